/*
 * CPU oracle for the elastic RTM hot path — TEST INFRASTRUCTURE ONLY.
 * See ertm_oracle.h for the grid convention and the reference lines each
 * piece restates.  Only tests/, the smoke check and bench.py's CPU-baseline
 * leg load this library; the CUDA product never does.
 */
#include "ertm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef REAL
#define REAL double
#endif
typedef REAL real;

/* The reference defines pai as 3.1415926 (3D_elastic_RTM/3D_zzzzz:1) and uses
 * it in the cosine sponge; the cubic sponge and the Ricker use PI from SU. */
#define REF_PAI 3.1415926
#define SU_PI 3.141592653589793

int orc_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int orc_real_size(void) { return (int)sizeof(real); }

/* ----------------------------------------------------------------------
 * Helpers
 * -------------------------------------------------------------------- */

/* Ricker wavelet, restating make_ricker_new (3D_elastic_RTM/zzzzz:139-160):
 * Bpar = sqrt(6)/(pi f), N = ceil(1.35 Bpar/dt), 2N+1 samples, peak at N,
 * w(t) = 0.5 (2 - u^2) exp(-u^2/4) with u = 2 sqrt(6) t / Bpar.
 * The reference computes in float; so does this function. */
int orc_ricker(double freq_hz, double dt_s, float *out, int maxn)
{
    float freq = (float)freq_hz, dt = (float)dt_s;
    if (freq == 0.0f) freq = 30.0f;
    if (dt == 0.0f) dt = 0.004f;
    float bpar = (float)(sqrt(6.0) / (SU_PI * freq));
    int n = (int)ceil(1.35 * bpar / dt);
    int np = 2 * n + 1;
    if (out == NULL) return np;
    if (np > maxn) return -np;
    out[n] = 1.0f;
    for (int i = 1; i <= n; i++) {
        float t = dt * (float)i;
        float u = (float)(2.0 * sqrt(6.0) * t / bpar);
        float v = (float)(0.5 * (2.0 - u * u) * exp(-u * u / 4.0));
        out[n + i] = v;
        out[n - i] = v;
    }
    return np;
}

/* Taylor coefficients of the staggered first derivative of half-width R:
 * sum_n c_n (2n-1)^(2m-1) = delta_{m,1}, m = 1..R (solved in double). */
void orc_coef_taylor(int R, double *coef)
{
    double A[8][9];
    for (int m = 0; m < R; m++) {
        for (int n = 0; n < R; n++) A[m][n] = pow(2.0 * n + 1.0, 2.0 * m + 1.0);
        A[m][R] = (m == 0) ? 1.0 : 0.0;
    }
    for (int c = 0; c < R; c++) {          /* Gauss-Jordan with partial pivoting */
        int p = c;
        for (int r = c + 1; r < R; r++) if (fabs(A[r][c]) > fabs(A[p][c])) p = r;
        for (int k = 0; k <= R; k++) { double t = A[c][k]; A[c][k] = A[p][k]; A[p][k] = t; }
        for (int r = 0; r < R; r++) {
            if (r == c) continue;
            double f = A[r][c] / A[c][c];
            for (int k = c; k <= R; k++) A[r][k] -= f * A[c][k];
        }
    }
    coef[0] = 0.0;
    for (int n = 0; n < R; n++) coef[n + 1] = A[n][R] / A[n][n];
    for (int n = R + 1; n < 8; n++) coef[n] = 0.0;
}

/* The reference's optimised 12th-order coefficients
 * (make_coe_optimized_new, 3D_elastic_RTM/zzzzz:202-210), as float values. */
void orc_coef_reference12(double *coef)
{
    static const float c[7] = {0.0f, 1.2213363647f, -0.096931457519f, 0.017447662353f,
                               -0.0029672895159f, 0.00035900539822f, -0.00002184781161f};
    for (int n = 0; n < 7; n++) coef[n] = (double)c[n];
    coef[7] = 0.0;
}

/* Sponge damping profile along one axis of n cells with widths w0 (low side)
 * and w1 (high side), values in 1/s.
 *  SPONGE_COS   : 3D cosine profile, coe_attenuation_3d_new2
 *                 (3D_elastic_RTM/3D_zzzzz:261-300): low side
 *                 coe*(1-cos(pai/2*(w0-i-1)/(w0-1))), high side coe*(1-cos(pai/2*i'/(w1-1))).
 *  SPONGE_CUBIC : 2D cubic profile, make_attenuation_new
 *                 (3D_elastic_RTM/zzzzz:238-280): coe*((w0-1-i)/(w0-1))^3, coe*(i'/(w1-1))^3.
 * The reference evaluates these in float; so does this function. The 3D
 * damping of a cell is the sum of its three axis profiles (3D_zzzzz:302-356).
 * Each value is rounded to float once, as `float * double` in the reference. */
void orc_sponge_profile(int kind, int n, int w0, int w1, double coe, double *out)
{
    float fc = (float)coe;
    for (int i = 0; i < n; i++) out[i] = 0.0;
    for (int i = 0; i < w0 && i < n; i++) {
        float v;
        if (kind == ORC_BOUNDARY_SPONGE_COS)
            v = (float)(fc * (1.0 - cos((REF_PAI / 2 * (w0 - i - 1) / (w0 - 1)))));
        else {
            float x = (float)((w0 - 1.0 - i) / (w0 - 1.0));
            v = (float)(fc * pow(x * 1.0, 3.0));
        }
        out[i] += v;
    }
    for (int q = 0; q < w1; q++) {
        int i = n - w1 + q;
        if (i < 0) continue;
        float v;
        if (kind == ORC_BOUNDARY_SPONGE_COS)
            v = (float)(fc * (1.0 - cos((REF_PAI / 2 * q / (w1 - 1)))));
        else {
            float x = (float)(q / (w1 - 1.0));
            v = (float)(fc * pow(x * 1.0, 3.0));
        }
        out[i] += v;
    }
}

/* C-PML coefficients (Komatitsch & Martin 2007, kappa = 1) along one axis.
 * stagger 0: integer points p = i; -1: p = i - 1/2 (x and y half points);
 * +1: p = i + 1/2 (z half points).  Distance into the layer is measured from
 * the last interior-side slab index (w0-1 on the low side, n-w1 on the high
 * side), so every point with nonzero damping lies inside the slab index ranges
 * [0,w0) and [n-w1,n).  d = d0 (dist/L)^2, d0 = -3 vmax ln(rc) / (2 L),
 * alpha = pi f0 (1 - dist/L), b = exp(-(d+alpha) dt), a = d (b-1)/(d+alpha). */
void orc_cpml_profile(int n, int w0, int w1, double h, double dt_s, double vmax,
                      double rc, double f0, int stagger, double *a, double *b)
{
    for (int i = 0; i < n; i++) {
        double p = i + 0.5 * stagger;
        double dist = 0.0, L = 1.0;
        if (w0 > 0 && p < w0 - 1) { dist = (w0 - 1) - p; L = w0; }
        else if (w1 > 0 && p > n - w1) { dist = p - (n - w1); L = w1; }
        if (dist <= 0.0) { a[i] = 0.0; b[i] = 1.0; continue; }
        double Lm = L * h, x = dist * h / Lm;
        double d0 = -3.0 * vmax * log(rc) / (2.0 * Lm);
        double d = d0 * x * x;
        double al = SU_PI * f0 * (1.0 - x);
        if (al < 0) al = 0;
        b[i] = exp(-(d + al) * dt_s);
        a[i] = d * (b[i] - 1.0) / (d + al);
    }
}

/* ----------------------------------------------------------------------
 * Propagation state
 * -------------------------------------------------------------------- */

enum { F_VX, F_VY, F_VZ, F_TXX, F_TYY, F_TZZ, F_TXY, F_TXZ, F_TYZ, F_TP, F_VXP, F_VYP, F_VZP, NF };
/* psi slots: stress derivatives then velocity derivatives */
enum {
    P_EXX, P_EYY, P_EZZ, P_DYVX, P_DXVY, P_DZVX, P_DXVZ, P_DZVY, P_DYVZ,
    P_DXTXX, P_DYTXY, P_DZTXZ, P_DXTXY, P_DYTYY, P_DZTYZ, P_DXTXZ, P_DYTYZ, P_DZTZZ, NP
};

typedef struct {
    orc_grid g;
    int two_d;
    int R, Ry;
    long px, py, pz, sy, sz, off0, total;
    real *f[NF];
    real *psi[NP];
    real *M, *MU, *LAM, *B;      /* padded like the fields */
    real *att;                   /* sponge damping per padded cell (sponge) */
    real *ax[2], *bx[2], *ay[2], *by[2], *az[2], *bz[2];   /* CPML: [0]=full [1]=half */
    real c[8];
    real dt, idx, idy, idz;
} orc_state;

#define AT(S, i, j, k) ((S)->off0 + (long)(k) * (S)->sz + (long)(j) * (S)->sy + (long)(i))

static real dplus(const real *f, long c, long s, const real *cf, int R)
{
    real acc = 0;
    for (int n = 1; n <= R; n++) acc += cf[n] * (f[c + n * s] - f[c - (n - 1) * s]);
    return acc;
}

static real dminus(const real *f, long c, long s, const real *cf, int R)
{
    real acc = 0;
    for (int n = 1; n <= R; n++) acc += cf[n] * (f[c + (n - 1) * s] - f[c - n * s]);
    return acc;
}

static void state_free(orc_state *S)
{
    if (!S) return;
    for (int i = 0; i < NF; i++) free(S->f[i]);
    for (int i = 0; i < NP; i++) free(S->psi[i]);
    free(S->M); free(S->MU); free(S->LAM); free(S->B); free(S->att);
    for (int h = 0; h < 2; h++) {
        free(S->ax[h]); free(S->bx[h]); free(S->ay[h]); free(S->by[h]);
        free(S->az[h]); free(S->bz[h]);
    }
    free(S);
}

static real *zalloc(long n) { return (real *)calloc((size_t)n, sizeof(real)); }

static orc_state *state_new(const orc_grid *g, const float *vp, const float *vs, const float *rho)
{
    if (g->nx <= 0 || g->ny <= 0 || g->nz <= 0 || (g->R != 4 && g->R != 6)) return NULL;
    orc_state *S = (orc_state *)calloc(1, sizeof(orc_state));
    if (!S) return NULL;
    S->g = *g;
    S->two_d = (g->ny == 1);
    S->R = g->R;
    S->Ry = S->two_d ? 0 : g->R;
    S->px = g->nx + 2L * S->R;
    S->py = g->ny + 2L * S->Ry;
    S->pz = g->nz + 2L * S->R;
    S->sy = S->px;
    S->sz = S->px * S->py;
    S->off0 = (long)S->R * S->sz + (long)S->Ry * S->sy + S->R;
    S->total = S->px * S->py * S->pz;
    for (int i = 0; i < NF; i++) if (!(S->f[i] = zalloc(S->total))) goto fail;
    if (!(S->M = zalloc(S->total)) || !(S->MU = zalloc(S->total)) ||
        !(S->LAM = zalloc(S->total)) || !(S->B = zalloc(S->total))) goto fail;
    for (int n = 0; n <= g->R; n++) S->c[n] = (real)g->coef[n];
    S->dt = (real)(g->dt_ms / 1000.0);
    S->idx = (real)(1.0 / g->dx);
    S->idy = (real)(1.0 / g->dy);
    S->idz = (real)(1.0 / g->dz);
    for (int k = 0; k < g->nz; k++)
        for (int j = 0; j < g->ny; j++)
            for (int i = 0; i < g->nx; i++) {
                long m = ((long)k * g->ny + j) * g->nx + i;
                long c = AT(S, i, j, k);
                real r = rho[m], p = vp[m], s = vs[m];
                S->M[c] = r * p * p;
                S->MU[c] = r * s * s;
                S->LAM[c] = S->M[c] - 2 * S->MU[c];
                S->B[c] = 1 / r;
            }
    double dts = g->dt_ms / 1000.0;
    if (g->boundary == ORC_BOUNDARY_CPML) {
        for (int i = 0; i < NP; i++) if (!(S->psi[i] = zalloc(S->total))) goto fail;
        int ns[3] = {g->nx, g->ny, g->nz};
        double hs[3] = {g->dx, g->dy, g->dz};
        real **A[3] = {S->ax, S->ay, S->az}, **Bb[3] = {S->bx, S->by, S->bz};
        double *ta = (double *)malloc(sizeof(double) * (ns[0] + ns[1] + ns[2]));
        double *tb = (double *)malloc(sizeof(double) * (ns[0] + ns[1] + ns[2]));
        if (!ta || !tb) { free(ta); free(tb); goto fail; }
        for (int ax = 0; ax < 3; ax++)
            for (int h = 0; h < 2; h++) {
                int stg = h == 0 ? 0 : (ax == 2 ? +1 : -1);
                int w0 = g->pml[2 * ax], w1 = g->pml[2 * ax + 1];
                if (ax == 1 && S->two_d) { w0 = w1 = 0; }
                orc_cpml_profile(ns[ax], w0, w1, hs[ax], dts, g->pml_vmax, g->pml_r, g->pml_f0,
                                 stg, ta, tb);
                A[ax][h] = zalloc(ns[ax]);
                Bb[ax][h] = zalloc(ns[ax]);
                if (!A[ax][h] || !Bb[ax][h]) { free(ta); free(tb); goto fail; }
                for (int i = 0; i < ns[ax]; i++) { A[ax][h][i] = (real)ta[i]; Bb[ax][h][i] = (real)tb[i]; }
            }
        free(ta); free(tb);
    } else {
        if (!(S->att = zalloc(S->total))) goto fail;
        double *px = (double *)malloc(sizeof(double) * g->nx);
        double *py = (double *)malloc(sizeof(double) * g->ny);
        double *pz = (double *)malloc(sizeof(double) * g->nz);
        if (!px || !py || !pz) { free(px); free(py); free(pz); goto fail; }
        orc_sponge_profile(g->boundary, g->nx, g->pml[0], g->pml[1], g->sponge_coef, px);
        if (S->two_d) { py[0] = 0.0; }
        else orc_sponge_profile(g->boundary, g->ny, g->pml[2], g->pml[3], g->sponge_coef, py);
        orc_sponge_profile(g->boundary, g->nz, g->pml[4], g->pml[5], g->sponge_coef, pz);
        for (int k = 0; k < g->nz; k++)
            for (int j = 0; j < g->ny; j++)
                for (int i = 0; i < g->nx; i++)
                    /* the reference accumulates z, then x, then y (3D_zzzzz:302-356) */
                    S->att[AT(S, i, j, k)] = (real)(((float)pz[k] + (float)px[i]) + (float)py[j]);
        free(px); free(py); free(pz);
    }
    return S;
fail:
    state_free(S);
    return NULL;
}

/* damping factors of the reference update f2 = g1*(g2*f1 + increment)
 * (2D_elastic_RTM/viscoelastic_equation.cu:151-180) */
static void damp(const orc_state *S, long c, real *g1, real *g2)
{
    if (S->att) {
        real a = S->att[c] * S->dt / 2;
        *g1 = 1 / (1 + a);
        *g2 = 1 - a;
    } else {
        *g1 = 1;
        *g2 = 1;
    }
}

static real cpml(const orc_state *S, int slot, long c, const real *a, const real *b, int idx, real d)
{
    if (!S->psi[0]) return d;
    real *p = S->psi[slot];
    p[c] = b[idx] * p[c] + a[idx] * d;
    return d + p[c];
}

static void stress_step(orc_state *S, int psplit)
{
    const orc_grid *g = &S->g;
    const int R = S->R;
    const real *vx = S->f[F_VX], *vy = S->f[F_VY], *vz = S->f[F_VZ];
    const long sy = S->sy, sz = S->sz;
    const real dt = S->dt;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < g->nz; k++)
        for (int j = 0; j < g->ny; j++)
            for (int i = 0; i < g->nx; i++) {
                long c = AT(S, i, j, k);
                real exx = dplus(vx, c, 1, S->c, R) * S->idx;
                real ezz = dminus(vz, c, sz, S->c, R) * S->idz;
                real dzvx = dplus(vx, c, sz, S->c, R) * S->idz;
                real dxvz = dminus(vz, c, 1, S->c, R) * S->idx;
                real eyy = 0, dyvx = 0, dxvy = 0, dzvy = 0, dyvz = 0;
                if (S->psi[0]) {
                    exx = cpml(S, P_EXX, c, S->ax[0], S->bx[0], i, exx);
                    ezz = cpml(S, P_EZZ, c, S->az[0], S->bz[0], k, ezz);
                    dzvx = cpml(S, P_DZVX, c, S->az[1], S->bz[1], k, dzvx);
                    dxvz = cpml(S, P_DXVZ, c, S->ax[1], S->bx[1], i, dxvz);
                }
                if (!S->two_d) {
                    eyy = dplus(vy, c, sy, S->c, R) * S->idy;
                    dyvx = dminus(vx, c, sy, S->c, R) * S->idy;
                    dxvy = dminus(vy, c, 1, S->c, R) * S->idx;
                    dzvy = dplus(vy, c, sz, S->c, R) * S->idz;
                    dyvz = dminus(vz, c, sy, S->c, R) * S->idy;
                    if (S->psi[0]) {
                        eyy = cpml(S, P_EYY, c, S->ay[0], S->by[0], j, eyy);
                        dyvx = cpml(S, P_DYVX, c, S->ay[1], S->by[1], j, dyvx);
                        dxvy = cpml(S, P_DXVY, c, S->ax[1], S->bx[1], i, dxvy);
                        dzvy = cpml(S, P_DZVY, c, S->az[1], S->bz[1], k, dzvy);
                        dyvz = cpml(S, P_DYVZ, c, S->ay[1], S->by[1], j, dyvz);
                    }
                }
                real g1, g2;
                damp(S, c, &g1, &g2);
                real M = S->M[c], L = S->LAM[c], U = S->MU[c];
                S->f[F_TXX][c] = g1 * (g2 * S->f[F_TXX][c] + dt * (M * exx + L * (eyy + ezz)));
                S->f[F_TZZ][c] = g1 * (g2 * S->f[F_TZZ][c] + dt * (M * ezz + L * (exx + eyy)));
                S->f[F_TXZ][c] = g1 * (g2 * S->f[F_TXZ][c] + dt * U * (dzvx + dxvz));
                if (!S->two_d) {
                    S->f[F_TYY][c] = g1 * (g2 * S->f[F_TYY][c] + dt * (M * eyy + L * (exx + ezz)));
                    S->f[F_TXY][c] = g1 * (g2 * S->f[F_TXY][c] + dt * U * (dyvx + dxvy));
                    S->f[F_TYZ][c] = g1 * (g2 * S->f[F_TYZ][c] + dt * U * (dzvy + dyvz));
                }
                if (psplit)
                    S->f[F_TP][c] = g1 * (g2 * S->f[F_TP][c] + dt * M * (exx + eyy + ezz));
            }
}

static void velocity_step(orc_state *S, int psplit)
{
    const orc_grid *g = &S->g;
    const int R = S->R;
    const real *txx = S->f[F_TXX], *tyy = S->f[F_TYY], *tzz = S->f[F_TZZ];
    const real *txy = S->f[F_TXY], *txz = S->f[F_TXZ], *tyz = S->f[F_TYZ], *tp = S->f[F_TP];
    const long sy = S->sy, sz = S->sz;
    const real dt = S->dt;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < g->nz; k++)
        for (int j = 0; j < g->ny; j++)
            for (int i = 0; i < g->nx; i++) {
                long c = AT(S, i, j, k);
                real dxtxx = dminus(txx, c, 1, S->c, R) * S->idx;
                real dztxz = dminus(txz, c, sz, S->c, R) * S->idz;
                real dxtxz = dplus(txz, c, 1, S->c, R) * S->idx;
                real dztzz = dplus(tzz, c, sz, S->c, R) * S->idz;
                real dytxy = 0, dxtxy = 0, dytyy = 0, dztyz = 0, dytyz = 0;
                if (S->psi[0]) {
                    dxtxx = cpml(S, P_DXTXX, c, S->ax[1], S->bx[1], i, dxtxx);
                    dztxz = cpml(S, P_DZTXZ, c, S->az[0], S->bz[0], k, dztxz);
                    dxtxz = cpml(S, P_DXTXZ, c, S->ax[0], S->bx[0], i, dxtxz);
                    dztzz = cpml(S, P_DZTZZ, c, S->az[1], S->bz[1], k, dztzz);
                }
                if (!S->two_d) {
                    dytxy = dplus(txy, c, sy, S->c, R) * S->idy;
                    dxtxy = dplus(txy, c, 1, S->c, R) * S->idx;
                    dytyy = dminus(tyy, c, sy, S->c, R) * S->idy;
                    dztyz = dminus(tyz, c, sz, S->c, R) * S->idz;
                    dytyz = dplus(tyz, c, sy, S->c, R) * S->idy;
                    if (S->psi[0]) {
                        dytxy = cpml(S, P_DYTXY, c, S->ay[0], S->by[0], j, dytxy);
                        dxtxy = cpml(S, P_DXTXY, c, S->ax[0], S->bx[0], i, dxtxy);
                        dytyy = cpml(S, P_DYTYY, c, S->ay[1], S->by[1], j, dytyy);
                        dztyz = cpml(S, P_DZTYZ, c, S->az[0], S->bz[0], k, dztyz);
                        dytyz = cpml(S, P_DYTYZ, c, S->ay[0], S->by[0], j, dytyz);
                    }
                }
                real g1, g2;
                damp(S, c, &g1, &g2);
                real b = S->B[c];
                S->f[F_VX][c] = g1 * (g2 * S->f[F_VX][c] + dt * b * (dxtxx + dytxy + dztxz));
                S->f[F_VZ][c] = g1 * (g2 * S->f[F_VZ][c] + dt * b * (dxtxz + dytyz + dztzz));
                if (!S->two_d)
                    S->f[F_VY][c] = g1 * (g2 * S->f[F_VY][c] + dt * b * (dxtxy + dytyy + dztyz));
                if (psplit) {
                    /* decoupled P velocity driven by the gradient of the P stress,
                     * the role of fwd_vxp_vzp_3D (3D_forward_or_back_together.cu:118) */
                    S->f[F_VXP][c] = g1 * (g2 * S->f[F_VXP][c] + dt * b * dminus(tp, c, 1, S->c, R) * S->idx);
                    S->f[F_VZP][c] = g1 * (g2 * S->f[F_VZP][c] + dt * b * dplus(tp, c, sz, S->c, R) * S->idz);
                    if (!S->two_d)
                        S->f[F_VYP][c] = g1 * (g2 * S->f[F_VYP][c] + dt * b * dminus(tp, c, sy, S->c, R) * S->idy);
                }
            }
}

static long rec_cell(const orc_state *S, const orc_shot *s, int r, int *ok)
{
    int irx = r % s->nrx, iry = r / s->nrx;
    int i = s->rx0 + irx * s->drx, j = s->ry0 + iry * s->dry;
    *ok = (i >= 0 && i < S->g.nx && j >= 0 && j < S->g.ny && s->rz >= 0 && s->rz < S->g.nz);
    return AT(S, i, j, s->rz);
}

static int image_pp_ps(real ex, real ey, real ez, real px, real py, real pz, real sx, real sy,
                       real sz, real *pp, real *ps);

/* One time step `it` of a pass, in the order of
 * 3D_elastic_RTM/3D_forward_or_back_together.cu:25-154 (model), :173-289 (source),
 * :310-452 (receiver). */
static void state_step(orc_state *S, const orc_shot *s, int mode, int it, int nsteps, float *data,
                       orc_excitation *ex, float *pp, float *ps, float *ptp)
{
    const int psplit = (mode != ORC_MODE_MODEL);
    const long nrec = (long)s->nrx * s->nry;
    const orc_grid *g = &S->g;
    if (mode == ORC_MODE_RECEIVER && data) {
        /* write_or_add_shot_3D_surface_three with add_receiver_bool (:328) */
        for (long r = 0; r < nrec; r++) {
            int ok;
            long c = rec_cell(S, s, (int)r, &ok);
            if (!ok) continue;
            for (int q = 0; q < 3; q++) {
                if (q == 1 && S->two_d) continue;
                real d = data[((long)q * nsteps + it) * nrec + r];
                real *f = S->f[F_VX + q];
                f[c] = (s->inject_mode == 2) ? d : f[c] + d;
            }
        }
    }
    if (mode != ORC_MODE_RECEIVER && it < s->nw) {
        /* add_source_3D into txx, tyy, tzz (:36-38) */
        long c = AT(S, s->sx, s->sy, s->sz);
        real w = s->wavelet[it];
        S->f[F_TXX][c] += w;
        S->f[F_TZZ][c] += w;
        if (!S->two_d) S->f[F_TYY][c] += w;
    }
    stress_step(S, psplit);
    velocity_step(S, psplit);
    if (mode == ORC_MODE_MODEL && data) {
        /* write_or_add_shot_3D_surface_three record flag 0 (:127) */
        for (long r = 0; r < nrec; r++) {
            int ok;
            long c = rec_cell(S, s, (int)r, &ok);
            for (int q = 0; q < 3; q++)
                data[((long)q * nsteps + it) * nrec + r] =
                    ok ? (float)S->f[F_VX + q][c] : 0.0f;
        }
    }
    if (mode == ORC_MODE_SOURCE && ex) {
        /* excitation amplitude / time of the P velocity, restating
         * caculate_ex_amp_time_new (2D_elastic_RTM/elastic_2D_kernel_3.cu:30-48) with the
         * vector and P-stress capture of cuda_cal_excitation_amp_time_new (:282):
         * strict '>' keeps the earliest maximum. */
#pragma omp parallel for schedule(static)
        for (int k = 0; k < g->nz; k++)
            for (int j = 0; j < g->ny; j++)
                for (int i = 0; i < g->nx; i++) {
                    long c = AT(S, i, j, k);
                    long m = ((long)k * g->ny + j) * g->nx + i;
                    real px = S->f[F_VXP][c], py = S->f[F_VYP][c], pz = S->f[F_VZP][c];
                    real a2 = px * px + py * py + pz * pz;
                    if (a2 > (real)ex->amp2[m]) {
                        ex->second2[m] = ex->amp2[m];
                        ex->amp2[m] = (float)a2;
                        ex->time[m] = it;
                        ex->evx[m] = (float)px;
                        ex->evy[m] = (float)py;
                        ex->evz[m] = (float)pz;
                        ex->etp[m] = (float)S->f[F_TP][c];
                    } else if (a2 > (real)ex->second2[m]) {
                        ex->second2[m] = (float)a2;
                    }
                }
    }
    if (mode == ORC_MODE_RECEIVER && ex) {
        /* imaging_inner_product_ex / imaging_correlation_ex, restating
         * 2D_elastic_RTM/elastic_2D_kernel_3.cu:542-576; a zero excitation vector
         * (0/0 in the reference) images as 0. */
#pragma omp parallel for schedule(static)
        for (int k = 0; k < g->nz; k++)
            for (int j = 0; j < g->ny; j++)
                for (int i = 0; i < g->nx; i++) {
                    long m = ((long)k * g->ny + j) * g->nx + i;
                    if (ex->time[m] != it) continue;
                    long c = AT(S, i, j, k);
                    real px = S->f[F_VXP][c], py = S->f[F_VYP][c], pz = S->f[F_VZP][c];
                    real vpp, vps;
                    if (image_pp_ps(ex->evx[m], ex->evy[m], ex->evz[m], px, py, pz,
                                    S->f[F_VX][c] - px, S->f[F_VY][c] - py, S->f[F_VZ][c] - pz,
                                    &vpp, &vps)) {
                        if (pp) pp[m] = (float)vpp;
                        if (ps) ps[m] = (float)vps;
                    }
                    real et = ex->etp[m];
                    if (ptp && et != 0) ptp[m] = (float)(S->f[F_TP][c] / et);
                }
    }
}

/* PP and PS of one cell (imaging_inner_product_ex_2D, elastic_2D_kernel_3.cu:559-580):
 * (e . r_P)/|e|^2 and (e . r_S)/|e|^2; returns 0 where |e|^2 == 0 */
static int image_pp_ps(real ex, real ey, real ez, real px, real py, real pz, real sx, real sy,
                       real sz, real *pp, real *ps)
{
    real den = ex * ex + ey * ey + ez * ez;
    if (!(den > 0)) return 0;
    *pp = (ex * px + ey * py + ez * pz) / den;
    *ps = (ex * sx + ey * sy + ez * sz) / den;
    return 1;
}

static void state_export(const orc_state *S, float *out)
{
    const orc_grid *g = &S->g;
    long n = (long)g->nx * g->ny * g->nz;
    for (int q = 0; q < NF; q++)
        for (int k = 0; k < g->nz; k++)
            for (int j = 0; j < g->ny; j++)
                for (int i = 0; i < g->nx; i++)
                    out[q * n + ((long)k * g->ny + j) * g->nx + i] = (float)S->f[q][AT(S, i, j, k)];
}

int orc_run_pass(const orc_grid *g, const float *vp, const float *vs, const float *rho,
                 const orc_shot *s, int mode, int nsteps, float *data,
                 orc_excitation *ex, float *img_pp, float *img_ps, float *img_tp,
                 float *final_fields)
{
    if (!g || !vp || !vs || !rho || !s || nsteps < 0) return -1;
    if (mode == ORC_MODE_RECEIVER && !ex) return -1;
    if (s->sx < 0 || s->sx >= g->nx || s->sy < 0 || s->sy >= g->ny || s->sz < 0 || s->sz >= g->nz)
        return -1;
    orc_state *S = state_new(g, vp, vs, rho);
    if (!S) return -2;
    long n = (long)g->nx * g->ny * g->nz;
    if (mode == ORC_MODE_SOURCE && ex) {
        memset(ex->amp2, 0, sizeof(float) * n);
        memset(ex->second2, 0, sizeof(float) * n);
        memset(ex->time, 0, sizeof(int) * n);
        memset(ex->evx, 0, sizeof(float) * n);
        memset(ex->evy, 0, sizeof(float) * n);
        memset(ex->evz, 0, sizeof(float) * n);
        memset(ex->etp, 0, sizeof(float) * n);
    }
    if (mode == ORC_MODE_RECEIVER) {
        if (img_pp) memset(img_pp, 0, sizeof(float) * n);
        if (img_ps) memset(img_ps, 0, sizeof(float) * n);
        if (img_tp) memset(img_tp, 0, sizeof(float) * n);
        for (int it = nsteps - 1; it >= 0; it--)
            state_step(S, s, mode, it, nsteps, data, ex, img_pp, img_ps, img_tp);
    } else {
        for (int it = 0; it < nsteps; it++)
            state_step(S, s, mode, it, nsteps, data, ex, img_pp, img_ps, img_tp);
    }
    if (final_fields) state_export(S, final_fields);
    state_free(S);
    return 0;
}

/* ----------------------------------------------------------------------
 * Stepping API for the CPU baseline: lets a caller time steps without the
 * allocation cost of a full pass.
 * -------------------------------------------------------------------- */
void *orc_state_create(const orc_grid *g, const float *vp, const float *vs, const float *rho)
{
    return state_new(g, vp, vs, rho);
}

void orc_state_step(void *st, const orc_shot *s, int mode, int it, int nsteps, float *data,
                    orc_excitation *ex, float *pp, float *ps, float *ptp)
{
    state_step((orc_state *)st, s, mode, it, nsteps, data, ex, pp, ps, ptp);
}

void orc_state_destroy(void *st) { state_free((orc_state *)st); }

/* ----------------------------------------------------------------------
 * Divergence / curl decomposition (decom_new, elastic_2D_kernel_2.cu:671-791)
 * -------------------------------------------------------------------- */
int orc_divcurl(const orc_grid *g, const float *vp, const float *vs,
                const float *vx, const float *vy, const float *vz,
                float *p, float *sx, float *sy, float *sz)
{
    if (!g || !vp || !vs || !vx || !vz || !p || !sy) return -1;
    int two_d = (g->ny == 1);
    if (!two_d && (!vy || !sx || !sz)) return -1;
    const int R = g->R;
    const int Ry = two_d ? 0 : R;
    long px = g->nx + 2L * R, py = g->ny + 2L * Ry, pz = g->nz + 2L * R;
    long ssy = px, ssz = px * py, off0 = (long)R * ssz + (long)Ry * ssy + R, tot = px * py * pz;
    real *X = zalloc(tot), *Y = zalloc(tot), *Z = zalloc(tot), *VS = zalloc(tot);
    if (!X || !Y || !Z || !VS) { free(X); free(Y); free(Z); free(VS); return -2; }
    real cf[8];
    for (int n = 0; n <= R; n++) cf[n] = (real)g->coef[n];
    for (int k = 0; k < g->nz; k++)
        for (int j = 0; j < g->ny; j++)
            for (int i = 0; i < g->nx; i++) {
                long m = ((long)k * g->ny + j) * g->nx + i;
                long c = off0 + k * ssz + j * ssy + i;
                X[c] = vx[m];
                Z[c] = vz[m];
                if (!two_d) Y[c] = vy[m];
                VS[c] = vs[m];
            }
    real ix = (real)(1.0 / g->dx), iy = (real)(1.0 / g->dy), iz = (real)(1.0 / g->dz);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < g->nz; k++)
        for (int j = 0; j < g->ny; j++)
            for (int i = 0; i < g->nx; i++) {
                long m = ((long)k * g->ny + j) * g->nx + i;
                long c = off0 + k * ssz + j * ssy + i;
                real div = dplus(X, c, 1, cf, R) * ix + dminus(Z, c, ssz, cf, R) * iz;
                if (!two_d) div += dplus(Y, c, ssy, cf, R) * iy;
                p[m] = (float)((real)vp[m] * div);
                /* shear velocity averaged over the four cells of the rotation plane
                 * (decom_new averages (i,k),(i,k+1),(i+1,k),(i+1,k+1)); cells past the
                 * grid edge contribute zero, as the reference's padded arrays do */
                real vxz = (VS[c] + VS[c + ssz] + VS[c + 1] + VS[c + 1 + ssz]) / 4;
                sy[m] = (float)(vxz * (dplus(X, c, ssz, cf, R) * iz - dminus(Z, c, 1, cf, R) * ix));
                if (!two_d) {
                    real vyz = (VS[c] + VS[c + ssz] + VS[c + ssy] + VS[c + ssy + ssz]) / 4;
                    real vxy = (VS[c] + VS[c + 1] + VS[c + ssy] + VS[c + 1 + ssy]) / 4;
                    sx[m] = (float)(vyz * (dminus(Z, c, ssy, cf, R) * iy - dplus(Y, c, ssz, cf, R) * iz));
                    sz[m] = (float)(vxy * (dminus(Y, c, 1, cf, R) * ix - dminus(X, c, ssy, cf, R) * iy));
                }
            }
    free(X); free(Y); free(Z); free(VS);
    return 0;
}

/* ----------------------------------------------------------------------
 * Born modelling and its exact adjoint (2D, sponge boundaries)
 * -------------------------------------------------------------------- */
typedef struct {
    int nx, nz, R;
    long px, pz, n;            /* padded extents (R halo on every side) */
    real c[8], dt, ix, iz;
    real *M, *U, *L, *B, *g1, *g2;
} born2d;

#define B2(S, i, k) (((long)(k) + (S)->R) * (S)->px + (i) + (S)->R)

static int born_setup(born2d *S, const orc_grid *g, const float *vp, const float *vs,
                      const float *rho)
{
    if (g->ny != 1 || g->boundary == ORC_BOUNDARY_CPML) return -1;
    memset(S, 0, sizeof *S);
    S->nx = g->nx; S->nz = g->nz; S->R = g->R;
    S->px = g->nx + 2L * g->R; S->pz = g->nz + 2L * g->R; S->n = S->px * S->pz;
    for (int q = 0; q <= g->R; q++) S->c[q] = (real)g->coef[q];
    S->dt = (real)(g->dt_ms / 1000.0);
    S->ix = (real)(1.0 / g->dx); S->iz = (real)(1.0 / g->dz);
    real **arr[6] = {&S->M, &S->U, &S->L, &S->B, &S->g1, &S->g2};
    for (int q = 0; q < 6; q++) if (!(*arr[q] = zalloc(S->n))) return -2;
    double *px = (double *)malloc(sizeof(double) * g->nx), *pz = (double *)malloc(sizeof(double) * g->nz);
    if (!px || !pz) { free(px); free(pz); return -2; }
    orc_sponge_profile(g->boundary, g->nx, g->pml[0], g->pml[1], g->sponge_coef, px);
    orc_sponge_profile(g->boundary, g->nz, g->pml[4], g->pml[5], g->sponge_coef, pz);
    for (int k = 0; k < g->nz; k++)
        for (int i = 0; i < g->nx; i++) {
            long c = B2(S, i, k), m = (long)k * g->nx + i;
            real r = rho[m], p = vp[m], s = vs[m];
            S->M[c] = r * p * p; S->U[c] = r * s * s; S->L[c] = S->M[c] - 2 * S->U[c]; S->B[c] = 1 / r;
            real a = (real)((float)pz[k] + (float)px[i]) * S->dt / 2;
            S->g1[c] = 1 / (1 + a); S->g2[c] = 1 - a;
        }
    free(px); free(pz);
    return 0;
}

static void born_free(born2d *S)
{
    free(S->M); free(S->U); free(S->L); free(S->B); free(S->g1); free(S->g2);
}

static real b_dpx(const born2d *S, const real *f, long c) { return dplus(f, c, 1, S->c, S->R) * S->ix; }
static real b_dmx(const born2d *S, const real *f, long c) { return dminus(f, c, 1, S->c, S->R) * S->ix; }
static real b_dpz(const born2d *S, const real *f, long c) { return dplus(f, c, S->px, S->c, S->R) * S->iz; }
static real b_dmz(const born2d *S, const real *f, long c) { return dminus(f, c, S->px, S->c, S->R) * S->iz; }

static void born_sources(real dm, real du, real rr, real e0xx, real e0zz, real e0xz, real a0x,
                         real a0z, real dt, real *sxx, real *szz, real *sxz, real *svx, real *svz);

/* one step of background (+ scattered when dM != NULL); stores v0 (start of
 * step) and a0 into keep[4] when keep != NULL */
static void born_step(const born2d *S, const orc_shot *s, int it, real *v0x, real *v0z, real *s0xx,
                      real *s0zz, real *s0xz, real *vx, real *vz, real *sxx, real *szz, real *sxz,
                      const real *dM, const real *dU, const real *rr, real **keep)
{
    const real dt = S->dt;
    if (it < s->nw) {
        long c = B2(S, s->sx, s->sz);
        s0xx[c] += s->wavelet[it];
        s0zz[c] += s->wavelet[it];
    }
    if (keep) {
        memcpy(keep[0], v0x, sizeof(real) * S->n);
        memcpy(keep[1], v0z, sizeof(real) * S->n);
    }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < S->nz; k++)
        for (int i = 0; i < S->nx; i++) {
            long c = B2(S, i, k);
            real e0xx = b_dpx(S, v0x, c), e0zz = b_dmz(S, v0z, c);
            real e0xz = b_dpz(S, v0x, c) + b_dmx(S, v0z, c);
            real g1 = S->g1[c], g2 = S->g2[c], M = S->M[c], L = S->L[c], U = S->U[c];
            s0xx[c] = g1 * (g2 * s0xx[c] + dt * (M * e0xx + L * e0zz));
            s0zz[c] = g1 * (g2 * s0zz[c] + dt * (M * e0zz + L * e0xx));
            s0xz[c] = g1 * (g2 * s0xz[c] + dt * U * e0xz);
            if (dM) {
                real exx = b_dpx(S, vx, c), ezz = b_dmz(S, vz, c);
                real exz = b_dpz(S, vx, c) + b_dmx(S, vz, c);
                real qxx, qzz, qxz, unused0, unused1;
                born_sources(dM[c], dU[c], 0, e0xx, e0zz, e0xz, 0, 0, dt, &qxx, &qzz, &qxz, &unused0,
                             &unused1);
                sxx[c] = g1 * (g2 * sxx[c] + dt * (M * exx + L * ezz) + qxx);
                szz[c] = g1 * (g2 * szz[c] + dt * (M * ezz + L * exx) + qzz);
                sxz[c] = g1 * (g2 * sxz[c] + dt * U * exz + qxz);
            }
        }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < S->nz; k++)
        for (int i = 0; i < S->nx; i++) {
            long c = B2(S, i, k);
            real g1 = S->g1[c], g2 = S->g2[c], b = S->B[c];
            real a0x = b * (b_dmx(S, s0xx, c) + b_dmz(S, s0xz, c));
            real a0z = b * (b_dpx(S, s0xz, c) + b_dpz(S, s0zz, c));
            if (keep) { keep[2][c] = a0x; keep[3][c] = a0z; }
            v0x[c] = g1 * (g2 * v0x[c] + dt * a0x);
            v0z[c] = g1 * (g2 * v0z[c] + dt * a0z);
            if (dM) {
                real ax = b * (b_dmx(S, sxx, c) + b_dmz(S, sxz, c));
                real az = b * (b_dpx(S, sxz, c) + b_dpz(S, szz, c));
                real q0, q1, q2, svx, svz;
                born_sources(0, 0, rr[c], 0, 0, 0, a0x, a0z, dt, &q0, &q1, &q2, &svx, &svz);
                vx[c] = g1 * (g2 * vx[c] + dt * ax + svx);
                vz[c] = g1 * (g2 * vz[c] + dt * az + svz);
            }
        }
}

/* Born secondary sources of one cell (the reference's dem_p terms,
 * cuda_cal_dem_parameter_viscoelastic_media_new, viscoelastic_equation.cu:2398-2505,
 * inversion_para 2, no attenuation): stress sources dt (dM exx + dL ezz,
 * dM ezz + dL exx, dU exz) and velocity sources -dt r_rho (ax, az) */
static void born_sources(real dm, real du, real rr, real e0xx, real e0zz, real e0xz, real a0x,
                         real a0z, real dt, real *sxx, real *szz, real *sxz, real *svx, real *svz)
{
    real dl = dm - 2 * du;
    *sxx = dt * (dm * e0xx + dl * e0zz);
    *szz = dt * (dm * e0zz + dl * e0xx);
    *sxz = dt * du * e0xz;
    *svx = -dt * rr * a0x;
    *svz = -dt * rr * a0z;
}

static int born_rec(const born2d *S, const orc_shot *s, int r, long *c)
{
    int irx = r % s->nrx, i = s->rx0 + irx * s->drx;
    if (i < 0 || i >= S->nx || s->rz < 0 || s->rz >= S->nz) return 0;
    *c = B2(S, i, s->rz);
    return 1;
}

int orc_born_forward(const orc_grid *g, const float *vp, const float *vs, const float *rho,
                     const orc_shot *s, int nt, const float *r_vp, const float *r_vs,
                     const float *r_rho, float *data)
{
    born2d S;
    if (!s || !data || nt < 1 || s->nry != 1) return -1;
    int rc = born_setup(&S, g, vp, vs, rho);
    if (rc) { born_free(&S); return rc; }
    real *f[13];
    for (int q = 0; q < 13; q++) if (!(f[q] = zalloc(S.n))) { rc = -2; }
    if (!rc) {
        real *dM = f[10], *dU = f[11], *rr = f[12];
        for (int k = 0; k < S.nz; k++)
            for (int i = 0; i < S.nx; i++) {
                long c = B2(&S, i, k), m = (long)k * S.nx + i;
                dM[c] = S.M[c] * ((real)r_rho[m] + 2 * (real)r_vp[m]);
                dU[c] = S.U[c] * ((real)r_rho[m] + 2 * (real)r_vs[m]);
                rr[c] = r_rho[m];
            }
        const long nrec = s->nrx;
        memset(data, 0, sizeof(float) * 3 * (size_t)nt * nrec);
        for (int it = 0; it < nt; it++) {
            born_step(&S, s, it, f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9], dM, dU,
                      rr, NULL);
            for (long r = 0; r < nrec; r++) {
                long c;
                if (!born_rec(&S, s, (int)r, &c)) continue;
                data[((long)0 * nt + it) * nrec + r] = (float)f[5][c];
                data[((long)2 * nt + it) * nrec + r] = (float)f[6][c];
            }
        }
    }
    for (int q = 0; q < 13; q++) free(f[q]);
    born_free(&S);
    return rc;
}

int orc_born_adjoint(const orc_grid *g, const float *vp, const float *vs, const float *rho,
                     const orc_shot *s, int nt, const float *residual, float *g_vp, float *g_vs,
                     float *g_rho)
{
    born2d S;
    if (!s || !residual || nt < 1 || s->nry != 1) return -1;
    int rc = born_setup(&S, g, vp, vs, rho);
    if (rc) { born_free(&S); return rc; }
    const long n = S.n;
    /* background history: v0 at the start of every step and a0 of every step */
    real *hist = (real *)malloc(sizeof(real) * (size_t)4 * n * nt);
    real *w[16];
    for (int q = 0; q < 16; q++) w[q] = zalloc(n);
    for (int q = 0; q < 16; q++) if (!w[q]) rc = -2;
    if (!hist) rc = -2;
    if (!rc) {
        real *v0x = w[0], *v0z = w[1], *s0xx = w[2], *s0zz = w[3], *s0xz = w[4];
        for (int it = 0; it < nt; it++) {
            real *keep[4] = {hist + (4L * it + 0) * n, hist + (4L * it + 1) * n,
                             hist + (4L * it + 2) * n, hist + (4L * it + 3) * n};
            born_step(&S, s, it, v0x, v0z, s0xx, s0zz, s0xz, NULL, NULL, NULL, NULL, NULL, NULL,
                      NULL, NULL, keep);
        }
        real *ax = w[5], *az = w[6], *hxx = w[7], *hzz = w[8], *hxz = w[9];
        real *gM = w[10], *gL = w[11], *gU = w[12], *gR = w[13], *tx = w[14], *tz = w[15];
        for (long q = 0; q < n; q++) ax[q] = az[q] = hxx[q] = hzz[q] = hxz[q] = 0;
        const long nrec = s->nrx;
        const real dt = S.dt;
        real *Qxx = (real *)calloc(n, sizeof(real)), *Qzz = (real *)calloc(n, sizeof(real));
        real *Qxz = (real *)calloc(n, sizeof(real));
        for (int it = nt - 1; it >= 0; it--) {
            const real *hv0x = hist + (4L * it + 0) * n, *hv0z = hist + (4L * it + 1) * n;
            const real *ha0x = hist + (4L * it + 2) * n, *ha0z = hist + (4L * it + 3) * n;
            for (long r = 0; r < nrec; r++) {          /* record^T */
                long c;
                if (!born_rec(&S, s, (int)r, &c)) continue;
                ax[c] += residual[((long)0 * nt + it) * nrec + r];
                az[c] += residual[((long)2 * nt + it) * nrec + r];
            }
            /* velocity update^T */
            for (long q = 0; q < n; q++) {
                tx[q] = S.B[q] * S.g1[q] * ax[q];
                tz[q] = S.B[q] * S.g1[q] * az[q];
            }
#pragma omp parallel for schedule(static)
            for (int k = 0; k < S.nz; k++)
                for (int i = 0; i < S.nx; i++) {
                    long c = B2(&S, i, k);
                    real g1 = S.g1[c];
                    gR[c] += -dt * (g1 * ax[c] * ha0x[c] + g1 * az[c] * ha0z[c]);
                    hxx[c] += -dt * b_dpx(&S, tx, c);
                    hxz[c] += -dt * (b_dpz(&S, tx, c) + b_dmx(&S, tz, c));
                    hzz[c] += -dt * b_dmz(&S, tz, c);
                }
            /* stress update^T */
            for (long q = 0; q < n; q++) {
                real g1 = S.g1[q];
                Qxx[q] = g1 * hxx[q]; Qzz[q] = g1 * hzz[q]; Qxz[q] = g1 * hxz[q];
                tx[q] = S.M[q] * Qxx[q] + S.L[q] * Qzz[q];     /* reused as M Qxx + L Qzz */
                tz[q] = S.L[q] * Qxx[q] + S.M[q] * Qzz[q];     /* L Qxx + M Qzz */
            }
            real *uq = hxx;                                    /* U Qxz, written after use */
#pragma omp parallel for schedule(static)
            for (int k = 0; k < S.nz; k++)
                for (int i = 0; i < S.nx; i++) {
                    long c = B2(&S, i, k);
                    real e0xx = b_dpx(&S, hv0x, c), e0zz = b_dmz(&S, hv0z, c);
                    real e0xz = b_dpz(&S, hv0x, c) + b_dmx(&S, hv0z, c);
                    gM[c] += dt * (Qxx[c] * e0xx + Qzz[c] * e0zz);
                    gL[c] += dt * (Qxx[c] * e0zz + Qzz[c] * e0xx);
                    gU[c] += dt * Qxz[c] * e0xz;
                }
            for (long q = 0; q < n; q++) uq[q] = S.U[q] * Qxz[q];
#pragma omp parallel for schedule(static)
            for (int k = 0; k < S.nz; k++)
                for (int i = 0; i < S.nx; i++) {
                    long c = B2(&S, i, k);
                    real g12 = S.g2[c] * S.g1[c];
                    ax[c] = g12 * ax[c] - dt * (b_dmx(&S, tx, c) + b_dmz(&S, uq, c));
                    az[c] = g12 * az[c] - dt * (b_dpz(&S, tz, c) + b_dpx(&S, uq, c));
                }
            for (long q = 0; q < n; q++) {
                real g2 = S.g2[q];
                hxx[q] = g2 * Qxx[q]; hzz[q] = g2 * Qzz[q]; hxz[q] = g2 * Qxz[q];
            }
        }
        for (int k = 0; k < S.nz; k++)
            for (int i = 0; i < S.nx; i++) {
                long c = B2(&S, i, k), m = (long)k * S.nx + i;
                real gm = gM[c] + gL[c], gu = gU[c] - 2 * gL[c];
                g_vp[m] = (float)(2 * S.M[c] * gm);
                g_vs[m] = (float)(2 * S.U[c] * gu);
                g_rho[m] = (float)(S.M[c] * gm + S.U[c] * gu + gR[c]);
            }
        free(Qxx); free(Qzz); free(Qxz);
    }
    for (int q = 0; q < 16; q++) free(w[q]);
    free(hist);
    born_free(&S);
    return rc;
}

/* ----------------------------------------------------------------------
 * Entry points used only to compare single pieces of the scheme with the
 * reference's own 2D kernels (tests/golden/ref_kernels_2d.npz)
 * -------------------------------------------------------------------- */

/* One stress half-step of the 2D scheme from given fields (nz*nx arrays):
 * the code of stress_step, without the P stress. */
int orc_stress_step_given(const orc_grid *g, const float *vp, const float *vs, const float *rho,
                          const float *vx, const float *vz, const float *txx, const float *tzz,
                          const float *txz, float *otxx, float *otzz, float *otxz)
{
    if (!g || g->ny != 1) return -1;
    orc_state *S = state_new(g, vp, vs, rho);
    if (!S) return -2;
    const float *in[5] = {vx, vz, txx, tzz, txz};
    const int fid[5] = {F_VX, F_VZ, F_TXX, F_TZZ, F_TXZ};
    for (int q = 0; q < 5; q++)
        for (int k = 0; k < g->nz; k++)
            for (int i = 0; i < g->nx; i++)
                S->f[fid[q]][AT(S, i, 0, k)] = in[q][(long)k * g->nx + i];
    stress_step(S, 0);
    float *out[3] = {otxx, otzz, otxz};
    const int oid[3] = {F_TXX, F_TZZ, F_TXZ};
    for (int q = 0; q < 3; q++)
        for (int k = 0; k < g->nz; k++)
            for (int i = 0; i < g->nx; i++)
                out[q][(long)k * g->nx + i] = (float)S->f[oid[q]][AT(S, i, 0, k)];
    state_free(S);
    return 0;
}

/* Born secondary sources for n cells (see born_sources): inputs per cell */
int orc_born_sources_given(long n, double dt_ms, const float *vp, const float *vs, const float *rho,
                           const float *rvp, const float *rvs, const float *rrho, const float *exx,
                           const float *ezz, const float *exz, const float *ax, const float *az,
                           float *osxx, float *oszz, float *osxz, float *osvx, float *osvz)
{
    real dt = (real)(dt_ms / 1000.0);
    for (long c = 0; c < n; c++) {
        real r = rho[c], p = vp[c], q = vs[c];
        real M = r * p * p, U = r * q * q;
        real dm = M * ((real)rrho[c] + 2 * (real)rvp[c]), du = U * ((real)rrho[c] + 2 * (real)rvs[c]);
        real a, b, d, e, f;
        born_sources(dm, du, rrho[c], exx[c], ezz[c], exz[c], ax[c], az[c], dt, &a, &b, &d, &e, &f);
        osxx[c] = (float)a; oszz[c] = (float)b; osxz[c] = (float)d; osvx[c] = (float)e; osvz[c] = (float)f;
    }
    return 0;
}

/* PP / PS of n cells with the oracle's imaging rule (2D: y components zero) */
int orc_image_given(long n, const float *ex, const float *ez, const float *rpx, const float *rpz,
                    const float *rsx, const float *rsz, float *pp, float *ps)
{
    for (long c = 0; c < n; c++) {
        real a = 0, b = 0;
        if (!image_pp_ps(ex[c], 0, ez[c], rpx[c], 0, rpz[c], rsx[c], 0, rsz[c], &a, &b)) a = b = 0;
        pp[c] = (float)a;
        ps[c] = (float)b;
    }
    return 0;
}
