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

/* Angle of the window sums, rounded as the reference does: float(atan(sxz / szz))
 * * 180 / pai1 in float arithmetic, pai1 = 3.1415926f (elastic_2D_kernel_3.cu:4, :204). */
static float angle_of_sums(double sxz, double szz)
{
    float a = (float)atan(sxz / szz);
    a = a * 180.0f;
    return a / 3.1415926f;
}

/* P-wave propagation angle at cell (i, k) of a 2D state (and, when asked, the
 * window's P energy), restating caculate_ex_angle_pp_only_RTM (source wavefield,
 * 5 x 5 window, hw = 2) and caculate_ex_angle_rp_only_RTM (receiver wavefield,
 * 9 x 9 window, hw = 4) (2D_elastic_RTM/elastic_2D_kernel_3.cu:132-284) on the
 * Poynting vector of sum_poynting (elastic_2D_kernel_2.cu:28-30), p = -tp (vxp, vzp):
 * over the (2 hw + 1)^2 cells around (i, k) (cells outside the grid count as zero),
 * sxz = sum px pz and szz = sum pz^2, angle = atan(sxz / szz) in degrees from the
 * z axis.  Returns 0 and leaves *out alone where szz == 0, as the reference does. */
static int window_angle(const orc_state *S, int i, int k, int hw, float *out, float *energy)
{
    const orc_grid *g = &S->g;
    double sxz = 0.0, szz = 0.0, sxx = 0.0;
    for (int dk = -hw; dk <= hw; dk++)
        for (int di = -hw; di <= hw; di++) {
            int ii = i + di, kk = k + dk;
            if (ii < 0 || ii >= g->nx || kk < 0 || kk >= g->nz) continue;
            long c = AT(S, ii, 0, kk);
            double tp = S->f[F_TP][c];
            double px = -tp * S->f[F_VXP][c], pz = -tp * S->f[F_VZP][c];
            sxz += px * pz;
            szz += pz * pz;
            sxx += px * px;
        }
    if (energy) *energy = (float)(sxx + szz);
    if (szz == 0.0) return 0;
    *out = angle_of_sums(sxz, szz);
    return 1;
}

static void capture_angles(const orc_state *S, const orc_excitation *ex, int it, int hw,
                           float *angle, float *energy)
{
    const orc_grid *g = &S->g;
    if (!S->two_d || !angle) return;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < g->nz; k++)
        for (int i = 0; i < g->nx; i++) {
            long m = (long)k * g->nx + i;
            if (ex->time[m] == it) window_angle(S, i, k, hw, &angle[m], energy ? &energy[m] : NULL);
        }
}

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
        capture_angles(S, ex, it, 2, ex->src_angle, ex->src_energy);
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
        capture_angles(S, ex, it, 4, ex->rcv_angle, ex->rcv_energy);
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
    if (mode == ORC_MODE_SOURCE && ex && ex->src_angle) memset(ex->src_angle, 0, sizeof(float) * n);
    if (mode == ORC_MODE_SOURCE && ex && ex->src_energy) memset(ex->src_energy, 0, sizeof(float) * n);
    if (mode == ORC_MODE_RECEIVER && ex->rcv_angle) memset(ex->rcv_angle, 0, sizeof(float) * n);
    if (mode == ORC_MODE_RECEIVER && ex->rcv_energy) memset(ex->rcv_energy, 0, sizeof(float) * n);
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

/* All 13 fields of a stepping state, [13][nz][ny][nx] (field order of the enum). */
void orc_state_fields(const void *st, float *out) { state_export((const orc_state *)st, out); }

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
    real *M, *U, *B, *g1, *g2; /* relaxed moduli pi = rho vp^2, mu = rho vs^2; buoyancy; damping */
    int nm;                    /* relaxation mechanisms (0: elastic) */
    real ra[3], rb[3];         /* memory-variable update r' = ra r + rb f */
    real tp, ts;               /* GSLS strengths of the P and S moduli */
    real kp, ks;               /* 1 + nm tp, 1 + nm ts: unrelaxed / relaxed */
} born2d;

#define B2(S, i, k) (((long)(k) + (S)->R) * (S)->px + (i) + (S)->R)

/* GSLS fit (tau method, first order in tau): relaxation frequencies
 * f_l = f0 10^(2 (l + 1/2) / nmech - 1) (log-spaced over about two decades
 * around f0), tau_sigma = 1 / (2 pi f_l); Q^-1(w) ~ tau S(w) with
 * S(w) = sum_l w tau_sigma / (1 + w^2 tau_sigma^2), fitted in least squares to a
 * constant 1/q at 32 log-spaced frequencies in [f0/4, 4 f0]:
 * tau = (1/q) sum S / sum S^2. */
void orc_visco_fit(int nmech, double qp, double qs, double f0, double *tau_sigma, double *tau_p,
                   double *tau_s)
{
    const double pi = 3.14159265358979323846;
    if (nmech < 1 || nmech > 3 || !(f0 > 0)) { *tau_p = *tau_s = 0; return; }
    for (int l = 0; l < nmech; l++) {
        double fl = f0 * pow(10.0, 2.0 * (l + 0.5) / nmech - 1.0);
        tau_sigma[l] = 1.0 / (2.0 * pi * fl);
    }
    double s1 = 0, s2 = 0;
    for (int j = 0; j < 32; j++) {
        double f = f0 / 4.0 * pow(16.0, j / 31.0), w = 2.0 * pi * f, S = 0;
        for (int l = 0; l < nmech; l++) S += w * tau_sigma[l] / (1.0 + w * w * tau_sigma[l] * tau_sigma[l]);
        s1 += S;
        s2 += S * S;
    }
    *tau_p = qp > 0 ? (1.0 / qp) * s1 / s2 : 0.0;
    *tau_s = qs > 0 ? (1.0 / qs) * s1 / s2 : 0.0;
}

static int born_setup(born2d *S, const orc_grid *g, const float *vp, const float *vs,
                      const float *rho)
{
    if (g->ny != 1 || g->boundary == ORC_BOUNDARY_CPML) return -1;
    if (g->visco_nmech < 0 || g->visco_nmech > 3) return -1;
    memset(S, 0, sizeof *S);
    S->nx = g->nx; S->nz = g->nz; S->R = g->R;
    S->px = g->nx + 2L * g->R; S->pz = g->nz + 2L * g->R; S->n = S->px * S->pz;
    for (int q = 0; q <= g->R; q++) S->c[q] = (real)g->coef[q];
    S->dt = (real)(g->dt_ms / 1000.0);
    S->ix = (real)(1.0 / g->dx); S->iz = (real)(1.0 / g->dz);
    S->nm = g->visco_nmech;
    S->kp = S->ks = 1;
    if (S->nm > 0) {
        double ts[3], tp, tsh;
        orc_visco_fit(S->nm, g->visco_qp, g->visco_qs, g->visco_f0, ts, &tp, &tsh);
        S->tp = (real)tp; S->ts = (real)tsh;
        S->kp = 1 + S->nm * S->tp; S->ks = 1 + S->nm * S->ts;
        for (int l = 0; l < S->nm; l++) {
            double h = g->dt_ms / 1000.0 / (2.0 * ts[l]);
            S->ra[l] = (real)((1.0 - h) / (1.0 + h));
            S->rb[l] = (real)(-2.0 * h / (1.0 + h));
        }
    }
    real **arr[5] = {&S->M, &S->U, &S->B, &S->g1, &S->g2};
    for (int q = 0; q < 5; q++) if (!(*arr[q] = zalloc(S->n))) return -2;
    double *px = (double *)malloc(sizeof(double) * g->nx), *pz = (double *)malloc(sizeof(double) * g->nz);
    if (!px || !pz) { free(px); free(pz); return -2; }
    orc_sponge_profile(g->boundary, g->nx, g->pml[0], g->pml[1], g->sponge_coef, px);
    orc_sponge_profile(g->boundary, g->nz, g->pml[4], g->pml[5], g->sponge_coef, pz);
    for (int k = 0; k < g->nz; k++)
        for (int i = 0; i < g->nx; i++) {
            long c = B2(S, i, k), m = (long)k * g->nx + i;
            real r = rho[m], p = vp[m], s = vs[m];
            S->M[c] = r * p * p; S->U[c] = r * s * s; S->B[c] = 1 / r;
            real a = (real)((float)pz[k] + (float)px[i]) * S->dt / 2;
            S->g1[c] = 1 / (1 + a); S->g2[c] = 1 - a;
        }
    free(px); free(pz);
    return 0;
}

static void born_free(born2d *S)
{
    free(S->M); free(S->U); free(S->B); free(S->g1); free(S->g2);
}

static real b_dpx(const born2d *S, const real *f, long c) { return dplus(f, c, 1, S->c, S->R) * S->ix; }
static real b_dmx(const born2d *S, const real *f, long c) { return dminus(f, c, 1, S->c, S->R) * S->ix; }
static real b_dpz(const born2d *S, const real *f, long c) { return dplus(f, c, S->px, S->c, S->R) * S->iz; }
static real b_dmz(const born2d *S, const real *f, long c) { return dminus(f, c, S->px, S->c, S->R) * S->iz; }

static void born_sources(real dm, real du, real rr, real e0xx, real e0zz, real e0xz, real a0x,
                         real a0z, real dt, real *sxx, real *szz, real *sxz, real *svx, real *svz);

/* isotropic combination of strain rates with moduli (m, u):
 * (m exx + (m-2u) ezz, m ezz + (m-2u) exx, u exz) */
static void iso(real m, real u, real exx, real ezz, real exz, real *o)
{
    o[0] = m * exx + (m - 2 * u) * ezz;
    o[1] = m * ezz + (m - 2 * u) * exx;
    o[2] = u * exz;
}

/* 2D state of one wavefield: velocities, stresses, memory variables r[comp][mech] */
typedef struct {
    real *vx, *vz, *sxx, *szz, *sxz;
    real *r[3][3];
} bstate;

/* one step of background (+ scattered when sc != NULL).  Stress with GSLS memory
 * variables (Crank-Nicolson decay, updated before the stress uses them):
 *   r_l' = ra_l r_l + rb_l f(e),  f = iso(pi tp, mu ts; e)
 *   sigma' = g1 (g2 sigma + dt (iso(pi kp, mu ks; e) + sum_l r_l'))
 * Scattered: the same with secondary sources iso(dpi kp, dmu ks; e0) in the stress
 * and iso(dpi tp, dmu ts; e0) in f, and -dt r_rho a0 in the velocity.  Stores v0
 * (start of step) and a0 into keep[4] when keep != NULL. */
static void born_step(const born2d *S, const orc_shot *s, int it, bstate *bg, bstate *sc,
                      const real *dpi, const real *dmu, const real *rr, real **keep)
{
    const real dt = S->dt;
    const int nm = S->nm;
    if (it < s->nw) {
        long c = B2(S, s->sx, s->sz);
        bg->sxx[c] += s->wavelet[it];
        bg->szz[c] += s->wavelet[it];
    }
    if (keep) {
        memcpy(keep[0], bg->vx, sizeof(real) * S->n);
        memcpy(keep[1], bg->vz, sizeof(real) * S->n);
    }
    real *bs[3] = {bg->sxx, bg->szz, bg->sxz};
    real *ss[3] = {sc ? sc->sxx : NULL, sc ? sc->szz : NULL, sc ? sc->sxz : NULL};
#pragma omp parallel for schedule(static)
    for (int k = 0; k < S->nz; k++)
        for (int i = 0; i < S->nx; i++) {
            long c = B2(S, i, k);
            real e0xx = b_dpx(S, bg->vx, c), e0zz = b_dmz(S, bg->vz, c);
            real e0xz = b_dpz(S, bg->vx, c) + b_dmx(S, bg->vz, c);
            real g1 = S->g1[c], g2 = S->g2[c], pi = S->M[c], mu = S->U[c];
            real E0[3], F0[3];
            iso(pi * S->kp, mu * S->ks, e0xx, e0zz, e0xz, E0);
            iso(pi * S->tp, mu * S->ts, e0xx, e0zz, e0xz, F0);
            for (int q = 0; q < 3; q++) {
                real sum = 0;
                for (int l = 0; l < nm; l++) {
                    real *r = bg->r[q][l];
                    r[c] = S->ra[l] * r[c] + S->rb[l] * F0[q];
                    sum += r[c];
                }
                bs[q][c] = g1 * (g2 * bs[q][c] + dt * (E0[q] + sum));
            }
            if (sc) {
                real exx = b_dpx(S, sc->vx, c), ezz = b_dmz(S, sc->vz, c);
                real exz = b_dpz(S, sc->vx, c) + b_dmx(S, sc->vz, c);
                real E[3], F[3], dE[3], dF[3], unused0, unused1;
                iso(pi * S->kp, mu * S->ks, exx, ezz, exz, E);
                iso(pi * S->tp, mu * S->ts, exx, ezz, exz, F);
                /* the reference's stress sources (dem_p), scaled by the GSLS strengths */
                born_sources(dpi[c] * S->kp, dmu[c] * S->ks, 0, e0xx, e0zz, e0xz, 0, 0, 1, &dE[0],
                             &dE[1], &dE[2], &unused0, &unused1);
                iso(dpi[c] * S->tp, dmu[c] * S->ts, e0xx, e0zz, e0xz, dF);
                for (int q = 0; q < 3; q++) {
                    real sum = 0;
                    for (int l = 0; l < nm; l++) {
                        real *r = sc->r[q][l];
                        r[c] = S->ra[l] * r[c] + S->rb[l] * (F[q] + dF[q]);
                        sum += r[c];
                    }
                    ss[q][c] = g1 * (g2 * ss[q][c] + dt * (E[q] + dE[q] + sum));
                }
            }
        }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < S->nz; k++)
        for (int i = 0; i < S->nx; i++) {
            long c = B2(S, i, k);
            real g1 = S->g1[c], g2 = S->g2[c], b = S->B[c];
            real a0x = b * (b_dmx(S, bg->sxx, c) + b_dmz(S, bg->sxz, c));
            real a0z = b * (b_dpx(S, bg->sxz, c) + b_dpz(S, bg->szz, c));
            if (keep) { keep[2][c] = a0x; keep[3][c] = a0z; }
            bg->vx[c] = g1 * (g2 * bg->vx[c] + dt * a0x);
            bg->vz[c] = g1 * (g2 * bg->vz[c] + dt * a0z);
            if (sc) {
                real ax = b * (b_dmx(S, sc->sxx, c) + b_dmz(S, sc->sxz, c));
                real az = b * (b_dpx(S, sc->sxz, c) + b_dpz(S, sc->szz, c));
                real q0, q1, q2, svx, svz;
                born_sources(0, 0, rr[c], 0, 0, 0, a0x, a0z, dt, &q0, &q1, &q2, &svx, &svz);
                sc->vx[c] = g1 * (g2 * sc->vx[c] + dt * ax + svx);
                sc->vz[c] = g1 * (g2 * sc->vz[c] + dt * az + svz);
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

/* allocate a zeroed state (memory variables for S->nm mechanisms) */
static int bstate_new(const born2d *S, bstate *b)
{
    memset(b, 0, sizeof *b);
    real **f[5] = {&b->vx, &b->vz, &b->sxx, &b->szz, &b->sxz};
    int bad = 0;
    for (int q = 0; q < 5; q++) if (!(*f[q] = zalloc(S->n))) bad = 1;
    for (int q = 0; q < 3; q++)
        for (int l = 0; l < S->nm; l++) if (!(b->r[q][l] = zalloc(S->n))) bad = 1;
    return bad ? -2 : 0;
}

static void bstate_free(bstate *b)
{
    free(b->vx); free(b->vz); free(b->sxx); free(b->szz); free(b->sxz);
    for (int q = 0; q < 3; q++)
        for (int l = 0; l < 3; l++) free(b->r[q][l]);
}

int orc_born_forward(const orc_grid *g, const float *vp, const float *vs, const float *rho,
                     const orc_shot *s, int nt, const float *r_vp, const float *r_vs,
                     const float *r_rho, float *data)
{
    born2d S;
    if (!s || !data || nt < 1 || s->nry != 1) return -1;
    int rc = born_setup(&S, g, vp, vs, rho);
    if (rc) { born_free(&S); return rc; }
    bstate bg, sc;
    real *dpi = zalloc(S.n), *dmu = zalloc(S.n), *rr = zalloc(S.n);
    rc = bstate_new(&S, &bg);
    if (!rc) rc = bstate_new(&S, &sc);
    if (!dpi || !dmu || !rr) rc = -2;
    if (!rc) {
        for (int k = 0; k < S.nz; k++)
            for (int i = 0; i < S.nx; i++) {
                long c = B2(&S, i, k), m = (long)k * S.nx + i;
                dpi[c] = S.M[c] * ((real)r_rho[m] + 2 * (real)r_vp[m]);
                dmu[c] = S.U[c] * ((real)r_rho[m] + 2 * (real)r_vs[m]);
                rr[c] = r_rho[m];
            }
        const long nrec = s->nrx;
        memset(data, 0, sizeof(float) * 3 * (size_t)nt * nrec);
        for (int it = 0; it < nt; it++) {
            born_step(&S, s, it, &bg, &sc, dpi, dmu, rr, NULL);
            for (long r = 0; r < nrec; r++) {
                long c;
                if (!born_rec(&S, s, (int)r, &c)) continue;
                data[((long)0 * nt + it) * nrec + r] = (float)sc.vx[c];
                data[((long)2 * nt + it) * nrec + r] = (float)sc.vz[c];
            }
        }
    }
    bstate_free(&bg); bstate_free(&sc);
    free(dpi); free(dmu); free(rr);
    born_free(&S);
    return rc;
}

/* Modelling pass of the Born background scheme (2D, sponge, GSLS memory
 * variables when g->visco_nmech > 0): records vx, vz at the receivers after
 * every step into data[3][nt][nrx] (vy row zero). */
int orc_visco_model(const orc_grid *g, const float *vp, const float *vs, const float *rho,
                    const orc_shot *s, int nt, float *data)
{
    born2d S;
    if (!s || !data || nt < 1 || s->nry != 1) return -1;
    int rc = born_setup(&S, g, vp, vs, rho);
    if (rc) { born_free(&S); return rc; }
    bstate bg;
    rc = bstate_new(&S, &bg);
    if (!rc) {
        const long nrec = s->nrx;
        memset(data, 0, sizeof(float) * 3 * (size_t)nt * nrec);
        for (int it = 0; it < nt; it++) {
            born_step(&S, s, it, &bg, NULL, NULL, NULL, NULL, NULL);
            for (long r = 0; r < nrec; r++) {
                long c;
                if (!born_rec(&S, s, (int)r, &c)) continue;
                data[((long)0 * nt + it) * nrec + r] = (float)bg.vx[c];
                data[((long)2 * nt + it) * nrec + r] = (float)bg.vz[c];
            }
        }
    }
    bstate_free(&bg);
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
    const int nm = S.nm;
    /* background history: v0 at the start of every step and a0 of every step */
    real *hist = (real *)malloc(sizeof(real) * (size_t)4 * n * nt);
    bstate bg;
    rc = bstate_new(&S, &bg);
    real *w[14], *lr[3][3] = {{0}};
    for (int q = 0; q < 14; q++) if (!(w[q] = zalloc(n))) rc = -2;
    for (int q = 0; q < 3; q++)
        for (int l = 0; l < nm; l++) if (!(lr[q][l] = zalloc(n))) rc = -2;
    if (!hist) rc = -2;
    if (!rc) {
        for (int it = 0; it < nt; it++) {
            real *keep[4] = {hist + (4L * it + 0) * n, hist + (4L * it + 1) * n,
                             hist + (4L * it + 2) * n, hist + (4L * it + 3) * n};
            born_step(&S, s, it, &bg, NULL, NULL, NULL, NULL, keep);
        }
        real *ax = w[0], *az = w[1], *hxx = w[2], *hzz = w[3], *hxz = w[4];
        real *gP = w[5], *gU = w[6], *gR = w[7], *tx = w[8], *tz = w[9];
        real *Sxx = w[10], *Szz = w[11], *Sxz = w[12], *Qb = w[13];
        (void)Qb;
        const long nrec = s->nrx;
        const real dt = S.dt;
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
            /* stress and memory-variable update^T: Q = g1 h is the adjoint of the
             * bracket; Lambda_l = lr_l + dt Q that of r_l'; P = sum_l rb_l Lambda_l
             * that of f; the strain adjoint S = dt E^T Q + F^T P */
#pragma omp parallel for schedule(static)
            for (int k = 0; k < S.nz; k++)
                for (int i = 0; i < S.nx; i++) {
                    long c = B2(&S, i, k);
                    real g1 = S.g1[c], pi = S.M[c], mu = S.U[c];
                    real Q[3] = {g1 * hxx[c], g1 * hzz[c], g1 * hxz[c]}, P[3] = {0, 0, 0};
                    for (int q = 0; q < 3; q++)
                        for (int l = 0; l < nm; l++) {
                            real lam = lr[q][l][c] + dt * Q[q];
                            P[q] += S.rb[l] * lam;
                            lr[q][l][c] = S.ra[l] * lam;
                        }
                    real e0xx = b_dpx(&S, hv0x, c), e0zz = b_dmz(&S, hv0z, c);
                    real e0xz = b_dpz(&S, hv0x, c) + b_dmx(&S, hv0z, c);
                    real div0 = e0xx + e0zz;
                    real tq = dt * Q[0], tz_ = dt * Q[1], tx_ = dt * Q[2];
                    gP[c] += (S.kp * (tq + tz_) + S.tp * (P[0] + P[1])) * div0;
                    gU[c] += S.ks * (-2 * tq * e0zz - 2 * tz_ * e0xx + tx_ * e0xz) +
                             S.ts * (-2 * P[0] * e0zz - 2 * P[1] * e0xx + P[2] * e0xz);
                    real E[3], F[3];
                    /* E^T and F^T are symmetric in (xx, zz): iso() gives them */
                    iso(pi * S.kp, mu * S.ks, tq, tz_, tx_, E);
                    iso(pi * S.tp, mu * S.ts, P[0], P[1], P[2], F);
                    Sxx[c] = E[0] + F[0];
                    Szz[c] = E[1] + F[1];
                    Sxz[c] = E[2] + F[2];
                    hxx[c] = S.g2[c] * Q[0];
                    hzz[c] = S.g2[c] * Q[1];
                    hxz[c] = S.g2[c] * Q[2];
                }
#pragma omp parallel for schedule(static)
            for (int k = 0; k < S.nz; k++)
                for (int i = 0; i < S.nx; i++) {
                    long c = B2(&S, i, k);
                    real g12 = S.g2[c] * S.g1[c];
                    ax[c] = g12 * ax[c] - (b_dmx(&S, Sxx, c) + b_dmz(&S, Sxz, c));
                    az[c] = g12 * az[c] - (b_dpz(&S, Szz, c) + b_dpx(&S, Sxz, c));
                }
        }
        for (int k = 0; k < S.nz; k++)
            for (int i = 0; i < S.nx; i++) {
                long c = B2(&S, i, k), m = (long)k * S.nx + i;
                g_vp[m] = (float)(2 * S.M[c] * gP[c]);
                g_vs[m] = (float)(2 * S.U[c] * gU[c]);
                g_rho[m] = (float)(S.M[c] * gP[c] + S.U[c] * gU[c] + gR[c]);
            }
    }
    for (int q = 0; q < 14; q++) free(w[q]);
    for (int q = 0; q < 3; q++)
        for (int l = 0; l < 3; l++) free(lr[q][l]);
    bstate_free(&bg);
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

/* Propagation angle on given 2D arrays (nz x nx, x fastest): the window angle of
 * window_angle over p = -tp (vxp, vzp), written at the cells whose excitation time
 * equals `it` (elsewhere `out` is left alone); hw = 2 (source, 5 x 5) or 4
 * (receiver, 9 x 9).  Pins the angle restatement to the reference's own
 * caculate_ex_angle_pp_only_RTM / _rp_only_RTM run on the same arrays. */
int orc_angle_given(int nx, int nz, int hw, int it, const float *tp, const float *vxp,
                    const float *vzp, const int *ex_time, float *out)
{
    if (nx <= 0 || nz <= 0 || hw < 0 || !tp || !vxp || !vzp || !ex_time || !out) return -1;
    for (int k = 0; k < nz; k++)
        for (int i = 0; i < nx; i++) {
            long m = (long)k * nx + i;
            if (ex_time[m] != it) continue;
            double sxz = 0.0, szz = 0.0;
            for (int dk = -hw; dk <= hw; dk++)
                for (int di = -hw; di <= hw; di++) {
                    int ii = i + di, kk = k + dk;
                    if (ii < 0 || ii >= nx || kk < 0 || kk >= nz) continue;
                    long q = (long)kk * nx + ii;
                    /* sum_poynting forms p in float (elastic_2D_kernel_2.cu:28-30) */
                    const float px = -tp[q] * vxp[q], pz = -tp[q] * vzp[q];
                    sxz += (double)px * (double)pz;
                    szz += (double)pz * (double)pz;
                }
            if (szz != 0.0) out[m] = angle_of_sums(sxz, szz);
        }
    return 0;
}
