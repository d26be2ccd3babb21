// Host set-up shared by every entry point that runs the step kernels: the
// padded-volume geometry, the difference coefficients, the absorbing-boundary
// profiles and the z-chunk rule.  The context path (ertm_api.cu) and the
// no-allocation modelling path (noalloc.cu) both call these, so the two can
// never drift apart.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "ertm_internal.cuh"

namespace ertm {

static long long rup(long long v, long long m) { return (v + m - 1) / m * m; }

Geom make_geom(int nx, int ny, int nz, int R)
{
    Geom g{};
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.R = R;
    g.two_d = (ny == 1);
    g.tyb = g.two_d ? TY2 : TY3;
    g.hx = XH;
    g.hy = g.two_d ? 0 : R;
    g.hz = R;
    g.px = rup(2LL * g.hx + rup(nx, TX), 32);
    g.py = 2LL * g.hy + rup(ny, g.tyb);
    g.pz = 2LL * g.hz + nz + 1;
    g.sy = g.px;
    g.sz = g.px * g.py;
    g.off0 = g.hz * g.sz + g.hy * g.sy + g.hx;
    g.total = g.px * g.py * g.pz;
    return g;
}

void stencil_coefs(int coef_kind, const float* user, int R, float coef[8])
{
    for (int n = 0; n < 8; n++) coef[n] = 0.f;
    if (coef_kind == ERTM_COEF_USER) {
        for (int n = 0; n <= R && n < 8; n++) coef[n] = user[n];
        return;
    }
    if (coef_kind == ERTM_COEF_REFERENCE12) {
        // the reference's 12-point set (3D_elastic_RTM/zzzzz:202-210)
        const float r12[7] = {0.0f, 1.2213363647f, -0.096931457519f, 0.017447662353f,
                              -0.0029672895159f, 0.00035900539822f, -0.00002184781161f};
        for (int n = 0; n < 7; n++) coef[n] = r12[n];
        return;
    }
    // Taylor weights of the staggered first derivative: sum_n c_n (2n-1)^(2m-1) = delta_m1,
    // solved by Gauss-Jordan elimination with partial pivoting in double
    double A[8][9];
    for (int m = 0; m < R; m++) {
        for (int n = 0; n < R; n++) A[m][n] = std::pow(2.0 * n + 1.0, 2.0 * m + 1.0);
        A[m][R] = (m == 0);
    }
    for (int cc = 0; cc < R; cc++) {
        int p = cc;
        for (int r = cc + 1; r < R; r++)
            if (std::fabs(A[r][cc]) > std::fabs(A[p][cc])) p = r;
        for (int k = 0; k <= R; k++) std::swap(A[cc][k], A[p][k]);
        for (int r = 0; r < R; r++) {
            if (r == cc) continue;
            const double f = A[r][cc] / A[cc][cc];
            for (int k = cc; k <= R; k++) A[r][k] -= f * A[cc][k];
        }
    }
    for (int n = 0; n < R; n++) coef[n + 1] = (float)(A[n][R] / A[n][n]);
}

void cpml_profile(int n, int w0, int w1, int stg, double h, double vmax, double rcoef, double f0,
                  double dts, int i0, int m, float* a, float* b)
{
    // C-PML (Komatitsch & Martin 2007) with kappa = 1: quadratic damping d, alpha
    // falling linearly from pi f0 at the inner edge to 0 at the outer edge;
    // the oracle's orc_cpml_profile computes the same values
    for (int q = 0; q < m; q++) {
        const double p = i0 + q + 0.5 * stg;
        double dist = 0.0, L = 1.0;
        if (w0 > 0 && p < w0 - 1) { dist = (w0 - 1) - p; L = w0; }
        else if (w1 > 0 && p > n - w1) { dist = p - (n - w1); L = w1; }
        if (dist <= 0.0) {
            a[q] = 0.f;
            b[q] = 1.f;
            continue;
        }
        const double Lm = L * h, x = dist * h / Lm;
        const double d = -3.0 * vmax * std::log(rcoef) / (2.0 * Lm) * x * x;
        double al = M_PI * f0 * (1.0 - x);
        if (al < 0) al = 0;
        const double bb = std::exp(-(d + al) * dts);
        b[q] = (float)bb;
        a[q] = (float)(d * (bb - 1.0) / (d + al));
    }
}

void sponge_profile(int n, int w0, int w1, int kind, float coe, int i0, int m, float* v)
{
    // coe_attenuation_3d_new2 (3D_elastic_RTM/3D_zzzzz:261-300): cosine ramp;
    // make_attenuation_new (3D_elastic_RTM/zzzzz:238-280): cubic ramp.  The
    // near-side ramp then the far-side ramp accumulate into a float, as the
    // reference's two loops do.
    const double pai = 3.1415926;   // 3D_zzzzz:1
    for (int q = 0; q < m; q++) {
        const int i = i0 + q;
        float acc = 0.f;
        if (i < w0) {
            float val;
            if (kind == ERTM_BOUNDARY_SPONGE_COS)
                val = (float)(coe * (1.0 - std::cos(pai / 2 * (w0 - i - 1) / (w0 - 1))));
            else {
                const float x = (float)((w0 - 1.0 - i) / (w0 - 1.0));
                val = (float)(coe * std::pow(x * 1.0, 3.0));
            }
            acc += val;
        }
        if (w1 > 0 && i >= n - w1) {
            const int k = i - (n - w1);
            float val;
            if (kind == ERTM_BOUNDARY_SPONGE_COS)
                val = (float)(coe * (1.0 - std::cos(pai / 2 * k / (w1 - 1))));
            else {
                const float x = (float)(k / (w1 - 1.0));
                val = (float)(coe * std::pow(x * 1.0, 3.0));
            }
            acc += val;
        }
        v[q] = acc;
    }
}

// z planes per CTA.  3D: chunks of about 32 planes, balanced over nz.  Timed on
// B200 at 480 x 480 x 380 (R = 4, C-PML), the step kernels get faster as the
// chunk shrinks from the whole column (380 planes) down to 32-48 planes
// (stress 1.92 -> 1.51 ms, velocity 1.98 -> 1.61 ms per launch), while below
// ~24 planes the z-queue fill of each chunk starts to cost more than the finer
// load balance gains.  2D: the chunk count minimises (waves of CTAs) x
// (planes per chunk + start-up of ~2R planes).
int choose_kchunk(const Geom& g, int R, int device)
{
    if (!g.two_d) {
        const int target = 32;
        const int chunks = std::max(1, (g.nz + target / 2) / target);
        return (g.nz + chunks - 1) / chunks;
    }
    const long long cols = (long long)((g.nx + TX - 1) / TX) * ((g.ny + g.tyb - 1) / g.tyb);
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        sms = 148;
    }
    const long long slots = (long long)sms * 8;
    const double startup = 2.0 * R;
    int best = g.nz;
    double best_cost = 1e300;
    for (int kc = g.nz; kc >= std::min(g.nz, 16); kc--) {
        const long long chunks = (g.nz + kc - 1) / kc;
        const long long waves = (cols * chunks + slots - 1) / slots;
        const double cost = (double)waves * (kc + startup);
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best = kc;
        }
    }
    return best;
}

}  // namespace ertm
