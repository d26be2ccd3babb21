// Born (linearised) modelling and its exact adjoint, 2D elastic or viscoelastic
// (generalised standard linear solid, up to 3 mechanisms), sponge boundaries.
//
// Viscoelastic stress (a = attenuation strengths tp, ts of the tau method; pi =
// rho vp^2, mu = rho vs^2 relaxed moduli; iso(m, u; e) = (m exx + (m-2u) ezz,
// m ezz + (m-2u) exx, u exz)):
//   r_l'   = ra_l r_l + rb_l iso(pi tp, mu ts; e)          (Crank-Nicolson decay)
//   sigma' = g1 (g2 sigma + dt (iso(pi kp, mu ks; e) + sum_l r_l'))
// with kp = 1 + nm tp, ks = 1 + nm ts (unrelaxed / relaxed); nm = 0 is elastic.
// This is the reference's memory-variable update (fwd_txxzzxzpp_viscoelastic_and_memory,
// 2D_elastic_RTM/viscoelastic_equation.cu:184-325, one mechanism) generalised to nm.
//
// The scattered field obeys the background scheme with secondary sources from
// relative perturbations (r_vp, r_vs, r_rho) of the migration model:
//   stress   += dt (dM e0_xx + dL e0_zz,  dM e0_zz + dL e0_xx,  dU e0_xz)
//   velocity += -dt r_rho a0
// dM = M (r_rho + 2 r_vp), dU = U (r_rho + 2 r_vs), dL = dM - 2 dU; e0 are the
// background strain rates at the start of the step and a0 = b div(sigma0) the
// background acceleration of the step.  These are the secondary sources of
// cuda_cal_dem_parameter_viscoelastic_media_new (2D_elastic_RTM/viscoelastic_equation.cu
// :2398-2505, inversion_para 2) without attenuation, and they make the Born
// operator the exact derivative of the discrete background scheme.
//
// The adjoint applies the transpose of every step in reverse order (D+ and D-
// transpose to -D- and -D+ on the zero-padded grid).  Per reverse step:
//   k_adj_vel : h_s <- g2 g1 h_s (completes the previous reverse step) + velocity^T
//               contribution; rho gradient from a0
//   k_adj_str : stress^T: velocity adjoint update, M/L/U gradients from e0
// The background history (v0 at the start of each step, a0 of each step) is
// rebuilt per segment from checkpoints of the background state.
//
// Compact 2D layout: cell (i,k) at (k+R)*px + (i+XH), zero halos.
#include <cuda_runtime.h>

#include "born.cuh"

namespace ertm {

namespace {

template <int R>
__device__ __forceinline__ float dpx(const float* __restrict__ f, long long c, const BornArgs& a)
{
    float s = 0.f;
#pragma unroll
    for (int n = 1; n <= R; n++) s = fmaf(a.cx[n], __ldg(f + c + n) - __ldg(f + c - n + 1), s);
    return s;
}
template <int R>
__device__ __forceinline__ float dmx(const float* __restrict__ f, long long c, const BornArgs& a)
{
    float s = 0.f;
#pragma unroll
    for (int n = 1; n <= R; n++) s = fmaf(a.cx[n], __ldg(f + c + n - 1) - __ldg(f + c - n), s);
    return s;
}
// Rows k-R .. k+R of one field at the thread's column, carried down the warp's z
// chunk: each row is loaded once (one aligned 128-byte line per warp) and every
// z stencil reads registers.  dpz / dmz are the forward / backward z differences
// at row k with the same terms in the same order as the x differences above.
template <int R>
struct ZWin {
    float w[2 * R + 1];
    template <typename F>
    __device__ __forceinline__ void init(F f, long long c, long long p)
    {
#pragma unroll
        for (int j = 0; j <= 2 * R; j++) w[j] = f(c + (long long)(j - R) * p);
    }
    // c: the next row's cell
    template <typename F>
    __device__ __forceinline__ void shift(F f, long long c, long long p)
    {
#pragma unroll
        for (int j = 0; j < 2 * R; j++) w[j] = w[j + 1];
        w[2 * R] = f(c + (long long)R * p);
    }
    __device__ __forceinline__ float dpz(const float* cz) const
    {
        float s = 0.f;
#pragma unroll
        for (int n = 1; n <= R; n++) s = fmaf(cz[n], w[R + n] - w[R - n + 1], s);
        return s;
    }
    __device__ __forceinline__ float dmz(const float* cz) const
    {
        float s = 0.f;
#pragma unroll
        for (int n = 1; n <= R; n++) s = fmaf(cz[n], w[R + n - 1] - w[R - n], s);
        return s;
    }
};

// read-only field (not written by the kernel that reads it)
struct Ld {
    const float* p;
    __device__ __forceinline__ float operator()(long long c) const { return __ldg(p + c); }
};
// product of the shared B g1 (shot-independent, index c - zo) and the shot's own
// field w: the velocity update's transposed operand
struct Prod {
    const float* bg;
    const float* w;
    long long zo;
    __device__ __forceinline__ float operator()(long long c) const { return __ldg(bg + (c - zo)) * __ldg(w + c); }
};
template <int R, typename F>
__device__ __forceinline__ float tdpx(F f, long long c, const BornArgs& a)
{
    float s = 0.f;
#pragma unroll
    for (int n = 1; n <= R; n++) s = fmaf(a.cx[n], f(c + n) - f(c - n + 1), s);
    return s;
}
template <int R, typename F>
__device__ __forceinline__ float tdmx(F f, long long c, const BornArgs& a)
{
    float s = 0.f;
#pragma unroll
    for (int n = 1; n <= R; n++) s = fmaf(a.cx[n], f(c + n - 1) - f(c - n), s);
    return s;
}

// Work of one warp: a strip of 32 allocated columns (cells i = 32 w + lane - BXH, so
// every row access is one aligned 128-byte line) and a chunk of a.kc rows, marched
// top to bottom; blockIdx.z is the shot.  Lanes outside the grid (i < 0 or
// i >= nx: zero halo columns) load and compute like the others and store nothing.
constexpr int WPB = 4;       // warps per block: adjacent strips
struct Strip {
    int i, k0, k1;
    bool act;                // the lane's cell is inside the grid
    long long c;             // cell (i, k0) of the shared volumes
    long long zo;            // shot offset of the per-shot volumes
};
__device__ __forceinline__ bool strip_of(const BornArgs& a, Strip& s)
{
    const int w = blockIdx.x * WPB + threadIdx.y;
    s.k0 = blockIdx.y * a.kc;
    if (32 * w - BXH >= a.nx || s.k0 >= a.nz) return false;
    s.k1 = min(s.k0 + a.kc, a.nz);
    s.i = 32 * w + (int)threadIdx.x - BXH;
    s.act = s.i >= 0 && s.i < a.nx;
    s.c = (long long)(s.k0 + a.R) * a.px + 32 * w + threadIdx.x;
    s.zo = (long long)blockIdx.z * a.ss;
    return true;
}

// cell (i, k) of the launch's shot blockIdx.z: c indexes the shared volumes,
// c + zo (zo = shot * ss) the shot's own volumes
__device__ __forceinline__ bool cell_of(const BornArgs& a, int& i, int& k, long long& c, long long& zo)
{
    i = blockIdx.x * blockDim.x + threadIdx.x;
    k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= a.nx || k >= a.nz) return false;
    c = (long long)(k + a.R) * a.px + i + BXH;
    zo = (long long)blockIdx.z * a.ss;
    return true;
}

// the shot's parameters: sx, sz, rx0, nrx, drx, rz
__device__ __forceinline__ int shot_par(const BornArgs& a, int q) { return __ldg(a.shot_tab + blockIdx.z * 8 + q); }

__device__ __forceinline__ int recv_of(const BornArgs& a, int i, int k)
{
    if (k != shot_par(a, 5)) return -1;
    int d = i - shot_par(a, 2);
    const int drx = shot_par(a, 4);
    if (d < 0 || d % drx) return -1;
    d /= drx;
    return d < shot_par(a, 3) ? d : -1;
}

__device__ __forceinline__ float* shot_traces(const BornArgs& a) { return a.traces + blockIdx.z * a.tstride; }

__device__ __forceinline__ void iso(float m, float u, float exx, float ezz, float exz, float* o)
{
    const float l = m - 2.f * u;
    o[0] = m * exx + l * ezz;
    o[1] = m * ezz + l * exx;
    o[2] = u * exz;
}

// ---- forward ---------------------------------------------------------------
template <int R, bool BORN, int NM>
__global__ void __launch_bounds__(32 * WPB) k_born_stress(BornArgs a, int it)
{
    Strip S;
    if (!strip_of(a, S)) return;
    const long long p = a.px, zo = S.zo;
    const float dt = a.dt;
    const float* v0x = a.v0x + zo;
    const float* v0z = a.v0z + zo;
    const float* vx = a.vx + zo;
    const float* vz = a.vz + zo;
    // z windows: v0x and vx feed forward z differences, v0z and vz backward ones
    ZWin<R> w0x, w0z, wx, wz;
    w0x.init(Ld{v0x}, S.c, p);
    w0z.init(Ld{v0z}, S.c, p);
    if (BORN) {
        wx.init(Ld{vx}, S.c, p);
        wz.init(Ld{vz}, S.c, p);
    }
    const bool src_step = it >= 0 && it < a.nw;
    const int sx = shot_par(a, 0), sz = shot_par(a, 1);
    long long c = S.c;
    for (int k = S.k0; k < S.k1; k++, c += p) {
        const long long cz = c + zo;
        const float e0xx = dpx<R>(v0x, c, a), e0zz = w0z.dmz(a.cz);
        const float e0xz = w0x.dpz(a.cz) + dmx<R>(v0z, c, a);
        if (S.act) {
            // every load of the row before any store: a store through one of the
            // state pointers could alias a later load, which would serialise the
            // memory-variable updates into one round trip each
            const float g1 = __ldg(a.g1 + c), g2 = __ldg(a.g2 + c), pi = __ldg(a.M + c), mu = __ldg(a.U + c);
            float o[3] = {a.s0xx[cz], a.s0zz[cz], a.s0xz[cz]};
            float r0v[3][NM > 0 ? NM : 1], rv[3][NM > 0 ? NM : 1], so[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int q = 0; q < 3; q++)
#pragma unroll
                for (int l = 0; l < NM; l++) r0v[q][l] = a.r0[q * 3 + l][cz];
            float exx = 0.f, ezz = 0.f, exz = 0.f, dpi = 0.f, dmu = 0.f;
            if (BORN) {
                so[0] = a.sxx[cz];
                so[1] = a.szz[cz];
                so[2] = a.sxz[cz];
#pragma unroll
                for (int q = 0; q < 3; q++)
#pragma unroll
                    for (int l = 0; l < NM; l++) rv[q][l] = a.r[q * 3 + l][cz];
                exx = dpx<R>(vx, c, a);
                ezz = wz.dmz(a.cz);
                exz = wx.dpz(a.cz) + dmx<R>(vz, c, a);
                dpi = __ldg(a.dM + c);
                dmu = __ldg(a.dU + c);
            }
            if (src_step && S.i == sx && k == sz) {
                // explosive source into the background
                const float w = __ldg(a.wavelet + (long long)blockIdx.z * a.wstride + it);
                o[0] += w;
                o[1] += w;
            }
            float E0[3], F0[3];
            iso(pi * a.kp, mu * a.ks, e0xx, e0zz, e0xz, E0);
            if (NM) iso(pi * a.tp, mu * a.ts, e0xx, e0zz, e0xz, F0);
            float ns0[3];
#pragma unroll
            for (int q = 0; q < 3; q++) {
                float sum = 0.f;
#pragma unroll
                for (int l = 0; l < NM; l++) {
                    r0v[q][l] = a.ra[l] * r0v[q][l] + a.rb[l] * F0[q];
                    sum += r0v[q][l];
                }
                ns0[q] = g1 * (g2 * o[q] + dt * (E0[q] + sum));
            }
            float nsc[3];
            if (BORN) {
                float E[3], dE[3], F[3], dF[3];
                iso(pi * a.kp, mu * a.ks, exx, ezz, exz, E);
                // the reference's stress sources (dem_p), scaled by the GSLS strengths
                iso(dpi * a.kp, dmu * a.ks, e0xx, e0zz, e0xz, dE);
                if (NM) {
                    iso(pi * a.tp, mu * a.ts, exx, ezz, exz, F);
                    iso(dpi * a.tp, dmu * a.ts, e0xx, e0zz, e0xz, dF);
                }
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    float sum = 0.f;
#pragma unroll
                    for (int l = 0; l < NM; l++) {
                        rv[q][l] = a.ra[l] * rv[q][l] + a.rb[l] * (F[q] + dF[q]);
                        sum += rv[q][l];
                    }
                    nsc[q] = g1 * (g2 * so[q] + dt * (E[q] + dE[q] + sum));
                }
            }
            // stores
            a.s0xx[cz] = ns0[0];
            a.s0zz[cz] = ns0[1];
            a.s0xz[cz] = ns0[2];
#pragma unroll
            for (int q = 0; q < 3; q++)
#pragma unroll
                for (int l = 0; l < NM; l++) a.r0[q * 3 + l][cz] = r0v[q][l];
            if (BORN) {
                a.sxx[cz] = nsc[0];
                a.szz[cz] = nsc[1];
                a.sxz[cz] = nsc[2];
#pragma unroll
                for (int q = 0; q < 3; q++)
#pragma unroll
                    for (int l = 0; l < NM; l++) a.r[q * 3 + l][cz] = rv[q][l];
            }
        }
        if (k + 1 < S.k1) {
            w0x.shift(Ld{v0x}, c + p, p);
            w0z.shift(Ld{v0z}, c + p, p);
            if (BORN) {
                wx.shift(Ld{vx}, c + p, p);
                wz.shift(Ld{vz}, c + p, p);
            }
        }
    }
}

template <int R, bool BORN, bool KEEP>
__global__ void __launch_bounds__(32 * WPB) k_born_velocity(BornArgs a, int it)
{
    Strip S;
    if (!strip_of(a, S)) return;
    const long long p = a.px, zo = S.zo;
    const float dt = a.dt;
    const float* s0xx = a.s0xx + zo;
    const float* s0xz = a.s0xz + zo;
    const float* s0zz = a.s0zz + zo;
    const float* sxx = a.sxx + zo;
    const float* sxz = a.sxz + zo;
    const float* szz = a.szz + zo;
    ZWin<R> w0xz, w0zz, wxz, wzz;      // sigma_xz: backward z difference; sigma_zz: forward
    w0xz.init(Ld{s0xz}, S.c, p);
    w0zz.init(Ld{s0zz}, S.c, p);
    if (BORN) {
        wxz.init(Ld{sxz}, S.c, p);
        wzz.init(Ld{szz}, S.c, p);
    }
    const int rz = a.traces ? shot_par(a, 5) : -1;
    long long c = S.c;
    for (int k = S.k0; k < S.k1; k++, c += p) {
        const long long cz = c + zo;
        const float b = __ldg(a.B + c);
        const float a0x = b * (dmx<R>(s0xx, c, a) + w0xz.dmz(a.cz));
        const float a0z = b * (dpx<R>(s0xz, c, a) + w0zz.dpz(a.cz));
        float ax = 0.f, az = 0.f;
        if (BORN) {
            ax = b * (dmx<R>(sxx, c, a) + wxz.dmz(a.cz));
            az = b * (dpx<R>(sxz, c, a) + wzz.dpz(a.cz));
        }
        if (S.act) {
            // every load of the row before any store (see k_born_stress)
            const float g1 = __ldg(a.g1 + c), g2 = __ldg(a.g2 + c);
            const float ov0x = a.v0x[cz], ov0z = a.v0z[cz];
            float ovx = 0.f, ovz = 0.f, r = 0.f;
            if (BORN) {
                ovx = a.vx[cz];
                ovz = a.vz[cz];
                r = __ldg(a.rr + c);
            }
            if (KEEP) {   // background history for the adjoint: v0 at the start of the step, a0
                a.kv0x[cz] = ov0x;
                a.kv0z[cz] = ov0z;
                a.ka0x[cz] = a0x;
                a.ka0z[cz] = a0z;
            }
            a.v0x[cz] = g1 * (g2 * ov0x + dt * a0x);
            a.v0z[cz] = g1 * (g2 * ov0z + dt * a0z);
            if (BORN) {
                const float nvx = g1 * (g2 * ovx + dt * (ax - r * a0x));
                const float nvz = g1 * (g2 * ovz + dt * (az - r * a0z));
                a.vx[cz] = nvx;
                a.vz[cz] = nvz;
                const int rec = k == rz ? recv_of(a, S.i, k) : -1;
                if (rec >= 0) {
                    const long long nrec = a.nrx, cs = (long long)a.nt * nrec;
                    float* d = shot_traces(a) + (long long)it * nrec + rec;
                    d[0] = nvx;
                    d[cs] = 0.f;
                    d[2 * cs] = nvz;
                }
            }
        }
        if (k + 1 < S.k1) {
            w0xz.shift(Ld{s0xz}, c + p, p);
            w0zz.shift(Ld{s0zz}, c + p, p);
            if (BORN) {
                wxz.shift(Ld{sxz}, c + p, p);
                wzz.shift(Ld{szz}, c + p, p);
            }
        }
    }
}

// ---- adjoint ---------------------------------------------------------------
// residual sample `it` of every shot's receivers into its velocity adjoint
// (grid: receivers x, shots y)
__global__ void k_adj_inject(BornArgs a, int it)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int sh = blockIdx.y;
    const int* t = a.shot_tab + sh * 8;
    if (r >= t[3]) return;
    const int i = t[2] + r * t[4], rz = t[5];
    if (i < 0 || i >= a.nx || rz < 0 || rz >= a.nz) return;
    const long long c = (long long)(rz + a.R) * a.px + i + BXH + (long long)sh * a.ss;
    const long long nrec = a.nrx, cs = (long long)a.nt * nrec;
    const float* d = a.traces + sh * a.tstride + (long long)it * nrec + r;
    a.ax[c] += d[0];
    a.az[c] += d[2 * cs];
}

// velocity update^T: h (the stress adjoint, already carried through g2 g1 by
// k_adj_mem) gains the velocity update's stencil transposed, applied to the
// products B g1 a^; rho gradient from a0
template <int R>
__global__ void __launch_bounds__(32 * WPB) k_adj_vel(BornArgs a)
{
    Strip S;
    if (!strip_of(a, S)) return;
    const long long p = a.px, zo = S.zo;
    const float dt = a.dt;
    const Prod tx{a.Bg1, a.ax, zo}, tz{a.Bg1, a.az, zo};
    ZWin<R> wx, wz;                    // products: forward z difference of x, backward of z
    wx.init(tx, S.c + zo, p);
    wz.init(tz, S.c + zo, p);
    long long c = S.c;
    for (int k = S.k0; k < S.k1; k++, c += p) {
        const long long cz = c + zo;
        const float dxx = tdpx<R>(tx, cz, a);
        const float dxz = wx.dpz(a.cz) + tdmx<R>(tz, cz, a);
        const float dzz = wz.dmz(a.cz);
        if (S.act) {
            // every load of the row before any store (see k_born_stress)
            const float g1 = __ldg(a.g1 + c);
            const float gr = a.gR[cz], hxx = a.hxx[cz], hxz = a.hxz[cz], hzz = a.hzz[cz];
            const float vax = __ldg(a.ax + cz), vaz = __ldg(a.az + cz);
            const float h0x = __ldg(a.ha0x + cz), h0z = __ldg(a.ha0z + cz);
            // rho gradient: -dt g1 (vx^ a0x + vz^ a0z)
            a.gR[cz] = gr + -dt * (g1 * vax * h0x + g1 * vaz * h0z);
            a.hxx[cz] = hxx - dt * dxx;
            a.hxz[cz] = hxz - dt * dxz;
            a.hzz[cz] = hzz - dt * dzz;
        }
        if (k + 1 < S.k1) {
            wx.shift(tx, cz + p, p);
            wz.shift(tz, cz + p, p);
        }
    }
}

// stress and memory-variable update^T of one cell: Q = g1 h is the adjoint of
// the stress bracket, Lambda_l = lr_l + dt Q that of r_l', P = sum_l rb_l Lambda_l
// that of f; writes the strain adjoint S = iso(pi kp, mu ks; dt Q) + iso(pi tp,
// mu ts; P) (both maps are symmetric), carries lr_l = ra_l Lambda_l and h = g2 Q,
// and accumulates the pi and mu gradients from the background strain rates.
template <int R, int NM>
__global__ void __launch_bounds__(32 * WPB) k_adj_mem(BornArgs a)
{
    Strip S;
    if (!strip_of(a, S)) return;
    const long long p = a.px, zo = S.zo;
    const float dt = a.dt;
    const float* hv0x = a.hv0x + zo;
    const float* hv0z = a.hv0z + zo;
    ZWin<R> wx, wz;
    wx.init(Ld{hv0x}, S.c, p);
    wz.init(Ld{hv0z}, S.c, p);
    long long c = S.c;
    for (int k = S.k0; k < S.k1; k++, c += p) {
        const long long cz = c + zo;
        const float e0xx = dpx<R>(hv0x, c, a), e0zz = wz.dmz(a.cz);
        const float e0xz = wx.dpz(a.cz) + dmx<R>(hv0z, c, a);
        if (S.act) {
            // every load of the row before any store (see k_born_stress)
            const float g1 = __ldg(a.g1 + c), g2 = __ldg(a.g2 + c), pi = __ldg(a.M + c), mu = __ldg(a.U + c);
            const float Q[3] = {g1 * a.hxx[cz], g1 * a.hzz[cz], g1 * a.hxz[cz]};
            float lv[3][NM > 0 ? NM : 1];
#pragma unroll
            for (int q = 0; q < 3; q++)
#pragma unroll
                for (int l = 0; l < NM; l++) lv[q][l] = a.lr[q * 3 + l][cz];
            const float gm = a.gM[cz], gu = a.gU[cz];
            float P[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int q = 0; q < 3; q++)
#pragma unroll
                for (int l = 0; l < NM; l++) {
                    const float lam = lv[q][l] + dt * Q[q];
                    P[q] += a.rb[l] * lam;
                    lv[q][l] = a.ra[l] * lam;
                }
            const float tq0 = dt * Q[0], tq1 = dt * Q[1], tq2 = dt * Q[2];
            const float ngm = gm + (a.kp * (tq0 + tq1) + a.tp * (P[0] + P[1])) * (e0xx + e0zz);
            const float ngu = gu + (a.ks * (-2.f * tq0 * e0zz - 2.f * tq1 * e0xx + tq2 * e0xz) +
                                    a.ts * (-2.f * P[0] * e0zz - 2.f * P[1] * e0xx + P[2] * e0xz));
            float E[3], F[3] = {0.f, 0.f, 0.f};
            iso(pi * a.kp, mu * a.ks, tq0, tq1, tq2, E);
            if (NM) iso(pi * a.tp, mu * a.ts, P[0], P[1], P[2], F);
#pragma unroll
            for (int q = 0; q < 3; q++)
#pragma unroll
                for (int l = 0; l < NM; l++) a.lr[q * 3 + l][cz] = lv[q][l];
            a.gM[cz] = ngm;
            a.gU[cz] = ngu;
            a.Sxx[cz] = E[0] + F[0];
            a.Szz[cz] = E[1] + F[1];
            a.Sxz[cz] = E[2] + F[2];
            a.hxx[cz] = g2 * Q[0];
            a.hzz[cz] = g2 * Q[1];
            a.hxz[cz] = g2 * Q[2];
        }
        if (k + 1 < S.k1) {
            wx.shift(Ld{hv0x}, c + p, p);
            wz.shift(Ld{hv0z}, c + p, p);
        }
    }
}

// velocity adjoint: a <- g2 g1 a (the velocity update^T) - D^T S (the stress
// update's stencils transposed), plus the next (earlier) step's residual
template <int R>
__global__ void __launch_bounds__(32 * WPB) k_adj_str(BornArgs a, int it_next)
{
    Strip S;
    if (!strip_of(a, S)) return;
    const long long p = a.px, zo = S.zo;
    const Ld sxx{a.Sxx + zo}, szz{a.Szz + zo}, sxz{a.Sxz + zo};
    ZWin<R> wxz, wzz;                  // S_xz: backward z difference; S_zz: forward
    wxz.init(sxz, S.c, p);
    wzz.init(szz, S.c, p);
    const int rz = it_next >= 0 ? shot_par(a, 5) : -1;
    long long c = S.c;
    for (int k = S.k0; k < S.k1; k++, c += p) {
        const long long cz = c + zo;
        const float dx = tdmx<R>(sxx, c, a) + wxz.dmz(a.cz);
        const float dz = wzz.dpz(a.cz) + tdpx<R>(sxz, c, a);
        if (S.act) {
            const float g12 = __ldg(a.g2 + c) * __ldg(a.g1 + c);
            float nx = g12 * a.ax[cz] - dx;
            float nz = g12 * a.az[cz] - dz;
            const int rec = k == rz ? recv_of(a, S.i, k) : -1;
            if (rec >= 0) {
                const long long nrec = a.nrx, cs = (long long)a.nt * nrec;
                const float* d = shot_traces(a) + (long long)it_next * nrec + rec;
                nx += d[0];
                nz += d[2 * cs];
            }
            a.ax[cz] = nx;
            a.az[cz] = nz;
        }
        if (k + 1 < S.k1) {
            wxz.shift(sxz, c + p, p);
            wzz.shift(szz, c + p, p);
        }
    }
}

// gradients w.r.t. (r_vp, r_vs, r_rho) on the contiguous nz x nx grid, summed over
// the launch's shots (in shot order) and added to the outputs when `accumulate`
__global__ void k_born_final(BornArgs a, float* gvp, float* gvs, float* grho, int accumulate)
{
    int i, k;
    long long c, zo;
    if (!cell_of(a, i, k, c, zo)) return;
    const long long m = (long long)k * a.nx + i;
    float gp = 0.f, gu = 0.f, gr = 0.f;
    for (int sh = 0; sh < a.nshot; sh++) {
        const long long q = c + sh * a.ss;
        gp += a.gM[q];
        gu += a.gU[q];
        gr += a.gR[q];
    }
    const float ovp = accumulate ? gvp[m] : 0.f, ovs = accumulate ? gvs[m] : 0.f;
    const float orho = accumulate ? grho[m] : 0.f;
    gvp[m] = ovp + 2.f * a.M[c] * gp;
    gvs[m] = ovs + 2.f * a.U[c] * gu;
    grho[m] = orho + (a.M[c] * gp + a.U[c] * gu + gr);
}

// model products (copied from the context's padded model, plane j = 0), damping
// factors and B g1 on the compact layout
__global__ void k_born_model(BornArgs a, const float* Mc, const float* Uc, const float* Bc,
                             long long csz, const float* att_x, const float* att_z, float* M,
                             float* U, float* Bg1, float* B, float* g1, float* g2)
{
    int i, k;
    long long c;
    long long zo;
    if (!cell_of(a, i, k, c, zo)) return;
    const long long m = (long long)k * csz + i;
    M[c] = Mc[m];
    U[c] = Uc[m];
    B[c] = Bc[m];
    const float at = att_z[k] + att_x[i];
    const float h = at * a.dt * 0.5f;
    g1[c] = 1.f / (1.f + h);
    g2[c] = 1.f - h;
    Bg1[c] = B[c] * g1[c];
}

__global__ void k_born_pert(BornArgs a, const float* rvp, const float* rvs, const float* rrho,
                            float* dM, float* dU, float* rr)
{
    int i, k;
    long long c;
    long long zo;
    if (!cell_of(a, i, k, c, zo)) return;
    const long long m = (long long)k * a.nx + i;
    dM[c] = a.M[c] * (rrho[m] + 2.f * rvp[m]);
    dU[c] = a.U[c] * (rrho[m] + 2.f * rvs[m]);
    rr[c] = rrho[m];
}

dim3 born_grid(const BornArgs& a, int shots = 1) { return dim3((a.nx + 31) / 32, (a.nz + 7) / 8, shots); }

// The marching kernels' arguments and grid: WPB strips per block, chunks of kc
// rows, one grid layer per shot.  kc is the longest chunk (32, 16 or 8 rows) that
// still gives about two waves of blocks on the device (a shorter chunk reloads
// the 2R rows of its z windows more often).
BornArgs march(const BornArgs& a, dim3& grid)
{
    static const int sms = [] {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n > 0 ? n : 148;
    }();
    BornArgs b = a;
    const long long xb = ((a.nx + BXH + 31) / 32 + WPB - 1) / WPB;
    b.kc = 8;
    for (int kc = 32; kc > 8; kc /= 2)
        if (xb * ((a.nz + kc - 1) / kc) * a.nshot >= 2LL * 7 * sms) {
            b.kc = kc;
            break;
        }
    grid = dim3((unsigned)xb, (a.nz + b.kc - 1) / b.kc, a.nshot);
    return b;
}

}  // namespace

cudaError_t born_launch_model(const BornArgs& a, const float* Mc, const float* Uc, const float* Bc,
                              long long csz, const float* att_x, const float* att_z, float* M,
                              float* U, float* Bg1, float* B, float* g1, float* g2, cudaStream_t s)
{
    k_born_model<<<born_grid(a), dim3(32, 8), 0, s>>>(a, Mc, Uc, Bc, csz, att_x, att_z, M, U, Bg1, B,
                                                      g1, g2);
    return cudaGetLastError();
}

cudaError_t born_launch_pert(const BornArgs& a, const float* rvp, const float* rvs,
                             const float* rrho, float* dM, float* dU, float* rr, cudaStream_t s)
{
    k_born_pert<<<born_grid(a), dim3(32, 8), 0, s>>>(a, rvp, rvs, rrho, dM, dU, rr);
    return cudaGetLastError();
}

namespace {
template <int R, int NM>
void step_r(const BornArgs& a0, int it, bool born, bool keep, cudaStream_t s)
{
    dim3 g;
    const BornArgs a = march(a0, g);
    const dim3 b(32, WPB);
    if (born) k_born_stress<R, true, NM><<<g, b, 0, s>>>(a, it);
    else k_born_stress<R, false, NM><<<g, b, 0, s>>>(a, it);
    if (born) k_born_velocity<R, true, false><<<g, b, 0, s>>>(a, it);
    else if (keep) k_born_velocity<R, false, true><<<g, b, 0, s>>>(a, it);
    else k_born_velocity<R, false, false><<<g, b, 0, s>>>(a, it);
}
template <int R, int NM>
void adj_r(const BornArgs& a0, int it, cudaStream_t s)
{
    dim3 g;
    const BornArgs a = march(a0, g);
    const dim3 b(32, WPB);
    k_adj_vel<R><<<g, b, 0, s>>>(a);
    k_adj_mem<R, NM><<<g, b, 0, s>>>(a);
    k_adj_str<R><<<g, b, 0, s>>>(a, it - 1);
}
template <int R>
void step_nm(const BornArgs& a, int it, bool born, bool keep, cudaStream_t s)
{
    switch (a.nm) {
    case 0: step_r<R, 0>(a, it, born, keep, s); break;
    case 1: step_r<R, 1>(a, it, born, keep, s); break;
    case 2: step_r<R, 2>(a, it, born, keep, s); break;
    default: step_r<R, 3>(a, it, born, keep, s); break;
    }
}
template <int R>
void adj_nm(const BornArgs& a, int it, cudaStream_t s)
{
    switch (a.nm) {
    case 0: adj_r<R, 0>(a, it, s); break;
    case 1: adj_r<R, 1>(a, it, s); break;
    case 2: adj_r<R, 2>(a, it, s); break;
    default: adj_r<R, 3>(a, it, s); break;
    }
}
}  // namespace

cudaError_t born_launch_step(const BornArgs& a, int it, bool born, bool keep, cudaStream_t s)
{
    if (a.R == 4) step_nm<4>(a, it, born, keep, s);
    else step_nm<6>(a, it, born, keep, s);
    return cudaGetLastError();
}

cudaError_t born_launch_adjoint_step(const BornArgs& a, int it, cudaStream_t s)
{
    if (a.R == 4) adj_nm<4>(a, it, s);
    else adj_nm<6>(a, it, s);
    return cudaGetLastError();
}

cudaError_t born_launch_inject(const BornArgs& a, int it, cudaStream_t s)
{
    if (a.nrx <= 0) return cudaSuccess;
    k_adj_inject<<<dim3((a.nrx + 127) / 128, a.nshot), 128, 0, s>>>(a, it);
    return cudaGetLastError();
}

cudaError_t born_launch_final(const BornArgs& a, float* gvp, float* gvs, float* grho, bool accumulate,
                              cudaStream_t s)
{
    k_born_final<<<born_grid(a), dim3(32, 8), 0, s>>>(a, gvp, gvs, grho, accumulate ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace ertm
