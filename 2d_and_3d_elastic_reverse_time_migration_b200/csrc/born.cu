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
template <int R>
__device__ __forceinline__ float dpz(const float* __restrict__ f, long long c, const BornArgs& a)
{
    const long long p = a.px;
    float s = 0.f;
#pragma unroll
    for (int n = 1; n <= R; n++) s = fmaf(a.cz[n], __ldg(f + c + n * p) - __ldg(f + c - (n - 1) * p), s);
    return s;
}
template <int R>
__device__ __forceinline__ float dmz(const float* __restrict__ f, long long c, const BornArgs& a)
{
    const long long p = a.px;
    float s = 0.f;
#pragma unroll
    for (int n = 1; n <= R; n++) s = fmaf(a.cz[n], __ldg(f + c + (n - 1) * p) - __ldg(f + c - n * p), s);
    return s;
}

// products of neighbours for the transposed stencils: f(c) = p(c - zo) q(c - zo) w(c),
// p and q shared by the shots of a launch, w the shot's own volume (offset zo)
struct Prod2 {
    const float* p;
    const float* q;
    const float* w;
    long long zo;
    __device__ __forceinline__ float operator()(long long c) const
    {
        return __ldg(p + (c - zo)) * __ldg(q + (c - zo)) * w[c];
    }
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
template <int R, typename F>
__device__ __forceinline__ float tdpz(F f, long long c, const BornArgs& a)
{
    const long long p = a.px;
    float s = 0.f;
#pragma unroll
    for (int n = 1; n <= R; n++) s = fmaf(a.cz[n], f(c + n * p) - f(c - (n - 1) * p), s);
    return s;
}
template <int R, typename F>
__device__ __forceinline__ float tdmz(F f, long long c, const BornArgs& a)
{
    const long long p = a.px;
    float s = 0.f;
#pragma unroll
    for (int n = 1; n <= R; n++) s = fmaf(a.cz[n], f(c + (n - 1) * p) - f(c - n * p), s);
    return s;
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
__global__ void k_born_stress(BornArgs a, int it)
{
    int i, k;
    long long c, zo;
    if (!cell_of(a, i, k, c, zo)) return;
    const long long cz = c + zo;
    const float dt = a.dt;
    const float g1 = a.g1[c], g2 = a.g2[c], pi = a.M[c], mu = a.U[c];
    const float *v0x = a.v0x + zo, *v0z = a.v0z + zo;
    const float e0xx = dpx<R>(v0x, c, a), e0zz = dmz<R>(v0z, c, a);
    const float e0xz = dpz<R>(v0x, c, a) + dmx<R>(v0z, c, a);
    float o[3] = {a.s0xx[cz], a.s0zz[cz], a.s0xz[cz]};
    if (it >= 0 && it < a.nw && i == shot_par(a, 0) && k == shot_par(a, 1)) {
        // explosive source into the background
        const float w = __ldg(a.wavelet + (long long)blockIdx.z * a.wstride + it);
        o[0] += w;
        o[1] += w;
    }
    float E0[3], F0[3];
    iso(pi * a.kp, mu * a.ks, e0xx, e0zz, e0xz, E0);
    if (NM) iso(pi * a.tp, mu * a.ts, e0xx, e0zz, e0xz, F0);
    float* s0[3] = {a.s0xx, a.s0zz, a.s0xz};
#pragma unroll
    for (int q = 0; q < 3; q++) {
        float sum = 0.f;
#pragma unroll
        for (int l = 0; l < NM; l++) {
            float* r = a.r0[q * 3 + l];
            const float v = a.ra[l] * r[cz] + a.rb[l] * F0[q];
            r[cz] = v;
            sum += v;
        }
        s0[q][cz] = g1 * (g2 * o[q] + dt * (E0[q] + sum));
    }
    if (BORN) {
        const float *vx = a.vx + zo, *vz = a.vz + zo;
        const float exx = dpx<R>(vx, c, a), ezz = dmz<R>(vz, c, a);
        const float exz = dpz<R>(vx, c, a) + dmx<R>(vz, c, a);
        const float dpi = a.dM[c], dmu = a.dU[c];
        float E[3], dE[3], F[3], dF[3];
        iso(pi * a.kp, mu * a.ks, exx, ezz, exz, E);
        // the reference's stress sources (dem_p), scaled by the GSLS strengths
        iso(dpi * a.kp, dmu * a.ks, e0xx, e0zz, e0xz, dE);
        if (NM) {
            iso(pi * a.tp, mu * a.ts, exx, ezz, exz, F);
            iso(dpi * a.tp, dmu * a.ts, e0xx, e0zz, e0xz, dF);
        }
        float* sc[3] = {a.sxx, a.szz, a.sxz};
#pragma unroll
        for (int q = 0; q < 3; q++) {
            float sum = 0.f;
#pragma unroll
            for (int l = 0; l < NM; l++) {
                float* r = a.r[q * 3 + l];
                const float v = a.ra[l] * r[cz] + a.rb[l] * (F[q] + dF[q]);
                r[cz] = v;
                sum += v;
            }
            sc[q][cz] = g1 * (g2 * sc[q][cz] + dt * (E[q] + dE[q] + sum));
        }
    }
}

template <int R, bool BORN, bool KEEP>
__global__ void k_born_velocity(BornArgs a, int it)
{
    int i, k;
    long long c, zo;
    if (!cell_of(a, i, k, c, zo)) return;
    const long long cz = c + zo;
    const float dt = a.dt;
    const float g1 = a.g1[c], g2 = a.g2[c], b = a.B[c];
    const float a0x = b * (dmx<R>(a.s0xx + zo, c, a) + dmz<R>(a.s0xz + zo, c, a));
    const float a0z = b * (dpx<R>(a.s0xz + zo, c, a) + dpz<R>(a.s0zz + zo, c, a));
    const float ov0x = a.v0x[cz], ov0z = a.v0z[cz];
    if (KEEP) {   // background history for the adjoint: v0 at the start of the step, a0
        a.kv0x[cz] = ov0x;
        a.kv0z[cz] = ov0z;
        a.ka0x[cz] = a0x;
        a.ka0z[cz] = a0z;
    }
    a.v0x[cz] = g1 * (g2 * ov0x + dt * a0x);
    a.v0z[cz] = g1 * (g2 * ov0z + dt * a0z);
    if (BORN) {
        const float ax = b * (dmx<R>(a.sxx + zo, c, a) + dmz<R>(a.sxz + zo, c, a));
        const float az = b * (dpx<R>(a.sxz + zo, c, a) + dpz<R>(a.szz + zo, c, a));
        const float r = a.rr[c];
        const float nvx = g1 * (g2 * a.vx[cz] + dt * (ax - r * a0x));
        const float nvz = g1 * (g2 * a.vz[cz] + dt * (az - r * a0z));
        a.vx[cz] = nvx;
        a.vz[cz] = nvz;
        const int rec = a.traces ? recv_of(a, i, k) : -1;
        if (rec >= 0) {
            const long long nrec = a.nrx, cs = (long long)a.nt * nrec;
            float* d = shot_traces(a) + (long long)it * nrec + rec;
            d[0] = nvx;
            d[cs] = 0.f;
            d[2 * cs] = nvz;
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
// k_adj_mem) gains the velocity update's stencil transposed; rho gradient from a0
template <int R>
__global__ void k_adj_vel(BornArgs a)
{
    int i, k;
    long long c, zo;
    if (!cell_of(a, i, k, c, zo)) return;
    const long long cz = c + zo;
    const float dt = a.dt;
    const float g1 = a.g1[c];
    // rho gradient: -dt g1 (vx^ a0x + vz^ a0z)
    a.gR[cz] += -dt * (g1 * a.ax[cz] * __ldg(a.ha0x + cz) + g1 * a.az[cz] * __ldg(a.ha0z + cz));
    // the shot's adjoint velocity through per-cell products B g1 a^ (shared B, g1)
    const Prod2 tx{a.B, a.g1, a.ax, zo}, tz{a.B, a.g1, a.az, zo};
    a.hxx[cz] = a.hxx[cz] - dt * tdpx<R>(tx, cz, a);
    a.hxz[cz] = a.hxz[cz] - dt * (tdpz<R>(tx, cz, a) + tdmx<R>(tz, cz, a));
    a.hzz[cz] = a.hzz[cz] - dt * tdmz<R>(tz, cz, a);
}

// stress and memory-variable update^T of one cell: Q = g1 h is the adjoint of
// the stress bracket, Lambda_l = lr_l + dt Q that of r_l', P = sum_l rb_l Lambda_l
// that of f; writes the strain adjoint S = iso(pi kp, mu ks; dt Q) + iso(pi tp,
// mu ts; P) (both maps are symmetric), carries lr_l = ra_l Lambda_l and h = g2 Q,
// and accumulates the pi and mu gradients from the background strain rates.
template <int R, int NM>
__global__ void k_adj_mem(BornArgs a)
{
    int i, k;
    long long c, zo;
    if (!cell_of(a, i, k, c, zo)) return;
    const long long cz = c + zo;
    const float dt = a.dt;
    const float g1 = a.g1[c], g2 = a.g2[c], pi = a.M[c], mu = a.U[c];
    const float Q[3] = {g1 * a.hxx[cz], g1 * a.hzz[cz], g1 * a.hxz[cz]};
    float P[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
        for (int l = 0; l < NM; l++) {
            float* lr = a.lr[q * 3 + l];
            const float lam = lr[cz] + dt * Q[q];
            P[q] += a.rb[l] * lam;
            lr[cz] = a.ra[l] * lam;
        }
    const float e0xx = dpx<R>(a.hv0x + zo, c, a), e0zz = dmz<R>(a.hv0z + zo, c, a);
    const float e0xz = dpz<R>(a.hv0x + zo, c, a) + dmx<R>(a.hv0z + zo, c, a);
    const float tq0 = dt * Q[0], tq1 = dt * Q[1], tq2 = dt * Q[2];
    a.gM[cz] += (a.kp * (tq0 + tq1) + a.tp * (P[0] + P[1])) * (e0xx + e0zz);
    a.gU[cz] += a.ks * (-2.f * tq0 * e0zz - 2.f * tq1 * e0xx + tq2 * e0xz) +
                a.ts * (-2.f * P[0] * e0zz - 2.f * P[1] * e0xx + P[2] * e0xz);
    float E[3], F[3] = {0.f, 0.f, 0.f};
    iso(pi * a.kp, mu * a.ks, tq0, tq1, tq2, E);
    if (NM) iso(pi * a.tp, mu * a.ts, P[0], P[1], P[2], F);
    a.Sxx[cz] = E[0] + F[0];
    a.Szz[cz] = E[1] + F[1];
    a.Sxz[cz] = E[2] + F[2];
    a.hxx[cz] = g2 * Q[0];
    a.hzz[cz] = g2 * Q[1];
    a.hxz[cz] = g2 * Q[2];
}

struct Load {
    const float* p;
    __device__ __forceinline__ float operator()(long long c) const { return p[c]; }
};

// velocity adjoint: a <- g2 g1 a (the velocity update^T) - D^T S (the stress
// update's stencils transposed), plus the next (earlier) step's residual
template <int R>
__global__ void k_adj_str(BornArgs a, int it_next)
{
    int i, k;
    long long c, zo;
    if (!cell_of(a, i, k, c, zo)) return;
    const long long cz = c + zo;
    const float g12 = a.g2[c] * a.g1[c];
    const Load sxx{a.Sxx}, szz{a.Szz}, sxz{a.Sxz};
    float nx = g12 * a.ax[cz] - (tdmx<R>(sxx, cz, a) + tdmz<R>(sxz, cz, a));
    float nz = g12 * a.az[cz] - (tdpz<R>(szz, cz, a) + tdpx<R>(sxz, cz, a));
    if (it_next >= 0) {
        const int rec = recv_of(a, i, k);
        if (rec >= 0) {
            const long long nrec = a.nrx, cs = (long long)a.nt * nrec;
            const float* d = shot_traces(a) + (long long)it_next * nrec + rec;
            nx += d[0];
            nz += d[2 * cs];
        }
    }
    a.ax[cz] = nx;
    a.az[cz] = nz;
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

// model products (copied from the context's padded model, plane j = 0) and damping
// factors on the compact layout
__global__ void k_born_model(BornArgs a, const float* Mc, const float* Uc, const float* Bc,
                             long long csz, const float* att_x, const float* att_z, float* M,
                             float* U, float* L, float* B, float* g1, float* g2)
{
    int i, k;
    long long c;
    long long zo;
    if (!cell_of(a, i, k, c, zo)) return;
    const long long m = (long long)k * csz + i;
    M[c] = Mc[m];
    U[c] = Uc[m];
    L[c] = M[c] - 2.f * U[c];
    B[c] = Bc[m];
    const float at = att_z[k] + att_x[i];
    const float h = at * a.dt * 0.5f;
    g1[c] = 1.f / (1.f + h);
    g2[c] = 1.f - h;
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

}  // namespace

cudaError_t born_launch_model(const BornArgs& a, const float* Mc, const float* Uc, const float* Bc,
                              long long csz, const float* att_x, const float* att_z, float* M,
                              float* U, float* L, float* B, float* g1, float* g2, cudaStream_t s)
{
    k_born_model<<<born_grid(a), dim3(32, 8), 0, s>>>(a, Mc, Uc, Bc, csz, att_x, att_z, M, U, L, B, g1,
                                                      g2);
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
void step_r(const BornArgs& a, int it, bool born, bool keep, cudaStream_t s)
{
    const dim3 g = born_grid(a, a.nshot), b(32, 8);
    if (born) k_born_stress<R, true, NM><<<g, b, 0, s>>>(a, it);
    else k_born_stress<R, false, NM><<<g, b, 0, s>>>(a, it);
    if (born) k_born_velocity<R, true, false><<<g, b, 0, s>>>(a, it);
    else if (keep) k_born_velocity<R, false, true><<<g, b, 0, s>>>(a, it);
    else k_born_velocity<R, false, false><<<g, b, 0, s>>>(a, it);
}
template <int R, int NM>
void adj_r(const BornArgs& a, int it, cudaStream_t s)
{
    const dim3 g = born_grid(a, a.nshot), b(32, 8);
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
