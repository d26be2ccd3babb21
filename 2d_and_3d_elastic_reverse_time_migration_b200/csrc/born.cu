// Born (linearised) modelling and its exact adjoint, 2D elastic, sponge boundaries.
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

// products of neighbours for the transposed stencils
struct Prod2 {   // f(c) = p(c) * q(c) * w(c)
    const float* p;
    const float* q;
    const float* w;
    __device__ __forceinline__ float operator()(long long c) const
    {
        return __ldg(p + c) * __ldg(q + c) * w[c];
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

__device__ __forceinline__ bool cell_of(const BornArgs& a, int& i, int& k, long long& c)
{
    i = blockIdx.x * blockDim.x + threadIdx.x;
    k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= a.nx || k >= a.nz) return false;
    c = (long long)(k + a.R) * a.px + i + BXH;
    return true;
}

__device__ __forceinline__ int recv_of(const BornArgs& a, int i, int k)
{
    if (k != a.rz) return -1;
    int d = i - a.rx0;
    if (d < 0 || d % a.drx) return -1;
    d /= a.drx;
    return d < a.nrx ? d : -1;
}

// ---- forward ---------------------------------------------------------------
template <int R, bool BORN>
__global__ void k_born_stress(BornArgs a, int it)
{
    int i, k;
    long long c;
    if (!cell_of(a, i, k, c)) return;
    const float dt = a.dt;
    const float g1 = a.g1[c], g2 = a.g2[c], M = a.M[c], L = a.L[c], U = a.U[c];
    const float e0xx = dpx<R>(a.v0x, c, a), e0zz = dmz<R>(a.v0z, c, a);
    const float e0xz = dpz<R>(a.v0x, c, a) + dmx<R>(a.v0z, c, a);
    float oxx = a.s0xx[c], ozz = a.s0zz[c];
    if (it < a.nw && i == a.ssx && k == a.ssz) {   // explosive source into the background
        const float w = __ldg(a.wavelet + it);
        oxx += w;
        ozz += w;
    }
    a.s0xx[c] = g1 * (g2 * oxx + dt * (M * e0xx + L * e0zz));
    a.s0zz[c] = g1 * (g2 * ozz + dt * (M * e0zz + L * e0xx));
    a.s0xz[c] = g1 * (g2 * a.s0xz[c] + dt * U * e0xz);
    if (BORN) {
        const float exx = dpx<R>(a.vx, c, a), ezz = dmz<R>(a.vz, c, a);
        const float exz = dpz<R>(a.vx, c, a) + dmx<R>(a.vz, c, a);
        const float dm = a.dM[c], du = a.dU[c], dl = dm - 2.f * du;
        a.sxx[c] = g1 * (g2 * a.sxx[c] + dt * (M * exx + L * ezz + dm * e0xx + dl * e0zz));
        a.szz[c] = g1 * (g2 * a.szz[c] + dt * (M * ezz + L * exx + dm * e0zz + dl * e0xx));
        a.sxz[c] = g1 * (g2 * a.sxz[c] + dt * (U * exz + du * e0xz));
    }
}

template <int R, bool BORN, bool KEEP>
__global__ void k_born_velocity(BornArgs a, int it)
{
    int i, k;
    long long c;
    if (!cell_of(a, i, k, c)) return;
    const float dt = a.dt;
    const float g1 = a.g1[c], g2 = a.g2[c], b = a.B[c];
    const float a0x = b * (dmx<R>(a.s0xx, c, a) + dmz<R>(a.s0xz, c, a));
    const float a0z = b * (dpx<R>(a.s0xz, c, a) + dpz<R>(a.s0zz, c, a));
    const float ov0x = a.v0x[c], ov0z = a.v0z[c];
    if (KEEP) {   // background history for the adjoint: v0 at the start of the step, a0
        a.kv0x[c] = ov0x;
        a.kv0z[c] = ov0z;
        a.ka0x[c] = a0x;
        a.ka0z[c] = a0z;
    }
    a.v0x[c] = g1 * (g2 * ov0x + dt * a0x);
    a.v0z[c] = g1 * (g2 * ov0z + dt * a0z);
    if (BORN) {
        const float ax = b * (dmx<R>(a.sxx, c, a) + dmz<R>(a.sxz, c, a));
        const float az = b * (dpx<R>(a.sxz, c, a) + dpz<R>(a.szz, c, a));
        const float r = a.rr[c];
        const float nvx = g1 * (g2 * a.vx[c] + dt * (ax - r * a0x));
        const float nvz = g1 * (g2 * a.vz[c] + dt * (az - r * a0z));
        a.vx[c] = nvx;
        a.vz[c] = nvz;
        const int rec = a.traces ? recv_of(a, i, k) : -1;
        if (rec >= 0) {
            const long long nrec = a.nrx, cs = (long long)a.nt * nrec;
            float* d = a.traces + (long long)it * nrec + rec;
            d[0] = nvx;
            d[cs] = 0.f;
            d[2 * cs] = nvz;
        }
    }
}

// ---- adjoint ---------------------------------------------------------------
__global__ void k_adj_inject(BornArgs a, int it)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nrx) return;
    const int i = a.rx0 + r * a.drx;
    if (i < 0 || i >= a.nx || a.rz < 0 || a.rz >= a.nz) return;
    const long long c = (long long)(a.rz + a.R) * a.px + i + BXH;
    const long long nrec = a.nrx, cs = (long long)a.nt * nrec;
    const float* d = a.traces + (long long)it * nrec + r;
    a.ax[c] += d[0];
    a.az[c] += d[2 * cs];
}

template <int R>
__global__ void k_adj_vel(BornArgs a)
{
    int i, k;
    long long c;
    if (!cell_of(a, i, k, c)) return;
    const float dt = a.dt;
    const float g1 = a.g1[c];
    // rho gradient: -dt g1 (vx^ a0x + vz^ a0z)
    a.gR[c] += -dt * (g1 * a.ax[c] * __ldg(a.ha0x + c) + g1 * a.az[c] * __ldg(a.ha0z + c));
    const Prod2 tx{a.B, a.g1, a.ax}, tz{a.B, a.g1, a.az};
    const float g12 = a.g2[c] * g1;
    a.hxx[c] = g12 * a.hxx[c] - dt * tdpx<R>(tx, c, a);
    a.hxz[c] = g12 * a.hxz[c] - dt * (tdpz<R>(tx, c, a) + tdmx<R>(tz, c, a));
    a.hzz[c] = g12 * a.hzz[c] - dt * tdmz<R>(tz, c, a);
}

template <int R>
__global__ void k_adj_str(BornArgs a, int it_next)
{
    int i, k;
    long long c;
    if (!cell_of(a, i, k, c)) return;
    const float dt = a.dt;
    const float g1 = a.g1[c];
    const float qxx = g1 * a.hxx[c], qzz = g1 * a.hzz[c], qxz = g1 * a.hxz[c];
    const float e0xx = dpx<R>(a.hv0x, c, a), e0zz = dmz<R>(a.hv0z, c, a);
    const float e0xz = dpz<R>(a.hv0x, c, a) + dmx<R>(a.hv0z, c, a);
    a.gM[c] += dt * (qxx * e0xx + qzz * e0zz);
    a.gL[c] += dt * (qxx * e0zz + qzz * e0xx);
    a.gU[c] += dt * qxz * e0xz;
    // neighbour products: M q_xx + L q_zz, L q_xx + M q_zz, U q_xz
    auto mx = [&](long long e) {
        const float ge = __ldg(a.g1 + e);
        return __ldg(a.M + e) * ge * a.hxx[e] + __ldg(a.L + e) * ge * a.hzz[e];
    };
    auto mz = [&](long long e) {
        const float ge = __ldg(a.g1 + e);
        return __ldg(a.L + e) * ge * a.hxx[e] + __ldg(a.M + e) * ge * a.hzz[e];
    };
    auto ux = [&](long long e) { return __ldg(a.U + e) * __ldg(a.g1 + e) * a.hxz[e]; };
    const float g12 = a.g2[c] * g1;
    float nx = g12 * a.ax[c] - dt * (tdmx<R>(mx, c, a) + tdmz<R>(ux, c, a));
    float nz = g12 * a.az[c] - dt * (tdpz<R>(mz, c, a) + tdpx<R>(ux, c, a));
    // residual of the next (earlier) step, injected at the receivers
    if (it_next >= 0) {
        const int rec = recv_of(a, i, k);
        if (rec >= 0) {
            const long long nrec = a.nrx, cs = (long long)a.nt * nrec;
            const float* d = a.traces + (long long)it_next * nrec + rec;
            nx += d[0];
            nz += d[2 * cs];
        }
    }
    a.ax[c] = nx;
    a.az[c] = nz;
}

// gradients w.r.t. (r_vp, r_vs, r_rho) on the contiguous nz x nx grid
__global__ void k_born_final(BornArgs a, float* gvp, float* gvs, float* grho)
{
    int i, k;
    long long c;
    if (!cell_of(a, i, k, c)) return;
    const long long m = (long long)k * a.nx + i;
    const float gm = a.gM[c] + a.gL[c], gu = a.gU[c] - 2.f * a.gL[c];
    gvp[m] = 2.f * a.M[c] * gm;
    gvs[m] = 2.f * a.U[c] * gu;
    grho[m] = a.M[c] * gm + a.U[c] * gu + a.gR[c];
}

// model products (copied from the context's padded model, plane j = 0) and damping
// factors on the compact layout
__global__ void k_born_model(BornArgs a, const float* Mc, const float* Uc, const float* Bc,
                             long long csz, const float* att_x, const float* att_z, float* M,
                             float* U, float* L, float* B, float* g1, float* g2)
{
    int i, k;
    long long c;
    if (!cell_of(a, i, k, c)) return;
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
    if (!cell_of(a, i, k, c)) return;
    const long long m = (long long)k * a.nx + i;
    dM[c] = a.M[c] * (rrho[m] + 2.f * rvp[m]);
    dU[c] = a.U[c] * (rrho[m] + 2.f * rvs[m]);
    rr[c] = rrho[m];
}

dim3 born_grid(const BornArgs& a) { return dim3((a.nx + 31) / 32, (a.nz + 7) / 8); }

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

cudaError_t born_launch_step(const BornArgs& a, int it, bool born, bool keep, cudaStream_t s)
{
    const dim3 g = born_grid(a), b(32, 8);
    if (a.R == 4) {
        if (born) k_born_stress<4, true><<<g, b, 0, s>>>(a, it);
        else k_born_stress<4, false><<<g, b, 0, s>>>(a, it);
        if (born) k_born_velocity<4, true, false><<<g, b, 0, s>>>(a, it);
        else if (keep) k_born_velocity<4, false, true><<<g, b, 0, s>>>(a, it);
        else k_born_velocity<4, false, false><<<g, b, 0, s>>>(a, it);
    } else {
        if (born) k_born_stress<6, true><<<g, b, 0, s>>>(a, it);
        else k_born_stress<6, false><<<g, b, 0, s>>>(a, it);
        if (born) k_born_velocity<6, true, false><<<g, b, 0, s>>>(a, it);
        else if (keep) k_born_velocity<6, false, true><<<g, b, 0, s>>>(a, it);
        else k_born_velocity<6, false, false><<<g, b, 0, s>>>(a, it);
    }
    return cudaGetLastError();
}

cudaError_t born_launch_adjoint_step(const BornArgs& a, int it, cudaStream_t s)
{
    const dim3 g = born_grid(a), b(32, 8);
    const int it_next = it - 1;
    if (a.R == 4) {
        k_adj_vel<4><<<g, b, 0, s>>>(a);
        k_adj_str<4><<<g, b, 0, s>>>(a, it_next);
    } else {
        k_adj_vel<6><<<g, b, 0, s>>>(a);
        k_adj_str<6><<<g, b, 0, s>>>(a, it_next);
    }
    return cudaGetLastError();
}

cudaError_t born_launch_inject(const BornArgs& a, int it, cudaStream_t s)
{
    if (a.nrx <= 0) return cudaSuccess;
    k_adj_inject<<<(a.nrx + 127) / 128, 128, 0, s>>>(a, it);
    return cudaGetLastError();
}

cudaError_t born_launch_final(const BornArgs& a, float* gvp, float* gvs, float* grho, cudaStream_t s)
{
    k_born_final<<<born_grid(a), dim3(32, 8), 0, s>>>(a, gvp, gvs, grho);
    return cudaGetLastError();
}

}  // namespace ertm
