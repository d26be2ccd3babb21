// Small kernels around the step kernels: layout conversion between the
// caller's contiguous volumes and the padded HBM layout, model preparation,
// receiver injection, the step counter, and the divergence/curl P/S split.
#include "ertm_internal.cuh"

namespace ertm {

namespace {

__global__ void k_scatter(Geom g, const float* __restrict__ src, float* __restrict__ dst)
{
    long long n = (long long)g.nx * g.ny * g.nz;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n;
         m += (long long)gridDim.x * blockDim.x) {
        int i = (int)(m % g.nx);
        long long t = m / g.nx;
        int j = (int)(t % g.ny);
        int k = (int)(t / g.ny);
        dst[k * g.sz + j * g.sy + i] = src[m];
    }
}

template <typename T>
__global__ void k_gather(Geom g, const T* __restrict__ src, T* __restrict__ dst)
{
    long long n = (long long)g.nx * g.ny * g.nz;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n;
         m += (long long)gridDim.x * blockDim.x) {
        int i = (int)(m % g.nx);
        long long t = m / g.nx;
        int j = (int)(t % g.ny);
        int k = (int)(t / g.ny);
        dst[m] = src[k * g.sz + j * g.sy + i];
    }
}

__global__ void k_sqrt_gather(Geom g, const float* __restrict__ src, float* __restrict__ dst)
{
    long long n = (long long)g.nx * g.ny * g.nz;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n;
         m += (long long)gridDim.x * blockDim.x) {
        int i = (int)(m % g.nx);
        long long t = m / g.nx;
        int j = (int)(t % g.ny);
        int k = (int)(t / g.ny);
        dst[m] = sqrtf(src[k * g.sz + j * g.sy + i]);
    }
}

// rho*vp^2, rho*vs^2, 1/rho from the caller's contiguous vp, vs, rho
__global__ void k_model(Geom g, const float* __restrict__ vp, const float* __restrict__ vs,
                        const float* __restrict__ rho, float* __restrict__ M,
                        float* __restrict__ MU, float* __restrict__ B)
{
    long long n = (long long)g.nx * g.ny * g.nz;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n;
         m += (long long)gridDim.x * blockDim.x) {
        int i = (int)(m % g.nx);
        long long t = m / g.nx;
        int j = (int)(t % g.ny);
        int k = (int)(t / g.ny);
        long long c = k * g.sz + j * g.sy + i;
        float r = rho[m], p = vp[m], s = vs[m];
        M[c] = r * p * p;
        MU[c] = r * s * s;
        B[c] = 1.f / r;
    }
}

// receiver injection of sample `it` (write_or_add_shot_3D_surface_three with
// add_receiver_bool, 3D_forward_or_back_together.cu:328)
__global__ void k_inject(KArgs a, int it)
{
    long long nrec = (long long)a.nrx * a.nry;
    long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= nrec) return;
    int ix = (int)(r % a.nrx), iy = (int)(r / a.nrx);
    int i = a.rx0 + ix * a.drx, j = a.ry0 + iy * a.dry;
    if (i < 0 || i >= a.nx || j < 0 || j >= a.ny || a.rz < 0 || a.rz >= a.nz) return;
    long long c = (long long)a.rz * a.sz + (long long)j * a.sy + i;
    const long long cs = (long long)a.nt * nrec;
    const float* d = a.traces + (long long)it * nrec + r;
    for (int q = 0; q < 3; q++) {
        if (q == 1 && a.f[F_VY] == nullptr) continue;
        float* f = a.f[F_VX + q];
        f[c] = (a.inject_mode == 2) ? d[q * cs] : f[c] + d[q * cs];
    }
}

__global__ void k_advance(int* it, int delta) { *it += delta; }

__global__ void k_axpy(long long n, const float* __restrict__ x, float* __restrict__ y)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        y[i] += x[i];
}
__global__ void k_set_int(int* p, int v) { *p = v; }

// P-wave propagation angle at the cells whose excitation time is the current step
// (caculate_ex_angle_pp_only_RTM / caculate_ex_angle_rp_only_RTM,
// 2D_elastic_RTM/elastic_2D_kernel_3.cu:132-284), from the Poynting vector of
// sum_poynting (elastic_2D_kernel_2.cu:28-30), p = -tp (vxp, vzp): over the
// (2 hw + 1)^2 cells around the cell (the reference's 5 x 5 source window, hw = 2,
// and 9 x 9 receiver window, hw = 4; cells outside the grid count as zero),
// sxz = sum px pz and szz = sum pz^2 (p in float, products and sums in double, as the
// reference: its Poynting arrays are float and it forms 1.0 * px * pz; a float product
// would underflow where the receiver wavefield is still only the stencil's numerical
// precursor), angle = atan(sxz / szz) in degrees from the z axis, rounded as the
// reference rounds it, written only where szz != 0.  Runs after the velocity kernel
// of the step and before the step counter advances.
__global__ void k_angle(Geom g, KArgs a, float* __restrict__ ang, int hw)
{
    const int it = *a.it_ptr;
    const float* tp = a.f[F_TP];
    const float* vxp = a.f[F_VXP];
    const float* vzp = a.f[F_VZP];
    const long long n = (long long)g.nx * g.nz;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n;
         m += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(m % g.nx), k = (int)(m / g.nx);
        const long long c = k * g.sz + i;
        if (a.ex_time[c] != it) continue;
        double sxz = 0.0, szz = 0.0;
        for (int dk = -hw; dk <= hw; dk++) {
            if (k + dk < 0 || k + dk >= g.nz) continue;
            for (int di = -hw; di <= hw; di++) {
                if (i + di < 0 || i + di >= g.nx) continue;
                const long long q = c + dk * g.sz + di;
                const float t = tp[q];
                const float px = -t * vxp[q], pz = -t * vzp[q];
                sxz += (double)px * (double)pz;
                szz += (double)pz * (double)pz;
            }
        }
        if (szz != 0.0) {
            // float(atan(sxz / szz)) * 180 / pai1 in float, pai1 = 3.1415926f
            // (elastic_2D_kernel_3.cu:4, :204)
            float d = (float)atan(sxz / szz);
            d = d * 180.0f;
            ang[c] = d / 3.1415926f;
        }
    }
}

template <int R>
__device__ __forceinline__ float dplus(const float* f, long long c, long long s, const float* cf)
{
    float acc = 0.f;
#pragma unroll
    for (int n = 1; n <= R; n++) acc = fmaf(cf[n], f[c + n * s] - f[c - (n - 1) * s], acc);
    return acc;
}

template <int R>
__device__ __forceinline__ float dminus(const float* f, long long c, long long s, const float* cf)
{
    float acc = 0.f;
#pragma unroll
    for (int n = 1; n <= R; n++) acc = fmaf(cf[n], f[c + (n - 1) * s] - f[c - n * s], acc);
    return acc;
}

// decom_new (2D_elastic_RTM/elastic_2D_kernel_2.cu:671-791) and its 3D extension.
// vp, vs are padded copies of the model velocities; outputs are contiguous.
template <int R>
__global__ void k_divcurl(Geom g, KArgs a, const float* __restrict__ vp,
                          const float* __restrict__ vs, float* __restrict__ p,
                          float* __restrict__ sx, float* __restrict__ sy, float* __restrict__ sz)
{
    long long n = (long long)g.nx * g.ny * g.nz;
    const float* X = a.f[F_VX];
    const float* Y = a.f[F_VY];
    const float* Z = a.f[F_VZ];
    const long long SY = g.sy, SZ = g.sz;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n;
         m += (long long)gridDim.x * blockDim.x) {
        int i = (int)(m % g.nx);
        long long t = m / g.nx;
        int j = (int)(t % g.ny);
        int k = (int)(t / g.ny);
        long long c = k * SZ + j * SY + i;
        float div = dplus<R>(X, c, 1, a.cx) + dminus<R>(Z, c, SZ, a.cz);
        if (!g.two_d) div += dplus<R>(Y, c, SY, a.cy);
        p[m] = vp[c] * div;
        float vxz = (vs[c] + vs[c + SZ] + vs[c + 1] + vs[c + 1 + SZ]) / 4.f;
        sy[m] = vxz * (dplus<R>(X, c, SZ, a.cz) - dminus<R>(Z, c, 1, a.cx));
        if (!g.two_d) {
            float vyz = (vs[c] + vs[c + SZ] + vs[c + SY] + vs[c + SY + SZ]) / 4.f;
            float vxy = (vs[c] + vs[c + 1] + vs[c + SY] + vs[c + 1 + SY]) / 4.f;
            sx[m] = vyz * (dminus<R>(Z, c, SY, a.cy) - dplus<R>(Y, c, SZ, a.cz));
            sz[m] = vxy * (dminus<R>(Y, c, 1, a.cx) - dminus<R>(X, c, SY, a.cy));
        }
    }
}

int grid_for(long long n)
{
    long long b = (n + 255) / 256;
    if (b > 148 * 32) b = 148 * 32;
    if (b < 1) b = 1;
    return (int)b;
}

}  // namespace

cudaError_t launch_scatter(const Geom& g, const float* src, float* dst, cudaStream_t s)
{
    k_scatter<<<grid_for((long long)g.nx * g.ny * g.nz), 256, 0, s>>>(g, src, dst);
    return cudaGetLastError();
}

cudaError_t launch_gather(const Geom& g, const float* src, float* dst, cudaStream_t s)
{
    k_gather<float><<<grid_for((long long)g.nx * g.ny * g.nz), 256, 0, s>>>(g, src, dst);
    return cudaGetLastError();
}

cudaError_t launch_gather_int(const Geom& g, const int* src, int* dst, cudaStream_t s)
{
    k_gather<int><<<grid_for((long long)g.nx * g.ny * g.nz), 256, 0, s>>>(g, src, dst);
    return cudaGetLastError();
}

cudaError_t launch_sqrt_gather(const Geom& g, const float* amp2, float* out, cudaStream_t s)
{
    k_sqrt_gather<<<grid_for((long long)g.nx * g.ny * g.nz), 256, 0, s>>>(g, amp2, out);
    return cudaGetLastError();
}

cudaError_t launch_model(const Geom& g, const float* vp, const float* vs, const float* rho,
                         float* M, float* MU, float* B, cudaStream_t s)
{
    k_model<<<grid_for((long long)g.nx * g.ny * g.nz), 256, 0, s>>>(g, vp, vs, rho, M, MU, B);
    return cudaGetLastError();
}

cudaError_t launch_inject(const KArgs& a, int it, cudaStream_t s)
{
    long long nrec = (long long)a.nrx * a.nry;
    if (nrec <= 0) return cudaSuccess;
    k_inject<<<(unsigned)((nrec + 255) / 256), 256, 0, s>>>(a, it);
    return cudaGetLastError();
}

cudaError_t launch_axpy(long long n, const float* x, float* y, cudaStream_t s)
{
    k_axpy<<<grid_for(n), 256, 0, s>>>(n, x, y);
    return cudaGetLastError();
}

cudaError_t launch_advance(int* it_ptr, int delta, cudaStream_t s)
{
    k_advance<<<1, 1, 0, s>>>(it_ptr, delta);
    return cudaGetLastError();
}

cudaError_t launch_set_int(int* p, int v, cudaStream_t s)
{
    k_set_int<<<1, 1, 0, s>>>(p, v);
    return cudaGetLastError();
}

cudaError_t launch_angle(const Geom& g, const KArgs& a, float* ang, int hw, cudaStream_t s)
{
    k_angle<<<grid_for((long long)g.nx * g.nz), 256, 0, s>>>(g, a, ang, hw);
    return cudaGetLastError();
}

cudaError_t launch_divcurl(int R, const Geom& g, const KArgs& a, const float* vp, const float* vs,
                           float* p, float* sx, float* sy, float* sz, cudaStream_t s)
{
    int nb = grid_for((long long)g.nx * g.ny * g.nz);
    if (R == 4) k_divcurl<4><<<nb, 256, 0, s>>>(g, a, vp, vs, p, sx, sy, sz);
    else k_divcurl<6><<<nb, 256, 0, s>>>(g, a, vp, vs, p, sx, sy, sz);
    return cudaGetLastError();
}

cudaError_t launch_stress(int R, const Geom& g, const KArgs& a, const StressMaps& m, bool cpml,
                          bool psplit, cudaStream_t s)
{
    return R == 4 ? launch_stress_r4(g, a, m, cpml, psplit, s)
                  : launch_stress_r6(g, a, m, cpml, psplit, s);
}

cudaError_t launch_velocity(int R, const Geom& g, const KArgs& a, const VelMaps& m, bool cpml,
                            int epi, bool record, cudaStream_t s)
{
    return R == 4 ? launch_velocity_r4(g, a, m, cpml, epi, record, s)
                  : launch_velocity_r6(g, a, m, cpml, epi, record, s);
}

cudaError_t launch_stress_multi(int R, dim3 grid, const StressMulti& P, bool cpml, cudaStream_t s)
{
    return R == 4 ? launch_stress_multi_r4(grid, P, cpml, s) : launch_stress_multi_r6(grid, P, cpml, s);
}

cudaError_t launch_velocity_multi(int R, dim3 grid, const VelMulti& P, bool cpml, int epi, cudaStream_t s)
{
    return R == 4 ? launch_velocity_multi_r4(grid, P, cpml, epi, s)
                  : launch_velocity_multi_r6(grid, P, cpml, epi, s);
}

}  // namespace ertm
