// Staggered-grid velocity–stress step kernels for sm_100a.
//
// One time step is two z-streaming kernels:
//   k_stress   : sigma(n+1) = f(sigma(n), v(n)) [+ P stress tp]      (+ source)
//   k_velocity : v(n+1) = f(v(n), sigma(n+1))   [+ P velocity v_P]   (+ epilogue)
// Each CTA owns a TX x TYB column of the x–y plane and a chunk of z planes:
// TYB consumer warps (one cell per thread) plus one producer warp.  One lane of
// the producer warp streams every input plane into a ring of shared-memory
// stages with TMA (cp.async.bulk.tensor, mbarrier completion, S planes ahead),
// refilling a stage as soon as every consumer warp has arrived on the stage's
// `empty` mbarrier.  There is no block-wide barrier in the z loop (warps drift
// apart by up to S-1 planes) and the issue cost stays off the consumers' path;
// C-PML memory variables, which live only in the absorbing slabs, come by
// 4-byte cp.async into a three-buffer ring, two planes ahead.
// Cell and slab offsets are 32-bit (a padded volume holds < 2^31 floats).
// The current plane of the fields that need x or y derivatives is staged in
// shared memory with an R-wide halo; the z derivatives come from a register
// queue of 2R+1 planes per field that slides down the column, so every
// value is read from HBM once per kernel (halo re-reads hit L2).
//
// Stencil operators (c_n already divided by the spacing):
//   D+ f[i] = sum_n c_n (f[i+n] - f[i-n+1])     (derivative at i+1/2)
//   D- f[i] = sum_n c_n (f[i+n-1] - f[i-n])     (derivative at i-1/2)
// Staggering (x and y like the reference's x, z like its z):
//   tii, tp at (i,j,k); vx (i-1/2,j,k); vy (i,j-1/2,k); vz (i,j,k+1/2);
//   txy (i-1/2,j-1/2,k); txz (i-1/2,j,k+1/2); tyz (i,j-1/2,k+1/2).
// The operator choice per derivative restates 2D_elastic_RTM/viscoelastic_equation.cu
// :137-176 (stress) and :1827-2122 (velocity); the update form
//   f(n+1) = g1 * (g2 * f(n) + dt * increment),  g1 = 1/(1+a dt/2), g2 = 1 - a dt/2
// is the reference's damped update (:151-180) with a = 0 (g1 = g2 = 1) under C-PML.
#pragma once

#include "ertm_internal.cuh"

namespace ertm {

__device__ __forceinline__ float cpml_upd(float* __restrict__ psi, long long p, float a, float b,
                                          float d)
{
    float v = fmaf(b, psi[p], a * d);
    psi[p] = v;
    return d + v;
}

template <bool Y>
__device__ __forceinline__ void damping(const KArgs& a, bool cpml, int i, int j, int k, float& g1,
                                        float& g2)
{
    if (cpml) {
        g1 = 1.f;
        g2 = 1.f;
    } else {
        // the reference accumulates the z, x, then y profiles (3D_zzzzz:302-356)
        float at = __ldg(a.att[2] + k) + __ldg(a.att[0] + i);
        if (Y) at = at + __ldg(a.att[1] + j);
        float h = at * a.dt * 0.5f;
        g1 = 1.f / (1.f + h);
        g2 = 1.f - h;
    }
}

__device__ __forceinline__ int receiver_index(const KArgs& a, int i, int j)
{
    int di = i - a.rx0, dj = j - a.ry0;
    if (di < 0 || dj < 0) return -1;
    if (di % a.drx || dj % a.dry) return -1;
    int ix = di / a.drx, iy = dj / a.dry;
    if (ix >= a.nrx || iy >= a.nry) return -1;
    return iy * a.nrx + ix;
}

// ---------------------------------------------------------------------------
// Asynchronous copy primitives
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// cp.async (global -> shared, 4 bytes) for the C-PML memory variables
__device__ __forceinline__ void cpa4(void* sdst, const void* gsrc)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(sdst)), "l"(gsrc)
                 : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cpa_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait on a stage: gives up after a fixed number of polls (each poll
// may suspend the thread for a while), so a lost copy cannot hang the GPU.
constexpr unsigned kWaitPolls = 1u << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity,
                                                  unsigned polls = kWaitPolls)
{
    for (unsigned n = 0; n < polls; n++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// the consumers' budget: the test hook's, else the default
__device__ __forceinline__ unsigned consumer_polls(const KArgs& a)
{
    return a.wait_polls ? a.wait_polls : kWaitPolls;
}
// the test hook's skipped copy: plane t of the first CTA of the grid
__device__ __forceinline__ bool skip_plane(const KArgs& a, int t)
{
    return a.skip_plane1 == t + 1 && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0;
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(smem_u32(bar))
                 : "memory");
}
// one plane of a 3D tiled tensor (coordinates in the padded volume)
__device__ __forceinline__ void tma3(float* dst, const CUtensorMap* map, int x, int y, int z,
                                     uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Box geometry of the staged tiles
template <int R, bool Y>
struct Boxes {
    static constexpr int TYB = Y ? TY3 : TY2;
    static constexpr int XB = xb_of(R);
    static constexpr int YB = Y ? R : 0;
    static constexpr int C = TX * TYB;                         // centre box
    static constexpr int XW = TX + 2 * XB;                      // x-halo box width
    static constexpr int X = XW * TYB;
    static constexpr int YH = TYB + 2 * YB;                     // y-halo box height
    static constexpr int Yb = TX * YH;
    static constexpr int XY = XW * YH;
    // shared-memory slot sizes: a TMA box must land on a 128-byte boundary, so
    // slots round up to 32 floats (a no-op for the 3D tiles; one-row 2D tiles
    // have 40- or 48-float halo boxes)
    static constexpr int XP = (X + 31) / 32 * 32;
    static constexpr int XYP = (XY + 31) / 32 * 32;
};

// Stage ring of NS stages: plane t goes to stage t % NS.  bars[s] ("full")
// completes when the TMA bytes of the stage's plane have landed; bars[NS + s]
// ("empty") when all TYB consumer warps have arrived after using the stage.

// Producer lane: issue planes 0 .. nk-1, refilling a stage as soon as its
// previous plane is released.  Every wait is bounded; before returning it
// waits (bounded) for the copies still in flight, so the block never exits
// with a TMA write into its shared memory pending.  False if a wait gave up.
// A consumer whose wait on a stage gives up stops at once without releasing
// that stage, so a stage is refilled only after every consumer saw its
// previous copy land: no copy is ever issued into a stage whose last copy is
// still pending.
template <int NS, class Issue>
__device__ __forceinline__ bool produce_planes(uint64_t* bars, int nk, unsigned polls, Issue issue)
{
    bool ok = true;
    int t = 0, skipped = -1;
    for (; t < nk; ++t) {
        if (t >= NS && !mbar_wait_bounded(&bars[NS + t % NS], ((t / NS) - 1) & 1, polls)) {
            ok = false;
            break;
        }
        if (!issue(t)) skipped = t;
    }
    // drain: every copy issued into the ring has landed before the block exits
    for (int u = (t > NS ? t - NS : 0); u < t; ++u)
        if (u != skipped && !mbar_wait_bounded(&bars[u % NS], (u / NS) & 1)) ok = false;
    return ok;
}

// ---------------------------------------------------------------------------
// Stress kernel
// ---------------------------------------------------------------------------
template <int R, bool Y, bool CPML, bool PS>
struct StressShape {
    using B = Boxes<R, Y>;
    static constexpr int NV = Y ? 3 : 2;                        // vx, vz, (vy)
    static constexpr int NSIG = Y ? 6 : 3;                      // txx tzz txz (tyy txy tyz)
    static constexpr int NC = NSIG + (PS ? 1 : 0) + 2;          // + tp + M + MU
    static constexpr int NP = CPML ? (Y ? 9 : 4) : 0;
    // stage: v tiles (XY), fronts (C), cells (C)
    static constexpr int OFF_FR = NV * B::XYP;
    static constexpr int OFF_C = OFF_FR + NV * B::C;
    static constexpr int STAGE = OFF_C + NC * B::C;             // floats
    static constexpr unsigned TX_BYTES = 4u * (NV * B::XY + NV * B::C + NC * B::C);   // box bytes
    static_assert(B::C % 32 == 0 && OFF_FR % 32 == 0 && OFF_C % 32 == 0 && STAGE % 32 == 0,
                  "TMA boxes must start on 128-byte boundaries");
    static constexpr int PSI = NP * B::C;                       // floats per psi buffer
    static constexpr int NS = 4;                                // ring stages
    static constexpr size_t BYTES = 4 * (size_t)(NS * STAGE + 3 * PSI) + 16 * NS;
};

// The stress step of one CTA: tile (blockIdx.x, blockIdx.y) of the x-y plane, z
// chunk bz of the grid described by `a`, whose TMA maps are `maps`.
template <int R, bool Y, bool CPML, bool PS>
__device__ __forceinline__ void stress_body(const StressMaps& maps, const KArgs& a, int bz)
{
    using SS = StressShape<R, Y, CPML, PS>;
    using B = typename SS::B;
    constexpr int NS = SS::NS;
    constexpr int TYB = B::TYB, XB = B::XB, XW = B::XW, CB = B::C;
    constexpr int NV = SS::NV, NSIG = SS::NSIG;
    constexpr int C_TP = NSIG, C_M = NSIG + (PS ? 1 : 0), C_MU = C_M + 1;
    extern __shared__ __align__(128) float sm[];
    float* psibuf = sm + NS * SS::STAGE;
    uint64_t* bars = reinterpret_cast<uint64_t*>(psibuf + 3 * SS::PSI);

    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool leader = (tx == 0 && ty == TYB);
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TYB;
    const int i = i0 + tx, j = j0 + ty;
    const int k0 = bz * a.kchunk;
    const int k1 = min(k0 + a.kchunk, a.nz);
    const int nk = k1 - k0;
    const int sy = (int)a.sy, sz = (int)a.sz;
    const bool act = (i < a.nx) && (j < a.ny);
    const int it = __ldg(a.it_ptr);
    const bool src_on = (it >= 0) && (it < a.nw);
    const bool src_here = src_on && (i == a.ssx) && (j == a.ssy);
    const float wsrc = src_on ? __ldg(a.wavelet + it) : 0.f;
    const int cell = ty * TX + tx;
    // padded-volume coordinates of the tile
    const int gx = i0 + XH, gy = j0 + (Y ? R : 0), gz0 = k0 + R;

    float* sig[6] = {a.f[F_TXX], a.f[F_TZZ], a.f[F_TXZ], a.f[F_TYY], a.f[F_TXY], a.f[F_TYZ]};
    float* tp = a.f[F_TP];
    const int cj = j * sy + i;

    auto issue = [&](int t) -> bool {   // leader only: all boxes of iteration t into stage t % S
        if (skip_plane(a, t)) return false;
        const int st = t % NS;
        float* S = sm + st * SS::STAGE;
        uint64_t* bar = &bars[st];
        const int z = gz0 + t;
        mbar_expect_tx(bar, SS::TX_BYTES);
#pragma unroll
        for (int f = 0; f < NV; f++) {
            tma3(S + f * B::XYP, &maps.v[f], gx - XB, gy - B::YB, z, bar);
            tma3(S + SS::OFF_FR + f * CB, &maps.vc[f], gx, gy, z + R, bar);
        }
#pragma unroll
        for (int q = 0; q < NSIG; q++) tma3(S + SS::OFF_C + q * CB, &maps.sig[q], gx, gy, z, bar);
        if (PS) tma3(S + SS::OFF_C + C_TP * CB, &maps.tp, gx, gy, z, bar);
        tma3(S + SS::OFF_C + C_M * CB, &maps.M, gx, gy, z, bar);
        tma3(S + SS::OFF_C + C_MU * CB, &maps.MU, gx, gy, z, bar);
        return true;
    };

    // C-PML: slab membership and profile coefficients of this column
    const int WX = a.w[0] + a.w[1], WY = a.w[2] + a.w[3];
    const bool inx = CPML && act && (i < a.w[0] || i >= a.nx - a.w[1]);
    const bool iny = CPML && Y && act && (j < a.w[2] || j >= a.ny - a.w[3]);
    const int slx = i < a.w[0] ? i : i - a.nx + WX;
    const int sly = j < a.w[2] ? j : j - a.ny + WY;
    float axf = 0.f, bxf = 1.f, axh = 0.f, bxh = 1.f, ayf = 0.f, byf = 1.f, ayh = 0.f, byh = 1.f;
    if (inx) {
        axf = __ldg(a.pa[0][0] + i); bxf = __ldg(a.pb[0][0] + i);
        axh = __ldg(a.pa[0][1] + i); bxh = __ldg(a.pb[0][1] + i);
    }
    if (iny) {
        ayf = __ldg(a.pa[1][0] + j); byf = __ldg(a.pb[1][0] + j);
        ayh = __ldg(a.pa[1][1] + j); byh = __ldg(a.pb[1][1] + j);
    }
    // psi slots: x: EXX DXVZ (DXVY), y: EYY DYVX DYVZ, z: EZZ DZVX (DZVY)
    constexpr int PX = 0, PY = Y ? 3 : 2, PZ = Y ? 6 : 2;
    auto issue_psi = [&](int p, int buf) {
        if (!CPML) return;
        float* Ps = psibuf + buf * SS::PSI;
        if (inx) {
            const int x = (p * a.ny + j) * WX + slx;
            cpa4(&Ps[(PX + 0) * CB + cell], a.psi[P_EXX] + x);
            cpa4(&Ps[(PX + 1) * CB + cell], a.psi[P_DXVZ] + x);
            if (Y) cpa4(&Ps[(PX + 2) * CB + cell], a.psi[P_DXVY] + x);
        }
        if (iny) {
            const int y = (p * WY + sly) * a.nx + i;
            cpa4(&Ps[(PY + 0) * CB + cell], a.psi[P_EYY] + y);
            cpa4(&Ps[(PY + 1) * CB + cell], a.psi[P_DYVX] + y);
            cpa4(&Ps[(PY + 2) * CB + cell], a.psi[P_DYVZ] + y);
        }
        if (act && (p < a.w[4] || p >= a.nz - a.w[5])) {
            const int sl = p < a.w[4] ? p : p - a.nz + a.w[4] + a.w[5];
            const int z = (sl * a.ny + j) * a.nx + i;
            cpa4(&Ps[(PZ + 0) * CB + cell], a.psi[P_EZZ] + z);
            cpa4(&Ps[(PZ + 1) * CB + cell], a.psi[P_DZVX] + z);
            if (Y) cpa4(&Ps[(PZ + 2) * CB + cell], a.psi[P_DZVY] + z);
        }
        cpa_commit();
    };

    if (leader) {
        for (int s = 0; s < NS; s++) {
            mbar_init(&bars[s], 1);
            mbar_init(&bars[NS + s], TYB);
        }
        mbar_fence_init();
    }
    __syncthreads();
    if (ty == TYB) {   // producer warp
        if (leader && !produce_planes<NS>(bars, nk, consumer_polls(a), issue) && a.err)
            atomicExch(a.err, DEV_WAIT_TIMEOUT);
        return;
    }

    // register queues of planes k-R .. k+R; the front (k+R) arrives with each stage
    const float* vsrc[3] = {a.f[F_VX], a.f[F_VZ], a.f[F_VY]};
    float qx[2 * R + 1], qy[2 * R + 1], qz[2 * R + 1];
#pragma unroll
    for (int q = 0; q < 2 * R; q++) {
        const int cc = (k0 + q - R) * sz + cj;
        qx[q] = vsrc[0][cc];
        qz[q] = vsrc[1][cc];
        if (Y) qy[q] = vsrc[2][cc];
    }
    issue_psi(k0, 0);
    if (nk > 1) issue_psi(k0 + 1, 1);
    else cpa_commit();
    cpa_wait_1();

    bool ok = true;
    const unsigned polls = consumer_polls(a);
    for (int t = 0; t < nk; ++t) {
        const int k = k0 + t;
        const int st = t % NS;
        if (!mbar_wait_bounded(&bars[st], (t / NS) & 1, polls)) {
            ok = false;          // stop here: the stage stays unreleased
            cpa_wait_all();
            break;
        }
        if (t + 2 < nk) issue_psi(k + 2, (t + 2) % 3);
        else cpa_commit();   // keep one group per iteration
        const float* S = sm + st * SS::STAGE;
        const float* Cc = S + SS::OFF_C;
        const float* Ps = psibuf + (t % 3) * SS::PSI;
        qx[2 * R] = S[SS::OFF_FR + 0 * CB + cell];
        qz[2 * R] = S[SS::OFF_FR + 1 * CB + cell];
        if (Y) qy[2 * R] = S[SS::OFF_FR + 2 * CB + cell];
        // tiles: (TX+2XB) wide, (TYB+2YB) high; the cell sits at row ty+YB, column tx+XB
        const float* Tx = S + 0 * B::XYP + (ty + B::YB) * XW + tx + XB;
        const float* Tz = S + 1 * B::XYP + (ty + B::YB) * XW + tx + XB;
        const float* Ty = S + 2 * B::XYP + (ty + B::YB) * XW + tx + XB;

        float exx = 0.f, dxvz = 0.f, dxvy = 0.f, eyy = 0.f, dyvx = 0.f, dyvz = 0.f;
        float ezz = 0.f, dzvx = 0.f, dzvy = 0.f;
#pragma unroll
        for (int n = 1; n <= R; n++) {
            exx = fmaf(a.cx[n], Tx[n] - Tx[1 - n], exx);
            dxvz = fmaf(a.cx[n], Tz[n - 1] - Tz[-n], dxvz);
            ezz = fmaf(a.cz[n], qz[R + n - 1] - qz[R - n], ezz);
            dzvx = fmaf(a.cz[n], qx[R + n] - qx[R - n + 1], dzvx);
            if (Y) {
                dxvy = fmaf(a.cx[n], Ty[n - 1] - Ty[-n], dxvy);
                eyy = fmaf(a.cy[n], Ty[n * XW] - Ty[(1 - n) * XW], eyy);
                dyvx = fmaf(a.cy[n], Tx[(n - 1) * XW] - Tx[-n * XW], dyvx);
                dyvz = fmaf(a.cy[n], Tz[(n - 1) * XW] - Tz[-n * XW], dyvz);
                dzvy = fmaf(a.cz[n], qy[R + n] - qy[R - n + 1], dzvy);
            }
        }

        if (act) {
            const int c = k * sz + cj;
            if (CPML) {
                if (inx) {
                    const int x = (k * a.ny + j) * WX + slx;
                    float p0 = fmaf(bxf, Ps[(PX + 0) * CB + cell], axf * exx);
                    float p1 = fmaf(bxh, Ps[(PX + 1) * CB + cell], axh * dxvz);
                    a.psi[P_EXX][x] = p0;
                    a.psi[P_DXVZ][x] = p1;
                    exx += p0;
                    dxvz += p1;
                    if (Y) {
                        float p2 = fmaf(bxh, Ps[(PX + 2) * CB + cell], axh * dxvy);
                        a.psi[P_DXVY][x] = p2;
                        dxvy += p2;
                    }
                }
                if (iny) {
                    const int y = (k * WY + sly) * a.nx + i;
                    float p0 = fmaf(byf, Ps[(PY + 0) * CB + cell], ayf * eyy);
                    float p1 = fmaf(byh, Ps[(PY + 1) * CB + cell], ayh * dyvx);
                    float p2 = fmaf(byh, Ps[(PY + 2) * CB + cell], ayh * dyvz);
                    a.psi[P_EYY][y] = p0;
                    a.psi[P_DYVX][y] = p1;
                    a.psi[P_DYVZ][y] = p2;
                    eyy += p0;
                    dyvx += p1;
                    dyvz += p2;
                }
                if (k < a.w[4] || k >= a.nz - a.w[5]) {
                    const int sl = k < a.w[4] ? k : k - a.nz + a.w[4] + a.w[5];
                    const int z = (sl * a.ny + j) * a.nx + i;
                    const float azf = __ldg(a.pa[2][0] + k), bzf = __ldg(a.pb[2][0] + k);
                    const float azh = __ldg(a.pa[2][1] + k), bzh = __ldg(a.pb[2][1] + k);
                    float p0 = fmaf(bzf, Ps[(PZ + 0) * CB + cell], azf * ezz);
                    float p1 = fmaf(bzh, Ps[(PZ + 1) * CB + cell], azh * dzvx);
                    a.psi[P_EZZ][z] = p0;
                    a.psi[P_DZVX][z] = p1;
                    ezz += p0;
                    dzvx += p1;
                    if (Y) {
                        float p2 = fmaf(bzh, Ps[(PZ + 2) * CB + cell], azh * dzvy);
                        a.psi[P_DZVY][z] = p2;
                        dzvy += p2;
                    }
                }
            }
            float g1, g2;
            damping<Y>(a, CPML, i, j, k, g1, g2);
            const float M = Cc[C_M * CB + cell], U = Cc[C_MU * CB + cell];
            const float L = M - 2.f * U;
            const float dt = a.dt;
            float oxx = Cc[0 * CB + cell], ozz = Cc[1 * CB + cell], oxz = Cc[2 * CB + cell];
            float oyy = 0.f, oxy = 0.f, oyz = 0.f;
            if (Y) {
                oyy = Cc[3 * CB + cell];
                oxy = Cc[4 * CB + cell];
                oyz = Cc[5 * CB + cell];
            }
            if (src_here && k == a.ssz) {     // add_source_3D into txx, tyy, tzz
                oxx += wsrc;
                ozz += wsrc;
                if (Y) oyy += wsrc;
            }
            if (ok) {
                sig[0][c] = g1 * (g2 * oxx + dt * (M * exx + L * (eyy + ezz)));
                sig[1][c] = g1 * (g2 * ozz + dt * (M * ezz + L * (exx + eyy)));
                sig[2][c] = g1 * (g2 * oxz + dt * U * (dzvx + dxvz));
                if (Y) {
                    sig[3][c] = g1 * (g2 * oyy + dt * (M * eyy + L * (exx + ezz)));
                    sig[4][c] = g1 * (g2 * oxy + dt * U * (dyvx + dxvy));
                    sig[5][c] = g1 * (g2 * oyz + dt * U * (dzvy + dyvz));
                }
                if (PS) tp[c] = g1 * (g2 * Cc[C_TP * CB + cell] + dt * M * (exx + eyy + ezz));
            }
        }

#pragma unroll
        for (int q = 0; q < 2 * R; q++) {
            qx[q] = qx[q + 1];
            qz[q] = qz[q + 1];
            if (Y) qy[q] = qy[q + 1];
        }
        cpa_wait_1();   // plane t+1's memory variables have landed
        __syncwarp();
        if (tx == 0) mbar_arrive(&bars[NS + st]);   // release the stage
    }
    if (!ok && a.err) atomicExch(a.err, DEV_WAIT_TIMEOUT);
}

// ---------------------------------------------------------------------------
// Velocity kernel
// ---------------------------------------------------------------------------
template <int R, bool Y, bool CPML, int EPI>
struct VelShape {
    using B = Boxes<R, Y>;
    static constexpr bool PS = (EPI != EPI_NONE);
    // tiles: txx (X), txz (X), txy (XY), tyy (Y), tyz (Y), tp (XY; X in 2D)
    static constexpr int O_TXX = 0;
    static constexpr int O_TXZ = O_TXX + B::XP;
    static constexpr int O_TXY = O_TXZ + B::XP;
    static constexpr int O_TYY = O_TXY + (Y ? B::XYP : 0);
    static constexpr int O_TYZ = O_TYY + (Y ? B::Yb : 0);
    static constexpr int O_TP = O_TYZ + (Y ? B::Yb : 0);
    static constexpr int O_FR = O_TP + (PS ? B::XYP : 0);
    // fronts: txz, tzz, (tyz), (tp)
    static constexpr int NFR = 2 + (Y ? 1 : 0) + (PS ? 1 : 0);
    static constexpr int FR_TYZ = 2, FR_TP = Y ? 3 : 2;
    // cells: vx, vz, (vy), (vxp, vzp, (vyp)), b, (excitation)
    static constexpr int C_VX = 0, C_VZ = 1, C_VY = 2;
    static constexpr int C_PX = Y ? 3 : 2;
    static constexpr int C_PZ = C_PX + 1, C_PY = C_PX + 2;
    static constexpr int C_B = PS ? C_PX + (Y ? 3 : 2) : C_PX;
    static constexpr int C_EX = C_B + 1;
    static constexpr int NC = C_B + 1 + (PS ? 1 : 0);
    static constexpr int O_C = O_FR + NFR * B::C;
    static constexpr int STAGE = O_C + NC * B::C;
    static constexpr unsigned TX_BYTES =    // box bytes (slots may be padded)
        4u * (2 * B::X + (Y ? B::XY + 2 * B::Yb : 0) + (PS ? B::XY : 0) + NFR * B::C + NC * B::C);
    static_assert(B::C % 32 == 0 && O_TXZ % 32 == 0 && O_TXY % 32 == 0 && O_TYY % 32 == 0 &&
                      O_TYZ % 32 == 0 && O_TP % 32 == 0 && O_FR % 32 == 0 && O_C % 32 == 0 &&
                      STAGE % 32 == 0,
                  "TMA boxes must start on 128-byte boundaries");
    static constexpr int NP = CPML ? (Y ? 9 : 4) : 0;
    static constexpr int PSI = NP * B::C;
    static constexpr int NS = 3;   // ring stages (4 would not leave room for 2 CTAs per SM)
    static constexpr size_t BYTES = 4 * (size_t)(NS * STAGE + 3 * PSI) + 16 * NS;
};

// The velocity step of one CTA (tile and chunk as in stress_body).
template <int R, bool Y, bool CPML, int EPI, bool REC>
__device__ __forceinline__ void velocity_body(const VelMaps& maps, const KArgs& a, int bz)
{
    using VS = VelShape<R, Y, CPML, EPI>;
    using B = typename VS::B;
    constexpr int NS = VS::NS;
    constexpr bool PS = VS::PS;
    constexpr int TYB = B::TYB, XB = B::XB, XW = B::XW, CB = B::C;
    extern __shared__ __align__(128) float sm[];
    float* psibuf = sm + NS * VS::STAGE;
    uint64_t* bars = reinterpret_cast<uint64_t*>(psibuf + 3 * VS::PSI);

    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool leader = (tx == 0 && ty == TYB);
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TYB;
    const int i = i0 + tx, j = j0 + ty;
    const int k0 = bz * a.kchunk;
    const int k1 = min(k0 + a.kchunk, a.nz);
    const int nk = k1 - k0;
    const int sy = (int)a.sy, sz = (int)a.sz;
    const bool act = (i < a.nx) && (j < a.ny);
    const int it = __ldg(a.it_ptr);
    const int rec = ((REC || EPI == EPI_IMAGE) && act) ? receiver_index(a, i, j) : -1;
    const long long nrec = (long long)a.nrx * a.nry;
    const int cell = ty * TX + tx;
    const int gx = i0 + XH, gy = j0 + (Y ? R : 0), gz0 = k0 + R;
    const int cj = j * sy + i;

    float* vx = a.f[F_VX];
    float* vy = a.f[F_VY];
    float* vz = a.f[F_VZ];
    float* vxp = a.f[F_VXP];
    float* vyp = a.f[F_VYP];
    float* vzp = a.f[F_VZP];

    auto issue = [&](int t) -> bool {
        if (skip_plane(a, t)) return false;
        const int st = t % NS;
        float* S = sm + st * VS::STAGE;
        uint64_t* bar = &bars[st];
        const int z = gz0 + t;
        mbar_expect_tx(bar, VS::TX_BYTES);
        tma3(S + VS::O_TXX, &maps.txx, gx - XB, gy, z, bar);
        tma3(S + VS::O_TXZ, &maps.txz, gx - XB, gy, z, bar);
        if (Y) {
            tma3(S + VS::O_TXY, &maps.txy, gx - XB, gy - R, z, bar);
            tma3(S + VS::O_TYY, &maps.tyy, gx, gy - R, z, bar);
            tma3(S + VS::O_TYZ, &maps.tyz, gx, gy - R, z, bar);
        }
        if (PS) tma3(S + VS::O_TP, &maps.tp, gx - XB, gy - B::YB, z, bar);
#pragma unroll
        for (int f = 0; f < VS::NFR; f++) tma3(S + VS::O_FR + f * CB, &maps.fr[f], gx, gy, z + R, bar);
#pragma unroll
        for (int q = 0; q < VS::NC; q++) tma3(S + VS::O_C + q * CB, &maps.c[q], gx, gy, z, bar);
        return true;
    };

    const int WX = a.w[0] + a.w[1], WY = a.w[2] + a.w[3];
    const bool inx = CPML && act && (i < a.w[0] || i >= a.nx - a.w[1]);
    const bool iny = CPML && Y && act && (j < a.w[2] || j >= a.ny - a.w[3]);
    const int slx = i < a.w[0] ? i : i - a.nx + WX;
    const int sly = j < a.w[2] ? j : j - a.ny + WY;
    float axf = 0.f, bxf = 1.f, axh = 0.f, bxh = 1.f, ayf = 0.f, byf = 1.f, ayh = 0.f, byh = 1.f;
    if (inx) {
        axf = __ldg(a.pa[0][0] + i); bxf = __ldg(a.pb[0][0] + i);
        axh = __ldg(a.pa[0][1] + i); bxh = __ldg(a.pb[0][1] + i);
    }
    if (iny) {
        ayf = __ldg(a.pa[1][0] + j); byf = __ldg(a.pb[1][0] + j);
        ayh = __ldg(a.pa[1][1] + j); byh = __ldg(a.pb[1][1] + j);
    }
    // psi slots: x: DXTXX DXTXZ (DXTXY), y: DYTXY DYTYY DYTYZ, z: DZTXZ DZTZZ (DZTYZ)
    constexpr int PX = 0, PY = Y ? 3 : 2, PZ = Y ? 6 : 2;
    auto issue_psi = [&](int p, int buf) {
        if (!CPML) return;
        float* Ps = psibuf + buf * VS::PSI;
        if (inx) {
            const int x = (p * a.ny + j) * WX + slx;
            cpa4(&Ps[(PX + 0) * CB + cell], a.psi[P_DXTXX] + x);
            cpa4(&Ps[(PX + 1) * CB + cell], a.psi[P_DXTXZ] + x);
            if (Y) cpa4(&Ps[(PX + 2) * CB + cell], a.psi[P_DXTXY] + x);
        }
        if (iny) {
            const int y = (p * WY + sly) * a.nx + i;
            cpa4(&Ps[(PY + 0) * CB + cell], a.psi[P_DYTXY] + y);
            cpa4(&Ps[(PY + 1) * CB + cell], a.psi[P_DYTYY] + y);
            cpa4(&Ps[(PY + 2) * CB + cell], a.psi[P_DYTYZ] + y);
        }
        if (act && (p < a.w[4] || p >= a.nz - a.w[5])) {
            const int sl = p < a.w[4] ? p : p - a.nz + a.w[4] + a.w[5];
            const int z = (sl * a.ny + j) * a.nx + i;
            cpa4(&Ps[(PZ + 0) * CB + cell], a.psi[P_DZTXZ] + z);
            cpa4(&Ps[(PZ + 1) * CB + cell], a.psi[P_DZTZZ] + z);
            if (Y) cpa4(&Ps[(PZ + 2) * CB + cell], a.psi[P_DZTYZ] + z);
        }
        cpa_commit();
    };

    if (leader) {
        for (int s = 0; s < NS; s++) {
            mbar_init(&bars[s], 1);
            mbar_init(&bars[NS + s], TYB);
        }
        mbar_fence_init();
    }
    __syncthreads();
    if (ty == TYB) {   // producer warp
        if (leader && !produce_planes<NS>(bars, nk, consumer_polls(a), issue) && a.err)
            atomicExch(a.err, DEV_WAIT_TIMEOUT);
        return;
    }

    const float* txz = a.f[F_TXZ];
    const float* tyz = a.f[F_TYZ];
    const float* tzz = a.f[F_TZZ];
    const float* tp = a.f[F_TP];
    float qxz[2 * R + 1], qyz[2 * R + 1], qzz[2 * R + 1], qtp[2 * R + 1];
#pragma unroll
    for (int q = 0; q < 2 * R; q++) {
        const int cc = (k0 + q - R) * sz + cj;
        qxz[q] = txz[cc];
        qzz[q] = tzz[cc];
        if (Y) qyz[q] = tyz[cc];
        if (PS) qtp[q] = tp[cc];
    }
    issue_psi(k0, 0);
    if (nk > 1) issue_psi(k0 + 1, 1);
    else cpa_commit();
    cpa_wait_1();

    bool ok = true;
    const unsigned polls = consumer_polls(a);
    for (int t = 0; t < nk; ++t) {
        const int k = k0 + t;
        const int st = t % NS;
        if (!mbar_wait_bounded(&bars[st], (t / NS) & 1, polls)) {
            ok = false;          // stop here: the stage stays unreleased
            cpa_wait_all();
            break;
        }
        if (t + 2 < nk) issue_psi(k + 2, (t + 2) % 3);
        else cpa_commit();   // keep one group per iteration
        const float* S = sm + st * VS::STAGE;
        const float* Cc = S + VS::O_C;
        const float* Ps = psibuf + (t % 3) * VS::PSI;
        qxz[2 * R] = S[VS::O_FR + 0 * CB + cell];
        qzz[2 * R] = S[VS::O_FR + 1 * CB + cell];
        if (Y) qyz[2 * R] = S[VS::O_FR + VS::FR_TYZ * CB + cell];
        if (PS) qtp[2 * R] = S[VS::O_FR + VS::FR_TP * CB + cell];
        const float* Txx = S + VS::O_TXX + ty * XW + tx + XB;
        const float* Txz = S + VS::O_TXZ + ty * XW + tx + XB;
        const float* Txy = S + VS::O_TXY + (ty + R) * XW + tx + XB;
        const float* Tyy = S + VS::O_TYY + (ty + R) * TX + tx;
        const float* Tyz = S + VS::O_TYZ + (ty + R) * TX + tx;
        const float* Ttp = S + VS::O_TP + (ty + B::YB) * XW + tx + XB;

        float dxtxx = 0.f, dytxy = 0.f, dztxz = 0.f;
        float dxtxy = 0.f, dytyy = 0.f, dztyz = 0.f;
        float dxtxz = 0.f, dytyz = 0.f, dztzz = 0.f;
        float dxtp = 0.f, dytp = 0.f, dztp = 0.f;
#pragma unroll
        for (int n = 1; n <= R; n++) {
            dxtxx = fmaf(a.cx[n], Txx[n - 1] - Txx[-n], dxtxx);
            dxtxz = fmaf(a.cx[n], Txz[n] - Txz[1 - n], dxtxz);
            dztxz = fmaf(a.cz[n], qxz[R + n - 1] - qxz[R - n], dztxz);
            dztzz = fmaf(a.cz[n], qzz[R + n] - qzz[R - n + 1], dztzz);
            if (Y) {
                dytxy = fmaf(a.cy[n], Txy[n * XW] - Txy[(1 - n) * XW], dytxy);
                dxtxy = fmaf(a.cx[n], Txy[n] - Txy[1 - n], dxtxy);
                dytyy = fmaf(a.cy[n], Tyy[(n - 1) * TX] - Tyy[-n * TX], dytyy);
                dztyz = fmaf(a.cz[n], qyz[R + n - 1] - qyz[R - n], dztyz);
                dytyz = fmaf(a.cy[n], Tyz[n * TX] - Tyz[(1 - n) * TX], dytyz);
            }
            if (PS) {
                dxtp = fmaf(a.cx[n], Ttp[n - 1] - Ttp[-n], dxtp);
                dztp = fmaf(a.cz[n], qtp[R + n] - qtp[R - n + 1], dztp);
                if (Y) dytp = fmaf(a.cy[n], Ttp[(n - 1) * XW] - Ttp[-n * XW], dytp);
            }
        }

        if (act) {
            const int c = k * sz + cj;
            if (CPML) {
                if (inx) {
                    const int x = (k * a.ny + j) * WX + slx;
                    float p0 = fmaf(bxh, Ps[(PX + 0) * CB + cell], axh * dxtxx);
                    float p1 = fmaf(bxf, Ps[(PX + 1) * CB + cell], axf * dxtxz);
                    a.psi[P_DXTXX][x] = p0;
                    a.psi[P_DXTXZ][x] = p1;
                    dxtxx += p0;
                    dxtxz += p1;
                    if (Y) {
                        float p2 = fmaf(bxf, Ps[(PX + 2) * CB + cell], axf * dxtxy);
                        a.psi[P_DXTXY][x] = p2;
                        dxtxy += p2;
                    }
                }
                if (iny) {
                    const int y = (k * WY + sly) * a.nx + i;
                    float p0 = fmaf(byf, Ps[(PY + 0) * CB + cell], ayf * dytxy);
                    float p1 = fmaf(byh, Ps[(PY + 1) * CB + cell], ayh * dytyy);
                    float p2 = fmaf(byf, Ps[(PY + 2) * CB + cell], ayf * dytyz);
                    a.psi[P_DYTXY][y] = p0;
                    a.psi[P_DYTYY][y] = p1;
                    a.psi[P_DYTYZ][y] = p2;
                    dytxy += p0;
                    dytyy += p1;
                    dytyz += p2;
                }
                if (k < a.w[4] || k >= a.nz - a.w[5]) {
                    const int sl = k < a.w[4] ? k : k - a.nz + a.w[4] + a.w[5];
                    const int z = (sl * a.ny + j) * a.nx + i;
                    const float azf = __ldg(a.pa[2][0] + k), bzf = __ldg(a.pb[2][0] + k);
                    const float azh = __ldg(a.pa[2][1] + k), bzh = __ldg(a.pb[2][1] + k);
                    float p0 = fmaf(bzf, Ps[(PZ + 0) * CB + cell], azf * dztxz);
                    float p1 = fmaf(bzh, Ps[(PZ + 1) * CB + cell], azh * dztzz);
                    a.psi[P_DZTXZ][z] = p0;
                    a.psi[P_DZTZZ][z] = p1;
                    dztxz += p0;
                    dztzz += p1;
                    if (Y) {
                        float p2 = fmaf(bzf, Ps[(PZ + 2) * CB + cell], azf * dztyz);
                        a.psi[P_DZTYZ][z] = p2;
                        dztyz += p2;
                    }
                }
            }
            float g1, g2;
            damping<Y>(a, CPML, i, j, k, g1, g2);
            const float b = Cc[VS::C_B * CB + cell];
            const float db = a.dt * b;
            float nvx = g1 * (g2 * Cc[VS::C_VX * CB + cell] + db * (dxtxx + dytxy + dztxz));
            float nvz = g1 * (g2 * Cc[VS::C_VZ * CB + cell] + db * (dxtxz + dytyz + dztzz));
            float nvy = 0.f;
            if (Y) nvy = g1 * (g2 * Cc[VS::C_VY * CB + cell] + db * (dxtxy + dytyy + dztyz));
            float npx = 0.f, npy = 0.f, npz = 0.f;
            if (PS) {
                // decoupled P velocity from the P-stress gradient (role of fwd_vxp_vzp_3D,
                // 3D_forward_or_back_together.cu:118); S velocity = v - v_P
                npx = g1 * (g2 * Cc[VS::C_PX * CB + cell] + db * dxtp);
                npz = g1 * (g2 * Cc[VS::C_PZ * CB + cell] + db * dztp);
                if (Y) npy = g1 * (g2 * Cc[VS::C_PY * CB + cell] + db * dytp);
                if (ok) {
                    vxp[c] = npx;
                    vzp[c] = npz;
                    if (Y) vyp[c] = npy;
                }
            }
            if (EPI == EPI_EXCITE && ok) {
                // caculate_ex_amp_time_new (2D_elastic_RTM/elastic_2D_kernel_3.cu:30-48):
                // strict '>' keeps the earliest maximum of |v_P|
                float a2 = npx * npx + npy * npy + npz * npz;
                if (a2 > Cc[VS::C_EX * CB + cell]) {
                    a.ex_amp2[c] = a2;
                    a.ex_time[c] = it;
                    a.ex_v[0][c] = npx;
                    if (Y) a.ex_v[1][c] = npy;
                    a.ex_v[2][c] = npz;
                    a.ex_tp[c] = qtp[R];
                }
            }
            if (EPI == EPI_IMAGE && ok) {
                // imaging_inner_product_ex / imaging_correlation_ex
                // (2D_elastic_RTM/elastic_2D_kernel_3.cu:542-576) at it == excitation time
                if (__float_as_int(Cc[VS::C_EX * CB + cell]) == it) {
                    float ex = a.ex_v[0][c], ey = Y ? a.ex_v[1][c] : 0.f, ez = a.ex_v[2][c];
                    float den = ex * ex + ey * ey + ez * ez;
                    if (den > 0.f) {   // a true division: 1/den overflows for denormal den
                        if (a.img[0]) a.img[0][c] = (ex * npx + ey * npy + ez * npz) / den;
                        if (a.img[1])
                            a.img[1][c] = (ex * (nvx - npx) + ey * (nvy - npy) + ez * (nvz - npz)) / den;
                    }
                    float et = a.ex_tp[c];
                    if (a.img[2] && et != 0.f) a.img[2][c] = qtp[R] / et;
                }
                // receiver injection of the next (earlier) sample, reference :328
                if (rec >= 0 && k == a.rz && it > 0) {
                    const float* d = a.traces + (long long)(it - 1) * nrec + rec;
                    const long long cs = (long long)a.nt * nrec;
                    if (a.inject_mode == 2) {
                        nvx = d[0];
                        nvz = d[2 * cs];
                        if (Y) nvy = d[cs];
                    } else {
                        nvx += d[0];
                        nvz += d[2 * cs];
                        if (Y) nvy += d[cs];
                    }
                }
            }
            if (ok) {
                vx[c] = nvx;
                vz[c] = nvz;
                if (Y) vy[c] = nvy;
            }
            if (REC && ok && rec >= 0 && k == a.rz) {
                // write_or_add_shot_3D_surface_three, record flag 0 (:127)
                float* d = a.traces + (long long)it * nrec + rec;
                const long long cs = (long long)a.nt * nrec;
                d[0] = nvx;
                d[cs] = nvy;
                d[2 * cs] = nvz;
            }
        }

#pragma unroll
        for (int q = 0; q < 2 * R; q++) {
            qxz[q] = qxz[q + 1];
            qzz[q] = qzz[q + 1];
            if (Y) qyz[q] = qyz[q + 1];
            if (PS) qtp[q] = qtp[q + 1];
        }
        cpa_wait_1();   // plane t+1's memory variables have landed
        __syncwarp();
        if (tx == 0) mbar_arrive(&bars[NS + st]);   // release the stage
    }
    if (!ok && a.err) atomicExch(a.err, DEV_WAIT_TIMEOUT);
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
template <int R, bool Y, bool CPML, bool PS>
__global__ void __launch_bounds__(TX * ((Y ? TY3 : TY2) + 1), Y ? CTAS3 : 1)
k_stress(const __grid_constant__ StressMaps maps, const __grid_constant__ KArgs a)
{
    stress_body<R, Y, CPML, PS>(maps, a, blockIdx.z);
}

template <int R, bool Y, bool CPML, int EPI, bool REC>
__global__ void __launch_bounds__(TX * ((Y ? TY3 : TY2) + 1), Y ? CTAS3 : 1)
k_velocity(const __grid_constant__ VelMaps maps, const __grid_constant__ KArgs a)
{
    velocity_body<R, Y, CPML, EPI, REC>(maps, a, blockIdx.z);
}

// Several 3D shots in one launch (the RTM passes: P/S split on, excitation or
// imaging epilogue).  Every shot has its own context-sized volumes, argument
// block and TMA maps, all in the parameter block (StressMulti / VelMulti);
// blockIdx.z covers the `chunks` z chunks of every shot in turn.  A CTA whose tile lies outside its
// shot's grid, or whose shot is idle at this step (step index >= it_hi: a shot
// with fewer steps than the launch), returns before touching anything.
template <int R, bool CPML>
__global__ void __launch_bounds__(TX * (TY3 + 1), CTAS3) k_stress_multi(const __grid_constant__ StressMulti P)
{
    const int shot = blockIdx.z / P.chunks;
    const KArgs& a = P.a[shot];
    if ((int)blockIdx.x * TX >= a.nx || (int)blockIdx.y * TY3 >= a.ny || __ldg(a.it_ptr) >= a.it_hi) return;
    stress_body<R, true, CPML, true>(P.m[shot], a, blockIdx.z - shot * P.chunks);
}

template <int R, bool CPML, int EPI>
__global__ void __launch_bounds__(TX * (TY3 + 1), CTAS3) k_velocity_multi(const __grid_constant__ VelMulti P)
{
    const int shot = blockIdx.z / P.chunks;
    const KArgs& a = P.a[shot];
    if ((int)blockIdx.x * TX >= a.nx || (int)blockIdx.y * TY3 >= a.ny || __ldg(a.it_ptr) >= a.it_hi) return;
    velocity_body<R, true, CPML, EPI, false>(P.m[shot], a, blockIdx.z - shot * P.chunks);
}

// ---------------------------------------------------------------------------
// Launch helpers (instantiated per R in launch_r4.cu / launch_r6.cu)
// ---------------------------------------------------------------------------
// One instantiation per kernel, so the shared-memory opt-in below is made for
// each kernel separately (the kernels share their function types), once per device.
template <typename MAPS, void (*K)(MAPS, KArgs)>
static cudaError_t launch_dyn(dim3 grid, dim3 block, size_t smem, const MAPS& m, const KArgs& a,
                              cudaStream_t st)
{
    static unsigned long long opted = 0;
    cudaError_t attr = smem_opt_in(K, smem, &opted);
    if (attr != cudaSuccess) return attr;
    K<<<grid, block, smem, st>>>(m, a);
    return cudaGetLastError();
}

template <int R, bool Y, bool C, bool P>
static cudaError_t launch_stress_y(dim3 grid, dim3 block, const StressMaps& m, const KArgs& a,
                                   cudaStream_t st)
{
    return launch_dyn<StressMaps, k_stress<R, Y, C, P>>(grid, block,
                                                         StressShape<R, Y, C, P>::BYTES, m, a, st);
}

inline dim3 step_grid(const Geom& g, const KArgs& a, int tyb)
{
    return dim3((g.nx + TX - 1) / TX, (g.ny + tyb - 1) / tyb, (g.nz + a.kchunk - 1) / a.kchunk);
}

template <int R>
cudaError_t launch_stress_t(const Geom& g, const KArgs& a, const StressMaps& m, bool cpml, bool ps,
                            cudaStream_t st)
{
    const bool Y = !g.two_d;
    const int tyb = Y ? TY3 : TY2;
    dim3 block(TX, tyb + 1), grid = step_grid(g, a, tyb);
    if (Y) {
        if (cpml) return ps ? launch_stress_y<R, true, true, true>(grid, block, m, a, st)
                            : launch_stress_y<R, true, true, false>(grid, block, m, a, st);
        return ps ? launch_stress_y<R, true, false, true>(grid, block, m, a, st)
                  : launch_stress_y<R, true, false, false>(grid, block, m, a, st);
    }
    if (cpml) return ps ? launch_stress_y<R, false, true, true>(grid, block, m, a, st)
                        : launch_stress_y<R, false, true, false>(grid, block, m, a, st);
    return ps ? launch_stress_y<R, false, false, true>(grid, block, m, a, st)
              : launch_stress_y<R, false, false, false>(grid, block, m, a, st);
}

template <int R, bool Y, bool C>
static cudaError_t launch_velocity_y(dim3 grid, dim3 block, const VelMaps& m, const KArgs& a,
                                     int epi, bool rec, cudaStream_t st)
{
    if (epi == EPI_EXCITE)
        return launch_dyn<VelMaps, k_velocity<R, Y, C, EPI_EXCITE, false>>(
            grid, block, VelShape<R, Y, C, EPI_EXCITE>::BYTES, m, a, st);
    if (epi == EPI_IMAGE)
        return launch_dyn<VelMaps, k_velocity<R, Y, C, EPI_IMAGE, false>>(
            grid, block, VelShape<R, Y, C, EPI_IMAGE>::BYTES, m, a, st);
    if (rec)
        return launch_dyn<VelMaps, k_velocity<R, Y, C, EPI_NONE, true>>(
            grid, block, VelShape<R, Y, C, EPI_NONE>::BYTES, m, a, st);
    return launch_dyn<VelMaps, k_velocity<R, Y, C, EPI_NONE, false>>(
        grid, block, VelShape<R, Y, C, EPI_NONE>::BYTES, m, a, st);
}

template <int R>
cudaError_t launch_velocity_t(const Geom& g, const KArgs& a, const VelMaps& m, bool cpml, int epi,
                              bool rec, cudaStream_t st)
{
    const bool Y = !g.two_d;
    const int tyb = Y ? TY3 : TY2;
    dim3 block(TX, tyb + 1), grid = step_grid(g, a, tyb);
    if (Y) return cpml ? launch_velocity_y<R, true, true>(grid, block, m, a, epi, rec, st)
                       : launch_velocity_y<R, true, false>(grid, block, m, a, epi, rec, st);
    return cpml ? launch_velocity_y<R, false, true>(grid, block, m, a, epi, rec, st)
                : launch_velocity_y<R, false, false>(grid, block, m, a, epi, rec, st);
}

template <typename P, void (*K)(P)>
static cudaError_t launch_dyn_multi(dim3 grid, size_t smem, const P& prm, cudaStream_t st)
{
    static unsigned long long opted = 0;
    cudaError_t attr = smem_opt_in(K, smem, &opted);
    if (attr != cudaSuccess) return attr;
    K<<<grid, dim3(TX, TY3 + 1), smem, st>>>(prm);
    return cudaGetLastError();
}

template <int R>
cudaError_t launch_stress_multi_t(dim3 grid, const StressMulti& P, bool cpml, cudaStream_t st)
{
    if (cpml)
        return launch_dyn_multi<StressMulti, k_stress_multi<R, true>>(grid, StressShape<R, true, true, true>::BYTES, P, st);
    return launch_dyn_multi<StressMulti, k_stress_multi<R, false>>(grid, StressShape<R, true, false, true>::BYTES, P, st);
}

template <int R>
cudaError_t launch_velocity_multi_t(dim3 grid, const VelMulti& P, bool cpml, int epi, cudaStream_t st)
{
    if (epi == EPI_EXCITE)
        return cpml ? launch_dyn_multi<VelMulti, k_velocity_multi<R, true, EPI_EXCITE>>(
                          grid, VelShape<R, true, true, EPI_EXCITE>::BYTES, P, st)
                    : launch_dyn_multi<VelMulti, k_velocity_multi<R, false, EPI_EXCITE>>(
                          grid, VelShape<R, true, false, EPI_EXCITE>::BYTES, P, st);
    if (epi == EPI_IMAGE)
        return cpml ? launch_dyn_multi<VelMulti, k_velocity_multi<R, true, EPI_IMAGE>>(
                          grid, VelShape<R, true, true, EPI_IMAGE>::BYTES, P, st)
                    : launch_dyn_multi<VelMulti, k_velocity_multi<R, false, EPI_IMAGE>>(
                          grid, VelShape<R, true, false, EPI_IMAGE>::BYTES, P, st);
    return cudaErrorInvalidValue;
}

}  // namespace ertm
