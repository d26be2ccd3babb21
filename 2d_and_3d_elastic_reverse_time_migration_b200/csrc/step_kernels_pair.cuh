// Cell-pair variants of the 3D step kernels (sm_100a).
//
// Same tiles, shared-memory stages, TMA tensor maps, mbarrier protocol and z
// chunks as k_stress / k_velocity (step_kernels.cuh), but each consumer thread
// updates two x-adjacent cells: a warp covers two rows of the 32 x 8 tile
// (16 lanes x 2 cells each), so a CTA has TYB/2 consumer warps plus the producer
// warp.  The pairing cuts instructions per cell:
//   * every shared-memory read of the staged planes is a 64-bit load: the x
//     stencils read their 2R+2-wide window once for both cells, the y stencils
//     and the per-cell values one float2 per row;
//   * the y and z stencils of both cells run as packed FP32 pairs (FFMA2,
//     __ffma2_rn); the x stencils, whose taps straddle the pairs, stay scalar on
//     the loaded window;
//   * z queues hold float2, loop control, waits, releases and stores (64-bit)
//     are shared by two cells.
// Per cell the stencil arithmetic is that of the single-cell kernels in the same
// order: a difference a - b is fma(-1, b, a) (one rounding, as a subtraction),
// each tap is fma(c_n, difference, sum); the compiler may fuse the update's
// products differently, so results agree to float rounding.  The memory
// variables of the C-PML, the source, receivers and the excitation / imaging
// epilogue are handled cell by cell.  2D grids keep the single-cell kernels (one
// tile row only).  Measured on B200 at 480 x 480 x 380 (R = 4, C-PML, source
// pass) the pairs are slower than the single-cell kernels (stress 1.517 against
// 1.447 ms, velocity 1.658 against 1.615 ms): those already move their DRAM
// traffic at ~89 % of the copy bandwidth, and half as many warps per SM hide
// less latency.  They stay an option (ertm_set_step_variant); the single-cell
// kernels are the default.
#pragma once

#include "step_kernels.cuh"

namespace ertm {

constexpr int PAIR_WARPS = TY3 / 2;   // consumer warps of a pair CTA (two tile rows each)

__device__ __forceinline__ float2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ void st2(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
// a - b per lane with one rounding (fma(-1, b, a) is exact up to the final rounding)
__device__ __forceinline__ float2 sub2(float2 a, float2 b)
{
    return __ffma2_rn(make_float2(-1.f, -1.f), b, a);
}
// acc + c (d) per lane, one rounding (fmaf(c, d, acc) per lane)
__device__ __forceinline__ float2 fma2(float c, float2 d, float2 acc)
{
    return __ffma2_rn(make_float2(c, c), d, acc);
}
__device__ __forceinline__ float lane_of(float2 v, int e) { return e ? v.y : v.x; }

// The x window of one staged row around a cell pair: 2R+2 values at row offsets
// base .. base+2R+1, base = (first cell) - R; cell e of the pair sits at R + e.
template <int R>
struct XWin {
    float v[2 * R + 2];
    __device__ __forceinline__ void load(const float* p)   // p: 8-byte aligned
    {
#pragma unroll
        for (int q = 0; q <= R; q++) {
            const float2 t = ld2(p + 2 * q);
            v[2 * q] = t.x;
            v[2 * q + 1] = t.y;
        }
    }
    // D+ f at cell e: sum_n c_n (f[i+n] - f[i-n+1])
    __device__ __forceinline__ float dp(const float* c, int e) const
    {
        float s = 0.f;
#pragma unroll
        for (int n = 1; n <= R; n++) s = fmaf(c[n], v[R + e + n] - v[R + e - n + 1], s);
        return s;
    }
    // D- f at cell e: sum_n c_n (f[i+n-1] - f[i-n])
    __device__ __forceinline__ float dm(const float* c, int e) const
    {
        float s = 0.f;
#pragma unroll
        for (int n = 1; n <= R; n++) s = fmaf(c[n], v[R + e + n - 1] - v[R + e - n], s);
        return s;
    }
};

// y stencils of a cell pair over a staged box with row pitch P (p: the pair's row)
template <int R, int P>
__device__ __forceinline__ float2 dyp2(const float* p, const float* c)   // D+
{
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int n = 1; n <= R; n++) s = fma2(c[n], sub2(ld2(p + n * P), ld2(p + (1 - n) * P)), s);
    return s;
}
template <int R, int P>
__device__ __forceinline__ float2 dym2(const float* p, const float* c)   // D-
{
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int n = 1; n <= R; n++) s = fma2(c[n], sub2(ld2(p + (n - 1) * P), ld2(p - n * P)), s);
    return s;
}
// z stencils of a cell pair on a register queue of 2R+1 planes (plane k at q[R])
template <int R>
__device__ __forceinline__ float2 dzp2(const float2* q, const float* c)   // D+
{
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int n = 1; n <= R; n++) s = fma2(c[n], sub2(q[R + n], q[R - n + 1]), s);
    return s;
}
template <int R>
__device__ __forceinline__ float2 dzm2(const float2* q, const float* c)   // D-
{
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int n = 1; n <= R; n++) s = fma2(c[n], sub2(q[R + n - 1], q[R - n]), s);
    return s;
}

// ---------------------------------------------------------------------------
// Stress kernel, cell pairs (3D)
// ---------------------------------------------------------------------------
template <int R, bool CPML, bool PS>
__global__ void __launch_bounds__(32 * (PAIR_WARPS + 1), CTAS3)
k_stress2(const __grid_constant__ StressMaps maps, const KArgs a)
{
    using SS = StressShape<R, true, CPML, PS>;
    using B = typename SS::B;
    constexpr int NS = SS::NS;
    constexpr int XB = B::XB, XW = B::XW, CB = B::C;
    constexpr int NV = SS::NV, NSIG = SS::NSIG;
    constexpr int C_TP = NSIG, C_M = NSIG + (PS ? 1 : 0), C_MU = C_M + 1;
    static_assert((XW % 2) == 0 && ((XB - R) % 2) == 0, "pair loads must be 8-byte aligned");
    extern __shared__ __align__(128) float sm[];
    float* psibuf = sm + NS * SS::STAGE;
    uint64_t* bars = reinterpret_cast<uint64_t*>(psibuf + 3 * SS::PSI);

    const int lane = threadIdx.x, wy = threadIdx.y;
    const bool leader = (lane == 0 && wy == PAIR_WARPS);
    const int r = 2 * wy + (lane >> 4);          // tile row of the pair
    const int ci = 2 * (lane & 15);              // tile column of the pair's first cell
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * B::TYB;
    const int i = i0 + ci, j = j0 + r;
    const int k0 = blockIdx.z * a.kchunk;
    const int k1 = min(k0 + a.kchunk, a.nz);
    const int nk = k1 - k0;
    const int sy = (int)a.sy, sz = (int)a.sz;
    const bool act[2] = {(i < a.nx) && (j < a.ny), (i + 1 < a.nx) && (j < a.ny)};
    const int it = __ldg(a.it_ptr);
    const bool src_on = (it >= 0) && (it < a.nw);
    const float wsrc = src_on ? __ldg(a.wavelet + it) : 0.f;
    const int cell = r * TX + ci;                // C-box index of the first cell
    const int gx = i0 + XH, gy = j0 + R, gz0 = k0 + R;

    float* sig[6] = {a.f[F_TXX], a.f[F_TZZ], a.f[F_TXZ], a.f[F_TYY], a.f[F_TXY], a.f[F_TYZ]};
    float* tp = a.f[F_TP];
    const int cj = j * sy + i;

    auto issue = [&](int t) -> bool {
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

    // C-PML: slab membership and profile coefficients of the pair's columns
    const int WX = a.w[0] + a.w[1], WY = a.w[2] + a.w[3];
    bool inx[2], iny;
    int slx[2];
    float axf[2], bxf[2], axh[2], bxh[2];
    float ayf = 0.f, byf = 1.f, ayh = 0.f, byh = 1.f;
#pragma unroll
    for (int e = 0; e < 2; e++) {
        inx[e] = CPML && act[e] && (i + e < a.w[0] || i + e >= a.nx - a.w[1]);
        slx[e] = i + e < a.w[0] ? i + e : i + e - a.nx + WX;
        axf[e] = 0.f; bxf[e] = 1.f; axh[e] = 0.f; bxh[e] = 1.f;
        if (inx[e]) {
            axf[e] = __ldg(a.pa[0][0] + i + e); bxf[e] = __ldg(a.pb[0][0] + i + e);
            axh[e] = __ldg(a.pa[0][1] + i + e); bxh[e] = __ldg(a.pb[0][1] + i + e);
        }
    }
    iny = CPML && act[0] && (j < a.w[2] || j >= a.ny - a.w[3]);
    const int sly = j < a.w[2] ? j : j - a.ny + WY;
    if (iny) {
        ayf = __ldg(a.pa[1][0] + j); byf = __ldg(a.pb[1][0] + j);
        ayh = __ldg(a.pa[1][1] + j); byh = __ldg(a.pb[1][1] + j);
    }
    // psi slots: x: EXX DXVZ DXVY, y: EYY DYVX DYVZ, z: EZZ DZVX DZVY (cell e at + e)
    constexpr int PX = 0, PY = 3, PZ = 6;
    auto issue_psi = [&](int p, int buf) {
        if (!CPML) return;
        float* Ps = psibuf + buf * SS::PSI;
#pragma unroll
        for (int e = 0; e < 2; e++) {
            if (inx[e]) {
                const int x = (p * a.ny + j) * WX + slx[e];
                cpa4(&Ps[(PX + 0) * CB + cell + e], a.psi[P_EXX] + x);
                cpa4(&Ps[(PX + 1) * CB + cell + e], a.psi[P_DXVZ] + x);
                cpa4(&Ps[(PX + 2) * CB + cell + e], a.psi[P_DXVY] + x);
            }
            if (iny && act[e]) {
                const int y = (p * WY + sly) * a.nx + i + e;
                cpa4(&Ps[(PY + 0) * CB + cell + e], a.psi[P_EYY] + y);
                cpa4(&Ps[(PY + 1) * CB + cell + e], a.psi[P_DYVX] + y);
                cpa4(&Ps[(PY + 2) * CB + cell + e], a.psi[P_DYVZ] + y);
            }
            if (act[e] && (p < a.w[4] || p >= a.nz - a.w[5])) {
                const int sl = p < a.w[4] ? p : p - a.nz + a.w[4] + a.w[5];
                const int z = (sl * a.ny + j) * a.nx + i + e;
                cpa4(&Ps[(PZ + 0) * CB + cell + e], a.psi[P_EZZ] + z);
                cpa4(&Ps[(PZ + 1) * CB + cell + e], a.psi[P_DZVX] + z);
                cpa4(&Ps[(PZ + 2) * CB + cell + e], a.psi[P_DZVY] + z);
            }
        }
        cpa_commit();
    };

    if (leader) {
        for (int s = 0; s < NS; s++) {
            mbar_init(&bars[s], 1);
            mbar_init(&bars[NS + s], PAIR_WARPS);
        }
        mbar_fence_init();
    }
    __syncthreads();
    if (wy == PAIR_WARPS) {   // producer warp
        if (leader && !produce_planes<NS>(bars, nk, consumer_polls(a), issue) && a.err)
            atomicExch(a.err, DEV_WAIT_TIMEOUT);
        return;
    }

    // register queues of planes k-R .. k+R (pairs); the front (k+R) arrives with each stage
    const float* vsrc[3] = {a.f[F_VX], a.f[F_VZ], a.f[F_VY]};
    float2 qx[2 * R + 1], qy[2 * R + 1], qz[2 * R + 1];
#pragma unroll
    for (int q = 0; q < 2 * R; q++) {
        const int cc = (k0 + q - R) * sz + cj;
        qx[q] = ld2(vsrc[0] + cc);
        qz[q] = ld2(vsrc[1] + cc);
        qy[q] = ld2(vsrc[2] + cc);
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
        qx[2 * R] = ld2(S + SS::OFF_FR + 0 * CB + cell);
        qz[2 * R] = ld2(S + SS::OFF_FR + 1 * CB + cell);
        qy[2 * R] = ld2(S + SS::OFF_FR + 2 * CB + cell);
        // the pair's row in the staged v tiles ((TX+2XB) wide, (TYB+2R) high)
        const float* Tx = S + 0 * B::XYP + (r + R) * XW + XB + ci;
        const float* Tz = S + 1 * B::XYP + (r + R) * XW + XB + ci;
        const float* Ty = S + 2 * B::XYP + (r + R) * XW + XB + ci;

        // x derivatives on the rows' windows (scalar per cell)
        XWin<R> wx, wz, wyy;
        wx.load(Tx - R);
        wz.load(Tz - R);
        wyy.load(Ty - R);
        float exx[2], dxvz[2], dxvy[2];
#pragma unroll
        for (int e = 0; e < 2; e++) {
            exx[e] = wx.dp(a.cx, e);
            dxvz[e] = wz.dm(a.cx, e);
            dxvy[e] = wyy.dm(a.cx, e);
        }
        // y and z derivatives as pairs
        const float2 eyy2 = dyp2<R, XW>(Ty, a.cy);
        const float2 dyvx2 = dym2<R, XW>(Tx, a.cy);
        const float2 dyvz2 = dym2<R, XW>(Tz, a.cy);
        const float2 ezz2 = dzm2<R>(qz, a.cz);
        const float2 dzvx2 = dzp2<R>(qx, a.cz);
        const float2 dzvy2 = dzp2<R>(qy, a.cz);

        const float2 oxx2 = ld2(Cc + 0 * CB + cell), ozz2 = ld2(Cc + 1 * CB + cell);
        const float2 oxz2 = ld2(Cc + 2 * CB + cell), oyy2 = ld2(Cc + 3 * CB + cell);
        const float2 oxy2 = ld2(Cc + 4 * CB + cell), oyz2 = ld2(Cc + 5 * CB + cell);
        const float2 M2 = ld2(Cc + C_M * CB + cell), U2 = ld2(Cc + C_MU * CB + cell);
        float2 otp2 = make_float2(0.f, 0.f);
        if (PS) otp2 = ld2(Cc + C_TP * CB + cell);
        float nxx[2], nzz[2], nxz[2], nyy[2], nxy[2], nyz[2], ntp[2];
        const int c = k * sz + cj;
#pragma unroll
        for (int e = 0; e < 2; e++) {
            float ex = exx[e], dxz = dxvz[e], dxy = dxvy[e];
            float ey = lane_of(eyy2, e), dyx = lane_of(dyvx2, e), dyz = lane_of(dyvz2, e);
            float ez = lane_of(ezz2, e), dzx = lane_of(dzvx2, e), dzy = lane_of(dzvy2, e);
            if (CPML && act[e]) {
                if (inx[e]) {
                    const int x = (k * a.ny + j) * WX + slx[e];
                    float p0 = fmaf(bxf[e], Ps[(PX + 0) * CB + cell + e], axf[e] * ex);
                    float p1 = fmaf(bxh[e], Ps[(PX + 1) * CB + cell + e], axh[e] * dxz);
                    float p2 = fmaf(bxh[e], Ps[(PX + 2) * CB + cell + e], axh[e] * dxy);
                    a.psi[P_EXX][x] = p0;
                    a.psi[P_DXVZ][x] = p1;
                    a.psi[P_DXVY][x] = p2;
                    ex += p0;
                    dxz += p1;
                    dxy += p2;
                }
                if (iny) {
                    const int y = (k * WY + sly) * a.nx + i + e;
                    float p0 = fmaf(byf, Ps[(PY + 0) * CB + cell + e], ayf * ey);
                    float p1 = fmaf(byh, Ps[(PY + 1) * CB + cell + e], ayh * dyx);
                    float p2 = fmaf(byh, Ps[(PY + 2) * CB + cell + e], ayh * dyz);
                    a.psi[P_EYY][y] = p0;
                    a.psi[P_DYVX][y] = p1;
                    a.psi[P_DYVZ][y] = p2;
                    ey += p0;
                    dyx += p1;
                    dyz += p2;
                }
                if (k < a.w[4] || k >= a.nz - a.w[5]) {
                    const int sl = k < a.w[4] ? k : k - a.nz + a.w[4] + a.w[5];
                    const int z = (sl * a.ny + j) * a.nx + i + e;
                    const float azf = __ldg(a.pa[2][0] + k), bzf = __ldg(a.pb[2][0] + k);
                    const float azh = __ldg(a.pa[2][1] + k), bzh = __ldg(a.pb[2][1] + k);
                    float p0 = fmaf(bzf, Ps[(PZ + 0) * CB + cell + e], azf * ez);
                    float p1 = fmaf(bzh, Ps[(PZ + 1) * CB + cell + e], azh * dzx);
                    float p2 = fmaf(bzh, Ps[(PZ + 2) * CB + cell + e], azh * dzy);
                    a.psi[P_EZZ][z] = p0;
                    a.psi[P_DZVX][z] = p1;
                    a.psi[P_DZVY][z] = p2;
                    ez += p0;
                    dzx += p1;
                    dzy += p2;
                }
            }
            float g1, g2;
            damping<true>(a, CPML, i + e, j, k, g1, g2);
            const float M = lane_of(M2, e), U = lane_of(U2, e);
            const float L = M - 2.f * U;
            const float dt = a.dt;
            float oxx = lane_of(oxx2, e), ozz = lane_of(ozz2, e), oyy = lane_of(oyy2, e);
            if (src_on && i + e == a.ssx && j == a.ssy && k == a.ssz) {   // add_source_3D
                oxx += wsrc;
                ozz += wsrc;
                oyy += wsrc;
            }
            nxx[e] = g1 * (g2 * oxx + dt * (M * ex + L * (ey + ez)));
            nzz[e] = g1 * (g2 * ozz + dt * (M * ez + L * (ex + ey)));
            nxz[e] = g1 * (g2 * lane_of(oxz2, e) + dt * U * (dzx + dxz));
            nyy[e] = g1 * (g2 * oyy + dt * (M * ey + L * (ex + ez)));
            nxy[e] = g1 * (g2 * lane_of(oxy2, e) + dt * U * (dyx + dxy));
            nyz[e] = g1 * (g2 * lane_of(oyz2, e) + dt * U * (dzy + dyz));
            ntp[e] = PS ? g1 * (g2 * lane_of(otp2, e) + dt * M * (ex + ey + ez)) : 0.f;
        }
        if (act[1]) {
            st2(sig[0] + c, make_float2(nxx[0], nxx[1]));
            st2(sig[1] + c, make_float2(nzz[0], nzz[1]));
            st2(sig[2] + c, make_float2(nxz[0], nxz[1]));
            st2(sig[3] + c, make_float2(nyy[0], nyy[1]));
            st2(sig[4] + c, make_float2(nxy[0], nxy[1]));
            st2(sig[5] + c, make_float2(nyz[0], nyz[1]));
            if (PS) st2(tp + c, make_float2(ntp[0], ntp[1]));
        } else if (act[0]) {
            sig[0][c] = nxx[0];
            sig[1][c] = nzz[0];
            sig[2][c] = nxz[0];
            sig[3][c] = nyy[0];
            sig[4][c] = nxy[0];
            sig[5][c] = nyz[0];
            if (PS) tp[c] = ntp[0];
        }

#pragma unroll
        for (int q = 0; q < 2 * R; q++) {
            qx[q] = qx[q + 1];
            qz[q] = qz[q + 1];
            qy[q] = qy[q + 1];
        }
        cpa_wait_1();   // plane t+1's memory variables have landed
        __syncwarp();
        if (lane == 0) mbar_arrive(&bars[NS + st]);   // release the stage
    }
    if (!ok && a.err) atomicExch(a.err, DEV_WAIT_TIMEOUT);
}

// ---------------------------------------------------------------------------
// Velocity kernel, cell pairs (3D)
// ---------------------------------------------------------------------------
template <int R, bool CPML, int EPI, bool REC>
__global__ void __launch_bounds__(32 * (PAIR_WARPS + 1), CTAS3)
k_velocity2(const __grid_constant__ VelMaps maps, const KArgs a)
{
    using VS = VelShape<R, true, CPML, EPI>;
    using B = typename VS::B;
    constexpr int NS = VS::NS;
    constexpr bool PS = VS::PS;
    constexpr int XB = B::XB, XW = B::XW, CB = B::C;
    static_assert((XW % 2) == 0 && ((XB - R) % 2) == 0, "pair loads must be 8-byte aligned");
    extern __shared__ __align__(128) float sm[];
    float* psibuf = sm + NS * VS::STAGE;
    uint64_t* bars = reinterpret_cast<uint64_t*>(psibuf + 3 * VS::PSI);

    const int lane = threadIdx.x, wy = threadIdx.y;
    const bool leader = (lane == 0 && wy == PAIR_WARPS);
    const int r = 2 * wy + (lane >> 4);
    const int ci = 2 * (lane & 15);
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * B::TYB;
    const int i = i0 + ci, j = j0 + r;
    const int k0 = blockIdx.z * a.kchunk;
    const int k1 = min(k0 + a.kchunk, a.nz);
    const int nk = k1 - k0;
    const int sy = (int)a.sy, sz = (int)a.sz;
    const bool act[2] = {(i < a.nx) && (j < a.ny), (i + 1 < a.nx) && (j < a.ny)};
    const int it = __ldg(a.it_ptr);
    int rec[2];
#pragma unroll
    for (int e = 0; e < 2; e++) rec[e] = ((REC || EPI == EPI_IMAGE) && act[e]) ? receiver_index(a, i + e, j) : -1;
    const long long nrec = (long long)a.nrx * a.nry;
    const int cell = r * TX + ci;
    const int gx = i0 + XH, gy = j0 + R, gz0 = k0 + R;
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
        tma3(S + VS::O_TXY, &maps.txy, gx - XB, gy - R, z, bar);
        tma3(S + VS::O_TYY, &maps.tyy, gx, gy - R, z, bar);
        tma3(S + VS::O_TYZ, &maps.tyz, gx, gy - R, z, bar);
        if (PS) tma3(S + VS::O_TP, &maps.tp, gx - XB, gy - B::YB, z, bar);
#pragma unroll
        for (int f = 0; f < VS::NFR; f++) tma3(S + VS::O_FR + f * CB, &maps.fr[f], gx, gy, z + R, bar);
#pragma unroll
        for (int q = 0; q < VS::NC; q++) tma3(S + VS::O_C + q * CB, &maps.c[q], gx, gy, z, bar);
        return true;
    };

    const int WX = a.w[0] + a.w[1], WY = a.w[2] + a.w[3];
    bool inx[2], iny;
    int slx[2];
    float axf[2], bxf[2], axh[2], bxh[2];
    float ayf = 0.f, byf = 1.f, ayh = 0.f, byh = 1.f;
#pragma unroll
    for (int e = 0; e < 2; e++) {
        inx[e] = CPML && act[e] && (i + e < a.w[0] || i + e >= a.nx - a.w[1]);
        slx[e] = i + e < a.w[0] ? i + e : i + e - a.nx + WX;
        axf[e] = 0.f; bxf[e] = 1.f; axh[e] = 0.f; bxh[e] = 1.f;
        if (inx[e]) {
            axf[e] = __ldg(a.pa[0][0] + i + e); bxf[e] = __ldg(a.pb[0][0] + i + e);
            axh[e] = __ldg(a.pa[0][1] + i + e); bxh[e] = __ldg(a.pb[0][1] + i + e);
        }
    }
    iny = CPML && act[0] && (j < a.w[2] || j >= a.ny - a.w[3]);
    const int sly = j < a.w[2] ? j : j - a.ny + WY;
    if (iny) {
        ayf = __ldg(a.pa[1][0] + j); byf = __ldg(a.pb[1][0] + j);
        ayh = __ldg(a.pa[1][1] + j); byh = __ldg(a.pb[1][1] + j);
    }
    // psi slots: x: DXTXX DXTXZ DXTXY, y: DYTXY DYTYY DYTYZ, z: DZTXZ DZTZZ DZTYZ
    constexpr int PX = 0, PY = 3, PZ = 6;
    auto issue_psi = [&](int p, int buf) {
        if (!CPML) return;
        float* Ps = psibuf + buf * VS::PSI;
#pragma unroll
        for (int e = 0; e < 2; e++) {
            if (inx[e]) {
                const int x = (p * a.ny + j) * WX + slx[e];
                cpa4(&Ps[(PX + 0) * CB + cell + e], a.psi[P_DXTXX] + x);
                cpa4(&Ps[(PX + 1) * CB + cell + e], a.psi[P_DXTXZ] + x);
                cpa4(&Ps[(PX + 2) * CB + cell + e], a.psi[P_DXTXY] + x);
            }
            if (iny && act[e]) {
                const int y = (p * WY + sly) * a.nx + i + e;
                cpa4(&Ps[(PY + 0) * CB + cell + e], a.psi[P_DYTXY] + y);
                cpa4(&Ps[(PY + 1) * CB + cell + e], a.psi[P_DYTYY] + y);
                cpa4(&Ps[(PY + 2) * CB + cell + e], a.psi[P_DYTYZ] + y);
            }
            if (act[e] && (p < a.w[4] || p >= a.nz - a.w[5])) {
                const int sl = p < a.w[4] ? p : p - a.nz + a.w[4] + a.w[5];
                const int z = (sl * a.ny + j) * a.nx + i + e;
                cpa4(&Ps[(PZ + 0) * CB + cell + e], a.psi[P_DZTXZ] + z);
                cpa4(&Ps[(PZ + 1) * CB + cell + e], a.psi[P_DZTZZ] + z);
                cpa4(&Ps[(PZ + 2) * CB + cell + e], a.psi[P_DZTYZ] + z);
            }
        }
        cpa_commit();
    };

    if (leader) {
        for (int s = 0; s < NS; s++) {
            mbar_init(&bars[s], 1);
            mbar_init(&bars[NS + s], PAIR_WARPS);
        }
        mbar_fence_init();
    }
    __syncthreads();
    if (wy == PAIR_WARPS) {   // producer warp
        if (leader && !produce_planes<NS>(bars, nk, consumer_polls(a), issue) && a.err)
            atomicExch(a.err, DEV_WAIT_TIMEOUT);
        return;
    }

    const float* txz = a.f[F_TXZ];
    const float* tyz = a.f[F_TYZ];
    const float* tzz = a.f[F_TZZ];
    const float* tp = a.f[F_TP];
    float2 qxz[2 * R + 1], qyz[2 * R + 1], qzz[2 * R + 1], qtp[2 * R + 1];
#pragma unroll
    for (int q = 0; q < 2 * R; q++) {
        const int cc = (k0 + q - R) * sz + cj;
        qxz[q] = ld2(txz + cc);
        qzz[q] = ld2(tzz + cc);
        qyz[q] = ld2(tyz + cc);
        if (PS) qtp[q] = ld2(tp + cc);
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
        qxz[2 * R] = ld2(S + VS::O_FR + 0 * CB + cell);
        qzz[2 * R] = ld2(S + VS::O_FR + 1 * CB + cell);
        qyz[2 * R] = ld2(S + VS::O_FR + VS::FR_TYZ * CB + cell);
        if (PS) qtp[2 * R] = ld2(S + VS::O_FR + VS::FR_TP * CB + cell);
        const float* Txx = S + VS::O_TXX + r * XW + XB + ci;
        const float* Txz = S + VS::O_TXZ + r * XW + XB + ci;
        const float* Txy = S + VS::O_TXY + (r + R) * XW + XB + ci;
        const float* Tyy = S + VS::O_TYY + (r + R) * TX + ci;
        const float* Tyz = S + VS::O_TYZ + (r + R) * TX + ci;
        const float* Ttp = S + VS::O_TP + (r + B::YB) * XW + XB + ci;

        // x derivatives on the rows' windows (scalar per cell)
        XWin<R> wxx, wxz, wxy, wtp;
        wxx.load(Txx - R);
        wxz.load(Txz - R);
        wxy.load(Txy - R);
        if (PS) wtp.load(Ttp - R);
        float dxtxx[2], dxtxz[2], dxtxy[2], dxtp[2] = {0.f, 0.f};
#pragma unroll
        for (int e = 0; e < 2; e++) {
            dxtxx[e] = wxx.dm(a.cx, e);
            dxtxz[e] = wxz.dp(a.cx, e);
            dxtxy[e] = wxy.dp(a.cx, e);
            if (PS) dxtp[e] = wtp.dm(a.cx, e);
        }
        // y and z derivatives as pairs
        const float2 dytxy2 = dyp2<R, XW>(Txy, a.cy);
        const float2 dytyy2 = dym2<R, TX>(Tyy, a.cy);
        const float2 dytyz2 = dyp2<R, TX>(Tyz, a.cy);
        const float2 dztxz2 = dzm2<R>(qxz, a.cz);
        const float2 dztzz2 = dzp2<R>(qzz, a.cz);
        const float2 dztyz2 = dzm2<R>(qyz, a.cz);
        float2 dytp2 = make_float2(0.f, 0.f), dztp2 = make_float2(0.f, 0.f);
        if (PS) {
            dytp2 = dym2<R, XW>(Ttp, a.cy);
            dztp2 = dzp2<R>(qtp, a.cz);
        }

        const float2 ovx2 = ld2(Cc + VS::C_VX * CB + cell), ovz2 = ld2(Cc + VS::C_VZ * CB + cell);
        const float2 ovy2 = ld2(Cc + VS::C_VY * CB + cell), b2 = ld2(Cc + VS::C_B * CB + cell);
        float2 opx2 = make_float2(0.f, 0.f), opy2 = opx2, opz2 = opx2, oex2 = opx2;
        if (PS) {
            opx2 = ld2(Cc + VS::C_PX * CB + cell);
            opz2 = ld2(Cc + VS::C_PZ * CB + cell);
            opy2 = ld2(Cc + VS::C_PY * CB + cell);
            oex2 = ld2(Cc + VS::C_EX * CB + cell);
        }
        const int c = k * sz + cj;
        float nvx[2], nvy[2], nvz[2], npx[2] = {0.f, 0.f}, npy[2] = {0.f, 0.f}, npz[2] = {0.f, 0.f};
#pragma unroll
        for (int e = 0; e < 2; e++) {
            float dxx = dxtxx[e], dxz = dxtxz[e], dxy = dxtxy[e];
            float dyxy = lane_of(dytxy2, e), dyyy = lane_of(dytyy2, e), dyyz = lane_of(dytyz2, e);
            float dzxz = lane_of(dztxz2, e), dzzz = lane_of(dztzz2, e), dzyz = lane_of(dztyz2, e);
            if (CPML && act[e]) {
                if (inx[e]) {
                    const int x = (k * a.ny + j) * WX + slx[e];
                    float p0 = fmaf(bxh[e], Ps[(PX + 0) * CB + cell + e], axh[e] * dxx);
                    float p1 = fmaf(bxf[e], Ps[(PX + 1) * CB + cell + e], axf[e] * dxz);
                    float p2 = fmaf(bxf[e], Ps[(PX + 2) * CB + cell + e], axf[e] * dxy);
                    a.psi[P_DXTXX][x] = p0;
                    a.psi[P_DXTXZ][x] = p1;
                    a.psi[P_DXTXY][x] = p2;
                    dxx += p0;
                    dxz += p1;
                    dxy += p2;
                }
                if (iny) {
                    const int y = (k * WY + sly) * a.nx + i + e;
                    float p0 = fmaf(byf, Ps[(PY + 0) * CB + cell + e], ayf * dyxy);
                    float p1 = fmaf(byh, Ps[(PY + 1) * CB + cell + e], ayh * dyyy);
                    float p2 = fmaf(byf, Ps[(PY + 2) * CB + cell + e], ayf * dyyz);
                    a.psi[P_DYTXY][y] = p0;
                    a.psi[P_DYTYY][y] = p1;
                    a.psi[P_DYTYZ][y] = p2;
                    dyxy += p0;
                    dyyy += p1;
                    dyyz += p2;
                }
                if (k < a.w[4] || k >= a.nz - a.w[5]) {
                    const int sl = k < a.w[4] ? k : k - a.nz + a.w[4] + a.w[5];
                    const int z = (sl * a.ny + j) * a.nx + i + e;
                    const float azf = __ldg(a.pa[2][0] + k), bzf = __ldg(a.pb[2][0] + k);
                    const float azh = __ldg(a.pa[2][1] + k), bzh = __ldg(a.pb[2][1] + k);
                    float p0 = fmaf(bzf, Ps[(PZ + 0) * CB + cell + e], azf * dzxz);
                    float p1 = fmaf(bzh, Ps[(PZ + 1) * CB + cell + e], azh * dzzz);
                    float p2 = fmaf(bzf, Ps[(PZ + 2) * CB + cell + e], azf * dzyz);
                    a.psi[P_DZTXZ][z] = p0;
                    a.psi[P_DZTZZ][z] = p1;
                    a.psi[P_DZTYZ][z] = p2;
                    dzxz += p0;
                    dzzz += p1;
                    dzyz += p2;
                }
            }
            float g1, g2;
            damping<true>(a, CPML, i + e, j, k, g1, g2);
            const float b = lane_of(b2, e);
            const float db = a.dt * b;
            nvx[e] = g1 * (g2 * lane_of(ovx2, e) + db * (dxx + dyxy + dzxz));
            nvz[e] = g1 * (g2 * lane_of(ovz2, e) + db * (dxz + dyyz + dzzz));
            nvy[e] = g1 * (g2 * lane_of(ovy2, e) + db * (dxy + dyyy + dzyz));
            if (PS) {
                // decoupled P velocity from the P-stress gradient (role of fwd_vxp_vzp_3D,
                // 3D_forward_or_back_together.cu:118); S velocity = v - v_P
                npx[e] = g1 * (g2 * lane_of(opx2, e) + db * dxtp[e]);
                npz[e] = g1 * (g2 * lane_of(opz2, e) + db * lane_of(dztp2, e));
                npy[e] = g1 * (g2 * lane_of(opy2, e) + db * lane_of(dytp2, e));
            }
            if (!act[e]) continue;
            const int ce = c + e;
            if (EPI == EPI_EXCITE) {
                // caculate_ex_amp_time_new (2D_elastic_RTM/elastic_2D_kernel_3.cu:30-48):
                // strict '>' keeps the earliest maximum of |v_P|
                const float a2 = npx[e] * npx[e] + npy[e] * npy[e] + npz[e] * npz[e];
                if (a2 > lane_of(oex2, e)) {
                    a.ex_amp2[ce] = a2;
                    a.ex_time[ce] = it;
                    a.ex_v[0][ce] = npx[e];
                    a.ex_v[1][ce] = npy[e];
                    a.ex_v[2][ce] = npz[e];
                    a.ex_tp[ce] = lane_of(qtp[R], e);
                }
            }
            if (EPI == EPI_IMAGE) {
                // imaging_inner_product_ex / imaging_correlation_ex
                // (2D_elastic_RTM/elastic_2D_kernel_3.cu:542-576) at it == excitation time
                if (__float_as_int(lane_of(oex2, e)) == it) {
                    const float ex = a.ex_v[0][ce], ey = a.ex_v[1][ce], ez = a.ex_v[2][ce];
                    const float den = ex * ex + ey * ey + ez * ez;
                    if (den > 0.f) {   // a true division: 1/den overflows for denormal den
                        if (a.img[0]) a.img[0][ce] = (ex * npx[e] + ey * npy[e] + ez * npz[e]) / den;
                        if (a.img[1])
                            a.img[1][ce] = (ex * (nvx[e] - npx[e]) + ey * (nvy[e] - npy[e]) +
                                            ez * (nvz[e] - npz[e])) / den;
                    }
                    const float et = a.ex_tp[ce];
                    if (a.img[2] && et != 0.f) a.img[2][ce] = lane_of(qtp[R], e) / et;
                }
                // receiver injection of the next (earlier) sample, reference :328
                if (rec[e] >= 0 && k == a.rz && it > 0) {
                    const float* d = a.traces + (long long)(it - 1) * nrec + rec[e];
                    const long long cs = (long long)a.nt * nrec;
                    if (a.inject_mode == 2) {
                        nvx[e] = d[0];
                        nvz[e] = d[2 * cs];
                        nvy[e] = d[cs];
                    } else {
                        nvx[e] += d[0];
                        nvz[e] += d[2 * cs];
                        nvy[e] += d[cs];
                    }
                }
            }
            if (REC && rec[e] >= 0 && k == a.rz) {
                // write_or_add_shot_3D_surface_three, record flag 0 (:127)
                float* d = a.traces + (long long)it * nrec + rec[e];
                const long long cs = (long long)a.nt * nrec;
                d[0] = nvx[e];
                d[cs] = nvy[e];
                d[2 * cs] = nvz[e];
            }
        }
        if (act[1]) {
            st2(vx + c, make_float2(nvx[0], nvx[1]));
            st2(vz + c, make_float2(nvz[0], nvz[1]));
            st2(vy + c, make_float2(nvy[0], nvy[1]));
            if (PS) {
                st2(vxp + c, make_float2(npx[0], npx[1]));
                st2(vzp + c, make_float2(npz[0], npz[1]));
                st2(vyp + c, make_float2(npy[0], npy[1]));
            }
        } else if (act[0]) {
            vx[c] = nvx[0];
            vz[c] = nvz[0];
            vy[c] = nvy[0];
            if (PS) {
                vxp[c] = npx[0];
                vzp[c] = npz[0];
                vyp[c] = npy[0];
            }
        }

#pragma unroll
        for (int q = 0; q < 2 * R; q++) {
            qxz[q] = qxz[q + 1];
            qzz[q] = qzz[q + 1];
            qyz[q] = qyz[q + 1];
            if (PS) qtp[q] = qtp[q + 1];
        }
        cpa_wait_1();   // plane t+1's memory variables have landed
        __syncwarp();
        if (lane == 0) mbar_arrive(&bars[NS + st]);   // release the stage
    }
    if (!ok && a.err) atomicExch(a.err, DEV_WAIT_TIMEOUT);
}

// ---------------------------------------------------------------------------
// Launch helpers of the 3D pair kernels (block: 32 x (PAIR_WARPS + 1))
// ---------------------------------------------------------------------------
template <int R, bool C, bool P>
static cudaError_t launch_stress_pair(dim3 grid, const StressMaps& m, const KArgs& a, cudaStream_t st)
{
    return launch_dyn<StressMaps, k_stress2<R, C, P>>(grid, dim3(32, PAIR_WARPS + 1),
                                                      StressShape<R, true, C, P>::BYTES, m, a, st);
}

template <int R, bool C>
static cudaError_t launch_velocity_pair(dim3 grid, const VelMaps& m, const KArgs& a, int epi, bool rec,
                                        cudaStream_t st)
{
    const dim3 block(32, PAIR_WARPS + 1);
    if (epi == EPI_EXCITE)
        return launch_dyn<VelMaps, k_velocity2<R, C, EPI_EXCITE, false>>(
            grid, block, VelShape<R, true, C, EPI_EXCITE>::BYTES, m, a, st);
    if (epi == EPI_IMAGE)
        return launch_dyn<VelMaps, k_velocity2<R, C, EPI_IMAGE, false>>(
            grid, block, VelShape<R, true, C, EPI_IMAGE>::BYTES, m, a, st);
    if (rec)
        return launch_dyn<VelMaps, k_velocity2<R, C, EPI_NONE, true>>(
            grid, block, VelShape<R, true, C, EPI_NONE>::BYTES, m, a, st);
    return launch_dyn<VelMaps, k_velocity2<R, C, EPI_NONE, false>>(
        grid, block, VelShape<R, true, C, EPI_NONE>::BYTES, m, a, st);
}

// 3D grids: the pair kernels when KArgs::pairs is set, else the single-cell kernels;
// 2D grids: the single-cell kernels (one tile row)
template <int R>
cudaError_t launch_stress_any(const Geom& g, const KArgs& a, const StressMaps& m, bool cpml, bool ps,
                              cudaStream_t st)
{
    if (g.two_d || !a.pairs) return launch_stress_t<R>(g, a, m, cpml, ps, st);
    const dim3 grid = step_grid(g, a, TY3);
    if (cpml) return ps ? launch_stress_pair<R, true, true>(grid, m, a, st)
                        : launch_stress_pair<R, true, false>(grid, m, a, st);
    return ps ? launch_stress_pair<R, false, true>(grid, m, a, st)
              : launch_stress_pair<R, false, false>(grid, m, a, st);
}

template <int R>
cudaError_t launch_velocity_any(const Geom& g, const KArgs& a, const VelMaps& m, bool cpml, int epi,
                                bool rec, cudaStream_t st)
{
    if (g.two_d || !a.pairs) return launch_velocity_t<R>(g, a, m, cpml, epi, rec, st);
    const dim3 grid = step_grid(g, a, TY3);
    return cpml ? launch_velocity_pair<R, true>(grid, m, a, epi, rec, st)
                : launch_velocity_pair<R, false>(grid, m, a, epi, rec, st);
}

}  // namespace ertm
