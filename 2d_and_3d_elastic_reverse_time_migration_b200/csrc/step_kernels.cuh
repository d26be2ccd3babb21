// Staggered-grid velocity–stress step kernels for sm_100a.
//
// One time step is two z-streaming kernels:
//   k_stress   : sigma(n+1) = f(sigma(n), v(n)) [+ P stress tp]      (+ source)
//   k_velocity : v(n+1) = f(v(n), sigma(n+1))   [+ P velocity v_P]   (+ epilogue)
// Each CTA owns a TX x TYB column of the x–y plane and a chunk of z planes.
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

// cp.async (sm_80+ async copy, global -> shared, 4 bytes): every input of
// plane k+1 is requested while plane k is computed.
__device__ __forceinline__ void cpa4(void* sdst, const void* gsrc)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Shared-memory stage of one z plane: NV halo tiles [SH][SW], NC per-cell
// arrays [TYB][TX], NP C-PML memory variables [TYB][TX].  Two stages alternate.
template <int R, bool Y, int NV, int NC, int NP>
struct Stage {
    static constexpr int TYB = Y ? TY3 : TY2;
    static constexpr int SW = TX + 2 * R;
    static constexpr int SH = Y ? TYB + 2 * R : TYB;
    static constexpr int TILE = SH * SW;
    static constexpr int CELL = TYB * TX;
    static constexpr int FLOATS = NV * TILE + (NC + NP) * CELL;
    static constexpr size_t BYTES = 2 * sizeof(float) * FLOATS;
};

// ---------------------------------------------------------------------------
// Stress kernel
// ---------------------------------------------------------------------------
template <int R, bool Y, bool CPML, bool PS>
struct StressShape {
    static constexpr int NV = Y ? 3 : 2;                          // vx, vz, (vy)
    static constexpr int NSIG = Y ? 6 : 3;                        // txx tzz txz (tyy txy tyz)
    static constexpr int NC = NSIG + (PS ? 1 : 0) + 2;            // + tp + M + MU
    static constexpr int NP = CPML ? (Y ? 9 : 4) : 0;
    using S = Stage<R, Y, NV, NC, NP>;
};

template <int R, bool Y, bool CPML, bool PS>
__global__ void __launch_bounds__(TX * (Y ? TY3 : TY2), 1)
k_stress(const KArgs a)
{
    using SS = StressShape<R, Y, CPML, PS>;
    using S = typename SS::S;
    constexpr int TYB = S::TYB, SW = S::SW, TILE = S::TILE, CELL = S::CELL;
    constexpr int NV = SS::NV, NC = SS::NC, NSIG = SS::NSIG;
    constexpr int YO = Y ? R : 0;
    // per-cell slots
    constexpr int C_TP = NSIG, C_M = NSIG + (PS ? 1 : 0), C_MU = C_M + 1;
    extern __shared__ __align__(16) float sm[];

    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = blockIdx.x * TX + tx;
    const int j = blockIdx.y * TYB + ty;
    const int k0 = blockIdx.z * a.kchunk;
    const int k1 = min(k0 + a.kchunk, a.nz);
    const long long sy = a.sy, sz = a.sz;
    const bool act = (i < a.nx) && (j < a.ny);
    const int it = __ldg(a.it_ptr);
    const bool src_here = (it < a.nw) && (i == a.ssx) && (j == a.ssy);
    const float wsrc = (it < a.nw) ? __ldg(a.wavelet + it) : 0.f;
    const int r = ty + YO, s = tx + R, cell = ty * TX + tx;

    const float* vsrc[3] = {a.f[F_VX], a.f[F_VZ], a.f[F_VY]};
    float* sig[6] = {a.f[F_TXX], a.f[F_TZZ], a.f[F_TXZ], a.f[F_TYY], a.f[F_TXY], a.f[F_TYZ]};
    float* tp = a.f[F_TP];
    const long long cj = (long long)j * sy + i;       // column offset of (i, j)
    const long long mj = (long long)j * a.msy + i;

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
    // psi slots in the stage: x: EXX DXVZ (DXVY), y: EYY DYVX DYVZ, z: EZZ DZVX (DZVY)
    constexpr int PX = 0, PY = Y ? 3 : 2, PZ = Y ? 6 : 2;

    auto issue = [&](int p, int st, float cvx, float cvz, float cvy) {
        float* T = sm + st * S::FLOATS;
        float* Cc = T + NV * TILE;
        float* Ps = Cc + NC * CELL;
        const long long cp = (long long)p * sz + cj;
        T[0 * TILE + r * SW + s] = cvx;
        T[1 * TILE + r * SW + s] = cvz;
        if (Y) T[2 * TILE + r * SW + s] = cvy;
#pragma unroll
        for (int f = 0; f < NV; f++) {
            if (tx < R) {
                cpa4(&T[f * TILE + r * SW + tx], vsrc[f] + cp - R);
                cpa4(&T[f * TILE + r * SW + tx + TX + R], vsrc[f] + cp + TX);
            }
            if (Y && ty < R) {
                cpa4(&T[f * TILE + ty * SW + s], vsrc[f] + cp - R * sy);
                cpa4(&T[f * TILE + (ty + TYB + R) * SW + s], vsrc[f] + cp + TYB * sy);
            }
        }
        if (act) {
#pragma unroll
            for (int q = 0; q < NSIG; q++) cpa4(&Cc[q * CELL + cell], sig[q] + cp);
            if (PS) cpa4(&Cc[C_TP * CELL + cell], tp + cp);
            const long long mp = (long long)p * a.msz + mj;
            cpa4(&Cc[C_M * CELL + cell], a.M + mp);
            cpa4(&Cc[C_MU * CELL + cell], a.MU + mp);
            if (CPML) {
                if (inx) {
                    const long long x = ((long long)p * a.ny + j) * WX + slx;
                    cpa4(&Ps[(PX + 0) * CELL + cell], a.psi[P_EXX] + x);
                    cpa4(&Ps[(PX + 1) * CELL + cell], a.psi[P_DXVZ] + x);
                    if (Y) cpa4(&Ps[(PX + 2) * CELL + cell], a.psi[P_DXVY] + x);
                }
                if (iny) {
                    const long long y = ((long long)p * WY + sly) * a.nx + i;
                    cpa4(&Ps[(PY + 0) * CELL + cell], a.psi[P_EYY] + y);
                    cpa4(&Ps[(PY + 1) * CELL + cell], a.psi[P_DYVX] + y);
                    cpa4(&Ps[(PY + 2) * CELL + cell], a.psi[P_DYVZ] + y);
                }
                if (p < a.w[4] || p >= a.nz - a.w[5]) {
                    const int sl = p < a.w[4] ? p : p - a.nz + a.w[4] + a.w[5];
                    const long long z = ((long long)sl * a.ny + j) * a.nx + i;
                    cpa4(&Ps[(PZ + 0) * CELL + cell], a.psi[P_EZZ] + z);
                    cpa4(&Ps[(PZ + 1) * CELL + cell], a.psi[P_DZVX] + z);
                    if (Y) cpa4(&Ps[(PZ + 2) * CELL + cell], a.psi[P_DZVY] + z);
                }
            }
        }
        cpa_commit();
    };

    // register queues of planes k-R .. k+R
    float qx[2 * R + 1], qy[2 * R + 1], qz[2 * R + 1];
#pragma unroll
    for (int q = 0; q <= 2 * R; q++) {
        const long long cc = (long long)(k0 + q - R) * sz + cj;
        qx[q] = vsrc[0][cc];
        qz[q] = vsrc[1][cc];
        if (Y) qy[q] = vsrc[2][cc];
    }
    issue(k0, 0, qx[R], qz[R], Y ? qy[R] : 0.f);
    cpa_wait_all();
    __syncthreads();

    for (int k = k0; k < k1; ++k) {
        const int st = (k - k0) & 1;
        const bool more = (k + 1 < k1);
        float fx = 0.f, fy = 0.f, fz = 0.f;
        if (more) {
            const long long cn = (long long)(k + 1 + R) * sz + cj;
            fx = vsrc[0][cn];
            fz = vsrc[1][cn];
            if (Y) fy = vsrc[2][cn];
            issue(k + 1, st ^ 1, qx[R + 1], qz[R + 1], Y ? qy[R + 1] : 0.f);
        }
        const float* T = sm + st * S::FLOATS;
        const float* Cc = T + NV * TILE;
        const float* Ps = Cc + NC * CELL;
        const float* Tx = T;
        const float* Tz = T + TILE;
        const float* Ty = T + 2 * TILE;

        float exx = 0.f, dxvz = 0.f, dxvy = 0.f, eyy = 0.f, dyvx = 0.f, dyvz = 0.f;
        float ezz = 0.f, dzvx = 0.f, dzvy = 0.f;
#pragma unroll
        for (int n = 1; n <= R; n++) {
            exx = fmaf(a.cx[n], Tx[r * SW + s + n] - Tx[r * SW + s - n + 1], exx);
            dxvz = fmaf(a.cx[n], Tz[r * SW + s + n - 1] - Tz[r * SW + s - n], dxvz);
            ezz = fmaf(a.cz[n], qz[R + n - 1] - qz[R - n], ezz);
            dzvx = fmaf(a.cz[n], qx[R + n] - qx[R - n + 1], dzvx);
            if (Y) {
                dxvy = fmaf(a.cx[n], Ty[r * SW + s + n - 1] - Ty[r * SW + s - n], dxvy);
                eyy = fmaf(a.cy[n], Ty[(r + n) * SW + s] - Ty[(r - n + 1) * SW + s], eyy);
                dyvx = fmaf(a.cy[n], Tx[(r + n - 1) * SW + s] - Tx[(r - n) * SW + s], dyvx);
                dyvz = fmaf(a.cy[n], Tz[(r + n - 1) * SW + s] - Tz[(r - n) * SW + s], dyvz);
                dzvy = fmaf(a.cz[n], qy[R + n] - qy[R - n + 1], dzvy);
            }
        }

        if (act) {
            const long long c = (long long)k * sz + cj;
            if (CPML) {
                if (inx) {
                    const long long x = ((long long)k * a.ny + j) * WX + slx;
                    float p0 = fmaf(bxf, Ps[(PX + 0) * CELL + cell], axf * exx);
                    float p1 = fmaf(bxh, Ps[(PX + 1) * CELL + cell], axh * dxvz);
                    a.psi[P_EXX][x] = p0;
                    a.psi[P_DXVZ][x] = p1;
                    exx += p0;
                    dxvz += p1;
                    if (Y) {
                        float p2 = fmaf(bxh, Ps[(PX + 2) * CELL + cell], axh * dxvy);
                        a.psi[P_DXVY][x] = p2;
                        dxvy += p2;
                    }
                }
                if (iny) {
                    const long long y = ((long long)k * WY + sly) * a.nx + i;
                    float p0 = fmaf(byf, Ps[(PY + 0) * CELL + cell], ayf * eyy);
                    float p1 = fmaf(byh, Ps[(PY + 1) * CELL + cell], ayh * dyvx);
                    float p2 = fmaf(byh, Ps[(PY + 2) * CELL + cell], ayh * dyvz);
                    a.psi[P_EYY][y] = p0;
                    a.psi[P_DYVX][y] = p1;
                    a.psi[P_DYVZ][y] = p2;
                    eyy += p0;
                    dyvx += p1;
                    dyvz += p2;
                }
                if (k < a.w[4] || k >= a.nz - a.w[5]) {
                    const int sl = k < a.w[4] ? k : k - a.nz + a.w[4] + a.w[5];
                    const long long z = ((long long)sl * a.ny + j) * a.nx + i;
                    const float azf = __ldg(a.pa[2][0] + k), bzf = __ldg(a.pb[2][0] + k);
                    const float azh = __ldg(a.pa[2][1] + k), bzh = __ldg(a.pb[2][1] + k);
                    float p0 = fmaf(bzf, Ps[(PZ + 0) * CELL + cell], azf * ezz);
                    float p1 = fmaf(bzh, Ps[(PZ + 1) * CELL + cell], azh * dzvx);
                    a.psi[P_EZZ][z] = p0;
                    a.psi[P_DZVX][z] = p1;
                    ezz += p0;
                    dzvx += p1;
                    if (Y) {
                        float p2 = fmaf(bzh, Ps[(PZ + 2) * CELL + cell], azh * dzvy);
                        a.psi[P_DZVY][z] = p2;
                        dzvy += p2;
                    }
                }
            }
            float g1, g2;
            damping<Y>(a, CPML, i, j, k, g1, g2);
            const float M = Cc[C_M * CELL + cell], U = Cc[C_MU * CELL + cell];
            const float L = M - 2.f * U;
            const float dt = a.dt;
            float oxx = Cc[0 * CELL + cell], ozz = Cc[1 * CELL + cell], oxz = Cc[2 * CELL + cell];
            float oyy = 0.f, oxy = 0.f, oyz = 0.f;
            if (Y) {
                oyy = Cc[3 * CELL + cell];
                oxy = Cc[4 * CELL + cell];
                oyz = Cc[5 * CELL + cell];
            }
            if (src_here && k == a.ssz) {     // add_source_3D into txx, tyy, tzz
                oxx += wsrc;
                ozz += wsrc;
                if (Y) oyy += wsrc;
            }
            sig[0][c] = g1 * (g2 * oxx + dt * (M * exx + L * (eyy + ezz)));
            sig[1][c] = g1 * (g2 * ozz + dt * (M * ezz + L * (exx + eyy)));
            sig[2][c] = g1 * (g2 * oxz + dt * U * (dzvx + dxvz));
            if (Y) {
                sig[3][c] = g1 * (g2 * oyy + dt * (M * eyy + L * (exx + ezz)));
                sig[4][c] = g1 * (g2 * oxy + dt * U * (dyvx + dxvy));
                sig[5][c] = g1 * (g2 * oyz + dt * U * (dzvy + dyvz));
            }
            if (PS) tp[c] = g1 * (g2 * Cc[C_TP * CELL + cell] + dt * M * (exx + eyy + ezz));
        }

#pragma unroll
        for (int q = 0; q < 2 * R; q++) {
            qx[q] = qx[q + 1];
            qz[q] = qz[q + 1];
            if (Y) qy[q] = qy[q + 1];
        }
        qx[2 * R] = fx;
        qz[2 * R] = fz;
        if (Y) qy[2 * R] = fy;
        cpa_wait_all();
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Velocity kernel
// ---------------------------------------------------------------------------
template <int R, bool Y, bool CPML, int EPI>
struct VelShape {
    static constexpr bool PS = (EPI != EPI_NONE);
    // tiles: txx, txz, (txy, tyy, tyz), (tp)
    static constexpr int T_TXX = 0, T_TXZ = 1, T_TXY = 2, T_TYY = 3, T_TYZ = 4;
    static constexpr int T_TP = Y ? 5 : 2;
    static constexpr int NV = (Y ? 5 : 2) + (PS ? 1 : 0);
    // cells: vx, vz, (vy), (vxp, vzp, (vyp)), b, (excitation amp2 / time)
    static constexpr int C_VX = 0, C_VZ = 1, C_VY = 2;
    static constexpr int C_PX = Y ? 3 : 2;
    static constexpr int C_PZ = C_PX + 1, C_PY = C_PX + 2;
    static constexpr int C_B = PS ? C_PX + (Y ? 3 : 2) : C_PX;
    static constexpr int C_EX = C_B + 1;
    static constexpr int NC = C_B + 1 + (PS ? 1 : 0);
    static constexpr int NP = CPML ? (Y ? 9 : 4) : 0;
    using S = Stage<R, Y, NV, NC, NP>;
};

template <int R, bool Y, bool CPML, int EPI, bool REC>
__global__ void __launch_bounds__(TX * (Y ? TY3 : TY2), 1)
k_velocity(const KArgs a)
{
    using VS = VelShape<R, Y, CPML, EPI>;
    using S = typename VS::S;
    constexpr bool PS = VS::PS;
    constexpr int TYB = S::TYB, SW = S::SW, TILE = S::TILE, CELL = S::CELL;
    constexpr int NV = VS::NV, NC = VS::NC;
    constexpr int YO = Y ? R : 0;
    extern __shared__ __align__(16) float sm[];

    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = blockIdx.x * TX + tx;
    const int j = blockIdx.y * TYB + ty;
    const int k0 = blockIdx.z * a.kchunk;
    const int k1 = min(k0 + a.kchunk, a.nz);
    const long long sy = a.sy, sz = a.sz;
    const bool act = (i < a.nx) && (j < a.ny);
    const int it = __ldg(a.it_ptr);
    const int rec = ((REC || EPI == EPI_IMAGE) && act) ? receiver_index(a, i, j) : -1;
    const long long nrec = (long long)a.nrx * a.nry;
    const int r = ty + YO, s = tx + R, cell = ty * TX + tx;
    const long long cj = (long long)j * sy + i;
    const long long mj = (long long)j * a.msy + i;

    const float* txx = a.f[F_TXX];
    const float* tyy = a.f[F_TYY];
    const float* tzz = a.f[F_TZZ];
    const float* txy = a.f[F_TXY];
    const float* txz = a.f[F_TXZ];
    const float* tyz = a.f[F_TYZ];
    const float* tp = a.f[F_TP];
    float* vx = a.f[F_VX];
    float* vy = a.f[F_VY];
    float* vz = a.f[F_VZ];
    float* vxp = a.f[F_VXP];
    float* vyp = a.f[F_VYP];
    float* vzp = a.f[F_VZP];

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

    auto issue = [&](int p, int st, float cxz, float cyz, float ctp) {
        float* T = sm + st * S::FLOATS;
        float* Cc = T + NV * TILE;
        float* Ps = Cc + NC * CELL;
        const long long cp = (long long)p * sz + cj;
        // centres: from the z queues where there is one, else copied
        T[VS::T_TXZ * TILE + r * SW + s] = cxz;
        cpa4(&T[VS::T_TXX * TILE + r * SW + s], txx + cp);
        if (Y) {
            T[VS::T_TYZ * TILE + r * SW + s] = cyz;
            cpa4(&T[VS::T_TXY * TILE + r * SW + s], txy + cp);
            cpa4(&T[VS::T_TYY * TILE + r * SW + s], tyy + cp);
        }
        if (PS) T[VS::T_TP * TILE + r * SW + s] = ctp;
        if (tx < R) {   // x halos: txx, txz, (txy), (tp)
            cpa4(&T[VS::T_TXX * TILE + r * SW + tx], txx + cp - R);
            cpa4(&T[VS::T_TXX * TILE + r * SW + tx + TX + R], txx + cp + TX);
            cpa4(&T[VS::T_TXZ * TILE + r * SW + tx], txz + cp - R);
            cpa4(&T[VS::T_TXZ * TILE + r * SW + tx + TX + R], txz + cp + TX);
            if (Y) {
                cpa4(&T[VS::T_TXY * TILE + r * SW + tx], txy + cp - R);
                cpa4(&T[VS::T_TXY * TILE + r * SW + tx + TX + R], txy + cp + TX);
            }
            if (PS) {
                cpa4(&T[VS::T_TP * TILE + r * SW + tx], tp + cp - R);
                cpa4(&T[VS::T_TP * TILE + r * SW + tx + TX + R], tp + cp + TX);
            }
        }
        if (Y && ty < R) {   // y halos: txy, tyy, tyz, (tp)
            const long long lo = cp - R * sy, hi = cp + TYB * sy;
            const int rl = ty * SW + s, rh = (ty + TYB + R) * SW + s;
            cpa4(&T[VS::T_TXY * TILE + rl], txy + lo);
            cpa4(&T[VS::T_TXY * TILE + rh], txy + hi);
            cpa4(&T[VS::T_TYY * TILE + rl], tyy + lo);
            cpa4(&T[VS::T_TYY * TILE + rh], tyy + hi);
            cpa4(&T[VS::T_TYZ * TILE + rl], tyz + lo);
            cpa4(&T[VS::T_TYZ * TILE + rh], tyz + hi);
            if (PS) {
                cpa4(&T[VS::T_TP * TILE + rl], tp + lo);
                cpa4(&T[VS::T_TP * TILE + rh], tp + hi);
            }
        }
        if (act) {
            cpa4(&Cc[VS::C_VX * CELL + cell], vx + cp);
            cpa4(&Cc[VS::C_VZ * CELL + cell], vz + cp);
            if (Y) cpa4(&Cc[VS::C_VY * CELL + cell], vy + cp);
            if (PS) {
                cpa4(&Cc[VS::C_PX * CELL + cell], vxp + cp);
                cpa4(&Cc[VS::C_PZ * CELL + cell], vzp + cp);
                if (Y) cpa4(&Cc[VS::C_PY * CELL + cell], vyp + cp);
            }
            cpa4(&Cc[VS::C_B * CELL + cell], a.B + (long long)p * a.msz + mj);
            if (EPI == EPI_EXCITE) cpa4(&Cc[VS::C_EX * CELL + cell], a.ex_amp2 + cp);
            if (EPI == EPI_IMAGE) cpa4(&Cc[VS::C_EX * CELL + cell], a.ex_time + cp);
            if (CPML) {
                if (inx) {
                    const long long x = ((long long)p * a.ny + j) * WX + slx;
                    cpa4(&Ps[(PX + 0) * CELL + cell], a.psi[P_DXTXX] + x);
                    cpa4(&Ps[(PX + 1) * CELL + cell], a.psi[P_DXTXZ] + x);
                    if (Y) cpa4(&Ps[(PX + 2) * CELL + cell], a.psi[P_DXTXY] + x);
                }
                if (iny) {
                    const long long y = ((long long)p * WY + sly) * a.nx + i;
                    cpa4(&Ps[(PY + 0) * CELL + cell], a.psi[P_DYTXY] + y);
                    cpa4(&Ps[(PY + 1) * CELL + cell], a.psi[P_DYTYY] + y);
                    cpa4(&Ps[(PY + 2) * CELL + cell], a.psi[P_DYTYZ] + y);
                }
                if (p < a.w[4] || p >= a.nz - a.w[5]) {
                    const int sl = p < a.w[4] ? p : p - a.nz + a.w[4] + a.w[5];
                    const long long z = ((long long)sl * a.ny + j) * a.nx + i;
                    cpa4(&Ps[(PZ + 0) * CELL + cell], a.psi[P_DZTXZ] + z);
                    cpa4(&Ps[(PZ + 1) * CELL + cell], a.psi[P_DZTZZ] + z);
                    if (Y) cpa4(&Ps[(PZ + 2) * CELL + cell], a.psi[P_DZTYZ] + z);
                }
            }
        }
        cpa_commit();
    };

    float qxz[2 * R + 1], qyz[2 * R + 1], qzz[2 * R + 1], qtp[2 * R + 1];
#pragma unroll
    for (int q = 0; q <= 2 * R; q++) {
        const long long cc = (long long)(k0 + q - R) * sz + cj;
        qxz[q] = txz[cc];
        qzz[q] = tzz[cc];
        if (Y) qyz[q] = tyz[cc];
        if (PS) qtp[q] = tp[cc];
    }
    issue(k0, 0, qxz[R], Y ? qyz[R] : 0.f, PS ? qtp[R] : 0.f);
    cpa_wait_all();
    __syncthreads();

    for (int k = k0; k < k1; ++k) {
        const int st = (k - k0) & 1;
        const bool more = (k + 1 < k1);
        float f_xz = 0.f, f_yz = 0.f, f_zz = 0.f, f_tp = 0.f;
        if (more) {
            const long long cn = (long long)(k + 1 + R) * sz + cj;
            f_xz = txz[cn];
            f_zz = tzz[cn];
            if (Y) f_yz = tyz[cn];
            if (PS) f_tp = tp[cn];
            issue(k + 1, st ^ 1, qxz[R + 1], Y ? qyz[R + 1] : 0.f, PS ? qtp[R + 1] : 0.f);
        }
        const float* T = sm + st * S::FLOATS;
        const float* Cc = T + NV * TILE;
        const float* Ps = Cc + NC * CELL;
        const float* Txx = T + VS::T_TXX * TILE;
        const float* Txz = T + VS::T_TXZ * TILE;
        const float* Txy = T + VS::T_TXY * TILE;
        const float* Tyy = T + VS::T_TYY * TILE;
        const float* Tyz = T + VS::T_TYZ * TILE;
        const float* Ttp = T + VS::T_TP * TILE;

        float dxtxx = 0.f, dytxy = 0.f, dztxz = 0.f;
        float dxtxy = 0.f, dytyy = 0.f, dztyz = 0.f;
        float dxtxz = 0.f, dytyz = 0.f, dztzz = 0.f;
        float dxtp = 0.f, dytp = 0.f, dztp = 0.f;
#pragma unroll
        for (int n = 1; n <= R; n++) {
            dxtxx = fmaf(a.cx[n], Txx[r * SW + s + n - 1] - Txx[r * SW + s - n], dxtxx);
            dxtxz = fmaf(a.cx[n], Txz[r * SW + s + n] - Txz[r * SW + s - n + 1], dxtxz);
            dztxz = fmaf(a.cz[n], qxz[R + n - 1] - qxz[R - n], dztxz);
            dztzz = fmaf(a.cz[n], qzz[R + n] - qzz[R - n + 1], dztzz);
            if (Y) {
                dytxy = fmaf(a.cy[n], Txy[(r + n) * SW + s] - Txy[(r - n + 1) * SW + s], dytxy);
                dxtxy = fmaf(a.cx[n], Txy[r * SW + s + n] - Txy[r * SW + s - n + 1], dxtxy);
                dytyy = fmaf(a.cy[n], Tyy[(r + n - 1) * SW + s] - Tyy[(r - n) * SW + s], dytyy);
                dztyz = fmaf(a.cz[n], qyz[R + n - 1] - qyz[R - n], dztyz);
                dytyz = fmaf(a.cy[n], Tyz[(r + n) * SW + s] - Tyz[(r - n + 1) * SW + s], dytyz);
            }
            if (PS) {
                dxtp = fmaf(a.cx[n], Ttp[r * SW + s + n - 1] - Ttp[r * SW + s - n], dxtp);
                dztp = fmaf(a.cz[n], qtp[R + n] - qtp[R - n + 1], dztp);
                if (Y) dytp = fmaf(a.cy[n], Ttp[(r + n - 1) * SW + s] - Ttp[(r - n) * SW + s], dytp);
            }
        }

        if (act) {
            const long long c = (long long)k * sz + cj;
            if (CPML) {
                if (inx) {
                    const long long x = ((long long)k * a.ny + j) * WX + slx;
                    float p0 = fmaf(bxh, Ps[(PX + 0) * CELL + cell], axh * dxtxx);
                    float p1 = fmaf(bxf, Ps[(PX + 1) * CELL + cell], axf * dxtxz);
                    a.psi[P_DXTXX][x] = p0;
                    a.psi[P_DXTXZ][x] = p1;
                    dxtxx += p0;
                    dxtxz += p1;
                    if (Y) {
                        float p2 = fmaf(bxf, Ps[(PX + 2) * CELL + cell], axf * dxtxy);
                        a.psi[P_DXTXY][x] = p2;
                        dxtxy += p2;
                    }
                }
                if (iny) {
                    const long long y = ((long long)k * WY + sly) * a.nx + i;
                    float p0 = fmaf(byf, Ps[(PY + 0) * CELL + cell], ayf * dytxy);
                    float p1 = fmaf(byh, Ps[(PY + 1) * CELL + cell], ayh * dytyy);
                    float p2 = fmaf(byf, Ps[(PY + 2) * CELL + cell], ayf * dytyz);
                    a.psi[P_DYTXY][y] = p0;
                    a.psi[P_DYTYY][y] = p1;
                    a.psi[P_DYTYZ][y] = p2;
                    dytxy += p0;
                    dytyy += p1;
                    dytyz += p2;
                }
                if (k < a.w[4] || k >= a.nz - a.w[5]) {
                    const int sl = k < a.w[4] ? k : k - a.nz + a.w[4] + a.w[5];
                    const long long z = ((long long)sl * a.ny + j) * a.nx + i;
                    const float azf = __ldg(a.pa[2][0] + k), bzf = __ldg(a.pb[2][0] + k);
                    const float azh = __ldg(a.pa[2][1] + k), bzh = __ldg(a.pb[2][1] + k);
                    float p0 = fmaf(bzf, Ps[(PZ + 0) * CELL + cell], azf * dztxz);
                    float p1 = fmaf(bzh, Ps[(PZ + 1) * CELL + cell], azh * dztzz);
                    a.psi[P_DZTXZ][z] = p0;
                    a.psi[P_DZTZZ][z] = p1;
                    dztxz += p0;
                    dztzz += p1;
                    if (Y) {
                        float p2 = fmaf(bzf, Ps[(PZ + 2) * CELL + cell], azf * dztyz);
                        a.psi[P_DZTYZ][z] = p2;
                        dztyz += p2;
                    }
                }
            }
            float g1, g2;
            damping<Y>(a, CPML, i, j, k, g1, g2);
            const float b = Cc[VS::C_B * CELL + cell];
            const float db = a.dt * b;
            float nvx = g1 * (g2 * Cc[VS::C_VX * CELL + cell] + db * (dxtxx + dytxy + dztxz));
            float nvz = g1 * (g2 * Cc[VS::C_VZ * CELL + cell] + db * (dxtxz + dytyz + dztzz));
            float nvy = 0.f;
            if (Y) nvy = g1 * (g2 * Cc[VS::C_VY * CELL + cell] + db * (dxtxy + dytyy + dztyz));
            float npx = 0.f, npy = 0.f, npz = 0.f;
            if (PS) {
                // decoupled P velocity from the P-stress gradient (role of fwd_vxp_vzp_3D,
                // 3D_forward_or_back_together.cu:118); S velocity = v - v_P
                npx = g1 * (g2 * Cc[VS::C_PX * CELL + cell] + db * dxtp);
                npz = g1 * (g2 * Cc[VS::C_PZ * CELL + cell] + db * dztp);
                if (Y) npy = g1 * (g2 * Cc[VS::C_PY * CELL + cell] + db * dytp);
                vxp[c] = npx;
                vzp[c] = npz;
                if (Y) vyp[c] = npy;
            }
            if (EPI == EPI_EXCITE) {
                // caculate_ex_amp_time_new (2D_elastic_RTM/elastic_2D_kernel_3.cu:30-48):
                // strict '>' keeps the earliest maximum of |v_P|
                float a2 = npx * npx + npy * npy + npz * npz;
                if (a2 > Cc[VS::C_EX * CELL + cell]) {
                    a.ex_amp2[c] = a2;
                    a.ex_time[c] = it;
                    a.ex_v[0][c] = npx;
                    if (Y) a.ex_v[1][c] = npy;
                    a.ex_v[2][c] = npz;
                    a.ex_tp[c] = qtp[R];
                }
            }
            if (EPI == EPI_IMAGE) {
                // imaging_inner_product_ex / imaging_correlation_ex
                // (2D_elastic_RTM/elastic_2D_kernel_3.cu:542-576) at it == excitation time
                if (__float_as_int(Cc[VS::C_EX * CELL + cell]) == it) {
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
            vx[c] = nvx;
            vz[c] = nvz;
            if (Y) vy[c] = nvy;
            if (REC && rec >= 0 && k == a.rz) {
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
        qxz[2 * R] = f_xz;
        qzz[2 * R] = f_zz;
        if (Y) qyz[2 * R] = f_yz;
        if (PS) qtp[2 * R] = f_tp;
        cpa_wait_all();
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Launch helpers (instantiated per R in launch_r4.cu / launch_r6.cu)
// ---------------------------------------------------------------------------
// One instantiation per kernel, so the shared-memory opt-in below is made for
// each kernel separately (the kernels all share one function type).
template <void (*K)(KArgs)>
static cudaError_t launch_dyn(dim3 grid, dim3 block, size_t smem, const KArgs& a, cudaStream_t st)
{
    // opt in to more than 48 KB of dynamic shared memory (once per kernel)
    static cudaError_t attr = cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem);
    if (attr != cudaSuccess) return attr;
    K<<<grid, block, smem, st>>>(a);
    return cudaGetLastError();
}

template <int R, bool Y, bool C, bool P>
static cudaError_t launch_stress_y(dim3 grid, dim3 block, const KArgs& a, cudaStream_t st)
{
    return launch_dyn<k_stress<R, Y, C, P>>(grid, block, StressShape<R, Y, C, P>::S::BYTES, a, st);
}

template <int R>
cudaError_t launch_stress_t(const Geom& g, const KArgs& a, bool cpml, bool ps, cudaStream_t st)
{
    const bool Y = !g.two_d;
    const int tyb = Y ? TY3 : TY2;
    dim3 block(TX, tyb);
    dim3 grid((g.nx + TX - 1) / TX, (g.ny + tyb - 1) / tyb, (g.nz + a.kchunk - 1) / a.kchunk);
    if (Y) {
        if (cpml) return ps ? launch_stress_y<R, true, true, true>(grid, block, a, st)
                            : launch_stress_y<R, true, true, false>(grid, block, a, st);
        return ps ? launch_stress_y<R, true, false, true>(grid, block, a, st)
                  : launch_stress_y<R, true, false, false>(grid, block, a, st);
    }
    if (cpml) return ps ? launch_stress_y<R, false, true, true>(grid, block, a, st)
                        : launch_stress_y<R, false, true, false>(grid, block, a, st);
    return ps ? launch_stress_y<R, false, false, true>(grid, block, a, st)
              : launch_stress_y<R, false, false, false>(grid, block, a, st);
}

template <int R, bool Y, bool C>
static cudaError_t launch_velocity_y(dim3 grid, dim3 block, const KArgs& a, int epi, bool rec,
                                     cudaStream_t st)
{
    if (epi == EPI_EXCITE)
        return launch_dyn<k_velocity<R, Y, C, EPI_EXCITE, false>>(
            grid, block, VelShape<R, Y, C, EPI_EXCITE>::S::BYTES, a, st);
    if (epi == EPI_IMAGE)
        return launch_dyn<k_velocity<R, Y, C, EPI_IMAGE, false>>(
            grid, block, VelShape<R, Y, C, EPI_IMAGE>::S::BYTES, a, st);
    if (rec)
        return launch_dyn<k_velocity<R, Y, C, EPI_NONE, true>>(
            grid, block, VelShape<R, Y, C, EPI_NONE>::S::BYTES, a, st);
    return launch_dyn<k_velocity<R, Y, C, EPI_NONE, false>>(
        grid, block, VelShape<R, Y, C, EPI_NONE>::S::BYTES, a, st);
}

template <int R>
cudaError_t launch_velocity_t(const Geom& g, const KArgs& a, bool cpml, int epi, bool rec,
                              cudaStream_t st)
{
    const bool Y = !g.two_d;
    const int tyb = Y ? TY3 : TY2;
    dim3 block(TX, tyb);
    dim3 grid((g.nx + TX - 1) / TX, (g.ny + tyb - 1) / tyb, (g.nz + a.kchunk - 1) / a.kchunk);
    if (Y) return cpml ? launch_velocity_y<R, true, true>(grid, block, a, epi, rec, st)
                       : launch_velocity_y<R, true, false>(grid, block, a, epi, rec, st);
    return cpml ? launch_velocity_y<R, false, true>(grid, block, a, epi, rec, st)
                : launch_velocity_y<R, false, false>(grid, block, a, epi, rec, st);
}

}  // namespace ertm
