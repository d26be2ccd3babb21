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

// ---------------------------------------------------------------------------
// Stress kernel
// ---------------------------------------------------------------------------
template <int R, bool Y, bool CPML, bool PS>
__global__ void __launch_bounds__(TX * (Y ? TY3 : TY2))
k_stress(const KArgs a)
{
    constexpr int TYB = Y ? TY3 : TY2;
    constexpr int SW = TX + 2 * R;
    constexpr int SH = Y ? TYB + 2 * R : TYB;
    constexpr int YO = Y ? R : 0;
    __shared__ float s_vx[SH][SW];
    __shared__ float s_vz[SH][SW];
    __shared__ float s_vy[Y ? SH : 1][Y ? SW : 1];

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

    const float* __restrict__ vx = a.f[F_VX];
    const float* __restrict__ vy = a.f[F_VY];
    const float* __restrict__ vz = a.f[F_VZ];
    float* __restrict__ txx = a.f[F_TXX];
    float* __restrict__ tyy = a.f[F_TYY];
    float* __restrict__ tzz = a.f[F_TZZ];
    float* __restrict__ txy = a.f[F_TXY];
    float* __restrict__ txz = a.f[F_TXZ];
    float* __restrict__ tyz = a.f[F_TYZ];
    float* __restrict__ tp = a.f[F_TP];

    long long c = (long long)k0 * sz + (long long)j * sy + i;
    long long cm = (long long)k0 * a.msz + (long long)j * a.msy + i;

    float qx[2 * R + 1], qy[2 * R + 1], qz[2 * R + 1];
#pragma unroll
    for (int q = 0; q <= 2 * R; q++) {
        long long cc = c + (long long)(q - R) * sz;
        qx[q] = vx[cc];
        qz[q] = vz[cc];
        if (Y) qy[q] = vy[cc];
    }

    const int r = ty + YO, s = tx + R;
    for (int k = k0; k < k1; ++k) {
        // prefetch: queue fronts of the next plane, this plane's old stresses and model
        const bool more = (k + 1 < k1);
        float nx_ = 0.f, ny_ = 0.f, nz_ = 0.f;
        if (more) {
            long long cn = c + (long long)(R + 1) * sz;
            nx_ = vx[cn];
            nz_ = vz[cn];
            if (Y) ny_ = vy[cn];
        }
        float oxx = 0.f, oyy = 0.f, ozz = 0.f, oxy = 0.f, oxz = 0.f, oyz = 0.f, otp = 0.f;
        float M = 0.f, U = 0.f;
        if (act) {
            oxx = txx[c];
            ozz = tzz[c];
            oxz = txz[c];
            if (Y) {
                oyy = tyy[c];
                oxy = txy[c];
                oyz = tyz[c];
            }
            if (PS) otp = tp[c];
            M = __ldg(a.M + cm);
            U = __ldg(a.MU + cm);
        }

        // stage plane k
        s_vx[r][s] = qx[R];
        s_vz[r][s] = qz[R];
        if (Y) s_vy[r][s] = qy[R];
        if (tx < R) {
            s_vx[r][tx] = vx[c - R];
            s_vx[r][tx + TX + R] = vx[c + TX];
            s_vz[r][tx] = vz[c - R];
            s_vz[r][tx + TX + R] = vz[c + TX];
            if (Y) {
                s_vy[r][tx] = vy[c - R];
                s_vy[r][tx + TX + R] = vy[c + TX];
            }
        }
        if (Y && ty < R) {
            s_vx[ty][s] = vx[c - R * sy];
            s_vx[ty + TYB + R][s] = vx[c + TYB * sy];
            s_vy[ty][s] = vy[c - R * sy];
            s_vy[ty + TYB + R][s] = vy[c + TYB * sy];
            s_vz[ty][s] = vz[c - R * sy];
            s_vz[ty + TYB + R][s] = vz[c + TYB * sy];
        }
        __syncthreads();

        float exx = 0.f, dxvz = 0.f, dxvy = 0.f, eyy = 0.f, dyvx = 0.f, dyvz = 0.f;
        float ezz = 0.f, dzvx = 0.f, dzvy = 0.f;
#pragma unroll
        for (int n = 1; n <= R; n++) {
            exx = fmaf(a.cx[n], s_vx[r][s + n] - s_vx[r][s - n + 1], exx);
            dxvz = fmaf(a.cx[n], s_vz[r][s + n - 1] - s_vz[r][s - n], dxvz);
            ezz = fmaf(a.cz[n], qz[R + n - 1] - qz[R - n], ezz);
            dzvx = fmaf(a.cz[n], qx[R + n] - qx[R - n + 1], dzvx);
            if (Y) {
                dxvy = fmaf(a.cx[n], s_vy[r][s + n - 1] - s_vy[r][s - n], dxvy);
                eyy = fmaf(a.cy[n], s_vy[r + n][s] - s_vy[r - n + 1][s], eyy);
                dyvx = fmaf(a.cy[n], s_vx[r + n - 1][s] - s_vx[r - n][s], dyvx);
                dyvz = fmaf(a.cy[n], s_vz[r + n - 1][s] - s_vz[r - n][s], dyvz);
                dzvy = fmaf(a.cz[n], qy[R + n] - qy[R - n + 1], dzvy);
            }
        }

        if (act) {
            if (CPML) {
                const int w0 = a.w[0], w1 = a.w[1];
                if (i < w0 || i >= a.nx - w1) {
                    int sl = i < w0 ? i : i - a.nx + w0 + w1;
                    long long p = ((long long)k * a.ny + j) * (w0 + w1) + sl;
                    exx = cpml_upd(a.psi[P_EXX], p, __ldg(a.pa[0][0] + i), __ldg(a.pb[0][0] + i), exx);
                    dxvz = cpml_upd(a.psi[P_DXVZ], p, __ldg(a.pa[0][1] + i), __ldg(a.pb[0][1] + i), dxvz);
                    if (Y)
                        dxvy = cpml_upd(a.psi[P_DXVY], p, __ldg(a.pa[0][1] + i), __ldg(a.pb[0][1] + i),
                                        dxvy);
                }
                if (Y) {
                    const int w2 = a.w[2], w3 = a.w[3];
                    if (j < w2 || j >= a.ny - w3) {
                        int sl = j < w2 ? j : j - a.ny + w2 + w3;
                        long long p = ((long long)k * (w2 + w3) + sl) * a.nx + i;
                        eyy = cpml_upd(a.psi[P_EYY], p, __ldg(a.pa[1][0] + j), __ldg(a.pb[1][0] + j), eyy);
                        dyvx = cpml_upd(a.psi[P_DYVX], p, __ldg(a.pa[1][1] + j), __ldg(a.pb[1][1] + j),
                                        dyvx);
                        dyvz = cpml_upd(a.psi[P_DYVZ], p, __ldg(a.pa[1][1] + j), __ldg(a.pb[1][1] + j),
                                        dyvz);
                    }
                }
                const int w4 = a.w[4], w5 = a.w[5];
                if (k < w4 || k >= a.nz - w5) {
                    int sl = k < w4 ? k : k - a.nz + w4 + w5;
                    long long p = ((long long)sl * a.ny + j) * a.nx + i;
                    ezz = cpml_upd(a.psi[P_EZZ], p, __ldg(a.pa[2][0] + k), __ldg(a.pb[2][0] + k), ezz);
                    dzvx = cpml_upd(a.psi[P_DZVX], p, __ldg(a.pa[2][1] + k), __ldg(a.pb[2][1] + k), dzvx);
                    if (Y)
                        dzvy = cpml_upd(a.psi[P_DZVY], p, __ldg(a.pa[2][1] + k), __ldg(a.pb[2][1] + k),
                                        dzvy);
                }
            }
            float g1, g2;
            damping<Y>(a, CPML, i, j, k, g1, g2);
            const float L = M - 2.f * U;
            const float dt = a.dt;
            if (src_here && k == a.ssz) {     // add_source_3D into txx, tyy, tzz
                oxx += wsrc;
                ozz += wsrc;
                if (Y) oyy += wsrc;
            }
            txx[c] = g1 * (g2 * oxx + dt * (M * exx + L * (eyy + ezz)));
            tzz[c] = g1 * (g2 * ozz + dt * (M * ezz + L * (exx + eyy)));
            txz[c] = g1 * (g2 * oxz + dt * U * (dzvx + dxvz));
            if (Y) {
                tyy[c] = g1 * (g2 * oyy + dt * (M * eyy + L * (exx + ezz)));
                txy[c] = g1 * (g2 * oxy + dt * U * (dyvx + dxvy));
                tyz[c] = g1 * (g2 * oyz + dt * U * (dzvy + dyvz));
            }
            if (PS) tp[c] = g1 * (g2 * otp + dt * M * (exx + eyy + ezz));
        }
        __syncthreads();

#pragma unroll
        for (int q = 0; q < 2 * R; q++) {
            qx[q] = qx[q + 1];
            qz[q] = qz[q + 1];
            if (Y) qy[q] = qy[q + 1];
        }
        qx[2 * R] = nx_;
        qz[2 * R] = nz_;
        if (Y) qy[2 * R] = ny_;
        c += sz;
        cm += a.msz;
    }
}

// ---------------------------------------------------------------------------
// Velocity kernel
// ---------------------------------------------------------------------------
template <int R, bool Y, bool CPML, int EPI, bool REC>
__global__ void __launch_bounds__(TX * (Y ? TY3 : TY2))
k_velocity(const KArgs a)
{
    constexpr bool PS = (EPI != EPI_NONE);
    constexpr int TYB = Y ? TY3 : TY2;
    constexpr int SW = TX + 2 * R;
    constexpr int SH = Y ? TYB + 2 * R : TYB;
    constexpr int YO = Y ? R : 0;
    __shared__ float s_txx[SH][SW];
    __shared__ float s_txz[SH][SW];
    __shared__ float s_txy[Y ? SH : 1][Y ? SW : 1];
    __shared__ float s_tyy[Y ? SH : 1][Y ? SW : 1];
    __shared__ float s_tyz[Y ? SH : 1][Y ? SW : 1];
    __shared__ float s_tp[PS ? SH : 1][PS ? SW : 1];

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

    const float* __restrict__ txx = a.f[F_TXX];
    const float* __restrict__ tyy = a.f[F_TYY];
    const float* __restrict__ tzz = a.f[F_TZZ];
    const float* __restrict__ txy = a.f[F_TXY];
    const float* __restrict__ txz = a.f[F_TXZ];
    const float* __restrict__ tyz = a.f[F_TYZ];
    const float* __restrict__ tp = a.f[F_TP];
    float* __restrict__ vx = a.f[F_VX];
    float* __restrict__ vy = a.f[F_VY];
    float* __restrict__ vz = a.f[F_VZ];
    float* __restrict__ vxp = a.f[F_VXP];
    float* __restrict__ vyp = a.f[F_VYP];
    float* __restrict__ vzp = a.f[F_VZP];

    long long c = (long long)k0 * sz + (long long)j * sy + i;
    long long cm = (long long)k0 * a.msz + (long long)j * a.msy + i;

    float qxz[2 * R + 1], qyz[2 * R + 1], qzz[2 * R + 1], qtp[2 * R + 1];
#pragma unroll
    for (int q = 0; q <= 2 * R; q++) {
        long long cc = c + (long long)(q - R) * sz;
        qxz[q] = txz[cc];
        qzz[q] = tzz[cc];
        if (Y) qyz[q] = tyz[cc];
        if (PS) qtp[q] = tp[cc];
    }

    const int r = ty + YO, s = tx + R;
    for (int k = k0; k < k1; ++k) {
        const bool more = (k + 1 < k1);
        float n_xz = 0.f, n_yz = 0.f, n_zz = 0.f, n_tp = 0.f;
        if (more) {
            long long cn = c + (long long)(R + 1) * sz;
            n_xz = txz[cn];
            n_zz = tzz[cn];
            if (Y) n_yz = tyz[cn];
            if (PS) n_tp = tp[cn];
        }
        float ovx = 0.f, ovy = 0.f, ovz = 0.f, opx = 0.f, opy = 0.f, opz = 0.f, b = 0.f;
        if (act) {
            ovx = vx[c];
            ovz = vz[c];
            if (Y) ovy = vy[c];
            if (PS) {
                opx = vxp[c];
                opz = vzp[c];
                if (Y) opy = vyp[c];
            }
            b = __ldg(a.B + cm);
        }

        s_txx[r][s] = txx[c];
        s_txz[r][s] = qxz[R];
        if (Y) {
            s_txy[r][s] = txy[c];
            s_tyy[r][s] = tyy[c];
            s_tyz[r][s] = qyz[R];
        }
        if (PS) s_tp[r][s] = qtp[R];
        if (tx < R) {
            s_txx[r][tx] = txx[c - R];
            s_txx[r][tx + TX + R] = txx[c + TX];
            s_txz[r][tx] = txz[c - R];
            s_txz[r][tx + TX + R] = txz[c + TX];
            if (Y) {
                s_txy[r][tx] = txy[c - R];
                s_txy[r][tx + TX + R] = txy[c + TX];
            }
            if (PS) {
                s_tp[r][tx] = tp[c - R];
                s_tp[r][tx + TX + R] = tp[c + TX];
            }
        }
        if (Y && ty < R) {
            s_txy[ty][s] = txy[c - R * sy];
            s_txy[ty + TYB + R][s] = txy[c + TYB * sy];
            s_tyy[ty][s] = tyy[c - R * sy];
            s_tyy[ty + TYB + R][s] = tyy[c + TYB * sy];
            s_tyz[ty][s] = tyz[c - R * sy];
            s_tyz[ty + TYB + R][s] = tyz[c + TYB * sy];
            if (PS) {
                s_tp[ty][s] = tp[c - R * sy];
                s_tp[ty + TYB + R][s] = tp[c + TYB * sy];
            }
        }
        __syncthreads();

        float dxtxx = 0.f, dytxy = 0.f, dztxz = 0.f;
        float dxtxy = 0.f, dytyy = 0.f, dztyz = 0.f;
        float dxtxz = 0.f, dytyz = 0.f, dztzz = 0.f;
        float dxtp = 0.f, dytp = 0.f, dztp = 0.f;
#pragma unroll
        for (int n = 1; n <= R; n++) {
            dxtxx = fmaf(a.cx[n], s_txx[r][s + n - 1] - s_txx[r][s - n], dxtxx);
            dxtxz = fmaf(a.cx[n], s_txz[r][s + n] - s_txz[r][s - n + 1], dxtxz);
            dztxz = fmaf(a.cz[n], qxz[R + n - 1] - qxz[R - n], dztxz);
            dztzz = fmaf(a.cz[n], qzz[R + n] - qzz[R - n + 1], dztzz);
            if (Y) {
                dytxy = fmaf(a.cy[n], s_txy[r + n][s] - s_txy[r - n + 1][s], dytxy);
                dxtxy = fmaf(a.cx[n], s_txy[r][s + n] - s_txy[r][s - n + 1], dxtxy);
                dytyy = fmaf(a.cy[n], s_tyy[r + n - 1][s] - s_tyy[r - n][s], dytyy);
                dztyz = fmaf(a.cz[n], qyz[R + n - 1] - qyz[R - n], dztyz);
                dytyz = fmaf(a.cy[n], s_tyz[r + n][s] - s_tyz[r - n + 1][s], dytyz);
            }
            if (PS) {
                dxtp = fmaf(a.cx[n], s_tp[r][s + n - 1] - s_tp[r][s - n], dxtp);
                dztp = fmaf(a.cz[n], qtp[R + n] - qtp[R - n + 1], dztp);
                if (Y) dytp = fmaf(a.cy[n], s_tp[r + n - 1][s] - s_tp[r - n][s], dytp);
            }
        }

        if (act) {
            if (CPML) {
                const int w0 = a.w[0], w1 = a.w[1];
                if (i < w0 || i >= a.nx - w1) {
                    int sl = i < w0 ? i : i - a.nx + w0 + w1;
                    long long p = ((long long)k * a.ny + j) * (w0 + w1) + sl;
                    dxtxx = cpml_upd(a.psi[P_DXTXX], p, __ldg(a.pa[0][1] + i), __ldg(a.pb[0][1] + i),
                                     dxtxx);
                    dxtxz = cpml_upd(a.psi[P_DXTXZ], p, __ldg(a.pa[0][0] + i), __ldg(a.pb[0][0] + i),
                                     dxtxz);
                    if (Y)
                        dxtxy = cpml_upd(a.psi[P_DXTXY], p, __ldg(a.pa[0][0] + i),
                                         __ldg(a.pb[0][0] + i), dxtxy);
                }
                if (Y) {
                    const int w2 = a.w[2], w3 = a.w[3];
                    if (j < w2 || j >= a.ny - w3) {
                        int sl = j < w2 ? j : j - a.ny + w2 + w3;
                        long long p = ((long long)k * (w2 + w3) + sl) * a.nx + i;
                        dytxy = cpml_upd(a.psi[P_DYTXY], p, __ldg(a.pa[1][0] + j),
                                         __ldg(a.pb[1][0] + j), dytxy);
                        dytyy = cpml_upd(a.psi[P_DYTYY], p, __ldg(a.pa[1][1] + j),
                                         __ldg(a.pb[1][1] + j), dytyy);
                        dytyz = cpml_upd(a.psi[P_DYTYZ], p, __ldg(a.pa[1][0] + j),
                                         __ldg(a.pb[1][0] + j), dytyz);
                    }
                }
                const int w4 = a.w[4], w5 = a.w[5];
                if (k < w4 || k >= a.nz - w5) {
                    int sl = k < w4 ? k : k - a.nz + w4 + w5;
                    long long p = ((long long)sl * a.ny + j) * a.nx + i;
                    dztxz = cpml_upd(a.psi[P_DZTXZ], p, __ldg(a.pa[2][0] + k), __ldg(a.pb[2][0] + k),
                                     dztxz);
                    dztzz = cpml_upd(a.psi[P_DZTZZ], p, __ldg(a.pa[2][1] + k), __ldg(a.pb[2][1] + k),
                                     dztzz);
                    if (Y)
                        dztyz = cpml_upd(a.psi[P_DZTYZ], p, __ldg(a.pa[2][0] + k),
                                         __ldg(a.pb[2][0] + k), dztyz);
                }
            }
            float g1, g2;
            damping<Y>(a, CPML, i, j, k, g1, g2);
            const float db = a.dt * b;
            float nvx = g1 * (g2 * ovx + db * (dxtxx + dytxy + dztxz));
            float nvz = g1 * (g2 * ovz + db * (dxtxz + dytyz + dztzz));
            float nvy = 0.f;
            if (Y) nvy = g1 * (g2 * ovy + db * (dxtxy + dytyy + dztyz));
            float npx = 0.f, npy = 0.f, npz = 0.f;
            if (PS) {
                // decoupled P velocity from the P-stress gradient (role of fwd_vxp_vzp_3D,
                // 3D_forward_or_back_together.cu:118); S velocity = v - v_P
                npx = g1 * (g2 * opx + db * dxtp);
                npz = g1 * (g2 * opz + db * dztp);
                if (Y) npy = g1 * (g2 * opy + db * dytp);
                vxp[c] = npx;
                vzp[c] = npz;
                if (Y) vyp[c] = npy;
            }
            if (EPI == EPI_EXCITE) {
                // caculate_ex_amp_time_new (2D_elastic_RTM/elastic_2D_kernel_3.cu:30-48):
                // strict '>' keeps the earliest maximum of |v_P|
                float a2 = npx * npx + npy * npy + npz * npz;
                if (a2 > a.ex_amp2[c]) {
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
                if (a.ex_time[c] == it) {
                    float ex = a.ex_v[0][c], ey = Y ? a.ex_v[1][c] : 0.f, ez = a.ex_v[2][c];
                    float den = ex * ex + ey * ey + ez * ez;
                    if (den > 0.f) {
                        float inv = 1.f / den;
                        if (a.img[0]) a.img[0][c] = (ex * npx + ey * npy + ez * npz) * inv;
                        if (a.img[1])
                            a.img[1][c] = (ex * (nvx - npx) + ey * (nvy - npy) + ez * (nvz - npz)) * inv;
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
        __syncthreads();

#pragma unroll
        for (int q = 0; q < 2 * R; q++) {
            qxz[q] = qxz[q + 1];
            qzz[q] = qzz[q + 1];
            if (Y) qyz[q] = qyz[q + 1];
            if (PS) qtp[q] = qtp[q + 1];
        }
        qxz[2 * R] = n_xz;
        qzz[2 * R] = n_zz;
        if (Y) qyz[2 * R] = n_yz;
        if (PS) qtp[2 * R] = n_tp;
        c += sz;
        cm += a.msz;
    }
}

// ---------------------------------------------------------------------------
// Launch helpers (instantiated per R in launch_r4.cu / launch_r6.cu)
// ---------------------------------------------------------------------------
template <int R>
cudaError_t launch_stress_t(const Geom& g, const KArgs& a, bool cpml, bool ps, cudaStream_t st)
{
    const bool Y = !g.two_d;
    const int tyb = Y ? TY3 : TY2;
    dim3 block(TX, tyb);
    dim3 grid((g.nx + TX - 1) / TX, (g.ny + tyb - 1) / tyb, (g.nz + a.kchunk - 1) / a.kchunk);
#define ERTM_S(YY, CC, PP) k_stress<R, YY, CC, PP><<<grid, block, 0, st>>>(a)
    if (Y) {
        if (cpml) { if (ps) ERTM_S(true, true, true); else ERTM_S(true, true, false); }
        else { if (ps) ERTM_S(true, false, true); else ERTM_S(true, false, false); }
    } else {
        if (cpml) { if (ps) ERTM_S(false, true, true); else ERTM_S(false, true, false); }
        else { if (ps) ERTM_S(false, false, true); else ERTM_S(false, false, false); }
    }
#undef ERTM_S
    return cudaGetLastError();
}

template <int R, bool Y, bool C>
static cudaError_t launch_velocity_y(dim3 grid, dim3 block, const KArgs& a, int epi, bool rec,
                                     cudaStream_t st)
{
    if (epi == EPI_EXCITE) k_velocity<R, Y, C, EPI_EXCITE, false><<<grid, block, 0, st>>>(a);
    else if (epi == EPI_IMAGE) k_velocity<R, Y, C, EPI_IMAGE, false><<<grid, block, 0, st>>>(a);
    else if (rec) k_velocity<R, Y, C, EPI_NONE, true><<<grid, block, 0, st>>>(a);
    else k_velocity<R, Y, C, EPI_NONE, false><<<grid, block, 0, st>>>(a);
    return cudaGetLastError();
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
