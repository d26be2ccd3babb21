// Learned LSRTM preconditioner: the U-Net's tensor-core kernels (BF16 inputs,
// FP32 accumulation in tensor memory) and its small elementwise kernels.
//
// Every convolution, transposed convolution and weight gradient is one GEMM
//   D[M x N] = sum_k A[m, k] B[n, k]          (A, B BF16; D FP32 in TMEM)
// issued with tcgen05.mma (kind::f16, M = 128 rows per CTA, N = BN <= 128
// columns, K = 16 per instruction) by one thread of the CTA.  The operands are
// staged in shared memory by all 128 threads through "loaders" that gather 8
// consecutive K elements (16 bytes) of one row: an implicit im2col for 3x3
// convolutions on NHWC activations, plain rows of K-major weights, or
// MN-major gathers (8 channels of one pixel) for the weight gradients.  The
// threads copy operand chunks into a ring of 3-4 shared-memory stages with
// cp.async (zero-fill for padding), several K tiles ahead of the tensor core;
// tcgen05.commit on a per-stage mbarrier tells them when a stage may be refilled.
// After the K loop each warp reads its 32 accumulator rows from TMEM
// (tcgen05.ld 32x32b) and an epilogue functor writes them (bias, ReLU, BF16
// store, scatter of a transposed convolution, or FP32 atomics for split-K
// weight gradients).
//
// Shared-memory operand layout (K-major, no swizzle): element (r, k) of an
// R-row, 64-column stage at byte ((k / 8) * R + r) * 16 + (k % 8) * 2, i.e. the
// 8 x 16-byte core matrices of the canonical layout with SBO = 128 bytes
// (next 8 rows) and LBO = R * 16 bytes (next 8 K elements).
//
// 3x3 convolutions of layers 128 pixels wide or wider (16-channel input
// groups) skip the im2col gather: k_conv3s stages the three input rows around
// a 128-pixel output row once per channel group and feeds the nine taps as
// operand windows shifted by one pixel (16 bytes) each (see its comment).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "ertm.h"
#include "ertm_internal.cuh"

namespace {

typedef __nv_bfloat16 bf16;

constexpr int BM = 128;      // rows per CTA (tcgen05 M)
constexpr int BK = 64;       // K elements per stage
constexpr int NT = 128;      // threads per CTA
constexpr unsigned kPolls = 1u << 24;

enum NnError { NN_OK = 0, NN_WAIT = 1 };

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned n)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(su32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, unsigned parity)
{
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(su32(b)), "r"(parity)
                 : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity)
{
    for (unsigned n = 0; n < kPolls; n++)
        if (mbar_try(b, parity)) return true;
    return false;
}

// shared-memory matrix descriptor: K-major, no swizzle, LBO = lbo bytes, SBO = 128 bytes
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((128u >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version for sm_100
    return d;                  // base offset 0, legacy LBO mode, layout SWIZZLE_NONE
}

// instruction descriptor of kind::f16: BF16 x BF16 -> F32, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_bf16(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v)
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = __uint_as_float(r[q]);
}

// ---------------------------------------------------------------------------
// Operand loaders: src(r, k) is the address of 16 bytes = 8 consecutive K
// elements of row r starting at k (k % 8 == 0), or nullptr where the operand is
// zero (rows or K past the bounds, convolution padding).
// ---------------------------------------------------------------------------

// NHWC activation view: pixel p = (n*H + y)*W + x, channels [off, off+C) of a
// pixel stride of cs channels
struct Act {
    const bf16* p;
    int nb, h, w, cs, off, c;
};

// implicit im2col of a 3x3, pad-1 convolution: row = output pixel, k = tap * C + c
struct LoadConv3 {
    Act x;
    int M, K;
    static constexpr bool MN = false;
    __device__ __forceinline__ const bf16* src(int r, int k) const
    {
        if (r >= M || k >= K) return nullptr;
        const int tap = k / x.c, c = k - tap * x.c;
        const int xx = r % x.w, t = r / x.w, yy = t % x.h, n = t / x.h;
        const int sy = yy + tap / 3 - 1, sx = xx + tap % 3 - 1;
        if (sy < 0 || sy >= x.h || sx < 0 || sx >= x.w) return nullptr;
        return x.p + ((long long)(n * x.h + sy) * x.w + sx) * x.cs + x.off + c;
    }
};

// rows of a K-major matrix [rows][ld]
struct LoadRows {
    const bf16* p;
    int rows, K, ld;
    static constexpr bool MN = false;
    __device__ __forceinline__ const bf16* src(int r, int k) const
    {
        if (r >= rows || k >= K) return nullptr;
        return p + (long long)r * ld + k;
    }
};

// transposed-convolution backward input: row = low-resolution pixel (n, i, j),
// k = (a*2 + b) * C + o reads dy at (2i+a, 2j+b), channel o (dy at 2h x 2w)
struct LoadUp2 {
    Act dy;      // high-resolution view (h, w = 2x the rows' grid)
    int M, K;
    static constexpr bool MN = false;
    __device__ __forceinline__ const bf16* src(int r, int k) const
    {
        if (r >= M || k >= K) return nullptr;
        const int ab = k / dy.c, o = k - ab * dy.c;
        const int lw = dy.w / 2, lh = dy.h / 2;
        const int j = r % lw, t = r / lw, i = t % lh, n = t / lh;
        const int y = 2 * i + (ab >> 1), x = 2 * j + (ab & 1);
        return dy.p + ((long long)(n * dy.h + y) * dy.w + x) * dy.cs + dy.off + o;
    }
};

// Weight-gradient operands are staged MN-major: one 16-byte chunk holds 8
// consecutive rows (channels, contiguous in NHWC memory) at one K index (pixel),
// so the gathers stay coalesced.  operator()(r, k) returns rows r .. r+7 (r % 8 == 0).

// rows = channels of an NHWC view, k = pixel
struct LoadChanMN {
    Act a;
    int rows, P;
    static constexpr bool MN = true;
    __device__ __forceinline__ const bf16* src(int r, int k) const
    {
        if (r >= rows || k >= P) return nullptr;
        return a.p + (long long)k * a.cs + a.off + r;
    }
};

// rows = (tap, c) of the 3x3 im2col, k = output pixel
struct LoadConv3MN {
    Act x;
    int rows, P;   // rows = 9 C
    static constexpr bool MN = true;
    __device__ __forceinline__ const bf16* src(int r, int k) const
    {
        if (r >= rows || k >= P) return nullptr;
        const int tap = r / x.c, c = r - tap * x.c;
        const int xx = k % x.w, t = k / x.w, yy = t % x.h, n = t / x.h;
        const int sy = yy + tap / 3 - 1, sx = xx + tap % 3 - 1;
        if (sy < 0 || sy >= x.h || sx < 0 || sx >= x.w) return nullptr;
        return x.p + ((long long)(n * x.h + sy) * x.w + sx) * x.cs + x.off + c;
    }
};

// rows = (a, b, o) of the 2x2 up-sampling gather of dy (high resolution), k = low-res pixel
struct LoadUp2MN {
    Act dy;
    int rows, P;   // rows = 4 C
    static constexpr bool MN = true;
    __device__ __forceinline__ const bf16* src(int r, int k) const
    {
        if (r >= rows || k >= P) return nullptr;
        const int ab = r / dy.c, o = r - ab * dy.c;
        const int lw = dy.w / 2, lh = dy.h / 2;
        const int j = k % lw, t = k / lw, i = t % lh, n = t / lh;
        const int y = 2 * i + (ab >> 1), x = 2 * j + (ab & 1);
        return dy.p + ((long long)(n * dy.h + y) * dy.w + x) * dy.cs + dy.off + o;
    }
};

// ---------------------------------------------------------------------------
// Epilogues: called with 8 consecutive columns n0..n0+7 of row m
// ---------------------------------------------------------------------------
// NHWC output (bias, optional ReLU): y[m][off + n]
struct EpiAct {
    bf16* y;
    int cs, off, N, M;
    const float* bias;
    int relu;
    __device__ __forceinline__ void operator()(int m, int n0, const float* v) const
    {
        if (m >= M) return;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int n = n0 + q;
            if (n >= N) break;
            float t = v[q] + (bias ? bias[n] : 0.f);
            if (relu) t = fmaxf(t, 0.f);
            y[(long long)m * cs + off + n] = __float2bfloat16(t);
        }
    }
};

// FP32 NHWC output without activation (network output)
struct EpiF32 {
    float* y;
    int cs, N, M;
    const float* bias;
    __device__ __forceinline__ void operator()(int m, int n0, const float* v) const
    {
        if (m >= M) return;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int n = n0 + q;
            if (n >= N) break;
            y[(long long)m * cs + n] = v[q] + (bias ? bias[n] : 0.f);
        }
    }
};

// input gradient: dx[m][off + n] = acc * (x[m][off + n] > 0) when mask is given
struct EpiGrad {
    bf16* dx;
    int cs, off, N, M;
    const bf16* mask;   // activation whose ReLU produced the layer input, same view
    __device__ __forceinline__ void operator()(int m, int n0, const float* v) const
    {
        if (m >= M) return;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int n = n0 + q;
            if (n >= N) break;
            const long long i = (long long)m * cs + off + n;
            float t = v[q];
            if (mask && !(__bfloat162float(mask[i]) > 0.f)) t = 0.f;
            dx[i] = __float2bfloat16(t);
        }
    }
};

// transposed 2x2 stride-2 convolution: column n = (a*2 + b) * C + o scatters to
// the high-resolution pixel (2i+a, 2j+b) of low-resolution row m
struct EpiUp2 {
    bf16* y;
    int cs, off, C, lh, lw, M;
    const float* bias;
    int relu;
    __device__ __forceinline__ void operator()(int m, int n0, const float* v) const
    {
        if (m >= M) return;
        const int j = m % lw, t = m / lw, i = t % lh, nb = t / lh;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int n = n0 + q;
            if (n >= 4 * C) break;
            const int ab = n / C, o = n - ab * C;
            const int yy = 2 * i + (ab >> 1), xx = 2 * j + (ab & 1);
            float s = v[q] + (bias ? bias[o] : 0.f);
            if (relu) s = fmaxf(s, 0.f);
            y[((long long)(nb * 2 * lh + yy) * 2 * lw + xx) * cs + off + o] = __float2bfloat16(s);
        }
    }
};

// FP32 accumulation (split-K weight gradients): g[m][n] += acc, or g[n][m] += acc
// when trans (the GEMM ran with the operands swapped)
struct EpiAtomic {
    float* g;
    int ld, N, M;
    int trans;
    __device__ __forceinline__ void operator()(int m, int n0, const float* v) const
    {
        if (m >= M) return;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int n = n0 + q;
            if (n >= N) break;
            atomicAdd(g + (trans ? (long long)n * ld + m : (long long)m * ld + n), v[q]);
        }
    }
};

// ---------------------------------------------------------------------------
// The GEMM kernel
// ---------------------------------------------------------------------------
// ring depth: four stages up to BN = 64 (up to 72 KB), three at BN = 128 (96 KB)
template <int BN>
struct Ring {
    static constexpr int N = BN >= 128 ? 3 : 4;
};
template <int BN>
struct Smem {
    static constexpr int NS = Ring<BN>::N;
    alignas(128) uint8_t a[NS][BM * BK * 2];
    alignas(128) uint8_t b[NS][BN * BK * 2];
    uint64_t bar[NS];
    uint32_t tmem;
};

__device__ __forceinline__ void cp16(void* sdst, const void* gsrc)
{
    // 16 bytes global -> shared, asynchronous; a null source zero-fills
    const uint32_t n = gsrc ? 16u : 0u;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(su32(sdst)),
                 "l"(gsrc ? gsrc : sdst), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// stage one operand tile: rows [r0, r0 + R), K chunk [k0, k0 + 64)
template <int R, class L>
__device__ __forceinline__ void stage(uint8_t* dst, const L& ld, int r0, int k0)
{
    constexpr int CH = R * (BK / 8);   // 16-byte chunks
    if constexpr (!L::MN) {
        // K-major: chunk = 8 K elements of one row; core matrix (8 rows x 16 B)
#pragma unroll 4
        for (int q = threadIdx.x; q < CH; q += NT) {
            const int r = q % R, j = q / R;    // consecutive threads take consecutive rows
            cp16(dst + ((size_t)j * R + r) * 16, ld.src(r0 + r, k0 + j * 8));
        }
    } else {
        // MN-major: chunk = 8 rows at one K; core matrix (8 K x 16 B), same SBO / LBO
        constexpr int RG = R / 8;
#pragma unroll 4
        for (int q = threadIdx.x; q < CH; q += NT) {
            const int rg = q % RG, k = q / RG;   // consecutive threads take consecutive row groups
            cp16(dst + ((size_t)(k >> 3) * RG + rg) * 128 + (k & 7) * 16, ld.src(r0 + rg * 8, k0 + k));
        }
    }
}

template <int BN, class LA, class LB, class EP>
__global__ void __launch_bounds__(NT) k_gemm(LA la, LB lb, EP ep, int M, int N, int K, int kt_per, int* err)
{
    extern __shared__ __align__(128) uint8_t smraw[];
    Smem<BN>& S = *reinterpret_cast<Smem<BN>*>(smraw);
    constexpr int TCOLS = BN < 32 ? 32 : BN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int KT = (K + BK - 1) / BK;
    const int kt0 = blockIdx.z * kt_per, kt1 = min(KT, kt0 + kt_per);

    constexpr int NS = Smem<BN>::NS;
    if (threadIdx.x == 0) {
        for (int q = 0; q < NS; q++) mbar_init(&S.bar[q], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&S.tmem)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem;
    constexpr uint32_t IDESC = idesc_bf16(BN) | (LA::MN ? 1u << 15 : 0u) | (LB::MN ? 1u << 16 : 0u);
    bool ok = true;
    const int nu = kt1 - kt0;
    // every thread copies its chunks of K tile u into slot u % NS with cp.async, one
    // commit group per tile (empty groups keep the count uniform)
    auto issue = [&](int u) {
        if (u < nu) {
            const int sl = u % NS;
            stage<BM>(S.a[sl], la, m0, (kt0 + u) * BK);
            stage<BN>(S.b[sl], lb, n0, (kt0 + u) * BK);
        }
        cp_commit();
    };
    for (int u = 0; u < NS - 1; u++) issue(u);
    for (int u = 0; u < nu; ++u) {
        cp_wait<NS - 2>();        // this thread's copies of tile u have landed
        proxy_fence();            // ... and are visible to the tensor core's async proxy
        __syncthreads();          // ... for every thread's chunks
        const int sl = u % NS;
        if (threadIdx.x == 0 && ok) {
            tc_fence_after();
            const uint32_t a0 = su32(S.a[sl]), b0 = su32(S.b[sl]);
#pragma unroll
            for (int j = 0; j < BK / 16; j++) {
                // K step j covers the core-matrix columns 2j, 2j+1
                const uint64_t da = sdesc(a0 + (uint32_t)(2 * j * BM * 16), BM * 16);
                const uint64_t db = sdesc(b0 + (uint32_t)(2 * j * BN * 16), BN * 16);
                umma(tmem, da, db, IDESC, (u > 0 || j > 0) ? 1u : 0u);
            }
            umma_commit(&S.bar[sl]);
        }
        // refill slot (u - 1) % NS with tile u + NS - 1 once tile u-1's MMAs read it
        const int un = u + NS - 1;
        if (un < nu && u >= 1 && ok) ok = mbar_wait(&S.bar[(u - 1) % NS], ((u - 1) / NS) & 1);
        issue(ok ? un : nu);
    }
    cp_wait<0>();
    if (nu > 0 && ok) ok = mbar_wait(&S.bar[(nu - 1) % NS], ((nu - 1) / NS) & 1);
    // the other stage's last commit precedes it, so every MMA has completed;
    // the TMEM loads below are warp-collective, so the decision is block-uniform
    const bool all_ok = __syncthreads_and(ok ? 1 : 0) != 0;
    tc_fence_after();
    if (nu > 0 && all_ok) {
        const int m = m0 + warp * 32 + lane;
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c = 0; c < BN; c += 8) {
            float v[8];
            tmem_ld8(trow + c, v);
            ep(m, n0 + c, v);
        }
    }
    if (!ok && err) atomicExch(err, NN_WAIT);
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
}

template <int BN, class LA, class LB, class EP>
cudaError_t gemm_bn(const LA& la, const LB& lb, const EP& ep, int M, int N, int K, int splitk, int* err,
                    cudaStream_t st)
{
    const int KT = (K + BK - 1) / BK;
    splitk = splitk < 1 ? 1 : (splitk > KT ? KT : splitk);
    const int kt_per = (KT + splitk - 1) / splitk;
    const int gz = (KT + kt_per - 1) / kt_per;
    const size_t smem = sizeof(Smem<BN>);
    static unsigned long long opted = 0;   // devices with the opt-in made
    cudaError_t attr = ertm::smem_opt_in(k_gemm<BN, LA, LB, EP>, smem, &opted);
    if (attr != cudaSuccess) return attr;
    dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, gz);
    k_gemm<BN, LA, LB, EP><<<grid, NT, smem, st>>>(la, lb, ep, M, N, K, kt_per, err);
    return cudaGetLastError();
}

// N tile: 16 <= BN <= 128, multiple of 16 (tcgen05 M = 128 needs N % 16 == 0)
template <class LA, class LB, class EP>
cudaError_t gemm(const LA& la, const LB& lb, const EP& ep, int M, int N, int K, int splitk, int* err,
                 cudaStream_t st)
{
    if (N <= 16) return gemm_bn<16>(la, lb, ep, M, N, K, splitk, err, st);
    if (N <= 32) return gemm_bn<32>(la, lb, ep, M, N, K, splitk, err, st);
    if (N <= 64) return gemm_bn<64>(la, lb, ep, M, N, K, splitk, err, st);
    return gemm_bn<128>(la, lb, ep, M, N, K, splitk, err, st);
}

// ---------------------------------------------------------------------------
// 3x3 convolution over rows of 128 pixels, taps as shifted operand windows
// ---------------------------------------------------------------------------
// For a layer whose width is a multiple of 128 and whose input channels come in
// groups of 16, a CTA computes RO output tiles of 128 x BN: 128 consecutive
// pixels of RO consecutive image rows.  Per group of 16 input channels a stage
// holds the RO + 2 input rows around those output rows, 130 pixels each (the
// padding column on either side, zero outside the image), as planes of 16-byte
// chunks (8 channels of one pixel per chunk, plane [row][chunk]), and the
// group's weights for the nine taps.  In the K-major no-swizzle layout of
// tcgen05 an operand row is one 16-byte chunk and 8 consecutive rows form a
// core matrix, so the A operand of tap (ky, kx) for output row r is the plane of
// input row r + ky read from pixel kx on: 9 RO MMAs of K = 16 per stage read the
// staged rows in place, each output row into its own TMEM accumulator.  A stage
// copies (RO + 2) x 130 pixels of input against RO x 128 x 9 for im2col tiles,
// and the weights once for RO rows.
constexpr int CV_PX = 130;                   // pixels per staged row
constexpr int CV_PLANE = CV_PX * 16;         // bytes of one [row][chunk] plane
template <int BN, int RO>
struct ConvSmem {
    static constexpr int NS = 3;
    static constexpr int A_BYTES = (RO + 2) * 2 * CV_PLANE;   // RO + 2 rows x 2 chunks
    static constexpr int A_PAD = (A_BYTES + 127) / 128 * 128;
    alignas(128) uint8_t a[NS][A_PAD];
    alignas(128) uint8_t b[NS][9 * 2 * BN * 16];   // [tap][chunk][BN rows x 16 B]
    uint64_t bar[NS];
    uint32_t tmem;
};
// TMEM columns of RO accumulators of BN columns (a power of two, at least 32)
constexpr int conv_tcols(int n) { return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : n <= 256 ? 256 : 512; }

template <int BN, int RO, class EP>
__global__ void __launch_bounds__(NT) k_conv3s(Act x, const bf16* __restrict__ w, int N, EP ep, int* err)
{
    extern __shared__ __align__(128) uint8_t smraw[];
    ConvSmem<BN, RO>& S = *reinterpret_cast<ConvSmem<BN, RO>*>(smraw);
    constexpr int NS = ConvSmem<BN, RO>::NS;
    constexpr int TCOLS = conv_tcols(RO * BN);
    static_assert(RO * BN <= 512, "TMEM columns");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n0 = blockIdx.y * BN;
    const int tiles_x = x.w / BM, groups_y = x.h / RO;
    const int x0 = (int)(blockIdx.x % tiles_x) * BM;
    const int t1 = (int)(blockIdx.x / tiles_x);
    const int y0 = (t1 % groups_y) * RO, nb = t1 / groups_y;
    const int G = x.c / 16, ldw = 9 * x.c;
    if (threadIdx.x == 0) {
        for (int q = 0; q < NS; q++) mbar_init(&S.bar[q], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&S.tmem)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem;
    constexpr uint32_t IDESC = idesc_bf16(BN);
    bool ok = true;
    // every thread copies its 16-byte chunks of channel group g into slot g % NS,
    // one commit group per group (empty groups keep the count uniform)
    auto issue = [&](int g) {
        if (g < G) {
            uint8_t* A = S.a[g % NS];
            uint8_t* Bs = S.b[g % NS];
            const int c0 = x.off + 16 * g;
            for (int q = threadIdx.x; q < (RO + 2) * CV_PX * 2; q += NT) {
                // consecutive threads take the two chunks of consecutive pixels
                const int kc = q & 1, pr = q >> 1, dy = pr / CV_PX, px = pr - dy * CV_PX;
                const int yy = y0 + dy - 1, xx = x0 + px - 1;
                const bf16* src = (yy >= 0 && yy < x.h && xx >= 0 && xx < x.w)
                                      ? x.p + ((long long)(nb * x.h + yy) * x.w + xx) * x.cs + c0 + 8 * kc
                                      : nullptr;
                cp16(A + (dy * 2 + kc) * CV_PLANE + px * 16, src);
            }
            for (int q = threadIdx.x; q < 9 * 2 * BN; q += NT) {
                const int r = q % BN, tk = q / BN, kc = tk & 1, tap = tk >> 1;
                const bf16* src = n0 + r < N ? w + (long long)(n0 + r) * ldw + tap * x.c + 16 * g + 8 * kc : nullptr;
                cp16(Bs + (tap * 2 + kc) * BN * 16 + r * 16, src);
            }
        }
        cp_commit();
    };
    for (int g = 0; g < NS - 1; g++) issue(g);
    for (int g = 0; g < G; ++g) {
        cp_wait<NS - 2>();        // this thread's copies of group g have landed
        proxy_fence();            // ... and are visible to the tensor core's async proxy
        __syncthreads();          // ... for every thread's chunks
        const int sl = g % NS;
        if (threadIdx.x == 0 && ok) {
            tc_fence_after();
            const uint32_t a0 = su32(S.a[sl]), b0 = su32(S.b[sl]);
#pragma unroll
            for (int r = 0; r < RO; r++)
#pragma unroll
                for (int tap = 0; tap < 9; tap++) {
                    const int ky = tap / 3, kx = tap % 3;
                    const uint64_t da = sdesc(a0 + (uint32_t)((r + ky) * 2 * CV_PLANE + kx * 16), CV_PLANE);
                    const uint64_t db = sdesc(b0 + (uint32_t)(tap * 2 * BN * 16), BN * 16);
                    umma(tmem + (uint32_t)(r * BN), da, db, IDESC, (g > 0 || tap > 0) ? 1u : 0u);
                }
            umma_commit(&S.bar[sl]);
        }
        // refill slot (g - 1) % NS with group g + NS - 1 once group g-1's MMAs read it
        const int gn = g + NS - 1;
        if (gn < G && g >= 1 && ok) ok = mbar_wait(&S.bar[(g - 1) % NS], ((g - 1) / NS) & 1);
        issue(ok ? gn : G);
    }
    cp_wait<0>();
    if (G > 0 && ok) ok = mbar_wait(&S.bar[(G - 1) % NS], ((G - 1) / NS) & 1);
    // the last group's commit follows every earlier one, so every MMA has completed;
    // the TMEM loads below are warp-collective, so the decision is block-uniform
    const bool all_ok = __syncthreads_and(ok ? 1 : 0) != 0;
    tc_fence_after();
    if (G > 0 && all_ok) {
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int r = 0; r < RO; r++) {
            const int m = ((nb * x.h + y0 + r) * x.w + x0) + warp * 32 + lane;
#pragma unroll 1
            for (int c = 0; c < BN; c += 8) {
                float v[8];
                tmem_ld8(trow + (uint32_t)(r * BN + c), v);
                ep(m, n0 + c, v);
            }
        }
    }
    if (!ok && err) atomicExch(err, NN_WAIT);
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
}

// the layer fits the row kernel: width a multiple of 128, input channels in
// groups of 16 starting on a 16-byte boundary of 16-byte-aligned pixels
bool conv3s_fits(const Act& x)
{
    return x.w % BM == 0 && x.c % 16 == 0 && x.off % 8 == 0 && x.cs % 8 == 0 &&
           (reinterpret_cast<uintptr_t>(x.p) & 15) == 0;
}

template <int BN, int RO, class EP>
cudaError_t conv3s_launch(const Act& x, const bf16* w, int N, const EP& ep, int* err, cudaStream_t st)
{
    const size_t smem = sizeof(ConvSmem<BN, RO>);
    static unsigned long long opted = 0;
    cudaError_t attr = ertm::smem_opt_in(k_conv3s<BN, RO, EP>, smem, &opted);
    if (attr != cudaSuccess) return attr;
    const long long tiles = (long long)x.nb * (x.h / RO) * (x.w / BM);
    dim3 grid((unsigned)tiles, (N + BN - 1) / BN);
    k_conv3s<BN, RO, EP><<<grid, NT, smem, st>>>(x, w, N, ep, err);
    return cudaGetLastError();
}

// two output rows per CTA where the height allows (the weights are staged once
// for both), else one
template <int BN, class EP>
cudaError_t conv3s_bn(const Act& x, const bf16* w, int N, const EP& ep, int* err, cudaStream_t st)
{
    return x.h % 2 == 0 ? conv3s_launch<BN, 2>(x, w, N, ep, err, st) : conv3s_launch<BN, 1>(x, w, N, ep, err, st);
}

// 3x3 convolution of x with weights w [N][9 * x.c] (tap-major K): the row kernel
// where the layer fits it, else the implicit-im2col GEMM
template <class EP>
cudaError_t conv3(const Act& x, const bf16* w, int N, const EP& ep, int* err, cudaStream_t st)
{
    if (conv3s_fits(x)) {
        if (N <= 16) return conv3s_bn<16>(x, w, N, ep, err, st);
        if (N <= 32) return conv3s_bn<32>(x, w, N, ep, err, st);
        if (N <= 64) return conv3s_bn<64>(x, w, N, ep, err, st);
        return conv3s_bn<128>(x, w, N, ep, err, st);
    }
    const int M = x.nb * x.h * x.w, K = 9 * x.c;
    LoadConv3 la{x, M, K};
    LoadRows lb{w, N, K, K};
    return gemm(la, lb, ep, M, N, K, 1, err, st);
}

// ---------------------------------------------------------------------------
// Elementwise kernels
// ---------------------------------------------------------------------------
// 2x2 max pooling of an NHWC view into a dense NHWC output with C channels
__global__ void k_pool_fwd(Act x, bf16* y, long long n)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(q % x.c);
        long long t = q / x.c;
        const int j = (int)(t % (x.w / 2));
        t /= (x.w / 2);
        const int i = (int)(t % (x.h / 2)), nb = (int)(t / (x.h / 2));
        float m = -3.0e38f;
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++)
                m = fmaxf(m, __bfloat162float(x.p[((long long)(nb * x.h + 2 * i + a) * x.w + 2 * j + b) * x.cs + x.off + c]));
        y[q] = __float2bfloat16(m);
    }
}

// max pooling backward: the gradient goes to the first maximum of each 2x2 window;
// adds into dx (NHWC view), masked by the ReLU of x when mask != 0
__global__ void k_pool_bwd(Act x, const bf16* dy, bf16* dx, long long n, int mask)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(q % x.c);
        long long t = q / x.c;
        const int j = (int)(t % (x.w / 2));
        t /= (x.w / 2);
        const int i = (int)(t % (x.h / 2)), nb = (int)(t / (x.h / 2));
        float m = -3.0e38f;
        long long best = -1;
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) {
                const long long e = ((long long)(nb * x.h + 2 * i + a) * x.w + 2 * j + b) * x.cs + x.off + c;
                const float v = __bfloat162float(x.p[e]);
                if (v > m) { m = v; best = e; }
            }
        const float g = __bfloat162float(dy[q]);
        if (best >= 0 && (!mask || m > 0.f)) dx[best] = __float2bfloat16(__bfloat162float(dx[best]) + g);
    }
}

// bias gradient: db[o] += sum over pixels of dy[p][off + o]
__global__ void k_bias_grad(Act dy, long long P, float* db)
{
    const int o = blockIdx.y;
    float s = 0.f;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x)
        s += __bfloat162float(dy.p[p * dy.cs + dy.off + o]);
    for (int k = 16; k; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
    __shared__ float part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
        atomicAdd(db + o, t);
    }
}

// mean-squared-error gradient of an FP32 NHWC output against a target, first C
// channels of cs: g = scale (y - t) (BF16, cs channels, zero in the padding);
// loss += sum (y - t)^2
__global__ void k_mse(const float* y, const float* t, int cs, int C, long long P, float scale, bf16* g, float* loss)
{
    float acc = 0.f;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P * cs; q += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(q % cs);
        float d = 0.f;
        if (c < C) {
            d = y[q] - t[(q / cs) * C + c];
            acc += d * d;
        }
        g[q] = __float2bfloat16(scale * d);
    }
    for (int k = 16; k; k >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, k);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

// Adam on FP32 master weights; writes the BF16 copy used by the GEMMs
__global__ void k_adam(float* w, const float* g, float* m, float* v, bf16* wb, long long n, float lr, float b1,
                       float b2, float eps, float c1, float c2)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const float gq = g[q];
        const float mq = b1 * m[q] + (1.f - b1) * gq;
        const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
        m[q] = mq;
        v[q] = vq;
        const float wq = w[q] - lr * (mq / c1) / (sqrtf(vq / c2) + eps);
        w[q] = wq;
        wb[q] = __float2bfloat16(wq);
    }
}

// weight re-layouts for the input gradients:
//  conv3: W[o][tap][c] (K = 9 Ci) -> Wf[c][8 - tap][o] (K = 9 Co)
//  up2:   U[(a*2+b)*Co + o][c] (K = Ci) -> Ut[c][(a*2+b)*Co + o] (K = 4 Co)
__global__ void k_flip3(const bf16* w, bf16* wf, int co, int ci)
{
    const long long n = (long long)co * 9 * ci;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(q % ci), tap = (int)((q / ci) % 9), o = (int)(q / (9LL * ci));
        wf[((long long)c * 9 + (8 - tap)) * co + o] = w[q];
    }
}
__global__ void k_transpose(const bf16* a, bf16* t, int rows, int cols)
{
    const long long n = (long long)rows * cols;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(q % cols), r = (int)(q / cols);
        t[(long long)c * rows + r] = a[q];
    }
}
__global__ void k_f32_to_bf16(const float* a, bf16* b, long long n)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        b[q] = __float2bfloat16(a[q]);
}

int grid_of(long long n) { return (int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16); }

int rc_of(cudaError_t e) { return e == cudaSuccess ? ERTM_OK : ERTM_ECUDA; }

Act act_of(const ertm_nn_act* a)
{
    return Act{reinterpret_cast<const bf16*>(a->data), a->n, a->h, a->w, a->cstride, a->coff, a->c};
}

// the operand copies move 16-byte chunks: every matrix starts on a 16-byte boundary
bool aligned16(const void* p) { return p && ((uintptr_t)p % 16) == 0; }
bool same_grid(const ertm_nn_act* a, const ertm_nn_act* b) { return a->n == b->n && a->h == b->h && a->w == b->w; }
bool act_ok(const ertm_nn_act* a)
{
    return a && a->data && a->n > 0 && a->h > 0 && a->w > 0 && a->c > 0 && a->c % 8 == 0 && a->coff % 8 == 0 &&
           a->cstride % 8 == 0 && a->coff + a->c <= a->cstride && ((uintptr_t)a->data % 16) == 0;
}
// a ReLU mask is read at the output's own element offsets
bool mask_ok(const ertm_nn_act* mask, const ertm_nn_act* dx)
{
    return !mask || (act_ok(mask) && same_grid(mask, dx) && mask->cstride == dx->cstride && mask->coff == dx->coff &&
                     mask->c == dx->c);
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int ertm_nn_gemm(const void* a, const void* b, float* d, int M, int N, int K, int* err, void* stream)
{
    if (!aligned16(a) || !aligned16(b) || !d || M < 1 || N < 1 || K < 1 || K % 8) return ERTM_EINVAL;
    LoadRows la{reinterpret_cast<const bf16*>(a), M, K, K};
    LoadRows lb{reinterpret_cast<const bf16*>(b), N, K, K};
    EpiF32 ep{d, N, N, M, nullptr};
    return rc_of(gemm(la, lb, ep, M, N, K, 1, err, (cudaStream_t)stream));
}

int ertm_nn_conv3x3(const ertm_nn_act* x, const void* w, const float* bias, const ertm_nn_act* y, int relu,
                    float* y32, int* err, void* stream)
{
    if (!act_ok(x) || !aligned16(w) || !y || (!y32 && !act_ok(y))) return ERTM_EINVAL;
    if (y->n != x->n || y->h != x->h || y->w != x->w) return ERTM_EINVAL;
    const int M = x->n * x->h * x->w, N = y->c;
    const bf16* wb = reinterpret_cast<const bf16*>(w);
    cudaStream_t st = (cudaStream_t)stream;
    if (y32) {
        EpiF32 ep{y32, y->cstride, N, M, bias};
        return rc_of(conv3(act_of(x), wb, N, ep, err, st));
    }
    EpiAct ep{reinterpret_cast<bf16*>(const_cast<void*>(y->data)), y->cstride, y->coff, N, M, bias, relu};
    return rc_of(conv3(act_of(x), wb, N, ep, err, st));
}

int ertm_nn_conv3x3_dgrad(const ertm_nn_act* dy, const void* wflip, const ertm_nn_act* dx, const ertm_nn_act* mask,
                          int* err, void* stream)
{
    if (!act_ok(dy) || !aligned16(wflip) || !act_ok(dx) || !same_grid(dy, dx)) return ERTM_EINVAL;
    if (!mask_ok(mask, dx)) return ERTM_EINVAL;
    const int M = dy->n * dy->h * dy->w, N = dx->c;
    EpiGrad ep{reinterpret_cast<bf16*>(const_cast<void*>(dx->data)), dx->cstride, dx->coff, N, M,
               mask ? reinterpret_cast<const bf16*>(mask->data) : nullptr};
    return rc_of(conv3(act_of(dy), reinterpret_cast<const bf16*>(wflip), N, ep, err, (cudaStream_t)stream));
}

int ertm_nn_conv3x3_wgrad(const ertm_nn_act* x, const ertm_nn_act* dy, float* dw, int splitk, int* err, void* stream)
{
    if (!act_ok(x) || !act_ok(dy) || !dw) return ERTM_EINVAL;
    const int P = x->n * x->h * x->w;
    const int co = dy->c, k9 = 9 * x->c;
    LoadChanMN ld_dy{act_of(dy), co, P};
    LoadConv3MN ld_x{act_of(x), k9, P};
    cudaStream_t st = (cudaStream_t)stream;
    // the longer of the two operands takes the 128-row side of the MMA
    if (k9 > co) {
        EpiAtomic ep{dw, k9, co, k9, 1};
        return rc_of(gemm(ld_x, ld_dy, ep, k9, co, P, splitk, err, st));
    }
    EpiAtomic ep{dw, k9, k9, co, 0};
    return rc_of(gemm(ld_dy, ld_x, ep, co, k9, P, splitk, err, st));
}

int ertm_nn_up2(const ertm_nn_act* x, const void* u, const float* bias, const ertm_nn_act* y, int relu, int* err,
                void* stream)
{
    if (!act_ok(x) || !aligned16(u) || !act_ok(y) || y->h != 2 * x->h || y->w != 2 * x->w || y->n != x->n)
        return ERTM_EINVAL;
    const int M = x->n * x->h * x->w, N = 4 * y->c, K = x->c;
    Act xa = act_of(x);
    // a plain-rows view of x works only for dense channels; use the 1x1 gather otherwise
    LoadRows lb{reinterpret_cast<const bf16*>(u), N, K, K};
    EpiUp2 ep{reinterpret_cast<bf16*>(const_cast<void*>(y->data)), y->cstride, y->coff, y->c, x->h, x->w, M, bias,
              relu};
    if (x->coff == 0 && x->cstride == x->c) {
        LoadRows la{xa.p, M, K, K};
        return rc_of(gemm(la, lb, ep, M, N, K, 1, err, (cudaStream_t)stream));
    }
    return ERTM_EINVAL;
}

int ertm_nn_up2_dgrad(const ertm_nn_act* dy, const void* ut, const ertm_nn_act* dx, const ertm_nn_act* mask,
                      int* err, void* stream)
{
    if (!act_ok(dy) || !aligned16(ut) || !act_ok(dx) || dy->h != 2 * dx->h || dy->w != 2 * dx->w || dy->n != dx->n ||
        !mask_ok(mask, dx))
        return ERTM_EINVAL;
    const int M = dx->n * dx->h * dx->w, N = dx->c, K = 4 * dy->c;
    LoadUp2 la{act_of(dy), M, K};
    LoadRows lb{reinterpret_cast<const bf16*>(ut), N, K, K};
    EpiGrad ep{reinterpret_cast<bf16*>(const_cast<void*>(dx->data)), dx->cstride, dx->coff, N, M,
               mask ? reinterpret_cast<const bf16*>(mask->data) : nullptr};
    return rc_of(gemm(la, lb, ep, M, N, K, 1, err, (cudaStream_t)stream));
}

int ertm_nn_up2_wgrad(const ertm_nn_act* x, const ertm_nn_act* dy, float* du, int splitk, int* err, void* stream)
{
    if (!act_ok(x) || !act_ok(dy) || !du || dy->h != 2 * x->h || dy->w != 2 * x->w) return ERTM_EINVAL;
    const int P = x->n * x->h * x->w;
    const int c4 = 4 * dy->c, ci = x->c;
    LoadUp2MN ld_dy{act_of(dy), c4, P};
    LoadChanMN ld_x{act_of(x), ci, P};
    cudaStream_t st = (cudaStream_t)stream;
    if (ci > c4) {
        EpiAtomic ep{du, ci, c4, ci, 1};
        return rc_of(gemm(ld_x, ld_dy, ep, ci, c4, P, splitk, err, st));
    }
    EpiAtomic ep{du, ci, ci, c4, 0};
    return rc_of(gemm(ld_dy, ld_x, ep, c4, ci, P, splitk, err, st));
}

int ertm_nn_pool2(const ertm_nn_act* x, void* y, void* stream)
{
    if (!act_ok(x) || !y || x->h % 2 || x->w % 2) return ERTM_EINVAL;
    const long long n = (long long)x->n * (x->h / 2) * (x->w / 2) * x->c;
    k_pool_fwd<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(act_of(x), reinterpret_cast<bf16*>(y), n);
    return rc_of(cudaGetLastError());
}

int ertm_nn_pool2_bwd(const ertm_nn_act* x, const void* dy, const ertm_nn_act* dx, int relu_mask, void* stream)
{
    if (!act_ok(x) || !dy || !act_ok(dx) || x->h % 2 || x->w % 2) return ERTM_EINVAL;
    if (dx->cstride != x->cstride || dx->coff != x->coff || dx->c != x->c) return ERTM_EINVAL;
    const long long n = (long long)x->n * (x->h / 2) * (x->w / 2) * x->c;
    // the gradient lands at the same offsets as x's elements (same view layout)
    Act xa = act_of(x);
    bf16* dxp = reinterpret_cast<bf16*>(const_cast<void*>(dx->data));
    k_pool_bwd<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(xa, reinterpret_cast<const bf16*>(dy), dxp, n,
                                                             relu_mask);
    return rc_of(cudaGetLastError());
}

int ertm_nn_bias_grad(const ertm_nn_act* dy, float* db, void* stream)
{
    if (!act_ok(dy) || !db) return ERTM_EINVAL;
    const long long P = (long long)dy->n * dy->h * dy->w;
    dim3 grid((unsigned)std::min<long long>((P + 255) / 256, 64), dy->c);
    k_bias_grad<<<grid, 256, 0, (cudaStream_t)stream>>>(act_of(dy), P, db);
    return rc_of(cudaGetLastError());
}

int ertm_nn_mse(const float* y, const float* target, int cstride, int c, long long pixels, float scale, void* grad,
                float* loss, void* stream)
{
    if (!y || !target || !grad || !loss || c > cstride || cstride % 8) return ERTM_EINVAL;
    k_mse<<<grid_of(pixels * cstride), 256, 0, (cudaStream_t)stream>>>(y, target, cstride, c, pixels, scale,
                                                                     reinterpret_cast<bf16*>(grad), loss);
    return rc_of(cudaGetLastError());
}

int ertm_nn_adam(float* w, const float* g, float* m, float* v, void* wb, long long n, float lr, float b1, float b2,
                 float eps, int step, void* stream)
{
    if (!w || !g || !m || !v || !wb || n < 0 || step < 1) return ERTM_EINVAL;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, reinterpret_cast<bf16*>(wb), n, lr, b1, b2, eps,
                                                         c1, c2);
    return rc_of(cudaGetLastError());
}

int ertm_nn_flip3(const void* w, void* wf, int co, int ci, void* stream)
{
    if (!w || !wf || co < 1 || ci < 1) return ERTM_EINVAL;
    k_flip3<<<grid_of((long long)co * 9 * ci), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<const bf16*>(w),
                                                                             reinterpret_cast<bf16*>(wf), co, ci);
    return rc_of(cudaGetLastError());
}

int ertm_nn_transpose(const void* a, void* t, int rows, int cols, void* stream)
{
    if (!a || !t || rows < 1 || cols < 1) return ERTM_EINVAL;
    k_transpose<<<grid_of((long long)rows * cols), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const bf16*>(a), reinterpret_cast<bf16*>(t), rows, cols);
    return rc_of(cudaGetLastError());
}

int ertm_nn_to_bf16(const float* a, void* b, long long n, void* stream)
{
    if (!a || !b || n < 0) return ERTM_EINVAL;
    k_f32_to_bf16<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(a, reinterpret_cast<bf16*>(b), n);
    return rc_of(cudaGetLastError());
}

}  // extern "C"
