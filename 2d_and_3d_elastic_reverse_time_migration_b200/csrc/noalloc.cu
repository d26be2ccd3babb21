// Observed-data modelling without any device allocation.
//
// ertm_forward_together_using_real_model_noalloc runs the same modelling pass
// as ertm_forward_together_using_real_model, but every buffer it needs beyond
// the caller's inputs and outputs (wavefields, model products, absorbing-layer
// profiles and memory variables, the step counter, the wavelet copy) lives in
// one file-scope device array of fixed size.  It is meant for callers that are
// not allowed to allocate device memory when they call in: plugin hosts whose
// execute step forbids allocation, real-time pipelines that fix their memory at
// start-up, and frameworks whose own allocator owns the GPU (an allocation
// behind its back fragments or exhausts its pool).  Such callers allocate the
// inputs and the output themselves and pass device pointers.
//
// Limits and rules, all enforced or documented here:
//  * the scratch array is kNoAllocBytes (64 MiB); a grid whose padded state
//    does not fit is rejected with ERTM_EINVAL and a message giving the need;
//  * every GPU that loads this file's module holds the array until exit;
//  * the array's device address is looked up once per device, on the first
//    call made with that device current (cudaGetSymbolAddress), and again
//    after the device's context changed (a device reset); make that first
//    call before any stream capture on the device;
//  * all calls share the array: calls that overlap on the GPU (two streams,
//    two host threads) race and give wrong results; the caller serialises them;
//  * the state is cleared at the start of every call, so the array's previous
//    contents never leak into a result.
// No cudaMalloc, cudaFree or allocating library routine is called.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "ertm.h"
#include "ertm_internal.cuh"

using namespace ertm;

namespace {

constexpr size_t kNoAllocBytes = size_t(64) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};
CUcontext g_scratch_ctx[kMaxDevices] = {nullptr};

thread_local char g_noalloc_err[512];

int nfail(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_noalloc_err, sizeof g_noalloc_err, fmt, ap);
    va_end(ap);
    return code;
}

// the CUDA context current on this thread (driver entry point, no -lcuda needed)
CUcontext current_context()
{
    static PFN_cuCtxGetCurrent_v4000 get = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return (PFN_cuCtxGetCurrent_v4000)p;
    }();
    CUcontext ctx = nullptr;
    if (!get || get(&ctx) != CUDA_SUCCESS) return nullptr;
    return ctx;
}

// Device address of the scratch array in the current context of device `dev`.
// The lookup (cudaGetSymbolAddress) is cached per device together with the
// context it was made in: after the caller resets the device, its new primary
// context loads the module afresh and the lookup is repeated.
int scratch_base(int dev, unsigned char** out)
{
    if (dev < 0 || dev >= kMaxDevices) return nfail(ERTM_EINVAL, "device %d not supported", dev);
    const CUcontext ctx = current_context();
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[dev] || !ctx || g_scratch_ctx[dev] != ctx) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return nfail(ERTM_ECUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
        g_scratch_ctx[dev] = ctx;
    }
    *out = static_cast<unsigned char*>(g_scratch_ptr[dev]);
    return ERTM_OK;
}

// a pointer the kernels on `dev` may use: device memory of that GPU, or managed memory
bool on_device(const void* p, int dev)
{
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (at.type == cudaMemoryTypeManaged) return true;
    return at.type == cudaMemoryTypeDevice && at.device == dev;
}

// bump allocator over the scratch array (256-byte aligned sub-buffers)
struct Carve {
    unsigned char* base;
    size_t used = 0;
    template <typename T>
    T* take(size_t n)
    {
        size_t off = (used + 255) & ~size_t(255);
        used = off + n * sizeof(T);
        return reinterpret_cast<T*>(base + off);
    }
};

int encode(CUtensorMap* m, const void* base, const Geom& g, int bx, int by)
{
    static PFN_cuTensorMapEncodeTiled_v12000 enc = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                             &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return (PFN_cuTensorMapEncodeTiled_v12000)p;
    }();
    if (!enc) return nfail(ERTM_ECUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)g.py, (cuuint64_t)g.pz};
    cuuint64_t strides[2] = {(cuuint64_t)g.px * 4, (cuuint64_t)(g.px * g.py) * 4};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims, strides,
                     box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return nfail(ERTM_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return ERTM_OK;
}

// largest |vp| of the caller's contiguous model, into *out (float bits, non-negative)
__global__ void k_noalloc_absmax(const float* __restrict__ v, long long n, float* out)
{
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(v[i]));
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax((int*)out, __float_as_int(m));
}

#define NCK(call)                                                                       \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return nfail(ERTM_ECUDA, "%s: %s", #call, cudaGetErrorString(e_));          \
    } while (0)

}  // namespace

namespace {

int run_noalloc(const ertm_config* cfg, const float* vp, const float* vs, const float* rho,
                const ertm_shot* s, float* data_out, void* stream)
{
    if (!cfg || !s) return nfail(ERTM_EINVAL, "config or shot is NULL");
    const ertm_config& c = *cfg;
    if (c.nx < 1 || c.ny < 1 || c.nz < 1 || !(c.dx > 0) || !(c.dy > 0) || !(c.dz > 0) ||
        !(c.dt_ms > 0) || c.nt < 1)
        return nfail(ERTM_EINVAL, "bad grid, spacing, dt or nt");
    if (c.order != 8 && c.order != 12) return nfail(ERTM_ENOTSUP, "order %d", c.order);
    if (c.boundary < 0 || c.boundary > 2 || c.coef_kind < 0 || c.coef_kind > 2)
        return nfail(ERTM_EINVAL, "boundary or coefficient kind");
    if (c.coef_kind == ERTM_COEF_REFERENCE12 && c.order != 12)
        return nfail(ERTM_EINVAL, "reference coefficients need order 12");
    const bool two_d = (c.ny == 1);
    const int ns[3] = {c.nx, c.ny, c.nz};
    for (int ax = 0; ax < 3; ax++) {
        if (c.pml[2 * ax] < 0 || c.pml[2 * ax + 1] < 0) return nfail(ERTM_EINVAL, "negative width");
        if (ax == 1 && two_d) continue;
        if (c.pml[2 * ax] + c.pml[2 * ax + 1] > ns[ax]) return nfail(ERTM_EINVAL, "widths exceed grid");
        if (c.boundary != ERTM_BOUNDARY_CPML && (c.pml[2 * ax] == 1 || c.pml[2 * ax + 1] == 1))
            return nfail(ERTM_EINVAL, "sponge widths must be 0 or >= 2");
    }
    if (s->sx < 0 || s->sx >= c.nx || s->sy < 0 || s->sy >= c.ny || s->sz < 0 || s->sz >= c.nz)
        return nfail(ERTM_EINVAL, "source cell outside the grid");
    if (s->nw < 0 || (s->nw > 0 && !s->wavelet) || s->nrx < 0 || s->nry < 0 || s->drx <= 0 ||
        s->dry <= 0)
        return nfail(ERTM_EINVAL, "bad wavelet or receiver grid");
    if (two_d && (s->nry > 1 || s->ry0 != 0 || s->sy != 0))
        return nfail(ERTM_EINVAL, "2D grid: receivers and source must sit at y = 0");
    const long long nrec = (long long)s->nrx * s->nry;
    if (c.device < 0) return nfail(ERTM_EINVAL, "device %d", c.device);
    const int dv = c.device;
    if (!on_device(vp, dv) || !on_device(vs, dv) || !on_device(rho, dv) ||
        (nrec > 0 && !on_device(data_out, dv)) || (s->nw > 0 && !on_device(s->wavelet, dv)))
        return nfail(ERTM_EINVAL, "vp, vs, rho, wavelet and data_out must be memory of device %d "
                     "(cudaMalloc on that device, or managed)", dv);
    NCK(cudaSetDevice(c.device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // geometry of the padded volumes (same layout as the context path)
    const int R = c.order / 2;
    const Geom g = make_geom(c.nx, c.ny, c.nz, R);

    // scratch plan: wavefields, model products, profiles, memory variables, counters
    static const int kAxis[NPSI] = {0, 1, 2, 1, 0, 2, 0, 2, 1, 0, 1, 2, 0, 1, 2, 0, 1, 2};
    static const bool k2D[NPSI] = {true, false, true, false, false, true, true, false, false,
                                   true, false, true, false, false, false, true, false, true};
    const int fields3[9] = {F_VX, F_VY, F_VZ, F_TXX, F_TYY, F_TZZ, F_TXY, F_TXZ, F_TYZ};
    const int fields2[5] = {F_VX, F_VZ, F_TXX, F_TZZ, F_TXZ};
    const int nf = two_d ? 5 : 9;
    const int* fl = two_d ? fields2 : fields3;
    const bool cpml = c.boundary == ERTM_BOUNDARY_CPML;
    long long psi_n[NPSI] = {0};
    size_t need = 0;
    {
        auto add = [&](size_t bytes) { need = ((need + 255) & ~size_t(255)) + bytes; };
        for (int q = 0; q < nf + 3; q++) add(4 * (size_t)g.total);
        for (int ax = 0; ax < 3; ax++) add(4 * 4 * (size_t)ns[ax] + 3 * 256);
        if (cpml)
            for (int p = 0; p < NPSI; p++) {
                if (two_d && !k2D[p]) continue;
                int ax = kAxis[p];
                long long w = c.pml[2 * ax] + c.pml[2 * ax + 1];
                psi_n[p] = ax == 0 ? (long long)c.nz * c.ny * w
                         : ax == 1 ? (long long)c.nz * w * c.nx
                                   : w * c.ny * c.nx;
                add(4 * (size_t)psi_n[p]);
            }
        add(64);
        add(4 * (size_t)(s->nw > 0 ? s->nw : 1));
    }
    if (need > kNoAllocBytes)
        return nfail(ERTM_EINVAL, "grid needs %.1f MiB of scratch; the no-allocation entry point "
                     "holds at most %.0f MiB", need / 1048576.0, kNoAllocBytes / 1048576.0);

    unsigned char* base = nullptr;
    int rc = scratch_base(c.device, &base);
    if (rc) return rc;
    Carve cv{base};
    float* fbase[NFIELD] = {nullptr};
    for (int q = 0; q < nf; q++) fbase[fl[q]] = cv.take<float>(g.total);
    float* mbase[3];
    for (int q = 0; q < 3; q++) mbase[q] = cv.take<float>(g.total);
    float* prof[3][4];
    for (int ax = 0; ax < 3; ax++)
        for (int h = 0; h < 4; h++) prof[ax][h] = cv.take<float>(ns[ax]);
    float* psi[NPSI] = {nullptr};
    for (int p = 0; p < NPSI; p++)
        if (psi_n[p]) psi[p] = cv.take<float>(psi_n[p]);
    int* counters = cv.take<int>(16);
    float* wav = cv.take<float>(s->nw > 0 ? s->nw : 1);

    // clear what must start at zero: halos and state of every volume, memory variables
    for (int q = 0; q < nf; q++) NCK(cudaMemsetAsync(fbase[fl[q]], 0, 4 * g.total, st));
    for (int q = 0; q < 3; q++) NCK(cudaMemsetAsync(mbase[q], 0, 4 * g.total, st));
    for (int p = 0; p < NPSI; p++)
        if (psi[p]) NCK(cudaMemsetAsync(psi[p], 0, 4 * psi_n[p], st));
    NCK(cudaMemsetAsync(counters, 0, 16 * sizeof(int), st));
    if (s->nw > 0) NCK(cudaMemcpyAsync(wav, s->wavelet, 4 * (size_t)s->nw, cudaMemcpyDeviceToDevice, st));

    // model products rho vp^2, rho vs^2, 1/rho into the padded layout
    NCK(launch_model(g, vp, vs, rho, mbase[0] + g.off0, mbase[1] + g.off0, mbase[2] + g.off0, st));
    // C-PML strength from the model's largest vp unless the caller fixed it
    float vmax = c.pml_vmax;
    if (cpml && !(vmax > 0)) {
        const long long n = (long long)c.nx * c.ny * c.nz;
        float* vm_d = reinterpret_cast<float*>(counters + 8);
        long long nb = (n + 255) / 256;
        k_noalloc_absmax<<<(unsigned)(nb < 148 * 16 ? nb : 148 * 16), 256, 0, st>>>(vp, n, vm_d);
        NCK(cudaGetLastError());
        NCK(cudaMemcpyAsync(&vmax, vm_d, sizeof(float), cudaMemcpyDeviceToHost, st));
        NCK(cudaStreamSynchronize(st));
        if (!(vmax > 0.f) || !std::isfinite(vmax))
            return nfail(ERTM_EINVAL, "model vp has no positive finite maximum");
    }

    // difference coefficients
    float coef[8];
    stencil_coefs(c.coef_kind, c.coef, R, coef);

    // boundary profiles, computed in stack chunks and copied synchronously
    const double dts = c.dt_ms / 1000.0;
    const double hs[3] = {c.dx, c.dy, c.dz};
    for (int ax = 0; ax < 3; ax++) {
        const int n = ns[ax];
        int w0 = c.pml[2 * ax], w1 = c.pml[2 * ax + 1];
        if (ax == 1 && two_d) w0 = w1 = 0;
        float chunk[4][256];
        for (int i0 = 0; i0 < n; i0 += 256) {
            const int m = n - i0 < 256 ? n - i0 : 256;
            if (cpml) {
                const double rcoef = c.pml_r > 0 ? c.pml_r : 1e-3;
                const double f0 = c.pml_f0 > 0 ? c.pml_f0 : 10.0;
                for (int h = 0; h < 2; h++) {
                    const int stg = h == 0 ? 0 : (ax == 2 ? 1 : -1);
                    cpml_profile(n, w0, w1, stg, hs[ax], vmax, rcoef, f0, dts, i0, m, chunk[2 * h],
                                 chunk[2 * h + 1]);
                }
            } else {
                sponge_profile(n, w0, w1, c.boundary, c.sponge_coef, i0, m, chunk[0]);
            }
            for (int h = 0; h < (cpml ? 4 : 1); h++)
                NCK(cudaMemcpyAsync(prof[ax][h] + i0, chunk[h], 4 * m, cudaMemcpyHostToDevice, st));
            NCK(cudaStreamSynchronize(st));
        }
    }

    // kernel arguments
    KArgs a;
    std::memset(&a, 0, sizeof a);
    for (int q = 0; q < NFIELD; q++) a.f[q] = fbase[q] ? fbase[q] + g.off0 : nullptr;
    a.M = mbase[0] + g.off0;
    a.MU = mbase[1] + g.off0;
    a.B = mbase[2] + g.off0;
    a.sy = a.msy = g.sy;
    a.sz = a.msz = g.sz;
    a.nx = g.nx; a.ny = g.ny; a.nz = g.nz;
    for (int n = 0; n < 8; n++) {
        a.cx[n] = (float)(coef[n] / c.dx);
        a.cy[n] = (float)(coef[n] / c.dy);
        a.cz[n] = (float)(coef[n] / c.dz);
    }
    a.dt = c.dt_ms / 1000.f;
    for (int ax = 0; ax < 3; ax++) {
        a.att[ax] = cpml ? nullptr : prof[ax][0];
        a.pa[ax][0] = cpml ? prof[ax][0] : nullptr;
        a.pb[ax][0] = cpml ? prof[ax][1] : nullptr;
        a.pa[ax][1] = cpml ? prof[ax][2] : nullptr;
        a.pb[ax][1] = cpml ? prof[ax][3] : nullptr;
    }
    for (int p = 0; p < NPSI; p++) a.psi[p] = psi[p];
    for (int q = 0; q < 6; q++) a.w[q] = c.pml[q];
    if (two_d) a.w[2] = a.w[3] = 0;
    a.ssx = s->sx; a.ssy = s->sy; a.ssz = s->sz; a.nw = s->nw; a.wavelet = wav;
    a.rx0 = s->rx0; a.nrx = s->nrx; a.drx = s->drx;
    a.ry0 = s->ry0; a.nry = s->nry; a.dry = s->dry; a.rz = s->rz;
    a.inject_mode = ERTM_INJECT_ADD;
    a.traces = data_out;
    a.nt = c.nt;
    a.it_ptr = counters;
    a.err = counters + 4;

    // z planes per CTA: the context path's rule
    a.kchunk = choose_kchunk(g, R, c.device);

    // tensor maps over the scratch volumes
    StressMaps sm;
    VelMaps vm;
    std::memset(&sm, 0, sizeof sm);
    std::memset(&vm, 0, sizeof vm);
    const int xw = TX + 2 * xb_of(R), yh = g.tyb + (two_d ? 0 : 2 * R);
    const int vv[3] = {F_VX, F_VZ, F_VY};
    for (int q = 0; q < (two_d ? 2 : 3); q++) {
        if ((rc = encode(&sm.v[q], fbase[vv[q]], g, xw, yh))) return rc;
        if ((rc = encode(&sm.vc[q], fbase[vv[q]], g, TX, g.tyb))) return rc;
    }
    const int sg[6] = {F_TXX, F_TZZ, F_TXZ, F_TYY, F_TXY, F_TYZ};
    for (int q = 0; q < (two_d ? 3 : 6); q++)
        if ((rc = encode(&sm.sig[q], fbase[sg[q]], g, TX, g.tyb))) return rc;
    if ((rc = encode(&sm.M, mbase[0], g, TX, g.tyb))) return rc;
    if ((rc = encode(&sm.MU, mbase[1], g, TX, g.tyb))) return rc;
    if ((rc = encode(&vm.txx, fbase[F_TXX], g, xw, g.tyb))) return rc;
    if ((rc = encode(&vm.txz, fbase[F_TXZ], g, xw, g.tyb))) return rc;
    if (!two_d) {
        if ((rc = encode(&vm.txy, fbase[F_TXY], g, xw, yh))) return rc;
        if ((rc = encode(&vm.tyy, fbase[F_TYY], g, TX, yh))) return rc;
        if ((rc = encode(&vm.tyz, fbase[F_TYZ], g, TX, yh))) return rc;
    }
    int n = 0;
    if ((rc = encode(&vm.c[n++], fbase[F_VX], g, TX, g.tyb))) return rc;
    if ((rc = encode(&vm.c[n++], fbase[F_VZ], g, TX, g.tyb))) return rc;
    if (!two_d && (rc = encode(&vm.c[n++], fbase[F_VY], g, TX, g.tyb))) return rc;
    if ((rc = encode(&vm.c[n++], mbase[2], g, TX, g.tyb))) return rc;
    n = 0;
    if ((rc = encode(&vm.fr[n++], fbase[F_TXZ], g, TX, g.tyb))) return rc;
    if ((rc = encode(&vm.fr[n++], fbase[F_TZZ], g, TX, g.tyb))) return rc;
    if (!two_d && (rc = encode(&vm.fr[n++], fbase[F_TYZ], g, TX, g.tyb))) return rc;

    // the modelling pass: record vx, vy, vz at the receivers for every step
    if (nrec > 0) NCK(cudaMemsetAsync(data_out, 0, 4 * 3 * (size_t)c.nt * nrec, st));
    NCK(launch_set_int(counters, 0, st));
    for (int step = 0; step < c.nt; step++) {
        NCK(launch_stress(R, g, a, sm, cpml, false, st));
        NCK(launch_velocity(R, g, a, vm, cpml, EPI_NONE, nrec > 0, st));
        NCK(launch_advance(counters, 1, st));
    }
    int err = 0;
    NCK(cudaMemcpyAsync(&err, counters + 4, sizeof(int), cudaMemcpyDeviceToHost, st));
    NCK(cudaStreamSynchronize(st));
    if (err) return nfail(ERTM_EDEVICE, "a step kernel's bounded wait expired (code %d)", err);
    return ERTM_OK;
}

}  // namespace

extern "C" int ertm_forward_together_using_real_model_noalloc(const ertm_config* cfg,
                                                              const float* vp, const float* vs,
                                                              const float* rho,
                                                              const ertm_shot* shot,
                                                              float* data_out, void* stream,
                                                              char* errbuf, size_t errlen)
{
    g_noalloc_err[0] = 0;
    int rc = run_noalloc(cfg, vp, vs, rho, shot, data_out, stream);
    if (errbuf && errlen) {
        size_t n = strnlen(g_noalloc_err, sizeof g_noalloc_err);
        if (n >= errlen) n = errlen - 1;
        std::memcpy(errbuf, g_noalloc_err, n);
        errbuf[n] = 0;
    }
    return rc;
}
