// Host side of libertm: the C ABI declared in include/ertm.h.
//
// The context replaces the reference's GPUdevice struct and its globals
// (3D_elastic_RTM/3D_elastic_modeling_typedef_struct:1-55,
//  3D_elastic_RTM/3D_elastic_modeling_parameter:1-141).  It owns every device
// buffer; passes are stream-ordered on the context stream and each public call
// synchronises that stream before returning.  The whole grid lives on one GPU
// (no z-slab decomposition, unlike the reference's exchange_device_nz_kernel_*).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "ertm.h"
#include "born.cuh"
#include "ertm_internal.cuh"

using namespace ertm;

namespace {

thread_local std::string g_create_error;

enum Mode { MODE_MODEL = 0, MODE_SOURCE = 1, MODE_RECEIVER = 2, MODE_PLAIN = 3 };

// axis of each C-PML memory-variable slot (0 x, 1 y, 2 z)
const int kPsiAxis[NPSI] = {0, 1, 2, 1, 0, 2, 0, 2, 1, 0, 1, 2, 0, 1, 2, 0, 1, 2};
// slots that exist in 2D (no y derivative, no vy/txy/tyz)
const bool kPsi2D[NPSI] = {true, false, true, false, false, true, true, false, false,
                           true, false, true, false, false, false, true, false, true};

}  // namespace

struct ertm_ctx {
    ertm_config cfg{};
    int R = 4;
    Geom g{};
    int cap_nx = 0, cap_ny = 0;      // grid the buffers were allocated for (ertm_set_grid)
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    float coef[8] = {0};

    float* f_base[NFIELD] = {nullptr};
    float* f[NFIELD] = {nullptr};
    // per model: M, MU, B, VP, VS (padded)
    float* m_base[2][5] = {{nullptr}};
    float* m[2][5] = {{nullptr}};
    bool model_set[2] = {false, false};
    float vpmax[2] = {0.f, 0.f};

    // boundary
    float* att[3] = {nullptr, nullptr, nullptr};
    float* pa[3][2] = {{nullptr}};
    float* pb[3][2] = {{nullptr}};
    float* psi[NPSI] = {nullptr};
    long long psi_n[NPSI] = {0};
    float profile_vmax = -1.f;
    bool att_ready = false;

    // excitation and images (padded)
    float* ex_amp2_base = nullptr;
    int* ex_time_base = nullptr;
    float* ex_v_base[3] = {nullptr};
    float* ex_tp_base = nullptr;
    float* img_base[3] = {nullptr};
    // propagation angles at the excitation time (2D, ertm_set_angles): [0] source
    // wavefield, written by the source pass; [1] receiver wavefield, receiver pass
    float* ang_base[2] = {nullptr, nullptr};
    bool angles = false;
    bool have_src_angle = false, have_rcv_angle = false;
    bool have_excitation = false;
    int last_shot_key = 0;

    // staging
    float* stage = nullptr;          // 3 contiguous volumes
    float* traces = nullptr;
    size_t traces_cap = 0;
    float* wavelet = nullptr;
    int wavelet_cap = 0;
    int* it_d = nullptr;
    float* vmax_d = nullptr;
    int* err_d = nullptr;

    // TMA tensor maps (box shapes C, X, Y, XY; see StressMaps / VelMaps)
    CUtensorMap mC[NFIELD], mX[NFIELD], mY[NFIELD], mXY[NFIELD];
    CUtensorMap mModel[2][3];
    CUtensorMap mExAmp, mExTime;

    // test hook of the device-error path (ertm_set_wait_fault)
    int skip_plane1 = 0;
    unsigned wait_polls = 0;
    // 3D step-kernel variant (ertm_set_step_variant): 0 one cell per thread, 1 cell pairs
    int pairs = 0;

    std::string err;
    long long launches = 0;

    // Born / adjoint state (2D, compact layout; allocated on first use).  Shared
    // volumes (model and perturbation products) once; per-shot volumes for a group
    // of `G` shots run by one launch per step, each type laid out [shot][n].
    struct BornState {
        bool ready = false;
        long long px = 0, n = 0;          // pitch and floats per compact volume
        float* shared = nullptr;          // the SV_* volumes
        float* sv[16] = {nullptr};
        float* block = nullptr;           // the PV_* volumes of G shots
        float* pv[64] = {nullptr};        // type q, shot 0 (shot s at + s * n)
        int G = 0;
        float* ckpt = nullptr;            // checkpoints: nck x 14 types x G shots
        long long ckpt_floats = 0;
        float* hist = nullptr;            // history: K x 4 types x G shots
        long long hist_floats = 0;
        int* tab = nullptr;               // shot table, G x 8 ints (device)
        int tab_cap = 0;
        float* wav = nullptr;             // wavelets, G x nw (device)
        long long wav_cap = 0;
    } born;
};

namespace {

int fail(ertm_ctx* c, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    else g_create_error = buf;
    return code;
}

#define CK(ctx, call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail((ctx), e_ == cudaErrorMemoryAllocation ? ERTM_ENOMEM : ERTM_ECUDA, \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

bool is_device_ptr(const void* p)
{
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }

bool field_used(const Geom& g, int f)
{
    if (!g.two_d) return true;
    return !(f == F_VY || f == F_TYY || f == F_TXY || f == F_TYZ || f == F_VYP);
}

int alloc_volume(ertm_ctx* c, float** base, float** origin)
{
    CK(c, cudaMalloc(base, sizeof(float) * c->g.total));
    CK(c, cudaMemsetAsync(*base, 0, sizeof(float) * c->g.total, c->stream));
    *origin = *base + c->g.off0;
    return ERTM_OK;
}

int ensure_stage(ertm_ctx* c)
{
    if (c->stage) return ERTM_OK;
    // sized for the allocated grid: ertm_set_grid may enlarge the active one later
    long long n = (long long)c->cap_nx * c->cap_ny * c->g.nz;
    CK(c, cudaMalloc(&c->stage, sizeof(float) * 3 * n));
    return ERTM_OK;
}

__global__ void k_absmax(const float* __restrict__ v, long long n, float* out)
{
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(v[i]));
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax((int*)out, __float_as_int(m));
}

// Fill host-side double profiles, upload as float.
int upload_profiles(ertm_ctx* c, float vmax)
{
    const ertm_config& cf = c->cfg;
    const Geom& g = c->g;
    const double dts = cf.dt_ms / 1000.0;
    int ns[3] = {g.nx, g.ny, g.nz};
    double hs[3] = {cf.dx, cf.dy, cf.dz};
    if (cf.boundary == ERTM_BOUNDARY_CPML) {
        if (c->profile_vmax == vmax) return ERTM_OK;
        double rc = cf.pml_r > 0 ? cf.pml_r : 1e-3;
        double f0 = cf.pml_f0 > 0 ? cf.pml_f0 : 10.0;
        for (int ax = 0; ax < 3; ax++) {
            int n = ns[ax];
            int w0 = cf.pml[2 * ax], w1 = cf.pml[2 * ax + 1];
            if (ax == 1 && g.two_d) w0 = w1 = 0;
            for (int h = 0; h < 2; h++) {
                int stg = h == 0 ? 0 : (ax == 2 ? 1 : -1);
                std::vector<float> a(n), b(n);
                cpml_profile(n, w0, w1, stg, hs[ax], vmax, rc, f0, dts, 0, n, a.data(), b.data());
                if (!c->pa[ax][h]) {
                    const int cap = ax == 0 ? c->cap_nx : ax == 1 ? c->cap_ny : g.nz;
                    CK(c, cudaMalloc(&c->pa[ax][h], sizeof(float) * cap));
                    CK(c, cudaMalloc(&c->pb[ax][h], sizeof(float) * cap));
                }
                CK(c, cudaMemcpyAsync(c->pa[ax][h], a.data(), sizeof(float) * n,
                                      cudaMemcpyHostToDevice, c->stream));
                CK(c, cudaMemcpyAsync(c->pb[ax][h], b.data(), sizeof(float) * n,
                                      cudaMemcpyHostToDevice, c->stream));
                CK(c, cudaStreamSynchronize(c->stream));
            }
        }
        c->profile_vmax = vmax;
        return ERTM_OK;
    }
    if (c->att_ready) return ERTM_OK;
    for (int ax = 0; ax < 3; ax++) {
        int n = ns[ax];
        std::vector<float> v(n, 0.f);
        if (!(ax == 1 && g.two_d))
            sponge_profile(n, cf.pml[2 * ax], cf.pml[2 * ax + 1], cf.boundary, cf.sponge_coef, 0, n,
                           v.data());
        if (!c->att[ax]) {
            const int cap = ax == 0 ? c->cap_nx : ax == 1 ? c->cap_ny : g.nz;
            CK(c, cudaMalloc(&c->att[ax], sizeof(float) * cap));
        }
        CK(c, cudaMemcpyAsync(c->att[ax], v.data(), sizeof(float) * n, cudaMemcpyHostToDevice,
                              c->stream));
    }
    CK(c, cudaStreamSynchronize(c->stream));
    c->att_ready = true;
    return ERTM_OK;
}

int validate_shot(ertm_ctx* c, const ertm_shot* s, bool need_source)
{
    if (!s) return fail(c, ERTM_EINVAL, "shot is NULL");
    const Geom& g = c->g;
    if (need_source) {
        if (s->sx < 0 || s->sx >= g.nx || s->sy < 0 || s->sy >= g.ny || s->sz < 0 || s->sz >= g.nz)
            return fail(c, ERTM_EINVAL, "source cell (%d,%d,%d) outside the %dx%dx%d grid", s->sx,
                        s->sy, s->sz, g.nx, g.ny, g.nz);
        if (s->nw < 0 || (s->nw > 0 && !s->wavelet))
            return fail(c, ERTM_EINVAL, "wavelet of %d samples with NULL pointer", s->nw);
    }
    if (s->nrx < 0 || s->nry < 0 || s->drx <= 0 || s->dry <= 0)
        return fail(c, ERTM_EINVAL, "bad receiver grid (nrx=%d nry=%d drx=%d dry=%d)", s->nrx,
                    s->nry, s->drx, s->dry);
    if (g.two_d && (s->nry > 1 || s->ry0 != 0 || s->sy != 0))
        return fail(c, ERTM_EINVAL, "2D grid: receivers and source must sit at y = 0");
    if (s->inject_mode != 0 && s->inject_mode != ERTM_INJECT_ADD && s->inject_mode != ERTM_INJECT_REPLACE)
        return fail(c, ERTM_EINVAL, "inject_mode %d", s->inject_mode);
    return ERTM_OK;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
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
    return fn;
}

// One tensor map over a whole padded volume (allocation base, [pz][py][px]) with a
// bx x by x 1 box.  TMA requires 16-byte aligned bases and strides: cudaMalloc bases
// are 256-byte aligned and the row pitch is a multiple of 128 bytes.
int encode_map(ertm_ctx* c, CUtensorMap* m, const void* base, bool is_int, int bx, int by)
{
    auto enc = tensor_map_encoder();
    if (!enc) return fail(c, ERTM_ECUDA, "cuTensorMapEncodeTiled unavailable");
    const Geom& g = c->g;
    cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)g.py, (cuuint64_t)g.pz};
    cuuint64_t strides[2] = {(cuuint64_t)g.px * 4, (cuuint64_t)(g.px * g.py) * 4};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = enc(m, is_int ? CU_TENSOR_MAP_DATA_TYPE_INT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                     const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(c, ERTM_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return ERTM_OK;
}

struct BoxDims {
    int c_x, c_y, x_x, y_y;
};
BoxDims box_dims(const ertm_ctx* c)
{
    const int tyb = c->g.tyb;
    const int xw = TX + 2 * xb_of(c->R);
    const int yh = tyb + (c->g.two_d ? 0 : 2 * c->R);
    return {TX, tyb, xw, yh};
}

// tensor maps of every field: centre boxes for all, halo boxes where a kernel
// differentiates along x / y: vx vy vz tp txy (XY), txx txz (X), tyy tyz (Y)
int build_field_maps(ertm_ctx* c)
{
    BoxDims b = box_dims(c);
    int rc;
    for (int q = 0; q < NFIELD; q++) {
        if (!c->f_base[q]) continue;
        if ((rc = encode_map(c, &c->mC[q], c->f_base[q], false, b.c_x, b.c_y))) return rc;
        if ((rc = encode_map(c, &c->mX[q], c->f_base[q], false, b.x_x, b.c_y))) return rc;
        if ((rc = encode_map(c, &c->mXY[q], c->f_base[q], false, b.x_x, b.y_y))) return rc;
        if ((rc = encode_map(c, &c->mY[q], c->f_base[q], false, b.c_x, b.y_y))) return rc;
    }
    return ERTM_OK;
}

StressMaps stress_maps(const ertm_ctx* c, int which)
{
    StressMaps m;
    std::memset(&m, 0, sizeof m);
    const int v[3] = {F_VX, F_VZ, F_VY};
    for (int q = 0; q < 3; q++) {
        m.v[q] = c->mXY[v[q]];
        m.vc[q] = c->mC[v[q]];
    }
    const int sg[6] = {F_TXX, F_TZZ, F_TXZ, F_TYY, F_TXY, F_TYZ};
    for (int q = 0; q < 6; q++) m.sig[q] = c->mC[sg[q]];
    m.tp = c->mC[F_TP];
    m.M = c->mModel[which][0];
    m.MU = c->mModel[which][1];
    return m;
}

VelMaps vel_maps(const ertm_ctx* c, int which, int epi)
{
    VelMaps m;
    std::memset(&m, 0, sizeof m);
    const bool Y = !c->g.two_d, ps = (epi != EPI_NONE);
    m.txx = c->mX[F_TXX];
    m.txz = c->mX[F_TXZ];
    m.txy = c->mXY[F_TXY];
    m.tp = c->mXY[F_TP];
    m.tyy = c->mY[F_TYY];
    m.tyz = c->mY[F_TYZ];
    int n = 0;
    m.c[n++] = c->mC[F_VX];
    m.c[n++] = c->mC[F_VZ];
    if (Y) m.c[n++] = c->mC[F_VY];
    if (ps) {
        m.c[n++] = c->mC[F_VXP];
        m.c[n++] = c->mC[F_VZP];
        if (Y) m.c[n++] = c->mC[F_VYP];
    }
    m.c[n++] = c->mModel[which][2];
    if (epi == EPI_EXCITE) m.c[n++] = c->mExAmp;
    if (epi == EPI_IMAGE) m.c[n++] = c->mExTime;
    n = 0;
    m.fr[n++] = c->mC[F_TXZ];
    m.fr[n++] = c->mC[F_TZZ];
    if (Y) m.fr[n++] = c->mC[F_TYZ];
    if (ps) m.fr[n++] = c->mC[F_TP];
    return m;
}

int ensure_traces(ertm_ctx* c, size_t n)
{
    if (c->traces_cap >= n) return ERTM_OK;
    if (c->traces) cudaFree(c->traces);
    c->traces = nullptr;
    c->traces_cap = 0;
    CK(c, cudaMalloc(&c->traces, sizeof(float) * n));
    c->traces_cap = n;
    return ERTM_OK;
}

int ensure_excitation(ertm_ctx* c)
{
    if (c->ex_amp2_base) return ERTM_OK;
    float* dummy;
    int rc;
    if ((rc = alloc_volume(c, &c->ex_amp2_base, &dummy))) return rc;
    CK(c, cudaMalloc(&c->ex_time_base, sizeof(int) * c->g.total));
    for (int q = 0; q < 3; q++) {
        if (q == 1 && c->g.two_d) continue;
        if ((rc = alloc_volume(c, &c->ex_v_base[q], &dummy))) return rc;
    }
    if ((rc = alloc_volume(c, &c->ex_tp_base, &dummy))) return rc;
    const int tyb = c->g.tyb;
    if ((rc = encode_map(c, &c->mExAmp, c->ex_amp2_base, false, TX, tyb))) return rc;
    if ((rc = encode_map(c, &c->mExTime, c->ex_time_base, true, TX, tyb))) return rc;
    return ERTM_OK;
}

int ensure_images(ertm_ctx* c)
{
    if (c->img_base[0]) return ERTM_OK;
    float* dummy;
    for (int q = 0; q < 3; q++) {
        int rc = alloc_volume(c, &c->img_base[q], &dummy);
        if (rc) return rc;
    }
    return ERTM_OK;
}

// Common kernel arguments for a pass in model `which`.
void fill_args(ertm_ctx* c, int which, const ertm_shot* s, KArgs& a)
{
    const Geom& g = c->g;
    std::memset(&a, 0, sizeof a);
    for (int q = 0; q < NFIELD; q++) a.f[q] = c->f[q];
    a.M = c->m[which][0];
    a.MU = c->m[which][1];
    a.B = c->m[which][2];
    a.sy = g.sy;
    a.sz = g.sz;
    a.msy = g.sy;
    a.msz = g.sz;
    a.nx = g.nx;
    a.ny = g.ny;
    a.nz = g.nz;
    a.kchunk = g.nz;
    for (int n = 0; n < 8; n++) {
        a.cx[n] = (float)(c->coef[n] / c->cfg.dx);
        a.cy[n] = (float)(c->coef[n] / c->cfg.dy);
        a.cz[n] = (float)(c->coef[n] / c->cfg.dz);
    }
    a.dt = c->cfg.dt_ms / 1000.f;
    for (int ax = 0; ax < 3; ax++) {
        a.att[ax] = c->att[ax];
        for (int h = 0; h < 2; h++) {
            a.pa[ax][h] = c->pa[ax][h];
            a.pb[ax][h] = c->pb[ax][h];
        }
    }
    for (int p = 0; p < NPSI; p++) a.psi[p] = c->psi[p];
    for (int q = 0; q < 6; q++) a.w[q] = c->cfg.pml[q];
    if (g.two_d) a.w[2] = a.w[3] = 0;
    if (s) {
        a.ssx = s->sx;
        a.ssy = s->sy;
        a.ssz = s->sz;
        a.nw = s->nw;
        a.rx0 = s->rx0;
        a.nrx = s->nrx;
        a.drx = s->drx;
        a.ry0 = s->ry0;
        a.nry = s->nry;
        a.dry = s->dry;
        a.rz = s->rz;
        a.inject_mode = s->inject_mode == 0 ? ERTM_INJECT_ADD : s->inject_mode;
    } else {
        a.nw = 0;
        a.drx = a.dry = 1;
        a.rz = -1;
    }
    a.wavelet = c->wavelet;
    a.nt = c->cfg.nt;
    a.it_ptr = c->it_d;
    a.ex_amp2 = c->ex_amp2_base ? c->ex_amp2_base + g.off0 : nullptr;
    a.ex_time = c->ex_time_base ? c->ex_time_base + g.off0 : nullptr;
    for (int q = 0; q < 3; q++) {
        a.ex_v[q] = c->ex_v_base[q] ? c->ex_v_base[q] + g.off0 : nullptr;
        a.img[q] = c->img_base[q] ? c->img_base[q] + g.off0 : nullptr;
    }
    a.ex_tp = c->ex_tp_base ? c->ex_tp_base + g.off0 : nullptr;
    a.err = c->err_d;
    a.skip_plane1 = c->skip_plane1;
    a.wait_polls = c->wait_polls;
    a.pairs = c->pairs;
}

int check_device_error(ertm_ctx* c)
{
    int e = 0;
    CK(c, cudaMemcpyAsync(&e, c->err_d, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    if (e) {
        CK(c, cudaMemsetAsync(c->err_d, 0, sizeof(int), c->stream));
        return fail(c, ERTM_EDEVICE, "a step kernel's bounded wait for its staged planes expired (code %d)", e);
    }
    return ERTM_OK;
}

// floats of C-PML memory-variable slot p on the active grid g
long long psi_count(const Geom& g, const ertm_config& c, int p)
{
    const int ax = kPsiAxis[p];
    const long long w = c.pml[2 * ax] + c.pml[2 * ax + 1];
    return ax == 0 ? (long long)g.nz * g.ny * w : ax == 1 ? (long long)g.nz * w * g.nx : w * g.ny * g.nx;
}

// Z-chunk autotuner (ertm_config.autotune = 1).  For each grid shape, stencil
// radius, boundary kind and device it times the plain step (stress + velocity,
// no source, no epilogue) for a few steps at every candidate chunk and keeps the
// fastest; the result is cached for the life of the process.  It runs before a
// pass resets the wavefields, so the trial steps leave no trace.
struct TuneKey {
    int device, nx, ny, nz, R, cpml;
    bool operator<(const TuneKey& o) const
    {
        return std::tie(device, nx, ny, nz, R, cpml) < std::tie(o.device, o.nx, o.ny, o.nz, o.R, o.cpml);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, int> g_tuned;

int autotune_kchunk(ertm_ctx* c, int which, int* out)
{
    const Geom& g = c->g;
    const bool cpml = c->cfg.boundary == ERTM_BOUNDARY_CPML;
    const TuneKey key{c->device, g.nx, g.ny, g.nz, c->R, cpml ? 1 : 0};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            *out = it->second;
            return ERTM_OK;
        }
    }
    std::vector<int> cand;
    const int base[] = {16, 24, 32, 48, 64, 96, 128};
    for (int v : base)
        if (v < g.nz) cand.push_back(v);
    cand.push_back(g.nz);
    KArgs a;
    fill_args(c, which, nullptr, a);
    a.traces = nullptr;
    a.wavelet = nullptr;
    CK(c, launch_set_int(c->it_d, 0, c->stream));   // the kernels read the step index
    const StressMaps sm = stress_maps(c, which);
    const VelMaps vm = vel_maps(c, which, EPI_NONE);
    cudaEvent_t e0, e1;
    CK(c, cudaEventCreate(&e0));
    CK(c, cudaEventCreate(&e1));
    int best = cand.back();
    float best_ms = 1e30f;
    cudaError_t e = cudaSuccess;
    for (int kc : cand) {
        a.kchunk = kc;
        for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {
            if (rep == 1) e = cudaEventRecord(e0, c->stream);
            if (e == cudaSuccess) e = launch_stress(c->R, g, a, sm, cpml, false, c->stream);
            if (e == cudaSuccess) e = launch_velocity(c->R, g, a, vm, cpml, EPI_NONE, false, c->stream);
            c->launches += 2;
        }
        if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) break;
        if (ms < best_ms) {
            best_ms = ms;
            best = kc;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return fail(c, ERTM_ECUDA, "autotune: %s", cudaGetErrorString(e));
    int rc = check_device_error(c);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[key] = best;
    }
    *out = best;
    return ERTM_OK;
}

int reset_state(ertm_ctx* c)
{
    for (int q = 0; q < NFIELD; q++)
        if (c->f_base[q]) CK(c, cudaMemsetAsync(c->f_base[q], 0, sizeof(float) * c->g.total, c->stream));
    for (int p = 0; p < NPSI; p++)
        if (c->psi[p]) CK(c, cudaMemsetAsync(c->psi[p], 0, sizeof(float) * c->psi_n[p], c->stream));
    return ERTM_OK;
}

int upload_wavelet(ertm_ctx* c, const ertm_shot* s)
{
    if (s->nw <= 0) return ERTM_OK;
    if (c->wavelet_cap < s->nw) {
        if (c->wavelet) cudaFree(c->wavelet);
        c->wavelet = nullptr;
        CK(c, cudaMalloc(&c->wavelet, sizeof(float) * s->nw));
        c->wavelet_cap = s->nw;
    }
    CK(c, cudaMemcpyAsync(c->wavelet, s->wavelet, sizeof(float) * s->nw, cudaMemcpyDefault, c->stream));
    return ERTM_OK;
}

// NVTX range for profilers (no-op unless a tool is attached): one per pass and per
// Born operator call, so timelines show shots, passes and CG operator calls.
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
};

// One pass of `nsteps` steps.  MODE_MODEL records into `traces` ([3][nt][nrec],
// device), MODE_RECEIVER injects from it.
// The time loop of a pass: `one_step` (which launches one step's kernels on
// c->stream) runs nsteps times, as a CUDA graph of kGraphSteps steps replayed
// back to back (the kernels read the step index from device memory, so one graph
// serves every chunk); the first step and the remainder are launched directly.
template <typename F>
int time_loop(ertm_ctx* c, int nsteps, F&& one_step)
{
    constexpr int kGraphSteps = 32;
    int done = 0;
    if (nsteps > 0) {
        CK(c, one_step());
        done = 1;
    }
    if (nsteps - done >= 2 * kGraphSteps) {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        CK(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int q = 0; q < kGraphSteps && e == cudaSuccess; q++) e = one_step();
        cudaError_t e2 = cudaStreamEndCapture(c->stream, &graph);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
        while (e == cudaSuccess && nsteps - done >= kGraphSteps) {
            e = cudaGraphLaunch(exec, c->stream);
            done += kGraphSteps;
        }
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fail(c, ERTM_ECUDA, "graph time loop: %s", cudaGetErrorString(e));
    }
    for (; done < nsteps; done++) CK(c, one_step());
    return ERTM_OK;
}

int run_pass(ertm_ctx* c, int which, const ertm_shot* s, int mode, int nsteps, float* traces)
{
    if (!c->model_set[which])
        return fail(c, ERTM_ESTATE, "%s model not set", which ? "migration" : "true");
    Range range(mode == MODE_SOURCE ? "ertm source pass" : mode == MODE_RECEIVER ? "ertm receiver pass"
                                                                               : "ertm modelling pass");
    int rc;
    float vmax = c->cfg.pml_vmax > 0 ? c->cfg.pml_vmax : c->vpmax[which];
    if ((rc = upload_profiles(c, vmax))) return rc;
    int kchunk = choose_kchunk(c->g, c->R, c->device);
    if (c->cfg.autotune == 1 && (rc = autotune_kchunk(c, which, &kchunk))) return rc;
    if ((rc = reset_state(c))) return rc;
    if (mode != MODE_RECEIVER && (rc = upload_wavelet(c, s))) return rc;
    KArgs a;
    fill_args(c, which, s, a);
    a.kchunk = kchunk;
    a.traces = traces;
    const bool cpml = c->cfg.boundary == ERTM_BOUNDARY_CPML;
    const int R = c->R;
    int epi = EPI_NONE;
    bool psplit = false, record = false;
    if (mode == MODE_SOURCE) { epi = EPI_EXCITE; psplit = true; }
    if (mode == MODE_RECEIVER) { epi = EPI_IMAGE; psplit = true; }
    if (mode == MODE_MODEL) record = (traces != nullptr);
    if (mode == MODE_RECEIVER) a.nw = 0;
    int it0 = (mode == MODE_RECEIVER) ? nsteps - 1 : 0;
    int dir = (mode == MODE_RECEIVER) ? -1 : 1;
    CK(c, launch_set_int(c->it_d, it0, c->stream));
    c->launches++;
    if (mode == MODE_RECEIVER && nsteps > 0) {
        CK(c, launch_inject(a, nsteps - 1, c->stream));
        c->launches++;
    }
    const StressMaps sm = stress_maps(c, which);
    const VelMaps vm = vel_maps(c, which, epi);
    float* ang = nullptr;
    if (c->angles && mode == MODE_SOURCE) ang = c->ang_base[0] + c->g.off0;
    if (c->angles && mode == MODE_RECEIVER) ang = c->ang_base[1] + c->g.off0;
    auto one_step = [&]() -> cudaError_t {
        cudaError_t e = launch_stress(R, c->g, a, sm, cpml, psplit, c->stream);
        if (e == cudaSuccess) e = launch_velocity(R, c->g, a, vm, cpml, epi, record, c->stream);
        if (e == cudaSuccess && ang)
            e = launch_angle(c->g, a, ang, mode == MODE_SOURCE ? 2 : 4, c->stream);
        if (e == cudaSuccess) e = launch_advance(c->it_d, dir, c->stream);
        return e;
    };
    if ((rc = time_loop(c, nsteps, one_step))) return rc;
    c->launches += (ang ? 4LL : 3LL) * nsteps;
    return check_device_error(c);
}

int copy_out_volume(ertm_ctx* c, const float* padded_origin, float* out)
{
    if (!out) return ERTM_OK;
    if (is_device_ptr(out)) {
        CK(c, launch_gather(c->g, padded_origin, out, c->stream));
        c->launches++;
        return ERTM_OK;
    }
    int rc = ensure_stage(c);
    if (rc) return rc;
    long long n = (long long)c->g.nx * c->g.ny * c->g.nz;
    CK(c, launch_gather(c->g, padded_origin, c->stage, c->stream));
    c->launches++;
    CK(c, cudaMemcpyAsync(out, c->stage, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return ERTM_OK;
}

long long nrec_of(const ertm_shot* s) { return (long long)s->nrx * s->nry; }

}  // namespace

extern "C" {

int ertm_abi_version(void) { return ERTM_ABI_VERSION; }

int ertm_create(const ertm_config* cfg, ertm_ctx** out)
{
    if (!out) return fail(nullptr, ERTM_EINVAL, "out is NULL");
    *out = nullptr;
    if (!cfg) return fail(nullptr, ERTM_EINVAL, "config is NULL");
    const ertm_config& c = *cfg;
    if (c.nx < 1 || c.ny < 1 || c.nz < 1)
        return fail(nullptr, ERTM_EINVAL, "grid %dx%dx%d", c.nx, c.ny, c.nz);
    if (!(c.dx > 0) || !(c.dy > 0) || !(c.dz > 0) || !(c.dt_ms > 0))
        return fail(nullptr, ERTM_EINVAL, "spacings and dt must be positive");
    if (c.nt < 1) return fail(nullptr, ERTM_EINVAL, "nt = %d", c.nt);
    if (c.order != 8 && c.order != 12)
        return fail(nullptr, ERTM_ENOTSUP, "order %d (8 or 12 supported)", c.order);
    if (c.boundary < 0 || c.boundary > 2) return fail(nullptr, ERTM_EINVAL, "boundary %d", c.boundary);
    if (c.coef_kind == ERTM_COEF_REFERENCE12 && c.order != 12)
        return fail(nullptr, ERTM_EINVAL, "reference coefficients need order 12");
    if (c.coef_kind < 0 || c.coef_kind > 2) return fail(nullptr, ERTM_EINVAL, "coef_kind %d", c.coef_kind);
    for (int q = 0; q < 6; q++)
        if (c.pml[q] < 0) return fail(nullptr, ERTM_EINVAL, "negative absorbing width");
    int ns[3] = {c.nx, c.ny, c.nz};
    for (int ax = 0; ax < 3; ax++) {
        if (ax == 1 && c.ny == 1) continue;
        if (c.pml[2 * ax] + c.pml[2 * ax + 1] > ns[ax])
            return fail(nullptr, ERTM_EINVAL, "absorbing widths exceed the grid on axis %d", ax);
        if (c.boundary != ERTM_BOUNDARY_CPML && (c.pml[2 * ax] == 1 || c.pml[2 * ax + 1] == 1))
            return fail(nullptr, ERTM_EINVAL, "sponge widths must be 0 or >= 2");
    }
    if (c.src_steps < 0 || c.src_steps > c.nt)
        return fail(nullptr, ERTM_EINVAL, "src_steps %d outside [0, nt]", c.src_steps);
    if (c.reserved[0]) return fail(nullptr, ERTM_EINVAL, "reserved fields must be zero");
    if (c.visco_nmech < 0 || c.visco_nmech > 3)
        return fail(nullptr, ERTM_EINVAL, "visco_nmech %d (0..3)", c.visco_nmech);
    if (c.visco_nmech > 0 && !(c.visco_qp > 0 && c.visco_qs > 0 && c.visco_f0 > 0))
        return fail(nullptr, ERTM_EINVAL, "viscoelastic Born needs positive visco_qp, visco_qs, visco_f0");
    if (c.autotune != 0 && c.autotune != 1) return fail(nullptr, ERTM_EINVAL, "autotune %d", c.autotune);
    if (c.checkpoint_every < 0) return fail(nullptr, ERTM_EINVAL, "checkpoint_every < 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(nullptr, ERTM_ECUDA, "no CUDA device");
    }
    if (c.device < 0 || c.device >= ndev) return fail(nullptr, ERTM_EINVAL, "device %d of %d", c.device, ndev);

    ertm_ctx* x = new (std::nothrow) ertm_ctx();
    if (!x) return fail(nullptr, ERTM_ENOMEM, "host allocation");
    x->cfg = c;
    x->R = c.order / 2;
    x->device = c.device;
    x->g = make_geom(c.nx, c.ny, c.nz, x->R);
    if (x->g.total >= (1LL << 31)) {   // the step kernels index a volume with 32-bit offsets
        const long long total = x->g.total;
        delete x;
        return fail(nullptr, ERTM_EINVAL, "grid too large: %lld floats per padded volume (limit 2^31)", total);
    }
    int rc = ERTM_OK;
    auto bail = [&](int code) {
        g_create_error = x->err;
        ertm_destroy(x);
        return code;
    };
    if (cudaSetDevice(c.device) != cudaSuccess) {
        fail(x, ERTM_ECUDA, "cudaSetDevice(%d)", c.device);
        return bail(ERTM_ECUDA);
    }
    if (cudaStreamCreateWithFlags(&x->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        fail(x, ERTM_ECUDA, "stream create");
        return bail(ERTM_ECUDA);
    }
    x->stream = x->own_stream;
    // difference coefficients
    stencil_coefs(c.coef_kind, c.coef, x->R, x->coef);
    for (int q = 0; q < NFIELD; q++) {
        if (!field_used(x->g, q)) continue;
        if ((rc = alloc_volume(x, &x->f_base[q], &x->f[q]))) return bail(rc);
    }
    x->cap_nx = c.nx;
    x->cap_ny = c.ny;
    if (c.boundary == ERTM_BOUNDARY_CPML) {
        const Geom& g = x->g;
        for (int p = 0; p < NPSI; p++) {
            if (g.two_d && !kPsi2D[p]) continue;
            const long long n = psi_count(g, c, p);
            x->psi_n[p] = n;
            if (n == 0) continue;
            if (cudaMalloc(&x->psi[p], sizeof(float) * n) != cudaSuccess) {
                cudaGetLastError();
                fail(x, ERTM_ENOMEM, "C-PML memory variables");
                return bail(ERTM_ENOMEM);
            }
        }
    }
    if (cudaMalloc(&x->it_d, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&x->vmax_d, sizeof(float)) != cudaSuccess ||
        cudaMalloc(&x->err_d, sizeof(int)) != cudaSuccess ||
        cudaMemsetAsync(x->it_d, 0, sizeof(int), x->stream) != cudaSuccess ||
        cudaMemsetAsync(x->err_d, 0, sizeof(int), x->stream) != cudaSuccess) {
        cudaGetLastError();
        fail(x, ERTM_ENOMEM, "counters");
        return bail(ERTM_ENOMEM);
    }
    if ((rc = build_field_maps(x))) return bail(rc);
    if (cudaStreamSynchronize(x->stream) != cudaSuccess) {
        fail(x, ERTM_ECUDA, "%s", cudaGetErrorString(cudaGetLastError()));
        return bail(ERTM_ECUDA);
    }
    *out = x;
    return ERTM_OK;
}

int ertm_destroy(ertm_ctx* c)
{
    if (!c) return ERTM_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int q = 0; q < NFIELD; q++) cudaFree(c->f_base[q]);
    for (int w = 0; w < 2; w++)
        for (int q = 0; q < 5; q++) cudaFree(c->m_base[w][q]);
    for (int ax = 0; ax < 3; ax++) {
        cudaFree(c->att[ax]);
        for (int h = 0; h < 2; h++) {
            cudaFree(c->pa[ax][h]);
            cudaFree(c->pb[ax][h]);
        }
    }
    for (int p = 0; p < NPSI; p++) cudaFree(c->psi[p]);
    cudaFree(c->ex_amp2_base);
    cudaFree(c->ex_time_base);
    for (int q = 0; q < 3; q++) {
        cudaFree(c->ex_v_base[q]);
        cudaFree(c->img_base[q]);
    }
    cudaFree(c->ex_tp_base);
    cudaFree(c->ang_base[0]);
    cudaFree(c->ang_base[1]);
    cudaFree(c->stage);
    cudaFree(c->traces);
    cudaFree(c->wavelet);
    cudaFree(c->it_d);
    cudaFree(c->vmax_d);
    cudaFree(c->err_d);
    cudaFree(c->born.shared);
    cudaFree(c->born.block);
    cudaFree(c->born.ckpt);
    cudaFree(c->born.hist);
    cudaFree(c->born.tab);
    cudaFree(c->born.wav);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return ERTM_OK;
}

int ertm_last_error(const ertm_ctx* c, char* buf, size_t len)
{
    if (!buf || len == 0) return ERTM_EINVAL;
    const std::string& s = c ? c->err : g_create_error;
    size_t n = std::min(len - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
    return ERTM_OK;
}

int ertm_set_stream(ertm_ctx* c, void* stream)
{
    if (!c) return ERTM_EINVAL;
    CK(c, cudaStreamSynchronize(c->stream));
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return ERTM_OK;
}

int ertm_set_grid(ertm_ctx* c, int nx, int ny, int nt, int src_steps)
{
    if (!c) return ERTM_EINVAL;
    if (nx < 1 || ny < 1 || nx > c->cap_nx || ny > c->cap_ny)
        return fail(c, ERTM_EINVAL, "active grid %dx%d outside the allocated %dx%d", nx, ny, c->cap_nx,
                    c->cap_ny);
    if (c->g.two_d && ny != 1) return fail(c, ERTM_EINVAL, "2D context: ny must be 1");
    if (nt < 1 || src_steps < 0 || src_steps > nt)
        return fail(c, ERTM_EINVAL, "nt = %d, src_steps = %d", nt, src_steps);
    const int ns[2] = {nx, ny};
    for (int ax = 0; ax < 2; ax++) {
        if (ax == 1 && c->g.two_d) continue;
        if (c->cfg.pml[2 * ax] + c->cfg.pml[2 * ax + 1] > ns[ax])
            return fail(c, ERTM_EINVAL, "absorbing widths exceed the active grid on axis %d", ax);
    }
    CK(c, cudaSetDevice(c->device));
    CK(c, cudaStreamSynchronize(c->stream));
    c->g.nx = nx;
    c->g.ny = ny;
    c->cfg.nx = nx;
    c->cfg.ny = ny;
    c->cfg.nt = nt;
    c->cfg.src_steps = src_steps;
    for (int p = 0; p < NPSI; p++)
        if (c->psi[p]) c->psi_n[p] = psi_count(c->g, c->cfg, p);
    c->profile_vmax = -1.f;
    c->att_ready = false;
    c->model_set[0] = c->model_set[1] = false;
    c->have_excitation = false;
    c->have_src_angle = c->have_rcv_angle = false;
    c->born.ready = false;
    return ERTM_OK;
}

int ertm_set_angles(ertm_ctx* c, int on)
{
    if (!c) return ERTM_EINVAL;
    if (on != 0 && on != 1) return fail(c, ERTM_EINVAL, "on = %d", on);
    if (on && !c->g.two_d) return fail(c, ERTM_ENOTSUP, "propagation angles need a 2D grid");
    CK(c, cudaSetDevice(c->device));
    if (on && !c->ang_base[0]) {
        float* dummy;
        for (int q = 0; q < 2; q++) {
            int rc = alloc_volume(c, &c->ang_base[q], &dummy);
            if (rc) return rc;
        }
    }
    if (!on) c->have_src_angle = c->have_rcv_angle = false;
    c->angles = on != 0;
    return ERTM_OK;
}

int ertm_get_angles(ertm_ctx* c, float* src_angle, float* rcv_angle)
{
    if (!c) return ERTM_EINVAL;
    if (!c->angles) return fail(c, ERTM_ESTATE, "angle capture is off");
    if (src_angle && !c->have_src_angle) return fail(c, ERTM_ESTATE, "no source pass with angles has run");
    if (rcv_angle && !c->have_rcv_angle) return fail(c, ERTM_ESTATE, "no receiver pass with angles has run");
    CK(c, cudaSetDevice(c->device));
    int rc = copy_out_volume(c, c->ang_base[0] + c->g.off0, src_angle);
    if (rc == ERTM_OK) rc = copy_out_volume(c, c->ang_base[1] + c->g.off0, rcv_angle);
    if (rc) return rc;
    CK(c, cudaStreamSynchronize(c->stream));
    return ERTM_OK;
}

int ertm_set_model(ertm_ctx* c, int which, const float* vp, const float* vs, const float* rho)
{
    if (!c) return ERTM_EINVAL;
    if (which != 0 && which != 1) return fail(c, ERTM_EINVAL, "which = %d", which);
    if (!vp || !vs || !rho) return fail(c, ERTM_EINVAL, "NULL model array");
    CK(c, cudaSetDevice(c->device));
    int rc;
    for (int q = 0; q < 5; q++) {
        if (c->m_base[which][q]) continue;
        if ((rc = alloc_volume(c, &c->m_base[which][q], &c->m[which][q]))) return rc;
        if (q < 3 && (rc = encode_map(c, &c->mModel[which][q], c->m_base[which][q], false, TX,
                                      c->g.tyb)))
            return rc;
    }
    if ((rc = ensure_stage(c))) return rc;
    const long long n = (long long)c->g.nx * c->g.ny * c->g.nz;
    const float* src[3] = {vp, vs, rho};
    for (int q = 0; q < 3; q++)
        CK(c, cudaMemcpyAsync(c->stage + q * n, src[q], sizeof(float) * n, cudaMemcpyDefault, c->stream));
    CK(c, launch_model(c->g, c->stage, c->stage + n, c->stage + 2 * n, c->m[which][0], c->m[which][1],
                       c->m[which][2], c->stream));
    CK(c, launch_scatter(c->g, c->stage, c->m[which][3], c->stream));
    CK(c, launch_scatter(c->g, c->stage + n, c->m[which][4], c->stream));
    CK(c, cudaMemsetAsync(c->vmax_d, 0, sizeof(float), c->stream));
    k_absmax<<<std::min<long long>((n + 255) / 256, 148 * 16), 256, 0, c->stream>>>(c->stage, n, c->vmax_d);
    CK(c, cudaGetLastError());
    c->launches += 4;
    float vm = 0.f;
    CK(c, cudaMemcpyAsync(&vm, c->vmax_d, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    if (!(vm > 0.f) || !std::isfinite(vm)) return fail(c, ERTM_EINVAL, "model vp has no positive finite maximum");
    c->vpmax[which] = vm;
    c->model_set[which] = true;
    return ERTM_OK;
}

int ertm_forward_together_using_real_model(ertm_ctx* c, const ertm_shot* s, float* data_out)
{
    if (!c) return ERTM_EINVAL;
    CK(c, cudaSetDevice(c->device));
    int rc = validate_shot(c, s, true);
    if (rc) return rc;
    const long long nrec = nrec_of(s);
    const size_t nd = 3 * (size_t)c->cfg.nt * nrec;
    const bool dev = is_device_ptr(data_out);
    float* traces = nullptr;
    if (data_out && nd) {
        if (dev) traces = data_out;
        else {
            if ((rc = ensure_traces(c, nd))) return rc;
            traces = c->traces;
        }
        CK(c, cudaMemsetAsync(traces, 0, sizeof(float) * nd, c->stream));
    }
    if ((rc = run_pass(c, 0, s, MODE_MODEL, c->cfg.nt, traces))) return rc;
    if (data_out && nd && !dev)
        CK(c, cudaMemcpyAsync(data_out, traces, sizeof(float) * nd, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return ERTM_OK;
}

int ertm_forward_together_using_smoothed_model(ertm_ctx* c, const ertm_shot* s)
{
    if (!c) return ERTM_EINVAL;
    CK(c, cudaSetDevice(c->device));
    int rc = validate_shot(c, s, true);
    if (rc) return rc;
    if ((rc = ensure_excitation(c))) return rc;
    const Geom& g = c->g;
    CK(c, cudaMemsetAsync(c->ex_amp2_base, 0, sizeof(float) * g.total, c->stream));
    CK(c, cudaMemsetAsync(c->ex_time_base, 0, sizeof(int) * g.total, c->stream));
    for (int q = 0; q < 3; q++)
        if (c->ex_v_base[q]) CK(c, cudaMemsetAsync(c->ex_v_base[q], 0, sizeof(float) * g.total, c->stream));
    CK(c, cudaMemsetAsync(c->ex_tp_base, 0, sizeof(float) * g.total, c->stream));
    if (c->angles) CK(c, cudaMemsetAsync(c->ang_base[0], 0, sizeof(float) * g.total, c->stream));
    int nsrc = c->cfg.src_steps > 0 ? c->cfg.src_steps : 2 * c->cfg.nt / 3;
    c->have_excitation = false;
    c->have_src_angle = false;
    if ((rc = run_pass(c, 1, s, MODE_SOURCE, nsrc, nullptr))) return rc;
    CK(c, cudaStreamSynchronize(c->stream));
    c->have_excitation = true;
    c->have_src_angle = c->angles;
    return ERTM_OK;
}

int ertm_backward_together_using_smoothed_model(ertm_ctx* c, const ertm_shot* s, const float* data_in,
                                                float* img_pp, float* img_ps, float* img_tp)
{
    if (!c) return ERTM_EINVAL;
    CK(c, cudaSetDevice(c->device));
    int rc = validate_shot(c, s, false);
    if (rc) return rc;
    if (!c->have_excitation) return fail(c, ERTM_ESTATE, "receiver pass before a source pass");
    if (!data_in && nrec_of(s) > 0) return fail(c, ERTM_EINVAL, "data_in is NULL");
    if ((rc = ensure_images(c))) return rc;
    const Geom& g = c->g;
    for (int q = 0; q < 3; q++) CK(c, cudaMemsetAsync(c->img_base[q], 0, sizeof(float) * g.total, c->stream));
    c->have_rcv_angle = false;
    if (c->angles) CK(c, cudaMemsetAsync(c->ang_base[1], 0, sizeof(float) * g.total, c->stream));
    const long long nrec = nrec_of(s);
    const size_t nd = 3 * (size_t)c->cfg.nt * nrec;
    float* traces = nullptr;
    if (nd) {
        if (is_device_ptr(data_in)) traces = const_cast<float*>(data_in);
        else {
            if ((rc = ensure_traces(c, nd))) return rc;
            CK(c, cudaMemcpyAsync(c->traces, data_in, sizeof(float) * nd, cudaMemcpyHostToDevice, c->stream));
            traces = c->traces;
        }
    }
    if ((rc = run_pass(c, 1, s, MODE_RECEIVER, c->cfg.nt, traces))) return rc;
    c->have_rcv_angle = c->angles;
    float* outs[3] = {img_pp, img_ps, img_tp};
    for (int q = 0; q < 3; q++)
        if ((rc = copy_out_volume(c, c->img_base[q] + g.off0, outs[q]))) return rc;
    CK(c, cudaStreamSynchronize(c->stream));
    return ERTM_OK;
}

int ertm_rtm_shot(ertm_ctx* c, const ertm_shot* s, const float* data_in, float* img_pp, float* img_ps,
                  float* img_tp)
{
    int rc = ertm_forward_together_using_smoothed_model(c, s);
    if (rc) return rc;
    return ertm_backward_together_using_smoothed_model(c, s, data_in, img_pp, img_ps, img_tp);
}

int ertm_rtm_batch(ertm_ctx* c, const ertm_shot* shots, int nshots, const float* const* data,
                   float* stack_pp, float* stack_ps, float* stack_tp)
{
    if (!c) return ERTM_EINVAL;
    if (nshots < 0 || (nshots > 0 && (!shots || !data))) return fail(c, ERTM_EINVAL, "bad shot list");
    CK(c, cudaSetDevice(c->device));
    const Geom& g = c->g;
    const long long n = (long long)g.nx * g.ny * g.nz;
    float* outs[3] = {stack_pp, stack_ps, stack_tp};
    // running sums in the padded layout, gathered once at the end
    float* acc = nullptr;
    CK(c, cudaMalloc(&acc, sizeof(float) * 3 * g.total));
    cudaError_t e = cudaMemsetAsync(acc, 0, sizeof(float) * 3 * g.total, c->stream);
    int rc = e == cudaSuccess ? ERTM_OK : fail(c, ERTM_ECUDA, "%s", cudaGetErrorString(e));
    for (int q = 0; q < nshots && rc == ERTM_OK; q++) {
        // one RTM shot (no per-shot image download), then stack its images
        rc = ertm_forward_together_using_smoothed_model(c, &shots[q]);
        if (rc == ERTM_OK)
            rc = ertm_backward_together_using_smoothed_model(c, &shots[q], data[q], nullptr, nullptr,
                                                             nullptr);
        for (int k = 0; rc == ERTM_OK && k < 3; k++) {
            e = launch_axpy(g.total, c->img_base[k], acc + k * g.total, c->stream);
            if (e != cudaSuccess) rc = fail(c, ERTM_ECUDA, "stack: %s", cudaGetErrorString(e));
            c->launches++;
        }
    }
    for (int k = 0; rc == ERTM_OK && k < 3; k++) rc = copy_out_volume(c, acc + k * g.total + g.off0, outs[k]);
    cudaStreamSynchronize(c->stream);
    cudaFree(acc);
    (void)n;
    return rc;
}

int ertm_rtm_multi(ertm_ctx* const* ctx, int n, const ertm_shot* shots, const float* const* data,
                   float* const* img_pp, float* const* img_ps, float* const* img_tp)
{
    if (!ctx || !ctx[0]) return fail(nullptr, ERTM_EINVAL, "ertm_rtm_multi: no contexts");
    ertm_ctx* c0 = ctx[0];
    if (n < 1 || n > ERTM_MULTI_MAX)
        return fail(c0, ERTM_EINVAL, "ertm_rtm_multi: %d shots (1 .. %d per call)", n, ERTM_MULTI_MAX);
    if (!shots || !data) return fail(c0, ERTM_EINVAL, "ertm_rtm_multi: shots or data is NULL");
    for (int q = 0; q < n; q++) {
        const ertm_ctx* c = ctx[q];
        if (!c) return fail(c0, ERTM_EINVAL, "ertm_rtm_multi: context %d is NULL", q);
        for (int r = 0; r < q; r++)
            if (ctx[r] == c) return fail(c0, ERTM_EINVAL, "ertm_rtm_multi: context %d repeats context %d", q, r);
        if (c->g.two_d) return fail(c0, ERTM_ENOTSUP, "ertm_rtm_multi: 3D grids only (context %d is 2D)", q);
        if (c->device != c0->device || c->g.nz != c0->g.nz || c->R != c0->R ||
            c->cfg.boundary != c0->cfg.boundary)
            return fail(c0, ERTM_EINVAL,
                        "ertm_rtm_multi: context %d differs from context 0 in device, nz, order or boundary", q);
        if (!c->model_set[1]) return fail(c0, ERTM_ESTATE, "ertm_rtm_multi: context %d has no migration model", q);
    }
    CK(c0, cudaSetDevice(c0->device));
    int rc;
    for (int q = 0; q < n; q++) {
        if ((rc = validate_shot(ctx[q], &shots[q], true))) {
            const std::string m = ctx[q]->err;
            return fail(c0, rc, "ertm_rtm_multi: shot %d: %s", q, m.c_str());
        }
        if (nrec_of(&shots[q]) > 0 && !data[q]) return fail(c0, ERTM_EINVAL, "ertm_rtm_multi: data %d is NULL", q);
    }
    // every context's earlier work is done; this call issues all of its work on
    // context 0's stream (the per-context helpers below use c->stream)
    for (int q = 0; q < n; q++) CK(c0, cudaStreamSynchronize(ctx[q]->stream));
    struct StreamSwap {
        ertm_ctx* const* ctx;
        int n;
        cudaStream_t saved[ERTM_MULTI_MAX];
        StreamSwap(ertm_ctx* const* c, int k, cudaStream_t st) : ctx(c), n(k)
        {
            for (int q = 0; q < n; q++) {
                saved[q] = ctx[q]->stream;
                ctx[q]->stream = st;
            }
        }
        ~StreamSwap()
        {
            for (int q = 0; q < n; q++) ctx[q]->stream = saved[q];
        }
    } swap(ctx, n, c0->stream);
    Range range("ertm rtm multi");
    const cudaStream_t st = c0->stream;
    const bool cpml = c0->cfg.boundary == ERTM_BOUNDARY_CPML;
    // every context's boundary profiles on the device before any kernel reads them
    // (the tuner's trial steps run on context 0)
    for (int q = 0; q < n; q++) {
        ertm_ctx* c = ctx[q];
        if ((rc = upload_profiles(c, c->cfg.pml_vmax > 0 ? c->cfg.pml_vmax : c->vpmax[1]))) return rc;
    }
    int kchunk = choose_kchunk(c0->g, c0->R, c0->device);
    if (c0->cfg.autotune == 1 && (rc = autotune_kchunk(c0, 1, &kchunk))) return rc;
    const int chunks = (c0->g.nz + kchunk - 1) / kchunk;
    unsigned gx = 0, gy = 0;
    for (int q = 0; q < n; q++) {
        gx = std::max(gx, (unsigned)((ctx[q]->g.nx + TX - 1) / TX));
        gy = std::max(gy, (unsigned)((ctx[q]->g.ny + TY3 - 1) / TY3));
    }
    const dim3 grid(gx, gy, (unsigned)(n * chunks));
    // the argument blocks travel by value in the kernels' parameter space
    std::unique_ptr<StressMulti> SP(new StressMulti());
    std::unique_ptr<VelMulti> VP(new VelMulti());
    std::memset(SP.get(), 0, sizeof(StressMulti));
    std::memset(VP.get(), 0, sizeof(VelMulti));
    SP->chunks = VP->chunks = chunks;
    auto args_of = [&](int q, float* traces, int it_hi, int epi) {
        ertm_ctx* c = ctx[q];
        KArgs& a = SP->a[q];
        fill_args(c, 1, &shots[q], a);
        a.kchunk = kchunk;
        a.traces = traces;
        a.it_ptr = c0->it_d;   // one step index for every shot of the call
        a.it_hi = it_hi;
        a.pairs = 0;
        if (epi == EPI_IMAGE) a.nw = 0;
        VP->a[q] = a;
        SP->m[q] = stress_maps(c, 1);
        VP->m[q] = vel_maps(c, 1, epi);
    };
    auto loop = [&](int epi, int nsteps, int dir) -> int {
        auto one_step = [&]() -> cudaError_t {
            cudaError_t e = launch_stress_multi(c0->R, grid, *SP, cpml, st);
            if (e == cudaSuccess) e = launch_velocity_multi(c0->R, grid, *VP, cpml, epi, st);
            if (e == cudaSuccess) e = launch_advance(c0->it_d, dir, st);
            return e;
        };
        int r = time_loop(c0, nsteps, one_step);
        c0->launches += 3LL * nsteps;
        return r;
    };

    // source pass: every shot from step 0; a shot with fewer source steps idles
    // (its CTAs return at once) for the rest of the pass
    int nsrc_max = 0;
    for (int q = 0; q < n; q++) {
        ertm_ctx* c = ctx[q];
        const Geom& g = c->g;
        if ((rc = ensure_excitation(c))) return rc;
        CK(c0, cudaMemsetAsync(c->ex_amp2_base, 0, sizeof(float) * g.total, st));
        CK(c0, cudaMemsetAsync(c->ex_time_base, 0, sizeof(int) * g.total, st));
        for (int k = 0; k < 3; k++)
            if (c->ex_v_base[k]) CK(c0, cudaMemsetAsync(c->ex_v_base[k], 0, sizeof(float) * g.total, st));
        CK(c0, cudaMemsetAsync(c->ex_tp_base, 0, sizeof(float) * g.total, st));
        c->have_excitation = false;
        const float vmax = c->cfg.pml_vmax > 0 ? c->cfg.pml_vmax : c->vpmax[1];
        if ((rc = upload_profiles(c, vmax))) return rc;
        if ((rc = reset_state(c))) return rc;
        if ((rc = upload_wavelet(c, &shots[q]))) return rc;
        const int nsrc = c->cfg.src_steps > 0 ? c->cfg.src_steps : 2 * c->cfg.nt / 3;
        args_of(q, nullptr, nsrc, EPI_EXCITE);
        nsrc_max = std::max(nsrc_max, nsrc);
    }
    CK(c0, launch_set_int(c0->it_d, 0, st));
    c0->launches++;
    if ((rc = loop(EPI_EXCITE, nsrc_max, 1))) return rc;
    for (int q = 0; q < n; q++) ctx[q]->have_excitation = true;

    // receiver pass: the step index runs down from the longest shot's last step;
    // a shot joins when it reaches its own last step (its first residual sample is
    // injected up front: its wavefields stay untouched until it joins)
    int nt_max = 0;
    for (int q = 0; q < n; q++) {
        ertm_ctx* c = ctx[q];
        const Geom& g = c->g;
        if ((rc = ensure_images(c))) return rc;
        for (int k = 0; k < 3; k++) CK(c0, cudaMemsetAsync(c->img_base[k], 0, sizeof(float) * g.total, st));
        const long long nrec = nrec_of(&shots[q]);
        const size_t nd = 3 * (size_t)c->cfg.nt * nrec;
        float* traces = nullptr;
        if (nd) {
            if (is_device_ptr(data[q])) traces = const_cast<float*>(data[q]);
            else {
                if ((rc = ensure_traces(c, nd))) return rc;
                CK(c0, cudaMemcpyAsync(c->traces, data[q], sizeof(float) * nd, cudaMemcpyHostToDevice, st));
                traces = c->traces;
            }
        }
        if ((rc = reset_state(c))) return rc;
        args_of(q, traces, c->cfg.nt, EPI_IMAGE);
        if (c->cfg.nt > 0) {
            CK(c0, launch_inject(SP->a[q], c->cfg.nt - 1, st));
            c0->launches++;
        }
        nt_max = std::max(nt_max, c->cfg.nt);
    }
    CK(c0, launch_set_int(c0->it_d, nt_max - 1, st));
    c0->launches++;
    if ((rc = loop(EPI_IMAGE, nt_max, -1))) return rc;
    for (int q = 0; q < n; q++) {
        ertm_ctx* c = ctx[q];
        float* outs[3] = {img_pp ? img_pp[q] : nullptr, img_ps ? img_ps[q] : nullptr,
                          img_tp ? img_tp[q] : nullptr};
        for (int k = 0; k < 3; k++)
            if ((rc = copy_out_volume(c, c->img_base[k] + c->g.off0, outs[k]))) return rc;
    }
    for (int q = 0; q < n; q++)
        if ((rc = check_device_error(ctx[q]))) {
            const std::string m = ctx[q]->err;
            return fail(c0, rc, "ertm_rtm_multi: shot %d: %s", q, m.c_str());
        }
    CK(c0, cudaStreamSynchronize(st));
    return ERTM_OK;
}

int ertm_get_wavefield(ertm_ctx* c, int field, float* out)
{
    if (!c) return ERTM_EINVAL;
    if (field < 0 || field >= NFIELD) return fail(c, ERTM_EINVAL, "field %d", field);
    if (!out) return fail(c, ERTM_EINVAL, "out is NULL");
    CK(c, cudaSetDevice(c->device));
    if (!c->f[field]) {
        long long n = (long long)c->g.nx * c->g.ny * c->g.nz;
        if (is_device_ptr(out)) CK(c, cudaMemsetAsync(out, 0, sizeof(float) * n, c->stream));
        else std::memset(out, 0, sizeof(float) * n);
        CK(c, cudaStreamSynchronize(c->stream));
        return ERTM_OK;
    }
    return copy_out_volume(c, c->f[field], out);
}

int ertm_get_excitation(ertm_ctx* c, float* amp, int32_t* time, float* evx, float* evy, float* evz,
                        float* etp)
{
    if (!c) return ERTM_EINVAL;
    if (!c->have_excitation) return fail(c, ERTM_ESTATE, "no source pass has run");
    CK(c, cudaSetDevice(c->device));
    const Geom& g = c->g;
    const long long n = (long long)g.nx * g.ny * g.nz;
    int rc = ensure_stage(c);
    if (rc) return rc;
    if (amp) {
        CK(c, launch_sqrt_gather(g, c->ex_amp2_base + g.off0, c->stage, c->stream));
        CK(c, cudaMemcpyAsync(amp, c->stage, sizeof(float) * n, cudaMemcpyDefault, c->stream));
    }
    if (time) {
        CK(c, launch_gather_int(g, c->ex_time_base + g.off0, (int*)c->stage, c->stream));
        CK(c, cudaMemcpyAsync(time, c->stage, sizeof(int) * n, cudaMemcpyDefault, c->stream));
    }
    CK(c, cudaStreamSynchronize(c->stream));
    float* outs[4] = {evx, evy, evz, etp};
    float* srcs[4] = {c->ex_v_base[0], c->ex_v_base[1], c->ex_v_base[2], c->ex_tp_base};
    for (int q = 0; q < 4; q++) {
        if (!outs[q]) continue;
        if (!srcs[q]) {
            if (is_device_ptr(outs[q])) CK(c, cudaMemsetAsync(outs[q], 0, sizeof(float) * n, c->stream));
            else std::memset(outs[q], 0, sizeof(float) * n);
            continue;
        }
        if ((rc = copy_out_volume(c, srcs[q] + g.off0, outs[q]))) return rc;
    }
    CK(c, cudaStreamSynchronize(c->stream));
    return ERTM_OK;
}

int ertm_divcurl(ertm_ctx* c, int which, float* p, float* sx, float* sy, float* sz)
{
    if (!c) return ERTM_EINVAL;
    if (which != 0 && which != 1) return fail(c, ERTM_EINVAL, "which = %d", which);
    if (!c->model_set[which]) return fail(c, ERTM_ESTATE, "model %d not set", which);
    if (!p || !sy || (!c->g.two_d && (!sx || !sz))) return fail(c, ERTM_EINVAL, "NULL output");
    CK(c, cudaSetDevice(c->device));
    const Geom& g = c->g;
    const long long n = (long long)g.nx * g.ny * g.nz;
    KArgs a;
    fill_args(c, which, nullptr, a);
    float* outs[4] = {p, sx, sy, sz};
    bool dev[4];
    float* tmp[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int q = 0; q < 4; q++) {
        dev[q] = is_device_ptr(outs[q]);
        if (!outs[q] || (g.two_d && (q == 1 || q == 3))) continue;
        if (dev[q]) tmp[q] = outs[q];
        else CK(c, cudaMalloc(&tmp[q], sizeof(float) * n));
    }
    cudaError_t e = launch_divcurl(c->R, g, a, c->m[which][3], c->m[which][4], tmp[0], tmp[1], tmp[2],
                                   tmp[3], c->stream);
    c->launches++;
    for (int q = 0; q < 4 && e == cudaSuccess; q++)
        if (tmp[q] && !dev[q])
            e = cudaMemcpyAsync(outs[q], tmp[q], sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    for (int q = 0; q < 4; q++)
        if (tmp[q] && !dev[q]) cudaFree(tmp[q]);
    if (e != cudaSuccess) return fail(c, ERTM_ECUDA, "divcurl: %s", cudaGetErrorString(e));
    return ERTM_OK;
}

int ertm_propagate(ertm_ctx* c, int which, const ertm_shot* s, int nsteps)
{
    if (!c) return ERTM_EINVAL;
    if (which != 0 && which != 1) return fail(c, ERTM_EINVAL, "which = %d", which);
    if (nsteps < 0) return fail(c, ERTM_EINVAL, "nsteps = %d", nsteps);
    CK(c, cudaSetDevice(c->device));
    int rc = validate_shot(c, s, true);
    if (rc) return rc;
    if ((rc = run_pass(c, which, s, MODE_MODEL, nsteps, nullptr))) return rc;
    CK(c, cudaStreamSynchronize(c->stream));
    return ERTM_OK;
}

int ertm_time_kernels(ertm_ctx* c, const ertm_shot* s, int nsteps, float* ms)
{
    if (!c || !ms) return ERTM_EINVAL;
    if (nsteps < 1) return fail(c, ERTM_EINVAL, "nsteps = %d", nsteps);
    CK(c, cudaSetDevice(c->device));
    int rc = validate_shot(c, s, true);
    if (rc) return rc;
    if (!c->model_set[1]) return fail(c, ERTM_ESTATE, "migration model not set");
    if ((rc = ensure_excitation(c))) return rc;
    float vmax = c->cfg.pml_vmax > 0 ? c->cfg.pml_vmax : c->vpmax[1];
    if ((rc = upload_profiles(c, vmax))) return rc;
    if ((rc = reset_state(c))) return rc;
    if ((rc = upload_wavelet(c, s))) return rc;
    KArgs a;
    fill_args(c, 1, s, a);
    a.kchunk = choose_kchunk(c->g, c->R, c->device);
    const bool cpml = c->cfg.boundary == ERTM_BOUNDARY_CPML;
    cudaEvent_t ev[3];
    for (int q = 0; q < 3; q++) CK(c, cudaEventCreate(&ev[q]));
    CK(c, launch_set_int(c->it_d, 0, c->stream));
    float tot[2] = {0.f, 0.f};
    const StressMaps sm = stress_maps(c, 1);
    const VelMaps vm = vel_maps(c, 1, EPI_EXCITE);
    for (int step = 0; step < nsteps; step++) {
        CK(c, cudaEventRecord(ev[0], c->stream));
        CK(c, launch_stress(c->R, c->g, a, sm, cpml, true, c->stream));
        CK(c, cudaEventRecord(ev[1], c->stream));
        CK(c, launch_velocity(c->R, c->g, a, vm, cpml, EPI_EXCITE, false, c->stream));
        CK(c, cudaEventRecord(ev[2], c->stream));
        CK(c, launch_advance(c->it_d, 1, c->stream));
        c->launches += 3;
        CK(c, cudaEventSynchronize(ev[2]));
        float t0, t1;
        CK(c, cudaEventElapsedTime(&t0, ev[0], ev[1]));
        CK(c, cudaEventElapsedTime(&t1, ev[1], ev[2]));
        tot[0] += t0;
        tot[1] += t1;
    }
    for (int q = 0; q < 3; q++) cudaEventDestroy(ev[q]);
    c->have_excitation = false;
    ms[0] = tot[0];
    ms[1] = tot[1];
    return check_device_error(c);
}

int64_t ertm_kernel_launches(const ertm_ctx* c) { return c ? c->launches : 0; }

int ertm_set_step_variant(ertm_ctx* c, int variant)
{
    if (!c) return ERTM_EINVAL;
    if (variant != ERTM_STEP_PAIRS && variant != ERTM_STEP_SINGLE)
        return fail(c, ERTM_EINVAL, "step variant %d", variant);
    c->pairs = variant == ERTM_STEP_PAIRS;
    return ERTM_OK;
}

int ertm_set_wait_fault(ertm_ctx* c, int plane, uint32_t polls)
{
    if (!c) return ERTM_EINVAL;
    if (plane < -1) return fail(c, ERTM_EINVAL, "plane = %d", plane);
    c->skip_plane1 = plane + 1;
    c->wait_polls = polls;
    return ERTM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Born modelling and adjoint (2D, sponge boundaries)
// ---------------------------------------------------------------------------
namespace {

// Shared compact volumes: model products, damping factors, perturbation products.
enum { SV_M, SV_U, SV_BG1, SV_B, SV_G1, SV_G2, SV_DM, SV_DU, SV_RR, SV_N };
// Per-shot compact volume types, each [shot][n] over a group of shots: background
// state (5 fields + 9 memory variables, contiguous so that a checkpoint of every shot
// is one copy), scattered state and memory variables, adjoint state, gradient
// accumulators (pi, unused, mu, rho), adjoint memory variables, strain-adjoint scratch.
enum { PV_BG = 0, PV_R0 = PV_BG + 5, PV_SC = PV_R0 + 9, PV_R = PV_SC + 5, PV_ADJ = PV_R + 9,
       PV_GRAD = PV_ADJ + 5, PV_LR = PV_GRAD + 4, PV_S = PV_LR + 9, PV_N = PV_S + 3 };
static_assert(PV_N <= 64 && SV_N <= 16, "BornState volume tables");
constexpr int kBornMaxShots = 256;   // shots per launch (grid z)

// GSLS fit (tau method, first order): relaxation frequencies
// f_l = f0 10^(2 (l + 1/2) / nm - 1), tau_sigma = 1 / (2 pi f_l);
// Q^-1(w) ~ tau S(w), S(w) = sum_l w tau_sigma / (1 + w^2 tau_sigma^2), fitted in
// least squares to constant 1/q at 32 log-spaced frequencies in [f0/4, 4 f0]
void visco_fit(int nm, double qp, double qs, double f0, double* tau_sigma, double* tp, double* ts)
{
    const double pi = 3.14159265358979323846;
    for (int l = 0; l < nm; l++) tau_sigma[l] = 1.0 / (2.0 * pi * f0 * std::pow(10.0, 2.0 * (l + 0.5) / nm - 1.0));
    double s1 = 0, s2 = 0;
    for (int j = 0; j < 32; j++) {
        const double w = 2.0 * pi * f0 / 4.0 * std::pow(16.0, j / 31.0);
        double S = 0;
        for (int l = 0; l < nm; l++) S += w * tau_sigma[l] / (1.0 + w * w * tau_sigma[l] * tau_sigma[l]);
        s1 += S;
        s2 += S * S;
    }
    *tp = (1.0 / qp) * s1 / s2;
    *ts = (1.0 / qs) * s1 / s2;
}

int born_check(ertm_ctx* c, const ertm_shot* shots, int nshots)
{
    if (!c->g.two_d) return fail(c, ERTM_ENOTSUP, "Born operators support 2D grids only");
    if (c->cfg.boundary == ERTM_BOUNDARY_CPML)
        return fail(c, ERTM_ENOTSUP, "Born operators support sponge boundaries only");
    if (!c->model_set[1]) return fail(c, ERTM_ESTATE, "migration model not set");
    if (!shots || nshots < 1) return fail(c, ERTM_EINVAL, "no shots");
    for (int i = 0; i < nshots; i++) {
        int rc = validate_shot(c, &shots[i], true);
        if (rc) return rc;
        if (shots[i].nrx != shots[0].nrx || shots[i].nw != shots[0].nw)
            return fail(c, ERTM_EINVAL, "shots of one call need the same receiver count and wavelet length");
    }
    return ERTM_OK;
}

// shared volumes and the argument block (shot-independent part); model products
// copied from the migration model
int born_prepare(ertm_ctx* c, BornArgs& a)
{
    auto& B = c->born;
    const Geom& g = c->g;
    int rc;
    if (!B.ready) {
        CK(c, cudaStreamSynchronize(c->stream));
        cudaFree(B.shared);
        cudaFree(B.block);
        cudaFree(B.ckpt);
        cudaFree(B.hist);
        B.shared = B.block = B.ckpt = B.hist = nullptr;
        B.G = 0;
        B.ckpt_floats = B.hist_floats = 0;
        B.px = round_up(2LL * BXH + round_up(g.nx, 32), 32);
        B.n = B.px * (g.nz + 2LL * c->R);
        CK(c, cudaMalloc(&B.shared, sizeof(float) * B.n * SV_N));
        CK(c, cudaMemsetAsync(B.shared, 0, sizeof(float) * B.n * SV_N, c->stream));
        for (int q = 0; q < SV_N; q++) B.sv[q] = B.shared + (size_t)q * B.n;
        B.ready = true;
    }
    if ((rc = upload_profiles(c, 0.f))) return rc;
    std::memset(&a, 0, sizeof a);
    a.nx = g.nx;
    a.nz = g.nz;
    a.R = c->R;
    a.px = B.px;
    for (int q = 0; q < 8; q++) {
        a.cx[q] = (float)(c->coef[q] / c->cfg.dx);
        a.cz[q] = (float)(c->coef[q] / c->cfg.dz);
    }
    a.dt = c->cfg.dt_ms / 1000.f;
    a.M = B.sv[SV_M]; a.U = B.sv[SV_U]; a.Bg1 = B.sv[SV_BG1]; a.B = B.sv[SV_B];
    a.g1 = B.sv[SV_G1]; a.g2 = B.sv[SV_G2];
    a.dM = B.sv[SV_DM]; a.dU = B.sv[SV_DU]; a.rr = B.sv[SV_RR];
    a.nm = c->cfg.visco_nmech;
    a.kp = a.ks = 1.f;
    a.tp = a.ts = 0.f;
    for (int l = 0; l < 3; l++) a.ra[l] = a.rb[l] = 0.f;
    if (a.nm > 0) {
        double tau[3], tp, ts;
        visco_fit(a.nm, c->cfg.visco_qp, c->cfg.visco_qs, c->cfg.visco_f0, tau, &tp, &ts);
        a.tp = (float)tp;
        a.ts = (float)ts;
        a.kp = (float)(1.0 + a.nm * tp);
        a.ks = (float)(1.0 + a.nm * ts);
        for (int l = 0; l < a.nm; l++) {
            const double h = c->cfg.dt_ms / 1000.0 / (2.0 * tau[l]);
            a.ra[l] = (float)((1.0 - h) / (1.0 + h));
            a.rb[l] = (float)(-2.0 * h / (1.0 + h));
        }
    }
    a.nt = c->cfg.nt;
    a.nshot = 1;
    a.ss = B.n;
    CK(c, born_launch_model(a, c->m[1][0], c->m[1][1], c->m[1][2], g.sz, c->att[0], c->att[2],
                            B.sv[SV_M], B.sv[SV_U], B.sv[SV_BG1], B.sv[SV_B], B.sv[SV_G1], B.sv[SV_G2],
                            c->stream));
    c->launches++;
    return ERTM_OK;
}

// per-shot volumes for a group of G shots (grown on demand; the type stride is G n)
int born_group_volumes(ertm_ctx* c, int G)
{
    auto& B = c->born;
    if (B.G < G) {
        CK(c, cudaStreamSynchronize(c->stream));
        cudaFree(B.block);
        B.block = nullptr;
        B.G = 0;
        CK(c, cudaMalloc(&B.block, sizeof(float) * B.n * PV_N * G));
        B.G = G;
    }
    return ERTM_OK;
}

// lay the per-shot volumes of a group of G shots out densely (type q at q G n, shot
// s at + s n) and point the per-shot arguments at them
void born_group_args(ertm_ctx* c, BornArgs& a, int G)
{
    auto& B = c->born;
    for (int q = 0; q < PV_N; q++) B.pv[q] = B.block + (size_t)q * G * B.n;
    a.nshot = G;
    a.ss = B.n;
    float** bg[5] = {&a.v0x, &a.v0z, &a.s0xx, &a.s0zz, &a.s0xz};
    float** sc[5] = {&a.vx, &a.vz, &a.sxx, &a.szz, &a.sxz};
    float** ad[5] = {&a.ax, &a.az, &a.hxx, &a.hzz, &a.hxz};
    for (int q = 0; q < 5; q++) {
        *bg[q] = B.pv[PV_BG + q];
        *sc[q] = B.pv[PV_SC + q];
        *ad[q] = B.pv[PV_ADJ + q];
    }
    a.gM = B.pv[PV_GRAD]; a.gL = B.pv[PV_GRAD + 1]; a.gU = B.pv[PV_GRAD + 2];
    a.gR = B.pv[PV_GRAD + 3];
    for (int q = 0; q < 9; q++) {
        a.r0[q] = B.pv[PV_R0 + q];
        a.r[q] = B.pv[PV_R + q];
        a.lr[q] = B.pv[PV_LR + q];
    }
    a.Sxx = B.pv[PV_S]; a.Szz = B.pv[PV_S + 1]; a.Sxz = B.pv[PV_S + 2];
}

// shot table and wavelets of shots[0..G) on the device
int born_group_shots(ertm_ctx* c, BornArgs& a, const ertm_shot* shots, int G)
{
    auto& B = c->born;
    const int nw = shots[0].nw;
    if (B.tab_cap < G) {
        cudaFree(B.tab);
        B.tab = nullptr;
        B.tab_cap = 0;
        CK(c, cudaMalloc(&B.tab, sizeof(int) * 8 * G));
        B.tab_cap = G;
    }
    const long long wn = (long long)G * (nw > 0 ? nw : 1);
    if (B.wav_cap < wn) {
        cudaFree(B.wav);
        B.wav = nullptr;
        B.wav_cap = 0;
        CK(c, cudaMalloc(&B.wav, sizeof(float) * wn));
        B.wav_cap = wn;
    }
    std::vector<int> tab(8 * (size_t)G, 0);
    for (int s = 0; s < G; s++) {
        const ertm_shot& sh = shots[s];
        int* t = &tab[8 * (size_t)s];
        t[0] = sh.sx; t[1] = sh.sz; t[2] = sh.rx0; t[3] = sh.nrx; t[4] = sh.drx; t[5] = sh.rz;
        if (nw > 0)
            CK(c, cudaMemcpyAsync(B.wav + (size_t)s * nw, sh.wavelet, sizeof(float) * nw, cudaMemcpyDefault,
                                  c->stream));
    }
    CK(c, cudaMemcpyAsync(B.tab, tab.data(), sizeof(int) * 8 * G, cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));   // the host table is a temporary
    a.shot_tab = B.tab;
    a.nw = nw;
    a.wavelet = B.wav;
    a.wstride = nw > 0 ? nw : 1;
    a.nrx = shots[0].nrx;
    return ERTM_OK;
}

int born_zero_types(ertm_ctx* c, int first, int count, int G)
{
    CK(c, cudaMemsetAsync(c->born.pv[first], 0, sizeof(float) * c->born.n * G * count, c->stream));
    return ERTM_OK;
}

// contiguous nz*nx device copies of up to three caller arrays (stage)
int born_stage_in(ertm_ctx* c, const float* const* src, int count, const float** out)
{
    int rc = ensure_stage(c);
    if (rc) return rc;
    const long long n = (long long)c->g.nx * c->g.nz;
    for (int q = 0; q < count; q++) {
        if (is_device_ptr(src[q])) {
            out[q] = src[q];
            continue;
        }
        CK(c, cudaMemcpyAsync(c->stage + q * n, src[q], sizeof(float) * n, cudaMemcpyHostToDevice,
                              c->stream));
        out[q] = c->stage + q * n;
    }
    return ERTM_OK;
}

// Shots per launch: at most `want`, bounded so that the group's volumes (and, for the
// adjoint, its checkpoints and history) take at most about 60 % of the free memory.
int born_group_size(ertm_ctx* c, int want, long long floats_per_shot)
{
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    // memory the context already holds for a group counts as available
    const long long held = (long long)c->born.G * c->born.n * PV_N + c->born.ckpt_floats + c->born.hist_floats;
    const double avail = 0.6 * (double)free_b + 4.0 * (double)held;
    long long g = (long long)(avail / (4.0 * (double)floats_per_shot));
    if (g > want) g = want;
    if (g > kBornMaxShots) g = kBornMaxShots;
    return g < 1 ? 1 : (int)g;
}

}  // namespace

extern "C" {

int ertm_born_forward_shots(ertm_ctx* c, const ertm_shot* shots, int nshots, const float* r_vp,
                            const float* r_vs, const float* r_rho, float* data_out)
{
    if (!c) return ERTM_EINVAL;
    Range range("ertm born forward");
    if (!r_vp || !r_vs || !r_rho || !data_out) return fail(c, ERTM_EINVAL, "NULL argument");
    CK(c, cudaSetDevice(c->device));
    int rc = born_check(c, shots, nshots);
    if (rc) return rc;
    BornArgs a;
    if ((rc = born_prepare(c, a))) return rc;
    const float* src[3] = {r_vp, r_vs, r_rho};
    const float* dev[3];
    if ((rc = born_stage_in(c, src, 3, dev))) return rc;
    auto& B = c->born;
    CK(c, born_launch_pert(a, dev[0], dev[1], dev[2], B.sv[SV_DM], B.sv[SV_DU], B.sv[SV_RR], c->stream));
    c->launches++;
    const int nt = c->cfg.nt;
    const long long nd = 3LL * nt * shots[0].nrx;   // floats of one shot's traces
    const bool dev_out = is_device_ptr(data_out);
    const int G = born_group_size(c, nshots, B.n * (long long)PV_N + (dev_out ? 0 : nd));
    if ((rc = born_group_volumes(c, G))) return rc;
    if (!dev_out && (rc = ensure_traces(c, (size_t)nd * G))) return rc;
    for (int s0 = 0; s0 < nshots; s0 += G) {
        const int g = std::min(G, nshots - s0);
        born_group_args(c, a, g);
        if ((rc = born_group_shots(c, a, shots + s0, g))) return rc;
        a.tstride = nd;
        a.traces = dev_out ? data_out + (size_t)s0 * nd : c->traces;
        // background and scattered states of the group (types BG .. R, contiguous)
        if ((rc = born_zero_types(c, PV_BG, PV_ADJ - PV_BG, g))) return rc;
        CK(c, cudaMemsetAsync(a.traces, 0, sizeof(float) * nd * g, c->stream));
        for (int it = 0; it < nt; it++) CK(c, born_launch_step(a, it, true, false, c->stream));
        c->launches += 2LL * nt;
        if (!dev_out)
            CK(c, cudaMemcpyAsync(data_out + (size_t)s0 * nd, a.traces, sizeof(float) * nd * g,
                                  cudaMemcpyDeviceToHost, c->stream));
    }
    CK(c, cudaStreamSynchronize(c->stream));
    return ERTM_OK;
}

int ertm_born_forward(ertm_ctx* c, const ertm_shot* s, const float* r_vp, const float* r_vs,
                      const float* r_rho, float* data_out)
{
    return ertm_born_forward_shots(c, s, 1, r_vp, r_vs, r_rho, data_out);
}

int ertm_born_adjoint_shots(ertm_ctx* c, const ertm_shot* shots, int nshots, const float* residual,
                            float* g_vp, float* g_vs, float* g_rho)
{
    if (!c) return ERTM_EINVAL;
    Range range("ertm born adjoint");
    if (!residual || !g_vp || !g_vs || !g_rho) return fail(c, ERTM_EINVAL, "NULL argument");
    CK(c, cudaSetDevice(c->device));
    int rc = born_check(c, shots, nshots);
    if (rc) return rc;
    BornArgs a;
    if ((rc = born_prepare(c, a))) return rc;
    auto& B = c->born;
    const int nt = c->cfg.nt;
    const int K = std::min(nt, c->cfg.checkpoint_every > 0 ? c->cfg.checkpoint_every : 200);
    const int nck = (nt + K - 1) / K;
    const int nbg = 5 + (a.nm ? 9 : 0);   // background volume types in a checkpoint
    const long long nd = 3LL * nt * shots[0].nrx;
    const bool dev_res = is_device_ptr(residual);
    const long long per_shot = B.n * ((long long)PV_N + 14LL * nck + 4LL * K) + (dev_res ? 0 : nd);
    const int G = born_group_size(c, nshots, per_shot);
    if ((rc = born_group_volumes(c, G))) return rc;
    const long long ck_need = 14LL * nck * G * B.n, hist_need = 4LL * K * G * B.n;
    if (B.ckpt_floats < ck_need) {
        cudaFree(B.ckpt);
        B.ckpt = nullptr;
        B.ckpt_floats = 0;
        CK(c, cudaMalloc(&B.ckpt, sizeof(float) * ck_need));
        B.ckpt_floats = ck_need;
    }
    if (B.hist_floats < hist_need) {
        cudaFree(B.hist);
        B.hist = nullptr;
        B.hist_floats = 0;
        CK(c, cudaMalloc(&B.hist, sizeof(float) * hist_need));
        B.hist_floats = hist_need;
    }
    if (!dev_res && (rc = ensure_traces(c, (size_t)nd * G))) return rc;
    // gradient targets: the caller's device arrays, or the stage for host arrays
    float* outs[3] = {g_vp, g_vs, g_rho};
    const long long n = (long long)c->g.nx * c->g.nz;
    bool dev[3];
    for (int q = 0; q < 3; q++) dev[q] = is_device_ptr(outs[q]);
    if (!(dev[0] && dev[1] && dev[2]) && (rc = ensure_stage(c))) return rc;
    float* tgt[3];
    for (int q = 0; q < 3; q++) tgt[q] = dev[q] ? outs[q] : c->stage + q * n;
    for (int s0 = 0; s0 < nshots; s0 += G) {
        const int g = std::min(G, nshots - s0);
        born_group_args(c, a, g);
        if ((rc = born_group_shots(c, a, shots + s0, g))) return rc;
        a.tstride = nd;
        if (dev_res) a.traces = const_cast<float*>(residual) + (size_t)s0 * nd;
        else {
            CK(c, cudaMemcpyAsync(c->traces, residual + (size_t)s0 * nd, sizeof(float) * nd * g,
                                  cudaMemcpyHostToDevice, c->stream));
            a.traces = c->traces;
        }
        const size_t ck_seg = (size_t)nbg * g * B.n;   // floats of one checkpoint of the group
        // 1. background forward, checkpointing every shot's state every K steps
        if ((rc = born_zero_types(c, PV_BG, 14, g))) return rc;
        // the group's background types (BG, R0) are contiguous: one copy per checkpoint
        auto save = [&](int seg) {
            return cudaMemcpyAsync(B.ckpt + seg * ck_seg, B.pv[PV_BG], sizeof(float) * ck_seg,
                                   cudaMemcpyDeviceToDevice, c->stream);
        };
        auto load = [&](int seg) {
            return cudaMemcpyAsync(B.pv[PV_BG], B.ckpt + seg * ck_seg, sizeof(float) * ck_seg,
                                   cudaMemcpyDeviceToDevice, c->stream);
        };
        for (int it = 0; it < nt; it++) {
            if (it % K == 0) CK(c, save(it / K));
            CK(c, born_launch_step(a, it, false, false, c->stream));
        }
        // 2. reverse sweep, one checkpoint segment at a time
        if ((rc = born_zero_types(c, PV_ADJ, PV_N - PV_ADJ, g))) return rc;   // adjoint, gradients, scratch
        CK(c, born_launch_inject(a, nt - 1, c->stream));
        for (int sg = nck - 1; sg >= 0; sg--) {
            const int t0 = sg * K, t1 = std::min(nt, t0 + K);
            CK(c, load(sg));
            for (int it = t0; it < t1; it++) {
                float* h = B.hist + (size_t)(it - t0) * 4 * g * B.n;
                a.kv0x = h;
                a.kv0z = h + g * B.n;
                a.ka0x = h + 2 * g * B.n;
                a.ka0z = h + 3 * g * B.n;
                CK(c, born_launch_step(a, it, false, true, c->stream));
            }
            for (int it = t1 - 1; it >= t0; it--) {
                const float* h = B.hist + (size_t)(it - t0) * 4 * g * B.n;
                a.hv0x = h;
                a.hv0z = h + g * B.n;
                a.ha0x = h + 2 * g * B.n;
                a.ha0z = h + 3 * g * B.n;
                CK(c, born_launch_adjoint_step(a, it, c->stream));
            }
        }
        c->launches += 2LL * nt * 2 + 3LL * nt + 1;
        // 3. gradients w.r.t. the relative perturbations, summed over the group's shots
        CK(c, born_launch_final(a, tgt[0], tgt[1], tgt[2], s0 > 0, c->stream));
        c->launches++;
    }
    for (int q = 0; q < 3; q++)
        if (!dev[q])
            CK(c, cudaMemcpyAsync(outs[q], tgt[q], sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return ERTM_OK;
}

int ertm_born_adjoint(ertm_ctx* c, const ertm_shot* s, const float* residual, float* g_vp,
                      float* g_vs, float* g_rho)
{
    return ertm_born_adjoint_shots(c, s, 1, residual, g_vp, g_vs, g_rho);
}

}  // extern "C"
