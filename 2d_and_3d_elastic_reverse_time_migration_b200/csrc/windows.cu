// Batched RTM over aperture windows of one shared model (ertm_rtm_windows).
//
// Every shot migrates on its own window: the shared migration model cropped to
// the window laterally (full depth), extended by the absorbing layers with edge
// values, and its images are added into one stacked volume of the model's size.
// The shots run in groups of up to ERTM_MULTI_MAX through ertm_rtm_multi: one
// context per shot of a group (allocated once for the largest window and shrunk
// to each shot's window with ertm_set_grid), all on one stream, and every time
// step of a group is one launch of each step kernel covering all of its shots.
// Shots are taken in decreasing order of cost, so a group's shots have similar
// sizes and step counts, and their images are stacked in that order: the sum
// does not depend on the group size.  Built on the public C ABI plus two small
// kernels (crop, stack); the reference migrates one shot per run on the full
// grid (3D_elastic_RTM/3D_output_file.cu:339-365).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ertm.h"

namespace {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// dst[k][j][i] = src[clamp(k+oz)][clamp(j+oy)][clamp(i+ox)] for the three model arrays
__global__ void k_crop_pad(const float* __restrict__ vp, const float* __restrict__ vs,
                           const float* __restrict__ rho, int NX, int NY, int NZ, int ox, int oy,
                           int oz, float* __restrict__ out, int nx, int ny, int nz)
{
    const long long n = (long long)nx * ny * nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % nx), j = (int)((q / nx) % ny), k = (int)(q / ((long long)nx * ny));
        const long long s = ((long long)clampi(k + oz, 0, NZ - 1) * NY + clampi(j + oy, 0, NY - 1)) * NX +
                            clampi(i + ox, 0, NX - 1);
        out[q] = vp[s];
        out[n + q] = vs[s];
        out[2 * n + q] = rho[s];
    }
}

// stack[k][y0+j][x0+i] += img[k+pz][j+py][i+px] over the window interior (wx x wy x NZ)
__global__ void k_stack_window(const float* __restrict__ img, int nx, int ny, int nz, int px, int py,
                               int pz, float* __restrict__ stack, int NX, int NY, int NZ, int x0,
                               int y0, int wx, int wy)
{
    const long long n = (long long)wx * wy * NZ, wn = (long long)nx * ny * nz, sn = (long long)NX * NY * NZ;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % wx), j = (int)((q / wx) % wy), k = (int)(q / ((long long)wx * wy));
        const long long w = ((long long)(k + pz) * ny + (j + py)) * nx + (i + px);
        const long long s = ((long long)k * NY + (j + y0)) * NX + (i + x0);
        for (int c = 0; c < 3; c++) stack[c * sn + s] += img[c * wn + w];
    }
}

void put_err(char* buf, size_t len, const std::string& m)
{
    if (!buf || !len) return;
    size_t n = std::min(len - 1, m.size());
    std::memcpy(buf, m.data(), n);
    buf[n] = 0;
}

struct Slot {
    ertm_ctx* ctx = nullptr;
    float* model = nullptr;   // 3 x cap cells (window grid)
    float* img = nullptr;     // 3 x cap cells (window grid)
};

}  // namespace

extern "C" int ertm_rtm_windows(const ertm_config* base, const float* vp, const float* vs,
                                const float* rho, int nshots, const ertm_window* win,
                                const ertm_shot* shots, const float* const* data, int lanes,
                                float* stack_pp, float* stack_ps, float* stack_tp, char* errbuf,
                                size_t errlen)
{
    auto bad = [&](int code, const std::string& m) {
        put_err(errbuf, errlen, m);
        return code;
    };
    if (!base || !vp || !vs || !rho) return bad(ERTM_EINVAL, "NULL config or model");
    if (nshots < 0 || (nshots > 0 && (!win || !shots || !data))) return bad(ERTM_EINVAL, "bad shot list");
    if (lanes < 1) return bad(ERTM_EINVAL, "lanes must be >= 1");
    const ertm_config& B = *base;
    const int NX = B.nx, NY = B.ny, NZ = B.nz;
    const bool two_d = (NY == 1);
    if (NX < 1 || NY < 1 || NZ < 1) return bad(ERTM_EINVAL, "model grid");
    const int* p = B.pml;
    const int pxl = p[0], pxr = p[1], pyl = two_d ? 0 : p[2], pyr = two_d ? 0 : p[3], pzt = p[4],
              pzb = p[5];
    // window grids and the capacity of a lane
    int cap_nx = 1, cap_ny = 1, cap_nt = 1;
    char msg[256];
    for (int i = 0; i < nshots; i++) {
        const ertm_window& w = win[i];
        const ertm_shot& s = shots[i];
        if (w.wx < 1 || w.wy < 1 || w.x0 < 0 || w.y0 < 0 || w.x0 + w.wx > NX || w.y0 + w.wy > NY ||
            (two_d && (w.wy != 1 || w.y0 != 0)) || w.nt < 1 || w.src_steps < 0 || w.src_steps > w.nt) {
            snprintf(msg, sizeof msg, "shot %d: window (%d,%d)+(%d,%d) nt %d outside the %dx%d model", i,
                     w.x0, w.y0, w.wx, w.wy, w.nt, NX, NY);
            return bad(ERTM_EINVAL, msg);
        }
        if (s.sx < w.x0 || s.sx >= w.x0 + w.wx || s.sy < w.y0 || s.sy >= w.y0 + w.wy || s.sz < 0 ||
            s.sz >= NZ) {
            snprintf(msg, sizeof msg, "shot %d: source (%d,%d,%d) outside its window", i, s.sx, s.sy, s.sz);
            return bad(ERTM_EINVAL, msg);
        }
        if (s.nrx * s.nry > 0 && !data[i]) {
            snprintf(msg, sizeof msg, "shot %d: data is NULL", i);
            return bad(ERTM_EINVAL, msg);
        }
        cap_nx = std::max(cap_nx, w.wx + pxl + pxr);
        cap_ny = std::max(cap_ny, two_d ? 1 : w.wy + pyl + pyr);
        cap_nt = std::max(cap_nt, w.nt);
    }
    const int nz_w = NZ + pzt + pzb;
    const long long ncap = (long long)cap_nx * cap_ny * nz_w, nmod = (long long)NX * NY * NZ;
    const int G = std::max(1, std::min({lanes, ERTM_MULTI_MAX, std::max(nshots, 1)}));
    if (cudaSetDevice(B.device) != cudaSuccess) {
        cudaGetLastError();
        return bad(ERTM_ECUDA, "cudaSetDevice");
    }

    // shared model, stack and one stream on the device
    const float* mdl[3] = {vp, vs, rho};
    float* dmodel = nullptr;
    float* stack = nullptr;
    cudaStream_t st = nullptr;
    std::vector<Slot> S(G);
    int rc = ERTM_OK;
    std::string err;
    auto cuda_fail = [&](cudaError_t e, const char* what) {
        if (rc == ERTM_OK) {
            rc = e == cudaErrorMemoryAllocation ? ERTM_ENOMEM : ERTM_ECUDA;
            err = std::string(what) + ": " + cudaGetErrorString(e);
        }
    };
    auto api_fail = [&](int r, ertm_ctx* c, const std::string& head) {
        if (rc == ERTM_OK) {
            char b[512];
            ertm_last_error(c, b, sizeof b);
            rc = r;
            err = head + b;
        }
    };
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) cuda_fail(e, "stream");
    if (rc == ERTM_OK && (e = cudaMalloc(&dmodel, sizeof(float) * 3 * nmod)) != cudaSuccess) cuda_fail(e, "model");
    for (int q = 0; q < 3 && rc == ERTM_OK; q++)
        if ((e = cudaMemcpy(dmodel + q * nmod, mdl[q], sizeof(float) * nmod, cudaMemcpyDefault)) != cudaSuccess)
            cuda_fail(e, "model copy");
    if (rc == ERTM_OK && (e = cudaMalloc(&stack, sizeof(float) * 3 * nmod)) != cudaSuccess) cuda_fail(e, "stack");
    if (rc == ERTM_OK && (e = cudaMemsetAsync(stack, 0, sizeof(float) * 3 * nmod, st)) != cudaSuccess)
        cuda_fail(e, "memset");
    for (int l = 0; l < G && rc == ERTM_OK; l++) {
        ertm_config c = B;
        c.nx = cap_nx;
        c.ny = cap_ny;
        c.nz = nz_w;
        c.nt = cap_nt;
        c.src_steps = 0;
        if (two_d) c.pml[2] = c.pml[3] = 0;
        int r = ertm_create(&c, &S[l].ctx);
        if (r) {
            api_fail(r, nullptr, "window context: ");
            break;
        }
        ertm_set_stream(S[l].ctx, st);
        if ((e = cudaMalloc(&S[l].model, sizeof(float) * 3 * ncap)) != cudaSuccess) { cuda_fail(e, "window model"); break; }
        if ((e = cudaMalloc(&S[l].img, sizeof(float) * 3 * ncap)) != cudaSuccess) { cuda_fail(e, "window image"); break; }
    }

    // largest windows first
    std::vector<int> order(nshots);
    for (int i = 0; i < nshots; i++) order[i] = i;
    auto cost = [&](int i) {
        const ertm_window& w = win[i];
        const int ss = w.src_steps ? w.src_steps : 2 * w.nt / 3;
        return (double)(w.wx + pxl + pxr) * (two_d ? 1 : w.wy + pyl + pyr) * (ss + w.nt);
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });

    for (int g0 = 0; g0 < nshots && rc == ERTM_OK; g0 += G) {
        const int m = std::min(G, nshots - g0);
        ertm_ctx* cx[ERTM_MULTI_MAX];
        ertm_shot sh[ERTM_MULTI_MAX];
        const float* dd[ERTM_MULTI_MAX];
        float* pp[ERTM_MULTI_MAX];
        float* ps[ERTM_MULTI_MAX];
        float* tp[ERTM_MULTI_MAX];
        for (int j = 0; j < m && rc == ERTM_OK; j++) {
            const int i = order[g0 + j];
            const ertm_window& w = win[i];
            Slot& sl = S[j];
            const int nx = w.wx + pxl + pxr, ny = two_d ? 1 : w.wy + pyl + pyr;
            const long long n = (long long)nx * ny * nz_w;
            int r = ertm_set_grid(sl.ctx, nx, ny, w.nt, w.src_steps);
            if (!r) {
                k_crop_pad<<<592, 256, 0, st>>>(dmodel, dmodel + nmod, dmodel + 2 * nmod, NX, NY, NZ,
                                                w.x0 - pxl, two_d ? 0 : w.y0 - pyl, -pzt, sl.model, nx, ny, nz_w);
                if ((e = cudaGetLastError()) != cudaSuccess) {
                    cuda_fail(e, "crop");
                    break;
                }
                r = ertm_set_model(sl.ctx, 1, sl.model, sl.model + n, sl.model + 2 * n);
            }
            if (r) {
                char head[64];
                snprintf(head, sizeof head, "shot %d: ", i);
                api_fail(r, sl.ctx, head);
                break;
            }
            ertm_shot s = shots[i];
            s.sx = s.sx - w.x0 + pxl;
            s.sy = two_d ? 0 : s.sy - w.y0 + pyl;
            s.sz = s.sz + pzt;
            s.rx0 = s.rx0 - w.x0 + pxl;
            s.ry0 = two_d ? 0 : s.ry0 - w.y0 + pyl;
            s.rz = s.rz + pzt;
            cx[j] = sl.ctx;
            sh[j] = s;
            dd[j] = data[i];
            pp[j] = sl.img;
            ps[j] = sl.img + n;
            tp[j] = sl.img + 2 * n;
        }
        if (rc != ERTM_OK) break;
        if (two_d) {
            // 2D windows: one shot per call through the single-shot path
            for (int j = 0; j < m && rc == ERTM_OK; j++) {
                int r = ertm_rtm_shot(cx[j], &sh[j], dd[j], pp[j], ps[j], tp[j]);
                if (r) api_fail(r, cx[j], "shot: ");
            }
        } else {
            int r = ertm_rtm_multi(cx, m, sh, dd, pp, ps, tp);
            if (r) api_fail(r, cx[0], "shots: ");
        }
        for (int j = 0; j < m && rc == ERTM_OK; j++) {
            const ertm_window& w = win[order[g0 + j]];
            const int nx = w.wx + pxl + pxr, ny = two_d ? 1 : w.wy + pyl + pyr;
            k_stack_window<<<592, 256, 0, st>>>(pp[j], nx, ny, nz_w, pxl, two_d ? 0 : pyl, pzt, stack, NX, NY,
                                                NZ, w.x0, two_d ? 0 : w.y0, w.wx, two_d ? 1 : w.wy);
            if ((e = cudaGetLastError()) != cudaSuccess) cuda_fail(e, "stack");
        }
    }

    // the outputs
    if (rc == ERTM_OK) {
        float* outs[3] = {stack_pp, stack_ps, stack_tp};
        for (int q = 0; q < 3 && rc == ERTM_OK; q++) {
            if (!outs[q]) continue;
            e = cudaMemcpyAsync(outs[q], stack + q * nmod, sizeof(float) * nmod, cudaMemcpyDefault, st);
            if (e != cudaSuccess) cuda_fail(e, "output copy");
        }
    }
    if (st && (e = cudaStreamSynchronize(st)) != cudaSuccess) cuda_fail(e, "windows");
    for (auto& sl : S) {
        if (sl.ctx) ertm_destroy(sl.ctx);
        cudaFree(sl.model);
        cudaFree(sl.img);
    }
    cudaFree(stack);
    cudaFree(dmodel);
    if (st) cudaStreamDestroy(st);
    if (rc != ERTM_OK) return bad(rc, err);
    put_err(errbuf, errlen, "");
    return ERTM_OK;
}
