// Batched RTM over aperture windows of one shared model (ertm_rtm_windows).
//
// Every shot migrates on its own window: the shared migration model cropped to
// the window laterally (full depth), extended by the absorbing layers with edge
// values, and its images are added into one stacked volume of the model's size.
// Shots run on `lanes` contexts at once, one host thread and one CUDA stream per
// lane, each context allocated for the largest window and shrunk to each shot's
// window with ertm_set_grid; a lane keeps its own stack and the stacks are summed
// in lane order at the end, so the result does not depend on how the shots were
// spread over the lanes beyond float summation order.  Built on the public C ABI
// plus two small kernels (crop, stack); the reference migrates one shot per run
// on the full grid (3D_elastic_RTM/3D_output_file.cu:339-365).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
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

__global__ void k_add(const float* __restrict__ a, float* __restrict__ b, long long n)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x)
        b[q] += a[q];
}

void put_err(char* buf, size_t len, const std::string& m)
{
    if (!buf || !len) return;
    size_t n = std::min(len - 1, m.size());
    std::memcpy(buf, m.data(), n);
    buf[n] = 0;
}

struct Lane {
    ertm_ctx* ctx = nullptr;
    cudaStream_t st = nullptr;
    float* model = nullptr;   // 3 x cap cells (window grid)
    float* img = nullptr;     // 3 x cap cells (window grid)
    float* stack = nullptr;   // 3 x model cells
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
    lanes = std::max(1, std::min(lanes, std::max(nshots, 1)));
    if (cudaSetDevice(B.device) != cudaSuccess) {
        cudaGetLastError();
        return bad(ERTM_ECUDA, "cudaSetDevice");
    }

    // shared model on the device
    const float* mdl[3] = {vp, vs, rho};
    float* dmodel = nullptr;
    std::vector<Lane> L(lanes);
    int rc = ERTM_OK;
    std::string err;
    auto cuda_fail = [&](cudaError_t e, const char* what) {
        if (rc == ERTM_OK) {
            rc = e == cudaErrorMemoryAllocation ? ERTM_ENOMEM : ERTM_ECUDA;
            err = std::string(what) + ": " + cudaGetErrorString(e);
        }
    };
    cudaError_t e = cudaMalloc(&dmodel, sizeof(float) * 3 * nmod);
    if (e != cudaSuccess) cuda_fail(e, "model");
    for (int q = 0; q < 3 && rc == ERTM_OK; q++)
        if ((e = cudaMemcpy(dmodel + q * nmod, mdl[q], sizeof(float) * nmod, cudaMemcpyDefault)) != cudaSuccess)
            cuda_fail(e, "model copy");
    for (int l = 0; l < lanes && rc == ERTM_OK; l++) {
        ertm_config c = B;
        c.nx = cap_nx;
        c.ny = cap_ny;
        c.nz = nz_w;
        c.nt = cap_nt;
        c.src_steps = 0;
        if (two_d) c.pml[2] = c.pml[3] = 0;
        int r = ertm_create(&c, &L[l].ctx);
        if (r) {
            char b[512];
            ertm_last_error(nullptr, b, sizeof b);
            rc = r;
            err = std::string("lane context: ") + b;
            break;
        }
        if ((e = cudaStreamCreateWithFlags(&L[l].st, cudaStreamNonBlocking)) != cudaSuccess) { cuda_fail(e, "stream"); break; }
        ertm_set_stream(L[l].ctx, L[l].st);
        if ((e = cudaMalloc(&L[l].model, sizeof(float) * 3 * ncap)) != cudaSuccess) { cuda_fail(e, "lane model"); break; }
        if ((e = cudaMalloc(&L[l].img, sizeof(float) * 3 * ncap)) != cudaSuccess) { cuda_fail(e, "lane image"); break; }
        if ((e = cudaMalloc(&L[l].stack, sizeof(float) * 3 * nmod)) != cudaSuccess) { cuda_fail(e, "lane stack"); break; }
        if ((e = cudaMemsetAsync(L[l].stack, 0, sizeof(float) * 3 * nmod, L[l].st)) != cudaSuccess) { cuda_fail(e, "memset"); break; }
    }

    // largest windows first, handed out dynamically
    std::vector<int> order(nshots);
    for (int i = 0; i < nshots; i++) order[i] = i;
    auto cost = [&](int i) {
        const ertm_window& w = win[i];
        const int ss = w.src_steps ? w.src_steps : 2 * w.nt / 3;
        return (double)(w.wx + pxl + pxr) * (two_d ? 1 : w.wy + pyl + pyr) * (ss + w.nt);
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::atomic<int> next{0};
    std::atomic<bool> stop{rc != ERTM_OK};
    std::mutex mu;

    auto worker = [&](int l) {
        cudaSetDevice(B.device);
        Lane& ln = L[l];
        auto lane_fail = [&](int code, const std::string& m) {
            std::lock_guard<std::mutex> lk(mu);
            if (rc == ERTM_OK) {
                rc = code;
                err = m;
            }
            stop = true;
        };
        while (!stop) {
            const int q = next.fetch_add(1);
            if (q >= nshots) break;
            const int i = order[q];
            const ertm_window& w = win[i];
            const int nx = w.wx + pxl + pxr, ny = two_d ? 1 : w.wy + pyl + pyr;
            const long long n = (long long)nx * ny * nz_w;
            int r = ertm_set_grid(ln.ctx, nx, ny, w.nt, w.src_steps);
            if (!r) {
                k_crop_pad<<<592, 256, 0, ln.st>>>(dmodel, dmodel + nmod, dmodel + 2 * nmod, NX, NY, NZ,
                                                    w.x0 - pxl, two_d ? 0 : w.y0 - pyl, -pzt, ln.model, nx,
                                                    ny, nz_w);
                cudaError_t ke = cudaGetLastError();
                if (ke != cudaSuccess) {
                    lane_fail(ERTM_ECUDA, std::string("crop: ") + cudaGetErrorString(ke));
                    break;
                }
                r = ertm_set_model(ln.ctx, 1, ln.model, ln.model + n, ln.model + 2 * n);
            }
            ertm_shot s = shots[i];
            s.sx = s.sx - w.x0 + pxl;
            s.sy = two_d ? 0 : s.sy - w.y0 + pyl;
            s.sz = s.sz + pzt;
            s.rx0 = s.rx0 - w.x0 + pxl;
            s.ry0 = two_d ? 0 : s.ry0 - w.y0 + pyl;
            s.rz = s.rz + pzt;
            if (!r) r = ertm_rtm_shot(ln.ctx, &s, data[i], ln.img, ln.img + n, ln.img + 2 * n);
            if (r) {
                char b[512];
                ertm_last_error(ln.ctx, b, sizeof b);
                char head[64];
                snprintf(head, sizeof head, "shot %d: ", i);
                lane_fail(r, std::string(head) + b);
                break;
            }
            k_stack_window<<<592, 256, 0, ln.st>>>(ln.img, nx, ny, nz_w, pxl, two_d ? 0 : pyl, pzt,
                                                    ln.stack, NX, NY, NZ, w.x0, two_d ? 0 : w.y0, w.wx,
                                                    two_d ? 1 : w.wy);
            cudaError_t ke = cudaGetLastError();
            if (ke != cudaSuccess) {
                lane_fail(ERTM_ECUDA, std::string("stack: ") + cudaGetErrorString(ke));
                break;
            }
        }
        cudaError_t se = cudaStreamSynchronize(ln.st);
        if (se != cudaSuccess) lane_fail(ERTM_ECUDA, std::string("lane: ") + cudaGetErrorString(se));
    };
    // Autotuning (base->autotune): tune every distinct window shape up front on
    // lane 0 alone, so no other lane's work disturbs the trial timings (a
    // zero-step pass runs the tuner, whose choice is cached per shape).
    if (rc == ERTM_OK && B.autotune == 1) {
        std::vector<std::pair<int, int>> shapes;
        for (int i = 0; i < nshots; i++)
            shapes.emplace_back(win[i].wx + pxl + pxr, two_d ? 1 : win[i].wy + pyl + pyr);
        std::sort(shapes.begin(), shapes.end());
        shapes.erase(std::unique(shapes.begin(), shapes.end()), shapes.end());
        for (auto& sh : shapes) {
            const long long n = (long long)sh.first * sh.second * nz_w;
            int r = ertm_set_grid(L[0].ctx, sh.first, sh.second, 1, 0);
            if (!r) {
                k_crop_pad<<<592, 256, 0, L[0].st>>>(dmodel, dmodel + nmod, dmodel + 2 * nmod, NX, NY, NZ, 0, 0,
                                                      0, L[0].model, sh.first, sh.second, nz_w);
                r = ertm_set_model(L[0].ctx, 1, L[0].model, L[0].model + n, L[0].model + 2 * n);
            }
            ertm_shot s{};
            s.nrx = s.nry = 0;
            s.drx = s.dry = 1;
            if (!r) r = ertm_propagate(L[0].ctx, 1, &s, 0);
            if (r) {
                char b[512];
                ertm_last_error(L[0].ctx, b, sizeof b);
                rc = r;
                err = std::string("autotune: ") + b;
                break;
            }
        }
    }
    if (rc == ERTM_OK) {
        std::vector<std::thread> th;
        for (int l = 0; l < lanes; l++) th.emplace_back(worker, l);
        for (auto& t : th) t.join();
    }

    // sum the lane stacks in lane order, then write the outputs
    if (rc == ERTM_OK) {
        for (int l = 1; l < lanes; l++) {
            cudaStreamSynchronize(L[l].st);
            k_add<<<592, 256, 0, L[0].st>>>(L[l].stack, L[0].stack, 3 * nmod);
        }
        float* outs[3] = {stack_pp, stack_ps, stack_tp};
        for (int q = 0; q < 3 && rc == ERTM_OK; q++) {
            if (!outs[q]) continue;
            e = cudaMemcpyAsync(outs[q], L[0].stack + q * nmod, sizeof(float) * nmod, cudaMemcpyDefault,
                                L[0].st);
            if (e != cudaSuccess) cuda_fail(e, "output copy");
        }
        if ((e = cudaStreamSynchronize(L[0].st)) != cudaSuccess) cuda_fail(e, "output");
    }
    for (auto& ln : L) {
        if (ln.ctx) ertm_destroy(ln.ctx);
        if (ln.st) cudaStreamDestroy(ln.st);
        cudaFree(ln.model);
        cudaFree(ln.img);
        cudaFree(ln.stack);
    }
    cudaFree(dmodel);
    if (rc != ERTM_OK) return bad(rc, err);
    put_err(errbuf, errlen, "");
    return ERTM_OK;
}
