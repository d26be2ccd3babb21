// On-disk formats of the reference and the direct-wave mute of recorded data.
//
// Volumes: raw float32, native (little-endian) byte order, written x-outer,
// z-inner: for ix, for iy, for iz (output_file_xyz / output_file_xyz_boundary,
// input_file_xyz / input_file_xyz_boundary, 3D_elastic_RTM/3D_zzzzz:1-139).  The
// library's arrays are (nz, ny, nx) with x fastest, so reading and writing
// transpose.  The "boundary" variants read into / write from the interior of
// a padded array (offsets bl in x, bf in y, bu in z), which is how the
// reference stores models with absorbing layers and cuts them off its images
// (result-pp-*, 3D_output_file.cu:309-428).
//
// Shot gathers: one raw float32 file per component ([nrec][nt], receiver-major
// with time fastest, receivers y-major); the library's trace layout is
// [3][nt][nrec].
//
// Direct-wave mute (cut_direct_shot_3D_surface_three_new, called per step at
// 3D_forward_or_back_together.cu:135; its body is not in the reference tree):
// restated from its arguments (receiver and source cells, velocity, spacings,
// dt, wavelet length, cut length) as zeroing every sample earlier than the
// straight-ray direct arrival t_d = |receiver - source| / v plus the wavelet
// length and `extra` samples.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "ertm.h"

namespace {

bool is_dev(const void* p)
{
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// samples of receiver r to zero
__host__ __device__ inline int mute_len(const ertm_shot& s, int r, float dx, float dy, float dz,
                                        float dt_s, float v, int extra)
{
    const int ix = r % s.nrx, iy = r / s.nrx;
    const float rx = (float)(s.rx0 + ix * s.drx), ry = (float)(s.ry0 + iy * s.dry), rz = (float)s.rz;
    const float ddx = (rx - s.sx) * dx, ddy = (ry - s.sy) * dy, ddz = (rz - s.sz) * dz;
    const float td = sqrtf(ddx * ddx + ddy * ddy + ddz * ddz) / v;
    return (int)ceilf(td / dt_s) + s.nw + extra;
}

__global__ void k_mute(float* d, ertm_shot s, int nt, float dx, float dy, float dz, float dt_s, float v,
                       int extra)
{
    const long long nrec = (long long)s.nrx * s.nry;
    const long long n = 3 * (long long)nt * nrec;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(q % nrec), it = (int)((q / nrec) % nt);
        if (it < mute_len(s, r, dx, dy, dz, dt_s, v, extra)) d[q] = 0.f;
    }
}

}  // namespace

extern "C" {

int ertm_write_volume_xyz(const char* path, const float* vol, int nxb, int nyb, int nzb, int nx, int ny, int nz,
                          int bl, int bf, int bu)
{
    if (!path || !vol || nx < 1 || ny < 1 || nz < 1 || bl < 0 || bf < 0 || bu < 0 || bl + nx > nxb ||
        bf + ny > nyb || bu + nz > nzb)
        return ERTM_EINVAL;
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return ERTM_EINVAL;
    std::vector<float> col(nz);
    int rc = ERTM_OK;
    for (int ix = 0; ix < nx && rc == ERTM_OK; ix++)
        for (int iy = 0; iy < ny && rc == ERTM_OK; iy++) {
            for (int iz = 0; iz < nz; iz++)
                col[iz] = vol[((long long)(iz + bu) * nyb + (iy + bf)) * nxb + ix + bl];
            if (std::fwrite(col.data(), sizeof(float), nz, fp) != (size_t)nz) rc = ERTM_EINVAL;
        }
    if (std::fclose(fp) != 0) rc = ERTM_EINVAL;
    return rc;
}

int ertm_read_volume_xyz(const char* path, float* vol, int nxb, int nyb, int nzb, int nx, int ny, int nz, int bl,
                         int bf, int bu)
{
    if (!path || !vol || nx < 1 || ny < 1 || nz < 1 || bl < 0 || bf < 0 || bu < 0 || bl + nx > nxb ||
        bf + ny > nyb || bu + nz > nzb)
        return ERTM_EINVAL;
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return ERTM_EINVAL;
    std::vector<float> col(nz);
    int rc = ERTM_OK;
    for (int ix = 0; ix < nx && rc == ERTM_OK; ix++)
        for (int iy = 0; iy < ny && rc == ERTM_OK; iy++) {
            if (std::fread(col.data(), sizeof(float), nz, fp) != (size_t)nz) {
                rc = ERTM_EINVAL;
                break;
            }
            for (int iz = 0; iz < nz; iz++)
                vol[((long long)(iz + bu) * nyb + (iy + bf)) * nxb + ix + bl] = col[iz];
        }
    std::fclose(fp);
    return rc;
}

int ertm_mute_direct(const ertm_shot* s, float* data, int nt, float dx, float dy, float dz, float dt_ms,
                     float v, int extra, void* stream)
{
    if (!s || !data || nt < 1 || !(v > 0) || !(dt_ms > 0) || s->nrx < 0 || s->nry < 0 || s->drx < 1 ||
        s->dry < 1 || extra < 0)
        return ERTM_EINVAL;
    const long long nrec = (long long)s->nrx * s->nry;
    const float dts = dt_ms / 1000.f;
    if (is_dev(data)) {
        const long long n = 3 * (long long)nt * nrec;
        const int blocks = (int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16);
        if (n == 0) return ERTM_OK;
        k_mute<<<blocks, 256, 0, (cudaStream_t)stream>>>(data, *s, nt, dx, dy, dz, dts, v, extra);
        if (cudaGetLastError() != cudaSuccess) return ERTM_ECUDA;
        return cudaStreamSynchronize((cudaStream_t)stream) == cudaSuccess ? ERTM_OK : ERTM_ECUDA;
    }
    for (long long r = 0; r < nrec; r++) {
        const int m = mute_len(*s, (int)r, dx, dy, dz, dts, v, extra);
        for (int c = 0; c < 3; c++)
            for (int it = 0; it < nt && it < m; it++) data[((long long)c * nt + it) * nrec + r] = 0.f;
    }
    return ERTM_OK;
}

}  // extern "C"
