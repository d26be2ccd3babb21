// Image and gradient post-filters.
//
// Host (the reference runs them on the CPU): the Laplacian filter of cpu_laplace
// (3D_elastic_RTM/zzzzz:1110-1147; the 2D copy `laplace` at 2D_elastic_RTM/zzzzz:1153)
// and the Hilbert transform along depth of suhilbt (3D_elastic_RTM/zzzzz:1018-1066;
// 2D copy at 2D_elastic_RTM/zzzzz:1061).  The reference applies both to the interior
// of a padded image; here the caller passes that interior.
//
// Host or device, chosen by where the array lives (the reference runs them as GPU
// kernels on its gradients, 2D_elastic_RTM/viscoelastic_equation.cu:2528-2988):
// the truncated Gaussian "bell" smoothing of cuda_bell_smooth{x,z}_new /
// cuda_bell_smooth_2d, and the cosine-power edge taper of
// cuda_attenuation_truncation; the angle-dependent compensation of PP/PS images and
// the angle-domain common-image gathers of 2D_elastic_RTM/elastic_2D_kernel_3.cu.
//
// Arrays are (nz, ny, nx), x fastest; ny = 1 is a 2D section.
#include <cuda_runtime.h>

#include <cmath>
#include <thread>
#include <vector>

#include "ertm.h"

namespace {

bool on_device(const void* p)
{
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

constexpr int kMaxBell = 64;

// Bell weights exp(-i^2 / (2 r)) for i = -r..r, computed once on the host in double
// and rounded to float, so the host and device passes use the same numbers.
struct BellW {
    float w[2 * kMaxBell + 1];
};

BellW bell_weights(int r)
{
    BellW b{};
    for (int i = -r; i <= r; i++) b.w[i + r] = (float)std::exp(-(double)i * i / 2.0 / r);
    return b;
}

// One smoothing pass along an axis of stride `st` and length `len`: the weights that
// fall inside the array are renormalised to sum 1 (the reference's truncation at the
// edges).  A cell's coordinate along the axis is (c / st) % len.
__host__ __device__ inline float bell_at(const float* g, long long c, long long st, int len, int r,
                                         const float* w)
{
    const int p = (int)((c / st) % len);
    float sum = 0.f, s = 0.f;
    for (int i = -r; i <= r; i++)
        if (p + i >= 0 && p + i < len) sum += w[i + r];
    for (int i = -r; i <= r; i++)
        if (p + i >= 0 && p + i < len) s += w[i + r] / sum * g[c + i * st];
    return s;
}

__global__ void k_bell(const float* __restrict__ g, float* __restrict__ out, long long n, long long st,
                       int len, int r, BellW bw)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
        out[c] = bell_at(g, c, st, len, r, bw.w);
}

// Taper factor of column ix: cos(pi/2 m / w)^power on the `left`+1 first columns
// (m = left - ix) and the `right` last ones (m = ix - nx + right).
__host__ __device__ inline float taper_at(int ix, int nx, int left, int right, int power)
{
    double f = 1.0;
    const double hp = 1.57079632679489661923;
    if (left > 0 && ix <= left) f *= pow(cos(hp * (left - ix) / left), power);
    if (right > 0 && ix >= nx - right) f *= pow(cos(hp * (ix - nx + right) / right), power);
    return (float)f;
}

// Aperture factor of column ix: 0 outside [x0, x1) (a side whose edge is negative is
// open), cos(pi/2 m / w)^power on the w columns inside each closed edge (m counts
// from the inner end of the ramp), 1 elsewhere.
__host__ __device__ inline float aperture_at(int ix, int x0, int x1, int w, int power)
{
    const double hp = 1.57079632679489661923;
    double f = 1.0;
    if (x0 >= 0) {
        if (ix < x0) return 0.f;
        if (ix < x0 + w) f *= pow(cos(hp * (x0 + w - ix) / w), power);
    }
    if (x1 >= 0) {
        if (ix >= x1) return 0.f;
        if (ix >= x1 - w) f *= pow(cos(hp * (ix - (x1 - w)) / w), power);
    }
    return (float)f;
}

__global__ void k_aperture(float* img, long long n, int nx, int x0, int x1, int w, int power)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
        img[c] *= aperture_at((int)(c % nx), x0, x1, w, power);
}

__global__ void k_taper(float* img, long long n, int nx, int left, int right, int power)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
        img[c] *= taper_at((int)(c % nx), nx, left, right, power);
}

// Angle-dependent amplitude compensation of one cell (open angle d = src - rcv, degrees),
// rounded as the reference's kernels round it: the angle in radians is formed in double
// with the float constant pai1 = 3.1415926f, the cosine or sine is stored as a float,
// and the division is done in double (elastic_2D_kernel_3.cu:622-761).
__host__ __device__ inline float compensate(float img, float src, float rcv, int kind)
{
    const double pai1 = (double)3.1415926f;
    const float d = src - rcv;
    switch (kind) {
    case ERTM_COMP_PP: {
        const float den = (fabsf(d) >= 87.5f && fabsf(d) <= 92.5f) ? 0.1f
                                                                   : (float)cos((double)d * pai1 / 180.0);
        return (float)((double)img / ((double)den + 0.0001));
    }
    case ERTM_COMP_PS: {
        const float den = fabsf(d) <= 2.5f ? 0.1f : (float)sin(fabs((double)d * pai1 / 180.0));
        return (float)((double)img / ((double)den + 0.0001));
    }
    case ERTM_COMP_PP_SIGN: {
        const float sgn = (float)cos((double)d * pai1 / 180.0);
        const float v = sgn <= 0.f ? -img : img;
        return (float)(-(double)v / ((double)fabsf(sgn) + 0.03));
    }
    default: {   // ERTM_COMP_PS_SIGN
        const float sgn = (float)fabs(sin((double)d * pai1 / 180.0));
        const float den = (float)((double)fabsf(sgn) + 0.1);
        return (float)(-(double)img / (double)den);
    }
    }
}

__global__ void k_compensate(const float* img, const float* src, const float* rcv, float* out, long long n,
                             int kind)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
        out[c] = compensate(img[c], src[c], rcv[c], kind);
}

// Angle bin of cell (ix, iz), or -1 when the cell is masked out or its angle is past
// the last bin.
__host__ __device__ inline int adcig_bin(float ang, int ix, int iz, int nang, float dangle, int sx, int zmin,
                                         float slope)
{
    if (!(iz > zmin && iz > slope * (ix - sx) && iz > slope * (sx - ix))) return -1;
    const int r = (int)((fabsf(ang) + 0.5f) / dangle);
    if (r >= nang) return -1;
    return ang >= 0.f ? nang + r : nang - r;
}

__global__ void k_adcig(const float* img, const float* ang, const float* normal, float* cig, int nx, int nz,
                        int nang, float dangle, int sx, int zmin, float slope)
{
    const long long n = (long long)nx * nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const float a = ang[c] - (normal ? normal[c] : 0.f);
        const int b = adcig_bin(a, (int)(c % nx), (int)(c / nx), nang, dangle, sx, zmin, slope);
        if (b >= 0) cig[b * n + c] += img[c];   // one cell per thread: no two threads share an address
    }
}

// Hilbert transform of columns [c0, c1) (one host thread's share of ertm_hilbert_z)
void hilbert_columns(const float* img, float* out, int nz, long long sz, long long c0, long long c1,
                     const double* cs, const double* sn)
{
    std::vector<double> col((size_t)nz), re((size_t)nz), im((size_t)nz);
    for (long long c = c0; c < c1; c++) {
        for (int t = 0; t < nz; t++) col[t] = img[t * sz + c];
        for (int w = 0; w < nz; w++) {
            double r = 0.0, i = 0.0;
            for (int t = 0; t < nz; t++) {
                const int q = (int)(((long long)w * t) % nz);
                r += col[t] * cs[q];
                i -= col[t] * sn[q];
            }
            if (w < nz / 2) { re[w] = i; im[w] = -r; }      // * (-i)
            else { re[w] = -i; im[w] = r; }                  // * (+i)
        }
        for (int t = 0; t < nz; t++) {
            double v = 0.0;
            for (int w = 0; w < nz; w++) {
                const int q = (int)(((long long)w * t) % nz);
                v += re[w] * cs[q] - im[w] * sn[q];
            }
            out[t * sz + c] = (float)(v / nz);
        }
    }
}

int grid_for(long long n)
{
    const long long b = (n + 255) / 256;
    return (int)(b < 148 * 16 ? b : 148 * 16);
}

}  // namespace

extern "C" {

// Laplacian image filter (cpu_laplace, zzzzz:1110-1147, extended to 3D with the y
// term): t = -(d2/dx2 + d2/dy2 + d2/dz2) r with second-order differences inside,
// t = -r on the outermost cells, then the outermost cells copy their inner
// neighbour (x edges, then y, then z, so a corner takes its diagonal inner
// neighbour), and r = vp^2 t / 4.  Arrays (nz, ny, nx), x fastest.  The reference's
// copy loop for the top and bottom rows indexes columns with the depth counter, so
// it reaches min(nx, nz) columns and its corners take a raw -r value; here every
// column is covered, and the interior matches the reference exactly.
int ertm_laplace_filter(float* img, const float* vp, int nx, int ny, int nz, float dx, float dy, float dz)
{
    if (!img || !vp || nx < 3 || nz < 3 || ny < 1 || (ny > 1 && ny < 3) || !(dx > 0) || !(dy > 0) ||
        !(dz > 0))
        return ERTM_EINVAL;
    const long long sy = nx, sz = (long long)nx * ny, n = sz * nz;
    std::vector<float> t(n);
    const double ix2 = 1.0 / ((double)dx * dx), iy2 = 1.0 / ((double)dy * dy), iz2 = 1.0 / ((double)dz * dz);
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                const long long c = k * sz + j * sy + i;
                const bool edge = i == 0 || i == nx - 1 || k == 0 || k == nz - 1 || (ny > 1 && (j == 0 || j == ny - 1));
                if (edge) {
                    t[c] = -img[c];
                    continue;
                }
                double lap = (img[c + 1] + img[c - 1] - 2.0 * img[c]) * ix2 +
                             (img[c + sz] + img[c - sz] - 2.0 * img[c]) * iz2;
                if (ny > 1) lap += (img[c + sy] + img[c - sy] - 2.0 * img[c]) * iy2;
                t[c] = (float)(-lap);
            }
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++) {
            const long long r = k * sz + j * sy;
            t[r] = t[r + 1];
            t[r + nx - 1] = t[r + nx - 2];
        }
    if (ny > 1)
        for (int k = 0; k < nz; k++)
            for (int i = 0; i < nx; i++) {
                t[k * sz + i] = t[k * sz + sy + i];
                t[k * sz + (ny - 1) * sy + i] = t[k * sz + (ny - 2) * sy + i];
            }
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            t[j * sy + i] = t[sz + j * sy + i];
            t[(nz - 1) * sz + j * sy + i] = t[(nz - 2) * sz + j * sy + i];
        }
    for (long long c = 0; c < n; c++) img[c] = vp[c] * vp[c] * t[c] / 4.0f;
    return ERTM_OK;
}

// Hilbert transform along depth of every (y, x) column (suhilbt, zzzzz:1018-1066):
// X = DFT(x) (forward e^{-i w t}), multiplied by -i for w < n/2 and by +i from n/2 on,
// y = Re(IDFT(X)) / n — the reference's direct O(n^2) transforms, in double.  The
// columns are split over the host's hardware threads.
int ertm_hilbert_z(const float* img, float* out, int nx, int ny, int nz)
{
    if (!img || !out || nx < 1 || ny < 1 || nz < 1) return ERTM_EINVAL;
    const double pi = 3.14159265358979323846;
    std::vector<double> cs((size_t)nz), sn((size_t)nz);
    for (int q = 0; q < nz; q++) {
        cs[q] = std::cos(2.0 * pi * q / nz);
        sn[q] = std::sin(2.0 * pi * q / nz);
    }
    const long long sz = (long long)nx * ny;
    const long long work = sz * (long long)nz * nz;
    unsigned nth = std::thread::hardware_concurrency();
    if (nth == 0) nth = 1;
    if (work < (1LL << 22)) nth = 1;
    if ((long long)nth > sz) nth = (unsigned)sz;
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nth; t++)
        pool.emplace_back(hilbert_columns, img, out, nz, sz, sz * t / nth, sz * (t + 1) / nth, cs.data(),
                          sn.data());
    for (auto& th : pool) th.join();
    return ERTM_OK;
}



// Truncated Gaussian smoothing (cuda_bell_smoothz_new / cuda_bell_smoothx_new,
// viscoelastic_equation.cu:2528-2566): one pass per axis named in `axes`
// (ERTM_AXIS_X | ERTM_AXIS_Y | ERTM_AXIS_Z), in the order z, y, x.  The reference's
// 2D form (cuda_bell_smooth_2d, :2568-2604) truncates its window to a rectangle, so
// its weights factor: it equals the z pass followed by the x pass.  Passes go
// through `work` (n floats, same memory space) when more than one axis is named;
// `in` may be `out` only when exactly two are (no pass then reads what it writes).  Host arrays run on the host, device arrays on
// `stream` (the call returns after the stream has finished the passes).
int ertm_bell_smooth(const float* in, float* out, float* work, int nx, int ny, int nz, int rbell, int axes,
                     void* stream)
{
    if (!in || !out || nx < 1 || ny < 1 || nz < 1 || rbell < 1 || rbell > kMaxBell || (axes & ~7) || !axes)
        return ERTM_EINVAL;
    const long long n = (long long)nx * ny * nz;
    struct Pass {
        long long st;
        int len;
    };
    Pass ps[3];
    int np = 0;
    if (axes & ERTM_AXIS_Z) ps[np++] = {(long long)nx * ny, nz};
    if (axes & ERTM_AXIS_Y) ps[np++] = {(long long)nx, ny};
    if (axes & ERTM_AXIS_X) ps[np++] = {1, nx};
    const bool dev = on_device(in);
    if (dev != on_device(out) || (np > 1 && (!work || dev != on_device(work)))) return ERTM_EINVAL;
    const BellW bw = bell_weights(rbell);
    // pass q reads src[q] and writes dst[q]; buffers alternate so that the last pass
    // lands in `out` and no pass reads the array it writes.
    const float* src = in;
    for (int q = 0; q < np; q++) {
        float* dst = ((np - 1 - q) % 2 == 0) ? out : work;
        if (dst == src) return ERTM_EINVAL;  // in == out with an odd pass count
        if (dev) {
            k_bell<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(src, dst, n, ps[q].st, ps[q].len, rbell, bw);
            if (cudaGetLastError() != cudaSuccess) return ERTM_ECUDA;
        } else {
            for (long long c = 0; c < n; c++) dst[c] = bell_at(src, c, ps[q].st, ps[q].len, rbell, bw.w);
        }
        src = dst;
    }
    if (dev) return cudaStreamSynchronize((cudaStream_t)stream) == cudaSuccess ? ERTM_OK : ERTM_ECUDA;
    return ERTM_OK;
}

// Edge taper in x (cuda_attenuation_truncation, viscoelastic_equation.cu:2881-2926,
// with its widths offset/3 and power 3 as arguments): column ix is multiplied by
// cos(pi/2 (left - ix) / left)^power for ix <= left and by
// cos(pi/2 (ix - nx + right) / right)^power for ix >= nx - right; a width of 0 leaves
// that side alone.
int ertm_taper_x(float* img, int nx, int ny, int nz, int left, int right, int power, void* stream)
{
    if (!img || nx < 1 || ny < 1 || nz < 1 || left < 0 || right < 0 || left >= nx || right > nx || power < 0)
        return ERTM_EINVAL;
    const long long n = (long long)nx * ny * nz;
    if (on_device(img)) {
        k_taper<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(img, n, nx, left, right, power);
        if (cudaGetLastError() != cudaSuccess) return ERTM_ECUDA;
        return cudaStreamSynchronize((cudaStream_t)stream) == cudaSuccess ? ERTM_OK : ERTM_ECUDA;
    }
    std::vector<float> f(nx);
    for (int i = 0; i < nx; i++) f[i] = taper_at(i, nx, left, right, power);
    for (long long c = 0; c < n; c++) img[c] *= f[c % nx];
    return ERTM_OK;
}

// Aperture mute of a gradient or image in x (cauda_zero_and_attenuation_truncation,
// viscoelastic_equation.cu:2928-2988, and its _old form, :2990-3045): columns
// outside [x0, x1) are zeroed and the w columns inside each edge ramp up with
// cos^power.  The reference's call: x0 = offset_left - receiver_offset when
// offset_left > receiver_offset (else open, -1), x1 = offset_left + receiver_offset
// when offset_right > receiver_offset, w = max(3, receiver_offset / offset_attenuation)
// and power 2 (the _old form: w = receiver_offset / 3, power 3).
int ertm_aperture_taper(float* img, int nx, int ny, int nz, int x0, int x1, int w, int power, void* stream)
{
    if (!img || nx < 1 || ny < 1 || nz < 1 || w < 1 || power < 0 || x0 < -1 || x1 < -1 ||
        (x0 >= 0 && x1 >= 0 && x1 < x0))
        return ERTM_EINVAL;
    const long long n = (long long)nx * ny * nz;
    if (on_device(img)) {
        k_aperture<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(img, n, nx, x0, x1, w, power);
        if (cudaGetLastError() != cudaSuccess) return ERTM_ECUDA;
        return cudaStreamSynchronize((cudaStream_t)stream) == cudaSuccess ? ERTM_OK : ERTM_ECUDA;
    }
    std::vector<float> f(nx);
    for (int i = 0; i < nx; i++) f[i] = aperture_at(i, x0, x1, w, power);
    for (long long c = 0; c < n; c++) img[c] *= f[c % nx];
    return ERTM_OK;
}

// Angle-dependent compensation of a PP or PS image (2D_elastic_RTM/elastic_2D_kernel_3.cu):
// with d = src_angle - rcv_angle in degrees,
//   ERTM_COMP_PP       img / (cos d + 1e-4), cos d replaced by 0.1 for 87.5 <= |d| <= 92.5
//                      (imaging_pp_compensate_dependent_angle_2D, :622-648)
//   ERTM_COMP_PS       img / (sin |d| + 1e-4), sin |d| replaced by 0.1 for |d| <= 2.5
//                      (imaging_ps_compensate_dependent_angle_2D, :650-676)
//   ERTM_COMP_PP_SIGN  -sign(cos d) img / (|cos d| + 0.03), sign(0) = -1
//                      (cuda_ex_com_pp_ps_sign + imaging_pp_compensate_dependent_angle_2D_new,
//                      :698-741)
//   ERTM_COMP_PS_SIGN  -img / (|sin d| + 0.1)  (imaging_ps_compensate_dependent_angle_2D_new,
//                      :743-761)
// The reference applies them cell by cell at the cell's excitation time, when the
// cell's image and both angles are final; here they run on the finished arrays.
int ertm_angle_compensate(const float* img, const float* src_angle, const float* rcv_angle, float* out,
                          long long n, int kind, void* stream)
{
    if (!img || !src_angle || !rcv_angle || !out || n < 0 || kind < ERTM_COMP_PP || kind > ERTM_COMP_PS_SIGN)
        return ERTM_EINVAL;
    const bool dev = on_device(img);
    if (on_device(src_angle) != dev || on_device(rcv_angle) != dev || on_device(out) != dev) return ERTM_EINVAL;
    if (n == 0) return ERTM_OK;
    if (dev) {
        k_compensate<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(img, src_angle, rcv_angle, out, n, kind);
        if (cudaGetLastError() != cudaSuccess) return ERTM_ECUDA;
        return cudaStreamSynchronize((cudaStream_t)stream) == cudaSuccess ? ERTM_OK : ERTM_ECUDA;
    }
    for (long long c = 0; c < n; c++) out[c] = compensate(img[c], src_angle[c], rcv_angle[c], kind);
    return ERTM_OK;
}

// Angle-domain common-image gathers of one shot (set_adcigs_for_ex,
// 2D_elastic_RTM/elastic_2D_kernel_3.cu:489-511): the angle of a cell is
// angle - normal (normal may be NULL: 0); r = (int)((|angle| + 0.5) / dangle); cells
// with r < nang, iz > zmin and iz > slope |ix - sx| add their image value to bin
// nang + r (angle >= 0) or nang - r (angle < 0) of cig [2 nang + 1][nz][nx], so bin b
// holds angles near (b - nang) dangle.  The reference's mask uses zmin 50, slope 1.2.
// Accumulates into cig; host or device arrays.
int ertm_adcig_bin(const float* img, const float* angle, const float* normal, float* cig, int nx, int nz,
                   int nang, float dangle, int sx, int zmin, float slope, void* stream)
{
    if (!img || !angle || !cig || nx < 1 || nz < 1 || nang < 1 || !(dangle > 0)) return ERTM_EINVAL;
    const bool dev = on_device(img);
    if (on_device(angle) != dev || on_device(cig) != dev || (normal && on_device(normal) != dev))
        return ERTM_EINVAL;
    const long long n = (long long)nx * nz;
    if (dev) {
        k_adcig<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(img, angle, normal, cig, nx, nz, nang, dangle, sx,
                                                              zmin, slope);
        if (cudaGetLastError() != cudaSuccess) return ERTM_ECUDA;
        return cudaStreamSynchronize((cudaStream_t)stream) == cudaSuccess ? ERTM_OK : ERTM_ECUDA;
    }
    for (long long c = 0; c < n; c++) {
        const float a = angle[c] - (normal ? normal[c] : 0.f);
        const int b = adcig_bin(a, (int)(c % nx), (int)(c / nx), nang, dangle, sx, zmin, slope);
        if (b >= 0) cig[b * n + c] += img[c];
    }
    return ERTM_OK;
}

}  // extern "C"
