// Internal types of libertm: device geometry, kernel argument block, launchers.
//
// HBM layout.  Every wavefield, model, excitation and image volume is one
// allocation of `Geom::total` floats with zero halos: x is padded by XH floats
// on both sides and the row pitch rounded up to 32 floats (128 B), y by R rows
// (3D only), z by R planes.  Pointers passed to kernels point at cell (0,0,0),
// so the stencil reads k*sz + j*sy + i +/- n without bounds checks; halo cells
// are never written and stay zero, which is the reference's `radius` padding
// (nnx_radius, viscoelastic_equation.cu:100).  Rows past nx and ny up to the
// tile size are allocated too and stay zero.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "ertm.h"

namespace ertm {

constexpr int TX = 32;        // x tile = one warp
constexpr int TY3 = 8;        // y tile of the 3D kernels
constexpr int CTAS3 = 2;      // resident CTAs per SM of the 3D step kernels
constexpr int TY2 = 1;        // y tile of the 2D kernels (a 2D grid has one y row)
constexpr int XH = 8;         // allocated x halo, floats (>= R, 32-byte aligned)

enum Field {
    F_VX, F_VY, F_VZ, F_TXX, F_TYY, F_TZZ, F_TXY, F_TXZ, F_TYZ, F_TP, F_VXP, F_VYP, F_VZP, NFIELD
};

// C-PML memory-variable slots: one per spatial derivative that enters an update.
enum Psi {
    P_EXX, P_EYY, P_EZZ, P_DYVX, P_DXVY, P_DZVX, P_DXVZ, P_DZVY, P_DYVZ,
    P_DXTXX, P_DYTXY, P_DZTXZ, P_DXTXY, P_DYTYY, P_DZTYZ, P_DXTXZ, P_DYTYZ, P_DZTZZ, NPSI
};

enum Epilogue { EPI_NONE = 0, EPI_EXCITE = 1, EPI_IMAGE = 2 };

struct Geom {
    int nx, ny, nz, R;
    int hx, hy, hz;
    long long px, py, pz;   // allocated extents
    long long sy, sz;       // strides (floats)
    long long off0;         // offset of cell (0,0,0)
    long long total;        // floats per volume
    int two_d;
    int tyb;                // y tile of the kernels for this grid
};

// Everything a step kernel reads; passed by value (param space).
struct KArgs {
    float* f[NFIELD];                // origin pointers
    const float* M;                  // rho*vp^2
    const float* MU;                 // rho*vs^2
    const float* B;                  // 1/rho
    long long sy, sz;                // field strides
    long long msy, msz;              // model strides
    int nx, ny, nz;
    int kchunk;
    float cx[8], cy[8], cz[8];       // c_n / h
    float dt;
    // sponge boundary: per-axis damping profiles (1/s), summed per cell
    const float* att[3];
    // C-PML: per axis, [0] integer points, [1] half points
    const float* pa[3][2];
    const float* pb[3][2];
    float* psi[NPSI];
    int w[6];
    // source (it < nw only)
    int ssx, ssy, ssz, nw;
    const float* wavelet;
    // receivers on a regular grid at depth rz
    int rx0, nrx, drx, ry0, nry, dry, rz;
    int inject_mode;
    float* traces;                   // [3][nt][nrec], recorded or injected
    int nt;
    const int* it_ptr;               // current step index (device)
    // excitation state and images (same geometry as the fields)
    float* ex_amp2;
    int* ex_time;
    float* ex_v[3];
    float* ex_tp;
    float* img[3];
    int* err;                        // device error word (0 = ok)
    // test hook of the device-error path (zero = off, so a zeroed KArgs is safe):
    // with skip_plane1 = t + 1 the first CTA of the grid does not issue the
    // staged copy of its chunk's plane t, so its consumers' bounded wait
    // (wait_polls polls; 0 = kWaitPolls) runs out
    int skip_plane1;
    unsigned wait_polls;
    // 3D step-kernel variant: 0 = one cell per thread (default), 1 = cell pairs
    int pairs;
    // several shots per launch only: the shot is idle while *it_ptr >= it_hi
    int it_hi;
};

// Device error codes written to KArgs::err
enum DeviceError { DEV_OK = 0, DEV_WAIT_TIMEOUT = 1 };

// TMA tensor maps of one step kernel, passed as a __grid_constant__ parameter.
// Every map covers a whole padded volume [pz][py][px]; the box shape is fixed
// per map: C = TX x TYB (centre), X = (TX+2XB) x TYB, Y = TX x (TYB+2R),
// XY = (TX+2XB) x (TYB+2R), one plane deep.
struct StressMaps {
    CUtensorMap v[3];      // vx, vz, vy      (XY boxes; X in 2D)
    CUtensorMap vc[3];     // vx, vz, vy      (C boxes: z-queue fronts)
    CUtensorMap sig[6];    // txx tzz txz tyy txy tyz (C)
    CUtensorMap tp;        // (C)
    CUtensorMap M, MU;     // (C)
};

struct VelMaps {
    CUtensorMap txx, txz;  // X boxes
    CUtensorMap txy, tp;   // XY boxes (X in 2D)
    CUtensorMap tyy, tyz;  // Y boxes
    CUtensorMap c[8];      // C boxes: vx vz vy vxp vzp vyp b excitation(amp2 or time)
    CUtensorMap fr[4];     // C boxes of txz tzz tyz tp: z-queue fronts
};

// Argument blocks of the multi-shot step kernels: up to kMultiMax shots per
// launch, each with its own argument block and TMA maps, all passed by value in
// the kernel's parameter block (3.1 KB per shot of the 32 KB it can hold), so
// that the TMA unit reads every descriptor from parameter space.
constexpr int kMultiMax = ERTM_MULTI_MAX;
struct StressMulti {
    KArgs a[kMultiMax];
    StressMaps m[kMultiMax];
    int chunks;                      // z chunks per shot
};
struct VelMulti {
    KArgs a[kMultiMax];
    VelMaps m[kMultiMax];
    int chunks;
};
static_assert(sizeof(VelMulti) <= 32764 && sizeof(StressMulti) <= 32764, "kernel parameter limit");

// x halo of the staged tiles: >= R and a multiple of 4 floats (16-byte TMA x start)
constexpr int xb_of(int R) { return R <= 4 ? 4 : 8; }

// Dynamic shared-memory opt-in of kernel `K` (a function attribute of the
// device's context): made once per device, on the first launch with that
// device current.  `done` is the kernel's own bit set of devices (one static
// per kernel instantiation at the call site).
template <typename KPTR>
inline cudaError_t smem_opt_in(KPTR K, size_t smem, unsigned long long* done)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (bit && (__atomic_load_n(done, __ATOMIC_ACQUIRE) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && bit) __atomic_fetch_or(done, bit, __ATOMIC_RELEASE);
    return e;
}

// Host set-up shared by the context path and the no-allocation path (setup.cu).
Geom make_geom(int nx, int ny, int nz, int R);
// difference coefficients c_0..c_R (c_0 = 0) for ERTM_COEF_* `coef_kind`
void stencil_coefs(int coef_kind, const float* user, int R, float coef[8]);
// C-PML a/b coefficients of one axis of n cells at integer (stg 0) or half points
// (stg +1 or -1), for cells i0 .. i0+m-1 into a[0..m), b[0..m)
void cpml_profile(int n, int w0, int w1, int stg, double h, double vmax, double rcoef, double f0,
                  double dts, int i0, int m, float* a, float* b);
// sponge damping (1/s, ERTM_BOUNDARY_SPONGE_COS or _CUBIC ramps) of one axis of n
// cells, for cells i0 .. i0+m-1 into v[0..m)
void sponge_profile(int n, int w0, int w1, int kind, float coe, int i0, int m, float* v);
// z planes per CTA of the step kernels for grid g on `device`
int choose_kchunk(const Geom& g, int R, int device);

// Launchers (one translation unit per stencil radius).
cudaError_t launch_stress(int R, const Geom& g, const KArgs& a, const StressMaps& m, bool cpml,
                          bool psplit, cudaStream_t s);
cudaError_t launch_velocity(int R, const Geom& g, const KArgs& a, const VelMaps& m, bool cpml,
                            int epi, bool record, cudaStream_t s);
cudaError_t launch_stress_r4(const Geom& g, const KArgs& a, const StressMaps& m, bool cpml,
                             bool psplit, cudaStream_t s);
cudaError_t launch_stress_r6(const Geom& g, const KArgs& a, const StressMaps& m, bool cpml,
                             bool psplit, cudaStream_t s);
cudaError_t launch_velocity_r4(const Geom& g, const KArgs& a, const VelMaps& m, bool cpml, int epi,
                               bool record, cudaStream_t s);
cudaError_t launch_velocity_r6(const Geom& g, const KArgs& a, const VelMaps& m, bool cpml, int epi,
                               bool record, cudaStream_t s);
cudaError_t launch_stress_multi_r4(dim3 grid, const StressMulti& P, bool cpml, cudaStream_t s);
cudaError_t launch_stress_multi_r6(dim3 grid, const StressMulti& P, bool cpml, cudaStream_t s);
cudaError_t launch_velocity_multi_r4(dim3 grid, const VelMulti& P, bool cpml, int epi, cudaStream_t s);
cudaError_t launch_velocity_multi_r6(dim3 grid, const VelMulti& P, bool cpml, int epi, cudaStream_t s);
// several 3D shots per launch (RTM passes): grid (x tiles, y tiles, shots x chunks)
cudaError_t launch_stress_multi(int R, dim3 grid, const StressMulti& P, bool cpml, cudaStream_t s);
cudaError_t launch_velocity_multi(int R, dim3 grid, const VelMulti& P, bool cpml, int epi, cudaStream_t s);

// Small kernels (aux.cu)
cudaError_t launch_scatter(const Geom& g, const float* src, float* dst, cudaStream_t s);
cudaError_t launch_gather(const Geom& g, const float* src, float* dst, cudaStream_t s);
cudaError_t launch_gather_int(const Geom& g, const int* src, int* dst, cudaStream_t s);
cudaError_t launch_model(const Geom& g, const float* vp, const float* vs, const float* rho,
                         float* M, float* MU, float* B, cudaStream_t s);
cudaError_t launch_inject(const KArgs& a, int it, cudaStream_t s);
cudaError_t launch_advance(int* it_ptr, int delta, cudaStream_t s);
cudaError_t launch_set_int(int* p, int v, cudaStream_t s);
cudaError_t launch_sqrt_gather(const Geom& g, const float* amp2, float* out, cudaStream_t s);
cudaError_t launch_axpy(long long n, const float* x, float* y, cudaStream_t s);   // y += x
// 2D propagation angle at the cells whose excitation step it is; window (2 hw + 1)^2:
// hw = 2 in the source pass, 4 in the receiver pass
cudaError_t launch_angle(const Geom& g, const KArgs& a, float* ang, int hw, cudaStream_t s);
cudaError_t launch_divcurl(int R, const Geom& g, const KArgs& a, const float* vp, const float* vs,
                           float* p, float* sx, float* sy, float* sz, cudaStream_t s);

}  // namespace ertm
