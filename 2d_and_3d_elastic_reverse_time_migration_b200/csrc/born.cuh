// Born modelling / adjoint kernels (2D, sponge boundaries, elastic or GSLS
// viscoelastic): argument block and launchers.
#pragma once

#include <cuda_runtime.h>

namespace ertm {

constexpr int BXH = 8;   // x halo of the compact 2D layout (floats)

struct BornArgs {
    int nx, nz, R;
    long long px;                          // row pitch; cell (i,k) at (k+R)*px + i + BXH
    float cx[8], cz[8];                    // c_n / h
    float dt;
    const float *M, *U, *Bg1, *B, *g1, *g2;// model products (Bg1 = B g1) and damping factors
    float *v0x, *v0z, *s0xx, *s0zz, *s0xz; // background state
    float *vx, *vz, *sxx, *szz, *sxz;      // scattered state
    const float *dM, *dU, *rr;             // perturbation products
    float *ax, *az, *hxx, *hzz, *hxz;      // adjoint state
    float *gM, *gL, *gU, *gR;              // gradient accumulators (pi, unused, mu, rho)
    // GSLS attenuation (nm = 0: elastic): memory variables r[q*3 + l] of stress
    // component q (xx, zz, xz) and mechanism l; r' = ra_l r + rb_l f
    int nm;
    float ra[3], rb[3];
    float tp, ts, kp, ks;                  // strengths; kp = 1 + nm tp, ks = 1 + nm ts
    float *r0[9], *r[9], *lr[9];           // background, scattered, adjoint memory variables
    float *Sxx, *Szz, *Sxz;                // strain adjoint of the reverse step (scratch)
    const float *hv0x, *hv0z, *ha0x, *ha0z;// background history read by the adjoint step
    float *kv0x, *kv0z, *ka0x, *ka0z;      // history slot written by a recording step
    int nw;
    const float* wavelet;                  // shot s's wavelet at wavelet + s * wstride
    int wstride;
    int nrx;                               // receivers per shot
    float* traces;                         // per shot [3][nt][nrx]: recorded (forward) or residual (adjoint)
    int nt;
    // Shots of one launch (blockIdx.z = shot): every per-shot volume above (states,
    // memory variables, adjoint, strain scratch, gradient accumulators, history) is
    // [shot][n] with the shot stride `ss` floats; shot s's source cell, receiver line
    // and traces come from shot_tab[s * 8 + 0..5] = (sx, sz, rx0, nrx, drx, rz) and
    // traces + s * tstride.  The model and perturbation products are shared.
    int nshot;
    long long ss;
    const int* shot_tab;
    long long tstride;
    int kc;                                // rows per warp of the step kernels (set by the launcher)
};

cudaError_t born_launch_model(const BornArgs& a, const float* Mc, const float* Uc, const float* Bc,
                              long long csz, const float* att_x, const float* att_z, float* M,
                              float* U, float* Bg1, float* B, float* g1, float* g2, cudaStream_t s);
cudaError_t born_launch_pert(const BornArgs& a, const float* rvp, const float* rvs,
                             const float* rrho, float* dM, float* dU, float* rr, cudaStream_t s);
cudaError_t born_launch_step(const BornArgs& a, int it, bool born, bool keep, cudaStream_t s);
cudaError_t born_launch_adjoint_step(const BornArgs& a, int it, cudaStream_t s);
cudaError_t born_launch_inject(const BornArgs& a, int it, cudaStream_t s);
// gradients summed over the launch's shots, written to (or, with accumulate, added to)
// the nz x nx outputs
cudaError_t born_launch_final(const BornArgs& a, float* gvp, float* gvs, float* grho, bool accumulate,
                              cudaStream_t s);

}  // namespace ertm
