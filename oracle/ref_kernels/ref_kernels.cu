// Golden-vector harness over the reference's own 2D CUDA kernels, compiled from
// the reference tree (paths passed by the Makefile).  Host wrappers copy small
// arrays in the reference's 2D layout (ix * (nz + 2 radius) + iz, radius-padded)
// to the device, launch one reference kernel and copy the result back.  Only
// tests/golden/make_golden_kernels.py calls it, to record fixtures.
#include "ref_shim.cuh"
#include REF_K2
#include REF_K3
#include REF_VISCO

#include <vector>

namespace {
struct Dev {
    std::vector<float*> p;
    float* put(const float* h, size_t n)
    {
        float* d = nullptr;
        cudaMalloc(&d, n * sizeof(float));
        if (h) cudaMemcpy(d, h, n * sizeof(float), cudaMemcpyHostToDevice);
        else cudaMemset(d, 0, n * sizeof(float));
        p.push_back(d);
        return d;
    }
    float* fill(float v, size_t n)
    {
        std::vector<float> h(n, v);
        return put(h.data(), n);
    }
    ~Dev() { for (float* d : p) cudaFree(d); }
};
int get(float* h, const float* d, size_t n)
{
    cudaDeviceSynchronize();
    cudaMemcpy(h, d, n * sizeof(float), cudaMemcpyDeviceToHost);
    return (int)cudaGetLastError();
}
}  // namespace

// fwd_txxzzxzpp_viscoelastic_and_memory_3parameterization (viscoelastic_equation.cu:184-325)
// with tao = strain = 1 (no attenuation: memory variables stay zero) and
// modul_p = vp^2, modul_s = vs^2: one elastic stress half-step with damping.
// nx % 32 == 0, nz % 16 == 0.  coe_x = dt/1000/dx (the reference host code that sets it is absent).
extern "C" int ref_stress_step(int nx, int nz, float dt_ms, float dx, float dz, const float* coe7,
                               const float* vp, const float* vs, const float* rho, const float* att,
                               const float* vx, const float* vz, const float* txx, const float* tzz,
                               const float* txz, float* otxx, float* otzz, float* otxz)
{
    const size_t n = (size_t)(nx + 2 * radius) * (nz + 2 * radius);
    Dev D;
    std::vector<float> mp(n), ms(n);
    for (size_t i = 0; i < n; i++) { mp[i] = vp[i] * vp[i]; ms[i] = vs[i] * vs[i]; }
    float *dvx = D.put(vx, n), *dvz = D.put(vz, n);
    float *t1xx = D.put(txx, n), *t1zz = D.put(tzz, n), *t1xz = D.put(txz, n);
    float *t2xx = D.put(nullptr, n), *t2zz = D.put(nullptr, n), *t2xz = D.put(nullptr, n);
    float *tp1 = D.put(nullptr, n), *tp2 = D.put(nullptr, n);
    float *mpd = D.put(mp.data(), n), *msd = D.put(ms.data(), n), *attd = D.put(att, n);
    float *rhod = D.put(rho, n), *vpd = D.put(vp, n), *vsd = D.put(vs, n);
    float* mem[8];
    for (int q = 0; q < 8; q++) mem[q] = D.put(nullptr, n);
    float *tao = D.fill(1.f, n), *sp = D.fill(1.f, n), *ss = D.fill(1.f, n);
    float* coe = D.put(coe7, 7);
    const float coe_x = dt_ms / 1000.f / dx, coe_z = dt_ms / 1000.f / dz;
    fwd_txxzzxzpp_viscoelastic_and_memory_3parameterization<<<dim3(nx / 32, nz / 16), dim3(32, 16)>>>(
        tp2, tp1, t2xx, t1xx, t2zz, t1zz, t2xz, t1xz, dvx, dvz, mpd, msd, attd, dt_ms, coe, coe_x,
        coe_z, nx, nz, rhod, mem[0], mem[1], mem[2], mem[3], mem[4], mem[5], mem[6], mem[7], vpd, vsd,
        tao, sp, ss);
    int e = get(otxx, t2xx, n);
    e |= get(otzz, t2zz, n);
    e |= get(otxz, t2xz, n);
    return e;
}

// decom_new (elastic_2D_kernel_2.cu:671-791): P = vp div v, S = vs curl v
extern "C" int ref_decom_new(int nx, int nz, float dx, float dz, const float* coe7, const float* vx,
                             const float* vz, const float* vp, const float* vs, float* p, float* s)
{
    const size_t n = (size_t)(nx + 2 * radius) * (nz + 2 * radius);
    Dev D;
    float *dvx = D.put(vx, n), *dvz = D.put(vz, n), *dp = D.put(nullptr, n), *ds = D.put(nullptr, n);
    float *vpd = D.put(vp, n), *vsd = D.put(vs, n), *coe = D.put(coe7, 7);
    decom_new<<<dim3(nx / 32, nz / 16), dim3(32, 16)>>>(dvx, dvz, dp, ds, vpd, vsd, coe, nx, nz, dx, dz);
    int e = get(p, dp, n);
    e |= get(s, ds, n);
    return e;
}

// imaging_inner_product_ex_2D (elastic_2D_kernel_3.cu:559-580) with every cell's
// excitation time equal to `it`; plain nx*nz arrays (no padding, no offsets)
extern "C" int ref_imaging(int nx, int nz, const float* ex, const float* ez, const float* rx,
                           const float* rz, float* out)
{
    const size_t n = (size_t)nx * nz;
    Dev D;
    float *dex = D.put(ex, n), *dez = D.put(ez, n), *drx = D.put(rx, n), *drz = D.put(rz, n);
    float *dt = D.put(nullptr, n), *amp = D.put(nullptr, n), *dout = D.put(nullptr, n);
    float* mx = D.fill(1.f, 1);
    imaging_inner_product_ex_2D<<<dim3((nx + 31) / 32, (nz + 15) / 16), dim3(32, 16)>>>(
        dout, amp, dex, dez, dt, drx, drz, nx, nz, nz, 0, 0, mx, 0);
    return get(out, dout, n);
}

// cuda_cal_dem_parameter_viscoelastic_media_new (viscoelastic_equation.cu:2398-2505),
// inversion_para 2 (relative vp, vs, rho perturbations), no attenuation.
// out: dem_p1, dem_p2, then dem_p[2..4] (stress sources), each padded n.
extern "C" int ref_dem_sources(int nx, int nz, float dt_ms, const float* vp, const float* vs,
                               const float* rho, const float* rvp, const float* rvs, const float* rrho,
                               const float* vx_x, const float* vx_z, const float* vz_x,
                               const float* vz_z, const float* vx_t, const float* vz_t, float* out)
{
    const size_t n = (size_t)(nx + 2 * radius2) * (nz + 2 * radius2);
    Dev D;
    float *d1 = D.put(nullptr, n), *d2 = D.put(nullptr, n), *dall = D.put(nullptr, 8 * n);
    float *a = D.put(vx_x, n), *b = D.put(vx_z, n), *c = D.put(vz_x, n), *d = D.put(vz_z, n);
    float *e = D.put(vx_t, n), *f = D.put(vz_t, n);
    float *z0 = D.put(nullptr, n), *z1 = D.put(nullptr, n), *z2 = D.put(nullptr, n);
    float *pvp = D.put(rvp, n), *pvs = D.put(rvs, n), *pr = D.put(rrho, n);
    float *vpd = D.put(vp, n), *vsd = D.put(vs, n), *rhod = D.put(rho, n);
    float *tao = D.fill(1.f, n), *sp = D.fill(1.f, n), *ss = D.fill(1.f, n);
    cuda_cal_dem_parameter_viscoelastic_media_new<<<dim3(nx / 32, nz / 16), dim3(32, 16)>>>(
        d1, d2, dall, a, b, c, d, e, f, z0, z1, z2, pvp, pvs, pr, nx, nz, vpd, vsd, rhod, tao, sp, ss,
        dt_ms, 2);
    int err = get(out, d1, n);
    err |= get(out + n, d2, n);
    err |= get(out + 2 * n, dall + 2 * n, 3 * n);
    return err;
}

// Device time of the reference's own 2D time step on an nx x nz interior
// (radius-padded, ix-major layout): the stress kernel
// fwd_txxzzxzpp_viscoelastic_and_memory_3parameterization
// (viscoelastic_equation.cu:184-325) then the velocity kernels
// adjoint_fwd_vx_viscoelastic and adjoint_fwd_vz_viscoelastic (:1827-2122),
// launched with the reference's tiles (32 x 16) and time-level ping-pong, as its
// driver would.  Inputs are smooth nonzero fields (the timing does not depend on
// the values); no result is read back.  nx % 32 == 0, nz % 16 == 0.
// ms[0], ms[1], ms[2]: total CUDA-event time of each kernel over nsteps steps
// (warm-up steps excluded).  Only bench.py calls it.
extern "C" int ref_time_step(int nx, int nz, int nsteps, int warmup, float dt_ms, float dx, float dz,
                             const float* coe7, float* ms)
{
    if (nx % 32 || nz % 16 || nsteps < 1) return -1;
    const size_t n = (size_t)(nx + 2 * radius) * (nz + 2 * radius);
    Dev D;
    std::vector<float> h(n);
    auto smooth = [&](float a, float b) {
        for (size_t i = 0; i < n; i++) h[i] = a + b * (float)((i * 2654435761u) % 1000u) / 1000.f;
        return D.put(h.data(), n);
    };
    float *vx[2] = {smooth(0.f, 1e-3f), smooth(0.f, 1e-3f)};
    float *vz[2] = {smooth(0.f, 1e-3f), smooth(0.f, 1e-3f)};
    float *txx[2] = {smooth(0.f, 1e-3f), smooth(0.f, 1e-3f)};
    float *tzz[2] = {smooth(0.f, 1e-3f), smooth(0.f, 1e-3f)};
    float *txz[2] = {smooth(0.f, 1e-3f), smooth(0.f, 1e-3f)};
    float *tp[2] = {smooth(0.f, 1e-3f), smooth(0.f, 1e-3f)};
    float* mem[2][4];
    for (int t = 0; t < 2; t++)
        for (int q = 0; q < 4; q++) mem[t][q] = D.put(nullptr, n);
    float *vp = smooth(2500.f, 500.f), *vs = smooth(1400.f, 300.f), *rho = smooth(2200.f, 100.f);
    float *mp = smooth(6.25e6f, 1e6f), *msd = smooth(1.96e6f, 4e5f), *att = smooth(0.f, 10.f);
    float *tao = D.fill(1.f, n), *sp = D.fill(1.f, n), *ss = D.fill(1.f, n);
    float* coe = D.put(coe7, 7);
    const float coe_x = dt_ms / 1000.f / dx, coe_z = dt_ms / 1000.f / dz;
    const dim3 grid(nx / 32, nz / 16), block(32, 16);
    cudaEvent_t ev[4];
    for (int q = 0; q < 4; q++) cudaEventCreate(&ev[q]);
    float tot[3] = {0.f, 0.f, 0.f};
    for (int s = 0; s < warmup + nsteps; s++) {
        const int a = s & 1, b = a ^ 1;   // time level a -> b
        cudaEventRecord(ev[0]);
        fwd_txxzzxzpp_viscoelastic_and_memory_3parameterization<<<grid, block>>>(
            tp[b], tp[a], txx[b], txx[a], tzz[b], tzz[a], txz[b], txz[a], vx[a], vz[a], mp, msd, att,
            dt_ms, coe, coe_x, coe_z, nx, nz, rho, mem[b][0], mem[a][0], mem[b][1], mem[a][1],
            mem[b][2], mem[a][2], mem[b][3], mem[a][3], vp, vs, tao, sp, ss);
        cudaEventRecord(ev[1]);
        adjoint_fwd_vx_viscoelastic<<<grid, block>>>(vx[b], vx[a], txx[b], txz[b], tzz[b], att, dx, dz,
                                                     dt_ms, coe, coe_x, coe_z, nx, nz, mp, msd, rho,
                                                     mem[b][0], mem[b][1], mem[b][2], mem[b][3], vp, vs,
                                                     tao, sp, ss);
        cudaEventRecord(ev[2]);
        adjoint_fwd_vz_viscoelastic<<<grid, block>>>(vz[b], vz[a], txx[b], txz[b], tzz[b], att, dx, dz,
                                                     dt_ms, coe, coe_x, coe_z, nx, nz, mp, msd, rho,
                                                     mem[b][0], mem[b][1], mem[b][2], mem[b][3], vp, vs,
                                                     tao, sp, ss);
        cudaEventRecord(ev[3]);
        cudaEventSynchronize(ev[3]);
        if (s >= warmup) {
            float t;
            for (int q = 0; q < 3; q++) {
                cudaEventElapsedTime(&t, ev[q], ev[q + 1]);
                tot[q] += t;
            }
        }
    }
    for (int q = 0; q < 4; q++) cudaEventDestroy(ev[q]);
    for (int q = 0; q < 3; q++) ms[q] = tot[q];
    return (int)cudaGetLastError();
}

// sum_poynting (elastic_2D_kernel_2.cu:8-30) then caculate_ex_angle_pp_only_RTM
// (hw_mode 0, 5 x 5 window) or caculate_ex_angle_rp_only_RTM (hw_mode 1, 9 x 9)
// (elastic_2D_kernel_3.cu:132-284) at step `it`.  Inputs radius-padded, ix-major;
// ex_time as the reference's float array.  `angle` (padded) keeps its input values
// where the kernel writes nothing.  nx % 32 == 0, nz % 16 == 0.
extern "C" int ref_angle(int nx, int nz, int hw_mode, int it, const float* tp, const float* vxp,
                         const float* vzp, const float* ex_time, float* angle)
{
    if (nx % 32 || nz % 16) return -1;
    const size_t n = (size_t)(nx + 2 * radius) * (nz + 2 * radius);
    Dev D;
    float *dtp = D.put(tp, n), *dvxp = D.put(vxp, n), *dvzp = D.put(vzp, n);
    float *zero = D.put(nullptr, n);
    float *px = D.put(nullptr, n), *pz = D.put(nullptr, n), *sx = D.put(nullptr, n), *sz = D.put(nullptr, n);
    float *det = D.put(ex_time, n), *dang = D.put(angle, n);
    const dim3 grid(nx / 32, nz / 16), block(32, 16);
    sum_poynting<<<grid, block>>>(px, pz, sx, sz, dvxp, dvzp, zero, zero, zero, zero, zero, dtp, nx, nz);
    if (hw_mode == 0)
        caculate_ex_angle_pp_only_RTM<<<grid, block>>>(dang, px, pz, det, it, nx, nz);
    else
        caculate_ex_angle_rp_only_RTM<<<grid, block>>>(dang, px, pz, det, it, nx, nz);
    return get(angle, dang, n);
}

// Angle-dependent compensation of an image, plain ix-major nx x nz arrays, every
// cell at its excitation step (ex_time = it = 0):
//   kind 0 imaging_pp_compensate_dependent_angle_2D, kind 1 imaging_ps_... (:622-676);
//   kind 2 caculate_ex_open_pp_ps + cuda_ex_com_pp_ps_sign(mark 0) +
//          imaging_pp_compensate_dependent_angle_2D_new;
//   kind 3 the same with mark 1 and imaging_ps_compensate_dependent_angle_2D_new (:678-761).
// out: the compensated image; for kinds 0 and 1 also rcv_out = the kernel's
// rewrite of the receiver angle (the open angle).
extern "C" int ref_compensate(int nx, int nz, int kind, const float* src, const float* rcv,
                              const float* img, float* out, float* rcv_out)
{
    const size_t n = (size_t)nx * nz;
    Dev D;
    float *ds = D.put(src, n), *dr = D.put(rcv, n), *di = D.put(img, n), *dout = D.put(nullptr, n);
    float *det = D.put(nullptr, n), *open = D.put(nullptr, n), *sgn = D.put(nullptr, n);
    const dim3 grid((nx + 31) / 32, (nz + 15) / 16), block(32, 16);
    if (kind == 0)
        imaging_pp_compensate_dependent_angle_2D<<<grid, block>>>(ds, dr, dout, di, det, nx, nz, nz, 0, 0, 0);
    else if (kind == 1)
        imaging_ps_compensate_dependent_angle_2D<<<grid, block>>>(ds, dr, dout, di, det, nx, nz, nz, 0, 0, 0);
    else {
        caculate_ex_open_pp_ps<<<grid, block>>>(open, ds, dr, nx, nz, nx, nz, 0, 0, 0, det);
        cuda_ex_com_pp_ps_sign<<<grid, block>>>(sgn, open, nx, nz, nx, nz, kind == 2 ? 0 : 1);
        if (kind == 2)
            imaging_pp_compensate_dependent_angle_2D_new<<<grid, block>>>(open, sgn, dout, di, det, nx, nz,
                                                                           nz, 0, 0);
        else
            imaging_ps_compensate_dependent_angle_2D_new<<<grid, block>>>(open, sgn, dout, di, det, nx, nz,
                                                                           nz, 0, 0);
    }
    int e = get(out, dout, n);
    if (rcv_out) e |= get(rcv_out, dr, n);
    return e;
}

// cuda_bell_smoothz_new (mode 0), cuda_bell_smoothx_new (mode 1) or
// cuda_bell_smooth_2d (mode 2) (viscoelastic_equation.cu:2528-2604); ix-major nx x nz.
extern "C" int ref_bell(int nx, int nz, int rbell, int mode, const float* g, float* out)
{
    const size_t n = (size_t)nx * nz;
    Dev D;
    float *dg = D.put(g, n), *dout = D.put(nullptr, n);
    const dim3 grid((nx + 31) / 32, (nz + 15) / 16), block(32, 16);
    if (mode == 0) cuda_bell_smoothz_new<<<grid, block>>>(dg, dout, rbell, nx, nz);
    else if (mode == 1) cuda_bell_smoothx_new<<<grid, block>>>(dg, dout, rbell, nx, nz);
    else cuda_bell_smooth_2d<<<grid, block>>>(dg, dout, rbell, nx, nz);
    return get(out, dout, n);
}

// cuda_attenuation_truncation (zero_mode 0, :2881-2926) or
// cauda_zero_and_attenuation_truncation (zero_mode 1, :2928-2988) in place on an
// ix-major nx x nz array.
extern "C" int ref_truncation(int nx, int nz, int zero_mode, int offset_left, int offset_right,
                              int receiver_offset, int offset_attenuation, float* g)
{
    const size_t n = (size_t)nx * nz;
    Dev D;
    float* dg = D.put(g, n);
    const dim3 grid((nx + 31) / 32, (nz + 15) / 16), block(32, 16);
    if (zero_mode == 0)
        cuda_attenuation_truncation<<<grid, block>>>(dg, nx, nz, offset_left, offset_right, receiver_offset);
    else
        cauda_zero_and_attenuation_truncation<<<grid, block>>>(dg, nx, nz, offset_left, offset_right,
                                                               receiver_offset, offset_attenuation);
    return get(g, dg, n);
}
