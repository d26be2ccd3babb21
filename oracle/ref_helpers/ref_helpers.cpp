// Golden-vector generator: runs the reference's own CPU helpers
// (3D_elastic_RTM/zzzzz and 3D_elastic_RTM/3D_zzzzz, included from the
// reference tree at build time) on small fixed inputs and prints JSON.
#include "su_shim.h"
#include REF_ZZZZZ
#include REF_3D_ZZZZZ

static void arr(const char *name, const float *v, long n, bool last = false)
{
    printf("\"%s\": [", name);
    for (long i = 0; i < n; i++) printf("%s%.9g", i ? "," : "", v[i]);
    printf("]%s\n", last ? "" : ",");
}

int main()
{
    printf("{\n");
    // make_ricker_new (zzzzz:139-160)
    const float fr[3] = {10.f, 15.f, 30.f};
    const float dts[3] = {0.0008f, 0.0005f, 0.001f};
    for (int q = 0; q < 3; q++) {
        int np = 0;
        float *w = make_ricker_new(fr[q], dts[q], &np);
        char nm[64];
        snprintf(nm, sizeof nm, "ricker_%g_%g", fr[q], dts[q]);
        arr(nm, w, np);
        free1float(w);
    }
    // make_coe_optimized_new (zzzzz:202-219)
    float coe[7] = {0};
    make_coe_optimized_new(coe);
    arr("coe_optimized12", coe, 7);
    // make_attenuation_new, 2D cubic damping (zzzzz:238-325): nx=20 nz=16, bu=5 bd=6 bl=4 br=7
    {
        int nx = 20, nz = 16, bu = 5, bd = 6, bl = 4, br = 7;
        int nxa = bl + nx + br, nza = bu + nz + bd;
        float *att = alloc1float((size_t)nxa * nza);
        make_attenuation_new(att, nx, nz, bu, bd, bl, br, 200.f);
        arr("att2d_cubic_ix_major", att, (long)nxa * nza);
        free1float(att);
    }
    // coe_attenuation_3d_new2, 3D cosine damping (3D_zzzzz:261-369)
    {
        int nx = 9, ny = 8, nz = 7, bu = 3, bd = 4, bl = 5, br = 3, bf = 2, bb = 4;
        int nxb = nx + bl + br, nyb = ny + bf + bb, nzb = nz + bu + bd;
        float *att = alloc1float((size_t)nxb * nyb * nzb);
        coe_attenuation_3d_new2(att, nx, ny, nz, bu, bd, bl, br, bf, bb, 150.f);
        arr("att3d_cos_z_major", att, (long)nxb * nyb * nzb);
        free1float(att);
    }
    // add_pml_layers_v_h, edge-replicating padding (3D_zzzzz:141-259)
    {
        int nx = 5, ny = 4, nz = 3, bl = 2, bf = 3, bu = 1;
        int nxb = nx + bl + 2, nyb = ny + bf + 1, nzb = nz + bu + 2;
        float *v = alloc1float((size_t)nxb * nyb * nzb);
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++)
                    v[(k + bu) * nxb * nyb + (j + bf) * nxb + i + bl] = 1000.f + 100.f * k + 10.f * j + i;
        add_pml_layers_v_h(v, nx, ny, nz, bl, bf, bu, nxb, nyb, nzb);
        arr("pad3d_z_major", v, (long)nxb * nyb * nzb);
        free1float(v);
    }
    // cpu_laplace (zzzzz:1110-1147) on an image of nx = 12, nz = 9 (nx >= nz keeps the
    // reference's row-copy loop inside the array), no boundary offsets; layout ix*nz+iz
    {
        int nx = 12, nz = 9;
        float *img = alloc1float((size_t)nx * nz), *vel = alloc1float((size_t)nx * nz);
        for (int ix = 0; ix < nx; ix++)
            for (int iz = 0; iz < nz; iz++) {
                img[ix * nz + iz] = (float)(sin(0.7 * ix + 0.3) * cos(0.45 * iz - 0.2) + 0.05 * ((ix * 7 + iz * 3) % 5));
                vel[ix * nz + iz] = 2000.f + 25.f * iz + 10.f * ix;
            }
        arr("laplace_in_ix_major", img, (long)nx * nz);
        arr("laplace_vel_ix_major", vel, (long)nx * nz);
        cpu_laplace(img, vel, nx, nz, nx, nz, 0, 0, 5.f, 4.f);
        arr("laplace_out_ix_major", img, (long)nx * nz);
        free1float(img);
        free1float(vel);
    }
    // suhilbt (zzzzz:1018-1066) along z, nx = 5 columns, nz = 16 and nz = 15; layout ix*nz+iz
    for (int nz = 15; nz <= 16; nz++) {
        int nx = 5;
        float *img = alloc1float((size_t)nx * nz), *out = alloc1float((size_t)nx * nz);
        for (int ix = 0; ix < nx; ix++)
            for (int iz = 0; iz < nz; iz++)
                img[ix * nz + iz] = (float)(cos(2 * PI * (ix + 1) * iz / nz + 0.1 * ix) + 0.3 * sin(0.9 * iz * iz / nz) - 0.1 * ix);
        suhilbt(img, out, nx, nz, nx, nz, 0, 0, 5.f, 5.f);
        char nm[64];
        snprintf(nm, sizeof nm, "hilbert_in_nz%d_ix_major", nz);
        arr(nm, img, (long)nx * nz);
        snprintf(nm, sizeof nm, "hilbert_out_nz%d_ix_major", nz);
        arr(nm, out, (long)nx * nz);
        free1float(img);
        free1float(out);
    }
    // vp_set_vs / vp_set_density (zzzzz:1261-1287)
    {
        float vp[4] = {1800.f, 2500.f, 3200.f, 4500.f}, vs[4], rho[4];
        vp_set_vs(vp, vs, 2, 2);
        vp_set_density(vp, rho, 2, 2);
        arr("vp_in", vp, 4);
        arr("vs_from_vp", vs, 4);
        arr("rho_from_vp", rho, 4, true);
    }
    printf("}\n");
    return 0;
}
