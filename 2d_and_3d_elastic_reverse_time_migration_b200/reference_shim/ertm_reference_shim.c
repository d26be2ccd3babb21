/* Shim a maintainer adds to the reference's 3D driver (the file that would hold
 * its missing main) to route the three per-shot calls of
 * 3D_elastic_RTM/3D_forward_or_back_together.cu (:9, :161, :296) to libertm.
 * It reads the reference's globals (3D_elastic_modeling_parameter:1-141) and
 * keeps the reference's function names, so the shot loop is unchanged.
 * Link with -lertm; include/ertm.h declares everything used here. */
#include "ertm.h"

static ertm_ctx *g_ertm;           /* replaces GPUdevice mgdevice[MAX_GPU_COUNT] */

/* after elastic_modeling_parameter_input() and the CPU model preparation */
static void ertm_setup(void)
{
    ertm_config c = {0};
    c.nx = nnx; c.ny = nny; c.nz = nnz;              /* padded grid (bl/br, bf/bb, bu/bd) */
    c.dx = dx; c.dy = dy; c.dz = dz; c.dt_ms = dt;   /* dt in ms, as the reference */
    c.nt = lt; c.src_steps = 2 * lt / 3;             /* 3D_forward_or_back_together.cu:173 */
    c.order = 12; c.coef_kind = ERTM_COEF_REFERENCE12;       /* radius 6, zzzzz:202 */
    c.boundary = ERTM_BOUNDARY_SPONGE_COS; c.sponge_coef = coe_att;  /* 3D_zzzzz:261 */
    c.pml[0] = bl; c.pml[1] = br; c.pml[2] = bf; c.pml[3] = bb; c.pml[4] = bu; c.pml[5] = bd;
    c.device = gpuid[0];
    if (ertm_create(&c, &g_ertm)) { char m[512]; ertm_last_error(NULL, m, sizeof m); err("%s", m); }
    /* velocity_pml / velocity1_pml / density_pml are nnz*nny*nnx, x fastest (3D_zzzzz:21) */
    ertm_set_model(g_ertm, 0, velocity_pml, velocity1_pml, density_pml);
    ertm_set_model(g_ertm, 1, s_velocity_pml, s_velocity1_pml, s_density_pml);
}

/* the reference passes interior positions plus the offsets bl, bb, bu to
 * add_source_3D and write_or_add_shot_3D_surface_three
 * (3D_forward_or_back_together.cu:36, :127); ertm_shot takes padded-grid cells */
static ertm_shot shot_of_globals(void)
{
    ertm_shot s = {0};
    s.sx = sx_real + bl; s.sy = sy_real + bb; s.sz = sz_real + bu;
    s.nw = wavelet_length; s.wavelet = wavelet;
    s.rx0 = receiver_start_x + bl; s.nrx = receiver_num_x; s.drx = receiver_interval_x;
    s.ry0 = receiver_start_y + bb; s.nry = receiver_num_y; s.dry = receiver_interval_y;
    s.rz = receiver_start_z + bu;
    s.inject_mode = add_receiver_bool ? ERTM_INJECT_ADD : ERTM_INJECT_REPLACE;
    return s;
}

/* the three reference calls, same names, same order in the shot loop */
void forward_together_using_real_model(GPUdevice *unused)
{
    ertm_shot s = shot_of_globals();
    /* obs_shot_all: [3][lt][nry*nrx], host or device memory */
    if (ertm_forward_together_using_real_model(g_ertm, &s, obs_shot_all)) { /* ertm_last_error */ }
}
void forward_together_using_smoothed_model(GPUdevice *unused)
{
    ertm_shot s = shot_of_globals();
    ertm_forward_together_using_smoothed_model(g_ertm, &s);
}
void backward_together_using_smoothed_model(GPUdevice *unused)
{
    ertm_shot s = shot_of_globals();
    ertm_backward_together_using_smoothed_model(g_ertm, &s, obs_shot_all,
                                                vresult_pp_h, vresult_ps_h, vresult_tp_h);
}
