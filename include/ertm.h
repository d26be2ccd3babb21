/*
 * ertm.h — C ABI of the B200 elastic reverse-time-migration library (libertm.so).
 *
 * Drop-in for the reference's per-shot "forward/backward together" calls
 * (3D_elastic_RTM/3D_forward_or_back_together.cu):
 *
 *   reference                                         this library
 *   forward_together_using_real_model(GPUdevice*)     ertm_forward_together_using_real_model
 *       (:9-155, observed-data modelling)
 *   forward_together_using_smoothed_model(GPUdevice*) ertm_forward_together_using_smoothed_model
 *       (:161-290, source pass + excitation capture)
 *   backward_together_using_smoothed_model(GPUdevice*) ertm_backward_together_using_smoothed_model
 *       (:296-453, receiver pass + excitation-amplitude imaging)
 *
 * The reference functions read ~60 globals (3D_elastic_RTM/3D_elastic_modeling_parameter:1-141)
 * and a GPUdevice struct (3D_elastic_modeling_typedef_struct:1-55); here they
 * are an `ertm_config` (grid, time step, stencil, boundary), an `ertm_shot`
 * (source and receiver geometry) and an opaque context that owns every device
 * buffer.  Errors abort the process in the reference (checkCudaErrors); here
 * every call returns an int status (0 = OK, negative = ERTM_E*) and
 * ertm_last_error() returns the message.  No exception crosses this boundary.
 *
 * Conventions
 *  - Arrays are float32, x fastest: cell (i,j,k) at k*ny*nx + j*nx + i
 *    (the reference's 3D device layout, 3D_zzzzz:21).  ny == 1 is a 2D x–z grid.
 *  - The grid includes the absorbing layers (the reference's nnx/nny/nnz).
 *  - dt is in milliseconds (reference parameter `dt`, dt_real = dt/1000,
 *    2D_elastic_RTM/viscoelastic_equation.cu:66).
 *  - Pointer arguments may be host (pageable or pinned) or device memory of the
 *    context's GPU; the library detects which.
 *  - Calls are ordered on the context's stream and return when their results
 *    are complete.  One context per host thread; a context is not re-entrant.
 *  - Traces are [3][nt][nrec] (vx, vy, vz; vy is zero in 2D), receiver r =
 *    iry*nrx + irx.
 */
#ifndef ERTM_H
#define ERTM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ERTM_ABI_VERSION 1

/* status codes */
#define ERTM_OK        0
#define ERTM_EINVAL   -1   /* bad argument or size */
#define ERTM_ENOMEM   -2   /* device or host allocation failed */
#define ERTM_ECUDA    -3   /* CUDA runtime error */
#define ERTM_ESTATE   -4   /* call out of order (e.g. receiver pass before source pass) */
#define ERTM_ENOTSUP  -5   /* configuration not supported by the library */
#define ERTM_EDEVICE  -6   /* a device-side check failed (bounded wait expired, bad index) */

/* absorbing boundary kinds */
#define ERTM_BOUNDARY_CPML          0  /* convolutional PML (default) */
#define ERTM_BOUNDARY_SPONGE_COS    1  /* reference 3D damping, 3D_zzzzz:261-369 */
#define ERTM_BOUNDARY_SPONGE_CUBIC  2  /* reference 2D damping, zzzzz:238-325 */

/* difference coefficient sets */
#define ERTM_COEF_TAYLOR        0  /* Taylor coefficients of order 2R */
#define ERTM_COEF_REFERENCE12   1  /* reference optimised 12th order, zzzzz:202-210 (R=6) */
#define ERTM_COEF_USER          2  /* ertm_config.coef[1..R] */

/* receiver injection mode of the receiver pass (reference add_receiver_bool) */
#define ERTM_INJECT_ADD      1
#define ERTM_INJECT_REPLACE  2

/* wavefield ids for ertm_get_wavefield */
enum {
    ERTM_F_VX = 0, ERTM_F_VY, ERTM_F_VZ, ERTM_F_TXX, ERTM_F_TYY, ERTM_F_TZZ,
    ERTM_F_TXY, ERTM_F_TXZ, ERTM_F_TYZ, ERTM_F_TP, ERTM_F_VXP, ERTM_F_VYP, ERTM_F_VZP,
    ERTM_NFIELDS
};

typedef struct ertm_ctx ertm_ctx;

typedef struct {
    int   nx, ny, nz;        /* grid incl. absorbing layers; ny == 1 -> 2D */
    float dx, dy, dz;        /* metres */
    float dt_ms;             /* time step, milliseconds */
    int   nt;                /* samples of a full record (reference `lt`) */
    int   src_steps;         /* steps of the source pass; 0 -> 2*nt/3 as the reference (:173) */
    int   order;             /* 8 (R=4) or 12 (R=6) */
    int   coef_kind;         /* ERTM_COEF_* */
    float coef[8];           /* used when coef_kind == ERTM_COEF_USER */
    int   boundary;          /* ERTM_BOUNDARY_* */
    int   pml[6];            /* absorbing widths x0,x1,y0,y1,z0,z1 in cells */
    float pml_r;             /* CPML reflection coefficient (default 1e-3 when 0) */
    float pml_f0;            /* CPML alpha frequency in Hz (default 10 when 0) */
    float pml_vmax;          /* CPML velocity; 0 -> max Vp of the model */
    float sponge_coef;       /* reference coe_attenuation (sponge kinds) */
    int   device;            /* CUDA device ordinal */
    int   checkpoint_every;  /* Born adjoint: background checkpoint interval; 0 -> 200 */
    int   autotune;          /* 1: time the z-chunk candidates of the step kernels once per
                                grid shape (cached for the process); 0: fixed rule */
    int   visco_nmech;       /* Born operators: GSLS relaxation mechanisms, 0 (elastic) .. 3 */
    float visco_qp, visco_qs;  /* constant quality factors fitted by the mechanisms */
    float visco_f0;          /* centre of the fitted band, Hz */
    int   reserved[1];       /* must be zero */
} ertm_config;

typedef struct {
    int sx, sy, sz;          /* explosive source cell (reference sx_real, sy_real, sz_real) */
    int nw;                  /* wavelet samples (reference wavelet_length) */
    const float *wavelet;    /* host or device, nw values */
    int rx0, nrx, drx;       /* receiver grid along x (receiver_start_x/num_x/interval_x) */
    int ry0, nry, dry;       /* along y; nry = 1 in 2D */
    int rz;                  /* receiver depth index (receiver_start_z) */
    int inject_mode;         /* ERTM_INJECT_*, receiver pass; 0 -> ADD */
} ertm_shot;

/* Aperture window of one shot over a shared model (ertm_rtm_windows). */
typedef struct {
    int x0, y0;              /* window origin, model cells (no absorbing layers) */
    int wx, wy;              /* window size, model cells; wy = 1, y0 = 0 in 2D */
    int nt;                  /* record length of this shot, steps */
    int src_steps;           /* source-pass steps; 0 -> 2*nt/3 */
} ertm_window;

/* ---- lifecycle --------------------------------------------------------- */

/* Replaces allocate_typedef_struct (3D_elastic_modeling_typedef_struct:57-210).
 * Validates the config, selects the device, allocates every device buffer. */
int ertm_create(const ertm_config *cfg, ertm_ctx **out);
int ertm_destroy(ertm_ctx *ctx);
/* Message of the last failing call on this context (or of a failed create
 * when ctx is NULL, thread-local). Always NUL-terminates. */
int ertm_last_error(const ertm_ctx *ctx, char *buf, size_t len);
/* Use the caller's cudaStream_t (NULL restores the context's own stream). */
int ertm_set_stream(ertm_ctx *ctx, void *cuda_stream);
int ertm_abi_version(void);

/* Shrink (or restore) the active grid of a context to nx x ny x cfg.nz cells,
 * nx <= cfg.nx and ny <= cfg.ny of ertm_create, with record length nt and
 * source-pass length src_steps (0 -> 2*nt/3).  The buffers stay allocated at the
 * create-time size; models, excitation and Born state are dropped (set the
 * models again).  No counterpart in the reference, whose buffers are sized once
 * per run (allocate_typedef_struct); it lets one context serve shots on
 * aperture windows of different sizes without reallocating. */
int ertm_set_grid(ertm_ctx *ctx, int nx, int ny, int nt, int src_steps);

/* Batched RTM over aperture windows of one shared migration model.
 * No single counterpart in the reference, which migrates one shot per run on
 * the full grid and writes one image per shot (3D_output_file.cu:339-365).
 *  base     spacings, dt, order, coefficients, boundary, absorbing widths and
 *           device of every window grid; base->nx, ny, nz are the shared model's
 *           size WITHOUT absorbing layers; base->nt, src_steps are ignored.
 *  vp,vs,rho  the shared migration model, nz*ny*nx floats (host or device).
 *  win[i], shots[i]  window and shot i.  Source and receiver cells are given in
 *           model cells; each window grid is the model cropped to the window,
 *           all depths, extended by the absorbing layers with edge values.
 *  data[i]  observed data of shot i, [3][win[i].nt][nrx*nry] (host or device).
 *  lanes    shots per launch (1 .. ERTM_MULTI_MAX; larger values are clamped):
 *           the shots run in groups of `lanes`, each group through
 *           ertm_rtm_multi on contexts sized for the largest window, so every
 *           time step of a group is one launch of each step kernel for all of
 *           its shots.  Groups are formed from the shots in decreasing order of
 *           cost (cells x steps) and their images are stacked in that order.
 *  stack_*  nz*ny*nx sums of the windows' PP / PS / TP images (host or device;
 *           NULL skips one).  errbuf receives a message on failure. */
int ertm_rtm_windows(const ertm_config *base, const float *vp, const float *vs, const float *rho,
                     int nshots, const ertm_window *win, const ertm_shot *shots,
                     const float *const *data, int lanes, float *stack_pp, float *stack_ps,
                     float *stack_tp, char *errbuf, size_t errlen);

/* Load a model: which = 0 true model (velocity/velocity1/density),
 * which = 1 migration model (s_velocity/s_velocity1/s_density).
 * vp, vs, rho: nz*ny*nx floats (host or device), copied. */
int ertm_set_model(ertm_ctx *ctx, int which, const float *vp, const float *vs, const float *rho);

/* ---- the reference's three per-shot calls ------------------------------ */

/* Observed-data modelling in the true model for cfg.nt steps
 * (3D_forward_or_back_together.cu:9-155).  data_out: [3][nt][nrec]. */
int ertm_forward_together_using_real_model(ertm_ctx *ctx, const ertm_shot *shot, float *data_out);

/* Source pass in the migration model for src_steps steps with excitation
 * amplitude/time capture of the P velocity (:161-290).  The excitation state
 * stays in the context for the receiver pass. */
int ertm_forward_together_using_smoothed_model(ertm_ctx *ctx, const ertm_shot *shot);

/* Receiver pass it = nt-1 .. 0 injecting data_in [3][nt][nrec] and applying
 * the vector excitation-amplitude imaging condition (:296-453):
 *   PP = (e_P . r_P)/|e_P|^2,  PS = (e_P . r_S)/|e_P|^2,  TP = r_tp / e_tp
 * at it == excitation time.  Images are nz*ny*nx (full grid); any may be NULL. */
int ertm_backward_together_using_smoothed_model(ertm_ctx *ctx, const ertm_shot *shot,
                                                const float *data_in, float *img_pp,
                                                float *img_ps, float *img_tp);

/* Source pass then receiver pass: one RTM shot. */
int ertm_rtm_shot(ertm_ctx *ctx, const ertm_shot *shot, const float *data_in,
                  float *img_pp, float *img_ps, float *img_tp);

/* RTM of `nshots` shots on this context's GPU with the images stacked on the
 * device (the reference's shot loop and per-shot image files,
 * 3D_output_file.cu:339-365, become one sum); data[q] is shot q's
 * [3][nt][nrec] record.  Outputs are nz*ny*nx (any may be NULL).  Several GPUs
 * split a shot list between contexts and add their stacks (one reduce). */
int ertm_rtm_batch(ertm_ctx *ctx, const ertm_shot *shots, int nshots, const float *const *data,
                   float *stack_pp, float *stack_ps, float *stack_tp);

/* Several 3D shots migrated together, each on its own context: one RTM shot
 * (source pass, receiver pass) per context, as ertm_rtm_shot would run it, but
 * every time step is one launch of each step kernel covering all n shots (the
 * reference runs one shot per program invocation, 3D_forward_or_back_together.cu
 * :29,34,125).  ctx[q] holds shot q's grid (its own nx, ny, nt, src_steps, e.g.
 * through ertm_set_grid) and migration model; all contexts are 3D, distinct, on
 * one device, with the same nz, order and boundary kind; 1 <= n <= ERTM_MULTI_MAX.
 * Shots with fewer steps than the longest idle at the end of the source pass and
 * at the start of the receiver pass.  data[q] is shot q's [3][nt_q][nrec_q]
 * record (host or device).  img_pp/ps/tp: NULL, or arrays of n outputs of
 * ctx[q]'s grid (host or device; NULL entries skip).  All work runs on ctx[0]'s
 * stream; afterwards each context holds its shot's excitation and images, the
 * same numbers as ertm_rtm_shot gives. */
#define ERTM_MULTI_MAX 10
int ertm_rtm_multi(ertm_ctx *const *ctx, int n, const ertm_shot *shots, const float *const *data,
                   float *const *img_pp, float *const *img_ps, float *const *img_tp);

/* ---- least-squares RTM operators (2D, sponge boundaries) ---------------
 * The linearised (Born) modelling of the reference's LSRTM
 * (demig_fwd_txxzzxzpp_viscoelastic_and_memory_3parameterization and
 * cuda_cal_dem_parameter_viscoelastic_media_new, 2D_elastic_RTM/viscoelastic_equation.cu
 * :328-477, :2398-2505, inversion_para 2, elastic case) and its exact adjoint
 * (the role of adjoint_fwd_vx/vz_viscoelastic, adjoint_fwd_memory_new and
 * cal_gradient_in_viscoelastic_media_new, :1827-2294), in the migration model.
 * Perturbations are relative: r_vp = dvp/vp, r_vs = dvs/vs, r_rho = drho/rho
 * (nz*ny*nx each).  data/residual are [3][nt][nrec] (vx, 0, vz).  The adjoint
 * returns F^T residual, i.e. the gradient of 0.5 |F r - d|^2 when the residual
 * is F r - d; its background wavefield is rebuilt from checkpoints every
 * cfg.checkpoint_every steps (no full wavefield history is kept).
 * 2D grids with a sponge boundary only (ERTM_ENOTSUP otherwise). */
int ertm_born_forward(ertm_ctx *ctx, const ertm_shot *shot, const float *r_vp,
                      const float *r_vs, const float *r_rho, float *data_out);
int ertm_born_adjoint(ertm_ctx *ctx, const ertm_shot *shot, const float *residual,
                      float *g_vp, float *g_vs, float *g_rho);
/* The same operators over `nshots` shots at once: the shots of a group share every
 * step kernel launch (one grid layer per shot), the group as large as about 60 % of
 * the free device memory allows (at most 256 shots).  The reference's LSRTM driver,
 * absent from its tree, would loop over shots calling its per-shot kernels
 * (viscoelastic_equation.cu:328-477, :1827-2294, :2398-2505).  All shots need the
 * same receiver count and wavelet length.  data_out / residual hold
 * [nshots][3][nt][nrec]; the adjoint returns the gradient summed over the shots
 * (in shot order).  Host or device pointers. */
int ertm_born_forward_shots(ertm_ctx *ctx, const ertm_shot *shots, int nshots, const float *r_vp,
                            const float *r_vs, const float *r_rho, float *data_out);
int ertm_born_adjoint_shots(ertm_ctx *ctx, const ertm_shot *shots, int nshots,
                            const float *residual, float *g_vp, float *g_vs, float *g_rho);

/* ---- inspection (the reference's output_3d_wavefiled_* / EA outputs,
 *      3D_output_file.cu:2-250) ------------------------------------------ */

/* Current wavefield `field` (ERTM_F_*) into out (nz*ny*nx). */
int ertm_get_wavefield(ertm_ctx *ctx, int field, float *out);
/* Excitation state of the last source pass (any pointer may be NULL):
 * amplitude |v_P|, time index, v_P vector and P stress at that time. */
int ertm_get_excitation(ertm_ctx *ctx, float *amp, int32_t *time, float *evx, float *evy,
                        float *evz, float *etp);

/* Divergence/curl P/S decomposition of the current velocity field
 * (decom_new, 2D_elastic_RTM/elastic_2D_kernel_2.cu:671-791; 3D extension):
 * p = vp * div v; 2D: sy = vs*(dvx/dz - dvz/dx); 3D: sx, sy, sz the curl
 * components.  Uses the model `which`.  sx, sz ignored in 2D. */
int ertm_divcurl(ertm_ctx *ctx, int which, float *p, float *sx, float *sy, float *sz);

/* Run `nsteps` plain propagation steps of the modelling pass from a zero
 * state in model `which` (0/1) without recording: for wavefield checks. */
int ertm_propagate(ertm_ctx *ctx, int which, const ertm_shot *shot, int nsteps);

/* Device time of each step kernel over `nsteps` propagation steps of the
 * source pass, measured with CUDA events on the context stream:
 * ms[0] stress kernel, ms[1] velocity kernel (totals over nsteps). */
int ertm_time_kernels(ertm_ctx *ctx, const ertm_shot *shot, int nsteps, float *ms);

/* Number of kernels this context has launched (for launch accounting). */
int64_t ertm_kernel_launches(const ertm_ctx *ctx);

/* Variant of the 3D step kernels (both compute the same numbers to float
 * rounding): one cell per thread (the default, the faster on B200) or two
 * x-adjacent cells per thread with packed FP32 pairs.  No counterpart in the
 * reference; for measurement and equivalence tests.  2D grids always use one
 * cell per thread. */
#define ERTM_STEP_SINGLE  0
#define ERTM_STEP_PAIRS   1
int ertm_set_step_variant(ertm_ctx *ctx, int variant);

/* Test hook of the device-error path.  No counterpart in the reference (it
 * aborts on any CUDA error, 3D_forward_or_back_together.cu:34).  With
 * plane >= 0 the first CTA of every step-kernel launch does not issue the
 * staged copy of its z plane `plane` (a copy that never lands), so the bounded
 * wait of its consumers runs out after `polls` polls (0: the default budget);
 * the kernel then stops writing, its producer waits (bounded) for the copies it
 * did issue, and the pass returns ERTM_EDEVICE with the context still usable.
 * plane = -1 turns the hook off (the default). */
int ertm_set_wait_fault(ertm_ctx *ctx, int plane, uint32_t polls);

/* ---- modelling without device allocation ------------------------------
 * No counterpart in the reference: an addition of this library.
 *
 * The same modelling pass as ertm_forward_together_using_real_model, for
 * callers that must not allocate GPU memory when they call in (a plugin host
 * whose execute step forbids it, a real-time pipeline whose memory is fixed at
 * start-up, a framework whose own allocator owns the device).  No context is
 * created and nothing is allocated: the caller passes pointers to memory of
 * GPU cfg->device (or managed memory) for vp, vs, rho (nz*ny*nx),
 * shot->wavelet and data_out ([3][nt][nrec]); memory of another GPU is
 * refused with ERTM_EINVAL.  The wavefields live in one fixed 64 MiB device
 * array inside the library, held by every GPU that loads it until the process
 * exits.  A grid whose state does not fit returns ERTM_EINVAL with the needed
 * size in errbuf.  The first call on a device looks up that array's address,
 * and so does the first call after the device's context changed
 * (cudaDeviceReset); make such a call before any stream capture on that
 * device.  Calls share the array: calls that overlap on the GPU race, so
 * serialise them; each call clears the state it uses.  Work is ordered on
 * `cuda_stream` (NULL: the legacy default stream) and is complete on return.
 * errbuf (may be NULL) receives a message on failure. */
int ertm_forward_together_using_real_model_noalloc(const ertm_config *cfg, const float *vp,
                                                   const float *vs, const float *rho,
                                                   const ertm_shot *shot, float *data_out,
                                                   void *cuda_stream, char *errbuf,
                                                   size_t errlen);

/* ---- files and recorded data (host code) ------------------------------ */

/* Raw float32 volume in the reference's file order, x outer and z inner
 * (output_file_xyz_boundary / input_file_xyz_boundary, 3D_elastic_RTM/3D_zzzzz:1-139):
 * the file holds nx*ny*nz values; the array is (nzb, nyb, nxb) with x fastest and
 * the file's volume sits at offsets (bl, bf, bu) in x, y, z.  Offsets 0 and
 * full sizes give output_file_xyz / input_file_xyz.  Host arrays. */
int ertm_write_volume_xyz(const char *path, const float *vol, int nxb, int nyb, int nzb, int nx,
                          int ny, int nz, int bl, int bf, int bu);
int ertm_read_volume_xyz(const char *path, float *vol, int nxb, int nyb, int nzb, int nx, int ny,
                         int nz, int bl, int bf, int bu);

/* Image post-filters (host arrays (nz, ny, nx), x fastest).  Laplacian filter of
 * cpu_laplace (3D_elastic_RTM/zzzzz:1110-1147; 3D adds the y term): in place,
 * img <- vp^2 (-laplacian(img)) / 4 with the reference's edge handling.  Hilbert
 * transform along depth of suhilbt (3D_elastic_RTM/zzzzz:1018-1066) into out.  Both
 * work on the image interior the reference cuts out of its padded arrays. */
int ertm_laplace_filter(float *img, const float *vp, int nx, int ny, int nz, float dx, float dy,
                        float dz);
int ertm_hilbert_z(const float *img, float *out, int nx, int ny, int nz);

/* Gradient post-filters, host or device arrays (nz, ny, nx).  Truncated Gaussian
 * smoothing with weights exp(-i^2 / (2 rbell)), |i| <= rbell <= 64, renormalised
 * where the window leaves the array, one pass per axis in `axes` (z, then y, then x)
 * — cuda_bell_smoothz_new / cuda_bell_smoothx_new / cuda_bell_smooth_2d
 * (2D_elastic_RTM/viscoelastic_equation.cu:2528-2604).  `work` (n floats, same
 * memory space) is needed with two or more axes; `in` may equal `out` with exactly
 * two.  Device arrays run on `stream`; the call returns when the passes are done. */
#define ERTM_AXIS_X 1
#define ERTM_AXIS_Y 2
#define ERTM_AXIS_Z 4
int ertm_bell_smooth(const float *in, float *out, float *work, int nx, int ny, int nz, int rbell,
                     int axes, void *stream);
/* Cosine-power edge taper in x of cuda_attenuation_truncation
 * (viscoelastic_equation.cu:2881-2926; there left = offset_left/3, right =
 * offset_right/3, power 3), in place, host or device. */
int ertm_taper_x(float *img, int nx, int ny, int nz, int left, int right, int power, void *stream);
/* Aperture mute in x of cauda_zero_and_attenuation_truncation
 * (viscoelastic_equation.cu:2928-3045): columns outside [x0, x1) become 0 (an edge
 * of -1 leaves that side open) and the w columns inside each edge ramp with
 * cos^power; in place, host or device. */
int ertm_aperture_taper(float *img, int nx, int ny, int nz, int x0, int x1, int w, int power,
                        void *stream);

/* Propagation angles (2D grids).  With capture on, the source pass records at each
 * cell the P-wave propagation angle of the source wavefield at the cell's
 * excitation time, and the receiver pass that of the receiver wavefield at the
 * same time: Poynting vector p = -tp (vxp, vzp), angle = atan(sum px pz / sum pz^2)
 * over the 5 x 5 (source pass) or 9 x 9 (receiver pass) cells around the cell, in
 * degrees from the z axis; a cell whose window sum of pz^2 is zero keeps 0.  Replaces caculate_ex_angle_pp_only_RTM /
 * caculate_ex_angle_rp_only_RTM on sum_poynting's vectors
 * (2D_elastic_RTM/elastic_2D_kernel_3.cu:132-284, elastic_2D_kernel_2.cu:8-30).
 * One extra kernel per step while on; ERTM_ENOTSUP on 3D grids.  ertm_get_angles
 * copies either array out (NULL skips; host or device pointers, (nz, 1, nx)). */
int ertm_set_angles(ertm_ctx *ctx, int on);
int ertm_get_angles(ertm_ctx *ctx, float *src_angle, float *rcv_angle);

/* Angle-dependent compensation of a PP or PS image from the two angle arrays
 * (elastic_2D_kernel_3.cu:622-761), n cells, host or device arrays (all alike). */
#define ERTM_COMP_PP       0  /* img / (cos d + 1e-4), 0.1 near 90 degrees */
#define ERTM_COMP_PS       1  /* img / (sin|d| + 1e-4), 0.1 near 0 degrees */
#define ERTM_COMP_PP_SIGN  2  /* -sign(cos d) img / (|cos d| + 0.03) */
#define ERTM_COMP_PS_SIGN  3  /* -img / (|sin d| + 0.1) */
int ertm_angle_compensate(const float *img, const float *src_angle, const float *rcv_angle,
                          float *out, long long n, int kind, void *stream);

/* Angle-domain common-image gathers of one shot, accumulated into
 * cig[2*nang+1][nz][nx] (set_adcigs_for_ex, elastic_2D_kernel_3.cu:489-511): a cell
 * with iz > zmin and iz > slope*|ix - sx| adds its image value to bin
 * nang +/- (int)((|angle - normal| + 0.5) / dangle) when that offset is below nang.
 * normal may be NULL.  The reference uses zmin = 50, slope = 1.2. */
int ertm_adcig_bin(const float *img, const float *angle, const float *normal, float *cig, int nx,
                   int nz, int nang, float dangle, int sx, int zmin, float slope, void *stream);

/* Direct-wave mute of recorded data [3][nt][nrx*nry] (host or device), replacing
 * cut_direct_shot_3D_surface_three_new (3D_forward_or_back_together.cu:135, body
 * not in the reference tree): zeroes every sample it < ceil(t_d / dt) + shot->nw
 * + extra, t_d = |receiver - source| / v (straight ray, spacings dx, dy, dz in m). */
int ertm_mute_direct(const ertm_shot *shot, float *data, int nt, float dx, float dy, float dz,
                     float dt_ms, float v, int extra, void *stream);

/* ---- learned LSRTM preconditioner: tensor-core network kernels --------
 * No counterpart in the reference (its LSRTM has no learned part).  Building
 * blocks of a 2D U-Net: BF16 NHWC activations, FP32 accumulation in tensor
 * memory (tcgen05.mma), FP32 master weights.  All pointers are device
 * pointers; calls are asynchronous on `stream` (NULL: the legacy stream).
 * `err` (device int, may be NULL) is set non-zero if a kernel's bounded wait
 * gave up.  Channel counts, offsets and strides are multiples of 8; activation
 * and weight pointers start on a 16-byte boundary; an input gradient has the
 * grid of its output gradient, and a ReLU mask the layout (grid, stride,
 * channel offset and count) of the gradient it masks (ERTM_EINVAL otherwise). */
typedef struct {
    const void *data;        /* BF16, pixel p = (n*h + y)*w + x at data + p*cstride + coff */
    int n, h, w;             /* batch, height, width */
    int cstride, coff, c;    /* channels per pixel in memory, first channel, channels used */
} ertm_nn_act;

/* D[M][N] = A[M][K] B[N][K]^T, A and B BF16 row-major (K contiguous, K % 8 == 0), D FP32 */
int ertm_nn_gemm(const void *a, const void *b, float *d, int M, int N, int K, int *err, void *stream);
/* 3x3 convolution, zero padding 1: y = relu?(conv(x, w) + bias); w BF16 [y.c][9][x.c];
 * output into the BF16 view y, or FP32 y32[pixel][y.cstride] when y32 != NULL */
int ertm_nn_conv3x3(const ertm_nn_act *x, const void *w, const float *bias, const ertm_nn_act *y,
                    int relu, float *y32, int *err, void *stream);
/* input gradient through a 3x3 convolution: dx = conv(dy, wflip) (* (mask > 0) when mask);
 * wflip from ertm_nn_flip3 */
int ertm_nn_conv3x3_dgrad(const ertm_nn_act *dy, const void *wflip, const ertm_nn_act *dx,
                          const ertm_nn_act *mask, int *err, void *stream);
/* weight gradient of a 3x3 convolution, accumulated: dw[dy.c][9][x.c] += ... (split-K) */
int ertm_nn_conv3x3_wgrad(const ertm_nn_act *x, const ertm_nn_act *dy, float *dw, int splitk,
                          int *err, void *stream);
/* 2x2 stride-2 transposed convolution: y[2i+a][2j+b][o] = relu?(sum_c x[i][j][c] u[(2a+b)*y.c+o][c]
 * + bias[o]); x dense (coff 0, cstride c) */
int ertm_nn_up2(const ertm_nn_act *x, const void *u, const float *bias, const ertm_nn_act *y,
                int relu, int *err, void *stream);
/* input gradient of ertm_nn_up2 (ut = u transposed, [x.c][4 y.c]), optional ReLU mask */
int ertm_nn_up2_dgrad(const ertm_nn_act *dy, const void *ut, const ertm_nn_act *dx,
                      const ertm_nn_act *mask, int *err, void *stream);
/* weight gradient of ertm_nn_up2, accumulated: du[4 dy.c][x.c] += ... */
int ertm_nn_up2_wgrad(const ertm_nn_act *x, const ertm_nn_act *dy, float *du, int splitk, int *err,
                      void *stream);
/* 2x2 max pooling into a dense BF16 output [n][h/2][w/2][x.c] */
int ertm_nn_pool2(const ertm_nn_act *x, void *y, void *stream);
/* its backward: adds dy into dx at the first maximum of each window (dx has x's layout);
 * relu_mask: only where that maximum is positive */
int ertm_nn_pool2_bwd(const ertm_nn_act *x, const void *dy, const ertm_nn_act *dx, int relu_mask,
                      void *stream);
/* db[o] += sum over pixels of dy[..][o] */
int ertm_nn_bias_grad(const ertm_nn_act *dy, float *db, void *stream);
/* grad = scale (y - target) over the first c of cstride channels (BF16, padding 0);
 * *loss += sum (y - target)^2 */
int ertm_nn_mse(const float *y, const float *target, int cstride, int c, long long pixels,
                float scale, void *grad, float *loss, void *stream);
/* Adam step `step` (1-based) on FP32 weights; writes the BF16 copy wb */
int ertm_nn_adam(float *w, const float *g, float *m, float *v, void *wb, long long n, float lr,
                 float b1, float b2, float eps, int step, void *stream);
/* wf[c][8-tap][o] = w[o][tap][c] (BF16) */
int ertm_nn_flip3(const void *w, void *wf, int co, int ci, void *stream);
/* t[cols][rows] = a[rows][cols] (BF16) */
int ertm_nn_transpose(const void *a, void *t, int rows, int cols, void *stream);
int ertm_nn_to_bf16(const float *a, void *b, long long n, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* ERTM_H */
