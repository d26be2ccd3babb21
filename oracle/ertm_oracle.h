/*
 * CPU oracle for the elastic RTM hot path — TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-loop restatement of the reference's staggered-grid
 * velocity–stress propagation, P/S split, excitation-amplitude capture and
 * excitation-amplitude imaging.  It exists to check the CUDA library and to
 * time a CPU baseline; nothing in the product links or calls it.
 *
 * Built twice from the same source (oracle/Makefile):
 *   liboracle64.so   REAL = double  (the parity oracle)
 *   liboracle32.so   REAL = float   (the OpenMP CPU baseline)
 * Every entry point below takes and returns float arrays; REAL is internal.
 *
 * Parity pinning: the helper functions (Ricker, difference coefficients,
 * sponge profiles) and the 2D kernels that survive in the reference are
 * checked against outputs of the reference's own code (tests/golden); the 3D
 * assembly has no reference implementation (its kernels are absent from the
 * reference tree), so the 3D oracle extends the 2D forms and is pinned only
 * through those pieces.
 *
 * Grid convention (shared with the CUDA library, x fastest):
 *   cell (i,j,k) -> k*ny*nx + j*nx + i,  ny == 1 means a 2D x–z grid.
 *   txx,tyy,tzz,tp at (i, j, k)
 *   vx at (i-1/2, j, k), vy at (i, j-1/2, k), vz at (i, j, k+1/2)
 *   txy at (i-1/2, j-1/2, k), txz at (i-1/2, j, k+1/2), tyz at (i, j-1/2, k+1/2)
 * which extends the 2D staggering of
 *   2D_elastic_RTM/viscoelastic_equation.cu:137-149 (stress, D+x vx, D-z vz)
 *   2D_elastic_RTM/viscoelastic_equation.cu:164-176 (shear, D-x vz, D+z vx)
 *   2D_elastic_RTM/viscoelastic_equation.cu:1827-1973 (vx: D-x txx, D-z txz)
 *   2D_elastic_RTM/viscoelastic_equation.cu:1976-2122 (vz: D+x txz, D+z tzz)
 * Fields outside [0,n) are zero (the reference pads every array by `radius`).
 */
#ifndef ERTM_ORACLE_H
#define ERTM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_BOUNDARY_CPML = 0, ORC_BOUNDARY_SPONGE_COS = 1, ORC_BOUNDARY_SPONGE_CUBIC = 2 };
enum { ORC_MODE_MODEL = 0, ORC_MODE_SOURCE = 1, ORC_MODE_RECEIVER = 2 };

typedef struct {
    int nx, ny, nz;          /* grid including absorbing layers; ny == 1 -> 2D */
    double dx, dy, dz;       /* metres */
    double dt_ms;            /* milliseconds, as the reference's `dt` */
    int R;                   /* stencil half-width: 4 (8th order) or 6 (12th order) */
    double coef[8];          /* coef[1..R] */
    int boundary;            /* ORC_BOUNDARY_* */
    int pml[6];              /* absorbing widths x0,x1,y0,y1,z0,z1 (cells) */
    double pml_r;            /* CPML target reflection coefficient */
    double pml_f0;           /* CPML alpha frequency (Hz) */
    double pml_vmax;         /* CPML reference velocity (m/s) */
    double sponge_coef;      /* reference `coe_attenuation` */
    int visco_nmech;         /* Born operators: relaxation mechanisms (0 elastic, 1..3 GSLS) */
    double visco_qp, visco_qs, visco_f0;   /* constant Q targets and reference frequency (Hz) */
} orc_grid;

/* GSLS relaxation of `nmech` mechanisms fitted to constant qp, qs around f0
 * (tau method, first order): tau_sigma[l] and the P and S strengths. */
void orc_visco_fit(int nmech, double qp, double qs, double f0, double *tau_sigma, double *tau_p,
                   double *tau_s);

typedef struct {
    int sx, sy, sz;          /* explosive source cell */
    int nw;                  /* wavelet samples */
    const float *wavelet;    /* one sample per step */
    int rx0, nrx, drx;       /* receiver grid along x */
    int ry0, nry, dry;       /* receiver grid along y (nry = 1 in 2D) */
    int rz;                  /* receiver depth index */
    int inject_mode;         /* 1 add (default), 2 replace */
} orc_shot;

/* Excitation state written by the source pass, read by the receiver pass.
 * All arrays nz*ny*nx. `amp2` is |v_P|^2 at the excitation time; `second2`
 * is the largest |v_P|^2 seen at any other step (used only to detect ties). */
typedef struct {
    float *amp2, *second2;
    int   *time;
    float *evx, *evy, *evz, *etp;
    /* 2D only, optional (NULL = off): P-wave propagation angle in degrees at the
     * excitation time, of the source wavefield (written by the source pass) and of
     * the receiver wavefield (written by the receiver pass); see orc_window_angle. */
    float *src_angle, *rcv_angle;
    /* optional (NULL = off): the window's P energy sum (px^2 + pz^2) at each angle
     * capture, to tell cells with a real wavefield from cells that only hold the
     * stencil's numerical precursor (where the angle means nothing) */
    float *src_energy, *rcv_energy;
} orc_excitation;

/* ---- model-independent helpers --------------------------------------- */
int  orc_ricker(double freq_hz, double dt_s, float *out, int maxn);
void orc_coef_taylor(int R, double *coef);
void orc_coef_reference12(double *coef);
void orc_sponge_profile(int kind, int n, int w0, int w1, double coe, double *out);
void orc_cpml_profile(int n, int w0, int w1, double h, double dt_s, double vmax,
                      double rc, double f0, int stagger, double *a, double *b);

/* ---- propagation passes ---------------------------------------------- */
/* Runs `nsteps` time steps of one pass in the model (vp, vs, rho).
 *  MODEL:    records vx,vy,vz at the receivers into data[3][nsteps][nrec]
 *            (it = 0 .. nsteps-1), source injected.
 *  SOURCE:   source injected; P/S split on; excitation capture into `ex`.
 *  RECEIVER: it = nsteps-1 .. 0; data[3][nsteps][nrec] injected; P/S split on;
 *            imaging into img_pp, img_ps, img_tp (nz*ny*nx, zeroed here).
 * If `final_fields` is non-NULL it receives 13 arrays of nz*ny*nx in the order
 *  vx vy vz txx tyy tzz txy txz tyz tp vxp vyp vzp  (state after the pass).
 * Returns 0 on success, negative on bad arguments / allocation failure. */
int orc_run_pass(const orc_grid *g, const float *vp, const float *vs, const float *rho,
                 const orc_shot *s, int mode, int nsteps, float *data,
                 orc_excitation *ex, float *img_pp, float *img_ps, float *img_tp,
                 float *final_fields);

/* Divergence / curl P/S decomposition of a velocity field (restates
 * 2D_elastic_RTM/elastic_2D_kernel_2.cu:671-791 decom_new, extended to 3D):
 *   P = vp * div v  at (i,j,k)
 *   2D: S = vs * (d vx/dz - d vz/dx) at the txz point
 *   3D: Sx = vs*(d vz/dy - d vy/dz) at tyz, Sy = vs*(d vx/dz - d vz/dx) at txz,
 *       Sz = vs*(d vy/dx - d vx/dy) at txy.
 * In 2D only p and sy are written. */
int orc_divcurl(const orc_grid *g, const float *vp, const float *vs,
                const float *vx, const float *vy, const float *vz,
                float *p, float *sx, float *sy, float *sz);

/* ---- Born modelling and its adjoint (2D, sponge boundaries) ----------
 * Linearised (first-order scattering) modelling for relative perturbations
 * r_vp, r_vs, r_rho of the model (vp, vs, rho): the scattered field obeys the
 * background scheme with secondary sources
 *   stress  : dt (dM e0_xx + dL e0_zz, dL e0_xx + dM e0_zz, dU e0_xz)
 *   velocity: -dt r_rho a0
 * with dM = M (r_rho + 2 r_vp), dU = U (r_rho + 2 r_vs), dL = dM - 2 dU, e0 the
 * background strain rates and a0 = b div(sigma0) the background acceleration —
 * the reference's secondary sources (cuda_cal_dem_parameter_viscoelastic_media_new,
 * 2D_elastic_RTM/viscoelastic_equation.cu:2398-2505, inversion_para 2) without
 * attenuation.  This is the exact derivative of orc_run_pass's discrete scheme.
 * born_forward records vx, vz of the scattered field into data[3][nt][nrec].
 * born_adjoint applies the exact transpose of born_forward to `residual`
 * ([3][nt][nrec]) and returns the gradients w.r.t. r_vp, r_vs, r_rho. */
/* Modelling pass of the Born background scheme (2D, sponge; viscoelastic when
 * g->visco_nmech > 0): data[3][nt][nrx] of vx, (0), vz after every step. */
int orc_visco_model(const orc_grid *g, const float *vp, const float *vs, const float *rho,
                    const orc_shot *s, int nt, float *data);
int orc_born_forward(const orc_grid *g, const float *vp, const float *vs, const float *rho,
                     const orc_shot *s, int nt, const float *r_vp, const float *r_vs,
                     const float *r_rho, float *data);
int orc_born_adjoint(const orc_grid *g, const float *vp, const float *vs, const float *rho,
                     const orc_shot *s, int nt, const float *residual, float *g_vp, float *g_vs,
                     float *g_rho);

/* Single pieces of the scheme on given inputs, for comparison with the
 * reference's own 2D kernels (see ertm_oracle.c). */
int orc_stress_step_given(const orc_grid *g, const float *vp, const float *vs, const float *rho,
                          const float *vx, const float *vz, const float *txx, const float *tzz,
                          const float *txz, float *otxx, float *otzz, float *otxz);
int orc_born_sources_given(long n, double dt_ms, const float *vp, const float *vs, const float *rho,
                           const float *rvp, const float *rvs, const float *rrho, const float *exx,
                           const float *ezz, const float *exz, const float *ax, const float *az,
                           float *osxx, float *oszz, float *osxz, float *osvx, float *osvz);
int orc_image_given(long n, const float *ex, const float *ez, const float *rpx, const float *rpz,
                    const float *rsx, const float *rsz, float *pp, float *ps);

/* Stepping state for callers that run a pass one step at a time (the CPU
 * baseline's timed sample, the angle tests): create, step (same arguments as one
 * iteration of orc_run_pass), read all 13 fields [13][nz][ny][nx], destroy. */
void *orc_state_create(const orc_grid *g, const float *vp, const float *vs, const float *rho);
void orc_state_step(void *st, const orc_shot *s, int mode, int it, int nsteps, float *data,
                    orc_excitation *ex, float *pp, float *ps, float *ptp);
void orc_state_fields(const void *st, float *out);
void orc_state_destroy(void *st);

/* Window propagation angle on given 2D arrays (see ertm_oracle.c). */
int orc_angle_given(int nx, int nz, int hw, int it, const float *tp, const float *vxp,
                    const float *vzp, const int *ex_time, float *out);

/* Threads used by the OpenMP loops (1 if built without OpenMP). */
int orc_threads(void);
/* sizeof(REAL) of the loaded library (8 or 4). */
int orc_real_size(void);

#ifdef __cplusplus
}
#endif
#endif
