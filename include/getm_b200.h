/* getm_b200.h -- C ABI of the B200 implementation of GETM's per-timestep 3D hot path.
 *
 * Every entry point is a drop-in for one GETM 2.5 subroutine (getm-model/code, cited per
 * function as path:line) or for a fused group of them. Arrays are DEVICE pointers in the
 * reference's own layout: a 3D field covers the haloed index space
 * (imin-2:imax+2, jmin-2:jmax+2, 0:kmax), i fastest, element (i,j,k) at
 *     base + (i-(imin-2)) + (j-(jmin-2))*sj + k*sk
 * (Fortran column-major when sj = imax-imin+5 and sk = sj*(jmax-jmin+5); padded pitches are
 * allowed). 2D fields use the same (i,j) addressing with no k term. Masks az/au/av/ax are int32
 * like the reference's integer masks.
 *
 * Calling convention: one host thread per context; every call is stream-ordered on the context's
 * stream and returns a status (0 = OK, < 0 = error, see GETM_ERR_*). No call exits the process:
 * where the reference calls stop / getm_error, the entry point returns an error code and the
 * Fortran-side wrapper turns it into getm_error.
 *
 * Suffixes: no suffix = FP64 (the reference's REALTYPE, cppdefs.h:130-131),
 *           _f32      = FP32 arithmetic for the same routine (the mixed-precision variant).
 */
#ifndef GETM_B200_H
#define GETM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------------------- */
#define GETM_OK 0
#define GETM_ERR_ARG (-1)         /* invalid argument (reference: stop '... is invalid') */
#define GETM_ERR_CUDA (-2)        /* a CUDA runtime call or kernel launch failed */
#define GETM_ERR_UNSUPPORTED (-3) /* valid in the reference but not provided here */
#define GETM_ERR_CHECK (-4)       /* a device-side check failed (range / NaN / iteration cap) */
#define GETM_ERR_TIMEOUT (-5)     /* a bounded device wait ran out */
#define GETM_ERR_NOMEM (-6)       /* device allocation failed */
#define GETM_ERR_STATE (-7)       /* call order violated (e.g. masks not initialised) */
#define GETM_ERR_TOO_LARGE (-8)   /* the domain exceeds a fixed size limit of the entry point */

/* ---- scheme / split / tag identifiers (values as in the reference) --------------------- */
/* advection.F90:55,60-62 ; advection_3d.F90:42 */
#define GETM_NOSPLIT 0
#define GETM_FULLSPLIT 1
#define GETM_HALFSPLIT 2
#define GETM_HVSPLIT 3
#define GETM_NOADV 0
#define GETM_UPSTREAM 1
#define GETM_UPSTREAM_2DH 2
#define GETM_P2 3
#define GETM_SUPERBEE 4
#define GETM_MUSCL 5
#define GETM_P2_PDM 6
#define GETM_J7 7
#define GETM_FCT 8
#define GETM_P2_2DH 9
/* halo_zones.F90:25-27 ; advection_3d.F90:42 */
#define GETM_H_TAG 10
#define GETM_D_TAG 20
#define GETM_U_TAG 31
#define GETM_V_TAG 32
#define GETM_W_TAG 33

/* ---- domain and context ---------------------------------------------------------------- */
/* The index space and Cartesian metrics of domain.F90 (imin..kmax, dx, dy, ard1=1/(dx*dy),
 * domain.F90:596). */
typedef struct getm_domain {
  int32_t imin, imax, jmin, jmax, kmax;
  int64_t sj, sk; /* element strides of j and k (the i stride is 1) */
  double dx, dy, ard1;
} getm_domain;

typedef struct getm_ctx getm_ctx;

/* Device pointers of one t_adv_grid (advection.F90:43-51): byte masks, 1 = .true. */
typedef struct getm_adv_grid {
  const uint8_t *mask_uflux, *mask_vflux, *mask_uupdate, *mask_vupdate, *mask_finalise;
  const int32_t *az;
} getm_adv_grid;

/* Creates a context on the current CUDA device; `stream` is a cudaStream_t (NULL = legacy
 * default stream). Replaces the allocation part of init_3d / init_advection (m3d.F90:88,
 * advection.F90:204). */
int getm_ctx_create(const getm_domain *dom, void *stream, getm_ctx **out);
int getm_ctx_destroy(getm_ctx *ctx);
int getm_ctx_set_stream(getm_ctx *ctx, void *stream);
/* Accumulated device-side warnings since the last call, e.g. the number of water columns whose
 * vertical-advection iteration estimate exceeded adv_ver_iterations (adv_split_w.F90:223-228
 * prints these). Synchronises the context's stream. */
int getm_ctx_take_warnings(getm_ctx *ctx, int64_t *n_warnings);
/* Per-stage device timers: the counterpart of the reference's tic/toc subsystem timers
 * (src/futils/getm_timers.F90:275-357). When enabled, every kernel launch of a stage is
 * bracketed by CUDA events on the context's stream; read accumulates (synchronising) the elapsed
 * device time and the launch count of a slot. */
#define GETM_TIM_ADV_U 0
#define GETM_TIM_ADV_V 1
#define GETM_TIM_ADV_W 2
#define GETM_TIM_ADV_FINALISE 3
#define GETM_TIM_VDIFF 4
#define GETM_TIM_COPY 5
#define GETM_TIM_TRACER_UV 6
#define GETM_TIM_TRACER_WVU 7
#define GETM_TIM_BC2D 8  /* 2D kernels of the mode-split step */
#define GETM_TIM_BC3D 9  /* other 3D kernels of the macro step */
#define GETM_TIM_IP 10   /* internal pressure */
#define GETM_TIM_MOM3D 11 /* uu/vv_momentum_3d */
#define GETM_TIM_ADJ_RECORD 12 /* forward tracer steps that write the adjoint tape */
#define GETM_TIM_ADJ 13        /* adjoint tracer steps */
#define GETM_NTIMERS 16
int getm_timers_enable(getm_ctx *ctx, int on);
int getm_timers_reset(getm_ctx *ctx);
int getm_timers_read(getm_ctx *ctx, int slot, double *total_ms, int64_t *launches);
const char *getm_timer_name(int slot);
/* Process-wide choice of the horizontal split-sweep kernels (no counterpart in the reference: a
 * tuning and testing switch). on != 0 (the default) runs the FP32 sweeps and the FP64 v sweeps in
 * the vectorised kernels wherever the rows and levels of the swept fields start on 16-byte
 * boundaries; on == 0 uses the shared-memory tile sweeps everywhere (the FP64 u sweep always
 * does). Both give identical results. Returns the previous setting. */
int getm_set_vector_sweeps(int on);
/* Process-wide choice for the mixed-precision step (no counterpart in the reference: a testing and
 * accuracy switch). on != 0 (the default) runs the barotropic micro steps of getm_time_loop on FP32
 * working copies of the 2D fields whenever the step has no open boundaries (the elevation and
 * Uint/Vint stay FP64); on == 0 keeps the micro steps on the FP64 state arrays, as the plain step
 * does. Returns the previous setting. */
int getm_set_fp32_micro_steps(int on);
/* Process-wide choice of the micro-step launches (no counterpart in the reference: a tuning and
 * testing switch). on != 0 (the default): getm_time_loop without open boundaries runs sealevel and
 * depth_update as one launch per micro step, the new elevations alternating between the z and zo
 * arrays (at the end of the call z and zo hold what the separate launches leave), forms each
 * Coriolis term inside the velocity update that reads it (the call's last term at its end), and
 * the mixed-precision micro step forms its bottom friction inside the momentum-advection kernels;
 * on == 0: the separate launches. Both give identical results. Returns the previous setting. */
int getm_set_fused_micro_step(int on);
/* Human-readable text of the last error on this context (never NULL). */
const char *getm_ctx_last_error(const getm_ctx *ctx);
const char *getm_version(void);

/* init_advection (advection.F90:204-354): builds the flux/update/finalise masks of the H, U and
 * V advection grids from the device masks az, au, av, ax (int32, E2DFIELD). Must precede any
 * advection call. The context keeps its own copies. */
int getm_init_advection(getm_ctx *ctx, const int32_t *az, const int32_t *au, const int32_t *av,
                        const int32_t *ax);
/* The mask set that do_advection_3d selects for `tag` (advection_3d.F90:262-277). */
int getm_adv_grid_for_tag(const getm_ctx *ctx, int tag, getm_adv_grid *out);

/* ---- split advection sweeps ------------------------------------------------------------ */
/* adv_split_u (src/2d/adv_split_u.F90:8-295) applied to `nk` consecutive k-levels (pointers
 * point at the first level, levels are sk apart; nk = 1 is the reference's 2D call). f and fi
 * may alias (the reference's in-place call, advection_3d.F90:446). adv may be NULL when the
 * caller does not need the advective increments. */
int getm_adv_split_u(getm_ctx *ctx, int nk, double dt, const double *f, double *fi, double *Di,
                     double *adv, const double *U, const double *DU, double splitfac, int scheme,
                     double AH, const uint8_t *mask_flux, const uint8_t *mask_update);
/* adv_split_v (src/2d/adv_split_v.F90:8-145), same conventions. */
int getm_adv_split_v(getm_ctx *ctx, int nk, double dt, const double *f, double *fi, double *Di,
                     double *adv, const double *V, const double *DV, double splitfac, int scheme,
                     double AH, const uint8_t *mask_flux, const uint8_t *mask_update);
/* adv_split_w (src/3d/adv_split_w.F90:7-360), full 3D fields; f and fi may alias. */
int getm_adv_split_w(getm_ctx *ctx, double dt, const double *f, double *fi, double *hi, double *adv,
                     const double *ww, double splitfac, int scheme, int tag, const int32_t *az,
                     int itersmax);
/* The same three sweeps in FP32 (the arithmetic of the mixed-precision step). */
int getm_adv_split_u_f32(getm_ctx *ctx, int nk, float dt, const float *f, float *fi, float *Di,
                         float *adv, const float *U, const float *DU, float splitfac, int scheme,
                         float AH, const uint8_t *mask_flux, const uint8_t *mask_update);
int getm_adv_split_v_f32(getm_ctx *ctx, int nk, float dt, const float *f, float *fi, float *Di,
                         float *adv, const float *V, const float *DV, float splitfac, int scheme,
                         float AH, const uint8_t *mask_flux, const uint8_t *mask_update);
int getm_adv_split_w_f32(getm_ctx *ctx, float dt, const float *f, float *fi, float *hi, float *adv,
                         const float *ww, float splitfac, int scheme, int tag, const int32_t *az,
                         int itersmax);

/* do_advection_3d (src/3d/advection_3d.F90:120-598): NOSPLIT / FULLSPLIT / HALFSPLIT / HVSPLIT
 * with the split schemes UPSTREAM, P2, SUPERBEE, MUSCL, P2_PDM (the 2DH schemes are not
 * provided: GETM_ERR_UNSUPPORTED). hires and advres are the optional outputs (NULL = absent).
 * adv_ver_iterations is the module variable of advection_3d.F90:41. */
int getm_do_advection_3d(getm_ctx *ctx, double dt, double *f, const double *uu, const double *vv,
                         const double *ww, const double *hu, const double *hv, const double *ho,
                         const double *hn, int split, int hscheme, int vscheme, double AH, int tag,
                         double *hires, double *advres, int adv_ver_iterations);
int getm_do_advection_3d_f32(getm_ctx *ctx, float dt, float *f, const float *uu, const float *vv,
                             const float *ww, const float *hu, const float *hv, const float *ho,
                             const float *hn, int split, int hscheme, int vscheme, float AH,
                             int tag, float *hires, float *advres, int adv_ver_iterations);

/* ---- vertical columns ------------------------------------------------------------------ */
/* getm_tridiagonal (src/futils/tridiagonal.F90:8-51) on ncol independent systems of size
 * 0:kmax. Coefficient arrays are laid out [k][col] (column fastest): au[k*ncol+c]. Levels fi..lt
 * are solved; value is written on fi..lt only. */
int getm_tridiagonal_columns(getm_ctx *ctx, int ncol, int kmax, int fi, int lt, const double *au,
                             const double *bu, const double *cu, const double *du, double *value);

/* Implicit vertical diffusion of a tracer on all wet interior columns (az==1, imin..imax x
 * jmin..jmax): the matrix assembly and solve of do_salinity (src/3d/salinity.F90:348-389) when
 * src == NULL, or of do_temperature (src/3d/temperature.F90:471-550) with src holding per layer
 * the radiation / surface-flux increment dry_z*dt*(rad1d(k)[+shf*rho_0_cpi]-rad1d(k-1)). */
int getm_tracer_vdiff(getm_ctx *ctx, double dt, double cnpar, double avmol, double *S,
                      const double *hn, const double *nuh, const int32_t *az, const double *src);
int getm_tracer_vdiff_f32(getm_ctx *ctx, float dt, float cnpar, float avmol, float *S,
                          const float *hn, const float *nuh, const int32_t *az, const float *src);

/* Fused tracer step = do_advection_3d(H_TAG) followed by the vertical-diffusion solve, i.e. the
 * body of do_salinity (salinity.F90:301-389) for fwf_int = 0 and no numerical-mixing analysis. */
int getm_tracer_step(getm_ctx *ctx, double dt, double *f, const double *uu, const double *vv,
                     const double *ww, const double *hu, const double *hv, const double *ho,
                     const double *hn, const double *nuh, int split, int hscheme, int vscheme,
                     double AH, double cnpar, double avmol, int adv_ver_iterations);
int getm_tracer_step_f32(getm_ctx *ctx, float dt, float *f, const float *uu, const float *vv,
                         const float *ww, const float *hu, const float *hv, const float *ho,
                         const float *hn, const float *nuh, int split, int hscheme, int vscheme,
                         float AH, float cnpar, float avmol, int adv_ver_iterations);

/* ---- the mode-split time step ----------------------------------------------------------- */
/* The module state that integrate_2d / integrate_3d read and write (variables_2d, variables_3d,
 * domain and the m2d/m3d/temperature/salinity/eqstate settings of the reference) as one table of
 * DEVICE pointers. 2D fields are FP64 (E2DFIELD); 3D fields (I3DFIELD) are FP64 when prec3d = 8
 * (the plain FP64 step) or FP32 when prec3d = 4 (the mixed-precision step, whose 2D substeps,
 * transport accumulation Uint/Vint and all vertical sums stay FP64). The table order is:
 *  f2:  z zo U V D DU DV UEx VEx fU fV ru rv ruu rvv Uint Vint Uinto Vinto SlUx SlVx Slru Slrv
 *       zub zvb zub0 zvb0 fwf H HU HV dry_z dry_u dry_v coru corv tausx tausy airp sseo ssen
 *       ssuo ssun ssvo ssvn Dn Dun Dvn rru rrv taubx tauby taub taus swr shf A g1 g2
 *  f3:  uu vv ww ho hn huo hun hvo hvn uuEx vvEx idpdx idpdy T S rho buoy num nuh rad tke eps
 *       Tlo Slo
 *  par: dtm dt cnpar min_depth crit_depth g rho_0 kappa avmmol avmolt avmols T0 S0 dtr0 dsr0
 *       ip_fac temp_AH salt_AH avmback avhback cp swr_bot_refl_frac swr_min_bot_frac
 *  ipar: M MM runtype vel2d_adv_split vel2d_adv_hor vel3d_adv_split vel3d_adv_hor
 *       vel3d_adv_ver temp_adv_split temp_adv_hor temp_adv_ver salt_adv_split salt_adv_hor
 *       salt_adv_ver adv_ver_iterations ufirst2d ufirst3d calc_temp calc_salt ip_method
 *       viscosity eqstate_method sealevel_check radiation nan_warned
 * ufirst2d / ufirst3d are the SAVEd alternation switches of momentum.F90:33 (initially 0) and
 * m3d.F90:504 (initially 1); the calls update them in the host-side struct. ip_method selects the
 * internal pressure gradient (internal_pressure.F90:80, 149-168): 1 = BLUMBERG_MELLOR,
 * 2 = BLUMBERG_MELLOR_LIN, 3 = Z_INTERPOL, 4 = SONG_WRIGHT, 5 = CHU_FAN, 6 = SHCHEPETKIN_MCWILLIAMS,
 * 7 = STELLING_VANKESTER (kmax <= 64, else GETM_ERR_UNSUPPORTED); other values GETM_ERR_ARG.
 * viscosity: 0 = CONSTANT_VISCOSITY (num, nuh as given), 1 = PARABOLIC_VISCOSITY (gotm.F90:131-143:
 * the profile from taub after stresses_3d, plus avmback / avhback; tke and eps receive the
 * profiles when not NULL). eqstate_method (eqstate.F90:31): 1 linear, 2 UNESCO80, 3 Jackett et al.
 * 2006 at zero pressure. radiation: 0 = do_temperature without sources (the reference with swr =
 * shf = 0), 1 = the short-wave radiation profile into rad (temperature.F90:452-465, from swr and
 * the attenuation A, g1, g2) and its absorption plus the surface heat flux shf as sources of the
 * temperature diffusion (temperature.F90:469-525, cp the heat capacity of parameters.F90:23, bottom
 * reflection when swr_bot_refl_frac > 0). sealevel_check (m2d.F90:82): every |sealevel_check|
 * micro steps the elevations are swept for NaN (sealevel_nan_check, sealevel.F90:172-314) until the
 * first finding, which sets nan_warned (the routine's SAVEd have_warned); sealevel_check > 0 makes a
 * finding an error: the call that made it returns GETM_ERR_CHECK (getm_time_loop at its end, after
 * finishing its steps; the reference stops at once). swr, shf, A, g1, g2 and rad may be NULL when
 * radiation = 0, tke and eps may always be NULL.
 * Tlo, Slo (no counterpart in the reference; FP32 states only, may be NULL): compensated storage of
 * the mixed step's temperature and salinity, as IEEE binary16 (2 bytes per element, the 3D layout of
 * the other fields). T is then the unevaluated sum T + e of an FP32 number and its carried rounding
 * error e (|e| <= half an ulp of T), stored as Tlo = e * 2^16 -- likewise S: every advection sweep
 * and diffusion solve adds its increment to T exactly and keeps the rounding error in e, so that the
 * increments smaller than half an ulp of T -- which plain FP32 storage loses at every update, and
 * which a tracer far from zero receives every sweep -- are kept to about 11 more bits. Valid for
 * |T| < 2^23. The fluxes and the equation of state read T alone. Start them at zero; NULL gives
 * plain FP32 storage. The FP64 step ignores them. */
#define GETM_NF2 59
#define GETM_NF3 24
#define GETM_NPD 23
#define GETM_NPI 25
typedef struct getm_bc_state {
  double *f2[GETM_NF2];
  void *f3[GETM_NF3];
  const int32_t *az, *au, *av, *ax;
  double par[GETM_NPD];
  int32_t ipar[GETM_NPI];
  int32_t prec3d; /* bytes per 3D element: 8 or 4 */
} getm_bc_state;

/* integrate_2d (src/2d/m2d.F90:412-490): one barotropic micro step -- bottom_friction (every MM
 * steps), uv_advect, momentum (alternating u/v order), Uint/Vint accumulation, sealevel and
 * depth_update. Closed boundaries (no update_2d_bdy), Am <= 0, An_method = 0, no residual. */
int getm_integrate_2d(getm_ctx *ctx, getm_bc_state *st, int loop);
/* integrate_3d (src/3d/m3d.F90:422-636): one baroclinic macro step for runtype 4 with sigma
 * coordinates: start_macro, bottom_friction_3d, internal pressure (ip_method), uu/vv_momentum_3d,
 * coordinates, ww_momentum_3d, uv_advect_3d, stresses_3d, gotm (PARABOLIC_VISCOSITY when
 * viscosity = 1), do_temperature / do_salinity (advection + implicit vertical diffusion; with
 * radiation = 1 the short-wave and surface heat-flux sources of temperature), do_eqstate
 * (eqstate_method), slow_bottom_friction, uv_advect of Uint/Vint, slow_terms and stop_macro.
 * The vertical grid is sigma coordinates with equidistant layers: every level of a column has the
 * same layer height (ho, hn, huo, hun, hvo, hvn), as sigma_coordinates and the initialisation
 * produce them; the step reads a column's height once where it needs it for all levels. */
int getm_integrate_3d(getm_ctx *ctx, getm_bc_state *st, int n);
/* The micro-step loop of time_loop (src/getm/integration.F90:98-172) for n = n0..n0+count-1:
 * integrate_2d every step, integrate_3d when runtype >= 2 and mod(n, M) == 0 (do_3d,
 * integration.F90:106). */
int getm_time_loop(getm_ctx *ctx, getm_bc_state *st, int n0, int count);

/* ---- the substeps of the mode-split step, one by one ------------------------------------
 * Each is one reference subroutine on the state table (same validation as getm_integrate_2d; the
 * 2D arithmetic of the 2D substeps is FP64, as in the plain step), for a host that keeps its own
 * integrate_2d / integrate_3d and swaps single calls. */
/* bottom_friction(runtype) (src/2d/bottom_friction.F90:8-250) */
int getm_bottom_friction(getm_ctx *ctx, getm_bc_state *st, int runtype);
/* uv_advect(U,V,DU,DV) (src/2d/uv_advect.F90:8-310): UEx, VEx */
int getm_uv_advect(getm_ctx *ctx, getm_bc_state *st);
/* momentum(n,tausx,tausy,airp) (src/2d/momentum.F90:8-60): umomentum and vmomentum in the order
 * of the SAVEd switch ufirst2d, which the call toggles; tausx, tausy, airp are the state's */
int getm_momentum(getm_ctx *ctx, getm_bc_state *st, int n);
/* umomentum(tausx,airp) (src/2d/momentum.F90:69-223): U, its mirror_bdy_2d copies, fV */
int getm_umomentum(getm_ctx *ctx, getm_bc_state *st);
/* vmomentum(tausy,airp) (src/2d/momentum.F90:232-386): V, its mirror_bdy_2d copies, fU */
int getm_vmomentum(getm_ctx *ctx, getm_bc_state *st);
/* update_2d_bdy(loop,bdy2d_ramp) (src/2d/update_2d_bdy.F90:8-186) with the context's open
 * boundaries (no-op without) */
int getm_update_2d_bdy(getm_ctx *ctx, getm_bc_state *st, int loop);
/* sealevel(loop) (src/2d/sealevel.F90:8-163): zo = z, the elevation update, and the NaN sweep of
 * sealevel_check (GETM_ERR_CHECK for sealevel_check > 0 and a finding) */
int getm_sealevel(getm_ctx *ctx, getm_bc_state *st, int loop);
/* depth_update() (src/2d/depth_update.F90:8-148): D, DU, DV and the drying factors */
int getm_depth_update(getm_ctx *ctx, getm_bc_state *st);
/* do_internal_pressure() (src/3d/internal_pressure.F90:181-274): idpdx, idpdy by ip_method */
int getm_internal_pressure(getm_ctx *ctx, getm_bc_state *st);
/* do_eqstate() (src/3d/eqstate.F90:94-261): rho and buoy by eqstate_method */
int getm_do_eqstate(getm_ctx *ctx, getm_bc_state *st);
/* gotm() (src/3d/gotm.F90:96-163) with PARABOLIC_VISCOSITY when viscosity = 1 (no-op for 0) */
int getm_gotm(getm_ctx *ctx, getm_bc_state *st);
/* the short-wave radiation profile rad of do_temperature (src/3d/temperature.F90:452-465) */
int getm_sw_radiation(getm_ctx *ctx, getm_bc_state *st);
/* sealevel_nan_check() (src/2d/sealevel.F90:172-314) on a device elevation field z (E2DFIELD,
 * FP64): the number of interior points that are not below HUGE (NaN, +Inf, HUGE; -Inf is not
 * counted, nor are halo points) into the HOST *num_nan, and the last of them in the reference's
 * loop order into *inan, *jnan (reference indices; may be NULL; 0 when none). Synchronises. */
int getm_sealevel_nan_check(getm_ctx *ctx, const double *z, int64_t *num_nan, int32_t *inan,
                            int32_t *jnan);

/* ---- open boundaries ------------------------------------------------------------------ */
/* The open-boundary description of bdy_spec.F90 (domain.F90:263-280 marks the points az = 2):
 * segments per side, in the order western (wi, wfj, wlj), northern (nj, nfi, nli), eastern
 * (ei, efj, elj), southern (sj, sfi, sli) -- seg holds 3 ints per segment, reference indices --
 * with a 2D type each (ZERO_GRADIENT 1, SOMMERFELD 2, CLAMPED 3, FLATHER_ELEV 4, cppdefs.h:65-68).
 * The nsbv = npoints boundary points are numbered in segment order (bdy_map). Elevation data
 * (bdy_data): `data` per point, or harmonic amp[p]*sin(2*pi*loop*dtm/period + phase[p]) at micro
 * step `loop` when amp != NULL; data_u / data_v = bdy_data_u / bdy_data_v of FLATHER_ELEV (NULL =
 * zero). All pointers are HOST arrays, copied by getm_set_open_boundaries. With boundaries set,
 * getm_integrate_2d / getm_integrate_3d / getm_time_loop apply update_2d_bdy (m2d.F90:475) and
 * the mirror_bdy_2d / mirror_bdy_3d copies of momentum.F90:190,353, uu_momentum_3d.F90:389,
 * vv_momentum_3d.F90:400 and m3d.F90:595,602. Call after getm_init_advection (the masks select
 * the mirrored points). */
typedef struct {
  int32_t nwb, nnb, neb, nsb;
  const int32_t *seg;
  const int32_t *type2d;
  int32_t ramp;    /* bdy2d_ramp (<= 1: no ramp) */
  int32_t npoints; /* nsbv */
  const double *data, *data_u, *data_v, *amp, *phase;
  double period;
} getm_bdy;
int getm_set_open_boundaries(getm_ctx *ctx, const getm_bdy *bdy);
/* New boundary data for the following steps (get_2d_bdy's job in the reference): HOST arrays of
 * npoints values each (data_u / data_v may be NULL); switches off harmonic data. */
int getm_set_bdy_data(getm_ctx *ctx, const double *data, const double *data_u, const double *data_v);

/* ---- hotstart: the restart file's fields ------------------------------------------------- */
/* The fields GETM writes to and reads from its restart file (write_restart_ncdf.F90:86-204,
 * read_restart_ncdf.F90), in the file's order, as indices into getm_bc_state.f2 / .f3:
 *   2D: z zo U SlUx Slru V SlVx Slrv; runtype >= 2 also ssen ssun ssvn sseo ssuo ssvo Uinto Vinto
 *   3D (runtype >= 2): uu vv ww uuEx vvEx tke eps num nuh hn; runtype >= 3 also T S
 * f2_ids / f3_ids (may be NULL) receive up to GETM_NF2 / GETM_NF3 indices; *n2, *n3 the counts. */
int getm_restart_fields(int runtype, int32_t *f2_ids, int32_t *n2, int32_t *f3_ids, int32_t *n3);
/* Device -> host for restart_file(WRITING) (output.F90:383): each restart field's extent in the file
 * -- the interior imin..imax x jmin..jmax (x levels 0..kmax), no halos (cppdefs.h:161-170) -- into
 * the HOST FP64 arrays host2[q] (nx*ny) and host3[q] (nx*ny*(kmax+1)), i fastest, in the order of
 * getm_restart_fields; FP32 3D fields are widened, a NULL tke / eps is written as zeros.
 * Synchronises. */
int getm_restart_write(getm_ctx *ctx, const getm_bc_state *st, int runtype, double *const *host2,
                       double *const *host3);
/* Host -> device for a hotstart (restart_file(READING), then postinit_2d / postinit_3d of
 * initialise.F90:331-334): the restart fields' interiors from host arrays laid out as above (FP32
 * 3D fields narrowed; halo values are kept), then postinit_2d (m2d.F90:358-400: where any U or V is
 * non-zero on a closed velocity point, U, Uinto / V, Vinto = 0 on all closed points; z = zo = -9999
 * on land; depth_update) and, for runtype >= 2, postinit_3d (m3d.F90:376-409: uu = 0 where au = 0,
 * vv = 0 where av = 0; on land tke = 0, num = nuh = 1e-15, T = S = -9999; the layer heights by
 * coordinates(hotstart)). The SAVEd switches in ipar (ufirst2d, ufirst3d) are the caller's. */
int getm_restart_read(getm_ctx *ctx, getm_bc_state *st, int runtype, const double *const *host2,
                      const double *const *host3);

/* ---- halo rows of a slab decomposition ---------------------------------------------------- */
/* The row exchange of the reference's parallel build (update_3d_halo / update_2d_halo,
 * src/futils/halo_mpi.F90:376-558) for a domain cut into slabs of rows (a 1D decomposition in j):
 * a rank sends its first and last two interior rows to its neighbours, which write them into their
 * halo rows. getm_halo_pack copies the rows j_first .. j_first+nrows-1 (reference indices of the
 * context's domain) of the levels 0 .. nk-1 of a field with elem_bytes-byte elements (4 or 8;
 * nk = 1 for a 2D field) into the packed device buffer buf, laid out [level][row][i];
 * getm_halo_unpack writes such a buffer back into those rows. The transfer between ranks is the
 * caller's (NCCL send/recv, or a device copy between two slabs of one process). */
int getm_halo_pack(getm_ctx *ctx, const void *f, int elem_bytes, int nk, int j_first, int nrows,
                   void *buf);
int getm_halo_unpack(getm_ctx *ctx, void *f, int elem_bytes, int nk, int j_first, int nrows,
                     const void *buf);

/* ---- adjoint of the tracer step ---------------------------------------------------------- */
/* No counterpart in the reference. The tracer step of getm_tracer_step (HALFSPLIT advection,
 * split schemes, adv_ver_iterations = 1, then implicit vertical diffusion) is differentiated in
 * reverse mode with the limiter branch of every face frozen at the forward pass's choice (the
 * step is then linear in the tracer, and the adjoint is its exact transpose).
 *
 * Tape of one step, written by getm_tracer_step_record: tape_codes = 5 planes of n3 bytes
 * (n3 = sk*(kmax+1); the branch of every face of the sweeps u/2, v/2, w, v/2, u/2) and tape_g =
 * the tracer after advection (one 3D field). getm_tracer_step_record advances f exactly as
 * getm_tracer_step does.
 * getm_tracer_step_adjoint turns fbar (cotangent of the step's output tracer) into the cotangent
 * of its input, in place, and ADDS the cotangent of nuh to nubar (zero it before the first step).
 * Velocities, layer heights and nuh are the step's (constant within the step). Other splits,
 * schemes or iteration counts return GETM_ERR_UNSUPPORTED. */
int getm_tracer_step_record(getm_ctx *ctx, double dt, double *f, const double *uu, const double *vv,
                            const double *ww, const double *hu, const double *hv, const double *ho,
                            const double *hn, const double *nuh, int split, int hscheme, int vscheme,
                            double AH, double cnpar, double avmol, uint8_t *tape_codes,
                            double *tape_g);
int getm_tracer_step_record_f32(getm_ctx *ctx, float dt, float *f, const float *uu, const float *vv,
                                const float *ww, const float *hu, const float *hv, const float *ho,
                                const float *hn, const float *nuh, int split, int hscheme,
                                int vscheme, float AH, float cnpar, float avmol,
                                uint8_t *tape_codes, float *tape_g);
int getm_tracer_step_adjoint(getm_ctx *ctx, double dt, double *fbar, double *nubar, const double *uu,
                             const double *vv, const double *ww, const double *hu, const double *hv,
                             const double *ho, const double *hn, const double *nuh, int split,
                             int hscheme, int vscheme, double AH, double cnpar, double avmol,
                             const uint8_t *tape_codes, const double *tape_g);
int getm_tracer_step_adjoint_f32(getm_ctx *ctx, float dt, float *fbar, float *nubar, const float *uu,
                                 const float *vv, const float *ww, const float *hu, const float *hv,
                                 const float *ho, const float *hn, const float *nuh, int split,
                                 int hscheme, int vscheme, float AH, float cnpar, float avmol,
                                 const uint8_t *tape_codes, const float *tape_g);
/* Gradient over nsteps steps with fixed velocities, heights and nuh, checkpointed: the forward
 * pass keeps f every `every` steps (f leaves holding the final tracer); the reverse pass recomputes
 * each block of steps from its checkpoint with the tape recorded and runs the adjoint steps
 * backwards. fbar: in = dJ/d(final tracer), out = dJ/d(initial tracer); nubar += dJ/d(nuh).
 * ms_forward / ms_reverse (may be NULL) receive the device time of the two passes. Device memory
 * used: ceil(nsteps/every) checkpoints + `every` tapes, plus 8 3D work arrays. */
int getm_tracer_gradient(getm_ctx *ctx, int nsteps, int every, double dt, double *f,
                         const double *uu, const double *vv, const double *ww, const double *hu,
                         const double *hv, const double *ho, const double *hn, const double *nuh,
                         int split, int hscheme, int vscheme, double AH, double cnpar, double avmol,
                         double *fbar, double *nubar, float *ms_forward, float *ms_reverse);
int getm_tracer_gradient_f32(getm_ctx *ctx, int nsteps, int every, float dt, float *f,
                             const float *uu, const float *vv, const float *ww, const float *hu,
                             const float *hv, const float *ho, const float *hn, const float *nuh,
                             int split, int hscheme, int vscheme, float AH, float cnpar,
                             float avmol, float *fbar, float *nubar, float *ms_forward,
                             float *ms_reverse);

/* ---- diagnostics ----------------------------------------------------------------------- */
/* Compensated (Neumaier) FP64 sum of f*h/ard1 over wet interior cells (az>=1, k=1..kmax):
 * the global tracer content. Deterministic (fixed reduction order). Result written to the HOST
 * double *out (the call synchronises the stream). No counterpart routine in the reference; it
 * backs the tracer-conservation checks. */
int getm_tracer_content(getm_ctx *ctx, const double *f, const double *h, const int32_t *az,
                        double *out);
int getm_tracer_content_f32(getm_ctx *ctx, const float *f, const float *h, const int32_t *az,
                            double *out);
/* check_3d_fields (src/futils/check_3d_fields.F90:8-59): counts cells of the interior with az>0
 * and k>=kmin (kmin = 0, the sigma-coordinate value) whose value is below minval or above
 * maxval (a NaN compares false both ways and is not counted, as in the reference). Count written
 * to the HOST int64 *status. */
int getm_check_3d_fields(getm_ctx *ctx, const double *f, const int32_t *az, double minval,
                         double maxval, int64_t *status);

/* ---- context-free, allocation-free variant ------------------------------------------- */
/* getm_tracer_vdiff without a context and without any device allocation. No counterpart in the
 * reference: it exists for callers that cannot allocate device memory while they step (they keep
 * no context, their device memory is fully committed, or they cannot afford the device-wide wait
 * of cudaFree). Same kernel, arguments and results as getm_tracer_vdiff (FP64).
 *
 * Scratch: one array with static storage in the library, sized for domains whose padded 3D index
 * space sk*(kmax+1) holds at most GETM_VDIFF_NOALLOC_MAX_CELLS elements (two FP64 coefficients
 * per element: 64 MiB of device memory, which the CUDA runtime reserves when it loads the module
 * holding it: at start-up, or at the first call where modules load lazily). A larger domain
 * returns GETM_ERR_TOO_LARGE and nothing runs. Nothing in the scratch has to start at zero.
 * Device and stream: the caller makes the device that owns the arrays current and passes a
 * stream of that device (NULL = legacy default stream). The first call on each device looks up
 * the scratch address there (a one-time set-up, no allocation); make that first call before any
 * stream capture begins. The address is kept per device together with the CUDA context it was
 * found in: a call in another context of the device (e.g. after cudaDeviceReset ended the primary
 * context) repeats that set-up.
 * Concurrency: all calls on one device share the one scratch array. Calls whose work overlaps in
 * time (on different streams, or from several host threads without ordering) race on it and give
 * wrong results; calls on one stream are ordered and safe. */
#define GETM_VDIFF_NOALLOC_MAX_CELLS 4194304LL
int getm_tracer_vdiff_noalloc(const getm_domain *dom, void *stream, double dt, double cnpar,
                              double avmol, double *S, const double *hn, const double *nuh,
                              const int32_t *az, const double *src);

#ifdef __cplusplus
}
#endif
#endif /* GETM_B200_H */
