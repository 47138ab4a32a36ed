// launch.h -- host-side launchers of the templated kernels (instantiated per precision in
// kernels_f64.cu / kernels_f32.cu). Each returns a cudaError_t as int (0 = success).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace gb {

struct Dev;

// Process-wide switch of the vectorised horizontal sweeps (getm_set_vector_sweeps; on by default).
bool vector_sweeps_enabled();
bool fused_micro_enabled();
// Process-wide switch of the FP32 working copies of the mixed step's micro steps
// (getm_set_fp32_micro_steps; on by default).
bool fp32_micro_steps_enabled();

constexpr int RED_BLOCKS = 1184;  // 8 x 148 SMs
constexpr int RED_THREADS = 256;

// lo (FP32 only; FP64 ignores it): compensated storage of a tracer, the carried rounding error of
// every cell in FP16, scaled to half an ulp of the cell's value, read and written by the updates
// (fv_update_lo); null for plain FP32 storage.
// Horizontal sweep over nk levels starting at the given level pointers. DIR 0 = u, 1 = v.
// code != nullptr also writes the limiter branch of every face (one byte per face, stored at the
// face's left / lower cell, same level pointer origin as f).
// f_b != nullptr sweeps a second tracer (f_b, fi_src_b -> fi_dst_b) with the same transports,
// heights and masks (then code and adv must be nullptr).
// adv_init: adv (nk levels from the level pointer) is not cleared by the caller; the sweep starts
// the sum, so that every cell of those levels ends as 0 + its flux divergence.
// du2d / di2d: DU / Di_src are 2D arrays (the first cell of the plane, not a level pointer) whose
// values hold at every level of the column.
template <class R, int DIR>
int run_sweep_h(const Dev& d, cudaStream_t s, int nk, R dt, R splitfac, int scheme, R AH, const R* f,
                const R* fi_src, R* fi_dst, const R* Di_src, R* Di_dst, R* adv, const R* U, const R* DU,
                const uint8_t* mflux, const uint8_t* mupd, uint8_t* code = nullptr, const R* f_b = nullptr,
                const R* fi_src_b = nullptr, R* fi_dst_b = nullptr, __half* lo = nullptr,
                __half* lo_b = nullptr, bool adv_init = false, bool du2d = false, bool di2d = false);

// Vertical sweep on full 3D fields (level-0 pointers); code as above (face k stored at level k;
// only without sub-iterations).
template <class R>
int run_sweep_w(const Dev& d, cudaStream_t s, R dt, R splitfac, int scheme, int kshift, int itersmax,
                const R* f, const R* fi_src, R* fi_dst, R* hi, R* adv, const R* ww, const int32_t* az,
                unsigned long long* warn, uint8_t* code = nullptr, __half* lo = nullptr);

// Depth-averaged momentum advection of one micro step with HALFSPLIT (adv2d_fused.cuh): UEx
// (dir 0, U-grid masks) or VEx (dir 1, V-grid masks) from U, V, DU, DV in one launch, arithmetic
// in T; Ex is FP64.
template <class T>
int run_uvadv2d_fused(const Dev& d, cudaStream_t s, int dir, T dt, int scheme, const double* U, const double* V,
                      const double* DU, const double* DV, const uint8_t* mflux_u, const uint8_t* mflux_v,
                      const uint8_t* mupd_u, const uint8_t* mupd_v, double* Ex);
// The bottom friction of the micro step (bottom_friction.F90:48-150), formed by the momentum
// advection kernel of the same component from the velocities it stages anyway: DIR 0 the U points
// (ru, ruu; zub for runtype 1), DIR 1 the V points (rv, rvv; zvb). FP32 arithmetic, the operations
// of k_bottom_friction_f32t (bc.cu) in the same order, so the same values. r == nullptr: off.
struct Bf2Args {
  const uint8_t* mask;  // au (DIR 0) / av (DIR 1), uint8 copies
  const uint8_t* au;    // DIR 1: the U points' mask for the velocity outside the interior
  float* zb;            // zub / zvb (FP32 working copies)
  const float* zb0;     // zub0 / zvb0
  float* r;             // ru / rv (FP32 working copies)
  float* rr;            // ruu / rvv
  float kappa, avmmol, min_depth;
  int runtype;
};
// both components in one launch (mu / mv: the U and the V grid's flux-u, flux-v, update-u,
// update-v masks; bfu / bfv: their bottom friction, may be null)
int run_uvadv2d_both_f32(const Dev& d, cudaStream_t s, float dt, int scheme, const float* U, const float* V,
                         const float* DU, const float* DV, const uint8_t* const* mu, const uint8_t* const* mv,
                         float* UEx, float* VEx, const Bf2Args* bfu, const Bf2Args* bfv);
// bf (may be null): also form the bottom friction of the micro step for this component's points
int run_uvadv2d_fused_f32(const Dev& d, cudaStream_t s, int dir, float dt, int scheme, const float* U,
                          const float* V, const float* DU, const float* DV, const uint8_t* mflux_u,
                          const uint8_t* mflux_v, const uint8_t* mupd_u, const uint8_t* mupd_v, float* Ex,
                          const Bf2Args* bf = nullptr);

// Vertical sweep of two tracers in place (H_TAG, no sub-iterations), heights updated once.
template <class R>
int run_sweep_w2(const Dev& d, cudaStream_t s, R dt, R splitfac, int scheme, R* fa, R* fb, R* hi, const R* ww,
                 const int32_t* az, __half* lo_a = nullptr, __half* lo_b = nullptr);

// ---- adjoint of the tracer step (adjoint.cuh) ----
// Layer heights before sweeps 2..5 of the HALFSPLIT sequence u/2 v/2 w v/2 u/2, from ho (levels
// 1..kmax): H1 after u/2, H2 after v/2, H3 after w, H4 after v/2.
template <class R>
int run_adj_heights(const Dev& d, cudaStream_t s, R dt, int sub, bool has_w, const R* ho, const R* uu,
                    const R* vv, const R* ww, const uint8_t* mupd_u, const uint8_t* mupd_v,
                    const int32_t* az, R* H1, R* H2, R* H3, R* H4);
// Adjoint of one horizontal sweep over nk levels (level pointers): gbar (cotangent of the sweep's
// output) -> fbar (cotangent of its input). Dio = heights before the sweep. copy0: also pass the
// level below the pointers' origin (level 0 of the 3D field) through.
template <class R, int DIR>
int run_adj_sweep_h(const Dev& d, cudaStream_t s, int nk, R dt, R splitfac, int scheme, R AH, const R* gbar,
                    R* fbar, const R* Dio, const R* U, const R* DU, const uint8_t* mflux, const uint8_t* mupd,
                    const uint8_t* code, bool copy0 = false);
// Adjoint of the vertical sweep (full 3D fields); hi = heights before the sweep.
template <class R>
int run_adj_sweep_w(const Dev& d, cudaStream_t s, R dt, R splitfac, int scheme, int kshift, const R* gbar,
                    R* fbar, const R* hi, const R* ww, const int32_t* az, const uint8_t* code);
// Adjoint of the implicit vertical diffusion: fbar (cotangent of the new tracer) -> gbar
// (cotangent of the old one); nubar += cotangent of nuh. g = old tracer, Sn = new tracer.
template <class R>
int run_adj_vdiff(const Dev& d, cudaStream_t s, R dt, R cnpar, R avmol, const R* fbar, R* gbar, R* nubar,
                  const R* g, const R* Sn, const R* hn, const R* nuh, const int32_t* az, R* rus, R* qus);

template <class R>
int run_finalise(const Dev& d, cudaStream_t s, R dt, R* f, const R* ho, const R* adv, const R* hi,
                 const uint8_t* mfin);

// rus/qus: two scratch 3D arrays (Thomas coefficients). The old tracer is read from Sin (default:
// S itself) and the new one written to S and, when given, to S2 as well; only the solved columns
// (interior, az == 1) are written.
template <class R>
int run_vdiff(const Dev& d, cudaStream_t s, R dt, R cnpar, R avmol, R* S, const R* hn, const R* nuh,
              const int32_t* az, const R* src, R* rus, R* qus, const R* Sin = nullptr, R* S2 = nullptr,
              __half* lo = nullptr);

// Two tracers (temperature a with its sources src_a, salinity b) diffused in one launch over the
// same heights and diffusivity; each with its own molecular diffusivity, scratch pair and
// compensated storage; each tracer's expressions are run_vdiff's. hn2d: hn is a 2D array of column
// heights (every level of a column has that height). qus_a == qus_b == nullptr: each tracer's
// elimination coefficients go to its rus array as interleaved (ru, qu) pairs (2 * sk * (kmax+1)
// elements).
template <class R>
int run_vdiff2(const Dev& d, cudaStream_t s, R dt, R cnpar, const R* hn, const R* nuh, const int32_t* az,
               R* Sa, R avmol_a, const R* src_a, R* rus_a, R* qus_a, __half* lo_a, R* Sb, R avmol_b, R* rus_b,
               R* qus_b, __half* lo_b, bool hn2d = false);

template <class R>
int run_tridiag(cudaStream_t s, int ncol, int kmax, int fi, int lt, const R* au, const R* bu, const R* cu,
                const R* du, R* value);

// Two-stage deterministic content reduction; partial must hold 2*RED_BLOCKS doubles.
template <class R>
int run_content(const Dev& d, cudaStream_t s, const R* f, const R* h, const int32_t* az, double* partial,
                double* out);

template <class R>
int run_check_range(const Dev& d, cudaStream_t s, const R* f, const int32_t* az, R lo, R hi,
                    unsigned long long* count);

int run_build_masks(const Dev& d, cudaStream_t s, const int32_t* az, const int32_t* au, const int32_t* av,
                    const int32_t* ax, uint8_t* planes);

// 3D kernels of the macro step (bc_kernels.cuh); scr = the scratch arrays (NB3, FP32 NB3F)
enum {
  BC3_BF3D = 0, BC3_ZZ, BC3_IP, BC3_UUMOM, BC3_VVMOM, BC3_SIGMA, BC3_WW, BC3_UVADV_PREP_U, BC3_UVADV_PREP_V,
  BC3_STRESSES, BC3_EQSTATE, BC3_SLOW_TERMS, BC3_UVADV_PREP_UV, BC3_ZZ_LIN, BC3_IP_LIN,
  BC3_IP_SW, BC3_IP_CF, BC3_SM_COLS, BC3_IP_SM, BC3_EQSTATE_UNESCO, BC3_EQSTATE_JACKETT, BC3_GOTM_PARABOLIC,
  BC3_SW_RADIATION, BC3_TEMP_SOURCE, BC3_IP_ZI, BC3_IP_SVK
};
// sealevel_nan_check sweep of the interior elevations (bc.cu, k_nan_sweep): cnt[0] +=
// findings, cnt[1] = max(cnt[1], last loop-order index + 1); skipped while cnt[2] != 0
int run_nan_sweep(const Dev& d, cudaStream_t s, const double* z, unsigned long long* cnt);
template <class R3>
struct Bc3;
// colh (may be null): the column-height planes of k_col_heights, which the FP32 momentum-advection
// set-up (BC3_UVADV_PREP_UV) then reads in place of the 3D heights
template <class R3>
int run_bc3(int which, const Dev& d, cudaStream_t st, const Bc3<R3>& s, R3* const* scr, const R3* colh = nullptr);
// the column heights of the macro step after sigma_coordinates (k_col_heights): NCOLH 2D planes
// (COL_* in bc_common.cuh)
template <class R3>
int run_col_heights(const Dev& d, cudaStream_t st, const Bc3<R3>& s, R3* out);

}  // namespace gb
