// ctx.cu -- context, mask set-up and the C-ABI entry points (include/getm_b200.h).
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"
#include <algorithm>

#include "launch.h"

#include "ctx_internal.h"

namespace gb {

std::atomic<int> g_vector_sweeps{1};
bool vector_sweeps_enabled() { return g_vector_sweeps.load(std::memory_order_relaxed) != 0; }

std::atomic<int> g_fused_micro{1};
bool fused_micro_enabled() { return g_fused_micro.load(std::memory_order_relaxed) != 0; }
std::atomic<int> g_fp32_micro{1};
bool fp32_micro_steps_enabled() { return g_fp32_micro.load(std::memory_order_relaxed) != 0; }



// init_advection (advection.F90:263-318) from az/au/av/ax.
__global__ void k_build_masks(Dev d, const int32_t* __restrict__ az, const int32_t* __restrict__ au,
                              const int32_t* __restrict__ av, const int32_t* __restrict__ ax, uint8_t* planes) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  const int ni = d.ni(), nj = d.nj();
  if (ii >= ni || jj >= nj) return;
  const long long c = (long long)ii + (long long)jj * d.sj;
  const long long n = d.sj * (long long)nj;
  const bool last_i = (ii == ni - 1), last_j = (jj == nj - 1);
  planes[P_UPDATEH * n + c] = az[c] == 1;
  planes[P_UFLUX * n + c] = (au[c] == 1 || au[c] == 2) && !last_i;
  planes[P_VFLUX * n + c] = (av[c] == 1 || av[c] == 2) && !last_j;
  planes[P_XFLUX * n + c] = ax[c] == 1 && !last_i && !last_j;
  planes[P_UUPDATEU * n + c] = au[c] == 1;
  planes[P_VUPDATEV * n + c] = av[c] == 1;
  // U grid u-flux = mask_updateH(i+1,j); V grid v-flux = mask_updateH(i,j+1)
  planes[P_UFLUX_U * n + c] = !last_i && az[c + 1] == 1;
  planes[P_VFLUX_V * n + c] = !last_j && az[c + d.sj] == 1;
}

int run_build_masks(const Dev& d, cudaStream_t s, const int32_t* az, const int32_t* au, const int32_t* av,
                    const int32_t* ax, uint8_t* planes) {
  dim3 blk(64, 4, 1);
  dim3 grd((d.ni() + 63) / 64, (d.nj() + 3) / 4, 1);
  k_build_masks<<<grd, blk, 0, s>>>(d, az, au, av, ax, planes);
  return (int)cudaGetLastError();
}

}  // namespace gb

using namespace gb;

// ---------------------------------------------------------------------------------------------
// do_advection_3d (advection_3d.F90:279-566) on device pointers (level-0 origin).
template <class R>
int do_adv3d(getm_ctx* ctx, R dt, R* f, const R* uu, const R* vv, const R* ww, const R* hu,
                    const R* hv, const R* ho, const R* hn, int split, int hs, int vs, R AH, int tag, R* hires,
                    R* advres, int iters, bool field_out, __half* lo, unsigned h2d) {
  (void)hn;
  if (!ctx) return GETM_ERR_ARG;
  if (!ctx->adv_ready) return fail(ctx, GETM_ERR_STATE, "getm_init_advection has not been called");
  getm_adv_grid g;
  if (!grid_for_tag(ctx, tag, &g)) return fail(ctx, GETM_ERR_ARG, "do_advection_3d: tag is invalid");
  if (!f || !ho) return fail(ctx, GETM_ERR_ARG, "do_advection_3d: null field");
  if (hs != NOADV && !is_split_scheme(hs)) {
    if (hs == UPSTREAM_2DH || hs == 7 || hs == 8 || hs == 9)
      return fail(ctx, GETM_ERR_UNSUPPORTED, "do_advection_3d: 2DH schemes are not provided");
    return fail(ctx, GETM_ERR_ARG, "do_advection_3d: hscheme is invalid");
  }
  if (vs != NOADV && !is_split_scheme(vs)) return fail(ctx, GETM_ERR_ARG, "do_advection_3d: vscheme is invalid");
  if (iters < 1) iters = 1;
  if (iters > 1 && ctx->dom.kmax > 128)
    return fail(ctx, GETM_ERR_UNSUPPORTED, "adv_ver_iterations > 1 needs kmax <= 128");
  const Dev& d = ctx->dev;
  cudaStream_t s = ctx->stream;
  const int kmax = d.kmax;
  const long long sk = d.sk;
  const long long n3 = n3d(d);
  const size_t bytes3 = (size_t)n3 * sizeof(R);
  const int kshift = (tag == GETM_W_TAG) ? 1 : 0;
  int rc = ensure_scratch(ctx, bytes3);
  if (rc) return rc;
  R* S = (R*)ctx->scr[0];
  R* H = hires ? hires : (R*)ctx->scr[1];
  const bool needs_adv = (hs != NOADV && vs != NOADV && (split == GETM_NOSPLIT || split == GETM_HVSPLIT)) ||
                         (hs != NOADV && vs == NOADV && split == GETM_NOSPLIT);
  R* A = advres ? advres : (needs_adv ? (R*)ctx->scr[2] : nullptr);
  // p_adv = 0 (advection_3d.F90:296): FULLSPLIT and HALFSPLIT clear level 0 and let their first u
  // sweep start the sum on levels 1..kmax; the other sequences clear the whole array
  const bool split_first_u = hs != NOADV && vs != NOADV && kmax >= 1 &&
                             (split == GETM_FULLSPLIT || split == GETM_HALFSPLIT);
  // h2d (callers inside the step): bit 0 hu, bit 1 hv, bit 2 ho are 2D arrays of column values
  // (the layer heights of equidistant sigma coordinates); only the FULLSPLIT and HALFSPLIT sweeps
  // take them
  if (h2d && (!split_first_u || hires)) return fail(ctx, GETM_ERR_STATE, "do_advection_3d: 2D heights need a split");
  if (A) GB_TRY(cudaMemsetAsync(A, 0, split_first_u ? (size_t)sk * sizeof(R) : bytes3, s), "memset adv");
  auto L = [&](auto* p, int k) { return p + (long long)k * sk; };
  const R half = R(0.5), one = R(1);
  unsigned long long* warn = ctx->cnt;

  if (hs == NOADV || vs == NOADV || kmax < 1) {
    // p_hi = ho over the whole array
    GB_TIMED(GETM_TIM_COPY, cudaMemcpyAsync(H, ho, bytes3, cudaMemcpyDeviceToDevice, s), "copy ho");
  } else if (hires || kshift == 1) {
    // level 0 of p_hi (the sweeps below write levels 1..kmax from ho); read only by the W-grid
    // vertical sweep (face 0) and returned in hires
    GB_TRY(cudaMemcpyAsync(H, ho, (size_t)sk * sizeof(R), cudaMemcpyDeviceToDevice, s), "copy ho(0)");
  }
  if (hs == NOADV && vs == NOADV) return GETM_OK;
  if (hs == NOADV) {
    if (kmax > 1) GB_TIMED(GETM_TIM_ADV_W, run_sweep_w<R>(d, s, dt, one, vs, kshift, iters, f, f, f, H, A, ww, g.az, warn), "w");
    return GETM_OK;
  }
  const int nk = kmax;
  if (vs == NOADV) {
    // per-level 2D do_advection (advection.F90:469-666) on levels 1..kmax
    if (split == GETM_NOSPLIT) {
      GB_TIMED(GETM_TIM_COPY, cudaMemcpyAsync(S, f, bytes3, cudaMemcpyDeviceToDevice, s), "copy f");
      GB_TIMED(GETM_TIM_ADV_U, (run_sweep_h<R, 0>(d, s, nk, dt, one, hs, AH, L(f, 1), L(S, 1), L(S, 1), L(H, 1), L(H, 1), L(A, 1),
                                L(uu, 1), L(hu, 1), g.mask_uflux, g.mask_uupdate)), "u");
      GB_TIMED(GETM_TIM_ADV_V, (run_sweep_h<R, 1>(d, s, nk, dt, one, hs, AH, L(f, 1), L(S, 1), L(S, 1), L(H, 1), L(H, 1), L(A, 1),
                                L(vv, 1), L(hv, 1), g.mask_vflux, g.mask_vupdate)), "v");
      GB_TIMED(GETM_TIM_ADV_FINALISE, run_finalise<R>(d, s, dt, f, ho, A, H, g.mask_finalise), "finalise");
    } else if (split == GETM_FULLSPLIT) {
      GB_TIMED(GETM_TIM_ADV_U, (run_sweep_h<R, 0>(d, s, nk, dt, one, hs, AH, L(f, 1), L(f, 1), L(S, 1), L(ho, 1), L(H, 1),
                                A ? L(A, 1) : nullptr, L(uu, 1), L(hu, 1), g.mask_uflux, g.mask_uupdate)), "u");
      GB_TIMED(GETM_TIM_ADV_V, (run_sweep_h<R, 1>(d, s, nk, dt, one, hs, AH, L(S, 1), L(S, 1), L(f, 1), L(H, 1), L(H, 1),
                                A ? L(A, 1) : nullptr, L(vv, 1), L(hv, 1), g.mask_vflux, g.mask_vupdate)), "v");
    } else if (split == GETM_HALFSPLIT) {
      GB_TIMED(GETM_TIM_COPY, cudaMemcpyAsync(S, f, bytes3, cudaMemcpyDeviceToDevice, s), "copy f");
      GB_TIMED(GETM_TIM_ADV_U, (run_sweep_h<R, 0>(d, s, nk, dt, half, hs, AH, L(S, 1), L(S, 1), L(f, 1), L(ho, 1), L(H, 1),
                                A ? L(A, 1) : nullptr, L(uu, 1), L(hu, 1), g.mask_uflux, g.mask_uupdate)), "u");
      GB_TIMED(GETM_TIM_ADV_V, (run_sweep_h<R, 1>(d, s, nk, dt, one, hs, AH, L(f, 1), L(f, 1), L(S, 1), L(H, 1), L(H, 1),
                                A ? L(A, 1) : nullptr, L(vv, 1), L(hv, 1), g.mask_vflux, g.mask_vupdate)), "v");
      GB_TIMED(GETM_TIM_ADV_U, (run_sweep_h<R, 0>(d, s, nk, dt, half, hs, AH, L(S, 1), L(S, 1), L(f, 1), L(H, 1), L(H, 1),
                                A ? L(A, 1) : nullptr, L(uu, 1), L(hu, 1), g.mask_uflux, g.mask_uupdate)), "u");
    } else {
      return fail(ctx, GETM_ERR_ARG, "do_advection: split is invalid");
    }
    return GETM_OK;
  }
  R* Al = A ? L(A, 1) : nullptr;
  // compensated storage of the tracer (FP32; the FULLSPLIT and HALFSPLIT sequences, whose updates
  // are all increments)
  __half* lw = (lo && field_out) ? lo : nullptr;
  __half* ll = lw ? L(lw, 1) : nullptr;
  const bool hu2 = h2d & 1u, hv2 = h2d & 2u, ho2 = h2d & 4u;
  const R* HUl = hu2 ? hu : L(hu, 1);
  const R* HVl = hv2 ? hv : L(hv, 1);
  const R* HOl = ho2 ? ho : L(ho, 1);
  switch (split) {
    case GETM_NOSPLIT:
      GB_TIMED(GETM_TIM_COPY, cudaMemcpyAsync(S, f, bytes3, cudaMemcpyDeviceToDevice, s), "copy f");
      GB_TIMED(GETM_TIM_ADV_U, (run_sweep_h<R, 0>(d, s, nk, dt, one, hs, AH, L(f, 1), L(S, 1), L(S, 1), L(ho, 1), L(H, 1), Al,
                                L(uu, 1), L(hu, 1), g.mask_uflux, g.mask_uupdate)), "u");
      GB_TIMED(GETM_TIM_ADV_V, (run_sweep_h<R, 1>(d, s, nk, dt, one, hs, AH, L(f, 1), L(S, 1), L(S, 1), L(H, 1), L(H, 1), Al,
                                L(vv, 1), L(hv, 1), g.mask_vflux, g.mask_vupdate)), "v");
      if (kmax > 1) GB_TIMED(GETM_TIM_ADV_W, run_sweep_w<R>(d, s, dt, one, vs, kshift, 1, f, S, S, H, A, ww, g.az, warn), "w");
      GB_TIMED(GETM_TIM_ADV_FINALISE, run_finalise<R>(d, s, dt, f, ho, A, H, g.mask_finalise), "finalise");
      break;
    case GETM_FULLSPLIT:
      GB_TIMED(GETM_TIM_ADV_U, (run_sweep_h<R, 0>(d, s, nk, dt, one, hs, AH, L(f, 1), L(f, 1), L(S, 1), HOl, L(H, 1), Al,
                                L(uu, 1), HUl, g.mask_uflux, g.mask_uupdate, nullptr, nullptr, nullptr, nullptr, ll,
                                nullptr, true, hu2, ho2)), "u");
      GB_TIMED(GETM_TIM_ADV_V, (run_sweep_h<R, 1>(d, s, nk, dt, one, hs, AH, L(S, 1), L(S, 1), L(f, 1), L(H, 1), L(H, 1), Al,
                                L(vv, 1), HVl, g.mask_vflux, g.mask_vupdate, nullptr, nullptr, nullptr, nullptr, ll,
                                nullptr, false, hv2)), "v");
      if (kmax > 1) GB_TIMED(GETM_TIM_ADV_W, run_sweep_w<R>(d, s, dt, one, vs, kshift, iters, f, f, f, H, A, ww, g.az, warn, nullptr, lw), "w");
      break;
    case GETM_HALFSPLIT:
      GB_TIMED(GETM_TIM_ADV_U, (run_sweep_h<R, 0>(d, s, nk, dt, half, hs, AH, L(f, 1), L(f, 1), L(S, 1), HOl, L(H, 1), Al,
                                L(uu, 1), HUl, g.mask_uflux, g.mask_uupdate, nullptr, nullptr, nullptr, nullptr, ll,
                                nullptr, true, hu2, ho2)), "u1");
      GB_TIMED(GETM_TIM_ADV_V, (run_sweep_h<R, 1>(d, s, nk, dt, half, hs, AH, L(S, 1), L(S, 1), L(f, 1), L(H, 1), L(H, 1), Al,
                                L(vv, 1), HVl, g.mask_vflux, g.mask_vupdate, nullptr, nullptr, nullptr, nullptr, ll,
                                nullptr, false, hv2)), "v1");
      if (kmax > 1) GB_TIMED(GETM_TIM_ADV_W, run_sweep_w<R>(d, s, dt, one, vs, kshift, iters, f, f, f, H, A, ww, g.az, warn, nullptr, lw), "w");
      GB_TIMED(GETM_TIM_ADV_V, (run_sweep_h<R, 1>(d, s, nk, dt, half, hs, AH, L(f, 1), L(f, 1), L(S, 1), L(H, 1), L(H, 1), Al,
                                L(vv, 1), HVl, g.mask_vflux, g.mask_vupdate, nullptr, nullptr, nullptr, nullptr, ll,
                                nullptr, false, hv2)), "v2");
      // the last sweep writes the field and heights only when the caller keeps them
      GB_TIMED(GETM_TIM_ADV_U, (run_sweep_h<R, 0>(d, s, nk, dt, half, hs, AH, L(S, 1), L(S, 1),
                                field_out ? L(f, 1) : nullptr, L(H, 1), (field_out || hires) ? L(H, 1) : nullptr,
                                Al, L(uu, 1), HUl, g.mask_uflux, g.mask_uupdate, nullptr, nullptr, nullptr, nullptr, ll,
                                nullptr, false, hu2)), "u2");
      break;
    case GETM_HVSPLIT:
      GB_TIMED(GETM_TIM_COPY, cudaMemcpyAsync(S, f, bytes3, cudaMemcpyDeviceToDevice, s), "copy f");
      GB_TIMED(GETM_TIM_ADV_U, (run_sweep_h<R, 0>(d, s, nk, dt, one, hs, AH, L(f, 1), L(S, 1), L(S, 1), L(ho, 1), L(H, 1), Al,
                                L(uu, 1), L(hu, 1), g.mask_uflux, g.mask_uupdate)), "u");
      GB_TIMED(GETM_TIM_ADV_V, (run_sweep_h<R, 1>(d, s, nk, dt, one, hs, AH, L(f, 1), L(S, 1), L(S, 1), L(H, 1), L(H, 1), Al,
                                L(vv, 1), L(hv, 1), g.mask_vflux, g.mask_vupdate)), "v");
      GB_TIMED(GETM_TIM_ADV_FINALISE, run_finalise<R>(d, s, dt, f, ho, A, H, g.mask_finalise), "finalise");
      if (kmax > 1) GB_TIMED(GETM_TIM_ADV_W, run_sweep_w<R>(d, s, dt, one, vs, kshift, iters, f, f, f, H, A, ww, g.az, warn), "w");
      break;
    default:
      return fail(ctx, GETM_ERR_ARG, "do_advection_3d: split is invalid");
  }
  return GETM_OK;
}

// Two tracers (temperature and salinity) advected together with HALFSPLIT on the H grid: the
// same sweeps as do_adv3d's HALFSPLIT branch for each field, with the heights hi evolved once.
template <class R>
int do_adv3d_pair(getm_ctx* ctx, R dt, R* fa, R* fb, const R* uu, const R* vv, const R* ww, const R* hu,
                  const R* hv, const R* ho, int hs, int vs, R AH, __half* lo_a, __half* lo_b, unsigned h2d) {
  getm_adv_grid g;
  grid_for_tag(ctx, GETM_H_TAG, &g);
  const Dev& d = ctx->dev;
  cudaStream_t s = ctx->stream;
  const int kmax = d.kmax;
  const long long sk = d.sk;
  int rc = ensure_scratch(ctx, (size_t)n3d(d) * sizeof(R));
  if (rc) return rc;
  R* Sa = (R*)ctx->scr[0];
  R* H = (R*)ctx->scr[1];
  R* Sb = (R*)ctx->scr[2];
  auto L = [&](auto* p, int k) { return p ? p + (long long)k * sk : p; };
  const R half = R(0.5), one = R(1);
  const int nk = kmax;
  __half* la = L(lo_a, 1);
  __half* lb = L(lo_b, 1);
  // h2d as in do_adv3d: hu, hv, ho as 2D arrays of column values
  const bool hu2 = h2d & 1u, hv2 = h2d & 2u, ho2 = h2d & 4u;
  const R* HUl = hu2 ? hu : L(hu, 1);
  const R* HVl = hv2 ? hv : L(hv, 1);
  const R* HOl = ho2 ? ho : L(ho, 1);
  GB_TIMED(GETM_TIM_ADV_U, (run_sweep_h<R, 0>(d, s, nk, dt, half, hs, AH, L(fa, 1), L(fa, 1), L(Sa, 1), HOl,
                            L(H, 1), nullptr, L(uu, 1), HUl, g.mask_uflux, g.mask_uupdate, nullptr, L(fb, 1),
                            L(fb, 1), L(Sb, 1), la, lb, false, hu2, ho2)), "u1");
  GB_TIMED(GETM_TIM_ADV_V, (run_sweep_h<R, 1>(d, s, nk, dt, half, hs, AH, L(Sa, 1), L(Sa, 1), L(fa, 1), L(H, 1),
                            L(H, 1), nullptr, L(vv, 1), HVl, g.mask_vflux, g.mask_vupdate, nullptr, L(Sb, 1),
                            L(Sb, 1), L(fb, 1), la, lb, false, hv2)), "v1");
  if (kmax > 1 && vs != NOADV)
    GB_TIMED(GETM_TIM_ADV_W, run_sweep_w2<R>(d, s, dt, one, vs, fa, fb, H, ww, g.az, lo_a, lo_b), "w");
  GB_TIMED(GETM_TIM_ADV_V, (run_sweep_h<R, 1>(d, s, nk, dt, half, hs, AH, L(fa, 1), L(fa, 1), L(Sa, 1), L(H, 1),
                            L(H, 1), nullptr, L(vv, 1), HVl, g.mask_vflux, g.mask_vupdate, nullptr, L(fb, 1),
                            L(fb, 1), L(Sb, 1), la, lb, false, hv2)), "v2");
  GB_TIMED(GETM_TIM_ADV_U, (run_sweep_h<R, 0>(d, s, nk, dt, half, hs, AH, L(Sa, 1), L(Sa, 1), L(fa, 1), L(H, 1),
                            L(H, 1), nullptr, L(uu, 1), HUl, g.mask_uflux, g.mask_uupdate, nullptr, L(Sb, 1),
                            L(Sb, 1), L(fb, 1), la, lb, false, hu2)), "u2");
  return GETM_OK;
}
template int do_adv3d_pair<double>(getm_ctx*, double, double*, double*, const double*, const double*, const double*,
                                   const double*, const double*, const double*, int, int, double, __half*, __half*, unsigned);
template int do_adv3d_pair<float>(getm_ctx*, float, float*, float*, const float*, const float*, const float*,
                                  const float*, const float*, const float*, int, int, float, __half*, __half*, unsigned);

template int do_adv3d<double>(getm_ctx*, double, double*, const double*, const double*, const double*,
                               const double*, const double*, const double*, const double*, int, int, int, double,
                               int, double*, double*, int, bool, __half*, unsigned);
template int do_adv3d<float>(getm_ctx*, float, float*, const float*, const float*, const float*, const float*,
                             const float*, const float*, const float*, int, int, int, float, int, float*, float*,
                             int, bool, __half*, unsigned);

template <class R>
static int sweep_h_api(getm_ctx* ctx, int dir, int nk, R dt, const R* f, R* fi, R* Di, R* adv, const R* U,
                       const R* DU, R splitfac, int scheme, R AH, const uint8_t* mflux, const uint8_t* mupd) {
  if (!ctx || !f || !fi || !Di || !U || !DU || !mflux || !mupd || nk < 1)
    return fail(ctx, GETM_ERR_ARG, "adv_split: bad argument");
  if (!is_split_scheme(scheme)) return fail(ctx, GETM_ERR_ARG, "adv_split: scheme is invalid");
  const Dev& d = ctx->dev;
  const R* src = f;
  if (f == fi) {
    // in-place call: fluxes must see the pre-sweep field (the reference's separate flux phase)
    const size_t bytes = (size_t)(d.sk * (long long)(nk - 1) + n2d(d)) * sizeof(R);
    int rc = ensure_scratch(ctx, (size_t)n3d(d) * sizeof(R) > bytes ? (size_t)n3d(d) * sizeof(R) : bytes);
    if (rc) return rc;
    GB_TRY(cudaMemcpyAsync(ctx->scr[0], f, bytes, cudaMemcpyDeviceToDevice, ctx->stream), "copy f");
    src = (const R*)ctx->scr[0];
  }
  int e = dir == 0 ? run_sweep_h<R, 0>(d, ctx->stream, nk, dt, splitfac, scheme, AH, src, fi, fi, Di, Di, adv, U,
                                       DU, mflux, mupd)
                   : run_sweep_h<R, 1>(d, ctx->stream, nk, dt, splitfac, scheme, AH, src, fi, fi, Di, Di, adv, U,
                                       DU, mflux, mupd);
  return cuda_fail(ctx, e, "adv_split");
}

template <class R>
static int vdiff_api(getm_ctx* ctx, R dt, R cnpar, R avmol, R* S, const R* hn, const R* nuh, const int32_t* az,
                     const R* src) {
  if (!ctx || !S || !hn || !nuh || !az) return fail(ctx, GETM_ERR_ARG, "tracer_vdiff: bad argument");
  int rc = ensure_scratch(ctx, (size_t)n3d(ctx->dev) * sizeof(R));
  if (rc) return rc;
  GB_TIMED(GETM_TIM_VDIFF,
           run_vdiff<R>(ctx->dev, ctx->stream, dt, cnpar, avmol, S, hn, nuh, az, src, (R*)ctx->scr[0], (R*)ctx->scr[1]),
           "tracer_vdiff");
  return GETM_OK;
}

template <class R>
int tracer_step_impl(getm_ctx* ctx, R dt, R* f, const R* uu, const R* vv, const R* ww, const R* hu, const R* hv,
                     const R* ho, const R* hn, const R* nuh, int split, int hs, int vs, R AH, R cnpar, R avmol,
                     int iters) {
  int rc = do_adv3d<R>(ctx, dt, f, uu, vv, ww, hu, hv, ho, hn, split, hs, vs, AH, GETM_H_TAG, nullptr, nullptr,
                       iters);
  if (rc) return rc;
  return vdiff_api<R>(ctx, dt, cnpar, avmol, f, hn, nuh, ctx->zmask, nullptr);
}
template int tracer_step_impl<double>(getm_ctx*, double, double*, const double*, const double*, const double*,
                                      const double*, const double*, const double*, const double*, const double*, int,
                                      int, int, double, double, double, int);
template int tracer_step_impl<float>(getm_ctx*, float, float*, const float*, const float*, const float*,
                                     const float*, const float*, const float*, const float*, const float*, int, int,
                                     int, float, float, float, int);

template <class R>
static int content_api(getm_ctx* ctx, const R* f, const R* h, const int32_t* az, double* out) {
  if (!ctx || !f || !h || !az || !out) return fail(ctx, GETM_ERR_ARG, "tracer_content: bad argument");
  GB_TRY(run_content<R>(ctx->dev, ctx->stream, f, h, az, ctx->red, ctx->red + 2 * RED_BLOCKS), "content");
  double r[2];
  GB_TRY(cudaMemcpyAsync(r, ctx->red + 2 * RED_BLOCKS, sizeof(r), cudaMemcpyDeviceToHost, ctx->stream), "read");
  GB_TRY(cudaStreamSynchronize(ctx->stream), "sync");
  *out = r[0];
  return GETM_OK;
}

namespace gb {

// Rows [r0, r0+nrows) (array rows, i.e. j - (jmin-2)) of nk consecutive levels of a field of elem
// bytes, copied to or from a packed buffer laid out [level][row][i] (the ni elements of a row are
// contiguous in both). 16-byte words where the whole block allows it, else elements.
template <class W>
__global__ void k_rows_copy(const Dev d, char* f, char* buf, int r0, int nrows, int nk, int words_per_row,
                            long long row_stride_w, long long level_stride_w, int to_buf) {
  const long long n = (long long)words_per_row * nrows * nk;
  W* fw = reinterpret_cast<W*>(f);
  W* bw = reinterpret_cast<W*>(buf);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long q = t % words_per_row, rk = t / words_per_row;
    const long long r = rk % nrows, k = rk / nrows;
    const long long fo = k * level_stride_w + (r0 + r) * row_stride_w + q;
    if (to_buf) bw[t] = fw[fo];
    else fw[fo] = bw[t];
  }
}

}  // namespace gb

static int rows_copy(getm_ctx* ctx, void* f, int elem_bytes, int nk, int j_first, int nrows, void* buf, int to_buf) {
  using namespace gb;
  if (!ctx || !f || !buf || (elem_bytes != 4 && elem_bytes != 8) || nk < 1 || nrows < 1) return GETM_ERR_ARG;
  const Dev& d = ctx->dev;
  const int r0 = j_first - (d.jmin - HALO);
  if (r0 < 0 || r0 + nrows > d.nj() || nk > d.kmax + 1)
    return fail(ctx, GETM_ERR_ARG, "halo rows: rows or levels outside the field");
  const long long row_bytes = (long long)d.ni() * elem_bytes;
  const long long sj_b = d.sj * elem_bytes, sk_b = d.sk * elem_bytes;
  const bool w16 = row_bytes % 16 == 0 && sj_b % 16 == 0 && sk_b % 16 == 0 &&
                   reinterpret_cast<uintptr_t>(f) % 16 == 0 && reinterpret_cast<uintptr_t>(buf) % 16 == 0;
  const int wb = w16 ? 16 : elem_bytes;
  const long long n = row_bytes / wb * nrows * nk;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 4 * 148);
  TimerScope ts(ctx, GETM_TIM_COPY);
  char* fc = static_cast<char*>(f);
  char* bc = static_cast<char*>(buf);
  if (wb == 16)
    k_rows_copy<int4><<<blocks, 256, 0, ctx->stream>>>(d, fc, bc, r0, nrows, nk, (int)(row_bytes / 16), sj_b / 16,
                                                       sk_b / 16, to_buf);
  else if (wb == 8)
    k_rows_copy<long long><<<blocks, 256, 0, ctx->stream>>>(d, fc, bc, r0, nrows, nk, (int)(row_bytes / 8), sj_b / 8,
                                                            sk_b / 8, to_buf);
  else
    k_rows_copy<int><<<blocks, 256, 0, ctx->stream>>>(d, fc, bc, r0, nrows, nk, (int)(row_bytes / 4), sj_b / 4,
                                                      sk_b / 4, to_buf);
  GB_TRY(cudaGetLastError(), "halo rows");
  return GETM_OK;
}

extern "C" {

const char* getm_version(void) { return "getm-b200 0.1 (sm_100a)"; }

int getm_ctx_create(const getm_domain* dom, void* stream, getm_ctx** out) {
  if (!dom || !out) return GETM_ERR_ARG;
  *out = nullptr;
  if (dom->imax < dom->imin || dom->jmax < dom->jmin || dom->kmax < 0) return GETM_ERR_ARG;
  const long long ni = dom->imax - dom->imin + 1 + 2 * HALO;
  const long long nj = dom->jmax - dom->jmin + 1 + 2 * HALO;
  if (dom->sj < ni || dom->sk < dom->sj * nj) return GETM_ERR_ARG;
  if (!(dom->dx > 0) || !(dom->dy > 0) || !(dom->ard1 > 0)) return GETM_ERR_ARG;
  getm_ctx* ctx = new getm_ctx();
  ctx->dom = *dom;
  ctx->dev = to_dev(*dom);
  ctx->stream = (cudaStream_t)stream;
  cudaGetDevice(&ctx->device);
  const long long n = n2d(ctx->dev);
  if (cudaMalloc(&ctx->planes, (size_t)n * NPLANES) != cudaSuccess ||
      cudaMalloc(&ctx->zmask, (size_t)n * 3 * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&ctx->red, (2 * RED_BLOCKS + 2) * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&ctx->cnt, GB_NCOUNTERS * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    getm_ctx_destroy(ctx);
    return GETM_ERR_NOMEM;
  }
  if (cudaMemsetAsync(ctx->cnt, 0, GB_NCOUNTERS * sizeof(unsigned long long), ctx->stream) != cudaSuccess) {
    getm_ctx_destroy(ctx);
    return GETM_ERR_CUDA;
  }
  *out = ctx;
  return GETM_OK;
}

int getm_ctx_destroy(getm_ctx* ctx) {
  if (!ctx) return GETM_OK;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream); else cudaDeviceSynchronize();
  cudaFree(ctx->planes);
  cudaFree(ctx->zmask);
  cudaFree(ctx->red);
  cudaFree(ctx->cnt);
  cudaFree(ctx->stage);
  for (auto p : ctx->scr) cudaFree(p);
  cudaFree(ctx->bc_scr3);
  cudaFree(ctx->bc_scr2);
  cudaFree(ctx->colh);
  cudaFree(ctx->w2);
  cudaFree(ctx->adj_scr);
  cudaFree(ctx->adj_store);
  for (void* p : {(void*)ctx->bdy.pts, (void*)ctx->bdy.data, (void*)ctx->bdy.data_u, (void*)ctx->bdy.data_v,
                  (void*)ctx->bdy.amp, (void*)ctx->bdy.phase, (void*)ctx->bdy.pairs})
    cudaFree(p);
  for (int t = 0; t < GETM_NTIMERS; ++t)
    for (auto& ev : ctx->pending[t]) ctx->pool.push_back(ev);
  for (auto& ev : ctx->pool) {
    cudaEventDestroy(ev.first);
    cudaEventDestroy(ev.second);
  }
  delete ctx;
  return GETM_OK;
}

int getm_ctx_set_stream(getm_ctx* ctx, void* stream) {
  if (!ctx) return GETM_ERR_ARG;
  ctx->stream = (cudaStream_t)stream;
  return GETM_OK;
}

int getm_ctx_take_warnings(getm_ctx* ctx, int64_t* n_warnings) {
  if (!ctx || !n_warnings) return GETM_ERR_ARG;
  // counters [0] (iteration cap of adv_split_w) and [2] (log-law arguments <= 1 of the slow
  // bottom friction); [1] belongs to check_3d_fields
  unsigned long long h[3] = {0, 0, 0};
  GB_TRY(cudaMemcpyAsync(h, ctx->cnt, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream), "read warnings");
  GB_TRY(cudaMemsetAsync(ctx->cnt, 0, sizeof(unsigned long long), ctx->stream), "reset warnings");
  GB_TRY(cudaMemsetAsync(ctx->cnt + 2, 0, sizeof(unsigned long long), ctx->stream), "reset warnings");
  GB_TRY(cudaStreamSynchronize(ctx->stream), "sync");
  *n_warnings = (int64_t)(h[0] + h[2]);
  return GETM_OK;
}

const char* getm_ctx_last_error(const getm_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

static const char* kTimerNames[GETM_NTIMERS] = {"adv_split_u", "adv_split_v", "adv_split_w", "adv_finalise",
                                                 "tracer_vdiff", "copy", "tracer_fused_uv",
                                                 "tracer_fused_wvu", "mode_split_2d", "macro_3d_other", "internal_pressure",
                                                 "uv_momentum_3d", "tracer_record", "tracer_adjoint", "reserved14",
                                                 "reserved15"};

const char* getm_timer_name(int slot) {
  return (slot >= 0 && slot < GETM_NTIMERS) ? kTimerNames[slot] : "";
}

static void drain_timers(getm_ctx* ctx) {
  for (int t = 0; t < GETM_NTIMERS; ++t) {
    for (auto& ev : ctx->pending[t]) {
      float ms = 0.f;
      cudaEventSynchronize(ev.second);
      cudaEventElapsedTime(&ms, ev.first, ev.second);
      ctx->total_ms[t] += ms;
      ctx->launches[t] += 1;
      ctx->pool.push_back(ev);
    }
    ctx->pending[t].clear();
  }
}

int getm_set_vector_sweeps(int on) {
  return gb::g_vector_sweeps.exchange(on != 0 ? 1 : 0);
}

int getm_set_fp32_micro_steps(int on) {
  return gb::g_fp32_micro.exchange(on != 0 ? 1 : 0);
}

int getm_set_fused_micro_step(int on) {
  return gb::g_fused_micro.exchange(on != 0 ? 1 : 0);
}

int getm_timers_enable(getm_ctx* ctx, int on) {
  if (!ctx) return GETM_ERR_ARG;
  ctx->timing = on != 0;
  return GETM_OK;
}

int getm_timers_reset(getm_ctx* ctx) {
  if (!ctx) return GETM_ERR_ARG;
  drain_timers(ctx);
  for (int t = 0; t < GETM_NTIMERS; ++t) {
    ctx->total_ms[t] = 0.0;
    ctx->launches[t] = 0;
  }
  return GETM_OK;
}

int getm_timers_read(getm_ctx* ctx, int slot, double* total_ms, int64_t* launches) {
  if (!ctx || slot < 0 || slot >= GETM_NTIMERS || !total_ms || !launches) return GETM_ERR_ARG;
  drain_timers(ctx);
  *total_ms = ctx->total_ms[slot];
  *launches = ctx->launches[slot];
  return GETM_OK;
}

int getm_init_advection(getm_ctx* ctx, const int32_t* az, const int32_t* au, const int32_t* av,
                        const int32_t* ax) {
  if (!ctx || !az || !au || !av || !ax) return fail(ctx, GETM_ERR_ARG, "init_advection: null mask");
  const long long n = n2d(ctx->dev);
  GB_TRY(run_build_masks(ctx->dev, ctx->stream, az, au, av, ax, ctx->planes), "build masks");
  GB_TRY(cudaMemcpyAsync(ctx->zmask, az, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream), "az");
  GB_TRY(cudaMemcpyAsync(ctx->zmask + n, au, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream), "au");
  GB_TRY(cudaMemcpyAsync(ctx->zmask + 2 * n, av, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream),
         "av");
  ctx->adv_ready = true;
  return GETM_OK;
}

int getm_adv_grid_for_tag(const getm_ctx* ctx, int tag, getm_adv_grid* out) {
  if (!ctx || !out) return GETM_ERR_ARG;
  if (!ctx->adv_ready) return GETM_ERR_STATE;
  return grid_for_tag(ctx, tag, out) ? GETM_OK : GETM_ERR_ARG;
}

int getm_adv_split_u(getm_ctx* ctx, int nk, double dt, const double* f, double* fi, double* Di, double* adv,
                     const double* U, const double* DU, double splitfac, int scheme, double AH,
                     const uint8_t* mask_flux, const uint8_t* mask_update) {
  return sweep_h_api<double>(ctx, 0, nk, dt, f, fi, Di, adv, U, DU, splitfac, scheme, AH, mask_flux, mask_update);
}

int getm_adv_split_v(getm_ctx* ctx, int nk, double dt, const double* f, double* fi, double* Di, double* adv,
                     const double* V, const double* DV, double splitfac, int scheme, double AH,
                     const uint8_t* mask_flux, const uint8_t* mask_update) {
  return sweep_h_api<double>(ctx, 1, nk, dt, f, fi, Di, adv, V, DV, splitfac, scheme, AH, mask_flux, mask_update);
}

extern "C++" {
template <class R>
static int sweep_w_api(getm_ctx* ctx, R dt, const R* f, R* fi, R* hi, R* adv, const R* ww, R splitfac, int scheme,
                       int tag, const int32_t* az, int itersmax) {
  if (!ctx || !f || !fi || !hi || !ww || !az) return fail(ctx, GETM_ERR_ARG, "adv_split_w: bad argument");
  if (scheme == NOADV) return GETM_OK;
  if (!is_split_scheme(scheme)) return fail(ctx, GETM_ERR_ARG, "adv_split_w: scheme is invalid");
  if (itersmax > 1 && ctx->dom.kmax > 128)
    return fail(ctx, GETM_ERR_UNSUPPORTED, "adv_split_w: itersmax > 1 needs kmax <= 128");
  const int kshift = (tag == GETM_W_TAG) ? 1 : 0;
  return cuda_fail(ctx,
                   run_sweep_w<R>(ctx->dev, ctx->stream, dt, splitfac, scheme, kshift, itersmax < 1 ? 1 : itersmax, f,
                                  fi, fi, hi, adv, ww, az, ctx->cnt),
                   "adv_split_w");
}
}  // extern "C++"

int getm_adv_split_w(getm_ctx* ctx, double dt, const double* f, double* fi, double* hi, double* adv,
                     const double* ww, double splitfac, int scheme, int tag, const int32_t* az, int itersmax) {
  return sweep_w_api<double>(ctx, dt, f, fi, hi, adv, ww, splitfac, scheme, tag, az, itersmax);
}

int getm_adv_split_u_f32(getm_ctx* ctx, int nk, float dt, const float* f, float* fi, float* Di, float* adv,
                         const float* U, const float* DU, float splitfac, int scheme, float AH,
                         const uint8_t* mask_flux, const uint8_t* mask_update) {
  return sweep_h_api<float>(ctx, 0, nk, dt, f, fi, Di, adv, U, DU, splitfac, scheme, AH, mask_flux, mask_update);
}

int getm_adv_split_v_f32(getm_ctx* ctx, int nk, float dt, const float* f, float* fi, float* Di, float* adv,
                         const float* V, const float* DV, float splitfac, int scheme, float AH,
                         const uint8_t* mask_flux, const uint8_t* mask_update) {
  return sweep_h_api<float>(ctx, 1, nk, dt, f, fi, Di, adv, V, DV, splitfac, scheme, AH, mask_flux, mask_update);
}

int getm_adv_split_w_f32(getm_ctx* ctx, float dt, const float* f, float* fi, float* hi, float* adv, const float* ww,
                         float splitfac, int scheme, int tag, const int32_t* az, int itersmax) {
  return sweep_w_api<float>(ctx, dt, f, fi, hi, adv, ww, splitfac, scheme, tag, az, itersmax);
}

int getm_do_advection_3d(getm_ctx* ctx, double dt, double* f, const double* uu, const double* vv,
                         const double* ww, const double* hu, const double* hv, const double* ho,
                         const double* hn, int split, int hscheme, int vscheme, double AH, int tag,
                         double* hires, double* advres, int adv_ver_iterations) {
  return do_adv3d<double>(ctx, dt, f, uu, vv, ww, hu, hv, ho, hn, split, hscheme, vscheme, AH, tag, hires,
                          advres, adv_ver_iterations);
}

int getm_do_advection_3d_f32(getm_ctx* ctx, float dt, float* f, const float* uu, const float* vv,
                             const float* ww, const float* hu, const float* hv, const float* ho, const float* hn,
                             int split, int hscheme, int vscheme, float AH, int tag, float* hires,
                             float* advres, int adv_ver_iterations) {
  return do_adv3d<float>(ctx, dt, f, uu, vv, ww, hu, hv, ho, hn, split, hscheme, vscheme, AH, tag, hires, advres,
                         adv_ver_iterations);
}

int getm_tridiagonal_columns(getm_ctx* ctx, int ncol, int kmax, int fi, int lt, const double* au,
                             const double* bu, const double* cu, const double* du, double* value) {
  if (!ctx || ncol < 0 || kmax < 1 || fi < 0 || lt > kmax || fi >= lt || !au || !bu || !cu || !du || !value)
    return fail(ctx, GETM_ERR_ARG, "tridiagonal: bad argument");
  if (ncol == 0) return GETM_OK;
  if ((size_t)2 * (kmax + 1) * 64 * sizeof(double) > 200 * 1024)
    return fail(ctx, GETM_ERR_UNSUPPORTED, "tridiagonal: kmax too large");
  return cuda_fail(ctx, run_tridiag<double>(ctx->stream, ncol, kmax, fi, lt, au, bu, cu, du, value), "tridiagonal");
}


int getm_tracer_vdiff(getm_ctx* ctx, double dt, double cnpar, double avmol, double* S, const double* hn,
                      const double* nuh, const int32_t* az, const double* src) {
  return vdiff_api<double>(ctx, dt, cnpar, avmol, S, hn, nuh, az, src);
}

int getm_tracer_vdiff_f32(getm_ctx* ctx, float dt, float cnpar, float avmol, float* S, const float* hn,
                          const float* nuh, const int32_t* az, const float* src) {
  return vdiff_api<float>(ctx, dt, cnpar, avmol, S, hn, nuh, az, src);
}


int getm_tracer_step(getm_ctx* ctx, double dt, double* f, const double* uu, const double* vv, const double* ww,
                     const double* hu, const double* hv, const double* ho, const double* hn, const double* nuh,
                     int split, int hscheme, int vscheme, double AH, double cnpar, double avmol,
                     int adv_ver_iterations) {
  return tracer_step_impl<double>(ctx, dt, f, uu, vv, ww, hu, hv, ho, hn, nuh, split, hscheme, vscheme, AH, cnpar, avmol,
                             adv_ver_iterations);
}

int getm_tracer_step_f32(getm_ctx* ctx, float dt, float* f, const float* uu, const float* vv, const float* ww,
                         const float* hu, const float* hv, const float* ho, const float* hn, const float* nuh,
                         int split, int hscheme, int vscheme, float AH, float cnpar, float avmol,
                         int adv_ver_iterations) {
  return tracer_step_impl<float>(ctx, dt, f, uu, vv, ww, hu, hv, ho, hn, nuh, split, hscheme, vscheme, AH, cnpar, avmol,
                            adv_ver_iterations);
}


int getm_tracer_content(getm_ctx* ctx, const double* f, const double* h, const int32_t* az, double* out) {
  return content_api<double>(ctx, f, h, az, out);
}

int getm_tracer_content_f32(getm_ctx* ctx, const float* f, const float* h, const int32_t* az, double* out) {
  return content_api<float>(ctx, f, h, az, out);
}

int getm_halo_pack(getm_ctx* ctx, const void* f, int elem_bytes, int nk, int j_first, int nrows, void* buf) {
  return rows_copy(ctx, const_cast<void*>(f), elem_bytes, nk, j_first, nrows, buf, 1);
}

int getm_halo_unpack(getm_ctx* ctx, void* f, int elem_bytes, int nk, int j_first, int nrows, const void* buf) {
  return rows_copy(ctx, f, elem_bytes, nk, j_first, nrows, const_cast<void*>(buf), 0);
}

int getm_check_3d_fields(getm_ctx* ctx, const double* f, const int32_t* az, double minval, double maxval,
                         int64_t* status) {
  if (!ctx || !f || !az || !status) return fail(ctx, GETM_ERR_ARG, "check_3d_fields: bad argument");
  GB_TRY(cudaMemsetAsync(ctx->cnt + 1, 0, sizeof(unsigned long long), ctx->stream), "reset");
  GB_TRY(run_check_range<double>(ctx->dev, ctx->stream, f, az, minval, maxval, ctx->cnt + 1), "check");
  unsigned long long h = 0;
  GB_TRY(cudaMemcpyAsync(&h, ctx->cnt + 1, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream), "read");
  GB_TRY(cudaStreamSynchronize(ctx->stream), "sync");
  *status = (int64_t)h;
  return GETM_OK;
}

}  // extern "C"
