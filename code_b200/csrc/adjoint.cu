// adjoint.cu -- host side of the tracer adjoint: the forward step that records the tape, the
// adjoint step, and the checkpointed gradient over many steps (C-ABI entry points).
//
// The tracer step is do_advection_3d(H_TAG) with HALFSPLIT (u/2 v/2 w v/2 u/2,
// advection_3d.F90:439-537) followed by the implicit vertical diffusion (salinity.F90:348-389).
// The reference has no adjoint; this one differentiates the discrete step exactly for frozen
// limiter branches (the branch of every face is recorded by the forward sweep).
//
// Tape of one step: five planes of branch codes (one byte per face and sweep, each plane laid out
// like a 3D field: n3 = sk*(kmax+1) bytes) followed by nothing else; and the tracer after
// advection (the diffusion's input), one 3D field of the step's precision.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "launch.h"

#include "ctx_internal.h"

namespace {

constexpr int ADJ_NSCR = 8;  // Sn, tmp, H1..H4, RU, QU

template <class R>
int check_adj_args(getm_ctx* ctx, int split, int hs, int vs, const void* f, const void* uu, const void* vv,
                   const void* ww, const void* hu, const void* hv, const void* ho, const void* hn,
                   const void* nuh) {
  if (!ctx) return GETM_ERR_ARG;
  if (!ctx->adv_ready) return fail(ctx, GETM_ERR_STATE, "getm_init_advection has not been called");
  if (!f || !uu || !vv || !ww || !hu || !hv || !ho || !hn || !nuh)
    return fail(ctx, GETM_ERR_ARG, "tracer adjoint: null field");
  if (split != GETM_HALFSPLIT) return fail(ctx, GETM_ERR_UNSUPPORTED, "tracer adjoint: only HALFSPLIT");
  if (!is_split_scheme(hs)) return fail(ctx, GETM_ERR_UNSUPPORTED, "tracer adjoint: hscheme must be a split scheme");
  if (vs != NOADV && !is_split_scheme(vs))
    return fail(ctx, GETM_ERR_UNSUPPORTED, "tracer adjoint: vscheme must be a split scheme or NOADV");
  return GETM_OK;
}

int ensure_adj_scratch(getm_ctx* ctx, size_t bytes) {
  if (ctx->adj_scr_bytes >= bytes) return GETM_OK;
  cudaFree(ctx->adj_scr);
  ctx->adj_scr = nullptr;
  ctx->adj_scr_bytes = 0;
  if (cudaMalloc(&ctx->adj_scr, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, GETM_ERR_NOMEM, "adjoint scratch allocation failed");
  }
  ctx->adj_scr_bytes = bytes;
  return GETM_OK;
}

// Forward tracer step (HALFSPLIT, itersmax = 1) that writes the tape: the same kernels and
// arguments as do_adv3d + vdiff_api, with branch recording switched on.
template <class R>
int step_record(getm_ctx* ctx, R dt, R* f, const R* uu, const R* vv, const R* ww, const R* hu, const R* hv,
                const R* ho, const R* hn, const R* nuh, int hs, int vs, R AH, R cnpar, R avmol, uint8_t* codes,
                R* g, R* sn = nullptr) {
  const Dev& d = ctx->dev;
  cudaStream_t s = ctx->stream;
  const long long n3 = n3d(d);
  const long long sk = d.sk;
  const int kmax = d.kmax;
  getm_adv_grid gr;
  grid_for_tag(ctx, GETM_H_TAG, &gr);
  int rc = ensure_scratch(ctx, (size_t)n3 * sizeof(R));
  if (rc) return rc;
  R* S = (R*)ctx->scr[0];
  R* H = (R*)ctx->scr[1];
  auto L = [&](auto* p, int k) { return p + (long long)k * sk; };
  auto plane = [&](int q) { return codes + (long long)q * n3; };
  const R half = R(0.5), one = R(1);
  // (level 0 of the heights is not read by the H-grid sweeps)
  const int nk = kmax;
  GB_TIMED(GETM_TIM_ADJ_RECORD, (run_sweep_h<R, 0>(d, s, nk, dt, half, hs, AH, L(f, 1), L(f, 1), L(S, 1), L(ho, 1),
                                 L(H, 1), nullptr, L(uu, 1), L(hu, 1), gr.mask_uflux, gr.mask_uupdate,
                                 L(plane(0), 1))), "u1");
  GB_TIMED(GETM_TIM_ADJ_RECORD, (run_sweep_h<R, 1>(d, s, nk, dt, half, hs, AH, L(S, 1), L(S, 1), L(f, 1), L(H, 1),
                                 L(H, 1), nullptr, L(vv, 1), L(hv, 1), gr.mask_vflux, gr.mask_vupdate,
                                 L(plane(1), 1))), "v1");
  if (vs != NOADV && kmax > 1)
    GB_TIMED(GETM_TIM_ADJ_RECORD, run_sweep_w<R>(d, s, dt, one, vs, 0, 1, f, f, f, H, nullptr, ww, gr.az, ctx->cnt,
                                                 plane(2)), "w");
  GB_TIMED(GETM_TIM_ADJ_RECORD, (run_sweep_h<R, 1>(d, s, nk, dt, half, hs, AH, L(f, 1), L(f, 1), L(S, 1), L(H, 1),
                                 L(H, 1), nullptr, L(vv, 1), L(hv, 1), gr.mask_vflux, gr.mask_vupdate,
                                 L(plane(3), 1))), "v2");
  GB_TIMED(GETM_TIM_ADJ_RECORD, (run_sweep_h<R, 0>(d, s, nk, dt, half, hs, AH, L(S, 1), L(S, 1), L(f, 1), L(H, 1),
                                 L(H, 1), nullptr, L(uu, 1), L(hu, 1), gr.mask_uflux, gr.mask_uupdate,
                                 L(plane(4), 1))), "u2");
  GB_TIMED(GETM_TIM_ADJ_RECORD, cudaMemcpyAsync(g, f, (size_t)n3 * sizeof(R), cudaMemcpyDeviceToDevice, s), "tape g");
  // the diffusion's result also goes to sn when the caller keeps the step outputs (only the solved
  // columns are written there -- the only ones the adjoint diffusion reads)
  GB_TIMED(GETM_TIM_ADJ_RECORD, run_vdiff<R>(d, s, dt, cnpar, avmol, f, hn, nuh, ctx->zmask, nullptr, (R*)ctx->scr[0],
                                             (R*)ctx->scr[1], nullptr, sn), "vdiff");
  return GETM_OK;
}

// Adjoint of one tracer step: fbar (cotangent of the step's output) becomes the cotangent of its
// input; nubar accumulates the cotangent of nuh. Sn_in = the step's output (the diffusion's
// result) when the caller kept it, else it is re-solved from g; heights_ready = the heights before
// sweeps 2..5 are already in the adjoint scratch (the velocities and layer heights are those of
// the previous call).
template <class R>
int step_adjoint(getm_ctx* ctx, R dt, R* fbar, R* nubar, const R* uu, const R* vv, const R* ww, const R* hu,
                 const R* hv, const R* ho, const R* hn, const R* nuh, int hs, int vs, R AH, R cnpar, R avmol,
                 const uint8_t* codes, const R* g, const R* Sn_in = nullptr, bool heights_ready = false) {
  const Dev& d = ctx->dev;
  cudaStream_t s = ctx->stream;
  const long long n3 = n3d(d);
  const long long sk = d.sk;
  const int kmax = d.kmax;
  getm_adv_grid gr;
  grid_for_tag(ctx, GETM_H_TAG, &gr);
  int rc = ensure_adj_scratch(ctx, (size_t)ADJ_NSCR * n3 * sizeof(R));
  if (rc) return rc;
  rc = ensure_scratch(ctx, (size_t)n3 * sizeof(R));
  if (rc) return rc;
  R* base = (R*)ctx->adj_scr;
  R *Sn = base, *tmp = base + n3, *H1 = base + 2 * n3, *H2 = base + 3 * n3, *H3 = base + 4 * n3,
    *H4 = base + 5 * n3, *RU = base + 6 * n3, *QU = base + 7 * n3;
  auto L = [&](auto* p, int k) { return p + (long long)k * sk; };
  auto plane = [&](int q) { return codes + (long long)q * n3; };
  const R half = R(0.5), one = R(1);
  const bool has_w = vs != NOADV && kmax > 1;
  // the diffusion's output: kept by the caller, or re-solved from its input on the tape
  const R* Sout = Sn_in;
  if (!Sout) {
    GB_TIMED(GETM_TIM_ADJ, cudaMemcpyAsync(Sn, g, (size_t)n3 * sizeof(R), cudaMemcpyDeviceToDevice, s), "copy g");
    GB_TIMED(GETM_TIM_ADJ, run_vdiff<R>(d, s, dt, cnpar, avmol, Sn, hn, nuh, ctx->zmask, nullptr, RU, QU), "vdiff");
    Sout = Sn;
  }
  GB_TIMED(GETM_TIM_ADJ, run_adj_vdiff<R>(d, s, dt, cnpar, avmol, fbar, tmp, nubar, g, Sout, hn, nuh, ctx->zmask,
                                          RU, QU), "adjoint vdiff");
  if (!heights_ready)
    GB_TIMED(GETM_TIM_ADJ, run_adj_heights<R>(d, s, dt, hs == UPSTREAM ? 0 : 1, has_w, ho, uu, vv, ww,
                                              gr.mask_uupdate, gr.mask_vupdate, gr.az, H1, H2, H3, H4), "heights");
  // u/2 (sweep 5): tmp -> fbar
  GB_TIMED(GETM_TIM_ADJ, (run_adj_sweep_h<R, 0>(d, s, kmax, dt, half, hs, AH, L(tmp, 1), L(fbar, 1), L(H4, 1),
                                                L(uu, 1), L(hu, 1), gr.mask_uflux, gr.mask_uupdate,
                                                L(plane(4), 1), true)), "adjoint u2");
  // v/2 (sweep 4): fbar -> tmp
  GB_TIMED(GETM_TIM_ADJ, (run_adj_sweep_h<R, 1>(d, s, kmax, dt, half, hs, AH, L(fbar, 1), L(tmp, 1), L(H3, 1),
                                                L(vv, 1), L(hv, 1), gr.mask_vflux, gr.mask_vupdate,
                                                L(plane(3), 1), true)), "adjoint v2");
  // w (sweep 3): tmp -> fbar
  if (has_w) {
    GB_TIMED(GETM_TIM_ADJ, run_adj_sweep_w<R>(d, s, dt, one, vs, 0, tmp, fbar, H2, ww, gr.az, plane(2)),
             "adjoint w");
  } else {
    GB_TRY(cudaMemcpyAsync(fbar, tmp, (size_t)n3 * sizeof(R), cudaMemcpyDeviceToDevice, s), "copy");
  }
  // v/2 (sweep 2): fbar -> tmp
  GB_TIMED(GETM_TIM_ADJ, (run_adj_sweep_h<R, 1>(d, s, kmax, dt, half, hs, AH, L(fbar, 1), L(tmp, 1), L(H1, 1),
                                                L(vv, 1), L(hv, 1), gr.mask_vflux, gr.mask_vupdate,
                                                L(plane(1), 1), true)), "adjoint v1");
  // u/2 (sweep 1): tmp -> fbar
  GB_TIMED(GETM_TIM_ADJ, (run_adj_sweep_h<R, 0>(d, s, kmax, dt, half, hs, AH, L(tmp, 1), L(fbar, 1), L(ho, 1),
                                                L(uu, 1), L(hu, 1), gr.mask_uflux, gr.mask_uupdate,
                                                L(plane(0), 1), true)), "adjoint u1");
  return GETM_OK;
}

template <class R>
int record_api(getm_ctx* ctx, R dt, R* f, const R* uu, const R* vv, const R* ww, const R* hu, const R* hv,
               const R* ho, const R* hn, const R* nuh, int split, int hs, int vs, R AH, R cnpar, R avmol,
               uint8_t* codes, R* g) {
  int rc = check_adj_args<R>(ctx, split, hs, vs, f, uu, vv, ww, hu, hv, ho, hn, nuh);
  if (rc) return rc;
  if (!codes || !g) return fail(ctx, GETM_ERR_ARG, "tracer_step_record: null tape");
  return step_record<R>(ctx, dt, f, uu, vv, ww, hu, hv, ho, hn, nuh, hs, vs, AH, cnpar, avmol, codes, g);
}

template <class R>
int adjoint_api(getm_ctx* ctx, R dt, R* fbar, R* nubar, const R* uu, const R* vv, const R* ww, const R* hu,
                const R* hv, const R* ho, const R* hn, const R* nuh, int split, int hs, int vs, R AH, R cnpar,
                R avmol, const uint8_t* codes, const R* g) {
  int rc = check_adj_args<R>(ctx, split, hs, vs, fbar, uu, vv, ww, hu, hv, ho, hn, nuh);
  if (rc) return rc;
  if (!nubar || !codes || !g) return fail(ctx, GETM_ERR_ARG, "tracer_step_adjoint: null argument");
  return step_adjoint<R>(ctx, dt, fbar, nubar, uu, vv, ww, hu, hv, ho, hn, nuh, hs, vs, AH, cnpar, avmol, codes, g);
}

// Checkpointed gradient: nsteps forward steps from f (f is advanced to the final state), keeping
// f every `every` steps; then, block by block from the last, the block's steps are recomputed from
// its checkpoint with the tape recorded, and the adjoint steps run in reverse. fbar enters as the
// cotangent of the final state and leaves as that of the initial state; nubar accumulates the
// cotangent of nuh (constant in time).
template <class R>
int gradient_api(getm_ctx* ctx, int nsteps, int every, R dt, R* f, const R* uu, const R* vv, const R* ww,
                 const R* hu, const R* hv, const R* ho, const R* hn, const R* nuh, int split, int hs, int vs, R AH,
                 R cnpar, R avmol, R* fbar, R* nubar, float* ms_forward, float* ms_reverse) {
  int rc = check_adj_args<R>(ctx, split, hs, vs, f, uu, vv, ww, hu, hv, ho, hn, nuh);
  if (rc) return rc;
  if (!fbar || !nubar || nsteps < 0 || every < 1) return fail(ctx, GETM_ERR_ARG, "tracer_gradient: bad argument");
  const Dev& d = ctx->dev;
  cudaStream_t s = ctx->stream;
  const long long n3 = n3d(d);
  const size_t fb = (size_t)n3 * sizeof(R);
  const int nblk = (nsteps + every - 1) / every;
  const int blk = nsteps < every ? nsteps : every;
  const size_t tape1 = 5 * (size_t)n3 + 2 * fb;  // codes + g + the step's output of one step
  const size_t need = (size_t)nblk * fb + (size_t)blk * tape1 + 256;
  if (ctx->adj_store_bytes < need) {
    cudaFree(ctx->adj_store);
    ctx->adj_store = nullptr;
    ctx->adj_store_bytes = 0;
    if (cudaMalloc(&ctx->adj_store, need) != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, GETM_ERR_NOMEM, "tracer_gradient: checkpoint allocation failed");
    }
    ctx->adj_store_bytes = need;
  }
  R* ckpt = (R*)ctx->adj_store;
  uint8_t* tape = (uint8_t*)ctx->adj_store + (size_t)nblk * fb;
  // g of step q of a block: tape + q*tape1 + 5*n3 (the codes come first); 5*n3 is not always a
  // multiple of the element size, so the g parts are placed after all code planes instead
  uint8_t* codes0 = tape;
  R* g0 = (R*)(tape + (size_t)blk * 5 * n3 + (256 - ((size_t)blk * 5 * n3) % 256) % 256);
  R* sn0 = g0 + (size_t)blk * n3;  // the output of each step of the block (the diffusion's result)
  if ((uint8_t*)(sn0 + (size_t)blk * n3) > (uint8_t*)ctx->adj_store + need)
    return fail(ctx, GETM_ERR_NOMEM, "tracer_gradient: tape layout");
  cudaEvent_t ev[3];
  for (auto& e : ev) GB_TRY(cudaEventCreate(&e), "event");
  struct EvFree {
    cudaEvent_t* e;
    ~EvFree() { for (int i = 0; i < 3; ++i) cudaEventDestroy(e[i]); }
  } evfree{ev};
  GB_TRY(cudaEventRecord(ev[0], s), "event");
  // the steps of the last block are taped while they run forward: the reverse starts with that
  // block, so it needs no checkpoint and is not recomputed
  const int last0 = (nblk - 1) * every;
  for (int n = 0; n < nsteps; ++n) {
    if (n >= last0) {
      const int q = n - last0;
      rc = step_record<R>(ctx, dt, f, uu, vv, ww, hu, hv, ho, hn, nuh, hs, vs, AH, cnpar, avmol,
                          codes0 + (size_t)q * 5 * n3, g0 + (size_t)q * n3, sn0 + (size_t)q * n3);
      if (rc) return rc;
      continue;
    }
    if (n % every == 0)
      GB_TRY(cudaMemcpyAsync(ckpt + (size_t)(n / every) * n3, f, fb, cudaMemcpyDeviceToDevice, s), "checkpoint");
    rc = tracer_step_impl<R>(ctx, dt, f, uu, vv, ww, hu, hv, ho, hn, nuh, split, hs, vs, AH, cnpar, avmol, 1);
    if (rc) return rc;
  }
  GB_TRY(cudaEventRecord(ev[1], s), "event");
  bool heights_done = false;
  // reverse: blocks from the last; the forward state of a block is rebuilt in scr-independent
  // storage (the checkpoint slot itself: its value is not needed again)
  for (int b = nblk - 1; b >= 0; --b) {
    const int n0 = b * every;
    const int cnt = (n0 + every <= nsteps) ? every : nsteps - n0;
    R* fw = ckpt + (size_t)b * n3;
    for (int q = 0; q < cnt && b != nblk - 1; ++q) {
      rc = step_record<R>(ctx, dt, fw, uu, vv, ww, hu, hv, ho, hn, nuh, hs, vs, AH, cnpar, avmol,
                          codes0 + (size_t)q * 5 * n3, g0 + (size_t)q * n3, sn0 + (size_t)q * n3);
      if (rc) return rc;
    }
    for (int q = cnt - 1; q >= 0; --q) {
      // velocities, heights and nuh are the same in every step: the heights before each sweep are
      // computed by the first adjoint step and reused
      rc = step_adjoint<R>(ctx, dt, fbar, nubar, uu, vv, ww, hu, hv, ho, hn, nuh, hs, vs, AH, cnpar, avmol,
                           codes0 + (size_t)q * 5 * n3, g0 + (size_t)q * n3, sn0 + (size_t)q * n3, heights_done);
      if (rc) return rc;
      heights_done = true;
    }
  }
  GB_TRY(cudaEventRecord(ev[2], s), "event");
  GB_TRY(cudaEventSynchronize(ev[2]), "sync");
  float a = 0.f, r = 0.f;
  GB_TRY(cudaEventElapsedTime(&a, ev[0], ev[1]), "elapsed");
  GB_TRY(cudaEventElapsedTime(&r, ev[1], ev[2]), "elapsed");
  if (ms_forward) *ms_forward = a;
  if (ms_reverse) *ms_reverse = r;
  return GETM_OK;
}

}  // namespace

extern "C" {

int getm_tracer_step_record(getm_ctx* ctx, double dt, double* f, const double* uu, const double* vv,
                            const double* ww, const double* hu, const double* hv, const double* ho, const double* hn,
                            const double* nuh, int split, int hscheme, int vscheme, double AH, double cnpar,
                            double avmol, uint8_t* tape_codes, double* tape_g) {
  return record_api<double>(ctx, dt, f, uu, vv, ww, hu, hv, ho, hn, nuh, split, hscheme, vscheme, AH, cnpar, avmol,
                            tape_codes, tape_g);
}
int getm_tracer_step_record_f32(getm_ctx* ctx, float dt, float* f, const float* uu, const float* vv,
                                const float* ww, const float* hu, const float* hv, const float* ho, const float* hn,
                                const float* nuh, int split, int hscheme, int vscheme, float AH, float cnpar,
                                float avmol, uint8_t* tape_codes, float* tape_g) {
  return record_api<float>(ctx, dt, f, uu, vv, ww, hu, hv, ho, hn, nuh, split, hscheme, vscheme, AH, cnpar, avmol,
                           tape_codes, tape_g);
}
int getm_tracer_step_adjoint(getm_ctx* ctx, double dt, double* fbar, double* nubar, const double* uu,
                             const double* vv, const double* ww, const double* hu, const double* hv, const double* ho,
                             const double* hn, const double* nuh, int split, int hscheme, int vscheme, double AH,
                             double cnpar, double avmol, const uint8_t* tape_codes, const double* tape_g) {
  return adjoint_api<double>(ctx, dt, fbar, nubar, uu, vv, ww, hu, hv, ho, hn, nuh, split, hscheme, vscheme, AH,
                             cnpar, avmol, tape_codes, tape_g);
}
int getm_tracer_step_adjoint_f32(getm_ctx* ctx, float dt, float* fbar, float* nubar, const float* uu,
                                 const float* vv, const float* ww, const float* hu, const float* hv, const float* ho,
                                 const float* hn, const float* nuh, int split, int hscheme, int vscheme, float AH,
                                 float cnpar, float avmol, const uint8_t* tape_codes, const float* tape_g) {
  return adjoint_api<float>(ctx, dt, fbar, nubar, uu, vv, ww, hu, hv, ho, hn, nuh, split, hscheme, vscheme, AH,
                            cnpar, avmol, tape_codes, tape_g);
}
int getm_tracer_gradient(getm_ctx* ctx, int nsteps, int every, double dt, double* f, const double* uu,
                         const double* vv, const double* ww, const double* hu, const double* hv, const double* ho,
                         const double* hn, const double* nuh, int split, int hscheme, int vscheme, double AH,
                         double cnpar, double avmol, double* fbar, double* nubar, float* ms_forward,
                         float* ms_reverse) {
  return gradient_api<double>(ctx, nsteps, every, dt, f, uu, vv, ww, hu, hv, ho, hn, nuh, split, hscheme, vscheme,
                              AH, cnpar, avmol, fbar, nubar, ms_forward, ms_reverse);
}
int getm_tracer_gradient_f32(getm_ctx* ctx, int nsteps, int every, float dt, float* f, const float* uu,
                             const float* vv, const float* ww, const float* hu, const float* hv, const float* ho,
                             const float* hn, const float* nuh, int split, int hscheme, int vscheme, float AH,
                             float cnpar, float avmol, float* fbar, float* nubar, float* ms_forward,
                             float* ms_reverse) {
  return gradient_api<float>(ctx, nsteps, every, dt, f, uu, vv, ww, hu, hv, ho, hn, nuh, split, hscheme, vscheme,
                             AH, cnpar, avmol, fbar, nubar, ms_forward, ms_reverse);
}

}  // extern "C"
