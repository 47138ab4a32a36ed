// ctx_internal.h -- the context object and helpers shared by the host-side units (ctx.cu, bc.cu).
#pragma once
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"
#include "launch.h"

#define GB_NCOUNTERS 8

namespace gb {
enum MaskPlane { P_UPDATEH = 0, P_UFLUX, P_VFLUX, P_XFLUX, P_UUPDATEU, P_VUPDATEV, P_UFLUX_U, P_VFLUX_V, NPLANES };

static inline long long n2d(const Dev& d) { return d.sj * (long long)d.nj(); }
static inline long long n3d(const Dev& d) { return d.sk * (long long)(d.kmax + 1); }
}  // namespace gb

struct getm_ctx {
  getm_domain dom;
  gb::Dev dev;
  cudaStream_t stream = nullptr;
  int device = 0;
  uint8_t* planes = nullptr;   // 8 byte masks of init_advection, n2d each (see MaskPlane)
  int32_t* zmask = nullptr;    // copies of az, au, av (n2d each)
  bool adv_ready = false;
  void* scr[3] = {nullptr, nullptr, nullptr};  // 3D scratch: tracer ping-pong, hi, adv
  size_t scr_bytes = 0;
  double* red = nullptr;                // reduction partials (2*RED_BLOCKS) + result (2)
  // device counters: [0] warnings, [1] range-check count, [2] slow bottom-friction log checks,
  // [3..5] the elevation NaN sweep of the micro steps (findings, last index + 1, latch)
  unsigned long long* cnt = nullptr;
  bool nan_swept = false;  // a NaN sweep was launched since its counters were last read
  // FP64 staging buffer of the restart-field transfers (getm_restart_read / _write)
  double* stage = nullptr;
  size_t stage_bytes = 0;
  std::string err;
  // per-stage device timers (the counterpart of getm_timers' tic/toc, getm_timers.F90:275-357)
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending[GETM_NTIMERS];
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
  double total_ms[GETM_NTIMERS] = {};
  long long launches[GETM_NTIMERS] = {};
  // scratch of the mode-split step: 3D temporaries of uv_advect_3d and the internal pressure
  // (NB3 arrays of bc_scr3_elem bytes per element) and 2D temporaries (NB2 FP64 arrays)
  void* bc_scr3 = nullptr;
  size_t bc_scr3_bytes = 0;
  double* bc_scr2 = nullptr;
  // the macro step's column heights (NCOLH 2D arrays of the 3D fields' type, run_col_heights),
  // read by the advection and diffusion launches after sigma_coordinates in place of the 3D heights
  void* colh = nullptr;
  // FP32 working copies of the 2D fields of the mixed-precision micro step (NF2 slots of n2d
  // floats; only the is_work2 fields are used)
  float* w2 = nullptr;
  // scratch of the tracer adjoint: ADJ_NSCR 3D arrays (adjoint.cu) and the checkpoints and tapes
  // of the checkpointed gradient
  void* adj_scr = nullptr;
  size_t adj_scr_bytes = 0;
  void* adj_store = nullptr;
  size_t adj_store_bytes = 0;
  // open boundaries (getm_set_open_boundaries): boundary points and mirror copies, device arrays
  struct Bdy {
    int npoints = 0;
    int side_first[5] = {0, 0, 0, 0, 0};  // points of side s: [side_first[s], side_first[s+1])
    int4* pts = nullptr;                   // (i, j, type, side) per point, reference indices
    double *data = nullptr, *data_u = nullptr, *data_v = nullptr, *amp = nullptr, *phase = nullptr;
    bool harmonic = false;
    double period = 0.0;
    int ramp = -1;
    // mirror copies (dst, src 2D offsets) per tag (0 U, 1 V, 2 H/D) and side
    long long* pairs = nullptr;
    int pair_first[3][5] = {};
  } bdy;
  bool has_bdy = false;
};

namespace {
// Records a CUDA event pair around one launch when timing is enabled.
struct TimerScope {
  getm_ctx* c;
  int slot;
  std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
  TimerScope(getm_ctx* c_, int slot_) : c(c_), slot(slot_) {
    if (!c || !c->timing) return;
    if (!c->pool.empty()) {
      ev = c->pool.back();
      c->pool.pop_back();
    } else {
      cudaEventCreate(&ev.first);
      cudaEventCreate(&ev.second);
    }
    cudaEventRecord(ev.first, c->stream);
  }
  ~TimerScope() {
    if (!ev.first) return;
    cudaEventRecord(ev.second, c->stream);
    c->pending[slot].push_back(ev);
  }
};
}  // namespace


using namespace gb;

static inline int fail(getm_ctx* c, int code, const char* what) {
  if (c) c->err = what;
  return code;
}

static inline int cuda_fail(getm_ctx* c, int e, const char* where) {
  if (e == 0) return GETM_OK;
  if (c) c->err = std::string(where) + ": " + cudaGetErrorString((cudaError_t)e);
  return GETM_ERR_CUDA;
}

#define GB_TRY(expr, where)                                   \
  do {                                                        \
    int _e = (int)(expr);                                     \
    if (_e != 0) return cuda_fail(ctx, _e, where);            \
  } while (0)

#define GB_TIMED(slot, expr, where)                           \
  do {                                                        \
    TimerScope _ts(ctx, slot);                                \
    int _e = (int)(expr);                                     \
    if (_e != 0) return cuda_fail(ctx, _e, where);            \
  } while (0)

static inline int ensure_scratch(getm_ctx* ctx, size_t bytes) {
  if (ctx->scr_bytes >= bytes) return GETM_OK;
  for (auto& p : ctx->scr) {
    if (p) cudaFree(p);
    p = nullptr;
  }
  ctx->scr_bytes = 0;
  for (auto& p : ctx->scr)
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, GETM_ERR_NOMEM, "scratch allocation failed");
    }
  ctx->scr_bytes = bytes;
  return GETM_OK;
}

static inline bool grid_for_tag(const getm_ctx* ctx, int tag, getm_adv_grid* g) {
  const long long n = n2d(ctx->dev);
  const uint8_t* P = ctx->planes;
  const int32_t* az = ctx->zmask;
  const int32_t* au = ctx->zmask + n;
  const int32_t* av = ctx->zmask + 2 * n;
  switch (tag) {
    case GETM_H_TAG:
    case GETM_D_TAG:
    case GETM_W_TAG:
      *g = {P + P_UFLUX * n, P + P_VFLUX * n, P + P_UPDATEH * n, P + P_UPDATEH * n, P + P_UPDATEH * n, az};
      return true;
    case GETM_U_TAG:
      *g = {P + P_UFLUX_U * n, P + P_XFLUX * n, P + P_UUPDATEU * n, P + P_UFLUX * n, P + P_UFLUX * n, au};
      return true;
    case GETM_V_TAG:
      *g = {P + P_XFLUX * n, P + P_VFLUX_V * n, P + P_VFLUX * n, P + P_VUPDATEV * n, P + P_VFLUX * n, av};
      return true;
    default:
      return false;
  }
}


// do_advection_3d (advection_3d.F90:120-598) on device pointers; defined in ctx.cu. lo: the
// tracer's compensated storage (FP32, FULLSPLIT / HALFSPLIT; null = none). h2d: bit 0 hu, bit 1 hv,
// bit 2 ho are 2D arrays of values shared by every level of a column (FULLSPLIT / HALFSPLIT only).
template <class R>
int do_adv3d(getm_ctx* ctx, R dt, R* f, const R* uu, const R* vv, const R* ww, const R* hu, const R* hv,
             const R* ho, const R* hn, int split, int hs, int vs, R AH, int tag, R* hires, R* advres, int iters,
             bool field_out = true, __half* lo = nullptr, unsigned h2d = 0);
// Two tracers advected together with HALFSPLIT on the H grid (ctx.cu); the caller has checked that
// hs is a split scheme, vs a split scheme or NOADV, and adv_ver_iterations = 1.
template <class R>
int do_adv3d_pair(getm_ctx* ctx, R dt, R* fa, R* fb, const R* uu, const R* vv, const R* ww, const R* hu,
                  const R* hv, const R* ho, int hs, int vs, R AH, __half* lo_a = nullptr, __half* lo_b = nullptr,
                  unsigned h2d = 0);

// Tracer step: do_advection_3d(H_TAG) then the implicit vertical diffusion (ctx.cu).
template <class R>
int tracer_step_impl(getm_ctx* ctx, R dt, R* f, const R* uu, const R* vv, const R* ww, const R* hu, const R* hv,
                     const R* ho, const R* hn, const R* nuh, int split, int hs, int vs, R AH, R cnpar, R avmol,
                     int iters);
