// kernels.cuh -- CUDA kernels of the hot path, templated on the arithmetic type R.
// Instantiated for double in kernels_f64.cu (built without FMA contraction so that every
// expression rounds exactly as the reference's) and for float in kernels_f32.cu.
#pragma once
#include <type_traits>
#include <cuda_fp16.h>
#include "common.cuh"
#include "launch.h"

namespace gb {

// ---------------------------------------------------------------------------------------------
// Horizontal split sweeps (adv_split_u.F90:205-285, adv_split_v.F90:63-135).
//
// The limiter scheme S is a template parameter. FP64 evaluates the reference's expressions in the
// reference's order (bit-identical results, IEEE division). FP32 -- the mixed-precision variant --
// evaluates the same interface values with fewer instructions: the ratio-based limiters are
// rewritten without the ratio (L(r)*deltaf from the magnitudes |deltafu|, |deltaf|, which equals
// the reference's value in exact arithmetic) and the remaining divisions by face quantities use
// the fast reciprocal (__fdividef, <= 2 ulp).

template <class R>
__device__ __forceinline__ R qdiv(R a, R b) {
  if constexpr (sizeof(R) == 4) return __fdividef(a, b);
  else return a / b;
}

// FP32 P2_PDM limiter in scaled form. With w = (1-cfl)/2 > 0 (Courant numbers below 1, the
// stability limit of the split schemes) the reference's candidates 2r/(cfl+1e-10),
// (1/2+x)+(1/2-x)r and 2/(1-cfl) (r = a/b, x = (1-2cfl)/6), multiplied by w*|deltaf| = w*b, are
// v1 = a(1-cfl)/(cfl+1e-10), v2 = w((1/2+x)b + (1/2-x)a) and b itself: the interface value is
// fu + sign(deltaf)*min(v1, v2, b) with one division instead of two (the third branch gives the
// downwind value). Every operation is an explicitly rounded intrinsic, so the branch comparisons
// of recon_code round exactly like the value of recon_s wherever they are inlined.
struct Pdm32 {
  float v1, v2;
};
__device__ __forceinline__ Pdm32 pdm32(float cfl, float a, float b) {
  const float omc = __fsub_rn(1.f, cfl);
  const float x = __fmul_rn(1.f / 6.f, __fsub_rn(1.f, __fmul_rn(2.f, cfl)));
  Pdm32 p;
  p.v1 = __fdividef(__fmul_rn(a, omc), __fadd_rn(cfl, 1.e-10f));
  p.v2 = __fmul_rn(__fmul_rn(0.5f, omc), __fmaf_rn(__fadd_rn(0.5f, x), b, __fmul_rn(__fsub_rn(0.5f, x), a)));
  return p;
}

// Interface value from (fuu, fu, fd) at Courant number cfl (advection.F90:785-879).
template <class R, int S>
__device__ __forceinline__ R recon_s(R cfl, R fuu, R fu, R fd) {
  if constexpr (sizeof(R) == 8) {
    return recon<R>(S, cfl, fuu, fu, fd);
  } else {
    const float df = fd - fu, du = fu - fuu;
    if constexpr (S == P2) {
      const float x = __fmul_rn(1.f / 6.f, __fsub_rn(1.f, __fmul_rn(2.f, cfl)));
      return __fadd_rn(fu, __fmul_rn(__fmul_rn(0.5f, __fsub_rn(1.f, cfl)),
                                     __fadd_rn(__fmul_rn(__fadd_rn(0.5f, x), df), __fmul_rn(__fsub_rn(0.5f, x), du))));
    } else if constexpr (S == SUPERBEE || S == MUSCL || S == P2_PDM) {
      if (!(df * du > 0.f)) return fu;
      const float a = fabsf(du), b = fabsf(df);  // L(r)*|deltaf| with r = a/b
      if constexpr (S == P2_PDM) {
        const Pdm32 p = pdm32(cfl, a, b);
        return fu + copysignf(fminf(fminf(p.v1, p.v2), b), df);
      } else {
        float Lb;
        if constexpr (S == SUPERBEE) Lb = fmaxf(fminf(2.f * a, b), fminf(a, 2.f * b));
        else Lb = fminf(fminf(2.f * a, 0.5f * (b + a)), 2.f * b);
        return __fadd_rn(fu, __fmul_rn(__fmul_rn(0.5f, __fsub_rn(1.f, cfl)), copysignf(Lb, df)));
      }
    } else {
      return fu;
    }
  }
}

// Limiter branch taken by recon_s for one face, for the adjoint (0 = first-order value fu).
//   SUPERBEE: 1 L=2r, 2 L=1, 3 L=r, 4 L=2;  MUSCL: 1 L=2r, 2 L=(1+r)/2, 3 L=2;
//   P2_PDM: 1 L=2r/(cfl+1e-10), 2 L=(1/2+x)+(1/2-x)r, 3 L=2/(1-cfl);  P2: 1.
// The comparisons are those of recon_s (the reference's MIN/MAX order in FP64, the magnitude form
// in FP32), so the code names the branch whose value the forward sweep used.
template <class R, int S>
__device__ __forceinline__ uint8_t recon_code(R cfl, R fuu, R fu, R fd) {
  if constexpr (S == P2) {
    return 1;
  } else if constexpr (S == SUPERBEE || S == MUSCL || S == P2_PDM) {
    const R df = fd - fu, du = fu - fuu;
    if (!(df * du > R(0))) return 0;
    R t1, t2, t3, t4;
    if constexpr (sizeof(R) == 8) {
      const R ratio = du / df;
      if constexpr (S == SUPERBEE) {
        t1 = R(2) * ratio; t2 = R(1); t3 = ratio; t4 = R(2);
      } else if constexpr (S == MUSCL) {
        t1 = R(2) * ratio; t2 = R(0.5) * (R(1) + ratio); t3 = R(2); t4 = R(0);
      } else {
        const R x = (R(1) / R(6)) * (R(1) - R(2) * cfl);
        t2 = (R(0.5) + x) + (R(0.5) - x) * ratio;
        t1 = R(2) * ratio / (cfl + R(1.e-10));
        t3 = R(2) / (R(1) - cfl); t4 = R(0);
      }
    } else {
      const float a = fabsf(du), b = fabsf(df);
      if constexpr (S == SUPERBEE) {
        t1 = 2.f * a; t2 = b; t3 = a; t4 = 2.f * b;
      } else if constexpr (S == MUSCL) {
        t1 = 2.f * a; t2 = 0.5f * (b + a); t3 = 2.f * b; t4 = 0.f;
      } else {  // the scaled candidates of recon_s (pdm32): the same order as t1, t2, t3
        const Pdm32 p = pdm32(cfl, a, b);
        t1 = p.v1; t2 = p.v2; t3 = b; t4 = 0.f;
      }
    }
    if constexpr (S == SUPERBEE) {
      const R m1 = (t2 < t1) ? t2 : t1, m2 = (t4 < t3) ? t4 : t3;
      const uint8_t c1 = (t2 < t1) ? 2 : 1, c2 = (t4 < t3) ? 4 : 3;
      return (m2 > m1) ? c2 : c1;
    } else {
      (void)t4;
      const R m = (t2 < t1) ? t2 : t1;
      const uint8_t c = (t2 < t1) ? 2 : 1;
      return (t3 < m) ? 3 : c;
    }
  } else {
    (void)cfl; (void)fuu; (void)fu; (void)fd;
    return 0;
  }
}

// Derivative of the interface value fu + A*(fu-fuu) + B*(fd-fu) for limiter branch `code`
// (the frozen-branch linearisation of recon_s).
template <class R, int S>
__device__ __forceinline__ void recon_coef(uint8_t code, R cfl, R& A, R& B) {
  A = R(0);
  B = R(0);
  if (code == 0) return;
  const R omc = R(1) - cfl;
  if constexpr (S == SUPERBEE) {
    if (code == 1) A = omc;
    else if (code == 2) B = R(0.5) * omc;
    else if (code == 3) A = R(0.5) * omc;
    else B = omc;
  } else if constexpr (S == MUSCL) {
    if (code == 1) A = omc;
    else if (code == 2) A = B = R(0.25) * omc;
    else B = omc;
  } else if constexpr (S == P2_PDM || S == P2) {
    if (S == P2 || code == 2) {
      const R x = (R(1) / R(6)) * (R(1) - R(2) * cfl);
      A = R(0.5) * omc * (R(0.5) - x);
      B = R(0.5) * omc * (R(0.5) + x);
    } else if (code == 1) {
      A = omc / (cfl + R(1.e-10));
    } else {
      B = R(1);
    }
  }
}

// Finite-volume update of one cell after a split step: hin = hio - dh is the new layer height and
// advn the flux divergence (adv_split_u.F90:274-279, adv_split_w.F90:289-292).
// FP64 keeps the reference's form (hio*fio - dt*advn)/hin, bit for bit. FP32 evaluates the same
// quantity as an increment, fio + (fio*dh - dt*advn)/hin: the rounding then acts on the small
// increment instead of on hio*fio, which removes the bias that (hio*fio)/hin carries in still water
// and keeps the FP32 tracer within ~1e-6 of FP64 over hundreds of steps.
template <class R>
__device__ __forceinline__ R fv_update(R hio, R dh, R hin, R fio, R dt, R advn) {
  if constexpr (sizeof(R) == 8) {
    (void)dh;
    return (hio * fio - dt * advn) / hin;
  } else {
    (void)hio;
    return __fadd_rn(fio, __fdividef(__fmaf_rn(fio, dh, -__fmul_rn(dt, advn)), hin));
  }
}

// Compensated storage of an FP32 tracer (the mixed step): the tracer is the unevaluated sum
// hi + lo of two FP32 numbers. An update adds its increment and the carried lo to hi exactly
// (Knuth's TwoSum): hi becomes the rounded sum and lo the rounding error, so increments smaller
// than half an ulp of hi -- which a plain FP32 update drops, and which a tracer far from zero
// (temperature near 15 C, salinity near 35) receives every sweep -- accumulate in lo until they
// reach hi instead of being lost. |lo| stays below half an ulp of hi. The fluxes are formed from
// hi alone, as in the plain update.
__device__ __forceinline__ float add_comp(float hi, float inc, float& lo) {
  const float b = __fadd_rn(inc, lo);
  const float s = __fadd_rn(hi, b);
  const float bb = __fsub_rn(s, hi);
  lo = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return s;
}
// The carried error is stored in FP16 as lo * 2^16 (an exact power-of-two scaling): |lo| <= half an
// ulp of hi, so the stored value stays below 1 for |hi| < 2^24 and keeps lo to 11 bits wherever it
// is a normal FP16 number (|lo| >= 2^-30, i.e. |hi| above about 2^-7; below, the tracer's own FP32
// spacing is already that fine); the tracer then holds about 35 significant bits in 6 bytes.
constexpr float LO_ENC = 65536.f, LO_DEC = 1.f / 65536.f;
// hi + inc with the carried error given as its stored (scaled) value slo
__device__ __forceinline__ float add_comp_scaled(float hi, float inc, float& slo) {
  float lo = __fmul_rn(slo, LO_DEC);
  const float s = add_comp(hi, inc, lo);
  slo = __fmul_rn(lo, LO_ENC);
  return s;
}
// fv_update with the compensated storage; slo: the cell's scaled carried error (read and written)
template <class R>
__device__ __forceinline__ R fv_update_lo(R hio, R dh, R hin, R fio, R dt, R advn, float& slo) {
  if constexpr (sizeof(R) == 8) {
    (void)slo;
    return fv_update<R>(hio, dh, hin, fio, dt, advn);
  } else {
    (void)hio;
    return add_comp_scaled(fio, __fdividef(__fmaf_rn(fio, dh, -__fmul_rn(dt, advn)), hin), slo);
  }
}
// the same on the FP16 array of the carried errors at element p
template <class R>
__device__ __forceinline__ R fv_update_lo(R hio, R dh, R hin, R fio, R dt, R advn, __half* lo, long long p) {
  float slo = __half2float(lo[p]);
  const R v = fv_update_lo<R>(hio, dh, hin, fio, dt, advn, slo);
  lo[p] = __float2half_rn(slo);
  return v;
}

// Flux through face q (between cells q and q+1) from staged values: f at q-1..q+2, flux masks at
// q-1..q+1. cdx = dti/dx (used by FP32 only).
// Courant number of a horizontal face (adv_split_u.F90:229-246); cdx = dti/dx is used by FP32.
template <class R>
__device__ __forceinline__ R face_cfl(bool pos, R Uf, R DUf, R dti, R cdx, R dxf) {
  if constexpr (sizeof(R) == 8) {
    (void)cdx;
    return pos ? Uf / DUf * dti / dxf : -Uf / DUf * dti / dxf;
  } else {
    (void)dti; (void)dxf;
    return __fdividef(fabsf(Uf) * cdx, DUf);
  }
}

// With REC the limiter branch is written to *code (0 when the face is not limited).
// FP32 without branch recording: the same values computed without branches (every candidate is
// evaluated and the result selected), so the lanes of a warp do not diverge on the masks, the
// flow direction or the limiter's extremum test; the operations and their rounding are those of
// the branching form below.
template <int S>
__device__ __forceinline__ float face_flux_f32(float Uf, float DUf, float fm1, float f0, float f1, float f2,
                                               bool mm1, bool m0, bool mp1, float cdx, float AH, bool use_AH,
                                               float dxf) {
  const bool pos = Uf > 0.f;
  float fu = pos ? f0 : f1;
  if constexpr (S != UPSTREAM) {
    const float fuu = pos ? fm1 : f2;
    const float fd = pos ? f1 : f0;
    const bool lim = pos ? mm1 : mp1;
    const float cfl = __fdividef(fabsf(Uf) * cdx, DUf);
    float val;
    if constexpr (S == P2_PDM) {
      const float df = fd - fu, du = fu - fuu;
      const Pdm32 p = pdm32(cfl, fabsf(du), fabsf(df));
      const float v = fu + copysignf(fminf(fminf(p.v1, p.v2), fabsf(df)), df);
      val = (df * du > 0.f) ? v : fu;
    } else {
      val = recon_s<float, S>(cfl, fuu, fu, fd);
    }
    fu = lim ? val : fu;
  }
  float fl = Uf * fu;
  if (use_AH) fl = fl - AH * DUf * (f1 - f0) / dxf;
  return m0 ? fl : 0.f;
}

template <class R, int S, bool REC = false>
__device__ __forceinline__ R face_flux_s(R Uf, R DUf, R fm1, R f0, R f1, R f2, bool mm1, bool m0, bool mp1,
                                         R dti, R cdx, R AH, bool use_AH, R dxf, uint8_t* code = nullptr) {
  if constexpr (sizeof(R) == 4 && !REC) {
    (void)dti; (void)code;
    return face_flux_f32<S>(Uf, DUf, fm1, f0, f1, f2, mm1, m0, mp1, cdx, AH, use_AH, dxf);
  }
  if (REC) *code = 0;
  if (!m0) return R(0);
  const bool pos = Uf > R(0);
  R fu = pos ? f0 : f1;
  if (S != UPSTREAM && (pos ? mm1 : mp1)) {
    const R fuu = pos ? fm1 : f2;
    const R fd = pos ? f1 : f0;
    const R cfl = face_cfl<R>(pos, Uf, DUf, dti, cdx, dxf);
    if (REC) *code = recon_code<R, S>(cfl, fuu, fu, fd);
    fu = recon_s<R, S>(cfl, fuu, fu, fd);
  }
  R fl = Uf * fu;
  if (use_AH) fl = fl - AH * DUf * (f1 - f0) / dxf;
  return fl;
}

// Tiled sweeps: a block stages the stencil source f, the face transports/heights and the flux
// masks of its tile in shared memory, computes each face flux of the tile once into shared memory
// and then updates its cells. A cell in the update range with mask_update takes fi/Di from the
// sources, every other cell copies them through when source and destination differ. f must not
// alias fi_dst (callers ping-pong); fi_src may be f or alias fi_dst, Di_src may alias Di_dst.
constexpr int TU = 128;             // u sweep: threads (faces) per block along i
constexpr int OWU = TU - 1;         // u sweep: cells updated per block
constexpr int TVX = 32, TVY = 8;    // v sweep: tile of 32 (i) x 8 (j) cells
constexpr int NKB = 8;              // levels per block (the 2D masks are staged once for them)

// Constants of one sweep, computed on the host in R (the same IEEE operations the reference
// performs per cell, so FP64 results are unchanged): dti = splitfac*dt, dxf = the face spacing
// along the sweep (DXU / DYV), dyf = the face width (DYU / DXV), cdx = dti/dxf.
template <class R>
struct SweepC {
  R dt, splitfac, AH, dti, dxf, dyf, ard1, cdx;
  R cdy, cadv;   // FP32 cell update: dti*dyf*ard1 and splitfac*dyf*ard1
  int adv_init;  // vectorised u sweep: start the flux-divergence sum adv instead of adding to it
  // level strides of the face depths (DU / DV) and of the heights read (Di_src): the 3D level
  // stride, or 0 for a 2D array of values that every level of a column shares (the layer heights
  // of equidistant sigma coordinates)
  long long skdu, skdi;
};

template <class R>
inline SweepC<R> sweep_consts(const Dev& d, int dir, R dt, R splitfac, R AH) {
  SweepC<R> c;
  c.dt = dt;
  c.splitfac = splitfac;
  c.AH = AH;
  c.dti = splitfac * dt;
  c.dxf = dir == 0 ? R(d.dx) : R(d.dy);
  c.dyf = dir == 0 ? R(d.dy) : R(d.dx);
  c.ard1 = R(d.ard1);
  c.cdx = c.dti / c.dxf;
  c.cdy = c.dti * c.dyf * c.ard1;
  c.cadv = splitfac * c.dyf * c.ard1;
  c.adv_init = 0;
  c.skdu = c.skdi = d.sk;
  return c;
}

// Height decrement and flux divergence of a cell between its faces lo and hi
// (adv_split_u.F90:274-276). FP64: the reference's expressions. FP32: one difference times a
// host constant, with explicitly rounded operations, so every sweep kernel that calls these
// rounds identically (no compiler-chosen contraction).
template <class R>
__device__ __forceinline__ R cell_dD(const SweepC<R>& C, R Uhi, R Ulo) {
  if constexpr (sizeof(R) == 8) return C.dti * (Uhi * C.dyf - Ulo * C.dyf) * C.ard1;
  else return __fmul_rn(__fsub_rn(Uhi, Ulo), C.cdy);
}
template <class R>
__device__ __forceinline__ R cell_advn(const SweepC<R>& C, R flhi, R fllo) {
  if constexpr (sizeof(R) == 8) return C.splitfac * (flhi * C.dyf - fllo * C.dyf) * C.ard1;
  else return __fmul_rn(__fsub_rn(flhi, fllo), C.cadv);
}

// The tracer fields of one sweep: the stencil source f, the field fi updated from fi_src into
// fi_dst (fi_src may be f or alias fi_dst). A sweep advects NF fields with the same transports,
// heights and masks -- temperature and salinity share them, so they are swept together: the
// layer heights, Courant numbers and masks are read and computed once for both.
template <class R>
struct TracerIO {
  const R* f;
  const R* fi_src;
  R* fi_dst;
  __half* lo = nullptr;  // FP32 compensated storage: the cells' scaled carried errors (may be null)
};
template <class R, int NF>
struct TracerSet {
  TracerIO<R> t[NF];
};

// Asynchronous global -> shared copies (cp.async, 4 or 8 bytes): the tile sweeps stage level k+1
// while they compute level k, so the loads of the next level are in flight during the face and
// update phases instead of stalling every warp at the start of each level.
template <class R>
__device__ __forceinline__ void cp_async(R* smem, const R* gmem) {
  static_assert(sizeof(R) == 4 || sizeof(R) == 8, "cp_async: 4 or 8 bytes");
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(sizeof(R)) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// u sweep (adv_split_u.F90:222-285) over one row segment, for up to NKB levels. The TU threads
// compute the TU faces i0-1 .. i0+TU-2 (one each) and update the OWU = TU-1 cells between them,
// so no warp computes a second face. Levels are double-buffered in shared memory: the copies of
// level k+1 (stencil source, transports, heights, own-cell inputs) are issued before level k is
// computed.
template <class R, int S, bool REC, int NF>
__global__ void __launch_bounds__(TU, sizeof(R) == 4 ? 16 : 8) k_sweep_u_tile(Dev d, SweepC<R> C, int nk, TracerSet<R, NF> F,
                                                     const R* Di_src, R* Di_dst, R* adv,
                                                     const R* __restrict__ U, const R* __restrict__ DU,
                                                     const uint8_t* __restrict__ mflux,
                                                     const uint8_t* __restrict__ mupd, uint8_t* code) {
  __shared__ R sf[2][NF][TU + 3];   // f(i0-2 .. i0+TU)
  __shared__ R sU[2][TU];           // U(i0-1 .. i0+TU-2)
  __shared__ R sDU[2][TU];
  __shared__ R sD[2][TU];           // Di_src of the own cells
  __shared__ R sfi[2][NF][TU];      // fi_src of the own cells (when it is not f)
  __shared__ R sA[2][TU];           // adv of the own cells (momentum sweeps)
  __shared__ uint8_t sm[TU + 3];    // mflux(i0-2 .. i0+TU)
  __shared__ R sfl[NF][TU];         // flux of faces i0-1 .. i0+TU-2
  const int t = threadIdx.x;
  const int ni = d.ni();
  const int ii0 = blockIdx.x * OWU;
  const long long crow = (long long)blockIdx.y * d.sj;
  const int k0 = blockIdx.z * NKB;
  const int k1 = min(k0 + NKB, nk);
  constexpr int sub = (S == UPSTREAM) ? 0 : 1;
  const bool use_AH = C.AH > R(0);
  // masks of the row (levels share them)
  for (int q = t; q < TU + 3; q += TU) {
    const int ii = ii0 - 2 + q;
    sm[q] = (ii >= 0 && ii < ni) ? mflux[crow + ii] : 0;
  }
  const int ii = ii0 + t;
  const bool own = t < OWU && ii < ni;
  const bool upd = own && (ii >= 1 + sub) && (ii <= ni - 2 - sub) && mupd[crow + ii];
  // tiles away from the ends of the row stage without bounds checks
  const bool inner = ii0 >= 2 && ii0 + TU + 1 <= ni;
  auto stage = [&](int k, int b) {
    const long long row = crow + (long long)k * d.sk;
    const R* Ur = U + row;
    const R* DUr = DU + crow + (long long)k * C.skdu;
    if (inner) {
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        const R* fr = F.t[n].f + row + (ii0 - 2);
        cp_async(&sf[b][n][t], fr + t);
        if (t < 3) cp_async(&sf[b][n][TU + t], fr + TU + t);
      }
      cp_async(&sU[b][t], Ur + ii0 - 1 + t);
      cp_async(&sDU[b][t], DUr + ii0 - 1 + t);
    } else {
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        const R* fr = F.t[n].f + row;
        for (int q = t; q < TU + 3; q += TU) {
          const int i2 = ii0 - 2 + q;
          if (i2 >= 0 && i2 < ni) cp_async(&sf[b][n][q], fr + i2);
          else sf[b][n][q] = R(0);
        }
      }
      const int i2 = ii0 - 1 + t;
      if (i2 >= 0 && i2 < ni) {
        cp_async(&sU[b][t], Ur + i2);
        cp_async(&sDU[b][t], DUr + i2);
      } else {
        sU[b][t] = R(0);
        sDU[b][t] = R(0);
      }
    }
    if (own) {
      cp_async(&sD[b][t], Di_src + crow + (long long)k * C.skdi + ii);
#pragma unroll
      for (int n = 0; n < NF; ++n)
        if (F.t[n].fi_src != F.t[n].f) cp_async(&sfi[b][n][t], F.t[n].fi_src + row + ii);
      if (NF == 1 && adv && upd) cp_async(&sA[b][t], adv + row + ii);
    }
    cp_async_commit();
  };
  if (k0 < k1) stage(k0, 0);
  for (int k = k0, b = 0; k < k1; ++k, b ^= 1) {
    const long long row = crow + (long long)k * d.sk;
    if (k + 1 < k1) {
      stage(k + 1, b ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    {
      const int q = t;
      const int fa = ii0 - 1 + q;
      const bool valid = fa >= sub && fa <= ni - 2 - sub;
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        R fl = R(0);
        uint8_t cd = 0;
        if (valid)
          fl = face_flux_s<R, S, REC>(sU[b][q], sDU[b][q], sf[b][n][q], sf[b][n][q + 1], sf[b][n][q + 2],
                                      sf[b][n][q + 3], sm[q] != 0, sm[q + 1] != 0, sm[q + 2] != 0, C.dti, C.cdx,
                                      C.AH, use_AH, C.dxf, &cd);
        sfl[n][q] = fl;
        if (REC && n == 0 && q >= 1 && fa < ni) code[row + fa] = cd;  // face fa is stored at its left cell
      }
    }
    __syncthreads();
    if (own) {
      const long long p = row + ii;
      const R Dio = sD[b][t];
      if (upd) {
        const R dD = cell_dD<R>(C, sU[b][t + 1], sU[b][t]);
        const R Dn = Dio - dD;
        if (Di_dst) Di_dst[p] = Dn;
#pragma unroll
        for (int n = 0; n < NF; ++n) {
          const R fio = F.t[n].fi_src == F.t[n].f ? sf[b][n][t + 2] : sfi[b][n][t];
          const R advn = cell_advn<R>(C, sfl[n][t + 1], sfl[n][t]);
          if (F.t[n].fi_dst) {
            if (F.t[n].lo) {
              F.t[n].fi_dst[p] = fv_update_lo<R>(Dio, dD, Dn, fio, C.dt, advn, F.t[n].lo, p);
            } else {
              F.t[n].fi_dst[p] = fv_update<R>(Dio, dD, Dn, fio, C.dt, advn);
            }
          }
          if (NF == 1 && adv) adv[p] = sA[b][t] + advn;
        }
      } else {
#pragma unroll
        for (int n = 0; n < NF; ++n)
          if (F.t[n].fi_dst && F.t[n].fi_dst != F.t[n].fi_src)
            F.t[n].fi_dst[p] = F.t[n].fi_src == F.t[n].f ? sf[b][n][t + 2] : sfi[b][n][t];
        if (Di_dst && Di_dst != Di_src) Di_dst[p] = Dio;
      }
    }
    __syncthreads();  // buffer b and sfl are restaged / rewritten for level k+2 / k+1
  }
}

// v sweep (adv_split_v.F90:79-135) over a tile of TVX x TVY cells, for up to NKB levels, with the
// levels double-buffered in shared memory like the u sweep.
template <class R, int S, bool REC, int NF>
__global__ void __launch_bounds__(TVX * TVY, sizeof(R) == 4 ? (NF == 1 ? 8 : 6) : (NF == 1 ? 4 : 3))
    k_sweep_v_tile(Dev d, SweepC<R> C, int nk, TracerSet<R, NF> F, const R* Di_src, R* Di_dst, R* adv,
                   const R* __restrict__ V, const R* __restrict__ DV, const uint8_t* __restrict__ mflux,
                   const uint8_t* __restrict__ mupd, uint8_t* code) {
  __shared__ R sf[2][NF][TVY + 4][TVX];  // f(j0-2 .. j0+TVY+1)
  __shared__ R sV[2][TVY + 1][TVX];      // V(j0-1 .. j0+TVY-1)
  __shared__ R sDV[2][TVY + 1][TVX];
  __shared__ R sD[2][TVY][TVX];          // Di_src of the own cells
  __shared__ R sfi[2][NF][TVY][TVX];     // fi_src of the own cells (when it is not f)
  __shared__ R sA[2][TVY][TVX];          // adv of the own cells (momentum sweeps)
  __shared__ uint8_t sm[TVY + 4][TVX];   // mflux(j0-2 .. j0+TVY+1)
  __shared__ R sfl[NF][TVY + 1][TVX];    // flux of faces j0-1 .. j0+TVY-1
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int ni = d.ni(), nj = d.nj();
  const int ii = blockIdx.x * TVX + tx;
  const int jj0 = blockIdx.y * TVY;
  const int k0 = blockIdx.z * NKB;
  const int k1 = min(k0 + NKB, nk);
  const bool iok = ii < ni;
  const long long sj = d.sj;
  constexpr int sub = (S == UPSTREAM) ? 0 : 1;
  const bool use_AH = C.AH > R(0);
  for (int q = ty; q < TVY + 4; q += TVY) {
    const int jj = jj0 - 2 + q;
    sm[q][tx] = (iok && jj >= 0 && jj < nj) ? mflux[(long long)jj * sj + ii] : 0;
  }
  const int jj = jj0 + ty;
  const bool own = iok && jj < nj;
  const long long c = (long long)jj * sj + ii;
  const bool upd = own && (jj >= 1 + sub) && (jj <= nj - 2 - sub) && mupd[c];
  // tiles away from the ends of the columns stage without bounds checks
  const bool inner = iok && jj0 >= 2 && jj0 + TVY + 2 <= nj;
  auto stage = [&](int k, int b) {
    const long long lev = (long long)k * d.sk;
    if (inner) {
      const long long b0 = lev + (long long)(jj0 - 2) * sj + ii;  // row jj0-2 of this column
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        const R* fc = F.t[n].f + b0;
        cp_async(&sf[b][n][ty][tx], fc + (long long)ty * sj);
        if (ty < 4) cp_async(&sf[b][n][TVY + ty][tx], fc + (long long)(TVY + ty) * sj);
      }
      const R* Vc = V + b0 + sj;  // row jj0-1
      const R* DVc = DV + (b0 - lev + (long long)k * C.skdu) + sj;
      cp_async(&sV[b][ty][tx], Vc + (long long)ty * sj);
      cp_async(&sDV[b][ty][tx], DVc + (long long)ty * sj);
      if (ty == 0) {
        cp_async(&sV[b][TVY][tx], Vc + (long long)TVY * sj);
        cp_async(&sDV[b][TVY][tx], DVc + (long long)TVY * sj);
      }
    } else {
#pragma unroll
      for (int n = 0; n < NF; ++n)
        for (int q = ty; q < TVY + 4; q += TVY) {
          const int j2 = jj0 - 2 + q;
          if (iok && j2 >= 0 && j2 < nj) cp_async(&sf[b][n][q][tx], F.t[n].f + lev + (long long)j2 * sj + ii);
          else sf[b][n][q][tx] = R(0);
        }
      for (int q = ty; q < TVY + 1; q += TVY) {
        const int j2 = jj0 - 1 + q;
        if (iok && j2 >= 0 && j2 < nj) {
          const long long c2 = lev + (long long)j2 * sj + ii;
          cp_async(&sV[b][q][tx], V + c2);
          cp_async(&sDV[b][q][tx], DV + (c2 - lev + (long long)k * C.skdu));
        } else {
          sV[b][q][tx] = R(0);
          sDV[b][q][tx] = R(0);
        }
      }
    }
    if (own) {
      cp_async(&sD[b][ty][tx], Di_src + (long long)k * C.skdi + c);
#pragma unroll
      for (int n = 0; n < NF; ++n)
        if (F.t[n].fi_src != F.t[n].f) cp_async(&sfi[b][n][ty][tx], F.t[n].fi_src + lev + c);
      if (NF == 1 && adv && upd) cp_async(&sA[b][ty][tx], adv + lev + c);
    }
    cp_async_commit();
  };
  if (k0 < k1) stage(k0, 0);
  for (int k = k0, b = 0; k < k1; ++k, b ^= 1) {
    const long long lev = (long long)k * d.sk;
    if (k + 1 < k1) {
      stage(k + 1, b ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    for (int q = ty; q < TVY + 1; q += TVY) {
      const int fa = jj0 - 1 + q;
      const bool valid = iok && fa >= sub && fa <= nj - 2 - sub;
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        R fl = R(0);
        uint8_t cd = 0;
        if (valid)
          fl = face_flux_s<R, S, REC>(sV[b][q][tx], sDV[b][q][tx], sf[b][n][q][tx], sf[b][n][q + 1][tx],
                                      sf[b][n][q + 2][tx], sf[b][n][q + 3][tx], sm[q][tx] != 0, sm[q + 1][tx] != 0,
                                      sm[q + 2][tx] != 0, C.dti, C.cdx, C.AH, use_AH, C.dxf, &cd);
        sfl[n][q][tx] = fl;
        if (REC && n == 0 && q >= 1 && iok && fa < nj) code[lev + (long long)fa * sj + ii] = cd;
      }
    }
    __syncthreads();
    if (own) {
      const long long p = lev + c;
      const R Dio = sD[b][ty][tx];
      if (upd) {
        const R dD = cell_dD<R>(C, sV[b][ty + 1][tx], sV[b][ty][tx]);
        const R Dn = Dio - dD;
        if (Di_dst) Di_dst[p] = Dn;
#pragma unroll
        for (int n = 0; n < NF; ++n) {
          const R fio = F.t[n].fi_src == F.t[n].f ? sf[b][n][ty + 2][tx] : sfi[b][n][ty][tx];
          const R advn = cell_advn<R>(C, sfl[n][ty + 1][tx], sfl[n][ty][tx]);
          if (F.t[n].fi_dst) {
            if (F.t[n].lo) {
              F.t[n].fi_dst[p] = fv_update_lo<R>(Dio, dD, Dn, fio, C.dt, advn, F.t[n].lo, p);
            } else {
              F.t[n].fi_dst[p] = fv_update<R>(Dio, dD, Dn, fio, C.dt, advn);
            }
          }
          if (NF == 1 && adv) adv[p] = sA[b][ty][tx] + advn;
        }
      } else {
#pragma unroll
        for (int n = 0; n < NF; ++n)
          if (F.t[n].fi_dst && F.t[n].fi_dst != F.t[n].fi_src)
            F.t[n].fi_dst[p] = F.t[n].fi_src == F.t[n].f ? sf[b][n][ty + 2][tx] : sfi[b][n][ty][tx];
        if (Di_dst && Di_dst != Di_src) Di_dst[p] = Dio;
      }
    }
    __syncthreads();  // buffer b and sfl are restaged / rewritten for level k+2 / k+1
  }
}

// ---------------------------------------------------------------------------------------------
// Vertical split sweep (adv_split_w.F90:158-307) without sub-iterations (itersmax = 1):
// one thread per water column, k-sequential, streaming with a register window so that every
// level of f and hi is read before it is overwritten -- f, fi and hi may therefore alias. The
// window reaches two levels ahead of the face being computed so that several loads per thread
// are in flight.
// Courant number of vertical face k (adv_split_w.F90:167-169) from the layer heights around it.
template <class R>
__device__ __forceinline__ R wface_cfl(R w, R dti, R hk, R hkp1) {
  if constexpr (sizeof(R) == 8) return fabs(w) * dti / (R(0.5) * (hk + hkp1));
  else return __fdividef(2.f * fabsf(w) * dti, hk + hkp1);
}

template <class R, int S, bool REC = false>
__device__ __forceinline__ R wface_s(int k, int kshift, int kmax, R dti, R w, R fkm1, R fk, R fkp1, R fkp2,
                                     R hk, R hkp1, uint8_t* code = nullptr) {
  const bool pos = w > R(0);
  R fu = pos ? fk : fkp1;
  if (REC) *code = 0;
  if (S != UPSTREAM && (pos ? (k > 1 - kshift) : (k < kmax - 1))) {
    const R fuu = pos ? fkm1 : fkp2;
    const R fd = pos ? fkp1 : fk;
    const R cfl = wface_cfl<R>(w, dti, hk, hkp1);
    if (REC) *code = recon_code<R, S>(cfl, fuu, fu, fd);
    fu = recon_s<R, S>(cfl, fuu, fu, fd);
  }
  return w * fu;
}

template <class R, int S, bool REC>
__global__ void __launch_bounds__(128) k_sweep_w(Dev d, R dt, R splitfac, int kshift,
                                                 const R* f, const R* fi_src, R* fi_dst, R* hi, R* adv,
                                                 const R* __restrict__ ww,
                                                 const int32_t* __restrict__ az, uint8_t* code, __half* lo = nullptr) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  // columns i = imin-2..imax+1, j = jmin-2..jmax+1 (adv_split_w.F90:160-162)
  if (ii >= d.ni() - 1 || jj >= d.nj() - 1) return;
  const long long c = (long long)ii + (long long)jj * d.sj;
  if (az[c] != 1) return;
  const int kmax = d.kmax;
  const long long sk = d.sk;
  const R dti = splitfac * dt;
  const bool fi_is_f = (fi_src == f);
  auto F = [&](int k) -> R { return (k >= 0 && k <= kmax) ? f[c + k * sk] : R(0); };
  auto H = [&](int k) -> R { return (k >= 0 && k <= kmax) ? hi[c + k * sk] : R(0); };
  auto W = [&](int k) -> R { return (k <= kmax) ? ww[c + k * sk] : R(0); };
  R wprev = R(0);  // wflux(k-1); wflux(0) = 0 unless W_TAG computes face 0
  if (kshift == 1) {
    uint8_t cd = 0;
    wprev = wface_s<R, S, REC>(0, 1, kmax, dti, ww[c], R(0), F(0), F(1), F(2), H(0), H(1), &cd);
    if (REC) code[c] = cd;
  }
  // window for face k = 1: f(0..4), hi(1..3), ww(0..2); the carried errors (compensated storage)
  // of levels 1, 2
  R a = F(0), b = F(1), e = F(2), g = F(3), g2 = F(4);
  R hA = H(1), hB = H(2), hC = H(3);
  R wkm1 = W(0), wk = W(1), wk1 = W(2);
  auto LO = [&](int k) -> float { return (lo && k <= kmax) ? __half2float(lo[c + k * sk]) : 0.f; };
  float lk = LO(1), lk1 = LO(2);
  for (int k = 1; k <= kmax - kshift; ++k) {
    // loads two levels ahead, issued before this level's stores (f/hi may alias fi/hi)
    const R gn = F(k + 4);
    const R hn3 = H(k + 3);
    const R wn = W(k + 2);
    const float ln = LO(k + 2);
    const R fio = fi_is_f ? b : fi_src[c + k * sk];
    const R advo = adv ? adv[c + k * sk] : R(0);
    R wfl = R(0);
    if (k <= kmax - 1) {
      uint8_t cd = 0;
      wfl = wface_s<R, S, REC>(k, kshift, kmax, dti, wk, a, b, e, g, hA, hB, &cd);
      if (REC) code[c + k * sk] = cd;
    }
    const R hio = hA;
    const R dh = dti * (wk - wkm1);
    const R hin = hio - dh;
    const R advn = splitfac * (wfl - wprev);
    if (lo) {
      float slo = lk;
      fi_dst[c + k * sk] = fv_update_lo<R>(hio, dh, hin, fio, dt, advn, slo);
      lo[c + k * sk] = __float2half_rn(slo);
    } else {
      fi_dst[c + k * sk] = fv_update<R>(hio, dh, hin, fio, dt, advn);
    }
    hi[c + k * sk] = hin;
    if (adv) adv[c + k * sk] = advo + advn;
    a = b; b = e; e = g; g = g2; g2 = gn;
    hA = hB; hB = hC; hC = hn3;
    wkm1 = wk; wk = wk1; wk1 = wn;
    lk = lk1; lk1 = ln;
    wprev = wfl;
  }
}

// Vertical sweep of two tracers in place (temperature and salinity with the same ww and hi, H_TAG,
// itersmax = 1): k_sweep_w's arithmetic for each field, the heights updated once.
template <class R, int S>
__global__ void __launch_bounds__(128) k_sweep_w2(Dev d, R dt, R splitfac, R* fa, R* fb, R* hi,
                                                  const R* __restrict__ ww, const int32_t* __restrict__ az,
                                                  __half* lo_a = nullptr, __half* lo_b = nullptr) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  if (ii >= d.ni() - 1 || jj >= d.nj() - 1) return;
  const long long c = (long long)ii + (long long)jj * d.sj;
  if (az[c] != 1) return;
  const int kmax = d.kmax;
  const long long sk = d.sk;
  const R dti = splitfac * dt;
  auto FA = [&](int k) -> R { return (k >= 0 && k <= kmax) ? fa[c + k * sk] : R(0); };
  auto FB = [&](int k) -> R { return (k >= 0 && k <= kmax) ? fb[c + k * sk] : R(0); };
  auto H = [&](int k) -> R { return (k >= 0 && k <= kmax) ? hi[c + k * sk] : R(0); };
  auto W = [&](int k) -> R { return (k <= kmax) ? ww[c + k * sk] : R(0); };
  R a0 = FA(0), a1 = FA(1), a2 = FA(2), a3 = FA(3), a4 = FA(4);
  R b0 = FB(0), b1 = FB(1), b2 = FB(2), b3 = FB(3), b4 = FB(4);
  R hA = H(1), hB = H(2), hC = H(3);
  R wkm1 = W(0), wk = W(1), wk1 = W(2);
  R wpa = R(0), wpb = R(0);
  // the carried errors (compensated storage) two levels ahead, like the window
  auto LO = [&](const __half* l, int k) -> float { return (l && k <= kmax) ? __half2float(l[c + k * sk]) : 0.f; };
  float la = LO(lo_a, 1), la1 = LO(lo_a, 2), lb = LO(lo_b, 1), lb1 = LO(lo_b, 2);
  for (int k = 1; k <= kmax; ++k) {
    const R an = FA(k + 4), bn = FB(k + 4);
    const R hn3 = H(k + 3);
    const R wn = W(k + 2);
    const float lan = LO(lo_a, k + 2), lbn = LO(lo_b, k + 2);
    R wfa = R(0), wfb = R(0);
    if (k <= kmax - 1) {
      wfa = wface_s<R, S>(k, 0, kmax, dti, wk, a0, a1, a2, a3, hA, hB);
      wfb = wface_s<R, S>(k, 0, kmax, dti, wk, b0, b1, b2, b3, hA, hB);
    }
    const R hio = hA;
    const R dh = dti * (wk - wkm1);
    const R hin = hio - dh;
    if (lo_a) {
      float slo = la;
      fa[c + k * sk] = fv_update_lo<R>(hio, dh, hin, a1, dt, splitfac * (wfa - wpa), slo);
      lo_a[c + k * sk] = __float2half_rn(slo);
    } else {
      fa[c + k * sk] = fv_update<R>(hio, dh, hin, a1, dt, splitfac * (wfa - wpa));
    }
    if (lo_b) {
      float slo = lb;
      fb[c + k * sk] = fv_update_lo<R>(hio, dh, hin, b1, dt, splitfac * (wfb - wpb), slo);
      lo_b[c + k * sk] = __float2half_rn(slo);
    } else {
      fb[c + k * sk] = fv_update<R>(hio, dh, hin, b1, dt, splitfac * (wfb - wpb));
    }
    hi[c + k * sk] = hin;
    a0 = a1; a1 = a2; a2 = a3; a3 = a4; a4 = an;
    b0 = b1; b1 = b2; b2 = b3; b3 = b4; b4 = bn;
    hA = hB; hB = hC; hC = hn3;
    wkm1 = wk; wk = wk1; wk1 = wn;
    la = la1; la1 = lan;
    lb = lb1; lb1 = lbn;
    wpa = wfa;
    wpb = wfb;
  }
}

// adv_split_w with sub-iterations (itersmax > 1, adv_split_w.F90:193-299): the column is held in
// thread-local arrays (kmax <= GB_KMAX_ITER). Counts columns whose estimate exceeded itersmax.
#ifndef GB_KMAX_ITER
#define GB_KMAX_ITER 128
#endif
template <class R>
__global__ void __launch_bounds__(64) k_sweep_w_iter(Dev d, R dt, R splitfac, int scheme, int kshift,
                                                     int itersmax, const R* f, const R* fi_src,
                                                     R* fi_dst, R* hi, R* adv,
                                                     const R* __restrict__ ww,
                                                     const int32_t* __restrict__ az,
                                                     unsigned long long* warn, __half* lo = nullptr) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  if (ii >= d.ni() - 1 || jj >= d.nj() - 1) return;
  const long long c = (long long)ii + (long long)jj * d.sj;
  if (az[c] != 1) return;
  const int kmax = d.kmax;
  const long long sk = d.sk;
  const R dti = splitfac * dt;
  R fo[GB_KMAX_ITER + 1], fia[GB_KMAX_ITER + 1], hia[GB_KMAX_ITER + 1], ada[GB_KMAX_ITER + 1],
      wfl[GB_KMAX_ITER + 1], cfl0[GB_KMAX_ITER + 1], cfls[GB_KMAX_ITER + 1];
  float loa[GB_KMAX_ITER + 1];  // the scaled carried errors of the column (compensated storage)
  for (int k = 0; k <= kmax; ++k) {
    fo[k] = f[c + k * sk];
    cfl0[k] = R(0);
  }
  for (int k = 1 - kshift; k <= kmax - 1; ++k)
    cfl0[k] = fabs(ww[c + k * sk]) * dti / (R(0.5) * (hi[c + k * sk] + hi[c + (k + 1) * sk]));
  wfl[0] = R(0);
  wfl[kmax] = R(0);
  int iters = 1;
  R itersm1 = R(1), dtik = dti, splitfack = splitfac;
  const R* faux = fo;
  int it = 1;
  while (it <= iters) {
    if (it == 1) {
      for (int k = 0; k <= kmax; ++k) {
        fia[k] = fi_src[c + k * sk];
        hia[k] = hi[c + k * sk];
        ada[k] = adv ? adv[c + k * sk] : R(0);
        loa[k] = lo ? __half2float(lo[c + k * sk]) : 0.f;
      }
      faux = fo;
      for (int k = 0; k <= kmax; ++k) cfls[k] = cfl0[k];
    } else if (scheme != UPSTREAM || iters < itersmax) {
      for (int k = 1 - kshift; k <= kmax - 1; ++k)
        cfls[k] = fabs(ww[c + k * sk]) * dti / (R(0.5) * (hia[k] + hia[k + 1]));
    }
    if (iters < itersmax) {
      int iters_new = 1;
      for (int k = 1 - kshift; k <= kmax - 1; ++k) {
        const int cn = (int)ceil(cfls[k]);
        iters_new = iters_new > cn ? iters_new : cn;
      }
      if (iters_new > iters) {
        if (iters_new > itersmax) {
          atomicAdd(warn, 1ull);
          iters = itersmax;
        } else {
          iters = iters_new;
        }
        itersm1 = R(1) / R(iters);
        dtik = dti * itersm1;
        splitfack = splitfac * itersm1;
        if (it > 1) {
          it = 1;
          continue;
        }
      }
    }
    for (int k = 1 - kshift; k <= kmax - 1; ++k) {
      const R w = ww[c + k * sk];
      R fu, fuu = R(0), fd = R(0);
      bool lim = false;
      if (w > R(0)) {
        fu = faux[k];
        if (scheme != UPSTREAM) lim = (k > 1 - kshift);
        if (lim) { fuu = faux[k - 1]; fd = faux[k + 1]; }
      } else {
        fu = faux[k + 1];
        if (scheme != UPSTREAM) lim = (k < kmax - 1);
        if (lim) { fuu = faux[k + 2]; fd = faux[k]; }
      }
      if (lim) fu = recon<R>(scheme, cfls[k] * itersm1, fuu, fu, fd);
      wfl[k] = w * fu;
    }
    for (int k = 1; k <= kmax - kshift; ++k) {
      const R hio = hia[k];
      const R dh = dtik * (ww[c + k * sk] - ww[c + (k - 1) * sk]);
      hia[k] = hio - dh;
      const R advn = splitfack * (wfl[k] - wfl[k - 1]);
      fia[k] = lo ? fv_update_lo<R>(hio, dh, hia[k], fia[k], dt, advn, loa[k])
                  : fv_update<R>(hio, dh, hia[k], fia[k], dt, advn);
      ada[k] = ada[k] + advn;
    }
    faux = fia;
    ++it;
  }
  for (int k = 1; k <= kmax - kshift; ++k) {
    fi_dst[c + k * sk] = fia[k];
    hi[c + k * sk] = hia[k];
    if (adv) adv[c + k * sk] = ada[k];
    if (lo) lo[c + k * sk] = __float2half_rn(loa[k]);
  }
}

// ---------------------------------------------------------------------------------------------
// Thomas solve of one column (tridiagonal.F90:35-48); ru/qu live in shared memory [k][tid].
template <class R>
struct ThomasSmem {
  R* ru;
  R* qu;
  int nt;
  __device__ R& RU(int k) { return ru[k * nt + threadIdx.x]; }
  __device__ R& QU(int k) { return qu[k * nt + threadIdx.x]; }
};

// One tracer of the implicit vertical diffusion: the old values are read from Sin and the new ones
// written to S (they may alias) and, when S2 is given, to S2 as well; src (may be null): the
// temperature form's sources; RU, QU: two scratch 3D arrays; lo: the compensated storage (FP32).
template <class R>
struct VdField {
  const R* Sin;
  R* S;
  const R* src;
  R* RU;
  R* QU;
  R* S2;
  __half* lo;
  R avmol;
};
template <class R, int NF>
struct VdSet {
  VdField<R> t[NF];
};

// Implicit vertical diffusion (salinity.F90:348-389; temperature form with src) of NF = 1 or 2
// tracers (do_temperature and do_salinity share hn and nuh). One thread per interior column; the
// matrix rows are built top-down as the elimination proceeds, ru(k+1)/qu(k+1) carried in registers
// and ru(k)/qu(k) stored in two scratch 3D arrays per tracer (full occupancy, no shared memory for
// them: holding them in shared memory measured 1.6x slower at kmax = 50, from the lower occupancy)
// for the back substitution. With two tracers the thread runs their two eliminations side by side
// (independent chains) and loads hn and nuh once.
// hsk: the level stride of hn (d.sk; 0 when hn is a 2D array of column heights)
template <class R, int NF, bool IL = false>
__global__ void __launch_bounds__(128) k_vdiff(Dev d, R dt, R cnpar, VdSet<R, NF> F, const R* __restrict__ hn,
                                               const R* __restrict__ nuh, const int32_t* __restrict__ az,
                                               long long hsk) {
  const int kmax = d.kmax;
  const int i = d.imin + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = d.jmin + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > d.imax || j > d.jmax) return;
  const long long c = d.ix(i, j);
  if (az[c] != 1 || kmax <= 1) return;
  const long long sk = d.sk;
  // the elimination coefficients ru(k), qu(k) of a tracer: two scratch arrays, or (IL) one array of
  // (ru, qu) pairs at RU (twice the elements), one 8- or 16-byte access per level
  using R2 = std::conditional_t<sizeof(R) == 4, float2, double2>;
  auto put_rq = [&](const VdField<R>& f, int k, R r, R q) {
    if constexpr (IL) {
      R2 v;
      v.x = r;
      v.y = q;
      reinterpret_cast<R2*>(f.RU)[c + k * sk] = v;
    } else {
      f.RU[c + k * sk] = r;
      f.QU[c + k * sk] = q;
    }
  };
  auto get_rq = [&](const VdField<R>& f, int k, R& r, R& q) {
    if constexpr (IL) {
      const R2 v = reinterpret_cast<const R2*>(f.RU)[c + k * sk];
      r = v.x;
      q = v.y;
    } else {
      r = f.RU[c + k * sk];
      q = f.QU[c + k * sk];
    }
  };
  // the new value of level k from the old one and the increment: a plain FP32 sum, or the
  // compensated sum of the carried error lo (the tracer's compensated storage)
  // (lin: the level's stored carried error, loaded ahead by the caller)
  auto new_level = [&](const VdField<R>& f, int k, R sold, R inc, float lin) -> R {
    if constexpr (sizeof(R) == 4) {
      if (f.lo) {
        float slo = lin;
        const float v = add_comp_scaled(sold, inc, slo);
        f.lo[c + k * sk] = __float2half_rn(slo);
        return v;
      }
    }
    return sold + inc;
  };
  auto lo_at = [&](const VdField<R>& f, int k) -> float {
    if constexpr (sizeof(R) == 4) return f.lo ? __half2float(f.lo[c + k * sk]) : 0.f;
    else return 0.f;
  };
  auto put = [&](const VdField<R>& f, int k, R v) {
    f.S[c + k * sk] = v;
    if (f.S2) f.S2[c + k * sk] = v;
  };
  const R co = R(2) * (R(1) - cnpar) * dt;
  const R cn = R(2) * cnpar * dt;
  // FP64 solves the reference's system for the new value. FP32 solves the same matrix for the
  // increment dS = S_new - S_old, whose right-hand side is the flux divergence at the old level,
  // (ao+an)(k)*(S(k+1)-S(k)) - (ao+an)(k-1)*(S(k)-S(k-1)) [+ src]; the rounding then acts on the
  // small increment rather than on h*S (bias-free over hundreds of steps).
  constexpr bool incr = sizeof(R) == 4;
  // The inputs of a level (hn, nuh, then per tracer the old value and src) are staged by cp.async
  // into the thread's own shared-memory slots, a ring of four levels with three in flight ahead
  // of the elimination (a serial chain per column), so the chain does not wait on their loads.
  constexpr int NQ = 2 + 2 * NF;
  __shared__ R sl[4][NQ][128];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  auto issue = [&](int lv) {
    if (lv >= 1) {
      R(*q)[128] = sl[lv & 3];
      cp_async(&q[0][tid], hn + c + lv * hsk);
      cp_async(&q[1][tid], nuh + c + lv * sk);
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        cp_async(&q[2 + 2 * n][tid], F.t[n].Sin + c + lv * sk);
        if (F.t[n].src) cp_async(&q[3 + 2 * n][tid], F.t[n].src + c + lv * sk);
      }
    }
    cp_async_commit();
  };
  auto get = [&](int lv, int q) -> R { return sl[lv & 3][q][tid]; };
  issue(kmax);
  issue(kmax - 1);
  issue(kmax - 2);
  issue(kmax - 3);
  cp_async_wait<2>();  // levels kmax and kmax-1
  // surface row k = kmax: au = a1, bu = a2, du = a4
  int k = kmax;
  R hnk = get(k, 0), hnkm1 = get(k - 1, 0);
  R nuk = get(k - 1, 1);
  R Sk[NF], Skm1[NF], src_n[NF], ao_km1[NF], an_km1[NF], ru[NF], qu[NF];
#pragma unroll
  for (int n = 0; n < NF; ++n) {
    const VdField<R>& f = F.t[n];
    const R nu = nuk + f.avmol;
    Sk[n] = get(k, 2 + 2 * n);
    Skm1[n] = get(k - 1, 2 + 2 * n);
    const R srck = f.src ? get(k, 3 + 2 * n) : R(0);
    src_n[n] = f.src ? get(k - 1, 3 + 2 * n) : R(0);  // the source of the next row
    ao_km1[n] = co * nu / (hnk + hnkm1);
    an_km1[n] = cn * nu / (hnk + hnkm1);
    const R a1 = -an_km1[n];
    const R a2 = hnk + an_km1[n];
    R a4 = incr ? -(ao_km1[n] + an_km1[n]) * (Sk[n] - Skm1[n]) : Sk[n] * (hnk - ao_km1[n]) + Skm1[n] * ao_km1[n];
    if (f.src) a4 = a4 + srck;
    ru[n] = a1 / a2;
    qu[n] = a4 / a2;
    put_rq(f, k, ru[n], qu[n]);
  }
  // inner rows k = kmax-1 .. 2
  for (k = kmax - 1; k >= 2; --k) {
    issue(k - 3);        // into the slot of level k+1, whose values were read in the row above
    cp_async_wait<2>();  // level k-1
    hnk = hnkm1;
    hnkm1 = get(k - 1, 0);
    nuk = get(k - 1, 1);
#pragma unroll
    for (int n = 0; n < NF; ++n) {
      const VdField<R>& f = F.t[n];
      const R ao_k = ao_km1[n], an_k = an_km1[n];  // aux at interface k (computed as k-1 of row k+1)
      const R nu = nuk + f.avmol;
      const R Skp1 = Sk[n];
      Sk[n] = Skm1[n];
      Skm1[n] = get(k - 1, 2 + 2 * n);
      const R srcv = src_n[n];
      if (f.src) src_n[n] = get(k - 1, 3 + 2 * n);
      ao_km1[n] = co * nu / (hnk + hnkm1);
      an_km1[n] = cn * nu / (hnk + hnkm1);
      const R a3 = -an_k;
      const R a1 = -an_km1[n];
      const R a2 = hnk + an_k + an_km1[n];
      R a4 = incr ? (ao_k + an_k) * (Skp1 - Sk[n]) - (ao_km1[n] + an_km1[n]) * (Sk[n] - Skm1[n])
                  : Skp1 * ao_k + Sk[n] * (hnk - ao_k - ao_km1[n]) + Skm1[n] * ao_km1[n];
      if (f.src) a4 = a4 + srcv;
      const R den = a2 - a3 * ru[n];
      ru[n] = a1 / den;
      qu[n] = (a4 - a3 * qu[n]) / den;
      put_rq(f, k, ru[n], qu[n]);
    }
  }
  cp_async_wait<0>();
  // bottom row k = 1 (fi): only qu
  R v[NF];
#pragma unroll
  for (int n = 0; n < NF; ++n) {
    const VdField<R>& f = F.t[n];
    const R ao_k = ao_km1[n], an_k = an_km1[n];
    const R Skp1 = Sk[n];  // S(2)
    const R S1 = Skm1[n];  // S(1)
    const R h1 = hnkm1;
    const R a3 = -an_k;
    const R a2 = h1 + an_k;
    R a4 = incr ? (ao_k + an_k) * (Skp1 - S1) : Skp1 * ao_k + S1 * (h1 - ao_k);
    if (f.src) a4 = a4 + src_n[n];  // src(1)
    v[n] = (a4 - a3 * qu[n]) / (a2 - a3 * ru[n]);
    put(f, 1, incr ? new_level(f, 1, S1, v[n], lo_at(f, 1)) : v[n]);
  }
  // back substitution upwards, with the next level's coefficients loaded one step ahead
  R qn[NF], rn[NF], sn[NF], qn2[NF], rn2[NF], sn2[NF];
  float ln[NF], ln2[NF];
#pragma unroll
  for (int n = 0; n < NF; ++n) {
    const VdField<R>& f = F.t[n];
    qn[n] = rn[n] = R(0);
    if (kmax >= 2) get_rq(f, 2, rn[n], qn[n]);
    sn[n] = (incr && kmax >= 2) ? f.Sin[c + 2 * sk] : R(0);
    ln[n] = kmax >= 2 ? lo_at(f, 2) : 0.f;
    qn2[n] = rn2[n] = R(0);
    if (kmax >= 3) get_rq(f, 3, rn2[n], qn2[n]);
    sn2[n] = (incr && kmax >= 3) ? f.Sin[c + 3 * sk] : R(0);
    ln2[n] = kmax >= 3 ? lo_at(f, 3) : 0.f;
  }
  for (k = 2; k <= kmax; ++k) {
#pragma unroll
    for (int n = 0; n < NF; ++n) {
      const VdField<R>& f = F.t[n];
      const R q = qn[n], r = rn[n], so = sn[n];
      const float lc = ln[n];
      qn[n] = qn2[n]; rn[n] = rn2[n]; sn[n] = sn2[n]; ln[n] = ln2[n];
      if (k + 2 <= kmax) {
        get_rq(f, k + 2, rn2[n], qn2[n]);
        if (incr) sn2[n] = f.Sin[c + (k + 2) * sk];
        ln2[n] = lo_at(f, k + 2);
      }
      v[n] = q - r * v[n];
      put(f, k, incr ? new_level(f, k, so, v[n], lc) : v[n]);
    }
  }
}

// getm_tridiagonal on ncol independent columns, coefficients laid out [k][col].
template <class R>
__global__ void __launch_bounds__(64) k_tridiag(int ncol, int kmax, int fi, int lt, const R* __restrict__ au,
                                                const R* __restrict__ bu, const R* __restrict__ cu,
                                                const R* __restrict__ du, R* value) {
  extern __shared__ unsigned char smem_raw[];
  ThomasSmem<R> sm{reinterpret_cast<R*>(smem_raw), reinterpret_cast<R*>(smem_raw) + (kmax + 1) * blockDim.x,
                   (int)blockDim.x};
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  auto A = [&](const R* a, int k) -> R { return a[(long long)k * ncol + col]; };
  sm.RU(lt) = A(au, lt) / A(bu, lt);
  sm.QU(lt) = A(du, lt) / A(bu, lt);
  for (int i = lt - 1; i >= fi + 1; --i) {
    const R den = A(bu, i) - A(cu, i) * sm.RU(i + 1);
    sm.RU(i) = A(au, i) / den;
    sm.QU(i) = (A(du, i) - A(cu, i) * sm.QU(i + 1)) / den;
  }
  sm.QU(fi) = (A(du, fi) - A(cu, fi) * sm.QU(fi + 1)) / (A(bu, fi) - A(cu, fi) * sm.RU(fi + 1));
  R v = sm.QU(fi);
  value[(long long)fi * ncol + col] = v;
  for (int i = fi + 1; i <= lt; ++i) {
    v = sm.QU(i) - sm.RU(i) * v;
    value[(long long)i * ncol + col] = v;
  }
}

// NOSPLIT finaliser (advection_3d.F90:416-423): f = (ho*f - dt*adv)/hi on mask_finalise columns,
// levels 1..kmax.
template <class R>
__global__ void k_finalise(Dev d, R dt, R* f, const R* __restrict__ ho, const R* __restrict__ adv,
                           const R* __restrict__ hi, const uint8_t* __restrict__ mfin) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  if (ii >= d.ni() || jj >= d.nj()) return;
  const long long c = (long long)ii + (long long)jj * d.sj;
  if (!mfin[c]) return;
  const long long p = c + (long long)(blockIdx.z + 1) * d.sk;
  f[p] = (ho[p] * f[p] - dt * adv[p]) / hi[p];
}

// ---------------------------------------------------------------------------------------------
// Deterministic compensated reduction of f*h/ard1 (Neumaier pairs combined in a fixed order).
struct Neu {
  double s, c;
};
__device__ __forceinline__ void neu_add(Neu& a, double x) {
  const double t = a.s + x;
  if (fabs(a.s) >= fabs(x)) a.c += (a.s - t) + x; else a.c += (x - t) + a.s;
  a.s = t;
}
__device__ __forceinline__ void neu_merge(Neu& a, const Neu& b) {
  neu_add(a, b.s);
  a.c += b.c;
}


template <class R>
__global__ void __launch_bounds__(RED_THREADS) k_content_partial(Dev d, const R* __restrict__ f,
                                                                 const R* __restrict__ h,
                                                                 const int32_t* __restrict__ az,
                                                                 double* partial) {
  __shared__ Neu sh[RED_THREADS];
  const int nx = d.imax - d.imin + 1, ny = d.jmax - d.jmin + 1;
  const long long ncell = (long long)nx * ny * d.kmax;
  const double area = 1.0 / d.ard1;
  Neu acc{0.0, 0.0};
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < ncell;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx);
    const long long r = q / nx;
    const int j = (int)(r % ny);
    const int k = 1 + (int)(r / ny);
    const long long c = d.ix(d.imin + i, d.jmin + j);
    if (az[c] < 1) continue;
    const long long p = c + (long long)k * d.sk;
    neu_add(acc, (double)f[p] * (double)h[p] * area);
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = RED_THREADS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) neu_merge(sh[threadIdx.x], sh[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = sh[0].s;
    partial[2 * blockIdx.x + 1] = sh[0].c;
  }
}

static __global__ void __launch_bounds__(RED_THREADS) k_content_final(const double* partial, int nb,
                                                                        double* out) {
  __shared__ Neu sh[RED_THREADS];
  Neu acc{0.0, 0.0};
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    neu_add(acc, partial[2 * b]);
    acc.c += partial[2 * b + 1];
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = RED_THREADS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) neu_merge(sh[threadIdx.x], sh[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sh[0].s + sh[0].c;
    out[1] = sh[0].c;
  }
}

template <class R>
__global__ void k_check_range(Dev d, const R* __restrict__ f, const int32_t* __restrict__ az, R lo, R hi,
                              unsigned long long* count) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = d.imax - d.imin + 1, ny = d.jmax - d.jmin + 1;
  if (ii >= nx || jj >= ny) return;
  const long long c = d.ix(d.imin + ii, d.jmin + jj);
  if (az[c] <= 0) return;
  unsigned long long n = 0;
  for (int k = 0; k <= d.kmax; ++k) {
    const R v = f[c + (long long)k * d.sk];
    if (v < lo || v > hi) ++n;
  }
  if (n) atomicAdd(count, n);
}

}  // namespace gb
