// kernels_inst.cuh -- launcher definitions; included once per precision by kernels_f64.cu and
// kernels_f32.cu with GB_REAL defined to the arithmetic type.
#pragma once
#include <cstdint>
#include <initializer_list>
#include <type_traits>

#include "kernels.cuh"
#include "sweeps_vec.cuh"

namespace gb {

// The vectorised sweeps of sweeps_vec.cuh apply when every row and level of the fields starts on
// a 16-byte boundary (byte masks: N bytes, FP16 carried errors: 2N bytes); the tile kernels serve
// every other layout (and all layouts when the vectorised sweeps are switched off, for comparison).
template <class R>
static bool vec_layout(const Dev& d, int nk, std::initializer_list<const void*> ptrs,
                       std::initializer_list<const void*> bytes, std::initializer_list<const void*> halves = {}) {
  constexpr long long N = 16 / sizeof(R);
  if (!vector_sweeps_enabled()) return false;
  if (d.sj % N != 0 || (nk > 1 && d.sk % N != 0)) return false;
  for (const void* p : ptrs)
    if (p && (reinterpret_cast<uintptr_t>(p) % 16) != 0) return false;
  for (const void* p : bytes)
    if (p && (reinterpret_cast<uintptr_t>(p) % N) != 0) return false;
  for (const void* p : halves)
    if (p && (reinterpret_cast<uintptr_t>(p) % (2 * N)) != 0) return false;
  return true;
}

// Calls F.template operator()<S>() with the scheme id as a compile-time constant; returns
// cudaErrorInvalidValue for an id that is not a split scheme.
template <class Fn>
static int dispatch_scheme(int scheme, Fn&& fn) {
  switch (scheme) {
    case UPSTREAM: return fn(std::integral_constant<int, UPSTREAM>());
    case P2: return fn(std::integral_constant<int, P2>());
    case SUPERBEE: return fn(std::integral_constant<int, SUPERBEE>());
    case MUSCL: return fn(std::integral_constant<int, MUSCL>());
    case P2_PDM: return fn(std::integral_constant<int, P2_PDM>());
    default: return (int)cudaErrorInvalidValue;
  }
}

template <class R, int DIR>
int run_sweep_h(const Dev& d, cudaStream_t s, int nk, R dt, R splitfac, int scheme, R AH, const R* f,
                const R* fi_src, R* fi_dst, const R* Di_src, R* Di_dst, R* adv, const R* U, const R* DU,
                const uint8_t* mflux, const uint8_t* mupd, uint8_t* code, const R* f_b, const R* fi_src_b,
                R* fi_dst_b, __half* lo, __half* lo_b, bool adv_init, bool du2d, bool di2d) {
  if (nk <= 0) return 0;
  if (f_b && (code || adv)) return (int)cudaErrorInvalidValue;
  SweepC<R> C = sweep_consts<R>(d, DIR, dt, splitfac, AH);
  if (du2d) C.skdu = 0;
  if (di2d) C.skdi = 0;
  bool comp = false;  // set below: the sweep updates compensated storage
  const int nz = (nk + NKB - 1) / NKB;
  return dispatch_scheme(scheme, [&](auto sc) {
    constexpr int S = decltype(sc)::value;
    auto go = [&](auto rec, auto set) {
      constexpr bool REC = decltype(rec)::value;
      constexpr int NF = sizeof(set.t) / sizeof(set.t[0]);
      // FP32: both directions vectorised; FP64: the v sweep (the FP64 u sweep measures faster in
      // the tile kernel, division-bound faces)
      const bool vec = (sizeof(R) == 4 || DIR == 1) &&
                       vec_layout<R>(d, nk,
                                     {set.t[0].f, set.t[0].fi_src, set.t[0].fi_dst, set.t[NF - 1].f,
                                      set.t[NF - 1].fi_src, set.t[NF - 1].fi_dst, Di_src, Di_dst, adv, U, DU},
                                     {mflux, mupd, code}, {set.t[0].lo, set.t[NF - 1].lo});
      // adv_init: the vectorised u sweep starts the sum itself; every other kernel adds to a
      // cleared one
      if (adv_init && adv && !(sizeof(R) == 4 && vec && DIR == 0)) {
        const cudaError_t e = cudaMemsetAsync(adv, 0, (size_t)nk * d.sk * sizeof(R), s);
        if (e != cudaSuccess) return (int)e;
      }
      if constexpr (sizeof(R) == 4) {
        constexpr int N = 16 / sizeof(R);
        if (vec && DIR == 0) {
          const int nseg = (d.ni() + UOWN * N - 1) / (UOWN * N);
          dim3 blk(32, UWB, 1);
          dim3 grd((nseg + UWB - 1) / UWB, d.nj(), nz);
          SweepC<R> Cu = C;
          Cu.adv_init = adv_init && adv ? 1 : 0;
          if (comp)
            k_sweep_u_vec<R, S, REC, NF, true><<<grd, blk, 0, s>>>(d, Cu, nk, set, Di_src, Di_dst, adv, U, DU,
                                                                   mflux, mupd, code);
          else
            k_sweep_u_vec<R, S, REC, NF, false><<<grd, blk, 0, s>>>(d, Cu, nk, set, Di_src, Di_dst, adv, U, DU,
                                                                    mflux, mupd, code);
          return (int)cudaGetLastError();
        }
        if (vec) {
          auto vl = [&](auto vn) {
            constexpr int VN = decltype(vn)::value;
            // rows per thread: VJS, halved while the grid would give fewer than ~24 warps per SM
            const long long nx = (d.ni() + 32 * VN - 1) / (32 * VN), nz = (nk + VKW - 1) / VKW;
            int rows = VJS;
            while (rows > 8 && nx * ((d.nj() + rows - 1) / rows) * nz * VKW < 148LL * 24) rows /= 2;
            dim3 blk(32, VKW, 1);
            dim3 grd((unsigned)nx, (d.nj() + rows - 1) / rows, (unsigned)nz);
            if (comp)
              k_sweep_v_vec<R, S, REC, NF, VN, true><<<grd, blk, 0, s>>>(d, C, nk, rows, set, Di_src, Di_dst, adv,
                                                                         U, DU, mflux, mupd, code);
            else
              k_sweep_v_vec<R, S, REC, NF, VN, false><<<grd, blk, 0, s>>>(d, C, nk, rows, set, Di_src, Di_dst, adv,
                                                                          U, DU, mflux, mupd, code);
            return (int)cudaGetLastError();
          };
          // float4 lanes for one field; float2 lanes for a tracer pair (72 registers against 116:
          // measured 4% faster at 2048x2048x50 from the higher occupancy; one field measured slower)
          if (NF == 2) return vl(std::integral_constant<int, 2>());
          return vl(std::integral_constant<int, 4>());
        }
      } else {
        // FP64: the j-marching v sweep on two-cell (16-byte) lanes (the 2048x2048x50 step's v
        // sweeps measured 18.8 ms against 25.2 ms in the tile kernel)
        constexpr int VN = 2;
        if (vec && DIR == 1) {
          const long long nx = (d.ni() + 32 * VN - 1) / (32 * VN), nz = (nk + VKW - 1) / VKW;
          int rows = VJS;
          while (rows > 8 && nx * ((d.nj() + rows - 1) / rows) * nz * VKW < 148LL * 24) rows /= 2;
          dim3 blk(32, VKW, 1);
          dim3 grd((unsigned)nx, (d.nj() + rows - 1) / rows, (unsigned)nz);
          k_sweep_v_vec<R, S, REC, NF, VN><<<grd, blk, 0, s>>>(d, C, nk, rows, set, Di_src, Di_dst, adv, U, DU,
                                                               mflux, mupd, code);
          return (int)cudaGetLastError();
        }
      }
      if (DIR == 0) {
        dim3 grd((d.ni() + OWU - 1) / OWU, d.nj(), nz);
        k_sweep_u_tile<R, S, REC, NF><<<grd, TU, 0, s>>>(d, C, nk, set, Di_src, Di_dst, adv, U, DU, mflux, mupd,
                                                         code);
      } else {
        dim3 blk(TVX, TVY, 1);
        dim3 grd((d.ni() + TVX - 1) / TVX, (d.nj() + TVY - 1) / TVY, nz);
        k_sweep_v_tile<R, S, REC, NF><<<grd, blk, 0, s>>>(d, C, nk, set, Di_src, Di_dst, adv, U, DU, mflux, mupd,
                                                          code);
      }
      return (int)cudaGetLastError();
    };
    // compensated storage (lo) only where the arithmetic is FP32
    if (sizeof(R) == 8) lo = lo_b = nullptr;
    comp = lo || lo_b;
    if (f_b) {
      TracerSet<R, 2> set{{{f, fi_src, fi_dst, lo}, {f_b, fi_src_b, fi_dst_b, lo_b}}};
      return go(std::false_type(), set);
    }
    TracerSet<R, 1> set{{{f, fi_src, fi_dst, lo}}};
    return code ? go(std::true_type(), set) : go(std::false_type(), set);
  });
}

template <class R>
int run_sweep_w2(const Dev& d, cudaStream_t s, R dt, R splitfac, int scheme, R* fa, R* fb, R* hi, const R* ww,
                 const int32_t* az, __half* lo_a, __half* lo_b) {
  if (sizeof(R) == 8) lo_a = lo_b = nullptr;
  return dispatch_scheme(scheme, [&](auto sc) {
    constexpr int S = decltype(sc)::value;
    dim3 blk(64, 2, 1);
    dim3 grd((d.ni() - 1 + blk.x - 1) / blk.x, (d.nj() - 1 + blk.y - 1) / blk.y, 1);
    k_sweep_w2<R, S><<<grd, blk, 0, s>>>(d, dt, splitfac, fa, fb, hi, ww, az, lo_a, lo_b);
    return (int)cudaGetLastError();
  });
}

template <class R>
int run_sweep_w(const Dev& d, cudaStream_t s, R dt, R splitfac, int scheme, int kshift, int itersmax,
                const R* f, const R* fi_src, R* fi_dst, R* hi, R* adv, const R* ww, const int32_t* az,
                unsigned long long* warn, uint8_t* code, __half* lo) {
  if (sizeof(R) == 8) lo = nullptr;
  if (itersmax > 1) {
    if (code) return (int)cudaErrorInvalidValue;
    dim3 blk(32, 2, 1);
    dim3 grd((d.ni() - 1 + blk.x - 1) / blk.x, (d.nj() - 1 + blk.y - 1) / blk.y, 1);
    k_sweep_w_iter<R><<<grd, blk, 0, s>>>(d, dt, splitfac, scheme, kshift, itersmax, f, fi_src, fi_dst, hi,
                                          adv, ww, az, warn, lo);
    return (int)cudaGetLastError();
  }
  return dispatch_scheme(scheme, [&](auto sc) {
    constexpr int S = decltype(sc)::value;
    dim3 blk(64, 2, 1);
    dim3 grd((d.ni() - 1 + blk.x - 1) / blk.x, (d.nj() - 1 + blk.y - 1) / blk.y, 1);
    if (code)
      k_sweep_w<R, S, true><<<grd, blk, 0, s>>>(d, dt, splitfac, kshift, f, fi_src, fi_dst, hi, adv, ww, az, code,
                                                lo);
    else
      k_sweep_w<R, S, false><<<grd, blk, 0, s>>>(d, dt, splitfac, kshift, f, fi_src, fi_dst, hi, adv, ww, az,
                                                 nullptr, lo);
    return (int)cudaGetLastError();
  });
}

template <class R>
int run_finalise(const Dev& d, cudaStream_t s, R dt, R* f, const R* ho, const R* adv, const R* hi,
                 const uint8_t* mfin) {
  dim3 blk(64, 4, 1);
  dim3 grd((d.ni() + blk.x - 1) / blk.x, (d.nj() + blk.y - 1) / blk.y, d.kmax);
  k_finalise<R><<<grd, blk, 0, s>>>(d, dt, f, ho, adv, hi, mfin);
  return (int)cudaGetLastError();
}

template <class R>
int run_vdiff(const Dev& d, cudaStream_t s, R dt, R cnpar, R avmol, R* S, const R* hn, const R* nuh,
              const int32_t* az, const R* src, R* rus, R* qus, const R* Sin, R* S2, __half* lo) {
  if (d.kmax <= 1) return 0;
  if (sizeof(R) == 8) lo = nullptr;
  const int nx = d.imax - d.imin + 1, ny = d.jmax - d.jmin + 1;
  dim3 blk(32, 4, 1);
  dim3 grd((nx + 31) / 32, (ny + 3) / 4, 1);
  VdSet<R, 1> F{{{Sin ? Sin : S, S, src, rus, qus, S2, lo, avmol}}};
  k_vdiff<R, 1><<<grd, blk, 0, s>>>(d, dt, cnpar, F, hn, nuh, az, d.sk);
  return (int)cudaGetLastError();
}

template <class R>
int run_vdiff2(const Dev& d, cudaStream_t s, R dt, R cnpar, const R* hn, const R* nuh, const int32_t* az,
               R* Sa, R avmol_a, const R* src_a, R* rus_a, R* qus_a, __half* lo_a, R* Sb, R avmol_b, R* rus_b,
               R* qus_b, __half* lo_b, bool hn2d) {
  if (d.kmax <= 1) return 0;
  if (sizeof(R) == 8) lo_a = lo_b = nullptr;
  const int nx = d.imax - d.imin + 1, ny = d.jmax - d.jmin + 1;
  dim3 blk(32, 4, 1);
  dim3 grd((nx + 31) / 32, (ny + 3) / 4, 1);
  VdSet<R, 2> F{{{Sa, Sa, src_a, rus_a, qus_a, nullptr, lo_a, avmol_a},
                 {Sb, Sb, nullptr, rus_b, qus_b, nullptr, lo_b, avmol_b}}};
  // qus_a == qus_b == nullptr: each tracer's (ru, qu) pairs interleaved in its rus array (two
  // elements per cell): one access per level instead of two
  if (!qus_a && !qus_b)
    k_vdiff<R, 2, true><<<grd, blk, 0, s>>>(d, dt, cnpar, F, hn, nuh, az, hn2d ? 0LL : d.sk);
  else
    k_vdiff<R, 2><<<grd, blk, 0, s>>>(d, dt, cnpar, F, hn, nuh, az, hn2d ? 0LL : d.sk);
  return (int)cudaGetLastError();
}

template <class R>
int run_tridiag(cudaStream_t s, int ncol, int kmax, int fi, int lt, const R* au, const R* bu, const R* cu,
                const R* du, R* value) {
  const int nt = 64;
  const size_t smem = 2 * (size_t)(kmax + 1) * nt * sizeof(R);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_tridiag<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  k_tridiag<R><<<(ncol + nt - 1) / nt, nt, smem, s>>>(ncol, kmax, fi, lt, au, bu, cu, du, value);
  return (int)cudaGetLastError();
}

template <class R>
int run_content(const Dev& d, cudaStream_t s, const R* f, const R* h, const int32_t* az, double* partial,
                double* out) {
  k_content_partial<R><<<RED_BLOCKS, RED_THREADS, 0, s>>>(d, f, h, az, partial);
  k_content_final<<<1, RED_THREADS, 0, s>>>(partial, RED_BLOCKS, out);
  return (int)cudaGetLastError();
}

template <class R>
int run_check_range(const Dev& d, cudaStream_t s, const R* f, const int32_t* az, R lo, R hi,
                    unsigned long long* count) {
  dim3 blk(64, 4, 1);
  const int nx = d.imax - d.imin + 1, ny = d.jmax - d.jmin + 1;
  dim3 grd((nx + blk.x - 1) / blk.x, (ny + blk.y - 1) / blk.y, 1);
  k_check_range<R><<<grd, blk, 0, s>>>(d, f, az, lo, hi, count);
  return (int)cudaGetLastError();
}

// explicit instantiations for GB_REAL
template int run_sweep_h<GB_REAL, 0>(const Dev&, cudaStream_t, int, GB_REAL, GB_REAL, int, GB_REAL,
                                     const GB_REAL*, const GB_REAL*, GB_REAL*, const GB_REAL*, GB_REAL*,
                                     GB_REAL*, const GB_REAL*, const GB_REAL*, const uint8_t*, const uint8_t*,
                                     uint8_t*, const GB_REAL*, const GB_REAL*, GB_REAL*, __half*, __half*, bool, bool,
                                     bool);
template int run_sweep_h<GB_REAL, 1>(const Dev&, cudaStream_t, int, GB_REAL, GB_REAL, int, GB_REAL,
                                     const GB_REAL*, const GB_REAL*, GB_REAL*, const GB_REAL*, GB_REAL*,
                                     GB_REAL*, const GB_REAL*, const GB_REAL*, const uint8_t*, const uint8_t*,
                                     uint8_t*, const GB_REAL*, const GB_REAL*, GB_REAL*, __half*, __half*, bool, bool,
                                     bool);
template int run_sweep_w2<GB_REAL>(const Dev&, cudaStream_t, GB_REAL, GB_REAL, int, GB_REAL*, GB_REAL*, GB_REAL*,
                                   const GB_REAL*, const int32_t*, __half*, __half*);
template int run_sweep_w<GB_REAL>(const Dev&, cudaStream_t, GB_REAL, GB_REAL, int, int, int, const GB_REAL*,
                                  const GB_REAL*, GB_REAL*, GB_REAL*, GB_REAL*, const GB_REAL*, const int32_t*,
                                  unsigned long long*, uint8_t*, __half*);
template int run_finalise<GB_REAL>(const Dev&, cudaStream_t, GB_REAL, GB_REAL*, const GB_REAL*, const GB_REAL*,
                                   const GB_REAL*, const uint8_t*);
template int run_vdiff<GB_REAL>(const Dev&, cudaStream_t, GB_REAL, GB_REAL, GB_REAL, GB_REAL*, const GB_REAL*,
                                const GB_REAL*, const int32_t*, const GB_REAL*, GB_REAL*, GB_REAL*, const GB_REAL*,
                                GB_REAL*, __half*);
template int run_vdiff2<GB_REAL>(const Dev&, cudaStream_t, GB_REAL, GB_REAL, const GB_REAL*, const GB_REAL*,
                                 const int32_t*, GB_REAL*, GB_REAL, const GB_REAL*, GB_REAL*, GB_REAL*, __half*,
                                 GB_REAL*, GB_REAL, GB_REAL*, GB_REAL*, __half*, bool);
template int run_tridiag<GB_REAL>(cudaStream_t, int, int, int, int, const GB_REAL*, const GB_REAL*,
                                  const GB_REAL*, const GB_REAL*, GB_REAL*);
template int run_content<GB_REAL>(const Dev&, cudaStream_t, const GB_REAL*, const GB_REAL*, const int32_t*,
                                  double*, double*);
template int run_check_range<GB_REAL>(const Dev&, cudaStream_t, const GB_REAL*, const int32_t*, GB_REAL,
                                      GB_REAL, unsigned long long*);

}  // namespace gb

// ---- fused 2D momentum advection ----
#include "adv2d_fused.cuh"
namespace gb {
template int run_uvadv2d_fused<GB_REAL>(const Dev&, cudaStream_t, int, GB_REAL, int, const double*, const double*,
                                        const double*, const double*, const uint8_t*, const uint8_t*,
                                        const uint8_t*, const uint8_t*, double*);
}  // namespace gb

// ---- adjoint of the tracer step ----
#include "adjoint.cuh"
namespace gb {
template int run_adj_heights<GB_REAL>(const Dev&, cudaStream_t, GB_REAL, int, bool, const GB_REAL*, const GB_REAL*,
                                      const GB_REAL*, const GB_REAL*, const uint8_t*, const uint8_t*,
                                      const int32_t*, GB_REAL*, GB_REAL*, GB_REAL*, GB_REAL*);
template int run_adj_sweep_h<GB_REAL, 0>(const Dev&, cudaStream_t, int, GB_REAL, GB_REAL, int, GB_REAL,
                                         const GB_REAL*, GB_REAL*, const GB_REAL*, const GB_REAL*, const GB_REAL*,
                                         const uint8_t*, const uint8_t*, const uint8_t*, bool);
template int run_adj_sweep_h<GB_REAL, 1>(const Dev&, cudaStream_t, int, GB_REAL, GB_REAL, int, GB_REAL,
                                         const GB_REAL*, GB_REAL*, const GB_REAL*, const GB_REAL*, const GB_REAL*,
                                         const uint8_t*, const uint8_t*, const uint8_t*, bool);
template int run_adj_sweep_w<GB_REAL>(const Dev&, cudaStream_t, GB_REAL, GB_REAL, int, int, const GB_REAL*,
                                      GB_REAL*, const GB_REAL*, const GB_REAL*, const int32_t*, const uint8_t*);
template int run_adj_vdiff<GB_REAL>(const Dev&, cudaStream_t, GB_REAL, GB_REAL, GB_REAL, const GB_REAL*, GB_REAL*,
                                    GB_REAL*, const GB_REAL*, const GB_REAL*, const GB_REAL*, const GB_REAL*,
                                    const int32_t*, GB_REAL*, GB_REAL*);
}  // namespace gb

// ---- mode-split macro step (3D kernels) ----
#include "bc_kernels.cuh"
namespace gb {
template int run_bc3<GB_REAL>(int, const Dev&, cudaStream_t, const Bc3<GB_REAL>&, GB_REAL* const*, const GB_REAL*);
template int run_col_heights<GB_REAL>(const Dev&, cudaStream_t, const Bc3<GB_REAL>&, GB_REAL*);
}  // namespace gb
