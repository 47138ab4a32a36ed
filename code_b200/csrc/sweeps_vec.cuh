// sweeps_vec.cuh -- vectorised horizontal split sweeps (adv_split_u.F90:222-285,
// adv_split_v.F90:79-135) for fields whose rows and levels start on 16-byte boundaries; the FP32
// sweeps run here (FP64 runs the tile kernels of kernels.cuh, measured faster for its
// division-bound faces).
//
// Every thread owns N = 16 / sizeof(R) consecutive cells along i (one float4 / double2), so each
// global access is a full 16-byte vector and a warp moves 512 contiguous bytes per row.
//  * v sweep: the thread marches along j over a segment of VJS rows of one level, keeping the
//    stencil rows j-1 .. j+2 and the flux of the face below in registers: every face flux is
//    computed once, no shared memory and no barrier.
//  * u sweep: the 32 lanes of a warp cover 32*N consecutive cells of one row; the stencil
//    neighbours across lanes come by warp shuffles, the flux of the face between two warps of a
//    block through shared memory (one barrier per level).
// Each face flux and cell update evaluates the same expressions as the tile kernels of
// kernels.cuh (face_flux_s, fv_update), so FP64 results are bit-identical to them.
#pragma once
#include <type_traits>
#include "kernels.cuh"

namespace gb {

template <class R, int N>
struct alignas(N * sizeof(R)) VecPack {
  R v[N];
};

template <class R, int N>
__device__ __forceinline__ void ldv(const R* p, R (&v)[N]) {
  const VecPack<R, N> x = *reinterpret_cast<const VecPack<R, N>*>(p);
#pragma unroll
  for (int m = 0; m < N; ++m) v[m] = x.v[m];
}
template <class R, int N>
__device__ __forceinline__ void stv(R* p, const R (&v)[N]) {
  VecPack<R, N> x;
#pragma unroll
  for (int m = 0; m < N; ++m) x.v[m] = v[m];
  *reinterpret_cast<VecPack<R, N>*>(p) = x;
}

// N values of one row starting at cell c0 (zero beyond ni); p points at cell c0
template <class R, int N>
__device__ __forceinline__ void ld_row(const R* p, bool full, int navail, R (&v)[N]) {
  if (full) {
    ldv<R, N>(p, v);
  } else {
#pragma unroll
    for (int m = 0; m < N; ++m) v[m] = m < navail ? p[m] : R(0);
  }
}
template <class R, int N>
__device__ __forceinline__ void st_row(R* p, bool full, int navail, const R (&v)[N]) {
  if (full) {
    stv<R, N>(p, v);
  } else {
#pragma unroll
    for (int m = 0; m < N; ++m)
      if (m < navail) p[m] = v[m];
  }
}
// The carried errors of N cells (compensated storage, FP16) as one raw vector of N halves (8, 4
// or 2 bytes), converted to and from floats.
template <int N>
using LoVec = std::conditional_t<N == 4, uint2, std::conditional_t<N == 2, uint32_t, uint16_t>>;
template <int N>
__device__ __forceinline__ void lo_unpack(const LoVec<N>& x, float (&v)[N]) {
  const __half* h = reinterpret_cast<const __half*>(&x);
#pragma unroll
  for (int m = 0; m < N; ++m) v[m] = __half2float(h[m]);
}
template <int N>
__device__ __forceinline__ LoVec<N> lo_pack(const float (&v)[N]) {
  LoVec<N> x;
  __half* h = reinterpret_cast<__half*>(&x);
#pragma unroll
  for (int m = 0; m < N; ++m) h[m] = __float2half_rn(v[m]);
  return x;
}
template <int N>
__device__ __forceinline__ void st_lo(__half* p, bool full, int navail, const float (&v)[N]) {
  if (full) {
    *reinterpret_cast<LoVec<N>*>(p) = lo_pack<N>(v);
  } else {
#pragma unroll
    for (int m = 0; m < N; ++m)
      if (m < navail) p[m] = __float2half_rn(v[m]);
  }
}
template <int N>
__device__ __forceinline__ void ld_mask(const uint8_t* p, bool full, int navail, uint8_t (&v)[N]) {
  if (full) {
    if constexpr (N == 4) {
      const uint32_t x = *reinterpret_cast<const uint32_t*>(p);
#pragma unroll
      for (int m = 0; m < 4; ++m) v[m] = (uint8_t)(x >> (8 * m));
    } else {
      const uint16_t x = *reinterpret_cast<const uint16_t*>(p);
#pragma unroll
      for (int m = 0; m < N; ++m) v[m] = (uint8_t)(x >> (8 * m));
    }
  } else {
#pragma unroll
    for (int m = 0; m < N; ++m) v[m] = m < navail ? p[m] : 0;
  }
}
// the N mask bytes of a row from cell c0 packed into one word (byte m = cell c0+m)
template <int N>
__device__ __forceinline__ uint32_t ld_mask_w(const uint8_t* p, bool full, int navail) {
  static_assert(N == 2 || N == 4, "mask words of 2 or 4 cells (aligned 16- or 32-bit loads)");
  if (full) {
    if constexpr (N == 4) return *reinterpret_cast<const uint32_t*>(p);
    else return *reinterpret_cast<const uint16_t*>(p);
  }
  uint32_t x = 0;
#pragma unroll
  for (int m = 0; m < N; ++m)
    if (m < navail) x |= (uint32_t)p[m] << (8 * m);
  return x;
}
__device__ __forceinline__ bool mbit(uint32_t w, int m) { return ((w >> (8 * m)) & 0xffu) != 0; }

template <int N>
__device__ __forceinline__ void st_codes(uint8_t* p, bool full, int navail, const uint8_t (&v)[N]) {
  static_assert(N == 2 || N == 4, "code words of 2 or 4 cells (aligned 16- or 32-bit stores)");
  if (full) {
    if constexpr (N == 4) {
      *reinterpret_cast<uint32_t*>(p) = (uint32_t)v[0] | ((uint32_t)v[1] << 8) | ((uint32_t)v[2] << 16) |
                                        ((uint32_t)v[3] << 24);
    } else {
      *reinterpret_cast<uint16_t*>(p) = (uint16_t)(v[0] | (v[1] << 8));
    }
  } else {
#pragma unroll
    for (int m = 0; m < N; ++m)
      if (m < navail) p[m] = v[m];
  }
}

// 16-byte asynchronous copy global -> shared that reads `bytes` (0..16) bytes and zero-fills the
// rest (rows outside the domain and cells beyond the row end read as zero, like the tile sweeps'
// staging). src must be a valid address even when bytes == 0.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}

// The same for a vector of B = 8 or 16 bytes (8: cp.async.ca, the only form below 16 bytes).
template <int B>
__device__ __forceinline__ void cp_async_v(void* smem, const void* gmem, int bytes) {
  if constexpr (B == 16) {
    cp_async16(smem, gmem, bytes);
  } else {
    static_assert(B == 8, "cp_async_v: 8 or 16 bytes");
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
  }
}

// The same for the raw carried-error vector of N cells (8 or 4 bytes; cp.async.ca), reading
// `bytes` of it and zero-filling the rest.
template <int N>
__device__ __forceinline__ void cp_async_lo(void* smem, const void* gmem, int bytes) {
  static_assert(N == 4 || N == 2, "carried errors of 4 or 2 cells");
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (N == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}

// Each thread stages the inputs of its next steps in its own slots of a shared-memory ring
// (slot [stage][array][thread]: a warp's 16-byte slots are contiguous) and reads back only what
// it copied itself, so the pipeline needs no barrier; a slot is refilled one step after it was
// read and consumed.
constexpr int VST = 3;   // pipeline depth (steps in flight)
constexpr int VJS = 64;  // v sweep: rows per thread (fewer on small domains, see vec_rows)
constexpr int VKW = 4;   // v sweep: levels per block (one warp each)

template <class R, int N>
__device__ __forceinline__ void lds_vec(const VecPack<R, N>& x, R (&v)[N]) {
#pragma unroll
  for (int m = 0; m < N; ++m) v[m] = x.v[m];
}

// VN: cells per lane (16 bytes of R by default; 2 FP32 cells halve the registers of a lane)
// LO: the tracers carry compensated storage (F.t[n].lo; FP32 only), which the kernel then stages
// and updates; without it the kernel holds none of that code
template <class R, int S, bool REC, int NF, int VN = 16 / sizeof(R), bool LO = false>
__global__ void __launch_bounds__(32 * VKW) k_sweep_v_vec(Dev d, SweepC<R> C, int nk, int rows, TracerSet<R, NF> F,
                                                        const R* Di_src, R* Di_dst, R* adv,
                                                        const R* __restrict__ V, const R* __restrict__ DV,
                                                        const uint8_t* __restrict__ mflux,
                                                        const uint8_t* __restrict__ mupd, uint8_t* code) {
  constexpr int N = VN;
  constexpr int VB = N * (int)sizeof(R);
  // slots: f(j+2) per field; for a single field also fi(j) and adv(j) (a tracer pair reads fi
  // directly in the rare case that it is not f); V, DV, Di of row j
  constexpr int XV = NF == 1 ? 2 : NF, XDV = XV + 1, XDI = XV + 2, XAD = XV + 3;
  constexpr int NA = NF == 1 ? 6 : NF + 3;
  constexpr int sub = (S == UPSTREAM) ? 0 : 1;
  __shared__ VecPack<R, N> sbuf[VST][NA][32 * VKW];
  // the carried errors of the tracers (compensated storage), staged with the other inputs
  __shared__ LoVec<N> slo[LO ? VST : 1][NF][32 * VKW];
  const int tid = threadIdx.y * 32 + threadIdx.x;
  const int ni = d.ni(), nj = d.nj();
  const int c0 = (blockIdx.x * 32 + threadIdx.x) * N;
  const int k = blockIdx.z * VKW + threadIdx.y;
  if (c0 >= ni || k >= nk) return;  // no barrier in this kernel
  const int navail = ni - c0;
  const bool full = navail >= N;
  const int vbytes = (full ? N : navail) * (int)sizeof(R);
  const int j0 = blockIdx.y * rows;
  const int j1 = min(j0 + rows, nj);
  const long long sj = d.sj;
  const long long base = (long long)k * d.sk + c0;  // cell (c0, row 0) of level k
  // the same cell of the face depths DV and of the heights Di_src (2D arrays: level stride 0)
  const long long based = (long long)k * C.skdu + c0, basei = (long long)k * C.skdi + c0;
  const bool use_AH = C.AH > R(0);
  bool fis_f[NF];
#pragma unroll
  for (int n = 0; n < NF; ++n) fis_f[n] = F.t[n].fi_src == F.t[n].f;
  auto row_at = [&](const R* a, long long b, int j, R (&v)[N]) {
    if (j < 0 || j >= nj) {
#pragma unroll
      for (int m = 0; m < N; ++m) v[m] = R(0);
    } else {
      ld_row<R, N>(a + b + (long long)j * sj, full, navail, v);
    }
  };
  auto row_of = [&](const R* a, int j, R (&v)[N]) { row_at(a, base, j, v); };
  auto mrow_of = [&](const uint8_t* a, int j) -> uint32_t {
    return (j < 0 || j >= nj) ? 0u : ld_mask_w<N>(a + (long long)j * sj + c0, full, navail);
  };
  // inputs of row step j into stage st (an empty group past the segment keeps the counting uniform)
  auto issue = [&](int j, int st) {
    if (j < j1) {
      const long long p = base + (long long)j * sj;
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        const bool in = j + 2 < nj;
        cp_async_v<VB>(&sbuf[st][n][tid], F.t[n].f + (in ? p + 2 * sj : p), in ? vbytes : 0);
        if (NF == 1 && !fis_f[n]) cp_async_v<VB>(&sbuf[st][1][tid], F.t[n].fi_src + p, vbytes);
      }
      cp_async_v<VB>(&sbuf[st][XV][tid], V + p, vbytes);
      cp_async_v<VB>(&sbuf[st][XDV][tid], DV + (based + (long long)j * sj), vbytes);
      cp_async_v<VB>(&sbuf[st][XDI][tid], Di_src + (basei + (long long)j * sj), vbytes);
      if (NF == 1 && adv) cp_async_v<VB>(&sbuf[st][XAD][tid], adv + p, vbytes);
      if constexpr (LO && (N == 2 || N == 4)) {
#pragma unroll
        for (int n = 0; n < NF; ++n)
          if (F.t[n].lo) cp_async_lo<N>(&slo[st][n][tid], F.t[n].lo + p, vbytes / (int)sizeof(R) * 2);
      }
    }
    cp_async_commit();
  };
  // face fa (between rows fa and fa+1) from the window w[0..3] = rows fa-1 .. fa+2 and the flux
  // masks mw[0..2] = rows fa-1 .. fa+1
  R w[NF][4][N];
  uint32_t mw0, mw1, mw2;
  R Vp[N], fl_old[NF][N];
#pragma unroll
  for (int q = 0; q < VST - 1; ++q) issue(j0 + q, q);
#pragma unroll
  for (int n = 0; n < NF; ++n) {
    row_of(F.t[n].f, j0 - 2, w[n][0]);
    row_of(F.t[n].f, j0 - 1, w[n][1]);
    row_of(F.t[n].f, j0, w[n][2]);
    row_of(F.t[n].f, j0 + 1, w[n][3]);
  }
  mw0 = mrow_of(mflux, j0 - 2);
  mw1 = mrow_of(mflux, j0 - 1);
  mw2 = mrow_of(mflux, j0);
  {
    R DVp[N];
    row_of(V, j0 - 1, Vp);
    row_at(DV, based, j0 - 1, DVp);
    const int fa = j0 - 1;
    const bool valid = fa >= sub && fa <= nj - 2 - sub;
#pragma unroll
    for (int n = 0; n < NF; ++n)
#pragma unroll
      for (int m = 0; m < N; ++m)
        fl_old[n][m] = valid ? face_flux_s<R, S, false>(Vp[m], DVp[m], w[n][0][m], w[n][1][m], w[n][2][m],
                                                        w[n][3][m], mbit(mw0, m), mbit(mw1, m), mbit(mw2, m),
                                                        C.dti, C.cdx, C.AH, use_AH, C.dxf)
                             : R(0);
  }
  // masks of the next two steps (flux masks of row j+1, update masks of row j), loaded two steps
  // ahead (2D: cached)
  uint32_t mf1 = mrow_of(mflux, j0 + 1), mu1 = mrow_of(mupd, j0);
  uint32_t mf2 = mrow_of(mflux, j0 + 2), mu2 = mrow_of(mupd, j0 + 1);
  int st = 0;
  for (int j = j0; j < j1; ++j) {
    issue(j + VST - 1, st == 0 ? VST - 1 : st - 1);
    mw0 = mw1;
    mw1 = mw2;
    mw2 = mf1;
    const uint32_t mu = mu1;
    mf1 = mf2;
    mu1 = mu2;
    if (j + 2 < j1) {
      mf2 = mrow_of(mflux, j + 3);
      mu2 = mrow_of(mupd, j + 2);
    }
    cp_async_wait<VST - 1>();
    R Vc[N], DVc[N], Dio[N];
    lds_vec<R, N>(sbuf[st][XV][tid], Vc);
    lds_vec<R, N>(sbuf[st][XDV][tid], DVc);
    lds_vec<R, N>(sbuf[st][XDI][tid], Dio);
    R fio[NF][N];
#pragma unroll
    for (int n = 0; n < NF; ++n) {
      R nw[N];
      lds_vec<R, N>(sbuf[st][n][tid], nw);
#pragma unroll
      for (int m = 0; m < N; ++m) {
        w[n][0][m] = w[n][1][m];
        w[n][1][m] = w[n][2][m];
        w[n][2][m] = w[n][3][m];
        w[n][3][m] = nw[m];
      }
      if (fis_f[n]) {
#pragma unroll
        for (int m = 0; m < N; ++m) fio[n][m] = w[n][1][m];
      } else {
        if constexpr (NF == 1) lds_vec<R, N>(sbuf[st][1][tid], fio[n]);
        else ld_row<R, N>(F.t[n].fi_src + base + (long long)j * sj, full, navail, fio[n]);
      }
    }
    const long long p = base + (long long)j * sj;
    const bool jin = j >= 1 + sub && j <= nj - 2 - sub;
    const bool fvalid = j >= sub && j <= nj - 2 - sub;
    R fl_new[NF][N];
    uint8_t cd[N];
#pragma unroll
    for (int n = 0; n < NF; ++n)
#pragma unroll
      for (int m = 0; m < N; ++m) {
        uint8_t c = 0;
        fl_new[n][m] = fvalid ? face_flux_s<R, S, REC>(Vc[m], DVc[m], w[n][0][m], w[n][1][m], w[n][2][m],
                                                       w[n][3][m], mbit(mw0, m), mbit(mw1, m), mbit(mw2, m),
                                                       C.dti, C.cdx, C.AH, use_AH, C.dxf, &c)
                              : R(0);
        if (n == 0) cd[m] = c;
      }
    if (REC) st_codes<N>(code + p, full, navail, cd);
    // update of row j
    bool any = false;
    R Dn[N], dDv[N];
#pragma unroll
    for (int m = 0; m < N; ++m) {
      const bool upd = jin && mbit(mu, m);
      any |= upd;
      dDv[m] = cell_dD<R>(C, Vc[m], Vp[m]);
      Dn[m] = upd ? Dio[m] - dDv[m] : Dio[m];
    }
    R ad[N];
    if (NF == 1 && adv) lds_vec<R, N>(sbuf[st][XAD][tid], ad);
#pragma unroll
    for (int n = 0; n < NF; ++n) {
      R fo[N];
      float lo[N];
      const bool comp = LO && F.t[n].lo && any;  // compensated storage: the cells' carried errors
      if constexpr (LO && (N == 2 || N == 4)) {
        if (comp) lo_unpack<N>(slo[st][n][tid], lo);
      }
#pragma unroll
      for (int m = 0; m < N; ++m) {
        const bool upd = jin && mbit(mu, m);
        const R advn = cell_advn<R>(C, fl_new[n][m], fl_old[n][m]);
        if (comp)
          fo[m] = upd ? fv_update_lo<R>(Dio[m], dDv[m], Dn[m], fio[n][m], C.dt, advn, lo[m]) : fio[n][m];
        else
          fo[m] = upd ? fv_update<R>(Dio[m], dDv[m], Dn[m], fio[n][m], C.dt, advn) : fio[n][m];
        if (NF == 1 && adv && upd) ad[m] = ad[m] + advn;
      }
      if (F.t[n].fi_dst && (any || F.t[n].fi_dst != F.t[n].fi_src)) st_row<R, N>(F.t[n].fi_dst + p, full, navail, fo);
      if (comp) st_lo<N>(F.t[n].lo + p, full, navail, lo);
    }
    if (Di_dst && (any || Di_dst != Di_src)) st_row<R, N>(Di_dst + p, full, navail, Dn);
    if (NF == 1 && adv && any) st_row<R, N>(adv + p, full, navail, ad);
#pragma unroll
    for (int m = 0; m < N; ++m) Vp[m] = Vc[m];
#pragma unroll
    for (int n = 0; n < NF; ++n)
#pragma unroll
      for (int m = 0; m < N; ++m) fl_old[n][m] = fl_new[n][m];
    st = st == VST - 1 ? 0 : st + 1;
  }
  cp_async_wait<0>();
}

// u sweep: a warp covers 32 vectors of one row and updates the cells of lanes 1..30 (UOWN = 30
// vectors): lane 0 supplies the two cells left of the segment and lane 31 the right neighbour and
// the flux through the segment's right face, all by shuffles, so a warp needs no shared memory
// exchange, no barrier and no divergent halo loads. Segments advance by 30 vectors; the warps of
// a block take consecutive segments of one row and loop over NKB levels, staging the levels
// ahead in their shared-memory ring like the v sweep.
constexpr int UOWN = 30;
constexpr int UWB = 4;  // warps (segments) per block

template <class R, int S, bool REC, int NF, bool LO = false>
__global__ void __launch_bounds__(32 * UWB) k_sweep_u_vec(Dev d, SweepC<R> C, int nk, TracerSet<R, NF> F,
                                                        const R* Di_src, R* Di_dst, R* adv,
                                                        const R* __restrict__ U, const R* __restrict__ DU,
                                                        const uint8_t* __restrict__ mflux,
                                                        const uint8_t* __restrict__ mupd, uint8_t* code) {
  constexpr int N = 16 / sizeof(R);
  // slots: f per field; for a single field also fi and adv; U, DU, Di
  constexpr int XU = NF == 1 ? 2 : NF, XDU = XU + 1, XDI = XU + 2, XAD = XU + 3;
  constexpr int NA = NF == 1 ? 6 : NF + 3;
  constexpr int sub = (S == UPSTREAM) ? 0 : 1;
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ VecPack<R, N> sbuf[VST][NA][32 * UWB];
  // the carried errors of the tracers (compensated storage), staged with the other inputs
  __shared__ LoVec<N> slo[LO ? VST : 1][NF][32 * UWB];
  const int lane = threadIdx.x;
  const int tid = threadIdx.y * 32 + lane;
  const int ni = d.ni();
  const int seg = blockIdx.x * UWB + threadIdx.y;
  const int s0 = seg * UOWN * N;  // first cell owned by the warp
  if (s0 >= ni) return;           // whole warp (no barrier in this kernel)
  const int c0 = s0 + (lane - 1) * N;
  const bool act = c0 >= 0 && c0 < ni;
  const int navail = ni - c0;
  const bool full = act && navail >= N;
  const int vbytes = act ? (full ? N : navail) * (int)sizeof(R) : 0;
  const bool own = act && lane >= 1 && lane <= UOWN;
  // adv_init: the sweep starts the flux-divergence sum, writing adv = 0 + its own term in every cell
  // it owns (the caller does not clear adv first)
  const bool ainit = C.adv_init != 0;
  const long long crow = (long long)blockIdx.y * d.sj;
  const int k0 = blockIdx.z * NKB;
  const int k1 = min(k0 + NKB, nk);
  const long long cc = act ? c0 : 0;  // a valid address for the lanes outside the row
  const bool use_AH = C.AH > R(0);
  bool fis_f[NF];
#pragma unroll
  for (int n = 0; n < NF; ++n) fis_f[n] = F.t[n].fi_src == F.t[n].f;
  // masks of the lane's cells and of the two cells to its left
  uint8_t mf[N + 2], mu[N];
  {
    uint8_t m[N];
    if (act) ld_mask<N>(mflux + crow + c0, full, navail, m);
    else
#pragma unroll
      for (int q = 0; q < N; ++q) m[q] = 0;
    if (own) ld_mask<N>(mupd + crow + c0, full, navail, mu);
    else
#pragma unroll
      for (int q = 0; q < N; ++q) mu[q] = 0;
    const uint32_t l2 = __shfl_up_sync(FULL, (uint32_t)m[N - 2], 1), l1 = __shfl_up_sync(FULL, (uint32_t)m[N - 1], 1);
    mf[0] = (uint8_t)l2;
    mf[1] = (uint8_t)l1;
#pragma unroll
    for (int q = 0; q < N; ++q) mf[q + 2] = m[q];
  }
  bool updm[N];
  bool any = false;
#pragma unroll
  for (int q = 0; q < N; ++q) {
    const int c = c0 + q;
    updm[q] = own && q < navail && mu[q] != 0 && c >= 1 + sub && c <= ni - 2 - sub;
    any |= updm[q];
  }
  auto issue = [&](int k, int st) {
    if (k < k1) {
      const long long p = crow + (long long)k * d.sk + cc;
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        cp_async16(&sbuf[st][n][tid], F.t[n].f + p, vbytes);
        if (NF == 1 && own && !fis_f[n]) cp_async16(&sbuf[st][1][tid], F.t[n].fi_src + p, vbytes);
      }
      cp_async16(&sbuf[st][XU][tid], U + p, vbytes);
      cp_async16(&sbuf[st][XDU][tid], DU + (crow + (long long)k * C.skdu + cc), vbytes);
      if (own) {
        cp_async16(&sbuf[st][XDI][tid], Di_src + (crow + (long long)k * C.skdi + cc), vbytes);
        if (NF == 1 && adv && any && !ainit) cp_async16(&sbuf[st][XAD][tid], adv + p, vbytes);
        if constexpr (LO && (N == 2 || N == 4)) {
#pragma unroll
          for (int n = 0; n < NF; ++n)
            if (F.t[n].lo && any) cp_async_lo<N>(&slo[st][n][tid], F.t[n].lo + p, vbytes / (int)sizeof(R) * 2);
        }
      }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int q = 0; q < VST - 1; ++q) issue(k0 + q, q);
  int st = 0;
  for (int k = k0; k < k1; ++k) {
    issue(k + VST - 1, st == 0 ? VST - 1 : st - 1);
    cp_async_wait<VST - 1>();
    const long long p = crow + (long long)k * d.sk + c0;
    R f[NF][N + 3];  // cells c0-2 .. c0+N
    R Uv[N + 1], DUv[N + 1];  // faces c0-1 .. c0+N-1
#pragma unroll
    for (int n = 0; n < NF; ++n) {
      R v[N];
      lds_vec<R, N>(sbuf[st][n][tid], v);
      f[n][0] = __shfl_up_sync(FULL, v[N - 2], 1);
      f[n][1] = __shfl_up_sync(FULL, v[N - 1], 1);
#pragma unroll
      for (int q = 0; q < N; ++q) f[n][q + 2] = v[q];
      f[n][N + 2] = __shfl_down_sync(FULL, v[0], 1);
    }
    {
      R u[N], du[N];
      lds_vec<R, N>(sbuf[st][XU][tid], u);
      lds_vec<R, N>(sbuf[st][XDU][tid], du);
      Uv[0] = __shfl_up_sync(FULL, u[N - 1], 1);
      DUv[0] = __shfl_up_sync(FULL, du[N - 1], 1);
#pragma unroll
      for (int q = 0; q < N; ++q) {
        Uv[q + 1] = u[q];
        DUv[q + 1] = du[q];
      }
    }
    // left faces of the lane's cells: face c0+m-1
    R fl[NF][N + 1];
    uint8_t cd[N + 1];
#pragma unroll
    for (int m = 0; m < N; ++m) {
      const int fa = c0 + m - 1;
      const bool valid = act && fa >= sub && fa <= ni - 2 - sub;
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        uint8_t c = 0;
        fl[n][m] = valid ? face_flux_s<R, S, REC>(Uv[m], DUv[m], f[n][m], f[n][m + 1], f[n][m + 2], f[n][m + 3],
                                                  mf[m] != 0, mf[m + 1] != 0, mf[m + 2] != 0, C.dti, C.cdx, C.AH,
                                                  use_AH, C.dxf, &c)
                         : R(0);
        if (n == 0) cd[m] = c;
      }
    }
    // right face of the last cell: the next lane's first face
#pragma unroll
    for (int n = 0; n < NF; ++n) fl[n][N] = __shfl_down_sync(FULL, fl[n][0], 1);
    cd[N] = (uint8_t)__shfl_down_sync(FULL, (uint32_t)cd[0], 1);
    const int stc = st;
    st = st == VST - 1 ? 0 : st + 1;
    if (!own) continue;
    if (REC) {
      uint8_t cv[N];  // faces c0 .. c0+N-1, stored at their left cells
#pragma unroll
      for (int q = 0; q < N; ++q) cv[q] = cd[q + 1];
      st_codes<N>(code + p, full, navail, cv);
    }
    R Dio[N], Dn[N], dDv[N];
    lds_vec<R, N>(sbuf[stc][XDI][tid], Dio);
#pragma unroll
    for (int q = 0; q < N; ++q) {
      dDv[q] = cell_dD<R>(C, Uv[q + 1], Uv[q]);
      Dn[q] = updm[q] ? Dio[q] - dDv[q] : Dio[q];
    }
    R ad[N];
    if (NF == 1 && adv && any && !ainit) lds_vec<R, N>(sbuf[stc][XAD][tid], ad);
    if (NF == 1 && adv && ainit) {
#pragma unroll
      for (int q = 0; q < N; ++q) ad[q] = R(0);
    }
#pragma unroll
    for (int n = 0; n < NF; ++n) {
      R fio[N], fo[N];
      if (fis_f[n]) {
#pragma unroll
        for (int q = 0; q < N; ++q) fio[q] = f[n][q + 2];
      } else {
        if constexpr (NF == 1) lds_vec<R, N>(sbuf[stc][1][tid], fio);
        else ld_row<R, N>(F.t[n].fi_src + p, full, navail, fio);
      }
      float lo[N];
      const bool comp = LO && F.t[n].lo && any;  // compensated storage: the cells' carried errors
      if constexpr (LO && (N == 2 || N == 4)) {
        if (comp) lo_unpack<N>(slo[stc][n][tid], lo);
      }
#pragma unroll
      for (int q = 0; q < N; ++q) {
        const R advn = cell_advn<R>(C, fl[n][q + 1], fl[n][q]);
        if (comp)
          fo[q] = updm[q] ? fv_update_lo<R>(Dio[q], dDv[q], Dn[q], fio[q], C.dt, advn, lo[q]) : fio[q];
        else
          fo[q] = updm[q] ? fv_update<R>(Dio[q], dDv[q], Dn[q], fio[q], C.dt, advn) : fio[q];
        if (NF == 1 && adv && updm[q]) ad[q] = ad[q] + advn;
      }
      if (F.t[n].fi_dst && (any || F.t[n].fi_dst != F.t[n].fi_src)) st_row<R, N>(F.t[n].fi_dst + p, full, navail, fo);
      if (comp) st_lo<N>(F.t[n].lo + p, full, navail, lo);
    }
    if (Di_dst && (any || Di_dst != Di_src)) st_row<R, N>(Di_dst + p, full, navail, Dn);
    if (NF == 1 && adv && (any || ainit)) st_row<R, N>(adv + p, full, navail, ad);
  }
  cp_async_wait<0>();
}

}  // namespace gb
