// adv2d_fused.cuh -- the depth-averaged momentum advection of one micro step (uv_advect.F90:94-300
// with split = HALFSPLIT) as ONE kernel per momentum component. Included by kernels_inst.cuh.
//
// uv_advect builds the advected quantity and the face transports of the U (or V) control volumes
// from U, V, DU, DV (uv_advect.F90:94-110 / :204-220) and runs do_advection (advection.F90:
// 362-702) on them: u/2, v, u/2 split sweeps whose flux divergences sum to UEx (VEx). Done as
// separate launches that is six passes over the 2D state per component. Here a block owns an
// FX x FY tile, stages U, V, DU, DV over the tile plus the halo the three sweeps need (4 cells in
// x for two u/2 sweeps, 2 in y for the v sweep) in shared memory, runs u/2 on the tile+halo, v on
// the tile widened in x, u/2 on the tile, and writes UEx once. Every flux and update is the
// expression of the split-sweep kernels (face_flux_s, fv_update) in the same order, so FP64
// results equal the three-sweep sequence bit for bit. The u sweeps pass face fluxes between
// neighbouring cells by warp shuffles (the two warps of a region row overlap by one column), the v
// sweep through shared memory; each thread's own cells keep their depth and flux-divergence sum
// in registers across the three sweeps.
#pragma once
#include "kernels.cuh"

namespace gb {

constexpr int FX = 56, FY = 16;             // own tile (region rows of two full warps)
constexpr int RW = FX + 8, RH = FY + 4;     // staged region: i in [-4, FX+3], j in [-2, FY+1]
constexpr int FTY = 8;                      // thread rows: a block is RW x FTY threads, lane x <-> region column
constexpr int FT = RW * FTY;                // threads per block

// k*(a*s - b*s)*c as single rounded operations in this order: the volume and flux differences of
// the cell updates. FP64: the plain operations (the FP64 build contracts nothing); FP32: explicit
// intrinsics, so that the result does not depend on which products the compiler contracts.
template <class T>
__device__ __forceinline__ T diff_scaled(T k, T a, T b, T s, T c) {
  if constexpr (sizeof(T) == 4) return __fmul_rn(__fmul_rn(k, __fsub_rn(__fmul_rn(a, s), __fmul_rn(b, s))), c);
  else return k * (a * s - b * s) * c;
}
template <class T>
__device__ __forceinline__ T add_r(T a, T b) {
  if constexpr (sizeof(T) == 4) return __fadd_rn(a, b);
  else return a + b;
}

template <class T>
struct Adv2dSmem {
  T F0[RH][RW];   // advected quantity; reused for the field after the v sweep
  T F1[RH][RW];   // after the first u/2 sweep
  T Di[RH][RW];   // staged control-volume depth (the sweeps carry their rows' updated depths in registers)
  T Ua[RH][RW], DUa[RH][RW], Va[RH][RW], DVa[RH][RW];  // face transports / depths
  T FL[RH][RW];   // face fluxes of the v sweep
  T Q[RH][RW];    // bottom friction: the other component's velocity V/DV (DIR 0) or U/DU (DIR 1)
  uint8_t mfu[RH][RW], mfv[RH][RW], mpu[RH][RW], mpv[RH][RW];
};


// DIR 0: UEx on the U grid (fadv = U/DU, faces between U points); DIR 1: VEx on the V grid.
// TI: the storage type of U, V, DU, DV and Ex (FP64 state arrays, or the FP32 working copies of
// the mixed-precision micro step)
template <class T, int S, int DIR, class TI>
__device__ __forceinline__ void uvadv2d_tile(const Dev& d, T dt, const TI* __restrict__ U, const TI* __restrict__ V,
                                             const TI* __restrict__ DU, const TI* __restrict__ DV,
                                             const uint8_t* __restrict__ mflux_u,
                                             const uint8_t* __restrict__ mflux_v,
                                             const uint8_t* __restrict__ mupd_u, const uint8_t* __restrict__ mupd_v,
                                             TI* __restrict__ Ex, const Bf2Args& bf) {
  extern __shared__ unsigned char smem_raw[];
  Adv2dSmem<T>& sm = *reinterpret_cast<Adv2dSmem<T>*>(smem_raw);
  const int ni = d.ni(), nj = d.nj();
  const long long sj = d.sj;
  const int ii0 = blockIdx.x * FX, jj0 = blockIdx.y * FY;
  constexpr int sub = (S == UPSTREAM) ? 0 : 1;
  const T half = T(0.5), one = T(1), zero = T(0);
  const T dxu = T(d.dx), dyu = T(d.dy), ard1 = T(d.ard1);
  // ---- stage: region cell (r, q) <-> array (jj0-2+r, ii0-4+q); thread (q, ty) takes column q
  const int q = threadIdx.x, ty = threadIdx.y;
  const int ii = ii0 - 4 + q;
  const bool iin = ii >= 0 && ii < ni;
  for (int r = ty; r < RH; r += FTY) {
    const int jj = jj0 - 2 + r;
    T f0 = zero, ua = zero, dua = zero, va = zero, dva = zero, dio = zero, oq = zero;
    uint8_t a = 0, b = 0, c2 = 0, e2 = 0;
    if (iin && jj >= 0 && jj < nj) {
      const long long c = (long long)jj * sj + ii;
      if constexpr (sizeof(T) == 4 && sizeof(TI) == 4)
        if (bf.r) oq = DIR == 0 ? __fdividef(float(V[c]), float(DV[c])) : __fdividef(float(U[c]), float(DU[c]));
      a = mflux_u[c];
      b = mflux_v[c];
      c2 = mupd_u[c];
      e2 = mupd_v[c];
      dio = T(DIR == 0 ? DU[c] : DV[c]);
      const long long cn = DIR == 0 ? c + 1 : c + sj;  // the next U (V) point
      const bool ok = DIR == 0 ? (ii <= ni - 2) : (jj <= nj - 2);
      if (ok) {
        // FP32 working copies: the approximate division (2 ulp); FP64 arrays: the reference's quotient
        if constexpr (sizeof(T) == 4 && sizeof(TI) == 4)
          f0 = DIR == 0 ? __fdividef(U[c], DU[c]) : __fdividef(V[c], DV[c]);
        else
          f0 = T(DIR == 0 ? U[c] / DU[c] : V[c] / DV[c]);
        ua = T(0.5 * (U[c] + U[cn]));
        va = T(0.5 * (V[c] + V[cn]));
        dua = T(0.5 * (DU[c] + DU[cn]));
        dva = T(0.5 * (DV[c] + DV[cn]));
      }
    }
    sm.F0[r][q] = f0;
    sm.Q[r][q] = oq;
    sm.Ua[r][q] = ua;
    sm.DUa[r][q] = dua;
    sm.Va[r][q] = va;
    sm.DVa[r][q] = dva;
    sm.Di[r][q] = dio;
    sm.mfu[r][q] = a;
    sm.mfv[r][q] = b;
    sm.mpu[r][q] = c2;
    sm.mpv[r][q] = e2;
  }
  __syncthreads();
  // ---- the sweeps. A thread takes region column qc of the rows below; the two warps of a row
  // overlap by one column (warp 0: qc = 0..31, warp 1: qc = 31..62; warp 1's copy of column 31,
  // `dup`, updates and stores nothing), so that the left face flux of every cell a u sweep updates
  // is the flux of the lane before it (a warp shuffle, no shared-memory round trip or barrier).
  // The own rows of a thread, r = 2 + ty + 8m (m = 0, 1), are the same in all three sweeps: their
  // depths and flux-divergence sums stay in registers.
  const int qc = q - (q >> 5);
  const bool dup = q == 32;
  const int iic = ii0 - 4 + qc;
  const bool qown = qc >= 4 && qc < FX + 4 && !dup;  // own cells q in [4, FX+4)
  T di[2], acc[2] = {zero, zero};
  // ---- sweep 1: u/2 on rows r in [0, RH), cells q in [2, RW-2), faces q in [1, RW-3]
  {
    const T dti = half * dt, cdx = dti / dxu;
    const bool fok = qc >= 1 && qc <= RW - 3 && iic >= sub && iic <= ni - 2 - sub;  // face between qc, qc+1
    const bool cok = iic >= 1 + sub && iic <= ni - 2 - sub;
    const bool upd = qc >= 2 && qc < RW - 2 && !dup;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      // the own rows, then the halo rows 0, 1, RH-2, RH-1 (thread rows 0..3)
      const int r = m < 2 ? 2 + ty + 8 * m : (ty < 2 ? ty : RH - 4 + ty);
      if (m == 2 && ty >= 4) continue;
      T fl = zero;
      if (fok)
        fl = face_flux_s<T, S>(sm.Ua[r][qc], sm.DUa[r][qc], sm.F0[r][qc - 1], sm.F0[r][qc], sm.F0[r][qc + 1],
                               sm.F0[r][qc + 2], sm.mfu[r][qc - 1] != 0, sm.mfu[r][qc] != 0,
                               sm.mfu[r][qc + 1] != 0, dti, cdx, zero, false, dxu);
      const T flm = __shfl_up_sync(0xffffffffu, fl, 1);  // the face between qc-1 and qc
      if (upd) {
        const T fio = sm.F0[r][qc];
        T fnew = fio;
        T Dio = sm.Di[r][qc];
        if (cok && sm.mpu[r][qc]) {
          const T dD = diff_scaled<T>(dti, sm.Ua[r][qc], sm.Ua[r][qc - 1], dyu, ard1);
          const T Dn = Dio - dD;
          const T advn = diff_scaled<T>(half, fl, flm, dyu, ard1);
          fnew = fv_update<T>(Dio, dD, Dn, fio, dt, advn);
          Dio = Dn;
          if (m < 2 && qown) acc[m] = add_r<T>(acc[m], advn);
        }
        if (m < 2) di[m] = Dio;
        sm.F1[r][qc] = fnew;
      }
    }
    __syncthreads();
  }
  // ---- sweep 2: v on columns q in [2, RW-2), cells r in [2, RH-2), faces r in [1, RH-3]
  {
    const T dti = one * dt, cdy = dti / dyu;
    const bool col = qc >= 2 && qc < RW - 2 && !dup;
    if (col)
      for (int r = 1 + ty; r <= RH - 3; r += FTY) {
        const int fa = jj0 - 2 + r;  // face between r and r+1
        T fl = zero;
        if (fa >= sub && fa <= nj - 2 - sub)
          fl = face_flux_s<T, S>(sm.Va[r][qc], sm.DVa[r][qc], sm.F1[r - 1][qc], sm.F1[r][qc], sm.F1[r + 1][qc],
                                 sm.F1[r + 2][qc], sm.mfv[r - 1][qc] != 0, sm.mfv[r][qc] != 0,
                                 sm.mfv[r + 1][qc] != 0, dti, cdy, zero, false, dyu);
        sm.FL[r][qc] = fl;
      }
    __syncthreads();
    if (col) {
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const int r = 2 + ty + 8 * m;
        const int jj = jj0 - 2 + r;
        const T fio = sm.F1[r][qc];
        T fnew = fio;
        if (jj >= 1 + sub && jj <= nj - 2 - sub && sm.mpv[r][qc]) {
          const T Dio = di[m];
          const T dD = diff_scaled<T>(dti, sm.Va[r][qc], sm.Va[r - 1][qc], dxu, ard1);
          const T Dn = Dio - dD;
          const T advn = diff_scaled<T>(one, sm.FL[r][qc], sm.FL[r - 1][qc], dxu, ard1);
          fnew = fv_update<T>(Dio, dD, Dn, fio, dt, advn);
          if (qown) acc[m] = add_r<T>(acc[m], advn);
        }
        sm.F0[r][qc] = fnew;  // the field after v (F0 is no longer needed)
      }
    }
    __syncthreads();
  }
  // ---- sweep 3: u/2 on the own rows, own cells q in [4, RW-4), faces q in [3, RW-5]
  {
    const T dti = half * dt, cdx = dti / dxu;
    const bool fok = qc >= 3 && qc <= RW - 5 && iic >= sub && iic <= ni - 2 - sub;
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      const int r = 2 + ty + 8 * m;
      T fl = zero;
      if (fok)
        fl = face_flux_s<T, S>(sm.Ua[r][qc], sm.DUa[r][qc], sm.F0[r][qc - 1], sm.F0[r][qc], sm.F0[r][qc + 1],
                               sm.F0[r][qc + 2], sm.mfu[r][qc - 1] != 0, sm.mfu[r][qc] != 0,
                               sm.mfu[r][qc + 1] != 0, dti, cdx, zero, false, dxu);
      const T flm = __shfl_up_sync(0xffffffffu, fl, 1);
      if (qown) {
        const int jj = jj0 - 2 + r;
        T a = acc[m];
        if (iic >= 1 + sub && iic <= ni - 2 - sub && jj < nj && sm.mpu[r][qc]) {
          const T advn = diff_scaled<T>(half, fl, flm, dyu, ard1);
          a = add_r<T>(a, advn);
        }
        if (iic < ni && jj < nj) Ex[(long long)jj * sj + iic] = (TI)a;
      }
    }
  }
  if constexpr (sizeof(T) == 4 && sizeof(TI) == 4) {
    if (bf.r && qown) {
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const int r = 2 + ty + 8 * m;
        const int jj = jj0 - 2 + r;
        if (iic >= ni || jj >= nj) continue;
        const long long c = (long long)jj * sj + iic;
        const int i = iic + d.imin - HALO, j = jj + d.jmin - HALO;
        const bool in = i >= d.imin && i <= d.imax && j >= d.jmin && j <= d.jmax;
        const float q4 = 0.25f;
        float uloc, vloc, HHl;
        bool on;
        if (DIR == 0) {
          on = i <= d.imax + HALO - 1 && bf.mask[c] > 0;
          if (!on) continue;
          vloc = in ? __fmul_rn(q4, __fadd_rn(__fadd_rn(__fadd_rn(sm.Q[r][qc], sm.Q[r][qc + 1]), sm.Q[r - 1][qc]),
                                              sm.Q[r - 1][qc + 1]))
                    : 0.f;
          uloc = __fdividef(float(U[c]), float(DU[c]));
          HHl = fmaxf(bf.min_depth, float(DU[c]));
        } else {
          on = j <= d.jmax + HALO - 1 && bf.mask[c] > 0;
          if (!on) continue;
          if (in)
            uloc = __fmul_rn(q4, __fadd_rn(__fadd_rn(__fadd_rn(sm.Q[r][qc], sm.Q[r][qc - 1]), sm.Q[r + 1][qc]),
                                           sm.Q[r + 1][qc - 1]));
          else
            uloc = (i <= d.imax + HALO - 1 && bf.au[c] > 0) ? sm.Q[r][qc] : 0.f;
          vloc = __fdividef(float(V[c]), float(DV[c]));
          HHl = fmaxf(bf.min_depth, float(DV[c]));
        }
        const BfLaw b = bf_law_f32(bf.zb[c], bf.zb0[c], HHl, uloc, vloc, bf.kappa, bf.avmmol, bf.runtype);
        if (bf.runtype == 1) bf.zb[c] = b.zn;
        bf.rr[c] = b.rr;
        bf.r[c] = b.r;
      }
    }
  }
}

template <class T, int S, int DIR, class TI>
__global__ void __launch_bounds__(FT) k_uvadv2d_fused(Dev d, T dt, const TI* __restrict__ U,
                                                      const TI* __restrict__ V, const TI* __restrict__ DU,
                                                      const TI* __restrict__ DV,
                                                      const uint8_t* __restrict__ mflux_u,
                                                      const uint8_t* __restrict__ mflux_v,
                                                      const uint8_t* __restrict__ mupd_u,
                                                      const uint8_t* __restrict__ mupd_v, TI* __restrict__ Ex,
                                                      Bf2Args bf) {
  uvadv2d_tile<T, S, DIR, TI>(d, dt, U, V, DU, DV, mflux_u, mflux_v, mupd_u, mupd_v, Ex, bf);
}

// Both components in one launch (blockIdx.z = 0: UEx on the U grid, 1: VEx on the V grid): the
// same tiles as two k_uvadv2d_fused launches, one grid, one tail. Four blocks per SM (32 registers,
// no spills; the shared memory holds four): the issue-bound sweeps then have 64 warps to choose
// from instead of 48.
struct Adv2dMasks {
  const uint8_t *mflux_u, *mflux_v, *mupd_u, *mupd_v;
};
template <class T, int S, class TI>
__global__ void __launch_bounds__(FT, 4) k_uvadv2d_both(Dev d, T dt, const TI* __restrict__ U, const TI* __restrict__ V,
                                                     const TI* __restrict__ DU, const TI* __restrict__ DV,
                                                     Adv2dMasks mu, Adv2dMasks mv, TI* __restrict__ UEx,
                                                     TI* __restrict__ VEx, Bf2Args bfu, Bf2Args bfv) {
  if (blockIdx.z == 0)
    uvadv2d_tile<T, S, 0, TI>(d, dt, U, V, DU, DV, mu.mflux_u, mu.mflux_v, mu.mupd_u, mu.mupd_v, UEx, bfu);
  else
    uvadv2d_tile<T, S, 1, TI>(d, dt, U, V, DU, DV, mv.mflux_u, mv.mflux_v, mv.mupd_u, mv.mupd_v, VEx, bfv);
}

template <class T, int S, int DIR, class TI>
int launch_uvadv2d_fused(const Dev& d, cudaStream_t s, T dt, const TI* U, const TI* V, const TI* DU, const TI* DV,
                         const uint8_t* mflux_u, const uint8_t* mflux_v, const uint8_t* mupd_u,
                         const uint8_t* mupd_v, TI* Ex, const Bf2Args& bf) {
  const size_t smem = sizeof(Adv2dSmem<T>);
  // opt-in above 48 KB of shared memory (a host-side setting of the current device's function)
  const cudaError_t e = cudaFuncSetAttribute(k_uvadv2d_fused<T, S, DIR, TI>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return (int)e;
  dim3 grd((d.ni() + FX - 1) / FX, (d.nj() + FY - 1) / FY, 1);
  k_uvadv2d_fused<T, S, DIR, TI><<<grd, dim3(RW, FTY, 1), smem, s>>>(d, dt, U, V, DU, DV, mflux_u, mflux_v, mupd_u,
                                                                      mupd_v, Ex, bf);
  return (int)cudaGetLastError();
}

template <class T, class TI>
int run_uvadv2d_fused_t(const Dev& d, cudaStream_t s, int dir, T dt, int scheme, const TI* U, const TI* V,
                        const TI* DU, const TI* DV, const uint8_t* mflux_u, const uint8_t* mflux_v,
                        const uint8_t* mupd_u, const uint8_t* mupd_v, TI* Ex, const Bf2Args& bf) {
  return dispatch_scheme(scheme, [&](auto sc) {
    constexpr int S = decltype(sc)::value;
    return dir == 0
               ? launch_uvadv2d_fused<T, S, 0, TI>(d, s, dt, U, V, DU, DV, mflux_u, mflux_v, mupd_u, mupd_v, Ex, bf)
               : launch_uvadv2d_fused<T, S, 1, TI>(d, s, dt, U, V, DU, DV, mflux_u, mflux_v, mupd_u, mupd_v, Ex, bf);
  });
}

template <class T>
int run_uvadv2d_fused(const Dev& d, cudaStream_t s, int dir, T dt, int scheme, const double* U, const double* V,
                      const double* DU, const double* DV, const uint8_t* mflux_u, const uint8_t* mflux_v,
                      const uint8_t* mupd_u, const uint8_t* mupd_v, double* Ex) {
  return run_uvadv2d_fused_t<T, double>(d, s, dir, dt, scheme, U, V, DU, DV, mflux_u, mflux_v, mupd_u, mupd_v, Ex,
                                        Bf2Args{});
}

// FP32 arithmetic on the FP32 working copies of the mixed-precision micro step (defined in the
// FP32 translation unit only)
#if defined(GB_REAL_IS_FLOAT)

int run_uvadv2d_fused_f32(const Dev& d, cudaStream_t s, int dir, float dt, int scheme, const float* U,
                          const float* V, const float* DU, const float* DV, const uint8_t* mflux_u,
                          const uint8_t* mflux_v, const uint8_t* mupd_u, const uint8_t* mupd_v, float* Ex,
                          const Bf2Args* bf) {
  return run_uvadv2d_fused_t<float, float>(d, s, dir, dt, scheme, U, V, DU, DV, mflux_u, mflux_v, mupd_u, mupd_v,
                                           Ex, bf ? *bf : Bf2Args{});
}

int run_uvadv2d_both_f32(const Dev& d, cudaStream_t s, float dt, int scheme, const float* U, const float* V,
                         const float* DU, const float* DV, const uint8_t* const* mu, const uint8_t* const* mv,
                         float* UEx, float* VEx, const Bf2Args* bfu, const Bf2Args* bfv) {
  return dispatch_scheme(scheme, [&](auto sc) {
    constexpr int S = decltype(sc)::value;
    const size_t smem = sizeof(Adv2dSmem<float>);
    const cudaError_t e = cudaFuncSetAttribute(k_uvadv2d_both<float, S, float>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    dim3 grd((d.ni() + FX - 1) / FX, (d.nj() + FY - 1) / FY, 2);
    k_uvadv2d_both<float, S, float><<<grd, dim3(RW, FTY, 1), smem, s>>>(
        d, dt, U, V, DU, DV, Adv2dMasks{mu[0], mu[1], mu[2], mu[3]}, Adv2dMasks{mv[0], mv[1], mv[2], mv[3]}, UEx,
        VEx, bfu ? *bfu : Bf2Args{}, bfv ? *bfv : Bf2Args{});
    return (int)cudaGetLastError();
  });
}
#endif

}  // namespace gb
