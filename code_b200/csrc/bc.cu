// bc.cu -- the mode-split time step on the device: 2D (barotropic) kernels, the drivers of
// integrate_2d / integrate_3d / the micro-step loop, and their C-ABI entry points.
// Built with --fmad=false: the FP64 arithmetic rounds exactly as written (as in the reference).
#include <algorithm>

#include "bc_common.cuh"
#include "ctx_internal.h"

namespace gb {

#define GB_IJ2                                                          \
  const int i = blockIdx.x * blockDim.x + threadIdx.x + d.imin - HALO; \
  const int j = blockIdx.y * blockDim.y + threadIdx.y + d.jmin - HALO; \
  if (i > d.imax + HALO || j > d.jmax + HALO) return;

struct W2 {
  const Dev& d;
  double* p;
  __device__ double& operator()(int i, int j) const { return p[d.ix(i, j)]; }
};
// a 2D field of the micro step: the FP32 working copy (mixed step) or the FP64 state array
template <class E>
struct A2 {
  const Dev& d;
  E* p;
  __device__ E& operator()(int i, int j) const { return p[d.ix(i, j)]; }
};
template <bool MIX, int Q>
__device__ __forceinline__ auto f2a(const Dev& d, const Bc2& s, const Bc2W& w) {
  if constexpr (MIX && is_work2(Q)) return A2<float>{d, w.w[Q]};
  else return A2<double>{d, s.f2[Q]};
}

struct M2 {
  const Dev& d;
  const int32_t* p;
  __device__ int operator()(int i, int j) const { return p[d.ix(i, j)]; }
};
struct M8 {
  const Dev& d;
  const uint8_t* p;
  __device__ int operator()(int i, int j) const { return p[d.ix(i, j)]; }
};
// mask q (0 az, 1 au, 2 av) of the micro step: the int32 state array, or its uint8 copy (mixed step)
template <bool MIX>
__device__ __forceinline__ auto m2a(const Dev& d, const Bc2& s, const Bc2W& w, int q) {
  if constexpr (MIX) return M8{d, w.m8[q]};
  else return M2{d, q == 0 ? s.az : q == 1 ? s.au : s.av};
}
__device__ __forceinline__ bool interior(const Dev& d, int i, int j) {
  return i >= d.imin && i <= d.imax && j >= d.jmin && j <= d.jmax;
}

// bottom_friction.F90:48-150: ru/rv from the depth-averaged velocities (log-law drag). Arithmetic
// type T: FP64 in the plain step (the reference's expressions and order), FP32 in the mixed step
// (inputs and outputs stay FP64 arrays).
template <class T, bool MIX>
__global__ void k_bottom_friction(Dev d, Bc2 s, Bc2W w, int runtype) {
  GB_IJ2
  auto U = f2a<MIX, U_>(d, s, w);
  auto V = f2a<MIX, V_>(d, s, w);
  auto DU_ = f2a<MIX, DU>(d, s, w);
  auto DV_ = f2a<MIX, DV>(d, s, w);
  auto ruu = f2a<MIX, RUU>(d, s, w);
  auto rvv = f2a<MIX, RVV>(d, s, w);
  auto ru = f2a<MIX, RU>(d, s, w);
  auto rv = f2a<MIX, RV>(d, s, w);
  W2 zub{d, s.f2[ZUB]}, zvb{d, s.f2[ZVB]}, zub0{d, s.f2[ZUB0]}, zvb0{d, s.f2[ZVB0]};
  M2 au{d, s.au}, av{d, s.av};
  const T kappa = T(s.par[P_KAPPA]), avmmol = T(s.par[P_AVMMOL]), min_depth = T(s.par[P_MIN_DEPTH]);
  const T q = T(0.25), h = T(0.5);
  auto qt = [](double a, double b) { return T(a) / T(b); };
  const bool in = interior(d, i, j);
  if (i <= d.imax + HALO - 1 && au(i, j) > 0) {
    // vloc: 4-point average on interior U points (0 elsewhere, as the reference's work array holds)
    const T vloc = in ? q * (qt(V(i, j), DV_(i, j)) + qt(V(i + 1, j), DV_(i + 1, j)) + qt(V(i, j - 1), DV_(i, j - 1)) +
                             qt(V(i + 1, j - 1), DV_(i + 1, j - 1)))
                      : T(0);
    const T uloc = qt(U(i, j), DU_(i, j));
    const T HHl = fmax(min_depth, T(DU_(i, j)));
    const T zb = T(zub(i, j));
    T x = kappa / log((zb + h * HHl) / zb);
    T r = x * x;
    if (runtype == 1) {
      const T fricvel = sqrt(r * (uloc * uloc + vloc * vloc));
      const T zn = fmin(HHl, T(zub0(i, j)) + T(0.1) * avmmol / fmax(avmmol, fricvel));
      zub(i, j) = zn;
      r = (zn + h * HHl) / zn;
      x = kappa / log(r);
      r = x * x;
    }
    ruu(i, j) = r;
    ru(i, j) = r * sqrt(uloc * uloc + vloc * vloc);
  }
  if (j <= d.jmax + HALO - 1 && av(i, j) > 0) {
    // uloc: 4-point average on interior V points; elsewhere the U-point quotient where au > 0
    T uloc;
    if (in)
      uloc = q * (qt(U(i, j), DU_(i, j)) + qt(U(i - 1, j), DU_(i - 1, j)) + qt(U(i, j + 1), DU_(i, j + 1)) +
                  qt(U(i - 1, j + 1), DU_(i - 1, j + 1)));
    else
      uloc = (i <= d.imax + HALO - 1 && au(i, j) > 0) ? qt(U(i, j), DU_(i, j)) : T(0);
    const T vloc = qt(V(i, j), DV_(i, j));
    const T HHl = fmax(min_depth, T(DV_(i, j)));
    const T zb = T(zvb(i, j));
    T x = kappa / log((zb + h * HHl) / zb);
    T r = x * x;
    if (runtype == 1) {
      const T fricvel = sqrt(r * (uloc * uloc + vloc * vloc));
      const T zn = fmin(HHl, T(zvb0(i, j)) + T(0.1) * avmmol / fmax(avmmol, fricvel));
      zvb(i, j) = zn;
      r = (zn + h * HHl) / zn;
      x = kappa / log(r);
      r = x * x;
    }
    rvv(i, j) = r;
    rv(i, j) = r * sqrt(uloc * uloc + vloc * vloc);
  }
}

// FP32 form of k_bottom_friction on a 32x8 tile: the velocity quotients U/DU and V/DV of the tile
// and its one-cell halo are formed once into shared memory (the 4-point averages of the U and V
// points read them from there); the drag itself is bf_law_f32, as in the fused momentum advection.
// MIX: the roughness arrays are the FP32 working copies.
template <bool MIX>
__global__ void __launch_bounds__(256) k_bottom_friction_f32t(Dev d, Bc2 s, Bc2W w, int runtype) {
  __shared__ float suq[10][34], svq[10][34];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = blockIdx.x * 32 + d.imin - HALO, j0 = blockIdx.y * 8 + d.jmin - HALO;
  auto U = f2a<MIX, U_>(d, s, w);
  auto V = f2a<MIX, V_>(d, s, w);
  auto DU_ = f2a<MIX, DU>(d, s, w);
  auto DV_ = f2a<MIX, DV>(d, s, w);
  for (int e = ty * 32 + tx; e < 340; e += 256) {
    const int r = e / 34, q = e % 34;
    const int ii = i0 - 1 + q, jj = j0 - 1 + r;
    float uq = 0.f, vq = 0.f;
    if (ii >= d.imin - HALO && ii <= d.imax + HALO && jj >= d.jmin - HALO && jj <= d.jmax + HALO) {
      uq = __fdividef(float(U(ii, jj)), float(DU_(ii, jj)));
      vq = __fdividef(float(V(ii, jj)), float(DV_(ii, jj)));
    }
    suq[r][q] = uq;
    svq[r][q] = vq;
  }
  __syncthreads();
  const int i = i0 + tx, j = j0 + ty;
  if (i > d.imax + HALO || j > d.jmax + HALO) return;
  auto UQ = [&](int di, int dj) { return suq[ty + 1 + dj][tx + 1 + di]; };
  auto VQ = [&](int di, int dj) { return svq[ty + 1 + dj][tx + 1 + di]; };
  auto ruu = f2a<MIX, RUU>(d, s, w);
  auto rvv = f2a<MIX, RVV>(d, s, w);
  auto ru = f2a<MIX, RU>(d, s, w);
  auto rv = f2a<MIX, RV>(d, s, w);
  auto zub = f2a<MIX, ZUB>(d, s, w);
  auto zvb = f2a<MIX, ZVB>(d, s, w);
  auto zub0 = f2a<MIX, ZUB0>(d, s, w);
  auto zvb0 = f2a<MIX, ZVB0>(d, s, w);
  M2 au{d, s.au}, av{d, s.av};
  const float kappa = float(s.par[P_KAPPA]), avmmol = float(s.par[P_AVMMOL]), min_depth = float(s.par[P_MIN_DEPTH]);
  const float q = 0.25f;
  const bool in = interior(d, i, j);
  if (i <= d.imax + HALO - 1 && au(i, j) > 0) {
    const float vloc = in ? __fmul_rn(q, __fadd_rn(__fadd_rn(__fadd_rn(VQ(0, 0), VQ(1, 0)), VQ(0, -1)), VQ(1, -1))) : 0.f;
    const float HHl = fmaxf(min_depth, float(DU_(i, j)));
    const BfLaw b = bf_law_f32(float(zub(i, j)), float(zub0(i, j)), HHl, UQ(0, 0), vloc, kappa, avmmol, runtype);
    if (runtype == 1) zub(i, j) = b.zn;
    ruu(i, j) = b.rr;
    ru(i, j) = b.r;
  }
  if (j <= d.jmax + HALO - 1 && av(i, j) > 0) {
    float uloc;
    if (in)
      uloc = __fmul_rn(q, __fadd_rn(__fadd_rn(__fadd_rn(UQ(0, 0), UQ(-1, 0)), UQ(0, 1)), UQ(-1, 1)));
    else
      uloc = (i <= d.imax + HALO - 1 && au(i, j) > 0) ? UQ(0, 0) : 0.f;
    const float HHl = fmaxf(min_depth, float(DV_(i, j)));
    const BfLaw b = bf_law_f32(float(zvb(i, j)), float(zvb0(i, j)), HHl, uloc, VQ(0, 0), kappa, avmmol, runtype);
    if (runtype == 1) zvb(i, j) = b.zn;
    rvv(i, j) = b.rr;
    rv(i, j) = b.r;
  }
}

// uv_advect.F90:94-110 (U grid) / :204-220 (V grid): quantities of the 2D momentum volumes, in
// the working type T of the 2D advection (FP64 in the plain step, FP32 in the mixed step), plus
// the control-volume depth Do (= DU or DV) in T.
template <int DIR, class T>
__global__ void k_uvadv2d_prep(Dev d, const double* Up, const double* Vp, const double* DUp, const double* DVp,
                               T* fadv, T* Uadv, T* Vadv, T* DUadv, T* DVadv, T* Do) {
  GB_IJ2
  W2 U{d, const_cast<double*>(Up)}, V{d, const_cast<double*>(Vp)}, DU_{d, const_cast<double*>(DUp)},
      DV_{d, const_cast<double*>(DVp)};
  const long long c = d.ix(i, j);
  if (Do) Do[c] = T(DIR == 0 ? DU_(i, j) : DV_(i, j));
  if (DIR == 0) {
    if (i > d.imax + HALO - 1) return;
    fadv[c] = T(U(i, j) / DU_(i, j));
    Uadv[c] = T(0.5 * (U(i, j) + U(i + 1, j)));
    Vadv[c] = T(0.5 * (V(i, j) + V(i + 1, j)));
    DUadv[c] = T(0.5 * (DU_(i, j) + DU_(i + 1, j)));
    DVadv[c] = T(0.5 * (DV_(i, j) + DV_(i + 1, j)));
  } else {
    if (j > d.jmax + HALO - 1) return;
    fadv[c] = T(V(i, j) / DV_(i, j));
    Uadv[c] = T(0.5 * (U(i, j) + U(i, j + 1)));
    Vadv[c] = T(0.5 * (V(i, j) + V(i, j + 1)));
    DUadv[c] = T(0.5 * (DU_(i, j) + DU_(i, j + 1)));
    DVadv[c] = T(0.5 * (DV_(i, j) + DV_(i, j + 1)));
  }
}

// FP32 advective increments of the mixed step widened into the FP64 UEx / VEx
__global__ void k_widen2d(Dev d, const float* a, double* out) {
  GB_IJ2
  const long long c = d.ix(i, j);
  out[c] = (double)a[c];
}

// NOSPLIT finaliser of the 2D driver (advection.F90:500-507)
template <class T>
__global__ void k_finalise2d(Dev d, T dt, T* f, const T* Do, const T* adv, const T* Di, const uint8_t* mfin) {
  GB_IJ2
  const long long c = d.ix(i, j);
  if (mfin[c]) f[c] = (Do[c] * f[c] - dt * adv[c]) / Di[c];
}

// momentum.F90:157-174 (umomentum, DIR 0) / :319-336 (vmomentum, DIR 1): depth-integrated
// transport update on U (V) points of the interior.
// COR: the kernel first forms the Coriolis term that this update needs from the other velocity
// (fV from V for the U update, fU from U for the V update; the expressions of k_coriolis) at
// every interior point and stores it, then updates its own velocity with it -- one launch where
// the momentum / Coriolis pair took two (the other velocity is not written by this kernel, so no
// point reads a value another thread changes).
template <int DIR, bool MIX, bool COR = false>
__global__ void k_momentum(Dev d, Bc2 s, Bc2W w) {
  GB_IJ2
  if (!interior(d, i, j)) return;
  if constexpr (COR) {
    if (DIR == 0) {  // fV on U points from V
      auto V = f2a<MIX, V_>(d, s, w);
      auto fV = f2a<MIX, FV>(d, s, w);
      W2 coru{d, s.f2[CORU]};
      M2 au{d, s.au};
      if (au(i, j) >= 1) {
        const double Vloc = 0.25 * ((double)V(i, j - 1) + (double)V(i + 1, j - 1) + (double)V(i, j) + (double)V(i + 1, j));
        fV(i, j) = coru(i, j) * Vloc;
      } else {
        fV(i, j) = 0.0;
      }
    } else {  // fU on V points from U
      auto U = f2a<MIX, U_>(d, s, w);
      auto fU = f2a<MIX, FU>(d, s, w);
      W2 corv{d, s.f2[CORV]};
      M2 av{d, s.av};
      if (av(i, j) >= 1) {
        const double Uloc = 0.25 * ((double)U(i - 1, j) + (double)U(i, j) + (double)U(i - 1, j + 1) + (double)U(i, j + 1));
        fU(i, j) = corv(i, j) * Uloc;
      } else {
        fU(i, j) = 0.0;
      }
    }
  }
  M2 mask{d, DIR == 0 ? s.au : s.av};
  if (!(mask(i, j) == 1 || mask(i, j) == 2)) return;
  auto X = f2a<MIX, DIR == 0 ? U_ : V_>(d, s, w);
  auto DX = f2a<MIX, DIR == 0 ? DU : DV>(d, s, w);
  auto D = f2a<MIX, D_>(d, s, w);
  auto airp = f2a<MIX, AIRP>(d, s, w);
  auto taus = f2a<MIX, DIR == 0 ? TAUSX : TAUSY>(d, s, w);
  auto Slr_ = f2a<MIX, DIR == 0 ? SLRU : SLRV>(d, s, w);
  auto dry = f2a<MIX, DIR == 0 ? DRY_U : DRY_V>(d, s, w);
  auto fC = f2a<MIX, DIR == 0 ? FV : FU>(d, s, w);
  auto Ex = f2a<MIX, DIR == 0 ? UEX : VEX>(d, s, w);
  auto Slx = f2a<MIX, DIR == 0 ? SLUX : SLVX>(d, s, w);
  auto r = f2a<MIX, DIR == 0 ? RU : RV>(d, s, w);
  W2 z{d, s.f2[Z]}, H{d, s.f2[HH]};
  const double g = s.par[P_G], rho_0 = s.par[P_RHO_0], dtm = s.par[P_DTM], min_depth = s.par[P_MIN_DEPTH];
  const double gamma = rho_0 * g;
  const double gammai = 1.0 / gamma;
  const int di = DIR == 0 ? 1 : 0, dj = DIR == 0 ? 0 : 1;
  const double zp = fmax(z(i + di, j + dj), -H(i, j) + fmin(min_depth, (double)D(i + di, j + dj)));
  const double zm = fmax(z(i, j), -H(i + di, j + dj) + fmin(min_depth, (double)D(i, j)));
  const double zx = (zp - zm + ((double)airp(i + di, j + dj) - (double)airp(i, j)) * gammai) / (DIR == 0 ? d.dx : d.dy);
  const double tau = 0.5 * ((double)taus(i, j) + (double)taus(i + di, j + dj));
  const double Slr = X(i, j) > 0.0 ? fmax((double)Slr_(i, j), 0.0) : fmin((double)Slr_(i, j), 0.0);
  const double Xo = X(i, j), DXo = DX(i, j), dryo = dry(i, j), fCo = fC(i, j), Exo = Ex(i, j), Slxo = Slx(i, j),
               ro = r(i, j);
  if (DIR == 0)
    X(i, j) = (Xo - dtm * (g * DXo * zx + dryo * (-tau / rho_0 - fCo + Exo + Slxo + Slr))) / (1.0 + dtm * ro / DXo);
  else
    X(i, j) = (Xo - dtm * (g * DXo * zx + dryo * (-tau / rho_0 + fCo + Exo + Slxo + Slr))) / (1.0 + dtm * ro / DXo);
}

// The mixed micro step's form of k_momentum: the same update with the elevation gradient's
// difference zp - zm taken in FP64 (the elevations are FP64) and every other operation in FP32 on
// the FP32 working copies (the Coriolis term with COR as well). Split into the Coriolis term and
// the update of one point (momentum_core_f32 from the point's inputs), which the one- and
// two-point kernels share.
//
// The Coriolis term of the DIR update at c (DIR 0: fV on U points from V at c-sj, c+1-sj, c, c+1;
// DIR 1: fU on V points from U at c-1, c, c-1+sj, c+sj), given those four values in that order.
template <int DIR>
__device__ __forceinline__ float cor_term_f32(const Bc2& s, const Bc2W& w, long long c, float a, float b, float e,
                                              float f) {
  const int m = DIR == 0 ? w.m8[1][c] : w.m8[2][c];
  return m >= 1 ? float(s.f2[DIR == 0 ? CORU : CORV][c]) * (0.25f * (a + b + e + f)) : 0.f;
}
// The new velocity of the DIR update at one point from its inputs: old value Xo, Coriolis term fCo,
// elevation, depth H, total depth D, air pressure and surface stress at the point (c) and at the
// next T point along the component (n), then the point's slow term, face depth, drying factor,
// advection term, slow advection term and drag coefficient.
template <int DIR>
__device__ __forceinline__ float momentum_core_f32(const Dev& d, const Bc2& s, float Xo, float fCo, double zc, double zn,
                                                   float Hc, float Hn, float Dc, float Dn, float ac, float an,
                                                   float tc, float tn, float sl, float DXo, float dryo, float Exo,
                                                   float Slxo, float ro) {
  const float g = float(s.par[P_G]), rho_0 = float(s.par[P_RHO_0]), dtm = float(s.par[P_DTM]);
  const double min_depth = s.par[P_MIN_DEPTH];
  const float gammai = 1.f / (rho_0 * g);
  const double zp = fmax(zn, -(double)Hc + fmin(min_depth, (double)Dn));
  const double zm = fmax(zc, -(double)Hn + fmin(min_depth, (double)Dc));
  const float zx = (float(zp - zm) + (an - ac) * gammai) / float(DIR == 0 ? d.dx : d.dy);
  const float tau = 0.5f * (tc + tn);
  const float Slr = Xo > 0.f ? fmaxf(sl, 0.f) : fminf(sl, 0.f);
  const float fc = DIR == 0 ? -fCo : fCo;
  return (Xo - dtm * (g * DXo * zx + dryo * (-tau / rho_0 + fc + Exo + Slxo + Slr))) / (1.f + dtm * ro / DXo);
}
// The new velocity of the DIR update at an interior point c whose mask is 1 or 2, from its old value
// Xo and the Coriolis term fCo.
template <int DIR>
__device__ __forceinline__ float momentum_new_f32(const Dev& d, const Bc2& s, const Bc2W& w, long long c, float Xo,
                                                  float fCo) {
  const long long dn = DIR == 0 ? 1 : d.sj;  // the next T point along the component
  const float* D = w.w[D_];
  const float* airp = w.w[AIRP];
  const float* taus = w.w[DIR == 0 ? TAUSX : TAUSY];
  const double* z = s.f2[Z];
  const float* H = w.w[HH];
  return momentum_core_f32<DIR>(d, s, Xo, fCo, z[c], z[c + dn], H[c], H[c + dn], D[c], D[c + dn], airp[c],
                                airp[c + dn], taus[c], taus[c + dn], w.w[DIR == 0 ? SLRU : SLRV][c],
                                w.w[DIR == 0 ? DU : DV][c], w.w[DIR == 0 ? DRY_U : DRY_V][c],
                                w.w[DIR == 0 ? UEX : VEX][c], w.w[DIR == 0 ? SLUX : SLVX][c],
                                w.w[DIR == 0 ? RU : RV][c]);
}

template <int DIR, bool COR>
__global__ void k_momentum_f32(Dev d, Bc2 s, Bc2W w) {
  GB_IJ2
  if (!interior(d, i, j)) return;
  const long long c = d.ix(i, j);
  if constexpr (COR) {
    if (DIR == 0) {  // fV on U points from V
      const float* V = w.w[V_];
      w.w[FV][c] = cor_term_f32<0>(s, w, c, V[c - d.sj], V[c + 1 - d.sj], V[c], V[c + 1]);
    } else {  // fU on V points from U
      const float* U = w.w[U_];
      w.w[FU][c] = cor_term_f32<1>(s, w, c, U[c - 1], U[c], U[c - 1 + d.sj], U[c + d.sj]);
    }
  }
  const int m = DIR == 0 ? w.m8[1][c] : w.m8[2][c];
  if (!(m == 1 || m == 2)) return;
  float* X = w.w[DIR == 0 ? U_ : V_];
  X[c] = momentum_new_f32<DIR>(d, s, w, c, X[c], w.w[DIR == 0 ? FV : FU][c]);
}

// k_momentum_f32 on two neighbouring points per thread (region columns 2t and 2t+1 of a row, for
// layouts with an even row pitch): the inputs are loaded as pairs (float2, double2, uchar2), the
// values at the next T point along the component are the pair's second element and one more load
// (DIR 0) or a second pair (DIR 1). The same expressions per point, so the same values.
__device__ __forceinline__ float2 ld_f2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ double2 ld_d2(const double* p) { return *reinterpret_cast<const double2*>(p); }
template <int DIR, bool COR>
__global__ void k_momentum_f32v(Dev d, Bc2 s, Bc2W w) {
  const int ii = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  if (ii >= d.ni() || jj >= d.nj()) return;
  const int i0 = ii + d.imin - HALO, j = jj + d.jmin - HALO;
  const bool in0 = interior(d, i0, j), in1 = interior(d, i0 + 1, j);
  if (!in0 && !in1) return;
  const long long c = (long long)jj * d.sj + ii;
  const long long sj = d.sj;
  const uchar2 mk = *reinterpret_cast<const uchar2*>(w.m8[DIR == 0 ? 1 : 2] + c);
  float* fCp = w.w[DIR == 0 ? FV : FU];
  float fC0, fC1;
  if constexpr (COR) {
    const double2 cor = ld_d2(s.f2[DIR == 0 ? CORU : CORV] + c);
    if (DIR == 0) {  // fV on U points from V at c-sj, c+1-sj, c, c+1
      const float* V = w.w[V_];
      const float2 vs = ld_f2(V + c - sj), vc = ld_f2(V + c);
      const float vs2 = V[c + 2 - sj], vc2 = V[c + 2];
      fC0 = mk.x >= 1 ? float(cor.x) * (0.25f * (vs.x + vs.y + vc.x + vc.y)) : 0.f;
      fC1 = mk.y >= 1 ? float(cor.y) * (0.25f * (vs.y + vs2 + vc.y + vc2)) : 0.f;
    } else {  // fU on V points from U at c-1, c, c-1+sj, c+sj
      const float* U = w.w[U_];
      const float2 uc = ld_f2(U + c), up = ld_f2(U + c + sj);
      const float um = U[c - 1], upm = U[c - 1 + sj];
      fC0 = mk.x >= 1 ? float(cor.x) * (0.25f * (um + uc.x + upm + up.x)) : 0.f;
      fC1 = mk.y >= 1 ? float(cor.y) * (0.25f * (uc.x + uc.y + up.x + up.y)) : 0.f;
    }
  } else {
    const float2 f = ld_f2(fCp + c);
    fC0 = f.x;
    fC1 = f.y;
  }
  const bool u0 = in0 && (mk.x == 1 || mk.x == 2), u1 = in1 && (mk.y == 1 || mk.y == 2);
  float* X = w.w[DIR == 0 ? U_ : V_];
  float r0 = 0.f, r1 = 0.f;
  if (u0 || u1) {
    const float* D = w.w[D_];
    const float* airp = w.w[AIRP];
    const float* taus = w.w[DIR == 0 ? TAUSX : TAUSY];
    const float* H = w.w[HH];
    const double* z = s.f2[Z];
    const float2 Xo = ld_f2(X + c), Hc = ld_f2(H + c), Dc = ld_f2(D + c), ac = ld_f2(airp + c), tc = ld_f2(taus + c);
    const double2 zc = ld_d2(z + c);
    double zn0, zn1;
    float Hn0, Hn1, Dn0, Dn1, an0, an1, tn0, tn1;
    if (DIR == 0) {
      zn0 = zc.y;
      zn1 = z[c + 2];
      Hn0 = Hc.y;
      Hn1 = H[c + 2];
      Dn0 = Dc.y;
      Dn1 = D[c + 2];
      an0 = ac.y;
      an1 = airp[c + 2];
      tn0 = tc.y;
      tn1 = taus[c + 2];
    } else {
      const double2 zn = ld_d2(z + c + sj);
      const float2 Hn = ld_f2(H + c + sj), Dn = ld_f2(D + c + sj), an = ld_f2(airp + c + sj), tn = ld_f2(taus + c + sj);
      zn0 = zn.x;
      zn1 = zn.y;
      Hn0 = Hn.x;
      Hn1 = Hn.y;
      Dn0 = Dn.x;
      Dn1 = Dn.y;
      an0 = an.x;
      an1 = an.y;
      tn0 = tn.x;
      tn1 = tn.y;
    }
    const float2 sl = ld_f2(w.w[DIR == 0 ? SLRU : SLRV] + c), DX = ld_f2(w.w[DIR == 0 ? DU : DV] + c),
                 dry = ld_f2(w.w[DIR == 0 ? DRY_U : DRY_V] + c), Ex = ld_f2(w.w[DIR == 0 ? UEX : VEX] + c),
                 Slx = ld_f2(w.w[DIR == 0 ? SLUX : SLVX] + c), ro = ld_f2(w.w[DIR == 0 ? RU : RV] + c);
    r0 = momentum_core_f32<DIR>(d, s, Xo.x, fC0, zc.x, zn0, Hc.x, Hn0, Dc.x, Dn0, ac.x, an0, tc.x, tn0, sl.x, DX.x,
                                dry.x, Ex.x, Slx.x, ro.x);
    r1 = momentum_core_f32<DIR>(d, s, Xo.y, fC1, zc.y, zn1, Hc.y, Hn1, Dc.y, Dn1, ac.y, an1, tc.y, tn1, sl.y, DX.y,
                                dry.y, Ex.y, Slx.y, ro.y);
  }
  if constexpr (COR) {
    if (in0) fCp[c] = fC0;
    if (in1) fCp[c + 1] = fC1;
  }
  if (u0) X[c] = r0;
  if (u1) X[c + 1] = r1;
}

// momentum.F90:193-216 / :356-379: Coriolis terms fU (after the U update) and fV (after V).
template <int DIR, bool MIX>
__global__ void k_coriolis(Dev d, Bc2 s, Bc2W w) {
  GB_IJ2
  if (!interior(d, i, j)) return;
  if constexpr (MIX) {  // FP32 arithmetic on the working copies, as k_momentum_f32 forms the terms
    const long long c = d.ix(i, j);
    if (DIR == 0) {
      const float* U = w.w[U_];
      w.w[FU][c] = w.m8[2][c] >= 1 ? float(s.f2[CORV][c]) * (0.25f * (U[c - 1] + U[c] + U[c - 1 + d.sj] + U[c + d.sj]))
                                : 0.f;
    } else {
      const float* V = w.w[V_];
      w.w[FV][c] = w.m8[1][c] >= 1 ? float(s.f2[CORU][c]) * (0.25f * (V[c - d.sj] + V[c + 1 - d.sj] + V[c] + V[c + 1]))
                                : 0.f;
    }
    return;
  }
  if (DIR == 0) {  // fU on V points from the new U
    auto U = f2a<MIX, U_>(d, s, w);
    auto fU = f2a<MIX, FU>(d, s, w);
    W2 corv{d, s.f2[CORV]};
    M2 av{d, s.av};
    if (av(i, j) >= 1) {
      const double Uloc = 0.25 * ((double)U(i - 1, j) + (double)U(i, j) + (double)U(i - 1, j + 1) + (double)U(i, j + 1));
      fU(i, j) = corv(i, j) * Uloc;
    } else {
      fU(i, j) = 0.0;
    }
  } else {  // fV on U points from the new V
    auto V = f2a<MIX, V_>(d, s, w);
    auto fV = f2a<MIX, FV>(d, s, w);
    W2 coru{d, s.f2[CORU]};
    M2 au{d, s.au};
    if (au(i, j) >= 1) {
      const double Vloc = 0.25 * ((double)V(i, j - 1) + (double)V(i + 1, j - 1) + (double)V(i, j) + (double)V(i + 1, j));
      fV(i, j) = coru(i, j) * Vloc;
    } else {
      fV(i, j) = 0.0;
    }
  }
}

// m2d.F90:471-472 (Uint, Vint accumulation, FP64) + sealevel.F90:89-112 (zo = z; z update).
template <bool MIX>
__global__ void k_accum_sealevel(Dev d, Bc2 s, Bc2W w, int accumulate) {
  GB_IJ2
  auto U = f2a<MIX, U_>(d, s, w);
  auto V = f2a<MIX, V_>(d, s, w);
  auto fwf = f2a<MIX, FWF>(d, s, w);
  W2 z{d, s.f2[Z]}, zo{d, s.f2[ZO]}, Uint{d, s.f2[UINT]}, Vint{d, s.f2[VINT]};
  auto az = m2a<MIX>(d, s, w, 0);
  const double dtm = s.par[P_DTM];
  if (accumulate) {
    Uint(i, j) = Uint(i, j) + U(i, j);
    Vint(i, j) = Vint(i, j) + V(i, j);
  }
  const double zold = z(i, j);
  zo(i, j) = zold;
  if (interior(d, i, j) && az(i, j) == 1)
    z(i, j) = zold - dtm * (((double)U(i, j) * d.dy - (double)U(i - 1, j) * d.dy) +
                            ((double)V(i, j) * d.dx - (double)V(i, j - 1) * d.dx)) * d.ard1 +
              dtm * fwf(i, j);
}

// depth_update.F90:55-110
template <bool MIX>
__global__ void k_depth_update(Dev d, Bc2 s, Bc2W w) {
  GB_IJ2
  auto D = f2a<MIX, D_>(d, s, w);
  auto DU_ = f2a<MIX, DU>(d, s, w);
  auto DV_ = f2a<MIX, DV>(d, s, w);
  auto dry_u = f2a<MIX, DRY_U>(d, s, w);
  auto dry_v = f2a<MIX, DRY_V>(d, s, w);
  auto H = f2a<MIX, HH>(d, s, w);
  auto HU_ = f2a<MIX, HU>(d, s, w);
  auto HV_ = f2a<MIX, HV>(d, s, w);
  W2 z{d, s.f2[Z]}, zo{d, s.f2[ZO]}, dry_z{d, s.f2[DRY_Z]};
  auto az = m2a<MIX>(d, s, w, 0);
  auto au = m2a<MIX>(d, s, w, 1);
  auto av = m2a<MIX>(d, s, w, 2);
  const double min_depth = s.par[P_MIN_DEPTH], crit_depth = s.par[P_CRIT_DEPTH];
  D(i, j) = z(i, j) + H(i, j);
  if (i <= d.imax + HALO - 1) {
    const double x = fmax(0.25 * (zo(i, j) + zo(i + 1, j) + z(i, j) + z(i + 1, j)), -HU_(i, j) + min_depth);
    DU_(i, j) = x + HU_(i, j);
  }
  if (j <= d.jmax + HALO - 1) {
    const double x = fmax(0.25 * (zo(i, j) + zo(i, j + 1) + z(i, j) + z(i, j + 1)), -HV_(i, j) + min_depth);
    DV_(i, j) = x + HV_(i, j);
  }
  const double d1 = 2 * min_depth;
  const double d2i = 1.0 / (crit_depth - 2 * min_depth);
  if (az(i, j) > 0) dry_z(i, j) = fmax(0.0, fmin(1.0, (D(i, j) - 0.5 * d1) * d2i));
  if (au(i, j) > 0) dry_u(i, j) = fmax(0.0, fmin(1.0, (DU_(i, j) - d1) * d2i));
  if (av(i, j) > 0) dry_v(i, j) = fmax(0.0, fmin(1.0, (DV_(i, j) - d1) * d2i));
}

// k_accum_sealevel and k_depth_update as one launch, for the micro-step loop without open
// boundaries. The elevations ping-pong between the state's z and zo arrays: s.f2[Z] holds the
// elevations before the step and is only read; the new ones go to s.f2[ZO], so the old array is
// exactly the reference's zo = z of sealevel.F90:89 and the caller swaps the two pointers after
// the launch. The depths of a U (V) point need the new elevation of the next T point, which the
// thread forms itself from the same inputs with the same expression (no thread reads a value
// that another writes). Same values as the two kernels, bit for bit. flags: bit 0 accumulates
// Uint/Vint; bit 1 writes the drying factor dry_z, which no micro-step kernel reads: the caller asks
// for it on the micro steps whose state a macro step or the host reads next.
template <bool MIX>
__global__ void k_sealevel_depth(Dev d, Bc2 s, Bc2W w, int flags) {
  const int accumulate = flags & 1;
  GB_IJ2
  auto U = f2a<MIX, U_>(d, s, w);
  auto V = f2a<MIX, V_>(d, s, w);
  auto D = f2a<MIX, D_>(d, s, w);
  auto DU_ = f2a<MIX, DU>(d, s, w);
  auto DV_ = f2a<MIX, DV>(d, s, w);
  auto dry_u = f2a<MIX, DRY_U>(d, s, w);
  auto dry_v = f2a<MIX, DRY_V>(d, s, w);
  auto fwf = f2a<MIX, FWF>(d, s, w);
  auto H = f2a<MIX, HH>(d, s, w);
  auto HU_ = f2a<MIX, HU>(d, s, w);
  auto HV_ = f2a<MIX, HV>(d, s, w);
  W2 zold{d, s.f2[Z]}, znew{d, s.f2[ZO]}, Uint{d, s.f2[UINT]}, Vint{d, s.f2[VINT]}, dry_z{d, s.f2[DRY_Z]};
  auto az = m2a<MIX>(d, s, w, 0);
  auto au = m2a<MIX>(d, s, w, 1);
  auto av = m2a<MIX>(d, s, w, 2);
  const double dtm = s.par[P_DTM];
  // sealevel.F90:94-108 at (ii, jj)
  auto zn = [&](int ii, int jj) -> double {
    const double zo_ = zold(ii, jj);
    if (interior(d, ii, jj) && az(ii, jj) == 1)
      return zo_ - dtm * (((double)U(ii, jj) * d.dy - (double)U(ii - 1, jj) * d.dy) +
                          ((double)V(ii, jj) * d.dx - (double)V(ii, jj - 1) * d.dx)) * d.ard1 +
             dtm * fwf(ii, jj);
    return zo_;
  };
  if (accumulate) {
    Uint(i, j) = Uint(i, j) + U(i, j);
    Vint(i, j) = Vint(i, j) + V(i, j);
  }
  const double z0 = zn(i, j);
  znew(i, j) = z0;
  // depth_update.F90:55-110
  const double min_depth = s.par[P_MIN_DEPTH], crit_depth = s.par[P_CRIT_DEPTH];
  D(i, j) = z0 + H(i, j);
  if (i <= d.imax + HALO - 1) {
    const double x = fmax(0.25 * (zold(i, j) + zold(i + 1, j) + z0 + zn(i + 1, j)), -HU_(i, j) + min_depth);
    DU_(i, j) = x + HU_(i, j);
  }
  if (j <= d.jmax + HALO - 1) {
    const double x = fmax(0.25 * (zold(i, j) + zold(i, j + 1) + z0 + zn(i, j + 1)), -HV_(i, j) + min_depth);
    DV_(i, j) = x + HV_(i, j);
  }
  const double d1 = 2 * min_depth;
  const double d2i = 1.0 / (crit_depth - 2 * min_depth);
  if ((flags & 2) && az(i, j) > 0) dry_z(i, j) = fmax(0.0, fmin(1.0, (D(i, j) - 0.5 * d1) * d2i));
  if (au(i, j) > 0) dry_u(i, j) = fmax(0.0, fmin(1.0, (DU_(i, j) - d1) * d2i));
  if (av(i, j) > 0) dry_v(i, j) = fmax(0.0, fmin(1.0, (DV_(i, j) - d1) * d2i));
}

// k_sealevel_depth<true> on two neighbouring points per thread (region columns 2t and 2t+1 of a row,
// even row pitch): paired loads of the FP32 working copies, the FP64 elevations and the masks; the
// new elevations of the pair, of the next point along the row and of the pair in the next row are
// formed once each (the one-point form forms three per point). The same expressions, so the same
// values; every load stays inside the haloed plane (the conditions are those of the one-point form).
__global__ void k_sealevel_depth_p(Dev d, Bc2 s, Bc2W w, int flags) {
  const int ii = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  if (ii >= d.ni() || jj >= d.nj()) return;
  const int i = ii + d.imin - HALO, j = jj + d.jmin - HALO;  // the pair's points: i, i+1
  const long long c = (long long)jj * d.sj + ii, sj = d.sj;
  const float *U = w.w[U_], *V = w.w[V_], *fwf = w.w[FWF], *H = w.w[HH], *HUa = w.w[HU], *HVa = w.w[HV];
  float *D = w.w[D_], *DUa = w.w[DU], *DVa = w.w[DV], *dry_u = w.w[DRY_U], *dry_v = w.w[DRY_V];
  const double* zold = s.f2[Z];
  const uint8_t *az = w.m8[0], *au = w.m8[1], *av = w.m8[2];
  const double dtm = s.par[P_DTM];
  // sealevel.F90:94-108 from a point's inputs
  auto zn_of = [&](bool upd, double zo_, float u0, float um, float v0, float vm, float f) -> double {
    return upd ? zo_ - dtm * (((double)u0 * d.dy - (double)um * d.dy) + ((double)v0 * d.dx - (double)vm * d.dx)) *
                           d.ard1 +
                     dtm * f
               : zo_;
  };
  const bool lastcol = i + 1 > d.imax + HALO - 1;  // the pair's second point has no DU (i+1 = imax+2)
  const bool dvrow = j <= d.jmax + HALO - 1;
  // row j: the pair and the point after it
  const bool in0 = interior(d, i, j), in1 = interior(d, i + 1, j), in2 = interior(d, i + 2, j);
  const double2 zo = ld_d2(zold + c);
  const uchar2 a01 = *reinterpret_cast<const uchar2*>(az + c);
  double z0, z1, z2 = 0.0, zo2 = 0.0;
  {
    float2 u = make_float2(0.f, 0.f), v = u, vs = u, f = u;
    float um = 0.f;
    if (in0 || in1 || in2) {  // (the point after the pair reads U at i+1)
      u = ld_f2(U + c);
      v = ld_f2(V + c);
      vs = ld_f2(V + c - sj);
      f = ld_f2(fwf + c);
    }
    if (in0) um = U[c - 1];
    z0 = zn_of(in0 && a01.x == 1, zo.x, u.x, um, v.x, vs.x, f.x);
    z1 = zn_of(in1 && a01.y == 1, zo.y, u.y, u.x, v.y, vs.y, f.y);
    if (!lastcol) {
      zo2 = zold[c + 2];
      if (in2 && az[c + 2] == 1) z2 = zn_of(true, zo2, U[c + 2], u.y, V[c + 2], V[c + 2 - sj], fwf[c + 2]);
      else z2 = zo2;
    }
  }
  // row j+1: the pair
  double2 zoN = make_double2(0.0, 0.0);
  double zN0 = 0.0, zN1 = 0.0;
  if (dvrow) {
    const bool n0 = interior(d, i, j + 1), n1 = interior(d, i + 1, j + 1);
    zoN = ld_d2(zold + c + sj);
    const uchar2 aN = *reinterpret_cast<const uchar2*>(az + c + sj);
    float2 u = make_float2(0.f, 0.f), v = u, vs = u, f = u;
    float um = 0.f;
    if (n0 || n1) {
      u = ld_f2(U + c + sj);
      v = ld_f2(V + c + sj);
      vs = ld_f2(V + c);
      f = ld_f2(fwf + c + sj);
    }
    if (n0) um = U[c - 1 + sj];
    zN0 = zn_of(n0 && aN.x == 1, zoN.x, u.x, um, v.x, vs.x, f.x);
    zN1 = zn_of(n1 && aN.y == 1, zoN.y, u.y, u.x, v.y, vs.y, f.y);
  }
  if (flags & 1) {
    double2 ui = ld_d2(s.f2[UINT] + c), vi = ld_d2(s.f2[VINT] + c);
    const float2 u = ld_f2(U + c), v = ld_f2(V + c);
    ui.x = ui.x + u.x;
    ui.y = ui.y + u.y;
    vi.x = vi.x + v.x;
    vi.y = vi.y + v.y;
    *reinterpret_cast<double2*>(s.f2[UINT] + c) = ui;
    *reinterpret_cast<double2*>(s.f2[VINT] + c) = vi;
  }
  *reinterpret_cast<double2*>(s.f2[ZO] + c) = make_double2(z0, z1);
  // depth_update.F90:55-110
  const double min_depth = s.par[P_MIN_DEPTH], crit_depth = s.par[P_CRIT_DEPTH];
  const float2 Hc = ld_f2(H + c), HUc = ld_f2(HUa + c), HVc = ld_f2(HVa + c);
  const float2 Dn = make_float2(float(z0 + Hc.x), float(z1 + Hc.y));
  *reinterpret_cast<float2*>(D + c) = Dn;
  float2 DUn, DVn;
  DUn.x = float(fmax(0.25 * (zo.x + zo.y + z0 + z1), -HUc.x + min_depth) + HUc.x);
  if (!lastcol) {
    DUn.y = float(fmax(0.25 * (zo.y + zo2 + z1 + z2), -HUc.y + min_depth) + HUc.y);
    *reinterpret_cast<float2*>(DUa + c) = DUn;
  } else {
    DUa[c] = DUn.x;
    DUn.y = DUa[c + 1];  // not updated at imax+2, as in the one-point form
  }
  if (dvrow) {
    DVn.x = float(fmax(0.25 * (zo.x + zoN.x + z0 + zN0), -HVc.x + min_depth) + HVc.x);
    DVn.y = float(fmax(0.25 * (zo.y + zoN.y + z1 + zN1), -HVc.y + min_depth) + HVc.y);
    *reinterpret_cast<float2*>(DVa + c) = DVn;
  } else {
    DVn = ld_f2(DVa + c);
  }
  const double d1 = 2 * min_depth;
  const double d2i = 1.0 / (crit_depth - 2 * min_depth);
  if (flags & 2) {
    if (a01.x > 0) s.f2[DRY_Z][c] = fmax(0.0, fmin(1.0, ((double)Dn.x - 0.5 * d1) * d2i));
    if (a01.y > 0) s.f2[DRY_Z][c + 1] = fmax(0.0, fmin(1.0, ((double)Dn.y - 0.5 * d1) * d2i));
  }
  const uchar2 mu = *reinterpret_cast<const uchar2*>(au + c), mv = *reinterpret_cast<const uchar2*>(av + c);
  if (mu.x > 0) dry_u[c] = float(fmax(0.0, fmin(1.0, ((double)DUn.x - d1) * d2i)));
  if (mu.y > 0) dry_u[c + 1] = float(fmax(0.0, fmin(1.0, ((double)DUn.y - d1) * d2i)));
  if (mv.x > 0) dry_v[c] = float(fmax(0.0, fmin(1.0, ((double)DVn.x - d1) * d2i)));
  if (mv.y > 0) dry_v[c + 1] = float(fmax(0.0, fmin(1.0, ((double)DVn.y - d1) * d2i)));
}

// exchanges the contents of two 2D FP64 arrays (the elevation ping-pong's last state)
__global__ void k_swap2(long long n2, double* a, double* b) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n2; c += (long long)gridDim.x * blockDim.x) {
    const double x = a[c];
    a[c] = b[c];
    b[c] = x;
  }
}

// start_macro.F90:54-86, first loop (T points) ...
__global__ void k_start_macro_t(Dev d, Bc2 s) {
  GB_IJ2
  W2 sseo{d, s.f2[SSEO]}, ssen{d, s.f2[SSEN]}, z{d, s.f2[Z]}, Dn{d, s.f2[DN]}, H{d, s.f2[HH]};
  sseo(i, j) = ssen(i, j);
  ssen(i, j) = z(i, j);
  Dn(i, j) = ssen(i, j) + H(i, j);
}
// ... then U and V points and Uint/M, Vint/M
__global__ void k_start_macro_uv(Dev d, Bc2 s, double split) {
  GB_IJ2
  W2 sseo{d, s.f2[SSEO]}, ssen{d, s.f2[SSEN]}, ssuo{d, s.f2[SSUO]}, ssun{d, s.f2[SSUN]}, HU_{d, s.f2[HU]},
      Dun{d, s.f2[DUN]}, ssvo{d, s.f2[SSVO]}, ssvn{d, s.f2[SSVN]}, HV_{d, s.f2[HV]}, Dvn{d, s.f2[DVN]},
      Uint{d, s.f2[UINT]}, Vint{d, s.f2[VINT]};
  const double min_depth = s.par[P_MIN_DEPTH];
  if (i <= d.imax + HALO - 1) {
    ssuo(i, j) = ssun(i, j);
    double v = 0.25 * (sseo(i, j) + sseo(i + 1, j) + ssen(i, j) + ssen(i + 1, j));
    v = fmax(v, -HU_(i, j) + min_depth);
    ssun(i, j) = v;
    Dun(i, j) = v + HU_(i, j);
  }
  if (j <= d.jmax + HALO - 1) {
    ssvo(i, j) = ssvn(i, j);
    double v = 0.25 * (sseo(i, j) + sseo(i, j + 1) + ssen(i, j) + ssen(i, j + 1));
    v = fmax(v, -HV_(i, j) + min_depth);
    ssvn(i, j) = v;
    Dvn(i, j) = v + HV_(i, j);
  }
  Uint(i, j) = split * Uint(i, j);
  Vint(i, j) = split * Vint(i, j);
}

// slow_bottom_friction.F90:53-93: depth-averaged velocities of the last macro step (scratch Ui/Vi)
__global__ void k_sbf_uv(Dev d, Bc2 s, double* Uip, double* Vip) {
  GB_IJ2
  W2 Uinto{d, s.f2[UINTO]}, Vinto{d, s.f2[VINTO]}, ssuo{d, s.f2[SSUO]}, ssvo{d, s.f2[SSVO]}, HU_{d, s.f2[HU]},
      HV_{d, s.f2[HV]}, Ui{d, Uip}, Vi{d, Vip};
  M2 au{d, s.au}, av{d, s.av};
  const bool in = interior(d, i, j);
  if (in)
    Ui(i, j) = au(i, j) >= 1 ? Uinto(i, j) / (ssuo(i, j) + HU_(i, j)) : 0.0;
  else
    Ui(i, j) = (j == d.jmax + 1 || i == d.imin - 1) ? Uinto(i, j) / (ssuo(i, j) + HU_(i, j)) : 0.0;
  if (in)
    Vi(i, j) = av(i, j) >= 1 ? Vinto(i, j) / (ssvo(i, j) + HV_(i, j)) : 0.0;
  else
    Vi(i, j) = (j == d.jmin - 1 || i == d.imax + 1) ? Vinto(i, j) / (ssvo(i, j) + HV_(i, j)) : 0.0;
}

// slow_bottom_friction.F90:95-170: ru, rv of the slow (macro) friction. Counts non-positive log
// arguments (the reference stops with 'Bottom friction coefficient infinite').
__global__ void k_sbf_r(Dev d, Bc2 s, const double* Uip, const double* Vip, unsigned long long* bad) {
  GB_IJ2
  if (!interior(d, i, j)) return;
  W2 ssun{d, s.f2[SSUN]}, ssvn{d, s.f2[SSVN]}, HU_{d, s.f2[HU]}, HV_{d, s.f2[HV]}, zub{d, s.f2[ZUB]},
      zvb{d, s.f2[ZVB]}, ru{d, s.f2[RU]}, rv{d, s.f2[RV]}, Ui{d, const_cast<double*>(Uip)},
      Vi{d, const_cast<double*>(Vip)};
  M2 au{d, s.au}, av{d, s.av};
  const double kappa = s.par[P_KAPPA], min_depth = s.par[P_MIN_DEPTH];
  if (au(i, j) >= 1) {
    const double HHl = fmax(min_depth, ssun(i, j) + HU_(i, j));
    double r = (zub(i, j) + 0.5 * HHl) / zub(i, j);
    if (!(r > 1.0)) atomicAdd(bad, 1ull);
    const double x = kappa / log(r);
    r = x * x;
    const double uloc = Ui(i, j);
    const double vloc = 0.25 * (Vi(i, j) + Vi(i + 1, j) + Vi(i, j - 1) + Vi(i + 1, j - 1));
    ru(i, j) = r * sqrt(uloc * uloc + vloc * vloc);
  } else {
    ru(i, j) = 0.0;
  }
  if (av(i, j) >= 1) {
    const double HHl = fmax(min_depth, ssvn(i, j) + HV_(i, j));
    double r = (zvb(i, j) + 0.5 * HHl) / zvb(i, j);
    if (!(r > 1.0)) atomicAdd(bad, 1ull);
    const double x = kappa / log(r);
    r = x * x;
    const double uloc = 0.25 * (Ui(i, j) + Ui(i - 1, j) + Ui(i, j + 1) + Ui(i - 1, j + 1));
    const double vloc = Vi(i, j);
    rv(i, j) = r * sqrt(uloc * uloc + vloc * vloc);
  } else {
    rv(i, j) = 0.0;
  }
}

// update_2d_bdy.F90:74-178: elevations of the open-boundary points [p0, p1) of one side (sides are
// launched in the reference's order W, N, E, S). Harmonic data: amp*sin(2*pi*loop*dtm/period+phase).
__global__ void k_bdy2d(Dev d, Bc2 s, const int4* __restrict__ pts, int p0, int p1, const double* data,
                        const double* data_u, const double* data_v, const double* amp, const double* phase,
                        double period, double fac, int loop) {
  const int p = p0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= p1) return;
  W2 z{d, s.f2[Z]}, D{d, s.f2[D_]}, U{d, s.f2[U_]}, DU_{d, s.f2[DU]}, V{d, s.f2[V_]}, DV_{d, s.f2[DV]},
      H{d, s.f2[HH]};
  const int4 q = pts[p];
  const int i = q.x, j = q.y, type = q.z, side = q.w;
  const double dtm = s.par[P_DTM], min_depth = s.par[P_MIN_DEPTH];
  const double g = (double)9.81f;  // the single-precision literal of update_2d_bdy.F90:92,96
  double bd;
  if (amp) {
    const double pi2 = 2.0 * 3.14159265358979323846;
    bd = amp[p] * sin(pi2 * (loop * dtm) / period + phase[p]);
  } else {
    bd = data[p];
  }
  const double bu = data_u ? data_u[p] : 0.0, bv = data_v ? data_v[p] : 0.0;
  double zn = z(i, j);
  switch (side) {
    case 0:  // western
      if (type == 1) zn = z(i + 1, j);
      else if (type == 2) zn = z(i, j) + dtm / d.dx * sqrt(g * D(i, j)) * (z(i + 1, j) - z(i, j));
      else if (type == 3) zn = fmax(fac * bd, -H(i, j) + min_depth);
      else {
        const double a = sqrt(DU_(i, j) / g) * (U(i, j) / DU_(i, j) - bu);
        zn = fmax(fac * (bd - a), -H(i, j) + min_depth);
      }
      break;
    case 1:  // northern
      if (type == 1) zn = z(i, j - 1);
      else if (type == 2) zn = z(i, j) - dtm / d.dy * sqrt(g * D(i, j)) * (z(i, j) - z(i, j - 1));
      else if (type == 3) zn = fmax(fac * bd, -H(i, j) + min_depth);
      else {
        const double a = sqrt(DV_(i, j) / g) * (V(i, j - 1) / DV_(i, j - 1) - bv);
        zn = fmax(fac * (bd + a), -H(i, j) + min_depth);
      }
      break;
    case 2:  // eastern
      if (type == 1) zn = z(i - 1, j);
      else if (type == 2) zn = z(i, j) - dtm / d.dx * sqrt(g * D(i, j)) * (z(i, j) - z(i - 1, j));
      else if (type == 3) zn = fmax(fac * bd, -H(i, j) + min_depth);
      else {
        const double a = sqrt(DU_(i, j) / g) * (U(i - 1, j) / DU_(i - 1, j) - bu);
        zn = fmax(fac * (bd + a), -H(i, j) + min_depth);
      }
      break;
    default:  // southern
      if (type == 1) zn = z(i, j + 1);
      else if (type == 2) zn = z(i, j) + dtm / d.dy * sqrt(g * D(i, j)) * (z(i, j + 1) - z(i, j));
      else if (type == 3) zn = fmax(fac * bd, -H(i, j) + min_depth);
      else {
        const double a = sqrt(DV_(i, j) / g) * (V(i, j) / DV_(i, j) - bv);
        zn = fmax(fac * (bd - a), -H(i, j) + min_depth);
      }
      break;
  }
  z(i, j) = zn;
}

// mirror_bdy_2d.F90 / mirror_bdy_3d.F90: f(dst) = f(src) for the (dst, src) 2D offsets of one side,
// on nl levels with stride sk.
template <class T>
__global__ void k_mirror(T* f, const long long* __restrict__ pairs, int n, int nl, long long sk) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const long long dst = pairs[2 * p], src = pairs[2 * p + 1];
  for (int k = 0; k < nl; ++k) f[dst + k * sk] = f[src + k * sk];
}

// sealevel.F90:172-314 (sealevel_nan_check): counts the interior elevations that are not below
// HUGE (NaN, +Inf, the largest double) into cnt[0] and keeps in cnt[1] one more than the largest
// loop-order index (j outer, i inner) of such a point, i.e. the last one the reference reports.
// With `latched`, cnt[2] != 0 (a finding of an earlier sweep: the reference's have_warned) skips the
// sweep.
__global__ void k_nan_sweep(Dev d, const double* __restrict__ z, unsigned long long* cnt, bool latched) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + d.imin;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + d.jmin;
  if (i > d.imax || j > d.jmax) return;
  if (latched && cnt[2] != 0) return;
  const double v = z[d.ix(i, j)];
  if (!(1.7976931348623157e308 > v)) {
    atomicAdd(&cnt[0], 1ull);
    const unsigned long long idx =
        (unsigned long long)(j - d.jmin) * (unsigned long long)(d.imax - d.imin + 1) + (unsigned long long)(i - d.imin);
    atomicMax(&cnt[1], idx + 1);
  }
}

// Restart fields (hotstart): the interior (imin..imax, jmin..jmax; levels 0..nl-1) of a field of
// type R to or from a packed FP64 buffer [level][j][i] -- the extent of a restart file without halos
// (cppdefs.h:161-170, _2D_W_HOT_ / _3D_W_HOT_).
template <class R>
__global__ void k_interior_copy(Dev d, R* f, double* buf, int nl, int to_buf) {
  const int nx = d.imax - d.imin + 1, ny = d.jmax - d.jmin + 1;
  const long long n = (long long)nx * ny * nl;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = d.imin + (int)(t % nx);
    const long long r = t / nx;
    const int j = d.jmin + (int)(r % ny), k = (int)(r / ny);
    const long long c = d.ix(i, j) + (long long)k * d.sk;
    if (to_buf) buf[t] = (double)f[c];
    else f[c] = (R)buf[t];
  }
}

// postinit_2d (m2d.F90:358-390), first half: flag[0] = 1 if any U /= 0 where au == 0 or V /= 0 where
// av == 0 (haloed plane)
__global__ void k_hot_check(Dev d, Bc2 s, unsigned long long* flag) {
  GB_IJ2
  M2 au{d, s.au}, av{d, s.av};
  W2 U{d, s.f2[U_]}, V{d, s.f2[V_]};
  if ((au(i, j) == 0 && U(i, j) != 0.0) || (av(i, j) == 0 && V(i, j) != 0.0)) atomicOr(flag, 1ull);
}

// postinit_2d (m2d.F90:380-396): the reset of U, Uinto / V, Vinto on closed velocity points when the
// check found any, and the elevations of land points set to -9999
__global__ void k_hot_reset2d(Dev d, Bc2 s, const unsigned long long* flag) {
  GB_IJ2
  M2 az{d, s.az}, au{d, s.au}, av{d, s.av};
  W2 U{d, s.f2[U_]}, V{d, s.f2[V_]}, Uinto{d, s.f2[UINTO]}, Vinto{d, s.f2[VINTO]}, z{d, s.f2[Z]}, zo{d, s.f2[ZO]};
  if (*flag) {
    if (au(i, j) == 0) {
      U(i, j) = 0.0;
      Uinto(i, j) = 0.0;
    }
    if (av(i, j) == 0) {
      V(i, j) = 0.0;
      Vinto(i, j) = 0.0;
    }
  }
  if (az(i, j) == 0) {
    z(i, j) = -9999.0;
    zo(i, j) = -9999.0;
  }
}

// postinit_3d (m3d.F90:376-405): uu = 0 on closed U points, vv = 0 on closed V points, and on land
// tke = 0, num = nuh = 1e-15 (single-precision literal), T = S = -9999; every level
template <class R3>
__global__ void k_hot_reset3d(Dev d, Bc2 s, R3* uu, R3* vv, R3* tke, R3* num, R3* nuh, R3* T, R3* S) {
  GB_IJ2
  M2 az{d, s.az}, au{d, s.au}, av{d, s.av};
  const long long c = d.ix(i, j);
  for (int k = 0; k <= d.kmax; ++k) {
    const long long q = c + (long long)k * d.sk;
    if (au(i, j) == 0) uu[q] = R3(0);
    if (av(i, j) == 0) vv[q] = R3(0);
    if (az(i, j) == 0) {
      if (tke) tke[q] = R3(0);
      num[q] = R3((double)1.e-15f);
      nuh[q] = R3((double)1.e-15f);
      S[q] = R3(-9999.0);
      T[q] = R3(-9999.0);
    }
  }
}

// stop_macro.F90:36-39
__global__ void k_stop_macro(Dev d, Bc2 s) {
  GB_IJ2
  W2 Uint{d, s.f2[UINT]}, Vint{d, s.f2[VINT]}, Uinto{d, s.f2[UINTO]}, Vinto{d, s.f2[VINTO]};
  Uinto(i, j) = Uint(i, j);
  Uint(i, j) = 0.0;
  Vinto(i, j) = Vint(i, j);
  Vint(i, j) = 0.0;
}

}  // namespace gb

namespace gb {

// after a sweep: a finding ends the sweeps (the reference's have_warned)
__global__ void k_nan_latch(unsigned long long* cnt) {
  if (cnt[0] != 0) cnt[2] = 1;
}

// one sweep into cnt[0..1] that neither reads nor sets a latch (getm_sealevel_nan_check)
int run_nan_sweep_once(const Dev& d, cudaStream_t s, const double* z, unsigned long long* cnt) {
  const dim3 blk(32, 4, 1);
  const dim3 g((d.imax - d.imin + 1 + 31) / 32, (d.jmax - d.jmin + 1 + 3) / 4, 1);
  k_nan_sweep<<<g, blk, 0, s>>>(d, z, cnt, false);
  return (int)cudaGetLastError();
}

int run_nan_sweep(const Dev& d, cudaStream_t s, const double* z, unsigned long long* cnt) {
  const dim3 blk(32, 4, 1);
  const dim3 g((d.imax - d.imin + 1 + 31) / 32, (d.jmax - d.jmin + 1 + 3) / 4, 1);
  k_nan_sweep<<<g, blk, 0, s>>>(d, z, cnt, true);
  k_nan_latch<<<1, 1, 0, s>>>(cnt);
  return (int)cudaGetLastError();
}

}  // namespace gb

// =============================================================================================
// host side
namespace {

using namespace gb;

const dim3 kBlk2(32, 4, 1);
dim3 grid2(const Dev& d) { return dim3((d.ni() + 31) / 32, (d.nj() + 3) / 4, 1); }

Bc2 to_bc2(const getm_bc_state* st) {
  Bc2 s;
  for (int q = 0; q < NF2; ++q) s.f2[q] = st->f2[q];
  s.az = st->az; s.au = st->au; s.av = st->av; s.ax = st->ax;
  for (int q = 0; q < NPD; ++q) s.par[q] = st->par[q];
  return s;
}

template <class R3>
Bc3<R3> to_bc3(const getm_bc_state* st) {
  Bc3<R3> s;
  for (int q = 0; q < NF2; ++q) s.f2[q] = st->f2[q];
  for (int q = 0; q < NF3; ++q) s.f3[q] = (R3*)st->f3[q];
  s.az = st->az; s.au = st->au; s.av = st->av; s.ax = st->ax;
  for (int q = 0; q < NPD; ++q) s.par[q] = st->par[q];
  return s;
}

int check_state(getm_ctx* ctx, const getm_bc_state* st) {
  if (!ctx || !st) return GETM_ERR_ARG;
  if (!ctx->adv_ready) return fail(ctx, GETM_ERR_STATE, "getm_init_advection has not been called");
  if (st->prec3d != 8 && st->prec3d != 4) return fail(ctx, GETM_ERR_ARG, "getm_bc_state.prec3d must be 8 or 4");
  const int* ip = st->ipar;
  for (int q = 0; q < NF2; ++q)
    if (!st->f2[q] && !(optional_f2(q) && !ip[I_RADIATION]))
      return fail(ctx, GETM_ERR_ARG, "getm_bc_state: null 2D field");
  for (int q = 0; q < NF3; ++q)
    if (!st->f3[q] && !(optional_f3(q) && (q != RAD || !ip[I_RADIATION])))
      return fail(ctx, GETM_ERR_ARG, "getm_bc_state: null 3D field");
  if (ip[I_VISCOSITY] != 0 && ip[I_VISCOSITY] != 1)
    return fail(ctx, GETM_ERR_ARG, "viscosity must be 0 (CONSTANT_VISCOSITY) or 1 (PARABOLIC_VISCOSITY)");
  if (ip[I_EQSTATE_METHOD] < 1 || ip[I_EQSTATE_METHOD] > 3)
    return fail(ctx, GETM_ERR_ARG, "eqstate_method must be 1..3 (eqstate.F90:56-68)");
  if (ip[I_RADIATION] != 0 && ip[I_RADIATION] != 1) return fail(ctx, GETM_ERR_ARG, "radiation must be 0 or 1");
  if (!st->az || !st->au || !st->av || !st->ax) return fail(ctx, GETM_ERR_ARG, "getm_bc_state: null mask");
  if (st->ipar[I_RUNTYPE] != 4 && st->ipar[I_RUNTYPE] != 2 && st->ipar[I_RUNTYPE] != 1 && st->ipar[I_RUNTYPE] != 3)
    return fail(ctx, GETM_ERR_ARG, "runtype must be 1..4");
  if (st->ipar[I_M] < 1 || st->ipar[I_MM] < 1) return fail(ctx, GETM_ERR_ARG, "M and MM must be >= 1");
  if (st->ipar[I_IP_METHOD] < 1 || st->ipar[I_IP_METHOD] > 7)
    return fail(ctx, GETM_ERR_ARG, "ip_method must be 1..7 (internal_pressure.F90:149-168)");
  if (st->ipar[I_IP_METHOD] == 7 && ctx->dom.kmax > 64)  // the work arrays of k_svk_cols (SVK_KMAX)
    return fail(ctx, GETM_ERR_UNSUPPORTED, "ip_method 7 (STELLING_VANKESTER): at most 64 levels");
  if ((size_t)2 * (ctx->dom.kmax + 1) * 64 * sizeof(double) > 200 * 1024)
    return fail(ctx, GETM_ERR_UNSUPPORTED, "kmax too large for the column solvers");
  return GETM_OK;
}

// mirror_bdy copies of one tag (0 U, 1 V, 2 H/D) on a 2D (nl = 1) or 3D (nl = kmax+1) field, side
// by side in the reference's order.
template <class T>
int mirror_bdy(getm_ctx* ctx, T* f, int tag, int nl) {
  if (!ctx->has_bdy) return GETM_OK;
  const auto& b = ctx->bdy;
  for (int side = 0; side < 4; ++side) {
    const int p0 = b.pair_first[tag][side], p1 = b.pair_first[tag][side + 1];
    if (p1 <= p0) continue;
    TimerScope ts(ctx, nl > 1 ? GETM_TIM_BC3D : GETM_TIM_BC2D);
    k_mirror<T><<<(p1 - p0 + 127) / 128, 128, 0, ctx->stream>>>(f, b.pairs + 2 * (long long)p0, p1 - p0, nl,
                                                                ctx->dev.sk);
    GB_TRY(cudaGetLastError(), "mirror_bdy");
  }
  return GETM_OK;
}

// update_2d_bdy (m2d.F90:475)
int bdy_2d(getm_ctx* ctx, const Bc2& s, int loop) {
  if (!ctx->has_bdy) return GETM_OK;
  const auto& b = ctx->bdy;
  double fac = 1.0;
  if (b.ramp > 1) fac = fmin(1.0, 4.0 * loop / (double)(float)b.ramp);
  for (int side = 0; side < 4; ++side) {
    const int p0 = b.side_first[side], p1 = b.side_first[side + 1];
    if (p1 <= p0) continue;
    TimerScope ts(ctx, GETM_TIM_BC2D);
    k_bdy2d<<<(p1 - p0 + 127) / 128, 128, 0, ctx->stream>>>(ctx->dev, s, b.pts, p0, p1, b.data, b.data_u, b.data_v,
                                                            b.harmonic ? b.amp : nullptr, b.phase, b.period, fac,
                                                            loop);
    GB_TRY(cudaGetLastError(), "update_2d_bdy");
  }
  return GETM_OK;
}

int ensure_bc_scratch(getm_ctx* ctx, size_t elem3) {
  const long long n3 = n3d(ctx->dev), n2 = n2d(ctx->dev);
  const size_t b3 = (size_t)(elem3 == 4 ? NB3F : NB3) * n3 * elem3;
  if (ctx->bc_scr3_bytes < b3) {
    if (ctx->bc_scr3) cudaFree(ctx->bc_scr3);
    ctx->bc_scr3 = nullptr;
    ctx->bc_scr3_bytes = 0;
    if (cudaMalloc(&ctx->bc_scr3, b3) != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, GETM_ERR_NOMEM, "mode-split 3D scratch allocation failed");
    }
    cudaMemsetAsync(ctx->bc_scr3, 0, b3, ctx->stream);
    ctx->bc_scr3_bytes = b3;
  }
  if (!ctx->bc_scr2) {
    if (cudaMalloc(&ctx->bc_scr2, (size_t)NB2 * n2 * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, GETM_ERR_NOMEM, "mode-split 2D scratch allocation failed");
    }
    cudaMemsetAsync(ctx->bc_scr2, 0, (size_t)NB2 * n2 * sizeof(double), ctx->stream);
  }
  if (!ctx->colh) {
    if (cudaMalloc(&ctx->colh, (size_t)NCOLH * n2 * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, GETM_ERR_NOMEM, "mode-split column-height allocation failed");
    }
  }
  return GETM_OK;
}

// do_advection (advection.F90:362-702) on 2D fields of type T, split schemes, with advres:
// p_Di starts as Do (read by the first sweep), p_adv = 0. f is a work field of the caller: when
// need_f is false its final value is not produced (uv_advect only keeps the increments).
template <class T>
int do_adv2d(getm_ctx* ctx, T dt, T* f, const T* U, const T* V, const T* DUa, const T* DVa, const T* Do, int split,
             int scheme, int tag, T* A, T* Di, T* S, bool need_f) {
  const Dev& d = ctx->dev;
  cudaStream_t s = ctx->stream;
  const long long n2 = n2d(d);
  const size_t b2 = (size_t)n2 * sizeof(T);
  getm_adv_grid g;
  if (!grid_for_tag(ctx, tag, &g)) return fail(ctx, GETM_ERR_ARG, "do_advection: tag is invalid");
  GB_TRY(cudaMemsetAsync(A, 0, b2, s), "zero adv");
  if (scheme == NOADV) return GETM_OK;
  if (!is_split_scheme(scheme)) return fail(ctx, GETM_ERR_UNSUPPORTED, "do_advection: 2DH schemes not provided");
  const T one = T(1), half = T(0.5), zero = T(0);
  switch (split) {
    case GETM_NOSPLIT:
      GB_TRY(cudaMemcpyAsync(S, f, b2, cudaMemcpyDeviceToDevice, s), "copy f");
      GB_TIMED(GETM_TIM_BC2D, (run_sweep_h<T, 0>(d, s, 1, dt, one, scheme, zero, f, S, S, Do, Di, A, U, DUa,
                                                  g.mask_uflux, g.mask_uupdate)), "u");
      GB_TIMED(GETM_TIM_BC2D, (run_sweep_h<T, 1>(d, s, 1, dt, one, scheme, zero, f, S, S, Di, Di, A, V, DVa,
                                                  g.mask_vflux, g.mask_vupdate)), "v");
      if (need_f) {
        k_finalise2d<T><<<grid2(d), kBlk2, 0, s>>>(d, dt, f, Do, A, Di, g.mask_finalise);
        GB_TRY(cudaGetLastError(), "finalise2d");
      }
      break;
    case GETM_FULLSPLIT:
      GB_TIMED(GETM_TIM_BC2D, (run_sweep_h<T, 0>(d, s, 1, dt, one, scheme, zero, f, f, S, Do, Di, A, U, DUa,
                                                  g.mask_uflux, g.mask_uupdate)), "u");
      GB_TIMED(GETM_TIM_BC2D, (run_sweep_h<T, 1>(d, s, 1, dt, one, scheme, zero, S, S, f, Di, Di, A, V, DVa,
                                                  g.mask_vflux, g.mask_vupdate)), "v");
      break;
    case GETM_HALFSPLIT:
      GB_TIMED(GETM_TIM_BC2D, (run_sweep_h<T, 0>(d, s, 1, dt, half, scheme, zero, f, f, S, Do, Di, A, U, DUa,
                                                  g.mask_uflux, g.mask_uupdate)), "u");
      GB_TIMED(GETM_TIM_BC2D, (run_sweep_h<T, 1>(d, s, 1, dt, one, scheme, zero, S, S, f, Di, Di, A, V, DVa,
                                                  g.mask_vflux, g.mask_vupdate)), "v");
      GB_TIMED(GETM_TIM_BC2D, (run_sweep_h<T, 0>(d, s, 1, dt, half, scheme, zero, f, f, S, Di, Di, A, U, DUa,
                                                  g.mask_uflux, g.mask_uupdate)), "u");
      if (need_f) GB_TRY(cudaMemcpyAsync(f, S, b2, cudaMemcpyDeviceToDevice, s), "copy back");
      break;
    default:
      return fail(ctx, GETM_ERR_ARG, "do_advection: split is invalid");
  }
  return GETM_OK;
}

// uv_advect.F90:94-300 on (U, V, DU, DV) -> UEx, VEx (split schemes). The plain step works in
// FP64 (bit for bit with the reference); the mixed step advects the depth-averaged momentum in
// FP32 and widens the increments into the FP64 UEx / VEx.
template <class T>
int uv_advect_2d_t(getm_ctx* ctx, const getm_bc_state* st, const double* U, const double* V, const double* DU_,
                   const double* DV_) {
  const Dev& d = ctx->dev;
  cudaStream_t s = ctx->stream;
  const long long n2 = n2d(d);
  const int split = st->ipar[I_VEL2D_SPLIT], hor = st->ipar[I_VEL2D_HOR];
  double* Ex[2] = {st->f2[UEX], st->f2[VEX]};
  if (hor == NOADV) {
    GB_TRY(cudaMemsetAsync(Ex[0], 0, n2 * sizeof(double), s), "UEx=0");
    GB_TRY(cudaMemsetAsync(Ex[1], 0, n2 * sizeof(double), s), "VEx=0");
    return GETM_OK;
  }
  if (split == GETM_HALFSPLIT && is_split_scheme(hor)) {
    // all three sweeps of each component in one launch (adv2d_fused.cuh)
    for (int dir = 0; dir < 2; ++dir) {
      getm_adv_grid g;
      grid_for_tag(ctx, dir == 0 ? GETM_U_TAG : GETM_V_TAG, &g);
      GB_TIMED(GETM_TIM_BC2D, run_uvadv2d_fused<T>(d, s, dir, T(st->par[P_DTM]), hor, U, V, DU_, DV_, g.mask_uflux,
                                                   g.mask_vflux, g.mask_uupdate, g.mask_vupdate, Ex[dir]),
               "uv_advect");
    }
    return GETM_OK;
  }
  // 2D scratch (NB2 FP64-sized arrays) viewed as T
  T* w = (T*)ctx->bc_scr2;
  T *fadv = w, *Uadv = w + n2, *Vadv = w + 2 * n2, *DUadv = w + 3 * n2, *DVadv = w + 4 * n2, *Di = w + 5 * n2,
    *S = w + 6 * n2, *Do = w + 7 * n2;
  constexpr bool is64 = sizeof(T) == 8;
  for (int dir = 0; dir < 2; ++dir) {
    T* A = is64 ? (T*)Ex[dir] : w + 8 * n2;
    {
      TimerScope ts(ctx, GETM_TIM_BC2D);
      if (dir == 0)
        k_uvadv2d_prep<0, T><<<grid2(d), kBlk2, 0, s>>>(d, U, V, DU_, DV_, fadv, Uadv, Vadv, DUadv, DVadv,
                                                         is64 ? nullptr : Do);
      else
        k_uvadv2d_prep<1, T><<<grid2(d), kBlk2, 0, s>>>(d, U, V, DU_, DV_, fadv, Uadv, Vadv, DUadv, DVadv,
                                                         is64 ? nullptr : Do);
      GB_TRY(cudaGetLastError(), "uv_advect prep");
    }
    const T* Dsrc = is64 ? (const T*)(dir == 0 ? DU_ : DV_) : Do;
    int rc = do_adv2d<T>(ctx, T(st->par[P_DTM]), fadv, Uadv, Vadv, DUadv, DVadv, Dsrc, split, hor,
                         dir == 0 ? GETM_U_TAG : GETM_V_TAG, A, Di, S, false);
    if (rc) return rc;
    if (!is64) {
      TimerScope ts(ctx, GETM_TIM_BC2D);
      k_widen2d<<<grid2(d), kBlk2, 0, s>>>(d, (const float*)A, Ex[dir]);
      GB_TRY(cudaGetLastError(), "widen");
    }
  }
  return GETM_OK;
}

int uv_advect_2d(getm_ctx* ctx, const getm_bc_state* st, const double* U, const double* V, const double* DU_,
                 const double* DV_) {
  return st->prec3d == 8 ? uv_advect_2d_t<double>(ctx, st, U, V, DU_, DV_)
                         : uv_advect_2d_t<float>(ctx, st, U, V, DU_, DV_);
}

#define GB_K2(kernel, ...)                                         \
  do {                                                             \
    TimerScope _ts(ctx, GETM_TIM_BC2D);                            \
    kernel<<<grid2(d), kBlk2, 0, ctx->stream>>>(__VA_ARGS__);      \
    GB_TRY(cudaGetLastError(), #kernel);                           \
  } while (0)

// sealevel.F90:115-117: the NaN sweep of the elevations every |sealevel_check| micro steps, until
// a sweep finds one (have_warned). The sweeps count on the device without a host synchronisation;
// nan_report reads the counters at the end of the call.
int nan_sweep_due(getm_ctx* ctx, const getm_bc_state* st, int loop) {
  const int chk = st->ipar[I_SEALEVEL_CHECK];
  if (chk == 0 || st->ipar[I_NAN_WARNED] || loop % std::abs(chk) != 0) return GETM_OK;
  TimerScope ts(ctx, GETM_TIM_BC2D);
  ctx->nan_swept = true;
  GB_TRY(run_nan_sweep(ctx->dev, ctx->stream, st->f2[Z], ctx->cnt + 3), "sealevel_nan_check");
  return GETM_OK;
}

// End of a call that swept: a finding sets nan_warned and, for sealevel_check > 0, is the error
// the reference stops with (getm_error 'NaN values encountered in elevations').
int nan_report(getm_ctx* ctx, getm_bc_state* st) {
  if (!ctx->nan_swept) return GETM_OK;
  ctx->nan_swept = false;
  unsigned long long h[2] = {0, 0};
  GB_TRY(cudaMemcpyAsync(h, ctx->cnt + 3, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream), "read NaN sweep");
  GB_TRY(cudaMemsetAsync(ctx->cnt + 3, 0, 3 * sizeof(unsigned long long), ctx->stream), "reset NaN sweep");
  GB_TRY(cudaStreamSynchronize(ctx->stream), "NaN sweep");
  if (h[0] == 0) return GETM_OK;
  st->ipar[I_NAN_WARNED] = 1;
  const Dev& d = ctx->dev;
  const long long nx = d.imax - d.imin + 1, last = (long long)h[1] - 1;
  char msg[160];
  snprintf(msg, sizeof msg, "NaN values encountered in elevations: %llu values, the last at i = %lld, j = %lld",
           h[0], d.imin + last % nx, d.jmin + last / nx);
  ctx->err = msg;
  return st->ipar[I_SEALEVEL_CHECK] > 0 ? GETM_ERR_CHECK : GETM_OK;
}

// bottom_friction.F90:8-250: ru, rv (and ruu, rvv; zub, zvb for runtype 1) from the transports;
// FP64 arithmetic for the FP64 state, FP32 arithmetic in the mixed step (on the working copies when
// wp is given)
int bottom_friction_2d(getm_ctx* ctx, const getm_bc_state* st, int runtype, const Bc2W* wp) {
  const Dev& d = ctx->dev;
  const Bc2 s = to_bc2(st);
  const Bc2W w = wp ? *wp : Bc2W{};
  const dim3 gt((d.ni() + 31) / 32, (d.nj() + 7) / 8, 1);
  TimerScope ts(ctx, GETM_TIM_BC2D);
  if (wp) k_bottom_friction_f32t<true><<<gt, dim3(32, 8, 1), 0, ctx->stream>>>(d, s, w, runtype);
  else if (st->prec3d == 8) k_bottom_friction<double, false><<<grid2(d), kBlk2, 0, ctx->stream>>>(d, s, w, runtype);
  else k_bottom_friction_f32t<false><<<gt, dim3(32, 8, 1), 0, ctx->stream>>>(d, s, w, runtype);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GETM_OK : cuda_fail(ctx, (int)e, "bottom_friction");
}

// the two-point kernels (velocity update, sealevel + depth_update) apply: an even row pitch and an
// even number of columns (a pair never straddles the plane's edge), pair-aligned FP64 and FP32 arrays
bool pairs_ok(const Dev& d, const Bc2& s, const Bc2W& w) {
  if (!vector_sweeps_enabled() || d.sj % 2 != 0 || d.ni() % 2 != 0) return false;
  for (int q : {Z, ZO, CORU, CORV, UINT, VINT})
    if (reinterpret_cast<uintptr_t>(s.f2[q]) % 16 != 0) return false;
  for (int q : {U_, V_, D_, DU, DV, FU, FV, HH, HU, HV, FWF, AIRP, TAUSX, TAUSY, SLRU, SLRV, DRY_U, DRY_V, UEX, VEX,
                SLUX, SLVX, RU, RV})
    if (reinterpret_cast<uintptr_t>(w.w[q]) % 8 != 0) return false;
  for (int q = 0; q < 3; ++q)
    if (reinterpret_cast<uintptr_t>(w.m8[q]) % 2 != 0) return false;
  return true;
}

// umomentum (DIR 0, momentum.F90:69-223) / vmomentum (DIR 1, :232-386): the transport update, the
// mirror_bdy_2d copies of the open boundaries (:190, :353) and the Coriolis term for the other
// velocity (:193-216, :356-379). Mixed micro step (wp): the update on the working copies, with
// the term it needs formed in the same launch when `cor` (see integrate_2d).
template <int DIR>
// fused (the FP64 micro-step loop without open boundaries; always for the mixed step): the update
// forms the Coriolis term it needs itself when `cor`, and the term of the other velocity is left to
// the next update (or to the end of the loop) instead of a k_coriolis launch after each update.
int momentum_2d(getm_ctx* ctx, const getm_bc_state* st, const Bc2W* wp, bool cor, bool fused = false) {
  const Dev& d = ctx->dev;
  const Bc2 s = to_bc2(st);
  const Bc2W w = wp ? *wp : Bc2W{};
  cudaStream_t cs = ctx->stream;
  {
    TimerScope ts(ctx, GETM_TIM_BC2D);
    if (!wp && fused && cor) k_momentum<DIR, false, true><<<grid2(d), kBlk2, 0, cs>>>(d, s, w);
    else if (!wp) k_momentum<DIR, false><<<grid2(d), kBlk2, 0, cs>>>(d, s, w);
    else if (pairs_ok(d, s, w)) {
      const dim3 gp((d.ni() / 2 + 31) / 32, (d.nj() + 3) / 4, 1);
      if (cor) k_momentum_f32v<DIR, true><<<gp, kBlk2, 0, cs>>>(d, s, w);
      else k_momentum_f32v<DIR, false><<<gp, kBlk2, 0, cs>>>(d, s, w);
    } else if (cor) k_momentum_f32<DIR, true><<<grid2(d), kBlk2, 0, cs>>>(d, s, w);
    else k_momentum_f32<DIR, false><<<grid2(d), kBlk2, 0, cs>>>(d, s, w);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, (int)e, DIR == 0 ? "umomentum" : "vmomentum");
  }
  if (wp || fused) return GETM_OK;
  int r;
  if ((r = mirror_bdy<double>(ctx, st->f2[DIR == 0 ? U_ : V_], DIR, 1))) return r;
  TimerScope ts(ctx, GETM_TIM_BC2D);
  k_coriolis<DIR, false><<<grid2(d), kBlk2, 0, cs>>>(d, s, w);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GETM_OK : cuda_fail(ctx, (int)e, "coriolis");
}

// m2d.F90:412-490 integrate_2d (closed boundaries; no residual; Am <= 0, An_method = 0)
// zswap (the micro-step loop without open boundaries): sealevel and depth_update as one launch that
// writes the new elevations into st->f2[ZO]; the caller then swaps st->f2[Z] and st->f2[ZO]. With
// zswap, dryz = false leaves dry_z as it is (a micro step that neither a macro step nor the
// caller follows).
int integrate_2d(getm_ctx* ctx, getm_bc_state* st, int loop, const Bc2W* wp = nullptr, bool first = false,
                 bool zswap = false, bool dryz = true) {
  const Dev& d = ctx->dev;
  const Bc2 s = to_bc2(st);
  int* ip = st->ipar;
  // wp != nullptr: the mixed-precision micro step on the FP32 working copies (no open boundaries)
  const bool mix = wp != nullptr;
  const Bc2W w = mix ? *wp : Bc2W{};
  auto k2 = [&](auto kernel, auto... args) -> int {
    TimerScope ts(ctx, GETM_TIM_BC2D);
    kernel<<<grid2(d), kBlk2, 0, ctx->stream>>>(args...);
    return (int)cudaGetLastError();
  };
  int rc = GETM_OK;
  const bool bf_due = (loop - 1) % ip[I_MM] == 0;
  // the mixed micro step forms the bottom friction inside its momentum-advection kernels (they
  // stage the same velocities); the separate kernel otherwise (and with the fused micro-step
  // kernels switched off, for the comparison of the two forms)
  const bool bf_fused = mix && bf_due && ip[I_VEL2D_HOR] != NOADV && fused_micro_enabled();
  if (bf_due && !bf_fused && (rc = bottom_friction_2d(ctx, st, ip[I_RUNTYPE], wp))) return rc;
  if (mix) {
    const int hor = ip[I_VEL2D_HOR];
    if (hor == NOADV) {
      GB_TRY(cudaMemsetAsync(w.w[UEX], 0, n2d(d) * sizeof(float), ctx->stream), "UEx=0");
      GB_TRY(cudaMemsetAsync(w.w[VEX], 0, n2d(d) * sizeof(float), ctx->stream), "VEx=0");
    } else {
      // both components in one launch: UEx and VEx each read U, V, DU, DV only
      const uint8_t* masks[2][4];
      Bf2Args bf[2]{};
      for (int dir = 0; dir < 2; ++dir) {
        getm_adv_grid g;
        grid_for_tag(ctx, dir == 0 ? GETM_U_TAG : GETM_V_TAG, &g);
        masks[dir][0] = g.mask_uflux;
        masks[dir][1] = g.mask_vflux;
        masks[dir][2] = g.mask_uupdate;
        masks[dir][3] = g.mask_vupdate;
        if (bf_fused) {
          bf[dir].mask = w.m8[dir == 0 ? 1 : 2];
          bf[dir].au = w.m8[1];
          bf[dir].zb = w.w[dir == 0 ? ZUB : ZVB];
          bf[dir].zb0 = w.w[dir == 0 ? ZUB0 : ZVB0];
          bf[dir].r = w.w[dir == 0 ? RU : RV];
          bf[dir].rr = w.w[dir == 0 ? RUU : RVV];
          bf[dir].kappa = float(st->par[P_KAPPA]);
          bf[dir].avmmol = float(st->par[P_AVMMOL]);
          bf[dir].min_depth = float(st->par[P_MIN_DEPTH]);
          bf[dir].runtype = ip[I_RUNTYPE];
        }
      }
      GB_TIMED(GETM_TIM_BC2D,
               run_uvadv2d_both_f32(d, ctx->stream, float(st->par[P_DTM]), hor, w.w[U_], w.w[V_], w.w[DU], w.w[DV],
                                    masks[0], masks[1], w.w[UEX], w.w[VEX], bf_fused ? &bf[0] : nullptr,
                                    bf_fused ? &bf[1] : nullptr),
               "uv_advect");
    }
  } else {
    rc = uv_advect_2d(ctx, st, st->f2[U_], st->f2[V_], st->f2[DU], st->f2[DV]);
    if (rc) return rc;
  }
  // umomentum / vmomentum: transport update, mirror_bdy_2d (momentum.F90:190,353), Coriolis term.
  // The mixed micro step forms each Coriolis term inside the update that uses it (k_momentum
  // with COR): the stored term was formed from the other velocity as it is now, so recomputing
  // it gives the same value. The first update of a getm_time_loop call (first) reads the stored
  // term instead -- the state's fU/fV, which need not match the velocities (a start from rest of
  // the Coriolis terms) -- and getm_time_loop forms the term of the last update at its end.
  // the FP64 loop without open boundaries forms the Coriolis terms like the mixed step (zswap)
  auto umom = [&](bool cor) -> int { return momentum_2d<0>(ctx, st, wp, cor, zswap); };
  auto vmom = [&](bool cor) -> int { return momentum_2d<1>(ctx, st, wp, cor, zswap); };
  if (ip[I_UFIRST2D]) {
    if ((rc = umom(!first)) || (rc = vmom(true))) return rc;
    ip[I_UFIRST2D] = 0;
  } else {
    if ((rc = vmom(!first)) || (rc = umom(true))) return rc;
    ip[I_UFIRST2D] = 1;
  }
  // update_2d_bdy sets the boundary elevations after the Uint accumulation and before sealevel
  // (m2d.F90:467-476); the accumulation does not touch z, so it runs inside the sealevel kernel
  if (zswap) {
    if (ctx->has_bdy) return fail(ctx, GETM_ERR_STATE, "integrate_2d: fused sealevel with open boundaries");
    const int flags = (ip[I_RUNTYPE] > 1 ? 1 : 0) | (dryz ? 2 : 0);
    if (mix && pairs_ok(d, s, w)) {
      TimerScope ts(ctx, GETM_TIM_BC2D);
      k_sealevel_depth_p<<<dim3((d.ni() / 2 + 31) / 32, (d.nj() + 3) / 4, 1), kBlk2, 0, ctx->stream>>>(d, s, w, flags);
      rc = (int)cudaGetLastError();
    } else {
      rc = mix ? k2(k_sealevel_depth<true>, d, s, w, flags) : k2(k_sealevel_depth<false>, d, s, w, flags);
    }
    if (rc) return cuda_fail(ctx, rc, "sealevel + depth_update");
    std::swap(st->f2[Z], st->f2[ZO]);
    return nan_sweep_due(ctx, st, loop);
  }
  if (!mix && (rc = bdy_2d(ctx, s, loop))) return rc;
  rc = mix ? k2(k_accum_sealevel<true>, d, s, w, ip[I_RUNTYPE] > 1 ? 1 : 0)
           : k2(k_accum_sealevel<false>, d, s, w, ip[I_RUNTYPE] > 1 ? 1 : 0);
  if (rc) return cuda_fail(ctx, rc, "sealevel");
  if ((rc = nan_sweep_due(ctx, st, loop))) return rc;
  rc = mix ? k2(k_depth_update<true>, d, s, w) : k2(k_depth_update<false>, d, s, w);
  if (rc) return cuda_fail(ctx, rc, "depth_update");
  return GETM_OK;
}

// uint8 copies of the masks az, au, av (values 0..3) for the mixed-precision micro step
__global__ void k_mask8(long long n2, const int32_t* az, const int32_t* au, const int32_t* av, uint8_t* m8,
                        long long pitch) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n2; c += (long long)gridDim.x * blockDim.x) {
    m8[c] = (uint8_t)az[c];
    m8[pitch + c] = (uint8_t)au[c];
    m8[2 * pitch + c] = (uint8_t)av[c];
  }
}

// Copies between the FP64 state and the FP32 working copies of the mixed-precision micro step:
// to_w != 0 fills the copies of the fields in `mask` (bit q = field q) from the state, to_w == 0
// writes them back.
struct FieldList {
  int n;
  int q[NF2];
};
// The 2D fields are contiguous planes of n2 elements; each grid row (blockIdx.y) copies one field,
// four elements per thread step (16-byte float4 / two double2 accesses when vec), grid-stride.
__global__ void k_sync_w2(long long n2, Bc2 s, Bc2W w, FieldList fl, int to_w, int vec) {
  const int q = fl.q[blockIdx.y];
  double* a = s.f2[q];
  float* b = w.w[q];
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long done = 0;
  if (vec) {
    const long long n4 = n2 / 4;
    for (long long t = t0; t < n4; t += stride) {
      if (to_w) {
        const double2 x = reinterpret_cast<const double2*>(a)[2 * t], y = reinterpret_cast<const double2*>(a)[2 * t + 1];
        reinterpret_cast<float4*>(b)[t] = make_float4((float)x.x, (float)x.y, (float)y.x, (float)y.y);
      } else {
        const float4 v = reinterpret_cast<const float4*>(b)[t];
        reinterpret_cast<double2*>(a)[2 * t] = make_double2(v.x, v.y);
        reinterpret_cast<double2*>(a)[2 * t + 1] = make_double2(v.z, v.w);
      }
    }
    done = n4 * 4;
  }
  for (long long c = done + t0; c < n2; c += stride) {
    if (to_w) b[c] = (float)a[c];
    else a[c] = (double)b[c];
  }
}

template <class R3>
int bc3(getm_ctx* ctx, const getm_bc_state* st, int which, int slot, unsigned skip = 0, const R3* colh = nullptr) {
  const Bc3<R3> s = to_bc3<R3>(st);
  const long long n3 = n3d(ctx->dev);
  R3* base = (R3*)ctx->bc_scr3;
  R3* scr[NB3F];
  const int nb = sizeof(R3) == 4 ? NB3F : NB3;
  // skip: scratch slots the kernel does not write (bit q = slot q)
  for (int q = 0; q < NB3F; ++q) scr[q] = (q < nb && !((skip >> q) & 1u)) ? base + q * n3 : nullptr;
  GB_TIMED(slot, (run_bc3<R3>(which, ctx->dev, ctx->stream, s, scr, colh)), "macro-step kernel");
  return GETM_OK;
}

// do_internal_pressure (internal_pressure.F90:181-274) with the configured method (check_state
// admits 1 to 7): heights of the layer interfaces (1, 5) or of the pressure points (2, 3, 4, 7; 6
// over the whole haloed domain, with its column integrals), then the gradients idpdx, idpdy
template <class R3>
int internal_pressure(getm_ctx* ctx, const getm_bc_state* st) {
  const int ipm = st->ipar[I_IP_METHOD];
  const bool centres = ipm == 2 || ipm == 3 || ipm == 4 || ipm == 7;
  const int ipk = ipm == 1   ? BC3_IP
                  : ipm == 2 ? BC3_IP_LIN
                  : ipm == 3 ? BC3_IP_ZI
                  : ipm == 7 ? BC3_IP_SVK
                  : ipm == 4 ? BC3_IP_SW
                  : ipm == 5 ? BC3_IP_CF
                             : BC3_IP_SM;
  int rc;
  // the FP32 Blumberg-Mellor integral forms its interface heights itself (k_ip with ZS)
  const bool zz_inside = sizeof(R3) == 4 && ipm == 1;
  if (!zz_inside &&
      (rc = bc3<R3>(ctx, st, ipm == 6 ? BC3_SM_COLS : centres ? BC3_ZZ_LIN : BC3_ZZ, GETM_TIM_BC3D)))
    return rc;
  return bc3<R3>(ctx, st, ipk, GETM_TIM_IP);
}

// m3d.F90:422-636 integrate_3d for runtype 4 (closed boundaries, sigma coordinates, linear EOS,
// Blumberg-Mellor internal pressure, prescribed viscosity)
template <class R3>
int integrate_3d(getm_ctx* ctx, getm_bc_state* st, int n) {
  (void)n;
  const Dev& d = ctx->dev;
  cudaStream_t s = ctx->stream;
  const Bc2 s2 = to_bc2(st);
  int* ip = st->ipar;
  const long long n3 = n3d(d);
  R3** f3 = (R3**)st->f3;
  int rc;
  // start_macro
  GB_K2(k_start_macro_t, d, s2);
  GB_K2(k_start_macro_uv, d, s2, 1.0 / (double)(float)ip[I_M]);
  if (d.kmax > 1 && (rc = bc3<R3>(ctx, st, BC3_BF3D, GETM_TIM_BC3D))) return rc;
  if (ip[I_RUNTYPE] == 4 && (rc = internal_pressure<R3>(ctx, st))) return rc;
  // m3d.F90 sets huo = hun, hvo = hvn here for uu/vv_momentum_3d; sigma_coordinates below then
  // recomputes huo/hvo from the same elevations, to the same values. The momentum kernels read
  // hun/hvn as their old heights instead, so the two 3D copies are not made.
  // uu/vv_momentum_3d, each followed by its mirror_bdy_3d (uu_momentum_3d.F90:389, vv_momentum_3d.F90:400)
  auto uum = [&]() -> int {
    int r = bc3<R3>(ctx, st, BC3_UUMOM, GETM_TIM_MOM3D);
    return r ? r : mirror_bdy<R3>(ctx, f3[UU], 0, d.kmax + 1);
  };
  auto vvm = [&]() -> int {
    int r = bc3<R3>(ctx, st, BC3_VVMOM, GETM_TIM_MOM3D);
    return r ? r : mirror_bdy<R3>(ctx, f3[VV], 1, d.kmax + 1);
  };
  if (ip[I_UFIRST3D]) {
    if ((rc = uum()) || (rc = vvm())) return rc;
    ip[I_UFIRST3D] = 0;
  } else {
    if ((rc = vvm()) || (rc = uum())) return rc;
    ip[I_UFIRST3D] = 1;
  }
  if ((rc = bc3<R3>(ctx, st, BC3_SIGMA, GETM_TIM_BC3D))) return rc;
  // the heights sigma_coordinates just set, as 2D planes of column values: the advection and
  // diffusion launches below read them in place of the 3D height arrays (equidistant sigma: every
  // level of a column has the same height)
  R3* colh = (R3*)ctx->colh;
  const long long n2 = n2d(d);
  auto CH = [&](int q) { return colh + (long long)q * n2; };
  GB_TIMED(GETM_TIM_BC3D, run_col_heights<R3>(d, s, to_bc3<R3>(st), colh), "column heights");
  if (d.kmax > 1) {
    if ((rc = bc3<R3>(ctx, st, BC3_WW, GETM_TIM_BC3D))) return rc;
    // uv_advect_3d (uv_advect_3d.F90:62-460); only the advection terms uuEx/vvEx are kept, so the
    // last sweep writes no field
    const int split = ip[I_VEL3D_SPLIT], hor = ip[I_VEL3D_HOR], ver = ip[I_VEL3D_VER];
    if (hor != NOADV || ver != NOADV) {
      R3* w = (R3*)ctx->bc_scr3;
      // FP32: both grids' quantities in one pass (U grid in scratch 0-5, V grid in 7-12); FP64: the
      // U grid, its advection, then the V grid into the same six arrays. With the split sweeps the
      // face depths huadv, hvadv and the control-volume heights come from the column heights (h2d)
      // and the set-up does not form them.
      const bool cols = (split == GETM_HALFSPLIT || split == GETM_FULLSPLIT) && is_split_scheme(hor) &&
                        is_split_scheme(ver);
      const unsigned h2d = cols ? 7u : 0u;
      const unsigned skip = cols ? ((1u << 4) | (1u << 5) | (1u << 11) | (1u << 12)) : 0u;
      R3* wv = sizeof(R3) == 4 ? w + 7 * n3 : w;
      R3 *fadv = w, *ua = w + n3, *va = w + 2 * n3, *wa = w + 3 * n3, *hua = w + 4 * n3, *hva = w + 5 * n3;
      R3 *fadvv = wv, *uav = wv + n3, *vav = wv + 2 * n3, *wav = wv + 3 * n3, *huav = wv + 4 * n3, *hvav = wv + 5 * n3;
      if (cols) {
        hua = CH(COL_HUA_U);
        hva = CH(COL_HVA_U);
        huav = CH(COL_HUA_V);
        hvav = CH(COL_HVA_V);
      }
      const R3* hou = cols ? CH(COL_HUN) : f3[HUN];
      const R3* hov = cols ? CH(COL_HVN) : f3[HVN];
      if ((rc = bc3<R3>(ctx, st, sizeof(R3) == 4 ? BC3_UVADV_PREP_UV : BC3_UVADV_PREP_U, GETM_TIM_BC3D, skip,
                        colh)))
        return rc;
      if ((rc = do_adv3d<R3>(ctx, R3(st->par[P_DT]), fadv, ua, va, wa, hua, hva, hou, hou, split, hor, ver, R3(0),
                             GETM_U_TAG, nullptr, f3[UUEX], ip[I_ADV_VER_ITERS], false, nullptr, h2d)))
        return rc;
      if (sizeof(R3) == 8 && (rc = bc3<R3>(ctx, st, BC3_UVADV_PREP_V, GETM_TIM_BC3D, skip))) return rc;
      if ((rc = do_adv3d<R3>(ctx, R3(st->par[P_DT]), fadvv, uav, vav, wav, huav, hvav, hov, hov, split, hor, ver,
                             R3(0), GETM_V_TAG, nullptr, f3[VVEX], ip[I_ADV_VER_ITERS], false, nullptr, h2d)))
        return rc;
    }
    if ((rc = bc3<R3>(ctx, st, BC3_STRESSES, GETM_TIM_BC3D))) return rc;
    // m3d.F90:570-575: gotm() with PARABOLIC_VISCOSITY (CONSTANT_VISCOSITY leaves num, nuh)
    if (ip[I_VISCOSITY] == 1 && (rc = bc3<R3>(ctx, st, BC3_GOTM_PARABOLIC, GETM_TIM_BC3D))) return rc;
  }
  if (ip[I_RUNTYPE] == 4) {
    const R3 dt = R3(st->par[P_DT]);
    // do_temperature's short-wave radiation and surface heat flux (temperature.F90:452-525): the
    // sources of the temperature diffusion in the tracer scratch, and (paired advection) the
    // top-level salinity before it is advected, which the freezing-point test of the heat flux reads
    const bool radn = ip[I_RADIATION] && ip[I_CALC_TEMP];
    // compensated storage of the tracers (FP16 scaled carried errors; null: plain storage)
    __half* tlo = (__half*)st->f3[TLO];
    __half* slo = (__half*)st->f3[SLO];
    R3* tsrc = nullptr;
    R3* s_top = nullptr;
    if (radn) {
      if ((rc = ensure_scratch(ctx, (size_t)n3 * sizeof(R3)))) return rc;
      tsrc = (R3*)ctx->scr[2];
      s_top = (R3*)(ctx->bc_scr2 + 7 * n2d(d));
    }
    auto temp_sources = [&](const R3* stop) -> int {
      const Bc3<R3> s3 = to_bc3<R3>(st);
      R3* sc[2] = {tsrc, const_cast<R3*>(stop)};
      GB_TIMED(GETM_TIM_VDIFF, (run_bc3<R3>(BC3_SW_RADIATION, d, s, s3, sc)), "short-wave radiation");
      if (d.kmax > 1) GB_TIMED(GETM_TIM_VDIFF, (run_bc3<R3>(BC3_TEMP_SOURCE, d, s, s3, sc)), "temperature sources");
      return GETM_OK;
    };
    // do_temperature and do_salinity advect with the same velocities and heights; with the same
    // schemes the two advections run as one paired sweep sequence (each field's arithmetic is
    // unchanged), followed by the two diffusion solves.
    const bool pair = ip[I_CALC_TEMP] && ip[I_CALC_SALT] && ip[I_TEMP_SPLIT] == GETM_HALFSPLIT &&
                      ip[I_SALT_SPLIT] == GETM_HALFSPLIT && ip[I_TEMP_HOR] == ip[I_SALT_HOR] &&
                      ip[I_TEMP_VER] == ip[I_SALT_VER] && is_split_scheme(ip[I_TEMP_HOR]) &&
                      (ip[I_TEMP_VER] == NOADV || is_split_scheme(ip[I_TEMP_VER])) &&
                      st->par[P_TEMP_AH] == st->par[P_SALT_AH] && ip[I_ADV_VER_ITERS] <= 1 && ctx->adv_ready;
    if (pair) {
      if (radn)
        GB_TRY(cudaMemcpyAsync(s_top, f3[SS] + (long long)d.kmax * d.sk, n2d(d) * sizeof(R3), cudaMemcpyDeviceToDevice,
                               s),
               "top-level salinity");
      if ((rc = do_adv3d_pair<R3>(ctx, dt, f3[TT], f3[SS], f3[UU], f3[VV], f3[WW], CH(COL_HUN), CH(COL_HVN),
                                  CH(COL_HO), ip[I_TEMP_HOR], ip[I_TEMP_VER], R3(st->par[P_TEMP_AH]), tlo, slo,
                                  7u)))
        return rc;
      if (radn && (rc = temp_sources(s_top))) return rc;
      // the two diffusion solves in one launch (shared hn, nuh); the elimination coefficients of
      // both tracers, as interleaved (ru, qu) pairs, in the macro-step scratch (its first four
      // slots, free at this point of the step)
      R3* b3 = (R3*)ctx->bc_scr3;
      GB_TIMED(GETM_TIM_VDIFF,
               run_vdiff2<R3>(d, s, dt, R3(st->par[P_CNPAR]), CH(COL_HN), f3[NUH], st->az, f3[TT],
                              R3(st->par[P_AVMOLT]), (const R3*)tsrc, b3 + 2 * n3, nullptr, tlo, f3[SS],
                              R3(st->par[P_AVMOLS]), b3, nullptr, slo, true),
               "vdiff T, S");
    }
    if (!pair && ip[I_CALC_TEMP]) {
      if ((rc = do_adv3d<R3>(ctx, dt, f3[TT], f3[UU], f3[VV], f3[WW], f3[HUN], f3[HVN], f3[HO], f3[HN],
                             ip[I_TEMP_SPLIT], ip[I_TEMP_HOR], ip[I_TEMP_VER], R3(st->par[P_TEMP_AH]), GETM_H_TAG,
                             nullptr, nullptr, ip[I_ADV_VER_ITERS], true, tlo)))
        return rc;
      if (radn && (rc = temp_sources(nullptr))) return rc;
      GB_TIMED(GETM_TIM_VDIFF, run_vdiff<R3>(d, s, dt, R3(st->par[P_CNPAR]), R3(st->par[P_AVMOLT]), f3[TT], f3[HN],
                                             f3[NUH], st->az, (const R3*)tsrc, (R3*)ctx->scr[0], (R3*)ctx->scr[1],
                                             nullptr, nullptr, tlo),
               "vdiff T");
    }
    if (!pair && ip[I_CALC_SALT]) {
      if ((rc = do_adv3d<R3>(ctx, dt, f3[SS], f3[UU], f3[VV], f3[WW], f3[HUN], f3[HVN], f3[HO], f3[HN],
                             ip[I_SALT_SPLIT], ip[I_SALT_HOR], ip[I_SALT_VER], R3(st->par[P_SALT_AH]), GETM_H_TAG,
                             nullptr, nullptr, ip[I_ADV_VER_ITERS], true, slo)))
        return rc;
      GB_TIMED(GETM_TIM_VDIFF, run_vdiff<R3>(d, s, dt, R3(st->par[P_CNPAR]), R3(st->par[P_AVMOLS]), f3[SS], f3[HN],
                                             f3[NUH], st->az, (const R3*)nullptr, (R3*)ctx->scr[0], (R3*)ctx->scr[1],
                                             nullptr, nullptr, slo),
               "vdiff S");
    }
    // m3d.F90:595,602
    if (ip[I_CALC_TEMP] && (rc = mirror_bdy<R3>(ctx, f3[TT], 2, d.kmax + 1))) return rc;
    if (ip[I_CALC_SALT] && (rc = mirror_bdy<R3>(ctx, f3[SS], 2, d.kmax + 1))) return rc;
    const int eos = ip[I_EQSTATE_METHOD] == 2 ? BC3_EQSTATE_UNESCO : ip[I_EQSTATE_METHOD] == 3 ? BC3_EQSTATE_JACKETT
                                                                                              : BC3_EQSTATE;
    if ((rc = bc3<R3>(ctx, st, eos, GETM_TIM_BC3D))) return rc;
  }
  if (d.kmax > 1) {
    const long long n2 = n2d(d);
    double* Ui = ctx->bc_scr2 + 8 * n2;
    double* Vi = ctx->bc_scr2 + 9 * n2;
    GB_K2(k_sbf_uv, d, s2, Ui, Vi);
    GB_K2(k_sbf_r, d, s2, Ui, Vi, ctx->cnt + 2);
    if ((rc = uv_advect_2d(ctx, st, st->f2[UINT], st->f2[VINT], st->f2[DUN], st->f2[DVN]))) return rc;
  }
  if ((rc = bc3<R3>(ctx, st, BC3_SLOW_TERMS, GETM_TIM_BC3D))) return rc;
  GB_K2(k_stop_macro, d, s2);
  return GETM_OK;
}

}  // namespace

extern "C" {

int getm_set_open_boundaries(getm_ctx* ctx, const getm_bdy* b) {
  if (!ctx || !b) return GETM_ERR_ARG;
  if (!ctx->adv_ready) return fail(ctx, GETM_ERR_STATE, "getm_init_advection has not been called");
  const Dev& d = ctx->dev;
  const int cnt[4] = {b->nwb, b->nnb, b->neb, b->nsb};
  const int nseg = cnt[0] + cnt[1] + cnt[2] + cnt[3];
  if (cnt[0] < 0 || cnt[1] < 0 || cnt[2] < 0 || cnt[3] < 0 || (nseg > 0 && (!b->seg || !b->type2d)))
    return fail(ctx, GETM_ERR_ARG, "open boundaries: bad segment description");
  // masks on the host (they select the mirrored points)
  const long long n2 = n2d(d);
  std::vector<int32_t> az(n2), au(n2), av(n2);
  GB_TRY(cudaMemcpyAsync(az.data(), ctx->zmask, n2 * 4, cudaMemcpyDeviceToHost, ctx->stream), "masks");
  GB_TRY(cudaMemcpyAsync(au.data(), ctx->zmask + n2, n2 * 4, cudaMemcpyDeviceToHost, ctx->stream), "masks");
  GB_TRY(cudaMemcpyAsync(av.data(), ctx->zmask + 2 * n2, n2 * 4, cudaMemcpyDeviceToHost, ctx->stream), "masks");
  GB_TRY(cudaStreamSynchronize(ctx->stream), "masks");
  auto ix = [&](int i, int j) { return (long long)(i - (d.imin - HALO)) + (long long)(j - (d.jmin - HALO)) * d.sj; };
  auto inside = [&](int i, int j) { return i >= d.imin && i <= d.imax && j >= d.jmin && j <= d.jmax; };
  // boundary points in segment order (bdy_map), side by side
  std::vector<int4> pts;
  auto& B = ctx->bdy;
  int l = 0;
  for (int side = 0; side < 4; ++side) {
    B.side_first[side] = (int)pts.size();
    for (int n = 0; n < cnt[side]; ++n, ++l) {
      const int pos = b->seg[3 * l], f = b->seg[3 * l + 1], e = b->seg[3 * l + 2], t = b->type2d[l];
      if (t < 1 || t > 4) return fail(ctx, GETM_ERR_ARG, "open boundaries: illegal 2D boundary type");
      for (int q = f; q <= e; ++q) {
        const int i = (side == 0 || side == 2) ? pos : q, j = (side == 0 || side == 2) ? q : pos;
        if (!inside(i, j)) return fail(ctx, GETM_ERR_ARG, "open boundaries: point outside the domain");
        pts.push_back(make_int4(i, j, t, side));
      }
    }
  }
  B.side_first[4] = (int)pts.size();
  const int np = (int)pts.size();
  if (b->npoints != np) return fail(ctx, GETM_ERR_ARG, "open boundaries: npoints does not match the segments");
  // mirror copies (mirror_bdy_2d.F90 / mirror_bdy_3d.F90), per tag and side
  std::vector<long long> pairs;
  auto seg = [&](int side, int n, int q) {
    int first = 0;
    for (int s2 = 0; s2 < side; ++s2) first += cnt[s2];
    return b->seg[3 * (first + n) + q];
  };
  auto in_array = [&](int i, int j) {
    return i >= d.imin - HALO && i <= d.imax + HALO && j >= d.jmin - HALO && j <= d.jmax + HALO;
  };
  for (int tag = 0; tag < 3; ++tag)
    for (int side = 0; side < 4; ++side) {
      B.pair_first[tag][side] = (int)(pairs.size() / 2);
      for (int n = 0; n < cnt[side]; ++n) {
        const int pos = seg(side, n, 0), f = seg(side, n, 1) - HALO, e = seg(side, n, 2) + HALO;
        for (int q = f; q <= e; ++q) {
          const int i = (side == 0 || side == 2) ? pos : q, j = (side == 0 || side == 2) ? q : pos;
          if (!in_array(i, j)) continue;
          int di = 0, dj = 0, si = 0, sj = 0;
          bool use = false;
          if (tag == 0 && (side == 1 || side == 3)) {  // U points, au == 3
            use = au[ix(i, j)] == 3;
            di = i; dj = j; si = i; sj = side == 1 ? j - 1 : j + 1;
          } else if (tag == 1 && (side == 0 || side == 2)) {  // V points, av == 3
            use = av[ix(i, j)] == 3;
            di = i; dj = j; si = side == 0 ? i + 1 : i - 1; sj = j;
          } else if (tag == 2) {  // boundary value into the point outside
            use = az[ix(i, j)] > 1;
            si = i; sj = j;
            di = side == 0 ? i - 1 : side == 2 ? i + 1 : i;
            dj = side == 1 ? j + 1 : side == 3 ? j - 1 : j;
          }
          if (use && in_array(di, dj) && in_array(si, sj)) {
            pairs.push_back(ix(di, dj));
            pairs.push_back(ix(si, sj));
          }
        }
      }
      B.pair_first[tag][side + 1] = (int)(pairs.size() / 2);
    }
  // device copies
  auto up = [&](auto*& dst, const auto* src, size_t count) -> int {
    cudaFree(dst);
    dst = nullptr;
    if (!src || count == 0) return GETM_OK;
    using E = std::remove_pointer_t<std::remove_reference_t<decltype(dst)>>;
    if (cudaMalloc((void**)&dst, count * sizeof(E)) != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, GETM_ERR_NOMEM, "open boundaries: allocation failed");
    }
    return cudaMemcpy(dst, src, count * sizeof(E), cudaMemcpyHostToDevice) == cudaSuccess
               ? GETM_OK
               : fail(ctx, GETM_ERR_CUDA, "open boundaries: copy failed");
  };
  int rc;
  if ((rc = up(B.pts, pts.data(), pts.size())) || (rc = up(B.pairs, pairs.data(), pairs.size())) ||
      (rc = up(B.data, b->data, np)) || (rc = up(B.data_u, b->data_u, np)) || (rc = up(B.data_v, b->data_v, np)) ||
      (rc = up(B.amp, b->amp, np)) || (rc = up(B.phase, b->phase, np)))
    return rc;
  if (b->amp && !b->phase) return fail(ctx, GETM_ERR_ARG, "open boundaries: harmonic data needs phase");
  if (!b->amp && !b->data && np > 0) return fail(ctx, GETM_ERR_ARG, "open boundaries: no elevation data");
  B.npoints = np;
  B.harmonic = b->amp != nullptr;
  B.period = b->period;
  B.ramp = b->ramp;
  if (B.harmonic && !(b->period > 0)) return fail(ctx, GETM_ERR_ARG, "open boundaries: period must be > 0");
  ctx->has_bdy = nseg > 0;
  return GETM_OK;
}

int getm_set_bdy_data(getm_ctx* ctx, const double* data, const double* data_u, const double* data_v) {
  if (!ctx || !data) return GETM_ERR_ARG;
  if (!ctx->has_bdy) return fail(ctx, GETM_ERR_STATE, "getm_set_open_boundaries has not been called");
  auto& B = ctx->bdy;
  const size_t nb = (size_t)B.npoints * sizeof(double);
  auto put = [&](double*& dst, const double* src) -> int {
    if (!src) {
      cudaFree(dst);
      dst = nullptr;
      return GETM_OK;
    }
    if (!dst && cudaMalloc((void**)&dst, nb) != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, GETM_ERR_NOMEM, "boundary data: allocation failed");
    }
    return cudaMemcpyAsync(dst, src, nb, cudaMemcpyHostToDevice, ctx->stream) == cudaSuccess
               ? GETM_OK
               : fail(ctx, GETM_ERR_CUDA, "boundary data: copy failed");
  };
  int rc;
  if ((rc = put(B.data, data)) || (rc = put(B.data_u, data_u)) || (rc = put(B.data_v, data_v))) return rc;
  // the host arrays may be reused by the caller right after the call
  GB_TRY(cudaStreamSynchronize(ctx->stream), "boundary data");
  B.harmonic = false;
  return GETM_OK;
}

int getm_integrate_2d(getm_ctx* ctx, getm_bc_state* st, int loop) {
  int rc = check_state(ctx, st);
  if (rc) return rc;
  if ((rc = ensure_bc_scratch(ctx, (size_t)st->prec3d))) return rc;
  rc = integrate_2d(ctx, st, loop);
  const int rn = nan_report(ctx, st);
  return rc ? rc : rn;
}

// ---- the substeps of integrate_2d / integrate_3d one by one (FP64 2D arithmetic of the state) ----
#define GB_BC_ENTRY                                            \
  int rc = check_state(ctx, st);                               \
  if (rc) return rc;                                           \
  if ((rc = ensure_bc_scratch(ctx, (size_t)st->prec3d))) return rc

int getm_bottom_friction(getm_ctx* ctx, getm_bc_state* st, int runtype) {
  GB_BC_ENTRY;
  if (runtype < 1 || runtype > 4) return fail(ctx, GETM_ERR_ARG, "runtype must be 1..4");
  return bottom_friction_2d(ctx, st, runtype, nullptr);
}

int getm_uv_advect(getm_ctx* ctx, getm_bc_state* st) {
  GB_BC_ENTRY;
  return uv_advect_2d(ctx, st, st->f2[U_], st->f2[V_], st->f2[DU], st->f2[DV]);
}

int getm_umomentum(getm_ctx* ctx, getm_bc_state* st) {
  GB_BC_ENTRY;
  return momentum_2d<0>(ctx, st, nullptr, false);
}

int getm_vmomentum(getm_ctx* ctx, getm_bc_state* st) {
  GB_BC_ENTRY;
  return momentum_2d<1>(ctx, st, nullptr, false);
}

int getm_momentum(getm_ctx* ctx, getm_bc_state* st, int n) {
  (void)n;
  GB_BC_ENTRY;
  int* ip = st->ipar;
  if (ip[I_UFIRST2D]) {
    if ((rc = momentum_2d<0>(ctx, st, nullptr, false)) || (rc = momentum_2d<1>(ctx, st, nullptr, false))) return rc;
    ip[I_UFIRST2D] = 0;
  } else {
    if ((rc = momentum_2d<1>(ctx, st, nullptr, false)) || (rc = momentum_2d<0>(ctx, st, nullptr, false))) return rc;
    ip[I_UFIRST2D] = 1;
  }
  return GETM_OK;
}

int getm_update_2d_bdy(getm_ctx* ctx, getm_bc_state* st, int loop) {
  GB_BC_ENTRY;
  return bdy_2d(ctx, to_bc2(st), loop);
}

int getm_sealevel(getm_ctx* ctx, getm_bc_state* st, int loop) {
  GB_BC_ENTRY;
  const Dev& d = ctx->dev;
  {
    TimerScope ts(ctx, GETM_TIM_BC2D);
    k_accum_sealevel<false><<<grid2(d), kBlk2, 0, ctx->stream>>>(d, to_bc2(st), Bc2W{}, 0);
    GB_TRY(cudaGetLastError(), "sealevel");
  }
  if ((rc = nan_sweep_due(ctx, st, loop))) return rc;
  return nan_report(ctx, st);
}

int getm_depth_update(getm_ctx* ctx, getm_bc_state* st) {
  GB_BC_ENTRY;
  const Dev& d = ctx->dev;
  TimerScope ts(ctx, GETM_TIM_BC2D);
  k_depth_update<false><<<grid2(d), kBlk2, 0, ctx->stream>>>(d, to_bc2(st), Bc2W{});
  GB_TRY(cudaGetLastError(), "depth_update");
  return GETM_OK;
}

int getm_internal_pressure(getm_ctx* ctx, getm_bc_state* st) {
  GB_BC_ENTRY;
  return st->prec3d == 8 ? internal_pressure<double>(ctx, st) : internal_pressure<float>(ctx, st);
}

int getm_do_eqstate(getm_ctx* ctx, getm_bc_state* st) {
  GB_BC_ENTRY;
  const int m = st->ipar[I_EQSTATE_METHOD];
  const int which = m == 2 ? BC3_EQSTATE_UNESCO : m == 3 ? BC3_EQSTATE_JACKETT : BC3_EQSTATE;
  return st->prec3d == 8 ? bc3<double>(ctx, st, which, GETM_TIM_BC3D) : bc3<float>(ctx, st, which, GETM_TIM_BC3D);
}

int getm_gotm(getm_ctx* ctx, getm_bc_state* st) {
  GB_BC_ENTRY;
  if (st->ipar[I_VISCOSITY] != 1) return GETM_OK;  // CONSTANT_VISCOSITY: num and nuh stay
  return st->prec3d == 8 ? bc3<double>(ctx, st, BC3_GOTM_PARABOLIC, GETM_TIM_BC3D)
                         : bc3<float>(ctx, st, BC3_GOTM_PARABOLIC, GETM_TIM_BC3D);
}

int getm_sw_radiation(getm_ctx* ctx, getm_bc_state* st) {
  GB_BC_ENTRY;
  if (!st->f3[RAD] || !st->f2[SWR] || !st->f2[ATT_A] || !st->f2[ATT_G1] || !st->f2[ATT_G2])
    return fail(ctx, GETM_ERR_ARG, "sw_radiation: swr, A, g1, g2 and rad are needed");
  return st->prec3d == 8 ? bc3<double>(ctx, st, BC3_SW_RADIATION, GETM_TIM_VDIFF)
                         : bc3<float>(ctx, st, BC3_SW_RADIATION, GETM_TIM_VDIFF);
}

// write_restart_ncdf.F90:86-204: the restart file's fields in its order, by runtype
static void restart_lists(int runtype, int* f2, int* n2, int* f3, int* n3) {
  static const int base2[] = {Z, ZO, U_, SLUX, SLRU, V_, SLVX, SLRV};
  static const int more2[] = {SSEN, SSUN, SSVN, SSEO, SSUO, SSVO, UINTO, VINTO};
  static const int base3[] = {UU, VV, WW, UUEX, VVEX, TKE, EPS, NUM, NUH, HN};
  static const int ts3[] = {TT, SS};
  int a = 0, b = 0;
  for (int q : base2) f2[a++] = q;
  if (runtype >= 2) {
    for (int q : more2) f2[a++] = q;
    for (int q : base3) f3[b++] = q;
    if (runtype >= 3)
      for (int q : ts3) f3[b++] = q;
  }
  *n2 = a;
  *n3 = b;
}

int getm_restart_fields(int runtype, int32_t* f2_ids, int32_t* n2, int32_t* f3_ids, int32_t* n3) {
  if (runtype < 1 || runtype > 4 || !n2 || !n3) return GETM_ERR_ARG;
  int a[NF2], b[NF3], na, nb;
  restart_lists(runtype, a, &na, b, &nb);
  for (int q = 0; q < na; ++q)
    if (f2_ids) f2_ids[q] = a[q];
  for (int q = 0; q < nb; ++q)
    if (f3_ids) f3_ids[q] = b[q];
  *n2 = na;
  *n3 = nb;
  return GETM_OK;
}

// One restart field through the context's FP64 staging buffer (to_host: device -> host).
static int restart_field(getm_ctx* ctx, void* f, int elem, int nl, double* host, int to_host) {
  const Dev& d = ctx->dev;
  const long long n = (long long)(d.imax - d.imin + 1) * (d.jmax - d.jmin + 1) * nl;
  if (ctx->stage_bytes < (size_t)n * sizeof(double)) {
    cudaFree(ctx->stage);
    ctx->stage = nullptr;
    ctx->stage_bytes = 0;
    if (cudaMalloc(&ctx->stage, (size_t)n * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, GETM_ERR_NOMEM, "restart staging buffer: allocation failed");
    }
    ctx->stage_bytes = (size_t)n * sizeof(double);
  }
  const int blocks = (int)std::min<long long>((n + 255) / 256, 8 * 148);
  if (!to_host) GB_TRY(cudaMemcpyAsync(ctx->stage, host, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream),
                       "restart upload");
  if (f) {
    TimerScope ts(ctx, GETM_TIM_COPY);
    if (elem == 8) k_interior_copy<double><<<blocks, 256, 0, ctx->stream>>>(d, (double*)f, ctx->stage, nl, to_host);
    else k_interior_copy<float><<<blocks, 256, 0, ctx->stream>>>(d, (float*)f, ctx->stage, nl, to_host);
    GB_TRY(cudaGetLastError(), "restart field");
  } else if (to_host) {
    GB_TRY(cudaMemsetAsync(ctx->stage, 0, n * sizeof(double), ctx->stream), "restart field");
  }
  if (to_host) {
    GB_TRY(cudaMemcpyAsync(host, ctx->stage, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
           "restart download");
  }
  // the staging buffer is reused by the next field
  GB_TRY(cudaStreamSynchronize(ctx->stream), "restart field");
  return GETM_OK;
}

int getm_restart_write(getm_ctx* ctx, const getm_bc_state* st, int runtype, double* const* host2,
                       double* const* host3) {
  int rc = check_state(ctx, st);
  if (rc) return rc;
  if (runtype < 1 || runtype > 4 || !host2 || (runtype >= 2 && !host3)) return GETM_ERR_ARG;
  int a[NF2], b[NF3], na, nb;
  restart_lists(runtype, a, &na, b, &nb);
  for (int q = 0; q < na; ++q)
    if ((rc = restart_field(ctx, st->f2[a[q]], 8, 1, host2[q], 1))) return rc;
  for (int q = 0; q < nb; ++q)
    if ((rc = restart_field(ctx, st->f3[b[q]], st->prec3d, ctx->dev.kmax + 1, host3[q], 1))) return rc;
  return GETM_OK;
}

int getm_restart_read(getm_ctx* ctx, getm_bc_state* st, int runtype, const double* const* host2,
                      const double* const* host3) {
  int rc = check_state(ctx, st);
  if (rc) return rc;
  if (runtype < 1 || runtype > 4 || !host2 || (runtype >= 2 && !host3)) return GETM_ERR_ARG;
  if ((rc = ensure_bc_scratch(ctx, (size_t)st->prec3d))) return rc;
  int a[NF2], b[NF3], na, nb;
  restart_lists(runtype, a, &na, b, &nb);
  for (int q = 0; q < na; ++q)
    if ((rc = restart_field(ctx, st->f2[a[q]], 8, 1, const_cast<double*>(host2[q]), 0))) return rc;
  for (int q = 0; q < nb; ++q)
    if (st->f3[b[q]] &&
        (rc = restart_field(ctx, st->f3[b[q]], st->prec3d, ctx->dev.kmax + 1, const_cast<double*>(host3[q]), 0)))
      return rc;
  // postinit_2d / postinit_3d of a hotstart (initialise.F90:331-334)
  const Dev& d = ctx->dev;
  const Bc2 s2 = to_bc2(st);
  unsigned long long* flag = ctx->cnt + 6;
  GB_TRY(cudaMemsetAsync(flag, 0, sizeof(unsigned long long), ctx->stream), "hotstart");
  {
    TimerScope ts(ctx, GETM_TIM_BC2D);
    k_hot_check<<<grid2(d), kBlk2, 0, ctx->stream>>>(d, s2, flag);
    k_hot_reset2d<<<grid2(d), kBlk2, 0, ctx->stream>>>(d, s2, flag);
    k_depth_update<false><<<grid2(d), kBlk2, 0, ctx->stream>>>(d, s2, Bc2W{});
    GB_TRY(cudaGetLastError(), "postinit_2d");
  }
  if (runtype >= 2) {
    TimerScope ts(ctx, GETM_TIM_BC3D);
    void** f3 = st->f3;
    if (st->prec3d == 8)
      k_hot_reset3d<double><<<grid2(d), kBlk2, 0, ctx->stream>>>(d, s2, (double*)f3[UU], (double*)f3[VV],
                                                               (double*)f3[TKE], (double*)f3[NUM], (double*)f3[NUH],
                                                               (double*)f3[TT], (double*)f3[SS]);
    else
      k_hot_reset3d<float><<<grid2(d), kBlk2, 0, ctx->stream>>>(d, s2, (float*)f3[UU], (float*)f3[VV], (float*)f3[TKE],
                                                              (float*)f3[NUM], (float*)f3[NUH], (float*)f3[TT],
                                                              (float*)f3[SS]);
    GB_TRY(cudaGetLastError(), "postinit_3d");
    rc = st->prec3d == 8 ? bc3<double>(ctx, st, BC3_SIGMA, GETM_TIM_BC3D) : bc3<float>(ctx, st, BC3_SIGMA, GETM_TIM_BC3D);
    if (rc) return rc;
  }
  return GETM_OK;
}

int getm_sealevel_nan_check(getm_ctx* ctx, const double* z, int64_t* num_nan, int32_t* inan, int32_t* jnan) {
  if (!ctx || !z || !num_nan) return GETM_ERR_ARG;
  const Dev& d = ctx->dev;
  unsigned long long* c = ctx->cnt + 6;  // counters [6] findings, [7] last index + 1; latch unused
  GB_TRY(cudaMemsetAsync(c, 0, 2 * sizeof(unsigned long long), ctx->stream), "reset");
  GB_TRY(run_nan_sweep_once(d, ctx->stream, z, c), "sealevel_nan_check");
  unsigned long long h[2] = {0, 0};
  GB_TRY(cudaMemcpyAsync(h, c, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream), "read");
  GB_TRY(cudaStreamSynchronize(ctx->stream), "sync");
  *num_nan = (int64_t)h[0];
  const long long nx = d.imax - d.imin + 1, last = (long long)h[1] - 1;
  if (inan) *inan = h[0] ? (int32_t)(d.imin + last % nx) : 0;
  if (jnan) *jnan = h[0] ? (int32_t)(d.jmin + last / nx) : 0;
  return GETM_OK;
}

int getm_integrate_3d(getm_ctx* ctx, getm_bc_state* st, int n) {
  int rc = check_state(ctx, st);
  if (rc) return rc;
  if ((rc = ensure_bc_scratch(ctx, (size_t)st->prec3d))) return rc;
  return st->prec3d == 8 ? integrate_3d<double>(ctx, st, n) : integrate_3d<float>(ctx, st, n);
}

static int time_loop(getm_ctx* ctx, getm_bc_state* st, int n0, int count, bool zswap);

int getm_time_loop(getm_ctx* ctx, getm_bc_state* st_user, int n0, int count) {
  int rc = check_state(ctx, st_user);
  if (rc) return rc;
  if ((rc = ensure_bc_scratch(ctx, (size_t)st_user->prec3d))) return rc;
  // Without open boundaries the micro steps update the elevations by pointer ping-pong between z
  // and zo (k_sealevel_depth) on a copy of the state table; after an odd number of swaps the two
  // arrays' contents are exchanged at the end, so the caller's z and zo hold what the reference's
  // would. The integer settings the steps update (ufirst2d/3d, nan_warned) are copied back.
  const bool zswap = !ctx->has_bdy && fused_micro_enabled();
  getm_bc_state loc = *st_user;
  rc = time_loop(ctx, zswap ? &loc : st_user, n0, count, zswap);
  if (zswap) {
    std::copy(loc.ipar, loc.ipar + NPI, st_user->ipar);
    if (loc.f2[Z] != st_user->f2[Z]) {
      k_swap2<<<592, 256, 0, ctx->stream>>>(n2d(ctx->dev), st_user->f2[Z], st_user->f2[ZO]);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess && rc == GETM_OK) rc = cuda_fail(ctx, (int)e, "elevation ping-pong");
    }
  }
  return rc;
}

static int time_loop(getm_ctx* ctx, getm_bc_state* st, int n0, int count, bool zswap) {
  int rc;
  // The mixed-precision step (FP32 3D fields) runs its micro steps on FP32 working copies of the
  // barotropic fields (is_work2) when the fused 2D momentum advection applies and there are no
  // open boundaries; the elevation and Uint/Vint stay FP64 throughout.
  const int* ip = st->ipar;
  const bool mix = st->prec3d == 4 && !ctx->has_bdy && fp32_micro_steps_enabled() &&
                   (ip[I_VEL2D_HOR] == NOADV ||
                    (ip[I_VEL2D_SPLIT] == GETM_HALFSPLIT && is_split_scheme(ip[I_VEL2D_HOR])));
  Bc2W w{};
  unsigned long long all = 0, written = 0, from3d = 0;
  if (mix) {
    const Dev& d = ctx->dev;
    const long long n2 = n2d(d);
    int nw = 0;
    for (int q = 0; q < NF2; ++q) nw += is_work2(q) ? 1 : 0;
    // nw FP32 planes, then the uint8 copies of az, au, av (3 planes, 16-byte aligned)
    const long long m8off = (long long)nw * n2 * (long long)sizeof(float);
    const long long m8pitch = (n2 + 15) / 16 * 16;
    if (!ctx->w2) {
      if (cudaMalloc(&ctx->w2, (size_t)(m8off + 3 * m8pitch)) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, GETM_ERR_NOMEM, "mixed-precision 2D working copies: allocation failed");
      }
    }
    int slot = 0;
    for (int q = 0; q < NF2; ++q) {
      w.w[q] = is_work2(q) ? ctx->w2 + (long long)(slot++) * n2 : nullptr;
      if (is_work2(q)) all |= 1ull << q;
    }
    uint8_t* m8 = reinterpret_cast<uint8_t*>(ctx->w2) + m8off;
    for (int q = 0; q < 3; ++q) w.m8[q] = m8 + q * m8pitch;
    k_mask8<<<592, 256, 0, ctx->stream>>>(n2, st->az, st->au, st->av, m8, m8pitch);
    GB_TRY(cudaGetLastError(), "uint8 masks");
    // written by the micro steps; written by the macro step and read by the micro steps
    for (int q : {U_, V_, D_, DU, DV, DRY_U, DRY_V, FU, FV, RU, RV, RUU, RVV, UEX, VEX}) written |= 1ull << q;
    if (st->ipar[I_RUNTYPE] == 1) written |= (1ull << ZUB) | (1ull << ZVB);  // renewed by the bottom friction
    for (int q : {SLUX, SLVX, SLRU, SLRV, RU, RV}) from3d |= 1ull << q;
  }
  auto sync = [&](unsigned long long mask, int to_w) -> int {
    TimerScope ts(ctx, GETM_TIM_COPY);
    FieldList fl{};
    for (int q = 0; q < NF2; ++q)
      if ((mask >> q) & 1ull) fl.q[fl.n++] = q;
    if (fl.n == 0) return GETM_OK;
    const long long n2 = n2d(ctx->dev);
    bool vec = n2 % 4 == 0;
    for (int m = 0; m < fl.n; ++m)
      vec = vec && reinterpret_cast<uintptr_t>(st->f2[fl.q[m]]) % 16 == 0 &&
            reinterpret_cast<uintptr_t>(w.w[fl.q[m]]) % 16 == 0;
    k_sync_w2<<<dim3(592, fl.n, 1), 256, 0, ctx->stream>>>(n2, to_bc2(st), w, fl, to_w, vec ? 1 : 0);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GETM_OK : cuda_fail(ctx, (int)e, "mixed-precision 2D copies");
  };
  if (mix && (rc = sync(all & ~((1ull << UEX) | (1ull << VEX)), 1))) return rc;
  bool dirty = false;  // working copies newer than the state
  for (int n = n0; n < n0 + count; ++n) {
    // do_3d (integration.F90:106): a macro step after every M-th micro step, for runtype >= 2
    const bool do_3d = st->ipar[I_RUNTYPE] >= 2 && n % st->ipar[I_M] == 0;
    const bool dryz = do_3d || n == n0 + count - 1;
    if ((rc = integrate_2d(ctx, st, n, mix ? &w : nullptr, n == n0, zswap, dryz))) return rc;
    dirty = mix;
    if (do_3d) {
      if (mix && (rc = sync(written, 0))) return rc;
      dirty = false;
      rc = st->prec3d == 8 ? integrate_3d<double>(ctx, st, n) : integrate_3d<float>(ctx, st, n);
      if (rc) return rc;
      // the macro step's 2D results into the working copies, unless the call ends here (the next
      // call fills every working copy from the state anyway)
      if (mix && n + 1 < n0 + count && (rc = sync(from3d, 1))) return rc;
    }
  }
  if ((mix || zswap) && count > 0) {
    // the Coriolis term of the last velocity update (fV after a V update, fU after a U update):
    // ufirst2d was toggled by the last micro step, so 0 means its order was u, v
    TimerScope ts(ctx, GETM_TIM_BC2D);
    const Bc2 s2 = to_bc2(st);
    const bool v_last = st->ipar[I_UFIRST2D] == 0;
    if (mix && v_last) k_coriolis<1, true><<<grid2(ctx->dev), kBlk2, 0, ctx->stream>>>(ctx->dev, s2, w);
    else if (mix) k_coriolis<0, true><<<grid2(ctx->dev), kBlk2, 0, ctx->stream>>>(ctx->dev, s2, w);
    else if (v_last) k_coriolis<1, false><<<grid2(ctx->dev), kBlk2, 0, ctx->stream>>>(ctx->dev, s2, w);
    else k_coriolis<0, false><<<grid2(ctx->dev), kBlk2, 0, ctx->stream>>>(ctx->dev, s2, w);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, (int)e, "coriolis");
  }
  if (dirty && (rc = sync(written, 0))) return rc;
  if (mix && !dirty && count > 0 && (rc = sync((1ull << FU) | (1ull << FV), 0))) return rc;
  return nan_report(ctx, st);
}

}  // extern "C"
