// common.cuh -- shared device-side definitions of the B200 hot-path library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/getm_b200.h"

namespace gb {

constexpr int HALO = 2;

// Index space of one context as the kernels see it (value copy of getm_domain).
struct Dev {
  int imin, imax, jmin, jmax, kmax;
  long long sj, sk;
  double dx, dy, ard1;
  // haloed extents
  __host__ __device__ int ni() const { return imax - imin + 1 + 2 * HALO; }
  __host__ __device__ int nj() const { return jmax - jmin + 1 + 2 * HALO; }
  // offset of (i,j) relative to the origin (imin-2, jmin-2)
  __host__ __device__ long long ix(int i, int j) const {
    return (long long)(i - (imin - HALO)) + (long long)(j - (jmin - HALO)) * sj;
  }
};

inline Dev to_dev(const getm_domain& d) {
  Dev v;
  v.imin = d.imin; v.imax = d.imax; v.jmin = d.jmin; v.jmax = d.jmax; v.kmax = d.kmax;
  v.sj = d.sj; v.sk = d.sk; v.dx = d.dx; v.dy = d.dy; v.ard1 = d.ard1;
  return v;
}

// Scheme ids (advection.F90:60-62)
enum : int { NOADV = 0, UPSTREAM = 1, UPSTREAM_2DH = 2, P2 = 3, SUPERBEE = 4, MUSCL = 5, P2_PDM = 6 };

__host__ __device__ inline bool is_split_scheme(int s) {
  return s == UPSTREAM || s == P2 || s == SUPERBEE || s == MUSCL || s == P2_PDM;
}

// Reference-exact min/max (Fortran MIN/MAX on ordered operands).
template <class R>
__device__ __forceinline__ R rmin(R a, R b) { return (b < a) ? b : a; }
template <class R>
__device__ __forceinline__ R rmax(R a, R b) { return (b > a) ? b : a; }

// advection.F90:854-879 adv_interfacial_reconstruction_p2
template <class R>
__device__ __forceinline__ R recon_p2(R cfl, R fu, R deltafu, R deltaf) {
  const R one6th = R(1) / R(6);
  R x = one6th * (R(1) - R(2) * cfl);
  return fu + R(0.5) * (R(1) - cfl) * ((R(0.5) + x) * deltaf + (R(0.5) - x) * deltafu);
}

// advection.F90:785-845 adv_interfacial_reconstruction. Same expression order as the
// reference so that an FP64 build without contraction reproduces it bit for bit.
template <class R>
__device__ __forceinline__ R recon(int scheme, R cfl, R fuu, R fu, R fd) {
  const R one6th = R(1) / R(6);
  R deltaf = fd - fu;
  R deltafu = fu - fuu;
  if (deltaf * deltafu > R(0)) {
    R ratio = deltafu / deltaf;
    R limiter;
    if (scheme == SUPERBEE) {
      limiter = rmax(rmin(R(2) * ratio, R(1)), rmin(ratio, R(2)));
    } else if (scheme == P2_PDM) {
      R x = one6th * (R(1) - R(2) * cfl);
      limiter = (R(0.5) + x) + (R(0.5) - x) * ratio;
      limiter = rmin(rmin(R(2) * ratio / (cfl + R(1.e-10)), limiter), R(2) / (R(1) - cfl));
    } else if (scheme == MUSCL) {
      limiter = rmin(rmin(R(2) * ratio, R(0.5) * (R(1) + ratio)), R(2));
    } else if (scheme == P2) {
      return recon_p2(cfl, fu, deltafu, deltaf);
    } else {
      return fu;
    }
    return fu + R(0.5) * limiter * (R(1) - cfl) * deltaf;
  }
  if (scheme == P2) return recon_p2(cfl, fu, deltafu, deltaf);
  return fu;
}

// FP32 log-law bottom drag of one velocity point (bottom_friction.F90:86-103 / :121-138), shared by
// every FP32 form of the bottom friction so that they give the same bits: from the roughness zb,
// the point's depth HH and the velocity components, the drag coefficient rr and r = rr*|u|; with
// runtype 1 the roughness is first renewed from the friction velocity (zn, which the caller
// stores). Every operation is explicitly rounded (no dependence on multiply-add contraction); the
// divisions outside the logarithm's argument are the approximate ones (2 ulp).
struct BfLaw {
  float zn, rr, r;
};
__device__ __forceinline__ BfLaw bf_law_f32(float zb, float zb0, float HH, float uloc, float vloc, float kappa,
                                            float avmmol, int runtype) {
  const float h = 0.5f;
  const float sp = __fadd_rn(__fmul_rn(uloc, uloc), __fmul_rn(vloc, vloc));
  float x = __fdividef(kappa, logf(__fdiv_rn(__fadd_rn(zb, __fmul_rn(h, HH)), zb)));
  float rr = __fmul_rn(x, x);
  BfLaw o;
  o.zn = zb;
  if (runtype == 1) {
    const float fricvel = __fsqrt_rn(__fmul_rn(rr, sp));
    const float zn = fminf(HH, __fadd_rn(zb0, __fdividef(__fmul_rn(0.1f, avmmol), fmaxf(avmmol, fricvel))));
    o.zn = zn;
    x = __fdividef(kappa, logf(__fdiv_rn(__fadd_rn(zn, __fmul_rn(h, HH)), zn)));
    rr = __fmul_rn(x, x);
  }
  o.rr = rr;
  o.r = __fmul_rn(rr, __fsqrt_rn(sp));
  return o;
}

}  // namespace gb
