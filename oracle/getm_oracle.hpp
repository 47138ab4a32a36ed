// getm_oracle.hpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of GETM 2.5's per-timestep 3D hot path (Fortran, getm-model/code), used as
// the parity oracle for the CUDA kernels in code_b200/csrc. Only tests/, the smoke check in
// __graft_entry__.py and bench.py's CPU-baseline leg load it; the product library never links it.
//
// Conventions (identical to the reference's I3DFIELD/E2DFIELD layout, cppdefs.h:146-159):
//   * arrays are Fortran column-major, i fastest, then j, then k;
//   * index origin is (imin-HALO, jmin-HALO, 0) with HALO = 2;
//   * element (i,j,k) sits at  (i-(imin-2)) + (j-(jmin-2))*sj + k*sk.
// Every routine keeps the reference's loop bounds, loop order and expression order (left-to-right
// evaluation, no fused multiply-add: build with -ffp-contract=off), so that a GPU kernel written
// without contraction reproduces it bit for bit in FP64.
//
// Parity pin: the reference ships no golden vectors or known-answer tests and cannot be compiled
// here (no Fortran compiler). The restatement is pinned by tests/golden/, whose fixtures are made
// by tests/golden/fortran_subset.py executing the reference's own Fortran source of these
// routines; see the header of that script for what it covers.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace gor {

constexpr int HALO = 2;

// |x| and ceil(x) found by argument-dependent lookup, so that the templates also accept the
// dual-number type of getm_tangent.hpp; for float/double they are std::fabs / std::ceil.
template <class R>
inline R absval(R x) {
  using std::fabs;
  return fabs(x);
}
template <class R>
inline int ceil_int(R x) {
  using std::ceil;
  return (int)ceil(x);
}

// advection.F90:55-62, advection_3d.F90:42
enum { NOSPLIT = 0, FULLSPLIT = 1, HALFSPLIT = 2, HVSPLIT = 3 };
enum { NOADV = 0, UPSTREAM = 1, UPSTREAM_2DH = 2, P2 = 3, SUPERBEE = 4, MUSCL = 5, P2_PDM = 6 };
// halo_zones.F90:25-27, advection_3d.F90:42
enum { H_TAG = 10, D_TAG = 20, U_TAG = 31, V_TAG = 32, W_TAG = 33 };

struct Dom {
  int imin, imax, jmin, jmax, kmax;
  long sj, sk;          // element strides of j and k
  double dx, dy, ard1;  // Cartesian metrics (DXU=DYU=...=dx/dy, ARCD1=ard1, cppdefs.h:34-62)
  long ix(int i, int j) const { return (long)(i - (imin - HALO)) + (long)(j - (jmin - HALO)) * sj; }
  long ix3(int i, int j, int k) const { return ix(i, j) + (long)k * sk; }
  long n2d() const { return sj * (long)(jmax - jmin + 1 + 2 * HALO); }
  long n3d() const { return sk * (long)(kmax + 1); }
};

// One t_adv_grid (advection.F90:43-51): logical masks as bytes, az as int32.
struct AdvGrid {
  const uint8_t *uflux, *vflux, *uupdate, *vupdate, *finalise;
  const int32_t *az;
};

// ---------------------------------------------------------------------------------------------
// advection.F90:785-845 adv_interfacial_reconstruction, :854-879 _p2
template <class R>
inline R recon_p2(R cfl, R fu, R deltafu, R deltaf) {
  const R one6th = R(1) / R(6);
  R x = one6th * (R(1) - R(2) * cfl);
  return fu + R(0.5) * (R(1) - cfl) * ((R(0.5) + x) * deltaf + (R(0.5) - x) * deltafu);
}

template <class R>
inline R fmin2(R a, R b) { return (b < a) ? b : a; }
template <class R>
inline R fmax2(R a, R b) { return (b > a) ? b : a; }

template <class R>
inline R adv_interfacial_reconstruction(int scheme, R cfl, R fuu, R fu, R fd) {
  const R one6th = R(1) / R(6);
  R deltaf = fd - fu;
  R deltafu = fu - fuu;
  if (deltaf * deltafu > R(0)) {
    R ratio = deltafu / deltaf;
    R limiter;
    switch (scheme) {
      case P2_PDM: {
        R x = one6th * (R(1) - R(2) * cfl);
        limiter = (R(0.5) + x) + (R(0.5) - x) * ratio;
        limiter = fmin2(fmin2(R(2) * ratio / (cfl + R(1.e-10)), limiter), R(2) / (R(1) - cfl));
        break;
      }
      case SUPERBEE:
        limiter = fmax2(fmin2(R(2) * ratio, R(1)), fmin2(ratio, R(2)));
        break;
      case MUSCL:
        limiter = fmin2(fmin2(R(2) * ratio, R(0.5) * (R(1) + ratio)), R(2));
        break;
      case P2:
        return recon_p2(cfl, fu, deltafu, deltaf);
      case UPSTREAM:
        return fu;
      default:
        // The Fortran select has no default: limiter would be undefined. Not reachable from the
        // split drivers, which only pass the five schemes above.
        return fu;
    }
    return fu + R(0.5) * limiter * (R(1) - cfl) * deltaf;
  }
  if (scheme == P2) return recon_p2(cfl, fu, deltafu, deltaf);
  return fu;
}

// ---------------------------------------------------------------------------------------------
// adv_split_u.F90:205-285. 2D fields (one k-level); f may alias fi.
template <class R>
void adv_split_u(const Dom& d, R dt, const R* f, R* fi, R* Di, R* adv, const R* U, const R* DU,
                 R splitfac, int scheme, R AH, const uint8_t* mask_flux, const uint8_t* mask_update) {
  const int isub = (scheme == UPSTREAM) ? 0 : 1;
  const bool use_AH = AH > R(0);
  const R dti = splitfac * dt;
  const R DX = R(d.dx), DY = R(d.dy), ARD1 = R(d.ard1);
  std::vector<R> uflux(d.n2d(), R(0));
#pragma omp parallel for schedule(static)
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j) {
    bool use_limiter = false;
    for (int i = d.imin - HALO + isub; i <= d.imax + HALO - 1 - isub; ++i) {
      long p = d.ix(i, j);
      if (mask_flux[p]) {
        R fu, fuu = R(0), fd = R(0), cfl = R(0);
        if (U[p] > R(0)) {
          fu = f[p];
          if (scheme != UPSTREAM) use_limiter = mask_flux[d.ix(i - 1, j)] != 0;
          if (use_limiter) {
            cfl = U[p] / DU[p] * dti / DX;
            fuu = f[d.ix(i - 1, j)];
            fd = f[d.ix(i + 1, j)];
          }
        } else {
          fu = f[d.ix(i + 1, j)];
          if (scheme != UPSTREAM) use_limiter = mask_flux[d.ix(i + 1, j)] != 0;
          if (use_limiter) {
            cfl = -U[p] / DU[p] * dti / DX;
            fuu = f[d.ix(i + 2, j)];
            fd = f[p];
          }
        }
        if (use_limiter) fu = adv_interfacial_reconstruction<R>(scheme, cfl, fuu, fu, fd);
        uflux[p] = U[p] * fu;
        if (use_AH) uflux[p] = uflux[p] - AH * DU[p] * (f[d.ix(i + 1, j)] - f[p]) / DX;
      } else {
        uflux[p] = R(0);
      }
    }
  }
#pragma omp parallel for schedule(static)
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j) {
    for (int i = d.imin - HALO + 1 + isub; i <= d.imax + HALO - 1 - isub; ++i) {
      long p = d.ix(i, j);
      if (mask_update[p]) {
        long pm = d.ix(i - 1, j);
        R Dio = Di[p];
        Di[p] = Dio - dti * (U[p] * DY - U[pm] * DY) * ARD1;
        R advn = splitfac * (uflux[p] * DY - uflux[pm] * DY) * ARD1;
        fi[p] = (Dio * fi[p] - dt * advn) / Di[p];
        adv[p] = adv[p] + advn;
      }
    }
  }
}

// adv_split_v.F90:63-135. mask_flux is indexed like the other fields (its dummy spans
// jmin-HALO:jmax+HALO-1, advection.F90:127; the last row is never read).
template <class R>
void adv_split_v(const Dom& d, R dt, const R* f, R* fi, R* Di, R* adv, const R* V, const R* DV,
                 R splitfac, int scheme, R AH, const uint8_t* mask_flux, const uint8_t* mask_update) {
  const int jsub = (scheme == UPSTREAM) ? 0 : 1;
  const bool use_AH = AH > R(0);
  const R dti = splitfac * dt;
  const R DX = R(d.dx), DY = R(d.dy), ARD1 = R(d.ard1);
  std::vector<R> vflux(d.n2d(), R(0));
#pragma omp parallel for schedule(static)
  for (int j = d.jmin - HALO + jsub; j <= d.jmax + HALO - 1 - jsub; ++j) {
    bool use_limiter = false;
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      long p = d.ix(i, j);
      if (mask_flux[p]) {
        R fu, fuu = R(0), fd = R(0), cfl = R(0);
        if (V[p] > R(0)) {
          fu = f[p];
          if (scheme != UPSTREAM) use_limiter = mask_flux[d.ix(i, j - 1)] != 0;
          if (use_limiter) {
            cfl = V[p] / DV[p] * dti / DY;
            fuu = f[d.ix(i, j - 1)];
            fd = f[d.ix(i, j + 1)];
          }
        } else {
          fu = f[d.ix(i, j + 1)];
          if (scheme != UPSTREAM) use_limiter = mask_flux[d.ix(i, j + 1)] != 0;
          if (use_limiter) {
            cfl = -V[p] / DV[p] * dti / DY;
            fuu = f[d.ix(i, j + 2)];
            fd = f[p];
          }
        }
        if (use_limiter) fu = adv_interfacial_reconstruction<R>(scheme, cfl, fuu, fu, fd);
        vflux[p] = V[p] * fu;
        if (use_AH) vflux[p] = vflux[p] - AH * DV[p] * (f[d.ix(i, j + 1)] - f[p]) / DY;
      } else {
        vflux[p] = R(0);
      }
    }
  }
#pragma omp parallel for schedule(static)
  for (int j = d.jmin - HALO + 1 + jsub; j <= d.jmax + HALO - 1 - jsub; ++j) {
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      long p = d.ix(i, j);
      if (mask_update[p]) {
        long pm = d.ix(i, j - 1);
        R Dio = Di[p];
        Di[p] = Dio - dti * (V[p] * DX - V[pm] * DX) * ARD1;
        R advn = splitfac * (vflux[p] * DX - vflux[pm] * DX) * ARD1;
        fi[p] = (Dio * fi[p] - dt * advn) / Di[p];
        adv[p] = adv[p] + advn;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------
// adv_split_w.F90:85-304 (the non-_POINTER_REMAP_ build; identical results). 3D fields; f may
// alias fi (the column of f is copied before any update, :184). Returns the number of columns
// whose iteration estimate exceeded itersmax (the reference prints a warning, :224-228).
template <class R>
long adv_split_w(const Dom& d, R dt, const R* f, R* fi, R* hi, R* adv, const R* ww, R splitfac,
                 int scheme, int tag, const int32_t* az, int itersmax) {
  if (scheme == NOADV) return 0;
  const int kmax = d.kmax;
  const int kshift = (tag == W_TAG) ? 1 : 0;
  const R dti = splitfac * dt;
  const bool iterate = itersmax > 1;
  long too_many = 0;
#pragma omp parallel for schedule(static) reduction(+ : too_many)
  for (int j = d.jmin - HALO; j <= d.jmax + HALO - 1; ++j) {
    bool use_limiter = false;
    std::vector<R> wflux(kmax + 1), fo(kmax + 1), fiaux(kmax + 1), hiaux(kmax + 1),
        advaux(kmax + 1), cfl0(kmax + 1), cflsv(kmax + 1);
    wflux[0] = R(0);
    wflux[kmax] = R(0);
    for (int i = d.imin - HALO; i <= d.imax + HALO - 1; ++i) {
      long c = d.ix(i, j);
      if (az[c] != 1) continue;
      if (scheme != UPSTREAM || iterate)
        for (int k = 1 - kshift; k <= kmax - 1; ++k)
          cfl0[k] = absval(ww[c + k * d.sk]) * dti /
                    (R(0.5) * (hi[c + k * d.sk] + hi[c + (k + 1) * d.sk]));
      R* cfls = iterate ? cflsv.data() : cfl0.data();
      int iters = 1;
      R itersm1 = R(1), dtik = dti, splitfack = splitfac;
      for (int k = 0; k <= kmax; ++k) fo[k] = f[c + k * d.sk];
      const R* faux = fo.data();
      int it = 1;
      while (it <= iters) {
        if (it == 1) {
          for (int k = 0; k <= kmax; ++k) {
            fiaux[k] = fi[c + k * d.sk];
            hiaux[k] = hi[c + k * d.sk];
            advaux[k] = adv[c + k * d.sk];
          }
          faux = fo.data();
        }
        if (iterate) {
          if (it == 1) {
            for (int k = 0; k <= kmax; ++k) cflsv[k] = cfl0[k];
          } else if (scheme != UPSTREAM || iters < itersmax) {
            for (int k = 1 - kshift; k <= kmax - 1; ++k)
              cflsv[k] = absval(ww[c + k * d.sk]) * dti / (R(0.5) * (hiaux[k] + hiaux[k + 1]));
          }
          if (iters < itersmax) {
            int iters_new = 1;
            for (int k = 1 - kshift; k <= kmax - 1; ++k)
              iters_new = std::max(iters_new, ceil_int(cflsv[k]));
            if (iters_new > iters) {
              if (iters_new > itersmax) {
                ++too_many;
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
        }
        for (int k = 1 - kshift; k <= kmax - 1; ++k) {
          R w = ww[c + k * d.sk];
          R fu, fuu = R(0), fd = R(0);
          if (w > R(0)) {
            fu = faux[k];
            if (scheme != UPSTREAM) use_limiter = (k > 1 - kshift);
            if (use_limiter) {
              fuu = faux[k - 1];
              fd = faux[k + 1];
            }
          } else {
            fu = faux[k + 1];
            if (scheme != UPSTREAM) use_limiter = (k < kmax - 1);
            if (use_limiter) {
              fuu = faux[k + 2];
              fd = faux[k];
            }
          }
          if (use_limiter) fu = adv_interfacial_reconstruction<R>(scheme, cfls[k] * itersm1, fuu, fu, fd);
          wflux[k] = w * fu;
        }
        for (int k = 1; k <= kmax - kshift; ++k) {
          R hio = hiaux[k];
          hiaux[k] = hio - dtik * (ww[c + k * d.sk] - ww[c + (k - 1) * d.sk]);
          R advn = splitfack * (wflux[k] - wflux[k - 1]);
          fiaux[k] = (hio * fiaux[k] - dt * advn) / hiaux[k];
          advaux[k] = advaux[k] + advn;
        }
        faux = fiaux.data();
        ++it;
      }
      for (int k = 1; k <= kmax - kshift; ++k) {
        fi[c + k * d.sk] = fiaux[k];
        hi[c + k * d.sk] = hiaux[k];
        adv[c + k * d.sk] = advaux[k];
      }
    }
  }
  return too_many;
}

// ---------------------------------------------------------------------------------------------
// advection.F90:362-702 do_advection (2D split driver; the split schemes only).
template <class R>
int do_advection(const Dom& d, const AdvGrid& g, R dt, R* f, const R* U, const R* V, const R* DU,
                 const R* DV, const R* Do, const R* /*Dn*/, int split, int scheme, R AH, R* Dires,
                 R* advres) {
  const long n = d.n2d();
  std::vector<R> Di_loc, adv_loc, fi;
  R* p_Di = Dires;
  if (!p_Di) { Di_loc.assign(n, R(0)); p_Di = Di_loc.data(); }
  R* p_adv = advres;
  if (!p_adv) { adv_loc.assign(n, R(0)); p_adv = adv_loc.data(); }
  // p_Di = Do over the whole array, p_adv = 0 (:459, :466)
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      p_Di[d.ix(i, j)] = Do[d.ix(i, j)];
      p_adv[d.ix(i, j)] = R(0);
    }
  if (scheme == NOADV) return 0;
  if (scheme != UPSTREAM && scheme != P2 && scheme != SUPERBEE && scheme != MUSCL && scheme != P2_PDM)
    return -1;
  switch (split) {
    case NOSPLIT: {
      fi.assign(f, f + n);
      adv_split_u<R>(d, dt, f, fi.data(), p_Di, p_adv, U, DU, R(1), scheme, AH, g.uflux, g.uupdate);
      adv_split_v<R>(d, dt, f, fi.data(), p_Di, p_adv, V, DV, R(1), scheme, AH, g.vflux, g.vupdate);
      for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
        for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
          long p = d.ix(i, j);
          if (g.finalise[p]) f[p] = (Do[p] * f[p] - dt * p_adv[p]) / p_Di[p];
        }
      break;
    }
    case FULLSPLIT:
      adv_split_u<R>(d, dt, f, f, p_Di, p_adv, U, DU, R(1), scheme, AH, g.uflux, g.uupdate);
      adv_split_v<R>(d, dt, f, f, p_Di, p_adv, V, DV, R(1), scheme, AH, g.vflux, g.vupdate);
      break;
    case HALFSPLIT:
      adv_split_u<R>(d, dt, f, f, p_Di, p_adv, U, DU, R(0.5), scheme, AH, g.uflux, g.uupdate);
      adv_split_v<R>(d, dt, f, f, p_Di, p_adv, V, DV, R(1), scheme, AH, g.vflux, g.vupdate);
      adv_split_u<R>(d, dt, f, f, p_Di, p_adv, U, DU, R(0.5), scheme, AH, g.uflux, g.uupdate);
      break;
    default:
      return -1;
  }
  return 0;
}

// ---------------------------------------------------------------------------------------------
// advection_3d.F90:120-598 do_advection_3d (split schemes). hires/advres may be null.
// Returns 0, or -1 for an invalid split/scheme (the reference stops), or the count of columns
// whose vertical iteration estimate exceeded adv_ver_iterations.
template <class R>
long do_advection_3d(const Dom& d, const AdvGrid& g, R dt, R* f, const R* uu, const R* vv,
                     const R* ww, const R* hu, const R* hv, const R* ho, const R* hn, int split,
                     int hscheme, int vscheme, R AH, int tag, R* hires, R* advres,
                     int adv_ver_iterations) {
  const long n3 = d.n3d();
  std::vector<R> hi_loc, adv_loc, fi;
  R* p_hi = hires;
  if (!p_hi) { hi_loc.resize(n3); p_hi = hi_loc.data(); }
  R* p_adv = advres;
  if (!p_adv) { adv_loc.resize(n3); p_adv = adv_loc.data(); }
  for (long q = 0; q < n3; ++q) { p_hi[q] = ho[q]; p_adv[q] = R(0); }
  const int kmax = d.kmax;
  auto lvl = [&](const R* a, int k) { return a + (long)k * d.sk; };
  auto lvlw = [&](R* a, int k) { return a + (long)k * d.sk; };
  long warn = 0;
  if (hscheme == NOADV && vscheme == NOADV) return 0;
  if (hscheme == NOADV) {
    if (kmax > 1)
      warn += adv_split_w<R>(d, dt, f, f, p_hi, p_adv, ww, R(1), vscheme, tag, g.az, adv_ver_iterations);
    return warn;
  }
  auto hvalid = [](int s) { return s == UPSTREAM || s == P2 || s == SUPERBEE || s == MUSCL || s == P2_PDM; };
  if (!hvalid(hscheme)) return -1;
  if (vscheme == NOADV) {
    // do_advection stops on split=HVSPLIT ('split is invalid', advection.F90:668-670)
    for (int k = 1; k <= kmax; ++k)
      if (do_advection<R>(d, g, dt, lvlw(f, k), lvl(uu, k), lvl(vv, k), lvl(hu, k), lvl(hv, k), lvl(ho, k),
                          lvl(hn, k), split, hscheme, AH, lvlw(p_hi, k), lvlw(p_adv, k)) != 0)
        return -1;
    return 0;
  }
  switch (split) {
    case NOSPLIT: {
      fi.assign(f, f + n3);
      for (int k = 1; k <= kmax; ++k) {
        adv_split_u<R>(d, dt, lvl(f, k), lvlw(fi.data(), k), lvlw(p_hi, k), lvlw(p_adv, k), lvl(uu, k),
                       lvl(hu, k), R(1), hscheme, AH, g.uflux, g.uupdate);
        adv_split_v<R>(d, dt, lvl(f, k), lvlw(fi.data(), k), lvlw(p_hi, k), lvlw(p_adv, k), lvl(vv, k),
                       lvl(hv, k), R(1), hscheme, AH, g.vflux, g.vupdate);
      }
      if (kmax > 1) warn += adv_split_w<R>(d, dt, f, fi.data(), p_hi, p_adv, ww, R(1), vscheme, tag, g.az, 1);
      for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
        for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
          long c = d.ix(i, j);
          if (!g.finalise[c]) continue;
          for (int k = 1; k <= kmax; ++k) {
            long p = c + k * d.sk;
            f[p] = (ho[p] * f[p] - dt * p_adv[p]) / p_hi[p];
          }
        }
      break;
    }
    case FULLSPLIT:
      for (int k = 1; k <= kmax; ++k)
        do_advection<R>(d, g, dt, lvlw(f, k), lvl(uu, k), lvl(vv, k), lvl(hu, k), lvl(hv, k), lvl(ho, k),
                        lvl(hn, k), FULLSPLIT, hscheme, AH, lvlw(p_hi, k), lvlw(p_adv, k));
      if (kmax > 1)
        warn += adv_split_w<R>(d, dt, f, f, p_hi, p_adv, ww, R(1), vscheme, tag, g.az, adv_ver_iterations);
      break;
    case HALFSPLIT:
      for (int k = 1; k <= kmax; ++k)
        adv_split_u<R>(d, dt, lvl(f, k), lvlw(f, k), lvlw(p_hi, k), lvlw(p_adv, k), lvl(uu, k), lvl(hu, k),
                       R(0.5), hscheme, AH, g.uflux, g.uupdate);
      for (int k = 1; k <= kmax; ++k)
        adv_split_v<R>(d, dt, lvl(f, k), lvlw(f, k), lvlw(p_hi, k), lvlw(p_adv, k), lvl(vv, k), lvl(hv, k),
                       R(0.5), hscheme, AH, g.vflux, g.vupdate);
      if (kmax > 1)
        warn += adv_split_w<R>(d, dt, f, f, p_hi, p_adv, ww, R(1), vscheme, tag, g.az, adv_ver_iterations);
      for (int k = 1; k <= kmax; ++k)
        adv_split_v<R>(d, dt, lvl(f, k), lvlw(f, k), lvlw(p_hi, k), lvlw(p_adv, k), lvl(vv, k), lvl(hv, k),
                       R(0.5), hscheme, AH, g.vflux, g.vupdate);
      for (int k = 1; k <= kmax; ++k)
        adv_split_u<R>(d, dt, lvl(f, k), lvlw(f, k), lvlw(p_hi, k), lvlw(p_adv, k), lvl(uu, k), lvl(hu, k),
                       R(0.5), hscheme, AH, g.uflux, g.uupdate);
      break;
    case HVSPLIT:
      for (int k = 1; k <= kmax; ++k)
        do_advection<R>(d, g, dt, lvlw(f, k), lvl(uu, k), lvl(vv, k), lvl(hu, k), lvl(hv, k), lvl(ho, k),
                        lvl(hn, k), NOSPLIT, hscheme, AH, lvlw(p_hi, k), lvlw(p_adv, k));
      if (kmax > 1)
        warn += adv_split_w<R>(d, dt, f, f, p_hi, p_adv, ww, R(1), vscheme, tag, g.az, adv_ver_iterations);
      break;
    default:
      return -1;
  }
  return warn;
}

// ---------------------------------------------------------------------------------------------
// tridiagonal.F90:35-48 getm_tridiagonal. Arrays indexed 0..kmax.
template <class R>
void getm_tridiagonal(int kmax, int fi, int lt, const R* au, const R* bu, const R* cu, const R* du,
                      R* value) {
  std::vector<R> ru(kmax + 1), qu(kmax + 1);
  ru[lt] = au[lt] / bu[lt];
  qu[lt] = du[lt] / bu[lt];
  for (int i = lt - 1; i >= fi + 1; --i) {
    ru[i] = au[i] / (bu[i] - cu[i] * ru[i + 1]);
    qu[i] = (du[i] - cu[i] * qu[i + 1]) / (bu[i] - cu[i] * ru[i + 1]);
  }
  qu[fi] = (du[fi] - cu[fi] * qu[fi + 1]) / (bu[fi] - cu[fi] * ru[fi + 1]);
  value[fi] = qu[fi];
  for (int i = fi + 1; i <= lt; ++i) value[i] = qu[i] - ru[i] * value[i - 1];
}

// ---------------------------------------------------------------------------------------------
// Implicit vertical diffusion of a tracer: salinity.F90:348-389 (src == null), or the
// temperature form temperature.F90:471-550 when src != null: src holds, per column, dry_z*dt times
// the radiation/surface-flux increment of each layer, i.e.
//   layer kmax: dry_z*dt*(rad1d(kmax)+shf*rho_0_cpi-rad1d(kmax-1)),
//   layer k<kmax: dry_z*dt*(rad1d(k)-rad1d(k-1)).
template <class R>
void tracer_vdiff(const Dom& d, R dt, R cnpar, R avmol, R* S, const R* hn, const R* nuh,
                  const int32_t* az, const R* src) {
  const int kmax = d.kmax;
  if (kmax <= 1) return;
#pragma omp parallel for schedule(static)
  for (int j = d.jmin; j <= d.jmax; ++j) {
    std::vector<R> auxo(kmax + 1), auxn(kmax + 1), a1(kmax + 1), a2(kmax + 1), a3(kmax + 1),
        a4(kmax + 1), Res(kmax + 1);
    for (int i = d.imin; i <= d.imax; ++i) {
      long c = d.ix(i, j);
      if (az[c] != 1) continue;
      auto A = [&](const R* a, int k) { return a[c + (long)k * d.sk]; };
      for (int k = 1; k <= kmax - 1; ++k) {
        auxo[k] = R(2) * (R(1) - cnpar) * dt * (A(nuh, k) + avmol) / (A(hn, k + 1) + A(hn, k));
        auxn[k] = R(2) * cnpar * dt * (A(nuh, k) + avmol) / (A(hn, k + 1) + A(hn, k));
      }
      int k = kmax;
      a1[k] = -auxn[k - 1];
      a2[k] = A(hn, k) + auxn[k - 1];
      a4[k] = A(S, k) * (A(hn, k) - auxo[k - 1]) + A(S, k - 1) * auxo[k - 1];
      if (src) a4[k] = a4[k] + A(src, k);
      for (k = 2; k <= kmax - 1; ++k) {
        a3[k] = -auxn[k];
        a1[k] = -auxn[k - 1];
        a2[k] = A(hn, k) + auxn[k] + auxn[k - 1];
        a4[k] = A(S, k + 1) * auxo[k] + A(S, k) * (A(hn, k) - auxo[k] - auxo[k - 1]) +
                A(S, k - 1) * auxo[k - 1];
        if (src) a4[k] = a4[k] + A(src, k);
      }
      k = 1;
      a3[k] = -auxn[k];
      a2[k] = A(hn, k) + auxn[k];
      a4[k] = A(S, k + 1) * auxo[k] + A(S, k) * (A(hn, k) - auxo[k]);
      if (src) a4[k] = a4[k] + A(src, k);
      getm_tridiagonal<R>(kmax, 1, kmax, a1.data(), a2.data(), a3.data(), a4.data(), Res.data());
      for (k = 1; k <= kmax; ++k) S[c + (long)k * d.sk] = Res[k];
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Tracer content sum_{wet interior cells} f*h/ard1 with Neumaier compensation (a diagnostic the
// reference does not have; used for the conservation checks).
template <class R>
double tracer_content(const Dom& d, const R* f, const R* h, const int32_t* az) {
  double s = 0.0, comp = 0.0;
  for (int k = 1; k <= d.kmax; ++k)
    for (int j = d.jmin; j <= d.jmax; ++j)
      for (int i = d.imin; i <= d.imax; ++i) {
        long c = d.ix(i, j);
        if (az[c] < 1) continue;
        long p = c + (long)k * d.sk;
        double x = (double)f[p] * (double)h[p] / d.ard1;
        double t = s + x;
        if (std::fabs(s) >= std::fabs(x)) comp += (s - t) + x; else comp += (x - t) + s;
        s = t;
      }
  return s + comp;
}

// ---------------------------------------------------------------------------------------------
// init_advection masks (advection.F90:263-318) from az/au/av/ax (int32, E2DFIELD). Writes the
// six byte masks of the H, U and V grids into out[0..17] in the order
//   H: uflux vflux uupdate vupdate finalise (5), U: same (5), V: same (5), plus xflux (1)
// -- see make_adv_grids for the exact mapping (pointer remaps of :287-318 resolved into copies).
struct AdvMasks {
  std::vector<uint8_t> updateH, uflux, vflux, xflux, uupdateU, vupdateV, uflux_U, vflux_V, xflux_U_unused;
};

inline void build_adv_masks(const Dom& d, const int32_t* az, const int32_t* au, const int32_t* av,
                            const int32_t* ax, AdvMasks& m) {
  const long n = d.n2d();
  m.updateH.assign(n, 0); m.uflux.assign(n, 0); m.vflux.assign(n, 0); m.xflux.assign(n, 0);
  m.uupdateU.assign(n, 0); m.vupdateV.assign(n, 0); m.uflux_U.assign(n, 0); m.vflux_V.assign(n, 0);
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      long p = d.ix(i, j);
      m.updateH[p] = az[p] == 1;
      m.uflux[p] = (au[p] == 1 || au[p] == 2) && i != d.imax + HALO;
      m.vflux[p] = (av[p] == 1 || av[p] == 2) && j != d.jmax + HALO;
      m.xflux[p] = ax[p] == 1 && i != d.imax + HALO && j != d.jmax + HALO;
      m.uupdateU[p] = au[p] == 1;
      m.vupdateV[p] = av[p] == 1;
    }
  // U grid u-flux mask: mask_updateH(i+1,j) (advection.F90:287-291); V grid v-flux mask:
  // mask_updateH(i,j+1) (:307). Entries with no source element stay false and are never read.
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      long p = d.ix(i, j);
      if (i + 1 <= d.imax + HALO) m.uflux_U[p] = m.updateH[d.ix(i + 1, j)];
      if (j + 1 <= d.jmax + HALO) m.vflux_V[p] = m.updateH[d.ix(i, j + 1)];
    }
}

inline AdvGrid adv_grid(const AdvMasks& m, int tag, const int32_t* az, const int32_t* au,
                        const int32_t* av) {
  AdvGrid g{};
  switch (tag) {
    case U_TAG:  // advection.F90:287-304
      g = {m.uflux_U.data(), m.xflux.data(), m.uupdateU.data(), m.uflux.data(), m.uflux.data(), au};
      break;
    case V_TAG:  // advection.F90:306-318
      g = {m.xflux.data(), m.vflux_V.data(), m.vflux.data(), m.vupdateV.data(), m.vflux.data(), av};
      break;
    default:  // H_TAG, D_TAG, W_TAG (advection.F90:278-284)
      g = {m.uflux.data(), m.vflux.data(), m.updateH.data(), m.updateH.data(), m.updateH.data(), az};
  }
  return g;
}

// Masks au/av/ax from az (domain.F90:292-346), over the haloed index range.
inline void derive_uvx_masks(const Dom& d, const int32_t* az, int32_t* au, int32_t* av, int32_t* ax) {
  const long n = d.n2d();
  std::fill(au, au + n, 0); std::fill(av, av + n, 0); std::fill(ax, ax + n, 0);
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO - 1; ++i) {
      int a = az[d.ix(i, j)], b = az[d.ix(i + 1, j)];
      int v = 0;
      if (a == 1 && b == 1) v = 1;
      if ((a == 1 && b == 2) || (a == 2 && b == 1)) v = 2;
      if (a == 2 && b == 2) v = 3;
      au[d.ix(i, j)] = v;
    }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO - 1; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      int a = az[d.ix(i, j)], b = az[d.ix(i, j + 1)];
      int v = 0;
      if (a == 1 && b == 1) v = 1;
      if ((a == 1 && b == 2) || (a == 2 && b == 1)) v = 2;
      if (a == 2 && b == 2) v = 3;
      av[d.ix(i, j)] = v;
    }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO - 1; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO - 1; ++i)
      if (az[d.ix(i, j)] >= 1 && az[d.ix(i, j + 1)] >= 1 && az[d.ix(i + 1, j)] >= 1 &&
          az[d.ix(i + 1, j + 1)] >= 1)
        ax[d.ix(i, j)] = 1;
}

}  // namespace gor
