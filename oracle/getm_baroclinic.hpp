// getm_baroclinic.hpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of GETM 2.5's mode-split time step (the barotropic micro step integrate_2d and
// the baroclinic macro step integrate_3d) for the closed-boundary, sigma-coordinate, prescribed
// viscosity configuration, used as the parity oracle of the CUDA baroclinic path. Each routine
// follows the reference file:line given beside it, with the same loop bounds and expression order
// (no contraction: build with -ffp-contract=off). Fields of the module state (variables_2d,
// variables_3d, domain) are passed as one table of pointers (BcState); 3D fields may be FP64 or
// FP32 (template R3), 2D fields are always FP64.
//
// Scope: runtype 4 (prognostic T and S); open boundaries of the four 2D types (update_2d_bdy,
// mirror_bdy_2d/3d); vert_cord = 1 with equidistant sigma; eqstate_method 1 (linear), 2 (UNESCO80)
// or 3 (Jackett et al. 2006); ip_method 1 to 7; num/nuh prescribed (CONSTANT_VISCOSITY) or
// the PARABOLIC_VISCOSITY profile of gotm(); short-wave radiation and surface heat flux in
// do_temperature; sealevel_nan_check; no numerical-mixing analysis; no rivers; An_method = 0 and
// Am = 0 (no horizontal momentum diffusion).
#pragma once
#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>

#include "getm_oracle.hpp"

namespace gor {

// Field tables: ORDER MATTERS (mirrored by code_b200/state.py and include/getm_b200.h).
enum F2 {
  Z, ZO, U_, V_, D_, DU, DV, UEX, VEX, FU, FV, RU, RV, RUU, RVV, UINT, VINT, UINTO, VINTO, SLUX, SLVX, SLRU, SLRV,
  ZUB, ZVB, ZUB0, ZVB0, FWF, HH, HU, HV, DRY_Z, DRY_U, DRY_V, CORU, CORV, TAUSX, TAUSY, AIRP, SSEO, SSEN, SSUO,
  SSUN, SSVO, SSVN, DN, DUN, DVN, RRU, RRV, TAUBX, TAUBY, TAUB, TAUS, SWR, SHF, ATT_A, ATT_G1, ATT_G2, NF2
};
enum F3 {
  UU, VV, WW, HO, HN, HUO, HUN, HVO, HVN, UUEX, VVEX, IDPDX, IDPDY, TT, SS, RHO, BUOY, NUM, NUH, RAD, TKE, EPS,
  TLO, SLO, NF3  // TLO, SLO: the mixed step's compensated storage (not read by the FP64 restatement)
};
enum PD {
  P_DTM, P_DT, P_CNPAR, P_MIN_DEPTH, P_CRIT_DEPTH, P_G, P_RHO_0, P_KAPPA, P_AVMMOL, P_AVMOLT, P_AVMOLS, P_T0, P_S0,
  P_DTR0, P_DSR0, P_IP_FAC, P_TEMP_AH, P_SALT_AH, P_AVMBACK, P_AVHBACK, P_CP, P_SWR_BOT_REFL_FRAC,
  P_SWR_MIN_BOT_FRAC, NPD
};
enum PI {
  I_M, I_MM, I_RUNTYPE, I_VEL2D_SPLIT, I_VEL2D_HOR, I_VEL3D_SPLIT, I_VEL3D_HOR, I_VEL3D_VER, I_TEMP_SPLIT, I_TEMP_HOR,
  I_TEMP_VER, I_SALT_SPLIT, I_SALT_HOR, I_SALT_VER, I_ADV_VER_ITERS, I_UFIRST2D, I_UFIRST3D, I_CALC_TEMP,
  I_CALC_SALT, I_IP_METHOD, I_VISCOSITY, I_EQSTATE_METHOD, I_SEALEVEL_CHECK, I_RADIATION, I_NAN_WARNED, NPI
};
// I_VISCOSITY: 0 = CONSTANT_VISCOSITY (num, nuh as given), 1 = PARABOLIC_VISCOSITY (gotm.F90:131-143)
// I_EQSTATE_METHOD: 1 linear, 2 UNESCO80, 3 Jackett et al. 2006 (eqstate.F90:94-261)
// I_RADIATION: 0 = no short-wave radiation or surface heat flux in do_temperature, 1 = both
// I_NAN_WARNED: the SAVEd have_warned of sealevel_nan_check (sealevel.F90:178)

// Open boundaries (domain.F90:263-280, bdy_spec.F90:225-290): segments per side -- western
// (wi, wfj..wlj), northern (nj, nfi..nli), eastern (ei, efj..elj), southern (sj, sfi..sli) -- with
// a 2D type each (cppdefs.h:65-69), and the elevation data of the boundary points in segment
// order (bdy_data; bdy_data_u/v for FLATHER_ELEV). With harmonic data the elevation of point p at
// micro step `loop` is amp[p]*sin(2*pi*loop*dtm/period + phase[p]) (the configurations' tide;
// the reference reads its boundary data from files).
enum { ZERO_GRADIENT = 1, SOMMERFELD = 2, CLAMPED = 3, FLATHER_ELEV = 4 };
struct Bdy {
  int nwb = 0, nnb = 0, neb = 0, nsb = 0;
  std::vector<int> seg;     // 3 ints per segment, sides in the order W, N, E, S
  std::vector<int> type2d;  // per segment
  int ramp = -1;            // bdy2d_ramp
  std::vector<double> data, data_u, data_v;  // per boundary point (used when amp is empty)
  std::vector<double> amp, phase;            // harmonic elevation per boundary point
  double period = 0.0;
  int nseg() const { return nwb + nnb + neb + nsb; }
};

template <class R3>
struct BcState {
  double* f2[NF2];
  R3* f3[NF3];
  const int32_t *az, *au, *av, *ax;
  double par[NPD];
  int ipar[NPI];
  const Bdy* bdy = nullptr;  // open boundaries (nullptr: closed domain)
};

// ---------------------------------------------------------------------------------------------
// 2D helpers
struct A2 {
  const Dom& d;
  double* p;
  double& operator()(int i, int j) const { return p[d.ix(i, j)]; }
};
struct M2 {
  const Dom& d;
  const int32_t* p;
  int operator()(int i, int j) const { return p[d.ix(i, j)]; }
};
template <class R>
struct A3 {
  const Dom& d;
  R* p;
  R& operator()(int i, int j, int k) const { return p[d.ix3(i, j, k)]; }
};

// bottom_friction.F90:48-150 (runtype>1 branch uses the stored ruu/rvv).
inline void bottom_friction(const Dom& d, BcState<double>* /*unused*/, double** f2, const int32_t* aup,
                            const int32_t* avp, const double* par, int runtype) {
  A2 U{d, f2[U_]}, V{d, f2[V_]}, DU_{d, f2[DU]}, DV_{d, f2[DV]}, ruu{d, f2[RUU]}, rvv{d, f2[RVV]}, ru{d, f2[RU]},
      rv{d, f2[RV]}, zub{d, f2[ZUB]}, zvb{d, f2[ZVB]}, zub0{d, f2[ZUB0]}, zvb0{d, f2[ZVB0]};
  M2 au{d, aup}, av{d, avp};
  const double kappa = par[P_KAPPA], avmmol = par[P_AVMMOL], min_depth = par[P_MIN_DEPTH];
  const long n = d.n2d();
  std::vector<double> uloc_(n, 0.0), vloc_(n, 0.0), HH_(n, 0.0), fricvel_(n, 0.0);
  A2 uloc{d, uloc_.data()}, vloc{d, vloc_.data()}, HH{d, HH_.data()}, fricvel{d, fricvel_.data()};
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) {
      if (au(i, j) > 0)
        vloc(i, j) = 0.25 * (V(i, j) / DV_(i, j) + V(i + 1, j) / DV_(i + 1, j) + V(i, j - 1) / DV_(i, j - 1) +
                             V(i + 1, j - 1) / DV_(i + 1, j - 1));
      else
        vloc(i, j) = 0.0;
    }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO - 1; ++i)
      if (au(i, j) > 0) {
        uloc(i, j) = U(i, j) / DU_(i, j);
        HH(i, j) = std::max(min_depth, DU_(i, j));
        double x = kappa / std::log((zub(i, j) + 0.5 * HH(i, j)) / zub(i, j));
        ruu(i, j) = x * x;
      }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO - 1; ++i)
      if (au(i, j) > 0) {
        if (runtype == 1) {
          fricvel(i, j) = std::sqrt(ruu(i, j) * (uloc(i, j) * uloc(i, j) + vloc(i, j) * vloc(i, j)));
          zub(i, j) = std::min(HH(i, j), zub0(i, j) + 0.1 * avmmol / std::max(avmmol, fricvel(i, j)));
          ruu(i, j) = (zub(i, j) + 0.5 * HH(i, j)) / zub(i, j);
          double x = kappa / std::log(ruu(i, j));
          ruu(i, j) = x * x;
        }
        ru(i, j) = ruu(i, j) * std::sqrt(uloc(i, j) * uloc(i, j) + vloc(i, j) * vloc(i, j));
      }
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) {
      if (av(i, j) > 0)
        uloc(i, j) = 0.25 * (U(i, j) / DU_(i, j) + U(i - 1, j) / DU_(i - 1, j) + U(i, j + 1) / DU_(i, j + 1) +
                             U(i - 1, j + 1) / DU_(i - 1, j + 1));
      else
        uloc(i, j) = 0.0;
    }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO - 1; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i)
      if (av(i, j) > 0) {
        vloc(i, j) = V(i, j) / DV_(i, j);
        HH(i, j) = std::max(min_depth, DV_(i, j));
        double x = kappa / std::log((zvb(i, j) + 0.5 * HH(i, j)) / zvb(i, j));
        rvv(i, j) = x * x;
      }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO - 1; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i)
      if (av(i, j) > 0) {
        if (runtype == 1) {
          fricvel(i, j) = std::sqrt(rvv(i, j) * (uloc(i, j) * uloc(i, j) + vloc(i, j) * vloc(i, j)));
          zvb(i, j) = std::min(HH(i, j), zvb0(i, j) + 0.1 * avmmol / std::max(avmmol, fricvel(i, j)));
          rvv(i, j) = (zvb(i, j) + 0.5 * HH(i, j)) / zvb(i, j);
          double x = kappa / std::log(rvv(i, j));
          rvv(i, j) = x * x;
        }
        rv(i, j) = rvv(i, j) * std::sqrt(uloc(i, j) * uloc(i, j) + vloc(i, j) * vloc(i, j));
      }
}

// uv_advect.F90:94-300 (split schemes only, vel2d_adv_hor != J7): 2D momentum advection on the
// U and V grids via do_advection with advres = UEx / VEx.
inline int uv_advect_2d(const Dom& d, const AdvMasks& m, const int32_t* az, const int32_t* au, const int32_t* av,
                        double dtm, const double* Up, const double* Vp, const double* DUp, const double* DVp,
                        int split, int hor, double* UEx, double* VEx) {
  const long n = d.n2d();
  if (hor == NOADV) {
    std::fill(UEx, UEx + n, 0.0);
    std::fill(VEx, VEx + n, 0.0);
    return 0;
  }
  A2 U{d, const_cast<double*>(Up)}, V{d, const_cast<double*>(Vp)}, DU_{d, const_cast<double*>(DUp)},
      DV_{d, const_cast<double*>(DVp)};
  // automatic arrays of the reference: undefined outside the loops; zero here
  std::vector<double> fadv_(n, 0.0), Uadv_(n, 0.0), Vadv_(n, 0.0), DUadv_(n, 0.0), DVadv_(n, 0.0);
  A2 fadv{d, fadv_.data()}, Uadv{d, Uadv_.data()}, Vadv{d, Vadv_.data()}, DUadv{d, DUadv_.data()},
      DVadv{d, DVadv_.data()};
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO - 1; ++i) {
      fadv(i, j) = U(i, j) / DU_(i, j);
      Uadv(i, j) = 0.5 * (U(i, j) + U(i + 1, j));
      Vadv(i, j) = 0.5 * (V(i, j) + V(i + 1, j));
      DUadv(i, j) = 0.5 * (DU_(i, j) + DU_(i + 1, j));
      DVadv(i, j) = 0.5 * (DV_(i, j) + DV_(i + 1, j));
    }
  AdvGrid gu = adv_grid(m, U_TAG, az, au, av);
  if (do_advection<double>(d, gu, dtm, fadv_.data(), Uadv_.data(), Vadv_.data(), DUadv_.data(), DVadv_.data(), DUp,
                           DUp, split, hor, 0.0, nullptr, UEx) != 0)
    return -1;
  for (int j = d.jmin - HALO; j <= d.jmax + HALO - 1; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      fadv(i, j) = V(i, j) / DV_(i, j);
      Uadv(i, j) = 0.5 * (U(i, j) + U(i, j + 1));
      Vadv(i, j) = 0.5 * (V(i, j) + V(i, j + 1));
      DUadv(i, j) = 0.5 * (DU_(i, j) + DU_(i, j + 1));
      DVadv(i, j) = 0.5 * (DV_(i, j) + DV_(i, j + 1));
    }
  AdvGrid gv = adv_grid(m, V_TAG, az, au, av);
  if (do_advection<double>(d, gv, dtm, fadv_.data(), Uadv_.data(), Vadv_.data(), DUadv_.data(), DVadv_.data(), DVp,
                           DVp, split, hor, 0.0, nullptr, VEx) != 0)
    return -1;
  return 0;
}

// update_2d_bdy.F90:74-178 -- elevations of the open-boundary points (after the Uint accumulation,
// before sealevel, m2d.F90:475).
inline void update_2d_bdy(const Dom& d, const Bdy& b, double** f2, const double* par, int loop) {
  A2 z{d, f2[Z]}, D{d, f2[D_]}, U{d, f2[U_]}, DU_{d, f2[DU]}, V{d, f2[V_]}, DV_{d, f2[DV]}, H{d, f2[HH]};
  const double dtm = par[P_DTM], min_depth = par[P_MIN_DEPTH];
  const double g = (double)9.81f;  // the single-precision literal of update_2d_bdy.F90:92,96
  double fac = 1.0;
  if (b.ramp > 1) fac = std::min(1.0, 4.0 * loop / (double)(float)b.ramp);
  auto data = [&](int k, int which) -> double {  // k: 1-based point index
    if (which == 0) {
      if (!b.amp.empty()) {
        const double pi2 = 2.0 * 3.14159265358979323846;
        return b.amp[k - 1] * std::sin(pi2 * (loop * dtm) / b.period + b.phase[k - 1]);
      }
      return b.data[k - 1];
    }
    const std::vector<double>& v = which == 1 ? b.data_u : b.data_v;
    return v.empty() ? 0.0 : v[k - 1];
  };
  int l = 0, k = 1;
  for (int n = 0; n < b.nwb; ++n, ++l) {
    const int i = b.seg[3 * l], jf = b.seg[3 * l + 1], jl = b.seg[3 * l + 2];
    for (int j = jf; j <= jl; ++j, ++k) switch (b.type2d[l]) {
        case ZERO_GRADIENT: z(i, j) = z(i + 1, j); break;
        case SOMMERFELD: z(i, j) = z(i, j) + dtm / d.dx * std::sqrt(g * D(i, j)) * (z(i + 1, j) - z(i, j)); break;
        case CLAMPED: z(i, j) = std::max(fac * data(k, 0), -H(i, j) + min_depth); break;
        case FLATHER_ELEV: {
          const double a = std::sqrt(DU_(i, j) / g) * (U(i, j) / DU_(i, j) - data(k, 1));
          z(i, j) = std::max(fac * (data(k, 0) - a), -H(i, j) + min_depth);
        } break;
      }
  }
  for (int n = 0; n < b.nnb; ++n, ++l) {
    const int j = b.seg[3 * l], if_ = b.seg[3 * l + 1], il = b.seg[3 * l + 2];
    for (int i = if_; i <= il; ++i, ++k) switch (b.type2d[l]) {
        case ZERO_GRADIENT: z(i, j) = z(i, j - 1); break;
        case SOMMERFELD: z(i, j) = z(i, j) - dtm / d.dy * std::sqrt(g * D(i, j)) * (z(i, j) - z(i, j - 1)); break;
        case CLAMPED: z(i, j) = std::max(fac * data(k, 0), -H(i, j) + min_depth); break;
        case FLATHER_ELEV: {
          const double a = std::sqrt(DV_(i, j) / g) * (V(i, j - 1) / DV_(i, j - 1) - data(k, 2));
          z(i, j) = std::max(fac * (data(k, 0) + a), -H(i, j) + min_depth);
        } break;
      }
  }
  for (int n = 0; n < b.neb; ++n, ++l) {
    const int i = b.seg[3 * l], jf = b.seg[3 * l + 1], jl = b.seg[3 * l + 2];
    for (int j = jf; j <= jl; ++j, ++k) switch (b.type2d[l]) {
        case ZERO_GRADIENT: z(i, j) = z(i - 1, j); break;
        case SOMMERFELD: z(i, j) = z(i, j) - dtm / d.dx * std::sqrt(g * D(i, j)) * (z(i, j) - z(i - 1, j)); break;
        case CLAMPED: z(i, j) = std::max(fac * data(k, 0), -H(i, j) + min_depth); break;
        case FLATHER_ELEV: {
          const double a = std::sqrt(DU_(i, j) / g) * (U(i - 1, j) / DU_(i - 1, j) - data(k, 1));
          z(i, j) = std::max(fac * (data(k, 0) + a), -H(i, j) + min_depth);
        } break;
      }
  }
  for (int n = 0; n < b.nsb; ++n, ++l) {
    const int j = b.seg[3 * l], if_ = b.seg[3 * l + 1], il = b.seg[3 * l + 2];
    for (int i = if_; i <= il; ++i, ++k) switch (b.type2d[l]) {
        case ZERO_GRADIENT: z(i, j) = z(i, j + 1); break;
        case SOMMERFELD: z(i, j) = z(i, j) + dtm / d.dy * std::sqrt(g * D(i, j)) * (z(i, j + 1) - z(i, j)); break;
        case CLAMPED: z(i, j) = std::max(fac * data(k, 0), -H(i, j) + min_depth); break;
        case FLATHER_ELEV: {
          const double a = std::sqrt(DV_(i, j) / g) * (V(i, j) / DV_(i, j) - data(k, 2));
          z(i, j) = std::max(fac * (data(k, 0) - a), -H(i, j) + min_depth);
        } break;
      }
  }
}

// mirror_bdy_2d.F90 / mirror_bdy_3d.F90: copies across the open boundaries. tag 0 = U_TAG (U points
// with au == 3 on northern/southern boundaries), 1 = V_TAG (av == 3 on western/eastern ones),
// 2 = H/D_TAG (the value of a boundary point, az > 1, into the point outside). nl levels of a
// field with level stride sk (nl = 1 for 2D fields).
template <class R>
inline void mirror_bdy(const Dom& d, const Bdy& b, const int32_t* azp, const int32_t* aup, const int32_t* avp,
                       R* f, int tag, int nl, long sk) {
  M2 az{d, azp}, au{d, aup}, av{d, avp};
  auto cp = [&](int id, int jd, int is, int js) {
    for (int k = 0; k < nl; ++k) f[d.ix(id, jd) + k * sk] = f[d.ix(is, js) + k * sk];
  };
  const int W = 0, N = b.nwb, E = N + b.nnb, S = E + b.neb;
  auto sg = [&](int l, int q) { return b.seg[3 * l + q]; };
  if (tag == 0) {
    for (int n = 0; n < b.nnb; ++n) {
      const int j = sg(N + n, 0);
      for (int i = sg(N + n, 1) - HALO; i <= sg(N + n, 2) + HALO; ++i)
        if (au(i, j) == 3) cp(i, j, i, j - 1);
    }
    for (int n = 0; n < b.nsb; ++n) {
      const int j = sg(S + n, 0);
      for (int i = sg(S + n, 1) - HALO; i <= sg(S + n, 2) + HALO; ++i)
        if (au(i, j) == 3) cp(i, j, i, j + 1);
    }
  } else if (tag == 1) {
    for (int n = 0; n < b.nwb; ++n) {
      const int i = sg(W + n, 0);
      for (int j = sg(W + n, 1) - HALO; j <= sg(W + n, 2) + HALO; ++j)
        if (av(i, j) == 3) cp(i, j, i + 1, j);
    }
    for (int n = 0; n < b.neb; ++n) {
      const int i = sg(E + n, 0);
      for (int j = sg(E + n, 1) - HALO; j <= sg(E + n, 2) + HALO; ++j)
        if (av(i, j) == 3) cp(i, j, i - 1, j);
    }
  } else {
    for (int n = 0; n < b.nwb; ++n) {
      const int i = sg(W + n, 0);
      for (int j = sg(W + n, 1) - HALO; j <= sg(W + n, 2) + HALO; ++j)
        if (az(i, j) > 1) cp(i - 1, j, i, j);
    }
    for (int n = 0; n < b.nnb; ++n) {
      const int j = sg(N + n, 0);
      for (int i = sg(N + n, 1) - HALO; i <= sg(N + n, 2) + HALO; ++i)
        if (az(i, j) > 1) cp(i, j + 1, i, j);
    }
    for (int n = 0; n < b.neb; ++n) {
      const int i = sg(E + n, 0);
      for (int j = sg(E + n, 1) - HALO; j <= sg(E + n, 2) + HALO; ++j)
        if (az(i, j) > 1) cp(i + 1, j, i, j);
    }
    for (int n = 0; n < b.nsb; ++n) {
      const int j = sg(S + n, 0);
      for (int i = sg(S + n, 1) - HALO; i <= sg(S + n, 2) + HALO; ++i)
        if (az(i, j) > 1) cp(i, j - 1, i, j);
    }
  }
}

// momentum.F90:69-223 umomentum, :232-386 vmomentum (CARTESIAN, no NEW_CORI).
inline void umomentum(const Dom& d, double** f2, const int32_t* aup, const int32_t* avp, const double* par,
                      const Bdy* bdy = nullptr, const int32_t* azp = nullptr) {
  A2 U{d, f2[U_]}, DU_{d, f2[DU]}, z{d, f2[Z]}, H{d, f2[HH]}, D{d, f2[D_]}, airp{d, f2[AIRP]}, tausx{d, f2[TAUSX]},
      Slru{d, f2[SLRU]}, dry_u{d, f2[DRY_U]}, fV{d, f2[FV]}, UEx{d, f2[UEX]}, SlUx{d, f2[SLUX]}, ru{d, f2[RU]},
      fU{d, f2[FU]}, corv{d, f2[CORV]};
  M2 au{d, aup}, av{d, avp};
  const double g = par[P_G], rho_0 = par[P_RHO_0], dtm = par[P_DTM], min_depth = par[P_MIN_DEPTH];
  const double gamma = rho_0 * g;
  const double gammai = 1.0 / gamma;
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (au(i, j) == 1 || au(i, j) == 2) {
        double zp = std::max(z(i + 1, j), -H(i, j) + std::min(min_depth, D(i + 1, j)));
        double zm = std::max(z(i, j), -H(i + 1, j) + std::min(min_depth, D(i, j)));
        double zx = (zp - zm + (airp(i + 1, j) - airp(i, j)) * gammai) / d.dx;
        double tausu = 0.5 * (tausx(i, j) + tausx(i + 1, j));
        double Slr = U(i, j) > 0.0 ? std::max(Slru(i, j), 0.0) : std::min(Slru(i, j), 0.0);
        U(i, j) = (U(i, j) - dtm * (g * DU_(i, j) * zx +
                                    dry_u(i, j) * (-tausu / rho_0 - fV(i, j) + UEx(i, j) + SlUx(i, j) + Slr))) /
                  (1.0 + dtm * ru(i, j) / DU_(i, j));
      }
  if (bdy) mirror_bdy<double>(d, *bdy, azp, aup, avp, f2[U_], 0, 1, 0);  // momentum.F90:190
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) {
      if (av(i, j) >= 1) {
        double Uloc = 0.25 * (U(i - 1, j) + U(i, j) + U(i - 1, j + 1) + U(i, j + 1));
        fU(i, j) = corv(i, j) * Uloc;
      } else {
        fU(i, j) = 0.0;
      }
    }
}

inline void vmomentum(const Dom& d, double** f2, const int32_t* aup, const int32_t* avp, const double* par,
                      const Bdy* bdy = nullptr, const int32_t* azp = nullptr) {
  A2 V{d, f2[V_]}, DV_{d, f2[DV]}, z{d, f2[Z]}, H{d, f2[HH]}, D{d, f2[D_]}, airp{d, f2[AIRP]}, tausy{d, f2[TAUSY]},
      Slrv{d, f2[SLRV]}, dry_v{d, f2[DRY_V]}, fU{d, f2[FU]}, VEx{d, f2[VEX]}, SlVx{d, f2[SLVX]}, rv{d, f2[RV]},
      fV{d, f2[FV]}, coru{d, f2[CORU]};
  M2 au{d, aup}, av{d, avp};
  const double g = par[P_G], rho_0 = par[P_RHO_0], dtm = par[P_DTM], min_depth = par[P_MIN_DEPTH];
  const double gamma = rho_0 * g;
  const double gammai = 1.0 / gamma;
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (av(i, j) == 1 || av(i, j) == 2) {
        double zp = std::max(z(i, j + 1), -H(i, j) + std::min(min_depth, D(i, j + 1)));
        double zm = std::max(z(i, j), -H(i, j + 1) + std::min(min_depth, D(i, j)));
        double zy = (zp - zm + (airp(i, j + 1) - airp(i, j)) * gammai) / d.dy;
        double tausv = 0.5 * (tausy(i, j) + tausy(i, j + 1));
        double Slr = V(i, j) > 0.0 ? std::max(Slrv(i, j), 0.0) : std::min(Slrv(i, j), 0.0);
        V(i, j) = (V(i, j) - dtm * (g * DV_(i, j) * zy +
                                    dry_v(i, j) * (-tausv / rho_0 + fU(i, j) + VEx(i, j) + SlVx(i, j) + Slr))) /
                  (1.0 + dtm * rv(i, j) / DV_(i, j));
      }
  if (bdy) mirror_bdy<double>(d, *bdy, azp, aup, avp, f2[V_], 1, 1, 0);  // momentum.F90:353
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) {
      if (au(i, j) >= 1) {
        double Vloc = 0.25 * (V(i, j - 1) + V(i + 1, j - 1) + V(i, j) + V(i + 1, j));
        fV(i, j) = coru(i, j) * Vloc;
      } else {
        fV(i, j) = 0.0;
      }
    }
}

// sealevel.F90:65-112
inline void sealevel(const Dom& d, double** f2, const int32_t* azp, const double* par) {
  A2 z{d, f2[Z]}, zo{d, f2[ZO]}, U{d, f2[U_]}, V{d, f2[V_]}, fwf{d, f2[FWF]};
  M2 az{d, azp};
  const double dtm = par[P_DTM];
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) zo(i, j) = z(i, j);
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (az(i, j) == 1)
        z(i, j) = z(i, j) - dtm * ((U(i, j) * d.dy - U(i - 1, j) * d.dy) + (V(i, j) * d.dx - V(i, j - 1) * d.dx)) * d.ard1 +
                  dtm * fwf(i, j);
}

// depth_update.F90:55-110
inline void depth_update(const Dom& d, double** f2, const int32_t* azp, const int32_t* aup, const int32_t* avp,
                         const double* par) {
  A2 D{d, f2[D_]}, z{d, f2[Z]}, zo{d, f2[ZO]}, H{d, f2[HH]}, HU_{d, f2[HU]}, HV_{d, f2[HV]}, DU_{d, f2[DU]},
      DV_{d, f2[DV]}, dry_z{d, f2[DRY_Z]}, dry_u{d, f2[DRY_U]}, dry_v{d, f2[DRY_V]};
  M2 az{d, azp}, au{d, aup}, av{d, avp};
  const double min_depth = par[P_MIN_DEPTH], crit_depth = par[P_CRIT_DEPTH];
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) D(i, j) = z(i, j) + H(i, j);
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO - 1; ++i) {
      double x = std::max(0.25 * (zo(i, j) + zo(i + 1, j) + z(i, j) + z(i + 1, j)), -HU_(i, j) + min_depth);
      DU_(i, j) = x + HU_(i, j);
    }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO - 1; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      double x = std::max(0.25 * (zo(i, j) + zo(i, j + 1) + z(i, j) + z(i, j + 1)), -HV_(i, j) + min_depth);
      DV_(i, j) = x + HV_(i, j);
    }
  const double d1 = 2 * min_depth;
  const double d2i = 1.0 / (crit_depth - 2 * min_depth);
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      if (az(i, j) > 0) dry_z(i, j) = std::max(0.0, std::min(1.0, (D(i, j) - 0.5 * d1) * d2i));
      if (au(i, j) > 0) dry_u(i, j) = std::max(0.0, std::min(1.0, (DU_(i, j) - d1) * d2i));
      if (av(i, j) > 0) dry_v(i, j) = std::max(0.0, std::min(1.0, (DV_(i, j) - d1) * d2i));
    }
}

// sealevel.F90:172-314 (sealevel_nan_check with sealevel_nandum): the number of interior
// elevations z that are not below HUGE(z) -- NaN, +Inf or the largest double -- and the last such
// point in the reference's loop order (j outer, i inner). The reference checks every point of the
// interior, land included.
inline long sealevel_nan_count(const Dom& d, const double* zp, int* inan, int* jnan) {
  A2 z{d, const_cast<double*>(zp)};
  const double ahuge = std::numeric_limits<double>::max();
  long num_nan = 0;
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (!(ahuge > z(i, j))) {
        ++num_nan;
        if (inan) *inan = i;
        if (jnan) *jnan = j;
      }
  return num_nan;
}

// m2d.F90:412-490 integrate_2d (closed boundaries, no residual, no uv_diffusion).
template <class R3>
int integrate_2d(const Dom& d, const AdvMasks& m, BcState<R3>& st, int loop) {
  double** f2 = st.f2;
  const double* par = st.par;
  int* ip = st.ipar;
  if ((loop - 1) % ip[I_MM] == 0) bottom_friction(d, nullptr, f2, st.au, st.av, par, ip[I_RUNTYPE]);
  if (uv_advect_2d(d, m, st.az, st.au, st.av, par[P_DTM], f2[U_], f2[V_], f2[DU], f2[DV], ip[I_VEL2D_SPLIT],
                   ip[I_VEL2D_HOR], f2[UEX], f2[VEX]) != 0)
    return -1;
  // momentum.F90:44-52: SAVEd toggle ufirst (initially .false.)
  if (ip[I_UFIRST2D]) {
    umomentum(d, f2, st.au, st.av, par, st.bdy, st.az);
    vmomentum(d, f2, st.au, st.av, par, st.bdy, st.az);
    ip[I_UFIRST2D] = 0;
  } else {
    vmomentum(d, f2, st.au, st.av, par, st.bdy, st.az);
    umomentum(d, f2, st.au, st.av, par, st.bdy, st.az);
    ip[I_UFIRST2D] = 1;
  }
  if (ip[I_RUNTYPE] > 1) {
    const long n = d.n2d();
    for (long q = 0; q < n; ++q) {
      f2[UINT][q] = f2[UINT][q] + f2[U_][q];
      f2[VINT][q] = f2[VINT][q] + f2[V_][q];
    }
  }
  if (st.bdy && st.bdy->nseg() > 0) update_2d_bdy(d, *st.bdy, f2, par, loop);  // m2d.F90:475
  sealevel(d, f2, st.az, par);
  // sealevel.F90:115-117: the NaN sweep every |sealevel_check| micro steps until the first
  // finding (have_warned); sealevel_check > 0 turns a finding into an error (getm_error)
  const int chk = ip[I_SEALEVEL_CHECK];
  if (chk != 0 && loop % std::abs(chk) == 0 && !ip[I_NAN_WARNED]) {
    if (sealevel_nan_count(d, f2[Z], nullptr, nullptr) > 0) {
      ip[I_NAN_WARNED] = 1;
      if (chk > 0) return -3;
    }
  }
  depth_update(d, f2, st.az, st.au, st.av, par);
  return 0;
}

// ---------------------------------------------------------------------------------------------
// start_macro.F90:54-86
inline void start_macro(const Dom& d, double** f2, const double* par, int M) {
  A2 sseo{d, f2[SSEO]}, ssen{d, f2[SSEN]}, z{d, f2[Z]}, Dn{d, f2[DN]}, H{d, f2[HH]}, ssuo{d, f2[SSUO]},
      ssun{d, f2[SSUN]}, HU_{d, f2[HU]}, Dun{d, f2[DUN]}, ssvo{d, f2[SSVO]}, ssvn{d, f2[SSVN]}, HV_{d, f2[HV]},
      Dvn{d, f2[DVN]};
  const double min_depth = par[P_MIN_DEPTH];
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      sseo(i, j) = ssen(i, j);
      ssen(i, j) = z(i, j);
      Dn(i, j) = ssen(i, j) + H(i, j);
    }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO - 1; ++i) {
      ssuo(i, j) = ssun(i, j);
      ssun(i, j) = 0.25 * (sseo(i, j) + sseo(i + 1, j) + ssen(i, j) + ssen(i + 1, j));
      ssun(i, j) = std::max(ssun(i, j), -HU_(i, j) + min_depth);
      Dun(i, j) = ssun(i, j) + HU_(i, j);
    }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO - 1; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      ssvo(i, j) = ssvn(i, j);
      ssvn(i, j) = 0.25 * (sseo(i, j) + sseo(i, j + 1) + ssen(i, j) + ssen(i, j + 1));
      ssvn(i, j) = std::max(ssvn(i, j), -HV_(i, j) + min_depth);
      Dvn(i, j) = ssvn(i, j) + HV_(i, j);
    }
  const double split = 1.0 / (double)(float)M;
  const long n = d.n2d();
  for (long q = 0; q < n; ++q) {
    f2[UINT][q] = split * f2[UINT][q];
    f2[VINT][q] = split * f2[VINT][q];
  }
}

// bottom_friction_3d.F90:50-130 (kumin = kvmin = 1)
template <class R3>
void bottom_friction_3d(const Dom& d, BcState<R3>& st) {
  double** f2 = st.f2;
  A2 zub{d, f2[ZUB]}, zvb{d, f2[ZVB]}, rru{d, f2[RRU]}, rrv{d, f2[RRV]};
  A3<R3> uu{d, st.f3[UU]}, vv{d, st.f3[VV]}, huo{d, st.f3[HUO]}, hvo{d, st.f3[HVO]}, hun{d, st.f3[HUN]},
      hvn{d, st.f3[HVN]};
  M2 au{d, st.au}, av{d, st.av};
  const double kappa = st.par[P_KAPPA], min_depth = st.par[P_MIN_DEPTH];
  const long n = d.n2d();
  std::vector<double> a_(n, 0.0), b_(n, 0.0), c_(n, 0.0), e_(n, 0.0);
  A2 uuloc{d, a_.data()}, uvloc{d, b_.data()}, vuloc{d, c_.data()}, vvloc{d, e_.data()};
  const int kk = 1;
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) {
      if (au(i, j) >= 1) {
        uuloc(i, j) = (double)uu(i, j, kk) / ((double)huo(i, j, kk));
        uvloc(i, j) = 0.25 * ((double)vv(i, j, kk) / (double)hvo(i, j, kk) + (double)vv(i + 1, j, kk) / (double)hvo(i + 1, j, kk) +
                              (double)vv(i, j - 1, kk) / (double)hvo(i, j - 1, kk) +
                              (double)vv(i + 1, j - 1, kk) / (double)hvo(i + 1, j - 1, kk));
      } else {
        uuloc(i, j) = 0.0;
        uvloc(i, j) = 0.0;
      }
    }
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) {
      if (av(i, j) >= 1) {
        vuloc(i, j) = 0.25 * ((double)uu(i, j, kk) / (double)huo(i, j, kk) + (double)uu(i - 1, j, kk) / (double)huo(i - 1, j, kk) +
                              (double)uu(i, j + 1, kk) / (double)huo(i, j + 1, kk) +
                              (double)uu(i - 1, j + 1, kk) / (double)huo(i - 1, j + 1, kk));
        vvloc(i, j) = (double)vv(i, j, kk) / ((double)hvo(i, j, kk));
      } else {
        vuloc(i, j) = 0.0;
        vvloc(i, j) = 0.0;
      }
    }
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (au(i, j) >= 1) {
        double hh = std::max(min_depth / d.kmax, (double)hun(i, j, kk));
        double r = (zub(i, j) + 0.5 * hh) / zub(i, j);
        r = kappa / std::log(r);
        r = r * r;
        rru(i, j) = r * std::sqrt(uuloc(i, j) * uuloc(i, j) + uvloc(i, j) * uvloc(i, j));
      }
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (av(i, j) >= 1) {
        double hh = std::max(min_depth / d.kmax, (double)hvn(i, j, kk));
        double r = (zvb(i, j) + 0.5 * hh) / zvb(i, j);
        r = kappa / std::log(r);
        r = r * r;
        rrv(i, j) = r * std::sqrt(vuloc(i, j) * vuloc(i, j) + vvloc(i, j) * vvloc(i, j));
      }
}

// ip_blumberg_mellor.F90:71-148
template <class R3>
void ip_blumberg_mellor(const Dom& d, BcState<R3>& st) {
  A3<R3> hn{d, st.f3[HN]}, hun{d, st.f3[HUN]}, hvn{d, st.f3[HVN]}, buoy{d, st.f3[BUOY]}, idpdx{d, st.f3[IDPDX]},
      idpdy{d, st.f3[IDPDY]};
  A2 H{d, st.f2[HH]};
  M2 az{d, st.az}, au{d, st.au}, av{d, st.av};
  const int kmax = d.kmax;
  const R3 dxm1 = R3(1.0 / d.dx), dym1 = R3(1.0 / d.dy);
  std::vector<R3> zz_(d.n3d(), R3(0));
  A3<R3> zz{d, zz_.data()};
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      idpdx(i, j, 0) = R3(0);
      idpdy(i, j, 0) = R3(0);
    }
  for (int j = d.jmin; j <= d.jmax + 1; ++j)
    for (int i = d.imin; i <= d.imax + 1; ++i)
      if (az(i, j) >= 1) {
        zz(i, j, 1) = R3(-H(i, j)) + hn(i, j, 1);
        for (int k = 2; k <= kmax; ++k) zz(i, j, k) = zz(i, j, k - 1) + hn(i, j, k);
      }
  const R3 half = R3(0.5);
#pragma omp parallel for schedule(static)
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (au(i, j) >= 1) {
        R3 grdl = (buoy(i + 1, j, kmax) - buoy(i, j, kmax)) * dxm1;
        R3 buoyl = half * (buoy(i + 1, j, kmax) + buoy(i, j, kmax));
        R3 prgr = grdl * half * hun(i, j, kmax);
        idpdx(i, j, kmax) = hun(i, j, kmax) * prgr;
        for (int k = kmax - 1; k >= 1; --k) {
          R3 grdu = grdl;
          grdl = (buoy(i + 1, j, k) - buoy(i, j, k)) * dxm1;
          R3 buoyu = buoyl;
          buoyl = half * (buoy(i + 1, j, k) + buoy(i, j, k));
          R3 dxz = (zz(i + 1, j, k) - zz(i, j, k)) * dxm1;
          prgr = prgr + half * (grdu + grdl) * half * (hun(i, j, k) + hun(i, j, k + 1)) - dxz * (buoyu - buoyl);
          idpdx(i, j, k) = hun(i, j, k) * prgr;
        }
      }
#pragma omp parallel for schedule(static)
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (av(i, j) >= 1) {
        R3 grdl = (buoy(i, j + 1, kmax) - buoy(i, j, kmax)) * dym1;
        R3 buoyl = half * (buoy(i, j + 1, kmax) + buoy(i, j, kmax));
        R3 prgr = grdl * half * hvn(i, j, kmax);
        idpdy(i, j, kmax) = hvn(i, j, kmax) * prgr;
        for (int k = kmax - 1; k >= 1; --k) {
          R3 grdu = grdl;
          grdl = (buoy(i, j + 1, k) - buoy(i, j, k)) * dym1;
          R3 buoyu = buoyl;
          buoyl = half * (buoy(i, j + 1, k) + buoy(i, j, k));
          R3 dyz = (zz(i, j + 1, k) - zz(i, j, k)) * dym1;
          prgr = prgr + half * (grdu + grdl) * half * (hvn(i, j, k) + hvn(i, j, k + 1)) - dyz * (buoyu - buoyl);
          idpdy(i, j, k) = hvn(i, j, k) * prgr;
        }
      }
}

// ip_blumberg_mellor_lin.F90:71-161: heights of the pressure points (layer centres), then per U
// and V column a downward integral of the along-sigma buoyancy gradient corrected by the slope of
// the pressure points times the mean vertical buoyancy gradient of the two columns. The lower
// bound kumin_pmz / kvmin_pmz is 1: the only value the reference assigns (adaptive_coordinates.F90:
// 237-238); with sigma coordinates it leaves the arrays unset. The V column starts its integral with
// hun(kmax) (ip_blumberg_mellor_lin.F90:143), as the reference does; the levels below use hvn.
template <class R3>
void ip_blumberg_mellor_lin(const Dom& d, BcState<R3>& st) {
  A3<R3> hn{d, st.f3[HN]}, hun{d, st.f3[HUN]}, hvn{d, st.f3[HVN]}, buoy{d, st.f3[BUOY]}, idpdx{d, st.f3[IDPDX]},
      idpdy{d, st.f3[IDPDY]};
  A2 H{d, st.f2[HH]};
  M2 az{d, st.az}, au{d, st.au}, av{d, st.av};
  const int kmax = d.kmax;
  const R3 dxm1 = R3(1.0 / d.dx), dym1 = R3(1.0 / d.dy);
  const R3 half = R3(0.5);
  std::vector<R3> zz_(d.n3d(), R3(0));
  A3<R3> zz{d, zz_.data()};
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      idpdx(i, j, 0) = R3(0);
      idpdy(i, j, 0) = R3(0);
    }
  for (int j = d.jmin; j <= d.jmax + 1; ++j)
    for (int i = d.imin; i <= d.imax + 1; ++i)
      if (az(i, j) >= 1) {
        zz(i, j, 1) = R3(-H(i, j)) + half * hn(i, j, 1);
        for (int k = 2; k <= kmax; ++k) zz(i, j, k) = zz(i, j, k - 1) + half * (hn(i, j, k - 1) + hn(i, j, k));
      }
  // one column; (oi, oj) = the neighbour across the face, hx = the face's layer heights, h0 = the
  // height that starts the integral, dm1 = 1/dx or 1/dy
  auto column = [&](int i, int j, int oi, int oj, A3<R3>& hx, R3 h0, A3<R3>& out, R3 dm1) {
    R3 dzl = (zz(i + oi, j + oj, kmax) - zz(i, j, kmax)) * dm1;
    R3 drl = (buoy(i + oi, j + oj, kmax) - buoy(i, j, kmax)) * dm1;
    R3 prgr = drl * half * h0;
    out(i, j, kmax) = hx(i, j, kmax) * prgr;
    for (int k = kmax - 1; k >= 1; --k) {
      const R3 dzu = dzl;
      dzl = (zz(i + oi, j + oj, k) - zz(i, j, k)) * dm1;
      const R3 dru = drl;
      drl = (buoy(i + oi, j + oj, k) - buoy(i, j, k)) * dm1;
      const R3 dzr2 = (buoy(i + oi, j + oj, k + 1) - buoy(i + oi, j + oj, k)) /
                      (zz(i + oi, j + oj, k + 1) - zz(i + oi, j + oj, k));
      const R3 dzr1 = (buoy(i, j, k + 1) - buoy(i, j, k)) / (zz(i, j, k + 1) - zz(i, j, k));
      const R3 aa = half * (drl + dru);
      const R3 bb = half * (dzl + dzu);
      const R3 cc = half * (dzr2 + dzr1);
      prgr = prgr + (aa - bb * cc) * half * (hx(i, j, k + 1) + hx(i, j, k));
      out(i, j, k) = hx(i, j, k) * prgr;
    }
  };
#pragma omp parallel for schedule(static)
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (au(i, j) >= 1) column(i, j, 1, 0, hun, hun(i, j, kmax), idpdx, dxm1);
#pragma omp parallel for schedule(static)
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (av(i, j) >= 1) column(i, j, 0, 1, hvn, hun(i, j, kmax), idpdy, dym1);
}

// Heights of the layer interfaces (centres = false, ip_blumberg_mellor.F90:81-90, ip_chu_fan.F90)
// or of the pressure points (centres = true, ip_blumberg_mellor_lin.F90:87-97, ip_song_wright.F90)
// of the columns i = imin..imax+1, j = jmin..jmax+1 with az >= 1; zero elsewhere.
template <class R3>
std::vector<R3> ip_heights(const Dom& d, BcState<R3>& st, bool centres) {
  A3<R3> hn{d, st.f3[HN]};
  A2 H{d, st.f2[HH]};
  M2 az{d, st.az};
  const R3 half = R3(0.5);
  std::vector<R3> zz_(d.n3d(), R3(0));
  A3<R3> zz{d, zz_.data()};
  for (int j = d.jmin; j <= d.jmax + 1; ++j)
    for (int i = d.imin; i <= d.imax + 1; ++i)
      if (az(i, j) >= 1) {
        if (centres) {
          zz(i, j, 1) = R3(-H(i, j)) + half * hn(i, j, 1);
          for (int k = 2; k <= d.kmax; ++k) zz(i, j, k) = zz(i, j, k - 1) + half * (hn(i, j, k - 1) + hn(i, j, k));
        } else {
          zz(i, j, 1) = R3(-H(i, j)) + hn(i, j, 1);
          for (int k = 2; k <= d.kmax; ++k) zz(i, j, k) = zz(i, j, k - 1) + hn(i, j, k);
        }
      }
  return zz_;
}

// ip_z_interpol.F90:61-168: pressure-point heights; per U (then V) column, downward from kmax-1,
// the neighbour buoyancies at the face's own pressure-point height zx(k), each found by a search
// from the top for the first neighbour level at or below zx(k) and interpolated between it and the
// level above. Where the search ends at level 1 or finds none, the reference keeps the value of
// the previous level -- or, at a column's first level, of the previous column in loop order (j
// outer, i inner, all U columns before all V columns) -- and 0 before any assignment (the
// reference's locals are unset there; executed from source they start at 0). That carried state
// makes the routine sequential in the loop order; it is restated here exactly so.
template <class R3>
void ip_z_interpol(const Dom& d, BcState<R3>& st) {
  A3<R3> hn{d, st.f3[HN]}, hun{d, st.f3[HUN]}, hvn{d, st.f3[HVN]}, buoy{d, st.f3[BUOY]}, idpdx{d, st.f3[IDPDX]},
      idpdy{d, st.f3[IDPDY]};
  A2 H{d, st.f2[HH]}, HU_{d, st.f2[HU]}, HV_{d, st.f2[HV]};
  M2 au{d, st.au}, av{d, st.av};
  const int kmax = d.kmax;
  const R3 dxm1 = R3(1.0 / d.dx), dym1 = R3(1.0 / d.dy), half = R3(0.5);
  std::vector<R3> zz_ = ip_heights(d, st, true);
  A3<R3> zz{d, zz_.data()};
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      idpdx(i, j, 0) = R3(0);
      idpdy(i, j, 0) = R3(0);
    }
  std::vector<R3> zx(kmax + 1);
  R3 buoyplus = R3(0), buoyminus = R3(0);
  // di, dj: the neighbour's offset; hx: hun or hvn; Hx: HU or HV; out: idpdx or idpdy
  auto column = [&](int i, int j, int di, int dj, A3<R3>& hx, A2& Hx, A3<R3>& out, R3 dm1) {
    zx[1] = R3(-Hx(i, j)) + half * hx(i, j, 1);
    for (int k = 2; k <= kmax; ++k) zx[k] = zx[k - 1] + half * (hx(i, j, k - 1) + hx(i, j, k));
    R3 grdl = half * hx(i, j, kmax) * (buoy(i + di, j + dj, kmax) - buoy(i, j, kmax)) * dm1;
    R3 prgr = grdl;
    out(i, j, kmax) = hx(i, j, kmax) * prgr;
    for (int k = kmax - 1; k >= 1; --k) {
      const R3 grdu = grdl;
      int kplus = kmax;
      for (; kplus >= 1; --kplus)
        if (zz(i + di, j + dj, kplus) <= zx[k]) break;
      int kminus = kmax;
      for (; kminus >= 1; --kminus)
        if (zz(i, j, kminus) <= zx[k]) break;
      if (kplus == kmax) buoyplus = buoy(i + di, j + dj, kplus);
      if (kplus < kmax && kplus > 1)
        buoyplus = ((zx[k] - zz(i + di, j + dj, kplus)) * buoy(i + di, j + dj, kplus + 1) +
                    (zz(i + di, j + dj, kplus + 1) - zx[k]) * buoy(i + di, j + dj, kplus)) /
                   (half * (hn(i + di, j + dj, kplus + 1) + hn(i + di, j + dj, kplus)));
      if (kminus == kmax) buoyminus = buoy(i, j, kminus);
      if (kminus < kmax && kminus > 1)
        buoyminus = ((zx[k] - zz(i, j, kminus)) * buoy(i, j, kminus + 1) +
                     (zz(i, j, kminus + 1) - zx[k]) * buoy(i, j, kminus)) /
                    (half * (hn(i, j, kminus + 1) + hn(i, j, kminus)));
      if (zx[k] > std::max(R3(-H(i + di, j + dj)), R3(-H(i, j))))
        grdl = half * hx(i, j, k) * (buoyplus - buoyminus) * dm1;
      else
        grdl = R3(0);
      prgr = prgr + grdu + grdl;
      out(i, j, k) = hx(i, j, k) * prgr;
    }
  };
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (au(i, j) >= 1) column(i, j, 1, 0, hun, HU_, idpdx, dxm1);
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (av(i, j) >= 1) column(i, j, 0, 1, hvn, HV_, idpdy, dym1);
}

// ip_stelling_vankester.F90:56-398: per U (then V) column the interface heights of both columns
// and the face's surface are merged into one sorted list zl (the reference's exchange sort); each
// interval of zl contributes its height times a limited buoyancy difference (the smaller of the two
// one-sided differences of the interpolated neighbour buoyancies, 0 where they differ in sign),
// and each level k takes the integral down to its pressure point zx(k). The work arrays lvel and
// dzfrac keep their values from the previous column wherever the interval loop does not reach a
// level; db is reset per U column but not per V column (the reference's V loop has no reset), and
// its V form takes max(dcn, dcm) when dcn = 0 where the U form takes min. Work arrays and db start
// at 0 (executed from source, the reference's locals do).
template <class R3>
void ip_stelling_vankester(const Dom& d, BcState<R3>& st) {
  A3<R3> hn{d, st.f3[HN]}, hun{d, st.f3[HUN]}, hvn{d, st.f3[HVN]}, buoy{d, st.f3[BUOY]}, idpdx{d, st.f3[IDPDX]},
      idpdy{d, st.f3[IDPDY]};
  A2 H{d, st.f2[HH]}, HU_{d, st.f2[HU]}, HV_{d, st.f2[HV]}, ssun{d, st.f2[SSUN]}, ssvn{d, st.f2[SSVN]};
  M2 az{d, st.az}, au{d, st.au}, av{d, st.av};
  const int kmax = d.kmax, lnum = 2 * kmax + 1;
  const R3 dxm1 = R3(1.0 / d.dx), dym1 = R3(1.0 / d.dy), half = R3(0.5);
  std::vector<R3> zz_ = ip_heights(d, st, true), zi_(d.n3d(), R3(0));
  A3<R3> zz{d, zz_.data()}, zi{d, zi_.data()};
  for (int j = d.jmin; j <= d.jmax + 1; ++j)
    for (int i = d.imin; i <= d.imax + 1; ++i)
      if (az(i, j) >= 1) {
        zi(i, j, 1) = R3(-H(i, j));
        for (int k = 2; k <= kmax; ++k) zi(i, j, k) = zi(i, j, k - 1) + hn(i, j, k - 1);
      }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      idpdx(i, j, 0) = R3(0);
      idpdy(i, j, 0) = R3(0);
    }
  std::vector<R3> zx(kmax + 1), zl(lnum + 1), dzl(lnum + 1), dzfrac(kmax + 1, R3(0));
  std::vector<int> lvel(kmax + 2, 0), m(lnum + 1), n(lnum + 1);
  R3 db = R3(0);
  auto column = [&](int i, int j, int di, int dj, A3<R3>& hx, A2& Hx, A2& ssx, A3<R3>& out, R3 dm1, bool vform) {
    const int i1 = i + di, j1 = j + dj;
    zx[1] = R3(-Hx(i, j)) + half * hx(i, j, 1);
    zl[1] = zi(i, j, 1);
    zl[2] = zi(i1, j1, 1);
    for (int k = 2; k <= kmax; ++k) {
      zx[k] = zx[k - 1] + half * (hx(i, j, k - 1) + hx(i, j, k));
      zl[2 * k - 1] = zi(i, j, k);
      zl[2 * k] = zi(i1, j1, k);
    }
    zl[lnum] = R3(ssx(i, j));
    for (bool changed = true; changed;) {
      changed = false;
      for (int l = 1; l <= lnum - 1; ++l)
        if (zl[l] > zl[l + 1]) {
          std::swap(zl[l], zl[l + 1]);
          changed = true;
        }
    }
    m[lnum] = kmax;
    n[lnum] = kmax;
    int kcount = kmax;
    lvel[kmax + 1] = lnum;
    for (int l = lnum - 1; l >= 1; --l) {
      dzl[l] = zl[l + 1] - zl[l];
      m[l] = m[l + 1];
      n[l] = n[l + 1];
      if (zl[l + 1] <= zi(i, j, m[l])) m[l] = std::max(1, m[l] - 1);
      if (zl[l + 1] <= zi(i1, j1, n[l])) n[l] = std::max(1, n[l] - 1);
      if (kcount > 0 && zx[kcount] > zl[l]) {
        lvel[kcount] = l;
        dzfrac[kcount] = zx[kcount] - zl[l];
        --kcount;
      }
    }
    R3 prgr = R3(0);
    if (!vform) db = R3(0);
    for (int k = kmax; k >= 1; --k) {
      for (int l = lvel[k + 1] - 1; l >= lvel[k]; --l) {
        const R3 zn = zz(i1, j1, n[l]), zm = zz(i, j, m[l]);
        R3 buoyminus, buoyplus;
        if (zn >= zz(i, j, kmax)) buoyminus = buoy(i, j, kmax);
        else if (zn <= zz(i, j, 1)) buoyminus = buoy(i, j, 1);
        else {
          const int klower = zn >= zm ? m[l] : m[l] - 1, kupper = zn >= zm ? m[l] + 1 : m[l];
          const R3 dzz = zz(i, j, kupper) - zz(i, j, klower);
          buoyminus = (zn - zz(i, j, klower)) / dzz * buoy(i, j, kupper) + (zz(i, j, kupper) - zn) / dzz * buoy(i, j, klower);
        }
        if (zm >= zz(i1, j1, kmax)) buoyplus = buoy(i1, j1, kmax);
        else if (zm <= zz(i1, j1, 1)) buoyplus = buoy(i1, j1, 1);
        else {
          const int klower = zm >= zn ? n[l] : n[l] - 1, kupper = zm >= zn ? n[l] + 1 : n[l];
          const R3 dzz = zz(i1, j1, kupper) - zz(i1, j1, klower);
          buoyplus = (zm - zz(i1, j1, klower)) / dzz * buoy(i1, j1, kupper) + (zz(i1, j1, kupper) - zm) / dzz * buoy(i1, j1, klower);
        }
        const R3 dcm = buoy(i1, j1, n[l]) - buoyminus;
        const R3 dcn = buoyplus - buoy(i, j, m[l]);
        if (dcn * dcm < R3(0)) db = R3(0);
        else if (!vform) db = dcn >= R3(0) ? std::min(dcn, dcm) : std::max(dcn, dcm);
        else {
          if (dcn >= R3(0)) db = std::min(dcn, dcm);
          if (dcn <= R3(0)) db = std::max(dcn, dcm);
        }
        prgr = prgr + dzl[l] * db * dm1;
      }
      out(i, j, k) = hx(i, j, k) * (prgr - dzfrac[k] * db * dm1);
    }
  };
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (au(i, j) >= 1) column(i, j, 1, 0, hun, HU_, ssun, idpdx, dxm1, false);
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (av(i, j) >= 1) column(i, j, 0, 1, hvn, HV_, ssvn, idpdy, dym1, true);
}

// ip_song_wright.F90:86-150: pressure-point heights; per column the gradient of the layer-mean
// buoyancy times the layer-mean height, less the change of the mean buoyancy times the slope of the
// pressure points. The V column's first slope term is scaled by 1/dx (ip_song_wright.F90:128), as
// in the reference.
template <class R3>
void ip_song_wright(const Dom& d, BcState<R3>& st) {
  A3<R3> hn{d, st.f3[HN]}, hun{d, st.f3[HUN]}, hvn{d, st.f3[HVN]}, buoy{d, st.f3[BUOY]}, idpdx{d, st.f3[IDPDX]},
      idpdy{d, st.f3[IDPDY]};
  M2 au{d, st.au}, av{d, st.av};
  const int kmax = d.kmax;
  const R3 dxm1 = R3(1.0 / d.dx), dym1 = R3(1.0 / d.dy), half = R3(0.5);
  std::vector<R3> zz_ = ip_heights(d, st, true);
  A3<R3> zz{d, zz_.data()};
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      idpdx(i, j, 0) = R3(0);
      idpdy(i, j, 0) = R3(0);
    }
  auto column = [&](int i, int j, int oi, int oj, A3<R3>& hx, A3<R3>& out, R3 dm1, R3 dm1top) {
    const int i1 = i + oi, j1 = j + oj;
    R3 grdl = half * hx(i, j, kmax) * (buoy(i1, j1, kmax) - buoy(i, j, kmax)) * dm1;
    R3 buoyl = half * (buoy(i1, j1, kmax) + buoy(i, j, kmax)) * (zz(i1, j1, kmax) - zz(i, j, kmax)) * dm1top;
    R3 prgr = grdl;
    out(i, j, kmax) = hx(i, j, kmax) * prgr;
    for (int k = kmax - 1; k >= 1; --k) {
      grdl = (half * (buoy(i1, j1, k) + buoy(i1, j1, k + 1)) * half * (hn(i1, j1, k) + hn(i1, j1, k + 1)) -
              half * (buoy(i, j, k) + buoy(i, j, k + 1)) * half * (hn(i, j, k) + hn(i, j, k + 1))) *
             dm1;
      const R3 buoyu = buoyl;
      buoyl = half * (buoy(i1, j1, k) + buoy(i, j, k)) * (zz(i1, j1, k) - zz(i, j, k)) * dm1;
      prgr = prgr + grdl - (buoyu - buoyl);
      out(i, j, k) = hx(i, j, k) * prgr;
    }
  };
#pragma omp parallel for schedule(static)
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (au(i, j) >= 1) column(i, j, 1, 0, hun, idpdx, dxm1, dxm1);
#pragma omp parallel for schedule(static)
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (av(i, j) >= 1) column(i, j, 0, 1, hvn, idpdy, dym1, dxm1);
}

// ip_chu_fan.F90:67-126: interface heights; the Blumberg-Mellor integral with a correction hc
// from the squared height differences of the four corners of each interface cell. The integral
// starts from the top gradient itself and the top level's term is hx*grad*hx/2, as in the reference.
template <class R3>
void ip_chu_fan(const Dom& d, BcState<R3>& st) {
  A3<R3> hun{d, st.f3[HUN]}, hvn{d, st.f3[HVN]}, buoy{d, st.f3[BUOY]}, idpdx{d, st.f3[IDPDX]},
      idpdy{d, st.f3[IDPDY]};
  M2 au{d, st.au}, av{d, st.av};
  const int kmax = d.kmax;
  const R3 dxm1 = R3(1.0 / d.dx), dym1 = R3(1.0 / d.dy), half = R3(0.5), sixth = R3(1.0 / 6);
  std::vector<R3> zz_ = ip_heights(d, st, false);
  A3<R3> zz{d, zz_.data()};
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      idpdx(i, j, 0) = R3(0);
      idpdy(i, j, 0) = R3(0);
    }
  auto column = [&](int i, int j, int oi, int oj, A3<R3>& hx, A3<R3>& out, R3 dm1) {
    const int i1 = i + oi, j1 = j + oj;
    R3 grdl = (buoy(i1, j1, kmax) - buoy(i, j, kmax)) * dm1;
    R3 buoyl = half * (buoy(i1, j1, kmax) + buoy(i, j, kmax));
    R3 prgr = grdl;
    out(i, j, kmax) = hx(i, j, kmax) * prgr * half * hx(i, j, kmax);
    for (int k = kmax - 1; k >= 1; --k) {
      const R3 grdu = grdl;
      grdl = (buoy(i1, j1, k) - buoy(i, j, k)) * dm1;
      const R3 buoyu = buoyl;
      buoyl = half * (buoy(i1, j1, k) + buoy(i, j, k));
      const R3 dz = (zz(i1, j1, k) - zz(i, j, k)) * dm1;
      const R3 a = zz(i1, j1, k) - zz(i1, j1, k + 1), b = zz(i, j, k) - zz(i, j, k + 1);
      const R3 c = zz(i1, j1, k + 1) - zz(i, j, k + 1), e = zz(i1, j1, k) - zz(i, j, k);
      R3 hc = a * a * (buoy(i1, j1, k) - buoy(i1, j1, k + 1));
      hc = hc - b * b * (buoy(i, j, k) - buoy(i, j, k + 1));
      hc = hc + c * c * (buoy(i1, j1, k + 1) - buoy(i, j, k + 1));
      hc = hc - e * e * (buoy(i1, j1, k) - buoy(i, j, k));
      hc = hc * dm1 * sixth / (zz(i, j, k) + zz(i1, j1, k) - zz(i, j, k + 1) - zz(i1, j1, k + 1));
      prgr = prgr + (grdu + grdl + hc) * half * (hx(i, j, k) + hx(i, j, k + 1)) - dz * (buoyu - buoyl);
      out(i, j, k) = hx(i, j, k) * prgr;
    }
  };
#pragma omp parallel for schedule(static)
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (au(i, j) >= 1) column(i, j, 1, 0, hun, idpdx, dxm1);
#pragma omp parallel for schedule(static)
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (av(i, j) >= 1) column(i, j, 0, 1, hvn, idpdy, dym1);
}

// ip_shchepetkin_mcwilliams.F90:61-262: pressure-point heights over the whole haloed domain; per
// column a pressure integral P with harmonic-mean vertical differences of buoyancy and height; per
// level the along-level pressure difference from P plus a horizontal flux term FC with
// harmonic-mean horizontal differences, less the elevation-slope term. Constants as the reference
// evaluates them: eps = 1.e-10 and OneFifth = 0.2 are single-precision literals widened to double,
// 1./12. a single-precision quotient (the factor t below).
template <class R3>
void ip_shchepetkin_mcwilliams(const Dom& d, BcState<R3>& st) {
  A3<R3> hn{d, st.f3[HN]}, hun{d, st.f3[HUN]}, hvn{d, st.f3[HVN]}, buoy{d, st.f3[BUOY]}, idpdx{d, st.f3[IDPDX]},
      idpdy{d, st.f3[IDPDY]};
  A2 H{d, st.f2[HH]}, sseo{d, st.f2[SSEO]};
  M2 az{d, st.az}, au{d, st.au}, av{d, st.av};
  const int kmax = d.kmax;
  const R3 dxm1 = R3(1.0 / d.dx), dym1 = R3(1.0 / d.dy), half = R3(0.5), two = R3(2.0), one = R3(1.0);
  const R3 eps = R3(double(1.e-10f)), fifth = R3(double(0.2f)), t = R3(double(1.0f / 12.0f));
  std::vector<R3> zz_(d.n3d(), R3(0)), P_(d.n3d(), R3(0));
  A3<R3> zz{d, zz_.data()}, P{d, P_.data()};
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i)
      if (az(i, j) >= 1) {
        zz(i, j, 1) = R3(-H(i, j)) + half * hn(i, j, 1);
        for (int k = 2; k <= kmax; ++k) zz(i, j, k) = zz(i, j, k - 1) + half * (hn(i, j, k - 1) + hn(i, j, k));
      }
  std::vector<R3> dR(kmax + 1), dZ(kmax + 1);
  for (int j = d.jmin; j <= d.jmax + 1; ++j)
    for (int i = d.imin; i <= d.imax + 1; ++i)
      if (az(i, j) >= 1) {
        for (int k = 1; k <= kmax - 1; ++k) {
          dR[k] = buoy(i, j, k + 1) - buoy(i, j, k);
          dZ[k] = zz(i, j, k + 1) - zz(i, j, k);
        }
        dR[kmax] = dR[kmax - 1];
        dZ[kmax] = dZ[kmax - 1];
        dR[0] = dR[1];
        dZ[0] = dZ[1];
        for (int k = kmax; k >= 1; --k) {
          const R3 cff = two * dR[k] * dR[k - 1];
          dR[k] = cff > eps ? cff / (dR[k] + dR[k - 1]) : R3(0);
          dZ[k] = two * dZ[k] * dZ[k - 1] / (dZ[k] + dZ[k - 1]);
        }
        const R3 cff1 = one / (zz(i, j, kmax) - zz(i, j, kmax - 1));
        const R3 cff2 = half * (buoy(i, j, kmax) - buoy(i, j, kmax - 1)) * half * hn(i, j, kmax) * cff1;
        P(i, j, kmax) = (buoy(i, j, kmax) + cff2) * half * hn(i, j, kmax);
        for (int k = kmax - 1; k >= 1; --k)
          P(i, j, k) = P(i, j, k + 1) +
                       half * ((buoy(i, j, k + 1) + buoy(i, j, k)) * (zz(i, j, k + 1) - zz(i, j, k)) -
                               fifth * ((dR[k + 1] - dR[k]) * (zz(i, j, k + 1) - zz(i, j, k) - t * (dZ[k + 1] + dZ[k])) -
                                        (dZ[k + 1] - dZ[k]) * (buoy(i, j, k + 1) - buoy(i, j, k) - t * (dR[k + 1] + dR[k]))));
      }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      idpdx(i, j, 0) = R3(0);
      idpdy(i, j, 0) = R3(0);
    }
  // harmonic mean of two neighbouring differences (ip_shchepetkin_mcwilliams.F90:172-186)
  auto harm = [&](R3 a, R3 b) {
    const R3 cff = two * a * b;
    return cff > eps ? cff * (one / (a + b)) : R3(0);
  };
  // one face at level k: columns c0 (i, j) and c1 (i+oi, j+oj), the differences to the columns
  // before c0 and after c1 along the direction
  auto face = [&](int i, int j, int oi, int oj, int k, A3<R3>& hx, R3 dm1) {
    const int im = i - oi, jm = j - oj, i1 = i + oi, j1 = j + oj, i2 = i + 2 * oi, j2 = j + 2 * oj;
    const R3 z0 = zz(i, j, k) - zz(im, jm, k), z1 = zz(i1, j1, k) - zz(i, j, k), z2 = zz(i2, j2, k) - zz(i1, j1, k);
    const R3 r0 = buoy(i, j, k) - buoy(im, jm, k), r1 = buoy(i1, j1, k) - buoy(i, j, k),
             r2 = buoy(i2, j2, k) - buoy(i1, j1, k);
    const R3 dZx0 = harm(z0, z1), dZx1 = harm(z1, z2), dRx0 = harm(r0, r1), dRx1 = harm(r1, r2);
    R3 AJ = P(i1, j1, k) - P(i, j, k);
    const R3 FC = half * ((buoy(i1, j1, k) + buoy(i, j, k)) * (zz(i1, j1, k) - zz(i, j, k)) -
                          fifth * ((dRx1 - dRx0) * (zz(i1, j1, k) - zz(i, j, k) - t * (dZx1 + dZx0)) -
                                   (dZx1 - dZx0) * (buoy(i1, j1, k) - buoy(i, j, k) - t * (dRx1 + dRx0))));
    AJ = AJ + FC;
    return AJ * dm1 * hx(i, j, k) -
           hx(i, j, k) * dm1 * R3(sseo(i1, j1) - sseo(i, j)) * half * (buoy(i1, j1, kmax) + buoy(i, j, kmax));
  };
#pragma omp parallel for schedule(static)
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) {
      if (au(i, j) >= 1)
        for (int k = kmax; k >= 1; --k) idpdx(i, j, k) = face(i, j, 1, 0, k, hun, dxm1);
      if (av(i, j) >= 1)
        for (int k = kmax; k >= 1; --k) idpdy(i, j, k) = face(i, j, 0, 1, k, hvn, dym1);
    }
}

// internal_pressure.F90:204-233: the configured method; nonzero for a method not provided here
template <class R3>
int do_internal_pressure(const Dom& d, BcState<R3>& st) {
  switch (st.ipar[I_IP_METHOD]) {
    case 1: ip_blumberg_mellor(d, st); return 0;
    case 2: ip_blumberg_mellor_lin(d, st); return 0;
    case 3: ip_z_interpol(d, st); return 0;
    case 4: ip_song_wright(d, st); return 0;
    case 5: ip_chu_fan(d, st); return 0;
    case 6: ip_shchepetkin_mcwilliams(d, st); return 0;
    case 7: ip_stelling_vankester(d, st); return 0;
    default: return -1;
  }
}

// uu_momentum_3d.F90:169-337 / vv_momentum_3d.F90:174-340 (kumin = kvmin = 1). dir 0 = uu.
template <class R3>
void uv_momentum_3d(const Dom& d, BcState<R3>& st, int dir) {
  double** f2 = st.f2;
  const double* par = st.par;
  const int kmax = d.kmax;
  A3<R3> uu{d, st.f3[dir == 0 ? UU : VV]}, vv{d, st.f3[dir == 0 ? VV : UU]};
  A3<R3> ho_{d, st.f3[dir == 0 ? HUO : HVO]}, hn_{d, st.f3[dir == 0 ? HUN : HVN]};
  A3<R3> Ex{d, st.f3[dir == 0 ? UUEX : VVEX]}, idp{d, st.f3[dir == 0 ? IDPDX : IDPDY]}, num{d, st.f3[NUM]};
  A2 dry{d, f2[dir == 0 ? DRY_U : DRY_V]}, cor{d, f2[dir == 0 ? CORU : CORV]}, taus{d, f2[dir == 0 ? TAUSX : TAUSY]},
      sseo{d, f2[SSEO]}, H{d, f2[HH]}, D{d, f2[D_]}, airp{d, f2[AIRP]}, rr{d, f2[dir == 0 ? RRU : RRV]},
      Uint{d, f2[dir == 0 ? UINT : VINT]}, sso{d, f2[dir == 0 ? SSUO : SSVO]}, HX{d, f2[dir == 0 ? HU : HV]};
  M2 mask{d, dir == 0 ? st.au : st.av};
  const double g = par[P_G], rho_0 = par[P_RHO_0], dt = par[P_DT], cnpar = par[P_CNPAR], avmmol = par[P_AVMMOL],
               min_depth = par[P_MIN_DEPTH], ip_fac = par[P_IP_FAC];
  const double gamma = g * rho_0;
  const double gammai = 1.0 / gamma, rho_0i = 1.0 / rho_0;
  const int di = dir == 0 ? 1 : 0, dj = dir == 0 ? 0 : 1;
  const double dxy = dir == 0 ? d.dx : d.dy;
#pragma omp parallel for schedule(static)
  for (int j = d.jmin; j <= d.jmax; ++j) {
    std::vector<double> dif(kmax + 1), auxn(kmax + 1), auxo(kmax + 1), a1(kmax + 1), a2(kmax + 1),
        a3(kmax + 1), a4(kmax + 1), Res(kmax + 1), ex(kmax + 1);
    for (int i = d.imin; i <= d.imax; ++i) {
      if (!(mask(i, j) == 1 || mask(i, j) == 2)) continue;
      const int kmn = 1;
      if (kmax > kmn) {
        for (int k = kmn; k <= kmax; ++k) {
          double loc, e;
          if (dir == 0) {
            loc = 0.25 * ((double)vv(i, j, k) + (double)vv(i + 1, j, k) + (double)vv(i, j - 1, k) + (double)vv(i + 1, j - 1, k));
            e = cor(i, j) * loc;
          } else {
            loc = 0.25 * ((double)vv(i, j, k) + (double)vv(i - 1, j, k) + (double)vv(i, j + 1, k) + (double)vv(i - 1, j + 1, k));
            e = -cor(i, j) * loc;
          }
          ex[k] = dry(i, j) * (e - (double)Ex(i, j, k) + ip_fac * (double)idp(i, j, k));
        }
        ex[kmax] = ex[kmax] + dry(i, j) * 0.5 * (taus(i, j) + taus(i + di, j + dj)) * rho_0i;
        for (int k = kmn; k <= kmax - 1; ++k) dif[k] = 0.5 * ((double)num(i, j, k) + (double)num(i + di, j + dj, k)) + avmmol;
        for (int k = kmn; k <= kmax - 1; ++k) {
          auxo[k] = 2.0 * (1.0 - cnpar) * dt * dif[k] / ((double)ho_(i, j, k + 1) + (double)ho_(i, j, k));
          auxn[k] = 2.0 * cnpar * dt * dif[k] / ((double)hn_(i, j, k + 1) + (double)hn_(i, j, k));
        }
        double zp = std::max(sseo(i + di, j + dj), -H(i, j) + std::min(min_depth, D(i + di, j + dj)));
        double zm = std::max(sseo(i, j), -H(i + di, j + dj) + std::min(min_depth, D(i, j)));
        double zx;
        if (dir == 0)
          zx = (zp - zm + (airp(i + 1, j) - airp(i, j)) * gammai) / dxy;
        else
          zx = (zp - zm + (airp(i, j + 1) - airp(i, j)) / gamma) / dxy;
        auto HOd = [&](int k) { return (double)ho_(i, j, k); };
        auto HNd = [&](int k) { return (double)hn_(i, j, k); };
        auto UUd = [&](int k) { return (double)uu(i, j, k); };
        int k = kmax;
        a1[k] = -auxn[k - 1] / HNd(k - 1);
        a2[k] = 1. + auxn[k - 1] / HNd(k);
        a4[k] = UUd(k) * (1 - auxo[k - 1] / HOd(k)) + UUd(k - 1) * auxo[k - 1] / HOd(k - 1) + dt * ex[k] -
                dt * 0.5 * (HOd(k) + HNd(k)) * g * zx;
        for (k = kmn + 1; k <= kmax - 1; ++k) {
          a3[k] = -auxn[k] / HNd(k + 1);
          a1[k] = -auxn[k - 1] / HNd(k - 1);
          a2[k] = 1.0 + (auxn[k] + auxn[k - 1]) / HNd(k);
          a4[k] = UUd(k + 1) * auxo[k] / HOd(k + 1) + UUd(k) * (1 - (auxo[k] + auxo[k - 1]) / HOd(k)) +
                  UUd(k - 1) * auxo[k - 1] / HOd(k - 1) + dt * ex[k] - dt * 0.5 * (HOd(k) + HNd(k)) * g * zx;
        }
        k = kmn;
        a3[k] = -auxn[k] / HNd(k + 1);
        a2[k] = 1.0 + auxn[k] / HNd(k) + dt * rr(i, j) / (0.5 * (HNd(k) + HOd(k)));
        a4[k] = UUd(k + 1) * auxo[k] / HOd(k + 1) + UUd(k) * (1 - auxo[k] / HOd(k)) + dt * ex[k] -
                dt * 0.5 * (HOd(k) + HNd(k)) * g * zx;
        getm_tridiagonal<double>(kmax, kmn, kmax, a1.data(), a2.data(), a3.data(), a4.data(), Res.data());
        double ResInt = 0.0;
        for (k = kmn; k <= kmax; ++k) ResInt = ResInt + Res[k];
        double Diff = (Uint(i, j) - ResInt) / (sso(i, j) + HX(i, j));
        for (k = kmn; k <= kmax; ++k) uu(i, j, k) = R3(Res[k] + HNd(k) * Diff);
      } else {
        uu(i, j, kmax) = R3(Uint(i, j));
      }
    }
  }
  // uu_momentum_3d.F90:389 / vv_momentum_3d.F90:400
  if (st.bdy) mirror_bdy<R3>(d, *st.bdy, st.az, st.au, st.av, st.f3[dir == 0 ? UU : VV], dir, kmax + 1, d.sk);
}

// sigma_coordinates.F90:85-113 (equidistant), all levels 0..kmax
template <class R3>
void sigma_coordinates(const Dom& d, BcState<R3>& st) {
  double** f2 = st.f2;
  A2 sseo{d, f2[SSEO]}, ssen{d, f2[SSEN]}, H{d, f2[HH]}, ssuo{d, f2[SSUO]}, ssun{d, f2[SSUN]}, HU_{d, f2[HU]},
      ssvo{d, f2[SSVO]}, ssvn{d, f2[SSVN]}, HV_{d, f2[HV]};
  A3<R3> ho{d, st.f3[HO]}, hn{d, st.f3[HN]}, huo{d, st.f3[HUO]}, hun{d, st.f3[HUN]}, hvo{d, st.f3[HVO]},
      hvn{d, st.f3[HVN]};
  const double kmaxm1 = 1.0 / (double)(float)d.kmax;
#pragma omp parallel for schedule(static)
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      const R3 a = R3((sseo(i, j) + H(i, j)) * kmaxm1), b = R3((ssen(i, j) + H(i, j)) * kmaxm1);
      for (int k = 0; k <= d.kmax; ++k) {
        ho(i, j, k) = a;
        hn(i, j, k) = b;
      }
    }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO - 1; ++i) {
      const R3 a = R3((ssuo(i, j) + HU_(i, j)) * kmaxm1), b = R3((ssun(i, j) + HU_(i, j)) * kmaxm1);
      for (int k = 0; k <= d.kmax; ++k) {
        huo(i, j, k) = a;
        hun(i, j, k) = b;
      }
    }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO - 1; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      const R3 a = R3((ssvo(i, j) + HV_(i, j)) * kmaxm1), b = R3((ssvn(i, j) + HV_(i, j)) * kmaxm1);
      for (int k = 0; k <= d.kmax; ++k) {
        hvo(i, j, k) = a;
        hvn(i, j, k) = b;
      }
    }
}

// ww_momentum_3d.F90:74-106 (kmin = 1)
template <class R3>
void ww_momentum_3d(const Dom& d, BcState<R3>& st) {
  A3<R3> ww{d, st.f3[WW]}, hn{d, st.f3[HN]}, ho{d, st.f3[HO]}, uu{d, st.f3[UU]}, vv{d, st.f3[VV]};
  M2 az{d, st.az};
  const R3 dtm1 = R3(1.0 / st.par[P_DT]);
  const R3 dx = R3(d.dx), dy = R3(d.dy), ard1 = R3(d.ard1);
  for (int k = 1; k <= d.kmax - 1; ++k)
#pragma omp parallel for schedule(static)
    for (int j = d.jmin; j <= d.jmax; ++j)
      for (int i = d.imin; i <= d.imax; ++i)
        if (az(i, j) == 1)
          ww(i, j, k) = ww(i, j, k - 1) - (hn(i, j, k) - ho(i, j, k)) * dtm1 -
                        (uu(i, j, k) * dy - uu(i - 1, j, k) * dy + vv(i, j, k) * dx - vv(i, j - 1, k) * dx) * ard1;
}

// uv_advect_3d.F90:62-460 (split schemes, no J7, no numerical analyses)
template <class R3>
int uv_advect_3d(const Dom& d, const AdvMasks& m, BcState<R3>& st) {
  const int* ip = st.ipar;
  const int split = ip[I_VEL3D_SPLIT], hor = ip[I_VEL3D_HOR], ver = ip[I_VEL3D_VER];
  if (hor == NOADV && ver == NOADV) return 0;
  const long n3 = d.n3d();
  std::vector<R3> f_(n3, R3(0)), ua_(n3, R3(0)), va_(n3, R3(0)), wa_(n3, R3(0)), hua_(n3, R3(0)), hva_(n3, R3(0));
  A3<R3> fadv{d, f_.data()}, uuadv{d, ua_.data()}, vvadv{d, va_.data()}, wwadv{d, wa_.data()}, huadv{d, hua_.data()},
      hvadv{d, hva_.data()};
  A3<R3> uu{d, st.f3[UU]}, vv{d, st.f3[VV]}, ww{d, st.f3[WW]}, ho{d, st.f3[HO]}, hn{d, st.f3[HN]}, hun{d, st.f3[HUN]},
      hvn{d, st.f3[HVN]};
  const R3 half = R3(0.5);
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) wwadv(i, j, 0) = R3(0);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= d.kmax; ++k)
    for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
      for (int i = d.imin - HALO; i <= d.imax + HALO - 1; ++i) {
        fadv(i, j, k) = uu(i, j, k) / hun(i, j, k);
        uuadv(i, j, k) = half * (uu(i, j, k) + uu(i + 1, j, k));
        vvadv(i, j, k) = half * (vv(i, j, k) + vv(i + 1, j, k));
        wwadv(i, j, k) = half * (ww(i, j, k) + ww(i + 1, j, k));
        huadv(i, j, k) = half * (ho(i + 1, j, k) + hn(i + 1, j, k));
        hvadv(i, j, k) = half * (hvn(i, j, k) + hvn(i + 1, j, k));
      }
  AdvGrid gu = adv_grid(m, U_TAG, st.az, st.au, st.av);
  if (do_advection_3d<R3>(d, gu, R3(st.par[P_DT]), f_.data(), ua_.data(), va_.data(), wa_.data(), hua_.data(),
                          hva_.data(), st.f3[HUN], st.f3[HUN], split, hor, ver, R3(0), U_TAG, nullptr, st.f3[UUEX],
                          ip[I_ADV_VER_ITERS]) < 0)
    return -1;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= d.kmax; ++k)
    for (int j = d.jmin - HALO; j <= d.jmax + HALO - 1; ++j)
      for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
        fadv(i, j, k) = vv(i, j, k) / hvn(i, j, k);
        uuadv(i, j, k) = half * (uu(i, j, k) + uu(i, j + 1, k));
        vvadv(i, j, k) = half * (vv(i, j, k) + vv(i, j + 1, k));
        wwadv(i, j, k) = half * (ww(i, j, k) + ww(i, j + 1, k));
        huadv(i, j, k) = half * (hun(i, j, k) + hun(i, j + 1, k));
        hvadv(i, j, k) = half * (ho(i, j + 1, k) + hn(i, j + 1, k));
      }
  AdvGrid gv = adv_grid(m, V_TAG, st.az, st.au, st.av);
  if (do_advection_3d<R3>(d, gv, R3(st.par[P_DT]), f_.data(), ua_.data(), va_.data(), wa_.data(), hua_.data(),
                          hva_.data(), st.f3[HVN], st.f3[HVN], split, hor, ver, R3(0), V_TAG, nullptr, st.f3[VVEX],
                          ip[I_ADV_VER_ITERS]) < 0)
    return -1;
  return 0;
}

// stresses_3d.F90:50-104 (taub/taus feed the turbulence closure only)
template <class R3>
void stresses_3d(const Dom& d, BcState<R3>& st) {
  double** f2 = st.f2;
  A2 rru{d, f2[RRU]}, rrv{d, f2[RRV]}, taubx{d, f2[TAUBX]}, tauby{d, f2[TAUBY]}, taub{d, f2[TAUB]}, taus{d, f2[TAUS]},
      tausx{d, f2[TAUSX]}, tausy{d, f2[TAUSY]};
  A3<R3> uu{d, st.f3[UU]}, vv{d, st.f3[VV]}, hun{d, st.f3[HUN]}, hvn{d, st.f3[HVN]};
  const double rho_0i = 1.0 / st.par[P_RHO_0];
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin - 1; i <= d.imax; ++i) taubx(i, j) = -(double)uu(i, j, 1) / (double)hun(i, j, 1) * rru(i, j);
  for (int j = d.jmin - 1; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) tauby(i, j) = -(double)vv(i, j, 1) / (double)hvn(i, j, 1) * rrv(i, j);
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) {
      double a = (double)uu(i - 1, j, 1) / (double)hun(i - 1, j, 1) * rru(i - 1, j);
      double b = (double)uu(i, j, 1) / (double)hun(i, j, 1) * rru(i, j);
      double c = (double)vv(i, j - 1, 1) / (double)hvn(i, j - 1, 1) * rrv(i, j - 1);
      double e = (double)vv(i, j, 1) / (double)hvn(i, j, 1) * rrv(i, j);
      taub(i, j) = std::sqrt(0.5 * (a * a + b * b + c * c + e * e));
      taus(i, j) = rho_0i * std::sqrt(tausx(i, j) * tausx(i, j) + tausy(i, j) * tausy(i, j));
    }
}

// eqstate.F90:496-534 (rho_from_theta_unesco80): UNESCO 1980 density at zero pressure. The
// coefficients are default-kind (single precision) literals in the reference, widened to double.
inline double rho_unesco80(double T, double S) {
  auto f = [](float c) { return (double)c; };
  const double T1 = T, T2 = T1 * T1, T3 = T1 * T2, T4 = T2 * T2, T5 = T1 * T4;
  const double S1 = S, S2 = S1 * S1, S3 = S1 * S2;
  double x = f(999.842594f) + f(6.793952e-02f) * T1 - f(9.09529e-03f) * T2 + f(1.001685e-04f) * T3;
  x = x - f(1.120083e-06f) * T4 + f(6.536332e-09f) * T5;
  x = x + S1 * (f(0.824493f) - f(4.0899e-03f) * T1 + f(7.6438e-05f) * T2 - f(8.2467e-07f) * T3);
  x = x + S1 * f(5.3875e-09f) * T4;
  x = x + std::sqrt(S3) * (-f(5.72466e-03f) + f(1.0227e-04f) * T1 - f(1.6546e-06f) * T2);
  x = x + f(4.8314e-04f) * S2;
  return x;
}

// eqstate.F90:540-590 (rho_from_theta at p = 0): the rational function of Jackett et al. (2006)
// for the density at zero pressure (double-precision coefficients).
inline double rho_jackett06(double s, double th) {
  const double th2 = th * th, sqrts = std::sqrt(s);
  const double anum = 9.9984085444849347e+02 +
                      th * (7.3471625860981584e+00 + th * (-5.3211231792841769e-02 + th * 3.6492439109814549e-04)) +
                      s * (2.5880571023991390e+00 - th * 6.7168282786692355e-03 + s * 1.9203202055760151e-03);
  const double aden =
      1.0000000000000000e+00 +
      th * (7.2815210113327091e-03 +
            th * (-4.4787265461983921e-05 + th * (3.3851002965802430e-07 + th * 1.3651202389758572e-10))) +
      s * (1.7632126669040377e-03 - th * (8.8066583251206474e-06 + th2 * 1.8832689434804897e-10) +
           sqrts * (5.7463776745432097e-06 + th2 * 1.4716275472242334e-09));
  return anum / aden;
}

// eqstate.F90:94-261 do_eqstate: density by the configured method -- 1 linear (:127-137, every
// point), 2 UNESCO80 (:148-156) or 3 Jackett et al. 2006 without pressure (:184-204), both on water
// columns (az > 0) only -- and the buoyancy -g/rho_0*(rho-rho_0) everywhere (:252-261). The
// thermal and haline coefficients alpha, beta that methods 2 and 3 also form (:158-176, :206-224)
// feed only the buoyancy frequency of the turbulence closure and are not formed here.
template <class R3>
void do_eqstate(const Dom& d, BcState<R3>& st) {
  A3<R3> rho{d, st.f3[RHO]}, buoy{d, st.f3[BUOY]}, T{d, st.f3[TT]}, S{d, st.f3[SS]};
  M2 az{d, st.az};
  const double* par = st.par;
  const int method = st.ipar[I_EQSTATE_METHOD];
  const R3 rho_0 = R3(par[P_RHO_0]), dtr0 = R3(par[P_DTR0]), dsr0 = R3(par[P_DSR0]), T0 = R3(par[P_T0]),
           S0 = R3(par[P_S0]);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= d.kmax; ++k)
    for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
      for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
        if (method == 2) {
          if (az(i, j) > 0) rho(i, j, k) = R3(rho_unesco80((double)T(i, j, k), (double)S(i, j, k)));
        } else if (method == 3) {
          if (az(i, j) > 0) rho(i, j, k) = R3(rho_jackett06((double)S(i, j, k), (double)T(i, j, k)));
        } else {
          rho(i, j, k) = rho_0 + dtr0 * (T(i, j, k) - T0) + dsr0 * (S(i, j, k) - S0);
        }
      }
  const R3 x = R3(-par[P_G] / par[P_RHO_0]);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= d.kmax; ++k)
    for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
      for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) buoy(i, j, k) = x * (rho(i, j, k) - rho_0);
}

// gotm.F90:96-163 with PARABOLIC_VISCOSITY (:131-143): per water column of the interior the
// prescribed profiles of turbulent kinetic energy, length scale, dissipation and eddy viscosity
// from the bottom stress taub and the bottom roughness, on the interfaces k = 1..kmax-1; num and nuh
// get the background values avmback / avhback added on every level (at k = 0 and kmax onto the
// values they held, which the reference copies through its 1D column arrays). tke and eps (may be
// null) receive the profiles. Single-precision literals as in the reference.
template <class R3>
void gotm_parabolic(const Dom& d, BcState<R3>& st) {
  A2 D{d, st.f2[D_]}, taub{d, st.f2[TAUB]}, zub{d, st.f2[ZUB]}, zvb{d, st.f2[ZVB]};
  A3<R3> hn{d, st.f3[HN]}, num{d, st.f3[NUM]}, nuh{d, st.f3[NUH]}, tke{d, st.f3[TKE]}, eps{d, st.f3[EPS]};
  M2 az{d, st.az};
  const int kmax = d.kmax;
  const double avmback = st.par[P_AVMBACK], avhback = st.par[P_AVHBACK];
  auto f = [](float c) { return (double)c; };
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) {
      if (az(i, j) < 1) continue;
      const double z0b = 0.5 * (std::max(zub(i - 1, j), zub(i, j)) + std::max(zvb(i, j - 1), zvb(i, j)));
      double zz = 0.0;
      for (int k = 1; k <= kmax - 1; ++k) {
        zz = zz + (double)hn(i, j, k);
        const double t = std::max(f(1.e-10f), f(3.333333f) * taub(i, j) * (1.0 - zz / D(i, j)));
        const double L = f(0.4f) * (zz + z0b) * std::sqrt(1.0 - zz / D(i, j));
        const double e = f(0.16431677f) * std::sqrt(t * t * t) / L;
        const double nu = f(0.09f) * t * t / e;
        if (st.f3[TKE]) tke(i, j, k) = R3(t);
        if (st.f3[EPS]) eps(i, j, k) = R3(e);
        num(i, j, k) = R3(nu + avmback);
        nuh(i, j, k) = R3(nu + avhback);
      }
      for (int k : {0, kmax}) {
        if (kmax < 1) break;
        num(i, j, k) = R3((double)num(i, j, k) + avmback);
        nuh(i, j, k) = R3((double)nuh(i, j, k) + avhback);
      }
    }
}

// temperature.F90:452-465: the short-wave radiation profile rad of the water columns (az >= 1) of
// the interior: swr at the surface, below it the two-band exponential decay A*exp(-z/g1) +
// (1-A)*exp(-z/g2) with the depth z under the surface.
template <class R3>
void sw_radiation(const Dom& d, BcState<R3>& st) {
  A2 swr{d, st.f2[SWR]}, A{d, st.f2[ATT_A]}, g1{d, st.f2[ATT_G1]}, g2{d, st.f2[ATT_G2]};
  A3<R3> hn{d, st.f3[HN]}, rad{d, st.f3[RAD]};
  M2 az{d, st.az};
  const int kmax = d.kmax;
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) {
      if (az(i, j) < 1) continue;
      const double swr_loc = swr(i, j);
      rad(i, j, kmax) = R3(swr_loc);
      double zz = 0.0;
      for (int k = kmax - 1; k >= 0; --k) {
        zz = zz + (double)hn(i, j, k + 1);
        rad(i, j, k) = R3(swr_loc * (A(i, j) * std::exp(-zz / g1(i, j)) + (1 - A(i, j)) * std::exp(-zz / g2(i, j))));
      }
    }
}

// temperature.F90:469-525: the source terms that do_temperature adds to the right-hand side of
// its diffusion matrix, per layer k = 1..kmax of the water columns (az == 1) of the interior:
// dry_z*dt*(rad1d(k) - rad1d(k-1)), plus shf*rho_0_cpi in the top layer. rad1d is rad less the
// bottom-reflected part (when swr_bot_refl_frac > 0 and enough light reaches the bottom) scaled by
// 1/(rho_0*cp); a cooling surface flux is dropped where the top layer is at the freezing point
// (T <= -0.0575*S, "the most primitive sea ice model"). S is the salinity before do_salinity.
template <class R3>
void temperature_source(const Dom& d, BcState<R3>& st, R3* srcp) {
  A2 shf{d, st.f2[SHF]}, A{d, st.f2[ATT_A]}, g1{d, st.f2[ATT_G1]}, g2{d, st.f2[ATT_G2]}, dry_z{d, st.f2[DRY_Z]};
  A3<R3> hn{d, st.f3[HN]}, rad{d, st.f3[RAD]}, T{d, st.f3[TT]}, S{d, st.f3[SS]}, src{d, srcp};
  M2 az{d, st.az};
  const int kmax = d.kmax;
  const double dt = st.par[P_DT];
  const double rho_0_cpi = 1.0 / (st.par[P_RHO_0] * st.par[P_CP]);
  const double refl = st.par[P_SWR_BOT_REFL_FRAC], minfrac = st.par[P_SWR_MIN_BOT_FRAC];
  std::vector<double> rad1d(kmax + 1);
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) {
      if (az(i, j) != 1) continue;
      double shf_loc = shf(i, j);
      if ((double)T(i, j, kmax) <= -((double)0.0575f * (double)S(i, j, kmax))) shf_loc = std::max(0.0, shf_loc);
      for (int k = 0; k <= kmax; ++k) rad1d[k] = (double)rad(i, j, k);
      if (refl > 0.0 && rad1d[0] / rad1d[kmax] > minfrac) {
        const double swr_refl = rad1d[0] * refl;
        rad1d[0] = rad1d[0] - swr_refl;
        double zz = 0.0;
        for (int k = 1; k <= kmax; ++k) {
          zz = zz + (double)hn(i, j, k);
          rad1d[k] = (double)rad(i, j, k) -
                     swr_refl * (A(i, j) * std::exp(-zz / g1(i, j)) + (1 - A(i, j)) * std::exp(-zz / g2(i, j)));
        }
      }
      for (int k = 0; k <= kmax; ++k) rad1d[k] = rad1d[k] * rho_0_cpi;
      for (int k = 1; k <= kmax - 1; ++k) src(i, j, k) = R3(dry_z(i, j) * dt * (rad1d[k] - rad1d[k - 1]));
      src(i, j, kmax) = R3(dry_z(i, j) * dt * (rad1d[kmax] + shf_loc * rho_0_cpi - rad1d[kmax - 1]));
    }
}

// slow_bottom_friction.F90:53-170
template <class R3>
void slow_bottom_friction(const Dom& d, BcState<R3>& st) {
  double** f2 = st.f2;
  A2 Uinto{d, f2[UINTO]}, Vinto{d, f2[VINTO]}, ssuo{d, f2[SSUO]}, ssun{d, f2[SSUN]}, ssvo{d, f2[SSVO]},
      ssvn{d, f2[SSVN]}, HU_{d, f2[HU]}, HV_{d, f2[HV]}, zub{d, f2[ZUB]}, zvb{d, f2[ZVB]}, ru{d, f2[RU]},
      rv{d, f2[RV]};
  M2 au{d, st.au}, av{d, st.av};
  const double kappa = st.par[P_KAPPA], min_depth = st.par[P_MIN_DEPTH];
  const long n = d.n2d();
  std::vector<double> Ui_(n, 0.0), Vi_(n, 0.0), ruu_(n, 0.0), rvv_(n, 0.0);
  A2 Ui{d, Ui_.data()}, Vi{d, Vi_.data()}, ruu{d, ruu_.data()}, rvv{d, rvv_.data()};
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      Ui(i, j) = au(i, j) >= 1 ? Uinto(i, j) / (ssuo(i, j) + HU_(i, j)) : 0.0;
  for (int i = d.imin - HALO; i <= d.imax + HALO; ++i)
    Ui(i, d.jmax + 1) = Uinto(i, d.jmax + 1) / (ssuo(i, d.jmax + 1) + HU_(i, d.jmax + 1));
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    Ui(d.imin - 1, j) = Uinto(d.imin - 1, j) / (ssuo(d.imin - 1, j) + HU_(d.imin - 1, j));
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      Vi(i, j) = av(i, j) >= 1 ? Vinto(i, j) / (ssvo(i, j) + HV_(i, j)) : 0.0;
  for (int i = d.imin - HALO; i <= d.imax + HALO; ++i)
    Vi(i, d.jmin - 1) = Vinto(i, d.jmin - 1) / (ssvo(i, d.jmin - 1) + HV_(i, d.jmin - 1));
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    Vi(d.imax + 1, j) = Vinto(d.imax + 1, j) / (ssvo(d.imax + 1, j) + HV_(d.imax + 1, j));
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (au(i, j) >= 1) {
        double HHl = std::max(min_depth, ssun(i, j) + HU_(i, j));
        ruu(i, j) = (zub(i, j) + 0.5 * HHl) / zub(i, j);
        double x = kappa / std::log(ruu(i, j));
        ruu(i, j) = x * x;
      }
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (av(i, j) >= 1) {
        double HHl = std::max(min_depth, ssvn(i, j) + HV_(i, j));
        rvv(i, j) = (zvb(i, j) + 0.5 * HHl) / zvb(i, j);
        double x = kappa / std::log(rvv(i, j));
        rvv(i, j) = x * x;
      }
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) {
      if (au(i, j) >= 1) {
        double uloc = Ui(i, j);
        double vloc = 0.25 * (Vi(i, j) + Vi(i + 1, j) + Vi(i, j - 1) + Vi(i + 1, j - 1));
        ru(i, j) = ruu(i, j) * std::sqrt(uloc * uloc + vloc * vloc);
      } else {
        ru(i, j) = 0.0;
      }
    }
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i) {
      if (av(i, j) >= 1) {
        double uloc = 0.25 * (Ui(i, j) + Ui(i - 1, j) + Ui(i, j + 1) + Ui(i - 1, j + 1));
        double vloc = Vi(i, j);
        rv(i, j) = rvv(i, j) * std::sqrt(uloc * uloc + vloc * vloc);
      } else {
        rv(i, j) = 0.0;
      }
    }
}

// slow_terms.F90:57-181 (kmax > 1, kumin = kvmin = 1)
template <class R3>
void slow_terms(const Dom& d, BcState<R3>& st) {
  double** f2 = st.f2;
  A2 UEx{d, f2[UEX]}, VEx{d, f2[VEX]}, SlUx{d, f2[SLUX]}, SlVx{d, f2[SLVX]}, Slru{d, f2[SLRU]}, Slrv{d, f2[SLRV]},
      Uint{d, f2[UINT]}, Vint{d, f2[VINT]}, ssuo{d, f2[SSUO]}, ssun{d, f2[SSUN]}, ssvo{d, f2[SSVO]}, ssvn{d, f2[SSVN]},
      HU_{d, f2[HU]}, HV_{d, f2[HV]}, ru{d, f2[RU]}, rv{d, f2[RV]}, rru{d, f2[RRU]}, rrv{d, f2[RRV]};
  A3<R3> uuEx{d, st.f3[UUEX]}, vvEx{d, st.f3[VVEX]}, idpdx{d, st.f3[IDPDX]}, idpdy{d, st.f3[IDPDY]}, uu{d, st.f3[UU]},
      vv{d, st.f3[VV]}, huo{d, st.f3[HUO]}, hun{d, st.f3[HUN]}, hvo{d, st.f3[HVO]}, hvn{d, st.f3[HVN]};
  M2 au{d, st.au}, av{d, st.av};
  const double ip_fac = st.par[P_IP_FAC];
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (au(i, j) >= 1) {
        double vs = -UEx(i, j);
        for (int k = 1; k <= d.kmax; ++k) vs = vs + (double)uuEx(i, j, k) - ip_fac * (double)idpdx(i, j, k);
        SlUx(i, j) = vs;
      }
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (av(i, j) >= 1) {
        double vs = -VEx(i, j);
        for (int k = 1; k <= d.kmax; ++k) vs = vs + (double)vvEx(i, j, k) - ip_fac * (double)idpdy(i, j, k);
        SlVx(i, j) = vs;
      }
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (au(i, j) >= 1)
        Slru(i, j) = -Uint(i, j) / (0.5 * (ssuo(i, j) + ssun(i, j)) + HU_(i, j)) * ru(i, j) +
                     (double)uu(i, j, 1) / (0.5 * ((double)huo(i, j, 1) + (double)hun(i, j, 1))) * rru(i, j);
  for (int j = d.jmin; j <= d.jmax; ++j)
    for (int i = d.imin; i <= d.imax; ++i)
      if (av(i, j) >= 1)
        Slrv(i, j) = -Vint(i, j) / (0.5 * (ssvo(i, j) + ssvn(i, j)) + HV_(i, j)) * rv(i, j) +
                     (double)vv(i, j, 1) / (0.5 * ((double)hvo(i, j, 1) + (double)hvn(i, j, 1))) * rrv(i, j);
}

// Hotstart (initialise.F90:295-334 with hotstart = .true.): after read_restart_ncdf has filled the
// restart fields, postinit_2d (m2d.F90:358-400) and postinit_3d (m3d.F90:376-409) re-derive the rest.
// postinit_2d: if any U /= 0 where au == 0 (or V /= 0 where av == 0), U, Uinto = 0 where au == 0
// and V, Vinto = 0 where av == 0; z = zo = -9999 on land (az == 0); depth_update. postinit_3d
// (runtype > 1): uu = 0 where au == 0, vv = 0 where av == 0; on land tke = 0, num = nuh = 1e-15
// (a single-precision literal), T = S = -9999; coordinates(hotstart), i.e. sigma_coordinates.
template <class R3>
void hotstart_postinit(const Dom& d, BcState<R3>& st, int runtype) {
  double** f2 = st.f2;
  A2 U{d, f2[U_]}, V{d, f2[V_]}, Uinto{d, f2[UINTO]}, Vinto{d, f2[VINTO]}, z{d, f2[Z]}, zo{d, f2[ZO]};
  M2 az{d, st.az}, au{d, st.au}, av{d, st.av};
  bool change = false;
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      if (au(i, j) == 0 && U(i, j) != 0.0) change = true;
      if (av(i, j) == 0 && V(i, j) != 0.0) change = true;
    }
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i) {
      if (change && au(i, j) == 0) {
        U(i, j) = 0.0;
        Uinto(i, j) = 0.0;
      }
      if (change && av(i, j) == 0) {
        V(i, j) = 0.0;
        Vinto(i, j) = 0.0;
      }
      if (az(i, j) == 0) {
        z(i, j) = -9999.0;
        zo(i, j) = -9999.0;
      }
    }
  depth_update(d, f2, st.az, st.au, st.av, st.par);
  if (runtype <= 1) return;
  A3<R3> uu{d, st.f3[UU]}, vv{d, st.f3[VV]}, tke{d, st.f3[TKE]}, num{d, st.f3[NUM]}, nuh{d, st.f3[NUH]},
      T{d, st.f3[TT]}, S{d, st.f3[SS]};
  for (int j = d.jmin - HALO; j <= d.jmax + HALO; ++j)
    for (int i = d.imin - HALO; i <= d.imax + HALO; ++i)
      for (int k = 0; k <= d.kmax; ++k) {
        if (au(i, j) == 0) uu(i, j, k) = R3(0);
        if (av(i, j) == 0) vv(i, j, k) = R3(0);
        if (az(i, j) == 0) {
          if (st.f3[TKE]) tke(i, j, k) = R3(0);
          num(i, j, k) = R3((double)1.e-15f);
          nuh(i, j, k) = R3((double)1.e-15f);
          S(i, j, k) = R3(-9999.0);
          T(i, j, k) = R3(-9999.0);
        }
      }
  sigma_coordinates(d, st);
}

// m3d.F90:422-636 integrate_3d for runtype 4 (see header for the configuration covered)
template <class R3>
int integrate_3d(const Dom& d, const AdvMasks& m, BcState<R3>& st, int n) {
  (void)n;
  double** f2 = st.f2;
  int* ip = st.ipar;
  const double* par = st.par;
  const long n3 = d.n3d();
  const long n2 = d.n2d();
  start_macro(d, f2, par, ip[I_M]);
  if (d.kmax > 1) bottom_friction_3d(d, st);
  if (ip[I_RUNTYPE] == 4 && do_internal_pressure(d, st) != 0) return -1;
  for (long q = 0; q < n3; ++q) {
    st.f3[HUO][q] = st.f3[HUN][q];
    st.f3[HVO][q] = st.f3[HVN][q];
  }
  if (ip[I_UFIRST3D]) {
    uv_momentum_3d(d, st, 0);
    uv_momentum_3d(d, st, 1);
    ip[I_UFIRST3D] = 0;
  } else {
    uv_momentum_3d(d, st, 1);
    uv_momentum_3d(d, st, 0);
    ip[I_UFIRST3D] = 1;
  }
  sigma_coordinates(d, st);
  if (d.kmax > 1) {
    ww_momentum_3d(d, st);
    if (uv_advect_3d(d, m, st) != 0) return -1;
    stresses_3d(d, st);
    if (ip[I_VISCOSITY] == 1) gotm_parabolic(d, st);  // m3d.F90:570-575
  }
  if (ip[I_RUNTYPE] == 4) {
    const R3 dt = R3(par[P_DT]);
    if (ip[I_CALC_TEMP]) {
      AdvGrid g = adv_grid(m, H_TAG, st.az, st.au, st.av);
      if (do_advection_3d<R3>(d, g, dt, st.f3[TT], st.f3[UU], st.f3[VV], st.f3[WW], st.f3[HUN], st.f3[HVN],
                              st.f3[HO], st.f3[HN], ip[I_TEMP_SPLIT], ip[I_TEMP_HOR], ip[I_TEMP_VER],
                              R3(par[P_TEMP_AH]), H_TAG, nullptr, nullptr, ip[I_ADV_VER_ITERS]) < 0)
        return -1;
      std::vector<R3> src;
      if (ip[I_RADIATION]) {  // temperature.F90:452-525
        sw_radiation(d, st);
        src.assign(n3, R3(0));
        if (d.kmax > 1) temperature_source(d, st, src.data());
      }
      tracer_vdiff<R3>(d, dt, R3(par[P_CNPAR]), R3(par[P_AVMOLT]), st.f3[TT], st.f3[HN], st.f3[NUH], st.az,
                       src.empty() ? nullptr : src.data());
    }
    if (ip[I_CALC_SALT]) {
      AdvGrid g = adv_grid(m, H_TAG, st.az, st.au, st.av);
      if (do_advection_3d<R3>(d, g, dt, st.f3[SS], st.f3[UU], st.f3[VV], st.f3[WW], st.f3[HUN], st.f3[HVN],
                              st.f3[HO], st.f3[HN], ip[I_SALT_SPLIT], ip[I_SALT_HOR], ip[I_SALT_VER],
                              R3(par[P_SALT_AH]), H_TAG, nullptr, nullptr, ip[I_ADV_VER_ITERS]) < 0)
        return -1;
      tracer_vdiff<R3>(d, dt, R3(par[P_CNPAR]), R3(par[P_AVMOLS]), st.f3[SS], st.f3[HN], st.f3[NUH], st.az, nullptr);
    }
    if (st.bdy) {  // m3d.F90:595,602
      if (ip[I_CALC_TEMP]) mirror_bdy<R3>(d, *st.bdy, st.az, st.au, st.av, st.f3[TT], 2, d.kmax + 1, d.sk);
      if (ip[I_CALC_SALT]) mirror_bdy<R3>(d, *st.bdy, st.az, st.au, st.av, st.f3[SS], 2, d.kmax + 1, d.sk);
    }
    do_eqstate(d, st);
  }
  if (d.kmax > 1) {
    slow_bottom_friction(d, st);
    if (uv_advect_2d(d, m, st.az, st.au, st.av, par[P_DTM], f2[UINT], f2[VINT], f2[DUN], f2[DVN], ip[I_VEL2D_SPLIT],
                     ip[I_VEL2D_HOR], f2[UEX], f2[VEX]) != 0)
      return -1;
  }
  slow_terms(d, st);
  // stop_macro.F90:36-39
  for (long q = 0; q < n2; ++q) {
    f2[UINTO][q] = f2[UINT][q];
    f2[UINT][q] = 0.0;
    f2[VINTO][q] = f2[VINT][q];
    f2[VINT][q] = 0.0;
  }
  return 0;
}

}  // namespace gor
