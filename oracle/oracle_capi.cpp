// oracle_capi.cpp -- TEST INFRASTRUCTURE ONLY: extern "C" entry points of the CPU oracle
// (getm_oracle.hpp) for the Python test harness (oracle/__init__.py, via ctypes).
// Suffix _d = FP64 (the reference's REALTYPE), _f = FP32.
#include "getm_oracle.hpp"
#include "getm_baroclinic.hpp"
#include "getm_tangent.hpp"

extern "C" {

typedef struct {
  int imin, imax, jmin, jmax, kmax;
  long long sj, sk;
  double dx, dy, ard1;
} or_dom;

static gor::Dom mk(const or_dom* o) {
  gor::Dom d;
  d.imin = o->imin; d.imax = o->imax; d.jmin = o->jmin; d.jmax = o->jmax; d.kmax = o->kmax;
  d.sj = (long)o->sj; d.sk = (long)o->sk; d.dx = o->dx; d.dy = o->dy; d.ard1 = o->ard1;
  return d;
}

void or_derive_uvx(const or_dom* o, const int32_t* az, int32_t* au, int32_t* av, int32_t* ax) {
  gor::derive_uvx_masks(mk(o), az, au, av, ax);
}

// out: 8 consecutive byte planes of n2d each:
// updateH, uflux, vflux, xflux, uupdateU, vupdateV, uflux_U, vflux_V
void or_build_masks(const or_dom* o, const int32_t* az, const int32_t* au, const int32_t* av,
                    const int32_t* ax, uint8_t* out) {
  gor::Dom d = mk(o);
  gor::AdvMasks m;
  gor::build_adv_masks(d, az, au, av, ax, m);
  const long n = d.n2d();
  const std::vector<uint8_t>* planes[8] = {&m.updateH, &m.uflux, &m.vflux, &m.xflux,
                                           &m.uupdateU, &m.vupdateV, &m.uflux_U, &m.vflux_V};
  for (int q = 0; q < 8; ++q) std::memcpy(out + q * n, planes[q]->data(), n);
}

#define OR_DEFINE(SUF, R)                                                                             \
  int or_recon_##SUF(int scheme, const R* cfl, const R* fuu, const R* fu, const R* fd, R* out,       \
                     long long n) {                                                                   \
    for (long long q = 0; q < n; ++q)                                                                 \
      out[q] = gor::adv_interfacial_reconstruction<R>(scheme, cfl[q], fuu[q], fu[q], fd[q]);          \
    return 0;                                                                                         \
  }                                                                                                   \
  void or_adv_split_u_##SUF(const or_dom* o, R dt, const R* f, R* fi, R* Di, R* adv, const R* U,      \
                            const R* DU, R splitfac, int scheme, R AH, const uint8_t* mflux,          \
                            const uint8_t* mupd) {                                                    \
    gor::adv_split_u<R>(mk(o), dt, f, fi, Di, adv, U, DU, splitfac, scheme, AH, mflux, mupd);        \
  }                                                                                                   \
  void or_adv_split_v_##SUF(const or_dom* o, R dt, const R* f, R* fi, R* Di, R* adv, const R* V,      \
                            const R* DV, R splitfac, int scheme, R AH, const uint8_t* mflux,          \
                            const uint8_t* mupd) {                                                    \
    gor::adv_split_v<R>(mk(o), dt, f, fi, Di, adv, V, DV, splitfac, scheme, AH, mflux, mupd);        \
  }                                                                                                   \
  long long or_adv_split_w_##SUF(const or_dom* o, R dt, const R* f, R* fi, R* hi, R* adv,            \
                                 const R* ww, R splitfac, int scheme, int tag, const int32_t* az,     \
                                 int itersmax) {                                                      \
    return gor::adv_split_w<R>(mk(o), dt, f, fi, hi, adv, ww, splitfac, scheme, tag, az, itersmax);   \
  }                                                                                                   \
  long long or_do_advection_3d_##SUF(const or_dom* o, const int32_t* az, const int32_t* au,          \
                                     const int32_t* av, const int32_t* ax, R dt, R* f, const R* uu,   \
                                     const R* vv, const R* ww, const R* hu, const R* hv, const R* ho, \
                                     const R* hn, int split, int hscheme, int vscheme, R AH, int tag, \
                                     R* hires, R* advres, int iters) {                                \
    gor::Dom d = mk(o);                                                                               \
    gor::AdvMasks m;                                                                                  \
    gor::build_adv_masks(d, az, au, av, ax, m);                                                       \
    gor::AdvGrid g = gor::adv_grid(m, tag, az, au, av);                                               \
    return gor::do_advection_3d<R>(d, g, dt, f, uu, vv, ww, hu, hv, ho, hn, split, hscheme, vscheme, \
                                   AH, tag, hires, advres, iters);                                    \
  }                                                                                                   \
  int or_do_advection_##SUF(const or_dom* o, const int32_t* az, const int32_t* au, const int32_t* av, \
                            const int32_t* ax, R dt, R* f, const R* U, const R* V, const R* DU,       \
                            const R* DV, const R* Do, const R* Dn, int split, int scheme, R AH,       \
                            int tag, R* Dires, R* advres) {                                           \
    gor::Dom d = mk(o);                                                                               \
    gor::AdvMasks m;                                                                                  \
    gor::build_adv_masks(d, az, au, av, ax, m);                                                       \
    gor::AdvGrid g = gor::adv_grid(m, tag, az, au, av);                                               \
    return gor::do_advection<R>(d, g, dt, f, U, V, DU, DV, Do, Dn, split, scheme, AH, Dires, advres); \
  }                                                                                                   \
  void or_tridiagonal_##SUF(int kmax, int fi, int lt, const R* au, const R* bu, const R* cu,          \
                            const R* du, R* value) {                                                  \
    gor::getm_tridiagonal<R>(kmax, fi, lt, au, bu, cu, du, value);                                    \
  }                                                                                                   \
  void or_tracer_vdiff_##SUF(const or_dom* o, R dt, R cnpar, R avmol, R* S, const R* hn,              \
                             const R* nuh, const int32_t* az, const R* src) {                         \
    gor::tracer_vdiff<R>(mk(o), dt, cnpar, avmol, S, hn, nuh, az, src);                               \
  }                                                                                                   \
  double or_tracer_content_##SUF(const or_dom* o, const R* f, const R* h, const int32_t* az) {        \
    return gor::tracer_content<R>(mk(o), f, h, az);                                                   \
  }                                                                                                   \
  /* nsteps of the tracer step (do_advection_3d then vertical diffusion, salinity.F90:301-389) */   \
  long long or_tracer_steps_##SUF(const or_dom* o, const int32_t* az, const int32_t* au,             \
                                  const int32_t* av, const int32_t* ax, int nsteps, R dt, R* f,       \
                                  const R* uu, const R* vv, const R* ww, const R* hu, const R* hv,    \
                                  const R* ho, const R* hn, const R* nuh, int split, int hscheme,     \
                                  int vscheme, R AH, R cnpar, R avmol, int iters) {                   \
    gor::Dom d = mk(o);                                                                               \
    gor::AdvMasks m;                                                                                  \
    gor::build_adv_masks(d, az, au, av, ax, m);                                                       \
    gor::AdvGrid g = gor::adv_grid(m, gor::H_TAG, az, au, av);                                        \
    long long warn = 0;                                                                               \
    for (int s = 0; s < nsteps; ++s) {                                                                \
      long r = gor::do_advection_3d<R>(d, g, dt, f, uu, vv, ww, hu, hv, ho, hn, split, hscheme,      \
                                       vscheme, AH, gor::H_TAG, nullptr, nullptr, iters);             \
      if (r < 0) return -1;                                                                           \
      warn += r;                                                                                      \
      gor::tracer_vdiff<R>(d, dt, cnpar, avmol, f, hn, nuh, az, nullptr);                             \
    }                                                                                                 \
    return warn;                                                                                      \
  }

OR_DEFINE(d, double)
OR_DEFINE(f, float)

// Tangent-linear tracer steps (getm_tangent.hpp): nsteps of the FP64 tracer step carrying the
// derivative in the direction (df, dnuh); f and df are advanced in place.
long long or_tracer_steps_tl(const or_dom* o, const int32_t* az, const int32_t* au, const int32_t* av,
                             const int32_t* ax, int nsteps, double dt, double* f, double* df, const double* uu,
                             const double* vv, const double* ww, const double* hu, const double* hv,
                             const double* ho, const double* hn, const double* nuh, const double* dnuh, int split,
                             int hscheme, int vscheme, double AH, double cnpar, double avmol) {
  using gor::Dual;
  gor::Dom d = mk(o);
  gor::AdvMasks m;
  gor::build_adv_masks(d, az, au, av, ax, m);
  gor::AdvGrid g = gor::adv_grid(m, gor::H_TAG, az, au, av);
  const long n3 = d.n3d();
  auto cst = [&](const double* a) {
    std::vector<Dual> v(n3);
    for (long q = 0; q < n3; ++q) v[q] = Dual(a[q]);
    return v;
  };
  std::vector<Dual> F(n3), NU(n3);
  for (long q = 0; q < n3; ++q) {
    F[q] = Dual(f[q], df[q]);
    NU[q] = Dual(nuh[q], dnuh ? dnuh[q] : 0.0);
  }
  std::vector<Dual> UU = cst(uu), VV = cst(vv), WW = cst(ww), HU = cst(hu), HV = cst(hv), HO = cst(ho),
                    HN = cst(hn);
  long long warn = 0;
  for (int s = 0; s < nsteps; ++s) {
    long r = gor::do_advection_3d<Dual>(d, g, Dual(dt), F.data(), UU.data(), VV.data(), WW.data(), HU.data(),
                                        HV.data(), HO.data(), HN.data(), split, hscheme, vscheme, Dual(AH), gor::H_TAG,
                                        nullptr, nullptr, 1);
    if (r < 0) return -1;
    warn += r;
    gor::tracer_vdiff<Dual>(d, Dual(dt), Dual(cnpar), Dual(avmol), F.data(), HN.data(), NU.data(), az, nullptr);
  }
  for (long q = 0; q < n3; ++q) {
    f[q] = F[q].v;
    df[q] = F[q].d;
  }
  return warn;
}

// ---- mode-split time loop (getm_baroclinic.hpp) -------------------------------------------------
// Open boundaries: the layout of getm_bdy in include/getm_b200.h.
typedef struct {
  int32_t nwb, nnb, neb, nsb;
  const int32_t* seg;
  const int32_t* type2d;
  int32_t ramp, npoints;
  const double *data, *data_u, *data_v, *amp, *phase;
  double period;
} or_bdy;

typedef struct {
  double* f2[gor::NF2];
  void* f3[gor::NF3];
  const int32_t *az, *au, *av, *ax;
  double par[gor::NPD];
  int ipar[gor::NPI];
  const or_bdy* bdy;  // NULL: closed domain
} or_bc;

int or_bc_sizes(int* out) {
  out[0] = gor::NF2;
  out[1] = gor::NF3;
  out[2] = gor::NPD;
  out[3] = gor::NPI;
  return 0;
}

extern "C++" {
static gor::Bdy to_bdy(const or_bdy* b) {
  gor::Bdy o;
  o.nwb = b->nwb; o.nnb = b->nnb; o.neb = b->neb; o.nsb = b->nsb;
  const int ns = o.nseg(), np = b->npoints;
  o.seg.assign(b->seg, b->seg + 3 * ns);
  o.type2d.assign(b->type2d, b->type2d + ns);
  o.ramp = b->ramp;
  auto cp = [&](const double* p, std::vector<double>& v) { if (p) v.assign(p, p + np); };
  cp(b->data, o.data); cp(b->data_u, o.data_u); cp(b->data_v, o.data_v); cp(b->amp, o.amp); cp(b->phase, o.phase);
  o.period = b->period;
  return o;
}

template <class R3>
static gor::BcState<R3> to_state(or_bc* s, gor::Bdy* bdy) {
  gor::BcState<R3> st;
  if (s->bdy) {
    *bdy = to_bdy(s->bdy);
    st.bdy = bdy;
  }
  for (int q = 0; q < gor::NF2; ++q) st.f2[q] = s->f2[q];
  for (int q = 0; q < gor::NF3; ++q) st.f3[q] = (R3*)s->f3[q];
  st.az = s->az; st.au = s->au; st.av = s->av; st.ax = s->ax;
  for (int q = 0; q < gor::NPD; ++q) st.par[q] = s->par[q];
  for (int q = 0; q < gor::NPI; ++q) st.ipar[q] = s->ipar[q];
  return st;
}
}  // extern "C++"

// time_loop (integration.F90:98-172): micro steps n = n0 .. n0+count-1, integrate_2d every step and
// integrate_3d when do_3d = (runtype >= 2 and mod(n, M) == 0) (integration.F90:106). The SAVEd
// momentum toggles are carried in ipar.
extern "C++" {
template <class R3>
static long long bc_steps(const or_dom* o, or_bc* s, int n0, int count) {
  gor::Dom d = mk(o);
  gor::AdvMasks m;
  gor::build_adv_masks(d, s->az, s->au, s->av, s->ax, m);
  gor::Bdy bdy;
  gor::BcState<R3> st = to_state<R3>(s, &bdy);
  for (int n = n0; n < n0 + count; ++n) {
    if (gor::integrate_2d(d, m, st, n) != 0) return -1;
    if (st.ipar[gor::I_RUNTYPE] >= 2 && n % st.ipar[gor::I_M] == 0)
      if (gor::integrate_3d(d, m, st, n) != 0) return -1;
  }
  for (int q = 0; q < gor::NPI; ++q) s->ipar[q] = st.ipar[q];
  return 0;
}
}  // extern "C++"

long long or_bc_steps_d(const or_dom* o, or_bc* s, int n0, int count) { return bc_steps<double>(o, s, n0, count); }
long long or_bc_steps_f(const or_dom* o, or_bc* s, int n0, int count) { return bc_steps<float>(o, s, n0, count); }

// single routines of the step (for routine-level parity tests)
enum {
  BC_BOTTOM_FRICTION = 0, BC_UV_ADVECT_2D, BC_UMOMENTUM, BC_VMOMENTUM, BC_SEALEVEL, BC_DEPTH_UPDATE,
  BC_START_MACRO, BC_BOTTOM_FRICTION_3D, BC_IP, BC_UU_MOMENTUM_3D, BC_VV_MOMENTUM_3D, BC_SIGMA, BC_WW,
  BC_UV_ADVECT_3D, BC_STRESSES_3D, BC_EQSTATE, BC_SLOW_BOTTOM_FRICTION, BC_SLOW_TERMS, BC_INTEGRATE_2D,
  BC_INTEGRATE_3D, BC_GOTM_PARABOLIC, BC_SW_RADIATION, BC_UPDATE_2D_BDY, BC_HOTSTART_POSTINIT
};

extern "C++" {
template <class R3>
static int bc_call(const or_dom* o, or_bc* s, int which, int arg) {
  gor::Dom d = mk(o);
  gor::AdvMasks m;
  gor::build_adv_masks(d, s->az, s->au, s->av, s->ax, m);
  gor::Bdy bdy;
  gor::BcState<R3> st = to_state<R3>(s, &bdy);
  int rc = 0;
  switch (which) {
    case BC_BOTTOM_FRICTION: gor::bottom_friction(d, nullptr, st.f2, st.au, st.av, st.par, st.ipar[gor::I_RUNTYPE]); break;
    case BC_UV_ADVECT_2D:
      rc = gor::uv_advect_2d(d, m, st.az, st.au, st.av, st.par[gor::P_DTM], st.f2[gor::U_], st.f2[gor::V_],
                             st.f2[gor::DU], st.f2[gor::DV], st.ipar[gor::I_VEL2D_SPLIT], st.ipar[gor::I_VEL2D_HOR],
                             st.f2[gor::UEX], st.f2[gor::VEX]);
      break;
    case BC_UMOMENTUM: gor::umomentum(d, st.f2, st.au, st.av, st.par, st.bdy, st.az); break;
    case BC_VMOMENTUM: gor::vmomentum(d, st.f2, st.au, st.av, st.par, st.bdy, st.az); break;
    case BC_SEALEVEL: gor::sealevel(d, st.f2, st.az, st.par); break;
    case BC_DEPTH_UPDATE: gor::depth_update(d, st.f2, st.az, st.au, st.av, st.par); break;
    case BC_START_MACRO: gor::start_macro(d, st.f2, st.par, st.ipar[gor::I_M]); break;
    case BC_BOTTOM_FRICTION_3D: gor::bottom_friction_3d(d, st); break;
    case BC_IP:
      if (gor::do_internal_pressure(d, st) != 0) return -1;
      break;
    case BC_UU_MOMENTUM_3D: gor::uv_momentum_3d(d, st, 0); break;
    case BC_VV_MOMENTUM_3D: gor::uv_momentum_3d(d, st, 1); break;
    case BC_SIGMA: gor::sigma_coordinates(d, st); break;
    case BC_WW: gor::ww_momentum_3d(d, st); break;
    case BC_UV_ADVECT_3D: rc = gor::uv_advect_3d(d, m, st); break;
    case BC_STRESSES_3D: gor::stresses_3d(d, st); break;
    case BC_EQSTATE: gor::do_eqstate(d, st); break;
    case BC_SLOW_BOTTOM_FRICTION: gor::slow_bottom_friction(d, st); break;
    case BC_SLOW_TERMS: gor::slow_terms(d, st); break;
    case BC_INTEGRATE_2D: rc = gor::integrate_2d(d, m, st, arg); break;
    case BC_INTEGRATE_3D: rc = gor::integrate_3d(d, m, st, arg); break;
    case BC_GOTM_PARABOLIC: gor::gotm_parabolic(d, st); break;
    case BC_SW_RADIATION: gor::sw_radiation(d, st); break;
    case BC_HOTSTART_POSTINIT: gor::hotstart_postinit(d, st, arg); break;
    case BC_UPDATE_2D_BDY:
      if (st.bdy && st.bdy->nseg() > 0) gor::update_2d_bdy(d, *st.bdy, st.f2, st.par, arg);
      break;
    default: return -2;
  }
  for (int q = 0; q < gor::NPI; ++q) s->ipar[q] = st.ipar[q];
  return rc;
}
}  // extern "C++"

int or_bc_call_d(const or_dom* o, or_bc* s, int which, int arg) { return bc_call<double>(o, s, which, arg); }

// sealevel_nan_check (sealevel.F90:172-314): count and last point (reference indices) of the
// interior elevations that are not below HUGE
long long or_sealevel_nan_check(const or_dom* o, const double* z, int* inan, int* jnan) {
  gor::Dom d = mk(o);
  return gor::sealevel_nan_count(d, z, inan, jnan);
}
int or_bc_call_f(const or_dom* o, or_bc* s, int which, int arg) { return bc_call<float>(o, s, which, arg); }

}  // extern "C"
