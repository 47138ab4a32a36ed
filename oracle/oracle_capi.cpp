// oracle_capi.cpp -- TEST INFRASTRUCTURE ONLY: extern "C" entry points of the CPU oracle
// (getm_oracle.hpp) for the Python test harness (oracle/__init__.py, via ctypes).
// Suffix _d = FP64 (the reference's REALTYPE), _f = FP32.
#include "getm_oracle.hpp"

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

}  // extern "C"
