// adjoint.cuh -- reverse-mode derivative of the tracer step (split advection + implicit vertical
// diffusion), templated on the arithmetic type R. Included by kernels_inst.cuh.
//
// With the limiter branches frozen, every split sweep is linear in the tracer: the interface value
// of a face is fu + A*(fu - fuu) + B*(fd - fu) with A, B fixed by the branch code recorded in the
// forward sweep and by the face's Courant number (recon_code / recon_coef in kernels.cuh), and
// the cell update is f_new = (hio*f - dt*(flux_e - flux_w)*...)/hin. The adjoint kernels apply
// the transpose of that linear map: the cotangent of each face flux is gathered from the two cells
// it updates, spread over the (up to) four cells of its stencil, and each cell collects the
// contributions of the faces whose stencils contain it -- a gather, so the result is deterministic
// and needs no atomics.
#pragma once
#include "kernels.cuh"

namespace gb {

// ---------------------------------------------------------------------------------------------
// Heights before sweeps 2..5 of u/2 v/2 w v/2 u/2 (the Di/hi updates of adv_split_u/v/w, in the
// forward sweeps' expressions). One thread per cell of levels 1..kmax.
template <class R>
__global__ void k_adj_heights(Dev d, R dt, int sub, int has_w, const R* __restrict__ ho, const R* __restrict__ uu,
                              const R* __restrict__ vv, const R* __restrict__ ww,
                              const uint8_t* __restrict__ mupd_u, const uint8_t* __restrict__ mupd_v,
                              const int32_t* __restrict__ az, R* H1, R* H2, R* H3, R* H4) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 1 + blockIdx.z;
  const int ni = d.ni(), nj = d.nj();
  if (ii >= ni || jj >= nj) return;
  const long long c = (long long)ii + (long long)jj * d.sj;
  const long long p = c + (long long)k * d.sk;
  const R dti = R(0.5) * dt;
  const bool upd_u = (ii >= 1 + sub) && (ii <= ni - 2 - sub) && mupd_u[c];
  const bool upd_v = (jj >= 1 + sub) && (jj <= nj - 2 - sub) && mupd_v[c];
  const bool upd_w = has_w && ii < ni - 1 && jj < nj - 1 && az[c] == 1;
  const R dyu = R(d.dy), dxv = R(d.dx), ard1 = R(d.ard1);
  R h = ho[p];
  if (upd_u) h = h - dti * (uu[p] * dyu - uu[p - 1] * dyu) * ard1;
  H1[p] = h;
  R dDv = R(0);
  if (upd_v) {
    dDv = dti * (vv[p] * dxv - vv[p - d.sj] * dxv) * ard1;
    h = h - dDv;
  }
  H2[p] = h;
  if (upd_w) h = h - dt * (ww[p] - ww[p - d.sk]);
  H3[p] = h;
  if (upd_v) h = h - dti * (vv[p] * dxv - vv[p - d.sj] * dxv) * ard1;
  H4[p] = h;
}

// ---------------------------------------------------------------------------------------------
// Adjoint of the u sweep over a row segment of TU cells, for up to NKB levels (the 2D masks are
// staged once). Staged per level: U, DU at cells i0-3 .. i0+TU+1, cotangents and heights at cells
// i0-2 .. i0+TU+1, branch codes of faces i0-2 .. i0+TU.
template <class R, int S>
__global__ void __launch_bounds__(TU) k_adj_sweep_u(Dev d, R dt, R splitfac, R AH, int nk, bool copy0,
                                                    const R* __restrict__ gbar, R* __restrict__ fbar,
                                                    const R* __restrict__ Dio, const R* __restrict__ U,
                                                    const R* __restrict__ DU, const uint8_t* __restrict__ mflux,
                                                    const uint8_t* __restrict__ mupd,
                                                    const uint8_t* __restrict__ code) {
  __shared__ R sU[TU + 5], sDU[TU + 5];
  __shared__ uint8_t sm[TU + 5], su[TU + 4];
  __shared__ R sg[TU + 4], skc[TU + 4], spc[TU + 4];
  __shared__ R sw[4][TU + 3];
  const int t = threadIdx.x;
  const int ni = d.ni();
  const int ii0 = blockIdx.x * TU;
  const long long crow = (long long)blockIdx.y * d.sj;
  const int k0 = blockIdx.z * NKB;
  const int k1 = min(k0 + NKB, nk);
  constexpr int sub = (S == UPSTREAM) ? 0 : 1;
  const R dti = splitfac * dt;
  const R dxf = R(d.dx), dyf = R(d.dy), ard1 = R(d.ard1);
  const R cdx = dti / dxf;
  const bool use_AH = AH > R(0);
  const R kfac = dt * splitfac * dyf * ard1;
  for (int q = t; q < TU + 5; q += TU) {
    const int ii = ii0 - 3 + q;
    sm[q] = (ii >= 0 && ii < ni) ? mflux[crow + ii] : 0;
  }
  for (int q = t; q < TU + 4; q += TU) {
    const int ii = ii0 - 2 + q;
    su[q] = (ii >= 0 && ii < ni && ii >= 1 + sub && ii <= ni - 2 - sub) ? mupd[crow + ii] : 0;
  }
  // level 0 (below the level pointers' origin) is not touched by the sweep: its cotangent passes
  if (copy0 && blockIdx.z == 0 && ii0 + t < ni) fbar[crow - d.sk + ii0 + t] = gbar[crow - d.sk + ii0 + t];
  for (int k = k0; k < k1; ++k) {
    const long long row = crow + (long long)k * d.sk;
    for (int q = t; q < TU + 5; q += TU) {
      const int ii = ii0 - 3 + q;
      const bool ok = ii >= 0 && ii < ni;
      sU[q] = ok ? U[row + ii] : R(0);
      sDU[q] = ok ? DU[row + ii] : R(0);
    }
    __syncthreads();
    // cells q <-> ii = ii0-2+q; U of its east face = sU[q+1], of its west face = sU[q]
    for (int q = t; q < TU + 4; q += TU) {
      const int ii = ii0 - 2 + q;
      R g = R(0), kc = R(0), pc = R(1);
      if (ii >= 0 && ii < ni) {
        g = gbar[row + ii];
        if (su[q]) {
          const R hio = Dio[row + ii];
          const R dD = dti * (sU[q + 1] * dyf - sU[q] * dyf) * ard1;
          const R hin = hio - dD;
          kc = kfac / hin;
          pc = hio / hin;
        }
      }
      sg[q] = g;
      skc[q] = kc;
      spc[q] = pc;
    }
    __syncthreads();
    // faces r <-> fa = ii0-2+r (between cells fa and fa+1); U index r+1, cells r and r+1
    for (int r = t; r < TU + 3; r += TU) {
      const int fa = ii0 - 2 + r;
      R wm1 = R(0), w0 = R(0), w1 = R(0), w2 = R(0);
      if (fa >= sub && fa <= ni - 2 - sub && sm[r + 1]) {
        const R Fb = -sg[r] * skc[r] + sg[r + 1] * skc[r + 1];
        const R Uf = sU[r + 1], DUf = sDU[r + 1];
        const bool pos = Uf > R(0);
        R A = R(0), B = R(0);
        if (S != UPSTREAM && (pos ? sm[r] : sm[r + 2])) {
          const R cfl = face_cfl<R>(pos, Uf, DUf, dti, cdx, dxf);
          recon_coef<R, S>(code[row + fa], cfl, A, B);
        }
        const R FU = Fb * Uf;
        const R cu = FU * (R(1) + A - B), cuu = -FU * A, cd = FU * B;
        if (pos) {
          wm1 = cuu; w0 = cu; w1 = cd;
        } else {
          w0 = cd; w1 = cu; w2 = cuu;
        }
        if (use_AH) {
          const R ka = Fb * AH * DUf / dxf;
          w0 = w0 + ka;
          w1 = w1 - ka;
        }
      }
      sw[0][r] = wm1;
      sw[1][r] = w0;
      sw[2][r] = w1;
      sw[3][r] = w2;
    }
    __syncthreads();
    const int ii = ii0 + t;
    // cell ii: q = t+2; faces ii+1, ii, ii-1, ii-2 <-> r = t+3, t+2, t+1, t
    if (ii < ni) fbar[row + ii] = sg[t + 2] * spc[t + 2] + sw[0][t + 3] + sw[1][t + 2] + sw[2][t + 1] + sw[3][t];
    __syncthreads();
  }
}

// Adjoint of the v sweep over a tile of TVX x TVY cells, for up to NKB levels.
template <class R, int S>
__global__ void __launch_bounds__(TVX * TVY) k_adj_sweep_v(Dev d, R dt, R splitfac, R AH, int nk, bool copy0,
                                                           const R* __restrict__ gbar, R* __restrict__ fbar,
                                                           const R* __restrict__ Dio, const R* __restrict__ V,
                                                           const R* __restrict__ DV,
                                                           const uint8_t* __restrict__ mflux,
                                                           const uint8_t* __restrict__ mupd,
                                                           const uint8_t* __restrict__ code) {
  __shared__ R sV[TVY + 5][TVX], sDV[TVY + 5][TVX];
  __shared__ uint8_t sm[TVY + 5][TVX], su[TVY + 4][TVX];
  __shared__ R sg[TVY + 4][TVX], skc[TVY + 4][TVX], spc[TVY + 4][TVX];
  __shared__ R sw[4][TVY + 3][TVX];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int ni = d.ni(), nj = d.nj();
  const int ii = blockIdx.x * TVX + tx;
  const int jj0 = blockIdx.y * TVY;
  const int k0 = blockIdx.z * NKB;
  const int k1 = min(k0 + NKB, nk);
  const bool iok = ii < ni;
  const long long sj = d.sj;
  constexpr int sub = (S == UPSTREAM) ? 0 : 1;
  const R dti = splitfac * dt;
  const R dxf = R(d.dy), dyf = R(d.dx), ard1 = R(d.ard1);  // DYV, DXV
  const R cdx = dti / dxf;
  const bool use_AH = AH > R(0);
  const R kfac = dt * splitfac * dyf * ard1;
  for (int q = ty; q < TVY + 5; q += TVY) {
    const int jj = jj0 - 3 + q;
    sm[q][tx] = (iok && jj >= 0 && jj < nj) ? mflux[(long long)jj * sj + ii] : 0;
  }
  for (int q = ty; q < TVY + 4; q += TVY) {
    const int jj = jj0 - 2 + q;
    su[q][tx] = (iok && jj >= 0 && jj < nj && jj >= 1 + sub && jj <= nj - 2 - sub) ? mupd[(long long)jj * sj + ii]
                                                                                   : 0;
  }
  // level 0 (below the level pointers' origin) is not touched by the sweep: its cotangent passes
  if (copy0 && blockIdx.z == 0 && iok && jj0 + ty < nj) {
    const long long c0 = (long long)(jj0 + ty) * sj + ii - d.sk;
    fbar[c0] = gbar[c0];
  }
  for (int k = k0; k < k1; ++k) {
    const long long lev = (long long)k * d.sk;
    for (int q = ty; q < TVY + 5; q += TVY) {
      const int jj = jj0 - 3 + q;
      const bool ok = iok && jj >= 0 && jj < nj;
      const long long c = lev + (long long)jj * sj + ii;
      sV[q][tx] = ok ? V[c] : R(0);
      sDV[q][tx] = ok ? DV[c] : R(0);
    }
    __syncthreads();
    for (int q = ty; q < TVY + 4; q += TVY) {
      const int jj = jj0 - 2 + q;
      R g = R(0), kc = R(0), pc = R(1);
      if (iok && jj >= 0 && jj < nj) {
        const long long c = lev + (long long)jj * sj + ii;
        g = gbar[c];
        if (su[q][tx]) {
          const R hio = Dio[c];
          const R dD = dti * (sV[q + 1][tx] * dyf - sV[q][tx] * dyf) * ard1;
          const R hin = hio - dD;
          kc = kfac / hin;
          pc = hio / hin;
        }
      }
      sg[q][tx] = g;
      skc[q][tx] = kc;
      spc[q][tx] = pc;
    }
    __syncthreads();
    for (int r = ty; r < TVY + 3; r += TVY) {
      const int fa = jj0 - 2 + r;
      R wm1 = R(0), w0 = R(0), w1 = R(0), w2 = R(0);
      if (iok && fa >= sub && fa <= nj - 2 - sub && sm[r + 1][tx]) {
        const R Fb = -sg[r][tx] * skc[r][tx] + sg[r + 1][tx] * skc[r + 1][tx];
        const R Vf = sV[r + 1][tx], DVf = sDV[r + 1][tx];
        const bool pos = Vf > R(0);
        R A = R(0), B = R(0);
        if (S != UPSTREAM && (pos ? sm[r][tx] : sm[r + 2][tx])) {
          const R cfl = face_cfl<R>(pos, Vf, DVf, dti, cdx, dxf);
          recon_coef<R, S>(code[lev + (long long)fa * sj + ii], cfl, A, B);
        }
        const R FV = Fb * Vf;
        const R cu = FV * (R(1) + A - B), cuu = -FV * A, cd = FV * B;
        if (pos) {
          wm1 = cuu; w0 = cu; w1 = cd;
        } else {
          w0 = cd; w1 = cu; w2 = cuu;
        }
        if (use_AH) {
          const R ka = Fb * AH * DVf / dxf;
          w0 = w0 + ka;
          w1 = w1 - ka;
        }
      }
      sw[0][r][tx] = wm1;
      sw[1][r][tx] = w0;
      sw[2][r][tx] = w1;
      sw[3][r][tx] = w2;
    }
    __syncthreads();
    const int jj = jj0 + ty;
    if (iok && jj < nj)
      fbar[lev + (long long)jj * sj + ii] = sg[ty + 2][tx] * spc[ty + 2][tx] + sw[0][ty + 3][tx] +
                                            sw[1][ty + 2][tx] + sw[2][ty + 1][tx] + sw[3][ty][tx];
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------
// Adjoint of the vertical sweep, one thread per column of the haloed plane; columns the forward
// sweep does not touch (and levels it does not update) pass the cotangent through. Faces are
// visited bottom-up with four rolling accumulators (cells k-1 .. k+2 of face k); cell k-1 is
// complete once face k has been added.
template <class R, int S>
__global__ void __launch_bounds__(128) k_adj_sweep_w(Dev d, R dt, R splitfac, int kshift, const R* __restrict__ gbar,
                                                     R* __restrict__ fbar, const R* __restrict__ hi,
                                                     const R* __restrict__ ww, const int32_t* __restrict__ az,
                                                     const uint8_t* __restrict__ code) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  if (ii >= d.ni() || jj >= d.nj()) return;
  const long long c = (long long)ii + (long long)jj * d.sj;
  const int kmax = d.kmax;
  const long long sk = d.sk;
  if (!(ii < d.ni() - 1 && jj < d.nj() - 1 && az[c] == 1)) {
    for (int k = 0; k <= kmax; ++k) fbar[c + k * sk] = gbar[c + k * sk];
    return;
  }
  const R dti = splitfac * dt;
  const int kup = kmax - kshift;  // levels 1..kup are updated
  auto G = [&](int k) -> R { return (k >= 0 && k <= kmax) ? gbar[c + k * sk] : R(0); };
  auto HI = [&](int k) -> R { return (k >= 0 && k <= kmax) ? hi[c + k * sk] : R(0); };
  auto W = [&](int k) -> R { return (k >= 0 && k <= kmax) ? ww[c + k * sk] : R(0); };
  // level data: g, hio, kc (flux cotangent factor), pc (pass-through factor)
  auto level = [&](int k, R wk, R wkm1, R hio, R& kc, R& pc) {
    kc = R(0);
    pc = R(1);
    if (k >= 1 && k <= kup) {
      const R hin = hio - dti * (wk - wkm1);
      kc = dt * splitfac / hin;
      pc = hio / hin;
    }
  };
  // window: cell k-1 (gm, pcm), cell k (g0, h0, kc0, pc0, w0 = w(k)), cell k+1 (g1, h1, kc1, pc1, w1)
  R wkm1 = W(-1);
  R w0 = W(0), w1 = W(1);
  R g0 = G(0), g1 = G(1), h0 = HI(0), h1 = HI(1);
  R kc0, pc0, kc1, pc1;
  level(0, w0, wkm1, h0, kc0, pc0);
  level(1, w1, w0, h1, kc1, pc1);
  R gm = R(0), pcm = R(1);
  R am1 = R(0), a0 = R(0), a1 = R(0), a2 = R(0);  // cells k-1, k, k+1, k+2
  for (int k = 0; k <= kmax + 1; ++k) {
    // face k between cells k and k+1
    if (k >= 1 - kshift && k <= kmax - 1) {
      const R Fb = -g0 * kc0 + g1 * kc1;
      const bool pos = w0 > R(0);
      R A = R(0), B = R(0);
      if (S != UPSTREAM && (pos ? (k > 1 - kshift) : (k < kmax - 1))) {
        const R cfl = wface_cfl<R>(w0, dti, h0, h1);
        recon_coef<R, S>(code[c + k * sk], cfl, A, B);
      }
      const R FW = Fb * w0;
      const R cu = FW * (R(1) + A - B), cuu = -FW * A, cdn = FW * B;
      if (pos) {
        am1 = am1 + cuu; a0 = a0 + cu; a1 = a1 + cdn;
      } else {
        a0 = a0 + cdn; a1 = a1 + cu; a2 = a2 + cuu;
      }
    }
    if (k >= 1) fbar[c + (k - 1) * sk] = gm * pcm + am1;
    // shift the window up by one level
    gm = g0; pcm = pc0;
    am1 = a0; a0 = a1; a1 = a2; a2 = R(0);
    const R w2 = W(k + 2), g2 = G(k + 2), h2 = HI(k + 2);
    R kc2, pc2;
    level(k + 2, w2, w1, h2, kc2, pc2);
    g0 = g1; h0 = h1; kc0 = kc1; pc0 = pc1; w0 = w1;
    g1 = g2; h1 = h2; kc1 = kc2; pc1 = pc2; w1 = w2;
  }
}

// ---------------------------------------------------------------------------------------------
// Adjoint of the implicit vertical diffusion (salinity.F90:348-389). The forward step solves
// A S_new = B S_old with the symmetric tridiagonal matrices
//   A = diag(h) - D(an),  B = diag(h) + D(ao),  (D(a) S)_k = a_k (S_{k+1}-S_k) - a_{k-1} (S_k-S_{k-1}),
//   an_k = cn (nuh_k+avmol)/(h_k+h_{k+1}),  ao_k = co (nuh_k+avmol)/(h_k+h_{k+1})  (interface k).
// So with lambda = A^{-1} fbar:  gbar = B lambda, and
//   nubar_k += (lambda_k - lambda_{k+1}) * (co (S_old,k+1 - S_old,k) + cn (S_new,k+1 - S_new,k))/(h_k+h_{k+1}).
// One thread per column of the haloed plane; columns without a solve pass fbar through.
template <class R>
__global__ void __launch_bounds__(128) k_adj_vdiff(Dev d, R dt, R cnpar, R avmol, const R* __restrict__ fbar,
                                                   R* __restrict__ gbar, R* nubar, const R* __restrict__ g,
                                                   const R* __restrict__ Sn, const R* __restrict__ hn,
                                                   const R* __restrict__ nuh, const int32_t* __restrict__ az,
                                                   R* RUs, R* QUs) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  if (ii >= d.ni() || jj >= d.nj()) return;
  const long long c = (long long)ii + (long long)jj * d.sj;
  const int kmax = d.kmax;
  const long long sk = d.sk;
  const int i = ii + d.imin - HALO, j = jj + d.jmin - HALO;
  const bool solved = kmax > 1 && i >= d.imin && i <= d.imax && j >= d.jmin && j <= d.jmax && az[c] == 1;
  if (!solved) {
    for (int k = 0; k <= kmax; ++k) gbar[c + k * sk] = fbar[c + k * sk];
    return;
  }
  auto L = [&](const R* a, int k) -> R { return a[c + k * sk]; };
  const R co = R(2) * (R(1) - cnpar) * dt;
  const R cn = R(2) * cnpar * dt;
  // elimination from the surface down (tridiagonal.F90:35-43 order), right-hand side fbar
  int k = kmax;
  R hnk = L(hn, k), hnkm1 = L(hn, k - 1);
  R an_km1 = cn * (L(nuh, k - 1) + avmol) / (hnk + hnkm1);
  R ru, qu;
  {
    const R a1 = -an_km1, a2 = hnk + an_km1;
    ru = a1 / a2;
    qu = L(fbar, k) / a2;
    RUs[c + k * sk] = ru;
    QUs[c + k * sk] = qu;
  }
  // the next level's loads are issued one iteration ahead (the elimination is a serial chain)
  R hn_n = L(hn, kmax - 2), nu_n = L(nuh, kmax - 2), fb_n = L(fbar, kmax - 1);
  for (k = kmax - 1; k >= 2; --k) {
    const R an_k = an_km1;
    hnk = hnkm1;
    hnkm1 = hn_n;
    const R nuv = nu_n, fbk = fb_n;
    if (k >= 3) {
      hn_n = L(hn, k - 2);
      nu_n = L(nuh, k - 2);
    }
    fb_n = L(fbar, k - 1);
    an_km1 = cn * (nuv + avmol) / (hnk + hnkm1);
    const R a3 = -an_k, a1 = -an_km1, a2 = hnk + an_k + an_km1;
    const R den = a2 - a3 * ru;
    ru = a1 / den;
    qu = (fbk - a3 * qu) / den;
    RUs[c + k * sk] = ru;
    QUs[c + k * sk] = qu;
  }
  R lam1;
  {
    const R an_k = an_km1;
    const R a3 = -an_k, a2 = hnkm1 + an_k;
    lam1 = (L(fbar, 1) - a3 * qu) / (a2 - a3 * ru);
  }
  // back substitution upwards, lambda(k) = qu(k) - ru(k) lambda(k-1), fused with the output pass:
  // once lambda(k) is known, level k-1 is complete --
  //   gbar(k-1) = h(k-1) l(k-1) + ao(k-1) (l(k) - l(k-1)) - ao(k-2) (l(k-1) - l(k-2)),
  //   nubar(k-1) += (l(k-1) - l(k)) (co (g(k) - g(k-1)) + cn (Sn(k) - Sn(k-1))) / (h(k-1) + h(k)).
  gbar[c] = L(fbar, 0);
  R lm = R(0), l0 = lam1;     // lambda(k-2), lambda(k-1)
  R ao_m = R(0);              // ao of the interface below level k-1
  R hk = L(hn, 1), gk = L(g, 1), sk0 = L(Sn, 1);  // h, g, Sn at level k-1
  // level k's inputs, loaded one iteration ahead
  R q_n = QUs[c + 2 * sk], r_n = RUs[c + 2 * sk], h_n = L(hn, 2), g_n = L(g, 2), s_n = L(Sn, 2), v_n = L(nuh, 1);
  for (k = 2; k <= kmax + 1; ++k) {
    R l1 = R(0), ao_k = R(0), hk1 = R(0), gk1 = R(0), sk1 = R(0);
    if (k <= kmax) {
      const R qk = q_n, rk = r_n, nuk = v_n;
      hk1 = h_n;
      gk1 = g_n;
      sk1 = s_n;
      if (k < kmax) {
        q_n = QUs[c + (k + 1) * sk];
        r_n = RUs[c + (k + 1) * sk];
        h_n = L(hn, k + 1);
        g_n = L(g, k + 1);
        s_n = L(Sn, k + 1);
        v_n = L(nuh, k);
      }
      l1 = qk - rk * l0;
      const R hs = hk + hk1;
      const R nu = nuk + avmol;
      ao_k = co * nu / hs;
      const R dl = l0 - l1;
      nubar[c + (k - 1) * sk] = nubar[c + (k - 1) * sk] + dl * (co * (gk1 - gk) + cn * (sk1 - sk0)) / hs;
    }
    gbar[c + (k - 1) * sk] = hk * l0 + ao_k * (l1 - l0) - ao_m * (l0 - lm);
    lm = l0;
    l0 = l1;
    ao_m = ao_k;
    hk = hk1;
    gk = gk1;
    sk0 = sk1;
  }
}

// ---------------------------------------------------------------------------------------------
// launchers

template <class R>
int run_adj_heights(const Dev& d, cudaStream_t s, R dt, int sub, bool has_w, const R* ho, const R* uu,
                    const R* vv, const R* ww, const uint8_t* mupd_u, const uint8_t* mupd_v,
                    const int32_t* az, R* H1, R* H2, R* H3, R* H4) {
  if (d.kmax < 1) return 0;
  dim3 blk(64, 4, 1);
  dim3 grd((d.ni() + blk.x - 1) / blk.x, (d.nj() + blk.y - 1) / blk.y, d.kmax);
  k_adj_heights<R><<<grd, blk, 0, s>>>(d, dt, sub, has_w ? 1 : 0, ho, uu, vv, ww, mupd_u, mupd_v, az, H1, H2,
                                       H3, H4);
  return (int)cudaGetLastError();
}

template <class R, int DIR>
int run_adj_sweep_h(const Dev& d, cudaStream_t s, int nk, R dt, R splitfac, int scheme, R AH, const R* gbar,
                    R* fbar, const R* Dio, const R* U, const R* DU, const uint8_t* mflux, const uint8_t* mupd,
                    const uint8_t* code, bool copy0) {
  if (nk <= 0) return 0;
  return dispatch_scheme(scheme, [&](auto sc) {
    constexpr int S = decltype(sc)::value;
    const int nz = (nk + NKB - 1) / NKB;
    if (DIR == 0) {
      dim3 grd((d.ni() + TU - 1) / TU, d.nj(), nz);
      k_adj_sweep_u<R, S><<<grd, TU, 0, s>>>(d, dt, splitfac, AH, nk, copy0, gbar, fbar, Dio, U, DU, mflux, mupd,
                                             code);
    } else {
      dim3 blk(TVX, TVY, 1);
      dim3 grd((d.ni() + TVX - 1) / TVX, (d.nj() + TVY - 1) / TVY, nz);
      k_adj_sweep_v<R, S><<<grd, blk, 0, s>>>(d, dt, splitfac, AH, nk, copy0, gbar, fbar, Dio, U, DU, mflux, mupd,
                                              code);
    }
    return (int)cudaGetLastError();
  });
}

template <class R>
int run_adj_sweep_w(const Dev& d, cudaStream_t s, R dt, R splitfac, int scheme, int kshift, const R* gbar,
                    R* fbar, const R* hi, const R* ww, const int32_t* az, const uint8_t* code) {
  return dispatch_scheme(scheme, [&](auto sc) {
    constexpr int S = decltype(sc)::value;
    dim3 blk(64, 2, 1);
    dim3 grd((d.ni() + blk.x - 1) / blk.x, (d.nj() + blk.y - 1) / blk.y, 1);
    k_adj_sweep_w<R, S><<<grd, blk, 0, s>>>(d, dt, splitfac, kshift, gbar, fbar, hi, ww, az, code);
    return (int)cudaGetLastError();
  });
}

template <class R>
int run_adj_vdiff(const Dev& d, cudaStream_t s, R dt, R cnpar, R avmol, const R* fbar, R* gbar, R* nubar,
                  const R* g, const R* Sn, const R* hn, const R* nuh, const int32_t* az, R* rus, R* qus) {
  dim3 blk(32, 4, 1);
  dim3 grd((d.ni() + blk.x - 1) / blk.x, (d.nj() + blk.y - 1) / blk.y, 1);
  k_adj_vdiff<R><<<grd, blk, 0, s>>>(d, dt, cnpar, avmol, fbar, gbar, nubar, g, Sn, hn, nuh, az, rus, qus);
  return (int)cudaGetLastError();
}

}  // namespace gb
