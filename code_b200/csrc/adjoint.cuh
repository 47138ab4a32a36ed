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
#include "sweeps_vec.cuh"

namespace gb {

// ---------------------------------------------------------------------------------------------
// Transposed cell and face operations of a horizontal split sweep, shared by the tile and the
// vectorised adjoint sweeps so that both round identically.
//  * adj_cell: the factors of cell (hio, Uhi, Ulo): kc = dt*splitfac*dyf*ard1/hin (the cotangent
//    of the flux difference per unit cotangent of the new value) and pc = hio/hin (pass-through).
//  * adj_face: the weights w[0..3] that face fa spreads its flux cotangent Fb over the cells
//    fa-1, fa, fa+1, fa+2 (frozen limiter branch `code`, optional AH diffusion).
template <class R>
__device__ __forceinline__ void adj_cell(R dti, R dyf, R ard1, R kfac, R hio, R Uhi, R Ulo, R& kc, R& pc) {
  const R dD = dti * (Uhi * dyf - Ulo * dyf) * ard1;
  const R hin = hio - dD;
  kc = kfac / hin;
  pc = hio / hin;
}
template <class R, int S>
__device__ __forceinline__ void adj_face(R Fb, R Uf, R DUf, bool mup, bool mdn, uint8_t code, R dti, R cdx, R dxf,
                                         R AH, bool use_AH, R (&w)[4]) {
  const bool pos = Uf > R(0);
  R A = R(0), B = R(0);
  if (S != UPSTREAM && (pos ? mup : mdn)) {
    const R cfl = face_cfl<R>(pos, Uf, DUf, dti, cdx, dxf);
    recon_coef<R, S>(code, cfl, A, B);
  }
  const R FU = Fb * Uf;
  const R cu = FU * (R(1) + A - B), cuu = -FU * A, cd = FU * B;
  if (pos) {
    w[0] = cuu; w[1] = cu; w[2] = cd; w[3] = R(0);
  } else {
    w[0] = R(0); w[1] = cd; w[2] = cu; w[3] = cuu;
  }
  if (use_AH) {
    const R ka = Fb * AH * DUf / dxf;
    w[1] = w[1] + ka;
    w[2] = w[2] - ka;
  }
}

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
// i0-2 .. i0+TU+1, branch codes of faces i0-2 .. i0+TU. Levels are double-buffered: the cp.async
// copies (and the code bytes, through registers) of level k+1 are issued before level k is
// computed.
template <class R, int S>
__global__ void __launch_bounds__(TU) k_adj_sweep_u(Dev d, R dt, R splitfac, R AH, int nk, bool copy0,
                                                    const R* __restrict__ gbar, R* __restrict__ fbar,
                                                    const R* __restrict__ Dio, const R* __restrict__ U,
                                                    const R* __restrict__ DU, const uint8_t* __restrict__ mflux,
                                                    const uint8_t* __restrict__ mupd,
                                                    const uint8_t* __restrict__ code) {
  __shared__ R sU[2][TU + 5], sDU[2][TU + 5];
  __shared__ R sG[2][TU + 4], sD[2][TU + 4];
  __shared__ uint8_t scd[2][TU + 3];
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
  __syncthreads();  // su is read by the staging below
  // level 0 (below the level pointers' origin) is not touched by the sweep: its cotangent passes
  if (copy0 && blockIdx.z == 0 && ii0 + t < ni) fbar[crow - d.sk + ii0 + t] = gbar[crow - d.sk + ii0 + t];
  auto stage = [&](int k, int b) {
    const long long row = crow + (long long)k * d.sk;
    for (int q = t; q < TU + 5; q += TU) {
      const int ii = ii0 - 3 + q;
      if (ii >= 0 && ii < ni) {
        cp_async(&sU[b][q], U + row + ii);
        cp_async(&sDU[b][q], DU + row + ii);
      } else {
        sU[b][q] = R(0);
        sDU[b][q] = R(0);
      }
    }
    for (int q = t; q < TU + 4; q += TU) {
      const int ii = ii0 - 2 + q;
      if (ii >= 0 && ii < ni) {
        cp_async(&sG[b][q], gbar + row + ii);
        if (su[q]) cp_async(&sD[b][q], Dio + row + ii);
      } else {
        sG[b][q] = R(0);
      }
    }
    cp_async_commit();
  };
  // code bytes of the faces r = t and r = t + TU (t < 3) of a level, through registers
  auto codes = [&](int k, uint8_t& c0, uint8_t& c1) {
    const long long row = crow + (long long)k * d.sk;
    const int fa0 = ii0 - 2 + t, fa1 = fa0 + TU;
    c0 = (S != UPSTREAM && fa0 >= 0 && fa0 < ni) ? code[row + fa0] : 0;
    c1 = (S != UPSTREAM && t < 3 && fa1 < ni) ? code[row + fa1] : 0;
  };
  uint8_t cn0 = 0, cn1 = 0;
  if (k0 < k1) {
    stage(k0, 0);
    codes(k0, cn0, cn1);
    scd[0][t] = cn0;
    if (t < 3) scd[0][TU + t] = cn1;
  }
  for (int k = k0, b = 0; k < k1; ++k, b ^= 1) {
    const long long row = crow + (long long)k * d.sk;
    if (k + 1 < k1) {
      stage(k + 1, b ^ 1);
      codes(k + 1, cn0, cn1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    // cells q <-> ii = ii0-2+q; U of its east face = sU[q+1], of its west face = sU[q]
    for (int q = t; q < TU + 4; q += TU) {
      R kc = R(0), pc = R(1);
      if (su[q]) adj_cell<R>(dti, dyf, ard1, kfac, sD[b][q], sU[b][q + 1], sU[b][q], kc, pc);
      sg[q] = sG[b][q];
      skc[q] = kc;
      spc[q] = pc;
    }
    __syncthreads();
    // faces r <-> fa = ii0-2+r (between cells fa and fa+1); U index r+1, cells r and r+1
    for (int r = t; r < TU + 3; r += TU) {
      const int fa = ii0 - 2 + r;
      R w[4] = {R(0), R(0), R(0), R(0)};
      if (fa >= sub && fa <= ni - 2 - sub && sm[r + 1]) {
        const R Fb = -sg[r] * skc[r] + sg[r + 1] * skc[r + 1];
        adj_face<R, S>(Fb, sU[b][r + 1], sDU[b][r + 1], sm[r] != 0, sm[r + 2] != 0, scd[b][r], dti, cdx, dxf, AH,
                       use_AH, w);
      }
      sw[0][r] = w[0];
      sw[1][r] = w[1];
      sw[2][r] = w[2];
      sw[3][r] = w[3];
    }
    __syncthreads();
    const int ii = ii0 + t;
    // cell ii: q = t+2; faces ii+1, ii, ii-1, ii-2 <-> r = t+3, t+2, t+1, t
    if (ii < ni) fbar[row + ii] = sg[t + 2] * spc[t + 2] + sw[0][t + 3] + sw[1][t + 2] + sw[2][t + 1] + sw[3][t];
    if (k + 1 < k1) {  // the codes of level k+1 (buffer b^1 was last read before this level's barriers)
      scd[b ^ 1][t] = cn0;
      if (t < 3) scd[b ^ 1][TU + t] = cn1;
    }
    __syncthreads();
  }
}

// Adjoint of the v sweep over a tile of TVX x TVY cells, for up to NKB levels, double-buffered
// like the u sweep.
template <class R, int S>
__global__ void __launch_bounds__(TVX * TVY) k_adj_sweep_v(Dev d, R dt, R splitfac, R AH, int nk, bool copy0,
                                                           const R* __restrict__ gbar, R* __restrict__ fbar,
                                                           const R* __restrict__ Dio, const R* __restrict__ V,
                                                           const R* __restrict__ DV,
                                                           const uint8_t* __restrict__ mflux,
                                                           const uint8_t* __restrict__ mupd,
                                                           const uint8_t* __restrict__ code) {
  __shared__ R sV[2][TVY + 5][TVX], sDV[2][TVY + 5][TVX];
  __shared__ R sG[2][TVY + 4][TVX], sD[2][TVY + 4][TVX];
  __shared__ uint8_t scd[2][TVY + 3][TVX];
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
  auto stage = [&](int k, int b) {
    const long long lev = (long long)k * d.sk;
    for (int q = ty; q < TVY + 5; q += TVY) {
      const int jj = jj0 - 3 + q;
      if (iok && jj >= 0 && jj < nj) {
        const long long c = lev + (long long)jj * sj + ii;
        cp_async(&sV[b][q][tx], V + c);
        cp_async(&sDV[b][q][tx], DV + c);
      } else {
        sV[b][q][tx] = R(0);
        sDV[b][q][tx] = R(0);
      }
    }
    for (int q = ty; q < TVY + 4; q += TVY) {
      const int jj = jj0 - 2 + q;
      if (iok && jj >= 0 && jj < nj) {
        const long long c = lev + (long long)jj * sj + ii;
        cp_async(&sG[b][q][tx], gbar + c);
        if (su[q][tx]) cp_async(&sD[b][q][tx], Dio + c);
      } else {
        sG[b][q][tx] = R(0);
      }
    }
    cp_async_commit();
  };
  // code bytes of the face rows r = ty and r = ty + TVY (ty < 3) of a level, through registers
  auto codes = [&](int k, uint8_t& c0, uint8_t& c1) {
    const long long lev = (long long)k * d.sk;
    const int fa0 = jj0 - 2 + ty, fa1 = fa0 + TVY;
    c0 = (S != UPSTREAM && iok && fa0 >= 0 && fa0 < nj) ? code[lev + (long long)fa0 * sj + ii] : 0;
    c1 = (S != UPSTREAM && iok && ty < 3 && fa1 < nj) ? code[lev + (long long)fa1 * sj + ii] : 0;
  };
  uint8_t cn0 = 0, cn1 = 0;
  if (k0 < k1) {
    stage(k0, 0);
    codes(k0, cn0, cn1);
    scd[0][ty][tx] = cn0;
    if (ty < 3) scd[0][TVY + ty][tx] = cn1;
  }
  for (int k = k0, b = 0; k < k1; ++k, b ^= 1) {
    const long long lev = (long long)k * d.sk;
    if (k + 1 < k1) {
      stage(k + 1, b ^ 1);
      codes(k + 1, cn0, cn1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    for (int q = ty; q < TVY + 4; q += TVY) {
      R kc = R(0), pc = R(1);
      if (su[q][tx]) adj_cell<R>(dti, dyf, ard1, kfac, sD[b][q][tx], sV[b][q + 1][tx], sV[b][q][tx], kc, pc);
      sg[q][tx] = sG[b][q][tx];
      skc[q][tx] = kc;
      spc[q][tx] = pc;
    }
    __syncthreads();
    for (int r = ty; r < TVY + 3; r += TVY) {
      const int fa = jj0 - 2 + r;
      R w[4] = {R(0), R(0), R(0), R(0)};
      if (iok && fa >= sub && fa <= nj - 2 - sub && sm[r + 1][tx]) {
        const R Fb = -sg[r][tx] * skc[r][tx] + sg[r + 1][tx] * skc[r + 1][tx];
        adj_face<R, S>(Fb, sV[b][r + 1][tx], sDV[b][r + 1][tx], sm[r][tx] != 0, sm[r + 2][tx] != 0, scd[b][r][tx],
                       dti, cdx, dxf, AH, use_AH, w);
      }
      sw[0][r][tx] = w[0];
      sw[1][r][tx] = w[1];
      sw[2][r][tx] = w[2];
      sw[3][r][tx] = w[3];
    }
    __syncthreads();
    const int jj = jj0 + ty;
    if (iok && jj < nj)
      fbar[lev + (long long)jj * sj + ii] = sg[ty + 2][tx] * spc[ty + 2][tx] + sw[0][ty + 3][tx] +
                                            sw[1][ty + 2][tx] + sw[2][ty + 1][tx] + sw[3][ty][tx];
    if (k + 1 < k1) {
      scd[b ^ 1][ty][tx] = cn0;
      if (ty < 3) scd[b ^ 1][TVY + ty][tx] = cn1;
    }
    __syncthreads();
  }
}

// Vectorised adjoint of the u sweep (FP32, 16-byte aligned layouts): the lane layout of
// k_sweep_u_vec -- a warp covers 32 float4 vectors of a row and lanes 1..30 own their cells. A
// lane computes the factors of its cells and the weights of their left faces c0-1 .. c0+N-2; the
// gather of a cell takes the weights of faces c+1, c, c-1, c-2, the outer ones by shuffles from
// the neighbouring lanes. Levels are staged two ahead by cp.async like the forward sweep.
template <class R, int S>
__global__ void __launch_bounds__(32 * UWB) k_adj_sweep_u_vec(Dev d, R dt, R splitfac, R AH, int nk, bool copy0,
                                                            const R* __restrict__ gbar, R* __restrict__ fbar,
                                                            const R* __restrict__ Dio, const R* __restrict__ U,
                                                            const R* __restrict__ DU,
                                                            const uint8_t* __restrict__ mflux,
                                                            const uint8_t* __restrict__ mupd,
                                                            const uint8_t* __restrict__ code) {
  static_assert(sizeof(R) == 4, "vectorised adjoint sweeps are FP32");
  constexpr int N = 4;
  constexpr int NA = 5;  // gbar, Dio, U, DU, codes
  constexpr int sub = (S == UPSTREAM) ? 0 : 1;
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ VecPack<R, N> sbuf[VST][NA][32 * UWB];
  const int lane = threadIdx.x;
  const int tid = threadIdx.y * 32 + lane;
  const int ni = d.ni();
  const int seg = blockIdx.x * UWB + threadIdx.y;
  const int s0 = seg * UOWN * N;
  if (s0 >= ni) return;  // whole warp (no barrier in this kernel)
  const int c0 = s0 + (lane - 1) * N;
  const bool act = c0 >= 0 && c0 < ni;
  const int navail = ni - c0;
  const bool full = act && navail >= N;
  const int vbytes = act ? (full ? N : navail) * (int)sizeof(R) : 0;
  const bool own = act && lane >= 1 && lane <= UOWN;
  const long long crow = (long long)blockIdx.y * d.sj;
  const int k0 = blockIdx.z * NKB;
  const int k1 = min(k0 + NKB, nk);
  const long long cc = act ? c0 : 0;
  const R dti = splitfac * dt;
  const R dxf = R(d.dx), dyf = R(d.dy), ard1 = R(d.ard1);
  const R cdx = dti / dxf;
  const bool use_AH = AH > R(0);
  const R kfac = dt * splitfac * dyf * ard1;
  // masks: flux masks of cells c0-2 .. c0+N-1, update masks of the lane's cells
  uint32_t mfw = 0, muw = 0;
  if (act) {
    mfw = ld_mask_w<N>(mflux + crow + c0, full, navail);
    muw = ld_mask_w<N>(mupd + crow + c0, full, navail);
  }
  const uint32_t mfl = __shfl_up_sync(FULL, mfw, 1);
  bool mfx[N + 2], su[N];
  mfx[0] = mbit(mfl, N - 2);
  mfx[1] = mbit(mfl, N - 1);
#pragma unroll
  for (int m = 0; m < N; ++m) {
    mfx[m + 2] = mbit(mfw, m);
    const int c = c0 + m;
    su[m] = act && m < navail && mbit(muw, m) && c >= 1 + sub && c <= ni - 2 - sub;
  }
  if (copy0 && blockIdx.z == 0 && own) {  // level 0 passes (not touched by the sweep)
    R v[N];
    ld_row<R, N>(gbar + crow - d.sk + c0, full, navail, v);
    st_row<R, N>(fbar + crow - d.sk + c0, full, navail, v);
  }
  auto issue = [&](int k, int st) {
    if (k < k1) {
      const long long p = crow + (long long)k * d.sk + cc;
      cp_async16(&sbuf[st][0][tid], gbar + p, vbytes);
      cp_async16(&sbuf[st][1][tid], Dio + p, vbytes);
      cp_async16(&sbuf[st][2][tid], U + p, vbytes);
      cp_async16(&sbuf[st][3][tid], DU + p, vbytes);
      if (S != UPSTREAM) {
        const int cb = act ? (full ? N : navail) : 0;
        if (cb == N) cp_async(reinterpret_cast<float*>(&sbuf[st][4][tid]), reinterpret_cast<const float*>(code + p));
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
    R g[N], hio[N], u[N], du[N];
    lds_vec<R, N>(sbuf[st][0][tid], g);
    lds_vec<R, N>(sbuf[st][1][tid], hio);
    lds_vec<R, N>(sbuf[st][2][tid], u);
    lds_vec<R, N>(sbuf[st][3][tid], du);
    uint32_t cw = 0;
    if (S != UPSTREAM) {
      if (full) {
        cw = *reinterpret_cast<const uint32_t*>(&sbuf[st][4][tid]);
      } else if (act) {
#pragma unroll
        for (int m = 0; m < N; ++m)
          if (m < navail) cw |= (uint32_t)code[p + m] << (8 * m);
      }
    }
    st = st == VST - 1 ? 0 : st + 1;
    const R uL = __shfl_up_sync(FULL, u[N - 1], 1);
    // cell factors
    R kc[N + 1], pc[N], gg[N + 1];  // index m+1 = cell c0+m; index 0 = cell c0-1 (left lane)
#pragma unroll
    for (int m = 0; m < N; ++m) {
      R kcm = R(0), pcm = R(1);
      if (su[m]) adj_cell<R>(dti, dyf, ard1, kfac, hio[m], u[m], m == 0 ? uL : u[m - 1], kcm, pcm);
      kc[m + 1] = kcm;
      pc[m] = pcm;
      gg[m + 1] = g[m];
    }
    kc[0] = __shfl_up_sync(FULL, kc[N], 1);
    gg[0] = __shfl_up_sync(FULL, gg[N], 1);
    const uint32_t cl = __shfl_up_sync(FULL, cw, 1);
    const R duL = __shfl_up_sync(FULL, du[N - 1], 1);
    // weights of the left faces fa = c0+m-1 (cells fa, fa+1 = index m, m+1)
    R w[N][4];
#pragma unroll
    for (int m = 0; m < N; ++m) {
      const int fa = c0 + m - 1;
#pragma unroll
      for (int q = 0; q < 4; ++q) w[m][q] = R(0);
      if (act && fa >= sub && fa <= ni - 2 - sub && mfx[m + 1]) {
        const R Fb = -gg[m] * kc[m] + gg[m + 1] * kc[m + 1];
        const uint8_t cd = (uint8_t)((m == 0 ? (cl >> (8 * (N - 1))) : (cw >> (8 * (m - 1)))) & 0xffu);
        adj_face<R, S>(Fb, m == 0 ? uL : u[m - 1], m == 0 ? duL : du[m - 1], mfx[m], mfx[m + 2], cd, dti, cdx, dxf,
                       AH, use_AH, w[m]);
      }
    }
    // neighbours' weights: wm1 of the next lane's faces 0 and 1, w0 of its face 0, w2 of the
    // previous lane's last face
    const R nm0 = __shfl_down_sync(FULL, w[0][0], 1), nm1 = __shfl_down_sync(FULL, w[1][0], 1);
    const R n00 = __shfl_down_sync(FULL, w[0][1], 1);
    const R p2 = __shfl_up_sync(FULL, w[N - 1][3], 1);
    if (!own) continue;
    R out[N];
#pragma unroll
    for (int m = 0; m < N; ++m) {
      // faces c+1 (left face index m+2), c (m+1), c-1 (m), c-2 (m-1)
      const R a = m + 2 < N ? w[m + 2][0] : (m + 2 == N ? nm0 : nm1);
      const R b = m + 1 < N ? w[m + 1][1] : n00;
      const R e = w[m][2];
      const R f = m >= 1 ? w[m - 1][3] : p2;
      out[m] = g[m] * pc[m] + a + b + e + f;
    }
    st_row<R, N>(fbar + p, full, navail, out);
  }
  cp_async_wait<0>();
}

// Vectorised adjoint of the v sweep (FP32, 16-byte aligned layouts): the lane layout of
// k_sweep_v_vec -- a lane owns 4 cells along i and marches `rows` rows in j of one level. At row
// step j it forms the factors of row j+2 and the weights of face j+1, and completes cell j from
// the weights of faces j+1, j, j-1, j-2 kept in registers. Rows are staged two steps ahead by
// cp.async.
template <class R, int S, int VN = 4>
__global__ void __launch_bounds__(32 * VKW) k_adj_sweep_v_vec(Dev d, R dt, R splitfac, R AH, int nk, int rows,
                                                            bool copy0, const R* __restrict__ gbar,
                                                            R* __restrict__ fbar, const R* __restrict__ Dio,
                                                            const R* __restrict__ V, const R* __restrict__ DV,
                                                            const uint8_t* __restrict__ mflux,
                                                            const uint8_t* __restrict__ mupd,
                                                            const uint8_t* __restrict__ code) {
  static_assert(sizeof(R) == 4, "vectorised adjoint sweeps are FP32");
  constexpr int N = VN;  // cells per lane (4: float4; 2: float2, half the registers)
  constexpr int VB = N * (int)sizeof(R);
  constexpr int NA = 5;  // gbar(j+2), Dio(j+2), V(j+2), DV(j+1), codes(j+1) (the codes staged for N = 4)
  constexpr int sub = (S == UPSTREAM) ? 0 : 1;
  __shared__ VecPack<R, N> sbuf[VST][NA][32 * VKW];
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
  const long long base = (long long)k * d.sk + c0;
  const R dti = splitfac * dt;
  const R dxf = R(d.dy), dyf = R(d.dx), ard1 = R(d.ard1);  // DYV, DXV
  const R cdx = dti / dxf;
  const bool use_AH = AH > R(0);
  const R kfac = dt * splitfac * dyf * ard1;
  if (copy0 && k == 0) {  // level 0 passes (not touched by the sweep)
    for (int j = j0; j < j1; ++j) {
      R v[N];
      ld_row<R, N>(gbar + base - d.sk + (long long)j * sj, full, navail, v);
      st_row<R, N>(fbar + base - d.sk + (long long)j * sj, full, navail, v);
    }
  }
  auto rowv = [&](const R* a, int j, R (&v)[N]) {
    if (j < 0 || j >= nj) {
#pragma unroll
      for (int m = 0; m < N; ++m) v[m] = R(0);
    } else {
      ld_row<R, N>(a + base + (long long)j * sj, full, navail, v);
    }
  };
  auto mrow = [&](const uint8_t* a, int j) -> uint32_t {
    return (j < 0 || j >= nj) ? 0u : ld_mask_w<N>(a + (long long)j * sj + c0, full, navail);
  };
  auto crow_of = [&](int j) -> uint32_t {  // code bytes of face row j
    if (S == UPSTREAM || j < 0 || j >= nj) return 0u;
    return ld_mask_w<N>(code + base + (long long)j * sj, full, navail);  // N bytes, N-byte aligned
  };
  // factors of row r from its cotangent, heights and the transports of its faces
  auto factors = [&](int r, const R (&g)[N], const R (&hio)[N], const R (&Vr)[N], const R (&Vrm1)[N],
                     uint32_t mu, R (&kc)[N], R (&pc)[N]) {
    const bool rin = r >= 1 + sub && r <= nj - 2 - sub;
#pragma unroll
    for (int m = 0; m < N; ++m) {
      kc[m] = R(0);
      pc[m] = R(1);
      if (rin && mbit(mu, m)) adj_cell<R>(dti, dyf, ard1, kfac, hio[m], Vr[m], Vrm1[m], kc[m], pc[m]);
    }
    (void)g;
  };
  // weights of face f from the factors of rows f, f+1 and its transport, masks and branch codes
  auto face = [&](int f, const R (&ga)[N], const R (&ka)[N], const R (&gb)[N], const R (&kb)[N], const R (&Vf)[N],
                  const R (&DVf)[N], uint32_t mdn_m1, uint32_t m0, uint32_t mp1, uint32_t cw, R (&w)[4][N]) {
    const bool fin = f >= sub && f <= nj - 2 - sub;
#pragma unroll
    for (int m = 0; m < N; ++m) {
      R ww[4] = {R(0), R(0), R(0), R(0)};
      if (fin && mbit(m0, m)) {
        const R Fb = -ga[m] * ka[m] + gb[m] * kb[m];
        adj_face<R, S>(Fb, Vf[m], DVf[m], mbit(mdn_m1, m), mbit(mp1, m), (uint8_t)((cw >> (8 * m)) & 0xffu), dti,
                       cdx, dxf, AH, use_AH, ww);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) w[q][m] = ww[q];
    }
  };
  auto issue = [&](int j, int st) {
    if (j < j1) {
      const long long p = base + (long long)j * sj;
      const bool r2 = j + 2 < nj;
      cp_async_v<VB>(&sbuf[st][0][tid], r2 ? gbar + p + 2 * sj : gbar + p, r2 ? vbytes : 0);
      cp_async_v<VB>(&sbuf[st][1][tid], r2 ? Dio + p + 2 * sj : Dio + p, r2 ? vbytes : 0);
      cp_async_v<VB>(&sbuf[st][2][tid], r2 ? V + p + 2 * sj : V + p, r2 ? vbytes : 0);
      const bool r1 = j + 1 < nj;
      cp_async_v<VB>(&sbuf[st][3][tid], r1 ? DV + p + sj : DV + p, r1 ? vbytes : 0);
      if (N == 4 && S != UPSTREAM && full && r1)
        cp_async(reinterpret_cast<float*>(&sbuf[st][4][tid]), reinterpret_cast<const float*>(code + p + sj));
    }
    cp_async_commit();
  };
#pragma unroll
  for (int q = 0; q < VST - 1; ++q) issue(j0 + q, q);
  // prologue: factors of rows j0-2 .. j0+1, weights of faces j0-2, j0-1, j0
  R gA[N], kA[N], pA[N];  // row j0-2, then reused
  R gB[N], kB[N], pB[N];  // row j0-1
  R gC[N], kC[N], pC[N];  // row j0   (the window: rows j, j+1 after the prologue)
  R gD[N], kD[N], pD[N];  // row j0+1
  R Vprev[N];             // V of row j0+1 (the south face of row j0+2)
  uint32_t mfw[4];        // flux masks of rows j0-3 .. j0 (face f uses rows f-1, f, f+1)
  {
    R Vm3[N], Vm2[N], Vm1[N], V0[N], hio[N];
    rowv(V, j0 - 3, Vm3);
    rowv(V, j0 - 2, Vm2);
    rowv(V, j0 - 1, Vm1);
    rowv(V, j0, V0);
    rowv(V, j0 + 1, Vprev);
    rowv(gbar, j0 - 2, gA);
    rowv(Dio, j0 - 2, hio);
    factors(j0 - 2, gA, hio, Vm2, Vm3, mrow(mupd, j0 - 2), kA, pA);
    rowv(gbar, j0 - 1, gB);
    rowv(Dio, j0 - 1, hio);
    factors(j0 - 1, gB, hio, Vm1, Vm2, mrow(mupd, j0 - 1), kB, pB);
    rowv(gbar, j0, gC);
    rowv(Dio, j0, hio);
    factors(j0, gC, hio, V0, Vm1, mrow(mupd, j0), kC, pC);
    rowv(gbar, j0 + 1, gD);
    rowv(Dio, j0 + 1, hio);
    factors(j0 + 1, gD, hio, Vprev, V0, mrow(mupd, j0 + 1), kD, pD);
    mfw[0] = mrow(mflux, j0 - 3);
    mfw[1] = mrow(mflux, j0 - 2);
    mfw[2] = mrow(mflux, j0 - 1);
    mfw[3] = mrow(mflux, j0);
    R DVr[N], w[4][N];
    // face j0-2: rows j0-2 (A), j0-1 (B)
    rowv(DV, j0 - 2, DVr);
    face(j0 - 2, gA, kA, gB, kB, Vm2, DVr, mfw[0], mfw[1], mfw[2], crow_of(j0 - 2), w);
    R s3a[N];
#pragma unroll
    for (int m = 0; m < N; ++m) s3a[m] = w[3][m];
    // face j0-1: rows j0-1 (B), j0 (C)
    rowv(DV, j0 - 1, DVr);
    face(j0 - 1, gB, kB, gC, kC, Vm1, DVr, mfw[1], mfw[2], mfw[3], crow_of(j0 - 1), w);
    R s2a[N], s3b[N];
#pragma unroll
    for (int m = 0; m < N; ++m) {
      s2a[m] = w[2][m];
      s3b[m] = w[3][m];
    }
    // face j0: rows j0 (C), j0+1 (D)
    const uint32_t mf1 = mrow(mflux, j0 + 1);
    rowv(DV, j0, DVr);
    face(j0, gC, kC, gD, kD, V0, DVr, mfw[2], mfw[3], mf1, crow_of(j0), w);
    R s1[N], s2b[N], s3c[N];
#pragma unroll
    for (int m = 0; m < N; ++m) {
      s1[m] = w[1][m];
      s2b[m] = w[2][m];
      s3c[m] = w[3][m];
    }
    // masks for the loop: face j+1 uses flux rows j, j+1, j+2; the factors of row j+2 its update mask
    uint32_t fm0 = mfw[3], fm1 = mf1;
    uint32_t mfn = mrow(mflux, j0 + 2), mun = mrow(mupd, j0 + 2);
    int st = 0;
    for (int j = j0; j < j1; ++j) {
      issue(j + VST - 1, st == 0 ? VST - 1 : st - 1);
      const uint32_t fm2 = mfn, mu2 = mun;
      if (j + 1 < j1) {
        mfn = mrow(mflux, j + 3);
        mun = mrow(mupd, j + 3);
      }
      cp_async_wait<VST - 1>();
      R gE[N], hE[N], VE[N], DVj1[N];
      lds_vec<R, N>(sbuf[st][0][tid], gE);
      lds_vec<R, N>(sbuf[st][1][tid], hE);
      lds_vec<R, N>(sbuf[st][2][tid], VE);
      lds_vec<R, N>(sbuf[st][3][tid], DVj1);
      uint32_t cw = 0;
      if (S != UPSTREAM && j + 1 < nj) {
        if (N == 4 && full) cw = *reinterpret_cast<const uint32_t*>(&sbuf[st][4][tid]);
        else cw = crow_of(j + 1);
      }
      st = st == VST - 1 ? 0 : st + 1;
      // factors of row j+2 (its south face is V(j+1) = Vprev)
      R kE[N], pE[N];
      factors(j + 2, gE, hE, VE, Vprev, mu2, kE, pE);
      // face j+1: rows j+1 (D), j+2 (E)
      face(j + 1, gD, kD, gE, kE, Vprev, DVj1, fm0, fm1, fm2, cw, w);
      R out[N];
#pragma unroll
      for (int m = 0; m < N; ++m) out[m] = gC[m] * pC[m] + w[0][m] + s1[m] + s2a[m] + s3a[m];
      st_row<R, N>(fbar + base + (long long)j * sj, full, navail, out);
#pragma unroll
      for (int m = 0; m < N; ++m) {
        s1[m] = w[1][m];
        s2a[m] = s2b[m];
        s2b[m] = w[2][m];
        s3a[m] = s3b[m];
        s3b[m] = s3c[m];
        s3c[m] = w[3][m];
        gC[m] = gD[m]; kC[m] = kD[m]; pC[m] = pD[m];
        gD[m] = gE[m]; kD[m] = kE[m]; pD[m] = pE[m];
        Vprev[m] = VE[m];
      }
      fm0 = fm1;
      fm1 = fm2;
    }
  }
  cp_async_wait<0>();
  (void)gA; (void)kA; (void)pA; (void)gB; (void)kB; (void)pB;
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
    if constexpr (sizeof(R) == 4) {
      if (DIR == 0 && vec_layout<R>(d, nk + (copy0 ? 1 : 0), {gbar, fbar, Dio, U, DU}, {mflux, mupd, code})) {
        constexpr int N = 4;
        const int nseg = (d.ni() + UOWN * N - 1) / (UOWN * N);
        dim3 blk(32, UWB, 1);
        dim3 grd((nseg + UWB - 1) / UWB, d.nj(), nz);
        k_adj_sweep_u_vec<R, S><<<grd, blk, 0, s>>>(d, dt, splitfac, AH, nk, copy0, gbar, fbar, Dio, U, DU, mflux,
                                                    mupd, code);
        return (int)cudaGetLastError();
      }
      if (DIR == 1 && vec_layout<R>(d, nk + (copy0 ? 1 : 0), {gbar, fbar, Dio, U, DU}, {mflux, mupd, code})) {
        constexpr int N = 2;  // two cells per lane (the kernel's VN)
        const long long nx = (d.ni() + 32 * N - 1) / (32 * N), nzv = (nk + VKW - 1) / VKW;
        int rows = VJS;
        while (rows > 8 && nx * ((d.nj() + rows - 1) / rows) * nzv * VKW < 148LL * 24) rows /= 2;
        dim3 blk(32, VKW, 1);
        dim3 grd((unsigned)nx, (d.nj() + rows - 1) / rows, (unsigned)nzv);
        k_adj_sweep_v_vec<R, S, 2><<<grd, blk, 0, s>>>(d, dt, splitfac, AH, nk, rows, copy0, gbar, fbar, Dio, U, DU,
                                                    mflux, mupd, code);
        return (int)cudaGetLastError();
      }
    }
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
