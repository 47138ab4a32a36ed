// bc_kernels.cuh -- 3D kernels of the mode-split macro step (integrate_3d), templated on the type
// R3 of the 3D fields (double: the plain FP64 step, bit for bit with the oracle; float: the
// mixed-precision step). 2D fields are always FP64. Included by kernels_inst.cuh.
#pragma once
#include "bc_common.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace gb {

template <class R3>
struct V3 {
  const Dev& d;
  R3* p;
  __device__ R3& operator()(int i, int j, int k) const { return p[d.ix(i, j) + (long long)k * d.sk]; }
};
struct V2 {
  const Dev& d;
  double* p;
  __device__ double& operator()(int i, int j) const { return p[d.ix(i, j)]; }
};
struct I2 {
  const Dev& d;
  const int32_t* p;
  __device__ int operator()(int i, int j) const { return p[d.ix(i, j)]; }
};

// thread -> reference index over the haloed plane
#define GB_IJ_HALO                                          \
  const int i = blockIdx.x * blockDim.x + threadIdx.x + d.imin - HALO; \
  const int j = blockIdx.y * blockDim.y + threadIdx.y + d.jmin - HALO; \
  if (i > d.imax + HALO || j > d.jmax + HALO) return;

// ---------------------------------------------------------------------------------------------
// bottom_friction_3d.F90:50-130 (kumin = kvmin = 1); 2D output rru, rrv. Bottom-layer quotients
// in FP64.
template <class R3>
__global__ void k_bf3d(Dev d, Bc3<R3> s) {
  GB_IJ_HALO
  if (i < d.imin || i > d.imax || j < d.jmin || j > d.jmax) return;
  V3<R3> uu{d, s.f3[UU]}, vv{d, s.f3[VV]}, huo{d, s.f3[HUO]}, hvo{d, s.f3[HVO]}, hun{d, s.f3[HUN]}, hvn{d, s.f3[HVN]};
  V2 zub{d, s.f2[ZUB]}, zvb{d, s.f2[ZVB]}, rru{d, s.f2[RRU]}, rrv{d, s.f2[RRV]};
  I2 au{d, s.au}, av{d, s.av};
  const double kappa = s.par[P_KAPPA], min_depth = s.par[P_MIN_DEPTH];
  auto q = [](R3 a, R3 b) { return (double)a / (double)b; };
  if (au(i, j) >= 1) {
    const double uuloc = q(uu(i, j, 1), huo(i, j, 1));
    const double uvloc = 0.25 * (q(vv(i, j, 1), hvo(i, j, 1)) + q(vv(i + 1, j, 1), hvo(i + 1, j, 1)) +
                                 q(vv(i, j - 1, 1), hvo(i, j - 1, 1)) + q(vv(i + 1, j - 1, 1), hvo(i + 1, j - 1, 1)));
    const double hh = fmax(min_depth / d.kmax, (double)hun(i, j, 1)) ;
    double r = (zub(i, j) + 0.5 * hh) / zub(i, j);
    r = kappa / log(r);
    r = r * r;
    rru(i, j) = r * sqrt(uuloc * uuloc + uvloc * uvloc);
  }
  if (av(i, j) >= 1) {
    const double vuloc = 0.25 * (q(uu(i, j, 1), huo(i, j, 1)) + q(uu(i - 1, j, 1), huo(i - 1, j, 1)) +
                                 q(uu(i, j + 1, 1), huo(i, j + 1, 1)) + q(uu(i - 1, j + 1, 1), huo(i - 1, j + 1, 1)));
    const double vvloc = q(vv(i, j, 1), hvo(i, j, 1));
    const double hh = fmax(min_depth / d.kmax, (double)hvn(i, j, 1));
    double r = (zvb(i, j) + 0.5 * hh) / zvb(i, j);
    r = kappa / log(r);
    r = r * r;
    rrv(i, j) = r * sqrt(vuloc * vuloc + vvloc * vvloc);
  }
}

// ip_blumberg_mellor.F90:83-92: interface heights zz of every wet T column (j <= jmax+1,
// i <= imax+1); zz is a scratch 3D array.
template <class R3>
__global__ void k_zz(Dev d, Bc3<R3> s, R3* zzp) {
  GB_IJ_HALO
  if (i < d.imin || i > d.imax + 1 || j < d.jmin || j > d.jmax + 1) return;
  I2 az{d, s.az};
  if (az(i, j) < 1) return;
  V3<R3> hn{d, s.f3[HN]}, zz{d, zzp};
  V2 H{d, s.f2[HH]};
  // equidistant sigma layers: the column's height, the same at every level
  const R3 h = hn(i, j, d.kmax);
  R3 z = R3(-H(i, j)) + h;
  zz(i, j, 1) = z;
  for (int k = 2; k <= d.kmax; ++k) {
    z = z + h;
    zz(i, j, k) = z;
  }
}

// ip_blumberg_mellor.F90:94-148: downward integral of the buoyancy gradient per U and V column.
// ZS (blocks of 32 x 4 points): the interface heights of the block's columns and of the next column
// and row (the neighbours across the faces) are formed into dynamic shared memory with k_zz's
// expressions, (kmax+1) x 5 x 33 values, instead of read from the zz array that k_zz writes.
constexpr int IPZ_W = 33, IPZ_H = 5;
template <class R3, bool ZS = false>
__global__ void k_ip(Dev d, Bc3<R3> s, const R3* zzp) {
  extern __shared__ unsigned char ip_smem[];
  R3* const zsm = reinterpret_cast<R3*>(ip_smem);
  auto zsh = [&](int k, int r, int q) -> R3& { return zsm[(k * IPZ_H + r) * IPZ_W + q]; };
  const int tx = threadIdx.x, ty = threadIdx.y;
  if constexpr (ZS) {
    const int i0 = blockIdx.x * 32 + d.imin - HALO, j0 = blockIdx.y * 4 + d.jmin - HALO;
    V3<R3> hn{d, s.f3[HN]};
    V2 H{d, s.f2[HH]};
    I2 az{d, s.az};
    for (int p = ty * 32 + tx; p < IPZ_W * IPZ_H; p += 128) {
      const int r = p / IPZ_W, q = p - r * IPZ_W;
      const int ii = i0 + q, jj = j0 + r;
      // k_zz at (ii, jj); dry columns and those outside the plane are never read
      if (ii > d.imax + HALO || jj > d.jmax + HALO || az(ii, jj) < 1) continue;
      const R3 h = hn(ii, jj, d.kmax);
      R3 z = R3(-H(ii, jj)) + h;
      zsh(1, r, q) = z;
      for (int k = 2; k <= d.kmax; ++k) {
        z = z + h;
        zsh(k, r, q) = z;
      }
    }
    __syncthreads();
  }
  GB_IJ_HALO
  V3<R3> hun{d, s.f3[HUN]}, hvn{d, s.f3[HVN]}, buoy{d, s.f3[BUOY]}, idpdx{d, s.f3[IDPDX]}, idpdy{d, s.f3[IDPDY]},
      zzg{d, const_cast<R3*>(zzp)};
  // the interface height at level k of the point (di = dj = 0) or of its neighbour (1, 0) / (0, 1)
  auto zz = [&](int ii, int jj, int k) -> R3 {
    if constexpr (ZS) return zsh(k, ty + (jj - j), tx + (ii - i));
    else return zzg(ii, jj, k);
  };
  idpdx(i, j, 0) = R3(0);
  idpdy(i, j, 0) = R3(0);
  if (i < d.imin || i > d.imax || j < d.jmin || j > d.jmax) return;
  I2 au{d, s.au}, av{d, s.av};
  const int kmax = d.kmax;
  const R3 half = R3(0.5);
  // the point's U and V columns side by side: each a downward integral with its face's layer
  // height (level-constant with equidistant sigma layers: read once) and its neighbour across the
  // face ((i+1, j) and (i, j+1)); the loads of B levels of both columns are issued before their
  // stores, the point's own buoyancy and interface heights loaded once for both
  const bool uc = au(i, j) >= 1, vc = av(i, j) >= 1;
  if (!uc && !vc) return;
  struct Col {
    R3 grdl, buoyl, hc, hk1, prgr, dm1;
  };
  auto start = [&](Col& c, V3<R3>& hx, V3<R3>& out, int oi, int oj, R3 dm1) {
    c.dm1 = dm1;
    c.grdl = (buoy(i + oi, j + oj, kmax) - buoy(i, j, kmax)) * dm1;
    c.buoyl = half * (buoy(i + oi, j + oj, kmax) + buoy(i, j, kmax));
    c.hc = hx(i, j, kmax);
    c.hk1 = c.hc;
    c.prgr = c.grdl * half * c.hk1;
    out(i, j, kmax) = c.hk1 * c.prgr;
  };
  auto level = [&](Col& c, V3<R3>& out, int k, R3 b1, R3 b0, R3 z1, R3 z0) {
    const R3 grdu = c.grdl;
    c.grdl = (b1 - b0) * c.dm1;
    const R3 buoyu = c.buoyl;
    c.buoyl = half * (b1 + b0);
    const R3 dz = (z1 - z0) * c.dm1;
    c.prgr = c.prgr + half * (grdu + c.grdl) * half * (c.hc + c.hk1) - dz * (buoyu - c.buoyl);
    out(i, j, k) = c.hc * c.prgr;
    c.hk1 = c.hc;
  };
  Col cu{}, cv{};
  if (uc) start(cu, hun, idpdx, 1, 0, R3(1.0 / d.dx));
  if (vc) start(cv, hvn, idpdy, 0, 1, R3(1.0 / d.dy));
  constexpr int B = sizeof(R3) == 4 ? 8 : 4;
  int k = kmax - 1;
  for (; k >= B; k -= B) {
    R3 b0[B], z0[B], bu[B], zu[B], bv[B], zv[B];
#pragma unroll
    for (int m = 0; m < B; ++m) {
      b0[m] = buoy(i, j, k - m);
      z0[m] = zz(i, j, k - m);
      bu[m] = uc ? buoy(i + 1, j, k - m) : R3(0);
      zu[m] = uc ? zz(i + 1, j, k - m) : R3(0);
      bv[m] = vc ? buoy(i, j + 1, k - m) : R3(0);
      zv[m] = vc ? zz(i, j + 1, k - m) : R3(0);
    }
#pragma unroll
    for (int m = 0; m < B; ++m) {
      if (uc) level(cu, idpdx, k - m, bu[m], b0[m], zu[m], z0[m]);
      if (vc) level(cv, idpdy, k - m, bv[m], b0[m], zv[m], z0[m]);
    }
  }
  for (; k >= 1; --k) {
    const R3 b0 = buoy(i, j, k), z0 = zz(i, j, k);
    if (uc) level(cu, idpdx, k, buoy(i + 1, j, k), b0, zz(i + 1, j, k), z0);
    if (vc) level(cv, idpdy, k, buoy(i, j + 1, k), b0, zz(i, j + 1, k), z0);
  }
}

// ip_blumberg_mellor_lin.F90:87-97: heights of the pressure points (layer centres) of the
// columns i = imin..imax+1, j = jmin..jmax+1 with az >= 1.
template <class R3>
__global__ void k_zz_lin(Dev d, Bc3<R3> s, R3* zzp) {
  GB_IJ_HALO
  if (i < d.imin || i > d.imax + 1 || j < d.jmin || j > d.jmax + 1) return;
  I2 az{d, s.az};
  if (az(i, j) < 1) return;
  V3<R3> hn{d, s.f3[HN]}, zz{d, zzp};
  V2 H{d, s.f2[HH]};
  const R3 half = R3(0.5);
  R3 hprev = hn(i, j, 1);
  R3 z = R3(-H(i, j)) + half * hprev;
  zz(i, j, 1) = z;
  int k = 2;
  for (; k + 3 <= d.kmax; k += 4) {  // four levels' loads before their stores
    R3 h[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) h[m] = hn(i, j, k + m);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      z = z + half * (hprev + h[m]);
      zz(i, j, k + m) = z;
      hprev = h[m];
    }
  }
  for (; k <= d.kmax; ++k) {
    const R3 h = hn(i, j, k);
    z = z + half * (hprev + h);
    zz(i, j, k) = z;
    hprev = h;
  }
}

// ip_blumberg_mellor_lin.F90:99-158: downward integral per U and V column of the along-sigma
// buoyancy gradient minus the slope of the pressure points times the mean vertical buoyancy
// gradient of the two columns; lower bound kumin_pmz = kvmin_pmz = 1 (the only value the reference
// assigns). The V integral starts from hun(kmax) as in the reference (ip_blumberg_mellor_lin.F90:
// 143); its levels below use hvn. Expressions in the reference's order.
template <class R3>
__global__ void k_ip_lin(Dev d, Bc3<R3> s, const R3* zzp) {
  GB_IJ_HALO
  V3<R3> hun{d, s.f3[HUN]}, hvn{d, s.f3[HVN]}, buoy{d, s.f3[BUOY]}, idpdx{d, s.f3[IDPDX]}, idpdy{d, s.f3[IDPDY]},
      zz{d, const_cast<R3*>(zzp)};
  idpdx(i, j, 0) = R3(0);
  idpdy(i, j, 0) = R3(0);
  if (i < d.imin || i > d.imax || j < d.jmin || j > d.jmax) return;
  I2 au{d, s.au}, av{d, s.av};
  const int kmax = d.kmax;
  const R3 half = R3(0.5);
  auto column = [&](V3<R3>& hx, R3 h0, V3<R3>& out, int oi, int oj, R3 dm1) {
    // the level k+1 values of both columns carried down in registers
    R3 b1 = buoy(i + oi, j + oj, kmax), b0 = buoy(i, j, kmax);
    R3 z1 = zz(i + oi, j + oj, kmax), z0 = zz(i, j, kmax), hk1 = hx(i, j, kmax);
    R3 dzl = (z1 - z0) * dm1;
    R3 drl = (b1 - b0) * dm1;
    R3 prgr = drl * half * h0;
    out(i, j, kmax) = hk1 * prgr;
    for (int k = kmax - 1; k >= 1; --k) {
      const R3 b1k = buoy(i + oi, j + oj, k), b0k = buoy(i, j, k);
      const R3 z1k = zz(i + oi, j + oj, k), z0k = zz(i, j, k), hk = hx(i, j, k);
      const R3 dzu = dzl;
      dzl = (z1k - z0k) * dm1;
      const R3 dru = drl;
      drl = (b1k - b0k) * dm1;
      const R3 dzr2 = (b1 - b1k) / (z1 - z1k);
      const R3 dzr1 = (b0 - b0k) / (z0 - z0k);
      const R3 aa = half * (drl + dru);
      const R3 bb = half * (dzl + dzu);
      const R3 cc = half * (dzr2 + dzr1);
      prgr = prgr + (aa - bb * cc) * half * (hk1 + hk);
      out(i, j, k) = hk * prgr;
      b1 = b1k; b0 = b0k; z1 = z1k; z0 = z0k; hk1 = hk;
    }
  };
  if (au(i, j) >= 1) column(hun, hun(i, j, kmax), idpdx, 1, 0, R3(1.0 / d.dx));
  if (av(i, j) >= 1) column(hvn, hun(i, j, kmax), idpdy, 0, 1, R3(1.0 / d.dy));
}

// ip_z_interpol.F90:61-168 (pressure-point heights from k_zz_lin). Per U (V) column, downward from
// kmax-1, the neighbour buoyancies at the face's own pressure-point height zx(k), found by a search
// from the top for the first neighbour level at or below zx(k) and interpolated with the level
// above. Where a search ends at level 1 or finds nothing the reference keeps buoyplus / buoyminus
// of the previous level -- at a column's first levels, of the previous column in its loop order (j
// outer, i inner, every U column before the V columns); both start at 0. The device form numbers
// the columns in that order (position p: U columns 0 .. nx*ny-1, then the V columns) and runs in
// three steps with the same results as the sequential loops:
//   1. k_zi_cols<1>: every column runs with carried values of 0, writes its gradients and records
//      whether it read a carried value before setting its own (need), and the last value it set
//      with key p (key -1: it set none);
//   2. k_zi_scan_blocks + k_zi_scan_aggs: an inclusive max-scan of the keys gives, for every
//      position, the nearest preceding column that set the value;
//   3. k_zi_cols<3>: the columns that read a carried value run again with it.
template <class R3>
struct ZiScr {
  R3* last_p;  // per position: the last buoyplus / buoyminus the column set
  R3* last_m;
  int* key_p;  // p where the column set the value, else -1; scanned in place (per block of 1024)
  int* key_m;
  int* need;   // bit 0: read buoyplus before setting it; bit 1: buoyminus
  int* agg_p;  // per block of 1024 positions: the block's largest key, then scanned
  int* agg_m;
  long long np;
};
constexpr int ZI_SCAN = 1024;

template <class R3>
struct ZiOut {
  R3 bp, bm;
  bool set_p, set_m, read_p, read_m;
};

// One column of ip_z_interpol with the carried values bp, bm coming in. zx(k) is formed upward in
// the output column first and read back level by level as the downward loop overwrites it. A
// level's search starts where the level above stopped whenever zx did not rise from that level (the
// levels above it failed the test there, so they fail it again): the same index as a search from the
// top, in fewer steps.
template <class R3>
__device__ ZiOut<R3> zi_column(const Dev& d, const Bc3<R3>& s, const R3* zzp, int i, int j, bool vg, R3 bp, R3 bm) {
  V3<R3> hn{d, s.f3[HN]}, buoy{d, s.f3[BUOY]}, zz{d, const_cast<R3*>(zzp)};
  V3<R3> hx{d, s.f3[vg ? HVN : HUN]}, out{d, s.f3[vg ? IDPDY : IDPDX]};
  V2 H{d, s.f2[HH]}, Hx{d, s.f2[vg ? HV : HU]};
  const int oi = vg ? 0 : 1, oj = vg ? 1 : 0;
  const int kmax = d.kmax;
  const R3 half = R3(0.5);
  const R3 dm1 = vg ? R3(1.0 / d.dy) : R3(1.0 / d.dx);
  ZiOut<R3> o{bp, bm, false, false, false, false};
  R3 z = R3(-Hx(i, j)) + half * hx(i, j, 1);
  out(i, j, 1) = z;
  for (int k = 2; k <= kmax; ++k) {
    z = z + half * (hx(i, j, k - 1) + hx(i, j, k));
    out(i, j, k) = z;
  }
  const R3 zbed = R3(-H(i + oi, j + oj)), zbed0 = R3(-H(i, j));
  R3 grdl = half * hx(i, j, kmax) * (buoy(i + oi, j + oj, kmax) - buoy(i, j, kmax)) * dm1;
  R3 prgr = grdl;
  out(i, j, kmax) = hx(i, j, kmax) * prgr;
  int kp = kmax, km = kmax;
  R3 zxa = R3(0);
  for (int k = kmax - 1; k >= 1; --k) {
    const R3 zx = out(i, j, k);
    if (!(k < kmax - 1 && zx <= zxa)) kp = km = kmax;
    zxa = zx;
    const R3 grdu = grdl;
    for (; kp >= 1; --kp)
      if (zz(i + oi, j + oj, kp) <= zx) break;
    for (; km >= 1; --km)
      if (zz(i, j, km) <= zx) break;
    if (kp == kmax) {
      o.bp = buoy(i + oi, j + oj, kp);
      o.set_p = true;
    }
    if (kp < kmax && kp > 1) {
      o.bp = ((zx - zz(i + oi, j + oj, kp)) * buoy(i + oi, j + oj, kp + 1) +
              (zz(i + oi, j + oj, kp + 1) - zx) * buoy(i + oi, j + oj, kp)) /
             (half * (hn(i + oi, j + oj, kp + 1) + hn(i + oi, j + oj, kp)));
      o.set_p = true;
    }
    if (km == kmax) {
      o.bm = buoy(i, j, km);
      o.set_m = true;
    }
    if (km < kmax && km > 1) {
      o.bm = ((zx - zz(i, j, km)) * buoy(i, j, km + 1) + (zz(i, j, km + 1) - zx) * buoy(i, j, km)) /
             (half * (hn(i, j, km + 1) + hn(i, j, km)));
      o.set_m = true;
    }
    if (zx > zbed && zx > zbed0) {  // zx(k) > max(-H(i+oi,j+oj), -H(i,j))
      o.read_p = o.read_p || !o.set_p;
      o.read_m = o.read_m || !o.set_m;
      grdl = half * hx(i, j, k) * (o.bp - o.bm) * dm1;
    } else {
      grdl = R3(0);
    }
    prgr = prgr + grdu + grdl;
    out(i, j, k) = hx(i, j, k) * prgr;
  }
  return o;
}

// the largest key at or before this thread's in its block (blockDim.x = ZI_SCAN)
static __device__ __forceinline__ int zi_block_max_scan(int v, int* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v = max(v, u);
  }
  if (lane == 31) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    int t = sh[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t = max(t, u);
    }
    sh[lane] = t;
  }
  __syncthreads();
  const int r = w > 0 ? max(v, sh[w - 1]) : v;
  __syncthreads();  // sh is reused by the caller's next scan
  return r;
}

template <class R3, int PASS>
__global__ void __launch_bounds__(128) k_zi_cols(Dev d, Bc3<R3> s, const R3* zzp, ZiScr<R3> z) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= z.np) return;
  const int nx = d.imax - d.imin + 1;
  const long long nn = z.np / 2;
  const bool vg = p >= nn;
  const long long q = vg ? p - nn : p;
  const int i = d.imin + (int)(q % nx), j = d.jmin + (int)(q / nx);
  I2 mask{d, vg ? s.av : s.au};
  if (mask(i, j) < 1) {
    if (PASS == 1) {
      z.key_p[p] = -1;
      z.key_m[p] = -1;
      z.need[p] = 0;
    }
    return;
  }
  if (PASS == 1) {
    const ZiOut<R3> o = zi_column<R3>(d, s, zzp, i, j, vg, R3(0), R3(0));
    z.last_p[p] = o.bp;
    z.last_m[p] = o.bm;
    z.key_p[p] = o.set_p ? (int)p : -1;
    z.key_m[p] = o.set_m ? (int)p : -1;
    z.need[p] = (o.read_p ? 1 : 0) | (o.read_m ? 2 : 0);
  } else {
    const int need = z.need[p];
    if (!need) return;
    // the nearest preceding position that set the value: the scanned key of p-1 within its block,
    // and the scanned aggregate of the blocks before it
    auto prev = [&](const int* key, const int* agg) {
      if (p == 0) return -1;
      const long long b = (p - 1) / ZI_SCAN;
      const int in_block = key[p - 1];
      return b > 0 ? max(in_block, agg[b - 1]) : in_block;
    };
    const int pp = (need & 1) ? prev(z.key_p, z.agg_p) : -1;
    const int pm = (need & 2) ? prev(z.key_m, z.agg_m) : -1;
    const R3 bp = pp >= 0 ? z.last_p[pp] : R3(0);
    const R3 bm = pm >= 0 ? z.last_m[pm] : R3(0);
    zi_column<R3>(d, s, zzp, i, j, vg, bp, bm);
  }
}

// in-place inclusive max-scan of both key arrays per block of ZI_SCAN positions; block maxima to agg
static __global__ void __launch_bounds__(ZI_SCAN) k_zi_scan_blocks(int* key_p, int* key_m, int* agg_p, int* agg_m,
                                                            long long np) {
  __shared__ int sh[32];
  const long long p = (long long)blockIdx.x * ZI_SCAN + threadIdx.x;
  int* keys[2] = {key_p, key_m};
  int* aggs[2] = {agg_p, agg_m};
  for (int a = 0; a < 2; ++a) {
    const int v = zi_block_max_scan(p < np ? keys[a][p] : -1, sh);
    if (p < np) keys[a][p] = v;
    if (threadIdx.x == ZI_SCAN - 1) aggs[a][blockIdx.x] = v;
  }
}

// in-place inclusive max-scan of the nb block maxima (one block, chunks of ZI_SCAN)
static __global__ void __launch_bounds__(ZI_SCAN) k_zi_scan_aggs(int* agg_p, int* agg_m, int nb) {
  __shared__ int sh[32];
  int* aggs[2] = {agg_p, agg_m};
  for (int a = 0; a < 2; ++a) {
    int carry = -1;
    for (int c0 = 0; c0 < nb; c0 += ZI_SCAN) {
      const int t = c0 + threadIdx.x;
      const int v = max(zi_block_max_scan(t < nb ? aggs[a][t] : -1, sh), carry);
      if (t < nb) aggs[a][t] = v;
      if (threadIdx.x == ZI_SCAN - 1) sh[0] = v;
      __syncthreads();
      carry = sh[0];
      __syncthreads();
    }
  }
}

// ip_stelling_vankester.F90:56-398 (pressure-point heights from k_zz_lin, interface heights zi
// from k_svk_zi). Per U (V) column the interface heights of both columns and the face's surface are
// sorted into zl (the reference's exchange sort, in the thread's local memory); each interval adds
// its height times the limited buoyancy difference db; level k takes the integral down to zx(k).
// The reference's work arrays lvel and dzfrac keep the previous column's values wherever the
// interval loop does not reach a level (kcount > 0 at its end), and db is not reset per V column.
// Every column whose loop reaches all levels sets them all before reading them, so the parallel
// pass (one thread per column) gives the sequential result; a column that does not reach them
// raises a flag, and then one thread redoes every column in the reference's loop order with the
// carried arrays (k_svk_serial). Levels up to SVK_KMAX.
constexpr int SVK_KMAX = 64;
constexpr int SVK_L = 2 * SVK_KMAX + 1;

template <class R3>
struct SvkWork {
  R3 zx[SVK_KMAX + 1], zl[SVK_L + 1], dzl[SVK_L + 1], dzfrac[SVK_KMAX + 1];
  int lvel[SVK_KMAX + 2], m[SVK_L + 1], n[SVK_L + 1];
};

template <class R3>
__global__ void k_svk_zi(Dev d, Bc3<R3> s, R3* zip) {
  GB_IJ_HALO
  if (i < d.imin || i > d.imax + 1 || j < d.jmin || j > d.jmax + 1) return;
  I2 az{d, s.az};
  if (az(i, j) < 1) return;
  V3<R3> hn{d, s.f3[HN]}, zi{d, zip};
  V2 H{d, s.f2[HH]};
  R3 z = R3(-H(i, j));
  zi(i, j, 1) = z;
  for (int k = 2; k <= d.kmax; ++k) {
    z = z + hn(i, j, k - 1);
    zi(i, j, k) = z;
  }
}

// one column; returns the levels the interval loop left unset (kcount). par: the parallel pass,
// which then writes nothing (the serial pass redoes the column with the carried arrays). Where the
// reference would read lvel below 1 (a level no column has reached yet; outside its work arrays)
// the interval loop stops at 1.
template <class R3>
__device__ int svk_column(const Dev& d, const Bc3<R3>& s, const R3* zzp, const R3* zip, int i, int j, bool vg,
                          SvkWork<R3>& w, R3& db, bool par) {
  V3<R3> buoy{d, s.f3[BUOY]}, zz{d, const_cast<R3*>(zzp)}, zi{d, const_cast<R3*>(zip)};
  V3<R3> hx{d, s.f3[vg ? HVN : HUN]}, out{d, s.f3[vg ? IDPDY : IDPDX]};
  V2 Hx{d, s.f2[vg ? HV : HU]}, ssx{d, s.f2[vg ? SSVN : SSUN]};
  const int di = vg ? 0 : 1, dj = vg ? 1 : 0, i1 = i + di, j1 = j + dj;
  const int kmax = d.kmax, lnum = 2 * kmax + 1;
  const R3 half = R3(0.5);
  const R3 dm1 = vg ? R3(1.0 / d.dy) : R3(1.0 / d.dx);
  w.zx[1] = R3(-Hx(i, j)) + half * hx(i, j, 1);
  w.zl[1] = zi(i, j, 1);
  w.zl[2] = zi(i1, j1, 1);
  for (int k = 2; k <= kmax; ++k) {
    w.zx[k] = w.zx[k - 1] + half * (hx(i, j, k - 1) + hx(i, j, k));
    w.zl[2 * k - 1] = zi(i, j, k);
    w.zl[2 * k] = zi(i1, j1, k);
  }
  w.zl[lnum] = R3(ssx(i, j));
  for (bool changed = true; changed;) {  // ends: every pass that swaps removes an inversion
    changed = false;
    for (int l = 1; l <= lnum - 1; ++l)
      if (w.zl[l] > w.zl[l + 1]) {
        const R3 t = w.zl[l + 1];
        w.zl[l + 1] = w.zl[l];
        w.zl[l] = t;
        changed = true;
      }
  }
  w.m[lnum] = kmax;
  w.n[lnum] = kmax;
  int kcount = kmax;
  w.lvel[kmax + 1] = lnum;
  for (int l = lnum - 1; l >= 1; --l) {
    w.dzl[l] = w.zl[l + 1] - w.zl[l];
    w.m[l] = w.m[l + 1];
    w.n[l] = w.n[l + 1];
    if (w.zl[l + 1] <= zi(i, j, w.m[l])) w.m[l] = max(1, w.m[l] - 1);
    if (w.zl[l + 1] <= zi(i1, j1, w.n[l])) w.n[l] = max(1, w.n[l] - 1);
    if (kcount > 0 && w.zx[kcount] > w.zl[l]) {
      w.lvel[kcount] = l;
      w.dzfrac[kcount] = w.zx[kcount] - w.zl[l];
      --kcount;
    }
  }
  if (par && kcount > 0) return kcount;
  R3 prgr = R3(0);
  if (!vg) db = R3(0);
  for (int k = kmax; k >= 1; --k) {
    for (int l = w.lvel[k + 1] - 1; l >= max(w.lvel[k], 1); --l) {
      const int ml = w.m[l], nl = w.n[l];
      const R3 zn = zz(i1, j1, nl), zm = zz(i, j, ml);
      R3 bminus, bplus;
      if (zn >= zz(i, j, kmax)) bminus = buoy(i, j, kmax);
      else if (zn <= zz(i, j, 1)) bminus = buoy(i, j, 1);
      else {
        const int kl = zn >= zm ? ml : ml - 1, ku = zn >= zm ? ml + 1 : ml;
        const R3 dzz = zz(i, j, ku) - zz(i, j, kl);
        bminus = (zn - zz(i, j, kl)) / dzz * buoy(i, j, ku) + (zz(i, j, ku) - zn) / dzz * buoy(i, j, kl);
      }
      if (zm >= zz(i1, j1, kmax)) bplus = buoy(i1, j1, kmax);
      else if (zm <= zz(i1, j1, 1)) bplus = buoy(i1, j1, 1);
      else {
        const int kl = zm >= zn ? nl : nl - 1, ku = zm >= zn ? nl + 1 : nl;
        const R3 dzz = zz(i1, j1, ku) - zz(i1, j1, kl);
        bplus = (zm - zz(i1, j1, kl)) / dzz * buoy(i1, j1, ku) + (zz(i1, j1, ku) - zm) / dzz * buoy(i1, j1, kl);
      }
      const R3 dcm = buoy(i1, j1, nl) - bminus;
      const R3 dcn = bplus - buoy(i, j, ml);
      const R3 mn = dcm < dcn ? dcm : dcn, mx = dcn < dcm ? dcm : dcn;
      if (dcn * dcm < R3(0)) db = R3(0);
      else if (!vg) db = dcn >= R3(0) ? mn : mx;
      else {
        if (dcn >= R3(0)) db = mn;
        if (dcn <= R3(0)) db = mx;
      }
      prgr = prgr + w.dzl[l] * db * dm1;
    }
    out(i, j, k) = hx(i, j, k) * (prgr - w.dzfrac[k] * db * dm1);
  }
  return kcount;
}

// the parallel pass: positions in loop order (U columns, then V); flag: some column left levels
template <class R3>
__global__ void __launch_bounds__(128) k_svk_cols(Dev d, Bc3<R3> s, const R3* zzp, const R3* zip, int* flag,
                                                  long long np) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int nx = d.imax - d.imin + 1;
  const long long nn = np / 2;
  const bool vg = p >= nn;
  const long long q = vg ? p - nn : p;
  const int i = d.imin + (int)(q % nx), j = d.jmin + (int)(q / nx);
  I2 mask{d, vg ? s.av : s.au};
  if (mask(i, j) < 1) return;
  SvkWork<R3> w;
  R3 db = R3(0);
  if (svk_column<R3>(d, s, zzp, zip, i, j, vg, w, db, true) > 0) atomicOr(flag, 1);
}

// the reference's loops in their order with the carried work arrays; only when flagged
template <class R3>
__global__ void k_svk_serial(Dev d, Bc3<R3> s, const R3* zzp, const R3* zip, const int* flag) {
  if (*flag == 0) return;
  SvkWork<R3> w;
  for (int k = 0; k <= SVK_KMAX; ++k) {
    w.dzfrac[k] = R3(0);
    w.lvel[k] = 0;
  }
  w.lvel[SVK_KMAX + 1] = 0;
  R3 db = R3(0);
  I2 au{d, s.au}, av{d, s.av};
  for (int g = 0; g < 2; ++g)
    for (int j = d.jmin; j <= d.jmax; ++j)
      for (int i = d.imin; i <= d.imax; ++i)
        if ((g ? av(i, j) : au(i, j)) >= 1) svk_column<R3>(d, s, zzp, zip, i, j, g == 1, w, db, false);
}

// ip_song_wright.F90:99-150 (pressure-point heights from k_zz_lin): per U and V column the
// gradient of the layer-mean buoyancy times the layer-mean height, less the change of the mean
// buoyancy times the slope of the pressure points. The V column's first slope term is scaled by
// 1/dx as in the reference (ip_song_wright.F90:128). Expressions in the reference's order.
template <class R3>
__global__ void k_ip_sw(Dev d, Bc3<R3> s, const R3* zzp) {
  GB_IJ_HALO
  V3<R3> hn{d, s.f3[HN]}, hun{d, s.f3[HUN]}, hvn{d, s.f3[HVN]}, buoy{d, s.f3[BUOY]}, idpdx{d, s.f3[IDPDX]},
      idpdy{d, s.f3[IDPDY]}, zz{d, const_cast<R3*>(zzp)};
  idpdx(i, j, 0) = R3(0);
  idpdy(i, j, 0) = R3(0);
  if (i < d.imin || i > d.imax || j < d.jmin || j > d.jmax) return;
  I2 au{d, s.au}, av{d, s.av};
  const int kmax = d.kmax;
  const R3 half = R3(0.5), dxm1 = R3(1.0 / d.dx), dym1 = R3(1.0 / d.dy);
  auto column = [&](V3<R3>& hx, V3<R3>& out, int oi, int oj, R3 dm1, R3 dm1top) {
    const int i1 = i + oi, j1 = j + oj;
    // level k+1 values of both columns carried down in registers
    R3 b1 = buoy(i1, j1, kmax), b0 = buoy(i, j, kmax), h1 = hn(i1, j1, kmax), h0 = hn(i, j, kmax);
    R3 grdl = half * hx(i, j, kmax) * (b1 - b0) * dm1;
    R3 buoyl = half * (b1 + b0) * (zz(i1, j1, kmax) - zz(i, j, kmax)) * dm1top;
    R3 prgr = grdl;
    out(i, j, kmax) = hx(i, j, kmax) * prgr;
    for (int k = kmax - 1; k >= 1; --k) {
      const R3 b1k = buoy(i1, j1, k), b0k = buoy(i, j, k), h1k = hn(i1, j1, k), h0k = hn(i, j, k);
      grdl = (half * (b1k + b1) * half * (h1k + h1) - half * (b0k + b0) * half * (h0k + h0)) * dm1;
      const R3 buoyu = buoyl;
      buoyl = half * (b1k + b0k) * (zz(i1, j1, k) - zz(i, j, k)) * dm1;
      prgr = prgr + grdl - (buoyu - buoyl);
      out(i, j, k) = hx(i, j, k) * prgr;
      b1 = b1k; b0 = b0k; h1 = h1k; h0 = h0k;
    }
  };
  if (au(i, j) >= 1) column(hun, idpdx, 1, 0, dxm1, dxm1);
  if (av(i, j) >= 1) column(hvn, idpdy, 0, 1, dym1, dxm1);
}

// ip_chu_fan.F90:67-126 (interface heights from k_zz): the Blumberg-Mellor integral with a
// correction hc from the squared height differences of the four corners of each interface cell;
// the integral starts from the top gradient itself and the top level's term is hx*grad*hx/2, as in
// the reference. Expressions in the reference's order.
template <class R3>
__global__ void k_ip_cf(Dev d, Bc3<R3> s, const R3* zzp) {
  GB_IJ_HALO
  V3<R3> hun{d, s.f3[HUN]}, hvn{d, s.f3[HVN]}, buoy{d, s.f3[BUOY]}, idpdx{d, s.f3[IDPDX]}, idpdy{d, s.f3[IDPDY]},
      zz{d, const_cast<R3*>(zzp)};
  idpdx(i, j, 0) = R3(0);
  idpdy(i, j, 0) = R3(0);
  if (i < d.imin || i > d.imax || j < d.jmin || j > d.jmax) return;
  I2 au{d, s.au}, av{d, s.av};
  const int kmax = d.kmax;
  const R3 half = R3(0.5), sixth = R3(1.0 / 6);
  auto column = [&](V3<R3>& hx, V3<R3>& out, int oi, int oj, R3 dm1) {
    const int i1 = i + oi, j1 = j + oj;
    R3 b1 = buoy(i1, j1, kmax), b0 = buoy(i, j, kmax), z1 = zz(i1, j1, kmax), z0 = zz(i, j, kmax);
    R3 hk1 = hx(i, j, kmax);
    R3 grdl = (b1 - b0) * dm1;
    R3 buoyl = half * (b1 + b0);
    R3 prgr = grdl;
    out(i, j, kmax) = hk1 * prgr * half * hk1;
    for (int k = kmax - 1; k >= 1; --k) {
      const R3 b1k = buoy(i1, j1, k), b0k = buoy(i, j, k), z1k = zz(i1, j1, k), z0k = zz(i, j, k);
      const R3 hk = hx(i, j, k);
      const R3 grdu = grdl;
      grdl = (b1k - b0k) * dm1;
      const R3 buoyu = buoyl;
      buoyl = half * (b1k + b0k);
      const R3 dz = (z1k - z0k) * dm1;
      const R3 a = z1k - z1, b = z0k - z0, c = z1 - z0, e = z1k - z0k;
      R3 hc = a * a * (b1k - b1);
      hc = hc - b * b * (b0k - b0);
      hc = hc + c * c * (b1 - b0);
      hc = hc - e * e * (b1k - b0k);
      hc = hc * dm1 * sixth / (z0k + z1k - z0 - z1);
      prgr = prgr + (grdu + grdl + hc) * half * (hk + hk1) - dz * (buoyu - buoyl);
      out(i, j, k) = hk * prgr;
      b1 = b1k; b0 = b0k; z1 = z1k; z0 = z0k; hk1 = hk;
    }
  };
  if (au(i, j) >= 1) column(hun, idpdx, 1, 0, R3(1.0 / d.dx));
  if (av(i, j) >= 1) column(hvn, idpdy, 0, 1, R3(1.0 / d.dy));
}

// ip_shchepetkin_mcwilliams.F90 constants as the reference evaluates them: eps = 1.e-10 and
// OneFifth = 0.2 are single-precision literals widened to double; 1./12. is a single-precision
// quotient.
template <class R3>
struct SmConst {
  static constexpr double eps = double(1.e-10f), fifth = double(0.2f), t = double(1.0f / 12.0f);
};

// ip_shchepetkin_mcwilliams.F90:61-145: pressure-point heights of every haloed column with az >= 1
// (into zz), and for the columns i = imin..imax+1, j = jmin..jmax+1 the pressure integral P from
// the harmonic means of the vertical buoyancy and height differences (marched down the column in
// registers). Expressions in the reference's order.
template <class R3>
__global__ void k_sm_cols(Dev d, Bc3<R3> s, R3* zzp, R3* Pp) {
  GB_IJ_HALO
  I2 az{d, s.az};
  V3<R3> hn{d, s.f3[HN]}, buoy{d, s.f3[BUOY]}, zz{d, zzp}, P{d, Pp};
  if (az(i, j) < 1) {
    // land: zz stays zero, as the reference's array does (allocated zero, written on water only,
    // internal_pressure.F90:135); the face terms of neighbouring water columns read it
    for (int k = 1; k <= d.kmax; ++k) zz(i, j, k) = R3(0);
    return;
  }
  V2 H{d, s.f2[HH]};
  const int kmax = d.kmax;
  const R3 half = R3(0.5), two = R3(2.0), one = R3(1.0);
  const R3 eps = R3(SmConst<R3>::eps), fifth = R3(SmConst<R3>::fifth), t = R3(SmConst<R3>::t);
  R3 z = R3(-H(i, j)) + half * hn(i, j, 1);
  zz(i, j, 1) = z;
  for (int k = 2; k <= kmax; ++k) {
    z = z + half * (hn(i, j, k - 1) + hn(i, j, k));
    zz(i, j, k) = z;
  }
  if (i < d.imin || i > d.imax + 1 || j < d.jmin || j > d.jmax + 1) return;
  // original differences o(k) = x(k+1) - x(k), k = 1..kmax-1, o(kmax) = o(kmax-1), o(0) = o(1);
  // harmonic means h(k) of o(k), o(k-1) for k = 1..kmax
  auto oR = [&](int k) {
    const int kk = k < 1 ? 1 : (k > kmax - 1 ? kmax - 1 : k);
    return buoy(i, j, kk + 1) - buoy(i, j, kk);
  };
  auto oZ = [&](int k) {
    const int kk = k < 1 ? 1 : (k > kmax - 1 ? kmax - 1 : k);
    return zz(i, j, kk + 1) - zz(i, j, kk);
  };
  auto hR = [&](int k) {
    const R3 a = oR(k), b = oR(k - 1);
    const R3 cff = two * a * b;
    return cff > eps ? cff / (a + b) : R3(0);
  };
  auto hZ = [&](int k) {
    const R3 a = oZ(k), b = oZ(k - 1);
    return two * a * b / (a + b);
  };
  const R3 cff1 = one / (zz(i, j, kmax) - zz(i, j, kmax - 1));
  const R3 cff2 = half * (buoy(i, j, kmax) - buoy(i, j, kmax - 1)) * half * hn(i, j, kmax) * cff1;
  R3 p = (buoy(i, j, kmax) + cff2) * half * hn(i, j, kmax);
  P(i, j, kmax) = p;
  R3 dR1 = hR(kmax), dZ1 = hZ(kmax);  // level k+1
  for (int k = kmax - 1; k >= 1; --k) {
    const R3 dR0 = hR(k), dZ0 = hZ(k);
    const R3 b1 = buoy(i, j, k + 1), b0 = buoy(i, j, k), z1 = zz(i, j, k + 1), z0 = zz(i, j, k);
    p = p + half * ((b1 + b0) * (z1 - z0) -
                    fifth * ((dR1 - dR0) * (z1 - z0 - t * (dZ1 + dZ0)) - (dZ1 - dZ0) * (b1 - b0 - t * (dR1 + dR0))));
    P(i, j, k) = p;
    dR1 = dR0;
    dZ1 = dZ0;
  }
}

// ip_shchepetkin_mcwilliams.F90:147-262: per U and V face of the interior and level, the pressure
// difference of the two columns plus the flux term FC from the harmonic means of the horizontal
// height and buoyancy differences (each thread forms the two means of its face from the columns
// before, at and after the face), less the elevation-slope term. Expressions in the reference's
// order.
template <class R3>
__global__ void k_ip_sm(Dev d, Bc3<R3> s, const R3* zzp, const R3* Pp) {
  GB_IJ_HALO
  V3<R3> hun{d, s.f3[HUN]}, hvn{d, s.f3[HVN]}, buoy{d, s.f3[BUOY]}, idpdx{d, s.f3[IDPDX]}, idpdy{d, s.f3[IDPDY]},
      zz{d, const_cast<R3*>(zzp)}, P{d, const_cast<R3*>(Pp)};
  V2 sseo{d, s.f2[SSEO]};
  idpdx(i, j, 0) = R3(0);
  idpdy(i, j, 0) = R3(0);
  if (i < d.imin || i > d.imax || j < d.jmin || j > d.jmax) return;
  I2 au{d, s.au}, av{d, s.av};
  const int kmax = d.kmax;
  const R3 half = R3(0.5), two = R3(2.0), one = R3(1.0);
  const R3 eps = R3(SmConst<R3>::eps), fifth = R3(SmConst<R3>::fifth), t = R3(SmConst<R3>::t);
  auto harm = [&](R3 a, R3 b) {
    const R3 cff = two * a * b;
    return cff > eps ? cff * (one / (a + b)) : R3(0);
  };
  auto column = [&](V3<R3>& hx, V3<R3>& out, int oi, int oj, R3 dm1) {
    const int im = i - oi, jm = j - oj, i1 = i + oi, j1 = j + oj, i2 = i + 2 * oi, j2 = j + 2 * oj;
    const R3 slope = R3(sseo(i1, j1) - sseo(i, j));
    for (int k = kmax; k >= 1; --k) {
      const R3 zm = zz(im, jm, k), z0 = zz(i, j, k), z1 = zz(i1, j1, k), z2 = zz(i2, j2, k);
      const R3 bm = buoy(im, jm, k), b0 = buoy(i, j, k), b1 = buoy(i1, j1, k), b2 = buoy(i2, j2, k);
      const R3 dZx0 = harm(z0 - zm, z1 - z0), dZx1 = harm(z1 - z0, z2 - z1);
      const R3 dRx0 = harm(b0 - bm, b1 - b0), dRx1 = harm(b1 - b0, b2 - b1);
      R3 AJ = P(i1, j1, k) - P(i, j, k);
      const R3 FC = half * ((b1 + b0) * (z1 - z0) -
                            fifth * ((dRx1 - dRx0) * (z1 - z0 - t * (dZx1 + dZx0)) -
                                     (dZx1 - dZx0) * (b1 - b0 - t * (dRx1 + dRx0))));
      AJ = AJ + FC;
      const R3 hk = hx(i, j, k);
      out(i, j, k) = AJ * dm1 * hk - hk * dm1 * slope * half * (buoy(i1, j1, kmax) + buoy(i, j, kmax));
    }
  };
  if (au(i, j) >= 1) column(hun, idpdx, 1, 0, R3(1.0 / d.dx));
  if (av(i, j) >= 1) column(hvn, idpdy, 0, 1, R3(1.0 / d.dy));
}

// uu_momentum_3d.F90:169-304 (DIR 0) / vv_momentum_3d.F90:174-315 (DIR 1), kumin = 1: explicit
// (the old heights huo/hvo equal hun/hvn at this point of integrate_3d, m3d.F90, and are read from
// hun/hvn);
// terms, implicit vertical viscosity and the transport correction to the depth-integrated
// transport Uint. One thread per column. The column arithmetic type T is FP64 for the FP64 step
// (the reference's expressions in the reference's order) and FP32 for the mixed step (divisions by
// the fast reciprocal); the depth integral of the solution and the transport correction are FP64
// in both. The elimination carries ru(k+1), qu(k+1) in registers and stores ru(k), qu(k) in two
// scratch 3D arrays (RUs, QUs) so that occupancy is not limited by shared memory; the back
// substitution overwrites QUs with Res(k) and the last pass writes uu = Res + hn*Diff.
// The layer heights (hun / hvn, which the reference passes as both the old and the new heights
// here) are level-constant in sigma coordinates with equidistant layers, the only vertical grid
// this kernel supports: the column's height is read once (at kmax) for every level. The nine
// inputs of a level (uu, num at the column and its neighbour, the other velocity at the four
// points of its average, the advection term, the pressure gradient) are staged by cp.async into
// the thread's own shared-memory slots ahead of the elimination (a ring of SL levels, SL - 2 of
// them in flight), and the back substitution and the last pass load ahead through registers, so
// the column's loads are in flight while its recurrence runs.
// SM: ru, qu (and the back substitution's Res) of the block's columns in dynamic shared memory
// ([kmax+1][NT] each) instead of the scratch arrays -- FP32 with kmax < 64, where the columns fit
// next to the staging ring at full occupancy of 64-thread blocks -- which removes their round
// trips through DRAM.
constexpr int UVM_SLOTS = 4;
constexpr int UVM_IN = 9;
constexpr int UVM_THREADS = 128;
template <class R3, int DIR, bool SM, int NT, int SL = UVM_SLOTS>
__global__ void __launch_bounds__(NT) k_uvmom3d(Dev d, Bc3<R3> s, R3* RUs, R3* QUs) {
  using T = R3;
  static_assert(SL == 4 || SL == 8, "a ring of 4 or 8 levels");
  __shared__ R3 sl[SL][UVM_IN][NT];
  extern __shared__ unsigned char uvm_cols[];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int kmax = d.kmax;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + d.imin;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + d.jmin;
  if (i > d.imax || j > d.jmax) return;  // no barrier in this kernel
  I2 mask{d, DIR == 0 ? s.au : s.av};
  if (!(mask(i, j) == 1 || mask(i, j) == 2)) return;
  V3<R3> uu{d, s.f3[DIR == 0 ? UU : VV]}, vv{d, s.f3[DIR == 0 ? VV : UU]}, hn{d, s.f3[DIR == 0 ? HUN : HVN]},
      Ex{d, s.f3[DIR == 0 ? UUEX : VVEX]}, idp{d, s.f3[DIR == 0 ? IDPDX : IDPDY]}, num{d, s.f3[NUM]}, RUg{d, RUs},
      QUg{d, QUs};
  R3* const sRU = reinterpret_cast<R3*>(uvm_cols);
  R3* const sQU = sRU + (long long)(d.kmax + 1) * NT;
  auto RU = [&](int, int, int k) -> R3& {
    if constexpr (SM) return sRU[k * NT + tid];
    else return RUg(i, j, k);
  };
  auto QU = [&](int, int, int k) -> R3& {
    if constexpr (SM) return sQU[k * NT + tid];
    else return QUg(i, j, k);
  };
  V2 dry{d, s.f2[DIR == 0 ? DRY_U : DRY_V]}, cor{d, s.f2[DIR == 0 ? CORU : CORV]},
      taus{d, s.f2[DIR == 0 ? TAUSX : TAUSY]}, sseo{d, s.f2[SSEO]}, H{d, s.f2[HH]}, D{d, s.f2[D_]},
      airp{d, s.f2[AIRP]}, rr{d, s.f2[DIR == 0 ? RRU : RRV]}, Uint{d, s.f2[DIR == 0 ? UINT : VINT]},
      sso{d, s.f2[DIR == 0 ? SSUO : SSVO]}, HX{d, s.f2[DIR == 0 ? HU : HV]};
  const double g = s.par[P_G], rho_0 = s.par[P_RHO_0], dt = s.par[P_DT], cnpar = s.par[P_CNPAR],
               avmmol = s.par[P_AVMMOL], min_depth = s.par[P_MIN_DEPTH], ip_fac = s.par[P_IP_FAC];
  const int di = DIR == 0 ? 1 : 0, dj = DIR == 0 ? 0 : 1;
  if (kmax <= 1) {
    uu(i, j, kmax) = R3(Uint(i, j));
    return;
  }
  const double gamma = g * rho_0;
  const double gammai = 1.0 / gamma, rho_0i = 1.0 / rho_0;
  const T dryij = T(dry(i, j)), corij = T(cor(i, j));
  const T ip_t = T(ip_fac), avm_t = T(avmmol), dt_t = T(dt), g_t = T(g);
  const T taus_top = T(dry(i, j) * 0.5 * (taus(i, j) + taus(i + di, j + dj)) * rho_0i);
  // the level's inputs into slot k % SL (an empty group for k < 0 keeps the counting uniform)
  auto issue = [&](int k) {
    if (k >= 0) {
      R3(*q)[NT] = sl[k & (SL - 1)];
      cp_async(&q[0][tid], &uu(i, j, k));
      cp_async(&q[1][tid], &num(i, j, k));
      cp_async(&q[2][tid], &num(i + di, j + dj, k));
      if (DIR == 0) {
        cp_async(&q[3][tid], &vv(i, j, k));
        cp_async(&q[4][tid], &vv(i + 1, j, k));
        cp_async(&q[5][tid], &vv(i, j - 1, k));
        cp_async(&q[6][tid], &vv(i + 1, j - 1, k));
      } else {
        cp_async(&q[3][tid], &vv(i, j, k));
        cp_async(&q[4][tid], &vv(i - 1, j, k));
        cp_async(&q[5][tid], &vv(i, j + 1, k));
        cp_async(&q[6][tid], &vv(i - 1, j + 1, k));
      }
      cp_async(&q[7][tid], &Ex(i, j, k));
      cp_async(&q[8][tid], &idp(i, j, k));
    }
    cp_async_commit();
  };
  auto in = [&](int k, int q) -> T { return T(sl[k & (SL - 1)][q][tid]); };
  const T hcol = T(hn(i, j, kmax));
  auto HO = [&](int) { return hcol; };
  auto HN = [&](int) { return hcol; };
  auto UU_ = [&](int k) { return in(k, 0); };
  auto exk = [&](int k) {
    T loc, e;
    if (DIR == 0) {
      loc = T(0.25) * (in(k, 3) + in(k, 4) + in(k, 5) + in(k, 6));
      e = corij * loc;
    } else {
      loc = T(0.25) * (in(k, 3) + in(k, 4) + in(k, 5) + in(k, 6));
      e = -corij * loc;
    }
    T x = dryij * (e - in(k, 7) + ip_t * in(k, 8));
    if (k == kmax) {
      if constexpr (sizeof(T) == 8) x = x + dryij * 0.5 * (taus(i, j) + taus(i + di, j + dj)) * rho_0i;
      else x = x + taus_top;
    }
    return x;
  };
  auto dif = [&](int k) { return T(0.5) * (in(k, 1) + in(k, 2)) + avm_t; };
#pragma unroll
  for (int m = 0; m <= SL - 2; ++m) issue(kmax - m);
  const T c_o = T(2.0 * (1.0 - cnpar) * dt), c_n = T(2.0 * cnpar * dt);
  const double zp = fmax(sseo(i + di, j + dj), -H(i, j) + fmin(min_depth, D(i + di, j + dj)));
  const double zm = fmax(sseo(i, j), -H(i + di, j + dj) + fmin(min_depth, D(i, j)));
  double zx;
  if (DIR == 0)
    zx = (zp - zm + (airp(i + 1, j) - airp(i, j)) * gammai) / d.dx;
  else
    zx = (zp - zm + (airp(i, j + 1) - airp(i, j)) / gamma) / d.dy;
  const T zx_t = T(zx);
  cp_async_wait<SL - 3>();  // levels kmax and kmax-1
  // column window: heights and velocity at k-1, k, k+1
  int k = kmax;
  T hok = HO(k), hnk = HN(k), hokm1 = HO(k - 1), hnkm1 = HN(k - 1);
  T uk = UU_(k), ukm1 = UU_(k - 1), ukp1 = T(0), hokp1 = T(0), hnkp1 = T(0);
  T difk = dif(k - 1);
  T ao_km1 = qdiv(c_o * difk, hok + hokm1), an_km1 = qdiv(c_n * difk, hnk + hnkm1);
  T ru, qu;
  {
    const T a1 = qdiv(-an_km1, hnkm1);
    const T a2 = T(1) + qdiv(an_km1, hnk);
    const T a4 = uk * (1 - qdiv(ao_km1, hok)) + qdiv(ukm1 * ao_km1, hokm1) + dt_t * exk(k) -
                 dt_t * T(0.5) * (hok + hnk) * g_t * zx_t;
    ru = qdiv(a1, a2);
    qu = qdiv(a4, a2);
    RU(i, j, k) = R3(ru);
    QU(i, j, k) = R3(qu);
  }
  for (k = kmax - 1; k >= 2; --k) {
    issue(k - (SL - 2));      // into the slot of level k+2, last read in the iteration of level k+2
    cp_async_wait<SL - 3>();  // level k-1
    const T ao_k = ao_km1, an_k = an_km1;
    hokp1 = hok; hnkp1 = hnk; ukp1 = uk;
    hok = hokm1; hnk = hnkm1; uk = ukm1;
    hokm1 = HO(k - 1); hnkm1 = HN(k - 1); ukm1 = UU_(k - 1);
    difk = dif(k - 1);
    ao_km1 = qdiv(c_o * difk, hok + hokm1);
    an_km1 = qdiv(c_n * difk, hnk + hnkm1);
    const T a3 = qdiv(-an_k, hnkp1);
    const T a1 = qdiv(-an_km1, hnkm1);
    const T a2 = T(1) + qdiv(an_k + an_km1, hnk);
    const T a4 = qdiv(ukp1 * ao_k, hokp1) + uk * (1 - qdiv(ao_k + ao_km1, hok)) + qdiv(ukm1 * ao_km1, hokm1) +
                 dt_t * exk(k) - dt_t * T(0.5) * (hok + hnk) * g_t * zx_t;
    const T den = a2 - a3 * ru;
    ru = qdiv(a1, den);
    qu = qdiv(a4 - a3 * qu, den);
    RU(i, j, k) = R3(ru);
    QU(i, j, k) = R3(qu);
  }
  T v;
  {
    k = 1;
    const T ao_k = ao_km1, an_k = an_km1;
    hokp1 = hok; hnkp1 = hnk; ukp1 = uk;
    hok = hokm1; hnk = hnkm1; uk = ukm1;
    const T a3 = qdiv(-an_k, hnkp1);
    const T a2 = T(1) + qdiv(an_k, hnk) + qdiv(dt_t * T(rr(i, j)), T(0.5) * (hnk + hok));
    const T a4 = qdiv(ukp1 * ao_k, hokp1) + uk * (1 - qdiv(ao_k, hok)) + dt_t * exk(k) -
                 dt_t * T(0.5) * (hok + hnk) * g_t * zx_t;
    v = qdiv(a4 - a3 * qu, a2 - a3 * ru);
  }
  cp_async_wait<0>();
  // back substitution (Res in QU) and its FP64 sum in ascending k; RU, QU two levels ahead
  double ResInt = 0.0;
  ResInt = ResInt + (double)v;
  QU(i, j, 1) = R3(v);
  T q1 = T(0), r1 = T(0), q2 = T(0), r2 = T(0);
  if (kmax >= 2) { q1 = T(QU(i, j, 2)); r1 = T(RU(i, j, 2)); }
  if (kmax >= 3) { q2 = T(QU(i, j, 3)); r2 = T(RU(i, j, 3)); }
  for (k = 2; k <= kmax; ++k) {
    const T qc = q1, rc = r1;
    q1 = q2; r1 = r2;
    if (k + 2 <= kmax) { q2 = T(QU(i, j, k + 2)); r2 = T(RU(i, j, k + 2)); }
    v = qc - rc * v;
    QU(i, j, k) = R3(v);
    ResInt = ResInt + (double)v;
  }
  const double Diff = (Uint(i, j) - ResInt) / (sso(i, j) + HX(i, j));
  // last pass, four independent levels at a time
  for (k = 1; k + 3 <= kmax; k += 4) {
    R3 q[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) q[m] = QU(i, j, k + m);
#pragma unroll
    for (int m = 0; m < 4; ++m) uu(i, j, k + m) = R3((double)q[m] + (double)hcol * Diff);
  }
  for (; k <= kmax; ++k) uu(i, j, k) = R3((double)QU(i, j, k) + (double)hcol * Diff);
}

// sigma_coordinates.F90:85-113 (equidistant sigma): layer heights of all levels 0..kmax. A thread
// covers up to LVC levels of one column (grid z = level chunk; one chunk for kmax < 64): the
// column's 2D inputs are read once, and its stores (six per level) are independent.
constexpr int LVC = 64;
template <class R3>
__global__ void k_sigma(Dev d, Bc3<R3> s) {
  GB_IJ_HALO
  const int k0 = blockIdx.z * LVC, k1 = min(k0 + LVC, d.kmax + 1);
  V2 sseo{d, s.f2[SSEO]}, ssen{d, s.f2[SSEN]}, H{d, s.f2[HH]}, ssuo{d, s.f2[SSUO]}, ssun{d, s.f2[SSUN]},
      HU_{d, s.f2[HU]}, ssvo{d, s.f2[SSVO]}, ssvn{d, s.f2[SSVN]}, HV_{d, s.f2[HV]};
  V3<R3> ho{d, s.f3[HO]}, hn{d, s.f3[HN]}, huo{d, s.f3[HUO]}, hun{d, s.f3[HUN]}, hvo{d, s.f3[HVO]}, hvn{d, s.f3[HVN]};
  const double kmaxm1 = 1.0 / (double)(float)d.kmax;
  {
    const R3 a = R3((sseo(i, j) + H(i, j)) * kmaxm1), b = R3((ssen(i, j) + H(i, j)) * kmaxm1);
    for (int k = k0; k < k1; ++k) {
      ho(i, j, k) = a;
      hn(i, j, k) = b;
    }
  }
  if (i <= d.imax + HALO - 1) {
    const R3 a = R3((ssuo(i, j) + HU_(i, j)) * kmaxm1), b = R3((ssun(i, j) + HU_(i, j)) * kmaxm1);
    for (int k = k0; k < k1; ++k) {
      huo(i, j, k) = a;
      hun(i, j, k) = b;
    }
  }
  if (j <= d.jmax + HALO - 1) {
    const R3 a = R3((ssvo(i, j) + HV_(i, j)) * kmaxm1), b = R3((ssvn(i, j) + HV_(i, j)) * kmaxm1);
    for (int k = k0; k < k1; ++k) {
      hvo(i, j, k) = a;
      hvn(i, j, k) = b;
    }
  }
}

// FP32 form of k_sigma for 16-byte aligned layouts: a thread covers 4 consecutive cells of a row
// and stores float4 vectors (a quarter of the store instructions of the scalar form, whose
// stores queue up behind one another).
template <int N>
__global__ void __launch_bounds__(128) k_sigma_vec(Dev d, Bc3<float> s) {
  const int ni = d.ni(), nj = d.nj();
  const int c0 = (blockIdx.x * blockDim.x + threadIdx.x) * N;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  if (c0 >= ni || jj >= nj) return;
  const long long c = (long long)jj * d.sj + c0;
  const int nall = min(N, ni - c0), nu = min(N, ni - 1 - c0);
  const bool vrow = jj <= nj - 2;
  const double kmaxm1 = 1.0 / (double)(float)d.kmax;
  float a0[N], b0[N], a1[N], b1[N], a2[N], b2[N];
#pragma unroll
  for (int m = 0; m < N; ++m) {
    const long long q = c + (m < nall ? m : 0);
    a0[m] = (float)((s.f2[SSEO][q] + s.f2[HH][q]) * kmaxm1);
    b0[m] = (float)((s.f2[SSEN][q] + s.f2[HH][q]) * kmaxm1);
    a1[m] = (float)((s.f2[SSUO][q] + s.f2[HU][q]) * kmaxm1);
    b1[m] = (float)((s.f2[SSUN][q] + s.f2[HU][q]) * kmaxm1);
    a2[m] = (float)((s.f2[SSVO][q] + s.f2[HV][q]) * kmaxm1);
    b2[m] = (float)((s.f2[SSVN][q] + s.f2[HV][q]) * kmaxm1);
  }
  // levels in gridDim.z chunks: more threads, each with fewer stores queued behind one another
  const int kc = (d.kmax + 1 + gridDim.z - 1) / gridDim.z;
  const int ka = blockIdx.z * kc, kb = min(d.kmax + 1, ka + kc);
  for (int k = ka; k < kb; ++k) {
    const long long p = c + (long long)k * d.sk;
    st_row<float, N>(s.f3[HO] + p, nall == N, nall, a0);
    st_row<float, N>(s.f3[HN] + p, nall == N, nall, b0);
    if (nu > 0) {
      st_row<float, N>(s.f3[HUO] + p, nu == N, nu, a1);
      st_row<float, N>(s.f3[HUN] + p, nu == N, nu, b1);
    }
    if (vrow) {
      st_row<float, N>(s.f3[HVO] + p, nall == N, nall, a2);
      st_row<float, N>(s.f3[HVN] + p, nall == N, nall, b2);
    }
  }
}

// ww_momentum_3d.F90:74-106 (kmin = 1): upward continuity integral per wet interior column.
// The layer height that k_sigma / k_sigma_vec store at every level of a column (equidistant sigma
// coordinates, sigma_coordinates.F90:85-113), formed with their expression from the column's
// elevation e (sseo, ssen, ssuo, ssun, ssvo, ssvn) and depth hx (H, HU, HV): the kernels that run
// after k_sigma in the same macro step take the heights from here instead of reading the 3D
// arrays back (the same values where k_sigma wrote them).
template <class R3>
__device__ __forceinline__ R3 sig_h(const Bc3<R3>& s, int e, int hx, long long c, double kmaxm1) {
  return R3((s.f2[e][c] + s.f2[hx][c]) * kmaxm1);
}

// The column heights of the macro step after k_sigma, as 2D planes of R3 (NCOLH of them, n2 apart):
// COL_HO, COL_HN, COL_HUN, COL_HVN = the values k_sigma stored at every level of ho, hn, hun, hvn;
// COL_HUA_U, COL_HVA_U, COL_HUA_V, COL_HVA_V = the face depths huadv, hvadv of the U and the V
// momentum grids (uv_advect_3d.F90:76-98, :267-289), which are the same at every level. Cells where
// k_sigma or uv_advect_3d form no value hold 0.
template <class R3>
__global__ void k_col_heights(Dev d, Bc3<R3> s, R3* out) {
  GB_IJ_HALO
  const int ni = d.ni(), nj = d.nj();
  const long long n2 = d.sj * (long long)nj;  // plane pitch (the 2D fields' size)
  const int ii = i - (d.imin - HALO), jj = j - (d.jmin - HALO);
  const long long c = d.ix(i, j);
  const double kmaxm1 = 1.0 / (double)(float)d.kmax;
  const R3 half = R3(0.5);
  auto ho = [&](long long q) { return sig_h<R3>(s, SSEO, HH, q, kmaxm1); };
  auto hn = [&](long long q) { return sig_h<R3>(s, SSEN, HH, q, kmaxm1); };
  auto hun = [&](long long q) { return sig_h<R3>(s, SSUN, HU, q, kmaxm1); };
  auto hvn = [&](long long q) { return sig_h<R3>(s, SSVN, HV, q, kmaxm1); };
  const bool ulast = ii == ni - 1, vlast = jj == nj - 1;
  out[COL_HO * n2 + c] = ho(c);
  out[COL_HN * n2 + c] = hn(c);
  out[COL_HUN * n2 + c] = ulast ? R3(0) : hun(c);
  out[COL_HVN * n2 + c] = vlast ? R3(0) : hvn(c);
  out[COL_HUA_U * n2 + c] = ulast ? R3(0) : half * (ho(c + 1) + hn(c + 1));
  out[COL_HVA_U * n2 + c] = (ulast || vlast) ? R3(0) : half * (hvn(c) + hvn(c + 1));
  out[COL_HUA_V * n2 + c] = (ulast || vlast) ? R3(0) : half * (hun(c) + hun(c + d.sj));
  out[COL_HVA_V * n2 + c] = vlast ? R3(0) : half * (ho(c + d.sj) + hn(c + d.sj));
}

// ww_momentum_3d.F90:74-106 with the layer heights of the column from sig_h (read after k_sigma)
template <class R3>
__global__ void k_ww(Dev d, Bc3<R3> s) {
  GB_IJ_HALO
  if (i < d.imin || i > d.imax || j < d.jmin || j > d.jmax) return;
  I2 az{d, s.az};
  if (az(i, j) != 1) return;
  V3<R3> ww{d, s.f3[WW]}, uu{d, s.f3[UU]}, vv{d, s.f3[VV]};
  const R3 dtm1 = R3(1.0 / s.par[P_DT]);
  const R3 dx = R3(d.dx), dy = R3(d.dy), ard1 = R3(d.ard1);
  const double kmaxm1 = 1.0 / (double)(float)d.kmax;
  const long long c = d.ix(i, j);
  const R3 hnc = sig_h<R3>(s, SSEN, HH, c, kmaxm1), hoc = sig_h<R3>(s, SSEO, HH, c, kmaxm1);
  // four levels' loads are issued before their four stores (the loads do not wait on the stores)
  R3 w = ww(i, j, 0);
  int k = 1;
  for (; k + 3 <= d.kmax - 1; k += 4) {
    R3 a[4][4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      a[m][0] = uu(i, j, k + m);
      a[m][1] = uu(i - 1, j, k + m);
      a[m][2] = vv(i, j, k + m);
      a[m][3] = vv(i, j - 1, k + m);
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      w = w - (hnc - hoc) * dtm1 - (a[m][0] * dy - a[m][1] * dy + a[m][2] * dx - a[m][3] * dx) * ard1;
      ww(i, j, k + m) = w;
    }
  }
  for (; k <= d.kmax - 1; ++k) {
    w = w - (hnc - hoc) * dtm1 -
        (uu(i, j, k) * dy - uu(i - 1, j, k) * dy + vv(i, j, k) * dx - vv(i, j - 1, k) * dx) * ard1;
    ww(i, j, k) = w;
  }
}

// uv_advect_3d.F90:76-98 (DIR 0, U grid) / :267-289 (DIR 1, V grid): the velocity, transports and
// heights of the momentum control volumes on levels 1..kmax; wwadv(:,:,0) = 0 (U grid).
template <class R3, int DIR>
__global__ void k_uvadv3d_prep(Dev d, Bc3<R3> s, R3* fadvp, R3* uuadvp, R3* vvadvp, R3* wwadvp, R3* huadvp,
                               R3* hvadvp) {
  GB_IJ_HALO
  const int k = blockIdx.z;  // one thread per cell and level 0..kmax (independent loads in flight)
  V3<R3> uu{d, s.f3[UU]}, vv{d, s.f3[VV]}, ww{d, s.f3[WW]}, ho{d, s.f3[HO]}, hn{d, s.f3[HN]}, hun{d, s.f3[HUN]},
      hvn{d, s.f3[HVN]};
  V3<R3> fadv{d, fadvp}, uuadv{d, uuadvp}, vvadv{d, vvadvp}, wwadv{d, wwadvp}, huadv{d, huadvp}, hvadv{d, hvadvp};
  const R3 half = R3(0.5);
  if (DIR == 0) {
    if (k == 0) {
      wwadv(i, j, 0) = R3(0);
      return;
    }
    if (i > d.imax + HALO - 1) return;
    fadv(i, j, k) = uu(i, j, k) / hun(i, j, k);
    uuadv(i, j, k) = half * (uu(i, j, k) + uu(i + 1, j, k));
    vvadv(i, j, k) = half * (vv(i, j, k) + vv(i + 1, j, k));
    wwadv(i, j, k) = half * (ww(i, j, k) + ww(i + 1, j, k));
    if (huadvp) huadv(i, j, k) = half * (ho(i + 1, j, k) + hn(i + 1, j, k));
    if (hvadvp) hvadv(i, j, k) = half * (hvn(i, j, k) + hvn(i + 1, j, k));
  } else {
    if (k == 0 || j > d.jmax + HALO - 1) return;
    fadv(i, j, k) = vv(i, j, k) / hvn(i, j, k);
    uuadv(i, j, k) = half * (uu(i, j, k) + uu(i, j + 1, k));
    vvadv(i, j, k) = half * (vv(i, j, k) + vv(i, j + 1, k));
    wwadv(i, j, k) = half * (ww(i, j, k) + ww(i, j + 1, k));
    if (huadvp) huadv(i, j, k) = half * (hun(i, j, k) + hun(i, j + 1, k));
    if (hvadvp) hvadv(i, j, k) = half * (ho(i, j + 1, k) + hn(i, j + 1, k));
  }
}

// FP32 form of k_uvadv3d_prep for 16-byte aligned layouts: a thread forms 4 consecutive cells of a
// row with float4 loads and stores (the i+1 neighbour of the last cell by one scalar load; the
// j+1 neighbours are the next row's vector). Same expressions, same cells written.
template <int DIR>
__global__ void __launch_bounds__(128) k_uvadv3d_prep_vec(Dev d, Bc3<float> s, float* fadvp, float* uuadvp,
                                                        float* vvadvp, float* wwadvp, float* huadvp, float* hvadvp) {
  constexpr int N = 4;
  const int ni = d.ni(), nj = d.nj();
  const int c0 = (blockIdx.x * blockDim.x + threadIdx.x) * N;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (c0 >= ni || jj >= nj) return;
  const long long p = (long long)k * d.sk + (long long)jj * d.sj + c0;
  // cells written: DIR 0 -- every cell but the last of the row (k >= 1); DIR 1 -- rows but the last
  int nw = min(N, ni - c0);
  if (k == 0) {
    if (DIR == 0) {
      const float z[N] = {0.f, 0.f, 0.f, 0.f};
      st_row<float, N>(wwadvp + p, nw == N, nw, z);
    }
    return;
  }
  if (DIR == 0) nw = min(nw, ni - 1 - c0);
  if (DIR == 1 && jj > nj - 2) return;
  if (nw <= 0) return;
  const bool fullr = c0 + N <= ni;  // loads of the whole vector are in the row
  auto ld = [&](int f, long long off, float (&v)[N]) { ld_row<float, N>(s.f3[f] + p + off, fullr, ni - c0, v); };
  float uu[N], vv[N], ww[N], ho[N], hn[N], hun[N], hvn[N];
  const float half = 0.5f;
  float fa[N], ua[N], va[N], wa[N], ha[N], hb[N];
  if (DIR == 0) {
    ld(UU, 0, uu); ld(VV, 0, vv); ld(WW, 0, ww); ld(HO, 0, ho); ld(HN, 0, hn); ld(HUN, 0, hun); ld(HVN, 0, hvn);
    // the i+1 neighbours of the last cell (only read when that cell is written)
    const bool nb = c0 + N < ni;
    const long long q = p + N;
    const float uue = nb ? s.f3[UU][q] : 0.f, vve = nb ? s.f3[VV][q] : 0.f, wwe = nb ? s.f3[WW][q] : 0.f,
                hoe = nb ? s.f3[HO][q] : 0.f, hne = nb ? s.f3[HN][q] : 0.f, hvne = nb ? s.f3[HVN][q] : 0.f;
#pragma unroll
    for (int m = 0; m < N; ++m) {
      const float u1 = m + 1 < N ? uu[m + 1] : uue, v1 = m + 1 < N ? vv[m + 1] : vve, w1 = m + 1 < N ? ww[m + 1] : wwe;
      const float o1 = m + 1 < N ? ho[m + 1] : hoe, n1 = m + 1 < N ? hn[m + 1] : hne,
                  h1 = m + 1 < N ? hvn[m + 1] : hvne;
      fa[m] = uu[m] / hun[m];
      ua[m] = half * (uu[m] + u1);
      va[m] = half * (vv[m] + v1);
      wa[m] = half * (ww[m] + w1);
      ha[m] = half * (o1 + n1);
      hb[m] = half * (hvn[m] + h1);
    }
  } else {
    float uu1[N], vv1[N], ww1[N], hun1[N], ho1[N], hn1[N];
    const long long sj = d.sj;
    ld(UU, 0, uu); ld(VV, 0, vv); ld(WW, 0, ww); ld(HUN, 0, hun); ld(HVN, 0, hvn);
    ld(UU, sj, uu1); ld(VV, sj, vv1); ld(WW, sj, ww1); ld(HUN, sj, hun1); ld(HO, sj, ho1); ld(HN, sj, hn1);
#pragma unroll
    for (int m = 0; m < N; ++m) {
      fa[m] = vv[m] / hvn[m];
      ua[m] = half * (uu[m] + uu1[m]);
      va[m] = half * (vv[m] + vv1[m]);
      wa[m] = half * (ww[m] + ww1[m]);
      ha[m] = half * (hun[m] + hun1[m]);
      hb[m] = half * (ho1[m] + hn1[m]);
    }
    (void)ho; (void)hn;
  }
  const bool fullw = nw == N;
  st_row<float, N>(fadvp + p, fullw, nw, fa);
  st_row<float, N>(uuadvp + p, fullw, nw, ua);
  st_row<float, N>(vvadvp + p, fullw, nw, va);
  st_row<float, N>(wwadvp + p, fullw, nw, wa);
  if (huadvp) st_row<float, N>(huadvp + p, fullw, nw, ha);
  if (hvadvp) st_row<float, N>(hvadvp + p, fullw, nw, hb);
}

// Both momentum grids' quantities in one pass (FP32, 16-byte aligned layouts): the inputs of a
// vector of 4 cells are read once for the U and the V grid; the same expressions and cells as
// k_uvadv3d_prep_vec<0> into u[0..5] and k_uvadv3d_prep_vec<1> into v[0..5] (fadv, uuadv, vvadv,
// wwadv, huadv, hvadv), with wwadv(:,:,0) = 0 of the U grid.
struct Prep6 {
  float* a[6];
};
template <int N = 4>
__global__ void __launch_bounds__(128) k_uvadv3d_prep_vec2(Dev d, Bc3<float> s, Prep6 u, Prep6 v,
                                                         const float* colh) {
  const int ni = d.ni(), nj = d.nj();
  const int c0 = (blockIdx.x * blockDim.x + threadIdx.x) * N;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (c0 >= ni || jj >= nj) return;
  const long long c = (long long)jj * d.sj + c0;  // the 2D index of the first cell
  const long long p = (long long)k * d.sk + c;
  const int nrow = min(N, ni - c0);
  if (k == 0) {
    const float z[N] = {0.f, 0.f, 0.f, 0.f};
    st_row<float, N>(u.a[3] + p, nrow == N, nrow, z);
    return;
  }
  const bool fullr = c0 + N <= ni;
  auto ld = [&](int f, long long off, float (&x)[N]) { ld_row<float, N>(s.f3[f] + p + off, fullr, ni - c0, x); };
  // heights: the 3D arrays, or (colh) the column planes of k_col_heights, the same values
  const long long n2 = d.sj * (long long)nj;
  auto ldh = [&](int f, int q, long long off, float (&x)[N]) {
    if (colh) ld_row<float, N>(colh + q * n2 + c + off, fullr, ni - c0, x);
    else ld_row<float, N>(s.f3[f] + p + off, fullr, ni - c0, x);
  };
  auto ldh1 = [&](int f, int q, long long off) -> float {
    return colh ? colh[q * n2 + c + off] : s.f3[f][p + off];
  };
  float uu[N], vv[N], ww[N], hun[N], hvn[N];
  ld(UU, 0, uu); ld(VV, 0, vv); ld(WW, 0, ww);
  ldh(HUN, COL_HUN, 0, hun); ldh(HVN, COL_HVN, 0, hvn);
  const float half = 0.5f;
  const int nwu = min(nrow, ni - 1 - c0);  // U grid: every cell but the last of the row
  if (nwu > 0) {
    const bool nb = c0 + N < ni;
    const long long q = p + N;
    const float uue = nb ? s.f3[UU][q] : 0.f, vve = nb ? s.f3[VV][q] : 0.f, wwe = nb ? s.f3[WW][q] : 0.f;
    float fa[N], ua[N], va[N], wa[N], ha[N], hb[N];
    const bool hout = u.a[4] || u.a[5];
    float ho[N], hn[N], hoe = 0.f, hne = 0.f, hvne = 0.f;
    if (hout) {
      ldh(HO, COL_HO, 0, ho); ldh(HN, COL_HN, 0, hn);
      if (nb) { hoe = ldh1(HO, COL_HO, N); hne = ldh1(HN, COL_HN, N); hvne = ldh1(HVN, COL_HVN, N); }
    }
#pragma unroll
    for (int m = 0; m < N; ++m) {
      const float u1 = m + 1 < N ? uu[m + 1] : uue, v1 = m + 1 < N ? vv[m + 1] : vve, w1 = m + 1 < N ? ww[m + 1] : wwe;
      fa[m] = uu[m] / hun[m];
      ua[m] = half * (uu[m] + u1);
      va[m] = half * (vv[m] + v1);
      wa[m] = half * (ww[m] + w1);
      if (hout) {
        const float o1 = m + 1 < N ? ho[m + 1] : hoe, n1 = m + 1 < N ? hn[m + 1] : hne,
                    h1 = m + 1 < N ? hvn[m + 1] : hvne;
        ha[m] = half * (o1 + n1);
        hb[m] = half * (hvn[m] + h1);
      }
    }
    const bool fw = nwu == N;
    st_row<float, N>(u.a[0] + p, fw, nwu, fa);
    st_row<float, N>(u.a[1] + p, fw, nwu, ua);
    st_row<float, N>(u.a[2] + p, fw, nwu, va);
    st_row<float, N>(u.a[3] + p, fw, nwu, wa);
    if (u.a[4]) st_row<float, N>(u.a[4] + p, fw, nwu, ha);
    if (u.a[5]) st_row<float, N>(u.a[5] + p, fw, nwu, hb);
  }
  if (jj <= nj - 2) {  // V grid: rows but the last
    const long long sj = d.sj;
    float uu1[N], vv1[N], ww1[N];
    ld(UU, sj, uu1); ld(VV, sj, vv1); ld(WW, sj, ww1);
    float fa[N], ua[N], va[N], wa[N], ha[N], hb[N];
    const bool hout = v.a[4] || v.a[5];
    float hun1[N], ho1[N], hn1[N];
    if (hout) { ldh(HUN, COL_HUN, sj, hun1); ldh(HO, COL_HO, sj, ho1); ldh(HN, COL_HN, sj, hn1); }
#pragma unroll
    for (int m = 0; m < N; ++m) {
      fa[m] = vv[m] / hvn[m];
      ua[m] = half * (uu[m] + uu1[m]);
      va[m] = half * (vv[m] + vv1[m]);
      wa[m] = half * (ww[m] + ww1[m]);
      if (hout) {
        ha[m] = half * (hun[m] + hun1[m]);
        hb[m] = half * (ho1[m] + hn1[m]);
      }
    }
    const bool fw = nrow == N;
    st_row<float, N>(v.a[0] + p, fw, nrow, fa);
    st_row<float, N>(v.a[1] + p, fw, nrow, ua);
    st_row<float, N>(v.a[2] + p, fw, nrow, va);
    st_row<float, N>(v.a[3] + p, fw, nrow, wa);
    if (v.a[4]) st_row<float, N>(v.a[4] + p, fw, nrow, ha);
    if (v.a[5]) st_row<float, N>(v.a[5] + p, fw, nrow, hb);
  }
}

// stresses_3d.F90:50-104 (bottom and surface stresses; FP64 from the bottom layer)
template <class R3>
__global__ void k_stresses(Dev d, Bc3<R3> s) {
  GB_IJ_HALO
  V3<R3> uu{d, s.f3[UU]}, vv{d, s.f3[VV]}, hun{d, s.f3[HUN]}, hvn{d, s.f3[HVN]};
  V2 rru{d, s.f2[RRU]}, rrv{d, s.f2[RRV]}, taubx{d, s.f2[TAUBX]}, tauby{d, s.f2[TAUBY]}, taub{d, s.f2[TAUB]},
      taus{d, s.f2[TAUS]}, tausx{d, s.f2[TAUSX]}, tausy{d, s.f2[TAUSY]};
  const double rho_0i = 1.0 / s.par[P_RHO_0];
  if (j >= d.jmin && j <= d.jmax && i >= d.imin - 1 && i <= d.imax)
    taubx(i, j) = -(double)uu(i, j, 1) / (double)hun(i, j, 1) * rru(i, j);
  if (j >= d.jmin - 1 && j <= d.jmax && i >= d.imin && i <= d.imax)
    tauby(i, j) = -(double)vv(i, j, 1) / (double)hvn(i, j, 1) * rrv(i, j);
  if (j >= d.jmin && j <= d.jmax && i >= d.imin && i <= d.imax) {
    const double a = (double)uu(i - 1, j, 1) / (double)hun(i - 1, j, 1) * rru(i - 1, j);
    const double b = (double)uu(i, j, 1) / (double)hun(i, j, 1) * rru(i, j);
    const double c = (double)vv(i, j - 1, 1) / (double)hvn(i, j - 1, 1) * rrv(i, j - 1);
    const double e = (double)vv(i, j, 1) / (double)hvn(i, j, 1) * rrv(i, j);
    taub(i, j) = sqrt(0.5 * (a * a + b * b + c * c + e * e));
    taus(i, j) = rho_0i * sqrt(tausx(i, j) * tausx(i, j) + tausy(i, j) * tausy(i, j));
  }
}

// eqstate.F90:127-137 (linear) + :252-261 (buoyancy) of one cell. FP64: the reference's expression.
// FP32: the buoyancy from the density anomaly dtr0*(T-T0) + dsr0*(S-S0) directly -- the same value
// in exact arithmetic, without forming rho_0 + anomaly and subtracting rho_0 again (in FP32 that
// cancellation keeps only ~1e-4 of the anomaly at rho ~ 1000 kg/m3); explicitly rounded operations,
// so the scalar and the vectorised kernel agree bit for bit.
template <class R3>
__device__ __forceinline__ void eos_lin(const Bc3<R3>& s, R3 t, R3 sal, R3& r, R3& b) {
  const R3 rho_0 = R3(s.par[P_RHO_0]), dtr0 = R3(s.par[P_DTR0]), dsr0 = R3(s.par[P_DSR0]), T0 = R3(s.par[P_T0]),
           S0 = R3(s.par[P_S0]);
  const R3 x = R3(-s.par[P_G] / s.par[P_RHO_0]);
  if constexpr (sizeof(R3) == 8) {
    r = rho_0 + dtr0 * (t - T0) + dsr0 * (sal - S0);
    b = x * (r - rho_0);
  } else {
    const float anom = __fmaf_rn(dsr0, __fsub_rn(sal, S0), __fmul_rn(dtr0, __fsub_rn(t, T0)));
    r = __fadd_rn(rho_0, anom);
    b = __fmul_rn(x, anom);
  }
}

// levels 1..kmax over the haloed plane, one thread per cell
template <class R3>
__global__ void k_eqstate(Dev d, Bc3<R3> s) {
  GB_IJ_HALO
  const int k = blockIdx.z + 1;
  V3<R3> rho{d, s.f3[RHO]}, buoy{d, s.f3[BUOY]}, T{d, s.f3[TT]}, S{d, s.f3[SS]};
  R3 r, b;
  eos_lin<R3>(s, T(i, j, k), S(i, j, k), r, b);
  rho(i, j, k) = r;
  buoy(i, j, k) = b;
}

// FP32, 16-byte aligned layouts: 4 consecutive cells per thread with float4 accesses
template <int N>
__global__ void __launch_bounds__(128) k_eqstate_vec(Dev d, Bc3<float> s) {
  const int ni = d.ni(), nj = d.nj();
  const int c0 = (blockIdx.x * blockDim.x + threadIdx.x) * N;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  if (c0 >= ni || jj >= nj) return;
  const long long p = (long long)(blockIdx.z + 1) * d.sk + (long long)jj * d.sj + c0;
  const int na = min(N, ni - c0);
  float t[N], sa[N], r[N], b[N];
  ld_row<float, N>(s.f3[TT] + p, na == N, na, t);
  ld_row<float, N>(s.f3[SS] + p, na == N, na, sa);
#pragma unroll
  for (int m = 0; m < N; ++m) eos_lin<float>(s, t[m], sa[m], r[m], b[m]);
  st_row<float, N>(s.f3[RHO] + p, na == N, na, r);
  st_row<float, N>(s.f3[BUOY] + p, na == N, na, b);
}

// eqstate.F90:496-534 (rho_from_theta_unesco80): UNESCO 1980 density at zero pressure; the
// coefficients are the reference's default-kind (single precision) literals, widened to double.
__device__ __forceinline__ double rho_unesco80(double T, double S) {
  const double T1 = T, T2 = T1 * T1, T3 = T1 * T2, T4 = T2 * T2, T5 = T1 * T4;
  const double S1 = S, S2 = S1 * S1, S3 = S1 * S2;
  double x = (double)999.842594f + (double)6.793952e-02f * T1 - (double)9.09529e-03f * T2 +
             (double)1.001685e-04f * T3;
  x = x - (double)1.120083e-06f * T4 + (double)6.536332e-09f * T5;
  x = x + S1 * ((double)0.824493f - (double)4.0899e-03f * T1 + (double)7.6438e-05f * T2 -
                (double)8.2467e-07f * T3);
  x = x + S1 * (double)5.3875e-09f * T4;
  x = x + sqrt(S3) * (-(double)5.72466e-03f + (double)1.0227e-04f * T1 - (double)1.6546e-06f * T2);
  x = x + (double)4.8314e-04f * S2;
  return x;
}

// eqstate.F90:540-590 (rho_from_theta at p = 0): the rational function of Jackett et al. (2006).
__device__ __forceinline__ double rho_jackett06(double s, double th) {
  const double th2 = th * th, sqrts = sqrt(s);
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

// eqstate.F90:144-261 with eqstate_method 2 (UNESCO80) or 3 (Jackett 2006): the density of the
// water columns (az > 0; land keeps its density) and the buoyancy -g/rho_0*(rho-rho_0) of every
// point of the haloed plane, levels 1..kmax. The density function is evaluated in FP64 for either
// storage type: in the mixed step the buoyancy is then formed from the FP64 density before it is
// rounded, which keeps the anomaly rho-rho_0 (a thousandth of rho) to FP32 precision. The thermal
// and haline expansion coefficients alpha, beta that the reference also forms feed only the
// turbulence closure's buoyancy frequency and are not formed.
template <class R3, int METHOD>
__global__ void k_eqstate_nl(Dev d, Bc3<R3> s) {
  GB_IJ_HALO
  const int k = blockIdx.z + 1;
  V3<R3> rho{d, s.f3[RHO]}, buoy{d, s.f3[BUOY]}, T{d, s.f3[TT]}, S{d, s.f3[SS]};
  I2 az{d, s.az};
  const double rho_0 = s.par[P_RHO_0];
  const double x = -s.par[P_G] / s.par[P_RHO_0];
  double r;
  if (az(i, j) > 0) {
    r = METHOD == 2 ? rho_unesco80((double)T(i, j, k), (double)S(i, j, k))
                    : rho_jackett06((double)S(i, j, k), (double)T(i, j, k));
    rho(i, j, k) = R3(r);
  } else {
    r = (double)rho(i, j, k);
  }
  if constexpr (sizeof(R3) == 8) buoy(i, j, k) = R3(x) * (R3(r) - R3(rho_0));
  else buoy(i, j, k) = R3(x * (r - rho_0));
}

// gotm.F90:96-163 with PARABOLIC_VISCOSITY (:131-143), after stresses_3d: per water column of the
// interior the profiles of turbulent kinetic energy, length scale, dissipation and eddy viscosity
// on the interfaces k = 1..kmax-1 from the bottom stress taub, the depth D and the bottom
// roughness (z0b from zub, zvb of the four velocity points), then num = profile + avmback and
// nuh = profile + avhback; at k = 0 and kmax the background is added to the stored values (the
// reference passes them through its column arrays). tke and eps receive the profiles when given.
// FP64 arithmetic with the reference's single-precision literals and expression order; one thread
// per column.
template <class R3>
__global__ void k_gotm_parabolic(Dev d, Bc3<R3> s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + d.imin;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + d.jmin;
  if (i > d.imax || j > d.jmax) return;
  I2 az{d, s.az};
  if (az(i, j) < 1) return;
  V2 D{d, s.f2[D_]}, taub{d, s.f2[TAUB]}, zub{d, s.f2[ZUB]}, zvb{d, s.f2[ZVB]};
  V3<R3> hn{d, s.f3[HN]}, num{d, s.f3[NUM]}, nuh{d, s.f3[NUH]}, tke{d, s.f3[TKE]}, eps{d, s.f3[EPS]};
  const int kmax = d.kmax;
  const double avmback = s.par[P_AVMBACK], avhback = s.par[P_AVHBACK];
  const double z0b = 0.5 * (fmax(zub(i - 1, j), zub(i, j)) + fmax(zvb(i, j - 1), zvb(i, j)));
  const double Dl = D(i, j), tb = taub(i, j);
  double zz = 0.0;
  for (int k = 1; k <= kmax - 1; ++k) {
    zz = zz + (double)hn(i, j, k);
    const double t = fmax((double)1.e-10f, (double)3.333333f * tb * (1.0 - zz / Dl));
    const double L = (double)0.4f * (zz + z0b) * sqrt(1.0 - zz / Dl);
    const double e = (double)0.16431677f * sqrt(t * t * t) / L;
    const double nu = (double)0.09f * t * t / e;
    if (s.f3[TKE]) tke(i, j, k) = R3(t);
    if (s.f3[EPS]) eps(i, j, k) = R3(e);
    num(i, j, k) = R3(nu + avmback);
    nuh(i, j, k) = R3(nu + avhback);
  }
  if (kmax >= 1) {
    num(i, j, 0) = R3((double)num(i, j, 0) + avmback);
    nuh(i, j, 0) = R3((double)nuh(i, j, 0) + avhback);
    num(i, j, kmax) = R3((double)num(i, j, kmax) + avmback);
    nuh(i, j, kmax) = R3((double)nuh(i, j, kmax) + avhback);
  }
}

// temperature.F90:452-465: the short-wave radiation rad of the water columns (az >= 1) of the
// interior, swr at the surface and below it swr*(A*exp(-z/g1) + (1-A)*exp(-z/g2)) with z the depth
// of the interface under the surface; one thread per column, FP64 arithmetic.
template <class R3>
__global__ void k_sw_radiation(Dev d, Bc3<R3> s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + d.imin;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + d.jmin;
  if (i > d.imax || j > d.jmax) return;
  I2 az{d, s.az};
  if (az(i, j) < 1) return;
  V2 swr{d, s.f2[SWR]}, A{d, s.f2[ATT_A]}, g1{d, s.f2[ATT_G1]}, g2{d, s.f2[ATT_G2]};
  V3<R3> hn{d, s.f3[HN]}, rad{d, s.f3[RAD]};
  const double swr_loc = swr(i, j), a = A(i, j), l1 = g1(i, j), l2 = g2(i, j);
  rad(i, j, d.kmax) = R3(swr_loc);
  double zz = 0.0;
  for (int k = d.kmax - 1; k >= 0; --k) {
    zz = zz + (double)hn(i, j, k + 1);
    rad(i, j, k) = R3(swr_loc * (a * exp(-zz / l1) + (1 - a) * exp(-zz / l2)));
  }
}

// temperature.F90:469-525: the sources that do_temperature adds to the right-hand side of its
// diffusion matrix, per layer of the water columns (az == 1) of the interior: dry_z*dt*(rad1d(k) -
// rad1d(k-1)), with shf*rho_0_cpi added in the top layer. rad1d = rad less the light reflected at
// the bottom (swr_bot_refl_frac > 0 and rad(0)/rad(kmax) > swr_min_bot_frac) times 1/(rho_0*cp); a
// cooling surface flux is dropped where the top layer is at the freezing point (T <= -0.0575*S).
// S_top: the top-level salinity before do_salinity (NULL: read S itself). The column's rad1d is
// formed level by level from the bottom up, so no column array is needed.
template <class R3>
__global__ void k_temp_source(Dev d, Bc3<R3> s, const R3* __restrict__ S_top, R3* __restrict__ srcp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + d.imin;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + d.jmin;
  if (i > d.imax || j > d.jmax) return;
  I2 az{d, s.az};
  if (az(i, j) != 1) return;
  const int kmax = d.kmax;
  V2 shf{d, s.f2[SHF]}, A{d, s.f2[ATT_A]}, g1{d, s.f2[ATT_G1]}, g2{d, s.f2[ATT_G2]}, dry_z{d, s.f2[DRY_Z]};
  V3<R3> hn{d, s.f3[HN]}, rad{d, s.f3[RAD]}, T{d, s.f3[TT]}, S{d, s.f3[SS]}, src{d, srcp};
  const double dt = s.par[P_DT];
  const double rho_0_cpi = 1.0 / (s.par[P_RHO_0] * s.par[P_CP]);
  const double refl = s.par[P_SWR_BOT_REFL_FRAC], minfrac = s.par[P_SWR_MIN_BOT_FRAC];
  double shf_loc = shf(i, j);
  const double stop = S_top ? (double)S_top[d.ix(i, j)] : (double)S(i, j, kmax);
  if ((double)T(i, j, kmax) <= -((double)0.0575f * stop)) shf_loc = fmax(0.0, shf_loc);
  const double rad0 = (double)rad(i, j, 0), radk = (double)rad(i, j, kmax);
  const bool reflect = refl > 0.0 && rad0 / radk > minfrac;
  const double swr_refl = reflect ? rad0 * refl : 0.0;
  const double a = A(i, j), l1 = g1(i, j), l2 = g2(i, j), dz = dry_z(i, j);
  // rad1d(k) before the scaling, k = 0..kmax
  double zz = 0.0;
  double below = reflect ? (rad0 - swr_refl) * rho_0_cpi : rad0 * rho_0_cpi;  // rad1d(k-1)
  for (int k = 1; k <= kmax; ++k) {
    double r = (double)rad(i, j, k);
    if (reflect) {
      zz = zz + (double)hn(i, j, k);
      r = r - swr_refl * (a * exp(-zz / l1) + (1 - a) * exp(-zz / l2));
    }
    const double here = r * rho_0_cpi;
    src(i, j, k) = k < kmax ? R3(dz * dt * (here - below)) : R3(dz * dt * (here + shf_loc * rho_0_cpi - below));
    below = here;
  }
}

// slow_terms.F90:57-181 (kmax > 1, kumin = kvmin = 1): vertical sums in FP64
template <class R3>
__global__ void k_slow_terms(Dev d, Bc3<R3> s) {
  GB_IJ_HALO
  if (i < d.imin || i > d.imax || j < d.jmin || j > d.jmax) return;
  V2 UEx{d, s.f2[UEX]}, VEx{d, s.f2[VEX]}, SlUx{d, s.f2[SLUX]}, SlVx{d, s.f2[SLVX]}, Slru{d, s.f2[SLRU]},
      Slrv{d, s.f2[SLRV]}, Uint{d, s.f2[UINT]}, Vint{d, s.f2[VINT]}, ssuo{d, s.f2[SSUO]}, ssun{d, s.f2[SSUN]},
      ssvo{d, s.f2[SSVO]}, ssvn{d, s.f2[SSVN]}, HU_{d, s.f2[HU]}, HV_{d, s.f2[HV]}, ru{d, s.f2[RU]}, rv{d, s.f2[RV]},
      rru{d, s.f2[RRU]}, rrv{d, s.f2[RRV]};
  V3<R3> uuEx{d, s.f3[UUEX]}, vvEx{d, s.f3[VVEX]}, idpdx{d, s.f3[IDPDX]}, idpdy{d, s.f3[IDPDY]}, uu{d, s.f3[UU]},
      vv{d, s.f3[VV]}, huo{d, s.f3[HUO]}, hun{d, s.f3[HUN]}, hvo{d, s.f3[HVO]}, hvn{d, s.f3[HVN]};
  I2 au{d, s.au}, av{d, s.av};
  const double ip_fac = s.par[P_IP_FAC];
  if (au(i, j) >= 1) {
    double vs = -UEx(i, j);
    for (int k = 1; k <= d.kmax; ++k) vs = vs + (double)uuEx(i, j, k) - ip_fac * (double)idpdx(i, j, k);
    SlUx(i, j) = vs;
    Slru(i, j) = -Uint(i, j) / (0.5 * (ssuo(i, j) + ssun(i, j)) + HU_(i, j)) * ru(i, j) +
                 (double)uu(i, j, 1) / (0.5 * ((double)huo(i, j, 1) + (double)hun(i, j, 1))) * rru(i, j);
  }
  if (av(i, j) >= 1) {
    double vs = -VEx(i, j);
    for (int k = 1; k <= d.kmax; ++k) vs = vs + (double)vvEx(i, j, k) - ip_fac * (double)idpdy(i, j, k);
    SlVx(i, j) = vs;
    Slrv(i, j) = -Vint(i, j) / (0.5 * (ssvo(i, j) + ssvn(i, j)) + HV_(i, j)) * rv(i, j) +
                 (double)vv(i, j, 1) / (0.5 * ((double)hvo(i, j, 1) + (double)hvn(i, j, 1))) * rrv(i, j);
  }
}

// ---------------------------------------------------------------------------------------------
// launchers
inline dim3 plane_grid(const Dev& d, dim3 blk, int nz = 1) {
  return dim3((d.ni() + blk.x - 1) / blk.x, (d.nj() + blk.y - 1) / blk.y, nz);
}

template <class R3>
int run_col_heights(const Dev& d, cudaStream_t st, const Bc3<R3>& s, R3* out) {
  const dim3 blk(64, 4, 1);
  k_col_heights<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s, out);
  return (int)cudaGetLastError();
}

template <class R3>
int run_bc3(int which, const Dev& d, cudaStream_t st, const Bc3<R3>& s, R3* const* scr, const R3* colh) {
  const dim3 blk(32, 4, 1);
  switch (which) {
    case BC3_BF3D: k_bf3d<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s); break;
    case BC3_ZZ: k_zz<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s, scr[6]); break;
    case BC3_IP:
      if constexpr (sizeof(R3) == 4) {  // the interface heights formed in shared memory (no k_zz)
        const size_t dyn = (size_t)(d.kmax + 1) * IPZ_H * IPZ_W * sizeof(R3);
        const cudaError_t e = cudaFuncSetAttribute(k_ip<R3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
        if (e != cudaSuccess) return (int)e;
        k_ip<R3, true><<<plane_grid(d, blk), blk, dyn, st>>>(d, s, nullptr);
      } else {
        k_ip<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s, scr[6]);
      }
      break;
    case BC3_ZZ_LIN: k_zz_lin<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s, scr[6]); break;
    case BC3_IP_LIN: k_ip_lin<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s, scr[6]); break;
    case BC3_IP_SW: k_ip_sw<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s, scr[6]); break;
    case BC3_IP_CF: k_ip_cf<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s, scr[6]); break;
    case BC3_IP_SVK: {  // zz (from k_zz_lin) in scr[6]; zi in scr[5]; the flag in scr[0]
      const long long np = 2LL * (d.imax - d.imin + 1) * (d.jmax - d.jmin + 1);
      int* flag = (int*)scr[0];
      cudaMemsetAsync(flag, 0, sizeof(int), st);
      k_svk_zi<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s, scr[5]);
      k_svk_cols<R3><<<(int)((np + 127) / 128), 128, 0, st>>>(d, s, scr[6], scr[5], flag, np);
      k_svk_serial<R3><<<1, 1, 0, st>>>(d, s, scr[6], scr[5], flag);
      break;
    }
    case BC3_IP_ZI: {  // zz (from k_zz_lin) in scr[6]; the carried-value records in scr[0..5]
      const long long np = 2LL * (d.imax - d.imin + 1) * (d.jmax - d.jmin + 1);
      const int nb = (int)((np + ZI_SCAN - 1) / ZI_SCAN);
      ZiScr<R3> z{scr[0], scr[4], (int*)scr[1], (int*)scr[5], (int*)scr[2], (int*)scr[3], (int*)scr[3] + nb, np};
      const int g = (int)((np + 127) / 128);
      k_zi_cols<R3, 1><<<g, 128, 0, st>>>(d, s, scr[6], z);
      k_zi_scan_blocks<<<nb, ZI_SCAN, 0, st>>>(z.key_p, z.key_m, z.agg_p, z.agg_m, np);
      k_zi_scan_aggs<<<1, ZI_SCAN, 0, st>>>(z.agg_p, z.agg_m, nb);
      k_zi_cols<R3, 3><<<g, 128, 0, st>>>(d, s, scr[6], z);
      break;
    }
    case BC3_SM_COLS: k_sm_cols<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s, scr[6], scr[0]); break;
    case BC3_IP_SM: k_ip_sm<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s, scr[6], scr[0]); break;
    case BC3_UUMOM:
    case BC3_VVMOM: {
      const int nx = d.imax - d.imin + 1, ny = d.jmax - d.jmin + 1;
      bool done = false;
      if constexpr (sizeof(R3) == 4) {
        if (d.kmax + 1 <= 64) {
          constexpr int NT = 64;
          const dim3 b2(32, 2, 1);
          const dim3 g2((nx + 31) / 32, (ny + 1) / 2, 1);
          const size_t dyn = 2 * (size_t)(d.kmax + 1) * NT * sizeof(R3);
          // a ring of eight levels (six in flight ahead of the elimination): with the coefficients
          // in shared memory a block of 64 columns holds few warps, so each column keeps more of
          // its loads in flight; above 48 KB of shared memory per block the launch opts in
          auto kern = which == BC3_UUMOM ? k_uvmom3d<R3, 0, true, NT, 8> : k_uvmom3d<R3, 1, true, NT, 8>;
          const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
          if (e != cudaSuccess) return (int)e;
          kern<<<g2, b2, dyn, st>>>(d, s, scr[0], scr[1]);
          done = true;
        }
      }
      if (!done) {
        const dim3 b2(32, 4, 1);
        const dim3 g2((nx + 31) / 32, (ny + 3) / 4, 1);
        if (which == BC3_UUMOM)
          k_uvmom3d<R3, 0, false, UVM_THREADS><<<g2, b2, 0, st>>>(d, s, scr[0], scr[1]);
        else
          k_uvmom3d<R3, 1, false, UVM_THREADS><<<g2, b2, 0, st>>>(d, s, scr[0], scr[1]);
      }
      break;
    }
    case BC3_SIGMA: {
      if constexpr (sizeof(R3) == 4) {
        bool ok = vector_sweeps_enabled() && d.sj % 4 == 0 && d.sk % 4 == 0;
        for (int f : {HO, HN, HUO, HUN, HVO, HVN}) ok = ok && reinterpret_cast<uintptr_t>(s.f3[f]) % 16 == 0;
        if (ok) {
          const dim3 gv((d.ni() + 4 * 32 - 1) / (4 * 32), (d.nj() + 3) / 4, 4);
          k_sigma_vec<4><<<gv, dim3(32, 4, 1), 0, st>>>(d, s);
          break;
        }
      }
      k_sigma<R3><<<plane_grid(d, blk, (d.kmax + LVC) / LVC), blk, 0, st>>>(d, s);
      break;
    }
    case BC3_WW: k_ww<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s); break;
    case BC3_UVADV_PREP_U:
    case BC3_UVADV_PREP_V: {
      const bool u = which == BC3_UVADV_PREP_U;
      if constexpr (sizeof(R3) == 4) {
        bool ok = vector_sweeps_enabled() && d.sj % 4 == 0 && d.sk % 4 == 0;
        for (int q = 0; q < 6 && ok; ++q) ok = !scr[q] || reinterpret_cast<uintptr_t>(scr[q]) % 16 == 0;
        for (int f : {UU, VV, WW, HO, HN, HUN, HVN})
          ok = ok && reinterpret_cast<uintptr_t>(s.f3[f]) % 16 == 0;
        if (ok) {
          const dim3 bv(32, 4, 1);
          const dim3 gv((d.ni() + 4 * 32 - 1) / (4 * 32), (d.nj() + 3) / 4, d.kmax + 1);
          if (u) k_uvadv3d_prep_vec<0><<<gv, bv, 0, st>>>(d, s, scr[0], scr[1], scr[2], scr[3], scr[4], scr[5]);
          else k_uvadv3d_prep_vec<1><<<gv, bv, 0, st>>>(d, s, scr[0], scr[1], scr[2], scr[3], scr[4], scr[5]);
          break;
        }
      }
      if (u)
        k_uvadv3d_prep<R3, 0><<<plane_grid(d, blk, d.kmax + 1), blk, 0, st>>>(d, s, scr[0], scr[1], scr[2], scr[3],
                                                                              scr[4], scr[5]);
      else
        k_uvadv3d_prep<R3, 1><<<plane_grid(d, blk, d.kmax + 1), blk, 0, st>>>(d, s, scr[0], scr[1], scr[2], scr[3],
                                                                              scr[4], scr[5]);
      break;
    }
    case BC3_UVADV_PREP_UV: {  // FP32 only: U grid into scr[0..5], V grid into scr[7..12]
      if constexpr (sizeof(R3) == 4) {
        bool ok = vector_sweeps_enabled() && d.sj % 4 == 0 && d.sk % 4 == 0;
        for (int q : {0, 1, 2, 3, 4, 5, 7, 8, 9, 10, 11, 12}) ok = ok && reinterpret_cast<uintptr_t>(scr[q]) % 16 == 0;
        for (int f : {UU, VV, WW, HO, HN, HUN, HVN})
          ok = ok && reinterpret_cast<uintptr_t>(s.f3[f]) % 16 == 0;
        ok = ok && reinterpret_cast<uintptr_t>(colh) % 16 == 0;
        if (ok) {
          const dim3 bv(32, 4, 1);
          const dim3 gv((d.ni() + 4 * 32 - 1) / (4 * 32), (d.nj() + 3) / 4, d.kmax + 1);
          k_uvadv3d_prep_vec2<4><<<gv, bv, 0, st>>>(d, s, Prep6{{scr[0], scr[1], scr[2], scr[3], scr[4], scr[5]}},
                                                    Prep6{{scr[7], scr[8], scr[9], scr[10], scr[11], scr[12]}},
                                                    colh);
        } else {
          k_uvadv3d_prep<R3, 0><<<plane_grid(d, blk, d.kmax + 1), blk, 0, st>>>(d, s, scr[0], scr[1], scr[2],
                                                                                scr[3], scr[4], scr[5]);
          k_uvadv3d_prep<R3, 1><<<plane_grid(d, blk, d.kmax + 1), blk, 0, st>>>(d, s, scr[7], scr[8], scr[9],
                                                                                scr[10], scr[11], scr[12]);
        }
        break;
      } else {
        return (int)cudaErrorInvalidValue;
      }
    }
    case BC3_STRESSES: k_stresses<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s); break;
    case BC3_EQSTATE_UNESCO: k_eqstate_nl<R3, 2><<<plane_grid(d, blk, d.kmax), blk, 0, st>>>(d, s); break;
    case BC3_EQSTATE_JACKETT: k_eqstate_nl<R3, 3><<<plane_grid(d, blk, d.kmax), blk, 0, st>>>(d, s); break;
    case BC3_GOTM_PARABOLIC: {
      const dim3 g((d.imax - d.imin + 1 + 31) / 32, (d.jmax - d.jmin + 1 + 3) / 4, 1);
      k_gotm_parabolic<R3><<<g, blk, 0, st>>>(d, s);
      break;
    }
    case BC3_SW_RADIATION: {
      const dim3 g((d.imax - d.imin + 1 + 31) / 32, (d.jmax - d.jmin + 1 + 3) / 4, 1);
      k_sw_radiation<R3><<<g, blk, 0, st>>>(d, s);
      break;
    }
    case BC3_TEMP_SOURCE: {  // scr[0] = the source array, scr[1] = the top-level salinity (may be null)
      const dim3 g((d.imax - d.imin + 1 + 31) / 32, (d.jmax - d.jmin + 1 + 3) / 4, 1);
      k_temp_source<R3><<<g, blk, 0, st>>>(d, s, scr[1], scr[0]);
      break;
    }
    case BC3_EQSTATE: {
      if constexpr (sizeof(R3) == 4) {
        bool ok = vector_sweeps_enabled() && d.sj % 4 == 0 && d.sk % 4 == 0;
        for (int f : {TT, SS, RHO, BUOY}) ok = ok && reinterpret_cast<uintptr_t>(s.f3[f]) % 16 == 0;
        if (ok) {
          const dim3 gv((d.ni() + 4 * 32 - 1) / (4 * 32), (d.nj() + 3) / 4, d.kmax);
          k_eqstate_vec<4><<<gv, dim3(32, 4, 1), 0, st>>>(d, s);
          break;
        }
      }
      k_eqstate<R3><<<plane_grid(d, blk, d.kmax), blk, 0, st>>>(d, s);
      break;
    }
    case BC3_SLOW_TERMS: k_slow_terms<R3><<<plane_grid(d, blk), blk, 0, st>>>(d, s); break;
    default: return (int)cudaErrorInvalidValue;
  }
  return (int)cudaGetLastError();
}

}  // namespace gb
