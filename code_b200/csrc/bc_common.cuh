// bc_common.cuh -- the state table of the mode-split step as the kernels see it.
// Field order is part of the C ABI (getm_bc_state, include/getm_b200.h).
#pragma once
#include "common.cuh"

namespace gb {

enum F2 {
  Z, ZO, U_, V_, D_, DU, DV, UEX, VEX, FU, FV, RU, RV, RUU, RVV, UINT, VINT, UINTO, VINTO, SLUX, SLVX, SLRU, SLRV,
  ZUB, ZVB, ZUB0, ZVB0, FWF, HH, HU, HV, DRY_Z, DRY_U, DRY_V, CORU, CORV, TAUSX, TAUSY, AIRP, SSEO, SSEN, SSUO,
  SSUN, SSVO, SSVN, DN, DUN, DVN, RRU, RRV, TAUBX, TAUBY, TAUB, TAUS, SWR, SHF, ATT_A, ATT_G1, ATT_G2, NF2
};
enum F3 {
  UU, VV, WW, HO, HN, HUO, HUN, HVO, HVN, UUEX, VVEX, IDPDX, IDPDY, TT, SS, RHO, BUOY, NUM, NUH, RAD, TKE, EPS,
  TLO, SLO, NF3
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
// fields a state may leave NULL: the radiation inputs and output when radiation = 0, tke and eps,
// and the compensated storage of T and S (Tlo, Slo)
constexpr bool optional_f2(int q) { return q == SWR || q == SHF || q == ATT_A || q == ATT_G1 || q == ATT_G2; }
constexpr bool optional_f3(int q) { return q == RAD || q == TKE || q == EPS || q == TLO || q == SLO; }

// 2D part (all FP64) -- passed to kernels by value
struct Bc2 {
  double* f2[NF2];
  const int32_t *az, *au, *av, *ax;
  double par[NPD];
};

// The mixed-precision micro step keeps FP32 working copies of the 2D fields that the barotropic
// kernels read and write every micro step (transports, depths, the momentum terms and the
// forcing; the static depths H, HU, HV, the freshwater flux and the bottom roughness zub0/zvb0 as
// read-only copies; the roughness zub/zvb, which the FP32 bottom friction reads as FP32 and renews
// with FP32 values, written back only when it renews them); the elevation, the accumulated
// transports Uint/Vint and the Coriolis factors stay FP64. The FP64 state is the authoritative
// copy between calls: the copies are filled at the start of getm_time_loop and written back
// before each macro step and at the end.
constexpr bool is_work2(int q) {
  return q == U_ || q == V_ || q == D_ || q == DU || q == DV || q == DRY_U || q == DRY_V || q == FU || q == FV ||
         q == RU || q == RV || q == RUU || q == RVV || q == UEX || q == VEX || q == SLUX || q == SLVX ||
         q == SLRU || q == SLRV || q == TAUSX || q == TAUSY || q == AIRP || q == HH || q == HU || q == HV ||
         q == FWF || q == ZUB || q == ZVB || q == ZUB0 || q == ZVB0;
}
struct Bc2W {
  float* w[NF2];         // FP32 working copy of field q (used where is_work2(q))
  const uint8_t* m8[3];  // uint8 copies of the masks az, au, av (their values are 0..3)
};

template <class R3>
struct Bc3 {
  double* f2[NF2];
  R3* f3[NF3];
  const int32_t *az, *au, *av, *ax;
  double par[NPD];
};

// number of 3D / 2D scratch arrays of the mode-split step
constexpr int NB3 = 7;   // fadv, uuadv, vvadv, wwadv, huadv, hvadv, zz
constexpr int NB3F = 13; // FP32: the same, then the V grid's six (both grids prepared in one pass)
// planes of the column heights (k_col_heights)
enum { COL_HO, COL_HN, COL_HUN, COL_HVN, COL_HUA_U, COL_HVA_U, COL_HUA_V, COL_HVA_V, NCOLH };
constexpr int NB2 = 10;  // fadv, Uadv, Vadv, DUadv, DVadv, Di, adv, S, Ui, Vi

}  // namespace gb
