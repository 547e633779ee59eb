// BSIM3 v3.2.2 (levels 9 / 49): set-up interface and the per-instance load.
//
// Restates, in the reference's order of floating-point operations:
//   model card and Model::processParams      src/DeviceModelPKG/OpenModels/src/N_DEV_MOSFET_B3.C:204-1820, 8458-8548, 8573-9080
//   Instance::processParams / constructor    N_DEV_MOSFET_B3.C:1845-1880, 2440-2500
//   Instance::updateTemperature              N_DEV_MOSFET_B3.C:3593-4488
//   Instance::updateIntermediateVars         N_DEV_MOSFET_B3.C:4496-7246
//   setupCapacitors_oldDAE / _newDAE         N_DEV_MOSFET_B3.C:7610-7867, 7544-7608
//   auxChargeCalculations                    N_DEV_MOSFET_B3.C:7447-7542
//   Master::updateState                      N_DEV_MOSFET_B3.C:9199-9270
//   Master::loadDAEVectors / loadDAEMatrices N_DEV_MOSFET_B3.C:9276-9613, 9624-9900
// for nqsMod = 0, capMod 0, 1, 2 or 3 and no instance initial conditions: the 4-terminal stamp in
// the BSIM4 load's staged layout, or with drain / source sheet resistance (RSH * NRD, RSH * NRS)
// the stamp on (D', G, S', B) plus the resistor couplings in the wide layout.
#pragma once

#include <string>
#include <vector>

#include "bsim4_eval.cuh"  // LoadFlags, RecPtr, staged layout constants
#include "bsim4_setup.h"   // ModelSpec, SetupOptions, RecordTable
#include "xd_consts.h"
#include "mos_cv.h"

#define XB3_FIELDS(F)                                                                               \
  /* model-level */                                                                                 \
  F(dtype) F(mobMod) F(capMod) F(xpart) F(tox) F(cox) F(factor1) F(vcrit) F(ijth)                   \
  /* temperature and instance */                                                                    \
  F(vtm) F(TempRatio) F(Nvtm) F(SourceSatCurrent) F(DrainSatCurrent) F(vjsm) F(IsEvjsm) F(vjdm)       \
  F(IsEvjdm) F(czbd) F(czbs) F(czbdsw) F(czbdswg) F(czbssw) F(czbsswg) F(PhiBTemp) F(PhiBSWTemp)    \
  F(PhiBSWGTemp) F(MJ) F(MJSW) F(MJSWG) F(mult) F(off) F(drainConductance) F(sourceConductance)   \
  /* size-binned and size-derived */                                                                \
  F(vbsc) F(phi) F(phis3) F(sqrtPhi) F(Xdep0) F(vbi) F(dvt2) F(dvt2w) F(dvt1) F(dvt0) F(dvt1w)       \
  F(dvt0w) F(weff) F(leff) F(nlx) F(k1ox) F(k2ox) F(kt1) F(kt1l) F(kt2) F(w0) F(eta0) F(etab)        \
  F(theta0vb0) F(vth0) F(k1) F(k3) F(k3b) F(nfactor) F(cdsc) F(cdscb) F(cdscd) F(cit) F(vfb) F(ngate) \
  F(voff) F(cdep0) F(dwg) F(dwb) F(rds0) F(prwg) F(prwb) F(xj) F(a0) F(ags) F(b0) F(b1) F(keta) F(ua) \
  F(ub) F(uc) F(u0temp) F(vsattemp) F(a1) F(a2) F(delta) F(pclm) F(litl) F(thetaRout) F(pdiblb)      \
  F(pvag) F(pscbe1) F(pscbe2) F(alpha0) F(alpha1) F(beta0) F(weffCV) F(leffCV) F(noff) F(voffcv)     \
  F(vfbzb) F(vfbcv) F(abulkCVfactor) F(acde) F(ldeb) F(moin) F(cgdo) F(cgso) F(cgbo) F(cgdl) F(cgsl) F(ckappa)

namespace xb3 {

enum Field {
#define XB3_ENUM(n) f_##n,
  XB3_FIELDS(XB3_ENUM)
#undef XB3_ENUM
  kNumFields
};

// Store slots (registerStoreLIDs order, N_DEV_MOSFET_B3.C:3058-3088) and the state slots the
// nqsMod = 0 load writes (registerStateLIDs order, :2993-3056; the reference reserves 12 state
// entries per instance, of which the first five carry these charges).
enum StoreSlot { s_vbd, s_vbs, s_vgs, s_vds, s_von, kNumStore };
enum StateSlot { t_qb, t_qg, t_qd, t_qbs, t_qbd, kNumState };

std::string build_records(const std::vector<xb4::ModelSpec> &models, int n_inst, const int *inst_model,
                          const std::vector<std::string> &inst_param_names, const double *inst_param_values,
                          const xb4::SetupOptions &opts, xb4::RecordTable &out);

struct LoadOut {
  double vec[xb4::kNumVec];
  double jf[xb4::kNumMat];
  double jq[xb4::kNumMat];
  double sto[kNumStore];
  double sta[kNumState];
  // With internal nodes (the BSIM4 wide layout): F at the external drain and source, dF/dx at
  // (D', D), (D, D'), (D, D), (S', S), (S, S'), (S, S).
  double vecx[2];
  double jfx[6];
};

// One BSIM3 instance. V = terminal voltages (D, G, S, B); sto_old = limiter history (currSto on
// Newton step 0, nextSto otherwise).
// SERIES = true: V holds (D', G, S', B) and Vx the external (D, S); the sheet-resistance
// resistors (N_DEV_MOSFET_B3.C:1849-1861, 7235-7236) load into vecx / jfx.
template <bool SERIES = false, class RV>
XD_HD void bsim3_load(const RV &P_, const double V[4], const double *sto_old, const xb4::LoadFlags &fl,
                      LoadOut &o, const double *Vx = nullptr) {
  using namespace xdc;
#define P(x) P_(f_##x)
  const double dtype = P(dtype);
  const double gmin = fl.gmin;
  const double M = P(mult);
  const bool OFF = P(off) != 0.0;
  const bool ChargeComputationNeeded = fl.tranop || fl.acop || fl.transient;

  // Node and branch voltages (:4690-4760).
  const double Vdp = V[0], Vg = V[1], Vsp = V[2], Vb = V[3];
  const double Vd = SERIES ? Vx[0] : Vdp, Vs = SERIES ? Vx[1] : Vsp;
  const double Vddp = Vd - Vdp, Vssp = Vs - Vsp;
  (void)Vddp; (void)Vssp;
  const double Vbsp = Vb - Vsp;
  const double Vgsp = Vg - Vsp;
  const double Vdpsp = Vdp - Vsp;
  double vbs = dtype * Vbsp;
  double vgs = dtype * Vgsp;
  double vds = dtype * Vdpsp;
  double vbd = vbs - vds;
  double vgd = vgs - vds;
  int origFlag = 1;
  const double vgs_orig = vgs, vds_orig = vds, vbs_orig = vbs, vbd_orig = vbd, vgd_orig = vgd;

  // Initial conditions and limiting (:4770-4960).
  if (fl.init_jct && !OFF && fl.voltlim) {
    vbs = 0.0;
    vgs = dtype * P(vth0) + 0.1;
    vds = 0.1;
    origFlag = 0;
    vbd = vbs - vds;
    vgd = vgs - vds;
  } else if ((fl.init_fix || fl.init_jct) && OFF) {
    vbs = vgs = vds = 0;
  }
  double vbs_old, vbd_old, vgs_old, vds_old, von_local;
  if (fl.newton_iter == 0 && fl.dcop) {
    vbs_old = vbs;
    vbd_old = vbd;
    vgs_old = vgs;
    vds_old = vds;
    von_local = 0.0;
  } else {
    vbs_old = sto_old[s_vbs];
    vbd_old = sto_old[s_vbd];
    vgs_old = sto_old[s_vgs];
    vds_old = sto_old[s_vds];
    von_local = sto_old[s_von];
  }
  const double vgdo = vgs_old - vds_old;
  if (fl.voltlim && !(fl.init_fix && OFF)) {
    int Check = 1;
    if (vds_old >= 0.0) {
      vgs = fetlim(vgs, vgs_old, von_local);
      vds = vgs - vgd;
      vds = limvds(vds, vds_old);
      vgd = vgs - vds;
    } else {
      vgd = fetlim(vgd, vgdo, von_local);
      vds = vgs - vgd;
      vds = -limvds(-vds, -vds_old);
      vgs = vgd + vds;
    }
    if (vds >= 0.0) {
      vbs = pnjlim(vbs, vbs_old, CONSTvt0, P(vcrit), &Check);
      vbd = vbs - vds;
    } else {
      vbd = pnjlim(vbd, vbd_old, CONSTvt0, P(vcrit), &Check);
      vbs = vbd + vds;
    }
    if (vgs_orig != vgs || vds_orig != vds || vbs_orig != vbs || vbd_orig != vbd || vgd_orig != vgd) origFlag = 0;
  }
  vbd = vbs - vds;
  vgd = vgs - vds;
  const double vgb = vgs - vbs;

  // Junction diodes (:5000-5110).
  const double Nvtm = P(Nvtm);
  double gbs, cbs, gbd, cbd;
  {
    const double SourceSatCurrent = P(SourceSatCurrent);
    if (SourceSatCurrent <= 0.0) {
      gbs = gmin;
      cbs = gbs * vbs;
    } else if (P(ijth) == 0.0) {
      const double evbs = exp(vbs / Nvtm);
      gbs = SourceSatCurrent * evbs / Nvtm + gmin;
      cbs = SourceSatCurrent * (evbs - 1.0) + gmin * vbs;
    } else if (vbs < P(vjsm)) {
      const double evbs = exp(vbs / Nvtm);
      gbs = SourceSatCurrent * evbs / Nvtm + gmin;
      cbs = SourceSatCurrent * (evbs - 1.0) + gmin * vbs;
    } else {
      const double T0 = P(IsEvjsm) / Nvtm;
      gbs = T0 + gmin;
      cbs = P(IsEvjsm) - SourceSatCurrent + T0 * (vbs - P(vjsm)) + gmin * vbs;
    }
    const double DrainSatCurrent = P(DrainSatCurrent);
    if (DrainSatCurrent <= 0.0) {
      gbd = gmin;
      cbd = gbd * vbd;
    } else if (P(ijth) == 0.0) {
      const double evbd = exp(vbd / Nvtm);
      gbd = DrainSatCurrent * evbd / Nvtm + gmin;
      cbd = DrainSatCurrent * (evbd - 1.0) + gmin * vbd;
    } else if (vbd < P(vjdm)) {
      const double evbd = exp(vbd / Nvtm);
      gbd = DrainSatCurrent * evbd / Nvtm + gmin;
      cbd = DrainSatCurrent * (evbd - 1.0) + gmin * vbd;
    } else {
      const double T0 = P(IsEvjdm) / Nvtm;
      gbd = T0 + gmin;
      cbd = P(IsEvjdm) - DrainSatCurrent + T0 * (vbd - P(vjdm)) + gmin * vbd;
    }
  }

  int mode;
  double Vds, Vgs, Vbs;
  if (vds >= 0.0) {
    mode = 1;
    Vds = vds;
    Vgs = vgs;
    Vbs = vbs;
  } else {
    mode = -1;
    Vds = -vds;
    Vgs = vgd;
    Vbs = vbd;
  }

  double T0, T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12, tmp, tmp1, tmp2, tmp3, tmp4;
  double dT0_dVg, dT0_dVd, dT0_dVb, dT1_dVg, dT1_dVd, dT1_dVb, dT2_dVg, dT2_dVd, dT2_dVb, dT3_dVg, dT3_dVd,
      dT3_dVb;
  // Effective body bias, surface potential, depletion width (:5155-5185).
  const double vbsc = P(vbsc), phi = P(phi), sqrtPhi = P(sqrtPhi);
  T0 = Vbs - vbsc - 0.001;
  T1 = sqrt(T0 * T0 - 0.004 * vbsc);
  double Vbseff = vbsc + 0.5 * (T0 + T1);
  double dVbseff_dVb = 0.5 * (1.0 + T0 / T1);
  if (Vbseff < Vbs) Vbseff = Vbs;
  double Phis, dPhis_dVb, sqrtPhis, dsqrtPhis_dVb;
  if (Vbseff > 0.0) {
    T0 = phi / (phi + Vbseff);
    Phis = phi * T0;
    dPhis_dVb = -T0 * T0;
    sqrtPhis = P(phis3) / (phi + 0.5 * Vbseff);
    dsqrtPhis_dVb = -0.5 * sqrtPhis * sqrtPhis / P(phis3);
  } else {
    Phis = phi - Vbseff;
    dPhis_dVb = -1.0;
    sqrtPhis = sqrt(Phis);
    dsqrtPhis_dVb = -0.5 / sqrtPhis;
  }
  const double Xdep = P(Xdep0) * sqrtPhis / sqrtPhi;
  const double dXdep_dVb = (P(Xdep0) / sqrtPhi) * dsqrtPhis_dVb;
  const double Leff = P(leff);
  const double Vtm = P(vtm);
  const double factor1 = P(factor1);

  // Threshold voltage (:5186-5290).
  T3 = sqrt(Xdep);
  const double V0 = P(vbi) - phi;
  T0 = P(dvt2) * Vbseff;
  if (T0 >= -0.5) {
    T1 = 1.0 + T0;
    T2 = P(dvt2);
  } else {
    T4 = 1.0 / (3.0 + 8.0 * T0);
    T1 = (1.0 + 3.0 * T0) * T4;
    T2 = P(dvt2) * T4 * T4;
  }
  const double lt1 = factor1 * T3 * T1;
  const double dlt1_dVb = factor1 * (0.5 / T3 * T1 * dXdep_dVb + T3 * T2);
  T0 = P(dvt2w) * Vbseff;
  if (T0 >= -0.5) {
    T1 = 1.0 + T0;
    T2 = P(dvt2w);
  } else {
    T4 = 1.0 / (3.0 + 8.0 * T0);
    T1 = (1.0 + 3.0 * T0) * T4;
    T2 = P(dvt2w) * T4 * T4;
  }
  const double ltw = factor1 * T3 * T1;
  const double dltw_dVb = factor1 * (0.5 / T3 * T1 * dXdep_dVb + T3 * T2);
  double Theta0, dTheta0_dVb;
  T0 = -0.5 * P(dvt1) * Leff / lt1;
  if (T0 > -CONSTEXP_THRESHOLD) {
    T1 = exp(T0);
    Theta0 = T1 * (1.0 + 2.0 * T1);
    dT1_dVb = -T0 / lt1 * T1 * dlt1_dVb;
    dTheta0_dVb = (1.0 + 4.0 * T1) * dT1_dVb;
  } else {
    T1 = CONSTMIN_EXP;
    Theta0 = T1 * (1.0 + 2.0 * T1);
    dTheta0_dVb = 0.0;
  }
  const double thetavth = P(dvt0) * Theta0;
  const double Delt_vth = thetavth * V0;
  const double dDelt_vth_dVb = P(dvt0) * dTheta0_dVb * V0;
  T0 = -0.5 * P(dvt1w) * P(weff) * Leff / ltw;
  if (T0 > -CONSTEXP_THRESHOLD) {
    T1 = exp(T0);
    T2 = T1 * (1.0 + 2.0 * T1);
    dT1_dVb = -T0 / ltw * T1 * dltw_dVb;
    dT2_dVb = (1.0 + 4.0 * T1) * dT1_dVb;
  } else {
    T1 = CONSTMIN_EXP;
    T2 = T1 * (1.0 + 2.0 * T1);
    dT2_dVb = 0.0;
  }
  T0 = P(dvt0w) * T2;
  T2 = T0 * V0;
  dT2_dVb = P(dvt0w) * dT2_dVb * V0;
  const double TempRatio = P(TempRatio);
  T0 = sqrt(1.0 + P(nlx) / Leff);
  T1 = P(k1ox) * (T0 - 1.0) * sqrtPhi + (P(kt1) + P(kt1l) / Leff + P(kt2) * Vbseff) * TempRatio;
  tmp2 = P(tox) * phi / (P(weff) + P(w0));
  T3 = P(eta0) + P(etab) * Vbseff;
  if (T3 < 1.0e-4) {
    T9 = 1.0 / (3.0 - 2.0e4 * T3);
    T3 = (2.0e-4 - T3) * T9;
    T4 = T9 * T9;
  } else {
    T4 = 1.0;
  }
  const double dDIBL_Sft_dVd = T3 * P(theta0vb0);
  const double DIBL_Sft = dDIBL_Sft_dVd * Vds;
  double Vth = dtype * P(vth0) - P(k1) * sqrtPhi + P(k1ox) * sqrtPhis - P(k2ox) * Vbseff - Delt_vth - T2 +
               (P(k3) + P(k3b) * Vbseff) * tmp2 + T1 - DIBL_Sft;
  const double von = Vth;
  double dVth_dVb = P(k1ox) * dsqrtPhis_dVb - P(k2ox) - dDelt_vth_dVb - dT2_dVb + P(k3b) * tmp2 -
                    P(etab) * Vds * P(theta0vb0) * T4 + P(kt2) * TempRatio;
  const double dVth_dVd = -dDIBL_Sft_dVd;

  // Subthreshold swing factor n (:5291-5312).
  const double cox = P(cox);
  double n, dn_dVb, dn_dVd;
  tmp2 = P(nfactor) * CONSTEPSSI / Xdep;
  tmp3 = P(cdsc) + P(cdscb) * Vbseff + P(cdscd) * Vds;
  tmp4 = (tmp2 + tmp3 * Theta0 + P(cit)) / cox;
  if (tmp4 >= -0.5) {
    n = 1.0 + tmp4;
    dn_dVb = (-tmp2 / Xdep * dXdep_dVb + tmp3 * dTheta0_dVb + P(cdscb) * Theta0) / cox;
    dn_dVd = P(cdscd) * Theta0 / cox;
  } else {
    T0 = 1.0 / (3.0 + 8.0 * tmp4);
    n = (1.0 + 3.0 * tmp4) * T0;
    T0 *= T0;
    dn_dVb = (-tmp2 / Xdep * dXdep_dVb + tmp3 * dTheta0_dVb + P(cdscb) * Theta0) / cox * T0;
    dn_dVd = P(cdscd) * Theta0 / cox * T0;
  }

  // Poly-gate depletion (:5313-5335).
  double Vgs_eff, dVgs_eff_dVg;
  T0 = P(vfb) + phi;
  if ((P(ngate) > 1.e18) && (P(ngate) < 1.e25) && (Vgs > T0)) {
    T1 = 1.0e6 * CONSTQ * CONSTEPSSI * P(ngate) / (cox * cox);
    T4 = sqrt(1.0 + 2.0 * (Vgs - T0) / T1);
    T2 = T1 * (T4 - 1.0);
    T3 = 0.5 * T2 * T2 / T1;
    T7 = 1.12 - T3 - 0.05;
    T6 = sqrt(T7 * T7 + 0.224);
    T5 = 1.12 - 0.5 * (T7 + T6);
    Vgs_eff = Vgs - T5;
    dVgs_eff_dVg = 1.0 - (0.5 - 0.5 / T4) * (1.0 + T7 / T6);
  } else {
    Vgs_eff = Vgs;
    dVgs_eff_dVg = 1.0;
  }
  double Vgst = Vgs_eff - Vth;

  // Effective Vgst (Vgsteff) for I-V (:5336-5380).
  double Vgsteff, dVgsteff_dVg, dVgsteff_dVd, dVgsteff_dVb;
  T10 = 2.0 * n * Vtm;
  double VgstNVt = Vgst / T10;
  const double ExpArg = (2.0 * P(voff) - Vgst) / T10;
  if (VgstNVt > CONSTEXP_THRESHOLD) {
    Vgsteff = Vgst;
    dVgsteff_dVg = dVgs_eff_dVg;
    dVgsteff_dVd = -dVth_dVd;
    dVgsteff_dVb = -dVth_dVb;
  } else if (ExpArg > CONSTEXP_THRESHOLD) {
    T0 = (Vgst - P(voff)) / (n * Vtm);
    const double ExpVgst = exp(T0);
    Vgsteff = Vtm * P(cdep0) / cox * ExpVgst;
    dVgsteff_dVg = Vgsteff / (n * Vtm);
    dVgsteff_dVd = -dVgsteff_dVg * (dVth_dVd + T0 * Vtm * dn_dVd);
    dVgsteff_dVb = -dVgsteff_dVg * (dVth_dVb + T0 * Vtm * dn_dVb);
    dVgsteff_dVg *= dVgs_eff_dVg;
  } else {
    const double ExpVgst = exp(VgstNVt);
    T1 = T10 * log(1.0 + ExpVgst);
    dT1_dVg = ExpVgst / (1.0 + ExpVgst);
    dT1_dVb = -dT1_dVg * (dVth_dVb + Vgst / n * dn_dVb) + T1 / n * dn_dVb;
    dT1_dVd = -dT1_dVg * (dVth_dVd + Vgst / n * dn_dVd) + T1 / n * dn_dVd;
    dT2_dVg = -cox / (Vtm * P(cdep0)) * exp(ExpArg);
    T2 = 1.0 - T10 * dT2_dVg;
    dT2_dVd = -dT2_dVg * (dVth_dVd - 2.0 * Vtm * ExpArg * dn_dVd) + (T2 - 1.0) / n * dn_dVd;
    dT2_dVb = -dT2_dVg * (dVth_dVb - 2.0 * Vtm * ExpArg * dn_dVb) + (T2 - 1.0) / n * dn_dVb;
    Vgsteff = T1 / T2;
    T3 = T2 * T2;
    dVgsteff_dVg = (T2 * dT1_dVg - T1 * dT2_dVg) / T3 * dVgs_eff_dVg;
    dVgsteff_dVd = (T2 * dT1_dVd - T1 * dT2_dVd) / T3;
    dVgsteff_dVb = (T2 * dT1_dVb - T1 * dT2_dVb) / T3;
  }

  // Effective width and source/drain resistance (:5381-5410).
  T9 = sqrtPhis - sqrtPhi;
  double Weff = P(weff) - 2.0 * (P(dwg) * Vgsteff + P(dwb) * T9);
  double dWeff_dVg = -2.0 * P(dwg);
  double dWeff_dVb = -2.0 * P(dwb) * dsqrtPhis_dVb;
  if (Weff < 2.0e-8) {
    T0 = 1.0 / (6.0e-8 - 2.0 * Weff);
    Weff = 2.0e-8 * (4.0e-8 - Weff) * T0;
    T0 *= T0 * 4.0e-16;
    dWeff_dVg *= T0;
    dWeff_dVb *= T0;
  }
  double Rds, dRds_dVg, dRds_dVb;
  const double rds0 = P(rds0);
  T0 = P(prwg) * Vgsteff + P(prwb) * T9;
  if (T0 >= -0.9) {
    Rds = rds0 * (1.0 + T0);
    dRds_dVg = rds0 * P(prwg);
    dRds_dVb = rds0 * P(prwb) * dsqrtPhis_dVb;
  } else {
    T1 = 1.0 / (17.0 + 20.0 * T0);
    Rds = rds0 * (0.8 + T0) * T1;
    T1 *= T1;
    dRds_dVg = rds0 * P(prwg) * T1;
    dRds_dVb = rds0 * P(prwb) * dsqrtPhis_dVb * T1;
  }

  // Bulk charge factor Abulk (:5411-5460).
  T1 = 0.5 * P(k1ox) / sqrtPhis;
  dT1_dVb = -T1 / sqrtPhis * dsqrtPhis_dVb;
  T9 = sqrt(P(xj) * Xdep);
  tmp1 = Leff + 2.0 * T9;
  T5 = Leff / tmp1;
  tmp2 = P(a0) * T5;
  tmp3 = P(weff) + P(b1);
  tmp4 = P(b0) / tmp3;
  T2 = tmp2 + tmp4;
  dT2_dVb = -T9 / tmp1 / Xdep * dXdep_dVb;
  T6 = T5 * T5;
  T7 = T5 * T6;
  double Abulk0 = 1.0 + T1 * T2;
  double dAbulk0_dVb = T1 * tmp2 * dT2_dVb + T2 * dT1_dVb;
  T8 = P(ags) * P(a0) * T7;
  double dAbulk_dVg = -T1 * T8;
  double Abulk = Abulk0 + dAbulk_dVg * Vgsteff;
  double dAbulk_dVb = dAbulk0_dVb - T8 * Vgsteff * (dT1_dVb + 3.0 * T1 * dT2_dVb);
  if (Abulk0 < 0.1) {
    T9 = 1.0 / (3.0 - 20.0 * Abulk0);
    Abulk0 = (0.2 - Abulk0) * T9;
    dAbulk0_dVb *= T9 * T9;
  }
  if (Abulk < 0.1) {
    T9 = 1.0 / (3.0 - 20.0 * Abulk);
    Abulk = (0.2 - Abulk) * T9;
    T10 = T9 * T9;
    dAbulk_dVb *= T10;
    dAbulk_dVg *= T10;
  }
  T2 = P(keta) * Vbseff;
  if (T2 >= -0.9) {
    T0 = 1.0 / (1.0 + T2);
    dT0_dVb = -P(keta) * T0 * T0;
  } else {
    T1 = 1.0 / (0.8 + T2);
    T0 = (17.0 + 20.0 * T2) * T1;
    dT0_dVb = -P(keta) * T1 * T1;
  }
  dAbulk_dVg *= T0;
  dAbulk_dVb = dAbulk_dVb * T0 + Abulk * dT0_dVb;
  dAbulk0_dVb = dAbulk0_dVb * T0 + Abulk0 * dT0_dVb;
  Abulk *= T0;
  Abulk0 *= T0;

  // Mobility (:5461-5510).
  const double tox = P(tox);
  const int mobMod = (int)P(mobMod);
  double Denomi, dDenomi_dVg, dDenomi_dVd, dDenomi_dVb;
  if (mobMod == 1) {
    T0 = Vgsteff + Vth + Vth;
    T2 = P(ua) + P(uc) * Vbseff;
    T3 = T0 / tox;
    T5 = T3 * (T2 + P(ub) * T3);
    dDenomi_dVg = (T2 + 2.0 * P(ub) * T3) / tox;
    dDenomi_dVd = dDenomi_dVg * 2.0 * dVth_dVd;
    dDenomi_dVb = dDenomi_dVg * 2.0 * dVth_dVb + P(uc) * T3;
  } else if (mobMod == 2) {
    T5 = Vgsteff / tox * (P(ua) + P(uc) * Vbseff + P(ub) * Vgsteff / tox);
    dDenomi_dVg = (P(ua) + P(uc) * Vbseff + 2.0 * P(ub) * Vgsteff / tox) / tox;
    dDenomi_dVd = 0.0;
    dDenomi_dVb = Vgsteff * P(uc) / tox;
  } else {
    T0 = Vgsteff + Vth + Vth;
    T2 = 1.0 + P(uc) * Vbseff;
    T3 = T0 / tox;
    T4 = T3 * (P(ua) + P(ub) * T3);
    T5 = T4 * T2;
    dDenomi_dVg = (P(ua) + 2.0 * P(ub) * T3) * T2 / tox;
    dDenomi_dVd = dDenomi_dVg * 2.0 * dVth_dVd;
    dDenomi_dVb = dDenomi_dVg * 2.0 * dVth_dVb + P(uc) * T4;
  }
  if (T5 >= -0.8) {
    Denomi = 1.0 + T5;
  } else {
    T9 = 1.0 / (7.0 + 10.0 * T5);
    Denomi = (0.6 + T5) * T9;
    T9 *= T9;
    dDenomi_dVg *= T9;
    dDenomi_dVd *= T9;
    dDenomi_dVb *= T9;
  }
  const double ueff = P(u0temp) / Denomi;
  T9 = -ueff / Denomi;
  const double dueff_dVg = T9 * dDenomi_dVg;
  const double dueff_dVd = T9 * dDenomi_dVd;
  const double dueff_dVb = T9 * dDenomi_dVb;

  // Saturation field, Lambda, Vdsat (:5511-5640).
  const double vsattemp = P(vsattemp);
  const double WVCox = Weff * vsattemp * cox;
  const double WVCoxRds = WVCox * Rds;
  const double Esat = 2.0 * vsattemp / ueff;
  const double EsatL = Esat * Leff;
  T0 = -EsatL / ueff;
  const double dEsatL_dVg = T0 * dueff_dVg;
  const double dEsatL_dVd = T0 * dueff_dVd;
  const double dEsatL_dVb = T0 * dueff_dVb;
  double Lambda, dLambda_dVg;
  const double a1 = P(a1);
  if (a1 == 0.0) {
    Lambda = P(a2);
    dLambda_dVg = 0.0;
  } else if (a1 > 0.0) {
    T0 = 1.0 - P(a2);
    T1 = T0 - P(a1) * Vgsteff - 0.0001;
    T2 = sqrt(T1 * T1 + 0.0004 * T0);
    Lambda = P(a2) + T0 - 0.5 * (T1 + T2);
    dLambda_dVg = 0.5 * P(a1) * (1.0 + T1 / T2);
  } else {
    T1 = P(a2) + P(a1) * Vgsteff - 0.0001;
    T2 = sqrt(T1 * T1 + 0.0004 * P(a2));
    Lambda = 0.5 * (T1 + T2);
    dLambda_dVg = 0.5 * P(a1) * (1.0 + T1 / T2);
  }
  const double Vgst2Vtm = Vgsteff + 2.0 * Vtm;
  if (Rds > 0) {
    tmp2 = dRds_dVg / Rds + dWeff_dVg / Weff;
    tmp3 = dRds_dVb / Rds + dWeff_dVb / Weff;
  } else {
    tmp2 = dWeff_dVg / Weff;
    tmp3 = dWeff_dVb / Weff;
  }
  double Vdsat, dVdsat_dVg, dVdsat_dVd, dVdsat_dVb;
  if ((Rds == 0.0) && (Lambda == 1.0)) {
    T0 = 1.0 / (Abulk * EsatL + Vgst2Vtm);
    tmp1 = 0.0;
    T1 = T0 * T0;
    T2 = Vgst2Vtm * T0;
    T3 = EsatL * Vgst2Vtm;
    Vdsat = T3 * T0;
    dT0_dVg = -(Abulk * dEsatL_dVg + EsatL * dAbulk_dVg + 1.0) * T1;
    dT0_dVd = -(Abulk * dEsatL_dVd) * T1;
    dT0_dVb = -(Abulk * dEsatL_dVb + dAbulk_dVb * EsatL) * T1;
    dVdsat_dVg = T3 * dT0_dVg + T2 * dEsatL_dVg + EsatL * T0;
    dVdsat_dVd = T3 * dT0_dVd + T2 * dEsatL_dVd;
    dVdsat_dVb = T3 * dT0_dVb + T2 * dEsatL_dVb;
  } else {
    tmp1 = dLambda_dVg / (Lambda * Lambda);
    T9 = Abulk * WVCoxRds;
    T8 = Abulk * T9;
    T7 = Vgst2Vtm * T9;
    T6 = Vgst2Vtm * WVCoxRds;
    T0 = 2.0 * Abulk * (T9 - 1.0 + 1.0 / Lambda);
    dT0_dVg = 2.0 * (T8 * tmp2 - Abulk * tmp1 + (2.0 * T9 + 1.0 / Lambda - 1.0) * dAbulk_dVg);
    dT0_dVb = 2.0 * (T8 * (2.0 / Abulk * dAbulk_dVb + tmp3) + (1.0 / Lambda - 1.0) * dAbulk_dVb);
    dT0_dVd = 0.0;
    T1 = Vgst2Vtm * (2.0 / Lambda - 1.0) + Abulk * EsatL + 3.0 * T7;
    dT1_dVg = (2.0 / Lambda - 1.0) - 2.0 * Vgst2Vtm * tmp1 + Abulk * dEsatL_dVg + EsatL * dAbulk_dVg +
              3.0 * (T9 + T7 * tmp2 + T6 * dAbulk_dVg);
    dT1_dVb = Abulk * dEsatL_dVb + EsatL * dAbulk_dVb + 3.0 * (T6 * dAbulk_dVb + T7 * tmp3);
    dT1_dVd = Abulk * dEsatL_dVd;
    T2 = Vgst2Vtm * (EsatL + 2.0 * T6);
    dT2_dVg = EsatL + Vgst2Vtm * dEsatL_dVg + T6 * (4.0 + 2.0 * Vgst2Vtm * tmp2);
    dT2_dVb = Vgst2Vtm * (dEsatL_dVb + 2.0 * T6 * tmp3);
    dT2_dVd = Vgst2Vtm * dEsatL_dVd;
    T3 = sqrt(T1 * T1 - 2.0 * T0 * T2);
    Vdsat = (T1 - T3) / T0;
    dT3_dVg = (T1 * dT1_dVg - 2.0 * (T0 * dT2_dVg + T2 * dT0_dVg)) / T3;
    dT3_dVd = (T1 * dT1_dVd - 2.0 * (T0 * dT2_dVd + T2 * dT0_dVd)) / T3;
    dT3_dVb = (T1 * dT1_dVb - 2.0 * (T0 * dT2_dVb + T2 * dT0_dVb)) / T3;
    (void)dT3_dVg;
    (void)dT3_dVd;
    (void)dT3_dVb;
    dVdsat_dVg = (dT1_dVg - (T1 * dT1_dVg - dT0_dVg * T2 - T0 * dT2_dVg) / T3 - Vdsat * dT0_dVg) / T0;
    dVdsat_dVb = (dT1_dVb - (T1 * dT1_dVb - dT0_dVb * T2 - T0 * dT2_dVb) / T3 - Vdsat * dT0_dVb) / T0;
    dVdsat_dVd = (dT1_dVd - (T1 * dT1_dVd - T0 * dT2_dVd) / T3) / T0;
  }

  // Effective Vds (:5641-5665).
  const double delta = P(delta);
  T1 = Vdsat - Vds - delta;
  dT1_dVg = dVdsat_dVg;
  dT1_dVd = dVdsat_dVd - 1.0;
  dT1_dVb = dVdsat_dVb;
  T2 = sqrt(T1 * T1 + 4.0 * delta * Vdsat);
  T0 = T1 / T2;
  T3 = 2.0 * delta / T2;
  dT2_dVg = T0 * dT1_dVg + T3 * dVdsat_dVg;
  dT2_dVd = T0 * dT1_dVd + T3 * dVdsat_dVd;
  dT2_dVb = T0 * dT1_dVb + T3 * dVdsat_dVb;
  double Vdseff = Vdsat - 0.5 * (T1 + T2);
  double dVdseff_dVg = dVdsat_dVg - 0.5 * (dT1_dVg + dT2_dVg);
  const double dVdseff_dVd = dVdsat_dVd - 0.5 * (dT1_dVd + dT2_dVd);
  double dVdseff_dVb = dVdsat_dVb - 0.5 * (dT1_dVb + dT2_dVb);
  if (Vds == 0.0) {
    Vdseff = 0.0;
    dVdseff_dVg = 0.0;
    dVdseff_dVb = 0.0;
  }

  // Vasat (:5666-5700).
  tmp4 = 1.0 - 0.5 * Abulk * Vdsat / Vgst2Vtm;
  T9 = WVCoxRds * Vgsteff;
  T8 = T9 / Vgst2Vtm;
  T0 = EsatL + Vdsat + 2.0 * T9 * tmp4;
  T7 = 2.0 * WVCoxRds * tmp4;
  dT0_dVg = dEsatL_dVg + dVdsat_dVg + T7 * (1.0 + tmp2 * Vgsteff) -
            T8 * (Abulk * dVdsat_dVg - Abulk * Vdsat / Vgst2Vtm + Vdsat * dAbulk_dVg);
  dT0_dVb = dEsatL_dVb + dVdsat_dVb + T7 * tmp3 * Vgsteff - T8 * (dAbulk_dVb * Vdsat + Abulk * dVdsat_dVb);
  dT0_dVd = dEsatL_dVd + dVdsat_dVd - T8 * Abulk * dVdsat_dVd;
  T9 = WVCoxRds * Abulk;
  T1 = 2.0 / Lambda - 1.0 + T9;
  dT1_dVg = -2.0 * tmp1 + WVCoxRds * (Abulk * tmp2 + dAbulk_dVg);
  dT1_dVb = dAbulk_dVb * WVCoxRds + T9 * tmp3;
  const double Vasat = T0 / T1;
  const double dVasat_dVg = (dT0_dVg - Vasat * dT1_dVg) / T1;
  const double dVasat_dVb = (dT0_dVb - Vasat * dT1_dVb) / T1;
  const double dVasat_dVd = dT0_dVd / T1;
  if (Vdseff > Vds) Vdseff = Vds;
  const double diffVds = Vds - Vdseff;

  // Channel-length modulation, DIBL, pvag, SCBE (:5701-5860).
  double VACLM, dVACLM_dVg, dVACLM_dVd, dVACLM_dVb;
  if ((P(pclm) > 0.0) && (diffVds > 1.0e-10)) {
    T0 = 1.0 / (P(pclm) * Abulk * P(litl));
    dT0_dVb = -T0 / Abulk * dAbulk_dVb;
    dT0_dVg = -T0 / Abulk * dAbulk_dVg;
    T2 = Vgsteff / EsatL;
    T1 = Leff * (Abulk + T2);
    dT1_dVg = Leff * ((1.0 - T2 * dEsatL_dVg) / EsatL + dAbulk_dVg);
    dT1_dVb = Leff * (dAbulk_dVb - T2 * dEsatL_dVb / EsatL);
    dT1_dVd = -T2 * dEsatL_dVd / Esat;
    T9 = T0 * T1;
    VACLM = T9 * diffVds;
    dVACLM_dVg = T0 * dT1_dVg * diffVds - T9 * dVdseff_dVg + T1 * diffVds * dT0_dVg;
    dVACLM_dVb = (dT0_dVb * T1 + T0 * dT1_dVb) * diffVds - T9 * dVdseff_dVb;
    dVACLM_dVd = T0 * dT1_dVd * diffVds + T9 * (1.0 - dVdseff_dVd);
  } else {
    VACLM = CONSTMAX_EXP;
    dVACLM_dVd = dVACLM_dVg = dVACLM_dVb = 0.0;
  }
  double VADIBL, dVADIBL_dVg, dVADIBL_dVd, dVADIBL_dVb;
  if (P(thetaRout) > 0.0) {
    T8 = Abulk * Vdsat;
    T0 = Vgst2Vtm * T8;
    dT0_dVg = Vgst2Vtm * Abulk * dVdsat_dVg + T8 + Vgst2Vtm * Vdsat * dAbulk_dVg;
    dT0_dVb = Vgst2Vtm * (dAbulk_dVb * Vdsat + Abulk * dVdsat_dVb);
    dT0_dVd = Vgst2Vtm * Abulk * dVdsat_dVd;
    T1 = Vgst2Vtm + T8;
    dT1_dVg = 1.0 + Abulk * dVdsat_dVg + Vdsat * dAbulk_dVg;
    dT1_dVb = Abulk * dVdsat_dVb + dAbulk_dVb * Vdsat;
    dT1_dVd = Abulk * dVdsat_dVd;
    T9 = T1 * T1;
    T2 = P(thetaRout);
    VADIBL = (Vgst2Vtm - T0 / T1) / T2;
    dVADIBL_dVg = (1.0 - dT0_dVg / T1 + T0 * dT1_dVg / T9) / T2;
    dVADIBL_dVb = (-dT0_dVb / T1 + T0 * dT1_dVb / T9) / T2;
    dVADIBL_dVd = (-dT0_dVd / T1 + T0 * dT1_dVd / T9) / T2;
    T7 = P(pdiblb) * Vbseff;
    if (T7 >= -0.9) {
      T3 = 1.0 / (1.0 + T7);
      VADIBL *= T3;
      dVADIBL_dVg *= T3;
      dVADIBL_dVb = (dVADIBL_dVb - VADIBL * P(pdiblb)) * T3;
      dVADIBL_dVd *= T3;
    } else {
      T4 = 1.0 / (0.8 + T7);
      T3 = (17.0 + 20.0 * T7) * T4;
      dVADIBL_dVg *= T3;
      dVADIBL_dVb = dVADIBL_dVb * T3 - VADIBL * P(pdiblb) * T4 * T4;
      dVADIBL_dVd *= T3;
      VADIBL *= T3;
    }
  } else {
    VADIBL = CONSTMAX_EXP;
    dVADIBL_dVd = dVADIBL_dVg = dVADIBL_dVb = 0.0;
  }
  T8 = P(pvag) / EsatL;
  T9 = T8 * Vgsteff;
  if (T9 > -0.9) {
    T0 = 1.0 + T9;
    dT0_dVg = T8 * (1.0 - Vgsteff * dEsatL_dVg / EsatL);
    dT0_dVb = -T9 * dEsatL_dVb / EsatL;
    dT0_dVd = -T9 * dEsatL_dVd / EsatL;
  } else {
    T1 = 1.0 / (17.0 + 20.0 * T9);
    T0 = (0.8 + T9) * T1;
    T1 *= T1;
    dT0_dVg = T8 * (1.0 - Vgsteff * dEsatL_dVg / EsatL) * T1;
    T9 *= T1 / EsatL;
    dT0_dVb = -T9 * dEsatL_dVb;
    dT0_dVd = -T9 * dEsatL_dVd;
  }
  tmp1 = VACLM * VACLM;
  tmp2 = VADIBL * VADIBL;
  tmp3 = VACLM + VADIBL;
  T1 = VACLM * VADIBL / tmp3;
  tmp3 *= tmp3;
  dT1_dVg = (tmp1 * dVADIBL_dVg + tmp2 * dVACLM_dVg) / tmp3;
  dT1_dVd = (tmp1 * dVADIBL_dVd + tmp2 * dVACLM_dVd) / tmp3;
  dT1_dVb = (tmp1 * dVADIBL_dVb + tmp2 * dVACLM_dVb) / tmp3;
  const double Va = Vasat + T0 * T1;
  const double dVa_dVg = dVasat_dVg + T1 * dT0_dVg + T0 * dT1_dVg;
  const double dVa_dVd = dVasat_dVd + T1 * dT0_dVd + T0 * dT1_dVd;
  const double dVa_dVb = dVasat_dVb + T1 * dT0_dVb + T0 * dT1_dVb;
  double VASCBE, dVASCBE_dVg, dVASCBE_dVd, dVASCBE_dVb;
  if (P(pscbe2) > 0.0) {
    if (diffVds > P(pscbe1) * P(litl) / CONSTEXP_THRESHOLD) {
      T0 = P(pscbe1) * P(litl) / diffVds;
      VASCBE = Leff * exp(T0) / P(pscbe2);
      T1 = T0 * VASCBE / diffVds;
      dVASCBE_dVg = T1 * dVdseff_dVg;
      dVASCBE_dVd = -T1 * (1.0 - dVdseff_dVd);
      dVASCBE_dVb = T1 * dVdseff_dVb;
    } else {
      VASCBE = CONSTMAX_EXP * Leff / P(pscbe2);
      dVASCBE_dVg = dVASCBE_dVd = dVASCBE_dVb = 0.0;
    }
  } else {
    VASCBE = CONSTMAX_EXP;
    dVASCBE_dVg = dVASCBE_dVd = dVASCBE_dVb = 0.0;
  }

  // Drain current (:5861-5935).
  const double CoxWovL = cox * Weff / Leff;
  const double beta = ueff * CoxWovL;
  const double dbeta_dVg = CoxWovL * dueff_dVg + beta * dWeff_dVg / Weff;
  const double dbeta_dVd = CoxWovL * dueff_dVd;
  const double dbeta_dVb = CoxWovL * dueff_dVb + beta * dWeff_dVb / Weff;
  T0 = 1.0 - 0.5 * Abulk * Vdseff / Vgst2Vtm;
  dT0_dVg = -0.5 * (Abulk * dVdseff_dVg - Abulk * Vdseff / Vgst2Vtm + Vdseff * dAbulk_dVg) / Vgst2Vtm;
  dT0_dVd = -0.5 * Abulk * dVdseff_dVd / Vgst2Vtm;
  dT0_dVb = -0.5 * (Abulk * dVdseff_dVb + dAbulk_dVb * Vdseff) / Vgst2Vtm;
  const double fgche1 = Vgsteff * T0;
  const double dfgche1_dVg = Vgsteff * dT0_dVg + T0;
  const double dfgche1_dVd = Vgsteff * dT0_dVd;
  const double dfgche1_dVb = Vgsteff * dT0_dVb;
  T9 = Vdseff / EsatL;
  const double fgche2 = 1.0 + T9;
  const double dfgche2_dVg = (dVdseff_dVg - T9 * dEsatL_dVg) / EsatL;
  const double dfgche2_dVd = (dVdseff_dVd - T9 * dEsatL_dVd) / EsatL;
  const double dfgche2_dVb = (dVdseff_dVb - T9 * dEsatL_dVb) / EsatL;
  const double gche = beta * fgche1 / fgche2;
  const double dgche_dVg = (beta * dfgche1_dVg + fgche1 * dbeta_dVg - gche * dfgche2_dVg) / fgche2;
  const double dgche_dVd = (beta * dfgche1_dVd + fgche1 * dbeta_dVd - gche * dfgche2_dVd) / fgche2;
  const double dgche_dVb = (beta * dfgche1_dVb + fgche1 * dbeta_dVb - gche * dfgche2_dVb) / fgche2;
  T0 = 1.0 + gche * Rds;
  T9 = Vdseff / T0;
  const double Idl = gche * T9;
  const double dIdl_dVg = (gche * dVdseff_dVg + T9 * dgche_dVg) / T0 - Idl * gche / T0 * dRds_dVg;
  const double dIdl_dVd = (gche * dVdseff_dVd + T9 * dgche_dVd) / T0;
  const double dIdl_dVb = (gche * dVdseff_dVb + T9 * dgche_dVb - Idl * dRds_dVb * gche) / T0;
  T9 = diffVds / Va;
  T0 = 1.0 + T9;
  const double Idsa = Idl * T0;
  const double dIdsa_dVg = T0 * dIdl_dVg - Idl * (dVdseff_dVg + T9 * dVa_dVg) / Va;
  const double dIdsa_dVd = T0 * dIdl_dVd + Idl * (1.0 - dVdseff_dVd - T9 * dVa_dVd) / Va;
  const double dIdsa_dVb = T0 * dIdl_dVb - Idl * (dVdseff_dVb + T9 * dVa_dVb) / Va;
  T9 = diffVds / VASCBE;
  T0 = 1.0 + T9;
  const double Ids = Idsa * T0;
  double Gm = T0 * dIdsa_dVg - Idsa * (dVdseff_dVg + T9 * dVASCBE_dVg) / VASCBE;
  double Gds = T0 * dIdsa_dVd + Idsa * (1.0 - dVdseff_dVd - T9 * dVASCBE_dVd) / VASCBE;
  double Gmb = T0 * dIdsa_dVb - Idsa * (dVdseff_dVb + T9 * dVASCBE_dVb) / VASCBE;
  Gds += Gm * dVgsteff_dVd;
  Gmb += Gm * dVgsteff_dVb;
  Gm *= dVgsteff_dVg;
  Gmb *= dVbseff_dVb;

  // Substrate current (:5936-5975).
  double Isub, Gbd, Gbb, Gbg;
  tmp = P(alpha0) + P(alpha1) * Leff;
  if ((tmp <= 0.0) || (P(beta0) <= 0.0)) {
    Isub = Gbd = Gbb = Gbg = 0.0;
  } else {
    T2 = tmp / Leff;
    if (diffVds > P(beta0) / CONSTEXP_THRESHOLD) {
      T0 = -P(beta0) / diffVds;
      T1 = T2 * diffVds * exp(T0);
      T3 = T1 / diffVds * (T0 - 1.0);
      dT1_dVg = T3 * dVdseff_dVg;
      dT1_dVd = T3 * (dVdseff_dVd - 1.0);
      dT1_dVb = T3 * dVdseff_dVb;
    } else {
      T3 = T2 * CONSTMIN_EXP;
      T1 = T3 * diffVds;
      dT1_dVg = -T3 * dVdseff_dVg;
      dT1_dVd = T3 * (1.0 - dVdseff_dVd);
      dT1_dVb = -T3 * dVdseff_dVb;
    }
    Isub = T1 * Idsa;
    Gbg = T1 * dIdsa_dVg + Idsa * dT1_dVg;
    Gbd = T1 * dIdsa_dVd + Idsa * dT1_dVd;
    Gbb = T1 * dIdsa_dVb + Idsa * dT1_dVb;
    Gbd += Gbg * dVgsteff_dVd;
    Gbb += Gbg * dVgsteff_dVb;
    Gbg *= dVgsteff_dVg;
    Gbb *= dVbseff_dVb;
  }
  const double cdrain = Ids, gds = Gds, gm = Gm, gmbs = Gmb, gbbs = Gbb, gbgs = Gbg, gbds = Gbd, csub = Isub;

  // Intrinsic charges (:5964-6930): capMod 0 (shared simple model), 1, 2, 3 (charge thickness).
  double qgate = 0.0, qdrn = 0.0, qsrc = 0.0, qbulk = 0.0;
  double cggb = 0.0, cgsb = 0.0, cgdb = 0.0, cdgb = 0.0, cdsb = 0.0, cddb = 0.0, cbgb = 0.0, cbsb = 0.0,
         cbdb = 0.0;
  const double xpart = P(xpart);
  if (((xpart < 0) || (!ChargeComputationNeeded))) {
    // no charges
  } else if ((int)P(capMod) == 0) {
    // capMod = 0 (:5975-6240), the simple charge model BSIM4 shares.
    xdc::CvCharges cv;
    xdc::cv_simple(Vbseff, Vbs, phi, Phis, dPhis_dVb, sqrtPhis, dsqrtPhis_dVb, P(vfbcv), P(k1ox), Vgs_eff,
                   dVgs_eff_dVg, cox * P(weffCV) * P(leffCV), Abulk0, dAbulk0_dVb, P(abulkCVfactor), Vds, xpart,
                   true, cv);
    qgate = cv.qgate, qbulk = cv.qbulk, qdrn = cv.qdrn;
    cggb = cv.cggb, cgsb = cv.cgsb, cgdb = cv.cgdb, cdgb = cv.cdgb, cdsb = cv.cdsb, cddb = cv.cddb;
    cbgb = cv.cbgb, cbsb = cv.cbsb, cbdb = cv.cbdb;
  } else {
    double VbseffCV, dVbseffCV_dVb;
    if (Vbseff < 0.0) {
      VbseffCV = Vbseff;
      dVbseffCV_dVb = 1.0;
    } else {
      VbseffCV = phi - Phis;
      dVbseffCV_dVb = -dPhis_dVb;
    }
    const double CoxWL = cox * P(weffCV) * P(leffCV);
    const double noff = n * P(noff);
    const double dnoff_dVd = P(noff) * dn_dVd;
    const double dnoff_dVb = P(noff) * dn_dVb;
    T0 = Vtm * noff;
    const double voffcv = P(voffcv);
    VgstNVt = (Vgst - voffcv) / T0;
    if (VgstNVt > CONSTEXP_THRESHOLD) {
      Vgsteff = Vgst - voffcv;
      dVgsteff_dVg = dVgs_eff_dVg;
      dVgsteff_dVd = -dVth_dVd;
      dVgsteff_dVb = -dVth_dVb;
    } else if (VgstNVt < -CONSTEXP_THRESHOLD) {
      Vgsteff = T0 * log(1.0 + CONSTMIN_EXP);
      dVgsteff_dVg = 0.0;
      dVgsteff_dVd = Vgsteff / noff;
      dVgsteff_dVb = dVgsteff_dVd * dnoff_dVb;
      dVgsteff_dVd *= dnoff_dVd;
    } else {
      const double ExpVgst = exp(VgstNVt);
      Vgsteff = T0 * log(1.0 + ExpVgst);
      dVgsteff_dVg = ExpVgst / (1.0 + ExpVgst);
      dVgsteff_dVd = -dVgsteff_dVg * (dVth_dVd + (Vgst - voffcv) / noff * dnoff_dVd) + Vgsteff / noff * dnoff_dVd;
      dVgsteff_dVb = -dVgsteff_dVg * (dVth_dVb + (Vgst - voffcv) / noff * dnoff_dVb) + Vgsteff / noff * dnoff_dVb;
      dVgsteff_dVg *= dVgs_eff_dVg;
    }
    double Cgg, Cgd, Cgb, Cbg, Cbd, Cbb, Csg, Csd, Csb;
    double Cgg1, Cgd1, Cgb1, Cbg1, Cbd1, Cbb1;
    double Qac0, Qsub0, dQac0_dVg, dQac0_dVb, dQsub0_dVg, dQsub0_dVd, dQsub0_dVb;
    double Vfbeff, dVfbeff_dVg, dVfbeff_dVb, V3, V4, AbulkCV, dAbulkCV_dVb, VdsatCV, VdseffCV, dVdseffCV_dVg,
        dVdseffCV_dVd, dVdseffCV_dVb;
    const double vfbzb = P(vfbzb);
    const double k1ox = P(k1ox);
    if ((int)P(capMod) == 1) {
      // capMod = 1 (:6330-6490): depletion charge from the zero-bias flat band, inversion charge
      // of the saturation or the linear region.
      const double Arg1 = Vgs_eff - VbseffCV - vfbzb - Vgsteff;
      if (Arg1 <= 0.0) {
        qgate = CoxWL * Arg1;
        Cgg = CoxWL * (dVgs_eff_dVg - dVgsteff_dVg);
        Cgd = -CoxWL * dVgsteff_dVd;
        Cgb = -CoxWL * (dVbseffCV_dVb + dVgsteff_dVb);
      } else {
        T0 = 0.5 * k1ox;
        T1 = sqrt(T0 * T0 + Arg1);
        T2 = CoxWL * T0 / T1;
        qgate = CoxWL * k1ox * (T1 - T0);
        Cgg = T2 * (dVgs_eff_dVg - dVgsteff_dVg);
        Cgd = -T2 * dVgsteff_dVd;
        Cgb = -T2 * (dVbseffCV_dVb + dVgsteff_dVb);
      }
      qbulk = -qgate;
      Cbg = -Cgg;
      Cbd = -Cgd;
      Cbb = -Cgb;
      const double One_Third_CoxWL = CoxWL / 3.0;
      const double Two_Third_CoxWL = 2.0 * One_Third_CoxWL;
      AbulkCV = Abulk0 * P(abulkCVfactor);
      dAbulkCV_dVb = P(abulkCVfactor) * dAbulk0_dVb;
      VdsatCV = Vgsteff / AbulkCV;
      if (VdsatCV < Vds) {
        const double dVdsatCV_dVg = 1.0 / AbulkCV;
        const double dVdsatCV_dVb = -VdsatCV * dAbulkCV_dVb / AbulkCV;
        T0 = Vgsteff - VdsatCV / 3.0;
        dT0_dVg = 1.0 - dVdsatCV_dVg / 3.0;
        dT0_dVb = -dVdsatCV_dVb / 3.0;
        qgate += CoxWL * T0;
        Cgg1 = CoxWL * dT0_dVg;
        Cgb1 = CoxWL * dT0_dVb + Cgg1 * dVgsteff_dVb;
        Cgd1 = Cgg1 * dVgsteff_dVd;
        Cgg1 *= dVgsteff_dVg;
        Cgg += Cgg1;
        Cgb += Cgb1;
        Cgd += Cgd1;
        T0 = VdsatCV - Vgsteff;
        dT0_dVg = dVdsatCV_dVg - 1.0;
        dT0_dVb = dVdsatCV_dVb;
        qbulk += One_Third_CoxWL * T0;
        Cbg1 = One_Third_CoxWL * dT0_dVg;
        Cbb1 = One_Third_CoxWL * dT0_dVb + Cbg1 * dVgsteff_dVb;
        Cbd1 = Cbg1 * dVgsteff_dVd;
        Cbg1 *= dVgsteff_dVg;
        Cbg += Cbg1;
        Cbb += Cbb1;
        Cbd += Cbd1;
        if (xpart > 0.5)
          T0 = -Two_Third_CoxWL;
        else if (xpart < 0.5)
          T0 = -0.4 * CoxWL;
        else
          T0 = -One_Third_CoxWL;
        qsrc = T0 * Vgsteff;
        Csg = T0 * dVgsteff_dVg;
        Csb = T0 * dVgsteff_dVb;
        Csd = T0 * dVgsteff_dVd;
      } else {
        T0 = AbulkCV * Vds;
        T1 = 12.0 * (Vgsteff - 0.5 * T0 + 1.e-20);
        T2 = Vds / T1;
        T3 = T0 * T2;
        dT3_dVg = -12.0 * T2 * T2 * AbulkCV;
        dT3_dVd = 6.0 * T0 * (4.0 * Vgsteff - T0) / T1 / T1 - 0.5;
        dT3_dVb = 12.0 * T2 * T2 * dAbulkCV_dVb * Vgsteff;
        qgate += CoxWL * (Vgsteff - 0.5 * Vds + T3);
        Cgg1 = CoxWL * (1.0 + dT3_dVg);
        Cgb1 = CoxWL * dT3_dVb + Cgg1 * dVgsteff_dVb;
        Cgd1 = CoxWL * dT3_dVd + Cgg1 * dVgsteff_dVd;
        Cgg1 *= dVgsteff_dVg;
        Cgg += Cgg1;
        Cgb += Cgb1;
        Cgd += Cgd1;
        qbulk += CoxWL * (1.0 - AbulkCV) * (0.5 * Vds - T3);
        Cbg1 = -CoxWL * ((1.0 - AbulkCV) * dT3_dVg);
        Cbb1 = -CoxWL * ((1.0 - AbulkCV) * dT3_dVb + (0.5 * Vds - T3) * dAbulkCV_dVb) + Cbg1 * dVgsteff_dVb;
        Cbd1 = -CoxWL * (1.0 - AbulkCV) * dT3_dVd + Cbg1 * dVgsteff_dVd;
        Cbg1 *= dVgsteff_dVg;
        Cbg += Cbg1;
        Cbb += Cbb1;
        Cbd += Cbd1;
        if (xpart > 0.5) {  // 0/100
          T1 = T1 + T1;
          qsrc = -CoxWL * (0.5 * Vgsteff + 0.25 * T0 - T0 * T0 / T1);
          Csg = -CoxWL * (0.5 + 24.0 * T0 * Vds / T1 / T1 * AbulkCV);
          Csb = -CoxWL * (0.25 * Vds * dAbulkCV_dVb - 12.0 * T0 * Vds / T1 / T1 * (4.0 * Vgsteff - T0) * dAbulkCV_dVb) +
                Csg * dVgsteff_dVb;
          Csd = -CoxWL * (0.25 * AbulkCV - 12.0 * AbulkCV * T0 / T1 / T1 * (4.0 * Vgsteff - T0)) + Csg * dVgsteff_dVd;
          Csg *= dVgsteff_dVg;
        } else if (xpart < 0.5) {  // 40/60
          T1 = T1 / 12.0;
          T2 = 0.5 * CoxWL / (T1 * T1);
          T3 = Vgsteff * (2.0 * T0 * T0 / 3.0 + Vgsteff * (Vgsteff - 4.0 * T0 / 3.0)) - 2.0 * T0 * T0 * T0 / 15.0;
          qsrc = -T2 * T3;
          T4 = 4.0 / 3.0 * Vgsteff * (Vgsteff - T0) + 0.4 * T0 * T0;
          Csg = -2.0 * qsrc / T1 - T2 * (Vgsteff * (3.0 * Vgsteff - 8.0 * T0 / 3.0) + 2.0 * T0 * T0 / 3.0);
          Csb = (qsrc / T1 * Vds + T2 * T4 * Vds) * dAbulkCV_dVb + Csg * dVgsteff_dVb;
          Csd = (qsrc / T1 + T2 * T4) * AbulkCV + Csg * dVgsteff_dVd;
          Csg *= dVgsteff_dVg;
        } else {  // 50/50
          qsrc = -0.5 * (qgate + qbulk);
          Csg = -0.5 * (Cgg1 + Cbg1);
          Csb = -0.5 * (Cgb1 + Cbb1);
          Csd = -0.5 * (Cgd1 + Cbd1);
        }
      }
      qdrn = -(qgate + qbulk + qsrc);
    } else if ((int)P(capMod) == 2) {
      const double Vfb = vfbzb;
      V3 = Vfb - Vgs_eff + VbseffCV - CONSTDELTA_3;
      if (Vfb <= 0.0) {
        T0 = sqrt(V3 * V3 - 4.0 * CONSTDELTA_3 * Vfb);
        T2 = -CONSTDELTA_3 / T0;
      } else {
        T0 = sqrt(V3 * V3 + 4.0 * CONSTDELTA_3 * Vfb);
        T2 = CONSTDELTA_3 / T0;
      }
      T1 = 0.5 * (1.0 + V3 / T0);
      Vfbeff = Vfb - 0.5 * (V3 + T0);
      dVfbeff_dVg = T1 * dVgs_eff_dVg;
      dVfbeff_dVb = -T1 * dVbseffCV_dVb;
      Qac0 = CoxWL * (Vfbeff - Vfb);
      dQac0_dVg = CoxWL * dVfbeff_dVg;
      dQac0_dVb = CoxWL * dVfbeff_dVb;
      T0 = 0.5 * k1ox;
      T3 = Vgs_eff - Vfbeff - VbseffCV - Vgsteff;
      if (k1ox == 0.0) {
        T1 = 0.0;
        T2 = 0.0;
      } else if (T3 < 0.0) {
        T1 = T0 + T3 / k1ox;
        T2 = CoxWL;
      } else {
        T1 = sqrt(T0 * T0 + T3);
        T2 = CoxWL * T0 / T1;
      }
      Qsub0 = CoxWL * k1ox * (T1 - T0);
      dQsub0_dVg = T2 * (dVgs_eff_dVg - dVfbeff_dVg - dVgsteff_dVg);
      dQsub0_dVd = -T2 * dVgsteff_dVd;
      dQsub0_dVb = -T2 * (dVfbeff_dVb + dVbseffCV_dVb + dVgsteff_dVb);
      AbulkCV = Abulk0 * P(abulkCVfactor);
      dAbulkCV_dVb = P(abulkCVfactor) * dAbulk0_dVb;
      VdsatCV = Vgsteff / AbulkCV;
      V4 = VdsatCV - Vds - CONSTDELTA_4;
      T0 = sqrt(V4 * V4 + 4.0 * CONSTDELTA_4 * VdsatCV);
      VdseffCV = VdsatCV - 0.5 * (V4 + T0);
      T1 = 0.5 * (1.0 + V4 / T0);
      T2 = CONSTDELTA_4 / T0;
      T3 = (1.0 - T1 - T2) / AbulkCV;
      dVdseffCV_dVg = T3;
      dVdseffCV_dVd = T1;
      dVdseffCV_dVb = -T3 * VdsatCV * dAbulkCV_dVb;
      if (Vds == 0.0) {
        VdseffCV = 0.0;
        dVdseffCV_dVg = 0.0;
        dVdseffCV_dVb = 0.0;
      }
      T0 = AbulkCV * VdseffCV;
      T1 = 12.0 * (Vgsteff - 0.5 * T0 + 1e-20);
      T2 = VdseffCV / T1;
      T3 = T0 * T2;
      T4 = (1.0 - 12.0 * T2 * T2 * AbulkCV);
      T5 = (6.0 * T0 * (4.0 * Vgsteff - T0) / (T1 * T1) - 0.5);
      T6 = 12.0 * T2 * T2 * Vgsteff;
      qgate = CoxWL * (Vgsteff - 0.5 * VdseffCV + T3);
      Cgg1 = CoxWL * (T4 + T5 * dVdseffCV_dVg);
      Cgd1 = CoxWL * T5 * dVdseffCV_dVd + Cgg1 * dVgsteff_dVd;
      Cgb1 = CoxWL * (T5 * dVdseffCV_dVb + T6 * dAbulkCV_dVb) + Cgg1 * dVgsteff_dVb;
      Cgg1 *= dVgsteff_dVg;
      T7 = 1.0 - AbulkCV;
      qbulk = CoxWL * T7 * (0.5 * VdseffCV - T3);
      T4 = -T7 * (T4 - 1.0);
      T5 = -T7 * T5;
      T6 = -(T7 * T6 + (0.5 * VdseffCV - T3));
      Cbg1 = CoxWL * (T4 + T5 * dVdseffCV_dVg);
      Cbd1 = CoxWL * T5 * dVdseffCV_dVd + Cbg1 * dVgsteff_dVd;
      Cbb1 = CoxWL * (T5 * dVdseffCV_dVb + T6 * dAbulkCV_dVb) + Cbg1 * dVgsteff_dVb;
      Cbg1 *= dVgsteff_dVg;
      if (xpart > 0.5) {
        T1 = T1 + T1;
        qsrc = -CoxWL * (0.5 * Vgsteff + 0.25 * T0 - T0 * T0 / T1);
        T7 = (4.0 * Vgsteff - T0) / (T1 * T1);
        T4 = -(0.5 + 24.0 * T0 * T0 / (T1 * T1));
        T5 = -(0.25 * AbulkCV - 12.0 * AbulkCV * T0 * T7);
        T6 = -(0.25 * VdseffCV - 12.0 * T0 * VdseffCV * T7);
        Csg = CoxWL * (T4 + T5 * dVdseffCV_dVg);
        Csd = CoxWL * T5 * dVdseffCV_dVd + Csg * dVgsteff_dVd;
        Csb = CoxWL * (T5 * dVdseffCV_dVb + T6 * dAbulkCV_dVb) + Csg * dVgsteff_dVb;
        Csg *= dVgsteff_dVg;
      } else if (xpart < 0.5) {
        T1 = T1 / 12.0;
        T2 = 0.5 * CoxWL / (T1 * T1);
        T3 = Vgsteff * (2.0 * T0 * T0 / 3.0 + Vgsteff * (Vgsteff - 4.0 * T0 / 3.0)) - 2.0 * T0 * T0 * T0 / 15.0;
        qsrc = -T2 * T3;
        T7 = 4.0 / 3.0 * Vgsteff * (Vgsteff - T0) + 0.4 * T0 * T0;
        T4 = -2.0 * qsrc / T1 - T2 * (Vgsteff * (3.0 * Vgsteff - 8.0 * T0 / 3.0) + 2.0 * T0 * T0 / 3.0);
        T5 = (qsrc / T1 + T2 * T7) * AbulkCV;
        T6 = (qsrc / T1 * VdseffCV + T2 * T7 * VdseffCV);
        Csg = (T4 + T5 * dVdseffCV_dVg);
        Csd = T5 * dVdseffCV_dVd + Csg * dVgsteff_dVd;
        Csb = (T5 * dVdseffCV_dVb + T6 * dAbulkCV_dVb) + Csg * dVgsteff_dVb;
        Csg *= dVgsteff_dVg;
      } else {
        qsrc = -0.5 * (qgate + qbulk);
        Csg = -0.5 * (Cgg1 + Cbg1);
        Csb = -0.5 * (Cgb1 + Cbb1);
        Csd = -0.5 * (Cgd1 + Cbd1);
      }
      qgate += Qac0 + Qsub0;
      qbulk -= (Qac0 + Qsub0);
      qdrn = -(qgate + qbulk + qsrc);
      Cgg = dQac0_dVg + dQsub0_dVg + Cgg1;
      Cgd = dQsub0_dVd + Cgd1;
      Cgb = dQac0_dVb + dQsub0_dVb + Cgb1;
      Cbg = Cbg1 - dQac0_dVg - dQsub0_dVg;
      Cbd = Cbd1 - dQsub0_dVd;
      Cbb = Cbb1 - dQac0_dVb - dQsub0_dVb;
    } else {
      // capMod 3: charge-thickness model.
      V3 = vfbzb - Vgs_eff + VbseffCV - CONSTDELTA_3;
      if (vfbzb <= 0.0) {
        T0 = sqrt(V3 * V3 - 4.0 * CONSTDELTA_3 * vfbzb);
        T2 = -CONSTDELTA_3 / T0;
      } else {
        T0 = sqrt(V3 * V3 + 4.0 * CONSTDELTA_3 * vfbzb);
        T2 = CONSTDELTA_3 / T0;
      }
      T1 = 0.5 * (1.0 + V3 / T0);
      Vfbeff = vfbzb - 0.5 * (V3 + T0);
      dVfbeff_dVg = T1 * dVgs_eff_dVg;
      dVfbeff_dVb = -T1 * dVbseffCV_dVb;
      const double Cox = cox;
      double Tox = 1.0e8 * tox;
      T0 = (Vgs_eff - VbseffCV - vfbzb) / Tox;
      dT0_dVg = dVgs_eff_dVg / Tox;
      dT0_dVb = -dVbseffCV_dVb / Tox;
      tmp = T0 * P(acde);
      double Tcen, dTcen_dVg, dTcen_dVd, dTcen_dVb;
      const double ldeb = P(ldeb);
      if ((-CONSTEXP_THRESHOLD < tmp) && (tmp < CONSTEXP_THRESHOLD)) {
        Tcen = ldeb * exp(tmp);
        dTcen_dVg = P(acde) * Tcen;
        dTcen_dVb = dTcen_dVg * dT0_dVb;
        dTcen_dVg *= dT0_dVg;
      } else if (tmp <= -CONSTEXP_THRESHOLD) {
        Tcen = ldeb * CONSTMIN_EXP;
        dTcen_dVg = dTcen_dVb = 0.0;
      } else {
        Tcen = ldeb * CONSTMAX_EXP;
        dTcen_dVg = dTcen_dVb = 0.0;
      }
      const double LINK = 1.0e-3 * tox;
      V3 = ldeb - Tcen - LINK;
      V4 = sqrt(V3 * V3 + 4.0 * LINK * ldeb);
      Tcen = ldeb - 0.5 * (V3 + V4);
      T1 = 0.5 * (1.0 + V3 / V4);
      dTcen_dVg *= T1;
      dTcen_dVb *= T1;
      double Ccen = CONSTEPSSI / Tcen;
      T2 = Cox / (Cox + Ccen);
      double Coxeff = T2 * Ccen;
      T3 = -Ccen / Tcen;
      double dCoxeff_dVg = T2 * T2 * T3;
      double dCoxeff_dVb = dCoxeff_dVg * dTcen_dVb;
      dCoxeff_dVg *= dTcen_dVg;
      double CoxWLcen = CoxWL * Coxeff / Cox;
      Qac0 = CoxWLcen * (Vfbeff - vfbzb);
      double QovCox = Qac0 / Coxeff;
      dQac0_dVg = CoxWLcen * dVfbeff_dVg + QovCox * dCoxeff_dVg;
      dQac0_dVb = CoxWLcen * dVfbeff_dVb + QovCox * dCoxeff_dVb;
      T0 = 0.5 * k1ox;
      T3 = Vgs_eff - Vfbeff - VbseffCV - Vgsteff;
      if (k1ox == 0.0) {
        T1 = 0.0;
        T2 = 0.0;
      } else if (T3 < 0.0) {
        T1 = T0 + T3 / k1ox;
        T2 = CoxWLcen;
      } else {
        T1 = sqrt(T0 * T0 + T3);
        T2 = CoxWLcen * T0 / T1;
      }
      Qsub0 = CoxWLcen * k1ox * (T1 - T0);
      QovCox = Qsub0 / Coxeff;
      dQsub0_dVg = T2 * (dVgs_eff_dVg - dVfbeff_dVg - dVgsteff_dVg) + QovCox * dCoxeff_dVg;
      dQsub0_dVd = -T2 * dVgsteff_dVd;
      dQsub0_dVb = -T2 * (dVfbeff_dVb + dVbseffCV_dVb + dVgsteff_dVb) + QovCox * dCoxeff_dVb;
      double DenomiQ;
      if (k1ox <= 0.0) {
        DenomiQ = 0.25 * P(moin) * Vtm;
        T0 = 0.5 * sqrtPhi;
      } else {
        DenomiQ = P(moin) * Vtm * k1ox * k1ox;
        T0 = k1ox * sqrtPhi;
      }
      T1 = 2.0 * T0 + Vgsteff;
      const double DeltaPhi = Vtm * log(1.0 + T1 * Vgsteff / DenomiQ);
      const double dDeltaPhi_dVg = 2.0 * Vtm * (T1 - T0) / (DenomiQ + T1 * Vgsteff);
      T3 = 4.0 * (Vth - vfbzb - phi);
      Tox += Tox;
      if (T3 >= 0.0) {
        T0 = (Vgsteff + T3) / Tox;
        dT0_dVd = (dVgsteff_dVd + 4.0 * dVth_dVd) / Tox;
        dT0_dVb = (dVgsteff_dVb + 4.0 * dVth_dVb) / Tox;
      } else {
        T0 = (Vgsteff + 1.0e-20) / Tox;
        dT0_dVd = dVgsteff_dVd / Tox;
        dT0_dVb = dVgsteff_dVb / Tox;
      }
      tmp = exp(0.7 * log(T0));
      T1 = 1.0 + tmp;
      T2 = 0.7 * tmp / (T0 * Tox);
      Tcen = 1.9e-9 / T1;
      dTcen_dVg = -1.9e-9 * T2 / T1 / T1;
      dTcen_dVd = Tox * dTcen_dVg;
      dTcen_dVb = dTcen_dVd * dT0_dVb;
      dTcen_dVd *= dT0_dVd;
      dTcen_dVg *= dVgsteff_dVg;
      Ccen = CONSTEPSSI / Tcen;
      T0 = Cox / (Cox + Ccen);
      Coxeff = T0 * Ccen;
      T1 = -Ccen / Tcen;
      dCoxeff_dVg = T0 * T0 * T1;
      const double dCoxeff_dVd = dCoxeff_dVg * dTcen_dVd;
      dCoxeff_dVb = dCoxeff_dVg * dTcen_dVb;
      dCoxeff_dVg *= dTcen_dVg;
      CoxWLcen = CoxWL * Coxeff / Cox;
      AbulkCV = Abulk0 * P(abulkCVfactor);
      dAbulkCV_dVb = P(abulkCVfactor) * dAbulk0_dVb;
      VdsatCV = (Vgsteff - DeltaPhi) / AbulkCV;
      V4 = VdsatCV - Vds - CONSTDELTA_4;
      T0 = sqrt(V4 * V4 + 4.0 * CONSTDELTA_4 * VdsatCV);
      VdseffCV = VdsatCV - 0.5 * (V4 + T0);
      T1 = 0.5 * (1.0 + V4 / T0);
      T2 = CONSTDELTA_4 / T0;
      T3 = (1.0 - T1 - T2) / AbulkCV;
      T4 = T3 * (1.0 - dDeltaPhi_dVg);
      dVdseffCV_dVg = T4;
      dVdseffCV_dVd = T1;
      dVdseffCV_dVb = -T3 * VdsatCV * dAbulkCV_dVb;
      if (Vds == 0.0) {
        VdseffCV = 0.0;
        dVdseffCV_dVg = 0.0;
        dVdseffCV_dVb = 0.0;
      }
      T0 = AbulkCV * VdseffCV;
      T1 = Vgsteff - DeltaPhi;
      T2 = 12.0 * (T1 - 0.5 * T0 + 1.0e-20);
      T3 = T0 / T2;
      T4 = 1.0 - 12.0 * T3 * T3;
      T5 = AbulkCV * (6.0 * T0 * (4.0 * T1 - T0) / (T2 * T2) - 0.5);
      T6 = T5 * VdseffCV / AbulkCV;
      qgate = CoxWLcen * (T1 - T0 * (0.5 - T3));
      QovCox = qgate / Coxeff;
      Cgg1 = CoxWLcen * (T4 * (1.0 - dDeltaPhi_dVg) + T5 * dVdseffCV_dVg);
      Cgd1 = CoxWLcen * T5 * dVdseffCV_dVd + Cgg1 * dVgsteff_dVd + QovCox * dCoxeff_dVd;
      Cgb1 = CoxWLcen * (T5 * dVdseffCV_dVb + T6 * dAbulkCV_dVb) + Cgg1 * dVgsteff_dVb + QovCox * dCoxeff_dVb;
      Cgg1 = Cgg1 * dVgsteff_dVg + QovCox * dCoxeff_dVg;
      T7 = 1.0 - AbulkCV;
      T8 = T2 * T2;
      T9 = 12.0 * T7 * T0 * T0 / (T8 * AbulkCV);
      T10 = T9 * (1.0 - dDeltaPhi_dVg);
      T11 = -T7 * T5 / AbulkCV;
      T12 = -(T9 * T1 / AbulkCV + VdseffCV * (0.5 - T0 / T2));
      qbulk = CoxWLcen * T7 * (0.5 * VdseffCV - T0 * VdseffCV / T2);
      QovCox = qbulk / Coxeff;
      Cbg1 = CoxWLcen * (T10 + T11 * dVdseffCV_dVg);
      Cbd1 = CoxWLcen * T11 * dVdseffCV_dVd + Cbg1 * dVgsteff_dVd + QovCox * dCoxeff_dVd;
      Cbb1 = CoxWLcen * (T11 * dVdseffCV_dVb + T12 * dAbulkCV_dVb) + Cbg1 * dVgsteff_dVb + QovCox * dCoxeff_dVb;
      Cbg1 = Cbg1 * dVgsteff_dVg + QovCox * dCoxeff_dVg;
      if (xpart > 0.5) {
        qsrc = -CoxWLcen * (T1 / 2.0 + T0 / 4.0 - 0.5 * T0 * T0 / T2);
        QovCox = qsrc / Coxeff;
        T2 += T2;
        T3 = T2 * T2;
        T7 = -(0.25 - 12.0 * T0 * (4.0 * T1 - T0) / T3);
        T4 = -(0.5 + 24.0 * T0 * T0 / T3) * (1.0 - dDeltaPhi_dVg);
        T5 = T7 * AbulkCV;
        T6 = T7 * VdseffCV;
        Csg = CoxWLcen * (T4 + T5 * dVdseffCV_dVg);
        Csd = CoxWLcen * T5 * dVdseffCV_dVd + Csg * dVgsteff_dVd + QovCox * dCoxeff_dVd;
        Csb = CoxWLcen * (T5 * dVdseffCV_dVb + T6 * dAbulkCV_dVb) + Csg * dVgsteff_dVb + QovCox * dCoxeff_dVb;
        Csg = Csg * dVgsteff_dVg + QovCox * dCoxeff_dVg;
      } else if (xpart < 0.5) {
        T2 = T2 / 12.0;
        T3 = 0.5 * CoxWLcen / (T2 * T2);
        T4 = T1 * (2.0 * T0 * T0 / 3.0 + T1 * (T1 - 4.0 * T0 / 3.0)) - 2.0 * T0 * T0 * T0 / 15.0;
        qsrc = -T3 * T4;
        QovCox = qsrc / Coxeff;
        T8 = 4.0 / 3.0 * T1 * (T1 - T0) + 0.4 * T0 * T0;
        T5 = -2.0 * qsrc / T2 - T3 * (T1 * (3.0 * T1 - 8.0 * T0 / 3.0) + 2.0 * T0 * T0 / 3.0);
        T6 = AbulkCV * (qsrc / T2 + T3 * T8);
        T7 = T6 * VdseffCV / AbulkCV;
        Csg = T5 * (1.0 - dDeltaPhi_dVg) + T6 * dVdseffCV_dVg;
        Csd = Csg * dVgsteff_dVd + T6 * dVdseffCV_dVd + QovCox * dCoxeff_dVd;
        Csb = Csg * dVgsteff_dVb + T6 * dVdseffCV_dVb + T7 * dAbulkCV_dVb + QovCox * dCoxeff_dVb;
        Csg = Csg * dVgsteff_dVg + QovCox * dCoxeff_dVg;
      } else {
        qsrc = -0.5 * qgate;
        Csg = -0.5 * Cgg1;
        Csd = -0.5 * Cgd1;
        Csb = -0.5 * Cgb1;
      }
      qgate += Qac0 + Qsub0 - qbulk;
      qbulk -= (Qac0 + Qsub0);
      qdrn = -(qgate + qbulk + qsrc);
      Cbg = Cbg1 - dQac0_dVg - dQsub0_dVg;
      Cbd = Cbd1 - dQsub0_dVd;
      Cbb = Cbb1 - dQac0_dVb - dQsub0_dVb;
      Cgg = Cgg1 - Cbg;
      Cgd = Cgd1 - Cbd;
      Cgb = Cgb1 - Cbb;
    }
    Cgb *= dVbseff_dVb;
    Cbb *= dVbseff_dVb;
    Csb *= dVbseff_dVb;
    cggb = Cgg;
    cgsb = -(Cgg + Cgd + Cgb);
    cgdb = Cgd;
    cdgb = -(Cgg + Cbg + Csg);
    cdsb = (Cgg + Cgd + Cgb + Cbg + Cbd + Cbb + Csg + Csd + Csb);
    cddb = -(Cgd + Cbd + Csd);
    cbgb = Cbg;
    cbsb = -(Cbg + Cbd + Cbb);
    cbdb = Cbd;
  }

  // Junction charges, overlap charges, capacitances (:6945-7245, 7544-7867).
  double qbs = 0.0, qbd = 0.0, capbs = 0.0, capbd = 0.0;
  double qg = 0.0, qd = 0.0, qb = 0.0;
  double CAPcggb = 0.0, CAPcgdb = 0.0, CAPcgsb = 0.0, CAPcdgb = 0.0, CAPcddb = 0.0, CAPcdsb = 0.0, CAPcsgb = 0.0,
         CAPcsdb = 0.0, CAPcssb = 0.0, CAPcbgb = 0.0, CAPcbdb = 0.0, CAPcbsb = 0.0;
  if (ChargeComputationNeeded) {
    const double czbd = P(czbd), czbs = P(czbs), czbdsw = P(czbdsw), czbdswg = P(czbdswg), czbssw = P(czbssw),
                 czbsswg = P(czbsswg);
    const double MJ = P(MJ), MJSW = P(MJSW), MJSWG = P(MJSWG);
    const double PhiBTemp = P(PhiBTemp), PhiBSWTemp = P(PhiBSWTemp), PhiBSWGTemp = P(PhiBSWGTemp);
    double arg, sarg;
    if (vbs == 0.0) {
      qbs = 0.0;
      capbs = czbs + czbssw + czbsswg;
    } else if (vbs < 0.0) {
      if (czbs > 0.0) {
        arg = 1.0 - vbs / PhiBTemp;
        if (MJ == 0.5)
          sarg = 1.0 / sqrt(arg);
        else
          sarg = exp(-MJ * log(arg));
        qbs = PhiBTemp * czbs * (1.0 - arg * sarg) / (1.0 - MJ);
        capbs = czbs * sarg;
      } else {
        qbs = 0.0;
        capbs = 0.0;
      }
      if (czbssw > 0.0) {
        arg = 1.0 - vbs / PhiBSWTemp;
        if (MJSW == 0.5)
          sarg = 1.0 / sqrt(arg);
        else
          sarg = exp(-MJSW * log(arg));
        qbs += PhiBSWTemp * czbssw * (1.0 - arg * sarg) / (1.0 - MJSW);
        capbs += czbssw * sarg;
      }
      if (czbsswg > 0.0) {
        arg = 1.0 - vbs / PhiBSWGTemp;
        if (MJSWG == 0.5)
          sarg = 1.0 / sqrt(arg);
        else
          sarg = exp(-MJSWG * log(arg));
        qbs += PhiBSWGTemp * czbsswg * (1.0 - arg * sarg) / (1.0 - MJSWG);
        capbs += czbsswg * sarg;
      }
    } else {
      T0 = czbs + czbssw + czbsswg;
      T1 = vbs * (czbs * MJ / PhiBTemp + czbssw * MJSW / PhiBSWTemp + czbsswg * MJSWG / PhiBSWGTemp);
      qbs = vbs * (T0 + 0.5 * T1);
      capbs = T0 + T1;
    }
    if (vbd == 0.0) {
      qbd = 0.0;
      capbd = czbd + czbdsw + czbdswg;
    } else if (vbd < 0.0) {
      if (czbd > 0.0) {
        arg = 1.0 - vbd / PhiBTemp;
        if (MJ == 0.5)
          sarg = 1.0 / sqrt(arg);
        else
          sarg = exp(-MJ * log(arg));
        qbd = PhiBTemp * czbd * (1.0 - arg * sarg) / (1.0 - MJ);
        capbd = czbd * sarg;
      } else {
        qbd = 0.0;
        capbd = 0.0;
      }
      if (czbdsw > 0.0) {
        arg = 1.0 - vbd / PhiBSWTemp;
        if (MJSW == 0.5)
          sarg = 1.0 / sqrt(arg);
        else
          sarg = exp(-MJSW * log(arg));
        qbd += PhiBSWTemp * czbdsw * (1.0 - arg * sarg) / (1.0 - MJSW);
        capbd += czbdsw * sarg;
      }
      if (czbdswg > 0.0) {
        arg = 1.0 - vbd / PhiBSWGTemp;
        if (MJSWG == 0.5)
          sarg = 1.0 / sqrt(arg);
        else
          sarg = exp(-MJSWG * log(arg));
        qbd += PhiBSWGTemp * czbdswg * (1.0 - arg * sarg) / (1.0 - MJSWG);
        capbd += czbdswg * sarg;
      }
    } else {
      T0 = czbd + czbdsw + czbdswg;
      T1 = vbd * (czbd * MJ / PhiBTemp + czbdsw * MJSW / PhiBSWTemp + czbdswg * MJSWG / PhiBSWGTemp);
      qbd = vbd * (T0 + 0.5 * T1);
      capbd = T0 + T1;
    }
    // Overlap capacitances (:7134-7205): constant (capMod 0), piecewise (1), smooth (2 / 3).
    const double weffCV = P(weffCV), ckappa = P(ckappa);
    double cgdo, qgdo, cgso, qgso;
    if ((int)P(capMod) == 0) {
      cgdo = P(cgdo);
      qgdo = P(cgdo) * vgd;
      cgso = P(cgso);
      qgso = P(cgso) * vgs;
    } else if ((int)P(capMod) == 1) {
      if (vgd < 0.0) {
        T1 = sqrt(1.0 - 4.0 * vgd / ckappa);
        cgdo = P(cgdo) + weffCV * P(cgdl) / T1;
        qgdo = P(cgdo) * vgd - weffCV * 0.5 * P(cgdl) * ckappa * (T1 - 1.0);
      } else {
        cgdo = P(cgdo) + weffCV * P(cgdl);
        qgdo = (weffCV * P(cgdl) + P(cgdo)) * vgd;
      }
      if (vgs < 0.0) {
        T1 = sqrt(1.0 - 4.0 * vgs / ckappa);
        cgso = P(cgso) + weffCV * P(cgsl) / T1;
        qgso = P(cgso) * vgs - weffCV * 0.5 * P(cgsl) * ckappa * (T1 - 1.0);
      } else {
        cgso = P(cgso) + weffCV * P(cgsl);
        qgso = (weffCV * P(cgsl) + P(cgso)) * vgs;
      }
    } else {
      T0 = vgd + CONSTDELTA_1;
      T1 = sqrt(T0 * T0 + 4.0 * CONSTDELTA_1);
      T2 = 0.5 * (T0 - T1);
      T3 = weffCV * P(cgdl);
      T4 = sqrt(1.0 - 4.0 * T2 / ckappa);
      cgdo = P(cgdo) + T3 - T3 * (1.0 - 1.0 / T4) * (0.5 - 0.5 * T0 / T1);
      qgdo = (P(cgdo) + T3) * vgd - T3 * (T2 + 0.5 * ckappa * (T4 - 1.0));
      T0 = vgs + CONSTDELTA_1;
      T1 = sqrt(T0 * T0 + 4.0 * CONSTDELTA_1);
      T2 = 0.5 * (T0 - T1);
      T3 = weffCV * P(cgsl);
      T4 = sqrt(1.0 - 4.0 * T2 / ckappa);
      cgso = P(cgso) + T3 - T3 * (1.0 - 1.0 / T4) * (0.5 - 0.5 * T0 / T1);
      qgso = (P(cgso) + T3) * vgs - T3 * (T2 + 0.5 * ckappa * (T4 - 1.0));
    }
    // setupCapacitors_oldDAE (charge bookkeeping only, nqsMod = 0).
    const double cgbo = P(cgbo);
    const double qgd = qgdo, qgs = qgso, qgb = cgbo * vgb;
    if (mode > 0) {
      qgate += qgd + qgs + qgb;
      qbulk -= qgb;
      qdrn -= qgd;
      qsrc = -(qgate + qbulk + qdrn);
    } else {
      qgate += qgd + qgs + qgb;
      qbulk -= qgb;
      qsrc = qdrn - qgs;
      qdrn = -(qgate + qbulk + qsrc);
    }
    // setupCapacitors_newDAE (nqsMod = 0).
    if (mode > 0) {
      CAPcggb = (cggb + cgdo + cgso + cgbo);
      CAPcgdb = (cgdb - cgdo);
      CAPcgsb = (cgsb - cgso);
      CAPcdgb = (cdgb - cgdo);
      CAPcddb = (cddb + capbd + cgdo);
      CAPcdsb = cdsb;
      CAPcsgb = -(cggb + cbgb + cdgb + cgso);
      CAPcsdb = -(cgdb + cbdb + cddb);
      CAPcssb = (capbs + cgso - (cgsb + cbsb + cdsb));
      CAPcbgb = (cbgb - cgbo);
      CAPcbdb = (cbdb - capbd);
      CAPcbsb = (cbsb - capbs);
    } else {
      CAPcggb = (cggb + cgdo + cgso + cgbo);
      CAPcgdb = (cgsb - cgdo);
      CAPcgsb = (cgdb - cgso);
      CAPcdgb = -(cggb + cbgb + cdgb + cgdo);
      CAPcddb = (capbd + cgdo - (cgsb + cbsb + cdsb));
      CAPcdsb = -(cgdb + cbdb + cddb);
      CAPcsgb = (cdgb - cgso);
      CAPcsdb = cdsb;
      CAPcssb = (cddb + capbs + cgso);
      CAPcbgb = (cbgb - cgbo);
      CAPcbdb = (cbsb - capbd);
      CAPcbsb = (cbdb - capbs);
    }
    qg = qgate;
    qd = qdrn - qbd;
    qb = qbulk + qbd + qbs;
  }

  // Master::updateState (:9199-9270).
  o.sto[s_vbs] = vbs;
  o.sto[s_vgs] = vgs;
  o.sto[s_vds] = vds;
  o.sto[s_vbd] = vbd;
  o.sto[s_von] = von;
  o.sta[t_qb] = qb;
  o.sta[t_qg] = qg;
  o.sta[t_qd] = qd;
  o.sta[t_qbs] = qbs;
  o.sta[t_qbd] = qbd;

  // Master::loadDAEVectors (:9276-9613). Local terminal order D=0, G=1, S=2, B=3; the drain and
  // source primes coincide with D and S.
  for (int k = 0; k < xb4::kNumVec; ++k) o.vec[k] = 0.0;
  double Gmv, Gmbs, FwdSum, RevSum, cdreq, ceqbd, ceqbs, gbbdp, gbbsp, gbdpg, gbdpdp, gbdpb, gbdpsp, gbspg, gbspdp,
      gbspb, gbspsp;
  const double cd = cdrain;
  if (mode >= 0) {
    Gmv = gm;
    Gmbs = gmbs;
    FwdSum = Gmv + Gmbs;
    RevSum = 0.0;
    cdreq = dtype * (cd);
    ceqbd = -dtype * (csub);
    ceqbs = 0.0;
    gbbdp = -gbds;
    gbbsp = (gbds + gbgs + gbbs);
    gbdpg = gbgs;
    gbdpdp = gbds;
    gbdpb = gbbs;
    gbdpsp = -(gbdpg + gbdpdp + gbdpb);
    gbspg = 0.0;
    gbspdp = 0.0;
    gbspb = 0.0;
    gbspsp = 0.0;
  } else {
    Gmv = -gm;
    Gmbs = -gmbs;
    FwdSum = 0.0;
    RevSum = -(Gmv + Gmbs);
    cdreq = -dtype * (cd);
    ceqbs = -dtype * (csub);
    ceqbd = 0.0;
    gbbsp = -gbds;
    gbbdp = (gbds + gbgs + gbbs);
    gbdpg = 0.0;
    gbdpsp = 0.0;
    gbdpb = 0.0;
    gbdpdp = 0.0;
    gbspg = gbgs;
    gbspsp = gbds;
    gbspb = gbbs;
    gbspdp = -(gbspg + gbspsp + gbspb);
  }
  if (dtype > 0) {
    ceqbs += (cbs);
    ceqbd += (cbd);
  } else {
    ceqbs -= (cbs);
    ceqbd -= (cbd);
  }
  if (SERIES) {
    // Resistor currents at the external nodes (:9355-9362); the primes take -Idrain / -Isource.
    const double gdr = P(drainConductance), gsr = P(sourceConductance);
    const double Idrain = gdr * Vddp, Isource = gsr * Vssp;
    o.vecx[0] = 0.0;
    o.vecx[1] = 0.0;
    if (gdr != 0.0) o.vecx[0] += Idrain * M;
    if (gsr != 0.0) o.vecx[1] += Isource * M;
    o.vec[3] += (ceqbs + ceqbd) * M;
    o.vec[0] += (-(ceqbd - cdreq) - Idrain) * M;
    o.vec[2] += (-(cdreq + ceqbs) - Isource) * M;
  } else {
    o.vec[3] += (ceqbs + ceqbd) * M;
    o.vec[0] += (-(ceqbd - cdreq)) * M;
    o.vec[2] += (-(cdreq + ceqbs)) * M;
  }
  if (fl.voltlim && !origFlag) {
    double cdreq_Jdxp, ceqbd_Jdxp, ceqbs_Jdxp = 0.0;
    if (mode >= 0) {
      cdreq_Jdxp = dtype * (-gds * (vds - vds_orig) - Gmv * (vgs - vgs_orig) - Gmbs * (vbs - vbs_orig));
      ceqbd_Jdxp = -dtype * (-gbds * (vds - vds_orig) - gbgs * (vgs - vgs_orig) - gbbs * (vbs - vbs_orig));
    } else {
      cdreq_Jdxp = -dtype * (gds * (vds - vds_orig) + Gmv * (vgd - vgd_orig) + Gmbs * (vbd - vbd_orig));
      ceqbd_Jdxp = -dtype * (gbds * (vds - vds_orig) - gbgs * (vgd - vgd_orig) - gbbs * (vbd - vbd_orig));
    }
    if (dtype > 0) {
      ceqbs_Jdxp += (-gbs * (vbs - vbs_orig));
      ceqbd_Jdxp += (-gbd * (vbd - vbd_orig));
    } else {
      ceqbs_Jdxp -= (-gbs * (vbs - vbs_orig));
      ceqbd_Jdxp -= (-gbd * (vbd - vbd_orig));
    }
    o.vec[8 + 3] += -(ceqbs_Jdxp + ceqbd_Jdxp) * M;
    o.vec[8 + 0] += (ceqbd_Jdxp - cdreq_Jdxp) * M;
    o.vec[8 + 2] += (cdreq_Jdxp + ceqbs_Jdxp) * M;
  }
  // auxChargeCalculations (:7447-7542) and the Q vector.
  double Qeqqg_Jdxp = 0.0, Qeqqb_Jdxp = 0.0, Qeqqd_Jdxp = 0.0;
  if (ChargeComputationNeeded && !origFlag) {
    const double vgb_orig = vgs_orig - vbs_orig;
    Qeqqg_Jdxp = -CAPcggb * (vgb - vgb_orig) + CAPcgdb * (vbd - vbd_orig) + CAPcgsb * (vbs - vbs_orig);
    Qeqqb_Jdxp = -CAPcbgb * (vgb - vgb_orig) + CAPcbdb * (vbd - vbd_orig) + CAPcbsb * (vbs - vbs_orig);
    Qeqqd_Jdxp = -CAPcdgb * (vgb - vgb_orig) + CAPcddb * (vbd - vbd_orig) + CAPcdsb * (vbs - vbs_orig);
  }
  double Qeqqg, Qeqqb, Qeqqd;
  if (dtype > 0) {
    Qeqqg = qg;
    Qeqqb = qb;
    Qeqqd = qd;
  } else {
    Qeqqg = -qg;
    Qeqqb = -qb;
    Qeqqd = -qd;
  }
  o.vec[4 + 1] += Qeqqg * M;
  o.vec[4 + 3] += (Qeqqb)*M;
  o.vec[4 + 0] += (-(-Qeqqd)) * M;
  o.vec[4 + 2] += (-(+Qeqqg + Qeqqb + Qeqqd)) * M;
  if (fl.voltlim) {
    if (!(dtype > 0)) {
      Qeqqg_Jdxp = -Qeqqg_Jdxp;
      Qeqqb_Jdxp = -Qeqqb_Jdxp;
      Qeqqd_Jdxp = -Qeqqd_Jdxp;
    }
    if (!origFlag) {
      o.vec[12 + 1] += -Qeqqg_Jdxp * M;
      o.vec[12 + 3] += -(+Qeqqb_Jdxp) * M;
      o.vec[12 + 0] += (-Qeqqd_Jdxp) * M;
      o.vec[12 + 2] += (+Qeqqg_Jdxp + Qeqqb_Jdxp + Qeqqd_Jdxp) * M;
    }
  }

  // Master::loadDAEMatrices (:9624-9900). The non-quasi-static terms (dxpart * ggt*, T1global *
  // ddxpart_*) are zero for nqsMod = 0, and the series-resistance terms are zero without RSH.
  for (int k = 0; k < xb4::kNumMat; ++k) {
    o.jf[k] = 0.0;
    o.jq[k] = 0.0;
  }
#define JF(r, c) o.jf[(r)*4 + (c)]
#define JQ(r, c) o.jq[(r)*4 + (c)]
  if (SERIES) {
    // The sheet-resistance couplings, in the reference's statement order (:9631-9647, 9705, 9739).
    const double gdr = P(drainConductance), gsr = P(sourceConductance);
    for (int k = 0; k < 6; ++k) o.jfx[k] = 0.0;
    o.jfx[2] += gdr * M;
    o.jfx[1] -= gdr * M;
    o.jfx[5] += gsr * M;
    o.jfx[4] -= gsr * M;
    JF(3, 1) += (-gbgs) * M;
    JF(3, 3) += (gbd + gbs - gbbs) * M;
    JF(3, 0) += (-gbd + gbbdp) * M;
    JF(3, 2) += (-gbs + gbbsp) * M;
    o.jfx[0] -= gdr * M;
    JF(0, 3) -= (gbd - Gmbs - gbdpb) * M;
    JF(0, 1) += (Gmv + gbdpg) * M;
    JF(0, 0) += (gdr + gds + gbd + RevSum + gbdpdp) * M;
    JF(0, 2) -= (gds + FwdSum - gbdpsp) * M;
    JF(2, 1) += (-Gmv + gbspg) * M;
    JF(2, 3) -= (gbs + Gmbs - gbspb) * M;
    o.jfx[3] -= gsr * M;
    JF(2, 0) -= (gds + RevSum - gbspdp) * M;
    JF(2, 2) += (gsr + gds + gbs + FwdSum + gbspsp) * M;
  } else {
    JF(3, 1) += (-gbgs) * M;
    JF(3, 3) += (gbd + gbs - gbbs) * M;
    JF(3, 0) += (-gbd + gbbdp) * M;
    JF(3, 2) += (-gbs + gbbsp) * M;
    JF(0, 3) -= (gbd - Gmbs - gbdpb) * M;
    JF(0, 1) += (Gmv + gbdpg) * M;
    JF(0, 0) += (gds + gbd + RevSum + gbdpdp) * M;
    JF(0, 2) -= (gds + FwdSum - gbdpsp) * M;
    JF(2, 1) += (-Gmv + gbspg) * M;
    JF(2, 3) -= (gbs + Gmbs - gbspb) * M;
    JF(2, 0) -= (gds + RevSum - gbspdp) * M;
    JF(2, 2) += (gds + gbs + FwdSum + gbspsp) * M;
  }
  if (!(!fl.dcop && fl.init_tran && fl.newton_iter == 0)) {
    JQ(1, 1) += (CAPcggb)*M;
    JQ(1, 3) -= (CAPcggb + CAPcgdb + CAPcgsb) * M;
    JQ(1, 0) += (CAPcgdb)*M;
    JQ(1, 2) += (CAPcgsb)*M;
    JQ(3, 1) += (CAPcbgb)*M;
    JQ(3, 3) += (-CAPcbgb - CAPcbdb - CAPcbsb) * M;
    JQ(3, 0) += (CAPcbdb)*M;
    JQ(3, 2) += (CAPcbsb)*M;
    JQ(0, 3) -= (+CAPcdgb + CAPcddb + CAPcdsb) * M;
    JQ(0, 1) += (CAPcdgb)*M;
    JQ(0, 0) += (+CAPcddb) * M;
    JQ(0, 2) -= (-CAPcdsb) * M;
    JQ(2, 1) += (CAPcsgb)*M;
    JQ(2, 3) -= (+CAPcsgb + CAPcsdb + CAPcssb) * M;
    JQ(2, 0) -= (-CAPcsdb) * M;
    JQ(2, 2) += (+CAPcssb) * M;
  }
#undef JF
#undef JQ
#undef P
}

}  // namespace xb3
