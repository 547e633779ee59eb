// MOSFET level 1 (Shichman-Hodges with Meyer capacitances): set-up and per-instance load.
//
// Restates, in the reference's order of floating-point operations:
//   model card and Model::processParams     src/DeviceModelPKG/OpenModels/src/N_DEV_MOSFET1.C:120-292, 3752-3955
//   instance defaults                        N_DEV_MOSFET1.C:1160-1262
//   Instance::updateTemperature              N_DEV_MOSFET1.C:3403-3655
//   Instance::updateIntermediateVars         N_DEV_MOSFET1.C:2584-3402
//   DeviceSupport::qmeyer                    src/DeviceModelPKG/Core/src/N_DEV_DeviceSupport.C:545-632
//   Master::updateState                      N_DEV_MOSFET1.C:4069-4160
//   Master::loadDAEVectors / loadDAEMatrices N_DEV_MOSFET1.C:4168-4396, 4407-4697
// for the reference's default Meyer back-averaging (NEWMEYER off) and without instance initial
// conditions. Without drain/source series resistance (RD = RS = 0, no sheet resistance) the
// drain and source primes collapse onto the terminals: the 4-terminal stamp, the same staged
// layout as the BSIM4 load. With it (SERIES = true) the primes are internal nodes and the
// resistors load into the BSIM4 wide layout (vecx / jfx).
#pragma once

#include <string>
#include <vector>

#include "bsim4_eval.cuh"  // LoadFlags, RecPtr, staged layout constants
#include "bsim4_setup.h"   // ModelSpec, SetupOptions, RecordTable
#include "xd_consts.h"

#define XM1_FIELDS(F)                                                                                 \
  F(dtype) F(gamma) F(lambda) F(mj) F(mjsw) F(vt) F(tPhi) F(tVbi) F(tVto) F(sourceVcrit) F(drainVcrit) \
  F(Beta) F(DrainSatCur) F(SourceSatCur) F(Cbd) F(Cbdsw) F(Cbs) F(Cbssw) F(tDepCap) F(tBulkPot)       \
  F(f2d) F(f3d) F(f4d) F(f2s) F(f3s) F(f4s) F(GateSourceOverlapCap) F(GateDrainOverlapCap)            \
  F(GateBulkOverlapCap) F(OxideCap) F(mult) F(off) F(drainConductance) F(sourceConductance)

namespace xm1 {

enum Field {
#define XM1_ENUM(n) f_##n,
  XM1_FIELDS(XM1_ENUM)
#undef XM1_ENUM
  kNumFields
};

// Store slots (registerStoreLIDs order, N_DEV_MOSFET1.C:1513-1540) and state slots
// (registerStateLIDs order, :1452-1510).
enum StoreSlot { s_vbd, s_vbs, s_vgs, s_vds, s_von, kNumStore };
enum StateSlot { t_qgs, t_qgd, t_qgb, t_capgs, t_capgd, t_capgb, t_qbd, t_qbs, kNumState };

std::string build_records(const std::vector<xb4::ModelSpec> &models, int n_inst, const int *inst_model,
                          const std::vector<std::string> &inst_param_names, const double *inst_param_values,
                          const xb4::SetupOptions &opts, xb4::RecordTable &out);

struct LoadOut {
  double vec[xb4::kNumVec];
  double jf[xb4::kNumMat];
  double jq[xb4::kNumMat];
  double sto[kNumStore];
  double sta[kNumState];
  // With internal nodes: F at the external drain and source, dF/dx at (D', D), (D, D'), (D, D),
  // (S', S), (S, S'), (S, S).
  double vecx[2];
  double jfx[6];
};

// Meyer gate capacitances (DeviceSupport::qmeyer).
XD_HD void qmeyer(double vgs, double vgd, double vgb, double von, double vdsat, double &capgs, double &capgd,
                  double &capgb, double phi, double cox) {
  (void)vgb;
  const double vgst = vgs - von;
  if (vgst <= -phi) {
    capgb = cox / 2;
    capgs = 0;
    capgd = 0;
  } else if (vgst <= -phi / 2) {
    capgb = -vgst * cox / (2 * phi);
    capgs = 0;
    capgd = 0;
  } else if (vgst <= 0) {
    capgb = -vgst * cox / (2 * phi);
    capgs = vgst * cox / (1.5 * phi) + cox / 3;
    capgd = 0;
  } else {
    const double vds = vgs - vgd;
    if (vdsat <= vds) {
      capgs = cox / 3;
      capgd = 0;
      capgb = 0;
    } else {
      const double vddif = 2.0 * vdsat - vds;
      const double vddif1 = vdsat - vds;
      const double vddif2 = vddif * vddif;
      capgd = cox * (1.0 - vdsat * vdsat / vddif2) / 3;
      capgs = cox * (1.0 - vddif1 * vddif1 / vddif2) / 3;
      capgb = 0;
    }
  }
}

// One MOSFET1 instance. V = terminal voltages (D, G, S, B); sto_old = limiter history (currSto on
// Newton step 0, nextSto otherwise); curr_sta / curr_sto = the previous accepted time point's state
// and store, read for Meyer back-averaging.
// SERIES = true: V holds (D', G, S', B) and Vx the external (D, S); the drain/source resistors
// (N_DEV_MOSFET1.C:1180-1220, 3302-3303) load into vecx / jfx.
template <bool SERIES = false, class RV>
XD_HD void mos1_load(const RV &P_, const double V[4], const double *sto_old, const double *curr_sta,
                     const double *curr_sto, const xb4::LoadFlags &fl, LoadOut &o, const double *Vx = nullptr) {
  using namespace xdc;
#define P(x) P_(f_##x)
  const double dtype = P(dtype);
  const double gmin = fl.gmin;
  const double M = P(mult);
  const bool OFF = P(off) != 0.0;
  const double vt = P(vt);
  const double DrainSatCur = P(DrainSatCur), SourceSatCur = P(SourceSatCur);
  const double Beta = P(Beta);
  const double Vdp = V[0], Vg = V[1], Vsp = V[2], Vb = V[3];
  const double Vd = SERIES ? Vx[0] : Vdp, Vs = SERIES ? Vx[1] : Vsp;
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
  if (fl.init_jct && !OFF && fl.voltlim) {
    vbs = -1;
    vgs = dtype * P(tVto);
    vds = 0;
    vbd = vbs - vds;
    vgd = vgs - vds;
  } else if ((fl.init_fix || fl.init_jct) && OFF) {
    vbs = vgs = vds = 0;
    vbd = vgd = 0;
  }
  double vbs_old, vbd_old, vgs_old, vds_old, Von;
  if (fl.newton_iter == 0 && fl.dcop) {
    vbs_old = vbs;
    vbd_old = vbd;
    vgs_old = vgs;
    vds_old = vds;
    Von = 0.0;
  } else {
    vbs_old = sto_old[s_vbs];
    vbd_old = sto_old[s_vbd];
    vgs_old = sto_old[s_vgs];
    vds_old = sto_old[s_vds];
    Von = dtype * sto_old[s_von];
  }
  const double vgd_old = vgs_old - vds_old;
  if (fl.voltlim) {
    if (!(fl.init_fix && OFF)) {
      int Check = 1;
      if (vds_old >= 0) {
        vgs = fetlim(vgs, vgs_old, Von);
        vds = vgs - vgd;
        vds = limvds(vds, vds_old);
        vgd = vgs - vds;
      } else {
        vgd = fetlim(vgd, vgd_old, Von);
        vds = vgs - vgd;
        vds = -limvds(-vds, -vds_old);
        vgs = vgd + vds;
      }
      if (vds >= 0.0) {
        vbs = pnjlim(vbs, vbs_old, vt, P(sourceVcrit), &Check);
        vbd = vbs - vds;
      } else {
        vbd = pnjlim(vbd, vbd_old, vt, P(drainVcrit), &Check);
        vbs = vbd + vds;
      }
    }
  }
  vbd = vbs - vds;
  vgd = vgs - vds;
  const double Vgb = vgs - vbs;
  if (vgs_orig != vgs || vds_orig != vds || vbs_orig != vbs || vbd_orig != vbd || vgd_orig != vgd) origFlag = 0;
  double gbs, cbs, gbd, cbd;
  if (vbs <= 0) {
    gbs = SourceSatCur / vt;
    gbs += gmin;
    cbs = gbs * vbs;
  } else {
    const double evbs = exp(dmin(CONSTMAX_EXP_ARG, vbs / vt));
    gbs = (SourceSatCur * evbs / vt + gmin);
    cbs = (SourceSatCur * (evbs - 1) + gmin * vbs);
  }
  if (vbd <= 0) {
    gbd = DrainSatCur / vt;
    gbd += gmin;
    cbd = gbd * vbd;
  } else {
    const double evbd = exp(dmin(CONSTMAX_EXP_ARG, vbd / vt));
    gbd = (DrainSatCur * evbd / vt + gmin);
    cbd = (DrainSatCur * (evbd - 1) + gmin * vbd);
  }
  const int mode = (vds >= 0) ? 1 : -1;
  double cdrain, gm, gds, gmbs, Vdsat;
  {
    const double tPhi = P(tPhi);
    const double gamma = P(gamma), lambda = P(lambda);
    const double vbx = (mode == 1 ? vbs : vbd);
    double sarg;
    if (vbx <= 0) {
      sarg = sqrt(tPhi - vbx);
    } else {
      sarg = sqrt(tPhi);
      sarg = sarg - vbx / (sarg + sarg);
      sarg = dmax(0.0, sarg);
    }
    Von = (P(tVbi) * dtype) + gamma * sarg;
    const double vgst = (mode == 1 ? vgs : vgd) - Von;
    Vdsat = dmax(vgst, 0.0);
    const double arg = (sarg <= 0) ? 0 : gamma / (sarg + sarg);
    if (vgst <= 0) {
      cdrain = 0;
      gm = 0;
      gds = 0;
      gmbs = 0;
    } else {
      const double betap = Beta * (1 + lambda * (vds * mode));
      if (vgst <= (vds * mode)) {
        cdrain = betap * vgst * vgst * .5;
        gm = betap * vgst;
        gds = lambda * Beta * vgst * vgst * .5;
        gmbs = gm * arg;
      } else {
        cdrain = betap * (vds * mode) * (vgst - .5 * (vds * mode));
        gm = betap * (vds * mode);
        gds = betap * (vgst - (vds * mode)) + lambda * Beta * (vds * mode) * (vgst - .5 * (vds * mode));
        gmbs = gm * arg;
      }
    }
  }
  const double von = dtype * Von;
  // Junction charges and capacitances (:3000-3110).
  const double Cbs = P(Cbs), Cbssw = P(Cbssw), Cbd = P(Cbd), Cbdsw = P(Cbdsw);
  const double tDepCap = P(tDepCap), tBulkPot = P(tBulkPot), MJ = P(mj), MJSW = P(mjsw);
  double qbs, capbs, qbd, capbd;
  if (Cbs != 0 || Cbssw != 0) {
    if (vbs < tDepCap) {
      const double arg = 1 - vbs / tBulkPot;
      double sarg, sargsw;
      if (MJ == MJSW) {
        if (MJ == .5)
          sarg = sargsw = 1 / sqrt(arg);
        else
          sarg = sargsw = exp(-MJ * log(arg));
      } else {
        if (MJ == .5)
          sarg = 1 / sqrt(arg);
        else
          sarg = exp(-MJ * log(arg));
        if (MJSW == .5)
          sargsw = 1 / sqrt(arg);
        else
          sargsw = exp(-MJSW * log(arg));
      }
      qbs = tBulkPot * (Cbs * (1 - arg * sarg) / (1 - MJ) + Cbssw * (1 - arg * sargsw) / (1 - MJSW));
      capbs = Cbs * sarg + Cbssw * sargsw;
    } else {
      qbs = P(f4s) + vbs * (P(f2s) + vbs * (P(f3s) / 2));
      capbs = P(f2s) + P(f3s) * vbs;
    }
  } else {
    qbs = 0;
    capbs = 0;
  }
  if (Cbd != 0 || Cbdsw != 0) {
    if (vbd < tDepCap) {
      const double arg = 1 - vbd / tBulkPot;
      double sarg, sargsw;
      if (MJ == .5 && MJSW == .5) {
        sarg = sargsw = 1 / sqrt(arg);
      } else {
        if (MJ == .5)
          sarg = 1 / sqrt(arg);
        else
          sarg = exp(-MJ * log(arg));
        if (MJSW == .5)
          sargsw = 1 / sqrt(arg);
        else
          sargsw = exp(-MJSW * log(arg));
      }
      qbd = tBulkPot * (Cbd * (1 - arg * sarg) / (1 - MJ) + Cbdsw * (1 - arg * sargsw) / (1 - MJSW));
      capbd = Cbd * sarg + Cbdsw * sargsw;
    } else {
      qbd = P(f4d) + vbd * (P(f2d) + vbd * P(f3d) / 2);
      capbd = P(f2d) + vbd * P(f3d);
    }
  } else {
    qbd = 0;
    capbd = 0;
  }
  // Meyer capacitances with back-averaging (:3110-3170).
  double capgs, capgd, capgb;
  if (mode > 0)
    qmeyer(vgs, vgd, Vgb, Von, Vdsat, capgs, capgd, capgb, P(tPhi), P(OxideCap));
  else
    qmeyer(vgd, vgs, Vgb, Von, Vdsat, capgd, capgs, capgb, P(tPhi), P(OxideCap));
  double Capgs, Capgd, Capgb;
  if (fl.dcop) {
    Capgs = 2.0 * capgs + P(GateSourceOverlapCap);
    Capgd = 2.0 * capgd + P(GateDrainOverlapCap);
    Capgb = 2.0 * capgb + P(GateBulkOverlapCap);
  } else {
    Capgs = (capgs + curr_sta[t_capgs] + P(GateSourceOverlapCap));
    Capgd = (capgd + curr_sta[t_capgd] + P(GateDrainOverlapCap));
    Capgb = (capgb + curr_sta[t_capgb] + P(GateBulkOverlapCap));
  }
  Capgs *= (Capgs < 0.0) ? -1.0 : 1.0;
  Capgd *= (Capgd < 0.0) ? -1.0 : 1.0;
  Capgb *= (Capgb < 0.0) ? -1.0 : 1.0;
  double Gm, Gmbs, nrmsum, revsum, cdreq;
  if (mode >= 0) {
    Gm = gm;
    Gmbs = gmbs;
    nrmsum = Gm + Gmbs;
    revsum = 0;
    cdreq = dtype * cdrain;
  } else {
    Gm = -gm;
    Gmbs = -gmbs;
    nrmsum = 0;
    revsum = -(Gm + Gmbs);
    cdreq = -(dtype)*cdrain;
  }
  // Master::updateState: store and state (:4069-4160).
  o.sto[s_vbd] = vbd;
  o.sto[s_vbs] = vbs;
  o.sto[s_vgs] = vgs;
  o.sto[s_vds] = vds;
  o.sto[s_von] = von;
  o.sta[t_capgs] = capgs;
  o.sta[t_capgd] = capgd;
  o.sta[t_capgb] = capgb;
  double qgs, qgd, qgb;
  if (fl.dcop) {
    qgs = Capgs * vgs;
    qgd = Capgd * vgd;
    qgb = Capgb * Vgb;
  } else {
    qgs = curr_sta[t_qgs];
    qgd = curr_sta[t_qgd];
    qgb = curr_sta[t_qgb];
    const double vgs1 = curr_sto[s_vgs];
    const double vbs1 = curr_sto[s_vbs];
    const double vds1 = curr_sto[s_vds];
    const double vgb1 = vgs1 - vbs1;
    const double vgd1 = vgs1 - vds1;
    qgs += Capgs * (vgs - vgs1);
    qgd += Capgd * (vgd - vgd1);
    qgb += Capgb * ((vgs - vbs) - vgb1);
  }
  o.sta[t_qgs] = qgs;
  o.sta[t_qgd] = qgd;
  o.sta[t_qgb] = qgb;
  o.sta[t_qbd] = qbd;
  o.sta[t_qbs] = qbs;

  // Master::loadDAEVectors (:4168-4396). Local order D'=0, G=1, S'=2, B=3 (the primes coincide
  // with D and S without series resistance).
  for (int k = 0; k < xb4::kNumVec; ++k) o.vec[k] = 0.0;
  const double ceqbs = dtype * (cbs), ceqbd = dtype * (cbd), ceqgb = 0.0, ceqgs = 0.0, ceqgd = 0.0;
  const double gdr = SERIES ? P(drainConductance) : 0.0, gsr = SERIES ? P(sourceConductance) : 0.0;
  const double Idrain = SERIES ? gdr * (Vd - Vdp) : 0.0, Isource = SERIES ? gsr * (Vs - Vsp) : 0.0;
  if (SERIES) {
    o.vecx[0] = 0.0;
    o.vecx[1] = 0.0;
    if (gdr != 0.0) o.vecx[0] += Idrain * M;
  }
  double coef = (ceqgs + ceqgd + ceqgb);
  o.vec[1] += coef * M;
  if (SERIES && gsr != 0.0) o.vecx[1] += Isource * M;
  coef = ceqbs + ceqbd - ceqgb;
  o.vec[3] += coef * M;
  coef = -Idrain - (ceqbd - cdreq + ceqgd);
  o.vec[0] += coef * M;
  coef = -Isource - (ceqbs + cdreq + ceqgs);
  o.vec[2] += coef * M;
  const double Qeqbs = dtype * (qbs), Qeqbd = dtype * (qbd), Qeqgb = dtype * (qgb), Qeqgs = dtype * (qgs),
               Qeqgd = dtype * (qgd);
  coef = (Qeqgs + Qeqgd + Qeqgb);
  o.vec[4 + 1] += coef * M;
  coef = Qeqbs + Qeqbd - Qeqgb;
  o.vec[4 + 3] += coef * M;
  coef = -(Qeqbd + Qeqgd);
  o.vec[4 + 0] += coef * M;
  coef = -(Qeqbs + Qeqgs);
  o.vec[4 + 2] += coef * M;
  const bool charges = fl.tranop || fl.acop || fl.transient;
  const double gcgd = charges ? Capgd : 0.0, gcgs = charges ? Capgs : 0.0, gcgb = charges ? Capgb : 0.0;
  const double gcbs = charges ? capbs : 0.0, gcbd = charges ? capbd : 0.0;
  if (!origFlag) {
    const double dvgx = (mode > 0) ? (vgs - vgs_orig) : (vgd - vgd_orig);
    const double dvbx = (mode > 0) ? (vbs - vbs_orig) : (vbd - vbd_orig);
    const double c4 = dtype * (+((gbd - gmin)) * (vbd - vbd_orig) + ((gbs - gmin)) * (vbs - vbs_orig));
    const double c5 = dtype * (-((gbd - gmin)) * (vbd - vbd_orig) + gds * (vds - vds_orig) + Gm * dvgx + Gmbs * dvbx);
    const double c6 = dtype * (-((gbs - gmin)) * (vbs - vbs_orig) - gds * (vds - vds_orig) - Gm * dvgx - Gmbs * dvbx);
    o.vec[8 + 3] += c4 * M;
    o.vec[8 + 0] += c5 * M;
    o.vec[8 + 2] += c6 * M;
    const double q2 = dtype * (gcgd * (vgd - vgd_orig) + gcgs * (vgs - vgs_orig) +
                               gcgb * (vgs - vgs_orig - vbs + vbs_orig));
    const double q4 = dtype * (-(gcgb) * (vgs - vgs_orig - vbs + vbs_orig) + (gcgb) * (vbd - vbd_orig) +
                               (gcbs) * (vbs - vbs_orig));
    const double q5 = dtype * (-(gcgd) * (vgd - vgd_orig) - (gcbd) * (vbd - vbd_orig));
    const double q6 = dtype * (-gcgs * (vgs - vgs_orig) - (gcbs) * (vbs - vbs_orig));
    o.vec[12 + 1] += q2 * M;
    o.vec[12 + 3] += q4 * M;
    o.vec[12 + 0] += q5 * M;
    o.vec[12 + 2] += q6 * M;
  }

  // Master::loadDAEMatrices (:4407-4697), NEWMEYER off.
  for (int k = 0; k < xb4::kNumMat; ++k) {
    o.jf[k] = 0.0;
    o.jq[k] = 0.0;
  }
#define JF(r, c) o.jf[(r)*4 + (c)]
#define JQ(r, c) o.jq[(r)*4 + (c)]
  if (SERIES) {
    // The resistor couplings in the reference's statement order (:4449-4452, 4482-4485, 4541,
    // 4578).
    for (int k = 0; k < 6; ++k) o.jfx[k] = 0.0;
    o.jfx[2] += gdr * M;
    o.jfx[1] -= gdr * M;
    o.jfx[5] += gsr * M;
    o.jfx[4] -= gsr * M;
    JF(3, 3) += (gbs + gbd) * M;
    JF(3, 0) -= gbd * M;
    JF(3, 2) -= gbs * M;
    o.jfx[0] -= gdr * M;
    JF(0, 1) += (Gm) * M;
    JF(0, 3) += (-gbd + Gmbs) * M;
    JF(0, 0) += (gdr + gds + gbd + revsum) * M;
    JF(0, 2) += (-gds - nrmsum) * M;
    JF(2, 1) -= (Gm) * M;
    o.jfx[3] -= gsr * M;
    JF(2, 3) -= (gbs + Gmbs) * M;
    JF(2, 0) -= (gds + revsum) * M;
    JF(2, 2) += (gsr + gds + gbs + nrmsum) * M;
  } else {
    const double drainConductance = 0.0, sourceConductance = 0.0;
    JF(0, 0) += drainConductance * M;
    JF(0, 0) -= drainConductance * M;
    JF(2, 2) += sourceConductance * M;
    JF(2, 2) -= sourceConductance * M;
    JF(3, 3) += (gbs + gbd) * M;
    JF(3, 0) -= gbd * M;
    JF(3, 2) -= gbs * M;
    JF(0, 0) -= drainConductance * M;
    JF(0, 1) += (Gm) * M;
    JF(0, 3) += (-gbd + Gmbs) * M;
    JF(0, 0) += (drainConductance + gds + gbd + revsum) * M;
    JF(0, 2) += (-gds - nrmsum) * M;
    JF(2, 1) -= (Gm) * M;
    JF(2, 2) -= sourceConductance * M;
    JF(2, 3) -= (gbs + Gmbs) * M;
    JF(2, 0) -= (gds + revsum) * M;
    JF(2, 2) += (sourceConductance + gds + gbs + nrmsum) * M;
  }
  JQ(1, 1) += (gcgd + gcgs + gcgb) * M;
  JQ(1, 3) -= gcgb * M;
  JQ(1, 0) -= gcgd * M;
  JQ(1, 2) -= gcgs * M;
  JQ(3, 1) -= gcgb * M;
  JQ(3, 3) += (+gcbs + gcbd + gcgb) * M;
  JQ(3, 0) -= +gcbd * M;
  JQ(3, 2) -= +gcbs * M;
  JQ(0, 1) += -gcgd * M;
  JQ(0, 3) += -gcbd * M;
  JQ(0, 0) += (+gcbd + gcgd) * M;
  JQ(2, 1) -= gcgs * M;
  JQ(2, 3) -= +gcbs * M;
  JQ(2, 2) += (+gcbs + gcgs) * M;
#undef JF
#undef JQ
#undef P
}

}  // namespace xm1
