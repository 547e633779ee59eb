// Charge models shared by the BSIM3 and BSIM4 loads.
//
// cv_simple: the simple intrinsic charge model (capMod = 0), the same sequence of operations in
// both models (src/DeviceModelPKG/OpenModels/src/N_DEV_MOSFET_B3.C:5975-6240,
// N_DEV_MOSFET_B4.C:10718-11012): accumulation, depletion and inversion regions with their own
// flat band (VFBCV) and threshold, and the 0/100, 40/60 and 50/50 charge partitions. BSIM4 passes
// CoxWL with the finger count, BSIM3 without; the two references differ in one term of the 40/60
// linear region (bsim3 selects BSIM3's). The reference overwrites its Vbseff, Vth, Vgst and
// Vdsat here; no later part of either load reads them, so they are locals.
#pragma once

#include <cmath>

#include "xd_consts.h"

namespace xdc {

struct CvCharges {
  double qgate, qbulk, qdrn;
  double cggb, cgsb, cgdb, cdgb, cdsb, cddb, cbgb, cbsb, cbdb;
};

XD_HD void cv_simple(double Vbseff, double Vbs, double phi, double Phis, double dPhis_dVb, double sqrtPhis,
                     double dsqrtPhis_dVb, double vfbcv, double k1ox, double Vgs_eff, double dVgs_eff_dVg,
                     double CoxWL, double Abulk0, double dAbulk0_dVb, double abulkCVfactor, double Vds,
                     double xpart_, bool bsim3, CvCharges &c) {
  double T0, T1, T2, T3, T4, T5, T6, T7 = 0.0, T8 = 0.0, T9, T10, T11, T12, tmp, tmp1;
  double Vbs0, dVbs0_dVb;
  if (Vbseff < 0.0) {
    Vbs0 = Vbs;
    dVbs0_dVb = 1.0;
  } else {
    Vbs0 = phi - Phis;
    dVbs0_dVb = -dPhis_dVb;
  }
  const double Vfb0 = vfbcv;
  const double k1ox0 = k1ox;
  const double Vth0 = Vfb0 + phi + k1ox0 * sqrtPhis;
  const double Vgst0 = Vgs_eff - Vth0;
  const double dVth0_dVb = k1ox0 * dsqrtPhis_dVb;
  const double Arg1 = Vgs_eff - Vbs0 - Vfb0;
  if (Arg1 <= 0.0) {  // accumulation
    c.qgate = CoxWL * Arg1;
    c.qbulk = -c.qgate;
    c.qdrn = 0.0;
    c.cggb = CoxWL * dVgs_eff_dVg;
    c.cgdb = 0.0;
    c.cgsb = CoxWL * (dVbs0_dVb - dVgs_eff_dVg);
    c.cdgb = 0.0;
    c.cddb = 0.0;
    c.cdsb = 0.0;
    c.cbgb = -CoxWL * dVgs_eff_dVg;
    c.cbdb = 0.0;
    c.cbsb = -c.cgsb;
  } else if (Vgst0 <= 0.0) {  // depletion
    T1 = 0.5 * k1ox0;
    T2 = sqrt(T1 * T1 + Arg1);
    c.qgate = CoxWL * k1ox0 * (T2 - T1);
    c.qbulk = -c.qgate;
    c.qdrn = 0.0;
    T0 = CoxWL * T1 / T2;
    c.cggb = T0 * dVgs_eff_dVg;
    c.cgdb = 0.0;
    c.cgsb = T0 * (dVbs0_dVb - dVgs_eff_dVg);
    c.cdgb = 0.0;
    c.cddb = 0.0;
    c.cdsb = 0.0;
    c.cbgb = -c.cggb;
    c.cbdb = 0.0;
    c.cbsb = -c.cgsb;
  } else {  // inversion
    const double One_Third_CoxWL = CoxWL / 3.0;
    const double Two_Third_CoxWL = 2.0 * One_Third_CoxWL;
    const double AbulkCV = Abulk0 * abulkCVfactor;
    const double dAbulkCV_dVb = abulkCVfactor * dAbulk0_dVb;
    const double Vdsat0 = Vgst0 / AbulkCV;
    const double dVdsat_dVg = dVgs_eff_dVg / AbulkCV;
    const double dVdsat_dVb = -(Vdsat0 * dAbulkCV_dVb + dVth0_dVb) / AbulkCV;
    const double xpart = xpart_;
    const bool sat = (xpart > 0.5) ? (Vdsat0 <= Vds) : (Vds >= Vdsat0);
    if (sat) {
      T1 = Vdsat0 / 3.0;
      c.qgate = CoxWL * (Vgs_eff - Vfb0 - phi - T1);
      T2 = -Two_Third_CoxWL * Vgst0;
      c.qbulk = -(c.qgate + T2);
      // drain share of the inversion charge: 0 (0/100), 0.4 (40/60), 0.5 (50/50)
      c.qdrn = (xpart > 0.5) ? 0.0 : ((xpart < 0.5) ? 0.4 * T2 : 0.5 * T2);
      c.cggb = One_Third_CoxWL * (3.0 - dVdsat_dVg) * dVgs_eff_dVg;
      T2 = -One_Third_CoxWL * dVdsat_dVb;
      c.cgsb = -(c.cggb + T2);
      c.cgdb = 0.0;
      if (xpart > 0.5) {
        c.cdgb = 0.0;
        c.cddb = 0.0;
        c.cdsb = 0.0;
      } else if (xpart < 0.5) {
        T3 = 0.4 * Two_Third_CoxWL;
        c.cdgb = -T3 * dVgs_eff_dVg;
        c.cddb = 0.0;
        T4 = T3 * dVth0_dVb;
        c.cdsb = -(T4 + c.cdgb);
      } else {
        c.cdgb = -One_Third_CoxWL * dVgs_eff_dVg;
        c.cddb = 0.0;
        T4 = One_Third_CoxWL * dVth0_dVb;
        c.cdsb = -(T4 + c.cdgb);
      }
      c.cbgb = -(c.cggb - Two_Third_CoxWL * dVgs_eff_dVg);
      T3 = -(T2 + Two_Third_CoxWL * dVth0_dVb);
      c.cbsb = -(c.cbgb + T3);
      c.cbdb = 0.0;
    } else {  // linear region
      const double Alphaz = Vgst0 / Vdsat0;
      T1 = 2.0 * Vdsat0 - Vds;
      T2 = Vds / (3.0 * T1);
      T3 = T2 * Vds;
      T9 = 0.25 * CoxWL;
      T4 = T9 * Alphaz;
      if (xpart > 0.5) {
        T7 = 2.0 * Vds - T1 - 3.0 * T3;
        T8 = T3 - T1 - 2.0 * Vds;
      }
      c.qgate = CoxWL * (Vgs_eff - Vfb0 - phi - 0.5 * (Vds - T3));
      if (xpart > 0.5) {
        T10 = T4 * T8;
        c.qdrn = T4 * T7;
        c.qbulk = -(c.qgate + c.qdrn + T10);
      }
      T5 = T3 / T1;
      c.cggb = CoxWL * (1.0 - T5 * dVdsat_dVg) * dVgs_eff_dVg;
      if (xpart > 0.5) {
        T11 = -CoxWL * T5 * dVdsat_dVb;
        c.cgdb = CoxWL * (T2 - 0.5 + 0.5 * T5);
        c.cgsb = -(c.cggb + T11 + c.cgdb);
      } else {
        tmp = -CoxWL * T5 * dVdsat_dVb;
        c.cgdb = CoxWL * (T2 - 0.5 + 0.5 * T5);
        c.cgsb = -(c.cggb + c.cgdb + tmp);
      }
      T6 = 1.0 / Vdsat0;
      const double dAlphaz_dVg = T6 * (1.0 - Alphaz * dVdsat_dVg);
      const double dAlphaz_dVb = -T6 * (dVth0_dVb + Alphaz * dVdsat_dVb);
      if (xpart > 0.5) {  // 0/100
        T7 = T9 * T7;
        T8 = T9 * T8;
        T9 = 2.0 * T4 * (1.0 - 3.0 * T5);
        c.cdgb = (T7 * dAlphaz_dVg - T9 * dVdsat_dVg) * dVgs_eff_dVg;
        T12 = T7 * dAlphaz_dVb - T9 * dVdsat_dVb;
        c.cddb = T4 * (3.0 - 6.0 * T2 - 3.0 * T5);
        c.cdsb = -(c.cdgb + T12 + c.cddb);
        T9 = 2.0 * T4 * (1.0 + T5);
        T10 = (T8 * dAlphaz_dVg - T9 * dVdsat_dVg) * dVgs_eff_dVg;
        T11 = T8 * dAlphaz_dVb - T9 * dVdsat_dVb;
        T12 = T4 * (2.0 * T2 + T5 - 1.0);
        T0 = -(T10 + T11 + T12);
        c.cbgb = -(c.cggb + c.cdgb + T10);
        c.cbdb = -(c.cgdb + c.cddb + T12);
        c.cbsb = -(c.cgsb + c.cdsb + T0);
      } else if (xpart < 0.5) {  // 40/60
        T6 = 8.0 * Vdsat0 * Vdsat0 - 6.0 * Vdsat0 * Vds + 1.2 * Vds * Vds;
        T8 = T2 / T1;
        T7 = Vds - T1 - T8 * T6;
        c.qdrn = T4 * T7;
        T7 *= T9;
        tmp = T8 / T1;
        tmp1 = T4 * (2.0 - 4.0 * tmp * T6 + T8 * (16.0 * Vdsat0 - 6.0 * Vds));
        c.cdgb = (T7 * dAlphaz_dVg - tmp1 * dVdsat_dVg) * dVgs_eff_dVg;
        T10 = T7 * dAlphaz_dVb - tmp1 * dVdsat_dVb;
        c.cddb = T4 * (2.0 - (1.0 / (3.0 * T1 * T1) + 2.0 * tmp) * T6 + T8 * (6.0 * Vdsat0 - 2.4 * Vds));
        c.cdsb = -(c.cdgb + T10 + c.cddb);
        T7 = 2.0 * (T1 + T3);
        c.qbulk = -(c.qgate - T4 * T7);
        T7 *= T9;
        T0 = 4.0 * T4 * (1.0 - T5);
        T12 = (-T7 * dAlphaz_dVg - c.cdgb - T0 * dVdsat_dVg) * dVgs_eff_dVg;
        T11 = -T7 * dAlphaz_dVb - T10 - T0 * dVdsat_dVb;
        T10 = -4.0 * T4 * (T2 - 0.5 + 0.5 * T5) - c.cddb;
        tmp = -(T10 + T11 + T12);
        c.cbgb = -(c.cggb + c.cdgb + T12);
        // BSIM3's drain-bulk term takes T11 here (N_DEV_MOSFET_B3.C:6208), BSIM4's T10 (B4.C:10941).
        c.cbdb = -(c.cgdb + c.cddb + (bsim3 ? T11 : T10));
        c.cbsb = -(c.cgsb + c.cdsb + tmp);
      } else {  // 50/50
        T7 = T1 + T3;
        c.qdrn = -T4 * T7;
        c.qbulk = -(c.qgate + c.qdrn + c.qdrn);
        T7 *= T9;
        T0 = T4 * (2.0 * T5 - 2.0);
        c.cdgb = (T0 * dVdsat_dVg - T7 * dAlphaz_dVg) * dVgs_eff_dVg;
        T12 = T0 * dVdsat_dVb - T7 * dAlphaz_dVb;
        c.cddb = T4 * (1.0 - 2.0 * T2 - T5);
        c.cdsb = -(c.cdgb + T12 + c.cddb);
        c.cbgb = -(c.cggb + 2.0 * c.cdgb);
        c.cbdb = -(c.cgdb + 2.0 * c.cddb);
        c.cbsb = -(c.cgsb + 2.0 * c.cdsb);
      }
    }
  }
}

}  // namespace xdc
