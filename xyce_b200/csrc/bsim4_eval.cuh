// BSIM4 (v4.6.1) per-instance load: voltage limiting, DC and charge model, and the stamp values
// for F, Q, dF/dx, dQ/dx and the limiter correction vectors, for one instance.
//
// One call evaluates one instance entirely in registers (one CUDA thread per instance on the
// device). It restates, in the reference's order of floating-point operations:
//   Instance::updateIntermediateVars    N_DEV_MOSFET_B4.C:7744-11918
//   Instance::setupCapacitors_oldDAE     N_DEV_MOSFET_B4.C:12616-13045 (charge bookkeeping only)
//   Instance::setupCapacitors_newDAE     N_DEV_MOSFET_B4.C:12357-12608
//   Master::updateState                  N_DEV_MOSFET_B4.C:16180-16293
//   Instance::setupFVectorVars           N_DEV_MOSFET_B4.C:13525-13855
//   Instance::auxChargeCalculations      N_DEV_MOSFET_B4.C:12216-12350
//   Master::loadDAEVectors / loadDAEMatrices  N_DEV_MOSFET_B4.C:16303-16567, 16577-17268
// for the configuration the set-up accepts: rgateMod = rbodyMod = trnqsMod = acnqsMod = rdsMod = 0,
// igcMod 0/1/2, igbMod 0/1, capMod 0/1/2, no source/drain resistance nodes, no initial conditions. With
// no internal nodes the 11 stamp rows collapse onto the 4 terminals D, G, S, B.
//
// Local stamp layout (terminal order D=0, G=1, S=2, B=3):
//   vec[0..3]   F,  vec[4..7] Q,  vec[8..11] dFdxdVp,  vec[12..15] dQdxdVp
//   jf[r*4+c]   dF_r/dx_c,  jq[r*4+c]  dQ_r/dx_c
// Within one slot the terms are accumulated in the reference's statement order.
#pragma once

#include "bsim4_fields.h"
#include "xd_consts.h"
#include "mos_cv.h"

namespace xb4 {

struct LoadFlags {
  int dcop, init_tran, newton_iter, init_jct, init_fix, transient, tranop, acop, voltlim, input_op;
  double gmin, pdt;
};

// Store slots (registerStoreLIDs order, N_DEV_MOSFET_B4.C:5267-5290) and state slots
// (registerStateLIDs order, :5200-5230).
enum StoreSlot { s_vbd, s_vbs, s_vgs, s_vds, s_vges, s_vgms, s_vdes, s_vses, s_vdbs, s_vsbs, s_vdbd, s_vged, s_vgmd, s_von, kNumStore };
enum StateSlot { t_qb, t_qg, t_qd, kNumState };
enum { kNumVec = 16, kNumMat = 16, kNumStage = kNumVec + 2 * kNumMat };
// Series-resistance layout (internal drain / source nodes): the four vectors get rows 4 and 5 for
// the external drain and source, the matrices six more slots for the resistor couplings.
enum { kSerVecRows = 6, kSerMat = kNumMat + 6, kSerStage = 4 * kSerVecRows + 2 * kSerMat };

// General topology (rgateMod 1-3, rbodyMod 1/2, rdsMod 1, trnqsMod 1, instance initial conditions,
// and the sheet-resistance D' / S' nodes): the reference's full stamp over 15 local nodes — the
// four terminals, the internal drain / source / gate / gate-mid / body / source-body / drain-body
// nodes, the NQS charge node (registerLIDs order, N_DEV_MOSFET_B4.C:5018-5079) and the three
// initial-condition branch currents. A node the instance does not have is the same unknown as the
// one it collapses onto (D' -> D, S' -> S, G' and GM -> G, B' / SB / DB -> B); an absent charge node
// or branch current has no unknown.
enum GenNode {
  g_D, g_G, g_S, g_B, g_DP, g_SP, g_GP, g_GM, g_BP, g_SB, g_DB, g_Q, g_IBS, g_IDS, g_IGS, kGenNodes
};
// The stamp's (row, column) pairs in the reference's jacStamp order (:4641-4755): rows D, G, S, B,
// D', S', G', GM, B', SB, DB, the charge row, then the three initial-condition rows with their two
// couplings each; the charge node's columns in rows D', S', G' last.
constexpr int kGenStamp[][2] = {
    {g_D, g_D},   {g_D, g_DP},   {g_D, g_SP},   {g_D, g_GP},   {g_D, g_BP},
    {g_G, g_G},   {g_G, g_DP},   {g_G, g_SP},   {g_G, g_GP},   {g_G, g_GM},   {g_G, g_BP},
    {g_S, g_S},   {g_S, g_DP},   {g_S, g_SP},   {g_S, g_GP},   {g_S, g_BP},
    {g_B, g_B},   {g_B, g_BP},   {g_B, g_SB},   {g_B, g_DB},
    {g_DP, g_D},  {g_DP, g_DP},  {g_DP, g_SP},  {g_DP, g_GP},  {g_DP, g_GM},  {g_DP, g_BP},  {g_DP, g_DB},
    {g_SP, g_S},  {g_SP, g_DP},  {g_SP, g_SP},  {g_SP, g_GP},  {g_SP, g_GM},  {g_SP, g_BP},  {g_SP, g_SB},
    {g_GP, g_G},  {g_GP, g_DP},  {g_GP, g_SP},  {g_GP, g_GP},  {g_GP, g_GM},  {g_GP, g_BP},
    {g_GM, g_G},  {g_GM, g_DP},  {g_GM, g_SP},  {g_GM, g_GP},  {g_GM, g_GM},  {g_GM, g_BP},
    {g_BP, g_B},  {g_BP, g_DP},  {g_BP, g_SP},  {g_BP, g_GP},  {g_BP, g_GM},  {g_BP, g_BP},  {g_BP, g_SB},
    {g_BP, g_DB},
    {g_SB, g_B},  {g_SB, g_SP},  {g_SB, g_BP},  {g_SB, g_SB},
    {g_DB, g_B},  {g_DB, g_DP},  {g_DB, g_BP},  {g_DB, g_DB},
    {g_Q, g_DP},  {g_Q, g_SP},   {g_Q, g_GP},   {g_Q, g_BP},   {g_Q, g_Q},
    {g_IBS, g_S}, {g_IBS, g_B},  {g_IBS, g_IBS}, {g_S, g_IBS}, {g_B, g_IBS},
    {g_IDS, g_D}, {g_IDS, g_S},  {g_IDS, g_IDS}, {g_D, g_IDS}, {g_S, g_IDS},
    {g_IGS, g_G}, {g_IGS, g_S},  {g_IGS, g_IGS}, {g_G, g_IGS}, {g_S, g_IGS},
    {g_DP, g_Q},  {g_SP, g_Q},   {g_GP, g_Q}};
constexpr int kGenSlots = sizeof(kGenStamp) / sizeof(kGenStamp[0]);
static_assert(kGenSlots == 85, "the general stamp has 62 device entries, 8 NQS entries and 15 initial-condition entries");
// Slot of (row, col) in kGenStamp; -1 if the stamp has no such entry.
constexpr int gen_slot(int r, int c) {
  for (int k = 0; k < kGenSlots; ++k)
    if (kGenStamp[k][0] == r && kGenStamp[k][1] == c) return k;
  return -1;
}
// The slot of (R, C) as a compile-time constant: a stamp statement whose entry is not in the table
// does not compile.
template <int R, int C>
struct GenSlotOf {
  static constexpr int value = gen_slot(R, C);
  static_assert(value >= 0, "the general stamp has no such entry");
};
// State slots of the general topology: the three intrinsic charges, then the gate-mid charge
// (rgateMod 3), the two junction charges (rbodyMod) and the NQS charges qcheq, qcdump (trnqsMod),
// in registerStateLIDs order (:5212-5238).
enum GenState { gt_qb, gt_qg, gt_qd, gt_qgmid, gt_qbs, gt_qbd, gt_qcheq, gt_qcdump, kGenState };
// Staging of one instance: 4 vectors x 15 rows, then dF/dx and dQ/dx over the 85 stamp slots.
enum { kGenVecRows = kGenNodes, kGenStage = 4 * kGenVecRows + 2 * kGenSlots };

struct LoadOut {
  double vec[kNumVec];
  double jf[kNumMat];
  double jq[kNumMat];
  // With internal nodes: F at the external drain and source, and dF/dx at (D', D), (D, D'),
  // (D, D), (S', S), (S, S'), (S, S); rows 0 and 2 of vec/jf/jq are then D' and S'.
  double vecx[2];
  double jfx[6];
  double sto[kNumStore];  // s_vged and s_vgmd are not written by the load (kept from the input)
  double sta[kNumState];
  bool write_curr_sta;    // first Newton step of the first transient step: also write currSta
  double vgb;             // this load's vgb (the next load's "vgb_orig")
  // General topology: vectors gv[v * 15 + node] (F, Q, dF/dx*dVp, dQ/dx*dVp), the two matrices over
  // the stamp slots, and the eight state slots (zero where the instance has no such charge).
  double gv[4 * kGenNodes];
  double gf[kGenSlots];
  double gq[kGenSlots];
  double gsta[kGenState];
};

// Field-major record view: field f of this instance's record.
struct RecPtr {
  const double *base;
  int stride;
  XD_HD double operator()(int f) const {
#if defined(__CUDA_ARCH__)
    return __ldg(base + (size_t)f * stride);
#else
    return base[(size_t)f * stride];
#endif
  }
};

XD_HD void poly_depletion(double phi, double ngate, double epsgate, double coxe, double Vgs_arg, double &Vgs_eff,
                          double &dVgs_eff_dVg) {
  if ((ngate > 1.0e18) && (ngate < 1.0e25) && (Vgs_arg > phi) && (epsgate != 0)) {
    double T1 = 1.0e6 * xdc::CONSTQ * epsgate * ngate / (coxe * coxe);
    double T8 = Vgs_arg - phi;
    double T4 = sqrt(1.0 + 2.0 * T8 / T1);
    double T2 = 2.0 * T8 / (T4 + 1.0);
    double T3 = 0.5 * T2 * T2 / T1;
    double T7 = 1.12 - T3 - 0.05;
    double T6 = sqrt(T7 * T7 + 0.224);
    double T5 = 1.12 - 0.5 * (T7 + T6);
    Vgs_eff = Vgs_arg - T5;
    dVgs_eff_dVg = 1.0 - (0.5 - 0.5 / T4) * (1.0 + T7 / T6);
  } else {
    Vgs_eff = Vgs_arg;
    dVgs_eff_dVg = 1.0;
  }
}

// V[4] = node voltages (D, G, S, B); sto_old = the store values the limiter compares against
// (currSto on Newton step 0 of a transient step, nextSto otherwise); vgb_orig = the previous load's
// vgb of this instance (0 before the first load), which the reference uses as the "original" vgb.
// FULL = false compiles the load for the common card only — capMod 2, no gate tunnelling
// (igcMod = igbMod = 0) — whatever the record says, so the default kernel carries none of the
// other branches in its registers or its code; families whose cards use capMod 0/1 or the
// tunnelling currents run the FULL = true instantiation.
// SERIES = true: V holds (D', G, S', B) and Vx the external (D, S); the linear drain and source
// resistances (rdsMod = 0, sheet resistance) load into vecx / jfx.

// Hand-off state between the two parts of the evaluation when they run as separate kernels: the
// DC part (limiting, junction diodes, drain current, GIDL / GISL, gate tunnelling) stores these per
// instance, and the charge-and-stamp part (charges, capacitances, store / state, stamps) reads them.
// Parameters and node voltages are not in it: the second part reads them again; everything it
// derives from them (branch voltages from the limited vds / vgs / vbs, Phis from Vbseff, ...) it
// recomputes with the same operations, so the split evaluation is bit-identical to the fused one.
enum MidSlot {
  m_vds, m_vgs, m_vbs, m_orig, m_von, m_gbs, m_cbs, m_gbd, m_cbd, m_cdrain, m_gds, m_gm, m_gmbs, m_csub,
  m_gbbs, m_gbgs, m_gbds, m_Igidl, m_ggidld, m_ggidlg, m_ggidlb, m_Igisl, m_ggisls, m_ggislg, m_ggislb,
  m_Abulk0, m_dAbulk0_dVb, m_Vbseff, m_dVbseff_dVb, m_Vgs_eff, m_dVgs_eff_dVg, m_Vgst, m_dVth_dVb, m_dVth_dVd,
  m_n, m_dn_dVb, m_dn_dVd,
  kNumMid,
  // Gate tunnelling currents (the full evaluation variants only).
  m_Igs = kNumMid, m_gIgsg, m_gIgss, m_Igd, m_gIgdg, m_gIgdd, m_Igcs, m_gIgcsg, m_gIgcsd, m_gIgcsb, m_Igcd,
  m_gIgcdg, m_gIgcdd, m_gIgcdb, m_Igb, m_gIgbg, m_gIgbd, m_gIgbb,
  kNumMidFull,
  // General topology: the limited gate, source / drain and body-network voltages, the gate
  // resistance conductances (rgateMod 2/3) and the bias-dependent S/D conductances (rdsMod 1).
  m_vges = kNumMidFull, m_vgms, m_vdes, m_vses, m_vdbs, m_vsbs, m_gcrg, m_gcrgg, m_gcrgd, m_gcrgs, m_gcrgb,
  m_gstot, m_gstotd, m_gstotg, m_gstots, m_gstotb, m_gdtot, m_gdtotd, m_gdtotg, m_gdtots, m_gdtotb,
  kNumMidGen
};
struct Mid {
  double v[kNumMidGen];
};

#define P(x) P_(f_##x)

// Node and branch voltages of one instance and their unlimited ("orig") copies, with the
// initial-condition overrides applied (:7932-8097).
struct Bias {
  double Vd, Vs, Vdp, Vsp, Vddp, Vssp;
  // General topology: body-network drops, gate-resistor drops (unlimited, untyped: :7966-8004).
  double Vdbb, Vdbbp, Vsbb, Vsbbp, Vbpb, Vgegp, Vgegm, Vgmgp;
  double vds, vgs, vbs, vges, vgms, vdbs, vsbs, vses, vdes, vbd, vdbd, vgd, vged, vgmd, vgmb, vbs_jct, vbd_jct;
  double vbd_orig, vbs_orig, vgs_orig, vds_orig, vgd_orig, vges_orig, vgms_orig, vdes_orig, vses_orig, vdbs_orig;
  double vsbs_orig, vdbd_orig, vged_orig, vgmd_orig, vbs_jct_orig, vbd_jct_orig, vgmb_orig;
  double qdef;  // NQS: the charge node's value, typed (:7950-7986); zero without trnqsMod
  int origFlag;
};

// V: with GEN the 15 local node values (GenNode order; collapsed nodes carry their representative's
// value), else the 4 (D', G, S', B) with Vx the external (D, S) under SERIES.
template <bool SERIES, bool GEN = false, class RV>
XD_HD void bsim4_bias(const RV &P_, const double *V, const LoadFlags &fl, const double *Vx, Bias &b) {
  using namespace xdc;
  const double dtype = P(dtype);
  const double vth0 = P(vth0);
  const bool OFF = P(off) != 0.0;
  const bool rbodyMod = GEN && P(rbodyMod) != 0.0;
  // Node and branch voltages (:7932-8030).
  double Vdp, Vge, Vsp, Vb, Vd, Vs, Vgp, Vbp, Vgm, Vdb, Vsb;
  if (GEN) {
    Vd = V[g_D]; Vs = V[g_S]; Vb = V[g_B]; Vsp = V[g_SP]; Vdp = V[g_DP];
    Vgp = V[g_GP]; Vbp = V[g_BP]; Vge = V[g_G]; Vgm = V[g_GM]; Vdb = V[g_DB]; Vsb = V[g_SB];
  } else {
    Vdp = V[0]; Vge = V[1]; Vsp = V[2]; Vb = V[3];
    Vd = SERIES ? Vx[0] : Vdp;
    Vs = SERIES ? Vx[1] : Vsp;
    Vgp = Vge; Vbp = Vb; Vgm = Vge; Vdb = Vb; Vsb = Vb;
  }
  const double Vddp = Vd - Vdp, Vssp = Vs - Vsp;
  double vds = dtype * (Vdp - Vsp);
  double vgs = dtype * (Vgp - Vsp);
  double vbs = dtype * (Vbp - Vsp);
  double vges = dtype * (Vge - Vsp);
  double vgms = dtype * (Vgm - Vsp);
  double vdbs = dtype * (Vdb - Vsp);
  double vsbs = dtype * (Vsb - Vsp);
  double vses = dtype * (Vs - Vsp);
  double vdes = dtype * (Vd - Vsp);
  double vbd = vbs - vds;
  double vdbd = vdbs - vds;
  double vgd = vgs - vds;
  double vged = vges - vds;
  double vgmd = vgms - vds;
  double vgmb = vgms - vbs;
  double vbs_jct = (!rbodyMod) ? vbs : vsbs;
  double vbd_jct = (!rbodyMod) ? vbd : vdbd;
  b.Vdbb = Vdb - Vb;
  b.Vdbbp = Vdb - Vbp;
  b.Vsbb = Vsb - Vb;
  b.Vsbbp = Vsb - Vbp;
  b.Vbpb = Vbp - Vb;
  b.Vgegp = Vge - Vgp;
  b.Vgegm = Vge - Vgm;
  b.Vgmgp = Vgm - Vgp;
  int origFlag = 1;
  const double vbd_orig = vbd, vbs_orig = vbs, vgs_orig = vgs, vds_orig = vds, vgd_orig = vgd;
  const double vges_orig = vges, vgms_orig = vgms, vdes_orig = vdes, vses_orig = vses, vdbs_orig = vdbs;
  const double vsbs_orig = vsbs, vdbd_orig = vdbd, vged_orig = vged, vgmd_orig = vgmd;
  const double vbs_jct_orig = vbs_jct, vbd_jct_orig = vbd_jct, vgmb_orig = vgmb;

  // Initial-condition handling (:8051-8097). inputOP with a flag vector is not modelled.
  if (fl.init_jct && !OFF && fl.voltlim) {
    vds = 0.1;
    vdes = 0.11;
    vses = -0.01;
    vgs = vges = vgms = dtype * vth0 + 0.1;
    origFlag = 0;
    vbs = vdbs = vsbs = 0.0;
    vbd = vbs - vds;
    vdbd = vdbs - vds;
    vgd = vgs - vds;
    vged = vges - vds;
    vgmd = vgms - vds;
  } else if ((fl.init_fix || fl.init_jct) && OFF) {
    vds = vgs = vbs = vges = vgms = 0.0;
    vds = vsbs = vdes = vses = 0.0;
  }
  // NQS: the charge node's value (:7950-7986), zeroed with the voltages of an OFF device (:8096).
  b.qdef = (GEN && P(trnqsMod) != 0.0) ? dtype * V[g_Q] : 0.0;
  if ((fl.init_fix || fl.init_jct) && OFF) b.qdef = 0.0;
  b.Vd = Vd; b.Vs = Vs; b.Vdp = Vdp; b.Vsp = Vsp; b.Vddp = Vddp; b.Vssp = Vssp;
  b.vds = vds; b.vgs = vgs; b.vbs = vbs; b.vges = vges; b.vgms = vgms; b.vdbs = vdbs; b.vsbs = vsbs;
  b.vses = vses; b.vdes = vdes; b.vbd = vbd; b.vdbd = vdbd; b.vgd = vgd; b.vged = vged; b.vgmd = vgmd;
  b.vgmb = vgmb; b.vbs_jct = vbs_jct; b.vbd_jct = vbd_jct;
  b.vbd_orig = vbd_orig; b.vbs_orig = vbs_orig; b.vgs_orig = vgs_orig; b.vds_orig = vds_orig;
  b.vgd_orig = vgd_orig; b.vges_orig = vges_orig; b.vgms_orig = vgms_orig; b.vdes_orig = vdes_orig;
  b.vses_orig = vses_orig; b.vdbs_orig = vdbs_orig; b.vsbs_orig = vsbs_orig; b.vdbd_orig = vdbd_orig;
  b.vged_orig = vged_orig; b.vgmd_orig = vgmd_orig; b.vbs_jct_orig = vbs_jct_orig;
  b.vbd_jct_orig = vbd_jct_orig; b.vgmb_orig = vgmb_orig;
  b.origFlag = origFlag;
}

// Charge-and-stamp part of the evaluation: charges and capacitances, store and state, the F / Q /
// limiter-vector stamps and the dF/dx, dQ/dx stamps (:10707-13855, 16195-17268), from the DC part's
// hand-off state m.
template <bool FULL = false, bool SERIES = false, bool GEN = false, class RV>
XD_HD void bsim4_finish(const RV &P_, const double *V, const LoadFlags &fl, double vgb_orig, const Mid &m,
                        LoadOut &o, const double *Vx) {
  using namespace xdc;
  const double dtype = P(dtype);
  const int capMod = FULL ? (int)P(capMod) : 2;
  const int igcMod = FULL ? (int)P(igcMod) : 0, igbMod = FULL ? (int)P(igbMod) : 0;
  const double nf = P(nf);
  const double M = P(mult);
  const bool ChargeComputationNeeded = (fl.tranop || fl.acop || fl.transient);
  const int rgateMod = GEN ? (int)P(rgateMod) : 0;
  const bool rbodyMod = GEN && P(rbodyMod) != 0.0;
  const bool rdsMod = GEN && P(rdsMod) != 0.0;
  Bias bias;
  bsim4_bias<SERIES, GEN>(P_, V, fl, Vx, bias);
  const double Vddp = bias.Vddp, Vssp = bias.Vssp;
  (void)Vddp; (void)Vssp;
  double vds = bias.vds, vgs = bias.vgs, vbs = bias.vbs, vges = bias.vges, vgms = bias.vgms, vdbs = bias.vdbs;
  double vsbs = bias.vsbs, vses = bias.vses, vdes = bias.vdes, vbd = bias.vbd, vdbd = bias.vdbd, vgd = bias.vgd;
  double vged = bias.vged, vgmd = bias.vgmd, vgmb = bias.vgmb, vbs_jct = bias.vbs_jct, vbd_jct = bias.vbd_jct;
  const double vbd_orig = bias.vbd_orig, vbs_orig = bias.vbs_orig, vgs_orig = bias.vgs_orig;
  const double vds_orig = bias.vds_orig, vgd_orig = bias.vgd_orig, vges_orig = bias.vges_orig;
  const double vgms_orig = bias.vgms_orig, vdes_orig = bias.vdes_orig, vses_orig = bias.vses_orig;
  const double vdbs_orig = bias.vdbs_orig, vsbs_orig = bias.vsbs_orig, vdbd_orig = bias.vdbd_orig;
  const double vged_orig = bias.vged_orig, vgmd_orig = bias.vgmd_orig, vbs_jct_orig = bias.vbs_jct_orig;
  const double vbd_jct_orig = bias.vbd_jct_orig, vgmb_orig = bias.vgmb_orig;
  (void)vdes_orig; (void)vses_orig; (void)vdbs_orig; (void)vsbs_orig; (void)vdbd_orig; (void)vged_orig;
  (void)vgmd_orig; (void)vges_orig; (void)vgms_orig;
  int origFlag = bias.origFlag;
  // The reference takes vgb_orig from the instance's vgb member before it is recomputed, i.e. the
  // previous load's value (:8026); in the limiter test below vgb therefore equals vgb_orig.
  double vgb = vgb_orig;
  vds = m.v[m_vds];
  vgs = m.v[m_vgs];
  vbs = m.v[m_vbs];
  origFlag = (int)m.v[m_orig];
  if (GEN) {
    vges = m.v[m_vges];
    vgms = m.v[m_vgms];
    vdes = m.v[m_vdes];
    vses = m.v[m_vses];
    vdbs = m.v[m_vdbs];
    vsbs = m.v[m_vsbs];
  }
  vbd = vbs - vds;
  vgd = vgs - vds;
  vgb = vgs - vbs;
  vged = vges - vds;
  vgmd = vgms - vds;
  vgmb = vgms - vbs;
  vdbd = vdbs - vds;
  vbs_jct = (!rbodyMod) ? vbs : vsbs;
  vbd_jct = (!rbodyMod) ? vbd : vdbd;
  (void)vged; (void)vgmd;
  double T0, T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12, T13, T14;
  double dT0_dVg, dT0_dVd, dT0_dVb, dT1_dVg, dT1_dVd, dT1_dVb, dT2_dVg, dT2_dVd, dT2_dVb;
  double dT3_dVg, dT3_dVd, dT3_dVb, dT4_dVd, dT5_dVg, dT5_dVd, dT5_dVb, dT6_dVg, dT6_dVd, dT6_dVb;
  double dT8_dVg, dT8_dVd, dT8_dVb, dT9_dVg, dT9_dVd, dT9_dVb, dT10_dVg, dT10_dVd, dT10_dVb;
  double tmp, tmp1, tmp2, tmp3, tmp4;
  const double Aseff = P(Aseff), Pseff = P(Pseff), Adeff = P(Adeff), Pdeff = P(Pdeff), weffCJ = P(weffCJ);
  (void)Pseff; (void)Pdeff;
  const double gbs = m.v[m_gbs], cbs = m.v[m_cbs], gbd = m.v[m_gbd], cbd = m.v[m_cbd];
  const int mode = vds >= 0.0 ? 1 : -1;
  const double Vds = mode > 0 ? vds : -vds;
  const double Vbs = mode > 0 ? vbs : vbd;
  const double epssub = CONSTEPSSI;
  const double phi = P(phi), sqrtPhi_p = P(sqrtPhi);
  const double Vbseff = m.v[m_Vbseff], dVbseff_dVb = m.v[m_dVbseff_dVb];
  const double Phis = phi - Vbseff;
  const double dPhis_dVb = -1.0;
  const double sqrtPhis = sqrt(Phis);
  const double dsqrtPhis_dVb = -0.5 / sqrtPhis;
  const double Vtm = P(vtm);
  const double k1ox = P(k1ox);
  const double coxe = P(coxe);
  const double coxp = P(coxp);
  const double dVth_dVb = m.v[m_dVth_dVb], dVth_dVd = m.v[m_dVth_dVd];
  const double n = m.v[m_n], dn_dVb = m.v[m_dn_dVb], dn_dVd = m.v[m_dn_dVd];
  const double von = m.v[m_von];
  const double Vgs_eff = m.v[m_Vgs_eff], dVgs_eff_dVg = m.v[m_dVgs_eff_dVg];
  const double Vgst = m.v[m_Vgst];
  const double Abulk0 = m.v[m_Abulk0], dAbulk0_dVb = m.v[m_dAbulk0_dVb];
  const double cdrain = m.v[m_cdrain], gds = m.v[m_gds], gm = m.v[m_gm], gmbs = m.v[m_gmbs];
  const double csub = m.v[m_csub], gbbs = m.v[m_gbbs], gbgs = m.v[m_gbgs], gbds = m.v[m_gbds];
  const double Igidl = m.v[m_Igidl], ggidld = m.v[m_ggidld], ggidlg = m.v[m_ggidlg], ggidlb = m.v[m_ggidlb];
  const double Igisl = m.v[m_Igisl], ggisls = m.v[m_ggisls], ggislg = m.v[m_ggislg], ggislb = m.v[m_ggislb];
  const double Igs = FULL ? m.v[m_Igs] : 0.0, gIgsg = FULL ? m.v[m_gIgsg] : 0.0, gIgss = FULL ? m.v[m_gIgss] : 0.0;
  const double Igd = FULL ? m.v[m_Igd] : 0.0, gIgdg = FULL ? m.v[m_gIgdg] : 0.0, gIgdd = FULL ? m.v[m_gIgdd] : 0.0;
  const double Igcs = FULL ? m.v[m_Igcs] : 0.0, gIgcsg = FULL ? m.v[m_gIgcsg] : 0.0;
  const double gIgcsd = FULL ? m.v[m_gIgcsd] : 0.0, gIgcsb = FULL ? m.v[m_gIgcsb] : 0.0;
  const double Igcd = FULL ? m.v[m_Igcd] : 0.0, gIgcdg = FULL ? m.v[m_gIgcdg] : 0.0;
  const double gIgcdd = FULL ? m.v[m_gIgcdd] : 0.0, gIgcdb = FULL ? m.v[m_gIgcdb] : 0.0;
  const double Igb = FULL ? m.v[m_Igb] : 0.0, gIgbg = FULL ? m.v[m_gIgbg] : 0.0;
  const double gIgbd = FULL ? m.v[m_gIgbd] : 0.0, gIgbb = FULL ? m.v[m_gIgbb] : 0.0;
  const double gIgbs = -(gIgbg + gIgbd + gIgbb);
  const double gIgcss = -(gIgcsg + gIgcsd + gIgcsb);
  const double gIgcds = -(gIgcdg + gIgcdd + gIgcdb);
  double Coxeff, dCoxeff_dVg, Tcen, dTcen_dVg, Denomi, Vgsteff, dVgsteff_dVg, dVgsteff_dVd, dVgsteff_dVb;

  // Intrinsic charges (:10707-11620): capMod 0, 1 or 2 (charge-thickness model).
  double qgate = 0, qdrn = 0, qbulk = 0, qsrc = 0;
  double cggb = 0, cgsb = 0, cgdb = 0, cdgb = 0, cdsb = 0, cddb = 0, cbgb = 0, cbsb = 0, cbdb = 0;
  if ((P(xpart) < 0) || (!ChargeComputationNeeded)) {
    // all zero
  } else if (capMod == 0) {
    // capMod = 0 (:10718-11012), the simple charge model BSIM3 shares.
    xdc::CvCharges cv;
    xdc::cv_simple(Vbseff, Vbs, phi, Phis, dPhis_dVb, sqrtPhis, dsqrtPhis_dVb, P(vfbcv), P(k1ox), Vgs_eff,
                   dVgs_eff_dVg, coxe * P(weffCV) * P(leffCV) * nf, Abulk0, dAbulk0_dVb, P(abulkCVfactor), Vds,
                   P(xpart), false, cv);
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
    const double CoxWL = coxe * P(weffCV) * P(leffCV) * nf;
    if (P(cvchargeMod) == 0.0) {
      const double noff = n * P(noff);
      const double dnoff_dVd = P(noff) * dn_dVd;
      const double dnoff_dVb = P(noff) * dn_dVb;
      T0 = Vtm * noff;
      const double voffcv = P(voffcv);
      const double VgstNVt = (Vgst - voffcv) / T0;
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
    } else {
      const double mstarcv = P(mstarcv);
      T0 = n * Vtm;
      T1 = mstarcv * Vgst;
      T2 = T1 / T0;
      if (T2 > CONSTEXP_THRESHOLD) {
        T10 = T1;
        dT10_dVg = mstarcv * dVgs_eff_dVg;
        dT10_dVd = -dVth_dVd * mstarcv;
        dT10_dVb = -dVth_dVb * mstarcv;
      } else if (T2 < -CONSTEXP_THRESHOLD) {
        T10 = Vtm * log(1.0 + CONSTMIN_EXP);
        dT10_dVg = 0.0;
        dT10_dVd = T10 * dn_dVd;
        dT10_dVb = T10 * dn_dVb;
        T10 *= n;
      } else {
        const double ExpVgst = exp(T2);
        T3 = Vtm * log(1.0 + ExpVgst);
        T10 = n * T3;
        dT10_dVg = mstarcv * ExpVgst / (1.0 + ExpVgst);
        dT10_dVb = T3 * dn_dVb - dT10_dVg * (dVth_dVb + Vgst * dn_dVb / n);
        dT10_dVd = T3 * dn_dVd - dT10_dVg * (dVth_dVd + Vgst * dn_dVd / n);
        dT10_dVg *= dVgs_eff_dVg;
      }
      T1 = P(voffcbncv) - (1.0 - mstarcv) * Vgst;
      T2 = T1 / T0;
      if (T2 < -CONSTEXP_THRESHOLD) {
        T3 = coxe * CONSTMIN_EXP / P(cdep0);
        T9 = mstarcv + T3 * n;
        dT9_dVg = 0.0;
        dT9_dVd = dn_dVd * T3;
        dT9_dVb = dn_dVb * T3;
      } else if (T2 > CONSTEXP_THRESHOLD) {
        T3 = coxe * CONSTMAX_EXP / P(cdep0);
        T9 = mstarcv + T3 * n;
        dT9_dVg = 0.0;
        dT9_dVd = dn_dVd * T3;
        dT9_dVb = dn_dVb * T3;
      } else {
        const double ExpVgst = exp(T2);
        T3 = coxe / P(cdep0);
        T4 = T3 * ExpVgst;
        T5 = T1 * T4 / T0;
        T9 = mstarcv + n * T4;
        dT9_dVg = T3 * (mstarcv - 1.0) * ExpVgst / Vtm;
        dT9_dVb = T4 * dn_dVb - dT9_dVg * dVth_dVb - T5 * dn_dVb;
        dT9_dVd = T4 * dn_dVd - dT9_dVg * dVth_dVd - T5 * dn_dVd;
        dT9_dVg *= dVgs_eff_dVg;
      }
      Vgsteff = T10 / T9;
      T11 = T9 * T9;
      dVgsteff_dVg = (T9 * dT10_dVg - T10 * dT9_dVg) / T11;
      dVgsteff_dVd = (T9 * dT10_dVd - T10 * dT9_dVd) / T11;
      dVgsteff_dVb = (T9 * dT10_dVb - T10 * dT9_dVb) / T11;
    }
    if (capMod == 1) {
      // capMod = 1 (:11139-11319): accumulation and depletion charges Qac0 / Qsub0 with the
      // zero-bias flat band, the inversion charge without the charge-thickness correction.
      const double Vfb1 = P(vfbzb);
      double V3 = Vfb1 - Vgs_eff + VbseffCV - CONSTDELTA_3;
      if (Vfb1 <= 0.0)
        T0 = sqrt(V3 * V3 - 4.0 * CONSTDELTA_3 * Vfb1);
      else
        T0 = sqrt(V3 * V3 + 4.0 * CONSTDELTA_3 * Vfb1);
      T1 = 0.5 * (1.0 + V3 / T0);
      const double Vfbeff = Vfb1 - 0.5 * (V3 + T0);
      const double dVfbeff_dVg = T1 * dVgs_eff_dVg;
      const double dVfbeff_dVb = -T1 * dVbseffCV_dVb;
      const double Qac0 = CoxWL * (Vfbeff - Vfb1);
      const double dQac0_dVg = CoxWL * dVfbeff_dVg;
      const double dQac0_dVb = CoxWL * dVfbeff_dVb;
      const double k1ox1 = P(k1ox);
      T0 = 0.5 * k1ox1;
      T3 = Vgs_eff - Vfbeff - VbseffCV - Vgsteff;
      if (k1ox1 == 0.0) {
        T1 = 0.0;
        T2 = 0.0;
      } else if (T3 < 0.0) {
        T1 = T0 + T3 / k1ox1;
        T2 = CoxWL;
      } else {
        T1 = sqrt(T0 * T0 + T3);
        T2 = CoxWL * T0 / T1;
      }
      const double Qsub0 = CoxWL * k1ox1 * (T1 - T0);
      const double dQsub0_dVg = T2 * (dVgs_eff_dVg - dVfbeff_dVg - dVgsteff_dVg);
      const double dQsub0_dVd = -T2 * dVgsteff_dVd;
      const double dQsub0_dVb = -T2 * (dVfbeff_dVb + dVbseffCV_dVb + dVgsteff_dVb);
      const double AbulkCV = Abulk0 * P(abulkCVfactor);
      const double dAbulkCV_dVb = P(abulkCVfactor) * dAbulk0_dVb;
      const double VdsatCV = Vgsteff / AbulkCV;
      T0 = VdsatCV - Vds - CONSTDELTA_4;
      dT0_dVg = 1.0 / AbulkCV;
      dT0_dVb = -VdsatCV * dAbulkCV_dVb / AbulkCV;
      T1 = sqrt(T0 * T0 + 4.0 * CONSTDELTA_4 * VdsatCV);
      dT1_dVg = (T0 + CONSTDELTA_4 + CONSTDELTA_4) / T1;
      dT1_dVd = -T0 / T1;
      dT1_dVb = dT1_dVg * dT0_dVb;
      dT1_dVg *= dT0_dVg;
      double VdseffCV, dVdseffCV_dVg, dVdseffCV_dVd, dVdseffCV_dVb;
      if (T0 >= 0.0) {
        VdseffCV = VdsatCV - 0.5 * (T0 + T1);
        dVdseffCV_dVg = 0.5 * (dT0_dVg - dT1_dVg);
        dVdseffCV_dVd = 0.5 * (1.0 - dT1_dVd);
        dVdseffCV_dVb = 0.5 * (dT0_dVb - dT1_dVb);
      } else {
        T3 = (CONSTDELTA_4 + CONSTDELTA_4) / (T1 - T0);
        T4 = 1.0 - T3;
        T5 = VdsatCV * T3 / (T1 - T0);
        VdseffCV = VdsatCV * T4;
        dVdseffCV_dVg = dT0_dVg * T4 + T5 * (dT1_dVg - dT0_dVg);
        dVdseffCV_dVd = T5 * (dT1_dVd + 1.0);
        dVdseffCV_dVb = dT0_dVb * (T4 - T5) + T5 * dT1_dVb;
      }
      if (Vds == 0.0) {  // the reference leaves dVdseffCV_dVd as computed
        VdseffCV = 0.0;
        dVdseffCV_dVg = 0.0;
        dVdseffCV_dVb = 0.0;
      }
      T0 = AbulkCV * VdseffCV;
      T1 = 12.0 * (Vgsteff - 0.5 * T0 + 1.0e-20);
      T2 = VdseffCV / T1;
      T3 = T0 * T2;
      T4 = (1.0 - 12.0 * T2 * T2 * AbulkCV);
      T5 = (6.0 * T0 * (4.0 * Vgsteff - T0) / (T1 * T1) - 0.5);
      T6 = 12.0 * T2 * T2 * Vgsteff;
      qgate = CoxWL * (Vgsteff - 0.5 * VdseffCV + T3);
      double Cgg1 = CoxWL * (T4 + T5 * dVdseffCV_dVg);
      const double Cgd1 = CoxWL * T5 * dVdseffCV_dVd + Cgg1 * dVgsteff_dVd;
      const double Cgb1 = CoxWL * (T5 * dVdseffCV_dVb + T6 * dAbulkCV_dVb) + Cgg1 * dVgsteff_dVb;
      Cgg1 *= dVgsteff_dVg;
      T7 = 1.0 - AbulkCV;
      qbulk = CoxWL * T7 * (0.5 * VdseffCV - T3);
      T4 = -T7 * (T4 - 1.0);
      T5 = -T7 * T5;
      T6 = -(T7 * T6 + (0.5 * VdseffCV - T3));
      double Cbg1 = CoxWL * (T4 + T5 * dVdseffCV_dVg);
      const double Cbd1 = CoxWL * T5 * dVdseffCV_dVd + Cbg1 * dVgsteff_dVd;
      const double Cbb1 = CoxWL * (T5 * dVdseffCV_dVb + T6 * dAbulkCV_dVb) + Cbg1 * dVgsteff_dVb;
      Cbg1 *= dVgsteff_dVg;
      double Csg, Csd, Csb;
      const double xpart = P(xpart);
      if (xpart > 0.5) {  // 0/100
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
      } else if (xpart < 0.5) {  // 40/60
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
      } else {  // 50/50
        qsrc = -0.5 * (qgate + qbulk);
        Csg = -0.5 * (Cgg1 + Cbg1);
        Csb = -0.5 * (Cgb1 + Cbb1);
        Csd = -0.5 * (Cgd1 + Cbd1);
      }
      qgate += Qac0 + Qsub0;
      qbulk -= (Qac0 + Qsub0);
      qdrn = -(qgate + qbulk + qsrc);
      const double Cgg = dQac0_dVg + dQsub0_dVg + Cgg1;
      const double Cgd = dQsub0_dVd + Cgd1;
      double Cgb = dQac0_dVb + dQsub0_dVb + Cgb1;
      const double Cbg = Cbg1 - dQac0_dVg - dQsub0_dVg;
      const double Cbd = Cbd1 - dQsub0_dVd;
      double Cbb = Cbb1 - dQac0_dVb - dQsub0_dVb;
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
    } else {
    // capMod == 2
    const double vfbzb = P(vfbzb);
    double V3 = vfbzb - Vgs_eff + VbseffCV - CONSTDELTA_3;
    if (vfbzb <= 0.0)
      T0 = sqrt(V3 * V3 - 4.0 * CONSTDELTA_3 * vfbzb);
    else
      T0 = sqrt(V3 * V3 + 4.0 * CONSTDELTA_3 * vfbzb);
    T1 = 0.5 * (1.0 + V3 / T0);
    const double Vfbeff = vfbzb - 0.5 * (V3 + T0);
    const double dVfbeff_dVg = T1 * dVgs_eff_dVg;
    const double dVfbeff_dVb = -T1 * dVbseffCV_dVb;
    const double Cox = coxp;
    double Tox = 1.0e8 * P(toxp);
    T0 = (Vgs_eff - VbseffCV - vfbzb) / Tox;
    dT0_dVg = dVgs_eff_dVg / Tox;
    dT0_dVb = -dVbseffCV_dVb / Tox;
    tmp = T0 * P(acde);
    const double ldeb = P(ldeb);
    double dTcen_dVb, dTcen_dVd;
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
    const double LINK = 1.0e-3 * P(toxp);
    V3 = ldeb - Tcen - LINK;
    const double V4 = sqrt(V3 * V3 + 4.0 * LINK * ldeb);
    Tcen = ldeb - 0.5 * (V3 + V4);
    T1 = 0.5 * (1.0 + V3 / V4);
    dTcen_dVg *= T1;
    dTcen_dVb *= T1;
    double Ccen = epssub / Tcen;
    T2 = Cox / (Cox + Ccen);
    Coxeff = T2 * Ccen;
    T3 = -Ccen / Tcen;
    dCoxeff_dVg = T2 * T2 * T3;
    double dCoxeff_dVb = dCoxeff_dVg * dTcen_dVb;
    dCoxeff_dVg *= dTcen_dVg;
    double CoxWLcen = CoxWL * Coxeff / coxe;
    const double Qac0 = CoxWLcen * (Vfbeff - vfbzb);
    double QovCox = Qac0 / Coxeff;
    const double dQac0_dVg = CoxWLcen * dVfbeff_dVg + QovCox * dCoxeff_dVg;
    const double dQac0_dVb = CoxWLcen * dVfbeff_dVb + QovCox * dCoxeff_dVb;
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
    const double Qsub0 = CoxWLcen * k1ox * (T1 - T0);
    QovCox = Qsub0 / Coxeff;
    const double dQsub0_dVg = T2 * (dVgs_eff_dVg - dVfbeff_dVg - dVgsteff_dVg) + QovCox * dCoxeff_dVg;
    const double dQsub0_dVd = -T2 * dVgsteff_dVd;
    const double dQsub0_dVb = -T2 * (dVfbeff_dVb + dVbseffCV_dVb + dVgsteff_dVb) + QovCox * dCoxeff_dVb;
    if (k1ox <= 0.0) {
      Denomi = 0.25 * P(moin) * Vtm;
      T0 = 0.5 * sqrtPhi_p;
    } else {
      Denomi = P(moin) * Vtm * k1ox * k1ox;
      T0 = k1ox * sqrtPhi_p;
    }
    T1 = 2.0 * T0 + Vgsteff;
    const double DeltaPhi = Vtm * log(1.0 + T1 * Vgsteff / Denomi);
    const double dDeltaPhi_dVg = 2.0 * Vtm * (T1 - T0) / (Denomi + T1 * Vgsteff);
    T0 = Vgsteff - DeltaPhi - 0.001;
    dT0_dVg = 1.0 - dDeltaPhi_dVg;
    T1 = sqrt(T0 * T0 + Vgsteff * 0.004);
    const double VgDP = 0.5 * (T0 + T1);
    const double dVgDP_dVg = 0.5 * (dT0_dVg + (T0 * dT0_dVg + 0.002) / T1);
    Tox += Tox;
    T0 = (Vgsteff + P(vtfbphi2)) / Tox;
    tmp = exp(P(bdos) * 0.7 * log(T0));
    T1 = 1.0 + tmp;
    T2 = P(bdos) * 0.7 * tmp / (T0 * Tox);
    Tcen = P(ados) * 1.9e-9 / T1;
    dTcen_dVg = -Tcen * T2 / T1;
    dTcen_dVd = dTcen_dVg * dVgsteff_dVd;
    dTcen_dVb = dTcen_dVg * dVgsteff_dVb;
    dTcen_dVg *= dVgsteff_dVg;
    Ccen = epssub / Tcen;
    T0 = Cox / (Cox + Ccen);
    Coxeff = T0 * Ccen;
    T1 = -Ccen / Tcen;
    dCoxeff_dVg = T0 * T0 * T1;
    const double dCoxeff_dVd = dCoxeff_dVg * dTcen_dVd;
    dCoxeff_dVb = dCoxeff_dVg * dTcen_dVb;
    dCoxeff_dVg *= dTcen_dVg;
    CoxWLcen = CoxWL * Coxeff / coxe;
    const double AbulkCV = Abulk0 * P(abulkCVfactor);
    const double dAbulkCV_dVb = P(abulkCVfactor) * dAbulk0_dVb;
    const double VdsatCV = VgDP / AbulkCV;
    T0 = VdsatCV - Vds - CONSTDELTA_4;
    dT0_dVg = dVgDP_dVg / AbulkCV;
    dT0_dVb = -VdsatCV * dAbulkCV_dVb / AbulkCV;
    T1 = sqrt(T0 * T0 + 4.0 * CONSTDELTA_4 * VdsatCV);
    dT1_dVg = (T0 + CONSTDELTA_4 + CONSTDELTA_4) / T1;
    dT1_dVd = -T0 / T1;
    dT1_dVb = dT1_dVg * dT0_dVb;
    dT1_dVg *= dT0_dVg;
    double VdseffCV, dVdseffCV_dVg, dVdseffCV_dVd, dVdseffCV_dVb;
    if (T0 >= 0.0) {
      VdseffCV = VdsatCV - 0.5 * (T0 + T1);
      dVdseffCV_dVg = 0.5 * (dT0_dVg - dT1_dVg);
      dVdseffCV_dVd = 0.5 * (1.0 - dT1_dVd);
      dVdseffCV_dVb = 0.5 * (dT0_dVb - dT1_dVb);
    } else {
      T3 = (CONSTDELTA_4 + CONSTDELTA_4) / (T1 - T0);
      T4 = 1.0 - T3;
      T5 = VdsatCV * T3 / (T1 - T0);
      VdseffCV = VdsatCV * T4;
      dVdseffCV_dVg = dT0_dVg * T4 + T5 * (dT1_dVg - dT0_dVg);
      dVdseffCV_dVd = T5 * (dT1_dVd + 1.0);
      dVdseffCV_dVb = dT0_dVb * (T4 - T5) + T5 * dT1_dVb;
    }
    if (Vds == 0.0) {
      VdseffCV = 0.0;
      dVdseffCV_dVg = 0.0;
      dVdseffCV_dVb = 0.0;
    }
    T0 = AbulkCV * VdseffCV;
    T1 = VgDP;
    T2 = 12.0 * (T1 - 0.5 * T0 + 1.0e-20);
    T3 = T0 / T2;
    T4 = 1.0 - 12.0 * T3 * T3;
    T5 = AbulkCV * (6.0 * T0 * (4.0 * T1 - T0) / (T2 * T2) - 0.5);
    T6 = T5 * VdseffCV / AbulkCV;
    qgate = CoxWLcen * (T1 - T0 * (0.5 - T3));
    QovCox = qgate / Coxeff;
    double Cgg1 = CoxWLcen * (T4 * dVgDP_dVg + T5 * dVdseffCV_dVg);
    const double Cgd1 = CoxWLcen * T5 * dVdseffCV_dVd + Cgg1 * dVgsteff_dVd + QovCox * dCoxeff_dVd;
    const double Cgb1 = CoxWLcen * (T5 * dVdseffCV_dVb + T6 * dAbulkCV_dVb) + Cgg1 * dVgsteff_dVb + QovCox * dCoxeff_dVb;
    Cgg1 = Cgg1 * dVgsteff_dVg + QovCox * dCoxeff_dVg;
    T7 = 1.0 - AbulkCV;
    T8 = T2 * T2;
    T9 = 12.0 * T7 * T0 * T0 / (T8 * AbulkCV);
    T10 = T9 * dVgDP_dVg;
    T11 = -T7 * T5 / AbulkCV;
    T12 = -(T9 * T1 / AbulkCV + VdseffCV * (0.5 - T0 / T2));
    qbulk = CoxWLcen * T7 * (0.5 * VdseffCV - T0 * VdseffCV / T2);
    QovCox = qbulk / Coxeff;
    double Cbg1 = CoxWLcen * (T10 + T11 * dVdseffCV_dVg);
    const double Cbd1 = CoxWLcen * T11 * dVdseffCV_dVd + Cbg1 * dVgsteff_dVd + QovCox * dCoxeff_dVd;
    const double Cbb1 = CoxWLcen * (T11 * dVdseffCV_dVb + T12 * dAbulkCV_dVb) + Cbg1 * dVgsteff_dVb + QovCox * dCoxeff_dVb;
    Cbg1 = Cbg1 * dVgsteff_dVg + QovCox * dCoxeff_dVg;
    double Csg, Csd, Csb;
    const double xpart = P(xpart);
    if (xpart > 0.5) {
      qsrc = -CoxWLcen * (T1 / 2.0 + T0 / 4.0 - 0.5 * T0 * T0 / T2);
      QovCox = qsrc / Coxeff;
      T2 += T2;
      T3 = T2 * T2;
      T7 = -(0.25 - 12.0 * T0 * (4.0 * T1 - T0) / T3);
      T4 = -(0.5 + 24.0 * T0 * T0 / T3) * dVgDP_dVg;
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
      Csg = T5 * dVgDP_dVg + T6 * dVdseffCV_dVg;
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
    const double Cbg = Cbg1 - dQac0_dVg - dQsub0_dVg;
    const double Cbd = Cbd1 - dQsub0_dVd;
    double Cbb = Cbb1 - dQac0_dVb - dQsub0_dVb;
    const double Cgg = Cgg1 - Cbg;
    const double Cgd = Cgd1 - Cbd;
    double Cgb = Cgb1 - Cbb;
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
  }

  // NQS (:11626-11637): the channel charge the charge node carries, its capacitances and the
  // relaxation conductance gtau = gcrg / (Cox W L) x 1e-9 (from the DC part's unscaled gcrg).
  const bool trnqsMod = GEN && P(trnqsMod) != 0.0;
  constexpr double ScalingFactor = 1.0e-9;
  const double qdef = bias.qdef;
  double qchqs = 0.0, cqgb = 0.0, cqdb = 0.0, cqsb = 0.0, cqbb = 0.0, gtau = 0.0, CoxWL = 0.0;
  if (trnqsMod) {
    qchqs = -(qbulk + qgate);
    cqgb = -(cggb + cbgb);
    cqdb = -(cgdb + cbdb);
    cqsb = -(cgsb + cbsb);
    cqbb = -(cqgb + cqdb + cqsb);
    CoxWL = P(coxe) * P(weffCV) * nf * P(leffCV);
    gtau = m.v[m_gcrg] / CoxWL * ScalingFactor;
  }
  double qcheq = qchqs;

  // Junction charges and capacitances (:11661-11810). Outside charge computation the reference
  // keeps the previous load's junction values; they only feed Q and dQ/dx, which a DC solve does
  // not use, and are zero here.
  double qbs = 0.0, qbd = 0.0, capbs = 0.0, capbd = 0.0;
  if (ChargeComputationNeeded) {
    const double czbd = P(DunitAreaTempJctCap) * Adeff;
    const double czbs = P(SunitAreaTempJctCap) * Aseff;
    const double czbdsw = P(DunitLengthSidewallTempJctCap) * Pdeff;
    const double czbdswg = P(DunitLengthGateSidewallTempJctCap) * weffCJ * nf;
    const double czbssw = P(SunitLengthSidewallTempJctCap) * Pseff;
    const double czbsswg = P(SunitLengthGateSidewallTempJctCap) * weffCJ * nf;
    const double MJS = P(SbulkJctBotGradingCoeff), MJSWS = P(SbulkJctSideGradingCoeff);
    const double MJSWGS = P(SbulkJctGateSideGradingCoeff);
    const double MJD = P(DbulkJctBotGradingCoeff), MJSWD = P(DbulkJctSideGradingCoeff);
    const double MJSWGD = P(DbulkJctGateSideGradingCoeff);
    double arg, sarg;
    if (vbs_jct == 0.0) {
      qbs = 0.0;
      capbs = czbs + czbssw + czbsswg;
    } else if (vbs_jct < 0.0) {
      if (czbs > 0.0) {
        arg = 1.0 - vbs_jct / P(PhiBS);
        if (MJS == 0.5)
          sarg = 1.0 / sqrt(arg);
        else
          sarg = exp(-MJS * log(arg));
        qbs = P(PhiBS) * czbs * (1.0 - arg * sarg) / (1.0 - MJS);
        capbs = czbs * sarg;
      } else {
        qbs = 0.0;
        capbs = 0.0;
      }
      if (czbssw > 0.0) {
        arg = 1.0 - vbs_jct / P(PhiBSWS);
        if (MJSWS == 0.5)
          sarg = 1.0 / sqrt(arg);
        else
          sarg = exp(-MJSWS * log(arg));
        qbs += P(PhiBSWS) * czbssw * (1.0 - arg * sarg) / (1.0 - MJSWS);
        capbs += czbssw * sarg;
      }
      if (czbsswg > 0.0) {
        arg = 1.0 - vbs_jct / P(PhiBSWGS);
        if (MJSWGS == 0.5)
          sarg = 1.0 / sqrt(arg);
        else
          sarg = exp(-MJSWGS * log(arg));
        qbs += P(PhiBSWGS) * czbsswg * (1.0 - arg * sarg) / (1.0 - MJSWGS);
        capbs += czbsswg * sarg;
      }
    } else {
      T0 = czbs + czbssw + czbsswg;
      T1 = vbs_jct * (czbs * MJS / P(PhiBS) + czbssw * MJSWS / P(PhiBSWS) + czbsswg * MJSWGS / P(PhiBSWGS));
      qbs = vbs_jct * (T0 + 0.5 * T1);
      capbs = T0 + T1;
    }
    if (vbd_jct == 0.0) {
      qbd = 0.0;
      capbd = czbd + czbdsw + czbdswg;
    } else if (vbd_jct < 0.0) {
      if (czbd > 0.0) {
        arg = 1.0 - vbd_jct / P(PhiBD);
        if (MJD == 0.5)
          sarg = 1.0 / sqrt(arg);
        else
          sarg = exp(-MJD * log(arg));
        qbd = P(PhiBD) * czbd * (1.0 - arg * sarg) / (1.0 - MJD);
        capbd = czbd * sarg;
      } else {
        qbd = 0.0;
        capbd = 0.0;
      }
      if (czbdsw > 0.0) {
        arg = 1.0 - vbd_jct / P(PhiBSWD);
        if (MJSWD == 0.5)
          sarg = 1.0 / sqrt(arg);
        else
          sarg = exp(-MJSWD * log(arg));
        qbd += P(PhiBSWD) * czbdsw * (1.0 - arg * sarg) / (1.0 - MJSWD);
        capbd += czbdsw * sarg;
      }
      if (czbdswg > 0.0) {
        arg = 1.0 - vbd_jct / P(PhiBSWGD);
        if (MJSWGD == 0.5)
          sarg = 1.0 / sqrt(arg);
        else
          sarg = exp(-MJSWGD * log(arg));
        qbd += P(PhiBSWGD) * czbdswg * (1.0 - arg * sarg) / (1.0 - MJSWGD);
        capbd += czbdswg * sarg;
      }
    } else {
      T0 = czbd + czbdsw + czbdswg;
      T1 = vbd_jct * (czbd * MJD / P(PhiBD) + czbdsw * MJSWD / P(PhiBSWD) + czbdswg * MJSWGD / P(PhiBSWGD));
      qbd = vbd_jct * (T0 + 0.5 * T1);
      capbd = T0 + T1;
    }
  }

  // Overlap capacitances (:11812-11890): constant for capMod 0, bias-dependent for 1 and 2; with
  // rgateMod 3 they sit between the gate-mid node and the drain / source.
  const double vgdx = (rgateMod == 3) ? vgmd : vgd, vgsx = (rgateMod == 3) ? vgms : vgs;
  // Gate resistor currents (:11824-11844).
  double Igate = 0.0, IgateMid = 0.0;
  if (GEN) {
    if (rgateMod == 1) {
      Igate = P(grgeltd) * (bias.Vgegp);
    } else if (rgateMod == 2) {
      Igate = (m.v[m_gcrg]) * (bias.Vgegp);
    } else if (rgateMod == 3) {
      Igate = P(grgeltd) * (bias.Vgegm);
      IgateMid = m.v[m_gcrg] * (bias.Vgmgp);
    }
  }
  double cgdo, qgdo, cgso, qgso;
  if (capMod == 0) {
    cgdo = P(cgdo);
    qgdo = P(cgdo) * vgdx;
    cgso = P(cgso);
    qgso = P(cgso) * vgsx;
  } else {
    T0 = vgdx + CONSTDELTA_1;
    T1 = sqrt(T0 * T0 + 4.0 * CONSTDELTA_1);
    T2 = 0.5 * (T0 - T1);
    T3 = P(weffCV) * P(cgdl);
    T4 = sqrt(1.0 - 4.0 * T2 / P(ckappad));
    cgdo = P(cgdo) + T3 - T3 * (1.0 - 1.0 / T4) * (0.5 - 0.5 * T0 / T1);
    qgdo = (P(cgdo) + T3) * vgdx - T3 * (T2 + 0.5 * P(ckappad) * (T4 - 1.0));
    T0 = vgsx + CONSTDELTA_1;
    T1 = sqrt(T0 * T0 + 4.0 * CONSTDELTA_1);
    T2 = 0.5 * (T0 - T1);
    T3 = P(weffCV) * P(cgsl);
    T4 = sqrt(1.0 - 4.0 * T2 / P(ckappas));
    cgso = P(cgso) + T3 - T3 * (1.0 - 1.0 / T4) * (0.5 - 0.5 * T0 / T1);
    qgso = (P(cgso) + T3) * vgsx - T3 * (T2 + 0.5 * P(ckappas) * (T4 - 1.0));
  }
  if (nf != 1.0) {
    cgdo *= nf;
    cgso *= nf;
    qgdo *= nf;
    qgso *= nf;
  }

  // Overlap and gate-bulk charge bookkeeping and the charge partition (setupCapacitors_oldDAE,
  // :12616-13045). With NQS the intrinsic charge is the charge node's: the terminal charges keep
  // only the overlap and gate-bulk parts, and the partition dxpart / sxpart follows qdrn / qcheq.
  const double cgbo = P(cgbo);
  double dxpart, sxpart;
  double ddxpart_dVd = 0.0, ddxpart_dVg = 0.0, ddxpart_dVb = 0.0, ddxpart_dVs = 0.0;
  double dsxpart_dVd = 0.0, dsxpart_dVg = 0.0, dsxpart_dVb = 0.0, dsxpart_dVs = 0.0;
  double ggtg = 0.0, ggtd = 0.0, ggts = 0.0, ggtb = 0.0, gqdef = 0.0;
  double qgmid = 0.0;  // rgateMod 3: the overlap and gate-bulk charge on the gate-mid node
  // The integration coefficient of the old DAE form; zero on the first Newton step out of the
  // operating point (:12618-12629).
  const double ag0 = (!fl.dcop && fl.init_tran && fl.newton_iter == 0) ? 0.0 : fl.pdt;
  if (trnqsMod) {
    qcheq = qchqs;
    const double T0q = qdef * ScalingFactor / CoxWL;
    const double gcg = m.v[m_gcrgg], gcd = m.v[m_gcrgd], gcs = m.v[m_gcrgs], gcb = m.v[m_gcrgb];
    ggtg = T0q * gcg;
    ggtd = T0q * (mode > 0 ? gcd : gcs);
    ggts = T0q * (mode > 0 ? gcs : gcd);
    ggtb = T0q * gcb;
    gqdef = ScalingFactor * ag0;
    const double xpart = P(xpart);
    if (mode > 0) {
      if (fabs(qcheq) <= 1.0e-5 * CoxWL) {
        dxpart = (xpart < 0.5) ? 0.4 : (xpart > 0.5) ? 0.0 : 0.5;
      } else {
        dxpart = qdrn / qcheq;
        const double Cdd = cddb, Csd = -(cgdb + cddb + cbdb);
        ddxpart_dVd = (Cdd - dxpart * (Cdd + Csd)) / qcheq;
        const double Cdg = cdgb, Csg = -(cggb + cdgb + cbgb);
        ddxpart_dVg = (Cdg - dxpart * (Cdg + Csg)) / qcheq;
        const double Cds = cdsb, Css = -(cgsb + cdsb + cbsb);
        ddxpart_dVs = (Cds - dxpart * (Cds + Css)) / qcheq;
        ddxpart_dVb = -(ddxpart_dVd + ddxpart_dVg + ddxpart_dVs);
      }
      sxpart = 1.0 - dxpart;
      dsxpart_dVd = -ddxpart_dVd;
      dsxpart_dVg = -ddxpart_dVg;
      dsxpart_dVs = -ddxpart_dVs;
      dsxpart_dVb = -(dsxpart_dVd + dsxpart_dVg + dsxpart_dVs);
    } else {
      if (fabs(qcheq) <= 1.0e-5 * CoxWL) {
        sxpart = (xpart < 0.5) ? 0.4 : (xpart > 0.5) ? 0.0 : 0.5;
      } else {
        sxpart = qdrn / qcheq;
        const double Css = cddb, Cds = -(cgdb + cddb + cbdb);
        dsxpart_dVs = (Css - sxpart * (Css + Cds)) / qcheq;
        const double Csg = cdgb, Cdg = -(cggb + cdgb + cbgb);
        dsxpart_dVg = (Csg - sxpart * (Csg + Cdg)) / qcheq;
        const double Csd = cdsb, Cdd = -(cgsb + cdsb + cbsb);
        dsxpart_dVd = (Csd - sxpart * (Csd + Cdd)) / qcheq;
        dsxpart_dVb = -(dsxpart_dVd + dsxpart_dVg + dsxpart_dVs);
      }
      dxpart = 1.0 - sxpart;
      ddxpart_dVd = -dsxpart_dVd;
      ddxpart_dVg = -dsxpart_dVg;
      ddxpart_dVs = -dsxpart_dVs;
      ddxpart_dVb = -(ddxpart_dVd + ddxpart_dVg + ddxpart_dVs);
    }
    if (rgateMod == 3) {
      const double qgmb = cgbo * vgmb;
      qgmid = qgdo + qgso + qgmb;
      qgate = 0.0;
      qbulk = -qgmb;
      qdrn = -qgdo;
      qsrc = (mode > 0) ? -(qgmid + qbulk + qdrn) : -qgso;
    } else {
      const double qgb = cgbo * vgb;
      qgate = qgdo + qgso + qgb;
      qbulk = -qgb;
      qdrn = -qgdo;
      qsrc = (mode > 0) ? -(qgate + qbulk + qdrn) : -qgso;
    }
  } else if (mode > 0) {
    qdrn -= qgdo;
    if (rgateMod == 3) {
      const double qgmb = cgbo * vgmb;
      qgmid = qgdo + qgso + qgmb;
      qbulk -= qgmb;
      qsrc = -(qgate + qgmid + qbulk + qdrn);
    } else {
      const double qgb = cgbo * vgb;
      qgate += qgdo + qgso + qgb;
      qbulk -= qgb;
      qsrc = -(qgate + qbulk + qdrn);
    }
    sxpart = 0.6;
    dxpart = 0.4;
  } else {
    qsrc = qdrn - qgso;
    if (rgateMod == 3) {
      const double qgmb = cgbo * vgmb;
      qgmid = qgdo + qgso + qgmb;
      qbulk -= qgmb;
      qdrn = -(qgate + qgmid + qbulk + qsrc);
    } else {
      const double qgb = cgbo * vgb;
      qgate += qgdo + qgso + qgb;
      qbulk -= qgb;
      qdrn = -(qgate + qbulk + qsrc);
    }
    sxpart = 0.4;
    dxpart = 0.6;
  }
  (void)qsrc; (void)ag0;

  // Capacitance matrix entries (setupCapacitors_newDAE, :12357-12608).
  double CAPcggb, CAPcgdb, CAPcgsb, CAPcgbb, CAPcdgb, CAPcsgb, CAPcbgb, CAPcddb, CAPcdsb, CAPcsdb, CAPcssb;
  double CAPcdbb, CAPcsbb, CAPcbdb, CAPcbsb, CAPcbbb;
  double CAPcdgmb = 0.0, CAPcsgmb = 0.0, CAPcbgmb = 0.0;
  double CAPcgmgmb = 0.0, CAPcgmdb = 0.0, CAPcgmsb = 0.0, CAPcgmbb = 0.0, CAPcdbdb = 0.0, CAPcsbsb = 0.0;
  double CAPcqgb = 0.0, CAPcqdb = 0.0, CAPcqsb = 0.0, CAPcqbb = 0.0;
  if (trnqsMod) {
    // NQS: the intrinsic capacitances sit on the charge node's row; the terminals keep the overlap
    // and junction parts (the trnqsMod != 0 branches of :12423-12480 and :12543-12600).
    CAPcqgb = cqgb;
    CAPcqdb = (mode > 0) ? cqdb : cqsb;
    CAPcqsb = (mode > 0) ? cqsb : cqdb;
    CAPcqbb = cqbb;
    if (rgateMod == 3) {
      CAPcgmgmb = (cgdo + cgso + cgbo);
      CAPcgmdb = -cgdo;
      CAPcgmsb = -cgso;
      CAPcgmbb = -cgbo;
      CAPcdgmb = CAPcgmdb;
      CAPcsgmb = CAPcgmsb;
      CAPcbgmb = CAPcgmbb;
      CAPcdgb = CAPcsgb = CAPcbgb = 0.0;
      CAPcggb = CAPcgdb = CAPcgsb = CAPcgbb = 0.0;
    } else {
      CAPcggb = (cgdo + cgso + cgbo);
      CAPcgdb = -cgdo;
      CAPcgsb = -cgso;
      CAPcgbb = -cgbo;
      CAPcdgb = CAPcgdb;
      CAPcsgb = CAPcgsb;
      CAPcbgb = CAPcgbb;
      CAPcdgmb = CAPcsgmb = CAPcbgmb = 0.0;
    }
    CAPcddb = (capbd + cgdo);
    CAPcdsb = CAPcsdb = 0.0;
    CAPcssb = (capbs + cgso);
    if (!rbodyMod) {
      CAPcdbb = -(CAPcdgb + CAPcddb + CAPcdgmb);
      CAPcsbb = -(CAPcsgb + CAPcssb + CAPcsgmb);
      CAPcbdb = -capbd;
      CAPcbsb = -capbs;
      CAPcdbdb = 0.0;
      CAPcsbsb = 0.0;
    } else {
      CAPcdbb = CAPcsbb = CAPcbdb = CAPcbsb = 0.0;
      CAPcdbdb = -capbd;
      CAPcsbsb = -capbs;
    }
    CAPcbbb = -(CAPcbdb + CAPcbgb + CAPcbsb + CAPcbgmb);
  } else if (GEN) {
    if (mode > 0) {
      if (rgateMod == 3) {
        CAPcgmgmb = (cgdo + cgso + cgbo);
        CAPcgmdb = -cgdo;
        CAPcgmsb = -cgso;
        CAPcgmbb = -cgbo;
        CAPcdgmb = CAPcgmdb;
        CAPcsgmb = CAPcgmsb;
        CAPcbgmb = CAPcgmbb;
        CAPcggb = cggb;
        CAPcgdb = cgdb;
        CAPcgsb = cgsb;
        CAPcgbb = -(CAPcggb + CAPcgdb + CAPcgsb);
        CAPcdgb = cdgb;
        CAPcsgb = -(cggb + cbgb + cdgb);
        CAPcbgb = cbgb;
      } else {
        CAPcggb = (cggb + cgdo + cgso + cgbo);
        CAPcgdb = (cgdb - cgdo);
        CAPcgsb = (cgsb - cgso);
        CAPcgbb = -(CAPcggb + CAPcgdb + CAPcgsb);
        CAPcdgb = (cdgb - cgdo);
        CAPcsgb = -(cggb + cbgb + cdgb + cgso);
        CAPcbgb = (cbgb - cgbo);
        CAPcdgmb = CAPcsgmb = CAPcbgmb = 0.0;
      }
      CAPcddb = (cddb + capbd + cgdo);
      CAPcdsb = cdsb;
      CAPcsdb = -(cgdb + cbdb + cddb);
      CAPcssb = (capbs + cgso - (cgsb + cbsb + cdsb));
      if (!rbodyMod) {
        CAPcdbb = -(CAPcdgb + CAPcddb + CAPcdsb + CAPcdgmb);
        CAPcsbb = -(CAPcsgb + CAPcsdb + CAPcssb + CAPcsgmb);
        CAPcbdb = (cbdb - capbd);
        CAPcbsb = (cbsb - capbs);
        CAPcdbdb = 0.0;
        CAPcsbsb = 0.0;
      } else {
        CAPcdbb = -(cddb + cdgb + cdsb);
        CAPcsbb = -(CAPcsgb + CAPcsdb + CAPcssb + CAPcsgmb) + capbs;
        CAPcbdb = cbdb;
        CAPcbsb = cbsb;
        CAPcdbdb = -capbd;
        CAPcsbsb = -capbs;
      }
      CAPcbbb = -(CAPcbdb + CAPcbgb + CAPcbsb + CAPcbgmb);
    } else {
      if (rgateMod == 3) {
        CAPcgmgmb = (cgdo + cgso + cgbo);
        CAPcgmdb = -cgdo;
        CAPcgmsb = -cgso;
        CAPcgmbb = -cgbo;
        CAPcdgmb = CAPcgmdb;
        CAPcsgmb = CAPcgmsb;
        CAPcbgmb = CAPcgmbb;
        CAPcggb = cggb;
        CAPcgdb = cgsb;
        CAPcgsb = cgdb;
        CAPcgbb = -(CAPcggb + CAPcgdb + CAPcgsb);
        CAPcdgb = -(cggb + cbgb + cdgb);
        CAPcsgb = cdgb;
        CAPcbgb = cbgb;
      } else {
        CAPcggb = (cggb + cgdo + cgso + cgbo);
        CAPcgdb = (cgsb - cgdo);
        CAPcgsb = (cgdb - cgso);
        CAPcgbb = -(CAPcggb + CAPcgdb + CAPcgsb);
        CAPcdgb = -(cggb + cbgb + cdgb + cgdo);
        CAPcsgb = (cdgb - cgso);
        CAPcbgb = (cbgb - cgbo);
        CAPcdgmb = CAPcsgmb = CAPcbgmb = 0.0;
      }
      CAPcddb = (capbd + cgdo - (cgsb + cbsb + cdsb));
      CAPcdsb = -(cgdb + cbdb + cddb);
      CAPcsdb = cdsb;
      CAPcssb = (cddb + capbs + cgso);
      if (!rbodyMod) {
        CAPcdbb = -(CAPcdgb + CAPcddb + CAPcdsb + CAPcdgmb);
        CAPcsbb = -(CAPcsgb + CAPcsdb + CAPcssb + CAPcsgmb);
        CAPcbdb = (cbsb - capbd);
        CAPcbsb = (cbdb - capbs);
        CAPcdbdb = 0.0;
        CAPcsbsb = 0.0;
      } else {
        CAPcdbb = -(CAPcdgb + CAPcddb + CAPcdsb + CAPcdgmb) + capbd;
        CAPcsbb = -(cddb + cdgb + cdsb);
        CAPcbdb = cbsb;
        CAPcbsb = cbdb;
        CAPcdbdb = -capbd;
        CAPcsbsb = -capbs;
      }
      CAPcbbb = -(CAPcbgb + CAPcbdb + CAPcbsb + CAPcbgmb);
    }
  } else if (mode > 0) {
    CAPcggb = (cggb + cgdo + cgso + cgbo);
    CAPcgdb = (cgdb - cgdo);
    CAPcgsb = (cgsb - cgso);
    CAPcgbb = -(CAPcggb + CAPcgdb + CAPcgsb);
    CAPcdgb = (cdgb - cgdo);
    CAPcsgb = -(cggb + cbgb + cdgb + cgso);
    CAPcbgb = (cbgb - cgbo);
    CAPcddb = (cddb + capbd + cgdo);
    CAPcdsb = cdsb;
    CAPcsdb = -(cgdb + cbdb + cddb);
    CAPcssb = (capbs + cgso - (cgsb + cbsb + cdsb));
    CAPcdbb = -(CAPcdgb + CAPcddb + CAPcdsb + CAPcdgmb);
    CAPcsbb = -(CAPcsgb + CAPcsdb + CAPcssb + CAPcsgmb);
    CAPcbdb = (cbdb - capbd);
    CAPcbsb = (cbsb - capbs);
    CAPcbbb = -(CAPcbdb + CAPcbgb + CAPcbsb + CAPcbgmb);
  } else {
    CAPcggb = (cggb + cgdo + cgso + cgbo);
    CAPcgdb = (cgsb - cgdo);
    CAPcgsb = (cgdb - cgso);
    CAPcgbb = -(CAPcggb + CAPcgdb + CAPcgsb);
    CAPcdgb = -(cggb + cbgb + cdgb + cgdo);
    CAPcsgb = (cdgb - cgso);
    CAPcbgb = (cbgb - cgbo);
    CAPcddb = (capbd + cgdo - (cgsb + cbsb + cdsb));
    CAPcdsb = -(cgdb + cbdb + cddb);
    CAPcsdb = cdsb;
    CAPcssb = (cddb + capbs + cgso);
    CAPcdbb = -(CAPcdgb + CAPcddb + CAPcdsb + CAPcdgmb);
    CAPcsbb = -(CAPcsgb + CAPcsdb + CAPcssb + CAPcsgmb);
    CAPcbdb = (cbsb - capbd);
    CAPcbsb = (cbdb - capbs);
    CAPcbbb = -(CAPcbgb + CAPcbdb + CAPcbsb + CAPcbgmb);
  }

  // Master::updateState: store and state (:16195-16242).
  o.sto[s_vbd] = vbd;
  o.sto[s_vbs] = vbs;
  o.sto[s_vgs] = vgs;
  o.sto[s_vds] = vds;
  o.sto[s_vges] = vges;
  o.sto[s_vgms] = vgms;
  o.sto[s_vdes] = vdes;
  o.sto[s_vses] = vses;
  o.sto[s_vdbs] = vdbs;
  o.sto[s_vsbs] = vsbs;
  o.sto[s_vdbd] = vdbd;
  o.sto[s_vged] = 0.0;
  o.sto[s_vgmd] = 0.0;
  o.sto[s_von] = von;
  const double qg = qgate;
  const double qd = qdrn - qbd;
  const double qb = (!rbodyMod) ? qbulk + qbd + qbs : qbulk;
  o.sta[t_qg] = qg;
  o.sta[t_qd] = qd;
  o.sta[t_qb] = qb;
  if (GEN) {
    o.gsta[gt_qb] = qb;
    o.gsta[gt_qg] = qg;
    o.gsta[gt_qd] = qd;
    o.gsta[gt_qgmid] = (rgateMod == 3) ? qgmid : 0.0;
    o.gsta[gt_qbs] = rbodyMod ? qbs : 0.0;
    o.gsta[gt_qbd] = rbodyMod ? qbd : 0.0;
    o.gsta[gt_qcheq] = trnqsMod ? qcheq : 0.0;
    o.gsta[gt_qcdump] = trnqsMod ? qdef * ScalingFactor : 0.0;
  }
  o.write_curr_sta = (!fl.dcop) && fl.init_tran && fl.newton_iter == 0;
  o.vgb = vgb;

  // setupFVectorVars (:13525-13855).
  const double gjbd = gbd, gjbs = gbs;
  double Gmv, Gmbsv, FwdSum, RevSum, ceqdrn, ceqdrn_Jdxp, ceqbd, ceqbd_Jdxp, ceqbs, ceqbs_Jdxp;
  double gbbdp, gbbsp, gbdpg, gbdpdp, gbdpb, gbdpsp, gbspg, gbspdp, gbspb, gbspsp;
  if (mode >= 0) {
    Gmv = gm;
    Gmbsv = gmbs;
    FwdSum = Gmv + Gmbsv;
    RevSum = 0.0;
    ceqdrn = dtype * cdrain;
    ceqdrn_Jdxp = dtype * (-gds * (vds - vds_orig) - Gmv * (vgs - vgs_orig) - Gmbsv * (vbs - vbs_orig));
    ceqbd = dtype * (csub + Igidl);
    ceqbd_Jdxp = dtype * (-(gbds + ggidld) * (vds - vds_orig) - (gbgs + ggidlg) * (vgs - vgs_orig) -
                          (gbbs + ggidlb) * (vbs - vbs_orig));
    ceqbs = dtype * Igisl;
    ceqbs_Jdxp = dtype * (+ggisls * (vds - vds_orig) - ggislg * (vgd - vgd_orig) - ggislb * (vbd - vbd_orig));
    gbbdp = -(gbds);
    gbbsp = gbds + gbgs + gbbs;
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
    Gmbsv = -gmbs;
    FwdSum = 0.0;
    RevSum = -(Gmv + Gmbsv);
    ceqdrn = -dtype * cdrain;
    ceqdrn_Jdxp = -dtype * (+gds * (vds - vds_orig) + Gmv * (vgd - vgd_orig) + Gmbsv * (vbd - vbd_orig));
    ceqbs = dtype * (csub + Igisl);
    ceqbs_Jdxp = dtype * (+(gbds + ggisls) * (vds - vds_orig) - (gbgs + ggislg) * (vgd - vgd_orig) -
                          (gbbs + ggislb) * (vbd - vbd_orig));
    ceqbd = dtype * Igidl;
    ceqbd_Jdxp = dtype * (-ggidld * (vds - vds_orig) - ggidlg * (vgs - vgs_orig) - ggidlb * (vbs - vbs_orig));
    gbbsp = -(gbds);
    gbbdp = gbds + gbgs + gbbs;
    gbdpg = 0.0;
    gbdpsp = 0.0;
    gbdpb = 0.0;
    gbdpdp = 0.0;
    gbspg = gbgs;
    gbspsp = gbds;
    gbspb = gbbs;
    gbspdp = -(gbspg + gbspsp + gbspb);
  }
  // Gate-current totals (:13112-13170, mode >= 0; :13243-13300, mode < 0).
  double ceqgcrg = 0.0, ceqgcrg_Jdxp = 0.0;
  double Istoteq = 0.0, Idtoteq = 0.0, Ibtoteq = 0.0, Igtoteq = 0.0;
  double Istoteq_Jdxp = 0.0, Idtoteq_Jdxp = 0.0, Ibtoteq_Jdxp = 0.0, Igtoteq_Jdxp = 0.0;
  double gIstotg = 0.0, gIstotd = 0.0, gIstots = 0.0, gIstotb = 0.0;
  double gIdtotg = 0.0, gIdtotd = 0.0, gIdtots = 0.0, gIdtotb = 0.0;
  double gIbtotg = 0.0, gIbtotd = 0.0, gIbtots = 0.0, gIbtotb = 0.0;
  double gIgtotg = 0.0, gIgtotd = 0.0, gIgtots = 0.0, gIgtotb = 0.0;
  if (mode >= 0) {
    if (igcMod) {
      gIstotg = gIgsg + gIgcsg;
      gIstotd = gIgcsd;
      gIstots = gIgss + gIgcss;
      gIstotb = gIgcsb;
      Istoteq = dtype * (Igs + Igcs);
      Istoteq_Jdxp = dtype * (-gIstotg * (vgs - vgs_orig) - gIgcsd * (vds - vds_orig) - gIgcsb * (vbs - vbs_orig));
      gIdtotg = gIgdg + gIgcdg;
      gIdtotd = gIgdd + gIgcdd;
      gIdtots = gIgcds;
      gIdtotb = gIgcdb;
      Idtoteq = dtype * (Igd + Igcd);
      Idtoteq_Jdxp = dtype * (-gIgdg * (vgd - vgd_orig) - gIgcdg * (vgs - vgs_orig) - gIgcdd * (vds - vds_orig) -
                              gIgcdb * (vbs - vbs_orig));
    }
    if (igbMod) {
      gIbtotg = gIgbg;
      gIbtotd = gIgbd;
      gIbtots = gIgbs;
      gIbtotb = gIgbb;
      Ibtoteq = dtype * Igb;
      Ibtoteq_Jdxp = dtype * (-gIgbg * (vgs - vgs_orig) - gIgbd * (vds - vds_orig) - gIgbb * (vbs - vbs_orig));
    }
  } else {
    if (igcMod) {
      gIstotg = gIgsg + gIgcdg;
      gIstotd = gIgcds;
      gIstots = gIgss + gIgcdd;
      gIstotb = gIgcdb;
      Istoteq = dtype * (Igs + Igcd);
      Istoteq_Jdxp = dtype * (-gIgsg * (vgs - vgs_orig) - gIgcdg * (vgd - vgd_orig) + gIgcdd * (vds - vds_orig) -
                              gIgcdb * (vbd - vbd_orig));
      gIdtotg = gIgdg + gIgcsg;
      gIdtotd = gIgdd + gIgcss;
      gIdtots = gIgcsd;
      gIdtotb = gIgcsb;
      Idtoteq = dtype * (Igd + Igcs);
      Idtoteq_Jdxp = dtype * (-(gIgdg + gIgcsg) * (vgd - vgd_orig) + gIgcsd * (vds - vds_orig) -
                              gIgcsb * (vbd - vbd_orig));
    }
    if (igbMod) {
      gIbtotg = gIgbg;
      gIbtotd = gIgbs;
      gIbtots = gIgbd;
      gIbtotb = gIgbb;
      Ibtoteq = dtype * Igb;
      Ibtoteq_Jdxp = dtype * (-gIgbg * (vgd - vgd_orig) + gIgbd * (vds - vds_orig) - gIgbb * (vbd - vbd_orig));
    }
  }
  if (igcMod != 0 || igbMod != 0) {
    gIgtotg = gIstotg + gIdtotg + gIbtotg;
    gIgtotd = gIstotd + gIdtotd + gIbtotd;
    gIgtots = gIstots + gIdtots + gIbtots;
    gIgtotb = gIstotb + gIdtotb + gIbtotb;
    Igtoteq = Istoteq + Idtoteq + Ibtoteq;
    Igtoteq_Jdxp = Istoteq_Jdxp + Idtoteq_Jdxp + Ibtoteq_Jdxp;
  }
  // Gate resistance (rgateMod 2 / 3): the reference scales the DC part's derivatives by the
  // gate-resistor drop in place and folds gcrg into gcrgg (:13637-13664, :13767-13795).
  double gcrg = GEN ? m.v[m_gcrg] : 0.0, gcrgg = GEN ? m.v[m_gcrgg] : 0.0, gcrgd = GEN ? m.v[m_gcrgd] : 0.0;
  double gcrgs = GEN ? m.v[m_gcrgs] : 0.0, gcrgb = GEN ? m.v[m_gcrgb] : 0.0;
  if (GEN) {
    double Tg = 0.0;
    if (rgateMod == 2)
      Tg = vges - vgs;
    else if (rgateMod == 3)
      Tg = vgms - vgs;
    if (rgateMod > 1) {
      if (mode >= 0) {
        gcrgd = gcrgd * Tg;
        gcrgg = gcrgg * Tg;
        gcrgs = gcrgs * Tg;
        gcrgb = gcrgb * Tg;
        ceqgcrg = 0.0;
        ceqgcrg_Jdxp = -(gcrgd * (vds - vds_orig) + gcrgg * (vgs - vgs_orig) + gcrgb * (vbs - vbs_orig));
      } else {
        const double tmp_gcrgd = gcrgd;
        gcrgd = gcrgs * Tg;
        gcrgg = gcrgg * Tg;
        gcrgs = tmp_gcrgd * Tg;
        gcrgb = gcrgb * Tg;
        ceqgcrg = 0.0;
        ceqgcrg_Jdxp = -(gcrgg * (vgd - vgd_orig) - gcrgs * (vds - vds_orig) + gcrgb * (vbd - vbd_orig));
      }
      gcrgg -= gcrg;
    } else {
      ceqgcrg = gcrg = gcrgd = gcrgg = gcrgs = gcrgb = 0.0;
      ceqgcrg_Jdxp = 0.0;
    }
  }
  // Bias-dependent S/D resistance (rdsMod 1, :13797-13820).
  double gstot = 0.0, gstotd = 0.0, gstotg = 0.0, gstots = 0.0, gstotb = 0.0;
  double gdtot = 0.0, gdtotd = 0.0, gdtotg = 0.0, gdtots = 0.0, gdtotb = 0.0;
  double ceqgstot = 0.0, ceqgstot_Jdxp = 0.0, ceqgdtot = 0.0, ceqgdtot_Jdxp = 0.0;
  if (rdsMod) {
    gstot = m.v[m_gstot]; gstotd = m.v[m_gstotd]; gstotg = m.v[m_gstotg]; gstots = m.v[m_gstots];
    gstotb = m.v[m_gstotb];
    gdtot = m.v[m_gdtot]; gdtotd = m.v[m_gdtotd]; gdtotg = m.v[m_gdtotg]; gdtots = m.v[m_gdtots];
    gdtotb = m.v[m_gdtotb];
    ceqgstot = 0.0;
    ceqgstot_Jdxp = dtype * (gstotd * (vds - vds_orig) + gstotg * (vgs - vgs_orig) + gstotb * (vbs - vbs_orig));
    gstots = gstots - gstot;
    ceqgdtot = 0.0;
    ceqgdtot_Jdxp = -dtype * (gdtotd * (vds - vds_orig) + gdtotg * (vgs - vgs_orig) + gdtotb * (vbs - vbs_orig));
    gdtotd = gdtotd - gdtot;
  }
  double ceqjs, ceqjs_Jdxp, ceqjd, ceqjd_Jdxp;
  if (dtype > 0) {
    ceqjs = (cbs);
    ceqjs_Jdxp = (-gbs * (vbs_jct - vbs_jct_orig));
    ceqjd = (cbd);
    ceqjd_Jdxp = (-gbd * (vbd_jct - vbd_jct_orig));
  } else {
    ceqjs = -(cbs);
    ceqjs_Jdxp = (gbs * (vbs_jct - vbs_jct_orig));
    ceqjd = -(cbd);
    ceqjd_Jdxp = (gbd * (vbd_jct - vbd_jct_orig));
    ceqgcrg = -ceqgcrg;
    ceqgcrg_Jdxp = -ceqgcrg_Jdxp;
  }
  (void)ceqgstot; (void)ceqgdtot;

  if constexpr (GEN) {
    // ---- General topology: the reference's loads over the 15 local nodes ----
    const bool lim = fl.voltlim && !origFlag;
    // Terminal resistor and body-network currents (:11896-11917).
    const double Idrain = rdsMod ? gdtot * Vddp : P(drainConductance) * Vddp;
    const double Isource = rdsMod ? gstot * Vssp : P(sourceConductance) * Vssp;
    double Idbb = 0.0, Idbbp = 0.0, Isbb = 0.0, Isbbp = 0.0, Ibpb = 0.0;
    if (rbodyMod) {
      Idbb = P(grbdb) * bias.Vdbb;
      Idbbp = P(grbpd) * bias.Vdbbp;
      Isbb = P(grbsb) * bias.Vsbb;
      Isbbp = P(grbps) * bias.Vsbbp;
      Ibpb = P(grbpb) * bias.Vbpb;
    }
    const double Igate_Jdxp = 0.0, IgateMid_Jdxp = 0.0;  // the reference leaves both at zero (:11826)
#define GV(v, node) o.gv[(v)*kGenNodes + (node)]
    for (int k = 0; k < 4 * kGenNodes; ++k) o.gv[k] = 0.0;
    // Master::loadDAEVectors (:16316-16564).
    GV(0, g_DP) += -(ceqjd - ceqbd - ceqdrn + Idtoteq) * M;
    GV(0, g_GP) -= -(-ceqgcrg + Igtoteq) * M;
    if (rgateMod == 1) {
      GV(0, g_G) -= -(Igate) * M;
      GV(0, g_GP) += -(Igate) * M;
    } else if (rgateMod == 2) {
      GV(0, g_G) -= -(Igate + ceqgcrg) * M;
      GV(0, g_GP) += -(Igate) * M;
    } else if (rgateMod == 3) {
      GV(0, g_G) -= -(Igate) * M;
      GV(0, g_GM) -= -(IgateMid - Igate + ceqgcrg) * M;
      GV(0, g_GP) += -(IgateMid) * M;
    }
    if (!rbodyMod) {
      GV(0, g_BP) += -(ceqbd + ceqbs - ceqjd - ceqjs + Ibtoteq) * M;
      GV(0, g_SP) += -(ceqdrn - ceqbs + ceqjs + Istoteq) * M;
    } else {
      GV(0, g_DB) -= -(ceqjd + Idbb + Idbbp) * M;
      GV(0, g_BP) += -(ceqbd + ceqbs + Ibtoteq + Idbbp + Isbbp - Ibpb) * M;
      GV(0, g_B) += -(Isbb + Idbb + Ibpb) * M;
      GV(0, g_SB) -= -(ceqjs + Isbb + Isbbp) * M;
      GV(0, g_SP) += -(ceqdrn - ceqbs + ceqjs + Istoteq) * M;
    }
    if (rdsMod) {
      GV(0, g_D) += -(-ceqgdtot) * M;
      GV(0, g_S) += -(ceqgstot) * M;
      GV(0, g_DP) += -(ceqgdtot) * M;
      GV(0, g_SP) += -(-ceqgstot) * M;
    }
    if (P(dExists) != 0.0) {
      GV(0, g_D) += -(-Idrain) * M;
      GV(0, g_DP) += -(Idrain) * M;
    }
    if (P(sExists) != 0.0) {
      GV(0, g_S) += -(-Isource) * M;
      GV(0, g_SP) += -(+Isource) * M;
    }
    // Instance initial conditions: a branch current enforcing the terminal voltage during the
    // operating point (:16373-16401); not scaled by the multiplier.
    if (fl.dcop && P(icVBSGiven) != 0.0) {
      const double coef = V[g_IBS];
      GV(0, g_B) += coef;
      GV(0, g_S) += -coef;
      GV(0, g_IBS) += (V[g_B] - V[g_S] - P(icVBS));
    }
    if (fl.dcop && P(icVDSGiven) != 0.0) {
      const double coef = V[g_IDS];
      GV(0, g_D) += coef;
      GV(0, g_S) += -coef;
      GV(0, g_IDS) += (V[g_D] - V[g_S] - P(icVDS));
    }
    if (fl.dcop && P(icVGSGiven) != 0.0) {
      const double coef = V[g_IGS];
      GV(0, g_G) += coef;
      GV(0, g_S) += -coef;
      GV(0, g_IGS) += (V[g_G] - V[g_S] - P(icVGS));
    }
    if (lim) {
      GV(2, g_DP) += (ceqjd_Jdxp - ceqbd_Jdxp - ceqdrn_Jdxp + Idtoteq_Jdxp) * M;
      GV(2, g_GP) -= (-ceqgcrg_Jdxp + Igtoteq_Jdxp) * M;
      if (rgateMod == 1) {
        GV(2, g_G) -= (Igate_Jdxp) * M;
        GV(2, g_GP) += (Igate_Jdxp) * M;
      } else if (rgateMod == 2) {
        GV(2, g_G) -= (Igate_Jdxp + ceqgcrg_Jdxp) * M;
        GV(2, g_GP) += (Igate_Jdxp) * M;
      } else if (rgateMod == 3) {
        GV(2, g_G) -= (Igate_Jdxp) * M;
        GV(2, g_GM) -= (IgateMid_Jdxp - Igate_Jdxp + ceqgcrg_Jdxp) * M;
        GV(2, g_GP) += (IgateMid_Jdxp) * M;
      }
      if (!rbodyMod) {
        GV(2, g_BP) += (ceqbd_Jdxp + ceqbs_Jdxp - ceqjd_Jdxp - ceqjs_Jdxp + Ibtoteq_Jdxp) * M;
        GV(2, g_SP) += (ceqdrn_Jdxp - ceqbs_Jdxp + ceqjs_Jdxp + Istoteq_Jdxp) * M;
      } else {
        GV(2, g_DB) -= (ceqjd_Jdxp) * M;
        GV(2, g_BP) += (ceqbd_Jdxp + ceqbs_Jdxp + Ibtoteq_Jdxp) * M;
        GV(2, g_SB) -= (ceqjs_Jdxp) * M;
        GV(2, g_SP) += (ceqdrn_Jdxp - ceqbs_Jdxp + ceqjs_Jdxp + Istoteq_Jdxp) * M;
      }
      if (rdsMod) {
        GV(2, g_D) -= (ceqgdtot_Jdxp) * M;
        GV(2, g_S) += (ceqgstot_Jdxp) * M;
        GV(2, g_DP) += (ceqgdtot_Jdxp) * M;
        GV(2, g_SP) -= (ceqgstot_Jdxp) * M;
      }
    }
    // auxChargeCalculations (:12216-12350).
    double Qeqqg_Jdxp = 0.0, Qeqqd_Jdxp = 0.0, Qeqqb_Jdxp = 0.0, Qeqqgmid_Jdxp = 0.0;
    double Qeqqjs_Jdxp = 0.0, Qeqqjd_Jdxp = 0.0;
    if (ChargeComputationNeeded && !origFlag) {
      Qeqqg_Jdxp = -CAPcggb * (vgb - vgb_orig) + CAPcgdb * (vbd - vbd_orig) + CAPcgsb * (vbs - vbs_orig);
      Qeqqd_Jdxp = -CAPcdgb * (vgb - vgb_orig) - CAPcdgmb * (vgmb - vgmb_orig) +
                   (CAPcddb + CAPcdbdb) * (vbd - vbd_orig) - CAPcdbdb * (vbd_jct - vbd_jct_orig) +
                   CAPcdsb * (vbs - vbs_orig);
      Qeqqb_Jdxp = -CAPcbgb * (vgb - vgb_orig) - CAPcbgmb * (vgmb - vgmb_orig) + CAPcbdb * (vbd - vbd_orig) +
                   CAPcbsb * (vbs - vbs_orig);
      if (rgateMod == 3)
        Qeqqgmid_Jdxp = +CAPcgmdb * (vbd - vbd_orig) + CAPcgmsb * (vbs - vbs_orig) - CAPcgmgmb * (vgmb - vgmb_orig);
      if (rbodyMod) {
        Qeqqjs_Jdxp = CAPcsbsb * (vbs_jct - vbs_jct_orig);
        Qeqqjd_Jdxp = CAPcdbdb * (vbd_jct - vbd_jct_orig);
      }
    }
    // NQS (:12232-12244, 12300-12322): the charge-node terms of the limiter vectors; outside charge
    // computation the partition is the fixed 40/60 one and gtau is formed again from gcrg as the
    // F-vector set-up left it (zero unless rgateMod 2 / 3).
    double Qqcheq_Jdxp = 0.0;
    if (trnqsMod) {
      if (ChargeComputationNeeded) {
        const double T0n = ggtg * (vgb - vgb_orig) - ggtd * (vbd - vbd_orig) - ggts * (vbs - vbs_orig);
        Qeqqg_Jdxp += T0n;
        const double T1n = qdef * gtau;
        Qeqqd_Jdxp -= dxpart * T0n + T1n * (ddxpart_dVg * (vgb - vgb_orig) - ddxpart_dVd * (vbd - vbd_orig) -
                                            ddxpart_dVs * (vbs - vbs_orig));
        Qqcheq_Jdxp = -(CAPcqgb * (vgb - vgb_orig) - CAPcqdb * (vbd - vbd_orig) - CAPcqsb * (vbs - vbs_orig)) + T0n;
      } else {
        sxpart = (1.0 - (dxpart = (mode > 0) ? 0.4 : 0.6));
        ddxpart_dVd = ddxpart_dVg = ddxpart_dVb = ddxpart_dVs = 0.0;
        dsxpart_dVd = dsxpart_dVg = dsxpart_dVb = dsxpart_dVs = 0.0;
        gtau = gcrg / CoxWL * ScalingFactor;
      }
    }
    const double sgn = dtype > 0 ? 1.0 : -1.0;
    (void)sgn;
    double Qeqqg, Qeqqd, Qeqqb, Qeqqgmid = 0.0, Qeqqjs = 0.0, Qeqqjd = 0.0;
    if (dtype > 0) {
      Qeqqg = qg;
      Qeqqd = qd;
      Qeqqb = qb;
      if (rbodyMod) {
        Qeqqjs = qbs;
        Qeqqjd = qbd;
      }
      if (rgateMod == 3) Qeqqgmid = qgmid;
    } else {
      Qeqqg = -qg;
      Qeqqd = -qd;
      Qeqqb = -qb;
      if (rbodyMod) {
        Qeqqjs = -qbs;
        Qeqqjd = -qbd;
      }
      if (rgateMod == 3) Qeqqgmid = -qgmid;
    }
    GV(1, g_DP) += -(-Qeqqd) * M;
    GV(1, g_GP) -= -(Qeqqg) * M;
    if (rgateMod == 3) GV(1, g_GM) -= -(+Qeqqgmid) * M;
    if (!rbodyMod) {
      GV(1, g_BP) += -(-Qeqqb) * M;
      GV(1, g_SP) += -(+Qeqqg + Qeqqb + Qeqqd + Qeqqgmid) * M;
    } else {
      GV(1, g_DB) -= -(Qeqqjd) * M;
      GV(1, g_BP) += -(-Qeqqb) * M;
      GV(1, g_SB) -= -(Qeqqjs) * M;
      GV(1, g_SP) += -(Qeqqd + Qeqqg + Qeqqb + Qeqqjd + Qeqqjs + Qeqqgmid) * M;
    }
    if (trnqsMod) {
      const double Qqdef = dtype > 0 ? qdef : -qdef, Qqcheq = dtype > 0 ? qcheq : -qcheq;
      GV(1, g_Q) += -(Qqcheq - Qqdef) * M;
    }
    if (lim) {
      GV(3, g_DP) += (-Qeqqd_Jdxp) * M;
      GV(3, g_GP) -= (Qeqqg_Jdxp) * M;
      if (rgateMod == 3) GV(3, g_GM) -= (+Qeqqgmid_Jdxp) * M;
      if (!rbodyMod) {
        GV(3, g_BP) += (-Qeqqb_Jdxp) * M;
        GV(3, g_SP) += (+Qeqqg_Jdxp + Qeqqb_Jdxp + Qeqqd_Jdxp + Qeqqgmid_Jdxp) * M;
      } else {
        GV(3, g_DB) -= (Qeqqjd_Jdxp) * M;
        GV(3, g_BP) += (-Qeqqb_Jdxp) * M;
        GV(3, g_SB) -= (+Qeqqjs_Jdxp) * M;
        GV(3, g_SP) += (+Qeqqd_Jdxp + Qeqqg_Jdxp + Qeqqb_Jdxp + Qeqqjd_Jdxp + Qeqqjs_Jdxp + Qeqqgmid_Jdxp) * M;
      }
      if (trnqsMod) GV(3, g_Q) += (Qqcheq_Jdxp) * M;
    }
#undef GV
    // Master::loadDAEMatrices, pointer form (:16577-16853 and :17102-17172).
    for (int k = 0; k < kGenSlots; ++k) {
      o.gf[k] = 0.0;
      o.gq[k] = 0.0;
    }
#define GF(r, c) o.gf[GenSlotOf<g_##r, g_##c>::value]
#define GQ(r, c) o.gq[GenSlotOf<g_##r, g_##c>::value]
    const double gjbd = !rbodyMod ? gbd : 0.0, gjbs = !rbodyMod ? gbs : 0.0;
    const double gdpr = !rdsMod ? P(drainConductance) : 0.0, gspr = !rdsMod ? P(sourceConductance) : 0.0;
    const double geltd = P(grgeltd);
    const double Tq = qdef * gtau;  // :16606
    if (rgateMod == 1) {
      GF(G, G) += (geltd) * M;
      GF(G, GP) -= (geltd) * M;
      GF(GP, G) -= (geltd) * M;
      GF(GP, GP) += (+geltd - ggtg + gIgtotg) * M;
      GF(GP, DP) += (-ggtd + gIgtotd) * M;
      GF(GP, SP) += (-ggts + gIgtots) * M;
      GF(GP, BP) += (-ggtb + gIgtotb) * M;
    } else if (rgateMod == 2) {
      GF(G, G) += (gcrg) * M;
      GF(G, GP) += (gcrgg) * M;
      GF(G, DP) += (gcrgd) * M;
      GF(G, SP) += (gcrgs) * M;
      GF(G, BP) += (gcrgb) * M;
      GF(GP, G) -= (gcrg) * M;
      GF(GP, GP) += (-gcrgg - ggtg + gIgtotg) * M;
      GF(GP, DP) += (-gcrgd - ggtd + gIgtotd) * M;
      GF(GP, SP) += (-gcrgs - ggts + gIgtots) * M;
      GF(GP, BP) += (-gcrgb - ggtb + gIgtotb) * M;
    } else if (rgateMod == 3) {
      GF(G, G) += (geltd) * M;
      GF(G, GM) -= (geltd) * M;
      GF(GM, G) -= (geltd) * M;
      GF(GM, GM) += (geltd + gcrg) * M;
      GF(GM, DP) += (gcrgd) * M;
      GF(GM, GP) += (gcrgg) * M;
      GF(GM, SP) += (gcrgs) * M;
      GF(GM, BP) += (gcrgb) * M;
      GF(GP, GM) -= (gcrg) * M;
      GF(GP, GP) += (-gcrgg - ggtg + gIgtotg) * M;
      GF(GP, DP) += (-gcrgd - ggtd + gIgtotd) * M;
      GF(GP, SP) += (-gcrgs - ggts + gIgtots) * M;
      GF(GP, BP) += (-gcrgb - ggtb + gIgtotb) * M;
    } else {
      GF(GP, GP) += (-ggtg + gIgtotg) * M;
      GF(GP, DP) += (-ggtd + gIgtotd) * M;
      GF(GP, SP) += (-ggts + gIgtots) * M;
      GF(GP, BP) += (-ggtb + gIgtotb) * M;
    }
    if (rdsMod) {
      GF(D, GP) += (gdtotg) * M;
      GF(D, SP) += (gdtots) * M;
      GF(D, BP) += (gdtotb) * M;
      GF(S, DP) += (gstotd) * M;
      GF(S, GP) += (gstotg) * M;
      GF(S, BP) += (gstotb) * M;
    }
    GF(DP, DP) += (gdpr + gds + gbd + Tq * ddxpart_dVd - gdtotd + RevSum + gbdpdp + dxpart * ggtd - gIdtotd) * M;
    GF(DP, D) -= (gdpr + gdtot) * M;
    GF(DP, GP) += (Gmv - gdtotg + gbdpg - gIdtotg + dxpart * ggtg + Tq * ddxpart_dVg) * M;
    GF(DP, SP) -= (gds + gdtots - dxpart * ggts + gIdtots - Tq * ddxpart_dVs + FwdSum - gbdpsp) * M;
    GF(DP, BP) -= (gjbd + gdtotb - Gmbsv - gbdpb + gIdtotb - Tq * ddxpart_dVb - dxpart * ggtb) * M;
    GF(D, DP) -= (gdpr - gdtotd) * M;
    GF(D, D) += (gdpr + gdtot) * M;
    GF(SP, DP) -= (gds + gstotd + RevSum - gbspdp - Tq * dsxpart_dVd - sxpart * ggtd + gIstotd) * M;
    GF(SP, GP) += (-Gmv - gstotg + gbspg + sxpart * ggtg + Tq * dsxpart_dVg - gIstotg) * M;
    GF(SP, SP) += (gspr + gds + gbs + Tq * dsxpart_dVs - gstots + FwdSum + gbspsp + sxpart * ggts - gIstots) * M;
    GF(SP, S) -= (gspr + gstot) * M;
    GF(SP, BP) -= (gjbs + gstotb + Gmbsv - gbspb - sxpart * ggtb - Tq * dsxpart_dVb + gIstotb) * M;
    GF(S, SP) -= (gspr - gstots) * M;
    GF(S, S) += (gspr + gstot) * M;
    GF(BP, DP) += (-gjbd + gbbdp - gIbtotd) * M;
    GF(BP, GP) += (-gbgs - gIbtotg) * M;
    GF(BP, SP) += (-gjbs + gbbsp - gIbtots) * M;
    GF(BP, BP) += (gjbd + gjbs - gbbs - gIbtotb) * M;
    GF(DP, DP) += (ggidld) * M;
    GF(DP, GP) += (ggidlg) * M;
    GF(DP, SP) -= ((ggidlg + ggidld + ggidlb)) * M;
    GF(DP, BP) += (ggidlb) * M;
    GF(BP, DP) -= (ggidld) * M;
    GF(BP, GP) -= (ggidlg) * M;
    GF(BP, SP) += ((ggidlg + ggidld + ggidlb)) * M;
    GF(BP, BP) -= (ggidlb) * M;
    GF(SP, DP) -= ((ggisls + ggislg + ggislb)) * M;
    GF(SP, GP) += (ggislg) * M;
    GF(SP, SP) += (ggisls) * M;
    GF(SP, BP) += (ggislb) * M;
    GF(BP, DP) += ((ggislg + ggisls + ggislb)) * M;
    GF(BP, GP) -= (ggislg) * M;
    GF(BP, SP) -= (ggisls) * M;
    GF(BP, BP) -= (ggislb) * M;
    if (rbodyMod) {
      GF(DP, DB) += (-gbd) * M;
      GF(SP, SB) -= (gbs) * M;
      GF(DB, DP) += (-gbd) * M;
      GF(DB, DB) += (gbd + P(grbpd) + P(grbdb)) * M;
      GF(DB, BP) -= (P(grbpd)) * M;
      GF(DB, B) -= (P(grbdb)) * M;
      GF(BP, DB) -= (P(grbpd)) * M;
      GF(BP, B) -= (P(grbpb)) * M;
      GF(BP, SB) -= (P(grbps)) * M;
      GF(BP, BP) += (P(grbpd) + P(grbps) + P(grbpb)) * M;
      GF(SB, SP) += (-gbs) * M;
      GF(SB, BP) -= (P(grbps)) * M;
      GF(SB, B) -= (P(grbsb)) * M;
      GF(SB, SB) += (gbs + P(grbps) + P(grbsb)) * M;
      GF(B, DB) -= (P(grbdb)) * M;
      GF(B, BP) -= (P(grbpb)) * M;
      GF(B, SB) -= (P(grbsb)) * M;
      GF(B, B) += (P(grbsb) + P(grbdb) + P(grbpb)) * M;
    }
    if (trnqsMod) {  // :16796-16807
      GF(Q, Q) += (gqdef + gtau) * M;
      GF(Q, GP) += (ggtg) * M;
      GF(Q, DP) += (ggtd) * M;
      GF(Q, SP) += (ggts) * M;
      GF(Q, BP) += (ggtb) * M;
      GF(DP, Q) += (dxpart * gtau) * M;
      GF(SP, Q) += (sxpart * gtau) * M;
      GF(GP, Q) -= (gtau) * M;
    }
    // Initial-condition rows (:16810-16853): the couplings during the operating point, the branch
    // current's own diagonal (assigned, the row belongs to this instance alone) otherwise.
    if (P(icVBSGiven) != 0.0) {
      if (fl.dcop) {
        GF(B, IBS) += 1.0;
        GF(S, IBS) += -1.0;
        GF(IBS, B) += 1.0;
        GF(IBS, S) += -1.0;
      } else {
        GF(IBS, IBS) = 1.0;
      }
    }
    if (P(icVDSGiven) != 0.0) {
      if (fl.dcop) {
        GF(D, IDS) += 1.0;
        GF(S, IDS) += -1.0;
        GF(IDS, D) += 1.0;
        GF(IDS, S) += -1.0;
      } else {
        GF(IDS, IDS) = 1.0;
      }
    }
    if (P(icVGSGiven) != 0.0) {
      if (fl.dcop) {
        GF(G, IGS) += 1.0;
        GF(S, IGS) += -1.0;
        GF(IGS, G) += 1.0;
        GF(IGS, S) += -1.0;
      } else {
        GF(IGS, IGS) = 1.0;
      }
    }
    if (!(!fl.dcop && fl.init_tran && fl.newton_iter == 0)) {
      if (rgateMod == 3) {
        GQ(GM, GM) += (+CAPcgmgmb) * M;
        GQ(GM, DP) += (CAPcgmdb) * M;
        GQ(GM, SP) += (CAPcgmsb) * M;
        GQ(GM, BP) += (CAPcgmbb) * M;
        GQ(DP, GM) += (CAPcdgmb) * M;
        GQ(SP, GM) += (CAPcsgmb) * M;
        GQ(BP, GM) += (CAPcbgmb) * M;
      }
      GQ(GP, GP) += (CAPcggb) * M;
      GQ(GP, DP) += (CAPcgdb) * M;
      GQ(GP, SP) += (CAPcgsb) * M;
      GQ(GP, BP) += (CAPcgbb) * M;
      GQ(DP, DP) += (CAPcddb) * M;
      GQ(DP, GP) += (+CAPcdgb) * M;
      GQ(DP, SP) -= (-CAPcdsb) * M;
      GQ(DP, BP) -= (-CAPcdbb) * M;
      GQ(SP, DP) -= (-CAPcsdb) * M;
      GQ(SP, GP) += (CAPcsgb) * M;
      GQ(SP, SP) += (CAPcssb) * M;
      GQ(SP, BP) -= (-CAPcsbb) * M;
      GQ(BP, DP) += (CAPcbdb) * M;
      GQ(BP, GP) += (CAPcbgb) * M;
      GQ(BP, SP) += (CAPcbsb) * M;
      GQ(BP, BP) += (CAPcbbb) * M;
      if (rbodyMod) {
        GQ(DP, DB) += (CAPcdbdb) * M;
        GQ(SP, SB) -= (-CAPcsbsb) * M;
        GQ(DB, DP) += (CAPcdbdb) * M;
        GQ(DB, DB) += (-CAPcdbdb) * M;
        GQ(SB, SP) += (CAPcsbsb) * M;
        GQ(SB, SB) += (-CAPcsbsb) * M;
      }
      if (trnqsMod) {  // :17181-17187
        GQ(Q, GP) += (-CAPcqgb) * M;
        GQ(Q, DP) += (-CAPcqdb) * M;
        GQ(Q, SP) += (-CAPcqsb) * M;
        GQ(Q, BP) += (-CAPcqbb) * M;
      }
    }
#undef GF
#undef GQ
    (void)Vx;
    return;
  }

  // Master::loadDAEVectors (:16316-16564). Local order D, G, S, B.
  const bool lim = fl.voltlim && !origFlag;
  for (int k = 0; k < kNumVec; ++k) o.vec[k] = 0.0;
  o.vec[0] += -(ceqjd - ceqbd - ceqdrn + Idtoteq) * M;
  o.vec[1] -= -(-ceqgcrg + Igtoteq) * M;
  o.vec[3] += -(ceqbd + ceqbs - ceqjd - ceqjs + Ibtoteq) * M;
  o.vec[2] += -(ceqdrn - ceqbs + ceqjs + Istoteq) * M;
  if (SERIES) {
    // Linear terminal resistor currents (:11901-11904, 16360-16370), where the node exists.
    o.vecx[0] = 0.0;
    o.vecx[1] = 0.0;
    if (P(dExists) != 0.0) {
      const double Idrain = P(drainConductance) * Vddp;
      o.vecx[0] += -(-Idrain) * M;
      o.vec[0] += -(Idrain)*M;
    }
    if (P(sExists) != 0.0) {
      const double Isource = P(sourceConductance) * Vssp;
      o.vecx[1] += -(-Isource) * M;
      o.vec[2] += -(+Isource) * M;
    }
  }
  if (lim) {
    o.vec[8 + 0] += (ceqjd_Jdxp - ceqbd_Jdxp - ceqdrn_Jdxp + Idtoteq_Jdxp) * M;
    o.vec[8 + 1] -= (-ceqgcrg_Jdxp + Igtoteq_Jdxp) * M;
    o.vec[8 + 3] += (ceqbd_Jdxp + ceqbs_Jdxp - ceqjd_Jdxp - ceqjs_Jdxp + Ibtoteq_Jdxp) * M;
    o.vec[8 + 2] += (ceqdrn_Jdxp - ceqbs_Jdxp + ceqjs_Jdxp + Istoteq_Jdxp) * M;
  }
  // auxChargeCalculations (:12216-12350).
  double Qeqqg_Jdxp = 0.0, Qeqqd_Jdxp = 0.0, Qeqqb_Jdxp = 0.0;
  if (ChargeComputationNeeded && !origFlag) {
    Qeqqg_Jdxp = -CAPcggb * (vgb - vgb_orig) + CAPcgdb * (vbd - vbd_orig) + CAPcgsb * (vbs - vbs_orig);
    Qeqqd_Jdxp = -CAPcdgb * (vgb - vgb_orig) - CAPcdgmb * (vgmb - vgmb_orig) +
                 (CAPcddb + 0.0) * (vbd - vbd_orig) - 0.0 * (vbd_jct - vbd_jct_orig) + CAPcdsb * (vbs - vbs_orig);
    Qeqqb_Jdxp = -CAPcbgb * (vgb - vgb_orig) - CAPcbgmb * (vgmb - vgmb_orig) + CAPcbdb * (vbd - vbd_orig) +
                 CAPcbsb * (vbs - vbs_orig);
  }
  const double Qeqqgmid_Jdxp = 0.0, Qeqqgmid = 0.0;
  double Qeqqg, Qeqqd, Qeqqb;
  if (dtype > 0) {
    Qeqqg = qg;
    Qeqqd = qd;
    Qeqqb = qb;
  } else {
    Qeqqg = -qg;
    Qeqqd = -qd;
    Qeqqb = -qb;
  }
  o.vec[4 + 0] += -(-Qeqqd) * M;
  o.vec[4 + 1] -= -(Qeqqg) * M;
  o.vec[4 + 3] += -(-Qeqqb) * M;
  o.vec[4 + 2] += -(+Qeqqg + Qeqqb + Qeqqd + Qeqqgmid) * M;
  if (lim) {
    o.vec[12 + 0] += (-Qeqqd_Jdxp) * M;
    o.vec[12 + 1] -= (Qeqqg_Jdxp) * M;
    o.vec[12 + 3] += (-Qeqqb_Jdxp) * M;
    o.vec[12 + 2] += (+Qeqqg_Jdxp + Qeqqb_Jdxp + Qeqqd_Jdxp + Qeqqgmid_Jdxp) * M;
  }

  // Master::loadDAEMatrices (:16577-17268). Rows/cols D=0 G=1 S=2 B=3.
  for (int k = 0; k < kNumMat; ++k) {
    o.jf[k] = 0.0;
    o.jq[k] = 0.0;
  }
  const double gdpr = P(drainConductance), gspr = P(sourceConductance);
  // No NQS charge on this path: ggt*, the partition's derivatives and Tq = qdef * gtau are zero.
  const double Tq = qdef * gtau;
#define JF(r, c) o.jf[(r)*4 + (c)]
#define JQ(r, c) o.jq[(r)*4 + (c)]
  JF(1, 1) += (-ggtg + gIgtotg) * M;
  JF(1, 0) += (-ggtd + gIgtotd) * M;
  JF(1, 2) += (-ggts + gIgtots) * M;
  JF(1, 3) += (-ggtb + gIgtotb) * M;
  JF(0, 0) += (gdpr + gds + gbd + Tq * ddxpart_dVd - gdtotd + RevSum + gbdpdp + dxpart * ggtd - gIdtotd) * M;
  if (SERIES) {
    for (int k = 0; k < 6; ++k) o.jfx[k] = 0.0;
  }
  // The resistor couplings (D', D), (D, D'), (D, D) and the source's: their own slots with internal
  // nodes, the collapsed (D, D) / (S, S) entry otherwise.
#define JRES(k, r) (*(SERIES ? &o.jfx[k] : &JF(r, r)))
  JRES(0, 0) -= (gdpr + gdtot) * M;
  JF(0, 1) += (Gmv - gdtotg + gbdpg - gIdtotg + dxpart * ggtg + Tq * ddxpart_dVg) * M;
  JF(0, 2) -= (gds + gdtots - dxpart * ggts + gIdtots - Tq * ddxpart_dVs + FwdSum - gbdpsp) * M;
  JF(0, 3) -= (gjbd + gdtotb - Gmbsv - gbdpb + gIdtotb - Tq * ddxpart_dVb - dxpart * ggtb) * M;
  JRES(1, 0) -= (gdpr - gdtotd) * M;
  JRES(2, 0) += (gdpr + gdtot) * M;
  JF(2, 0) -= (gds + gstotd + RevSum - gbspdp - Tq * dsxpart_dVd - sxpart * ggtd + gIstotd) * M;
  JF(2, 1) += (-Gmv - gstotg + gbspg + sxpart * ggtg + Tq * dsxpart_dVg - gIstotg) * M;
  JF(2, 2) += (gspr + gds + gbs + Tq * dsxpart_dVs - gstots + FwdSum + gbspsp + sxpart * ggts - gIstots) * M;
  JRES(3, 2) -= (gspr + gstot) * M;
  JF(2, 3) -= (gjbs + gstotb + Gmbsv - gbspb - sxpart * ggtb - Tq * dsxpart_dVb + gIstotb) * M;
  JRES(4, 2) -= (gspr - gstots) * M;
  JRES(5, 2) += (gspr + gstot) * M;
#undef JRES
  JF(3, 0) += (-gjbd + gbbdp - gIbtotd) * M;
  JF(3, 1) += (-gbgs - gIbtotg) * M;
  JF(3, 2) += (-gjbs + gbbsp - gIbtots) * M;
  JF(3, 3) += (gjbd + gjbs - gbbs - gIbtotb) * M;
  JF(0, 0) += (ggidld) * M;
  JF(0, 1) += (ggidlg) * M;
  JF(0, 2) -= ((ggidlg + ggidld + ggidlb)) * M;
  JF(0, 3) += (ggidlb) * M;
  JF(3, 0) -= (ggidld) * M;
  JF(3, 1) -= (ggidlg) * M;
  JF(3, 2) += ((ggidlg + ggidld + ggidlb)) * M;
  JF(3, 3) -= (ggidlb) * M;
  JF(2, 0) -= ((ggisls + ggislg + ggislb)) * M;
  JF(2, 1) += (ggislg) * M;
  JF(2, 2) += (ggisls) * M;
  JF(2, 3) += (ggislb) * M;
  JF(3, 0) += ((ggislg + ggisls + ggislb)) * M;
  JF(3, 1) -= (ggislg) * M;
  JF(3, 2) -= (ggisls) * M;
  JF(3, 3) -= (ggislb) * M;
  if (!(!fl.dcop && fl.init_tran && fl.newton_iter == 0)) {
    JQ(1, 1) += (CAPcggb) * M;
    JQ(1, 0) += (CAPcgdb) * M;
    JQ(1, 2) += (CAPcgsb) * M;
    JQ(1, 3) += (CAPcgbb) * M;
    JQ(0, 0) += (CAPcddb) * M;
    JQ(0, 1) += (+CAPcdgb) * M;
    JQ(0, 2) -= (-CAPcdsb) * M;
    JQ(0, 3) -= (-CAPcdbb) * M;
    JQ(2, 0) -= (-CAPcsdb) * M;
    JQ(2, 1) += (CAPcsgb) * M;
    JQ(2, 2) += (CAPcssb) * M;
    JQ(2, 3) -= (-CAPcsbb) * M;
    JQ(3, 0) += (CAPcbdb) * M;
    JQ(3, 1) += (CAPcbgb) * M;
    JQ(3, 2) += (CAPcbsb) * M;
    JQ(3, 3) += (CAPcbbb) * M;
  }
#undef JF
#undef JQ
}

// V[4] = node voltages (D, G, S, B); sto_old = the store values the limiter compares against
// (currSto on Newton step 0 of a transient step, nextSto otherwise); vgb_orig = the previous load's
// vgb of this instance (0 before the first load), which the reference uses as the "original" vgb.
// FULL = false compiles the load for the common card only — capMod 2, no gate tunnelling
// (igcMod = igbMod = 0) — whatever the record says, so the default kernel carries none of the
// other branches in its registers or its code; families whose cards use capMod 0/1 or the
// tunnelling currents run the FULL = true instantiation.
// SERIES = true: V holds (D', G, S', B) and Vx the external (D, S); the linear drain and source
// resistances (rdsMod = 0, sheet resistance) load into vecx / jfx.
// PART = 0: the whole evaluation; 1: the DC part only, which fills *mid; 2: the charge-and-stamp
// part only, from *mid (the DC part of the same instance, same inputs).
// GEN = true: the general topology; V holds the 15 local node values, sto_old all 14 store slots,
// and the outputs go to gv / gf / gq / gsta (the variant is compiled FULL and without SERIES).
template <bool FULL = false, bool SERIES = false, int PART = 0, bool GEN = false, class RV>
XD_HD void bsim4_load(const RV &P_, const double *V, const double *sto_old, const LoadFlags &fl, double vgb_orig,
                      LoadOut &o, const double *Vx = nullptr, Mid *mid = nullptr) {
  using namespace xdc;
  static_assert(!GEN || (FULL && !SERIES), "the general topology is evaluated by the full, non-series load");
  if constexpr (PART == 2) {
    bsim4_finish<FULL, SERIES, GEN>(P_, V, fl, vgb_orig, *mid, o, Vx);
    return;
  }
  const double dtype = P(dtype);
  const int mobMod = (int)P(mobMod);
  const int dioMod = (int)P(dioMod);
  const int tempMod = (int)P(tempMod);
  const int capMod = FULL ? (int)P(capMod) : 2;
  const double gmin = fl.gmin;
  const double nf = P(nf);
  const double vth0 = P(vth0);
  const double M = P(mult);
  const bool OFF = P(off) != 0.0;

  const bool ChargeComputationNeeded = (fl.tranop || fl.acop || fl.transient);

  const int rgateMod = GEN ? (int)P(rgateMod) : 0;
  const bool rbodyMod = GEN && P(rbodyMod) != 0.0;
  const bool rdsMod = GEN && P(rdsMod) != 0.0;
  Bias bias;
  bsim4_bias<SERIES, GEN>(P_, V, fl, Vx, bias);
  const double Vddp = bias.Vddp, Vssp = bias.Vssp;
  (void)Vddp; (void)Vssp;
  double vds = bias.vds, vgs = bias.vgs, vbs = bias.vbs, vges = bias.vges, vgms = bias.vgms, vdbs = bias.vdbs;
  double vsbs = bias.vsbs, vses = bias.vses, vdes = bias.vdes, vbd = bias.vbd, vdbd = bias.vdbd, vgd = bias.vgd;
  double vged = bias.vged, vgmd = bias.vgmd, vgmb = bias.vgmb, vbs_jct = bias.vbs_jct, vbd_jct = bias.vbd_jct;
  const double vbd_orig = bias.vbd_orig, vbs_orig = bias.vbs_orig, vgs_orig = bias.vgs_orig;
  const double vds_orig = bias.vds_orig, vgd_orig = bias.vgd_orig, vges_orig = bias.vges_orig;
  const double vgms_orig = bias.vgms_orig, vdes_orig = bias.vdes_orig, vses_orig = bias.vses_orig;
  const double vdbs_orig = bias.vdbs_orig, vsbs_orig = bias.vsbs_orig, vdbd_orig = bias.vdbd_orig;
  const double vged_orig = bias.vged_orig, vgmd_orig = bias.vgmd_orig, vbs_jct_orig = bias.vbs_jct_orig;
  const double vbd_jct_orig = bias.vbd_jct_orig, vgmb_orig = bias.vgmb_orig;
  (void)vdes_orig; (void)vses_orig; (void)vdbs_orig; (void)vsbs_orig; (void)vdbd_orig; (void)vged_orig;
  (void)vgmd_orig; (void)vges_orig; (void)vgms_orig;
  int origFlag = bias.origFlag;
  // The reference takes vgb_orig from the instance's vgb member before it is recomputed, i.e. the
  // previous load's value (:8026); in the limiter test below vgb therefore equals vgb_orig.
  double vgb = vgb_orig;
  // Previous-iterate voltages for limiting (:8099-8166).
  double vbd_old, vbs_old, vgs_old, vds_old, von_local;
  double vges_old = 0.0, vgms_old = 0.0, vdes_old = 0.0, vses_old = 0.0, vdbs_old = 0.0, vsbs_old = 0.0;
  double vdbd_old = 0.0, vged_old = 0.0, vgmd_old = 0.0;
  if (fl.newton_iter == 0 && fl.dcop) {
    vbd_old = vbd;
    vbs_old = vbs;
    vgs_old = vgs;
    vds_old = vds;
    von_local = 0.0;
    if (GEN) {
      vges_old = vges; vgms_old = vgms; vdes_old = vdes; vses_old = vses; vdbs_old = vdbs; vsbs_old = vsbs;
      vdbd_old = vdbd; vged_old = vged; vgmd_old = vgmd;
    }
  } else {
    vbd_old = sto_old[s_vbd];
    vbs_old = sto_old[s_vbs];
    vgs_old = sto_old[s_vgs];
    vds_old = sto_old[s_vds];
    von_local = sto_old[s_von];
    if (GEN) {
      // vged / vgmd are never written by the load: their "old" values are whatever the store holds.
      vges_old = sto_old[s_vges]; vgms_old = sto_old[s_vgms]; vdes_old = sto_old[s_vdes];
      vses_old = sto_old[s_vses]; vdbs_old = sto_old[s_vdbs]; vsbs_old = sto_old[s_vsbs];
      vdbd_old = sto_old[s_vdbd]; vged_old = sto_old[s_vged]; vgmd_old = sto_old[s_vgmd];
    }
  }
  const double vgd_old = vgs_old - vds_old;
  (void)vdbd_old;

  if (fl.voltlim && !(fl.init_fix && OFF)) {
    int Check = 0;
    if (fl.newton_iter >= 0 && !(fl.init_jct)) {
      if (vds_old >= 0.0) {
        vgs = fetlim(vgs, vgs_old, von_local);
        vds = vgs - vgd;
        vds = limvds(vds, vds_old);
        vgd = vgs - vds;
        if (GEN) {
          if (rgateMod == 3) {
            vges = fetlim(vges, vges_old, von_local);
            vgms = fetlim(vgms, vgms_old, von_local);
          } else if ((rgateMod == 1) || (rgateMod == 2)) {
            vges = fetlim(vges, vges_old, von_local);
            vged = vges - vds;
          }
          if (rdsMod) {
            vdes = limvds(vdes, vdes_old);
            vses = -limvds(-vses, -vses_old);
          }
        }
      } else {
        vgd = fetlim(vgd, vgd_old, von_local);
        vds = vgs - vgd;
        vds = -limvds(-vds, -vds_old);
        vgs = vgd + vds;
        if (GEN) {
          if (rgateMod == 3) {
            vged = fetlim(vged, vged_old, von_local);
            vges = vged + vds;
            vgmd = fetlim(vgmd, vgmd_old, von_local);
            vgms = vgmd + vds;
          }
          if ((rgateMod == 1) || (rgateMod == 2)) {
            vged = fetlim(vged, vged_old, von_local);
            vges = vged + vds;
          }
          if (rdsMod) {
            vdes = -limvds(-vdes, -vdes_old);
            vses = limvds(vses, vses_old);
          }
        }
      }
      if (vds >= 0.0) {
        vbs = pnjlim(vbs, vbs_old, CONSTvt0, P(vcrit), &Check);
        vbd = vbs - vds;
        if (rbodyMod) {
          int Check1 = 0, Check2 = 0;
          vdbs = pnjlim(vdbs, vdbs_old, CONSTvt0, P(vcrit), &Check1);
          vdbd = vdbs - vds;
          vsbs = pnjlim(vsbs, vsbs_old, CONSTvt0, P(vcrit), &Check2);
        }
      } else {
        vbd = pnjlim(vbd, vbd_old, CONSTvt0, P(vcrit), &Check);
        vbs = vbd + vds;
        if (rbodyMod) {
          int Check1 = 0, Check2 = 0;
          vdbd = pnjlim(vdbd, vdbd_old, CONSTvt0, P(vcrit), &Check1);
          vdbs = vdbd + vds;
          const double vsbd_old = vsbs_old - vds_old;
          double vsbd = vsbs - vds;
          vsbd = pnjlim(vsbd, vsbd_old, CONSTvt0, P(vcrit), &Check2);
          vsbs = vsbd + vds;
        }
      }
    }
    (void)Check;
    if (fabs(vbd_orig - vbd) > kMachPrec || fabs(vbs_orig - vbs) > kMachPrec || fabs(vgs_orig - vgs) > kMachPrec ||
        fabs(vds_orig - vds) > kMachPrec || fabs(vgd_orig - vgd) > kMachPrec || fabs(vges_orig - vges) > kMachPrec ||
        fabs(vgms_orig - vgms) > kMachPrec || fabs(vdes_orig - vdes) > kMachPrec ||
        fabs(vses_orig - vses) > kMachPrec || fabs(vdbs_orig - vdbs) > kMachPrec ||
        fabs(vsbs_orig - vsbs) > kMachPrec || fabs(vdbd_orig - vdbd) > kMachPrec ||
        fabs(vbs_jct_orig - vbs_jct) > kMachPrec || fabs(vbd_jct_orig - vbd_jct) > kMachPrec ||
        fabs(vgmb_orig - vgmb) > kMachPrec || fabs(vgb_orig - vgb) > kMachPrec ||
        fabs(vged_orig - vged) > kMachPrec || fabs(vgmd_orig - vgmd) > kMachPrec) {
      origFlag = 0;
    }
  }
  vbd = vbs - vds;
  vgd = vgs - vds;
  vgb = vgs - vbs;
  vged = vges - vds;
  vgmd = vgms - vds;
  vgmb = vgms - vbs;
  vdbd = vdbs - vds;
  vbs_jct = (!rbodyMod) ? vbs : vsbs;
  vbd_jct = (!rbodyMod) ? vbd : vdbd;

  double T0, T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12, T13, T14;
  double dT0_dVg, dT0_dVd, dT0_dVb, dT1_dVg, dT1_dVd, dT1_dVb, dT2_dVg, dT2_dVd, dT2_dVb;
  double dT3_dVg, dT3_dVd, dT3_dVb, dT4_dVd, dT5_dVg, dT5_dVd, dT5_dVb, dT6_dVg, dT6_dVd, dT6_dVb;
  double dT8_dVg, dT8_dVd, dT8_dVb, dT9_dVg, dT9_dVd, dT9_dVb, dT10_dVg, dT10_dVd, dT10_dVb;
  double tmp, tmp1, tmp2, tmp3, tmp4;

  // Source/drain junction diodes (:8420-8660).
  const double Aseff = P(Aseff), Pseff = P(Pseff), Adeff = P(Adeff), Pdeff = P(Pdeff), weffCJ = P(weffCJ);
  double gbs, cbs, gbd, cbd;
  {
    const double Nvtms = P(vtm) * P(SjctEmissionCoeff);
    double SourceSatCurrent;
    if ((Aseff <= 0.0) && (Pseff <= 0.0))
      SourceSatCurrent = 1.0e-14;
    else
      SourceSatCurrent = Aseff * P(SjctTempSatCurDensity) + Pseff * P(SjctSidewallTempSatCurDensity) +
                         weffCJ * nf * P(SjctGateSidewallTempSatCurDensity);
    if (SourceSatCurrent <= 0.0) {
      gbs = gmin;
      cbs = gbs * vbs_jct;
    } else {
      switch (dioMod) {
        case 0: {
          double evbs = exp(vbs_jct / Nvtms);
          T1 = P(xjbvs) * exp(-(P(bvs) + vbs_jct) / Nvtms);
          gbs = SourceSatCurrent * (evbs + T1) / Nvtms + gmin;
          cbs = SourceSatCurrent * (evbs + P(XExpBVS) - T1 - 1.0) + gmin * vbs_jct;
          break;
        }
        case 1:
          T2 = vbs_jct / Nvtms;
          if (T2 < -CONSTEXP_THRESHOLD) {
            gbs = gmin;
            cbs = SourceSatCurrent * (CONSTMIN_EXP - 1.0) + gmin * vbs_jct;
          } else if (vbs_jct <= P(vjsmFwd)) {
            double evbs = exp(T2);
            gbs = SourceSatCurrent * evbs / Nvtms + gmin;
            cbs = SourceSatCurrent * (evbs - 1.0) + gmin * vbs_jct;
          } else {
            T0 = P(IVjsmFwd) / Nvtms;
            gbs = T0 + gmin;
            cbs = P(IVjsmFwd) - SourceSatCurrent + T0 * (vbs_jct - P(vjsmFwd)) + gmin * vbs_jct;
          }
          break;
        default: {
          double evbs, devbs_dvb;
          if (vbs_jct < P(vjsmRev)) {
            T0 = vbs_jct / Nvtms;
            if (T0 < -CONSTEXP_THRESHOLD) {
              evbs = CONSTMIN_EXP;
              devbs_dvb = 0.0;
            } else {
              evbs = exp(T0);
              devbs_dvb = evbs / Nvtms;
            }
            T1 = evbs - 1.0;
            T2 = P(IVjsmRev) + P(SslpRev) * (vbs_jct - P(vjsmRev));
            gbs = devbs_dvb * T2 + T1 * P(SslpRev) + gmin;
            cbs = T1 * T2 + gmin * vbs_jct;
          } else if (vbs_jct <= P(vjsmFwd)) {
            T0 = vbs_jct / Nvtms;
            if (T0 < -CONSTEXP_THRESHOLD) {
              evbs = CONSTMIN_EXP;
              devbs_dvb = 0.0;
            } else {
              evbs = exp(T0);
              devbs_dvb = evbs / Nvtms;
            }
            T1 = (P(bvs) + vbs_jct) / Nvtms;
            if (T1 > CONSTEXP_THRESHOLD) {
              T2 = CONSTMIN_EXP;
              T3 = 0.0;
            } else {
              T2 = exp(-T1);
              T3 = -T2 / Nvtms;
            }
            gbs = SourceSatCurrent * (devbs_dvb - P(xjbvs) * T3) + gmin;
            cbs = SourceSatCurrent * (evbs + P(XExpBVS) - 1.0 - P(xjbvs) * T2) + gmin * vbs_jct;
          } else {
            gbs = P(SslpFwd) + gmin;
            cbs = P(IVjsmFwd) + P(SslpFwd) * (vbs_jct - P(vjsmFwd)) + gmin * vbs_jct;
          }
          break;
        }
      }
    }
    const double Nvtmd = P(vtm) * P(DjctEmissionCoeff);
    double DrainSatCurrent;
    if ((Adeff <= 0.0) && (Pdeff <= 0.0))
      DrainSatCurrent = 1.0e-14;
    else
      DrainSatCurrent = Adeff * P(DjctTempSatCurDensity) + Pdeff * P(DjctSidewallTempSatCurDensity) +
                        weffCJ * nf * P(DjctGateSidewallTempSatCurDensity);
    if (DrainSatCurrent <= 0.0) {
      gbd = gmin;
      cbd = gbd * vbd_jct;
    } else {
      switch (dioMod) {
        case 0: {
          double evbd = exp(vbd_jct / Nvtmd);
          T1 = P(xjbvd) * exp(-(P(bvd) + vbd_jct) / Nvtmd);
          gbd = DrainSatCurrent * (evbd + T1) / Nvtmd + gmin;
          cbd = DrainSatCurrent * (evbd + P(XExpBVD) - T1 - 1.0) + gmin * vbd_jct;
          break;
        }
        case 1:
          T2 = vbd_jct / Nvtmd;
          if (T2 < -CONSTEXP_THRESHOLD) {
            gbd = gmin;
            cbd = DrainSatCurrent * (CONSTMIN_EXP - 1.0) + gmin * vbd_jct;
          } else if (vbd_jct <= P(vjdmFwd)) {
            double evbd = exp(T2);
            gbd = DrainSatCurrent * evbd / Nvtmd + gmin;
            cbd = DrainSatCurrent * (evbd - 1.0) + gmin * vbd_jct;
          } else {
            T0 = P(IVjdmFwd) / Nvtmd;
            gbd = T0 + gmin;
            cbd = P(IVjdmFwd) - DrainSatCurrent + T0 * (vbd_jct - P(vjdmFwd)) + gmin * vbd_jct;
          }
          break;
        default: {
          double evbd, devbd_dvb;
          if (vbd_jct < P(vjdmRev)) {
            T0 = vbd_jct / Nvtmd;
            if (T0 < -CONSTEXP_THRESHOLD) {
              evbd = CONSTMIN_EXP;
              devbd_dvb = 0.0;
            } else {
              evbd = exp(T0);
              devbd_dvb = evbd / Nvtmd;
            }
            T1 = evbd - 1.0;
            T2 = P(IVjdmRev) + P(DslpRev) * (vbd_jct - P(vjdmRev));
            gbd = devbd_dvb * T2 + T1 * P(DslpRev) + gmin;
            cbd = T1 * T2 + gmin * vbd_jct;
          } else if (vbd_jct <= P(vjdmFwd)) {
            T0 = vbd_jct / Nvtmd;
            if (T0 < -CONSTEXP_THRESHOLD) {
              evbd = CONSTMIN_EXP;
              devbd_dvb = 0.0;
            } else {
              evbd = exp(T0);
              devbd_dvb = evbd / Nvtmd;
            }
            T1 = (P(bvd) + vbd_jct) / Nvtmd;
            if (T1 > CONSTEXP_THRESHOLD) {
              T2 = CONSTMIN_EXP;
              T3 = 0.0;
            } else {
              T2 = exp(-T1);
              T3 = -T2 / Nvtmd;
            }
            gbd = DrainSatCurrent * (devbd_dvb - P(xjbvd) * T3) + gmin;
            cbd = DrainSatCurrent * (evbd + P(XExpBVD) - 1.0 - P(xjbvd) * T2) + gmin * vbd_jct;
          } else {
            gbd = P(DslpFwd) + gmin;
            cbd = P(IVjdmFwd) + P(DslpFwd) * (vbd_jct - P(vjdmFwd)) + gmin * vbd_jct;
          }
          break;
        }
      }
    }
  }

  // Trap-assisted tunnelling and recombination for reverse bias (:8661-8760).
  {
    const double vtm0 = P(vtm0);
    const double Nvtmrssws = vtm0 * P(njtsswstemp);
    const double Nvtmrsswgs = vtm0 * P(njtsswgstemp);
    const double Nvtmrss = vtm0 * P(njtsstemp);
    const double Nvtmrsswd = vtm0 * P(njtsswdtemp);
    const double Nvtmrsswgd = vtm0 * P(njtsswgdtemp);
    const double Nvtmrsd = vtm0 * P(njtsdtemp);
    double e1, e2, e3, e4, e5, e6, d1, d2, d3, d4, d5, d6;
    const double vtss = P(vtss), vtsd = P(vtsd), vtssws = P(vtssws), vtsswd = P(vtsswd), vtsswgs = P(vtsswgs),
                 vtsswgd = P(vtsswgd);
    if ((vtss - vbs_jct) < (vtss * 1e-3)) {
      T9 = 1.0e3; T0 = -vbs_jct / Nvtmrss * T9; dexp(T0, e1, T10); d1 = T10 / Nvtmrss * T9;
    } else {
      T9 = 1.0 / (vtss - vbs_jct); T0 = -vbs_jct / Nvtmrss * vtss * T9;
      dT0_dVb = vtss / Nvtmrss * (T9 + vbs_jct * T9 * T9); dexp(T0, e1, T10); d1 = T10 * dT0_dVb;
    }
    if ((vtsd - vbd_jct) < (vtsd * 1e-3)) {
      T9 = 1.0e3; T0 = -vbd_jct / Nvtmrsd * T9; dexp(T0, e2, T10); d2 = T10 / Nvtmrsd * T9;
    } else {
      T9 = 1.0 / (vtsd - vbd_jct); T0 = -vbd_jct / Nvtmrsd * vtsd * T9;
      dT0_dVb = vtsd / Nvtmrsd * (T9 + vbd_jct * T9 * T9); dexp(T0, e2, T10); d2 = T10 * dT0_dVb;
    }
    if ((vtssws - vbs_jct) < (vtssws * 1e-3)) {
      T9 = 1.0e3; T0 = -vbs_jct / Nvtmrssws * T9; dexp(T0, e3, T10); d3 = T10 / Nvtmrssws * T9;
    } else {
      T9 = 1.0 / (vtssws - vbs_jct); T0 = -vbs_jct / Nvtmrssws * vtssws * T9;
      dT0_dVb = vtssws / Nvtmrssws * (T9 + vbs_jct * T9 * T9); dexp(T0, e3, T10); d3 = T10 * dT0_dVb;
    }
    if ((vtsswd - vbd_jct) < (vtsswd * 1e-3)) {
      T9 = 1.0e3; T0 = -vbd_jct / Nvtmrsswd * T9; dexp(T0, e4, T10); d4 = T10 / Nvtmrsswd * T9;
    } else {
      T9 = 1.0 / (vtsswd - vbd_jct); T0 = -vbd_jct / Nvtmrsswd * vtsswd * T9;
      dT0_dVb = vtsswd / Nvtmrsswd * (T9 + vbd_jct * T9 * T9); dexp(T0, e4, T10); d4 = T10 * dT0_dVb;
    }
    if ((vtsswgs - vbs_jct) < (vtsswgs * 1e-3)) {
      T9 = 1.0e3; T0 = -vbs_jct / Nvtmrsswgs * T9; dexp(T0, e5, T10); d5 = T10 / Nvtmrsswgs * T9;
    } else {
      T9 = 1.0 / (vtsswgs - vbs_jct); T0 = -vbs_jct / Nvtmrsswgs * vtsswgs * T9;
      dT0_dVb = vtsswgs / Nvtmrsswgs * (T9 + vbs_jct * T9 * T9); dexp(T0, e5, T10); d5 = T10 * dT0_dVb;
    }
    if ((vtsswgd - vbd_jct) < (vtsswgd * 1e-3)) {
      T9 = 1.0e3; T0 = -vbd_jct / Nvtmrsswgd * T9; dexp(T0, e6, T10); d6 = T10 / Nvtmrsswgd * T9;
    } else {
      T9 = 1.0 / (vtsswgd - vbd_jct); T0 = -vbd_jct / Nvtmrsswgd * vtsswgd * T9;
      dT0_dVb = vtsswgd / Nvtmrsswgd * (T9 + vbd_jct * T9 * T9); dexp(T0, e6, T10); d6 = T10 * dT0_dVb;
    }
    gbs += P(SjctTempRevSatCur) * d1 + P(SswTempRevSatCur) * d3 + P(SswgTempRevSatCur) * d5;
    cbs -= P(SjctTempRevSatCur) * (e1 - 1.0) + P(SswTempRevSatCur) * (e3 - 1.0) + P(SswgTempRevSatCur) * (e5 - 1.0);
    gbd += P(DjctTempRevSatCur) * d2 + P(DswTempRevSatCur) * d4 + P(DswgTempRevSatCur) * d6;
    cbd -= P(DjctTempRevSatCur) * (e2 - 1.0) + P(DswTempRevSatCur) * (e4 - 1.0) + P(DswgTempRevSatCur) * (e6 - 1.0);
  }

  // Operating mode (:8761-8780).
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
  (void)Vgs;
  const double epsrox = P(epsrox_m);
  const double toxe = P(toxe_m);
  const double epssub = CONSTEPSSI;
  (void)epsrox;

  // Effective body bias, threshold voltage (:8819-9030).
  const double vbsc = P(vbsc);
  double Vbseff, dVbseff_dVb;
  T0 = Vbs - vbsc - 0.001;
  T1 = sqrt(T0 * T0 - 0.004 * vbsc);
  if (T0 >= 0.0) {
    Vbseff = vbsc + 0.5 * (T0 + T1);
    dVbseff_dVb = 0.5 * (1.0 + T0 / T1);
  } else {
    T2 = -0.002 / (T1 - T0);
    Vbseff = vbsc * (1.0 + T2);
    dVbseff_dVb = T2 * vbsc / T1;
  }
  const double phi = P(phi), sqrtPhi_p = P(sqrtPhi);
  T9 = 0.95 * phi;
  T0 = T9 - Vbseff - 0.001;
  T1 = sqrt(T0 * T0 + 0.004 * T9);
  Vbseff = T9 - 0.5 * (T0 + T1);
  dVbseff_dVb *= 0.5 * (1.0 + T0 / T1);
  const double Phis = phi - Vbseff;
  const double dPhis_dVb = -1.0;
  const double sqrtPhis = sqrt(Phis);
  const double dsqrtPhis_dVb = -0.5 / sqrtPhis;
  const double Xdep = P(Xdep0) * sqrtPhis / sqrtPhi_p;
  const double dXdep_dVb = (P(Xdep0) / sqrtPhi_p) * dsqrtPhis_dVb;
  const double Leff = P(leff);
  const double Vtm = P(vtm);
  const double Vtm0 = P(vtm0);
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
  const double factor1 = P(factor1);
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
  T0 = P(dvt1) * Leff / lt1;
  if (T0 < CONSTEXP_THRESHOLD) {
    T1 = exp(T0);
    T2 = T1 - 1.0;
    T3 = T2 * T2;
    T4 = T3 + 2.0 * T1 * CONSTMIN_EXP;
    Theta0 = T1 / T4;
    dT1_dVb = -T0 * T1 * dlt1_dVb / lt1;
    dTheta0_dVb = dT1_dVb * (T4 - 2.0 * T1 * (T2 + CONSTMIN_EXP)) / T4 / T4;
  } else {
    Theta0 = 1.0 / (CONSTMAX_EXP - 2.0);
    dTheta0_dVb = 0.0;
  }
  const double thetavth = P(dvt0) * Theta0;
  const double Delt_vth = thetavth * V0;
  const double dDelt_vth_dVb = P(dvt0) * dTheta0_dVb * V0;
  T0 = P(dvt1w) * P(weff) * Leff / ltw;
  if (T0 < CONSTEXP_THRESHOLD) {
    T1 = exp(T0);
    T2 = T1 - 1.0;
    T3 = T2 * T2;
    T4 = T3 + 2.0 * T1 * CONSTMIN_EXP;
    T5 = T1 / T4;
    dT1_dVb = -T0 * T1 * dltw_dVb / ltw;
    dT5_dVb = dT1_dVb * (T4 - 2.0 * T1 * (T2 + CONSTMIN_EXP)) / T4 / T4;
  } else {
    T5 = 1.0 / (CONSTMAX_EXP - 2.0);
    dT5_dVb = 0.0;
  }
  T0 = P(dvt0w) * T5;
  T2 = T0 * V0;
  dT2_dVb = P(dvt0w) * dT5_dVb * V0;
  const double TempRatio = P(temp) / P(tnom) - 1.0;
  T0 = sqrt(1.0 + P(lpe0) / Leff);
  const double k1ox = P(k1ox);
  T1 = k1ox * (T0 - 1.0) * sqrtPhi_p + (P(kt1) + P(kt1l) / Leff + P(kt2) * Vbseff) * TempRatio;
  const double Vth_NarrowW = toxe * phi / (P(weff) + P(w0));
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
  const double Lpe_Vb = sqrt(1.0 + P(lpeb) / Leff);
  const double k2ox = P(k2ox);
  double Vth = dtype * vth0 + (k1ox * sqrtPhis - P(k1) * sqrtPhi_p) * Lpe_Vb - k2ox * Vbseff - Delt_vth - T2 +
               (P(k3) + P(k3b) * Vbseff) * Vth_NarrowW + T1 - DIBL_Sft;
  double dVth_dVb = Lpe_Vb * k1ox * dsqrtPhis_dVb - k2ox - dDelt_vth_dVb - dT2_dVb + P(k3b) * Vth_NarrowW -
                    P(etab) * Vds * P(theta0vb0) * T4 + P(kt2) * TempRatio;
  double dVth_dVd = -dDIBL_Sft_dVd;
  const double coxe = P(coxe);
  tmp1 = epssub / Xdep;
  tmp2 = P(nfactor) * tmp1;
  tmp3 = P(cdsc) + P(cdscb) * Vbseff + P(cdscd) * Vds;
  tmp4 = (tmp2 + tmp3 * Theta0 + P(cit)) / coxe;
  double n, dn_dVb, dn_dVd;
  if (tmp4 >= -0.5) {
    n = 1.0 + tmp4;
    dn_dVb = (-tmp2 / Xdep * dXdep_dVb + tmp3 * dTheta0_dVb + P(cdscb) * Theta0) / coxe;
    dn_dVd = P(cdscd) * Theta0 / coxe;
  } else {
    T0 = 1.0 / (3.0 + 8.0 * tmp4);
    n = (1.0 + 3.0 * tmp4) * T0;
    T0 *= T0;
    dn_dVb = (-tmp2 / Xdep * dXdep_dVb + tmp3 * dTheta0_dVb + P(cdscb) * Theta0) / coxe * T0;
    dn_dVd = P(cdscd) * Theta0 / coxe * T0;
  }
  if (P(dvtp0) > 0.0) {
    T0 = -P(dvtp1) * Vds;
    if (T0 < -CONSTEXP_THRESHOLD) {
      T2 = CONSTMIN_EXP;
      dT2_dVd = 0.0;
    } else {
      T2 = exp(T0);
      dT2_dVd = -P(dvtp1) * T2;
    }
    T3 = Leff + P(dvtp0) * (1.0 + T2);
    dT3_dVd = P(dvtp0) * dT2_dVd;
    if (tempMod < 2) {
      T4 = Vtm * log(Leff / T3);
      dT4_dVd = -Vtm * dT3_dVd / T3;
    } else {
      T4 = Vtm0 * log(Leff / T3);
      dT4_dVd = -Vtm0 * dT3_dVd / T3;
    }
    const double dDITS_Sft_dVd = dn_dVd * T4 + n * dT4_dVd;
    const double dDITS_Sft_dVb = T4 * dn_dVb;
    Vth -= n * T4;
    dVth_dVd -= dDITS_Sft_dVd;
    dVth_dVb -= dDITS_Sft_dVb;
  }
  const double von = Vth;

  // Poly-gate depletion (:9033-9060).
  double vgs_eff, dvgs_eff_dvg, vgd_eff, dvgd_eff_dvg;
  T0 = P(vfb) + phi;
  T1 = CONSTEPSSI;
  poly_depletion(T0, P(ngate), T1, coxe, vgs, vgs_eff, dvgs_eff_dvg);
  poly_depletion(T0, P(ngate), T1, coxe, vgd, vgd_eff, dvgd_eff_dvg);
  double Vgs_eff, dVgs_eff_dVg;
  if (mode > 0) {
    Vgs_eff = vgs_eff;
    dVgs_eff_dVg = dvgs_eff_dvg;
  } else {
    Vgs_eff = vgd_eff;
    dVgs_eff_dVg = dvgd_eff_dvg;
  }
  const double Vgst = Vgs_eff - Vth;

  // Effective gate overdrive Vgsteff (:9061-9150).
  const double mstar = P(mstar);
  T0 = n * Vtm;
  T1 = mstar * Vgst;
  T2 = T1 / T0;
  if (T2 > CONSTEXP_THRESHOLD) {
    T10 = T1;
    dT10_dVg = mstar * dVgs_eff_dVg;
    dT10_dVd = -dVth_dVd * mstar;
    dT10_dVb = -dVth_dVb * mstar;
  } else if (T2 < -CONSTEXP_THRESHOLD) {
    T10 = Vtm * log(1.0 + CONSTMIN_EXP);
    dT10_dVg = 0.0;
    dT10_dVd = T10 * dn_dVd;
    dT10_dVb = T10 * dn_dVb;
    T10 *= n;
  } else {
    const double ExpVgst = exp(T2);
    T3 = Vtm * log(1.0 + ExpVgst);
    T10 = n * T3;
    dT10_dVg = mstar * ExpVgst / (1.0 + ExpVgst);
    dT10_dVb = T3 * dn_dVb - dT10_dVg * (dVth_dVb + Vgst * dn_dVb / n);
    dT10_dVd = T3 * dn_dVd - dT10_dVg * (dVth_dVd + Vgst * dn_dVd / n);
    dT10_dVg *= dVgs_eff_dVg;
  }
  T1 = P(voffcbn) - (1.0 - mstar) * Vgst;
  T2 = T1 / T0;
  if (T2 < -CONSTEXP_THRESHOLD) {
    T3 = coxe * CONSTMIN_EXP / P(cdep0);
    T9 = mstar + T3 * n;
    dT9_dVg = 0.0;
    dT9_dVd = dn_dVd * T3;
    dT9_dVb = dn_dVb * T3;
  } else if (T2 > CONSTEXP_THRESHOLD) {
    T3 = coxe * CONSTMAX_EXP / P(cdep0);
    T9 = mstar + T3 * n;
    dT9_dVg = 0.0;
    dT9_dVd = dn_dVd * T3;
    dT9_dVb = dn_dVb * T3;
  } else {
    const double ExpVgst = exp(T2);
    T3 = coxe / P(cdep0);
    T4 = T3 * ExpVgst;
    T5 = T1 * T4 / T0;
    T9 = mstar + n * T4;
    dT9_dVg = T3 * (mstar - 1.0) * ExpVgst / Vtm;
    dT9_dVb = T4 * dn_dVb - dT9_dVg * dVth_dVb - T5 * dn_dVb;
    dT9_dVd = T4 * dn_dVd - dT9_dVg * dVth_dVd - T5 * dn_dVd;
    dT9_dVg *= dVgs_eff_dVg;
  }
  double Vgsteff = T10 / T9;
  T11 = T9 * T9;
  double dVgsteff_dVg = (T9 * dT10_dVg - T10 * dT9_dVg) / T11;
  double dVgsteff_dVd = (T9 * dT10_dVd - T10 * dT9_dVd) / T11;
  double dVgsteff_dVb = (T9 * dT10_dVb - T10 * dT9_dVb) / T11;

  // Effective width and source/drain series resistance (:9155-9200).
  T9 = sqrtPhis - sqrtPhi_p;
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
  if (rdsMod) {
    Rds = dRds_dVg = dRds_dVb = 0.0;
  } else {
    T0 = 1.0 + P(prwg) * Vgsteff;
    dT0_dVg = -P(prwg) / T0 / T0;
    T1 = P(prwb) * T9;
    dT1_dVb = P(prwb) * dsqrtPhis_dVb;
    T2 = 1.0 / T0 + T1;
    T3 = T2 + sqrt(T2 * T2 + 0.01);
    dT3_dVg = 1.0 + T2 / (T3 - T2);
    dT3_dVb = dT3_dVg * dT1_dVb;
    dT3_dVg *= dT0_dVg;
    T4 = P(rds0) * 0.5;
    Rds = P(rdswmin) + T3 * T4;
    dRds_dVg = T4 * dT3_dVg;
    dRds_dVb = T4 * dT3_dVb;
  }

  // Bulk charge factor Abulk (:9201-9260).
  T9 = 0.5 * k1ox * Lpe_Vb / sqrtPhis;
  T1 = T9 + k2ox - P(k3b) * Vth_NarrowW;
  dT1_dVb = -T9 / sqrtPhis * dsqrtPhis_dVb;
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

  // Mobility (:9261-9340).
  T14 = 0.0;
  double Denomi, dDenomi_dVg, dDenomi_dVd, dDenomi_dVb;
  if (mobMod == 0) {
    T0 = Vgsteff + Vth + Vth - T14;
    T2 = P(ua) + P(uc) * Vbseff;
    T3 = T0 / toxe;
    T12 = sqrt(Vth * Vth + 0.0001);
    T9 = 1.0 / (Vgsteff + 2 * T12);
    T10 = T9 * toxe;
    T8 = P(ud) * T10 * T10 * Vth;
    T6 = T8 * Vth;
    T5 = T3 * (T2 + P(ub) * T3) + T6;
    T7 = -2.0 * T6 * T9;
    T11 = T7 * Vth / T12;
    dDenomi_dVg = (T2 + 2.0 * P(ub) * T3) / toxe;
    T13 = 2.0 * (dDenomi_dVg + T11 + T8);
    dDenomi_dVd = T13 * dVth_dVd;
    dDenomi_dVb = T13 * dVth_dVb + P(uc) * T3;
    dDenomi_dVg += T7;
  } else if (mobMod == 1) {
    T0 = Vgsteff + Vth + Vth - T14;
    T2 = 1.0 + P(uc) * Vbseff;
    T3 = T0 / toxe;
    T4 = T3 * (P(ua) + P(ub) * T3);
    T12 = sqrt(Vth * Vth + 0.0001);
    T9 = 1.0 / (Vgsteff + 2 * T12);
    T10 = T9 * toxe;
    T8 = P(ud) * T10 * T10 * Vth;
    T6 = T8 * Vth;
    T5 = T4 * T2 + T6;
    T7 = -2.0 * T6 * T9;
    T11 = T7 * Vth / T12;
    dDenomi_dVg = (P(ua) + 2.0 * P(ub) * T3) * T2 / toxe;
    T13 = 2.0 * (dDenomi_dVg + T11 + T8);
    dDenomi_dVd = T13 * dVth_dVd;
    dDenomi_dVb = T13 * dVth_dVb + P(uc) * T4;
    dDenomi_dVg += T7;
  } else {
    T0 = (Vgsteff + P(vtfbphi1)) / toxe;
    T1 = exp(P(eu) * log(T0));
    dT1_dVg = T1 * P(eu) / T0 / toxe;
    T2 = P(ua) + P(uc) * Vbseff;
    T3 = T0 / toxe;
    T12 = sqrt(Vth * Vth + 0.0001);
    T9 = 1.0 / (Vgsteff + 2 * T12);
    T10 = T9 * toxe;
    T8 = P(ud) * T10 * T10 * Vth;
    T6 = T8 * Vth;
    T5 = T1 * T2 + T6;
    T7 = -2.0 * T6 * T9;
    T11 = T7 * Vth / T12;
    dDenomi_dVg = T2 * dT1_dVg + T7;
    T13 = 2.0 * (T11 + T8);
    dDenomi_dVd = T13 * dVth_dVd;
    dDenomi_dVb = T13 * dVth_dVb + T1 * P(uc);
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

  // Saturation velocity, Vdsat (:9341-9460).
  const double vsattemp = P(vsattemp);
  const double WVCox = Weff * vsattemp * coxe;
  const double WVCoxRds = WVCox * Rds;
  const double Esat = 2.0 * vsattemp / ueff;
  double EsatL = Esat * Leff;
  T0 = -EsatL / ueff;
  double dEsatL_dVg = T0 * dueff_dVg;
  double dEsatL_dVd = T0 * dueff_dVd;
  double dEsatL_dVb = T0 * dueff_dVb;
  const double a1 = P(a1);
  double Lambda, dLambda_dVg;
  if (a1 == 0.0) {
    Lambda = P(a2);
    dLambda_dVg = 0.0;
  } else if (a1 > 0.0) {
    T0 = 1.0 - P(a2);
    T1 = T0 - a1 * Vgsteff - 0.0001;
    T2 = sqrt(T1 * T1 + 0.0004 * T0);
    Lambda = P(a2) + T0 - 0.5 * (T1 + T2);
    dLambda_dVg = 0.5 * a1 * (1.0 + T1 / T2);
  } else {
    T1 = P(a2) + a1 * Vgsteff - 0.0001;
    T2 = sqrt(T1 * T1 + 0.0004 * P(a2));
    Lambda = 0.5 * (T1 + T2);
    dLambda_dVg = 0.5 * a1 * (1.0 + T1 / T2);
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
    dVdsat_dVg = (dT1_dVg - (T1 * dT1_dVg - dT0_dVg * T2 - T0 * dT2_dVg) / T3 - Vdsat * dT0_dVg) / T0;
    dVdsat_dVb = (dT1_dVb - (T1 * dT1_dVb - dT0_dVb * T2 - T0 * dT2_dVb) / T3 - Vdsat * dT0_dVb) / T0;
    dVdsat_dVd = (dT1_dVd - (T1 * dT1_dVd - T0 * dT2_dVd) / T3) / T0;
  }

  // Effective Vds (:9461-9500).
  const double delta = P(delta);
  T1 = Vdsat - Vds - delta;
  dT1_dVg = dVdsat_dVg;
  dT1_dVd = dVdsat_dVd - 1.0;
  dT1_dVb = dVdsat_dVb;
  T2 = sqrt(T1 * T1 + 4.0 * delta * Vdsat);
  T0 = T1 / T2;
  T9 = 2.0 * delta;
  T3 = T9 / T2;
  dT2_dVg = T0 * dT1_dVg + T3 * dVdsat_dVg;
  dT2_dVd = T0 * dT1_dVd + T3 * dVdsat_dVd;
  dT2_dVb = T0 * dT1_dVb + T3 * dVdsat_dVb;
  double Vdseff, dVdseff_dVg, dVdseff_dVd, dVdseff_dVb;
  if (T1 >= 0.0) {
    Vdseff = Vdsat - 0.5 * (T1 + T2);
    dVdseff_dVg = dVdsat_dVg - 0.5 * (dT1_dVg + dT2_dVg);
    dVdseff_dVd = dVdsat_dVd - 0.5 * (dT1_dVd + dT2_dVd);
    dVdseff_dVb = dVdsat_dVb - 0.5 * (dT1_dVb + dT2_dVb);
  } else {
    T4 = T9 / (T2 - T1);
    T5 = 1.0 - T4;
    T6 = Vdsat * T4 / (T2 - T1);
    Vdseff = Vdsat * T5;
    dVdseff_dVg = dVdsat_dVg * T5 + T6 * (dT2_dVg - dT1_dVg);
    dVdseff_dVd = dVdsat_dVd * T5 + T6 * (dT2_dVd - dT1_dVd);
    dVdseff_dVb = dVdsat_dVb * T5 + T6 * (dT2_dVb - dT1_dVb);
  }
  if (Vds == 0.0) {
    Vdseff = 0.0;
    dVdseff_dVg = 0.0;
    dVdseff_dVb = 0.0;
  }
  if (Vdseff > Vds) Vdseff = Vds;
  const double diffVds = Vds - Vdseff;

  // Velocity overshoot (lambda) (:9501-9545).
  if ((P(lambdaGiven) != 0.0) && (P(lambda_m) > 0.0)) {
    T1 = Leff * ueff;
    T2 = P(lambda) / T1;
    T3 = -T2 / T1 * Leff;
    dT2_dVd = T3 * dueff_dVd;
    dT2_dVg = T3 * dueff_dVg;
    dT2_dVb = T3 * dueff_dVb;
    T5 = 1.0 / (Esat * P(litl));
    T4 = -T5 / EsatL;
    dT5_dVg = dEsatL_dVg * T4;
    dT5_dVd = dEsatL_dVd * T4;
    dT5_dVb = dEsatL_dVb * T4;
    T6 = 1.0 + diffVds * T5;
    dT6_dVg = dT5_dVg * diffVds - dVdseff_dVg * T5;
    dT6_dVd = dT5_dVd * diffVds + (1.0 - dVdseff_dVd) * T5;
    dT6_dVb = dT5_dVb * diffVds - dVdseff_dVb * T5;
    T7 = 2.0 / (T6 * T6 + 1.0);
    T8 = 1.0 - T7;
    T9 = T6 * T7 * T7;
    dT8_dVg = T9 * dT6_dVg;
    dT8_dVd = T9 * dT6_dVd;
    dT8_dVb = T9 * dT6_dVb;
    T10 = 1.0 + T2 * T8;
    dT10_dVg = dT2_dVg * T8 + T2 * dT8_dVg;
    dT10_dVd = dT2_dVd * T8 + T2 * dT8_dVd;
    dT10_dVb = dT2_dVb * T8 + T2 * dT8_dVb;
    if (T10 == 1.0) dT10_dVg = dT10_dVd = dT10_dVb = 0.0;
    dEsatL_dVg *= T10;
    dEsatL_dVg += EsatL * dT10_dVg;
    dEsatL_dVd *= T10;
    dEsatL_dVd += EsatL * dT10_dVd;
    dEsatL_dVb *= T10;
    dEsatL_dVb += EsatL * dT10_dVb;
    EsatL *= T10;
  }

  // Vasat (:9546-9565).
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

  // Quantum-mechanical effective oxide capacitance and beta (:9566-9590).
  tmp1 = P(vtfbphi2);
  tmp2 = 2.0e8 * P(toxp);
  dT0_dVg = 1.0 / tmp2;
  T0 = (Vgsteff + tmp1) * dT0_dVg;
  tmp3 = exp(P(bdos) * 0.7 * log(T0));
  T1 = 1.0 + tmp3;
  T2 = P(bdos) * 0.7 * tmp3 / T0;
  double Tcen = P(ados) * 1.9e-9 / T1;
  double dTcen_dVg = -Tcen * T2 * dT0_dVg / T1;
  const double coxp = P(coxp);
  double Coxeff = epssub * coxp / (epssub + coxp * Tcen);
  double dCoxeff_dVg = -Coxeff * Coxeff * dTcen_dVg / epssub;
  const double CoxeffWovL = Coxeff * Weff / Leff;
  const double beta = ueff * CoxeffWovL;
  T3 = ueff / Leff;
  const double dbeta_dVg = CoxeffWovL * dueff_dVg + T3 * (Weff * dCoxeff_dVg + Coxeff * dWeff_dVg);
  const double dbeta_dVd = CoxeffWovL * dueff_dVd;
  const double dbeta_dVb = CoxeffWovL * dueff_dVb + T3 * Coxeff * dWeff_dVb;
  (void)dbeta_dVd; (void)dbeta_dVb;

  // Linear-region current Idl (:9591-9640).
  const double AbovVgst2Vtm = Abulk / Vgst2Vtm;
  T0 = 1.0 - 0.5 * Vdseff * AbovVgst2Vtm;
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
  const double Idl = gche / T0;
  T1 = (1.0 - Idl * Rds) / T0;
  T2 = Idl * Idl;
  const double dIdl_dVg = T1 * dgche_dVg - T2 * dRds_dVg;
  const double dIdl_dVd = T1 * dgche_dVd;
  const double dIdl_dVb = T1 * dgche_dVb - T2 * dRds_dVb;

  // Output resistance terms: FP, PvagTerm, CLM, DIBL, DITS, SCBE (:9641-9800).
  double FP, dFP_dVg;
  if (P(fprout) <= 0.0) {
    FP = 1.0;
    dFP_dVg = 0.0;
  } else {
    T9 = P(fprout) * sqrt(Leff) / Vgst2Vtm;
    FP = 1.0 / (1.0 + T9);
    dFP_dVg = FP * FP * T9 / Vgst2Vtm;
  }
  double PvagTerm, dPvagTerm_dVg, dPvagTerm_dVb, dPvagTerm_dVd;
  T8 = P(pvag) / EsatL;
  T9 = T8 * Vgsteff;
  if (T9 > -0.9) {
    PvagTerm = 1.0 + T9;
    dPvagTerm_dVg = T8 * (1.0 - Vgsteff * dEsatL_dVg / EsatL);
    dPvagTerm_dVb = -T9 * dEsatL_dVb / EsatL;
    dPvagTerm_dVd = -T9 * dEsatL_dVd / EsatL;
  } else {
    T4 = 1.0 / (17.0 + 20.0 * T9);
    PvagTerm = (0.8 + T9) * T4;
    T4 *= T4;
    dPvagTerm_dVg = T8 * (1.0 - Vgsteff * dEsatL_dVg / EsatL) * T4;
    T9 *= T4 / EsatL;
    dPvagTerm_dVb = -T9 * dEsatL_dVb;
    dPvagTerm_dVd = -T9 * dEsatL_dVd;
  }
  double Cclm, dCclm_dVg, dCclm_dVd, dCclm_dVb, VACLM, dVACLM_dVg, dVACLM_dVd, dVACLM_dVb;
  if ((P(pclm) > CONSTMIN_EXP) && (diffVds > 1.0e-10)) {
    T0 = 1.0 + Rds * Idl;
    dT0_dVg = dRds_dVg * Idl + Rds * dIdl_dVg;
    dT0_dVd = Rds * dIdl_dVd;
    dT0_dVb = dRds_dVb * Idl + Rds * dIdl_dVb;
    T2 = Vdsat / Esat;
    T1 = Leff + T2;
    dT1_dVg = (dVdsat_dVg - T2 * dEsatL_dVg / Leff) / Esat;
    dT1_dVd = (dVdsat_dVd - T2 * dEsatL_dVd / Leff) / Esat;
    dT1_dVb = (dVdsat_dVb - T2 * dEsatL_dVb / Leff) / Esat;
    Cclm = FP * PvagTerm * T0 * T1 / (P(pclm) * P(litl));
    dCclm_dVg = Cclm * (dFP_dVg / FP + dPvagTerm_dVg / PvagTerm + dT0_dVg / T0 + dT1_dVg / T1);
    dCclm_dVb = Cclm * (dPvagTerm_dVb / PvagTerm + dT0_dVb / T0 + dT1_dVb / T1);
    dCclm_dVd = Cclm * (dPvagTerm_dVd / PvagTerm + dT0_dVd / T0 + dT1_dVd / T1);
    VACLM = Cclm * diffVds;
    dVACLM_dVg = dCclm_dVg * diffVds - dVdseff_dVg * Cclm;
    dVACLM_dVb = dCclm_dVb * diffVds - dVdseff_dVb * Cclm;
    dVACLM_dVd = dCclm_dVd * diffVds + (1.0 - dVdseff_dVd) * Cclm;
  } else {
    VACLM = Cclm = CONSTMAX_EXP;
    dVACLM_dVd = dVACLM_dVg = dVACLM_dVb = 0.0;
    dCclm_dVd = dCclm_dVg = dCclm_dVb = 0.0;
  }
  double VADIBL, dVADIBL_dVg, dVADIBL_dVd, dVADIBL_dVb;
  if (P(thetaRout) > CONSTMIN_EXP) {
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
    dVADIBL_dVg = dVADIBL_dVg * PvagTerm + VADIBL * dPvagTerm_dVg;
    dVADIBL_dVb = dVADIBL_dVb * PvagTerm + VADIBL * dPvagTerm_dVb;
    dVADIBL_dVd = dVADIBL_dVd * PvagTerm + VADIBL * dPvagTerm_dVd;
    VADIBL *= PvagTerm;
  } else {
    VADIBL = CONSTMAX_EXP;
    dVADIBL_dVd = dVADIBL_dVg = dVADIBL_dVb = 0.0;
  }
  const double Va = Vasat + VACLM;
  const double dVa_dVg = dVasat_dVg + dVACLM_dVg;
  const double dVa_dVb = dVasat_dVb + dVACLM_dVb;
  const double dVa_dVd = dVasat_dVd + dVACLM_dVd;
  T0 = P(pditsd) * Vds;
  if (T0 > CONSTEXP_THRESHOLD) {
    T1 = CONSTMAX_EXP;
    dT1_dVd = 0;
  } else {
    T1 = exp(T0);
    dT1_dVd = T1 * P(pditsd);
  }
  double VADITS, dVADITS_dVg, dVADITS_dVd;
  if (P(pdits) > CONSTMIN_EXP) {
    T2 = 1.0 + P(pditsl) * Leff;
    VADITS = (1.0 + T2 * T1) / P(pdits);
    dVADITS_dVg = VADITS * dFP_dVg;
    dVADITS_dVd = FP * T2 * dT1_dVd / P(pdits);
    VADITS *= FP;
  } else {
    VADITS = CONSTMAX_EXP;
    dVADITS_dVg = dVADITS_dVd = 0;
  }
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

  // Drain current with CLM, DIBL, DITS, SCBE (:9801-9870).
  T9 = diffVds / VADIBL;
  T0 = 1.0 + T9;
  double Idsa = Idl * T0;
  double dIdsa_dVg = T0 * dIdl_dVg - Idl * (dVdseff_dVg + T9 * dVADIBL_dVg) / VADIBL;
  double dIdsa_dVd = T0 * dIdl_dVd + Idl * (1.0 - dVdseff_dVd - T9 * dVADIBL_dVd) / VADIBL;
  double dIdsa_dVb = T0 * dIdl_dVb - Idl * (dVdseff_dVb + T9 * dVADIBL_dVb) / VADIBL;
  T9 = diffVds / VADITS;
  T0 = 1.0 + T9;
  dIdsa_dVg = T0 * dIdsa_dVg - Idsa * (dVdseff_dVg + T9 * dVADITS_dVg) / VADITS;
  dIdsa_dVd = T0 * dIdsa_dVd + Idsa * (1.0 - dVdseff_dVd - T9 * dVADITS_dVd) / VADITS;
  dIdsa_dVb = T0 * dIdsa_dVb - Idsa * dVdseff_dVb / VADITS;
  Idsa *= T0;
  T0 = log(Va / Vasat);
  dT0_dVg = dVa_dVg / Va - dVasat_dVg / Vasat;
  dT0_dVb = dVa_dVb / Va - dVasat_dVb / Vasat;
  dT0_dVd = dVa_dVd / Va - dVasat_dVd / Vasat;
  T1 = T0 / Cclm;
  T9 = 1.0 + T1;
  dT9_dVg = (dT0_dVg - T1 * dCclm_dVg) / Cclm;
  dT9_dVb = (dT0_dVb - T1 * dCclm_dVb) / Cclm;
  dT9_dVd = (dT0_dVd - T1 * dCclm_dVd) / Cclm;
  dIdsa_dVg = dIdsa_dVg * T9 + Idsa * dT9_dVg;
  dIdsa_dVb = dIdsa_dVb * T9 + Idsa * dT9_dVb;
  dIdsa_dVd = dIdsa_dVd * T9 + Idsa * dT9_dVd;
  Idsa *= T9;

  // Substrate current (:9871-9910).
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
    T4 = Idsa * Vdseff;
    Isub = T1 * T4;
    Gbg = T1 * (dIdsa_dVg * Vdseff + Idsa * dVdseff_dVg) + T4 * dT1_dVg;
    Gbd = T1 * (dIdsa_dVd * Vdseff + Idsa * dVdseff_dVd) + T4 * dT1_dVd;
    Gbb = T1 * (dIdsa_dVb * Vdseff + Idsa * dVdseff_dVb) + T4 * dT1_dVb;
    Gbd += Gbg * dVgsteff_dVd;
    Gbb += Gbg * dVgsteff_dVb;
    Gbg *= dVgsteff_dVg;
    Gbb *= dVbseff_dVb;
  }
  double csub = Isub, gbbs = Gbb, gbgs = Gbg, gbds = Gbd;

  // Drain current and conductances (:9911-9990).
  T9 = diffVds / VASCBE;
  T0 = 1.0 + T9;
  const double Ids = Idsa * T0;
  double Gm = T0 * dIdsa_dVg - Idsa * (dVdseff_dVg + T9 * dVASCBE_dVg) / VASCBE;
  double Gds = T0 * dIdsa_dVd + Idsa * (1.0 - dVdseff_dVd - T9 * dVASCBE_dVd) / VASCBE;
  double Gmb = T0 * dIdsa_dVb - Idsa * (dVdseff_dVb + T9 * dVASCBE_dVb) / VASCBE;
  tmp1 = Gds + Gm * dVgsteff_dVd;
  tmp2 = Gmb + Gm * dVgsteff_dVb;
  tmp3 = Gm;
  Gm = (Ids * dVdseff_dVg + Vdseff * tmp3) * dVgsteff_dVg;
  Gds = Ids * (dVdseff_dVd + dVdseff_dVg * dVgsteff_dVd) + Vdseff * tmp1;
  Gmb = (Ids * (dVdseff_dVb + dVdseff_dVg * dVgsteff_dVb) + Vdseff * tmp2) * dVbseff_dVb;
  double cdrain = Ids * Vdseff;
  if ((P(vtlGiven) != 0.0) && (P(vtl_m) > 0.0)) {
    T12 = 1.0 / Leff / CoxeffWovL;
    T11 = T12 / Vgsteff;
    T10 = -T11 / Vgsteff;
    const double vs = cdrain * T11;
    const double dvs_dVg = Gm * T11 + cdrain * T10 * dVgsteff_dVg;
    const double dvs_dVd = Gds * T11 + cdrain * T10 * dVgsteff_dVd;
    const double dvs_dVb = Gmb * T11 + cdrain * T10 * dVgsteff_dVb;
    T0 = 2 * CONSTMM;
    T1 = vs / (P(vtl) * P(tfactor));
    double Fsevl, dFsevl_dVg, dFsevl_dVd, dFsevl_dVb;
    if (T1 > 0.0) {
      T2 = 1.0 + exp(T0 * log(T1));
      T3 = (T2 - 1.0) * T0 / vs;
      Fsevl = 1.0 / exp(log(T2) / T0);
      dT2_dVg = T3 * dvs_dVg;
      dT2_dVd = T3 * dvs_dVd;
      dT2_dVb = T3 * dvs_dVb;
      T4 = -1.0 / T0 * Fsevl / T2;
      dFsevl_dVg = T4 * dT2_dVg;
      dFsevl_dVd = T4 * dT2_dVd;
      dFsevl_dVb = T4 * dT2_dVb;
    } else {
      Fsevl = 1.0;
      dFsevl_dVg = 0.0;
      dFsevl_dVd = 0.0;
      dFsevl_dVb = 0.0;
    }
    Gm *= Fsevl;
    Gm += cdrain * dFsevl_dVg;
    Gmb *= Fsevl;
    Gmb += cdrain * dFsevl_dVb;
    Gds *= Fsevl;
    Gds += cdrain * dFsevl_dVd;
    cdrain *= Fsevl;
  }
  double gds = Gds, gm = Gm, gmbs = Gmb;

  // Gate resistance conductance for rgateMod 2 / 3 and the NQS time constant (:9954-9989).
  double gcrg = 0.0, gcrgg = 0.0, gcrgd = 0.0, gcrgs = 0.0, gcrgb = 0.0;
  if (GEN && (rgateMod > 1 || P(trnqsMod) != 0.0)) {
    T9 = P(xrcrg2) * P(vtm);
    T0 = T9 * beta;
    dT0_dVd = (dbeta_dVd + dbeta_dVg * dVgsteff_dVd) * T9;
    dT0_dVb = (dbeta_dVb + dbeta_dVg * dVgsteff_dVb) * T9;
    dT0_dVg = dbeta_dVg * T9;
    gcrg = P(xrcrg1) * (T0 + Ids);
    gcrgd = P(xrcrg1) * (dT0_dVd + tmp1);
    gcrgb = P(xrcrg1) * (dT0_dVb + tmp2) * dVbseff_dVb;
    gcrgg = P(xrcrg1) * (dT0_dVg + tmp3) * dVgsteff_dVg;
    if (nf != 1.0) {
      gcrg *= nf;
      gcrgg *= nf;
      gcrgd *= nf;
      gcrgb *= nf;
    }
    if (rgateMod == 2) {
      T10 = P(grgeltd) * P(grgeltd);
      T11 = P(grgeltd) + gcrg;
      gcrg = P(grgeltd) * gcrg / T11;
      T12 = T10 / T11 / T11;
      gcrgg *= T12;
      gcrgd *= T12;
      gcrgb *= T12;
    }
    gcrgs = -(gcrgg + gcrgd + gcrgb);
  }
  // Bias-dependent external source / drain resistance, rdsMod = 1 (:9991-10061). It replaces the
  // poly-depleted vgs_eff / vgd_eff that GIDL / GISL read below with the S/D-resistance ones, as the
  // reference's shared members do.
  double gstot = 0.0, gstotd = 0.0, gstotg = 0.0, gstots = 0.0, gstotb = 0.0;
  double gdtot = 0.0, gdtotd = 0.0, gdtotg = 0.0, gdtots = 0.0, gdtotb = 0.0;
  if (rdsMod) {
    T0 = vgs - P(vfbsd);
    T1 = sqrt(T0 * T0 + 1.0e-4);
    vgs_eff = 0.5 * (T0 + T1);
    dvgs_eff_dvg = vgs_eff / T1;
    T0 = 1.0 + P(prwg) * vgs_eff;
    double dT0_dvg = -P(prwg) / T0 / T0 * dvgs_eff_dvg;
    T1 = -P(prwb) * vbs;
    double dT1_dvb = -P(prwb);
    T2 = 1.0 / T0 + T1;
    T3 = T2 + sqrt(T2 * T2 + 0.01);
    double dT3_dvg = T3 / (T3 - T2);
    double dT3_dvb = dT3_dvg * dT1_dvb;
    dT3_dvg *= dT0_dvg;
    T4 = P(rs0) * 0.5;
    const double Rs = P(rswmin) + T3 * T4;
    const double dRs_dvg = T4 * dT3_dvg;
    const double dRs_dvb = T4 * dT3_dvb;
    T0 = 1.0 + P(sourceConductance) * Rs;
    gstot = P(sourceConductance) / T0;
    T0 = -gstot * gstot;
    const double dgstot_dvd = 0.0;
    const double dgstot_dvg = T0 * dRs_dvg;
    const double dgstot_dvb = T0 * dRs_dvb;
    const double dgstot_dvs = -(dgstot_dvg + dgstot_dvb + dgstot_dvd);
    T0 = vgd - P(vfbsd);
    T1 = sqrt(T0 * T0 + 1.0e-4);
    vgd_eff = 0.5 * (T0 + T1);
    dvgd_eff_dvg = vgd_eff / T1;
    T0 = 1.0 + P(prwg) * vgd_eff;
    dT0_dvg = -P(prwg) / T0 / T0 * dvgd_eff_dvg;
    T1 = -P(prwb) * vbd;
    dT1_dvb = -P(prwb);
    T2 = 1.0 / T0 + T1;
    T3 = T2 + sqrt(T2 * T2 + 0.01);
    dT3_dvg = T3 / (T3 - T2);
    dT3_dvb = dT3_dvg * dT1_dvb;
    dT3_dvg *= dT0_dvg;
    T4 = P(rd0) * 0.5;
    const double Rd = P(rdwmin) + T3 * T4;
    const double dRd_dvg = T4 * dT3_dvg;
    const double dRd_dvb = T4 * dT3_dvb;
    T0 = 1.0 + P(drainConductance) * Rd;
    gdtot = P(drainConductance) / T0;
    T0 = -gdtot * gdtot;
    const double dgdtot_dvs = 0.0;
    const double dgdtot_dvg = T0 * dRd_dvg;
    const double dgdtot_dvb = T0 * dRd_dvb;
    const double dgdtot_dvd = -(dgdtot_dvg + dgdtot_dvb + dgdtot_dvs);
    gstotd = vses * dgstot_dvd;
    gstotg = vses * dgstot_dvg;
    gstots = vses * dgstot_dvs;
    gstotb = vses * dgstot_dvb;
    T2 = vdes - vds;
    gdtotd = T2 * dgdtot_dvd;
    gdtotg = T2 * dgdtot_dvg;
    gdtots = T2 * dgdtot_dvs;
    gdtotb = T2 * dgdtot_dvb;
  }

  // GIDL and GISL (:10063-10180). vgs_eff / vgd_eff here are the poly-depleted gate voltages
  // (rdsMod 0) or the S/D-resistance ones (rdsMod 1).
  T0 = 3.0 * toxe;
  T1 = (vds - vgs_eff - P(egidl)) / T0;
  double Igidl, Ggidld, Ggidlg, Ggidlb;
  if ((P(agidl) <= 0.0) || (P(bgidl) <= 0.0) || (T1 <= 0.0) || (P(cgidl) <= 0.0) || (vbd > 0.0)) {
    Igidl = Ggidld = Ggidlg = Ggidlb = 0.0;
  } else {
    dT1_dVd = 1.0 / T0;
    dT1_dVg = -dvgs_eff_dvg * dT1_dVd;
    T2 = P(bgidl) / T1;
    if (T2 < 100.0) {
      Igidl = P(agidl) * weffCJ * T1 * exp(-T2);
      T3 = Igidl * (1.0 + T2) / T1;
      Ggidld = T3 * dT1_dVd;
      Ggidlg = T3 * dT1_dVg;
    } else {
      Igidl = P(agidl) * weffCJ * 3.720075976e-44;
      Ggidld = Igidl * dT1_dVd;
      Ggidlg = Igidl * dT1_dVg;
      Igidl *= T1;
    }
    T4 = vbd * vbd;
    T5 = -vbd * T4;
    T6 = P(cgidl) + T5;
    T7 = T5 / T6;
    T8 = 3.0 * P(cgidl) * T4 / T6 / T6;
    Ggidld = Ggidld * T7 + Igidl * T8;
    Ggidlg = Ggidlg * T7;
    Ggidlb = -Igidl * T8;
    Igidl *= T7;
  }
  double ggidld = Ggidld, ggidlg = Ggidlg, ggidlb = Ggidlb;
  T1 = (-vds - vgd_eff - P(egisl)) / T0;
  double Igisl, Ggisls, Ggislg, Ggislb;
  if ((P(agisl) <= 0.0) || (P(bgisl) <= 0.0) || (T1 <= 0.0) || (P(cgisl) <= 0.0) || (vbs > 0.0)) {
    Igisl = Ggisls = Ggislg = Ggislb = 0.0;
  } else {
    dT1_dVd = 1.0 / T0;
    dT1_dVg = -dvgd_eff_dvg * dT1_dVd;
    T2 = P(bgisl) / T1;
    if (T2 < 100.0) {
      Igisl = P(agisl) * weffCJ * T1 * exp(-T2);
      T3 = Igisl * (1.0 + T2) / T1;
      Ggisls = T3 * dT1_dVd;
      Ggislg = T3 * dT1_dVg;
    } else {
      Igisl = P(agisl) * weffCJ * 3.720075976e-44;
      Ggisls = Igisl * dT1_dVd;
      Ggislg = Igisl * dT1_dVg;
      Igisl *= T1;
    }
    T4 = vbs * vbs;
    T5 = -vbs * T4;
    T6 = P(cgisl) + T5;
    T7 = T5 / T6;
    T8 = 3.0 * P(cgisl) * T4 / T6 / T6;
    Ggisls = Ggisls * T7 + Igisl * T8;
    Ggislg = Ggislg * T7;
    Ggislb = -Igisl * T8;
    Igisl *= T7;
  }
  double ggisls = Ggisls, ggislg = Ggislg, ggislb = Ggislb;
  // Gate tunnelling currents (:10183-10600): gate to channel (igcMod, partitioned between source
  // and drain), gate to source / drain overlap (with igcMod) and gate to bulk (igbMod).
  const int igcMod = FULL ? (int)P(igcMod) : 0, igbMod = FULL ? (int)P(igbMod) : 0;
  double Igcs = 0.0, gIgcsg = 0.0, gIgcsd = 0.0, gIgcsb = 0.0;
  double Igcd = 0.0, gIgcdg = 0.0, gIgcdd = 0.0, gIgcdb = 0.0;
  double Igs = 0.0, gIgsg = 0.0, gIgss = 0.0, Igd = 0.0, gIgdg = 0.0, gIgdd = 0.0;
  double Igb = 0.0, gIgbg = 0.0, gIgbd = 0.0, gIgbb = 0.0;
  if (igcMod != 0 || igbMod != 0) {
    double Vfb_g = P(vfbzb);
    double Voxacc = 0.0, dVoxacc_dVg = 0.0, dVoxacc_dVb = 0.0;
    double Voxdepinv = 0.0, dVoxdepinv_dVg = 0.0, dVoxdepinv_dVd = 0.0, dVoxdepinv_dVb = 0.0;
    {
      const double V3 = Vfb_g - Vgs_eff + Vbseff - CONSTDELTA_3;
      if (Vfb_g <= 0.0)
        T0 = sqrt(V3 * V3 - 4.0 * CONSTDELTA_3 * Vfb_g);
      else
        T0 = sqrt(V3 * V3 + 4.0 * CONSTDELTA_3 * Vfb_g);
      T1 = 0.5 * (1.0 + V3 / T0);
      const double Vfbeff = Vfb_g - 0.5 * (V3 + T0);
      const double dVfbeff_dVg = T1 * dVgs_eff_dVg;
      const double dVfbeff_dVb = -T1;
      Voxacc = Vfb_g - Vfbeff;
      dVoxacc_dVg = -dVfbeff_dVg;
      dVoxacc_dVb = -dVfbeff_dVb;
      if (Voxacc < 0.0) {
        Voxacc = dVoxacc_dVg = dVoxacc_dVb = 0.0;
      }
      const double k1ox = P(k1ox);
      T0 = 0.5 * k1ox;
      T3 = Vgs_eff - Vfbeff - Vbseff - Vgsteff;
      if (k1ox == 0.0) {
        Voxdepinv = dVoxdepinv_dVg = dVoxdepinv_dVd = dVoxdepinv_dVb = 0.0;
      } else if (T3 < 0.0) {
        Voxdepinv = -T3;
        dVoxdepinv_dVg = -dVgs_eff_dVg + dVfbeff_dVg + dVgsteff_dVg;
        dVoxdepinv_dVd = dVgsteff_dVd;
        dVoxdepinv_dVb = dVfbeff_dVb + 1.0 + dVgsteff_dVb;
      } else {
        T1 = sqrt(T0 * T0 + T3);
        T2 = T0 / T1;
        Voxdepinv = k1ox * (T1 - T0);
        dVoxdepinv_dVg = T2 * (dVgs_eff_dVg - dVfbeff_dVg - dVgsteff_dVg);
        dVoxdepinv_dVd = -T2 * dVgsteff_dVd;
        dVoxdepinv_dVb = -T2 * (dVfbeff_dVb + 1.0 + dVgsteff_dVb);
      }
      Voxdepinv += Vgsteff;
      dVoxdepinv_dVg += dVgsteff_dVg;
      dVoxdepinv_dVd += dVgsteff_dVd;
      dVoxdepinv_dVb += dVgsteff_dVb;
    }
    const double vtmg = (tempMod < 2) ? Vtm : Vtm0;
    double Vaux = 0.0, dVaux_dVg = 0.0, dVaux_dVd = 0.0, dVaux_dVb = 0.0, VxNVt = 0.0;
    if (igcMod) {
      T0 = vtmg * P(nigc);
      if (igcMod == 1) {
        VxNVt = (Vgs_eff - dtype * vth0) / T0;
        if (VxNVt > CONSTEXP_THRESHOLD) {
          Vaux = Vgs_eff - dtype * vth0;
          dVaux_dVg = dVgs_eff_dVg;
          dVaux_dVd = 0.0;
          dVaux_dVb = 0.0;
        }
      } else {
        VxNVt = (Vgs_eff - von) / T0;
        if (VxNVt > CONSTEXP_THRESHOLD) {
          Vaux = Vgs_eff - von;
          dVaux_dVg = dVgs_eff_dVg;
          dVaux_dVd = -dVth_dVd;
          dVaux_dVb = -dVth_dVb;
        }
      }
      if (VxNVt < -CONSTEXP_THRESHOLD) {
        Vaux = T0 * log(1.0 + CONSTMIN_EXP);
        dVaux_dVg = dVaux_dVd = dVaux_dVb = 0.0;
      } else if ((VxNVt >= -CONSTEXP_THRESHOLD) && (VxNVt <= CONSTEXP_THRESHOLD)) {
        const double ExpVxNVt = exp(VxNVt);
        Vaux = T0 * log(1.0 + ExpVxNVt);
        dVaux_dVg = ExpVxNVt / (1.0 + ExpVxNVt);
        if (igcMod == 1) {
          dVaux_dVd = 0.0;
          dVaux_dVb = 0.0;
        } else {
          dVaux_dVd = -dVgs_eff_dVg * dVth_dVd;
          dVaux_dVb = -dVgs_eff_dVg * dVth_dVb;
        }
        dVaux_dVg *= dVgs_eff_dVg;
      }
      T2 = Vgs_eff * Vaux;
      dT2_dVg = dVgs_eff_dVg * Vaux + Vgs_eff * dVaux_dVg;
      dT2_dVd = Vgs_eff * dVaux_dVd;
      dT2_dVb = Vgs_eff * dVaux_dVb;
      T11 = P(Aechvb);
      T12 = P(Bechvb);
      T3 = P(aigc) * P(cigc) - P(bigc);
      T4 = P(bigc) * P(cigc);
      T5 = T12 * (P(aigc) + T3 * Voxdepinv - T4 * Voxdepinv * Voxdepinv);
      if (T5 > CONSTEXP_THRESHOLD) {
        T6 = CONSTMAX_EXP;
        dT6_dVg = dT6_dVd = dT6_dVb = 0.0;
      } else if (T5 < -CONSTEXP_THRESHOLD) {
        T6 = CONSTMIN_EXP;
        dT6_dVg = dT6_dVd = dT6_dVb = 0.0;
      } else {
        T6 = exp(T5);
        dT6_dVg = T6 * T12 * (T3 - 2.0 * T4 * Voxdepinv);
        dT6_dVd = dT6_dVg * dVoxdepinv_dVd;
        dT6_dVb = dT6_dVg * dVoxdepinv_dVb;
        dT6_dVg *= dVoxdepinv_dVg;
      }
      const double Igc = T11 * T2 * T6;
      const double dIgc_dVg = T11 * (T2 * dT6_dVg + T6 * dT2_dVg);
      const double dIgc_dVd = T11 * (T2 * dT6_dVd + T6 * dT2_dVd);
      const double dIgc_dVb = T11 * (T2 * dT6_dVb + T6 * dT2_dVb);
      double Pigcd, dPigcd_dVg, dPigcd_dVd, dPigcd_dVb;
      if (P(pigcdGiven) != 0.0) {
        Pigcd = P(pigcd);
        dPigcd_dVg = dPigcd_dVd = dPigcd_dVb = 0.0;
      } else {
        T11 = P(Bechvb) * toxe;
        T12 = Vgsteff + 1.0e-20;
        T13 = T11 / T12 / T12;
        T14 = -T13 / T12;
        Pigcd = T13 * (1.0 - 0.5 * Vdseff / T12);
        dPigcd_dVg = T14 * (2.0 + 0.5 * (dVdseff_dVg - 3.0 * Vdseff / T12));
        dPigcd_dVd = 0.5 * T14 * dVdseff_dVd;
        dPigcd_dVb = 0.5 * T14 * dVdseff_dVb;
      }
      T7 = -Pigcd * Vdseff;
      double dT7_dVg = -Vdseff * dPigcd_dVg - Pigcd * dVdseff_dVg;
      double dT7_dVd = -Vdseff * dPigcd_dVd - Pigcd * dVdseff_dVd + dT7_dVg * dVgsteff_dVd;
      double dT7_dVb = -Vdseff * dPigcd_dVb - Pigcd * dVdseff_dVb + dT7_dVg * dVgsteff_dVb;
      dT7_dVg *= dVgsteff_dVg;
      dT7_dVb *= dVbseff_dVb;
      T8 = T7 * T7 + 2.0e-4;
      dT8_dVg = 2.0 * T7;
      dT8_dVd = dT8_dVg * dT7_dVd;
      dT8_dVb = dT8_dVg * dT7_dVb;
      dT8_dVg *= dT7_dVg;
      if (T7 > CONSTEXP_THRESHOLD) {
        T9 = CONSTMAX_EXP;
        dT9_dVg = dT9_dVd = dT9_dVb = 0.0;
      } else if (T7 < -CONSTEXP_THRESHOLD) {
        T9 = CONSTMIN_EXP;
        dT9_dVg = dT9_dVd = dT9_dVb = 0.0;
      } else {
        T9 = exp(T7);
        dT9_dVg = T9 * dT7_dVg;
        dT9_dVd = T9 * dT7_dVd;
        dT9_dVb = T9 * dT7_dVb;
      }
      T0 = T8 * T8;
      T1 = T9 - 1.0 + 1.0e-4;
      T10 = (T1 - T7) / T8;
      dT10_dVg = (dT9_dVg - dT7_dVg - T10 * dT8_dVg) / T8;
      dT10_dVd = (dT9_dVd - dT7_dVd - T10 * dT8_dVd) / T8;
      dT10_dVb = (dT9_dVb - dT7_dVb - T10 * dT8_dVb) / T8;
      Igcs = Igc * T10;
      const double dIgcs_dVg = dIgc_dVg * T10 + Igc * dT10_dVg;
      const double dIgcs_dVd = dIgc_dVd * T10 + Igc * dT10_dVd;
      const double dIgcs_dVb = dIgc_dVb * T10 + Igc * dT10_dVb;
      T1 = T9 - 1.0 - 1.0e-4;
      T10 = (T7 * T9 - T1) / T8;
      dT10_dVg = (dT7_dVg * T9 + (T7 - 1.0) * dT9_dVg - T10 * dT8_dVg) / T8;
      dT10_dVd = (dT7_dVd * T9 + (T7 - 1.0) * dT9_dVd - T10 * dT8_dVd) / T8;
      dT10_dVb = (dT7_dVb * T9 + (T7 - 1.0) * dT9_dVb - T10 * dT8_dVb) / T8;
      Igcd = Igc * T10;
      const double dIgcd_dVg = dIgc_dVg * T10 + Igc * dT10_dVg;
      const double dIgcd_dVd = dIgc_dVd * T10 + Igc * dT10_dVd;
      const double dIgcd_dVb = dIgc_dVb * T10 + Igc * dT10_dVb;
      gIgcsg = dIgcs_dVg;
      gIgcsd = dIgcs_dVd;
      gIgcsb = dIgcs_dVb * dVbseff_dVb;
      gIgcdg = dIgcd_dVg;
      gIgcdd = dIgcd_dVd;
      gIgcdb = dIgcd_dVb * dVbseff_dVb;
      // Gate to source and drain overlap tunnelling, on the terminal (not mode-ordered) voltages.
      const double vfbsd_t = P(vfbsd) + P(vfbsdoff);
      T0 = vgs - vfbsd_t;
      double vgx_eff = sqrt(T0 * T0 + 1.0e-4);
      double dvgx_eff_dvg = T0 / vgx_eff;
      T2 = vgs * vgx_eff;
      dT2_dVg = vgs * dvgx_eff_dvg + vgx_eff;
      T11 = P(AechvbEdgeS);
      T12 = P(BechvbEdge);
      T3 = P(aigs) * P(cigs) - P(bigs);
      T4 = P(bigs) * P(cigs);
      T5 = T12 * (P(aigs) + T3 * vgx_eff - T4 * vgx_eff * vgx_eff);
      if (T5 > CONSTEXP_THRESHOLD) {
        T6 = CONSTMAX_EXP;
        dT6_dVg = 0.0;
      } else if (T5 < -CONSTEXP_THRESHOLD) {
        T6 = CONSTMIN_EXP;
        dT6_dVg = 0.0;
      } else {
        T6 = exp(T5);
        dT6_dVg = T6 * T12 * (T3 - 2.0 * T4 * vgx_eff) * dvgx_eff_dvg;
      }
      Igs = T11 * T2 * T6;
      const double dIgs_dVg = T11 * (T2 * dT6_dVg + T6 * dT2_dVg);
      const double dIgs_dVs = -dIgs_dVg;
      T0 = vgd - vfbsd_t;
      vgx_eff = sqrt(T0 * T0 + 1.0e-4);
      dvgx_eff_dvg = T0 / vgx_eff;
      T2 = vgd * vgx_eff;
      dT2_dVg = vgd * dvgx_eff_dvg + vgx_eff;
      T11 = P(AechvbEdgeD);
      T3 = P(aigd) * P(cigd) - P(bigd);
      T4 = P(bigd) * P(cigd);
      T5 = T12 * (P(aigd) + T3 * vgx_eff - T4 * vgx_eff * vgx_eff);
      if (T5 > CONSTEXP_THRESHOLD) {
        T6 = CONSTMAX_EXP;
        dT6_dVg = 0.0;
      } else if (T5 < -CONSTEXP_THRESHOLD) {
        T6 = CONSTMIN_EXP;
        dT6_dVg = 0.0;
      } else {
        T6 = exp(T5);
        dT6_dVg = T6 * T12 * (T3 - 2.0 * T4 * vgx_eff) * dvgx_eff_dvg;
      }
      Igd = T11 * T2 * T6;
      const double dIgd_dVg = T11 * (T2 * dT6_dVg + T6 * dT2_dVg);
      const double dIgd_dVd = -dIgd_dVg;
      gIgsg = dIgs_dVg;
      gIgss = dIgs_dVs;
      gIgdg = dIgd_dVg;
      gIgdd = dIgd_dVd;
    }
    if (igbMod) {
      T0 = vtmg * P(nigbacc);
      T1 = -Vgs_eff + Vbseff + Vfb_g;
      VxNVt = T1 / T0;
      if (VxNVt > CONSTEXP_THRESHOLD) {
        Vaux = T1;
        dVaux_dVg = -dVgs_eff_dVg;
        dVaux_dVb = 1.0;
      } else if (VxNVt < -CONSTEXP_THRESHOLD) {
        Vaux = T0 * log(1.0 + CONSTMIN_EXP);
        dVaux_dVg = dVaux_dVb = 0.0;
      } else {
        const double ExpVxNVt = exp(VxNVt);
        Vaux = T0 * log(1.0 + ExpVxNVt);
        dVaux_dVb = ExpVxNVt / (1.0 + ExpVxNVt);
        dVaux_dVg = -dVaux_dVb * dVgs_eff_dVg;
      }
      T2 = (Vgs_eff - Vbseff) * Vaux;
      dT2_dVg = dVgs_eff_dVg * Vaux + (Vgs_eff - Vbseff) * dVaux_dVg;
      dT2_dVb = -Vaux + (Vgs_eff - Vbseff) * dVaux_dVb;
      T11 = 4.97232e-7 * P(weff) * P(leff) * P(ToxRatio);
      T12 = -7.45669e11 * toxe;
      T3 = P(aigbacc) * P(cigbacc) - P(bigbacc);
      T4 = P(bigbacc) * P(cigbacc);
      T5 = T12 * (P(aigbacc) + T3 * Voxacc - T4 * Voxacc * Voxacc);
      if (T5 > CONSTEXP_THRESHOLD) {
        T6 = CONSTMAX_EXP;
        dT6_dVg = dT6_dVb = 0.0;
      } else if (T5 < -CONSTEXP_THRESHOLD) {
        T6 = CONSTMIN_EXP;
        dT6_dVg = dT6_dVb = 0.0;
      } else {
        T6 = exp(T5);
        dT6_dVg = T6 * T12 * (T3 - 2.0 * T4 * Voxacc);
        dT6_dVb = dT6_dVg * dVoxacc_dVb;
        dT6_dVg *= dVoxacc_dVg;
      }
      const double Igbacc = T11 * T2 * T6;
      const double dIgbacc_dVg = T11 * (T2 * dT6_dVg + T6 * dT2_dVg);
      const double dIgbacc_dVb = T11 * (T2 * dT6_dVb + T6 * dT2_dVb);
      T0 = vtmg * P(nigbinv);
      T1 = Voxdepinv - P(eigbinv);
      VxNVt = T1 / T0;
      if (VxNVt > CONSTEXP_THRESHOLD) {
        Vaux = T1;
        dVaux_dVg = dVoxdepinv_dVg;
        dVaux_dVd = dVoxdepinv_dVd;
        dVaux_dVb = dVoxdepinv_dVb;
      } else if (VxNVt < -CONSTEXP_THRESHOLD) {
        Vaux = T0 * log(1.0 + CONSTMIN_EXP);
        dVaux_dVg = dVaux_dVd = dVaux_dVb = 0.0;
      } else {
        const double ExpVxNVt = exp(VxNVt);
        Vaux = T0 * log(1.0 + ExpVxNVt);
        dVaux_dVg = ExpVxNVt / (1.0 + ExpVxNVt);
        dVaux_dVd = dVaux_dVg * dVoxdepinv_dVd;
        dVaux_dVb = dVaux_dVg * dVoxdepinv_dVb;
        dVaux_dVg *= dVoxdepinv_dVg;
      }
      T2 = (Vgs_eff - Vbseff) * Vaux;
      dT2_dVg = dVgs_eff_dVg * Vaux + (Vgs_eff - Vbseff) * dVaux_dVg;
      dT2_dVd = (Vgs_eff - Vbseff) * dVaux_dVd;
      dT2_dVb = -Vaux + (Vgs_eff - Vbseff) * dVaux_dVb;
      T11 *= 0.75610;
      T12 *= 1.31724;
      T3 = P(aigbinv) * P(cigbinv) - P(bigbinv);
      T4 = P(bigbinv) * P(cigbinv);
      T5 = T12 * (P(aigbinv) + T3 * Voxdepinv - T4 * Voxdepinv * Voxdepinv);
      if (T5 > CONSTEXP_THRESHOLD) {
        T6 = CONSTMAX_EXP;
        dT6_dVg = dT6_dVd = dT6_dVb = 0.0;
      } else if (T5 < -CONSTEXP_THRESHOLD) {
        T6 = CONSTMIN_EXP;
        dT6_dVg = dT6_dVd = dT6_dVb = 0.0;
      } else {
        T6 = exp(T5);
        dT6_dVg = T6 * T12 * (T3 - 2.0 * T4 * Voxdepinv);
        dT6_dVd = dT6_dVg * dVoxdepinv_dVd;
        dT6_dVb = dT6_dVg * dVoxdepinv_dVb;
        dT6_dVg *= dVoxdepinv_dVg;
      }
      const double Igbinv = T11 * T2 * T6;
      const double dIgbinv_dVg = T11 * (T2 * dT6_dVg + T6 * dT2_dVg);
      const double dIgbinv_dVd = T11 * (T2 * dT6_dVd + T6 * dT2_dVd);
      const double dIgbinv_dVb = T11 * (T2 * dT6_dVb + T6 * dT2_dVb);
      Igb = Igbinv + Igbacc;
      gIgbg = dIgbinv_dVg + dIgbacc_dVg;
      gIgbd = dIgbinv_dVd;
      gIgbb = (dIgbinv_dVb + dIgbacc_dVb) * dVbseff_dVb;
    }
  }

  // Multi-finger scaling (:10601-10640).
  if (nf != 1.0) {
    cdrain *= nf; gds *= nf; gm *= nf; gmbs *= nf;
    gbbs *= nf; gbgs *= nf; gbds *= nf; csub *= nf;
    Igidl *= nf; ggidld *= nf; ggidlg *= nf; ggidlb *= nf;
    Igisl *= nf; ggisls *= nf; ggislg *= nf; ggislb *= nf;
    Igcs *= nf; gIgcsg *= nf; gIgcsd *= nf; gIgcsb *= nf;
    Igcd *= nf; gIgcdg *= nf; gIgcdd *= nf; gIgcdb *= nf;
    Igs *= nf; gIgsg *= nf; gIgss *= nf;
    Igd *= nf; gIgdg *= nf; gIgdd *= nf;
    Igb *= nf; gIgbg *= nf; gIgbd *= nf; gIgbb *= nf;
  }
  const double gIgbs = -(gIgbg + gIgbd + gIgbb);
  const double gIgcss = -(gIgcsg + gIgcsd + gIgcsb);
  const double gIgcds = -(gIgcdg + gIgcdd + gIgcdb);

  // Hand-off to the charge-and-stamp part.
  Mid hm;
  hm.v[m_vds] = vds;
  hm.v[m_vgs] = vgs;
  hm.v[m_vbs] = vbs;
  hm.v[m_orig] = (double)origFlag;
  hm.v[m_von] = von;
  hm.v[m_gbs] = gbs;
  hm.v[m_cbs] = cbs;
  hm.v[m_gbd] = gbd;
  hm.v[m_cbd] = cbd;
  hm.v[m_cdrain] = cdrain;
  hm.v[m_gds] = gds;
  hm.v[m_gm] = gm;
  hm.v[m_gmbs] = gmbs;
  hm.v[m_csub] = csub;
  hm.v[m_gbbs] = gbbs;
  hm.v[m_gbgs] = gbgs;
  hm.v[m_gbds] = gbds;
  hm.v[m_Igidl] = Igidl;
  hm.v[m_ggidld] = ggidld;
  hm.v[m_ggidlg] = ggidlg;
  hm.v[m_ggidlb] = ggidlb;
  hm.v[m_Igisl] = Igisl;
  hm.v[m_ggisls] = ggisls;
  hm.v[m_ggislg] = ggislg;
  hm.v[m_ggislb] = ggislb;
  hm.v[m_Abulk0] = Abulk0;
  hm.v[m_dAbulk0_dVb] = dAbulk0_dVb;
  hm.v[m_Vbseff] = Vbseff;
  hm.v[m_dVbseff_dVb] = dVbseff_dVb;
  hm.v[m_Vgs_eff] = Vgs_eff;
  hm.v[m_dVgs_eff_dVg] = dVgs_eff_dVg;
  hm.v[m_Vgst] = Vgst;
  hm.v[m_dVth_dVb] = dVth_dVb;
  hm.v[m_dVth_dVd] = dVth_dVd;
  hm.v[m_n] = n;
  hm.v[m_dn_dVb] = dn_dVb;
  hm.v[m_dn_dVd] = dn_dVd;
  if constexpr (FULL) {
    hm.v[m_Igs] = Igs;
    hm.v[m_gIgsg] = gIgsg;
    hm.v[m_gIgss] = gIgss;
    hm.v[m_Igd] = Igd;
    hm.v[m_gIgdg] = gIgdg;
    hm.v[m_gIgdd] = gIgdd;
    hm.v[m_Igcs] = Igcs;
    hm.v[m_gIgcsg] = gIgcsg;
    hm.v[m_gIgcsd] = gIgcsd;
    hm.v[m_gIgcsb] = gIgcsb;
    hm.v[m_Igcd] = Igcd;
    hm.v[m_gIgcdg] = gIgcdg;
    hm.v[m_gIgcdd] = gIgcdd;
    hm.v[m_gIgcdb] = gIgcdb;
    hm.v[m_Igb] = Igb;
    hm.v[m_gIgbg] = gIgbg;
    hm.v[m_gIgbd] = gIgbd;
    hm.v[m_gIgbb] = gIgbb;
  }
  if constexpr (GEN) {
    hm.v[m_vges] = vges;
    hm.v[m_vgms] = vgms;
    hm.v[m_vdes] = vdes;
    hm.v[m_vses] = vses;
    hm.v[m_vdbs] = vdbs;
    hm.v[m_vsbs] = vsbs;
    hm.v[m_gcrg] = gcrg;
    hm.v[m_gcrgg] = gcrgg;
    hm.v[m_gcrgd] = gcrgd;
    hm.v[m_gcrgs] = gcrgs;
    hm.v[m_gcrgb] = gcrgb;
    hm.v[m_gstot] = gstot;
    hm.v[m_gstotd] = gstotd;
    hm.v[m_gstotg] = gstotg;
    hm.v[m_gstots] = gstots;
    hm.v[m_gstotb] = gstotb;
    hm.v[m_gdtot] = gdtot;
    hm.v[m_gdtotd] = gdtotd;
    hm.v[m_gdtotg] = gdtotg;
    hm.v[m_gdtots] = gdtots;
    hm.v[m_gdtotb] = gdtotb;
  }
  (void)gIgbs; (void)gIgcss; (void)gIgcds;
  if constexpr (PART == 1) {
    *mid = hm;
    return;
  }
  bsim4_finish<FULL, SERIES, GEN>(P_, V, fl, vgb_orig, hm, o, Vx);
}
#undef P

}  // namespace xb4
