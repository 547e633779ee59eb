// Host-side BSIM4 set-up: model-card defaults, temperature and geometry precompute.
//
// Follows the reference's set-up sequence for one BSIM4 instance, in the same floating-point
// order, so that the load kernel sees the same constants the reference's evaluation sees:
//   model card defaults and dependent defaults   N_DEV_MOSFET_B4.C:15661-16066 (Model::Model)
//   junction-potential clamps                     N_DEV_MOSFET_B4.C:14740-14780 (Model::processParams)
//   instance defaults                             N_DEV_MOSFET_B4.C:4586-4618  (Instance::Instance)
//   mode selection                                N_DEV_MOSFET_B4.C:3621-3677  (Instance::processParams)
//   temperature / size / instance precompute      N_DEV_MOSFET_B4.C:5640-7743  (updateTemperature)
//   geometry helpers                              N_DEV_MOSFET_B4.C:14322-14462 (NumFingerDiff, PAeffGeo)
// The size-dependent set is created once per (L, W, NF) per model, at the first instance's
// temperature, exactly as the reference caches SizeDependParam objects.

#include "bsim4_setup.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <tuple>

#include "bsim4_fields.h"
#include "xd_consts.h"

namespace xb4 {
namespace {

using namespace xdc;

struct Card {
#define B4P(name, mem, dflt) double mem = dflt;
#include "bsim4_card.inc"
#undef B4P
  std::set<std::string> given;
  int dtype = 1;
  bool g(const char *n) const { return given.count(n) != 0; }
};

struct CardSetter {
  std::map<std::string, double Card::*> by_name;
  CardSetter() {
#define B4P(name, mem, dflt) by_name[name] = &Card::mem;
#include "bsim4_card.inc"
#undef B4P
  }
};

const CardSetter &card_setter() {
  static CardSetter s;
  return s;
}

std::string upper(std::string s) {
  for (auto &c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

// Size-dependent parameter set (one per (L, W, NF) per model).
struct Size {
#define B4BIN(mem, base, l, w, p) double mem = 0.0;
#include "bsim4_bins.inc"
#undef B4BIN
  double Length = 0, Width = 0, NFinger = 0;
  double dl = 0, dlc = 0, dw = 0, dwc = 0, dwj = 0, leff = 0, weff = 0, leffCV = 0, weffCV = 0, weffCJ = 0;
  double abulkCVfactor = 0, vsattemp = 0, rds0 = 0, rdswmin = 0, rd0 = 0, rdwmin = 0, rs0 = 0, rswmin = 0;
  double u0temp = 0, tfactor = 0, lc = 0, phi = 0, sqrtPhi = 0, phis3 = 0, Xdep0 = 0, sqrtXdep0 = 0;
  double litl = 0, vbi = 0, vfbsd = 0, cdep0 = 0, ToxRatio = 0, ToxRatioEdge = 0, Aechvb = 0, Bechvb = 0;
  double AechvbEdgeS = 0, AechvbEdgeD = 0, BechvbEdge = 0, mstar = 0, mstarcv = 0, voffcbn = 0;
  double voffcbncv = 0, ldeb = 0, k1ox = 0, theta0vb0 = 0, thetaRout = 0, vfbzbfactor = 0, ku0 = 0;
  double kvth0 = 0, ku0temp = 0, inv_od_ref = 0, rho_ref = 0, cgdo = 0, cgso = 0, cgbo = 0;
};

// Model after the temperature pass (the reference writes these back into the model object).
struct ModelState {
  Card c;
  double coxe = 0, coxp = 0, vcrit = 0, factor1 = 0, vtm0 = 0, Eg0 = 0, vtm = 0;
  double SjctTempSatCurDensity = 0, SjctSidewallTempSatCurDensity = 0, SjctGateSidewallTempSatCurDensity = 0;
  double DjctTempSatCurDensity = 0, DjctSidewallTempSatCurDensity = 0, DjctGateSidewallTempSatCurDensity = 0;
  double SunitAreaTempJctCap = 0, DunitAreaTempJctCap = 0, SunitLengthSidewallTempJctCap = 0;
  double DunitLengthSidewallTempJctCap = 0, SunitLengthGateSidewallTempJctCap = 0;
  double DunitLengthGateSidewallTempJctCap = 0, PhiBS = 0, PhiBD = 0, PhiBSWS = 0, PhiBSWD = 0;
  double PhiBSWGS = 0, PhiBSWGD = 0;
  double njtsstemp = 0, njtsswstemp = 0, njtsswgstemp = 0, njtsdtemp = 0, njtsswdtemp = 0, njtsswgdtemp = 0;
  bool temp_done = false;
  double temp_seen = 0;
  std::vector<std::unique_ptr<Size>> sizes;
};

struct InstParams {
  double temp = 0, l = 5.0e-6, w = 5.0e-6, nf = 1.0, sa = 0, sb = 0, sd = 0, sca = 0, scb = 0, scc = 0, sc = 0;
  double drainArea = 0, sourceArea = 0, drainPerimeter = 0, sourcePerimeter = 0, drainSquares = 1.0,
         sourceSquares = 1.0, rbdb = 0, rbsb = 0, rbpb = 0, rbps = 0, rbpd = 0, delvto = 0, xgw = 0, ngcon = 0,
         mult = 1.0, off = 0, trnqsMod = 0, acnqsMod = 0, rbodyMod = 0, rgateMod = 0, geoMod = 0, rgeoMod = 0,
         min = 0, icVDS = 0, icVGS = 0, icVBS = 0;
  std::set<std::string> given;
  bool g(const char *n) const { return given.count(n) != 0; }
};

// ---- Model card: defaults, dependent defaults, clamps (Model::Model, Model::processParams) ----
std::string process_model(const ModelSpec &spec, const SetupOptions &opts, Card &m) {
  m.dtype = spec.pmos ? CONSTPMOS : CONSTNMOS;
  const CardSetter &cs = card_setter();
  for (const auto &kv : spec.params) {
    std::string n = upper(kv.first);
    if (n == "LEVEL" || n == "VERSION") continue;
    auto it = cs.by_name.find(n);
    if (it == cs.by_name.end()) return "unknown BSIM4 model parameter " + n;
    double v = kv.second;
    if (n == "TNOM") v += CONSTCtoK;
    m.*(it->second) = v;
    m.given.insert(n);
  }
  if (!m.g("TNOM")) m.tnom = opts.tnom_c + CONSTCtoK;
  if (!m.g("TOXP")) m.toxp = m.toxe;
  if (!m.g("TOXM")) m.toxm = m.toxe;
  if (!m.g("DSUB")) m.dsub = m.drout;
  if (!m.g("VTH0")) m.vth0 = (m.dtype == CONSTNMOS) ? 0.7 : -0.7;
  if (!m.g("VDDEOT")) m.vddeot = (m.dtype == CONSTNMOS) ? 1.5 : -1.5;
  if (!m.g("EU")) m.eu = (m.dtype == CONSTNMOS) ? 1.67 : 1.0;
  if (!m.g("UA")) m.ua = (m.mobMod == 2) ? 1.0E-15 : 1.0E-9;
  if (!m.g("UC")) m.uc = (m.mobMod == 1) ? -0.0465 : -0.0465E-9;
  if (!m.g("UC1")) m.uc1 = (m.mobMod == 1) ? -0.056 : -0.056E-9;
  if (!m.g("U0")) m.u0 = (m.dtype == CONSTNMOS) ? 0.067 : 0.025;
  if (!m.g("AIGC")) m.aigc = (m.dtype == CONSTNMOS) ? 1.36E-2 : 9.80E-3;
  if (!m.g("BIGC")) m.bigc = (m.dtype == CONSTNMOS) ? 1.71E-3 : 7.59E-4;
  if (!m.g("CIGC")) m.cigc = (m.dtype == CONSTNMOS) ? 0.075 : 0.03;
  if (m.g("AIGSD")) {
    m.aigs = m.aigd = m.aigsd;
  } else {
    m.aigsd = (m.dtype == CONSTNMOS) ? 1.36E-2 : 9.80E-3;
    if (!m.g("AIGS")) m.aigs = m.aigsd;
    if (!m.g("AIGD")) m.aigd = m.aigsd;
  }
  if (m.g("BIGSD")) {
    m.bigs = m.bigd = m.bigsd;
  } else {
    m.bigsd = (m.dtype == CONSTNMOS) ? 1.71E-3 : 7.59E-4;
    if (!m.g("BIGS")) m.bigs = m.bigsd;
    if (!m.g("BIGD")) m.bigd = m.bigsd;
  }
  if (m.g("CIGSD")) {
    m.cigs = m.cigd = m.cigsd;
  } else {
    m.cigsd = (m.dtype == CONSTNMOS) ? 0.075 : 0.03;
    if (!m.g("CIGS")) m.cigs = m.cigsd;
    if (!m.g("CIGD")) m.cigd = m.cigsd;
  }
  if (!m.g("IJTHDFWD")) m.ijthdfwd = m.ijthsfwd;
  if (!m.g("IJTHDREV")) m.ijthdrev = m.ijthsrev;
  if (!m.g("XJBVD")) m.xjbvd = m.xjbvs;
  if (!m.g("BVD")) m.bvd = m.bvs;
  if (!m.g("CKAPPAD")) m.ckappad = m.ckappas;
  if (!m.g("DMCI")) m.dmci = m.dmcg;
  if (!m.g("LLC")) m.Llc = m.Ll;
  if (!m.g("LWC")) m.Lwc = m.Lw;
  if (!m.g("LWLC")) m.Lwlc = m.Lwl;
  if (!m.g("WLC")) m.Wlc = m.Wl;
  if (!m.g("WWC")) m.Wwc = m.Ww;
  if (!m.g("WWLC")) m.Wwlc = m.Wwl;
  if (!m.g("DWC")) m.dwc = m.Wint;
  if (!m.g("DLC")) m.dlc = m.Lint;
  if (!m.g("AGISL") && m.g("AGIDL")) m.agisl = m.agidl;
  if (!m.g("BGISL") && m.g("BGIDL")) m.bgisl = m.bgidl;
  if (!m.g("CGISL") && m.g("CGIDL")) m.cgisl = m.cgidl;
  if (!m.g("EGISL") && m.g("EGIDL")) m.egisl = m.egidl;
  if (!m.g("DLCIG")) m.dlcig = m.Lint;
  if (!m.g("DLCIGD")) m.dlcigd = m.g("DLCIG") ? m.dlcig : m.Lint;
  if (!m.g("DWJ")) m.dwj = m.dwc;
  if (!m.g("CF")) m.cf = 2.0 * m.epsrox * ((CONSTEPS0) / (M_PI)) * log(1.0 + 0.4E-6 / m.toxe);
  if (!m.g("JSD")) m.DjctSatCurDensity = m.SjctSatCurDensity;
  if (!m.g("JSWD")) m.DjctSidewallSatCurDensity = m.SjctSidewallSatCurDensity;
  if (!m.g("JSWGD")) m.DjctGateSidewallSatCurDensity = m.SjctGateSidewallSatCurDensity;
  if (!m.g("PBD")) m.DbulkJctPotential = m.SbulkJctPotential;
  if (!m.g("NJD")) m.DjctEmissionCoeff = m.SjctEmissionCoeff;
  if (!m.g("XTID")) m.DjctTempExponent = m.SjctTempExponent;
  if (!m.g("MJD")) m.DbulkJctBotGradingCoeff = m.SbulkJctBotGradingCoeff;
  if (!m.g("MJSWD")) m.DbulkJctSideGradingCoeff = m.SbulkJctSideGradingCoeff;
  if (!m.g("MJSWGS")) m.SbulkJctGateSideGradingCoeff = m.SbulkJctSideGradingCoeff;
  if (!m.g("MJSWGD")) m.DbulkJctGateSideGradingCoeff = m.SbulkJctGateSideGradingCoeff;
  if (!m.g("PBSWD")) m.DsidewallJctPotential = m.SsidewallJctPotential;
  if (!m.g("PBSWGS")) m.SGatesidewallJctPotential = m.SsidewallJctPotential;
  if (!m.g("PBSWGD")) m.DGatesidewallJctPotential = m.DsidewallJctPotential;
  if (!m.g("CJD")) m.DunitAreaJctCap = m.SunitAreaJctCap;
  if (!m.g("CJSWD")) m.DunitLengthSidewallJctCap = m.SunitLengthSidewallJctCap;
  if (!m.g("CJSWGS")) m.SunitLengthGateSidewallJctCap = m.SunitLengthSidewallJctCap;
  if (!m.g("CJSWGD")) m.DunitLengthGateSidewallJctCap = m.SunitLengthGateSidewallJctCap;
  if (!m.g("JTSD")) m.jtsd = m.jtss;
  if (!m.g("JTSSWD")) m.jtsswd = m.jtssws;
  if (!m.g("JTSSWGD")) m.jtsswgd = m.jtsswgs;
  if (!m.g("NJTSD") && m.g("NJTS")) m.njtsd = m.njts;
  if (!m.g("NJTSSWD") && m.g("NJTSSW")) m.njtsswd = m.njtssw;
  if (!m.g("NJTSSWGD") && m.g("NJTSSWG")) m.njtsswgd = m.njtsswg;
  if (!m.g("XTSD")) m.xtsd = m.xtss;
  if (!m.g("XTSSWD")) m.xtsswd = m.xtssws;
  if (!m.g("XTSSWGD")) m.xtsswgd = m.xtsswgs;
  if (!m.g("TNJTSD") && m.g("TNJTS")) m.tnjtsd = m.tnjts;
  if (!m.g("TNJTSSWD") && m.g("TNJTSSW")) m.tnjtsswd = m.tnjtssw;
  if (!m.g("TNJTSSWGD") && m.g("TNJTSSWG")) m.tnjtsswgd = m.tnjtsswg;
  if (!m.g("VTSD")) m.vtsd = m.vtss;
  if (!m.g("VTSSWD")) m.vtsswd = m.vtssws;
  if (!m.g("VTSSWGD")) m.vtsswgd = m.vtsswgs;
  if (!m.g("LAGISL") && m.g("LAGIDL")) m.lagisl = m.lagidl;
  if (!m.g("LBGISL") && m.g("LBGIDL")) m.lbgisl = m.lbgidl;
  if (!m.g("LCGISL") && m.g("LCGIDL")) m.lcgisl = m.lcgidl;
  if (!m.g("LEGISL") && m.g("LEGIDL")) m.legisl = m.legidl;
  const bool sd_a = !(!m.g("AIGSD") && (m.g("AIGS") || m.g("AIGD")));
  const bool sd_b = !(!m.g("BIGSD") && (m.g("BIGS") || m.g("BIGD")));
  const bool sd_c = !(!m.g("CIGSD") && (m.g("CIGS") || m.g("CIGD")));
  if (sd_a) m.laigs = m.laigd = m.laigsd;
  if (sd_b) m.lbigs = m.lbigd = m.lbigsd;
  if (sd_c) m.lcigs = m.lcigd = m.lcigsd;
  if (!m.g("WAGISL") && m.g("WAGIDL")) m.wagisl = m.wagidl;
  if (!m.g("WBGISL") && m.g("WBGIDL")) m.wbgisl = m.wbgidl;
  if (!m.g("WCGISL") && m.g("WCGIDL")) m.wcgisl = m.wcgidl;
  if (!m.g("WEGISL") && m.g("WEGIDL")) m.wegisl = m.wegidl;
  if (sd_a) m.waigs = m.waigd = m.waigsd;
  if (sd_b) m.wbigs = m.wbigd = m.wbigsd;
  if (sd_c) m.wcigs = m.wcigd = m.wcigsd;
  if (!m.g("PAGISL") && m.g("PAGIDL")) m.pagisl = m.pagidl;
  if (!m.g("PBGISL") && m.g("PBGIDL")) m.pbgisl = m.pbgidl;
  if (!m.g("PCGISL") && m.g("PCGIDL")) m.pcgisl = m.pcgidl;
  if (!m.g("PEGISL") && m.g("PEGIDL")) m.pegisl = m.pegidl;
  if (sd_a) m.paigs = m.paigd = m.paigsd;
  if (sd_b) m.pbigs = m.pbigd = m.pbigsd;
  if (sd_c) m.pcigs = m.pcigd = m.pcigsd;
  // Model::processParams
  if (m.SbulkJctPotential < 0.1) m.SbulkJctPotential = 0.1;
  if (m.SsidewallJctPotential < 0.1) m.SsidewallJctPotential = 0.1;
  if (m.SGatesidewallJctPotential < 0.1) m.SGatesidewallJctPotential = 0.1;
  if (m.DbulkJctPotential < 0.1) m.DbulkJctPotential = 0.1;
  if (m.DsidewallJctPotential < 0.1) m.DsidewallJctPotential = 0.1;
  if (m.DGatesidewallJctPotential < 0.1) m.DGatesidewallJctPotential = 0.1;

  // Features outside the load kernel's scope are refused here rather than mis-evaluated.
  if (m.mtrlMod != 0) return "BSIM4 mtrlMod != 0 is not supported";
  if (m.rdsMod != 0 && m.rdsMod != 1) return "BSIM4 rdsMod must be 0 or 1";
  if (m.igcMod < 0 || m.igcMod > 2) return "BSIM4 igcMod must be 0, 1 or 2";
  if (m.igbMod < 0 || m.igbMod > 1) return "BSIM4 igbMod must be 0 or 1";
  if (m.rgateMod < 0 || m.rgateMod > 3 || m.rgateMod != (int)m.rgateMod) return "BSIM4 rgateMod must be 0, 1, 2 or 3";
  if (m.rbodyMod < 0 || m.rbodyMod > 2 || m.rbodyMod != (int)m.rbodyMod) return "BSIM4 rbodyMod must be 0, 1 or 2";
  // The transient NQS charge model (trnqsMod 1) adds the charge node; acnqsMod only sets the AC
  // small-signal time constant (taunet, N_DEV_MOSFET_B4.C:11639-11642), which no DC or transient
  // load reads.
  if (m.trnqsMod != 0 && m.trnqsMod != 1) return "BSIM4 trnqsMod must be 0 or 1";
  if (m.acnqsMod != 0 && m.acnqsMod != 1) return "BSIM4 acnqsMod must be 0 or 1";
  if (m.capMod < 0 || m.capMod > 2) return "BSIM4 capMod must be 0, 1 or 2";
  if (m.dioMod < 0 || m.dioMod > 2) return "BSIM4 dioMod must be 0, 1 or 2";
  if (m.mobMod < 0 || m.mobMod > 2) return "BSIM4 mobMod must be 0, 1 or 2";
  // tnoiMod selects the thermal-noise model: outside a noise analysis it adds no nodes
  // (N_DEV_MOSFET_B4.C:3687) and feeds only the noise charge (:10674), so every value loads alike.
  if (m.tnoiMod < 0 || m.tnoiMod > 1) return "BSIM4 tnoiMod must be 0 or 1";
  return std::string();
}

// ---- Model-level part of the temperature pass (updateTemperature, B4.C:5670-6030) ----
void model_temperature(ModelState &ms, double temp) {
  Card &m = ms.c;
  const double Tnom = m.tnom;
  if ((m.g("TOXE")) && (m.g("TOXP")) && (m.g("DTOX")) && (m.toxe != (m.toxp + m.dtox))) {
    // toxe, toxp and dtox all given and inconsistent: dtox ignored
  } else if ((m.g("TOXE")) && (!m.g("TOXP"))) {
    m.toxp = m.toxe - m.dtox;
  } else if ((!m.g("TOXE")) && (m.g("TOXP"))) {
    m.toxe = m.toxp + m.dtox;
  }
  const double epsrox = m.epsrox;
  const double toxe = m.toxe;
  const double epssub = CONSTEPSSI;
  ms.coxe = epsrox * CONSTEPS0 / toxe;
  ms.coxp = m.epsrox * CONSTEPS0 / m.toxp;
  if (!m.g("CGDO")) {
    if (m.g("DLC") && (m.dlc > 0.0))
      m.cgdo = m.dlc * ms.coxe - m.cgdl;
    else
      m.cgdo = 0.6 * m.xj * ms.coxe;
  }
  if (!m.g("CGSO")) {
    if (m.g("DLC") && (m.dlc > 0.0))
      m.cgso = m.dlc * ms.coxe - m.cgsl;
    else
      m.cgso = 0.6 * m.xj * ms.coxe;
  }
  if (!m.g("CGBO")) m.cgbo = 2.0 * m.dwc * ms.coxe;
  ms.vcrit = CONSTvt0 * log(CONSTvt0 / (CONSTroot2 * 1.0e-14));
  ms.factor1 = sqrt(epssub / (epsrox * CONSTEPS0) * toxe);
  const double Vtm0 = ms.vtm0 = CONSTKboQ * Tnom;
  const double Eg0 = 1.16 - 7.02e-4 * Tnom * Tnom / (Tnom + 1108.0);
  ms.Eg0 = Eg0;
  ms.vtm = CONSTKboQ * temp;
  const double Eg = 1.16 - 7.02e-4 * temp * temp / (temp + 1108.0);
  if (temp != Tnom) {
    double T0 = Eg0 / Vtm0 - Eg / ms.vtm;
    double T1 = log(temp / Tnom);
    double T2 = T0 + m.SjctTempExponent * T1;
    double T3 = exp(T2 / m.SjctEmissionCoeff);
    ms.SjctTempSatCurDensity = m.SjctSatCurDensity * T3;
    ms.SjctSidewallTempSatCurDensity = m.SjctSidewallSatCurDensity * T3;
    ms.SjctGateSidewallTempSatCurDensity = m.SjctGateSidewallSatCurDensity * T3;
    T2 = T0 + m.DjctTempExponent * T1;
    T3 = exp(T2 / m.DjctEmissionCoeff);
    ms.DjctTempSatCurDensity = m.DjctSatCurDensity * T3;
    ms.DjctSidewallTempSatCurDensity = m.DjctSidewallSatCurDensity * T3;
    ms.DjctGateSidewallTempSatCurDensity = m.DjctGateSidewallSatCurDensity * T3;
  } else {
    ms.SjctTempSatCurDensity = m.SjctSatCurDensity;
    ms.SjctSidewallTempSatCurDensity = m.SjctSidewallSatCurDensity;
    ms.SjctGateSidewallTempSatCurDensity = m.SjctGateSidewallSatCurDensity;
    ms.DjctTempSatCurDensity = m.DjctSatCurDensity;
    ms.DjctSidewallTempSatCurDensity = m.DjctSidewallSatCurDensity;
    ms.DjctGateSidewallTempSatCurDensity = m.DjctGateSidewallSatCurDensity;
  }
  if (ms.SjctTempSatCurDensity < 0.0) ms.SjctTempSatCurDensity = 0.0;
  if (ms.SjctSidewallTempSatCurDensity < 0.0) ms.SjctSidewallTempSatCurDensity = 0.0;
  if (ms.SjctGateSidewallTempSatCurDensity < 0.0) ms.SjctGateSidewallTempSatCurDensity = 0.0;
  if (ms.DjctTempSatCurDensity < 0.0) ms.DjctTempSatCurDensity = 0.0;
  if (ms.DjctSidewallTempSatCurDensity < 0.0) ms.DjctSidewallTempSatCurDensity = 0.0;
  if (ms.DjctGateSidewallTempSatCurDensity < 0.0) ms.DjctGateSidewallTempSatCurDensity = 0.0;
  const double delTemp = temp - Tnom;
  double T0 = m.tcj * delTemp;
  if (T0 >= -1.0) {
    ms.SunitAreaTempJctCap = m.SunitAreaJctCap * (1.0 + T0);
    ms.DunitAreaTempJctCap = m.DunitAreaJctCap * (1.0 + T0);
  } else {
    if (m.SunitAreaJctCap > 0.0) ms.SunitAreaTempJctCap = 0.0;
    if (m.DunitAreaJctCap > 0.0) ms.DunitAreaTempJctCap = 0.0;
  }
  T0 = m.tcjsw * delTemp;
  if (T0 >= -1.0) {
    ms.SunitLengthSidewallTempJctCap = m.SunitLengthSidewallJctCap * (1.0 + T0);
    ms.DunitLengthSidewallTempJctCap = m.DunitLengthSidewallJctCap * (1.0 + T0);
  } else {
    if (m.SunitLengthSidewallJctCap > 0.0) ms.SunitLengthSidewallTempJctCap = 0.0;
    if (m.DunitLengthSidewallJctCap > 0.0) ms.DunitLengthSidewallTempJctCap = 0.0;
  }
  T0 = m.tcjswg * delTemp;
  if (T0 >= -1.0) {
    ms.SunitLengthGateSidewallTempJctCap = m.SunitLengthGateSidewallJctCap * (1.0 + T0);
    ms.DunitLengthGateSidewallTempJctCap = m.DunitLengthGateSidewallJctCap * (1.0 + T0);
  } else {
    if (m.SunitLengthGateSidewallJctCap > 0.0) ms.SunitLengthGateSidewallTempJctCap = 0.0;
    if (m.DunitLengthGateSidewallJctCap > 0.0) ms.DunitLengthGateSidewallTempJctCap = 0.0;
  }
  ms.PhiBS = m.SbulkJctPotential - m.tpb * delTemp;
  if (ms.PhiBS < 0.01) ms.PhiBS = 0.01;
  ms.PhiBD = m.DbulkJctPotential - m.tpb * delTemp;
  if (ms.PhiBD < 0.01) ms.PhiBD = 0.01;
  ms.PhiBSWS = m.SsidewallJctPotential - m.tpbsw * delTemp;
  if (ms.PhiBSWS <= 0.01) ms.PhiBSWS = 0.01;
  ms.PhiBSWD = m.DsidewallJctPotential - m.tpbsw * delTemp;
  if (ms.PhiBSWD <= 0.01) ms.PhiBSWD = 0.01;
  ms.PhiBSWGS = m.SGatesidewallJctPotential - m.tpbswg * delTemp;
  if (ms.PhiBSWGS <= 0.01) ms.PhiBSWGS = 0.01;
  ms.PhiBSWGD = m.DGatesidewallJctPotential - m.tpbswg * delTemp;
  if (ms.PhiBSWGD <= 0.01) ms.PhiBSWGD = 0.01;
  if (m.ijthdfwd <= 0.0) m.ijthdfwd = 0.1;
  if (m.ijthsfwd <= 0.0) m.ijthsfwd = 0.1;
  if (m.ijthdrev <= 0.0) m.ijthdrev = 0.1;
  if (m.ijthsrev <= 0.0) m.ijthsrev = 0.1;
  if ((m.xjbvd <= 0.0) && (m.dioMod == 2))
    m.xjbvd = 1.0;
  else if ((m.xjbvd < 0.0) && (m.dioMod == 0))
    m.xjbvd = 1.0;
  if (m.bvd <= 0.0) m.bvd = 10.0;
  if ((m.xjbvs <= 0.0) && (m.dioMod == 2))
    m.xjbvs = 1.0;
  else if ((m.xjbvs < 0.0) && (m.dioMod == 0))
    m.xjbvs = 1.0;
  if (m.bvs <= 0.0) m.bvs = 10.0;
}

double ni_at(const ModelState &ms) {
  const double Tnom = ms.c.tnom;
  const double Vtm0 = ms.vtm0;
  return 1.45e10 * (Tnom / 300.15) * sqrt(Tnom / 300.15) * exp(21.5565981 - ms.Eg0 / (2.0 * Vtm0));
}

// ---- Size-dependent set (updateTemperature, B4.C:6035-7115) ----
Size *get_size(ModelState &ms, const InstParams &ip, double temp, std::string &err) {
  for (auto &s : ms.sizes)
    if (s->Length == ip.l && s->Width == ip.w && s->NFinger == ip.nf) return s.get();
  const Card &m = ms.c;
  const double nf = ip.nf;
  const double Tnom = m.tnom;
  const double TRatio = temp / Tnom;
  const double delTemp = temp - Tnom;
  const double epssub = CONSTEPSSI;
  const double toxe = m.toxe;
  const double epsrox = m.epsrox;
  const double Vtm0 = ms.vtm0;
  const double Eg0 = ms.Eg0;
  const double ni = ni_at(ms);
  const double Ldrn = ip.l;
  std::unique_ptr<Size> sp(new Size());
  Size &p = *sp;
  p.Length = ip.l;
  p.Width = ip.w;
  p.NFinger = ip.nf;
  const double Lnew = ip.l + m.xl;
  const double Wnew = ip.w / nf + m.xw;
  double T0 = pow(Lnew, m.Lln);
  double T1 = pow(Wnew, m.Lwn);
  double tmp1 = m.Ll / T0 + m.Lw / T1 + m.Lwl / (T0 * T1);
  p.dl = m.Lint + tmp1;
  double tmp2 = m.Llc / T0 + m.Lwc / T1 + m.Lwlc / (T0 * T1);
  p.dlc = m.dlc + tmp2;
  double T2 = pow(Lnew, m.Wln);
  double T3 = pow(Wnew, m.Wwn);
  tmp1 = m.Wl / T2 + m.Ww / T3 + m.Wwl / (T2 * T3);
  p.dw = m.Wint + tmp1;
  tmp2 = m.Wlc / T2 + m.Wwc / T3 + m.Wwlc / (T2 * T3);
  p.dwc = m.dwc + tmp2;
  p.dwj = m.dwj + tmp2;
  p.leff = Lnew - 2.0 * p.dl;
  if (p.leff <= 0.0) { err = "BSIM4: effective channel length <= 0"; return nullptr; }
  p.weff = Wnew - 2.0 * p.dw;
  if (p.weff <= 0.0) { err = "BSIM4: effective channel width <= 0"; return nullptr; }
  p.leffCV = Lnew - 2.0 * p.dlc;
  if (p.leffCV <= 0.0) { err = "BSIM4: effective channel length for C-V <= 0"; return nullptr; }
  p.weffCV = Wnew - 2.0 * p.dwc;
  if (p.weffCV <= 0.0) { err = "BSIM4: effective channel width for C-V <= 0"; return nullptr; }
  p.weffCJ = Wnew - 2.0 * p.dwj;
  if (p.weffCJ <= 0.0) { err = "BSIM4: effective channel width for S/D junctions <= 0"; return nullptr; }
  double Inv_L, Inv_W, Inv_LW;
  if (m.binUnit == 1) {
    Inv_L = 1.0e-6 / p.leff;
    Inv_W = 1.0e-6 / p.weff;
    Inv_LW = 1.0e-12 / (p.leff * p.weff);
  } else {
    Inv_L = 1.0 / p.leff;
    Inv_W = 1.0 / p.weff;
    Inv_LW = 1.0 / (p.leff * p.weff);
  }
#define B4BIN(mem, base, l, w, pp) p.mem = m.base + m.l * Inv_L + m.w * Inv_W + m.pp * Inv_LW;
#include "bsim4_bins.inc"
#undef B4BIN
  p.abulkCVfactor = 1.0 + pow((p.clc / p.leffCV), p.cle);
  T0 = (TRatio - 1.0);
  const double PowWeffWr = pow(p.weffCJ * 1.0e6, p.wr) * nf;
  T1 = T2 = T3 = 0.0;
  double T4 = 0.0;
  if (m.tempMod == 0) {
    p.ua = p.ua + p.ua1 * T0;
    p.ub = p.ub + p.ub1 * T0;
    p.uc = p.uc + p.uc1 * T0;
    p.ud = p.ud + p.ud1 * T0;
    p.vsattemp = p.vsat - p.at * T0;
    double T10 = p.prt * T0;
    if (m.rdsMod) {
      T1 = p.rdw + T10;
      T2 = m.rdwmin + T10;
      T3 = p.rsw + T10;
      T4 = m.rswmin + T10;
    }
    p.rds0 = (p.rdsw + T10) * nf / PowWeffWr;
    p.rdswmin = (m.rdswmin + T10) * nf / PowWeffWr;
  } else {
    p.ua = p.ua * (1.0 + p.ua1 * delTemp);
    p.ub = p.ub * (1.0 + p.ub1 * delTemp);
    p.uc = p.uc * (1.0 + p.uc1 * delTemp);
    p.ud = p.ud * (1.0 + p.ud1 * delTemp);
    p.vsattemp = p.vsat * (1.0 - p.at * delTemp);
    double T10 = 1.0 + p.prt * delTemp;
    if (m.rdsMod) {
      T1 = p.rdw * T10;
      T2 = m.rdwmin * T10;
      T3 = p.rsw * T10;
      T4 = m.rswmin * T10;
    }
    p.rds0 = p.rdsw * T10 * nf / PowWeffWr;
    p.rdswmin = m.rdswmin * T10 * nf / PowWeffWr;
  }
  if (T1 < 0.0) T1 = 0.0;
  if (T2 < 0.0) T2 = 0.0;
  p.rd0 = T1 / PowWeffWr;
  p.rdwmin = T2 / PowWeffWr;
  if (T3 < 0.0) T3 = 0.0;
  if (T4 < 0.0) T4 = 0.0;
  p.rs0 = T3 / PowWeffWr;
  p.rswmin = T4 / PowWeffWr;
  if (p.u0 > 1.0) p.u0 = p.u0 / 1.0e4;
  double T5 = 1.0 - p.up * exp(-p.leff / p.lp);
  p.u0temp = p.u0 * T5 * pow(TRatio, p.ute);
  if (p.eu < 0.0) p.eu = 0.0;
  p.vfbsdoff = p.vfbsdoff * (1.0 + p.tvfbsdoff * delTemp);
  p.voff = p.voff * (1.0 + p.tvoff * delTemp);
  if ((m.g("VTL")) && (m.vtl > 0.0)) {
    if (m.lc < 0.0)
      p.lc = 0.0;
    else
      p.lc = m.lc;
    T0 = p.leff / (p.xn * p.leff + p.lc);
    p.tfactor = (1.0 - T0) / (1.0 + T0);
  }
  p.cgdo = (m.cgdo + p.cf) * p.weffCV;
  p.cgso = (m.cgso + p.cf) * p.weffCV;
  p.cgbo = m.cgbo * p.leffCV * nf;
  if (!m.g("NDEP") && m.g("GAMMA1")) {
    T0 = p.gamma1 * ms.coxe;
    p.ndep = 3.01248e22 * T0 * T0;
  }
  p.phi = Vtm0 * log(p.ndep / ni) + p.phin + 0.4;
  p.sqrtPhi = sqrt(p.phi);
  p.phis3 = p.sqrtPhi * p.phi;
  p.Xdep0 = sqrt(2.0 * epssub / (Charge_q * p.ndep * 1.0e6)) * p.sqrtPhi;
  p.sqrtXdep0 = sqrt(p.Xdep0);
  p.litl = sqrt(3.0 * p.xj * toxe);
  p.vbi = Vtm0 * log(p.nsd * p.ndep / (ni * ni));
  if (p.ngate > 0.0)
    p.vfbsd = Vtm0 * log(p.ngate / p.nsd);
  else
    p.vfbsd = 0.0;
  p.cdep0 = sqrt(Charge_q * epssub * p.ndep * 1.0e6 / 2.0 / p.phi);
  p.ToxRatio = exp(p.ntox * log(m.toxref / toxe)) / toxe / toxe;
  p.ToxRatioEdge = exp(p.ntox * log(m.toxref / (toxe * p.poxedge))) / toxe / toxe / p.poxedge / p.poxedge;
  p.Aechvb = (m.dtype == CONSTNMOS) ? 4.97232e-7 : 3.42537e-7;
  p.Bechvb = (m.dtype == CONSTNMOS) ? 7.45669e11 : 1.16645e12;
  p.AechvbEdgeS = p.Aechvb * p.weff * m.dlcig * p.ToxRatioEdge;
  p.AechvbEdgeD = p.Aechvb * p.weff * m.dlcigd * p.ToxRatioEdge;
  p.BechvbEdge = -p.Bechvb * m.toxe * p.poxedge;
  p.Aechvb *= p.weff * p.leff * p.ToxRatio;
  p.Bechvb *= -toxe;
  p.mstar = 0.5 + atan(p.minv) / M_PI;
  p.mstarcv = 0.5 + atan(p.minvcv) / M_PI;
  p.voffcbn = p.voff + m.voffl / p.leff;
  p.voffcbncv = p.voffcv + m.voffcvl / p.leff;
  p.ldeb = sqrt(epssub * Vtm0 / (Charge_q * p.ndep * 1.0e6)) / 3.0;
  p.acde *= pow((p.ndep / 2.0e16), -0.25);
  if (m.g("K1") || m.g("K2")) {
    if (!m.g("K1")) p.k1 = 0.53;
    if (!m.g("K2")) p.k2 = -0.0186;
  } else {
    if (!m.g("VBX")) p.vbx = p.phi - 7.7348e-4 * p.ndep * p.xt * p.xt;
    if (p.vbx > 0.0) p.vbx = -p.vbx;
    if (p.vbm > 0.0) p.vbm = -p.vbm;
    if (!m.g("GAMMA1")) p.gamma1 = 5.753e-12 * sqrt(p.ndep) / ms.coxe;
    if (!m.g("GAMMA2")) p.gamma2 = 5.753e-12 * sqrt(p.nsub) / ms.coxe;
    T0 = p.gamma1 - p.gamma2;
    T1 = sqrt(p.phi - p.vbx) - p.sqrtPhi;
    T2 = sqrt(p.phi * (p.phi - p.vbm)) - p.phi;
    p.k2 = T0 * T1 / (2.0 * T2 + p.vbm);
    p.k1 = p.gamma2 - 2.0 * p.k2 * sqrt(p.phi - p.vbm);
  }
  if (!m.g("VFB")) {
    if (m.g("VTH0"))
      p.vfb = m.dtype * p.vth0 - p.phi - p.k1 * p.sqrtPhi;
    else
      p.vfb = -1.0;
  }
  if (!m.g("VTH0")) p.vth0 = m.dtype * (p.vfb + p.phi + p.k1 * p.sqrtPhi);
  p.k1ox = p.k1 * toxe / m.toxm;
  double tmp = sqrt(epssub / (epsrox * CONSTEPS0) * toxe * p.Xdep0);
  T0 = p.dsub * p.leff / tmp;
  if (T0 < CONSTEXP_THRESHOLD) {
    T1 = exp(T0);
    T2 = T1 - 1.0;
    T3 = T2 * T2;
    T4 = T3 + 2.0 * T1 * CONSTMIN_EXP;
    p.theta0vb0 = T1 / T4;
  } else {
    p.theta0vb0 = 1.0 / (CONSTMAX_EXP - 2.0);
  }
  T0 = p.drout * p.leff / tmp;
  if (T0 < CONSTEXP_THRESHOLD) {
    T1 = exp(T0);
    T2 = T1 - 1.0;
    T3 = T2 * T2;
    T4 = T3 + 2.0 * T1 * CONSTMIN_EXP;
    T5 = T1 / T4;
  } else {
    T5 = 1.0 / (CONSTMAX_EXP - 2.0);
  }
  p.thetaRout = p.pdibl1 * T5 + p.pdibl2;
  tmp = sqrt(p.Xdep0);
  tmp1 = p.vbi - p.phi;
  tmp2 = ms.factor1 * tmp;
  T0 = p.dvt1w * p.weff * p.leff / tmp2;
  double T8, T9;
  if (T0 < CONSTEXP_THRESHOLD) {
    T1 = exp(T0);
    T2 = T1 - 1.0;
    T3 = T2 * T2;
    T4 = T3 + 2.0 * T1 * CONSTMIN_EXP;
    T8 = T1 / T4;
  } else {
    T8 = 1.0 / (CONSTMAX_EXP - 2.0);
  }
  T0 = p.dvt0w * T8;
  T8 = T0 * tmp1;
  T0 = p.dvt1 * p.leff / tmp2;
  if (T0 < CONSTEXP_THRESHOLD) {
    T1 = exp(T0);
    T2 = T1 - 1.0;
    T3 = T2 * T2;
    T4 = T3 + 2.0 * T1 * CONSTMIN_EXP;
    T9 = T1 / T4;
  } else {
    T9 = 1.0 / (CONSTMAX_EXP - 2.0);
  }
  T9 = p.dvt0 * T9 * tmp1;
  T4 = toxe * p.phi / (p.weff + p.w0);
  T0 = sqrt(1.0 + p.lpe0 / p.leff);
  T3 = 0.0;
  if ((m.tempMod == 1) || (m.tempMod == 0)) T3 = (p.kt1 + p.kt1l / p.leff) * (TRatio - 1.0);
  if (m.tempMod == 2) T3 = -p.kt1 * (TRatio - 1.0);
  T5 = p.k1ox * (T0 - 1.0) * p.sqrtPhi + T3;
  p.vfbzbfactor = -T8 - T9 + p.k3 * T4 + T5 - p.phi - p.k1 * p.sqrtPhi;
  double wlod = m.wlod;
  if (m.wlod < 0.0) wlod = 0.0;
  T0 = pow(Lnew, m.llodku0);
  const double W_tmp = Wnew + wlod;
  T1 = pow(W_tmp, m.wlodku0);
  tmp1 = m.lku0 / T0 + m.wku0 / T1 + m.pku0 / (T0 * T1);
  p.ku0 = 1.0 + tmp1;
  T0 = pow(Lnew, m.llodvth);
  T1 = pow(W_tmp, m.wlodvth);
  tmp1 = m.lkvth0 / T0 + m.wkvth0 / T1 + m.pkvth0 / (T0 * T1);
  p.kvth0 = 1.0 + tmp1;
  p.kvth0 = sqrt(p.kvth0 * p.kvth0 + DELTA);
  T0 = (TRatio - 1.0);
  p.ku0temp = p.ku0 * (1.0 + m.tku0 * T0) + DELTA;
  const double Inv_saref = 1.0 / (m.saref + 0.5 * Ldrn);
  const double Inv_sbref = 1.0 / (m.sbref + 0.5 * Ldrn);
  p.inv_od_ref = Inv_saref + Inv_sbref;
  p.rho_ref = m.ku0 / p.ku0temp * p.inv_od_ref;
  ms.sizes.push_back(std::move(sp));
  return ms.sizes.back().get();
}

void num_finger_diff(double nf_arg, int minSD, double &nuIntD, double &nuEndD, double &nuIntS, double &nuEndS) {
  int NF = static_cast<int>(nf_arg);
  if ((NF % 2) != 0) {
    nuEndD = nuEndS = 1.0;
    nuIntD = nuIntS = 2.0 * std::max((nf_arg - 1.0) / 2.0, 0.0);
  } else {
    if (minSD == 1) {
      nuEndD = 2.0;
      nuIntD = 2.0 * std::max((nf_arg / 2.0 - 1.0), 0.0);
      nuEndS = 0.0;
      nuIntS = nf_arg;
    } else {
      nuEndD = 0.0;
      nuIntD = nf_arg;
      nuEndS = 2.0;
      nuIntS = 2.0 * std::max((nf_arg / 2.0 - 1.0), 0.0);
    }
  }
}

void pa_eff_geo(double nf_arg, int geo, int minSD, double Weffcj, double DMCG, double DMCI, double DMDG, double &Ps,
                double &Pd, double &As, double &Ad) {
  double nuIntD = 0, nuEndD = 0, nuIntS = 0, nuEndS = 0;
  if (geo < 9) num_finger_diff(nf_arg, minSD, nuIntD, nuEndD, nuIntS, nuEndS);
  const double T0 = DMCG + DMCI, T1 = DMCG + DMCG, T2 = DMDG + DMDG;
  const double PSiso = T0 + T0 + Weffcj, PDiso = PSiso, PSsha = T1, PDsha = T1, PSmer = T2, PDmer = T2;
  const double ASiso = T0 * Weffcj, ADiso = ASiso, ASsha = DMCG * Weffcj, ADsha = ASsha, ASmer = DMDG * Weffcj,
               ADmer = ASmer;
  switch (geo) {
    case 0: Ps = nuEndS * PSiso + nuIntS * PSsha; Pd = nuEndD * PDiso + nuIntD * PDsha;
            As = nuEndS * ASiso + nuIntS * ASsha; Ad = nuEndD * ADiso + nuIntD * ADsha; break;
    case 1: Ps = nuEndS * PSiso + nuIntS * PSsha; Pd = (nuEndD + nuIntD) * PDsha;
            As = nuEndS * ASiso + nuIntS * ASsha; Ad = (nuEndD + nuIntD) * ADsha; break;
    case 2: Ps = (nuEndS + nuIntS) * PSsha; Pd = nuEndD * PDiso + nuIntD * PDsha;
            As = (nuEndS + nuIntS) * ASsha; Ad = nuEndD * ADiso + nuIntD * ADsha; break;
    case 3: Ps = (nuEndS + nuIntS) * PSsha; Pd = (nuEndD + nuIntD) * PDsha;
            As = (nuEndS + nuIntS) * ASsha; Ad = (nuEndD + nuIntD) * ADsha; break;
    case 4: Ps = nuEndS * PSiso + nuIntS * PSsha; Pd = nuEndD * PDmer + nuIntD * PDsha;
            As = nuEndS * ASiso + nuIntS * ASsha; Ad = nuEndD * ADmer + nuIntD * ADsha; break;
    case 5: Ps = (nuEndS + nuIntS) * PSsha; Pd = nuEndD * PDmer + nuIntD * PDsha;
            As = (nuEndS + nuIntS) * ASsha; Ad = nuEndD * ADmer + nuIntD * ADsha; break;
    case 6: Ps = nuEndS * PSmer + nuIntS * PSsha; Pd = nuEndD * PDiso + nuIntD * PDsha;
            As = nuEndS * ASmer + nuIntS * ASsha; Ad = nuEndD * ADiso + nuIntD * ADsha; break;
    case 7: Ps = nuEndS * PSmer + nuIntS * PSsha; Pd = (nuEndD + nuIntD) * PDsha;
            As = nuEndS * ASmer + nuIntS * ASsha; Ad = (nuEndD + nuIntD) * ADsha; break;
    case 8: Ps = nuEndS * PSmer + nuIntS * PSsha; Pd = nuEndD * PDmer + nuIntD * PDsha;
            As = nuEndS * ASmer + nuIntS * ASsha; Ad = nuEndD * ADmer + nuIntD * ADsha; break;
    case 9: Ps = PSiso + (nf_arg - 1.0) * PSsha; Pd = nf_arg * PDsha;
            As = ASiso + (nf_arg - 1.0) * ASsha; Ad = nf_arg * ADsha; break;
    case 10: Ps = nf_arg * PSsha; Pd = PDiso + (nf_arg - 1.0) * PDsha;
             As = nf_arg * ASsha; Ad = ADiso + (nf_arg - 1.0) * ADsha; break;
    default: break;
  }
}

double dio_ijth_vjm(double Nvtm, double Ijth, double Isb, double XExpBV) {
  const double Tc = XExpBV;
  const double Tb = 1.0 + Ijth / Isb - Tc;
  const double EVjmovNv = 0.5 * (Tb + sqrt(Tb * Tb + 4.0 * Tc));
  return Nvtm * log(EVjmovNv);
}

// ---- Instance-level part (updateTemperature, B4.C:7116-7570) -> one record ----
std::string instance_record(ModelState &ms, const InstParams &ipin, const SetupOptions &opts, std::vector<double> &rec) {
  InstParams ip = ipin;
  Card &m = ms.c;
  // Instance::Instance defaults for parameters not given on the instance line.
  if (!ip.g("RBDB")) ip.rbdb = m.rbdb;
  if (!ip.g("RBSB")) ip.rbsb = m.rbsb;
  if (!ip.g("RBPB")) ip.rbpb = m.rbpb;
  if (!ip.g("RBPS")) ip.rbps = m.rbps;
  if (!ip.g("RBPD")) ip.rbpd = m.rbpd;
  if (!ip.g("XGW")) ip.xgw = m.xgw;
  if (!ip.g("NGCON")) ip.ngcon = m.ngcon;
  if (!ip.g("SD")) ip.sd = 2.0 * m.dmcg;
  if (!ip.g("TEMP")) ip.temp = opts.temp_c + CONSTCtoK;
  if (!ip.g("AD")) ip.drainArea = 0.0;
  if (!ip.g("AS")) ip.sourceArea = 0.0;
  // Instance::processParams mode selection (:3618-3672): an instance value outside the range falls
  // back to the model's.
  if (!ip.g("RBODYMOD") || (ip.rbodyMod != 0 && ip.rbodyMod != 1 && ip.rbodyMod != 2)) ip.rbodyMod = m.rbodyMod;
  if (!ip.g("RGATEMOD") || (ip.rgateMod != 0 && ip.rgateMod != 1 && ip.rgateMod != 2 && ip.rgateMod != 3))
    ip.rgateMod = m.rgateMod;
  if (!ip.g("GEOMOD")) ip.geoMod = m.geoMod;
  if (!ip.g("RGEOMOD")) ip.rgeoMod = 0;
  if (!ip.g("TRNQSMOD") || (ip.trnqsMod != 0 && ip.trnqsMod != 1)) ip.trnqsMod = m.trnqsMod;
  if (!ip.g("ACNQSMOD") || (ip.acnqsMod != 0 && ip.acnqsMod != 1)) ip.acnqsMod = m.acnqsMod;
  // Geometry-derived source / drain resistance (RdseffGeo) applies where a sheet resistance or
  // rdsMod asks for a resistance and the instance gives no squares.
  if (ip.rgeoMod != 0 && (m.sheetResistance > 0.0 || m.rdsMod != 0) && (!ip.g("NRD") || !ip.g("NRS")))
    return "BSIM4 rgeoMod != 0 without NRD / NRS (geometry-derived source/drain resistance) is not supported";
  const double temp = ip.temp;
  if (!ms.temp_done) {
    model_temperature(ms, temp);
    ms.temp_done = true;
    ms.temp_seen = temp;
  } else if (temp != ms.temp_seen) {
    return "BSIM4 instances of one model must share one temperature";
  }
  std::string err;
  Size *pp = get_size(ms, ip, temp, err);
  if (!pp) return err;
  const Size &p = *pp;
  const double nf = ip.nf;
  const double Tnom = m.tnom;
  const double TRatio = temp / Tnom;
  const double toxe = m.toxe;
  const double Ldrn = ip.l;
  const double Wdrn = ip.w / nf;
  const double Lnew = ip.l + m.xl;
  double T0, T1, T2, T3, T4, T5, T6, T7, T9, T10;
  double u0temp, vth0, vsattemp, eta0, k2;
  if ((ip.sa > 0.0) && (ip.sb > 0.0) && ((nf == 1.0) || ((nf > 1.0) && (ip.sd > 0.0)))) {
    double Inv_sa = 0, Inv_sb = 0;
    double kvsat = m.kvsat;
    if (m.kvsat < -1.0) kvsat = -1.0;
    if (m.kvsat > 1.0) kvsat = 1.0;
    for (int i = 0; i < nf; i++) {
      T0 = 1.0 / nf / (ip.sa + 0.5 * Ldrn + i * (ip.sd + Ldrn));
      T1 = 1.0 / nf / (ip.sb + 0.5 * Ldrn + i * (ip.sd + Ldrn));
      Inv_sa += T0;
      Inv_sb += T1;
    }
    const double Inv_ODeff = Inv_sa + Inv_sb;
    const double rho = m.ku0 / p.ku0temp * Inv_ODeff;
    T0 = (1.0 + rho) / (1.0 + p.rho_ref);
    u0temp = p.u0temp * T0;
    T1 = (1.0 + kvsat * rho) / (1.0 + kvsat * p.rho_ref);
    vsattemp = p.vsattemp * T1;
    const double OD_offset = Inv_ODeff - p.inv_od_ref;
    const double dvth0_lod = m.kvth0 / p.kvth0 * OD_offset;
    const double dk2_lod = m.stk2 / pow(p.kvth0, m.lodk2) * OD_offset;
    const double deta0_lod = m.steta0 / pow(p.kvth0, m.lodeta0) * OD_offset;
    vth0 = p.vth0 + dvth0_lod;
    eta0 = p.eta0 + deta0_lod;
    k2 = p.k2 + dk2_lod;
  } else {
    u0temp = p.u0temp;
    vth0 = p.vth0;
    vsattemp = p.vsattemp;
    eta0 = p.eta0;
    k2 = p.k2;
  }
  if (m.wpemod) {
    double sca = ip.sca, scb = ip.scb, scc = ip.scc;
    if ((!ip.g("SCA")) && (!ip.g("SCB")) && (!ip.g("SCC"))) {
      if ((ip.g("SC")) && (ip.sc > 0.0)) {
        T1 = ip.sc + Wdrn;
        T2 = 1.0 / m.scref;
        sca = m.scref * m.scref / (ip.sc * T1);
        scb = ((0.1 * ip.sc + 0.01 * m.scref) * exp(-10.0 * ip.sc * T2) -
               (0.1 * T1 + 0.01 * m.scref) * exp(-10.0 * T1 * T2)) / Wdrn;
        scc = ((0.05 * ip.sc + 0.0025 * m.scref) * exp(-20.0 * ip.sc * T2) -
               (0.05 * T1 + 0.0025 * m.scref) * exp(-20.0 * T1 * T2)) / Wdrn;
      }
    }
    const double sceff = sca + m.web * scb + m.wec * scc;
    vth0 += p.kvth0we * sceff;
    k2 += p.k2we * sceff;
    T3 = 1.0 + p.ku0we * sceff;
    if (T3 <= 0.0) T3 = 0.0;
    u0temp *= T3;
  }
  vth0 += ip.delvto;
  const double vfb = p.vfb + m.dtype * ip.delvto;
  T3 = m.dtype * vth0 - vfb - p.phi;
  T4 = T3 + T3;
  T5 = 2.5 * T3;
  double vtfbphi1 = (m.dtype == CONSTNMOS) ? T4 : T5;
  if (vtfbphi1 < 0.0) vtfbphi1 = 0.0;
  double vtfbphi2 = 4.0 * T3;
  if (vtfbphi2 < 0.0) vtfbphi2 = 0.0;
  double vbsc;
  if (k2 < 0.0) {
    T0 = 0.5 * p.k1 / k2;
    vbsc = 0.9 * (p.phi - T0 * T0);
    if (vbsc > -3.0)
      vbsc = -3.0;
    else if (vbsc < -30.0)
      vbsc = -30.0;
  } else {
    vbsc = -30.0;
  }
  if (vbsc > p.vbm) vbsc = p.vbm;
  const double k2ox = k2 * toxe / m.toxm;
  const double vfbzb = p.vfbzbfactor + m.dtype * vth0;
  // Body resistance network (:7218-7309): rbodyMod 2 scales the resistances with geometry; the
  // conductances get gbmin added, and a resistance below 1 mOhm becomes 1e3 S.
  double rbdb = ip.rbdb, rbsb = ip.rbsb, rbpb = ip.rbpb, rbps = ip.rbps, rbpd = ip.rbpd;
  double grbdb = 0.0, grbpb = 0.0, grbps = 0.0, grbsb = 0.0, grbpd = 0.0;
  {
    const double lnl = log(p.leff * 1.0e6);
    const double lnw = log(p.weff * 1.0e6);
    const double lnnf = log(nf);
    int bodymode = 5;
    if ((!m.g("RBPS0")) || (!m.g("RBPD0")))
      bodymode = 1;
    else if ((!m.g("RBSBX0") && !m.g("RBSBY0")) || (!m.g("RBDBX0") && !m.g("RBDBY0")))
      bodymode = 3;
    if (ip.rbodyMod == 2) {
      if (bodymode == 5) {
        const double rbsbx = exp(log(m.rbsbx0) + m.rbsdbxl * lnl + m.rbsdbxw * lnw + m.rbsdbxnf * lnnf);
        const double rbsby = exp(log(m.rbsby0) + m.rbsdbyl * lnl + m.rbsdbyw * lnw + m.rbsdbynf * lnnf);
        rbsb = rbsbx * rbsby / (rbsbx + rbsby);
        const double rbdbx = exp(log(m.rbdbx0) + m.rbsdbxl * lnl + m.rbsdbxw * lnw + m.rbsdbxnf * lnnf);
        const double rbdby = exp(log(m.rbdby0) + m.rbsdbyl * lnl + m.rbsdbyw * lnw + m.rbsdbynf * lnnf);
        rbdb = rbdbx * rbdby / (rbdbx + rbdby);
      }
      if ((bodymode == 3) || (bodymode == 5)) {
        rbps = exp(log(m.rbps0) + m.rbpsl * lnl + m.rbpsw * lnw + m.rbpsnf * lnnf);
        rbpd = exp(log(m.rbpd0) + m.rbpdl * lnl + m.rbpdw * lnw + m.rbpdnf * lnnf);
      }
      const double rbpbx = exp(log(m.rbpbx0) + m.rbpbxl * lnl + m.rbpbxw * lnw + m.rbpbxnf * lnnf);
      const double rbpby = exp(log(m.rbpby0) + m.rbpbyl * lnl + m.rbpbyw * lnw + m.rbpbynf * lnnf);
      rbpb = rbpbx * rbpby / (rbpbx + rbpby);
    }
    if ((ip.rbodyMod == 1) || ((ip.rbodyMod == 2) && (bodymode == 5))) {
      grbdb = (rbdb < 1.0e-3) ? 1.0e3 : m.gbmin + 1.0 / rbdb;
      grbpb = (rbpb < 1.0e-3) ? 1.0e3 : m.gbmin + 1.0 / rbpb;
      grbps = (rbps < 1.0e-3) ? 1.0e3 : m.gbmin + 1.0 / rbps;
      grbsb = (rbsb < 1.0e-3) ? 1.0e3 : m.gbmin + 1.0 / rbsb;
      grbpd = (rbpd < 1.0e-3) ? 1.0e3 : m.gbmin + 1.0 / rbpd;
    }
    if ((ip.rbodyMod == 2) && (bodymode == 3)) {
      grbdb = grbsb = m.gbmin;
      grbpb = (rbpb < 1.0e-3) ? 1.0e3 : m.gbmin + 1.0 / rbpb;
      grbps = (rbps < 1.0e-3) ? 1.0e3 : m.gbmin + 1.0 / rbps;
      grbpd = (rbpd < 1.0e-3) ? 1.0e3 : m.gbmin + 1.0 / rbpd;
    }
    if ((ip.rbodyMod == 2) && (bodymode == 1)) {
      grbdb = grbsb = m.gbmin;
      grbps = grbpd = 1.0e3;
      grbpb = (rbpb < 1.0e-3) ? 1.0e3 : m.gbmin + 1.0 / rbpb;
    }
  }
  double grgeltd = m.rshg * (ip.xgw + p.weffCJ / 3.0 / ip.ngcon) / (ip.ngcon * nf * (Lnew - m.xgl));
  if (grgeltd > 0.0)
    grgeltd = 1.0 / grgeltd;
  else
    grgeltd = 1.0e3;
  const double DMCGeff = m.dmcg - m.dmcgt;
  const double DMCIeff = m.dmci;
  const double DMDGeff = m.dmdg - m.dmcgt;
  double Pseff = 0, Pdeff = 0, Aseff = 0, Adeff = 0, dumPs = 0, dumPd = 0, dumAs = 0, dumAd = 0;
  const int geoMod = (int)ip.geoMod, minSD = (int)ip.min;
  if (ip.g("PS")) {
    if (m.perMod == 0)
      Pseff = ip.sourcePerimeter;
    else
      Pseff = ip.sourcePerimeter - p.weffCJ * nf;
  } else {
    pa_eff_geo(nf, geoMod, minSD, p.weffCJ, DMCGeff, DMCIeff, DMDGeff, Pseff, dumPd, dumAs, dumAd);
  }
  if (ip.g("PD")) {
    if (m.perMod == 0)
      Pdeff = ip.drainPerimeter;
    else
      Pdeff = ip.drainPerimeter - p.weffCJ * nf;
  } else {
    pa_eff_geo(nf, geoMod, minSD, p.weffCJ, DMCGeff, DMCIeff, DMDGeff, dumPs, Pdeff, dumAs, dumAd);
  }
  if (ip.g("AS"))
    Aseff = ip.sourceArea;
  else
    pa_eff_geo(nf, geoMod, minSD, p.weffCJ, DMCGeff, DMCIeff, DMDGeff, dumPs, dumPd, Aseff, dumAd);
  if (ip.g("AD"))
    Adeff = ip.drainArea;
  else
    pa_eff_geo(nf, geoMod, minSD, p.weffCJ, DMCGeff, DMCIeff, DMDGeff, dumPs, dumPd, dumAs, Adeff);
  // Source / drain series resistance (:7378-7447): sheet resistance times the given number of
  // squares; no squares (rdsMod 1) or a zero product give 1e3 S. The internal node exists with
  // rdsMod 1, or when the sheet resistance and the squares are both positive (:3684-3760).
  double sourceConductance = 0.0, drainConductance = 0.0;
  if (m.rdsMod != 0 || ip.g("NRS")) {
    sourceConductance = ip.g("NRS") ? m.sheetResistance * ip.sourceSquares : 0.0;
    sourceConductance = (sourceConductance > 0.0) ? 1.0 / sourceConductance : 1.0e3;
  }
  if (m.rdsMod != 0 || ip.g("NRD")) {
    drainConductance = ip.g("NRD") ? m.sheetResistance * ip.drainSquares : 0.0;
    drainConductance = (drainConductance > 0.0) ? 1.0 / drainConductance : 1.0e3;
  }
  const bool dExists = m.rdsMod != 0 || (m.sheetResistance > 0.0 && ip.g("NRD") && ip.drainSquares > 0.0);
  const bool sExists = m.rdsMod != 0 || (m.sheetResistance > 0.0 && ip.g("NRS") && ip.sourceSquares > 0.0);
  double XExpBVS = 0, XExpBVD = 0, vjsmFwd = 0, vjsmRev = 0, vjdmFwd = 0, vjdmRev = 0;
  double IVjsmFwd = 0, IVjsmRev = 0, IVjdmFwd = 0, IVjdmRev = 0, SslpFwd = 0, SslpRev = 0, DslpFwd = 0, DslpRev = 0;
  const double Nvtms = ms.vtm * m.SjctEmissionCoeff;
  double SourceSatCurrent;
  if ((Aseff <= 0.0) && (Pseff <= 0.0))
    SourceSatCurrent = 1.0e-14;
  else
    SourceSatCurrent = Aseff * ms.SjctTempSatCurDensity + Pseff * ms.SjctSidewallTempSatCurDensity +
                       p.weffCJ * nf * ms.SjctGateSidewallTempSatCurDensity;
  if (SourceSatCurrent > 0.0) {
    switch ((int)m.dioMod) {
      case 0:
        if ((m.bvs / Nvtms) > CONSTEXP_THRESHOLD)
          XExpBVS = m.xjbvs * CONSTMIN_EXP;
        else
          XExpBVS = m.xjbvs * exp(-m.bvs / Nvtms);
        break;
      case 1:
        vjsmFwd = dio_ijth_vjm(Nvtms, m.ijthsfwd, SourceSatCurrent, 0.0);
        IVjsmFwd = SourceSatCurrent * exp(vjsmFwd / Nvtms);
        break;
      case 2: {
        if ((m.bvs / Nvtms) > CONSTEXP_THRESHOLD) {
          XExpBVS = m.xjbvs * CONSTMIN_EXP;
        } else {
          XExpBVS = exp(-m.bvs / Nvtms);
          XExpBVS *= m.xjbvs;
        }
        vjsmFwd = dio_ijth_vjm(Nvtms, m.ijthsfwd, SourceSatCurrent, XExpBVS);
        T0 = exp(vjsmFwd / Nvtms);
        IVjsmFwd = SourceSatCurrent * (T0 - XExpBVS / T0 + XExpBVS - 1.0);
        SslpFwd = SourceSatCurrent * (T0 + XExpBVS / T0) / Nvtms;
        T2 = m.ijthsrev / SourceSatCurrent;
        if (T2 < 1.0) T2 = 10.0;
        vjsmRev = -m.bvs - Nvtms * log((T2 - 1.0) / m.xjbvs);
        T1 = m.xjbvs * exp(-(m.bvs + vjsmRev) / Nvtms);
        IVjsmRev = SourceSatCurrent * (1.0 + T1);
        SslpRev = -SourceSatCurrent * T1 / Nvtms;
        break;
      }
      default: break;
    }
  }
  const double Nvtmd = ms.vtm * m.DjctEmissionCoeff;
  double DrainSatCurrent;
  if ((Adeff <= 0.0) && (Pdeff <= 0.0))
    DrainSatCurrent = 1.0e-14;
  else
    DrainSatCurrent = Adeff * ms.DjctTempSatCurDensity + Pdeff * ms.DjctSidewallTempSatCurDensity +
                      p.weffCJ * nf * ms.DjctGateSidewallTempSatCurDensity;
  if (DrainSatCurrent > 0.0) {
    switch ((int)m.dioMod) {
      case 0:
        if ((m.bvd / Nvtmd) > CONSTEXP_THRESHOLD)
          XExpBVD = m.xjbvd * CONSTMIN_EXP;
        else
          XExpBVD = m.xjbvd * exp(-m.bvd / Nvtmd);
        break;
      case 1:
        vjdmFwd = dio_ijth_vjm(Nvtmd, m.ijthdfwd, DrainSatCurrent, 0.0);
        IVjdmFwd = DrainSatCurrent * exp(vjdmFwd / Nvtmd);
        break;
      case 2: {
        if ((m.bvd / Nvtmd) > CONSTEXP_THRESHOLD) {
          XExpBVD = m.xjbvd * CONSTMIN_EXP;
        } else {
          XExpBVD = exp(-m.bvd / Nvtmd);
          XExpBVD *= m.xjbvd;
        }
        vjdmFwd = dio_ijth_vjm(Nvtmd, m.ijthdfwd, DrainSatCurrent, XExpBVD);
        T0 = exp(vjdmFwd / Nvtmd);
        IVjdmFwd = DrainSatCurrent * (T0 - XExpBVD / T0 + XExpBVD - 1.0);
        DslpFwd = DrainSatCurrent * (T0 + XExpBVD / T0) / Nvtmd;
        T2 = m.ijthdrev / DrainSatCurrent;
        if (T2 < 1.0) T2 = 10.0;
        vjdmRev = -m.bvd - Nvtmd * log((T2 - 1.0) / m.xjbvd);
        T1 = m.xjbvd * exp(-(m.bvd + vjdmRev) / Nvtmd);
        IVjdmRev = DrainSatCurrent * (1.0 + T1);
        DslpRev = -DrainSatCurrent * T1 / Nvtmd;
        break;
      }
      default: break;
    }
  }
  T0 = (TRatio - 1.0);
  ms.njtsstemp = m.njts * (1.0 + m.tnjts * T0);
  ms.njtsswstemp = m.njtssw * (1.0 + m.tnjtssw * T0);
  ms.njtsswgstemp = m.njtsswg * (1.0 + m.tnjtsswg * T0);
  ms.njtsdtemp = m.njtsd * (1.0 + m.tnjtsd * T0);
  ms.njtsswdtemp = m.njtsswd * (1.0 + m.tnjtsswd * T0);
  ms.njtsswgdtemp = m.njtsswgd * (1.0 + m.tnjtsswgd * T0);
  T7 = ms.Eg0 / ms.vtm * T0;
  double e1, e2, e3, e4, e5, e6;
  T9 = m.xtss * T7; dexp2(T9, e1);
  T9 = m.xtsd * T7; dexp2(T9, e2);
  T9 = m.xtssws * T7; dexp2(T9, e3);
  T9 = m.xtsswd * T7; dexp2(T9, e4);
  T9 = m.xtsswgs * T7; dexp2(T9, e5);
  T9 = m.xtsswgd * T7; dexp2(T9, e6);
  T10 = p.weffCJ * nf;
  const double SjctTempRevSatCur = e1 * Aseff * m.jtss;
  const double DjctTempRevSatCur = e2 * Adeff * m.jtsd;
  const double SswTempRevSatCur = e3 * Pseff * m.jtssws;
  const double DswTempRevSatCur = e4 * Pdeff * m.jtsswd;
  const double SswgTempRevSatCur = e5 * T10 * m.jtsswgs;
  const double DswgTempRevSatCur = e6 * T10 * m.jtsswgd;
  (void)T6;

  rec.assign(kNumFields, 0.0);
#define R(f) rec[f_##f]
  R(dtype) = m.dtype; R(mobMod) = m.mobMod; R(capMod) = m.capMod; R(dioMod) = m.dioMod; R(rdsMod) = m.rdsMod;
  R(igcMod) = m.igcMod; R(igbMod) = m.igbMod; R(tempMod) = m.tempMod; R(mtrlMod) = m.mtrlMod;
  R(cvchargeMod) = m.cvchargeMod; R(tnoiMod) = m.tnoiMod; R(xpart) = m.xpart; R(vtm) = ms.vtm; R(vtm0) = ms.vtm0;
  R(coxe) = ms.coxe; R(coxp) = ms.coxp; R(toxe_m) = m.toxe; R(toxp) = m.toxp; R(toxm) = m.toxm;
  R(epsrox_m) = m.epsrox; R(eot) = m.eot; R(epsrsub) = m.epsrsub; R(epsrgate) = m.epsrgate; R(factor1) = ms.factor1;
  R(vcrit) = ms.vcrit; R(SjctEmissionCoeff) = m.SjctEmissionCoeff; R(DjctEmissionCoeff) = m.DjctEmissionCoeff;
  R(SjctTempSatCurDensity) = ms.SjctTempSatCurDensity;
  R(SjctSidewallTempSatCurDensity) = ms.SjctSidewallTempSatCurDensity;
  R(SjctGateSidewallTempSatCurDensity) = ms.SjctGateSidewallTempSatCurDensity;
  R(DjctTempSatCurDensity) = ms.DjctTempSatCurDensity;
  R(DjctSidewallTempSatCurDensity) = ms.DjctSidewallTempSatCurDensity;
  R(DjctGateSidewallTempSatCurDensity) = ms.DjctGateSidewallTempSatCurDensity;
  R(xjbvs) = m.xjbvs; R(xjbvd) = m.xjbvd; R(bvs) = m.bvs; R(bvd) = m.bvd;
  R(njtsstemp) = ms.njtsstemp; R(njtsswstemp) = ms.njtsswstemp; R(njtsswgstemp) = ms.njtsswgstemp;
  R(njtsdtemp) = ms.njtsdtemp; R(njtsswdtemp) = ms.njtsswdtemp; R(njtsswgdtemp) = ms.njtsswgdtemp;
  R(vtss) = m.vtss; R(vtsd) = m.vtsd; R(vtssws) = m.vtssws; R(vtsswd) = m.vtsswd; R(vtsswgs) = m.vtsswgs;
  R(vtsswgd) = m.vtsswgd; R(phig) = m.phig; R(easub) = m.easub; R(Eg0) = ms.Eg0; R(ados) = m.ados; R(bdos) = m.bdos;
  R(pditsl) = m.pditsl; R(lambdaGiven) = m.g("LAMBDA") ? 1.0 : 0.0; R(vtlGiven) = m.g("VTL") ? 1.0 : 0.0;
  R(tnom) = m.tnom; R(DunitAreaTempJctCap) = ms.DunitAreaTempJctCap; R(SunitAreaTempJctCap) = ms.SunitAreaTempJctCap;
  R(DunitLengthSidewallTempJctCap) = ms.DunitLengthSidewallTempJctCap;
  R(DunitLengthGateSidewallTempJctCap) = ms.DunitLengthGateSidewallTempJctCap;
  R(SunitLengthSidewallTempJctCap) = ms.SunitLengthSidewallTempJctCap;
  R(SunitLengthGateSidewallTempJctCap) = ms.SunitLengthGateSidewallTempJctCap;
  R(SbulkJctBotGradingCoeff) = m.SbulkJctBotGradingCoeff; R(SbulkJctSideGradingCoeff) = m.SbulkJctSideGradingCoeff;
  R(SbulkJctGateSideGradingCoeff) = m.SbulkJctGateSideGradingCoeff;
  R(DbulkJctBotGradingCoeff) = m.DbulkJctBotGradingCoeff; R(DbulkJctSideGradingCoeff) = m.DbulkJctSideGradingCoeff;
  R(DbulkJctGateSideGradingCoeff) = m.DbulkJctGateSideGradingCoeff;
  R(PhiBS) = ms.PhiBS; R(PhiBSWS) = ms.PhiBSWS; R(PhiBSWGS) = ms.PhiBSWGS; R(PhiBD) = ms.PhiBD;
  R(PhiBSWD) = ms.PhiBSWD; R(PhiBSWGD) = ms.PhiBSWGD; R(lambda_m) = m.lambda; R(vtl_m) = m.vtl;
  R(phi) = p.phi; R(sqrtPhi) = p.sqrtPhi; R(Xdep0) = p.Xdep0; R(leff) = p.leff; R(vbi) = p.vbi; R(dvt2) = p.dvt2;
  R(dvt2w) = p.dvt2w; R(dvt1) = p.dvt1; R(dvt0) = p.dvt0; R(dvt1w) = p.dvt1w; R(weff) = p.weff; R(dvt0w) = p.dvt0w;
  R(lpe0) = p.lpe0; R(k1ox) = p.k1ox; R(kt1) = p.kt1; R(kt1l) = p.kt1l; R(kt2) = p.kt2; R(w0) = p.w0;
  R(etab) = p.etab; R(theta0vb0) = p.theta0vb0; R(lpeb) = p.lpeb; R(k1) = p.k1; R(k3) = p.k3; R(k3b) = p.k3b;
  R(cit) = p.cit; R(nfactor) = p.nfactor; R(cdsc) = p.cdsc; R(cdscb) = p.cdscb; R(cdscd) = p.cdscd;
  R(dvtp0) = p.dvtp0; R(dvtp1) = p.dvtp1; R(ngate) = p.ngate; R(mstar) = p.mstar; R(voffcbn) = p.voffcbn;
  R(cdep0) = p.cdep0; R(dwg) = p.dwg; R(dwb) = p.dwb; R(prwg) = p.prwg; R(prwb) = p.prwb; R(rds0) = p.rds0;
  R(rdswmin) = p.rdswmin; R(xj) = p.xj; R(a0) = p.a0; R(b1) = p.b1; R(b0) = p.b0; R(ags) = p.ags; R(keta) = p.keta;
  R(ua) = p.ua; R(uc) = p.uc; R(ub) = p.ub; R(ud) = p.ud; R(eu) = p.eu; R(a1) = p.a1; R(a2) = p.a2;
  R(delta) = p.delta; R(lambda) = p.lambda; R(litl) = p.litl; R(fprout) = p.fprout; R(pvag) = p.pvag;
  R(pclm) = p.pclm; R(thetaRout) = p.thetaRout; R(pdiblb) = p.pdiblb; R(pditsd) = p.pditsd; R(pdits) = p.pdits;
  R(pscbe1) = p.pscbe1; R(pscbe2) = p.pscbe2; R(alpha0) = p.alpha0; R(alpha1) = p.alpha1; R(beta0) = p.beta0;
  R(vtl) = p.vtl; R(tfactor) = p.tfactor; R(xrcrg1) = p.xrcrg1; R(xrcrg2) = p.xrcrg2; R(vfbsd) = p.vfbsd;
  R(egidl) = p.egidl; R(agidl) = p.agidl; R(bgidl) = p.bgidl; R(cgidl) = p.cgidl; R(weffCJ) = p.weffCJ;
  R(egisl) = p.egisl; R(agisl) = p.agisl; R(bgisl) = p.bgisl; R(cgisl) = p.cgisl;
  R(vfbcv) = p.vfbcv; R(Aechvb) = p.Aechvb; R(Bechvb) = p.Bechvb; R(AechvbEdgeS) = p.AechvbEdgeS;
  R(AechvbEdgeD) = p.AechvbEdgeD; R(BechvbEdge) = p.BechvbEdge; R(ToxRatio) = p.ToxRatio; R(aigc) = p.aigc;
  R(bigc) = p.bigc; R(cigc) = p.cigc; R(nigc) = p.nigc; R(pigcd) = p.pigcd; R(pigcdGiven) = m.g("PIGCD") ? 1 : 0;
  R(vfbsdoff) = p.vfbsdoff; R(aigs) = p.aigs; R(bigs) = p.bigs; R(cigs) = p.cigs; R(aigd) = p.aigd; R(bigd) = p.bigd;
  R(cigd) = p.cigd; R(nigbacc) = p.nigbacc; R(aigbacc) = p.aigbacc; R(bigbacc) = p.bigbacc; R(cigbacc) = p.cigbacc;
  R(nigbinv) = p.nigbinv; R(eigbinv) = p.eigbinv; R(aigbinv) = p.aigbinv; R(bigbinv) = p.bigbinv;
  R(cigbinv) = p.cigbinv;
  R(abulkCVfactor) = p.abulkCVfactor; R(weffCV) = p.weffCV; R(leffCV) = p.leffCV; R(noff) = p.noff;
  R(voffcv) = p.voffcv; R(mstarcv) = p.mstarcv; R(voffcbncv) = p.voffcbncv; R(acde) = p.acde; R(ldeb) = p.ldeb;
  R(moin) = p.moin; R(cgbo) = p.cgbo; R(cgdo) = p.cgdo; R(cgso) = p.cgso; R(cgdl) = p.cgdl; R(cgsl) = p.cgsl;
  R(ckappad) = p.ckappad; R(ckappas) = p.ckappas;
  R(vth0) = vth0; R(eta0) = eta0; R(k2ox) = k2ox; R(vfb) = vfb; R(vbsc) = vbsc; R(u0temp) = u0temp;
  R(vsattemp) = vsattemp; R(vtfbphi1) = vtfbphi1; R(vtfbphi2) = vtfbphi2; R(vfbzb) = vfbzb; R(nf) = nf;
  R(mult) = ip.mult; R(Aseff) = Aseff; R(Pseff) = Pseff; R(Adeff) = Adeff; R(Pdeff) = Pdeff; R(XExpBVS) = XExpBVS;
  R(XExpBVD) = XExpBVD; R(vjsmFwd) = vjsmFwd; R(vjsmRev) = vjsmRev; R(vjdmFwd) = vjdmFwd; R(vjdmRev) = vjdmRev;
  R(IVjsmFwd) = IVjsmFwd; R(IVjsmRev) = IVjsmRev; R(IVjdmFwd) = IVjdmFwd; R(IVjdmRev) = IVjdmRev;
  R(SslpFwd) = SslpFwd; R(SslpRev) = SslpRev; R(DslpFwd) = DslpFwd; R(DslpRev) = DslpRev;
  R(SjctTempRevSatCur) = SjctTempRevSatCur; R(SswTempRevSatCur) = SswTempRevSatCur;
  R(SswgTempRevSatCur) = SswgTempRevSatCur; R(DjctTempRevSatCur) = DjctTempRevSatCur;
  R(DswTempRevSatCur) = DswTempRevSatCur; R(DswgTempRevSatCur) = DswgTempRevSatCur;
  R(drainConductance) = drainConductance; R(sourceConductance) = sourceConductance; R(grgeltd) = grgeltd;
  R(dExists) = dExists ? 1.0 : 0.0; R(sExists) = sExists ? 1.0 : 0.0;
  R(rgateMod) = ip.rgateMod; R(rbodyMod) = ip.rbodyMod; R(rd0) = p.rd0; R(rdwmin) = p.rdwmin; R(rs0) = p.rs0;
  R(rswmin) = p.rswmin; R(grbpd) = grbpd; R(grbps) = grbps; R(grbpb) = grbpb; R(grbsb) = grbsb; R(grbdb) = grbdb;
  R(icVBS) = ip.icVBS; R(icVDS) = ip.icVDS; R(icVGS) = ip.icVGS;
  R(icVBSGiven) = ip.g("IC3") ? 1.0 : 0.0; R(icVDSGiven) = ip.g("IC1") ? 1.0 : 0.0;
  R(icVGSGiven) = ip.g("IC2") ? 1.0 : 0.0; R(trnqsMod) = ip.trnqsMod;
  R(temp) = temp; R(off) = ip.off;
#undef R
  return std::string();
}

bool set_inst_param(InstParams &ip, const std::string &name, double v) {
  static const std::map<std::string, double InstParams::*> tbl = {
      {"TEMP", &InstParams::temp}, {"L", &InstParams::l}, {"W", &InstParams::w}, {"NF", &InstParams::nf},
      {"SA", &InstParams::sa}, {"SB", &InstParams::sb}, {"SD", &InstParams::sd}, {"SCA", &InstParams::sca},
      {"SCB", &InstParams::scb}, {"SCC", &InstParams::scc}, {"SC", &InstParams::sc},
      {"AD", &InstParams::drainArea}, {"AS", &InstParams::sourceArea}, {"PD", &InstParams::drainPerimeter},
      {"PS", &InstParams::sourcePerimeter}, {"NRD", &InstParams::drainSquares},
      {"NRS", &InstParams::sourceSquares}, {"RBDB", &InstParams::rbdb}, {"RBSB", &InstParams::rbsb},
      {"RBPB", &InstParams::rbpb}, {"RBPS", &InstParams::rbps}, {"RBPD", &InstParams::rbpd},
      {"DELVTO", &InstParams::delvto}, {"XGW", &InstParams::xgw}, {"NGCON", &InstParams::ngcon},
      {"M", &InstParams::mult}, {"TRNQSMOD", &InstParams::trnqsMod}, {"ACNQSMOD", &InstParams::acnqsMod},
      {"RBODYMOD", &InstParams::rbodyMod}, {"RGATEMOD", &InstParams::rgateMod}, {"GEOMOD", &InstParams::geoMod},
      {"RGEOMOD", &InstParams::rgeoMod}, {"MIN", &InstParams::min}, {"OFF", &InstParams::off}};
  // The instance's initial conditions IC = (VDS, VGS, VBS) (:266-315).
  if (name == "IC1" || name == "IC2" || name == "IC3") {
    (name == "IC1" ? ip.icVDS : name == "IC2" ? ip.icVGS : ip.icVBS) = v;
    ip.given.insert(name);
    return true;
  }
  auto it = tbl.find(name);
  if (it == tbl.end()) return false;
  ip.*(it->second) = (name == "TEMP") ? v + CONSTCtoK : v;
  ip.given.insert(name);
  return true;
}

}  // namespace

std::string build_records(const std::vector<ModelSpec> &models, int n_inst, const int *inst_model,
                          const std::vector<std::string> &inst_param_names, const double *inst_param_values,
                          const SetupOptions &opts, RecordTable &out) {
  std::vector<std::unique_ptr<ModelState>> ms;
  for (const auto &spec : models) {
    std::unique_ptr<ModelState> s(new ModelState());
    std::string e = process_model(spec, opts, s->c);
    if (!e.empty()) return e;
    ms.push_back(std::move(s));
  }
  std::vector<std::string> names;
  for (const auto &n : inst_param_names) names.push_back(upper(n));
  const size_t np = names.size();
  // Instances with the same model and the same instance-line values share one record.
  std::map<std::pair<int, std::vector<double>>, int> key_to_rec;
  std::vector<std::vector<double>> recs;
  out.inst_rec.assign(n_inst, -1);
  for (int i = 0; i < n_inst; ++i) {
    const int mi = inst_model[i];
    if (mi < 0 || mi >= (int)ms.size()) return "instance model index out of range";
    std::vector<double> key(np);
    for (size_t k = 0; k < np; ++k) {
      double v = inst_param_values[(size_t)i * np + k];
      key[k] = std::isnan(v) ? -1.0e300 : v;
    }
    auto kk = std::make_pair(mi, key);
    auto it = key_to_rec.find(kk);
    if (it != key_to_rec.end()) {
      out.inst_rec[i] = it->second;
      continue;
    }
    InstParams ip;
    for (size_t k = 0; k < np; ++k) {
      double v = inst_param_values[(size_t)i * np + k];
      if (std::isnan(v)) continue;
      if (!set_inst_param(ip, names[k], v)) return "unknown BSIM4 instance parameter " + names[k];
    }
    std::vector<double> rec;
    std::string e = instance_record(*ms[mi], ip, opts, rec);
    if (!e.empty()) return e;
    const int r = (int)recs.size();
    recs.push_back(std::move(rec));
    key_to_rec[kk] = r;
    out.inst_rec[i] = r;
  }
  out.n_records = (int)recs.size();
  out.tab.assign((size_t)kNumFields * recs.size(), 0.0);
  for (size_t r = 0; r < recs.size(); ++r)
    for (int f = 0; f < kNumFields; ++f) out.tab[(size_t)f * recs.size() + r] = recs[r][f];
  return std::string();
}

}  // namespace xb4
