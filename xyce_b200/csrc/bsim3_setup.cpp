// Host-side BSIM3 set-up: model card, model processing, temperature and geometry precompute.
//
// Follows the reference's set-up sequence for one BSIM3 instance, in the same floating-point
// order, so that the load kernel sees the constants the reference's evaluation sees:
//   model card defaults and dependent defaults   N_DEV_MOSFET_B3.C:8573-9080 (Model::Model)
//   Model::processParams                          N_DEV_MOSFET_B3.C:8458-8548
//   instance defaults                             N_DEV_MOSFET_B3.C:2440-2500 (Instance::Instance)
//   series resistance                             N_DEV_MOSFET_B3.C:1845-1880 (Instance::processParams)
//   temperature / size / instance precompute      N_DEV_MOSFET_B3.C:3593-4488 (updateTemperature)
// The size-dependent set is created once per (L, W) per model, at the first instance's
// temperature, exactly as the reference caches SizeDependParam objects.

#include <cctype>
#include <cmath>
#include <map>
#include <memory>
#include <set>

#include "bsim3.h"

namespace xb3 {
namespace {

using namespace xdc;

constexpr double CONSTEg0 = 1.16;
constexpr double CONSTalphaEg = 7.02e-4;
constexpr double CONSTbetaEg = 1108.0;
constexpr double CONSTNi0 = 1.45e10;

struct Card {
#define B3P(name, mem, dflt) double mem = dflt;
#include "bsim3_card.inc"
#undef B3P
  std::set<std::string> given;
  int dtype = 1;
  bool g(const char *n) const { return given.count(n) != 0; }
  // Model::processParams results.
  double cox = 0, vcrit = 0, factor1 = 0, Vtm0 = 0, Eg0 = 0, ni = 0;
};

const std::map<std::string, double Card::*> &card_table() {
  static const std::map<std::string, double Card::*> t = {
#define B3P(name, mem, dflt) {name, &Card::mem},
#include "bsim3_card.inc"
#undef B3P
  };
  return t;
}

std::string upper(std::string s) {
  for (auto &c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

// Size-dependent parameter set (one per (L, W) per model).
struct Size {
#define B3BIN(mem, base, l, w, p) double mem = 0.0;
#include "bsim3_bins.inc"
#undef B3BIN
  double Length = 0, Width = 0;
  double dl = 0, dlc = 0, dw = 0, dwc = 0, leff = 0, weff = 0, leffCV = 0, weffCV = 0, abulkCVfactor = 0;
  double u0temp = 0, vsattemp = 0, rds0 = 0, cgdo = 0, cgso = 0, cgbo = 0, tconst = 0, phi = 0, sqrtPhi = 0;
  double phis3 = 0, Xdep0 = 0, sqrtXdep0 = 0, litl = 0, vbi = 0, cdep0 = 0, ldeb = 0, vbsc = 0, k1ox = 0, k2ox = 0;
  double theta0vb0 = 0, thetaRout = 0, vfbzb = 0;
};

struct ModelState {
  Card c;
  std::vector<std::unique_ptr<Size>> sizes;
  bool temp_done = false;
  double temp_seen = 0;
};

struct InstParams {
  double temp = 0, l = 0, w = 0, drainArea = 0, sourceArea = 0, drainSquares = 1.0, sourceSquares = 1.0,
         drainPerimeter = 0, sourcePerimeter = 0, mult = 1.0, nqsMod = 0, off = 0;
  std::set<std::string> given;
  bool g(const char *n) const { return given.count(n) != 0; }
};

bool set_inst(InstParams &ip, const std::string &name, double v) {
  static const std::map<std::string, double InstParams::*> tbl = {
      {"TEMP", &InstParams::temp},          {"L", &InstParams::l},
      {"W", &InstParams::w},                {"AD", &InstParams::drainArea},
      {"AS", &InstParams::sourceArea},      {"NRD", &InstParams::drainSquares},
      {"NRS", &InstParams::sourceSquares},  {"PD", &InstParams::drainPerimeter},
      {"PS", &InstParams::sourcePerimeter}, {"M", &InstParams::mult},
      {"NQSMOD", &InstParams::nqsMod},      {"OFF", &InstParams::off}};
  if (name == "IC1" || name == "IC2" || name == "IC3") {
    ip.given.insert(name);
    return true;
  }
  auto it = tbl.find(name);
  if (it == tbl.end()) return false;
  ip.*(it->second) = (name == "TEMP") ? v + CONSTCtoK : v;
  ip.given.insert(name);
  return true;
}

// ---- Model card: Model::Model dependent defaults and Model::processParams ----
std::string process_model(const xb4::ModelSpec &spec, const xb4::SetupOptions &opts, Card &m) {
  m.dtype = spec.pmos ? CONSTPMOS : CONSTNMOS;
  for (const auto &kv : spec.params) {
    const std::string n = upper(kv.first);
    if (n == "LEVEL" || n == "VERSION") continue;
    auto it = card_table().find(n);
    if (it == card_table().end()) return "unknown BSIM3 model parameter " + n;
    double v = kv.second;
    if (n == "TNOM") v += CONSTCtoK;
    m.*(it->second) = v;
    m.given.insert(n);
  }
  if (!m.g("TNOM")) m.tnom = opts.tnom_c + CONSTCtoK;
  if (!m.g("VTH0")) m.vth0 = (m.dtype == CONSTNMOS) ? 0.7 : -0.7;
  if (!m.g("UC")) m.uc = (m.mobMod == 3) ? -0.0465 : -0.0465e-9;
  if (!m.g("UC1")) m.uc1 = (m.mobMod == 3) ? -0.056 : -0.056e-9;
  if (!m.g("U0")) m.u0 = (m.dtype == CONSTNMOS) ? 0.067 : 0.025;
  if (m.capMod < 0 || m.capMod > 3)
    return "BSIM3 capMod " + std::to_string((int)m.capMod) + " is not supported (capMod 0 to 3 are)";
  // Model::processParams.
  m.cox = 3.453133e-11 / m.tox;
  if (!m.g("TOXM")) m.toxm = m.tox;
  if (!m.g("DSUB")) m.dsub = m.drout;
  if (!m.g("LLC")) m.Llc = m.Ll;
  if (!m.g("LWC")) m.Lwc = m.Lw;
  if (!m.g("LWLC")) m.Lwlc = m.Lwl;
  if (!m.g("WLC")) m.Wlc = m.Wl;
  // The reference keys this default on WWL rather than WWC, so WWC keeps its own default.
  if (!m.g("WWL")) m.Wwlc = m.Wwl;
  if (!m.g("WWLC")) m.Wwlc = m.Wwl;
  if (!m.g("DWC")) m.dwc = m.Wint;
  if (!m.g("DLC")) m.dlc = m.Lint;
  if (!m.g("CF")) {
    const double C1 = 2.0 * CONSTEPSOX;
    const double C5 = M_PI;
    const double C2 = 1.0 + (0.4e-6 / m.tox);
    const double C3 = log(C2);
    m.cf = C1 * C3 / C5;
  }
  if (!m.g("CGDO")) {
    if (m.g("DLC") && (m.dlc > 0.0))
      m.cgdo = m.dlc * m.cox - m.cgdl;
    else
      m.cgdo = 0.6 * m.xj * m.cox;
  }
  if (!m.g("CGSO")) {
    if (m.g("DLC") && (m.dlc > 0.0))
      m.cgso = m.dlc * m.cox - m.cgsl;
    else
      m.cgso = 0.6 * m.xj * m.cox;
  }
  if (!m.g("CGBO")) m.cgbo = 2.0 * m.dwc * m.cox;
  if (!m.g("CJSWG")) m.unitLengthGateSidewallJctCap = m.unitLengthSidewallJctCap;
  if (!m.g("PBSWG")) m.GatesidewallJctPotential = m.sidewallJctPotential;
  if (!m.g("MJSWG")) m.bulkJctGateSideGradingCoeff = m.bulkJctSideGradingCoeff;
  if (m.bulkJctPotential < 0.1) m.bulkJctPotential = 0.1;
  if (m.sidewallJctPotential < 0.1) m.sidewallJctPotential = 0.1;
  if (m.GatesidewallJctPotential < 0.1) m.GatesidewallJctPotential = 0.1;
  m.vcrit = CONSTvt0 * log(CONSTvt0 / (CONSTroot2 * 1.0e-14));
  m.factor1 = sqrt(CONSTEPSSI / CONSTEPSOX * m.tox);
  m.Vtm0 = CONSTKoverQ * m.tnom;
  m.Eg0 = CONSTEg0 - CONSTalphaEg * m.tnom * m.tnom / (m.tnom + CONSTbetaEg);
  m.ni = CONSTNi0 * (m.tnom / CONSTREFTEMP) * sqrt(m.tnom / CONSTREFTEMP) * exp(21.5565981 - m.Eg0 / (2.0 * m.Vtm0));
  return std::string();
}

// ---- Size-dependent set (the new-SizeDependParam branch of updateTemperature) ----
Size *get_size(ModelState &ms, const InstParams &ip, double temp, std::string &err) {
  const Card &m = ms.c;
  for (auto &s : ms.sizes)
    if (s->Length == ip.l && s->Width == ip.w) return s.get();
  std::unique_ptr<Size> sp(new Size());
  Size &p = *sp;
  const double Tnom = m.tnom;
  const double TRatio = temp / Tnom;
  const double Vtm0 = m.Vtm0, ni = m.ni;
  const double Ldrn = ip.l, Wdrn = ip.w;
  p.Length = Ldrn;
  p.Width = Wdrn;
  double T0 = pow(Ldrn, m.Lln);
  double T1 = pow(Wdrn, m.Lwn);
  double tmp1 = m.Ll / T0 + m.Lw / T1 + m.Lwl / (T0 * T1);
  p.dl = m.Lint + tmp1;
  double tmp2 = m.Llc / T0 + m.Lwc / T1 + m.Lwlc / (T0 * T1);
  p.dlc = m.dlc + tmp2;
  double T2 = pow(Ldrn, m.Wln);
  double T3 = pow(Wdrn, m.Wwn);
  tmp1 = m.Wl / T2 + m.Ww / T3 + m.Wwl / (T2 * T3);
  p.dw = m.Wint + tmp1;
  tmp2 = m.Wlc / T2 + m.Wwc / T3 + m.Wwlc / (T2 * T3);
  p.dwc = m.dwc + tmp2;
  p.leff = ip.l - 2.0 * p.dl;
  p.weff = ip.w - 2.0 * p.dw;
  p.leffCV = ip.l - 2.0 * p.dlc;
  p.weffCV = ip.w - 2.0 * p.dwc;
  if (p.leff <= 0.0 || p.weff <= 0.0 || p.leffCV <= 0.0 || p.weffCV <= 0.0) {
    err = "BSIM3 effective channel length or width <= 0";
    return nullptr;
  }
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
#define B3BIN(mem, base, l, w, pp) p.mem = m.base + m.l * Inv_L + m.w * Inv_W + m.pp * Inv_LW;
#include "bsim3_bins.inc"
#undef B3BIN
  p.abulkCVfactor = 1.0 + pow((p.clc / p.leffCV), p.cle);
  T0 = (TRatio - 1.0);
  p.ua = p.ua + p.ua1 * T0;
  p.ub = p.ub + p.ub1 * T0;
  p.uc = p.uc + p.uc1 * T0;
  if (p.u0 > 1.0) p.u0 = p.u0 / 1.0e4;
  p.u0temp = p.u0 * pow(TRatio, p.ute);
  p.vsattemp = p.vsat - p.at * T0;
  p.rds0 = (p.rdsw + p.prt * T0) / pow(p.weff * 1E6, p.wr);
  p.cgdo = (m.cgdo + p.cf) * p.weffCV;
  p.cgso = (m.cgso + p.cf) * p.weffCV;
  p.cgbo = m.cgbo * p.leffCV;
  T0 = p.leffCV * p.leffCV;
  p.tconst = p.u0temp * p.elm / (m.cox * p.weffCV * p.leffCV * T0);
  if (!m.g("NCH") && m.g("GAMMA1")) {
    T0 = p.gamma1 * m.cox;
    p.npeak = 3.021E22 * T0 * T0;
  }
  p.phi = 2.0 * Vtm0 * log(p.npeak / ni);
  p.sqrtPhi = sqrt(p.phi);
  p.phis3 = p.sqrtPhi * p.phi;
  p.Xdep0 = sqrt(2.0 * CONSTEPSSI / (CONSTQ * p.npeak * 1.0e6)) * p.sqrtPhi;
  p.sqrtXdep0 = sqrt(p.Xdep0);
  p.litl = sqrt(3.0 * p.xj * m.tox);
  p.vbi = Vtm0 * log(1.0e20 * p.npeak / (ni * ni));
  p.cdep0 = sqrt(CONSTQ * CONSTEPSSI * p.npeak * 1.0e6 / 2.0 / p.phi);
  p.ldeb = sqrt(CONSTEPSSI * Vtm0 / (CONSTQ * p.npeak * 1.0e6)) / 3.0;
  p.acde *= pow((p.npeak / 2.0e16), -0.25);
  if (m.g("K1") || m.g("K2")) {
    if (!m.g("K1")) p.k1 = 0.53;
    if (!m.g("K2")) p.k2 = -0.0186;
  } else {
    if (!m.g("VBX")) p.vbx = p.phi - 7.7348e-4 * p.npeak * p.xt * p.xt;
    if (p.vbx > 0.0) p.vbx = -p.vbx;
    if (p.vbm > 0.0) p.vbm = -p.vbm;
    if (!m.g("GAMMA1")) p.gamma1 = 5.753e-12 * sqrt(p.npeak) / m.cox;
    if (!m.g("GAMMA2")) p.gamma2 = 5.753e-12 * sqrt(p.nsub) / m.cox;
    T0 = p.gamma1 - p.gamma2;
    T1 = sqrt(p.phi - p.vbx) - p.sqrtPhi;
    T2 = sqrt(p.phi * (p.phi - p.vbm)) - p.phi;
    p.k2 = T0 * T1 / (2.0 * T2 + p.vbm);
    p.k1 = p.gamma2 - 2.0 * p.k2 * sqrt(p.phi - p.vbm);
  }
  if (p.k2 < 0.0) {
    T0 = 0.5 * p.k1 / p.k2;
    p.vbsc = 0.9 * (p.phi - T0 * T0);
    if (p.vbsc > -3.0)
      p.vbsc = -3.0;
    else if (p.vbsc < -30.0)
      p.vbsc = -30.0;
  } else {
    p.vbsc = -30.0;
  }
  if (p.vbsc > p.vbm) p.vbsc = p.vbm;
  if (!m.g("VFB")) {
    if (m.g("VTH0"))
      p.vfb = m.dtype * p.vth0 - p.phi - p.k1 * p.sqrtPhi;
    else
      p.vfb = -1.0;
  }
  if (!m.g("VTH0")) p.vth0 = m.dtype * (p.vfb + p.phi + p.k1 * p.sqrtPhi);
  p.k1ox = p.k1 * m.tox / m.toxm;
  p.k2ox = p.k2 * m.tox / m.toxm;
  T1 = sqrt(CONSTEPSSI / CONSTEPSOX * m.tox * p.Xdep0);
  T0 = exp(-0.5 * p.dsub * p.leff / T1);
  p.theta0vb0 = (T0 + 2.0 * T0 * T0);
  T0 = exp(-0.5 * p.drout * p.leff / T1);
  T2 = (T0 + 2.0 * T0 * T0);
  p.thetaRout = p.pdibl1 * T2 + p.pdibl2;
  const double tmp = sqrt(p.Xdep0);
  tmp1 = p.vbi - p.phi;
  tmp2 = m.factor1 * tmp;
  T0 = -0.5 * p.dvt1w * p.weff * p.leff / tmp2;
  if (T0 > -CONSTEXP_THRESHOLD) {
    T1 = exp(T0);
    T2 = T1 * (1.0 + 2.0 * T1);
  } else {
    T1 = CONSTMIN_EXP;
    T2 = T1 * (1.0 + 2.0 * T1);
  }
  T0 = p.dvt0w * T2;
  T2 = T0 * tmp1;
  T0 = -0.5 * p.dvt1 * p.leff / tmp2;
  if (T0 > -CONSTEXP_THRESHOLD) {
    T1 = exp(T0);
    T3 = T1 * (1.0 + 2.0 * T1);
  } else {
    T1 = CONSTMIN_EXP;
    T3 = T1 * (1.0 + 2.0 * T1);
  }
  T3 = p.dvt0 * T3 * tmp1;
  const double T4 = m.tox * p.phi / (p.weff + p.w0);
  T0 = sqrt(1.0 + p.nlx / p.leff);
  const double T5 = p.k1ox * (T0 - 1.0) * p.sqrtPhi + (p.kt1 + p.kt1l / p.leff) * (TRatio - 1.0);
  const double tmp3 = m.dtype * p.vth0 - T2 - T3 + p.k3 * T4 + T5;
  p.vfbzb = tmp3 - p.phi - p.k1 * p.sqrtPhi;
  ms.sizes.push_back(std::move(sp));
  return ms.sizes.back().get();
}

std::string instance_record(ModelState &ms, const InstParams &ipin, const xb4::SetupOptions &opts,
                            std::vector<double> &rec) {
  InstParams ip = ipin;
  const Card &m = ms.c;
  // Instance::Instance defaults.
  if (!ip.g("TEMP")) ip.temp = opts.temp_c + CONSTCtoK;
  if (!ip.g("L")) ip.l = m.model_l;
  if (!ip.g("W")) ip.w = m.model_w;
  if (!ip.g("AD")) ip.drainArea = 0.0;
  if (!ip.g("AS")) ip.sourceArea = 0.0;
  if (ip.nqsMod != 0) return "BSIM3 nqsMod != 0 is not supported";
  if (ip.g("IC1") || ip.g("IC2") || ip.g("IC3")) return "BSIM3 instance initial conditions are not supported";
  // Instance::processParams (:1849-1861): series conductances from the sheet resistance; a
  // nonzero one gives the instance its internal drain / source node (:1863-1865).
  double drainConductance = m.sheetResistance * ip.drainSquares;
  drainConductance = (drainConductance > 0.0) ? 1.0 / drainConductance : 0.0;
  double sourceConductance = m.sheetResistance * ip.sourceSquares;
  sourceConductance = (sourceConductance > 0.0) ? 1.0 / sourceConductance : 0.0;
  const double temp = ip.temp;
  if (!ms.temp_done) {
    ms.temp_done = true;
    ms.temp_seen = temp;
  } else if (temp != ms.temp_seen) {
    return "BSIM3 instances of one model must share one temperature";
  }
  // updateTemperature: temperature-dependent junction values.
  const double Tnom = m.tnom;
  const double vtm = CONSTKoverQ * temp;
  const double Eg = CONSTEg0 - CONSTalphaEg * temp * temp / (temp + CONSTbetaEg);
  double jctTempSatCurDensity, jctSidewallTempSatCurDensity;
  if (temp != Tnom) {
    const double T0 = m.Eg0 / m.Vtm0 - Eg / vtm + m.jctTempExponent * log(temp / Tnom);
    const double T1 = exp(T0 / m.jctEmissionCoeff);
    jctTempSatCurDensity = m.jctSatCurDensity * T1;
    jctSidewallTempSatCurDensity = m.jctSidewallSatCurDensity * T1;
  } else {
    jctTempSatCurDensity = m.jctSatCurDensity;
    jctSidewallTempSatCurDensity = m.jctSidewallSatCurDensity;
  }
  if (jctTempSatCurDensity < 0.0) jctTempSatCurDensity = 0.0;
  if (jctSidewallTempSatCurDensity < 0.0) jctSidewallTempSatCurDensity = 0.0;
  const double delTemp = temp - Tnom;
  double T0 = m.tcj * delTemp;
  const double unitAreaJctCapTemp = (T0 >= -1.0) ? m.unitAreaJctCap * (1.0 + T0) : 0.0;
  T0 = m.tcjsw * delTemp;
  const double unitLengthSidewallJctCapTemp = (T0 >= -1.0) ? m.unitLengthSidewallJctCap * (1.0 + T0) : 0.0;
  T0 = m.tcjswg * delTemp;
  const double unitLengthGateSidewallJctCapTemp =
      (T0 >= -1.0) ? m.unitLengthGateSidewallJctCap * (1.0 + T0) : 0.0;
  double PhiBTemp = m.bulkJctPotential - m.tpb * delTemp;
  if (PhiBTemp < 0.01) PhiBTemp = 0.01;
  double PhiBSWTemp = m.sidewallJctPotential - m.tpbsw * delTemp;
  if (PhiBSWTemp <= 0.01) PhiBSWTemp = 0.01;
  double PhiBSWGTemp = m.GatesidewallJctPotential - m.tpbswg * delTemp;
  if (PhiBSWGTemp <= 0.01) PhiBSWGTemp = 0.01;
  std::string err;
  const Size *pp = get_size(ms, ip, temp, err);
  if (!pp) return err;
  const Size &p = *pp;
  const double Nvtm = vtm * m.jctEmissionCoeff;
  double SourceSatCurrent, DrainSatCurrent, vjsm = 0, IsEvjsm = 0, vjdm = 0, IsEvjdm = 0;
  if ((ip.sourceArea <= 0.0) && (ip.sourcePerimeter <= 0.0))
    SourceSatCurrent = 1.0e-14;
  else
    SourceSatCurrent = ip.sourceArea * jctTempSatCurDensity + ip.sourcePerimeter * jctSidewallTempSatCurDensity;
  if ((SourceSatCurrent > 0.0) && (m.ijth > 0.0)) {
    vjsm = Nvtm * log(m.ijth / SourceSatCurrent + 1.0);
    IsEvjsm = SourceSatCurrent * exp(vjsm / Nvtm);
  }
  if ((ip.drainArea <= 0.0) && (ip.drainPerimeter <= 0.0))
    DrainSatCurrent = 1.0e-14;
  else
    DrainSatCurrent = ip.drainArea * jctTempSatCurDensity + ip.drainPerimeter * jctSidewallTempSatCurDensity;
  if ((DrainSatCurrent > 0.0) && (m.ijth > 0.0)) {
    vjdm = Nvtm * log(m.ijth / DrainSatCurrent + 1.0);
    IsEvjdm = DrainSatCurrent * exp(vjdm / Nvtm);
  }
  // Junction capacitances of updateIntermediateVars (:6950-6985), constant per instance.
  const double czbd = unitAreaJctCapTemp * ip.drainArea;
  const double czbs = unitAreaJctCapTemp * ip.sourceArea;
  double czbdsw, czbdswg, czbssw, czbsswg;
  if (ip.drainPerimeter < p.weff) {
    czbdswg = unitLengthGateSidewallJctCapTemp * ip.drainPerimeter;
    czbdsw = 0.0;
  } else {
    czbdsw = unitLengthSidewallJctCapTemp * (ip.drainPerimeter - p.weff);
    czbdswg = unitLengthGateSidewallJctCapTemp * p.weff;
  }
  if (ip.sourcePerimeter < p.weff) {
    czbssw = 0.0;
    czbsswg = unitLengthGateSidewallJctCapTemp * ip.sourcePerimeter;
  } else {
    czbssw = unitLengthSidewallJctCapTemp * (ip.sourcePerimeter - p.weff);
    czbsswg = unitLengthGateSidewallJctCapTemp * p.weff;
  }
  rec.assign(kNumFields, 0.0);
#define R(x) rec[f_##x]
  R(dtype) = m.dtype;
  R(mobMod) = m.mobMod;
  R(capMod) = m.capMod;
  R(xpart) = m.xpart;
  R(tox) = m.tox;
  R(cox) = m.cox;
  R(factor1) = m.factor1;
  R(vcrit) = m.vcrit;
  R(ijth) = m.ijth;
  R(vtm) = vtm;
  R(TempRatio) = temp / m.tnom - 1.0;
  R(Nvtm) = Nvtm;
  R(SourceSatCurrent) = SourceSatCurrent;
  R(DrainSatCurrent) = DrainSatCurrent;
  R(vjsm) = vjsm;
  R(IsEvjsm) = IsEvjsm;
  R(vjdm) = vjdm;
  R(IsEvjdm) = IsEvjdm;
  R(czbd) = czbd;
  R(czbs) = czbs;
  R(czbdsw) = czbdsw;
  R(czbdswg) = czbdswg;
  R(czbssw) = czbssw;
  R(czbsswg) = czbsswg;
  R(PhiBTemp) = PhiBTemp;
  R(PhiBSWTemp) = PhiBSWTemp;
  R(PhiBSWGTemp) = PhiBSWGTemp;
  R(MJ) = m.bulkJctBotGradingCoeff;
  R(MJSW) = m.bulkJctSideGradingCoeff;
  R(MJSWG) = m.bulkJctGateSideGradingCoeff;
  R(mult) = ip.mult;
  R(off) = ip.off;
  R(drainConductance) = drainConductance;
  R(sourceConductance) = sourceConductance;
#define S(x) R(x) = p.x;
  S(vbsc) S(phi) S(phis3) S(sqrtPhi) S(Xdep0) S(vbi) S(dvt2) S(dvt2w) S(dvt1) S(dvt0) S(dvt1w) S(dvt0w)
  S(weff) S(leff) S(nlx) S(k1ox) S(k2ox) S(kt1) S(kt1l) S(kt2) S(w0) S(eta0) S(etab) S(theta0vb0) S(vth0)
  S(k1) S(k3) S(k3b) S(nfactor) S(cdsc) S(cdscb) S(cdscd) S(cit) S(vfb) S(ngate) S(voff) S(cdep0) S(dwg)
  S(dwb) S(rds0) S(prwg) S(prwb) S(xj) S(a0) S(ags) S(b0) S(b1) S(keta) S(ua) S(ub) S(uc) S(u0temp)
  S(vsattemp) S(a1) S(a2) S(delta) S(pclm) S(litl) S(thetaRout) S(pdiblb) S(pvag) S(pscbe1) S(pscbe2)
  S(alpha0) S(alpha1) S(beta0) S(weffCV) S(leffCV) S(noff) S(voffcv) S(vfbzb) S(vfbcv) S(abulkCVfactor) S(acde)
  S(ldeb) S(moin) S(cgdo) S(cgso) S(cgbo) S(cgdl) S(cgsl) S(ckappa)
#undef S
#undef R
  return std::string();
}

}  // namespace

std::string build_records(const std::vector<xb4::ModelSpec> &models, int n_inst, const int *inst_model,
                          const std::vector<std::string> &inst_param_names, const double *inst_param_values,
                          const xb4::SetupOptions &opts, xb4::RecordTable &out) {
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
      const double v = inst_param_values[(size_t)i * np + k];
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
      const double v = inst_param_values[(size_t)i * np + k];
      if (std::isnan(v)) continue;
      if (!set_inst(ip, names[k], v)) return "unknown BSIM3 instance parameter " + names[k];
    }
    std::vector<double> rec;
    std::string e = instance_record(*ms[mi], ip, opts, rec);
    if (!e.empty()) return e;
    key_to_rec[kk] = (int)recs.size();
    out.inst_rec[i] = (int)recs.size();
    recs.push_back(std::move(rec));
  }
  out.n_records = (int)recs.size();
  out.tab.assign((size_t)kNumFields * recs.size(), 0.0);
  for (size_t r = 0; r < recs.size(); ++r)
    for (int f = 0; f < kNumFields; ++f) out.tab[(size_t)f * recs.size() + r] = recs[r][f];
  return std::string();
}

}  // namespace xb3
