// MOSFET level 1 set-up: model card, model processing and instance temperature precompute.
// Follows src/DeviceModelPKG/OpenModels/src/N_DEV_MOSFET1.C (Model::Model :3856-3955,
// Model::processParams :3752-3833, Instance::Instance :1160-1262, updateTemperature :3403-3655)
// in the same floating-point order.
#include <cctype>
#include <cmath>
#include <map>
#include <set>

#include "mos1.h"

namespace xm1 {
namespace {

using namespace xdc;

// Level-1 card parameters: netlist name, default (N_DEV_MOSFET1.C:120-292).
struct Card {
  double model_l = 1e-4, model_w = 1e-4, vt0 = 0.0, transconductance = 2e-5, gamma = 0.0, phi = 0.6, lambda = 0.0,
         drainResistance = 0.0, sourceResistance = 0.0, capBD = 0.0, capBS = 0.0, jctSatCur = 1e-14,
         bulkJctPotential = 0.8, gateSourceOverlapCapFactor = 0.0, gateDrainOverlapCapFactor = 0.0,
         gateBulkOverlapCapFactor = 0.0, sheetResistance = 0.0, bulkCapFactor = 0.0, bulkJctBotGradingCoeff = 0.5,
         sideWallCapFactor = 0.0, bulkJctSideGradingCoeff = 0.5, jctSatCurDensity = 0.0, oxideThickness = 1e-7,
         latDiff = 0.0, surfaceMobility = 600.0, surfaceMobility0 = 600.0, fwdCapDepCoeff = 0.5,
         substrateDoping = 0.0, surfaceStateDensity = 0.0, tnom = 27.0, fNcoef = 0.0, fNexp = 1.0, gateType = 0;
  int dtype = CONSTNMOS;
  bool capBDGiven = false, capBSGiven = false;
  std::set<std::string> given;
  bool g(const char *n) const { return given.count(n) != 0; }
  // processParams results
  double fact1 = 0, vtnom = 0, egfet1 = 0, pbfact1 = 0, oxideCapFactor = 0;
};

const std::map<std::string, double Card::*> &card_table() {
  static const std::map<std::string, double Card::*> t = {
      {"L", &Card::model_l}, {"W", &Card::model_w}, {"VTO", &Card::vt0}, {"KP", &Card::transconductance},
      {"GAMMA", &Card::gamma}, {"PHI", &Card::phi}, {"LAMBDA", &Card::lambda}, {"RD", &Card::drainResistance},
      {"RS", &Card::sourceResistance}, {"CBD", &Card::capBD}, {"CBS", &Card::capBS}, {"IS", &Card::jctSatCur},
      {"PB", &Card::bulkJctPotential}, {"CGSO", &Card::gateSourceOverlapCapFactor},
      {"CGDO", &Card::gateDrainOverlapCapFactor}, {"CGBO", &Card::gateBulkOverlapCapFactor},
      {"RSH", &Card::sheetResistance}, {"CJ", &Card::bulkCapFactor}, {"MJ", &Card::bulkJctBotGradingCoeff},
      {"CJSW", &Card::sideWallCapFactor}, {"MJSW", &Card::bulkJctSideGradingCoeff},
      {"JS", &Card::jctSatCurDensity}, {"TOX", &Card::oxideThickness}, {"LD", &Card::latDiff},
      {"UO", &Card::surfaceMobility}, {"U0", &Card::surfaceMobility0}, {"FC", &Card::fwdCapDepCoeff},
      {"NSUB", &Card::substrateDoping}, {"NSS", &Card::surfaceStateDensity}, {"TNOM", &Card::tnom},
      {"KF", &Card::fNcoef}, {"AF", &Card::fNexp}, {"TPG", &Card::gateType}};
  return t;
}

std::string upper(std::string s) {
  for (auto &c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

std::string process_model(const xb4::ModelSpec &spec, const xb4::SetupOptions &opts, Card &m) {
  m.dtype = spec.pmos ? CONSTPMOS : CONSTNMOS;
  for (const auto &kv : spec.params) {
    const std::string n = upper(kv.first);
    if (n == "LEVEL") continue;
    auto it = card_table().find(n);
    if (it == card_table().end()) return "unknown MOSFET level-1 model parameter " + n;
    m.*(it->second) = (n == "TNOM") ? kv.second + CONSTCtoK : kv.second;
    m.given.insert(n);
  }
  if (!m.g("TNOM")) m.tnom = opts.tnom_c + CONSTCtoK;
  m.capBDGiven = m.g("CBD") || m.capBD != 0;
  m.capBSGiven = m.g("CBS") || m.capBS != 0;
  if (m.g("U0")) {
    if (m.g("UO")) return "MOSFET level 1: both UO and U0 given";
    m.surfaceMobility = m.surfaceMobility0;
  }
  // Model::processParams
  m.fact1 = m.tnom / CONSTREFTEMP;
  m.vtnom = m.tnom * CONSTKoverQ;
  const double kt1 = CONSTboltz * m.tnom;
  m.egfet1 = 1.16 - (7.02e-4 * m.tnom * m.tnom) / (m.tnom + 1108);
  const double arg1 = -m.egfet1 / (kt1 + kt1) + 1.1150877 / (CONSTboltz * (CONSTREFTEMP + CONSTREFTEMP));
  m.pbfact1 = -2 * m.vtnom * (1.5 * log(m.fact1) + CONSTQ * arg1);
  if (!m.g("TOX") || m.oxideThickness == 0) {
    m.oxideCapFactor = 0;
  } else {
    m.oxideCapFactor = 3.9 * 8.854214871e-12 / m.oxideThickness;
    if (!m.g("KP")) {
      if (!m.g("UO") && !m.g("U0")) m.surfaceMobility = 600;
      m.transconductance = m.surfaceMobility * m.oxideCapFactor * 1e-4;
    }
    if (m.g("NSUB")) {
      if (m.substrateDoping * 1e6 > 1.45e16) {
        if (!m.g("PHI")) {
          m.phi = 2 * m.vtnom * log(m.substrateDoping * 1e6 / 1.45e16);
          m.phi = dmax(0.1, m.phi);
        }
        const double fermis = m.dtype * .5 * m.phi;
        double wkfng = 3.2;
        if (!m.g("TPG")) m.gateType = 1;
        if (m.gateType != 0) {
          const double fermig = m.dtype * m.gateType * .5 * m.egfet1;
          wkfng = 3.25 + .5 * m.egfet1 - fermig;
        }
        const double wkfngs = wkfng - (3.25 + .5 * m.egfet1 + fermis);
        if (!m.g("GAMMA"))
          m.gamma = sqrt(2 * 11.70 * 8.854214871e-12 * CONSTQ * m.substrateDoping * 1e6) / m.oxideCapFactor;
        if (!m.g("VTO")) {
          if (!m.g("NSS")) m.surfaceStateDensity = 0;
          const double vfb = wkfngs - m.surfaceStateDensity * 1e4 * CONSTQ / m.oxideCapFactor;
          m.vt0 = vfb + m.dtype * (m.gamma * sqrt(m.phi) + m.phi);
        }
      } else {
        return "MOSFET level 1: NSUB < Ni";
      }
    }
  }
  return std::string();
}

struct InstParams {
  double temp = 0, l = 0, w = 0, drainArea = 0, sourceArea = 0, drainSquares = 1.0, sourceSquares = 1.0,
         drainPerimeter = 0, sourcePerimeter = 0, mult = 1.0, off = 0;
  std::set<std::string> given;
  bool g(const char *n) const { return given.count(n) != 0; }
};

bool set_inst(InstParams &ip, const std::string &n, double v) {
  static const std::map<std::string, double InstParams::*> t = {
      {"TEMP", &InstParams::temp}, {"L", &InstParams::l}, {"W", &InstParams::w}, {"AD", &InstParams::drainArea},
      {"AS", &InstParams::sourceArea}, {"NRD", &InstParams::drainSquares}, {"NRS", &InstParams::sourceSquares},
      {"PD", &InstParams::drainPerimeter}, {"PS", &InstParams::sourcePerimeter}, {"M", &InstParams::mult},
      {"OFF", &InstParams::off}};
  if (n == "IC1" || n == "IC2" || n == "IC3") {
    ip.given.insert(n);
    return true;
  }
  auto it = t.find(n);
  if (it == t.end()) return false;
  ip.*(it->second) = (n == "TEMP") ? v + CONSTCtoK : v;
  ip.given.insert(n);
  return true;
}

std::string instance_record(const Card &m, InstParams ip, const xb4::SetupOptions &opts, std::vector<double> &rec) {
  if (ip.g("IC1") || ip.g("IC2") || ip.g("IC3")) return "MOSFET level 1 instance initial conditions are not supported";
  if (!ip.g("TEMP")) ip.temp = opts.temp_c + CONSTCtoK;
  if (!ip.g("L")) ip.l = m.model_l;
  if (!ip.g("W")) ip.w = m.model_w;
  if (!ip.g("AD")) ip.drainArea = 0.0;
  if (!ip.g("AS")) ip.sourceArea = 0.0;
  if (ip.l - 2 * m.latDiff <= 0) return "MOSFET level 1: effective channel length less than zero";
  const double EffectiveLength = ip.l - 2 * m.latDiff;
  const double GateSourceOverlapCap = m.gateSourceOverlapCapFactor * ip.w;
  const double GateDrainOverlapCap = m.gateDrainOverlapCapFactor * ip.w;
  const double GateBulkOverlapCap = m.gateBulkOverlapCapFactor * EffectiveLength;
  const double OxideCap = m.oxideCapFactor * EffectiveLength * ip.w;
  // updateTemperature
  const double temp = ip.temp;
  const double tnom = m.tnom;
  const double vt = temp * CONSTKoverQ;
  const double ratio = temp / tnom;
  const double fact2 = temp / CONSTREFTEMP;
  const double kt = temp * CONSTboltz;
  const double egfet = 1.16 - (7.02e-4 * temp * temp) / (temp + 1108);
  double arg = -egfet / (kt + kt) + 1.1150877 / (CONSTboltz * (CONSTREFTEMP + CONSTREFTEMP));
  const double pbfact = -2 * vt * (1.5 * log(fact2) + CONSTQ * arg);
  const double ratio4 = ratio * sqrt(ratio);
  const double tTransconductance = m.transconductance / ratio4;
  const double phio = (m.phi - m.pbfact1) / m.fact1;
  const double tPhi = fact2 * phio + pbfact;
  const double tVbi = m.vt0 - m.dtype * (m.gamma * sqrt(m.phi)) + .5 * (m.egfet1 - egfet) + m.dtype * .5 * (tPhi - m.phi);
  const double tVto = tVbi + m.dtype * m.gamma * sqrt(tPhi);
  const double tSatCur = m.jctSatCur * exp(-egfet / vt + m.egfet1 / m.vtnom);
  const double tSatCurDens = m.jctSatCurDensity * exp(-egfet / vt + m.egfet1 / m.vtnom);
  const double pbo = (m.bulkJctPotential - m.pbfact1) / m.fact1;
  const double gmaold = (m.bulkJctPotential - pbo) / pbo;
  double capfact = 1 / (1 + m.bulkJctBotGradingCoeff * (4e-4 * (m.tnom - CONSTREFTEMP) - gmaold));
  double tCbd = m.capBD * capfact;
  double tCbs = m.capBS * capfact;
  double tCj = m.bulkCapFactor * capfact;
  capfact = 1 / (1 + m.bulkJctSideGradingCoeff * (4e-4 * (m.tnom - CONSTREFTEMP) - gmaold));
  double tCjsw = m.sideWallCapFactor * capfact;
  const double tBulkPot = fact2 * pbo + pbfact;
  const double gmanew = (tBulkPot - pbo) / pbo;
  capfact = (1 + m.bulkJctBotGradingCoeff * (4e-4 * (temp - CONSTREFTEMP) - gmanew));
  tCbd *= capfact;
  tCbs *= capfact;
  tCj *= capfact;
  capfact = (1 + m.bulkJctSideGradingCoeff * (4e-4 * (temp - CONSTREFTEMP) - gmanew));
  tCjsw *= capfact;
  const double tDepCap = m.fwdCapDepCoeff * tBulkPot;
  double sourceVcrit, drainVcrit;
  if ((m.jctSatCurDensity == 0) || (ip.drainArea == 0) || (ip.sourceArea == 0)) {
    sourceVcrit = drainVcrit = vt * log(vt / (CONSTroot2 * m.jctSatCur));
  } else {
    drainVcrit = vt * log(vt / (CONSTroot2 * m.jctSatCurDensity * ip.drainArea));
    sourceVcrit = vt * log(vt / (CONSTroot2 * m.jctSatCurDensity * ip.sourceArea));
  }
  const double MJ = m.bulkJctBotGradingCoeff, MJSW = m.bulkJctSideGradingCoeff, FC = m.fwdCapDepCoeff;
  double czbd = m.capBDGiven ? tCbd : (m.g("CJ") ? tCj * ip.drainArea : 0);
  double czbdsw = m.g("CJSW") ? tCjsw * ip.drainPerimeter : 0;
  arg = 1 - FC;
  double sarg = exp((-MJ) * log(arg));
  double sargsw = exp((-MJSW) * log(arg));
  const double f2d = czbd * (1 - FC * (1 + MJ)) * sarg / arg + czbdsw * (1 - FC * (1 + MJSW)) * sargsw / arg;
  const double f3d = czbd * MJ * sarg / arg / tBulkPot + czbdsw * MJSW * sargsw / arg / tBulkPot;
  const double f4d = czbd * tBulkPot * (1 - arg * sarg) / (1 - MJ) + czbdsw * tBulkPot * (1 - arg * sargsw) / (1 - MJSW) -
                     f3d / 2 * (tDepCap * tDepCap) - tDepCap * f2d;
  double czbs = m.capBSGiven ? tCbs : (m.g("CJ") ? tCj * ip.sourceArea : 0);
  double czbssw = m.g("CJSW") ? tCjsw * ip.sourcePerimeter : 0;
  arg = 1 - FC;
  sarg = exp((-MJ) * log(arg));
  sargsw = exp((-MJSW) * log(arg));
  const double f2s = czbs * (1 - FC * (1 + MJ)) * sarg / arg + czbssw * (1 - FC * (1 + MJSW)) * sargsw / arg;
  const double f3s = czbs * MJ * sarg / arg / tBulkPot + czbssw * MJSW * sargsw / arg / tBulkPot;
  const double f4s = czbs * tBulkPot * (1 - arg * sarg) / (1 - MJ) + czbssw * tBulkPot * (1 - arg * sargsw) / (1 - MJSW) -
                     f3s / 2 * (tDepCap * tDepCap) - tDepCap * f2s;
  // updateIntermediateVars' instance constants.
  double DrainSatCur, SourceSatCur;
  if ((tSatCurDens == 0) || (ip.drainArea == 0) || (ip.sourceArea == 0)) {
    DrainSatCur = tSatCur;
    SourceSatCur = tSatCur;
  } else {
    DrainSatCur = tSatCurDens * ip.drainArea;
    SourceSatCur = tSatCurDens * ip.sourceArea;
  }
  const double Beta = tTransconductance * ip.w / EffectiveLength;
  // Series resistance (:1180-1220): RD / RS win over the sheet resistance; a conductance that is
  // nonzero gives the instance an internal node.
  double drainConductance = 0, sourceConductance = 0;
  if (m.drainResistance != 0)
    drainConductance = 1 / m.drainResistance;
  else if (m.g("RSH") && m.sheetResistance != 0)
    drainConductance = 1 / (m.sheetResistance * ip.drainSquares);
  if (m.sourceResistance != 0)
    sourceConductance = 1 / m.sourceResistance;
  else if (m.g("RSH") && m.sheetResistance != 0)
    sourceConductance = 1 / (m.sheetResistance * ip.sourceSquares);
  if (!std::isfinite(drainConductance) || !std::isfinite(sourceConductance))
    return "MOSFET level 1: RSH with NRD or NRS = 0 gives an infinite series conductance";
  rec.assign(kNumFields, 0.0);
#define R(f) rec[f_##f]
  R(dtype) = m.dtype; R(gamma) = m.gamma; R(lambda) = m.lambda; R(mj) = MJ; R(mjsw) = MJSW; R(vt) = vt;
  R(tPhi) = tPhi; R(tVbi) = tVbi; R(tVto) = tVto; R(sourceVcrit) = sourceVcrit; R(drainVcrit) = drainVcrit;
  R(Beta) = Beta; R(DrainSatCur) = DrainSatCur; R(SourceSatCur) = SourceSatCur; R(Cbd) = czbd; R(Cbdsw) = czbdsw;
  R(Cbs) = czbs; R(Cbssw) = czbssw; R(tDepCap) = tDepCap; R(tBulkPot) = tBulkPot; R(f2d) = f2d; R(f3d) = f3d;
  R(f4d) = f4d; R(f2s) = f2s; R(f3s) = f3s; R(f4s) = f4s; R(GateSourceOverlapCap) = GateSourceOverlapCap;
  R(GateDrainOverlapCap) = GateDrainOverlapCap; R(GateBulkOverlapCap) = GateBulkOverlapCap; R(OxideCap) = OxideCap;
  R(mult) = ip.mult; R(off) = ip.off; R(drainConductance) = drainConductance;
  R(sourceConductance) = sourceConductance;
#undef R
  return std::string();
}

}  // namespace

std::string build_records(const std::vector<xb4::ModelSpec> &models, int n_inst, const int *inst_model,
                          const std::vector<std::string> &inst_param_names, const double *inst_param_values,
                          const xb4::SetupOptions &opts, xb4::RecordTable &out) {
  std::vector<Card> cards(models.size());
  for (size_t m = 0; m < models.size(); ++m) {
    std::string e = process_model(models[m], opts, cards[m]);
    if (!e.empty()) return e;
  }
  std::vector<std::string> names;
  for (const auto &n : inst_param_names) names.push_back(upper(n));
  const size_t np = names.size();
  std::map<std::pair<int, std::vector<double>>, int> key_to_rec;
  std::vector<std::vector<double>> recs;
  out.inst_rec.assign(n_inst, -1);
  for (int i = 0; i < n_inst; ++i) {
    const int mi = inst_model[i];
    if (mi < 0 || mi >= (int)cards.size()) return "instance model index out of range";
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
      if (!set_inst(ip, names[k], v)) return "unknown MOSFET level-1 instance parameter " + names[k];
    }
    std::vector<double> rec;
    std::string e = instance_record(cards[mi], ip, opts, rec);
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

}  // namespace xm1
