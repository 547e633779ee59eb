// Per-record constants read by the BSIM4 load kernel.
//
// One record holds everything the evaluation of one instance needs that does not depend on the
// node voltages: model-level temperature-adjusted values, the size-binned parameter set for the
// instance's (L, W, NF), and the instance-level values computed at temperature setup
// (src/DeviceModelPKG/OpenModels/src/N_DEV_MOSFET_B4.C:5640-7743). Instances whose model card and
// instance parameters coincide share a record. Records are stored field-major in device memory
// (field f of record r at tab[f * n_records + r]), so a warp of instances that share a record
// broadcasts each load and a warp of per-instance records loads one coalesced line per field.
#pragma once

#define XB4_FIELDS(F)                                                                            \
  /* model-level */                                                                              \
  F(dtype) F(mobMod) F(capMod) F(dioMod) F(rdsMod) F(igcMod) F(igbMod) F(tempMod) F(mtrlMod)    \
  F(cvchargeMod) F(tnoiMod) F(xpart) F(vtm) F(vtm0) F(coxe) F(coxp) F(toxe_m) F(toxp) F(toxm)    \
  F(epsrox_m) F(eot) F(epsrsub) F(epsrgate) F(factor1) F(vcrit) F(SjctEmissionCoeff)             \
  F(DjctEmissionCoeff) F(SjctTempSatCurDensity) F(SjctSidewallTempSatCurDensity)                 \
  F(SjctGateSidewallTempSatCurDensity) F(DjctTempSatCurDensity) F(DjctSidewallTempSatCurDensity) \
  F(DjctGateSidewallTempSatCurDensity) F(xjbvs) F(xjbvd) F(bvs) F(bvd) F(njtsstemp)              \
  F(njtsswstemp) F(njtsswgstemp) F(njtsdtemp) F(njtsswdtemp) F(njtsswgdtemp) F(vtss) F(vtsd)      \
  F(vtssws) F(vtsswd) F(vtsswgs) F(vtsswgd) F(phig) F(easub) F(Eg0) F(ados) F(bdos) F(pditsl)     \
  F(lambdaGiven) F(vtlGiven) F(tnom) F(DunitAreaTempJctCap) F(SunitAreaTempJctCap)               \
  F(DunitLengthSidewallTempJctCap) F(DunitLengthGateSidewallTempJctCap)                          \
  F(SunitLengthSidewallTempJctCap) F(SunitLengthGateSidewallTempJctCap) F(SbulkJctBotGradingCoeff) \
  F(SbulkJctSideGradingCoeff) F(SbulkJctGateSideGradingCoeff) F(DbulkJctBotGradingCoeff)         \
  F(DbulkJctSideGradingCoeff) F(DbulkJctGateSideGradingCoeff) F(PhiBS) F(PhiBSWS) F(PhiBSWGS)     \
  F(PhiBD) F(PhiBSWD) F(PhiBSWGD) F(lambda_m) F(vtl_m)                                            \
  /* size-binned and size-derived */                                                             \
  F(phi) F(sqrtPhi) F(Xdep0) F(leff) F(vbi) F(dvt2) F(dvt2w) F(dvt1) F(dvt0) F(dvt1w) F(weff)      \
  F(dvt0w) F(lpe0) F(k1ox) F(kt1) F(kt1l) F(kt2) F(w0) F(etab) F(theta0vb0) F(lpeb) F(k1) F(k3)    \
  F(k3b) F(cit) F(nfactor) F(cdsc) F(cdscb) F(cdscd) F(dvtp0) F(dvtp1) F(ngate) F(mstar)          \
  F(voffcbn) F(cdep0) F(dwg) F(dwb) F(prwg) F(prwb) F(rds0) F(rdswmin) F(xj) F(a0) F(b1) F(b0)   \
  F(ags) F(keta) F(ua) F(uc) F(ub) F(ud) F(eu) F(a1) F(a2) F(delta) F(lambda) F(litl) F(fprout)   \
  F(pvag) F(pclm) F(thetaRout) F(pdiblb) F(pditsd) F(pdits) F(pscbe1) F(pscbe2) F(alpha0)         \
  F(alpha1) F(beta0) F(vtl) F(tfactor) F(xrcrg1) F(xrcrg2) F(vfbsd) F(egidl) F(agidl) F(bgidl)    \
  F(cgidl) F(weffCJ) F(egisl) F(agisl) F(bgisl) F(cgisl) F(abulkCVfactor) F(weffCV) F(leffCV)     \
  F(noff) F(voffcv) F(mstarcv) F(voffcbncv) F(acde) F(ldeb) F(moin) F(cgbo) F(cgdo) F(cgso)       \
  F(cgdl) F(cgsl) F(ckappad) F(ckappas) F(vfbcv) F(Aechvb) F(Bechvb) F(AechvbEdgeS) F(AechvbEdgeD)  \
  F(BechvbEdge) F(ToxRatio) F(aigc) F(bigc) F(cigc) F(nigc) F(pigcd) F(pigcdGiven) F(vfbsdoff)      \
  F(aigs) F(bigs) F(cigs) F(aigd) F(bigd) F(cigd) F(nigbacc) F(aigbacc) F(bigbacc) F(cigbacc)       \
  F(nigbinv) F(eigbinv) F(aigbinv) F(bigbinv) F(cigbinv)                                           \
  /* instance-level */                                                                           \
  F(vth0) F(eta0) F(k2ox) F(vfb) F(vbsc) F(u0temp) F(vsattemp) F(vtfbphi1) F(vtfbphi2) F(vfbzb)   \
  F(nf) F(mult) F(Aseff) F(Pseff) F(Adeff) F(Pdeff) F(XExpBVS) F(XExpBVD) F(vjsmFwd) F(vjsmRev)   \
  F(vjdmFwd) F(vjdmRev) F(IVjsmFwd) F(IVjsmRev) F(IVjdmFwd) F(IVjdmRev) F(SslpFwd) F(SslpRev)     \
  F(DslpFwd) F(DslpRev) F(SjctTempRevSatCur) F(SswTempRevSatCur) F(SswgTempRevSatCur)            \
  F(DjctTempRevSatCur) F(DswTempRevSatCur) F(DswgTempRevSatCur) F(drainConductance)              \
  F(sourceConductance) F(grgeltd) F(temp) F(off) F(dExists) F(sExists)                           \
  /* general topology: gate / body resistance modes, rdsMod 1 S/D resistance, body network, NQS */ \
  F(rgateMod) F(rbodyMod) F(rd0) F(rdwmin) F(rs0) F(rswmin) F(grbpd) F(grbps) F(grbpb) F(grbsb)   \
  F(grbdb) F(icVBS) F(icVDS) F(icVGS) F(icVBSGiven) F(icVDSGiven) F(icVGSGiven) F(trnqsMod)

namespace xb4 {
enum Field {
#define XB4_ENUM(n) f_##n,
  XB4_FIELDS(XB4_ENUM)
#undef XB4_ENUM
  kNumFields
};
}  // namespace xb4
