// N_DEV_GpuMosfetB4.C — the reference-side binding of the B200 device load for BSIM4 (see the
// header for what it does and why). Compiled against the reference's headers and linked with
// libxyce_b200.so and the CUDA runtime.
#include <Xyce_config.h>

#include "N_DEV_GpuMosfetB4.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>

#include <N_DEV_Configuration.h>
#include <N_DEV_Const.h>
#include <N_DEV_DeviceBlock.h>
#include <N_DEV_DeviceOptions.h>
#include <N_DEV_ExternData.h>
#include <N_DEV_SolverState.h>
#include <N_LAS_Matrix.h>

#include "../../include/xyce_devload.h"

namespace Xyce {
namespace Device {
namespace GpuMosfetB4 {

namespace {

// The instances' own state and store LIDs (the reference keeps them in protected members of
// DeviceInstance and offers no getter for the store's): a pointer to the base class member, named
// through a derived class, reads them from any instance.
// The same holds for the node LIDs: DeviceInstance::getDevLIDs is filled only by the numerical
// Jacobian test (N_DEV_DeviceInstance.C:383-388), so the binding reads the external and internal
// LID vectors registerLIDs stored.
struct LidAccess : public DeviceInstance {
  static const std::vector<int> &sta(const DeviceInstance &d) { return d.*(&LidAccess::staLIDVec); }
  static const std::vector<int> &sto(const DeviceInstance &d) { return d.*(&LidAccess::stoLIDVec); }
  // External LIDs (D, G, S, B), then the internal ones in the instance's registerLIDs order.
  static std::vector<int> nodes(const DeviceInstance &d) {
    std::vector<int> v = d.*(&LidAccess::extLIDVec);
    const std::vector<int> &in = d.*(&LidAccess::intLIDVec);
    v.insert(v.end(), in.begin(), in.end());
    return v;
  }
};

void check_cuda(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("GPU MOSFET binding: ") + what + ": " + cudaGetErrorString(e));
}

void check_xd(int rc, const char *what) {
  if (rc != 0) throw std::runtime_error(std::string("GPU MOSFET binding: ") + what + ": " + xd_last_error());
}

// The given, numeric parameters of a netlist line as (name, value) pairs.
std::vector<std::pair<std::string, double> > numeric_params(const std::vector<Param> &ps) {
  std::vector<std::pair<std::string, double> > out;
  for (size_t k = 0; k < ps.size(); ++k)
    if (ps[k].given() && ps[k].isNumeric()) out.push_back(std::make_pair(ps[k].uTag(), ps[k].getImmutableValue<double>()));
  return out;
}

// xd_flags from the solver state and device options the reference's loads read
// (N_DEV_SolverState.h:93-204, N_DEV_DeviceOptions.h).
xd_flags flags_from(const SolverState &ss, const DeviceOptions &dopt) {
  xd_flags f;
  f.dcop = ss.dcopFlag ? 1 : 0;
  f.init_tran = ss.initTranFlag ? 1 : 0;
  f.newton_iter = ss.newtonIter;
  f.init_jct = ss.initJctFlag ? 1 : 0;
  f.init_fix = ss.initFixFlag ? 1 : 0;
  f.transient = ss.transientFlag ? 1 : 0;
  f.tranop = ss.tranopFlag ? 1 : 0;
  f.acop = ss.acopFlag ? 1 : 0;
  f.voltlim = dopt.voltageLimiterFlag ? 1 : 0;
  f.input_op = ss.inputOPFlag ? 1 : 0;
  f.gmin = dopt.gmin;
  f.pdt = ss.pdt;
  return f;
}

}  // namespace

Master::Master(const Configuration &configuration, const FactoryBlock &factory_block, const SolverState &ss,
               const DeviceOptions &dopts, int cuda_device)
    : MOSFET_B4::Master(configuration, factory_block, ss, dopts), device_(cuda_device), ctx_(0), ready_(false), n_(0),
      n_rows_(0), n_unknowns_(0), nnz_(0), ground_(-1), d_sol_(0), d_jf_(0), d_jq_(0), stream_(0) {
  d_sta_[0] = d_sta_[1] = d_sto_[0] = d_sto_[1] = 0;
  for (int k = 0; k < 4; ++k) d_vec_[k] = 0;
}

Master::~Master() { release(); }

void Master::release() {
  if (ctx_) xd_destroy(ctx_);
  ctx_ = 0;
  double *bufs[] = {d_sol_, d_sta_[0], d_sta_[1], d_sto_[0], d_sto_[1], d_vec_[0], d_vec_[1], d_vec_[2], d_vec_[3],
                    d_jf_, d_jq_};
  for (size_t k = 0; k < sizeof(bufs) / sizeof(bufs[0]); ++k) cudaFree(bufs[k]);
  d_sol_ = d_jf_ = d_jq_ = 0;
  d_sta_[0] = d_sta_[1] = d_sto_[0] = d_sto_[1] = 0;
  for (int k = 0; k < 4; ++k) d_vec_[k] = 0;
  if (stream_) cudaStreamDestroy((cudaStream_t)stream_);
  stream_ = 0;
  ready_ = false;
}

MOSFET_B4::Model *Master::addModel(const ModelBlock &model_block, const FactoryBlock &factory_block) {
  Card c;
  c.name = model_block.getName();
  std::string t = model_block.getType();
  std::transform(t.begin(), t.end(), t.begin(), ::toupper);
  c.pmos = t == "PMOS";
  c.params = numeric_params(model_block.params);
  MOSFET_B4::Model *m = MOSFET_B4::Master::addModel(model_block, factory_block);
  // A card given twice replaces the earlier one, as the reference's model map does.
  for (size_t k = 0; k < cards_.size(); ++k)
    if (equal_nocase(cards_[k].name, c.name)) {
      cards_[k] = c;
      return m;
    }
  cards_.push_back(c);
  return m;
}

MOSFET_B4::Instance *Master::addInstance(const InstanceBlock &instance_block, const FactoryBlock &factory_block) {
  Line l;
  l.model = instance_block.getModelName();
  l.params = numeric_params(instance_block.params);
  lines_.push_back(l);
  return MOSFET_B4::Master::addInstance(instance_block, factory_block);
}

// Builds the library context once the topology has registered every instance (LIDs, state / store
// LIDs, Jacobian offsets): cards and lines as recorded, node LIDs from the instances, the pattern
// from the dF/dx matrix.
bool Master::setup() {
  if (ready_) return true;
  const std::vector<MOSFET_B4::Instance *> insts(getInstanceBegin(), getInstanceEnd());
  n_ = (int)insts.size();
  if (n_ != (int)lines_.size()) throw std::runtime_error("GPU MOSFET binding: instance count changed after set-up");
  if (n_ == 0) return ready_ = true;
  const ExternData &ext = insts[0]->getExternData();
  N_LAS_Matrix &J = *ext.dFdxMatrixPtr;
  n_rows_ = J.getLocalNumRows();
  ground_ = n_rows_ - 1;  // the overlap map with ground puts ground last
  n_unknowns_ = n_rows_ - 1;
  rowptr_.assign(1, 0);
  std::vector<int> colind;
  pos_.clear();
  for (int r = 0; r < n_unknowns_; ++r) {
    int len = 0;
    double *vals = 0;
    int *idx = 0;
    J.extractLocalRowView(r, len, vals, idx);
    // The library takes each row's columns in ascending order; pos_ maps the matrix's storage
    // order to that order.
    std::vector<int> order(len);
    for (int j = 0; j < len; ++j) order[j] = j;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return idx[a] < idx[b]; });
    std::vector<int> rank(len);
    for (int j = 0; j < len; ++j) {
      rank[order[j]] = j;
      colind.push_back(idx[order[j]]);
    }
    pos_.insert(pos_.end(), rank.begin(), rank.end());
    rowptr_.push_back((int)colind.size());
  }
  nnz_ = rowptr_.back();
  // Family description.
  std::vector<int> is_pmos, nparams, inst_model(n_), nodes(4 * (size_t)n_), internal(2 * (size_t)n_, -1);
  std::vector<const char *> pnames;
  std::vector<double> pvals;
  for (size_t m = 0; m < cards_.size(); ++m) {
    is_pmos.push_back(cards_[m].pmos ? 1 : 0);
    nparams.push_back((int)cards_[m].params.size());
    for (size_t k = 0; k < cards_[m].params.size(); ++k) {
      pnames.push_back(cards_[m].params[k].first.c_str());
      pvals.push_back(cards_[m].params[k].second);
    }
  }
  std::vector<std::string> inames;
  for (int i = 0; i < n_; ++i)
    for (size_t k = 0; k < lines_[i].params.size(); ++k)
      if (std::find(inames.begin(), inames.end(), lines_[i].params[k].first) == inames.end())
        inames.push_back(lines_[i].params[k].first);
  std::vector<double> ivals((size_t)n_ * std::max<size_t>(1, inames.size()), NAN);
  for (int i = 0; i < n_; ++i) {
    int mi = -1;
    for (size_t m = 0; m < cards_.size(); ++m)
      if (equal_nocase(cards_[m].name, lines_[i].model)) mi = (int)m;
    if (mi < 0) throw std::runtime_error("GPU MOSFET binding: instance model card not found: " + lines_[i].model);
    inst_model[i] = mi;
    for (size_t k = 0; k < lines_[i].params.size(); ++k) {
      const size_t col = std::find(inames.begin(), inames.end(), lines_[i].params[k].first) - inames.begin();
      ivals[(size_t)i * inames.size() + col] = lines_[i].params[k].second;
    }
    const std::vector<int> lids = LidAccess::nodes(*insts[i]);  // D, G, S, B, then internal D', S'
    if (lids.size() < 4) throw std::runtime_error("GPU MOSFET binding: instance without its four terminal LIDs");
    for (int k = 0; k < 4; ++k) nodes[4 * (size_t)i + k] = lids[k] == ground_ ? -1 : lids[k];
  }
  std::vector<const char *> inptr;
  for (size_t k = 0; k < inames.size(); ++k) inptr.push_back(inames[k].c_str());
  xd_mosfet_family fam;
  fam.level = 14;
  fam.n_models = (int)cards_.size();
  fam.model_is_pmos = is_pmos.data();
  fam.model_nparams = nparams.data();
  fam.model_param_names = pnames.data();
  fam.model_param_values = pvals.data();
  fam.n_inst = n_;
  fam.inst_model = inst_model.data();
  fam.inst_nodes = nodes.data();
  fam.n_inst_params = (int)inames.size();
  fam.inst_param_names = inptr.data();
  fam.inst_param_values = ivals.data();
  fam.temp_c = getDeviceOptions().temp.getImmutableValue<double>() - CONSTCtoK;
  fam.tnom_c = getDeviceOptions().tnom - CONSTCtoK;
  // Internal variables: which instances the library expects them on must match the reference's
  // topology (both follow the same rules). Gate / body resistance, rdsMod 1, the NQS charge node
  // and instance initial conditions take the general topology (XD_GEN_INTERNAL internal variables
  // per instance, registerLIDs order); otherwise only the drain / source ones can exist.
  fam.inst_internal = 0;
  fam.inst_internal_gen = 0;
  std::vector<int> gflags((size_t)XD_GEN_INTERNAL * n_);
  const int general = xd_internal_nodes_gen(&fam, gflags.data());
  if (general < 0) check_xd(general, "xd_internal_nodes_gen");
  std::vector<int> internal_gen(general ? (size_t)XD_GEN_INTERNAL * n_ : 0, -1);
  bool any = false;
  for (int i = 0; i < n_; ++i) {
    const std::vector<int> lids = LidAccess::nodes(*insts[i]);
    const int *fl = &gflags[(size_t)XD_GEN_INTERNAL * i];
    int want = 0;
    for (int k = 0; k < XD_GEN_INTERNAL; ++k) want += fl[k];
    if ((int)lids.size() - 4 != want)
      throw std::runtime_error("GPU MOSFET binding: internal nodes differ from the reference's topology");
    int next = 4;
    for (int k = 0; k < XD_GEN_INTERNAL; ++k) {
      const int lid = fl[k] ? lids[next++] : -1;
      if (general) internal_gen[(size_t)XD_GEN_INTERNAL * i + k] = lid;
      if (!general && k < 2) internal[2 * (size_t)i + k] = lid;
    }
    any = any || want > 0;
  }
  if (general)
    fam.inst_internal_gen = internal_gen.data();
  else
    fam.inst_internal = any ? internal.data() : 0;
  xd_csr pat;
  pat.n_rows = n_unknowns_;
  pat.rowptr = rowptr_.data();
  pat.colind = colind.data();
  check_cuda(cudaSetDevice(device_), "cudaSetDevice");
  check_xd(xd_create(&fam, &pat, device_, &ctx_), "xd_create");
  // State / store permutation: slot s of instance i lives at the instance's s-th LID. With the
  // general topology the library keeps eight state slots (qb, qg, qd, qgmid, qbs, qbd, qcheq,
  // qcdump) and an instance registers qgmid only with rgateMod 3, qbs / qbd only with rbodyMod and
  // qcheq / qcdump only with trnqsMod (registerStateLIDs, N_DEV_MOSFET_B4.C:5212-5238): the slots
  // it lacks get no LID (-1).
  const int nst = xd_num_state_slots(ctx_), nso = xd_num_store_slots(ctx_);
  sta_lid_.assign((size_t)nst * n_, -1);
  sto_lid_.resize((size_t)nso * n_);
  for (int i = 0; i < n_; ++i) {
    const std::vector<int> &st = LidAccess::sta(*insts[i]), &so = LidAccess::sto(*insts[i]);
    if ((int)so.size() < nso)
      throw std::runtime_error("GPU MOSFET binding: store registration differs from the library's");
    if (general) {
      const int *fl = &gflags[(size_t)XD_GEN_INTERNAL * i];
      const bool rg3 = fl[3] != 0, rb = fl[4] != 0, nqs = fl[7] != 0;
      const int want = 3 + (rg3 ? 1 : 0) + (rb ? 2 : 0) + (nqs ? 2 : 0);
      if ((int)st.size() != want)
        throw std::runtime_error("GPU MOSFET binding: state registration differs from the library's");
      int next = 0;
      for (int s = 0; s < nst; ++s) {
        const bool has = s < 3 || (s == 3 && rg3) || ((s == 4 || s == 5) && rb) || (s > 5 && nqs);
        sta_lid_[(size_t)s * n_ + i] = has ? st[next++] : -1;
      }
    } else {
      if ((int)st.size() < nst)
        throw std::runtime_error("GPU MOSFET binding: state registration differs from the library's");
      for (int s = 0; s < nst; ++s) sta_lid_[(size_t)s * n_ + i] = st[s];
    }
    for (int s = 0; s < nso; ++s) sto_lid_[(size_t)s * n_ + i] = so[s];
  }
  cudaStream_t st;
  check_cuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
  stream_ = st;
  const size_t nu = std::max(1, n_unknowns_), nz = std::max(1, nnz_);
  check_cuda(cudaMalloc(&d_sol_, nu * sizeof(double)), "allocation");
  for (int k = 0; k < 2; ++k) {
    check_cuda(cudaMalloc(&d_sta_[k], sta_lid_.size() * sizeof(double)), "allocation");
    check_cuda(cudaMalloc(&d_sto_[k], sto_lid_.size() * sizeof(double)), "allocation");
    h_sta_[k].resize(sta_lid_.size());
    h_sto_[k].resize(sto_lid_.size());
  }
  for (int k = 0; k < 4; ++k) {
    check_cuda(cudaMalloc(&d_vec_[k], nu * sizeof(double)), "allocation");
    h_vec_[k].resize(nu);
  }
  check_cuda(cudaMalloc(&d_jf_, nz * sizeof(double)), "allocation");
  check_cuda(cudaMalloc(&d_jq_, nz * sizeof(double)), "allocation");
  h_sol_.resize(nu);
  h_jf_.resize(nz);
  h_jq_.resize(nz);
  return ready_ = true;
}

bool Master::updateState(double *solVec, double *staVec, double *stoVec) {
  setup();
  if (n_ == 0) return true;
  const ExternData &ext = (*getInstanceBegin())->getExternData();
  double *currSta = ext.currStaVectorRawPtr;
  const double *currSto = ext.currStoVectorRawPtr;
  cudaStream_t st = (cudaStream_t)stream_;
  std::copy(solVec, solVec + n_unknowns_, h_sol_.begin());
  for (size_t k = 0; k < sta_lid_.size(); ++k) {
    const int lid = sta_lid_[k];
    h_sta_[0][k] = lid >= 0 ? staVec[lid] : 0.0;
    h_sta_[1][k] = lid >= 0 ? currSta[lid] : 0.0;
  }
  for (size_t k = 0; k < sto_lid_.size(); ++k) {
    h_sto_[0][k] = stoVec[sto_lid_[k]];
    h_sto_[1][k] = currSto[sto_lid_[k]];
  }
  check_cuda(cudaMemcpyAsync(d_sol_, h_sol_.data(), n_unknowns_ * sizeof(double), cudaMemcpyHostToDevice, st), "copy");
  for (int k = 0; k < 2; ++k) {
    check_cuda(cudaMemcpyAsync(d_sta_[k], h_sta_[k].data(), h_sta_[k].size() * sizeof(double), cudaMemcpyHostToDevice, st),
               "copy");
    check_cuda(cudaMemcpyAsync(d_sto_[k], h_sto_[k].data(), h_sto_[k].size() * sizeof(double), cudaMemcpyHostToDevice, st),
               "copy");
  }
  const xd_flags f = flags_from(getSolverState(), getDeviceOptions());
  check_xd(xd_update_state(ctx_, &f, d_sol_, d_sta_[0], d_sta_[1], d_sto_[0], d_sto_[1], st), "xd_update_state");
  check_cuda(cudaMemcpyAsync(h_sta_[0].data(), d_sta_[0], h_sta_[0].size() * sizeof(double), cudaMemcpyDeviceToHost, st),
             "copy");
  check_cuda(cudaMemcpyAsync(h_sta_[1].data(), d_sta_[1], h_sta_[1].size() * sizeof(double), cudaMemcpyDeviceToHost, st),
             "copy");
  check_cuda(cudaMemcpyAsync(h_sto_[0].data(), d_sto_[0], h_sto_[0].size() * sizeof(double), cudaMemcpyDeviceToHost, st),
             "copy");
  check_cuda(cudaStreamSynchronize(st), "synchronize");
  for (size_t k = 0; k < sta_lid_.size(); ++k) {
    if (sta_lid_[k] < 0) continue;
    staVec[sta_lid_[k]] = h_sta_[0][k];
    currSta[sta_lid_[k]] = h_sta_[1][k];
  }
  for (size_t k = 0; k < sto_lid_.size(); ++k) stoVec[sto_lid_[k]] = h_sto_[0][k];
  return true;
}

bool Master::loadDAEVectors(double *solVec, double *fVec, double *qVec, double *bVec, double *storeLeadF,
                            double *storeLeadQ) {
  (void)solVec; (void)bVec; (void)storeLeadF; (void)storeLeadQ;  // BSIM4 loads neither B nor lead currents
  if (n_ == 0) return true;
  const ExternData &ext = (*getInstanceBegin())->getExternData();
  double *out[4] = {fVec, qVec, ext.dFdxdVpVectorRawPtr, ext.dQdxdVpVectorRawPtr};
  cudaStream_t st = (cudaStream_t)stream_;
  for (int k = 0; k < 4; ++k) check_cuda(cudaMemsetAsync(d_vec_[k], 0, n_unknowns_ * sizeof(double), st), "memset");
  check_xd(xd_load_vectors(ctx_, d_vec_[0], d_vec_[1], d_vec_[2], d_vec_[3], st), "xd_load_vectors");
  for (int k = 0; k < 4; ++k)
    check_cuda(cudaMemcpyAsync(h_vec_[k].data(), d_vec_[k], n_unknowns_ * sizeof(double), cudaMemcpyDeviceToHost, st),
               "copy");
  check_cuda(cudaStreamSynchronize(st), "synchronize");
  for (int k = 0; k < 4; ++k)
    for (int i = 0; i < n_unknowns_; ++i) out[k][i] += h_vec_[k][i];
  return true;
}

bool Master::loadDAEMatrices(N_LAS_Matrix &dFdx, N_LAS_Matrix &dQdx) {
  if (n_ == 0) return true;
  cudaStream_t st = (cudaStream_t)stream_;
  check_cuda(cudaMemsetAsync(d_jf_, 0, nnz_ * sizeof(double), st), "memset");
  check_cuda(cudaMemsetAsync(d_jq_, 0, nnz_ * sizeof(double), st), "memset");
  check_xd(xd_load_matrices(ctx_, d_jf_, d_jq_, st), "xd_load_matrices");
  check_cuda(cudaMemcpyAsync(h_jf_.data(), d_jf_, nnz_ * sizeof(double), cudaMemcpyDeviceToHost, st), "copy");
  check_cuda(cudaMemcpyAsync(h_jq_.data(), d_jq_, nnz_ * sizeof(double), cudaMemcpyDeviceToHost, st), "copy");
  check_cuda(cudaStreamSynchronize(st), "synchronize");
  // Add row by row through the matrices' own row views (dF/dx and dQ/dx share one graph).
  for (int r = 0; r < n_unknowns_; ++r) {
    int len = 0, lenq = 0;
    double *vf = 0, *vq = 0;
    int *idx = 0, *idq = 0;
    dFdx.extractLocalRowView(r, len, vf, idx);
    dQdx.extractLocalRowView(r, lenq, vq, idq);
    const int b = rowptr_[r];
    if (len != rowptr_[r + 1] - b || lenq != len)
      throw std::runtime_error("GPU MOSFET binding: the matrices' pattern changed after set-up");
    for (int j = 0; j < len; ++j) {
      vf[j] += h_jf_[b + pos_[b + j]];
      vq[j] += h_jq_[b + pos_[b + j]];
    }
  }
  return true;
}

namespace {
Device *factory(const Configuration &configuration, const FactoryBlock &factory_block) {
  return new Master(configuration, factory_block, factory_block.solverState_, factory_block.deviceOptions_);
}
struct GpuTraits : public MOSFET_B4::Traits {
  static Device *factory(const Configuration &c, const FactoryBlock &fb) { return GpuMosfetB4::factory(c, fb); }
};
}  // namespace

void registerDevice() {
  Config<GpuTraits>::addConfiguration()
      .registerDevice("m", 14)
      .registerDevice("m", 54)
      .registerModelType("pmos", 14)
      .registerModelType("nmos", 14)
      .registerModelType("pmos", 54)
      .registerModelType("nmos", 54);
}

}  // namespace GpuMosfetB4
}  // namespace Device
}  // namespace Xyce
