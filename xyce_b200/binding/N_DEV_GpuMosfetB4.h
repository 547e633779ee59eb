// N_DEV_GpuMosfetB4.h — the reference-side binding of the B200 device load for BSIM4.
//
// A device master for the reference simulator that keeps the reference's BSIM4 model and instance
// objects for everything around the load (parameter processing, topology: LIDs, state and store
// LIDs, Jacobian offsets), and performs the three per-iteration calls the device manager makes —
// Device::updateState, Device::loadDAEVectors and Device::loadDAEMatrices
// (src/DeviceModelPKG/Core/include/N_DEV_Device.h:315, 361, 384) — through the C ABI of
// libxyce_b200.so (include/xyce_devload.h) on a CUDA device instead of instance by instance on the
// host (MOSFET_B4::Master, src/DeviceModelPKG/OpenModels/src/N_DEV_MOSFET_B4.C:16180-17268).
//
// It derives from the reference's MOSFET_B4::Master, so a netlist sees the same device: the same
// model and instance parameters, the same internal nodes and the same state / store registration.
// The first updateState after the topology has registered every instance's LIDs and Jacobian
// offsets builds the library context from the recorded .MODEL cards and instance lines, the
// instances' node LIDs and the dF/dx matrix's pattern.
//
// Layout conversions the binding performs on every call:
//   - node LIDs: the reference's vectors carry the ground node as their last entry (the overlap map
//     with ground, src/LinearAlgebraServicesPKG/src/N_LAS_Builder.C:416-440); the library takes
//     the unknowns without ground and ground as -1;
//   - state / store: the reference hands each instance its own LIDs
//     (registerStateLIDs / registerStoreLIDs, N_DEV_MOSFET_B4.C:5200, 5267); the library's blocks are
//     slot-major ([slot * n + i]); the binding gathers and scatters through the instances' LIDs;
//   - outputs: the library writes the family's sums into device buffers, which the binding adds into
//     the reference's F, Q, dF/dx*dVp, dQ/dx*dVp vectors and dF/dx, dQ/dx matrices (the devices'
//     += contract, N_LOA_NonlinearEquationLoader.C:128-133, 226-227).
//
// Registration: GpuMosfetB4::registerDevice() registers the binding for "m" levels 14 and 54 in
// place of MOSFET_B4::registerDevice() (N_DEV_MOSFET_B4.C:17276-17285); call one or the other.
#ifndef Xyce_N_DEV_GpuMosfetB4_h
#define Xyce_N_DEV_GpuMosfetB4_h

#include <string>
#include <utility>
#include <vector>

#include <N_DEV_MOSFET_B4.h>

struct xd_ctx;

namespace Xyce {
namespace Device {
namespace GpuMosfetB4 {

class Master : public MOSFET_B4::Master {
 public:
  Master(const Configuration &configuration, const FactoryBlock &factory_block, const SolverState &ss,
         const DeviceOptions &dopts, int cuda_device = 0);
  virtual ~Master();

  virtual MOSFET_B4::Model *addModel(const ModelBlock &model_block, const FactoryBlock &factory_block);
  virtual MOSFET_B4::Instance *addInstance(const InstanceBlock &instance_block, const FactoryBlock &factory_block);

  virtual bool updateState(double *solVec, double *staVec, double *stoVec);
  virtual bool loadDAEVectors(double *solVec, double *fVec, double *qVec, double *bVec, double *storeLeadF,
                              double *storeLeadQ);
  virtual bool loadDAEMatrices(N_LAS_Matrix &dFdx, N_LAS_Matrix &dQdx);

 private:
  struct Card {
    std::string name;
    bool pmos;
    std::vector<std::pair<std::string, double> > params;
  };
  struct Line {
    std::string model;
    std::vector<std::pair<std::string, double> > params;
  };
  bool setup();
  void release();

  int device_;
  std::vector<Card> cards_;
  std::vector<Line> lines_;
  xd_ctx *ctx_;
  bool ready_;
  int n_, n_rows_, n_unknowns_, nnz_, ground_;
  std::vector<int> rowptr_, pos_;                // pattern over the unknowns; pos_: storage order -> sorted order
  std::vector<int> sta_lid_, sto_lid_;           // sta_lid_[s * n + i]: reference LID of slot s of instance i
  std::vector<double> h_sol_, h_sta_[2], h_sto_[2], h_vec_[4], h_jf_, h_jq_;
  double *d_sol_, *d_sta_[2], *d_sto_[2], *d_vec_[4], *d_jf_, *d_jq_;
  void *stream_;
};

// Registers the binding for "m" levels 14 / 54 and the nmos / pmos model types of those levels.
void registerDevice();

}  // namespace GpuMosfetB4
}  // namespace Device
}  // namespace Xyce

#endif
