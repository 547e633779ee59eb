// B200 device-load library: BSIM4 evaluation kernel, deterministic gather assembly, C ABI.
//
// Per Newton iteration (xd_load):
//   1. bsim4_eval_kernel — one thread per instance. Gathers the 4 terminal voltages, reads the
//      previous iterate's limited voltages, evaluates the model in FP64 registers and writes
//      its 48 local stamp values slot-major into the context's staging array (coalesced: one
//      128-byte line per warp per slot), plus its store/state entries.
//   2. gather kernels — one output entry per thread (or per block for entries with many
//      contributions). Each entry sums its contributions in a fixed order (instance order, then
//      local slot order: the reference's summation order) through a precomputed
//      stamp-to-output map and adds the sum into the caller's vector / CSR value array. No
//      atomics: every run produces bit-identical results.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/xyce_devload.h"
#include "../../include/xyce_tia.h"
#include "bsim4_eval.cuh"
#include "bsim4_setup.h"
#include "bsim3.h"
#include "mos1.h"
#include "tia_long.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *where) {
  return fail(-3, std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e));
}

#define XD_CUDA(call)                                     \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
  } while (0)

constexpr int kLongThreshold = 32;   // entries with more contributions take the chunked path
constexpr int kChunk = 1024;         // contributions per chunk on the chunked path
constexpr int kChunkBlock = 128;

// Stamp-to-output gather map for one group of outputs (the four vectors, or the two matrices).
struct GatherMap {
  int n_short = 0, n_long = 0, n_chunks = 0;
  int *d_short_dst = nullptr, *d_short_ptr = nullptr;  // thread-per-entry path
  int *d_long_dst = nullptr, *d_long_chunk = nullptr;  // chunked path: entry -> [first chunk, next)
  int *d_chunk_begin = nullptr;                        // chunk -> [first contribution, next)
  double *d_partial = nullptr;                         // [NOUT][n_chunks] chunk partial sums
  int *d_src = nullptr;  // staging index within one output's slot range
  size_t n_src = 0;
};

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

// Model families the library evaluates (the reference's device levels).
enum Family { kFamilyMos1 = 1, kFamilyBsim3 = 3, kFamilyBsim4 = 4 };

struct xd_ctx {
  int family = kFamilyBsim4;
  int device = 0;
  int n = 0;
  int n_unknowns = 0;
  int nnz = 0;
  int n_rec = 0;
  double *d_tab = nullptr;
  int *d_rec = nullptr;
  int4 *d_nodes = nullptr;
  double *d_vgb = nullptr;
  double *d_stage = nullptr;
  GatherMap vmap, mmap;
  int eval_variant = 0;
  bool needs_full = false;  // some BSIM4 record uses capMod 0/1 or the gate tunnelling currents
  // Internal drain / source nodes (series resistance): d_ext holds each instance's external drain
  // and source, d_nodes its intrinsic (D', G, S', B); the staging layout widens to 6 vector rows
  // and 22 matrix slots.
  bool series = false;
  int2 *d_ext = nullptr;
  int vec_rows = 4, mat_slots = xb4::kNumMat, stage_slots = xb4::kNumStage;
  int resident_blocks[32] = {};  // per persistent launch shape: blocks resident on the whole device
  // The last evaluation was xd_load_static_scratch: its staged stamps are in the library's static
  // array, so d_stage does not hold them and the calls that read d_stage refuse until the next
  // xd_update_state.
  bool stage_static = false;
  // Hand-off state between the two kernels of a split evaluation (kNumMid slots per instance,
  // slot-major); allocated for the BSIM4 families the split launch shapes evaluate.
  double *d_mid = nullptr;
  // General topology (BSIM4 gate / body resistance, rdsMod 1, instance initial conditions): each
  // instance's 15 local nodes as unknowns (slot-major [node * n + i]; collapsed nodes carry their
  // representative's unknown, ground, an absent charge node and absent branch currents -1), 15
  // vector rows and 85 matrix slots of staging, and 8 state slots per instance.
  bool gen = false;
  int *d_gmap = nullptr;
};

namespace {

// Writes one instance's evaluation results: the staged stamps (the 4-terminal layout, or with SERIES
// the wide one: 6 vector rows, 22 matrix slots), the store and state entries, and vgb.
template <bool SERIES>
__device__ __forceinline__ void bsim4_write_one(int i, int n, const xb4::LoadOut &o, double *__restrict__ next_sta,
                                                double *__restrict__ curr_sta, double *__restrict__ next_sto,
                                                double *__restrict__ vgb, double *__restrict__ stage) {
  if (SERIES) {
    // Wide layout: vector v, row r at (v * 6 + r); rows 4 and 5 (external D, S) carry F only.
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int r = 0; r < 4; ++r) stage[(size_t)(v * xb4::kSerVecRows + r) * n + i] = o.vec[v * 4 + r];
    stage[(size_t)4 * n + i] = o.vecx[0];
    stage[(size_t)5 * n + i] = o.vecx[1];
    const size_t mf = 4 * xb4::kSerVecRows, mq = mf + xb4::kSerMat;
#pragma unroll
    for (int k = 0; k < xb4::kNumMat; ++k) stage[(mf + k) * n + i] = o.jf[k];
#pragma unroll
    for (int k = 0; k < 6; ++k) stage[(mf + xb4::kNumMat + k) * n + i] = o.jfx[k];
#pragma unroll
    for (int k = 0; k < xb4::kNumMat; ++k) stage[(mq + k) * n + i] = o.jq[k];
  } else {
#pragma unroll
    for (int k = 0; k < xb4::kNumVec; ++k) stage[(size_t)k * n + i] = o.vec[k];
#pragma unroll
    for (int k = 0; k < xb4::kNumMat; ++k) stage[(size_t)(xb4::kNumVec + k) * n + i] = o.jf[k];
#pragma unroll
    for (int k = 0; k < xb4::kNumMat; ++k) stage[(size_t)(xb4::kNumVec + xb4::kNumMat + k) * n + i] = o.jq[k];
  }
#pragma unroll
  for (int k = 0; k < xb4::kNumStore; ++k)
    if (k != xb4::s_vged && k != xb4::s_vgmd) next_sto[(size_t)k * n + i] = o.sto[k];
#pragma unroll
  for (int k = 0; k < xb4::kNumState; ++k) next_sta[(size_t)k * n + i] = o.sta[k];
  if (o.write_curr_sta) {
#pragma unroll
    for (int k = 0; k < xb4::kNumState; ++k) curr_sta[(size_t)k * n + i] = o.sta[k];
  }
  vgb[i] = o.vgb;
}

// One instance's node voltages (D, G, S, B; ground reads 0 V) and, with SERIES, its external
// drain and source voltages.
template <bool SERIES>
__device__ __forceinline__ void bsim4_gather_v(int i, const int4 *__restrict__ nodes, const int2 *__restrict__ ext,
                                               const double *__restrict__ sol, double V[4], double Vx[2]) {
  const int4 nd = nodes[i];
  V[0] = nd.x >= 0 ? sol[nd.x] : 0.0;
  V[1] = nd.y >= 0 ? sol[nd.y] : 0.0;
  V[2] = nd.z >= 0 ? sol[nd.z] : 0.0;
  V[3] = nd.w >= 0 ? sol[nd.w] : 0.0;
  if (SERIES) {
    const int2 ex = ext[i];
    Vx[0] = ex.x >= 0 ? sol[ex.x] : 0.0;
    Vx[1] = ex.y >= 0 ? sol[ex.y] : 0.0;
  } else {
    Vx[0] = Vx[1] = 0.0;
  }
}

// The store values the limiter compares against (currSto on Newton step 0, nextSto otherwise).
__device__ __forceinline__ void bsim4_sto_old(int i, int n, const double *__restrict__ next_sto,
                                              const double *__restrict__ curr_sto, const xb4::LoadFlags &fl,
                                              double sto_old[xb4::kNumStore]) {
  const double *so = (fl.newton_iter == 0) ? curr_sto : next_sto;
#pragma unroll
  for (int k = 0; k < xb4::kNumStore; ++k) sto_old[k] = 0.0;
  sto_old[xb4::s_vbd] = so[(size_t)xb4::s_vbd * n + i];
  sto_old[xb4::s_vbs] = so[(size_t)xb4::s_vbs * n + i];
  sto_old[xb4::s_vgs] = so[(size_t)xb4::s_vgs * n + i];
  sto_old[xb4::s_vds] = so[(size_t)xb4::s_vds * n + i];
  sto_old[xb4::s_von] = so[(size_t)xb4::s_von * n + i];
}

// One instance's evaluation and staging. SERIES: the family has internal drain / source nodes; ext
// holds the external drain and source of each instance and the staging layout is the wide one
// (6 vector rows, 22 matrix slots).
template <bool FULL, bool SERIES>
__device__ __forceinline__ void bsim4_eval_one(
    int i, int n, const double *__restrict__ tab, int nrec, const int *__restrict__ rec,
    const int4 *__restrict__ nodes, const double *__restrict__ sol, double *__restrict__ next_sta,
    double *__restrict__ curr_sta, double *__restrict__ next_sto, const double *__restrict__ curr_sto,
    double *__restrict__ vgb, double *__restrict__ stage, const xb4::LoadFlags &fl, const int2 *__restrict__ ext) {
  double V[4], Vx[2], sto_old[xb4::kNumStore];
  bsim4_gather_v<SERIES>(i, nodes, ext, sol, V, Vx);
  bsim4_sto_old(i, n, next_sto, curr_sto, fl, sto_old);
  xb4::RecPtr rp{tab + rec[i], nrec};
  xb4::LoadOut o;
  xb4::bsim4_load<FULL, SERIES>(rp, V, sto_old, fl, vgb[i], o, Vx);
  bsim4_write_one<SERIES>(i, n, o, next_sta, curr_sta, next_sto, vgb, stage);
}

// Split evaluation, first kernel: the DC part of one instance (limiting, junction diodes, drain
// current, GIDL / GISL, gate tunnelling); its hand-off state goes to mid, slot-major.
// Split evaluation, first kernel's body: the DC part of instance i into the hand-off buffer.
template <bool FULL, bool SERIES>
__device__ __forceinline__ void bsim4_dc_one(int i, int n, const double *__restrict__ tab, int nrec,
                                             const int *__restrict__ rec, const int4 *__restrict__ nodes,
                                             const double *__restrict__ sol, const double *__restrict__ next_sto,
                                             const double *__restrict__ curr_sto, const double *__restrict__ vgb,
                                             const xb4::LoadFlags &fl, const int2 *__restrict__ ext,
                                             double *__restrict__ mid) {
  double V[4], Vx[2], sto_old[xb4::kNumStore];
  bsim4_gather_v<SERIES>(i, nodes, ext, sol, V, Vx);
  bsim4_sto_old(i, n, next_sto, curr_sto, fl, sto_old);
  xb4::RecPtr rp{tab + rec[i], nrec};
  xb4::LoadOut o;
  xb4::Mid m;
  xb4::bsim4_load<FULL, SERIES, 1>(rp, V, sto_old, fl, vgb[i], o, Vx, &m);
  constexpr int nm = FULL ? xb4::kNumMidFull : xb4::kNumMid;
#pragma unroll
  for (int f = 0; f < nm; ++f) mid[(size_t)f * n + i] = m.v[f];
}

template <int BLOCK, int MINB, bool FULL, bool SERIES>
__global__ void __launch_bounds__(BLOCK, MINB) bsim4_dc_kernel(
    int n, const double *__restrict__ tab, int nrec, const int *__restrict__ rec, const int4 *__restrict__ nodes,
    const double *__restrict__ sol, const double *__restrict__ next_sto, const double *__restrict__ curr_sto,
    const double *__restrict__ vgb, xb4::LoadFlags fl, const int2 *__restrict__ ext, double *__restrict__ mid) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bsim4_dc_one<FULL, SERIES>(i, n, tab, nrec, rec, nodes, sol, next_sto, curr_sto, vgb, fl, ext, mid);
}

// The same DC part under an explicit register budget instead of launch bounds (112 registers a
// thread, in 64- or 96-thread blocks): an autotuner candidate that times within noise of 128 x 4
// on the scale circuit (the register file still holds 16 of its warps per SM).
template <int REGS>
__global__ void __maxnreg__(REGS) bsim4_dc_kernel_regs(
    int n, const double *__restrict__ tab, int nrec, const int *__restrict__ rec, const int4 *__restrict__ nodes,
    const double *__restrict__ sol, const double *__restrict__ next_sto, const double *__restrict__ curr_sto,
    const double *__restrict__ vgb, xb4::LoadFlags fl, const int2 *__restrict__ ext, double *__restrict__ mid) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bsim4_dc_one<false, false>(i, n, tab, nrec, rec, nodes, sol, next_sto, curr_sto, vgb, fl, ext, mid);
}

// Split evaluation, second kernel: charges, capacitances, store / state and the stamps of one
// instance from the DC part's hand-off state; writes the same outputs as bsim4_eval_kernel.
template <int BLOCK, int MINB, bool FULL, bool SERIES>
__global__ void __launch_bounds__(BLOCK, MINB) bsim4_charge_stamp_kernel(
    int n, const double *__restrict__ tab, int nrec, const int *__restrict__ rec, const int4 *__restrict__ nodes,
    const double *__restrict__ sol, double *__restrict__ next_sta, double *__restrict__ curr_sta,
    double *__restrict__ next_sto, double *__restrict__ vgb, double *__restrict__ stage, xb4::LoadFlags fl,
    const int2 *__restrict__ ext, const double *__restrict__ mid) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double V[4], Vx[2];
  bsim4_gather_v<SERIES>(i, nodes, ext, sol, V, Vx);
  xb4::Mid m;
  constexpr int nm = FULL ? xb4::kNumMidFull : xb4::kNumMid;
#pragma unroll
  for (int f = 0; f < nm; ++f) m.v[f] = mid[(size_t)f * n + i];
  xb4::RecPtr rp{tab + rec[i], nrec};
  xb4::LoadOut o;
  xb4::bsim4_load<FULL, SERIES, 2>(rp, V, nullptr, fl, vgb[i], o, Vx, &m);
  bsim4_write_one<SERIES>(i, n, o, next_sta, curr_sta, next_sto, vgb, stage);
}

// General topology: the 15 local nodes' values of instance i (absent nodes and ground read 0 V).
__device__ __forceinline__ void bsim4_gen_gather(int i, int n, const int *__restrict__ gmap,
                                                 const double *__restrict__ sol, double *V) {
#pragma unroll
  for (int k = 0; k < xb4::kGenNodes; ++k) {
    const int u = gmap[(size_t)k * n + i];
    V[k] = u >= 0 ? sol[u] : 0.0;
  }
}

// General topology: one instance's staged stamps (15 vector rows x 4, 85 dF/dx and 85 dQ/dx
// slots), store (vged / vgmd kept from the input), eight state slots and carried vgb.
__device__ __forceinline__ void bsim4_gen_write(int i, int n, const xb4::LoadOut &o, double *__restrict__ next_sta,
                                                double *__restrict__ curr_sta, double *__restrict__ next_sto,
                                                double *__restrict__ vgb, double *__restrict__ stage) {
#pragma unroll
  for (int k = 0; k < 4 * xb4::kGenNodes; ++k) stage[(size_t)k * n + i] = o.gv[k];
  const size_t mf = 4 * xb4::kGenNodes, mq = mf + xb4::kGenSlots;
#pragma unroll
  for (int k = 0; k < xb4::kGenSlots; ++k) stage[(mf + k) * n + i] = o.gf[k];
#pragma unroll
  for (int k = 0; k < xb4::kGenSlots; ++k) stage[(mq + k) * n + i] = o.gq[k];
#pragma unroll
  for (int k = 0; k < xb4::kNumStore; ++k)
    if (k != xb4::s_vged && k != xb4::s_vgmd) next_sto[(size_t)k * n + i] = o.sto[k];
#pragma unroll
  for (int k = 0; k < xb4::kGenState; ++k) next_sta[(size_t)k * n + i] = o.gsta[k];
  if (o.write_curr_sta) {
#pragma unroll
    for (int k = 0; k < xb4::kGenState; ++k) curr_sta[(size_t)k * n + i] = o.gsta[k];
  }
  vgb[i] = o.vgb;
}

// General topology: one thread per instance over the 15 local nodes; the full store block is read
// (the limiters of the gate, source / drain and body-network voltages compare against it) and the
// eight state slots written.
template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) bsim4_gen_kernel(
    int n, const double *__restrict__ tab, int nrec, const int *__restrict__ rec, const int *__restrict__ gmap,
    const double *__restrict__ sol, double *__restrict__ next_sta, double *__restrict__ curr_sta,
    double *__restrict__ next_sto, const double *__restrict__ curr_sto, double *__restrict__ vgb,
    double *__restrict__ stage, xb4::LoadFlags fl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double V[xb4::kGenNodes], sto_old[xb4::kNumStore];
  bsim4_gen_gather(i, n, gmap, sol, V);
  const double *so = (fl.newton_iter == 0) ? curr_sto : next_sto;
#pragma unroll
  for (int k = 0; k < xb4::kNumStore; ++k) sto_old[k] = so[(size_t)k * n + i];
  xb4::RecPtr rp{tab + rec[i], nrec};
  xb4::LoadOut o;
  xb4::bsim4_load<true, false, 0, true>(rp, V, sto_old, fl, vgb[i], o);
  bsim4_gen_write(i, n, o, next_sta, curr_sta, next_sto, vgb, stage);
}

// General topology, split like bsim4_dc_kernel / bsim4_charge_stamp_kernel: the DC part writes the
// general hand-off state (kNumMidGen doubles per instance, slot-major), the charge-and-stamp part
// reads it; together they load what bsim4_gen_kernel loads, bit for bit.
template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) bsim4_gen_dc_kernel(
    int n, const double *__restrict__ tab, int nrec, const int *__restrict__ rec, const int *__restrict__ gmap,
    const double *__restrict__ sol, const double *__restrict__ next_sto, const double *__restrict__ curr_sto,
    const double *__restrict__ vgb, xb4::LoadFlags fl, double *__restrict__ mid) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double V[xb4::kGenNodes], sto_old[xb4::kNumStore];
  bsim4_gen_gather(i, n, gmap, sol, V);
  const double *so = (fl.newton_iter == 0) ? curr_sto : next_sto;
#pragma unroll
  for (int k = 0; k < xb4::kNumStore; ++k) sto_old[k] = so[(size_t)k * n + i];
  xb4::RecPtr rp{tab + rec[i], nrec};
  xb4::LoadOut o;
  xb4::Mid m;
  xb4::bsim4_load<true, false, 1, true>(rp, V, sto_old, fl, vgb[i], o, nullptr, &m);
#pragma unroll
  for (int f = 0; f < xb4::kNumMidGen; ++f) mid[(size_t)f * n + i] = m.v[f];
}

template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) bsim4_gen_cs_kernel(
    int n, const double *__restrict__ tab, int nrec, const int *__restrict__ rec, const int *__restrict__ gmap,
    const double *__restrict__ sol, double *__restrict__ next_sta, double *__restrict__ curr_sta,
    double *__restrict__ next_sto, double *__restrict__ vgb, double *__restrict__ stage, xb4::LoadFlags fl,
    const double *__restrict__ mid) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double V[xb4::kGenNodes];
  bsim4_gen_gather(i, n, gmap, sol, V);
  xb4::Mid m;
#pragma unroll
  for (int f = 0; f < xb4::kNumMidGen; ++f) m.v[f] = mid[(size_t)f * n + i];
  xb4::RecPtr rp{tab + rec[i], nrec};
  xb4::LoadOut o;
  xb4::bsim4_load<true, false, 2, true>(rp, V, nullptr, fl, vgb[i], o, nullptr, &m);
  bsim4_gen_write(i, n, o, next_sta, curr_sta, next_sto, vgb, stage);
}

// One thread per instance. PERSIST: the grid is one wave of resident blocks that walks the
// instances with a grid stride, so the warps resident on an SM start together and run through the
// model's long straight-line code at about the same point, sharing its instruction-cache lines
// (a grid of one block per 128 instances refills an SM as blocks finish, which leaves the resident
// blocks a fraction of the code apart).
template <int BLOCK, int MINB, bool FULL, bool SERIES, bool PERSIST = false>
__global__ void __launch_bounds__(BLOCK, MINB) bsim4_eval_kernel(
    int n, const double *__restrict__ tab, int nrec, const int *__restrict__ rec, const int4 *__restrict__ nodes,
    const double *__restrict__ sol, double *__restrict__ next_sta, double *__restrict__ curr_sta,
    double *__restrict__ next_sto, const double *__restrict__ curr_sto, double *__restrict__ vgb,
    double *__restrict__ stage, xb4::LoadFlags fl, const int2 *__restrict__ ext) {
  if (PERSIST) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
      bsim4_eval_one<FULL, SERIES>(i, n, tab, nrec, rec, nodes, sol, next_sta, curr_sta, next_sto, curr_sto, vgb,
                                   stage, fl, ext);
  } else {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
      bsim4_eval_one<FULL, SERIES>(i, n, tab, nrec, rec, nodes, sol, next_sta, curr_sta, next_sto, curr_sto, vgb,
                                   stage, fl, ext);
  }
}

// MOSFET level 1: one thread per instance; reads the previous time point's Meyer state for
// back-averaging. SERIES: the nodes are (D', G, S', B), ext the external (D, S), and the staging
// is the wide layout.
template <int BLOCK, int MINB, bool SERIES>
__global__ void __launch_bounds__(BLOCK, MINB) mos1_eval_kernel(
    int n, const double *__restrict__ tab, int nrec, const int *__restrict__ rec, const int4 *__restrict__ nodes,
    const double *__restrict__ sol, double *__restrict__ next_sta, const double *__restrict__ curr_sta,
    double *__restrict__ next_sto, const double *__restrict__ curr_sto, double *__restrict__ stage,
    xb4::LoadFlags fl, const int2 *__restrict__ ext) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 nd = nodes[i];
  double V[4];
  V[0] = nd.x >= 0 ? sol[nd.x] : 0.0;
  V[1] = nd.y >= 0 ? sol[nd.y] : 0.0;
  V[2] = nd.z >= 0 ? sol[nd.z] : 0.0;
  V[3] = nd.w >= 0 ? sol[nd.w] : 0.0;
  const double *so = (fl.newton_iter == 0) ? curr_sto : next_sto;
  double sto_old[xm1::kNumStore], csto[xm1::kNumStore], csta[xm1::kNumState];
#pragma unroll
  for (int k = 0; k < xm1::kNumStore; ++k) {
    sto_old[k] = so[(size_t)k * n + i];
    csto[k] = curr_sto[(size_t)k * n + i];
  }
#pragma unroll
  for (int k = 0; k < xm1::kNumState; ++k) csta[k] = curr_sta[(size_t)k * n + i];
  xb4::RecPtr rp{tab + rec[i], nrec};
  xm1::LoadOut o;
  if (SERIES) {
    const int2 ex = ext[i];
    double Vx[2];
    Vx[0] = ex.x >= 0 ? sol[ex.x] : 0.0;
    Vx[1] = ex.y >= 0 ? sol[ex.y] : 0.0;
    xm1::mos1_load<true>(rp, V, sto_old, csta, csto, fl, o, Vx);
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int r = 0; r < 4; ++r) stage[(size_t)(v * xb4::kSerVecRows + r) * n + i] = o.vec[v * 4 + r];
    stage[(size_t)4 * n + i] = o.vecx[0];
    stage[(size_t)5 * n + i] = o.vecx[1];
    const size_t mf = 4 * xb4::kSerVecRows, mq = mf + xb4::kSerMat;
#pragma unroll
    for (int k = 0; k < xb4::kNumMat; ++k) stage[(mf + k) * n + i] = o.jf[k];
#pragma unroll
    for (int k = 0; k < 6; ++k) stage[(mf + xb4::kNumMat + k) * n + i] = o.jfx[k];
#pragma unroll
    for (int k = 0; k < xb4::kNumMat; ++k) stage[(mq + k) * n + i] = o.jq[k];
  } else {
    xm1::mos1_load<false>(rp, V, sto_old, csta, csto, fl, o);
#pragma unroll
    for (int k = 0; k < xb4::kNumVec; ++k) stage[(size_t)k * n + i] = o.vec[k];
#pragma unroll
    for (int k = 0; k < xb4::kNumMat; ++k) stage[(size_t)(xb4::kNumVec + k) * n + i] = o.jf[k];
#pragma unroll
    for (int k = 0; k < xb4::kNumMat; ++k) stage[(size_t)(xb4::kNumVec + xb4::kNumMat + k) * n + i] = o.jq[k];
  }
#pragma unroll
  for (int k = 0; k < xm1::kNumStore; ++k) next_sto[(size_t)k * n + i] = o.sto[k];
#pragma unroll
  for (int k = 0; k < xm1::kNumState; ++k) next_sta[(size_t)k * n + i] = o.sta[k];
}

template <int NOUT, bool ABS>
struct OutSet {
  double *out[NOUT];
  size_t base[NOUT];  // staging offset of each output's slot range
  int assign = 0;     // 1: store the family's sum (=) instead of adding it (+=)
};

// acc[o] += the staged values stage[base[o] + src[k]] for k in [b, e), in k order. The sources are
// read kGatherBatch at a time, all their loads issued before the first add, so that a target with
// many sources (a node row of the vector map) waits for one round of loads per batch instead of one
// per source; the adds keep the sequential order.
constexpr int kGatherBatch = 4;
template <int NOUT, bool ABS>
__device__ __forceinline__ void sum_sources(int b, int e, const int *__restrict__ src,
                                            const double *__restrict__ stage, const size_t *base, double *acc) {
  for (int k = b; k < e; k += kGatherBatch) {
    size_t s[kGatherBatch];
#pragma unroll
    for (int j = 0; j < kGatherBatch; ++j) s[j] = k + j < e ? (size_t)src[k + j] : 0;
    double v[kGatherBatch][NOUT];
#pragma unroll
    for (int j = 0; j < kGatherBatch; ++j)
#pragma unroll
      for (int o = 0; o < NOUT; ++o) v[j][o] = k + j < e ? stage[base[o] + s[j]] : 0.0;
#pragma unroll
    for (int j = 0; j < kGatherBatch; ++j)
      if (k + j < e) {
#pragma unroll
        for (int o = 0; o < NOUT; ++o) acc[o] += ABS ? fabs(v[j][o]) : v[j][o];
      }
  }
}

template <int NOUT, bool ABS>
__global__ void gather_short_kernel(int nt, const int *__restrict__ dst, const int *__restrict__ ptr,
                                    const int *__restrict__ src, const double *__restrict__ stage,
                                    OutSet<NOUT, ABS> os) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int b = ptr[t], e = ptr[t + 1];
  double acc[NOUT];
#pragma unroll
  for (int o = 0; o < NOUT; ++o) acc[o] = 0.0;
  sum_sources<NOUT, ABS>(b, e, src, stage, os.base, acc);
  const int d = dst[t];
#pragma unroll
  for (int o = 0; o < NOUT; ++o)
    if (os.out[o]) {
      if (os.assign)
        os.out[o][d] = acc[o];
      else
        os.out[o][d] += acc[o];
    }
}

// Entries with many contributions (the supply rail's row, for instance) are split into fixed
// chunks of kChunk consecutive contributions. Pass 1: one block per chunk sums its chunk with a
// fixed strided split and a fixed-shape tree into a per-chunk partial. Pass 2: one warp per
// entry combines its chunk partials in a fixed tree and adds the result to the output. Both the
// split and the trees are fixed by the map, so the result is bit-identical run to run.
template <int NOUT, bool ABS>
__global__ void __launch_bounds__(kChunkBlock) gather_chunk_kernel(const int *__restrict__ chunk_begin,
                                                                   const int *__restrict__ src,
                                                                   const double *__restrict__ stage,
                                                                   double *__restrict__ partial, int n_chunks,
                                                                   OutSet<NOUT, ABS> os) {
  __shared__ double red[NOUT][kChunkBlock];
  const int c = blockIdx.x;
  const int b = chunk_begin[c], e = chunk_begin[c + 1];
  double acc[NOUT];
#pragma unroll
  for (int o = 0; o < NOUT; ++o) acc[o] = 0.0;
  for (int k = b + threadIdx.x; k < e; k += kChunkBlock) {
    const size_t s = (size_t)src[k];
#pragma unroll
    for (int o = 0; o < NOUT; ++o) {
      const double v = stage[os.base[o] + s];
      acc[o] += ABS ? fabs(v) : v;
    }
  }
#pragma unroll
  for (int o = 0; o < NOUT; ++o) red[o][threadIdx.x] = acc[o];
  __syncthreads();
  for (int w = kChunkBlock / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
#pragma unroll
      for (int o = 0; o < NOUT; ++o) red[o][threadIdx.x] += red[o][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int o = 0; o < NOUT; ++o) partial[(size_t)o * n_chunks + c] = red[o][0];
  }
}

// One block per long entry: threads take the entry's chunk partials with a fixed stride, then a
// fixed tree (a single warp walking ~1,000 partials of a supply rail's entry was a serial tail of
// the gather).
constexpr int kCombineBlock = 256;
template <int NOUT, bool ABS>
__global__ void __launch_bounds__(kCombineBlock) gather_combine_kernel(int n_long, const int *__restrict__ dst,
                                                                       const int *__restrict__ first_chunk,
                                                                       const double *__restrict__ partial,
                                                                       int n_chunks, OutSet<NOUT, ABS> os) {
  __shared__ double red[NOUT][kCombineBlock];
  const int t = blockIdx.x, tid = threadIdx.x;
  const int b = first_chunk[t], e = first_chunk[t + 1];
  double acc[NOUT];
#pragma unroll
  for (int o = 0; o < NOUT; ++o) acc[o] = 0.0;
  for (int k = b + tid; k < e; k += kCombineBlock) {
#pragma unroll
    for (int o = 0; o < NOUT; ++o) acc[o] += partial[(size_t)o * n_chunks + k];
  }
#pragma unroll
  for (int o = 0; o < NOUT; ++o) red[o][tid] = acc[o];
  __syncthreads();
  for (int w = kCombineBlock / 2; w > 0; w >>= 1) {
    if (tid < w) {
#pragma unroll
      for (int o = 0; o < NOUT; ++o) red[o][tid] += red[o][tid + w];
    }
    __syncthreads();
  }
  if (tid == 0) {
    const int d = dst[t];
#pragma unroll
    for (int o = 0; o < NOUT; ++o)
      if (os.out[o]) {
        if (os.assign)
          os.out[o][d] = red[o][0];
        else
          os.out[o][d] += red[o][0];
      }
  }
}

template <int NOUT, bool ABS>
int run_gather(const GatherMap &m, const double *stage, const OutSet<NOUT, ABS> &os, cudaStream_t st,
               bool short_part = true) {
  if (short_part && m.n_short > 0) {
    const int blk = 256;
    gather_short_kernel<NOUT, ABS><<<(m.n_short + blk - 1) / blk, blk, 0, st>>>(m.n_short, m.d_short_dst,
                                                                               m.d_short_ptr, m.d_src, stage, os);
  }
  if (m.n_long > 0) {
    gather_chunk_kernel<NOUT, ABS><<<m.n_chunks, kChunkBlock, 0, st>>>(m.d_chunk_begin, m.d_src, stage, m.d_partial,
                                                                       m.n_chunks, os);
    gather_combine_kernel<NOUT, ABS><<<m.n_long, kCombineBlock, 0, st>>>(
        m.n_long, m.d_long_dst, m.d_long_chunk, m.d_partial, m.n_chunks, os);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "gather launch");
  return 0;
}

// Builds a gather map from (target, source) pairs listed in summation order.
// tgt_of[k] = target index or -1 (dropped); the map keeps, per target, sources in list order.
int build_map(const std::vector<int> &tgt_of, const std::vector<int> &src_of, int n_targets, GatherMap &m) {
  std::vector<int> count(n_targets, 0);
  for (int t : tgt_of)
    if (t >= 0) ++count[t];
  // Order targets: short ones first, long ones in a separate list; both keep ascending target.
  std::vector<int> short_dst, long_dst, short_ptr(1, 0);
  std::vector<long long> start(n_targets, -1);
  size_t n_src = 0;
  for (int t = 0; t < n_targets; ++t)
    if (count[t] > 0 && count[t] <= kLongThreshold) {
      start[t] = (long long)n_src;
      n_src += count[t];
      short_dst.push_back(t);
      short_ptr.push_back((int)n_src);
    }
  std::vector<int> long_chunk(1, 0), chunk_begin;
  for (int t = 0; t < n_targets; ++t)
    if (count[t] > kLongThreshold) {
      start[t] = (long long)n_src;
      for (int k = 0; k < count[t]; k += kChunk) chunk_begin.push_back((int)(n_src + k));
      n_src += count[t];
      long_dst.push_back(t);
      long_chunk.push_back((int)chunk_begin.size());
    }
  chunk_begin.push_back((int)n_src);
  if (n_src > (size_t)0x7fffffff) return fail(-1, "too many stamp contributions for 32-bit gather indices");
  std::vector<int> src(n_src);
  std::vector<long long> fillp(start);
  for (size_t k = 0; k < tgt_of.size(); ++k) {
    const int t = tgt_of[k];
    if (t < 0) continue;
    src[(size_t)fillp[t]++] = src_of[k];
  }
  m.n_short = (int)short_dst.size();
  m.n_long = (int)long_dst.size();
  m.n_chunks = (int)chunk_begin.size() - 1;
  m.n_src = n_src;
  auto up = [](int **d, const std::vector<int> &h) -> cudaError_t {
    if (h.empty()) {
      *d = nullptr;
      return cudaSuccess;
    }
    cudaError_t e = cudaMalloc(d, h.size() * sizeof(int));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*d, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice);
  };
  XD_CUDA(up(&m.d_short_dst, short_dst));
  XD_CUDA(up(&m.d_short_ptr, short_ptr));
  XD_CUDA(up(&m.d_long_dst, long_dst));
  XD_CUDA(up(&m.d_long_chunk, long_chunk));
  XD_CUDA(up(&m.d_chunk_begin, chunk_begin));
  if (m.n_chunks > 0) XD_CUDA(cudaMalloc(&m.d_partial, (size_t)4 * m.n_chunks * sizeof(double)));
  XD_CUDA(up(&m.d_src, src));
  return 0;
}

void free_map(GatherMap &m) {
  cudaFree(m.d_short_dst);
  cudaFree(m.d_short_ptr);
  cudaFree(m.d_long_dst);
  cudaFree(m.d_long_chunk);
  cudaFree(m.d_chunk_begin);
  cudaFree(m.d_partial);
  cudaFree(m.d_src);
  m = GatherMap();
}

// FP64 FMA throughput probe: 8 independent accumulator chains x 8 FMAs per iteration per thread.
__global__ void __launch_bounds__(256) fma_probe_kernel(double *out, int iters) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = 1.0 + 1e-9 * (t + k);
  const double b = 0.999999999, c = 1e-12;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
#pragma unroll
      for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
    }
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  out[t] = s;
}

// Launch shapes of the evaluation kernel. The kernel is register-bound (hundreds of live FP64
// intermediates); the shapes trade occupancy against spills. xd_create times each on the
// circuit and keeps the fastest.
// BSIM3: one thread per instance. SERIES: internal drain / source nodes (ext = external D, S),
// wide staging layout, as for BSIM4.
template <int BLOCK, int MINB, bool SERIES>
__global__ void __launch_bounds__(BLOCK, MINB) bsim3_eval_kernel(
    int n, const double *__restrict__ tab, int nrec, const int *__restrict__ rec, const int4 *__restrict__ nodes,
    const double *__restrict__ sol, double *__restrict__ next_sta, double *__restrict__ curr_sta,
    double *__restrict__ next_sto, const double *__restrict__ curr_sto, double *__restrict__ stage,
    xb4::LoadFlags fl, const int2 *__restrict__ ext) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 nd = nodes[i];
  double V[4];
  V[0] = nd.x >= 0 ? sol[nd.x] : 0.0;
  V[1] = nd.y >= 0 ? sol[nd.y] : 0.0;
  V[2] = nd.z >= 0 ? sol[nd.z] : 0.0;
  V[3] = nd.w >= 0 ? sol[nd.w] : 0.0;
  const double *so = (fl.newton_iter == 0) ? curr_sto : next_sto;
  double sto_old[xb3::kNumStore];
#pragma unroll
  for (int k = 0; k < xb3::kNumStore; ++k) sto_old[k] = so[(size_t)k * n + i];
  xb4::RecPtr rp{tab + rec[i], nrec};
  xb3::LoadOut o;
  if (SERIES) {
    const int2 ex = ext[i];
    double Vx[2];
    Vx[0] = ex.x >= 0 ? sol[ex.x] : 0.0;
    Vx[1] = ex.y >= 0 ? sol[ex.y] : 0.0;
    xb3::bsim3_load<true>(rp, V, sto_old, fl, o, Vx);
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int r = 0; r < 4; ++r) stage[(size_t)(v * xb4::kSerVecRows + r) * n + i] = o.vec[v * 4 + r];
    stage[(size_t)4 * n + i] = o.vecx[0];
    stage[(size_t)5 * n + i] = o.vecx[1];
    const size_t mf = 4 * xb4::kSerVecRows, mq = mf + xb4::kSerMat;
#pragma unroll
    for (int k = 0; k < xb4::kNumMat; ++k) stage[(mf + k) * n + i] = o.jf[k];
#pragma unroll
    for (int k = 0; k < 6; ++k) stage[(mf + xb4::kNumMat + k) * n + i] = o.jfx[k];
#pragma unroll
    for (int k = 0; k < xb4::kNumMat; ++k) stage[(mq + k) * n + i] = o.jq[k];
  } else {
    xb3::bsim3_load<false>(rp, V, sto_old, fl, o);
#pragma unroll
    for (int k = 0; k < xb4::kNumVec; ++k) stage[(size_t)k * n + i] = o.vec[k];
#pragma unroll
    for (int k = 0; k < xb4::kNumMat; ++k) stage[(size_t)(xb4::kNumVec + k) * n + i] = o.jf[k];
#pragma unroll
    for (int k = 0; k < xb4::kNumMat; ++k) stage[(size_t)(xb4::kNumVec + xb4::kNumMat + k) * n + i] = o.jq[k];
  }
#pragma unroll
  for (int k = 0; k < xb3::kNumStore; ++k) next_sto[(size_t)k * n + i] = o.sto[k];
#pragma unroll
  for (int k = 0; k < xb3::kNumState; ++k) next_sta[(size_t)k * n + i] = o.sta[k];
  // Master::updateState also seeds the previous time point's charges on the first step of a
  // transient (N_DEV_MOSFET_B3.C:9248-9262).
  if (!fl.dcop && fl.init_tran && fl.newton_iter == 0) {
#pragma unroll
    for (int k = 0; k < xb3::kNumState; ++k) curr_sta[(size_t)k * n + i] = o.sta[k];
  }
}

struct EvalVariant {
  int family;    // the model family the candidate evaluates
  int block, min_blocks;
  bool full;     // BSIM4: compiled with every supported option (capMod 0/1, gate tunnelling), not only the common card
  bool series;   // BSIM4: internal drain / source nodes, wide staging layout (BSIM3 / MOSFET1 take either layout)
  bool persist;  // one wave of resident blocks with a grid-stride loop
  bool split;    // two kernels: the DC part (min_blocks), then charges and stamps (min_blocks2)
  int min_blocks2;
  bool gen;      // BSIM4 general topology (15 local nodes, 85 stamp slots; split: the general hand-off)
};
constexpr int B4 = 4, B3 = 3, M1 = 1;  // kFamilyBsim4, kFamilyBsim3, kFamilyMos1
constexpr EvalVariant kEvalVariants[] = {
    {B4, 128, 1, false, false, false, false, 0}, {B4, 128, 2, false, false, false, false, 0},
    {B4, 128, 3, false, false, false, false, 0}, {B4, 128, 4, false, false, false, false, 0},
    {B4, 64, 4, false, false, false, false, 0},  {B4, 256, 2, false, false, false, false, 0},
    {B4, 128, 2, true, false, false, false, 0},  {B4, 128, 3, true, false, false, false, 0},
    {B4, 128, 2, true, true, false, false, 0},   {B4, 128, 3, true, true, false, false, 0},
    {B4, 128, 3, false, false, true, false, 0},  {B4, 128, 3, true, false, true, false, 0},
    {B4, 128, 3, false, false, false, true, 3},  {B4, 128, 4, false, false, false, true, 4},
    {B4, 128, 5, false, false, false, true, 5},  {B4, 128, 4, false, false, false, true, 3},
    {B3, 128, 1, false, false, false, false, 0}, {B3, 128, 2, false, false, false, false, 0},
    {B3, 128, 3, false, false, false, false, 0}, {B3, 64, 4, false, false, false, false, 0},
    {M1, 128, 1, false, false, false, false, 0}, {M1, 128, 4, false, false, false, false, 0},
    {M1, 256, 2, false, false, false, false, 0}, {M1, 64, 8, false, false, false, false, 0},
    {B4, 128, 1, true, false, false, false, 0, true}, {B4, 128, 2, true, false, false, false, 0, true},
    {B4, 128, 2, true, false, false, true, 2, true},  {B4, 128, 3, true, false, false, true, 3, true},
    {B4, 96, 6, false, false, false, true, 4},        {B4, 64, 9, false, false, false, true, 4}};
constexpr int kFirstFullVariant = 6, kFirstSeriesVariant = 8, kFirstBsim3Variant = 16, kFirstMos1Variant = 20;
constexpr int kFirstGenVariant = 24;
// A variant computes a context's loads exactly if it is for the context's family and, for BSIM4, its
// staging layout is the context's and it is a full one or the context's cards use only the common
// options; a split one also needs the context's hand-off buffer.
bool variant_fits(const xd_ctx *ctx, int v) {
  const EvalVariant &e = kEvalVariants[v];
  if (e.family != ctx->family) return false;
  if (ctx->family != kFamilyBsim4) return true;
  if (e.gen || ctx->gen) return e.gen == ctx->gen && (!e.split || ctx->d_mid != nullptr);
  return e.series == ctx->series && (e.full || !ctx->needs_full) && (!e.split || ctx->d_mid != nullptr);
}
constexpr int kNumEvalVariants = sizeof(kEvalVariants) / sizeof(kEvalVariants[0]);
static_assert(kNumEvalVariants <= 32, "resident_blocks holds 32 launch shapes");

// The persistent launch shapes' kernels (for the occupancy query).
const void *persistent_eval_kernel(int v) {
  switch (v) {
    case 10: return (const void *)bsim4_eval_kernel<128, 3, false, false, true>;
    case 11: return (const void *)bsim4_eval_kernel<128, 3, true, false, true>;
    default: return nullptr;
  }
}

// One wave of each persistent shape: resident blocks per SM (the occupancy calculator) x SMs.
int size_persistent_grids(xd_ctx *ctx) {
  int sms = 0;
  cudaError_t ce = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "multiprocessor count query");
  for (int v = 0; v < kNumEvalVariants; ++v) {
    if (!kEvalVariants[v].persist) continue;
    int per_sm = 0;
    const void *fn = persistent_eval_kernel(v);
    if (!fn) return fail(-3, "persistent launch shape without a kernel");
    ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kEvalVariants[v].block, 0);
    if (ce != cudaSuccess) return cuda_fail(ce, "occupancy query");
    ctx->resident_blocks[v] = std::max(1, per_sm) * std::max(1, sms);
  }
  return 0;
}

void launch_eval(int v, const xd_ctx *ctx, const xb4::LoadFlags &fl, const double *sol, double *next_sta,
                 double *curr_sta, double *next_sto, const double *curr_sto, double *stage, cudaStream_t st) {
  const int n = ctx->n;
  if (ctx->family == kFamilyMos1) {
    const int blk = kEvalVariants[v].block, grid = (n + blk - 1) / blk;
#define XD_M1_ARGS(E) n, ctx->d_tab, ctx->n_rec, ctx->d_rec, ctx->d_nodes, sol, next_sta, curr_sta, next_sto, curr_sto, \
                      stage, fl, E
#define XD_M1(B, M)                                                                         \
  if (ctx->series)                                                                          \
    mos1_eval_kernel<B, M, true><<<grid, blk, 0, st>>>(XD_M1_ARGS(ctx->d_ext));             \
  else                                                                                      \
    mos1_eval_kernel<B, M, false><<<grid, blk, 0, st>>>(XD_M1_ARGS(nullptr));
    switch (v - kFirstMos1Variant) {
      case 0: XD_M1(128, 1); break;
      case 1: XD_M1(128, 4); break;
      case 2: XD_M1(256, 2); break;
      default: XD_M1(64, 8); break;
    }
#undef XD_M1
#undef XD_M1_ARGS
    return;
  }
  if (ctx->family == kFamilyBsim3) {
    const int blk = kEvalVariants[v].block, grid = (n + blk - 1) / blk;
#define XD_B3_ARGS(E) n, ctx->d_tab, ctx->n_rec, ctx->d_rec, ctx->d_nodes, sol, next_sta, curr_sta, next_sto, curr_sto, \
                      stage, fl, E
#define XD_B3(B, M)                                                                         \
  if (ctx->series)                                                                          \
    bsim3_eval_kernel<B, M, true><<<grid, blk, 0, st>>>(XD_B3_ARGS(ctx->d_ext));            \
  else                                                                                      \
    bsim3_eval_kernel<B, M, false><<<grid, blk, 0, st>>>(XD_B3_ARGS(nullptr));
    switch (v - kFirstBsim3Variant) {
      case 0: XD_B3(128, 1); break;
      case 1: XD_B3(128, 2); break;
      case 2: XD_B3(128, 3); break;
      default: XD_B3(64, 4); break;
    }
#undef XD_B3
#undef XD_B3_ARGS
    return;
  }
  const int blk = kEvalVariants[v].block;
  int grid = (n + blk - 1) / blk;
  if (kEvalVariants[v].gen) {
#define XD_GEN_ARGS n, ctx->d_tab, ctx->n_rec, ctx->d_rec, ctx->d_gmap, sol, next_sta, curr_sta, next_sto, curr_sto, \
                    ctx->d_vgb, stage, fl
#define XD_GEN_DC_ARGS n, ctx->d_tab, ctx->n_rec, ctx->d_rec, ctx->d_gmap, sol, next_sto, curr_sto, ctx->d_vgb, fl, \
                       ctx->d_mid
#define XD_GEN_CS_ARGS n, ctx->d_tab, ctx->n_rec, ctx->d_rec, ctx->d_gmap, sol, next_sta, curr_sta, next_sto, \
                       ctx->d_vgb, stage, fl, ctx->d_mid
    switch (v - kFirstGenVariant) {
      case 0:
        bsim4_gen_kernel<128, 1><<<grid, blk, 0, st>>>(XD_GEN_ARGS);
        break;
      case 1:
        bsim4_gen_kernel<128, 2><<<grid, blk, 0, st>>>(XD_GEN_ARGS);
        break;
      case 2:
        bsim4_gen_dc_kernel<128, 2><<<grid, blk, 0, st>>>(XD_GEN_DC_ARGS);
        bsim4_gen_cs_kernel<128, 2><<<grid, blk, 0, st>>>(XD_GEN_CS_ARGS);
        break;
      default:
        bsim4_gen_dc_kernel<128, 3><<<grid, blk, 0, st>>>(XD_GEN_DC_ARGS);
        bsim4_gen_cs_kernel<128, 3><<<grid, blk, 0, st>>>(XD_GEN_CS_ARGS);
        break;
    }
#undef XD_GEN_ARGS
#undef XD_GEN_DC_ARGS
#undef XD_GEN_CS_ARGS
    return;
  }
  if (kEvalVariants[v].persist) grid = std::max(1, std::min(grid, ctx->resident_blocks[v]));
  if (kEvalVariants[v].split) {
#define XD_DC_ARGS n, ctx->d_tab, ctx->n_rec, ctx->d_rec, ctx->d_nodes, sol, next_sto, curr_sto, ctx->d_vgb, fl, ctx->d_ext, \
                   ctx->d_mid
#define XD_CS_ARGS n, ctx->d_tab, ctx->n_rec, ctx->d_rec, ctx->d_nodes, sol, next_sta, curr_sta, next_sto, ctx->d_vgb, \
                   stage, fl, ctx->d_ext, ctx->d_mid
    switch (v) {
      case 12:
        bsim4_dc_kernel<128, 3, false, false><<<grid, blk, 0, st>>>(XD_DC_ARGS);
        bsim4_charge_stamp_kernel<128, 3, false, false><<<grid, blk, 0, st>>>(XD_CS_ARGS);
        break;
      case 13:
        bsim4_dc_kernel<128, 4, false, false><<<grid, blk, 0, st>>>(XD_DC_ARGS);
        bsim4_charge_stamp_kernel<128, 4, false, false><<<grid, blk, 0, st>>>(XD_CS_ARGS);
        break;
      case 14:
        bsim4_dc_kernel<128, 5, false, false><<<grid, blk, 0, st>>>(XD_DC_ARGS);
        bsim4_charge_stamp_kernel<128, 5, false, false><<<grid, blk, 0, st>>>(XD_CS_ARGS);
        break;
      case 15:
        bsim4_dc_kernel<128, 4, false, false><<<grid, blk, 0, st>>>(XD_DC_ARGS);
        bsim4_charge_stamp_kernel<128, 3, false, false><<<grid, blk, 0, st>>>(XD_CS_ARGS);
        break;
      default: {
        // The DC part under a 112-register budget in 96- or 64-thread blocks, the charge / stamp
        // part in 128 x 4. Each sub-partition's register file still holds 4 warps at that budget (16
        // per SM): the budget changes the schedule and the spills, not the occupancy.
        const int grid128 = (n + 127) / 128;
        bsim4_dc_kernel_regs<112><<<grid, blk, 0, st>>>(XD_DC_ARGS);
        bsim4_charge_stamp_kernel<128, 4, false, false><<<grid128, 128, 0, st>>>(XD_CS_ARGS);
        break;
      }
    }
#undef XD_DC_ARGS
#undef XD_CS_ARGS
    return;
  }
#define XD_EVAL_ARGS n, ctx->d_tab, ctx->n_rec, ctx->d_rec, ctx->d_nodes, sol, next_sta, curr_sta, next_sto, curr_sto, \
                     ctx->d_vgb, stage, fl, ctx->d_ext
  switch (v) {
    case 0: bsim4_eval_kernel<128, 1, false, false><<<grid, blk, 0, st>>>(XD_EVAL_ARGS); break;
    case 1: bsim4_eval_kernel<128, 2, false, false><<<grid, blk, 0, st>>>(XD_EVAL_ARGS); break;
    case 2: bsim4_eval_kernel<128, 3, false, false><<<grid, blk, 0, st>>>(XD_EVAL_ARGS); break;
    case 3: bsim4_eval_kernel<128, 4, false, false><<<grid, blk, 0, st>>>(XD_EVAL_ARGS); break;
    case 4: bsim4_eval_kernel<64, 4, false, false><<<grid, blk, 0, st>>>(XD_EVAL_ARGS); break;
    case 5: bsim4_eval_kernel<256, 2, false, false><<<grid, blk, 0, st>>>(XD_EVAL_ARGS); break;
    case 6: bsim4_eval_kernel<128, 2, true, false><<<grid, blk, 0, st>>>(XD_EVAL_ARGS); break;
    case 7: bsim4_eval_kernel<128, 3, true, false><<<grid, blk, 0, st>>>(XD_EVAL_ARGS); break;
    case 8: bsim4_eval_kernel<128, 2, true, true><<<grid, blk, 0, st>>>(XD_EVAL_ARGS); break;
    case 9: bsim4_eval_kernel<128, 3, true, true><<<grid, blk, 0, st>>>(XD_EVAL_ARGS); break;
    case 10: bsim4_eval_kernel<128, 3, false, false, true><<<grid, blk, 0, st>>>(XD_EVAL_ARGS); break;
    case 11: bsim4_eval_kernel<128, 3, true, false, true><<<grid, blk, 0, st>>>(XD_EVAL_ARGS); break;
    default: break;
  }
#undef XD_EVAL_ARGS
}

// Internal drain / source nodes per instance: BSIM4 where the sheet resistance and the squares are
// positive (record flags), BSIM3 and MOSFET1 where the series conductance is nonzero.
void internal_flags(int family, const xb4::RecordTable &rt, std::vector<unsigned char> &dint,
                    std::vector<unsigned char> &sint) {
  const size_t nr = (size_t)rt.n_records;
  for (size_t i = 0; i < rt.inst_rec.size(); ++i) {
    const size_t r = (size_t)rt.inst_rec[i];
    if (family == kFamilyBsim4) {
      dint[i] = rt.tab[(size_t)xb4::f_dExists * nr + r] != 0.0;
      sint[i] = rt.tab[(size_t)xb4::f_sExists * nr + r] != 0.0;
    } else if (family == kFamilyBsim3) {
      dint[i] = rt.tab[(size_t)xb3::f_drainConductance * nr + r] != 0.0;
      sint[i] = rt.tab[(size_t)xb3::f_sourceConductance * nr + r] != 0.0;
    } else {
      dint[i] = rt.tab[(size_t)xm1::f_drainConductance * nr + r] != 0.0;
      sint[i] = rt.tab[(size_t)xm1::f_sourceConductance * nr + r] != 0.0;
    }
  }
}

// General topology, per instance: which of the internal variables (D', S', G', GM, B', SB, DB, the
// NQS charge and the three initial-condition branch currents, registerLIDs order) it has
// (:3684-3769, 4996-5099).
constexpr int kGenInternal = XD_GEN_INTERNAL;
static_assert(kGenInternal == xb4::kGenNodes - 4, "the internal variables are the local nodes after D, G, S, B");
void gen_flags(const xb4::RecordTable &rt, std::vector<unsigned char> &flags) {
  const size_t nr = (size_t)rt.n_records, n = rt.inst_rec.size();
  flags.assign((size_t)kGenInternal * n, 0);
  auto f = [&](xb4::Field fld, size_t r) { return rt.tab[(size_t)fld * nr + r]; };
  for (size_t i = 0; i < n; ++i) {
    const size_t r = (size_t)rt.inst_rec[i];
    const int rg = (int)f(xb4::f_rgateMod, r);
    const bool rb = f(xb4::f_rbodyMod, r) != 0.0;
    unsigned char *fl = &flags[(size_t)kGenInternal * i];
    fl[0] = f(xb4::f_dExists, r) != 0.0;
    fl[1] = f(xb4::f_sExists, r) != 0.0;
    fl[2] = rg > 0;
    fl[3] = rg == 3;
    fl[4] = fl[5] = fl[6] = rb;
    fl[7] = f(xb4::f_trnqsMod, r) != 0.0;
    fl[8] = f(xb4::f_icVBSGiven, r) != 0.0;
    fl[9] = f(xb4::f_icVDSGiven, r) != 0.0;
    fl[10] = f(xb4::f_icVGSGiven, r) != 0.0;
  }
}
// A BSIM4 family needs the general topology when a record uses gate or body resistance, rdsMod 1,
// the NQS charge node or an instance initial condition.
bool family_needs_gen(const xb4::RecordTable &rt) {
  const size_t nr = (size_t)rt.n_records;
  auto f = [&](xb4::Field fld, size_t r) { return rt.tab[(size_t)fld * nr + r]; };
  for (size_t r = 0; r < nr; ++r)
    if (f(xb4::f_rgateMod, r) != 0.0 || f(xb4::f_rbodyMod, r) != 0.0 || f(xb4::f_rdsMod, r) != 0.0 ||
        f(xb4::f_trnqsMod, r) != 0.0 || f(xb4::f_icVBSGiven, r) != 0.0 || f(xb4::f_icVDSGiven, r) != 0.0 ||
        f(xb4::f_icVGSGiven, r) != 0.0)
      return true;
  return false;
}

// Times every launch shape on the circuit's own instances at a synthetic operating point (node
// voltages spread over 0..1.2 V, transient flags) in scratch buffers, and returns the fastest.
int autotune_eval(xd_ctx *ctx, int &best) {
  best = ctx->family == kFamilyMos1    ? kFirstMos1Variant
         : ctx->family == kFamilyBsim3 ? kFirstBsim3Variant
         : ctx->gen                    ? kFirstGenVariant
         : ctx->series                 ? kFirstSeriesVariant
                                       : (ctx->needs_full ? kFirstFullVariant : 0);
  const int n = ctx->n;
  if (n < 4096) return 0;
  // State and store blocks of the family's size (BSIM4 3 / 14 or, general topology, 6 / 14; BSIM3
  // 5 / 5; MOSFET1 8 / 5 slots).
  const size_t nsta = ctx->family == kFamilyMos1 ? xm1::kNumState
                      : ctx->family == kFamilyBsim3 ? xb3::kNumState
                      : ctx->gen ? (size_t)xb4::kGenState : (size_t)xb4::kNumState;
  const size_t nsto = ctx->family == kFamilyMos1 ? xm1::kNumStore
                      : ctx->family == kFamilyBsim3 ? xb3::kNumStore : xb4::kNumStore;
  double *sol = nullptr, *sta = nullptr, *sto = nullptr;
  cudaError_t ce;
  if ((ce = cudaMalloc(&sol, std::max(1, ctx->n_unknowns) * sizeof(double))) != cudaSuccess ||
      (ce = cudaMalloc(&sta, (size_t)2 * nsta * n * sizeof(double))) != cudaSuccess ||
      (ce = cudaMalloc(&sto, (size_t)2 * nsto * n * sizeof(double))) != cudaSuccess) {
    cudaFree(sol); cudaFree(sta); cudaFree(sto);
    return cuda_fail(ce, "autotune allocation");
  }
  std::vector<double> h(std::max(1, ctx->n_unknowns));
  for (size_t k = 0; k < h.size(); ++k) h[k] = 1.2 * (double)((k * 2654435761u) % 1000u) / 999.0;
  cudaMemcpy(sol, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemset(sta, 0, (size_t)2 * nsta * n * sizeof(double));
  cudaMemset(sto, 0, (size_t)2 * nsto * n * sizeof(double));
  xb4::LoadFlags fl{};
  fl.transient = 1; fl.newton_iter = 1; fl.voltlim = 1; fl.gmin = 1e-12;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best_ms = 1e30f;
  for (int v = 0; v < kNumEvalVariants; ++v) {
    if (!variant_fits(ctx, v)) continue;
    launch_eval(v, ctx, fl, sol, sta, sta + (size_t)nsta * n, sto, sto + (size_t)nsto * n,
                ctx->d_stage, 0);
    cudaEventRecord(e0, 0);
    for (int r = 0; r < 3; ++r)
      launch_eval(v, ctx, fl, sol, sta, sta + (size_t)nsta * n, sto, sto + (size_t)nsto * n,
                  ctx->d_stage, 0);
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (cudaGetLastError() == cudaSuccess && ms < best_ms) {
      best_ms = ms;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sol);
  cudaFree(sta);
  cudaFree(sto);
  // The tuning runs advanced the per-instance vgb memory; a fresh context starts from 0.
  cudaMemset(ctx->d_vgb, 0, (size_t)n * sizeof(double));
  ce = cudaDeviceSynchronize();
  if (ce != cudaSuccess) return cuda_fail(ce, "autotune");
  return 0;
}

xb4::LoadFlags to_flags(const xd_flags &f) {
  xb4::LoadFlags l;
  l.dcop = f.dcop;
  l.init_tran = f.init_tran;
  l.newton_iter = f.newton_iter;
  l.init_jct = f.init_jct;
  l.init_fix = f.init_fix;
  l.transient = f.transient;
  l.tranop = f.tranop;
  l.acop = f.acop;
  l.voltlim = f.voltlim;
  l.input_op = f.input_op;
  l.gmin = f.gmin;
  l.pdt = f.pdt;
  return l;
}

}  // namespace

// Error reporting for the library's other translation units (xd_last_error reads it).
int xd_internal_fail(int code, const std::string &msg) { return fail(code, msg); }

extern "C" {

const char *xd_last_error(void) { return g_err.c_str(); }

int xd_internal_nodes_gen(const xd_mosfet_family *fam, int *flags) {
  g_err.clear();
  if (!fam || !flags) return fail(-1, "null argument");
  if (fam->n_inst < 0 || fam->n_models <= 0) return fail(-1, "bad instance or model count");
  if (fam->level != 14 && fam->level != 54) return fail(-1, "the general topology is BSIM4's (level 14 / 54)");
  const int n = fam->n_inst;
  std::vector<xb4::ModelSpec> models(fam->n_models);
  size_t off = 0;
  for (int m = 0; m < fam->n_models; ++m) {
    models[m].pmos = fam->model_is_pmos[m] != 0;
    for (int k = 0; k < fam->model_nparams[m]; ++k, ++off)
      models[m].params.push_back({fam->model_param_names[off], fam->model_param_values[off]});
  }
  std::vector<std::string> ipn;
  for (int k = 0; k < fam->n_inst_params; ++k) ipn.push_back(fam->inst_param_names[k]);
  xb4::SetupOptions opts;
  opts.temp_c = fam->temp_c;
  opts.tnom_c = fam->tnom_c;
  xb4::RecordTable rt;
  const std::string e = xb4::build_records(models, n, fam->inst_model, ipn, fam->inst_param_values, opts, rt);
  if (!e.empty()) return fail(-2, e);
  std::vector<unsigned char> gf;
  gen_flags(rt, gf);
  for (size_t k = 0; k < gf.size(); ++k) flags[k] = gf[k];
  return family_needs_gen(rt) ? 1 : 0;
}

int xd_general_stamp(int *rows, int *cols) {
  if (!rows || !cols) return fail(-1, "null argument");
  for (int k = 0; k < xb4::kGenSlots; ++k) {
    rows[k] = xb4::kGenStamp[k][0];
    cols[k] = xb4::kGenStamp[k][1];
  }
  return xb4::kGenSlots;
}

int xd_internal_nodes(const xd_mosfet_family *fam, int *flags) {
  g_err.clear();
  if (!fam || !flags) return fail(-1, "null argument");
  if (fam->n_inst < 0 || fam->n_models <= 0) return fail(-1, "bad instance or model count");
  const int n = fam->n_inst;
  for (int k = 0; k < 2 * n; ++k) flags[k] = 0;
  const bool b4 = fam->level == 14 || fam->level == 54, b3 = fam->level == 9 || fam->level == 49;
  if (!b4 && !b3 && fam->level != 1) return fail(-1, "unsupported MOSFET level");
  std::vector<xb4::ModelSpec> models(fam->n_models);
  size_t off = 0;
  for (int m = 0; m < fam->n_models; ++m) {
    models[m].pmos = fam->model_is_pmos[m] != 0;
    for (int k = 0; k < fam->model_nparams[m]; ++k, ++off)
      models[m].params.push_back({fam->model_param_names[off], fam->model_param_values[off]});
  }
  std::vector<std::string> ipn;
  for (int k = 0; k < fam->n_inst_params; ++k) ipn.push_back(fam->inst_param_names[k]);
  xb4::SetupOptions opts;
  opts.temp_c = fam->temp_c;
  opts.tnom_c = fam->tnom_c;
  xb4::RecordTable rt;
  const std::string e =
      b4   ? xb4::build_records(models, n, fam->inst_model, ipn, fam->inst_param_values, opts, rt)
      : b3 ? xb3::build_records(models, n, fam->inst_model, ipn, fam->inst_param_values, opts, rt)
           : xm1::build_records(models, n, fam->inst_model, ipn, fam->inst_param_values, opts, rt);
  if (!e.empty()) return fail(-2, e);
  std::vector<unsigned char> dint(n, 0), sint(n, 0);
  internal_flags(b4 ? kFamilyBsim4 : (b3 ? kFamilyBsim3 : kFamilyMos1), rt, dint, sint);
  for (int i = 0; i < n; ++i) {
    flags[2 * i] = dint[i];
    flags[2 * i + 1] = sint[i];
  }
  return 0;
}

int xd_num_instances(const xd_ctx *ctx) { return ctx ? ctx->n : -1; }
int xd_num_state_slots(const xd_ctx *ctx) {
  if (!ctx) return -1;
  return ctx->family == kFamilyMos1 ? (int)xm1::kNumState
         : ctx->family == kFamilyBsim3 ? (int)xb3::kNumState
         : ctx->gen                    ? (int)xb4::kGenState
                                       : (int)xb4::kNumState;
}
int xd_num_store_slots(const xd_ctx *ctx) {
  if (!ctx) return -1;
  return ctx->family == kFamilyMos1 ? (int)xm1::kNumStore
         : ctx->family == kFamilyBsim3 ? (int)xb3::kNumStore
                                       : (int)xb4::kNumStore;
}

int xd_destroy(xd_ctx *ctx) {
  if (!ctx) return 0;
  DeviceGuard g(ctx->device);
  cudaFree(ctx->d_tab);
  cudaFree(ctx->d_rec);
  cudaFree(ctx->d_nodes);
  cudaFree(ctx->d_vgb);
  cudaFree(ctx->d_stage);
  cudaFree(ctx->d_ext);
  cudaFree(ctx->d_mid);
  cudaFree(ctx->d_gmap);
  free_map(ctx->vmap);
  free_map(ctx->mmap);
  delete ctx;
  return 0;
}

int xd_create(const xd_mosfet_family *fam, const xd_csr *pat, int cuda_device, xd_ctx **out) {
  g_err.clear();
  if (!fam || !pat || !out) return fail(-1, "null argument");
  *out = nullptr;
  int family;
  if (fam->level == 14 || fam->level == 54)
    family = kFamilyBsim4;
  else if (fam->level == 9 || fam->level == 49)
    family = kFamilyBsim3;
  else if (fam->level == 1)
    family = kFamilyMos1;
  else
    return fail(-2, "MOSFET level " + std::to_string(fam->level) +
                        " is not implemented (levels 1, 9, 49, 14, 54 are)");
  if (fam->n_inst < 0 || fam->n_models <= 0) return fail(-1, "bad instance or model count");
  if ((long long)fam->n_inst * xb4::kGenStage >= (1LL << 31)) return fail(-1, "too many instances");
  if (pat->n_rows < 0 || !pat->rowptr || (pat->rowptr[pat->n_rows] > 0 && !pat->colind))
    return fail(-1, "bad CSR pattern");
  const int n = fam->n_inst;
  const int nu = pat->n_rows;
  // Model cards and per-record constants.
  std::vector<xb4::ModelSpec> models(fam->n_models);
  size_t off = 0;
  for (int m = 0; m < fam->n_models; ++m) {
    models[m].pmos = fam->model_is_pmos[m] != 0;
    for (int k = 0; k < fam->model_nparams[m]; ++k, ++off)
      models[m].params.push_back({fam->model_param_names[off], fam->model_param_values[off]});
  }
  std::vector<std::string> ipn;
  for (int k = 0; k < fam->n_inst_params; ++k) ipn.push_back(fam->inst_param_names[k]);
  xb4::SetupOptions opts;
  opts.temp_c = fam->temp_c;
  opts.tnom_c = fam->tnom_c;
  xb4::RecordTable rt;
  std::string e =
      family == kFamilyMos1    ? xm1::build_records(models, n, fam->inst_model, ipn, fam->inst_param_values, opts, rt)
      : family == kFamilyBsim3 ? xb3::build_records(models, n, fam->inst_model, ipn, fam->inst_param_values, opts, rt)
                               : xb4::build_records(models, n, fam->inst_model, ipn, fam->inst_param_values, opts, rt);
  if (!e.empty()) return fail(-2, e);
  // General topology (BSIM4): the caller passed the 11 internal variables per instance, or the
  // cards need them.
  const bool gen = family == kFamilyBsim4 && (fam->inst_internal_gen != nullptr || family_needs_gen(rt));
  if (gen && !fam->inst_internal_gen)
    return fail(-1, "the instances use gate or body resistance, rdsMod 1, the NQS charge node or initial conditions: "
                    "pass their internal "
                    "unknowns in inst_internal_gen (xd_internal_nodes_gen lists which instances have which)");
  if (gen && fam->inst_internal)
    return fail(-1, "pass the internal unknowns in inst_internal_gen only (it includes the drain and source ones)");
  if (fam->inst_internal_gen && family != kFamilyBsim4)
    return fail(-1, "inst_internal_gen is for BSIM4 families");
  // Internal drain / source nodes (series resistance): which instances have them.
  std::vector<unsigned char> dint(n, 0), sint(n, 0);
  bool series = false;
  internal_flags(family, rt, dint, sint);
  if (!gen)
    for (int i = 0; i < n; ++i) series = series || dint[i] || sint[i];
  if (series && !fam->inst_internal)
    return fail(-1, "instances have internal drain/source nodes (series resistance): pass their unknowns in "
                    "inst_internal (xd_internal_nodes lists which instances have them)");
  // Node indices and gather maps (registerLIDs / registerJacLIDs equivalent). With internal nodes
  // the intrinsic device sits on (D', G, S', B) and ext keeps the external drain and source.
  std::vector<int4> nodes(n);
  std::vector<int2> ext(series ? n : 0);
  for (int i = 0; i < n; ++i) {
    int v[4];
    for (int k = 0; k < 4; ++k) {
      v[k] = fam->inst_nodes[4 * (size_t)i + k];
      if (v[k] >= nu) return fail(-1, "instance node index beyond the pattern's unknowns");
      if (v[k] < 0) v[k] = -1;
    }
    if (fam->inst_internal) {
      for (int k = 0; k < 2; ++k) {
        const int u = fam->inst_internal[2 * (size_t)i + k];
        const bool has = k == 0 ? dint[i] : sint[i];
        if (has && (u < 0 || u >= nu))
          return fail(-1, "instance " + std::to_string(i) + " needs an internal " + (k == 0 ? "drain" : "source") +
                              " node inside the pattern's unknowns");
        if (!has && u >= 0)
          return fail(-1, "instance " + std::to_string(i) + " has no internal " + (k == 0 ? "drain" : "source") +
                              " node (RSH and NRD/NRS not both positive)");
      }
    }
    if (series) {
      ext[i] = make_int2(v[0], v[2]);
      if (dint[i]) v[0] = fam->inst_internal[2 * (size_t)i];
      if (sint[i]) v[2] = fam->inst_internal[2 * (size_t)i + 1];
    }
    nodes[i] = make_int4(v[0], v[1], v[2], v[3]);
  }
  auto csr_pos = [&](int r, int c, int &p) -> bool {
    p = -1;
    if (r < 0 || c < 0) return true;
    const int *b = pat->colind + pat->rowptr[r], *en = pat->colind + pat->rowptr[r + 1];
    const int *q = std::lower_bound(b, en, c);
    if (q == en || *q != c) return false;
    p = (int)(q - pat->colind);
    return true;
  };
  const int vrows = gen ? xb4::kGenVecRows : series ? xb4::kSerVecRows : 4;
  std::vector<int> vt, vs, mt, ms, gmap;
  if (gen) {
    // Local node -> unknown (collapsed nodes onto their representative, -1 for ground and for
    // absent branch currents), then the gather maps: per instance, vector rows in node order and
    // matrix entries in stamp-slot order.
    std::vector<unsigned char> gfl;
    gen_flags(rt, gfl);
    gmap.assign((size_t)xb4::kGenNodes * n, -1);
    vt.reserve((size_t)xb4::kGenVecRows * n);
    vs.reserve((size_t)xb4::kGenVecRows * n);
    mt.reserve((size_t)xb4::kGenSlots * n);
    ms.reserve((size_t)xb4::kGenSlots * n);
    static const char *const kNames[kGenInternal] = {"drain'", "source'", "gate'", "gate-mid", "body'",
                                                     "source-body", "drain-body", "charge", "IBS", "IDS", "IGS"};
    for (int i = 0; i < n; ++i) {
      int nd[xb4::kGenNodes];
      for (int k = 0; k < 4; ++k) {
        nd[k] = fam->inst_nodes[4 * (size_t)i + k];
        if (nd[k] >= nu) return fail(-1, "instance node index beyond the pattern's unknowns");
        if (nd[k] < 0) nd[k] = -1;
      }
      // Representatives of the collapsible nodes: D' -> D, S' -> S, G' / GM -> G, B' / SB / DB -> B.
      const int rep[kGenInternal] = {nd[0], nd[2], nd[1], nd[1], nd[3], nd[3], nd[3], -1, -1, -1, -1};
      for (int k = 0; k < kGenInternal; ++k) {
        const int u = fam->inst_internal_gen[(size_t)kGenInternal * i + k];
        const bool has = gfl[(size_t)kGenInternal * i + k] != 0;
        if (has && (u < 0 || u >= nu))
          return fail(-1, "instance " + std::to_string(i) + " needs an internal " + kNames[k] +
                              " unknown inside the pattern's unknowns");
        if (!has && u >= 0)
          return fail(-1, "instance " + std::to_string(i) + " has no internal " + kNames[k] + " variable");
        nd[4 + k] = has ? u : rep[k];
      }
      for (int k = 0; k < xb4::kGenNodes; ++k) {
        gmap[(size_t)k * n + i] = nd[k];
        vt.push_back(nd[k]);
        vs.push_back(k * n + i);
      }
      for (int k = 0; k < xb4::kGenSlots; ++k) {
        int p;
        if (!csr_pos(nd[xb4::kGenStamp[k][0]], nd[xb4::kGenStamp[k][1]], p))
          return fail(-1, "CSR pattern lacks an entry the instance's general stamp touches");
        mt.push_back(p);
        ms.push_back(k * n + i);
      }
      nodes[i] = make_int4(nd[0], nd[1], nd[2], nd[3]);
    }
  }
  vt.reserve((size_t)vrows * n);
  vs.reserve((size_t)vrows * n);
  mt.reserve((size_t)(series ? xb4::kSerMat : 16) * n);
  ms.reserve((size_t)(series ? xb4::kSerMat : 16) * n);
  // Each instance's vector rows in the order the family's loadDAEVectors adds them (BSIM4: D', G',
  // B', S' then the external D, S, N_DEV_MOSFET_B4.C:16316-16370; BSIM3: D, S, B, D', S' with the
  // gate's charge first, N_DEV_MOSFET_B3.C:9357-9366, 9554-9557; MOSFET1: D, G, S, B, D', S',
  // N_DEV_MOSFET1.C:4222-4236): where two rows of an instance are the same unknown (bulk tied to
  // source), the sum then adds them in the reference's order.
  static const int kVecOrder[3][6] = {{0, 1, 3, 2, 4, 5}, {4, 5, 1, 3, 0, 2}, {4, 1, 5, 3, 0, 2}};
  const int *vorder = kVecOrder[family == kFamilyBsim4 ? 0 : family == kFamilyBsim3 ? 1 : 2];
  for (int i = 0; !gen && i < n; ++i) {
    const int nd[4] = {nodes[i].x, nodes[i].y, nodes[i].z, nodes[i].w};
    for (int k = 0; k < 6; ++k) {
      const int r = vorder[k];
      if (r >= 4 && !series) continue;
      vt.push_back(r < 4 ? nd[r] : (r == 4 ? ext[i].x : ext[i].y));
      vs.push_back(r * n + i);
    }
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) {
        int p;
        if (!csr_pos(nd[r], nd[c], p)) return fail(-1, "CSR pattern lacks an entry the instance stamps");
        mt.push_back(p);
        ms.push_back((r * 4 + c) * n + i);
      }
    if (series) {
      // (D', D), (D, D'), (D, D), (S', S), (S, S'), (S, S): the order of LoadOut::jfx.
      const int rc[6][2] = {{nd[0], ext[i].x}, {ext[i].x, nd[0]}, {ext[i].x, ext[i].x},
                            {nd[2], ext[i].y}, {ext[i].y, nd[2]}, {ext[i].y, ext[i].y}};
      for (int k = 0; k < 6; ++k) {
        int p;
        if (!csr_pos(rc[k][0], rc[k][1], p))
          return fail(-1, "CSR pattern lacks a series-resistance entry the instance stamps");
        mt.push_back(p);
        ms.push_back((xb4::kNumMat + k) * n + i);
      }
    }
  }
  int rc = cudaSetDevice(cuda_device);
  if (rc != cudaSuccess) return cuda_fail((cudaError_t)rc, "cudaSetDevice");
  xd_ctx *ctx = new xd_ctx();
  ctx->family = family;
  ctx->device = cuda_device;
  ctx->n = n;
  ctx->n_unknowns = nu;
  ctx->nnz = pat->rowptr[nu];
  ctx->n_rec = rt.n_records;
  ctx->series = series;
  ctx->gen = gen;
  if (series) {
    ctx->vec_rows = xb4::kSerVecRows;
    ctx->mat_slots = xb4::kSerMat;
    ctx->stage_slots = xb4::kSerStage;
  }
  if (gen) {
    ctx->vec_rows = xb4::kGenVecRows;
    ctx->mat_slots = xb4::kGenSlots;
    ctx->stage_slots = xb4::kGenStage;
    ctx->needs_full = true;
  }
  if (family == kFamilyBsim4)
    for (int r = 0; r < rt.n_records; ++r)
      if (rt.tab[(size_t)xb4::f_igcMod * rt.n_records + r] != 0.0 ||
          rt.tab[(size_t)xb4::f_igbMod * rt.n_records + r] != 0.0 ||
          rt.tab[(size_t)xb4::f_capMod * rt.n_records + r] != 2.0)
        ctx->needs_full = true;
  auto cleanup = [&](int code) {
    xd_destroy(ctx);
    return code;
  };
  cudaError_t ce;
  if ((ce = cudaMalloc(&ctx->d_tab, std::max<size_t>(1, rt.tab.size()) * sizeof(double))) != cudaSuccess ||
      (ce = cudaMemcpy(ctx->d_tab, rt.tab.data(), rt.tab.size() * sizeof(double), cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (ce = cudaMalloc(&ctx->d_rec, std::max(1, n) * sizeof(int))) != cudaSuccess ||
      (ce = cudaMemcpy(ctx->d_rec, rt.inst_rec.data(), n * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (ce = cudaMalloc(&ctx->d_nodes, std::max(1, n) * sizeof(int4))) != cudaSuccess ||
      (ce = cudaMemcpy(ctx->d_nodes, nodes.data(), n * sizeof(int4), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (ce = cudaMalloc(&ctx->d_vgb, std::max(1, n) * sizeof(double))) != cudaSuccess ||
      (ce = cudaMemset(ctx->d_vgb, 0, std::max(1, n) * sizeof(double))) != cudaSuccess ||
      (ce = cudaMalloc(&ctx->d_stage, std::max<size_t>(1, (size_t)ctx->stage_slots * n) * sizeof(double))) !=
          cudaSuccess ||
      (ce = cudaMemset(ctx->d_stage, 0, std::max<size_t>(1, (size_t)ctx->stage_slots * n) * sizeof(double))) !=
          cudaSuccess)
    return cleanup(cuda_fail(ce, "xd_create allocation"));
  if (series && ((ce = cudaMalloc(&ctx->d_ext, std::max(1, n) * sizeof(int2))) != cudaSuccess ||
                 (ce = cudaMemcpy(ctx->d_ext, ext.data(), n * sizeof(int2), cudaMemcpyHostToDevice)) != cudaSuccess))
    return cleanup(cuda_fail(ce, "xd_create allocation"));
  if (gen && ((ce = cudaMalloc(&ctx->d_gmap, std::max<size_t>(1, gmap.size()) * sizeof(int))) != cudaSuccess ||
              (ce = cudaMemcpy(ctx->d_gmap, gmap.data(), gmap.size() * sizeof(int), cudaMemcpyHostToDevice)) !=
                  cudaSuccess))
    return cleanup(cuda_fail(ce, "xd_create allocation"));
  // Hand-off state of the split evaluation: the common card's, or the general topology's.
  if (family == kFamilyBsim4 && !series && !gen && !ctx->needs_full && n > 0 &&
      (ce = cudaMalloc(&ctx->d_mid, (size_t)xb4::kNumMid * n * sizeof(double))) != cudaSuccess)
    return cleanup(cuda_fail(ce, "xd_create allocation"));
  if (gen && n > 0 && (ce = cudaMalloc(&ctx->d_mid, (size_t)xb4::kNumMidGen * n * sizeof(double))) != cudaSuccess)
    return cleanup(cuda_fail(ce, "xd_create allocation"));
  if ((rc = build_map(vt, vs, nu, ctx->vmap)) != 0) return cleanup(rc);
  if ((rc = build_map(mt, ms, ctx->nnz, ctx->mmap)) != 0) return cleanup(rc);
  if ((rc = size_persistent_grids(ctx)) != 0) return cleanup(rc);
  if ((rc = autotune_eval(ctx, ctx->eval_variant)) != 0) return cleanup(rc);
  *out = ctx;
  return 0;
}

int xd_update_state(xd_ctx *ctx, const xd_flags *flags, const double *d_sol, double *d_next_sta, double *d_curr_sta,
                    double *d_next_sto, const double *d_curr_sto, void *stream) {
  if (!ctx || !flags) return fail(-1, "null argument");
  if (ctx->n == 0) return 0;
  if (!d_sol || !d_next_sta || !d_next_sto || !d_curr_sto || !d_curr_sta) return fail(-1, "null device buffer");
  if (flags->input_op) return fail(-2, "inputOP loads are not supported");
  DeviceGuard g(ctx->device);
  cudaStream_t st = (cudaStream_t)stream;
  launch_eval(ctx->eval_variant, ctx, to_flags(*flags), d_sol, d_next_sta, d_curr_sta, d_next_sto, d_curr_sto,
              ctx->d_stage, st);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "bsim4_eval_kernel launch");
  ctx->stage_static = false;
  return 0;
}

// The calls that read the context's staged stamps (d_stage) refuse after a static-scratch load.
static int check_stage_current(const xd_ctx *ctx) {
  if (ctx->stage_static)
    return fail(-1, "the last evaluation of this context was xd_load_static_scratch, whose staged stamps are in "
                    "the library's static array, not in the context; call xd_update_state first");
  return 0;
}

static int load_vectors_impl(xd_ctx *ctx, double *f, double *q, double *fx, double *qx, bool abs_mode, cudaStream_t st,
                             int assign = 0) {
  const size_t n = (size_t)ctx->n, r = (size_t)ctx->vec_rows;
  if (abs_mode) {
    OutSet<4, true> os{{f, q, fx, qx}, {0, r * n, 2 * r * n, 3 * r * n}};
    return run_gather(ctx->vmap, ctx->d_stage, os, st);
  }
  OutSet<4, false> os{{f, q, fx, qx}, {0, r * n, 2 * r * n, 3 * r * n}, assign};
  return run_gather(ctx->vmap, ctx->d_stage, os, st);
}

static int load_matrices_impl(xd_ctx *ctx, double *jf, double *jq, bool abs_mode, cudaStream_t st, int assign = 0) {
  const size_t n = (size_t)ctx->n, b = 4 * (size_t)ctx->vec_rows * n, m = (size_t)ctx->mat_slots * n;
  if (abs_mode) {
    OutSet<2, true> os{{jf, jq}, {b, b + m}};
    return run_gather(ctx->mmap, ctx->d_stage, os, st);
  }
  OutSet<2, false> os{{jf, jq}, {b, b + m}, assign};
  return run_gather(ctx->mmap, ctx->d_stage, os, st);
}

int xd_load_vectors(xd_ctx *ctx, double *d_f, double *d_q, double *d_dfdxdvp, double *d_dqdxdvp, void *stream) {
  if (!ctx) return fail(-1, "null context");
  if (ctx->n == 0) return 0;
  if (int rc = check_stage_current(ctx)) return rc;
  DeviceGuard g(ctx->device);
  return load_vectors_impl(ctx, d_f, d_q, d_dfdxdvp, d_dqdxdvp, false, (cudaStream_t)stream);
}

int xd_load_matrices(xd_ctx *ctx, double *d_dfdx_vals, double *d_dqdx_vals, void *stream) {
  if (!ctx) return fail(-1, "null context");
  if (ctx->n == 0) return 0;
  if (int rc = check_stage_current(ctx)) return rc;
  DeviceGuard g(ctx->device);
  return load_matrices_impl(ctx, d_dfdx_vals, d_dqdx_vals, false, (cudaStream_t)stream);
}

int xd_load(xd_ctx *ctx, const xd_flags *flags, const double *d_sol, double *d_next_sta, double *d_curr_sta,
            double *d_next_sto, const double *d_curr_sto, double *d_f, double *d_q, double *d_dfdxdvp,
            double *d_dqdxdvp, double *d_dfdx_vals, double *d_dqdx_vals, void *stream) {
  int rc = xd_update_state(ctx, flags, d_sol, d_next_sta, d_curr_sta, d_next_sto, d_curr_sto, stream);
  if (rc) return rc;
  if ((rc = xd_load_vectors(ctx, d_f, d_q, d_dfdxdvp, d_dqdxdvp, stream))) return rc;
  return xd_load_matrices(ctx, d_dfdx_vals, d_dqdx_vals, stream);
}

int xd_load_assign(xd_ctx *ctx, const xd_flags *flags, const double *d_sol, double *d_next_sta, double *d_curr_sta,
                   double *d_next_sto, const double *d_curr_sto, double *d_f, double *d_q, double *d_dfdxdvp,
                   double *d_dqdxdvp, double *d_dfdx_vals, double *d_dqdx_vals, void *stream) {
  int rc = xd_update_state(ctx, flags, d_sol, d_next_sta, d_curr_sta, d_next_sto, d_curr_sto, stream);
  if (rc) return rc;
  if (ctx->n == 0) return 0;
  DeviceGuard g(ctx->device);
  if ((rc = load_vectors_impl(ctx, d_f, d_q, d_dfdxdvp, d_dqdxdvp, false, (cudaStream_t)stream, 1))) return rc;
  return load_matrices_impl(ctx, d_dfdx_vals, d_dqdx_vals, false, (cudaStream_t)stream, 1);
}

int xd_load_vectors_staged(xd_ctx *ctx, const double *d_stage16, double *d_f, double *d_q, double *d_dfdxdvp,
                           double *d_dqdxdvp, int assign, void *stream) {
  if (!ctx) return fail(-1, "null context");
  if (ctx->n == 0) return 0;
  if (!d_stage16) return fail(-1, "null staged array");
  if (ctx->series || ctx->gen)
    return fail(-1, "staged vectors take the 4-terminal layout; this family has internal nodes");
  DeviceGuard g(ctx->device);
  const size_t n = (size_t)ctx->n;
  OutSet<4, false> os{{d_f, d_q, d_dfdxdvp, d_dqdxdvp}, {0, 4 * n, 8 * n, 12 * n}, assign ? 1 : 0};
  return run_gather(ctx->vmap, d_stage16, os, (cudaStream_t)stream);
}

int xd_load_abs(xd_ctx *ctx, double *d_f, double *d_q, double *d_dfdxdvp, double *d_dqdxdvp, double *d_dfdx_vals,
                double *d_dqdx_vals, void *stream) {
  if (!ctx) return fail(-1, "null context");
  if (ctx->n == 0) return 0;
  if (int rc = check_stage_current(ctx)) return rc;
  DeviceGuard g(ctx->device);
  int rc = load_vectors_impl(ctx, d_f, d_q, d_dfdxdvp, d_dqdxdvp, true, (cudaStream_t)stream);
  if (rc) return rc;
  return load_matrices_impl(ctx, d_dfdx_vals, d_dqdx_vals, true, (cudaStream_t)stream);
}

int xd_launches_per_load(const xd_ctx *ctx) {
  if (!ctx) return -1;
  if (ctx->n == 0) return 0;
  const int eval = (ctx->family == kFamilyBsim4 && kEvalVariants[ctx->eval_variant].split) ? 2 : 1;
  return eval + (ctx->vmap.n_short > 0) + 2 * (ctx->vmap.n_long > 0) + (ctx->mmap.n_short > 0) +
         2 * (ctx->mmap.n_long > 0);
}

int xd_eval_launch_shape(const xd_ctx *ctx, int *block, int *min_blocks) {
  if (!ctx || !block || !min_blocks) return fail(-1, "null argument");
  *block = kEvalVariants[ctx->eval_variant].block;
  *min_blocks = kEvalVariants[ctx->eval_variant].min_blocks;
  return 0;
}

int xd_num_eval_variants(void) { return kNumEvalVariants; }

int xd_eval_variant_info(int v, int *block, int *min_blocks) {
  if (v < 0 || v >= kNumEvalVariants || !block || !min_blocks) return fail(-1, "bad variant query");
  *block = kEvalVariants[v].block;
  *min_blocks = kEvalVariants[v].min_blocks;
  return 0;
}

int xd_eval_variant_persistent(int v) {
  if (v < 0 || v >= kNumEvalVariants) return fail(-1, "bad variant query");
  return kEvalVariants[v].persist ? 1 : 0;
}

int xd_eval_variant_split(int v) {
  if (v < 0 || v >= kNumEvalVariants) return fail(-1, "bad variant query");
  return kEvalVariants[v].split ? 1 : 0;
}

int xd_eval_variant_general(int v) {
  if (v < 0 || v >= kNumEvalVariants) return fail(-1, "bad variant query");
  return kEvalVariants[v].gen ? 1 : 0;
}

int xd_get_eval_variant(const xd_ctx *ctx) { return ctx ? ctx->eval_variant : -1; }

int xd_set_eval_variant(xd_ctx *ctx, int v) {
  if (!ctx || v < 0 || v >= kNumEvalVariants) return fail(-1, "bad evaluation variant");
  if (!variant_fits(ctx, v))
    return fail(-1, "this evaluation variant does not fit the family: it is compiled for capMod 2 without gate "
                    "tunnelling, or for another staging layout (internal drain / source nodes)");
  ctx->eval_variant = v;
  return 0;
}

int xd_probe_fp64_fma(double *d_out, int blocks, int iters, void *stream) {
  if (!d_out || blocks <= 0 || iters <= 0) return fail(-1, "bad probe arguments");
  fma_probe_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(d_out, iters);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "fma_probe_kernel launch");
  return 0;
}

int xd_num_stage_slots(const xd_ctx *ctx) { return ctx ? ctx->stage_slots : -1; }

int xd_copy_stamps(xd_ctx *ctx, double *h_out, void *stream) {
  if (!ctx || !h_out) return fail(-1, "null argument");
  if (int rc = check_stage_current(ctx)) return rc;
  DeviceGuard g(ctx->device);
  cudaStream_t st = (cudaStream_t)stream;
  XD_CUDA(cudaMemcpyAsync(h_out, ctx->d_stage, (size_t)ctx->stage_slots * ctx->n * sizeof(double),
                          cudaMemcpyDeviceToHost, st));
  XD_CUDA(cudaStreamSynchronize(st));
  return 0;
}


}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Allocation-free load. Scratch for the staged stamps and the chunk partial sums lives in a
// file-scope device array instead of context buffers, so xd_load_static_scratch itself never
// allocates. Capacity: XD_STATIC_MAX_INSTANCES instances (48 staged doubles each) plus
// 4 * XD_STATIC_MAX_INSTANCES chunk partials — 52 * 16384 doubles = 6.8 MB, held by every GPU
// that loads the library until the process exits.
namespace {

constexpr size_t kStaticStage = (size_t)XD_STATIC_MAX_INSTANCES * xb4::kNumStage;
constexpr size_t kStaticPartial = (size_t)4 * XD_STATIC_MAX_INSTANCES;
static __device__ __align__(256) double g_static_scratch[kStaticStage + kStaticPartial];

// Device address of g_static_scratch on the current device. In host code the symbol names a
// host-side stand-in, never a device address, so kernels only ever get the address
// cudaGetSymbolAddress returns. Resolved on every call (it allocates nothing and costs little
// next to the evaluation): an address kept from an earlier call would dangle once the device's
// primary context had been reset and created again.
int static_scratch_on(int dev, double **out) {
  (void)dev;
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_static_scratch)");
  *out = static_cast<double *>(p);
  return 0;
}

template <int NOUT>
int run_gather_static(const GatherMap &m, const double *stage, double *partial, const OutSet<NOUT, false> &os,
                      cudaStream_t st) {
  if (m.n_short > 0) {
    const int blk = 256;
    gather_short_kernel<NOUT, false><<<(m.n_short + blk - 1) / blk, blk, 0, st>>>(m.n_short, m.d_short_dst,
                                                                                m.d_short_ptr, m.d_src, stage, os);
  }
  if (m.n_long > 0) {
    gather_chunk_kernel<NOUT, false><<<m.n_chunks, kChunkBlock, 0, st>>>(m.d_chunk_begin, m.d_src, stage, partial,
                                                                         m.n_chunks, os);
    gather_combine_kernel<NOUT, false><<<m.n_long, kCombineBlock, 0, st>>>(
        m.n_long, m.d_long_dst, m.d_long_chunk, partial, m.n_chunks, os);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "gather launch");
  return 0;
}

}  // namespace

extern "C" {

int xd_load_static_scratch(xd_ctx *ctx, const xd_flags *flags, const double *d_sol, double *d_next_sta,
                           double *d_curr_sta, double *d_next_sto, const double *d_curr_sto, double *d_f, double *d_q,
                           double *d_dfdxdvp, double *d_dqdxdvp, double *d_dfdx_vals, double *d_dqdx_vals,
                           void *stream) {
  if (!ctx || !flags) return fail(-1, "null argument");
  if (ctx->series || ctx->gen)
    return fail(-1, "xd_load_static_scratch: the static scratch holds the 4-terminal layout; this family has "
                    "internal nodes");
  if (ctx->n > XD_STATIC_MAX_INSTANCES)
    return fail(-1, "xd_load_static_scratch: " + std::to_string(ctx->n) + " instances exceed the static scratch "
                    "capacity of " + std::to_string(XD_STATIC_MAX_INSTANCES) + "; use xd_load");
  if (4 * (size_t)ctx->vmap.n_chunks > kStaticPartial || 2 * (size_t)ctx->mmap.n_chunks > kStaticPartial)
    return fail(-1, "xd_load_static_scratch: gather partials exceed the static scratch capacity; use xd_load");
  if (ctx->n == 0) return 0;
  if (!d_sol || !d_next_sta || !d_next_sto || !d_curr_sto || !d_curr_sta) return fail(-1, "null device buffer");
  if (flags->input_op) return fail(-2, "inputOP loads are not supported");
  DeviceGuard g(ctx->device);
  double *scratch = nullptr;
  int rc = static_scratch_on(ctx->device, &scratch);
  if (rc) return rc;
  double *stage = scratch;
  double *partial = scratch + kStaticStage;
  cudaStream_t st = (cudaStream_t)stream;
  // Every staged slot of every instance is written by the evaluation before the gathers read it,
  // and every chunk partial is written before it is combined, so nothing needs clearing.
  launch_eval(ctx->eval_variant, ctx, to_flags(*flags), d_sol, d_next_sta, d_curr_sta, d_next_sto, d_curr_sto, stage,
              st);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "bsim4_eval_kernel launch");
  const size_t n = (size_t)ctx->n;
  OutSet<4, false> vs{{d_f, d_q, d_dfdxdvp, d_dqdxdvp}, {0, 4 * n, 8 * n, 12 * n}};
  if ((rc = run_gather_static(ctx->vmap, stage, partial, vs, st))) return rc;
  OutSet<2, false> ms{{d_dfdx_vals, d_dqdx_vals}, {16 * n, 32 * n}};
  if ((rc = run_gather_static(ctx->mmap, stage, partial, ms, st))) return rc;
  ctx->stage_static = true;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Fused load and combine. One Newton iterate's device load and the time-integration combine
// without the family's dF/dx and dQ/dx in between: the evaluation kernel stages the instances'
// stamps as usual, the few entries with more than kLongThreshold contributions (supply-rail
// couplings) are summed by the chunked gathers into the family's buffers, then
//   * fused_entry_kernel, a thread per CSR entry, forms the family's dF/dx and dQ/dx sum straight
//     from the staged stamps (same sources, same order as the gather kernels) and the Newton matrix
//     entry from it with the linear devices' terms;
//   * the vector gather forms the family's F, Q and limiter-vector sums (a thread per row), and
//     fused_row_kernel, a warp per row, the residual from them, with the linear devices' terms
//     summed in tia_combine_kernel's order (a long row's from its chunk sums, tia_long.h), and the
//     diagonal entry again where a gmin shunt is on.
// The family's dF/dx and dQ/dx are never written to memory (except for the long entries) or read
// back; the results are bit-identical to xd_load_assign followed by xd_tia_combine. (The row
// kernel summing the row's vector sources on one lane, instead of the thread-per-row gather, took
// 0.34 against 0.28 ms for the separate load and combine at 200k unknowns.) Entries are
// independent work items, so a row of 10^5 entries (a supply rail) costs no more than 10^5 short
// rows: one warp per row walking such a row's staged sources (an index, a source list, then the
// stamps, three dependent loads per entry) took ~6 ms at 200k unknowns.

int xd_tia_internal_pattern(const xd_tia *t, int *device, int *n_rows, int *nnz, const int **rowptr,
                            const int **colind);

struct xd_tia_fused {
  xd_tia *tia = nullptr;
  xd_ctx *fam = nullptr;
  int device = 0, n_rows = 0, nnz = 0;
  const int *d_rowptr = nullptr, *d_colind = nullptr;
  int2 *d_ent = nullptr;   // per CSR entry: (first source in the matrix map, count); count -1 = long entry
  int *d_diag = nullptr;   // per row: position of its diagonal entry, or -1
  XdLongRows lrows;        // the combine object's long rows (tia_long.h)
};

namespace {

constexpr int kFusedWarps = 8;
constexpr int kEntryBlock = 256;

// The family's dF/dx and dQ/dx of CSR entry k: its staged sources summed in the matrix map's
// order (as gather_short_kernel sums them), or the chunked gathers' sum for a long entry.
template <bool TRAN>
__device__ __forceinline__ void fused_entry_sums(int k, const int2 *__restrict__ ent, const int *__restrict__ msrc,
                                                 const double *__restrict__ stage, size_t mb_f, size_t mb_q,
                                                 const double *__restrict__ long_dfdx,
                                                 const double *__restrict__ long_dqdx, double &jf, double &jq) {
  const int2 e = ent[k];
  if (e.y < 0) {
    jf = long_dfdx[k];
    jq = TRAN ? long_dqdx[k] : 0.0;
    return;
  }
  double acc[2] = {0.0, 0.0};
  const size_t base[2] = {mb_f, mb_q};
  sum_sources<TRAN ? 2 : 1, false>(e.x, e.x + e.y, msrc, stage, base, acc);
  jf = acc[0];
  jq = acc[1];
}

// Newton matrix entry from the family's sums and the linear devices' constants, in
// tia_combine_kernel's operation order (the gmin shunt, on diagonals only, by the row kernel).
template <bool TRAN>
__device__ __forceinline__ double fused_matrix_entry(int k, double jf, double jq, double shunt, const xd_tia_coef &c,
                                                     const double *__restrict__ lin_f,
                                                     const double *__restrict__ lin_q) {
  if (lin_f) jf += lin_f[k];
  if (shunt != 0.0) jf += shunt;
  if (!TRAN) return jf;
  if (lin_q) jq += lin_q[k];
  return c.qscale * jq + c.fscale * jf;
}

template <bool TRAN>
__global__ void __launch_bounds__(kEntryBlock) fused_entry_kernel(
    int nnz, xd_tia_coef c, const int2 *__restrict__ ent, const int *__restrict__ msrc,
    const double *__restrict__ stage, size_t mb_f, size_t mb_q, const double *__restrict__ long_dfdx,
    const double *__restrict__ long_dqdx, const double *__restrict__ lin_f, const double *__restrict__ lin_q,
    double *__restrict__ jac) {
  const int k = blockIdx.x * kEntryBlock + threadIdx.x;
  if (k >= nnz) return;
  double jf, jq;
  fused_entry_sums<TRAN>(k, ent, msrc, stage, mb_f, mb_q, long_dfdx, long_dqdx, jf, jq);
  jac[k] = fused_matrix_entry<TRAN>(k, jf, jq, 0.0, c, lin_f, lin_q);
}

template <bool TRAN>
__global__ void __launch_bounds__(32 * kFusedWarps) fused_row_kernel(
    int n_rows, const int *__restrict__ rowptr, const int *__restrict__ colind, const int *__restrict__ diag,
    xd_tia_coef c, const double *__restrict__ x, const int2 *__restrict__ ent, const int *__restrict__ msrc,
    const double *__restrict__ stage, size_t mb_f, size_t mb_q, const double *__restrict__ long_dfdx,
    const double *__restrict__ long_dqdx, const double *__restrict__ fam_f, const double *__restrict__ fam_q,
    const double *__restrict__ fam_fx, const double *__restrict__ fam_qx, const double *__restrict__ lin_f,
    const double *__restrict__ lin_q, int limiter, const double *__restrict__ b, const double *__restrict__ qn0,
    const double *__restrict__ fhist, double *__restrict__ jac, double *__restrict__ rhs,
    double *__restrict__ q_tot, double *__restrict__ f_tot, XdLongRows L) {
  const int row = blockIdx.x * kFusedWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n_rows) return;
  const int beg = rowptr[row], end = rowptr[row + 1];
  // The linear devices' currents and charges of the row, lane-strided then a shuffle tree, as
  // tia_combine_kernel sums them; a long row's from its chunk sums, as there.
  double af = 0.0, aq = 0.0;
  if (end - beg > kLongRowEntries) {
    bool hd;
    long_row_sums(L, long_row_index(L, row), lane, af, aq, hd);
  } else if (lin_f || (TRAN && lin_q)) {
    for (int k = beg + lane; k < end; k += 32) {
      const double xc = x[colind[k]];
      if (lin_f) af += lin_f[k] * xc;
      if (TRAN && lin_q) aq += lin_q[k] * xc;
    }
  }
  if (end - beg <= kLongRowEntries) {
#pragma unroll
    for (int w = 16; w > 0; w >>= 1) {
      af += __shfl_down_sync(0xffffffffu, af, w);
      aq += __shfl_down_sync(0xffffffffu, aq, w);
    }
  }
  if (lane != 0) return;
  // The shunt goes on rows whose diagonal is in the pattern (the node rows): F and J together.
  const int dk = diag[row];
  const bool has_diag = c.gshunt != 0.0 && dk >= 0;
  if (has_diag) {
    double jf, jq;
    fused_entry_sums<TRAN>(dk, ent, msrc, stage, mb_f, mb_q, long_dfdx, long_dqdx, jf, jq);
    jac[dk] = fused_matrix_entry<TRAN>(dk, jf, jq, c.gshunt, c, lin_f, lin_q);
  }
  // The family's vector sums for the row, from the vector gather (rows it does not stamp keep
  // their zero values, as with the assigning load).
  const double ff = fam_f[row], fq = fam_q[row], ffx = fam_fx[row], fqx = fam_qx[row];
  double F = ff + af;
  if (has_diag) F += c.gshunt * x[row];
  if (b) F -= b[row];
  if (f_tot) f_tot[row] = F;
  if (!TRAN) {
    double r = -F;
    if (limiter) r = r + ffx;
    rhs[row] = r;
    return;
  }
  const double Q = fq + aq;
  if (q_tot) q_tot[row] = Q;
  double r = (Q - qn0[row]) * c.inv_h + c.fscale * F;
  if (c.hist_scale != 0.0) r = r + c.hist_scale * fhist[row];
  r = -r;
  if (limiter) r = r + c.qscale * fqx;
  if (limiter) r = r + c.fscale * ffx;
  rhs[row] = r;
}

// Per-target (first source, count) of a gather map over n_targets outputs: short targets get
// their range in the map's source list, long ones count -1, the others (0, 0).
int map_ranges(const GatherMap &m, int n_targets, std::vector<int2> &out) {
  out.assign((size_t)n_targets, make_int2(0, 0));
  std::vector<int> dst(m.n_short), ptr(m.n_short + 1), ldst(m.n_long);
  if (m.n_short > 0) {
    XD_CUDA(cudaMemcpy(dst.data(), m.d_short_dst, dst.size() * sizeof(int), cudaMemcpyDeviceToHost));
    XD_CUDA(cudaMemcpy(ptr.data(), m.d_short_ptr, ptr.size() * sizeof(int), cudaMemcpyDeviceToHost));
  }
  if (m.n_long > 0) XD_CUDA(cudaMemcpy(ldst.data(), m.d_long_dst, ldst.size() * sizeof(int), cudaMemcpyDeviceToHost));
  for (int t = 0; t < m.n_short; ++t) out[(size_t)dst[t]] = make_int2(ptr[t], ptr[t + 1] - ptr[t]);
  for (int t = 0; t < m.n_long; ++t) out[(size_t)ldst[t]] = make_int2(0, -1);
  return 0;
}

}  // namespace

extern "C" {

int xd_tia_fused_create(xd_tia *tia, xd_ctx *fam, xd_tia_fused **out) {
  if (!tia || !fam || !out) return fail(-1, "null argument");
  *out = nullptr;
  int device, n_rows, nnz;
  const int *rowptr, *colind;
  int rc = xd_tia_internal_pattern(tia, &device, &n_rows, &nnz, &rowptr, &colind);
  if (rc) return rc;
  if (device != fam->device) return fail(-1, "the combine object and the family are on different devices");
  if (n_rows != fam->n_unknowns || nnz != fam->nnz)
    return fail(-1, "the combine object's pattern is not the family's pattern");
  DeviceGuard g(device);
  std::vector<int2> ent;
  if ((rc = map_ranges(fam->mmap, nnz, ent)) != 0) return rc;
  // Each row's diagonal position (the gmin shunt's entry), from the pattern.
  std::vector<int> hp((size_t)n_rows + 1), hc((size_t)nnz), dpos((size_t)n_rows, -1);
  XD_CUDA(cudaMemcpy(hp.data(), rowptr, hp.size() * sizeof(int), cudaMemcpyDeviceToHost));
  if (nnz > 0) XD_CUDA(cudaMemcpy(hc.data(), colind, hc.size() * sizeof(int), cudaMemcpyDeviceToHost));
  for (int r = 0; r < n_rows; ++r)
    for (int k = hp[r]; k < hp[r + 1]; ++k)
      if (hc[k] == r) {
        dpos[r] = k;
        break;
      }
  xd_tia_fused *f = new xd_tia_fused();
  f->tia = tia;
  f->fam = fam;
  f->device = device;
  f->n_rows = n_rows;
  f->nnz = nnz;
  f->d_rowptr = rowptr;
  f->d_colind = colind;
  xd_tia_internal_long_rows(tia, &f->lrows);
  cudaError_t ce;
  if ((ce = cudaMalloc(&f->d_ent, std::max<size_t>(1, ent.size()) * sizeof(int2))) != cudaSuccess ||
      (ce = cudaMemcpy(f->d_ent, ent.data(), ent.size() * sizeof(int2), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (ce = cudaMalloc(&f->d_diag, std::max<size_t>(1, dpos.size()) * sizeof(int))) != cudaSuccess ||
      (ce = cudaMemcpy(f->d_diag, dpos.data(), dpos.size() * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess) {
    cudaFree(f->d_ent);
    cudaFree(f->d_diag);
    delete f;
    return cuda_fail(ce, "xd_tia_fused_create allocation");
  }
  *out = f;
  return 0;
}

int xd_tia_fused_destroy(xd_tia_fused *f) {
  if (!f) return 0;
  DeviceGuard g(f->device);
  cudaFree(f->d_ent);
  cudaFree(f->d_diag);
  delete f;
  return 0;
}

int xd_tia_load_combine(xd_tia_fused *fu, const xd_flags *flags, const xd_tia_coef *coef, const double *d_x,
                        double *d_next_sta, double *d_curr_sta, double *d_next_sto, const double *d_curr_sto,
                        double *d_fam_f, double *d_fam_q, double *d_fam_fx, double *d_fam_qx, double *d_fam_dfdx,
                        double *d_fam_dqdx, const double *d_lin_dfdx, const double *d_lin_dqdx, int limiter,
                        const double *d_b, const double *d_qn0, const double *d_fhist, double *d_jac,
                        double *d_rhs, double *d_q_tot, double *d_f_tot, void *stream) {
  if (!fu || !flags || !coef) return fail(-1, "null argument");
  if (fu->n_rows == 0) return 0;
  if (!d_x || !d_fam_f || !d_fam_q || !d_fam_fx || !d_fam_qx || !d_fam_dfdx || !d_fam_dqdx || !d_jac || !d_rhs)
    return fail(-1, "null device buffer");
  if (coef->mode != 0 && (!d_qn0 || (coef->hist_scale != 0.0 && !d_fhist)))
    return fail(-1, "null device buffer for a time step");
  xd_ctx *ctx = fu->fam;
  int rc = xd_update_state(ctx, flags, d_x, d_next_sta, d_curr_sta, d_next_sto, d_curr_sto, stream);
  if (rc) return rc;
  DeviceGuard g(fu->device);
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = (size_t)ctx->n, r = (size_t)ctx->vec_rows;
  const size_t mb = 4 * r * n, mm = (size_t)ctx->mat_slots * n;
  if (ctx->n > 0) {
    // The family's vector sums (all rows, a thread per row), and its long matrix entries' sums
    // (chunked) into its buffers.
    OutSet<4, false> vs{{d_fam_f, d_fam_q, d_fam_fx, d_fam_qx}, {0, r * n, 2 * r * n, 3 * r * n}, 1};
    if ((rc = run_gather(ctx->vmap, ctx->d_stage, vs, st))) return rc;
    OutSet<2, false> ms{{d_fam_dfdx, d_fam_dqdx}, {mb, mb + mm}, 1};
    if ((rc = run_gather(ctx->mmap, ctx->d_stage, ms, st, false))) return rc;
  }
  // Long rows: their chunks' linear-device sums (their matrix entries come from the entry kernel).
  if ((rc = xd_tia_internal_long_chunks(fu->tia, coef, d_x, nullptr, nullptr, d_lin_dfdx, d_lin_dqdx, nullptr, st)))
    return rc;
  const int row_blocks = (fu->n_rows + kFusedWarps - 1) / kFusedWarps;
  const int ent_blocks = (fu->nnz + kEntryBlock - 1) / kEntryBlock;
#define XD_ENTRY_ARGS                                                                                               \
  fu->nnz, *coef, fu->d_ent, ctx->mmap.d_src, ctx->d_stage, mb, mb + mm, d_fam_dfdx, d_fam_dqdx, d_lin_dfdx,         \
      d_lin_dqdx, d_jac
#define XD_ROW_ARGS                                                                                                 \
  fu->n_rows, fu->d_rowptr, fu->d_colind, fu->d_diag, *coef, d_x, fu->d_ent, ctx->mmap.d_src, ctx->d_stage, mb,   \
      mb + mm, d_fam_dfdx, d_fam_dqdx, d_fam_f, d_fam_q, d_fam_fx, d_fam_qx, d_lin_dfdx, d_lin_dqdx, limiter, d_b,   \
      d_qn0, d_fhist, d_jac, d_rhs, d_q_tot, d_f_tot, fu->lrows
  if (coef->mode != 0) {
    if (ent_blocks > 0) fused_entry_kernel<true><<<ent_blocks, kEntryBlock, 0, st>>>(XD_ENTRY_ARGS);
    fused_row_kernel<true><<<row_blocks, 32 * kFusedWarps, 0, st>>>(XD_ROW_ARGS);
  } else {
    if (ent_blocks > 0) fused_entry_kernel<false><<<ent_blocks, kEntryBlock, 0, st>>>(XD_ENTRY_ARGS);
    fused_row_kernel<false><<<row_blocks, 32 * kFusedWarps, 0, st>>>(XD_ROW_ARGS);
  }
#undef XD_ENTRY_ARGS
#undef XD_ROW_ARGS
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "fused load-and-combine launch");
  return 0;
}

}  // extern "C"
