/*
 * xyce_devload.h — C ABI of the B200 MOSFET device-load library (libxyce_b200.so).
 *
 * The library evaluates MOSFET instances and stamps F, Q, dF/dx, dQ/dx and the limiter
 * correction vectors into caller-owned device memory. It replaces, for one MOSFET family, the
 * three calls the reference's device manager makes on every Newton iteration:
 *
 *   xd_update_state   <- Device::updateState(solVec, staVec, stoVec)
 *                        src/DeviceModelPKG/Core/include/N_DEV_Device.h:315,
 *                        BSIM4 Master::updateState  src/DeviceModelPKG/OpenModels/src/N_DEV_MOSFET_B4.C:16180
 *   xd_load_vectors   <- Device::loadDAEVectors(solVec, fVec, qVec, bVec, storeLeadF, storeLeadQ)
 *                        N_DEV_Device.h:361, BSIM4 Master::loadDAEVectors  N_DEV_MOSFET_B4.C:16303
 *   xd_load_matrices  <- Device::loadDAEMatrices(dFdx, dQdx)
 *                        N_DEV_Device.h:384, BSIM4 Master::loadDAEMatrices N_DEV_MOSFET_B4.C:16577
 *
 * and the set-up the reference performs when a device is added and its Jacobian entries are
 * registered (DeviceMgr::addDeviceModel / addDeviceInstance, N_DEV_DeviceMgr.C:1272, 1446;
 * Instance::registerLIDs / registerStateLIDs / registerStoreLIDs / registerJacLIDs / setupPointers,
 * N_DEV_MOSFET_B4.C:4996-5626; CktGraphBasic::registerJacLIDswithDevs, N_TOP_CktGraphBasic.C:1092):
 *
 *   xd_create         <- addDeviceModel + addDeviceInstance + register*LIDs + setupPointers
 *   xd_destroy        <- DeviceMgr destructor for the family's Device object
 *
 * Conventions
 *   - Every function returns int: 0 = success, < 0 = error (argument, unsupported model feature
 *     or CUDA error). xd_last_error() describes the last error on the calling thread.
 *   - Loads follow the reference's contract: the caller zeroes the outputs once per Newton
 *     iteration (N_LOA_NonlinearEquationLoader.C:128-133, 226-227) and every device adds (+=)
 *     its contributions, so several families and other devices can share the same outputs.
 *   - Device pointers (d_*) are caller-owned device memory on the context's CUDA device. All
 *     work is ordered on the given CUDA stream (a cudaStream_t passed as void*; NULL = legacy
 *     default stream). Nothing is allocated or freed after xd_create.
 *   - Vector layout: one entry per unknown, indexed 0 .. n_unknowns-1; ground is not stored and
 *     reads as 0 V. Matrices are CSR value arrays for the pattern given at xd_create.
 *   - State/store layout: a family owns a contiguous block of the state (store) vector laid out
 *     slot-major: entry (slot s, instance i) at [s * n_inst + i]. BSIM4 has 3 state slots
 *     (qb, qg, qd) and 14 store slots (vbd vbs vgs vds vges vgms vdes vses vdbs vsbs vdbd vged
 *     vgmd von) — the reference's per-instance registration order (N_DEV_MOSFET_B4.C:5200, 5267).
 *   - Results are deterministic: no atomics; every output entry is summed in a fixed order.
 */
#ifndef XYCE_DEVLOAD_H
#define XYCE_DEVLOAD_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct xd_ctx xd_ctx;

/* Solver state the loads read (SolverState / DeviceOptions fields,
 * src/DeviceModelPKG/Core/include/N_DEV_SolverState.h:93-204, N_DEV_DeviceOptions.h). */
typedef struct xd_flags {
  int dcop;        /* dcopFlag: DC operating point                        */
  int init_tran;   /* initTranFlag: first time step of a transient         */
  int newton_iter; /* newtonIter: Newton iteration count within the step   */
  int init_jct;    /* initJctFlag: junction initialisation (first DCOP it) */
  int init_fix;    /* initFixFlag                                          */
  int transient;   /* transientFlag                                        */
  int tranop;      /* tranopFlag: DCOP phase of a transient                */
  int acop;        /* acopFlag                                             */
  int voltlim;     /* voltageLimiterFlag (.OPTIONS DEVICE VOLTLIM)         */
  int input_op;    /* inputOPFlag (not modelled: must be 0)                */
  double gmin;     /* DeviceOptions::gmin                                  */
  double pdt;      /* SolverState::pdt (alpha/dt)                          */
} xd_flags;

/* One MOSFET family (one reference Device object): its .MODEL cards and instances. */
typedef struct xd_mosfet_family {
  int level;                             /* 14 or 54 = BSIM4                                  */
  int n_models;                          /* number of .MODEL cards                            */
  const int *model_is_pmos;              /* [n_models] 0 = NMOS, 1 = PMOS                     */
  const int *model_nparams;              /* [n_models] (name, value) pairs per card           */
  const char *const *model_param_names;  /* concatenated over cards, netlist names            */
  const double *model_param_values;      /* same order                                        */
  int n_inst;                            /* number of instances                               */
  const int *inst_model;                 /* [n_inst] card index                               */
  const int *inst_nodes;                 /* [4*n_inst] D, G, S, B unknown index; -1 = ground  */
  int n_inst_params;                     /* instance-line parameter names                     */
  const char *const *inst_param_names;   /* e.g. "L", "W", "NF", "AD", "DELVTO", "M"          */
  const double *inst_param_values;       /* [n_inst * n_inst_params]; NaN = not given         */
  double temp_c;                         /* .OPTIONS DEVICE TEMP (Celsius)                    */
  double tnom_c;                         /* .OPTIONS DEVICE TNOM (Celsius)                    */
  const int *inst_internal;              /* [2*n_inst] internal drain, source unknown (D', S')
                                            or -1 where the node collapses onto D / S; null if
                                            no instance has one (see xd_internal_nodes)        */
  const int *inst_internal_gen;          /* BSIM4 general topology: [XD_GEN_INTERNAL*n_inst]
                                            the unknowns of D', S', G', GM, B', SB, DB, Q,
                                            IBS, IDS, IGS per instance, -1 where absent (see
                                            xd_internal_nodes_gen); null otherwise. Required
                                            when the cards use rgateMod, rbodyMod, rdsMod 1,
                                            trnqsMod 1 or instance ICs; then inst_internal
                                            must be null                                      */
} xd_mosfet_family;

/* Internal variables per instance of the BSIM4 general topology, in the reference's registerLIDs
 * order (N_DEV_MOSFET_B4.C:5018-5099): drain', source', gate' (rgateMod 1-3), gate-mid (rgateMod 3),
 * body', source-body, drain-body (rbodyMod 1/2), the NQS charge (trnqsMod 1), then the branch
 * currents of the initial conditions IC3 = VBS, IC1 = VDS, IC2 = VGS. */
#define XD_GEN_INTERNAL 11

/* Jacobian sparsity pattern over the unknowns (host memory, read during xd_create only).
 * Column indices must be sorted within each row and must include every entry the family's
 * stamps touch (the reference's topology builds the same union of device stamps). */
typedef struct xd_csr {
  int n_rows;          /* number of unknowns                 */
  const int *rowptr;   /* [n_rows + 1]                       */
  const int *colind;   /* [rowptr[n_rows]]                   */
} xd_csr;

/* Builds the family on CUDA device `cuda_device`: processes model cards (defaults,
 * temperature, size binning), uploads per-instance constants, and precomputes the
 * stamp-to-output gather maps. Fails (< 0) on unsupported model features. */
int xd_create(const xd_mosfet_family *family, const xd_csr *pattern, int cuda_device, xd_ctx **out);

/* Topology query before xd_create, as the reference's instances report their internal variables
 * (N_DEV_MOSFET_B4.C:3684-3760, registerLIDs :4996-5060; N_DEV_MOSFET_B3.C:1849-1865;
 * N_DEV_MOSFET1.C:1180-1253):
 * flags[2i] / flags[2i+1] = 1 when instance i has an internal drain / source node (BSIM4 with
 * rdsMod = 0: sheet resistance RSH with NRD / NRS > 0; BSIM3: RSH times NRD / NRS, 1 square by
 * default, nonzero; MOSFET1: RD / RS nonzero, else RSH times NRD / NRS nonzero). The caller allocates those unknowns (the reference numbers them after the
 * external ones, in instance order, drain first) and passes them in inst_internal. Host-only. */
int xd_internal_nodes(const xd_mosfet_family *family, int *flags);

/* The general topology's query (BSIM4 only): flags[XD_GEN_INTERNAL*i + k] = 1 when instance i has
 * internal variable k (order above; N_DEV_MOSFET_B4.C:3684-3769). The caller numbers them as the
 * reference does, after the external unknowns, instance by instance in that order, and passes
 * them in inst_internal_gen. A node the instance does not have is the same unknown as its
 * terminal (D' -> D, S' -> S, G' and GM -> G, B' / SB / DB -> B); an absent branch current has
 * none. Returns 1 when the family needs the general topology (inst_internal_gen is then required),
 * 0 when it does not (passing inst_internal_gen is still allowed: the general evaluation loads the
 * same values), < 0 on error. Host-only. */
int xd_internal_nodes_gen(const xd_mosfet_family *family, int *flags);

/* The general topology's stamp: rows[k], cols[k] (local nodes D=0, G, S, B, D', S', G', GM, B', SB,
 * DB, Q, IBS, IDS, IGS = 14) of its 85 Jacobian entries, in the reference's jacStamp order
 * (N_DEV_MOSFET_B4.C:4641-4795) with the charge node's columns of rows D', S', G' last; returns the
 * count. The pattern must hold every entry whose two nodes are unknowns after collapsing.
 * Host-only. */
int xd_general_stamp(int *rows, int *cols);

/* Releases all device memory of the context. */
int xd_destroy(xd_ctx *ctx);

/* Description of the last error on the calling thread ("" if none). */
const char *xd_last_error(void);

int xd_num_instances(const xd_ctx *ctx);
int xd_num_state_slots(const xd_ctx *ctx); /* per instance: 3 for BSIM4 (qb, qg, qd); 8 with the
                                              general topology (then qgmid, qbs, qbd, qcheq,
                                              qcdump, zero where the instance has no such
                                              charge)                                           */
int xd_num_store_slots(const xd_ctx *ctx); /* per instance: 14 for BSIM4 */

/* Evaluates every instance at the solution d_sol. Reads the previous iterate's limited
 * voltages from d_next_sto (newton_iter > 0) or d_curr_sto (newton_iter == 0), writes the new
 * store entries into d_next_sto (except vged/vgmd, which the reference does not write) and the
 * charges into d_next_sta; on the first Newton step of the first transient step it also writes
 * the charges into d_curr_sta (N_DEV_MOSFET_B4.C:16254-16289). The stamp values are kept in the
 * context for the following xd_load_vectors / xd_load_matrices calls. */
int xd_update_state(xd_ctx *ctx, const xd_flags *flags, const double *d_sol, double *d_next_sta,
                    double *d_curr_sta, double *d_next_sto, const double *d_curr_sto, void *stream);

/* Adds the family's F, Q, dF/dx*dVp and dQ/dx*dVp contributions (last xd_update_state). */
int xd_load_vectors(xd_ctx *ctx, double *d_f, double *d_q, double *d_dfdxdvp, double *d_dqdxdvp,
                    void *stream);

/* Adds the family's dF/dx and dQ/dx contributions into CSR value arrays of the pattern. */
int xd_load_matrices(xd_ctx *ctx, double *d_dfdx_vals, double *d_dqdx_vals, void *stream);

/* xd_update_state + xd_load_vectors + xd_load_matrices in one call. */
int xd_load(xd_ctx *ctx, const xd_flags *flags, const double *d_sol, double *d_next_sta, double *d_curr_sta,
            double *d_next_sto, const double *d_curr_sto, double *d_f, double *d_q, double *d_dfdxdvp,
            double *d_dqdxdvp, double *d_dfdx_vals, double *d_dqdx_vals, void *stream);

/* Like xd_load, but stores (=) the family's sum into every vector entry and CSR value the family
 * stamps, instead of adding to it; entries the family does not stamp are not touched. For a
 * caller that keeps one set of output buffers per device family (zeroed once when allocated),
 * this removes the zeroing pass the reference's loader makes before every load
 * (N_LOA_NonlinearEquationLoader.C:128-133, 226-227). No counterpart in the reference: its
 * devices only accumulate. */
int xd_load_assign(xd_ctx *ctx, const xd_flags *flags, const double *d_sol, double *d_next_sta,
                   double *d_curr_sta, double *d_next_sto, const double *d_curr_sto, double *d_f,
                   double *d_q, double *d_dfdxdvp, double *d_dqdxdvp, double *d_dfdx_vals,
                   double *d_dqdx_vals, void *stream);

/* Assembles vector stamps computed outside the library (by the learned surrogate, for instance):
 * d_stage16 holds 16 x n_inst doubles in the layout of the first 16 slots of xd_copy_stamps (F, Q,
 * dFdxdVp, dQdxdVp at D, G, S, B), summed into the four vectors through the family's gather map
 * with the same order and determinism as xd_load_vectors; assign != 0 stores instead of adding.
 * No counterpart in the reference. */
int xd_load_vectors_staged(xd_ctx *ctx, const double *d_stage16, double *d_f, double *d_q, double *d_dfdxdvp,
                           double *d_dqdxdvp, int assign, void *stream);

/* Test and error-bound support: like the two load calls, but adds |term| instead of term, so the
 * outputs hold, per entry, the sum of absolute contributions (the scale of the rounding error of
 * that entry's sum). */
int xd_load_abs(xd_ctx *ctx, double *d_f, double *d_q, double *d_dfdxdvp, double *d_dqdxdvp,
                double *d_dfdx_vals, double *d_dqdx_vals, void *stream);

/* Copies the per-instance local stamps of the last xd_update_state to host memory:
 * [48 * n_inst] doubles, slot-major (slot k of instance i at [k * n_inst + i]); slots 0-15 are
 * the F, Q, dFdxdVp, dQdxdVp terminal entries (D, G, S, B each), 16-31 dF/dx and 32-47 dQ/dx
 * as 4x4 row-major terminal blocks. A family with internal drain / source nodes has the wide
 * layout, [68 * n_inst]: each vector takes 6 rows (D', G, S', B, then the external D and S,
 * F only), dF/dx and dQ/dx take 22 slots each (the 4x4 block on D', G, S', B, then (D', D),
 * (D, D'), (D, D), (S', S), (S, S'), (S, S)). The general topology's layout is [230 * n_inst]:
 * each vector 15 rows (the local nodes of xd_general_stamp), then dF/dx and dQ/dx over its 85
 * stamp slots. xd_num_stage_slots gives the count. Synchronises the stream. */
int xd_copy_stamps(xd_ctx *ctx, double *h_out, void *stream);
int xd_num_stage_slots(const xd_ctx *ctx); /* staged values per instance: 48, 68 or 230 */

/* Diagnostics. xd_launches_per_load: kernels one xd_load enqueues (eval + gathers).
 * xd_probe_fp64_fma: runs `blocks` x 256 threads, each doing `iters` x 64 independent-chain
 * FP64 FMAs in registers, and writes one checksum per thread into d_out (blocks*256 doubles);
 * timing it gives the FP64 FMA-pipe throughput the evaluation kernel is measured against. */
int xd_launches_per_load(const xd_ctx *ctx);
/* Launch shape (threads per block, minimum resident blocks per SM) that xd_create's autotuner
 * selected for the evaluation kernel after timing every candidate on the circuit. */
int xd_eval_launch_shape(const xd_ctx *ctx, int *block, int *min_blocks);
/* The autotuner's candidates: xd_num_eval_variants() of them; xd_eval_variant_info gives the
 * launch shape of candidate v; xd_get_eval_variant / xd_set_eval_variant read and override the
 * context's choice (every candidate computes identical results; tests force each in turn). The
 * common candidates are compiled for BSIM4 capMod 2 without gate tunnelling; a family whose cards
 * use capMod 0/1 or igcMod/igbMod runs only the full ones, and xd_set_eval_variant refuses the
 * others for it. */
int xd_num_eval_variants(void);
int xd_eval_variant_info(int v, int *block, int *min_blocks);
/* 1 when candidate v is a persistent shape (one wave of resident blocks walking the instances with
 * a grid stride), 0 when it launches one block per `block` instances, < 0 for a bad v. */
int xd_eval_variant_persistent(int v);
/* 1 when candidate v splits the evaluation into two kernels — the DC part (limiting, junction
 * diodes, drain current, GIDL / GISL, gate tunnelling) and then charges, capacitances and stamps —
 * which hand per-instance state over through a buffer the context allocates at xd_create; each
 * kernel is smaller than the fused one (fewer registers, a smaller instruction footprint). Its
 * results are bit-identical to the fused candidates'. 0 otherwise, < 0 for a bad v. */
int xd_eval_variant_split(int v);
/* 1 when candidate v evaluates BSIM4's general topology (the only candidates a general-topology
 * family fits), 0 otherwise, < 0 for a bad v. */
int xd_eval_variant_general(int v);
int xd_get_eval_variant(const xd_ctx *ctx);
int xd_set_eval_variant(xd_ctx *ctx, int v);
int xd_probe_fp64_fma(double *d_out, int blocks, int iters, void *stream);

/* Allocation-free load (no counterpart in the reference: it is for callers of this library).
 *
 * Same work and same results as xd_load, but the scratch the load needs between evaluation and
 * assembly (48 staged values per instance and the chunk partial sums) lives in one fixed array
 * inside the library — a file-scope __device__ array of XD_STATIC_MAX_INSTANCES * 52 doubles
 * (6.8 MB) that every GPU loading the library holds until the process exits — instead of the
 * context's own buffers. The call itself performs no cudaMalloc, cudaFree or other allocation.
 * It is meant for callers that cannot allocate device memory when they load: a solver that has
 * handed all device memory to its own pool allocator, or that runs its Newton loop under a
 * fixed memory budget, still needs the context (xd_create allocates once at set-up) but gets
 * no per-call or per-context scratch from this entry point.
 *
 *   - Families with more than XD_STATIC_MAX_INSTANCES instances are rejected (< 0, see
 *     xd_last_error); use xd_load for them.
 *   - The first call on a device resolves the array's device address (cudaGetSymbolAddress)
 *     with that device current; make that first call before any stream capture.
 *   - Every call, from every context on the device, shares the one array and it keeps the last
 *     call's contents. Calls whose work overlaps on the GPU (different streams, or different
 *     host threads without ordering) race on it; order them on one stream.
 *   - Nothing in the array needs to start at zero: each call writes every staged value and
 *     every partial it later reads.
 *   - The staged stamps of a static load stay in the array, not in the context: after it,
 *     xd_load_vectors, xd_load_matrices, xd_load_abs and xd_copy_stamps on the same context
 *     return an error until the next xd_update_state (or xd_load) refills the context's own.
 *   - The array's device address is kept per device for the life of the process, so the call
 *     assumes the device's primary context is not reset (cudaDeviceReset) while the library is
 *     loaded.
 *   - Families with internal drain / source nodes (series resistance) are rejected: their
 *     staging layout is wider than the array's. */
#define XD_STATIC_MAX_INSTANCES 16384
int xd_load_static_scratch(xd_ctx *ctx, const xd_flags *flags, const double *d_sol, double *d_next_sta,
                           double *d_curr_sta, double *d_next_sto, const double *d_curr_sto, double *d_f,
                           double *d_q, double *d_dfdxdvp, double *d_dqdxdvp, double *d_dfdx_vals,
                           double *d_dqdx_vals, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* XYCE_DEVLOAD_H */
