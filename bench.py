"""BSIM4 device-load throughput on B200 (loads/s, eval + stamp), with roofline and CPU baseline.

One step = one full device load of every BSIM4 instance of the workload at a fixed Newton
iterate: update_state + loadDAEVectors + loadDAEMatrices through the C ABI (``xd_load_assign``,
which stores the family's sums into its own F, Q, dF/dx*dVp, dQ/dx*dVp, dF/dx and dQ/dx buffers,
so the reference loader's zeroing pass before every load is not needed). Metric: instances x
steps / device time.

Default workload: the scale configuration — a seeded random INV/NAND2/NOR2 netlist of about
1M BSIM4 MOSFETs with RC wire ladders (~3M R/C), node voltages uniform in 0-1.2 V, transient
flags (charges computed, limiting on, newton_iter > 0). The per-step working set (staging,
maps, CSR values) is several hundred MB, larger than the 126 MB L2, so no flush is needed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--mos M]

With N > 1 (torchrun), every rank loads its own replica circuit (seed + rank): the path has no
exchange step ("replicas only"); value = all ranks' instances x steps / max rank time.
--impl reference times the reference's own CPU load (the oracle library built from the
reference sources) on the host cores instead, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BSIM4 device loads/s (eval+stamp)"
UNIT = "loads/s"
# Algorithmic HBM bytes per instance per load of the evaluation kernel: reads 4 voltages (32),
# node indices (16), record index (4), 5 store values (40), vgb (8); writes 48 stamp values (384),
# 12 store (96), 3 state (24), vgb (8).
EVAL_BYTES_PER_INST = 32 + 16 + 4 + 40 + 8 + 384 + 96 + 24 + 8
# DRAM bytes per instance of one evaluation (dram__bytes_read.sum + dram__bytes_write.sum), for
# roofline.traffic. Fused kernel: one ncu capture at 199,832 instances of the same generator,
# 90 + 326 B. Split kernels (the bias / DC stage, a 37-double hand-off per instance, then the
# charge / stamp stage): one capture of both launches at 999,694 instances, the benchmark's own
# size, 88.4 + 274.0 MB and 351.2 + 588.9 MB, i.e. 362 + 940 B; the hand-off adds 2 x 296 B to the
# 612 algorithmic bytes.
EVAL_DRAM_BYTES_PER_INST_NCU = 90 + 326
SPLIT_DRAM_BYTES_PER_INST_NCU = 362 + 940
# FP64 operations per instance of one evaluation (ncu thread-instruction counters of the same
# capture: 2,621 DFMA (2 flops each) + 844 DMUL + 511 DADD per instance), for the evaluation
# kernel's compute roofline against the FP64 FMA-pipe probe.
EVAL_FP64_FLOPS_PER_INST = 2 * 2621 + 844 + 511


def replica_totals(dist, n, ms, device):
    """Whole-job figures of the replicas: the instances all ranks loaded (each rank's circuit is its
    own seeded replica, so the counts differ slightly) and the slowest rank's time per step."""
    if dist is None:
        return n, ms
    import torch

    t_n = torch.tensor([float(n)], dtype=torch.float64, device=device)
    t_ms = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t_n, op=dist.ReduceOp.SUM)
    dist.all_reduce(t_ms, op=dist.ReduceOp.MAX)
    return int(round(float(t_n.item()))), float(t_ms.item())


def replica_seed(seed, rank):
    """The seed of rank `rank`'s replica circuit."""
    return seed + rank


def eval_shape(lib, h):
    """The evaluation kernel's launch shape that the autotuner picked for a context."""
    import ctypes

    blk, minb = ctypes.c_int(), ctypes.c_int()
    v = lib.xd_get_eval_variant(h)
    lib.xd_eval_variant_info(v, ctypes.byref(blk), ctypes.byref(minb))
    return {"variant": v, "block": blk.value, "min_blocks_per_sm": minb.value,
            "persistent": lib.xd_eval_variant_persistent(v) == 1, "split": lib.xd_eval_variant_split(v) == 1}


def other_families(c, rowptr, colind, sol, dev_id, args):
    """Load throughput of the BSIM3 (level 9) and MOSFET1 (level 1) families on the same circuit and
    iterate as the BSIM4 step (xd_load_assign, transient flags, limiting on), CUDA events around
    10 steps after 3 warm-up steps. BSIM3 takes the ring oscillator's cards, MOSFET1 the defaults."""
    import ctypes

    import torch

    from xyce_b200 import ModelCard, MosfetDevice, SolverFlags, _native, netlist

    lib = _native.load()
    out = {}
    nu, nnz = c.n_unknowns, int(rowptr[-1])
    f64 = dict(dtype=torch.float64, device=f"cuda:{dev_id}")
    for name, level, cards in (("bsim3", 9, netlist.ring_bsim3_cards()),
                               ("mosfet1", 1, [ModelCard(False, {}), ModelCard(True, {})])):
        fam = MosfetDevice(cards, c.mos_type, c.mos_nodes, {"L": c.mos_l.astype(float), "W": c.mos_w.astype(float)},
                           (rowptr, colind), nu, device=dev_id, level=level)
        sta = [torch.zeros(fam.n_state, **f64) for _ in range(2)]
        sto = [torch.zeros(fam.n_store, **f64) for _ in range(2)]
        bufs = [torch.zeros(nu, **f64) for _ in range(4)] + [torch.zeros(nnz, **f64) for _ in range(2)]
        p = lambda t: ctypes.c_void_p(t.data_ptr())
        fam.load(SolverFlags(newton_iter=1, voltlim=0), sol, sta[0], sta[1], sto[0], sto[1], *bufs)

        def step():
            fl = SolverFlags(newton_iter=1).to_c()
            _native.check(lib.xd_load_assign(fam._h, ctypes.byref(fl), p(sol), p(sta[0]), p(sta[1]), p(sto[0]),
                                             p(sto[1]), *[p(b) for b in bufs],
                                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
                          "xd_load_assign")

        for _ in range(3):
            step()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(10):
            step()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 10
        out[name] = {"ms_per_step": ms, "loads_per_s": c.n_mos / (ms * 1e-3)}
        fam.close()
    return out


def general_family(args, dev_id, n_mos=200_000):
    """Load throughput of BSIM4's general topology: a seeded gate netlist whose NMOS cards use gate
    resistance with a gate-mid node (rgateMod 3), the body network (rbodyMod 1), bias-dependent S/D
    resistance (rdsMod 1) and the NQS charge node, and whose PMOS cards use rgateMod 2 with the
    five-resistor body network (rbodyMod 2): 15 local nodes and 85 stamp entries per instance.
    xd_load_assign with transient flags and limiting on, every evaluation launch shape that fits
    (fused and split) timed over 10 steps after 3 warm-up steps, and the autotuner's pick."""
    import ctypes

    import torch

    from xyce_b200 import ModelCard, MosfetDevice, SolverFlags, _native, netlist
    from xyce_b200.device import internal_nodes

    lib = _native.load()
    c = netlist.random_logic(n_mos, seed=args.seed + 7)
    n = c.n_mos
    cards = [ModelCard(False, {"RGATEMOD": 3, "RBODYMOD": 1, "RDSMOD": 1, "TRNQSMOD": 1, "RSH": 20.0}),
             ModelCard(True, {"RGATEMOD": 2, "RBODYMOD": 2, "RBPS0": 60.0, "RBPD0": 70.0})]
    extra = {"NRD": np.full(n, 2.0), "NRS": np.full(n, 1.5)}
    cards, im, nd, params = netlist.mosfet_family(c, cards, extra)
    flags, general = internal_nodes(cards, im, nd, params, general=True)
    assert general
    c = netlist.with_internal_nodes(c, flags)
    rowptr, colind = netlist.jacobian_pattern(c)
    nu, nnz = c.n_unknowns, int(rowptr[-1])
    fam = MosfetDevice(cards, im, nd, params, (rowptr, colind), nu, device=dev_id, level=14,
                       inst_internal=c.mos_internal)
    f64 = dict(dtype=torch.float64, device=f"cuda:{dev_id}")
    sol = torch.as_tensor(np.random.default_rng(args.seed).uniform(0.0, 1.2, nu), **f64)
    sta = [torch.zeros(fam.n_state, **f64) for _ in range(2)]
    sto = [torch.zeros(fam.n_store, **f64) for _ in range(2)]
    bufs = [torch.zeros(nu, **f64) for _ in range(4)] + [torch.zeros(nnz, **f64) for _ in range(2)]
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    fam.load(SolverFlags(newton_iter=1, voltlim=0), sol, sta[0], sta[1], sto[0], sto[1], *bufs)
    picked = lib.xd_get_eval_variant(fam._h)

    def time_steps():
        fl = SolverFlags(newton_iter=1).to_c()
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

        def step():
            _native.check(lib.xd_load_assign(fam._h, ctypes.byref(fl), p(sol), p(sta[0]), p(sta[1]), p(sto[0]),
                                             p(sto[1]), *[p(b) for b in bufs], st), "xd_load_assign")

        for _ in range(3):
            step()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(10):
            step()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 10

    shapes = {}
    for v in range(lib.xd_num_eval_variants()):
        if lib.xd_eval_variant_general(v) == 1 and lib.xd_set_eval_variant(fam._h, v) == 0:
            blk, minb = ctypes.c_int(), ctypes.c_int()
            lib.xd_eval_variant_info(v, ctypes.byref(blk), ctypes.byref(minb))
            key = f"{'split' if lib.xd_eval_variant_split(v) == 1 else 'fused'} {blk.value}x{minb.value}"
            shapes[key] = time_steps()
    lib.xd_set_eval_variant(fam._h, picked)
    ms = time_steps()
    fam.close()
    return {"workload": f"seeded INV/NAND2/NOR2 netlist, {n} BSIM4 MOSFETs with the general topology (NMOS rgateMod 3, "
                        f"rbodyMod 1, rdsMod 1, trnqsMod 1; PMOS rgateMod 2, rbodyMod 2), {int(flags.sum())} internal "
                        f"unknowns, {nnz} Jacobian nnz",
            "ms_per_step": ms, "loads_per_s": n / (ms * 1e-3), "eval_variant": picked,
            "ms_per_step_by_launch_shape": shapes}


def batched_section(args, dev_id):
    """The batched Monte-Carlo sweep: 256 circuits (sizes log-uniform 1k-20k MOSFETs, per-circuit
    DELVTO ~ N(0, 30 mV) and TOXE x U[0.98, 1.02]) merged into one block-diagonal system, every
    device load one evaluation launch over all circuits; timed as direct calls and as replays of
    a CUDA graph that captured the load (output zeroing + update_state + both gathers)."""
    import ctypes

    import torch

    from xyce_b200 import MosfetDevice, SolverFlags, _native, netlist

    b = netlist.batched_sweep(256, 1000, 20000, seed=args.seed)
    c = b.circuit
    rowptr, colind = netlist.jacobian_pattern(c)
    dev = MosfetDevice(b.cards, b.inst_model, c.mos_nodes, b.inst_params, (rowptr, colind), c.n_unknowns,
                       device=dev_id, level=14)
    n, nu, nnz = c.n_mos, c.n_unknowns, int(rowptr[-1])
    f64 = dict(dtype=torch.float64, device=f"cuda:{dev_id}")
    sol = torch.as_tensor(np.random.default_rng(args.seed).uniform(0, 1.2, nu), **f64)
    sta_n, sta_c = torch.zeros(3 * n, **f64), torch.zeros(3 * n, **f64)
    sto_n, sto_c = torch.zeros(14 * n, **f64), torch.zeros(14 * n, **f64)
    out = [torch.zeros(nu, **f64) for _ in range(4)] + [torch.zeros(nnz, **f64) for _ in range(2)]
    dev.load(SolverFlags(newton_iter=1, voltlim=0), sol, sta_n, sta_c, sto_n, sto_c, *out)
    flags = SolverFlags(newton_iter=1)

    def step():
        for v in out:
            v.zero_()
        dev.load(flags, sol, sta_n, sta_c, sto_n, sto_c, *out)

    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(3):
            step()
    torch.cuda.current_stream().wait_stream(s)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        step()
    res = {}
    for mode in ("direct", "cuda_graph"):
        for _ in range(3):
            graph.replay() if mode == "cuda_graph" else step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            graph.replay() if mode == "cuda_graph" else step()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        res[mode] = {"ms_per_load": ms, "loads_per_s": n / (ms * 1e-3)}
    shape = eval_shape(_native.load(), dev._h)
    dev.close()
    return {"workload": f"256 seeded gate netlists (sizes log-uniform 1k-20k, {n} BSIM4 MOSFETs in all, {nu} "
                        f"unknowns, {nnz} nnz), per-circuit DELVTO ~ N(0, 30 mV) and TOXE x U[0.98, 1.02] "
                        f"(512 model cards), one evaluation launch per load",
            "circuits": int(len(b.sizes)), "mosfets": n, **res,
            "eval_launch_shape": shape}


def placed_transient(args, n_mos=None, ns=None):
    """A gate netlist with placed wiring (a pin takes one of the 64 most recently opened fan-out
    slots; 100k MOSFETs and placed_ns by default, or n_mos MOSFETs for ns) through a transient on
    the GPU: fused device loads and combine, and the refactorization of every Newton matrix on the
    device, one host factorization at the start. Operating point from the logic-level starting
    iterate, then 0 - ns at 10 ps steps with the reference's transient Newton tolerances; the
    device state stays resident across the run."""
    import ctypes

    import torch

    from xyce_b200 import MosfetDevice, SolverFlags, netlist
    from xyce_b200.transient import GpuTransient, NewtonParams

    n_mos = args.placed_mos if n_mos is None else n_mos
    ns = args.placed_ns if ns is None else ns
    c = netlist.random_logic(n_mos, seed=args.seed, n_inputs=64, locality=64)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = netlist.mosfet_family(c, None)
    fam = MosfetDevice(cards, im, nd, params, (rowptr, colind), c.n_unknowns, level=14)
    g = GpuTransient(c, fam, rowptr, colind, solver="rf")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dc_its = g.dcop(x0=netlist.logic_initial_guess(c))
    torch.cuda.synchronize()
    dc_s = time.perf_counter() - t0
    st = g.stats
    f0, h0, l0 = st.factorizations, st.host_factorizations, st.loads
    t0 = time.perf_counter()
    _, w = g.run(ns * 1e-9, 10e-12, params=NewtonParams.transient(),
                 record=np.arange(0, c.n_nodes, 997))
    torch.cuda.synchronize()
    run_s = time.perf_counter() - t0
    its = int(sum(st.newton_iters))
    # Per-iteration parts, timed alone on the final state: device load + combine, refactor, solve.
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    fl = SolverFlags(newton_iter=1, pdt=1e11, gmin=g.gmin)
    zero = torch.zeros_like(g.x)
    ev[0].record()
    for _ in range(5):
        g._load_combine_raw(fl, 1, 1e-11, 2, zero, zero)  # the transient's path (fused where available)
    ev[1].record()
    for _ in range(5):
        g._load_raw(fl)
        g._combine(1, 1e-11, 2, zero, zero)
    ev[2].record()
    torch.cuda.synchronize()
    ref_ms = []
    for _ in range(3):
        t = time.perf_counter()
        g._lib.xd_rf_refactor(g._rf, ctypes.c_void_p(g.jac.data_ptr()))
        torch.cuda.synchronize()
        ref_ms.append((time.perf_counter() - t) * 1e3)
    x = g.rhs.clone()
    t = time.perf_counter()
    for _ in range(3):
        g._lib.xd_rf_solve(g._rf, ctypes.c_void_p(x.data_ptr()))
    torch.cuda.synchronize()
    solve_ms = (time.perf_counter() - t) * 1e3 / 3
    # The same refactorization and solve through cuSOLVER's refactorization library (comparison).
    ref_lib_ms = []
    for _ in range(3):
        t = time.perf_counter()
        g._lib.xd_rf_refactor_library(g._rf, ctypes.c_void_p(g.jac.data_ptr()))
        torch.cuda.synchronize()
        ref_lib_ms.append((time.perf_counter() - t) * 1e3)
    x = g.rhs.clone()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(3):
        g._lib.xd_rf_solve_library(g._rf, ctypes.c_void_p(x.data_ptr()))
    torch.cuda.synchronize()
    solve_lib_ms = (time.perf_counter() - t) * 1e3 / 3
    lev_l, lev_u = ctypes.c_int(), ctypes.c_int()
    g._lib.xd_rf_levels(g._rf, ctypes.byref(lev_l), ctypes.byref(lev_u))
    nnz_f, nlev, nupd = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
    g._lib.xd_rf_stats(g._rf, ctypes.byref(nnz_f), ctypes.byref(nlev), ctypes.byref(nupd))
    res = {"workload": f"seeded INV/NAND2/NOR2 netlist with placed wiring (fan-out U{{1..4}}, a pin takes one of "
                       f"the 64 most recent open slots), {c.n_mos} BSIM4 MOSFETs, {c.res_nodes.shape[0]} R + "
                       f"{c.cap_nodes.shape[0]} C wire parasitics, 64 PWL inputs, {c.n_unknowns} unknowns, "
                       f"{g.nnz} nnz; operating point, then 0-{ns:g} ns at 10 ps steps, reference "
                       f"transient Newton tolerances",
           "operating_point_s": dc_s, "operating_point_newton_iters": int(dc_its),
           "gpu_s_per_run": run_s, "steps": len(st.newton_iters), "failed_steps": st.failed_steps,
           "newton_iters_per_step": float(np.mean(st.newton_iters)),
           "ms_per_newton_iteration": run_s * 1e3 / max(1, its),
           "matrices": st.factorizations - f0, "host_factorizations": st.host_factorizations - h0,
           "solves": st.solves, "refinement_solves": st.refinements,
           "first_solve_backward_error": {q: float(np.quantile(st.first_solve_berr, v)) for q, v in
                                          (("median", 0.5), ("p90", 0.9), ("max", 1.0))} if st.first_solve_berr else None,
           "per_iteration_ms": {"device_loads_and_combine": ev[0].elapsed_time(ev[1]) / 5,
                                "device_loads_then_combine_unfused": ev[1].elapsed_time(ev[2]) / 5,
                                "refactorization": min(ref_ms), "refactorization_cusolver": min(ref_lib_ms),
                                "triangular_solves": solve_ms, "triangular_solves_cusolver": solve_lib_ms},
           "factor_levels": [lev_l.value, lev_u.value],
           "factors": {"entries": nnz_f.value, "elimination_levels": nlev.value, "updates": nupd.value},
           "swing_v": [float(w.min()), float(w.max())]}
    g.close()
    fam.close()
    return res


def transient_section(args):
    """Transient wall time per run, GPU path vs the oracle's loads through the same driver, and
    the learned warm start against the plain GPU path (Newton iterations per step)."""
    import torch

    from oracle.transient import OracleTransient
    from xyce_b200 import Bsim3Device, MosfetDevice, SolverFlags, netlist, surrogate as S
    from xyce_b200.transient import GpuTransient, NewtonParams

    out = {}
    if args.placed_only:
        out["placed_netlist"] = placed_transient(args)
        if args.scale_mos > 0:
            out["scale_1m"] = placed_transient(args, args.scale_mos, args.scale_ns)
        return out
    # BSIM3 ring oscillator: operating point, 0.1 V kick on node 1, 0-20 ns at 10 ps steps.
    c = netlist.inverter_ring(101, vdd=1.8)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards = netlist.ring_bsim3_cards()
    fam = Bsim3Device(cards, c.mos_type, c.mos_nodes, {"L": c.mos_l, "W": c.mos_w}, (rowptr, colind),
                      c.n_unknowns)
    runs = {}
    for name, mk in (("gpu", lambda: GpuTransient(c, fam, rowptr, colind)),
                     ("cpu_oracle", lambda: OracleTransient(c, cards, rowptr, colind, level=9))):
        tr = mk()
        tr.dcop()
        x0 = tr.x.clone()
        x0[1] += 0.1
        tr.set_initial_state(x0)
        if name == "gpu":
            torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, w = tr.run(20e-9, 10e-12, params=NewtonParams.transient(), record=[1, 51])
        if name == "gpu":
            torch.cuda.synchronize()
        runs[name] = (time.perf_counter() - t0, tr.stats, w)
    g_s, g_st, g_w = runs["gpu"]
    c_s, c_st, _ = runs["cpu_oracle"]
    out["ring_bsim3"] = {
        "workload": "101-stage BSIM3 ring oscillator, W/L 1u/0.18u (PMOS 2u), VDD 1.8 V, 5 fF/stage, operating "
                    "point + 0.1 V kick on node 1, 0-20 ns, 10 ps steps, reference transient Newton tolerances",
        "gpu_s_per_run": g_s, "cpu_oracle_s_per_run": c_s, "cpu_cores": 1,
        "gpu_newton_iters_per_step": float(np.mean(g_st.newton_iters)),
        "gpu_ms_per_newton_iteration": g_s * 1e3 / max(1, int(sum(g_st.newton_iters))),
        "gpu_static_pivot_fallbacks": g_st.static_pivot_fallbacks,
        "cpu_newton_iters_per_step": float(np.mean(c_st.newton_iters)), "steps": len(g_st.newton_iters),
        "node1_swing_v": [float(g_w[:, 0].min()), float(g_w[:, 0].max())]}
    fam.close()
    # Learned warm start on the placed gate netlist (the placed-netlist transient's circuit).
    t0 = time.perf_counter()
    sur = S.BsimSurrogate(seed=0)
    rep = sur.train(n_samples=args.surrogate_samples // 2, epochs=8)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    n_ws = args.placed_mos if args.placed_mos > 0 else 100_000
    c = netlist.random_logic(n_ws, seed=args.seed, n_inputs=64, locality=64)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = netlist.mosfet_family(c, None)
    res, waves = {}, {}
    for mode in ("plain", "warm_start"):
        fam = MosfetDevice(cards, im, nd, params, (rowptr, colind), c.n_unknowns, level=14)
        g = GpuTransient(c, fam, rowptr, colind, solver="rf")
        g.predictor = "linear"
        if mode == "warm_start":
            g.surrogate = S.SurrogateLoads(sur, fam, c.mos_type, c.mos_nodes, c.mos_w, c.mos_l)
        g.dcop(x0=netlist.logic_initial_guess(c))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, waves[mode] = g.run(args.placed_ns * 1e-9, 10e-12, params=NewtonParams.transient(),
                               record=np.arange(0, c.n_nodes, 97))
        torch.cuda.synchronize()
        st = g.stats
        res[mode] = {"s_per_run": time.perf_counter() - t0,
                     "exact_newton_iters_per_step": float(np.mean(st.newton_iters)),
                     "chord_iters_per_step": float(np.mean(st.chord_iters)) if st.chord_iters else 0.0,
                     "matrices": st.factorizations, "surrogate_loads": st.surrogate_loads}
        if mode == "warm_start":
            # One surrogate load against one exact FP64 load of the same instances, at the final point.
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            fl = SolverFlags(newton_iter=1, pdt=1e11, gmin=g.gmin)
            e[0].record()
            for _ in range(5):
                g._surrogate_load()
            e[1].record()
            for _ in range(5):
                g._load_raw(fl)
            e[2].record()
            torch.cuda.synchronize()
            res["load_ms"] = {"surrogate": e[0].elapsed_time(e[1]) / 5, "exact_fp64": e[1].elapsed_time(e[2]) / 5}
        g.close()
        fam.close()
    if args.placed_mos > 0:
        out["placed_netlist"] = placed_transient(args)
    if args.scale_mos > 0:
        # The scale configuration's transient: ~1M BSIM4 MOSFETs with placed wiring and ~3M R/C,
        # 2 ns, device-resident state.
        out["scale_1m"] = placed_transient(args, args.scale_mos, args.scale_ns)
    out["warm_start_placed"] = {
        "workload": f"the placed netlist: {c.n_mos} BSIM4 MOSFETs, {c.n_unknowns} unknowns, operating point, "
                    f"0-{args.placed_ns:g} ns at 10 ps, linear predictor on both paths, GPU refactorization",
        "plain": res["plain"], "warm_start": res["warm_start"], "load_ms": res["load_ms"],
        "max_waveform_difference_v": float(np.abs(waves["plain"] - waves["warm_start"]).max()),
        "surrogate": {"train_s": train_s, "samples": 2 * (args.surrogate_samples // 2),
                      "heldout_rel_error_median_p95": {t: {k: [round(v["rel_median"], 4), round(v["rel_p95"], 4)]
                                                           for k, v in r.items()} for t, r in rep.items()}}}
    return out


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mos", type=int, default=1_000_000)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--wire-segments", type=int, default=4)
    ap.add_argument("--cpu-sample", type=int, default=20000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-transient", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--surrogate-samples", type=int, default=20_000_000,
                    help="surrogate training samples in all (half per device type)")
    ap.add_argument("--placed-mos", type=int, default=100_000, help="MOSFETs of the placed-netlist transient (0: skip)")
    ap.add_argument("--placed-ns", type=float, default=1.0, help="length of the placed-netlist transient (ns)")
    ap.add_argument("--scale-mos", type=int, default=0,
                    help="MOSFETs of the scale transient (placed wiring; 0: skip; 1000000 for the scale configuration)")
    ap.add_argument("--scale-ns", type=float, default=2.0, help="length of the scale transient (ns)")
    ap.add_argument("--eval-variant", type=int, default=-1,
                    help="pin the BSIM4 evaluation launch shape (xd_set_eval_variant; default: the autotuner's pick)")
    ap.add_argument("--placed-only", action="store_true",
                    help="transient section: only the placed-netlist transient (for profiling its solve)")
    return ap.parse_args()


def build_workload(n_mos, seed, wire_segments):
    from xyce_b200 import netlist

    c = netlist.random_logic(n_mos, seed=seed, wire_segments=wire_segments)
    rowptr, colind = netlist.jacobian_pattern(c)
    return c, rowptr, colind


def family(c):
    from xyce_b200 import ModelCard

    cards = [ModelCard(False, {}), ModelCard(True, {})]
    return cards, c.mos_type.astype(np.int32), c.mos_nodes.astype(np.int32), {"L": c.mos_l, "W": c.mos_w}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, gpu_index):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        self.gpu = gpu_index

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        try:
            rows = [l.strip().split(", ") for l in open(self.path) if l.strip()]
        except Exception:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if len(r) > 5 + k and "Active" in r[5 + k]
                          and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(args, omp=False, sample=None, min_seconds=10.0):
    """Reference CPU load (oracle library = the reference's own device code) on a bounded sample.
    Serial: the plain build (no libm interposer) when present; omp: the OpenMP build."""
    from oracle import xyce_ref as xr
    from oracle.run import OracleRun

    sample = sample or args.cpu_sample
    c, rowptr, colind = build_workload(sample, args.seed, args.wire_segments)
    cards, im, nd, params = family(c)
    orc = OracleRun(c, cards, im, nd, params, rowptr, colind)
    plain = not omp and xr.available(plain=True)
    if omp or plain:
        # Same circuit through the OpenMP build (updateState parallel) or the plain serial build.
        orc.ref = xr.RefCircuit(14, [(m.pmos, dict(m.params)) for m in cards], im, nd, params, c.n_unknowns, omp=omp,
                                plain=plain)
        orc.ref.set_pattern(*_oracle_pattern(c, nd, rowptr, colind))
    n = im.shape[0]
    sol = np.random.default_rng(args.seed).uniform(0.0, 1.2, c.n_unknowns)
    from xyce_b200 import SolverFlags

    z3, z14 = np.zeros(3 * n), np.zeros(14 * n)
    r = orc.load(SolverFlags(newton_iter=1, voltlim=0), sol, z3, z3, z14, z14)
    orc.load(SolverFlags(newton_iter=1), sol, r["next_sta"], z3, r["next_sto"], z14)
    reps, dt = 1, orc.ref.time_loads(1)
    while dt < min_seconds and reps < 10000:
        reps = max(reps * 2, int(reps * min_seconds / max(dt, 1e-3) * 1.1))
        dt = orc.ref.time_loads(reps)
    return n * reps / dt, n, reps, dt, ("openmp" if omp else ("serial" if plain else "serial, libm interposer"))


def _oracle_pattern(c, inst_nodes, rowptr, colind):
    nu = c.n_unknowns
    pairs = [np.stack([np.repeat(np.arange(nu), np.diff(rowptr)), colind], 1)]
    nd = np.where(inst_nodes < 0, nu, inst_nodes).astype(np.int64)
    pairs.append(np.stack([np.repeat(nd, 4, axis=1).reshape(-1), np.tile(nd, (1, 4)).reshape(-1)], 1))
    pr = np.concatenate(pairs, 0)
    key = np.unique(pr[:, 0] * (nu + 1) + pr[:, 1])
    rows, cols = key // (nu + 1), (key % (nu + 1)).astype(np.int32)
    orp = np.zeros(nu + 2, dtype=np.int64)
    np.add.at(orp, rows + 1, 1)
    return np.cumsum(orp).astype(np.int32), cols


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference(args, rank):
    if rank != 0:
        return
    from oracle import xyce_ref as xr

    if not xr.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle library (reference sources compiled) not built"}))
        return
    omp = xr.available(omp=True)
    cores = host_cores()
    if omp:
        os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    samples = []
    for _ in range(args.warmup):
        cpu_baseline(args, omp=omp, min_seconds=1.0)
    for _ in range(args.steps):
        v, n, reps, dt, _ = cpu_baseline(args, omp=omp, min_seconds=2.0)
        samples.append((v, dt))
    value = statistics.median([s[0] for s in samples])
    total = sum(s[1] for s in samples)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / max(1, args.steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"random INV/NAND2/NOR2 logic, BSIM4, sample of {args.cpu_sample} MOSFETs "
                                   f"(generator of the {args.mos}-MOSFET scale circuit), fixed Newton iterate"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores if omp else 1, "kind": "reference",
                             "sample": f"{args.cpu_sample} BSIM4 instances x repeated loads, >=2 s per step; "
                                       f"{'OpenMP build (updateState parallel over instances)' if omp else 'serial build'}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch

    from xyce_b200 import Bsim4Device, SolverFlags, _native

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev_id = local
    c, rowptr, colind = build_workload(args.mos, replica_seed(args.seed, rank), args.wire_segments)
    cards, im, nd, params = family(c)
    n = im.shape[0]
    nu, nnz = c.n_unknowns, int(rowptr[-1])
    dev = Bsim4Device(cards, im, nd, params, (rowptr, colind), nu, device=dev_id)
    lib = _native.load()
    launches = lib.xd_launches_per_load(dev._h)
    import ctypes

    if args.eval_variant >= 0:
        _native.check(lib.xd_set_eval_variant(dev._h, args.eval_variant), "xd_set_eval_variant")
    shape = eval_shape(lib, dev._h)
    stream = torch.cuda.current_stream()
    f64 = dict(dtype=torch.float64, device=f"cuda:{dev_id}")
    rng = np.random.default_rng(args.seed + 17 * rank)
    sol_h = rng.uniform(0.0, 1.2, nu)
    sol = torch.as_tensor(sol_h, **f64)
    sta_n, sta_c = torch.zeros(3 * n, **f64), torch.zeros(3 * n, **f64)
    sto_n, sto_c = torch.zeros(14 * n, **f64), torch.zeros(14 * n, **f64)
    out = {k: torch.zeros(nu, **f64) for k in ("f", "q", "fx", "qx")}
    out["jf"], out["jq"] = torch.zeros(nnz, **f64), torch.zeros(nnz, **f64)
    # Consistent previous iterate: one load at the same voltages without limiting.
    dev.load(SolverFlags(newton_iter=1, voltlim=0), sol, sta_n, sta_c, sto_n, sto_c, *out.values())
    flags = SolverFlags(newton_iter=1)
    import ctypes as _ct

    def step():
        # xd_load_assign: the family's sums are stored straight into its own output buffers (zeroed
        # once above), so the caller's zeroing pass of the reference's loader is not needed.
        fl = flags.to_c()
        p = lambda t: _ct.c_void_p(t.data_ptr())
        _native.check(lib.xd_load_assign(dev._h, _ct.byref(fl), p(sol), p(sta_n), p(sta_c), p(sto_n), p(sto_c),
                                         p(out["f"]), p(out["q"]), p(out["fx"]), p(out["qx"]), p(out["jf"]),
                                         p(out["jq"]), _ct.c_void_p(torch.cuda.current_stream().cuda_stream)),
                      "xd_load_assign")

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev_id) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    n_all, ms_max = replica_totals(dist, n, ms, f"cuda:{dev_id}")
    value = n_all / (ms_max * 1e-3)

    # Per-kernel device time on the launching stream (eval kernel vs gathers).
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    t_eval, t_vec, t_mat, reps = 0.0, 0.0, 0.0, max(5, args.steps)
    for _ in range(reps):
        for v in out.values():
            v.zero_()
        evs[0].record(stream)
        dev.update_state(flags, sol, sta_n, sta_c, sto_n, sto_c)
        evs[1].record(stream)
        dev.load_dae_vectors(out["f"], out["q"], out["fx"], out["qx"])
        evs[2].record(stream)
        dev.load_dae_matrices(out["jf"], out["jq"])
        evs[3].record(stream)
        torch.cuda.synchronize()
        t_eval += evs[0].elapsed_time(evs[1])
        t_vec += evs[1].elapsed_time(evs[2])
        t_mat += evs[2].elapsed_time(evs[3])
    t_eval, t_vec, t_mat = t_eval / reps, t_vec / reps, t_mat / reps

    # FP64 FMA pipe throughput (project probe) for the evaluation kernel's compute roofline.
    probe = torch.zeros(148 * 8 * 256, **f64)
    iters = 2000
    lib.xd_probe_fp64_fma(probe.data_ptr(), 148 * 8, iters, stream.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    lib.xd_probe_fp64_fma(probe.data_ptr(), 148 * 8, iters, stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    fp64_peak_tflops = 2.0 * 148 * 8 * 256 * iters * 64 / (e0.elapsed_time(e1) * 1e-3) / 1e12

    # End to end through the C ABI with host buffers: every step copies its iterate and store in
    # from pinned host memory and every output (F, Q, both limiter vectors, both CSR value arrays,
    # state, store) back out. Two buffer sets and two streams pipeline consecutive steps: step
    # k's load runs while step k-1's results travel back over PCIe.
    pin = lambda t: torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    s_comp, s_copy = torch.cuda.Stream(), torch.cuda.Stream()
    sets = []
    for _ in range(2):
        d = {"sol": torch.empty_like(sol), "sta_n": torch.zeros_like(sta_n), "sto_n": torch.zeros_like(sto_n)}
        d.update({k: torch.zeros_like(v) for k, v in out.items()})
        h = {k: pin(v) for k, v in d.items() if k not in ("sol",)}
        h_in = {"sol": pin(sol), "sto_n": pin(sto_n)}
        h_in["sol"].copy_(torch.as_tensor(sol_h))
        h_in["sto_n"].copy_(sto_n.cpu())
        sets.append((d, h, h_in, torch.cuda.Event(), torch.cuda.Event()))
    h2d = (sol.numel() + sto_n.numel()) * 8
    d2h = sum(v.numel() for v in out.values()) * 8 + (sta_n.numel() + sto_n.numel()) * 8

    def e2e_step(k):
        d, h, h_in, computed, copied = sets[k % 2]
        s_comp.wait_event(copied)
        with torch.cuda.stream(s_comp):
            d["sol"].copy_(h_in["sol"], non_blocking=True)
            d["sto_n"].copy_(h_in["sto_n"], non_blocking=True)
            for key in ("f", "q", "fx", "qx", "jf", "jq"):
                d[key].zero_()
            dev.load(flags, d["sol"], d["sta_n"], sta_c, d["sto_n"], sto_c, d["f"], d["q"], d["fx"], d["qx"], d["jf"],
                     d["jq"], stream=s_comp)
            computed.record(s_comp)
        s_copy.wait_event(computed)
        with torch.cuda.stream(s_copy):
            for key in ("f", "q", "fx", "qx", "jf", "jq", "sta_n", "sto_n"):
                h[key].copy_(d[key], non_blocking=True)
            copied.record(s_copy)

    for k in range(4):
        e2e_step(k)
    torch.cuda.synchronize()
    e0.record(s_comp)
    for k in range(args.steps):
        e2e_step(k)
    e1.record(s_copy)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    _, e2e_ms = replica_totals(dist, n, e2e_ms, f"cuda:{dev_id}")
    e2e_value = n_all / (e2e_ms * 1e-3)
    # The link the end-to-end step is bound by: the same device-to-host copies of one step's
    # outputs, alone (no load, no host-to-device traffic), from the same buffers.
    d_set, h_set = sets[0][0], sets[0][1]
    e0.record(s_copy)
    for _ in range(3):
        with torch.cuda.stream(s_copy):
            for key in ("f", "q", "fx", "qx", "jf", "jq", "sta_n", "sto_n"):
                h_set[key].copy_(d_set[key], non_blocking=True)
    e1.record(s_copy)
    torch.cuda.synchronize()
    d2h_alone_gbs = d2h * 3 / (e0.elapsed_time(e1) * 1e-3) / 1e9
    d2h_e2e_gbs = d2h / (e2e_ms * 1e-3) / 1e9

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import xyce_ref as xr

        if xr.available():
            v, ns, reps_c, dt, build = cpu_baseline(args)
            cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"{ns} BSIM4 instances of the same generator x {reps_c} full loads ({dt:.1f} s), "
                             f"reference build -O2 ({build}), fixed Newton iterate"}
    hbm_peak, peak_src = measured_peaks()
    eval_achieved = EVAL_BYTES_PER_INST * n / (t_eval * 1e-3) / 1e9
    fp64_achieved = EVAL_FP64_FLOPS_PER_INST * n / (t_eval * 1e-3) / 1e12
    if shape["split"]:
        # The DC part under a register budget (bsim4_dc_kernel_regs) runs in 64- or 96-thread blocks.
        dc = "bsim4_dc_kernel" if shape["block"] == 128 else "bsim4_dc_kernel_regs"
        eval_kernel, dram_per_inst = f"{dc} + bsim4_charge_stamp_kernel", SPLIT_DRAM_BYTES_PER_INST_NCU
    else:
        eval_kernel, dram_per_inst = "bsim4_eval_kernel", EVAL_DRAM_BYTES_PER_INST_NCU
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"scale circuit: seeded random INV/NAND2/NOR2 logic, {n} BSIM4 MOSFETs per GPU, "
                               f"{c.res_nodes.shape[0]} R + {c.cap_nodes.shape[0]} C wire parasitics, "
                               f"{nnz} Jacobian nnz, fixed Newton iterate (node voltages U[0,1.2] V)",
                   "instances_per_gpu": n, "nnz": nnz, "parallelism": f"replicas x{world}",
                   "l2": "working set > 126 MB L2 (staging + maps + CSR values), no flush"},
        "gpu_launches": launches * args.steps,
        "roofline": {"bound": "fp64", "kernel": eval_kernel, "achieved": fp64_achieved,
                     "peak": fp64_peak_tflops, "unit": "TFLOP/s", "frac": fp64_achieved / fp64_peak_tflops,
                     "traffic": dram_per_inst * n,
                     "note": f"binding bound: the FP64 pipe ({EVAL_FP64_FLOPS_PER_INST} FP64 flops per instance, "
                             "executed-instruction count); peak = the FP64 FMA probe timed in this run "
                             "(the measured-peaks file has no FP64 figure); traffic = ncu DRAM bytes per "
                             f"instance ({dram_per_inst} B) x instances",
                     "hbm": {"achieved": eval_achieved, "peak": hbm_peak, "unit": "GB/s",
                             "frac": eval_achieved / hbm_peak, "peak_source": peak_src,
                             "algorithmic_bytes_per_instance": EVAL_BYTES_PER_INST}},
        "kernels_ms": {"eval": t_eval, "gather_vectors": t_vec, "gather_matrices": t_mat},
        "eval_launch_shape": shape,
        "fp64": {"probe_peak_tflops": fp64_peak_tflops, "flops_per_instance": EVAL_FP64_FLOPS_PER_INST,
                 "eval_achieved_tflops": EVAL_FP64_FLOPS_PER_INST * n / (t_eval * 1e-3) / 1e12,
                 "eval_frac": EVAL_FP64_FLOPS_PER_INST * n / (t_eval * 1e-3) / 1e12 / fp64_peak_tflops},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "link": {"bound": "device-to-host copy", "achieved_gbs": d2h_e2e_gbs,
                         "copies_alone_gbs": d2h_alone_gbs, "frac": d2h_e2e_gbs / d2h_alone_gbs}},
        "clocks": clk.summary(),
    }
    if cpu is not None:
        result["cpu_baseline"] = cpu
    if rank == 0 and world == 1 and not args.no_batched:
        result["other_families"] = other_families(c, rowptr, colind, sol, dev_id, args)
        result["other_families"]["bsim4_general_topology"] = general_family(args, dev_id)
        result["batched"] = batched_section(args, dev_id)
    if rank == 0 and world == 1 and not args.no_transient:
        from oracle import xyce_ref as xr

        if xr.available():
            result["transient"] = transient_section(args)
    if rank == 0:
        print(json.dumps(result))
    dev.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
