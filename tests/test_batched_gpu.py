"""Batched Monte-Carlo sweep: many circuits, each with its own threshold shift (DELVTO) and oxide
thickness (TOXE, per-circuit model cards), merged block-diagonally and loaded by one evaluation
launch; parity of every circuit's loads against the oracle, and a CUDA-graph replay of the load
that matches the direct call bit for bit."""
import numpy as np
import pytest

from xyce_b200 import MosfetDevice, SolverFlags, netlist

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from tests.gpu_parity import GpuRun, check_step, waveform_errors  # noqa: E402
from tests.parity import OracleRun  # noqa: E402


def test_batched_sweep_parity_against_oracle():
    b = netlist.batched_sweep(24, 100, 2000, seed=1)
    c = b.circuit
    rowptr, colind = netlist.jacobian_pattern(c)
    dev = MosfetDevice(b.cards, b.inst_model, c.mos_nodes, b.inst_params, (rowptr, colind), c.n_unknowns, level=14)
    orc = OracleRun(c, b.cards, b.inst_model, c.mos_nodes, b.inst_params, rowptr, colind, level=14,
                    n_sta_slots=dev.n_state_slots)
    gpu = GpuRun(dev, int(rowptr[-1]), c.n_unknowns)
    n = c.n_mos
    rng = np.random.default_rng(3)
    sta, sto = np.zeros(3 * n), np.zeros(14 * n)
    for step, fl in enumerate([SolverFlags(newton_iter=1, voltlim=0), SolverFlags(newton_iter=1),
                               SolverFlags(newton_iter=2)]):
        sol = rng.uniform(0.0, 1.2, c.n_unknowns)
        r = orc.load_with_sensitivity(fl, sol, sta, sta, sto, sto)
        g = gpu.load(fl, sol, sta, sta, sto, sto)
        check_step(step, fl, g, r, n, True, rowptr, 14, 3, 14, vspan=1.2)
        sta, sto = r["next_sta"], r["next_sto"]
    dev.close()


def test_cuda_graph_replay_matches_direct_load():
    b = netlist.batched_sweep(16, 200, 3000, seed=2)
    c = b.circuit
    rowptr, colind = netlist.jacobian_pattern(c)
    dev = MosfetDevice(b.cards, b.inst_model, c.mos_nodes, b.inst_params, (rowptr, colind), c.n_unknowns, level=14)
    n, nu, nnz = c.n_mos, c.n_unknowns, int(rowptr[-1])
    f64 = dict(dtype=torch.float64, device="cuda")
    sol = torch.as_tensor(np.random.default_rng(0).uniform(0, 1.2, nu), **f64)
    sta_n, sta_c = torch.zeros(3 * n, **f64), torch.zeros(3 * n, **f64)
    sto_n, sto_c = torch.zeros(14 * n, **f64), torch.zeros(14 * n, **f64)
    out = [torch.zeros(nu, **f64) for _ in range(4)] + [torch.zeros(nnz, **f64) for _ in range(2)]
    flags = SolverFlags(newton_iter=1, voltlim=0)

    def step():
        for v in out:
            v.zero_()
        dev.load(flags, sol, sta_n, sta_c, sto_n, sto_c, *out)

    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        step()
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    direct = [v.clone() for v in out]
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        step()
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize()
    for a, d in zip(out, direct):
        assert torch.equal(a, d)
    dev.close()


def test_batched_sweep_transient_waveforms_match_per_circuit_oracle_runs():
    """The merged sweep through one transient on the GPU (one evaluation launch per load for all
    circuits, refactorization path), against separate oracle runs of single circuits of the sweep
    (their own TOXE cards and DELVTO): every compared circuit's node waveforms within reltol 1e-3 /
    abstol 1e-12. Newton tolerances are tight, so the merged system's shared convergence test
    cannot show in the waveforms."""
    from tests.parity import family_inputs
    from oracle.transient import OracleTransient
    from xyce_b200 import ModelCard
    from xyce_b200.transient import GpuTransient, NewtonParams

    seed, n_c, lo, hi = 3, 8, 200, 1500
    b = netlist.batched_sweep(n_c, lo, hi, seed=seed)
    c = b.circuit
    rowptr, colind = netlist.jacobian_pattern(c)
    tight = NewtonParams(max_iter=40, rhs_tol=1e-9, delta_x_tol=1e-3, abs_tol=1e-9, rel_tol=1e-6,
                         update_weights_each_iter=False)
    tight_dc = NewtonParams(rhs_tol=1e-12, delta_x_tol=1e-3, abs_tol=1e-12, rel_tol=1e-6)
    fam = MosfetDevice(b.cards, b.inst_model, c.mos_nodes, b.inst_params, (rowptr, colind), c.n_unknowns, level=14)
    g = GpuTransient(c, fam, rowptr, colind, solver="rf")
    g.dcop(tight_dc)
    tg, wg = g.run(0.8e-9, 10e-12, params=tight, record=np.arange(c.n_nodes))
    g.close()
    fam.close()
    worst = {}
    for k in (0, 3, 7):
        ck = netlist.random_logic(int(b.sizes[k]), seed=seed * 100003 + k + 1, wire_segments=2)
        assert ck.n_nodes == b.node_offset[k + 1] - b.node_offset[k]
        cards = [ModelCard(False, {"TOXE": 3.0e-9 * b.toxe_factor[k]}),
                 ModelCard(True, {"TOXE": 3.0e-9 * b.toxe_factor[k]})]
        extra = {"DELVTO": np.full(ck.n_mos, b.delvto[k])}
        rp, ci = netlist.jacobian_pattern(ck)
        o = OracleTransient(ck, cards, rp, ci, level=14, extra_params=extra)
        o.dcop(tight_dc)
        to, wo = o.run(0.8e-9, 10e-12, params=tight, record=np.arange(ck.n_nodes))
        assert np.array_equal(tg, to)
        mine = wg[:, b.node_offset[k]:b.node_offset[k + 1]]
        worst[k], point = waveform_errors(mine, wo)
        assert worst[k] <= 1.0 and point <= 1.0, (k, worst[k], point)
        assert (wo.max(0) - wo.min(0)).max() > 0.5  # inputs switch inside the window
    print("batched sweep: worst waveform error / bound per circuit", worst)
