"""GPU parity of the BSIM4 device load against the oracle (the reference's own device code).

Every test drives the same instances, the same solution / state / store inputs and the same
solver flags through (a) the oracle library and (b) the C ABI of libxyce_b200.so on cuda:0,
and compares F, Q, dF/dx*dVp, dQ/dx*dVp, the dF/dx and dQ/dx CSR values, and the new state and
store entries. Tolerance per entry: |gpu - ref| <= 1e-12 * max(|gpu|, |ref|) + 1e-14 * S
(+ 1e-14 * R for Jacobian entries), where S is the entry's sum of absolute contributions
(reported by xd_load_abs): the two sides sum the same terms in different orders, and S bounds
the rounding difference that ordering can cause; R is the largest magnitude in the entry's row,
the scale of the rounding residue left where capacitances cancel analytically.
"""
import numpy as np
import pytest

from tests.parity import family_inputs
from xyce_b200 import Bsim4Device, ModelCard, SolverFlags, netlist

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from tests.gpu_parity import GpuRun, run_sequence as _run_sequence  # noqa: E402


TRANSIENT_SEQ = [SolverFlags(newton_iter=1, voltlim=0), SolverFlags(newton_iter=1), SolverFlags(newton_iter=2),
                 SolverFlags(newton_iter=0), SolverFlags(newton_iter=0, init_tran=1),
                 SolverFlags(newton_iter=1, init_tran=1), SolverFlags(newton_iter=3)]
DC_SEQ = [SolverFlags(dcop=1, transient=0, newton_iter=0, init_jct=1), SolverFlags(dcop=1, transient=0, newton_iter=1),
          SolverFlags(dcop=1, transient=0, tranop=1, newton_iter=2), SolverFlags(dcop=1, transient=0, newton_iter=3)]


def test_parity_random_logic_default_cards():
    c = netlist.random_logic(4000, seed=11)
    worst = _run_sequence(c, None, TRANSIENT_SEQ + DC_SEQ)
    print("worst error / tolerance:", worst)


def test_parity_large_swings_limiting_active():
    c = netlist.random_logic(3000, seed=5)
    cards = [ModelCard(False, {"DIOMOD": 2}), ModelCard(True, {"DIOMOD": 0})]
    worst = _run_sequence(c, cards, [SolverFlags(newton_iter=1, voltlim=0)] +
                          [SolverFlags(newton_iter=k) for k in range(1, 6)], vrange=(-1.5, 4.0), seed=3)
    print("worst error / tolerance:", worst)


def test_parity_model_card_variants():
    c = netlist.random_logic(2000, seed=7)
    rng = np.random.default_rng(2)
    n = c.n_mos
    cards = [ModelCard(False, {"MOBMOD": 1, "DIOMOD": 2, "TOXE": 2.5e-9, "VTH0": 0.45, "U0": 0.04, "NDEP": 2e17,
                               "CJS": 1e-3, "CJSWS": 2e-10, "XPART": 1, "JSS": 1e-6, "LAMBDA": 0.2, "PCLM": 1.0,
                               "AGIDL": 1e-9, "BGIDL": 1e9, "CGIDL": 0.5, "EGIDL": 0.2}),
             ModelCard(True, {"MOBMOD": 2, "DIOMOD": 0, "TNOM": 25, "VTH0": -0.42, "XPART": 0.5, "CJS": 1e-3,
                              "CJSWGS": 3e-10, "CVCHARGEMOD": 1, "VTL": 2e5, "TEMPMOD": 1, "K1": 0.5, "K2": -0.02})]
    extra = {"NF": rng.choice([1.0, 2.0, 3.0], n), "AD": np.where(rng.random(n) < .5, np.nan, 1e-12),
             "PS": np.where(rng.random(n) < .5, np.nan, 3e-6), "SA": np.where(rng.random(n) < .3, 1e-6, np.nan),
             "SB": np.where(rng.random(n) < .3, 1e-6, np.nan), "DELVTO": rng.normal(0, 0.03, n),
             "M": rng.choice([1.0, 2.0], n)}
    worst = _run_sequence(c, cards, TRANSIENT_SEQ, extra_params=extra, vrange=(-0.5, 1.8))
    print("worst error / tolerance:", worst)


def _num_variants():
    from xyce_b200 import _native
    return _native.load().xd_num_eval_variants()


@pytest.mark.parametrize("v", [0, 1, 2, 3, 4, 5, 6, 7, 10, 11, 12, 13, 14, 15])
def test_parity_every_eval_launch_variant(v):
    """The autotuner may pick any launch shape of the evaluation kernel; each is held to the
    oracle, with an instance count that leaves a partial last block."""
    if v >= _num_variants():
        pytest.skip("no such variant")
    c = netlist.random_logic(1500, seed=21)
    worst = _run_sequence(c, None, TRANSIENT_SEQ[:3] + DC_SEQ[:2], eval_variant=v)
    print("variant", v, "worst error / tolerance:", worst)


def test_eval_launch_variants_bitwise_identical():
    c = netlist.random_logic(5000, seed=4)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c)
    n = im.shape[0]
    sol = np.random.default_rng(1).uniform(0, 1.2, c.n_unknowns)
    sto = np.random.default_rng(2).uniform(-0.2, 1.2, 14 * n)
    z3 = np.zeros(3 * n)
    ref = None
    for v in range(_num_variants()):
        dev = Bsim4Device(cards, im, nd, params, (rowptr, colind), c.n_unknowns)
        if dev._lib.xd_set_eval_variant(dev._h, v) != 0:
            dev.close()  # a variant for another staging layout (internal nodes)
            continue
        gpu = GpuRun(dev, int(rowptr[-1]), c.n_unknowns)
        out = gpu.load(SolverFlags(newton_iter=1), sol, z3, z3, sto.copy(), sto.copy())
        dev.close()
        if ref is None:
            ref = out
            continue
        for k in ref:
            if k == "abs":
                continue
            assert np.array_equal(ref[k], out[k], equal_nan=True), (v, k)


@pytest.mark.parametrize("capmod,xpart,cvc", [(0, 0.0, 0), (0, 0.5, 0), (0, 1.0, 0), (1, 0.0, 0), (1, 0.5, 1),
                                               (1, 1.0, 0)])
def test_parity_capmod_0_and_1(capmod, xpart, cvc):
    """The simple (capMod 0) and the non-charge-thickness (capMod 1) charge models, every charge
    partition, both threshold forms of the C-V gate overdrive (cvchargeMod), biases that reach
    accumulation, depletion, the linear and the saturation regions."""
    c = netlist.random_logic(1500, seed=31)
    cards = [ModelCard(False, {"CAPMOD": capmod, "XPART": xpart, "CVCHARGEMOD": cvc}),
             ModelCard(True, {"CAPMOD": capmod, "XPART": xpart, "CVCHARGEMOD": cvc, "VFBCV": -0.8})]
    worst = _run_sequence(c, cards, TRANSIENT_SEQ[:4] + DC_SEQ[2:3], vrange=(-0.4, 1.6), seed=capmod + 7)
    print("capMod", capmod, "xpart", xpart, "worst error / tolerance:", worst)


@pytest.mark.parametrize("igc,igb,cards_extra", [
    (1, 0, {}), (2, 0, {"PIGCD": 1.5}), (0, 1, {}), (2, 1, {"TOXE": 1.4e-9, "NF": 2.0, "AIGSD": 0.012}),
])
def test_parity_gate_tunnelling(igc, igb, cards_extra):
    """Gate tunnelling currents: gate to channel partitioned to source and drain (igcMod 1, with the
    bias-dependent partition, and 2 with a given PIGCD), gate to source / drain overlap, gate to
    bulk in accumulation and inversion (igbMod 1), thin oxide so the currents matter, multi-finger
    scaling; both operating modes (the random iterate puts drain below source on many devices)."""
    c = netlist.random_logic(1500, seed=41 + igc + 2 * igb)
    common = {"IGCMOD": igc, "IGBMOD": igb, "TOXE": cards_extra.get("TOXE", 1.8e-9)}
    common.update({k: v for k, v in cards_extra.items() if k not in ("TOXE", "NF")})
    cards = [ModelCard(False, dict(common, TNOIMOD=1)), ModelCard(True, dict(common))]
    extra = {"NF": np.full(c.n_mos, cards_extra["NF"])} if "NF" in cards_extra else None
    worst = _run_sequence(c, cards, TRANSIENT_SEQ[:4] + DC_SEQ[:2], extra_params=extra, vrange=(-0.6, 1.8),
                          seed=igc + igb)
    print("igcMod", igc, "igbMod", igb, "worst error / tolerance:", worst)


def test_gate_tunnelling_family_refuses_variants_without_it():
    from xyce_b200 import _native

    c = netlist.random_logic(200, seed=3)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c, [ModelCard(False, {"IGCMOD": 1}), ModelCard(True, {})])
    dev = Bsim4Device(cards, im, nd, params, (rowptr, colind), c.n_unknowns)
    lib = _native.load()
    ok = []
    for v in range(lib.xd_num_eval_variants()):
        ok.append(lib.xd_set_eval_variant(dev._h, v) == 0)
    dev.close()
    # 6, 7 and 11 are the full ones; 8, 9 are for internal nodes; 10 is a persistent common one;
    # 12-15 split the common evaluation into two kernels; 16-23 are for BSIM3 and MOSFET1; 24-27
    # for the general topology (24, 25 fused, 26, 27 split); 28, 29 split the common evaluation with
    # the DC part at 112 registers in 96- or 64-thread blocks.
    assert ok == ([False] * 6 + [True] * 2 + [False] * 2 + [False] + [True] + [False] * 4 + [False] * 8 + [False] * 4
                  + [False] * 2)


@pytest.mark.parametrize("variant", ["all", "mixed"])
def test_parity_series_resistance_internal_nodes(variant):
    """Drain / source sheet resistance (RSH x NRD / NRS, rdsMod = 0): internal D' / S' nodes
    numbered as the reference numbers them, the linear resistor currents and couplings, and the
    intrinsic device on (D', G, S', B). "mixed" also has instances without squares (no node) and
    with zero squares (no node, the reference's 1e3 S fallback conductance on the collapsed
    entries)."""
    from xyce_b200.device import internal_nodes

    c = netlist.random_logic(1500, seed=51)
    n = c.n_mos
    rng = np.random.default_rng(5)
    cards = [ModelCard(False, {"RSH": 25.0}), ModelCard(True, {"RSH": 40.0})]
    if variant == "all":
        nrd, nrs = np.full(n, 2.0), np.full(n, 1.5)
    else:
        nrd = np.where(rng.random(n) < 0.5, rng.uniform(0.5, 3.0, n), np.nan)
        nrs = np.where(rng.random(n) < 0.3, 0.0, rng.uniform(0.5, 3.0, n))
    extra = {"NRD": nrd, "NRS": nrs}
    cards_, im, nd, params = family_inputs(c, cards, extra)
    flags = internal_nodes(cards_, im, nd, params)
    assert flags.any()
    c2 = netlist.with_internal_nodes(c, flags)
    worst = _run_sequence(c2, cards, TRANSIENT_SEQ[:4] + DC_SEQ[:2], extra_params=extra, vrange=(-0.3, 1.5))
    print("series", variant, int(flags.sum()), "internal nodes; worst error / tolerance:", worst)


def test_parity_inverter_ring_bsim4():
    c = netlist.inverter_ring(101, vdd=1.8)
    worst = _run_sequence(c, None, TRANSIENT_SEQ, vrange=(0.0, 1.8))
    print("worst error / tolerance:", worst)


def test_load_is_deterministic():
    c = netlist.random_logic(20000, seed=1)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c)
    dev = Bsim4Device(cards, im, nd, params, (rowptr, colind), c.n_unknowns)
    gpu = GpuRun(dev, int(rowptr[-1]), c.n_unknowns)
    n = im.shape[0]
    sol = np.random.default_rng(0).uniform(0, 1.2, c.n_unknowns)
    z3, z14 = np.zeros(3 * n), np.zeros(14 * n)
    a = gpu.load(SolverFlags(), sol, z3, z3, z14, z14)
    # vgb state advanced by the first load: reload twice from the same inputs and compare bitwise.
    b = gpu.load(SolverFlags(), sol, z3, z3, z14, z14)
    c2 = gpu.load(SolverFlags(), sol, z3, z3, z14, z14)
    for k in ("f", "q", "dfdxdvp", "dqdxdvp", "dfdx", "dqdx", "next_sta", "next_sto"):
        assert np.array_equal(b[k], c2[k]), k
    dev.close()


def test_unsupported_card_is_refused():
    c = netlist.inverter_ring(5)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c, [ModelCard(False, {"MTRLMOD": 1}), ModelCard(True, {})])
    from xyce_b200._native import NativeError
    with pytest.raises(NativeError, match="mtrlMod"):
        Bsim4Device(cards, im, nd, params, (rowptr, colind), c.n_unknowns)


def test_persistent_eval_variants_walk_every_instance():
    """The persistent launch shapes run one wave of resident blocks over more instances than the
    wave holds (a grid-stride loop with a partial last stride); their loads equal the one-block-
    per-128-instances shape bit for bit."""
    from xyce_b200 import _native

    lib = _native.load()
    c = netlist.random_logic(100000, seed=8)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c)
    n = im.shape[0]
    assert n > 148 * 4 * 128
    sol = np.random.default_rng(3).uniform(0, 1.2, c.n_unknowns)
    sto = np.random.default_rng(4).uniform(-0.2, 1.2, 14 * n)
    z3 = np.zeros(3 * n)
    outs = {}
    for v in [2] + [v for v in range(lib.xd_num_eval_variants()) if lib.xd_eval_variant_persistent(v) == 1]:
        dev = Bsim4Device(cards, im, nd, params, (rowptr, colind), c.n_unknowns)
        assert dev._lib.xd_set_eval_variant(dev._h, v) == 0
        gpu = GpuRun(dev, int(rowptr[-1]), c.n_unknowns)
        outs[v] = gpu.load(SolverFlags(newton_iter=1), sol, z3, z3, sto.copy(), sto.copy())
        dev.close()
    assert len(outs) == 3
    for v, out in outs.items():
        for k in out:
            if k != "abs":
                assert np.array_equal(out[k], outs[2][k], equal_nan=True), (v, k)


def test_split_evaluation_equals_fused_bitwise():
    """The split launch shapes (DC part, then charges and stamps, handing per-instance state over
    through the context's buffer) give the fused evaluation's results bit for bit over a flag
    sequence that takes every path of the hand-off: limiting off and on, the first step of a
    transient (current state written too), junction initialisation and a DC load; the carried vgb
    of each load feeds the next."""
    from xyce_b200 import _native

    lib = _native.load()
    c = netlist.random_logic(20000, seed=12)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c)
    n = im.shape[0]
    seq = [SolverFlags(newton_iter=1, voltlim=0), SolverFlags(newton_iter=0, init_tran=1),
           SolverFlags(newton_iter=2), SolverFlags(dcop=1, transient=0, newton_iter=0, init_jct=1),
           SolverFlags(dcop=1, transient=0, tranop=1, newton_iter=1)]
    rng = np.random.default_rng(9)
    sols = [rng.uniform(-0.3, 1.5, c.n_unknowns) for _ in seq]
    split = [v for v in range(lib.xd_num_eval_variants())
             if lib.xd_eval_variant_split(v) == 1 and lib.xd_eval_variant_general(v) == 0]
    assert split
    outs = {}
    for v in [10] + split:
        dev = Bsim4Device(cards, im, nd, params, (rowptr, colind), c.n_unknowns)
        assert dev._lib.xd_set_eval_variant(dev._h, v) == 0
        gpu = GpuRun(dev, int(rowptr[-1]), c.n_unknowns)
        sta_n, sta_c, sto_n, sto_c = np.zeros(3 * n), np.zeros(3 * n), np.zeros(14 * n), np.zeros(14 * n)
        res = []
        for flags, sol in zip(seq, sols):
            g = gpu.load(flags, sol, sta_n, sta_c, sto_n, sto_c)
            res.append(g)
            sta_n, sta_c, sto_n = g["next_sta"], g["curr_sta"], g["next_sto"]
        outs[v] = res
        dev.close()
    for v in split:
        for step, (a, b) in enumerate(zip(outs[10], outs[v])):
            for k in a:
                if k != "abs":
                    assert np.array_equal(a[k], b[k], equal_nan=True), (v, step, k)
