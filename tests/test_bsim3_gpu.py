"""GPU parity of the BSIM3 (level 9) load against the oracle (the reference's own
N_DEV_MOSFET_B3.C), with the same per-entry tolerance as the BSIM4 tests: F, Q, dF/dx, dQ/dx,
the limiter vectors, the store and the state after every step of a DC-then-transient sequence."""
import numpy as np
import pytest

from xyce_b200 import Bsim3Device, ModelCard, SolverFlags, netlist

pytestmark = pytest.mark.gpu

pytest.importorskip("torch")

from tests.gpu_parity import GpuRun, run_sequence  # noqa: E402
from tests.parity import family_inputs  # noqa: E402

SEQ = [SolverFlags(dcop=1, transient=0, newton_iter=0, init_jct=1), SolverFlags(dcop=1, transient=0, newton_iter=1),
       SolverFlags(dcop=1, transient=0, tranop=1, newton_iter=2), SolverFlags(newton_iter=0, init_tran=1, pdt=1e11),
       SolverFlags(newton_iter=1, pdt=1e11), SolverFlags(newton_iter=2, pdt=1e11), SolverFlags(newton_iter=0, pdt=2e11),
       SolverFlags(newton_iter=1, pdt=2e11)]

# capMod 2 / 3, xpart 0 / 0.5 / 1, mobMod 1 / 2 / 3, poly depletion, K1/K2 given, gamma1 given,
# substrate current on, CLM / SCBE off, sidewall junctions.
VARIANT_CARDS = [
    [ModelCard(False, {"CAPMOD": 2, "XPART": 1, "MOBMOD": 2, "TOX": 4e-9, "JSW": 1e-10, "CJSWG": 3e-10}),
     ModelCard(True, {"CAPMOD": 3, "XPART": 0.5, "MOBMOD": 3, "K1": 0.5, "K2": -0.02, "NGATE": 1e20, "TNOM": 25})],
    [ModelCard(False, {"XPART": 1, "IJTH": 0, "CGDL": 1e-10, "CGSL": 1e-10, "RDSW": 0, "GAMMA1": 0.5, "PCLM": 0,
                       "PSCBE2": 0, "ALPHA0": 1e-6, "BETA0": 20}),
     ModelCard(True, {"XPART": 0.5, "VFB": -0.9, "A1": -0.1, "KETA": -0.5, "NCH": 3e17, "VBX": 0.5})],
]


def _junction_params(n, seed):
    rng = np.random.default_rng(seed)
    return {"AD": np.where(rng.random(n) < .5, np.nan, 2e-12), "AS": np.where(rng.random(n) < .5, np.nan, 2e-12),
            "PD": np.where(rng.random(n) < .3, 0.5e-6, 6e-6), "PS": np.full(n, 6e-6)}


def test_bsim3_parity_ring_default_cards():
    """The 101-stage ring oscillator's devices: W/L = 1u/0.18u (PMOS W = 2u), VDD = 1.8 V."""
    c = netlist.inverter_ring(101, vdd=1.8)
    worst = run_sequence(c, [ModelCard(False, {}), ModelCard(True, {})], SEQ, vrange=(0.0, 1.8), level=9)
    print("worst error / tolerance:", worst)


def test_bsim3_parity_random_logic_large_swings():
    c = netlist.random_logic(4000, seed=33, vdd=1.8, length=0.18e-6)
    worst = run_sequence(c, [ModelCard(False, {}), ModelCard(True, {})], SEQ, vrange=(-0.6, 2.6),
                         extra_params=_junction_params(c.n_mos, 5), level=9)
    print("worst error / tolerance:", worst)


@pytest.mark.parametrize("k", range(len(VARIANT_CARDS)))
def test_bsim3_parity_card_variants(k):
    c = netlist.random_logic(3000, seed=40 + k, vdd=1.8, length=0.18e-6)
    worst = run_sequence(c, VARIANT_CARDS[k], SEQ, vrange=(-0.3, 2.1), extra_params=_junction_params(c.n_mos, k),
                         level=9)
    print("worst error / tolerance:", worst)


@pytest.mark.parametrize("capmod,xpart", [(0, 0.0), (0, 0.5), (0, 1.0), (1, 0.0), (1, 0.5), (1, 1.0)])
def test_bsim3_parity_capmod_0_and_1(capmod, xpart):
    """The simple charge model (capMod 0, its own flat band VFBCV) and capMod 1 with its piecewise
    overlap capacitances (CGDL / CGSL), every charge partition, over accumulation to saturation."""
    c = netlist.random_logic(2000, seed=61 + capmod, vdd=1.8, length=0.18e-6)
    cards = [ModelCard(False, {"CAPMOD": capmod, "XPART": xpart, "CGDL": 2e-10, "CGSL": 2e-10}),
             ModelCard(True, {"CAPMOD": capmod, "XPART": xpart, "VFBCV": -0.7, "CGDL": 1e-10, "CGSL": 3e-10})]
    worst = run_sequence(c, cards, SEQ, vrange=(-0.5, 2.2), extra_params=_junction_params(c.n_mos, capmod),
                         level=9)
    print("capMod", capmod, "xpart", xpart, "worst error / tolerance:", worst)


def test_bsim3_parity_series_resistance_internal_nodes():
    """Drain / source sheet resistance (RSH x NRD / NRS, the squares default to 1): internal D' / S'
    nodes numbered as the reference numbers them, some instances with zero source squares (no
    source node)."""
    from xyce_b200.device import internal_nodes
    from tests.parity import family_inputs

    c = netlist.random_logic(2000, seed=71, vdd=1.8, length=0.18e-6)
    n = c.n_mos
    rng = np.random.default_rng(9)
    cards = [ModelCard(False, {"RSH": 30.0}), ModelCard(True, {"RSH": 45.0})]
    extra = {"NRD": rng.uniform(0.5, 3.0, n), "NRS": np.where(rng.random(n) < 0.3, 0.0, rng.uniform(0.5, 3.0, n))}
    cards_, im, nd, params = family_inputs(c, cards, extra)
    flags = internal_nodes(cards_, im, nd, params, level=9)
    assert flags.any() and not flags.all()
    c2 = netlist.with_internal_nodes(c, flags)
    worst = run_sequence(c2, cards, SEQ, vrange=(-0.3, 2.1), extra_params=extra, level=9)
    print("BSIM3 series:", int(flags.sum()), "internal nodes; worst error / tolerance:", worst)


def test_bsim3_load_is_deterministic():
    c = netlist.random_logic(20000, seed=2, vdd=1.8, length=0.18e-6)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c)
    dev = Bsim3Device(cards, im, nd, params, (rowptr, colind), c.n_unknowns)
    gpu = GpuRun(dev, int(rowptr[-1]), c.n_unknowns)
    n = im.shape[0]
    sol = np.random.default_rng(0).uniform(0, 1.8, c.n_unknowns)
    z5 = np.zeros(5 * n)
    a = gpu.load(SolverFlags(), sol, z5, z5, z5, z5)
    b = gpu.load(SolverFlags(), sol, z5, z5, z5, z5)
    for key in ("f", "q", "dfdxdvp", "dqdxdvp", "dfdx", "dqdx", "next_sta", "next_sto"):
        assert np.array_equal(a[key], b[key]), key
    dev.close()


def _family_variants(level):
    from xyce_b200 import _native
    from xyce_b200.device import MosfetDevice

    lib = _native.load()
    c = netlist.random_logic(200, seed=3)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c, netlist.ring_bsim3_cards() if level == 9 else None)
    dev = MosfetDevice(cards, im, nd, params, (rowptr, colind), c.n_unknowns, level=level)
    vs = [v for v in range(lib.xd_num_eval_variants()) if lib.xd_set_eval_variant(dev._h, v) == 0]
    dev.close()
    return vs


@pytest.mark.parametrize("level", [9, 1])
def test_launch_shape_candidates_parity_and_bitwise(level):
    """BSIM3 and MOSFET1 have their own launch-shape candidates, which the autotuner times per
    circuit. Each is held to the oracle, with a partial last block, and all give the same loads
    bit for bit."""
    variants = _family_variants(level)
    assert len(variants) >= 4
    c = netlist.random_logic(1500, seed=22)
    cards = netlist.ring_bsim3_cards() if level == 9 else [ModelCard(False, {}), ModelCard(True, {})]
    seq = SEQ[:2] + SEQ[3:6]
    for v in variants:
        worst = run_sequence(c, cards, seq, vrange=(-0.3, 1.8), level=level, eval_variant=v, charges_in_dc=level == 1)
        print("level", level, "variant", v, "worst error / tolerance:", worst)
    from xyce_b200.device import MosfetDevice

    rowptr, colind = netlist.jacobian_pattern(c)
    cards_, im, nd, params = family_inputs(c, cards)
    n = im.shape[0]
    rng = np.random.default_rng(5)
    sol = rng.uniform(-0.3, 1.8, c.n_unknowns)
    ref = None
    for v in variants:
        dev = MosfetDevice(cards_, im, nd, params, (rowptr, colind), c.n_unknowns, level=level)
        assert dev._lib.xd_set_eval_variant(dev._h, v) == 0
        z_sta, z_sto = np.zeros(dev.n_state), np.zeros(dev.n_store)
        out = GpuRun(dev, int(rowptr[-1]), c.n_unknowns).load(SolverFlags(newton_iter=1), sol, z_sta, z_sta, z_sto,
                                                              z_sto)
        dev.close()
        if ref is None:
            ref = out
            continue
        for k in out:
            if k != "abs":
                assert np.array_equal(out[k], ref[k], equal_nan=True), (level, v, k)
