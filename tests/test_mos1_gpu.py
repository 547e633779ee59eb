"""GPU parity of the level-1 MOSFET load (Shichman-Hodges + Meyer back-averaging) against the
oracle (the reference's own N_DEV_MOSFET1.C), with the same tolerance as the BSIM4 tests."""
import numpy as np
import pytest

from xyce_b200 import ModelCard, SolverFlags, netlist

pytestmark = pytest.mark.gpu

pytest.importorskip("torch")

from tests.gpu_parity import run_sequence  # noqa: E402

CARDS = [ModelCard(False, {"VTO": 0.7, "KP": 1e-4, "GAMMA": 0.4, "LAMBDA": 0.02, "CGSO": 1e-10, "CGDO": 1e-10,
                           "CGBO": 2e-10, "CJ": 1e-4, "CJSW": 1e-10, "TOX": 1e-8, "MJ": 0.4}),
         ModelCard(True, {"VTO": -0.7, "KP": 4e-5, "TOX": 2e-8, "NSUB": 1e16, "CBD": 1e-15, "CBS": 1e-15,
                          "IS": 1e-13})]
SEQ = [SolverFlags(dcop=1, transient=0, newton_iter=0, init_jct=1), SolverFlags(dcop=1, transient=0, newton_iter=1),
       SolverFlags(dcop=1, transient=0, tranop=1, newton_iter=2), SolverFlags(newton_iter=0, init_tran=1),
       SolverFlags(newton_iter=1), SolverFlags(newton_iter=2), SolverFlags(newton_iter=0), SolverFlags(newton_iter=1)]


def test_mos1_parity_random_logic():
    c = netlist.random_logic(3000, seed=21)
    n = c.n_mos
    rng = np.random.default_rng(4)
    extra = {"AD": np.where(rng.random(n) < .5, np.nan, 2e-12), "AS": np.where(rng.random(n) < .5, np.nan, 2e-12),
             "PD": np.full(n, 6e-6), "PS": np.full(n, 6e-6)}
    worst = run_sequence(c, CARDS, SEQ, vrange=(-0.5, 2.5), extra_params=extra, level=1, charges_in_dc=True)
    print("worst error / tolerance:", worst)


def test_mos1_parity_default_cards_ring():
    c = netlist.inverter_ring(51, vdd=1.8)
    worst = run_sequence(c, [ModelCard(False, {}), ModelCard(True, {})], SEQ, vrange=(0.0, 1.8), level=1,
                         charges_in_dc=True)
    print("worst error / tolerance:", worst)


def test_mos1_parity_series_resistance_internal_nodes():
    """Drain / source series resistance: NMOS with RD (which wins over the sheet resistance) and
    RSH x NRS, PMOS with RS alone (its drain collapses onto the terminal); the internal D' / S'
    nodes are numbered as the reference numbers them (N_DEV_MOSFET1.C:1180-1220, 1248-1253)."""
    from xyce_b200.device import internal_nodes
    from tests.parity import family_inputs

    c = netlist.random_logic(2000, seed=23)
    n = c.n_mos
    rng = np.random.default_rng(6)
    cards = [ModelCard(False, dict(CARDS[0].params, RD=20.0, RSH=30.0)), ModelCard(True, dict(CARDS[1].params, RS=15.0))]
    extra = {"NRD": rng.uniform(0.5, 3.0, n), "NRS": rng.uniform(0.5, 3.0, n)}
    cards_, im, nd, params = family_inputs(c, cards, extra)
    flags = internal_nodes(cards_, im, nd, params, level=1)
    nmos = c.mos_type == 0
    assert (flags[:, 0] == nmos).all() and flags[:, 1].all()
    c2 = netlist.with_internal_nodes(c, flags)
    worst = run_sequence(c2, cards, SEQ, vrange=(-0.5, 2.5), extra_params=extra, level=1, charges_in_dc=True)
    print("MOSFET1 series:", int(flags.sum()), "internal nodes; worst error / tolerance:", worst)
