"""Oracle parity of the BSIM4 load at the benchmarked sizes.

The throughput in bench.py is measured on the scale circuit (seeded INV/NAND2/NOR2 logic with ~1M
BSIM4 MOSFETs and 4-segment RC wires, node voltages U[0, 1.2] V, transient flags). This file runs
that exact circuit, iterate and flag sequence through the evaluation launch shape the autotuner
picks for it, and compares every output entry — F, Q, dF/dx*dVp, dQ/dx*dVp, both CSR value arrays,
state and store — with the reference's own load (the oracle library), within the parity tolerance,
as the small parity tests do. The same is done for the 100k-MOSFET gate netlist with 64 inputs.

Sequence per circuit: (1) a load without limiting from zero state, (2) the benchmark's timed load
(same iterate, limiting on, Newton iteration 1), (3) a load at a second random iterate, where the
limiters act on most instances. Besides the pass/fail, each output reports how many entries agree
at plain 1e-12 relative without any floor; the fraction that needed a floor must stay small.
"""
import numpy as np
import pytest

from xyce_b200 import MosfetDevice, SolverFlags, netlist

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from tests.gpu_parity import GpuRun, check_step, log_strict  # noqa: E402
from tests.parity import OracleRun, family_inputs, stamp_counts  # noqa: E402

# bench.py's default workload (scale circuit, seed 2026) and the 100k gate netlist.
CASES = {
    "scale_1m": dict(n_mos_target=1_000_000, seed=2026, wire_segments=4),
    "gates_100k": dict(n_mos_target=100_000, seed=7, n_inputs=64),
}
# Largest fraction of an output's entries allowed to need a tolerance floor (the rest must agree
# at plain 1e-12 relative). The limiter vectors are sums of per-instance terms built to cancel
# (the source entry is minus the others, each a capacitance or conductance times a voltage step):
# where a node's terms nearly cancel, a one-ulp difference of an exp / log result in one term is
# far above 1e-12 of the small total, so more of their entries rely on the row-scaled floor.
MAX_FLOOR_FRACTION = {"dfdxdvp": 0.1, "dqdxdvp": 0.1}
DEFAULT_MAX_FLOOR_FRACTION = 1e-2


@pytest.mark.parametrize("case", list(CASES))
def test_oracle_parity_at_benchmark_size(case):
    c = netlist.random_logic(**CASES[case])
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c)
    dev = MosfetDevice(cards, im, nd, params, (rowptr, colind), c.n_unknowns, level=14)
    variant = dev._lib.xd_get_eval_variant(dev._h)
    orc = OracleRun(c, cards, im, nd, params, rowptr, colind)
    gpu = GpuRun(dev, int(rowptr[-1]), c.n_unknowns)
    n = im.shape[0]
    rng = np.random.default_rng(CASES[case]["seed"])
    sol1 = rng.uniform(0.0, 1.2, c.n_unknowns)
    sol2 = rng.uniform(0.0, 1.2, c.n_unknowns)
    seq = [(SolverFlags(newton_iter=1, voltlim=0), sol1), (SolverFlags(newton_iter=1), sol1),
           (SolverFlags(newton_iter=2), sol2)]
    sta_n, sta_c = np.zeros(3 * n), np.zeros(3 * n)
    sto_n, sto_c = np.zeros(14 * n), np.zeros(14 * n)
    strict, worst = {}, {}
    counts = stamp_counts(rowptr, colind, nd, c.n_unknowns)
    for step, (flags, sol) in enumerate(seq):
        r = orc.load_with_sensitivity(flags, sol, sta_n, sta_c, sto_n, sto_c)
        g = gpu.load(flags, sol, sta_n, sta_c, sto_n, sto_c)
        rep = check_step(step, flags, g, r, n, True, rowptr, 14, 3, 14, vspan=1.2, strict=strict, counts=counts)
        for k, v in rep.items():
            worst[k] = max(worst.get(k, 0.0), v)
        sta_n, sta_c, sto_n = r["next_sta"], r["curr_sta"], r["next_sto"]
    dev.close()
    log_strict(strict)
    print(f"{case}: {n} instances, evaluation variant {variant}, worst error / tolerance {worst}")
    for key, (tot, ok, idx, cls) in strict.items():
        frac = (tot - ok) / max(1, tot)
        print(f"  {key}: {ok}/{tot} within plain 1e-12 relative, {tot - ok} needed a floor ({frac:.2e}: "
              f"summation order {cls[0]}, cancellation {cls[1]}, libm ulp {cls[2]})")
        limit = MAX_FLOOR_FRACTION.get(key, DEFAULT_MAX_FLOOR_FRACTION)
        assert frac <= limit, f"{key}: {frac:.3g} of the entries needed a tolerance floor"
