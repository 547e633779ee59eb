"""The reference-side binding (xyce_b200/binding/N_DEV_GpuMosfetB4.C) driven by the reference's own
device loop (GPU).

The binding is compiled against the reference's headers into the oracle harness
(oracle/_ref/libxyce_ref_gpu.so, `make -C oracle binding`) as the BSIM4 device master: the
reference's model and instance objects are created, their LIDs, state / store LIDs and Jacobian
offsets registered by the harness exactly as the reference's topology does, and the harness then
makes the device manager's calls — zeroing, Device::updateState, loadDAEVectors, loadDAEMatrices —
on the binding, which runs them through libxyce_b200.so. The outputs, in the reference's own
vectors and matrices, must equal the product's direct C-ABI load bit for bit (the binding only
permutes and adds into zeroed outputs) and match the reference's CPU load within the parity
tolerance, over a transient and DC flag sequence with limiting active, with and without internal
drain / source nodes, and with the general topology (gate and body resistance, rdsMod 1, the NQS
charge node, instance initial conditions).
"""
import numpy as np
import pytest

from oracle import xyce_ref as xr
from xyce_b200 import ModelCard, MosfetDevice, SolverFlags, netlist
from xyce_b200.device import internal_nodes

pytestmark = pytest.mark.gpu

pytest.importorskip("torch")

from tests.gpu_parity import GpuRun, check_step  # noqa: E402
from tests.parity import OracleRun, family_inputs  # noqa: E402

SEQ = [SolverFlags(dcop=1, transient=0, newton_iter=0, init_jct=1), SolverFlags(dcop=1, transient=0, newton_iter=1),
       SolverFlags(newton_iter=0, init_tran=1), SolverFlags(newton_iter=1), SolverFlags(newton_iter=2)]


@pytest.mark.parametrize("topology", ["plain", "series", "general"])
def test_reference_device_loop_through_gpu_binding(topology):
    if not xr.available(gpu=True):
        pytest.fail("oracle/_ref/libxyce_ref_gpu.so is not built (make -C oracle binding)")
    c = netlist.random_logic(2500, seed=61)
    n = c.n_mos
    cards, extra = None, None
    if topology == "series":
        cards = [ModelCard(False, {"RSH": 25.0}), ModelCard(True, {"RSH": 40.0})]
        extra = {"NRD": np.full(n, 2.0), "NRS": np.where(np.arange(n) % 3 == 0, np.nan, 1.5)}
    elif topology == "general":
        cards = [ModelCard(False, {"RGATEMOD": 3, "RBODYMOD": 1, "RDSMOD": 1, "RSH": 20.0}),
                 ModelCard(True, {"RGATEMOD": 1, "RBODYMOD": 2, "RBPS0": 60.0, "RBPD0": 70.0, "TRNQSMOD": 1})]
        # Initial conditions on NMOS instances (drain / source nodes exist: the reference places the
        # couplings in the branch currents' columns there).
        ic = (np.arange(n) % 9 == 0) & (c.mos_type == netlist.NMOS)
        extra = {"NRD": np.full(n, 2.0), "NRS": np.full(n, 1.5), "IC2": np.where(ic, 0.8, np.nan)}
    cards, im, nd, params = family_inputs(c, cards, extra)
    if topology == "series":
        c = netlist.with_internal_nodes(c, internal_nodes(cards, im, nd, params))
    elif topology == "general":
        c = netlist.with_internal_nodes(c, internal_nodes(cards, im, nd, params, general=True)[0])
    rowptr, colind = netlist.jacobian_pattern(c)
    ref = OracleRun(c, cards, im, nd, params, rowptr, colind)
    bnd = OracleRun(c, cards, im, nd, params, rowptr, colind, gpu_binding=True)
    dev = MosfetDevice(cards, im, nd, params, (rowptr, colind), c.n_unknowns, inst_internal=c.mos_internal)
    direct = GpuRun(dev, int(rowptr[-1]), c.n_unknowns)
    rng = np.random.default_rng(8)
    ns = dev.n_state_slots
    assert ns == ref.n_sta_slots
    sta_n, sta_c, sto_n, sto_c = np.zeros(ns * n), np.zeros(ns * n), np.zeros(14 * n), np.zeros(14 * n)
    for step, flags in enumerate(SEQ):
        sol = rng.uniform(-0.3, 1.5, c.n_unknowns)
        r = ref.load_with_sensitivity(flags, sol, sta_n, sta_c, sto_n, sto_c)
        b = bnd.load(flags, sol, sta_n, sta_c, sto_n, sto_c)
        g = direct.load(flags, sol, sta_n, sta_c, sto_n, sto_c)
        # The binding adds the library's sums into zeroed reference outputs: the direct load's values.
        for k in ("f", "q", "dfdxdvp", "dqdxdvp", "dfdx", "dqdx", "next_sta", "next_sto", "curr_sta"):
            assert np.array_equal(b[k], g[k]), (step, k)
        # And the reference's own load within the parity tolerance.
        b["abs"] = g["abs"]
        charges = bool(flags.transient or flags.tranop or flags.acop)
        check_step(step, flags, b, r, n, charges, rowptr, 14, ns, 14, vspan=1.8)
        sta_n, sta_c, sto_n = r["next_sta"], r["curr_sta"], r["next_sto"]
        if flags.newton_iter == 0 or flags.dcop:
            sto_c = r["next_sto"].copy()
    dev.close()
