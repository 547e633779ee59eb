"""BSIM4's general topology: gate resistance (rgateMod 1-3), the body resistance network (rbodyMod
1/2), bias-dependent source / drain resistance (rdsMod 1), the transient NQS charge model
(trnqsMod 1: a charge node, the charge partition by qdrn / qcheq) and instance initial conditions
(IC1-3), each with the internal nodes and branch currents the reference gives it
(src/DeviceModelPKG/OpenModels/src/N_DEV_MOSFET_B4.C: nodes :3684-3769, registerLIDs :4996-5099,
jacStamp :4641-4795, NQS :11626-11637, 12616-13045, 12216-12322, the loads :16303-16853 and
:17102-17187).

CPU: the library's stamp table and topology query against the reference's own instances (the
oracle library): the same internal variables per instance, numbered the same way, and a pattern
that holds every entry the reference's stamps touch. GPU: the load through the C ABI against the
oracle over DC and transient flag sequences with limiting active, within the parity tolerance of
the other BSIM4 tests, for each mode on its own and all of them mixed in one family.
"""
import numpy as np
import pytest

from oracle import xyce_ref as xr
from xyce_b200 import ModelCard, SolverFlags, netlist
from xyce_b200.device import GEN_INTERNAL, general_stamp, internal_nodes

from tests.parity import OracleRun, family_inputs

pytestmark = pytest.mark.skipif(not xr.available(), reason="oracle library not built")

# Sheet resistance with squares on every instance keeps the reference from falling back to its
# 1e3 S conductance (and from warning about it) where rdsMod 1 asks for S/D resistors.
_RS = {"RSH": 20.0}
BODY5 = {"RBPS0": 60.0, "RBPD0": 70.0, "RBSBX0": 120.0, "RBSBY0": 150.0, "RBDBX0": 110.0, "RBDBY0": 140.0,
         "RBPBX0": 90.0, "RBPBY0": 80.0, "RBSDBXL": 0.1, "RBPBXW": -0.2}
CASES = {
    "rgate1": [ModelCard(False, {"RGATEMOD": 1, "RSHG": 5.0}), ModelCard(True, {"RGATEMOD": 1, "RSHG": 8.0})],
    "rgate2": [ModelCard(False, {"RGATEMOD": 2, "XRCRG1": 14.0, "XRCRG2": 1.5}),
               ModelCard(True, {"RGATEMOD": 2, "RSHG": 3.0})],
    "rgate3": [ModelCard(False, {"RGATEMOD": 3, "RSHG": 4.0, "CAPMOD": 1}),
               ModelCard(True, {"RGATEMOD": 3, "XRCRG1": 10.0})],
    "rbody1": [ModelCard(False, {"RBODYMOD": 1, "RBDB": 40.0, "RBSB": 30.0}),
               ModelCard(True, {"RBODYMOD": 1, "GBMIN": 1e-10})],
    "rbody2": [ModelCard(False, {"RBODYMOD": 2, **BODY5}), ModelCard(True, {"RBODYMOD": 2, "RBPS0": 55.0,
                                                                             "RBPD0": 65.0})],
    "rds1": [ModelCard(False, {"RDSMOD": 1, "RDSW": 150.0, "RDW": 80.0, "RSW": 90.0, "RDWMIN": 5.0, "RSWMIN": 4.0,
                               "PRWG": 0.1, "PRWB": 0.05, **_RS}),
             ModelCard(True, {"RDSMOD": 1, "RDW": 120.0, "RSW": 100.0, **_RS})],
    "mixed": [ModelCard(False, {"RGATEMOD": 3, "RBODYMOD": 1, "RDSMOD": 1, "IGCMOD": 1, "RDW": 60.0, "RSW": 70.0,
                                **_RS}),
              ModelCard(True, {"RGATEMOD": 2, "RBODYMOD": 2, "CAPMOD": 0, **BODY5})],
    "nqs": [ModelCard(False, {"TRNQSMOD": 1}), ModelCard(True, {"TRNQSMOD": 1, "XRCRG1": 10.0, "XPART": 0.5})],
    # NQS with the gate-resistance modes that scale gcrg in place (the NQS conductances take the
    # unscaled values) and with the body network's extra state slots before the NQS ones.
    "nqs_rgate": [ModelCard(False, {"TRNQSMOD": 1, "RGATEMOD": 2, "XPART": 1.0}),
                  ModelCard(True, {"TRNQSMOD": 1, "RGATEMOD": 3, "RBODYMOD": 1, "CAPMOD": 1, "RSHG": 4.0})],
    # Instances switching NQS off (and on) against their model's setting.
    "nqs_mixed": [ModelCard(False, {"TRNQSMOD": 1, "RDSMOD": 1, "RDW": 60.0, "RSW": 70.0, **_RS}),
                  ModelCard(True, {"RGATEMOD": 1, "RSHG": 8.0, "CAPMOD": 0})],
}


def _extra(case, n, rng, nmos):
    extra = {"NRD": np.full(n, 2.0), "NRS": np.full(n, 1.5)} if case in ("rds1", "mixed", "nqs_mixed") else {}
    if case == "nqs_mixed":
        extra["TRNQSMOD"] = np.where(rng.random(n) < 0.3, np.where(nmos, 0.0, 1.0), np.nan)
    if case == "mixed":
        # Instance overrides of the modes, and initial conditions on some instances: on the NMOS
        # ones, whose drain / source nodes exist (rdsMod 1), where the reference places the
        # initial-condition couplings in the branch currents' columns (see
        # test_reference_ic_coupling_placement for the instances where it does not).
        extra["RGATEMOD"] = np.where(rng.random(n) < 0.2, 1.0, np.nan)
        extra["RBODYMOD"] = np.where(rng.random(n) < 0.2, 0.0, np.nan)
        extra["IC1"] = np.where(nmos & (rng.random(n) < 0.2), 0.4, np.nan)
        extra["IC2"] = np.where(nmos & (rng.random(n) < 0.2), 0.9, np.nan)
        extra["IC3"] = np.where(nmos & (rng.random(n) < 0.2), -0.2, np.nan)
    return extra


def _circuit(case, n_mos=600, seed=21):
    c = netlist.random_logic(n_mos, seed=seed)
    extra = _extra(case, c.n_mos, np.random.default_rng(seed), c.mos_type == netlist.NMOS)
    cards, im, nd, params = family_inputs(c, CASES[case], extra)
    flags, general = internal_nodes(cards, im, nd, params, general=True)
    assert general
    return netlist.with_internal_nodes(c, flags), cards, extra, flags


def test_general_stamp_table_matches_library():
    assert np.array_equal(general_stamp(), netlist.GEN_STAMP)
    assert GEN_INTERNAL == 11 and netlist.GEN_NODES == 15 and general_stamp().shape[0] == 85


@pytest.mark.parametrize("case", list(CASES))
def test_topology_matches_reference_instances(case):
    """The internal variables the library lists per instance are the ones the reference's instances
    register (count and numbering), and the pattern holds every entry their stamps touch
    (OracleRun asserts the latter)."""
    c, cards, extra, flags = _circuit(case, n_mos=300)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards_, im, nd, params = family_inputs(c, cards, extra)
    orc = OracleRun(c, cards_, im, nd, params, rowptr, colind)
    assert orc.ref.n_unknowns == c.n_unknowns
    counts = np.array([orc.ref.num_internal(i) for i in range(c.n_mos)])
    assert np.array_equal(counts, flags.sum(1))
    # State slots: 3 + qgmid (rgateMod 3) + qbs, qbd (rbodyMod) + qcheq, qcdump (trnqsMod).
    assert orc.n_sta_slots == 8
    assert int((orc.sta_off >= 0).sum()) == orc.ref.n_state


def test_plain_family_refuses_nothing_and_needs_no_general_topology():
    c = netlist.random_logic(200, seed=3)
    cards, im, nd, params = family_inputs(c)
    flags, general = internal_nodes(cards, im, nd, params, general=True)
    assert not general and not flags.any()


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES))
def test_general_topology_parity(case):
    pytest.importorskip("torch")
    from tests.gpu_parity import run_sequence

    c, cards, extra, flags = _circuit(case)
    tran = [SolverFlags(newton_iter=1, voltlim=0), SolverFlags(newton_iter=1), SolverFlags(newton_iter=2),
            SolverFlags(newton_iter=0, init_tran=1), SolverFlags(newton_iter=1, init_tran=1),
            SolverFlags(newton_iter=3)]
    dc = [SolverFlags(dcop=1, transient=0, newton_iter=0, init_jct=1), SolverFlags(dcop=1, transient=0, newton_iter=1),
          SolverFlags(dcop=1, transient=0, tranop=1, newton_iter=2)]
    worst = run_sequence(c, cards, dc + tran, extra_params=extra, vrange=(-0.4, 1.6), seed=4)
    print(case, int(flags.sum()), "internal variables; worst error / tolerance:", worst)


def _ic_placement(rgate, rbody, nrd, nrs, ics):
    """Where the reference writes the initial-condition couplings of a 3-stage inverter ring whose
    instances all use (rgateMod, rbodyMod, NRD given, NRS given) and the initial conditions `ics`:
    the difference of its dF/dx in DC and in a time step (the couplings load only in DC, the branch
    current's diagonal only in a step; the rest of dF/dx is the same) as {(row, col): value}, and
    the same set placed in the branch currents' columns. Also the circuit and pattern."""
    from xyce_b200.device import SolverFlags as _F  # noqa: F401

    c0 = netlist.inverter_ring(3)
    n = c0.n_mos
    base = {"RGATEMOD": rgate, "RBODYMOD": rbody, "RSH": 10.0}
    extra = {}
    if nrd:
        extra["NRD"] = np.full(n, 1.0)
    if nrs:
        extra["NRS"] = np.full(n, 1.0)
    for name in ics:
        extra[name] = np.full(n, 0.3)
    cards, im, nd, params = family_inputs(c0, [ModelCard(False, dict(base)), ModelCard(True, dict(base))], extra)
    flags, _ = internal_nodes(cards, im, nd, params, general=True)
    c = netlist.with_internal_nodes(c0, flags)
    rowptr, colind = netlist.jacobian_pattern(c)
    orc = OracleRun(c, cards, im, nd, params, rowptr, colind)
    sol = np.random.default_rng(1).uniform(0.0, 1.0, c.n_unknowns)
    z8, z14 = np.zeros(8 * n), np.zeros(14 * n)
    dc = orc.load(SolverFlags(dcop=1, transient=0, newton_iter=1, voltlim=0), sol, z8, z8, z14, z14)
    tr = orc.load(SolverFlags(newton_iter=1, voltlim=0), sol, z8, z8, z14, z14)
    d = dc["dfdx"] - tr["dfdx"]
    prow = np.repeat(np.arange(c.n_unknowns), np.diff(rowptr))
    got = {(int(prow[k]), int(colind[k])): round(float(d[k])) for k in np.flatnonzero(np.abs(d) > 0.5)}
    loc = netlist.general_local_nodes(c)
    want = {}
    for i in range(n):
        for ic_node, term in ((12, 3), (13, 0), (14, 1)):  # (IBS, B), (IDS, D), (IGS, G)
            if loc[i, ic_node] < 0:
                continue
            for r_, c_, v in ((loc[i, term], loc[i, ic_node], 1), (loc[i, 2], loc[i, ic_node], -1),
                              (loc[i, ic_node], loc[i, term], 1), (loc[i, ic_node], loc[i, 2], -1),
                              (loc[i, ic_node], loc[i, ic_node], -1)):
                if r_ >= 0 and c_ >= 0:
                    want[(int(r_), int(c_))] = want.get((int(r_), int(c_)), 0) + v
    want = {k: v for k, v in want.items() if v != 0}
    return got, want, c, orc, sol


@pytest.mark.parametrize("rgate,rbody,nrd,nrs,ic,consistent", [
    (1, 0, 0, 0, "IC1", True), (2, 0, 0, 1, "IC3", True), (0, 1, 1, 1, "IC2", True), (3, 1, 1, 1, "IC1", True),
    (0, 1, 0, 1, "IC3", True), (3, 0, 0, 1, "IC2", True),
    (0, 1, 0, 0, "IC1", False), (3, 0, 0, 0, "IC3", False), (1, 1, 1, 0, "IC2", False), (2, 1, 0, 1, "IC1", False)])
def test_reference_ic_coupling_placement(rgate, rbody, nrd, nrs, ic, consistent):
    """The reference places an initial condition's couplings in row D (IC1 = VDS) and row S (every
    initial condition) in the branch current's column, except where that row absorbed its prime
    node's row (no drain' / source') while gate-mid or body-network nodes exist (rgateMod 3 or
    rbodyMod): there the coupling lands one column early, on the node before the branch current
    (its Jacobian offsets, MOSFET_B4 registerJacLIDs :5313-5400 over jacStampMap's merged rows,
    N_DEV_DeviceInstance.C:636-900). Its dF/dx is then not the derivative of its own F, which loads
    the coupling at the branch current (:16373-16401); the finite difference below shows it. The
    library places the couplings in the branch currents' columns always, so it equals the reference
    in the consistent configurations, which the parity tests use."""
    got, want, c, orc, sol = _ic_placement(rgate, rbody, nrd, nrs, [ic])
    assert (got == want) == consistent, (got, want)
    if not consistent:
        # A coupling the reference's dF/dx misplaces, against a finite difference of its own F
        # (linear in the branch current): F changes by the coupling in that row and column.
        miss = [k for k, v in want.items() if got.get(k, 0) != v and k[0] != k[1]]
        if not miss:
            return
        r_, c_ = miss[0]
        n = c.n_mos
        z8, z14 = np.zeros(8 * n), np.zeros(14 * n)
        fl = SolverFlags(dcop=1, transient=0, newton_iter=1, voltlim=0)
        x1 = sol.copy()
        x1[c_] += 1.0
        f0 = orc.load(fl, sol, z8, z8, z14, z14)["f"]
        f1 = orc.load(fl, x1, z8, z8, z14, z14)["f"]
        if c_ >= c.n_nodes + c.n_vsrc:  # a branch current: F is linear in it
            assert f1[r_] - f0[r_] == pytest.approx(want[(r_, c_)], abs=1e-9)


@pytest.mark.gpu
def test_general_launch_shapes_equal_bitwise():
    """Every launch shape of the general topology — fused, and split into the DC part and the
    charge-and-stamp part handing the general state over through the context's buffer — gives the
    same loads bit for bit over a flag sequence that takes each path of the hand-off (limiting off
    and on, the first transient step, junction initialisation, a DC load), NQS instances included."""
    pytest.importorskip("torch")
    from tests.gpu_parity import GpuRun
    from xyce_b200 import MosfetDevice, _native

    lib = _native.load()
    c, cards, extra, flags = _circuit("nqs_rgate", n_mos=3000, seed=5)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards_, im, nd, params = family_inputs(c, cards, extra)
    n = im.shape[0]
    seq = [SolverFlags(newton_iter=1, voltlim=0), SolverFlags(newton_iter=0, init_tran=1),
           SolverFlags(newton_iter=2), SolverFlags(dcop=1, transient=0, newton_iter=0, init_jct=1),
           SolverFlags(dcop=1, transient=0, tranop=1, newton_iter=1)]
    rng = np.random.default_rng(3)
    sols = [rng.uniform(-0.3, 1.5, c.n_unknowns) for _ in seq]
    shapes = [v for v in range(lib.xd_num_eval_variants()) if lib.xd_eval_variant_general(v) == 1]
    assert any(lib.xd_eval_variant_split(v) == 1 for v in shapes)
    outs = {}
    for v in shapes:
        dev = MosfetDevice(cards_, im, nd, params, (rowptr, colind), c.n_unknowns, inst_internal=c.mos_internal)
        assert dev._lib.xd_set_eval_variant(dev._h, v) == 0
        gpu = GpuRun(dev, int(rowptr[-1]), c.n_unknowns)
        ns = dev.n_state_slots
        sta_n, sta_c, sto_n, sto_c = np.zeros(ns * n), np.zeros(ns * n), np.zeros(14 * n), np.zeros(14 * n)
        res = []
        for fl, sol in zip(seq, sols):
            g = gpu.load(fl, sol, sta_n, sta_c, sto_n, sto_c)
            res.append(g)
            sta_n, sta_c, sto_n = g["next_sta"], g["curr_sta"], g["next_sto"]
        outs[v] = res
        dev.close()
    ref = outs[shapes[0]]
    for v in shapes[1:]:
        for step, (a, b) in enumerate(zip(ref, outs[v])):
            for k in a:
                if k != "abs":
                    assert np.array_equal(a[k], b[k], equal_nan=True), (v, step, k)
