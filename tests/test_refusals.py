"""Host-side set-up refuses the model options the B200 load does not implement, before any device
memory is touched (so these run without a GPU). A refused card must never fall back to another
implementation: xd_create returns an error and the Python mirror raises."""
import numpy as np
import pytest

from xyce_b200 import ModelCard, MosfetDevice, netlist
from xyce_b200._native import NativeError


def _make(level, cards, extra=None):
    c = netlist.inverter_ring(5)
    rowptr, colind = netlist.jacobian_pattern(c)
    params = {"L": c.mos_l.astype(float), "W": c.mos_w.astype(float)}
    if extra:
        params.update({k: np.full(c.n_mos, v) for k, v in extra.items()})
    return MosfetDevice(cards, c.mos_type, c.mos_nodes, params, (rowptr, colind), c.n_unknowns, level=level)


NMOS_PMOS = [ModelCard(False, {}), ModelCard(True, {})]


@pytest.mark.parametrize("level,cards,extra,match", [
    (3, NMOS_PMOS, None, "not implemented"),
    # Gate resistance is loaded through the general topology: without its internal unknowns the
    # family is refused, naming the field that carries them.
    (14, [ModelCard(False, {"RGATEMOD": 1}), ModelCard(True, {})], None, "inst_internal_gen"),
    (14, [ModelCard(False, {"RGATEMOD": 4}), ModelCard(True, {})], None, "rgateMod must be 0, 1, 2 or 3"),
    (14, [ModelCard(False, {"RBODYMOD": 3}), ModelCard(True, {})], None, "rbodyMod must be 0, 1 or 2"),
    (14, [ModelCard(False, {"RDSMOD": 2}), ModelCard(True, {})], None, "rdsMod must be 0 or 1"),
    # The NQS charge node is a general-topology internal variable too.
    (14, [ModelCard(False, {"TRNQSMOD": 1}), ModelCard(True, {})], None, "inst_internal_gen"),
    (14, [ModelCard(False, {"TRNQSMOD": 2}), ModelCard(True, {})], None, "trnqsMod must be 0 or 1"),
    (14, NMOS_PMOS, {"IC3": 0.2}, "inst_internal_gen"),
    (14, [ModelCard(False, {"CAPMOD": 3}), ModelCard(True, {})], None, "capMod must be 0, 1 or 2"),
    (14, [ModelCard(False, {"IGCMOD": 3}), ModelCard(True, {})], None, "igcMod must be 0, 1 or 2"),
    (14, [ModelCard(False, {}), ModelCard(True, {"IGBMOD": 2})], None, "igbMod must be 0 or 1"),
    (14, [ModelCard(False, {"RSH": 10.0}), ModelCard(True, {})], {"RGEOMOD": 1}, "rgeoMod"),
    (14, [ModelCard(False, {"RSH": 10.0}), ModelCard(True, {"RSH": 5.0})], {"NRD": 2.0, "NRS": 1.5},
     "inst_internal"),
    (14, [ModelCard(False, {"NOSUCH": 1.0}), ModelCard(True, {})], None, "unknown BSIM4 model parameter"),
    (9, [ModelCard(False, {"CAPMOD": 4}), ModelCard(True, {})], None, "capMod"),
    (9, [ModelCard(False, {"RSH": 10.0}), ModelCard(True, {})], None, "inst_internal"),
    (9, NMOS_PMOS, {"NQSMOD": 1}, "nqsMod"),
    (9, NMOS_PMOS, {"IC1": 0.5}, "initial conditions"),
    (9, [ModelCard(False, {"NPEAK": 1e17}), ModelCard(True, {})], None, "unknown BSIM3 model parameter NPEAK"),
    (1, [ModelCard(False, {"RD": 10.0}), ModelCard(True, {})], None, "inst_internal"),
    (1, [ModelCard(False, {"RSH": 10.0}), ModelCard(True, {})], {"NRD": 0.0}, "infinite series conductance"),
    (1, NMOS_PMOS, {"IC2": 0.5}, "initial conditions"),
])
def test_unsupported_option_is_refused(level, cards, extra, match):
    with pytest.raises(NativeError, match=match):
        _make(level, cards, extra)


def test_mixed_instance_temperatures_are_refused():
    c = netlist.inverter_ring(5)
    rowptr, colind = netlist.jacobian_pattern(c)
    temp = np.where(np.arange(c.n_mos) % 4 < 2, 27.0, 60.0)
    for level in (9, 14):
        params = {"L": c.mos_l.astype(float), "W": c.mos_w.astype(float), "TEMP": temp}
        # Instances alternate PMOS / NMOS, so each model's instances see both temperatures.
        with pytest.raises(NativeError, match="share one temperature"):
            MosfetDevice(NMOS_PMOS, c.mos_type, c.mos_nodes, params, (rowptr, colind), c.n_unknowns, level=level)


def test_internal_node_query_follows_sheet_resistance():
    """RSH with NRD / NRS > 0 gives an instance internal drain / source nodes; without RSH, or
    with zero squares, the node collapses (the reference's createNode rule)."""
    from xyce_b200.device import internal_nodes

    c = netlist.inverter_ring(5)
    n = c.n_mos
    cards = [ModelCard(False, {"RSH": 10.0}), ModelCard(True, {})]
    nrd = np.where(np.arange(n) % 3 == 0, 2.0, np.where(np.arange(n) % 3 == 1, 0.0, np.nan))
    params = {"L": c.mos_l.astype(float), "W": c.mos_w.astype(float), "NRD": nrd, "NRS": np.full(n, 1.0)}
    flags = internal_nodes(cards, c.mos_type, c.mos_nodes, params)
    nmos = c.mos_type == 0
    assert (flags[:, 0] == (nmos & (np.arange(n) % 3 == 0))).all()
    assert (flags[:, 1] == nmos).all()
    c2 = netlist.with_internal_nodes(c, flags)
    assert c2.n_unknowns == c.n_unknowns + int(flags.sum())
    got = c2.mos_internal[flags]
    assert (np.sort(got) == np.arange(c.n_unknowns, c2.n_unknowns)).all()
    rowptr, colind = netlist.jacobian_pattern(c2)
    assert rowptr.shape[0] == c2.n_unknowns + 1


def test_internal_node_query_bsim3():
    """BSIM3 gives an instance internal nodes whenever RSH times the squares (1 by default) is
    positive (N_DEV_MOSFET_B3.C:1849-1865)."""
    from xyce_b200.device import internal_nodes

    c = netlist.inverter_ring(5)
    n = c.n_mos
    cards = [ModelCard(False, {"RSH": 10.0}), ModelCard(True, {})]
    params = {"L": c.mos_l.astype(float), "W": c.mos_w.astype(float),
              "NRS": np.where(np.arange(n) % 2 == 0, 0.0, 2.0)}
    flags = internal_nodes(cards, c.mos_type, c.mos_nodes, params, level=9)
    nmos = c.mos_type == 0
    assert (flags[:, 0] == nmos).all()
    assert (flags[:, 1] == (nmos & (np.arange(n) % 2 == 1))).all()


def test_internal_node_query_mos1():
    """MOSFET1: RD / RS give the node whatever the squares; otherwise RSH x NRD / NRS (1 by
    default) does; with neither the node collapses (N_DEV_MOSFET1.C:1180-1220)."""
    from xyce_b200.device import internal_nodes

    c = netlist.inverter_ring(5)
    n = c.n_mos
    cards = [ModelCard(False, {"RD": 10.0}), ModelCard(True, {"RSH": 20.0})]
    params = {"L": c.mos_l.astype(float), "W": c.mos_w.astype(float), "NRS": np.full(n, 2.0)}
    flags = internal_nodes(cards, c.mos_type, c.mos_nodes, params, level=1)
    nmos = c.mos_type == 0
    assert (flags[:, 0] == True).all()  # noqa: E712
    assert (flags[:, 1] == ~nmos).all()
    none = internal_nodes(NMOS_PMOS, c.mos_type, c.mos_nodes, params, level=1)
    assert not none.any()


def test_static_pivot_setup_refuses_bad_systems():
    """xd_slu_create checks its arguments and factors on the host before touching a GPU: sizes
    outside 1..XD_DENSE_MAX_N, a bad threshold, a malformed pattern and a singular matrix are
    refused with an error."""
    import ctypes

    from xyce_b200 import _native

    lib = _native.load()

    def create(n, rowptr, colind, vals, tol=1e-3):
        rp = np.ascontiguousarray(rowptr, np.int32)
        ci = np.ascontiguousarray(colind, np.int32)
        v = np.ascontiguousarray(vals, np.float64)
        h = ctypes.c_void_p()
        rc = lib.xd_slu_create(n, rp.ctypes.data_as(_native._ip), ci.ctypes.data_as(_native._ip),
                               v.ctypes.data_as(_native._dp), tol, 0, ctypes.byref(h))
        return rc, lib.xd_last_error().decode()

    eye = lambda n: (np.arange(n + 1), np.arange(n), np.ones(n))
    n = _native.XD_DENSE_MAX_N + 1
    rc, msg = create(n, *eye(n))
    assert rc < 0 and "n must be" in msg
    rc, msg = create(4, *eye(4), tol=0.0)
    assert rc < 0 and "tol" in msg
    rc, msg = create(2, [0, 1, 2], [0, 5], [1.0, 1.0])
    assert rc < 0 and "CSR" in msg
    # Two identical rows: singular.
    rc, msg = create(2, [0, 2, 4], [0, 1, 0, 1], [1.0, 2.0, 1.0, 2.0])
    assert rc == -2 and "singular" in msg
