"""The allocation-free load entry point against the regular one (GPU).

xd_load_static_scratch is for callers that cannot allocate device memory at load time (a solver
that gave all device memory to its own pool, or that runs its Newton loop under a fixed memory
budget): its scratch is a fixed array inside the library instead of context buffers. This test
calls it through the C ABI and checks that two loads in a row give bit-identical F, Q, limiter
vectors, Jacobian values, state and store to xd_load on an identical second context pinned to the
same evaluation launch shape (the two run the same kernels over the same gather map in the same
order), for a BSIM4, a BSIM3 and a MOSFET1 family. It also checks that a family larger than the
array, and a family with internal drain / source nodes, are refused, and that the calls that read
the context's own staged stamps refuse to run after a static load.

The file name sorts last so that a run stopping at the first failure has run everything else.
"""
import ctypes

import numpy as np
import pytest

from tests.parity import family_inputs
from xyce_b200 import ModelCard, MosfetDevice, SolverFlags, _native, netlist
from xyce_b200.device import internal_nodes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

MAX_INSTANCES = 16384  # XD_STATIC_MAX_INSTANCES in include/xyce_devload.h
OUTPUTS = ("f", "q", "fx", "qx", "jf", "jq")


def _buffers(dev, nu, nnz, sol):
    f64 = dict(dtype=torch.float64, device="cuda")
    return dict(sol=torch.as_tensor(sol, **f64), nsta=torch.zeros(dev.n_state, **f64),
                csta=torch.zeros(dev.n_state, **f64), nsto=torch.zeros(dev.n_store, **f64),
                csto=torch.zeros(dev.n_store, **f64), f=torch.zeros(nu, **f64), q=torch.zeros(nu, **f64),
                fx=torch.zeros(nu, **f64), qx=torch.zeros(nu, **f64), jf=torch.zeros(nnz, **f64),
                jq=torch.zeros(nnz, **f64))


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _static_load(lib, dev, flags, b, stream=None):
    cflags = flags.to_c()
    return lib.xd_load_static_scratch(dev._h, ctypes.byref(cflags), _p(b["sol"]), _p(b["nsta"]), _p(b["csta"]),
                                      _p(b["nsto"]), _p(b["csto"]), _p(b["f"]), _p(b["q"]), _p(b["fx"]),
                                      _p(b["qx"]), _p(b["jf"]), _p(b["jq"]), stream)


FAMILIES = {
    "bsim4": (14, None, 6000),
    "bsim3": (9, netlist.ring_bsim3_cards, 3000),
    "mosfet1": (1, lambda: [ModelCard(False, {}), ModelCard(True, {})], 3000),
}


@pytest.mark.parametrize("family", list(FAMILIES))
def test_static_scratch_load_matches_regular_load_twice(family):
    level, mk_cards, size = FAMILIES[family]
    lib = _native.load()
    c = netlist.random_logic(size, seed=77)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c, mk_cards() if mk_cards else None)
    n, nu, nnz = im.shape[0], c.n_unknowns, int(rowptr[-1])
    assert n <= MAX_INSTANCES
    regular = MosfetDevice(cards, im, nd, params, (rowptr, colind), nu, level=level)
    static = MosfetDevice(cards, im, nd, params, (rowptr, colind), nu, level=level)
    # Same launch shape on both contexts, so the comparison can be exact.
    assert lib.xd_set_eval_variant(static._h, lib.xd_get_eval_variant(regular._h)) == 0
    rng = np.random.default_rng(5)
    sol1 = rng.uniform(0.0, 1.2, nu)
    sol2 = sol1 + rng.uniform(-0.3, 0.3, nu)
    a = _buffers(regular, nu, nnz, sol1)
    b = _buffers(static, nu, nnz, sol1)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # A transient's first step (initTran, Newton step 0: the current state is written too), then a
    # later Newton iteration at a moved iterate.
    seq = [(sol1, SolverFlags(newton_iter=0, init_tran=1)), (sol2, SolverFlags(newton_iter=2))]
    for call, (sol, flags) in enumerate(seq):
        for buf in (a, b):
            buf["sol"].copy_(torch.as_tensor(sol))
            for k in OUTPUTS:
                buf[k].zero_()
        regular.load(flags, a["sol"], a["nsta"], a["csta"], a["nsto"], a["csto"], a["f"], a["q"], a["fx"], a["qx"],
                     a["jf"], a["jq"])
        rc = _static_load(lib, static, flags, b, stream)
        assert rc == 0, lib.xd_last_error().decode()
        torch.cuda.synchronize()
        for k in OUTPUTS + ("nsta", "nsto", "csta"):
            assert torch.equal(a[k], b[k]), f"{family} call {call}: {k} differs from xd_load"
        assert bool(torch.isfinite(b["f"]).all()) and bool(b["jf"].abs().sum() > 0)
    regular.close()
    static.close()


def test_stage_reading_calls_refuse_after_a_static_load():
    """A static load leaves its staged stamps in the library's array, not in the context: the
    calls that read the context's staged stamps refuse until the next xd_update_state."""
    lib = _native.load()
    c = netlist.random_logic(2000, seed=79)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c)
    nu, nnz = c.n_unknowns, int(rowptr[-1])
    dev = MosfetDevice(cards, im, nd, params, (rowptr, colind), nu)
    b = _buffers(dev, nu, nnz, np.random.default_rng(1).uniform(0.0, 1.2, nu))
    assert _static_load(lib, dev, SolverFlags(newton_iter=1), b) == 0
    with pytest.raises(_native.NativeError, match="static"):
        dev.load_dae_vectors(b["f"], b["q"], b["fx"], b["qx"])
    with pytest.raises(_native.NativeError, match="static"):
        dev.load_abs(b["f"], b["q"], b["fx"], b["qx"], b["jf"], b["jq"])
    dev.update_state(SolverFlags(newton_iter=1), b["sol"], b["nsta"], b["csta"], b["nsto"], b["csto"])
    dev.load_dae_vectors(b["f"], b["q"], b["fx"], b["qx"])
    torch.cuda.synchronize()
    dev.close()


def test_static_scratch_refuses_oversized_family():
    lib = _native.load()
    c = netlist.random_logic(MAX_INSTANCES + 2000, seed=78)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c)
    n, nu, nnz = im.shape[0], c.n_unknowns, int(rowptr[-1])
    assert n > MAX_INSTANCES
    dev = MosfetDevice(cards, im, nd, params, (rowptr, colind), nu)
    b = _buffers(dev, nu, nnz, np.zeros(nu))
    assert _static_load(lib, dev, SolverFlags(), b) < 0
    assert "exceed" in lib.xd_last_error().decode()
    dev.close()


def test_static_scratch_refuses_internal_node_family():
    """Families with internal drain / source nodes stage a wider layout than the array holds."""
    lib = _native.load()
    c = netlist.random_logic(1500, seed=51)
    n = c.n_mos
    cards = [ModelCard(False, {"RSH": 25.0}), ModelCard(True, {"RSH": 40.0})]
    extra = {"NRD": np.full(n, 2.0), "NRS": np.full(n, 1.5)}
    cards_, im, nd, params = family_inputs(c, cards, extra)
    flags = internal_nodes(cards_, im, nd, params)
    c2 = netlist.with_internal_nodes(c, flags)
    rowptr, colind = netlist.jacobian_pattern(c2)
    dev = MosfetDevice(cards_, im, nd, params, (rowptr, colind), c2.n_unknowns, inst_internal=c2.mos_internal)
    b = _buffers(dev, c2.n_unknowns, int(rowptr[-1]), np.zeros(c2.n_unknowns))
    assert _static_load(lib, dev, SolverFlags(), b) < 0
    assert "internal" in lib.xd_last_error().decode()
    dev.close()
