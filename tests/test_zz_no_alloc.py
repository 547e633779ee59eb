"""The allocation-free load entry point against the regular one (GPU).

xd_load_static_scratch is for callers that cannot allocate device memory at load time (a solver
that gave all device memory to its own pool, or that runs its Newton loop under a fixed memory
budget): its scratch is a fixed array inside the library instead of context buffers. This test
calls it through the C ABI and checks that two loads in a row give the same F, Q, limiter
vectors, Jacobian values, state and store as xd_load on an identical second context, within
the parity tolerance. It also checks that a family larger than the array is refused.

The file name sorts last so that a run stopping at the first failure has run everything else.
"""
import ctypes

import numpy as np
import pytest

from tests.parity import ABS_SUM_FLOOR, RTOL, compare, family_inputs
from xyce_b200 import Bsim4Device, SolverFlags, _native, netlist

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

MAX_INSTANCES = 16384  # XD_STATIC_MAX_INSTANCES in include/xyce_devload.h


def _buffers(n, nu, nnz, sol):
    f64 = dict(dtype=torch.float64, device="cuda")
    return dict(sol=torch.as_tensor(sol, **f64), nsta=torch.zeros(3 * n, **f64), csta=torch.zeros(3 * n, **f64),
                nsto=torch.zeros(14 * n, **f64), csto=torch.zeros(14 * n, **f64), f=torch.zeros(nu, **f64),
                q=torch.zeros(nu, **f64), fx=torch.zeros(nu, **f64), qx=torch.zeros(nu, **f64),
                jf=torch.zeros(nnz, **f64), jq=torch.zeros(nnz, **f64))


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _outputs(b):
    return ("f", "q", "fx", "qx", "jf", "jq")


def test_static_scratch_load_matches_regular_load_twice():
    lib = _native.load()
    c = netlist.random_logic(6000, seed=77)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c)
    n, nu, nnz = im.shape[0], c.n_unknowns, int(rowptr[-1])
    assert n <= MAX_INSTANCES
    regular = Bsim4Device(cards, im, nd, params, (rowptr, colind), nu)
    static = Bsim4Device(cards, im, nd, params, (rowptr, colind), nu)
    rng = np.random.default_rng(5)
    sol1 = rng.uniform(0.0, 1.2, nu)
    sol2 = sol1 + rng.uniform(-0.3, 0.3, nu)
    a = _buffers(n, nu, nnz, sol1)
    b = _buffers(n, nu, nnz, sol1)
    stream = torch.cuda.current_stream()
    for call, (sol, flags) in enumerate([(sol1, SolverFlags(newton_iter=1)), (sol2, SolverFlags(newton_iter=2))]):
        for buf in (a, b):
            buf["sol"].copy_(torch.as_tensor(sol))
            for k in _outputs(buf):
                buf[k].zero_()
        regular.load(flags, a["sol"], a["nsta"], a["csta"], a["nsto"], a["csto"], a["f"], a["q"], a["fx"], a["qx"],
                     a["jf"], a["jq"])
        cflags = flags.to_c()
        rc = lib.xd_load_static_scratch(static._h, ctypes.byref(cflags), _p(b["sol"]), _p(b["nsta"]), _p(b["csta"]),
                                        _p(b["nsto"]), _p(b["csto"]), _p(b["f"]), _p(b["q"]), _p(b["fx"]),
                                        _p(b["qx"]), _p(b["jf"]), _p(b["jq"]), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.xd_last_error().decode()
        s = {k: torch.zeros_like(a[k]) for k in _outputs(a)}
        regular.load_abs(s["f"], s["q"], s["fx"], s["qx"], s["jf"], s["jq"])
        torch.cuda.synchronize()
        for k in _outputs(a):
            bad, worst = compare(k, b[k].cpu().numpy(), a[k].cpu().numpy(), s[k].cpu().numpy(), RTOL, ABS_SUM_FLOOR,
                                 rowptr=rowptr if k in ("jf", "jq") else None)
            assert bad == 0, f"call {call}: {k} differs from xd_load ({worst:.3g}x tolerance)"
        for k in ("nsta", "nsto"):
            bad, worst = compare(k, b[k].cpu().numpy(), a[k].cpu().numpy(), np.abs(a[k].cpu().numpy()).max(), RTOL,
                                 ABS_SUM_FLOOR)
            assert bad == 0, f"call {call}: {k} differs from xd_load ({worst:.3g}x tolerance)"
    regular.close()
    static.close()


def test_static_scratch_refuses_oversized_family():
    lib = _native.load()
    c = netlist.random_logic(MAX_INSTANCES + 2000, seed=78)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c)
    n, nu, nnz = im.shape[0], c.n_unknowns, int(rowptr[-1])
    assert n > MAX_INSTANCES
    dev = Bsim4Device(cards, im, nd, params, (rowptr, colind), nu)
    b = _buffers(n, nu, nnz, np.zeros(nu))
    cflags = SolverFlags().to_c()
    rc = lib.xd_load_static_scratch(dev._h, ctypes.byref(cflags), _p(b["sol"]), _p(b["nsta"]), _p(b["csta"]),
                                    _p(b["nsto"]), _p(b["csto"]), _p(b["f"]), _p(b["q"]), _p(b["fx"]), _p(b["qx"]),
                                    _p(b["jf"]), _p(b["jq"]), None)
    assert rc < 0
    assert "exceed" in lib.xd_last_error().decode()
    dev.close()
