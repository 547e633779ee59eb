"""The fused device load and combine (xd_tia_load_combine) against the two calls it replaces,
xd_load_assign into the family's buffers followed by xd_tia_combine (GPU).

Both run on identical inputs; the Newton matrix, the residual, Q and F totals and the family's
vectors must be bit-identical, in DC mode with a gmin shunt, and in time-step mode with backward
Euler and trapezoid coefficients, with and without the limiter corrections. The circuit's supply
rail gives rows and entries with more contributions than the thread-per-entry path takes, so the
chunked path is covered too. A whole transient with the fused path reproduces the unfused
transient's waveforms bit for bit."""
import ctypes

import numpy as np
import pytest

from xyce_b200 import MosfetDevice, SolverFlags, _native, netlist

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from xyce_b200.transient import GpuTransient, LinearDevices, NewtonParams, tia_coef  # noqa: E402


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("mode,order,gshunt,limiter", [(0, 1, 1e-3, 1), (1, 1, 0.0, 1), (1, 2, 0.0, 0),
                                                       (1, 2, 0.0, 1)])
def test_fused_load_combine_bitwise(mode, order, gshunt, limiter):
    lib = _native.load()
    c = netlist.random_logic(12000, seed=31, n_inputs=16)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = netlist.mosfet_family(c)
    nu, nnz = c.n_unknowns, int(rowptr[-1])
    # Two fresh contexts: an evaluation advances the context's per-instance vgb memory (the next
    # load's vgb_orig), so the fused call gets a context that has not loaded yet, as the unfused one.
    fam = MosfetDevice(cards, im, nd, params, (rowptr, colind), nu)
    fam2 = MosfetDevice(cards, im, nd, params, (rowptr, colind), nu)
    assert lib.xd_set_eval_variant(fam2._h, lib.xd_get_eval_variant(fam._h)) == 0
    csr = _native.XdCsr(nu, rowptr.ctypes.data_as(_native._ip), colind.ctypes.data_as(_native._ip))
    tia = ctypes.c_void_p()
    _native.check(lib.xd_tia_create(ctypes.byref(csr), 0, ctypes.byref(tia)), "xd_tia_create")
    fused = ctypes.c_void_p()
    _native.check(lib.xd_tia_fused_create(tia, fam2._h, ctypes.byref(fused)), "xd_tia_fused_create")
    lin = LinearDevices(c, rowptr, colind)
    f64 = dict(dtype=torch.float64, device="cuda")
    T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), **f64)
    rng = np.random.default_rng(3)
    x = T(rng.uniform(-0.2, 1.4, nu))
    # b is per unknown: the sources' values on their branch rows, zero elsewhere.
    bvec = np.zeros(nu)
    bvec[lin.branch] = lin.source_values(0.3e-9)
    lin_f, lin_q, b = T(lin.lin_f), T(lin.lin_q), T(bvec)
    assert b.shape[0] == nu and lin_f.shape[0] == nnz
    qn0, fhist = T(rng.normal(0, 1e-15, nu)), T(rng.normal(0, 1e-4, nu))
    n = fam.n
    sets = []
    for _ in range(2):
        d = dict(nsta=torch.zeros(3 * n, **f64), csta=torch.zeros(3 * n, **f64), nsto=T(rng.uniform(0, 1, 14 * n)),
                 csto=torch.zeros(14 * n, **f64), f=torch.zeros(nu, **f64), q=torch.zeros(nu, **f64),
                 fx=torch.zeros(nu, **f64), qx=torch.zeros(nu, **f64), jf=torch.zeros(nnz, **f64),
                 jq=torch.zeros(nnz, **f64), jac=torch.zeros(nnz, **f64), rhs=torch.zeros(nu, **f64),
                 qtot=torch.zeros(nu, **f64), ftot=torch.zeros(nu, **f64))
        sets.append(d)
    sets[1]["nsto"].copy_(sets[0]["nsto"])
    flags = SolverFlags(newton_iter=1, dcop=int(mode == 0), transient=int(mode != 0), tranop=int(mode == 0))
    coef = tia_coef(mode, 2e-12, order, gshunt)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    a, f = sets
    cf = flags.to_c()
    _native.check(lib.xd_load_assign(fam._h, ctypes.byref(cf), _p(x), _p(a["nsta"]), _p(a["csta"]), _p(a["nsto"]),
                                     _p(a["csto"]), _p(a["f"]), _p(a["q"]), _p(a["fx"]), _p(a["qx"]), _p(a["jf"]),
                                     _p(a["jq"]), st), "xd_load_assign")
    _native.check(lib.xd_tia_combine(tia, ctypes.byref(coef), _p(x), _p(a["jf"]), _p(a["jq"]), _p(lin_f), _p(lin_q),
                                     _p(a["f"]), _p(a["q"]), _p(a["fx"]) if limiter else None,
                                     _p(a["qx"]) if limiter else None, _p(b), _p(qn0), _p(fhist), _p(a["jac"]),
                                     _p(a["rhs"]), _p(a["qtot"]), _p(a["ftot"]), st), "xd_tia_combine")
    _native.check(lib.xd_tia_load_combine(fused, ctypes.byref(cf), ctypes.byref(coef), _p(x), _p(f["nsta"]),
                                          _p(f["csta"]), _p(f["nsto"]), _p(f["csto"]), _p(f["f"]), _p(f["q"]),
                                          _p(f["fx"]), _p(f["qx"]), _p(f["jf"]), _p(f["jq"]), _p(lin_f), _p(lin_q),
                                          limiter, _p(b), _p(qn0), _p(fhist), _p(f["jac"]), _p(f["rhs"]),
                                          _p(f["qtot"]), _p(f["ftot"]), st), "xd_tia_load_combine")
    torch.cuda.synchronize()
    keys = ["jac", "rhs", "ftot", "f", "fx", "nsto"] + (["qtot", "q", "qx", "nsta"] if mode else [])
    for k in keys:
        assert torch.equal(a[k], f[k]), k
    assert float(a["jac"].abs().max()) > 0
    lib.xd_tia_fused_destroy(fused)
    lib.xd_tia_destroy(tia)
    fam.close()
    fam2.close()


def test_fused_transient_matches_unfused_bitwise():
    c = netlist.random_logic(1200, seed=7, n_inputs=16)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = netlist.mosfet_family(c)
    waves = {}
    for fused in (False, True):
        fam = MosfetDevice(cards, im, nd, params, (rowptr, colind), c.n_unknowns)
        g = GpuTransient(c, fam, rowptr, colind, fused=fused)
        g.dcop()
        _, waves[fused] = g.run(0.2e-9, 10e-12, params=NewtonParams.transient(), record=np.arange(c.n_nodes))
        g.close()
        fam.close()
    assert np.array_equal(waves[False], waves[True])
