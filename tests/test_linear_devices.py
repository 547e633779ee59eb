"""The circuits' linear devices against the reference's own resistor, capacitor and voltage-source
code (oracle: src/DeviceModelPKG/OpenModels/src/N_DEV_Resistor.C, N_DEV_Capacitor.C,
N_DEV_Vsrc.C and the piecewise-linear source data N_DEV_SourceData.C, compiled by
oracle/Makefile).

The transient drivers load the resistors, capacitors and independent sources of a gate netlist as
constant CSR stamps (``LinearDevices``: lin_f, lin_q) and a source vector b(t): F = lin_f x - b,
Q = lin_q x, dF/dx = lin_f, dQ/dx = lin_q. The reference's devices, loaded through the same device
calls as the MOSFETs, give F, Q, dF/dx and dQ/dx of the same devices at the same x and time; the
two must agree per entry (1e-12 relative plus 1e-14 of the entry's absolute sum, as for the
MOSFET loads), and the source values bit for bit — at the PWL points, between them, before the
first and after the last. Not probed: a time exactly equal to a source's last point, where the
reference's segment search finds no point later than the time and keeps the segment index of its
previous evaluation (PWLinData::updateSource, N_DEV_SourceData.C:1408-1425), so its value there
depends on the call history; the restatement takes the last segment. The GPU test does the same for the device-side source evaluation
(xd_pwl_eval) and for the combine's F and Q totals with the MOSFET contributions zero.
"""
import numpy as np
import pytest

from oracle import xyce_ref as xr
from xyce_b200 import SolverFlags, netlist
from xyce_b200.transient import LinearDevices

pytestmark = pytest.mark.skipif(not xr.available(), reason="oracle library not built")


class LinearOracle:
    """The reference's R, C and V devices of a circuit, each family on the circuit's pattern."""

    def __init__(self, c, rowptr, colind):
        nu = c.n_unknowns
        self.c, self.nu = c, nu
        self.fams = []
        if c.res_nodes.shape[0]:
            self.fams.append(xr.RefLinear("r", c.res_nodes, {"R": c.res_value}, nu))
        if c.cap_nodes.shape[0]:
            self.fams.append(xr.RefLinear("c", c.cap_nodes, {"C": c.cap_value}, nu))
        pwl = list(c.vsrc_pwl) + [None] * (c.n_vsrc - len(c.vsrc_pwl))
        # The sources' branch unknowns are their internal variables, after the nodes.
        self.fams.append(xr.RefLinear("v", c.vsrc_nodes, {"DCV0": c.vsrc_dc}, c.n_nodes, pwl=pwl))
        prow = np.repeat(np.arange(nu), np.diff(rowptr))
        for f in self.fams:
            assert f.n_unknowns == nu
            pairs = [np.stack([prow, colind], 1)]
            for i in range(f.n):
                sr, sc = f.stamp(i)
                pairs.append(np.stack([sr, sc], 1).astype(np.int64))
            pr = np.concatenate(pairs, 0)
            key = np.unique(pr[:, 0] * (nu + 1) + pr[:, 1])
            rows, cols = key // (nu + 1), (key % (nu + 1)).astype(np.int32)
            orp = np.zeros(nu + 2, dtype=np.int64)
            np.add.at(orp, rows + 1, 1)
            f.set_pattern(np.cumsum(orp).astype(np.int32), cols)
            f.map = np.searchsorted(rows * (nu + 1) + cols, prow * (nu + 1) + colind)

    def load(self, x, t):
        """F, Q, dF/dx, dQ/dx (on the circuit's pattern) summed over the three families, and each
        entry's absolute sum; t = None loads the DC source values."""
        nu = self.nu
        out = {k: np.zeros(nu) for k in ("f", "q")}
        out.update({k: np.zeros(len(self.fams[0].map)) for k in ("dfdx", "dqdx")})
        ab = {k: np.zeros_like(v) for k, v in out.items()}
        flags = xr.make_flags(**(vars(SolverFlags(dcop=1, transient=0)) if t is None else vars(SolverFlags())))
        s = np.zeros(nu + 1)
        s[:nu] = x
        for f in self.fams:
            f.set_time(0.0 if t is None else t)
            r = f.load(flags, s, np.zeros(1), np.zeros(1), np.zeros(1), np.zeros(1))
            for k, v in (("f", r.f[:nu]), ("q", r.q[:nu]), ("dfdx", r.dfdx[f.map]), ("dqdx", r.dqdx[f.map])):
                out[k] += v
                ab[k] += np.abs(v)
        return out, ab


def _circuit():
    c = netlist.random_logic(400, seed=13, n_inputs=8)
    rowptr, colind = netlist.jacobian_pattern(c)
    return c, rowptr, colind


def _close(name, a, b, ab):
    bad = np.abs(a - b) > 1e-12 * np.maximum(np.abs(a), np.abs(b)) + 1e-14 * ab
    assert not bad.any(), f"{name}: {int(bad.sum())} entries differ, first {np.flatnonzero(bad)[:5]}"


def test_linear_device_stamps_match_reference_devices():
    c, rowptr, colind = _circuit()
    lin = LinearDevices(c, rowptr, colind)
    orc = LinearOracle(c, rowptr, colind)
    rng = np.random.default_rng(4)
    times = sorted({float(t) for p in c.vsrc_pwl if p is not None for t in p[0]})
    last = {float(p[0][-1]) for p in c.vsrc_pwl if p is not None}
    inner = [t for t in times if t not in last and t > 0.0]
    probe = [None, 0.0, inner[0], inner[len(inner) // 2], 0.5 * (times[1] + times[2]), max(last) * 1.5]
    for t in probe:
        x = rng.uniform(-0.2, 1.4, c.n_unknowns)
        ref, ab = orc.load(x, t)
        b = np.zeros(c.n_unknowns)
        b[lin.branch] = lin.source_values(t)
        f = np.zeros(c.n_unknowns)
        q = np.zeros(c.n_unknowns)
        prow = np.repeat(np.arange(c.n_unknowns), np.diff(rowptr))
        np.add.at(f, prow, lin.lin_f * x[colind])
        np.add.at(q, prow, lin.lin_q * x[colind])
        f -= b
        _close("dfdx", lin.lin_f, ref["dfdx"], ab["dfdx"])
        _close("dqdx", lin.lin_q, ref["dqdx"], ab["dqdx"])
        _close("F", f, ref["f"], ab["f"] + np.abs(b) + np.abs(f))
        _close("Q", q, ref["q"], ab["q"] + np.abs(q))
        # Source values bit for bit: the branch rows' F at x = 0 is minus the source value.
        zero, _ = orc.load(np.zeros(c.n_unknowns), t)
        assert np.array_equal(-zero["f"][lin.branch], lin.source_values(t)), t


@pytest.mark.gpu
def test_device_sources_and_combine_match_reference_devices():
    import ctypes

    import torch

    from xyce_b200 import _native
    from xyce_b200.transient import tia_coef

    lib = _native.load()
    c, rowptr, colind = _circuit()
    lin = LinearDevices(c, rowptr, colind)
    orc = LinearOracle(c, rowptr, colind)
    nu, nnz = c.n_unknowns, int(rowptr[-1])
    counts = np.array([0 if p is None else len(p[0]) for p in c.vsrc_pwl], dtype=np.int32)
    tv = np.array([x for p in c.vsrc_pwl if p is not None for pair in zip(p[0], p[1]) for x in pair])
    rows = np.ascontiguousarray(lin.branch, dtype=np.int32)
    dc = np.ascontiguousarray(c.vsrc_dc, dtype=np.float64)
    pwl = ctypes.c_void_p()
    _native.check(lib.xd_pwl_create(c.n_vsrc, rows.ctypes.data_as(_native._ip), counts.ctypes.data_as(_native._ip),
                                    tv.ctypes.data_as(_native._dp), dc.ctypes.data_as(_native._dp), None, None, 0,
                                    ctypes.byref(pwl)), "xd_pwl_create")
    csr = _native.XdCsr(nu, rowptr.ctypes.data_as(_native._ip), colind.ctypes.data_as(_native._ip))
    tia = ctypes.c_void_p()
    _native.check(lib.xd_tia_create(ctypes.byref(csr), 0, ctypes.byref(tia)), "xd_tia_create")
    f64 = dict(dtype=torch.float64, device="cuda")
    T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), **f64)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    zn, zz = torch.zeros(nu, **f64), torch.zeros(nnz, **f64)
    lin_f, lin_q = T(lin.lin_f), T(lin.lin_q)
    times = sorted({float(t) for q in c.vsrc_pwl if q is not None for t in q[0]})
    last = {float(q[0][-1]) for q in c.vsrc_pwl if q is not None}
    inner = [t for t in times if t not in last and t > 0.0]
    rng = np.random.default_rng(5)
    for t in [None, 0.0, inner[0], inner[-1], 0.37 * (times[2] + times[3]), max(last) * 2.0]:
        b = torch.zeros(nu, **f64)
        _native.check(lib.xd_pwl_eval(pwl, 0.0 if t is None else t, 0 if t is None else 1, p(b), None), "xd_pwl_eval")
        torch.cuda.synchronize()
        want = np.zeros(nu)
        want[lin.branch] = lin.source_values(t)
        assert np.array_equal(b.cpu().numpy(), want), t
        x = rng.uniform(-0.2, 1.4, nu)
        ref, ab = orc.load(x, t)
        jac, rhs, qt, ft = torch.zeros(nnz, **f64), torch.zeros(nu, **f64), torch.zeros(nu, **f64), torch.zeros(nu, **f64)
        coef = tia_coef(1, 1e-11, 1)
        _native.check(lib.xd_tia_combine(tia, ctypes.byref(coef), p(T(x)), p(zz), p(zz), p(lin_f), p(lin_q), p(zn),
                                         p(zn), None, None, p(b), p(zn), None, p(jac), p(rhs), p(qt), p(ft), None),
                      "xd_tia_combine")
        torch.cuda.synchronize()
        _close("F", ft.cpu().numpy(), ref["f"], ab["f"] + np.abs(want))
        _close("Q", qt.cpu().numpy(), ref["q"], ab["q"])
        jw = coef.qscale * ref["dqdx"] + coef.fscale * ref["dfdx"]
        _close("J", jac.cpu().numpy(), jw, coef.qscale * ab["dqdx"] + ab["dfdx"])
    lib.xd_tia_destroy(tia)
    lib.xd_pwl_destroy(pwl)
