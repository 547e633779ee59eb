"""GPU sparse refactorization (include/xyce_rf.h) for the transient's Newton matrices: solutions
against scipy after refactoring with new values in the same pattern, and a transient with the
refactorization against the same transient with the dense GPU LU."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

from xyce_b200 import MosfetDevice, _native, netlist
from xyce_b200.transient import GpuTransient, NewtonParams

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from tests.gpu_parity import waveform_errors  # noqa: E402
from tests.parity import family_inputs  # noqa: E402


def _pair(c, solver):
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c, None)
    fam = MosfetDevice(cards, im, nd, params, (rowptr, colind), c.n_unknowns, level=14)
    return GpuTransient(c, fam, rowptr, colind, solver=solver), fam


def test_refactor_and_solve_match_scipy():
    c = netlist.random_logic(3000, seed=9)
    g, fam = _pair(c, "rf")
    rng = np.random.default_rng(0)
    rows = np.repeat(np.arange(g.nu), np.diff(g.rowptr))
    for k in range(3):
        vals = rng.uniform(-1e-3, 1e-3, g.nnz)
        vals[rows == g.colind] = rng.uniform(5e-3, 1e-2, int((rows == g.colind).sum()))
        g.jac.copy_(torch.as_tensor(vals, device="cuda"))
        b = rng.standard_normal(g.nu)
        g.rhs.copy_(torch.as_tensor(b, device="cuda"))
        x = g._solve().cpu().numpy()
        A = sp.csr_matrix((vals, g.colind, g.rowptr), shape=(g.nu, g.nu))
        res = np.abs(A @ x - b).max() / np.abs(b).max()
        assert res < 1e-9, (k, res)
    assert g.stats.host_factorizations == 1  # later matrices were refactored on the GPU
    g.close()
    fam.close()


def test_transient_with_gpu_refactorization_matches_dense():
    c = netlist.random_logic(800, seed=7, n_inputs=8)
    tight = NewtonParams(max_iter=40, rhs_tol=1e-9, delta_x_tol=1e-3, abs_tol=1e-9, rel_tol=1e-6,
                         update_weights_each_iter=False)
    # The default operating-point tolerances admit millivolt differences between two Newton paths
    # (deltaXTol 1 on relTol 1e-3 weights); tightened, both solvers land on the same point.
    tight_dc = NewtonParams(rhs_tol=1e-12, delta_x_tol=1e-3, abs_tol=1e-12, rel_tol=1e-6)
    waves = []
    for solver in ("dense", "rf"):
        g, fam = _pair(c, solver)
        g.dcop(tight_dc)
        _, w = g.run(0.5e-9, 10e-12, params=tight, record=np.arange(c.n_nodes))
        waves.append(w)
        if solver == "rf":
            # Most Newton matrices were refactored on the GPU, not factored on the host.
            assert g.stats.host_factorizations < g.stats.factorizations // 4, g.stats
        g.close()
        fam.close()
    assert np.abs(waves[0] - waves[1]).max() < 1e-8


def test_placed_netlist_transient_refactorization_matches_oracle():
    """A placed (locality-wired) BSIM4 gate netlist: operating point from the logic-level starting
    iterate, then 0.3 ns on the GPU refactorization path, against the same driver on the oracle's
    loads with a host LU; waveforms within reltol 1e-3 / abstol 1e-12."""
    from oracle.transient import OracleTransient

    c = netlist.random_logic(2500, seed=4, n_inputs=16, locality=64)
    tight = NewtonParams(max_iter=40, rhs_tol=1e-9, delta_x_tol=1e-3, abs_tol=1e-9, rel_tol=1e-6,
                         update_weights_each_iter=False)
    tight_dc = NewtonParams(rhs_tol=1e-12, delta_x_tol=1e-3, abs_tol=1e-12, rel_tol=1e-6)
    rec = np.arange(0, c.n_nodes, max(1, c.n_nodes // 50))
    x0 = netlist.logic_initial_guess(c)
    g, fam = _pair(c, "rf")
    rowptr, colind = netlist.jacobian_pattern(c)
    o = OracleTransient(c, None, rowptr, colind, level=14, solver="splu")
    waves = []
    for s in (g, o):
        s.dcop(tight_dc, x0=x0)
        waves.append(s.run(0.3e-9, 10e-12, params=tight, record=rec))
    (tg, wg), (to, wo) = waves
    assert np.array_equal(tg, to)
    worst, point = waveform_errors(wg, wo)
    assert worst <= 1.0 and point <= 1.0, (worst, point)
    assert g.stats.host_factorizations < g.stats.factorizations // 4, g.stats
    print("placed netlist: worst error / bound", worst, "per point", point, "host factorizations", g.stats.host_factorizations,
          "of", g.stats.factorizations)
    g.close()
    fam.close()


def test_triangular_solve_kernels_match_library_and_repeat_bitwise():
    """The library's own forward / back substitution (one warp per row, no level barriers) on a
    placed netlist's factors: the same solution as the refactorization library's solve to rounding,
    backward error at rounding level, and bit-identical results when repeated (its sums do not
    depend on the order in which rows finish)."""
    c = netlist.random_logic(20000, seed=5, locality=64)
    g, fam = _pair(c, "rf")
    rng = np.random.default_rng(1)
    rows = np.repeat(np.arange(g.nu), np.diff(g.rowptr))
    vals = rng.uniform(-1e-3, 1e-3, g.nnz)
    vals[rows == g.colind] = rng.uniform(5e-3, 1e-2, int((rows == g.colind).sum()))
    g.jac.copy_(torch.as_tensor(vals, device="cuda"))
    g.rhs.copy_(torch.as_tensor(rng.standard_normal(g.nu), device="cuda"))
    g._solve()  # host factorization of this matrix, refactorization set up
    b = rng.standard_normal(g.nu)
    outs = []
    for fn in ("xd_rf_solve", "xd_rf_solve", "xd_rf_solve_library"):
        x = torch.as_tensor(b, device="cuda").clone()
        torch.cuda.synchronize()
        _native.check(getattr(g._lib, fn)(g._rf, ctypes.c_void_p(x.data_ptr())), fn)
        torch.cuda.synchronize()
        outs.append(x.cpu().numpy())
    A = sp.csr_matrix((vals, g.colind, g.rowptr), shape=(g.nu, g.nu))
    for x in outs:
        berr = np.max(np.abs(b - A @ x) / (abs(A) @ np.abs(x) + np.abs(b)))
        assert berr < 1e-13, berr
    assert np.array_equal(outs[0], outs[1])
    assert np.max(np.abs(outs[0] - outs[2])) <= 1e-11 * np.max(np.abs(outs[2]))
    g.close()
    fam.close()


def _diag_dominant(g, seed):
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(g.nu), np.diff(g.rowptr))
    vals = rng.uniform(-1e-3, 1e-3, g.nnz)
    vals[rows == g.colind] = rng.uniform(5e-3, 1e-2, int((rows == g.colind).sum()))
    return vals


def test_own_refactorization_matches_library_and_repeats_bitwise():
    """The library's own refactorization (xd_rf_refactor: right-looking over pivot levels)
    against cuSOLVER's (xd_rf_refactor_library) on a placed netlist's pattern with new values in
    the kept pivot order: the same solution to rounding, backward error at rounding level, and
    bit-identical factors when repeated."""
    c = netlist.random_logic(20000, seed=5, locality=64)
    g, fam = _pair(c, "rf")
    vals = _diag_dominant(g, 1)
    g.jac.copy_(torch.as_tensor(vals, device="cuda"))
    g.rhs.copy_(torch.as_tensor(np.ones(g.nu), device="cuda"))
    g._solve()  # host factorization of this matrix, refactorization set up
    nnz_f, nlev, nupd = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
    _native.check(g._lib.xd_rf_stats(g._rf, ctypes.byref(nnz_f), ctypes.byref(nlev), ctypes.byref(nupd)), "xd_rf_stats")
    vals2 = _diag_dominant(g, 2)
    d2 = torch.as_tensor(vals2, device="cuda")
    b = np.random.default_rng(3).standard_normal(g.nu)
    A = sp.csr_matrix((vals2, g.colind, g.rowptr), shape=(g.nu, g.nu))
    facs, xs = [], []
    for fn, solve in (("xd_rf_refactor", "xd_rf_solve"), ("xd_rf_refactor", "xd_rf_solve"),
                      ("xd_rf_refactor_library", "xd_rf_solve_library")):
        torch.cuda.synchronize()
        _native.check(getattr(g._lib, fn)(g._rf, ctypes.c_void_p(d2.data_ptr())), fn)
        if fn == "xd_rf_refactor":
            f = np.zeros(nnz_f.value)
            _native.check(g._lib.xd_rf_copy_factors(g._rf, f.ctypes.data_as(_native._dp)), "xd_rf_copy_factors")
            facs.append(f)
        x = torch.as_tensor(b, device="cuda").clone()
        torch.cuda.synchronize()
        _native.check(getattr(g._lib, solve)(g._rf, ctypes.c_void_p(x.data_ptr())), solve)
        torch.cuda.synchronize()
        xs.append(x.cpu().numpy())
    # New values in the kept pivot order: backward errors at rounding level, the same for both.
    berrs = [np.max(np.abs(b - A @ x) / (abs(A) @ np.abs(x) + np.abs(b))) for x in xs]
    assert max(berrs) < 1e-11, berrs
    assert berrs[0] < 10 * berrs[2] + 1e-15, berrs
    assert np.array_equal(facs[0], facs[1])
    assert np.array_equal(xs[0], xs[1])
    assert np.max(np.abs(xs[0] - xs[2])) <= 1e-11 * np.max(np.abs(xs[2]))
    print(f"factors {nnz_f.value} entries, {nlev.value} elimination levels, {nupd.value} updates")
    g.close()
    fam.close()


def test_own_refactorization_reports_a_zero_pivot():
    """A matrix whose first pivot in the kept order is exactly zero: xd_rf_refactor returns an
    error (the transient driver then factors afresh on the host) instead of factors with infinities."""
    c = netlist.random_logic(2000, seed=8, locality=64)
    g, fam = _pair(c, "rf")
    vals = _diag_dominant(g, 4)
    g.jac.copy_(torch.as_tensor(vals, device="cuda"))
    g.rhs.copy_(torch.as_tensor(np.ones(g.nu), device="cuda"))
    g._solve()
    P, Q = g._rf_keep[9], g._rf_keep[10]
    r, col = int(P[0]), int(Q[0])
    k = g.rowptr[r] + int(np.flatnonzero(g.colind[g.rowptr[r]:g.rowptr[r + 1]] == col)[0])
    bad = vals.copy()
    bad[k] = 0.0
    d = torch.as_tensor(bad, device="cuda")
    torch.cuda.synchronize()
    rc = g._lib.xd_rf_refactor(g._rf, ctypes.c_void_p(d.data_ptr()))
    assert rc < 0
    assert "zero pivot in row 0" in g._lib.xd_last_error().decode()
    # The same object refactors a good matrix afterwards.
    d.copy_(torch.as_tensor(vals, device="cuda"))
    torch.cuda.synchronize()
    assert g._lib.xd_rf_refactor(g._rf, ctypes.c_void_p(d.data_ptr())) == 0
    g.close()
    fam.close()
