"""The transient driver on the GPU (device loads by xd_load_assign, Newton matrix and residual by
xd_tia_combine) against the same driver on the oracle's loads: the combine kernel against its
numpy restatement, and node waveforms of a BSIM3 ring oscillator and of a BSIM4 gate netlist
with RC wires and PWL inputs, within reltol = 1e-3 of the oracle's (of each node's scale, and point
by point with the reference's 1e-6 V node tolerance)."""
import ctypes

import numpy as np
import pytest

from xyce_b200 import MosfetDevice, netlist
from xyce_b200.transient import GpuTransient, NewtonParams, tia_coef

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from tests.gpu_parity import waveform_errors  # noqa: E402
from tests.parity import family_inputs  # noqa: E402
from oracle.transient import OracleTransient  # noqa: E402

# Tight Newton tolerances for the comparisons: both sides converge far below the waveform bound,
# so differences in iteration counts cannot show up as waveform differences.
TIGHT = NewtonParams(max_iter=40, rhs_tol=1e-9, delta_x_tol=1e-3, abs_tol=1e-9, rel_tol=1e-6,
                     update_weights_each_iter=False)


def _pair(c, cards, level, extra=None):
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c, cards, extra)
    fam = MosfetDevice(cards, im, nd, params, (rowptr, colind), c.n_unknowns, level=level)
    g = GpuTransient(c, fam, rowptr, colind)
    o = OracleTransient(c, cards, rowptr, colind, level=level, extra_params=extra)
    return g, o


def _check_waves(tg, wg, to, wo):
    """Node waveforms within reltol of each node's scale and, point by point, within reltol of the
    value plus the reference's voltage tolerance (tests/gpu_parity.py waveform_errors)."""
    assert np.array_equal(tg, to), "time points differ"
    worst, point = waveform_errors(wg, wo)
    assert worst <= 1.0, f"waveforms differ: worst {worst:.3g}x of reltol x node scale"
    assert point <= 1.0, f"waveforms differ: worst {point:.3g}x of the per-point reltol / vntol bound"
    print("worst error / per-point bound", point)
    return worst


def test_combine_kernel_matches_numpy():
    c = netlist.random_logic(2000, seed=5)
    g, o = _pair(c, None, 14)
    rng = np.random.default_rng(1)
    nu, nnz = g.nu, g.nnz
    T = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    g.x.copy_(T(rng.uniform(0, 1.2, nu)))
    for buf in (g.f, g.q, g.jf, g.jq, g.b):
        buf.copy_(T(rng.standard_normal(buf.shape[0])))
    qn0, fh = T(rng.standard_normal(nu)), T(rng.standard_normal(nu))
    rows = np.repeat(np.arange(nu), np.diff(g.rowptr))
    diag = (rows == g.colind).astype(float)
    has_diag = np.zeros(nu)
    has_diag[rows[rows == g.colind]] = 1.0
    assert has_diag[:c.n_nodes].all() and not has_diag[c.n_nodes:].any()  # branch rows have no diagonal
    for mode, h, order, gsh in ((0, None, 1, 0.0), (1, 1e-11, 1, 0.0), (1, 3e-12, 2, 0.0), (0, None, 1, 1e-3)):
        g.gshunt = gsh
        g._combine(mode, h, order, qn0, fh)
        x = g.x.cpu().numpy()
        A_f = o.Af
        jf = g.jf.cpu().numpy() + g.lin.lin_f + gsh * diag
        F = g.f.cpu().numpy() + A_f @ x + gsh * has_diag * x - g.b.cpu().numpy()
        if mode == 0:
            jac, rhs = jf, -F
        else:
            cf = tia_coef(mode, h, order)
            jq = g.jq.cpu().numpy() + g.lin.lin_q
            Q = g.q.cpu().numpy() + o.Aq @ x
            jac = cf.qscale * jq + cf.fscale * jf
            rhs = -((Q - qn0.cpu().numpy()) * cf.inv_h + cf.fscale * F + cf.hist_scale * fh.cpu().numpy())
            assert np.allclose(g.qtot.cpu().numpy(), Q, rtol=1e-13, atol=1e-30)
        assert np.allclose(g.jac.cpu().numpy(), jac, rtol=1e-13, atol=1e-30), mode
        assert np.allclose(g.rhs.cpu().numpy(), rhs, rtol=1e-12, atol=1e-18 * np.abs(rhs).max()), mode
        assert np.allclose(g.ftot.cpu().numpy(), F, rtol=1e-12, atol=1e-18 * np.abs(F).max()), mode
    g.gshunt = 0.0
    g.close()


def test_ring_oscillator_bsim3_waveforms_match_oracle():
    """101-stage BSIM3 ring, VDD = 1.8 V, 5 fF per stage, 10 ps steps.

    Started from alternating rails (one stage inconsistent, so one edge travels round the ring),
    not from the operating point plus a kick: at the operating point every stage sits at its
    metastable point, where any rounding difference grows like exp(t / tau), tau = C / g_m ~ 50 ps,
    so two correct implementations part ways within ~2 ns whatever their accuracy."""
    c = netlist.inverter_ring(101, vdd=1.8)
    g, o = _pair(c, netlist.ring_bsim3_cards(), 9)
    rec = [1, 2, 26, 51, 76, 101]
    for s in (g, o):
        s.dcop()
        x0 = s.x.clone()
        x0[1:102] = torch.as_tensor(np.where(np.arange(1, 102) % 2 == 1, 1.8, 0.0), dtype=torch.float64)
        s.set_initial_state(x0)
    tg, wg = g.run(6e-9, 10e-12, params=TIGHT, record=rec)
    to, wo = o.run(6e-9, 10e-12, params=TIGHT, record=rec)
    worst = _check_waves(tg, wg, to, wo)
    # The ring is switching: node 1 has swung rail to rail within the window.
    assert wg[:, 0].max() > 1.7 and wg[:, 0].min() < 0.1
    print("ring: worst waveform error / bound", worst, "GPU Newton its/step", np.mean(g.stats.newton_iters))
    g.close()


def test_ring_oscillator_bsim3_kick_start_matches_oracle():
    """The ring on the configuration's own stimulus: the operating point, a 0.1 V kick on node 1,
    10 ps steps. Every stage starts at its metastable point, where rounding differences between two
    correct implementations grow like exp(t / tau), tau ~ 50 ps, so the comparison covers the first
    nanosecond (a 1e-16 difference grows ~5e8-fold by then, far inside the bound); the oscillation
    itself is compared from the alternating start above."""
    c = netlist.inverter_ring(101, vdd=1.8)
    g, o = _pair(c, netlist.ring_bsim3_cards(), 9)
    rec = [1, 2, 26, 51, 76, 101]
    for s in (g, o):
        s.dcop()
        x0 = s.x.clone()
        x0[1] += 0.1
        s.set_initial_state(x0)
    tg, wg = g.run(1e-9, 10e-12, params=TIGHT, record=rec)
    to, wo = o.run(1e-9, 10e-12, params=TIGHT, record=rec)
    worst = _check_waves(tg, wg, to, wo)
    # The kick has moved node 1 and its neighbour away from the operating point.
    assert np.abs(wg[-1, :2] - wg[0, :2]).max() > 1e-3
    print("ring kick: worst waveform error / bound", worst)
    g.close()


def test_gate_netlist_bsim4_waveforms_match_oracle():
    """BSIM4 INV/NAND2/NOR2 netlist with RC wires and 64 PWL inputs (50 ps edges), 1 ns."""
    c = netlist.random_logic(1200, seed=7, n_inputs=16)
    g, o = _pair(c, None, 14)
    rec = np.arange(0, c.n_nodes, max(1, c.n_nodes // 40))
    for s in (g, o):
        s.dcop()
    tg, wg = g.run(1e-9, 10e-12, params=TIGHT, record=rec)
    to, wo = o.run(1e-9, 10e-12, params=TIGHT, record=rec)
    worst = _check_waves(tg, wg, to, wo)
    print("gates: worst waveform error / bound", worst, "GPU Newton its/step", np.mean(g.stats.newton_iters))
    g.close()


def test_graph_replayed_newton_matches_eager_bitwise():
    """Each Newton iteration replayed as a CUDA graph computes exactly what the eager iteration
    does: same iteration counts, bit-identical waveforms (ring from the operating point plus a
    kick, reference transient tolerances, so the run includes step-size and order changes)."""
    c = netlist.inverter_ring(101, vdd=1.8)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c, netlist.ring_bsim3_cards())
    out = []
    for graphs in (False, True):
        fam = MosfetDevice(cards, im, nd, params, (rowptr, colind), c.n_unknowns, level=9)
        g = GpuTransient(c, fam, rowptr, colind, graphs=graphs)
        assert g.graphs == graphs
        g.dcop()
        x0 = g.x.clone()
        x0[1] += 0.1
        g.set_initial_state(x0)
        t, w = g.run(2e-9, 10e-12, record=np.arange(c.n_unknowns))
        out.append((t, w, list(g.stats.newton_iters), g.stats.wall_s))
        g.close()
        fam.close()
    assert out[0][2] == out[1][2]
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    print(f"ring 2 ns: eager {out[0][3]:.3f} s, graphs {out[1][3]:.3f} s")


def test_small_dense_solve_matches_numpy():
    """The one-SM dense solve (include/xyce_tia.h) against numpy on circuit-like sparse matrices
    (row pivoting needed: zero diagonals of source branch rows), a dense matrix, the size limit,
    a singular matrix (info set, solution not finite), and solves with kept factors."""
    from xyce_b200 import _native

    lib = _native.load()
    rng = np.random.default_rng(3)
    T = lambda a, dt=torch.float64: torch.as_tensor(a, dtype=dt, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    for n, density in ((1, 1.0), (7, 0.5), (33, 0.1), (103, 0.03), (160, 0.02), (150, 1.0)):
        A = np.where(rng.random((n, n)) < density, rng.standard_normal((n, n)), 0.0)
        A[np.arange(n), np.arange(n)] += np.where(rng.random(n) < 0.2, 0.0, 3.0)  # some zero diagonals
        A[np.arange(n), (np.arange(n) + 1) % n] += 1.0  # keeps it nonsingular with zero diagonals
        rows, cols = np.nonzero(np.ones((n, n)) if density == 1.0 else (A != 0) | np.eye(n, dtype=bool))
        rowptr = np.zeros(n + 1, np.int32)
        np.add.at(rowptr, rows + 1, 1)
        rowptr = np.cumsum(rowptr).astype(np.int32)
        colind = cols.astype(np.int32)
        csr = _native.XdCsr(n, rowptr.ctypes.data_as(_native._ip), colind.ctypes.data_as(_native._ip))
        h = ctypes.c_void_p()
        assert lib.xd_tia_create(ctypes.byref(csr), 0, ctypes.byref(h)) == 0
        vals, b = T(A[rows, cols]), T(rng.standard_normal(n))
        lu, piv, x, info = T(np.zeros(n * n)), T(np.zeros(n), torch.int32), T(np.zeros(n)), T([7], torch.int32)
        assert lib.xd_tia_dense_solve(h, p(vals), p(b), p(lu), p(piv), p(x), p(info), None) == 0
        torch.cuda.synchronize()
        ref = np.linalg.solve(A, b.cpu().numpy())
        err = np.abs(x.cpu().numpy() - ref).max() / np.abs(ref).max()
        assert int(info.item()) == 0 and err < 1e-10, (n, err)
        b2 = T(rng.standard_normal(n))
        x2 = T(np.zeros(n))
        assert lib.xd_tia_dense_resolve(h, p(lu), p(piv), p(b2), p(x2), None) == 0
        torch.cuda.synchronize()
        ref2 = np.linalg.solve(A, b2.cpu().numpy())
        assert np.abs(x2.cpu().numpy() - ref2).max() / np.abs(ref2).max() < 1e-10, n
        if n == 33:
            A0 = A.copy()
            A0[:, 5] = 0.0  # singular: column 5 has no pivot
            assert lib.xd_tia_dense_solve(h, p(T(A0[rows, cols])), p(b), None, None, p(x), p(info), None) == 0
            torch.cuda.synchronize()
            assert int(info.item()) > 0 and not np.isfinite(x.cpu().numpy()).all()
        lib.xd_tia_destroy(h)
    # Beyond the size limit the call is refused.
    n = _native.XD_DENSE_MAX_N + 1
    rowptr = np.arange(n + 1, dtype=np.int32)
    colind = np.arange(n, dtype=np.int32)
    csr = _native.XdCsr(n, rowptr.ctypes.data_as(_native._ip), colind.ctypes.data_as(_native._ip))
    h = ctypes.c_void_p()
    assert lib.xd_tia_create(ctypes.byref(csr), 0, ctypes.byref(h)) == 0
    v = T(np.ones(n))
    assert lib.xd_tia_dense_solve(h, p(v), p(v), None, None, p(v), None, None) < 0
    lib.xd_tia_destroy(h)


def test_static_pivot_small_solve_matches_numpy_and_falls_back():
    """The static-pivot solve (xd_slu_*): orders and fill from one matrix, later matrices of the
    same pattern solved without a pivot search, against numpy; factors kept for a chord solve
    (xd_slu_resolve); a matrix whose pivots fail the 1e-3 threshold test stops it (info = step + 1)
    and the pivoting solve queued behind it gives the right answer."""
    from xyce_b200 import _native

    lib = _native.load()
    rng = np.random.default_rng(11)
    T = lambda a, dt=torch.float64: torch.as_tensor(a, dtype=dt, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    for n, density in ((7, 0.5), (33, 0.1), (103, 0.03), (160, 0.02)):
        A = np.where(rng.random((n, n)) < density, rng.standard_normal((n, n)), 0.0)
        A[np.arange(n), np.arange(n)] += np.where(rng.random(n) < 0.2, 0.0, 3.0)
        A[np.arange(n), (np.arange(n) + 1) % n] += 1.0
        A[0, 0] = 2.0  # column 0 holds at least two entries (this and row n - 1's), for the fallback case
        mask = (A != 0) | np.eye(n, dtype=bool)
        rows, cols = np.nonzero(mask)
        rowptr = np.zeros(n + 1, np.int32)
        np.add.at(rowptr, rows + 1, 1)
        rowptr = np.cumsum(rowptr).astype(np.int32)
        colind = cols.astype(np.int32)
        csr = _native.XdCsr(n, rowptr.ctypes.data_as(_native._ip), colind.ctypes.data_as(_native._ip))
        tia, slu = ctypes.c_void_p(), ctypes.c_void_p()
        assert lib.xd_tia_create(ctypes.byref(csr), 0, ctypes.byref(tia)) == 0
        v0 = np.ascontiguousarray(A[rows, cols])
        assert lib.xd_slu_create(n, rowptr.ctypes.data_as(_native._ip), colind.ctypes.data_as(_native._ip),
                                 v0.ctypes.data_as(_native._dp), 1e-3, 0, ctypes.byref(slu)) == 0
        lu, piv, x, info = T(np.zeros(n * n)), T(np.zeros(n), torch.int32), T(np.zeros(n)), T([7], torch.int32)
        for k in range(3):
            Ak = np.where(mask, A * (1 + 0.05 * rng.standard_normal((n, n))), 0.0)
            b = T(rng.standard_normal(n))
            assert lib.xd_slu_solve(slu, p(T(Ak[rows, cols])), p(b), p(lu), p(x), p(info), None) == 0
            torch.cuda.synchronize()
            assert int(info.item()) == 0, (n, k)
            ref = np.linalg.solve(Ak, b.cpu().numpy())
            assert np.abs(x.cpu().numpy() - ref).max() / np.abs(ref).max() < 1e-10, (n, k)
            b2, x2 = T(rng.standard_normal(n)), T(np.zeros(n))
            assert lib.xd_slu_resolve(slu, p(lu), p(b2), p(x2), None) == 0
            torch.cuda.synchronize()
            ref2 = np.linalg.solve(Ak, b2.cpu().numpy())
            assert np.abs(x2.cpu().numpy() - ref2).max() / np.abs(ref2).max() < 1e-10, (n, k)
        # Entries rescaled by 10^U(-6, 6): some static pivot fails its threshold test (info > 0) and the
        # pivoting solve queued behind it answers; every attempt's answer is checked.
        failed = 0
        for attempt in range(20):
            A1 = np.where(mask, A * 10.0 ** rng.uniform(-6, 6, (n, n)), 0.0)
            b = T(rng.standard_normal(n))
            vals1 = T(A1[rows, cols])
            assert lib.xd_slu_solve(slu, p(vals1), p(b), p(lu), p(x), p(info), None) == 0
            assert lib.xd_tia_dense_solve_fallback(tia, p(vals1), p(b), p(lu), p(piv), p(x), p(info), None) == 0
            torch.cuda.synchronize()
            xs, bs = x.cpu().numpy(), b.cpu().numpy()
            berr = np.abs(A1 @ xs - bs).max() / (np.abs(A1).max() * np.abs(xs).max() + np.abs(bs).max())
            assert berr < 1e-13, (n, attempt, berr)  # backward error: A1 may be badly conditioned
            fb = T([0], torch.int32)
            assert lib.xd_slu_solve(slu, p(vals1), p(b), None, p(x), p(fb), None) == 0
            torch.cuda.synchronize()
            failed += int(fb.item()) > 0
            if failed:
                break
        assert failed, n
        info.fill_(0)
        # With info 0 on entry the fallback does nothing.
        x.fill_(123.0)
        assert lib.xd_tia_dense_solve_fallback(tia, p(vals1), p(b), p(lu), p(piv), p(x), p(info), None) == 0
        torch.cuda.synchronize()
        assert float(x[0].item()) == 123.0
        lib.xd_slu_destroy(slu)
        lib.xd_tia_destroy(tia)


def test_newton_update_and_residual_norm_kernels():
    """xd_tia_newton_update / xd_tia_residual_norm against numpy: the update, refreshed and kept
    weights, the weighted RMS norm, the residual's max norm, a non-finite residual reported as NaN
    and the flag passed through."""
    from xyce_b200 import _native

    lib = _native.load()
    rng = np.random.default_rng(5)
    T = lambda a, dt=torch.float64: torch.as_tensor(a, dtype=dt, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    for n in (1, 103, 5000):
        rowptr = np.arange(n + 1, dtype=np.int32)
        colind = np.arange(n, dtype=np.int32)
        csr = _native.XdCsr(n, rowptr.ctypes.data_as(_native._ip), colind.ctypes.data_as(_native._ip))
        h = ctypes.c_void_p()
        assert lib.xd_tia_create(ctypes.byref(csr), 0, ctypes.byref(h)) == 0
        x, dx, xref = rng.standard_normal(n), rng.standard_normal(n) * 1e-3, rng.standard_normal(n)
        w0 = 1e-3 * np.abs(xref) + 1e-6
        for upd in (0, 1):
            dx_, xref_ = T(dx), T(xref)
            xd, wd, norms = T(x), T(w0), T(np.zeros(3))
            assert lib.xd_tia_newton_update(h, p(xd), p(dx_), p(xref_), p(wd), 1e-3, 1e-6, upd, p(norms), None) == 0
            torch.cuda.synchronize()
            xn = x + dx
            wn = 1e-3 * np.maximum(np.abs(xref), np.abs(xn)) + 1e-6 if upd else w0
            assert np.array_equal(xd.cpu().numpy(), xn)
            assert np.array_equal(wd.cpu().numpy(), wn)
            ref = np.sqrt(np.mean((dx / wn) ** 2))
            assert abs(float(norms[0]) - ref) <= 1e-13 * ref
        rhs = rng.standard_normal(n)
        flag = T([3], torch.int32)
        norms = T(np.zeros(3))
        assert lib.xd_tia_residual_norm(h, p(T(rhs)), p(flag), p(norms), None) == 0
        torch.cuda.synchronize()
        assert float(norms[1]) == np.abs(rhs).max() and float(norms[2]) == 3.0
        rhs[n // 2] = np.nan
        assert lib.xd_tia_residual_norm(h, p(T(rhs)), None, p(norms), None) == 0
        torch.cuda.synchronize()
        assert np.isnan(float(norms[1])) and float(norms[2]) == 0.0
        lib.xd_tia_destroy(h)
