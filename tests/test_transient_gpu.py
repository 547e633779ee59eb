"""The transient driver on the GPU (device loads by xd_load_assign, Newton matrix and residual by
xd_tia_combine) against the same driver on the oracle's loads: the combine kernel against its
numpy restatement, and node waveforms of a BSIM3 ring oscillator and of a BSIM4 gate netlist
with RC wires and PWL inputs, within reltol = 1e-3 / abstol = 1e-12 of the oracle's."""
import ctypes

import numpy as np
import pytest

from xyce_b200 import MosfetDevice, netlist
from xyce_b200.transient import GpuTransient, NewtonParams, tia_coef

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from tests.parity import family_inputs  # noqa: E402
from tests.transient_oracle import OracleTransient  # noqa: E402

# Tight Newton tolerances for the comparisons: both sides converge far below the waveform bound,
# so differences in iteration counts cannot show up as waveform differences.
TIGHT = NewtonParams(max_iter=40, rhs_tol=1e-9, delta_x_tol=1e-3, abs_tol=1e-9, rel_tol=1e-6,
                     update_weights_each_iter=False)
RELTOL, ABSTOL = 1e-3, 1e-12


def _pair(c, cards, level, extra=None):
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c, cards, extra)
    fam = MosfetDevice(cards, im, nd, params, (rowptr, colind), c.n_unknowns, level=level)
    g = GpuTransient(c, fam, rowptr, colind)
    o = OracleTransient(c, cards, rowptr, colind, level=level, extra_params=extra)
    return g, o


def _check_waves(tg, wg, to, wo):
    assert np.array_equal(tg, to), "time points differ"
    scale = np.abs(wo).max(axis=0, keepdims=True)
    err = np.abs(wg - wo)
    bound = RELTOL * scale + ABSTOL
    worst = float((err / bound).max())
    assert worst <= 1.0, f"waveforms differ: worst {worst:.3g}x of reltol/abstol"
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
    for mode, h, order in ((0, None, 1), (1, 1e-11, 1), (1, 3e-12, 2)):
        g._combine(mode, h, order, qn0, fh)
        x = g.x.cpu().numpy()
        A_f = o.Af
        jf = g.jf.cpu().numpy() + g.lin.lin_f
        F = g.f.cpu().numpy() + A_f @ x - g.b.cpu().numpy()
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
