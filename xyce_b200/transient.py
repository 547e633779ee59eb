"""Transient analysis on the B200 device loads: the callers either side of the hot path.

Restates, for the circuits this package generates (MOSFETs of one family, resistors, capacitors,
DC and piecewise-linear voltage sources), the reference's transient driver:

* linear devices — resistor, capacitor and independent voltage source loads
  (src/DeviceModelPKG/OpenModels/src/N_DEV_Resistor.C:1075-1161, N_DEV_Capacitor.C:1821-2002,
  N_DEV_Vsrc.C:941-1028); their dF/dx and dQ/dx do not depend on the solution, so they are
  assembled once as CSR value arrays, and source values enter through b(t). PWL sources follow
  PWLinData::updateSource (src/DeviceModelPKG/Core/src/N_DEV_SourceData.C:1371-1480).
* the one-step integrator (N_TIA_OneStep.C: backward Euler on the first step after the operating
  point, trapezoid after it), its Jacobian J = (1/h) dQ/dx + f dF/dx and residual with the
  devices' voltage-limiter corrections (N_TIA_OneStep.C:272-336, 470-497) — formed on the GPU by
  ``xd_tia_combine``.
* the damped-Newton loop with its convergence test (N_NLS_DampedNewton.C:485-600, 1792-1900) and
  the parameters the reference uses for DC operating points and for transient steps
  (N_NLS_NLParams.C:90-160).

Every device load and the combine run as CUDA kernels on device-resident buffers; the host only
sees two scalars per Newton iteration (the residual's max norm and the update's weighted norm).
The linear system is solved by a dense LU on the GPU for small circuits, by GPU sparse
refactorization (one host factorization fixes pivots and fill, ``xd_rf_*`` refactors every later
matrix on the device) or by a host sparse LU (SuperLU through scipy): the linear solve is outside
the device-load path.

Step control is fixed-step (the largest step the analysis allows), halving on Newton failure.
"""
from __future__ import annotations

import ctypes
import math
import warnings
import time as _time
from dataclasses import dataclass, field

import numpy as np

from . import _native
from .device import MosfetDevice, SolverFlags


@dataclass
class NewtonParams:
    """N_NLS_NLParams defaults: DC operating point, and the transient overrides (:120-131)."""

    max_iter: int = 200
    rhs_tol: float = 1e-6
    delta_x_tol: float = 1.0
    abs_tol: float = 1e-12
    rel_tol: float = 1e-3
    update_weights_each_iter: bool = True

    @staticmethod
    def dc() -> "NewtonParams":
        return NewtonParams()

    @staticmethod
    def transient() -> "NewtonParams":
        return NewtonParams(max_iter=20, rhs_tol=1e-2, delta_x_tol=0.33, abs_tol=1e-6, rel_tol=1e-2,
                            update_weights_each_iter=False)


def pwl_value(times, values, t: float) -> float:
    """PWLinData::updateSource without delay or repeat (N_DEV_SourceData.C:1371-1490), with its own
    arithmetic: linear between points, zero-valued start at t = 0 when the first point is later,
    the last value after the last point (formed as the reference forms it, from the segment
    (0, v_last) - (1, v_last))."""
    n = len(times)
    if t > times[n - 1]:
        v = float(values[n - 1])
        value = (1.0 - t) * v / 1.0
        value += (-0.0 + t) * v / 1.0
        return value
    loc = n - 1
    for i in range(n):
        if t < times[i]:
            loc = i
            break
    if loc == 0:
        t1, v1 = 0.0, 0.0
    else:
        t1, v1 = float(times[loc - 1]), float(values[loc - 1])
    t2, v2 = float(times[loc]), float(values[loc])
    if t1 == t2:
        return v2
    length = t2 - t1
    return (t2 - t) * v1 / length + (-t1 + t) * v2 / length


class LinearDevices:
    """Resistors, capacitors and voltage sources of a circuit as constant CSR stamps."""

    def __init__(self, c, rowptr, colind):
        self.c = c
        nu = c.n_unknowns
        nnz = int(rowptr[-1])
        rows = np.repeat(np.arange(nu), np.diff(rowptr))
        key = rows.astype(np.int64) * nu + colind

        def pos(r, cc):
            k = np.searchsorted(key, np.asarray(r, np.int64) * nu + np.asarray(cc, np.int64))
            assert np.all(key[k] == np.asarray(r, np.int64) * nu + cc), "pattern lacks a linear-device entry"
            return k

        self.lin_f = np.zeros(nnz)
        self.lin_q = np.zeros(nnz)

        def add2(vals, nodes, g):
            a, b = nodes[:, 0], nodes[:, 1]
            for r, cc, s in ((a, a, 1.0), (a, b, -1.0), (b, a, -1.0), (b, b, 1.0)):
                m = (r >= 0) & (cc >= 0)
                np.add.at(vals, pos(r[m], cc[m]), s * g[m])

        if c.res_nodes.shape[0]:
            add2(self.lin_f, c.res_nodes.astype(np.int64), 1.0 / c.res_value)
        if c.cap_nodes.shape[0]:
            add2(self.lin_q, c.cap_nodes.astype(np.int64), c.cap_value.astype(float))
        self.branch = np.arange(c.n_nodes, c.n_nodes + c.n_vsrc)
        if c.n_vsrc:
            p, n = c.vsrc_nodes[:, 0].astype(np.int64), c.vsrc_nodes[:, 1].astype(np.int64)
            for r, cc, s in ((p, self.branch, 1.0), (n, self.branch, -1.0), (self.branch, p, 1.0),
                             (self.branch, n, -1.0)):
                m = (r >= 0) & (cc >= 0)
                np.add.at(self.lin_f, pos(r[m], cc[m]), s)

    def source_values(self, t: float | None) -> np.ndarray:
        """Source values at time t (None: the DC values)."""
        c = self.c
        v = np.array(c.vsrc_dc, dtype=float)
        if t is not None:
            for k, p in enumerate(c.vsrc_pwl):
                if p is not None:
                    v[k] = pwl_value(p[0], p[1], t)
        return v


@dataclass
class StepStats:
    newton_iters: list = field(default_factory=list)
    times: list = field(default_factory=list)
    failed_steps: int = 0
    wall_s: float = 0.0
    loads: int = 0
    factorizations: int = 0
    host_factorizations: int = 0
    surrogate_loads: int = 0
    static_pivot_fallbacks: int = 0
    chord_iters: list = field(default_factory=list)
    surrogate_error: list = field(default_factory=list)
    solves: int = 0                 # triangular solves with the GPU refactorization's factors
    refinements: int = 0            # of which iterative-refinement steps
    first_solve_berr: list = field(default_factory=list)  # backward error after each first solve


class TransientBase:
    """Operating point and fixed-step transient of a circuit: the integrator and Newton loop.

    Subclasses supply the two per-iterate steps, ``_load(flags)`` (every device's F, Q, dF/dx,
    dQ/dx at self.x) and ``_combine(mode, h, order, qn0, fhist)`` (Newton matrix, residual, Q and F
    totals); the buffers are torch tensors on ``dev``.
    ``solver``: "dense" (LU on ``dev``, small circuits), "rf" (GPU sparse refactorization, device
    backends), "splu" (host sparse LU) or "auto".
    """

    def __init__(self, c, n_state, n_store, rowptr, colind, dev, solver="auto", gmin=1e-12):
        import torch

        self.torch = torch
        self.c = c
        self.nu = c.n_unknowns
        self.nnz = int(rowptr[-1])
        self.rowptr = np.ascontiguousarray(rowptr, np.int32)
        self.colind = np.ascontiguousarray(colind, np.int32)
        self.dev = dev
        self.gmin = gmin
        self.gshunt = 0.0  # node-to-ground conductance during gmin stepping
        self.limiting = True  # device voltage limiting, with its corrections in the Newton residual
        self.lin = LinearDevices(c, self.rowptr, self.colind)
        z = lambda k: torch.zeros(k, dtype=torch.float64, device=self.dev)
        self.next_sta, self.curr_sta = z(n_state), z(n_state)
        self.next_sto, self.curr_sto = z(n_store), z(n_store)
        self.jac, self.rhs, self.qtot, self.ftot = z(self.nnz), z(self.nu), z(self.nu), z(self.nu)
        self.b = z(self.nu)
        self.x = z(self.nu)
        self._branch = torch.as_tensor(self.lin.branch, device=self.dev)
        if solver == "auto":
            solver = "dense" if self.nu <= 4096 else "splu"
        self.solver = solver
        if solver == "dense":
            rows = np.repeat(np.arange(self.nu), np.diff(self.rowptr))
            self._flat = torch.as_tensor(rows.astype(np.int64) * self.nu + self.colind, device=self.dev)
            self._dense = torch.zeros(self.nu * self.nu, dtype=torch.float64, device=self.dev)
        self.stats = StepStats()

    def _set_sources(self, t):
        vals = self.lin.source_values(t)
        self.b.zero_()
        if len(vals):
            self.b[self._branch] = self.torch.as_tensor(vals, dtype=self.torch.float64, device=self.dev)

    def _load(self, flags: SolverFlags):
        raise NotImplementedError

    def _combine(self, mode, h=None, order=1, qn0=None, fhist=None):
        raise NotImplementedError

    def _sync(self):
        pass

    # -- learned warm start ------------------------------------------------------------------------
    surrogate = None  # set to an object with load(x, f, q, fx, qx, stream) to enable the warm start
    chord_max = 3
    chord_tol = 1e-4
    chord_step_cap = 0.5  # volts
    chord_monotone = True  # stop the chord iterations when the surrogate residual grows
    predictor = "none"  # Newton start: "none" (the last point) or "linear" (extrapolation of the last two)

    def _surrogate_load(self):
        raise NotImplementedError

    def _anchor(self, f_sn, q_sn):
        """f <- f_anchor + (f - f_sn), likewise q: anchored surrogate vectors."""
        self.f.sub_(f_sn).add_(self.f_anchor)
        self.q.sub_(q_sn).add_(self.q_anchor)

    def _save_anchor(self):
        """Exact MOSFET F and Q at the accepted point (the last load was there)."""
        if self.surrogate is not None:
            self.f_anchor = self.f.clone()
            self.q_anchor = self.q.clone()

    def _surrogate_warm_start(self, h, order, qn0, fhist, x_n):
        """Chord iterations on anchored surrogate loads: the MOSFETs' F and Q at an iterate x are
        the exact FP64 values at the last accepted point x_n plus the surrogate's change from x_n
        to x, so the surrogate's level errors cancel and only its slope errors remain; the linear
        devices are exact and the matrix is the last exact factorization. This moves self.x towards
        the solution before the exact FP64 Newton iterations take over; the exact loads always make
        the final, converged evaluation."""
        lim = self.limiting
        self.limiting = False  # the surrogate has no limiter corrections
        n_it = 0
        x_start = self.x.clone()
        self.x.copy_(x_n)
        self._surrogate_load()
        f_sn, q_sn = self.f.clone(), self.q.clone()
        self.x.copy_(x_start)
        best_x, best_r = self.x.clone(), math.inf
        try:
            for _ in range(self.chord_max + 1):
                self._surrogate_load()
                self._anchor(f_sn, q_sn)
                self._combine(1, h, order, qn0, fhist)
                r = float(self.rhs.abs().max())
                if not math.isfinite(r) or (self.chord_monotone and r >= best_r):
                    break  # the surrogate residual stopped falling: keep the best iterate
                if r < best_r or not self.chord_monotone:
                    best_x.copy_(self.x)
                    best_r = min(r, best_r)
                if n_it == self.chord_max:
                    break
                dx = self._solve_factored()
                step = float(dx.abs().max())
                if not math.isfinite(step):
                    break
                if step > self.chord_step_cap:
                    dx *= self.chord_step_cap / step
                self.x += dx
                n_it += 1
                if step <= self.chord_tol:
                    best_x.copy_(self.x)
                    break
        finally:
            self.limiting = lim
            self.x.copy_(best_x)
            self.f.copy_(self.f_anchor)
            self.q.copy_(self.q_anchor)
        self.stats.chord_iters.append(n_it)
        self.stats.surrogate_loads += n_it

    def _solve(self):
        """Factors the current Newton matrix (kept for chord iterations) and solves with rhs."""
        torch = self.torch
        if self.solver == "rf":
            return self._solve_rf()
        if self.solver == "dense":
            self._dense.zero_()
            self._dense[self._flat] = self.jac
            LU, piv, _ = torch.linalg.lu_factor_ex(self._dense.view(self.nu, self.nu))
            self._lu = (LU, piv)  # a singular matrix gives a non-finite step: a Newton failure
        else:
            import scipy.sparse as sp
            import scipy.sparse.linalg as spl
            J = sp.csr_matrix((self.jac.cpu().numpy(), self.colind, self.rowptr), shape=(self.nu, self.nu))
            self.stats.factorizations += 1
            try:
                self._lu = spl.splu(J.tocsc())
            except RuntimeError:  # exactly singular: a Newton failure, as with the dense factorization
                self._lu = None
                return torch.full_like(self.rhs, float("nan"))
            return self._solve_factored()
        self.stats.factorizations += 1
        return self._solve_factored()

    def _solve_rf(self):
        raise NotImplementedError("the GPU refactorization needs a device backend")

    def _solve_factored(self):
        """Solves with the last factorization (a chord step when the matrix has moved on)."""
        torch = self.torch
        if self.solver == "rf":
            x = self.rhs.clone()
            _native.check(self._lib.xd_rf_solve(self._rf, ctypes.c_void_p(x.data_ptr())), "xd_rf_solve")
            return x
        if self.solver == "dense":
            LU, piv = self._lu
            return torch.linalg.lu_solve(LU, piv, self.rhs.view(-1, 1)).view(-1)
        dx = self._lu.solve(self.rhs.cpu().numpy())
        return torch.as_tensor(dx, device=self.dev)

    def _newton(self, prm: NewtonParams, flags_for_iter, mode, h=None, order=1, qn0=None, fhist=None):
        """Newton iterations from self.x; returns the number of updates or -1 (no convergence).

        As in DampedNewton::solve, the residual is re-evaluated at each updated iterate and the
        convergence test (:1792-1830) takes its max norm together with the weighted RMS norm of the
        update just made, weights rel_tol * max(|x_ref|, |x|) + abs_tol (:325-350) with x_ref the
        iterate the solve started from; a transient solve fixes the weights at its start. So the
        last load of a converged solve is at the converged point, and Q and F there are current.
        """
        torch = self.torch
        x_ref = self.x.clone()
        w = prm.rel_tol * x_ref.abs() + prm.abs_tol
        self._load_and_combine(flags_for_iter(0), mode, h, order, qn0, fhist)
        for it in range(1, prm.max_iter + 1):
            dx = self._solve()
            w, wrms = self._update(dx, x_ref, w, prm)
            self._load_and_combine(flags_for_iter(it), mode, h, order, qn0, fhist)
            max_rhs = self._residual_max()
            if not (math.isfinite(max_rhs) and math.isfinite(wrms)):
                return -1
            if max_rhs <= prm.rhs_tol and wrms <= prm.delta_x_tol:
                return it
        return -1

    def _update(self, dx, x_ref, w, prm):
        """x += dx; the weights (refreshed when the parameters say so) and the update's weighted
        RMS norm."""
        torch = self.torch
        self.x += dx
        if prm.update_weights_each_iter:
            w = prm.rel_tol * torch.maximum(x_ref.abs(), self.x.abs()) + prm.abs_tol
        return w, float(torch.sqrt(torch.mean((dx / w) ** 2)))

    def _residual_max(self):
        return float(self.rhs.abs().max())

    def _load_and_combine(self, flags, mode, h=None, order=1, qn0=None, fhist=None):
        """The device loads at self.x, then the combine (one fused pass where the backend has it)."""
        self._load(flags)
        self._combine(mode, h, order, qn0, fhist)

    def _history_here(self):
        """Q and F at the current point (after a load there) into q_tot / f_tot."""
        zero = self.torch.zeros_like(self.x)
        self._combine(1, 1.0, 1, zero, None)

    # -- analyses -----------------------------------------------------------------------------------
    def dcop(self, params: NewtonParams | None = None, x0=None, t0: float = 0.0) -> int:
        """Operating point at time t0 (sources at their transient values, as the reference does
        for the operating point of a transient), with charges computed (tranop); leaves Q(t0) and
        F(t0) in q_tot / f_tot and the device history rotated. Newton from x0 (zero if not given)
        first; if it fails,
        gmin stepping as the reference's continuation does it (N_NLS_NOX_Interface.C:1351-1380,
        N_NLS_NOX_AugmentLinSys_GStepping.C:125-131): a shunt conductance 10^p - 10^-4 from every
        unknown to ground, p stepped from 4 to -4 by natural continuation with an adaptive step
        (first step -2, halved on a failed stage, grown by the LOCA rule with aggressiveness 0.01;
        at most 400 stages of at most 20 Newton iterations), each stage starting from the last
        converged one. Returns the total number of Newton updates."""
        prm = params or NewtonParams.dc()
        start = self.torch.zeros_like(self.x)
        if x0 is not None:
            start.copy_(self.torch.as_tensor(x0, dtype=self.torch.float64))
        self._set_sources(t0)

        # The first load of a solve from zero initialises the junction voltages (the models ignore
        # the iterate there); a supplied starting iterate (x0, as a .NODESET gives) is evaluated
        # from the first load on.
        def flags(it, first=True):
            return SolverFlags(dcop=1, transient=0, tranop=1, newton_iter=it,
                               init_jct=1 if (it == 0 and first and x0 is None) else 0, gmin=self.gmin,
                               voltlim=int(self.limiting))

        self.x.copy_(start)
        self.gshunt = 0.0
        total = self._newton(prm, flags, mode=0)
        if total < 0:
            total = self._gmin_stepping(prm, start, flags)
        self.gshunt = 0.0
        self._history_here()
        self._accept_point()
        return total

    def _gmin_stepping(self, prm: NewtonParams, start, flags) -> int:
        p, p_end, step = 4.0, -4.0, -2.0
        max_stages, stage_iters, aggressiveness, min_step = 400, 20, 0.01, 1e-6
        stage_prm = NewtonParams(max_iter=min(stage_iters, prm.max_iter), rhs_tol=prm.rhs_tol,
                                 delta_x_tol=prm.delta_x_tol, abs_tol=prm.abs_tol, rel_tol=prm.rel_tol,
                                 update_weights_each_iter=prm.update_weights_each_iter)
        self.x.copy_(start)
        for t in (self.next_sta, self.next_sto, self.curr_sta, self.curr_sto):
            t.zero_()
        total, first, saved = 0, True, None
        p_try = p
        for _ in range(max_stages):
            self.gshunt = 10.0 ** p_try - 10.0 ** p_end
            n_it = self._newton(stage_prm, lambda it, first=first: flags(it, first), mode=0)
            if n_it >= 0:
                total += n_it
                first = False
                self.curr_sto.copy_(self.next_sto)
                saved = [t.clone() for t in (self.x, self.next_sta, self.next_sto, self.curr_sto)]
                p = p_try
                if p <= p_end:
                    return total
                frac = (stage_iters - n_it) / (stage_iters - 1)
                step *= 1.0 + aggressiveness * max(frac, 0.0) ** 2
            else:
                if saved is None:
                    break  # the heavily shunted start itself failed
                for t, v in zip((self.x, self.next_sta, self.next_sto, self.curr_sto), saved):
                    t.copy_(v)
                step *= 0.5
                if abs(step) < min_step:
                    break
            p_try = max(p + step, p_end)
        self.gshunt = 0.0
        raise RuntimeError(f"operating point did not converge (gmin stepping stopped at 10^{p_try:.3g} S)")

    def _accept_point(self):
        """The accepted point's device history becomes the current one."""
        self.curr_sta.copy_(self.next_sta)
        self.curr_sto.copy_(self.next_sto)
        self._save_anchor()

    def set_initial_state(self, x, t0: float = 0.0):
        """Starts the transient from x (an operating point with a kick, say): one load at x gives
        Q(t0), F(t0) and the device history."""
        self.x.copy_(self.torch.as_tensor(x, dtype=self.torch.float64))
        self._set_sources(t0)
        self._load(SolverFlags(dcop=1, transient=0, tranop=1, newton_iter=1, gmin=self.gmin,
                               voltlim=int(self.limiting)))
        self._history_here()
        self._accept_point()

    def run(self, tstop: float, hmax: float, params: NewtonParams | None = None, record=None, warm_start=None,
            min_step: float = 1e-18):
        """Fixed-step transient from the current state to tstop. ``record``: unknown indices whose
        waveforms are returned. ``warm_start(t, h, x_n, x_nm1)``: optional initial Newton iterate.
        Returns (times, waveforms [n_points, len(record)])."""
        torch = self.torch
        prm = params or NewtonParams.transient()
        rec = np.arange(self.nu) if record is None else np.asarray(record)
        rec_t = torch.as_tensor(rec, device=self.dev)
        t = 0.0
        h = hmax
        qn0 = self.qtot.clone()
        fhist = self.ftot.clone()
        x_n = self.x.clone()
        x_nm1 = None
        h_prev = hmax
        times, waves = [0.0], [self.x[rec_t].cpu().numpy()]
        first = True
        t_start = _time.perf_counter()
        while t < tstop * (1 - 1e-12):
            h = min(h, tstop - t)
            order = 1 if first else 2
            self._set_sources(t + h)
            if warm_start is not None:
                self.x.copy_(warm_start(t, h, x_n, x_nm1))
            elif x_nm1 is not None and self.predictor == "linear":
                self.x.copy_(x_n + (x_n - x_nm1) * (h / h_prev))
            else:
                self.x.copy_(x_n)
            if self.surrogate is not None and not first and getattr(self, "_lu", None) is not None:
                self._surrogate_warm_start(h, order, qn0, fhist, x_n)

            def flags(it, first=first, h=h):
                return SolverFlags(transient=1, newton_iter=it, init_tran=1 if first else 0, pdt=1.0 / h,
                                   gmin=self.gmin, voltlim=int(self.limiting))

            n_it = self._newton(prm, flags, mode=1, h=h, order=order, qn0=qn0, fhist=fhist)
            if n_it < 0:
                self.stats.failed_steps += 1
                # Restore the device history of the last accepted point and retry with half the step.
                self.next_sta.copy_(self.curr_sta)
                self.next_sto.copy_(self.curr_sto)
                h *= 0.5
                if h < min_step:
                    raise RuntimeError(f"time step too small at t = {t:.6g}")
                continue
            t += h
            first = False
            # Accept: the last load was at the converged point, so q_tot / f_tot are Q and F there.
            qn0.copy_(self.qtot)
            fhist.copy_(self.ftot)
            self._accept_point()
            x_nm1, x_n = x_n, self.x.clone()
            h_prev = h
            self.stats.newton_iters.append(n_it)
            self.stats.times.append(t)
            times.append(t)
            waves.append(self.x[rec_t].cpu().numpy())
            h = min(hmax, h * 2.0)
        self._sync()
        self.stats.wall_s += _time.perf_counter() - t_start
        return np.array(times), np.stack(waves)


class GpuTransient(TransientBase):
    """The transient on one CUDA device: MOSFET loads by ``xd_load_assign`` and the combine with
    the linear devices by ``xd_tia_combine``, on device-resident buffers.

    ``family``: the circuit's MOSFETs as one ``MosfetDevice`` built on the pattern (rowptr, colind).
    """

    def __init__(self, c, family: MosfetDevice, rowptr, colind, device=0, solver="auto", gmin=1e-12,
                 graphs=True, static_pivot=True, fused=True):
        import torch

        if solver == "auto":
            # Up to XD_DENSE_MAX_N unknowns the one-SM solves; above, the sparse refactorization
            # (on the 1,228-MOSFET gate netlist, 2,534 unknowns, 0.22 s for 1 ns against 1.65 s with
            # a dense LU of every Newton matrix).
            solver = "dense" if c.n_unknowns <= _native.XD_DENSE_MAX_N else "rf"
        super().__init__(c, family.n_state, family.n_store, rowptr, colind, torch.device("cuda", device), solver,
                         gmin)
        self.fam = family
        # With the dense solve, each Newton iteration (factor, solve, update, norms, device loads,
        # combine) replays as one CUDA graph, one per distinct (flags, step, method) combination.
        self.graphs = bool(graphs) and self.solver == "dense"
        self._graphs = {}
        self._graph_pool = None
        lib = _native.load()
        self._lib = lib
        csr = _native.XdCsr(self.nu, self.rowptr.ctypes.data_as(_native._ip), self.colind.ctypes.data_as(_native._ip))
        h = ctypes.c_void_p()
        _native.check(lib.xd_tia_create(ctypes.byref(csr), int(device), ctypes.byref(h)), "xd_tia_create")
        self._tia = h
        # Source values at each time point on the device (xd_pwl_eval): the branch rows of b.
        nv = c.n_vsrc
        counts = np.array([0 if p is None else len(p[0]) for p in c.vsrc_pwl] + [0] * (nv - len(c.vsrc_pwl)),
                          dtype=np.int32)[:nv]
        tv = np.array([x for p in c.vsrc_pwl if p is not None for pair in zip(p[0], p[1]) for x in pair] or [0.0],
                      dtype=np.float64)
        rows = np.ascontiguousarray(self.lin.branch, dtype=np.int32)
        dc = np.ascontiguousarray(c.vsrc_dc, dtype=np.float64)
        hp = ctypes.c_void_p()
        _native.check(lib.xd_pwl_create(nv, rows.ctypes.data_as(_native._ip), counts.ctypes.data_as(_native._ip),
                                        tv.ctypes.data_as(_native._dp), dc.ctypes.data_as(_native._dp), None, None,
                                        int(device), ctypes.byref(hp)), "xd_pwl_create")
        self._pwl = hp
        # Fused load and combine (xd_tia_load_combine): the Newton matrix and residual straight from
        # the evaluation's staged stamps, bit-identical to xd_load_assign + xd_tia_combine.
        self._fused = None
        if fused:
            hf = ctypes.c_void_p()
            _native.check(lib.xd_tia_fused_create(h, family._h, ctypes.byref(hf)), "xd_tia_fused_create")
            self._fused = hf
        T = lambda a: torch.as_tensor(a, dtype=torch.float64, device=self.dev).contiguous()
        z = lambda k: torch.zeros(k, dtype=torch.float64, device=self.dev)
        self.lin_f, self.lin_q = T(self.lin.lin_f), T(self.lin.lin_q)
        # Circuits of at most XD_DENSE_MAX_N unknowns take the library's one-SM dense solve.
        self._small = self.solver == "dense" and self.nu <= _native.XD_DENSE_MAX_N
        if self._small:
            self._lu_d = z(self.nu * self.nu)
            self._piv_d = torch.zeros(self.nu, dtype=torch.int32, device=self.dev)
            self._dx_d = z(self.nu)
        # Small systems: static-pivot refactorization (xd_slu_*) with the pivoting solve queued
        # behind it for the matrices whose pivots fail its threshold test; the order is taken from
        # a host factorization of the first matrix and taken again after a fallback.
        self.static_pivot = bool(static_pivot) and self._small
        self._slu = None
        self._slu_stale = False
        self._info_d = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self._fallback_d = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self._e_norms = z(3)  # the eager iterations' norms (the graph-replayed ones use their own)
        # Family outputs (stored by xd_load_assign; entries the family does not stamp stay zero).
        self.f, self.q, self.fx, self.qx = z(self.nu), z(self.nu), z(self.nu), z(self.nu)
        self.jf, self.jq = z(self.nnz), z(self.nnz)

    def close(self):
        self._graphs = {}
        if getattr(self, "_slu", None) is not None and self._slu.value:
            self._lib.xd_slu_destroy(self._slu)
            self._slu = None
        if getattr(self, "_pwl", None) is not None and self._pwl.value:
            self._lib.xd_pwl_destroy(self._pwl)
            self._pwl = None
        if getattr(self, "_fused", None) is not None and self._fused.value:
            self._lib.xd_tia_fused_destroy(self._fused)
            self._fused = None
        if getattr(self, "_tia", None) is not None and self._tia.value:
            self._lib.xd_tia_destroy(self._tia)
            self._tia = None
        if getattr(self, "_rf", None) is not None and self._rf.value:
            self._lib.xd_rf_destroy(self._rf)
            self._rf = None

    def _rf_setup(self):
        """Host factorization of the current matrix (pivot order, fill) and the GPU refactorization
        set-up from it: P A Q = L U with (P A Q)[i][j] = A[P[i]][Q[j]]."""
        import scipy.sparse as sp
        import scipy.sparse.linalg as spl

        if getattr(self, "_rf", None) is not None and self._rf.value:
            self._lib.xd_rf_destroy(self._rf)
            self._rf = None
        vals = self.jac.cpu().numpy()
        # SuperLU drops entries that are exactly zero, but the refactorization needs L + U to hold
        # every position of the pattern (a DC matrix has zeros where later matrices have
        # capacitances): factor with a placeholder far below every pivot in those positions.
        scale = float(np.abs(vals).max()) or 1.0
        sym = np.where(vals == 0.0, scale * 1e-30, vals)
        A = sp.csr_matrix((sym, self.colind, self.rowptr), shape=(self.nu, self.nu))
        # Fill-reducing order on A + A^T with threshold pivoting that prefers the diagonal (a row
        # swap only when the diagonal is below 0.1 of the column's largest entry), as circuit
        # solvers such as KLU factor: strict partial pivoting destroys the order's sparsity on
        # MNA matrices (66M instead of 2M nonzeros at 200k unknowns).
        lu = spl.splu(A.tocsc(), permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.1,
                      options=dict(SymmetricMode=True))
        P = np.argsort(lu.perm_r).astype(np.int32)
        Q = np.argsort(lu.perm_c).astype(np.int32)
        L = lu.L.tocsr()
        U = lu.U.tocsr()
        L.sort_indices()
        U.sort_indices()
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        arrs = [i32(self.rowptr), i32(self.colind), f64(vals), i32(L.indptr), i32(L.indices), f64(L.data),
                i32(U.indptr), i32(U.indices), f64(U.data), P, Q]
        self._rf_keep = arrs
        ip = lambda a: a.ctypes.data_as(_native._ip)
        dp = lambda a: a.ctypes.data_as(_native._dp)
        h = ctypes.c_void_p()
        _native.check(self._lib.xd_rf_create(self.nu, self.nnz, ip(arrs[0]), ip(arrs[1]), dp(arrs[2]), int(L.nnz),
                                             ip(arrs[3]), ip(arrs[4]), dp(arrs[5]), int(U.nnz), ip(arrs[6]),
                                             ip(arrs[7]), dp(arrs[8]), ip(P), ip(Q), self.dev.index or 0,
                                             ctypes.byref(h)), "xd_rf_create")
        self._rf = h
        self.stats.host_factorizations += 1

    def _rf_try_setup(self):
        """_rf_setup, with a singular matrix (the library's zero pivot, or the host factorization's)
        reported as False, like a failed dense factorization, so that Newton fails the step."""
        try:
            self._rf_setup()
            return True
        except (_native.NativeError, RuntimeError):
            if getattr(self, "_rf", None) is not None and self._rf.value:
                self._lib.xd_rf_destroy(self._rf)
            self._rf = None
            return False

    def _solve_rf(self):
        torch = self.torch
        self.stats.factorizations += 1
        self._lu = True
        nan = lambda: torch.full_like(self.rhs, float("nan"))
        fresh = False
        if getattr(self, "_rf", None) is None or not self._rf.value:
            if not self._rf_try_setup():
                return nan()
            fresh = True
        else:
            torch.cuda.current_stream(self.dev).synchronize()  # values complete before the library reads them
            rc = self._lib.xd_rf_refactor(self._rf, ctypes.c_void_p(self.jac.data_ptr()))
            if rc != 0:
                # A zero pivot in the kept pivot order (the matrices of a DC solve and of a time step
                # differ in which entries dominate): factor this matrix afresh on the host.
                if not self._rf_try_setup():
                    return nan()
                fresh = True
        x = self._rf_solve_refined(self.rhs, accept=fresh)
        if x is None and not fresh:
            # The kept pivot order does not suit this matrix: factor it afresh on the host.
            if not self._rf_try_setup():
                return nan()
            x = self._rf_solve_refined(self.rhs, accept=True)
        return nan() if x is None else x

    def _rf_matrices(self):
        torch = self.torch
        if getattr(self, "_rf_crow", None) is None:
            self._rf_crow = torch.as_tensor(self.rowptr.astype(np.int64), device=self.dev)
            self._rf_col = torch.as_tensor(self.colind.astype(np.int64), device=self.dev)
        mk = lambda v: torch.sparse_csr_tensor(self._rf_crow, self._rf_col, v, size=(self.nu, self.nu),
                                               check_invariants=False)
        with warnings.catch_warnings():  # torch marks its sparse CSR support as beta
            warnings.simplefilter("ignore", UserWarning)
            return mk(self.jac), mk(self.jac.abs())

    def _rf_solve_refined(self, b, tol=1e-10, max_refine=3, accept=False):
        """Solve with the current factors, then iterative refinement (r = b - J x, x += J^-1 r) until
        the componentwise backward error max_i |r_i| / (|J| |x| + |b|)_i is at most tol (a stable
        factorization gives a few ulps after one refinement step), at most max_refine times. Returns
        None when the error stays above tol, or the last iterate when accept is set."""
        torch = self.torch
        J, Ja = self._rf_matrices()
        x = b.clone()
        torch.cuda.current_stream(self.dev).synchronize()
        _native.check(self._lib.xd_rf_solve(self._rf, ctypes.c_void_p(x.data_ptr())), "xd_rf_solve")
        torch.cuda.synchronize(self.dev)
        self.stats.solves += 1
        ab = b.abs()
        for k in range(max_refine + 1):
            if not bool(torch.isfinite(x).all()):
                return None
            r = b - J @ x
            den = Ja @ x.abs() + ab
            err = torch.where(r == 0, torch.zeros_like(r), r.abs() / den.clamp_min(1e-300))
            e = float(err.max())
            if k == 0:
                self.stats.first_solve_berr.append(e)
            if e <= tol:
                return x
            if k == max_refine:
                return x if accept else None
            d = r.contiguous()
            torch.cuda.current_stream(self.dev).synchronize()
            _native.check(self._lib.xd_rf_solve(self._rf, ctypes.c_void_p(d.data_ptr())), "xd_rf_solve")
            torch.cuda.synchronize(self.dev)
            self.stats.solves += 1
            self.stats.refinements += 1
            x = x + d
        return None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ptr(self, t):
        return None if t is None else ctypes.c_void_p(t.data_ptr())

    # -- graph-replayed Newton iterations (dense solve) ---------------------------------------------
    def _iteration_body(self, prm, flags1, mode, h, order, qn0, fhist):
        """One Newton update and the evaluation at the new iterate, as _newton does it eagerly:
        factor and solve, x += dx, the weighted update norm, the device loads and the combine at
        the new x, and the residual's max norm; the two norms land in the pinned host buffer."""
        torch = self.torch
        if self._small:
            self._dense_solve(self._dx_d)
            dx, LU, piv = self._dx_d, None, None
        else:
            self._dense.zero_()
            self._dense[self._flat] = self.jac
            LU, piv, _ = torch.linalg.lu_factor_ex(self._dense.view(self.nu, self.nu))
            dx = torch.linalg.lu_solve(LU, piv, self.rhs.view(-1, 1)).view(-1)
        self._device_update(dx, self._g_xref, self._g_w, prm, self._g_norms)
        self._load_combine_raw(flags1, mode, h, order, qn0, fhist)
        self._device_residual_norm(self._g_norms)
        self._g_host.copy_(self._g_norms, non_blocking=True)
        return "small" if self._small else (LU, piv)

    def _graph_for(self, prm, flags1, mode, h, order, qn0, fhist):
        torch = self.torch
        # The static-pivot set-up reads the current matrix on the host (never while capturing); a new
        # order drops the graphs that launch the old one's kernels.
        self._slu_ready()
        key = (mode, h, order, self.gshunt, self.limiting, prm.rel_tol, prm.abs_tol, prm.update_weights_each_iter,
               tuple(sorted(vars(flags1).items())), self._ptr(qn0).value if qn0 is not None else 0,
               self._ptr(fhist).value if fhist is not None else 0)
        g = self._graphs.get(key)
        if g is not None:
            return g
        if not hasattr(self, "_g_host"):
            z = lambda k: torch.zeros(k, dtype=torch.float64, device=self.dev)
            self._g_xref, self._g_w, self._g_norms = z(self.nu), z(self.nu), z(3)
            self._g_host = torch.zeros(3, dtype=torch.float64, pin_memory=True)
            if not self._small:
                # Library handles and workspaces come into being outside any capture.
                eye = torch.eye(self.nu, dtype=torch.float64, device=self.dev)
                torch.linalg.lu_solve(*torch.linalg.lu_factor_ex(eye)[:2], eye[:, :1])
            self._graph_pool = torch.cuda.graph_pool_handle()
            torch.cuda.synchronize(self.dev)
        # Capture from a copy of the state: capturing runs nothing, but the buffers are restored to
        # be safe against any eager work a library does while it is captured.
        keep = [t.clone() for t in (self.x, self.next_sta, self.next_sto, self.jac, self.rhs)]
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, pool=self._graph_pool):
            lu = self._iteration_body(prm, flags1, mode, h, order, qn0, fhist)
        for t, k in zip((self.x, self.next_sta, self.next_sto, self.jac, self.rhs), keep):
            t.copy_(k)
        self._graphs[key] = (graph, lu)
        return self._graphs[key]

    def _newton(self, prm: NewtonParams, flags_for_iter, mode, h=None, order=1, qn0=None, fhist=None):
        self._first_solve = True
        if not self.graphs:
            return super()._newton(prm, flags_for_iter, mode, h, order, qn0, fhist)
        f1, f2 = flags_for_iter(1), flags_for_iter(2)
        f2.newton_iter = 1
        if f1 != f2:  # the iterations' flags differ beyond newton_iter >= 1: no single graph
            return super()._newton(prm, flags_for_iter, mode, h, order, qn0, fhist)
        torch = self.torch
        self._load_and_combine(flags_for_iter(0), mode, h, order, qn0, fhist)
        graph, lu = self._graph_for(prm, f1, mode, h, order, qn0, fhist)  # loads and combine leave x as it was
        self._g_xref.copy_(self.x)
        self._g_w.copy_(prm.rel_tol * self._g_xref.abs() + prm.abs_tol)
        stream = torch.cuda.current_stream(self.dev)
        for it in range(1, prm.max_iter + 1):
            graph.replay()
            self._lu = lu
            self.stats.factorizations += 1
            self.stats.loads += 1
            stream.synchronize()
            wrms, max_rhs = float(self._g_host[0]), float(self._g_host[1])
            self._lu_from_slu = self._slu is not None and self._g_host[2] == 0
            if self._g_host[2] != 0:
                self._note_fallback()
            if not (math.isfinite(max_rhs) and math.isfinite(wrms)):
                return -1
            if max_rhs <= prm.rhs_tol and wrms <= prm.delta_x_tol:
                return it
        return -1

    def _device_update(self, dx, x_ref, w, prm, norms):
        p = self._ptr
        _native.check(self._lib.xd_tia_newton_update(self._tia, p(self.x), p(dx.contiguous()), p(x_ref), p(w),
                                                     prm.rel_tol, prm.abs_tol, int(prm.update_weights_each_iter),
                                                     p(norms), self._stream()), "xd_tia_newton_update")

    def _device_residual_norm(self, norms):
        p = self._ptr
        _native.check(self._lib.xd_tia_residual_norm(self._tia, p(self.rhs), p(self._fallback_d), p(norms),
                                                     self._stream()), "xd_tia_residual_norm")

    def _update(self, dx, x_ref, w, prm):
        if not self.graphs and not self._small:
            return super()._update(dx, x_ref, w, prm)
        w = w.clone()  # written in place when the weights are refreshed
        self._device_update(dx, x_ref, w, prm, self._e_norms)
        return w, float(self._e_norms[0].item())

    def _residual_max(self):
        if not self.graphs and not self._small:
            return super()._residual_max()
        self._device_residual_norm(self._e_norms)
        return float(self._e_norms[1].item())

    def _slu_ready(self, renew=True):
        """The static-pivot solve's order and pattern, taken from the current matrix when there is
        none, or (renew) again when one failed a pivot since; False when the matrix is singular (that
        solve then uses the pivoting kernel alone). Orders are renewed only at the first solve of a
        Newton solve, in the eager and the graph-replayed iterations alike, so that both use the
        same orders. Host work: never called while a graph is captured."""
        if not self.static_pivot:
            return False
        if self._slu is not None and not (self._slu_stale and renew):
            return True
        if self._slu is not None:
            self._lib.xd_slu_destroy(self._slu)
            self._slu = None
            self._lu_from_slu = False
            self._graphs = {}  # they launch the old order's kernels
        vals = np.ascontiguousarray(self.jac.cpu().numpy())
        h = ctypes.c_void_p()
        rc = self._lib.xd_slu_create(self.nu, self.rowptr.ctypes.data_as(_native._ip),
                                     self.colind.ctypes.data_as(_native._ip), vals.ctypes.data_as(_native._dp),
                                     1e-3, self.dev.index or 0, ctypes.byref(h))
        self._slu_stale = False
        if rc != 0:
            return False
        self._slu = h
        return True

    def _note_fallback(self):
        self.stats.static_pivot_fallbacks += 1
        self._slu_stale = True

    def _dense_solve(self, out):
        p = self._ptr
        if self._slu is not None:
            _native.check(self._lib.xd_slu_solve(self._slu, p(self.jac), p(self.rhs), p(self._lu_d), p(out),
                                                 p(self._info_d), self._stream()), "xd_slu_solve")
            self._fallback_d.copy_(self._info_d)
            _native.check(self._lib.xd_tia_dense_solve_fallback(self._tia, p(self.jac), p(self.rhs), p(self._lu_d),
                                                                p(self._piv_d), p(out), p(self._info_d),
                                                                self._stream()), "xd_tia_dense_solve_fallback")
            return
        _native.check(self._lib.xd_tia_dense_solve(self._tia, p(self.jac), p(self.rhs), p(self._lu_d),
                                                   p(self._piv_d), p(out), None, self._stream()),
                      "xd_tia_dense_solve")

    def _solve(self):
        if not self._small:
            return super()._solve()
        self._slu_ready(renew=getattr(self, "_first_solve", True))
        self._first_solve = False
        self._dense_solve(self._dx_d)
        if self._slu is not None:
            fell_back = int(self._fallback_d.item()) != 0
            self._lu_from_slu = not fell_back  # which kernel's factors _lu_d holds
            if fell_back:
                self._note_fallback()
        self._lu = "small"
        self.stats.factorizations += 1
        return self._dx_d.clone()

    def _solve_factored(self):
        if not self._small:
            return super()._solve_factored()
        out = self.torch.empty_like(self.rhs)
        p = self._ptr
        if self._slu is not None and getattr(self, "_lu_from_slu", False):
            _native.check(self._lib.xd_slu_resolve(self._slu, p(self._lu_d), p(self.rhs), p(out), self._stream()),
                          "xd_slu_resolve")
            return out
        _native.check(self._lib.xd_tia_dense_resolve(self._tia, p(self._lu_d), p(self._piv_d), p(self.rhs), p(out),
                                                     self._stream()), "xd_tia_dense_resolve")
        return out

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def _sync(self):
        self.torch.cuda.synchronize(self.dev)

    def _load(self, flags: SolverFlags):
        self._load_raw(flags)
        self.stats.loads += 1

    def _load_raw(self, flags: SolverFlags):
        c = flags.to_c()
        p = self._ptr
        _native.check(self._lib.xd_load_assign(self.fam._h, ctypes.byref(c), p(self.x), p(self.next_sta),
                                               p(self.curr_sta), p(self.next_sto), p(self.curr_sto), p(self.f),
                                               p(self.q), p(self.fx), p(self.qx), p(self.jf), p(self.jq),
                                               self._stream()), "xd_load_assign")

    def _set_sources(self, t):
        _native.check(self._lib.xd_pwl_eval(self._pwl, 0.0 if t is None else float(t), 0 if t is None else 1,
                                            self._ptr(self.b), self._stream()), "xd_pwl_eval")

    def _load_and_combine(self, flags, mode, h=None, order=1, qn0=None, fhist=None):
        self._load_combine_raw(flags, mode, h, order, qn0, fhist)
        self.stats.loads += 1

    def _load_combine_raw(self, flags, mode, h=None, order=1, qn0=None, fhist=None):
        if self._fused is None:
            self._load_raw(flags)
            self._combine(mode, h, order, qn0, fhist)
            return
        c = flags.to_c()
        coef = tia_coef(mode, h, order, self.gshunt)
        p = self._ptr
        _native.check(self._lib.xd_tia_load_combine(self._fused, ctypes.byref(c), ctypes.byref(coef), p(self.x),
                                                    p(self.next_sta), p(self.curr_sta), p(self.next_sto),
                                                    p(self.curr_sto), p(self.f), p(self.q), p(self.fx), p(self.qx),
                                                    p(self.jf), p(self.jq), p(self.lin_f), p(self.lin_q),
                                                    1 if self.limiting else 0, p(self.b), p(qn0), p(fhist),
                                                    p(self.jac), p(self.rhs), p(self.qtot), p(self.ftot),
                                                    self._stream()), "xd_tia_load_combine")

    def _surrogate_load(self):
        self.surrogate.load(self.x, self.f, self.q, self.fx, self.qx, self._stream())

    def _combine(self, mode, h=None, order=1, qn0=None, fhist=None):
        coef = tia_coef(mode, h, order, self.gshunt)
        p = self._ptr
        _native.check(self._lib.xd_tia_combine(self._tia, ctypes.byref(coef), p(self.x), p(self.jf), p(self.jq),
                                               p(self.lin_f), p(self.lin_q), p(self.f), p(self.q),
                                               p(self.fx) if self.limiting else None,
                                               p(self.qx) if self.limiting else None, p(self.b),
                                               p(qn0), p(fhist), p(self.jac), p(self.rhs), p(self.qtot),
                                               p(self.ftot), self._stream()), "xd_tia_combine")


def tia_coef(mode, h=None, order=1, gshunt=0.0) -> _native.XdTiaCoef:
    """Coefficients of the one-step method: backward Euler (order 1) or trapezoid (order 2)."""
    coef = _native.XdTiaCoef()
    coef.mode = mode
    coef.gshunt = gshunt
    if mode:
        coef.qscale = coef.inv_h = 1.0 / h
        coef.fscale = 0.5 if order == 2 else 1.0
        coef.hist_scale = 0.5 if order == 2 else 0.0
    else:
        coef.qscale, coef.fscale, coef.inv_h, coef.hist_scale = 0.0, 1.0, 0.0, 0.0
    return coef
