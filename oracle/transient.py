"""The transient driver of xyce_b200.transient run on the oracle: the reference's own device loads
(compiled from its sources, oracle/) and a numpy restatement of the combine step, on CPU tensors.

Test infrastructure: the GPU transient is compared with this one step by step, through the same
integrator and Newton loop, so that waveform differences measure the device-load path alone.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch

from oracle.run import OracleRun
from xyce_b200.netlist import mosfet_family as family_inputs
from xyce_b200.device import SolverFlags
from xyce_b200.transient import TransientBase


class OracleTransient(TransientBase):
    def __init__(self, c, cards, rowptr, colind, level=14, extra_params=None, solver="auto", gmin=1e-12):
        cards, im, nd, params = family_inputs(c, cards, extra_params)
        self.orc = OracleRun(c, cards, im, nd, params, rowptr, colind, level=level)
        n = im.shape[0]
        super().__init__(c, self.orc.n_sta_slots * n, self.orc.n_sto_slots * n, rowptr, colind, torch.device("cpu"),
                         solver, gmin)
        nu = self.nu
        self.Af = sp.csr_matrix((self.lin.lin_f, self.colind, self.rowptr), shape=(nu, nu))
        self.Aq = sp.csr_matrix((self.lin.lin_q, self.colind, self.rowptr), shape=(nu, nu))
        self._r = None
        rows = np.repeat(np.arange(nu), np.diff(self.rowptr))
        self._diag = (rows == self.colind).astype(float)
        self._has_diag = np.zeros(nu)
        self._has_diag[rows[rows == self.colind]] = 1.0  # the shunt's rows: node rows, not branch rows

    def _load(self, flags: SolverFlags):
        r = self.orc.load(flags, self.x.numpy(), self.next_sta.numpy(), self.curr_sta.numpy(), self.next_sto.numpy(),
                          self.curr_sto.numpy())
        self.next_sta.copy_(torch.as_tensor(r["next_sta"]))
        self.curr_sta.copy_(torch.as_tensor(r["curr_sta"]))
        self.next_sto.copy_(torch.as_tensor(r["next_sto"]))
        self._r = r
        self.stats.loads += 1

    def _combine(self, mode, h=None, order=1, qn0=None, fhist=None):
        r = self._r
        x = self.x.numpy()
        jf = r["dfdx"] + self.lin.lin_f
        F = r["f"] + self.Af @ x
        if self.gshunt:
            jf = jf + self.gshunt * self._diag
            F = F + self.gshunt * self._has_diag * x
        F = F - self.b.numpy()
        self.ftot.copy_(torch.as_tensor(F))
        if mode == 0:
            self.jac.copy_(torch.as_tensor(jf))
            rhs = -F
            if self.limiting:
                rhs = rhs + r["dfdxdvp"]
            self.rhs.copy_(torch.as_tensor(rhs))
            return
        inv_h = 1.0 / h
        fs = 0.5 if order == 2 else 1.0
        jq = r["dqdx"] + self.lin.lin_q
        Q = r["q"] + self.Aq @ x
        self.qtot.copy_(torch.as_tensor(Q))
        self.jac.copy_(torch.as_tensor(inv_h * jq + fs * jf))
        res = (Q - qn0.numpy()) * inv_h + fs * F
        if order == 2:
            res = res + 0.5 * fhist.numpy()
        res = -res
        if self.limiting:
            res = res + inv_h * r["dqdxdvp"]
            res = res + fs * r["dfdxdvp"]
        self.rhs.copy_(torch.as_tensor(res))
