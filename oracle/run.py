"""The reference's own device objects driven over a circuit: the oracle side of every device-load
parity check (test infrastructure).

OracleRun builds the reference's MOSFET instances (oracle/_ref, compiled from the reference's
sources by oracle/Makefile) for a circuit's MOSFET family, numbers their internal nodes as the
reference's topology does, registers the product's Jacobian pattern (plus the entries the
reference's stamps reach), and loads them through the reference's own updateState /
loadDAEVectors / loadDAEMatrices (N_DEV_DeviceMgr.C, N_DEV_MOSFET_B4.C:5200-5267 for the state and
store LIDs). Outputs come back in the product's layouts: unknown-indexed vectors, the product's
CSR order, slot-major state and store.

Only the tests, the smoke check and the bench's CPU-baseline and reference legs use this module.
"""
from __future__ import annotations

import numpy as np

from oracle import xyce_ref as xr
from xyce_b200 import netlist
from xyce_b200.device import SolverFlags

# One-ulp libm perturbation seeds for the conditioning reruns, and the outputs compared.
SENS_SEEDS = (101, 202)
OUTPUT_KEYS = ("f", "q", "dfdxdvp", "dqdxdvp", "dfdx", "dqdx", "next_sta", "next_sto")


def flags_dict(f: SolverFlags) -> dict:
    return dict(dcop=f.dcop, init_tran=f.init_tran, newton_iter=f.newton_iter, init_jct=f.init_jct,
                init_fix=f.init_fix, transient=f.transient, tranop=f.tranop, acop=f.acop, voltlim=f.voltlim,
                input_op=f.input_op, gmin=f.gmin, pdt=f.pdt)


class OracleRun:
    """The reference's own device objects for the circuit's MOSFETs, on the product's pattern."""

    def __init__(self, c: netlist.Circuit, cards, inst_model, inst_nodes, params, rowptr, colind, level=14,
                 n_sta_slots=None, gpu_binding=False):
        self.c = c
        models = [(m.pmos, dict(m.params)) for m in cards]
        nu = c.n_unknowns
        # The reference numbers its internal nodes after the external unknowns, in instance order.
        # gpu_binding: the reference's own device loop with the product's binding as the device master.
        self.ref = xr.RefCircuit(level, models, inst_model, inst_nodes, params, nu - c.n_internal,
                                 gpu_binding=gpu_binding)
        assert self.ref.n_unknowns == nu, "the oracle's internal nodes differ from the circuit's"
        n = inst_model.shape[0]
        # Oracle pattern: the product's pattern plus the ground row / column entries the stamps hit.
        g = nu
        pairs = [np.stack([np.repeat(np.arange(nu), np.diff(rowptr)), colind], 1)]
        nd = np.where(inst_nodes < 0, g, inst_nodes).astype(np.int64)
        rr = np.repeat(nd, 4, axis=1).reshape(-1)
        cc = np.tile(nd, (1, 4)).reshape(-1)
        pairs.append(np.stack([rr, cc], 1))
        extra_pairs = np.zeros((0, 2), dtype=np.int64)
        if c.n_internal:
            # With internal nodes the reference's stamps reach beyond the terminal block: add them.
            # Its stamp can hold entries the product's pattern lacks (the sheet-resistance stamp
            # has the external drain's couplings to G', S', B', which only rdsMod 1 loads); each
            # load below checks that the reference leaves those at zero, so that nothing the
            # reference loads drops out of the comparison.
            ref_pairs = []
            for i in range(n):
                sr, sc = self.ref.stamp(i)
                ref_pairs.append(np.stack([np.asarray(sr, np.int64), np.asarray(sc, np.int64)], 1))
            pairs += ref_pairs
            rp = np.concatenate(ref_pairs, 0)
            rp = rp[(rp[:, 0] < g) & (rp[:, 1] < g)]
            prow_ = np.repeat(np.arange(nu), np.diff(rowptr)).astype(np.int64)
            have = np.isin(rp[:, 0] * (nu + 1) + rp[:, 1], prow_ * (nu + 1) + colind)
            extra_pairs = np.unique(rp[~have], axis=0)
        pr = np.concatenate(pairs, 0)
        key = np.unique(pr[:, 0] * (nu + 1) + pr[:, 1])
        rows, cols = key // (nu + 1), (key % (nu + 1)).astype(np.int32)
        orp = np.zeros(nu + 2, dtype=np.int64)
        np.add.at(orp, rows + 1, 1)
        orp = np.cumsum(orp).astype(np.int32)
        self.ref.set_pattern(orp, cols)
        # Map each product CSR entry to the oracle CSR entry with the same (row, col).
        prow = np.repeat(np.arange(nu), np.diff(rowptr))
        okey = rows * (nu + 1) + cols
        self.map = np.searchsorted(okey, prow * (nu + 1) + colind)
        self.extra = np.searchsorted(okey, extra_pairs[:, 0] * (nu + 1) + extra_pairs[:, 1])
        self.n = n
        self.sta_base = np.array([self.ref.state_base(i) for i in range(n)], dtype=np.int64)
        self.sto_base = np.array([self.ref.store_base(i) for i in range(n)], dtype=np.int64)
        # The reference may reserve more state entries per instance than the load writes (BSIM3
        # reserves 12 and writes the first 5 without NQS); the product keeps only the written ones.
        self.n_sta_slots = self.ref.n_state // max(1, n) if n_sta_slots is None else n_sta_slots
        self.n_sto_slots = self.ref.n_store // max(1, n)
        # sta_off[s, i]: the oracle's state entry of product slot s of instance i (-1: none).
        self.sta_off = self.sta_base[None, :] + np.arange(self.n_sta_slots)[:, None]
        if c.mos_internal is not None and c.mos_internal.shape[1] == netlist.GEN_NODES - 4:
            # General topology: the product keeps (qb, qg, qd, qgmid, qbs, qbd, qcheq, qcdump); an
            # instance registers qgmid only with rgateMod 3, qbs / qbd only with rbodyMod and
            # qcheq / qcdump only with trnqsMod (registerStateLIDs, N_DEV_MOSFET_B4.C:5212-5238).
            rg3 = (c.mos_internal[:, 3] >= 0).astype(np.int64)
            rb = c.mos_internal[:, 4] >= 0
            nq = c.mos_internal[:, 7] >= 0
            self.n_sta_slots = 8
            b = self.sta_base
            q0 = b + 3 + rg3 + 2 * rb.astype(np.int64)
            self.sta_off = np.stack([b, b + 1, b + 2, np.where(rg3 == 1, b + 3, -1), np.where(rb, b + 3 + rg3, -1),
                                     np.where(rb, b + 4 + rg3, -1), np.where(nq, q0, -1), np.where(nq, q0 + 1, -1)])

    def to_aos_sto(self, soa):
        """Product slot-major store block -> oracle per-instance layout."""
        out = np.zeros(max(1, self.ref.n_store))
        for s in range(self.n_sto_slots):
            out[self.sto_base + s] = soa[s * self.n:(s + 1) * self.n]
        return out

    def to_aos_sta(self, soa):
        out = np.zeros(max(1, self.ref.n_state))
        for s in range(self.n_sta_slots):
            has = self.sta_off[s] >= 0
            out[self.sta_off[s][has]] = soa[s * self.n:(s + 1) * self.n][has]
        return out

    def from_aos_sto(self, aos):
        return np.concatenate([aos[self.sto_base + s] for s in range(self.n_sto_slots)])

    def from_aos_sta(self, aos):
        return np.concatenate([np.where(self.sta_off[s] >= 0, aos[np.maximum(self.sta_off[s], 0)], 0.0)
                               for s in range(self.n_sta_slots)])

    def load(self, flags: SolverFlags, sol, next_sta_soa, curr_sta_soa, next_sto_soa, curr_sto_soa,
             perturb_seed=None):
        nu = self.c.n_unknowns
        s = np.zeros(nu + 1)
        s[:nu] = sol
        out = self.ref.load(xr.make_flags(**flags_dict(flags)), s, self.to_aos_sta(next_sta_soa),
                            self.to_aos_sta(curr_sta_soa), self.to_aos_sto(next_sto_soa),
                            self.to_aos_sto(curr_sto_soa), perturb_seed=perturb_seed)
        if self.extra.size:
            assert not out.dfdx[self.extra].any() and not out.dqdx[self.extra].any(), \
                "the reference loads entries outside the product's pattern"
        return dict(f=out.f[:nu], q=out.q[:nu], dfdxdvp=out.dfdxdvp[:nu], dqdxdvp=out.dqdxdvp[:nu],
                    dfdx=out.dfdx[self.map], dqdx=out.dqdx[self.map], next_sta=self.from_aos_sta(out.next_sta),
                    curr_sta=self.from_aos_sta(out.curr_sta), next_sto=self.from_aos_sto(out.next_sto))

    def load_with_sensitivity(self, flags: SolverFlags, sol, next_sta_soa, curr_sta_soa, next_sto_soa,
                              curr_sto_soa):
        """The load, plus r["sens"][key]: per entry, the largest change over the one-ulp-perturbed
        reruns. The perturbed runs go first so that the device objects' carried state (BSIM4
        keeps the previous load's vgb) ends as the unperturbed load leaves it."""
        pert = [self.load(flags, sol, next_sta_soa, curr_sta_soa, next_sto_soa, curr_sto_soa, perturb_seed=sd)
                for sd in SENS_SEEDS]
        r = self.load(flags, sol, next_sta_soa, curr_sta_soa, next_sto_soa, curr_sto_soa)
        r["sens"] = {k: np.max([np.abs(p[k] - r[k]) for p in pert], axis=0) for k in OUTPUT_KEYS}
        return r
