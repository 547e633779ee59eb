"""Generates the committed golden fixtures from the oracle (the reference's own device code).

    python tests/golden/make_golden.py

Each fixture holds one small seeded circuit, a sequence of solver-flag steps, and for every
step the inputs (solution, state, store) and the oracle's outputs (F, Q, dFdxdVp, dQdxdVp,
dF/dx and dQ/dx on the product's CSR pattern, new state and store). Tests use them to pin the
oracle build and to check the CUDA path where the oracle library is not available.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.parity import OracleRun, family_inputs, flags_dict  # noqa: E402
from xyce_b200 import ModelCard, SolverFlags, netlist  # noqa: E402

CASES = {
    "bsim4_logic_default": dict(n=240, seed=101, cards=None, vrange=(0.0, 1.2)),
    "bsim4_logic_swing": dict(n=200, seed=102, cards=[ModelCard(False, {"DIOMOD": 2}), ModelCard(True, {"DIOMOD": 0})],
                              vrange=(-1.5, 4.0)),
    "bsim4_ring_card": dict(n=0, seed=103, cards=[ModelCard(False, {"MOBMOD": 1, "TOXE": 2.5e-9, "VTH0": 0.45}),
                                                   ModelCard(True, {"MOBMOD": 2, "VTH0": -0.42, "XPART": 0.5})],
                            vrange=(0.0, 1.8)),
}
SEQ = [SolverFlags(newton_iter=1, voltlim=0), SolverFlags(newton_iter=1), SolverFlags(newton_iter=2),
       SolverFlags(newton_iter=0, init_tran=1), SolverFlags(dcop=1, transient=0, newton_iter=1)]


def make(name, spec):
    c = netlist.inverter_ring(15, vdd=1.8) if spec["n"] == 0 else netlist.random_logic(spec["n"], seed=spec["seed"])
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c, spec["cards"])
    orc = OracleRun(c, cards, im, nd, params, rowptr, colind)
    n = im.shape[0]
    rng = np.random.default_rng(spec["seed"])
    sta_n, sta_c, sto_n, sto_c = np.zeros(3 * n), np.zeros(3 * n), np.zeros(14 * n), np.zeros(14 * n)
    out = dict(rowptr=rowptr, colind=colind, inst_model=im, inst_nodes=nd, L=params["L"], W=params["W"],
               n_unknowns=c.n_unknowns, n_steps=len(SEQ))
    cards_txt = [f"{int(m.pmos)}:" + ",".join(f"{k}={v!r}" for k, v in m.params.items()) for m in cards]
    out["cards"] = np.array(cards_txt)
    for s, fl in enumerate(SEQ):
        sol = rng.uniform(spec["vrange"][0], spec["vrange"][1], c.n_unknowns)
        r = orc.load(fl, sol, sta_n, sta_c, sto_n, sto_c)
        out[f"s{s}_flags"] = np.array([flags_dict(fl)[k] for k in ("dcop", "init_tran", "newton_iter", "init_jct",
                                                                   "init_fix", "transient", "tranop", "acop",
                                                                   "voltlim", "input_op", "gmin", "pdt")])
        for k, v in dict(sol=sol, in_next_sta=sta_n, in_curr_sta=sta_c, in_next_sto=sto_n, in_curr_sto=sto_c).items():
            out[f"s{s}_{k}"] = v
        for k, v in r.items():
            out[f"s{s}_{k}"] = v
        sta_n, sta_c, sto_n = r["next_sta"], r["curr_sta"], r["next_sto"]
        if fl.newton_iter == 0:
            sto_c = r["next_sto"].copy()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


if __name__ == "__main__":
    for name, spec in CASES.items():
        make(name, spec)
        print("wrote", name)
