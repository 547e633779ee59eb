"""Golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py from the oracle).

* The oracle reproduces every fixture bit for bit (pins the oracle build: shims, harness, flags).
* The CUDA path matches every fixture within the parity tolerance (needs no oracle library).
"""
import glob
import os

import numpy as np
import pytest

from tests.parity import ABS_SUM_FLOOR, RTOL, compare
from xyce_b200 import ModelCard, SolverFlags, netlist

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
FLAG_KEYS = ("dcop", "init_tran", "newton_iter", "init_jct", "init_fix", "transient", "tranop", "acop", "voltlim",
             "input_op", "gmin", "pdt")


def _cards(z):
    out = []
    for t in z["cards"]:
        pm, rest = str(t).split(":", 1)
        params = {}
        for kv in filter(None, rest.split(",")):
            k, v = kv.split("=")
            params[k] = float(v)
        out.append(ModelCard(bool(int(pm)), params))
    return out


def _flags(arr):
    d = {k: (float(v) if k in ("gmin", "pdt") else int(v)) for k, v in zip(FLAG_KEYS, arr)}
    return SolverFlags(**d)


def _circuit(z):
    nu = int(z["n_unknowns"])
    c = netlist.Circuit(n_nodes=nu, mos_type=z["inst_model"], mos_nodes=z["inst_nodes"], mos_w=z["W"], mos_l=z["L"],
                        res_nodes=np.zeros((0, 2), np.int32), res_value=np.zeros(0),
                        cap_nodes=np.zeros((0, 2), np.int32), cap_value=np.zeros(0),
                        vsrc_nodes=np.zeros((0, 2), np.int32), vsrc_dc=np.zeros(0))
    return c


def test_fixtures_exist():
    assert len(FIXTURES) >= 3


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_oracle_reproduces_golden(path):
    from oracle import xyce_ref as xr

    if not xr.available():
        pytest.skip("oracle library not built")
    from tests.parity import OracleRun

    z = np.load(path)
    c = _circuit(z)
    cards = _cards(z)
    orc = OracleRun(c, cards, z["inst_model"], z["inst_nodes"], {"L": z["L"], "W": z["W"]}, z["rowptr"], z["colind"])
    for s in range(int(z["n_steps"])):
        fl = _flags(z[f"s{s}_flags"])
        r = orc.load(fl, z[f"s{s}_sol"], z[f"s{s}_in_next_sta"], z[f"s{s}_in_curr_sta"], z[f"s{s}_in_next_sto"],
                     z[f"s{s}_in_curr_sto"])
        for k in ("f", "q", "dfdxdvp", "dqdxdvp", "dfdx", "dqdx", "next_sta", "next_sto"):
            assert np.array_equal(r[k], z[f"s{s}_{k}"]), (s, k)


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_gpu_matches_golden(path):
    torch = pytest.importorskip("torch")
    from xyce_b200 import Bsim4Device

    z = np.load(path)
    nu = int(z["n_unknowns"])
    n = z["inst_model"].shape[0]
    nnz = int(z["rowptr"][-1])
    dev = Bsim4Device(_cards(z), z["inst_model"], z["inst_nodes"], {"L": z["L"], "W": z["W"]},
                      (z["rowptr"], z["colind"]), nu)
    cu = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")
    for s in range(int(z["n_steps"])):
        fl = _flags(z[f"s{s}_flags"])
        sol, nsta, csta = cu(z[f"s{s}_sol"]), cu(z[f"s{s}_in_next_sta"]), cu(z[f"s{s}_in_curr_sta"])
        nsto, csto = cu(z[f"s{s}_in_next_sto"]), cu(z[f"s{s}_in_curr_sto"])
        o = {k: torch.zeros(nu, dtype=torch.float64, device="cuda") for k in ("f", "q", "dfdxdvp", "dqdxdvp")}
        o["dfdx"] = torch.zeros(nnz, dtype=torch.float64, device="cuda")
        o["dqdx"] = torch.zeros(nnz, dtype=torch.float64, device="cuda")
        dev.load(fl, sol, nsta, csta, nsto, csto, o["f"], o["q"], o["dfdxdvp"], o["dqdxdvp"], o["dfdx"], o["dqdx"])
        a = {k: torch.zeros_like(v) for k, v in o.items()}
        dev.load_abs(a["f"], a["q"], a["dfdxdvp"], a["dqdxdvp"], a["dfdx"], a["dqdx"])
        torch.cuda.synchronize()
        charges = bool(fl.transient or fl.tranop or fl.acop)
        keys = ["f", "dfdxdvp", "dfdx"] + (["q", "dqdxdvp", "dqdx"] if charges else [])
        for k in keys:
            bad, worst = compare(k, o[k].cpu().numpy(), z[f"s{s}_{k}"], a[k].cpu().numpy(), RTOL, ABS_SUM_FLOOR,
                                 rowptr=z["rowptr"] if k in ("dfdx", "dqdx") else None)
            assert bad == 0, f"{os.path.basename(path)} step {s}: {k} {bad} entries off ({worst:.3g}x tolerance)"
        written = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 13]
        g = nsto.cpu().numpy().reshape(14, n)[written]
        r = z[f"s{s}_next_sto"].reshape(14, n)[written]
        assert compare("sto", g, r)[0] == 0
    dev.close()
