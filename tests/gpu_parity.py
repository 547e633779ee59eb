"""GPU-side parity machinery shared by the family test files (needs torch and a CUDA device)."""
import os

import numpy as np
import torch

from tests.parity import (ABS_SUM_FLOOR, RTOL, OracleRun, compare, family_inputs, floor_classes, row_max,
                          strict_split)
from xyce_b200 import MosfetDevice, netlist


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


class GpuRun:
    def __init__(self, dev: MosfetDevice, nnz: int, n_unknowns: int):
        self.dev, self.nnz, self.nu = dev, nnz, n_unknowns

    def load(self, flags, sol, next_sta, curr_sta, next_sto, curr_sto):
        nu, nnz = self.nu, self.nnz
        t = dict(sol=_dev(sol), next_sta=_dev(next_sta), curr_sta=_dev(curr_sta), next_sto=_dev(next_sto),
                 curr_sto=_dev(curr_sto))
        outs = {k: torch.zeros(nu, dtype=torch.float64, device="cuda") for k in ("f", "q", "dfdxdvp", "dqdxdvp")}
        outs["dfdx"] = torch.zeros(nnz, dtype=torch.float64, device="cuda")
        outs["dqdx"] = torch.zeros(nnz, dtype=torch.float64, device="cuda")
        self.dev.update_state(flags, t["sol"], t["next_sta"], t["curr_sta"], t["next_sto"], t["curr_sto"])
        self.dev.load_dae_vectors(outs["f"], outs["q"], outs["dfdxdvp"], outs["dqdxdvp"])
        self.dev.load_dae_matrices(outs["dfdx"], outs["dqdx"])
        sums = {k: torch.zeros_like(v) for k, v in outs.items()}
        self.dev.load_abs(sums["f"], sums["q"], sums["dfdxdvp"], sums["dqdxdvp"], sums["dfdx"], sums["dqdx"])
        torch.cuda.synchronize()
        res = {k: v.cpu().numpy() for k, v in outs.items()}
        res["next_sta"] = t["next_sta"].cpu().numpy()
        res["curr_sta"] = t["curr_sta"].cpu().numpy()
        res["next_sto"] = t["next_sto"].cpu().numpy()
        res["abs"] = {k: v.cpu().numpy() for k, v in sums.items()}
        return res


# Per parity test: (test id, {output: [entries, entries within plain 1e-12 relative, indices that
# needed a floor]}); tests/conftest.py prints it after the run and writes it to $PARITY_REPORT.
STRICT_LOG = []


def log_strict(strict):
    STRICT_LOG.append((os.environ.get("PYTEST_CURRENT_TEST", "").split(" ")[0], strict))


# Store slots each family writes (BSIM4 leaves vged / vgmd untouched, N_DEV_MOSFET_B4.C:16195-16210).
STORE_WRITTEN = {14: [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 13], 9: [0, 1, 2, 3, 4], 1: [0, 1, 2, 3, 4]}


def _tally(strict, key, got, ref, classes=(0, 0, 0)):
    """Adds (entries, entries within plain 1e-12 relative) of one output to `strict`, a dict of
    [entries, strict passes, first few indices that needed a floor, [summation-order,
    cancellation, libm-ulp] counts of the floors those entries needed (tests.parity.floor_classes)]."""
    if strict is None:
        return
    tot, ok, idx = strict_split(got, ref)
    t = strict.setdefault(key, [0, 0, [], [0, 0, 0]])
    t[0] += tot
    t[1] += ok
    if len(t[2]) < 8:
        t[2].extend(int(i) for i in idx[:8 - len(t[2])])
    for j in range(3):
        t[3][j] += classes[j]


def check_step(step, flags, g, r, n, charges=True, rowptr=None, level=14, n_sta=3, n_sto=14, vspan=None,
               strict=None, counts=None):
    """Compares one load of every output within the parity tolerance. With `strict` (a dict), also
    counts per output how many entries pass at plain 1e-12 relative, without any floor. `counts`
    (output -> contributions per entry, tests.parity.stamp_counts) widens the abs-sum floor of
    entries summed from very many instances to the summation-order bound."""
    report = {}
    keys = ["f", "dfdxdvp", "dfdx"] + (["q", "dqdxdvp", "dqdx"] if charges else [])
    for k in keys:
        detail = []
        vec_scale = None
        if vspan is not None and rowptr is not None and k in ("dfdxdvp", "dqdxdvp"):
            m = "dfdx" if k == "dfdxdvp" else "dqdx"
            vec_scale = vspan * np.maximum(row_max(rowptr, r[m]), row_max(rowptr, g[m]))
        kw = dict(rowptr=rowptr if k in ("dfdx", "dqdx") else None, sens=r["sens"][k] if "sens" in r else None,
                  vec_scale=vec_scale, nterms=None if counts is None else counts.get(k))
        bad, worst = compare(k, g[k], r[k], g["abs"][k], RTOL, ABS_SUM_FLOOR, detail=detail, **kw)
        report[k] = worst
        _tally(strict, k, g[k], r[k], floor_classes(g[k], r[k], g["abs"][k], RTOL, ABS_SUM_FLOOR, **kw))
        assert bad == 0, (f"step {step} {flags}: {k} has {bad} entries out of tolerance (worst {worst:.3g}x); "
                          f"(name, index, gpu, ref, allowed): {detail}")
    gs = g["next_sto"].reshape(n_sto, n)[STORE_WRITTEN[level]]
    rs = r["next_sto"].reshape(n_sto, n)[STORE_WRITTEN[level]]
    ss = r["sens"]["next_sto"].reshape(n_sto, n)[STORE_WRITTEN[level]] if "sens" in r else None
    bad, worst = compare("sto", gs, rs, sens=ss)
    _tally(strict, "next_sto", gs, rs, floor_classes(gs, rs, sens=ss))
    assert bad == 0, f"step {step}: store out of tolerance ({worst:.3g}x)"
    if charges:
        # Charges are sums of cancelling terms: the floor is 1e-14 of the instance's largest charge.
        scale = np.abs(r["next_sta"]).reshape(n_sta, n).max(0)
        detail = []
        bad, worst = compare("sta", g["next_sta"].reshape(n_sta, n), r["next_sta"].reshape(n_sta, n),
                             np.broadcast_to(scale, (n_sta, n)), RTOL, ABS_SUM_FLOOR, detail=detail,
                             sens=r["sens"]["next_sta"].reshape(n_sta, n) if "sens" in r else None)
        report["sta"] = worst
        _tally(strict, "next_sta", g["next_sta"], r["next_sta"],
               floor_classes(g["next_sta"].reshape(n_sta, n), r["next_sta"].reshape(n_sta, n),
                             np.broadcast_to(scale, (n_sta, n)), RTOL, ABS_SUM_FLOOR,
                             sens=r["sens"]["next_sta"].reshape(n_sta, n) if "sens" in r else None))
        assert bad == 0, f"step {step}: state out of tolerance ({worst:.3g}x): {detail}"
        if level in (9, 14) and flags.init_tran and flags.newton_iter == 0 and not flags.dcop:
            assert np.allclose(g["curr_sta"], g["next_sta"], rtol=0, atol=0)
    return report


def run_sequence(c, cards, seqs, vrange=(0.0, 1.2), seed=0, extra_params=None, charges_in_dc=False, level=14,
                 eval_variant=None):
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, inst_model, inst_nodes, params = family_inputs(c, cards, extra_params)
    dev = MosfetDevice(cards, inst_model, inst_nodes, params, (rowptr, colind), c.n_unknowns, level=level,
                       inst_internal=c.mos_internal)
    if eval_variant is not None:
        assert dev._lib.xd_set_eval_variant(dev._h, eval_variant) == 0
    orc = OracleRun(c, cards, inst_model, inst_nodes, params, rowptr, colind, level=level,
                    n_sta_slots=dev.n_state_slots)
    gpu = GpuRun(dev, int(rowptr[-1]), c.n_unknowns)
    n = inst_model.shape[0]
    n_sta, n_sto = dev.n_state_slots, dev.n_store_slots
    assert (n_sta, n_sto) == (orc.n_sta_slots, orc.n_sto_slots)
    rng = np.random.default_rng(seed)
    sta_n, sta_c = np.zeros(n_sta * n), np.zeros(n_sta * n)
    sto_n, sto_c = np.zeros(n_sto * n), np.zeros(n_sto * n)
    worst, strict = {}, {}
    for step, flags in enumerate(seqs):
        sol = rng.uniform(vrange[0], vrange[1], c.n_unknowns)
        r = orc.load_with_sensitivity(flags, sol, sta_n, sta_c, sto_n, sto_c)
        g = gpu.load(flags, sol, sta_n, sta_c, sto_n, sto_c)
        charges = bool(flags.transient or flags.tranop or flags.acop) or charges_in_dc
        rep = check_step(step, flags, g, r, n, charges, rowptr, level, n_sta, n_sto, vspan=vrange[1] - vrange[0],
                         strict=strict)
        for k, v in rep.items():
            worst[k] = max(worst.get(k, 0.0), v)
        # Both sides continue from the oracle's state and store; a step that ends a time point
        # (Newton step 0 of a new step, or any DC step) also becomes the "current" history.
        sta_n, sta_c, sto_n = r["next_sta"], r["curr_sta"], r["next_sto"]
        if flags.newton_iter == 0 or flags.dcop:
            sto_c = r["next_sto"].copy()
            if level == 1:
                sta_c = r["next_sta"].copy()
    dev.close()
    log_strict(strict)
    return worst




# Waveform comparison. RELTOL is the configs' transient reltol; VNTOL the reference's default node
# voltage tolerance (the absolute part of its per-point Newton weights, N_NLS_NLParams.C).
WAVE_RELTOL, WAVE_VNTOL = 1e-3, 1e-6


def waveform_errors(wg, wo):
    """Worst error of waveforms wg against wo (points x nodes) as fractions of two bounds: per node,
    reltol times the node's largest magnitude over the window; per point, reltol times the larger
    of the two values there plus VNTOL. Both must be at most 1."""
    err = np.abs(wg - wo)
    scaled = float((err / (WAVE_RELTOL * np.abs(wo).max(axis=0, keepdims=True) + 1e-12)).max())
    point = float((err / (WAVE_RELTOL * np.maximum(np.abs(wg), np.abs(wo)) + WAVE_VNTOL)).max())
    return scaled, point
