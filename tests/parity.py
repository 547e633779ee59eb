"""Shared helpers for parity tests: the same circuit through the oracle and through the C ABI."""
from __future__ import annotations

import math

import numpy as np

from oracle.run import OUTPUT_KEYS, SENS_SEEDS, OracleRun, flags_dict  # noqa: F401 (re-exported)
from xyce_b200 import netlist
from xyce_b200.device import ModelCard, SolverFlags  # noqa: F401

# Tolerance per entry: |a - b| <= RTOL * max(|a|, |b|) + ABS_SUM_FLOOR * S + ROW_FLOOR * R, where S
# is the entry's sum of absolute contributions (the two implementations sum the same terms in
# different orders) and, for Jacobian entries, R is the largest magnitude in the entry's row: an
# entry that is itself the rounding residue of cancelling capacitances (charge conservation makes
# some dQ/dx sums vanish analytically) carries noise of the order of eps times the row's scale,
# which any difference in the last bit of a capacitance changes. The limiter vectors dF/dx*dVp and
# dQ/dx*dVp are Jacobian rows times voltage steps, formed per instance as sums of terms that can
# cancel (the source entry is minus the gate, bulk and drain ones), so for them R is the matching
# Jacobian row's largest magnitude times V, the span of the node voltages (the largest step).
RTOL = 1e-12
ABS_SUM_FLOOR = 1e-14
ROW_FLOOR = 1e-14
# Conditioning: the oracle can rerun a load with every exp / log / log10 / pow result moved by one
# ulp (oracle/libm_perturb.C). The largest change of an entry over SENS_SEEDS such runs measures
# how much that entry depends on the last bit of the elementary functions; the GPU's functions and
# the host C library's may differ by an ulp, so each entry's tolerance also admits SENS_FACTOR
# times that change. Well-conditioned entries move by ~1e-16 relative and keep the 1e-12 bound;
# the ones this opens up are values formed by cancellation (the drain-bulk transconductance of a
# device deep in cut-off, for instance), which no implementation with a different libm can pin.
SENS_FACTOR = 4.0


def row_scale(rowptr, vals_a, vals_b):
    """Per-entry max |value| over the entry's CSR row (max over both operands)."""
    m = np.maximum(np.abs(vals_a), np.abs(vals_b))
    rows = np.repeat(np.arange(len(rowptr) - 1), np.diff(rowptr))
    rmax = np.zeros(len(rowptr) - 1)
    np.maximum.at(rmax, rows, m)
    return rmax[rows]


def row_max(rowptr, vals):
    """Per-row max |value| of CSR values (0 for an empty row)."""
    rows = np.repeat(np.arange(len(rowptr) - 1), np.diff(rowptr))
    rmax = np.zeros(len(rowptr) - 1)
    np.maximum.at(rmax, rows, np.abs(vals))
    return rmax


# (cards, inst_model, inst_nodes, inst_params) of a circuit's MOSFETs.
family_inputs = netlist.mosfet_family


def stamp_counts(rowptr, colind, inst_nodes, n_unknowns):
    """Contributions per output entry of a 4-terminal family: per vector row, the instance
    terminals on it; per CSR entry, the (row, column) terminal pairs of all instances on it."""
    nd = np.asarray(inst_nodes, dtype=np.int64).reshape(-1, 4)
    t = nd.reshape(-1)
    vec = np.bincount(t[t >= 0], minlength=n_unknowns).astype(np.float64)
    r = np.repeat(nd, 4, axis=1).reshape(-1)
    c = np.tile(nd, (1, 4)).reshape(-1)
    keep = (r >= 0) & (c >= 0)
    r, c = r[keep], c[keep]
    # CSR position of each pair (rows' columns are sorted, so (row, col) keys ascend).
    prow = np.repeat(np.arange(n_unknowns), np.diff(rowptr)).astype(np.int64)
    full = prow * (n_unknowns + 1) + np.asarray(colind, dtype=np.int64)
    pos = np.searchsorted(full, r * (n_unknowns + 1) + c)
    mat = np.bincount(pos, minlength=int(rowptr[-1])).astype(np.float64)
    return {"f": vec, "q": vec, "dfdxdvp": vec, "dqdxdvp": vec, "dfdx": mat, "dqdx": mat}


def strict_split(got, ref, rtol=RTOL):
    """(entries, entries within the plain bound |a - b| <= rtol * max(|a|, |b|), indices of the
    others): how many entries needed one of the floors of compare() to pass."""
    got = np.asarray(got).reshape(-1)
    ref = np.asarray(ref).reshape(-1)
    d = np.abs(got - ref)
    ok = d <= rtol * np.maximum(np.abs(got), np.abs(ref))
    return int(ok.size), int(np.count_nonzero(ok)), np.flatnonzero(~ok)


def _allowances(got, ref, abs_sum, rtol, floor, rowptr, sens, vec_scale, nterms):
    """compare()'s allowed error per entry, cumulatively by floor: plain relative; + the abs-sum
    (summation-order) floor; + the row / vector-scale (cancellation) floor; + the libm sensitivity."""
    a0 = rtol * np.maximum(np.abs(got), np.abs(ref))
    a1 = a0
    if abs_sum is not None:
        fl = floor
        if nterms is not None:
            fl = np.maximum(floor, 2.0 * np.maximum(np.asarray(nterms, dtype=np.float64) - 1.0, 0.0) * 2.0 ** -53)
        a1 = a1 + fl * np.asarray(abs_sum)
    a2 = a1
    if rowptr is not None:
        a2 = a2 + ROW_FLOOR * row_scale(rowptr, got, ref)
    if vec_scale is not None:
        a2 = a2 + ROW_FLOOR * np.asarray(vec_scale)
    a3 = a2
    if sens is not None:
        a3 = a3 + SENS_FACTOR * np.asarray(sens).reshape(a3.shape)
    return a0, a1, a2, a3


def floor_classes(got, ref, abs_sum=None, rtol=RTOL, floor=ABS_SUM_FLOOR, rowptr=None, sens=None, vec_scale=None,
                  nterms=None):
    """Of the entries outside plain rtol relative: how many pass once the abs-sum floor is added
    (summation order), how many need the row / vector-scale floor too (cancellation residue), and
    how many the libm sensitivity as well (one-ulp conditioning)."""
    got = np.asarray(got)
    ref = np.asarray(ref)
    d = np.abs(got - ref)
    a0, a1, a2, a3 = _allowances(got, ref, abs_sum, rtol, floor, rowptr, sens, vec_scale, nterms)
    return (int(np.count_nonzero((d > a0) & (d <= a1))), int(np.count_nonzero((d > a1) & (d <= a2))),
            int(np.count_nonzero((d > a2) & (d <= a3))))


def compare(name, got, ref, abs_sum=None, rtol=RTOL, floor=ABS_SUM_FLOOR, rowptr=None, detail=None, sens=None,
            vec_scale=None, nterms=None):
    """Returns (n_bad, worst ratio of |diff| to the allowed error). With rowptr (CSR values), adds
    the row-scaled floor; with vec_scale (per-entry R of a limiter vector), ROW_FLOOR times it;
    with sens (the oracle's one-ulp sensitivity of each entry), adds SENS_FACTOR times it. With
    nterms (each entry's number of summed contributions), the abs-sum floor is at least the bound
    of recursive summation, (n - 1) u S per side with u = 2^-53: an entry summed from a million
    instances (a supply rail) differs by summation order alone far above 1e-14 S. If `detail` is
    a list, the worst offenders are appended to it."""
    got = np.asarray(got)
    ref = np.asarray(ref)
    d = np.abs(got - ref)
    allow = _allowances(got, ref, abs_sum, rtol, floor, rowptr, sens, vec_scale, nterms)[3]
    allow = np.maximum(allow, 1e-300)
    ratio = d / allow
    bad = int(np.count_nonzero(d > allow))
    worst = float(ratio.max()) if ratio.size else 0.0
    if detail is not None and bad:
        for k in np.argsort(-ratio)[:5]:
            detail.append((name, int(k), float(got.flat[k]), float(ref.flat[k]), float(allow.flat[k])))
    return bad, worst
