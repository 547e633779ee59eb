"""The oracle itself (the reference's device code compiled by oracle/Makefile): sanity and pins.

These run on CPU. The oracle is test infrastructure; parity tests compare the CUDA path to it.
"""
import numpy as np
import pytest

from oracle import xyce_ref as xr

pytestmark = pytest.mark.skipif(not xr.available(), reason="oracle library not built")


def _one_nmos(params=None, level=14):
    ref = xr.RefCircuit(level, [(False, {})], np.array([0]), np.array([[0, 1, -1, -1]]),
                        params or {"L": np.array([0.18e-6]), "W": np.array([1e-6])}, 2)
    rows, cols = ref.stamp(0)
    nv = ref.n_unknowns + 1
    ent = sorted(set(zip(rows.tolist(), cols.tolist())))
    rowptr = np.zeros(nv + 1, dtype=np.int32)
    for r, _ in ent:
        rowptr[r + 1] += 1
    rowptr = np.cumsum(rowptr).astype(np.int32)
    ref.set_pattern(rowptr, np.array([c for _, c in ent], dtype=np.int32))
    return ref


def test_bsim4_default_topology_has_no_internal_nodes():
    ref = _one_nmos()
    assert ref.n_unknowns == 2
    assert ref.n_state == 3 and ref.n_store == 14


def test_bsim4_kcl_and_symmetry_of_charge():
    ref = _one_nmos()
    sol = np.array([1.0, 1.2, 0.0])
    out = ref.load(xr.make_flags(newton_iter=1, voltlim=0), sol, np.zeros(3), np.zeros(3), np.zeros(14), np.zeros(14))
    # Drain current flows into the drain (F > 0 at the drain for an on NMOS) and the gate draws none.
    assert out.f[0] > 1e-5 and out.f[1] == 0.0
    # Charge is conserved: Q summed over all terminals (including ground) is zero.
    assert abs(out.q.sum()) < 1e-18
    # Store keeps the limited branch voltages: vds = 1.0, vgs = 1.2.
    assert out.next_sto[3] == pytest.approx(1.0) and out.next_sto[2] == pytest.approx(1.2)


def test_finite_difference_jacobian_matches_dfdx():
    """TESTJAC-style check (N_DEV_NumericalJacobian.C:175) of the oracle's own dF/dx."""
    ref = _one_nmos()
    f0 = xr.make_flags(newton_iter=1, voltlim=0)
    sol = np.array([0.8, 1.0, 0.0])

    def F(s):
        return ref.load(f0, s, np.zeros(3), np.zeros(3), np.zeros(14), np.zeros(14))

    base = F(sol)
    h = 1e-7
    for j in range(2):
        s2 = sol.copy()
        s2[j] += h
        fd = (F(s2).f - base.f) / h
        # dfdx entry (row 0, col j) in the 2x2 (+ground) pattern: row 0 columns are [0, 1, 2]
        assert fd[0] == pytest.approx(base.dfdx[j], rel=1e-4, abs=1e-12)


def test_bsim3_default_topology_has_no_internal_nodes():
    ref = _one_nmos(level=9)
    assert ref.n_unknowns == 2
    # 12 state entries are reserved per instance (5 used without NQS) and 5 store entries.
    assert ref.n_state == 12 and ref.n_store == 5


@pytest.mark.parametrize("level", [9, 14])
def test_finite_difference_jacobians_both_families(level):
    """dF/dx and dQ/dx of the oracle against central differences of F and Q (transient flags)."""
    ref = _one_nmos(level=level)
    ns, no = ref.n_state, ref.n_store
    f0 = xr.make_flags(newton_iter=1, voltlim=0)
    sol = np.array([0.9, 1.1, 0.0])

    def load(s):
        return ref.load(f0, s, np.zeros(ns), np.zeros(ns), np.zeros(no), np.zeros(no))

    base = load(sol)
    h = 1e-6
    for j in range(2):
        sp, sm = sol.copy(), sol.copy()
        sp[j] += h
        sm[j] -= h
        lp, lm = load(sp), load(sm)
        fd_f = (lp.f - lm.f) / (2 * h)
        fd_q = (lp.q - lm.q) / (2 * h)
        for r in range(2):
            k = 3 * r + j  # row r of the 2 x (2 + ground) pattern
            assert fd_f[r] == pytest.approx(base.dfdx[k], rel=1e-5, abs=1e-12)
            assert fd_q[r] == pytest.approx(base.dqdx[k], rel=1e-5, abs=1e-22)


def test_gpu_binding_library_loads_and_builds_the_reference_topology():
    """The harness built with the product's BSIM4 binding as its device master loads without a GPU,
    and creating a family through it registers the reference's own topology (the GPU is touched
    only by the first load)."""
    if not xr.available(gpu=True):
        pytest.skip("binding harness not built (make -C oracle binding)")
    lib = xr.load_library(gpu=True)
    assert hasattr(lib, "xref_create_gpu_binding")
    ref = xr.RefCircuit(14, [(False, {}), (True, {"RSH": 10.0})], np.array([0, 1]),
                        np.array([[0, 1, -1, -1], [0, 1, 2, 2]]),
                        {"L": np.array([0.18e-6] * 2), "W": np.array([1e-6] * 2), "NRD": np.array([np.nan, 2.0])}, 3,
                        gpu_binding=True)
    assert ref.n_unknowns == 4  # the PMOS instance's internal drain node
    assert ref.n_state == 6 and ref.n_store == 28
