"""Workload generators and the Jacobian pattern (host logic, no GPU)."""
import numpy as np
import pytest

from xyce_b200 import netlist


def test_random_logic_shapes_and_determinism():
    a = netlist.random_logic(3000, seed=3)
    b = netlist.random_logic(3000, seed=3)
    assert np.array_equal(a.mos_nodes, b.mos_nodes) and np.array_equal(a.res_value, b.res_value)
    assert abs(a.n_mos - 3000) < 50
    assert a.mos_nodes.max() < a.n_nodes and a.mos_nodes.min() >= -1
    assert np.all((a.res_value >= 10) & (a.res_value <= 1000))
    assert np.all((a.cap_value >= 0.1e-15) & (a.cap_value <= 10e-15))
    # Gate types appear in equal measure (INV 2 MOSFETs, NAND2/NOR2 4 MOSFETs).
    assert a.meta["n_gates"] * 10 / 3 == pytest.approx(a.n_mos, rel=0.05)


def test_random_logic_is_acyclic():
    c = netlist.random_logic(2000, seed=9)
    # Every gate's input pins come from nets created earlier (primary inputs or earlier gates).
    assert c.meta["n_inputs"] == 64


def test_pattern_covers_every_stamp_and_is_sorted():
    c = netlist.random_logic(1500, seed=4)
    rowptr, colind = netlist.jacobian_pattern(c)
    assert rowptr.shape[0] == c.n_unknowns + 1
    for r in range(c.n_unknowns):
        row = colind[rowptr[r]:rowptr[r + 1]]
        assert np.all(np.diff(row) > 0)
    entries = set(zip(np.repeat(np.arange(c.n_unknowns), np.diff(rowptr)).tolist(), colind.tolist()))
    for nd in c.mos_nodes[:200]:
        for a in nd:
            for b in nd:
                if a >= 0 and b >= 0:
                    assert (a, b) in entries


def test_inverter_ring():
    c = netlist.inverter_ring(101)
    assert c.n_mos == 202 and c.n_nodes == 102
    assert np.all(c.mos_nodes[0::2, 2] == 0)  # PMOS sources on VDD
