"""Seeded synthetic circuits and the Jacobian pattern they induce.

The reference reads SPICE netlists; the workloads here are generated instead, from a seed:

* ``random_logic``  — a random gate-level digital netlist of BSIM4 MOSFETs in INV / NAND2 / NOR2
  gates (gate type uniform), fan-out uniform in 1..4, each fan-out branch an RC wire (segment R
  log-uniform in 10-1000 ohm, C log-uniform in 0.1-10 fF), driven by primary inputs with
  piecewise-linear sources (50 ps edges). Gates only read nets created before them, so the
  logic is acyclic.
* ``inverter_ring`` — an odd-stage CMOS inverter ring with a load capacitor per stage.

The unknowns follow the reference's modified nodal analysis: one unknown per circuit node
(ground is not an unknown) and one per voltage-source branch current. ``jacobian_pattern``
forms the union of all device stamps as a CSR pattern with sorted columns, which is what the
reference's topology builds before devices register their Jacobian offsets
(src/TopoManagerPKG/src/N_TOP_CktGraphBasic.C:1092-1142).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

NMOS, PMOS = 0, 1


@dataclass
class Circuit:
    n_nodes: int                          # circuit nodes (unknowns 0 .. n_nodes-1)
    mos_type: np.ndarray                  # [n_mos] NMOS / PMOS
    mos_nodes: np.ndarray                 # [n_mos, 4] D, G, S, B (-1 = ground)
    mos_w: np.ndarray                     # [n_mos] width (m)
    mos_l: np.ndarray                     # [n_mos] length (m)
    res_nodes: np.ndarray                 # [n_res, 2]
    res_value: np.ndarray                 # [n_res] ohm
    cap_nodes: np.ndarray                 # [n_cap, 2]
    cap_value: np.ndarray                 # [n_cap] farad
    vsrc_nodes: np.ndarray                # [n_vsrc, 2] (+, -)
    vsrc_dc: np.ndarray                   # [n_vsrc] DC value (V)
    vsrc_pwl: list = field(default_factory=list)  # per source: None or (times, values)
    vdd: float = 1.2
    meta: dict = field(default_factory=dict)
    # Internal variables of the MOSFETs: [n_mos, 2] drain / source nodes (series resistance), or
    # [n_mos, 11] for the BSIM4 general topology (D', S', G', GM, B', SB, DB, the NQS charge Q and
    # the IBS, IDS, IGS branch currents), unknown indices, -1 where the instance has none. They come after the nodes
    # and the source branches, instance by instance in that order (the reference's numbering).
    mos_internal: np.ndarray | None = None
    n_internal: int = 0

    @property
    def n_mos(self) -> int:
        return int(self.mos_type.shape[0])

    @property
    def n_vsrc(self) -> int:
        return int(self.vsrc_nodes.shape[0])

    @property
    def n_unknowns(self) -> int:
        return self.n_nodes + self.n_vsrc + self.n_internal

    def mos_intrinsic_nodes(self) -> np.ndarray:
        """[n_mos, 4] (D', G, S', B): the intrinsic device's nodes (D / S where no internal node)."""
        m = self.mos_nodes.copy()
        if self.mos_internal is not None:
            for k, col in ((0, 0), (1, 2)):
                has = self.mos_internal[:, k] >= 0
                m[has, col] = self.mos_internal[has, k]
        return m

    def branch_index(self, k: int) -> int:
        return self.n_nodes + k


def _pairs_2term(nodes: np.ndarray) -> np.ndarray:
    a, b = nodes[:, 0], nodes[:, 1]
    rows = np.concatenate([a, a, b, b])
    cols = np.concatenate([a, b, a, b])
    return np.stack([rows, cols], 1)


# The BSIM4 general topology's stamp over its 15 local nodes (D, G, S, B, D', S', G', GM, B', SB, DB,
# Q, IBS, IDS, IGS = 0..14), in the reference's jacStamp order (N_DEV_MOSFET_B4.C:4641-4795), the
# charge node's columns of rows D', S', G' last; the library reports the same table
# (xd_general_stamp).
_D, _G, _S, _B, _DP, _SP, _GP, _GM, _BP, _SB, _DB, _Q, _IBS, _IDS, _IGS = range(15)
GEN_NODES = 15
GEN_STAMP = np.array(
    [(_D, _D), (_D, _DP), (_D, _SP), (_D, _GP), (_D, _BP),
     (_G, _G), (_G, _DP), (_G, _SP), (_G, _GP), (_G, _GM), (_G, _BP),
     (_S, _S), (_S, _DP), (_S, _SP), (_S, _GP), (_S, _BP),
     (_B, _B), (_B, _BP), (_B, _SB), (_B, _DB),
     (_DP, _D), (_DP, _DP), (_DP, _SP), (_DP, _GP), (_DP, _GM), (_DP, _BP), (_DP, _DB),
     (_SP, _S), (_SP, _DP), (_SP, _SP), (_SP, _GP), (_SP, _GM), (_SP, _BP), (_SP, _SB),
     (_GP, _G), (_GP, _DP), (_GP, _SP), (_GP, _GP), (_GP, _GM), (_GP, _BP),
     (_GM, _G), (_GM, _DP), (_GM, _SP), (_GM, _GP), (_GM, _GM), (_GM, _BP),
     (_BP, _B), (_BP, _DP), (_BP, _SP), (_BP, _GP), (_BP, _GM), (_BP, _BP), (_BP, _SB), (_BP, _DB),
     (_SB, _B), (_SB, _SP), (_SB, _BP), (_SB, _SB),
     (_DB, _B), (_DB, _DP), (_DB, _BP), (_DB, _DB),
     (_Q, _DP), (_Q, _SP), (_Q, _GP), (_Q, _BP), (_Q, _Q),
     (_IBS, _S), (_IBS, _B), (_IBS, _IBS), (_S, _IBS), (_B, _IBS),
     (_IDS, _D), (_IDS, _S), (_IDS, _IDS), (_D, _IDS), (_S, _IDS),
     (_IGS, _G), (_IGS, _S), (_IGS, _IGS), (_G, _IGS), (_S, _IGS),
     (_DP, _Q), (_SP, _Q), (_GP, _Q)], dtype=np.int64)


def general_local_nodes(c: Circuit) -> np.ndarray:
    """[n_mos, 15] unknown of each local node of the general topology: a node the instance does
    not have is its terminal's unknown (D' -> D, S' -> S, G' and GM -> G, B' / SB / DB -> B), an
    absent charge node or branch current -1, ground -1."""
    nd = c.mos_nodes.astype(np.int64)
    internal = c.mos_internal.astype(np.int64)
    rep = nd[:, [0, 2, 1, 1, 3, 3, 3]]
    loc = np.full((nd.shape[0], GEN_NODES), -1, dtype=np.int64)
    loc[:, :4] = nd
    loc[:, 4:11] = np.where(internal[:, :7] >= 0, internal[:, :7], rep)
    loc[:, 11:] = internal[:, 7:]
    return loc


def jacobian_pattern(c: Circuit):
    """CSR (rowptr, colind) over the unknowns: union of MOSFET 4x4, R/C 2x2 and V-source stamps."""
    parts = []
    m = c.mos_intrinsic_nodes().astype(np.int64)
    r = np.repeat(m, 4, axis=1)
    cc = np.tile(m, (1, 4))
    parts.append(np.stack([r.reshape(-1), cc.reshape(-1)], 1))
    if c.mos_internal is not None and c.mos_internal.shape[1] == GEN_NODES - 4:
        # The general topology's stamp after collapsing (pairs with ground or an absent branch
        # current drop out below).
        loc = general_local_nodes(c)
        parts.append(np.stack([loc[:, GEN_STAMP[:, 0]].reshape(-1), loc[:, GEN_STAMP[:, 1]].reshape(-1)], 1))
    elif c.mos_internal is not None:
        # Series resistances: (D', D), (D, D'), (D, D) and the source's.
        for k, col in ((0, 0), (1, 2)):
            has = c.mos_internal[:, k] >= 0
            a, b = c.mos_internal[has, k].astype(np.int64), c.mos_nodes[has, col].astype(np.int64)
            parts.append(np.stack([np.concatenate([a, b, b]), np.concatenate([b, a, b])], 1))
    if c.res_nodes.shape[0]:
        parts.append(_pairs_2term(c.res_nodes.astype(np.int64)))
    if c.cap_nodes.shape[0]:
        parts.append(_pairs_2term(c.cap_nodes.astype(np.int64)))
    if c.n_vsrc:
        br = np.arange(c.n_nodes, c.n_nodes + c.n_vsrc, dtype=np.int64)
        p, n = c.vsrc_nodes[:, 0].astype(np.int64), c.vsrc_nodes[:, 1].astype(np.int64)
        parts.append(np.stack([np.concatenate([p, br, n, br]), np.concatenate([br, p, br, n])], 1))
    pr = np.concatenate(parts, 0)
    pr = pr[(pr[:, 0] >= 0) & (pr[:, 1] >= 0)]
    nu = c.n_unknowns
    key = np.unique(pr[:, 0] * nu + pr[:, 1])
    rows = key // nu
    cols = (key % nu).astype(np.int32)
    rowptr = np.zeros(nu + 1, dtype=np.int64)
    np.add.at(rowptr, rows + 1, 1)
    rowptr = np.cumsum(rowptr).astype(np.int32)
    return rowptr, cols


def with_internal_nodes(c: Circuit, flags) -> Circuit:
    """The circuit with an internal unknown for every True in flags ([n_mos, 2] drain / source, or
    [n_mos, 11] for the BSIM4 general topology, from ``device.internal_nodes``), numbered after all
    other unknowns, instance by instance in column order."""
    import dataclasses

    flags = np.asarray(flags, dtype=bool)
    flags = flags.reshape(c.n_mos, -1)
    internal = np.full(flags.shape, -1, dtype=np.int64)
    base = c.n_nodes + c.n_vsrc
    order = np.flatnonzero(flags.reshape(-1))
    internal.reshape(-1)[order] = base + np.arange(order.shape[0])
    return dataclasses.replace(c, mos_internal=internal, n_internal=int(order.shape[0]))


def _loguniform(rng, lo, hi, n):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n))


def random_logic(n_mos_target: int, seed: int = 0, n_inputs: int = 64, wire_segments: int = 2, vdd: float = 1.2,
                 wn: float = 1e-6, wp: float = 2e-6, length: float = 0.18e-6, edge: float = 50e-12,
                 locality: int = 0) -> Circuit:
    """Random INV/NAND2/NOR2 netlist with about ``n_mos_target`` MOSFETs (see module doc).

    ``locality`` = 0: a gate pin takes any open fan-out slot of an earlier net (the wiring is an
    expander graph: a direct factorization of its matrix fills in almost completely). K > 0: a pin
    takes one of the K most recently opened slots, as in a placed netlist where a gate drives
    nearby gates; the fan-out distribution is unchanged."""
    rng = np.random.default_rng(seed)
    # Gate types: 0 INV (2 MOSFETs, 1 input), 1 NAND2 (4, 2), 2 NOR2 (4, 2); mean 10/3 MOSFETs.
    n_gates = max(1, int(round(n_mos_target * 3 / 10)))
    gtype = rng.integers(0, 3, n_gates)
    n_pins = np.where(gtype == 0, 1, 2)
    node = 0
    VDD = node
    node += 1
    inputs = np.arange(node, node + n_inputs)
    node += n_inputs
    outs = np.arange(node, node + n_gates)
    node += n_gates
    mids = np.full(n_gates, -1)
    nm = gtype != 0
    mids[nm] = np.arange(node, node + int(nm.sum()))
    node += int(nm.sum())
    # Fan-out slots: each net (primary input or gate output) offers U{1..4} branch slots; a gate
    # pin takes a random open slot of an earlier net (or, if none is open, a random earlier net).
    net_src = np.concatenate([inputs, outs])
    fan = rng.integers(1, 5, net_src.shape[0])
    pin_net = np.empty(int(n_pins.sum()), dtype=np.int64)
    pool = []
    pool.extend(np.repeat(np.arange(n_inputs), fan[:n_inputs]).tolist())
    pin = 0
    for g in range(n_gates):
        for _ in range(int(n_pins[g])):
            if pool:
                j = int(rng.integers(max(0, len(pool) - locality) if locality > 0 else 0, len(pool)))
                pool[j], pool[-1] = pool[-1], pool[j]
                pin_net[pin] = pool.pop()
            else:
                pin_net[pin] = int(rng.integers(0, n_inputs + g))
            pin += 1
        pool.extend([n_inputs + g] * int(fan[n_inputs + g]))
    stub_nets = np.array(pool, dtype=np.int64)
    # Each pin (and each unused slot) is reached through an RC ladder of `wire_segments` segments.
    n_branch = pin_net.shape[0] + stub_nets.shape[0]
    branch_net = np.concatenate([pin_net, stub_nets])
    ladder = np.arange(node, node + n_branch * wire_segments).reshape(n_branch, wire_segments)
    node += n_branch * wire_segments
    drv = net_src[branch_net]
    seg_from = np.concatenate([drv[:, None], ladder[:, :-1]], 1)
    res_nodes = np.stack([seg_from.reshape(-1), ladder.reshape(-1)], 1)
    res_value = _loguniform(rng, 10.0, 1000.0, res_nodes.shape[0])
    cap_nodes = np.stack([ladder.reshape(-1), np.full(ladder.size, -1)], 1)
    cap_value = _loguniform(rng, 0.1e-15, 10e-15, cap_nodes.shape[0])
    pin_node = ladder[: pin_net.shape[0], -1]
    # Transistors.
    typ, nod = [], []
    first_pin = np.concatenate([[0], np.cumsum(n_pins)[:-1]])
    for g in range(n_gates):
        o = outs[g]
        a = pin_node[first_pin[g]]
        if gtype[g] == 0:
            typ += [PMOS, NMOS]
            nod += [[o, a, VDD, VDD], [o, a, -1, -1]]
            continue
        b = pin_node[first_pin[g] + 1]
        m = mids[g]
        if gtype[g] == 1:  # NAND2: PMOS in parallel, NMOS in series
            typ += [PMOS, PMOS, NMOS, NMOS]
            nod += [[o, a, VDD, VDD], [o, b, VDD, VDD], [o, a, m, -1], [m, b, -1, -1]]
        else:  # NOR2: PMOS in series, NMOS in parallel
            typ += [PMOS, PMOS, NMOS, NMOS]
            nod += [[m, a, VDD, VDD], [o, b, m, VDD], [o, a, -1, -1], [o, b, -1, -1]]
    mos_type = np.array(typ, dtype=np.int32)
    mos_nodes = np.array(nod, dtype=np.int32)
    mos_w = np.where(mos_type == PMOS, wp, wn)
    mos_l = np.full(mos_type.shape[0], length)
    # Sources: VDD, and one PWL source per primary input (random bit sequence, 50 ps edges).
    vsrc_nodes = np.stack([np.concatenate([[VDD], inputs]), np.full(n_inputs + 1, -1)], 1)
    vsrc_dc = np.concatenate([[vdd], np.zeros(n_inputs)])
    pwl = [None]
    period = 1e-9
    for k in range(n_inputs):
        bits = rng.integers(0, 2, 12)
        t, v = [0.0], [vdd * bits[0]]
        for j in range(1, bits.shape[0]):
            t0 = j * period * 0.5 + rng.uniform(0, 0.2e-9)
            t += [t0, t0 + edge]
            v += [v[-1], vdd * bits[j]]
        pwl.append((np.array(t), np.array(v)))
    return Circuit(n_nodes=node, mos_type=mos_type, mos_nodes=mos_nodes, mos_w=mos_w, mos_l=mos_l,
                   res_nodes=res_nodes.astype(np.int32), res_value=res_value, cap_nodes=cap_nodes.astype(np.int32),
                   cap_value=cap_value, vsrc_nodes=vsrc_nodes.astype(np.int32), vsrc_dc=vsrc_dc, vsrc_pwl=pwl,
                   vdd=vdd, meta=dict(kind="random_logic", seed=seed, n_gates=n_gates, n_inputs=n_inputs,
                                      logic=dict(gtype=gtype, outs=outs, mids=mids, inputs=inputs, net_src=net_src,
                                                 pin_net=pin_net, first_pin=first_pin, n_pins=n_pins,
                                                 branch_net=branch_net, ladder=ladder, vdd_node=VDD)))


def logic_initial_guess(c: Circuit, t: float = 0.0) -> np.ndarray:
    """Node voltages of a random_logic netlist at the logic levels its inputs set at time t: the
    primary inputs' source values propagated through the gates in order (every gate reads earlier
    nets only), each wire ladder at its driving net's voltage, series-stack middle nodes at the
    rail their conducting transistor ties them to. A starting iterate for the operating point's
    Newton solve, as a .NODESET gives one; the solve itself settles the analogue values."""
    lg = c.meta["logic"]
    x = np.zeros(c.n_unknowns)
    vdd = c.vdd
    x[lg["vdd_node"]] = vdd
    n_in = lg["inputs"].shape[0]
    net_v = np.zeros(lg["net_src"].shape[0])
    for k in range(n_in):
        times, vals = c.vsrc_pwl[1 + k]
        net_v[k] = _pwl_at(times, vals, t)
    hi = lambda v: v > 0.5 * vdd
    gtype, first, pin_net = lg["gtype"], lg["first_pin"], lg["pin_net"]
    mids = lg["mids"]
    for g in range(gtype.shape[0]):
        a = hi(net_v[pin_net[first[g]]])
        if gtype[g] == 0:
            out = not a
        else:
            b = hi(net_v[pin_net[first[g] + 1]])
            if gtype[g] == 1:  # NAND2: middle node between the series NMOS
                out = not (a and b)
                x[mids[g]] = 0.0 if b else (vdd if a else 0.0)
            else:  # NOR2: middle node between the series PMOS
                out = not (a or b)
                x[mids[g]] = vdd if not a else (vdd if out else 0.0)
        net_v[n_in + g] = vdd if out else 0.0
        x[lg["outs"][g]] = net_v[n_in + g]
    x[lg["inputs"]] = net_v[:n_in]
    x[lg["ladder"]] = net_v[lg["branch_net"]][:, None]
    return x


def _pwl_at(times, values, t):
    if t <= times[0]:
        return float(values[0]) if times[0] == 0.0 else 0.0
    if t >= times[-1]:
        return float(values[-1])
    k = int(np.searchsorted(times, t, side="right"))
    t0, t1, v0, v1 = times[k - 1], times[k], values[k - 1], values[k]
    return float(v0 + (v1 - v0) * (t - t0) / (t1 - t0))


# Model cards for the BSIM3 ring-oscillator workload (W/L = 1u/0.18u, PMOS W = 2u, VDD = 1.8 V).
# An empty BSIM3 card makes the threshold ~2 V at L = 0.18u (VTH0 is then derived from VFB = -1
# and a body factor K1 ~ 1.9 computed from the default doping and 15 nm oxide), above the supply,
# so the ring would never switch. These project-chosen round values keep every other parameter at
# its card default and give thresholds near 0.6 V and on-currents of a few hundred uA.
RING_BSIM3_NMOS = {"TOX": 4e-9, "VTH0": 0.45, "K1": 0.55, "K2": 0.0, "U0": 400.0, "VSAT": 1e5}
RING_BSIM3_PMOS = {"TOX": 4e-9, "VTH0": -0.45, "K1": 0.55, "K2": 0.0, "U0": 120.0, "VSAT": 8e4}


def mosfet_family(c: Circuit, cards=None, extra_params=None):
    """(cards, inst_model, inst_nodes, inst_params) of the circuit's MOSFETs for ``MosfetDevice``:
    one NMOS and one PMOS card (default parameters unless ``cards`` is given), each instance's
    card by its type, its D, G, S, B unknowns, and L / W plus ``extra_params`` per instance."""
    from .device import ModelCard

    if cards is None:
        cards = [ModelCard(False, {}), ModelCard(True, {})]
    inst_model = c.mos_type.astype(np.int32)
    params = {"L": c.mos_l.astype(float), "W": c.mos_w.astype(float)}
    if extra_params:
        params.update(extra_params)
    return cards, inst_model, c.mos_nodes.astype(np.int32), params


def ring_bsim3_cards():
    from .device import ModelCard
    return [ModelCard(False, dict(RING_BSIM3_NMOS)), ModelCard(True, dict(RING_BSIM3_PMOS))]


def inverter_ring(stages: int = 101, vdd: float = 1.8, wn: float = 1e-6, wp: float = 2e-6, length: float = 0.18e-6,
                  cload: float = 5e-15) -> Circuit:
    """Odd-stage CMOS inverter ring with a load capacitor on every stage output."""
    VDD = 0
    out = np.arange(1, stages + 1)
    inp = np.roll(out, 1)
    typ = np.tile([PMOS, NMOS], stages)
    nod = np.empty((2 * stages, 4), dtype=np.int32)
    nod[0::2] = np.stack([out, inp, np.full(stages, VDD), np.full(stages, VDD)], 1)
    nod[1::2] = np.stack([out, inp, np.full(stages, -1), np.full(stages, -1)], 1)
    w = np.where(typ == PMOS, wp, wn)
    return Circuit(n_nodes=stages + 1, mos_type=typ.astype(np.int32), mos_nodes=nod, mos_w=w,
                   mos_l=np.full(2 * stages, length), res_nodes=np.zeros((0, 2), np.int32), res_value=np.zeros(0),
                   cap_nodes=np.stack([out, np.full(stages, -1)], 1).astype(np.int32),
                   cap_value=np.full(stages, cload), vsrc_nodes=np.array([[VDD, -1]], np.int32),
                   vsrc_dc=np.array([vdd]), vsrc_pwl=[None], vdd=vdd, meta=dict(kind="inverter_ring", stages=stages))


@dataclass
class Batch:
    """Several circuits merged into one block-diagonal system (one family, one launch)."""

    circuit: Circuit              # merged circuit (unknowns of circuit k are contiguous)
    cards: list                   # model cards: 2 per circuit (NMOS, PMOS)
    inst_model: np.ndarray        # card index per MOSFET
    inst_params: dict             # instance-line parameters (L, W, DELVTO)
    node_offset: np.ndarray       # [n_circuits + 1] first node of each circuit
    mos_offset: np.ndarray        # [n_circuits + 1] first MOSFET of each circuit
    sizes: np.ndarray             # MOSFETs per circuit
    delvto: np.ndarray            # per-circuit threshold shift (V)
    toxe_factor: np.ndarray       # per-circuit oxide-thickness factor


def batched_sweep(n_circuits: int = 256, min_mos: int = 1000, max_mos: int = 20000, seed: int = 0,
                  sigma_vth: float = 0.030, toxe_spread: float = 0.02, toxe_nominal: float = 3.0e-9,
                  wire_segments: int = 2) -> Batch:
    """A Monte-Carlo sweep: n_circuits random gate netlists (``random_logic``, sizes log-uniform in
    [min_mos, max_mos]), each with its own threshold shift ~ N(0, sigma_vth) (instance DELVTO on
    all its MOSFETs) and oxide thickness TOXE x U[1 - spread, 1 + spread] (its own NMOS/PMOS model
    cards), merged into one block-diagonal circuit whose unknowns keep each circuit contiguous.
    Node unknowns of every circuit come first, then every circuit's source branches."""
    from .device import ModelCard

    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(min_mos), np.log(max_mos), n_circuits)).astype(int)
    delvto = rng.normal(0.0, sigma_vth, n_circuits)
    toxe = rng.uniform(1 - toxe_spread, 1 + toxe_spread, n_circuits)
    parts = [random_logic(int(m), seed=seed * 100003 + k + 1, wire_segments=wire_segments) for k, m in enumerate(sizes)]
    node_off = np.zeros(n_circuits + 1, dtype=np.int64)
    mos_off = np.zeros(n_circuits + 1, dtype=np.int64)
    for k, p in enumerate(parts):
        node_off[k + 1] = node_off[k] + p.n_nodes
        mos_off[k + 1] = mos_off[k] + p.n_mos

    def shift(a, off):
        a = np.asarray(a, dtype=np.int64)
        return np.where(a >= 0, a + off, -1)

    mos_nodes = np.concatenate([shift(p.mos_nodes, node_off[k]) for k, p in enumerate(parts)]).astype(np.int32)
    res_nodes = np.concatenate([shift(p.res_nodes, node_off[k]) for k, p in enumerate(parts)]).astype(np.int32)
    cap_nodes = np.concatenate([shift(p.cap_nodes, node_off[k]) for k, p in enumerate(parts)]).astype(np.int32)
    vsrc_nodes = np.concatenate([shift(p.vsrc_nodes, node_off[k]) for k, p in enumerate(parts)]).astype(np.int32)
    merged = Circuit(n_nodes=int(node_off[-1]), mos_type=np.concatenate([p.mos_type for p in parts]),
                     mos_nodes=mos_nodes, mos_w=np.concatenate([p.mos_w for p in parts]),
                     mos_l=np.concatenate([p.mos_l for p in parts]), res_nodes=res_nodes,
                     res_value=np.concatenate([p.res_value for p in parts]), cap_nodes=cap_nodes,
                     cap_value=np.concatenate([p.cap_value for p in parts]), vsrc_nodes=vsrc_nodes,
                     vsrc_dc=np.concatenate([p.vsrc_dc for p in parts]),
                     vsrc_pwl=[w for p in parts for w in p.vsrc_pwl], vdd=parts[0].vdd,
                     meta=dict(kind="batched_sweep", n_circuits=n_circuits, seed=seed))
    cards = []
    for k in range(n_circuits):
        cards.append(ModelCard(False, {"TOXE": toxe_nominal * toxe[k]}))
        cards.append(ModelCard(True, {"TOXE": toxe_nominal * toxe[k]}))
    circ = np.repeat(np.arange(n_circuits), np.diff(mos_off))
    inst_model = (2 * circ + merged.mos_type).astype(np.int32)
    params = {"L": merged.mos_l.astype(float), "W": merged.mos_w.astype(float), "DELVTO": delvto[circ]}
    return Batch(merged, cards, inst_model, params, node_off, mos_off, sizes, delvto, toxe)
