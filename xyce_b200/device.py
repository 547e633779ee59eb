"""Host-side mirror of the reference's MOSFET Device interface, backed by the B200 kernels.

``MosfetDevice`` plays the role of one of the reference's MOSFET ``Master`` objects inside the
device manager — ``Bsim4Device`` for ``MOSFET_B4::Master``
(src/DeviceModelPKG/OpenModels/src/N_DEV_MOSFET_B4.C:16180-17268), ``Bsim3Device`` for
``MOSFET_B3::Master`` (N_DEV_MOSFET_B3.C:9199-9900), ``Mos1Device`` for
``MOSFET1::Master`` (N_DEV_MOSFET1.C:4069-4697): one object per MOSFET family, created from
.MODEL cards and instance lines, with the three per-iteration calls of ``Device``
(src/DeviceModelPKG/Core/include/N_DEV_Device.h:315, 361, 384):

    update_state(sol, sta, sto)          <- Device::updateState
    load_dae_vectors(f, q, dfdxdvp, dqdxdvp) <- Device::loadDAEVectors
    load_dae_matrices(dfdx, dqdx)        <- Device::loadDAEMatrices

Buffers are float64 CUDA tensors (torch is used only to own device memory and streams); the
work runs in hand-written sm_100a kernels through the C ABI of ``include/xyce_devload.h``.
Errors raise ``NativeError`` (the reference reports fatal errors by throwing
``std::runtime_error``, src/ErrorHandlingPKG/src/N_ERH_Messenger.C:373).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _native

BSIM4_STATE_SLOTS = ("qb", "qg", "qd")
BSIM4_STORE_SLOTS = ("vbd", "vbs", "vgs", "vds", "vges", "vgms", "vdes", "vses", "vdbs", "vsbs", "vdbd",
                     "vged", "vgmd", "von")


@dataclass
class SolverFlags:
    """The SolverState / DeviceOptions fields a MOSFET load reads (N_DEV_SolverState.h:93-204)."""

    dcop: int = 0
    init_tran: int = 0
    newton_iter: int = 1
    init_jct: int = 0
    init_fix: int = 0
    transient: int = 1
    tranop: int = 0
    acop: int = 0
    voltlim: int = 1
    input_op: int = 0
    gmin: float = 1e-12
    pdt: float = 0.0

    def to_c(self) -> _native.XdFlags:
        f = _native.XdFlags()
        for k in ("dcop", "init_tran", "newton_iter", "init_jct", "init_fix", "transient", "tranop", "acop",
                  "voltlim", "input_op"):
            setattr(f, k, int(getattr(self, k)))
        f.gmin = float(self.gmin)
        f.pdt = float(self.pdt)
        return f


@dataclass
class ModelCard:
    """A .MODEL card: ``pmos`` selects the type; ``params`` maps netlist names to values."""

    pmos: bool = False
    params: dict = field(default_factory=dict)


def _ptr(t):
    if t is None:
        return None
    if not t.is_cuda or t.dtype.itemsize != 8:
        raise _native.NativeError("device buffers must be float64 CUDA tensors")
    if not t.is_contiguous():
        raise _native.NativeError("device buffers must be contiguous")
    return ctypes.c_void_p(t.data_ptr())


def _stream_handle(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def _family_struct(models, inst_model, inst_nodes, inst_params, level, temp_c, tnom_c, inst_internal=None):
    """The ``xd_mosfet_family`` struct of a family, with the arrays it points into (keep them alive)."""
    inst_model = np.ascontiguousarray(inst_model, dtype=np.int32)
    n = int(inst_model.shape[0])
    nodes = np.ascontiguousarray(np.asarray(inst_nodes, dtype=np.int32).reshape(-1))
    if nodes.shape[0] != 4 * n:
        raise _native.NativeError("inst_nodes must have shape [n, 4]")
    is_pmos = np.array([1 if m.pmos else 0 for m in models], dtype=np.int32)
    nparams = np.array([len(m.params) for m in models], dtype=np.int32)
    names, values = [], []
    for m in models:
        for k, v in m.params.items():
            names.append(str(k).encode())
            values.append(float(v))
    cnames = (ctypes.c_char_p * max(1, len(names)))(*names)
    vals = np.ascontiguousarray(values if values else [0.0], dtype=np.float64)
    pnames = list(inst_params.keys())
    cpnames = (ctypes.c_char_p * max(1, len(pnames)))(*[p.encode() for p in pnames])
    pv = np.full((n, max(1, len(pnames))), math.nan)
    for k, p in enumerate(pnames):
        pv[:, k] = np.asarray(inst_params[p], dtype=np.float64)
    pv = np.ascontiguousarray(pv)
    keep = [inst_model, nodes, is_pmos, nparams, vals, pv, cnames, cpnames]
    fam = _native.XdMosfetFamily()
    fam.level = int(level)
    fam.n_models = len(models)
    fam.model_is_pmos = is_pmos.ctypes.data_as(_native._ip)
    fam.model_nparams = nparams.ctypes.data_as(_native._ip)
    fam.model_param_names = cnames
    fam.model_param_values = vals.ctypes.data_as(_native._dp)
    fam.n_inst = n
    fam.inst_model = inst_model.ctypes.data_as(_native._ip)
    fam.inst_nodes = nodes.ctypes.data_as(_native._ip)
    fam.n_inst_params = len(pnames)
    fam.inst_param_names = cpnames
    fam.inst_param_values = pv.ctypes.data_as(_native._dp)
    fam.temp_c = float(temp_c)
    fam.tnom_c = float(tnom_c)
    if inst_internal is not None:
        # [n, 2]: drain / source internal nodes; [n, 11]: the BSIM4 general topology's internal
        # variables (GEN_INTERNAL order).
        arr = np.asarray(inst_internal, dtype=np.int32)
        internal = np.ascontiguousarray(arr.reshape(-1))
        keep.append(internal)
        if arr.ndim == 2 and arr.shape == (n, GEN_INTERNAL):
            fam.inst_internal_gen = internal.ctypes.data_as(_native._ip)
        elif internal.shape[0] == 2 * n:
            fam.inst_internal = internal.ctypes.data_as(_native._ip)
        else:
            raise _native.NativeError(f"inst_internal must have shape [n, 2] or [n, {GEN_INTERNAL}]")
    return fam, keep


# The BSIM4 general topology's internal variables per instance, in the reference's registerLIDs
# order (N_DEV_MOSFET_B4.C:5018-5099); the columns of an [n, 11] ``inst_internal``.
GEN_INTERNAL_NAMES = ("drain'", "source'", "gate'", "gate-mid", "body'", "source-body", "drain-body", "charge",
                      "IBS", "IDS", "IGS")
GEN_INTERNAL = len(GEN_INTERNAL_NAMES)


def internal_nodes(models, inst_model, inst_nodes, inst_params, level=14, temp_c=27.0, tnom_c=27.0, general=False):
    """Which instances have which internal variables: the topology query the reference's instances
    answer before their unknowns are numbered. ``general=False``: [n, 2] bool, the internal drain /
    source nodes (``xd_internal_nodes``). ``general=True`` (BSIM4): ([n, 11] bool in GEN_INTERNAL
    order, whether the family needs the general topology) from ``xd_internal_nodes_gen``."""
    fam, keep = _family_struct(models, inst_model, inst_nodes, inst_params, level, temp_c, tnom_c)
    n = int(np.asarray(inst_model).shape[0])
    lib = _native.load()
    if general:
        flags = np.zeros(GEN_INTERNAL * n, dtype=np.int32)
        rc = lib.xd_internal_nodes_gen(ctypes.byref(fam), flags.ctypes.data_as(_native._ip))
        _native.check(min(rc, 0), "xd_internal_nodes_gen")
        return flags.reshape(n, GEN_INTERNAL).astype(bool), rc == 1
    flags = np.zeros(2 * n, dtype=np.int32)
    _native.check(lib.xd_internal_nodes(ctypes.byref(fam), flags.ctypes.data_as(_native._ip)), "xd_internal_nodes")
    return flags.reshape(n, 2).astype(bool)


def general_stamp():
    """The general topology's 85 (row, col) local-node pairs (``xd_general_stamp``)."""
    lib = _native.load()
    rows, cols = np.zeros(128, dtype=np.int32), np.zeros(128, dtype=np.int32)
    k = lib.xd_general_stamp(rows.ctypes.data_as(_native._ip), cols.ctypes.data_as(_native._ip))
    _native.check(min(k, 0), "xd_general_stamp")
    return np.stack([rows[:k], cols[:k]], 1)


class MosfetDevice:
    """One MOSFET family (one reference Device object) on one CUDA device.

    models:        list of ``ModelCard``
    inst_model:    int array [n]      card index per instance
    inst_nodes:    int array [n, 4]   D, G, S, B unknown indices (-1 = ground)
    inst_params:   dict name -> float array [n] (NaN = not given), e.g. L, W, NF, AD, DELVTO, M
    pattern:       (rowptr, colind) CSR pattern of the Jacobian over the unknowns
    inst_internal: int array [n, 2] internal drain / source unknowns (-1 = none), required when
                   ``internal_nodes`` reports some; or, for the BSIM4 general topology (gate / body
                   resistance, rdsMod 1, NQS, instance ICs), [n, 11] in GEN_INTERNAL order
    """

    level = 14

    def __init__(self, models, inst_model, inst_nodes, inst_params, pattern, n_unknowns, device=0,
                 temp_c=27.0, tnom_c=27.0, level=None, inst_internal=None):
        if level is not None:
            self.level = int(level)
        lib = _native.load()
        self._lib = lib
        self.device = int(device)
        self.n = int(np.asarray(inst_model).shape[0])
        self.n_unknowns = int(n_unknowns)
        fam, keep = _family_struct(models, inst_model, inst_nodes, inst_params, self.level, temp_c, tnom_c,
                                   inst_internal)
        rowptr = np.ascontiguousarray(pattern[0], dtype=np.int32)
        colind = np.ascontiguousarray(pattern[1], dtype=np.int32)
        if rowptr.shape[0] != self.n_unknowns + 1:
            raise _native.NativeError("pattern rowptr must have n_unknowns + 1 entries")
        keep += [rowptr, colind]
        csr = _native.XdCsr(self.n_unknowns, rowptr.ctypes.data_as(_native._ip), colind.ctypes.data_as(_native._ip))
        h = ctypes.c_void_p()
        _native.check(lib.xd_create(ctypes.byref(fam), ctypes.byref(csr), self.device, ctypes.byref(h)), "xd_create")
        self._keep = keep
        self._h = h
        self.nnz = int(rowptr[-1])
        self.n_state_slots = lib.xd_num_state_slots(h)
        self.n_store_slots = lib.xd_num_store_slots(h)
        self.n_state = self.n_state_slots * self.n
        self.n_store = self.n_store_slots * self.n

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.xd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def update_state(self, flags: SolverFlags, sol, next_sta, curr_sta, next_sto, curr_sto, stream=None):
        c = flags.to_c()
        _native.check(self._lib.xd_update_state(self._h, ctypes.byref(c), _ptr(sol), _ptr(next_sta), _ptr(curr_sta),
                                                _ptr(next_sto), _ptr(curr_sto), _stream_handle(stream)),
                      "xd_update_state")

    def load_dae_vectors(self, f, q, dfdxdvp, dqdxdvp, stream=None):
        _native.check(self._lib.xd_load_vectors(self._h, _ptr(f), _ptr(q), _ptr(dfdxdvp), _ptr(dqdxdvp),
                                                _stream_handle(stream)), "xd_load_vectors")

    def load_dae_matrices(self, dfdx_vals, dqdx_vals, stream=None):
        _native.check(self._lib.xd_load_matrices(self._h, _ptr(dfdx_vals), _ptr(dqdx_vals), _stream_handle(stream)),
                      "xd_load_matrices")

    def load(self, flags, sol, next_sta, curr_sta, next_sto, curr_sto, f, q, dfdxdvp, dqdxdvp, dfdx, dqdx,
             stream=None):
        c = flags.to_c()
        _native.check(self._lib.xd_load(self._h, ctypes.byref(c), _ptr(sol), _ptr(next_sta), _ptr(curr_sta),
                                         _ptr(next_sto), _ptr(curr_sto), _ptr(f), _ptr(q), _ptr(dfdxdvp),
                                         _ptr(dqdxdvp), _ptr(dfdx), _ptr(dqdx), _stream_handle(stream)), "xd_load")

    def load_abs(self, f, q, dfdxdvp, dqdxdvp, dfdx, dqdx, stream=None):
        _native.check(self._lib.xd_load_abs(self._h, _ptr(f), _ptr(q), _ptr(dfdxdvp), _ptr(dqdxdvp), _ptr(dfdx),
                                            _ptr(dqdx), _stream_handle(stream)), "xd_load_abs")

    def copy_stamps(self, stream=None) -> np.ndarray:
        """The staged stamps, [slots, n] (48 slots for the 4-terminal layout, 68 with internal drain /
        source nodes, 230 for the general topology)."""
        slots = self._lib.xd_num_stage_slots(self._h)
        out = np.zeros(slots * self.n, dtype=np.float64)
        _native.check(self._lib.xd_copy_stamps(self._h, ctypes.c_void_p(out.ctypes.data), _stream_handle(stream)),
                      "xd_copy_stamps")
        return out.reshape(slots, self.n)


class Bsim4Device(MosfetDevice):
    """BSIM4 v4.6.1 (levels 14/54): the reference's MOSFET_B4::Master."""

    level = 14


class Bsim3Device(MosfetDevice):
    """BSIM3 v3.2.2 (levels 9/49): the reference's MOSFET_B3::Master."""

    level = 9


class Mos1Device(MosfetDevice):
    """Level-1 MOSFET (Shichman-Hodges, Meyer capacitances): the reference's MOSFET1::Master."""

    level = 1


BSIM3_STATE_SLOTS = ("qb", "qg", "qd", "qbs", "qbd")
BSIM3_STORE_SLOTS = ("vbd", "vbs", "vgs", "vds", "von")
MOS1_STATE_SLOTS = ("qgs", "qgd", "qgb", "capgs", "capgd", "capgb", "qbd", "qbs")
MOS1_STORE_SLOTS = ("vbd", "vbs", "vgs", "vds", "von")
