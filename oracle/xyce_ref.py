"""ctypes front end of the oracle library (oracle/_ref/libxyce_ref.so).

TEST INFRASTRUCTURE ONLY. The library is the reference's own MOSFET1 / BSIM3 / BSIM4 device
code (src/DeviceModelPKG/OpenModels/src/N_DEV_MOSFET{1,_B3,_B4}.C) compiled unmodified by
oracle/Makefile, driven by oracle/ref_harness.C through the same Device::updateState /
loadDAEVectors / loadDAEMatrices calls the reference's DeviceMgr makes
(src/DeviceModelPKG/Core/src/N_DEV_DeviceMgr.C:2117-2123, 2452-2461, 2256-2261).
Only tests/, the smoke check and bench.py's CPU baseline may import this module.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libxyce_ref.so")
LIB_OMP_PATH = os.path.join(_HERE, "_ref", "libxyce_ref_omp.so")
# Serial build without the libm interposer (oracle/libm_perturb.C): the CPU baseline's timing.
LIB_PLAIN_PATH = os.path.join(_HERE, "_ref", "libxyce_ref_plain.so")
# The harness with the product's reference-side binding (xyce_b200/binding) as the BSIM4 device
# master: the reference's Device calls run through libxyce_b200.so on the GPU.
LIB_GPU_PATH = os.path.join(_HERE, "_ref", "libxyce_ref_gpu.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class XrefFlags(ctypes.Structure):
    _fields_ = [
        ("dcop", ctypes.c_int), ("init_tran", ctypes.c_int), ("newton_iter", ctypes.c_int),
        ("init_jct", ctypes.c_int), ("init_fix", ctypes.c_int), ("transient", ctypes.c_int),
        ("tranop", ctypes.c_int), ("acop", ctypes.c_int), ("voltlim", ctypes.c_int),
        ("input_op", ctypes.c_int), ("gmin", ctypes.c_double), ("pdt", ctypes.c_double),
    ]


_LIBS: dict = {}


def _path(omp: bool, plain: bool, gpu: bool = False) -> str:
    if gpu:
        return LIB_GPU_PATH
    return LIB_OMP_PATH if omp else (LIB_PLAIN_PATH if plain else LIB_PATH)


def available(omp: bool = False, plain: bool = False, gpu: bool = False) -> bool:
    return os.path.exists(_path(omp, plain, gpu))


def load_library(omp: bool = False, plain: bool = False, gpu: bool = False):
    path = _path(omp, plain, gpu)
    if path in _LIBS:
        return _LIBS[path]
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library not built: {path} (run make -C oracle)")
    lib = ctypes.CDLL(path)
    create_args = [ctypes.c_int, ctypes.c_int, _ip, _ip, ctypes.POINTER(ctypes.c_char_p), _dp, ctypes.c_int, _ip, _ip,
                   ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), _dp, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    lib.xref_create.restype = ctypes.c_void_p
    lib.xref_create.argtypes = create_args
    if hasattr(lib, "xref_create_gpu_binding"):
        lib.xref_create_gpu_binding.restype = ctypes.c_void_p
        lib.xref_create_gpu_binding.argtypes = create_args
    lib.xref_destroy.argtypes = [ctypes.c_void_p]
    if hasattr(lib, "xref_create_linear"):
        lib.xref_create_linear.restype = ctypes.c_void_p
        lib.xref_create_linear.argtypes = [ctypes.c_char_p, ctypes.c_int, _ip, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_char_p), _dp, _ip, _dp, ctypes.c_int,
                                           ctypes.c_char_p, ctypes.c_int]
        lib.xref_set_time.argtypes = [ctypes.c_void_p, ctypes.c_double]
        lib.xref_set_time.restype = None
    if hasattr(lib, "xref_set_perturbation"):
        lib.xref_set_perturbation.argtypes = [ctypes.c_int, ctypes.c_ulonglong]
        lib.xref_set_perturbation.restype = None
    for name in ("xref_num_unknowns", "xref_num_state", "xref_num_store"):
        getattr(lib, name).argtypes = [ctypes.c_void_p]
        getattr(lib, name).restype = ctypes.c_int
    for name in ("xref_num_internal", "xref_state_base", "xref_store_base", "xref_stamp_count",
                 "xref_num_state_inst"):
        getattr(lib, name).argtypes = [ctypes.c_void_p, ctypes.c_int]
        getattr(lib, name).restype = ctypes.c_int
    lib.xref_stamp.argtypes = [ctypes.c_void_p, ctypes.c_int, _ip, _ip]
    lib.xref_stamp.restype = ctypes.c_int
    lib.xref_set_pattern.argtypes = [ctypes.c_void_p, ctypes.c_int, _ip, _ip]
    lib.xref_set_pattern.restype = ctypes.c_int
    lib.xref_load.argtypes = [ctypes.c_void_p, ctypes.POINTER(XrefFlags), _dp, _dp, _dp, _dp, _dp, _dp,
                              _dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_int]
    lib.xref_load.restype = ctypes.c_int
    lib.xref_time_loads.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.xref_time_loads.restype = ctypes.c_double
    lib.xref_last_error.argtypes = [ctypes.c_void_p]
    lib.xref_last_error.restype = ctypes.c_char_p
    _LIBS[path] = lib
    return lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


@dataclass
class RefLoad:
    f: np.ndarray
    q: np.ndarray
    dfdxdvp: np.ndarray
    dqdxdvp: np.ndarray
    dfdx: np.ndarray
    dqdx: np.ndarray
    next_sta: np.ndarray
    curr_sta: np.ndarray
    next_sto: np.ndarray


class RefCircuit:
    """The reference's device objects for one MOSFET family over one set of instances.

    models: list of (is_pmos, {NAME: value}) model cards.
    inst_model: int array [n]; inst_nodes: int array [n, 4] (D, G, S, B; -1 = ground);
    inst_params: {NAME: float array [n]} (NaN = not given).
    """

    def __init__(self, level, models, inst_model, inst_nodes, inst_params, n_nodes, omp=False, plain=False,
                 gpu_binding=False):
        self.lib = load_library(omp, plain, gpu_binding)
        self.level = level
        is_pmos = np.array([1 if m[0] else 0 for m in models], dtype=np.int32)
        nparams = np.array([len(m[1]) for m in models], dtype=np.int32)
        names, values = [], []
        for _, card in models:
            for k, v in card.items():
                names.append(k.encode())
                values.append(float(v))
        self._names = (ctypes.c_char_p * max(1, len(names)))(*names)
        vals = np.array(values if values else [0.0], dtype=np.float64)
        inst_model = np.ascontiguousarray(inst_model, dtype=np.int32)
        inst_nodes = np.ascontiguousarray(inst_nodes, dtype=np.int32).reshape(-1)
        n = inst_model.shape[0]
        pnames = list(inst_params.keys())
        self._pnames = (ctypes.c_char_p * max(1, len(pnames)))(*[p.encode() for p in pnames])
        pvals = np.full((n, max(1, len(pnames))), math.nan)
        for k, p in enumerate(pnames):
            pvals[:, k] = np.asarray(inst_params[p], dtype=np.float64)
        pvals = np.ascontiguousarray(pvals)
        err = ctypes.create_string_buffer(512)
        create = self.lib.xref_create_gpu_binding if gpu_binding else self.lib.xref_create
        h = create(level, len(models), _iptr(is_pmos), _iptr(nparams), self._names, _dptr(vals), n,
                                 _iptr(inst_model), _iptr(inst_nodes), len(pnames), self._pnames, _dptr(pvals),
                                 int(n_nodes), err, 512)
        if not h:
            raise RuntimeError(f"oracle create failed: {err.value.decode()}")
        self.h = ctypes.c_void_p(h)
        self.n = n
        self.n_nodes = int(n_nodes)
        self.n_unknowns = self.lib.xref_num_unknowns(self.h)
        self.n_state = self.lib.xref_num_state(self.h)
        self.n_store = self.lib.xref_num_store(self.h)
        self.nnz = None

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.lib.xref_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def num_internal(self, i):
        return self.lib.xref_num_internal(self.h, i)

    def state_base(self, i):
        return self.lib.xref_state_base(self.h, i)

    def store_base(self, i):
        return self.lib.xref_store_base(self.h, i)

    def stamp(self, i):
        k = self.lib.xref_stamp_count(self.h, i)
        r = np.zeros(max(1, k), dtype=np.int32)
        c = np.zeros(max(1, k), dtype=np.int32)
        self.lib.xref_stamp(self.h, i, _iptr(r), _iptr(c))
        return r[:k], c[:k]

    def set_pattern(self, rowptr, colind):
        self._rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self._colind = np.ascontiguousarray(colind, dtype=np.int32)
        rc = self.lib.xref_set_pattern(self.h, self._rowptr.shape[0] - 1, _iptr(self._rowptr), _iptr(self._colind))
        if rc != 0:
            raise RuntimeError(f"oracle pattern rejected (code {rc})")
        self.nnz = int(self._rowptr[-1])

    def load(self, flags: XrefFlags, next_sol, next_sta, curr_sta, next_sto, curr_sto, curr_sol=None,
             repetitions=1, perturb_seed=None) -> RefLoad:
        """One reference load. With ``perturb_seed``, every exp/log/log10/pow result inside the load
        is moved by one ulp (direction drawn from the seed); see libm_perturb.C."""
        nv = self.n_unknowns + 1
        next_sol = np.ascontiguousarray(next_sol, dtype=np.float64)
        assert next_sol.shape[0] == nv
        ns = max(1, self.n_state)
        no = max(1, self.n_store)
        nsta = np.zeros(ns); nsta[: len(next_sta)] = next_sta
        csta = np.zeros(ns); csta[: len(curr_sta)] = curr_sta
        nsto = np.zeros(no); nsto[: len(next_sto)] = next_sto
        csto = np.zeros(no); csto[: len(curr_sto)] = curr_sto
        csol = None if curr_sol is None else np.ascontiguousarray(curr_sol, dtype=np.float64)
        out = RefLoad(np.zeros(nv), np.zeros(nv), np.zeros(nv), np.zeros(nv), np.zeros(self.nnz),
                      np.zeros(self.nnz), nsta, csta, nsto)
        if perturb_seed is not None:
            if not hasattr(self.lib, "xref_set_perturbation"):
                raise RuntimeError("this oracle build has no libm perturbation (serial library only)")
            self.lib.xref_set_perturbation(1, ctypes.c_ulonglong(int(perturb_seed)))
        try:
            rc = self.lib.xref_load(self.h, ctypes.byref(flags), _dptr(next_sol),
                                    _dptr(csol) if csol is not None else None, _dptr(nsta), _dptr(csta),
                                    _dptr(nsto), _dptr(csto), _dptr(out.f), _dptr(out.q), _dptr(out.dfdxdvp),
                                    _dptr(out.dqdxdvp),
                                    _dptr(out.dfdx), _dptr(out.dqdx), int(repetitions))
        finally:
            if perturb_seed is not None:
                self.lib.xref_set_perturbation(0, ctypes.c_ulonglong(0))
        if rc != 0:
            raise RuntimeError(f"oracle load failed: {self.lib.xref_last_error(self.h).decode()}")
        out.next_sta = nsta[: self.n_state]
        out.curr_sta = csta[: self.n_state]
        out.next_sto = nsto[: self.n_store]
        return out

    def time_loads(self, repetitions: int) -> float:
        return float(self.lib.xref_time_loads(self.h, int(repetitions)))


class RefLinear(RefCircuit):
    """The reference's resistors ("r", instance parameter R), capacitors ("c", C) or independent
    voltage sources ("v", DCV0; pwl[i] = (times, values) for a piecewise-linear transient value) over
    2-node instances (inst_nodes [n, 2], -1 = ground). A source's branch current is its internal
    unknown, numbered after the n_nodes nodes in instance order."""

    def __init__(self, letter, inst_nodes, inst_params, n_nodes, pwl=None):
        self.lib = load_library()
        self.level = 1
        inst_nodes = np.ascontiguousarray(inst_nodes, dtype=np.int32).reshape(-1)
        n = inst_nodes.shape[0] // 2
        pnames = list(inst_params.keys())
        self._pnames = (ctypes.c_char_p * max(1, len(pnames)))(*[p.encode() for p in pnames])
        pvals = np.full((n, max(1, len(pnames))), math.nan)
        for k, p in enumerate(pnames):
            pvals[:, k] = np.asarray(inst_params[p], dtype=np.float64)
        pvals = np.ascontiguousarray(pvals)
        counts = np.zeros(max(1, n), dtype=np.int32)
        tv = [0.0]
        if pwl is not None:
            tv = []
            for i, p in enumerate(pwl):
                if p is not None:
                    counts[i] = len(p[0])
                    for t, v in zip(p[0], p[1]):
                        tv += [float(t), float(v)]
        tv = np.ascontiguousarray(tv if tv else [0.0], dtype=np.float64)
        err = ctypes.create_string_buffer(512)
        h = self.lib.xref_create_linear(letter.encode(), n, _iptr(inst_nodes), len(pnames), self._pnames, _dptr(pvals),
                                        _iptr(counts), _dptr(tv), int(n_nodes), err, 512)
        if not h:
            raise RuntimeError(f"oracle create failed: {err.value.decode()}")
        self.h = ctypes.c_void_p(h)
        self.n = n
        self.n_nodes = int(n_nodes)
        self.n_unknowns = self.lib.xref_num_unknowns(self.h)
        self.n_state = self.lib.xref_num_state(self.h)
        self.n_store = self.lib.xref_num_store(self.h)
        self.nnz = None

    def set_time(self, t: float):
        self.lib.xref_set_time(self.h, float(t))


def make_flags(**kw) -> XrefFlags:
    """Flags default to a transient Newton iterate past the first: charges computed, limiting on."""
    f = XrefFlags()
    f.dcop = kw.get("dcop", 0)
    f.init_tran = kw.get("init_tran", 0)
    f.newton_iter = kw.get("newton_iter", 1)
    f.init_jct = kw.get("init_jct", 0)
    f.init_fix = kw.get("init_fix", 0)
    f.transient = kw.get("transient", 1)
    f.tranop = kw.get("tranop", 0)
    f.acop = kw.get("acop", 0)
    f.voltlim = kw.get("voltlim", 1)
    f.input_op = kw.get("input_op", 0)
    f.gmin = kw.get("gmin", 1e-12)
    f.pdt = kw.get("pdt", 0.0)
    return f
