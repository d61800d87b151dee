"""ctypes binding of the CPU FP64 oracle (oracle/kyn_oracle.cpp).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by __graft_entry__.smoke() as
the checker, and by bench.py's CPU-baseline leg.  The product package never
imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libkyn_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_long)

FIELD = {"x0": 0, "x": 1, "q": 2, "q_prev": 3, "q_delta": 4, "v": 5, "vd": 6, "a": 7, "f": 8,
         "lambda": 9, "tangent": 10, "output": 11}
WIDTH = {"x0": 7, "x": 7, "q": 7, "q_prev": 7, "q_delta": 6, "v": 6, "vd": 6, "a": 6, "f": 6,
         "lambda": 6, "tangent": 36, "output": 3}


def build(force: bool = False) -> str:
    """Compile the oracle (and its FLOP-counting build) with its Makefile (g++,
    no GPU needed)."""
    flops = os.path.join(_HERE, "_build", "libkyn_oracle_flops.so")
    deps = [os.path.join(_HERE, f) for f in ("kyn_oracle.cpp", "kyn_oracle.h")]
    deps.append(os.path.join(_HERE, "..", "include", "kynema_b200.h"))
    stale = any(not os.path.exists(x) or any(os.path.getmtime(d) > os.path.getmtime(x) for d in deps)
                for x in (_LIB_PATH, flops))
    if force or stale:
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_model_create.restype = ctypes.c_void_p
        L.orc_model_create.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
        L.orc_model_destroy.argtypes = [ctypes.c_void_p]
        L.orc_model_info.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_set_solver_mode.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_set_loads.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_set_prescribed.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _ip]
        L.orc_predict_and_assemble.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_get_state.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_get_crs.argtypes = [ctypes.c_void_p, _ip, _ip, _dp]
        L.orc_get_system_vectors.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_get_convergence.argtypes = [ctypes.c_void_p, _dp, _ip]
        L.orc_get_element_terms.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_run_batch.restype = ctypes.c_long
        L.orc_run_batch.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.c_int,
                                    _dp, _ip]
        L.orc_run_batch_record.restype = ctypes.c_long
        L.orc_run_batch_record.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                           ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp,
                                           ctypes.c_int, _dp, _ip, _ip]
        L.orc_crs_build.restype = ctypes.c_long
        L.orc_crs_build.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _lp, _lp,
                                    ctypes.c_int, ctypes.c_int, _lp, _lp, ctypes.c_int, _lp,
                                    _lp, _lp, _lp, _lp, _lp, _lp, ctypes.c_int]
        _lib = L
    return _lib


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class OracleModel:
    """One model in the oracle; mirrors State/Solver reads of the reference."""

    def __init__(self, packed, solver_mode: int = 0):
        """solver_mode 0: dense partial-pivot LU of the bordered system;
        1: boundary-condition elimination + LU without pivoting."""
        self.packed = packed  # keeps numpy arrays alive
        err = ctypes.create_string_buffer(256)
        h = lib().orc_model_create(ctypes.byref(packed.desc), err, 256)
        if not h:
            raise ValueError("oracle rejected model: " + err.value.decode())
        self.h = ctypes.c_void_p(h)
        from openturbine_b200.model import KynModelInfo  # plain struct layout
        info = KynModelInfo()
        lib().orc_model_info(self.h, ctypes.byref(info))
        self.info = info
        if solver_mode:
            lib().orc_set_solver_mode(self.h, solver_mode)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_model_destroy(self.h)
            self.h = None

    def set_node_fx(self, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        lib().orc_set_loads(self.h, 0, _d(v))

    def set_state_f(self, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        lib().orc_set_loads(self.h, 1, _d(v))

    def set_prescribed(self, cid: int, u) -> None:
        v = np.ascontiguousarray(u, dtype=np.float64)
        lib().orc_set_prescribed(self.h, cid, _d(v))

    def step(self, params) -> tuple[int, int]:
        it = ctypes.c_int(0)
        c = params.to_c()
        st = lib().orc_step(self.h, ctypes.byref(c), ctypes.byref(it))
        return st, it.value

    def predict_and_assemble(self, params) -> None:
        c = params.to_c()
        lib().orc_predict_and_assemble(self.h, ctypes.byref(c))

    def state(self, field: str) -> np.ndarray:
        rows = self.info.num_constraints if field in ("lambda", "output") else self.info.num_nodes
        out = np.zeros((rows, WIDTH[field]))
        lib().orc_get_state(self.h, FIELD[field], _d(out))
        return out

    def crs(self):
        n, nnz = self.info.num_dofs, self.info.nnz
        rp = np.zeros(n + 1, dtype=np.int32)
        ci = np.zeros(nnz, dtype=np.int32)
        vals = np.zeros(nnz)
        lib().orc_get_crs(self.h, rp.ctypes.data_as(_ip), ci.ctypes.data_as(_ip), _d(vals))
        return rp, ci, vals

    def system_vectors(self):
        n = self.info.num_dofs
        b, x = np.zeros(n), np.zeros(n)
        lib().orc_get_system_vectors(self.h, _d(b), _d(x))
        return b, x

    def convergence(self) -> np.ndarray:
        out = np.zeros(256)
        n = ctypes.c_int(0)
        lib().orc_get_convergence(self.h, _d(out), ctypes.byref(n))
        return out[: n.value].copy()

    def element_terms(self, beam: int, n_nodes: int):
        r = np.zeros((n_nodes, 6))
        s = np.zeros((n_nodes, n_nodes, 6, 6))
        lib().orc_get_element_terms(self.h, beam, _d(r), _d(s))
        return r, s


def run_batch(models: list, params, steps: int, amp=None, freq=None, nthreads: int = 0):
    """Advance every model `steps` steps with OpenMP over models (CPU baseline)."""
    arr = (ctypes.c_void_p * len(models))(*[m.h.value for m in models])
    secs = ctypes.c_double(0.0)
    iters = ctypes.c_int(0)
    c = params.to_c()
    a = np.ascontiguousarray(amp, dtype=np.float64) if amp is not None else None
    f = np.ascontiguousarray(freq, dtype=np.float64) if freq is not None else None
    conv = lib().orc_run_batch(arr, len(models), ctypes.byref(c), steps,
                               _d(a) if a is not None else None,
                               _d(f) if f is not None else None, nthreads,
                               ctypes.byref(secs), ctypes.byref(iters))
    return int(conv), secs.value, iters.value


def run_batch_record(models: list, params, first_step: int, steps: int, amp, freq,
                     nthreads: int = 0):
    """Advance every model `steps` steps from time step `first_step` (tip load
    amp sin(2 pi freq t)) with OpenMP over models; returns (status, iters,
    seconds) with status/iters of shape (models, steps)."""
    n = len(models)
    arr = (ctypes.c_void_p * n)(*[m.h.value for m in models])
    secs = ctypes.c_double(0.0)
    st = np.zeros((n, steps), dtype=np.int32)
    it = np.zeros((n, steps), dtype=np.int32)
    c = params.to_c()
    a = np.ascontiguousarray(amp, dtype=np.float64)
    f = np.ascontiguousarray(freq, dtype=np.float64)
    lib().orc_run_batch_record(arr, n, ctypes.byref(c), first_step, steps, _d(a), _d(f), nthreads,
                               ctypes.byref(secs), st.ctypes.data_as(_ip), it.ctypes.data_as(_ip))
    return st, it, secs.value


def crs_build(num_system_dofs, num_dofs, active_dofs, fmap, elem_nodes, constraints=None,
              sort_rows=True):
    """ComputeRowPtrs / ComputeColInds on raw connectivity (unit-test form).

    elem_nodes: list of per-element node lists.  constraints: list of dicts with
    base_active, target_active, base_table[6], target_table[6], row_range (2,).
    """
    L = lib()
    ad = np.ascontiguousarray(active_dofs, dtype=np.int64)
    fm = np.ascontiguousarray(fmap, dtype=np.int64)
    ne = len(elem_nodes)
    mx = max([len(e) for e in elem_nodes] + [1])
    npe = np.array([len(e) for e in elem_nodes] or [0], dtype=np.int64)
    en = np.zeros((max(ne, 1), mx), dtype=np.int64)
    for i, e in enumerate(elem_nodes):
        en[i, : len(e)] = e
    cons = constraints or []
    nc = len(cons)
    ba = np.array([c["base_active"] for c in cons] or [0], dtype=np.int64)
    ta = np.array([c["target_active"] for c in cons] or [0], dtype=np.int64)
    bt = np.array([c["base_table"] for c in cons] or [[0] * 6], dtype=np.int64)
    tt = np.array([c["target_table"] for c in cons] or [[0] * 6], dtype=np.int64)
    rr = np.array([c["row_range"] for c in cons] or [[0, 0]], dtype=np.int64)
    lp = lambda a: a.ctypes.data_as(_lp)  # noqa: E731
    rp = np.zeros(num_dofs + 1, dtype=np.int64)
    nnz = L.orc_crs_build(num_system_dofs, num_dofs, len(ad), lp(ad), lp(fm), ne, mx, lp(npe),
                          lp(en), nc, lp(ba), lp(ta), lp(bt), lp(tt), lp(rr), lp(rp), None,
                          int(sort_rows))
    ci = np.zeros(max(nnz, 1), dtype=np.int64)
    L.orc_crs_build(num_system_dofs, num_dofs, len(ad), lp(ad), lp(fm), ne, mx, lp(npe),
                    lp(en), nc, lp(ba), lp(ta), lp(bt), lp(tt), lp(rr), lp(rp), lp(ci),
                    int(sort_rows))
    return rp, ci[:nnz]
