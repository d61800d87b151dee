"""ctypes binding of libkynema_b200.so (the C ABI in include/kynema_b200.h).

Product path: every call goes to the sm_100a library.  There is no CPU
fallback -- ``Context()`` raises if the library is missing or no CUDA device
is visible.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .model import KynModelInfo, KynStepParams, Model, PackedModel, StepParameters

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libkynema_b200.so")

OK, NOT_CONVERGED = 0, 1
ERR = {-1: "INVALID", -2: "UNSUPPORTED", -3: "CUDA", -4: "BUDGET", -5: "NONFINITE",
       -6: "SINGULAR", -7: "NOT_FOUND", -8: "NO_DEVICE"}
FIELD = {"x0": 0, "x": 1, "q": 2, "q_prev": 3, "q_delta": 4, "v": 5, "vd": 6, "a": 7, "f": 8,
         "lambda": 9, "tangent": 10, "output": 11}
WIDTH = {"x0": 7, "x": 7, "q": 7, "q_prev": 7, "q_delta": 6, "v": 6, "vd": 6, "a": 6, "f": 6,
         "lambda": 6, "tangent": 36, "output": 3}
LOAD_NODE_FX, LOAD_STATE_F = 0, 1
OPT_RECORD_SYSTEM, OPT_PHASE_TIMING, OPT_CUDA_GRAPH, OPT_LINEAR_SOLVER = 1, 2, 3, 4
OPT_RESET_SOLVE_STATS, OPT_BULK_SECTIONS = 5, 6
SOLVER_GAUSS_JORDAN, SOLVER_PANEL_LU = 0, 1

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lib = None


class KynError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERR.get(code, code)}: {msg}")
        self.code = code


def load_library():
    """Load the CUDA library; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m openturbine_b200.build` "
            "(nvcc, sm_100a); there is no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    L.kyn_model_describe.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int), ctypes.c_char_p, ctypes.c_int]
    L.kyn_ctx_create.restype = ctypes.c_void_p
    L.kyn_ctx_create.argtypes = [ctypes.c_int, ctypes.c_size_t]
    L.kyn_ctx_destroy.argtypes = [ctypes.c_void_p]
    L.kyn_last_error.restype = ctypes.c_char_p
    L.kyn_last_error.argtypes = [ctypes.c_void_p]
    L.kyn_ctx_used_bytes.restype = ctypes.c_size_t
    L.kyn_ctx_used_bytes.argtypes = [ctypes.c_void_p]
    L.kyn_ctx_set_option.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64]
    L.kyn_model_create.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.kyn_model_destroy.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.kyn_model_clone.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.kyn_model_info_get.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    L.kyn_model_set_loads.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]
    L.kyn_model_set_prescribed.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]
    L.kyn_step.argtypes = [ctypes.c_void_p, _ip, ctypes.c_int, ctypes.c_void_p, _ip, _ip]
    L.kyn_step_async.argtypes = [ctypes.c_void_p, _ip, ctypes.c_int, ctypes.c_void_p]
    L.kyn_step_wait.argtypes = [ctypes.c_void_p, _ip, _ip]
    L.kyn_get_state.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]
    L.kyn_get_convergence.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _ip]
    L.kyn_get_crs.argtypes = [ctypes.c_void_p, ctypes.c_int, _ip, _ip, _dp]
    L.kyn_get_system_vectors.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
    L.kyn_set_loads_batch.argtypes = [ctypes.c_void_p, _ip, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_void_p, ctypes.c_int]
    L.kyn_get_state_batch.argtypes = [ctypes.c_void_p, _ip, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_void_p, ctypes.c_int]
    L.kyn_set_prescribed_batch.argtypes = [ctypes.c_void_p, _ip, ctypes.c_int, ctypes.c_void_p,
                                           ctypes.c_int]
    L.kyn_set_state.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]
    L.kyn_state_write.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
                                  ctypes.POINTER(ctypes.c_size_t)]
    L.kyn_state_read.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
    L.kyn_state_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.kyn_autotune.argtypes = [ctypes.c_void_p, _ip, ctypes.c_int, ctypes.c_void_p]
    L.kyn_tuned_threads.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.kyn_tuned_solver.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.kyn_set_loads_batch_static.argtypes = [ctypes.c_void_p, _ip, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_void_p, ctypes.c_int]
    L.kyn_ctx_stat.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
    L.kyn_ctx_stream.restype = ctypes.c_void_p
    L.kyn_ctx_stream.argtypes = [ctypes.c_void_p]
    _lib = L
    return L


def describe(model: Model | PackedModel):
    """Host-only check of a model description (kyn_model_describe): the sizes
    and the CRS graph (row_ptrs, col_inds) that kyn_model_create would build,
    without a GPU.  Raises RuntimeError with the library's reason when the
    description is invalid or outside this path."""
    L = load_library()
    pm = model.pack() if isinstance(model, Model) else model
    info = KynModelInfo()
    err = ctypes.create_string_buffer(256)
    rc = L.kyn_model_describe(ctypes.byref(pm.desc), ctypes.byref(info), None, None, err, 256)
    if rc < 0:
        raise RuntimeError(f"kyn_model_describe: {ERR.get(rc, rc)}: {err.value.decode()}")
    rp = np.zeros(info.num_dofs + 1, dtype=np.int32)
    ci = np.zeros(info.nnz, dtype=np.int32)
    rc = L.kyn_model_describe(ctypes.byref(pm.desc), ctypes.byref(info), rp.ctypes.data_as(_ip),
                              ci.ctypes.data_as(_ip), err, 256)
    if rc < 0:
        raise RuntimeError(f"kyn_model_describe: {ERR.get(rc, rc)}: {err.value.decode()}")
    return info, rp, ci


class Context:
    """A device context (kyn_ctx): owns resident models on one GPU."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self.lib = load_library()
        h = self.lib.kyn_ctx_create(device, hbm_budget_bytes)
        if not h:
            raise KynError(-8, f"kyn_ctx_create({device}) failed: no CUDA device")
        self.h = ctypes.c_void_p(h)
        self._packed: dict[int, PackedModel] = {}
        self._info: dict[int, KynModelInfo] = {}

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.kyn_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> int:
        if rc < 0:
            raise KynError(rc, self.lib.kyn_last_error(self.h).decode())
        return rc

    def set_cuda_graph(self, on: bool = True) -> None:
        """Replay each model set's step launches from a captured CUDA graph."""
        self._check(self.lib.kyn_ctx_set_option(self.h, OPT_CUDA_GRAPH, int(on)))

    def set_linear_solver(self, solver: int) -> None:
        """SOLVER_GAUSS_JORDAN (registers, default) or SOLVER_PANEL_LU for the
        free-block solve of the step kernel."""
        self._check(self.lib.kyn_ctx_set_option(self.h, OPT_LINEAR_SOLVER, int(solver)))

    def set_record_system(self, on: bool = True) -> None:
        self._check(self.lib.kyn_ctx_set_option(self.h, OPT_RECORD_SYSTEM, int(on)))

    @property
    def used_bytes(self) -> int:
        return int(self.lib.kyn_ctx_used_bytes(self.h))

    # models
    def create_model(self, model: Model | PackedModel) -> int:
        pm = model.pack() if isinstance(model, Model) else model
        mid = self._check(self.lib.kyn_model_create(self.h, ctypes.byref(pm.desc)))
        self._packed[mid] = pm
        info = KynModelInfo()
        self._check(self.lib.kyn_model_info_get(self.h, mid, ctypes.byref(info)))
        self._info[mid] = info
        return mid

    def clone_model(self, mid: int) -> int:
        """A copy of model `mid` in its current state (kyn_model_clone)."""
        nid = self._check(self.lib.kyn_model_clone(self.h, mid))
        self._packed[nid] = self._packed.get(mid)
        self._info[nid] = self._info[mid]
        return nid

    def destroy_model(self, mid: int) -> None:
        self._check(self.lib.kyn_model_destroy(self.h, mid))
        self._packed.pop(mid, None)
        self._info.pop(mid, None)

    def info(self, mid: int) -> KynModelInfo:
        return self._info[mid]

    def set_node_fx(self, mid: int, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._check(self.lib.kyn_model_set_loads(self.h, mid, LOAD_NODE_FX, v.ctypes.data_as(_dp)))

    def set_state_f(self, mid: int, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._check(self.lib.kyn_model_set_loads(self.h, mid, LOAD_STATE_F, v.ctypes.data_as(_dp)))

    def set_prescribed(self, mid: int, cid: int, u) -> None:
        v = np.ascontiguousarray(u, dtype=np.float64)
        self._check(self.lib.kyn_model_set_prescribed(self.h, mid, cid, v.ctypes.data_as(_dp)))

    def set_control(self, mid: int, cid: int, value: float) -> None:
        """The commanded angle of a RotationControl constraint, or the torque
        of a RevoluteJoint (the value the reference reads through its control
        pointer before each step)."""
        self.set_prescribed(mid, cid, [float(value), 0.0, 0.0, 1.0, 0.0, 0.0, 0.0])

    # stepping
    def step(self, ids, params: StepParameters):
        ids_a = np.ascontiguousarray(ids, dtype=np.int32)
        n = ids_a.shape[0]
        st = np.zeros(n, dtype=np.int32)
        it = np.zeros(n, dtype=np.int32)
        c = params.to_c()
        self._check(self.lib.kyn_step(self.h, ids_a.ctypes.data_as(_ip), n, ctypes.byref(c),
                                      st.ctypes.data_as(_ip), it.ctypes.data_as(_ip)))
        return st, it

    def step_async(self, ids, params: StepParameters) -> None:
        self._ids_async = np.ascontiguousarray(ids, dtype=np.int32)
        c = params.to_c()
        self._check(self.lib.kyn_step_async(self.h, self._ids_async.ctypes.data_as(_ip),
                                            self._ids_async.shape[0], ctypes.byref(c)))

    def step_wait(self):
        n = self._ids_async.shape[0]
        st = np.zeros(n, dtype=np.int32)
        it = np.zeros(n, dtype=np.int32)
        self._check(self.lib.kyn_step_wait(self.h, st.ctypes.data_as(_ip), it.ctypes.data_as(_ip)))
        return st, it

    @property
    def stream_handle(self) -> int:
        """cudaStream_t of the context (for events / torch.cuda.ExternalStream)."""
        return int(self.lib.kyn_ctx_stream(self.h) or 0)

    def stat(self, which: int) -> int:
        v = ctypes.c_int64(0)
        self._check(self.lib.kyn_ctx_stat(self.h, which, ctypes.byref(v)))
        return int(v.value)

    @property
    def kernel_launches(self) -> int:
        return self.stat(1)

    @property
    def allocations(self) -> int:
        """Device and pinned-host allocations made by this context so far."""
        return self.stat(3)

    def set_bulk_sections(self, on: bool) -> None:
        """Stage each iteration's sections with one bulk copy (default) or let
        every quadrature point load its own."""
        self._check(self.lib.kyn_ctx_set_option(self.h, OPT_BULK_SECTIONS, int(on)))

    def reset_solve_stats(self) -> None:
        self._check(self.lib.kyn_ctx_set_option(self.h, OPT_RESET_SOLVE_STATS, 1))

    def solve_stats(self) -> dict:
        """Gauss-Jordan solve counters since the context was created (backward
        errors of FP64 solves, FP32 refinement sweeps)."""
        import struct
        mx = struct.unpack("<d", struct.pack("<q", self.stat(6)))[0]
        return {"checked": self.stat(4), "guard_trips": self.stat(5), "max_backward_error": mx,
                "refine_sweeps": self.stat(7), "refine_short": self.stat(8)}

    def batch_ids(self, ids) -> np.ndarray:
        return np.ascontiguousarray(ids, dtype=np.int32)

    def set_loads_batch(self, ids: np.ndarray, which: int, ptr: int, on_device: bool) -> None:
        """Loads for many models from one array at address `ptr` (host or device)."""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        self._check(self.lib.kyn_set_loads_batch(self.h, ids.ctypes.data_as(_ip), ids.shape[0],
                                                 which, ctypes.c_void_p(ptr), int(on_device)))

    def set_prescribed_batch(self, ids: np.ndarray, ptr: int, on_device: bool) -> None:
        """Prescribed motion [constraints of the listed models][7] from one array."""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        self._check(self.lib.kyn_set_prescribed_batch(self.h, ids.ctypes.data_as(_ip), ids.shape[0],
                                                      ctypes.c_void_p(ptr), int(on_device)))

    def set_state(self, mid: int, field: str, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._check(self.lib.kyn_set_state(self.h, mid, FIELD[field], v.ctypes.data_as(_dp)))

    def write_restart(self, mid: int) -> bytes:
        """The model's restart record (WriteStateToFile format)."""
        n = ctypes.c_size_t(0)
        self._check(self.lib.kyn_state_write(self.h, mid, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        self._check(self.lib.kyn_state_write(self.h, mid, buf, n.value, ctypes.byref(n)))
        return buf.raw

    def read_restart(self, mid: int, record: bytes) -> None:
        self._check(self.lib.kyn_state_read(self.h, mid, record, len(record)))

    def copy_state(self, dst: int, src: int) -> None:
        self._check(self.lib.kyn_state_copy(self.h, dst, src))

    def autotune(self, ids, params) -> None:
        """Pick threads per CTA for each size class of these models by timing
        copies of them (the models themselves are not advanced)."""
        arr = np.ascontiguousarray(ids, dtype=np.int32)
        c = params.to_c()
        self._check(self.lib.kyn_autotune(self.h, arr.ctypes.data_as(_ip), arr.shape[0],
                                          ctypes.byref(c)))

    def tuned_threads(self, mid: int, precision: int = 0) -> int:
        return self._check(self.lib.kyn_tuned_threads(self.h, mid, precision))

    def tuned_solver(self, mid: int, precision: int = 0) -> int:
        """KYN_SOLVER_* the step uses for the model (tuned, else the context's)."""
        return self._check(self.lib.kyn_tuned_solver(self.h, mid, precision))

    def set_loads_batch_static(self, ids: np.ndarray, which: int, ptr: int,
                               on_device: bool) -> None:
        """set_loads_batch that allocates nothing: staging in the library's fixed
        device array (limits and sharing rules in include/kynema_b200.h)."""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        self._check(self.lib.kyn_set_loads_batch_static(
            self.h, ids.ctypes.data_as(_ip), ids.shape[0], which, ctypes.c_void_p(ptr),
            int(on_device)))

    def get_state_batch(self, ids: np.ndarray, field: str, ptr: int, on_device: bool) -> None:
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        self._check(self.lib.kyn_get_state_batch(self.h, ids.ctypes.data_as(_ip), ids.shape[0],
                                                 FIELD[field], ctypes.c_void_p(ptr),
                                                 int(on_device)))

    # results
    def state(self, mid: int, field: str) -> np.ndarray:
        info = self._info[mid]
        rows = info.num_constraints if field in ("lambda", "output") else info.num_nodes
        out = np.zeros((rows, WIDTH[field]))
        self._check(self.lib.kyn_get_state(self.h, mid, FIELD[field], out.ctypes.data_as(_dp)))
        return out

    def convergence(self, mid: int) -> np.ndarray:
        out = np.zeros(64)
        n = ctypes.c_int(0)
        self._check(self.lib.kyn_get_convergence(self.h, mid, out.ctypes.data_as(_dp),
                                                 ctypes.byref(n)))
        return out[: n.value].copy()

    def crs(self, mid: int, values: bool = True):
        info = self._info[mid]
        rp = np.zeros(info.num_dofs + 1, dtype=np.int32)
        ci = np.zeros(info.nnz, dtype=np.int32)
        vals = np.zeros(info.nnz) if values else None
        self._check(self.lib.kyn_get_crs(self.h, mid, rp.ctypes.data_as(_ip),
                                         ci.ctypes.data_as(_ip),
                                         vals.ctypes.data_as(_dp) if values else None))
        return rp, ci, vals

    def system_vectors(self, mid: int):
        n = self._info[mid].num_dofs
        b, x = np.zeros(n), np.zeros(n)
        self._check(self.lib.kyn_get_system_vectors(self.h, mid, b.ctypes.data_as(_dp),
                                                    x.ctypes.data_as(_dp)))
        return b, x
