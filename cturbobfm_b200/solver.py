"""Python binding of the C ABI in include/ctbfm.h (ctypes).

``Solver`` mirrors the reference's ``Solver(Config&, Mesh&)`` + ``solve()``
(include/solver.hpp:45-53) for one operating point given by an input.ini in the
reference's format. All computation happens in libctbfm.so on the GPU; this
module only moves host buffers across the C boundary. There is no CPU
fallback: a missing library or device raises.
"""

from __future__ import annotations

import ctypes
import os
from typing import Dict, Optional

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libctbfm.so")

CTBFM_OK = 0
CTBFM_E_CONFIG = 1
CTBFM_E_CUDA = 2
CTBFM_E_DIVERGED = 3
CTBFM_E_ARGUMENT = 4
CTBFM_E_UNSUPPORTED = 5

STATUS_RUNNING, STATUS_CONVERGED, STATUS_DIVERGED, STATUS_DEVICE_ERROR = 0, 1, 2, 3
STAGE_MODES = ("split", "fused", "persistent")
PRECISION_FP64, PRECISION_FP32_KAHAN = 0, 1


class CtbfmError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


class SolverDiverged(CtbfmError):
    pass


class Info(ctypes.Structure):
    _fields_ = [
        ("ni", ctypes.c_int64),
        ("nj", ctypes.c_int64),
        ("nk", ctypes.c_int64),
        ("topology", ctypes.c_int32),
        ("n_stages", ctypes.c_int32),
        ("iteration", ctypes.c_int64),
        ("max_iterations", ctypes.c_int64),
        ("status", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("time", ctypes.c_double),
        ("device_bytes", ctypes.c_int64),
        ("face_tile", ctypes.c_int32 * 3),
        ("fused_stage", ctypes.c_int32),
        ("persistent_stage", ctypes.c_int32),
        ("tuned_stage_ms", ctypes.c_double * 3),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [(f, ctypes.c_int64) for f in ("rounds", "rebuilds", "promotions", "reruns")] + \
        [(f, ctypes.c_double) for f in ("wait_s", "process_s", "rebuild_s", "promote_s", "release_s", "batch_s",
                                        "prepare_s", "enqueue_s", "admit_s")]


class Result(ctypes.Structure):
    _fields_ = [
        ("id", ctypes.c_int64),
        ("status", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("iterations", ctypes.c_int64),
        ("t_submit", ctypes.c_double),
        ("t_admit", ctypes.c_double),
        ("t_done", ctypes.c_double),
        ("massflow", ctypes.c_double * 6),
        ("turbo", ctypes.c_double * 4),
        ("error", ctypes.c_int32),
        ("message", ctypes.c_char * 240),
    ]


class PatchDesc(ctypes.Structure):
    """ctbfm_patch: one row of boundaries.csv."""

    _fields_ = [("name", ctypes.c_char_p)] + [(f, ctypes.c_int64) for f in
                                              ("i_min", "i_max", "j_min", "j_max", "k_min", "k_max")]


class CaseDesc(ctypes.Structure):
    """ctbfm_case_desc: settings, grid arrays and patches held in memory."""

    _fields_ = [
        ("ni", ctypes.c_int64),
        ("nj", ctypes.c_int64),
        ("nk", ctypes.c_int64),
        ("x", ctypes.POINTER(ctypes.c_double)),
        ("y", ctypes.POINTER(ctypes.c_double)),
        ("z", ctypes.POINTER(ctypes.c_double)),
        ("n_fields", ctypes.c_int32),
        ("field_names", ctypes.POINTER(ctypes.c_char_p)),
        ("fields", ctypes.POINTER(ctypes.POINTER(ctypes.c_double))),
        ("n_patches", ctypes.c_int32),
        ("patches", ctypes.POINTER(PatchDesc)),
        ("n_settings", ctypes.c_int32),
        ("keys", ctypes.POINTER(ctypes.c_char_p)),
        ("values", ctypes.POINTER(ctypes.c_char_p)),
        ("directory", ctypes.c_char_p),
    ]


def case_desc(case, directory: Optional[str] = None):
    """The ctbfm_case_desc of a ``cases.Case`` (its settings, grid arrays and
    patches, each patch's type and values under the patch's name as in
    input.ini) and the objects that keep its buffers alive. Files the case
    names (a fluid table, the Chima scaling functions) are written to
    ``directory``, against which the settings that name files resolve."""
    if case.table is not None or case.files:
        if directory is None:
            raise ValueError(f"case {case.name} names input files: pass a directory to write them to")
        case.write_side_files(directory)
    ni, nj, nk = case.shape
    arrays = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (case.x, case.y, case.z)]
    names = list(case.fields.keys())
    cols = [np.ascontiguousarray(case.fields[n], dtype=np.float64).reshape(-1) for n in names]
    settings = dict(case.settings)
    for p in case.patches:
        settings[p.name] = p.spec
    keys = [k.encode() for k in settings]
    vals = [str(v).encode() for v in settings.values()]
    pats = (PatchDesc * max(len(case.patches), 1))()
    pnames = [p.name.encode() for p in case.patches]
    for q, p in enumerate(case.patches):
        pats[q] = PatchDesc(pnames[q], p.i_min, p.i_max, p.j_min, p.j_max, p.k_min, p.k_max)
    fname_arr = (ctypes.c_char_p * max(len(names), 1))(*[n.encode() for n in names])
    col_arr = (ctypes.POINTER(ctypes.c_double) * max(len(cols), 1))(*[_ptr(c) for c in cols])
    key_arr = (ctypes.c_char_p * max(len(keys), 1))(*keys)
    val_arr = (ctypes.c_char_p * max(len(vals), 1))(*vals)
    d = CaseDesc(ni, nj, nk, _ptr(arrays[0]), _ptr(arrays[1]), _ptr(arrays[2]), len(names), fname_arr, col_arr,
                 len(case.patches), pats, len(keys), key_arr, val_arr,
                 os.path.abspath(directory).encode() if directory else None)
    return d, (arrays, cols, keys, vals, pnames, pats, fname_arr, col_arr, key_arr, val_arr)


_lib = None

# Every symbol include/ctbfm.h declares, with its ctypes signature.
_DP = ctypes.POINTER(ctypes.c_double)
_VP = ctypes.c_void_p
_I64 = ctypes.c_int64
SIGNATURES = {
    "ctbfm_create_from_ini": ([ctypes.c_char_p, ctypes.POINTER(_VP)], ctypes.c_int),
    "ctbfm_create": ([ctypes.POINTER(CaseDesc), ctypes.POINTER(_VP)], ctypes.c_int),
    "ctbfm_destroy": ([_VP], None),
    "ctbfm_set_stream": ([_VP, _VP], ctypes.c_int),
    "ctbfm_get_info": ([_VP, ctypes.POINTER(Info)], ctypes.c_int),
    "ctbfm_step": ([_VP, _I64, ctypes.POINTER(_I64)], ctypes.c_int),
    "ctbfm_enqueue": ([_VP, _I64], ctypes.c_int),
    "ctbfm_autotune": ([_VP], ctypes.c_int),
    "ctbfm_solve": ([_VP, ctypes.POINTER(_I64)], ctypes.c_int),
    "ctbfm_compute_residual": ([_VP] + [_DP] * 6, ctypes.c_int),
    "ctbfm_compute_residual_noalloc": ([_VP] + [_DP] * 6, ctypes.c_int),
    "ctbfm_get_state": ([_VP] + [_DP] * 5, ctypes.c_int),
    "ctbfm_set_state": ([_VP] + [_DP] * 5, ctypes.c_int),
    "ctbfm_get_lognorm": ([_VP, _DP], ctypes.c_int),
    "ctbfm_write_solution": ([_VP, ctypes.c_char_p], ctypes.c_int),
    "ctbfm_get_history": ([_VP, _I64, _DP, _DP, _DP, _DP, ctypes.POINTER(_I64)], ctypes.c_int),
    "ctbfm_get_turbo": ([_VP, _DP, _DP], ctypes.c_int),
    "ctbfm_get_history_time": ([_VP, _I64, _DP, ctypes.POINTER(_I64)], ctypes.c_int),
    "ctbfm_profile_kernels": ([_VP, ctypes.c_int, _DP], ctypes.c_int),
    "ctbfm_batch_create": ([ctypes.POINTER(_VP), ctypes.c_int32, ctypes.POINTER(_VP)], ctypes.c_int),
    "ctbfm_batch_destroy": ([_VP], None),
    "ctbfm_batch_set_stream": ([_VP, _VP], ctypes.c_int),
    "ctbfm_batch_enqueue": ([_VP, _I64], ctypes.c_int),
    "ctbfm_batch_autotune": ([_VP], ctypes.c_int),
    "ctbfm_batch_stage_kernels": ([_VP, ctypes.POINTER(ctypes.c_int32), _DP], ctypes.c_int),
    "ctbfm_batch_step": ([_VP, _I64, ctypes.POINTER(_I64)], ctypes.c_int),
    "ctbfm_batch_status": ([_VP, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(_I64), _DP, _DP], ctypes.c_int),
    "ctbfm_promote_fp64": ([_VP], ctypes.c_int),
    "ctbfm_server_create": ([ctypes.c_uint64, ctypes.c_int32, _I64, _I64, _I64, ctypes.c_int32,
                             ctypes.POINTER(_VP)], ctypes.c_int),
    "ctbfm_server_destroy": ([_VP], None),
    "ctbfm_server_set_promotion": ([_VP, ctypes.c_double], ctypes.c_int),
    "ctbfm_server_get_stats": ([_VP, ctypes.POINTER(ServerStats)], ctypes.c_int),
    "ctbfm_server_submit": ([_VP, ctypes.c_char_p, ctypes.POINTER(_I64)], ctypes.c_int),
    "ctbfm_server_submit_case": ([_VP, ctypes.POINTER(CaseDesc), ctypes.POINTER(_I64)], ctypes.c_int),
    "ctbfm_server_pump": ([_VP, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
    "ctbfm_server_results": ([_VP, ctypes.POINTER(Result), ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)],
                             ctypes.c_int),
    "ctbfm_last_error": ([], ctypes.c_char_p),
    "ctbfm_version": ([], ctypes.c_char_p),
}


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libctbfm.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise CtbfmError(CTBFM_E_CUDA, f"{path} is missing: build it with cturbobfm_b200.build.build()")
        lib = ctypes.CDLL(path)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_DP)


def _check(rc: int):
    if rc != CTBFM_OK:
        msg = load_library().ctbfm_last_error().decode()
        if rc == CTBFM_E_DIVERGED:
            raise SolverDiverged(rc, msg)
        raise CtbfmError(rc, msg)


class Solver:
    """One operating point on the current CUDA device."""

    def __init__(self, ini_path: str):
        lib = load_library()
        h = _VP()
        _check(lib.ctbfm_create_from_ini(os.path.abspath(ini_path).encode(), ctypes.byref(h)))
        self._adopt(h)

    @classmethod
    def from_case(cls, case, directory: Optional[str] = None) -> "Solver":
        """A solver built from a ``cases.Case`` held in memory (ctbfm_create):
        no input.ini, grid or boundaries file is written. ``directory`` takes
        the other files the case names and is where settings that name files
        resolve."""
        desc, keep = case_desc(case, directory)
        h = _VP()
        _check(load_library().ctbfm_create(ctypes.byref(desc), ctypes.byref(h)))
        del keep
        self = cls.__new__(cls)
        self._adopt(h)
        return self

    def _adopt(self, h):
        self._h = h
        inf = self.info()
        self.shape = (int(inf.ni), int(inf.nj), int(inf.nk))
        self.n = self.shape[0] * self.shape[1] * self.shape[2]
        self.n_stages = int(inf.n_stages)

    def close(self):
        if getattr(self, "_h", None):
            load_library().ctbfm_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stage_kernels(self):
        """(mode, {mode: ms}) as Batch.stage_kernels, from ctbfm_get_info."""
        inf = self.info()
        mode = "persistent" if inf.persistent_stage else ("fused" if inf.fused_stage else "split")
        return mode, {k: float(v) for k, v in zip(STAGE_MODES, inf.tuned_stage_ms)}

    def promote_fp64(self):
        """Continues a fp32_kahan solve in FP64 (no-op for FP64 solvers)."""
        _check(load_library().ctbfm_promote_fp64(self._h))

    def info(self) -> Info:
        inf = Info()
        _check(load_library().ctbfm_get_info(self._h, ctypes.byref(inf)))
        return inf

    def set_stream(self, stream_ptr: Optional[int]):
        _check(load_library().ctbfm_set_stream(self._h, _VP(stream_ptr or 0)))

    def step(self, n_iter: int) -> int:
        done = _I64()
        _check(load_library().ctbfm_step(self._h, int(n_iter), ctypes.byref(done)))
        return int(done.value)

    def enqueue(self, n_iter: int):
        _check(load_library().ctbfm_enqueue(self._h, int(n_iter)))

    def autotune(self):
        """ctbfm_autotune: face tiles and stage fusion, timed now."""
        _check(load_library().ctbfm_autotune(self._h))

    def solve(self) -> int:
        done = _I64()
        _check(load_library().ctbfm_solve(self._h, ctypes.byref(done)))
        return int(done.value)

    def residual(self):
        dt = np.zeros(self.n)
        r = np.zeros((5, self.n))
        _check(load_library().ctbfm_compute_residual(self._h, _ptr(dt), *[_ptr(r[v]) for v in range(5)]))
        return dt, r

    def residual_noalloc(self):
        """ctbfm_compute_residual_noalloc: the residual evaluation without any
        device allocation (face-flux scratch in the library's static array)."""
        dt = np.zeros(self.n)
        r = np.zeros((5, self.n))
        _check(load_library().ctbfm_compute_residual_noalloc(self._h, _ptr(dt), *[_ptr(r[v]) for v in range(5)]))
        return dt, r

    def state(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        u = np.zeros((5, self.n)) if out is None else out
        _check(load_library().ctbfm_get_state(self._h, *[_ptr(u[v]) for v in range(5)]))
        return u

    def set_state(self, u: np.ndarray):
        u = np.ascontiguousarray(u, dtype=np.float64)
        _check(load_library().ctbfm_set_state(self._h, *[_ptr(u[v]) for v in range(5)]))

    def write_solution(self, path: str) -> str:
        """ctbfm_write_solution: the current state as a volume CSV in the
        reference's format (Output::writeSolution, src/output.cpp:384-447),
        readable back as a restart file. Returns the path."""
        _check(load_library().ctbfm_write_solution(self._h, os.fspath(path).encode()))
        return os.fspath(path)

    def lognorm(self) -> np.ndarray:
        out = np.zeros(5)
        _check(load_library().ctbfm_get_lognorm(self._h, _ptr(out)))
        return out

    def history(self) -> Dict[str, np.ndarray]:
        lib = load_library()
        rows = _I64()
        _check(lib.ctbfm_get_history(self._h, 0, None, None, None, None, ctypes.byref(rows)))
        n = int(rows.value)
        ln, mf, tp, hub = np.zeros((n, 5)), np.zeros((n, 6)), np.zeros((n, 4)), np.zeros(n)
        t = np.zeros(n)
        if n:
            _check(lib.ctbfm_get_history(self._h, n, _ptr(ln), _ptr(mf), _ptr(tp), _ptr(hub), ctypes.byref(rows)))
            _check(lib.ctbfm_get_history_time(self._h, n, _ptr(t), ctypes.byref(rows)))
        return {"lognorm": ln, "massflow": mf, "turbo": tp, "hub": hub, "time": t}

    def turbo(self):
        mf, tp = np.zeros(6), np.zeros(4)
        _check(load_library().ctbfm_get_turbo(self._h, _ptr(mf), _ptr(tp)))
        return mf, tp

    KERNELS = ("k_bint", "k_dt", "k_pre", "k_faces_I", "k_faces_J", "k_faces_K", "k_nodes", "k_periodic",
               "k_finalize", "k_prim", "k_stage")

    def profile_kernels(self, reps: int = 20) -> Dict[str, float]:
        """Average device time per launch (ms) of each kernel kind, CUDA events."""
        out = np.zeros(len(self.KERNELS))
        _check(load_library().ctbfm_profile_kernels(self._h, int(reps), _ptr(out)))
        return {k: float(v) for k, v in zip(self.KERNELS, out)}

    @property
    def iteration(self) -> int:
        return int(self.info().iteration)

    @property
    def status(self) -> int:
        return int(self.info().status)

    @property
    def time(self) -> float:
        return float(self.info().time)


class Batch:
    """Solvers of one GPU_PRECISION advanced together (ctbfm_batch_*): one
    launch per kernel family for all members. The solvers stay usable for
    queries between steps and must outlive the batch."""

    def __init__(self, solvers):
        lib = load_library()
        self.solvers = list(solvers)
        arr = (_VP * len(self.solvers))(*[s._h for s in self.solvers])
        h = _VP()
        _check(lib.ctbfm_batch_create(arr, len(self.solvers), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            load_library().ctbfm_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.solvers)

    def set_stream(self, stream_ptr: Optional[int]):
        _check(load_library().ctbfm_batch_set_stream(self._h, _VP(stream_ptr or 0)))

    def enqueue(self, n_iter: int):
        _check(load_library().ctbfm_batch_enqueue(self._h, int(n_iter)))

    def autotune(self):
        """ctbfm_batch_autotune: face tiles and stage fusion, timed now."""
        _check(load_library().ctbfm_batch_autotune(self._h))

    def stage_kernels(self):
        """(mode, {mode: ms}): the batch's stage kernels ("split", "fused" or
        "persistent") and the autotuner's time of one stage in each (0: not
        timed) (ctbfm_batch_stage_kernels)."""
        f = ctypes.c_int32(0)
        ms = np.zeros(3)
        _check(load_library().ctbfm_batch_stage_kernels(self._h, ctypes.byref(f), _ptr(ms)))
        return STAGE_MODES[f.value], {k: float(v) for k, v in zip(STAGE_MODES, ms)}

    def step(self, n_iter: int) -> int:
        done = _I64(0)
        _check(load_library().ctbfm_batch_step(self._h, int(n_iter), ctypes.byref(done)))
        return int(done.value)

    def status(self) -> Dict[str, np.ndarray]:
        m = len(self.solvers)
        st = np.zeros(m, np.int32)
        it = np.zeros(m, np.int64)
        ln = np.zeros((m, 5))
        bd = np.zeros(m)
        _check(load_library().ctbfm_batch_status(self._h, st.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                 it.ctypes.data_as(ctypes.POINTER(_I64)), _ptr(ln), _ptr(bd)))
        return {"status": st, "iterations": it, "lognorm": ln, "best_drop": bd}


class Server:
    """Continuous batching of operating-point solves (ctbfm_server_*)."""

    def __init__(self, budget_bytes: int = 0, max_active: int = 1024, chunk: int = 200, stall_window: int = 0,
                 host_threads: int = 4, max_active_nodes: int = 0, promote_orders: float = 0.0):
        h = _VP()
        _check(load_library().ctbfm_server_create(int(budget_bytes), int(max_active), int(max_active_nodes), int(chunk),
                                                  int(stall_window), int(host_threads), ctypes.byref(h)))
        self._h = h
        if promote_orders > 0:
            _check(load_library().ctbfm_server_set_promotion(h, float(promote_orders)))

    def close(self):
        if getattr(self, "_h", None):
            load_library().ctbfm_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, ini_path: str) -> int:
        rid = _I64(0)
        _check(load_library().ctbfm_server_submit(self._h, os.path.abspath(ini_path).encode(), ctypes.byref(rid)))
        return int(rid.value)

    def submit_case(self, case, directory: Optional[str] = None) -> int:
        """Queues a ``cases.Case`` held in memory (ctbfm_server_submit_case)."""
        desc, keep = case_desc(case, directory)
        rid = _I64(0)
        _check(load_library().ctbfm_server_submit_case(self._h, ctypes.byref(desc), ctypes.byref(rid)))
        del keep
        return int(rid.value)

    def stats(self) -> Dict[str, float]:
        """Where the pumping thread's time went (ctbfm_server_get_stats)."""
        st = ServerStats()
        _check(load_library().ctbfm_server_get_stats(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def pump(self):
        a, w = ctypes.c_int32(0), ctypes.c_int32(0)
        _check(load_library().ctbfm_server_pump(self._h, ctypes.byref(a), ctypes.byref(w)))
        return int(a.value), int(w.value)

    def results(self, max_results: int = 4096):
        buf = (Result * max_results)()
        n = ctypes.c_int32(0)
        _check(load_library().ctbfm_server_results(self._h, buf, max_results, ctypes.byref(n)))
        out = []
        for r in buf[: n.value]:
            out.append({"id": r.id, "status": r.status, "precision": r.precision, "iterations": r.iterations,
                        "t_submit": r.t_submit, "t_admit": r.t_admit, "t_done": r.t_done,
                        "massflow": list(r.massflow), "turbo": list(r.turbo), "error": r.error,
                        "message": r.message.decode(errors="replace")})
        return out
