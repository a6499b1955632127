"""Python access to the CPU oracle (test infrastructure only).

Two checkers live here:
  * ``Oracle``: ctypes binding of liboracle.so, the plain-C restatement of the
    reference's explicit loop (ctbfm_oracle.c);
  * ``ref_harness``: runs oracle/_ref/ref_harness, the reference solver built
    from its own sources (refbuild/Makefile), in a case directory and parses
    its binary dump.

Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module; the product library never does.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_HARNESS = os.path.join(REF_DIR, "ref_harness")
REF_CLI = os.path.join(REF_DIR, "turbobfm")

_lib = None


def build() -> str:
    """Compiles liboracle.so (gcc, seconds)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        lib.oracle_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(vp)]
        lib.oracle_create.restype = ctypes.c_int
        lib.oracle_destroy.argtypes = [vp]
        lib.oracle_last_error.restype = ctypes.c_char_p
        lib.oracle_shape.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        lib.oracle_run.argtypes = [vp, ctypes.c_long, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_int)]
        lib.oracle_run.restype = ctypes.c_int
        lib.oracle_residual.argtypes = [vp] + [dp] * 6
        lib.oracle_residual.restype = ctypes.c_int
        lib.oracle_get_state.argtypes = [vp] + [dp] * 5
        lib.oracle_get_nuhat.argtypes = [vp, dp]
        lib.oracle_get_nuhat.restype = ctypes.c_int
        lib.oracle_set_state.argtypes = [vp] + [dp] * 5
        lib.oracle_history.argtypes = [vp, dp, dp, dp, dp]
        lib.oracle_history.restype = ctypes.c_long
        lib.oracle_time.argtypes = [vp]
        lib.oracle_time.restype = ctypes.c_double
        _lib = lib
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class OracleError(RuntimeError):
    pass


class Oracle:
    """The reference algorithm on the CPU, one serial FP64 instance."""

    def __init__(self, ini_path: str):
        lib = _load()
        h = ctypes.c_void_p()
        if lib.oracle_create(os.path.abspath(ini_path).encode(), ctypes.byref(h)) != 0:
            raise OracleError(lib.oracle_last_error().decode())
        self._h = h
        shp = (ctypes.c_longlong * 3)()
        lib.oracle_shape(h, shp)
        self.shape = (int(shp[0]), int(shp[1]), int(shp[2]))
        self.n = self.shape[0] * self.shape[1] * self.shape[2]

    def close(self):
        if self._h:
            _load().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, n_iter: int) -> Dict[str, int]:
        done = ctypes.c_long()
        conv = ctypes.c_int()
        rc = _load().oracle_run(self._h, n_iter, ctypes.byref(done), ctypes.byref(conv))
        return {"status": rc, "iterations": done.value, "converged": conv.value}

    def residual(self):
        dt = np.zeros(self.n)
        r = np.zeros((5, self.n))
        _load().oracle_residual(self._h, _ptr(dt), *[_ptr(r[c]) for c in range(5)])
        return dt, r

    def state(self) -> np.ndarray:
        u = np.zeros((5, self.n))
        _load().oracle_get_state(self._h, *[_ptr(u[c]) for c in range(5)])
        return u

    def nuhat(self) -> np.ndarray:
        """The Spalart-Allmaras working variable per node (zeros without it)."""
        out = np.zeros(self.n)
        _load().oracle_get_nuhat(self._h, _ptr(out))
        return out

    def set_state(self, u: np.ndarray):
        u = np.ascontiguousarray(u, dtype=np.float64)
        _load().oracle_set_state(self._h, *[_ptr(u[c]) for c in range(5)])

    def history(self) -> Dict[str, np.ndarray]:
        lib = _load()
        n = lib.oracle_history(self._h, None, None, None, None)
        ln, mf, tp, hub = np.zeros((n, 5)), np.zeros((n, 6)), np.zeros((n, 4)), np.zeros(n)
        lib.oracle_history(self._h, _ptr(ln), _ptr(mf), _ptr(tp), _ptr(hub))
        return {"lognorm": ln, "massflow": mf, "turbo": tp, "hub": hub}

    @property
    def time(self) -> float:
        return _load().oracle_time(self._h)


def reference_root() -> str:
    """Where the reference's sources are read for the reference build: the
    CTBFM_REFERENCE environment variable, else the REF default of the build
    recipe (oracle/refbuild/Makefile)."""
    env = os.environ.get("CTBFM_REFERENCE")
    if env:
        return env
    mk = os.path.join(os.path.dirname(os.path.abspath(__file__)), "refbuild", "Makefile")
    for line in open(mk):
        if line.startswith("REF ?="):
            return line.split("=", 1)[1].strip()
    return ""


def ref_available() -> bool:
    return os.path.exists(REF_HARNESS)


def ref_harness(mode: str, ini_path: str, n_iter: Optional[int] = None,
                timeout: float = 600.0) -> Dict[str, np.ndarray]:
    """Runs the reference build in the case directory and parses its dump."""
    case_dir = os.path.dirname(os.path.abspath(ini_path))
    out = os.path.join(case_dir, f"ref_{mode}.bin")
    args = [REF_HARNESS, mode, os.path.basename(ini_path)]
    if mode == "steps":
        args.append(str(int(n_iter)))
    args.append(out)
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", "1")
    r = subprocess.run(args, cwd=case_dir, capture_output=True, text=True, timeout=timeout, env=env)
    if r.returncode != 0:
        raise OracleError(f"ref_harness {mode} failed: {r.stderr.strip()[-400:]}")
    raw = np.fromfile(out, dtype=np.uint8)
    ni, nj, nk = np.frombuffer(raw[:24].tobytes(), dtype=np.int64)
    n = int(ni * nj * nk)
    off = 24
    res: Dict[str, np.ndarray] = {"shape": np.array([ni, nj, nk])}

    def take(count, dtype=np.float64):
        nonlocal off
        a = np.frombuffer(raw[off:off + 8 * count].tobytes(), dtype=dtype)
        off += 8 * count
        return a

    if mode == "run":
        res["state"] = take(5 * n).reshape(5, n)
    elif mode == "residual":
        res["dt"] = take(n)
        res["residual"] = take(5 * n).reshape(5, n)
    elif mode == "steps":
        done = int(take(1, np.int64)[0])
        res["iterations"] = done
        res["converged"] = int(take(1, np.int64)[0])
        res["time"] = float(take(1)[0])
        res["state"] = take(5 * n).reshape(5, n)
        res["lognorm"] = take(5 * done).reshape(done, 5)
        res["massflow"] = take(6 * done).reshape(done, 6)
        res["turbo"] = take(4 * done).reshape(done, 4)
        res["hub"] = take(done)
        if off + 8 * n <= raw.size:  # the Spalart-Allmaras working variable
            res["nuhat"] = take(n)
    return res
