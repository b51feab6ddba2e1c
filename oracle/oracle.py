"""ORACLE -- test infrastructure only (ctypes front end of getrates_oracle.c).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use this module, as the checker: the product path never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Dict, Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the C restatement (gcc + make, no reference sources needed)."""
    src = os.path.join(_HERE, "getrates_oracle.c")
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = ctypes.CDLL(_LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.oracle_getrates.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int64, dp, dp, dp, dp,
                                         ctypes.c_int]
        _lib.oracle_rates.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int64, dp, dp, dp, dp, dp, dp,
                                      dp, dp, dp, ctypes.c_int]
        _lib.oracle_check_blob.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
        for f in (_lib.oracle_getrates, _lib.oracle_rates, _lib.oracle_check_blob):
            f.restype = ctypes.c_int
    return _lib


def _dp(a: Optional[np.ndarray]):
    if a is None:
        return ctypes.POINTER(ctypes.c_double)()
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def check_blob(blob: bytes) -> int:
    buf = ctypes.create_string_buffer(blob, len(blob))
    return lib().oracle_check_blob(buf, len(blob))


def getrates(blob: bytes, P: np.ndarray, T: np.ndarray, Y: np.ndarray, nthreads: int = 0) -> np.ndarray:
    """wdot[ns, ng] (mol/cm^3/s) for P[ng] (dyne/cm^2), T[ng] (K), Y[ns, ng]."""
    P = np.ascontiguousarray(P, np.float64)
    T = np.ascontiguousarray(T, np.float64)
    Y = np.ascontiguousarray(Y, np.float64)
    ns, ng = Y.shape
    w = np.empty((ns, ng))
    buf = ctypes.create_string_buffer(blob, len(blob))
    rc = lib().oracle_getrates(buf, len(blob), ng, _dp(P), _dp(T), _dp(Y), _dp(w), nthreads)
    if rc:
        raise ValueError(f"oracle rejected the mechanism blob (code {rc})")
    return w


def rates(blob: bytes, P, T, Y, nr: int, nthreads: int = 0) -> Dict[str, np.ndarray]:
    """wdot plus per-reaction kf, kb, qf, qb [nr, ng] (file order) and the
    gross rate S[ns, ng]."""
    P = np.ascontiguousarray(P, np.float64)
    T = np.ascontiguousarray(T, np.float64)
    Y = np.ascontiguousarray(Y, np.float64)
    ns, ng = Y.shape
    out = {"wdot": np.empty((ns, ng)), "S": np.empty((ns, ng))}
    for k in ("kf", "kb", "qf", "qb"):
        out[k] = np.empty((nr, ng))
    buf = ctypes.create_string_buffer(blob, len(blob))
    rc = lib().oracle_rates(buf, len(blob), ng, _dp(P), _dp(T), _dp(Y), _dp(out["wdot"]), _dp(out["kf"]),
                            _dp(out["kb"]), _dp(out["qf"]), _dp(out["qb"]), _dp(out["S"]), nthreads)
    if rc:
        raise ValueError(f"oracle rejected the mechanism blob (code {rc})")
    return out


def errors(w_test: np.ndarray, w_ref: np.ndarray, S: Optional[np.ndarray] = None) -> Dict[str, float]:
    """The three error measures applied to every reported result.

    err_norm  max_k |dw_k| / max_k |w_k| per point (the reference mini-app's
              normwise error, chemistry_mini_app.j2:57-69);
    err_elem  |dw| / max(|w|, 1e-20) per element (tests/test_getrates.py:89-91);
    err_gross |dw| / S per element, S = sum_r |nu| (|qf| + |qb|).
    """
    d = np.abs(w_test - w_ref)
    den = np.abs(w_ref).max(axis=0)
    norm = d.max(axis=0) / np.where(den > 0, den, 1.0)
    elem = d / np.maximum(np.abs(w_ref), 1e-20)
    out = {"norm_max": float(norm.max()), "norm_median": float(np.median(norm)),
           "elem_max": float(elem.max()), "elem_median": float(np.median(elem))}
    if S is not None:
        g = d / np.where(S > 0, S, 1.0)
        out.update(gross_max=float(g.max()), gross_median=float(np.median(g)))
    return out
