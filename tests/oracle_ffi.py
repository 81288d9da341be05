"""ctypes binding of the oracle (oracle/liblnorm_oracle.so): the CPU
restatement of the reference solver, used only as the checker in tests, the
smoke check and the bench's CPU-baseline leg."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "_build" / "liblnorm_oracle.so"
REF_BIN = ORACLE_DIR / "_ref" / "L_OpenMP"

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not ORACLE_LIB.exists():
            build()
        L = C.CDLL(str(ORACLE_LIB))
        L.or_run_cli.argtypes = [C.c_char_p, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_char,
                                 C.c_int, C.c_int, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t,
                                 C.c_char_p, C.c_size_t, C.POINTER(C.c_int64)]
        L.or_run_cli.restype = C.c_int
        L.or_preprocess.argtypes = [C.c_char_p, C.c_size_t, C.c_int, C.c_char, C.c_int,
                                    C.POINTER(C.c_int64), C.c_size_t, C.POINTER(C.c_int),
                                    C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.POINTER(C.c_int)]
        L.or_preprocess.restype = C.c_int
        L.or_enumerate.argtypes = [C.POINTER(C.c_int64), C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_uint64, C.c_uint64, C.c_int, C.POINTER(C.c_int64),
                                   C.POINTER(C.c_uint64)]
        L.or_enumerate.restype = C.c_int
        L.or_total.argtypes = [C.c_int, C.c_int]
        L.or_total.restype = C.c_uint64
        L.or_labels.argtypes = [C.c_uint64, C.c_int, C.c_int, C.POINTER(C.c_int32)]
        L.or_labels.restype = None
        L.or_value.argtypes = [C.POINTER(C.c_int64), C.c_int, C.c_int, C.c_int, C.c_int,
                               C.POINTER(C.c_int32)]
        L.or_value.restype = C.c_int64
        _lib = L
    return _lib


def run_cli(text: str, d: int, stat: str = "n", marginal: bool = False,
            blocks: int = 512, threads: int = 32, nthreads: int = 0):
    """Full CLI pipeline: returns (rc, stdout, strategy_name, strategy_text, value)."""
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    raw = text.encode()
    out = C.create_string_buffer(1 << 20)
    strat = C.create_string_buffer(1 << 16)
    name = C.create_string_buffer(64)
    val = C.c_int64(0)
    rc = lib().or_run_cli(raw, len(raw), blocks, threads, d, (stat or "n")[0].encode(),
                          int(marginal), nthreads, out, len(out), strat, len(strat), name,
                          len(name), C.byref(val))
    return rc, out.value.decode(), name.value.decode(), strat.value.decode(), int(val.value)


def preprocess(text: str, d: int, stat: str = "n", marginal: bool = False):
    """Reduced matrix (last row fixed), effective d and marginal flag."""
    raw = text.encode()
    cap = 1 << 22
    red = (C.c_int64 * cap)()
    r, c, de, me, tr = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
    rc = lib().or_preprocess(raw, len(raw), d, (stat or "n")[0].encode(), int(marginal), red, cap,
                             C.byref(r), C.byref(c), C.byref(de), C.byref(me), C.byref(tr))
    if rc not in (0, -1):
        raise ValueError(f"oracle rejected input (rc={rc})")
    a = np.frombuffer(red, dtype=np.int64, count=r.value * c.value).reshape(r.value, c.value).copy()
    return dict(rc=rc, matrix=a, d=de.value, marginal=me.value, transposed=tr.value)


def enumerate_max(a: np.ndarray, d: int, marginal: bool = False, lo: int = 0, hi: int = 0,
                  nthreads: int = 0):
    """(max value, smallest Gray index attaining it) over [lo, hi)."""
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    a = np.ascontiguousarray(a, dtype=np.int64)
    v, n = C.c_int64(), C.c_uint64()
    rc = lib().or_enumerate(a.ctypes.data_as(C.POINTER(C.c_int64)), a.shape[0], a.shape[1], d,
                            int(marginal), lo, hi, nthreads, C.byref(v), C.byref(n))
    if rc != 0:
        raise ValueError("bad range")
    return int(v.value), int(n.value)


def total(rows: int, d: int) -> int:
    return int(lib().or_total(rows, d))


def labels(N: int, rows: int, d: int) -> np.ndarray:
    out = (C.c_int32 * max(rows - 1, 1))()
    lib().or_labels(N, rows, d, out)
    return np.frombuffer(out, dtype=np.int32, count=max(rows - 1, 0)).copy()


def value(a: np.ndarray, d: int, marginal: bool, labs) -> int:
    a = np.ascontiguousarray(a, dtype=np.int64)
    lab = np.ascontiguousarray(np.asarray(labs, dtype=np.int32))
    if lab.size == 0:
        lab = np.zeros(1, dtype=np.int32)
    return int(lib().or_value(a.ctypes.data_as(C.POINTER(C.c_int64)), a.shape[0], a.shape[1], d,
                              int(marginal), lab.ctypes.data_as(C.POINTER(C.c_int32))))
