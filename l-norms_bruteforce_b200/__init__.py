"""Python binding of the B200-native exact L_d-norm solver (liblnorms_b200.so).

The stages mirror the reference's pipeline (istvanmarton/L-norms_BruteForce,
L_CUDA.cu:414-439): read and preprocess a matrix (``Problem``), solve on the
GPU (``Problem.solve`` / ``solve_reduced`` / ``Plan``), and report the value
line and the strategy file in the original indexing (``Problem.report``).
``lnorm`` runs the whole pipeline in one call, like ``./L_CUDA``.

There is no CPU fallback: without the built library or a CUDA device every
solve raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "lib" / "liblnorms_b200.so"
CLI_PATH = PKG_DIR / "lib" / "L_CUDA"

LD_OK = 0
STATUS = {0: "LD_OK", 1: "LD_ERR_ARG", 2: "LD_ERR_INPUT", 3: "LD_ERR_LIMIT", 4: "LD_ERR_CUDA",
          5: "LD_ERR_NODEV", 6: "LD_ERR_IO", 7: "LD_ERR_TIMEOUT", 8: "LD_ERR_NOMEM"}
KERNEL_TABLE, KERNEL_WIDE = 1, 2


class LdError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class Result(C.Structure):
    _fields_ = [("value", C.c_int64), ("gray_index", C.c_uint64), ("labelings", C.c_uint64),
                ("kernel_ms", C.c_float), ("kernel_kind", C.c_int32), ("lane_bits", C.c_int32),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64), ("evaluated", C.c_uint64)]


class Options(C.Structure):
    _fields_ = [("device", C.c_int32), ("low_rows", C.c_int32), ("threads_per_block", C.c_int32),
                ("blocks", C.c_int32), ("tile", C.c_int32), ("kernel", C.c_int32),
                ("lane_bits", C.c_int32), ("shard_index", C.c_int32), ("shard_count", C.c_int32),
                ("prune_policy", C.c_int32), ("enumerate_all", C.c_int32), ("batch_split", C.c_int32),
                ("column_split", C.c_int32), ("paired_walks", C.c_int32), ("pack16", C.c_int32),
                ("walk_fetch", C.c_int32), ("batch_row_search", C.c_int32), ("stream", C.c_void_p)]


class ProblemInfo(C.Structure):
    _fields_ = [("rows_in", C.c_int32), ("cols_in", C.c_int32), ("rows", C.c_int32),
                ("cols", C.c_int32), ("d_user", C.c_int32), ("d", C.c_int32),
                ("marginal_user", C.c_int32), ("marginal", C.c_int32), ("transposed", C.c_int32),
                ("max_rows", C.c_int32), ("labelings", C.c_uint64)]


class PruneStats(C.Structure):
    _fields_ = [("walks_total", C.c_uint64), ("walks_kept", C.c_uint64), ("highs_total", C.c_uint64),
                ("highs_visited", C.c_uint64), ("highs_kept", C.c_uint64), ("block", C.c_uint64),
                ("incumbent", C.c_int64), ("bound_ms", C.c_float), ("scan_ms", C.c_float),
                ("pruned", C.c_int32), ("low_rows", C.c_int32), ("walk_rows", C.c_int32)]


# Every exported symbol of include/lnorms_b200.h: (name, restype, argtypes)
_P = C.c_void_p
_I64P = C.POINTER(C.c_int64)
_I32P = C.POINTER(C.c_int32)
_F32P = C.POINTER(C.c_float)
SIGNATURES = [
    ("ld_options_init", None, [C.POINTER(Options)]),
    ("ld_problem_from_text", C.c_int, [C.c_char_p, C.c_size_t, C.c_int32, C.c_char, C.c_int32, C.POINTER(_P)]),
    ("ld_problem_from_file", C.c_int, [C.c_char_p, C.c_int32, C.c_char, C.c_int32, C.POINTER(_P)]),
    ("ld_problem_from_matrix", C.c_int, [_I64P, C.c_int32, C.c_int32, C.c_int32, C.c_char, C.c_int32, C.POINTER(_P)]),
    ("ld_problem_destroy", None, [_P]),
    ("ld_problem_get_info", C.c_int, [_P, C.POINTER(ProblemInfo)]),
    ("ld_problem_reduced", C.c_int, [_P, _I64P, C.c_size_t]),
    ("ld_problem_log", C.c_char_p, [_P]),
    ("ld_problem_check_launch", C.c_int, [_P, C.c_int32, C.c_int32]),
    ("ld_problem_solve", C.c_int, [_P, C.POINTER(Options), C.POINTER(Result)]),
    ("ld_solve_reduced", C.c_int, [_I64P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(Options),
                                   C.POINTER(Result), _I32P]),
    ("ld_solve_reduced_noalloc", C.c_int, [_I64P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                           C.c_void_p, C.POINTER(Result), _I32P]),
    ("ld_solve_pruned", C.c_int, [_I64P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(Options),
                                  _I32P, C.POINTER(Result), _I32P, C.POINTER(PruneStats)]),
    ("ld_local_search", C.c_int, [_I64P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _I32P, C.c_int32,
                                  C.c_int32, C.c_int32, _I64P, _I32P]),
    ("ld_batch_create", C.c_int, [C.c_int32, C.POINTER(_I64P), _I32P, _I32P, _I32P, _I32P, C.POINTER(Options),
                                  C.c_int32, C.POINTER(_P)]),
    ("ld_batch_launch", C.c_int, [_P]),
    ("ld_batch_results", C.c_int, [_P, _I64P, C.POINTER(C.c_uint64), C.POINTER(C.c_float)]),
    ("ld_batch_describe", C.c_int, [_P, C.c_char_p, C.c_size_t]),
    ("ld_batch_evaluated", C.c_int, [_P, C.POINTER(C.c_uint64)]),
    ("ld_batch_destroy", None, [_P]),
    ("ld_gray_labels", C.c_int, [C.c_uint64, C.c_int32, C.c_int32, _I32P]),
    ("ld_problem_report", C.c_int, [_P, C.POINTER(Result), _I32P, C.c_int32, _I32P, C.c_char_p, C.c_size_t]),
    ("ld_plan_create", C.c_int, [_I64P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(Options), C.POINTER(_P)]),
    ("ld_plan_launch", C.c_int, [_P]),
    ("ld_plan_result", C.c_int, [_P, C.POINTER(Result), _I32P]),
    ("ld_plan_range", C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("ld_plan_describe", C.c_int, [_P, C.c_char_p, C.c_size_t]),
    ("ld_plan_stream", C.c_void_p, [_P]),
    ("ld_plan_result_device", C.c_void_p, [_P]),
    ("ld_plan_destroy", None, [_P]),
    ("ld_mlp_create", C.c_int, [C.c_int32, C.c_uint64, C.c_float, C.c_int32, C.POINTER(_P)]),
    ("ld_mlp_param_count", C.c_int64, []),
    ("ld_mlp_get_params", C.c_int, [_P, _F32P]),
    ("ld_mlp_set_params", C.c_int, [_P, _F32P]),
    ("ld_mlp_forward", C.c_int, [_P, _F32P, C.c_int32, _F32P]),
    ("ld_mlp_gradients", C.c_int, [_P, _F32P, _F32P, _F32P, C.c_int32, _F32P, _F32P]),
    ("ld_mlp_train_step", C.c_int, [_P, _F32P, _F32P, _F32P, C.c_int32, C.c_float, _F32P]),
    ("ld_mlp_destroy", None, [_P]),
    ("ld_tc_gemm", C.c_int, [C.POINTER(C.c_uint16), C.POINTER(C.c_uint16), C.c_int32, C.c_int32, C.c_int32,
                             _F32P, C.c_int32]),
    ("ld_cli_main", C.c_int, [C.c_int, C.POINTER(C.c_char_p)]),
    ("ld_symmetry_walk_ok", C.c_int32, [C.c_int32, C.c_int32, C.c_uint64]),
    ("ld_symmetry_walks", C.c_int, [C.c_int32, C.c_int32, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("ld_symmetry_walk_at", C.c_int, [C.c_int32, C.c_int32, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("ld_solve_resumable", C.c_int, [_I64P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int32,
                                     C.c_char_p, C.c_int32, C.POINTER(C.c_int32), C.c_void_p, _I32P]),
    ("ld_spectral_basis", C.c_int, [_I64P, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_double),
                                    C.POINTER(C.c_int32)]),
    ("ld_strategy_value", C.c_int, [C.c_char_p, C.c_size_t, C.c_int32, C.c_char, C.c_int32, _I32P, C.c_int32,
                                    _I64P]),
    ("ld_verify_main", C.c_int, [C.c_int, C.POINTER(C.c_char_p)]),
    ("ld_measure_int32_peak", C.c_int, [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("ld_last_error", C.c_char_p, []),
    ("ld_version", C.c_char_p, []),
]

_lib = None


def lib():
    """The loaded solver library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with "
                              f"`make -C {PKG_DIR}` (or __graft_entry__.build())")
        L = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(st: int) -> None:
    if st != LD_OK:
        raise LdError(st, lib().ld_last_error().decode(errors="replace"))


def options(**kw) -> Options:
    o = Options()
    lib().ld_options_init(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _as_i64(a) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(a, dtype=np.int64))
    if a.ndim != 2:
        raise ValueError("matrix must be 2-D")
    return a


@dataclass
class Solution:
    value: int
    gray_index: int
    labels: np.ndarray          # labels of reduced rows 0..R-2 (second->strategy)
    labelings: int
    kernel_ms: float
    kernel_kind: int
    lane_bits: int
    h2d_bytes: int = 0
    d2h_bytes: int = 0
    evaluated: int = 0          # labelings the kernels computed a value for


def _solution(res: Result, labels: np.ndarray) -> Solution:
    return Solution(int(res.value), int(res.gray_index), labels, int(res.labelings),
                    float(res.kernel_ms), int(res.kernel_kind), int(res.lane_bits),
                    int(res.h2d_bytes), int(res.d2h_bytes), int(res.evaluated))


def solve_reduced(a, d: int, marginal: bool = False, opts: Options | None = None) -> Solution:
    """calc_Lnorm on an already reduced matrix (last row fixed / marginal row)."""
    a = _as_i64(a)
    r, c = a.shape
    labels = np.zeros(max(r - 1, 1), dtype=np.int32)
    res = Result()
    _check(lib().ld_solve_reduced(a.ctypes.data_as(_I64P), r, c, d, int(marginal),
                                  C.byref(opts) if opts is not None else None, C.byref(res),
                                  labels.ctypes.data_as(_I32P)))
    return _solution(res, labels[: max(r - 1, 0)])


def solve_reduced_noalloc(a, d: int, marginal: bool = False, device: int = 0, stream: int = 0) -> Solution:
    """ld_solve_reduced without any device allocation (its working memory is a
    fixed 64 KiB device array inside the library); for callers that must not
    allocate GPU memory.  d <= 3, <= 64 columns (128 with 8-bit sums)."""
    a = _as_i64(a)
    r, c = a.shape
    labels = np.zeros(max(r - 1, 1), dtype=np.int32)
    res = Result()
    _check(lib().ld_solve_reduced_noalloc(a.ctypes.data_as(_I64P), r, c, d, int(marginal), device,
                                          C.c_void_p(stream or None), C.byref(res),
                                          labels.ctypes.data_as(_I32P)))
    return _solution(res, labels[: max(r - 1, 0)])


def solve_resumable(a, d: int, marginal: bool = False, pieces: int = 16, checkpoint: str = "",
                    max_pieces: int = 0, opts: Options | None = None):
    """Exhaustive solve in `pieces` shards run one after another, with a
    checkpoint file written after each; a later call with the same matrix
    and split continues where the file says.  At most `max_pieces` pieces
    run per call (0: all).  Returns (done, Solution): once done, the
    Solution equals solve_reduced's; before that it holds the best so far."""
    a = _as_i64(a)
    r, c = a.shape
    labels = np.zeros(max(r - 1, 1), dtype=np.int32)
    res, done = Result(), C.c_int32()
    _check(lib().ld_solve_resumable(a.ctypes.data_as(_I64P), r, c, d, int(marginal),
                                    C.byref(opts) if opts is not None else None, pieces, str(checkpoint).encode(),
                                    max_pieces, C.byref(done), C.byref(res), labels.ctypes.data_as(_I32P)))
    return bool(done.value), _solution(res, labels[: max(r - 1, 0)])


def local_search(a, d: int, marginal: bool = False, starts=None, n_random: int = 64, seed: int = 0,
                 max_rounds: int = 0, device: int = 0):
    """Steepest-ascent single-row moves from each start (random starts when
    `starts` is None).  Returns (values[n], labels[n, R-1])."""
    a = _as_i64(a)
    r, c = a.shape
    labs_per = 2 if d == 1 else d
    if starts is None:
        starts = np.random.default_rng(seed).integers(0, labs_per, size=(n_random, r - 1))
    starts = np.ascontiguousarray(np.asarray(starts, dtype=np.int32).reshape(-1, r - 1))
    n = starts.shape[0]
    values = np.zeros(n, dtype=np.int64)
    labels = np.zeros((n, r - 1), dtype=np.int32)
    _check(lib().ld_local_search(a.ctypes.data_as(_I64P), r, c, d, int(marginal),
                                 starts.ctypes.data_as(_I32P), n, max_rounds, device,
                                 values.ctypes.data_as(_I64P), labels.ctypes.data_as(_I32P)))
    return values, labels


def solve_pruned(a, d: int, marginal: bool = False, incumbent=None, opts: Options | None = None):
    """Exact solve that skips labeling blocks whose integer upper bound is
    below the incumbent's value (a labeling of rows 0..R-2).  Returns
    (Solution, stats dict); the Solution equals solve_reduced's."""
    a = _as_i64(a)
    r, c = a.shape
    labels = np.zeros(max(r - 1, 1), dtype=np.int32)
    inc = None
    if incumbent is not None:
        inc = np.ascontiguousarray(np.asarray(incumbent, dtype=np.int32).reshape(-1))
    res, st = Result(), PruneStats()
    _check(lib().ld_solve_pruned(a.ctypes.data_as(_I64P), r, c, d, int(marginal),
                                 C.byref(opts) if opts is not None else None,
                                 inc.ctypes.data_as(_I32P) if inc is not None else None, C.byref(res),
                                 labels.ctypes.data_as(_I32P), C.byref(st)))
    return _solution(res, labels[: max(r - 1, 0)]), {f: getattr(st, f) for f, _ in PruneStats._fields_}


def gray_labels(index: int, rows: int, d: int) -> np.ndarray:
    out = np.zeros(max(rows - 1, 1), dtype=np.int32)
    _check(lib().ld_gray_labels(index, rows, d, out.ctypes.data_as(_I32P)))
    return out[: max(rows - 1, 0)]


def symmetry_walk_ok(d: int, prefix_digits: int, w: int) -> bool:
    """Whether walk number w (its top `prefix_digits` base-d digits) can hold
    the smallest Gray index of a label-permutation class (d >= 3)."""
    return bool(lib().ld_symmetry_walk_ok(d, prefix_digits, w))


def symmetry_walks(d: int, prefix_digits: int, lo: int, hi: int) -> int:
    """Walk numbers in [lo, hi) that pass symmetry_walk_ok."""
    n = C.c_uint64()
    _check(lib().ld_symmetry_walks(d, prefix_digits, lo, hi, C.byref(n)))
    return int(n.value)


def symmetry_walk_at(d: int, prefix_digits: int, rank: int) -> int:
    """The passing walk number of the given rank (increasing order)."""
    w = C.c_uint64()
    _check(lib().ld_symmetry_walk_at(d, prefix_digits, rank, C.byref(w)))
    return int(w.value)


def spectral_basis(a, k: int = 3) -> np.ndarray:
    """The k leading eigenvectors of A^T A (cols x k, float64), each with
    its largest-magnitude component positive (ld_spectral_basis)."""
    a = _as_i64(a)
    r, c = a.shape
    out = np.zeros((c, k), dtype=np.float64)
    _check(lib().ld_spectral_basis(a.ctypes.data_as(_I64P), r, c, k,
                                   out.ctypes.data_as(C.POINTER(C.c_double)), None))
    return out


def strategy_value(text: str, d: int, stat: str = "n", marginal: bool = False, strategy=()) -> int:
    """The value, on the matrix text as read, of the labeling a strategy
    file records (one entry per input row, or per column when the d = 1
    problem is transposed; +1/-1 for d = 1, 0..d-1 otherwise)."""
    raw = text.encode()
    lab = np.ascontiguousarray(np.asarray(list(strategy), dtype=np.int32).reshape(-1))
    buf = lab if lab.size else np.zeros(1, dtype=np.int32)
    v = C.c_int64()
    _check(lib().ld_strategy_value(raw, len(raw), d, (stat or "n")[0].encode(), int(marginal),
                                   buf.ctypes.data_as(_I32P), int(lab.size), C.byref(v)))
    return int(v.value)


def int32_peak(device: int = 0):
    """(sustained int32 ALU ops/s, fastest launch ms) of the device."""
    ops, ms = C.c_double(), C.c_double()
    _check(lib().ld_measure_int32_peak(device, C.byref(ops), C.byref(ms)))
    return float(ops.value), float(ms.value)


class Problem:
    """Read + preprocess (matrix_read and load_parameters of the reference)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def from_text(cls, text: str | bytes, d: int, stat: str = "n", marginal: bool = False):
        raw = text.encode() if isinstance(text, str) else text
        h = C.c_void_p()
        _check(lib().ld_problem_from_text(raw, len(raw), d, (stat or "n")[0].encode(), int(marginal),
                                          C.byref(h)))
        return cls(h)

    @classmethod
    def from_file(cls, path, d: int, stat: str = "n", marginal: bool = False):
        h = C.c_void_p()
        _check(lib().ld_problem_from_file(str(path).encode(), d, (stat or "n")[0].encode(),
                                          int(marginal), C.byref(h)))
        return cls(h)

    @classmethod
    def from_matrix(cls, a, d: int, stat: str = "n", marginal: bool = False):
        a = _as_i64(a)
        h = C.c_void_p()
        _check(lib().ld_problem_from_matrix(a.ctypes.data_as(_I64P), a.shape[0], a.shape[1], d,
                                            (stat or "n")[0].encode(), int(marginal), C.byref(h)))
        return cls(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.ld_problem_destroy(h)
            self._h = None

    @property
    def info(self) -> dict:
        inf = ProblemInfo()
        _check(lib().ld_problem_get_info(self._h, C.byref(inf)))
        return {f: getattr(inf, f) for f, _ in ProblemInfo._fields_}

    @property
    def reduced(self) -> np.ndarray:
        inf = self.info
        out = np.zeros(max(inf["rows"] * inf["cols"], 1), dtype=np.int64)
        _check(lib().ld_problem_reduced(self._h, out.ctypes.data_as(_I64P), out.size))
        return out[: inf["rows"] * inf["cols"]].reshape(inf["rows"], inf["cols"])

    @property
    def log(self) -> str:
        return lib().ld_problem_log(self._h).decode()

    def check_launch(self, blocks: int = 512, threads: int = 32) -> None:
        _check(lib().ld_problem_check_launch(self._h, blocks, threads))

    def solve(self, opts: Options | None = None) -> Result:
        res = Result()
        _check(lib().ld_problem_solve(self._h, C.byref(opts) if opts is not None else None,
                                      C.byref(res)))
        return res

    def report(self, res: Result):
        """(value line appended to the log, strategy file name, strategy file text)."""
        n = max(self.info["rows_in"], self.info["cols_in"])
        strat = np.zeros(max(n, 1), dtype=np.int32)
        cnt = C.c_int32()
        name = C.create_string_buffer(64)
        _check(lib().ld_problem_report(self._h, C.byref(res), strat.ctypes.data_as(_I32P), strat.size,
                                       C.byref(cnt), name, len(name)))
        text = "".join(f"{int(v)}\n" for v in strat[: cnt.value])
        return name.value.decode(), text


def _is_path(source) -> bool:
    if isinstance(source, os.PathLike):
        return True
    if isinstance(source, str) and "\n" not in source:
        try:
            return Path(source).is_file()
        except OSError:
            return False
    return False


def lnorm(source, d: int, stat: str = "n", marginal: bool = False, blocks: int = 512,
          threads: int = 32, opts: Options | None = None):
    """Whole pipeline (like ./L_CUDA): returns (value, stdout_text, strategy_name, strategy_text)."""
    if _is_path(source):
        p = Problem.from_file(source, d, stat, marginal)
    elif isinstance(source, (str, bytes)):
        p = Problem.from_text(source, d, stat, marginal)
    else:
        p = Problem.from_matrix(source, d, stat, marginal)
    p.check_launch(blocks, threads)
    if p.info["rows"] == 0:
        res = Result()
        zero = True
    else:
        res = p.solve(opts)
        zero = False
    name, text = p.report(res)
    out = p.log
    if zero:  # main() prints this line itself, before the value (L_CUDA.cu:432)
        lines = out.splitlines(keepends=True)
        out = "".join(lines[:-1]) + "This is a zero matrix.\n" + lines[-1]
    return int(res.value), out, name, text


class Plan:
    """A device-resident reduced matrix for repeated solves."""

    def __init__(self, a, d: int, marginal: bool = False, opts: Options | None = None):
        a = _as_i64(a)
        self.rows, self.cols = a.shape
        self.d = d
        h = C.c_void_p()
        _check(lib().ld_plan_create(a.ctypes.data_as(_I64P), a.shape[0], a.shape[1], d, int(marginal),
                                    C.byref(opts) if opts is not None else None, C.byref(h)))
        self._h = h

    def launch(self) -> None:
        _check(lib().ld_plan_launch(self._h))

    def result(self) -> Solution:
        res = Result()
        labels = np.zeros(max(self.rows - 1, 1), dtype=np.int32)
        _check(lib().ld_plan_result(self._h, C.byref(res), labels.ctypes.data_as(_I32P)))
        return _solution(res, labels[: max(self.rows - 1, 0)])

    def solve(self) -> Solution:
        self.launch()
        return self.result()

    @property
    def range(self):
        lo, hi = C.c_uint64(), C.c_uint64()
        _check(lib().ld_plan_range(self._h, C.byref(lo), C.byref(hi)))
        return int(lo.value), int(hi.value)

    @property
    def stream(self) -> int:
        return int(lib().ld_plan_stream(self._h) or 0)

    @property
    def result_device_ptr(self) -> int:
        """Device address of the 16-byte {value, index} result of the last launch."""
        return int(lib().ld_plan_result_device(self._h) or 0)

    def describe(self) -> str:
        buf = C.create_string_buffer(256)
        _check(lib().ld_plan_describe(self._h, buf, len(buf)))
        return buf.value.decode()

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().ld_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.ld_plan_destroy(self._h)
            self._h = None


class Batch:
    """Many reduced matrices solved together: per lane class a persistent
    kernel over a device work queue, all captured in one CUDA graph."""

    def __init__(self, mats, ds, margs=None, opts: Options | None = None, autotune: bool = True):
        self._mats = [_as_i64(m) for m in mats]
        n = len(self._mats)
        self.n = n
        ptrs = (_I64P * n)(*[m.ctypes.data_as(_I64P) for m in self._mats])
        rows = np.array([m.shape[0] for m in self._mats], dtype=np.int32)
        cols = np.array([m.shape[1] for m in self._mats], dtype=np.int32)
        dd = np.ascontiguousarray(np.asarray(ds, dtype=np.int32).reshape(n))
        mm = np.ascontiguousarray(np.zeros(n, dtype=np.int32) if margs is None
                                  else np.asarray(margs, dtype=np.int32).reshape(n))
        h = C.c_void_p()
        _check(lib().ld_batch_create(n, ptrs, rows.ctypes.data_as(_I32P), cols.ctypes.data_as(_I32P),
                                     dd.ctypes.data_as(_I32P), mm.ctypes.data_as(_I32P),
                                     C.byref(opts) if opts is not None else None, int(autotune), C.byref(h)))
        self._h = h

    def launch(self) -> None:
        _check(lib().ld_batch_launch(self._h))

    def results(self):
        """(values int64[n], gray indices uint64[n], device ms of the launch)."""
        v = np.zeros(self.n, dtype=np.int64)
        g = np.zeros(self.n, dtype=np.uint64)
        ms = C.c_float()
        _check(lib().ld_batch_results(self._h, v.ctypes.data_as(_I64P), g.ctypes.data_as(C.POINTER(C.c_uint64)),
                                      C.byref(ms)))
        return v, g, float(ms.value)

    def solve(self):
        self.launch()
        return self.results()

    def describe(self) -> str:
        buf = C.create_string_buffer(4096)
        _check(lib().ld_batch_describe(self._h, buf, len(buf)))
        return buf.value.decode()

    def evaluated(self) -> np.ndarray:
        """Labelings the kernels compute a value for, per matrix (uint64[n])."""
        e = np.zeros(self.n, dtype=np.uint64)
        _check(lib().ld_batch_evaluated(self._h, e.ctypes.data_as(C.POINTER(C.c_uint64))))
        return e

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().ld_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.ld_batch_destroy(self._h)
            self._h = None


# ---------------------------------------------------------------------------
# proposal network (tensor-core MLP 44 -> 256 -> 256 -> 44)

MLP_IN = 44
MLP_HIDDEN = 256
MLP_OUT = 44
MLP_SHAPES = [("W1", (MLP_HIDDEN, MLP_IN)), ("b1", (MLP_HIDDEN,)), ("W2", (MLP_HIDDEN, MLP_HIDDEN)),
              ("b2", (MLP_HIDDEN,)), ("W3", (MLP_OUT, MLP_HIDDEN)), ("b3", (MLP_OUT,))]


def _f32(a, shape=None) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    if shape is not None and a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


def unflatten_params(flat: np.ndarray) -> dict:
    out, off = {}, 0
    for name, shape in MLP_SHAPES:
        n = int(np.prod(shape))
        out[name] = flat[off:off + n].reshape(shape)
        off += n
    return out


def flatten_params(p: dict) -> np.ndarray:
    return np.concatenate([np.asarray(p[name], dtype=np.float32).reshape(-1) for name, _ in MLP_SHAPES])


class Mlp:
    """The proposal network on one GPU: forward, gradients and Adam steps run
    on the library's tensor-core kernels (bf16 operands, fp32 accumulate)."""

    def __init__(self, batch: int = 1024, seed: int = 0, device: int = 0, skip: float = 0.0):
        h = C.c_void_p()
        _check(lib().ld_mlp_create(int(batch), int(seed), float(skip), int(device), C.byref(h)))
        self._h = h
        self.batch = int(batch)
        self.skip = float(skip)

    @staticmethod
    def param_count() -> int:
        return int(lib().ld_mlp_param_count())

    def get_params(self) -> dict:
        flat = np.zeros(self.param_count(), dtype=np.float32)
        _check(lib().ld_mlp_get_params(self._h, flat.ctypes.data_as(_F32P)))
        return unflatten_params(flat)

    def set_params(self, params: dict) -> None:
        flat = _f32(flatten_params(params))
        _check(lib().ld_mlp_set_params(self._h, flat.ctypes.data_as(_F32P)))

    def forward(self, x) -> np.ndarray:
        x = _f32(x)
        rows = x.shape[0]
        out = np.zeros((rows, MLP_OUT), dtype=np.float32)
        _check(lib().ld_mlp_forward(self._h, x.ctypes.data_as(_F32P), rows, out.ctypes.data_as(_F32P)))
        return out

    def gradients(self, x, t, mask):
        x, t, mask = _f32(x), _f32(t), _f32(mask)
        flat = np.zeros(self.param_count(), dtype=np.float32)
        loss = C.c_float()
        _check(lib().ld_mlp_gradients(self._h, x.ctypes.data_as(_F32P), t.ctypes.data_as(_F32P),
                                      mask.ctypes.data_as(_F32P), x.shape[0], flat.ctypes.data_as(_F32P),
                                      C.byref(loss)))
        return unflatten_params(flat), float(loss.value)

    def train_step(self, x, t, mask, lr: float = 1e-3) -> float:
        x, t, mask = _f32(x), _f32(t), _f32(mask)
        loss = C.c_float()
        _check(lib().ld_mlp_train_step(self._h, x.ctypes.data_as(_F32P), t.ctypes.data_as(_F32P),
                                       mask.ctypes.data_as(_F32P), x.shape[0], float(lr), C.byref(loss)))
        return float(loss.value)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().ld_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.ld_mlp_destroy(self._h)
            self._h = None


def tc_gemm(a_bits: np.ndarray, b_bits: np.ndarray, device: int = 0) -> np.ndarray:
    """C = A B^T on the tensor cores; A, B are bf16 bit patterns (uint16)."""
    a = np.ascontiguousarray(a_bits, dtype=np.uint16)
    b = np.ascontiguousarray(b_bits, dtype=np.uint16)
    M, K = a.shape
    N = b.shape[0]
    if b.shape[1] != K:
        raise ValueError("inner dimensions differ")
    c = np.zeros((M, N), dtype=np.float32)
    _check(lib().ld_tc_gemm(a.ctypes.data_as(C.POINTER(C.c_uint16)), b.ctypes.data_as(C.POINTER(C.c_uint16)),
                            M, N, K, c.ctypes.data_as(_F32P), int(device)))
    return c
