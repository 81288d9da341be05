"""Generate the golden fixtures (tests/golden/cases.json) by running the
reference's own OpenMP solver, oracle/_ref/L_OpenMP, built from the
reference sources by oracle/Makefile.

Each case stores the matrix file's text, the CLI tail (d, flag, m), the
reference's stdout and its strategy file.  The reference has no tests or
fixtures of its own, so these outputs are what pins the oracle and the
product.  Run from the repository root:

    make -C oracle REF_DIR=<reference checkout> && python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "l-norms_bruteforce_b200"))
import workloads as W  # noqa: E402

REF = ROOT / "oracle" / "_ref" / "L_OpenMP"
OUT = Path(__file__).resolve().parent / "cases.json"


def run_ref(text: str, tail: list[str], nthreads: int = 8, timeout: int = 600) -> dict:
    with tempfile.TemporaryDirectory() as td:
        (Path(td) / "m.txt").write_text(text)
        p = subprocess.run([str(REF), str(nthreads), "m.txt", *tail], cwd=td, capture_output=True,
                           text=True, timeout=timeout)
        files = sorted(Path(td).glob("strategy_*.txt"))
        strat_name = files[0].name if files else ""
        strat = files[0].read_text() if files else ""
    return dict(rc=p.returncode, stdout=p.stdout, strategy_name=strat_name, strategy=strat)


def work(a: np.ndarray, d: int) -> int:
    r = a.shape[0]
    return 2 ** (r - 1) if d <= 2 else d ** (r - 1)


def planted(rng: np.random.Generator, r: int, c: int, lo: int, hi: int) -> np.ndarray:
    """A random matrix with planted parallel / anti-parallel / zero lines and
    single-signed columns, so every preprocessing rule fires."""
    a = rng.integers(lo, hi + 1, size=(r, c), dtype=np.int64)
    k = rng.integers(0, 6)
    for _ in range(k):
        kind = rng.integers(0, 7)
        i, j = rng.integers(0, r), rng.integers(0, r)
        p, q = rng.integers(0, c), rng.integers(0, c)
        mult = int(rng.choice([1, 2, 3, -1, -2]))
        if kind == 0 and i != j:
            a[j] = mult * a[i]
        elif kind == 1 and p != q:
            a[:, q] = mult * a[:, p]
        elif kind == 2:
            a[i] = 0
        elif kind == 3:
            a[:, p] = 0
        elif kind == 4:
            a[:, p] = np.abs(a[:, p])
        elif kind == 5:
            a[:, p] = -np.abs(a[:, p])
        elif kind == 6 and i != j:
            a[j] = a[i]
    return a


def main() -> None:
    if not REF.exists():
        sys.exit("build the reference first: make -C oracle REF_DIR=<reference checkout>")
    rng = np.random.default_rng(20261203)
    cases = []

    def add(name, text, tail, nthreads=8):
        r = run_ref(text, tail, nthreads)
        cases.append(dict(name=name, text=text, tail=tail, nthreads=nthreads, **r))

    # known answers
    add("chsh", "1 1\n1 -1\n", ["1"])
    add("reset_d5_3x3", "1 2 3\n-1 0 2\n4 4 -4\n", ["5"])

    flags = ["n", "y", "r", "c", "Y", "R", "C", "x"]
    # random small matrices over every d and flag
    for t in range(260):
        d = int(rng.choice([1, 1, 1, 2, 2, 3, 3, 4, 5, 6, 7, 8, 9, 10]))
        maxr = {1: 14, 2: 14, 3: 10, 4: 8, 5: 7, 6: 6, 7: 6, 8: 5, 9: 5, 10: 5}[d]
        r = int(rng.integers(1, maxr + 1))
        c = int(rng.integers(1, 13))
        lo, hi = (-4, 4) if t % 3 else (-60, 60)
        a = planted(rng, r, c, lo, hi) if t % 2 else rng.integers(lo, hi + 1, size=(r, c))
        if work(a, d) > (1 << 21):
            continue
        f = flags[t % len(flags)]
        tail = [str(d)]
        marg = d == 1 and rng.random() < 0.4
        if f != "n":
            tail.append(f)
        if marg:
            tail.append("m" if rng.random() < 0.8 else "M")
        add(f"rand{t}_d{d}_{r}x{c}_{f}{'_m' if marg else ''}", W.matrix_text(a), tail,
            nthreads=int(rng.choice([1, 3, 8])))

    # marginal edge cases: zero first row / column, both zero, transposed LM
    base = rng.integers(-3, 4, size=(7, 9))
    for nm, mod in [("row0zero", lambda a: a.__setitem__((0, slice(None)), 0)),
                    ("col0zero", lambda a: a.__setitem__((slice(None), 0), 0)),
                    ("both0", lambda a: (a.__setitem__((0, slice(None)), 0),
                                         a.__setitem__((slice(None), 0), 0)))]:
        a = base.copy(); mod(a)
        for f in ["y", "r", "c", "n"]:
            tail = ["1", f, "m"] if f != "n" else ["1", "m"]
            add(f"marg_{nm}_{f}", W.matrix_text(a), tail)
    a = rng.integers(-3, 4, size=(12, 5))
    add("marg_transposed", W.matrix_text(a), ["1", "y", "m"])
    add("marg_transposed_noprep", W.matrix_text(a), ["1", "m"])
    # transpose for d == 1 only
    a = rng.integers(-9, 10, size=(15, 6))
    add("transpose_d1", W.matrix_text(a), ["1"])
    add("notranspose_d2", W.matrix_text(a[:10]), ["2"])
    # zero matrices, single row / column
    z = np.zeros((4, 5), dtype=np.int64)
    add("zero_d1_y", W.matrix_text(z), ["1", "y"])
    add("zero_d3_c", W.matrix_text(z), ["3", "c"])
    add("zero_d1_noprep", W.matrix_text(z), ["1"])
    add("single_row_d1", "3 -4 5\n", ["1"])
    add("single_row_d2", "3 -4 5\n", ["2"])
    add("single_col_d1", "3\n-4\n5\n1\n", ["1"])
    add("single_entry_lm", "-5\n", ["1", "m"])
    # parsing: scientific notation, separators, CRLF, blank lines, long rows
    a = rng.integers(-20, 21, size=(6, 6))
    sci = "".join(" ".join(f"{float(v):.8e}" for v in row) + "\n" for row in a)
    add("sci_notation", sci, ["1"])
    add("separators", "1,2;3\t-4\r\n\n  5 6 -7 8\n\n9|10|11|12\r\n", ["2", "y"])
    add("long_first_row", "1 2 3 4 5\n6 7 8\n-1 2 -3\n", ["1"])
    add("decimal_tokens", "1.9 -2.5 3\n4 5.0 -6\n7 8 9.99\n", ["1"])
    # d-reset: d >= reduced rows
    add("reset_d4_rows3", W.matrix_text(rng.integers(-5, 6, size=(3, 4))), ["4"])
    add("reset_d2_rows1", "2 -3 4\n", ["2"])
    add("reset_d3_rows2_y", "1 2\n2 4\n3 -1\n", ["3", "y"])
    # mid-size cases for every kernel family
    add("mid_L1_20x33", W.matrix_text(rng.integers(-30, 31, size=(20, 33))), ["1"])
    add("mid_LM_18x12", W.matrix_text(rng.integers(-7, 8, size=(18, 12))), ["1", "m"])
    add("mid_L2_18x40", W.matrix_text(rng.integers(-9, 10, size=(18, 40))), ["2"])
    add("mid_L3_12x20", W.matrix_text(rng.integers(-9, 10, size=(12, 20))), ["3"])
    add("mid_L4_9x17", W.matrix_text(rng.integers(-9, 10, size=(9, 17))), ["4"])
    add("mid_L7_7x9", W.matrix_text(rng.integers(-9, 10, size=(7, 9))), ["7"])
    add("mid_L10_6x70", W.matrix_text(rng.integers(-9, 10, size=(6, 70))), ["10"])
    add("wide_L1_12x300", W.matrix_text(rng.integers(-50, 51, size=(12, 300))), ["1"])
    add("wide_L2_10x150", W.matrix_text(rng.integers(-50, 51, size=(10, 150))), ["2"])
    add("pm1_L1_22x9", W.matrix_text(rng.choice([-1, 1], size=(22, 9))), ["1"])

    # the benchmark configurations that the reference finishes in seconds
    for inst in (W.config1(), W.config2(), W.config3()):
        add(inst.name, W.matrix_text(inst.matrix), inst.argv_tail())

    OUT.write_text(json.dumps(cases, indent=0))
    print(f"wrote {len(cases)} cases to {OUT}")


if __name__ == "__main__":
    main()
