"""The oracle (CPU restatement) against the reference's own outputs and
against an independent pure-Python brute force on tiny cases."""
import itertools

import numpy as np
import pytest

import oracle_ffi as O
from helpers import GOLDEN, split_tail, without_launch_line as lines_without_launch


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_oracle_matches_reference(case):
    d, stat, marg = split_tail(case["tail"])
    rc, out, name, strat, _ = O.run_cli(case["text"], d, stat, marg)
    assert rc == 0
    assert lines_without_launch(out) == lines_without_launch(case["stdout"])
    assert name == case["strategy_name"]
    assert strat == case["strategy"]


def brute(a, d, marginal):
    """Independent brute force: every labeling, last row fixed."""
    r, c = a.shape
    dd = 2 if d <= 2 else d
    best = None
    for labs in itertools.product(range(dd), repeat=r - 1):
        if d == 1:
            s = np.array([2 * x - 1 for x in labs] + [1])
            col = s @ a
            v = int(col[0] + np.abs(col[1:]).sum()) if marginal else int(np.abs(col).sum())
        else:
            v = 0
            for m in range(dd):
                sel = np.array([x == m for x in labs] + [m == 0])
                v += int(np.abs(a[sel].sum(axis=0)).sum())
        if best is None or v > best:
            best = v
    return best


@pytest.mark.parametrize("seed", range(40))
def test_oracle_vs_python_bruteforce(seed):
    rng = np.random.default_rng(seed)
    d = int(rng.choice([1, 1, 2, 3, 4, 5]))
    r = int(rng.integers(1, {1: 9, 2: 9, 3: 7, 4: 6, 5: 5}[d] + 1))
    c = int(rng.integers(1, 8))
    a = rng.integers(-6, 7, size=(r, c)).astype(np.int64)
    marg = d == 1 and seed % 3 == 0
    v, n = O.enumerate_max(a, d, marg, nthreads=int(rng.integers(1, 5)))
    assert v == brute(a, d, marg)
    assert O.value(a, d, marg, O.labels(n, r, d)) == v


def test_known_answers():
    assert O.run_cli("1 1\n1 -1\n", 1)[4] == 2          # CHSH local bound
    assert O.run_cli("1 2 3\n-1 0 2\n4 4 -4\n", 5)[4] == 21


def test_tie_break_is_smallest_gray_index():
    rng = np.random.default_rng(7)
    a = rng.integers(-2, 3, size=(9, 4)).astype(np.int64)
    for d in (1, 2, 3):
        v, n = O.enumerate_max(a, d, False, nthreads=1)
        total = O.total(9, d)
        first = next(k for k in range(total)
                     if O.value(a, d, False, O.labels(k, 9, d)) == v)
        assert n == first
        # independent of the worker count
        assert O.enumerate_max(a, d, False, nthreads=7) == (v, n)


def test_int64_range_exact():
    """Entries whose column sums overflow int32 are exact in int64."""
    a = np.array([[2_000_000_000, -1_500_000_000], [1_900_000_000, 7], [-3, 2_100_000_000]],
                 dtype=np.int64)
    v, _ = O.enumerate_max(a, 1, False, nthreads=1)
    assert v == brute(a, 1, False)
    assert v > 2**31
