"""The column-split table kernel (split_kernel.cuh): matrices too wide for one
thread's register vectors, where S lanes share each high index and hold a
slice of the columns each.  Bit-exact against the oracle (value and smallest
Gray index) at 65, 100, 200 and 256 columns for L_1, LM, d = 2, 3, 4 in
32-bit and 8-bit lanes; every group size forced on the same matrices; label
symmetry, shards and ties; and the wide kernel (column_split = -1) agrees."""
import numpy as np
import pytest

import oracle_ffi as O

pytestmark = pytest.mark.gpu

# rows per d: few enough that the oracle enumerates in well under a second
ROWS = {1: 15, 2: 14, 3: 9, 4: 8}


def _matrix(rng, d, cols, narrow):
    r = ROWS[d]
    amp = 3 if narrow else 400
    if narrow and d >= 2:
        amp = 1            # d >= 2 needs the full column sum within 8 bits
    return rng.integers(-amp, amp + 1, size=(r, cols)).astype(np.int64)


def _split_of(ld, a, d, marg, **kw):
    plan = ld.Plan(a, d, marg, ld.options(**kw))
    desc = plan.describe()
    sol = plan.solve()
    plan.close()
    return sol, desc


@pytest.mark.parametrize("cols", [65, 100, 200, 256])
@pytest.mark.parametrize("kind", ["L1", "LM", "d2", "d3", "d4"])
@pytest.mark.parametrize("narrow", [False, True], ids=["int32", "int8"])
def test_wide_matrices_match_the_oracle(ld, kind, cols, narrow):
    d = {"L1": 1, "LM": 1, "d2": 2, "d3": 3, "d4": 4}[kind]
    marg = kind == "LM"
    rng = np.random.default_rng(cols * 7 + d + 100 * marg + 1000 * narrow)
    a = _matrix(rng, d, cols, narrow)
    if marg:
        a[-1, :] = rng.integers(-3, 4, size=cols)       # the marginal row
        a[:, 0] = rng.integers(-3, 4, size=a.shape[0])  # the marginal column
    sol, desc = _split_of(ld, a, d, marg)
    # the unsplit kernel holds up to 64 int32 / 32 8-bit words per vector
    # for d <= 3, 16 / 8 for d >= 4
    words = (cols + 3) // 4 if narrow else cols
    limit = (32 if narrow else 64) if d <= 3 else (8 if narrow else 16)
    assert sol.kernel_kind == ld.KERNEL_TABLE, desc
    assert (" split=0" not in desc) == (words > limit), desc
    assert (sol.value, sol.gray_index) == O.enumerate_max(a, d, marg), desc
    assert sol.lane_bits == (8 if narrow else 32), desc


@pytest.mark.parametrize("S", [2, 4, 8])
@pytest.mark.parametrize("d", [1, 2, 3, 4, 6, 10])
def test_every_group_size_on_the_same_matrix(ld, S, d):
    """Forced group sizes, including matrices the unsplit kernel also takes."""
    rng = np.random.default_rng(10 * S + d)
    rows = {1: 14, 2: 13, 3: 9, 4: 8, 6: 7, 10: 6}[d]
    cols = {1: 40, 2: 30, 3: 24, 4: 20, 6: 12, 10: 8}[d]
    a = rng.integers(-50, 51, size=(rows, cols)).astype(np.int64)
    ref = O.enumerate_max(a, d, False)
    sol, desc = _split_of(ld, a, d, False, column_split=S)
    assert f" split={S}" in desc, desc
    assert (sol.value, sol.gray_index) == ref, desc


@pytest.mark.parametrize("d", [3, 4, 5])
def test_label_symmetry_and_every_walk(ld, d):
    rng = np.random.default_rng(70 + d)
    a = rng.integers(-30, 31, size=({3: 10, 4: 8, 5: 7}[d], 120)).astype(np.int64)
    ref = O.enumerate_max(a, d, False)
    sym, desc = _split_of(ld, a, d, False, column_split=8)
    full, _ = _split_of(ld, a, d, False, column_split=8, enumerate_all=1)
    assert (sym.value, sym.gray_index) == ref == (full.value, full.gray_index), desc
    assert sym.evaluated < full.evaluated == full.labelings


@pytest.mark.parametrize("d", [1, 3])
def test_shards_combine_to_the_oracle(ld, d):
    rng = np.random.default_rng(5 + d)
    a = rng.integers(-200, 201, size=({1: 16, 3: 10}[d], 150)).astype(np.int64)
    ref = O.enumerate_max(a, d, False)
    best = None
    for i in range(3):
        sol, desc = _split_of(ld, a, d, False, shard_index=i, shard_count=3)
        assert " split=0" not in desc
        cand = (sol.value, -sol.gray_index)
        best = cand if best is None or cand > best else best
    assert (best[0], -best[1]) == ref


def test_ties_keep_the_smallest_index(ld):
    a = np.ones((13, 130), dtype=np.int64)
    a[1::2] *= -1
    a[:, 64:] *= 2
    for d in (1, 2, 3):
        rr = a[: {1: 13, 2: 12, 3: 8}[d]]
        sol, desc = _split_of(ld, rr, d, False)
        assert " split=0" not in desc
        assert (sol.value, sol.gray_index) == O.enumerate_max(rr, d, False), (d, desc)


def test_wide_kernel_agrees(ld):
    rng = np.random.default_rng(9)
    for d, rows in ((1, 14), (2, 12), (3, 8)):
        a = rng.integers(-99, 100, size=(rows, 180)).astype(np.int64)
        split, desc = _split_of(ld, a, d, False)
        wide, wdesc = _split_of(ld, a, d, False, column_split=-1)
        assert " split=0" not in desc and wdesc.startswith("wide")
        assert (split.value, split.gray_index) == (wide.value, wide.gray_index)


@pytest.mark.parametrize("d", [1, 2, 3])
@pytest.mark.parametrize("blocks", [1, 2, 3])
def test_paired_walks_match_single_walks_and_oracle(ld, d, blocks):
    """Two high indices per thread against each table read (d = 1, 2, 3),
    forced onto small matrices by a small grid; an odd walk count leaves one
    thread a lone walk, which it runs twice."""
    rng = np.random.default_rng(40 * d + blocks)
    rows = {1: 17, 2: 16, 3: 11}[d]
    for amp, cols in ((1, 30), (60, 8)):         # 8-bit and 32-bit lanes (paired: <= 8 words)
        a = rng.integers(-amp, amp + 1, size=(rows, cols)).astype(np.int64)
        ref = O.enumerate_max(a, d, False)
        # few low rows: thousands of walks, so even one block has two per thread
        pair, desc = _split_of(ld, a, d, False, blocks=blocks, low_rows=3)
        one, desc1 = _split_of(ld, a, d, False, blocks=blocks, low_rows=3, paired_walks=-1)
        assert " pair=1" in desc and " pair=0" in desc1, (desc, desc1)
        assert (pair.value, pair.gray_index) == ref == (one.value, one.gray_index), desc
        assert pair.evaluated == one.evaluated


def test_paired_walks_with_label_symmetry_and_shards(ld):
    rng = np.random.default_rng(77)
    a = rng.integers(-9, 10, size=(12, 24)).astype(np.int64)
    ref = O.enumerate_max(a, 3, False)
    best = None
    for i in range(2):
        sol, desc = _split_of(ld, a, 3, False, blocks=2, low_rows=2, shard_index=i, shard_count=2)
        assert " pair=1" in desc and " sym=0" not in desc, desc
        cand = (sol.value, -sol.gray_index)
        best = cand if best is None or cand > best else best
    assert (best[0], -best[1]) == ref


@pytest.mark.parametrize("d,marg", [(1, False), (1, True), (2, False), (3, False), (5, False)])
def test_packed_maxima_at_the_16_bit_bound(ld, d, marg):
    """Two running maxima per word (p16=1) whenever sum |A| + 2K < 65536:
    totals just below the bound use it, just above do not, and both give the
    oracle's answer; pack16 = -1 turns it off."""
    rows = {1: 14, 2: 12, 3: 9, 5: 7}[d]
    for total, want in ((65000, 1), (66500, 0)):
        rng = np.random.default_rng(total + d)
        a = rng.integers(1, 100, size=(rows, 12)).astype(np.int64) * rng.choice([-1, 1], size=(rows, 12))
        if marg:
            a[:, 0] = rng.integers(-3, 4, size=rows)
        # scale column 1 so that sum |A| (+ 2K) lands on the target
        k = int(np.abs(a[:, 0]).sum()) if marg else 0
        rest = int(np.abs(a).sum() - np.abs(a[:, 1]).sum()) + 2 * k
        a[:, 1] = np.sign(a[:, 1]) * ((total - rest) // rows)
        a[0, 1] += np.sign(a[0, 1]) * ((total - rest) % rows)
        assert int(np.abs(a).sum()) + 2 * k == total
        ref = O.enumerate_max(a, d, marg)
        sol, desc = _split_of(ld, a, d, marg)
        off, desc_off = _split_of(ld, a, d, marg, pack16=-1)
        assert f" p16={want}" in desc and " p16=0" in desc_off, (desc, desc_off)
        assert (sol.value, sol.gray_index) == ref == (off.value, off.gray_index), desc


@pytest.mark.parametrize("d", [1, 2, 3, 4])
def test_fetched_walks_match_the_static_split_on_every_launch(ld, d):
    """Warps fetching walks from a counter (the default) against the fixed
    split (walk_fetch = -1): the same answer as the oracle, launch after
    launch of one plan (the last block resets the counter), with ties."""
    rng = np.random.default_rng(90 + d)
    rows = {1: 18, 2: 17, 3: 11, 4: 9}[d]
    a = rng.integers(-2, 3, size=(rows, 9)).astype(np.int64)
    a[1] = a[0]                               # equal rows: many tied labelings
    ref = O.enumerate_max(a, d, False)
    for kw in ({}, {"blocks": 3, "low_rows": 3}):
        plan = ld.Plan(a, d, False, ld.options(**kw))
        assert " fetch=1" in plan.describe()
        for _ in range(3):
            sol = plan.solve()
            assert (sol.value, sol.gray_index) == ref
        plan.close()
        stat, desc = _split_of(ld, a, d, False, walk_fetch=-1, **kw)
        assert " fetch=0" in desc and (stat.value, stat.gray_index) == ref
