"""Label symmetry on the GPU (d >= 3).  The table kernel skips the walks
that hold no smallest index of a label-permutation class (the default); its
value and smallest Gray index equal the oracle's and those of the run that
evaluates every walk, over walk lengths, low-row counts, lane widths, tied
and mostly-zero matrices, and shards."""
import numpy as np
import pytest

import oracle_ffi as O

pytestmark = pytest.mark.gpu

ROWS = {3: 11, 4: 9, 5: 8, 6: 7, 7: 7, 8: 6, 9: 6, 10: 6}


def matrices(d, rng):
    r = ROWS[d]
    yield rng.choice([-1, 1], size=(r, 9))                                  # many ties
    yield rng.integers(-3, 4, size=(r, 20))                                 # 8-bit lanes
    a = rng.integers(-40, 41, size=(r + 1, 7))                              # 32-bit lanes
    a[2] = a[0]                                                             # tied rows
    yield a
    yield (rng.random((r, 6)) < 0.3) * rng.integers(1, 3, size=(r, 6))     # mostly zero


@pytest.mark.parametrize("d", [3, 4, 5, 6, 7, 8, 9, 10])
def test_symmetry_matches_oracle(ld, d):
    rng = np.random.default_rng(500 + d)
    for a in matrices(d, rng):
        a = np.ascontiguousarray(a, dtype=np.int64)
        ref = O.enumerate_max(a, d, False)
        for opts in (dict(), dict(tile=1), dict(tile=2), dict(low_rows=0, tile=1), dict(low_rows=1),
                     dict(low_rows=2, tile=0)):
            plan = ld.Plan(a, d, False, ld.options(kernel=1, **opts))
            desc = plan.describe()
            sol = plan.solve()
            plan.close()
            assert (sol.value, sol.gray_index) == ref, (opts, desc)
            assert sol.labelings == O.total(a.shape[0], d)
            if " sym=0 " not in desc:
                assert sol.evaluated < sol.labelings, desc
            full = ld.solve_reduced(a, d, False, ld.options(kernel=1, enumerate_all=1, **opts))
            assert (full.value, full.gray_index) == ref, opts
            assert full.evaluated == full.labelings


def test_symmetry_skips_half_the_walks_at_d3(ld):
    """3^19 labelings (20 rows, +-1 entries): the walks that run are the
    classes' share, about half."""
    rng = np.random.default_rng(77)
    a = rng.choice([-1, 1], size=(20, 30)).astype(np.int64)
    sym = ld.solve_reduced(a, 3, False)
    full = ld.solve_reduced(a, 3, False, ld.options(enumerate_all=1))
    assert (sym.value, sym.gray_index) == (full.value, full.gray_index)
    assert 0.49 < sym.evaluated / sym.labelings < 0.52
    assert sym.kernel_ms < 0.7 * full.kernel_ms


@pytest.mark.parametrize("d,count", [(3, 2), (3, 3), (4, 4), (5, 3)])
def test_symmetric_shards_tile_balance_and_combine(ld, d, count):
    rng = np.random.default_rng(40 * d + count)
    r = {3: 13, 4: 10, 5: 9}[d]
    a = rng.integers(-9, 10, size=(r, 14)).astype(np.int64)
    a[3] = a[1]
    full = O.enumerate_max(a, d, False)
    plan = ld.Plan(a, d, False, ld.options(kernel=1))
    desc = plan.describe()
    whole = plan.solve()
    plan.close()
    geo = dict(kv.split("=") for kv in desc.split() if "=" in kv)
    block = int(geo["B"]) * d ** int(geo["fw"])          # labelings per walk
    assert int(geo["sym"]) > 0, desc
    parts, ranges, work = [], [], []
    for s in range(count):
        plan = ld.Plan(a, d, False, ld.options(kernel=1, shard_index=s, shard_count=count))
        ranges.append(plan.range)
        sol = plan.solve()
        plan.close()
        parts.append((sol.value, -sol.gray_index))
        work.append(sol.evaluated)
    assert ranges[0][0] == 0 and ranges[-1][1] == O.total(r, d)
    assert all(ranges[i][1] == ranges[i + 1][0] for i in range(count - 1))
    best = max(parts)
    assert (best[0], -best[1]) == full
    # the shards split the walks that run evenly (to one walk)
    assert sum(work) == whole.evaluated
    assert max(work) - min(work) <= block, (work, block)


@pytest.mark.parametrize("d", [3, 4, 5, 6, 8, 10])
@pytest.mark.parametrize("lanes", [32, 64])
def test_wide_kernel_symmetry(ld, d, lanes):
    """The column-parallel kernel hands warps the passing walks by rank: value
    and index equal the oracle's and the full run's, for 32- and 64-bit sums,
    on wide and tie-heavy matrices."""
    rng = np.random.default_rng(900 + 10 * d + lanes)
    # 1e6 .. 5e6 labelings: enough that walks by rank beat evaluating every
    # index (the plan's estimate keeps full enumeration for small solves)
    r = {3: 15, 4: 12, 5: 10, 6: 9, 8: 8, 10: 7}[d]
    mats = [rng.choice([-1, 1], size=(r, 70)), rng.integers(-3, 4, size=(r, 40))]
    if lanes == 64:
        mats.append(rng.integers(-2 ** 40, 2 ** 40, size=(r, 9)))
    for a in mats:
        a = np.ascontiguousarray(a, dtype=np.int64)
        ref = O.enumerate_max(a, d, False)
        plan = ld.Plan(a, d, False, ld.options(kernel=2, lane_bits=lanes))
        desc = plan.describe()
        sol = plan.solve()
        plan.close()
        assert (sol.value, sol.gray_index) == ref, desc
        assert " sym=0 " not in desc and sol.evaluated < sol.labelings, desc
        full = ld.solve_reduced(a, d, False, ld.options(kernel=2, lane_bits=lanes, enumerate_all=1))
        assert (full.value, full.gray_index) == ref
        assert full.evaluated == full.labelings


@pytest.mark.parametrize("d,count", [(3, 3), (4, 2), (6, 4)])
def test_wide_kernel_symmetric_shards(ld, d, count):
    rng = np.random.default_rng(70 + d)
    r = {3: 12, 4: 9, 6: 7}[d]
    a = rng.integers(-5, 6, size=(r, 50)).astype(np.int64)
    ref = O.enumerate_max(a, d, False)
    whole = ld.solve_reduced(a, d, False, ld.options(kernel=2))
    parts, ranges, work = [], [], []
    for s in range(count):
        plan = ld.Plan(a, d, False, ld.options(kernel=2, shard_index=s, shard_count=count))
        ranges.append(plan.range)
        sol = plan.solve()
        plan.close()
        parts.append((sol.value, -sol.gray_index))
        work.append(sol.evaluated)
    assert ranges[0][0] == 0 and ranges[-1][1] == O.total(r, d)
    assert all(ranges[i][1] == ranges[i + 1][0] for i in range(count - 1))
    best = max(parts)
    assert (best[0], -best[1]) == ref
    assert sum(work) == whole.evaluated


def test_pruned_search_symmetry(ld):
    """d = 3 pruned search: the walk bound also drops walks that hold no
    class minimum; value and index stay the oracle's, and fewer walks are
    kept than with every walk evaluated."""
    rng = np.random.default_rng(91)
    for t in range(4):
        a = rng.choice([-1, 1], size=(14, 12)) if t % 2 else rng.integers(-3, 4, size=(14, 10))
        a = np.ascontiguousarray(a, dtype=np.int64)
        a[4] = a[2]
        ref = O.enumerate_max(a, 3, False)
        vals, labs = ld.local_search(a, 3, False, n_random=16, seed=t)
        inc = labs[int(np.argmax(vals))]
        sym, st = ld.solve_pruned(a, 3, False, inc, ld.options(prune_policy=1))
        full, stf = ld.solve_pruned(a, 3, False, inc, ld.options(prune_policy=1, enumerate_all=1))
        assert (sym.value, sym.gray_index) == ref == (full.value, full.gray_index)
        assert st["pruned"] == 1 and stf["pruned"] == 1
        assert st["walks_kept"] < stf["walks_kept"], (st, stf)
