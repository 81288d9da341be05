"""The batched path (persistent kernel per lane class over a device work
queue, captured in a CUDA graph) gives every matrix the value and Gray
index the single-matrix solver gives."""
import numpy as np
import pytest

import oracle_ffi as O

pytestmark = pytest.mark.gpu


def mixed_batch(seed, n=48):
    rng = np.random.default_rng(seed)
    mats, ds, ms = [], [], []
    for t in range(n):
        kind = t % 8
        if kind == 0:      # int8-sized d=1
            a = rng.integers(-3, 4, size=(int(rng.integers(6, 20)), int(rng.integers(2, 40))))
            d, m = 1, 0
        elif kind == 1:    # LM
            a = rng.integers(-20, 21, size=(int(rng.integers(6, 18)), int(rng.integers(2, 30))))
            d, m = 1, 1
        elif kind == 2:    # d = 2
            a = rng.integers(-30, 31, size=(int(rng.integers(6, 18)), int(rng.integers(2, 48))))
            d, m = 2, 0
        elif kind == 3:    # d = 3, small entries
            a = rng.integers(-2, 3, size=(int(rng.integers(4, 11)), int(rng.integers(2, 32))))
            d, m = 3, 0
        elif kind == 4:    # d = 4: own plan (wide kernel)
            a = rng.integers(-9, 10, size=(int(rng.integers(3, 8)), int(rng.integers(2, 20))))
            d, m = 4, 0
        elif kind == 5:    # wider than the classes: own plan
            a = rng.integers(-9, 10, size=(int(rng.integers(4, 10)), int(rng.integers(65, 90))))
            d, m = 1, 0
        elif kind == 6:    # 64-bit sums: own plan
            a = rng.integers(-2**40, 2**40, size=(int(rng.integers(3, 10)), int(rng.integers(2, 9))))
            d, m = 1, 0
        else:              # single row
            a = rng.integers(-9, 10, size=(1, int(rng.integers(1, 9))))
            d, m = int(rng.choice([1, 2, 3])), 0
        mats.append(np.asarray(a, dtype=np.int64)); ds.append(d); ms.append(m)
    return mats, ds, ms


@pytest.mark.parametrize("autotune", [False, True])
def test_batch_matches_single_solves(ld, autotune):
    mats, ds, ms = mixed_batch(3)
    b = ld.Batch(mats, ds, ms, autotune=autotune)
    v, g, t = b.solve()
    for p, (a, d, m) in enumerate(zip(mats, ds, ms)):
        ref = O.enumerate_max(a, d, bool(m))
        assert (int(v[p]), int(g[p])) == ref, (p, a.shape, d, m, b.describe())
    # the captured graph replays to the same results
    v2, g2, t2 = b.solve()
    assert np.array_equal(v, v2) and np.array_equal(g, g2)
    assert t > 0 and t2 > 0
    b.close()


def test_batch_of_config4_sample(ld, workloads):
    """A slice of the 4096-matrix configuration (entries N(0, 20^2), d in
    {1,2,3}); matrices with more than 2^22 labelings are left out so the
    oracle check stays fast."""
    insts = [i for i in workloads.config4(count=400, seed=4)]
    mats, ds = [], []
    for inst in insts:
        p = ld.Problem.from_matrix(inst.matrix, inst.d)
        info = p.info
        if info["labelings"] > (1 << 22):
            continue
        mats.append(p.reduced); ds.append(info["d"])
    assert len(mats) > 50
    b = ld.Batch(mats, ds, autotune=True)
    v, g, _ = b.solve()
    for p, (a, d) in enumerate(zip(mats, ds)):
        sol = ld.solve_reduced(a, d)
        assert (int(v[p]), int(g[p])) == (sol.value, sol.gray_index), p
    b.close()


def test_batch_label_symmetry(ld):
    """d = 3 entries (and a d = 4 own plan) skip the walks that hold no class
    minimum; values and Gray indices equal the oracle's and the full run's."""
    rng = np.random.default_rng(31)
    mats, ds = [], []
    for t in range(24):
        r = int(rng.integers(5, 14))
        if t % 3 == 0:
            a = rng.choice([-1, 1], size=(r, int(rng.integers(3, 24))))       # many ties
        elif t % 3 == 1:
            a = rng.integers(-2, 3, size=(r, int(rng.integers(2, 40))))
        else:
            a = rng.integers(-30, 31, size=(r, int(rng.integers(2, 16))))
            a[1] = a[0]
        mats.append(np.asarray(a, dtype=np.int64)); ds.append(3)
    mats.append(rng.integers(-3, 4, size=(8, 12)).astype(np.int64)); ds.append(4)
    b = ld.Batch(mats, ds)
    v, g, _ = b.solve()
    ev = b.evaluated()
    b.close()
    full = ld.Batch(mats, ds, opts=ld.options(enumerate_all=1))
    vf, gf, _ = full.solve()
    evf = full.evaluated()
    full.close()
    for p, (a, d) in enumerate(zip(mats, ds)):
        ref = O.enumerate_max(a, d, False)
        assert (int(v[p]), int(g[p])) == ref, (p, a.shape)
        assert (int(vf[p]), int(gf[p])) == ref, (p, a.shape)
        assert int(evf[p]) == O.total(a.shape[0], d)
    big = [p for p, a in enumerate(mats) if a.shape[0] >= 10]
    assert big and all(ev[p] < evf[p] for p in big)


@pytest.mark.parametrize("split", [1, -1])
def test_batch_column_split(ld, split):
    """Wide int32 classes (40..64 words) on the column-split instances (two
    threads per high index, one shuffle per entry) and on the plain ones:
    the oracle's values and Gray indices, d = 1 (and LM), 2, 3, ties."""
    rng = np.random.default_rng(60 + split)
    mats, ds, ms = [], [], []
    for t in range(18):
        d = 1 + t % 3
        r = int(rng.integers(4, {1: 16, 2: 15, 3: 10}[d]))
        c = int(rng.integers(33, 65))
        a = rng.integers(-300, 301, size=(r, c))
        if t % 4 == 0:
            a[1] = a[0]
        m = int(d == 1 and t % 2 == 0)
        mats.append(np.asarray(a, dtype=np.int64)); ds.append(d); ms.append(m)
    b = ld.Batch(mats, ds, ms, opts=ld.options(batch_split=split), autotune=True)
    desc = b.describe()
    v, g, _ = b.solve()
    b.close()
    assert ("column split" in desc) == (split == 1), desc
    for p, (a, d, m) in enumerate(zip(mats, ds, ms)):
        assert (int(v[p]), int(g[p])) == O.enumerate_max(a, d, bool(m)), (p, a.shape, d, m, desc)


def test_config4_tail_matches_oracle(ld, workloads):
    """The d = 3 tail of the 4096-matrix workload (more than 3^20 labelings
    each, solved one by one outside the batch replay): its smallest
    matrices, all 27 of 22 rows (3^21 labelings), against values the
    oracle computed on the CPU (tests/golden/make_tail_golden.py; one to
    three minutes each there, 20-45 ms each here)."""
    import json
    from pathlib import Path
    gold = json.loads((Path(__file__).parent / "golden" / "config4_tail.json").read_text())
    insts = workloads.config4()
    assert len(gold) == 27
    for g in gold:
        p = ld.Problem.from_matrix(insts[g["index"]].matrix, insts[g["index"]].d)
        red = p.reduced
        assert red.shape == (g["rows"], g["cols"]) and p.info["d"] == 3
        sol = ld.solve_reduced(red, 3)
        assert (sol.value, sol.gray_index) == (g["value"], g["gray_index"]), g["index"]
