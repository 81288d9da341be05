"""Parity of the CUDA path with the oracle and the reference's own outputs.

Everything goes through the C-ABI (ctypes) or the drop-in executable.  The
bar is bit-exact: the same value and the same (smallest) Gray index, hence
the same strategy file.
"""
import subprocess

import numpy as np
import pytest

import oracle_ffi as O
from helpers import GOLDEN, split_tail, without_launch_line

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_pipeline_matches_reference(ld, case):
    d, stat, marg = split_tail(case["tail"])
    value, out, name, strat = ld.lnorm(case["text"], d, stat, marg, 512, 32)
    assert without_launch_line(out) == without_launch_line(case["stdout"])
    assert name == case["strategy_name"]
    assert strat == case["strategy"]


CLI_CASES = [c for c in GOLDEN if c["name"].startswith(("config", "chsh", "reset", "marg_", "zero",
                                                       "single", "sci", "separators", "mid_", "wide_"))]


@pytest.mark.parametrize("case", CLI_CASES, ids=[c["name"] for c in CLI_CASES])
def test_cli_matches_reference(ld, case, tmp_path):
    (tmp_path / "m.txt").write_text(case["text"])
    p = subprocess.run([str(ld.CLI_PATH), "512", "32", "m.txt", *case["tail"]], cwd=tmp_path,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    assert without_launch_line(p.stdout) == without_launch_line(case["stdout"])
    files = list(tmp_path.glob("strategy_*.txt"))
    assert [f.name for f in files] == [case["strategy_name"]]
    assert files[0].read_text() == case["strategy"]


def random_case(seed):
    rng = np.random.default_rng(1000 + seed)
    d = int(rng.choice([1, 1, 1, 2, 2, 3, 3, 4, 5, 6, 8, 10]))
    maxr = {1: 22, 2: 21, 3: 13, 4: 10, 5: 9, 6: 8, 8: 7, 10: 6}[d]
    r = int(rng.integers(1, maxr + 1))
    c = int(rng.choice([1, 2, 3, 5, 8, 13, 24, 31, 40, 64, 65, 100]))
    amp = int(rng.choice([1, 3, 20, 300, 40000]))
    a = rng.integers(-amp, amp + 1, size=(r, c)).astype(np.int64)
    marg = d == 1 and rng.random() < 0.3
    return a, d, marg


@pytest.mark.parametrize("seed", range(120))
def test_random_against_oracle(ld, seed):
    a, d, marg = random_case(seed)
    sol = ld.solve_reduced(a, d, marg)
    v, n = O.enumerate_max(a, d, marg)
    assert (sol.value, sol.gray_index) == (v, n)
    assert np.array_equal(sol.labels, O.labels(n, a.shape[0], d))
    assert sol.labelings == O.total(a.shape[0], d)


FORCED = [dict(kernel=1, lane_bits=8), dict(kernel=1, lane_bits=32),
          dict(kernel=2, lane_bits=32), dict(kernel=2, lane_bits=64),
          dict(kernel=1, low_rows=0), dict(kernel=1, low_rows=1), dict(kernel=1, low_rows=3, tile=2),
          dict(kernel=1, blocks=1), dict(kernel=1, blocks=3, tile=1), dict(kernel=2, blocks=1)]


@pytest.mark.parametrize("d", [1, 2, 3])
@pytest.mark.parametrize("marg", [False, True])
@pytest.mark.parametrize("forced", FORCED, ids=[str(f) for f in FORCED])
def test_every_kernel_path(ld, d, marg, forced):
    if marg and d != 1:
        pytest.skip("marginals are d == 1 only")
    rng = np.random.default_rng(d * 7 + marg)
    r = {1: 17, 2: 16, 3: 11}[d]
    a = rng.integers(-3, 4, size=(r, 9)).astype(np.int64)
    if forced.get("lane_bits") == 8 and marg:
        a[:, 0] = rng.integers(-1, 2, size=r)   # keep 2*sum|A_i0| within int8
    sol = ld.solve_reduced(a, d, marg, ld.options(**forced))
    v, n = O.enumerate_max(a, d, marg)
    assert (sol.value, sol.gray_index) == (v, n)
    if "lane_bits" in forced:
        assert sol.lane_bits == forced["lane_bits"]
    assert sol.kernel_kind == forced["kernel"]


@pytest.mark.parametrize("d", [1, 2, 3, 4])
def test_ties_resolve_to_smallest_index(ld, d):
    """Many labelings share the maximum; the reported index must be the
    first in Gray order (strict '>' per worker, strict '<' across workers)."""
    a = np.ones((9 if d < 4 else 7, 4), dtype=np.int64)
    a[::2] *= -1
    for opts in (ld.options(), ld.options(blocks=1), ld.options(kernel=2)):
        sol = ld.solve_reduced(a, d, False, opts)
        assert (sol.value, sol.gray_index) == O.enumerate_max(a, d, False)


def test_int64_entries(ld):
    rng = np.random.default_rng(5)
    for d in (1, 2, 3, 5):
        a = rng.integers(-2**40, 2**40, size=(8, 6)).astype(np.int64)
        sol = ld.solve_reduced(a, d)
        assert sol.lane_bits == 64
        assert (sol.value, sol.gray_index) == O.enumerate_max(a, d, False)
    # int32 entries whose column sums overflow int32
    a = rng.integers(2**30, 2**31 - 1, size=(10, 5)).astype(np.int64)
    sol = ld.solve_reduced(a, 1)
    assert sol.value > 2**31 and sol.lane_bits == 64
    assert (sol.value, sol.gray_index) == O.enumerate_max(a, 1, False)


@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("count", [2, 3, 5])
def test_shards_tile_the_index_space(ld, kernel, count):
    rng = np.random.default_rng(count)
    a = rng.integers(-9, 10, size=(19, 23)).astype(np.int64)
    full = O.enumerate_max(a, 1, False)
    parts, ranges = [], []
    for s in range(count):
        plan = ld.Plan(a, 1, False, ld.options(kernel=kernel, shard_index=s, shard_count=count))
        lo, hi = plan.range
        sol = plan.solve()
        assert (sol.value, sol.gray_index) == O.enumerate_max(a, 1, False, lo, hi)
        parts.append((sol.value, -sol.gray_index))
        ranges.append((lo, hi))
        plan.close()
    assert ranges[0][0] == 0 and ranges[-1][1] == O.total(19, 1)
    assert all(ranges[i][1] == ranges[i + 1][0] for i in range(count - 1))
    best = max(parts)
    assert (best[0], -best[1]) == full


def test_plan_relaunch_is_stable(ld):
    rng = np.random.default_rng(9)
    a = rng.integers(-20, 21, size=(26, 30)).astype(np.int64)
    plan = ld.Plan(a, 1)
    first = plan.solve()
    for _ in range(3):
        again = plan.solve()
        assert (again.value, again.gray_index) == (first.value, first.gray_index)
        assert again.kernel_ms > 0
    plan.close()
    assert (first.value, first.gray_index) == O.enumerate_max(a, 1, False)


@pytest.mark.parametrize("shape", [(1, 1), (1, 7), (2, 1), (2, 2), (3, 1), (5, 130), (12, 2100), (4, 4096)])
@pytest.mark.parametrize("d", [1, 2, 3])
def test_edge_shapes(ld, shape, d):
    rng = np.random.default_rng(shape[0] * 1000 + shape[1] + d)
    a = rng.integers(-50, 51, size=shape).astype(np.int64)
    sol = ld.solve_reduced(a, d)
    assert (sol.value, sol.gray_index) == O.enumerate_max(a, d, False)


def test_full_size_witness_and_invariances(ld, workloads):
    """At sizes the oracle cannot enumerate: the returned index is a witness
    of the value, and the value is invariant under column permutation and
    column negation, and under negating a free row (d = 1)."""
    a = workloads.lowrank(36, 44, np.random.default_rng(77))
    base = ld.solve_reduced(a, 1)
    assert O.value(a, 1, False, O.labels(base.gray_index, 36, 1)) == base.value
    rng = np.random.default_rng(1)
    perm = rng.permutation(44)
    sign = rng.choice([-1, 1], size=44)
    b = a[:, perm] * sign[None, :]
    assert ld.solve_reduced(b, 1).value == base.value
    c = a.copy()
    c[3] *= -1
    assert ld.solve_reduced(c, 1).value == base.value
    # sharded over 4 = whole
    parts = [ld.solve_reduced(a, 1, False, ld.options(shard_index=s, shard_count=4)) for s in range(4)]
    best = max((p.value, -p.gray_index) for p in parts)
    assert (best[0], -best[1]) == (base.value, base.gray_index)


@pytest.mark.parametrize("seed", range(16))
def test_mixed_lane_widths(ld, seed):
    """d = 1 matrices whose columns split between 8-bit and 32-bit lanes
    (most columns small, a few large), with and without marginals, over
    several low-row counts."""
    rng = np.random.default_rng(500 + seed)
    r = int(rng.integers(8, 21))
    c = int(rng.integers(3, 40))
    a = rng.integers(-3, 4, size=(r, c)).astype(np.int64)
    for col in rng.choice(c, size=int(rng.integers(1, min(c, 4) + 1)), replace=False):
        a[:, col] = rng.integers(-90, 91, size=r)
    marg = bool(seed % 2)
    ref = O.enumerate_max(a, 1, marg)
    for k in (-1, 0, 3, 7, min(r - 1, 10)):
        plan = ld.Plan(a, 1, marg, ld.options(kernel=1, low_rows=k))
        sol = plan.solve()
        assert (sol.value, sol.gray_index) == ref, plan.describe()
        plan.close()


def test_config2_uses_mixed_lanes(ld, workloads):
    inst = workloads.config2()
    p = ld.Problem.from_matrix(inst.matrix, 1, "y", True)
    plan = ld.Plan(p.reduced, 1, True)
    desc = plan.describe()
    assert "int8x4 words=0" not in desc, desc
    sol = plan.solve()
    golden = next(c for c in GOLDEN if c["name"] == inst.name)
    assert f"LM is: {sol.value}" in golden["stdout"]
    assert (sol.value, sol.gray_index) == (398, 3585128208)
    plan.close()


@pytest.mark.parametrize("seed", range(16))
def test_lm_linear_column(ld, seed):
    """LM with the marginal column in a 32-bit word of its own runs the
    instances that add it linearly; value and Gray index match the oracle
    for one or two 32-bit words and 0..16 int8x4 words, including ties."""
    rng = np.random.default_rng(500 + seed)
    r = int(rng.integers(6, 21))
    c = int(rng.integers(1, 66)) if seed % 4 else int(rng.integers(1, 5))
    a = rng.integers(-2, 3, size=(r, c)).astype(np.int64)
    a[:, 0] = rng.integers(-60, 61, size=r)                 # forces a 32-bit marginal column
    if seed % 3 == 0 and c > 2:
        a[:, 1] = rng.integers(-90, 91, size=r)             # and a second 32-bit column
    if seed % 5 == 0:
        a[1] = a[0]                                         # tied rows
    ref = O.enumerate_max(a, 1, True)
    plan = ld.Plan(a, 1, True)
    desc = plan.describe()
    if "int32 words=1 " in desc or "int32 words=2 " in desc:
        assert "lin=1" in desc, desc
    sol = plan.solve()
    assert (sol.value, sol.gray_index) == ref, desc
    plan.close()


@pytest.mark.parametrize("d", [4, 5, 6, 7, 8, 9, 10])
@pytest.mark.parametrize("lanes", ["int8", "int32"])
def test_table_kernel_d4_to_d10(ld, d, lanes):
    """The table decomposition for L_4 .. L_10: value and smallest Gray
    index equal the oracle's and the wide kernel's, for 8-bit and 32-bit
    lanes (widths padded to a multiple of 4 words), with tied rows."""
    rng = np.random.default_rng(1000 * d + (lanes == "int32"))
    for t in range(3):
        r = {4: 9, 5: 8, 6: 7, 7: 7, 8: 6, 9: 6, 10: 6}[d] + t % 2
        if lanes == "int8":
            c = int(rng.integers(2, 33))
            a = rng.integers(-3, 4, size=(r, c)).astype(np.int64)
        else:
            c = int(rng.integers(2, 17))
            a = rng.integers(-40, 41, size=(r, c)).astype(np.int64)
        if t == 2:
            a[1] = a[0]
        ref = O.enumerate_max(a, d, False)
        plan = ld.Plan(a, d, False)
        desc = plan.describe()
        assert desc.startswith("table"), desc
        sol = plan.solve()
        plan.close()
        assert (sol.value, sol.gray_index) == ref, desc
        wide = ld.solve_reduced(a, d, False, ld.options(kernel=2))
        assert (wide.value, wide.gray_index) == ref
        # walks of several high indices (the base-d step) and every low-row count
        for opts in (dict(tile=1), dict(tile=3), dict(low_rows=0, tile=2), dict(low_rows=1, tile=2),
                     dict(low_rows=2, tile=1)):
            plan = ld.Plan(a, d, False, ld.options(kernel=1, **opts))
            desc = plan.describe()
            sol = plan.solve()
            plan.close()
            assert (sol.value, sol.gray_index) == ref, (opts, desc)


def test_plans_sharing_a_kernel_keep_their_shared_memory(ld):
    """Two plans on the same kernel instance: the one created second needs
    less dynamic shared memory; the first still launches (the per-function
    limit is only ever raised)."""
    rng = np.random.default_rng(31)
    big = rng.integers(-3, 4, size=(22, 24)).astype(np.int64)
    small = rng.integers(-3, 4, size=(8, 24)).astype(np.int64)
    pa = ld.Plan(big, 1)
    pb = ld.Plan(small, 1)
    da, db = pa.describe(), pb.describe()
    assert da.split(" k=")[0] == db.split(" k=")[0]               # same instance
    assert int(da.split("smem=")[1].split()[0]) > int(db.split("smem=")[1].split()[0])
    sa = pa.solve()
    assert (sa.value, sa.gray_index) == O.enumerate_max(big, 1, False)
    sb = pb.solve()
    assert (sb.value, sb.gray_index) == O.enumerate_max(small, 1, False)
    pa.close()
    pb.close()


@pytest.mark.parametrize("kind", ["l1", "lm"])
def test_paired_walks(ld, kind):
    """Launches with at least two walks per thread use the instance that
    walks two high indices per thread; value and Gray index match the
    oracle, also split into 3 shards (uneven walk counts) and with tied rows."""
    rng = np.random.default_rng(77 if kind == "l1" else 78)
    if kind == "l1":
        a = rng.integers(-3, 4, size=(29, 30)).astype(np.int64)
        a[5] = a[3]
        marg = False
    else:
        a = rng.integers(-2, 3, size=(29, 20)).astype(np.int64)
        a[:, 0] = rng.integers(-60, 61, size=29)
        marg = True
    ref = O.enumerate_max(a, 1, marg)
    plan = ld.Plan(a, 1, marg)
    desc = plan.describe()
    assert "pair=1" in desc, desc
    if marg:
        assert "lin=1" in desc, desc
    sol = plan.solve()
    plan.close()
    assert (sol.value, sol.gray_index) == ref, desc
    best = None
    for i in range(3):
        sh = ld.solve_reduced(a, 1, marg, ld.options(shard_index=i, shard_count=3))
        cand = (sh.value, -sh.gray_index)
        best = cand if best is None or cand > best else best
    assert (best[0], -best[1]) == ref


def test_lm_linear_column_is_chosen(ld):
    rng = np.random.default_rng(9)
    a = rng.integers(-2, 3, size=(14, 23)).astype(np.int64)
    a[:, 0] = rng.integers(-60, 61, size=14)
    plan = ld.Plan(a, 1, True)
    assert "int32 words=1 " in plan.describe() and "lin=1" in plan.describe()
    assert (plan.solve().value, plan.solve().gray_index) == O.enumerate_max(a, 1, True)
    plan.close()


def prune_cases():
    rng = np.random.default_rng(77)
    for t in range(18):
        d = [1, 1, 2, 3][t % 4]
        marg = d == 1 and t % 3 == 0
        r = {1: int(rng.integers(12, 24)), 2: int(rng.integers(12, 20)), 3: int(rng.integers(8, 13))}[d]
        c = int(rng.integers(2, 30))
        if t % 2:
            u, v = rng.standard_normal((r, 2)), rng.standard_normal((2, c))
            a = np.rint(4 * u @ v).astype(np.int64) + rng.integers(-1, 2, size=(r, c))
        else:
            a = rng.integers(-6, 7, size=(r, c)).astype(np.int64)
        yield t, a, d, marg


@pytest.mark.parametrize("case", list(prune_cases()), ids=lambda c: f"p{c[0]}")
def test_pruned_equals_plain(ld, case):
    _, a, d, marg = case
    ref = O.enumerate_max(a, d, marg)
    vals, labs = ld.local_search(a, d, marg, n_random=32, seed=1)
    for lab in labs[:3]:
        assert O.value(a, d, marg, lab) in vals
    best = labs[int(np.argmax(vals))]
    opt = O.labels(ref[1], a.shape[0], d)
    for inc in (None, best, opt, labs[int(np.argmin(vals))]):
        for policy in (0, 1):           # automatic fallback, and always scan the survivors
            sol, st = ld.solve_pruned(a, d, marg, inc, ld.options(prune_policy=policy))
            assert (sol.value, sol.gray_index) == ref, st
            if inc is not None:
                assert st["incumbent"] == O.value(a, d, marg, inc)
            if policy == 1 and st["walk_rows"] > 0:
                assert st["pruned"] == 1


def test_pruned_falls_back_to_plain_when_bounds_prune_little(ld):
    """Random N(0, 20^2) matrices with d = 3 keep most walk prefixes: the
    automatic policy runs the plain enumeration, with the same answer."""
    rng = np.random.default_rng(7)
    a = np.rint(rng.normal(0, 20, size=(16, 24))).astype(np.int64)
    ref = O.enumerate_max(a, 3, False)
    vals, labs = ld.local_search(a, 3, False, n_random=64, seed=1)
    sol, st = ld.solve_pruned(a, 3, False, labs[int(np.argmax(vals))])
    assert (sol.value, sol.gray_index) == ref
    assert st["pruned"] == 0 and st["walks_kept"] * 4 > st["walks_total"]
    sol, st = ld.solve_pruned(a, 3, False, labs[int(np.argmax(vals))], ld.options(prune_policy=1))
    assert (sol.value, sol.gray_index) == ref and st["pruned"] == 1


def test_pruned_skips_most_blocks_on_low_rank(ld, workloads):
    """With the optimum as incumbent on a low-rank 36x44 matrix, the bounds
    prune most walks and most high indices, and the answer is unchanged."""
    a = workloads.lowrank(36, 44, np.random.default_rng(77))
    plain = ld.solve_reduced(a, 1)
    sol, st = ld.solve_pruned(a, 1, False, O.labels(plain.gray_index, 36, 1))
    assert (sol.value, sol.gray_index) == (plain.value, plain.gray_index)
    assert st["pruned"] == 1
    assert st["walks_kept"] < st["walks_total"] // 4
    assert st["highs_kept"] < st["highs_total"] // 100


@pytest.mark.parametrize("cols", [33, 41, 48, 57, 64])
def test_d3_above_32_words(ld, cols):
    """d = 3 with more than 32 column words keeps H1, H2 and forms H1+H2 on
    the fly; d = 2 up to 64 words."""
    rng = np.random.default_rng(cols)
    a = rng.integers(-60, 61, size=(9, cols)).astype(np.int64)
    for d in (2, 3):
        plan = ld.Plan(a, d, False, ld.options(kernel=1, lane_bits=32))
        sol = plan.solve()
        assert (sol.value, sol.gray_index) == O.enumerate_max(a, d, False), plan.describe()
        plan.close()
