"""Label symmetry for d >= 3, on the CPU.

The table kernel skips a walk (a block of high indices whose top P digits,
the walk number, are fixed) when no index in it can be the smallest Gray
index of its class under permutations of labels 1..d-1.  These tests pin:
the premise (the value is invariant under those permutations: the fixed row
has label 0), the soundness of the walk test (every class minimum lies in a
walk that passes), the exactness of the whole scheme (maximum and smallest
index equal to the oracle's on tie-heavy matrices), and the library's copy
of the test and its digit-DP counts against the model here."""
import itertools

import numpy as np
import pytest

import oracle_ffi as O


def reflected_labels(N, ndig, d):
    out = []
    for _ in range(ndig):
        r = N % (2 * d)
        out.append(r if r < d else 2 * d - 1 - r)
        N //= d
    return out


def index_of(labels, d):
    """Inverse of reflected_labels: the Gray index whose digits carry these
    labels (digit 0 first)."""
    N, par = 0, 0
    for lab in reversed(labels):
        n = d - 1 - lab if par else lab
        N = N * d + n
        par = (par ^ (n & 1)) if d % 2 else (n & 1)
    return N


def walk_ok(w, P, d):
    """The kernel's walk test (walk_holds_class_min): reading the P digits of
    w from the top, each label's first appearance takes the smallest digit
    any unseen label could take there."""
    used, par = {0}, 0
    for q in range(P - 1, -1, -1):
        if d - len(used) <= 1:
            break
        n = (w // d ** q) % d
        lab = d - 1 - n if par else n
        if lab not in used:
            unused = [x for x in range(d) if x not in used]
            if lab != (max(unused) if par else min(unused)):
                return False
            used.add(lab)
        par = (par ^ (n & 1)) if d % 2 else (n & 1)
    return True


def class_min(N, ndig, d):
    labs = reflected_labels(N, ndig, d)
    best = N
    for perm in itertools.permutations(range(1, d)):
        m = [0] + list(perm)
        best = min(best, index_of([m[x] for x in labs], d))
    return best


@pytest.mark.parametrize("d,ndig", [(3, 7), (4, 5), (5, 4), (6, 4)])
def test_index_of_inverts_the_code(d, ndig):
    for N in range(d ** ndig):
        assert index_of(reflected_labels(N, ndig, d), d) == N


@pytest.mark.parametrize("d", [3, 4, 5, 7])
def test_value_is_invariant_under_label_permutations(d):
    rng = np.random.default_rng(d)
    rows = 7
    a = rng.integers(-4, 5, size=(rows, 6))
    for _ in range(40):
        labs = rng.integers(0, d, size=rows - 1)
        v = O.value(a, d, False, labs)
        for perm in itertools.islice(itertools.permutations(range(1, d)), 12):
            m = np.array([0] + list(perm))
            assert O.value(a, d, False, m[labs]) == v


@pytest.mark.parametrize("d,ndig", [(3, 8), (4, 6), (5, 5), (6, 4)])
def test_every_class_minimum_is_in_a_passing_walk(d, ndig):
    for low in range(0, ndig):          # digits below the walk number (k + fw)
        P = ndig - low
        for N in range(d ** ndig):
            if class_min(N, ndig, d) == N:
                assert walk_ok(N // d ** low, P, d), (d, ndig, low, N)


@pytest.mark.parametrize("d,ndig", [(3, 8), (4, 6), (5, 5)])
def test_skipped_walks_hold_no_class_minimum(d, ndig):
    """The converse at the level of whole prefixes: the test is exact for
    walks of one index (it skips every non-minimum it can see)."""
    mins = {N for N in range(d ** ndig) if class_min(N, ndig, d) == N}
    for N in range(d ** ndig):
        assert walk_ok(N, ndig, d) == (N in mins)


def exact_scan(a, d, low):
    """Maximum and smallest index over the walks that pass, walk number =
    N // d^low, as the kernel evaluates them."""
    R = a.shape[0]
    ndig = R - 1
    P = ndig - low
    best, best_n = None, None
    for N in range(d ** ndig):
        if P > 0 and not walk_ok(N // d ** low, P, d):
            continue
        v = O.value(a, d, False, reflected_labels(N, ndig, d))
        if best is None or v > best:
            best, best_n = v, N
    return best, best_n


@pytest.mark.parametrize("d,rows", [(3, 7), (4, 6), (5, 5), (6, 5)])
@pytest.mark.parametrize("kind", ["pm1", "small", "zeroish"])
def test_symmetric_scan_equals_oracle(d, rows, kind):
    rng = np.random.default_rng(rows * 31 + d)
    for trial in range(3):
        if kind == "pm1":
            a = rng.choice([-1, 1], size=(rows, 5))
        elif kind == "small":
            a = rng.integers(-2, 3, size=(rows, 4))
        else:
            a = (rng.random((rows, 4)) < 0.3).astype(np.int64) * rng.integers(1, 3, size=(rows, 4))
        ref = O.enumerate_max(a, d, False, nthreads=1)
        for low in range(0, rows - 1):
            assert exact_scan(a, d, low) == ref, (d, rows, kind, trial, low)


# ---- the library's copy (symmetry.c) ----------------------------------------

@pytest.mark.parametrize("d,P", [(3, 1), (3, 6), (4, 5), (5, 4), (7, 3), (10, 3)])
def test_library_walk_test_matches_model(ld, d, P):
    for w in range(d ** P):
        assert ld.symmetry_walk_ok(d, P, w) == walk_ok(w, P, d), (d, P, w)


@pytest.mark.parametrize("d,P", [(3, 7), (4, 6), (5, 5), (6, 4), (9, 3), (10, 4)])
def test_library_counts_match_model(ld, d, P):
    passing = np.cumsum([0] + [walk_ok(w, P, d) for w in range(d ** P)])
    rng = np.random.default_rng(d * 7 + P)
    W = d ** P
    cases = [(0, W), (0, 0), (W, W), (0, 1), (W - 1, W)] + \
        [tuple(sorted(rng.integers(0, W + 1, size=2))) for _ in range(40)]
    for lo, hi in cases:
        assert ld.symmetry_walks(d, P, int(lo), int(hi)) == passing[hi] - passing[lo], (d, P, lo, hi)


def orbit_count(d, P):
    """Classes of P-digit label strings under permutations of labels 1..d-1:
    choose the i positions with a nonzero label, then split them into at
    most d-1 unlabelled blocks (Stirling numbers of the second kind)."""
    from math import comb
    S = [[0] * (P + 1) for _ in range(P + 1)]
    S[0][0] = 1
    for n in range(1, P + 1):
        for m in range(1, n + 1):
            S[n][m] = m * S[n - 1][m] + S[n - 1][m - 1]
    return sum(comb(P, i) * sum(S[i][m] for m in range(0, min(i, d - 1) + 1)) for i in range(P + 1))


def test_library_counts_large_prefixes(ld):
    """Over all d^P walk numbers the passing ones are exactly the class
    minima, one per class."""
    for d, P in [(3, 8), (4, 6), (3, 39), (4, 31), (5, 27), (7, 22), (10, 18)]:
        assert ld.symmetry_walks(d, P, 0, d ** P) == orbit_count(d, P), (d, P)
    assert ld.symmetry_walks(2, 40, 5, 17) == 12    # d <= 2: every walk
    with pytest.raises(ld.LdError):
        ld.symmetry_walks(3, 41, 0, 1)              # 3^41 >= 2^63


@pytest.mark.parametrize("d,P", [(3, 1), (3, 7), (4, 6), (5, 5), (6, 4), (8, 4), (10, 3)])
def test_library_walk_of_rank_lists_the_passing_walks(ld, d, P):
    passing = [w for w in range(d ** P) if walk_ok(w, P, d)]
    assert [ld.symmetry_walk_at(d, P, r) for r in range(len(passing))] == passing
    with pytest.raises(ld.LdError):
        ld.symmetry_walk_at(d, P, len(passing))


def test_library_walk_of_rank_long_prefixes(ld):
    rng = np.random.default_rng(3)
    for d, P in [(3, 39), (4, 31), (7, 22), (10, 18)]:
        K = ld.symmetry_walks(d, P, 0, d ** P)
        for r in [0, 1, K - 1] + [int(x) for x in rng.integers(0, K, size=20)]:
            w = ld.symmetry_walk_at(d, P, r)
            assert walk_ok(w, P, d)
            assert ld.symmetry_walks(d, P, 0, w) == r     # rank = passing walks below it


def test_library_argument_checks(ld):
    assert ld.symmetry_walk_ok(2, 10, 5) and ld.symmetry_walk_ok(1, 10, 7)     # d <= 2: every walk
    assert not ld.symmetry_walk_ok(3, 2, 9)                                    # not a 2-digit number
    with pytest.raises(ld.LdError):
        ld.symmetry_walks(3, 4, 10, 5)                                         # lo > hi
    with pytest.raises(ld.LdError):
        ld.symmetry_walks(3, 4, 0, 3 ** 4 + 1)                                 # beyond d^P
    with pytest.raises(ld.LdError):
        ld.symmetry_walks(11, 2, 0, 1)                                         # d > 10
    assert ld.symmetry_walk_at(2, 5, 7) == 7
