"""Host side of the learned proposals: Gray index <-> sign vector <-> labels
against the oracle, feature layout, and training-example alignment."""
import numpy as np
import pytest

import oracle_ffi as O


@pytest.fixture(scope="module")
def L(ld):
    import lnorms_b200.learned as L
    return L


def lowrank(seed, n, m=44):
    import lnorms_b200.workloads as W
    return W.lowrank(n, m, np.random.default_rng(seed))


@pytest.mark.parametrize("seed", range(6))
def test_gray_signs_match_oracle(L, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(3, 20))
    a = rng.integers(-9, 10, size=(n, 7))
    idx = int(rng.integers(0, 2 ** (n - 1)))
    s = L.signs_from_gray(idx, n)
    labs = O.labels(idx, n, 1)
    np.testing.assert_array_equal(L.labels_from_signs(s), labs)
    np.testing.assert_array_equal(L.labels_from_signs(-s), labs)     # global flip: same labeling
    assert int(L.l1_value(a, s)) == O.value(a, 1, False, labs)


def test_oracle_optimum_signs(L):
    a = lowrank(1, 14, 10)
    v, idx = O.enumerate_max(a, 1)
    s = L.signs_from_gray(idx, 14)
    assert int(L.l1_value(a, s)) == v


def test_row_features_layout(L):
    a = lowrank(2, 20)
    v = L.spectral_basis(a)
    assert v.shape == (44, 3)
    np.testing.assert_allclose(v.T @ v, np.eye(3), atol=1e-10)
    dirs = L.hemisphere(32)
    assert np.all(dirs[:, 2] >= 0)
    np.testing.assert_allclose(np.linalg.norm(dirs, axis=1), 1.0)
    x = L.row_features(a, v, dirs)
    assert x.shape == (32, 44) and x.dtype == np.float32
    assert np.all(x[:, 20:] == 0)
    rms = np.sqrt(np.mean(x[:, :20].astype(np.float64) ** 2, axis=1))
    assert np.all((rms > 0.5) & (rms <= 1.0 + 1e-5))
    with pytest.raises(ValueError):
        L.row_features(np.ones((45, 44)), v, dirs)


def test_spectral_basis_matches_lapack(ld, L):
    """The library's subspace iteration gives LAPACK's leading eigenvectors
    of A^T A (up to sign) on the learned search's matrices, each with its
    largest-magnitude component positive."""
    for seed, n in ((1, 16), (2, 28), (3, 44), (4, 20)):
        a = lowrank(seed, n)
        v = ld.spectral_basis(a)
        _, u = np.linalg.eigh(a.T.astype(np.float64) @ a.astype(np.float64))
        ref = u[:, ::-1][:, :3]
        np.testing.assert_allclose(np.abs(np.sum(v * ref, axis=0)), 1.0, atol=1e-9)
        idx = np.argmax(np.abs(v), axis=0)
        assert np.all(v[idx, np.arange(3)] > 0)
        np.testing.assert_allclose(v.T @ v, np.eye(3), atol=1e-10)


def test_spectral_basis_edge_cases(ld):
    # rank 1 and 2: the leading vectors span the row space, the rest is an
    # orthonormal completion
    for rows in (1, 2):
        a = np.random.default_rng(rows).integers(-5, 6, size=(rows, 12)).astype(np.int64)
        v = ld.spectral_basis(a)
        np.testing.assert_allclose(v.T @ v, np.eye(3), atol=1e-9)
        g = a.T.astype(np.float64) @ a
        top = np.linalg.eigvalsh(g)[::-1][:rows]
        np.testing.assert_allclose(np.diag(v.T @ g @ v)[:rows], top, rtol=1e-9)
    # a zero matrix and fewer columns than vectors
    np.testing.assert_allclose(ld.spectral_basis(np.zeros((3, 5), dtype=np.int64)).T
                               @ ld.spectral_basis(np.zeros((3, 5), dtype=np.int64)), np.eye(3), atol=1e-12)
    v = ld.spectral_basis(np.array([[3, 4], [1, -2]], dtype=np.int64))
    assert v.shape == (2, 3) and np.all(v[:, 2] == 0)
    with pytest.raises(ld.LdError):
        ld.spectral_basis(np.ones((3, 65), dtype=np.int64))


def test_training_examples_are_aligned(L):
    mats = [lowrank(s, n) for s, n in ((3, 16), (4, 21), (5, 12))]
    signs = []
    for a in mats:
        _, idx = O.enumerate_max(a, 1)
        signs.append(L.signs_from_gray(idx, a.shape[0]))
    xp, tp, mp = L.training_examples(mats, signs, perturb=2, grid_nearest=0)
    x, t, m = L.training_examples(mats, signs, perturb=2, grid_nearest=0, placed=False)
    # a placement moves each example's rows to n distinct slots, unchanged
    for j, a in enumerate(np.repeat(np.arange(3), 3)):
        n = mats[a].shape[0]
        slots = np.flatnonzero(mp[j])
        assert len(slots) == n
        assert sorted(np.abs(xp[j, slots])) == sorted(np.abs(x[j, :n]))
        score_p = float(np.sum(xp[j] * (2 * tp[j] - 1) * mp[j]))
        score = float(np.sum(x[j] * (2 * t[j] - 1) * m[j]))
        assert abs(score_p - score) < 1e-4
    assert x.shape == (9, 44) and t.shape == (9, 44) and m.shape == (9, 44)
    for j, a in enumerate(np.repeat(np.arange(3), 3)):
        n = mats[a].shape[0]
        assert m[j, :n].all() and not m[j, n:].any()
        s = 2 * t[j, :n] - 1
        assert abs(abs(s @ signs[a]) - n) < 1e-9          # target is +-s*
        assert float(x[j, :n] @ s) >= 0                    # aligned with the scores
    # the optimal direction's sign pattern is close to the optimum
    s0 = np.where(x[0, :16] >= 0, 1, -1)
    assert abs(int(s0 @ signs[0])) >= 12
    # grid directions nearest to the optimum join each matrix's examples
    xg, tg, mg = L.training_examples(mats, signs, perturb=1, grid_nearest=2, placed=False)
    assert xg.shape == (12, 44)
    for j in range(12):
        n = mats[j // 4].shape[0]
        assert float(xg[j, :n] @ (2 * tg[j, :n] - 1)) >= 0


def test_random_and_spectral_proposals(L):
    a = lowrank(6, 24)
    p = L.Proposer("random", directions=16, samples=1)
    s = p.propose(a)
    assert s.shape == (16, 24) and set(np.unique(s)) <= {-1, 1}
    p = L.Proposer("spectral", directions=16, samples=1)
    s = p.propose(a)
    assert s.shape == (16, 24)
    with pytest.raises(ValueError):
        L.Proposer("other")
