"""Resumable solves on the GPU: a solve interrupted after some pieces and
resumed from its checkpoint gives the oracle's value and Gray index, with
the work of one uninterrupted solve; a changed geometry is refused."""
import numpy as np
import pytest

import oracle_ffi as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("d,shape,pieces", [(3, (13, 9), 5), (1, (21, 30), 7), (4, (10, 8), 4), (2, (16, 12), 4)])
def test_interrupted_solve_resumes(ld, tmp_path, d, shape, pieces):
    rng = np.random.default_rng(d * 100 + pieces)
    a = rng.integers(-4, 5, size=shape).astype(np.int64)
    a[2] = a[1]                                   # ties
    ref = O.enumerate_max(a, d, False)
    whole = ld.solve_reduced(a, d, False)
    ck = tmp_path / "solve.ckpt"
    done, part = ld.solve_resumable(a, d, False, pieces=pieces, checkpoint=ck, max_pieces=2)
    assert not done and ck.exists()
    assert "next 2" in ck.read_text()
    assert part.value <= ref[0]
    done, _ = ld.solve_resumable(a, d, False, pieces=pieces, checkpoint=ck, max_pieces=1)
    assert not done and "next 3" in ck.read_text()
    done, sol = ld.solve_resumable(a, d, False, pieces=pieces, checkpoint=ck)
    assert done
    assert (sol.value, sol.gray_index) == ref
    assert list(sol.labels) == list(whole.labels)
    assert (sol.labelings, sol.evaluated) == (whole.labelings, whole.evaluated)
    # a finished checkpoint answers again without running anything
    done, again = ld.solve_resumable(a, d, False, pieces=pieces, checkpoint=ck)
    assert done and (again.value, again.gray_index) == ref


def test_wide_matrix_in_pieces(ld, tmp_path):
    rng = np.random.default_rng(5)
    a = rng.integers(-50, 51, size=(12, 80)).astype(np.int64)
    done, sol = ld.solve_resumable(a, 1, False, pieces=4, checkpoint=tmp_path / "w.ckpt")
    assert done and (sol.value, sol.gray_index) == O.enumerate_max(a, 1, False)


def test_changed_geometry_is_refused(ld, tmp_path):
    rng = np.random.default_rng(6)
    a = rng.integers(-4, 5, size=(13, 9)).astype(np.int64)
    ck = tmp_path / "solve.ckpt"
    done, _ = ld.solve_resumable(a, 3, False, pieces=5, checkpoint=ck, max_pieces=1, opts=ld.options(tile=1))
    assert not done
    # walks of 27 instead of 3 high indices: the pieces' boundaries move
    with pytest.raises(ld.LdError):
        ld.solve_resumable(a, 3, False, pieces=5, checkpoint=ck, opts=ld.options(tile=3))
    # the checkpoint is untouched and the original options continue it
    done, sol = ld.solve_resumable(a, 3, False, pieces=5, checkpoint=ck, opts=ld.options(tile=1))
    assert done and (sol.value, sol.gray_index) == O.enumerate_max(a, 3, False)
