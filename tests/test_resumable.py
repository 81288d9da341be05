"""Resumable solves, host side (no GPU): the checkpoint file's format, and
the checks made before any device work (another problem's checkpoint,
an unreadable file, a finished solve answered from the file alone)."""
import struct

import numpy as np
import pytest

import oracle_ffi as O


def fingerprint(a, d, marginal, pieces, enumerate_all=0):
    """FNV-1a 64 over (rows, cols, d, marginal, pieces, enumerate_all) as
    int32 and the matrix as int64, little-endian (the library's)."""
    h = 1469598103934665603
    data = struct.pack("<6i", a.shape[0], a.shape[1], d, int(marginal), pieces, enumerate_all)
    data += np.ascontiguousarray(a, dtype="<i8").tobytes()
    for byte in data:
        h ^= byte
        h = (h * 1099511628211) & (2 ** 64 - 1)
    return h


def write_checkpoint(path, fp, pieces, nxt, covered, value, index, labelings=0, evaluated=0, ms=0.0):
    path.write_text(f"lnorms-checkpoint 1\nfingerprint {fp:016x}\npieces {pieces}\nnext {nxt}\n"
                    f"covered {covered}\nvalue {value}\nindex {index}\nlabelings {labelings}\n"
                    f"evaluated {evaluated}\nkernel_ms {ms:.6f}\n")


def test_finished_checkpoint_is_answered_from_the_file(ld, tmp_path):
    a = np.random.default_rng(1).integers(-5, 6, size=(9, 7)).astype(np.int64)
    v, n = O.enumerate_max(a, 3, False)
    total = O.total(9, 3)
    ck = tmp_path / "solve.ckpt"
    write_checkpoint(ck, fingerprint(a, 3, False, 4), 4, 4, total, v, n, total, total // 2, 1.5)
    done, sol = ld.solve_resumable(a, 3, False, pieces=4, checkpoint=ck)
    assert done
    assert (sol.value, sol.gray_index, sol.labelings, sol.evaluated) == (v, n, total, total // 2)
    assert list(sol.labels) == list(O.labels(n, 9, 3))


def test_checkpoint_of_another_problem_is_refused(ld, tmp_path):
    a = np.random.default_rng(2).integers(-5, 6, size=(8, 5)).astype(np.int64)
    ck = tmp_path / "solve.ckpt"
    write_checkpoint(ck, fingerprint(a, 2, False, 4), 4, 1, 10, 3, 3)
    # another split, another order, every walk evaluated: all refused
    for kw in (dict(d=2, pieces=5), dict(d=3, pieces=4), dict(d=2, pieces=4, opts=ld.options(enumerate_all=1))):
        with pytest.raises(ld.LdError) as e:
            ld.solve_resumable(a, kw["d"], False, pieces=kw["pieces"], checkpoint=ck, opts=kw.get("opts"))
        assert e.value.status == 1
    other = a.copy()
    other[0, 0] += 1
    with pytest.raises(ld.LdError):
        ld.solve_resumable(other, 2, False, pieces=4, checkpoint=ck)


def test_unreadable_checkpoint_is_refused(ld, tmp_path):
    a = np.ones((5, 4), dtype=np.int64)
    ck = tmp_path / "solve.ckpt"
    ck.write_text("not a checkpoint\n")
    with pytest.raises(ld.LdError) as e:
        ld.solve_resumable(a, 1, False, pieces=2, checkpoint=ck)
    assert e.value.status == 6
    with pytest.raises(ld.LdError):
        ld.solve_resumable(a, 1, False, pieces=0, checkpoint=tmp_path / "x.ckpt")
