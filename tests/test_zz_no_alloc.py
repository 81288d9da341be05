"""The no-allocation entry point (ld_solve_reduced_noalloc).

It is for callers that must not allocate GPU memory while they solve: code
inside a process whose other framework holds nearly all device memory, or a
loop that cannot afford the device-wide synchronisation of cudaMalloc /
cudaFree.  Its working memory is one fixed device array inside the library.
Its output must equal the allocating entry point's exactly, on consecutive
calls that reuse that array.  This file is collected last so that a run
that stops at the first failure has run every other test before it."""
import numpy as np
import pytest


def _cases():
    rng = np.random.default_rng(31)
    yield rng.integers(-9, 10, size=(22, 30)).astype(np.int64), 1, False     # 8-bit lanes
    yield rng.integers(-500, 501, size=(21, 40)).astype(np.int64), 1, False  # 32-bit lanes
    yield rng.integers(-5, 6, size=(20, 17)).astype(np.int64), 1, True       # LM
    yield rng.integers(-40, 41, size=(16, 23)).astype(np.int64), 2, False    # d = 2, 32-bit lanes
    yield rng.integers(-3, 4, size=(18, 24)).astype(np.int64), 2, False      # d = 2, 8-bit lanes
    yield rng.choice([-1, 1], size=(12, 30)).astype(np.int64), 3, False      # d = 3, 8-bit lanes
    yield rng.integers(-50, 51, size=(11, 40)).astype(np.int64), 3, False    # d = 3, 32-bit lanes
    yield rng.integers(-50, 51, size=(10, 64)).astype(np.int64), 3, False    # d = 3, 64 columns
    yield rng.integers(-9, 10, size=(8, 128)).astype(np.int64), 1, False     # 128 columns, 8-bit lanes
    yield rng.integers(-300, 301, size=(30, 64)).astype(np.int64), 1, False  # 30 rows x 64 columns


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_and_oracle_twice(ld):
    import oracle_ffi as O
    for a, d, marg in _cases():
        ref = ld.solve_reduced(a, d, marg)
        assert (ref.value, ref.gray_index) == O.enumerate_max(a, d, marg)
        for _ in range(2):                      # the scratch array is reused
            got = ld.solve_reduced_noalloc(a, d, marg)
            assert (got.value, got.gray_index) == (ref.value, ref.gray_index), (a.shape, d, marg)
            assert np.array_equal(got.labels, ref.labels)
            assert got.labelings == ref.labelings
            # d = 3 skips the walks that hold no smallest index of a label class
            assert got.evaluated < got.labelings if d == 3 else got.evaluated == got.labelings


def test_noalloc_rejects_sizes_beyond_its_scratch(ld):
    """Rejected before any device work, so this runs without a GPU."""
    with pytest.raises(ld.LdError) as e:
        ld.solve_reduced_noalloc(np.ones((5, 70), dtype=np.int64) * 1000, 1)
    assert e.value.status == 3 and "columns" in str(e.value)
    with pytest.raises(ld.LdError) as e:
        ld.solve_reduced_noalloc(np.ones((5, 7), dtype=np.int64), 4)
    assert e.value.status == 3
    with pytest.raises(ld.LdError) as e:
        ld.solve_reduced_noalloc(np.ones((64, 7), dtype=np.int64), 1)
    assert e.value.status == 3
    for d in (2, 3):                            # 65 columns in 32-bit lanes, every d
        with pytest.raises(ld.LdError) as e:
            ld.solve_reduced_noalloc(np.ones((5, 65), dtype=np.int64) * 1000, d)
        assert e.value.status == 3 and "64 columns" in str(e.value)
