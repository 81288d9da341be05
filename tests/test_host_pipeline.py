"""The product's host stages (read, preprocess, launch line, report) on the
CPU, against the reference's outputs.  The labeling that the GPU would
return is supplied by the oracle, so everything but the kernel is checked
here without a device."""
import numpy as np
import pytest

import oracle_ffi as O
from helpers import GOLDEN, split_tail, without_launch_line


def _result(ld, value, index):
    r = ld.Result()
    r.value = value
    r.gray_index = index
    return r


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_host_pipeline_matches_reference(ld, case):
    d, stat, marg = split_tail(case["tail"])
    p = ld.Problem.from_text(case["text"], d, stat, marg)
    p.check_launch(512, 32)
    info = p.info
    # reduced matrix and effective d/marginal agree with the oracle's restatement
    ref = O.preprocess(case["text"], d, stat, marg)
    assert (info["rows"], info["cols"]) == ref["matrix"].shape
    assert info["d"] == ref["d"] and info["marginal"] == ref["marginal"]
    assert np.array_equal(p.reduced, ref["matrix"])
    if info["rows"] == 0:
        value, index = 0, 0
    else:
        value, index = O.enumerate_max(p.reduced, info["d"], bool(info["marginal"]))
    name, text = p.report(_result(ld, value, index))
    out = p.log
    if info["rows"] == 0:
        lines = out.splitlines(keepends=True)
        out = "".join(lines[:-1]) + "This is a zero matrix.\n" + lines[-1]
    assert without_launch_line(out) == without_launch_line(case["stdout"])
    assert name == case["strategy_name"]
    assert text == case["strategy"]


@pytest.mark.parametrize("blocks,threads", [(512, 32), (1, 1), (7, 1000), (100000, 3)])
def test_launch_line_matches_reference_clamp(ld, blocks, threads):
    """num_ofBlock line: threads clamped to the labeling count, blocks to
    count / threads (L_CUDA.cu:267-270)."""
    text = "1 2 3 0 1\n4 5 6 1 1\n7 8 10 2 1\n1 0 1 3 1\n"   # 4 rows -> 8 labelings
    p = ld.Problem.from_text(text, 1)
    p.check_launch(blocks, threads)
    total = 8
    t = min(threads, total)
    b = 0 if t == 0 else min(blocks, total // t)
    assert f"num_ofBlock: {b}, num_ofThread in block: {t}\n" in p.log


def test_limits(ld):
    # 64 independent rows with d=1 exceed maxRows = 63 (L_CUDA.cu:277)
    rng = np.random.default_rng(0)
    a = rng.integers(-9, 10, size=(64, 70))
    p = ld.Problem.from_matrix(a, 2)
    with pytest.raises(ld.LdError) as e:
        p.check_launch()
    assert e.value.status == 3
    assert "Matrix is too large. The matrix has 64 rows after reduction." in p.log
    # more than 4096 columns (L_CUDA.cu:278)
    p = ld.Problem.from_matrix(np.ones((2, 4097), dtype=np.int64) * np.array([[1], [2]]) +
                               np.arange(4097)[None, :] % 3, 2)
    with pytest.raises(ld.LdError):
        p.check_launch()
    assert "The length variable 4096 should be greater or equal than 4097." in p.log


def test_malformed_input_is_rejected(ld):
    with pytest.raises(ld.LdError) as e:
        ld.Problem.from_text("1 2 3\n4 5\n6 7 8\n", 1)     # a row shorter than the last
    assert e.value.status == 2
    with pytest.raises(ld.LdError):
        ld.Problem.from_text("  \n\n ; \n", 1)              # no entries
    with pytest.raises(ld.LdError):
        ld.Problem.from_text("1 2\n", 11)                   # d beyond RANK_OF_NORM


def test_parser_rules(ld):
    # separators, scientific notation truncation, decimal tokens, long first row
    p = ld.Problem.from_text("3.9e0, -2.5E1;7\r\n\n1.9 -0.5 4e-1 99\n-1 2 3\n", 2)
    assert p.info["rows_in"] == 3 and p.info["cols_in"] == 3
    q = ld.Problem.from_matrix(np.array([[3, -25, 7], [1, 0, 0], [-1, 2, 3]]), 2)
    assert np.array_equal(p.reduced, q.reduced)


def test_gray_labels_match_oracle(ld):
    for d, rows in [(1, 12), (2, 9), (3, 8), (4, 7), (7, 5), (10, 4)]:
        total = O.total(rows, d)
        for n in list(range(min(total, 200))) + [total - 1, total // 3]:
            assert np.array_equal(ld.gray_labels(n, rows, d), O.labels(n, rows, d))


def test_reduction_order_independent_of_input_magnitude(ld):
    """Grouping by canonical direction agrees with pairwise cross products
    for lines whose gcd is not 1 and for int64-sized entries."""
    big = 3_000_000_000
    a = np.array([[2, 4, 6, 0], [1, 2, 3, 0], [-3, -6, -9, 0], [5, 1, 0, 2], [big, 2 * big, 3 * big, 0]])
    text = "".join(" ".join(map(str, r)) + "\n" for r in a)
    for d in (1, 2):
        p = ld.Problem.from_text(text, d, "y")
        ref = O.preprocess(text, d, "y")
        assert np.array_equal(p.reduced, ref["matrix"])
        ref_lines = O.run_cli(text, d, "y")[1].splitlines()
        ref_lines = ref_lines[:next(i for i, ln in enumerate(ref_lines) if ln.startswith("num_ofBlock"))]
        assert p.log.splitlines() == ref_lines
