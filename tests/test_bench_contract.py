"""bench.py's pure helpers: the roofline's per-labeling issue-slot count
from a plan description, the plain-method count, and the bounded CPU sample
of a workload (no GPU needed)."""
import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def bench(ld):
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    old = sys.argv
    sys.argv = ["bench.py"]
    try:
        spec.loader.exec_module(mod)
    finally:
        sys.argv = old
    return mod


def test_issue_slots_from_plan_description(bench):
    d = "table D=1 int32 words=1 int8x4 words=9 lin=1 k=9 B=512 fw=1 walks=8388608 blocks=1184 tpb=128 smem=26352"
    assert bench.issue_ops_per_labeling(d, 1, 37)[0] == 18          # 9 vabsdiff4, column 0 linear
    d = "table D=1 int32 words=1 int8x4 words=9 lin=0 k=9 B=512 fw=1 walks=8388608 blocks=1184 tpb=128 smem=26352"
    assert bench.issue_ops_per_labeling(d, 1, 37)[0] == 20
    d = "table D=3 int32 words=0 int8x4 words=8 lin=0 k=5 B=243 fw=0 walks=4782969 blocks=1036 tpb=128 smem=24064"
    assert bench.issue_ops_per_labeling(d, 3, 30)[0] == 48
    assert bench.issue_ops_per_labeling("wide PC=2 multi=0 int32 blocks=1 tpb=2", 5, 37)[0] == 6 * 37


def test_plain_method_count(bench):
    assert bench.ops_per_labeling(1, 37) == 111
    assert bench.ops_per_labeling(3, 30) == 180


def test_reference_sample_keeps_columns_and_fixed_row(bench, ld, workloads):
    inst = workloads.config2()
    a, tail, n, what = bench.reference_sample(inst, ld, 1 << 20)
    assert tail == ["1", "m"]
    assert a.shape[1] == 37 and n == 2 ** (a.shape[0] - 1) <= 1 << 20
    p = ld.Problem.from_matrix(inst.matrix, inst.d, inst.stat, inst.marginal)
    red = p.reduced
    np.testing.assert_array_equal(a[0], red[-1])          # the marginal row goes first in the file
    np.testing.assert_array_equal(a[1:], red[: a.shape[0] - 1])


def test_clock_sampler_without_a_device(bench):
    c = bench.ClockSampler(0)
    out = c.stop()
    assert set(out) >= {"sm_mhz", "sm_max_mhz", "reasons"}
