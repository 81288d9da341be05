"""bench.py's pure helpers: the roofline's per-labeling issue-slot count
from a plan description, the plain-method count, and the bounded CPU sample
of a workload (no GPU needed)."""
import importlib.util
import json
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


def test_workload_config_is_the_libraries_reduction(bench, ld):
    """The bench line's `config` (shared by both arms) names the reduced
    shape and labeling count the library's preprocessing produces."""
    for cfg in (1, 2, 3, 5):
        inst = bench.instance(cfg)
        c = bench.workload_config(inst)
        info = ld.Problem.from_matrix(inst.matrix, inst.d, inst.stat, inst.marginal).info
        assert (c["rows"], c["cols"], c["labelings_per_step"]) == (info["rows"], info["cols"], info["labelings"])


def test_reference_output_reduced_shape(bench, ld):
    """The reference arm reads the reduced shape off the reference's own
    stdout; on every golden case with a value line it equals the shape the
    library's preprocessing leaves."""
    import json
    cases = json.loads((ROOT / "tests" / "golden" / "cases.json").read_text())
    checked = 0
    for case in cases:
        if case["rc"] != 0 or " is: " not in case["stdout"] or "zero matrix" in case["stdout"]:
            continue
        value, rows, cols = bench.reference_output(case["stdout"])
        tail = case["tail"]
        d = int(tail[0])
        stat = tail[1] if len(tail) > 1 and tail[1] not in ("m", "M") else "n"
        marg = any(t in ("m", "M") for t in tail[1:]) and d == 1
        p = ld.Problem.from_text(case["text"], d, stat, marg)
        info = p.info
        assert (rows, cols) == (info["rows"], info["cols"]), case["name"]
        checked += 1
    assert checked > 200


def test_reference_arm_runs_the_full_file_without_the_library(tmp_path):
    """`--impl reference` runs L_OpenMP on the whole input file with the
    workload's flags and never maps liblnorms_b200.so into its process."""
    import subprocess
    if not (ROOT / "oracle" / "_ref" / "L_OpenMP").exists():
        pytest.skip("reference binary not built")
    code = ("import runpy, sys, json\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', '--config', '1']\n"
            "runpy.run_path('bench.py', run_name='__main__')\n"
            "print(json.dumps({'mapped': 'liblnorms_b200' in open('/proc/self/maps').read()}))\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]
    line, mapped = lines[0], lines[1]
    assert mapped == {"mapped": False}
    assert line["impl"] == "reference" and line["config"]["labelings_per_step"] == 2 ** 23
    assert line["details"]["reduced"] == [24, 24]


def test_issue_slots_of_the_column_split_count_real_columns(bench):
    d = ("table D=1 int32 words=256 int8x4 words=0 lin=0 pair=0 k=6 B=64 fw=4 walks=1 run=1 sym=0 "
         "blocks=1 tpb=128 smem=1 split=8 p16=0")
    assert bench.issue_ops_per_labeling(d, 1, 200)[0] == 400
    d = ("table D=3 int32 words=0 int8x4 words=64 lin=0 pair=0 k=3 B=27 fw=0 walks=1 run=1 sym=5 "
         "blocks=1 tpb=128 smem=1 split=4 p16=1")
    assert bench.issue_ops_per_labeling(d, 3, 250)[0] == 2 * 3 * 63
