"""The reference-side binding: the reference's own L_OpenMP.c program, compiled
unmodified, with its calc_Lnorm (L_OpenMP.c:241-297) replaced by a call to
ld_solve_reduced (oracle/binding_calc_lnorm.c, linked by `make -C oracle
binding` into oracle/_ref/L_OpenMP_b200).  The reference's main, argument
checks, parser, preprocessing and print_results run around the library's
solve; on the golden cases its stdout and strategy file must equal the
reference's own, byte for byte."""
import json
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "oracle" / "_ref" / "L_OpenMP_b200"


def _cases():
    cases = json.loads((ROOT / "tests" / "golden" / "cases.json").read_text())
    ok = [c for c in cases if c["rc"] == 0]
    # every configuration case, then up to 12 cases of each kind of output
    # (marginals, transposed, d reset, zero matrix, united lines, plain)
    kinds = {}
    for c in ok:
        out = c["stdout"]
        kind = ("config" if c["name"].startswith("config") else "LM" if "LM is" in out else
                "transposed" if "transposed" in out else "reset" if "less than or equal" in out else
                "zero" if "zero matrix" in out else "united" if "was added" in out or "subtracted" in out
                else "plain")
        kinds.setdefault(kind, []).append(c)
    return [c for kind, cs in kinds.items() for c in (cs if kind == "config" else cs[:: max(1, len(cs) // 12)])]


def _run(case, tmp):
    (tmp / "m.txt").write_text(case["text"])
    for f in tmp.glob("strategy_*.txt"):
        f.unlink()
    p = subprocess.run([str(BIN), str(case["nthreads"]), "m.txt", *case["tail"]], cwd=tmp,
                       capture_output=True, text=True, timeout=300)
    strategy = (tmp / case["strategy_name"]).read_text() if case.get("strategy_name") and \
        (tmp / case["strategy_name"]).exists() else None
    return p, strategy


def test_binding_calls_the_library_not_the_reference_body(tmp_path):
    """Without a GPU the library's solve fails, so the program stops with
    the library's error: the reference's OpenMP body is not what runs."""
    torch = pytest.importorskip("torch")
    if not BIN.exists():
        pytest.skip("binding not built (needs the reference sources)")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the gpu test covers the binding")
    case = {"text": "1 1\n1 -1\n", "tail": ["1"], "nthreads": 2, "strategy_name": "strategy_L1.txt"}
    p, strategy = _run(case, tmp_path)
    assert p.returncode != 0
    assert "CUDA" in p.stderr and "L1 is:" not in p.stdout and strategy is None


@pytest.mark.gpu
def test_reference_main_around_the_library_matches_golden(tmp_path):
    if not BIN.exists():
        pytest.skip("binding not built (needs the reference sources)")
    cases = _cases()
    assert len(cases) > 50
    for case in cases:
        p, strategy = _run(case, tmp_path)
        assert p.returncode == 0, (case["name"], p.stderr[-500:])
        assert p.stdout == case["stdout"], case["name"]
        if case.get("strategy_name") and "zero matrix" not in case["stdout"]:
            assert strategy == case["strategy"], case["name"]
