"""The strategy verifier on the CPU: the value it recomputes for each of the
reference's own strategy files (the golden cases, generated by the
reference's L_OpenMP) equals the value the reference printed, through the
library call and through the L_verify executable."""
import re
import subprocess

import numpy as np
import pytest

from helpers import GOLDEN, split_tail

CASES = [c for c in GOLDEN if c["rc"] == 0 and c["strategy"].strip()]


def printed_value(stdout):
    m = re.search(r"^L(?:M|\d+) is: (-?\d+)$", stdout, re.M)
    return int(m.group(1))


def test_golden_cases_present():
    assert len(CASES) > 250


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_reference_strategy_value(ld, case):
    d, stat, marg = split_tail(case["tail"])
    strategy = [int(x) for x in case["strategy"].split()]
    assert ld.strategy_value(case["text"], d, stat, marg, strategy) == printed_value(case["stdout"])


@pytest.mark.parametrize("name", ["chsh", "config2_LM_40x40_y_m", "reset_d5_3x3"])
def test_verify_executable(ld, name, tmp_path):
    case = next((c for c in CASES if c["name"] == name), None)
    if case is None:
        pytest.skip(f"no golden case {name}")
    (tmp_path / "m.txt").write_text(case["text"])
    (tmp_path / case["strategy_name"]).write_text(case["strategy"])
    exe = ld.CLI_PATH.parent / "L_verify"
    p = subprocess.run([str(exe), "m.txt", case["strategy_name"], *case["tail"]], cwd=tmp_path,
                       capture_output=True, text=True, timeout=60)
    assert p.returncode == 0, p.stderr
    line = re.search(r"^L(?:M|\d+) is: -?\d+$", case["stdout"], re.M).group(0)
    assert p.stdout.strip() == line


def test_verifier_rejects_bad_strategies(ld):
    text = "1 2 3\n4 5 6\n-1 0 2\n"
    assert ld.strategy_value(text, 1, "n", False, [1, -1, 1]) == abs(1 - 4 - 1) + abs(2 - 5) + abs(3 - 6 + 2)
    with pytest.raises(ld.LdError):
        ld.strategy_value(text, 1, "n", False, [1, -1])          # wrong length
    with pytest.raises(ld.LdError):
        ld.strategy_value(text, 1, "n", False, [1, 0, 1])        # not a sign
    with pytest.raises(ld.LdError):
        ld.strategy_value(text, 2, "n", False, [0, 2, 1])        # label beyond d - 1


def test_verifier_finds_a_worse_strategy(ld):
    """A strategy that is not optimal verifies to a smaller value."""
    case = next(c for c in CASES if c["name"] == "chsh")
    d, stat, marg = split_tail(case["tail"])
    best = [int(x) for x in case["strategy"].split()]
    worse = [-x for x in best[:-1]] + best[-1:]
    assert ld.strategy_value(case["text"], d, stat, marg, worse) <= printed_value(case["stdout"])


def test_verifier_hand_cases(ld):
    # d = 1, no preprocessing: signs on rows
    text = "1 2\n3 -4\n"
    assert ld.strategy_value(text, 1, "n", False, [1, 1]) == abs(1 + 3) + abs(2 - 4)
    assert ld.strategy_value(text, 1, "n", False, [1, -1]) == abs(1 - 3) + abs(2 + 4)
    # LM: column 0 enters signed
    assert ld.strategy_value(text, 1, "n", True, [1, -1]) == (1 - 3) + abs(2 + 4)
    # d = 1 with more rows than columns is transposed: signs on columns
    tall = "1 2\n3 4\n5 -6\n"
    assert ld.strategy_value(tall, 1, "n", False, [1, -1]) == abs(1 - 2) + abs(3 - 4) + abs(5 + 6)
    with pytest.raises(ld.LdError):
        ld.strategy_value(tall, 1, "n", False, [1, -1, 1])                     # rows, not columns
    # d = 3: labels group rows into messages
    t3 = "1 0\n0 2\n3 3\n"
    assert ld.strategy_value(t3, 3, "n", False, [0, 1, 1]) == 1 + 0 + 3 + 5
