"""Shared test helpers."""
import json
from pathlib import Path

GOLDEN = json.loads((Path(__file__).parent / "golden" / "cases.json").read_text())


def split_tail(tail):
    """argv tail (d [flag] [m]) -> (d, stat, marginal), as arguments_CUDA
    reads it (L_CUDA.cu:392-409)."""
    d = int(tail[0])
    stat = tail[1][0] if len(tail) > 1 else "n"
    marg = False
    if d == 1 and len(tail) == 2:
        marg = tail[1][0] in "mM"
    elif d == 1 and len(tail) >= 3:
        marg = tail[2][0] in "mM"
    return d, stat, marg


def without_launch_line(s):
    """Drop the worker-count line, which differs between the OpenMP and
    CUDA front ends ("number of threads: .." vs "num_ofBlock: ..")."""
    return [ln for ln in s.splitlines()
            if not ln.startswith("number of threads:") and not ln.startswith("num_ofBlock:")]
