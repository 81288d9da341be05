"""Oracle values for the smallest d = 3 matrices of the 4096-matrix batch
workload's tail (the d = 3 matrices with more than 3^20 labelings, solved
one by one outside the batch replay).

    python tests/golden/make_tail_golden.py [count]      (27: every 22-row tail matrix)

Regenerates the workload with its seeded generator, reduces each matrix
with the library's preprocessing (no flag: the matrix as read), picks the
`count` tail matrices with the fewest labelings (the 27 of 22 rows have
3^21 labelings each) and enumerates them with the oracle
(oracle/lnorm_oracle.c, all host threads; one to three minutes each on 8
cores).  Writes tests/golden/config4_tail.json,
which tests/test_gpu_batch.py compares the GPU's single solves with."""
import json
import os
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT))


def main():
    count = int(sys.argv[1]) if len(sys.argv) > 1 else 27
    from conftest import load_package
    import oracle_ffi as O
    ld = load_package()
    import lnorms_b200.workloads as W
    tail = []
    for idx, inst in enumerate(W.config4()):
        p = ld.Problem.from_matrix(inst.matrix, inst.d)
        info = p.info
        if info["d"] == 3 and info["labelings"] > 3 ** 20:
            tail.append((int(info["labelings"]), p.reduced.shape[1], idx, p.reduced))
    tail.sort(key=lambda x: (x[0], x[1]))
    out = []
    for lab, cols, idx, red in tail[:count]:
        t0 = time.perf_counter()
        v, n = O.enumerate_max(red, 3, False, 0, 0, os.cpu_count() or 1)
        out.append({"index": idx, "rows": int(red.shape[0]), "cols": int(red.shape[1]), "labelings": lab,
                    "value": int(v), "gray_index": int(n), "oracle_s": time.perf_counter() - t0})
        print(out[-1], flush=True)
    (ROOT / "tests" / "golden" / "config4_tail.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
