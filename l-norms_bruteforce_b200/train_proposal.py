"""Train the proposal network on the GPU and write its weights.

    python l-norms_bruteforce_b200/train_proposal.py --out PATH.npz [--count 20000]

1. draws `count` low-rank matrices with 16..28 rows and 44 columns (the
   distribution of the 44 x 44 low-rank workload, fewer rows),
2. solves them exactly with one batched launch of the solver,
3. builds (row scores, optimal signs) examples around each optimum's
   spectral direction and trains the network with the library's
   tensor-core forward / backward kernels and Adam,
4. compares proposal modes on held-out matrices of the same distribution
   and writes a JSON summary next to the weights.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import sys
import time
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent


def load_package():
    if "lnorms_b200" in sys.modules:
        return sys.modules["lnorms_b200"]
    spec = importlib.util.spec_from_file_location("lnorms_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["lnorms_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(PKG_DIR / "data" / "proposal_net.npz"))
    ap.add_argument("--count", type=int, default=20000)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--perturb", type=int, default=1)
    ap.add_argument("--holdout", type=int, default=256)
    ap.add_argument("--holdout44", type=int, default=32)
    ap.add_argument("--directions", type=int, default=64)
    ap.add_argument("--samples", type=int, default=1)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()

    load_package()
    import lnorms_b200.learned as L
    import lnorms_b200.workloads as W

    summary = {"count": args.count}
    t0 = time.perf_counter()
    mats = W.config5_training(args.count)
    signs, values, ms = L.solve_training_set(mats, device=args.device)
    summary["solve_s"] = time.perf_counter() - t0
    summary["solve_device_ms"] = ms
    summary["labelings"] = int(sum(2 ** (a.shape[0] - 1) for a in mats))
    for a, s, v in zip(mats[:64], signs[:64], values[:64]):
        assert int(L.l1_value(a, s)) == int(v), "Gray index and value disagree"

    t0 = time.perf_counter()
    x, t, m = L.training_examples(mats, signs, perturb=args.perturb)
    summary["examples"] = int(x.shape[0])
    summary["features_s"] = time.perf_counter() - t0

    t0 = time.perf_counter()
    net, hist = L.train(x, t, m, epochs=args.epochs, device=args.device,
                        log=lambda s: print(s, flush=True))
    summary["train_s"] = time.perf_counter() - t0
    summary["loss_history"] = hist
    params = net.get_params()
    net.close()
    params["skip"] = np.float32(L.SKIP)
    out = Path(args.out)
    out.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(out, **params)

    hold = W.config5_training(args.holdout, seed=56)
    hsigns, hvals, _ = L.solve_training_set(hold, device=args.device)
    res = []
    budgets = [(2, 1), (4, 1), (8, 1), (32, 1), (args.directions, args.samples)]
    for directions, samples in budgets:
        for mode in L.PROPOSAL_MODES:      # equal proposal counts per mode
            p = L.Proposer(mode, directions=directions, samples=samples,
                           params=params if mode == "network" else None, device=args.device)
            res.append(L.evaluate(hold, hvals, p))
            p.close()
            print(json.dumps(res[-1]), flush=True)
    summary["holdout"] = res

    # 44-row matrices (the workload's shape, never seen in training): exact
    # optima from the pruned enumeration, which is exact for any incumbent
    rng = np.random.default_rng(4444)
    big = [W.lowrank(44, 44, rng) for _ in range(args.holdout44)]
    ref = L.Proposer("spectral", directions=64, samples=1, device=args.device)
    bvals = [L.solve_learned(a, ref)[0].value for a in big]
    ref.close()
    res44 = []
    for directions, samples in budgets:
        for mode in L.PROPOSAL_MODES:
            p = L.Proposer(mode, directions=directions, samples=samples,
                           params=params if mode == "network" else None, device=args.device)
            res44.append(L.evaluate(big, bvals, p))
            p.close()
            print("n=44", json.dumps(res44[-1]), flush=True)
    summary["holdout44"] = res44
    out.with_suffix(".json").write_text(json.dumps(summary, indent=1))
    print(json.dumps({k: v for k, v in summary.items() if k != "loss_history"}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
