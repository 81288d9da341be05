"""Learned proposals for the exact L_1 search (no counterpart in the reference).

The exact answer never depends on this module: it only supplies the
incumbent that the pruned enumeration (`solve_pruned`) compares its block
bounds against, and the pruned enumeration returns the plain enumeration's
value and Gray index for any incumbent.

Proposal scheme (L_1, non-marginal; sign vectors s in {-1,+1}^n, value
|A^T s|_1):

* Spectral directions.  V holds the top three right singular vectors of
  the matrix (m x 3).  A direction c on the unit sphere of R^3 gives row
  scores x(c) = A V c; sign(x(c)) is the classical rank-3 candidate, and
  sweeping c over a hemisphere covers the sign patterns of the rank-3 part.
* The network.  Its 44 inputs are the row scores x(c) scaled to unit RMS
  and clipped to [-8, 8], one per input slot; a matrix with n <= 44 rows
  occupies n slots (a placement), the others are zero.  Its 44 outputs are
  the logits of s_i = +1 per slot, with a parameter-free residual path
  (logit = network + SKIP * x) so that it learns corrections to the
  spectral sign rather than the sign itself.  It is trained on optimal
  labelings that the solver computes for small matrices of the same
  distribution (n in [16, 28]): the training direction is c* = V^T A^T s*
  normalised (the optimum's column sums seen in the spectral space) plus
  perturbed copies of it, the target is s* sign-aligned with x(c*), and
  every example gets a random placement, so that all 44 slots are trained
  although no training matrix has 44 rows.  Training directions are c*, a
  perturbed copy, and the grid directions nearest to c* (the grid the
  proposals use).  For each direction the proposals are the network's most
  likely labelings under `samples` different placements (placement 0 is the
  identity; the default is one).
* Every proposal is polished on the GPU by single-row-move local search
  (`local_search`), and the best polished value becomes the incumbent.

`PROPOSAL_MODES` names the ablations the tests and the bench compare:
"random" (uniform starts), "spectral" (sign(x(c)) starts) and "network".
"""
from __future__ import annotations

import time
from pathlib import Path

import numpy as np

N_MAX = 44
SKIP = 4.0
WEIGHTS = Path(__file__).resolve().parent / "data" / "proposal_net.npz"
PROPOSAL_MODES = ("random", "spectral", "network")


def _pkg():
    import sys
    return sys.modules[__name__.rsplit(".", 1)[0]]


# ---- features ---------------------------------------------------------------

def spectral_basis(a: np.ndarray, k: int = 3) -> np.ndarray:
    """Top-k right singular vectors (m x k) of a (rows x cols) matrix: the
    eigenvectors of A^T A with the k largest eigenvalues, from the library's
    subspace iteration (ld_spectral_basis; each vector's largest component
    positive).  A direction and its negation give the same labeling, so the
    sign rule does not matter to the proposals.  Matrices wider than 64
    columns use LAPACK through numpy."""
    if a.shape[1] <= 64 and k <= 8:
        return _pkg().spectral_basis(a, k)
    a = np.asarray(a, dtype=np.float64)
    _, u = np.linalg.eigh(a.T @ a)
    v = u[:, ::-1][:, :k]
    if v.shape[1] < k:
        v = np.concatenate([v, np.zeros((v.shape[0], k - v.shape[1]))], axis=1)
    return v


def hemisphere(count: int) -> np.ndarray:
    """`count` near-uniform unit vectors of R^3 with z >= 0 (Fibonacci)."""
    i = np.arange(count) + 0.5
    z = 1.0 - i / count                       # (0, 1]
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = i * np.pi * (3.0 - np.sqrt(5.0))
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


def row_features(a: np.ndarray, v: np.ndarray, dirs: np.ndarray) -> np.ndarray:
    """Network inputs (len(dirs) x 44): scaled row scores A V c per direction."""
    a = np.asarray(a, dtype=np.float64)
    n = a.shape[0]
    if n > N_MAX:
        raise ValueError(f"the proposal network handles at most {N_MAX} rows")
    x = (a @ v @ np.asarray(dirs, dtype=np.float64).T).T          # dirs x n
    rms = np.sqrt(np.mean(x * x, axis=1, keepdims=True)) + 1e-12
    out = np.zeros((x.shape[0], N_MAX), dtype=np.float32)
    out[:, :n] = np.clip(x / rms, -8.0, 8.0)
    return out


def optimal_direction(a: np.ndarray, v: np.ndarray, s: np.ndarray) -> np.ndarray:
    c = v.T @ (np.asarray(a, dtype=np.float64).T @ s)
    nrm = np.linalg.norm(c)
    return c / nrm if nrm > 0 else np.array([0.0, 0.0, 1.0])


# ---- labelings --------------------------------------------------------------

def signs_from_gray(index: int, rows: int) -> np.ndarray:
    """Sign vector (+-1, last row +1) of a d == 1 Gray index: label bit i of
    row i is ((N + 2^i) >> (i + 1)) & 1, and label 1 means +1."""
    i = np.arange(rows - 1, dtype=np.uint64)
    bits = ((np.uint64(index) + (np.uint64(1) << i)) >> (i + np.uint64(1))) & np.uint64(1)
    return np.concatenate([np.where(bits == 1, 1, -1), [1]]).astype(np.int64)


def labels_from_signs(s: np.ndarray) -> np.ndarray:
    """Labels of rows 0..n-2 (1 = +1) after flipping s so its last row is +1."""
    s = np.asarray(s)
    s = s * np.where(s[..., -1:] < 0, -1, 1)
    return (s[..., :-1] > 0).astype(np.int32)


def l1_value(a: np.ndarray, s: np.ndarray) -> np.ndarray:
    return np.abs(np.asarray(s, dtype=np.int64) @ np.asarray(a, dtype=np.int64)).sum(axis=-1)


# ---- training data ----------------------------------------------------------

def place(x: np.ndarray, n: int, slots: np.ndarray) -> np.ndarray:
    """Move the first n entries of each row of x to the given slots."""
    out = np.zeros_like(x)
    out[..., slots] = x[..., :n]
    return out


def training_examples(mats, signs, perturb: int = 1, sigma: float = 0.2, grid_nearest: int = 2,
                      grid_sizes=(2, 4, 8, 16, 32, 64), seed: int = 0, placed: bool = True):
    """(x, t, mask) arrays.  Per matrix: the optimal direction c*, `perturb`
    noisy copies of it, and the `grid_nearest` directions nearest to +-c* of
    the hemisphere grid the proposals use (grid size drawn from
    `grid_sizes`), so that training sees the directions inference uses.
    Targets are the optimal sign vector aligned with x; each example gets a
    random placement of the rows over the 44 slots."""
    rng = np.random.default_rng(seed)
    rng_place = np.random.default_rng(seed + 1)
    grids = {g: hemisphere(g) for g in grid_sizes}
    xs, ts, ms = [], [], []
    for a, s in zip(mats, signs):
        n = a.shape[0]
        v = spectral_basis(a)
        c0 = optimal_direction(a, v, s)
        dirs = [c0]
        for _ in range(perturb):
            c = c0 + sigma * rng.standard_normal(3)
            dirs.append(c / np.linalg.norm(c))
        if grid_nearest:
            g = grids[grid_sizes[int(rng.integers(len(grid_sizes)))]]
            cos = g @ c0
            for k in np.argsort(-np.abs(cos))[:grid_nearest]:
                dirs.append(g[k] * (1.0 if cos[k] >= 0 else -1.0))
        x = row_features(a, v, np.array(dirs))
        for j in range(len(dirs)):
            sa = s if float(x[j, :n] @ s) >= 0 else -s
            t = np.zeros(N_MAX, dtype=np.float32)
            t[:n] = (sa > 0)
            m = np.zeros(N_MAX, dtype=np.float32)
            m[:n] = 1.0
            xj = x[j]
            if placed:
                slots = rng_place.permutation(N_MAX)[:n]
                xj, t, m = place(xj, n, slots), place(t, n, slots), place(m, n, slots)
            xs.append(xj)
            ts.append(t)
            ms.append(m)
    return np.array(xs), np.array(ts), np.array(ms)


def solve_training_set(mats, device: int = 0):
    """Optimal sign vectors of raw matrices from one batched exact solve."""
    ld = _pkg()
    batch = ld.Batch(mats, [1] * len(mats), opts=ld.options(device=device))
    values, gray, ms = batch.solve()
    batch.close()
    signs = [signs_from_gray(int(g), a.shape[0]) for a, g in zip(mats, gray)]
    return signs, values, ms


def train(x, t, m, epochs: int = 30, batch: int = 1024, lr: float = 2e-3, seed: int = 0, device: int = 0,
          log=None):
    """Train a fresh network on the device; returns (Mlp, per-epoch mean losses)."""
    ld = _pkg()
    net = ld.Mlp(batch=batch, seed=seed, device=device, skip=SKIP)
    rng = np.random.default_rng(seed)
    history = []
    n = x.shape[0]
    for ep in range(epochs):
        order = rng.permutation(n)
        rate = lr * 0.5 * (1 + np.cos(np.pi * ep / epochs))      # cosine decay
        total, cnt = 0.0, 0
        for i in range(0, n - batch + 1, batch):
            idx = order[i:i + batch]
            total += net.train_step(x[idx], t[idx], m[idx], lr=rate)
            cnt += 1
        history.append(total / max(cnt, 1))
        if log:
            log(f"epoch {ep}: loss {history[-1]:.4f} lr {rate:.2e}")
    return net, history


# ---- proposals --------------------------------------------------------------

class Proposer:
    """Generates start labelings for the local search in one of the
    PROPOSAL_MODES; "network" loads the trained weights (or takes params).
    count() = directions * samples proposals in every mode."""

    def __init__(self, mode: str = "network", directions: int = 64, samples: int = 1,
                 params: dict | None = None, device: int = 0, seed: int = 0):
        if mode not in PROPOSAL_MODES:
            raise ValueError(f"mode must be one of {PROPOSAL_MODES}")
        self.mode, self.directions, self.samples, self.seed = mode, directions, samples, seed
        self.device = device
        self.net = None
        if mode == "network":
            ld = _pkg()
            if params is None:
                if not WEIGHTS.exists():
                    raise FileNotFoundError(f"{WEIGHTS} is missing: run train_proposal.py")
                with np.load(WEIGHTS) as f:
                    params = {k: f[k] for k in f.files}
            params = dict(params)
            skip = float(params.pop("skip", SKIP))
            rows = directions * samples
            self.net = ld.Mlp(batch=max(128, -(-rows // 128) * 128), seed=0, device=device, skip=skip)
            self.net.set_params(params)

    def count(self) -> int:
        return self.directions * self.samples

    def propose(self, a: np.ndarray) -> np.ndarray:
        """count() sign vectors (+-1) for the rows of `a`."""
        n = a.shape[0]
        rng = np.random.default_rng(self.seed)
        if self.mode == "random":
            return rng.choice([-1, 1], size=(self.count(), n))
        v = spectral_basis(a)
        x = row_features(a, v, hemisphere(self.directions))
        if self.mode == "spectral":
            x = row_features(a, v, hemisphere(self.count()))
            return np.where(x[:, :n] >= 0, 1, -1)
        slots = [np.arange(n)] + [rng.permutation(N_MAX)[:n] for _ in range(self.samples - 1)]
        z = self.net.forward(np.concatenate([place(x, n, sl) for sl in slots], axis=0))
        z = np.concatenate([z[k * len(x):(k + 1) * len(x)][:, sl] for k, sl in enumerate(slots)], axis=0)
        return np.where(z >= 0, 1, -1)

    def close(self):
        if self.net is not None:
            self.net.close()
            self.net = None


def incumbent(a: np.ndarray, proposer: Proposer, max_rounds: int = 0):
    """Best local-search-polished proposal: (value, labels, stats)."""
    ld = _pkg()
    t0 = time.perf_counter()
    s = proposer.propose(a)
    t1 = time.perf_counter()
    raw = l1_value(a, s)
    values, labels = ld.local_search(a, 1, False, starts=labels_from_signs(s), max_rounds=max_rounds,
                                     device=proposer.device)
    t2 = time.perf_counter()
    best = int(np.argmax(values))
    return int(values[best]), labels[best], {"proposals": int(s.shape[0]), "raw_best": int(raw.max()),
                                             "raw_mean": float(raw.mean()), "polished_best": int(values[best]),
                                             "polished_mean": float(values.mean()),
                                             "propose_s": t1 - t0, "local_search_s": t2 - t1}


def solve_learned(a, proposer: Proposer | None = None, opts=None):
    """Exact L_1 solve of a reduced matrix: learned incumbent, then the pruned
    enumeration.  Returns (Solution, stats); the Solution equals the plain
    enumeration's (value and Gray index) whatever the incumbent."""
    ld = _pkg()
    a = np.ascontiguousarray(np.asarray(a, dtype=np.int64))
    own = proposer is None
    if own:
        proposer = Proposer("network")
    try:
        t0 = time.perf_counter()
        value, labels, st = incumbent(a, proposer)
        t1 = time.perf_counter()
        sol, pst = ld.solve_pruned(a, 1, False, labels, opts)
        t2 = time.perf_counter()
    finally:
        if own:
            proposer.close()
    st.update({"incumbent": value, "incumbent_s": t1 - t0, "pruned_s": t2 - t1, "total_s": t2 - t0})
    st.update({f"prune_{k}": v for k, v in pst.items()})
    return sol, st


def evaluate(mats, optimum, proposer: Proposer) -> dict:
    """Incumbent quality of one proposal mode over matrices with known optimum
    values: how often the polished incumbent is already optimal, the mean
    relative gap, and the mean raw (unpolished) best proposal / optimum."""
    hits, gaps, raw, secs = 0, [], [], 0.0
    for a, opt in zip(mats, optimum):
        value, _, st = incumbent(np.asarray(a, dtype=np.int64), proposer)
        hits += int(value == int(opt))
        gaps.append((int(opt) - value) / max(int(opt), 1))
        raw.append(st["raw_best"] / max(int(opt), 1))
        secs += st["propose_s"] + st["local_search_s"]
    k = max(len(gaps), 1)
    return {"mode": proposer.mode, "proposals": proposer.count(), "matrices": len(gaps),
            "optimal_rate": hits / k, "mean_gap": float(np.mean(gaps)) if gaps else 0.0,
            "raw_best_ratio": float(np.mean(raw)) if raw else 0.0, "seconds": secs}


def solve_learned_batch(mats, proposer: Proposer, opts=None):
    """Exact L_1 solves of many reduced matrices (each <= 44 rows): the
    proposals of every matrix come from one forward pass of the network
    over all their directions; then per matrix the polished incumbent and
    the pruned enumeration.  Returns [(Solution, stats)] in input order; each
    Solution equals the plain enumeration's."""
    ld = _pkg()
    mats = [np.ascontiguousarray(np.asarray(a, dtype=np.int64)) for a in mats]
    if proposer.mode != "network":
        return [solve_learned(a, proposer, opts) for a in mats]
    t0 = time.perf_counter()
    dirs = hemisphere(proposer.directions)
    feats = [row_features(a, spectral_basis(a), dirs) for a in mats]
    z = proposer.net.forward(np.concatenate(feats, axis=0))
    t1 = time.perf_counter()
    out = []
    for p, a in enumerate(mats):
        n = a.shape[0]
        zp = z[p * len(dirs):(p + 1) * len(dirs), :n]
        s = np.where(zp >= 0, 1, -1)
        t2 = time.perf_counter()
        values, labels = ld.local_search(a, 1, False, starts=labels_from_signs(s), device=proposer.device)
        best = int(np.argmax(values))
        t3 = time.perf_counter()
        sol, pst = ld.solve_pruned(a, 1, False, labels[best], opts)
        t4 = time.perf_counter()
        st = {"incumbent": int(values[best]), "raw_best": int(l1_value(a, s).max()),
              "propose_s": (t1 - t0) / len(mats), "local_search_s": t3 - t2, "pruned_s": t4 - t3}
        st.update({f"prune_{k}": v for k, v in pst.items()})
        out.append((sol, st))
    return out
