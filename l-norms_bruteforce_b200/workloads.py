"""Seeded synthetic inputs with the shapes and value distributions of the five
benchmark configurations of the brute-force L_d solver.

The reference (istvanmarton/L-norms_BruteForce) ships no datasets; its own
perf tooling draws square matrices with uniform integers (gen_mtx.m:1-5).
These generators follow the five benchmark recipes:

* ``config1``: 24x24, uniform integers in [-10, 10], L_1, no preprocessing.
* ``config2``: 40x40 with marginals (flags ``y m``): row 0 / column 0 uniform
  in [-5, 5], body uniform in {-1, 0, 1}; a 34x37 core plus 4 duplicated
  rows, 2 all-zero rows and 3 duplicated columns at seeded positions, so
  uniting and zero-line removal reduce it back to 34x37 (2^33 labelings).
* ``config3``: 20x30 entries in {-1, +1}, d = 3 (3^19 labelings).
* ``config4``: a batch of matrices, n ~ U[16, 32], m ~ U[16, 64],
  d in {1, 2, 3} with p = .6/.3/.1, entries round(N(0, 20^2)).
* ``config5``: 44x44 low rank, A = round(5 U V) + U{-2..2} noise, U 44x3,
  V 3x44 standard Gaussian, L_1 (2^43 labelings).

All generators use numpy's PCG64 ``default_rng(seed)`` so the same seed gives
the same matrix on every machine with this numpy.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Instance:
    """One solve: the matrix as read from a file, and the CLI arguments."""
    name: str
    matrix: np.ndarray            # int64, rows x cols, as written to the file
    d: int
    stat: str = "n"               # preprocessing flag character (y/r/c or other)
    marginal: bool = False
    meta: dict = field(default_factory=dict)

    def argv_tail(self) -> list[str]:
        """The ``d [flag] [m]`` part of the CLI (README.md:23)."""
        out = [str(self.d)]
        if self.stat not in ("n", ""):
            out.append(self.stat)
            if self.marginal:
                out.append("m")
        elif self.marginal:
            out.append("m")
        return out


def matrix_text(a: np.ndarray, sep: str = " ") -> str:
    """Plain text form accepted by the reference parser (one row per line)."""
    return "".join(sep.join(str(int(v)) for v in row) + "\n" for row in a)


def config1(seed: int = 1) -> Instance:
    rng = np.random.default_rng(seed)
    a = rng.integers(-10, 11, size=(24, 24), dtype=np.int64)
    return Instance("config1_L1_24x24", a, d=1)


def config2(seed: int = 2) -> Instance:
    rng = np.random.default_rng(seed)
    core_r, core_c = 34, 37
    core = rng.integers(-1, 2, size=(core_r, core_c), dtype=np.int64)
    core[0, :] = rng.integers(-5, 6, size=core_c)
    core[:, 0] = rng.integers(-5, 6, size=core_r)
    rows = [core[i].copy() for i in range(core_r)]
    # 4 duplicated rows (full copies, marginal entry included) and 2 zero rows,
    # inserted at positions >= 1 so the marginal row stays first
    for _ in range(4):
        src = rows[int(rng.integers(1, len(rows)))].copy()
        rows.insert(int(rng.integers(1, len(rows) + 1)), src)
    for _ in range(2):
        rows.insert(int(rng.integers(1, len(rows) + 1)), np.zeros(core_c, dtype=np.int64))
    a = np.stack(rows)
    cols = [a[:, j].copy() for j in range(core_c)]
    for _ in range(3):
        src = cols[int(rng.integers(1, len(cols)))].copy()
        cols.insert(int(rng.integers(1, len(cols) + 1)), src)
    a = np.stack(cols, axis=1)
    assert a.shape == (40, 40)
    return Instance("config2_LM_40x40_y_m", a, d=1, stat="y", marginal=True,
                    meta={"core": [core_r, core_c]})


def config3(seed: int = 3) -> Instance:
    rng = np.random.default_rng(seed)
    a = rng.choice(np.array([-1, 1], dtype=np.int64), size=(20, 30))
    return Instance("config3_L3_20x30_pm1", a, d=3)


def config4(count: int = 4096, seed: int = 4,
            n_range=(16, 32), m_range=(16, 64),
            d_probs=(0.6, 0.3, 0.1)) -> list[Instance]:
    rng = np.random.default_rng(seed)
    out = []
    for t in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        m = int(rng.integers(m_range[0], m_range[1] + 1))
        d = int(rng.choice(np.array([1, 2, 3]), p=np.array(d_probs)))
        a = np.rint(rng.normal(0.0, 20.0, size=(n, m))).astype(np.int64)
        out.append(Instance(f"config4_{t}_n{n}_m{m}_d{d}", a, d=d))
    return out


def wide(cols: int, d: int = 1, rows: int = 0, amp: int = 40, seed: int = 6) -> Instance:
    """A matrix wider than one thread's register vectors hold (the
    reference's CLI takes up to 4096 columns, functions.h:2): rows x cols
    uniform integers in [-amp, amp] (32-bit lanes), no flag.  Default rows:
    2^31 labelings for d <= 2, 3^20 for d = 3."""
    rows = rows or {1: 32, 2: 32, 3: 21}.get(d, 12)
    rng = np.random.default_rng(seed)
    a = rng.integers(-amp, amp + 1, size=(rows, cols), dtype=np.int64)
    return Instance(f"wide_L{d}_{rows}x{cols}", a, d=d)


def lowrank(n: int, m: int, rng: np.random.Generator, rank: int = 3,
            scale: float = 5.0, noise: int = 2) -> np.ndarray:
    """round(scale * U V) + uniform integer noise in [-noise, noise]."""
    u = rng.standard_normal((n, rank))
    v = rng.standard_normal((rank, m))
    a = np.rint(scale * (u @ v)).astype(np.int64)
    return a + rng.integers(-noise, noise + 1, size=(n, m), dtype=np.int64)


def config5(seed: int = 5, n: int = 44, m: int = 44) -> Instance:
    rng = np.random.default_rng(seed)
    return Instance(f"config5_L1_{n}x{m}_lowrank", lowrank(n, m, rng), d=1)


def config5_training(count: int = 20000, seed: int = 55, n_range=(16, 28),
                     m: int = 44) -> list[np.ndarray]:
    """Same-distribution matrices with fewer rows, for the proposal network."""
    rng = np.random.default_rng(seed)
    return [lowrank(int(rng.integers(n_range[0], n_range[1] + 1)), m, rng)
            for _ in range(count)]


CONFIGS = {1: config1, 2: config2, 3: config3, 5: config5}
