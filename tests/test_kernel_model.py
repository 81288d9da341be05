"""A numpy model of the table kernel's arithmetic, checked against the
oracle on the CPU.  It pins the decomposition the CUDA kernel relies on:
N = h * B + j with the high rows' labels the Gray word of h, the low rows'
labels the Gray word of j read backwards for odd h, the per-D table vectors
and the register vectors they are compared against."""
import numpy as np
import pytest

import oracle_ffi as O


def gray_labels(x, ndig, d):
    return O.labels(x, ndig + 1, d) if ndig > 0 else np.zeros(0, dtype=np.int32)


def table_model(a, d, marginal, k):
    """(max value, smallest Gray index) computed the way the kernel does."""
    R, C = a.shape
    F = R - 1
    base = 2 if d <= 2 else d
    B = base ** k
    nh = F - k
    K = int(np.abs(a[:, 0]).sum()) if marginal else 0
    tot = a.sum(axis=0)
    # table: vectors per low labeling j (Gray order)
    table = []
    for j in range(B):
        lab = gray_labels(j, k, d)
        if d == 1:
            L = sum(((1 if lab[i] else -1) * a[i] for i in range(k)), np.zeros(C, dtype=np.int64))
            table.append([-L])
        else:
            Ls = [sum((a[i] for i in range(k) if lab[i] == m), np.zeros(C, dtype=np.int64)) for m in range(3)]
            if d == 2:
                table.append([-Ls[1], tot - Ls[1]])
            else:
                table.append([-Ls[1], -Ls[2], tot - Ls[1] - Ls[2]])
    best, bestN = None, None
    for h in range(base ** nh):
        lab = gray_labels(h, nh, d)
        if d == 1:
            H = a[R - 1].copy()
            if marginal:
                H[0] += K
            for t in range(nh):
                H += (1 if lab[t] else -1) * a[k + t]
            regs = [H]
        else:
            Hm = [sum((a[k + t] for t in range(nh) if lab[t] == m), np.zeros(C, dtype=np.int64))
                  for m in range(3)]
            regs = [Hm[1], Hm[1]] if d == 2 else [Hm[1], Hm[2], Hm[1] + Hm[2]]
        for jj in range(B):
            je = B - 1 - jj if h & 1 else jj
            v = sum(int(np.abs(r - e).sum()) for r, e in zip(regs, table[je])) - K
            N = h * B + jj
            if best is None or v > best or (v == best and N < bestN):
                best, bestN = v, N
    return best, bestN


@pytest.mark.parametrize("seed", range(24))
def test_table_decomposition_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    d = [1, 2, 3][seed % 3]
    marginal = d == 1 and seed % 2 == 1
    R = int(rng.integers(2, {1: 10, 2: 10, 3: 7}[d]))
    C = int(rng.integers(1, 6))
    a = rng.integers(-4, 5, size=(R, C)).astype(np.int64)
    k = int(rng.integers(0, R))       # 0 .. F low rows
    assert table_model(a, d, marginal, k) == O.enumerate_max(a, d, marginal, nthreads=1)


# ---- d >= 4: the generic base-D step and the low-entry inverse ------------

def reflected_labels(N, ndig, d):
    """Labels of digits 0..ndig-1 of N in the reflected base-d code."""
    out = []
    for _ in range(ndig):
        r = N % (2 * d)
        out.append(r if r < d else 2 * d - 1 - r)
        N //= d
    return out


def low_entry(N, k, d):
    """The isolated low word (table entry) whose labels equal the low
    digits' labels of N; the kernel inverts this map (block_pos_of_entry)."""
    lab = reflected_labels(N, k, d)
    e, p = 0, 0
    for t in range(k - 1, -1, -1):
        digit = d - 1 - lab[t] if p else lab[t]
        e = e * d + digit
        p = (digit & 1) if d % 2 == 0 else ((p + digit) & 1)
    return e


@pytest.mark.parametrize("d", [4, 5, 6, 7, 8, 9, 10])
def test_reflected_code_matches_oracle(d):
    rows = 6
    for N in range(0, d ** (rows - 1), max(1, d ** (rows - 1) // 97)):
        assert reflected_labels(N, rows - 1, d) == list(O.labels(N, rows, d))


@pytest.mark.parametrize("d", [4, 5, 6, 8, 10])
@pytest.mark.parametrize("k", [0, 1, 2, 3])
def test_low_entry_inverts_the_low_labels(d, k):
    B = d ** k
    for h in range(0, 7):
        seen = set()
        for jj in range(B):
            N = h * B + jj
            e = low_entry(N, k, d)
            assert 0 <= e < B
            assert reflected_labels(e, k, d) == reflected_labels(N, k, d)
            seen.add(e)
        assert len(seen) == B                        # a bijection for every h


def block_pos_of_entry(e, k, p0, d):
    """The kernel's block_pos_of_entry: the position j in a block of high
    index h (p0 = h & 1) whose low labels are those of the isolated table
    entry e; the inverse of low_entry.  One top-down pass over e's digits:
    e's own labels (reflection pe, the entry read alone) and j's digits
    (reflection p, starting from the high index's)."""
    pw = d ** (k - 1) if k > 0 else 1
    j, pe, p, rem = 0, 0, p0, e
    for _ in range(k):
        ne = rem // pw
        rem -= ne * pw
        lab = d - 1 - ne if pe else ne
        pe = (ne & 1) if d % 2 == 0 else ((pe + ne) & 1)
        n = d - 1 - lab if p else lab
        p = (n & 1) if d % 2 == 0 else ((p + n) & 1)
        j = j * d + n
        pw //= d
    return j


@pytest.mark.parametrize("d,k", [(4, 1), (4, 3), (5, 2), (5, 3), (6, 2), (7, 2), (8, 2), (9, 2), (10, 2), (3, 4)])
def test_block_pos_inverts_low_entry(d, k):
    B = d ** k
    for h in range(0, 4 * d + 3):
        seen = set()
        for jj in range(B):
            e = low_entry(h * B + jj, k, d)
            assert block_pos_of_entry(e, k, h & 1, d) == jj, (d, k, h, jj)
            seen.add(e)
        assert len(seen) == B       # a bijection of the block onto the table


@pytest.mark.parametrize("d", [4, 5, 6, 9, 10])
def test_generic_step_moves_one_row(d):
    """The kernel's step for D >= 4: walking h within a walk, digit i (the
    lowest nonzero base-d digit of u) moves from label a to label b with
    par = (h / d^(i+1)) odd."""
    ndig, fw = 5, 3
    WL = d ** fw
    for wk in (0, 1, 2, 5):
        h0 = wk * WL
        prev = reflected_labels(h0, ndig, d)
        for u in range(1, WL):
            h = h0 + u
            q, i = u, 0
            while q % d == 0:
                q //= d
                i += 1
            c = q % d
            par = (h // d ** (i + 1)) & 1
            b = d - 1 - c if par else c
            a = d - c if par else c - 1
            cur = reflected_labels(h, ndig, d)
            changed = [t for t in range(ndig) if cur[t] != prev[t]]
            assert changed == [i] and prev[i] == a and cur[i] == b, (h, i, a, b)
            prev = cur
