"""The multi-rank path on CPU: two gloo ranks each enumerate their shard of
the Gray-index space (with the oracle, since this runs without GPUs) and
exchange only the 16-byte (value, index) candidate; both must end with the
single-process answer, including on ties and with an empty shard.  A rank
that fails before the exchange makes the other's collective fail instead of
hanging."""
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, a, d, marg, shard_units, fail_rank, out):
    import datetime

    sys.path.insert(0, str(ROOT / "tests"))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    from conftest import load_package
    import oracle_ffi as O

    load_package()
    import lnorms_b200.distributed as D

    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                                world_size=world, timeout=datetime.timedelta(seconds=10))
        total = O.total(a.shape[0], d)
        lo, hi = D.shard_bounds(shard_units, rank, world)
        scale = total // shard_units
        lo, hi = lo * scale, hi * scale
        if rank == fail_rank:
            raise RuntimeError("rank failed before the exchange")
        if lo < hi:
            v, n = O.enumerate_max(a, d, marg, lo, hi, 1)
        else:
            v, n = np.iinfo(np.int64).min, np.iinfo(np.int64).max
        host = D.combine(int(v), int(n))
        # the tensor form bench.py queues on the solver's stream (same exchange)
        import torch
        tv, ti = D.combine_tensor(torch.tensor([int(v), int(n)], dtype=torch.int64))
        if (int(tv.item()), int(ti.item())) != host:
            raise AssertionError(f"combine_tensor {(int(tv.item()), int(ti.item()))} != combine {host}")
        out.put((rank, "ok", host))
        dist.destroy_process_group()
    except Exception as e:   # reported to the parent
        out.put((rank, "error", repr(e)))


def _run(world, a, d, marg, shard_units, fail_rank=-1):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, a, d, marg, shard_units, fail_rank, out))
             for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r, status, payload = out.get(timeout=120)
        res[r] = (status, payload)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return res


@pytest.mark.parametrize("d,marg", [(1, False), (1, True), (2, False), (3, False)])
def test_two_ranks_combine_to_the_single_answer(d, marg):
    import oracle_ffi as O
    rng = np.random.default_rng(d + 10 * marg)
    r = {1: 13, 2: 12, 3: 8}[d]
    a = rng.integers(-3, 4, size=(r, 6)).astype(np.int64)
    total = O.total(r, d)
    units = total // (3 if d == 3 else 2)   # shards on coarser units, like the library's walks
    res = _run(2, a, d, marg, units)
    ref = O.enumerate_max(a, d, marg)
    assert res[0] == ("ok", ref) and res[1] == ("ok", ref)


def test_ties_keep_the_smallest_index_and_empty_shard():
    import oracle_ffi as O
    a = np.ones((7, 3), dtype=np.int64)
    a[1::2] *= -1                               # many maximizers, in both shards
    res = _run(2, a, 1, False, 2)
    ref = O.enumerate_max(a, 1, False)
    assert res[0] == ("ok", ref) and res[1] == ("ok", ref)
    res = _run(3, a, 1, False, 2)              # 2 units over 3 ranks: one shard is empty
    assert all(res[r] == ("ok", ref) for r in range(3))


def test_failed_rank_surfaces_as_an_error():
    a = np.arange(24, dtype=np.int64).reshape(8, 3) - 11
    res = _run(2, a, 1, False, 4, fail_rank=1)
    assert res[1][0] == "error"
    assert res[0][0] == "error"                # the survivor's exchange errors out, it does not hang


def test_shard_bounds_tile():
    sys.path.insert(0, str(ROOT))
    from conftest import load_package
    load_package()
    import lnorms_b200.distributed as D
    for units in (0, 1, 5, 1000, 2**40 + 7):
        for count in (1, 2, 3, 8):
            spans = [D.shard_bounds(units, i, count) for i in range(count)]
            assert spans[0][0] == 0 and spans[-1][1] == units
            assert all(spans[i][1] == spans[i + 1][0] for i in range(count - 1))
