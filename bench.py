#!/usr/bin/env python3
"""Benchmark of the exact L_d solver (plain Gray-code enumeration).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config 2] [--impl ours|reference]

One step is one complete exact solve of the workload (configuration 2 by
default: the 40x40 marginal Bell expression with flags `y m`, reduced to
34x37, 2^33 labelings).  `value` is labelings/s over K device-timed steps
(CUDA events on the solver's stream, L2 flushed between steps, inputs
resident); `e2e` is the same metric through the public API from host
buffers (upload, solve, 16-byte result read, strategy report).  With N > 1
(torchrun) every rank enumerates its shard of the same solve and the ranks
combine the 16-byte (value, Gray index) candidate with two NCCL all-reduces;
the time is the max over ranks.

`--impl reference` times the reference's own OpenMP solver (oracle/_ref,
built from the reference sources) on the host cores instead.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "l-norms_bruteforce_b200"
REF_BIN = ROOT / "oracle" / "_ref" / "L_OpenMP"


def load_package():
    if "lnorms_b200" in sys.modules:
        return sys.modules["lnorms_b200"]
    spec = importlib.util.spec_from_file_location("lnorms_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["lnorms_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_workloads():
    """workloads.py on its own (it needs numpy only), so that the reference
    arm never maps the solver library into its process."""
    name = "lnorms_b200_workloads"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, PKG_DIR / "workloads.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def instance(cfg: int, wide_cols: int = 0, wide_d: int = 1):
    W = load_workloads()
    if wide_cols:
        return W.wide(wide_cols, wide_d)
    return {1: W.config1, 2: W.config2, 3: W.config3, 5: W.config5}[cfg]()


def reduced_shape(inst) -> tuple[int, int]:
    """Rows x columns left by the preprocessing: the generator's core for
    configuration 2 (its planted copies unite and its zero rows vanish), the
    input shape for the configurations without a flag (a d = 1 matrix with
    more rows than columns is transposed)."""
    if "core" in inst.meta:
        return tuple(int(x) for x in inst.meta["core"])
    r, c = inst.matrix.shape
    return (c, r) if inst.d == 1 and r > c else (r, c)


def workload_config(inst) -> dict:
    """The `config` object of the bench line, identical in both arms: what
    the workload is, not how an arm runs it."""
    rows, cols = reduced_shape(inst)
    base = 2 if inst.d <= 2 else inst.d
    labelings = base ** (rows - 1)
    flags = " ".join(inst.argv_tail()[1:]) or "none"
    r0, c0 = inst.matrix.shape
    return {"workload": (f"{inst.name}: {r0}x{c0} integer matrix, d={inst.d}"
                         f"{' with marginals' if inst.marginal else ''}, flags {flags}; preprocessing leaves "
                         f"{rows}x{cols}, {labelings} labelings"),
            "rows": rows, "cols": cols, "d": inst.d, "marginal": bool(inst.marginal), "flags": flags,
            "labelings_per_step": labelings,
            "l2": "GPU arm: flushed between steps (512 MiB write outside the timed events); inputs of a few KB"}


def ops_per_labeling(d: int, cols: int) -> int:
    """Integer work per labeling of the plain incremental method: update +
    |.| + accumulate per column (3m) for L_1/LM; two changed message vectors
    (6m) for d >= 2."""
    return 3 * cols if d == 1 else 6 * cols


def issue_ops_per_labeling(desc: str, d: int, cols: int) -> tuple[int, str]:
    """int32 ALU issue slots the chosen kernel spends per labeling.

    Table kernel: one absolute-difference-accumulate instruction (sad on a
    32-bit lane, vabsdiff4 on four 8-bit lanes) per column word per sum
    vector (D vectors per labeling: 1 for L_1/LM, 2 or 3 for d = 2, 3); both
    issue at half the ALU pipe's add/xor rate, so each costs 2 slots of the
    int32 add/xor peak.  The LM instances that add the marginal column
    linearly skip its word.  Wide kernel: the plain count."""
    f = dict(kv.split("=") for kv in desc.replace("int32 words", "int32_words")
             .replace("int8x4 words", "int8x4_words").split() if "=" in kv)
    if desc.startswith("table") and "int32_words" in f:
        D, wb, wa = int(f["D"]), int(f["int32_words"]), int(f["int8x4_words"])
        if int(f.get("split", 0)) > 0:
            # column split: the words of the actual columns (the padding to
            # S x PW words is not counted as work)
            words = cols if wb > 0 else (cols + 3) // 4
            return 2 * D * words, (f"2 slots x D={D} x {words} {'int32' if wb > 0 else 'int8x4'} words "
                                   f"(column split over {f['split']} lanes, unpadded)")
        if int(f.get("lin", 0)):
            # the LM marginal column is added linearly, once per high index
            return 2 * (D * (wb + wa) - 1), f"2 slots x ({wb - 1} int32 + {wa} int8x4 words; column 0 linear)"
        return 2 * D * (wb + wa), f"2 slots x D={D} x ({wb} int32 + {wa} int8x4 words)"
    return ops_per_labeling(d, cols), "plain count (wide kernel)"


# DRAM traffic of one launch of the config-2 table kernel, from the ncu
# capture summarised in profiles/table_kernel_config2_LM_34x37.md
# (dram__bytes_read.sum + dram__bytes_write.sum); the kernel is ALU-bound and
# reads only its matrix image.
TRAFFIC_BYTES = {2: 62208}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and throttle reasons sampled every 10 ms through NVML (read
    only) while the timed region runs; falls back to `nvidia-smi -lms 200`."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, index: int, interval: float = 0.01):
        import threading
        self.samples, self.reasons = [], set()
        self.sm_max = None
        self.proc = None
        self._stop = threading.Event()
        try:
            import pynvml as N
            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByIndex(index)
            self.sm_max = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))
            get_reasons = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                N.nvmlDeviceGetCurrentClocksThrottleReasons

            def loop():
                while not self._stop.is_set():
                    self.samples.append(float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)))
                    r = get_reasons(h)
                    for nm, bit in self.REASONS.items():
                        if r & bit:
                            self.reasons.add(nm)
                    self._stop.wait(interval)

            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            while not self.samples and self.thread.is_alive():
                time.sleep(0.001)
        except Exception:
            self.thread = None
            self._start_smi(index)

    def _start_smi(self, index):
        fields = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                  "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={index}", f"--query-gpu={fields}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.thread is not None:
            self._stop.set()
            self.thread.join(timeout=2)
            sm = self.samples
            smax = [self.sm_max] if self.sm_max else sm
            reasons = self.reasons
            source = "nvml 10 ms"
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.file.flush()
            rows = [ln.split(",") for ln in Path(self.file.name).read_text().splitlines() if ln.strip()]
            os.unlink(self.file.name)
            sm, smax, reasons = [], [], set()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for r in rows:
                try:
                    sm.append(float(r[1])); smax.append(float(r[2]))
                except (ValueError, IndexError):
                    continue
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            source = "nvidia-smi 200 ms"
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock source"], "samples": 0}
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        loaded = [s for s in sm if s >= 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "source": source}


# ---------------------------------------------------------------- CPU side
def write_matrix(path: Path, a: np.ndarray) -> None:
    path.write_text("".join(" ".join(str(int(v)) for v in row) + "\n" for row in a))


def run_reference_binary(a: np.ndarray, tail: list[str], threads: int) -> tuple[float, str]:
    with tempfile.TemporaryDirectory() as td:
        write_matrix(Path(td) / "m.txt", a)
        t0 = time.perf_counter()
        p = subprocess.run([str(REF_BIN), str(threads), "m.txt", *tail], cwd=td, capture_output=True,
                           text=True, timeout=900)
        dt = time.perf_counter() - t0
    if p.returncode != 0:
        raise RuntimeError(f"reference solver failed: {p.stdout[-300:]} {p.stderr[-300:]}")
    return dt, p.stdout


def reference_sample(inst, ld, target_labelings: int):
    """A bounded sample of the workload for the CPU: the reduced matrix with
    free rows dropped until at most target_labelings remain (same columns,
    so the per-labeling work is the workload's).  Returned as the file the
    reference reads: marginal row first, flag `m` only."""
    p = ld.Problem.from_matrix(inst.matrix, inst.d, inst.stat, inst.marginal)
    info = p.info
    red = p.reduced
    rows = info["rows"]
    base = 2 if info["d"] <= 2 else info["d"]
    keep = rows
    while keep > 1 and base ** (keep - 1) > target_labelings:
        keep -= 1
    sub = np.concatenate([red[: keep - 1], red[-1:]], axis=0)   # fixed row stays last
    labelings = base ** (keep - 1)
    if info["marginal"]:
        a = np.concatenate([sub[-1:], sub[:-1]], axis=0)         # the reference swaps it back
        tail = [str(info["d"]), "m"]
    else:
        a, tail = sub, [str(info["d"])]
    return a, tail, labelings, f"reduced {inst.name} cut to {keep} rows x {info['cols']} cols"


def cpu_baseline(inst, ld, target_seconds: float = 15.0) -> dict:
    """The reference's L_OpenMP on this host's cores: the full input file
    when that takes at most about twice target_seconds (configuration 2:
    about 4-11 s), else a bounded sample of the reduced matrix."""
    threads = os.cpu_count() or 1
    # calibrate on a small sample, then size the timed sample to ~target_seconds
    a, tail, n0, _ = reference_sample(inst, ld, 1 << 24)
    if REF_BIN.exists():
        t0, _ = run_reference_binary(a, tail, threads)
        rate = n0 / max(t0, 1e-3)
        cfg = workload_config(inst)
        n = cfg["labelings_per_step"]
        if n / rate <= 2 * target_seconds:
            t, out = run_reference_binary(inst.matrix, inst.argv_tail(), threads)
            value_line, rows, cols = reference_output(out)
            return {"value": n / t, "unit": "labelings/s", "cores": threads, "kind": "reference",
                    "sample": f"L_OpenMP.c built from the reference sources, {threads} threads, the full "
                              f"{inst.name} input file with flags {cfg['flags']} ({rows}x{cols} after its "
                              f"preprocessing, {n} labelings, value {value_line}, {t:.2f} s)"}
        a, tail, n, what = reference_sample(inst, ld, int(rate * target_seconds))
        t, _ = run_reference_binary(a, tail, threads)
        return {"value": n / t, "unit": "labelings/s", "cores": threads, "kind": "reference",
                "sample": f"L_OpenMP.c built from the reference sources, {threads} threads, {what} "
                          f"({n} labelings, {t:.2f} s)"}
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ffi as O   # the oracle restatement, when the reference binary is absent
    red_p = ld.Problem.from_matrix(inst.matrix, inst.d, inst.stat, inst.marginal)
    info = red_p.info
    red = red_p.reduced
    t0 = time.perf_counter()
    O.enumerate_max(red, info["d"], bool(info["marginal"]), 0, 1 << 24, threads)
    rate = (1 << 24) / max(time.perf_counter() - t0, 1e-3)
    n = int(min(O.total(info["rows"], info["d"]), rate * target_seconds))
    t0 = time.perf_counter()
    O.enumerate_max(red, info["d"], bool(info["marginal"]), 0, n, threads)
    t = time.perf_counter() - t0
    return {"value": n / t, "unit": "labelings/s", "cores": threads, "kind": "port",
            "sample": f"oracle restatement, {threads} threads, first {n} labelings of {inst.name}"}


def reference_output(stdout: str) -> tuple[int, int, int]:
    """(value, reduced rows, reduced columns) from the reference's stdout:
    the `L.. is: v` line and the preprocessing messages (functions.h:76,
    131-285): each removed zero line and each line united into another
    takes one row or column off the matrix as read; a transposed matrix
    swaps the two."""
    value, rows, cols, dr, dc, transposed = None, None, None, 0, 0, False
    gone = ("entries are zeros", "was added to", "was subtracted from")
    for ln in stdout.splitlines():
        s = ln.strip()
        if s.startswith("rows:") and "cols:" in s:
            rows = int(s.split(",")[0].split(":")[1])
            cols = int(s.split("cols:")[1])
        elif " is: " in s:
            value = int(s.split(" is: ")[1])
        elif s.startswith(("row ", "col ")) and any(m in s for m in gone):
            if s.startswith("row "):
                dr += 1
            else:
                dc += 1
        elif s == "The entries of the first row and column are zeros.":
            dr, dc = dr + 1, dc + 1   # the zero marginal row and column are dropped
        elif s == "Matrix was transposed.":
            transposed = True
    if value is None or rows is None:
        raise RuntimeError(f"unexpected reference output: {stdout[-300:]}")
    rows, cols = rows - dr, cols - dc
    return (value, cols, rows) if transposed else (value, rows, cols)


def run_reference_arm(args) -> None:
    """The reference's own OpenMP solver (L_OpenMP.c, compiled unmodified
    from its sources into oracle/_ref/) on the full workload: each step runs
    it once on the configuration's input file with the configuration's
    flags (`L_OpenMP threads m.txt 1 y m` for configuration 2), so it reads,
    preprocesses and enumerates every labeling itself.  This process loads
    numpy and the workload generator only, never the solver library."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    if args.config == 4 or args.method != "plain":
        print(json.dumps({"impl": "reference", "unavailable": "the reference solves one matrix per process "
                          "by plain enumeration; it has no batched or pruned form"}))
        return
    if not REF_BIN.exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/L_OpenMP was not built "
                          "(make -C oracle needs the reference sources)"}))
        return
    inst = instance(args.config, args.wide, args.wide_d)
    cfg = workload_config(inst)
    threads = os.cpu_count() or 1
    tail = inst.argv_tail()
    outs = []
    for _ in range(args.warmup):
        run_reference_binary(inst.matrix, tail, threads)
    times = []
    for _ in range(args.steps):
        dt, out = run_reference_binary(inst.matrix, tail, threads)
        times.append(dt)
        outs.append(reference_output(out))
    value_line, rows, cols = outs[-1]
    if (rows, cols) != (cfg["rows"], cfg["cols"]) or any(o != outs[0] for o in outs):
        raise RuntimeError(f"reference reduced the workload to {rows}x{cols} (expected {cfg['rows']}x"
                           f"{cfg['cols']}) or its steps disagree: {outs[:3]}")
    total = sum(times)
    n = cfg["labelings_per_step"]
    value = n * args.steps / total
    sample = (f"L_OpenMP.c compiled unmodified from the reference sources, {threads} threads, the full "
              f"{inst.name} input file with flags {cfg['flags']} per step ({n} labelings after its own "
              f"preprocessing; printed value {value_line}); whole-process wall clock")
    line = {
        "impl": "reference", "metric": "exact L_d labelings/s (plain enumeration)", "value": value,
        "unit": "labelings/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator of the configuration)",
        "config": cfg,
        "cpu_baseline": {"value": value, "unit": "labelings/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "labelings/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "details": {"value": value_line, "reduced": [rows, cols]},
    }
    print(json.dumps(line))


REF_GPU_BIN = ROOT / "oracle" / "_ref" / "L_CUDA"


def run_reference_gpu(args) -> None:
    """The reference's own CUDA solver (L_CUDA.cu built for sm_100a from its
    sources) on the same workload file and flags, timed as its README times
    it: wall clock of the whole process.  Its launch shape (blocks x
    threads, CLI arguments) is swept and the fastest kept.  The process's
    fixed cost (CUDA context, parsing) is measured on a 2 x 2 matrix and
    reported, and subtracted in `value_minus_startup`."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.config == 4 or args.method != "plain":
        print(json.dumps({"impl": "reference-gpu", "unavailable": "the reference solves one matrix per "
                          "process by plain enumeration"}))
        return
    if not REF_GPU_BIN.exists():
        print(json.dumps({"impl": "reference-gpu", "unavailable": "oracle/_ref/L_CUDA was not built "
                          "(make -C oracle needs the reference sources)"}))
        return
    ld = load_package()
    inst = instance(args.config)
    info = ld.Problem.from_matrix(inst.matrix, inst.d, inst.stat, inst.marginal).info
    tail = inst.argv_tail()

    def run(a, blocks, threads, tail_args):
        with tempfile.TemporaryDirectory() as td:
            write_matrix(Path(td) / "m.txt", a)
            t0 = time.perf_counter()
            p = subprocess.run([str(REF_GPU_BIN), str(blocks), str(threads), "m.txt", *tail_args], cwd=td,
                               capture_output=True, text=True, timeout=600)
            dt = time.perf_counter() - t0
        if p.returncode != 0:
            raise RuntimeError(f"reference GPU solver failed: {p.stdout[-300:]} {p.stderr[-300:]}")
        return dt, p.stdout

    startup = min(run(np.array([[1, 2], [3, 4]]), 1, 1, ["1"])[0] for _ in range(3))
    shapes = [(512, 32), (148 * 8, 128), (148 * 16, 128), (148 * 32, 256), (148 * 64, 256)]
    if args.ref_launch:
        shapes = [tuple(int(x) for x in args.ref_launch.split("x"))]
    sweep = {}
    for b, t in shapes:
        dt, out = run(inst.matrix, b, t, tail)
        sweep[f"{b}x{t}"] = dt
        if dt > 120:
            break
    best = min(sweep, key=sweep.get)
    b, t = (int(x) for x in best.split("x"))
    for _ in range(args.warmup):
        run(inst.matrix, b, t, tail)
    times, out = [], ""
    for _ in range(args.steps):
        dt, out = run(inst.matrix, b, t, tail)
        times.append(dt)
    value_line = next((ln for ln in out.splitlines() if " is: " in ln), "")
    wall = statistics.mean(times)
    n = int(info["labelings"])
    line = {
        "impl": "reference-gpu", "metric": "exact L_d labelings/s (plain enumeration)", "value": n / wall,
        "unit": "labelings/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * wall, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic (seeded generator of the configuration)",
        "config": {"workload": workload_name(inst, info), "launch": best, "sweep_s": sweep,
                   "output": value_line.strip()},
        "value_minus_startup": n / max(wall - startup, 1e-6), "startup_s": startup,
        "note": "L_CUDA.cu compiled from the reference sources for sm_100a (oracle/_ref/L_CUDA); whole-process "
                "wall clock, as the reference's README measures it",
    }
    print(json.dumps(line))


def workload_name(inst, info) -> str:
    return (f"{inst.name}: d={info['d_user']}{' marginal' if info['marginal_user'] else ''}, "
            f"flag {inst.stat}, {info['rows_in']}x{info['cols_in']} -> {info['rows']}x{info['cols']}, "
            f"{info['labelings']} labelings")


# ---------------------------------------------------------------- GPU side
class DeviceView:
    """Zero-copy view of a device int64 pair (the plan's result slot)."""

    def __init__(self, ptr: int):
        self.__cuda_array_interface__ = {"shape": (2,), "typestr": "<i8", "data": (ptr, False),
                                         "version": 3, "strides": None}


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    ld = load_package()
    import lnorms_b200.distributed as D
    inst = instance(args.config, args.wide, args.wide_d)
    cfg = workload_config(inst)
    prob = ld.Problem.from_matrix(inst.matrix, inst.d, inst.stat, inst.marginal)
    info = prob.info
    red = prob.reduced
    d, marg = info["d"], bool(info["marginal"])
    if (info["rows"], info["cols"], int(info["labelings"])) != (cfg["rows"], cfg["cols"], cfg["labelings_per_step"]):
        raise RuntimeError(f"preprocessing left {info['rows']}x{info['cols']}, the workload says "
                           f"{cfg['rows']}x{cfg['cols']}")
    knobs = dict(column_split=args.column_split, walk_fetch=args.walk_fetch, pack16=args.pack16,
                 paired_walks=args.paired_walks, tile=args.tile)
    opts = ld.options(device=local, shard_index=rank, shard_count=world, **knobs)
    plan = ld.Plan(red, d, marg, opts)
    lo, hi = plan.range
    total_labelings = info["labelings"]
    stream = torch.cuda.ExternalStream(plan.stream, device=torch.device("cuda", local))
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")   # > 126 MB L2

    def step():
        plan.launch()

    # the cross-rank (value, Gray index) combine: distributed.combine_tensor,
    # on the plan's device result slot, queued on the solver's stream
    combine = D.combine_tensor

    # the plan's result slot, viewed as a tensor for the cross-rank combine
    res_view = None
    if world > 1:
        res_view = torch.as_tensor(DeviceView(plan.result_device_ptr), device="cuda")

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
            if world > 1:
                combine(res_view)
                dist.barrier()
        sol0 = plan.result() if args.warmup else None
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        for i in range(args.steps):
            starts[i].record(stream)
            step()
            if world > 1:
                combine(res_view)
            stops[i].record(stream)
            flush.fill_(i & 0xFF)   # outside the timed events, same stream
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        clk = clocks.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, stops)]
    my_total = sum(step_ms)
    t = torch.tensor([my_total], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    sol = plan.result()
    value = total_labelings * args.steps / (total_ms * 1e-3)

    # end to end through the public API: host matrix in, value + strategy out
    e2e_ms, h2d, d2h = [], 0, 0
    for i in range(args.warmup + args.steps):
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        p = ld.Problem.from_matrix(inst.matrix, inst.d, inst.stat, inst.marginal)
        res = p.solve(ld.options(device=local, shard_index=rank, shard_count=world, **knobs))
        if world > 1:
            res.value, res.gray_index = D.combine(int(res.value), int(res.gray_index),
                                                  device=torch.device("cuda", local))
        p.report(res)
        dt = (time.perf_counter() - t0) * 1e3
        if i >= args.warmup:
            e2e_ms.append(dt)
            h2d, d2h = int(res.h2d_bytes), int(res.d2h_bytes)
    e2e_t = torch.tensor([sum(e2e_ms)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = total_labelings * args.steps / (float(e2e_t.item()) * 1e-3)

    if rank == 0:
        kernel_ms = statistics.mean(step_ms)
        desc = plan.describe()
        opl = ops_per_labeling(d, info["cols"])
        iopl, iwhat = issue_ops_per_labeling(desc, d, info["cols"])
        peak_ops, _ = ld.int32_peak(local)
        # labelings the kernel computed a value for (d >= 3: the walks that
        # hold no smallest index of a label-permutation class are skipped)
        evaluated = int(sol.evaluated)
        rate = evaluated / (kernel_ms * 1e-3)
        achieved = iopl * rate
        line = {
            "metric": "exact L_d labelings/s (plain enumeration)", "value": value, "unit": "labelings/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generator of the configuration)",
            "config": cfg,
            "details": {"evaluated_per_step": evaluated if world == 1 else None,
                        "label_symmetry": (f"{evaluated / (hi - lo):.4f} of the labelings evaluated: walks that "
                                           f"hold no smallest index of a class under permutations of labels "
                                           f"1..{d - 1} are skipped") if d >= 3 and evaluated < hi - lo else None,
                        "parallelism": f"gray-index shards x{world}" if world > 1 else "single GPU",
                        "kernel": desc, "value": sol.value, "gray_index": sol.gray_index},
            "roofline": {"bound": "int32", "achieved": achieved / 1e12, "peak": peak_ops / 1e12,
                         "unit": "Tops/s", "frac": achieved / peak_ops,
                         "traffic": TRAFFIC_BYTES.get(args.config) if world == 1 and not args.wide else None,
                         "ops_per_labeling": iopl,
                         "plain_method": {"ops_per_labeling": opl, "achieved": opl * rate / 1e12,
                                          "x_peak": opl * rate / peak_ops},
                         "note": f"achieved = {iopl} int32 issue slots per labeling ({iwhat}) x evaluated "
                                 f"labelings/s; "
                                 f"peak = int32 add/xor microbenchmark measured in this run; plain_method "
                                 f"counts the {'3m' if d == 1 else '6m'} ops the plain enumeration spends per "
                                 f"labeling (m={info['cols']}), which the table decomposition avoids"},
            "e2e": {"value": e2e_value, "unit": "labelings/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": statistics.mean(e2e_ms)},
            "gpu_launches": args.steps,
            "clocks": clk,
        }
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_baseline(inst, ld)
        if world == 1 and args.config5_count > 0:
            line["config5"] = config5_leg(ld, local, args.config5_count, steps=3, warmup=2)
        assert sol0 is None or (sol0.value == sol.value and sol0.gray_index == sol.gray_index)
        print(json.dumps(line))
    plan.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def config5_leg(ld, local: int, count: int, steps: int, warmup: int) -> dict:
    """The metric's other half, on configuration 5 (44x44 low rank, L_1,
    2^43 labelings): one plain enumeration against the exact learned-pruned
    search, batched over `count` matrices of the same distribution (seeds
    5 .. 5 + count - 1; seed 5 is configuration 5 itself), with network
    proposals and, as the method without the network, uniform random ones,
    8 proposals per matrix and (`budget_2`) 2.
    Times are wall clock per matrix from host matrix to host answer, taken
    after the configuration-2 events; the answer for configuration 5 must
    equal the plain enumeration's (value and Gray index)."""
    import lnorms_b200.learned as L

    W = load_workloads()
    inst = W.config5()
    red = ld.Problem.from_matrix(inst.matrix, inst.d, inst.stat, inst.marginal).reduced
    plan = ld.Plan(red, 1, False, ld.options(device=local))
    t0 = time.perf_counter()
    ref = plan.solve()
    plain_s = time.perf_counter() - t0
    desc = plan.describe()
    plan.close()
    mats = [ld.Problem.from_matrix(W.config5(seed=5 + i).matrix, 1).reduced for i in range(count)]
    total = 2 ** (red.shape[0] - 1)
    out = {"workload": f"{inst.name}: {red.shape[0]}x{red.shape[1]}, {total} labelings per matrix",
           "plain": {"s_per_matrix": plain_s, "kernel_ms": ref.kernel_ms, "labelings_per_s": total / plain_s,
                     "kernel": desc, "value": ref.value, "gray_index": ref.gray_index},
           "batch": count, "proposals_per_matrix": 8}
    runs = [(8, "network", "learned_pruned", out), (8, "random", "random_pruned", out)]
    small = {"proposals_per_matrix": 2}
    runs += [(2, "network", "learned_pruned", small), (2, "random", "random_pruned", small)]
    for budget, mode, key, dst in runs:
        proposer = L.Proposer(mode, directions=budget, samples=1, device=local)
        for _ in range(warmup):
            res = L.solve_learned_batch(mats, proposer)
        walls = []
        for _ in range(steps):
            t0 = time.perf_counter()
            res = L.solve_learned_batch(mats, proposer)
            walls.append(time.perf_counter() - t0)
        proposer.close()
        first = res[0][0]
        if (first.value, first.gray_index) != (ref.value, ref.gray_index):
            raise AssertionError(f"{key}: {(first.value, first.gray_index)} != plain "
                                 f"{(ref.value, ref.gray_index)}")
        ms = 1e3 * statistics.mean(walls) / count
        dst[key] = {"ms_per_matrix": ms, "speedup_vs_plain": plain_s * 1e3 / ms,
                    "labelings_per_s": total / (ms * 1e-3),
                    "walks_kept_mean": statistics.mean(r[1]["prune_walks_kept"] for r in res),
                    "incumbent_optimal": sum(int(r[1]["incumbent"] == r[0].value) for r in res)}
    out["budget_2"] = small
    out["target"] = "learned-pruned >= 5x faster than the plain GPU enumeration"
    return out


def run_batch(args) -> None:
    """The 4096-matrix batch (n in [16, 32], m in [16, 64], d in {1, 2, 3}):
    one step = one replay of the batch's CUDA graph (persistent kernels per
    lane class over a device work queue).  The d = 3 matrices with more than
    3^20 labelings (the tail: about 2.2e16 labelings, 251 matrices) stay out
    of the replay.  value = labelings of the replayed matrices per second of
    device time.  Outside the timed region every replayed result is checked
    against a single solve (ld_solve_reduced) of the same matrix, and with
    --tail-rows N every tail matrix of at most N rows is solved exactly, one
    solve each; the rest of the tail is listed with its labelings and the
    time the measured d = 3 rate gives it."""
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    ld = load_package()
    W = load_workloads()
    mats, ds, total, slots = [], [], 0, 0
    tail = []   # (index in the workload, reduced matrix, labelings)
    for idx, inst in enumerate(W.config4()[: args.batch_count or None]):
        p = ld.Problem.from_matrix(inst.matrix, inst.d)
        info = p.info
        if info["d"] == 3 and info["labelings"] > 3 ** 20:
            tail.append((idx, p.reduced, int(info["labelings"])))
            continue
        mats.append(p.reduced)
        ds.append(info["d"])
        total += int(info["labelings"])
    opts = ld.options(device=local, batch_split=args.batch_split, threads_per_block=args.batch_tpb)
    t0 = time.perf_counter()
    b = ld.Batch(mats, ds, opts=opts, autotune=True)
    create_s = time.perf_counter() - t0
    # int32 issue slots: one sad (2 slots) per column per sum vector (all of
    # this workload's sums need 32-bit lanes) per labeling the kernels
    # evaluate (d = 3: label symmetry skips about half)
    evaluated = b.evaluated()
    slots = sum(2 * dd * m.shape[1] * int(e) for dd, m, e in zip(ds, mats, evaluated))
    n_eval = int(evaluated.sum())
    for _ in range(args.warmup):
        v0, g0, _ = b.solve()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    ms = []
    for _ in range(args.steps):
        v, g, t = b.solve()
        ms.append(t)
    clk = clocks.stop()
    assert np.array_equal(v, v0) and np.array_equal(g, g0)
    desc = b.describe()
    b.close()
    # end to end through the public API: host matrices in, values out
    e2e = []
    for _ in range(max(1, min(args.steps, 3))):
        t0 = time.perf_counter()
        bb = ld.Batch(mats, ds, opts=opts, autotune=True)
        ve, ge, _ = bb.solve()
        bb.close()
        e2e.append(time.perf_counter() - t0)
        assert np.array_equal(ve, v0)
    # full-scale check: every replayed result against a single solve
    t0 = time.perf_counter()
    bad = []
    for i, (m, dd) in enumerate(zip(mats, ds)):
        sol = ld.solve_reduced(m, dd, False, ld.options(device=local))
        if (sol.value, sol.gray_index) != (int(v0[i]), int(g0[i])):
            bad.append(i)
    check_s = time.perf_counter() - t0
    if bad:
        raise AssertionError(f"{len(bad)} batch results differ from single solves, first {bad[:5]}")
    # the d = 3 tail: exact single solves up to --tail-rows rows
    tail_out = None
    if tail:
        solved, rest = [], []
        skip = {int(x) for x in args.tail_skip.split(",") if x.strip()}
        for idx, m, lab in sorted(tail, key=lambda x: x[2]):
            if idx in skip:
                continue
            if args.tail_min_rows <= m.shape[0] <= args.tail_rows:
                t0 = time.perf_counter()
                sol = ld.solve_reduced(m, 3, False, ld.options(device=local))
                solved.append({"index": idx, "rows": m.shape[0], "cols": m.shape[1], "labelings": lab,
                               "value": sol.value, "gray_index": sol.gray_index, "kernel_ms": sol.kernel_ms,
                               "wall_s": time.perf_counter() - t0})
                if args.tail_out:   # after every solve, so that a stopped run keeps what it solved
                    Path(args.tail_out).write_text(json.dumps({"solved": solved}, indent=1))
            elif m.shape[0] > args.tail_rows:
                rest.append({"index": idx, "rows": m.shape[0], "cols": m.shape[1], "labelings": lab})
        rate = (sum(x["labelings"] for x in solved) / max(1e-9, sum(x["kernel_ms"] for x in solved) * 1e-3)
                if solved else None)
        if rate:   # cost of each remaining matrix at the measured rate, scaled by columns
            mean_cols = sum(x["cols"] for x in solved) / len(solved)
            for x in rest:
                x["est_s"] = x["labelings"] / rate * (x["cols"] / mean_cols)
        tail_out = {"matrices": len(tail), "labelings": sum(x[2] for x in tail),
                    "solved": len(solved), "solved_labelings": sum(x["labelings"] for x in solved),
                    "solved_kernel_s": sum(x["kernel_ms"] for x in solved) * 1e-3,
                    "solved_wall_s": sum(x["wall_s"] for x in solved),
                    "rate_labelings_per_s": rate, "max_rows_solved": args.tail_rows,
                    "remaining": len(rest), "remaining_labelings": sum(x["labelings"] for x in rest),
                    "remaining_est_s": sum(x.get("est_s", 0.0) for x in rest)}
        if args.tail_out:
            Path(args.tail_out).write_text(json.dumps({"summary": tail_out, "solved": solved, "remaining": rest},
                                                      indent=1))
    if rank != 0:
        return
    dev_s = sum(ms) * 1e-3
    h2d = sum(m.size * 8 for m in mats)
    peak_ops, _ = ld.int32_peak(local)
    achieved = slots * args.steps / dev_s
    line = {
        "metric": "exact L_d labelings/s (batched solves)", "value": total * args.steps / dev_s,
        "unit": "labelings/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dev_s / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator of the configuration)",
        "config": {"workload": f"config4: {len(mats)} of {args.batch_count or 4096} matrices, {total} labelings",
                   "matrices": len(mats), "labelings_per_step": total, "evaluated_per_step": n_eval,
                   "tail": {"matrices": len(tail), "labelings": sum(x[2] for x in tail),
                            "why": "d = 3 with more than 3^20 labelings: solved one by one outside the replay"},
                   "batch": desc, "create_s": create_s,
                   "l2": "not flushed: the batch's inputs are a few MB and stay resident"},
        "checked_against_single_solves": {"matrices": len(mats), "mismatches": 0, "s": check_s},
        "tail": tail_out,
        "e2e": {"value": total / statistics.mean(e2e), "unit": "labelings/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": len(mats) * 16, "s_per_step": statistics.mean(e2e)},
        "roofline": {"bound": "int32", "achieved": achieved / 1e12, "peak": peak_ops / 1e12, "unit": "Tops/s",
                     "frac": achieved / peak_ops, "traffic": None, "ops_per_labeling": slots / max(n_eval, 1),
                     "note": "2 int32 issue slots (one sad) per column per sum vector per evaluated labeling, unpadded "
                             "columns, averaged over the batch; peak = int32 add/xor microbenchmark measured "
                             "in this run"},
        # per replay: one persistent kernel per lane class, the fold, and the own plans' kernels
        "gpu_launches": len(ms) * (int(desc.split(" classes")[0].split()[-1]) + 1
                                   + int(desc.split(" own plans")[0].split()[-1])),
        "clocks": clk,
    }
    print(json.dumps(line))


def run_search_batch(args, ld, L, inst, info, proposer, local, world, rank) -> None:
    """`--count N`: N independent matrices of the workload's distribution
    (seeds 5 .. 5 + N - 1 of the generator) solved exactly per step, the
    network's proposals for all of them from one forward pass."""
    import lnorms_b200.workloads as W
    mats = [W.config5(seed=5 + i).matrix for i in range(args.count)]
    for _ in range(args.warmup):
        ref = L.solve_learned_batch(mats, proposer)
    clocks = ClockSampler(local)
    walls = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        res = L.solve_learned_batch(mats, proposer)
        walls.append(time.perf_counter() - t0)
    clk = clocks.stop()
    proposer.close()
    for (s0, _), (s1, _) in zip(ref, res):
        assert (s0.value, s0.gray_index) == (s1.value, s1.gray_index)
    if rank != 0:
        return
    wall = sum(walls)
    total = info["labelings"] * args.count
    line = {
        "metric": f"exact L_1 labelings/s ({args.method} search, batched)", "value": total * args.steps / wall,
        "unit": "labelings/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * wall / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator of the configuration)",
        "config": {"workload": f"{args.count} matrices of {inst.name}'s distribution (seeds 5..{4 + args.count})",
                   "labelings_per_step": total, "proposals_per_matrix": proposer.count(),
                   "ms_per_matrix": 1e3 * wall / args.steps / args.count,
                   "values": [r[0].value for r in res][:8]},
        "e2e": {"value": total * args.steps / wall, "unit": "labelings/s"},
        "roofline": None,
        "clocks": clk,
    }
    print(json.dumps(line))


def run_search(args) -> None:
    """Exact solve by the pruned enumeration with an incumbent from
    local-search-polished proposals: `--method learned` (the trained
    network's proposals) or `--method pruned` (uniform random proposals, the
    method without the network).  One step = one exact solve of the
    workload from host matrix to host answer; value = labelings the solve
    covers (all of them, enumerated or proved dominated) per second."""
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ld = load_package()
    import lnorms_b200.learned as L
    inst = instance(args.config)
    prob = ld.Problem.from_matrix(inst.matrix, inst.d, inst.stat, inst.marginal)
    info = prob.info
    red = prob.reduced
    if info["d"] != 1 or info["marginal"]:
        raise SystemExit("the learned search handles L_1 without marginals")
    mode = "network" if args.method == "learned" else "random"
    proposer = L.Proposer(mode, directions=args.proposals, samples=1, device=local)
    if args.count > 1:
        run_search_batch(args, ld, L, inst, info, proposer, local, world, rank)
        return
    for _ in range(args.warmup):
        sol0, _ = L.solve_learned(red, proposer)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    walls, stats = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        sol, st = L.solve_learned(red, proposer)
        walls.append(time.perf_counter() - t0)
        stats.append(st)
    clk = clocks.stop()
    count = proposer.count()
    proposer.close()
    assert (sol.value, sol.gray_index) == (sol0.value, sol0.gray_index)
    total = info["labelings"]
    plain = None
    if args.with_plain:
        plan = ld.Plan(red, 1, False, ld.options(device=local))
        t0 = time.perf_counter()
        ref = plan.solve()
        plain = {"wall_s": time.perf_counter() - t0, "kernel_ms": ref.kernel_ms,
                 "value": ref.value, "gray_index": ref.gray_index}
        plan.close()
        assert (ref.value, ref.gray_index) == (sol.value, sol.gray_index)
    if rank != 0:
        return
    last = stats[-1]
    wall = sum(walls)
    line = {
        "metric": f"exact L_1 labelings/s ({args.method} search)", "value": total * args.steps / wall,
        "unit": "labelings/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * wall / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator of the configuration)",
        "config": {"workload": workload_name(inst, info), "rows": info["rows"], "cols": info["cols"], "d": 1,
                   "labelings_per_step": total, "proposals": count, "proposal_mode": mode,
                   "value": sol.value, "gray_index": sol.gray_index,
                   "l2": "not flushed: every step re-uploads its inputs from host memory"},
        "breakdown_ms": {"incumbent": 1e3 * statistics.mean(s["incumbent_s"] for s in stats),
                         "pruned_total": 1e3 * statistics.mean(s["pruned_s"] for s in stats),
                         "bound_kernel": statistics.mean(s["prune_bound_ms"] for s in stats),
                         "scan_kernel": statistics.mean(s["prune_scan_ms"] for s in stats)},
        "search": {"incumbent": last["incumbent"], "raw_best": last["raw_best"],
                   "walks_total": last["prune_walks_total"], "walks_kept": last["prune_walks_kept"],
                   "highs_total": last["prune_highs_total"], "highs_kept": last["prune_highs_kept"],
                   "low_rows": last["prune_low_rows"], "walk_rows": last["prune_walk_rows"]},
        "e2e": {"value": total * args.steps / wall, "unit": "labelings/s",
                "h2d_bytes_per_step": int(sol.h2d_bytes), "d2h_bytes_per_step": int(sol.d2h_bytes)},
        "roofline": None,
        "clocks": clk,
    }
    if plain:
        line["plain_gpu"] = plain
        line["speedup_vs_plain_gpu"] = plain["wall_s"] / (wall / args.steps)
    print(json.dumps(line))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", type=int, default=2, choices=[1, 2, 3, 4, 5],
                    help="workload; 4 runs the batched solver over the 4096-matrix batch")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"])
    ap.add_argument("--wide", type=int, default=0,
                    help="plain runs: instead of a configuration, a seeded matrix with this many columns "
                         "(the column-split table kernel's workload)")
    ap.add_argument("--wide-d", type=int, default=1, help="order d of the --wide matrix")
    for knob, what in (("column-split", "lanes per high index (2, 4, 8; -1 never; 0 auto)"),
                       ("walk-fetch", "0 warps fetch walks from a counter, -1 fixed split"),
                       ("pack16", "0 packed 16-bit maxima when values allow, -1 never"),
                       ("paired-walks", "0 two high indices per thread when possible, -1 never"),
                       ("tile", "high-row digits per walk (0 auto)")):
        ap.add_argument(f"--{knob}", type=int, default=0, help=f"plain runs, table kernel knob: {what}")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--method", default="plain", choices=["plain", "pruned", "learned"],
                    help="plain enumeration (the headline), or the exact pruned search with an "
                         "incumbent from random (pruned) or network (learned) proposals")
    ap.add_argument("--proposals", type=int, default=8, help="proposals per solve (pruned / learned)")
    ap.add_argument("--count", type=int, default=1,
                    help="pruned / learned: solve this many matrices of the workload's distribution per step")
    ap.add_argument("--batch-split", type=int, default=0, choices=(-1, 0, 1),
                    help="config 4: column-split instances of the wide int32 classes "
                         "(0 = the autotuner picks, 1 = always, -1 = never)")
    ap.add_argument("--batch-tpb", type=int, default=0, choices=(0, 64, 128),
                    help="config 4: threads per CTA of every lane class (0 = the autotuner picks)")
    ap.add_argument("--tail-rows", type=int, default=0,
                    help="config 4: also solve the d = 3 tail matrices of at most this many rows, one by one")
    ap.add_argument("--tail-min-rows", type=int, default=0,
                    help="config 4: solve only the tail matrices with at least this many rows (a later part)")
    ap.add_argument("--tail-skip", default="",
                    help="config 4: comma-separated workload indices of tail matrices solved in an earlier part")
    ap.add_argument("--tail-out", default="", help="config 4: write the tail's per-matrix results to this JSON file")
    ap.add_argument("--batch-count", type=int, default=0,
                    help="config 4: the first N of the 4096 matrices (0 = all; for small profiling runs)")
    ap.add_argument("--ref-launch", default="",
                    help="reference-gpu: blocks x threads to use (e.g. 9472x256) instead of the sweep")
    ap.add_argument("--config5-count", type=int, default=32,
                    help="plain runs: also time configuration 5, plain against the batched learned- and "
                         "random-pruned exact search over this many matrices (0 = skip)")
    ap.add_argument("--with-plain", action="store_true",
                    help="also time one plain enumeration of the workload (pruned / learned)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.impl == "reference-gpu":
        run_reference_gpu(args)
    elif args.config == 4:
        run_batch(args)
    elif args.method != "plain":
        run_search(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
