#!/usr/bin/env python
"""Benchmark: bitmask stream compaction throughput on B200.

Default workload (N=1): one column of n = 2^28 float32 with an iid Bernoulli(0.5) mask
(LSB-first uint32 words), compacted by the library's plain call. One step = one
compaction of that column with inputs resident in HBM.

  metric : compaction GB/s, algorithmic bytes per call B = n*w + ceil(n/8) + count*w
           (payload read + mask read + selected payload written) over the step time
  e2e    : the same metric through the host-buffer entry path: pinned host payload and
           mask copied in, compaction, count and selected payload copied back, per step;
           beside it the time of the step's copies alone (pcie_bound_ms), its bound
  --impl reference : the reference's own CPU compaction (generate_validation,
           src/data_generator.cuh:171-188, compiled from its sources into
           oracle/_ref/libcsref.so) on all host threads, same metric, bounded sample.

Multi-GPU (torchrun, one rank per GPU): every rank compacts its own column; there is no
data-path collective (the column shards with no exchange), scaling is weak, the step
time is the max over ranks and value = total bytes of all ranks / that time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "compaction GB/s (payload read + mask read + selected written) per single call"
UNIT = "GB/s"

WORKLOADS = {
    # name: (n, elem_bytes, float_unit, mask kind, mask param)
    "f32_n2^28_p0.5": (1 << 28, 4, True, "bernoulli", 0.5),
    "f32_n2^26_p0.5": (1 << 26, 4, True, "bernoulli", 0.5),
    "f32_n2^28_p0.001": (1 << 28, 4, True, "bernoulli", 0.001),
    "f32_n2^28_p0.01": (1 << 28, 4, True, "bernoulli", 0.01),
    "f32_n2^28_p0.1": (1 << 28, 4, True, "bernoulli", 0.1),
    "f32_n2^28_p0.9": (1 << 28, 4, True, "bernoulli", 0.9),
    "f32_n2^28_p0.99": (1 << 28, 4, True, "bernoulli", 0.99),
    "u32_n2^20_p0.5": (1 << 20, 4, False, "bernoulli", 0.5),
    # short columns (the size sweep below configuration 1's and above it)
    "u32_n2^16_p0.5": (1 << 16, 4, False, "bernoulli", 0.5),
    "u32_n2^18_p0.5": (1 << 18, 4, False, "bernoulli", 0.5),
    "u32_n2^22_p0.5": (1 << 22, 4, False, "bernoulli", 0.5),
    "u32_n2^24_p0.5": (1 << 24, 4, False, "bernoulli", 0.5),
    "u8_n2^22_p0.5": (1 << 22, 1, False, "bernoulli", 0.5),
    "u64_n2^20_p0.5": (1 << 20, 8, False, "bernoulli", 0.5),
    "u8_n2^29_runs8": (1 << 29, 1, False, "runs", 8.0),
    "u16_n2^29_runs64": (1 << 29, 2, False, "runs", 64.0),
    "u32_n2^29_runs4096": (1 << 29, 4, False, "runs", 4096.0),
    "u64_n2^29_runs64": (1 << 29, 8, False, "runs", 64.0),
    "u64_n2^29_dense10": (1 << 29, 8, False, "dense", 0.1),
    "u8_n2^29_p0.5": (1 << 29, 1, False, "bernoulli", 0.5),
    "u16_n2^29_p0.5": (1 << 29, 2, False, "bernoulli", 0.5),
    "u32_n2^29_p0.5": (1 << 29, 4, False, "bernoulli", 0.5),
    "u64_n2^29_p0.5": (1 << 29, 8, False, "bernoulli", 0.5),
    "u8_n2^27_p0.5": (1 << 27, 1, False, "bernoulli", 0.5),  # u8 case small enough for a full ncu capture
    # periodic selection (no mask in memory): pattern 0b10110010 over 8 elements, p = 0.5
    "f32_n2^28_pattern8": (1 << 28, 4, True, "pattern", (0b10110010, 8)),
    # selection evaluated on the device from the payload: x > 0.5 over uniform [0, 1), p = 0.5
    "f32_n2^28_pred_gt0.5": (1 << 28, 4, True, "predicate", (">", 0.5)),
}
DEFAULT_WORKLOAD = "f32_n2^28_p0.5"
BATCH_WORKLOAD = "batch256"  # 256 uneven columns in one plan (lengths log-uniform [2^10, 2^24])
SERVE_WORKLOAD = "serve"  # Poisson request arrivals over a 32 GiB device-resident pool
PAYLOAD_SEED = 0x5EED0001
MASK_SEED = 0x5EED0002


def describe(name: str) -> str:
    n, w, fu, kind, param = WORKLOADS[name]
    typ = {1: "uint8", 2: "uint16", 4: "float32" if fu else "uint32", 8: "uint64"}[w]
    lg = n.bit_length() - 1
    if kind == "bernoulli":
        m = f"iid Bernoulli(p={param}) mask"
    elif kind == "pattern":
        return (f"single column n=2^{lg} {typ}, periodic selection {param[0]:#b} over {param[1]} elements "
                f"(no mask in memory)")
    elif kind == "predicate":
        return f"single column n=2^{lg} {typ}, selection x {param[0]} {param[1]} evaluated on the device (no mask input)"
    elif kind == "runs":
        m = f"alternating runs, geometric lengths mean {int(param)}, selectivity 0.5"
    else:
        m = f"single dense block (first {int(param * 100)}% set)"
    return f"single column n=2^{lg} {typ}, {m}, LSB-first uint32 words"


def algorithmic_bytes(n: int, w: int, count: int) -> int:
    return n * w + (n + 7) // 8 + count * w


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def load_traffic(workload: str, algo: str = "3pass"):
    """DRAM bytes per launch of the workload's dominant kernel from an ncu capture: the
    3-pass writeout under the workload's name, the 1-pass kernel under "<workload>/1pass"."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text()).get(workload if algo == "3pass" else f"{workload}/{algo}")
    return d["traffic"] if d else None


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
    """Polls SM clock and clock-event reasons through NVML while the timed region runs."""

    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
        0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
        0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting",
    }

    def __init__(self, device_index: int):
        self.samples: list[int] = []
        self.reasons = 0
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:  # noqa: BLE001 - clocks are reported as unavailable
            self.nv = None

    def _sample(self):
        try:
            self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
            self.reasons |= int(self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
        except Exception:  # noqa: BLE001
            pass

    def _run(self):
        while not self._stop.is_set():
            self._sample()
            time.sleep(0.002)

    def start(self):
        if self.nv is None:
            return
        self._sample()
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def stop(self):
        if self.nv is None:
            return
        self._sample()
        self._stop.set()
        self._t.join()

    def result(self) -> dict:
        if self.nv is None or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["nvml unavailable"]}
        names = [v for k, v in self.REASONS.items() if self.reasons & k and v != "gpu_idle"]
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz, "reasons": names,
                "samples": len(self.samples)}


# ------------------------------------------------------------------------------ dist
def dist_init(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(x: float, dist, device) -> float:
    """The maximum of x over all ranks of the process group (the job's time is the slowest
    rank's); x itself without a process group. `device` is where the collective's tensor
    lives (a CUDA device for NCCL, cpu for gloo)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world: int, bytes_per_rank: int, seconds: float) -> float:
    """Whole-job GB/s: every rank moved bytes_per_rank in at most `seconds` (the max over ranks)."""
    return world * bytes_per_rank / seconds / 1e9


# ------------------------------------------------------------------------------ reference arm
def cpu_reference_run(workload: str, steps: int, warmup: int, sample_n: int | None = None, budget_s: float = 60.0,
                      single_thread_reps: int = 0):
    """Time the reference's own CPU compaction (oracle/_ref) or, if absent, the oracle port,
    on every host thread, over the workload's whole column (or its first sample_n elements);
    with single_thread_reps, also the reference's serial generate_validation on one thread."""
    import numpy as np

    from oracle import Oracle, Reference

    n, w, fu, kind, param = WORKLOADS[workload]
    ns = min(n, sample_n or n)
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    o = Oracle.instance()
    payload = o.payload(ns, w, PAYLOAD_SEED, float_unit=fu)
    if kind == "bernoulli":
        words = o.mask_bernoulli(ns, param, MASK_SEED)
    elif kind == "runs":
        words = o.mask_runs(ns, param, MASK_SEED)
    elif kind == "pattern":
        words = o.mask_pattern(ns, param[0], param[1])
    elif kind == "predicate":
        import operator

        cmp = {">": operator.gt, ">=": operator.ge, "<": operator.lt, "<=": operator.le}[param[0]]
        bits = cmp(payload.view(np.float32) if fu else payload, param[1])
        b = np.packbits(bits.astype(np.uint8), bitorder="little")
        words = np.concatenate([b, np.zeros((-len(b)) % 4, np.uint8)]).view(np.uint32)
    else:
        words = o.mask_dense_prefix(ns, param)
    out = np.empty(ns, dtype=payload.dtype)
    if Reference.available():
        ref = Reference()
        msb = o.rev8(words.view(np.uint8))[: ns // 8]  # the reference's MSB-first byte packing
        scratch = np.empty(ns, dtype=payload.dtype)
        kindname = "reference"

        def step():
            return ref.lib.ref_generate_validation_mt(payload.ctypes.data, msb.ctypes.data, out.ctypes.data,
                                                      scratch.ctypes.data, ns, w, threads)
    else:
        kindname = "port"

        def step():
            return o.lib.oracle_compact_mt(payload.ctypes.data, words.ctypes.data, out.ctypes.data, ns, w, threads)

    count = 0
    for _ in range(warmup):
        count = step()
    times = []
    t_start = time.perf_counter()
    for _ in range(steps):
        t0 = time.perf_counter()
        count = step()
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > budget_s:
            break
    t = statistics.mean(times)
    gbs = algorithmic_bytes(ns, w, count) / t / 1e9
    what = ("the reference's generate_validation per 8-element-aligned slice + stitch" if kindname == "reference"
            else "oracle_compact_mt")
    sample = (f"{'whole column' if ns == n else f'first {ns} of {n} elements'} ({describe(workload)}), "
              f"{len(times)} timed reps of {what} on {threads} threads")
    r = {"value": gbs, "unit": UNIT, "cores": threads, "kind": kindname, "sample": sample, "ms_per_step": t * 1e3,
         "reps": len(times), "count": count, "n": ns}
    if single_thread_reps and kindname == "reference":
        # the reference's own serial path, as it runs in its driver (src/main.cu:128)
        st = []
        for _ in range(single_thread_reps):
            t0 = time.perf_counter()
            ref.lib.ref_generate_validation(payload.ctypes.data, msb.ctypes.data, scratch.ctypes.data, ns, w)
            st.append(time.perf_counter() - t0)
        ts = min(st)
        r["single_thread"] = {"value": algorithmic_bytes(ns, w, count) / ts / 1e9, "unit": UNIT, "cores": 1,
                              "ms_per_step": ts * 1e3, "reps": len(st),
                              "what": "generate_validation (src/data_generator.cuh:171-188), one thread, whole column"}
    return r


def line_config(workload: str, count: int, B: int, world: int) -> dict:
    """The `config` of a bench line; both arms (ours and --impl reference) report the same."""
    n, w, fu, kind, param = WORKLOADS[workload]
    return {"workload": describe(workload), "n": n, "elem_bytes": w, "selected": count, "bytes_per_step": B,
            "l2": ("inputs larger than L2 (no flush needed)" if n * w > L2_BYTES else
                   "inputs fit in L2: a 256 MiB buffer is written before every timed step, each step timed alone"),
            "parallelism": f"replicas: one independent column per GPU x{world}"}


def run_reference_arm(args, workload: str):
    world, rank, _ = dist_init(args.gpus)
    if rank != 0:
        return 0
    try:
        r = cpu_reference_run(workload, args.steps, args.warmup, budget_s=120.0, single_thread_reps=2)
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build failed to run: {e}"}))
        return 0
    n, w, fu, kind, param = WORKLOADS[workload]
    pattern_or_pred = kind in ("pattern", "predicate")
    B = n * w + r["count"] * w if pattern_or_pred else algorithmic_bytes(n, w, r["count"])
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": r["reps"], "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if fu else f"u{8 * w}", "data": "synthetic",
        "config": line_config(workload, r["count"], B, args.gpus),
        "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "single_thread": r.get("single_thread"),
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------ our arm
def make_inputs(cs, torch, workload: str, dev):
    n, w, fu, kind, param = WORKLOADS[workload]
    dt = {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[w]
    d_in = torch.empty(n, dtype=dt, device=dev)
    cs.gen_payload(d_in, n, PAYLOAD_SEED, float_unit=fu)
    d_mask = torch.empty((n + 31) // 32, dtype=torch.int32, device=dev)
    if kind == "bernoulli":
        cs.gen_mask_bernoulli(d_mask, n, param, MASK_SEED)
    elif kind == "runs":
        cs.gen_mask_runs(d_mask, n, param, MASK_SEED)
    elif kind == "pattern":
        cs.gen_mask_pattern(d_mask, n, param[0], param[1])  # the same selection, for the masked variants
    elif kind == "predicate":  # the same selection as mask words, for the masked variants
        d_tmp = torch.empty_like(d_in)
        d_cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        cs.compressstore_if(d_in, d_tmp, n, cs.predicate(param[0], param[1], dtype=torch.float32 if fu else d_in.dtype),
                            d_cnt, d_mask_out=d_mask)
        del d_tmp
    else:
        cs.gen_mask_dense_prefix(d_mask, n, param)
    d_out = torch.empty(n, dtype=dt, device=dev)
    d_count = torch.zeros(1, dtype=torch.int64, device=dev)
    return n, w, d_in, d_mask, d_out, d_count


def verify(torch, d_in, d_mask, d_out, count, n) -> None:
    """Independent device-side check: count = mask popcount and output = masked_select."""
    shifts = torch.arange(32, device=d_in.device, dtype=torch.int32)
    bits = ((d_mask.view(-1, 1) >> shifts) & 1).view(-1)[:n].bool()
    exp_count = int(bits.sum().item())
    if count != exp_count:
        raise AssertionError(f"count {count} != mask popcount {exp_count}")
    ref = torch.masked_select(d_in, bits)
    if not torch.equal(d_out[:count], ref):
        raise AssertionError("output differs from masked_select")
    del bits, ref


L2_BYTES = 126e6


class L2Flush:
    """Per-step timing for workloads whose inputs fit in L2 (126 MB): before every timed
    step a 256 MiB buffer is written (evicting the step's inputs), then the step runs between
    its own pair of CUDA events on the stream. Everything is queued ahead on the stream, so
    the events bracket the step's device time and not the host's launch rate."""

    def __init__(self, torch, device):
        self.buf = torch.empty(256 << 20, dtype=torch.uint8, device=device)
        self.torch = torch

    def time(self, fn, steps: int, warmup: int, stream) -> float:
        torch = self.torch
        for i in range(warmup):
            self.buf.fill_(i & 0xff)
            fn()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i, (e0, e1) in enumerate(ev):
            self.buf.fill_((i + 7) & 0xff)
            e0.record(stream)
            fn()
            e1.record(stream)
        ev[-1][1].synchronize()
        return sum(e0.elapsed_time(e1) for e0, e1 in ev) / steps  # ms


def time_steps(torch, fn, steps: int, warmup: int, stream, flush: "L2Flush | None" = None) -> float:
    """Mean device time of one step (ms); with `flush`, L2 is flushed before every step."""
    if flush is not None:
        return flush.time(fn, steps, warmup, stream)
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps  # ms


def batch_measure(dev, rank: int, steps: int, warmup: int) -> dict:
    """256 columns, lengths log-uniform in [2^10, 2^24], widths {4, 8}, iid masks with p
    uniform in [0.01, 0.99] (seeded): elements/s of one batched plan (CS_ALGO_AUTO: each
    column's form from the batch table; graph replay) against the per-call loop of the same
    columns (cs_batch_run_per_call: one plain compressstore per column, a C-side loop).
    Every column of both is checked bit-exact against the plain call before timing."""
    import numpy as np
    import torch

    import gpu_compressstore2_b200 as cs

    rng = np.random.default_rng(20240604 + rank)
    ncols = 256
    lens = np.exp(rng.uniform(np.log(2 ** 10), np.log(2 ** 24), ncols)).astype(np.int64)
    widths = rng.choice([4, 8], ncols)
    ps = rng.uniform(0.01, 0.99, ncols)
    cols, refs = [], []
    counts = torch.zeros(ncols, dtype=torch.int64, device=dev)
    ref_counts = torch.zeros(ncols, dtype=torch.int64, device=dev)
    for i in range(ncols):
        n, w = int(lens[i]), int(widths[i])
        dt = torch.int32 if w == 4 else torch.int64
        d_in = torch.empty(n, dtype=dt, device=dev)
        cs.gen_payload(d_in, n, 7000 + i)
        d_mask = torch.empty((n + 31) // 32, dtype=torch.int32, device=dev)
        cs.gen_mask_bernoulli(d_mask, n, float(ps[i]), 8000 + i)
        cols.append((d_in, d_mask, torch.empty(n, dtype=dt, device=dev), n, counts[i:i + 1]))
        refs.append(torch.empty(n, dtype=dt, device=dev))
    elems = int(lens.sum())
    stream = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(stream):
        b = cs.Batch(cols, stream=stream)
        b.run(stream=stream)
        b.capture_graph(stream=stream)
        b.run(stream=stream)
        b.check(stream=stream)
        # bit-exact: every column of the plan == the plain call
        for i, c in enumerate(cols):
            cs.compressstore(c[0], c[1], refs[i], c[3], ref_counts[i:i + 1], stream=stream)
        stream.synchronize()
        if not torch.equal(counts, ref_counts):
            raise AssertionError("batched counts differ from the plain calls")
        for i, c in enumerate(cols):
            k = int(counts[i].item())
            if not torch.equal(c[2][:k], refs[i][:k]):
                raise AssertionError(f"column {i}: batched output differs from the plain call")
        del refs
        B = sum(int(lens[i]) * int(widths[i]) + (int(lens[i]) + 7) // 8 + int(counts[i].item()) * int(widths[i])
                for i in range(ncols))

        def timed(f, k):
            for _ in range(warmup):
                f()
            stream.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(k):
                f()
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1) / k

        sampler = ClockSampler(dev.index or 0)
        launches0 = cs.launch_count()
        sampler.start()
        ms_batch = timed(lambda: b.run(stream=stream), steps)
        sampler.stop()
        launches = (cs.launch_count() - launches0) // (steps + warmup) * steps
        ms_loop = timed(lambda: b.run_per_call(stream=stream), max(3, steps // 2))
        b.check(stream=stream)
        one_pass = b.one_pass_columns
        b.close()
    value = elems / (ms_batch * 1e-3)
    loop_value = elems / (ms_loop * 1e-3)
    return {"value": value, "unit": "elements/s", "ms_per_step": ms_batch, "elements": elems, "bytes_per_step": B,
            "achieved_gbs": B / (ms_batch * 1e-3) / 1e9, "one_pass_columns": one_pass,
            "per_call_loop": {"value": loop_value, "unit": "elements/s", "ms_per_step": ms_loop,
                              "loop": "cs_batch_run_per_call (C-side loop of plain calls)"},
            "batched_over_per_call": value / loop_value, "gpu_launches": launches, "clocks": sampler.result(),
            "checked": "every column == plain call (counts and bytes)"}


def run_batch(args):
    import torch

    world, rank, local = dist_init(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    r = batch_measure(dev, rank, args.steps, args.warmup)
    if rank == 0:
        peaks = load_peaks()
        line = {
            "metric": "batched compaction elements/s (256 uneven columns, one plan)", "value": r["value"],
            "unit": "elements/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32/u64", "data": "synthetic",
            "config": {"workload": "256 columns, lengths log-uniform [2^10, 2^24], widths {4, 8}, iid masks p~U[0.01,0.99]",
                       "elements": r["elements"], "bytes_per_step": r["bytes_per_step"], "graph": True,
                       "one_pass_columns": r["one_pass_columns"]},
            "per_call_loop": r["per_call_loop"], "batched_over_per_call": r["batched_over_per_call"],
            "roofline": {"bound": "hbm", "achieved": r["achieved_gbs"], "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": r["achieved_gbs"] / peaks["hbm_gbs"], "traffic": None, "peak_source": peaks["source"]},
            "gpu_launches": r["gpu_launches"], "clocks": r["clocks"],
        }
        print(json.dumps(line))
    return 0


def serve_measure(dev, rank: int, k: int, loads, pool_gib: float, budget_gib: int,
                  modes=(("batch", "SERVE_BATCH", 3), ("per_call", "SERVE_PER_CALL", 1),
                         ("per_call_3slots", "SERVE_PER_CALL", 3))) -> dict:
    """Serving loop: Poisson arrivals at each offered load; request n log-uniform in
    [2^12, 2^26] uint32/float32 elements with an iid mask, p uniform in [0.01, 0.99], drawn
    from a device-resident pool of payload + mask (64 regions, each with its own payload kind,
    uint32 or float32 alternating, and its own mask p; a request is a 128-element-aligned
    slice of one region). Each offered load is replayed by the library's native load
    generator (cs_server_replay) against continuous batching and against one plain call per
    request (one or three in flight); throughput counts algorithmic bytes (payload + mask
    read + selected written) over the time to the last completion. Outputs of a burst of
    mixed requests are checked bit-exact against the plain call first."""
    import numpy as np
    import torch

    import gpu_compressstore2_b200 as cs

    regions = 64
    pool_bytes = int(pool_gib * (1 << 30))
    region_n = (pool_bytes // regions * 8 // 33) // 4096 * 4096  # 4 B payload + 1/8 B mask per element
    pool_n = region_n * regions
    rng = np.random.default_rng(20241203 + rank)
    region_p = rng.uniform(0.01, 0.99, regions)
    d_pool = torch.empty(pool_n, dtype=torch.int32, device=dev)
    d_mpool = torch.empty(pool_n // 32, dtype=torch.int32, device=dev)
    for r in range(regions):
        cs.gen_payload(d_pool[r * region_n:(r + 1) * region_n], region_n, 9100 + r, float_unit=(r % 2 == 1))
        cs.gen_mask_bernoulli(d_mpool[r * region_n // 32:(r + 1) * region_n // 32], region_n, float(region_p[r]),
                              9300 + r)
    torch.cuda.synchronize()
    base_in, base_mask = d_pool.data_ptr(), d_mpool.data_ptr()

    def draw(count):
        ns = np.exp(rng.uniform(np.log(2 ** 12), np.log(2 ** 26), count)).astype(np.int64)
        rs = rng.integers(0, regions, count)
        offs = rs * region_n + rng.integers(0, (region_n - ns) // 128 + 1) * 128
        return ns, rs, offs

    def requests(ns, offs):
        return [cs.Server.request(base_in + int(o) * 4, base_mask + int(o) // 8, int(n), 4) for n, o in zip(ns, offs)]

    # bit-exactness of a mixed burst against the plain call
    vk = 64
    ns, rs, offs = draw(vk)
    verified = 0
    with cs.Server(out_budget_bytes=budget_gib << 30) as srv:
        tickets = [srv.submit(base_in + int(o) * 4, base_mask + int(o) // 8, int(n), 4) for n, o in zip(ns, offs)]
        tmp = torch.empty(int(ns.max()), dtype=torch.int32, device=dev)
        cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        mixed = 0
        for t, n, o in zip(tickets, ns, offs):
            res = srv.wait(t, timeout_s=60)
            if res.status != 0:
                raise AssertionError(f"serve request failed: {cs._lib.lib().cs_status_string(res.status)}")
            n, o = int(n), int(o)
            cs.compressstore(d_pool[o:o + n], d_mpool[o // 32:o // 32 + (n + 31) // 32], tmp, n, cnt)
            kk = int(cnt.item())
            if kk != res.count or not torch.equal(srv.output(t, res), tmp[:kk]):
                raise AssertionError("served output differs from the plain call")
            mixed += res.batch_size > 1
            srv.release(t)
            verified += 1

    ns, rs, offs = draw(k)
    reqs = requests(ns, offs)
    est_bytes = ns * 4 + (ns + 7) // 8 + (ns * region_p[rs] * 4)
    mean_bytes = float(est_bytes.mean())
    sampler = ClockSampler(dev.index or 0)
    sweep = []
    sampler.start()
    for gbs in loads:
        lam = gbs * 1e9 / mean_bytes  # requests per second
        arrivals = np.cumsum(rng.exponential(1e9 / lam, k)).astype(np.int64)
        point = {"offered_gbs": gbs, "offered_rps": lam}
        for name, mode, slots in modes:
            with cs.Server(out_budget_bytes=budget_gib << 30, mode=getattr(cs, mode), slots=slots) as srv:
                srv.replay(reqs[:8], np.zeros(8, dtype=np.int64))  # warm-up
                st0 = srv.stats()
                res = srv.replay(reqs, arrivals)
                st1 = srv.stats()
            bad = [r for r in res if r.status != 0]
            if bad:
                raise AssertionError(f"{len(bad)} served requests failed ({name})")
            lat = np.array([r.latency_ns for r in res], dtype=np.float64)
            done = arrivals + lat
            counts = np.array([r.count for r in res], dtype=np.int64)
            total = float((ns * 4 + (ns + 7) // 8 + counts * 4).sum())
            span = float(done.max())
            point[name] = {
                "achieved_gbs": total / span, "achieved_rps": k / span * 1e9,
                "p50_ms": float(np.percentile(lat, 50)) / 1e6, "p99_ms": float(np.percentile(lat, 99)) / 1e6,
                "mean_queue_ms": float(np.mean([r.queue_ns for r in res])) / 1e6,
                "mean_batch": float(np.mean([r.batch_size for r in res])),
                "batches": st1["batches"] - st0["batches"],
                "gpu_launches": st1["kernel_launches"] - st0["kernel_launches"],
                "arena_peak_bytes": st1["arena_peak"],
            }
        sweep.append(point)
    sampler.stop()
    del d_pool, d_mpool
    torch.cuda.empty_cache()
    return {"sweep": sweep, "clocks": sampler.result(), "requests_per_load": k, "regions": regions,
            "pool_bytes": pool_n * 4 + pool_n // 8, "verified_mixed_vs_plain": {"requests": verified,
                                                                                "ran_in_a_mix": int(mixed)}}


def run_serve(args):
    import torch

    world, rank, local = dist_init(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    loads = [float(x) for x in args.serve_loads.split(",")]
    r = serve_measure(dev, rank, args.serve_requests, loads, args.serve_pool_gib, args.serve_budget_gib)
    sweep = r["sweep"]
    if rank == 0:
        best = max(sweep, key=lambda p: p["batch"]["achieved_gbs"])
        peaks = load_peaks()
        line = {
            "metric": "serving throughput (algorithmic GB/s at the best offered load) with p50/p99 latency",
            "value": best["batch"]["achieved_gbs"], "unit": "GB/s", "n_gpus": world, "steps": r["requests_per_load"],
            "warmup": 8, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32/f32", "data": "synthetic",
            "config": {"workload": "Poisson arrivals, n log-uniform [2^12, 2^26] uint32/float32, iid masks "
                                   "p~U[0.01,0.99], 32 GiB device-resident pool",
                       "pool_bytes": r["pool_bytes"], "requests_per_load": r["requests_per_load"],
                       "regions": r["regions"], "out_budget_gib": args.serve_budget_gib, "slots": 3, "max_batch": 64},
            "p50_ms": best["batch"]["p50_ms"], "p99_ms": best["batch"]["p99_ms"],
            "per_call_at_best": best["per_call"], "per_call_3slots_at_best": best["per_call_3slots"],
            "sweep": sweep,
            "verified_mixed_vs_plain": r["verified_mixed_vs_plain"],
            "roofline": {"bound": "hbm", "achieved": best["batch"]["achieved_gbs"], "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": best["batch"]["achieved_gbs"] / peaks["hbm_gbs"], "traffic": None,
                         "peak_source": peaks["source"]},
            "gpu_launches": best["batch"]["gpu_launches"], "clocks": r["clocks"],
        }
        print(json.dumps(line))
    return 0


REF_GPU_BIN = ROOT / "baseline" / "_ref" / "ref_gpu_bench"
# (chunk lengths, block sizes, grid sizes) the reference GPU compositions are swept over in
# the bench: the neighbourhood of their best points on B200 from the full sweep of the
# reference driver's ranges (chunk 32..8192, block 32..1024, grid 32..2048; profiles/).
REF_GPU_SWEEP = ("1024,4096,8192", "256,1024", "1024,2048")


def reference_gpu_run(workload: str, reps: int = 5, sweep=REF_GPU_SWEEP, timeout_s: float = 300.0) -> dict:
    """Time the reference's own GPU compositions bench10 / bench7 / bench8 (compiled from its
    sources into baseline/_ref by baseline/Makefile) on this GPU, in a child process, over a
    small (chunk, block, grid) sweep; each configuration's output is checked byte for byte
    against the library's plain call on the same inputs. Returns {bench: best result} or
    {"unavailable": why}."""
    import subprocess

    n, w, fu, kind, param = WORKLOADS[workload]
    if not REF_GPU_BIN.exists():
        return {"unavailable": "baseline/_ref/ref_gpu_bench not built (needs the reference sources)"}
    if kind != "bernoulli" or w not in (4, 8) or n % 8192 or n >= 1 << 32:
        return {"unavailable": "the reference's GPU path runs 4/8-byte iid-mask columns below 2^32 elements"}
    cmd = [str(REF_GPU_BIN), str(n), str(w), str(param), str(PAYLOAD_SEED), str(MASK_SEED), str(reps), *sweep,
           "bench10,bench7,bench8"]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s)
    except subprocess.TimeoutExpired:
        return {"unavailable": f"ref_gpu_bench exceeded {timeout_s:.0f} s"}
    if r.returncode != 0:
        return {"unavailable": f"ref_gpu_bench exit {r.returncode}: {(r.stderr or r.stdout)[-300:]}"}
    d = json.loads(r.stdout.strip().splitlines()[-1])
    if not all(x["ok"] for x in d["results"]):
        bad = [f"{x['bench']}({x['chunk']},{x['block']},{x['grid']})" for x in d["results"] if not x["ok"]]
        return {"unavailable": f"reference GPU output differs from the library's: {bad}"}
    d["sweep"] = {"chunk": sweep[0], "block": sweep[1], "grid": sweep[2], "reps": reps}
    return d


def kernel_roofline(cs, torch, args, n, w, d_in, d_mask, d_out, d_count, B, step_ms, stream, peaks, workload):
    """Roofline of the dominant kernel, timed alone with CUDA events on its stream.

    1-pass: the step is the single k_compact_tma launch, so the step time is its time.
    3-pass: k_compact_tma (writeout) is launched alone through cs_writeout, over the same
    inputs with the chunk offsets of the same chunk length, and timed; its algorithmic bytes
    are the call's (every payload byte read once, mask read, selected written; the counts and
    offsets it also reads are under 0.3% of that)."""
    algo, chunk = args.algo, 0
    if algo == "auto":
        a = ctypes.c_int32()
        c = ctypes.c_uint32()
        cs.lib().cs_tune_get(w, n, ctypes.byref(a), ctypes.byref(c))
        algo = {cs.ALGO_1PASS: "1pass", cs.ALGO_3PASS: "3pass", cs.ALGO_NAIVE: "naive"}[a.value]
        chunk = int(c.value)
    if algo != "3pass":
        kms = step_ms
        kernel = "k_compact_tma (1-pass: the whole step is this one kernel)" if algo == "1pass" else \
            f"whole {algo} step"
        launches_timed = args.steps
    else:
        chunk = chunk or 1024
        nchunks = (n + chunk - 1) // chunk
        counts = torch.empty(nchunks, dtype=torch.int32, device=d_in.device)
        offsets = torch.empty(nchunks, dtype=torch.int64, device=d_in.device)
        total = torch.empty(1, dtype=torch.int64, device=d_in.device)
        cs.popc_chunks(d_mask, n, chunk, counts, stream=stream)
        cs.chunk_prefix_sum(counts, nchunks, offsets, total, stream=stream)
        kms = time_steps(torch, lambda: cs.writeout(d_in, d_mask, d_out, n, offsets, counts, chunk, stream=stream),
                         args.steps, 3, stream)
        torch.cuda.synchronize()
        verify(torch, d_in, d_mask, d_out, int(total.item()), n)
        kernel = f"k_compact_tma (3-pass writeout, chunk length {chunk}), launched alone through cs_writeout"
        launches_timed = args.steps
        del counts, offsets, total
    achieved = B / (kms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": load_traffic(workload, algo),
            "peak_source": peaks["source"],
            "kernel": kernel, "kernel_ms": kms, "launches_timed": launches_timed, "bytes_per_launch": B}


def run_ours(args, workload: str):
    import torch

    import gpu_compressstore2_b200 as cs

    world, rank, local = dist_init(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    stream = torch.cuda.current_stream()
    n, w, d_in, d_mask, d_out, d_count = make_inputs(cs, torch, workload, dev)
    fu = WORKLOADS[workload][2]

    algo = {"auto": cs.ALGO_AUTO, "1pass": cs.ALGO_1PASS, "3pass": cs.ALGO_3PASS, "naive": cs.ALGO_NAIVE}[args.algo]
    kind, param = WORKLOADS[workload][3], WORKLOADS[workload][4]
    pattern_path = kind == "pattern"
    pred_path = kind == "predicate"
    pred = cs.predicate(param[0], param[1], dtype=torch.float32 if fu else d_in.dtype) if pred_path else None

    def step():
        if pattern_path:
            cs.compressstore_pattern(d_in, d_out, n, param[0], param[1], d_count)
        elif pred_path:
            cs.compressstore_if(d_in, d_out, n, pred, d_count)
        else:
            cs.compressstore(d_in, d_mask, d_out, n, d_count, algo=algo)

    # warm-up and correctness check before timing
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    cs.compressstore_check()
    count = int(d_count.item())
    verify(torch, d_in, d_mask, d_out, count, n)
    # a periodic or predicate selection reads no mask: payload read + selected written
    B = n * w + count * w if (pattern_path or pred_path) else algorithmic_bytes(n, w, count)

    # timed region (inputs that fit in L2 are evicted from it before every step)
    flush = L2Flush(torch, dev) if n * w <= L2_BYTES else None
    sampler = ClockSampler(local)
    # the sampler thread starts (and takes its first sample) before the bracketing barrier and
    # synchronize, so its start-up does not delay the first step's launch
    sampler.start()
    time.sleep(0.01)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    launches0 = cs.launch_count()
    ms = time_steps(torch, step, args.steps, 0, stream, flush)
    sampler.stop()
    launches = cs.launch_count() - launches0
    torch.cuda.synchronize()
    ms = max_over_ranks(ms, pg, dev)
    if pg:
        pg.barrier()
    value = job_throughput(world, B, ms * 1e-3)

    peaks = load_peaks()
    if pattern_path or pred_path:
        achieved = B / (ms * 1e-3) / 1e9
        kname = ("k_pattern (the whole step is this one kernel)" if pattern_path else
                 "whole step: k_pred_blocks + sparse gather + k_compact_tma (payload read twice)")
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": achieved / peaks["hbm_gbs"], "traffic": load_traffic(workload),
                    "peak_source": peaks["source"], "kernel": kname,
                    "kernel_ms": ms, "launches_timed": args.steps, "bytes_per_launch": B}
    else:
        roofline = kernel_roofline(cs, torch, args, n, w, d_in, d_mask, d_out, d_count, B, ms, stream, peaks,
                                   workload)

    # variants at the same workload (N=1 only, rank 0)
    variants = {}
    if world == 1 and not args.no_variants:
        for name, algo in (("1pass", cs.ALGO_1PASS), ("3pass", cs.ALGO_3PASS), ("naive", cs.ALGO_NAIVE)):
            def f(a=algo):
                cs.compressstore(d_in, d_mask, d_out, n, d_count, algo=a)
            vms = time_steps(torch, f, max(3, args.steps // 2), 2, stream, flush)
            variants[name] = {"ms": vms, "gbs": B / (vms * 1e-3) / 1e9}
        # CS_ALGO_AUTO told the fraction the workload selects (cs_config.selectivity)
        stated = {"bernoulli": param, "runs": 0.5, "dense": param}.get(kind, 0.0)
        if stated:
            def f():
                cs.compressstore(d_in, d_mask, d_out, n, d_count, algo=cs.ALGO_AUTO, selectivity=stated)
            vms = time_steps(torch, f, max(3, args.steps // 2), 2, stream, flush)
            variants["auto_stated"] = {"ms": vms, "gbs": B / (vms * 1e-3) / 1e9, "selectivity": stated}
        cub = cs.CubFlagged(n, w, device=dev)
        vms = time_steps(torch, lambda: cub(d_in, d_mask, d_out, n, d_count), max(3, args.steps // 2), 2, stream,
                         flush)
        variants["cub_flagged"] = {"ms": vms, "gbs": B / (vms * 1e-3) / 1e9}
        torch.cuda.synchronize()
        verify(torch, d_in, d_mask, d_out, int(d_count.item()), n)
        del cub
        torch.cuda.empty_cache()
        # the reference's own GPU compositions, at their best swept configuration; GB/s of
        # the same algorithmic bytes over the reference's own timings.total
        ref = reference_gpu_run(workload)
        if "unavailable" in ref:
            variants["ref_gpu"] = ref
        else:
            for bench, best in ref["best"].items():
                variants[f"ref_{bench}"] = {"ms": best["total_ms_min"], "gbs": B / (best["total_ms_min"] * 1e-3) / 1e9,
                                            "proc_ms": best["proc_ms"], "chunk": best["chunk"],
                                            "block": best["block"], "grid": best["grid"],
                                            "timing": "reference timings.total (its CUDA events), min over reps",
                                            "checked": "output == library plain call, every swept point"}

    # end to end through the public host-buffer call: pinned host payload and mask in, count
    # and selected payload back, every step (compressstore_host pipelines the copies)
    e2e = None
    if not args.no_e2e and not pattern_path and not pred_path:
        h_in = torch.empty(d_in.shape, dtype=d_in.dtype, pin_memory=True)
        h_mask = torch.empty(d_mask.shape, dtype=d_mask.dtype, pin_memory=True)
        h_in.copy_(d_in)
        h_mask.copy_(d_mask)
        h_out = torch.empty(d_out.shape, dtype=d_out.dtype, pin_memory=True)
        torch.cuda.synchronize()

        def e2e_step():
            return cs.compressstore_host(h_in, h_mask, h_out, n)

        k = e2e_step()
        if k != count or not torch.equal(h_out[:k], d_out[:k].cpu()):
            raise AssertionError("host-buffer path differs from the device path")
        e2e_step()
        ke = max(3, min(args.steps, 10))
        if pg:
            pg.barrier()
        step_ms = []
        t0 = time.perf_counter()
        for _ in range(ke):
            t1 = time.perf_counter()
            k = e2e_step()
            step_ms.append((time.perf_counter() - t1) * 1e3)
        et = (time.perf_counter() - t0) / ke
        et = max_over_ranks(et, pg, dev)
        # The same step's copies with no compaction: the H2D of payload + mask beside the D2H
        # of the selected payload, on two streams. Their time is the PCIe bound of the step.
        s_h2d, s_d2h = torch.cuda.Stream(), torch.cuda.Stream()

        def copies_only():
            with torch.cuda.stream(s_h2d):
                d_in.copy_(h_in, non_blocking=True)  # the same bytes d_in already holds
                d_mask.copy_(h_mask, non_blocking=True)
            with torch.cuda.stream(s_d2h):
                h_out[:k].copy_(d_out[:k], non_blocking=True)
            torch.cuda.synchronize()

        copies_only()
        bound = []
        for _ in range(3):
            t1 = time.perf_counter()
            copies_only()
            bound.append(time.perf_counter() - t1)
        bound_ms = sorted(bound)[1] * 1e3
        pieces = (n * w + (32 << 20) - 1) // (32 << 20)
        e2e = {"value": job_throughput(world, B, et), "unit": UNIT, "h2d_bytes_per_step": n * w + d_mask.numel() * 4,
               "d2h_bytes_per_step": k * w + 8 * pieces, "ms_per_step": et * 1e3,
               "step_ms": [round(x, 2) for x in step_ms],
               "pcie_bound_ms": round(bound_ms, 3), "frac_of_pcie_bound": round(bound_ms / (et * 1e3), 3),
               "path": "compressstore_host: pinned host buffers, 32 MB pieces, H2D/compute/D2H overlapped"}
        del h_in, h_mask, h_out

    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        try:
            r = cpu_reference_run(workload, steps=20, warmup=1, budget_s=20.0, single_thread_reps=1)
            cpu = {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")}
            if "single_thread" in r:
                cpu["single_thread"] = r["single_thread"]
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": None, "sample": f"unavailable: {e}"}

    # the systems forms, measured in the same run (N=1, default workload): a short batch256
    # timing and one serving point, each with its own clocks and parity check
    systems = {}
    if world == 1 and rank == 0 and workload == DEFAULT_WORKLOAD and not args.no_systems:
        torch.cuda.empty_cache()
        try:
            systems["batch"] = batch_measure(dev, 0, steps=10, warmup=3)
            systems["batch"]["workload"] = ("256 columns, lengths log-uniform [2^10, 2^24], widths {4, 8}, "
                                            "iid masks p~U[0.01,0.99], graph replay")
        except Exception as e:  # noqa: BLE001
            systems["batch"] = {"unavailable": f"{type(e).__name__}: {e}"}
        torch.cuda.empty_cache()
        try:
            # 2000 requests (about 15 ms of arrivals), so the drain after the last arrival is a
            # few percent of the span
            sv = serve_measure(dev, 0, k=2000, loads=[6000.0], pool_gib=32.0, budget_gib=4,
                               modes=(("batch", "SERVE_BATCH", 3), ("per_call_3slots", "SERVE_PER_CALL", 3)))
            pt = sv["sweep"][0]
            systems["serve"] = {"offered_gbs": pt["offered_gbs"], "continuous_batching": pt["batch"],
                                "per_call_3_in_flight": pt["per_call_3slots"], "clocks": sv["clocks"],
                                "requests": sv["requests_per_load"], "pool_bytes": sv["pool_bytes"],
                                "verified_mixed_vs_plain": sv["verified_mixed_vs_plain"],
                                "workload": "Poisson arrivals, n log-uniform [2^12, 2^26] uint32/float32, iid masks "
                                            "p~U[0.01,0.99], 32 GiB device-resident pool"}
        except Exception as e:  # noqa: BLE001
            systems["serve"] = {"unavailable": f"{type(e).__name__}: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if fu else f"u{8 * w}", "data": "synthetic",
            "config": line_config(workload, count, B, world), "algo": args.algo,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": sampler.result(), "variants": variants, **systems,
        }
        print(json.dumps(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD,
                    choices=sorted(WORKLOADS) + [BATCH_WORKLOAD, SERVE_WORKLOAD])
    ap.add_argument("--algo", choices=["auto", "1pass", "3pass", "naive"], default="auto")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-systems", action="store_true", help="skip the batch and serve keys of the default line")
    ap.add_argument("--serve-requests", type=int, default=3000, help="requests per offered load (serve)")
    ap.add_argument("--serve-loads", default="500,1000,2000,3000,4000,5000,6000",
                    help="offered loads in algorithmic GB/s (serve)")
    ap.add_argument("--serve-pool-gib", type=float, default=32.0)
    ap.add_argument("--serve-budget-gib", type=int, default=4)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        if args.workload in (BATCH_WORKLOAD, SERVE_WORKLOAD):
            print(json.dumps({"impl": "reference", "unavailable": f"the reference has no {args.workload} form"}))
            return 0
        return run_reference_arm(args, args.workload)
    if args.workload == BATCH_WORKLOAD:
        return run_batch(args)
    if args.workload == SERVE_WORKLOAD:
        return run_serve(args)
    return run_ours(args, args.workload)


if __name__ == "__main__":
    sys.exit(main())
