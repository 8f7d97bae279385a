"""Autotuner for CS_ALGO_AUTO: measures the candidate algorithms and chunk lengths per
(element width, size bucket) on this GPU and installs the fastest in the library's table.

The reference picks chunk length, block and grid by an exhaustive sweep inside every run
(src/main.cu:168-190) and keeps the fastest per phase in SQL views (eval/eval.db); here the
sweep runs once per GPU model, and its result is a small text table (``cs_tune_save``
format) that ``cs_tune_load`` or the ``CS_TUNE_TABLE`` environment variable installs.

Each candidate is timed on masks of five selectivities, one per selectivity bucket (inputs
smaller than 512 MB with L2 flushed before every call, as the bench times them). The sum of
its times at 0.01, 0.5 and 0.99 decides the (width, size) entry, which a call takes when its
selectivity is unknown: the plain call cannot measure it before it runs without a pass of its
own. The fastest candidate at each selectivity becomes that selectivity bucket's entry
(``sel`` lines), which a call takes when its caller states the fraction it expects
(``cs_config.selectivity``). Within the 3-pass
hybrid the per-unit choice between the TMA writeout and the sparse gather is made at run time
from the pass-1 counts, so the dense / sparse split needs no table entry.

The batched form has a table of its own, keyed by (element width, size bucket, selectivity
bucket), because inside a plan the passes are shared by all columns: a column's form there is
a trade between reading its mask twice (3-pass) and waiting on look-backs (1-pass), not
launch latency. ``tune_batch`` times, per bucket, a plan of equal columns forced to each form
and keeps the faster (``batch`` lines of the table file).

Usage: python -m gpu_compressstore2_b200.autotune [--out FILE] [--max-log2 N] [--reps R]
                                                  [--plain-only | --batch-only]
"""
from __future__ import annotations

import argparse
import ctypes
import time
from pathlib import Path

from . import _lib

DEFAULT_TABLE = _lib.TUNE_TABLE

# candidates: (algo, chunk_length)
CANDIDATES = [
    (_lib.ALGO_1PASS, 1024),
    (_lib.ALGO_3PASS, 1024),
    (_lib.ALGO_3PASS, 2048),
    (_lib.ALGO_3PASS, 4096),
]
SELECTIVITIES = (0.01, 0.1, 0.5, 0.9, 0.99)  # one per selectivity bucket (cs_tune_sel_bucket)
# the (width, size) entry, for calls whose selectivity is unknown: the best sum over these
UNKNOWN_SELECTIVITIES = (0.01, 0.5, 0.99)


def bucket_sizes(max_log2: int) -> list[tuple[int, list[int]]]:
    """(size_bucket, [n]) with both sizes of the bucket: bucket b holds log2(n) in {2b, 2b+1}."""
    out = []
    for b in range(5, max_log2 // 2 + 1):
        out.append((b, [1 << lg for lg in (2 * b, 2 * b + 1) if lg <= max_log2]))
    return out


L2_FLUSH_BELOW = 512 << 20  # working sets smaller than this are timed with L2 flushed per call


def _time_call(torch, fn, reps: int, stream, flush=None) -> float:
    """Milliseconds per call. With `flush` (a device buffer larger than L2) every call is timed
    alone after the buffer is rewritten, so small inputs are read from DRAM as in the bench
    (the median); otherwise back-to-back calls (the mean)."""
    for _ in range(2):
        if flush is not None:
            flush.fill_(1)
        fn()
    stream.synchronize()
    if flush is not None:
        times = []
        for _ in range(reps):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        times.sort()
        return times[len(times) // 2]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def tune(widths=(1, 2, 4, 8), max_log2: int = 30, reps: int = 5, max_bytes: int = 8 << 30, verbose: bool = True):
    """Measure every candidate at both sizes of each bucket; returns {(w, bucket): (algo, chunk,
    {candidate: ms}, {sel_bucket: (algo, chunk)})}: the best sum over SELECTIVITIES and sizes,
    and the best sum over the sizes at each selectivity."""
    import torch

    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    stream = torch.cuda.Stream()
    results = {}
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(stream):
        for w in widths:
            dt = {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[w]
            for b, sizes in bucket_sizes(max_log2):
                sizes = [n for n in sizes if n * w <= max_bytes]
                if not sizes:
                    continue
                per_sel = {c: [0.0] * len(SELECTIVITIES) for c in CANDIDATES}  # candidate -> ms per selectivity
                for n in sizes:
                    d_in = torch.empty(n, dtype=dt, device="cuda")
                    cs.gen_payload(d_in, n, 11 + b, stream=stream)
                    d_out = torch.empty_like(d_in)
                    d_count = torch.zeros(1, dtype=torch.int64, device="cuda")
                    masks = []
                    for i, p in enumerate(SELECTIVITIES):
                        m = torch.empty(cs.mask_words(n) + 4, dtype=torch.int32, device="cuda")
                        cs.gen_mask_bernoulli(m, n, p, 100 + i, stream=stream)
                        masks.append(m)
                    for algo, chunk in CANDIDATES:
                        cfg = _lib.CsConfig(algo, chunk, 0, 0, 0)
                        for i, m in enumerate(masks):
                            args = (d_in.data_ptr(), m.data_ptr(), d_out.data_ptr(), n, w, d_count.data_ptr(),
                                    ctypes.byref(cfg), stream.cuda_stream)

                            def call(args=args):
                                _lib.check(L.compressstore_cfg(*args), "compressstore_cfg")

                            per_sel[(algo, chunk)][i] += _time_call(torch, call, reps, stream,
                                                                    flush_buf if n * w < L2_FLUSH_BELOW else None)
                    del d_in, d_out, masks
                    torch.cuda.empty_cache()
                times = {c: sum(t for p, t in zip(SELECTIVITIES, v) if p in UNKNOWN_SELECTIVITIES)
                         for c, v in per_sel.items()}
                best = min(times, key=times.get)
                sel_best = {}
                for i, p in enumerate(SELECTIVITIES):
                    sel_best[int(L.cs_tune_sel_bucket(p))] = min(per_sel, key=lambda c: per_sel[c][i])
                results[(w, b)] = (best[0], best[1], times, sel_best)
                if verbose:
                    desc = " ".join(f"{a}/{c}:{t * 1e3:.1f}us" for (a, c), t in times.items())
                    sel = " ".join(f"p={p}:{a}/{c}" for p, (a, c) in zip(SELECTIVITIES, sel_best.values()))
                    lg = "/".join(str(n.bit_length() - 1) for n in sizes)
                    print(f"w={w} bucket={b} n=2^{lg}: best algo={best[0]} chunk={best[1]}  [{desc}]  "
                          f"by selectivity [{sel}]", flush=True)
    return results


BATCH_SELECTIVITIES = SELECTIVITIES


def tune_batch(widths=(1, 2, 4, 8), buckets=range(5, 13), reps: int = 10, elems: int = 1 << 26,
               verbose: bool = True):
    """Per (width, size bucket, selectivity bucket): time a plan of equal columns (n in the
    middle of the bucket, enough columns for ~`elems` elements, at least 8, at most 512)
    forced to the 1-pass and to the 3-pass form (graph replay); returns
    {(w, bucket, sel_bucket): (algo, {algo: ms})}."""
    import torch

    import gpu_compressstore2_b200 as cs

    L = cs.lib()
    results = {}
    stream = torch.cuda.Stream()
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(stream):
        for w in widths:
            dt = {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[w]
            for b in buckets:
                n = 1 << (2 * b + 1)
                k = max(8, min(512, elems // n))
                d_in = torch.empty(k * n, dtype=dt, device="cuda")
                cs.gen_payload(d_in, k * n, 31 + b, stream=stream)
                d_out = torch.empty_like(d_in)
                d_mask = torch.empty(k * n // 32, dtype=torch.int32, device="cuda")
                counts = torch.zeros(k, dtype=torch.int64, device="cuda")
                cols = [(d_in[i * n:(i + 1) * n], d_mask[i * n // 32:(i + 1) * n // 32], d_out[i * n:(i + 1) * n], n,
                         counts[i:i + 1]) for i in range(k)]
                for p in BATCH_SELECTIVITIES:
                    cs.gen_mask_bernoulli(d_mask, k * n, p, 77 + b, stream=stream)
                    times = {}
                    for algo in (_lib.ALGO_1PASS, _lib.ALGO_3PASS):
                        plan = cs.Batch(cols, stream=stream, algo=algo)
                        plan.capture_graph(stream=stream)
                        times[algo] = _time_call(torch, lambda: plan.run(stream=stream), reps, stream,
                                                 flush_buf if k * n * w < L2_FLUSH_BELOW else None)
                        plan.check(stream=stream)
                        plan.close()
                    best = min(times, key=times.get)
                    sb = int(L.cs_tune_sel_bucket(p))
                    results[(w, b, sb)] = (best, times)
                    if verbose:
                        print(f"batch w={w} bucket={b} n=2^{2 * b + 1} x{k} p={p}: best algo={best}  "
                              f"[1pass:{times[_lib.ALGO_1PASS] * 1e3:.1f}us 3pass:{times[_lib.ALGO_3PASS] * 1e3:.1f}us]",
                              flush=True)
                del d_in, d_out, d_mask, cols
                torch.cuda.empty_cache()
    return results


def install_batch(results) -> None:
    L = _lib.lib()
    for (w, b, sb), (algo, _) in results.items():
        _lib.check(L.cs_tune_batch_set(w, b, sb, algo), "cs_tune_batch_set")


def install(results) -> None:
    """Put measured choices in the library's table (every untuned bucket keeps the default)."""
    L = _lib.lib()
    for (w, b), (algo, chunk, _, sel_best) in results.items():
        _lib.check(L.cs_tune_set(w, b, algo, chunk), "cs_tune_set")
        for sb, (a, c) in sel_best.items():
            _lib.check(L.cs_tune_sel_set(w, b, sb, a, c), "cs_tune_sel_set")


def save(path: Path) -> None:
    _lib.check(_lib.lib().cs_tune_save(str(path).encode()), "cs_tune_save")


def load(path: Path = DEFAULT_TABLE) -> bool:
    """Install a saved table; False when the file does not exist."""
    path = Path(path)
    if not path.exists():
        return False
    _lib.check(_lib.lib().cs_tune_load(str(path).encode()), f"cs_tune_load({path})")
    return True


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default=str(DEFAULT_TABLE))
    ap.add_argument("--max-log2", type=int, default=30)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--plain-only", action="store_true")
    ap.add_argument("--batch-only", action="store_true")
    args = ap.parse_args()
    t0 = time.time()
    entries = 0
    if not args.batch_only:
        res = tune(max_log2=args.max_log2, reps=args.reps)
        install(res)
        entries += len(res)
    if not args.plain_only:
        bres = tune_batch(reps=2 * args.reps)
        install_batch(bres)
        entries += len(bres)
    save(Path(args.out))
    print(f"wrote {args.out} ({entries} entries) in {time.time() - t0:.0f} s")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
