"""Autotuner: choose, per length bucket, the kernel shape of each path.

A bucket is a query word count w = ceil(m/32) (1..1024). Its candidate
shapes are every compiled variant that holds w words: one candidate per lane
with W = w words (w <= 32), and a candidate spread over L = ceil(w/W) lanes
for each multi-lane width W (the persistent kernel carries W <= 16). For every
bucket 1..32 and a sample of longer ones, each shape is timed on a seeded
workload of reads of 32*w bases, about 1e13 cells (20K..4M candidates) so
that every shape runs many waves (CUDA events, best of three after a warm-up);
the fastest wins. Unsampled long buckets take the width of the nearest
sampled bucket above them, with L = ceil(w/W).

The batched path has a second table for large batches ("batched_large", used
from 150K candidates on): every bucket of 33..512 words takes the multi-lane
shape that the cost model ranks first (model_shape), over every width from 4
to 16 words. The model counts idle lanes and padding rows, and on 500K
long-read candidates its shapes ran 5% faster than the sampled ones. In small
batches the many shapes they use run side by side in the persistent kernel
and thrash its instruction cache, so small batches keep the sampled table.

    python myers-gpu_b200/autotune.py [--out PATH] [--quick]
    python myers-gpu_b200/autotune.py --refill-batched-long   # no GPU: rewrite batched_large in the cache

writes autotune_b200.json next to the library (the runtime loads it at
start); the file also keeps every measurement.
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

LONG_SAMPLE = [33, 36, 40, 44, 48, 56, 64, 72, 80, 96, 112, 128, 160, 192, 224, 256, 320, 384, 448, 512, 640, 768,
               896, 1024]
DIST = 0.2


def candidate_shapes(mg, w, path):
    out = []
    if w <= 32:
        out.append((w - 1, 1))
    for v, W, multi in mg.variants():
        if not multi:
            continue
        if path == mg.PATH_BATCHED and W > 16 and w <= 512:
            continue
        L = math.ceil(w / W)
        if 2 <= L <= 32:
            out.append((v, L))
    return out


def model_shape(w, widths):
    """The multi-lane shape (W, L) of a bucket of w words that the cost model
    ranks first: the lanes a candidate occupies (32 / floor(32/L), so idle
    lanes count) times the instructions of one lane-step (10W + 16)."""
    best = None
    for W in widths:
        L = math.ceil(w / W)
        if not 2 <= L <= 32:
            continue
        cost = (32.0 / (32 // L)) * (10 * W + 16)
        if best is None or cost < best[0]:
            best = (cost, W, L)
    return None if best is None else [best[1], best[2]]


BATCHED_MODEL_WORDS = range(33, 513)  # buckets the persistent kernel's widths (<= 16) hold


def refill_batched_long(table, widths):
    """The large-batch table of the batched path: buckets of 33..512 words by
    model_shape."""
    for w in BATCHED_MODEL_WORDS:
        shape = model_shape(w, [W for W in widths if W <= 16])
        if shape:
            table[str(w)] = shape


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "autotune_b200.json"))
    ap.add_argument("--quick", action="store_true", help="fewer buckets (smoke runs)")
    ap.add_argument("--refill-batched-long", action="store_true",
                    help="rewrite the batched path's long buckets of an existing cache by the cost model")
    args = ap.parse_args()
    if args.refill_batched_long:
        os.environ["MYERS_AUTOTUNE"] = "0"
        import myersgpu as mg
        widths = sorted(W for _, W, multi in mg.variants() if multi)
        with open(args.out) as f:
            cache = json.load(f)
        cache["batched_large"] = {}
        refill_batched_long(cache["batched_large"], widths)
        cache["method"] = cache["method"].split("; batched")[0] + \
            "; batched_large (batches of 150K candidates or more), 33..512 words: the cost model over " + \
            "multi-lane widths " + ",".join(str(W) for W in widths if W <= 16)
        with open(args.out, "w") as f:
            json.dump(cache, f)
        print("rewrote", args.out)
        return
    os.environ["MYERS_AUTOTUNE"] = "0"  # tune against the cost model, not an older cache
    import torch

    import myersgpu as mg
    torch.cuda.set_device(0)
    ref_size = 200_000_000
    ref_words = mg.make_reference(ref_size, 77)
    ref = mg.Reference(ref_words, ref_size)
    buckets = list(range(1, 33)) + LONG_SAMPLE
    if args.quick:
        buckets = [1, 4, 13, 32, 64, 313]
    measured = {"plain": {}, "batched": {}}
    t_start = time.time()
    stream = torch.cuda.current_stream()
    for w in buckets:
        m = 32 * w
        cells = 1.4 * m * m
        # large batches (about 1e13 cells: many waves of the widest shapes), so
        # the choice is the shape that sustains the highest throughput rather
        # than the one that best fills a GPU too large for the batch
        n_cands = int(min(4_000_000, max(20_000, 1e13 / cells)))
        s = mg.spec(ref_size, max(1, n_cands // 11), 1000 + w, lengths=m, cands=11)
        wl = mg.make_workload(s, ref_words)
        n = len(wl["cands"])

        def dev(a):
            return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).cuda()

        d_peq, d_qi, d_c = dev(wl["peq"]), dev(wl["qinfo"]), dev(wl["cands"])
        d_res = torch.empty(n * 8, dtype=torch.uint8, device="cuda")
        ctx = mg.Context(n)
        for pname, path in (("plain", mg.PATH_PLAIN), ("batched", mg.PATH_BATCHED)):
            rows = []
            for v, L in candidate_shapes(mg, w, path):
                mg.set_shape_override(path, w, v, L)
                times = []
                for rep in range(4):
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    ctx.verify(ref, d_peq.data_ptr(), len(wl["peq"]), d_qi.data_ptr(), len(wl["qinfo"]),
                               d_c.data_ptr(), n, DIST, d_res.data_ptr(), path=path, stream=stream.cuda_stream,
                               min_size=m, max_size=m)
                    b.record(stream)
                    torch.cuda.synchronize()
                    if rep:
                        times.append(a.elapsed_time(b))
                mg.set_shape_override(path, w, -1)
                rows.append([v, L, mg.lib.myersVariantWords(v), n / (min(times) / 1e3)])
            best = max(rows, key=lambda r: r[3])
            measured[pname][w] = {"shape": best[:3], "cand_s": best[3], "all": rows, "m": m, "candidates": n}
        ctx.close()
        print(f"w={w:5d} m={m:6d} n={n:8d} plain={measured['plain'][w]['shape']} "
              f"batched={measured['batched'][w]['shape']} ({time.time() - t_start:.0f}s)", flush=True)

    table = {"plain": {}, "batched": {}, "batched_large": {}}
    widths = {W: v for v, W, multi in mg.variants() if multi}
    refill_batched_long(table["batched_large"], sorted(widths))
    for pname in ("plain", "batched"):
        sampled = sorted(measured[pname])
        for w in range(1, 1025):
            if w in measured[pname]:
                v, L, W = measured[pname][w]["shape"]
                table[pname][w] = [W, L]
                continue
            above = [x for x in sampled if x >= w]
            ref_w = above[0] if above else sampled[-1]
            v, L, W = measured[pname][ref_w]["shape"]
            if L == 1:  # a single-lane winner above 32 words cannot happen; keep the cost model
                continue
            for W2 in sorted(widths):
                if W2 < W:
                    continue
                if pname == "batched" and W2 > 16 and w <= 512:
                    continue
                L2 = math.ceil(w / W2)
                if 2 <= L2 <= 32:
                    table[pname][w] = [W2, L2]
                    break
    props = torch.cuda.get_device_properties(0)
    out = {"device": props.name, "sms": props.multi_processor_count, "distance": DIST,
           "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
           "method": "per bucket: every compiled shape timed on reads of 32*w bases (about 1e13 cells, 20K..4M candidates), best of 3 after a warm-up",
           "format": "plain/batched: words -> [W words per lane, L lanes per candidate]",
           "plain": {str(k): v for k, v in table["plain"].items()},
           "batched": {str(k): v for k, v in table["batched"].items()},
           "batched_large": table["batched_large"],
           "measured": {p: {str(k): v for k, v in measured[p].items()} for p in measured}}
    with open(args.out, "w") as f:
        json.dump(out, f)
    ref.close()
    print("wrote", args.out)


if __name__ == "__main__":
    main()
