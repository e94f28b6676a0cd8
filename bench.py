"""Benchmark of Myers candidate verification on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload 1..5]
                    [--path plain|batched] [--impl ours|reference]

One step = one verification pass over the whole batch of the workload (all
candidates of all reads, inputs resident in HBM). Default workload: 1M reads
of 1,000 bases, 11 candidates each (11M candidates), over a 3.1 Gbase
synthetic reference -- the full-shape plain Myers configuration. Prints one
JSON line (rank 0).

  value     candidates/s over the timed steps, kernels on HBM-resident inputs
            (N GPUs: each rank verifies its own seeded batch; the sum of
            candidates / the slowest rank's time)
  e2e       the same metric through the drop-in C API (initMyers /
            sendMyersBuffer / receiveMyersBuffer) from pinned host buffers:
            H2D of PEQ, query info and candidates and D2H of the results are
            inside the timed region
  roofline  the Myers kernel against the measured integer-ALU peak (3-input
            logic ops/s probed in this run): achieved = word-steps x 11 ops
            per launch / launch time
  parity    a seeded random 10% of the timed results against the reference's
            own CPU Myers (computeAllQueriesCPU, compiled from its sources
            into oracle/_ref), bit for bit
  cpu_baseline  that same reference run: its candidates / its seconds on the
            host cores
  configs   (1 GPU, default workload) the other configurations, each with its
            own timing, clocks, roofline fraction and reference parity sample:
            plain-100b, batched-mixed (batched and plain, full size and a
            110K-candidate batch), batched-long, plain-1000b and batched-mixed
            under Ukkonen's cut-off, and a short serving sweep

--impl reference times the reference's own CPU implementation instead (the
GPU path of the reference targets sm_20..sm_50 only).
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "myers-gpu_b200"))

DIST = 0.2
OPS_PER_WORD_STEP = 11  # the fused recurrence: PEQ select + 10 logic/add/shift ops
L2_NOTE = "L2 flushed before every timed step (256 MiB write, untimed)"

WORKLOAD_NAMES = {
    1: "plain-100b: 16 Mbase ref, 100K reads x 100 b, 11 cand/read (1.1M candidates)",
    2: "plain-1000b: 3.1 Gbase ref, 1M reads x 1000 b, 11 cand/read (11M candidates)",
    3: "batched-mixed: 3.1 Gbase ref, 2M reads of 100..1000 b, 1+Poisson(10) cand/read",
    4: "batched-long: 3.1 Gbase ref, 100K reads of 1000..10000 b, 1+Poisson(4) cand/read",
    5: "serving-mix: 3.1 Gbase ref, 300K requests of one read (100..1000 b) and 1..64 candidates",
}
# offered rates (candidates/s) of the serving sweep in the default line: the
# low end and the region around the knee
SERVING_RATES_SHORT = [1e6, 2e7, 5e7, 7e7, 7.8e7, 8.2e7, 8.6e7, 9e7, 9.5e7]
SERVING_RATES_FULL = [1e4, 1e5, 1e6, 2e6, 5e6, 1e7, 2e7, 3e7, 4e7, 5e7, 6e7, 7e7, 7.5e7, 8e7, 8.2e7, 8.4e7, 8.6e7,
                      8.8e7, 9e7, 9.2e7, 9.5e7, 1e8, 1.1e8]


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", type=int, default=2, choices=[1, 2, 3, 4, 5])
    ap.add_argument("--path", default=None, choices=["plain", "batched"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="fraction of the workload's reads (tests)")
    ap.add_argument("--parity-frac", type=float, default=0.1,
                    help="fraction of the timed results checked against the reference's CPU Myers")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="no reference parity / CPU baseline run")
    ap.add_argument("--no-configs", action="store_true", help="only the selected workload (no other configurations)")
    ap.add_argument("--lane-words", type=int, default=12, help="serving: words per lane of the latency shapes")
    ap.add_argument("--slots", type=int, default=4, help="serving: batches in flight")
    ap.add_argument("--max-batch", type=int, default=0, help="serving: candidates per batch (0: the server's default)")
    ap.add_argument("--no-graphs", action="store_true", help="serving: launch batches without CUDA graphs")
    ap.add_argument("--cutoff", type=float, default=None,
                    help="Ukkonen's cut-off: report minima above (uint32)(m * CUTOFF) as no match, skipping rows")
    ap.add_argument("--shape", type=int, default=0,
                    help="verify every length bucket with multi-lane lanes of this many words (0: tuned shapes)")
    ap.add_argument("--traceback", action="store_true",
                    help="time the traceback of the workload's candidates within --tb-bound x m")
    ap.add_argument("--tb-bound", type=float, default=0.2, help="traceback: score bound as a fraction of m")
    ap.add_argument("--tb-scratch-gb", type=float, default=16.0, help="traceback: scratch for the stored bands")
    return ap.parse_args()


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.skip = 0
        self.pokes = []
        self.nvml = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = (pynvml, pynvml.nvmlDeviceGetHandleByIndex(gpu_index))
        except Exception:  # no NVML: the nvidia-smi rows alone
            self.nvml = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        # wait for the first row, so that the sampler runs when the timed region starts;
        # rows written before the region are dropped
        t0 = time.time()
        while time.time() - t0 < 5 and os.path.getsize(self.out.name) == 0:
            time.sleep(0.01)
        self.out.flush()
        self.skip = len(open(self.out.name).read().strip().splitlines())

    def poke(self):
        """One NVML reading, taken while queued steps run (covers timed regions
        shorter than the sampler's 200 ms period)."""
        if self.nvml is None:
            return
        nv, h = self.nvml
        try:
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        except Exception:
            return
        masks = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}
        self.pokes.append((float(sm), float(smax), {n for n, m in masks.items() if bits & m}))

    def stop(self):
        rows = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.out.flush()
            self.out.seek(0)
            rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.strip()][self.skip:]
        os.unlink(self.out.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for name, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        for c, cmax, rs in self.pokes:
            sm.append(c)
            smax = cmax
            reasons |= rs
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def reduce_over_ranks(dist, elapsed_s, n_cands, cells, device):
    """Whole-job numbers of a replicas run: the slowest rank's timed seconds,
    and the candidates and DP cells all ranks verified."""
    import torch
    t = torch.tensor([elapsed_s], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    tot = torch.tensor([float(n_cands), float(cells)], dtype=torch.float64, device=device)
    dist.all_reduce(tot)
    return float(t.item()), float(tot[0].item()), float(tot[1].item())


def all_ranks_true(dist, flag, device="cuda"):
    """True on every rank iff `flag` is true on every rank."""
    import torch
    t = torch.tensor([1 if flag else 0], dtype=torch.int32, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN)
    return bool(t.item())


_REF_CACHE = {}


def reference_words(ms, k):
    """The packed synthetic reference of workload k: 16 Mbases for plain-100b,
    one shared 3.1 Gbase reference for the others (generated once)."""
    s = ms.workload_spec(k)
    key = (s.ref_size, 1000 + (s.seed if k == 1 else 0))
    if key not in _REF_CACHE:
        _REF_CACHE[key] = ms.make_reference(*key)
    return _REF_CACHE[key], int(s.ref_size)


def make_inputs(ms, k, scale, seed_offset, num_reads=None):
    s = ms.workload_spec(k, scale=scale)
    s.seed += 7919 * seed_offset
    if num_reads is not None:
        s.num_reads = min(s.num_reads, num_reads)
    ref_words, ref_size = reference_words(ms, k)
    w = ms.make_workload(s, ref_words)
    return s, ref_words, ref_size, w


def write_ref_file(tmp, ref_words, ref_size):
    """The reference as a .4bits.ref file (u32 words, u32 bases, words), the
    format the drop-in initMyers loads."""
    fn = os.path.join(tmp, f"bench.{ref_size}.4bits.ref")
    if not os.path.exists(fn):
        with open(fn, "wb") as f:
            f.write(np.array([len(ref_words), ref_size], dtype=np.uint32).tobytes())
            ref_words.tofile(f)
    return fn


def workload_units(ms, w):
    cells, word_steps = ms.cells(w["qinfo"], w["cands"], DIST)
    return float(cells.sum()), float(word_steps.sum())


def device_run(mg, ref, w, path, steps, warmup, local=0, dist=None, cutoff=None):
    """Time `steps` verification passes of workload w (inputs resident in HBM)
    with CUDA events on the launching stream, L2 flushed before every step,
    clocks sampled during the timed region. Returns per-step milliseconds, the
    last step's results, the launches per step and the clock record."""
    import torch
    n = len(w["cands"])
    ctx = mg.Context(n)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).to("cuda")

    d_peq, d_qi, d_c = dev(w["peq"]), dev(w["qinfo"]), dev(w["cands"])
    d_res = torch.empty(n * 8, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    lengths = w["qinfo"]["size"]
    lo, hi = int(lengths.min()), int(lengths.max())

    def step():
        ctx.verify(ref, d_peq.data_ptr(), len(w["peq"]), d_qi.data_ptr(), len(w["qinfo"]), d_c.data_ptr(), n, DIST,
                   d_res.data_ptr(), path=path, stream=stream.cuda_stream, min_size=lo, max_size=hi, cutoff=cutoff)

    try:
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        launches = ctx.launches()
        clocks = ClockSampler(local)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        clocks.start()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, b in evs:
            flush.zero_()
            a.record(stream)
            step()
            b.record(stream)
        clocks.poke()
        torch.cuda.synchronize()
        clk = clocks.stop()
        del flush
        if dist is not None:
            dist.barrier()
        step_ms = [a.elapsed_time(b) for a, b in evs]
        res = d_res.cpu().numpy().view(mg.RES).copy()
    finally:
        ctx.close()
        del d_peq, d_qi, d_c, d_res
        torch.cuda.empty_cache()
    return {"step_ms": step_ms, "res": res, "launches": launches, "clocks": clk}


def reference_parity(w, res, ref_words, ref_size, frac, seed, threads, padded=None, cutoff=None):
    """Check a seeded random fraction of the results against the reference's
    own CPU Myers (computeAllQueriesCPU of
    src-integration/myers-reorderBuffer-padding.c:178-208, compiled into
    oracle/_ref; reads beyond its 4096-base cap through its computeMyers,
    :97-176), or the restated oracle where oracle/_ref is not built. Returns
    (parity record, CPU rate record of that same run)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    n = len(w["cands"])
    k = max(1, min(n, int(math.ceil(frac * n))))
    idx = np.arange(n) if k >= n else np.sort(np.random.default_rng(seed).choice(n, size=k, replace=False))
    sub = np.ascontiguousarray(w["cands"][idx])
    if orc.have_reference():
        expect, sec = orc.reference_verify_aligned(w["peq"], w["qinfo"], sub, ref_words, ref_size, DIST,
                                                   nthreads=threads, padded=padded)
        kind, who = "reference", "the reference's computeAllQueriesCPU (oracle/_ref)"
    else:
        t = time.perf_counter()
        expect = orc.verify(w["peq"], w["qinfo"], sub, ref_words, ref_size, DIST, nthreads=threads)
        sec = time.perf_counter() - t
        kind, who = "port", "the restated oracle (oracle/myers_oracle.c)"
    if cutoff is not None:
        expect = orc.apply_cutoff(expect, w["qinfo"], sub, cutoff)
    mism = int(np.count_nonzero(res[idx] != expect))
    parity = {"candidates": int(k), "fraction": k / n, "oracle": who, "bit_exact": mism == 0, "mismatches": mism}
    m = w["qinfo"]["size"][sub["query"]].astype(np.float64)
    f = np.float32(1.0) + np.float32(2.0) * np.float32(DIST)
    wb = np.floor(m.astype(np.float32) * f).astype(np.float64)
    cells = float((m * 8 * (np.floor(wb / 8) + np.where(wb % 8 != 0, 2, 1))).sum())
    what = "all" if k >= n else f"a seeded random {100 * k / n:.0f}% ({k})"
    cpu = {"value": k / sec, "unit": "candidates/s", "cores": threads, "kind": kind, "gcups": cells / sec / 1e9,
           "sample": f"{what} of the {n} candidates of the same workload, {sec:.1f} s, OpenMP over {threads} threads"}
    return parity, cpu


def roofline(peak, word_steps, kernel_s):
    achieved = word_steps * OPS_PER_WORD_STEP / kernel_s
    return {"bound": "int32-alu", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "Tops/s",
            "frac": achieved / peak}


def run_reference(args):
    import myerssynth as ms  # the generator only: no CUDA library in this process
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    k = args.workload
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    threads = host_threads()
    kind = "reference" if orc.have_reference() else "port"
    per_step = max(1.0, min(10.0, 120.0 / max(1, args.steps + args.warmup)))
    s, ref_words, ref_size, w = make_inputs(ms, k, args.scale, 0, num_reads=max(1, 2000 // (10 if k in (2, 4) else 1)))
    padded = orc.pad_reference(ref_words) if kind == "reference" else None

    def run(w):
        if kind == "reference":
            return orc.reference_verify_aligned(w["peq"], w["qinfo"], w["cands"], ref_words, ref_size, DIST,
                                                nthreads=threads, padded=padded)[1]
        t = time.perf_counter()
        orc.verify(w["peq"], w["qinfo"], w["cands"], ref_words, ref_size, DIST, nthreads=threads)
        return time.perf_counter() - t

    sec = max(run(w), 1e-4)
    full = ms.workload_spec(k, scale=args.scale)
    total_reads = full.num_reads
    full_cands = len(ms.make_workload(full, ref_words)["cands"])
    s.num_reads = int(max(len(w["qinfo"]), min(total_reads, per_step / (sec / len(w["qinfo"])))))
    w = ms.make_workload(s, ref_words)
    for _ in range(args.warmup):
        run(w)
    times = [run(w) for _ in range(args.steps)]
    t = float(np.mean(times))
    cps = len(w["cands"]) / t
    cells, _ = ms.cells(w["qinfo"], w["cands"], DIST)
    line = {"impl": "reference", "metric": "candidates/s", "value": cps, "unit": "candidates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded)", "gcups": float(cells.sum() / t / 1e9),
            "config": {"workload": WORKLOAD_NAMES[k], "candidates_per_gpu": full_cands, "distance": DIST,
                       "window": "aligned",
                       "path": "the reference's CPU Myers (computeAllQueriesCPU)" if kind == "reference"
                       else "CPU port of the reference algorithm",
                       "l2": "host caches (CPU)", "parallelism": f"{threads} host threads",
                       "sample_candidates_per_step": len(w["cands"]),
                       "sample_fraction": len(w["cands"]) / full_cands},
            "cpu_baseline": {"value": cps, "unit": "candidates/s", "cores": threads, "kind": kind,
                             "sample": f"each step: first {s.num_reads} reads ({len(w['cands'])} candidates, "
                                       f"{100 * len(w['cands']) / full_cands:.1f}% of the workload), "
                                       f"OpenMP over {threads} threads"},
            "e2e": {"value": cps, "unit": "candidates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch

    import myersgpu as mg
    import myerssynth as ms
    world, rank, local, dist = dist_setup(args)
    torch.cuda.set_device(local)
    k = args.workload
    path = {"plain": mg.PATH_PLAIN, "batched": mg.PATH_BATCHED}[args.path or ("batched" if k in (3, 4, 5) else "plain")]
    s, ref_words, ref_size, w = make_inputs(ms, k, args.scale, rank)
    n_cands = len(w["cands"])
    lengths = w["qinfo"]["size"]
    cells, ws_total = workload_units(ms, w)

    ref = mg.Reference(ref_words, ref_size)
    shape_note = None
    if args.shape:
        # one multi-lane shape per length bucket: lanes of args.shape words
        v = [v for v, W, multi in mg.variants() if multi and W == args.shape]
        if not v:
            raise SystemExit(f"no multi-lane shape with {args.shape} words per lane")
        for words in np.unique((lengths.astype(np.int64) + 31) // 32):
            mg.set_shape_override(path, int(words), v[0], max(2, -(-int(words) // args.shape)))
        shape_note = f"every bucket: lanes of {args.shape} words (override)"

    run = device_run(mg, ref, w, path, args.steps, args.warmup, local, dist, args.cutoff)
    step_ms, res, clk = run["step_ms"], run["res"], run["clocks"]
    elapsed = sum(step_ms) / 1e3
    if dist is not None:
        elapsed, all_cands, all_cells = reduce_over_ranks(dist, elapsed, n_cands, cells, "cuda")
    else:
        all_cands, all_cells = float(n_cands), cells
    value = all_cands * args.steps / elapsed
    gcups = all_cells * args.steps / elapsed / 1e9

    # roofline: the dominant kernel is the whole step on the plain single-launch path
    peak = mg.probe_int_peak(4000)
    kernel_s = float(np.mean(step_ms)) / 1e3
    roof = roofline(peak, ws_total, kernel_s)
    _, word_steps = ms.cells(w["qinfo"], w["cands"], DIST)
    hbm_bytes = float(len(w["peq"]) * 80 + len(w["qinfo"]) * 8 + n_cands * (16 + 8)
                      + (word_steps / np.ceil(w["qinfo"]["size"][w["cands"]["query"]] / 32) / 2).sum())
    peaks_file = os.path.join(ROOT, "MEASURED_PEAKS.json")
    hbm_peak = json.load(open(peaks_file)).get("hbm_gbs") if os.path.exists(peaks_file) else 6650.0
    traffic = None
    prof = os.path.join(ROOT, "profiles", f"traffic_workload{k}.json")
    if os.path.exists(prof):
        traffic = json.load(open(prof))["dram_bytes_per_candidate"] * n_cands
    roof.update({"traffic": traffic,
                 "peak_source": "3-input logic op probe (LOP3, 8 independent chains) in this run",
                 "ops_per_word_step": OPS_PER_WORD_STEP,
                 "hbm": {"achieved_gbs": hbm_bytes / kernel_s / 1e9, "peak_gbs": hbm_peak,
                         "frac": hbm_bytes / kernel_s / 1e9 / hbm_peak}})

    tmp = tempfile.TemporaryDirectory()
    # end to end through the drop-in API
    e2e = None
    if not args.no_e2e and args.cutoff is None:
        e2e = run_e2e(mg, args, write_ref_file(tmp.name, ref_words, ref_size), ref_size, w, path, dist)
        if "_results" in e2e:
            e2e["results_equal_device"] = bool(np.array_equal(e2e.pop("_results"), res))
        if dist is not None:
            # whole job: all ranks' candidates over the slowest rank's seconds
            # (every rank takes part in the same reductions, even without a value)
            ok = bool(e2e.get("value"))
            el_e2e = n_cands * args.steps / e2e["value"] if ok else float("inf")
            el_max, all_c, _ = reduce_over_ranks(dist, el_e2e, n_cands, 0.0, "cuda")
            ok = all_ranks_true(dist, ok)
            same = all_ranks_true(dist, e2e.get("results_equal_device", False))
            if ok:
                e2e["value"] = all_c * args.steps / el_max
                e2e["h2d_bytes_per_step"] *= world
                e2e["d2h_bytes_per_step"] *= world
                e2e["results_equal_device"] = same
            else:
                e2e = {"value": None, "unit": "candidates/s", "note": "a rank's buffers were too small"}

    # parity of the timed results: 1 GPU against the reference's own CPU Myers
    # on a seeded 10% (its time is the CPU baseline); N GPUs, where all ranks
    # share the host, a 2,000-candidate sample per rank against the restated oracle
    cpu = None
    threads = host_threads()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    padded = orc.pad_reference(ref_words) if orc.have_reference() and world == 1 and not args.no_cpu else None
    if world == 1 and not args.no_cpu:
        parity, cpu = reference_parity(w, res, ref_words, ref_size, args.parity_frac, 11, threads, padded,
                                       args.cutoff)
    else:
        idx = np.random.default_rng(rank).choice(n_cands, size=min(2000, n_cands), replace=False)
        expect = orc.verify(w["peq"], w["qinfo"], w["cands"][idx], ref_words, ref_size, DIST)
        if args.cutoff is not None:
            expect = orc.apply_cutoff(expect, w["qinfo"], w["cands"][idx], args.cutoff)
        ok = bool(np.array_equal(res[idx], expect))
        if dist is not None:
            ok = all_ranks_true(dist, ok)
        parity = {"candidates": int(len(idx)) * world, "fraction": len(idx) / n_cands,
                  "oracle": "the restated oracle (oracle/myers_oracle.c)", "bit_exact": ok}
    del w, res

    configs = None
    if rank == 0 and world == 1 and k == 2 and not args.no_configs and args.scale == 1.0 and args.cutoff is None:
        configs = run_configs(mg, ms, args, ref, peak, tmp.name, threads, padded)
    ref.close()
    tmp.cleanup()
    if rank == 0:
        line = {
            "metric": "candidates/s", "value": value, "unit": "candidates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)",
            "gcups": gcups,
            "config": {"workload": WORKLOAD_NAMES[k], "candidates_per_gpu": n_cands, "distance": DIST,
                       "window": "aligned", "path": "batched" if path == mg.PATH_BATCHED else "plain",
                       "l2": L2_NOTE, "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       **({"shapes": shape_note} if shape_note else {}),
                       **({"cutoff": args.cutoff} if args.cutoff is not None else {})},
            "roofline": roof, "e2e": e2e, "cpu_baseline": cpu, "clocks": clk,
            "gpu_launches": run["launches"] * args.steps,
            "parity_sample": parity,
        }
        if configs is not None:
            line["configs"] = configs
            line["targets"] = targets_summary(value, configs)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def config_record(mg, ms, ref, w, path, steps, warmup, peak, ref_words, ref_size, threads, padded, parity_frac,
                  seed, cutoff=None):
    """One configuration's figures: device-resident candidates/s with its
    clocks, the roofline fraction, and a reference parity sample whose time
    is the CPU baseline."""
    n = len(w["cands"])
    cells, ws = workload_units(ms, w)
    r = device_run(mg, ref, w, path, steps, warmup, cutoff=cutoff)
    t = float(np.mean(r["step_ms"])) / 1e3
    rec = {"path": "batched" if path == mg.PATH_BATCHED else "plain", "candidates": n, "value": n / t,
           "unit": "candidates/s", "ms_per_step": t * 1e3, "steps": steps, "warmup": warmup, "gcups": cells / t / 1e9,
           "roofline_frac": roofline(peak, ws, t)["frac"], "launches_per_step": r["launches"], "clocks": r["clocks"]}
    if parity_frac > 0:
        rec["parity_sample"], rec["cpu_baseline"] = reference_parity(w, r["res"], ref_words, ref_size, parity_frac,
                                                                     seed, threads, padded, cutoff)
    return rec, r["res"]


def run_configs(mg, ms, args, ref3, peak, tmp, threads, padded3):
    """The benchmark's other configurations, each on the same GPU in this run:
    plain-100b (with its e2e), batched-mixed on both paths at full size and at
    110K candidates (with the batched path's e2e), batched-long on both paths,
    the cut-off on plain-1000b and batched-mixed, the traceback of
    plain-1000b, and a short serving sweep. Steps per configuration are capped so the whole
    line stays within a few minutes."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    steps, warmup = min(args.steps, 10), min(args.warmup, 3)
    out = {}

    # plain-100b: its own 16 Mbase reference; all of its candidates checked
    _, rw1, rs1, w1 = make_inputs(ms, 1, 1.0, 0)
    ref1 = mg.Reference(rw1, rs1)
    try:
        rec, res = config_record(mg, ms, ref1, w1, mg.PATH_PLAIN, max(steps, 20), warmup, peak, rw1, rs1, threads,
                                 orc.pad_reference(rw1) if padded3 is not None else None, 1.0, 101)
        e2e = run_e2e(mg, argparse.Namespace(steps=steps, warmup=warmup), write_ref_file(tmp, rw1, rs1), rs1, w1,
                      mg.PATH_PLAIN)
        if "_results" in e2e:
            e2e["results_equal_device"] = bool(np.array_equal(e2e.pop("_results"), res))
        rec["e2e"] = e2e
    finally:
        ref1.close()
    out["plain-100b"] = {"workload": WORKLOAD_NAMES[1], **rec}
    del w1, res

    rw, rs = reference_words(ms, 3)
    fn = write_ref_file(tmp, rw, rs)
    # batched-mixed at full size, both paths
    _, _, _, w3 = make_inputs(ms, 3, 1.0, 0)
    b, resb = config_record(mg, ms, ref3, w3, mg.PATH_BATCHED, steps, warmup, peak, rw, rs, threads, padded3,
                            args.parity_frac, 303)
    e2e = run_e2e(mg, argparse.Namespace(steps=steps, warmup=warmup), fn, rs, w3, mg.PATH_BATCHED)
    if "_results" in e2e:
        e2e["results_equal_device"] = bool(np.array_equal(e2e.pop("_results"), resb))
    b["e2e"] = e2e
    p, resp = config_record(mg, ms, ref3, w3, mg.PATH_PLAIN, steps, warmup, peak, rw, rs, threads, padded3, 0.0, 0)
    p["results_equal_batched"] = bool(np.array_equal(resp, resb))
    out["batched-mixed"] = {"workload": WORKLOAD_NAMES[3], "batched": b, "plain": p,
                            "batched_over_plain": b["value"] / p["value"]}
    del w3, resb, resp

    # batched-mixed, a 110K-candidate batch (0.5% of the reads): where one
    # persistent launch and per-shape launches differ most
    _, _, _, ws3 = make_inputs(ms, 3, 0.005, 0)
    bs, resb = config_record(mg, ms, ref3, ws3, mg.PATH_BATCHED, max(steps, 20), warmup, peak, rw, rs, threads,
                             padded3, 1.0, 304)
    ps, resp = config_record(mg, ms, ref3, ws3, mg.PATH_PLAIN, max(steps, 20), warmup, peak, rw, rs, threads,
                             padded3, 0.0, 0)
    ps["results_equal_batched"] = bool(np.array_equal(resp, resb))
    out["batched-mixed-110k"] = {"workload": WORKLOAD_NAMES[3] + ", first 0.5% of the reads", "batched": bs,
                                 "plain": ps, "batched_over_plain": bs["value"] / ps["value"]}
    del ws3, resb, resp

    # batched-long, both paths
    _, _, _, w4 = make_inputs(ms, 4, 1.0, 0)
    b4, resb = config_record(mg, ms, ref3, w4, mg.PATH_BATCHED, min(steps, 5), warmup, peak, rw, rs, threads,
                             padded3, args.parity_frac, 404)
    p4, resp = config_record(mg, ms, ref3, w4, mg.PATH_PLAIN, min(steps, 5), warmup, peak, rw, rs, threads,
                             padded3, 0.0, 0)
    p4["results_equal_batched"] = bool(np.array_equal(resp, resb))
    out["batched-long"] = {"workload": WORKLOAD_NAMES[4], "batched": b4, "plain": p4,
                           "batched_over_plain": b4["value"] / p4["value"]}
    del w4, resb, resp

    # plain-1000b under Ukkonen's cut-off at 0.08 m: the two-pass plain path
    # (its roofline fraction counts the full DP's word-steps, so it can exceed 1)
    _, _, _, w2 = make_inputs(ms, 2, 1.0, 0)
    cut, _ = config_record(mg, ms, ref3, w2, mg.PATH_PLAIN, steps, warmup, peak, rw, rs, threads, padded3, 0.02,
                           205, cutoff=0.08)
    out["plain-1000b-cutoff-0.08"] = {"workload": WORKLOAD_NAMES[2] + ", Ukkonen's cut-off at 0.08 m",
                                      "cutoff": 0.08, **cut}
    # traceback of plain-1000b: the alignments of the candidates scoring at most 0.2 m
    out["traceback-plain-1000b"] = {"workload": "traceback of " + WORKLOAD_NAMES[2],
                                    **traceback_record(mg, ref3, rw, rs, w2, min(steps, 5), warmup, 16.0, 0.2)}
    del w2

    # batched-mixed under the cut-off at 0.08 m: the two passes as two
    # persistent launches
    _, _, _, w3 = make_inputs(ms, 3, 1.0, 0)
    cutb, _ = config_record(mg, ms, ref3, w3, mg.PATH_BATCHED, steps, warmup, peak, rw, rs, threads, padded3,
                            0.02, 306, cutoff=0.08)
    out["batched-mixed-cutoff-0.08"] = {"workload": WORKLOAD_NAMES[3] + ", Ukkonen's cut-off at 0.08 m",
                                        "cutoff": 0.08, **cutb}
    del w3

    # serving: a short sweep around the knee
    out["serving"] = serving_sweep(mg, ms, args, ref3, rw, rs, SERVING_RATES_SHORT, steps=min(steps, 5),
                                   warmup=warmup, threads=threads, padded=padded3)
    return out


def targets_summary(value_plain_1000b, configs):
    """The targets, as measured in this line."""
    sv = configs["serving"]
    records = []  # every per-path record of every configuration
    for c in configs.values():
        records += [c[p] for p in ("batched", "plain") if p in c] or [c]
    samples = [r["parity_sample"] for r in records if "parity_sample" in r]
    same = ([r["results_equal_batched"] for r in records if "results_equal_batched" in r]
            + [r["e2e"]["results_equal_device"] for r in records if "results_equal_device" in (r.get("e2e") or {})]
            + [sv["results_equal_to_batched"]])
    return {
        "cutoff_0.08_over_plain_1000b": configs["plain-1000b-cutoff-0.08"]["value"] / value_plain_1000b,
        "cutoff_0.08_over_batched_mixed": (configs["batched-mixed-cutoff-0.08"]["value"] /
                                           configs["batched-mixed"]["batched"]["value"]),
        "batched_over_plain_mixed_full": configs["batched-mixed"]["batched_over_plain"],
        "batched_over_plain_mixed_110k": configs["batched-mixed-110k"]["batched_over_plain"],
        "batched_over_plain_long": configs["batched-long"]["batched_over_plain"],
        "serving_frac_of_batched_at_p99_le_5ms": sv["served_frac_of_batched"],
        "serving_p99_ms": (sv["best"] or {}).get("p99_ms"),
        "reference_parity_candidates": int(sum(p["candidates"] for p in samples)),
        "bit_exact_everywhere": all(p["bit_exact"] for p in samples) and all(same),
        "plain_1000b_cand_s": value_plain_1000b,
        "traceback_plain_1000b_alignments_s": configs["traceback-plain-1000b"]["value"],
    }


def run_e2e(mg, args, ref_file, ref_size, w, path, dist=None):
    """The metric through the drop-in API from pinned host buffers: every
    step copies its inputs in and its results out. When the resident
    reference is much larger than L2 (3.1 Gbase: 1.55 GB), steps stream
    through two buffers, as callers of the API do (one buffer's copies
    overlap the other's kernels). With a reference that fits L2, steps run
    one at a time on one buffer, with L2 flushed between them."""
    n_cands = len(w["cands"])
    nb = 2 if ref_size // 2 > (1 << 30) else 1
    need = len(w["peq"]) * 80 + len(w["qinfo"]) * 8 + n_cands * 32
    mg.lib.myersSetMemoryBudget(nb * (int(need * 1.3) + (64 << 20)))
    avg = int(w["qinfo"]["size"].mean())
    cpq = max(1, n_cands // max(1, len(w["qinfo"])))
    bufs = mg.Buffers(ref_file, num_buffers=nb, avg_query_size=avg, cands_per_query=cpq)
    try:
        bufs.set_path(path)
        for b in range(nb):
            ne, nq, nc = bufs.capacity(b)
            if ne < len(w["peq"]) or nq < len(w["qinfo"]) or nc < n_cands:
                return {"value": None, "unit": "candidates/s", "note": f"buffer capacity too small {(ne, nq, nc)}"}
            v_peq, v_qi, v_c, v_res = bufs.views(b)
            v_peq[: len(w["peq"])] = w["peq"]
            v_qi[: len(w["qinfo"])] = w["qinfo"]
            v_c[:n_cands] = w["cands"]

        def send(b):
            bufs.send(b, DIST, len(w["peq"]), len(w["qinfo"]), n_cands)

        for _ in range(max(1, args.warmup)):
            for b in range(nb):
                send(b)
            for b in range(nb):
                mg.check(bufs.receive(b), "receive")
        import torch
        el = 0.0
        if nb == 1:
            flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
            for _ in range(args.steps):
                flush.zero_()  # L2 flushed before every step, outside the timed call
                torch.cuda.synchronize()
                t = time.perf_counter()
                send(0)
                mg.check(bufs.receive(0), "receive")
                el += time.perf_counter() - t
            del flush
        else:
            torch.cuda.synchronize()
            if dist is not None:
                dist.barrier()  # ranks start the timed region together
            t = time.perf_counter()
            for i in range(min(nb, args.steps)):
                send(i % nb)
            for i in range(args.steps):
                mg.check(bufs.receive(i % nb), "receive")
                if i + nb < args.steps:
                    send((i + nb) % nb)
            el = time.perf_counter() - t
        # every step's results equal the device-resident run's (checked by the caller)
        res = bufs.views(0)[3][:n_cands].copy()
        h2d = len(w["peq"]) * 80 + len(w["qinfo"]) * 8 + n_cands * 16
        how = ("two buffers in flight: step i sends on buffer i % 2 once that buffer's step i-2 is received"
               if nb == 2 else "one buffer, one step at a time, L2 flushed between steps")
        return {"value": n_cands * args.steps / el, "unit": "candidates/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(n_cands * 8), "buffers": nb, "steps": args.steps,
                "api": "initMyers buffers: fill pinned host buffers (untimed), then sendMyersBuffer + "
                       "receiveMyersBuffer per step (H2D, kernels, D2H timed on the host clock); " + how,
                "_results": res}
    finally:
        bufs.close()
        mg.lib.myersSetMemoryBudget(0)


def serving_sweep(mg, ms, args, ref, ref_words, ref_size, rates, steps, warmup, threads, padded=None):
    """Open-loop Poisson arrivals of requests (one read of 100..1000 bases and
    1..64 candidates) into the serving loop at the given offered rates; p50/p99
    latency (arrival -> results on the host) and throughput per rate, beside
    the batched kernel's throughput on the same requests as one batch."""
    import torch
    # a pool of 300K requests (~9.8M candidates): ~0.1 s of load at the top rates
    s = ms.workload_spec(5, scale=3.0 * args.scale)
    w = ms.make_workload(s, ref_words)
    off = np.concatenate([[0], np.cumsum(w["ncands"])]).astype(np.uint32)
    n_req, n_cands = len(w["qinfo"]), len(w["cands"])
    mean_c = n_cands / n_req

    # batched kernel on all requests at once, inputs resident (the comparison point)
    ctx = mg.Context(n_cands)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).to("cuda")

    d_peq, d_qi, d_c = dev(w["peq"]), dev(w["qinfo"]), dev(w["cands"])
    d_res = torch.empty(n_cands * 8, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream()

    def step():
        ctx.verify(ref, d_peq.data_ptr(), len(w["peq"]), d_qi.data_ptr(), n_req, d_c.data_ptr(), n_cands, DIST,
                   d_res.data_ptr(), path=mg.PATH_BATCHED, stream=st.cuda_stream, min_size=100, max_size=1000)

    for _ in range(warmup):
        step()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(steps):
        step()
    b.record(st)
    torch.cuda.synchronize()
    batched_cps = n_cands * steps / (a.elapsed_time(b) / 1e3)
    batched_res = d_res.cpu().numpy().view(mg.RES).copy()
    # the same, with the shapes the server picks (latency shapes), to split the
    # serving gap into shape cost and serving-loop cost
    same_cps = None
    if args.lane_words > 0:
        # the server's latency policy: the cheapest multi-lane shape with lanes
        # of at most lane_words words (lanes x (10W + 16) per column step)
        multi = [(v, W) for v, W, m in mg.variants() if m and W <= 16]

        def latency_shape(wd):
            best = None
            for v, W in multi:
                L = -(-wd // W)
                if (W > args.lane_words and W != multi[0][1]) or not 2 <= L <= 32:
                    continue
                cost = (32.0 / (32 // L)) * (10 * W + 16)
                if best is None or cost < best[0]:
                    best = (cost, v, L)
            return best[1], best[2]

        words = range(args.lane_words + 1, 33)
        for wd in words:
            mg.set_shape_override(mg.PATH_BATCHED, wd, *latency_shape(wd))
        for _ in range(2):
            step()
        a.record(st)
        for _ in range(steps):
            step()
        b.record(st)
        torch.cuda.synchronize()
        same_cps = n_cands * steps / (a.elapsed_time(b) / 1e3)
        for wd in words:
            mg.set_shape_override(mg.PATH_BATCHED, wd, -1)
    ctx.close()
    del d_peq, d_qi, d_c, d_res
    torch.cuda.empty_cache()

    rng = np.random.default_rng(5)
    sweep, same = [], True
    clocks = ClockSampler(0)
    with mg.Server(ref, distance=DIST, slots=args.slots, lane_words=args.lane_words, graphs=not args.no_graphs,
                   max_batch_candidates=args.max_batch) as srv:
        clocks.start()
        for rate in rates:
            k = int(min(n_req, max(300, rate * 1.0 / mean_c)))  # about one second of load
            gaps = rng.exponential(mean_c / rate * 1e9, size=k)
            arrivals = np.cumsum(gaps).astype(np.uint64)
            stt, lat, res, wall = srv.replay(w["peq"], w["qinfo"][:k], off[:k + 1], w["cands"]["position"], arrivals)
            ok = lat < np.iinfo(np.uint64).max
            cands_done = int(off[k]) if ok.all() else int(sum(off[i + 1] - off[i] for i in np.nonzero(ok)[0]))
            same &= bool(np.array_equal(res[:off[k]], batched_res[:off[k]]))
            sweep.append({"offered_cand_s": rate, "requests": k, "refused": int((~ok).sum()),
                          "throughput_cand_s": cands_done / (wall / 1e9),
                          "p50_ms": float(np.percentile(lat[ok], 50) / 1e6), "p99_ms": float(np.percentile(lat[ok], 99) / 1e6),
                          "status": int(stt)})
            clocks.poke()
        stats = srv.stats()
    clk = clocks.stop()
    good = [r for r in sweep if r["p99_ms"] <= 5.0 and r["refused"] == 0]
    best = max(good, key=lambda r: r["throughput_cand_s"]) if good else None
    value = best["throughput_cand_s"] if best else 0.0
    rec = {"workload": WORKLOAD_NAMES[5], "requests": n_req, "candidates": n_cands,
           "served_cand_s_at_p99_le_5ms": value, "best": best, "batched_cand_s": batched_cps,
           "served_frac_of_batched": value / batched_cps, "batched_same_shapes_cand_s": same_cps,
           "served_frac_of_batched_same_shapes": (value / same_cps) if same_cps else None,
           "results_equal_to_batched": same, "batches": stats["batches"],
           "largest_batch_candidates": stats["batchCandidatesMax"],
           "server": {"slots": stats["slots"], "max_batch_candidates": stats["maxBatchCandidates"],
                      "budget": "16 GiB", "lane_words": args.lane_words, "graphs": not args.no_graphs},
           "sweep": sweep, "clocks": clk}
    if threads:
        rec["parity_sample"], rec["cpu_baseline"] = reference_parity(w, batched_res, ref_words, ref_size,
                                                                     args.parity_frac, 505, threads, padded)
    return rec


def run_serving(args):
    """Workload 5 alone: the full offered-rate sweep."""
    import torch

    import myersgpu as mg
    import myerssynth as ms
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    torch.cuda.set_device(0)
    ref_words, ref_size = reference_words(ms, 5)
    ref = mg.Reference(ref_words, ref_size)
    try:
        rec = serving_sweep(mg, ms, args, ref, ref_words, ref_size, SERVING_RATES_FULL, args.steps, args.warmup,
                            0 if args.no_cpu else host_threads())
    finally:
        ref.close()
    value = rec["served_cand_s_at_p99_le_5ms"]
    line = {"metric": "candidates/s served at p99 <= 5 ms", "value": value, "unit": "candidates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded), open-loop Poisson arrivals",
            "config": {"workload": WORKLOAD_NAMES[5], "requests": rec["requests"], "candidates": rec["candidates"],
                       "distance": DIST, "server": rec["server"]},
            "serving": {k: v for k, v in rec.items() if k not in ("clocks", "server", "workload")},
            "e2e": {"value": value, "unit": "candidates/s",
                    "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                    "api": "myersServerSubmit/Wait through the replay driver: arrival to results on the host"},
            "clocks": rec["clocks"], "gpu_launches": None}
    print(json.dumps(line), flush=True)


def traceback_record(mg, ref, ref_words, ref_size, w, steps, warmup, scratch_gb, bound):
    """Traceback of the candidates whose score is within bound x the longest
    read: one step = one myersTraceback call over the verified batch
    (selection, the band-storing forward pass and the walk), inputs and
    results resident. Returns the timing, roofline, parity and CPU-baseline
    fields of a record."""
    import torch
    n = len(w["cands"])
    m_of = w["qinfo"]["size"][w["cands"]["query"]].astype(np.int64)
    max_score = int(bound * int(m_of.max()))
    ctx = mg.Context(n)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).to("cuda")

    d_peq, d_qi, d_c = dev(w["peq"]), dev(w["qinfo"]), dev(w["cands"])
    d_res = torch.empty(n * 8, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    ctx.verify(ref, d_peq.data_ptr(), len(w["peq"]), d_qi.data_ptr(), len(w["qinfo"]), d_c.data_ptr(), n, DIST,
               d_res.data_ptr(), path=mg.PATH_BATCHED, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    res = d_res.cpu().numpy().view(mg.RES)
    max_ops = 256  # runs per candidate: about 2 per edit of a traced alignment, plus one
    d_ops = torch.empty(n * max_ops, dtype=torch.int32, device="cuda")
    d_aln = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    tb = mg.Traceback(n, int(scratch_gb * (1 << 30)))
    try:
        def step():
            return tb.run(ref, d_peq.data_ptr(), len(w["peq"]), d_qi.data_ptr(), len(w["qinfo"]), d_c.data_ptr(),
                          d_res.data_ptr(), n, DIST, max_score, d_ops.data_ptr(), max_ops, d_aln.data_ptr(),
                          stream=stream.cuda_stream)

        for _ in range(warmup):
            traced = step()
        torch.cuda.synchronize()
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        clocks = ClockSampler(0)
        clocks.start()
        times = []
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            traced = step()
            b.record(stream)
            clocks.poke()
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b) / 1e3)
        clk = clocks.stop()
        del flush
        chunks = int(tb.chunks())
    finally:
        tb.close()
        ctx.close()
    t = float(np.mean(times))
    aln = d_aln.cpu().numpy().view(mg.ALN)
    ops = d_ops.cpu().numpy().view(np.uint32).reshape(n, max_ops)
    del d_peq, d_qi, d_c, d_res, d_ops, d_aln
    torch.cuda.empty_cache()
    sel = (res["score"] != mg.NO_RESULT) & (res["score"] <= max_score)
    # work of the forward pass: ceil(m/32) words x (end column + 1) columns per traced candidate
    ws = float((np.ceil(m_of[sel] / 32.0) * (res["column"][sel].astype(np.float64) + 1)).sum())
    peak = mg.probe_int_peak(4000)
    achieved = ws * OPS_PER_WORD_STEP / t
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    idx = np.nonzero(sel)[0]
    pick = np.random.default_rng(5).choice(idx, size=min(300, len(idx)), replace=False)
    e_aln, e_ops = orc.traceback(w["peq"], w["qinfo"], w["cands"][pick], res[pick], ref_words, ref_size, DIST,
                                 max_score, max_ops)
    # records compared whole; ops where they fit (else both leave them unspecified)
    ok = np.array_equal(aln[pick].view(np.uint32), e_aln.view(np.uint32)) and all(
        np.array_equal(ops[i, :e_aln["num_ops"][j]], e_ops[j, :e_aln["num_ops"][j]])
        for j, i in enumerate(pick) if e_aln["num_ops"][j] <= max_ops)
    overflow = int((aln["num_ops"][sel] > max_ops).sum())
    # CPU baseline: the oracle's DP traceback on a bounded sample, all host threads
    cores = host_threads()
    sample = idx[: max(1, min(len(idx), 4000))]
    t0 = time.perf_counter()
    orc.traceback(w["peq"], w["qinfo"], w["cands"][sample], res[sample], ref_words, ref_size, DIST, max_score,
                  max_ops, nthreads=cores)
    cpu_s = time.perf_counter() - t0
    return {
        "value": traced / t, "unit": "alignments/s", "ms_per_step": t * 1e3, "steps": steps, "warmup": warmup,
        "traced": int(traced), "candidates": n, "max_score": max_score, "max_ops": max_ops,
        "scratch_gib": scratch_gb,
        "roofline": {"bound": "int32-alu", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "Tops/s",
                     "frac": achieved / peak, "traffic": None,
                     "note": "whole call (selection, host read of the count, forward pass, walk) against the "
                             "forward pass's word-steps x 11"},
        "cpu_baseline": {"value": len(sample) / cpu_s, "unit": "alignments/s", "cores": cores, "kind": "port",
                         "sample": f"{len(sample)} traced candidates, the oracle's O(mn) DP traceback"},
        "parity_sample": {"candidates": int(len(pick)), "bit_exact": bool(ok)},
        "ops_overflow": overflow, "clocks": clk, "gpu_launches": 1 + 2 * chunks,
    }


def run_traceback(args):
    """The traceback line for one workload (--traceback)."""
    import torch

    import myersgpu as mg
    import myerssynth as ms
    torch.cuda.set_device(0)
    k = args.workload
    _, ref_words, ref_size, w = make_inputs(ms, k, args.scale, 0)
    ref = mg.Reference(ref_words, ref_size)
    try:
        r = traceback_record(mg, ref, ref_words, ref_size, w, args.steps, args.warmup, args.tb_scratch_gb,
                             args.tb_bound)
    finally:
        ref.close()
    line = {
        "metric": "alignments/s", "value": r["value"], "unit": "alignments/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)",
        "config": {"workload": "traceback of " + WORKLOAD_NAMES[k], "traced": r["traced"], "candidates": r["candidates"],
                   "max_score": r["max_score"], "max_ops": r["max_ops"], "scratch_gib": r["scratch_gib"],
                   "l2": L2_NOTE},
        **{key: r[key] for key in ("roofline", "cpu_baseline", "parity_sample", "ops_overflow", "clocks",
                                   "gpu_launches")},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.traceback:
        run_traceback(args)
    elif args.workload == 5:
        run_serving(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
