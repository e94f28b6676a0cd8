"""GPU parity of Ukkonen's cut-off (myersVerifyCutoffAsync, myersSetCutoff)
against the oracle: the reference-pinned results with the cut-off contract
applied (oracle.apply_cutoff: a minimum above (uint32_t)(m * cutoff) becomes
{NO_MATCH, NO_MATCH}; everything else unchanged). Integer outputs: bit-exact.
On the plain path the cut-off settles most candidates from the DP of a
prefix of their query and runs the rest in full, so these tests compare exact
scores and first columns wherever the minimum is within the bound, including
minima equal to it, and the no-match marker everywhere else."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIST = 0.2
CUTOFFS = [0.0, 0.04, 0.08, 0.2, 0.35, 1.0]


@pytest.fixture(scope="module")
def gpu(mg, cuda_ok):
    import torch
    torch.cuda.init()
    return mg


@pytest.fixture(scope="module")
def data(gpu):
    ref_size = 8_000_000
    ref_words = gpu.make_reference(ref_size, 4321)
    ref = gpu.Reference(ref_words, ref_size)
    ws = {k: gpu.make_workload(gpu.workload_spec(k, scale=sc, ref_size=ref_size), ref_words)
          for k, sc in ((1, 0.02), (2, 0.003), (3, 0.002), (4, 0.002), (5, 0.004))}
    yield ref_words, ref_size, ref, ws
    ref.close()


def _verify(gpu, ref, w, cutoff, window, path, min_size=0, max_size=0):
    ctx = gpu.Context(len(w["cands"]))
    try:
        return gpu.verify_torch(ctx, ref, w["peq"], w["qinfo"], w["cands"], DIST, window=window, path=path,
                                min_size=min_size, max_size=max_size, cutoff=cutoff)
    finally:
        ctx.close()


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("path", ["plain", "batched"])
def test_workloads_cutoff_vs_oracle(gpu, orc, data, k, path):
    ref_words, ref_size, ref, ws = data
    w = ws[k]
    full = orc.verify(w["peq"], w["qinfo"], w["cands"], ref_words, ref_size, DIST)
    p = gpu.PATH_PLAIN if path == "plain" else gpu.PATH_BATCHED
    for cutoff in CUTOFFS:
        got = _verify(gpu, ref, w, cutoff, gpu.WINDOW_ALIGNED, p)
        expect = orc.apply_cutoff(full, w["qinfo"], w["cands"], cutoff)
        bad = np.nonzero(got != expect)[0]
        assert bad.size == 0, (cutoff, len(bad), got[bad[:5]], expect[bad[:5]])


def test_exact_window_cutoff(gpu, orc, data):
    ref_words, ref_size, ref, ws = data
    w = ws[2]
    full = orc.verify(w["peq"], w["qinfo"], w["cands"], ref_words, ref_size, DIST, exact=True)
    for cutoff in (0.05, 0.2):
        got = _verify(gpu, ref, w, cutoff, gpu.WINDOW_EXACT, gpu.PATH_PLAIN, 1000, 1000)
        assert np.array_equal(got, orc.apply_cutoff(full, w["qinfo"], w["cands"], cutoff))


def test_minimum_at_the_bound(gpu, orc, data):
    """Bounds placed at the true minima of candidates of one length (1,000
    bases, one candidate per lane of 32 words): a minimum equal to the bound is
    reported exactly, one above it is not."""
    ref_words, ref_size, ref, ws = data
    w = ws[2]  # 1000-base reads
    full = orc.verify(w["peq"], w["qinfo"], w["cands"], ref_words, ref_size, DIST)
    scores = full["score"][full["score"] != orc.NO_RESULT]
    picks = np.unique(np.percentile(scores, [1, 5, 10, 50]).astype(np.int64))
    for s in picks:
        cutoff = float(np.float32(s) / np.float32(1000))
        bound = int(orc.cutoff_bound(np.array([1000]), cutoff)[0])
        expect = orc.apply_cutoff(full, w["qinfo"], w["cands"], cutoff)
        got = _verify(gpu, ref, w, cutoff, gpu.WINDOW_ALIGNED, gpu.PATH_PLAIN, 1000, 1000)
        assert np.array_equal(got, expect), (s, bound)
        assert (full["score"] == bound).any() or bound != s


def test_golden_fixtures_under_cutoff(gpu, orc, golden_verify):
    """The reference's own outputs (every pos % 8, lengths 1..4096, windows at
    the reference's end, out-of-range positions) with the contract applied."""
    g = golden_verify
    ref = gpu.Reference(g["ref"], g["ref_size"])
    try:
        for cutoff in (0.0, 0.1, 0.3):
            expect = orc.apply_cutoff(g["res_aligned"], g["qinfo"], g["cands"], cutoff)
            for path in (gpu.PATH_PLAIN, gpu.PATH_BATCHED):
                ctx = gpu.Context(len(g["cands"]))
                try:
                    got = gpu.verify_torch(ctx, ref, g["peq"], g["qinfo"], g["cands"], g["distance"], path=path,
                                           cutoff=cutoff)
                finally:
                    ctx.close()
                bad = np.nonzero(got != expect)[0]
                assert bad.size == 0, (cutoff, path, len(bad), got[bad[:5]], expect[bad[:5]])
    finally:
        ref.close()


def test_dropin_buffer_cutoff(gpu, orc, data, tmp_path):
    ref_words, ref_size, ref, ws = data
    w = ws[3]
    fn = str(tmp_path / "r.4bits.ref")
    with open(fn, "wb") as f:
        f.write(np.array([len(ref_words), ref_size], dtype=np.uint32).tobytes())
        ref_words.tofile(f)
    full = orc.verify(w["peq"], w["qinfo"], w["cands"], ref_words, ref_size, DIST)
    with gpu.Buffers(fn, num_buffers=1, avg_query_size=400, cands_per_query=11) as bufs:
        bufs.set_cutoff(0.1)
        res, st = gpu.verify_buffers(bufs, w["peq"], w["qinfo"], w["cands"], DIST)
        assert st == gpu.SUCCESS
        assert np.array_equal(res, orc.apply_cutoff(full, w["qinfo"], w["cands"], 0.1))
        bufs.set_cutoff(None)
        res, st = gpu.verify_buffers(bufs, w["peq"], w["qinfo"], w["cands"], DIST)
        assert st == gpu.SUCCESS and np.array_equal(res, full)


@pytest.mark.parametrize("mult", ["0.25", "1", "100"])
def test_prefix_multiplier_extremes(mult):
    """The first pass's prefix length comes from MYERS_CUTOFF_PREFIX (read once
    per process). A tiny multiplier sends almost every candidate to the second
    pass; a huge one makes the first pass run every query in full. Both must
    give the contract's results (a child process per setting)."""
    import os
    import subprocess
    import sys
    code = r'''
import sys, numpy as np
sys.path.insert(0, "myers-gpu_b200"); sys.path.insert(0, "oracle")
import myersgpu as mg, oracle as orc
ref_size = 3_000_000
rw = mg.make_reference(ref_size, 99)
ref = mg.Reference(rw, ref_size)
for k, sc in ((2, 0.002), (3, 0.001), (4, 0.001)):
    w = mg.make_workload(mg.workload_spec(k, scale=sc, ref_size=ref_size), rw)
    full = orc.verify(w["peq"], w["qinfo"], w["cands"], rw, ref_size, 0.2)
    for cutoff in (0.03, 0.1, 0.25):
        exp = orc.apply_cutoff(full, w["qinfo"], w["cands"], cutoff)
        for path in (mg.PATH_PLAIN, mg.PATH_BATCHED):
            ctx = mg.Context(len(w["cands"]))
            got = mg.verify_torch(ctx, ref, w["peq"], w["qinfo"], w["cands"], 0.2, cutoff=cutoff, path=path)
            ctx.close()
            assert np.array_equal(got, exp), (k, cutoff, path, int((got != exp).sum()))
ref.close()
print("ok")
'''
    from conftest import ROOT
    env = dict(os.environ, MYERS_CUTOFF_PREFIX=mult)
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0 and "ok" in out.stdout, out.stderr[-2000:]
