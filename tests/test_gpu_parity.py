"""GPU parity: the CUDA path, called through the C ABI, against the oracle
(the reference's own CPU Myers via golden vectors, and the restated oracle on
seeded workloads). Integer outputs: bit-exact."""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIST = 0.2


@pytest.fixture(scope="module")
def gpu(mg, cuda_ok):
    import torch
    torch.cuda.init()
    return mg


def _run(mg, ref_words, ref_size, peq, qinfo, cands, window, path, distance=DIST, min_size=0, max_size=0):
    ref = mg.Reference(ref_words, ref_size)
    ctx = mg.Context(max(1, len(cands)))
    try:
        res = mg.verify_torch(ctx, ref, peq, qinfo, cands, distance, window=window, path=path, min_size=min_size,
                              max_size=max_size)
        return res, ctx.launches(), ctx.flags()
    finally:
        ctx.close()
        ref.close()


@pytest.mark.parametrize("path", ["plain", "batched"])
def test_golden_aligned(gpu, golden_verify, path):
    g = golden_verify
    p = gpu.PATH_PLAIN if path == "plain" else gpu.PATH_BATCHED
    res, launches, flags = _run(gpu, g["ref"], g["ref_size"], g["peq"], g["qinfo"], g["cands"], gpu.WINDOW_ALIGNED, p,
                                distance=g["distance"])
    bad = np.nonzero(res != g["res_aligned"])[0]
    assert bad.size == 0, (bad[:10], res[bad[:10]], g["res_aligned"][bad[:10]])
    assert launches >= 1 and flags == 0


@pytest.mark.parametrize("path", ["plain", "batched"])
def test_golden_exact(gpu, golden_verify, path):
    g = golden_verify
    p = gpu.PATH_PLAIN if path == "plain" else gpu.PATH_BATCHED
    m = g["exact_mask"]
    res, _, _ = _run(gpu, g["ref"], g["ref_size"], g["peq"], g["qinfo"], g["cands"], gpu.WINDOW_EXACT, p,
                     distance=g["distance"])
    assert np.array_equal(res[m], g["res_exact"][m])


WORKLOADS = [(1, 0.05), (2, 0.004), (3, 0.002), (4, 0.003), (5, 0.004)]


@pytest.fixture(scope="module")
def workloads(gpu):
    ref_size = 8_000_000
    ref = gpu.make_reference(ref_size, 1234)
    out = {}
    for k, scale in WORKLOADS:
        out[k] = gpu.make_workload(gpu.workload_spec(k, scale=scale, ref_size=ref_size), ref)
    return ref, ref_size, out


@pytest.mark.parametrize("k", [k for k, _ in WORKLOADS])
@pytest.mark.parametrize("window", ["aligned", "exact"])
@pytest.mark.parametrize("path", ["plain", "batched"])
def test_workloads_vs_oracle(gpu, orc, workloads, k, window, path):
    ref, ref_size, ws = workloads
    w = ws[k]
    exact = window == "exact"
    expect = orc.verify(w["peq"], w["qinfo"], w["cands"], ref, ref_size, DIST, exact=exact)
    p = gpu.PATH_PLAIN if path == "plain" else gpu.PATH_BATCHED
    res, launches, flags = _run(gpu, ref, ref_size, w["peq"], w["qinfo"], w["cands"],
                                gpu.WINDOW_EXACT if exact else gpu.WINDOW_ALIGNED, p)
    bad = np.nonzero(res != expect)[0]
    assert bad.size == 0, (len(bad), bad[:5], res[bad[:5]], expect[bad[:5]])
    assert flags == 0


def test_uniform_length_single_launch(gpu, orc, workloads):
    ref, ref_size, ws = workloads
    w = ws[1]
    res, launches, _ = _run(gpu, ref, ref_size, w["peq"], w["qinfo"], w["cands"], gpu.WINDOW_ALIGNED,
                            gpu.PATH_PLAIN, min_size=100, max_size=100)
    assert launches == 1
    assert np.array_equal(res, orc.verify(w["peq"], w["qinfo"], w["cands"], ref, ref_size, DIST))


def _forced_shape(gpu, orc, workloads, W, L, path):
    ref, ref_size, ws = workloads
    w = ws[3]
    v = [x for x, ww, multi in gpu.variants() if multi and ww == W][0]
    words = sorted(set(((w["lengths"] + 31) // 32).tolist()))
    try:
        for wd in words:
            if W * L >= wd:
                gpu.set_shape_override(path, wd, v, L)
        res, _, _ = _run(gpu, ref, ref_size, w["peq"], w["qinfo"], w["cands"], gpu.WINDOW_ALIGNED, path)
    finally:
        for wd in words:
            gpu.set_shape_override(path, wd, -1)
    assert np.array_equal(res, orc.verify(w["peq"], w["qinfo"], w["cands"], ref, ref_size, DIST))


@pytest.mark.parametrize("variant_L", [(4, 2), (4, 9), (5, 7), (6, 6), (7, 5), (8, 4), (9, 4), (10, 3), (11, 3),
                                       (12, 3), (13, 3), (14, 2), (15, 3), (16, 2), (32, 2)])
def test_every_multi_shape(gpu, orc, workloads, variant_L):
    """Force each multi-lane variant (including L not dividing 32) on reads
    of up to 1000 bases in the plain kernel and compare with the oracle."""
    _forced_shape(gpu, orc, workloads, *variant_L, gpu.PATH_PLAIN)


@pytest.mark.parametrize("variant_L", [(4, 8), (5, 7), (6, 6), (7, 5), (8, 4), (9, 4), (10, 4), (11, 3), (12, 3),
                                       (13, 3), (14, 3), (15, 2), (16, 2)])
def test_every_multi_shape_persistent(gpu, orc, workloads, variant_L):
    """The same in the persistent kernel (the serving loop's latency shapes
    run there): every multi-lane width it carries."""
    _forced_shape(gpu, orc, workloads, *variant_L, gpu.PATH_BATCHED)


def test_all_lengths_1_to_300(gpu, orc):
    """Every query length 1..300 (every single-lane W up to 10 and every
    top-alignment shift), both windows."""
    rng = np.random.default_rng(7)
    ref_size = 200_000
    ref = gpu.make_reference(ref_size, 77)
    peq, qinfo, cands = [], [], []
    entry = 0
    for q, m in enumerate(range(1, 301)):
        read = bytes(rng.choice(list(b"ACGTN"), size=m, p=[0.245, 0.245, 0.245, 0.245, 0.02]).astype(np.uint8))
        peq.append(orc.pack_peq(read).reshape(-1, 20))
        qinfo.append((entry, m))
        entry += (m + 127) // 128
        for _ in range(4):
            cands.append((q, int(rng.integers(0, ref_size - 500))))
    peq = np.concatenate(peq).ravel().view(gpu.QRY_ENTRY)
    qinfo = np.array(qinfo, dtype=np.uint32).view(gpu.QINFO).ravel()
    c = np.zeros(len(cands), dtype=gpu.CAND)
    c["query"] = [x[0] for x in cands]
    c["position"] = [x[1] for x in cands]
    for exact in (False, True):
        expect = orc.verify(peq, qinfo, c, ref, ref_size, DIST, exact=exact)
        for path in (gpu.PATH_PLAIN, gpu.PATH_BATCHED):
            res, _, _ = _run(gpu, ref, ref_size, peq, qinfo, c, gpu.WINDOW_EXACT if exact else gpu.WINDOW_ALIGNED,
                             path)
            assert np.array_equal(res, expect)


def test_long_queries_up_to_max(gpu, orc):
    """Queries at the multi-lane limits (16384 batched, 32768 plain)."""
    rng = np.random.default_rng(3)
    ref_size = 400_000
    ref = gpu.make_reference(ref_size, 5)
    peq, qinfo, cands = [], [], []
    entry = 0
    for q, m in enumerate([4097, 10000, 16384, 20000, 32768]):
        start = int(rng.integers(0, ref_size - 2 * m))
        codes = [(int(ref[(start + k) // 8]) >> (4 * ((start + k) % 8))) & 0xF for k in range(m)]
        read = bytes(b"ACGTN"[c] if rng.random() > 0.05 else b"ACGT"[rng.integers(0, 4)] for c in codes)
        peq.append(orc.pack_peq(read).reshape(-1, 20))
        qinfo.append((entry, m))
        entry += (m + 127) // 128
        cands.append((q, max(0, start - m // 5)))
        cands.append((q, int(rng.integers(0, ref_size - 2 * m))))
    peq = np.concatenate(peq).ravel().view(gpu.QRY_ENTRY)
    qinfo = np.array(qinfo, dtype=np.uint32).view(gpu.QINFO).ravel()
    c = np.zeros(len(cands), dtype=gpu.CAND)
    c["query"] = [x[0] for x in cands]
    c["position"] = [x[1] for x in cands]
    expect = orc.verify(peq, qinfo, c, ref, ref_size, DIST)
    for path in (gpu.PATH_PLAIN, gpu.PATH_BATCHED):
        res, _, flags = _run(gpu, ref, ref_size, peq, qinfo, c, gpu.WINDOW_ALIGNED, path)
        assert np.array_equal(res, expect)
        assert flags == 0


def test_invalid_indices_are_flagged(gpu, orc):
    """Bad query indices and PEQ entries give {0, MAX} and a flag, never a
    wild read; the valid candidates around them are unaffected."""
    ref_size = 100_000
    ref = gpu.make_reference(ref_size, 8)
    w = gpu.make_workload(gpu.workload_spec(1, scale=0.001, ref_size=ref_size), ref)
    cands = w["cands"].copy()
    qinfo = w["qinfo"].copy()
    cands[3]["query"] = len(qinfo) + 10           # query out of range
    qinfo[5]["posEntry"] = len(w["peq"]) + 100     # PEQ entries out of range
    expect = orc.verify(w["peq"], w["qinfo"], w["cands"], ref, ref_size, DIST)
    for path in (gpu.PATH_PLAIN, gpu.PATH_BATCHED):
        res, _, flags = _run(gpu, ref, ref_size, w["peq"], qinfo, cands, gpu.WINDOW_ALIGNED, path)
        assert res[3]["score"] == gpu.NO_RESULT
        bad5 = cands["query"] == 5
        assert (res[bad5]["score"] == gpu.NO_RESULT).all()
        ok = (cands["query"] != 5) & (np.arange(len(cands)) != 3)
        assert np.array_equal(res[ok], expect[ok])
        assert flags & 2 and flags & 4


def test_empty_and_zero_length(gpu, orc):
    ref_size = 10_000
    ref = gpu.make_reference(ref_size, 2)
    peq = np.zeros(1, dtype=gpu.QRY_ENTRY)
    qinfo = np.array([(0, 0)], dtype=np.uint32).view(gpu.QINFO).ravel()
    c = np.zeros(3, dtype=gpu.CAND)
    c["position"] = [0, 5000, ref_size + 1]
    for path in (gpu.PATH_PLAIN, gpu.PATH_BATCHED):
        res, _, _ = _run(gpu, ref, ref_size, peq, qinfo, c, gpu.WINDOW_ALIGNED, path)
        assert res.tolist() == orc.verify(peq, qinfo, c, ref, ref_size, DIST).tolist()
        assert res.tolist() == [(0, 0), (0, 0), (0, gpu.NO_RESULT)]
        res0, launches, _ = _run(gpu, ref, ref_size, peq, qinfo, c[:0], gpu.WINDOW_ALIGNED, path)
        assert len(res0) == 0 and launches == 0


def _write_ref_file(path, words, size):
    with open(path, "wb") as f:
        f.write(np.array([len(words), size], dtype=np.uint32).tobytes())
        f.write(np.asarray(words, dtype=np.uint32).tobytes())


@pytest.mark.parametrize("path", ["plain", "batched"])
def test_dropin_buffers(gpu, orc, workloads, path):
    """The reference's call sequence: initMyers, fill the pinned buffers
    through the getters, send, receive, read results, endMyers."""
    ref, ref_size, ws = workloads
    with tempfile.TemporaryDirectory() as tmp:
        fn = os.path.join(tmp, "g.4bits.ref")
        _write_ref_file(fn, ref, ref_size)
        gpu.lib.myersSetMemoryBudget(256 << 20)
        bufs = gpu.Buffers(fn, num_buffers=2, avg_query_size=400, cands_per_query=10)
        try:
            bufs.set_path(gpu.PATH_PLAIN if path == "plain" else gpu.PATH_BATCHED)
            for i, k in enumerate((3, 5)):
                w = ws[k]
                res, st = gpu.verify_buffers(bufs, w["peq"], w["qinfo"], w["cands"], DIST, buffer=i)
                assert st == gpu.SUCCESS
                assert np.array_equal(res, orc.verify(w["peq"], w["qinfo"], w["cands"], ref, ref_size, DIST))
            # capacity errors are returned, not fatal
            ne, nq, nc = bufs.capacity(0)
            st = gpu.lib.myersSend(bufs.handles[0], DIST, ne + 1, 1, 1)
            assert st == gpu.E_CAPACITY
        finally:
            bufs.close()
            gpu.lib.myersSetMemoryBudget(0)


def test_dropin_graph_replay(gpu, orc, workloads):
    """Sends replayed as CUDA graphs: consecutive sends of other sizes (graph
    updated in place), other length mixes and kernel paths (new topology),
    window modes and an empty send all give the results of plain stream
    launches and the oracle's."""
    ref, ref_size, ws = workloads
    with tempfile.TemporaryDirectory() as tmp:
        fn = os.path.join(tmp, "g.4bits.ref")
        _write_ref_file(fn, ref, ref_size)
        gpu.lib.myersSetMemoryBudget(256 << 20)
        bufs = gpu.Buffers(fn, num_buffers=2, avg_query_size=400, cands_per_query=10)
        try:
            bufs.set_graphs(True, 0)
            bufs.set_graphs(False, 1)
            w3, w5 = ws[3], ws[5]
            sends = []
            for k, nq in ((3, 40), (3, 7), (5, 60), (3, 40)):
                w = ws[k]
                qi = w["qinfo"][:nq]
                last = qi[-1]
                ne = int(last["posEntry"]) + (int(last["size"]) + 127) // 128
                sends.append((w["peq"][:ne], qi, w["cands"][w["cands"]["query"] < nq]))
            empty = (w3["peq"][:1], w3["qinfo"][:1], w3["cands"][:0])
            plan = [(gpu.PATH_BATCHED, gpu.WINDOW_ALIGNED, s) for s in sends] + \
                   [(gpu.PATH_PLAIN, gpu.WINDOW_ALIGNED, s) for s in sends] + \
                   [(gpu.PATH_BATCHED, gpu.WINDOW_EXACT, sends[2]), (gpu.PATH_BATCHED, gpu.WINDOW_ALIGNED, empty),
                    (gpu.PATH_PLAIN, gpu.WINDOW_ALIGNED, sends[0])]
            for path, window, (peq, qinfo, cands) in plan:
                expect = orc.verify(peq, qinfo, cands, ref, ref_size, DIST, exact=window == gpu.WINDOW_EXACT)
                for i in (0, 1):
                    bufs.set_path(path, i)
                    bufs.set_window_mode(window, i)
                    res, st = gpu.verify_buffers(bufs, peq, qinfo, cands, DIST, buffer=i)
                    assert st == gpu.SUCCESS
                    assert np.array_equal(res, expect), (path, window, len(cands), i)
        finally:
            bufs.close()
            gpu.lib.myersSetMemoryBudget(0)


def test_concurrent_contexts_on_two_streams(gpu, orc, workloads):
    """Two contexts verifying different batches at the same time on two
    streams (a plain launch whose warps take tiles from the context's counter,
    and the persistent kernel on the other): each batch's results equal the
    oracle's. Contexts share no device state."""
    import torch
    ref_words, ref_size, ws = workloads
    ref = gpu.Reference(ref_words, ref_size)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1)).cuda()

    jobs = []
    for k, path in ((2, gpu.PATH_PLAIN), (3, gpu.PATH_BATCHED)):
        w = ws[k]
        n = len(w["cands"])
        jobs.append(dict(w=w, path=path, ctx=gpu.Context(n), stream=torch.cuda.Stream(),
                         d=(dev(w["peq"]), dev(w["qinfo"]), dev(w["cands"])),
                         res=torch.empty(n * 8, dtype=torch.uint8, device="cuda")))
    try:
        for _ in range(2):  # twice: the counters start again at every launch
            for j in jobs:
                w, (d_peq, d_qi, d_c) = j["w"], j["d"]
                j["ctx"].verify(ref, d_peq.data_ptr(), len(w["peq"]), d_qi.data_ptr(), len(w["qinfo"]),
                                d_c.data_ptr(), len(w["cands"]), DIST, j["res"].data_ptr(), path=j["path"],
                                stream=j["stream"].cuda_stream)
            torch.cuda.synchronize()
            for j in jobs:
                w = j["w"]
                got = j["res"].cpu().numpy().view(gpu.RES)
                assert np.array_equal(got, orc.verify(w["peq"], w["qinfo"], w["cands"], ref_words, ref_size, DIST))
    finally:
        for j in jobs:
            j["ctx"].close()
        ref.close()


@pytest.mark.parametrize("path", ["plain", "batched"])
def test_one_candidate_per_read(gpu, orc, workloads, path):
    """With fewer than two candidates per read, reads of 513..1,024 bases run
    on lanes of at most 16 words (a warp's 32 candidates then come from 32
    reads, more than the 16 PEQ slots of one-lane shapes of more than 16
    words): every 11th candidate of 1,000-base and mixed reads."""
    ref, ref_size, ws = workloads
    p = gpu.PATH_PLAIN if path == "plain" else gpu.PATH_BATCHED
    for k in (2, 3):
        w = ws[k]
        sel = np.ascontiguousarray(w["cands"][::11])
        assert len(sel) < 2 * len(w["qinfo"])
        res, _, _ = _run(gpu, ref, ref_size, w["peq"], w["qinfo"], sel, gpu.WINDOW_ALIGNED, p)
        assert np.array_equal(res, orc.verify(w["peq"], w["qinfo"], sel, ref, ref_size, DIST)), k


@pytest.mark.parametrize("env", [{"MYERS_LARGE_BATCH": "1", "MYERS_SMALL_BATCH": "0"},
                                 {"MYERS_SMALL_BATCH": "0"}], ids=["large", "tuned"])
def test_batch_size_shapes(env):
    """The batched path picks its shapes by batch size. Below 280K candidates
    reads of up to 1,024 bases take lanes of at most 12 words (what the other
    tests' small batches run). Longer reads, and every read from 280K, take the
    large-batch table (every lane width) from 150K candidates and the tuned
    table below that. The thresholds (MYERS_SMALL_BATCH,
    MYERS_LARGE_BATCH, read once per process, so in a child) are moved here so
    small batches of long and mixed reads run the large-batch and the tuned
    tables, compared with the oracle on both paths."""
    import subprocess
    import sys
    from conftest import ROOT
    code = r'''
import sys, numpy as np
sys.path.insert(0, "myers-gpu_b200"); sys.path.insert(0, "oracle")
import myersgpu as mg, oracle as orc
ref_size = 4_000_000
rw = mg.make_reference(ref_size, 31)
ref = mg.Reference(rw, ref_size)
for k, sc in ((4, 0.003), (3, 0.001)):
    w = mg.make_workload(mg.workload_spec(k, scale=sc, ref_size=ref_size), rw)
    expect = orc.verify(w["peq"], w["qinfo"], w["cands"], rw, ref_size, 0.2)
    for path in (mg.PATH_BATCHED, mg.PATH_PLAIN):
        ctx = mg.Context(len(w["cands"]))
        got = mg.verify_torch(ctx, ref, w["peq"], w["qinfo"], w["cands"], 0.2, path=path)
        ctx.close()
        assert np.array_equal(got, expect), (k, path, int((got != expect).sum()))
ref.close()
print("ok")
'''
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=dict(os.environ, **env),
                         capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0 and "ok" in out.stdout, out.stderr[-2000:]
