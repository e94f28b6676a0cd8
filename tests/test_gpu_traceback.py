"""GPU traceback against the oracle's: the same start column, op count and
run-length ops for every candidate, on the workload shapes (short, mixed,
long reads), both window modes, tight and loose score bounds, tiny scratch
(many passes), too little room for the ops, and inconsistent results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIST = 0.2


@pytest.fixture(scope="module")
def tbdata(mg, cuda_ok):
    import torch
    torch.cuda.init()
    ref_size = 6_000_000
    ref_words = mg.make_reference(ref_size, 99)
    ref = mg.Reference(ref_words, ref_size)
    ws = {k: mg.make_workload(mg.workload_spec(k, scale=sc, ref_size=ref_size), ref_words)
          for k, sc in ((1, 0.01), (3, 0.0004), (5, 0.002))}
    yield dict(ref=ref, ref_words=ref_words, ref_size=ref_size, ws=ws)
    ref.close()


def _check(mg, orc, d, w, max_score, max_ops, exact=False, results=None, scratch=1 << 30, nthreads=0):
    window = mg.WINDOW_EXACT if exact else mg.WINDOW_ALIGNED
    if results is None:
        results = orc.verify(w["peq"], w["qinfo"], w["cands"], d["ref_words"], d["ref_size"], DIST, exact=exact)
    e_aln, e_ops = orc.traceback(w["peq"], w["qinfo"], w["cands"], results, d["ref_words"], d["ref_size"], DIST,
                                 max_score, max_ops, exact=exact, nthreads=nthreads)
    with mg.Traceback(len(w["cands"]), scratch) as tb:
        g_aln, g_ops = mg.traceback_torch(tb, d["ref"], w["peq"], w["qinfo"], w["cands"], results, DIST, max_score,
                                          max_ops, window=window)
        chunks = tb.chunks()
    assert np.array_equal(g_aln.view(np.uint32).reshape(-1, 4), e_aln.view(np.uint32).reshape(-1, 4))
    fit = e_aln["num_ops"] <= max_ops
    for k in np.nonzero(fit)[0]:
        n = int(e_aln["num_ops"][k])
        assert np.array_equal(g_ops[k, :n], e_ops[k, :n]), k
    return e_aln, chunks


@pytest.mark.parametrize("k", [1, 3, 5])
@pytest.mark.parametrize("exact", [False, True])
def test_traceback_matches_oracle(mg, orc, tbdata, k, exact):
    w = tbdata["ws"][k]
    m = w["qinfo"]["size"][w["cands"]["query"]]
    # every candidate (decoys included: wide bands), then a mapper's bound
    aln, _ = _check(mg, orc, tbdata, w, 10 ** 6, 1024, exact=exact)
    assert (aln["num_ops"] < orc.TB_INCONSISTENT).all()
    aln, _ = _check(mg, orc, tbdata, w, int(0.08 * m.max()), 512, exact=exact)
    traced = aln["num_ops"] < orc.TB_INCONSISTENT
    assert 0 < traced.sum() < len(aln)


def test_traceback_long_reads(mg, orc, tbdata):
    """Reads of 1,000-10,000 bases: several lanes of up to 16 words."""
    w = mg.make_workload(mg.workload_spec(4, scale=0.0003, ref_size=tbdata["ref_size"]), tbdata["ref_words"])
    res = orc.verify(w["peq"], w["qinfo"], w["cands"], tbdata["ref_words"], tbdata["ref_size"], DIST)
    m = w["qinfo"]["size"][w["cands"]["query"]]
    aln, _ = _check(mg, orc, tbdata, w, int(0.15 * m.max()), 4096, results=res, nthreads=4)
    assert (aln["num_ops"] < orc.TB_INCONSISTENT).sum() > 0


def test_traceback_small_scratch_and_ops(mg, orc, tbdata):
    w = tbdata["ws"][5]
    aln, chunks = _check(mg, orc, tbdata, w, 10 ** 6, 1024, scratch=4 << 20)
    assert chunks > 1
    # room for 3 runs only: the count is reported, the record otherwise the same
    aln, _ = _check(mg, orc, tbdata, w, 10 ** 6, 3)
    assert (aln["num_ops"][aln["num_ops"] < orc.TB_INCONSISTENT] > 3).any()


def test_traceback_inconsistent_and_edges(mg, orc, tbdata):
    w = tbdata["ws"][1]
    res = orc.verify(w["peq"], w["qinfo"], w["cands"], tbdata["ref_words"], tbdata["ref_size"], DIST)
    bad = res.copy()
    bad["score"][::3] += 1                    # not what the inputs give at that column
    bad["column"][1::7] = 10_000              # past the window
    bad["score"][2::11] = 0xFFFFFFFF          # no result: not traced
    aln, _ = _check(mg, orc, tbdata, w, 10 ** 6, 256, results=bad)
    assert (aln["num_ops"] == orc.TB_INCONSISTENT).sum() > len(aln) // 4
    assert (aln["num_ops"][2::11] == orc.TB_NOT_TRACED).all()
    # an empty query and a window off the end of the reference
    peq = w["peq"][:1].copy()
    qinfo = np.array([(0, 0), (0, 100)], dtype=np.uint32).view(mg.QINFO).ravel()
    c = np.zeros(3, dtype=mg.CAND)
    c["query"] = [0, 1, 1]
    c["position"] = [50, 1000, tbdata["ref_size"] - 10]
    ww = dict(peq=peq, qinfo=qinfo, cands=c)
    aln, _ = _check(mg, orc, tbdata, ww, 10 ** 6, 256)
    assert aln["num_ops"][0] == 0 and aln["start_column"][0] == 1
    assert aln["num_ops"][2] == orc.TB_NOT_TRACED
