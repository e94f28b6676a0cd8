"""GPU tests of the serving loop: each request's result is the same alone and
in the mix (continuous batching, concurrent submitters), equal to the oracle;
admission refuses what does not fit instead of failing."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIST = 0.2


@pytest.fixture(scope="module")
def serving(mg, cuda_ok):
    import torch
    torch.cuda.init()
    ref_size = 6_000_000
    ref_words = mg.make_reference(ref_size, 55)
    w = mg.make_workload(mg.workload_spec(5, scale=0.004, ref_size=ref_size), ref_words)  # 400 requests
    off = np.concatenate([[0], np.cumsum(w["ncands"])]).astype(np.uint32)
    ref = mg.Reference(ref_words, ref_size)
    yield dict(ref_words=ref_words, ref_size=ref_size, w=w, off=off, ref=ref)
    ref.close()


def _request(w, off, i):
    q = w["qinfo"][i]
    e = (int(q["size"]) + 127) // 128
    return w["peq"][q["posEntry"]:q["posEntry"] + e], int(q["size"]), w["cands"]["position"][off[i]:off[i + 1]]


def test_alone_equals_mix_equals_oracle(mg, orc, serving):
    w, off = serving["w"], serving["off"]
    expect = orc.verify(w["peq"], w["qinfo"], w["cands"], serving["ref_words"], serving["ref_size"], DIST)
    n = len(w["qinfo"])
    with mg.Server(serving["ref"], distance=DIST, slots=3, max_batch_candidates=4096) as srv:
        # alone: one request at a time, each waited for before the next
        alone = []
        for i in range(n):
            peq, m, pos = _request(w, off, i)
            st, t = srv.submit(peq, m, pos)
            assert st == mg.SUCCESS
            st, r = srv.wait(t, len(pos))
            assert st == mg.SUCCESS
            alone.append(r)
        alone = np.concatenate(alone)
        assert srv.stats()["batches"] == n
        # in the mix: open-loop arrivals much faster than the GPU drains them
        arrivals = np.cumsum(np.random.default_rng(1).exponential(2000.0, size=n)).astype(np.uint64)
        st, lat, mix, wall = srv.replay(w["peq"], w["qinfo"], off, w["cands"]["position"], arrivals)
        assert st == mg.SUCCESS and (lat < np.iinfo(np.uint64).max).all()
        s = srv.stats()
        assert s["batches"] < 2 * n          # requests shared batches
        assert s["batchCandidatesMax"] > 64  # more than one request's worth in a batch
    assert np.array_equal(alone, expect)
    assert np.array_equal(mix, expect)


def test_concurrent_submitters(mg, orc, serving):
    w, off = serving["w"], serving["off"]
    expect = orc.verify(w["peq"], w["qinfo"], w["cands"], serving["ref_words"], serving["ref_size"], DIST)
    n = len(w["qinfo"])
    out = [None] * n
    errors = []
    with mg.Server(serving["ref"], distance=DIST, slots=4, max_batch_candidates=2048) as srv:
        def worker(k):
            try:
                for i in range(k, n, 4):
                    peq, m, pos = _request(w, off, i)
                    st, t = srv.submit(peq, m, pos)
                    assert st == mg.SUCCESS
                    st, r = srv.wait(t, len(pos))
                    assert st == mg.SUCCESS
                    out[i] = r
            except AssertionError as e:  # pragma: no cover - reported below
                errors.append(e)
        threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    assert not errors
    assert np.array_equal(np.concatenate(out), expect)


def test_admission(mg, serving):
    w, off = serving["w"], serving["off"]
    with mg.Server(serving["ref"], distance=DIST, slots=1, max_batch_candidates=128, max_queued=4,
                   max_query_size=1000) as srv:
        peq, m, pos = _request(w, off, 0)
        # a request longer than the configured reads, or with more candidates than a slot
        st, _ = srv.submit(np.zeros(9, dtype=mg.QRY_ENTRY), 1100, pos[:1])
        assert st == mg.E_QUERY_TOO_LONG
        st, _ = srv.submit(peq, m, np.zeros(129, dtype=np.uint64))
        assert st == mg.E_CAPACITY
        # flooding a 4-deep queue: some submissions are refused, the rest complete
        tickets, refused = [], 0
        for i in range(200):
            peq, m, pos = _request(w, off, i % len(w["qinfo"]))
            st, t = srv.submit(peq, m, pos)
            if st == mg.E_BUSY:
                refused += 1
            else:
                assert st == mg.SUCCESS
                tickets.append((t, len(pos)))
        for t, k in tickets:
            st, _ = srv.wait(t, k)
            assert st == mg.SUCCESS
        s = srv.stats()
        assert refused > 0 and s["refused"] == refused
        assert s["completed"] == len(tickets)
        st, _ = srv.poll(tickets[0][0], 1)  # already taken
        assert st == mg.E_INVALID_ARGUMENT
