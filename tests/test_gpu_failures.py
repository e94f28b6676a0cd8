"""Host-side refusals that need a device to reach: a memory budget too small
for one buffer or one serving slot, and batches larger than the buffer or
context holds. Each is reported as a status before anything is enqueued; none
makes the GPU fault. The reference exits the process on every error
(src-api/myersGPU.c:24-47) and sizes buffers from 95% of free memory
(myersGPU.c:323-333); here the budget is the caller's and the status comes
back."""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIST = 0.2


@pytest.fixture(scope="module")
def small(mg, cuda_ok, tmp_path_factory):
    import torch
    torch.cuda.init()
    ref_size = 2_000_000
    ref_words = mg.make_reference(ref_size, 77)
    path = str(tmp_path_factory.mktemp("ref") / "small.4bits.ref")
    with open(path, "wb") as f:
        f.write(np.array([len(ref_words), ref_size], dtype=np.uint32).tobytes())
        ref_words.tofile(f)
    w = mg.make_workload(mg.workload_spec(1, scale=0.01, ref_size=ref_size), ref_words)  # 1,000 reads x 100 b
    return dict(path=path, ref_words=ref_words, ref_size=ref_size, w=w)


def test_budget_smaller_than_one_buffer(mg, small):
    arr = C.POINTER(C.c_void_p)()
    mg.lib.myersSetMemoryBudget(1)
    try:
        st = mg.lib.myersInit(C.byref(arr), 2, small["path"].encode(), 100, 11)
    finally:
        mg.lib.myersSetMemoryBudget(0)
    assert st == mg.E_INSUFFICIENT_MEM_GPU, mg.error_string(st)
    assert not arr


def test_send_beyond_capacity_is_refused(mg, orc, small):
    w = small["w"]
    # a budget for about 4,000 candidates of 100 bases per buffer
    mg.lib.myersSetMemoryBudget(400_000)
    try:
        bufs = mg.Buffers(small["path"], num_buffers=1, avg_query_size=100, cands_per_query=11)
    finally:
        mg.lib.myersSetMemoryBudget(0)
    try:
        ne, nq, nc = bufs.capacity(0)
        assert 0 < nc < len(w["cands"])
        st = mg.lib.myersSend(bufs.handles[0], DIST, ne, nq, nc + 1)
        assert st == mg.E_CAPACITY
        assert bufs.receive(0) == mg.E_CAPACITY  # the refused send is what receive reports
        # the buffer still works for a batch that fits
        nreads = min(nq, ne, nc // 11)
        sub_q = w["qinfo"][:nreads]
        sub_c = w["cands"][:11 * nreads]
        res, st = mg.verify_buffers(bufs, w["peq"][:nreads], sub_q, sub_c, DIST)
        assert st == mg.SUCCESS
        expect = orc.verify(w["peq"], w["qinfo"], sub_c, small["ref_words"], small["ref_size"], DIST)
        assert np.array_equal(res, expect)
    finally:
        bufs.close()


def test_context_capacity(mg, small):
    import torch
    w = small["w"]
    ref = mg.Reference(small["ref_words"], small["ref_size"])
    ctx = mg.Context(100)
    try:
        d = torch.empty(16, dtype=torch.uint8, device="cuda")
        p = d.data_ptr()
        st = mg.lib.myersVerifyAsync(ctx.h, ref.h, p, 1, p, 1, p, 101, C.c_float(DIST), mg.WINDOW_ALIGNED,
                                     mg.PATH_BATCHED, p, None)
        assert st == mg.E_CAPACITY
        assert ctx.launches() == 0
    finally:
        ctx.close()
        ref.close()


def test_server_budget_too_small(mg, small):
    ref = mg.Reference(small["ref_words"], small["ref_size"])
    try:
        with pytest.raises(mg.MyersError) as e:
            mg.Server(ref, distance=DIST, slots=4, budget=1024, max_query_size=1000)
        assert e.value.status == mg.E_INSUFFICIENT_MEM_GPU
    finally:
        ref.close()
