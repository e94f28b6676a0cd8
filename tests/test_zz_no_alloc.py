"""The entry point that allocates nothing (myersVerifyNoAllocAsync), for
callers that cannot call cudaMalloc -- programs whose own allocator owns all
device memory, services whose memory budget is fixed once they run. Called through the C ABI on two batches in a row, its results
must equal those of the allocating entry point (myersVerifyRangeAsync, batched
path) bit for bit: integer outputs, no tolerance. This file is collected last
so a stop-at-first-failure run has run every other test before it."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIST = 0.2


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).cuda()


def test_no_alloc_matches_allocating_entry_point(mg, orc, cuda_ok):
    import torch
    torch.cuda.init()
    ref_size = 4_000_003
    ref_words = mg.make_reference(ref_size, 2024)
    d_ref = torch.from_numpy(ref_words.view(np.int32)).cuda()       # the caller's own reference copy
    batches = [mg.make_workload(mg.workload_spec(3, scale=0.004, ref_size=ref_size), ref_words),   # 100..1000 b
               mg.make_workload(mg.workload_spec(4, scale=0.0005, ref_size=ref_size), ref_words)]  # 1..10 kb
    ref = mg.Reference(ref_words, ref_size)
    stream = torch.cuda.current_stream()
    free_before_second = None
    try:
        for call, w in enumerate(batches):
            n = len(w["cands"])
            assert 0 < n <= mg.NOALLOC_MAX_CANDIDATES
            dp, dq, dc = _dev(torch, w["peq"]), _dev(torch, w["qinfo"]), _dev(torch, w["cands"])
            d_new = torch.full((n * 8,), 0xAB, dtype=torch.uint8, device="cuda")
            lo, hi = int(w["qinfo"]["size"].min()), int(w["qinfo"]["size"].max())
            torch.cuda.synchronize()
            if call == 1:
                free_before_second = torch.cuda.mem_get_info()[0]
            st = mg.lib.myersVerifyNoAllocAsync(d_ref.data_ptr(), len(ref_words), ref_size, dp.data_ptr(),
                                                len(w["peq"]), dq.data_ptr(), len(w["qinfo"]), dc.data_ptr(), n,
                                                DIST, mg.WINDOW_ALIGNED, lo, hi, d_new.data_ptr(),
                                                stream.cuda_stream)
            assert st == mg.SUCCESS, mg.error_string(st)
            torch.cuda.synchronize()
            if call == 1:
                assert torch.cuda.mem_get_info()[0] == free_before_second
            got = d_new.cpu().numpy().view(mg.RES)
            ctx = mg.Context(n)
            try:
                expect = mg.verify_torch(ctx, ref, w["peq"], w["qinfo"], w["cands"], DIST, path=mg.PATH_BATCHED,
                                         min_size=lo, max_size=hi)
            finally:
                ctx.close()
            assert np.array_equal(got, expect)
            assert np.array_equal(got, orc.verify(w["peq"], w["qinfo"], w["cands"], ref_words, ref_size, DIST))
    finally:
        ref.close()


def test_no_alloc_rejects_oversized_batch(mg, cuda_ok):
    n = mg.NOALLOC_MAX_CANDIDATES + 1
    st = mg.lib.myersVerifyNoAllocAsync(C.c_void_p(16), 1, 8, C.c_void_p(16), 1, C.c_void_p(16), 1, C.c_void_p(16),
                                        n, DIST, mg.WINDOW_ALIGNED, 0, 0, C.c_void_p(16), None)
    assert st == mg.E_CAPACITY
