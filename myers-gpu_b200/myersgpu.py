"""Python bindings of the Myers B200 library (ctypes over the C ABI).

The product is libmyers_b200.so: CUDA kernels for sm_100a behind the C ABI
declared in include/myers-interface.h (a drop-in for the reference's
src-api/myers-interface.h). This module only binds that ABI, and re-exports the
seeded workload generator of myerssynth.py; there is no Python compute path. If
the library is missing, importing this module raises.

Record layouts (numpy dtypes) match the C structs byte for byte:
  QRY_ENTRY  qryEntry_t  80 B  bitmap[5][4] u32  (128 query bases)
  CAND       candInfo_t  16 B  u32 query, 4 B padding, u64 position
  QINFO      qryInfo_t    8 B  u32 posEntry, u32 size
  RES        resEntry_t   8 B  u32 column, u32 score
"""
import ctypes as C
import os

import numpy as np

# the record layouts and the seeded workload generator (no CUDA code)
from myerssynth import (CAND, GENOME, PAD_WORD, QINFO, QRY_ENTRY, RES, SynthSpec, cells,  # noqa: F401
                        make_reference, make_workload, spec, workload_spec)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmyers_b200.so")


SUCCESS = 0
E_OPENING_FILE, E_READING_FILE, E_INSUFFICIENT_MEM_GPU, E_ALLOCATE_MEM, E_INCOMPATIBLE_GPU = 1, 2, 3, 4, 5
E_INVALID_ARGUMENT, E_CAPACITY, E_QUERY_TOO_LONG, E_CUDA, E_TIMEOUT, E_NOT_READY, E_BUSY = 6, 7, 8, 9, 10, 11, 12
WINDOW_ALIGNED, WINDOW_EXACT = 0, 1
PATH_PLAIN, PATH_BATCHED = 0, 1
NO_RESULT = 0xFFFFFFFF
NO_MATCH = 0xFFFFFFFF  # column and score of a candidate above the cut-off bound
MAX_QUERY_BASES = 32768
NOALLOC_MAX_CANDIDATES = 262144


class MyersError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"{what}: {error_string(status)} (status {status})")


def _load(path):
    if not os.path.exists(path):
        raise ImportError(f"{os.path.basename(path)} is not built: run myers-gpu_b200/build.py")
    return C.CDLL(path)


lib = _load(LIB_PATH)

_P, _U32, _U64, _I32, _F = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_float
_PP = C.POINTER(C.c_void_p)


def _sig(fn, res, *args):
    f = getattr(lib, fn)
    f.restype = res
    f.argtypes = list(args)
    return f


_sig("myersGetErrorString", C.c_char_p, _I32)
for _g in ("getPEQBuffer", "getCandidatesBuffer", "getPEQInfoBuffer", "getResultsBuffer"):
    _sig(_g, _P, _P)
for _g in ("getMaxPEQEntries", "getMaxCandidates", "getMaxQueries"):
    _sig(_g, _U32, _P)
_sig("myersInit", _I32, C.POINTER(_PP), _U32, C.c_char_p, C.c_int32, C.c_int32)
_sig("myersSend", _I32, _P, _F, _U32, _U32, _U32)
_sig("myersReceive", _I32, _P)
_sig("myersEnd", _I32, C.POINTER(_PP))
_sig("myersSetWindowMode", _I32, _P, _I32)
_sig("myersSetKernelPath", _I32, _P, _I32)
_sig("myersSetGraphs", _I32, _P, _I32)
_sig("myersSetMemoryBudget", _I32, _U64)
_sig("myersGetDevice", _I32, _P)
_sig("myersGetLastStatus", _I32, _P)
_sig("myersBufferLastLaunches", _U32, _P)
_sig("myersReferenceCreate", _I32, _PP, _P, _U64, _U64)
_sig("myersReferenceLoad", _I32, _PP, C.c_char_p)
_sig("myersReferenceDestroy", _I32, _P)
_sig("myersReferenceSize", _U64, _P)
_sig("myersContextCreate", _I32, _PP, _U64)
_sig("myersContextDestroy", _I32, _P)
_sig("myersVerifyAsync", _I32, _P, _P, _P, _U32, _P, _U32, _P, _U32, _F, _I32, _I32, _P, _P)
_sig("myersVerifyRangeAsync", _I32, _P, _P, _P, _U32, _P, _U32, _P, _U32, _F, _I32, _I32, _U32, _U32, _P, _P)
_sig("myersVerifyCutoffAsync", _I32, _P, _P, _P, _U32, _P, _U32, _P, _U32, _F, _I32, _I32, _F, _U32, _U32, _P,
     _P)
_sig("myersSetCutoff", _I32, _P, _F)
_sig("myersVerifyNoAllocAsync", _I32, _P, _U64, _U64, _P, _U32, _P, _U32, _P, _U32, _F, _I32, _U32, _U32, _P, _P)
_sig("myersContextLastLaunches", _U32, _P)
_sig("myersPackPEQAsync", _I32, _P, _P, _U64, _P, _P, _U32, _P, _U32, _P)
_sig("myersPackReferenceAsync", _I32, _P, _U64, _P, _U64, _P)
_sig("myersServerCreate", _I32, _PP, _P, _P)
_sig("myersServerSubmit", _I32, _P, _P, _U32, _P, _U32, C.POINTER(_U64))
_sig("myersServerPoll", _I32, _P, _U64, _P)
_sig("myersServerWait", _I32, _P, _U64, _P, _U32)
_sig("myersServerStats", _I32, _P, _P)
_sig("myersServerDestroy", _I32, _P)
_sig("myersServerReplay", _I32, _P, _P, _P, _P, _P, _U32, _P, _P, _P, C.POINTER(_U64))
_sig("myersContextFlags", _I32, _P, C.POINTER(_U32), _I32)
_sig("myersNumVariants", _I32)
_sig("myersVariantWords", _I32, _I32)
_sig("myersVariantIsMulti", _I32, _I32)
_sig("myersShapeOf", _I32, _I32, _U32, C.POINTER(_I32), C.POINTER(_I32), C.POINTER(_I32))
_sig("myersSetShapeOverride", _I32, _I32, _U32, _I32, _I32)
_sig("myersTunedShapes", _I32, _I32)
_sig("myersProbeIntPeak", _I32, C.POINTER(C.c_double), _I32)
_sig("myersTracebackCreate", _I32, _PP, _U64, _U64)
_sig("myersTracebackDestroy", _I32, _P)
_sig("myersTraceback", _I32, _P, _P, _P, _U32, _P, _U32, _P, _P, _U32, _F, _I32, _U32, _P, _U32, _P, _P)
_sig("myersTracebackLastCount", _U32, _P)
_sig("myersTracebackLastChunks", _U32, _P)

# Every symbol the C header declares (the CPU tests check the exports).
EXPORTED = (
    "getPEQBuffer getCandidatesBuffer getPEQInfoBuffer getResultsBuffer getMaxPEQEntries "
    "getMaxCandidates getMaxQueries initMyers sendMyersBuffer receiveMyersBuffer endMyers "
    "myersGetErrorString myersInit myersSend myersReceive myersEnd myersSetWindowMode "
    "myersSetKernelPath myersSetGraphs myersSetMemoryBudget myersGetDevice myersGetLastStatus myersReferenceCreate "
    "myersReferenceLoad myersReferenceDestroy myersReferenceSize myersContextCreate myersContextDestroy "
    "myersVerifyAsync myersVerifyRangeAsync myersVerifyCutoffAsync myersSetCutoff myersVerifyNoAllocAsync myersContextLastLaunches myersContextFlags "
    "myersPackPEQAsync myersPackReferenceAsync "
    "myersBufferLastLaunches myersNumVariants myersVariantWords myersVariantIsMulti myersShapeOf "
    "myersSetShapeOverride myersTunedShapes myersProbeIntPeak myersServerCreate myersServerSubmit myersServerPoll myersServerWait "
    "myersServerStats myersServerDestroy myersServerReplay myersTracebackCreate myersTracebackDestroy "
    "myersTraceback myersTracebackLastCount myersTracebackLastChunks"
).split()

ALN = np.dtype([("start_column", "<u4"), ("num_ops", "<u4"), ("score", "<u4"), ("end_column", "<u4")])
TB_NOT_TRACED = 0xFFFFFFFF
TB_INCONSISTENT = 0xFFFFFFFE


def error_string(status):
    return lib.myersGetErrorString(status).decode()


def check(status, what=""):
    if status != SUCCESS:
        raise MyersError(status, what)
    return status


# ---------------------------------------------------------------------------
# shapes


def shape_of(query_size, path=PATH_PLAIN):
    v, L, W = _I32(), _I32(), _I32()
    check(lib.myersShapeOf(path, query_size, C.byref(v), C.byref(L), C.byref(W)), "myersShapeOf")
    return v.value, L.value, W.value


def set_shape_override(path, words, variant, L=1):
    check(lib.myersSetShapeOverride(path, words, variant, L), "myersSetShapeOverride")


def variants():
    """(variant, W, is_multi) of every compiled kernel variant."""
    return [(v, lib.myersVariantWords(v), bool(lib.myersVariantIsMulti(v))) for v in range(lib.myersNumVariants())]


def probe_int_peak(iters=2000):
    x = C.c_double()
    check(lib.myersProbeIntPeak(C.byref(x), iters), "myersProbeIntPeak")
    return x.value


# ---------------------------------------------------------------------------
# drop-in buffers (initMyers / sendMyersBuffer / receiveMyersBuffer / endMyers)


class Buffers:
    """The reference API's buffers: library-owned pinned host arrays filled in
    place, one stream per buffer (status-returning entry points)."""

    def __init__(self, ref_file, num_buffers=1, avg_query_size=1000, cands_per_query=10):
        self._arr = _PP()
        check(lib.myersInit(C.byref(self._arr), num_buffers, ref_file.encode(), avg_query_size, cands_per_query),
              "myersInit")
        self.handles = [self._arr[i] for i in range(num_buffers)]

    def __len__(self):
        return len(self.handles)

    def capacity(self, i=0):
        h = self.handles[i]
        return lib.getMaxPEQEntries(h), lib.getMaxQueries(h), lib.getMaxCandidates(h)

    def views(self, i=0):
        """numpy views of buffer i's pinned arrays: (peq, qinfo, cands, results)."""
        h = self.handles[i]
        ne, nq, nc = self.capacity(i)

        def view(ptr, n, dt):
            raw = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint8)), shape=(n * dt.itemsize,))
            return raw.view(dt)

        return (view(lib.getPEQBuffer(h), ne, QRY_ENTRY), view(lib.getPEQInfoBuffer(h), nq, QINFO),
                view(lib.getCandidatesBuffer(h), nc, CAND), view(lib.getResultsBuffer(h), nc, RES))

    def set_window_mode(self, mode, i=None):
        for h in (self.handles if i is None else [self.handles[i]]):
            check(lib.myersSetWindowMode(h, mode), "myersSetWindowMode")

    def set_path(self, path, i=None):
        for h in (self.handles if i is None else [self.handles[i]]):
            check(lib.myersSetKernelPath(h, path), "myersSetKernelPath")

    def set_cutoff(self, cutoff, i=None):
        """Ukkonen's cut-off for the next sends (None: off)."""
        for h in (self.handles if i is None else [self.handles[i]]):
            check(lib.myersSetCutoff(h, -1.0 if cutoff is None else cutoff), "myersSetCutoff")

    def set_graphs(self, enable, i=None):
        for h in (self.handles if i is None else [self.handles[i]]):
            check(lib.myersSetGraphs(h, int(bool(enable))), "myersSetGraphs")

    def send(self, i, distance, num_entries, num_queries, num_cands):
        return check(lib.myersSend(self.handles[i], distance, num_entries, num_queries, num_cands), "myersSend")

    def receive(self, i):
        return lib.myersReceive(self.handles[i])

    def launches(self, i=0):
        return lib.myersBufferLastLaunches(self.handles[i])

    def close(self):
        if self._arr:
            check(lib.myersEnd(C.byref(self._arr)), "myersEnd")
            self._arr = _PP()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def verify_buffers(bufs, peq, qinfo, cands, distance, buffer=0):
    """Fill buffer `buffer` from numpy arrays, send, receive; returns
    (results copy, status of receive)."""
    v_peq, v_qi, v_c, v_res = bufs.views(buffer)
    v_peq[: len(peq)] = peq
    v_qi[: len(qinfo)] = qinfo
    v_c[: len(cands)] = cands
    bufs.send(buffer, distance, len(peq), len(qinfo), len(cands))
    st = bufs.receive(buffer)
    return v_res[: len(cands)].copy(), st


# ---------------------------------------------------------------------------
# device-resident reference and stream-ordered verification


class Reference:
    def __init__(self, words=None, size=None, path=None):
        self.h = C.c_void_p()
        if path is not None:
            check(lib.myersReferenceLoad(C.byref(self.h), path.encode()), "myersReferenceLoad")
        else:
            w = np.ascontiguousarray(words, dtype=np.uint32)
            check(lib.myersReferenceCreate(C.byref(self.h), w.ctypes.data, w.size, size), "myersReferenceCreate")

    @property
    def size(self):
        return lib.myersReferenceSize(self.h)

    def close(self):
        if self.h:
            lib.myersReferenceDestroy(self.h)
            self.h = C.c_void_p()


class Context:
    def __init__(self, max_candidates):
        self.h = C.c_void_p()
        check(lib.myersContextCreate(C.byref(self.h), max_candidates), "myersContextCreate")

    def verify(self, ref, d_peq, n_entries, d_qinfo, n_queries, d_cands, n_cands, distance, d_results,
               window=WINDOW_ALIGNED, path=PATH_PLAIN, stream=0, min_size=0, max_size=0, cutoff=None):
        """Enqueue on `stream` (a cudaStream_t as int). Pointers are device
        addresses. `cutoff` (a fraction of the query length) selects Ukkonen's
        cut-off (myersVerifyCutoffAsync)."""
        if cutoff is not None:
            return check(lib.myersVerifyCutoffAsync(self.h, ref.h, d_peq, n_entries, d_qinfo, n_queries, d_cands,
                                                    n_cands, distance, window, path, cutoff, min_size, max_size,
                                                    d_results, stream), "myersVerifyCutoffAsync")
        return check(lib.myersVerifyRangeAsync(self.h, ref.h, d_peq, n_entries, d_qinfo, n_queries, d_cands, n_cands,
                                               distance, window, path, min_size, max_size, d_results, stream),
                     "myersVerifyRangeAsync")

    def launches(self):
        return lib.myersContextLastLaunches(self.h)

    def flags(self, clear=True):
        f = _U32()
        check(lib.myersContextFlags(self.h, C.byref(f), int(clear)), "myersContextFlags")
        return f.value

    def close(self):
        if self.h:
            lib.myersContextDestroy(self.h)
            self.h = C.c_void_p()


class Traceback:
    """Work space of myersTraceback: ids of up to max_candidates candidates
    and scratch_bytes of device memory for the stored band of each traced
    candidate."""

    def __init__(self, max_candidates, scratch_bytes=1 << 30):
        self.h = C.c_void_p()
        check(lib.myersTracebackCreate(C.byref(self.h), max_candidates, scratch_bytes), "myersTracebackCreate")

    def run(self, ref, d_peq, n_entries, d_qinfo, n_queries, d_cands, d_results, n_cands, distance, max_score,
            d_ops, max_ops, d_alns, window=WINDOW_ALIGNED, stream=0):
        """Enqueue on `stream`; pointers are device addresses. Returns the
        number of candidates traced."""
        check(lib.myersTraceback(self.h, ref.h, d_peq, n_entries, d_qinfo, n_queries, d_cands, d_results, n_cands,
                                 distance, window, max_score, d_ops, max_ops, d_alns, stream), "myersTraceback")
        return lib.myersTracebackLastCount(self.h)

    def chunks(self):
        return lib.myersTracebackLastChunks(self.h)

    def close(self):
        if self.h:
            lib.myersTracebackDestroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def traceback_torch(tb, ref, peq, qinfo, cands, results, distance, max_score, max_ops, window=WINDOW_ALIGNED):
    """Trace numpy inputs (results from a verification of the same inputs)
    on the current torch stream; returns (ALN records, ops (n, max_ops))."""
    import torch

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1)).cuda()

    n = len(cands)
    d_peq, d_qi, d_c, d_r = dev(peq), dev(qinfo), dev(cands), dev(results)
    d_ops = torch.zeros(max(1, n) * max_ops, dtype=torch.int32, device="cuda")
    d_aln = torch.zeros(max(1, n) * 16, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    tb.run(ref, d_peq.data_ptr(), len(peq), d_qi.data_ptr(), len(qinfo), d_c.data_ptr(), d_r.data_ptr(), n,
           distance, max_score, d_ops.data_ptr(), max_ops, d_aln.data_ptr(), window=window,
           stream=stream.cuda_stream)
    torch.cuda.synchronize()
    aln = d_aln.cpu().numpy()[: n * 16].view(ALN)
    ops = d_ops.cpu().numpy().view(np.uint32)[: n * max_ops].reshape(n, max_ops)
    return aln, ops


def verify_torch(ctx, ref, peq, qinfo, cands, distance, window=WINDOW_ALIGNED, path=PATH_PLAIN, min_size=0,
                 max_size=0, device="cuda", cutoff=None):
    """Copy numpy inputs to the GPU with torch, verify, return numpy results."""
    import torch

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).to(device)

    d_peq, d_qi, d_c = dev(peq), dev(qinfo), dev(cands)
    d_res = torch.empty(len(cands) * RES.itemsize, dtype=torch.uint8, device=device)
    stream = torch.cuda.current_stream().cuda_stream
    ctx.verify(ref, d_peq.data_ptr(), len(peq), d_qi.data_ptr(), len(qinfo), d_c.data_ptr(), len(cands), distance,
               d_res.data_ptr(), window=window, path=path, stream=stream, min_size=min_size, max_size=max_size,
               cutoff=cutoff)
    torch.cuda.synchronize()
    return d_res.cpu().numpy().view(RES)


# ---------------------------------------------------------------------------
# serving loop


class ServerConfig(C.Structure):
    _fields_ = [("budgetBytes", C.c_uint64), ("slots", C.c_uint32), ("maxBatchCandidates", C.c_uint32),
                ("maxQueued", C.c_uint32), ("distance", C.c_float), ("windowMode", C.c_int), ("path", C.c_int),
                ("maxQuerySize", C.c_uint32), ("laneWords", C.c_uint32), ("useGraphs", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("refused", C.c_uint64), ("completed", C.c_uint64),
                ("batches", C.c_uint64), ("batchCandidatesMax", C.c_uint64), ("candidatesCompleted", C.c_uint64),
                ("slots", C.c_uint32), ("maxBatchCandidates", C.c_uint32), ("maxBatchQueries", C.c_uint32),
                ("maxBatchEntries", C.c_uint32)]


class Server:
    """Continuous-batching request loop over a resident reference."""

    def __init__(self, ref, distance=0.2, slots=0, budget=0, max_batch_candidates=0, max_queued=0,
                 window=WINDOW_ALIGNED, path=PATH_BATCHED, max_query_size=0, lane_words=0, graphs=True):
        cfg = ServerConfig(budget, slots, max_batch_candidates, max_queued, distance, window, path, max_query_size,
                           lane_words, int(graphs))
        self.h = C.c_void_p()
        check(lib.myersServerCreate(C.byref(self.h), ref.h, C.byref(cfg)), "myersServerCreate")

    def submit(self, peq_entries, query_size, positions):
        """Returns (status, ticket); status E_BUSY means the request was refused."""
        peq_entries = np.ascontiguousarray(peq_entries)
        pos = np.ascontiguousarray(positions, dtype=np.uint64)
        t = C.c_uint64()
        st = lib.myersServerSubmit(self.h, peq_entries.ctypes.data, query_size, pos.ctypes.data, len(pos),
                                   C.byref(t))
        return st, t.value

    def wait(self, ticket, n, timeout_ms=60000):
        out = np.empty(n, dtype=RES)
        st = lib.myersServerWait(self.h, ticket, out.ctypes.data, timeout_ms)
        return st, out

    def poll(self, ticket, n):
        out = np.empty(n, dtype=RES)
        return lib.myersServerPoll(self.h, ticket, out.ctypes.data), out

    def stats(self):
        s = ServerStats()
        check(lib.myersServerStats(self.h, C.byref(s)), "myersServerStats")
        return {f: getattr(s, f) for f, _ in s._fields_}

    def replay(self, peq, qinfo, cand_offset, positions, arrival_ns):
        """Open-loop replay; returns (status, latency_ns per request, results, wall_ns)."""
        n = len(qinfo)
        lat = np.empty(n, dtype=np.uint64)
        res = np.empty(int(cand_offset[-1]), dtype=RES)
        wall = C.c_uint64()
        peq, qinfo = np.ascontiguousarray(peq), np.ascontiguousarray(qinfo)
        off = np.ascontiguousarray(cand_offset, dtype=np.uint32)
        pos = np.ascontiguousarray(positions, dtype=np.uint64)
        arr = np.ascontiguousarray(arrival_ns, dtype=np.uint64)
        st = lib.myersServerReplay(self.h, peq.ctypes.data, qinfo.ctypes.data, off.ctypes.data, pos.ctypes.data, n,
                                   arr.ctypes.data, lat.ctypes.data, res.ctypes.data, C.byref(wall))
        return st, lat, res, wall.value

    def close(self):
        if self.h:
            lib.myersServerDestroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
