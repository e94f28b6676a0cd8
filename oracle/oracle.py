"""Test infrastructure only: ctypes bindings of the CPU oracle.

  liboracle.so            the C restatement (myers_oracle.c)
  _ref/libref_padding.so  the reference's own aligned-window CPU Myers
  _ref/libref_exact.so    the reference's own exact-window CPU Myers

Only the tests, the smoke check and the benchmark's CPU-baseline leg use
this module, as the checker. Inputs use the API record layouts (numpy dtypes
of myersgpu: QRY_ENTRY, QINFO, CAND, RES).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
PAD_WORD = 0x44444444
RES = np.dtype([("column", "<u4"), ("score", "<u4")])


def build(ref_src=None):
    """Compile the oracle (and _ref/, when `ref_src` names a checkout of the
    reference's sources)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE] + ([f"REF={ref_src}"] if ref_src else []), check=True)


def _lib(name, required=True):
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        if required:
            raise ImportError(f"{name} is not built (make -C oracle)")
        return None
    return C.CDLL(path)


_orc = _lib("liboracle.so")
_orc.orc_verify.restype = None
_orc.orc_verify.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_uint64,
                            C.c_float, C.c_int, C.c_void_p, C.c_int]
_orc.orc_window_bases.restype = C.c_uint32
_orc.orc_window_bases.argtypes = [C.c_uint32, C.c_float]
_orc.orc_pack_reference.restype = None
_orc.orc_pack_reference.argtypes = [C.c_char_p, C.c_uint64, C.c_void_p]
_orc.orc_pack_peq.restype = None
_orc.orc_pack_peq.argtypes = [C.c_char_p, C.c_uint32, C.c_void_p]
_orc.orc_traceback.restype = None
_orc.orc_traceback.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                               C.c_uint64, C.c_float, C.c_int, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                               C.c_int]

ALN = np.dtype([("start_column", "<u4"), ("num_ops", "<u4"), ("score", "<u4"), ("end_column", "<u4")])
TB_NOT_TRACED = 0xFFFFFFFF
TB_INCONSISTENT = 0xFFFFFFFE
OP_CODES = {7: "=", 8: "X", 1: "I", 2: "D"}


def window_bases(m, distance):
    return _orc.orc_window_bases(m, distance)


def verify(peq, qinfo, cands, ref_words, ref_size, distance, exact=False, nthreads=0):
    """Restated reference algorithm over all candidates (OpenMP)."""
    peq = np.ascontiguousarray(peq)
    qinfo = np.ascontiguousarray(qinfo)
    cands = np.ascontiguousarray(cands)
    ref_words = np.ascontiguousarray(ref_words, dtype=np.uint32)
    res = np.empty(len(cands), dtype=RES)
    _orc.orc_verify(peq.ctypes.data, qinfo.ctypes.data, cands.ctypes.data, len(cands), ref_words.ctypes.data,
                    ref_words.size, ref_size, distance, int(exact), res.ctypes.data, nthreads)
    return res


NO_RESULT = 0xFFFFFFFF
NO_MATCH = 0xFFFFFFFF


def cutoff_bound(m, cutoff):
    """The cut-off bound of queries of m bases: (uint32_t)(m * cutoff) with
    the product in float32 (the window sizing's convention)."""
    return np.floor(np.asarray(m, dtype=np.float32) * np.float32(cutoff)).astype(np.int64)


def apply_cutoff(results, qinfo, cands, cutoff):
    """The cut-off contract on full results: a verified candidate whose
    minimum score exceeds the bound of its query becomes {NO_MATCH, NO_MATCH};
    everything else is unchanged. The contract of GEMTools'
    gt_map_block_bpm_get_distance__cutoff (GEMTools/src/gt_map_align_bpm.c:
    141-210), which returns a distance and position only within its
    max_distance, on results pinned to the reference's CPU Myers."""
    out = np.array(results, copy=True)
    m = qinfo["size"][cands["query"]]
    sel = (out["score"] != NO_RESULT) & (out["score"].astype(np.int64) > cutoff_bound(m, cutoff))
    out["column"][sel] = NO_MATCH
    out["score"][sel] = NO_MATCH
    return out


def traceback(peq, qinfo, cands, results, ref_words, ref_size, distance, max_score, max_ops, exact=False,
              nthreads=0):
    """Alignments of the candidates whose score is <= max_score: returns
    (records of ALN, ops as a (len(cands), max_ops) u32 array; row k holds
    num_ops[k] run-length ops, length << 4 | SAM code)."""
    peq = np.ascontiguousarray(peq)
    qinfo = np.ascontiguousarray(qinfo)
    cands = np.ascontiguousarray(cands)
    results = np.ascontiguousarray(results)
    ref_words = np.ascontiguousarray(ref_words, dtype=np.uint32)
    aln = np.empty(len(cands), dtype=ALN)
    ops = np.zeros((len(cands), max(1, max_ops)), dtype=np.uint32)
    _orc.orc_traceback(peq.ctypes.data, qinfo.ctypes.data, cands.ctypes.data, results.ctypes.data, len(cands),
                       ref_words.ctypes.data, ref_words.size, ref_size, distance, int(exact), max_score,
                       ops.ctypes.data, max_ops, aln.ctypes.data, nthreads)
    return aln, ops


def cigar(ops, n):
    """SAM-style string of the first n run-length ops."""
    return "".join(f"{int(o) >> 4}{OP_CODES[int(o) & 15]}" for o in ops[:n])


def pack_reference(ascii_bases):
    b = bytes(ascii_bases)
    out = np.empty((len(b) + 7) // 8, dtype=np.uint32)
    _orc.orc_pack_reference(b, len(b), out.ctypes.data)
    return out


def pack_peq(read):
    b = bytes(read)
    out = np.zeros(((len(b) + 127) // 128) * 20, dtype=np.uint32)
    _orc.orc_pack_peq(b, len(b), out.ctypes.data)
    return out


# ---- the reference's own CPU Myers ----

_pad = _lib(os.path.join("_ref", "libref_padding.so"), required=False)
_exa = _lib(os.path.join("_ref", "libref_exact.so"), required=False)
if _pad is not None:
    _pad.refshim_verify_aligned.restype = C.c_int
    _pad.refshim_verify_aligned.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                            C.c_void_p, C.c_uint32, C.c_uint32, C.c_float, C.c_void_p, C.c_int,
                                            C.c_int, C.POINTER(C.c_double)]
if _exa is not None:
    _exa.refshim_verify_exact.restype = C.c_int
    _exa.refshim_verify_exact.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                          C.c_uint32, C.c_uint32, C.c_float, C.c_void_p, C.c_int,
                                          C.POINTER(C.c_double)]


def have_reference():
    return _pad is not None and _exa is not None


def pad_reference(ref_words):
    """The packed reference followed by 16 words of N: the reference's CPU
    code reads up to two words past the packed array. Callers that check
    several batches against one reference pass this to the calls below
    (`padded=`) instead of having each call copy the reference."""
    return np.concatenate([np.asarray(ref_words, dtype=np.uint32), np.full(16, PAD_WORD, dtype=np.uint32)])


def reference_verify_aligned(peq, qinfo, cands, ref_words, ref_size, distance, nthreads=0, uncapped=True,
                             padded=None):
    """The reference's computeAllQueriesCPU (aligned window). Returns
    (results, seconds of its compute region, including the direct
    computeMyers calls of the reads beyond its 4096-base cap)."""
    if _pad is None:
        raise RuntimeError("oracle/_ref/libref_padding.so is not built")
    peq = np.ascontiguousarray(peq)
    qinfo = np.ascontiguousarray(qinfo)
    cands = np.ascontiguousarray(cands)
    w = pad_reference(ref_words) if padded is None else padded
    res = np.empty(len(cands), dtype=RES)
    sec = C.c_double()
    rc = _pad.refshim_verify_aligned(peq.ctypes.data, len(peq), qinfo.ctypes.data, len(qinfo), cands.ctypes.data,
                                     len(cands), w.ctypes.data, len(ref_words), ref_size, distance, res.ctypes.data,
                                     nthreads, int(uncapped), C.byref(sec))
    if rc:
        raise RuntimeError(f"refshim_verify_aligned failed ({rc})")
    return res, sec.value


def reference_verify_exact(peq, qinfo, cands, ref_words, ref_size, distance, nthreads=0, padded=None):
    """The reference's exact-window CPU Myers (one query length only)."""
    if _exa is None:
        raise RuntimeError("oracle/_ref/libref_exact.so is not built")
    peq = np.ascontiguousarray(peq)
    qinfo = np.ascontiguousarray(qinfo)
    cands = np.ascontiguousarray(cands)
    w = pad_reference(ref_words) if padded is None else padded
    res = np.empty(len(cands), dtype=RES)
    sec = C.c_double()
    rc = _exa.refshim_verify_exact(peq.ctypes.data, qinfo.ctypes.data, len(qinfo), cands.ctypes.data, len(cands),
                                   w.ctypes.data, len(ref_words), ref_size, distance, res.ctypes.data, nthreads,
                                   C.byref(sec))
    if rc:
        raise RuntimeError(f"refshim_verify_exact failed ({rc})")
    return res, sec.value


def dp_semiglobal(query, text):
    """Textbook O(m*n) semi-global edit distance (D[0][j] = 0, D[i][0] = i)
    of two code sequences; returns (min score over columns 1..n with the
    first-minimum tie-break starting from (m, 0), its column - 1). Pure
    Python: tiny cases only. Follows the DP of src/sw.c:187-236."""
    m, n = len(query), len(text)
    prev = [0] * (n + 1)
    for i in range(1, m + 1):
        cur = [i] + [0] * n
        qi = query[i - 1]
        for j in range(1, n + 1):
            cur[j] = min(prev[j - 1] + (0 if qi == text[j - 1] else 1), prev[j] + 1, cur[j - 1] + 1)
        prev = cur
    best, col = m, 0
    for j in range(1, n + 1):
        if prev[j] < best:
            best, col = prev[j], j - 1
    return best, col
