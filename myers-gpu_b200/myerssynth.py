"""Seeded synthetic workloads of the Myers benchmark, and the record layouts.

Binds libmyers_synth.so (host C, OpenMP; myers-gpu_b200/csrc/synth.c) with
ctypes. It loads no CUDA code, so CPU-only users (the CPU baseline of the
benchmark, the oracle's tests) can generate the same seeded inputs as the
GPU path without loading libmyers_b200.so.

Record layouts (numpy dtypes) match the C structs of include/myers-interface.h
byte for byte:
  QRY_ENTRY  qryEntry_t  80 B  bitmap[5][4] u32  (128 query bases)
  CAND       candInfo_t  16 B  u32 query, 4 B padding, u64 position
  QINFO      qryInfo_t    8 B  u32 posEntry, u32 size
  RES        resEntry_t   8 B  u32 column, u32 score
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SYNTH_PATH = os.path.join(HERE, "libmyers_synth.so")

QRY_ENTRY = np.dtype([("bitmap", "<u4", (5, 4))])
CAND = np.dtype([("query", "<u4"), ("pad", "<u4"), ("position", "<u8")])
QINFO = np.dtype([("posEntry", "<u4"), ("size", "<u4")])
RES = np.dtype([("column", "<u4"), ("score", "<u4")])
assert QRY_ENTRY.itemsize == 80 and CAND.itemsize == 16 and QINFO.itemsize == 8 and RES.itemsize == 8

if not os.path.exists(SYNTH_PATH):
    raise ImportError("libmyers_synth.so is not built: run myers-gpu_b200/build.py")
synth = C.CDLL(SYNTH_PATH)


class SynthSpec(C.Structure):
    _fields_ = [
        ("ref_size", C.c_uint64), ("num_reads", C.c_uint32),
        ("len_kind", C.c_uint32), ("len_fixed", C.c_uint32), ("len_lo", C.c_uint32), ("len_hi", C.c_uint32),
        ("len_set_n", C.c_uint32), ("len_set", C.c_uint32 * 16), ("len_weights", C.c_double * 16),
        ("mut_kind", C.c_uint32), ("sub", C.c_double), ("ins", C.c_double), ("del_", C.c_double),
        ("rate_lo", C.c_double), ("rate_hi", C.c_double), ("indel_mean", C.c_double),
        ("cand_kind", C.c_uint32), ("cand_fixed", C.c_uint32), ("cand_lambda", C.c_double),
        ("cand_cap", C.c_uint32), ("cand_lo", C.c_uint32), ("cand_hi", C.c_uint32),
        ("jitter", C.c_uint32), ("distance", C.c_float), ("seed", C.c_uint64),
    ]


synth.synth_reference.restype = C.c_int
synth.synth_reference.argtypes = [C.c_uint64, C.c_double, C.c_uint32, C.c_uint32, C.c_uint64, C.c_void_p, C.c_uint64]
synth.synth_plan.restype = C.c_int
synth.synth_plan.argtypes = [C.POINTER(SynthSpec), C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64),
                             C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
synth.synth_fill.restype = C.c_int
synth.synth_fill.argtypes = [C.POINTER(SynthSpec), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_void_p, C.c_void_p, C.c_void_p]

PAD_WORD = 0x44444444


def make_reference(size, seed, n_frac=0.001, run=(50, 500), pad_words=0):
    """Packed reference of `size` bases (i.i.d. ACGT with N runs); returns the
    ceil(size/8) words plus `pad_words` words of N."""
    nw = (size + 7) // 8 + pad_words
    words = np.empty(nw, dtype=np.uint32)
    rc = synth.synth_reference(size, n_frac, run[0], run[1], seed, words.ctypes.data, nw)
    if rc:
        raise RuntimeError(f"synth_reference failed ({rc})")
    return words


def spec(ref_size, num_reads, seed, distance=0.2, lengths=100, length_weights=None, length_range=None,
         uniform_lengths=None, sub=0.04, ins=0.005, dele=0.005, rate_range=None, indel_mean=1.0, cands=11,
         cand_poisson=None, cand_cap=0, cand_range=None, jitter=8):
    s = SynthSpec()
    s.ref_size, s.num_reads, s.seed, s.distance, s.jitter = ref_size, num_reads, seed, distance, jitter
    if length_range is not None:
        s.len_kind, s.len_lo, s.len_hi = 2, length_range[0], length_range[1]
    elif uniform_lengths is not None:
        s.len_kind, s.len_set_n = 3, len(uniform_lengths)
        for i, v in enumerate(uniform_lengths):
            s.len_set[i] = v
    elif length_weights is not None:
        s.len_kind, s.len_set_n = 1, len(lengths)
        for i, (v, w) in enumerate(zip(lengths, length_weights)):
            s.len_set[i], s.len_weights[i] = v, w
    else:
        s.len_kind, s.len_fixed = 0, lengths
    if rate_range is not None:
        s.mut_kind, s.rate_lo, s.rate_hi = 1, rate_range[0], rate_range[1]
    else:
        s.mut_kind, s.sub, s.ins, s.del_ = 0, sub, ins, dele
    s.indel_mean = indel_mean
    if cand_poisson is not None:
        s.cand_kind, s.cand_lambda, s.cand_cap = 1, cand_poisson, cand_cap
    elif cand_range is not None:
        s.cand_kind, s.cand_lo, s.cand_hi = 2, cand_range[0], cand_range[1]
    else:
        s.cand_kind, s.cand_fixed = 0, cands
    return s


def make_workload(s, ref_words, ascii=False):
    """Reads and candidates for spec `s` over `ref_words`. Returns a dict with
    peq (QRY_ENTRY), qinfo (QINFO), cands (CAND), lengths, ncands, true_pos
    and, if asked, the reads as one ASCII byte string (bases back to back)."""
    n = s.num_reads
    lengths = np.empty(n, dtype=np.uint32)
    ncands = np.empty(n, dtype=np.uint32)
    te, tc, tb = C.c_uint64(), C.c_uint64(), C.c_uint64()
    synth.synth_plan(C.byref(s), lengths.ctypes.data, ncands.ctypes.data, C.byref(te), C.byref(tc), C.byref(tb))
    peq = np.empty(te.value, dtype=QRY_ENTRY)
    qinfo = np.empty(n, dtype=QINFO)
    cands = np.empty(tc.value, dtype=CAND)
    true_pos = np.empty(n, dtype=np.uint64)
    asc = np.empty(tb.value, dtype=np.uint8) if ascii else None
    rc = synth.synth_fill(C.byref(s), ref_words.ctypes.data, lengths.ctypes.data, ncands.ctypes.data,
                          qinfo.ctypes.data, peq.ctypes.data, cands.ctypes.data,
                          asc.ctypes.data if ascii else None, true_pos.ctypes.data)
    if rc:
        raise RuntimeError(f"synth_fill failed ({rc})")
    out = dict(peq=peq, qinfo=qinfo, cands=cands, lengths=lengths, ncands=ncands, true_pos=true_pos)
    if ascii:
        out["ascii"] = asc
    return out


# The workloads of the benchmark, by number. `scale` shrinks the read count
# (and, for the 16 Mbase one, nothing else) for tests.
GENOME = 3_100_000_000


def workload_spec(k, seed=None, scale=1.0, ref_size=None):
    if k == 1:
        return spec(ref_size or 16_000_000, max(1, int(100_000 * scale)), seed or 101, lengths=100,
                    sub=0.04, ins=0.005, dele=0.005, cands=11)
    if k == 2:
        return spec(ref_size or GENOME, max(1, int(1_000_000 * scale)), seed or 202, lengths=1000,
                    sub=0.05, ins=0.005, dele=0.005, cands=11)
    if k == 3:
        return spec(ref_size or GENOME, max(1, int(2_000_000 * scale)), seed or 303,
                    lengths=[100, 200, 400, 600, 800, 1000], length_weights=[30, 20, 15, 15, 10, 10],
                    rate_range=(0.02, 0.08), cand_poisson=10.0, cand_cap=64)
    if k == 4:
        return spec(ref_size or GENOME, max(1, int(100_000 * scale)), seed or 404, length_range=(1000, 10000),
                    sub=0.03, ins=0.06, dele=0.03, indel_mean=1.5, cand_poisson=4.0)
    if k == 5:
        return spec(ref_size or GENOME, max(1, int(100_000 * scale)), seed or 505,
                    uniform_lengths=list(range(100, 1001, 100)), rate_range=(0.02, 0.08), cand_range=(1, 64))
    raise ValueError(k)


def cells(qinfo, cands, distance=0.2, exact=False):
    """DP cells (m x columns) of the candidates, as the throughput unit."""
    m = qinfo["size"][cands["query"]].astype(np.float64)
    f = np.float32(1.0) + np.float32(2.0) * np.float32(distance)
    w = np.floor(m.astype(np.float32) * f).astype(np.float64)
    n = w if exact else 8 * (np.floor(w / 8) + np.where(w % 8 != 0, 2, 1))
    return m * n, np.ceil(m / 32) * n
