"""Generate the golden fixtures in this directory from the reference's own code.

Run where the reference sources are present (they are compiled into
oracle/_ref/ by `make -C oracle REF=<reference checkout>`):

    python tests/golden/make_golden.py

Writes:
  packers.npz   a small multi-FASTA and GEM .prof text, and what the
                reference's packers made of them (genReference-4bits: the
                .4bits.ref bytes; genCandidate-reorder: the .gem.qry bytes)
  verify.npz    seeded inputs (packed reference, PEQ, query info, candidates)
                with the reference CPU Myers' results: aligned windows from
                src-integration/myers-reorderBuffer-padding.c, exact windows
                from src/myers-4bits.c (fixed-length groups only)

The fixtures hold only data: synthetic sequences and the numbers the
reference's code computed from them.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "myers-gpu_b200"))

import myersgpu as mg  # noqa: E402
import oracle as orc  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref")
DIST = 0.2


def rand_bases(rng, n, n_frac=0.02, lower_frac=0.1):
    b = rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), size=n)
    n_mask = rng.random(n) < n_frac
    b[n_mask] = ord("N")
    low = rng.random(n) < lower_frac
    b[low] = b[low] | 0x20  # lower case (the packers accept both)
    return b


def packers(rng, tmp):
    # multi-FASTA with two records, lines of 60, odd total length
    seq = rand_bases(rng, 5003)
    fa = os.path.join(tmp, "g.fa")
    with open(fa, "wb") as f:
        f.write(b">chr1 test\n")
        for i in range(0, 3000, 60):
            f.write(bytes(seq[i:min(i + 60, 3000)]) + b"\n")
        f.write(b">chr2\n")
        for i in range(3000, 5003, 60):
            f.write(bytes(seq[i:min(i + 60, 5003)]) + b"\n")
    subprocess.run([os.path.join(REF_BIN, "genReference-4bits"), fa], check=True, capture_output=True)
    ref_bytes = open(fa + ".5003.4bits.ref", "rb").read()
    # GEM .prof: read \t area:strand:pos:score ... (genCandidate-reorder.c:114-179)
    lines, reads = [], []
    for q, m in enumerate([100, 128, 129, 300, 257, 1000, 31, 33]):
        r = rand_bases(rng, m, n_frac=0.01)
        reads.append(bytes(r))
        cands = "\t".join(f"chr1:+:{int(p)}:{int(s)}" for p, s in zip(rng.integers(0, 4000, 3), rng.integers(0, 9, 3)))
        lines.append(bytes(r) + b"\t" + cands.encode())
    prof = os.path.join(tmp, "c.prof")
    with open(prof, "wb") as f:
        f.write(b"\n".join(lines) + b"\n")
    subprocess.run([os.path.join(REF_BIN, "genCandidate-reorder"), prof], check=True, capture_output=True)
    out = [p for p in os.listdir(tmp) if p.startswith("c.prof.") and p.endswith(".gem.qry")]
    qry_bytes = open(os.path.join(tmp, out[0]), "rb").read()
    fa_text = open(fa, "rb").read()
    prof_text = open(prof, "rb").read()
    return dict(fasta=np.frombuffer(fa_text, np.uint8), ref_file=np.frombuffer(ref_bytes, np.uint8),
                prof=np.frombuffer(prof_text, np.uint8), qry_file=np.frombuffer(qry_bytes, np.uint8))


def edge_cases(rng, ref_words, ref_size, start_query, start_entry):
    """Hand-placed candidates: every pos%8, windows at the reference end,
    out-of-range positions, lengths at word and entry boundaries."""
    lengths = [1, 2, 31, 32, 33, 63, 64, 65, 127, 128, 129, 255, 256, 257, 511, 512, 513, 1023, 1024, 1025, 4096]
    peqs, qinfo, cands = [], [], []
    entry = start_entry
    for qi, m in enumerate(lengths):
        q = start_query + qi
        # read copied from the reference with a few substitutions
        p0 = int(rng.integers(0, ref_size - 2 * m - 64))
        codes = [(int(ref_words[(p0 + k) // 8]) >> (4 * ((p0 + k) % 8))) & 0xF for k in range(m)]
        for k in rng.integers(0, m, max(1, m // 25)):
            codes[k] = int(rng.integers(0, 5))
        read = bytes(b"ACGTN"[c] for c in codes)
        peqs.append(orc.pack_peq(read).reshape(-1, 20))
        qinfo.append((entry, m))
        entry += (m + 127) // 128
        w = orc.window_bases(m, DIST)
        pos_list = [p0 - m // 5 + d for d in range(-3, 5)]            # all pos%8 around the true start
        pos_list += [max(0, p0 - m // 5 + 1000 * k) for k in range(1, 3)]
        pos_list += [ref_size - w - 1, ref_size - w - 2, ref_size - w - 9]   # last valid windows
        pos_list += [ref_size - w, ref_size - 1, ref_size, ref_size + 5]     # out of range
        for p in pos_list:
            cands.append((q, max(0, p)))
    peq = np.concatenate(peqs).ravel().view(mg.QRY_ENTRY)
    qi = np.array(qinfo, dtype=np.uint32).view(mg.QINFO).ravel()
    c = np.zeros(len(cands), dtype=mg.CAND)
    c["query"] = [x[0] for x in cands]
    c["position"] = [x[1] for x in cands]
    return peq, qi, c


def concat_workloads(parts):
    peq, qinfo, cands = [], [], []
    ne = nq = 0
    for p, q, c in parts:
        q = q.copy()
        c = c.copy()
        q["posEntry"] += ne
        c["query"] += nq
        peq.append(p)
        qinfo.append(q)
        cands.append(c)
        ne += len(p)
        nq += len(q)
    return np.concatenate(peq), np.concatenate(qinfo), np.concatenate(cands)


def verify_fixture(rng):
    ref_size = 400_003  # not a multiple of 8: the last word is partial
    ref = mg.make_reference(ref_size, 11, n_frac=0.002)
    parts, groups = [], []
    for k, scale in [(1, 0.004), (2, 0.0003), (3, 0.00015), (4, 0.0003), (5, 0.0006)]:
        w = mg.make_workload(mg.workload_spec(k, scale=scale, ref_size=ref_size), ref)
        parts.append((w["peq"], w["qinfo"], w["cands"]))
        groups.append(k)
    ne = sum(len(p[0]) for p in parts)
    nq = sum(len(p[1]) for p in parts)
    parts.append(edge_cases(rng, ref, ref_size, 0, 0))
    groups.append(0)
    peq, qinfo, cands = concat_workloads(parts)
    group = np.concatenate([np.full(len(p[2]), g, dtype=np.uint8) for p, g in zip(parts, groups)])
    res, _ = orc.reference_verify_aligned(peq, qinfo, cands, ref, ref_size, DIST, uncapped=True)
    # exact windows: the reference oracle takes one query length per call
    ex = np.zeros(len(cands), dtype=orc.RES)
    ex_mask = np.zeros(len(cands), dtype=bool)
    off = 0
    for (p, q, c), g in zip(parts, groups):
        if g in (1, 2):
            r, _ = orc.reference_verify_exact(p, q, c, ref, ref_size, DIST)
            ex[off:off + len(c)] = r
            ex_mask[off:off + len(c)] = True
        off += len(c)
    return dict(ref_words=ref, ref_size=np.uint64(ref_size), distance=np.float32(DIST),
                peq=peq.view(np.uint32).reshape(-1, 20), qinfo=qinfo.view(np.uint32).reshape(-1, 2),
                cand_query=cands["query"], cand_pos=cands["position"], group=group,
                res_aligned=res.view(np.uint32).reshape(-1, 2), res_exact=ex.view(np.uint32).reshape(-1, 2),
                exact_mask=ex_mask)


def main():
    if not orc.have_reference():
        sys.exit("oracle/_ref is not built (make -C oracle REF=<reference checkout>)")
    rng = np.random.default_rng(20241203)
    with tempfile.TemporaryDirectory() as tmp:
        np.savez_compressed(os.path.join(HERE, "packers.npz"), **packers(rng, tmp))
    np.savez_compressed(os.path.join(HERE, "verify.npz"), **verify_fixture(rng))
    for f in ("packers.npz", "verify.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
