"""CPU tests: the oracle against the reference's golden vectors and a textbook
DP, the packers against the reference's packers, the workload generator."""
import os

import numpy as np
import pytest

from conftest import GOLDEN


def test_oracle_matches_reference_aligned(golden_verify, orc):
    g = golden_verify
    res = orc.verify(g["peq"], g["qinfo"], g["cands"], g["ref"], g["ref_size"], g["distance"])
    assert np.array_equal(res, g["res_aligned"].astype(res.dtype))


def test_oracle_matches_reference_exact(golden_verify, orc):
    g = golden_verify
    m = g["exact_mask"]
    res = orc.verify(g["peq"], g["qinfo"], g["cands"], g["ref"], g["ref_size"], g["distance"], exact=True)
    assert np.array_equal(res[m], g["res_exact"][m].astype(res.dtype))


def test_golden_covers_edges(golden_verify):
    g = golden_verify
    sizes = g["qinfo"]["size"]
    pos = g["cands"]["position"]
    assert set(np.unique(pos % 8)) == set(range(8))
    for m in (1, 31, 32, 33, 127, 128, 129, 1024, 1025, 4096):
        assert m in sizes
    assert (g["res_aligned"]["score"] == 0xFFFFFFFF).sum() > 0          # out-of-range windows
    assert sizes.max() > 4096                                            # beyond the API's old cap


def _codes(ref_words, start, n):
    return [(int(ref_words[(start + k) // 8]) >> (4 * ((start + k) % 8))) & 0xF for k in range(n)]


@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_textbook_dp(orc, mg, seed):
    rng = np.random.default_rng(seed)
    ref_size = 3000
    ascii_ref = bytes(rng.choice(list(b"ACGTN"), size=ref_size, p=[0.24, 0.24, 0.24, 0.24, 0.04]).astype(np.uint8))
    words = orc.pack_reference(ascii_ref)
    peq, qinfo, cands, expect_a, expect_e = [], [], [], [], []
    entry = 0
    for q in range(12):
        m = int(rng.integers(1, 80))
        read = bytes(rng.choice(list(b"ACGTN"), size=m).astype(np.uint8))
        peq.append(orc.pack_peq(read).reshape(-1, 20))
        qinfo.append((entry, m))
        entry += (m + 127) // 128
        W = orc.window_bases(m, 0.2)
        for _ in range(3):
            pos = int(rng.integers(0, ref_size - W - 20))
            cands.append((q, pos))
            qc = ["ACGTN".index(chr(b)) for b in read]
            E = W // 8 + (2 if W % 8 else 1)
            start = pos - pos % 8
            expect_a.append(orc.dp_semiglobal(qc, _codes(words, start, 8 * E)))
            expect_e.append(orc.dp_semiglobal(qc, _codes(words, pos, W)))
    peq = np.concatenate(peq).ravel().view(mg.QRY_ENTRY)
    qinfo = np.array(qinfo, dtype=np.uint32).view(mg.QINFO).ravel()
    c = np.zeros(len(cands), dtype=mg.CAND)
    c["query"] = [x[0] for x in cands]
    c["position"] = [x[1] for x in cands]
    ra = orc.verify(peq, qinfo, c, words, ref_size, 0.2)
    re_ = orc.verify(peq, qinfo, c, words, ref_size, 0.2, exact=True)
    assert [(int(r["score"]), int(r["column"])) for r in ra] == expect_a
    assert [(int(r["score"]), int(r["column"])) for r in re_] == expect_e


def test_reference_packer_format(orc):
    d = np.load(os.path.join(GOLDEN, "packers.npz"))
    fasta = d["fasta"].tobytes()
    seq = b"".join(line for line in fasta.split(b"\n") if line and not line.startswith(b">"))
    ref_file = d["ref_file"].tobytes()
    num_entries, size = np.frombuffer(ref_file[:8], dtype=np.uint32)
    assert size == len(seq) and num_entries == (len(seq) + 7) // 8
    ref_words = np.frombuffer(ref_file[8:], dtype=np.uint32)
    mine = orc.pack_reference(seq)
    full = size // 8  # the reference packs the partial last word from stale bytes
    assert np.array_equal(mine[:full], ref_words[:full])
    last_mask = (1 << (4 * (size % 8))) - 1
    assert (int(mine[full]) & last_mask) == (int(ref_words[full]) & last_mask)


def test_reference_peq_format(orc, mg):
    d = np.load(os.path.join(GOLDEN, "packers.npz"))
    prof = d["prof"].tobytes().strip().split(b"\n")
    qry = d["qry_file"].tobytes()
    hdr = np.frombuffer(qry[:20], dtype=np.uint32)
    _, tot_entries, _, nq, nc = (int(x) for x in hdr)
    off = 20
    peq = np.frombuffer(qry[off:off + 80 * tot_entries], dtype=np.uint32).reshape(-1, 20)
    off += 80 * tot_entries
    cands = np.frombuffer(qry[off:off + 16 * nc], dtype=mg.CAND)
    off += 16 * nc
    qinfo = np.frombuffer(qry[off:off + 8 * nq], dtype=mg.QINFO)
    assert nq == len(prof)
    entry = 0
    for i, line in enumerate(prof):
        read = line.split(b"\t")[0]
        assert qinfo[i]["size"] == len(read) and qinfo[i]["posEntry"] == entry
        ne = (len(read) + 127) // 128
        assert np.array_equal(orc.pack_peq(read).reshape(-1, 20), peq[entry:entry + ne])
        entry += ne
        for j, tok in enumerate(line.split(b"\t")[1:]):
            assert cands[3 * i + j]["query"] == i
            assert cands[3 * i + j]["position"] == int(tok.split(b":")[2])


def test_synth_deterministic(mg):
    r1 = mg.make_reference(1_000_000, 5)
    r2 = mg.make_reference(1_000_000, 5)
    assert np.array_equal(r1, r2)
    codes = (r1[:, None] >> (4 * np.arange(8, dtype=np.uint32))) & 0xF
    frac_n = (codes.ravel()[:1_000_000] == 4).mean()
    assert 0.0 < frac_n < 0.01
    s = mg.workload_spec(3, scale=0.0005, ref_size=100_000)
    a = mg.make_workload(s, r1)
    b = mg.make_workload(s, r1)
    for k in ("peq", "qinfo", "cands"):
        assert np.array_equal(a[k], b[k])
    assert set(np.unique(a["lengths"])) <= {100, 200, 400, 600, 800, 1000}


def test_synth_thread_independent(mg):
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, 'myers-gpu_b200'); import myersgpu as mg, numpy as np;"
            "r = mg.make_reference(300_000, 9); w = mg.make_workload(mg.workload_spec(5, scale=0.002, ref_size=300_000), r);"
            "print(int(r.sum() % 1000003), int(w['cands']['position'].sum() % 1000003), int(w['peq'].view(np.uint32).sum()))")
    root = os.path.dirname(GOLDEN.rstrip("/")).rsplit("/", 1)[0]
    outs = set()
    for t in ("1", "3"):
        env = dict(os.environ, OMP_NUM_THREADS=t)
        outs.add(subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True, text=True,
                                check=True).stdout)
    assert len(outs) == 1


def _dp_traceback(qc, tc, end_col):
    """Pure-Python DP and traceback with the stated step order (diagonal,
    query base alone, text base alone) from (m, end_col + 1). Returns
    (start column, ops as (code, length) runs)."""
    m, n = len(qc), end_col + 1
    D = [[0] * (n + 1) for _ in range(m + 1)]
    for i in range(1, m + 1):
        D[i][0] = i
        for j in range(1, n + 1):
            D[i][j] = min(D[i - 1][j - 1] + (qc[i - 1] != tc[j - 1]), D[i - 1][j] + 1, D[i][j - 1] + 1)
    i, j, rev = m, n, []
    while i > 0:
        if j > 0 and D[i - 1][j - 1] + (qc[i - 1] != tc[j - 1]) == D[i][j]:
            rev.append("=" if qc[i - 1] == tc[j - 1] else "X")
            i, j = i - 1, j - 1
        elif D[i - 1][j] + 1 == D[i][j]:
            rev.append("I")
            i -= 1
        else:
            rev.append("D")
            j -= 1
    runs = []
    for op in reversed(rev):
        if runs and runs[-1][0] == op:
            runs[-1][1] += 1
        else:
            runs.append([op, 1])
    return j, [(o, k) for o, k in runs]


@pytest.mark.parametrize("exact", [False, True])
def test_oracle_traceback_matches_textbook(orc, mg, exact):
    """The oracle's traceback (the definition the GPU path is checked
    against) equals an independent pure-Python DP traceback, and every
    alignment is consistent: query bases = m, text bases = end - start + 1,
    edit cost = score."""
    rng = np.random.default_rng(11 + exact)
    ref_size = 4000
    ascii_ref = bytes(rng.choice(list(b"ACGTN"), size=ref_size, p=[0.24, 0.24, 0.24, 0.24, 0.04]).astype(np.uint8))
    words = orc.pack_reference(ascii_ref)
    peq, qinfo, cands, reads = [], [], [], []
    entry = 0
    for q in range(10):
        m = int(rng.integers(1, 60))
        read = bytes(rng.choice(list(b"ACGTN"), size=m).astype(np.uint8))
        reads.append(["ACGTN".index(chr(b)) for b in read])
        peq.append(orc.pack_peq(read).reshape(-1, 20))
        qinfo.append((entry, m))
        entry += (m + 127) // 128
        W = orc.window_bases(m, 0.2)
        for _ in range(4):
            cands.append((q, int(rng.integers(0, ref_size - W - 20))))
    peq = np.concatenate(peq).ravel().view(mg.QRY_ENTRY)
    qinfo = np.array(qinfo, dtype=np.uint32).view(mg.QINFO).ravel()
    c = np.zeros(len(cands), dtype=mg.CAND)
    c["query"] = [x[0] for x in cands]
    c["position"] = [x[1] for x in cands]
    res = orc.verify(peq, qinfo, c, words, ref_size, 0.2, exact=exact)
    aln, ops = orc.traceback(peq, qinfo, c, res, words, ref_size, 0.2, 10 ** 6, 256, exact=exact)
    names = {7: "=", 8: "X", 1: "I", 2: "D"}
    for k, (q, pos) in enumerate(cands):
        m = len(reads[q])
        W = orc.window_bases(m, 0.2)
        start = pos if exact else pos - pos % 8
        ncols = W if exact else 8 * (W // 8 + (2 if W % 8 else 1))
        tc = _codes(words, start, ncols)
        tc = [0 if t > 4 else t for t in tc]
        a0, runs = _dp_traceback(reads[q], tc, int(res["column"][k]))
        got = [(names[int(o) & 15], int(o) >> 4) for o in ops[k, : aln["num_ops"][k]]]
        assert (int(aln["start_column"][k]), got) == (a0, runs)
        n_q = sum(n for o, n in got if o in "=XI")
        n_t = sum(n for o, n in got if o in "=XD")
        cost = sum(n for o, n in got if o in "XID")
        assert n_q == m and n_t == int(res["column"][k]) - a0 + 1 and cost == int(res["score"][k])
    # a bound below every score traces nothing; a wrong score is caught
    aln0, _ = orc.traceback(peq, qinfo, c, res, words, ref_size, 0.2, 0, 16, exact=exact)
    assert ((aln0["num_ops"] == orc.TB_NOT_TRACED) | (res["score"] == 0)).all()
    bad = res.copy()
    bad["score"] += 1
    aln1, _ = orc.traceback(peq, qinfo, c, bad, words, ref_size, 0.2, 10 ** 6, 16, exact=exact)
    assert (aln1["num_ops"] == orc.TB_INCONSISTENT).all()


def test_cutoff_contract_on_reference_outputs(mg, orc, golden_verify):
    """apply_cutoff keeps every result whose score is within (uint32)(m *
    cutoff) (float32) and marks the others, leaving unverified candidates
    ({0, 0xFFFFFFFF}) as they are."""
    g = golden_verify
    res = g["res_aligned"]
    m = g["qinfo"]["size"][g["cands"]["query"]]
    for cutoff in (0.0, 0.05, 0.2, 2.0):
        out = orc.apply_cutoff(res, g["qinfo"], g["cands"], cutoff)
        for i in range(0, len(res), 7):
            bound = int(np.float32(int(m[i])) * np.float32(cutoff))
            if res[i]["score"] == orc.NO_RESULT or res[i]["score"] <= bound:
                assert out[i] == res[i]
            else:
                assert out[i]["score"] == orc.NO_MATCH and out[i]["column"] == orc.NO_MATCH
