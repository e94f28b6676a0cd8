"""GPU tests of the device packers against the oracle's packers and the
reference's own packer output (tests/golden/packers.npz)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).cuda()


def test_pack_peq_matches_host_packers(mg, orc, cuda_ok):
    import torch
    ref_size = 1_000_000
    ref = mg.make_reference(ref_size, 9)
    w = mg.make_workload(mg.workload_spec(3, scale=0.001, ref_size=ref_size), ref, ascii=True)
    rng = np.random.default_rng(0)
    asc = w["ascii"].copy()
    low = rng.random(asc.size) < 0.1
    asc[low] |= 0x20                      # lower case packs the same
    other = rng.random(asc.size) < 0.002
    asc[other] = ord("X")                 # other characters pack as N
    lengths = w["qinfo"]["size"].astype(np.uint64)
    offsets = np.concatenate([[0], np.cumsum(lengths)]).astype(np.uint64)
    expect = np.concatenate([orc.pack_peq(bytes(asc[offsets[i]:offsets[i + 1]])).reshape(-1, 20)
                             for i in range(len(lengths))])
    stream = torch.cuda.current_stream().cuda_stream
    # every device buffer stays referenced while the kernels may use it
    d_asc, d_asc_plain = _dev(torch, asc), _dev(torch, w["ascii"])
    d_off, d_qi = _dev(torch, offsets), _dev(torch, w["qinfo"])
    bad = w["qinfo"].copy()
    bad[0]["posEntry"] = len(w["peq"])
    d_bad = _dev(torch, bad)
    d_out = torch.full((len(w["peq"]) * 80,), 0x5A, dtype=torch.uint8, device="cuda")
    ctx = mg.Context(1)
    try:
        st = mg.lib.myersPackPEQAsync(ctx.h, d_asc.data_ptr(), asc.size, d_off.data_ptr(), d_qi.data_ptr(),
                                      len(lengths), d_out.data_ptr(), len(w["peq"]), stream)
        assert st == mg.SUCCESS
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().view(np.uint32).reshape(-1, 20)
        assert np.array_equal(got, expect)
        # the generator's own (unmodified) reads pack to its PEQ entries
        d_out.fill_(0)
        mg.lib.myersPackPEQAsync(ctx.h, d_asc_plain.data_ptr(), asc.size, d_off.data_ptr(), d_qi.data_ptr(),
                                 len(lengths), d_out.data_ptr(), len(w["peq"]), stream)
        torch.cuda.synchronize()
        assert np.array_equal(d_out.cpu().numpy().view(mg.QRY_ENTRY), w["peq"])
        assert ctx.flags() == 0
        # a read whose entries fall outside the buffer is skipped and flagged
        mg.lib.myersPackPEQAsync(ctx.h, d_asc.data_ptr(), asc.size, d_off.data_ptr(), d_bad.data_ptr(),
                                 len(lengths), d_out.data_ptr(), len(w["peq"]), stream)
        torch.cuda.synchronize()
        assert ctx.flags() & 4
        # so is one whose bytes would run past the ASCII buffer
        mg.lib.myersPackPEQAsync(ctx.h, d_asc.data_ptr(), asc.size - 1, d_off.data_ptr(), d_qi.data_ptr(),
                                 len(lengths), d_out.data_ptr(), len(w["peq"]), stream)
        torch.cuda.synchronize()
        assert ctx.flags() & 4
    finally:
        ctx.close()


def test_pack_reference_matches_reference_packer(mg, orc, cuda_ok):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    d = np.load(os.path.join(GOLDEN, "packers.npz"))
    fasta = d["fasta"].tobytes()
    seq = np.frombuffer(b"".join(l for l in fasta.split(b"\n") if l and not l.startswith(b">")), dtype=np.uint8)
    ref_file = d["ref_file"].tobytes()
    n_entries, size = np.frombuffer(ref_file[:8], dtype=np.uint32)
    ref_words = np.frombuffer(ref_file[8:], dtype=np.uint32)
    d_seq = _dev(torch, seq)
    d_words = torch.empty(int(n_entries) * 4, dtype=torch.uint8, device="cuda")
    st = mg.lib.myersPackReferenceAsync(d_seq.data_ptr(), len(seq), d_words.data_ptr(), int(n_entries), stream)
    assert st == mg.SUCCESS
    torch.cuda.synchronize()
    got = d_words.cpu().numpy().view(np.uint32)
    full = int(size) // 8
    assert np.array_equal(got[:full], ref_words[:full])
    mask = (1 << (4 * (int(size) % 8))) - 1
    assert (int(got[full]) & mask) == (int(ref_words[full]) & mask)
    assert np.array_equal(got, orc.pack_reference(seq.tobytes()))
    # a larger random sequence with every character class
    rng = np.random.default_rng(3)
    big = rng.choice(np.frombuffer(b"ACGTacgtNnXR-", dtype=np.uint8), size=1_000_003)
    nw = (len(big) + 7) // 8 + 2
    d_bigseq = _dev(torch, big)
    d_big = torch.empty(nw * 4, dtype=torch.uint8, device="cuda")
    mg.lib.myersPackReferenceAsync(d_bigseq.data_ptr(), len(big), d_big.data_ptr(), nw, stream)
    torch.cuda.synchronize()
    got = d_big.cpu().numpy().view(np.uint32)
    exp = orc.pack_reference(big.tobytes())
    assert np.array_equal(got[:len(exp)], exp) and (got[len(exp):] == 0x44444444).all()
