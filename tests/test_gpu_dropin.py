"""Drop-in check: the reference's own sample driver (src-api/test.c,
unmodified) linked against libmyers_b200.so (oracle/_ref/sample0), run on a
packed reference and .gem.qry query files, its results file checked against
the oracle. This is the reference's call sequence end to end: initMyers, the
getters, sendMyersBuffer/receiveMyersBuffer from OpenMP threads, endMyers."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SAMPLE0 = os.path.join(ROOT, "oracle", "_ref", "sample0")


def write_ref(path, words, size):
    with open(path, "wb") as f:
        f.write(np.array([len(words), size], dtype=np.uint32).tobytes())
        f.write(np.asarray(words, dtype=np.uint32).tobytes())


def write_qry(path, w):
    # the layout src-api/test.c:30-66 reads: 5 u32 header, PEQ entries,
    # 16-byte candidates, query info
    with open(path, "wb") as f:
        f.write(np.array([int(w["qinfo"]["size"].sum()), len(w["peq"]), 0, len(w["qinfo"]), len(w["cands"])],
                         dtype=np.uint32).tobytes())
        f.write(w["peq"].tobytes())
        f.write(w["cands"].tobytes())
        f.write(w["qinfo"].tobytes())


@pytest.mark.skipif(not os.path.exists(SAMPLE0), reason="oracle/_ref/sample0 not built")
def test_reference_sample_driver(mg, orc, cuda_ok, tmp_path):
    ref_size = 3_000_001
    ref = mg.make_reference(ref_size, 31)
    fn_ref = str(tmp_path / "g.4bits.ref")
    write_ref(fn_ref, ref, ref_size)
    ws = [mg.make_workload(mg.workload_spec(k, scale=sc, ref_size=ref_size), ref) for k, sc in ((3, 0.002), (1, 0.05))]
    qfiles = []
    for i, w in enumerate(ws):
        q = str(tmp_path / f"q{i}.gem.qry")
        write_qry(q, w)
        qfiles.append(q)
    env = dict(os.environ, OMP_NUM_THREADS="2", MYERS_MEMORY_BUDGET=str(512 << 20))
    out = subprocess.run([SAMPLE0, "0.2", fn_ref, *qfiles], capture_output=True, text=True, env=env, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = open(qfiles[0] + ".gem-int.pad.gpu").read().split("\n")
    total = int(lines[0])
    rows = np.array([list(map(int, l.split())) for l in lines[1:1 + total]], dtype=np.int64)
    expect = np.concatenate([orc.verify(w["peq"], w["qinfo"], w["cands"], ref, ref_size, 0.2) for w in ws])
    assert total == len(expect)
    assert np.array_equal(rows[:, 0], np.arange(total))
    assert np.array_equal(rows[:, 1], expect["score"].astype(np.int64))
    assert np.array_equal(rows[:, 2], expect["column"].astype(np.int64))
