import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "myers-gpu_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a)")


@pytest.fixture(scope="session")
def mg():
    import myersgpu
    return myersgpu


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle


@pytest.fixture(scope="session")
def golden_verify(mg):
    d = np.load(os.path.join(GOLDEN, "verify.npz"))
    peq = np.ascontiguousarray(d["peq"]).view(mg.QRY_ENTRY).ravel()
    qinfo = np.ascontiguousarray(d["qinfo"]).view(mg.QINFO).ravel()
    cands = np.zeros(len(d["cand_query"]), dtype=mg.CAND)
    cands["query"] = d["cand_query"]
    cands["position"] = d["cand_pos"]
    res_a = np.ascontiguousarray(d["res_aligned"]).view(mg.RES).ravel()
    res_e = np.ascontiguousarray(d["res_exact"]).view(mg.RES).ravel()
    return dict(ref=d["ref_words"], ref_size=int(d["ref_size"]), distance=float(d["distance"]), peq=peq,
                qinfo=qinfo, cands=cands, group=d["group"], res_aligned=res_a, res_exact=res_e,
                exact_mask=d["exact_mask"])


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
