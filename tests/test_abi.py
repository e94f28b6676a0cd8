"""CPU tests of the C ABI: the library loads, exports every symbol the header
declares, and its host-only logic (shape choice, argument checks) behaves."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def header_functions():
    text = open(os.path.join(ROOT, "include", "myers-interface.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text)
    skip = {"if", "sizeof", "defined", "for", "while", "return"}
    return sorted(set(n for n in names if n not in skip and not n.isupper()))


def test_exports_every_declared_symbol(mg):
    declared = header_functions()
    assert "initMyers" in declared and "myersVerifyAsync" in declared
    lib = ctypes.CDLL(mg.LIB_PATH)
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(mg.EXPORTED) == sorted(set(mg.EXPORTED))
    assert set(mg.EXPORTED) == set(declared)


def test_reference_getter_names(mg):
    # the reference API (src-api/myers-interface.h:31-46)
    for n in ("getPEQBuffer", "getCandidatesBuffer", "getPEQInfoBuffer", "getResultsBuffer", "getMaxPEQEntries",
              "getMaxCandidates", "getMaxQueries", "initMyers", "sendMyersBuffer", "receiveMyersBuffer", "endMyers"):
        assert hasattr(mg.lib, n)


def test_error_strings(mg):
    for st in range(13):
        assert mg.error_string(st).startswith("Myers")
    assert "Unknown" in mg.error_string(99)


def test_shape_choice(mg):
    """Whatever picks the shape (autotuner cache or cost model), it must hold
    the query, and the batched path must only pick shapes its persistent
    kernel carries (or, beyond 16384 bases, multi-lane shapes it launches
    plainly)."""
    for path in (mg.PATH_PLAIN, mg.PATH_BATCHED):
        for m in (1, 31, 32, 33, 100, 513, 1000, 1024, 1025, 3000, 10000, 16384, 20000, 32768):
            v, L, W = mg.shape_of(m, path)
            multi = bool(mg.lib.myersVariantIsMulti(v))
            assert W == mg.lib.myersVariantWords(v)
            assert 1 <= L <= 32 and L * W * 32 >= m
            assert multi or L == 1
            if path == mg.PATH_BATCHED and multi and m <= 16384:
                assert W <= 16
    with pytest.raises(mg.MyersError):
        mg.shape_of(0)
    with pytest.raises(mg.MyersError):
        mg.shape_of(mg.MAX_QUERY_BASES + 1)


def test_cost_model_without_cache():
    """With the autotuner's cache disabled, the built-in cost model gives one
    candidate per lane up to 1024 bases."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, 'myers-gpu_b200'); import myersgpu as mg;"
            "assert mg.lib.myersTunedShapes(0) == 0;"
            "print([mg.shape_of(m, p)[1:] for p in (0, 1) for m in (1, 100, 1000, 1024, 1025, 10000)])")
    env = dict(__import__('os').environ, MYERS_AUTOTUNE="0")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, check=True)
    shapes = eval(out.stdout)
    assert shapes[:4] == [(1, 1), (1, 4), (1, 32), (1, 32)] and shapes[6:10] == [(1, 1), (1, 4), (1, 32), (1, 32)]
    assert shapes[4][0] > 1 and shapes[5][0] > 1


def test_shape_override(mg):
    v0 = mg.shape_of(1000, mg.PATH_PLAIN)
    multi8 = [v for v, w, multi in mg.variants() if multi and w == 8][0]
    mg.set_shape_override(mg.PATH_PLAIN, 32, multi8, 4)
    assert mg.shape_of(1000, mg.PATH_PLAIN) == (multi8, 4, 8)
    with pytest.raises(mg.MyersError):
        mg.set_shape_override(mg.PATH_PLAIN, 32, multi8, 3)    # 3 x 8 words < 32
    mg.set_shape_override(mg.PATH_PLAIN, 32, -1)
    assert mg.shape_of(1000, mg.PATH_PLAIN) == v0


def test_bad_arguments_without_gpu(mg):
    arr = ctypes.POINTER(ctypes.c_void_p)()
    assert mg.lib.myersInit(ctypes.byref(arr), 0, b"x", 0, 0) == mg.E_INVALID_ARGUMENT
    assert mg.lib.myersSend(None, 0.2, 0, 0, 0) == mg.E_INVALID_ARGUMENT
    assert mg.lib.myersReceive(None) == mg.E_INVALID_ARGUMENT
    assert mg.lib.myersVerifyAsync(None, None, None, 0, None, 0, None, 0, 0.2, 0, 0, None, None) == \
        mg.E_INVALID_ARGUMENT
    assert mg.lib.getMaxCandidates(None) == 0
