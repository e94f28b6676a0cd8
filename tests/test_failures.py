"""Host-side failure paths of the C ABI, on the CPU: each error here is
detected before any device work, so no GPU is needed. The reference's
convention (src-api/myersGPU.c:24-47) is to print the error and end the
process; the status-returning entry points report the same error as a code
instead (MYERS_E_OPENING_FILE, MYERS_E_READING_FILE, ...)."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

from conftest import ROOT


def _ref_file(path, words, size, truncate_to=None):
    data = np.array([len(words), size], dtype=np.uint32).tobytes() + np.asarray(words, dtype=np.uint32).tobytes()
    with open(path, "wb") as f:
        f.write(data if truncate_to is None else data[:truncate_to])
    return path


def test_reference_load_missing_file(mg, tmp_path):
    h = C.c_void_p()
    assert mg.lib.myersReferenceLoad(C.byref(h), str(tmp_path / "absent.4bits.ref").encode()) == mg.E_OPENING_FILE
    assert not h


def test_reference_load_truncated_or_inconsistent_file(mg, tmp_path):
    words = np.full(100, 0x01234012, dtype=np.uint32)
    cases = {
        "empty": _ref_file(tmp_path / "empty.ref", words, 800, truncate_to=0),
        "header cut": _ref_file(tmp_path / "hdr.ref", words, 800, truncate_to=6),
        "words cut": _ref_file(tmp_path / "short.ref", words, 800, truncate_to=8 + 4 * 40),
        "more bases than words hold": _ref_file(tmp_path / "bases.ref", words, 801),
    }
    for what, path in cases.items():
        h = C.c_void_p()
        st = mg.lib.myersReferenceLoad(C.byref(h), str(path).encode())
        assert st == mg.E_READING_FILE, (what, mg.error_string(st))
        assert not h


def test_init_reports_file_errors(mg, tmp_path):
    arr = C.POINTER(C.c_void_p)()
    assert mg.lib.myersInit(C.byref(arr), 2, str(tmp_path / "absent.ref").encode(), 1000, 10) == mg.E_OPENING_FILE
    short = _ref_file(tmp_path / "short.ref", np.zeros(64, dtype=np.uint32), 512, truncate_to=100)
    assert mg.lib.myersInit(C.byref(arr), 2, str(short).encode(), 1000, 10) == mg.E_READING_FILE
    assert not arr


def test_fatal_convention_of_the_reference_calls(tmp_path):
    """initMyers, like the reference's, prints the error and exits with
    EXIT_FAILURE (no return to the caller)."""
    code = ("import ctypes as C, sys; sys.path.insert(0, 'myers-gpu_b200'); import myersgpu as mg;"
            "arr = C.POINTER(C.c_void_p)();"
            f"mg.lib.initMyers(C.byref(arr), 1, {str(tmp_path / 'absent.ref')!r}.encode(), 1000, 10);"
            "print('returned')")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert out.returncode == 1
    assert "returned" not in out.stdout
    assert "Myers - Error: opening file in initMyers" in out.stderr


def test_no_alloc_argument_checks(mg):
    p = C.c_void_p(256)
    # a reference size that would overflow the word count, and a batch beyond the static scratch
    assert mg.lib.myersVerifyNoAllocAsync(p, (1 << 62), 8, p, 1, p, 1, p, 1, 0.2, mg.WINDOW_ALIGNED, 0, 0, p,
                                          None) == mg.E_INVALID_ARGUMENT
    assert mg.lib.myersVerifyNoAllocAsync(p, 1, 9, p, 1, p, 1, p, 1, 0.2, mg.WINDOW_ALIGNED, 0, 0, p,
                                          None) == mg.E_INVALID_ARGUMENT
    assert mg.lib.myersVerifyNoAllocAsync(p, 1, 8, p, 1, p, 1, p, mg.NOALLOC_MAX_CANDIDATES + 1, 0.2,
                                          mg.WINDOW_ALIGNED, 0, 0, p, None) == mg.E_CAPACITY
    assert mg.lib.myersVerifyNoAllocAsync(p, 1, 8, p, 1, p, 1, p, 1, float("nan"), mg.WINDOW_ALIGNED, 0, 0, p,
                                          None) == mg.E_INVALID_ARGUMENT
    assert mg.lib.myersVerifyNoAllocAsync(p, 1, 8, p, 1, p, 1, p, 1, 0.2, 7, 0, 0, p, None) == mg.E_INVALID_ARGUMENT
    # an empty batch is a no-op
    assert mg.lib.myersVerifyNoAllocAsync(None, 0, 0, None, 0, None, 0, None, 0, 0.2, mg.WINDOW_ALIGNED, 0, 0, None,
                                          None) == mg.SUCCESS


def test_server_and_traceback_argument_checks(mg):
    h = C.c_void_p()
    assert mg.lib.myersServerCreate(C.byref(h), None, None) == mg.E_INVALID_ARGUMENT
    assert mg.lib.myersServerSubmit(None, None, 100, None, 1, None) == mg.E_INVALID_ARGUMENT
    assert mg.lib.myersTracebackCreate(None, 1, 1) == mg.E_INVALID_ARGUMENT
