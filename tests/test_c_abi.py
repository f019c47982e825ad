"""The drop-in boundary without a GPU: the library loads, exports exactly the
declared entry points, and the frozen layouts hold (tests/c/contract.c:20-40
and tests/c/abi_symbols.txt of the reference)."""
import ctypes
import os
import re
import subprocess

import pytest

import semper_b200 as sb

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header, pattern):
    text = open(os.path.join(REPO, "include", header)).read()
    return sorted(set(re.findall(pattern, text)))


def test_library_exports_exactly_the_declared_symbols():
    lib = sb.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", sb.LIB_PATH], capture_output=True, text=True, check=True)
    exported = sorted(line.split()[-1] for line in out.stdout.splitlines() if line.strip())
    c_api = _declared("semper_c.h", r"\b(semper_[a-z_]+)\s*\(")
    dic_api = _declared("semper_dic_cuda.h", r"\b(dic_cuda_[a-z0-9_]+)\s*\(")
    ext_api = _declared("semper_b200_ext.h", r"\b(semper_b200_[a-z0-9_]+)\s*\(")
    assert c_api == sorted(sb.C_SYMBOLS)
    assert ext_api == sorted(sb.EXT_SYMBOLS)
    assert exported == sorted(c_api + dic_api + ext_api)
    for name in exported:
        assert hasattr(lib, name)


def test_reference_abi_symbol_list():
    # tests/c/abi_symbols.txt of the reference lists these eleven, sorted.
    assert sorted(sb.C_SYMBOLS) == [
        "semper_cancel", "semper_create", "semper_destroy", "semper_incremental_cancel",
        "semper_incremental_create", "semper_incremental_destroy", "semper_incremental_init",
        "semper_incremental_process", "semper_run", "semper_set_reference", "semper_version"]


def test_frozen_layouts():
    assert ctypes.sizeof(sb.SemperParams) == 32
    offs = [getattr(sb.SemperParams, f).offset for f, _ in sb.SemperParams._fields_]
    assert offs == [0, 4, 8, 12, 16, 20, 24, 28]
    assert ctypes.sizeof(sb.IncrementalInfo) == 24
    assert sb.TASK_DT.itemsize == 40 and sb.RESULT_DT.itemsize == 48


def test_version_and_null_handles():
    lib = sb.lib()
    assert re.fullmatch(r"\d+\.\d+\.\d+", sb.version())
    prm = sb.params((0, 0, 64, 64), 8, 15, 15)
    buf = (ctypes.c_float * 8)()
    assert lib.semper_run(None, None, 0, None, 0, ctypes.byref(prm), buf, 8, None, 0, sb.PROGRESS_CB(), None) == -3
    assert lib.semper_set_reference(None, None, 0, None, 0, 64, 64) == -3
    assert lib.semper_incremental_init(None, None, 0, None, 0, 64, 64, ctypes.byref(prm), 0) == -3
    assert lib.semper_incremental_process(None, None, 0, buf, 8, None, 0, None, sb.PROGRESS_CB(), None) == -3
    lib.semper_cancel(None)
    lib.semper_incremental_cancel(None)
    lib.semper_destroy(None)
    lib.semper_incremental_destroy(None)


def test_no_device_is_an_error_not_a_fallback():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError):
        sb.Engine()
