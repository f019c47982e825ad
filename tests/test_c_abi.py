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


def _exports(path, demangle=False):
    args = ["nm", "-D", "--defined-only"] + (["-C"] if demangle else []) + [path]
    out = subprocess.run(args, capture_output=True, text=True, check=True)
    return sorted(line.split(None, 2)[-1] for line in out.stdout.splitlines() if line.strip())


def test_drop_in_library_exports_exactly_the_reference_abi():
    """libsemper_c.so, the drop-in for the reference's C library, exports the
    eleven symbols of tests/c/abi_symbols.txt and nothing else (the
    reference's CI diffs its export list against that file)."""
    sb.lib()
    assert _exports(sb.C_LIB_PATH) == sorted(sb.C_SYMBOLS)


def test_full_library_exports_exactly_the_declared_symbols():
    lib = sb.lib()
    exported = _exports(sb.LIB_PATH)
    c_names = [e for e in exported if not e.startswith("_Z")]
    c_api = _declared("semper_c.h", r"\b(semper_[a-z_]+)\s*\(")
    dic_api = _declared("semper_dic_cuda.h", r"\b(dic_cuda_[a-z0-9_]+)\s*\(")
    ext_api = _declared("semper_b200_ext.h", r"\b(semper_b200_[a-z0-9_]+)\s*\(")
    assert c_api == sorted(sb.C_SYMBOLS)
    assert ext_api == sorted(sb.EXT_SYMBOLS)
    assert c_names == sorted(c_api + dic_api + ext_api)
    for name in c_names:
        assert hasattr(lib, name)
    # the C++ API of include/semper/*.hpp, and nothing else of C++
    cxx = [e for e in _exports(sb.LIB_PATH, demangle=True) if "::" in e]
    assert cxx and all(e.startswith("Semper::pipeline::") for e in cxx)
    names = {e.split("(")[0] for e in cxx}
    for want in ["Semper::pipeline::run_full_field", "Semper::pipeline::ReferenceCache::set_from_gray",
                 "Semper::pipeline::ReferenceCache::reset", "Semper::pipeline::IncrementalSession::init",
                 "Semper::pipeline::IncrementalSession::process_frame", "Semper::pipeline::request_cancel",
                 "Semper::pipeline::clear_cancel", "Semper::pipeline::cancel_requested",
                 "Semper::pipeline::detail::global_cancel_token"]:
        assert want in names, want


def test_cxx_api_headers_build_and_link(tmp_path):
    """A caller of the reference's C++ API builds and links against the
    library (no OpenCV here: the gray-view overloads only)."""
    src = tmp_path / "caller.cpp"
    src.write_text(
        "#include <semper/incremental.hpp>\n#include <semper/pipeline.hpp>\n"
        "using namespace Semper::pipeline;\n"
        "int main() {\n"
        "  ReferenceCache cache; FullFieldParams p; float out[8]; float met[24];\n"
        "  CancelToken tok; { CancelScope scope(tok); }\n"
        "  int rc = run_full_field(cache, GrayView(), GrayView(), p, out, 8, met, 24);\n"
        "  rc += run_full_field(cache, GrayView(), GrayView(), p, out, 8, met, 24, tok);\n"
        "  IncrementalSession s; IncrementalParams ip; ip.field = p;\n"
        "  rc += s.init(GrayView(), GrayView(), ip) + s.max_points() + s.frames_processed();\n"
        "  request_cancel(); clear_cancel(); return rc + (cancel_requested() ? 1 : 0) + kSeedFailed;\n"
        "}\n")
    lib_dir = os.path.dirname(sb.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-I", os.path.join(REPO, "include"), str(src), "-o",
                    str(tmp_path / "caller"), "-L", lib_dir, "-lsemper_b200", f"-Wl,-rpath,{lib_dir}"], check=True)


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
