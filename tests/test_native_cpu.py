"""CPU tests of the native code that need no GPU: the team-FFT index maps
(emulated on the host thread by thread) and the C ABI library's exports."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_team_fft_emulation(tmp_path):
    exe = tmp_path / "fft_emulation"
    src = os.path.join(ROOT, "tests", "native", "fft_emulation.cu")
    subprocess.run(["nvcc", "-std=c++17", "-O1", "-Wno-deprecated-gpu-targets", "-o", str(exe), src], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASS" in r.stdout


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "qaf.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(qaf_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    import qaf
    if not os.path.exists(qaf.LIB_PATH):
        import sys
        sys.path.insert(0, os.path.join(ROOT, "nature-control_b200"))
        import build
        build.build(verbose=False)
    return qaf.lib()


def test_library_exports_every_declared_symbol(lib):
    import qaf
    syms = header_symbols()
    assert sorted(qaf.EXPORTS) == syms
    for s in syms:
        assert hasattr(lib, s), s


def test_library_host_only_calls(lib):
    import qaf
    assert "sm_100a" in qaf.version()
    assert qaf.supported(1024, qaf.F32) and qaf.supported(128, qaf.F64)
    # powers of two in [16, 1024] and 3 * 2^k in [48, 768] (the reference's 768 = 512 * 3 / 2)
    for n in (48, 96, 192, 384, 768):
        assert qaf.supported(n, qaf.F32) and qaf.supported(n, qaf.F64), n
    for n in (2048, 1536, 24, 12, 80, 100):
        assert not qaf.supported(n, qaf.F32), n
    h = ctypes.c_void_p()
    bad = qaf.MeshDesc(7, 8, 1.0, 1.0, qaf.F64)
    assert lib.qaf_mesh_create(ctypes.byref(bad), ctypes.byref(h)) == qaf.ERR_INVALID
    assert b"even" in lib.qaf_last_error()
    bad = qaf.MeshDesc(8, 8, -1.0, 1.0, qaf.F64)
    assert lib.qaf_mesh_create(ctypes.byref(bad), ctypes.byref(h)) == qaf.ERR_INVALID
    good = qaf.MeshDesc(32, 32, 1.0, 1.0, qaf.F32)
    assert lib.qaf_mesh_create(ctypes.byref(good), ctypes.byref(h)) == qaf.OK
    pb, sb = ctypes.c_size_t(), ctypes.c_size_t()
    assert lib.qaf_mesh_sizes(h, ctypes.byref(pb), ctypes.byref(sb)) == qaf.OK
    assert pb.value == 32 * 32 * 4 and sb.value == 17 * 32 * 8
    assert lib.qaf_state_advance(h, None, qaf.IFRK4, 1, None) == qaf.ERR_INVALID
    assert lib.qaf_mesh_destroy(h) == qaf.OK
