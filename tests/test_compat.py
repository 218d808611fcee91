"""include/qaf_compat.cuh: a driver written against the reference's names
(Mesh, Field, FwdTrans, curr_func, wnonl_func, integrate_func0D..4D, dealias,
SpecSet, IF::IFRK2, IF::IFE, ...) compiles against libqaf and gives what the
fused path gives."""
import json
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "native", "compat_driver.cu")
OUT = os.path.join(HERE, "native", "_build")
LIBDIR = os.path.join(ROOT, "nature-control_b200", "qaf")


def _build(fp32: bool) -> str:
    os.makedirs(OUT, exist_ok=True)
    exe = os.path.join(OUT, "compat_driver_f32" if fp32 else "compat_driver")
    if not os.path.exists(os.path.join(LIBDIR, "libqaf.so")):
        pytest.skip("libqaf.so is not built")
    if os.path.exists(exe) and os.path.getmtime(exe) >= max(os.path.getmtime(SRC), os.path.getmtime(
            os.path.join(ROOT, "include", "qaf_compat.cuh")), os.path.getmtime(os.path.join(LIBDIR, "libqaf.so"))):
        return exe
    cmd = ["nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-I", os.path.join(ROOT, "include"),
           "-o", exe, SRC, "-L", LIBDIR, "-lqaf", "-Xlinker", "-rpath", "-Xlinker", LIBDIR]
    if fp32:
        cmd.insert(1, "-DQAF_COMPAT_FP32")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return exe


@pytest.mark.parametrize("fp32", [False, True])
def test_reference_style_driver_compiles(fp32):
    assert os.path.exists(_build(fp32))


@pytest.mark.gpu
@pytest.mark.parametrize("integ,n,steps", [("rk4", 64, 20), ("rk2", 64, 10), ("ife", 32, 10), ("rk4", 128, 5)])
def test_reference_style_loop_matches_fused_step_fp64(cuda, integ, n, steps):
    r = subprocess.run([_build(False), str(n), str(steps), integ], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("rel_w", "rel_r1", "rel_r2"):
        assert out[k] <= 1e-12, out


@pytest.mark.gpu
@pytest.mark.parametrize("fp32,bar", [(False, 1e-12), (True, 1e-5)])
def test_friction_driver_settings_768(cuda, fp32, bar):
    # friction.cu's own grid and parameters: Nx = 512 * 3 / 2 = 768, Lx = 66 pi,
    # Re = Er = 0.1, Rf = 0.00075, alpha = 0.2, dt = 0.002
    r = subprocess.run([_build(fp32), "768", "10", "rk4", "friction"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("rel_w", "rel_r1", "rel_r2"):
        assert out[k] <= bar, out


@pytest.mark.gpu
def test_reference_style_loop_matches_fused_step_fp32(cuda):
    r = subprocess.run([_build(True), "64", "20", "rk4"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("rel_w", "rel_r1", "rel_r2"):
        assert out[k] <= 1e-5, out
