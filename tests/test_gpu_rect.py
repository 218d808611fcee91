"""Grids with nx != ny. The reference's Mesh takes any Nx, Ny, Lx, Ly
(Basic/Mesh.cuh:61-73); here the row kernels and row transforms run at the
nx-point length and the column ones at the ny-point length, each size a
power of two in [16, 1024] or 3 * 2^k in [48, 768]. Checked against the FP64
oracle (which takes nx, ny), against goldens of the reference's own build
(tests/golden, group "rect") and live against that build."""
import numpy as np
import pytest
import torch

import oracle as O
import qaf
from conftest import golden

pytestmark = pytest.mark.gpu

L16 = 16 * np.pi


def dev(a, mesh):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype=mesh.complex_dtype)


def devr(a, mesh):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype=mesh.real_dtype)


def host(t):
    a = t.detach().cpu().numpy()
    return a.astype(np.complex128) if np.iscomplexobj(a) else a.astype(np.float64)


RECT = [(64, 128), (128, 64), (96, 64), (64, 192), (1024, 256), (256, 768), (48, 16)]


@pytest.mark.parametrize("dtype", [qaf.F64, qaf.F32])
@pytest.mark.parametrize("nx,ny", RECT)
def test_rect_transforms_against_oracle(cuda, nx, ny, dtype):
    m = qaf.Mesh(nx, ny, lx=L16, ly=L16 * ny / nx, dtype=dtype)
    rng = np.random.default_rng(nx * 7 + ny)
    x = rng.standard_normal((ny, nx))
    tol = 1e-14 if dtype == qaf.F64 else 1e-6
    assert O.rel_l2(host(m.fwd_trans(devr(x, m))), O.fwd(x)) < tol
    S = rng.standard_normal((ny, nx // 2 + 1)) + 1j * rng.standard_normal((ny, nx // 2 + 1))
    assert O.rel_l2(host(m.bwd_trans(dev(S, m))), O.bwd(S, nx)) < tol
    assert O.rel_l2(host(m.bwd_trans(m.fwd_trans(devr(x, m)))), x) < tol


@pytest.mark.parametrize("dtype", [qaf.F64, qaf.F32])
@pytest.mark.parametrize("nx,ny", [(64, 128), (128, 64), (96, 64), (64, 48)])
def test_rect_nonlinear_against_oracle(cuda, nx, ny, dtype):
    Ly = L16 * ny / nx
    m = qaf.Mesh(nx, ny, lx=L16, ly=Ly, dtype=dtype)
    p = O.params(n=nx, ny=ny, L=L16, Ly=Ly)
    rng = np.random.default_rng(nx + 3 * ny)
    st = [(rng.standard_normal((ny, nx // 2 + 1)) + 1j * rng.standard_normal((ny, nx // 2 + 1))) * 1e-3 * (nx / 32)
          for _ in range(3)]
    st[0] *= 30
    ref = O.nonlinear(p, *st)
    got = m.nonlinear(qaf.Params(), *[dev(a, m) for a in st])
    tol = 2e-12 if dtype == qaf.F64 else 2e-5
    for g, o in zip(got, ref):
        assert O.rel_l2(host(g), o) < tol


@pytest.mark.parametrize("integ", [qaf.IFRK4, qaf.IFRK2, qaf.IFE])
@pytest.mark.parametrize("nx,ny", [(64, 128), (128, 64), (192, 64)])
def test_rect_steps_against_oracle_f64(cuda, nx, ny, integ):
    Ly = L16 * ny / nx
    m = qaf.Mesh(nx, ny, lx=L16, ly=Ly, dtype=qaf.F64)
    p = O.params(n=nx, ny=ny, L=L16, Ly=Ly)
    s0 = O.initial_spectra(8, nx, ny=ny)
    ref = O.step(p, *s0, 5, integ)
    st = [dev(a, m) for a in s0]
    m.step(qaf.Params(), *st, nsteps=5, integrator=integ)
    m.check_finite()
    for g, o in zip(st, ref):
        assert O.rel_l2(host(g), o) < 1e-13


def test_rect_f32_100_steps_against_oracle(cuda):
    nx, ny = 128, 64
    Ly = L16 * ny / nx
    m = qaf.Mesh(nx, ny, lx=L16, ly=Ly, dtype=qaf.F32)
    s0 = O.initial_spectra(9, nx, ny=ny)
    ref = O.step(O.params(n=nx, ny=ny, L=L16, Ly=Ly), *s0, 100)
    st = [dev(a, m) for a in s0]
    m.step(qaf.Params(), *st, nsteps=100)
    for g, o in zip(st, ref):
        assert O.rel_l2(host(g), o) < 1e-4


def test_rect_nonlinear_and_steps_match_reference_build(cuda):
    g = golden("ref_nl_rect96x64.npz")
    m = qaf.Mesh(96, 64, lx=L16, ly=L16 * 64 / 96, dtype=qaf.F64)
    out = m.nonlinear(qaf.Params(), dev(g["w"], m), dev(g["r1"], m), dev(g["r2"], m))
    for a, key in zip(out, ("wn", "r1n", "r2n")):
        assert O.rel_l2(host(a), g[key]) < 1e-13
    g = golden("ref_run64x128.npz")
    for dtype, bar in ((qaf.F64, 1e-13), (qaf.F32, 2e-5)):
        m = qaf.Mesh(64, 128, lx=L16, ly=2 * L16, dtype=dtype)
        st = [dev(g[f"{k}_0"], m) for k in ("w", "r1", "r2")]
        prev = 0
        for s in (1, 20):
            m.step(qaf.Params(), *st, nsteps=s - prev)
            prev = s
            for t, k in zip(st, ("w", "r1", "r2")):
                assert O.rel_l2(host(t), g[f"{k}_{s}"]) < bar, (dtype, s, k)


def test_rect_diagnostics_and_restart(cuda, tmp_path):
    nx, ny = 64, 128
    Ly = 2 * L16
    m = qaf.Mesh(nx, ny, lx=L16, ly=Ly, dtype=qaf.F64)
    p = O.params(n=nx, ny=ny, L=L16, Ly=Ly)
    s0 = O.initial_spectra(10, nx, ny=ny)
    ref = O.step(p, *s0, 3)
    m.load(*[dev(a, m) for a in s0])
    m.advance(qaf.Params(), 3)
    w, _, _ = m.store()
    e, z, spec = m.diagnostics(w, nshells=16)
    eo, zo, speco = O.diagnostics(p, ref[0], 16)
    assert abs(e - eo) <= 1e-12 * abs(eo) and abs(z - zo) <= 1e-12 * abs(zo)
    assert np.allclose(spec, speco, rtol=1e-10, atol=1e-300)
    path = str(tmp_path / "rect.qafstate")
    m.save(path, step=3)
    m2 = qaf.Mesh(nx, ny, lx=L16, ly=Ly, dtype=qaf.F64)
    assert m2.restore(path) == 3
    m.advance(qaf.Params(), 2)
    m2.advance(qaf.Params(), 2)
    for a, b in zip(m.store(), m2.store()):
        assert torch.equal(a, b)


@pytest.mark.parametrize("dtype,bar", [(qaf.F64, 1e-12), (qaf.F32, 1e-4)])
def test_rect_100_steps_match_reference_build_live(cuda, tmp_path, dtype, bar):
    # 256 x 512 (Lx = 16 pi, Ly = 32 pi), IF-RK4 dt = 1e-3, seed 18, 100 steps,
    # against the reference's build run live from the same initial spectra
    from test_gpu_parity import _harness
    nx, ny = 256, 512
    out = _harness(tmp_path, "run", "--n", str(nx), "--ny", str(ny), "--L", repr(L16), "--Ly", repr(2 * L16),
                   "--steps", "100", "--seed", "18", "--dumps", "0,100")
    s0 = O.read_dump(out + "_s0.bin")["fields"]
    ref = O.read_dump(out + "_s100.bin")["fields"]
    assert s0[0].shape == (ny, nx // 2 + 1)
    m = qaf.Mesh(nx, ny, lx=L16, ly=2 * L16, dtype=dtype)
    st = [dev(a, m) for a in s0]
    m.step(qaf.Params(), *st, nsteps=100)
    m.check_finite()
    for t, r, k in zip(st, ref, ("w", "r1", "r2")):
        err = O.rel_l2(host(t), r)
        assert err < bar, (k, err)
