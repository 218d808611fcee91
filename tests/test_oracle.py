"""CPU tests of the FP64 host oracle: pinned to the golden vectors produced by
the reference's own CUDA build (tests/golden/, see make_golden.py) and to the
analytic known-answer tests of the reference's unit tests."""
import json
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, golden
from golden.make_golden import kat_fields

L16 = 16 * np.pi


def test_seeded_generator_numpy_equals_c_header():
    for seed in (0, 1, 5, 123456789):
        a = O.random_q_init(seed, 24)
        b = O.random_q_init_c(seed, 24)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    w, r1, r2 = O.random_q_init(0, 64)
    assert np.all(w == 0) and r1.min() >= -0.01 and r1.max() < 0.01 and abs(r2.mean()) < 1e-3


def test_couple_init_numpy_equals_c_header():
    # the smooth initial state of UnitTest/TimeIntegration/couple/couple.cu:4-35
    for seed, n, L in ((0, 32, 8 * np.pi), (9, 64, 8 * np.pi), (2, 48, 66 * np.pi)):
        a = O.couple_init(seed, n, L)
        b = O.couple_init_c(seed, n, L)
        for x, y in zip(a, b):
            assert np.abs(x - y).max() <= 1e-16
    w, r1, r2 = O.couple_init(0, 64, 8 * np.pi)
    S = 2 * np.sqrt(r1 * r1 + r2 * r2)
    assert np.all(w == 0) and 0.19 < S.min() and S.max() < 0.21


@pytest.mark.parametrize("n", [8, 12, 16, 30, 64, 128, 768])
def test_transforms_match_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n))
    X = O.fwd(x)
    assert O.rel_l2(X, np.fft.rfft2(x)) < 1e-15 * 8
    assert O.rel_l2(O.bwd(X), x) < 1e-15 * 8


@pytest.mark.parametrize("n", [8, 32, 128])
def test_bwd_sees_only_hermitian_part_of_edge_columns(n):
    # cuFFT Z2D, as called by the reference's BwdTrans, was measured to use only
    # the Hermitian part of the kx = 0 and kx = n/2 columns; numpy's irfft2 does the same
    rng = np.random.default_rng(n + 1)
    X = rng.standard_normal((n, n // 2 + 1)) + 1j * rng.standard_normal((n, n // 2 + 1))
    assert O.rel_l2(O.bwd(X), np.fft.irfft2(X, s=(n, n))) < 1e-14
    assert O.rel_l2(O.bwd(X), O.bwd(O.hermitian_part(X))) < 1e-14


def test_mesh_tables_and_mask():
    p = O.params(n=128)
    kx, ky, k2, cut = O.tables(p)
    dk = 2 * np.pi / L16
    assert np.allclose(kx[0, :], dk * np.arange(65))
    assert np.allclose(ky[:, 0], dk * np.r_[np.arange(65), np.arange(-63, 0)])
    assert np.allclose(k2, kx ** 2 + ky ** 2)
    # asymmetric 2/3 mask of cutoff_func: kx <= 42, ky in [-41, 42]
    keep_i = np.where(cut[0, :] > 0)[0]
    keep_j = np.where(cut[:, 0] > 0)[0]
    assert keep_i.max() == 42 and keep_i.min() == 0 and len(keep_i) == 43
    kyk = np.round(ky[keep_j, 0] / dk).astype(int)
    assert kyk.min() == -41 and kyk.max() == 42


def test_field_operator_identities():
    # UnitTest/Fld/Fld.cu:21-63: phi = sin(x+y) on L = 66 pi (wave number 33 dk = 1,
    # so the grid needs more than 66 points)
    n, L = 128, 66 * np.pi
    p = O.params(n=n, L=L)
    x = np.arange(n) * L / n
    X, Y = np.meshgrid(x, x)
    ph = O.fwd(np.sin(X + Y))
    k = 2 * np.pi / L
    # with L = 66 pi the modes sin(x+y) live at wave number 33 dk = 1
    assert np.allclose(O.bwd(O.laplacian(p, ph)), -2 * np.sin(X + Y) * (33 * k) ** 2, atol=1e-12)
    assert np.allclose(O.bwd(O.xderiv(p, ph)), np.cos(X + Y) * 33 * k, atol=1e-12)
    assert np.allclose(-O.bwd(O.yderiv(p, ph)), -np.cos(X + Y) * 33 * k, atol=1e-12)
    u, v = O.vel(p, O.laplacian(p, ph))
    assert np.allclose(O.bwd(u), -np.cos(X + Y), atol=1e-12)
    assert np.allclose(O.bwd(v), np.cos(X + Y), atol=1e-12)


@pytest.mark.parametrize("k", range(5))
def test_nonlinear_known_answers(k):
    # UnitTest/Nonlinear/nlterms{k}.cu: N = 128 (the closed forms are band
    # limited below 64), L = 2 pi, Re = Er = 0.1, Ra = 0.2, lambda = 0.1.
    p = O.params(n=128, L=2 * np.pi, re=0.1, er=0.1, alpha=0.2, lam=0.1, rf=0.000075)
    w, r1, r2, e0, e1, e2 = kat_fields(k)
    nl = O.nonlinear(p, O.fwd(w), O.fwd(r1), O.fwd(r2))
    dev = [np.abs(O.bwd(a) - b).max() / np.abs(b).max() for a, b in zip(nl, (e0, e1, e2))]
    # N_w sums terms ~100x larger than itself (1/(Er Re) = 100): cancellation
    assert dev[0] < 2e-7
    # nlterms3's closed form for N_r1 carries the rounded literal 0.0342282
    assert dev[1] < (2e-8 if k == 3 else 1e-12)
    assert dev[2] < 1e-12
    ref = json.load(open(os.path.join(GOLDEN, "ref_kat_summary.json")))[f"kat{k}"]["max_rel_dev_from_closed_form"]
    # the reference's own build sits at the same distance from the closed forms
    for a, b in zip(dev, ref):
        assert a < 10 * b + 1e-13


@pytest.mark.parametrize("n", [32, 64, 96, 192])
def test_nonlinear_matches_reference_build(n):
    g = golden(f"ref_nl_rand{n}.npz")
    p = O.params(n=n)
    out = O.nonlinear(p, g["w"], g["r1"], g["r2"])
    for a, b in zip(out, (g["wn"], g["r1n"], g["r2n"])):
        # raw spectra, non-Hermitian kx = 0 / n/2 columns included
        assert O.rel_l2(a, b) < 5e-15


def test_initial_state_matches_reference_build():
    g = golden("ref_run32.npz")
    w, r1, r2 = O.initial_spectra(5, 32)
    for a, name in zip((w, r1, r2), ("w_0", "r1_0", "r2_0")):
        assert O.rel_l2(O.hermitian_part(a), O.hermitian_part(g[name])) < 1e-15


def test_rk4_steps_match_reference_build_32():
    g = golden("ref_run32.npz")
    p = O.params(n=32)
    st = (g["w_0"], g["r1_0"], g["r2_0"])
    prev = 0
    for s in (1, 2, 10, 20):
        st = O.step(p, *st, s - prev)
        prev = s
        for a, name in zip(st, ("w", "r1", "r2")):
            assert O.rel_l2(a, g[f"{name}_{s}"]) < 1e-14, (s, name)


@pytest.mark.parametrize("n", [96, 192])
def test_rk4_steps_match_reference_build_3x2k(n):
    # 3 * 2^k grids: the oracle's mixed-radix transform against the reference's
    # build (cuFFT), including its initial FwdTrans of the seeded fields
    g = golden(f"ref_run{n}.npz")
    p = O.params(n=n)
    w, r1, r2 = O.initial_spectra(14 if n == 96 else 15, n)
    for a, name in zip((w, r1, r2), ("w_0", "r1_0", "r2_0")):
        assert O.rel_l2(O.hermitian_part(a), O.hermitian_part(g[name])) < 1e-15
    st = (g["w_0"], g["r1_0"], g["r2_0"])
    prev = 0
    for s in (1, 20):
        st = O.step(p, *st, s - prev)
        prev = s
        for a, name in zip(st, ("w", "r1", "r2")):
            assert O.rel_l2(a, g[f"{name}_{s}"]) < 1e-14, (s, name)


def test_rect_grids_match_reference_build():
    # nx != ny, Lx != Ly: one nonlinear evaluation at 96 x 64 and 20 IF-RK4
    # steps at 64 x 128, each against the reference's build (Mesh(Nx, Ny, Lx, Ly))
    g = golden("ref_nl_rect96x64.npz")
    p = O.params(n=96, ny=64, L=16 * np.pi, Ly=16 * np.pi * 64 / 96)
    out = O.nonlinear(p, g["w"], g["r1"], g["r2"])
    for a, b in zip(out, (g["wn"], g["r1n"], g["r2n"])):
        assert O.rel_l2(a, b) < 5e-15
    g = golden("ref_run64x128.npz")
    p = O.params(n=64, ny=128, L=16 * np.pi, Ly=32 * np.pi)
    w, r1, r2 = O.initial_spectra(17, 64, ny=128)
    for a, name in zip((w, r1, r2), ("w_0", "r1_0", "r2_0")):
        assert O.rel_l2(O.hermitian_part(a), O.hermitian_part(g[name])) < 1e-15
    st = (g["w_0"], g["r1_0"], g["r2_0"])
    prev = 0
    for s in (1, 20):
        st = O.step(p, *st, s - prev)
        prev = s
        for a, name in zip(st, ("w", "r1", "r2")):
            assert O.rel_l2(a, g[f"{name}_{s}"]) < 1e-14, (s, name)


def test_rk4_100_steps_match_reference_build_64():
    g = golden("ref_run64_s100.npz")
    p = O.params(n=64)
    st = O.step(p, *O.initial_spectra(0, 64), 100)
    for a, name in zip(st, ("w", "r1", "r2")):
        assert O.rel_l2(a, g[name]) < 1e-13


def test_taylor_green_decay_is_exact():
    # UnitTest/TimeIntegration/Taylor: w0 = -2 cos x cos y, Q = 0, Re = 40, Rf = 0,
    # dt = 0.02; the nonlinear terms vanish, so w(t) = w0 exp(-2 t / Re)
    n = 32
    p = O.params(n=n, L=2 * np.pi, re=40, er=40, rf=0, alpha=0.2, dt=0.02)
    x = np.arange(n) * 2 * np.pi / n
    X, Y = np.meshgrid(x, x)
    w0 = -2 * np.cos(X) * np.cos(Y)
    z = np.zeros_like(w0)
    st = O.step(p, O.fwd(w0), O.fwd(z), O.fwd(z), 50)
    assert np.allclose(O.bwd(st[0]), w0 * np.exp(-2 * 50 * 0.02 / 40), atol=1e-13)
    assert np.abs(O.bwd(st[1])).max() < 1e-14


def smooth_state(n):
    """An analytic state with r1^2 + r2^2 > 0 everywhere (so S is smooth) whose
    spectrum stays far below the 2/3 cutoff over short times."""
    x = np.arange(n) * 2 * np.pi / n
    X, Y = np.meshgrid(x, x)
    w = 0.5 * np.sin(X) * np.cos(Y)
    r1 = 0.3 + 0.1 * np.cos(X + Y)
    r2 = 0.1 * np.sin(X) + 0.05 * np.cos(2 * Y)
    return O.fwd(w), O.fwd(r1), O.fwd(r2)


def test_integrators_converge_at_their_order():
    # The reference dealiases the state once per step (friction.cu:253-255), not
    # each product; for states with energy at the cutoff that adds an O(dt)
    # consistency error for every integrator, so the order is checked on a
    # smooth, resolved state.
    n = 32
    s0 = smooth_state(n)
    T = 0.2
    mk = lambda dt: O.params(n=n, L=2 * np.pi, re=1.0, er=1.0, rf=0.1, dt=dt)
    ref = O.step(mk(T / 512), *s0, 512, O.IFRK4)
    for integ, order in ((O.IFE, 1), (O.IFRK2, 2), (O.IFRK4, 4)):
        errs = []
        for m in (8, 16):
            st = O.step(mk(T / m), *s0, m, integ)
            errs.append(O.rel_l2(st[1], ref[1]))
        rate = np.log2(errs[0] / errs[1])
        assert rate > order - 0.3, (integ, errs, rate)


def test_diagnostics_definitions():
    n, L = 32, 16 * np.pi
    p = O.params(n=n, L=L)
    w = O.dealias(p, O.fwd(O.random_q_init(3, n, -1, 1)[1]))
    e, z, spec = O.diagnostics(p, w, nshells=24)
    wp = O.bwd(w)
    assert np.isclose(z, 0.5 * np.mean(wp ** 2), rtol=1e-12)
    u, v = O.vel(p, w)
    up, vp = O.bwd(u), O.bwd(v)
    assert np.isclose(e, 0.5 * np.mean(up ** 2 + vp ** 2), rtol=1e-12)
    # the shells tile the stored half plane, each point counted once (EnergySpec.cu:81-96);
    # the post-processor starts from a physical snapshot, i.e. from the Hermitian part
    # of the kx = 0 column, which the asymmetric 2/3 mask leaves non-Hermitian at ky = N/3
    dk = 2 * np.pi / L
    kx, ky, k2, _ = O.tables(p)
    uh, vh = O.vel(p, O.hermitian_part(w))
    m2 = np.abs(uh) ** 2 + np.abs(vh) ** 2
    k = 0.0
    for s in range(24):
        k += dk
    assert np.isclose(spec.sum() * 2 * dk * n ** 4, m2[k2 < k * k].sum(), rtol=1e-12)


COUPLE = dict(re=0.1, er=0.1, rf=0.000075, lam=0.1, alpha=0.2, dt=0.001)


def test_step_without_dealias_is_step_before_truncation():
    # one step: the friction step's state = the coupled step's state times the 2/3 mask
    p = O.params(n=32)
    s0 = O.initial_spectra(1, 32)
    a = O.step(p, *s0, 1)
    b = O.step(O.params(n=32, no_dealias=1), *s0, 1)
    cut = O.tables(p)[3]
    for x, y in zip(a, b):
        assert np.array_equal(x, y * cut)
        assert np.abs(y * (1 - cut)).max() > 0


def test_coupled_step_matches_reference_build_64():
    # the reference's coupled step (couple.cu:179-215: no dealias kernels) with
    # its parameters, from the reference build's own state 0
    g = golden("ref_couple64.npz")
    p = O.params(n=64, L=8 * np.pi, no_dealias=1, **COUPLE)
    st = (g["w_0"], g["r1_0"], g["r2_0"])
    prev = 0
    for s in (1, 10):
        st = O.step(p, *st, s - prev)
        prev = s
        for a, name in zip(st, ("w", "r1", "r2")):
            assert O.rel_l2(a, g[f"{name}_{s}"]) < 1e-14, (s, name)
    w0, r10, r20 = (O.fwd(a) for a in O.couple_init(9, 64, 8 * np.pi))
    assert O.rel_l2(O.hermitian_part(r10), O.hermitian_part(g["r1_0"])) < 1e-15


def test_w_only_truncation_step():
    # dealias/couple.cu:226-229 truncates wnew only: one step gives the friction
    # step's w and the coupled step's r1, r2
    s0 = O.initial_spectra(1, 32)
    full = O.step(O.params(n=32), *s0, 1)
    none = O.step(O.params(n=32, no_dealias=1), *s0, 1)
    w_only = O.step(O.params(n=32, no_dealias=2), *s0, 1)
    assert np.array_equal(w_only[0], full[0])
    assert np.array_equal(w_only[1], none[1]) and np.array_equal(w_only[2], none[2])


def test_w_only_truncation_matches_reference_build_64():
    g = golden("ref_dealiasw64.npz")
    p = O.params(n=64, L=8 * np.pi, no_dealias=2, **COUPLE)
    st = (g["w_0"], g["r1_0"], g["r2_0"])
    prev = 0
    for s in (1, 10):
        st = O.step(p, *st, s - prev)
        prev = s
        for a, name in zip(st, ("w", "r1", "r2")):
            assert O.rel_l2(a, g[f"{name}_{s}"]) < 1e-14, (s, name)
