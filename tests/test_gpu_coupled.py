"""The coupled runs of UnitTest/TimeIntegration (couple/, less/): the IF-RK4
step without the per-step 2/3 truncation (couple.cu:179-215), the coupled
parameters (couple.cu:81-88: Re = Er = 0.1, Rf = 7.5e-5, lambda = 0.1,
Ra = 0.2, dt = 1e-3) and the smooth initial state (couple.cu:4-35).

Parity: the fused path against the reference's own build of that step
(golden ref_couple64.npz) and against the FP64 oracle; the dealias/ variant
(w truncated, r1 and r2 not, golden ref_dealiasw64.npz); the lowered linear
coefficient of less/ (L_Q = -k^2 + 0.995, less/Qsolver.cuh:38,50) against the
oracle. Long run: the observation recorded in couple/remark — over 40 time
units on 512^2 (L = 66 pi) the scalar order S = 2 |(r1, r2)| stays near 1
(<= 1.03 there) and the points with S > 1.02 self-suppress to fewer than
1.6% (4000 of 262144)."""
import math

import numpy as np
import pytest
import torch

import oracle as O
import qaf
from conftest import golden

pytestmark = pytest.mark.gpu

COUPLE = dict(re=0.1, er=0.1, rf=0.000075, lam=0.1, alpha=0.2, dt=0.001)


def dev(a, mesh):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype=mesh.complex_dtype)


def host(t):
    return t.detach().cpu().numpy().astype(np.complex128)


def couple_params(**kw):
    return qaf.Params(**{**COUPLE, "no_dealias": 1, **kw})


def couple_oracle_params(n, L, **kw):
    return O.params(n=n, L=L, **{**COUPLE, "no_dealias": 1, **kw})


def test_no_dealias_matches_reference_build_64(cuda):
    # the reference's coupled step (no dealias kernels), FP64, from its own
    # state 0; bar: relative L2 1e-12 per 10 steps, 1e-10 after 1000
    g = golden("ref_couple64.npz")
    m = qaf.Mesh(64, lx=8 * math.pi, dtype=qaf.F64)
    st = [dev(g[f"{k}_0"], m) for k in ("w", "r1", "r2")]
    prev = 0
    for s, bar in ((1, 1e-13), (10, 1e-12), (1000, 1e-10)):
        m.step(couple_params(), *st, nsteps=s - prev)
        prev = s
        for t, k in zip(st, ("w", "r1", "r2")):
            assert O.rel_l2(host(t), g[f"{k}_{s}"]) < bar, (s, k)
    # the modes outside the 2/3 mask stay populated: the step really skipped the truncation
    cut = O.tables(O.params(n=64, L=8 * math.pi))[3]
    assert np.abs(host(st[1]) * (1 - cut)).max() > 0


def test_w_only_truncation_matches_reference_build_64(cuda):
    # dealias/couple.cu:226-229: wnew truncated by the 2/3 mask, r1 and r2 not
    g = golden("ref_dealiasw64.npz")
    m = qaf.Mesh(64, lx=8 * math.pi, dtype=qaf.F64)
    st = [dev(g[f"{k}_0"], m) for k in ("w", "r1", "r2")]
    prev = 0
    for s, bar in ((1, 1e-13), (10, 1e-12), (200, 1e-11)):
        m.step(couple_params(no_dealias=2), *st, nsteps=s - prev)
        prev = s
        for t, k in zip(st, ("w", "r1", "r2")):
            assert O.rel_l2(host(t), g[f"{k}_{s}"]) < bar, (s, k)
    cut = O.tables(O.params(n=64, L=8 * math.pi))[3]
    assert np.abs(host(st[0]) * (1 - cut)).max() == 0          # w truncated
    assert np.abs(host(st[1]) * (1 - cut)).max() > 0           # r1 not


@pytest.mark.parametrize("dtype,steps,bar", [(qaf.F64, 20, 1e-12), (qaf.F32, 100, 1e-4)])
def test_no_dealias_against_oracle(cuda, dtype, steps, bar):
    n, L = 64, 8 * math.pi
    s0 = [O.fwd(a) for a in O.couple_init(3, n, L)]
    ref = O.step(couple_oracle_params(n, L), *s0, steps)
    m = qaf.Mesh(n, lx=L, dtype=dtype)
    st = [dev(a, m) for a in s0]
    m.load(*st)
    m.advance(couple_params(), nsteps=steps)
    m.store(*st)
    for t, o in zip(st, ref):
        assert O.rel_l2(host(t), o) < bar


def test_lowered_linear_coefficient_against_oracle(cuda):
    # less/: L_Q = -k^2 + 0.995 (with the friction solver's dealias kept here)
    n = 64
    s0 = O.initial_spectra(4, n)
    for no_dealias in (0, 1):
        ref = O.step(O.params(n=n, q_lin=0.995, no_dealias=no_dealias), *s0, 10)
        m = qaf.Mesh(n, lx=16 * math.pi, dtype=qaf.F64)
        st = [dev(a, m) for a in s0]
        m.step(qaf.Params(q_lin=0.995, no_dealias=no_dealias), *st, nsteps=10)
        for t, o in zip(st, ref):
            assert O.rel_l2(host(t), o) < 1e-13


def test_no_dealias_ensemble_equals_single_grids(cuda):
    sizes = [64, 128, 64]
    L = 8 * math.pi
    ens = qaf.Ensemble(sizes, couple_params(), [0.2, 0.25, 0.15], lx=L, dtype=qaf.F64)
    s0 = [[O.fwd(a) for a in O.couple_init(10 + k, n, L)] for k, n in enumerate(sizes)]
    for k, n in enumerate(sizes):
        m = ens.mesh(k)
        ens.load(k, *[dev(a, m) for a in s0[k]])
    ens.advance(15)
    for k, n in enumerate(sizes):
        m = qaf.Mesh(n, lx=L, dtype=qaf.F64)
        st = [dev(a, m) for a in s0[k]]
        m.step(couple_params(alpha=[0.2, 0.25, 0.15][k]), *st, nsteps=15)
        for a, b in zip(ens.store(k), st):
            assert O.rel_l2(host(a), host(b)) < 1e-13


@pytest.mark.parametrize("dtype", [qaf.F64, qaf.F32])
def test_coupled_smooth_run_keeps_order_bounded(cuda, dtype):
    # couple.cu as run by the reference: 512^2, L = 66 pi, 40 time units. The
    # smooth pattern (|k|^2 = 8) decays within one time unit, the order then
    # grows out of the noise and saturates near S = 1 from t ~ 20 on; the
    # share of points above 1.02 peaks at the onset and then self-suppresses.
    # Bounds (held for every noise seed measured, 0-2): max S <= 1.04 (the
    # remark saw <= 1.03 for its one rand() realisation), time-mean share of
    # S > 1.02 over t in [20, 40] below 1.6%.
    n, L = 512, 66 * math.pi
    m = qaf.Mesh(n, lx=L, dtype=dtype)
    m.load(*[m.fwd_trans(torch.from_numpy(a).to("cuda", m.real_dtype).contiguous())
             for a in O.couple_init(0, n, L)])
    p = couple_params()
    smax, late = 0.0, []
    for c in range(100):                       # S sampled every 0.4 time units
        m.advance(p, 400)
        _, r1, r2 = m.store()
        a, b = m.bwd_trans(r1), m.bwd_trans(r2)
        S = 2 * torch.sqrt(a * a + b * b)
        top = S.max().item()
        assert math.isfinite(top)
        smax = max(smax, top)
        if (c + 1) * 0.4 >= 20 - 1e-9:
            late.append((S > 1.02).double().mean().item())
    assert smax <= 1.04
    assert top > 1.0                           # the ordered state formed and persists
    assert sum(late) / len(late) < 0.016


@pytest.mark.parametrize("dtype,bar", [(qaf.F64, 1e-12), (qaf.F32, 1e-4)])
def test_q_only_run_against_oracle(cuda, dtype, bar):
    # decoupledQ/Qpure.cu:80-238: w frozen at its initial 0, Q alone
    # (lambda = 0.1, Re = 40, dt = 0.02, L = 2 pi, r1 = 0.9 (sin^2(x+y) - 1/2),
    # r2 = 0.9 sin(x+y) cos(x+y)). With the active stress off (Er = inf, so
    # 1/(Er Re) = 0, and Ra = 0) w stays exactly 0 and u = v = 0: that run.
    # (Its stage 4 calls integrate_func2D where integrate_func4D belongs,
    # Qpure.cu:212-213; the scheme here is the correct IF-RK4.)
    n, L = 64, 2 * math.pi
    x = np.arange(n) * L / n
    X, Y = np.meshgrid(x, x)
    s0 = [O.fwd(np.zeros((n, n))), O.fwd(0.9 * (np.sin(X + Y) ** 2 - 0.5)), O.fwd(0.9 * np.sin(X + Y) * np.cos(X + Y))]
    kw = dict(re=40.0, rf=0.0, lam=0.1, alpha=0.0, dt=0.02)
    ref = O.step(O.params(n=n, L=L, er=float("inf"), **kw), *s0, 50)
    m = qaf.Mesh(n, lx=L, dtype=dtype)
    st = [dev(a, m) for a in s0]
    m.step(qaf.Params(er=float("inf"), **kw), *st, nsteps=50)
    # w stays 0 up to roundoff: the row pass transforms two real fields as one
    # complex FFT, so w's physical values carry its partner's rounding (the
    # oracle, transforming each field alone, keeps it exactly 0)
    assert float(st[0].abs().max()) <= bar * float(st[1].abs().max())
    for t, o in zip(st[1:], ref[1:]):
        assert O.rel_l2(host(t), o) < bar
