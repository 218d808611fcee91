"""The discrete adjoint (qaf_adjoint_*) against the oracle's tangent-linear model
and against central finite differences of the GPU forward map.

For J = L + <gT, s_T> (L the mean enstrophy of the last `window` states, gT a
fixed weight on the final state) the adjoint's gradient g must satisfy
<g, d> = dJ/de along every direction d of the initial spectra and of the
activity field; the oracle's TLM gives dJ/de in FP64 on the CPU.
"""
import math
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import oracle as O  # noqa: E402

L = 16 * math.pi


def _setup(n, seed, dt=1e-2, advect=1, amp=0.5, no_dealias=0):
    p = O.params(n=n, L=L, dt=dt, alpha=1.0, rf=0.1, advect_omega=advect, no_dealias=no_dealias)
    s0 = O.initial_spectra(seed, n, lo=-amp, hi=amp)
    rng = np.random.default_rng(seed + 1000)
    alpha = 1.0 + 0.1 * rng.standard_normal((n, n))
    gT = [rng.standard_normal(s0[0].shape) + 1j * rng.standard_normal(s0[0].shape) for _ in range(3)]
    gT = [1e-3 * g for g in gT]
    return p, s0, alpha, gT, rng


def _qaf_params(qaf, dt, advect=1, no_dealias=0):
    return qaf.Params(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=dt, q_lin=1.0, advect_omega=advect,
                      no_dealias=no_dealias)


def _dev(x, cdt):
    import torch
    return torch.as_tensor(np.ascontiguousarray(x)).to(device="cuda", dtype=cdt)


def _gpu_grad(qaf, n, dtype, s0, alpha, gT, nsteps, K, window, dt, advect=1, const_alpha=False, no_dealias=0):
    import torch
    mesh = qaf.Mesh(n, n, L, L, dtype)
    cdt, rdt = mesh.complex_dtype, mesh.real_dtype
    p = _qaf_params(qaf, dt, advect, no_dealias)
    if not const_alpha:
        p.alpha_field = _dev(alpha, rdt)
    adj = qaf.Adjoint(mesh, nsteps, K, window)
    loss, final = adj.forward(p, *[_dev(s, cdt) for s in s0])
    g = adj.backward([_dev(x, cdt) for x in gT] if gT is not None else None, grad_loss=1.0)
    torch.cuda.synchronize()
    return loss, final, [x.cpu().numpy() for x in g[:3]], g[3].cpu().numpy()


def _dot(g, d):
    return float(sum(np.sum(a.real * b.real + a.imag * b.imag) for a, b in zip(g, d)))


def _tlm_dJ(p, s0, alpha, d, dal, gT, nsteps, window):
    _, dsT, _, dL = O.step_tlm(p, *s0, *d, nsteps, window, alpha_field=alpha, dalpha_field=dal)
    return dL + (_dot(gT, dsT) if gT is not None else 0.0)


@pytest.mark.parametrize("advect,no_dealias", [(1, 0), (0, 0), (1, 1), (1, 2)])
def test_gradient_matches_oracle_tlm_fp64(cuda, advect, no_dealias):
    import qaf
    n, T, K, Wn, dt = 32, 12, 5, 4, 1e-2
    p, s0, alpha, gT, rng = _setup(n, 3, dt, advect, no_dealias=no_dealias)
    loss, _, g, ga = _gpu_grad(qaf, n, qaf.F64, s0, alpha, gT, T, K, Wn, dt, advect, no_dealias=no_dealias)
    _, _, L_ref, _ = O.step_tlm(p, *s0, *[np.zeros_like(s0[0])] * 3, T, Wn, alpha_field=alpha)
    assert abs(loss - L_ref) <= 1e-10 * abs(L_ref)
    for trial in range(3):
        d = [rng.standard_normal(s0[0].shape) + 1j * rng.standard_normal(s0[0].shape) for _ in range(3)]
        dal = rng.standard_normal((n, n))
        want = _tlm_dJ(p, s0, alpha, d, dal, gT, T, Wn)
        got = _dot(g, d) + float(np.sum(ga * dal))
        assert abs(got - want) <= 1e-9 * abs(want), (trial, got, want)


@pytest.mark.parametrize("n", [16, 64, 128, 256, 512])
def test_gradient_matches_oracle_tlm_all_sizes(cuda, n):
    """Every launch shape of the adjoint kernels (field-parallel up to 256^2, column-sequential above)."""
    import qaf
    T, K, Wn, dt = 3, 2, 2, 5e-3
    p, s0, alpha, gT, rng = _setup(n, 21, dt)
    _, _, g, ga = _gpu_grad(qaf, n, qaf.F64, s0, alpha, gT, T, K, Wn, dt)
    d = [rng.standard_normal(s0[0].shape) + 1j * rng.standard_normal(s0[0].shape) for _ in range(3)]
    dal = rng.standard_normal((n, n))
    want = _tlm_dJ(p, s0, alpha, d, dal, gT, T, Wn)
    got = _dot(g, d) + float(np.sum(ga * dal))
    assert abs(got - want) <= 1e-9 * abs(want), (got, want)


def test_gradient_separate_directions_fp64(cuda):
    """State-only and activity-only directions, loss-only and final-state-only objectives."""
    import qaf
    n, T, K, Wn, dt = 32, 8, 3, 3, 1e-2
    p, s0, alpha, gT, rng = _setup(n, 5, dt)
    z = [np.zeros_like(s0[0])] * 3
    d = [rng.standard_normal(s0[0].shape) + 1j * rng.standard_normal(s0[0].shape) for _ in range(3)]
    dal = rng.standard_normal((n, n))
    # loss only
    _, _, g, ga = _gpu_grad(qaf, n, qaf.F64, s0, alpha, None, T, K, Wn, dt)
    want = _tlm_dJ(p, s0, alpha, d, None, None, T, Wn)
    assert abs(_dot(g, d) - want) <= 1e-9 * abs(want)
    want = _tlm_dJ(p, s0, alpha, z, dal, None, T, Wn)
    assert abs(float(np.sum(ga * dal)) - want) <= 1e-9 * abs(want)
    # final state only (no loss window)
    _, _, g, ga = _gpu_grad(qaf, n, qaf.F64, s0, alpha, gT, T, K, 0, dt)
    want = _tlm_dJ(p, s0, alpha, d, dal, gT, T, 0)
    got = _dot(g, d) + float(np.sum(ga * dal))
    assert abs(got - want) <= 1e-9 * abs(want)


def test_constant_activity_gradient_is_field_sum(cuda):
    import qaf
    n, T, K, Wn, dt = 32, 6, 4, 3, 1e-2
    p, s0, _, _, _ = _setup(n, 7, dt)
    ones = np.ones((n, n))
    _, _, _, ga = _gpu_grad(qaf, n, qaf.F64, s0, ones, None, T, K, Wn, dt, const_alpha=True)
    want = _tlm_dJ(p, s0, ones, [np.zeros_like(s0[0])] * 3, ones, None, T, Wn)
    assert abs(float(ga.sum()) - want) <= 1e-9 * abs(want)


def test_checkpoint_interval_does_not_change_gradients(cuda):
    import qaf
    n, T, Wn, dt = 32, 9, 4, 1e-2
    _, s0, alpha, gT, _ = _setup(n, 9, dt)
    ref = _gpu_grad(qaf, n, qaf.F64, s0, alpha, gT, T, T, Wn, dt)
    for K in (1, 4):
        got = _gpu_grad(qaf, n, qaf.F64, s0, alpha, gT, T, K, Wn, dt)
        assert abs(got[0] - ref[0]) <= 1e-14 * abs(ref[0])   # enstrophy sums use atomics
        for a, b in zip(got[2], ref[2]):
            assert np.array_equal(a, b)
        assert np.array_equal(got[3], ref[3])


def test_central_differences_16_directions_fp64(cuda):
    """Central differences of the GPU forward (FP64) along 16 random directions."""
    import qaf
    import torch
    n, T, K, Wn, dt = 64, 20, 8, 5, 5e-3
    _, s0, alpha, _, rng = _setup(n, 11, dt)
    _, _, g, ga = _gpu_grad(qaf, n, qaf.F64, s0, alpha, None, T, K, Wn, dt)
    mesh = qaf.Mesh(n, n, L, L, qaf.F64)
    adj = qaf.Adjoint(mesh, T, K, Wn)

    def loss_at(s, a):
        p = _qaf_params(qaf, dt)
        p.alpha_field = _dev(a, torch.float64)
        return adj.forward(p, *[_dev(x, torch.complex128) for x in s], final_state=False)[0]

    scale = max(np.abs(s0[1]).max(), 1e-30)
    for k in range(16):
        d = [rng.standard_normal(s0[0].shape) + 1j * rng.standard_normal(s0[0].shape) for _ in range(3)]
        d = [x * scale for x in d]
        dal = rng.standard_normal((n, n))
        eps = 1e-5
        lp = loss_at([s0[f] + eps * d[f] for f in range(3)], alpha + eps * dal)
        lm = loss_at([s0[f] - eps * d[f] for f in range(3)], alpha - eps * dal)
        fd = (lp - lm) / (2 * eps)
        ad = _dot(g, d) + float(np.sum(ga * dal))
        assert abs(fd - ad) <= 1e-6 * abs(ad) + 1e-14, (k, fd, ad)


def test_fp32_gradient_close_to_fp64(cuda):
    import qaf
    n, T, K, Wn, dt = 64, 16, 8, 4, 5e-3
    _, s0, alpha, gT, _ = _setup(n, 13, dt)
    l64, _, g64, ga64 = _gpu_grad(qaf, n, qaf.F64, s0, alpha, gT, T, K, Wn, dt)
    l32, _, g32, ga32 = _gpu_grad(qaf, n, qaf.F32, s0, alpha, gT, T, K, Wn, dt)
    assert abs(l32 - l64) <= 1e-4 * abs(l64)
    for a, b in zip(g32, g64):
        assert O.rel_l2(a, b) <= 1e-3
    assert O.rel_l2(ga32, ga64) <= 1e-3


def test_autograd_wrapper_matches_raw_api(cuda):
    import torch

    import qaf
    import qaf.autograd as QA
    n, T, K, Wn, dt = 32, 6, 4, 3, 1e-2
    _, s0, alpha, gT, _ = _setup(n, 15, dt)
    mesh = qaf.Mesh(n, n, L, L, qaf.F64)
    leaves = [_dev(s, torch.complex128).requires_grad_() for s in s0]
    al = _dev(alpha, torch.float64).requires_grad_()
    loss, wT, r1T, r2T = QA.rollout(mesh, _qaf_params(qaf, dt), *leaves, al, nsteps=T, checkpoint_every=K,
                                    loss_window=Wn)
    gTt = [_dev(x, torch.complex128) for x in gT]
    # J = loss + <gT, s_T> with the real inner product
    J = loss + sum((torch.conj(g) * s).real.sum() for g, s in zip(gTt, (wT, r1T, r2T)))
    J.backward()
    _, _, g, ga = _gpu_grad(qaf, n, qaf.F64, s0, alpha, gT, T, K, Wn, dt)
    for leaf, want in zip(leaves, g):
        assert O.rel_l2(leaf.grad.cpu().numpy(), want) <= 1e-12
    assert O.rel_l2(al.grad.cpu().numpy(), ga) <= 1e-12


def test_fwd_trans_adjoint(cuda):
    """<F x, a> = <x, F^T a> for the FwdTrans autograd wrapper."""
    import torch

    import qaf
    import qaf.autograd as QA
    n = 32
    mesh = qaf.Mesh(n, n, L, L, qaf.F64)
    rng = np.random.default_rng(3)
    x = _dev(rng.standard_normal((n, n)), torch.float64).requires_grad_()
    a = _dev(rng.standard_normal((n, n // 2 + 1)) + 1j * rng.standard_normal((n, n // 2 + 1)), torch.complex128)
    y = QA.fwd_trans(mesh, x)
    (torch.conj(a) * y).real.sum().backward()
    lhs = float((torch.conj(a) * y.detach()).real.sum())
    rhs = float((x.detach() * x.grad).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_invalid_arguments(cuda):
    import qaf
    mesh = qaf.Mesh(32, 32, L, L, qaf.F64)
    for args in ((0, 4, 0), (4, 0, 0), (4, 4, 5), (4, 4, -1)):
        with pytest.raises(qaf.QafError):
            qaf.Adjoint(mesh, *args)
    adj = qaf.Adjoint(mesh, 4, 2, 2)
    with pytest.raises(qaf.QafError):
        adj.backward()          # no forward yet
