"""Batched ensembles (qaf_ensemble_*) against the same instances stepped one by one.

Each instance of an ensemble is an independent run of friction.cu's loop with
its own grid size, activity and friction; the batched stepper must give every
instance what a single mesh gives it (same kernels, same tables), and the
single-mesh path is itself checked against the oracle in test_gpu_parity.py.
"""
import math

import pytest

pytestmark = pytest.mark.gpu

L = 16 * math.pi


def _rel(a, b):
    import torch
    return (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()


def _single(qaf, n, p, seed, nsteps, dtype):
    m = qaf.Mesh(n, n, L, L, dtype)
    w, r1, r2 = m.random_q(seed)
    m.load(w, r1, r2)
    m.advance(p, nsteps)
    out = m.store()
    return out, m.last_diagnostics()


def _params(qaf, alpha, rf):
    return qaf.Params(re=1.0, er=1.0, rf=rf, lam=0.1, alpha=alpha, dt=1e-3)


@pytest.mark.parametrize("dtype,tol", [("F64", 1e-13), ("F32", 2e-6)])
def test_mixed_sizes_match_single_meshes(cuda, dtype, tol):
    import qaf
    dt = getattr(qaf, dtype)
    sizes = [64, 128, 64, 256, 128, 64, 32]
    alpha = [0.5 + 0.25 * k for k in range(len(sizes))]
    rf = [0.02 * k for k in range(len(sizes))]
    seeds = [11 + 7 * k for k in range(len(sizes))]
    shared = _params(qaf, 1.0, 0.0)
    ens = qaf.Ensemble(sizes, shared, alpha, rf, lx=L, dtype=dt)
    ens.init_random(seeds)
    nsteps = 6
    ens.advance(nsteps)
    diags = ens.diagnostics()
    for k, n in enumerate(sizes):
        (w, r1, r2), (e1, z1) = _single(qaf, n, _params(qaf, alpha[k], rf[k]), seeds[k], nsteps, dt)
        ew, er1, er2 = ens.store(k)
        for got, want in ((ew, w), (er1, r1), (er2, r2)):
            assert _rel(got, want) <= tol, (k, n)
        # energy and enstrophy are quadratic in the state: about twice its
        # relative difference (the batch and single-grid column kernels may
        # differ in their shared/register twiddles and inlining, i.e. in FP32
        # rounding)
        e2, z2 = diags[k]
        dtol = 1e-9 if dtype == "F64" else 4 * tol
        assert abs(e2 - e1) <= dtol * abs(e1) and abs(z2 - z1) <= dtol * abs(z1), (k, e1, e2, z1, z2)


def test_many_instances_fp32(cuda):
    """A larger FP32 ensemble: every instance against its single-mesh run."""
    import qaf
    sizes = [64] * 24 + [128] * 12 + [256] * 4
    alpha = [0.2 + 0.05 * (k % 17) for k in range(len(sizes))]
    rf = [0.01 * (k % 5) for k in range(len(sizes))]
    seeds = list(range(100, 100 + len(sizes)))
    ens = qaf.Ensemble(sizes, _params(qaf, 1.0, 0.0), alpha, rf, lx=L, dtype=qaf.F32)
    ens.init_random(seeds)
    ens.advance(4)
    for k in (0, 5, 23, 24, 30, 35, 36, 39):
        (w, r1, r2), _ = _single(qaf, sizes[k], _params(qaf, alpha[k], rf[k]), seeds[k], 4, qaf.F32)
        ew, er1, er2 = ens.store(k)
        assert _rel(ew, w) <= 2e-6 and _rel(er1, r1) <= 2e-6 and _rel(er2, r2) <= 2e-6, k


def test_advance_in_pieces_equals_one_call(cuda):
    import qaf
    sizes = [64, 128]
    p = _params(qaf, 1.0, 0.1)
    a = qaf.Ensemble(sizes, p, [1.0, 0.7], lx=L, dtype=qaf.F64)
    b = qaf.Ensemble(sizes, p, [1.0, 0.7], lx=L, dtype=qaf.F64)
    a.init_random([3, 4])
    b.init_random([3, 4])
    a.advance(5)
    for _ in range(5):
        b.advance(1)
    for k in range(2):
        for x, y in zip(a.store(k), b.store(k)):
            assert _rel(x, y) == 0.0


def test_load_store_round_trip_and_reload(cuda):
    """store(load(x)) returns x's Hermitian-consistent content; a reload restarts from it."""
    import qaf
    import torch
    p = _params(qaf, 1.0, 0.0)
    ens = qaf.Ensemble([64, 64], p, [1.0, 1.0], lx=L, dtype=qaf.F64)
    m = ens.mesh(0)
    w, r1, r2 = m.random_q(5)
    ens.load(1, w, r1, r2)
    ens.load(0, w, r1, r2)
    ens.advance(3)
    a = ens.store(0)
    b = ens.store(1)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    ens.load(0, w, r1, r2)
    ens.advance(3)
    for x, y in zip(ens.store(0), a):
        assert torch.equal(x, y)


def test_invalid_arguments(cuda):
    import qaf
    p = _params(qaf, 1.0, 0.0)
    with pytest.raises(qaf.QafError):
        qaf.Ensemble([64, 100], p, [1.0, 1.0], lx=L)
    with pytest.raises(qaf.QafError):
        qaf.Ensemble([], p, [], lx=L)
    with pytest.raises(qaf.QafError):
        qaf.Ensemble([64], p, [float("nan")], lx=L)
    ens = qaf.Ensemble([64], p, [1.0], lx=L)
    with pytest.raises(qaf.QafError):
        qaf._check(qaf.lib().qaf_ensemble_advance(ens._h, -1, None))
    with pytest.raises((qaf.QafError, IndexError)):
        ens.store(1)


def test_set_controls_between_steps(cuda):
    """New activity/friction mid-run equals a single mesh stepped with the two parameter sets in turn."""
    import qaf
    sizes = [64, 128, 64]
    a0, r0 = [1.0, 0.6, 1.4], [0.05, 0.1, 0.2]
    a1, r1_ = [1.8, 0.9, 0.5], [0.3, 0.02, 0.1]
    seeds = [21, 22, 23]
    ens = qaf.Ensemble(sizes, _params(qaf, 1.0, 0.0), a0, r0, lx=L, dtype=qaf.F64)
    ens.init_random(seeds)
    ens.advance(2)
    ens.set_controls(a1, r1_)
    ens.advance(3)
    for k, n in enumerate(sizes):
        m = qaf.Mesh(n, n, L, L, qaf.F64)
        m.load(*m.random_q(seeds[k]))
        m.advance(_params(qaf, a0[k], r0[k]), 2)
        m.advance(_params(qaf, a1[k], r1_[k]), 3)
        for got, want in zip(ens.store(k), m.store()):
            assert _rel(got, want) <= 1e-13, k
