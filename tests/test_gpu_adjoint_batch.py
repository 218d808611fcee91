"""The batched adjoint (qaf_adjoint_batch_*) against the single-instance adjoint,
instance by instance: same losses, same gradients (the single-instance adjoint is
itself pinned to the oracle's tangent-linear model in test_gpu_adjoint.py)."""
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


def _params(qaf, dt):
    return qaf.Params(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=dt, q_lin=1.0, advect_omega=1)


def _case(n, ninst, seed):
    rng = np.random.default_rng(seed)
    states = [O.initial_spectra(seed + k, n, lo=-0.5, hi=0.5) for k in range(ninst)]
    alphas = [1.0 + 0.1 * rng.standard_normal((n, n)) for _ in range(ninst)]
    gT = [[1e-3 * (rng.standard_normal(states[0][0].shape) + 1j * rng.standard_normal(states[0][0].shape))
           for _ in range(3)] for _ in range(ninst)]
    return states, alphas, gT


def _dev(x, dt):
    import torch
    return torch.as_tensor(np.ascontiguousarray(x)).to(device="cuda", dtype=dt)


@pytest.mark.parametrize("dtype_name,tol", [("F64", 1e-11), ("F32", 2e-5)])
@pytest.mark.parametrize("const_alpha", [False, True])
def test_batch_matches_single_instances(cuda, dtype_name, tol, const_alpha):
    import torch

    import qaf
    dtype = getattr(qaf, dtype_name)
    n, ninst, T, K, Wn, dt = 32, 3, 6, 4, 2, 1e-2
    states, alphas, gT = _case(n, ninst, 40)
    glosses = [1.0, 0.5, 2.0]
    batch = qaf.AdjointBatch(ninst, n, _params(qaf, dt), T, K, Wn, lx=L, dtype=dtype)
    cdt, rdt = batch.mesh.complex_dtype, batch.mesh.real_dtype
    s0 = [_dev(np.stack([states[k][f] for k in range(ninst)]), cdt) for f in range(3)]
    al = None if const_alpha else _dev(np.stack(alphas), rdt)
    losses, final = batch.forward(*s0, alpha=al)
    gTb = [_dev(np.stack([gT[k][f] for k in range(ninst)]), cdt) for f in range(3)]
    gw, g1, g2, ga = batch.backward(gTb, glosses)
    torch.cuda.synchronize()
    for k in range(ninst):
        mesh = qaf.Mesh(n, n, L, L, dtype)
        p = _params(qaf, dt)
        if not const_alpha:
            p.alpha_field = _dev(alphas[k], rdt)
        adj = qaf.Adjoint(mesh, T, K, Wn)
        loss, fin = adj.forward(p, *[_dev(states[k][f], cdt) for f in range(3)])
        g = adj.backward([_dev(gT[k][f], cdt) for f in range(3)], grad_loss=glosses[k])
        torch.cuda.synchronize()
        assert abs(losses[k] - loss) <= tol * abs(loss), k
        for f in range(3):
            assert O.rel_l2(final[f][k].cpu().numpy(), fin[f].cpu().numpy()) <= tol, (k, f)
            assert O.rel_l2((gw, g1, g2)[f][k].cpu().numpy(), g[f].cpu().numpy()) <= tol * 10, (k, f)
        assert O.rel_l2(ga[k].cpu().numpy(), g[3].cpu().numpy()) <= tol * 10, k


def test_batch_invalid_arguments(cuda):
    import qaf
    p = _params(qaf, 1e-3)
    with pytest.raises(qaf.QafError):
        qaf.AdjointBatch(2, 512, p, 4, 2, 1, lx=L)
    with pytest.raises(qaf.QafError):
        qaf.AdjointBatch(0, 64, p, 4, 2, 1, lx=L)
    b = qaf.AdjointBatch(2, 32, p, 4, 2, 1, lx=L)
    with pytest.raises(qaf.QafError):
        b.backward()
