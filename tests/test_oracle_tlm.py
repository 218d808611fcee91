"""The oracle's tangent-linear model (the reference gradient of the GPU adjoint)
against central finite differences of the oracle's own forward map."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import oracle as O  # noqa: E402


def _case(n, seed, advect=1):
    p = O.params(n=n, L=16 * np.pi, dt=1e-2, alpha=1.0, rf=0.1, advect_omega=advect)
    s0 = O.initial_spectra(seed, n, lo=-0.5, hi=0.5)
    rng = np.random.default_rng(seed)
    shape = s0[0].shape
    d = [rng.standard_normal(shape) + 1j * rng.standard_normal(shape) for _ in range(3)]
    al = 1.0 + 0.1 * rng.standard_normal((n, n))
    dal = rng.standard_normal((n, n))
    return p, s0, d, al, dal


def _loss(p, s, al, T, Wn):
    z = [np.zeros_like(s[0])] * 3
    return O.step_tlm(p, *s, *z, T, Wn, alpha_field=al)[2]


@pytest.mark.parametrize("advect", [1, 0])
def test_tlm_matches_central_differences(advect):
    p, s0, d, al, dal = _case(16, 3, advect)
    T, Wn = 6, 3
    _, _, L, dL = O.step_tlm(p, *s0, *d, T, Wn, alpha_field=al, dalpha_field=dal)
    eps = 1e-5
    plus = _loss(p, [s0[f] + eps * d[f] for f in range(3)], al + eps * dal, T, Wn)
    minus = _loss(p, [s0[f] - eps * d[f] for f in range(3)], al - eps * dal, T, Wn)
    fd = (plus - minus) / (2 * eps)
    assert abs(fd - dL) <= 1e-8 * abs(dL)


def test_tlm_forward_part_is_oracle_step():
    p, s0, d, al, _ = _case(16, 5)
    st, _, _, _ = O.step_tlm(p, *s0, *d, 4, 0, alpha_field=al)
    ref = O.step(p, *s0, 4, alpha_field=al)
    for a, b in zip(st, ref):
        assert np.array_equal(a, b)


def test_tlm_is_linear_in_the_tangent():
    p, s0, d, al, dal = _case(16, 7)
    _, t1, _, l1 = O.step_tlm(p, *s0, *d, 3, 2, alpha_field=al, dalpha_field=dal)
    _, t2, _, l2 = O.step_tlm(p, *s0, *[2.5 * x for x in d], 3, 2, alpha_field=al, dalpha_field=2.5 * dal)
    assert abs(l2 - 2.5 * l1) <= 1e-12 * abs(l2)
    for a, b in zip(t1, t2):
        assert O.rel_l2(b, 2.5 * a) <= 1e-12
