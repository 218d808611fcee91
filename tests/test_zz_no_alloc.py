"""The allocation-free step (qaf_step_noalloc).

For callers that cannot allocate device memory when they step (work captured
into a CUDA graph, plug-ins whose host owns the device memory, loops that must
not allocate once running), the library offers one entry point that keeps all
of its scratch in a fixed device array compiled into the library. This test
calls it through the C ABI and checks it against the ordinary qaf_step on the
same inputs, twice in a row (the array keeps the previous call's contents, so
the second call must not depend on them), and checks that grids larger than
the array's 128 x 128 limit are refused.

It lives in its own file, collected last, so that a run stopping at the first
failure has already run every other test."""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
import qaf

pytestmark = pytest.mark.gpu

L16 = 16 * np.pi


def _dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype=dtype)


def _noalloc(n, dtype, p, state, nsteps, status=None):
    cp = p.c()
    return qaf.lib().qaf_step_noalloc(n, L16, L16, dtype, ctypes.byref(cp), qaf.IFRK4,
                                      *[ctypes.c_void_p(t.data_ptr()) for t in state], nsteps,
                                      ctypes.c_void_p(status.data_ptr() if status is not None else None),
                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("n,dtype,tol", [(64, qaf.F64, 1e-12), (128, qaf.F64, 1e-12), (128, qaf.F32, 1e-5)])
def test_noalloc_step_matches_step_twice(cuda, n, dtype, tol):
    # qaf_step's tables come from long-double host arithmetic, the noalloc
    # path's from double on the device: equal to rounding, hence a tolerance
    m = qaf.Mesh(n, lx=L16, dtype=dtype)
    p = qaf.Params(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=1e-3)
    ref = [_dev(a, m.complex_dtype) for a in O.initial_spectra(0, n)]
    got = [t.clone() for t in ref]
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    for call in range(2):
        m.step(p, *ref, nsteps=3)
        assert _noalloc(n, dtype, p, got, 3, status) == qaf.OK, qaf.lib().qaf_last_error()
        torch.cuda.synchronize()
        assert int(status.item()) == 0, call
        for a, b in zip(got, ref):
            err = O.rel_l2(a.cpu().numpy().astype(np.complex128), b.cpu().numpy().astype(np.complex128))
            assert err < tol, (call, err)


def test_noalloc_status_reports_a_lost_copy(cuda):
    # the call cannot see a kernel failure when it returns (its work is only
    # queued), so the status word carries it: here a copy wait that runs out,
    # made on purpose by the library's test hook (an armed copy never issued)
    n = 64
    p = qaf.Params()
    s0 = [_dev(a, torch.complex128) for a in O.initial_spectra(2, n)]
    st = [t.clone() for t in s0]
    status = torch.zeros((1,), dtype=torch.int32, device="cuda")
    assert qaf.lib().qaf_test_lose_copy(0, 256) == qaf.OK
    assert _noalloc(n, qaf.F64, p, st, 1, status) == qaf.OK
    torch.cuda.synchronize()
    assert int(status.item()) & 2
    # the next call starts from cleared flags and is right again
    st = [t.clone() for t in s0]
    assert _noalloc(n, qaf.F64, p, st, 1, status) == qaf.OK
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    ref = O.step(O.params(n=n), *O.initial_spectra(2, n), 1)
    for a, b in zip(st, ref):
        assert O.rel_l2(a.cpu().numpy(), b) < 1e-12


def test_noalloc_takes_no_device_memory_and_refuses_large_grids(cuda):
    n = 64
    p = qaf.Params()
    st = [_dev(a, torch.complex128) for a in O.initial_spectra(1, n)]
    assert _noalloc(n, qaf.F64, p, st, 1) == qaf.OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert _noalloc(n, qaf.F64, p, st, 2) == qaf.OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    big = [torch.zeros((256, 129), dtype=torch.complex128, device="cuda") for _ in range(3)]
    assert _noalloc(256, qaf.F64, p, big, 1) == qaf.ERR_INVALID
    assert b"128" in qaf.lib().qaf_last_error()
