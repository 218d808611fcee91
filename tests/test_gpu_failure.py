"""Failure detection and one-time set-up.

* The column kernel's copy waits are bounded: a copy that never lands makes
  the wait give up, the CTA stops at the next item boundary with nothing in
  flight, and the step reports QAF_ERR_CUDA. The failure is made on purpose
  and without any fault: the library's test hook arms one copy's barrier and
  never issues the copy, with a low poll limit so the wait gives up quickly.
  The next step on the same mesh must be right again.
* Kernel attributes and the persistent grid size are set up once per device,
  under a lock: first calls from several host threads at once, and a step on
  a second device after the first (skipped with one device).
"""
import subprocess
import sys
import textwrap
import time

import numpy as np
import pytest
import torch

import oracle as O
import qaf

pytestmark = pytest.mark.gpu

L16 = 16 * np.pi


def _dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype=dtype)


@pytest.mark.parametrize("dtype,slab", [(qaf.F64, 0), (qaf.F64, 2), (qaf.F32, 1)])
def test_lost_copy_is_reported_and_the_next_step_is_right(cuda, dtype, slab):
    n = 64
    m = qaf.Mesh(n, lx=L16, dtype=dtype)
    p = qaf.Params()
    s0 = O.initial_spectra(3, n)
    st = [_dev(a, m.complex_dtype) for a in s0]
    m.step(p, *st, nsteps=1)
    m.check_finite()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    assert qaf.lib().qaf_test_lose_copy(slab, 256) == qaf.OK
    m.step(p, *st, nsteps=1)
    with pytest.raises(qaf.QafError) as ei:
        m.check_finite()   # synchronises the stream
    elapsed = time.perf_counter() - t0
    assert ei.value.status == qaf.ERR_CUDA
    assert "timed out" in str(ei.value)
    # a given-up wait ends its CTA's work at the next item: no long stall
    assert elapsed < 2.0, elapsed
    # the flags were cleared by the check; a fresh step is right again
    st = [_dev(a, m.complex_dtype) for a in s0]
    m.step(p, *st, nsteps=2)
    m.check_finite()
    ref = O.step(O.params(n=n), *s0, 2)
    tol = 1e-12 if dtype == qaf.F64 else 1e-5
    for a, b in zip(st, ref):
        assert O.rel_l2(a.cpu().numpy().astype(np.complex128), b) < tol


def test_hook_rejects_bad_arguments():
    assert qaf.lib().qaf_test_lose_copy(-1, 10) == qaf.ERR_INVALID
    assert qaf.lib().qaf_test_lose_copy(0, 0) == qaf.ERR_INVALID


_THREADS = textwrap.dedent("""
    import sys, threading
    sys.path[:0] = {paths!r}
    import numpy as np, torch
    import oracle as O, qaf
    torch.cuda.set_device(0)
    n = 96 if qaf.supported(96, qaf.F32) else 32
    s0 = O.initial_spectra(4, n)
    p = qaf.Params()
    out, errs = [None] * 8, []
    go = threading.Barrier(8)
    def work(k):
        try:
            m = qaf.Mesh(n, lx=16 * np.pi, dtype=qaf.F32)
            st = [torch.from_numpy(a).to("cuda", dtype=torch.complex64) for a in s0]
            go.wait()
            m.step(p, *st, nsteps=2)
            torch.cuda.synchronize()
            out[k] = [t.cpu().numpy() for t in st]
        except Exception as e:
            errs.append(repr(e))
    ts = [threading.Thread(target=work, args=(k,)) for k in range(8)]
    for t in ts: t.start()
    for t in ts: t.join()
    assert not errs, errs
    for k in range(1, 8):
        for a, b in zip(out[k], out[0]):
            assert np.array_equal(a, b), k
    ref = O.step(O.params(n=n), *s0, 2)
    for a, b in zip(out[0], ref):
        assert O.rel_l2(a.astype(np.complex128), b) < 1e-5
    print("threads ok", n)
""")


def test_first_calls_from_many_threads_at_once(cuda):
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    paths = [os.path.join(root, "nature-control_b200"), os.path.join(root, "oracle")]
    r = subprocess.run([sys.executable, "-c", _THREADS.format(paths=paths)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "threads ok" in r.stdout


@pytest.mark.skipif(not torch.cuda.is_available() or torch.cuda.device_count() < 2, reason="needs two GPUs")
def test_step_on_a_second_device_after_the_first(cuda):
    n = 64
    s0 = O.initial_spectra(5, n)
    ref = O.step(O.params(n=n), *s0, 2)
    for dev in (0, 1):
        with torch.cuda.device(dev):
            m = qaf.Mesh(n, lx=L16, dtype=qaf.F64)
            st = [torch.from_numpy(a).to(f"cuda:{dev}") for a in s0]
            m.step(qaf.Params(), *st, nsteps=2)
            m.check_finite()
            for a, b in zip(st, ref):
                assert O.rel_l2(a.cpu().numpy(), b) < 1e-12
