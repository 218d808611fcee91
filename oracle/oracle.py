"""Python face of the FP64 host oracle (oracle/qaf_oracle.cpp).

TEST INFRASTRUCTURE ONLY. The tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use it as the checker; the product never imports
it. Besides the ctypes bindings it holds:

* ``random_q_init`` — a numpy restatement of include/qaf_init.h (SplitMix64),
  bit-identical to the C generator used by the library and the driver around
  the reference's CUDA build;
* ``read_dump`` — the reader of that driver's binary dumps
  ("QAFDUMP1" header, fields in the reference's layouts).
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

IFE, IFRK2, IFRK4 = 0, 1, 2


class Params(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double),
        ("re", ctypes.c_double), ("er", ctypes.c_double), ("rf", ctypes.c_double), ("lam", ctypes.c_double),
        ("alpha", ctypes.c_double), ("dt", ctypes.c_double), ("q_lin", ctypes.c_double),
        ("advect_omega", ctypes.c_int), ("emulate_symmetry", ctypes.c_int), ("no_dealias", ctypes.c_int),
    ]


def params(n=128, L=16 * np.pi, re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=1e-3, q_lin=1.0,
           advect_omega=1, emulate_symmetry=1, ny=None, Ly=None, no_dealias=0) -> Params:
    return Params(n, ny or n, L, Ly or L, re, er, rf, lam, alpha, dt, q_lin, advect_omega, emulate_symmetry,
                  no_dealias)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        pp = ctypes.POINTER(Params)
        L.oracle_fwd.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
        L.oracle_bwd.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
        L.oracle_bwd_mutating.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
        L.oracle_tables.argtypes = [pp, dp, dp, dp, dp]
        for name in ("oracle_xderiv", "oracle_yderiv", "oracle_laplacian"):
            getattr(L, name).argtypes = [pp, dp, dp]
        L.oracle_vel.argtypes = [pp, dp, dp, dp]
        L.oracle_step_tlm.argtypes = [pp, dp, dp, dp, dp, dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, dp, dp]
        L.oracle_dealias.argtypes = [pp, dp]
        L.oracle_if_tables.argtypes = [pp, ctypes.c_int, ctypes.c_double, dp, dp]
        L.oracle_nonlinear.argtypes = [pp, dp, dp, dp, dp, dp, dp, dp, dp]
        L.oracle_step.argtypes = [pp, ctypes.c_int, dp, dp, dp, dp, ctypes.c_int]
        L.oracle_diagnostics.argtypes = [pp, dp, dp, dp, dp, ctypes.c_int]
        L.oracle_random_q_init.argtypes = [ctypes.c_ulonglong, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, dp, dp, dp]
        L.oracle_random_q_init.restype = None
        L.oracle_couple_init.argtypes = [ctypes.c_ulonglong, ctypes.c_int, ctypes.c_double, ctypes.c_double, dp, dp, dp]
        L.oracle_couple_init.restype = None
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _spec(a):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a


def _check(rc):
    if rc != 0:
        raise ValueError(f"oracle call failed with status {rc}")


def spec_shape(p: Params):
    return (p.ny, p.nx // 2 + 1)


def fwd(phys):
    phys = np.ascontiguousarray(phys, dtype=np.float64)
    ny, nx = phys.shape
    out = np.empty((ny, nx // 2 + 1), np.complex128)
    _check(lib().oracle_fwd(nx, ny, _p(phys), _p(out)))
    return out


def bwd(spec, nx=None):
    spec = _spec(spec)
    ny, nxh = spec.shape
    nx = nx or 2 * (nxh - 1)
    out = np.empty((ny, nx), np.float64)
    _check(lib().oracle_bwd(nx, ny, _p(spec), _p(out)))
    return out


def tables(p: Params):
    shp = spec_shape(p)
    kx, ky, k2, cut = (np.empty(shp) for _ in range(4))
    _check(lib().oracle_tables(ctypes.byref(p), _p(kx), _p(ky), _p(k2), _p(cut)))
    return kx, ky, k2, cut


def _unary(name, p, a):
    a = _spec(a)
    out = np.empty_like(a)
    _check(getattr(lib(), name)(ctypes.byref(p), _p(a), _p(out)))
    return out


def xderiv(p, a):
    return _unary("oracle_xderiv", p, a)


def yderiv(p, a):
    return _unary("oracle_yderiv", p, a)


def laplacian(p, a):
    return _unary("oracle_laplacian", p, a)


def vel(p, w):
    w = _spec(w)
    u, v = np.empty_like(w), np.empty_like(w)
    _check(lib().oracle_vel(ctypes.byref(p), _p(w), _p(u), _p(v)))
    return u, v


def dealias(p, a):
    a = _spec(a).copy()
    _check(lib().oracle_dealias(ctypes.byref(p), _p(a)))
    return a


def if_tables(p, which, dt):
    shp = spec_shape(p)
    IF, IFh = np.empty(shp), np.empty(shp)
    _check(lib().oracle_if_tables(ctypes.byref(p), which, dt, _p(IF), _p(IFh)))
    return IF, IFh


def nonlinear(p, w, r1, r2, alpha_field=None, want_phys=False):
    w, r1, r2 = _spec(w), _spec(r1), _spec(r2)
    wn, r1n, r2n = np.empty_like(w), np.empty_like(w), np.empty_like(w)
    phys = np.empty((9, p.ny, p.nx)) if want_phys else None
    af = None if alpha_field is None else np.ascontiguousarray(alpha_field, dtype=np.float64)
    _check(lib().oracle_nonlinear(ctypes.byref(p), _p(af), _p(w), _p(r1), _p(r2), _p(wn), _p(r1n), _p(r2n),
                                  _p(phys)))
    return (wn, r1n, r2n, phys) if want_phys else (wn, r1n, r2n)


def step(p, w, r1, r2, nsteps, integrator=IFRK4, alpha_field=None):
    """Return the state after ``nsteps`` steps (inputs are not modified)."""
    w, r1, r2 = _spec(w).copy(), _spec(r1).copy(), _spec(r2).copy()
    af = None if alpha_field is None else np.ascontiguousarray(alpha_field, dtype=np.float64)
    _check(lib().oracle_step(ctypes.byref(p), integrator, _p(af), _p(w), _p(r1), _p(r2), nsteps))
    return w, r1, r2


def step_tlm(p, w, r1, r2, dw, dr1, dr2, nsteps, loss_window, alpha_field=None, dalpha_field=None):
    """IF-RK4 with its tangent-linear model: returns (final state, final tangent,
    loss, dloss), loss the mean enstrophy 0.5 mean(w^2) of the states after the
    last ``loss_window`` steps and dloss its derivative along the tangent."""
    w, r1, r2 = _spec(w).copy(), _spec(r1).copy(), _spec(r2).copy()
    dw, dr1, dr2 = _spec(dw).copy(), _spec(dr1).copy(), _spec(dr2).copy()
    af = None if alpha_field is None else np.ascontiguousarray(alpha_field, dtype=np.float64)
    daf = None if dalpha_field is None else np.ascontiguousarray(dalpha_field, dtype=np.float64)
    loss, dloss = ctypes.c_double(), ctypes.c_double()
    _check(lib().oracle_step_tlm(ctypes.byref(p), _p(af), _p(daf), _p(w), _p(r1), _p(r2), _p(dw), _p(dr1), _p(dr2),
                                 nsteps, loss_window, ctypes.byref(loss), ctypes.byref(dloss)))
    return (w, r1, r2), (dw, dr1, dr2), loss.value, dloss.value


def diagnostics(p, w, nshells=0):
    w = _spec(w)
    e, z = ctypes.c_double(), ctypes.c_double()
    spec = np.empty(max(nshells, 1))
    _check(lib().oracle_diagnostics(ctypes.byref(p), _p(w), ctypes.byref(e), ctypes.byref(z),
                                    _p(spec) if nshells else None, nshells))
    return e.value, z.value, (spec[:nshells] if nshells else None)


# ---- seeded initial condition: numpy restatement of include/qaf_init.h ----
_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def uniform(seed, first, count, lo, hi):
    k = np.arange(first, first + count, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (k + np.uint64(1)) * _GAMMA
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return lo + (hi - lo) * u


def random_q_init(seed, n, lo=-0.01, hi=0.01, ny=None):
    ny = ny or n
    np_ = n * ny
    w = np.zeros((ny, n))
    r1 = uniform(seed, 0, np_, lo, hi).reshape(ny, n)
    r2 = uniform(seed, np_, np_, lo, hi).reshape(ny, n)
    return w, r1, r2


def couple_init(seed, n, L, amp=1e-3):
    """Smooth initial state of UnitTest/TimeIntegration/couple/couple.cu:4-35 with
    seeded noise (qaf_couple_init of include/qaf_init.h): w = 0,
    r1 = 0.2 (sin^2(x+y) - 1/2) + amp u, r2 = 0.2 sin(x+y) cos(x+y) + amp u'."""
    np_ = n * n
    i = np.arange(n)
    ph = (i[None, :] * (L / n)) + (i[:, None] * (L / n))
    s, c = np.sin(ph), np.cos(ph)
    r1 = 0.2 * (s * s - 0.5) + amp * uniform(seed, 0, np_, 0.0, 1.0).reshape(n, n)
    r2 = 0.2 * s * c + amp * uniform(seed, np_, np_, 0.0, 1.0).reshape(n, n)
    return np.zeros((n, n)), r1, r2


def random_q_init_c(seed, n, lo=-0.01, hi=0.01):
    """The same initial state from the C header (through the oracle library)."""
    w, r1, r2 = (np.empty((n, n)) for _ in range(3))
    lib().oracle_random_q_init(seed, n, n, lo, hi, _p(w), _p(r1), _p(r2))
    return w, r1, r2


def couple_init_c(seed, n, L, amp=1e-3):
    """The coupled-run initial state from the C header (through the oracle library)."""
    w, r1, r2 = (np.empty((n, n)) for _ in range(3))
    lib().oracle_couple_init(seed, n, L, amp, _p(w), _p(r1), _p(r2))
    return w, r1, r2


def initial_spectra(seed, n, **kw):
    """Spectral initial state as the reference driver builds it: FwdTrans of the
    physical fields (friction.cu:165-185); the following BwdTrans only
    symmetrises the kx=0 column, which for a real field changes it by rounding."""
    w, r1, r2 = random_q_init(seed, n, **kw)
    return fwd(w), fwd(r1), fwd(r2)


# ---- binary dumps of the driver around the reference's CUDA build ----
def read_dump(path):
    with open(path, "rb") as f:
        raw = f.read()
    if raw[:8] != b"QAFDUMP1":
        raise ValueError(f"{path}: not a QAFDUMP1 file")
    nx, ny, nxh, rb, nf, kind = struct.unpack("<6i", raw[8:32])
    (step_,) = struct.unpack("<q", raw[32:40])
    body = raw[40:]
    if kind == 0:
        dt = np.complex128 if rb == 8 else np.complex64
        per = ny * nxh
        arr = np.frombuffer(body, dtype=dt, count=nf * per).reshape(nf, ny, nxh)
    else:
        dt = np.float64 if rb == 8 else np.float32
        per = ny * nx
        arr = np.frombuffer(body, dtype=dt, count=nf * per).reshape(nf, ny, nx)
    return {"nx": nx, "ny": ny, "step": step_, "kind": kind, "fields": [a.copy() for a in arr]}


def hermitian_part(spec):
    """Replace the kx=0 and kx=nx/2 columns by their Hermitian parts: the part
    of a stored half-spectrum that a C2R can see."""
    s = np.array(spec, dtype=np.complex128, copy=True)
    ny = s.shape[0]
    idx = (-np.arange(ny)) % ny
    for c in (0, s.shape[1] - 1):
        col = s[:, c].copy()
        s[:, c] = 0.5 * (col + np.conj(col[idx]))
    return s


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
