"""qaf — Python face of the B200 pseudo-spectral active-nematic solver.

A thin ctypes binding of the C ABI in include/qaf.h (libqaf.so, built in this
directory by ``nature-control_b200/build.py``). Device memory and streams come
from PyTorch CUDA tensors; every computation runs in the library's CUDA
kernels. There is no CPU fallback: without the built library, or without a
GPU, the calls raise.

The names follow the reference's header-only API (whpy/nature-control):
``Mesh`` (Basic/Mesh.cuh:48-113), ``fwd_trans``/``bwd_trans`` (FwdTrans /
BwdTrans, FldOp/QFldfuncs.cuh:45-55), ``xderiv``/``yderiv``/``laplacian``/
``vel`` (:165-224), ``nonlinear`` (curr_func + wnonl_func + r1nonl_func +
r2nonl_func, InertialFriction/friction/Qsolver.cuh:166-312), ``step`` (the
IF-RK4 loop of InertialFriction/friction/friction.cu:212-259, and the IF-RK2 /
IF-Euler integrators of TimeIntegration/).
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqaf.so")

F32, F64 = 0, 1
IFE, IFRK2, IFRK4 = 0, 1, 2
OK, ERR_INVALID, ERR_UNSUPPORTED, ERR_CUDA, ERR_NONFINITE, ERR_ALLOC = range(6)

# Every symbol include/qaf.h declares (the tests check the library exports them).
EXPORTS = [
    "qaf_version", "qaf_last_error", "qaf_supported", "qaf_mesh_create", "qaf_mesh_destroy", "qaf_mesh_sizes",
    "qaf_field_alloc", "qaf_field_free", "qaf_mesh_tables", "qaf_fwd_trans", "qaf_bwd_trans", "qaf_symmetrize",
    "qaf_xderiv", "qaf_yderiv", "qaf_laplacian", "qaf_vel", "qaf_dealias", "qaf_if_tables", "qaf_integrate",
    "qaf_nonlinear", "qaf_step", "qaf_step_host", "qaf_last_diagnostics", "qaf_check_finite", "qaf_diagnostics",
    "qaf_state_load", "qaf_state_advance", "qaf_state_store", "qaf_last_diagnostics_async", "qaf_state_save", "qaf_state_restore", "qaf_state_advance_timed", "qaf_launch_count",
    "qaf_test_lose_copy",
    "qaf_init_random_q", "qaf_step_noalloc", "qaf_ensemble_create", "qaf_ensemble_destroy",
    "qaf_ensemble_init_random", "qaf_ensemble_load", "qaf_ensemble_store", "qaf_ensemble_advance",
    "qaf_ensemble_diagnostics", "qaf_ensemble_set_controls", "qaf_adjoint_create", "qaf_adjoint_destroy",
    "qaf_adjoint_forward", "qaf_adjoint_backward", "qaf_autotune", "qaf_autotune_load", "qaf_autotune_reset",
    "qaf_set_variant", "qaf_variant_choice", "qaf_variant_list", "qaf_adjoint_batch_create",
    "qaf_adjoint_batch_destroy", "qaf_adjoint_batch_forward", "qaf_adjoint_batch_backward",
]


class QafError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"qaf status {status}: {msg}")
        self.status = status


class NonFiniteError(QafError):
    pass


class MeshDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("lx", ctypes.c_double), ("ly", ctypes.c_double),
                ("dtype", ctypes.c_int)]


class CParams(ctypes.Structure):
    _fields_ = [("re", ctypes.c_double), ("er", ctypes.c_double), ("rf", ctypes.c_double),
                ("lam", ctypes.c_double), ("alpha", ctypes.c_double), ("alpha_field", ctypes.c_void_p),
                ("dt", ctypes.c_double), ("q_lin", ctypes.c_double), ("advect_omega", ctypes.c_int),
                ("no_dealias", ctypes.c_int)]


@dataclass
class Params:
    """Physical parameters (InertialFriction/friction/friction.cu:100-105 names)."""
    re: float = 1.0
    er: float = 1.0
    rf: float = 0.1
    lam: float = 0.1
    alpha: float = 1.0
    dt: float = 1e-3
    q_lin: float = 1.0
    advect_omega: int = 1
    no_dealias: int = 0      # 1: no 2/3 truncation per step (the coupled runs); 2: of w only (dealias/couple.cu)
    alpha_field: Optional[object] = field(default=None, repr=False)   # torch tensor (ny, nx) on the device

    def c(self) -> CParams:
        ptr = None
        if self.alpha_field is not None:
            ptr = self.alpha_field.data_ptr()
        return CParams(self.re, self.er, self.rf, self.lam, self.alpha, ptr, self.dt, self.q_lin, self.advect_omega,
                       self.no_dealias)


_lib = None


def lib():
    """Load libqaf.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python nature-control_b200/build.py` "
                              "(or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        vp, cp = ctypes.c_void_p, ctypes.c_int
        L.qaf_version.restype = ctypes.c_char_p
        L.qaf_last_error.restype = ctypes.c_char_p
        L.qaf_supported.argtypes = [cp, cp]
        L.qaf_mesh_create.argtypes = [ctypes.POINTER(MeshDesc), ctypes.POINTER(vp)]
        L.qaf_mesh_destroy.argtypes = [vp]
        L.qaf_mesh_sizes.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
        L.qaf_mesh_tables.argtypes = [vp, vp, vp, vp, vp]
        for n in ("qaf_fwd_trans", "qaf_bwd_trans", "qaf_xderiv", "qaf_yderiv", "qaf_laplacian"):
            getattr(L, n).argtypes = [vp, vp, vp, vp]
        L.qaf_symmetrize.argtypes = [vp, vp, vp]
        L.qaf_dealias.argtypes = [vp, vp, vp]
        L.qaf_vel.argtypes = [vp, vp, vp, vp, vp]
        L.qaf_if_tables.argtypes = [vp, ctypes.POINTER(CParams), cp, vp, vp, vp]
        L.qaf_integrate.argtypes = [vp, cp, cp, vp, vp, vp, vp, vp, vp, ctypes.c_double, vp]
        L.qaf_nonlinear.argtypes = [vp, ctypes.POINTER(CParams), vp, vp, vp, vp, vp, vp, vp]
        L.qaf_nonlinear_dbg.argtypes = [vp, ctypes.POINTER(CParams), vp, vp, vp, vp, vp, vp, vp, vp]
        L.qaf_step.argtypes = [vp, ctypes.POINTER(CParams), cp, vp, vp, vp, cp, vp]
        L.qaf_step_host.argtypes = [vp, ctypes.POINTER(CParams), cp, vp, vp, vp, cp]
        L.qaf_last_diagnostics.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.qaf_last_diagnostics_async.argtypes = [vp, vp, vp]
        L.qaf_state_save.argtypes = [vp, ctypes.c_char_p, ctypes.c_uint64, vp]
        L.qaf_state_restore.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64), vp]
        L.qaf_check_finite.argtypes = [vp, vp]
        L.qaf_diagnostics.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double), cp, vp]
        L.qaf_state_load.argtypes = [vp, vp, vp, vp, vp]
        L.qaf_state_store.argtypes = [vp, vp, vp, vp, vp]
        L.qaf_state_advance.argtypes = [vp, ctypes.POINTER(CParams), cp, cp, vp]
        L.qaf_state_advance_timed.argtypes = [vp, ctypes.POINTER(CParams), cp, cp, ctypes.POINTER(ctypes.c_double), vp]
        L.qaf_launch_count.argtypes = [vp]
        L.qaf_launch_count.restype = ctypes.c_uint64
        L.qaf_init_random_q.argtypes = [vp, ctypes.c_uint64, ctypes.c_double, ctypes.c_double, vp, vp, vp, vp]
        L.qaf_step_noalloc.argtypes = [cp, ctypes.c_double, ctypes.c_double, cp, ctypes.POINTER(CParams), cp,
                                       vp, vp, vp, cp, vp, vp]
        L.qaf_test_lose_copy.argtypes = [cp, ctypes.c_uint]
        dp = ctypes.POINTER(ctypes.c_double)
        L.qaf_ensemble_create.argtypes = [cp, ctypes.POINTER(cp), ctypes.c_double, ctypes.c_double, cp,
                                          ctypes.POINTER(CParams), dp, dp, ctypes.POINTER(vp)]
        L.qaf_ensemble_destroy.argtypes = [vp]
        L.qaf_ensemble_init_random.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.c_double,
                                               ctypes.c_double, vp]
        L.qaf_ensemble_load.argtypes = [vp, cp, vp, vp, vp, vp]
        L.qaf_ensemble_store.argtypes = [vp, cp, vp, vp, vp, vp]
        L.qaf_ensemble_advance.argtypes = [vp, cp, vp]
        L.qaf_ensemble_diagnostics.argtypes = [vp, dp, vp]
        L.qaf_ensemble_set_controls.argtypes = [vp, dp, dp, vp]
        L.qaf_adjoint_create.argtypes = [vp, cp, cp, cp, ctypes.POINTER(vp)]
        L.qaf_adjoint_destroy.argtypes = [vp]
        L.qaf_adjoint_forward.argtypes = [vp, ctypes.POINTER(CParams), vp, vp, vp, vp, vp, vp, dp, vp]
        L.qaf_adjoint_backward.argtypes = [vp, vp, vp, vp, ctypes.c_double, vp, vp, vp, vp, vp]
        sp = ctypes.c_char_p
        L.qaf_autotune.argtypes = [cp, cp, cp, sp, sp, cp, dp]
        L.qaf_autotune_load.argtypes = [sp]
        L.qaf_autotune_reset.argtypes = []
        L.qaf_set_variant.argtypes = [cp, cp, cp, sp, sp]
        L.qaf_variant_choice.argtypes = [cp, cp, cp, sp, cp]
        L.qaf_variant_list.argtypes = [cp, cp, sp, cp]
        L.qaf_adjoint_batch_create.argtypes = [cp, cp, ctypes.c_double, ctypes.c_double, cp, ctypes.POINTER(CParams),
                                               cp, cp, cp, ctypes.POINTER(vp)]
        L.qaf_adjoint_batch_destroy.argtypes = [vp]
        L.qaf_adjoint_batch_forward.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, dp, vp]
        L.qaf_adjoint_batch_backward.argtypes = [vp, vp, vp, vp, dp, vp, vp, vp, vp, vp]
        _lib = L
    return _lib


def _check(status):
    if status != OK:
        msg = lib().qaf_last_error().decode(errors="replace")
        if status == ERR_NONFINITE:
            raise NonFiniteError(status, msg)
        raise QafError(status, msg)


def version() -> str:
    return lib().qaf_version().decode()


def supported(n: int, dtype: int = F32) -> bool:
    return bool(lib().qaf_supported(n, dtype))


def autotune(n: int, dtype: int = F32, ninst: int = 1, cache: Optional[str] = None):
    """Time the launch shapes of the fused step kernels for n x n on `ninst`
    synthetic instances and keep the fastest; returns (choice, us per step)."""
    buf = ctypes.create_string_buffer(128)
    us = ctypes.c_double()
    _check(lib().qaf_autotune(n, dtype, ninst, cache.encode() if cache else None, buf, 128, ctypes.byref(us)))
    return buf.value.decode(), us.value


def autotune_load(path: str):
    """Apply the records of an autotuner cache that match this GPU."""
    _check(lib().qaf_autotune_load(path.encode()))


def autotune_reset():
    """Back to the built-in launch shapes."""
    _check(lib().qaf_autotune_reset())


def set_variant(n: int, dtype: int, batched: bool, col: str = "default", row: str = "default"):
    _check(lib().qaf_set_variant(n, dtype, 1 if batched else 0, col.encode(), row.encode()))


def variant_choice(n: int, dtype: int = F32, batched: bool = False) -> str:
    buf = ctypes.create_string_buffer(128)
    _check(lib().qaf_variant_choice(n, dtype, 1 if batched else 0, buf, 128))
    return buf.value.decode()


def variant_list(n: int, dtype: int = F32):
    buf = ctypes.create_string_buffer(512)
    _check(lib().qaf_variant_list(n, dtype, buf, 512))
    return buf.value.decode().split()


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    import torch
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


class Mesh:
    """Grid geometry, wave numbers, 2/3 mask and scratch (Basic/Mesh.cuh:48-113).

    Fields are torch CUDA tensors: physical (ny, nx) real, spectral
    (ny, nx//2+1) complex, in the reference's index order (x fastest).
    """

    def __init__(self, nx: int, ny: Optional[int] = None, lx: float = 2 * math.pi, ly: Optional[float] = None,
                 dtype: int = F64):
        self.nx, self.ny = nx, ny or nx
        self.lx, self.ly = lx, ly or lx
        self.dtype = dtype
        self.nxh = nx // 2 + 1
        h = ctypes.c_void_p()
        _check(lib().qaf_mesh_create(ctypes.byref(MeshDesc(self.nx, self.ny, self.lx, self.ly, dtype)), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.qaf_mesh_destroy(h)
            self._h = None

    # -- tensors --------------------------------------------------------
    @property
    def real_dtype(self):
        import torch
        return torch.float64 if self.dtype == F64 else torch.float32

    @property
    def complex_dtype(self):
        import torch
        return torch.complex128 if self.dtype == F64 else torch.complex64

    def new_spec(self):
        import torch
        return torch.zeros((self.ny, self.nxh), dtype=self.complex_dtype, device="cuda")

    def new_phys(self):
        import torch
        return torch.zeros((self.ny, self.nx), dtype=self.real_dtype, device="cuda")

    def _chk_spec(self, t):
        if tuple(t.shape) != (self.ny, self.nxh) or t.dtype != self.complex_dtype:
            raise ValueError(f"spectrum must be {(self.ny, self.nxh)} {self.complex_dtype}, got {tuple(t.shape)} {t.dtype}")
        return _ptr(t)

    def _chk_phys(self, t):
        if tuple(t.shape) != (self.ny, self.nx) or t.dtype != self.real_dtype:
            raise ValueError(f"physical field must be {(self.ny, self.nx)} {self.real_dtype}, got {tuple(t.shape)} {t.dtype}")
        return _ptr(t)

    def tables(self):
        """kx, ky, k^2, cutoff as numpy arrays (waveinit / cutoff_func, Mesh.cuh:6-46)."""
        import numpy as np
        dt = np.float64 if self.dtype == F64 else np.float32
        arrs = [np.empty((self.ny, self.nxh), dt) for _ in range(4)]
        _check(lib().qaf_mesh_tables(self._h, *[a.ctypes.data_as(ctypes.c_void_p) for a in arrs]))
        return arrs

    # -- transforms and operators ---------------------------------------
    def fwd_trans(self, phys, spec=None):
        spec = self.new_spec() if spec is None else spec
        _check(lib().qaf_fwd_trans(self._h, self._chk_phys(phys), self._chk_spec(spec), _stream()))
        return spec

    def bwd_trans(self, spec, phys=None):
        phys = self.new_phys() if phys is None else phys
        _check(lib().qaf_bwd_trans(self._h, self._chk_spec(spec), self._chk_phys(phys), _stream()))
        return phys

    def symmetrize(self, spec):
        _check(lib().qaf_symmetrize(self._h, self._chk_spec(spec), _stream()))
        return spec

    def _unary(self, name, x, out):
        out = self.new_spec() if out is None else out
        _check(getattr(lib(), name)(self._h, self._chk_spec(x), self._chk_spec(out), _stream()))
        return out

    def xderiv(self, x, out=None):
        return self._unary("qaf_xderiv", x, out)

    def yderiv(self, x, out=None):
        return self._unary("qaf_yderiv", x, out)

    def laplacian(self, x, out=None):
        return self._unary("qaf_laplacian", x, out)

    def vel(self, w):
        u, v = self.new_spec(), self.new_spec()
        _check(lib().qaf_vel(self._h, self._chk_spec(w), self._chk_spec(u), self._chk_spec(v), _stream()))
        return u, v

    def dealias(self, x):
        _check(lib().qaf_dealias(self._h, self._chk_spec(x), _stream()))
        return x

    def if_tables(self, p: Params, which: int):
        import torch
        IF = torch.empty((self.ny, self.nxh), dtype=self.real_dtype, device="cuda")
        IFh = torch.empty_like(IF)
        cp = p.c()
        _check(lib().qaf_if_tables(self._h, ctypes.byref(cp), which, _ptr(IF), _ptr(IFh), _stream()))
        return IF, IFh

    def integrate(self, integ, stage, old, curr, new, nonl, IF, IFh, dt):
        nl = None if nonl is None else self._chk_spec(nonl)
        cu = None if curr is None else self._chk_spec(curr)
        _check(lib().qaf_integrate(self._h, integ, stage, self._chk_spec(old), cu, self._chk_spec(new), nl,
                                   _ptr(IF), _ptr(IFh), dt, _stream()))

    # -- hot path -------------------------------------------------------
    def nonlinear(self, p: Params, w, r1, r2, want_phys=False):
        """N_w, N_r1, N_r2 at the given spectra; with want_phys also the row
        pass's physical fields (w r1 r2 u v du/dx du/dy+dv/dx Lap r1 Lap r2 S p11 p12 p21)."""
        import torch
        outs = [self.new_spec() for _ in range(3)]
        cp = p.c()
        if want_phys:
            phys = torch.zeros((13, self.ny, self.nx), dtype=self.real_dtype, device="cuda")
            _check(lib().qaf_nonlinear_dbg(self._h, ctypes.byref(cp), self._chk_spec(w), self._chk_spec(r1),
                                           self._chk_spec(r2), *[self._chk_spec(o) for o in outs], _ptr(phys),
                                           _stream()))
            return (*outs, phys)
        _check(lib().qaf_nonlinear(self._h, ctypes.byref(cp), self._chk_spec(w), self._chk_spec(r1),
                                   self._chk_spec(r2), *[self._chk_spec(o) for o in outs], _stream()))
        return tuple(outs)

    def step(self, p: Params, w, r1, r2, nsteps: int = 1, integrator: int = IFRK4):
        """Advance the spectral state (w, r1, r2) in place by nsteps steps."""
        cp = p.c()
        _check(lib().qaf_step(self._h, ctypes.byref(cp), integrator, self._chk_spec(w), self._chk_spec(r1),
                              self._chk_spec(r2), nsteps, _stream()))
        return w, r1, r2

    def random_q(self, seed: int, lo: float = -0.01, hi: float = 0.01):
        """Seeded initial spectra (w = 0, r1, r2 ~ U(lo, hi); include/qaf_init.h)."""
        w, r1, r2 = self.new_spec(), self.new_spec(), self.new_spec()
        _check(lib().qaf_init_random_q(self._h, seed, lo, hi, self._chk_spec(w), self._chk_spec(r1),
                                       self._chk_spec(r2), _stream()))
        return w, r1, r2

    # -- resident state (load once, advance, store snapshots) -----------
    def load(self, w, r1, r2):
        _check(lib().qaf_state_load(self._h, self._chk_spec(w), self._chk_spec(r1), self._chk_spec(r2), _stream()))

    def store(self, w=None, r1=None, r2=None):
        w = self.new_spec() if w is None else w
        r1 = self.new_spec() if r1 is None else r1
        r2 = self.new_spec() if r2 is None else r2
        _check(lib().qaf_state_store(self._h, self._chk_spec(w), self._chk_spec(r1), self._chk_spec(r2), _stream()))
        return w, r1, r2

    def save(self, path: str, step: int = 0):
        """Write the resident state to a checkpoint file (exact, with a step counter)."""
        _check(lib().qaf_state_save(self._h, str(path).encode(), int(step), _stream()))

    def restore(self, path: str) -> int:
        """Load the resident state from a checkpoint file; returns its step counter."""
        st = ctypes.c_uint64()
        _check(lib().qaf_state_restore(self._h, str(path).encode(), ctypes.byref(st), _stream()))
        return st.value

    def advance(self, p: Params, nsteps: int = 1, integrator: int = IFRK4):
        cp = p.c()
        _check(lib().qaf_state_advance(self._h, ctypes.byref(cp), integrator, nsteps, _stream()))

    def advance_timed(self, p: Params, nsteps: int = 1, integrator: int = IFRK4):
        """Advance with CUDA events around each kernel: (row_ms, col_ms, launches)."""
        cp = p.c()
        out = (ctypes.c_double * 3)()
        _check(lib().qaf_state_advance_timed(self._h, ctypes.byref(cp), integrator, nsteps, out, _stream()))
        return out[0], out[1], int(out[2])

    def launch_count(self) -> int:
        return int(lib().qaf_launch_count(self._h))

    def last_diagnostics(self):
        """(energy, enstrophy) of the state left by the last step()."""
        out = (ctypes.c_double * 2)()
        _check(lib().qaf_last_diagnostics(self._h, out))
        return out[0], out[1]

    def last_diagnostics_async(self, out=None):
        """Enqueue a read-back of (energy, enstrophy) of the last step into `out`
        (a float64 tensor of 2, pinned host memory or on the device; a new pinned
        one if None) without synchronising; valid once the stream reaches it."""
        import torch
        if out is None:
            out = torch.empty(2, dtype=torch.float64).pin_memory()
        if out.dtype != torch.float64 or out.numel() < 2 or not out.is_contiguous():
            raise ValueError("out must be a contiguous float64 tensor of 2")
        if not out.is_cuda and not out.is_pinned():
            raise ValueError("out must be pinned host memory or a device tensor")
        _check(lib().qaf_last_diagnostics_async(self._h, ctypes.c_void_p(out.data_ptr()), _stream()))
        return out

    def check_finite(self):
        _check(lib().qaf_check_finite(self._h, _stream()))

    def diagnostics(self, w, nshells: int = 0):
        """(energy, enstrophy, spectrum[nshells]) of a vorticity spectrum."""
        import numpy as np
        e, z = ctypes.c_double(), ctypes.c_double()
        spec = np.zeros(max(nshells, 1))
        _check(lib().qaf_diagnostics(self._h, self._chk_spec(w), ctypes.byref(e), ctypes.byref(z),
                                     spec.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nshells, _stream()))
        return e.value, z.value, (spec[:nshells] if nshells else None)


class Ensemble:
    """Many independent instances advanced together with IF-RK4.

    Instance k has grid n[k] x n[k] (one of the supported sizes), activity
    alpha[k] and friction rf[k]; Re, Er, lambda, dt and q_lin come from the
    shared Params. The reference runs one grid per process (friction.cu);
    this is the batched form of that loop.
    """

    def __init__(self, n, p: Params, alpha, rf=None, lx: float = 2 * math.pi, ly: Optional[float] = None,
                 dtype: int = F32, tune: bool = False, tune_cache: Optional[str] = None):
        """tune: time the launch shapes for each grid size first (tune_cache:
        read the choices from this JSON-lines file when it has them, else tune
        and record them there)."""
        self.n = [int(v) for v in n]
        if tune_cache is not None and os.path.exists(tune_cache):
            autotune_load(tune_cache)
        if tune:
            for size in sorted(set(self.n)):
                count = self.n.count(size)
                if tune_cache is not None and os.path.exists(tune_cache) and \
                        variant_choice(size, dtype, count > 1) != "col:default row:default":
                    continue
                autotune(size, dtype, count, tune_cache)
        self.tuned = {size: variant_choice(size, dtype, self.n.count(size) > 1) for size in sorted(set(self.n))}
        k = len(self.n)
        self.alpha = [float(v) for v in alpha]
        self.rf = [float(p.rf)] * k if rf is None else [float(v) for v in rf]
        if len(self.alpha) != k or len(self.rf) != k:
            raise ValueError("alpha and rf need one value per instance")
        self.lx, self.ly, self.dtype, self.params = lx, ly or lx, dtype, p
        self._meshes = {}
        cp = p.c()
        h = ctypes.c_void_p()
        na = (ctypes.c_int * k)(*self.n)
        aa = (ctypes.c_double * k)(*self.alpha)
        ra = (ctypes.c_double * k)(*self.rf)
        _check(lib().qaf_ensemble_create(k, na, self.lx, self.ly, dtype, ctypes.byref(cp), aa, ra, ctypes.byref(h)))
        self._h = h

    def __len__(self):
        return len(self.n)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.qaf_ensemble_destroy(h)
            self._h = None

    def mesh(self, k: int) -> Mesh:
        """A Mesh with instance k's geometry (for tensors and transforms)."""
        n = self.n[k]
        if n not in self._meshes:
            self._meshes[n] = Mesh(n, n, self.lx, self.ly, self.dtype)
        return self._meshes[n]

    def init_random(self, seeds, lo: float = -0.01, hi: float = 0.01):
        sa = (ctypes.c_uint64 * len(self.n))(*[int(v) for v in seeds])
        _check(lib().qaf_ensemble_init_random(self._h, sa, lo, hi, _stream()))

    def load(self, k: int, w, r1, r2):
        m = self.mesh(k)
        _check(lib().qaf_ensemble_load(self._h, k, m._chk_spec(w), m._chk_spec(r1), m._chk_spec(r2), _stream()))

    def store(self, k: int):
        m = self.mesh(k)
        w, r1, r2 = m.new_spec(), m.new_spec(), m.new_spec()
        _check(lib().qaf_ensemble_store(self._h, k, m._chk_spec(w), m._chk_spec(r1), m._chk_spec(r2), _stream()))
        return w, r1, r2

    def advance(self, nsteps: int = 1):
        _check(lib().qaf_ensemble_advance(self._h, nsteps, _stream()))

    def set_controls(self, alpha, rf=None):
        """New per-instance activity (and friction) for the following steps."""
        k = len(self.n)
        alpha = [float(v) for v in alpha]
        rf = self.rf if rf is None else [float(v) for v in rf]
        if len(alpha) != k or len(rf) != k:
            raise ValueError("alpha and rf need one value per instance")
        self.alpha, self.rf = alpha, rf
        aa = (ctypes.c_double * k)(*self.alpha)
        ra = (ctypes.c_double * k)(*self.rf)
        _check(lib().qaf_ensemble_set_controls(self._h, aa, ra, _stream()))

    def diagnostics(self):
        """[(energy, enstrophy)] per instance after the last step."""
        k = len(self.n)
        out = (ctypes.c_double * (2 * k))()
        _check(lib().qaf_ensemble_diagnostics(self._h, out, _stream()))
        return [(out[2 * i], out[2 * i + 1]) for i in range(k)]


class Adjoint:
    """Reverse-mode gradients of `nsteps` IF-RK4 steps on `mesh` (include/qaf.h,
    qaf_adjoint_*): of the mean enstrophy of the states after the last
    `loss_window` steps and of any function of the final state, with respect
    to the initial spectra and the activity field Ra(x). The state is kept
    every `checkpoint_every` steps and each segment is recomputed once during
    the backward sweep. The mesh's resident state is overwritten."""

    def __init__(self, mesh: Mesh, nsteps: int, checkpoint_every: int = 64, loss_window: int = 0):
        self.mesh, self.nsteps, self.K, self.window = mesh, nsteps, checkpoint_every, loss_window
        h = ctypes.c_void_p()
        _check(lib().qaf_adjoint_create(mesh._h, nsteps, checkpoint_every, loss_window, ctypes.byref(h)))
        self._h = h
        self._alpha = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.qaf_adjoint_destroy(h)
            self._h = None

    def forward(self, p: Params, w0, r1_0, r2_0, final_state: bool = True):
        """Run the steps; returns (loss, (wT, r1T, r2T) or None)."""
        m = self.mesh
        self._alpha = p.alpha_field          # must outlive the backward call
        cp = p.c()
        out = (m.new_spec(), m.new_spec(), m.new_spec()) if final_state else None
        ptrs = [m._chk_spec(t) for t in out] if out else [None, None, None]
        loss = ctypes.c_double()
        _check(lib().qaf_adjoint_forward(self._h, ctypes.byref(cp), m._chk_spec(w0), m._chk_spec(r1_0),
                                         m._chk_spec(r2_0), *ptrs, ctypes.byref(loss), _stream()))
        return loss.value, out

    def backward(self, grad_final=None, grad_loss: float = 1.0, want_alpha: bool = True):
        """Gradients (gw0, gr1_0, gr2_0, galpha) given dL/d(final state) (or None) and dL/d(loss)."""
        m = self.mesh
        g = [None, None, None]
        keep = []
        if grad_final is not None:
            keep = [t.contiguous() if t is not None else None for t in grad_final]
            g = [m._chk_spec(t) if t is not None else None for t in keep]
        gw, g1, g2 = m.new_spec(), m.new_spec(), m.new_spec()
        ga = m.new_phys() if want_alpha else None
        _check(lib().qaf_adjoint_backward(self._h, *g, float(grad_loss), m._chk_spec(gw), m._chk_spec(g1),
                                          m._chk_spec(g2), m._chk_phys(ga) if ga is not None else None,
                                          _stream()))
        return gw, g1, g2, ga


class AdjointBatch:
    """`ninst` instances of one n x n grid (n <= 256) with their own initial
    spectra and activity fields, stepped and differentiated together
    (qaf_adjoint_batch_*): each stage of the forward, recompute and adjoint is
    one launch for the whole batch. Tensors hold the instances along dim 0."""

    def __init__(self, ninst: int, n: int, p: Params, nsteps: int, checkpoint_every: int = 64, loss_window: int = 1,
                 lx: float = 2 * math.pi, dtype: int = F32):
        self.ninst, self.n, self.nsteps, self.dtype = ninst, n, nsteps, dtype
        self.mesh = Mesh(n, n, lx, lx, dtype)          # tensor shapes and dtypes
        cp = p.c()
        h = ctypes.c_void_p()
        _check(lib().qaf_adjoint_batch_create(ninst, n, lx, lx, dtype, ctypes.byref(cp), nsteps, checkpoint_every,
                                              loss_window, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.qaf_adjoint_batch_destroy(h)
            self._h = None

    def _spec(self):
        import torch
        return torch.zeros((self.ninst, self.n, self.n // 2 + 1), dtype=self.mesh.complex_dtype, device="cuda")

    def _chk(self, t, real=False):
        shape = (self.ninst, self.n, self.n) if real else (self.ninst, self.n, self.n // 2 + 1)
        dt = self.mesh.real_dtype if real else self.mesh.complex_dtype
        if tuple(t.shape) != shape or t.dtype != dt:
            raise ValueError(f"expected {shape} {dt}, got {tuple(t.shape)} {t.dtype}")
        return _ptr(t)

    def forward(self, w0, r1_0, r2_0, alpha=None, final_state: bool = True):
        """Returns (losses (list of ninst floats), (wT, r1T, r2T) or None)."""
        out = (self._spec(), self._spec(), self._spec()) if final_state else None
        ptrs = [self._chk(t) for t in out] if out else [None, None, None]
        losses = (ctypes.c_double * self.ninst)()
        _check(lib().qaf_adjoint_batch_forward(self._h, self._chk(w0), self._chk(r1_0), self._chk(r2_0),
                                               self._chk(alpha, True) if alpha is not None else None, *ptrs, losses,
                                               _stream()))
        return list(losses), out

    def backward(self, grad_final=None, grad_losses=None, want_alpha: bool = True):
        """(gw0, gr1_0, gr2_0, galpha) for dL/d(final states) (or None) and dL/dloss_k (or None)."""
        import torch
        keep = [t.contiguous() if t is not None else None for t in grad_final] if grad_final is not None else []
        g = [self._chk(t) if t is not None else None for t in keep] if keep else [None, None, None]
        gl = (ctypes.c_double * self.ninst)(*[float(v) for v in grad_losses]) if grad_losses is not None else None
        gw, g1, g2 = self._spec(), self._spec(), self._spec()
        ga = torch.zeros((self.ninst, self.n, self.n), dtype=self.mesh.real_dtype, device="cuda") if want_alpha else None
        _check(lib().qaf_adjoint_batch_backward(self._h, *g, gl, self._chk(gw), self._chk(g1), self._chk(g2),
                                                self._chk(ga, True) if ga is not None else None, _stream()))
        return gw, g1, g2, ga

