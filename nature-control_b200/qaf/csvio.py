"""Physical-field CSV files in the reference's format.

The reference's drivers start from ``./init/{w,r1,r2}_init.csv`` (file_init,
InertialFriction/friction/friction.cu:62-97, 164-185) and every 1000 steps
write ``{step}w.csv``, ``{step}r1.csv``, ``{step}r2.csv`` and ``{step}S.csv``
(field_visual, BasicUtils/BasicUtils.cuh:38-50; friction.cu:262-278). A file
holds one line per grid row j (ny lines); line j holds the values f[j*nx + i],
i = 0..nx-1, each followed by a comma, printed as a C++ stream prints a double
by default: %g with 6 significant digits.

These files round the state to 6 digits; Mesh.save/Mesh.restore keep it exact.
The functions here let runs move between the reference and this library:

    w, r1, r2 = qaf.csvio.load_state(mesh, "init/")          # file_init + FwdTrans
    qaf.csvio.write_snapshot(mesh, 25000)                     # 25000w.csv ... 25000S.csv
"""
from __future__ import annotations

import math
import os
from typing import Optional

import numpy as np


def format_value(v: float) -> str:
    """A double as a default-formatted C++ output stream prints it (%g, 6 digits)."""
    if math.isnan(v):
        return "-nan" if math.copysign(1.0, v) < 0 else "nan"
    if math.isinf(v):
        return "-inf" if v < 0 else "inf"
    return "%g" % v


def write_field(path: str, field) -> None:
    """field_visual: an (ny, nx) array (numpy or torch, any device) to `path`."""
    a = _host(field)
    if a.ndim != 2:
        raise ValueError("a physical field is a 2D array (ny, nx)")
    with open(path, "w") as f:
        for row in a:
            f.write("".join(format_value(float(v)) + "," for v in row))
            f.write("\n")


def read_field(path: str, nx: Optional[int] = None, ny: Optional[int] = None) -> np.ndarray:
    """file_init: the (ny, nx) float64 field in `path`.

    Like the reference, a line's values are the comma-separated tokens up to
    the last comma or the end of the line (a trailing comma adds no value).
    Where the reference prints "no such file!" or "size not match!", this
    raises FileNotFoundError / ValueError."""
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    rows = []
    with open(path) as f:
        for line in f:
            line = line.rstrip("\n").rstrip("\r")
            toks = line.split(",")
            if toks and toks[-1] == "":
                toks = toks[:-1]
            rows.append([float(t) for t in toks])
    if not rows or any(len(r) != len(rows[0]) for r in rows):
        raise ValueError(f"{path}: rows of unequal length")
    a = np.asarray(rows, dtype=np.float64)
    if (ny is not None and a.shape[0] != ny) or (nx is not None and a.shape[1] != nx):
        raise ValueError(f"{path}: size {a.shape[1]} x {a.shape[0]} does not match the mesh {nx} x {ny}")
    return a


def load_state(mesh, directory: str = "init", names=("w_init.csv", "r1_init.csv", "r2_init.csv")):
    """The reference's start from CSV files: read w, r1, r2, FwdTrans each,
    make the spectra the mesh's resident state (Mesh.load) and return them."""
    import torch
    ny, nx = mesh.ny, mesh.nx
    spec = []
    for name in names:
        a = read_field(os.path.join(directory, name), nx, ny)
        spec.append(mesh.fwd_trans(torch.from_numpy(a).to("cuda", mesh.real_dtype).contiguous()))
    mesh.load(*spec)
    return tuple(spec)


def write_snapshot(mesh, step: int, directory: str = ".", spectra=None) -> list:
    """The reference's periodic output: {step}w.csv, {step}r1.csv, {step}r2.csv
    and {step}S.csv (S = 2 sqrt(r1^2 + r2^2), S_func) of the mesh's resident
    state, or of `spectra` = (w, r1, r2) when given. Returns the paths."""
    import torch
    w, r1, r2 = spectra if spectra is not None else mesh.store()
    pw, p1, p2 = (mesh.bwd_trans(x) for x in (w, r1, r2))
    S = 2 * torch.sqrt(p1 * p1 + p2 * p2)
    paths = []
    for name, f in (("w", pw), ("r1", p1), ("r2", p2), ("S", S)):
        path = os.path.join(directory, f"{step}{name}.csv")
        write_field(path, f)
        paths.append(path)
    return paths


def _host(field) -> np.ndarray:
    if isinstance(field, np.ndarray):
        return field.astype(np.float64, copy=False)
    try:
        import torch
        if isinstance(field, torch.Tensor):
            return field.detach().to("cpu", torch.float64).numpy()
    except ImportError:
        pass
    return np.asarray(field, dtype=np.float64)
