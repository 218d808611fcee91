"""A run that moves between the reference and this library through the
reference's CSV snapshots: write_snapshot writes {step}w/r1/r2/S.csv of the
resident state; load_state starts a mesh from such files, as file_init +
FwdTrans do (InertialFriction/friction/friction.cu:164-185). The format keeps
6 significant digits, so the round trip holds to that."""
import math
import os

import numpy as np
import pytest
import torch

import oracle as O
import qaf
from qaf import csvio

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [qaf.F64, qaf.F32])
def test_snapshot_round_trip(cuda, tmp_path, dtype):
    n, L = 64, 16 * math.pi
    m = qaf.Mesh(n, lx=L, dtype=dtype)
    s0 = [torch.from_numpy(a).to("cuda", m.complex_dtype) for a in O.initial_spectra(2, n, lo=-0.5, hi=0.5)]
    m.load(*s0)
    m.advance(qaf.Params(), 20)
    paths = csvio.write_snapshot(m, 20, str(tmp_path))
    assert [os.path.basename(p) for p in paths] == ["20w.csv", "20r1.csv", "20r2.csv", "20S.csv"]
    w, r1, r2 = m.store()
    phys = [m.bwd_trans(x).cpu().numpy().astype(np.float64) for x in (w, r1, r2)]
    got = [csvio.read_field(p, n, n) for p in paths]
    for a, b in zip(got[:3], phys):
        assert np.all(np.abs(a - b) <= 5e-6 * np.abs(b) + 1e-30)
    S = 2 * np.sqrt(phys[1] ** 2 + phys[2] ** 2)
    assert np.allclose(got[3], S, rtol=1e-5, atol=0)

    # start a second mesh from the snapshot, as the reference's restart does.
    # A physical snapshot holds the Hermitian part of the spectra only: the
    # asymmetric 2/3 mask leaves the kx = 0 column non-Hermitian at ky = N/3
    # (its partner row is zeroed), a part that no C2R sees; the reference's
    # CSV restart drops it too.
    H = O.hermitian_part
    m2 = qaf.Mesh(n, lx=L, dtype=dtype)
    spec = csvio.load_state(m2, str(tmp_path), names=("20w.csv", "20r1.csv", "20r2.csv"))
    for a, b in zip(spec, (w, r1, r2)):
        a, b = H(a.cpu().numpy().astype(np.complex128)), H(b.cpu().numpy().astype(np.complex128))
        assert np.linalg.norm(a - b) <= 5e-6 * np.linalg.norm(b)
    # the restarted run is the oracle's run from the same files. (It is not
    # the uninterrupted run to 6 digits: with the partner row zeroed every
    # step, the (N/3, 0) mode's physical amplitude is half its stored value,
    # which the snapshot halves again; Mesh.save/restore restart exactly.)
    ref = O.step(O.params(n=n), *[O.fwd(f) for f in got[:3]], 10)
    m2.advance(qaf.Params(), 10)
    bar = 1e-12 if dtype == qaf.F64 else 1e-4
    for a, b in zip(m2.store(), ref):
        assert O.rel_l2(a.cpu().numpy().astype(np.complex128), b) < bar


def test_load_state_rejects_a_size_mismatch(cuda, tmp_path):
    for name in ("w_init.csv", "r1_init.csv", "r2_init.csv"):
        csvio.write_field(str(tmp_path / name), np.zeros((32, 32)))
    m = qaf.Mesh(64, lx=16 * math.pi, dtype=qaf.F64)
    with pytest.raises(ValueError):
        csvio.load_state(m, str(tmp_path))
