"""Launch-shape autotuner: the cache format and the names (CPU), and every
launch variant against the built-in shapes (GPU)."""
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "nature-control_b200"))

import qaf  # noqa: E402


def _lib_or_skip():
    if not os.path.exists(qaf.LIB_PATH):
        pytest.skip("libqaf.so is not built")
    return qaf.lib()


@pytest.fixture
def fresh_table():
    _lib_or_skip()
    qaf.autotune_reset()
    yield
    qaf.autotune_reset()


def test_variant_names(fresh_table):
    names = qaf.variant_list(256, qaf.F32)
    assert names[:2] == ["col:default", "row:default"]
    assert "col:e16" in names and "row:e8r2" in names
    assert qaf.variant_list(256, qaf.F64) == ["col:default", "row:default"]
    assert qaf.variant_choice(256, qaf.F32, False) == "col:default row:default"
    qaf.set_variant(256, qaf.F32, True, "col:e16", "row:e8r2")
    assert qaf.variant_choice(256, qaf.F32, True) == "col:e16 row:e8r2"
    assert qaf.variant_choice(256, qaf.F32, False) == "col:default row:default"
    with pytest.raises(qaf.QafError):
        qaf.set_variant(256, qaf.F32, False, "col:e99", "default")
    with pytest.raises(qaf.QafError):
        qaf.set_variant(256, qaf.F64, False, "col:e16", "default")


def test_cache_load_applies_matching_records(fresh_table, tmp_path):
    path = tmp_path / "tune.jsonl"
    path.write_text(
        '{"device": "*", "dtype": "f32", "n": 128, "batched": 1, "col": "col:e16", "row": "row:e16r8", "us_per_step": 12.5}\n'
        '{"device": "some other GPU", "dtype": "f32", "n": 64, "batched": 0, "col": "col:e4", "row": "row:default", "us_per_step": 3}\n'
        '{"device": "*", "dtype": "f32", "n": 256, "batched": 0, "col": "col:e77", "row": "row:default", "us_per_step": 1}\n'
        'not json at all\n')
    qaf.autotune_load(str(path))
    assert qaf.variant_choice(128, qaf.F32, True) == "col:e16 row:e16r8"
    assert qaf.variant_choice(64, qaf.F32, False) == "col:default row:default"     # other device
    assert qaf.variant_choice(256, qaf.F32, False) == "col:default row:default"    # unknown shape
    with pytest.raises(qaf.QafError):
        qaf.autotune_load(str(tmp_path / "missing.jsonl"))


def _rel(a, b):
    import torch
    return (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [64, 128, 256, 1024])
def test_every_variant_matches_builtin_shapes(cuda, fresh_table, n):
    """Single meshes and batched groups, every column and row shape, against the built-in ones (FP32)."""
    import torch
    L = 16 * 3.141592653589793
    p = qaf.Params(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=1e-3)
    steps = 3 if n < 1024 else 1
    m = qaf.Mesh(n, n, L, L, qaf.F32)
    s0 = m.random_q(5)
    m.load(*s0)
    m.advance(p, steps)
    ref = m.store()
    names = qaf.variant_list(n, qaf.F32)
    cols = [x for x in names if x.startswith("col:")]
    rows = [x for x in names if x.startswith("row:")]
    for c in cols:
        for r in rows:
            qaf.set_variant(n, qaf.F32, False, c, r)
            m.load(*s0)
            m.advance(p, steps)
            for got, want in zip(m.store(), ref):
                assert _rel(got, want) <= 1e-5, (c, r)
    if n <= 256:
        for c in cols:
            for r in rows:
                qaf.set_variant(n, qaf.F32, True, c, r)
                ens = qaf.Ensemble([n, n, n], p, [1.0, 1.0, 1.0], [0.1, 0.1, 0.1], lx=L, dtype=qaf.F32)
                for k in range(3):
                    ens.load(k, *s0)
                ens.advance(steps)
                for k in range(3):
                    for got, want in zip(ens.store(k), ref):
                        assert _rel(got, want) <= 1e-5, (c, r, k)
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_autotune_records_and_reloads(cuda, fresh_table, tmp_path):
    path = str(tmp_path / "tune.jsonl")
    choice, us = qaf.autotune(128, qaf.F32, 6, path)
    assert us > 0 and choice.startswith("col:") and " row:" in choice
    assert qaf.variant_choice(128, qaf.F32, True) == choice
    text = open(path).read()
    assert '"n": 128' in text and '"batched": 1' in text
    choice, _ = qaf.autotune(128, qaf.F32, 6, path)  # same key: replaced, not appended (near-ties may flip)
    assert open(path).read().count('"n": 128') == 1
    qaf.autotune_reset()
    assert qaf.variant_choice(128, qaf.F32, True) == "col:default row:default"
    qaf.autotune_load(path)
    assert qaf.variant_choice(128, qaf.F32, True) == choice
    choice64, _ = qaf.autotune(64, qaf.F64, 1, None)  # FP64 has the built-in shapes only
    assert choice64 == "col:default row:default"


@pytest.mark.gpu
def test_tuned_ensemble_matches_untuned(cuda, fresh_table, tmp_path):
    L = 16 * 3.141592653589793
    p = qaf.Params(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=1e-3)
    sizes = [64, 128, 64, 256]
    a = qaf.Ensemble(sizes, p, [1.0] * 4, [0.1] * 4, lx=L, dtype=qaf.F32)
    b = qaf.Ensemble(sizes, p, [1.0] * 4, [0.1] * 4, lx=L, dtype=qaf.F32, tune=True,
                     tune_cache=str(tmp_path / "t.jsonl"))
    for e in (a, b):
        e.init_random([1, 2, 3, 4])
        e.advance(4)
    for k in range(4):
        for x, y in zip(b.store(k), a.store(k)):
            assert _rel(x, y) <= 1e-5
