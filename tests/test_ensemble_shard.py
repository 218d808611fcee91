"""Ensemble sharding over ranks (host logic; CPU, gloo for world size 2)."""
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "nature-control_b200"))

from qaf.shard import draw_ensemble, gather_by_instance, instance_cost, rank_cost, shard_instances  # noqa: E402


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shard_covers_each_instance_once_and_balances(world):
    n, _, _, _ = draw_ensemble(256, 3)
    parts = shard_instances(n, world)
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(256))
    costs = [rank_cost(n, p) for p in parts]
    mean = sum(costs) / world
    assert max(costs) - mean <= instance_cost(max(n)) + 1e-9
    assert shard_instances(n, world) == parts          # deterministic


def test_shard_more_ranks_than_instances():
    parts = shard_instances([64, 256], 4)
    assert sorted(len(p) for p in parts) == [0, 0, 1, 1]
    assert parts[0] == [1]                             # the largest goes first, to rank 0


def test_draw_is_seeded_and_in_range():
    a = draw_ensemble(64, 11)
    b = draw_ensemble(64, 11)
    assert a == b
    n, al, rf, seeds = a
    assert set(n) <= {64, 128, 256}
    assert all(0.5 <= v < 2.0 for v in al) and all(0.01 <= v < 0.5 for v in rf)
    assert len(set(seeds)) == 64


def test_gather_single_process():
    assert gather_by_instance([2, 0, 1], ["c", "a", "b"], 3) == ["a", "b", "c"]
    with pytest.raises(ValueError):
        gather_by_instance([0, 0], [1, 2], 2)
    with pytest.raises(ValueError):
        gather_by_instance([0], [1], 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, sizes, seeds, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    os.environ["QAF_ORACLE_THREADS"] = "1"
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = shard_instances(sizes, world)[rank]
        vals = []
        for k in mine:
            p = O.params(n=sizes[k], dt=1e-3)
            w, r1, r2 = O.step(p, *O.initial_spectra(seeds[k], sizes[k]), 2)
            vals.append(float(abs(w).sum() + abs(r1).sum()))
        out = gather_by_instance(mine, vals, len(sizes))
        q.put((rank, mine, out))
    finally:
        dist.destroy_process_group()


def test_sharded_ensemble_two_gloo_ranks():
    """Two CPU ranks each step their shard with the oracle; the gathered table equals one process's."""
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    sizes = [16, 32, 16, 32, 16]
    seeds = [5, 6, 7, 8, 9]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, sizes, seeds, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert sorted(res[0][1] + res[1][1]) == list(range(5))
    assert res[0][2] == res[1][2]
    want = []
    for k in range(5):
        p = O.params(n=sizes[k], dt=1e-3)
        w, r1, r2 = O.step(p, *O.initial_spectra(seeds[k], sizes[k]), 2)
        want.append(float(abs(w).sum() + abs(r1).sum()))
    assert res[0][2] == want
