"""Host logic of the batched ensemble (C5), on CPU: the seeded member draw, the shard plan over ranks, and the
metric gather over a world-size-2 gloo process group (the ensemble's only collective)."""
import os
import socket

import numpy as np
import pytest

from outbreaklab_b200 import ensemble as E, sounding as S, workloads as W


def test_members_follow_the_configuration():
    cs = E.draw_members(24, 5)
    assert len(cs) == 24
    for c in cs:
        assert 128 <= c.nx <= 384 and 128 <= c.ny <= 320 and c.nx % 8 == 0 and c.ny % 8 == 0
        assert c.dx in (1000.0, 1500.0, 2000.0) and c.dt == 6.0 * c.dx / 1000.0 and c.nz == 40 and c.scheme == 1
        assert 10.0 <= c.wk["shear_u"] <= 35.0
        a = S.analyze(S.parse_sharppy(W.weisman_klemp_sharppy(**c.wk)))
        assert 1500.0 <= a.P["mlcape"] <= 4000.0
        for (x, y) in c.bubbles:
            assert 0 < x < c.nx * c.dx and 0 < y < c.ny * c.dx
    again = E.draw_members(24, 5)
    assert [(c.nx, c.ny, c.dx, c.wk) for c in cs] == [(c.nx, c.ny, c.dx, c.wk) for c in again]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shard_plan_covers_and_balances(world):
    cs = E.draw_members(24, 5)
    plan = E.plan_shards(cs, world)
    flat = sorted(i for p in plan for i in p)
    assert flat == list(range(24))
    loads = [sum(cs[i].cells for i in p) for p in plan]
    # greedy largest-first: the spread is at most the largest member
    assert max(loads) - min(loads) <= max(c.cells for c in cs)


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as td
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world)
    local = {"cells": 1000 * (rank + 1), "steps": 10, "device_ms": 5.0 + rank,
             "latency_ms_all": [[1.0 + rank, 2.0 + rank, 3.0 + rank]] * (rank + 1)}
    res = E.gather(local, (torch, td))
    out.put((rank, res))
    td.destroy_process_group()


def test_gather_over_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        g = res[r]
        assert g["ranks"] == 2
        # total cell-steps (1000*10 + 2000*10) over the slowest rank's 6 ms
        assert np.isclose(g["cell_steps_per_s"], 30000 / 0.006)
        lat = np.array([1, 2, 3] + [2, 3, 4] * 2, float)
        assert np.isclose(g["latency_ms_p50"], np.percentile(lat, 50))
        assert np.isclose(g["latency_ms_p99"], np.percentile(lat, 99))


def test_tile_cache_roundtrip(tmp_path):
    from outbreaklab_b200 import ensemble as E
    cs = E.draw_members(3, seed=2)
    c = E.TileCache(str(tmp_path / "sub" / "tiles.json"))
    sig = E.TileCache.signature(cs, "B200")
    assert c.get(sig) is None
    c.put(sig, [64, 32, 32, 128, 16, 128], [0.1, 0.2, 0.3, 0.05, 0.07, 1.5])
    assert c.get(sig) == [64, 32, 32, 128, 16, 128]
    # another member set or device has its own entry
    assert c.get(E.TileCache.signature(cs[:2], "B200")) is None
    assert c.get(E.TileCache.signature(cs, "H100")) is None
    c.put(E.TileCache.signature(cs[:2], "B200"), [32] * 5 + [256], [1.0] * 6)
    assert c.get(sig) == [64, 32, 32, 128, 16, 128]
    # an unreadable file is an empty cache
    with open(c.path, "w") as f:
        f.write("{not json")
    assert c.get(sig) is None
