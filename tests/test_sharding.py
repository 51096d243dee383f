"""Multi-rank host logic on CPU: scenario sharding, instance balancing and the
result gather, run as two gloo ranks (the same code path the GPU ranks take,
with the oracle standing in for the device solve)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from cupf import grids as G
from cupf.sharding import balance_instances, gather_rows, instance_cost, scenario_shard


@pytest.mark.parametrize("total,world", [(0, 2), (1, 2), (7, 2), (1024, 8), (1000, 3), (5, 8)])
def test_scenario_shard_tiles(total, world):
    spans = [scenario_shard(total, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == total
    for (a, b), (c, _) in zip(spans, spans[1:]):
        assert b == c
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1


def test_scenario_shard_rejects_bad_rank():
    with pytest.raises(ValueError):
        scenario_shard(10, 2, 2)


def test_balance_uneven_batch():
    """The uneven multi-grid batch: 118/500/2,000/10,000 buses x 256/128/96/32."""
    inst = [(118, 256), (500, 128), (2000, 96), (10000, 32)]
    costs = [instance_cost(n, b) for n, b in inst for _ in range(1)]
    for world in (1, 2, 4):
        a = balance_instances(costs, world)
        assert sorted(i for r in a for i in r) == list(range(len(costs)))
    # deterministic
    assert balance_instances(costs, 2) == balance_instances(costs, 2)


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist
    from oracle.oracle import Oracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = G.grid_118()
        total = 10
        S = g.scenarios(total, seed=21)
        V0 = g.flat_start(total)
        a, b = scenario_shard(total, rank, world)
        r = Oracle().solve_many(g, S[a:b], V0[a:b], 1e-8, 10, 1)
        local = torch.from_numpy(np.ascontiguousarray(r["V"]).view(np.float64))
        full = gather_rows(local, world)
        if rank == 0:
            np.save(out_path, full.numpy())
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_equals_single_process(tmp_path):
    from oracle.oracle import Oracle

    out = tmp_path / "v.npy"
    mp.spawn(_rank_main, args=(2, _free_port(), str(out)), nprocs=2, join=True)
    got = np.load(out).view(np.complex128)
    g = G.grid_118()
    S = g.scenarios(10, seed=21)
    want = Oracle().solve_many(g, S, g.flat_start(10), 1e-8, 10, 1)["V"]
    assert np.array_equal(got, want)
