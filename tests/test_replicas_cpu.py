"""The replica (N > 1) path on CPU: two gloo ranks shard a set of catalogs,
compute each one's power-spectrum multipoles independently, and the gathered
results equal the serial run; the MAX-over-ranks timing reduction and the
whole-job rate are checked on the same process group."""
import os
import socket

import numpy as np
import pytest

from cosmonpc_b200 import replicas


def test_shard_covers_units_once():
    for n_units in (0, 1, 5, 8, 13):
        for world in (1, 2, 3, 8):
            got = [i for r in range(world) for i in replicas.shard(n_units, r, world)]
            assert got == list(range(n_units))
            sizes = [len(replicas.shard(n_units, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def _catalog(seed, n=3000, L=500.0):
    return np.random.default_rng(seed).uniform(0.0, L, size=(n, 3))


def _pk(seed):
    from oracle.box import paint_field, _fwd, KGeom

    L, n = 500.0, 16
    pos = _catalog(seed, L=L)
    c = _fwd(paint_field(pos, np.ones(len(pos)), n, L, "cic", True))
    geo = KGeom(n, L)
    edges = np.linspace(0.02, 0.18, 5)
    out = []
    for ell in (0, 2):
        mu = np.nan_to_num(geo.khat[2])
        leg = 0.5 * (3.0 * mu * mu - 1.0) if ell else 1.0
        p = (np.abs(c) ** 2 * leg).real
        idx = np.digitize(geo.knorm, edges) - 1
        out.append([p[idx == b].mean() for b in range(len(edges) - 1)])
    return np.array(out)


def _rank_main(rank, world, port, n_units, base_seed, q):
    try:
        _rank_body(rank, world, port, n_units, base_seed, q)
    except BaseException as e:  # report to the parent instead of leaving it waiting
        q.put(("error", rank, repr(e)))
        raise


def _rank_body(rank, world, port, n_units, base_seed, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = {u: _pk(replicas.unit_seed(base_seed, u)) for u in replicas.shard(n_units, rank, world)}
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t = replicas.max_over_ranks(0.5 + rank)
        if rank == 0:
            merged = {}
            for d in gathered:
                merged.update(d)
            q.put((merged, t, replicas.job_rate(len(mine), t, world)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_equal_serial():
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    n_units, base_seed, world = 5, 20261208, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n_units, base_seed, q)) for r in range(world)]
    for p in procs:
        p.start()
    msg = q.get(timeout=240)
    assert msg[0] != "error", msg
    merged, t, rate = msg
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(merged) == list(range(n_units))
    for u in range(n_units):
        np.testing.assert_array_equal(merged[u], _pk(replicas.unit_seed(base_seed, u)))
    assert t == 1.5  # the slowest rank
    assert rate == pytest.approx(3 * 2 / 1.5)
