"""Multi-process ensemble logic on CPU (gloo, world size 2): every rank takes
its cost-balanced shard of the cells and the per-cell results are gathered on
every rank, with no collective inside the step."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sides, out_q):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    import conftest  # noqa: F401  (puts the package on sys.path)
    import torch.distributed as dist

    from pf_kks_gpu.ensemble import cell_cost, gather_results, partition

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [cell_cost(n, n, 10) for n in sides]
        shard = partition(costs, world)[rank]
        # stand-in for the per-cell GPU run: a value that identifies the cell and its rank
        local = {i: {"rank": rank, "side": sides[i]} for i in shard}
        merged = gather_results(local)
        out_q.put((rank, shard, merged))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_shard_and_gather():
    sides = [128, 192, 256, 384, 512, 256, 128, 512]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sides, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=90) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    shards = {r: s for r, s, _ in results}
    assert sorted(shards[0] + shards[1]) == list(range(len(sides)))
    assert not set(shards[0]) & set(shards[1])
    for _, _, merged in results:
        assert sorted(merged) == list(range(len(sides)))
        for i, v in merged.items():
            assert v["side"] == sides[i] and i in shards[v["rank"]]


class _FakeEnsemble:
    """CPU stand-in for pf_kks_gpu.ensemble.Ensemble: a cell 'advances' by
    recording its step count; results() reports it like the real class."""

    def __init__(self, members, precision="mixed", device=0, tune=False):
        self.sides = [cfg.nx for cfg, _ in members]
        self.tags = [state for _, state in members]
        self.steps = [0] * len(members)

    def run(self, n_steps):
        self.steps = [a + b for a, b in zip(self.steps, n_steps)]
        return [0] * len(self.steps)

    def results(self, fields=False):
        return [{"status": 0, "istep": k, "side": n, "tag": t} for k, n, t in zip(self.steps, self.sides, self.tags)]

    def close(self):
        pass


def _sharded_worker(rank, world, port, sides, out_q):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    import conftest  # noqa: F401
    import torch.distributed as dist

    from pf_kks_gpu.ensemble import run_sharded
    from pf_kks_gpu.workloads import base_config

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        built = []

        def lazy(i):
            def make():
                built.append(i)
                return f"state{i}"
            return make

        members = [(base_config(nx=n, ny=n), lazy(i)) for i, n in enumerate(sides)]
        steps = [10 + i for i in range(len(sides))]
        merged, shard, status = run_sharded(members, steps, make_ensemble=_FakeEnsemble)
        out_q.put((rank, shard, sorted(built), merged, status))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_run_sharded_two_ranks():
    """run_sharded: each rank builds and runs only its shard (the lazy
    states of the other rank's cells are never made), and every rank ends
    with every cell's result, each from the rank that ran it."""
    sides = [128, 192, 256, 384, 512, 256, 128]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, world, port, sides, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=90) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    shards = {r: s for r, s, _, _, _ in results}
    assert sorted(shards[0] + shards[1]) == list(range(len(sides)))
    for rank, shard, built, merged, status in results:
        assert built == sorted(shard)
        assert status == [0] * len(shard)
        assert sorted(merged) == list(range(len(sides)))
        for i, r in merged.items():
            assert r["side"] == sides[i] and r["tag"] == f"state{i}" and r["istep"] == 10 + i
            assert i in shards[r["rank"]]
