"""Multi-rank host logic on CPU process groups (gloo, world size 2): the model
partition, the max/sum reductions of the benchmark, and that sharding the
models over ranks changes no result (models are independent)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from openturbine_b200 import sharding as S


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_is_balanced_and_complete():
    rng = np.random.default_rng(3)
    nodes = rng.integers(5, 22, size=200)
    costs = [S.beam_cost(int(n), int(n) + 2) for n in nodes]
    for world in (1, 2, 4, 8):
        parts = S.partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(200))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-9
    assert S.partition(costs, 3) == S.partition(costs, 3)


def _worker(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle.oracle_py import OracleModel, run_batch
    from openturbine_b200 import workloads as W
    draws = W.draw_batch(12, first_id=4000)
    costs = [S.beam_cost(d.num_nodes, d.num_nodes + 2) for d in draws]
    mine = S.partition(costs, world)[rank]
    models = [OracleModel(W.batch_cantilever_model(draws[i]).pack()) for i in mine]
    conv, _, _ = run_batch(models, W.batch_params(), 3, [draws[i].amp for i in mine],
                           [draws[i].freq for i in mine], 1)
    q = {i: m.state("q") for i, m in zip(mine, models)}
    gathered = [None] * world
    dist.all_gather_object(gathered, q)
    total = S.sum_over_ranks(conv, dist)
    tmax = S.max_over_ranks(float(rank + 1), dist)
    if rank == 0:
        merged = {}
        for g in gathered:
            merged.update(g)
        np.savez(out_path, total=total, tmax=tmax,
                 **{f"q{i}": merged[i] for i in sorted(merged)})
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_oracle_equals_single_process(tmp_path):
    out = str(tmp_path / "ranks.npz")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    res = np.load(out)
    assert res["tmax"] == 2.0
    from oracle.oracle_py import OracleModel, run_batch
    from openturbine_b200 import workloads as W
    draws = W.draw_batch(12, first_id=4000)
    models = [OracleModel(W.batch_cantilever_model(d).pack()) for d in draws]
    conv, _, _ = run_batch(models, W.batch_params(), 3, [d.amp for d in draws],
                           [d.freq for d in draws], 1)
    assert res["total"] == conv
    for i, m in enumerate(models):
        np.testing.assert_array_equal(res[f"q{i}"], m.state("q"))


def _bench_worker(rank, world, port, out_path):
    """The benchmark's own multi-rank pieces on gloo: each rank takes its weak-
    scaling batch (bench.rank_draws), advances it on the oracle and reduces its
    timed region and converged beam-steps with bench.job_rate, as bench.py does
    with NCCL under torchrun."""
    import sys
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    import bench
    from oracle.oracle_py import OracleModel, run_batch
    from openturbine_b200 import workloads as W
    draws = bench.rank_draws(rank, 6, nodes=7)
    models = [OracleModel(W.batch_cantilever_model(d).pack()) for d in draws]
    conv, _, _ = run_batch(models, W.batch_params(), 2, [d.amp for d in draws],
                           [d.freq for d in draws], 1)
    local_ms = 10.0 * (rank + 1)          # a stand-in timed region per rank
    t_ms, units, rate = bench.job_rate(local_ms, conv, dist)
    ids = [d.model_id for d in draws]
    gathered = [None] * world
    dist.all_gather_object(gathered, (ids, conv))
    if rank == 0:
        np.savez(out_path, t_ms=t_ms, units=units, rate=rate,
                 ids=np.array([i for g in gathered for i in g[0]]),
                 convs=np.array([g[1] for g in gathered]))
    dist.barrier()
    dist.destroy_process_group()


def test_bench_multirank_reduction_and_shards(tmp_path):
    out = str(tmp_path / "bench_ranks.npz")
    mp.spawn(_bench_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    res = np.load(out)
    # the slowest rank's time, the units of every rank, their ratio
    assert res["t_ms"] == 20.0
    assert res["units"] == res["convs"].sum()
    assert res["rate"] == res["convs"].sum() / 0.02
    # weak scaling: each rank has its own batch, no model twice
    assert sorted(res["ids"].tolist()) == list(range(12))
