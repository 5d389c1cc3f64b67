"""Multi-rank path on CPU (gloo, world size 2): individuals are sharded across
ranks with no data-path collective; gathering the shards reproduces the
single-process evaluation, and the timing reduction takes the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from tests.helpers import synthetic_dir


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, d, pop, out_dir):
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle import oracle
    s = oracle.OracleSet(d)
    shard = np.array_split(np.arange(len(pop)), world)[rank]
    fit = torch.tensor(s.fitness(pop[shard]))
    sizes = [len(x) for x in np.array_split(np.arange(len(pop)), world)]
    gathered = [torch.zeros(n, dtype=torch.float64) for n in sizes]
    dist.all_gather(gathered, fit)
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        np.save(os.path.join(out_dir, "fit.npy"), torch.cat(gathered).numpy())
        np.save(os.path.join(out_dir, "tmax.npy"), t.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_population_equals_single_process(tmp_path, built_oracle):
    d, data = synthetic_dir(built_oracle, 2, 8, str(tmp_path / "set"))
    pop = np.random.default_rng(0).uniform(0, 1, size=(10, 9)).astype(np.float32)
    mp.start_processes(_worker, args=(2, _free_port(), d, pop, str(tmp_path)), nprocs=2, start_method="spawn")
    fit = np.load(tmp_path / "fit.npy")
    want = built_oracle.OracleSet(d).fitness(pop)
    np.testing.assert_array_equal(fit, want)
    assert float(np.load(tmp_path / "tmax.npy")[0]) == 2.0


def _bench_worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import bench
    d = bench.Dist(backend="gloo")
    d.barrier()
    # rank r timed its K = 4 steps at (r + 1) ms each: the job took the slowest rank's 8 ms
    value, ms = bench.whole_job_rate(d, 1000.0, [float(rank + 1)] * 4)
    if rank == 0:
        np.save(os.path.join(out_dir, "rate.npy"), np.array([value, ms, d.world]))
    d.barrier()
    d.close()


def test_bench_dist_aggregation(tmp_path):
    """bench.py's multi-rank plumbing (the Dist barrier and max-over-ranks timer, the whole-job
    rate) on two gloo ranks."""
    mp.start_processes(_bench_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    value, ms, world = np.load(tmp_path / "rate.npy")
    assert world == 2
    assert ms == 2.0                                 # slowest rank: 4 steps x 2 ms
    assert value == 2 * 1000.0 * 4 / (8.0 / 1e3)     # both ranks' units over the slowest rank's time
