"""The engine's multi-rank path on one GPU: individuals are sharded across two ranks (processes),
each rank evaluates its shard with its own engine on cuda:0, and the fitness values are gathered
over a gloo process group (the path that bench.py --gpus N takes, one rank per GPU, with no
data-path collective).  The ranks' kernels never wait on one another -- they only share the GPU --
so this is a plain two-process run.  Gathering the shards must reproduce the single-process
evaluation bit for bit (work items never mix individuals' sums, and every reduction is in a fixed
order), and bench.py's whole-job rate takes the slowest rank's time.
Reference: the reference evaluates one population per process (fitness.cu:316-333)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from gpuga_b200 import PATH_BATCHED, Fitness, synth

pytestmark = pytest.mark.gpu

P = 45


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _data():
    data = synth.make(2, Nc=24, seed=17)
    with Fitness(arrays=data) as e0:
        return synth.fill_targets(data, lambda _d, p: e0.find_force64(p))


def _worker(rank, world, port, data, pop, out_dir):
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import bench
    d = bench.Dist(backend="gloo")
    shards = np.array_split(np.arange(len(pop)), world)
    mine = shards[rank]
    with Fitness(arrays=data, device=0) as e:
        fit = np.asarray(e.compute(len(mine), pop[mine], path=PATH_BATCHED), dtype=np.float64)
    # gloo gathers equal sizes: every shard padded to the largest, trimmed afterwards
    width = max(len(s) for s in shards)
    padded = torch.full((width,), float("nan"), dtype=torch.float64)
    padded[:len(mine)] = torch.from_numpy(fit.copy())
    gathered = [torch.zeros(width, dtype=torch.float64) for _ in shards]
    dist.all_gather(gathered, padded)
    gathered = [g[:len(s)] for g, s in zip(gathered, shards)]
    # the whole-job rate over the slowest rank's time, as bench.py reports it
    value, ms = bench.whole_job_rate(d, float(len(mine)), [float(rank + 1)])
    if rank == 0:
        np.save(os.path.join(out_dir, "fit.npy"), torch.cat(gathered).numpy())
        np.save(os.path.join(out_dir, "rate.npy"), np.array([value, ms]))
    d.barrier()
    d.close()


def test_sharded_engine_equals_single_process(tmp_path):
    data = _data()
    pop = synth.population(data, P, seed=9)
    mp.start_processes(_worker, args=(2, _free_port(), data, pop, str(tmp_path)), nprocs=2, start_method="spawn")
    got = np.load(tmp_path / "fit.npy")
    with Fitness(arrays=data, device=0) as e:
        want = np.asarray(e.compute(P, pop, path=PATH_BATCHED))
    assert np.array_equal(got, want)
    value, ms = np.load(tmp_path / "rate.npy")
    assert ms == 2.0  # the slower rank's time
