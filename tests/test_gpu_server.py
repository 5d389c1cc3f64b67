"""Serving loop: concurrent fitting jobs with continuous batching.

Each job's result must be the same alone and in the mix: the best-fitness
history and the final elite of a job run among others equal, bit for bit, the
same job run on its own engine with the GA alone (the batched kernels never
mix jobs inside a CTA and reduce in a fixed order)."""
import time

import numpy as np
import pytest

from gpuga_b200 import GA, Fitness, Server, _lib
from tests.helpers import synthetic_dir

pytestmark = pytest.mark.gpu

GENS = 6


@pytest.fixture(scope="module")
def job_dirs(built_oracle, tmp_path_factory):
    dirs = []
    # parent_number = P/2, a multiple of 10; the NN2B job (4) brings its per-pair scratch and pair
    # lists into the shared launch sets
    for cfg, Nc, P in [(1, 8, 40), (2, 12, 60), (3, 4, 20), (1, 6, 40), (4, 4, 20)]:
        d, data = synthetic_dir(built_oracle, cfg, Nc, str(tmp_path_factory.mktemp(f"job{cfg}_{Nc}")))
        with open(f"{d}/ga.in", "w") as f:
            f.write(f"maximum_generation 50\npopulation_size {P}\nparent_number {P // 2}\nmutation_rate 0.2\n")
        dirs.append(d)
    return dirs


def alone(d, seed):
    with Fitness(d) as e:
        ga = GA(e, input_dir=d, seed=seed)
        best = []
        for _ in range(GENS):
            ga.step()
            best.append(ga.state(_pop_size(d))[2][0])
        elite = ga.state(_pop_size(d))[1][0].copy()
        ga.close()
    return np.array(best, np.float32), elite


def _pop_size(d):
    for line in open(f"{d}/ga.in"):
        if line.startswith("population_size"):
            return int(line.split()[1])
    return 200


def test_jobs_are_the_same_alone_and_in_the_mix(job_dirs):
    refs = [alone(d, 1000 + k) for k, d in enumerate(job_dirs)]
    with Server(device=0, hbm_budget_bytes=120e9, max_jobs=32) as srv:
        srv.hold(True)  # load every job first, so that all of them share every window
        ids = [srv.submit(d, seed=1000 + k, generations=GENS) for k, d in enumerate(job_dirs)]
        deadline = time.time() + 120
        while any(srv.poll(j)[3] == Server.QUEUED for j in ids) and time.time() < deadline:
            time.sleep(0.01)
        srv.hold(False)
        assert srv.drain(300) == _lib.OK
        st = srv.stats()
        assert st["jobs_finished"] == len(job_dirs)
        assert st["peak_resident_jobs"] == len(job_dirs)  # all of them shared the launches
        assert st["batches"] == GENS
        assert st["p99_gen_ms"] >= st["p50_gen_ms"] > 0
        assert st["p99_wall_gen_ms"] >= st["p50_wall_gen_ms"] > 0
        assert st["p99_first_window_ms"] >= st["p50_first_window_ms"] > 0
        for jid, d, (best, elite) in zip(ids, job_dirs, refs):
            status, done, total, state = srv.poll(jid)
            assert (status, done, total, state) == (_lib.OK, GENS, GENS, Server.DONE)
            got_best, got_elite = srv.result(jid, GENS, elite.size)
            np.testing.assert_array_equal(got_best, best)
            np.testing.assert_array_equal(got_elite, elite)


def test_budget_admission_and_late_arrivals(job_dirs):
    """A budget that holds one job at a time serialises them; late arrivals still finish."""
    with Server(device=0, hbm_budget_bytes=2.5e8, max_jobs=8) as srv:
        ids = [srv.submit(job_dirs[0], seed=1, generations=GENS)]
        time.sleep(0.05)
        ids.append(srv.submit(job_dirs[1], seed=2, generations=GENS))
        ids.append(srv.submit(job_dirs[3], seed=3, generations=GENS))
        assert srv.drain(300) == _lib.OK
        for jid in ids:
            assert srv.poll(jid)[0] == _lib.OK
        assert srv.stats()["jobs_finished"] == 3


def test_over_budget_and_cancel(job_dirs):
    with Server(device=0, hbm_budget_bytes=1e6, max_jobs=4) as srv:
        with pytest.raises(_lib.GpugaError) as ei:
            srv.submit(job_dirs[1], generations=GENS)
        assert ei.value.status == _lib.ERR_BUDGET
    with Server(device=0, hbm_budget_bytes=120e9, max_jobs=1) as srv:
        first = srv.submit(job_dirs[0], seed=5, generations=40)
        queued = srv.submit(job_dirs[3], seed=6, generations=40)
        srv.cancel(queued)
        srv.cancel(first)
        assert srv.drain(300) == _lib.OK
        assert srv.poll(queued)[0] == _lib.ERR_CANCELLED
        assert srv.poll(first)[3] == Server.CANCELLED


def test_engine_jobs_share_one_training_set(job_dirs):
    """Two jobs on one engine (different seeds) run together and match their solo runs."""
    d = job_dirs[1]
    with Fitness(d) as e:
        solo = []
        for seed in (11, 12):
            # a server job of G generations runs the GA with maximum_generation = G
            ga = GA(e, seed=seed, population_size=40, parent_number=20, mutation_rate=0.2, maximum_generation=GENS)
            hist = []
            for _ in range(GENS):
                ga.step()
                hist.append(ga.state(40)[2][0])
            solo.append(np.array(hist, np.float32))
            ga.close()
        with Server(device=0) as srv:
            ids = [srv.submit_engine(e, 40, 20, 0.2, GENS, seed=s) for s in (11, 12)]
            assert srv.drain(300) == _lib.OK
            for jid, want in zip(ids, solo):
                got, _ = srv.result(jid, GENS, e.number_of_variables)
                np.testing.assert_array_equal(got, want)
