"""Cell-list neighbor build and configurations beyond the reference's size limit.

The reference scans all Na^2 pairs of a configuration in one CUDA block, so a
configuration holds at most 1024 atoms (neighbor.cu:30-66).  The engine builds
lists for large configurations from cell lists in O(N) (gpuga_options
neighbor_cells), with the same FP32 pair test and neighbor order, and gives
force configurations whose f_ij scratch does not fit shared memory a global
scratch.  Lists must be identical to the O(Na^2) scan and to the oracle, and
results identical between the two builds."""
import numpy as np
import pytest

from gpuga_b200 import PATH_PLAIN64, Fitness, synth
from tests.helpers import oracle_targets

pytestmark = pytest.mark.gpu


def _kw(data):
    return dict(nn2b_r1=float(data["nn2b_r1"]), nn2b_r2=float(data["nn2b_r2"])) if "nn2b_r1" in data else {}


@pytest.mark.parametrize("workload,Nc", [(1, 6), (2, 40), (3, 12), (4, 10)])
def test_cell_lists_equal_the_pair_scan(workload, Nc):
    data = synth.make(workload, Nc=Nc)
    with Fitness(arrays=data, neighbor_cells=2, **_kw(data)) as scan, \
            Fitness(arrays=data, neighbor_cells=1, **_kw(data)) as cells:
        a, b = scan.neighbors(), cells.neighbors()
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])
        pop = synth.population(data, 64, seed=5)
        np.testing.assert_array_equal(scan.compute(64, pop), cells.compute(64, pop))


@pytest.fixture(scope="module")
def large_set(built_oracle, tmp_path_factory):
    """4096-atom force and energy/virial configurations next to small ones; FP64 teacher targets."""
    data = synth.diamond_set([8, 2, 8, 3], Nc_force=2, seed=21, P=64)
    data = synth.fill_targets(data, oracle_targets(built_oracle))
    d = synth.write_dir(data, str(tmp_path_factory.mktemp("large")))
    return data, built_oracle.OracleSet(d)


def test_large_configuration_lists_match_the_oracle(large_set):
    data, s = large_set
    oNN, onl = s.neighbors()
    with Fitness(arrays=data) as e:  # automatic: cell lists for the 4096-atom configurations
        assert e.max_Na == 4096
        NN, nbr = e.neighbors()
        np.testing.assert_array_equal(NN, oNN)
        np.testing.assert_array_equal(nbr, onl)


def test_large_configuration_fitness_and_forces(large_set):
    data, s = large_set
    P = 64
    pop = synth.population(data, P, seed=9)
    with Fitness(arrays=data) as e:
        fit = e.compute(P, pop)
        fit64 = e.compute(P, pop, path=PATH_PLAIN64)
        np.testing.assert_allclose(fit, fit64, rtol=1e-6)
        assert np.array_equal(np.argsort(fit, kind="stable"), np.argsort(fit64, kind="stable"))
        # per-atom forces of the force configurations (4096-atom one through the global scratch)
        Fb = e.batched_forces(pop[:4])
        for k in range(4):
            F, _, _ = e.find_force64(s.decode(pop[k]))
            Nf = e.N_force
            want = np.stack([F[:Nf], F[e.N:e.N + Nf], F[2 * e.N:2 * e.N + Nf]])
            scale = np.abs(want).max()
            np.testing.assert_allclose(Fb[k], want, atol=2e-5 * scale, rtol=0)
        # the oracle's FP64 fitness of the first individuals
        np.testing.assert_allclose(fit[:4], s.fitness(pop[:4]), rtol=1e-6)
