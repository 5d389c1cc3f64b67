"""The engine's GA (host C++, libgpuga_b200.so) against the oracle's restatement of
ga.cu:27-212, both driven by the same fitness, must print identical ga.out lines."""
import numpy as np
import pytest

from gpuga_b200 import GA


def _fitness_fn(pmin, pmax):
    target = np.linspace(0.1, 0.9, len(pmin)).astype(np.float32)

    def f(pop):
        return np.sum((pop - target) ** 2, axis=1).astype(np.float32)
    return f


@pytest.mark.parametrize("d,P,parents,rate,G", [(9, 40, 20, 0.2, 25), (13, 200, 100, 0.2, 12), (15, 60, 30, 1.0, 8)])
def test_host_ga_matches_oracle_ga(d, P, parents, rate, G, built_oracle):
    pmin = np.linspace(-1, 1, d).astype(np.float32)
    pmax = pmin + np.linspace(0.5, 2.0, d).astype(np.float32)
    fn = _fitness_fn(pmin, pmax)
    text, final = built_oracle.ga_run(d, pmin, pmax, P, parents, rate, 1000, G, 12345678, fn)
    ga = GA(host_callback=fn, num_vars=d, pmin=pmin, pmax=pmax, population_size=P, parent_number=parents,
            mutation_rate=rate, maximum_generation=1000, seed=12345678)
    lines = [ga.step() for _ in range(G)]
    assert "".join(lines) == text
    gen, pop, fit = ga.state(P)
    assert gen == G
    np.testing.assert_array_equal(pop.reshape(-1), final.reshape(-1))


def test_ga_with_nan_fitness_keeps_order(built_oracle):
    """NaN fitness values never move in the insertion sort (ga.cu:110)."""
    d, P = 9, 20
    pmin = np.zeros(d, np.float32)
    pmax = np.ones(d, np.float32)

    def fn(pop):
        f = np.sum(pop, axis=1).astype(np.float32)
        f[::3] = np.nan
        return f
    text, _ = built_oracle.ga_run(d, pmin, pmax, P, 10, 0.2, 100, 5, 7, fn)
    ga = GA(host_callback=fn, num_vars=d, pmin=pmin, pmax=pmax, population_size=P, parent_number=10,
            mutation_rate=0.2, maximum_generation=100, seed=7)
    assert "".join(ga.step() for _ in range(5)) == text


def test_mutation_never_touches_the_elite(built_oracle):
    d, P = 9, 40
    pmin = np.zeros(d, np.float32)
    pmax = np.ones(d, np.float32)
    ga = GA(host_callback=lambda pop: np.arange(len(pop), dtype=np.float32), num_vars=d, pmin=pmin, pmax=pmax,
            population_size=P, parent_number=20, mutation_rate=1.0, maximum_generation=10, seed=3)
    ga.step()
    _, pop0, _ = ga.state(P)
    elite = pop0[0].copy()
    ga.step()
    _, pop1, _ = ga.state(P)
    np.testing.assert_array_equal(pop1[0], elite)
