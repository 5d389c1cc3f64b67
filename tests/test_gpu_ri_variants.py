"""RI extensions on the GPU against the oracle: potential type 4 (anion charge -q) and the
opt-in damped-Coulomb self energy (gpuga_options.ri_self_energy).

Tolerances as in the main parity file: FP64 path 1e-9 of each quantity's scale; batched
fitness relative 1e-6 per individual with the FP64 ranking; per-config energies 2e-6 of the
set's energy scale.  Type 0 with the self energy off is the reference's ri.cu and is covered
there; here every other combination, plus the statement that switching the self energy on
changes energies only."""
import numpy as np
import pytest

from gpuga_b200 import PATH_BATCHED, PATH_PLAIN64, Fitness, synth
from tests.helpers import oracle_targets

pytestmark = pytest.mark.gpu

FIT_RTOL = 1e-6
MODES = [(4, False), (0, True), (4, True)]


@pytest.fixture(scope="module")
def ri_sets(built_oracle, tmp_path_factory):
    cache = {}

    def get(pt, self_on):
        if (pt, self_on) not in cache:
            data = synth.make(3, Nc=10)
            data["potential_type"] = pt
            data["ri_self_energy"] = self_on
            data = synth.fill_targets(data, oracle_targets(built_oracle))
            d = synth.write_dir(data, str(tmp_path_factory.mktemp(f"ri{pt}{int(self_on)}")))
            s = built_oracle.OracleSet(d)
            s.set_ri_self(self_on)
            cache[(pt, self_on)] = (d, s, data)
        return cache[(pt, self_on)]

    return get


@pytest.mark.parametrize("pt,self_on", MODES)
def test_fp64_path_matches_oracle(ri_sets, pt, self_on):
    d, s, _ = ri_sets(pt, self_on)
    with Fitness(d, ri_self_energy=self_on) as e:
        assert e.potential_type == pt
        rng = np.random.default_rng(pt)
        p = s.decode(rng.uniform(0, 1, size=15).astype(np.float32))
        F, W, pe = e.find_force64(p)
        oF, oW, ope = s.find_force(p)
        for a, b in ((F, oF), (W, oW), (pe, ope)):
            assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max()
        pop = rng.uniform(0, 1, size=(5, 15)).astype(np.float32)
        np.testing.assert_allclose(e.compute(5, pop, path=PATH_PLAIN64), s.fitness(pop), rtol=1e-9)


@pytest.mark.parametrize("pt,self_on", MODES)
def test_batched_fitness_and_energies_match_oracle(ri_sets, pt, self_on):
    d, s, data = ri_sets(pt, self_on)
    P = 45
    pop = np.vstack([data["teacher01"][None, :], synth.population(data, P - 1, seed=13)])
    with Fitness(d, ri_self_energy=self_on) as e:
        fit = e.compute(P, pop, path=PATH_BATCHED)
        ofit = s.fitness(pop)
        rel = np.abs(fit - ofit) / np.abs(ofit)
        assert rel[1:].max() <= FIT_RTOL
        assert fit[0] < 1e-3 * np.median(fit[1:])  # the teacher reproduces the targets it made
        order, oorder = np.argsort(fit[1:], kind="stable"), np.argsort(ofit[1:], kind="stable")
        assert np.array_equal(order, oorder)
        E, _, _ = e.config_results(P)
        Ncf = s.Nc_force
        for p in (0, 1, P - 1):
            oF, oW, ope = s.find_force(s.decode(pop[p]))
            oE, _ = s.config_sums(oW, ope)
            assert np.abs(E[p, Ncf:] - oE[Ncf:]).max() <= 2e-6 * np.abs(oE[Ncf:]).max()


def test_self_energy_changes_energies_only(ri_sets):
    """Forces and virials of the batched path are bit-identical with the self energy on or off;
    the energies differ by the FP64 self term -K_C q^2 S(rc) sum_i (q_i / q)^2."""
    d, s, data = ri_sets(4, True)
    pop = synth.population(data, 33, seed=3)
    with Fitness(d, ri_self_energy=False) as off, Fitness(d, ri_self_energy=True) as on:
        off.compute(33, pop)
        on.compute(33, pop)
        E0, W0, F0 = off.config_results(33)
        E1, W1, F1 = on.config_results(33)
        np.testing.assert_array_equal(W0, W1)
        np.testing.assert_array_equal(F0, F1)
        np.testing.assert_array_equal(off.batched_forces(pop[:4]), on.batched_forces(pop[:4]))
        qsum = data["Na"].astype(np.float64)  # type 4: every ion carries |q|
        alpha, kc = 0.2, 14.399645
        from math import erfc, exp, pi, sqrt
        Ncf = s.Nc_force
        for p in (0, 17, 32):
            prm = s.decode(pop[p])
            rc = prm[10]
            S = alpha / sqrt(pi) + erfc(alpha * rc) / rc + alpha / sqrt(pi) * exp(-alpha * alpha * rc * rc)
            want = -kc * prm[0] ** 2 * S * qsum
            np.testing.assert_allclose(E1[p, Ncf:] - E0[p, Ncf:], want[Ncf:], rtol=1e-9)
