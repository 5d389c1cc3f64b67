"""Fitness precision of the batched FP32 path against the FP64 path, on populations large enough
to see the tail of the error distribution.

The FP32 rounding of a derived per-individual constant (the bond-order exponent -1/(2n), the
pair-set factors sqrt(2S) A, D0/(S-1), ...) is the same for every bond of that individual, so it
does not average out over the thousands of bonds of a configuration; near equilibrium it reaches
the virial amplified by the cancellation in fr' - b fa'.  The batched kernels carry the FP64
remainders of these constants.  Targets (stated here, checked below):
  * the benchmark's minimal-Tersoff Si set (500 configurations, S fixed at 2): relative fitness
    error <= 1e-6 for every one of 400 random individuals (measured 1.4e-7; smaller sets of the
    same kind have shown tails up to 1.5e-6, individuals near the optimum up to 1.7e-6);
  * S free in [1.5, 2.5] (the reference's wurtzite examples): <= 2e-5; what remains there is the
    FP32 evaluation of fr, fa, b and of the force assembly (all three in FP64 brought it to 8e-8,
    at 3.4 times the time).
"""
import numpy as np
import pytest

from gpuga_b200 import PATH_BATCHED, PATH_PLAIN64, Fitness, synth

pytestmark = pytest.mark.gpu


def _set(S_free: bool):
    data = synth.make(2)
    if S_free:
        data["pmin"][3], data["pmax"][3] = 1.5, 2.5
        data["teacher01"][3] = 0.37
    with Fitness(arrays=data) as e0:
        data = synth.fill_targets(data, lambda _d, p: e0.find_force64(p))
    return data


@pytest.mark.parametrize("S_free,tol", [(False, 1e-6), (True, 2e-5)])
def test_random_population_error_tail(S_free, tol):
    data = _set(S_free)
    P = 400
    pop = synth.population(data, P, seed=12)
    with Fitness(arrays=data) as e:
        fit = np.asarray(e.compute(P, pop, path=PATH_BATCHED))
        f64 = np.asarray(e.compute(P, pop, path=PATH_PLAIN64))
    rel = np.abs(fit - f64) / np.abs(f64)
    assert rel.max() <= tol, f"max relative fitness error {rel.max():.3e} (p99 {np.percentile(rel, 99):.3e})"
    order, oorder = np.argsort(fit, kind="stable"), np.argsort(f64, kind="stable")
    if not np.array_equal(order, oorder):
        srt = np.sort(f64)
        assert (np.diff(srt) / np.abs(srt[1:])).min() <= 2 * tol


@pytest.mark.parametrize("cutoff,zmax", [(3.0, 4), (3.9, 16)])
def test_free_S_and_wide_lists_against_the_oracle(built_oracle, tmp_path, cutoff, zmax):
    """The instantiation that carries the constants' remainders (S free), on 4-neighbor lists and on
    up to 16-neighbor lists (cutoff 3.9 A: the second shell enters the list with fc = 0 beyond R2), against
    the FP64 oracle: relative fitness error <= 2e-5, per-config virials <= 2e-6 of scale."""
    from tests.helpers import oracle_targets
    data = synth.make(2, Nc=24, seed=31)
    data["cutoff"] = cutoff
    data["pmin"][3], data["pmax"][3] = 1.5, 2.5
    data["teacher01"][3] = 0.37
    data = synth.fill_targets(data, oracle_targets(built_oracle))
    d = synth.write_dir(data, str(tmp_path / "set"))
    s = built_oracle.OracleSet(d)
    P = 40
    pop = synth.population(data, P, seed=8)
    with Fitness(d) as e:
        NN, _ = e.neighbors()
        assert zmax // 2 < int(NN.max()) <= zmax  # the 4- or 16-slot kernel class
        fit = np.asarray(e.compute(P, pop))
        E, W, _ = e.config_results(P)
    ofit = s.fitness(pop)
    assert (np.abs(fit - ofit) / np.abs(ofit)).max() <= 2e-5
    Ncf = s.Nc_force
    for p in (0, P - 1):
        oF, oW, ope = s.find_force(s.decode(pop[p]))
        _, oWc = s.config_sums(oW, ope)
        oWm = oWc.reshape(6, s.Nc).T
        assert np.abs(W[p, Ncf:] - oWm[Ncf:]).max() <= 2e-6 * np.abs(oWm[Ncf:]).max()
