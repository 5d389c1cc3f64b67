"""GPU parity: the CUDA paths of libgpuga_b200.so against the FP64 CPU oracle.

Tolerances (stated here, checked below):
  * neighbor lists: bit-exact (integer work);
  * FP64 path (plain64 / find_force64): relative 1e-9 of each quantity's scale;
  * batched mixed-precision path (FP32 pair/three-body math with FP64 where
    differences cancel, FP64 sums): fitness relative error <= 1e-6 for every
    individual, per-config energies and virials <= 2e-6 of the set's scale,
    forces <= 2e-5 of the force scale, and the ranking of each population equals
    the FP64 ranking (no near-tie exemption).
"""
import os

import numpy as np
import pytest

from gpuga_b200 import PATH_BATCHED, PATH_PLAIN32, PATH_PLAIN64, Fitness, synth
from tests.helpers import config_totals, read_elite, reference_outputs, synthetic_dir

pytestmark = pytest.mark.gpu

FIT_RTOL = 1e-6
FIXTURES = ["si_diamond", "wurzite_Si", "wurzite_GaAs", "nn2b", "hfo2"]


def engine_for(d, oracle_set, **kw):
    if oracle_set.potential_type == 3:
        kw.setdefault("nn2b_r1", 7.0)
        kw.setdefault("nn2b_r2", 8.0)
    return Fitness(d, **kw)


@pytest.fixture(scope="module")
def sets(golden, built_oracle, tmp_path_factory):
    cache = {}

    def get(name):
        if name not in cache:
            if name.startswith("synth"):
                cfg, Nc = {"synth1": (1, 20), "synth2": (2, 40), "synth3": (3, 10), "synth4": (4, 8)}[name]
                d, data = synthetic_dir(built_oracle, cfg, Nc, str(tmp_path_factory.mktemp(name)))
                s = built_oracle.OracleSet(d)
                kw = {}
                if cfg == 4:
                    s.set_nn2b(data["nn2b_r1"], data["nn2b_r2"], False)
                    kw = dict(nn2b_r1=data["nn2b_r1"], nn2b_r2=data["nn2b_r2"])
                cache[name] = (d, s, kw)
            else:
                d = golden(name)
                s = built_oracle.OracleSet(d)
                cache[name] = (d, s, {})
        return cache[name]

    return get


ALL = FIXTURES + ["synth1", "synth2", "synth3", "synth4"]


@pytest.mark.parametrize("name", ALL)
def test_neighbor_list_bit_exact(name, sets):
    d, s, kw = sets(name)
    e = engine_for(d, s, **kw)
    NN, nbr = e.neighbors()
    oNN, onl = s.neighbors()
    np.testing.assert_array_equal(NN, oNN)
    np.testing.assert_array_equal(nbr, onl)
    NNr, NL = e.neighbors_reference_layout()
    np.testing.assert_array_equal(NNr, oNN)
    # reference layout NL[k*N + i]
    off = np.concatenate([[0], np.cumsum(oNN)])
    i = np.arange(s.N)
    for k in range(int(oNN.max())):
        m = oNN > k
        np.testing.assert_array_equal(NL[k * s.N + i[m]], onl[off[:-1][m] + k])


@pytest.mark.parametrize("name", ALL)
def test_fp64_path_matches_oracle(name, sets):
    d, s, kw = sets(name)
    e = engine_for(d, s, **kw)
    rng = np.random.default_rng(3)
    x = rng.uniform(0, 1, size=s.num_vars).astype(np.float32)
    p = s.decode(x)
    np.testing.assert_array_equal(e.decode(x).astype(np.float64), p)
    F, W, pe = e.find_force64(p)
    oF, oW, ope = s.find_force(p)
    for a, b in ((F, oF), (W, oW), (pe, ope)):
        scale = max(np.abs(b).max(), 1e-30)
        assert np.abs(a - b).max() <= 1e-9 * scale
    pop = rng.uniform(0, 1, size=(5, s.num_vars)).astype(np.float32)
    fit = e.compute(5, pop, path=PATH_PLAIN64)
    ofit = s.fitness(pop)
    np.testing.assert_allclose(fit, ofit, rtol=1e-9)


def _check_batched(e, s, pop, label):
    P = pop.shape[0]
    fit, comps = e.compute(P, pop, path=PATH_BATCHED, components=True)
    ofit, ocomps = s.fitness(pop, with_components=True)
    finite = np.isfinite(ofit)
    assert np.array_equal(np.isfinite(fit), finite), label
    rel = np.abs(fit[finite] - ofit[finite]) / np.abs(ofit[finite])
    assert rel.max() <= FIT_RTOL, f"{label}: max rel fitness error {rel.max():.3e}"
    order, oorder = np.argsort(fit, kind="stable"), np.argsort(ofit, kind="stable")
    assert np.array_equal(order, oorder), f"{label}: ranking differs from the FP64 ranking"
    return rel.max()


@pytest.mark.parametrize("name", ALL)
def test_batched_fitness_matches_oracle(name, sets):
    d, s, kw = sets(name)
    e = engine_for(d, s, **kw)
    P = 37 if s.N < 20000 else 8  # a partial warp of individuals
    pop = synth.population({"pmin": s.pmin}, P, seed=11)
    _check_batched(e, s, pop, name)


@pytest.mark.parametrize("name", ["si_diamond", "synth1", "synth2", "synth3"])
def test_batched_config_results_and_forces(name, sets):
    d, s, kw = sets(name)
    e = engine_for(d, s, **kw)
    P = 6
    pop = synth.population({"pmin": s.pmin}, P, seed=5)
    e.compute(P, pop)
    E, W, F2 = e.config_results(P)
    forces = e.batched_forces(pop)
    Ncf = s.Nc_force
    for p in range(P):
        prm = s.decode(pop[p])
        oF, oW, ope = s.find_force(prm)
        oE, oWc = s.config_sums(oW, ope)
        escale = np.abs(oE[Ncf:]).max()
        assert np.abs(E[p, Ncf:] - oE[Ncf:]).max() <= 2e-6 * escale
        oWm = oWc.reshape(6, s.Nc).T
        wscale = np.abs(oWm[Ncf:]).max()
        assert np.abs(W[p, Ncf:] - oWm[Ncf:]).max() <= 2e-6 * wscale
        Nf = s.N_force
        oFf = np.stack([oF[:Nf], oF[s.N:s.N + Nf], oF[2 * s.N:2 * s.N + Nf]])
        fscale = np.abs(oFf).max()
        assert np.abs(forces[p] - oFf).max() <= 2e-5 * fscale


def test_batched_near_teacher_population(sets):
    """Individuals close to the optimum (small errors, the hardest case for relative error)."""
    d, s, kw = sets("synth2")
    e = engine_for(d, s, **kw)
    data_like = {"pmin": s.pmin, "teacher01": np.full(s.num_vars, 0.5, np.float32)}
    pop = synth.population(data_like, 64, seed=2, near_teacher=0.05)
    _check_batched(e, s, pop, "near-teacher")


def test_graph_and_eager_identical_and_deterministic(sets):
    d, s, kw = sets("synth2")
    pop = synth.population({"pmin": s.pmin}, 70, seed=9)
    a = engine_for(d, s, use_graph=True).compute(70, pop)
    b = engine_for(d, s, use_graph=False).compute(70, pop)
    np.testing.assert_array_equal(a, b)
    e = engine_for(d, s)
    c1 = e.compute(70, pop)
    c2 = e.compute(70, pop)
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_array_equal(a, c1)


def test_result_is_the_same_alone_and_in_a_mix(sets):
    """An individual's fitness does not depend on the rest of the population."""
    d, s, kw = sets("synth2")
    e = engine_for(d, s)
    pop = synth.population({"pmin": s.pmin}, 96, seed=4)
    mix = e.compute(96, pop)
    for idx in (0, 31, 32, 95):
        alone = e.compute(1, pop[idx:idx + 1])
        assert alone[0] == mix[idx]


def test_plain32_path_close_to_fp64(sets):
    d, s, kw = sets("si_diamond")
    e = engine_for(d, s)
    pop = synth.population({"pmin": s.pmin}, 4, seed=1)
    f32 = e.compute(4, pop, path=PATH_PLAIN32)
    f64 = e.compute(4, pop, path=PATH_PLAIN64)
    np.testing.assert_allclose(f32, f64, rtol=1e-3)


@pytest.mark.parametrize("name", ["si_diamond", "wurzite_Si", "nn2b", "hfo2"])
def test_predict_reproduces_reference_outputs(name, sets, tmp_path):
    d, s, kw = sets(name)
    e = engine_for(d, s, **kw)
    p = read_elite(d)
    # elite01 such that the FP32 decode gives the printed parameters (min == max entries are exact)
    span = (s.pmax.astype(np.float64) - s.pmin)
    x = np.where(span > 0, (p - s.pmin) / np.where(span > 0, span, 1), 0.0).astype(np.float32)
    e.predict(str(tmp_path), x)
    fo, eo, vo = reference_outputs(d)
    mf, me, mv = reference_outputs(str(tmp_path))
    assert mf.shape == fo.shape and me.shape == eo.shape and mv.shape == vo.shape
    np.testing.assert_allclose(mf[:, 3:], fo[:, 3:], rtol=1e-5, atol=1e-6)
    tol_e = 3e-4 if name == "nn2b" else 3e-5
    assert np.abs(mf[:, :3] - fo[:, :3]).max() <= 1e-4 * np.abs(fo[:, :3]).max()
    assert np.abs(me[:, 0] - eo[:, 0]).max() <= tol_e * max(np.abs(eo[:, 0]).max(), 1e-3)
    assert np.abs(mv[:, 0] - vo[:, 0]).max() <= 1e-4 * np.abs(vo[:, 0]).max()
