"""Pins the CPU oracle against the reference's own regression outputs.

Each golden set holds the reference's inputs, the last ga.out line (the elite
predict() evaluated, ga.cu:84-91) and the force/energy/virial files predict()
wrote (fitness.cu:335-390).  The reference computed them in FP32 with
fast-math and printed the elite with 6 significant digits, so the bar is a
relative error of ~1e-4 of each quantity's scale.
"""
import numpy as np
import pytest

from tests.helpers import config_totals, read_elite, reference_outputs

# relative tolerance of energies; nn2b's elite has 141 weights printed with 6 digits
SETS = {"si_diamond": 3e-5, "si_diamond_example": 3e-5, "nn2b": 3e-4, "wurzite_Si": 3e-5, "wurzite_GaAs": 3e-5,
        "hfo2": 3e-5}


@pytest.mark.parametrize("name", list(SETS))
def test_oracle_reproduces_reference_outputs(name, golden, built_oracle):
    d = golden(name)
    s = built_oracle.OracleSet(d)
    params = read_elite(d)
    assert len(params) == s.num_vars
    F, W, pe = s.find_force(params)
    Fp, E, Wp = config_totals(s, F, W, pe)
    fo, eo, vo = reference_outputs(d)
    assert fo.shape == (s.N_force, 6) and eo.shape == (s.Nc - s.Nc_force, 2)
    # the reference columns are the parsed targets
    fr = s.arrays()["force_ref"].reshape(3, s.N)[:, :s.N_force].T
    np.testing.assert_allclose(fo[:, 3:], fr, rtol=1e-5, atol=1e-6)
    fscale = np.abs(fo[:, :3]).max()
    assert np.abs(Fp - fo[:, :3]).max() <= 1e-4 * fscale
    escale = max(np.abs(eo[:, 0]).max(), 1e-3)
    assert np.abs(E - eo[:, 0]).max() <= SETS[name] * escale
    vscale = np.abs(vo[:, 0]).max()
    assert np.abs(Wp - vo[:, 0]).max() <= 1e-4 * vscale


@pytest.mark.parametrize("name,rtol", [("si_diamond", 1e-5), ("si_diamond_example", 1e-5), ("nn2b", 1e-3),
                                       ("wurzite_Si", 1e-5), ("wurzite_GaAs", 1e-5), ("hfo2", 1e-5)])
def test_oracle_fitness_matches_reference_ga_out(name, rtol, golden, built_oracle):
    """The best fitness the reference printed for its elite (ga.cu:141) is recomputed by the oracle."""
    d = golden(name)
    s = built_oracle.OracleSet(d)
    with open(f"{d}/ga_last.out") as f:
        printed = float(f.read().split()[1])
    F, W, pe = s.find_force(read_elite(d))
    import ctypes as C
    comps = np.zeros(3)
    lib = built_oracle.lib()
    fit = lib.oracle_fitness_arrays(s._h, *(a.ctypes.data_as(C.c_void_p) for a in (F, W, pe, comps)))
    assert abs(fit - printed) <= rtol * printed


def test_oracle_neighbor_counts(golden, built_oracle):
    """Coordination numbers the reference prints at start-up (neighbor.cu:78-82)."""
    s = built_oracle.OracleSet(golden("si_diamond"))
    NN, nl = s.neighbors()
    counts = np.bincount(NN)
    assert counts.argmax() == 4 and NN.min() == 3 and NN.max() == 12  # polytype / strained cells
    assert nl.size == NN.sum()
    # lists are ascending and symmetric
    off = np.concatenate([[0], np.cumsum(NN)])
    for i in range(0, s.N, 97):
        li = nl[off[i]:off[i + 1]]
        assert np.all(np.diff(li) > 0)
        for j in li:
            assert i in nl[off[j]:off[j + 1]]


def test_oracle_fma_modes_agree_on_fixtures(golden, built_oracle):
    """The three FP32 contraction patterns give the same lists on the reference data."""
    d = golden("wurzite_Si")
    lists = [built_oracle.OracleSet(d, fma_mode=m).neighbors() for m in (0, 1, 2)]
    for NN, nl in lists[1:]:
        np.testing.assert_array_equal(NN, lists[0][0])
        np.testing.assert_array_equal(nl, lists[0][1])
