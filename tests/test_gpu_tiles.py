"""Force-item tiles of the batched Tersoff path and their autotuner.

Each Tersoff force configuration's work items can be tiled several ways (gpuga_options.tiles:
1 the fixed rule, 2 half the individuals per item, 3 a quarter, 4 32 individuals with the f_ij
scratch in global memory, 5 the fixed rule without staged geometry; 0 lets the autotuner pick per
configuration size).  The per-atom arithmetic is the same in every tile and each individual's
squared force errors are summed in a canonical order, so every tile -- and therefore whatever the
autotuner picks -- must give bit-identical fitness values, components and per-configuration
results.  Reference: the reference has one launch shape, <<<Nc, max_Na>>> with get_block_size
(fitness.cu:481-490, minimal_tersoff.cu:421-431).
"""
import numpy as np
import pytest

from gpuga_b200 import PATH_BATCHED, Fitness, synth
from tests.helpers import golden_subset

pytestmark = pytest.mark.gpu


def _sets(golden, tmp_path):
    w2 = synth.make(2, Nc=24, seed=17)  # diamond cells of 8, 64, 216 and 512 atoms
    free = synth.make(2, Nc=16, seed=23)
    free["pmin"][3], free["pmax"][3] = 1.5, 2.5  # S free: the instantiation with remainders
    out = []
    for data in (w2, free):
        with Fitness(arrays=data) as e0:
            data = synth.fill_targets(data, lambda _d, p: e0.find_force64(p))
        out.append(("arrays", data))
    out.append(("dir", golden_subset(golden("wurzite_GaAs"), str(tmp_path / "gaas"), 4, 4)))  # two atom types
    return out


def _run(kind, src, tiles, P, pop):
    e = Fitness(arrays=src, tiles=tiles) if kind == "arrays" else Fitness(src, tiles=tiles)
    with e:
        fit, comps = e.compute(P, pop, path=PATH_BATCHED, components=True)
        E, W, F2 = e.config_results(P)
        codes, _ = e.plan_tiles(P)
        return np.asarray(fit), np.asarray(comps), E, W, F2, codes, e.Nc_force


def test_every_tile_gives_the_same_bits(golden, tmp_path):
    for kind, src in _sets(golden, tmp_path):
        nv = len(src["pmin"]) if kind == "arrays" else 13
        P = 45  # a partial group of individuals in most tiles
        pop = np.random.default_rng(5).uniform(0, 1, size=(P, nv)).astype(np.float32)
        ref = _run(kind, src, 1, P, pop)
        for tiles in (2, 3, 4, 5, 0):
            got = _run(kind, src, tiles, P, pop)
            for a, b in zip(got[:5], ref[:5]):
                assert np.array_equal(a, b), f"{kind} tiles={tiles}: results differ from the fixed rule"
            codes, Ncf = got[5], got[6]
            if tiles:
                assert np.all(codes[:Ncf] == tiles) and np.all(codes[Ncf:] == 0)
            else:
                assert np.all((codes[:Ncf] >= 1) & (codes[:Ncf] <= 5)) and np.all(codes[Ncf:] == 0)


def test_fast_form_for_bonds_inside_r1_gives_the_same_bits():
    """Atoms whose bonds all lie inside r1 take a form without the cutoff terms when every lane of
    their warp agrees (tersoff_atom's vote).  With r1 a fitted parameter in [2.5, 2.9] A, many
    atoms of the diamond cells have bonds beyond some individuals' r1, so which form an atom takes
    depends on the atoms and individuals that share its warp: the tiles (different warp
    compositions in force items) and an individual alone or in a population (different lanes in
    energy/virial items) must still give identical bits.  Reference: the cutoff function and its
    use, minimal_tersoff.cu:77-90 and 191-316."""
    data = synth.make(2, Nc=16, seed=31)
    data["pmin"][7], data["pmax"][7] = 2.5, 2.9  # r1 per individual (r2 stays 3.2)
    with Fitness(arrays=data) as e0:
        data = synth.fill_targets(data, lambda _d, p: e0.find_force64(p))
    P = 40
    pop = np.random.default_rng(11).uniform(0, 1, size=(P, len(data["pmin"]))).astype(np.float32)
    ref = _run("arrays", data, 1, P, pop)
    for tiles in (2, 3, 4):
        got = _run("arrays", data, tiles, P, pop)
        for a, b in zip(got[:5], ref[:5]):
            assert np.array_equal(a, b), f"tiles={tiles}: results differ from the fixed rule"
    with Fitness(arrays=data, tiles=1) as e:
        for i in (0, 17, 39):
            alone = np.asarray(e.compute(1, pop[i:i + 1], path=PATH_BATCHED))
            assert alone[0] == ref[0][i], f"individual {i}: alone {alone[0]!r} vs in the population {ref[0][i]!r}"
