"""NN2B network widths across the batched kernel's register classes (8, 12, 16, 32 neurons, with
and without a width of the class's own size; above 16 one pair per weight load) against the FP64
path: relative fitness error <= 1e-6 per individual and the FP64 ranking, on random individuals.
Each unordered pair is evaluated once in force items and energy/virial items walk the
configuration's pair list at every width.  Reference: nn2b.cu:49-173 (widths up to 10 there)."""
import numpy as np
import pytest

from gpuga_b200 import PATH_BATCHED, PATH_PLAIN64, Fitness, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("neurons", [3, 8, 11, 12, 20, 32])
def test_width_against_fp64(neurons):
    data = synth.make(4, Nc=8, neurons=neurons, seed=60 + neurons)
    kw = dict(nn2b_r1=data["nn2b_r1"], nn2b_r2=data["nn2b_r2"])
    with Fitness(arrays=data, **kw) as e0:
        data = synth.fill_targets(data, lambda _d, p: e0.find_force64(p))
    P = 40
    pop = synth.population(data, P, seed=5)
    with Fitness(arrays=data, **kw) as e:
        fit = np.asarray(e.compute(P, pop, path=PATH_BATCHED))
        f64 = np.asarray(e.compute(P, pop, path=PATH_PLAIN64))
    rel = np.abs(fit - f64) / np.abs(f64)
    assert rel.max() <= 1e-6, f"n = {neurons}: max relative fitness error {rel.max():.3e}"
    assert np.array_equal(np.argsort(fit, kind="stable"), np.argsort(f64, kind="stable"))
