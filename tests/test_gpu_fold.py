"""Where each individual's fitness is folded (gpuga_options.fitness_fold): in the work item that
finishes the individual's last configuration (1: a per-individual atomic count, reset by the
folding item for the next generation) or in a launch of its own (2, and the default 0).  The fold is the same fixed-order FP64 sum in every case, so fitness values and
components must be bit-identical -- generation after generation, which also checks that the counts
return to zero.  Reference: fitness.cu:329-331, 392-555 (the reference folds on the host)."""
import ctypes as C

import numpy as np
import pytest

from gpuga_b200 import PATH_BATCHED, Fitness, _lib, synth

pytestmark = pytest.mark.gpu


def _sets():
    out = []
    for workload, Nc in ((2, 24), (3, 6), (4, 8)):
        data = synth.make(workload, Nc=Nc, seed=40 + workload)
        kw = dict(nn2b_r1=data["nn2b_r1"], nn2b_r2=data["nn2b_r2"]) if workload == 4 else {}
        with Fitness(arrays=data, **kw) as e0:
            data = synth.fill_targets(data, lambda _d, p: e0.find_force64(p))
        out.append((workload, data, kw))
    return out


def _kernels(e, P):
    k = C.c_int()
    _lib.check(_lib.load().gpuga_plan_kernels(e.handle, P, C.byref(k)))
    return k.value


@pytest.mark.parametrize("index", [0, 1, 2])
def test_fold_placement_gives_the_same_bits(index):
    workload, data, kw = _sets()[index]
    P = 45
    pops = [synth.population(data, P, seed=70 + g) for g in range(3)]
    results = {}
    for fold in (1, 2, 0):
        with Fitness(arrays=data, fitness_fold=fold, **kw) as e:
            got = []
            for pop in pops:  # three generations through the same plan
                fit, comps = e.compute(P, pop, path=PATH_BATCHED, components=True)
                got.append((np.asarray(fit).copy(), np.asarray(comps).copy()))
            results[fold] = (got, _kernels(e, P))
    (ref, k1), (sep, k2), (auto, k0) = results[1], results[2], results[0]
    assert k2 == k1 + 1  # the separate fold is one more launch
    assert k0 == k2      # the default is the fold launch
    for g, (a, b, c) in enumerate(zip(ref, sep, auto)):
        for what, x, y, z in zip(("fitness", "components"), a, b, c):
            rel = float(np.max(np.abs(x - y) / np.abs(y)))
            assert np.array_equal(x, y), (f"workload {workload}, generation {g}: {what} folded in the items differ "
                                          f"from the fold launch (max rel {rel:.3e}, {int(np.sum(x != y))} values)")
            assert np.array_equal(x, z)
