"""Seeded synthetic workloads: deterministic, in the reference's formats, and the
teacher parameter vector reproduces its own targets (fitness ~ FP32 rounding)."""
import numpy as np
import pytest

from gpuga_b200 import synth
from tests.helpers import synthetic_dir


def test_generator_is_deterministic():
    a = synth.make(2, Nc=12)
    b = synth.make(2, Nc=12)
    for k in ("Na", "r", "box9", "type", "teacher01"):
        np.testing.assert_array_equal(a[k], b[k])
    assert not np.array_equal(synth.make(2, seed=9, Nc=12)["r"], a["r"])


@pytest.mark.parametrize("cfg,Nc,sizes", [(1, 20, {64}), (2, 40, {8, 64, 216, 512}), (3, 12, None), (4, 10, {64, 216})])
def test_workload_shapes(cfg, Nc, sizes):
    data = synth.make(cfg, Nc=Nc)
    assert len(data["Na"]) == Nc and data["Nc_force"] == Nc // 2
    if sizes:
        assert set(int(n) for n in data["Na"]) <= sizes
    if cfg == 3:
        assert data["Na"].min() >= 96 and data["Na"].max() <= 324
        assert set(np.unique(data["type"])) == {0, 1}


@pytest.mark.parametrize("cfg,Nc", [(1, 6), (2, 10), (3, 4), (4, 4)])
def test_teacher_reproduces_targets(cfg, Nc, tmp_path, built_oracle):
    d, data = synthetic_dir(built_oracle, cfg, Nc, str(tmp_path))
    s = built_oracle.OracleSet(d)
    if cfg == 4:
        s.set_nn2b(data["nn2b_r1"], data["nn2b_r2"], False)
    fit = s.fitness(np.vstack([data["teacher01"], synth.population(data, 2, seed=1)]))
    assert fit[0] < 1e-5
    assert np.all(fit[1:] > 100 * fit[0])


def test_full_size_workload2_statistics():
    data = synth.make(2)
    assert len(data["Na"]) == 500
    assert 90000 < int(data["Na"].sum()) < 115000
