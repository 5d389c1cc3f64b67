"""Device-resident GA loop (gpuga_ga_advance) against the host GA.

The device loop draws the same random choices from the same std::mt19937
stream and applies them on the GPU, so after any number of generations the
ga.out lines, the population, the fitness vector and the random stream (the
generations that follow) are identical to stepping the host GA -- bit for
bit, because both score the population with the same batched launches."""
import numpy as np
import pytest

from gpuga_b200 import GA, Fitness, _lib
from tests.helpers import synthetic_dir

pytestmark = pytest.mark.gpu


def host_steps(e, n, **kw):
    ga = GA(e, **kw)
    lines = "".join(ga.step() for _ in range(n))
    return ga, lines


def assert_same_state(a, b, P):
    ga, pa, fa = a.state(P)
    gb, pb, fb = b.state(P)
    assert ga == gb
    np.testing.assert_array_equal(pa, pb)
    np.testing.assert_array_equal(fa, fb)


@pytest.mark.parametrize("window", [1, 8, 32])
def test_device_loop_matches_host_steps_si_diamond(golden, window):
    d = golden("si_diamond")
    with Fitness(d) as e:
        kw = dict(seed=12345678, population_size=200, parent_number=100, mutation_rate=0.2, maximum_generation=1000)
        host, want = host_steps(e, 45, **kw)
        dev = GA(e, **kw)
        dev.set_device_loop(True, window)
        got = dev.advance(45)
        assert got == want
        assert_same_state(host, dev, 200)
        # the random stream continues identically
        assert dev.step() == host.step()
        assert_same_state(host, dev, 200)
        host.close()
        dev.close()


@pytest.mark.parametrize("cfg,Nc,P", [(1, 6, 40), (3, 4, 20), (4, 4, 20)])
def test_device_loop_matches_host_steps_synthetic(built_oracle, tmp_path, cfg, Nc, P):
    d, _ = synthetic_dir(built_oracle, cfg, Nc, str(tmp_path / "set"))
    with Fitness(d) as e:
        kw = dict(seed=7, population_size=P, parent_number=P // 2, mutation_rate=0.3, maximum_generation=30)
        host, want = host_steps(e, 30, **kw)
        dev = GA(e, **kw)
        dev.set_device_loop(True, 7)
        # interleaved: device window, host steps, device again
        got = dev.advance(11)
        got += "".join(dev.step() for _ in range(4))
        got += dev.advance(100)  # clipped to the 15 generations left
        assert got == want
        assert_same_state(host, dev, P)
        host.close()
        dev.close()


def test_run_writes_the_host_loop_ga_out(golden, tmp_path):
    """gpuga_ga_run on the device loop writes the same ga.out and prediction files as the host loop."""
    import shutil
    outs = {}
    for loop in (0, 1):
        d = str(tmp_path / f"si{loop}")
        shutil.copytree(golden("si_diamond"), d)
        with open(f"{d}/ga.in", "w") as f:
            f.write("maximum_generation 60\npopulation_size 100\nparent_number 50\nmutation_rate 0.2\n")
        with Fitness(d) as e:
            ga = GA(e, input_dir=d, seed=3)
            ga.set_device_loop(bool(loop), 16)
            ga.run(d)
            ga.close()
        outs[loop] = [open(f"{d}/{n}").read() for n in ("ga.out", "force.out", "energy.out", "virial.out")]
    assert outs[0] == outs[1]


def _host_insertion_order(f32):
    """The reference's insertion sort (ga.cu:105-119) on FP32 values, as an index permutation."""
    f = list(f32)
    idx = list(range(len(f)))
    for i in range(1, len(f)):
        key, j = f[i], i - 1
        while j >= 0 and f[j] > key:
            f[j + 1] = f[j]
            idx[j + 1] = idx[j]
            j -= 1
        f[j + 1] = key
        idx[j + 1] = i
    return np.array(idx), np.array(f, np.float32)


@pytest.mark.parametrize("P", [1, 7, 256, 1000, 2003])
def test_rank_is_the_insertion_sort_order(P):
    rng = np.random.default_rng(P)
    fit = rng.choice([0.5, 0.25, 1.0, 2.0], size=P) + rng.integers(0, 3, P) * 1e-9  # ties after FP32 rounding
    fit[rng.random(P) < 0.05] = np.nan
    fit[rng.random(P) < 0.02] = -0.0
    fit[rng.random(P) < 0.02] = 0.0
    fit[rng.random(P) < 0.02] = np.inf
    order = np.zeros(P, np.int32)
    srt = np.zeros(P, np.float32)
    L = _lib.load()
    _lib.check(L.gpuga_ga_rank_device(0, P, fit.ctypes.data, order.ctypes.data, srt.ctypes.data))
    want_idx, want_f = _host_insertion_order(fit.astype(np.float32))
    np.testing.assert_array_equal(order, want_idx)
    np.testing.assert_array_equal(srt.view(np.uint32), want_f.view(np.uint32))
