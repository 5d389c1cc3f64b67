"""The gpuga command-line driver (the reference's main.cu interface): stdin lists
input directories; each gets ga.out, force.out, energy.out and virial.out."""
import os
import subprocess

import numpy as np
import pytest

from gpuga_b200 import GA, Fitness, _lib
from tests.helpers import synthetic_dir

pytestmark = pytest.mark.gpu


def test_cli_runs_a_fit_and_matches_the_library_ga(built_oracle, tmp_path):
    d, data = synthetic_dir(built_oracle, 1, 6, str(tmp_path / "fit"))
    with open(os.path.join(d, "ga.in"), "w") as f:
        f.write("maximum_generation 5\npopulation_size 40\nparent_number 20\nmutation_rate 0.2\n")
    r = subprocess.run([_lib.CLI_PATH, "--seed", "12345678"], input=f"1\n{d}\n", capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Finished running gpuga." in r.stdout
    lines = open(os.path.join(d, "ga.out")).read().splitlines()
    assert len(lines) == 5 and lines[0].startswith("0 ")
    with Fitness(d) as e:
        ga = GA(e, input_dir=d, seed=12345678)
        mine = [ga.step().rstrip("\n") for _ in range(5)]
        ga.close()
        assert lines == mine
        fo = np.loadtxt(os.path.join(d, "force.out"), ndmin=2)
        eo = np.loadtxt(os.path.join(d, "energy.out"), ndmin=2)
        vo = np.loadtxt(os.path.join(d, "virial.out"), ndmin=2)
        assert fo.shape == (e.N_force, 6)
        assert eo.shape == (e.Nc - e.Nc_force, 2)
        assert vo.shape == (6 * (e.Nc - e.Nc_force), 2)


def test_cli_reports_input_errors(tmp_path):
    r = subprocess.run([_lib.CLI_PATH], input=f"1\n{tmp_path}\n", capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert "potential.in" in r.stderr


def test_cli_host_loop_matches_device_loop(built_oracle, tmp_path):
    """--host-loop (selection on the host each generation) writes the same ga.out as the default
    device-resident GA loop."""
    import shutil
    d, _ = synthetic_dir(built_oracle, 1, 6, str(tmp_path / "a"))
    with open(os.path.join(d, "ga.in"), "w") as f:
        f.write("maximum_generation 12\npopulation_size 40\nparent_number 20\nmutation_rate 0.2\n")
    d2 = str(tmp_path / "b")
    shutil.copytree(d, d2)
    outs = []
    for dd, extra in ((d, []), (d2, ["--host-loop"])):
        r = subprocess.run([_lib.CLI_PATH, "--seed", "7"] + extra, input=f"1\n{dd}\n", capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        outs.append(open(os.path.join(dd, "ga.out")).read())
    assert outs[0] == outs[1]
