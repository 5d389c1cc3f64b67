"""gpuga_b200.train_tool against the reference's own DFT -> train.in converter.

tests/golden/train_tool/<set>/train.in was written by the reference program
(develop/wurzite/<set>/construct_train_in.cpp, built unmodified;
tests/golden/make_train_tool_fixture.py) from the DFT files beside it.  The
tool, given the settings compiled into that copy, must write the same text."""
import os
import subprocess
import sys

import pytest

from gpuga_b200 import train_tool

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "train_tool")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# the compile-time settings of each reference copy (construct_train_in.cpp:46-55, 143, 222-233)
SETTINGS = {
    "GaAs": dict(cells=(4, 4, 3), delta_e=0.0, stress_kbar=True, force_types="zero",
                 z_bands=((1.5, 4.5), (7.5, 10.5), (13.5, 17.0)), ev_type_map=[0, 1, 1, 0], ev_map_skip_last=3,
                 ev_types="zero", max_cell_size=4),
    "Si": dict(cells=(4, 4, 3), delta_e=1.31684, stress_kbar=True, force_types="file",
               z_bands=((1.5, 4.5), (7.5, 10.5), (13.5, 17.0)), ev_type_map=[0, 1, 1, 0], ev_map_skip_last=3,
               ev_types="file", max_cell_size=4),
}


def _files(name):
    tok = open(os.path.join(GOLD, name, "input.txt")).read().split()
    return int(tok[0]), [os.path.join(GOLD, name, f) for f in tok[2:]]


@pytest.mark.parametrize("name", sorted(SETTINGS))
def test_same_train_in_as_the_reference_converter(name):
    nf, files = _files(name)
    got = train_tool.build(files, nf, **SETTINGS[name])
    want = open(os.path.join(GOLD, name, "train.in")).read()
    assert got == want


def test_command_line(tmp_path):
    args = ["--cells", "4", "4", "3", "--force-types", "zero", "--z-bands", "1.5:4.5,7.5:10.5,13.5:17",
            "--ev-type-map", "0,1,1,0", "--ev-map-skip-last", "3", "--ev-types", "zero", "--max-cell-size", "4",
            "--dir", os.path.join(GOLD, "GaAs"), "--output", str(tmp_path / "train.in")]
    with open(os.path.join(GOLD, "GaAs", "input.txt")) as f:
        subprocess.run([sys.executable, "-m", "gpuga_b200.train_tool"] + args, stdin=f, check=True, cwd=ROOT)
    assert open(tmp_path / "train.in").read() == open(os.path.join(GOLD, "GaAs", "train.in")).read()


def test_written_set_parses_and_cell_size_is_checked(tmp_path):
    """The converted set is a valid training set for the engine's parser; oversize cells are refused."""
    nf, files = _files("GaAs")
    with pytest.raises(ValueError):
        train_tool.build(files, nf, cells=(1, 1, 1), max_cell_size=1)
    text = train_tool.build(files, nf, **SETTINGS["GaAs"])
    lines = text.splitlines()
    nc, ncf = (int(v) for v in lines[0].split())
    assert (nc, ncf) == (7, 2)
    na = [int(v) for v in lines[1:1 + nc]]
    assert na[:2] == [192, 192] and all(n % 48 == 0 for n in na[2:])
