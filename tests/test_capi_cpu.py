"""C ABI checks that need no GPU: every declared symbol is exported, and the
host-side parsers follow the reference's rules (fitness.cu:59-314, ga.cu:214-316)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from gpuga_b200 import _lib, synth
from tests.conftest import ROOT

HEADER = os.path.join(ROOT, "include", "gpuga.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(gpuga_[a-z0-9_]+)\s*\(", text)
    return sorted(set(n for n in names if not n.endswith("_cb")))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python bindings cover the whole ABI
    assert set(names) <= set(_lib.PROTOTYPES) | {"gpuga_calibrate_fp32"}


def test_version_and_defaults():
    L = _lib.load()
    assert L.gpuga_version().decode().startswith("gpuga-b200")
    o = _lib.Options()
    L.gpuga_default_options(C.byref(o))
    assert (o.device, o.path, o.use_graph, o.nn2b_consistent) == (0, 0, 1, 0)
    assert (o.nn2b_r1, o.nn2b_r2) == (7.0, 8.0)


def parse(d):
    sz = np.zeros(11, np.int32)
    st = _lib.load().gpuga_parse_inputs(d.encode(), sz.ctypes.data_as(C.c_void_p))
    return st, sz


@pytest.mark.parametrize("name,ga", [("si_diamond", [200, 100, 1000]), ("wurzite_Si", [400, 200, 1000]),
                                     ("nn2b", [200, 100, 1000]), ("hfo2", [200, 100, 1000])])
def test_parse_golden_sets_like_the_oracle(name, ga, golden, built_oracle):
    d = golden(name)
    st, sz = parse(d)
    assert st == 0, _lib.load().gpuga_last_error()
    s = built_oracle.OracleSet(d)
    assert list(sz[:8]) == [s.potential_type, s.num_vars, s.num_neurons, s.Nc, s.Nc_force, s.N, s.N_force, s.max_Na]
    assert list(sz[8:]) == ga


def _write(d, potential=None, train=None, ga=None):
    os.makedirs(d, exist_ok=True)
    if potential is not None:
        open(os.path.join(d, "potential.in"), "w").write(potential)
    if train is not None:
        open(os.path.join(d, "train.in"), "w").write(train)
    if ga is not None:
        open(os.path.join(d, "ga.in"), "w").write(ga)
    return d


POT1 = "potential_type 1\ncutoff 3\nweight_force 0.1\nweight_energy 0.2\nweight_virial 0.7\n" + \
       "".join(f"p{k} 1 2\n" for k in range(9))
BOX = "5 0 0 0 5 0 0 0 5\n"
TRAIN_OK = "2 1\n2\n2\n" + BOX + "0 0 0 0 0 0 0\n0 1 1 1 0 0 0\n-1 0 0 0 0 0 0\n" + BOX + "0 0 0 0\n0 1 1 1\n"


def test_parse_minimal_valid_set(tmp_path):
    d = _write(str(tmp_path), POT1, TRAIN_OK)
    st, sz = parse(d)
    assert st == 0
    assert list(sz[:8]) == [1, 9, 0, 2, 1, 4, 2, 2]


@pytest.mark.parametrize("train,msg", [
    ("1 1\n2\n", "configurations should >= 2"),
    ("2 0\n2\n2\n", "force configurations should >= 1"),
    ("2 2\n2\n2\n", "potential configurations should >= 1"),
    ("2 1\n1\n2\n", "should >= 2"),
    ("2 1\n2\n2\n" + BOX + "0 0 0 0 0 0\n", "reading error"),
])
def test_train_in_validation(tmp_path, train, msg):
    d = _write(str(tmp_path), POT1, train)
    st, _ = parse(d)
    assert st == _lib.ERR_PARSE
    assert msg in _lib.load().gpuga_last_error().decode()


@pytest.mark.parametrize("pot,status", [
    ("potential_type 7\n", _lib.ERR_UNSUPPORTED),
    ("potential_type 1\ncutoff 3\nweight_force -1\n", _lib.ERR_PARSE),
    ("potential_type 1\ncutoff 3\nweight_force 1\nweight_energy 1\nweight_virial 1\nD0 1\n", _lib.ERR_PARSE),
    ("potential_type 3\n", _lib.ERR_PARSE),
])
def test_potential_in_validation(tmp_path, pot, status):
    d = _write(str(tmp_path), pot, TRAIN_OK)
    st, _ = parse(d)
    assert st == status


def test_missing_files_are_io_errors(tmp_path):
    st, _ = parse(str(tmp_path))
    assert st == _lib.ERR_IO


@pytest.mark.parametrize("ga,ok", [
    ("maximum_generation 10\npopulation_size 40 # comment\nparent_number 20\nmutation_rate 0.5\n", True),
    ("population_size 0x28\n", True),           # strtol base 0 (read_file.cu:81)
    ("population_size 25\n", False),            # multiple of 10
    ("population_size 10\n", False),            # >= 20
    ("parent_number 5\n", False),
    ("mutation_rate 1.5\n", False),
    ("mutation_rate abc\n", False),
    ("maximum_generation 0\n", False),
    ("maximum_generation 10 20\n", False),
    ("bogus_keyword 1\n", False),
    ("# only a comment\n\n", True),
])
def test_ga_in_rules(tmp_path, ga, ok):
    d = _write(str(tmp_path), POT1, TRAIN_OK, ga)
    st, sz = parse(d)
    assert (st == 0) == ok, _lib.load().gpuga_last_error()
    if ga.startswith("population_size 0x28"):
        assert sz[8] == 40


def test_synthetic_sets_parse(tmp_path):
    for cfg, Nc in [(1, 4), (2, 6), (3, 4), (4, 4)]:
        data = synth.make(cfg, Nc=Nc)
        d = synth.write_dir(data, str(tmp_path / f"w{cfg}"))
        st, sz = parse(d)
        assert st == 0, _lib.load().gpuga_last_error()
        assert sz[3] == Nc and sz[4] == Nc // 2 and sz[5] == int(data["Na"].sum())


def test_cli_rejects_unknown_options_with_usage():
    """The gpuga driver parses its options before touching a GPU: an unknown one prints the usage."""
    import os
    import subprocess
    if not os.path.exists(_lib.CLI_PATH):
        pytest.skip("gpuga CLI not built")
    r = subprocess.run([_lib.CLI_PATH, "--no-such-option"], input="0\n", capture_output=True, text=True, timeout=60)
    assert r.returncode == 2
    for opt in ("--host-loop", "--ri-self-energy", "--nn2b-taper", "--neighbor-cells"):
        assert opt in r.stderr
