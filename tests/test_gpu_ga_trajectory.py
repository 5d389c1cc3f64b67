"""GA trajectory parity with the reference program itself.

tests/golden/si_diamond/ga_ref_linux.out is the ga.out the unmodified reference
(src/*.cu, seeded GA) wrote on a B200 for tests/si_diamond
(tests/golden/make_ref_ga_fixture.py).  The gpuga CLI with the same seed must
select the same elite in every one of the 1000 generations: the decoded
parameters of every line are identical text, and the printed best fitness
agrees to within 2e-5 relative (the reference computes it in FP32 with
fast-math, this engine sums in FP64)."""
import os
import subprocess

import pytest

from gpuga_b200 import _lib
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(GOLDEN, "si_diamond", "ga_ref_linux.out")


@pytest.mark.skipif(not os.path.exists(FIXTURE), reason="reference trajectory fixture not recorded")
def test_cli_follows_the_reference_trajectory(golden, tmp_path):
    import shutil
    d = str(tmp_path / "si")
    shutil.copytree(golden("si_diamond"), d)
    r = subprocess.run([_lib.CLI_PATH, "--seed", "12345678"], input=f"1\n{d}\n", capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    ours = open(os.path.join(d, "ga.out")).read().splitlines()
    ref = open(FIXTURE).read().splitlines()
    assert len(ours) == len(ref) == 1000
    for a, b in zip(ours, ref):
        fa, fb = a.split(), b.split()
        assert fa[0] == fb[0]
        assert fa[2:] == fb[2:], f"generation {fa[0]}: elite differs"
        assert abs(float(fa[1]) - float(fb[1])) <= 2e-5 * abs(float(fb[1]))
