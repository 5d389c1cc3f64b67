"""Records the reference's own GA trajectory on tests/si_diamond (needs a GPU).

Runs the unmodified reference program built with the seeded GA
(oracle/_ref/gpuga_ref: src/*.cu, -DDEBUG => std::mt19937(12345678), Linux
libstdc++) on the committed si_diamond fixture and stores its ga.out as
tests/golden/si_diamond/ga_ref_linux.out.  (ga1.out in the same folder comes
from the Windows build, whose <random> distributions differ from libstdc++'s.)

    python tests/golden/make_ref_ga_fixture.py
"""
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.conftest import materialize  # noqa: E402


def main() -> None:
    exe = os.path.join(ROOT, "oracle", "_ref", "gpuga_ref")
    d = materialize("si_diamond", tempfile.mkdtemp(prefix="gpuga_refga_"))
    r = subprocess.run([exe], input=f"1\n{d}\n", capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        raise SystemExit(f"reference run failed: {r.stderr[-500:]}")
    shutil.copy(os.path.join(d, "ga.out"), os.path.join(HERE, "si_diamond", "ga_ref_linux.out"))
    print("wrote", os.path.join(HERE, "si_diamond", "ga_ref_linux.out"))


if __name__ == "__main__":
    main()
