"""Golden fixtures for gpuga_b200.train_tool from the reference's own converter.

Builds develop/wurzite/{GaAs,Si}/construct_train_in.cpp (each copy carries its
own compile-time settings) with g++ into oracle/_ref/, runs each on a subset of
that directory's DFT files (2 force configurations, 5 energy/virial
configurations, the last 3 from other_poly/ as in the reference's input.txt)
and stores, under tests/golden/train_tool/<set>/, the input files, input.txt
and the train.in the reference program wrote.

    python tests/golden/make_train_tool_fixture.py [path/to/reference]
"""
import os
import shutil
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
import sys

REFERENCE = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GPUGA_REFERENCE", "/root/reference")
REF = os.path.join(REFERENCE, "develop", "wurzite")

FILES = ["random/data_0", "random/data_1", "HIDROSTATIC/data_-0.010000", "BIAXIAL_0/data_-0.010000",
         "other_poly/data-bcc", "other_poly/data-rocksalt", "other_poly/data-zb"]


def main() -> None:
    os.makedirs(os.path.join(ROOT, "oracle", "_ref"), exist_ok=True)
    for name in ("GaAs", "Si"):
        exe = os.path.join(ROOT, "oracle", "_ref", f"construct_train_in_{name}")
        subprocess.run(["g++", "-O3", "-o", exe, os.path.join(REF, name, "construct_train_in.cpp")], check=True)
        dst = os.path.join(HERE, "train_tool", name)
        shutil.rmtree(dst, ignore_errors=True)
        work = tempfile.mkdtemp(prefix="gpuga_tt_")
        for f in FILES:
            for d in (dst, work):
                os.makedirs(os.path.join(d, os.path.dirname(f)), exist_ok=True)
                shutil.copy(os.path.join(REF, name, f), os.path.join(d, f))
        listing = "2 5\n" + "\n".join(FILES) + "\n"
        with open(os.path.join(dst, "input.txt"), "w") as f:
            f.write(listing)
        subprocess.run([exe], input=listing, text=True, cwd=work, check=True)
        shutil.copy(os.path.join(work, "train.in"), os.path.join(dst, "train.in"))
        shutil.rmtree(work)
        print("wrote", dst)


if __name__ == "__main__":
    main()
