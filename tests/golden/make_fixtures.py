"""Regenerate the reference fixtures under tests/golden/ from a GPUGA checkout.

Usage:  python tests/golden/make_fixtures.py /path/to/GPUGA

Copies the reference's own regression inputs and outputs (data files only,
no source): the training sets (gzip-compressed), potential.in / ga.in, the
last line of each ga.out (the elite the reference's predict() used,
ga.cu:84-91) and the force/energy/virial outputs it wrote.
"""
import gzip
import os
import shutil
import sys

SETS = {
    # name: (directory in the reference, output suffix, ga.out name)
    "si_diamond": ("tests/si_diamond", "1", "ga1.out"),
    "si_diamond_example": ("examples/si_diamond", "", "ga.out"),
    "hfo2": ("develop/hfo2", "", "ga.out"),
    "nn2b": ("develop/nn2b", "", "ga.out"),
    "wurzite_Si": ("develop/wurzite/Si", "", "ga.out"),
    "wurzite_GaAs": ("develop/wurzite/GaAs", "", "ga.out"),
}


def main(ref_root: str) -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    for name, (rel, suffix, ga_name) in SETS.items():
        src = os.path.join(ref_root, rel)
        dst = os.path.join(here, name)
        os.makedirs(dst, exist_ok=True)
        with open(os.path.join(src, "train.in"), "rb") as f, open(os.path.join(dst, "train.in.gz"), "wb") as raw:
            with gzip.GzipFile(fileobj=raw, mode="wb", compresslevel=9, mtime=0, filename="") as g:
                shutil.copyfileobj(f, g)
        for fn in ("potential.in", "ga.in"):
            shutil.copy(os.path.join(src, fn), os.path.join(dst, fn))
        for kind in ("force", "energy", "virial"):
            shutil.copy(os.path.join(src, f"{kind}{suffix}.out"), os.path.join(dst, f"{kind}.out"))
        with open(os.path.join(src, ga_name)) as f:
            lines = f.read().splitlines()
        with open(os.path.join(dst, "ga_last.out"), "w") as f:
            f.write(lines[-1] + "\n")
        if name == "si_diamond":
            # the full trajectory of the seeded (-DDEBUG) regression run
            shutil.copy(os.path.join(src, ga_name), os.path.join(dst, "ga.out"))
    print("fixtures written to", here)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
