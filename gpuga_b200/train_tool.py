"""DFT data -> train.in (the reference's develop/wurzite/*/construct_train_in.cpp).

Reads, like the reference program, from standard input: `Nc_force Nc_energy`
followed by one DFT file name per configuration (force configurations first),
and writes train.in.  A force file holds `Na`, the box (9 numbers, cell
vectors a, b, c as rows) and Na lines `type x y z fx fy fz`; an energy/virial
file holds `Na`, `energy` and six virial (or stress) components, the box, and
Na lines `type x y z`.  Energy/virial cells are replicated NA x NB x NC times
(energy and virial scale with the cell count); stresses from VASP in kbar are
turned into virials (x volume / 1602.18); DELTA_E shifts the energy per atom.

The reference sets these through compile-time constants; here they are
options, with the same meaning:

  --cells NA NB NC            NA, NB, NC (construct_train_in.cpp:47-49)
  --delta-e E                 DELTA_E, eV per atom (:52)
  --no-stress-kbar            STRESS_IN_KBAR = false (:51)
  --force-types {file,zero}   force configurations keep the file's types, or start from 0
                              (the GaAs/GaP/InAs/InP/ZnSe copies, :143)
  --z-bands lo:hi,...         CHANGE_TYPE for force configurations: type 1 where lo < z < hi
                              for any band (:144-150; those copies use 1.5:4.5,7.5:10.5,13.5:17)
  --ev-type-map t0,t1,...     CHANGE_TYPE for energy/virial configurations: the m-th atom of
                              the cell gets type t_m (TYPE[], :55) ...
  --ev-map-skip-last K        ... except the last K configurations (n < Nc - 3, :222)
  --ev-types {file,zero}      types of the configurations the map does not cover (:233)
  --max-cell-size N           CELL_SIZE, the largest energy/virial cell (:46)

Arithmetic follows the reference's FP32 operation order (numbers are read as
FP32, products and sums of FP32 values are rounded to FP32, the kbar factor is
formed in FP64) and numbers are printed with %g, so the same inputs give the
same train.in text.

    python -m gpuga_b200.train_tool --cells 4 4 3 --z-bands 1.5:4.5,7.5:10.5,13.5:17 \\
        --force-types zero --ev-type-map 0,1,1,0 --ev-map-skip-last 3 < input.txt
"""
from __future__ import annotations

import argparse
import ctypes
import os
import sys

import numpy as np

_libc = ctypes.CDLL(None)
_libc.strtof.restype = ctypes.c_float
_libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]

f32 = np.float32


def _read_f32(tok: str) -> np.float32:
    """FP32 parse of one token, as fscanf("%f") (strtof, one rounding)."""
    return f32(_libc.strtof(tok.encode(), None))


def _g(x) -> str:
    return "%g" % float(x)


class _Tokens:
    def __init__(self, path: str):
        with open(path) as f:
            self.tok = f.read().split()
        self.path = path
        self.k = 0

    def _next(self) -> str:
        if self.k >= len(self.tok):
            raise ValueError(f"Reading error: {self.path} ended early")
        self.k += 1
        return self.tok[self.k - 1]

    def int(self) -> int:
        return int(self._next())

    def f32(self) -> np.float32:
        return _read_f32(self._next())


def _in_bands(z: np.float32, bands) -> bool:
    return any(lo < float(z) < hi for lo, hi in bands)


def build(files: list[str], nc_force: int, cells=(1, 1, 1), delta_e: float = 0.0, stress_kbar: bool = True,
          force_types: str = "file", z_bands=(), ev_type_map=None, ev_map_skip_last: int = 0,
          ev_types: str = "file", max_cell_size: int | None = None) -> str:
    """train.in text for the DFT files (force configurations first)."""
    NA, NB, NC = (int(c) for c in cells)
    NABC = NA * NB * NC
    Nc = len(files)
    if not 0 <= nc_force <= Nc:
        raise ValueError("invalid number of force configurations")
    out = [f"{Nc} {nc_force}\n"]
    Na = []
    for n, path in enumerate(files):
        na = _Tokens(path).int()
        if n >= nc_force:
            if max_cell_size is not None and na > max_cell_size:
                raise ValueError(f"{path}: {na} atoms, more than the cell size {max_cell_size}")
            na *= NABC
        Na.append(na)
        out.append(f"{na}\n")
    for n in range(nc_force):
        t = _Tokens(files[n])
        na = t.int()
        box = [t.f32() for _ in range(9)]
        out.append("".join(_g(b) + " " for b in box) + "\n")
        for _ in range(na):
            typ = t.int()
            r = [t.f32() for _ in range(3)]
            f = [t.f32() for _ in range(3)]
            if force_types == "zero":
                typ = 0
            if z_bands and _in_bands(r[2], z_bands):
                typ = 1
            out.append(f"{typ} " + " ".join(_g(v) for v in r + f) + "\n")
    de = f32(delta_e)
    for n in range(nc_force, Nc):
        t = _Tokens(files[n])
        na = t.int()
        energy = t.f32()
        virial = [t.f32() for _ in range(6)]
        box = [t.f32() for _ in range(9)]
        energy = f32(f32(f32(f32(energy / f32(na)) + de) * f32(na)) * f32(NABC))
        virial = [f32(v * f32(NABC)) for v in virial]
        if stress_kbar:
            b = box
            vol = f32(f32(b[0] * f32(b[4] * b[8] - b[5] * b[7])) + f32(b[1] * f32(b[5] * b[6] - b[3] * b[8]))) \
                + f32(b[2] * f32(b[3] * b[7] - b[4] * b[6]))
            vol = f32(vol)
            factor = float(vol) / 1602.18  # float / double literal: FP64
            virial = [f32(float(v) * factor) for v in virial]
        out.append(" ".join(_g(v) for v in [energy] + virial) + "\n")
        out.append("".join(_g(box[k] * f32(NA)) + " " for k in range(3))
                   + "".join(_g(box[k] * f32(NB)) + " " for k in range(3, 6))
                   + "".join(_g(box[k] * f32(NC)) + " " for k in range(6, 9)) + "\n")
        types, rs = [], []
        for _ in range(na):
            types.append(t.int())
            rs.append([t.f32() for _ in range(3)])
        use_map = ev_type_map is not None and n < Nc - ev_map_skip_last
        for ia in range(NA):
            for ib in range(NB):
                for ic in range(NC):
                    a, bb, c = f32(ia), f32(ib), f32(ic)
                    d = [f32(f32(f32(box[k] * a) + f32(box[3 + k] * bb)) + f32(box[6 + k] * c)) for k in range(3)]
                    for m in range(na):
                        if use_map:
                            typ = ev_type_map[m]
                        else:
                            typ = types[m] if ev_types == "file" else 0
                        out.append(f"{typ} " + " ".join(_g(f32(rs[m][k] + d[k])) for k in range(3)) + "\n")
    return "".join(out)


def _bands(s: str):
    if not s:
        return ()
    return tuple(tuple(float(v) for v in b.split(":")) for b in s.split(","))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="DFT data -> train.in (construct_train_in.cpp)")
    ap.add_argument("--cells", type=int, nargs=3, default=[1, 1, 1], metavar=("NA", "NB", "NC"))
    ap.add_argument("--delta-e", type=float, default=0.0)
    ap.add_argument("--no-stress-kbar", action="store_true")
    ap.add_argument("--force-types", choices=["file", "zero"], default="file")
    ap.add_argument("--z-bands", default="")
    ap.add_argument("--ev-type-map", default="")
    ap.add_argument("--ev-map-skip-last", type=int, default=0)
    ap.add_argument("--ev-types", choices=["file", "zero"], default="file")
    ap.add_argument("--max-cell-size", type=int, default=None)
    ap.add_argument("--output", default="train.in")
    ap.add_argument("--dir", default=".", help="directory the file names are relative to")
    a = ap.parse_args(argv)
    tok = sys.stdin.read().split()
    nc_force, nc_energy = int(tok[0]), int(tok[1])
    files = [os.path.join(a.dir, f) for f in tok[2:2 + nc_force + nc_energy]]
    if len(files) != nc_force + nc_energy:
        print("Reading error: not enough file names", file=sys.stderr)
        return 1
    text = build(files, nc_force, a.cells, a.delta_e, not a.no_stress_kbar, a.force_types, _bands(a.z_bands),
                 [int(v) for v in a.ev_type_map.split(",")] if a.ev_type_map else None, a.ev_map_skip_last,
                 a.ev_types, a.max_cell_size)
    with open(os.path.join(a.dir, a.output) if not os.path.isabs(a.output) else a.output, "w") as f:
        f.write(text)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
