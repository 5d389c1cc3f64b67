"""Seeded synthetic training sets in GPUGA's formats.

Five workloads (sizes from the benchmark definitions of this project):

  1  minimal-Tersoff Si: 20 periodic 64-atom diamond cells (2x2x2 conventional,
     a = 5.43 A), isotropic strain U(-2 %, +2 %), displacements N(0, 0.05 A),
     cutoff 3.0 A, population 100.
  2  batched minimal-Tersoff Si: 500 configurations of 8/64/216/512 atoms
     (1..4^3 diamond supercells), strain U(+-3 %), displacements N(0, 0.1 A),
     population 1000.
  3  rigid-ion binary oxide: 300 configurations of 96..324 atoms in
     wurtzite-type (4-atom units) and fluorite-type (12-atom cells) lattices,
     strain U(+-2 %), displacements N(0, 0.08 A), cutoff 8 A, population 400.
  4  NN 2-body Si: MLP 1-16-16-1 (321 weights), 200 diamond cells of 64 or 216
     atoms, displacements N(0, 0.15 A), cutoff 5 A with a 4..5 A taper,
     teacher weights N(0, 0.3), population 200.
  5  serving mix: jobs drawn from workloads 1-3 with 20..500 configurations.

Every set splits its configurations as the reference requires (force
configurations first, fitness.cu:95-148): Nc_force = floor(Nc / 2).  Targets
come from a teacher parameter vector through a caller-supplied evaluator
``evaluate(data, params_fp64) -> (F[3N], W[6N], pe[N])``.
"""
from __future__ import annotations

import os

import numpy as np

DIAMOND = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                    [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]], np.float64)
FLUORITE_CATION = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]], np.float64)
FLUORITE_ANION = np.array([[x, y, z] for x in (.25, .75) for y in (.25, .75) for z in (.25, .75)], np.float64)

# bounds of examples/si_diamond/potential.in (D0, alpha, r0, S, n, beta, h, R1, R2)
SI_TERSOFF_BOUNDS = np.array([[2.9, 3.3], [1.3, 1.5], [2.2, 2.4], [2, 2], [0.5, 0.8], [0, 0.4], [-0.8, -0.6],
                              [2.8, 2.8], [3.2, 3.2]], np.float32)
# Q0, A00 rho00 C00, A01 rho01 C01, A11 rho11 C11, Coulomb cutoff, D0 alpha r0 S
RI_BOUNDS = np.array([[2.0, 2.6], [0, 0], [1, 1], [0, 0], [1000, 3000], [0.25, 0.35], [0, 50],
                      [10000, 25000], [0.12, 0.20], [10, 40], [8, 8], [0, 0.5], [1, 2], [2.0, 2.5], [2, 2]],
                     np.float32)


def _f32(x):
    return np.asarray(x, np.float32)


def _decode(pmin, pmax, x01):
    """FP32 decode of fitness.cu:320-324 (no contraction)."""
    a = _f32(pmin)
    b = _f32(_f32(pmax) - a)
    return _f32(a + _f32(b * _f32(x01)))


def _structure(frac_unit, lattice, reps):
    n1, n2, n3 = reps
    shifts = np.array([[i, j, k] for i in range(n1) for j in range(n2) for k in range(n3)], np.float64)
    frac = (frac_unit[None, :, :] + shifts[:, None, :]).reshape(-1, 3) / np.array([n1, n2, n3], np.float64)
    cell = lattice * np.array([n1, n2, n3], np.float64)[:, None]  # rows = cell vectors
    return frac, cell


def _config(rng, frac, cell, types, strain, sigma):
    eps = rng.uniform(-strain, strain)
    cell = cell * (1.0 + eps)
    pos = frac @ cell + rng.normal(0.0, sigma, size=(len(frac), 3))
    return pos, cell, np.asarray(types, np.int32)


def _assemble(configs, Nc_force, spec):
    Na = np.array([len(c[0]) for c in configs], np.int32)
    N = int(Na.sum())
    r = np.zeros(3 * N, np.float32)
    box9 = np.zeros(9 * len(configs), np.float32)
    types = np.zeros(N, np.int32)
    o = 0
    for c, (pos, cell, t) in enumerate(configs):
        n = len(pos)
        for k in range(3):
            r[k * N + o:k * N + o + n] = pos[:, k]
        box9[9 * c:9 * c + 9] = cell.reshape(-1)  # file order: a, b, c vectors
        types[o:o + n] = t
        o += n
    d = dict(spec)
    d.update(Na=Na, Nc_force=int(Nc_force), type=types, r=r, box9=box9,
             pe_ref=np.zeros(len(configs), np.float32), virial_ref=np.zeros(6 * len(configs), np.float32),
             force_ref=np.zeros(3 * N, np.float32))
    return d


def make(config: int, seed: int | None = None, Nc: int | None = None, neurons: int | None = None) -> dict:
    """Geometry, bounds, weights, GA sizes and the teacher for one workload (targets still zero).
    `neurons` sets the NN2B hidden width of workload 4 (16 by default; the reference holds at most 10)."""
    seed = config if seed is None else seed
    rng = np.random.default_rng(seed)
    a_si = 5.43
    if config in (1, 2):
        if config == 1:
            Nc = Nc or 20
            reps_list = [2] * Nc
            strain, sigma, P = 0.02, 0.05, 100
        else:
            Nc = Nc or 500
            reps_list = list(rng.choice([1, 2, 3, 4], size=Nc))
            strain, sigma, P = 0.03, 0.1, 1000
        lat = np.eye(3) * a_si
        configs = []
        for n in reps_list:
            frac, cell = _structure(DIAMOND, lat, (n, n, n))
            configs.append(_config(rng, frac, cell, np.zeros(len(frac)), strain, sigma))
        spec = dict(potential_type=1, num_neurons=0, cutoff=3.0, w_force=0.05, w_energy=0.15, w_stress=0.8,
                    pmin=SI_TERSOFF_BOUNDS[:, 0].copy(), pmax=SI_TERSOFF_BOUNDS[:, 1].copy(),
                    ga=dict(population_size=P, parent_number=P // 2, mutation_rate=0.2, maximum_generation=1000))
        teacher = rng.uniform(0, 1, size=9).astype(np.float32)
    elif config == 3:
        Nc = Nc or 300
        a_w, c_w, u = 3.25, 5.21, 0.382
        wz_lat = np.array([[a_w, 0, 0], [-a_w / 2, a_w * np.sqrt(3) / 2, 0], [0, 0, c_w]])
        wz_frac = np.array([[1 / 3, 2 / 3, 0], [2 / 3, 1 / 3, .5], [1 / 3, 2 / 3, u], [2 / 3, 1 / 3, .5 + u]])
        wz_types = [0, 0, 1, 1]
        fl_lat = np.eye(3) * 5.10
        fl_frac = np.vstack([FLUORITE_CATION, FLUORITE_ANION])
        fl_types = [0] * 4 + [1] * 8
        wz_reps = [(4, 3, 2), (3, 3, 3), (4, 4, 2), (3, 3, 4), (4, 4, 3), (5, 5, 2), (3, 3, 6), (5, 4, 3),
                   (4, 4, 4), (6, 4, 3), (9, 3, 3)]
        fl_reps = [(2, 2, 2), (3, 2, 2), (4, 2, 2), (3, 3, 2), (4, 3, 2), (3, 3, 3)]
        configs = []
        for c in range(Nc):
            if rng.uniform() < 0.5:
                reps = wz_reps[rng.integers(len(wz_reps))]
                frac, cell = _structure(wz_frac, wz_lat, reps)
                t = np.tile(wz_types, int(np.prod(reps)))
            else:
                reps = fl_reps[rng.integers(len(fl_reps))]
                frac, cell = _structure(fl_frac, fl_lat, reps)
                t = np.tile(fl_types, int(np.prod(reps)))
            configs.append(_config(rng, frac, cell, t, 0.02, 0.08))
        spec = dict(potential_type=0, num_neurons=0, cutoff=8.0, w_force=0.1, w_energy=0.2, w_stress=0.7,
                    pmin=RI_BOUNDS[:, 0].copy(), pmax=RI_BOUNDS[:, 1].copy(),
                    ga=dict(population_size=400, parent_number=200, mutation_rate=0.2, maximum_generation=1000))
        teacher = rng.uniform(0, 1, size=15).astype(np.float32)
    elif config == 4:
        Nc = Nc or 200
        n = neurons or 16
        nv = n * (n + 4) + 1
        lat = np.eye(3) * a_si
        configs = []
        for c in range(Nc):
            reps = 2 if rng.uniform() < 0.5 else 3
            frac, cell = _structure(DIAMOND, lat, (reps, reps, reps))
            configs.append(_config(rng, frac, cell, np.zeros(len(frac)), 0.0, 0.15))
        spec = dict(potential_type=3, num_neurons=n, cutoff=5.0, w_force=0.4, w_energy=0.3, w_stress=0.3,
                    pmin=np.full(nv, -3.0, np.float32), pmax=np.full(nv, 3.0, np.float32), nn2b_r1=4.0,
                    nn2b_r2=5.0,
                    ga=dict(population_size=200, parent_number=100, mutation_rate=0.2, maximum_generation=1000))
        w = np.clip(rng.normal(0.0, 0.3, size=nv), -3, 3)
        teacher = ((w + 3.0) / 6.0).astype(np.float32)
    else:
        raise ValueError(f"unknown workload {config}")
    data = _assemble(configs, len(configs) // 2, spec)
    data["teacher01"] = teacher
    data["name"] = f"workload{config}"
    return data


def diamond_set(reps_list, Nc_force: int, seed: int = 11, strain: float = 0.03, sigma: float = 0.1,
                P: int = 64) -> dict:
    """Minimal-Tersoff Si set of diamond supercells reps x reps x reps (8 reps^3 atoms each), with the
    bounds and teacher draw of workload 2 -- e.g. a few configurations of thousands of atoms."""
    rng = np.random.default_rng(seed)
    configs = []
    for n in reps_list:
        frac, cell = _structure(DIAMOND, np.eye(3) * 5.43, (n, n, n))
        configs.append(_config(rng, frac, cell, np.zeros(len(frac)), strain, sigma))
    spec = dict(potential_type=1, num_neurons=0, cutoff=3.0, w_force=0.05, w_energy=0.15, w_stress=0.8,
                pmin=SI_TERSOFF_BOUNDS[:, 0].copy(), pmax=SI_TERSOFF_BOUNDS[:, 1].copy(),
                ga=dict(population_size=P, parent_number=P // 2, mutation_rate=0.2, maximum_generation=1000))
    data = _assemble(configs, Nc_force, spec)
    data["teacher01"] = rng.uniform(0, 1, size=9).astype(np.float32)
    data["name"] = "diamond_set"
    return data


def teacher_params(data) -> np.ndarray:
    return _decode(data["pmin"], data["pmax"], data["teacher01"]).astype(np.float64)


def fill_targets(data: dict, evaluate) -> dict:
    """Targets from the teacher: config energies and virials (E/V configs) and per-atom forces (force configs)."""
    F, W, pe = evaluate(data, teacher_params(data))
    Na = data["Na"]
    N = int(Na.sum())
    Nc = len(Na)
    starts = np.concatenate([[0], np.cumsum(Na)[:-1]])
    E = np.add.reduceat(pe, starts)
    Wc = np.stack([np.add.reduceat(W[k * N:(k + 1) * N], starts) for k in range(6)])
    out = dict(data)
    Ncf = data["Nc_force"]
    pe_ref = np.zeros(Nc, np.float32)
    pe_ref[Ncf:] = E[Ncf:]
    vir = np.zeros(6 * Nc, np.float32)
    for k in range(6):
        vir[k * Nc + Ncf:(k + 1) * Nc] = Wc[k, Ncf:]
    Nf = int(Na[:Ncf].sum())
    fref = np.zeros(3 * N, np.float32)
    for k in range(3):
        fref[k * N:k * N + Nf] = F[k * N:k * N + Nf]
    out.update(pe_ref=pe_ref, virial_ref=vir, force_ref=fref)
    return out


def write_dir(data: dict, path: str) -> str:
    """Writes potential.in, train.in and ga.in in the reference's formats."""
    os.makedirs(path, exist_ok=True)
    pt = int(data["potential_type"])
    names = {1: ["D0", "alpha", "r0", "S", "n", "beta", "h", "R1", "R2"],
             0: ["Q0", "A00", "rho00", "C00", "A01", "rho01", "C01", "A11", "rho11", "C11", "cutoff", "D0",
                 "alpha", "r0", "S"]}
    names[4] = names[0]
    with open(os.path.join(path, "potential.in"), "w") as f:
        f.write(f"potential_type {pt}\n")
        if pt == 3:
            f.write(f"num_neurons {int(data['num_neurons'])}\n")
        f.write(f"cutoff {float(data['cutoff']):.9g}\n")
        f.write(f"weight_force {float(data['w_force']):.9g}\nweight_energy {float(data['w_energy']):.9g}\n"
                f"weight_virial {float(data['w_stress']):.9g}\n")
        if pt != 3:
            for nm, lo, hi in zip(names.get(pt, [f"p{m}" for m in range(len(data['pmin']))]), data["pmin"],
                                  data["pmax"]):
                f.write(f"{nm} {float(lo):.9g} {float(hi):.9g}\n")
    ga = data.get("ga", {})
    with open(os.path.join(path, "ga.in"), "w") as f:
        f.write(f"maximum_generation {ga.get('maximum_generation', 1000)}\n")
        f.write(f"population_size {ga.get('population_size', 200)}\n")
        f.write(f"parent_number {ga.get('parent_number', 100)}\n")
        f.write(f"mutation_rate {ga.get('mutation_rate', 0.2)}\n")
    Na = data["Na"]
    Nc = len(Na)
    N = int(Na.sum())
    Ncf = int(data["Nc_force"])
    r, box9, t = data["r"], data["box9"], data["type"]
    fref, pe_ref, vir = data["force_ref"], data["pe_ref"], data["virial_ref"]
    lines = [f"{Nc} {Ncf}"]
    lines += [str(int(n)) for n in Na]
    o = 0
    g = lambda v: f"{float(np.float32(v)):.9g}"  # noqa: E731  (round-trips FP32 exactly)
    for c in range(Nc):
        if c >= Ncf:
            lines.append(" ".join(g(v) for v in [pe_ref[c]] + [vir[k * Nc + c] for k in range(6)]))
        lines.append(" ".join(g(v) for v in box9[9 * c:9 * c + 9]))
        for k in range(int(Na[c])):
            i = o + k
            row = [str(int(t[i])), g(r[i]), g(r[N + i]), g(r[2 * N + i])]
            if c < Ncf:
                row += [g(fref[i]), g(fref[N + i]), g(fref[2 * N + i])]
            lines.append(" ".join(row))
        o += int(Na[c])
    with open(os.path.join(path, "train.in"), "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def population(data: dict, P: int, seed: int = 7, near_teacher: float | None = None) -> np.ndarray:
    """A population in [0,1]; with near_teacher=s, individuals scatter N(0, s) around the teacher."""
    rng = np.random.default_rng(seed)
    d = len(data["pmin"])
    if near_teacher is None:
        return rng.uniform(0, 1, size=(P, d)).astype(np.float32)
    x = data["teacher01"][None, :] + rng.normal(0, near_teacher, size=(P, d))
    return np.clip(x, 0, 1).astype(np.float32)
