"""Shared helpers of the test suite (reference outputs, synthetic sets)."""
import os
import tempfile

import numpy as np

from gpuga_b200 import synth


def read_elite(directory: str) -> np.ndarray:
    """Decoded parameters of the last ga.out line (the elite predict() used, ga.cu:84-91)."""
    with open(os.path.join(directory, "ga_last.out")) as f:
        return np.array([float(v) for v in f.read().split()[2:]], np.float64)


def reference_outputs(directory: str):
    fo = np.loadtxt(os.path.join(directory, "force.out"), ndmin=2)
    eo = np.loadtxt(os.path.join(directory, "energy.out"), ndmin=2)
    vo = np.loadtxt(os.path.join(directory, "virial.out"), ndmin=2)
    return fo, eo, vo


def config_totals(s, F, W, pe):
    """Split per-atom arrays into (force-config forces [Nf,3], E of E/V configs, W of E/V configs [6*nEV])."""
    N, Nf, Nc, Ncf = s.N, s.N_force, s.Nc, s.Nc_force
    Fp = np.stack([F[:Nf], F[N:N + Nf], F[2 * N:2 * N + Nf]], 1)
    E, Wc = s.config_sums(W, pe)
    Wp = np.concatenate([Wc[k * Nc + Ncf:(k + 1) * Nc] for k in range(6)])
    return Fp, E[Ncf:], Wp


def oracle_targets(oracle_mod):
    def evaluate(data, params):
        d = synth.write_dir(data, tempfile.mkdtemp(prefix="gpuga_synth_"))
        s = oracle_mod.OracleSet(d)
        if int(data["potential_type"]) == 3:
            s.set_nn2b(data.get("nn2b_r1", 7.0), data.get("nn2b_r2", 8.0), False)
        if data.get("ri_self_energy"):
            s.set_ri_self(True)
        return s.find_force(params)
    return evaluate


def synthetic_dir(oracle_mod, config: int, Nc: int, tmpdir: str, seed=None) -> tuple[str, dict]:
    data = synth.make(config, seed=seed, Nc=Nc)
    data = synth.fill_targets(data, oracle_targets(oracle_mod))
    return synth.write_dir(data, tmpdir), data


def golden_subset(src: str, dst: str, n_force: int, n_ev: int) -> str:
    """A smaller copy of a training set: its first n_force force configurations and first n_ev
    energy/virial configurations, train.in in the reference format (fitness.cu:95-148), the other
    input files unchanged."""
    import shutil
    os.makedirs(dst, exist_ok=True)
    for fn in os.listdir(src):
        if fn != "train.in":
            shutil.copy(os.path.join(src, fn), os.path.join(dst, fn))
    with open(os.path.join(src, "train.in")) as f:
        lines = [ln for ln in f.read().splitlines() if ln.strip()]
    Nc, Ncf = (int(v) for v in lines[0].split()[:2])
    Na = [int(lines[1 + c].split()[0]) for c in range(Nc)]
    blocks, pos = [], 1 + Nc
    for c in range(Nc):
        n = Na[c] + 1 + (1 if c >= Ncf else 0)
        blocks.append(lines[pos:pos + n])
        pos += n
    keep = list(range(min(n_force, Ncf))) + list(range(Ncf, min(Ncf + n_ev, Nc)))
    kf = min(n_force, Ncf)
    out = [f"{len(keep)} {kf}"] + [str(Na[c]) for c in keep]
    for c in keep:
        out += blocks[c]
    with open(os.path.join(dst, "train.in"), "w") as f:
        f.write("\n".join(out) + "\n")
    return dst
