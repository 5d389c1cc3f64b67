"""Degenerate and ragged configurations on the batched path, against the FP64 oracle.

Each potential's set gets, both as force configurations and as energy/virial configurations, two
atoms 17 A apart in a 20 A box (no neighbors; the reference's input rules ask for >= 2 atoms per
configuration), a dimer (one bond per atom) and a dimer with a third atom beyond the cutoff, next
to ordinary configurations of the workload.  Atoms without neighbors
must contribute exactly nothing, single-bond atoms must take the zeta = 0 branch of the bond order
(minimal_tersoff.cu:178-185), and the work-item planning must cope with configurations of 2-3
atoms beside hundreds.  Tolerances as in the main parity file: fitness 1e-6 relative, energies
2e-6 of the set's scale, forces 2e-5 of the force scale.
"""
import numpy as np
import pytest

from gpuga_b200 import Fitness, synth
from tests.helpers import oracle_targets

pytestmark = pytest.mark.gpu

SPEC_KEYS = ("potential_type", "num_neurons", "cutoff", "w_force", "w_energy", "w_stress", "pmin", "pmax", "ga",
             "nn2b_r1", "nn2b_r2")


def _split(data):
    Na, r, box9, t = data["Na"], data["r"], data["box9"], data["type"]
    N = int(Na.sum())
    out, o = [], 0
    for c, n in enumerate(Na):
        pos = np.stack([r[o:o + n], r[N + o:N + o + n], r[2 * N + o:2 * N + o + n]], 1).astype(np.float64)
        out.append((pos, box9[9 * c:9 * c + 9].reshape(3, 3).astype(np.float64), t[o:o + n].copy()))
        o += n
    return out


def _edge_set(workload, built_oracle):
    base = synth.make(workload, Nc=4, seed=5)
    spec = {k: base[k] for k in SPEC_KEYS if k in base}
    cfgs = _split(base)
    Ncf = int(base["Nc_force"])
    box = np.eye(3) * 20.0
    d = {1: 2.35, 3: 2.1, 4: 2.4}[workload]
    t2 = np.array([0, 1 if workload == 3 else 0], np.int32)
    lone = (np.array([[5.0, 5.0, 5.0], [15.0, 15.0, 15.0]]), box, t2.copy())
    dimer = (np.array([[5.0, 5.0, 5.0], [5.0 + d, 5.0, 5.0]]), box, t2)
    trio = (np.array([[5.0, 5.0, 5.0], [5.0, 5.0 + d, 5.0], [15.0, 15.0, 15.0]]), box,
            np.array([0, t2[1], t2[1]], np.int32))
    edge = [lone, dimer, trio]
    configs = edge + cfgs[:Ncf] + edge + cfgs[Ncf:]
    data = synth._assemble(configs, len(edge) + Ncf, spec)
    data["teacher01"] = base["teacher01"]
    return synth.fill_targets(data, oracle_targets(built_oracle))


def _oracle_set(built_oracle, data, tmp_path):
    s = built_oracle.OracleSet(synth.write_dir(data, str(tmp_path / "set")))
    if int(data["potential_type"]) == 3:
        s.set_nn2b(float(data["nn2b_r1"]), float(data["nn2b_r2"]), False)
    return s


@pytest.mark.parametrize("workload", [1, 3, 4])
def test_lone_atoms_dimers_and_ragged_sizes(workload, built_oracle, tmp_path):
    data = _edge_set(workload, built_oracle)
    s = _oracle_set(built_oracle, data, tmp_path)
    kw = dict(nn2b_r1=float(data["nn2b_r1"]), nn2b_r2=float(data["nn2b_r2"])) if workload == 4 else {}
    P = 40
    pop = synth.population(data, P, seed=3)
    with Fitness(arrays=data, **kw) as e:
        NN, _ = e.neighbors()
        assert NN.min() == 0  # the lone atoms and the far third atoms
        fit = np.asarray(e.compute(P, pop))
        E, _, _ = e.config_results(P)
        forces = e.batched_forces(pop[:3])
    ofit = s.fitness(pop)
    assert (np.abs(fit - ofit) / np.abs(ofit)).max() <= 1e-6
    Ncf, Nf = s.Nc_force, s.N_force
    for p in range(3):
        oF, oW, ope = s.find_force(s.decode(pop[p]))
        oE, _ = s.config_sums(oW, ope)
        assert np.abs(E[p, Ncf:] - oE[Ncf:]).max() <= 2e-6 * np.abs(oE[Ncf:]).max()
        assert E[p, Ncf] == 0.0  # the configuration of two isolated atoms
        oFf = np.stack([oF[:Nf], oF[s.N:s.N + Nf], oF[2 * s.N:2 * s.N + Nf]])
        assert np.abs(forces[p] - oFf).max() <= 2e-5 * np.abs(oFf).max()
        assert np.all(forces[p][:, :2] == 0.0)  # the isolated atoms of the first force configuration
