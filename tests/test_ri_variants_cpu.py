"""RI extensions in the oracle: the charge-neutral variant (potential type 4, anion charge -q)
and the opt-in damped-Coulomb self energy.

ri.cu:40-43 hard-codes cation +q and anion -q/2; type 0 keeps that, type 4 is the ratio -1
variant for 1:1 lattices.  The self energy follows develop/hfo2/find_E.m:10-13 (computed there
and multiplied by 0, so it is off by default).  Both are pinned against a numpy all-pairs sum
of the RI pair energy (ri.cu:77-110) on boxes wider than twice the cutoff, where the single-image
neighbor list is the plain minimum image."""
import math
import os

import numpy as np
import pytest

from gpuga_b200 import synth

KC, ALPHA = 14.399645, 0.2


def _small_set(tmp_path, pt):
    """Two cubic 20 A boxes (cutoff 8 A < half the box) of 6 and 9 ions."""
    rng = np.random.default_rng(4)
    pos, types, Na = [], [], []
    for n in (6, 9):
        pts = []
        while len(pts) < n:  # no pair closer than 1.6 A
            x = rng.uniform(0, 20, 3)
            if all(np.linalg.norm((x - y) - 20 * np.round((x - y) / 20)) > 1.6 for y in pts):
                pts.append(x)
        pos.append(np.array(pts))
        types.append(rng.integers(0, 2, n).astype(np.int32))
        Na.append(n)
    Na = np.array(Na, np.int32)
    N = int(Na.sum())
    allp = np.vstack(pos)
    r = np.concatenate([allp[:, 0], allp[:, 1], allp[:, 2]]).astype(np.float32)
    b = synth.RI_BOUNDS
    data = dict(potential_type=pt, num_neurons=0, cutoff=8.0, w_force=0.1, w_energy=0.2, w_stress=0.7,
                pmin=b[:, 0].astype(np.float32), pmax=b[:, 1].astype(np.float32), Na=Na, Nc_force=1, r=r,
                box9=np.tile(np.array([20, 0, 0, 0, 20, 0, 0, 0, 20], np.float32), 2),
                type=np.concatenate(types), pe_ref=np.zeros(2, np.float32), virial_ref=np.zeros(12, np.float32),
                force_ref=np.zeros(3 * N, np.float32))
    return synth.write_dir(data, str(tmp_path / f"ri{pt}")), data


def _numpy_energy(data, p, pt, self_on):
    """Config energies from ri.cu:77-110 pair by pair (i < j), FP64, plus the find_E.m self term."""
    q0 = p[0]
    ratio = -1.0 if pt == 4 else -0.5
    qq = [q0 * q0 * KC, ratio * q0 * q0 * KC, ratio * ratio * q0 * q0 * KC]
    a = [p[1], p[4], p[7]]
    rho = [p[2], p[5], p[8]]
    c = [p[3], p[6], p[9]]
    rc, d0, al, r0, s = p[10], p[11], p[12], p[13], p[14]
    v_rc = math.erfc(ALPHA * rc) / rc
    dv_rc = -math.erfc(ALPHA * rc) / rc ** 2 - 2 * ALPHA / math.sqrt(math.pi) * math.exp(-ALPHA ** 2 * rc ** 2) / rc
    selfk = ALPHA / math.sqrt(math.pi) + 0.5 * math.erfc(ALPHA * rc) / rc + 0.5 * (
        math.erfc(ALPHA * rc) / rc + 2 * ALPHA / math.sqrt(math.pi) * math.exp(-ALPHA ** 2 * rc ** 2))
    Na = data["Na"]
    N = int(Na.sum())
    r = data["r"].astype(np.float64)
    xyz = np.stack([r[:N], r[N:2 * N], r[2 * N:]], 1)
    out, o = [], 0
    for n in Na:
        E = 0.0
        for i in range(o, o + n):
            for j in range(i + 1, o + n):
                v = xyz[j] - xyz[i]
                v -= 20.0 * np.round(v / 20.0)
                d = float(np.linalg.norm(v))
                if d >= data["cutoff"]:
                    continue
                t = int(data["type"][i] + data["type"][j])
                E += a[t] * math.exp(-d / rho[t]) - c[t] / d ** 6
                E += qq[t] * (math.erfc(ALPHA * d) / d - v_rc - dv_rc * (d - rc))
                if t == 1:
                    E += d0 / (s - 1) * math.exp(-math.sqrt(2 * s) * al * (d - r0))
                    E -= s * d0 / (s - 1) * math.exp(-math.sqrt(2 / s) * al * (d - r0))
        if self_on:
            E -= selfk * sum(qq[0] if data["type"][i] == 0 else qq[2] for i in range(o, o + n))
        out.append(E)
        o += n
    return np.array(out)


@pytest.mark.parametrize("pt,self_on", [(0, False), (4, False), (0, True), (4, True)])
def test_oracle_ri_variants_match_the_pair_sum(tmp_path, built_oracle, pt, self_on):
    d, data = _small_set(tmp_path, pt)
    s = built_oracle.OracleSet(d)
    assert s.potential_type == pt and s.num_vars == 15
    s.set_ri_self(self_on)
    rng = np.random.default_rng(pt + 10 * self_on)
    for _ in range(3):
        p = s.decode(rng.uniform(0, 1, 15).astype(np.float32))
        F, W, pe = s.find_force(p)
        E, _ = s.config_sums(W, pe)
        want = _numpy_energy(data, p, pt, self_on)
        np.testing.assert_allclose(E, want, rtol=1e-11, atol=1e-11 * np.abs(want).max())


def test_self_energy_shifts_only_the_energy(tmp_path, built_oracle):
    """The self term is a per-atom constant: forces and virials are unchanged."""
    d, _ = _small_set(tmp_path, 4)
    s = built_oracle.OracleSet(d)
    p = s.decode(np.full(15, 0.4, np.float32))
    F0, W0, pe0 = s.find_force(p)
    s.set_ri_self(True)
    F1, W1, pe1 = s.find_force(p)
    np.testing.assert_array_equal(F0, F1)
    np.testing.assert_array_equal(W0, W1)
    assert np.all(pe1 < pe0)


def test_type4_potential_in_round_trips(tmp_path):
    """potential.in with type 4 carries 15 bounded parameters, like type 0 (fitness.cu:237-240)."""
    d, data = _small_set(tmp_path, 4)
    txt = open(os.path.join(d, "potential.in")).read().split("\n")
    assert txt[0] == "potential_type 4"
    assert sum(1 for ln in txt if ln.strip()) == 1 + 4 + 15


def test_library_parses_type4_like_the_oracle(tmp_path, built_oracle):
    import ctypes as C

    from gpuga_b200 import _lib
    d, _ = _small_set(tmp_path, 4)
    sz = np.zeros(11, np.int32)
    assert _lib.load().gpuga_parse_inputs(d.encode(), sz.ctypes.data_as(C.c_void_p)) == 0
    s = built_oracle.OracleSet(d)
    assert list(sz[:8]) == [4, 15, 0, s.Nc, s.Nc_force, s.N, s.N_force, s.max_Na]
