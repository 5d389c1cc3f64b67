"""Neighbor lists and the minimum-image rule pinned to the reference build itself.

oracle/_ref/ref_probe links the unmodified neighbor.cu:30-66 and mic.cuh:20-32 of the
reference (compiled from its own sources by oracle/Makefile, target `ref`).  This test runs it
on the five fixture sets and on 2 M random (box, displacement) inputs, and requires
bit-identical results from

  * the engine's lists (gpuga_engine_neighbors, reference layout NN[N], NL[k*N + i]), and
  * the oracle's FP32 replay with FMA pattern 0, fma(a2, b2, fma(a0, b0, a1 * b1)).

It is skipped where the reference build is absent.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

from gpuga_b200 import Fitness

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROBE = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
SETS = ["si_diamond", "hfo2", "nn2b", "wurzite_Si", "wurzite_GaAs"]

needs_probe = pytest.mark.skipif(not os.access(PROBE, os.X_OK), reason="reference build (oracle/_ref) not present")


def _run_probe(*args):
    subprocess.run([PROBE, *map(str, args)], check=True, stdout=subprocess.DEVNULL, timeout=600)


@needs_probe
@pytest.mark.parametrize("name", SETS)
def test_neighbor_lists_match_the_reference_build(name, golden, built_oracle, tmp_path):
    d = golden(name)
    out = str(tmp_path / "nl.bin")
    _run_probe("neighbors", d, out)
    with open(out, "rb") as f:
        N, M = struct.unpack("ii", f.read(8))
        ref_NN = np.frombuffer(f.read(4 * N), np.int32)
        ref_NL = np.frombuffer(f.read(4 * N * M), np.int32).reshape(M, N)
    with Fitness(d) as e:
        NN, NL = e.neighbors_reference_layout()
        NL = NL.reshape(-1, N)
    assert np.array_equal(NN, ref_NN)
    for i in range(N):
        assert np.array_equal(NL[:NN[i], i], ref_NL[:ref_NN[i], i]), f"atom {i}"
    oNN, onl = built_oracle.OracleSet(d).neighbors()
    assert np.array_equal(oNN, ref_NN)
    ref_csr = np.concatenate([ref_NL[:ref_NN[i], i] for i in range(N)])
    assert np.array_equal(onl, ref_csr)


@needs_probe
def test_minimum_image_matches_the_reference_build(built_oracle, tmp_path):
    n = 2_000_000
    out = str(tmp_path / "mic.bin")
    _run_probe("mic", n, 20240611, out)
    with open(out, "rb") as f:
        (m,) = struct.unpack("i", f.read(4))
        h = np.frombuffer(f.read(4 * 18 * m), np.float32)
        xyz = np.frombuffer(f.read(4 * 3 * m), np.float32)
        ref = np.frombuffer(f.read(4 * 4 * m), np.float32)
    assert m == n
    got = built_oracle.mic_batch(0, h, xyz)
    mism = np.flatnonzero(got.view(np.uint32) != ref.view(np.uint32))
    assert mism.size == 0, f"{mism.size} of {4 * n} values differ, first at {mism[:5]}"
