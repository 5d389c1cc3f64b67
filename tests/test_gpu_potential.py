"""The reference's plug-in boundary on device arrays in its own layouts:
gpuga_neighbor_compute (Neighbor::compute, neighbor.cu:68-83) and the
gpuga_potential_* calls (Potential, potential.cuh:22-41), FP32 results checked
against the FP64 oracle.

Tolerance: FP32 outputs within 3e-5 of each array's scale (forces, per-atom
virials and site energies), neighbor lists bit-exact."""
import ctypes as C

import numpy as np
import pytest
import torch

from gpuga_b200 import _lib
from tests.helpers import read_elite

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def ptr(t):
    return C.c_void_p(t.data_ptr())


def reference_arrays(s):
    a = s.arrays()
    return {k: dev(v) for k, v in a.items()}


@pytest.mark.parametrize("name", ["si_diamond", "wurzite_Si", "nn2b", "hfo2"])
def test_potential_interface_matches_oracle(name, golden, built_oracle):
    L = _lib.load()
    d = golden(name)
    s = built_oracle.OracleSet(d)
    a = reference_arrays(s)
    N, M, Nc = s.N, s.max_Na, s.Nc
    NN = torch.zeros(N, dtype=torch.int32, device="cuda")
    NL = torch.full((M * N,), -1, dtype=torch.int32, device="cuda")
    _lib.check(L.gpuga_neighbor_compute(Nc, N, M, ptr(a["Na"]), ptr(a["Na_sum"]), ptr(a["r"]), ptr(a["h"]),
                                        C.c_float(s.cutoff), ptr(NN), ptr(NL), None))
    torch.cuda.synchronize()
    oNN, onl = s.neighbors()
    np.testing.assert_array_equal(NN.cpu().numpy(), oNN)
    off = np.concatenate([[0], np.cumsum(oNN)])
    NLh = NL.cpu().numpy()
    for k in range(int(oNN.max())):
        m = oNN > k
        np.testing.assert_array_equal(NLh[k * N + np.arange(N)[m]], onl[off[:-1][m] + k])

    pot = C.c_void_p()
    _lib.check(L.gpuga_potential_create(s.potential_type, s.num_neurons, C.byref(pot)))
    try:
        _lib.check(L.gpuga_potential_initialize(pot, N, M))
        params = read_elite(d).astype(np.float32)
        _lib.check(L.gpuga_potential_update(pot, params.ctypes.data_as(C.c_void_p), len(params)))
        f = torch.zeros(3 * N, dtype=torch.float32, device="cuda")
        w = torch.zeros(6 * N, dtype=torch.float32, device="cuda")
        pe = torch.zeros(N, dtype=torch.float32, device="cuda")
        _lib.check(L.gpuga_potential_find_force(pot, Nc, N, ptr(a["Na"]), ptr(a["Na_sum"]), M, ptr(a["type"]),
                                                ptr(a["h"]), ptr(NN), ptr(NL), ptr(a["r"]), ptr(f), ptr(w), ptr(pe),
                                                None))
        torch.cuda.synchronize()
    finally:
        L.gpuga_potential_destroy(pot)
    oF, oW, ope = s.find_force(params.astype(np.float64))
    for got, want in ((f, oF), (w, oW), (pe, ope)):
        g = got.cpu().numpy().astype(np.float64)
        scale = np.abs(want).max()
        assert np.abs(g - want).max() <= 3e-5 * scale


def test_potential_argument_checks():
    L = _lib.load()
    pot = C.c_void_p()
    assert L.gpuga_potential_create(9, 0, C.byref(pot)) == _lib.ERR_UNSUPPORTED
    _lib.check(L.gpuga_potential_create(1, 0, C.byref(pot)))
    try:
        bad = np.zeros(3, np.float32)
        assert L.gpuga_potential_update(pot, bad.ctypes.data_as(C.c_void_p), 3) == _lib.ERR_ARG
        x = torch.zeros(8, dtype=torch.int32, device="cuda")
        rc = L.gpuga_potential_find_force(pot, 1, 2, ptr(x), ptr(x), 2, ptr(x), ptr(x), ptr(x), ptr(x), ptr(x),
                                          ptr(x), ptr(x), ptr(x), None)
        assert rc == _lib.ERR_ARG  # not initialised
    finally:
        L.gpuga_potential_destroy(pot)
