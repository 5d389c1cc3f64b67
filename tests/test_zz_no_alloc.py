"""gpuga_potential_find_force_noalloc: the allocation-free Potential::find_force.

Callers that may not call cudaMalloc when they need forces (a host that gives
its whole device-memory budget to its own allocator, a plug-in interface that
forbids device allocation after initialisation) use this entry point; its
scratch is a fixed array inside the library.  Two calls in a row must agree
with the allocating entry point (gpuga_potential_create / _update /
_find_force) within the tolerance of the Potential tests (3e-5 of each array's
scale), and a problem larger than the fixed scratch is refused cleanly.

This file is named to run last: it also checks that the shared array gives the
same answer after every other test has used the library."""
import ctypes as C

import numpy as np
import pytest
import torch

from gpuga_b200 import _lib
from tests.helpers import golden_subset, read_elite

pytestmark = pytest.mark.gpu

RTOL_OF_SCALE = 3e-5


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _within(got, want):
    g = got.cpu().numpy().astype(np.float64)
    w = want.cpu().numpy().astype(np.float64)
    scale = max(np.abs(w).max(), 1e-30)
    return np.abs(g - w).max() <= RTOL_OF_SCALE * scale


def _synthetic(name, tmp_path):
    """A small rigid-ion set (4 configurations of the rigid-ion benchmark geometry) and a Tersoff set
    whose scratch, N * max_Na * 56 bytes, sits just under the fixed 64 MiB (2328 atoms x 512)."""
    from gpuga_b200 import synth
    if name == "synth_ri":
        data = synth.make(3, Nc=4)
    else:
        data = synth.diamond_set([4, 4, 4, 4, 3, 2], Nc_force=3)
    d = synth.write_dir(data, str(tmp_path / name))
    return d, synth.teacher_params(data)


# golden sets beyond the fixed scratch are cut to a few configurations (force, energy/virial)
SUBSETS = {"wurzite_GaAs": (4, 8), "hfo2": (1, 1)}


@pytest.mark.parametrize("name", ["si_diamond", "wurzite_GaAs", "hfo2", "nn2b", "synth_ri", "near_limit"])
def test_noalloc_matches_allocating_entry_point(name, golden, built_oracle, tmp_path):
    L = _lib.load()
    if name.startswith("synth") or name == "near_limit":
        d, params = _synthetic(name, tmp_path)
    else:
        d = golden(name)
        if name in SUBSETS:
            d = golden_subset(d, str(tmp_path / name), *SUBSETS[name])
        params = read_elite(d)
    s = built_oracle.OracleSet(d)
    if name == "near_limit":
        need = s.N * s.max_Na * 56
        assert 0.95 * (64 << 20) < need < (64 << 20)
    a = {k: _dev(v) for k, v in s.arrays().items()}
    N, M, Nc = s.N, s.max_Na, s.Nc
    NN = torch.zeros(N, dtype=torch.int32, device="cuda")
    NL = torch.zeros(M * N, dtype=torch.int32, device="cuda")
    _lib.check(L.gpuga_neighbor_compute(Nc, N, M, _ptr(a["Na"]), _ptr(a["Na_sum"]), _ptr(a["r"]), _ptr(a["h"]),
                                        C.c_float(s.cutoff), _ptr(NN), _ptr(NL), None))
    params = np.ascontiguousarray(params, dtype=np.float32)
    pp = params.ctypes.data_as(C.c_void_p)

    def outputs():
        return (torch.zeros(3 * N, dtype=torch.float32, device="cuda"),
                torch.zeros(6 * N, dtype=torch.float32, device="cuda"),
                torch.zeros(N, dtype=torch.float32, device="cuda"))

    args = (Nc, N, _ptr(a["Na"]), _ptr(a["Na_sum"]), M, _ptr(a["type"]), _ptr(a["h"]), _ptr(NN), _ptr(NL),
            _ptr(a["r"]))
    # the existing, allocating entry point
    pot = C.c_void_p()
    _lib.check(L.gpuga_potential_create(s.potential_type, s.num_neurons, C.byref(pot)))
    try:
        _lib.check(L.gpuga_potential_initialize(pot, N, M))
        _lib.check(L.gpuga_potential_update(pot, pp, len(params)))
        ref = outputs()
        _lib.check(L.gpuga_potential_find_force(pot, *args, *(_ptr(t) for t in ref), None))
        torch.cuda.synchronize()
    finally:
        L.gpuga_potential_destroy(pot)
    # two calls in a row of the allocation-free one
    for _ in range(2):
        out = outputs()
        _lib.check(L.gpuga_potential_find_force_noalloc(s.potential_type, s.num_neurons, pp, len(params), *args,
                                                        *(_ptr(t) for t in out), None))
        torch.cuda.synchronize()
        for got, want in zip(out, ref):
            assert _within(got, want)


def test_noalloc_refuses_problems_beyond_its_scratch():
    L = _lib.load()
    params = np.zeros(9, np.float32)
    x = torch.zeros(16, dtype=torch.int32, device="cuda")
    N, M = 1 << 20, 1024  # 1M atoms x 1024 slots: far beyond the fixed scratch
    rc = L.gpuga_potential_find_force_noalloc(1, 0, params.ctypes.data_as(C.c_void_p), 9, 1, N, _ptr(x), _ptr(x), M,
                                              _ptr(x), _ptr(x), _ptr(x), _ptr(x), _ptr(x), _ptr(x), _ptr(x), _ptr(x),
                                              None)
    assert rc == _lib.ERR_ARG
    assert b"limit" in L.gpuga_last_error()
