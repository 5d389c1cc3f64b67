"""ctypes front-end of the CPU oracle (oracle/oracle.cpp) -- test infrastructure.

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  It is the checker, never the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    """Compile oracle/oracle.cpp into oracle/_build/liboracle.so (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.oracle_load.restype = C.c_void_p
        L.oracle_load.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.c_int]
        L.oracle_free.argtypes = [C.c_void_p]
        L.oracle_info.argtypes = [C.c_void_p, C.c_void_p]
        L.oracle_scalars.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_bounds.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_arrays.argtypes = [C.c_void_p] + [C.c_void_p] * 8
        L.oracle_neighbors.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_set_nn2b.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int]
        L.oracle_set_ri_self.argtypes = [C.c_void_p, C.c_int]
        L.oracle_decode.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_find_force.argtypes = [C.c_void_p] + [C.c_void_p] * 4
        L.oracle_config_sums.argtypes = [C.c_void_p] + [C.c_void_p] * 4
        L.oracle_fitness.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_fitness_arrays.restype = C.c_double
        L.oracle_fitness_arrays.argtypes = [C.c_void_p] + [C.c_void_p] * 4
        L.oracle_num_threads.restype = C.c_int
        L.oracle_mic_batch.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_ga_run.restype = C.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


FITNESS_CB = C.CFUNCTYPE(None, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_void_p)


class OracleSet:
    """A training set parsed and neighbor-listed by the oracle (FP32 rules of
    the reference), with FP64 force/energy/virial and fitness evaluation."""

    def __init__(self, directory: str, fma_mode: int = 0):
        L = lib()
        err = C.create_string_buffer(256)
        h = L.oracle_load(directory.encode(), fma_mode, err, 256)
        if not h:
            raise ValueError(f"oracle: {err.value.decode()}")
        self._h = C.c_void_p(h)
        info = np.zeros(9, np.int32)
        L.oracle_info(self._h, _p(info))
        (self.potential_type, self.num_vars, self.num_neurons, self.Nc, self.Nc_force, self.N,
         self.N_force, self.max_Na, self.num_bonds) = (int(v) for v in info)
        fw = np.zeros(4, np.float32)
        norms = np.zeros(3, np.float64)
        L.oracle_scalars(self._h, _p(fw), _p(norms))
        self.cutoff, self.w_force, self.w_energy, self.w_stress = (float(v) for v in fw)
        self.norm_force, self.norm_energy, self.norm_virial = (float(v) for v in norms)
        self.pmin = np.zeros(self.num_vars, np.float32)
        self.pmax = np.zeros(self.num_vars, np.float32)
        L.oracle_bounds(self._h, _p(self.pmin), _p(self.pmax))

    def close(self):
        if getattr(self, "_h", None):
            lib().oracle_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def arrays(self) -> dict:
        N, Nc = self.N, self.Nc
        out = dict(Na=np.zeros(Nc, np.int32), Na_sum=np.zeros(Nc, np.int32), type=np.zeros(N, np.int32),
                   r=np.zeros(3 * N, np.float32), h=np.zeros(18 * Nc, np.float32),
                   pe_ref=np.zeros(Nc, np.float32), virial_ref=np.zeros(6 * Nc, np.float32),
                   force_ref=np.zeros(3 * N, np.float32))
        lib().oracle_arrays(self._h, *(_p(out[k]) for k in
                                       ("Na", "Na_sum", "type", "r", "h", "pe_ref", "virial_ref", "force_ref")))
        return out

    def neighbors(self):
        NN = np.zeros(self.N, np.int32)
        nl = np.zeros(self.num_bonds, np.int32)
        lib().oracle_neighbors(self._h, _p(NN), _p(nl))
        return NN, nl

    def set_nn2b(self, r1: float = 7.0, r2: float = 8.0, consistent: bool = False):
        lib().oracle_set_nn2b(self._h, r1, r2, int(consistent))

    def set_ri_self(self, on: bool) -> None:
        """RI: subtract the damped-Coulomb self energy (develop/hfo2/find_E.m:10-13)."""
        lib().oracle_set_ri_self(self._h, int(on))

    def decode(self, x01) -> np.ndarray:
        x = np.ascontiguousarray(x01, np.float32)
        p = np.zeros(self.num_vars, np.float64)
        lib().oracle_decode(self._h, _p(x), _p(p))
        return p

    def find_force(self, params):
        p = np.ascontiguousarray(params, np.float64)
        F = np.zeros(3 * self.N)
        W = np.zeros(6 * self.N)
        pe = np.zeros(self.N)
        lib().oracle_find_force(self._h, _p(p), _p(F), _p(W), _p(pe))
        return F, W, pe

    def config_sums(self, W, pe):
        E = np.zeros(self.Nc)
        Wc = np.zeros(6 * self.Nc)
        lib().oracle_config_sums(self._h, _p(np.ascontiguousarray(W)), _p(np.ascontiguousarray(pe)), _p(E), _p(Wc))
        return E, Wc

    def fitness(self, pop01, with_components: bool = False):
        pop = np.ascontiguousarray(pop01, np.float32)
        P = pop.shape[0]
        fit = np.zeros(P)
        comps = np.zeros((P, 3))
        lib().oracle_fitness(self._h, P, _p(pop), _p(fit), _p(comps))
        return (fit, comps) if with_components else fit


def mic_batch(mode: int, h: np.ndarray, xyz: np.ndarray) -> np.ndarray:
    """FP32 minimum-image displacement and squared distance (mic.cuh:20-32, neighbor.cu:59)."""
    n = len(xyz) // 3
    h = np.ascontiguousarray(h, np.float32)
    xyz = np.ascontiguousarray(xyz, np.float32)
    out = np.zeros(4 * n, np.float32)
    lib().oracle_mic_batch(mode, n, _p(h), _p(xyz), _p(out))
    return out


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def ga_run(num_vars, pmin, pmax, population_size, parent_number, mutation_rate, maximum_generation,
           generations, seed, fitness_fn):
    """Reference GA (ga.cu:27-212) driven by ``fitness_fn(pop[P,d] float32) -> float32[P]``.
    Returns (ga.out text, final population)."""
    L = lib()
    d = num_vars

    def cb(P, pop_ptr, fit_ptr, user):
        pop = np.ctypeslib.as_array(pop_ptr, shape=(P * d,)).reshape(P, d).copy()
        f = np.asarray(fitness_fn(pop), np.float32)
        out = np.ctypeslib.as_array(fit_ptr, shape=(P,))
        out[:] = f

    c_cb = FITNESS_CB(cb)
    L.oracle_ga_run.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int,
                                C.c_uint, FITNESS_CB, C.c_void_p, C.c_char_p, C.c_int, C.c_void_p]
    mn = np.ascontiguousarray(pmin, np.float32)
    mx = np.ascontiguousarray(pmax, np.float32)
    n_out = 1 << 16
    while True:
        buf = C.create_string_buffer(n_out)
        final = np.zeros(population_size * d, np.float32)
        rc = L.oracle_ga_run(d, _p(mn), _p(mx), population_size, parent_number, mutation_rate, maximum_generation,
                             generations, seed, c_cb, None, buf, n_out, _p(final))
        if rc >= 0:
            return buf.value.decode(), final.reshape(population_size, d)
        n_out = -rc + 16
