"""Python mirror of GPUGA's host interfaces over the C ABI.

``Fitness`` follows src/fitness.cuh:30-83 (constructor from an input
directory, ``compute(P, population, fitness)``, ``predict(dir, elite)``,
``number_of_variables``, ``parameters_min``/``parameters_max``) and ``GA``
follows src/ga.cuh:20-58.  Arrays are numpy; the work happens in
libgpuga_b200.so on the GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import PATH_BATCHED, PATH_PLAIN32, PATH_PLAIN64, check


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def options(device: int = 0, path: int = PATH_BATCHED, use_graph: bool = True, nn2b_consistent: bool = False,
            nn2b_r1: float = 7.0, nn2b_r2: float = 8.0, verbose: bool = False, neighbor_cells: int = 0,
            ri_self_energy: bool = False, tiles: int = 0, fitness_fold: int = 0) -> _lib.Options:
    o = _lib.Options()
    _lib.load().gpuga_default_options(C.byref(o))
    o.device, o.path, o.use_graph = device, path, int(use_graph)
    o.nn2b_consistent, o.nn2b_r1, o.nn2b_r2, o.verbose = int(nn2b_consistent), nn2b_r1, nn2b_r2, int(verbose)
    o.neighbor_cells = neighbor_cells
    o.ri_self_energy = int(ri_self_energy)
    o.tiles = tiles
    o.fitness_fold = fitness_fold
    return o


class Fitness:
    """Training set + potential resident on one GPU (Fitness::Fitness, fitness.cu:30-38)."""

    def __init__(self, input_dir: str | None = None, *, arrays: dict | None = None, **opts):
        L = _lib.load()
        self._h = C.c_void_p()
        o = options(**opts)
        if input_dir is not None:
            check(L.gpuga_engine_create(input_dir.encode(), C.byref(o), C.byref(self._h)))
        else:
            a = arrays
            Na = np.ascontiguousarray(a["Na"], np.int32)
            keep = dict(
                weights=np.asarray([a["w_force"], a["w_energy"], a["w_stress"]], np.float32),
                pmin=np.ascontiguousarray(a["pmin"], np.float32), pmax=np.ascontiguousarray(a["pmax"], np.float32),
                type=np.ascontiguousarray(a["type"], np.int32), r=np.ascontiguousarray(a["r"], np.float32),
                box9=np.ascontiguousarray(a["box9"], np.float32),
                pe_ref=np.ascontiguousarray(a["pe_ref"], np.float32),
                virial_ref=np.ascontiguousarray(a["virial_ref"], np.float32),
                force_ref=np.ascontiguousarray(a["force_ref"], np.float32))
            check(L.gpuga_engine_create_from_arrays(
                int(a["potential_type"]), int(a.get("num_neurons", 0)), float(a["cutoff"]), _p(keep["weights"]),
                _p(keep["pmin"]), _p(keep["pmax"]), int(len(Na)), int(a["Nc_force"]), _p(Na), _p(keep["type"]),
                _p(keep["r"]), _p(keep["box9"]), _p(keep["pe_ref"]), _p(keep["virial_ref"]), _p(keep["force_ref"]),
                C.byref(o), C.byref(self._h)))
        info = np.zeros(10, np.int32)
        check(L.gpuga_engine_info(self._h, _p(info)))
        (self.potential_type, self.number_of_variables, self.num_neurons, self.Nc, self.Nc_force, self.N,
         self.N_force, self.max_Na, self.num_bonds, self.max_neighbors) = (int(v) for v in info)
        self.parameters_min = np.zeros(self.number_of_variables, np.float32)
        self.parameters_max = np.zeros(self.number_of_variables, np.float32)
        check(L.gpuga_engine_bounds(self._h, _p(self.parameters_min), _p(self.parameters_max)))
        norms = np.zeros(3)
        check(L.gpuga_engine_norms(self._h, _p(norms)))
        self.norm_force, self.norm_energy, self.norm_virial = (float(v) for v in norms)

    # -------------------------------------------------------------- lifetime
    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.load().gpuga_engine_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # -------------------------------------------------------------- hot path
    def compute(self, population_size: int, population: np.ndarray, fitness: np.ndarray | None = None,
                path: int = PATH_BATCHED, components: bool = False):
        """Fitness::compute (fitness.cu:316-333): population [P, d] in [0, 1] -> fitness [P] (FP64)."""
        pop = np.ascontiguousarray(population, np.float32).reshape(population_size, self.number_of_variables)
        out = np.zeros(population_size, np.float64)
        comps = np.zeros((population_size, 3), np.float64)
        check(_lib.load().gpuga_fitness_ex(self._h, path, population_size, _p(pop), _p(out), _p(comps)))
        if fitness is not None:
            fitness[:] = out
        return (out, comps) if components else out

    def config_results(self, population_size: int):
        """Per (individual, configuration) results of the last batched evaluation."""
        P, Nc = population_size, self.Nc
        E = np.zeros((P, Nc))
        W = np.zeros((P, Nc, 6))
        F2 = np.zeros((P, Nc))
        check(_lib.load().gpuga_last_config_results(self._h, P, _p(E), _p(W), _p(F2)))
        return E, W, F2

    def batched_forces(self, population: np.ndarray) -> np.ndarray:
        pop = np.ascontiguousarray(population, np.float32)
        P = pop.shape[0]
        out = np.zeros((P, 3, self.N_force), np.float32)
        check(_lib.load().gpuga_batched_forces(self._h, P, _p(pop), _p(out)))
        return out

    def find_force64(self, params):
        p = np.ascontiguousarray(params, np.float64)
        F, W, pe = np.zeros(3 * self.N), np.zeros(6 * self.N), np.zeros(self.N)
        check(_lib.load().gpuga_find_force64(self._h, _p(p), _p(F), _p(W), _p(pe)))
        return F, W, pe

    def find_force32(self, params):
        p = np.ascontiguousarray(params, np.float32)
        F = np.zeros(3 * self.N, np.float32)
        W = np.zeros(6 * self.N, np.float32)
        pe = np.zeros(self.N, np.float32)
        check(_lib.load().gpuga_find_force32(self._h, _p(p), _p(F), _p(W), _p(pe)))
        return F, W, pe

    def decode(self, x01) -> np.ndarray:
        x = np.ascontiguousarray(x01, np.float32)
        out = np.zeros(self.number_of_variables, np.float32)
        check(_lib.load().gpuga_decode(self._h, _p(x), _p(out)))
        return out

    def predict(self, input_dir: str, elite) -> None:
        """Fitness::predict (fitness.cu:335-390): writes force.out, energy.out, virial.out."""
        e = np.ascontiguousarray(elite, np.float32)
        check(_lib.load().gpuga_predict(self._h, input_dir.encode(), _p(e)))

    def plan_tiles(self, population_size: int):
        """(per-configuration force-item tile codes, autotuner host time in ms) of the plan for P."""
        t = np.zeros(self.Nc, np.int32)
        ms = C.c_double()
        check(_lib.load().gpuga_plan_tiles(self._h, population_size, _p(t), self.Nc, C.byref(ms)))
        return t, ms.value

    def neighbors(self):
        """(NN[N], nbr[num_bonds]) in CSR form, ascending neighbor indices."""
        NN = np.zeros(self.N, np.int32)
        nbr = np.zeros(max(self.num_bonds, 1), np.int32)
        check(_lib.load().gpuga_engine_neighbors_csr(self._h, _p(NN), _p(nbr)))
        return NN, nbr[: self.num_bonds]

    def neighbors_reference_layout(self):
        NN = np.zeros(self.N, np.int32)
        NL = np.zeros(self.N * self.max_Na, np.int32)
        check(_lib.load().gpuga_engine_neighbors(self._h, _p(NN), _p(NL)))
        return NN, NL


class Server:
    """Continuous-batching server: many fitting jobs, one GPU, shared launches (gpuga_server_*)."""

    QUEUED, RUNNING, DONE, FAILED, CANCELLED = range(5)

    def __init__(self, device: int = 0, hbm_budget_bytes: float = 120e9, max_jobs: int = 32):
        self._h = C.c_void_p()
        check(_lib.load().gpuga_server_create(device, float(hbm_budget_bytes), max_jobs, C.byref(self._h)))

    def submit(self, input_dir: str, seed: int = 12345678, generations: int = 0) -> int:
        jid = C.c_int()
        check(_lib.load().gpuga_server_submit(self._h, input_dir.encode(), seed, generations, C.byref(jid)))
        return jid.value

    def submit_engine(self, fitness: "Fitness", population_size: int, parent_number: int, mutation_rate: float,
                      generations: int, seed: int = 12345678) -> int:
        jid = C.c_int()
        check(_lib.load().gpuga_server_submit_engine(self._h, fitness.handle, population_size, parent_number,
                                                     mutation_rate, generations, seed, C.byref(jid)))
        return jid.value

    def poll(self, job_id: int):
        """(status, generations done, generations total, state)."""
        prog = np.zeros(3, np.int32)
        st = _lib.load().gpuga_server_poll(self._h, job_id, _p(prog))
        return st, int(prog[0]), int(prog[1]), int(prog[2])

    def result(self, job_id: int, generations: int, num_vars: int):
        best = np.zeros(generations, np.float32)
        elite = np.zeros(num_vars, np.float32)
        check(_lib.load().gpuga_server_result(self._h, job_id, _p(best), _p(elite)))
        return best, elite

    def cancel(self, job_id: int) -> None:
        check(_lib.load().gpuga_server_cancel(self._h, job_id))

    def hold(self, on: bool = True) -> None:
        """While held no new scheduling window starts; jobs are still admitted and set up."""
        check(_lib.load().gpuga_server_hold(self._h, int(on)))

    def drain(self, timeout_s: float = 0.0) -> int:
        return _lib.load().gpuga_server_drain(self._h, float(timeout_s))

    def stats(self) -> dict:
        keys = ("batches", "jobs_finished", "p50_gen_ms", "p99_gen_ms", "evals_per_s", "device_bytes",
                "peak_resident_jobs", "total_evals", "p50_wall_gen_ms", "p99_wall_gen_ms", "busy_s",
                "p50_first_window_ms", "p99_first_window_ms")
        s = np.zeros(len(keys))
        check(_lib.load().gpuga_server_stats(self._h, _p(s), len(keys)))
        return dict(zip(keys, (float(v) for v in s)))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.load().gpuga_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class GA:
    """GA of src/ga.cu driven by a Fitness (GA::GA + GA::compute one generation at a time)."""

    def __init__(self, fitness: Fitness | None = None, input_dir: str | None = None, seed: int = 12345678, *,
                 population_size: int = 200, parent_number: int = 100, mutation_rate: float = 0.2,
                 maximum_generation: int = 1000, host_callback=None, num_vars: int | None = None,
                 pmin=None, pmax=None):
        L = _lib.load()
        self._h = C.c_void_p()
        self._keep = None
        if host_callback is not None:
            d = num_vars

            def cb(P, pop_ptr, fit_ptr, user):
                pop = np.ctypeslib.as_array(pop_ptr, shape=(P * d,)).reshape(P, d).copy()
                np.ctypeslib.as_array(fit_ptr, shape=(P,))[:] = np.asarray(host_callback(pop), np.float32)

            c_cb = _lib.FITNESS_CB(cb)
            mn = np.ascontiguousarray(pmin, np.float32)
            mx = np.ascontiguousarray(pmax, np.float32)
            self._keep = (c_cb, mn, mx)
            check(L.gpuga_ga_create_host(d, _p(mn), _p(mx), population_size, parent_number, mutation_rate,
                                         maximum_generation, seed, c_cb, None, C.byref(self._h)))
            self.num_vars = d
        elif input_dir is not None:
            check(L.gpuga_ga_create(fitness.handle, input_dir.encode(), seed, C.byref(self._h)))
            self.num_vars = fitness.number_of_variables
        else:
            check(L.gpuga_ga_create_params(fitness.handle, population_size, parent_number, mutation_rate,
                                           maximum_generation, seed, C.byref(self._h)))
            self.num_vars = fitness.number_of_variables
        self.fitness_obj = fitness

    def step(self) -> str:
        buf = C.create_string_buffer(64 + 20 * self.num_vars)
        check(_lib.load().gpuga_ga_step(self._h, buf, len(buf)))
        return buf.value.decode()

    def run(self, input_dir: str) -> None:
        check(_lib.load().gpuga_ga_run(self._h, input_dir.encode()))

    def advance(self, generations: int) -> str:
        """`generations` generations on the device-resident loop; returns their ga.out lines."""
        buf = C.create_string_buffer(generations * (64 + 20 * self.num_vars) + 1)
        check(_lib.load().gpuga_ga_advance(self._h, generations, buf, len(buf)))
        return buf.value.decode()

    def set_device_loop(self, enable: bool, window: int = 0) -> None:
        check(_lib.load().gpuga_ga_set_device_loop(self._h, int(enable), window))

    def state(self, population_size: int):
        gen = C.c_int()
        pop = np.zeros((population_size, self.num_vars), np.float32)
        fit = np.zeros(population_size, np.float32)
        check(_lib.load().gpuga_ga_state(self._h, C.byref(gen), _p(pop), _p(fit)))
        return gen.value, pop, fit

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.load().gpuga_ga_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
