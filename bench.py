#!/usr/bin/env python
"""Benchmark: fitness evaluations per second (individual x atoms) of one GA generation.

A step is one generation's fitness evaluation of the whole population over the
whole training set (GPUGA's Fitness::compute, fitness.cu:316-333).  The default
workload is the batched minimal-Tersoff Si set: 500 periodic diamond
configurations of 8/64/216/512 atoms (~1e5 atoms), population 1000, seeded
synthetic data (no public dataset exists for this path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours:       value = units / device time with populations resident in HBM
            (gpuga_fitness_device); e2e = the same through gpuga_fitness with
            host buffers (H2D population + D2H fitness inside the timed region).
reference:  the reference's own implementation of this path, its CUDA build
            (src/*.cu compiled unmodified into oracle/_ref/ref_probe), timing
            Fitness::compute on the same workload and GPU.
Multi-GPU (torchrun): every rank evaluates its own population of the same size
(individuals are independent: weak scaling, no data-path collective); time is
the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fitness evals/s (indiv x atoms)"
UNIT = "indiv*atoms/s"
FLUSH_BYTES = 256 << 20  # > 126 MB L2


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", type=int, default=2, choices=[1, 2, 3, 4])
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU-baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-individuals", type=int, default=400,
                    help="individuals scored on the plain FP64 path (speed-up denominator and error sample)")
    ap.add_argument("--configs", type=int, default=None, help="override the workload's configuration count")
    ap.add_argument("--population", type=int, default=None, help="override the workload's population size")
    ap.add_argument("--neurons", type=int, default=None,
                    help="NN2B hidden width of workload 4 (default 16; the reference arm needs <= 10)")
    ap.add_argument("--serving", action="store_true", help="serving benchmark (workload 5) instead")
    ap.add_argument("--serving-jobs", type=int, default=32)
    ap.add_argument("--serving-generations", type=int, default=20)
    ap.add_argument("--serving-seconds", type=float, default=4.0,
                    help="bounded serving block: seconds every job keeps running after the last arrival")
    ap.add_argument("--no-serving", action="store_true", help="skip the bounded serving block")
    ap.add_argument("--tiles", type=int, default=0, choices=range(6),
                    help="Tersoff force-item tiles: 0 autotune (default), 1-5 one tile for every configuration")
    ap.add_argument("--fitness-fold", type=int, default=0, choices=range(3),
                    help="fitness fold: 0 (default) or 2 in its own launch, 1 in the work items")
    ap.add_argument("--ga-generations", type=int, default=20,
                    help="generations of the full GA loop timed on the host and on the device loop (0 = skip)")
    return ap.parse_args()


# ----------------------------------------------------------------------------- plumbing
class Dist:
    """One process per GPU (torchrun environment): the barrier and the max-over-ranks timer.
    backend: "nccl" on GPUs (the default when CUDA is available), "gloo" for the CPU tests."""

    def __init__(self, backend: str | None = None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.device = "cpu"
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
            timeout = datetime.timedelta(seconds=300)
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
                self.device = f"cuda:{self.local_rank}"
                dist.init_process_group("nccl", timeout=timeout, device_id=torch.device("cuda", self.local_rank))
            else:
                dist.init_process_group(backend, timeout=timeout)
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


TILE_NAMES = {1: "fixed rule", 2: "half G", 3: "quarter G", 4: "32 per item, global scratch", 5: "unstaged"}


def tile_summary(e, data, P) -> dict | None:
    """The autotuner's force-item tile per force-configuration size (Tersoff sets)."""
    if int(data["potential_type"]) not in (1, 2):
        return None
    codes, tune_ms = e.plan_tiles(P)
    Na, Ncf = np.asarray(data["Na"]), int(data["Nc_force"])
    by_size = {}
    for c in range(Ncf):
        by_size.setdefault(int(Na[c]), TILE_NAMES.get(int(codes[c]), str(int(codes[c]))))
    return {"autotuned": True, "tune_ms": tune_ms, "force_tile_by_atoms": dict(sorted(by_size.items()))}


def whole_job_rate(dist: Dist, units_per_rank_step: float, step_ms) -> tuple:
    """Whole-job throughput of K timed steps: every rank processed units_per_rank_step per step
    (weak scaling), the job took the slowest rank's total device time.  Returns (units/s,
    ms per step of the slowest rank)."""
    total_ms = dist.max(float(sum(step_ms)))
    return dist.world * units_per_rank_step * len(step_ms) / (total_ms / 1e3), total_ms / len(step_ms)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(prefix="gpuga_clocks_", suffix=".csv")
        os.close(fd)
        phys = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[self.device:self.device + 1]
        idx = phys[0] if phys and phys[0] else str(self.device)
        self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                      "-lms", "200", "-i", idx], stdout=open(self.path, "w"),
                                     stderr=subprocess.DEVNULL)

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def _ncu_counts(tag: str):
    """Lines `<tag>: key=value ...` of profiles/ncu_counts.txt (figures from ncu captures)."""
    try:
        lines = open(os.path.join(ROOT, "profiles", "ncu_counts.txt")).read().splitlines()
    except OSError:
        return []
    return [dict(tok.split("=", 1) for tok in ln.split()[1:]) for ln in lines if ln.startswith(tag + ":")]


def ncu_traffic(kernel: str, workload: int, units: float):
    """DRAM bytes (read + write) of one launch of `kernel` from an ncu capture of the same launch
    shape, or None when that shape was not captured."""
    for kv in _ncu_counts("traffic"):
        if int(kv["workload"]) == workload and kv["kernel"] == kernel and float(kv["units"]) == units:
            return float(kv["bytes"])
    return None


def ncu_inst_per_unit(kernel: str, workload: int):
    """Warp instructions per (individual, atom) of `kernel` from an ncu capture (the work-item shapes,
    hence the count per unit, depend on the configurations only)."""
    for kv in _ncu_counts("inst"):
        if int(kv["workload"]) == workload and kv["kernel"] == kernel:
            return float(kv["warp_inst_per_unit"])
    return None


# ----------------------------------------------------------------------------- workload
def oracle_evaluator():
    from oracle import oracle

    def evaluate(data, params):
        d = tempfile.mkdtemp(prefix="gpuga_ref_t_")
        from gpuga_b200 import synth
        synth.write_dir(data, d)
        s = oracle.OracleSet(d)
        if int(data["potential_type"]) == 3:
            s.set_nn2b(data.get("nn2b_r1", 7.0), data.get("nn2b_r2", 8.0), False)
        out = s.find_force(params)
        s.close()
        shutil.rmtree(d, ignore_errors=True)
        return out
    return evaluate


TILES = 0  # force-item tiles of the batched Tersoff path (0: autotuned per configuration size)
FOLD = 0   # where the fitness is folded (0/2: its own launch, 1: in the work items)


def engine_opts(data, device):
    kw = dict(device=device)
    if TILES:
        kw.update(tiles=TILES)
    if FOLD:
        kw.update(fitness_fold=FOLD)
    if int(data["potential_type"]) == 3:
        kw.update(nn2b_r1=float(data["nn2b_r1"]), nn2b_r2=float(data["nn2b_r2"]))
    return kw


def build_workload(workload: int, device: int, Nc=None, P=None, neurons=None):
    """Synthetic set with teacher targets evaluated by the engine's own FP64 path."""
    from gpuga_b200 import Fitness, synth
    data = synth.make(workload, Nc=Nc, neurons=neurons)
    if P:
        data["ga"] = dict(data["ga"], population_size=P, parent_number=P // 2)
    with Fitness(arrays=data, **engine_opts(data, device)) as e0:
        def evaluate(_data, params):
            return e0.find_force64(params)
        data = synth.fill_targets(data, evaluate)
    return data, Fitness(arrays=data, **engine_opts(data, device))


# ----------------------------------------------------------------------------- our arm
def run_ours(args, dist: Dist):
    import torch

    from gpuga_b200 import PATH_PLAIN64, _lib, synth
    dev = dist.local_rank
    torch.cuda.set_device(dev)
    L = _lib.load()
    data, e = build_workload(args.workload, dev, args.configs, args.population, args.neurons)
    P = int(data["ga"]["population_size"])
    d = e.number_of_variables
    Natoms = e.N
    nsteps, nwarm = args.steps, max(args.warmup, 3)
    pops_h = [synth.population(data, P, seed=1000 * dist.rank + k) for k in range(nsteps + nwarm)]
    pops = torch.from_numpy(np.stack(pops_h)).to(f"cuda:{dev}")
    fit = torch.empty(P, dtype=torch.float64, device=f"cuda:{dev}")
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{dev}")
    stream = torch.cuda.current_stream()
    h = e.handle

    def dev_step(k):
        _lib.check(L.gpuga_fitness_device(h, P, C.c_void_p(pops[k].data_ptr()), C.c_void_p(fit.data_ptr()),
                                          C.c_void_p(stream.cuda_stream)))

    n_launch = C.c_int()
    _lib.check(L.gpuga_plan_info(h, P, C.byref(n_launch), None, 0))
    tiles = tile_summary(e, data, P)
    n_kernels = C.c_int()
    _lib.check(L.gpuga_plan_kernels(h, P, C.byref(n_kernels)))
    kernels_per_step = n_kernels.value  # decode + item launches (+ the fitness fold's own launch)

    # ---- value: device-resident inputs, device time per step, L2 flushed between steps
    for k in range(nwarm):
        dev_step(k)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    clocks.start()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nsteps)]
    for k in range(nsteps):
        flush.zero_()
        evs[k][0].record(stream)
        dev_step(nwarm + k)
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    value, ms_per_step = whole_job_rate(dist, P * Natoms, step_ms)
    fit_dev = fit.cpu().numpy().copy()

    # ---- per-launch device times (separate pass of K steps; the launches of a step run one after
    # another on this stream while timing is on, each bracketed by its own events)
    _lib.check(L.gpuga_kernel_timing(h, P, 1))
    for k in range(nsteps):
        flush.zero_()
        dev_step(nwarm + k)
    torch.cuda.synchronize()
    rows = np.zeros((n_launch.value, 8))
    _lib.check(L.gpuga_plan_info(h, P, None, C.c_void_p(rows.ctypes.data), n_launch.value))
    _lib.check(L.gpuga_kernel_timing(h, P, 0))
    peak_fp32 = C.c_double()
    _lib.check(L.gpuga_calibrate_fp32(dev, C.byref(peak_fp32)))
    kinds = {0: "tersoff_batched", 1: "pair_batched<RI>", 2: "pair_batched<NN2B>"}
    launches = []
    for r in rows:
        items = {0: "energy_virial", 1: "force", 2: "force+energy_virial"}[int(r[2])]
        launches.append({"kernel": f"{kinds[int(r[0])]}<{int(r[1])},{items}>",
                         "ctas": int(r[3]), "units": r[4], "flops": r[5], "sfu_calls": r[6], "ms": r[7],
                         "tflops": (r[5] / (r[7] * 1e-3) / 1e12) if r[7] > 0 else None})
    dom = max(launches, key=lambda x: x["ms"])
    gen_flops = sum(x["flops"] for x in launches)
    traffic = ncu_traffic(dom["kernel"], args.workload, dom["units"])
    # instruction-issue bound of the same launch: warp instructions (ncu count per unit) issued per
    # second against 4 schedulers x SMs x SM clock
    ipu = ncu_inst_per_unit(dom["kernel"], args.workload)
    issue = None
    if ipu and dom["ms"] > 0:
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        mhz = (clock_info or {}).get("sm_mhz") or measured_peaks().get("sm_max_mhz") or 1965.0
        achieved = ipu * dom["units"] / (dom["ms"] * 1e-3)
        peak = 4.0 * sms * mhz * 1e6
        issue = {"warp_inst_per_unit": ipu, "achieved_warp_inst_per_s": achieved, "peak_warp_inst_per_s": peak,
                 "frac": achieved / peak, "source": "ncu smsp__inst_executed, profiles/ncu_counts.txt"}
    roofline = {"bound": "fp32", "kernel": dom["kernel"], "achieved": dom["tflops"], "peak": peak_fp32.value,
                "unit": "TFLOP/s", "frac": dom["tflops"] / peak_fp32.value if dom["tflops"] else None,
                "traffic": traffic, "peak_source": "measured: FFMA-chain calibration kernel on this GPU",
                "algorithmic": "FP32 flops of the batched formulation (FMA=2), transcendentals separate",
                "ms_per_launch": dom["ms"], "launches": launches,
                "issue": issue,
                "hbm": ({"achieved_gbs": traffic / (dom["ms"] * 1e-3) / 1e9,
                         "peak_gbs": measured_peaks().get("hbm_gbs"),
                         "frac": traffic / (dom["ms"] * 1e-3) / 1e9 / measured_peaks()["hbm_gbs"]}
                        if traffic and dom["ms"] > 0 and measured_peaks().get("hbm_gbs") else None),
                "generation": {"flops": gen_flops, "ms": ms_per_step,
                               "achieved": gen_flops / (ms_per_step * 1e-3) / 1e12,
                               "frac": gen_flops / (ms_per_step * 1e-3) / 1e12 / peak_fp32.value}}

    # ---- e2e through the public C ABI with host buffers
    e2e_ms = []
    out = np.zeros(P, np.float64)
    for k in range(nwarm):
        e.compute(P, pops_h[k], out)
    dist.barrier()
    for k in range(nsteps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _lib.check(L.gpuga_fitness(h, P, C.c_void_p(pops_h[nwarm + k].ctypes.data), C.c_void_p(out.ctypes.data)))
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_total = dist.max(sum(e2e_ms))
    e2e_value = dist.world * P * Natoms * nsteps / (e2e_total / 1e3)
    e2e_sorted = sorted(e2e_ms)
    p50 = float(np.percentile(e2e_sorted, 50))
    p99 = float(np.percentile(e2e_sorted, 99))

    # ---- whole GA generations (fitness + selection/crossover/mutation): host loop vs device loop
    ga_loop = measure_ga_loops(e, P, args.ga_generations) if args.ga_generations > 0 else None

    # ---- plain FP64 one-individual-per-launch path (denominator of the batched speed-up)
    npl = min(args.plain_individuals, P)
    plain_pop = pops_h[nwarm + nsteps - 1][:npl]
    e.compute(1, plain_pop[:1], path=PATH_PLAIN64)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fit64 = e.compute(npl, plain_pop, path=PATH_PLAIN64)
    t_plain = time.perf_counter() - t0
    plain_value = npl * Natoms / t_plain
    batched = np.asarray(e.compute(P, pops_h[nwarm + nsteps - 1]))[:npl]
    rel = np.abs(batched - fit64) / np.abs(fit64)
    rank_same = bool(np.array_equal(np.argsort(batched, kind="stable"), np.argsort(fit64, kind="stable")))

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": nsteps, "warmup": nwarm,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 pair/3-body math, f64 accumulation", "data": DATA,
        "config": workload_config(args, data, P, e.Nc, Natoms, e.num_bonds, dist.world),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": P * d * 4,
                "d2h_bytes_per_step": P * 8 * 4, "latency_ms": {"p50": p50, "p99": p99}},
        "gpu_launches": kernels_per_step * nsteps,
        "roofline": roofline,
        "plain_fp64": {"value": plain_value, "unit": UNIT, "individuals": npl,
                       "speedup_batched_vs_plain_fp64": value / plain_value,
                       "max_rel_fitness_err_vs_fp64": float(rel.max()),
                       "p99_rel_fitness_err_vs_fp64": float(np.percentile(rel, 99)), "ranking_identical": rank_same},
        "ga_loop": ga_loop,
        "tiles": tiles,
        "clocks": clock_info,
        "measured_peaks": {k: measured_peaks().get(k) for k in ("hbm_gbs", "bf16_tflops", "sm_max_mhz")},
        "fitness_checksum": float(np.sum(fit_dev)),
    }
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(data, args.cpu_seconds)
    e.close()
    if dist.world == 1 and not args.no_serving:
        # bounded serving block (32 jobs of workloads 1-3, Poisson arrivals), a single-GPU feature
        result["serving"] = run_serving(args, steady=True)
    return result


def measure_ga_loops(e, P: int, gens: int) -> dict:
    """Wall time per GA generation (ga.cu:78-92: fitness, sort, output line, crossover, mutation) with the
    host loop (gpuga_ga_step) and the device-resident loop (gpuga_ga_advance); both give identical
    ga.out lines, which is checked here too."""
    from gpuga_b200 import GA
    kw = dict(seed=12345678, population_size=P, parent_number=P // 2, mutation_rate=0.2,
              maximum_generation=gens + 3)
    host = GA(e, **kw)
    for _ in range(3):
        host.step()
    t0 = time.perf_counter()
    host_lines = "".join(host.step() for _ in range(gens))
    t_host = time.perf_counter() - t0
    dev = GA(e, **kw)
    dev.set_device_loop(True, 32)
    dev.advance(3)
    t0 = time.perf_counter()
    dev_lines = dev.advance(gens)
    t_dev = time.perf_counter() - t0
    host.close()
    dev.close()
    return {"generations": gens, "host_loop_ms_per_gen": t_host * 1e3 / gens,
            "device_loop_ms_per_gen": t_dev * 1e3 / gens, "identical_ga_out": host_lines == dev_lines}


def cpu_baseline(data, budget_s: float) -> dict:
    """FP64 OpenMP oracle on the host cores over a bounded sample of the same population."""
    from gpuga_b200 import synth
    from oracle import oracle
    oracle.build()
    d = synth.write_dir(data, tempfile.mkdtemp(prefix="gpuga_cpu_"))
    s = oracle.OracleSet(d)
    pop = synth.population(data, 4096, seed=99)
    t0 = time.perf_counter()
    s.fitness(pop[:1])
    t1 = time.perf_counter() - t0
    n = int(max(1, min(len(pop), budget_s / max(t1, 1e-3))))
    t0 = time.perf_counter()
    s.fitness(pop[:n])
    dt = time.perf_counter() - t0
    s.close()
    shutil.rmtree(d, ignore_errors=True)
    return {"value": n * int(data["Na"].sum()) / dt, "unit": UNIT,
            "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{n} individuals x full training set ({int(data['Na'].sum())} atoms), FP64 OpenMP oracle, "
                      f"{dt:.1f} s"}


# ----------------------------------------------------------------------------- reference arm
DATA = "synthetic (seeded generator, teacher targets)"


def workload_config(args, data, P, Nc, N, bonds, world) -> dict:
    """The `config` object of both arms (same keys and values for the same workload)."""
    name = (f"batched minimal-Tersoff Si: {Nc} diamond configs of 8/64/216/512 atoms" if args.workload == 2
            else data["name"])
    return {"workload": name, "population": P, "configs": Nc, "atoms": N, "bonds": bonds,
            "units_per_step": P * N, "l2": "flushed between steps (256 MiB write, outside the step timing)",
            "parallelism": f"replicas{world} (population per GPU, weak)"}


def run_reference(args, dist: Dist):
    probe = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
    if dist.rank != 0:
        return None
    if not os.path.exists(probe):
        return {"impl": "reference", "unavailable": "oracle/_ref/ref_probe was not built (needs the reference sources)"}
    from gpuga_b200 import synth
    data = synth.make(args.workload, Nc=args.configs, neurons=args.neurons)
    if args.population:
        data["ga"] = dict(data["ga"], population_size=args.population)
    if args.workload == 4 and int(data["num_neurons"]) > 10:
        return {"impl": "reference", "unavailable": "the reference NN2B holds at most 10 neurons (nn2b.cuh:27-33); "
                                                    "run with --neurons 10"}
    data = synth.fill_targets(data, oracle_evaluator())
    d = synth.write_dir(data, tempfile.mkdtemp(prefix="gpuga_ref_"))
    P = int(data["ga"]["population_size"])
    N = int(data["Na"].sum())
    from oracle import oracle
    bonds = oracle.OracleSet(d).num_bonds  # the same neighbor rule as the engine (bit-exact lists)
    r = subprocess.run([probe, "time", d, str(P), str(args.steps), str(max(args.warmup, 3)), "12345678"],
                       capture_output=True, text=True, timeout=3000)
    shutil.rmtree(d, ignore_errors=True)
    # the reference's start-up banner may leave the last line unterminated (neighbor.cu:78-82)
    line = [ln[ln.index("REF_TIME ") + len("REF_TIME "):] for ln in r.stdout.splitlines() if "REF_TIME " in ln]
    if r.returncode != 0 or not line:
        return {"impl": "reference", "unavailable": f"ref_probe failed (rc={r.returncode}): {r.stderr[-300:]}"}
    rt = json.loads(line[0])
    ms = rt["ms"]
    value = P * N * len(ms) / (sum(ms) / 1e3)
    sample = (f"reference CUDA build (GPUGA src/*.cu unmodified, nvcc -O3 --use_fast_math sm_100a) "
              f"Fitness::compute, P={P}, {N} atoms, {len(ms)} generations on the GPU, wall time per generation")
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": len(ms),
            "warmup": max(args.warmup, 3), "ms_per_step": sum(ms) / len(ms), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (fast-math)", "data": DATA,
            "config": workload_config(args, data, P, len(data["Na"]), N, bonds, 1),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "latency_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99))}}


# ----------------------------------------------------------------------------- serving
def _serving_jobs(args, rng):
    """Job directories of the serving mix: workloads 1-3 with 20..500 configurations, seeded synthetic
    data with teacher targets; plus the plain FP64 one-individual-per-launch rate of each potential."""
    from gpuga_b200 import PATH_PLAIN64, Fitness, synth
    jobs, plain_rate = [], {}
    tmp = tempfile.mkdtemp(prefix="gpuga_serving_")
    for k in range(args.serving_jobs):
        cfg = rng.choice([1, 2, 3])
        Nc = rng.randint(20, 500) if cfg != 1 else 20
        data = synth.make(cfg, seed=100 + k, Nc=Nc)
        with Fitness(arrays=data, **engine_opts(data, 0)) as e0:
            data = synth.fill_targets(data, lambda _d, p, e0=e0: e0.find_force64(p))
            if cfg not in plain_rate:  # plain FP64 one-individual-per-launch rate of this potential
                pop = synth.population(data, 4, seed=1)
                e0.compute(1, pop[:1], path=PATH_PLAIN64)
                t0 = time.perf_counter()
                e0.compute(4, pop, path=PATH_PLAIN64)
                plain_rate[cfg] = 4 * e0.N / (time.perf_counter() - t0)
        d = synth.write_dir(data, os.path.join(tmp, f"job{k}"))
        jobs.append((d, cfg, int(data["ga"]["population_size"]), int(data["Na"].sum())))
    return jobs, plain_rate, tmp


def run_serving(args, steady: bool = False) -> dict:
    """Continuous batching: 32 fitting jobs drawn from workloads 1-3 (20..500 configurations each)
    arriving as a Poisson process (2 jobs/s) into a server with a 120 GB budget.  Reports the
    aggregate evals/s, the per-generation latency (device time of a generation of all resident
    jobs, and the wall-clock time per generation each running job saw, stalls included), the time
    from a job's submission to the harvest of its first window, and the one-job-at-a-time
    plain-FP64 estimate for the same work.

    steady=False: every job runs --serving-generations generations.  steady=True (the bounded block
    of the default benchmark): every job runs until --serving-seconds after the last arrival and is
    then cancelled, so that all jobs are resident together for a while."""
    import random

    from gpuga_b200 import Server
    rng = random.Random(5)
    jobs, plain_rate, tmp = _serving_jobs(args, rng)
    gens = 10 ** 6 if steady else args.serving_generations
    with Server(device=0, hbm_budget_bytes=120e9, max_jobs=32) as srv:
        t0 = time.perf_counter()
        ids = []
        for k, (d, cfg, P, N) in enumerate(jobs):
            ids.append(srv.submit(d, seed=1000 + k, generations=gens))
            if k + 1 < len(jobs):
                time.sleep(rng.expovariate(2.0))
        if steady:
            time.sleep(args.serving_seconds)
            for j in ids:
                srv.cancel(j)
        rc = srv.drain(3000)
        wall = time.perf_counter() - t0
        st = srv.stats()
        done = [srv.poll(j)[1] for j in ids]
    shutil.rmtree(tmp, ignore_errors=True)
    units = [P * N * g for (_, _, P, N), g in zip(jobs, done)]
    total_units = float(sum(units))
    serial_plain_s = sum(u / plain_rate[cfg] for u, (_, cfg, _, _) in zip(units, jobs))
    return {"metric": "serving: aggregate fitness evals/s (indiv x atoms), 32 concurrent jobs", "value": st["evals_per_s"],
            "unit": UNIT, "n_gpus": 1, "jobs": len(jobs),
            "generations_per_job": (f"until cancelled {args.serving_seconds:g} s after the last arrival" if steady
                                    else gens),
            "generations_done": {"min": int(min(done)), "max": int(max(done)), "total": int(sum(done))},
            "status": rc if not steady else "cancelled after the steady-state period",
            "latency_ms": {"device_p50": st["p50_gen_ms"], "device_p99": st["p99_gen_ms"],
                           "wall_p50": st["p50_wall_gen_ms"], "wall_p99": st["p99_wall_gen_ms"],
                           "first_window_p50": st["p50_first_window_ms"],
                           "first_window_p99": st["p99_first_window_ms"]},
            "wall_s": wall, "busy_s": st["busy_s"],
            "peak_resident_jobs": st["peak_resident_jobs"], "generation_batches": st["batches"],
            "total_units": total_units, "arrivals": "Poisson, 2 jobs/s",
            "one_at_a_time_plain_fp64_s_estimate": serial_plain_s,
            "speedup_vs_one_at_a_time_plain_fp64": serial_plain_s / max(wall, 1e-9),
            "speedup_busy_vs_one_at_a_time_plain_fp64": serial_plain_s / max(st["busy_s"], 1e-9),
            "data": "synthetic (workloads 1-3, 20-500 configurations, teacher targets)"}


def main():
    global TILES, FOLD
    args = parse_args()
    TILES, FOLD = args.tiles, args.fitness_fold
    if args.serving:
        print(json.dumps(run_serving(args)))
        return 0
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return 0
        res = run_reference(args, _RankZero())
        print(json.dumps(res))
        return 0
    dist = Dist()
    try:
        res = run_ours(args, dist)
        if dist.rank == 0:
            print(json.dumps(res))
    finally:
        dist.close()
    return 0


class _RankZero:
    rank = 0
    world = 1


if __name__ == "__main__":
    sys.exit(main())
