"""Benchmark of the B200 SPM step (KAPSEL smoothed-profile method).

Workload (the headline configuration): 256^3 periodic grid, 1000 colloids
a=5, xi=2, seeded non-overlapping positions, random unit quaternions,
Gaussian velocities sd=1e-3, LJ repulsion (sigma=2a, eps=1, cutoff
2^(1/6) sigma), dt=0.05, no thermal noise.  A step is one
Time_evolution_hydro (sp_3d_ns.cxx:41-194) on device-resident state.

  value      FP32-mixed steps/s, whole job (N replicas, one per GPU)
  e2e        same metric through the C ABI with host particle records:
             every step uploads the Np particle records from pinned host
             memory, runs the step and reads them back
  fp64       FP64 GPU path steps/s on the same workload
  accuracy   relative L2 errors of u, phi, x, v, omega, FP32-mixed vs FP64,
             every 50 of 500 steps from the same initial state
  roofline   dominant kernel achieved GB/s vs measured peak, and every
             kernel family of both precisions (roofline.kernels)
  cpu_baseline  the reference program built from its sources (oracle/_ref),
             OpenMP, all host cores, on a bounded sample of the same workload

`--impl reference` runs that reference program alone on rank 0 (other ranks
exit) for the same metric on a bounded number of steps.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(npx=8, npy=8, npz=8, n_particles=1000, a=5.0, a_xi=2.0, dt=0.05)
METRIC = "SPM steps/s 256³ 1000 colloids, FP32-mixed vs FP64 GPU @≤1e-5; p99 serve lat"
UNIT = "steps/s"


def workload_config():
    from kapsel3_b200.udf import SPMConfig
    return SPMConfig(**WORKLOAD)


def workload_particles(cfg):
    from kapsel3_b200.udf import make_particles
    return make_particles(cfg, seed=2024, v_sd=1e-3, random_orientation=True)


def config_block():
    return {"workload": "SPM step, 256^3 periodic grid, 1000 colloids a=5 xi=2, LJ 12:6 WCA, dt=0.05, no noise",
            "grid": [256, 256, 256], "colloids": 1000, "radius": 5.0, "xi": 2.0, "dt": 0.05,
            "l2": "inputs larger than L2 (one field is 135 MB FP64 / 67 MB FP32; 11 fields resident)",
            "parallelism": "replicas (one independent run per GPU, no collective)"}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """Samples SM clock and throttle reasons through NVML on a thread while
    the timed region runs.  start() returns once the first sample is taken
    and stop() takes a last one, so even a short timed region is covered."""

    def __init__(self):
        self.samples = []
        self._stop = threading.Event()
        self._ready = threading.Event()
        self._t = None
        self._h = None
        self._nvml = None
        try:
            import pynvml
            pynvml.nvmlInit()
            idx = int(os.environ.get("LOCAL_RANK", "0"))
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            self._h = pynvml.nvmlDeviceGetHandleByIndex(idx if vis is None else 0 if "," not in vis else idx)
            self._smax = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self._nvml = pynvml
        except Exception as e:  # no NVML: report that
            self.error = str(e)

    def _sample(self):
        n = self._nvml
        sm = n.nvmlDeviceGetClockInfo(self._h, n.NVML_CLOCK_SM)
        reasons = n.nvmlDeviceGetCurrentClocksEventReasons(self._h)
        self.samples.append((sm, self._smax, reasons))

    def start(self):
        if self._nvml is None:
            return

        def run():
            try:
                self._sample()
                self._ready.set()
                while not self._stop.is_set():
                    time.sleep(0.02)
                    self._sample()
            except Exception:
                self._ready.set()
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()
        self._ready.wait(timeout=5)

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=2)
        if self._nvml is not None:
            try:
                self._sample()
            except Exception:
                pass
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        names = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
                 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
                 0x100: "display_clock_setting"}
        mask = 0
        for s in self.samples:
            mask |= int(s[2])
        return {"sm_mhz": float(np.median([s[0] for s in self.samples])), "sm_max_mhz": float(self.samples[0][1]),
                "reasons": [v for k, v in names.items() if mask & k], "samples": len(self.samples)}


# --------------------------------------------------------------- reference
def reference_available():
    from oracle import ref_runner
    return ref_runner.available(omp=True)


def time_reference(cfg, parts, nsteps, threads):
    """Runs the reference program (oracle/_ref, OpenMP build) for nsteps+1
    steps and returns steps/s over steps 1..nsteps (step 0 excluded: it
    includes first-touch of every array)."""
    from kapsel3_b200.udf import write_udf_keys
    from oracle import ref_runner
    import dataclasses
    c = dataclasses.replace(cfg, gts=1, num_snap=nsteps)
    d = tempfile.mkdtemp(prefix="kapsel_bench_ref_")
    keys, stamps = os.path.join(d, "run.keys"), os.path.join(d, "stamps.txt")
    write_udf_keys(keys, c, parts, out_dir=os.path.join(d, "avs"))
    ref_runner.run_reference(keys, dump_path=None, omp=True, threads=threads, step_times_path=stamps,
                             timeout=1800)
    t = np.loadtxt(stamps)
    # stamp i is taken at the start of step i (after i completed steps)
    dts = np.diff(t)[1:]
    return float(1.0 / np.mean(dts)), len(dts)


def resident_program_leg():
    """The reference program itself with its main loop advanced on the GPU
    (oracle/_ref/kapsel_gpu_resident: the unmodified reference objects plus
    kapsel3_b200/shim/kapsel_b200_resident.cxx) against the same program on
    the CPU (kapsel_ref_omp, GCC_OMP flags, all host threads), both end to
    end on the 128^3 / 200-colloid thermostat configuration.  The resident
    run outputs a frame every 50 steps (host copies of zeta, phi and the
    particles at each); steps/s over steps 50..200 from the program's own
    per-frame wall-clock stamps.  None when the programs are not built."""
    from kapsel3_b200.udf import SPMConfig, make_particles, write_udf_keys
    from oracle import ref_runner
    if not (ref_runner.available(gpu_resident=True) and ref_runner.available(omp=True)):
        return None
    threads = os.cpu_count() or 1
    cfg = SPMConfig(npx=7, npy=7, npz=7, n_particles=200, a=5.0, a_xi=2.0, dt=0.05, kbt=1e-4, gts=50, num_snap=4)
    parts = make_particles(cfg, seed=2024, v_sd=1e-3, random_orientation=True)
    d = tempfile.mkdtemp(prefix="kapsel_bench_resident_")
    keys, stamps = os.path.join(d, "run.keys"), os.path.join(d, "stamps.txt")
    write_udf_keys(keys, cfg, parts, out_dir=os.path.join(d, "avs"))
    ref_runner.run_reference(keys, dump_path=None, gpu_resident=True, threads=threads, step_times_path=stamps,
                             timeout=600)
    t = np.loadtxt(stamps)  # one stamp per frame: ts = 0, 50, ..., 200
    resident = float((len(t) - 2) * cfg.gts / (t[-1] - t[1]))
    ref_v, ref_n = time_reference(cfg, parts, 4, threads)
    return {"config": "128^3 grid, 200 colloids a=5 xi=2, kT=1e-4 thermostat, dt=0.05, a frame every 50 steps",
            "resident_program_steps_per_s": resident, "reference_program_steps_per_s": ref_v,
            "ratio": resident / ref_v, "reference_sample": f"{ref_n} steps, OMP_NUM_THREADS={threads}",
            "resident_sample": f"steps 50..{cfg.gts * cfg.num_snap} (frames at every 50th step included)"}


def port_baseline(cfg, parts, nsteps):
    """Fallback when the reference program is not built: the numpy oracle."""
    from oracle.spm_oracle import OracleSPM
    o = OracleSPM(cfg, parts)
    o.step()
    t0 = time.perf_counter()
    for _ in range(nsteps):
        o.step()
    return nsteps / (time.perf_counter() - t0), nsteps


def cpu_baseline(cfg, parts):
    threads = os.cpu_count() or 1
    if reference_available():
        v, n = time_reference(cfg, parts, 3, threads)
        return {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": f"{n} steps of the full 256^3/1000-colloid workload (steps 2..{n + 1} of a fresh run), "
                          f"reference program built from its sources, GCC_OMP flags, OMP_NUM_THREADS={threads}"}
    v, n = port_baseline(cfg, parts, 1)
    return {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{n} step of the full workload with the numpy restatement (reference program not built)"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cfg = workload_config()
    parts = workload_particles(cfg)
    threads = os.cpu_count() or 1
    nsteps = max(1, min(args.steps, 4))
    if reference_available():
        v, n = time_reference(cfg, parts, nsteps + 1, threads)
        kind = "reference"
        sample = (f"{n} steps of the full workload after one warm-up step, reference program built from its own "
                  f"sources (GCC_OMP flags), OMP_NUM_THREADS={threads}")
    else:
        v, n = port_baseline(cfg, parts, min(nsteps, 2))
        kind, threads = "port", 1
        sample = f"{n} steps with the numpy restatement (reference program not built)"
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus, "steps": n,
            "warmup": 1, "ms_per_step": 1000.0 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded initial state)",
            "config": config_block(),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------- GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-stream leg")
    ap.add_argument("--serve-runs", type=int, default=256)
    ap.add_argument("--profile-run", choices=["fp32", "fp64", "electrolyte", "squirmer"], default=None,
                    help="only run warm-up + timed steps of one precision (for ncu captures)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.profile_run:
        return profile_run(args)

    import torch
    import torch.distributed as dist
    from kapsel3_b200 import _native as N
    from kapsel3_b200.spm import SPMRun, pack_particles

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    W, K = max(3, args.warmup), max(1, args.steps)
    cfg = workload_config()
    parts = workload_particles(cfg)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    results = {}
    stream = torch.cuda.current_stream().cuda_stream
    for prec, name in ((N.SPM_PREC_FP32_MIXED, "fp32"), (N.SPM_PREC_FP64, "fp64")):
        run = SPMRun(cfg, precision=prec, stream=stream)
        run.initialize(parts)
        run.step(W)
        run.synchronize()
        run.kernel_launches(reset=True)
        barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler()
        clocks.start()
        ms = run.time_steps(K)
        cl = clocks.stop()
        torch.cuda.synchronize()
        barrier()
        ms = max_over_ranks(ms)
        launches = run.kernel_launches(reset=True)
        results[name] = dict(ms=ms, clocks=cl, launches=launches)
        # e2e through the C ABI: particle records from pinned host memory in,
        # step, records out, every step.
        L = N.lib()
        n = cfg.n_particles
        rec_t = torch.from_numpy(run.particles_record()).pin_memory()
        rec = rec_t.numpy()
        ptr = rec.ctypes.data_as(C.POINTER(C.c_double))
        for _ in range(2):
            N.check(L.spm_set_particles(run.h, ptr), "spm_set_particles")
            N.check(L.spm_step(run.h, 1), "spm_step")
            N.check(L.spm_get_particles(run.h, ptr), "spm_get_particles")
        barrier()
        t0 = time.perf_counter()
        for _ in range(K):
            N.check(L.spm_set_particles(run.h, ptr), "spm_set_particles")
            N.check(L.spm_step(run.h, 1), "spm_step")
            N.check(L.spm_get_particles(run.h, ptr), "spm_get_particles")
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        results[name]["e2e"] = dict(value=world * K / e2e_s, h2d=n * N.SPM_PARTICLE_WORDS * 8,
                                    d2h=n * N.SPM_PARTICLE_WORDS * 8)
        # every kernel family timed inside real steps (CUDA events on the stream each runs on)
        results[name]["kernels"] = profile_kernels(run, K)
        run.close()

    # accuracy: FP32-mixed vs FP64 over the precision configuration's 500 steps (independent of --steps)
    acc = accuracy_check(cfg, parts)
    serving = None if args.no_serve else serving_leg(rank, world, args.serve_runs, barrier, max_over_ranks)

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0
    fp32, fp64 = results["fp32"], results["fp64"]
    value = world * K / (fp32["ms"] / 1000.0)
    peaks = read_peaks()
    tables = {p: kernel_table(results[p]["kernels"], K, peaks["hbm_gbs"]) for p in ("fp32", "fp64")}
    dom = max((r for r in tables["fp32"] if r["bytes_per_launch"] > 0), key=lambda r: r["us_per_step"])
    roof = {"bound": "hbm", "kernel": dom["kernel"], "achieved": dom["achieved_gbs"], "peak": peaks["hbm_gbs"],
            "unit": "GB/s", "frac": dom["frac"], "traffic": read_traffic(dom["kernel"]),
            "traffic_source": TRAFFIC_FILE,
            "peak_source": peaks["source"], "bytes_per_launch": dom["bytes_per_launch"],
            "avg_launch_us": dom["us_per_launch"],
            "note": ("dominant = the FP32-mixed kernel family with the most device time per step; algorithmic "
                     "bytes per launch over its CUDA-event duration inside real steps (kernels[] holds every "
                     "family, both precisions)"),
            "kernels": tables}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": fp32["ms"] / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 fields / f64 particle reductions", "data": "synthetic (seeded initial state)",
        "config": config_block(),
        "fp64": {"value": world * K / (fp64["ms"] / 1000.0), "unit": UNIT, "ms_per_step": fp64["ms"] / K,
                 "clocks": fp64["clocks"],
                 "e2e": {"value": fp64["e2e"]["value"], "unit": UNIT, "h2d_bytes_per_step": fp64["e2e"]["h2d"],
                         "d2h_bytes_per_step": fp64["e2e"]["d2h"]}},
        "fp32_over_fp64": fp64["ms"] / fp32["ms"],
        "accuracy": acc,
        "e2e": {"value": fp32["e2e"]["value"], "unit": UNIT, "h2d_bytes_per_step": fp32["e2e"]["h2d"],
                "d2h_bytes_per_step": fp32["e2e"]["d2h"]},
        "roofline": roof,
        "step_hbm": {"algorithmic_gb_per_step_fp32": step_bytes(cfg, 4) / 1e9,
                     "achieved_gbs": step_bytes(cfg, 4) / (fp32["ms"] / K / 1000.0) / 1e9,
                     "frac_of_peak": step_bytes(cfg, 4) / (fp32["ms"] / K / 1000.0) / 1e9 / peaks["hbm_gbs"]},
        "clocks": fp32["clocks"],
        "gpu_launches": fp32["launches"],
    }
    if serving is not None:
        line["serving"] = serving
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg, parts)
        line["resident_reference_program"] = resident_program_leg()
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def serving_leg(rank, world, n_runs, barrier, max_over_ranks):
    """The serving stream: n_runs requests, exponential inter-arrivals at
    20/s, cubic side uniform over {32, 64, 128}, Np uniform in [1, 300]
    capped per side by packability, a=4, xi=2, 200 FP32-mixed steps each,
    device-memory budget 150 GB.  Each replica (GPU) serves every world-th
    request of the stream through its own native request loop; arrivals are
    real time.  A seeded random sample of 48 of each replica's runs (at
    least 32 of them complete in any run of this workload) keeps its final
    velocity and is re-run alone in FP64 for its error."""
    from kapsel3_b200 import _native as N
    from kapsel3_b200.serve import Server, partition, run_stream, serving_workload
    from kapsel3_b200.spm import SPMRun, unpack_particles

    w = serving_workload(n_runs=n_runs, rate_per_s=20.0, sides=(32, 64, 128), np_max=300, a=4.0, a_xi=2.0,
                         nsteps=200, seed=2024)
    mine = partition(w["requests"], rank, world)
    rng = np.random.default_rng(7 + rank)
    sample = set(int(i) for i in rng.choice(len(mine), size=min(SERVE_FP64_SAMPLE, len(mine)), replace=False))
    barrier()
    with Server(budget_bytes=150 << 30, use_graph=True, pool_capacity=8) as srv:
        res = run_stream(srv, mine, realtime=True, keep_velocity_ids=sample)
    per_side = {}
    for i in sorted(sample):
        r, out = mine[i], res["results"][i]
        if out["state"] != N.SPM_REQ_DONE:
            continue
        with SPMRun(r.cfg, precision=N.SPM_PREC_FP64) as run:
            run.initialize(unpack_particles(r.particles))
            run.step(r.nsteps)
            u64 = run.velocity()
        d = np.linalg.norm(out["velocity"] - u64) / max(np.linalg.norm(u64), 1e-300)
        per_side.setdefault(str(r.cfg.shape[0]), []).append(float(d))
    all_errs = [e for v in per_side.values() for e in v]
    errs = {"sample": "seeded random runs of this replica, re-run alone in FP64", "runs": len(all_errs),
            "max": max(all_errs) if all_errs else None,
            "median": float(np.median(all_errs)) if all_errs else None,
            "meets_1e-5": bool(all_errs) and max(all_errs) <= 1e-5,
            "per_side_max": {k: max(v) for k, v in sorted(per_side.items())},
            "per_side_runs": {k: len(v) for k, v in sorted(per_side.items())}}
    st = res["stats"]
    lat = res["latencies"]
    busy = max_over_ranks(st["busy_s"])
    steps_total = st["run_steps"] * world  # equal shares up to one request
    done = sum(1 for o in res["results"] if o["state"] == N.SPM_REQ_DONE)
    return {
        "runs": n_runs, "completed_rank0": done, "requested_rank0": len(mine),
        "arrivals": "exponential, 20/s, seeded", "sides": [32, 64, 128], "np_cap": w["np_cap"],
        "steps_per_run": 200, "dtype": "f32 fields / f64 particle reductions", "budget_gb": 150,
        "steps_per_s": steps_total / busy if busy > 0 else None,
        "step_latency_ms": {"p50": float(np.percentile(lat, 50)) if len(lat) else None,
                            "p99": max_over_ranks(float(np.percentile(lat, 99))) if len(lat) else None,
                            "max": float(lat.max()) if len(lat) else None},
        "pool_step_device_ms": {"p50": st["pool_step_device_p50_ms"], "p99": st["pool_step_device_p99_ms"]},
        "max_resident_runs": st["max_active"], "graph_captures": st["graph_captures"],
        "worker_phase_max_ms": {k: round(st[k + "_max_ms"], 3)
                                for k in ("pool_create", "admit", "pool_destroy", "launch", "finish")},
        "peak_device_gb": st["peak_bytes"] / 1e9, "wall_s": res["wall_s"],
        "fp64_rel_velocity_error": errs,
        "latency_definition": "host time between consecutive step completions of a run (first: from admission)",
    }


def profile_run(args):
    """Warm-up + timed steps of one precision, nothing else: the command the
    ncu launch lists and captures under profiles/ were taken with."""
    from kapsel3_b200 import _native as N
    from kapsel3_b200.spm import SPMRun
    from kapsel3_b200.udf import EQ_EL, SPMConfig, make_particles
    if args.profile_run in ("electrolyte", "squirmer"):
        # the Electrolyte and squirmer workloads of the profiles/ launch lists (FP64)
        if args.profile_run == "electrolyte":
            cfg = SPMConfig(npx=7, npy=7, npz=7, n_particles=50, a=5.0, a_xi=2.0, dt=0.005, equation=EQ_EL, kbt=1.0,
                            salt=True, valency=(1.0, -1.0), onsager=(1.0, 1.0), debye_length=4.0,
                            surface_charge=-20.0, e_field="DC", e_ext=(0.05, 0.0, 0.0), dielectric=1.0)
            parts = make_particles(cfg, seed=3, v_sd=1e-3, random_orientation=True)
        else:
            cfg = SPMConfig(npx=6, npy=6, npz=6, n_particles=50, a=5.0, a_xi=2.0, dt=0.1, janus_axis="Z",
                            janus_propulsion="SQUIRMER", slip_vel=0.015, slip_mode=2.0, slip_tol=0.005, slip_iter=4)
            parts = make_particles(cfg, seed=9, random_orientation=True)
        with SPMRun(cfg, precision=N.SPM_PREC_FP64) as run:
            run.initialize(parts)
            run.step(args.warmup)
            run.synchronize()
            ms = run.time_steps(args.steps)
            print(json.dumps({"profile_run": args.profile_run, "grid": cfg.shape, "steps": args.steps,
                              "ms_per_step": ms / args.steps}), flush=True)
        return 0
    cfg = workload_config()
    if os.environ.get("SPM_PROFILE_GRID"):
        import dataclasses
        k = int(os.environ["SPM_PROFILE_GRID"])
        cfg = dataclasses.replace(cfg, npx=k, npy=k, npz=k)
    parts = workload_particles(cfg)
    prec = N.SPM_PREC_FP32_MIXED if args.profile_run == "fp32" else N.SPM_PREC_FP64
    with SPMRun(cfg, precision=prec) as run:
        run.initialize(parts)
        run.step(args.warmup)
        run.synchronize()
        ms = run.time_steps(args.steps)
        print(json.dumps({"profile_run": args.profile_run, "grid": cfg.shape, "steps": args.steps,
                          "ms_per_step": ms / args.steps}), flush=True)
    return 0


def step_bytes(cfg, w):
    """Algorithmic HBM bytes of one step: (2*20 + 12) field passes of
    S_w = N^2 (N+2) w bytes plus 13 words per stencil cell (FP64 words for
    the particle side)."""
    nx, ny, nz = cfg.shape
    S = nx * ny * (nz + 2) * w
    return 52 * S + cfg.n_particles * 1935 * 13 * 8


TRAFFIC_FILE = "profiles/spm_step_fp32_256cubed_dram_traffic.md"
SERVE_FP64_SAMPLE = 48


def read_traffic(kernel):
    """DRAM bytes per launch of a kernel family from the committed ncu
    capture (dram__bytes_read.sum + dram__bytes_write.sum per launch, lines
    `traffic_bytes_per_launch[<family>]: <bytes>`); None if absent."""
    try:
        for line in open(os.path.join(ROOT, TRAFFIC_FILE)):
            if line.startswith(f"traffic_bytes_per_launch[{kernel}]:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def profile_kernels(run, K):
    from kapsel3_b200 import _native as N
    buf = C.create_string_buffer(1 << 16)
    N.check(N.lib().spm_profile_kernels(run.h, K, buf, len(buf)), "spm_profile_kernels")
    return json.loads(buf.value.decode())


def kernel_table(prof, K, peak):
    """Per kernel family: launches and device time per step, time and
    algorithmic bytes per launch, achieved GB/s and the fraction of the
    measured HBM peak (0 for kernels without an HBM-bound byte count)."""
    rows = []
    for k in prof["kernels"]:
        us, b = k["us_per_launch"], k["bytes_per_launch"]
        gbs = b / (us * 1e-6) / 1e9 if us > 0 and b > 0 else 0.0
        rows.append({"kernel": k["name"], "launches_per_step": k["launches"] / K, "us_per_launch": us,
                     "us_per_step": k["us_total"] / K, "bytes_per_launch": b, "achieved_gbs": gbs,
                     "frac": gbs / peak})
    rows.sort(key=lambda r: -r["us_per_step"])
    return rows


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured (MEASURED_PEAKS.json)"}
    except Exception:
        return {"hbm_gbs": 6650.0, "source": "fallback 6.65 TB/s"}


def accuracy_check(cfg, parts, steps=500, every=50):
    """The precision form's error report (the 256^3 / 1000-colloid
    configuration at its full length, 500 steps): FP32-mixed and FP64 runs
    from the same state advance side by side; every 50 steps the relative L2
    error of u, phi and particle x, v, omega against FP64."""
    from kapsel3_b200 import _native as N
    from kapsel3_b200.spm import SPMRun

    def rel(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    series = []
    with SPMRun(cfg, precision=N.SPM_PREC_FP32_MIXED) as r32, SPMRun(cfg, precision=N.SPM_PREC_FP64) as r64:
        r32.initialize(parts)
        r64.initialize(parts)
        for ts in range(every, steps + 1, every):
            r32.step(every)
            r64.step(every)
            p32, p64 = r32.particles(), r64.particles()
            e = {"ts": ts, "u": rel(r32.velocity(), r64.velocity()), "phi": rel(r32.phi(), r64.phi())}
            for k in ("x", "v", "omega"):
                e[k] = rel(p32[k], p64[k])
            series.append(e)
    last = series[-1]
    worst = max(max(e[k] for k in ("u", "phi", "x", "v", "omega")) for e in series)
    return {"steps": steps, "every": every, "series": series, "rel_l2_u": last["u"], "rel_l2_phi": last["phi"],
            "rel_l2_x": last["x"], "rel_l2_v": last["v"], "rel_l2_omega": last["omega"], "max_over_series": worst,
            "meets_1e-5": worst <= 1e-5}


if __name__ == "__main__":
    sys.exit(main())
