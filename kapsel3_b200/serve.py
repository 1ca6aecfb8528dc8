"""Serving form of the SPM step over the C ABI: run pools and the request loop.

`Pool` wraps spm_pool_* (same-grid runs with batched FFT stages, stepped from
a captured CUDA graph); `Server` wraps spm_server_* (the native persistent
request loop: admission by device-memory budget, resident run state, pools
stepped continuously, per-step latency).  `serving_workload` builds the
request stream of the serving benchmark: exponential inter-arrival times,
cubic grids drawn from a set of sides, particle counts drawn uniformly and
capped at what random sequential addition can place in the box.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _native as N
from .spm import pack_particles, params_from_config, unpack_particles
from .udf import SPMConfig, make_particles


class Pool:
    """Runs of one grid size and precision sharing one device arena."""

    def __init__(self, cfg: SPMConfig, precision: int = N.SPM_PREC_FP32_MIXED, capacity: int = 4):
        self.L = N.lib()
        self.cfg = cfg
        self.precision = precision
        p = params_from_config(cfg, precision)
        h = C.c_void_p()
        N.check(self.L.spm_pool_create(C.byref(p), capacity, None, C.byref(h)), "spm_pool_create")
        self.h = h
        self.runs: List[int] = []

    def close(self):
        if self.h:
            self.L.spm_pool_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def admit(self, cfg: SPMConfig, particles, mt_seed: int = 0) -> C.c_void_p:
        p = params_from_config(cfg, self.precision, mt_seed)
        rec = particles if isinstance(particles, np.ndarray) else pack_particles(particles, cfg.n_particles)
        rec = np.ascontiguousarray(rec, dtype=np.float64)
        run = C.c_void_p()
        N.check(self.L.spm_pool_admit(self.h, C.byref(p), N.dptr(rec) if rec.size else None, C.byref(run)),
                "spm_pool_admit")
        return run

    def release(self, run: C.c_void_p):
        N.check(self.L.spm_pool_release(self.h, run), "spm_pool_release")

    def size(self):
        n, cap = C.c_int(), C.c_int()
        N.check(self.L.spm_pool_size(self.h, C.byref(n), C.byref(cap)), "spm_pool_size")
        return n.value, cap.value

    def step(self, n: int = 1, use_graph: bool = True):
        N.check(self.L.spm_pool_step(self.h, n, 1 if use_graph else 0), "spm_pool_step")

    def synchronize(self):
        ms = C.c_float()
        n, _ = self.size()
        errs = (C.c_uint * max(n, 1))()
        N.check(self.L.spm_pool_synchronize(self.h, C.byref(ms), errs), "spm_pool_synchronize")
        return ms.value, [errs[i] for i in range(n)]

    def stats(self):
        k, cap = C.c_longlong(), C.c_int()
        N.check(self.L.spm_pool_stats(self.h, C.byref(k), C.byref(cap)), "spm_pool_stats")
        return dict(graph_kernels=k.value, captures=cap.value)

    # per-run getters through the whole-run C ABI
    def particles(self, run, n: int) -> np.ndarray:
        rec = np.zeros((n, N.SPM_PARTICLE_WORDS))
        if n:
            N.check(self.L.spm_get_particles(run, N.dptr(rec)), "spm_get_particles")
        return rec

    def velocity(self, run, shape) -> np.ndarray:
        nx, ny, nz = shape
        nf = nx * ny * 2 * (nz // 2 + 1)
        u = [np.zeros(nf) for _ in range(3)]
        N.check(self.L.spm_get_velocity(run, *[N.dptr(a) for a in u]), "spm_get_velocity")
        return np.stack([a.reshape(nx, ny, -1)[:, :, :nz] for a in u])


@dataclasses.dataclass
class Request:
    arrival_s: float
    cfg: SPMConfig
    particles: np.ndarray  # packed records
    nsteps: int
    seed: int


def max_packable(side: int, a: float = 4.0, seed: int = 0, tries: int = 20000, limit: int = 1 << 30) -> int:
    """Largest particle count random sequential addition places in a cubic box
    of `side` points (overlap length 1.05 * 2a, the reference's rule), for a
    fixed seed and `tries` consecutive failed attempts; stops at `limit`."""
    cfg = SPMConfig(npx=side.bit_length() - 1, npy=side.bit_length() - 1, npz=side.bit_length() - 1, a=a)
    L = side * cfg.dx
    rmin = 1.05 * 2 * a * cfg.dx
    rng = np.random.default_rng(seed)
    x = np.zeros((0, 3))
    fails = 0
    while fails < tries and len(x) < limit:
        c = rng.random(3) * L
        if len(x):
            dd = x - c
            dd -= np.rint(dd / L) * L
            if np.min((dd ** 2).sum(1)) <= rmin * rmin:
                fails += 1
                continue
        x = np.vstack([x, c])
        fails = 0
    return len(x)


def serving_workload(n_runs: int = 256, rate_per_s: float = 20.0, sides: Sequence[int] = (32, 64, 128),
                     np_max: int = 300, a: float = 4.0, a_xi: float = 2.0, nsteps: int = 200,
                     seed: int = 2024, pack_fraction: float = 0.5) -> Dict:
    """Seeded request stream: exponential inter-arrivals at `rate_per_s`, cubic
    side uniform over `sides`, Np uniform in [1, np_max] capped per side at
    `pack_fraction` of the random-sequential-addition maximum (so placement
    with the reference's overlap rule always succeeds quickly)."""
    rng = np.random.default_rng(seed)
    caps = {s: max(1, min(np_max, int(pack_fraction * max_packable(
        s, a, seed=seed, limit=int(np_max / pack_fraction) + 1)))) for s in sides}
    t = 0.0
    reqs = []
    for i in range(n_runs):
        t += rng.exponential(1.0 / rate_per_s)
        side = int(rng.choice(sides))
        npart = int(rng.integers(1, np_max + 1))
        npart = min(npart, caps[side])
        lg = side.bit_length() - 1
        cfg = SPMConfig(npx=lg, npy=lg, npz=lg, n_particles=npart, a=a, a_xi=a_xi, dt=0.05)
        ps = make_particles(cfg, seed=seed * 1000 + i, v_sd=1e-3, random_orientation=True)
        reqs.append(Request(t, cfg, pack_particles(ps, npart), nsteps, seed * 1000 + i))
    return dict(requests=reqs, np_cap=caps)


def partition(requests: List[Request], rank: int, world: int) -> List[Request]:
    """Share of a request stream served by replica `rank` of `world` (one
    server per GPU, runs never span GPUs): every world-th request."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return requests[rank::world]


class Server:
    """The native request loop (spm_server_*)."""

    def __init__(self, budget_bytes: int = 150 << 30, use_graph: bool = True, pool_capacity: int = 8,
                 steps_per_launch: int = 1, device: int = 0, pool_idle_s: Optional[float] = None):
        self.L = N.lib()
        cfg = N.SpmServerConfig()
        N.check(self.L.spm_server_config_default(C.byref(cfg)), "spm_server_config_default")
        cfg.budget_bytes = budget_bytes
        cfg.use_graph = 1 if use_graph else 0
        cfg.pool_initial_capacity = pool_capacity
        cfg.steps_per_launch = steps_per_launch
        cfg.device = device
        if pool_idle_s is not None:
            cfg.pool_idle_s = pool_idle_s
        h = C.c_void_p()
        N.check(self.L.spm_server_create(C.byref(cfg), C.byref(h)), "spm_server_create")
        self.h = h

    def close(self):
        if self.h:
            self.L.spm_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, cfg: SPMConfig, particles: np.ndarray, nsteps: int,
               precision: int = N.SPM_PREC_FP32_MIXED, keep_velocity: bool = False) -> int:
        p = params_from_config(cfg, precision)
        rec = np.ascontiguousarray(particles, dtype=np.float64)
        rid = C.c_longlong()
        N.check(self.L.spm_server_submit(self.h, C.byref(p), N.dptr(rec) if rec.size else None, nsteps,
                                         N.SPM_REQ_KEEP_VELOCITY if keep_velocity else 0, C.byref(rid)),
                "spm_server_submit")
        return rid.value

    def try_submit(self, *a, **k):
        """submit() that returns (status, message) instead of raising."""
        try:
            return 0, self.submit(*a, **k)
        except N.SpmError as e:
            return 1, str(e)

    def cancel(self, rid: int):
        N.check(self.L.spm_server_cancel(self.h, rid), "spm_server_cancel")

    def wait(self, rid: int, timeout_s: float = -1.0) -> int:
        st = C.c_int()
        N.check(self.L.spm_server_wait(self.h, rid, timeout_s, C.byref(st)), "spm_server_wait")
        return st.value

    def status(self, rid: int):
        st, code, steps = C.c_int(), C.c_int(), C.c_int()
        msg = C.create_string_buffer(512)
        N.check(self.L.spm_server_status(self.h, rid, C.byref(st), C.byref(code), C.byref(steps), msg, 512),
                "spm_server_status")
        return dict(state=st.value, status=code.value, steps=steps.value, message=msg.value.decode())

    def result(self, rid: int, n_particles: int, shape=None) -> Dict:
        rec = np.zeros((max(n_particles, 0), N.SPM_PARTICLE_WORDS))
        t, lat = C.c_double(), C.c_double()
        us = [None, None, None]
        if shape is not None:
            nx, ny, nz = shape
            nf = nx * ny * 2 * (nz // 2 + 1)
            us = [np.zeros(nf) for _ in range(3)]
        N.check(self.L.spm_server_result(self.h, rid, N.dptr(rec) if rec.size else None,
                                         *[N.dptr(a) if a is not None else None for a in us],
                                         C.byref(t), C.byref(lat)), "spm_server_result")
        out = dict(particles=rec, time=t.value, latency_s=lat.value)
        if shape is not None:
            nx, ny, nz = shape
            out["velocity"] = np.stack([a.reshape(nx, ny, -1)[:, :, :nz] for a in us])
        return out

    def forget(self, rid: int):
        N.check(self.L.spm_server_forget(self.h, rid), "spm_server_forget")

    def stats(self) -> Dict:
        s = N.SpmServerStats()
        N.check(self.L.spm_server_get_stats(self.h, C.byref(s)), "spm_server_get_stats")
        return {name: getattr(s, name) for name, _ in N.SpmServerStats._fields_}

    def latencies(self) -> np.ndarray:
        n = C.c_size_t()
        N.check(self.L.spm_server_latencies(self.h, None, 0, C.byref(n)), "spm_server_latencies")
        buf = (C.c_float * max(n.value, 1))()
        N.check(self.L.spm_server_latencies(self.h, buf, n.value, C.byref(n)), "spm_server_latencies")
        return np.frombuffer(buf, dtype=np.float32, count=n.value).copy()


def run_stream(server: Server, requests: List[Request], realtime: bool = True,
               keep_velocity_ids: Optional[set] = None, timeout_s: float = 600.0) -> Dict:
    """Submits `requests` at their arrival times (wall clock from now; all at
    once if not realtime), waits for all of them and returns per-request
    results and server statistics."""
    keep_velocity_ids = keep_velocity_ids or set()
    t0 = time.perf_counter()
    ids = []
    for i, r in enumerate(requests):
        if realtime:
            dt = r.arrival_s - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
        ids.append(server.submit(r.cfg, r.particles, r.nsteps, keep_velocity=i in keep_velocity_ids))
    out = []
    for i, rid in enumerate(ids):
        st = server.wait(rid, timeout_s)
        rec = dict(id=rid, state=st)
        if st == N.SPM_REQ_DONE:
            rec.update(server.result(rid, requests[i].cfg.n_particles,
                                     requests[i].cfg.shape if i in keep_velocity_ids else None))
        else:
            rec.update(server.status(rid))
        out.append(rec)
    wall = time.perf_counter() - t0
    return dict(results=out, stats=server.stats(), latencies=server.latencies(), wall_s=wall)


__all__ = ["Pool", "Server", "Request", "serving_workload", "run_stream", "max_packable", "partition",
           "unpack_particles"]
