"""Serving form on the GPU: run pools and the native request loop.

Parity bar: a run advanced inside a pool (batched FFT stages, CUDA-graph
replay, slot compaction, arena growth) matches the same run advanced alone in
its own context.  In FP64 the two differ only by the summation order of
float atomics in the shared-profile scatters (a few ulps where three or more
particles overlap one grid cell), so the bar is 1e-12 relative.  A FP32-mixed
run in the mix of the request loop matches the same request served alone
within 1e-6 relative velocity error, and FP32-mixed against FP64 within 1e-5.

Fault tests inject every failure on the host (bad requests, budget, cancel,
a failing device allocation); none faults or hangs the GPU."""
import ctypes as C

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.serve import Pool, Server, serving_workload
from kapsel3_b200.spm import SPMRun, pack_particles, unpack_particles
from kapsel3_b200.udf import EQ_LE, SPMConfig, make_particles

pytestmark = pytest.mark.gpu

TOL_POOL64 = 1e-12
TOL_MIX32 = 1e-6
TOL_32_VS_64 = 1e-5


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _case(npart, seed, side_lg=5, kbt=0.0, body=(0.0, 0.0, 0.0)):
    cfg = SPMConfig(npx=side_lg, npy=side_lg, npz=side_lg, n_particles=npart, a=4.0, a_xi=2.0, dt=0.05, kbt=kbt,
                    body_force=body)
    parts = make_particles(cfg, seed=seed, v_sd=1e-3, random_orientation=True)
    return cfg, pack_particles(parts, npart)


def _lone(cfg, rec, nsteps, prec):
    with SPMRun(cfg, precision=prec) as r:
        r.initialize(unpack_particles(rec))
        r.step(nsteps)
        return r.particles_record(), r.velocity()


def _cmp(rec_a, u_a, rec_b, u_b):
    pa, pb = unpack_particles(rec_a), unpack_particles(rec_b)
    return max(rel(u_a, u_b), rel(pa["x"], pb["x"]), rel(pa["v"], pb["v"]), rel(pa["omega"], pb["omega"]))


CASES = [_case(2, 11, body=(1e-3, 0, 0)), _case(5, 12, kbt=1e-5), _case(9, 13)]


@pytest.mark.parametrize("use_graph", [True, False])
def test_pool_runs_match_lone_runs(gpu, use_graph):
    nsteps = 12
    with Pool(CASES[0][0], precision=N.SPM_PREC_FP64, capacity=4) as pool:
        runs = [pool.admit(cfg, rec) for cfg, rec in CASES]
        for _ in range(nsteps):
            pool.step(1, use_graph=use_graph)
        _, errs = pool.synchronize()
        assert errs == [0, 0, 0]
        got = [(pool.particles(r, cfg.n_particles), pool.velocity(r, cfg.shape)) for r, (cfg, _) in zip(runs, CASES)]
        if use_graph:
            st = pool.stats()
            assert st["captures"] == 1 and st["graph_kernels"] > 0
    for (cfg, rec), (p, u) in zip(CASES, got):
        p0, u0 = _lone(cfg, rec, nsteps, N.SPM_PREC_FP64)
        assert _cmp(p, u, p0, u0) <= TOL_POOL64


def test_pool_release_and_growth_keep_runs_exact(gpu):
    """Capacity 1 grows to 2 and 4; releasing the first run moves the last
    one into its slot; the graph is re-captured each time."""
    n1, n2 = 5, 7
    with Pool(CASES[0][0], precision=N.SPM_PREC_FP64, capacity=1) as pool:
        runs = [pool.admit(cfg, rec) for cfg, rec in CASES]
        assert pool.size() == (3, 4)
        pool.step(n1)
        pool.release(runs[0])
        assert pool.size() == (2, 4)
        pool.step(n2)
        pool.synchronize()
        got = [(pool.particles(r, cfg.n_particles), pool.velocity(r, cfg.shape))
               for r, (cfg, _) in zip(runs[1:], CASES[1:])]
        assert pool.stats()["captures"] == 2
    for (cfg, rec), (p, u) in zip(CASES[1:], got):
        p0, u0 = _lone(cfg, rec, n1 + n2, N.SPM_PREC_FP64)
        assert _cmp(p, u, p0, u0) <= TOL_POOL64


def test_pool_fp32_mixed_close_to_fp64(gpu):
    nsteps = 10
    with Pool(CASES[0][0], precision=N.SPM_PREC_FP32_MIXED, capacity=4) as pool:
        runs = [pool.admit(cfg, rec) for cfg, rec in CASES]
        pool.step(nsteps)
        pool.synchronize()
        got = [pool.velocity(r, cfg.shape) for r, (cfg, _) in zip(runs, CASES)]
    for (cfg, rec), u in zip(CASES, got):
        _, u64 = _lone(cfg, rec, nsteps, N.SPM_PREC_FP64)
        assert rel(u, u64) <= TOL_32_VS_64


def test_pool_rejects_mismatched_runs(gpu):
    cfg, rec = CASES[0]
    with Pool(cfg, precision=N.SPM_PREC_FP64) as pool:
        other, orec = _case(2, 3, side_lg=6)
        with pytest.raises(N.SpmError):
            pool.admit(other, orec)
        le = SPMConfig(npx=5, npy=5, npz=5, n_particles=2, equation=EQ_LE, shear_rate=0.01)
        with pytest.raises(N.SpmError):
            Pool(le)
        assert pool.size()[0] == 0


def _serve(reqs, **kw):
    with Server(**kw) as srv:
        ids = [srv.submit(cfg, rec, n, keep_velocity=True) for cfg, rec, n in reqs]
        states = [srv.wait(i, 300.0) for i in ids]
        assert states == [N.SPM_REQ_DONE] * len(ids), [srv.status(i) for i in ids]
        out = [srv.result(i, cfg.n_particles, cfg.shape) for i, (cfg, _, _) in zip(ids, reqs)]
        return out, srv.stats()


def test_request_alone_equals_request_in_mix(gpu):
    target = (*_case(6, 21), 30)
    mix = [(*_case(3, 22), 25), (*_case(40, 23, side_lg=6), 30), target, (*_case(8, 24), 17),
           (*_case(1, 25, side_lg=6), 40)]
    alone, _ = _serve([target])
    mixed, stats = _serve(mix)
    a, m = alone[0], mixed[2]
    pa, pm = unpack_particles(a["particles"]), unpack_particles(m["particles"])
    err = max(rel(m["velocity"], a["velocity"]), rel(pm["x"], pa["x"]), rel(pm["v"], pa["v"]))
    assert err <= TOL_MIX32, err
    assert stats["completed"] == len(mix) and stats["max_active"] >= 2
    assert stats["run_steps"] == sum(n for _, _, n in mix)
    assert stats["step_latency_p99_ms"] >= stats["step_latency_p50_ms"] > 0


def test_budget_admission_queues_until_memory_frees(gpu):
    cfg, rec = _case(4, 31, side_lg=6)
    arena_b = __import__("ctypes").c_size_t()
    run_b = __import__("ctypes").c_size_t()
    from kapsel3_b200.spm import params_from_config
    p = params_from_config(cfg, N.SPM_PREC_FP32_MIXED)
    L = N.lib()
    N.check(L.spm_pool_device_bytes(p, 2, arena_b, run_b), "spm_pool_device_bytes")
    # room for one pool of two runs, not for a growth to four
    budget = arena_b.value + 2 * run_b.value + 1024
    reqs = [(cfg, rec, 20) for _ in range(5)]
    out, stats = _serve(reqs, budget_bytes=budget, pool_capacity=2)
    assert stats["completed"] == 5 and stats["max_active"] <= 2
    assert stats["peak_bytes"] <= budget
    for o in out[1:]:
        assert np.array_equal(o["particles"][:, :3], out[0]["particles"][:, :3]) or \
            rel(o["particles"][:, :3], out[0]["particles"][:, :3]) <= TOL_MIX32


def test_server_host_side_faults(gpu):
    cfg, rec = _case(3, 41)
    with Server(budget_bytes=4 << 30) as srv:
        bad = SPMConfig(npx=2, npy=5, npz=5, n_particles=3)
        assert srv.try_submit(bad, rec, 10)[0] != 0                       # malformed grid
        le = SPMConfig(npx=5, npy=5, npz=5, n_particles=3, equation=EQ_LE, shear_rate=0.01)
        assert srv.try_submit(le, rec, 10)[0] != 0                        # not served by pools
        out_of_box = rec.copy()
        out_of_box[0, 0] = 1e6
        assert srv.try_submit(cfg, out_of_box, 10)[0] != 0                # particle outside the box
        huge = SPMConfig(npx=9, npy=9, npz=9, n_particles=3)
        assert srv.try_submit(huge, rec, 10)[0] != 0                      # larger than the budget
        # cancelled while running or queued
        long_id = srv.submit(cfg, rec, 100000)
        srv.cancel(long_id)
        assert srv.wait(long_id, 60.0) == N.SPM_REQ_CANCELLED
        # a failing device allocation fails that request only
        N.check(N.lib().spm_debug_fail_allocations(1), "inject")
        bad_id = srv.submit(cfg, rec, 5)
        assert srv.wait(bad_id, 60.0) == N.SPM_REQ_FAILED
        st = srv.status(bad_id)
        assert st["status"] == 3, st                                      # SPM_ERR_NOMEM
        N.check(N.lib().spm_debug_fail_allocations(0), "inject off")
        ok_id = srv.submit(cfg, rec, 5)
        assert srv.wait(ok_id, 60.0) == N.SPM_REQ_DONE
        s = srv.stats()
        assert s["rejected"] == 4 and s["cancelled"] == 1 and s["failed"] == 1 and s["completed"] == 1


def test_serving_stream_small(gpu):
    """A short seeded stream with real-time arrivals across three grid sizes."""
    w = serving_workload(n_runs=12, rate_per_s=40.0, sides=(32, 64), np_max=30, nsteps=20, seed=7)
    from kapsel3_b200.serve import run_stream
    with Server() as srv:
        res = run_stream(srv, w["requests"])
    assert all(r["state"] == N.SPM_REQ_DONE for r in res["results"])
    assert res["stats"]["run_steps"] == 12 * 20
    assert len(res["latencies"]) == 12 * 20


def test_retired_memory_returns_to_the_pool_without_a_stall(gpu):
    """Pools and runs take their device memory from the library's stream-ordered
    memory pool: destroying a pool while another steps does not wait for the
    device (the worker's longest pool destruction stays at milliseconds), the
    freed blocks are handed out again, and spm_release_cached_memory returns
    the unused part to the driver with the library still usable."""
    w = serving_workload(n_runs=16, rate_per_s=200.0, sides=(32, 64), np_max=20, nsteps=30, seed=11)
    from kapsel3_b200.serve import run_stream
    with Server(pool_idle_s=0.0) as srv:
        res = run_stream(srv, w["requests"])
    st = res["stats"]
    assert all(r["state"] == N.SPM_REQ_DONE for r in res["results"])
    assert st["pool_destroy_max_ms"] < 100.0, st
    held = C.c_size_t()
    N.check(N.lib().spm_release_cached_memory(C.byref(held)), "spm_release_cached_memory")
    cfg1 = SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.05)
    with SPMRun(cfg1) as run:
        run.initialize(make_particles(cfg1, seed=1))
        run.step(2)
        assert np.isfinite(run.particles()["v"]).all()
