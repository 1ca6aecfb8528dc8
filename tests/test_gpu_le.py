"""Lees-Edwards (sheared) GPU step against the reference program's fixtures
(tests/golden/le_*.npz) and the oracle: particle trajectories, retained
vorticity modes, degree_oblique, and every term of the reference's per-step
shear-stress line (Mean_shear_stress, sp_3d_ns.h:296-339)."""
import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from kapsel3_b200.udf import EQ_LE, SPMConfig, make_particles
from oracle.spm_oracle import OracleSPMLE
from tests.golden_util import check_state, fixture_names, load, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10
LE_FIXTURES = [n for n in fixture_names() if n.startswith("le_")]
# stress-line columns (reference) <- shear_state() entries
COLS = {"shear_rate": (1, 0), "strain": (3, 1), "lj": (4, 2), "hydro_old": (5, 3), "hydro_new": (6, 4),
        "reynolds": (7, 5), "fluid": (8, 6), "apparent": (10, 7)}


@pytest.mark.parametrize("name", LE_FIXTURES)
def test_le_matches_reference_fixture(gpu, name):
    cfg, parts, z = load(name)
    assert cfg.equation == EQ_LE
    steps = set(int(s) for s in z["field_steps"])
    nframes = len(z["traj_ts"])
    with SPMRun(cfg) as run:
        run.initialize(parts)
        for ts in range(nframes):
            p = run.particles()
            zeta = run.zeta()[0] if ts in steps else None
            worst, errs = check_state(z, ts, cfg, p["x"], p["v"], p["omega"], p["q"], p["f_hydro_previous"],
                                      zeta=zeta, tol=TOL)
            assert worst < TOL, (name, ts, errs)
            deg, st = run.shear_state()
            assert abs(deg - z["traj_degree_oblique"][ts]) < 1e-13
            if ts + 1 < nframes:
                run.step(1)
                deg, st = run.shear_state()
                ref = z["stress_lines"][ts]
                for k, (ci, si) in COLS.items():
                    assert abs(st[si] - ref[ci]) <= 6e-8 * abs(ref[ci]) + 1e-18, (name, ts, k, st[si], ref[ci])


def _le_case():
    cfg = SPMConfig(npx=5, npy=5, npz=5, n_particles=6, a=3.5, a_xi=2.0, dt=0.05, equation=EQ_LE, shear_rate=0.05,
                    kbt=0.0)
    parts = make_particles(cfg, seed=29, v_sd=1e-3, random_orientation=True, min_dist_factor=0.93)
    return cfg, parts


def test_le_fp64_tracks_oracle_with_lj(gpu):
    cfg, parts = _le_case()
    o = OracleSPMLE(cfg, parts)
    with SPMRun(cfg) as run:
        run.initialize(parts)
        for s in range(16):
            run.step(1)
            o.step()
            p = run.particles()
            assert rel(p["x"], o.x) < TOL and rel(p["v"], o.v) < TOL and rel(p["omega"], o.omega) < TOL
            _, st = run.shear_state()
            assert abs(st[2] - o.stress["lj"]) <= 1e-9 * max(abs(o.stress["lj"]), 1e-30) + 1e-30
            assert abs(st[4] - o.stress["hydro_new"]) <= 1e-9 * abs(o.stress["hydro_new"])
        u = run.velocity()
    assert rel(u, o.velocity_field_obl()) < TOL


def test_le_fp32_mixed_close_to_fp64(gpu):
    cfg, parts = _le_case()
    res = {}
    for prec in (N.SPM_PREC_FP64, N.SPM_PREC_FP32_MIXED):
        with SPMRun(cfg, precision=prec) as run:
            run.initialize(parts)
            run.step(10)
            res[prec] = (run.velocity(), run.particles(), run.shear_state()[1])
    (u64, p64, s64), (u32, p32, s32) = res[N.SPM_PREC_FP64], res[N.SPM_PREC_FP32_MIXED]
    assert rel(u32, u64) < 1e-5
    assert rel(p32["x"], p64["x"]) < 1e-7
    assert abs(s32[7] - s64[7]) <= 1e-4 * abs(s64[7])
