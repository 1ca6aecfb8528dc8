"""Janus particles against the reference program built from its sources
(oracle/_ref/kapsel_ref), on the same seeded inputs: particle state, zeta and
the real-space velocity after every step, FP64, within 1e-10 relative.

Cases: squirmers with the self-consistent slip iteration (the SW_JANUS_SLIP
branch of Time_evolution_hydro, sp_3d_ns.cxx:121-161) as in the reference's
squirmer example (B1, alpha = 2, SLIP_tol 0.005, SLIP_iter 4), pushers with
rotlet terms converging to a tight tolerance, tumblers with a body-frame
force and torque (self_propulsion), and obstacles with the thermostat on
(fixed particles that draw no noise), also in a Lees-Edwards box (the
obstacle branches of the _OBL particle solvers)."""
import dataclasses

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from kapsel3_b200.udf import EQ_LE, SPMConfig, make_particles, write_udf_keys
from oracle import ref_runner

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


CASES = {
    "squirmer_example": SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.05,
                                  janus_axis="Z", janus_propulsion="SQUIRMER", slip_vel=0.015, slip_mode=2.0,
                                  slip_tol=0.005, slip_iter=4, gts=1, num_snap=8),
    "pushers_rotlet": SPMConfig(npx=5, npy=5, npz=6, n_particles=3, a=4.0, a_xi=2.0, dt=0.05,
                                janus_axis="X", janus_propulsion="SQUIRMER", slip_vel=0.02, slip_mode=-3.0,
                                rotlet_c1=0.01, rotlet_c2=-0.005, slip_tol=1e-6, slip_iter=30, gts=1, num_snap=8),
    "tumblers": SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=4.0, a_xi=2.0, dt=0.05, janus_axis="Z",
                          janus_propulsion="TUMBLER", janus_force=(0.02, 0.0, -0.01),
                          janus_torque=(0.0, 0.01, 0.03), gts=1, num_snap=8),
    "obstacles_thermostat": SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.05, kbt=1e-3,
                                      janus_propulsion="OBSTACLE", body_force=(1e-3, 0.0, 0.0), gts=1,
                                      num_snap=6),
}


@pytest.mark.skipif(not ref_runner.available(), reason="oracle/_ref is not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_janus_particles_match_the_reference_program(gpu, name, tmp_path):
    cfg = CASES[name]
    parts = make_particles(cfg, seed=13, v_sd=1e-3, random_orientation=True)
    keys, dump = str(tmp_path / "in.keys"), str(tmp_path / "d.bin")
    write_udf_keys(keys, cfg, parts, out_dir=str(tmp_path / "avs"))
    ref_runner.run_reference(keys, dump, fields_every=1, timeout=600, body_force=cfg.body_force)
    frames = ref_runner.read_dump(dump)["frames"]
    assert len(frames) == cfg.mstep + 1
    with SPMRun(cfg, precision=N.SPM_PREC_FP64) as run:
        run.initialize(parts)
        for fr in frames:
            if fr["ts"] > 0:
                run.step(1)
            p = run.particles()
            for k in ("x", "v", "omega", "q"):
                assert rel(p[k], fr[k]) <= TOL, (name, fr["ts"], k, rel(p[k], fr[k]))
            z, _ = run.zeta()
            assert rel(z, fr["zeta"]) <= TOL, (name, fr["ts"], "zeta", rel(z, fr["zeta"]))
            if fr["ts"] > 0:
                u = run.velocity()
                assert rel(u, fr["u"]) <= TOL, (name, fr["ts"], "u", rel(u, fr["u"]))
    if name == "obstacles_thermostat":
        assert not p["v"].any() and np.array_equal(p["x"], parts["x"])


OBSTACLES_LE = SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=4.0, a_xi=2.0, dt=0.05, equation=EQ_LE,
                         shear_rate=0.05, kbt=1e-3, janus_propulsion="OBSTACLE", body_force=(1e-3, 0.0, 0.0),
                         gts=1, num_snap=6)


@pytest.mark.skipif(not ref_runner.available(), reason="oracle/_ref is not built")
def test_obstacles_under_lees_edwards_match_the_reference_program(gpu, tmp_path):
    """Obstacles in a sheared box with the thermostat on: the obstacle branches
    of MD_solver_velocity_*_OBL and MD_solver_position_*_OBL
    (particle_solver.cxx:283-432) -- fixed, drawing no noise, out of the LJ
    pairs, their momentum_depend_fr (the body force) still feeding the
    hydrodynamic stress.  Particles, degree_oblique, the retained vorticity
    modes and every term of the shear-stress line after every step."""
    from tests.golden_util import retained

    cfg = OBSTACLES_LE
    parts = make_particles(cfg, seed=17, v_sd=1e-3, random_orientation=True)
    keys, dump = str(tmp_path / "in.keys"), str(tmp_path / "d.bin")
    write_udf_keys(keys, cfg, parts, out_dir=str(tmp_path / "avs"))
    err = ref_runner.run_reference(keys, dump, fields_every=1, timeout=600, body_force=cfg.body_force)
    frames = ref_runner.read_dump(dump)["frames"]
    assert len(frames) == cfg.mstep + 1
    lines = [[float(v) for v in l.split()] for l in err.splitlines()
             if l and not l.startswith("#") and len(l.split()) == 12]
    assert len(lines) >= cfg.mstep
    # stress-line columns <- shear_state() entries (Mean_shear_stress, sp_3d_ns.h:296-339)
    cols = {"shear_rate": (1, 0), "strain": (3, 1), "lj": (4, 2), "hydro_old": (5, 3), "hydro_new": (6, 4),
            "reynolds": (7, 5), "fluid": (8, 6), "apparent": (10, 7)}
    with SPMRun(cfg, precision=N.SPM_PREC_FP64) as run:
        run.initialize(parts)
        for fr in frames:
            if fr["ts"] > 0:
                run.step(1)
                deg, st = run.shear_state()
                assert abs(deg - fr["degree_oblique"]) < 1e-13
                ref = lines[fr["ts"] - 1]
                for k, (ci, si) in cols.items():
                    assert abs(st[si] - ref[ci]) <= 6e-8 * abs(ref[ci]) + 1e-14, (fr["ts"], k, st[si], ref[ci])
            p = run.particles()
            for k in ("x", "v", "omega", "q", "f_hydro_previous"):
                assert rel(p[k], fr[k]) <= TOL, (fr["ts"], k, rel(p[k], fr[k]))
            z, _ = run.zeta()
            assert rel(retained(cfg, z), retained(cfg, fr["zeta"])) <= TOL, (fr["ts"], "zeta")
    assert not p["v"].any() and np.array_equal(p["x"], parts["x"])


@pytest.mark.parametrize("prop", ["TUMBLER", "SQUIRMER"])
def test_self_propelled_janus_outside_navier_stokes_is_refused(gpu, prop):
    """The reference stops a run with tumblers or squirmers under any other
    solver (input.cxx:1509-1512)."""
    base = CASES["tumblers" if prop == "TUMBLER" else "squirmer_example"]
    cfg = dataclasses.replace(base, equation=EQ_LE, shear_rate=0.05)
    with pytest.raises(N.SpmError, match="tumblers and squirmers are served"):
        with SPMRun(cfg, precision=N.SPM_PREC_FP64):
            pass


def test_squirmers_fp32_mixed_close_to_fp64(gpu):
    cfg = CASES["pushers_rotlet"]
    parts = make_particles(cfg, seed=13, v_sd=1e-3, random_orientation=True)
    out = {}
    for prec in (N.SPM_PREC_FP64, N.SPM_PREC_FP32_MIXED):
        with SPMRun(cfg, precision=prec) as run:
            run.initialize(parts)
            run.step(6)
            out[prec] = run.particles()["v"], run.velocity()
    assert rel(out[N.SPM_PREC_FP32_MIXED][0], out[N.SPM_PREC_FP64][0]) <= 1e-5
    assert rel(out[N.SPM_PREC_FP32_MIXED][1], out[N.SPM_PREC_FP64][1]) <= 1e-5
