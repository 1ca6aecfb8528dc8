"""Rigid bodies on the GPU beyond the per-step fixture comparison (every
rigid fixture is also stepped by tests/test_gpu_golden.py):

* the body state a run reports (spm_get_rigid) against its beads: every
  bead carries its body's angular velocity, the beads keep their distances,
  and a body's centre takes the Adams-Bashforth step of its velocities;
* the FP32-mixed field path against FP64 on a rigid fixture;
* checkpoint / restart of a rigid run (the bodies' state, their previous
  forces and the MT19937 state of the rigid thermostat);
* a fixed body keeps the velocity it was given and the angular velocity
  its body-frame Rigid_omega had in space at the start (Rigid_motion fix;
  init_set_vGs, rigid.h:248-251)."""
import os

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from tests.golden_util import load, rel

pytestmark = pytest.mark.gpu


def _first(cfg):
    first = [0]
    for beads, count, *_ in cfg.rigid:
        for _ in range(int(count)):
            first.append(first[-1] + int(beads))
    return first


def _rotate(q, v):
    """q v q* for a unit quaternion q = (s, x, y, z)."""
    s, u = q[0], np.asarray(q[1:])
    return v + 2.0 * s * np.cross(u, v) + 2.0 * np.cross(u, np.cross(u, v))


@pytest.mark.parametrize("name", ["rigid_species_dof_thermostat", "example10_rigid_free_sedimenting"])
def test_body_state_matches_its_beads(gpu, name):
    cfg, parts, z = load(name)
    first = _first(cfg)
    with SPMRun(cfg) as run:
        run.initialize(parts)
        b0 = run.rigid_bodies()
        p0 = run.particles()
        run.step(8)
        b8 = run.rigid_bodies()
        run.step(1)
        b9 = run.rigid_bodies()
        run.step(1)
        b1 = run.rigid_bodies()
        p1 = run.particles()
    nb = len(first) - 1
    assert b1["xg"].shape == (nb, 3) and b1["mass"].shape == (nb,)
    for b in range(nb):
        sl = slice(first[b], first[b + 1])
        if cfg.kbt == 0.0:  # the rigid thermostat leaves the beads' angular velocities behind (fluct.cxx:40-95)
            assert (p1["omega"][sl] == b1["wg"][b]).all()
        d0 = np.linalg.norm(p0["x_nopbc"][sl, None] - p0["x_nopbc"][None, sl], axis=-1)
        d1 = np.linalg.norm(p1["x_nopbc"][sl, None] - p1["x_nopbc"][None, sl], axis=-1)
        assert np.abs(d1 - d0).max() < 1e-10
        # the centre without the wrap takes the second-order Adams-Bashforth step (solver_Rigid_Position)
        moved = b1["xg_nopbc"][b] - b9["xg_nopbc"][b]
        want = 0.5 * cfg.dt * (3.0 * b9["vg"][b] - b8["vg"][b])
        assert np.abs(moved - want).max() <= 1e-9 * np.abs(want).max() + 1e-15
        assert b1["mass"][b] == b0["mass"][b] > 0


def test_fp32_mixed_rigid_follows_fp64(gpu):
    cfg, parts, z = load("rigid_32_free_gravity")
    out = {}
    for prec in (N.SPM_PREC_FP64, N.SPM_PREC_FP32_MIXED):
        with SPMRun(cfg, precision=prec) as run:
            run.initialize(parts)
            run.step(60)
            out[prec] = run.particles()
    for k in ("x", "v", "omega"):
        assert rel(out[N.SPM_PREC_FP32_MIXED][k], out[N.SPM_PREC_FP64][k]) < 1e-4, k
    # and FP64 is the reference's trajectory
    assert rel(out[N.SPM_PREC_FP64]["v"], z["traj_v"][60]) < 1e-10


def test_rigid_checkpoint_continues_like_the_original(gpu, tmp_path):
    cfg, parts, z = load("rigid_species_dof_thermostat")
    path = os.path.join(tmp_path, "rigid.ck")
    with SPMRun(cfg) as a:
        a.initialize(parts)
        a.step(7)
        a.save_state(path)
        a.step(6)
        pa, ba = a.particles(), a.rigid_bodies()
    with SPMRun(cfg) as b:
        b.load_state(path)
        assert b.time()[0] == 7
        b.step(6)
        pb, bb = b.particles(), b.rigid_bodies()
    for k in ("x", "v", "omega", "q"):
        assert rel(pb[k], pa[k]) < 1e-12, k
    for k in ("xg", "vg", "wg"):
        assert rel(bb[k], ba[k]) < 1e-12, k
    assert rel(pb["v"], z["traj_v"][13]) < 1e-10


def test_fixed_body_keeps_its_motion(gpu):
    cfg, parts, z = load("rigid_32_fixed_motion")
    vel = np.array(cfg.rigid[0][4])
    w_body = np.array(cfg.rigid[0][5])
    first = _first(cfg)
    with SPMRun(cfg) as run:
        run.initialize(parts)
        q0 = run.particles()["q"]
        for _ in range(4):
            run.step(10)
            bodies = run.rigid_bodies()
            for b in range(len(first) - 1):
                assert np.abs(bodies["vg"][b] - vel).max() < 1e-15
                # the body-frame angular velocity turned to space once, by the initial orientation
                # (init_set_vGs, rigid.h:248-251), and kept there
                w = _rotate(q0[first[b]], w_body)
                assert np.abs(bodies["wg"][b] - w).max() < 1e-12 * np.linalg.norm(w_body)


@pytest.mark.skipif(not __import__("oracle.ref_runner", fromlist=["x"]).available(),
                    reason="reference program not built (oracle/_ref)")
@pytest.mark.parametrize("ac", [False, True])
def test_rigid_bodies_under_sustained_shear_match_the_reference(gpu, ac, tmp_path):
    """Rigid bodies in a Shear_Navier_Stokes box (as the reference's
    Examples/08/s001_t000_rigid.udf): the reference program's particles and
    zeta after every step within 1e-10, and its stress line."""
    import dataclasses

    from kapsel3_b200.udf import EQ_SNS, make_rigid_bodies, write_udf_keys
    from oracle import ref_runner

    cfg, _, _ = load("rigid_32_free_gravity")
    cfg = dataclasses.replace(cfg, equation=EQ_SNS, shear_rate=0.03, shear_ac=ac, shear_frequency=0.4,
                              rigid_gravity=(0.0, 0.0, 0.0), gts=1, num_snap=6)
    parts = make_rigid_bodies(cfg, seed=31)
    keys, dump = str(tmp_path / "in.keys"), str(tmp_path / "d.bin")
    write_udf_keys(keys, cfg, parts, out_dir=str(tmp_path / "avs"))
    err = ref_runner.run_reference(keys, dump, fields_every=1, timeout=600)
    frames = ref_runner.read_dump(dump)["frames"]
    width = 6 if ac else 5
    lines = []
    for line in err.splitlines():
        f = line.split()
        if len(f) == width and not line.startswith("#"):
            try:
                lines.append([float(v) for v in f])
            except ValueError:
                pass
    with SPMRun(cfg) as run:
        run.initialize(parts)
        for fr in frames:
            if fr["ts"] > 0:
                run.step(1)
                deg, st = run.shear_state()
                ours = [run.time()[1], st[0], st[1], st[2]] + ([st[4], st[5]] if ac else [st[3]])
                for a, b in zip(ours, lines[fr["ts"] - 1]):
                    assert abs(a - b) <= 6e-8 * abs(b) + 1e-14, (fr["ts"], ours, lines[fr["ts"] - 1])
            p = run.particles()
            for k in ("x", "v", "omega", "q"):
                assert rel(p[k], fr[k]) < 1e-10, (fr["ts"], k, rel(p[k], fr[k]))
            z, _ = run.zeta()
            assert rel(z, fr["zeta"]) < 1e-10, (fr["ts"], "zeta")


def _rigid_le_case(kbt):
    """Two bent three-bead bodies in a 32^3 Lees-Edwards box: body 0 reaches
    over the y boundary and its centre crosses it in the first steps (vG_y
    0.5), one bead of body 1 sits 1.08 SIGMA from a bead of body 0 (inside
    the WCA cutoff), so the bodies' Lennard-Jones force, torque and stress
    act from the first step."""
    import dataclasses

    from kapsel3_b200.udf import EQ_LE

    cfg, _, _ = load("rigid_32_free_gravity")
    cfg = dataclasses.replace(cfg, equation=EQ_LE, shear_rate=0.05, rigid_gravity=(0.0, 0.0, 0.0), kbt=kbt,
                              rigid=((3, 2, 1.5, "free", (0.0, 0.5, 0.0), (0.0, 0.0, 0.02)),), gts=1, num_snap=8)
    s, h = 3.6, 3.6 * np.sin(np.deg2rad(60.0))
    a0 = np.array([10.0, 30.94, 16.0])
    body0 = [a0, a0 + [s, 0.0, 0.0], a0 + [s + s / 2, h, 0.0]]
    b0 = a0 + [0.0, 0.0, 1.08 * 6.0]
    body1 = [b0, b0 + [-s, 0.0, 0.0], b0 + [-s - s / 2, -h, 0.0]]
    x = np.array(body0 + body1)
    n = len(x)
    parts = dict(x=x, v=np.zeros((n, 3)), q=np.tile(np.array([1.0, 0.0, 0.0, 0.0]), (n, 1)), omega=np.zeros((n, 3)))
    return cfg, parts


@pytest.mark.skipif(not __import__("oracle.ref_runner", fromlist=["x"]).available(),
                    reason="reference program not built (oracle/_ref)")
@pytest.mark.parametrize("kbt", [0.0, 1e-4])
def test_rigid_bodies_under_lees_edwards_match_the_reference(gpu, kbt, tmp_path):
    """Rigid bodies in a Lees-Edwards box (as the reference's
    Examples/08/helixes_shear0005.udf; solver_Rigid_Position_OBL,
    set_Particle_Velocities_OBL, the bodies' LJ and hydrodynamic stress): the
    reference program's particles, degree_oblique and retained zeta after
    every step within 1e-10, and every column of its stress line."""
    from kapsel3_b200.udf import write_udf_keys
    from oracle import ref_runner
    from tests.golden_util import retained

    cfg, parts = _rigid_le_case(kbt)
    keys, dump = str(tmp_path / "in.keys"), str(tmp_path / "d.bin")
    write_udf_keys(keys, cfg, parts, out_dir=str(tmp_path / "avs"))
    err = ref_runner.run_reference(keys, dump, fields_every=1, timeout=600)
    frames = ref_runner.read_dump(dump)["frames"]
    lines = [[float(v) for v in l.split()] for l in err.splitlines()
             if l and not l.startswith("#") and len(l.split()) == 12]
    # stress-line columns <- shear_state() entries (Mean_shear_stress, sp_3d_ns.h:296-339)
    cols = {"shear_rate": (1, 0), "strain": (3, 1), "lj": (4, 2), "hydro_old": (5, 3), "hydro_new": (6, 4),
            "reynolds": (7, 5), "fluid": (8, 6), "apparent": (10, 7)}
    assert any(abs(l[4]) > 0 for l in lines), "the bodies' LJ stress never acted"
    crossed = False
    with SPMRun(cfg) as run:
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
                assert rel(p[k], fr[k]) < 1e-10, (fr["ts"], k, rel(p[k], fr[k]))
            crossed |= bool(run.rigid_bodies()["xg"][0][1] < 16.0)
            z, _ = run.zeta()
            assert rel(retained(cfg, z), retained(cfg, fr["zeta"])) < 1e-10, (fr["ts"], "zeta")
    assert crossed, "body 0's centre did not cross the y boundary"
