"""Generates the golden fixtures of tests/golden/ by running the reference
program itself (oracle/_ref, built from the unmodified KAPSEL sources by
oracle/ref_build/Makefile) on seeded inputs.

    python tests/golden/make_golden.py

Each fixture stores the run's UDF-level description (SPMConfig fields + the
seeded initial particle state) and, for every step, the particle state the
reference dumped (x, v, omega, q, f_hydro_previous, torque_hydro_previous),
plus at a few steps the retained (2/3-rule) modes of zeta, uk_dc and
checksums of the velocity field.  Only this script reads the reference; the
tests read the .npz files.
"""
from __future__ import annotations

import dataclasses
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from kapsel3_b200.udf import EQ_LE, SPMConfig, make_particles, make_rigid_bodies, write_udf_keys  # noqa: E402
from kapsel3_b200.spm import config_from_udf, read_udf  # noqa: E402
from oracle import ref_runner  # noqa: E402

CASES = {
    # C1 of the benchmark plan: 32^3, two spheres a=4, body force 1e-3 along x
    "c1_32_two_spheres_body_force": dict(
        cfg=dict(npx=5, npy=5, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.05, body_force=(1e-3, 0.0, 0.0),
                 num_snap=100),
        init=dict(seed=1, v_sd=0.0, random_orientation=False), field_steps=(1, 100)),
    # thermostat (MT19937 + polar Box-Muller) with random orientations
    "thermostat_32_four_spheres": dict(
        cfg=dict(npx=5, npy=5, npz=5, n_particles=4, a=4.0, a_xi=2.0, dt=0.05, kbt=1e-4, num_snap=40),
        init=dict(seed=7, v_sd=1e-3, random_orientation=True), field_steps=(40,)),
    # non-cubic grid, lc = 1 on y (LJ pair multiplicity 3 per axis), close pairs
    "noncubic_lj_multiplicity": dict(
        cfg=dict(npx=5, npy=4, npz=6, n_particles=5, a=3.0, a_xi=2.0, dt=0.05, kbt=1e-5,
                 body_force=(0.0, 2e-3, -1e-3), num_snap=30),
        init=dict(seed=5, v_sd=2e-3, random_orientation=True, min_dist_factor=0.92), field_steps=(30,)),
    # Lees-Edwards: one sphere crosses the sheared y boundary, thermostat on
    "le_32_boundary_crossing": dict(
        cfg=dict(npx=5, npy=5, npz=5, n_particles=5, a=3.5, a_xi=2.0, dt=0.05, kbt=1e-5, equation=EQ_LE,
                 shear_rate=0.02, num_snap=40),
        init=dict(seed=13, v_sd=1e-3, random_orientation=True), field_steps=(40,),
        tweak=dict(index=0, x=(6.3, 31.998, 16.2), v=(0.0, 0.08, 0.0))),
    # C2 of the benchmark plan: 128^3, 200 spheres a=5, random orientations,
    # Gaussian velocities, thermostat kT=1e-4 (MT19937 seed 0), 1000 steps;
    # particle state every 50 steps (GTS=50), velocity checksums and the z=0
    # plane of u at steps 500 and 1000 (zeta modes are not stored at this size)
    "c2_128_200_spheres_thermostat": dict(
        cfg=dict(npx=7, npy=7, npz=7, n_particles=200, a=5.0, a_xi=2.0, dt=0.05, kbt=1e-4, gts=50, num_snap=20),
        init=dict(seed=2, v_sd=1e-3, random_orientation=True), field_steps=(500, 1000), fields_every=10,
        zeta=False),
    # Lees-Edwards: strain passes XYaspect = 1, the oblique grid is remapped
    "le_32_strain_remap": dict(
        cfg=dict(npx=5, npy=5, npz=5, n_particles=3, a=3.0, a_xi=2.0, dt=0.05, equation=EQ_LE, shear_rate=0.6,
                 num_snap=40),
        init=dict(seed=17, v_sd=1e-3, random_orientation=False), field_steps=(40,)),
    # rigid bodies (object_type rigid): two 4-bead bodies moving with a fixed
    # velocity and angular velocity (Rigid_motion fix), the first one across
    # the x edge of the box
    "rigid_32_fixed_motion": dict(
        cfg=dict(npx=5, npy=5, npz=5, n_particles=8, a=3.0, a_xi=2.0, dt=0.05, num_snap=40,
                 rigid=((4, 2, 1.0, "fix", (2e-3, -1e-3, 0.0), (0.0, 3e-3, 1e-3)),)),
        init=dict(seed=21, straddle=True), field_steps=(40,)),
    # free 3-bead bodies, MASS_RATIO 1.5, under gravity along -y
    "rigid_32_free_gravity": dict(
        cfg=dict(npx=5, npy=5, npz=5, n_particles=6, a=3.0, a_xi=2.0, dt=0.05, num_snap=60,
                 rigid=((3, 2, 1.5, "free", (0.0, 0.0, 0.0), (0.0, 0.0, 0.0)),), rigid_gravity=(0.0, 1e-3, 0.0)),
        init=dict(seed=22), field_steps=(60,)),
    # two species, non-cubic grid: free 3-bead bodies with two degrees of
    # freedom switched off (switch.free_rigid) and a fixed 4-bead body of
    # MASS_RATIO 2, thermostat on
    "rigid_species_dof_thermostat": dict(
        cfg=dict(npx=5, npy=5, npz=6, n_particles=10, a=3.0, a_xi=2.0, dt=0.05, kbt=1e-5, num_snap=40,
                 rigid=((3, 2, 1.0, "free", (0.0, 0.0, 0.0), (0.0, 0.0, 0.0)),
                        (4, 1, 2.0, "fix", (1e-3, 0.0, 0.0), (0.0, 0.0, 2e-3))),
                 rigid_dof=((0, (True, True, False), (False, True, True)),)),
        init=dict(seed=23), field_steps=(40,)),
    # the reference's own example inputs, shortened to a few dozen steps with
    # every step kept: Examples/12/a2_N65_Rer02.udf (65 one-bead bodies of
    # MASS_RATIO 1.5 spinning at a fixed body-frame rate, gravity along -z,
    # the x rotation switched off by switch.free_rigid; its flat wall and
    # Quincke switches, outside the step, turned off) and Examples/10/
    # input_rigid_free1.udf (a free 65-bead body sedimenting along -y on a
    # 64 x 128 x 64 grid)
    "example12_65_spinning_bodies": dict(example="Examples/12/a2_N65_Rer02.udf", num_snap=30, field_steps=(30,),
                                         overrides={"switch.wall.type": "NONE", "switch.quincke.type": "OFF"}),
    "example10_rigid_free_sedimenting": dict(example="Examples/10/input_rigid_free1.udf", num_snap=20,
                                             field_steps=(20,), zeta=False),
}


def retained_modes(cfg: SPMConfig, zeta: np.ndarray) -> np.ndarray:
    d = cfg.derived()
    nx, ny, nz = cfg.shape
    kx = np.arange(nx)
    kx = np.where(kx > nx // 2, kx - nx, kx)
    ky = np.arange(ny)
    ky = np.where(ky > ny // 2, ky - ny, ky)
    ix = np.where(np.abs(kx) < d["TRN_X"])[0]
    iy = np.where(np.abs(ky) < d["TRN_Y"])[0]
    return zeta[:, ix][:, :, iy][:, :, :, :d["TRN_Z"]]


def make_case(name, spec):
    if "example" in spec:
        tree = ref_runner.reference_tree()
        if tree is None:
            raise SystemExit("the reference sources are needed for " + spec["example"])
        kv = read_udf(os.path.join(tree, spec["example"]))
        kv.update(spec.get("overrides", {}))
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "example.keys")
            with open(path, "w") as f:
                f.writelines(f"{k} = {v}\n" for k, v in kv.items())
            cfg, parts = config_from_udf(path)
        cfg.gts, cfg.num_snap = 1, spec["num_snap"]
        init = dict(example=spec["example"], overrides=spec.get("overrides", {}))
    else:
        cfg = SPMConfig(**spec["cfg"])
        init = dict(spec["init"])
        parts = make_rigid_bodies(cfg, **init) if cfg.rigid else make_particles(cfg, **init)
    if "tweak" in spec:
        t = spec["tweak"]
        parts["x"][t["index"]] = t["x"]
        parts["v"][t["index"]] = t["v"]
    with tempfile.TemporaryDirectory() as td:
        keys = os.path.join(td, "run.keys")
        dump = os.path.join(td, "run.dump")
        write_udf_keys(keys, cfg, parts, out_dir=os.path.join(td, "avs"))
        err = ref_runner.run_reference(keys, dump_path=dump, fields_every=spec.get("fields_every", 1),
                                       body_force=cfg.body_force, timeout=4 * 3600.0)
        d = ref_runner.read_dump(dump)
    frames = d["frames"]
    out = {"config_json": np.array(json.dumps(dataclasses.asdict(cfg))),
           "init_json": np.array(json.dumps(init))}
    for k in ("x", "v", "omega"):
        out["init_" + k] = parts[k]
    out["init_q"] = parts["q"]
    for k in ("x", "x_nopbc", "v", "omega", "q", "f_hydro_previous", "torque_hydro_previous", "fr_previous"):
        out["traj_" + k] = np.stack([f[k] for f in frames])
    out["traj_uk_dc"] = np.stack([f["uk_dc"] for f in frames])
    out["traj_ts"] = np.array([f["ts"] for f in frames])
    out["traj_degree_oblique"] = np.array([f["degree_oblique"] for f in frames])
    if cfg.equation == EQ_LE:
        # Mean_shear_stress lines (sp_3d_ns.h:325-339): time, shear_rate,
        # degree_oblique, strain, lj, hydro_old, hydro_new, reynolds, fluid,
        # interfacial, apparent, viscosity
        rows = [[float(v) for v in l.split()] for l in err.splitlines()
                if l and not l.startswith("#") and len(l.split()) == 12]
        out["stress_lines"] = np.array(rows)
    by_ts = {int(f["ts"]): f for f in frames}
    fs = [s for s in spec["field_steps"] if s in by_ts]
    out["field_steps"] = np.array(fs)
    for s in fs:
        f = by_ts[s]
        if spec.get("zeta", True):
            out[f"zeta_retained_{s}"] = retained_modes(cfg, f["zeta"])
        if "u" not in f:
            out[f"phi_plane_{s}"] = f["phi"][:, :, 0].copy()
            continue
        u = f["u"]
        out[f"u_checksums_{s}"] = np.array([np.sum(u[c]) for c in range(3)] +
                                           [np.sum(u[c] ** 2) for c in range(3)] +
                                           [np.abs(u).max()])
        out[f"u_plane_{s}"] = u[:, :, :, 0].copy()       # z = 0 plane of every component
        out[f"phi_plane_{s}"] = f["phi"][:, :, 0].copy()
        out[f"phi_sum_{s}"] = np.array(f["phi"].sum())
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{path}: {os.path.getsize(path)} bytes, {len(frames)} frames")


def main():
    if not ref_runner.available():
        raise SystemExit("build the reference first: make -C oracle/ref_build")
    names = sys.argv[1:] or sorted(CASES)
    for n in names:
        make_case(n, CASES[n])


if __name__ == "__main__":
    main()
