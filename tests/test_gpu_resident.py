"""The reference program with its time evolution resident on the GPU.

oracle/_ref/kapsel_gpu_resident is the unmodified reference program (its
objects built from the reference's sources) linked with
kapsel3_b200/shim/kapsel_b200_resident.cxx: after the program's own
initialisation the Time_evolution pointer of its main loop
(sp_3d_ns.cxx:10, 954) runs spm_step on device-resident state, and host
copies are refreshed only before output frames and the restart file.  Its FP64
trajectory must match the pure reference program's (the golden fixtures)
within 1e-10: positions, velocities, angular velocities, orientations,
f_hydro_previous and uk_dc at every frame, and for Lees-Edwards also
degree_oblique."""
import os
import tempfile

import numpy as np
import pytest

from kapsel3_b200.udf import write_udf_keys
from oracle import ref_runner
from tests.golden_util import load, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.mark.parametrize("name", ["c1_32_two_spheres_body_force", "thermostat_32_four_spheres",
                                  "le_32_boundary_crossing", "rigid_32_free_gravity", "rigid_32_fixed_motion",
                                  "rigid_species_dof_thermostat"])
def test_resident_reference_program_matches_reference(gpu, name):
    if not ref_runner.available(gpu_resident=True):
        pytest.skip("oracle/_ref/kapsel_gpu_resident is not built (make -C oracle/ref_build gpu)")
    cfg, parts, z = load(name)
    with tempfile.TemporaryDirectory() as td:
        keys = os.path.join(td, "run.keys")
        dump = os.path.join(td, "run.dump")
        write_udf_keys(keys, cfg, parts, out_dir=os.path.join(td, "avs"))
        err = ref_runner.run_reference(keys, dump_path=dump, fields_every=0, body_force=cfg.body_force,
                                       gpu_resident=True, threads=4, timeout=600.0)
        frames = ref_runner.read_dump(dump)["frames"]
    assert "resident on the GPU" in err
    assert len(frames) == len(z["traj_ts"])
    for i, f in enumerate(frames):
        for k in ("x", "v", "omega", "q", "f_hydro_previous"):
            e = rel(f[k], z["traj_" + k][i])
            assert e <= TOL, (name, i, k, e)
        assert rel(f["uk_dc"], z["traj_uk_dc"][i]) <= TOL or np.abs(f["uk_dc"]).max() < 1e-300
        if "traj_degree_oblique" in z.files:
            assert abs(f["degree_oblique"] - z["traj_degree_oblique"][i]) <= TOL * max(1.0, abs(
                z["traj_degree_oblique"][i]))


def _frames(keys, tmp, name, fields_every=0, **kw):
    dump = os.path.join(tmp, name + ".dump")
    err = ref_runner.run_reference(keys, dump_path=dump, fields_every=fields_every, timeout=600.0, **kw)
    return err, ref_runner.read_dump(dump)["frames"]


def _same(fa, fb, what):
    assert [f["ts"] for f in fa] == [f["ts"] for f in fb], what
    for a, b in zip(fa, fb):
        for k in ("x", "v", "omega", "q", "f_hydro_previous"):
            e = rel(a[k], b[k])
            assert e <= TOL, (what, a["ts"], k, e)


def _live_cases():
    from kapsel3_b200.udf import EQ_SNS, SPMConfig
    from tests.test_gpu_janus import CASES as JANUS
    return {
        "shear_ns_dc_thermostat": SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=4.0, a_xi=2.0, dt=0.05,
                                            equation=EQ_SNS, shear_rate=0.02, kbt=1e-4, gts=2, num_snap=5),
        "two_species_thermostat": SPMConfig(npx=5, npy=5, npz=5, n_particles=5, a=3.5, a_xi=2.0, dt=0.05, kbt=1e-4,
                                            species=((3, 1.0, 0.0), (2, 2.5, 0.0)), gts=2, num_snap=5),
        "tumblers": JANUS["tumblers"],
        "squirmers": JANUS["squirmer_example"],
    }


@pytest.mark.parametrize("name", ["shear_ns_dc_thermostat", "two_species_thermostat", "tumblers", "squirmers"])
def test_resident_loop_serves_more_runs(gpu, name, tmp_path):
    """Shear_Navier_Stokes, several species and Janus particles through the
    resident loop: the same frames as the reference program run alone."""
    if not ref_runner.available(gpu_resident=True):
        pytest.skip("oracle/_ref/kapsel_gpu_resident is not built")
    from kapsel3_b200.udf import make_particles
    cfg = _live_cases()[name]
    parts = make_particles(cfg, seed=37, v_sd=1e-3, random_orientation=True)
    keys = os.path.join(str(tmp_path), "run.keys")
    write_udf_keys(keys, cfg, parts, out_dir=os.path.join(str(tmp_path), "avs"))
    _, ref = _frames(keys, str(tmp_path), "ref")
    err, res = _frames(keys, str(tmp_path), "res", gpu_resident=True, threads=4)
    assert "resident on the GPU" in err
    _same(res, ref, name)


def test_resident_loop_resumes_from_a_restart_file(gpu, tmp_path):
    """A resumed run (resume.Calculation = CONTINUE): the reference's first
    pass steps the input state, restores the saved one, and the resident loop
    takes the restored state over; the frames equal the reference program's
    own resumed run, thermostat included."""
    if not ref_runner.available(gpu_resident=True):
        pytest.skip("oracle/_ref/kapsel_gpu_resident is not built")
    from kapsel3_b200.udf import SPMConfig, make_particles, read_udf_keys
    cfg = SPMConfig(npx=5, npy=5, npz=5, n_particles=4, a=3.5, a_xi=2.0, dt=0.05, kbt=1e-4, gts=1, num_snap=5)
    parts = make_particles(cfg, seed=43, v_sd=1e-3, random_orientation=True)
    tmp = str(tmp_path)
    keys = os.path.join(tmp, "run.keys")
    write_udf_keys(keys, cfg, parts, out_dir=os.path.join(tmp, "avs"))
    res = os.path.join(tmp, "restart.keys")
    ref_runner.run_reference(keys, restart_path=res, timeout=600.0)
    kv = read_udf_keys(res)
    kv["output.Num_snap"] = "12"
    cont = os.path.join(tmp, "continue.keys")
    with open(cont, "w") as f:
        f.writelines(f"{k} = {v}\n" for k, v in kv.items())
    _, ref = _frames(cont, tmp, "ref")
    err, out = _frames(cont, tmp, "res", gpu_resident=True, threads=4)
    assert "resident on the GPU" in err and ref and ref[0]["ts"] == 6
    _same(out, ref, "resumed")


@pytest.mark.parametrize("name", ["salt_ac", "saltfree_dc"])
def test_resident_loop_serves_electrolyte_runs(gpu, name, tmp_path):
    """Electrolyte runs through the resident loop: the reference initialises
    the ions (salt with an AC field; counterions under a DC field), hands
    them over with Total_solute
    (spm_set_solute) and gets them back at every frame; the frames' particles,
    retained zeta and k-space concentrations equal the reference program's own
    run within 1e-10."""
    if not ref_runner.available(gpu_resident=True):
        pytest.skip("oracle/_ref/kapsel_gpu_resident is not built")
    import dataclasses

    from kapsel3_b200.udf import make_particles
    from tests.golden_util import retained
    from tests.test_gpu_electrolyte import CASES as EL

    cfg = dataclasses.replace(EL[name], gts=2, num_snap=4)
    parts = make_particles(cfg, seed=47, v_sd=1e-3, random_orientation=True)
    keys = os.path.join(str(tmp_path), "run.keys")
    write_udf_keys(keys, cfg, parts, out_dir=os.path.join(str(tmp_path), "avs"))
    _, ref = _frames(keys, str(tmp_path), "ref", fields_every=1)
    err, res = _frames(keys, str(tmp_path), "res", fields_every=1, gpu_resident=True, threads=4)
    assert "resident on the GPU" in err
    _same(res, ref, name)
    for a, b in zip(res, ref):
        assert rel(retained(cfg, a["zeta"]), retained(cfg, b["zeta"])) <= TOL, (name, a["ts"], "zeta")
        assert a["conc"].shape == b["conc"].shape
        for n in range(b["conc"].shape[0]):
            assert rel(a["conc"][n], b["conc"][n]) <= TOL, (name, a["ts"], "conc", n)


def test_resident_loop_applies_gravity_to_heavy_spheres(gpu, tmp_path):
    """Spheres heavier than the fluid under gravity (gravity.G, G_direction,
    MASS_RATIO 2): the resident loop maps Add_f_gravity's force on each
    sphere (md_force.cxx:306-315) and its frames equal the reference
    program's own."""
    if not ref_runner.available(gpu_resident=True):
        pytest.skip("oracle/_ref/kapsel_gpu_resident is not built")
    from kapsel3_b200.udf import SPMConfig, make_particles, read_udf_keys
    cfg = SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=3.5, a_xi=2.0, dt=0.05, mass_ratio=2.0, gts=2, num_snap=4)
    parts = make_particles(cfg, seed=53, v_sd=1e-3, random_orientation=True)
    keys = os.path.join(str(tmp_path), "run.keys")
    write_udf_keys(keys, cfg, parts, out_dir=os.path.join(str(tmp_path), "avs"))
    kv = read_udf_keys(keys)
    kv["gravity.G"], kv["gravity.G_direction"] = "0.002", "-Y"
    with open(keys, "w") as f:
        f.writelines(f"{k} = {v}\n" for k, v in kv.items())
    _, ref = _frames(keys, str(tmp_path), "ref")
    err, res = _frames(keys, str(tmp_path), "res", gpu_resident=True, threads=4)
    assert "resident on the GPU" in err
    _same(res, ref, "gravity")
    assert abs(ref[-1]["v"][:, 1]).max() > 1e-4  # the spheres sink along -y
