"""Restart files of the reference program (resume.cxx), both ways, against
the reference program run here (oracle/_ref):

* reference -> GPU: the reference runs N1 + 1 steps and writes its restart
  file; the reference resumed from it and this library resumed from it
  (kapsel3_b200.spm.resume_run: set-up, the reference's discarded first
  step, spm_load_restart) agree on every following step within 1e-10;
* GPU -> reference: a GPU run writes the restart file (spm_save_restart)
  and the reference program resumes from it; a GPU run resumed from the same
  file follows the reference within 1e-10; without noise the uninterrupted
  GPU run does too.

Covered: Navier_Stokes with a body force, with the thermostat (the resumed
generator restarts from its seed and draws one discarded step, as the
reference's does), Lees-Edwards with a nonzero degree_oblique, Electrolyte
with salt and an AC field (the ion concentrations are part of the file), and
the reference's restart file rewritten as a UDF file."""
import dataclasses
import os

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun, resume_run
from kapsel3_b200.udf import EQ_EL, EQ_LE, SPMConfig, make_particles, read_udf_keys, write_udf_from_keys, write_udf_keys
from oracle import ref_runner
from tests.golden_util import retained

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_runner.available(), reason="reference program not built (oracle/_ref)")]
TOL = 1e-10
N1, N2 = 6, 8

CASES = {
    "ns_body_force": SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=3.5, a_xi=2.0, dt=0.05,
                               body_force=(1e-3, 0.0, -5e-4)),
    "ns_thermostat": SPMConfig(npx=5, npy=5, npz=5, n_particles=4, a=3.5, a_xi=2.0, dt=0.05, kbt=1e-4),
    "lees_edwards": SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=3.5, a_xi=2.0, dt=0.05, equation=EQ_LE,
                              shear_rate=0.05, kbt=1e-5),
    "electrolyte_salt_ac": SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=4.0, a_xi=2.0, dt=0.01, equation=EQ_EL,
                                     kbt=1.0, salt=True, valency=(1.0, -1.0), onsager=(1.0, 1.5), debye_length=5.0,
                                     surface_charge=-12.0, e_field="AC", e_ext=(0.1, 0.05, 0.0), e_frequency=4.0),
}


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0))


def _keys(tmp, name, cfg, parts):
    path = os.path.join(tmp, name)
    write_udf_keys(path, cfg, parts, out_dir=os.path.join(tmp, "avs"))
    return path


def _extend(src, dst, num_snap):
    """The restart key file with output.Num_snap raised, so that the resumed
    reference program runs on (its MSTEP = Num_snap * GTS)."""
    kv = read_udf_keys(src)
    kv["output.Num_snap"] = str(num_snap)
    with open(dst, "w") as f:
        f.writelines(f"{k} = {v}\n" for k, v in kv.items())
    return dst


def _follow(run, frames, what):
    """Steps `run` through the reference's frames (state after ts steps)
    and compares particles and the retained (2/3-rule) modes of zeta at each
    (the modes outside are truncated before they are read)."""
    assert frames and run.time()[0] == frames[0]["ts"], (run.time(), frames[0]["ts"])
    for f in frames:
        if run.time()[0] < f["ts"]:
            run.step(f["ts"] - run.time()[0])
        p = run.particles()
        errs = {k: rel(p[k], f[k]) for k in ("x", "v", "omega", "q", "f_hydro_previous")}
        if "zeta" in f:
            zeta, uk = run.zeta()
            errs["zeta"] = rel(retained(run.cfg, zeta), retained(run.cfg, f["zeta"]))
            # the mean velocity against the flow's velocity scale, within 1e-8: an Electrolyte run's
            # uk_dc is the small remainder of a charge-neutral force sum, whose order of summation
            # differs between the programs (uninterrupted runs differ by ~5e-10 of the scale too)
            scale = max(np.linalg.norm(f["uk_dc"]), float(np.abs(f["u"]).max()) if "u" in f else 0.0)
            uk_err = float(np.linalg.norm(uk - f["uk_dc"])) / (scale if scale > 0 else 1.0)
            assert uk_err < 1e-8, (what, f["ts"], "uk_dc", uk_err)
        for n in range(f["conc"].shape[0] if "conc" in f else 0):  # Electrolyte: the ion concentrations
            errs[f"conc{n}"] = rel(run.concentration(n), f["conc"][n])
        assert max(errs.values()) < TOL, (what, f["ts"], errs)
        assert abs(run.time()[1] - f["time"]) <= 1e-12 * abs(f["time"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_restart_resumes_on_gpu(gpu, name, tmp_path):
    cfg = dataclasses.replace(CASES[name], num_snap=N1)
    parts = make_particles(cfg, seed=19, v_sd=1e-3, random_orientation=True)
    tmp = str(tmp_path)
    res = os.path.join(tmp, "ref_restart.keys")
    ref_runner.run_reference(_keys(tmp, "run.keys", cfg, parts), body_force=cfg.body_force, restart_path=res)
    cont = _extend(res, os.path.join(tmp, "ref_continue.keys"), N1 + N2)
    dump = os.path.join(tmp, "resumed.dump")
    ref_runner.run_reference(cont, dump_path=dump, fields_every=1, body_force=cfg.body_force)
    frames = ref_runner.read_dump(dump)["frames"]
    assert [f["ts"] for f in frames] == list(range(N1 + 1, N1 + N2 + 1))
    with resume_run(cont, config=cfg) as run:
        if cfg.equation == EQ_LE:
            deg, _ = run.shear_state()
            assert deg == frames[0]["degree_oblique"] != 0.0
        _follow(run, frames, "restart key file of the reference")
    if name == "ns_body_force":  # the same file as a UDF file
        udf = os.path.join(tmp, "ref_continue.udf")
        write_udf_from_keys(udf, read_udf_keys(cont))
        with SPMRun(cfg) as run:
            run.initialize(parts)
            run.step(1)
            run.load_restart(udf)
            _follow(run, frames, "restart UDF file")


@pytest.mark.parametrize("name", ["ns_body_force", "ns_thermostat"])
def test_gpu_restart_resumes_in_reference(gpu, name, tmp_path):
    cfg = dataclasses.replace(CASES[name], num_snap=N1)
    parts = make_particles(cfg, seed=23, v_sd=1e-3, random_orientation=True)
    tmp = str(tmp_path)
    keys = _keys(tmp, "run.keys", cfg, parts)
    res = os.path.join(tmp, "gpu_restart.keys")
    with SPMRun(cfg) as run:
        run.initialize(parts)
        run.step(N1 + 1)  # what the reference's run of MSTEP = N1 takes
        run.save_restart(res, keys)
        later = None
        if cfg.kbt == 0.0:
            run.step(N2 - 1)
            later = run.particles()
    cont = _extend(res, os.path.join(tmp, "gpu_continue.keys"), N1 + N2)
    dump = os.path.join(tmp, "resumed.dump")
    ref_runner.run_reference(cont, dump_path=dump, fields_every=1, body_force=cfg.body_force)
    frames = ref_runner.read_dump(dump)["frames"]
    assert [f["ts"] for f in frames] == list(range(N1 + 1, N1 + N2 + 1))
    with resume_run(cont, config=cfg) as run:
        _follow(run, frames, "restart key file of this library")
    if later is not None:  # no noise: the uninterrupted run is the resumed one
        for k in ("x", "v", "omega", "q"):
            assert rel(later[k], frames[-1][k]) < TOL, k


def test_restart_refuses_another_grid(gpu, tmp_path):
    cfg = dataclasses.replace(CASES["ns_body_force"], num_snap=2)
    parts = make_particles(cfg, seed=5)
    tmp = str(tmp_path)
    res = os.path.join(tmp, "r.keys")
    with SPMRun(cfg) as run:
        run.initialize(parts)
        run.step(3)
        run.save_restart(res)
    other = dataclasses.replace(cfg, npz=6)
    with SPMRun(other) as run:
        run.initialize(parts)
        with pytest.raises(N.SpmError, match="not the context's grid"):
            run.load_restart(res)


@pytest.mark.parametrize("fixture", ["rigid_32_free_gravity", "rigid_species_dof_thermostat"])
def test_rigid_restart_both_ways(gpu, fixture, tmp_path):
    """Rigid bodies in the restart file (Particles[] hold the bodies, then
    GR_body, GR_masses and GR_moments_body; resume.cxx:253-379, 925-1100):
    the reference's file resumes on the GPU, and this library's file resumes
    in the reference program; both resumed runs follow the reference's own
    resumed run within 1e-10 (bodies under gravity; two species with
    switched-off degrees of freedom and the thermostat)."""
    from tests.golden_util import load

    cfg, parts, _ = load(fixture)
    cfg = dataclasses.replace(cfg, num_snap=N1, gts=1)
    tmp = str(tmp_path)
    keys = _keys(tmp, "run.keys", cfg, parts)
    # reference -> GPU
    res = os.path.join(tmp, "ref_restart.keys")
    ref_runner.run_reference(keys, restart_path=res)
    cont = _extend(res, os.path.join(tmp, "ref_continue.keys"), N1 + N2)
    dump = os.path.join(tmp, "resumed.dump")
    ref_runner.run_reference(cont, dump_path=dump, fields_every=1)
    frames = ref_runner.read_dump(dump)["frames"]
    assert [f["ts"] for f in frames] == list(range(N1 + 1, N1 + N2 + 1))
    with resume_run(cont, config=cfg) as run:
        _follow(run, frames, "rigid restart file of the reference")
    # GPU -> reference
    mine = os.path.join(tmp, "gpu_restart.keys")
    with SPMRun(cfg) as run:
        run.initialize(parts)
        run.step(N1 + 1)
        run.save_restart(mine, keys)
    cont2 = _extend(mine, os.path.join(tmp, "gpu_continue.keys"), N1 + N2)
    dump2 = os.path.join(tmp, "resumed2.dump")
    ref_runner.run_reference(cont2, dump_path=dump2, fields_every=1)
    frames2 = ref_runner.read_dump(dump2)["frames"]
    assert [f["ts"] for f in frames2] == list(range(N1 + 1, N1 + N2 + 1))
    with resume_run(cont2, config=cfg) as run:
        _follow(run, frames2, "rigid restart file of this library")
