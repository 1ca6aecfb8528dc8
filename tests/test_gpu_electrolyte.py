"""Electrolyte runs (charged colloids with mobile ions; NSsolute_solver_Euler
and the Electrolyte branch of Time_evolution_hydro) against the reference
program built from its sources (oracle/_ref/kapsel_ref), on the same seeded
inputs: particle state, zeta, the real-space velocity and the k-space ion
concentrations after every step, FP64, within 1e-10 relative.

Cases: counterions only (saltfree) under a DC field, a salt solution
(positive and negative ions) without a field, a salt solution under an AC
field along x and y, two colloids inside the Lennard-Jones range (the
Force() call of the velocity update), and the Poisson-Boltzmann initial
profiles of Init_rho_ion: counterions alone (with and without a field, the
latter followed by the steady-state relaxation), salt around one colloid
(the potential iteration) and salt around two colloids under a field
(uniform start and steady state).  The initial ion fields are compared
from step 0.  The legacy AVS files of an
Electrolyte run (Output_charge_field_data) match the reference's own."""
import os

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from kapsel3_b200.udf import EQ_EL, SPMConfig, make_particles, write_udf_keys
from oracle import ref_runner

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


CASES = {
    "saltfree_dc": SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.01, equation=EQ_EL, kbt=1.0,
                             dielectric=1.0, salt=False, valency=(1.0, 0.0), onsager=(1.0, 1.0), surface_charge=-10.0,
                             e_field="DC", e_ext=(0.1, 0.0, 0.0), gts=1, num_snap=8),
    "salt_nofield": SPMConfig(npx=5, npy=5, npz=4, n_particles=3, a=3.0, a_xi=2.0, dt=0.01, equation=EQ_EL, kbt=1.0,
                              dielectric=2.0, salt=True, valency=(1.0, -1.0), onsager=(1.5, 1.0), debye_length=4.0,
                              surface_charge=20.0, gts=1, num_snap=8),
    "salt_ac": SPMConfig(npx=5, npy=4, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.01, equation=EQ_EL, kbt=1.0,
                         dielectric=1.0, salt=True, valency=(2.0, -1.0), onsager=(1.0, 2.0), debye_length=6.0,
                         surface_charge=-15.0, e_field="AC", e_ext=(0.2, -0.1, 0.0), e_frequency=5.0, gts=1,
                         num_snap=8),
}


CASES["salt_lj_contact"] = SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.01, equation=EQ_EL,
                                     kbt=1.0, salt=True, valency=(1.0, -1.0), onsager=(1.0, 1.0),
                                     debye_length=5.0, surface_charge=10.0, gts=1, num_snap=8)

# obstacles (fixed particles, out of the LJ pairs: obstacle_chain,
# interaction.h:29-35) in contact, in a DC field
CASES["salt_dc_obstacles"] = SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.01,
                                       equation=EQ_EL, kbt=1.0, salt=True, valency=(1.0, -1.0), onsager=(1.0, 1.0),
                                       debye_length=5.0, surface_charge=10.0, janus_propulsion="OBSTACLE",
                                       e_field="DC", e_ext=(0.1, 0.0, 0.0), gts=1, num_snap=8)


PB = dict(npx=5, npy=5, npz=5, a=4.0, a_xi=2.0, dt=0.01, equation=EQ_EL, kbt=1.0, init_pb=True, gts=1, num_snap=4)
CASES["pb_counterions"] = SPMConfig(n_particles=1, dielectric=1.0, valency=(1.0, 0.0), onsager=(1.0, 1.0),
                                    surface_charge=-10.0, **PB)
CASES["pb_counterions_dc"] = SPMConfig(n_particles=2, dielectric=2.0, valency=(2.0, 0.0), onsager=(1.0, 1.0),
                                       surface_charge=-12.0, e_field="DC", e_ext=(0.05, 0.0, 0.0), **PB)
CASES["pb_salt_one"] = SPMConfig(n_particles=1, dielectric=1.0, salt=True, valency=(1.0, -1.0), onsager=(1.0, 1.0),
                                 debye_length=4.0, surface_charge=-15.0, **PB)
CASES["pb_salt_two_dc"] = SPMConfig(n_particles=2, dielectric=1.0, salt=True, valency=(1.0, -1.0),
                                    onsager=(1.0, 1.5), debye_length=5.0, surface_charge=10.0, e_field="DC",
                                    e_ext=(0.0, 0.05, 0.0), **PB)


def _particles(name, cfg):
    parts = make_particles(cfg, seed=7, v_sd=1e-3, random_orientation=True)
    if name in ("salt_lj_contact", "salt_dc_obstacles"):
        # centres 8.6 apart: inside the cut-off 2^(1/6) SIGMA = 8.98 (SIGMA = 2 A DX)
        parts["x"][0] = (12.0, 16.0, 15.5)
        parts["x"][1] = (20.6, 16.0, 15.5)
    return parts


@pytest.mark.skipif(not ref_runner.available(), reason="oracle/_ref is not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_electrolyte_matches_the_reference_program(gpu, name, tmp_path):
    cfg = CASES[name]
    parts = _particles(name, cfg)
    keys, dump = str(tmp_path / "in.keys"), str(tmp_path / "d.bin")
    write_udf_keys(keys, cfg, parts, out_dir=str(tmp_path / "avs"))
    ref_runner.run_reference(keys, dump, fields_every=1, timeout=600)
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
            for n in range(fr["conc"].shape[0]):
                c = run.concentration(n)
                assert rel(c, fr["conc"][n]) <= TOL, (name, fr["ts"], "conc", n, rel(c, fr["conc"][n]))
    if cfg.janus_propulsion == "OBSTACLE":
        assert not p["v"].any() and np.array_equal(p["x"], parts["x"])


def test_electrolyte_parameter_checks(gpu):
    base = dict(npx=5, npy=5, npz=5, n_particles=2, a=4.0, equation=EQ_EL, kbt=1.0, surface_charge=-10.0,
                valency=(1.0, 0.0))
    for bad, msg in ((dict(surface_charge=0.0), "Surface_charge"), (dict(valency=(-1.0, 0.0)), "opposite sign"),
                     (dict(init_pb=True, salt=True, valency=(2.0, -1.0), n_particles=1, debye_length=5.0),
                      "Poisson_Boltzmann"), (dict(salt=True, valency=(1.0, 1.0)), "salt")):
        with pytest.raises(N.SpmError, match=msg):
            SPMRun(SPMConfig(**{**base, **bad}), precision=N.SPM_PREC_FP64)


@pytest.mark.parametrize("name", ["salt_ac", "pb_counterions_dc"])
def test_electrolyte_fp32_mixed_close_to_fp64(gpu, name):
    """FP32 fields and transforms (plain FP32 zeta and concentrations) with
    FP64 particle work and sums: velocities, the flow and the ion
    concentrations within 1e-5 of the FP64 run after a few dozen steps."""
    cfg = CASES[name]
    parts = make_particles(cfg, seed=41, v_sd=1e-3, random_orientation=True)
    out = {}
    for prec in (N.SPM_PREC_FP64, N.SPM_PREC_FP32_MIXED):
        with SPMRun(cfg, precision=prec) as run:
            run.initialize(parts)
            run.step(30)
            out[prec] = (run.particles()["v"], run.velocity(), [run.concentration(n) for n in range(2 if cfg.salt else 1)])
    v32, u32, c32 = out[N.SPM_PREC_FP32_MIXED]
    v64, u64, c64 = out[N.SPM_PREC_FP64]
    assert rel(v32, v64) <= 1e-5 and rel(u32, u64) <= 1e-5, (rel(v32, v64), rel(u32, u64))
    for a, b in zip(c32, c64):
        assert rel(a, b) <= 1e-5, rel(a, b)


AVS_REF = os.path.join(ref_runner.REF_DIR, "kapsel_ref_avs")


@pytest.mark.skipif(not os.access(AVS_REF, os.X_OK), reason="oracle/_ref/kapsel_ref_avs is not built")
def test_electrolyte_avs_files_match_the_reference_program(gpu, tmp_path):
    """Headers byte for byte; the seven float fields (u, phi, surface charge
    4 pi RADIUS^2, ion charge density, Coulomb potential) and the particle
    files to FP32 rounding."""
    cfg = SPMConfig(npx=5, npy=4, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.01, equation=EQ_EL, kbt=1.0,
                    salt=True, valency=(2.0, -1.0), onsager=(1.0, 2.0), debye_length=6.0, surface_charge=-15.0,
                    e_field="DC", e_ext=(0.1, 0.0, 0.05), gts=2, num_snap=2)
    parts = make_particles(cfg, seed=5, v_sd=1e-3, random_orientation=True)
    keys = str(tmp_path / "in.keys")
    write_udf_keys(keys, cfg, parts, out_dir=str(tmp_path / "ref"))
    ref_runner.run_reference_avs(keys)
    with SPMRun(cfg, precision=N.SPM_PREC_FP64) as run:
        run.initialize(parts)
        run.avs_open(str(tmp_path / "gpu"), "frame", cfg.num_snap)
        for ts in range(cfg.mstep + 1):
            if ts % cfg.gts == 0:
                run.avs_frame()
            run.step(1)
        run.avs_close()
    ref, ours = tmp_path / "ref", tmp_path / "gpu"
    for name in ("frame.fld", "framep.fld", "frame.cod"):
        assert (ours / name).read_bytes() == (ref / name).read_bytes(), name
    nx, ny, nz = cfg.shape
    for ts in range(0, cfg.mstep + 1, cfg.gts):
        a = np.fromfile(ours / "avs" / f"frame_{ts}.dat", dtype=np.float32).reshape(7, nz, ny, nx)
        b = np.fromfile(ref / "avs" / f"frame_{ts}.dat", dtype=np.float32).reshape(7, nz, ny, nx)
        for f in range(7):
            scale = max(float(np.abs(b[f]).max()), 1e-30)
            assert float(np.abs(a[f] - b[f]).max()) <= 2e-6 * scale, (ts, f)
        for ext in ("cod", "dat"):
            pa = np.fromfile(ours / "avs" / f"framep_{ts}.{ext}", dtype=np.float32)
            pb = np.fromfile(ref / "avs" / f"framep_{ts}.{ext}", dtype=np.float32)
            np.testing.assert_allclose(pa, pb, rtol=2e-6, atol=1e-6)
