"""Shear_Navier_Stokes (a periodic box whose mean shear is sustained on fluid
planes, NS_solver_slavedEuler_Shear_PBC, fluid_solver.cxx:377-409) against
the reference program built from its sources: particle state, zeta and u
after every step, FP64 within 1e-10 relative; the FP32-mixed form within
1e-5 of FP64.  Cases: DC steady shear (u_x fixed on the planes y = LY/4,
3LY/4) and AC oscillatory shear (the zigzag profile times cos(omega t))."""
import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from kapsel3_b200.udf import EQ_SNS, SPMConfig, make_particles, write_udf_keys
from oracle import ref_runner

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


CASES = {
    "dc": SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=4.0, a_xi=2.0, dt=0.05, equation=EQ_SNS, shear_rate=0.02,
                    kbt=1e-4, gts=1, num_snap=8),
    # heavier particles: the density field of Calc_shear_stress / the inertia
    # stress is no longer uniform
    "ac_heavy": SPMConfig(npx=5, npy=5, npz=4, n_particles=3, a=3.5, a_xi=2.0, dt=0.05, equation=EQ_SNS,
                          shear_rate=0.05, shear_ac=True, shear_frequency=0.3, mass_ratio=2.0, gts=1, num_snap=6),
    "dc_heavy": SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=4.0, a_xi=2.0, dt=0.05, equation=EQ_SNS,
                          shear_rate=0.02, mass_ratio=2.5, gts=1, num_snap=6),
    "ac": SPMConfig(npx=5, npy=5, npz=4, n_particles=2, a=3.5, a_xi=2.0, dt=0.05, equation=EQ_SNS, shear_rate=0.05,
                    shear_ac=True, shear_frequency=0.3, gts=1, num_snap=8),
}


@pytest.mark.skipif(not ref_runner.available(), reason="oracle/_ref is not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_shear_ns_matches_the_reference_program(gpu, name, tmp_path):
    cfg = CASES[name]
    parts = make_particles(cfg, seed=23, v_sd=1e-3, random_orientation=True)
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


def test_shear_ns_fp32_mixed_close_to_fp64(gpu):
    cfg = CASES["dc"]
    parts = make_particles(cfg, seed=23, v_sd=1e-3, random_orientation=True)
    out = {}
    for prec in (N.SPM_PREC_FP64, N.SPM_PREC_FP32_MIXED):
        with SPMRun(cfg, precision=prec) as run:
            run.initialize(parts)
            run.step(10)
            out[prec] = run.particles()["v"], run.velocity()
    assert rel(out[N.SPM_PREC_FP32_MIXED][0], out[N.SPM_PREC_FP64][0]) <= 1e-5
    assert rel(out[N.SPM_PREC_FP32_MIXED][1], out[N.SPM_PREC_FP64][1]) <= 1e-5


@pytest.mark.skipif(not ref_runner.available(), reason="oracle/_ref is not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_shear_ns_stress_line_matches_the_reference_program(gpu, name, tmp_path):
    """The shear-stress line the reference prints after every step
    (Update_strain, sp_3d_ns.h:205-214; Mean_shear_stress, :319-340):
    DC time, shear rate, strain, shear stress, viscosity; AC time, shear
    rate, strain, shear stress, inertia stress, their sum.  The reference
    prints 8 significant digits."""
    cfg = CASES[name]
    parts = make_particles(cfg, seed=29, v_sd=1e-3, random_orientation=True)
    keys = str(tmp_path / "in.keys")
    write_udf_keys(keys, cfg, parts, out_dir=str(tmp_path / "avs"))
    err = ref_runner.run_reference(keys, timeout=600)
    width = 6 if cfg.shear_ac else 5
    rows = []
    for line in err.splitlines():
        f = line.split()
        if len(f) == width and not line.startswith("#"):
            try:
                rows.append([float(v) for v in f])
            except ValueError:
                pass
    assert len(rows) == cfg.mstep + 1
    with SPMRun(cfg, precision=N.SPM_PREC_FP64) as run:
        run.initialize(parts)
        for ref in rows:
            run.step(1)
            deg, st = run.shear_state()
            ours = [run.time()[1], st[0], st[1], st[2]] + ([st[4], st[5]] if cfg.shear_ac else [st[3]])
            assert deg == 0.0
            for i, (a, b) in enumerate(zip(ours, ref)):
                assert abs(a - b) <= 6e-8 * abs(b) + 1e-14, (name, run.time()[0], i, a, b)
