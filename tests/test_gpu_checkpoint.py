"""Checkpoint / restart of device state (spm_save_state / spm_load_state).

A run saved after n1 steps and restored into a fresh context continues like
the original: after n2 more steps the particle state and zeta agree within
1e-12 relative (the shared-profile scatters use float atomics, whose order
may differ where three or more profiles overlap a cell).  Covered: FP64
Navier_Stokes with the thermostat (MT19937 state), FP32-mixed (compensated
zeta words), Lees-Edwards (degree_oblique and its device scalars) and
Electrolyte (ion concentrations and Total_solute; AC field in time).  A
checkpoint is refused by a context with other parameters (a Shear_Navier_Stokes
state by a run with another sustained profile), and a truncated file is
refused."""
import os

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from kapsel3_b200.udf import EQ_EL, EQ_LE, EQ_SNS, SPMConfig, make_particles

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


CASES = {
    "ns_fp64_thermostat": (SPMConfig(npx=5, npy=5, npz=5, n_particles=4, a=4.0, a_xi=2.0, dt=0.05, kbt=1e-4),
                           N.SPM_PREC_FP64),
    "ns_fp32_mixed": (SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=4.0, a_xi=2.0, dt=0.05,
                                body_force=(1e-3, 0.0, 0.0)), N.SPM_PREC_FP32_MIXED),
    "lees_edwards_fp64": (SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=3.5, a_xi=2.0, dt=0.05, equation=EQ_LE,
                                    shear_rate=0.3, kbt=1e-5), N.SPM_PREC_FP64),
    "electrolyte_salt_ac": (SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=4.0, a_xi=2.0, dt=0.01, equation=EQ_EL,
                                      kbt=1.0, salt=True, valency=(1.0, -1.0), onsager=(1.0, 1.5), debye_length=5.0,
                                      surface_charge=-12.0, e_field="AC", e_ext=(0.1, 0.05, 0.0), e_frequency=4.0),
                            N.SPM_PREC_FP64),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_restored_run_continues_like_the_original(gpu, name, tmp_path):
    cfg, prec = CASES[name]
    parts = make_particles(cfg, seed=31, v_sd=1e-3, random_orientation=True)
    path = os.path.join(tmp_path, "run.ck")
    with SPMRun(cfg, precision=prec) as a:
        a.initialize(parts)
        a.step(7)
        a.save_state(path)
        a.step(6)
        pa, (za, dca), ta = a.particles(), a.zeta(), a.time()
        sa = a.shear_state() if cfg.equation == EQ_LE else None
        ca = [a.concentration(n) for n in range(2)] if cfg.equation == EQ_EL else []
    with SPMRun(cfg, precision=prec) as b:
        b.load_state(path)
        assert b.time()[0] == 7
        b.step(6)
        pb, (zb, dcb), tb = b.particles(), b.zeta(), b.time()
        sb = b.shear_state() if cfg.equation == EQ_LE else None
        cb = [b.concentration(n) for n in range(2)] if cfg.equation == EQ_EL else []
    assert ta == tb
    for k in ("x", "v", "omega", "q", "f_hydro_previous"):
        assert rel(pb[k], pa[k]) <= TOL, (name, k)
    assert rel(zb, za) <= TOL and rel(dcb, dca) <= TOL
    for n, (x, y) in enumerate(zip(ca, cb)):
        assert rel(y, x) <= TOL, (name, "conc", n)
    if sa is not None:
        assert sb[0] == sa[0]
        assert rel(sb[1], sa[1]) <= TOL


def test_checkpoint_is_refused_by_another_run(gpu, tmp_path):
    cfg, prec = CASES["ns_fp64_thermostat"]
    parts = make_particles(cfg, seed=3)
    path = os.path.join(tmp_path, "run.ck")
    with SPMRun(cfg, precision=prec) as a:
        a.initialize(parts)
        a.step(2)
        a.save_state(path)
    other = SPMConfig(npx=5, npy=5, npz=5, n_particles=4, a=4.0, a_xi=2.0, dt=0.04, kbt=1e-4)
    with SPMRun(other, precision=prec) as b:
        with pytest.raises(N.SpmError):
            b.load_state(path)
    with SPMRun(cfg, precision=N.SPM_PREC_FP32_MIXED) as b:
        with pytest.raises(N.SpmError):
            b.load_state(path)
    data = open(path, "rb").read()
    short = os.path.join(tmp_path, "short.ck")
    open(short, "wb").write(data[: len(data) // 2])
    with SPMRun(cfg, precision=prec) as b:
        with pytest.raises(N.SpmError, match="truncated"):
            b.load_state(short)


def test_shear_checkpoint_keeps_its_profile(gpu, tmp_path):
    """A Shear_Navier_Stokes state restores only into a run with the same
    sustained profile: an AC state is refused by a DC run and by an AC run of
    another frequency."""
    ac = SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.05, equation=EQ_SNS, shear_rate=0.01,
                   shear_ac=True, shear_frequency=0.2)
    parts = make_particles(ac, seed=5)
    path = os.path.join(tmp_path, "ac.ck")
    with SPMRun(ac) as a:
        a.initialize(parts)
        a.step(2)
        a.save_state(path)
    with SPMRun(ac) as b:
        b.load_state(path)
    for other in (SPMConfig(**{**ac.__dict__, "shear_ac": False, "shear_frequency": 0.0}),
                  SPMConfig(**{**ac.__dict__, "shear_frequency": 0.3})):
        with SPMRun(other) as b:
            with pytest.raises(N.SpmError):
                b.load_state(path)
