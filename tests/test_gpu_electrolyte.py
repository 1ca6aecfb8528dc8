"""Electrolyte runs (charged colloids with mobile ions; NSsolute_solver_Euler
and the Electrolyte branch of Time_evolution_hydro) against the reference
program built from its sources (oracle/_ref/kapsel_ref), on the same seeded
inputs: particle state, zeta, the real-space velocity and the k-space ion
concentrations after every step, FP64, within 1e-10 relative.

Cases: counterions only (saltfree) under a DC field, a salt solution
(positive and negative ions) without a field, and a salt solution under an
AC field along x and y."""
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


@pytest.mark.skipif(not ref_runner.available(), reason="oracle/_ref is not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_electrolyte_matches_the_reference_program(gpu, name, tmp_path):
    cfg = CASES[name]
    parts = make_particles(cfg, seed=7, v_sd=1e-3, random_orientation=True)
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


def test_electrolyte_parameter_checks(gpu):
    base = dict(npx=5, npy=5, npz=5, n_particles=2, a=4.0, equation=EQ_EL, kbt=1.0, surface_charge=-10.0,
                valency=(1.0, 0.0))
    for bad, msg in ((dict(surface_charge=0.0), "Surface_charge"), (dict(valency=(-1.0, 0.0)), "opposite sign"),
                     (dict(init_pb=True), "Poisson_Boltzmann"), (dict(salt=True, valency=(1.0, 1.0)), "salt")):
        with pytest.raises(N.SpmError, match=msg):
            SPMRun(SPMConfig(**{**base, **bad}), precision=N.SPM_PREC_FP64)
    with pytest.raises(N.SpmError, match="FP64"):
        SPMRun(SPMConfig(**base), precision=N.SPM_PREC_FP32_MIXED)
