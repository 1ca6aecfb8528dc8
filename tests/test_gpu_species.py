"""Several particle species (Particle_spec[0..], Component_Number > 1)
against the reference program built from its sources (oracle/_ref/
kapsel_ref): particle state, zeta, u and, for Electrolyte runs, the ion
concentrations after every step, FP64, within 1e-10 relative.

Cases: two species of different MASS_RATIO with the thermostat on (IMASS,
IMOI and the noise of each species, p[n].spec in record order), colloids of
opposite charge in a salt solution (Surface_charge_e[p.spec] on the surface
charge field, counterions of each sign), and counterions around two
species of the same sign."""
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


EL = dict(a=4.0, a_xi=2.0, dt=0.01, equation=EQ_EL, kbt=1.0, gts=1, num_snap=6)
CASES = {
    "ns_two_species_thermostat": SPMConfig(npx=5, npy=5, npz=5, n_particles=4, a=4.0, a_xi=2.0, dt=0.05, kbt=1e-4,
                                           species=((2, 1.0, 0.0), (2, 3.0, 0.0)), gts=1, num_snap=8),
    "el_opposite_charges_salt": SPMConfig(npx=5, npy=5, npz=5, n_particles=4, salt=True, valency=(1.0, -1.0),
                                          onsager=(1.0, 1.0), debye_length=5.0, surface_charge=12.0,
                                          species=((2, 1.0, 12.0), (2, 1.5, -8.0)), **EL),
    "el_counterions_two_species": SPMConfig(npx=5, npy=5, npz=5, n_particles=3, valency=(1.0, 0.0),
                                            onsager=(1.0, 1.0), surface_charge=-10.0,
                                            species=((1, 1.0, -10.0), (2, 2.0, -4.0)), e_field="DC",
                                            e_ext=(0.05, 0.0, 0.0), **EL),
}


@pytest.mark.skipif(not ref_runner.available(), reason="oracle/_ref is not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_species_match_the_reference_program(gpu, name, tmp_path):
    cfg = CASES[name]
    parts = make_particles(cfg, seed=17, v_sd=1e-3, random_orientation=True)
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
            for n in range(fr["conc"].shape[0] if "conc" in fr else 0):
                c = run.concentration(n)
                assert rel(c, fr["conc"][n]) <= TOL, (name, fr["ts"], "conc", n, rel(c, fr["conc"][n]))
