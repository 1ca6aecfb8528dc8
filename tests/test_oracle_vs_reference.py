"""Live pin of the oracle against the reference program built from its
sources (oracle/_ref).  Skipped where the reference build is absent (the GPU
box); tests/test_golden_oracle.py covers that case with fixtures."""
import os
import tempfile

import numpy as np
import pytest

from kapsel3_b200.udf import SPMConfig, make_particles, write_udf_keys
from oracle import ref_runner
from oracle.spm_oracle import MT19937, OracleSPM

pytestmark = pytest.mark.skipif(not ref_runner.available(), reason="reference program not built here")


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("seed,np_,kbt,ro", [(21, 3, 0.0, False), (22, 5, 2e-4, True)])
def test_oracle_tracks_reference(seed, np_, kbt, ro):
    cfg = SPMConfig(npx=5, npy=5, npz=5, n_particles=np_, a=3.5, a_xi=2.0, dt=0.05, kbt=kbt, num_snap=12,
                    body_force=(0.0, 0.0, 5e-4))
    parts = make_particles(cfg, seed=seed, v_sd=1e-3, random_orientation=ro)
    with tempfile.TemporaryDirectory() as td:
        keys, dump = os.path.join(td, "k"), os.path.join(td, "d")
        write_udf_keys(keys, cfg, parts, out_dir=os.path.join(td, "avs"))
        ref_runner.run_reference(keys, dump, fields_every=4, body_force=cfg.body_force)
        frames = ref_runner.read_dump(dump)["frames"]
    o = OracleSPM(cfg, parts)
    for f in frames:
        assert rel(o.x, f["x"]) < 1e-13 and rel(o.v, f["v"]) < 1e-12
        if "u" in f:
            assert rel(o.velocity_field(), f["u"]) < 1e-12
            assert rel(o.phi, f["phi"]) < 1e-12
        o.step()


def test_mt19937_known_answer():
    # init_genrand(5489): first outputs of the published reference generator
    mt = MT19937(5489)
    assert [mt.genrand_int32() for _ in range(3)] == [3499211612, 581869302, 3890346734]
