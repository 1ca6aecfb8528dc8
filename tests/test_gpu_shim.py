"""The drop-in boundary, end to end: the reference program itself (built
from its unmodified sources) with its boundary functions -- NS_solver_slavedEuler,
Zeta_k2u_k, U_k2zeta_k, Solenoidal_uk, Make_phi_particle_sum,
Make_u_particle_sum, Calc_f_hydro_correct_precision and the Lennard-Jones
cell-list forces -- linked to the B200 library through
kapsel3_b200/shim/kapsel_b200_shim.cxx (-Wl,--wrap).  Its own main loop,
integrators and remaining CPU FFTs run unchanged; its FP64 trajectory must
match the pure reference program's (the golden fixtures) within 1e-10."""
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
                                  "noncubic_lj_multiplicity"])
def test_reference_program_with_gpu_boundary_matches_reference(gpu, name):
    if not ref_runner.available(gpu_shim=True):
        pytest.skip("oracle/_ref/kapsel_gpu is not built (make -C oracle/ref_build gpu, needs the reference sources)")
    cfg, parts, z = load(name)
    with tempfile.TemporaryDirectory() as td:
        keys = os.path.join(td, "run.keys")
        dump = os.path.join(td, "run.dump")
        write_udf_keys(keys, cfg, parts, out_dir=os.path.join(td, "avs"))
        ref_runner.run_reference(keys, dump_path=dump, fields_every=0, body_force=cfg.body_force, gpu_shim=True,
                                 timeout=600.0)
        frames = ref_runner.read_dump(dump)["frames"]
    assert len(frames) == len(z["traj_ts"])
    worst = 0.0
    for i, f in enumerate(frames):
        for k in ("x", "v", "omega", "q", "f_hydro_previous"):
            e = rel(f[k], z["traj_" + k][i])
            worst = max(worst, e)
            assert e <= TOL, (name, i, k, e)
        assert rel(f["uk_dc"], z["traj_uk_dc"][i]) <= TOL or np.abs(f["uk_dc"]).max() < 1e-300
    assert worst <= TOL
