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
                                  "le_32_boundary_crossing"])
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
