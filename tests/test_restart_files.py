"""The reference program's restart files without a GPU: the key file the
reference writes (Save_Restart_udf, resume.cxx:10-74, through the UDF
stand-in of oracle/ref_build) parses as an input with all its parameters,
and the same keys written as a UDF file (udf.write_udf_from_keys) read back
through this library's UDF reader unchanged, so spm_load_restart sees the
same section in either form.  The GPU side is tests/test_gpu_restart.py."""
import ctypes as C
import os

import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import config_from_udf, read_udf
from kapsel3_b200.udf import SPMConfig, make_particles, read_udf_keys, write_udf_from_keys, write_udf_keys
from oracle import ref_runner

pytestmark = pytest.mark.skipif(not ref_runner.available(), reason="reference program not built (oracle/_ref)")


@pytest.fixture(scope="module")
def restart_keys(tmp_path_factory):
    tmp = str(tmp_path_factory.mktemp("restart"))
    cfg = SPMConfig(npx=4, npy=4, npz=5, n_particles=2, a=2.5, a_xi=2.0, dt=0.05, kbt=1e-5, num_snap=2)
    parts = make_particles(cfg, seed=3, v_sd=1e-3, random_orientation=True)
    keys = os.path.join(tmp, "run.keys")
    write_udf_keys(keys, cfg, parts, out_dir=os.path.join(tmp, "avs"))
    res = os.path.join(tmp, "restart.keys")
    ref_runner.run_reference(keys, restart_path=res)
    return cfg, res


def test_reference_restart_file_holds_the_saved_section(restart_keys):
    cfg, res = restart_keys
    kv = read_udf_keys(res)
    assert kv["resume.Calculation"] == "CONTINUE"
    p = "resume.CONTINUE.Saved_Data."
    nx, ny, nz_ = cfg.shape[0], cfg.shape[1], cfg.shape[2] + 2
    assert f"{p}Zeta[{nx - 1}][{ny - 1}][{nz_ - 1}].zeta1" in kv and f"{p}Zeta[{nx}][0][0].zeta0" not in kv
    assert int(kv[p + "jikan.ts"]) == 2 and float(kv[p + "jikan.time"]) == pytest.approx(3 * cfg.dt)
    for j in range(cfg.n_particles):
        for f in ("R", "R_raw", "v", "v_old", "omega", "omega_old", "f_hydro_previous", "fr_previous"):
            assert f"{p}Particles[{j}].{f}.z" in kv
    # the parameters come along: the file is an input of its own
    got, parts = config_from_udf(res)
    assert got.shape == cfg.shape and got.n_particles == cfg.n_particles and got.kbt == cfg.kbt


def test_restart_keys_as_udf_file_read_back_unchanged(restart_keys, tmp_path):
    _, res = restart_keys
    kv = read_udf_keys(res)
    udf = str(tmp_path / "restart.udf")
    write_udf_from_keys(udf, kv)
    back = read_udf(udf)
    assert back == kv
    pk, pu = N.SpmParams(), N.SpmParams()
    assert N.lib().spm_params_from_udf_keys(res.encode(), C.byref(pk), None, 0) == 0
    assert N.lib().spm_params_from_udf(udf.encode(), C.byref(pu), None, 0) == 0
    assert bytes(pk) == bytes(pu)
