"""Legacy AVS output (spm_avs_open / spm_avs_frame / spm_avs_close) against
the files the reference program writes itself (oracle/_ref/kapsel_ref_avs:
avs_output.cxx, avs_output_p.cxx, output.cxx:129-191) for the same run.

Headers (.fld, p.fld, .cod) must be identical byte for byte.  The float
fields (u, phi, the five strain components) and the particle files agree
to FP32 rounding: the FP64 states of the two programs differ by ~1e-12
relative after a few steps, so a float may land one ulp apart.  The
reference never computes its pressure column (output.cxx:168); this
writer's is zero."""
import os

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from kapsel3_b200.udf import EQ_LE, SPMConfig, make_particles, write_udf_keys
from oracle import ref_runner

pytestmark = pytest.mark.gpu

AVS_REF = os.path.join(ref_runner.REF_DIR, "kapsel_ref_avs")


def _our_frames(cfg, parts, out_dir, prec=N.SPM_PREC_FP64):
    with SPMRun(cfg, precision=prec) as run:
        run.initialize(parts)
        run.avs_open(out_dir, "frame", cfg.num_snap)
        # the reference's main loop: output at ts % GTS == 0, then the step,
        # for ts = 0..MSTEP (sp_3d_ns.cxx:857-875)
        for ts in range(cfg.mstep + 1):
            if ts % cfg.gts == 0:
                run.avs_frame()
            run.step(1)
        run.avs_close()


def _fields(path, cfg):
    nx, ny, nz = cfg.shape
    return np.fromfile(path, dtype=np.float32).reshape(10, nz, ny, nx)


LE_CASE = SPMConfig(npx=5, npy=5, npz=4, n_particles=3, a=3.5, a_xi=2.0, dt=0.05, gts=2, num_snap=3,
                    equation=EQ_LE, shear_rate=0.5, kbt=1e-5)


@pytest.mark.skipif(not os.access(AVS_REF, os.X_OK), reason="oracle/_ref/kapsel_ref_avs is not built")
@pytest.mark.parametrize("equation", ["navier_stokes", "lees_edwards"])
def test_avs_files_match_the_reference_program(gpu, tmp_path, equation):
    """Lees-Edwards frames take u and the stress from the oblique grid and
    components to Cartesian ones, u with the mean flow of Shear_rate_eff
    (U_oblique2u, Stress_oblique2Stress; output.cxx:133-146)."""
    if equation == "lees_edwards":
        cfg = LE_CASE
    else:
        cfg = SPMConfig(npx=5, npy=4, npz=6, n_particles=3, a=4.0, a_xi=2.0, dt=0.05, gts=2, num_snap=2)
    parts = make_particles(cfg, seed=3, v_sd=1e-3, random_orientation=True)
    keys = str(tmp_path / "in.keys")
    write_udf_keys(keys, cfg, parts, out_dir=str(tmp_path / "ref"))
    ref_runner.run_reference_avs(keys)
    _our_frames(cfg, parts, str(tmp_path / "gpu"))
    ref, ours = tmp_path / "ref", tmp_path / "gpu"
    for name in ("frame.fld", "framep.fld", "frame.cod"):
        assert (ours / name).read_bytes() == (ref / name).read_bytes(), name
    for ts in range(0, cfg.mstep + 1, cfg.gts):
        a = _fields(ours / "avs" / f"frame_{ts}.dat", cfg)
        b = _fields(ref / "avs" / f"frame_{ts}.dat", cfg)
        for f in range(10):
            if f == 4:  # pressure
                assert not a[f].any()
                continue
            scale = max(float(np.abs(b[f]).max()), 1e-30)
            assert float(np.abs(a[f] - b[f]).max()) <= 2e-6 * scale, (ts, f)
        for ext in ("cod", "dat"):
            pa = np.fromfile(ours / "avs" / f"framep_{ts}.{ext}", dtype=np.float32)
            pb = np.fromfile(ref / "avs" / f"framep_{ts}.{ext}", dtype=np.float32)
            assert pa.shape == pb.shape
            np.testing.assert_allclose(pa, pb, rtol=2e-6, atol=1e-6)


def test_avs_fp32_run_and_errors(gpu, tmp_path):
    cfg = SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.05, gts=1, num_snap=3)
    parts = make_particles(cfg, seed=4)
    _our_frames(cfg, parts, str(tmp_path / "fp32"), prec=N.SPM_PREC_FP32_MIXED)
    for ts in range(cfg.mstep + 1):
        a = _fields(tmp_path / "fp32" / "avs" / f"frame_{ts}.dat", cfg)
        assert np.isfinite(a).all()
        assert 0.9 < a[3].max() < 1.1  # phi inside a particle
    text = (tmp_path / "fp32" / "frame.fld").read_text()
    assert text.count("EOT") == cfg.mstep + 1
    with SPMRun(cfg) as run:
        run.initialize(parts)
        with pytest.raises(N.SpmError, match="spm_avs_open was not called"):
            run.avs_frame()
