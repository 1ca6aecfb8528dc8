"""Hand-written 3D real FFT against numpy.fft (the FFTW r2c convention the
reference produces from Ooura's rdft3d + rdft3dsort + conjugation,
fft_wrapper.h:641-681)."""
import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from kapsel3_b200.udf import SPMConfig

pytestmark = pytest.mark.gpu

SHAPES = [(3, 3, 3), (4, 4, 4), (5, 5, 5), (6, 5, 4), (4, 6, 5), (7, 7, 7), (5, 4, 8), (8, 8, 8), (9, 3, 3),
          (3, 3, 6), (4, 3, 9)]


@pytest.mark.parametrize("np3", SHAPES)
@pytest.mark.parametrize("prec", [N.SPM_PREC_FP64, N.SPM_PREC_FP32_MIXED])
def test_fft_matches_numpy(gpu, np3, prec):
    cfg = SPMConfig(npx=np3[0], npy=np3[1], npz=np3[2], n_particles=0, lj_truncate="NONE")
    rng = np.random.default_rng(sum(np3) + 7 * prec)
    a = rng.standard_normal(cfg.shape)
    with SPMRun(cfg, precision=prec) as run:
        ak = run.A2a_k(a)
        ref = np.fft.rfftn(a)
        tol = 1e-13 if prec == N.SPM_PREC_FP64 else 3e-6
        err = np.abs(ak - ref).max() / np.abs(ref).max()
        assert err < tol, err
        # inverse of a Hermitian spectrum (numpy's own) returns the field
        back = run.A_k2a(ref)
        err2 = np.abs(back - a).max() / np.abs(a).max()
        assert err2 < tol, err2
