"""Precision form against the FP64 path on the benchmark workloads.

C3: 256^3, 1000 colloids a=5, seeded state, no noise.  The FP32-mixed path
(FP32 fields / FFT / projection / advection, zeta kept as a compensated
FP32 pair, FP64 particle reductions, integrators and k = 0 mode) stays within
1e-5 relative L2 of the FP64 GPU path in the velocity field, phi and particle
x, v, omega at every 50th of 500 steps (the configuration's full length).

C4: 128^3 Lees-Edwards, shear rate 1e-3, 400 colloids a=4: the mean apparent
shear stress (Mean_shear_stress, sp_3d_ns.h:325) over 2000 steps (the
configuration's full length) agrees within 1e-5 relative."""
import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from kapsel3_b200.udf import EQ_LE, SPMConfig, make_particles

pytestmark = pytest.mark.gpu
TOL = 1e-5


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def test_c3_fp32_mixed_tracks_fp64(gpu):
    cfg = SPMConfig(npx=8, npy=8, npz=8, n_particles=1000, a=5.0, a_xi=2.0, dt=0.05)
    parts = make_particles(cfg, seed=2024, v_sd=1e-3, random_orientation=True)
    with SPMRun(cfg, precision=N.SPM_PREC_FP32_MIXED) as r32, SPMRun(cfg, precision=N.SPM_PREC_FP64) as r64:
        r32.initialize(parts)
        r64.initialize(parts)
        for ts in range(50, 501, 50):
            r32.step(50)
            r64.step(50)
            p32, p64 = r32.particles(), r64.particles()
            errs = dict(u=rel(r32.velocity(), r64.velocity()), phi=rel(r32.phi(), r64.phi()),
                        x=rel(p32["x"], p64["x"]), v=rel(p32["v"], p64["v"]), omega=rel(p32["omega"], p64["omega"]))
            assert max(errs.values()) <= TOL, (ts, errs)


def test_c4_lees_edwards_stress_fp32_mixed_vs_fp64(gpu):
    cfg = SPMConfig(npx=7, npy=7, npz=7, n_particles=400, a=4.0, a_xi=2.0, dt=0.05, equation=EQ_LE,
                    shear_rate=1e-3)
    parts = make_particles(cfg, seed=4, v_sd=1e-3, random_orientation=True)
    means = {}
    for prec in (N.SPM_PREC_FP32_MIXED, N.SPM_PREC_FP64):
        with SPMRun(cfg, precision=prec) as r:
            r.initialize(parts)
            app = []
            for _ in range(2000):
                r.step(1)
                app.append(r.shear_state()[1][7])
            means[prec] = float(np.mean(app))
    err = abs(means[N.SPM_PREC_FP32_MIXED] - means[N.SPM_PREC_FP64]) / abs(means[N.SPM_PREC_FP64])
    assert err <= TOL, (means, err)
