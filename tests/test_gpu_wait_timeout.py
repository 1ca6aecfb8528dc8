"""Bounded device waits of the TMA transform passes.

Every wait of a pass on its ring of tile buffers is bounded by the GPU's
global timer (spm_set_wait_limit, default 1 s).  Here the limit is set to
1 ms and the test switch spm_debug_skip_tma_loads makes the next pass issue
no tile load at all: its waits run out with nothing in flight, the pass
stops, and the next synchronising call reports SPM_ERR_DEVICE with the
timeout message.  The context then serves again: re-initialised, it steps
like a run that never timed out (1e-12).  No GPU is faulted or hung: the
flag that nothing sets is an mbarrier phase that no load completes.
"""
import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from kapsel3_b200.udf import SPMConfig, make_particles

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


@pytest.mark.parametrize("prec", [N.SPM_PREC_FP64, N.SPM_PREC_FP32_MIXED])
def test_wait_runs_out_then_context_recovers(gpu, prec):
    cfg = SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.05, body_force=(1e-3, 0.0, 0.0))
    parts = make_particles(cfg, seed=7, v_sd=1e-3, random_orientation=True)
    with SPMRun(cfg, precision=prec) as ref:
        ref.initialize(parts)
        ref.step(3)
        want_p, (want_z, want_dc) = ref.particles(), ref.zeta()
    with SPMRun(cfg, precision=prec) as run:
        L = run.L
        run.initialize(parts)
        run.step(1)  # graph replay captured with the default limit
        assert L.spm_set_wait_limit(run.h, 1e-3) == 0
        assert L.spm_debug_skip_tma_loads(run.h, 1) == 0
        run.step(1)
        with pytest.raises(N.SpmError, match="TMA pipeline wait timed out"):
            run.synchronize()
        # the switch disarmed itself after one pass; the error word was cleared
        assert L.spm_set_wait_limit(run.h, 1.0) == 0
        run.synchronize()
        run.initialize(parts)
        run.step(3)
        got_p, (got_z, got_dc) = run.particles(), run.zeta()
    for k in ("x", "v", "omega", "q"):
        assert rel(got_p[k], want_p[k]) <= 1e-12, k
    assert rel(got_z, want_z) <= 1e-12 and rel(got_dc, want_dc) <= 1e-12


def test_wait_limit_arguments(gpu):
    cfg = SPMConfig(npx=3, npy=3, npz=3, n_particles=0, lj_truncate="NONE")
    with SPMRun(cfg) as run:
        # 1 = SPM_ERR_ARG
        assert run.L.spm_set_wait_limit(run.h, 0.0) == 1
        assert run.L.spm_set_wait_limit(run.h, 120.0) == 1
        assert run.L.spm_debug_skip_tma_loads(run.h, -1) == 1
