"""GPU FP64 path against the fixtures produced by the reference program
itself (tests/golden/): every step's particle state and the retained zeta
modes / velocity checksums at the stored steps, within 1e-10."""
import numpy as np
import pytest

from kapsel3_b200.spm import SPMRun
from tests.golden_util import check_state, fixture_names, load

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.mark.parametrize("name", fixture_names())
def test_gpu_matches_reference_fixture(gpu, name):
    cfg, parts, z = load(name)
    steps = set(int(s) for s in z["field_steps"])
    frame_ts = [int(t) for t in z["traj_ts"]]
    with SPMRun(cfg) as run:
        run.initialize(parts)
        done = 0
        for i, ts in enumerate(frame_ts):
            if ts > done:
                run.step(ts - done)
                done = ts
            p = run.particles()
            zeta = u = None
            if ts in steps:
                zeta, _ = run.zeta()
                u = run.velocity()
            worst, errs = check_state(z, i, cfg, p["x"], p["v"], p["omega"], p["q"], p["f_hydro_previous"],
                                      zeta=zeta, u=u, tol=TOL, ts=ts)
            assert worst < TOL, (name, ts, errs)
