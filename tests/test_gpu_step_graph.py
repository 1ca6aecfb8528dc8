"""spm_step replays a captured CUDA graph of the Navier_Stokes step for a
lone run.  The replayed run must advance exactly like the directly launched
one (SPM_NO_GRAPH=1): same step counter and time, same kernel-launch count,
the same state up to the order of the float atomics in the shared-profile
scatters (1e-12 relative), and a zeta set by the host between steps is
truncated before the next replay."""
import os

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from kapsel3_b200.udf import SPMConfig, make_particles

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def _run(cfg, parts, prec, graph, zeta_mid=None):
    old = os.environ.get("SPM_NO_GRAPH")
    os.environ["SPM_NO_GRAPH"] = "0" if graph else "1"
    try:
        run = SPMRun(cfg, precision=prec)
    finally:
        if old is None:
            del os.environ["SPM_NO_GRAPH"]
        else:
            os.environ["SPM_NO_GRAPH"] = old
    with run:
        run.initialize(parts)
        run.kernel_launches(reset=True)
        run.step(4)
        if zeta_mid is not None:
            run.set_zeta(*zeta_mid)
        run.step(3)
        return run.particles(), run.zeta(), run.time(), run.kernel_launches()


@pytest.mark.parametrize("prec", [N.SPM_PREC_FP64, N.SPM_PREC_FP32_MIXED])
def test_graph_replay_matches_direct_launches(gpu, prec):
    cfg = SPMConfig(npx=5, npy=5, npz=6, n_particles=4, a=4.0, a_xi=2.0, dt=0.05, kbt=1e-4)
    parts = make_particles(cfg, seed=21, v_sd=1e-3, random_orientation=True)
    pa, (za, da), ta, la = _run(cfg, parts, prec, graph=True)
    pb, (zb, db), tb, lb = _run(cfg, parts, prec, graph=False)
    assert ta == tb and la == lb
    for k in ("x", "v", "omega", "q", "f_hydro_previous"):
        assert rel(pa[k], pb[k]) <= 1e-12, k
    assert rel(za, zb) <= 1e-12 and rel(da, db) <= 1e-12


def test_host_zeta_between_replays(gpu):
    cfg = SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.05)
    parts = make_particles(cfg, seed=5)
    with SPMRun(cfg) as probe:
        probe.initialize(parts)
        probe.step(2)
        z, dc = probe.zeta()
    rng = np.random.default_rng(1)
    z = z + 1e-4 * (rng.standard_normal(z.shape) + 1j * rng.standard_normal(z.shape))
    pa, (za, _), _, _ = _run(cfg, parts, N.SPM_PREC_FP64, graph=True, zeta_mid=(z, dc))
    pb, (zb, _), _, _ = _run(cfg, parts, N.SPM_PREC_FP64, graph=False, zeta_mid=(z, dc))
    assert rel(za, zb) <= 1e-12
    assert rel(pa["v"], pb["v"]) <= 1e-12
