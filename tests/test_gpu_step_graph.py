"""spm_step replays a captured CUDA graph of the Navier_Stokes step, and of
the Electrolyte step once its ion fields are inside the 2/3 box, for a lone
run.  The replayed run must advance exactly like the directly launched one
(SPM_NO_GRAPH=1): same step counter and time, same kernel-launch count, the
same state up to the order of the float atomics in the shared-profile
scatters (1e-12 relative); a zeta set by the host between steps is truncated
before the next replay, and an AC field follows a time set by the host."""
import os

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from kapsel3_b200.udf import EQ_EL, SPMConfig, make_particles

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def _run(cfg, parts, prec, graph, zeta_mid=None, time_mid=None):
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
        if time_mid is not None:
            run.set_time(*time_mid)
        run.step(3)
        conc = [run.concentration(n) for n in range(2)] if cfg.equation == EQ_EL else []
        return run.particles(), run.zeta(), run.time(), run.kernel_launches(), conc


@pytest.mark.parametrize("prec", [N.SPM_PREC_FP64, N.SPM_PREC_FP32_MIXED])
def test_graph_replay_matches_direct_launches(gpu, prec):
    cfg = SPMConfig(npx=5, npy=5, npz=6, n_particles=4, a=4.0, a_xi=2.0, dt=0.05, kbt=1e-4)
    parts = make_particles(cfg, seed=21, v_sd=1e-3, random_orientation=True)
    pa, (za, da), ta, la, _ = _run(cfg, parts, prec, graph=True)
    pb, (zb, db), tb, lb, _ = _run(cfg, parts, prec, graph=False)
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
    pa, (za, _), _, _, _ = _run(cfg, parts, N.SPM_PREC_FP64, graph=True, zeta_mid=(z, dc))
    pb, (zb, _), _, _, _ = _run(cfg, parts, N.SPM_PREC_FP64, graph=False, zeta_mid=(z, dc))
    assert rel(za, zb) <= 1e-12
    assert rel(pa["v"], pb["v"]) <= 1e-12


@pytest.mark.parametrize("prec", [N.SPM_PREC_FP64, N.SPM_PREC_FP32_MIXED])
@pytest.mark.parametrize("set_time", [False, True])
def test_electrolyte_graph_replay_matches_direct_launches(gpu, prec, set_time):
    """Salt with an AC field: the field's phase comes from the time on the
    device, so a replayed step uses the field of its own time, also after
    the host moved the time (spm_set_time) between replays."""
    cfg = SPMConfig(npx=5, npy=4, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.01, equation=EQ_EL, kbt=1.0,
                    salt=True, valency=(1.0, -1.0), onsager=(1.0, 1.5), debye_length=5.0, surface_charge=-12.0,
                    e_field="AC", e_ext=(0.1, 0.05, 0.0), e_frequency=4.0)
    parts = make_particles(cfg, seed=13, v_sd=1e-3, random_orientation=True)
    tm = (4, 0.3125) if set_time else None
    pa, (za, da), ta, la, ca = _run(cfg, parts, prec, graph=True, time_mid=tm)
    pb, (zb, db), tb, lb, cb = _run(cfg, parts, prec, graph=False, time_mid=tm)
    assert ta == tb and la == lb
    if set_time:
        assert ta[0] == 7 and abs(ta[1] - (0.3125 + 3 * 0.01)) < 1e-12
        # the field's phase moved with the time: the run differs from one that kept its time
        pc = _run(cfg, parts, prec, graph=True)[0]
        assert rel(pa["v"], pc["v"]) > 1e-9
    for k in ("x", "v", "omega", "q", "f_hydro_previous"):
        assert rel(pa[k], pb[k]) <= 1e-12, k
    assert rel(za, zb) <= 1e-12 and rel(da, db) <= 1e-12
    for a, b in zip(ca, cb):
        assert rel(a, b) <= 1e-12
