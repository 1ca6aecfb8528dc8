"""Each reference solver boundary exposed by the C ABI, called with host
arrays in the reference layout, against the oracle's restatement of the same
reference function (FP64, 1e-11)."""
import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun, pack_particles
from kapsel3_b200.udf import SPMConfig, make_particles
from oracle.spm_oracle import OracleSPM

pytestmark = pytest.mark.gpu
TOL = 1e-11


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


@pytest.fixture(scope="module")
def setup():
    cfg = SPMConfig(npx=5, npy=4, npz=5, n_particles=4, a=3.0, a_xi=2.0, dt=0.05, kbt=0.0)
    parts = make_particles(cfg, seed=9, v_sd=1e-2, random_orientation=True)
    parts["omega"] = np.random.default_rng(1).normal(0, 1e-2, (4, 3))
    o = OracleSPM(cfg, parts)
    for _ in range(3):
        o.step()
    run = SPMRun(cfg)
    yield cfg, parts, o, run
    run.close()


def test_zeta_u_maps(gpu, setup):
    cfg, parts, o, run = setup
    uk = run.Zeta_k2u_k(o.zeta, o.uk_dc)
    assert rel(uk, o.zeta_k2u_k(o.zeta, o.uk_dc)) < TOL
    z, dc = run.U_k2zeta_k(uk)
    zr, dcr = o.u_k2zeta_k(uk)
    assert rel(z, zr) < TOL and np.allclose(dc, dcr, rtol=1e-13, atol=0)


def test_solenoidal_uk(gpu, setup):
    cfg, parts, o, run = setup
    rng = np.random.default_rng(4)
    uk = o.fft(rng.standard_normal((3,) + cfg.shape))
    assert rel(run.Solenoidal_uk(uk), o.solenoidal_uk(uk)) < TOL


def test_ns_solver(gpu, setup):
    cfg, parts, o, run = setup
    ref = OracleSPM(cfg, parts)
    ref.zeta, ref.uk_dc = o.zeta.copy(), o.uk_dc.copy()
    ref.ns_solver_slaved_euler()
    got = run.NS_solver_slavedEuler(o.zeta, o.uk_dc)
    assert rel(got, ref.zeta) < TOL


def test_phi_and_up(gpu, setup):
    cfg, parts, o, run = setup
    rec = pack_particles(dict(x=o.x, v=o.v, omega=o.omega, q=o.q), cfg.n_particles)
    phi, phs = run.Make_phi_particle_sum(rec)
    o.make_phi_particle_sum()
    assert rel(phs, o.phi_sum) < TOL and rel(phi, o.phi) < TOL
    up = run.Make_u_particle_sum(rec, o.phi_sum)
    assert rel(up, o.make_u_particle_sum()) < TOL
    phi2, up2 = run.Make_phi_u_particle(rec)
    assert rel(phi2, o.phi) < TOL and rel(up2, o.make_u_particle_sum()) < 1e-10


def test_make_f_sole_and_hydro(gpu, setup):
    cfg, parts, o, run = setup
    o.make_phi_particle_sum()
    up = o.make_u_particle_sum()
    f = run.Make_f_particle_dt_sole(o.u, up, o.phi)
    assert rel(f, o.solenoidal_u(up - o.phi[None] * o.u)) < TOL
    rec = pack_particles(dict(x=o.x, v=o.v, omega=o.omega, q=o.q), cfg.n_particles)
    out = run.Calc_f_hydro_correct_precision(rec, o.phi_sum, o.u)
    o.calc_f_hydro()
    assert rel(out[:, 26:29], o.f_hydro) < TOL and rel(out[:, 32:35], o.torque_hydro) < TOL


def test_lennard_jones(gpu, setup):
    cfg, parts, o, run = setup
    x = o.x.copy()
    x[1] = x[0] + np.array([6.2, 0.0, 0.0])  # inside the cutoff 2^(1/6)*6
    x %= o.L
    rec = pack_particles(dict(x=x, v=o.v, omega=o.omega, q=o.q), cfg.n_particles)
    out = run.Calc_f_Lennard_Jones(rec)
    o2 = OracleSPM(cfg, dict(x=x, v=o.v, omega=o.omega, q=o.q))
    o2.fr[:] = 0.0
    o2.calc_f_lennard_jones()
    assert np.abs(o2.fr).max() > 0
    assert rel(out[:, 38:41], o2.fr) < TOL


def test_fft_roundtrip_host(gpu, setup):
    cfg, parts, o, run = setup
    a = np.random.default_rng(2).standard_normal(cfg.shape)
    ak = run.A2a_k(a)
    assert rel(ak, np.fft.rfftn(a)) < 1e-14
    assert rel(run.A_k2a(ak), a) < 1e-14
