"""Host side of rigid bodies (object_type rigid) without a GPU: the UDF
round trip of Rigid_spec[] / switch.free_rigid / gravity, the checks the
library makes before it allocates anything (spm_device_bytes runs them),
and the reference's example inputs."""
import ctypes as C
import glob
import os

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import config_from_udf, params_from_config, read_udf
from kapsel3_b200.udf import SPMConfig, make_rigid_bodies, write_udf, write_udf_keys
from oracle import ref_runner

REFERENCE_TREE = ref_runner.reference_tree() or ""

BASE = dict(npx=5, npy=5, npz=6, a=3.0, a_xi=2.0, dt=0.05, kbt=1e-5,
            rigid=((3, 2, 1.0, "free", (0.0, 0.0, 0.0), (0.0, 0.0, 0.0)),
                   (4, 1, 2.0, "fix", (1e-3, 0.0, 0.0), (0.0, 0.0, 2e-3))),
            rigid_dof=((0, (True, True, False), (False, True, True)),), rigid_gravity=(0.0, 0.0, 2e-3))


def _cfg(**kw):
    c = dict(BASE)
    c.update(kw)
    c["n_particles"] = sum(int(b) * int(n) for b, n, *_ in c["rigid"])
    return SPMConfig(**c)


def _bytes(p):
    n = C.c_size_t()
    return N.lib().spm_device_bytes(C.byref(p), C.byref(n)), n.value


def test_rigid_params_from_config():
    p = params_from_config(_cfg(), N.SPM_PREC_FP64, 0)
    assert p.rigid == 1 and p.n_species == 2 and p.n_particles == 10
    assert list(p.rigid_beads)[:2] == [3, 4] and list(p.rigid_count)[:2] == [2, 1]
    assert list(p.species_count)[:2] == [6, 4] and list(p.species_mass_ratio)[:2] == [1.0, 2.0]
    assert [list(r) for r in p.rigid_free][:2] == [[1, 1, 0, 0, 1, 1], [0, 0, 0, 0, 0, 0]]
    assert list(p.rigid_velocity[1]) == [1e-3, 0.0, 0.0] and list(p.rigid_omega[1]) == [0.0, 0.0, 2e-3]
    assert list(p.rigid_gravity) == [0.0, 0.0, 2e-3]
    assert _bytes(p)[0] == 0


@pytest.mark.parametrize("writer", ["keys", "udf"])
def test_rigid_udf_round_trip(tmp_path, writer):
    cfg = _cfg()
    parts = make_rigid_bodies(cfg, seed=4, straddle=True)
    if writer == "keys":
        path = str(tmp_path / "run.keys")
        write_udf_keys(path, cfg, parts)
        p = N.SpmParams()
        rec = np.zeros((cfg.n_particles, N.SPM_PARTICLE_WORDS))
        assert N.lib().spm_params_from_udf_keys(path.encode(), C.byref(p), N.dptr(rec), cfg.n_particles) == 0
        want = params_from_config(cfg, N.SPM_PREC_FP64, 0)
        for f in ("rigid", "n_particles", "n_species"):
            assert getattr(p, f) == getattr(want, f), f
        for f in ("rigid_beads", "rigid_count", "species_count", "species_mass_ratio", "rigid_gravity"):
            assert list(getattr(p, f)) == list(getattr(want, f)), f
        for f in ("rigid_free", "rigid_velocity", "rigid_omega"):
            assert [list(r) for r in getattr(p, f)] == [list(r) for r in getattr(want, f)], f
        assert np.array_equal(rec[:, 0:3], parts["x"])
    else:
        path = str(tmp_path / "run.udf")
        write_udf(path, cfg, parts)
        got, gparts = config_from_udf(path)
        assert tuple(tuple(r) for r in got.rigid) == tuple(tuple(r) for r in cfg.rigid)
        assert got.rigid_gravity == cfg.rigid_gravity and got.n_particles == cfg.n_particles
        # switch.free_rigid comes back for every species (the unlisted ones keep Rigid_motion)
        assert got.rigid_dof[0] == cfg.rigid_dof[0]
        assert got.rigid_dof[1] == (1, (False, False, False), (False, False, False))
        assert np.array_equal(gparts["x"], parts["x"])


@pytest.mark.parametrize("change, message", [
    (dict(equation="Electrolyte", surface_charge=-1.0, valency=(1.0, 0.0), kbt=1.0), b"Lees-Edwards runs"),
    (dict(rotation=False), b"ROTATION ON"),
    (dict(body_force=(1e-3, 0.0, 0.0)), b"no constant body force"),
    (dict(rigid_gravity=(1e-3, 1e-3, 0.0)), b"one axis"),
])
def test_rigid_out_of_scope_is_refused(change, message):
    p = params_from_config(_cfg(**change), N.SPM_PREC_FP64, 0)
    rc, _ = _bytes(p)
    assert rc == N.SPM_ERR_ARG and message in N.lib().spm_last_error()


def test_rigid_bead_count_mismatch_is_refused():
    p = params_from_config(_cfg(), N.SPM_PREC_FP64, 0)
    p.n_particles = 9
    assert _bytes(p)[0] == N.SPM_ERR_ARG and b"add up to n_particles" in N.lib().spm_last_error()
    p = params_from_config(SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=3.0), N.SPM_PREC_FP64, 0)
    p.rigid_gravity[1] = 1e-3
    assert _bytes(p)[0] == N.SPM_ERR_ARG and b"spherical particles take body_force" in N.lib().spm_last_error()


def test_rigid_bodies_generator():
    cfg = _cfg()
    parts = make_rigid_bodies(cfg, seed=9, straddle=True)
    assert parts["x"].shape == (10, 3)
    assert parts["x"][0, 0] == pytest.approx(0.98 * 32)
    d = cfg.derived()
    L = np.array([d["LX"], d["LY"], d["LZ"]])
    first = [0, 3, 6, 10]
    for b in range(3):
        body = parts["x"][first[b]:first[b + 1]]
        steps = np.linalg.norm(np.diff(body, axis=0), axis=1)
        assert np.allclose(steps, 1.2 * cfg.a)
        r = body - body.mean(0)
        inertia = (r ** 2).sum() * np.eye(3) - r.T @ r
        ev = np.linalg.eigvalsh(inertia)
        assert np.min(np.diff(ev)) > 1e-3 * ev[-1]  # no equal principal moments
        for c in range(b + 1, 3):
            other = parts["x"][first[c]:first[c + 1]]
            dd = body[:, None] - other[None]
            dd -= np.rint(dd / L) * L
            assert np.sqrt((dd ** 2).sum(-1)).min() > 1.05 * d["SIGMA"]


def _rigid_examples():
    files = glob.glob(os.path.join(REFERENCE_TREE, "Examples", "*", "*.udf")) if REFERENCE_TREE else []
    out = []
    for f in sorted(files):
        if os.path.basename(f) in ("define.udf", "kapsel_unit.udf"):
            continue
        if read_udf(f).get("object_type.type") == "rigid":
            out.append(f)
    return out


@pytest.mark.skipif(not _rigid_examples(), reason="reference tree not present")
def test_reference_rigid_examples_pass_the_checks():
    """Every rigid example input of the reference parses unless it switches
    on a force outside the step (Examples/12: a flat wall and Quincke
    rotation); the others, Navier_Stokes, Shear_Navier_Stokes and the
    Lees-Edwards one (Examples/08/helixes_shear0005.udf), pass the library's
    checks (gravity included)."""
    ns = le = 0
    for f in _rigid_examples():
        p = N.SpmParams()
        kv = read_udf(f)
        if kv.get("switch.wall.type", "NONE") != "NONE":
            assert N.lib().spm_params_from_udf(f.encode(), C.byref(p), None, 0) == N.SPM_ERR_ARG, f
            assert b"outside the spectral SPM step" in N.lib().spm_last_error()
            continue
        assert N.lib().spm_params_from_udf(f.encode(), C.byref(p), None, 0) == 0, f
        rc, nbytes = _bytes(p)
        assert rc == 0 and nbytes > 0, (f, N.lib().spm_last_error())
        ns += p.equation in (N.SPM_EQ_NAVIER_STOKES, N.SPM_EQ_SHEAR_NAVIER_STOKES)
        le += p.equation == N.SPM_EQ_LEES_EDWARDS
    assert ns >= 6 and le >= 1
