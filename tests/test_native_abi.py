"""The C ABI library loads and exports every symbol include/kapsel_spm.h
declares; host-side parameter handling (no GPU work)."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.udf import SPMConfig, make_particles, write_udf_keys


def test_library_exports_every_declared_symbol():
    L = N.lib()
    syms = N.declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_params_default_and_bytes():
    L = N.lib()
    p = N.SpmParams()
    assert L.spm_params_default(C.byref(p)) == 0
    assert (p.npx, p.dx, p.dt, p.lj_truncate, p.rotation) == (5, 1.0, 0.05, 1, 1)
    p.npx = p.npy = p.npz = 8
    p.n_particles = 1000
    nb = C.c_size_t()
    assert L.spm_device_bytes(C.byref(p), C.byref(nb)) == 0
    assert 11 * 256 * 256 * 129 * 16 <= nb.value < 13 * 256 * 256 * 129 * 16
    p.npx = 12
    assert L.spm_device_bytes(C.byref(p), C.byref(nb)) == 1
    assert b"NPX" in L.spm_last_error()


def test_udf_key_file_roundtrip():
    cfg = SPMConfig(npx=5, npy=6, npz=4, n_particles=3, a=3.0, a_xi=2.0, dt=0.04, kbt=1e-4,
                    fix_cell=(True, False, True), rotation=False, mass_ratio=1.0)
    parts = make_particles(cfg, seed=3, v_sd=1e-3, random_orientation=True)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "in.keys")
        write_udf_keys(path, cfg, parts)
        p = N.SpmParams()
        rec = np.zeros((3, N.SPM_PARTICLE_WORDS))
        rc = N.lib().spm_params_from_udf_keys(path.encode(), C.byref(p), N.dptr(rec), 3)
        assert rc == 0, N.lib().spm_last_error()
    assert (p.npx, p.npy, p.npz, p.n_particles) == (5, 6, 4, 3)
    assert (p.a, p.a_xi, p.dt, p.kbt) == (3.0, 2.0, 0.04, 1e-4)
    assert list(p.fix_cell) == [1, 0, 1] and p.rotation == 0 and p.equation == N.SPM_EQ_NAVIER_STOKES
    np.testing.assert_array_equal(rec[:, 0:3], parts["x"])
    np.testing.assert_array_equal(rec[:, 6:9], parts["v"])
    # ROTATION OFF: Init_Particle sets the identity orientation
    np.testing.assert_array_equal(rec[:, 18:22], np.tile([1.0, 0.0, 0.0, 0.0], (3, 1)))


def test_udf_rejects_out_of_scope_equation():
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "in.keys")
        open(path, "w").write("constitutive_eq.type = Navier_Stokes_FDM\n")
        p = N.SpmParams()
        assert N.lib().spm_params_from_udf_keys(path.encode(), C.byref(p), None, 0) == 1
        assert b"Navier_Stokes_FDM" in N.lib().spm_last_error()


def test_create_without_device_fails_cleanly():
    if os.environ.get("CUDA_VISIBLE_DEVICES", None) == "" or not _gpu_visible():
        p = N.SpmParams()
        N.lib().spm_params_default(C.byref(p))
        h = C.c_void_p()
        assert N.lib().spm_create(C.byref(p), None, C.byref(h)) == 5
    else:
        pytest.skip("a GPU is visible")


def _gpu_visible():
    n = C.c_int()
    N.lib().spm_device_count(C.byref(n))
    return n.value > 0


def test_janus_parameter_checks():
    """Janus runs are Navier_Stokes only; a SQUIRMER needs an axis, B1 > 0 and
    a slip iteration budget (input.cxx:1410-1466, 1868-1872).  derive()
    runs without a device."""
    L = N.lib()
    nb = C.c_size_t()
    def bytes_rc(**kw):
        p = N.SpmParams()
        L.spm_params_default(C.byref(p))
        p.n_particles = 2
        for k, v in kw.items():
            setattr(p, k, v)
        return L.spm_device_bytes(C.byref(p), C.byref(nb)), L.spm_last_error().decode()
    ok = dict(janus_propulsion=N.SPM_JANUS_SQUIRMER, janus_axis=N.SPM_AXIS_Z, slip_vel=0.01)
    assert bytes_rc(**ok)[0] == 0
    assert bytes_rc(janus_propulsion=N.SPM_JANUS_TUMBLER)[0] == 0
    for bad, msg in ((dict(ok, janus_axis=N.SPM_AXIS_NONE), "janus_axis"), (dict(ok, slip_vel=0.0), "B1"),
                     (dict(ok, slip_iter=0), "SLIP_iter"), (dict(ok, equation=N.SPM_EQ_LEES_EDWARDS), "Navier_Stokes"),
                     (dict(janus_propulsion=7), "janus_propulsion")):
        rc, err = bytes_rc(**bad)
        assert rc == 1 and msg in err, (bad, err)  # SPM_ERR_ARG
