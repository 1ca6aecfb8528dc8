"""UDF input files: the reader of the OCTA UDF format (schema blocks, data
block, \\include) and the loader built on it (spm_params_from_udf), which
reads a run as Gourmet_file_io (input.cxx:677-2556) and Init_Particle
(init_particle.cxx:12-453) do.

Pins:
- a UDF file written from a run description loads to exactly the parameters
  and particle records of the equivalent UDF key file;
- uniform_random placement and random orientation reproduce glibc's rand()
  stream after srand(10) (drawn here through ctypes from the C library
  itself) and, when the reference program is built, its initial frame;
- every example input shipped with the reference parses, and those of
  spherical particles under Navier_Stokes, Shear_Navier_Stokes,
  Lees-Edwards or Electrolyte load, squirmers and several species included
  (only where the reference tree is present).
No GPU work."""
import ctypes as C
import glob
import math
import os

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import config_from_udf, read_udf
from kapsel3_b200.udf import EQ_LE, SPMConfig, make_particles, udf_keys, write_udf, write_udf_keys
from oracle import ref_runner

REFERENCE_TREE = ref_runner.reference_tree() or ""
OUTSIDE_SWITCHES = (("switch.pin.type", "NO"), ("switch.wall.type", "NONE"), ("switch.quincke.type", "OFF"),
                    ("switch.multipole.type", "OFF"))


def load(path, n, keys=False):
    p = N.SpmParams()
    rec = np.zeros((max(n, 1), N.SPM_PARTICLE_WORDS))
    fn = N.lib().spm_params_from_udf_keys if keys else N.lib().spm_params_from_udf
    rc = fn(path.encode(), C.byref(p), N.dptr(rec), n)
    return rc, p, rec[:n]


CASES = {
    "ns": SPMConfig(npx=5, npy=6, npz=4, n_particles=3, a=3.0, a_xi=2.0, dt=0.04, kbt=1e-4,
                    fix_cell=(True, False, True), rotation=True),
    "le_no_rotation": SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.05, equation=EQ_LE,
                                shear_rate=0.25, rotation=False, lj_truncate="OFF", lj_powers="24:12"),
    "body_force": SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, body_force=(1e-3, 0.0, 0.0)),
    "squirmer": SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, janus_axis="Y", janus_propulsion="SQUIRMER",
                          slip_vel=0.015, slip_mode=-2.5, rotlet_c1=0.003, rotlet_c2=-0.001, slip_tol=2e-3,
                          slip_iter=7),
    "two_species": SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=4.0, species=((1, 1.0, 0.0), (2, 2.5, 0.0))),
    "tumbler": SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, janus_axis="Z", janus_propulsion="TUMBLER",
                         janus_force=(0.01, 0.0, -0.02), janus_torque=(0.0, 0.005, 0.0)),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("include", [False, True])
def test_udf_file_loads_like_the_key_file(name, include, tmp_path):
    cfg = CASES[name]
    parts = make_particles(cfg, seed=5, v_sd=1e-3, random_orientation=True)
    keys, udf = str(tmp_path / "in.keys"), str(tmp_path / "in.udf")
    write_udf_keys(keys, cfg, parts)
    write_udf(udf, cfg, parts, define_path=str(tmp_path / "define.udf") if include else None)
    rc_k, pk, rk = load(keys, cfg.n_particles, keys=True)
    rc_u, pu, ru = load(udf, cfg.n_particles)
    assert rc_k == 0 and rc_u == 0, N.lib().spm_last_error()
    assert bytes(pk) == bytes(pu)
    np.testing.assert_array_equal(rk, ru)
    assert read_udf(udf) == udf_keys(cfg, parts)


def test_config_from_udf_round_trip(tmp_path):
    cfg = CASES["le_no_rotation"]
    parts = make_particles(cfg, seed=2, v_sd=1e-3)
    path = str(tmp_path / "in.udf")
    write_udf(path, cfg, parts)
    got, gp = config_from_udf(path)
    for f in ("npx", "npy", "npz", "equation", "shear_rate", "n_particles", "a", "a_xi", "dt", "lj_powers",
              "lj_truncate", "rotation", "fix_cell", "gts", "num_snap"):
        assert getattr(got, f) == getattr(cfg, f), f
    np.testing.assert_array_equal(gp["x"], parts["x"])
    np.testing.assert_array_equal(gp["v"], parts["v"])
    # ROTATION OFF: the orientation is the identity (init_particle.cxx:369-374)
    np.testing.assert_array_equal(gp["q"], np.tile([1.0, 0, 0, 0], (cfg.n_particles, 1)))


def test_user_specify_quaternions_are_normalised(tmp_path):
    cfg = CASES["ns"]
    parts = make_particles(cfg, seed=8, random_orientation=True)
    parts["q"] = parts["q"] * np.array([[1.5], [0.5], [2.0]])
    path = str(tmp_path / "in.udf")
    write_udf(path, cfg, parts)
    rc, _, rec = load(path, cfg.n_particles)
    assert rc == 0
    q = parts["q"]
    inv = 1.0 / np.sqrt(q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1] + q[:, 2] * q[:, 2] + q[:, 3] * q[:, 3])
    np.testing.assert_array_equal(rec[:, 18:22], q * inv[:, None])
    np.testing.assert_array_equal(rec[:, 22:26], rec[:, 18:22])


# ---------------------------------------------------------------------------
# uniform_random placement and random orientation
# ---------------------------------------------------------------------------
def _glibc_init(cfg, orientation):
    """Init_Particle's uniform_random branch and orientation, drawn from the
    C library's own rand() after srand(10)."""
    libc = C.CDLL("libc.so.6")
    libc.srand(10)
    rmax = 2147483647.0
    L = [float(1 << n) * cfg.dx for n in (cfg.npx, cfg.npy, cfg.npz)]
    overlap = (2.0 * (cfg.a * cfg.dx)) * 1.05
    x = []
    for i in range(cfg.n_particles):
        while True:
            c = [libc.rand() / rmax * L[d] for d in range(3)]
            ok = True
            for xj in x:
                s2 = 0.0
                for d in range(3):
                    r = xj[d] - c[d]
                    q = r / L[d]
                    r -= float(int(q + 0.5) if q >= 0 else int(q - 0.5)) * L[d]
                    s2 += r * r
                if math.sqrt(s2) <= overlap:
                    ok = False
                    break
            if ok:
                break
        x.append(c)

    def ra():
        return 2.0 * (libc.rand() - rmax * 0.5) / rmax

    def circle():
        while True:
            u, v = ra(), ra()
            if u * u + v * v <= 1:
                return u, v

    q = []
    for _ in range(cfg.n_particles):
        if orientation == "random" and cfg.rotation:
            u0, u1 = circle()
            u2, u3 = circle()
            s = math.sqrt((1.0 - (u0 * u0 + u1 * u1)) / (u2 * u2 + u3 * u3))
            q.append([u0, u1, u2 * s, u3 * s])
        else:
            q.append([1.0, 0.0, 0.0, 0.0])
    return np.array(x), np.array(q)


def _uniform_random_keys(cfg, orientation, path):
    zeros = {name: np.zeros((cfg.n_particles, w)) for name, w in (("x", 3), ("v", 3), ("q", 4), ("omega", 3))}
    k = udf_keys(cfg, zeros)
    k = {a: b for a, b in k.items() if ".user_specify.Particles[" not in a}
    k["switch.INIT_distribution.type"] = "uniform_random"
    k["switch.INIT_orientation"] = orientation
    with open(path, "w") as f:
        f.write("".join(f"{a} = {b}\n" for a, b in k.items()))


@pytest.mark.parametrize("orientation", ["random", "space_align", "user_specify"])
@pytest.mark.parametrize("grid", [4, 7])
def test_uniform_random_follows_glibc_rand(orientation, grid, tmp_path):
    # 16^3 box: fewer than 3 cells of the overlap length per axis (all
    # pairs tested); 128^3: the cell grid
    cfg = SPMConfig(npx=grid, npy=grid, npz=grid, n_particles=3 if grid == 4 else 400, a=3.0, a_xi=2.0)
    path = str(tmp_path / "in.keys")
    _uniform_random_keys(cfg, orientation, path)
    rc, _, rec = load(path, cfg.n_particles, keys=True)
    assert rc == 0, N.lib().spm_last_error()
    x, q = _glibc_init(cfg, orientation)
    np.testing.assert_array_equal(rec[:, 0:3], x)
    np.testing.assert_array_equal(rec[:, 3:6], x)
    np.testing.assert_array_equal(rec[:, 18:22], q)
    np.testing.assert_array_equal(rec[:, 6:9], 0.0)


@pytest.mark.skipif(not ref_runner.available(), reason="oracle/_ref is not built")
def test_uniform_random_matches_the_reference_program(tmp_path):
    cfg = SPMConfig(npx=5, npy=5, npz=5, n_particles=6, a=3.0, a_xi=2.0, dt=0.05)
    path = str(tmp_path / "in.keys")
    _uniform_random_keys(cfg, "random", path)
    rc, _, rec = load(path, cfg.n_particles, keys=True)
    assert rc == 0
    dump = str(tmp_path / "d.bin")
    ref_runner.run_reference(path, dump, fields_every=0, timeout=300)
    f0 = ref_runner.read_dump(dump)["frames"][0]
    assert f0["ts"] == 0
    np.testing.assert_array_equal(f0["x"], rec[:, 0:3])
    np.testing.assert_array_equal(f0["q"], rec[:, 18:22])


def test_uniform_random_gives_up_when_the_box_is_full(tmp_path):
    cfg = SPMConfig(npx=3, npy=3, npz=3, n_particles=40, a=3.0)
    path = str(tmp_path / "in.keys")
    _uniform_random_keys(cfg, "space_align", path)
    rc, _, _ = load(path, cfg.n_particles, keys=True)
    assert rc == 1 and b"uniform_random" in N.lib().spm_last_error()


# ---------------------------------------------------------------------------
# reader errors
# ---------------------------------------------------------------------------
SCHEMA = "\\begin{def}\nmesh: {NPX: int NPY: int NPZ: int}\nA: double [L] \"radius\"\nv[]: {x: float}\n\\end{def}\n"


@pytest.mark.parametrize("data,message", [
    ("mesh: {5, 5, 5}\nA: 4.0\nB: 1\n", "not in the schema"),
    ("mesh: {5, 5, 5, 5}\n", "too many values"),
    ("mesh: {5, 5}\n", "expected a value"),
    ("v: {1.0}\n", "expected '['"),
    ("mesh: {5, 5, 5}\n", "unterminated data"),
])
def test_reader_reports_malformed_data(data, message, tmp_path):
    path = str(tmp_path / "bad.udf")
    end = "" if message == "unterminated data" else "\\end{data}\n"
    open(path, "w").write(SCHEMA + "\\begin{data}\n" + data + end)
    need = C.c_size_t()
    assert N.lib().spm_udf_read_keys(path.encode(), None, 0, C.byref(need)) == 1
    assert message.encode() in N.lib().spm_last_error()


def test_reader_arrays_units_comments_and_include(tmp_path):
    (tmp_path / "schema.udf").write_text(
        "\\begin{header}\n\\begin{def}\nEngineType: string\n\\end{def}\n\\begin{data}\nEngineType: \"x\"\n"
        "\\end{data}\n\\end{header}\n\\begin{unit}\n[L]=1[nm]\n\\end{unit}\n\\begin{global_def}\n"
        "class V3:{x: float[unit], y: float[unit], z: float[unit]}[unit]\n"
        "sel: select {'a','b'} \"a comment\"   // trailing comment\n"
        "grid[][]: int\nparts[]: {R: V3 [L], tag: string}\n\\end{global_def}\n")
    path = tmp_path / "in.udf"
    path.write_text("\ufeff// leading byte-order mark and comment\n\\include{\"schema.udf\"}\n\\begin{data}\n"
                    "sel: \"b\"\ngrid: [[1, 2], [3]]\nparts: [{{1.5 2.5 -3.5e-002} \"p0\"}, {{0,0,0},\"p1\"}]\n"
                    "\\end{data}\n", encoding="utf-8")
    kv = read_udf(str(path))
    assert kv == {"sel": "b", "grid[0][0]": "1", "grid[0][1]": "2", "grid[1][0]": "3",
                  "parts[0].R.x": "1.5", "parts[0].R.y": "2.5", "parts[0].R.z": "-3.5e-002", "parts[0].tag": "p0",
                  "parts[1].R.x": "0", "parts[1].R.y": "0", "parts[1].R.z": "0", "parts[1].tag": "p1"}
    need = C.c_size_t()
    assert N.lib().spm_udf_read_keys(str(tmp_path / "missing.udf").encode(), None, 0, C.byref(need)) == 1
    assert b"cannot open" in N.lib().spm_last_error()


# ---------------------------------------------------------------------------
# the reference's own example inputs (only where the reference tree exists)
# ---------------------------------------------------------------------------
def _reference_inputs():
    files = sorted(glob.glob(os.path.join(REFERENCE_TREE, "sample", "input.udf")) +
                   glob.glob(os.path.join(REFERENCE_TREE, "Examples", "*", "*.udf")))
    return [f for f in files if os.path.basename(f) not in ("define.udf", "kapsel_unit.udf")]


@pytest.mark.skipif(not _reference_inputs(), reason="reference tree not present")
def test_every_reference_example_parses_and_in_scope_ones_load():
    loaded = loaded_rigid = 0
    for f in _reference_inputs():
        kv = read_udf(f)
        assert kv["constitutive_eq.type"] and kv["object_type.type"], f
        p = N.SpmParams()
        rc = N.lib().spm_params_from_udf(f.encode(), C.byref(p), None, 0)
        spherical = kv["object_type.type"] == "spherical_particle"
        ps = "object_type.spherical_particle.Particle_spec[0]."
        janus = spherical and kv[ps + "janus_propulsion"] != "OFF"
        eq_ok = kv["constitutive_eq.type"] in ("Navier_Stokes", "Shear_Navier_Stokes") or (
            kv["constitutive_eq.type"] in (EQ_LE, "Electrolyte") and not janus)
        rigid = kv["object_type.type"] == "rigid"
        # pinning, flat walls, Quincke rotation and multipoles are refused when switched on
        switches_off = all(kv.get(k, off) == off for k, off in OUTSIDE_SWITCHES)
        in_scope = eq_ok and (spherical or rigid) and switches_off
        assert (rc == 0) == in_scope, (f, N.lib().spm_last_error())
        if rc == 0:
            loaded += 1
            assert (p.npx, p.npy, p.npz) == tuple(int(kv[f"mesh.NP{a}"]) for a in "XYZ")
            if rigid:
                loaded_rigid += 1
                _check_rigid_keys(kv, p)
            counts = []
            while f"object_type.spherical_particle.Particle_spec[{len(counts)}].Particle_number" in kv:
                counts.append(int(kv[f"object_type.spherical_particle.Particle_spec[{len(counts)}].Particle_number"]))
            if not rigid:
                assert p.n_particles == sum(counts)
            if len(counts) > 1 and not rigid:
                assert p.n_species == len(counts) and list(p.species_count)[:len(counts)] == counts
                for i in range(len(counts)):
                    sp = f"object_type.spherical_particle.Particle_spec[{i}]."
                    assert p.species_mass_ratio[i] == float(kv[sp + "MASS_RATIO"])
                    assert p.species_surface_charge[i] == float(kv[sp + "Surface_charge"])
            assert p.a == float(kv["A"]) and p.a_xi == float(kv["A_XI"])
            eq = kv["constitutive_eq.type"]
            assert p.eta == float(kv[f"constitutive_eq.{eq}.ETA"])
            if eq in (EQ_LE, "Shear_Navier_Stokes"):
                ft = kv[f"constitutive_eq.{eq}.External_field.type"]
                assert p.shear_rate == float(kv[f"constitutive_eq.{eq}.External_field.{ft}.Shear_rate"])
                assert p.shear_ac == (ft == "AC")
            if eq == "Electrolyte":
                e = "constitutive_eq.Electrolyte."
                assert p.equation == N.SPM_EQ_ELECTROLYTE and p.dielectric == float(kv[e + "Dielectric_cst"])
                assert p.salt == (kv[e + "Add_salt.type"] == "salt")
                assert p.surface_charge == float(kv["object_type.spherical_particle.Particle_spec[0].Surface_charge"])
                if p.salt:
                    assert p.debye_length == float(kv[e + "Add_salt.salt.Debye_length"])
                    assert list(p.valency) == [float(kv[e + "Add_salt.salt.Valency_positive_ion"]),
                                               float(kv[e + "Add_salt.salt.Valency_negative_ion"])]
            if janus:
                jp = ("OFF", "TUMBLER", "SQUIRMER", "OBSTACLE")[p.janus_propulsion]
                assert jp == kv[ps + "janus_propulsion"]
                assert ("NONE", "X", "Y", "Z")[p.janus_axis] == kv[ps + "janus_axis"]
                if jp == "SQUIRMER":
                    assert p.slip_vel == float(kv[ps + "janus_slip_vel"])
                    assert p.slip_mode == float(kv[ps + "janus_slip_mode"])
                    assert p.slip_tol == float(kv["switch.SLIP_tol"])
                    assert p.slip_iter == int(kv["switch.SLIP_iter"])
            if kv["time_increment.type"] == "manual":
                assert p.dt == float(kv["time_increment.manual.delta_t"])
            elif eq != "Electrolyte":
                # DT = factor / (NU * KMAX2), KMAX2 from the 2/3-rule wavenumbers
                k2 = sum((2 * math.pi / ((1 << n) * p.dx) * (((1 << n) + 2) // 3)) ** 2 for n in (p.npx, p.npy, p.npz))
                assert p.dt == pytest.approx(float(kv["time_increment.auto.factor"]) / (p.eta / p.rho * k2), rel=1e-14)
    assert loaded >= 4 and loaded_rigid >= 6


def _check_rigid_keys(kv, p):
    """Rigid_spec[] (input.cxx:1583-1700), switch.free_rigid (input.cxx:1961-2008) and the rigid gravity
    (md_force.cxx:317-322) as the parser stores them."""
    spec = "object_type.rigid.Rigid_spec[{}]."
    nsp = 0
    while spec.format(nsp) + "Beads_number" in kv:
        nsp += 1
    assert p.rigid == 1 and p.n_species == (nsp if nsp > 1 else 0)
    total = 0
    for s in range(nsp):
        sp = spec.format(s)
        beads, count = int(kv[sp + "Beads_number"]), int(kv[sp + "Chain_number"])
        assert (p.rigid_beads[s], p.rigid_count[s]) == (beads, count)
        total += beads * count
        free = [kv[sp + "Rigid_motion"] == "free"] * 6
        dof = 0
        while kv.get("switch.free_rigid.type") == "YES" and f"switch.free_rigid.YES.DOF[{dof}].spec_id" in kv:
            t = f"switch.free_rigid.YES.DOF[{dof}]."
            if int(kv[t + "spec_id"]) == s:
                free = [kv[t + k + "." + a] == "YES" for k in ("vel", "omega") for a in "xyz"]
            dof += 1
        assert [bool(x) for x in p.rigid_free[s]] == free
        for d, a in enumerate("xyz"):
            assert p.rigid_velocity[s][d] == float(kv[sp + "Rigid_velocity." + a])
            assert p.rigid_omega[s][d] == float(kv[sp + "Rigid_omega." + a])
    assert p.n_particles == total
    g = [0.0] * 3
    if float(kv["gravity.G"]) != 0.0:
        g["XYZ".index(kv["gravity.G_direction"][1])] = float(kv["gravity.G"])
    assert list(p.rigid_gravity) == g


def test_janus_config_round_trip(tmp_path):
    for name in ("squirmer", "tumbler", "two_species"):
        cfg = CASES[name]
        parts = make_particles(cfg, seed=3, random_orientation=True)
        path = str(tmp_path / f"{name}.udf")
        write_udf(path, cfg, parts)
        got, _ = config_from_udf(path)
        for f in ("janus_axis", "janus_propulsion", "janus_force", "janus_torque", "slip_vel", "slip_mode",
                  "rotlet_c1", "rotlet_c2", "slip_tol", "slip_iter", "species"):
            assert getattr(got, f) == getattr(cfg, f), (name, f)
