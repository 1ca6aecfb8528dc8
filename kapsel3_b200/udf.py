"""UDF-driven run description for the SPM step.

KAPSEL reads every run parameter from a UDF file through OCTA's `UDFManager`
(input.cxx:677-2556).  That library is not available here, so a run is
described by a flat *key file*: one ``<udf.path> = <value>`` line per UDF
field the reference reads, keyed by exactly the paths `Gourmet_file_io` asks
for (e.g. ``mesh.NPX``, ``constitutive_eq.Navier_Stokes.ETA``,
``switch.INIT_distribution.user_specify.Particles[3].R.x``).  The same file
drives both the reference program (through its UDF stand-in) and this
package's C++ loader (`spm_config_from_udf_keys`), so both consume identical
inputs.

`SPMConfig` carries the physical parameters the step needs; `derived()`
reproduces the derived globals of `Set_global_parameters`
(input.cxx:425-604).  `make_particles` is the seeded initial-condition
generator used for every parity and benchmark case.
"""
from __future__ import annotations

import dataclasses
import math
import os
import re
from typing import Dict, Optional

import numpy as np

EQ_NS = "Navier_Stokes"
EQ_LE = "Shear_Navier_Stokes_Lees_Edwards"
EQ_EL = "Electrolyte"
EQ_SNS = "Shear_Navier_Stokes"


@dataclasses.dataclass
class SPMConfig:
    """Parameters of one SPM run (the UDF fields the step reads)."""

    npx: int = 5                 # mesh.NPX: NX = 1 << NPX (input.cxx:1752)
    npy: int = 5
    npz: int = 5
    dx: float = 1.0              # constitutive_eq.<type>.DX
    rho: float = 1.0
    eta: float = 1.0
    kbt: float = 0.0
    alpha_v: float = 1.0
    alpha_o: float = 1.0
    equation: str = EQ_NS        # constitutive_eq.type
    shear_rate: float = 0.0      # ...Lees_Edwards / Shear_Navier_Stokes .External_field.<DC|AC>.Shear_rate
    shear_ac: bool = False       # Shear_Navier_Stokes: AC oscillatory shear (else DC)
    shear_frequency: float = 0.0  # Shear_Navier_Stokes AC: Frequency
    n_particles: int = 2         # Particle_spec[0].Particle_number
    mass_ratio: float = 1.0
    a: float = 4.0               # A (radius in units of DX)
    a_xi: float = 2.0            # A_XI (interface thickness in units of DX)
    epsilon: float = 1.0         # EPSILON
    lj_powers: str = "12:6"
    lj_truncate: str = "ON"
    rotation: bool = True
    fix_cell: tuple = (True, True, True)
    dt: float = 0.05             # time_increment.manual.delta_t
    gts: int = 1                 # output.GTS
    num_snap: int = 1            # output.Num_snap (MSTEP = GTS*Num_snap)
    body_force: tuple = (0.0, 0.0, 0.0)  # constant force on every particle
    # Electrolyte (constitutive_eq.Electrolyte, input.cxx:834-930)
    dielectric: float = 1.0      # Dielectric_cst
    salt: bool = False           # Add_salt: salt (two ion species) or saltfree (counterions)
    init_pb: bool = False        # INIT_profile: Poisson_Boltzmann or Uniform
    valency: tuple = (-1.0, 0.0)  # saltfree: (counterion, -); salt: (positive, negative)
    onsager: tuple = (1.0, 1.0)  # Onsager coefficients in the same order
    debye_length: float = 10.0   # salt: Debye_length
    surface_charge: float = 0.0  # Particle_spec[0].Surface_charge
    e_field: str = "OFF"         # Electric_field: OFF, DC or AC
    e_ext: tuple = (0.0, 0.0, 0.0)  # Ex, Ey, Ez
    e_frequency: float = 0.0     # AC Frequency
    # Janus particles (Particle_spec[0].janus_*, input.cxx:1403-1470)
    janus_axis: str = "NONE"           # NONE, X, Y, Z
    janus_propulsion: str = "OFF"      # OFF, TUMBLER, SQUIRMER, OBSTACLE
    janus_force: tuple = (0.0, 0.0, 0.0)   # TUMBLER, body frame
    janus_torque: tuple = (0.0, 0.0, 0.0)  # TUMBLER, body frame
    slip_vel: float = 0.0              # SQUIRMER: janus_slip_vel (B1)
    slip_mode: float = 0.0             # SQUIRMER: janus_slip_mode (alpha = B2/B1)
    rotlet_c1: float = 0.0             # SQUIRMER: janus_rotlet_C1
    rotlet_c2: float = 0.0             # SQUIRMER: janus_rotlet_dipole_C2
    slip_tol: float = 1e-5             # switch.SLIP_tol
    slip_iter: int = 100               # switch.SLIP_iter
    # Several particle species: ((count, MASS_RATIO, Surface_charge), ...) for Particle_spec[0..], the
    # counts adding up to n_particles (species 0 first); empty: one species (n_particles, mass_ratio,
    # surface_charge)
    species: tuple = ()
    # Rigid bodies (object_type.type = rigid, Rigid_spec[0..]): one entry per rigid species,
    # (Beads_number, Chain_number, MASS_RATIO, Rigid_motion "free"/"fix", Rigid_velocity (3),
    # Rigid_omega (3)); n_particles is then the sum of Beads_number * Chain_number.  rigid_dof
    # overrides the degrees of freedom (switch.free_rigid): ((spec_id, (vx, vy, vz), (wx, wy, wz)), ...)
    # with booleans.
    rigid: tuple = ()
    rigid_dof: tuple = ()
    rigid_gravity: tuple = (0.0, 0.0, 0.0)  # gravity.G placed on the axis of gravity.G_direction

    # ------------------------------------------------------------------
    @property
    def shape(self):
        return (1 << self.npx, 1 << self.npy, 1 << self.npz)

    def derived(self) -> Dict[str, float]:
        """Derived globals, as `Set_global_parameters` (input.cxx:425-604)
        and the particle section of `Gourmet_file_io` (input.cxx:1701-1707,
        1807-1827) compute them."""
        nx, ny, nz = self.shape
        radius = self.a * self.dx
        xi = self.a_xi * self.dx
        sigma = 2.0 * radius
        mass = self.mass_ratio * self.rho * 4.0 / 3.0 * math.pi * radius ** 3
        moi = 2.0 / 5.0 * mass * radius ** 2
        pw = {"12:6": 6.0, "24:12": 12.0, "36:18": 18.0}[self.lj_powers]
        if self.lj_truncate == "ON":
            a_r_cutoff = 2.0 ** (1.0 / pw)
        elif self.lj_truncate == "OFF":
            a_r_cutoff = min(min(nx, ny, nz) * self.dx * 0.5 / sigma, 2.5)
        else:
            a_r_cutoff = 0.0
        if self.equation == EQ_LE:
            lj_dia = min((sigma + xi) / 2.0 ** (1.0 / pw), sigma)
        else:
            lj_dia = sigma
        return dict(
            NX=nx, NY=ny, NZ=nz, HNZ_=nz // 2 + 1, NZ_=2 * (nz // 2 + 1),
            TRN_X=(nx + 2) // 3, TRN_Y=(ny + 2) // 3, TRN_Z=(nz + 2) // 3,
            RADIUS=radius, XI=xi, HXI=0.5 * xi, SIGMA=sigma,
            MASS=mass, IMASS=1.0 / mass, MOI=moi, IMOI=1.0 / moi,
            NU=self.eta / self.rho, DX3=self.dx ** 3,
            LX=nx * self.dx, LY=ny * self.dx, LZ=nz * self.dx,
            WAVE_X=2 * math.pi / (nx * self.dx), WAVE_Y=2 * math.pi / (ny * self.dx),
            WAVE_Z=2 * math.pi / (nz * self.dx),
            A_R_cutoff=a_r_cutoff, LJ_dia=lj_dia,
            Ivolume=1.0 / (nx * ny * nz * self.dx ** 3),
        )

    @property
    def mstep(self) -> int:
        return self.gts * self.num_snap


def make_particles(cfg: SPMConfig, seed: int, v_sd: float = 0.0,
                   random_orientation: bool = False,
                   min_dist_factor: float = 1.05,
                   max_tries: int = 200000) -> Dict[str, np.ndarray]:
    """Seeded, non-overlapping uniform positions (random sequential addition
    with the reference's overlap length 1.05*SIGMA, init_particle.cxx:65-82),
    optional random unit quaternions and Gaussian velocities.  Deterministic
    for a given seed (numpy PCG64)."""
    rng = np.random.default_rng(seed)
    d = cfg.derived()
    L = np.array([d["LX"], d["LY"], d["LZ"]])
    rmin = min_dist_factor * d["SIGMA"]
    n = cfg.n_particles
    x = np.zeros((n, 3))
    tries = 0
    for i in range(n):
        while True:
            tries += 1
            if tries > max_tries:
                raise ValueError(f"cannot place {n} particles of radius {cfg.a} in {cfg.shape}")
            c = rng.random(3) * L
            if i == 0:
                break
            dd = x[:i] - c
            dd -= np.rint(dd / L) * L
            if np.min(np.sqrt((dd ** 2).sum(1))) > rmin:
                break
        x[i] = c
    v = rng.normal(0.0, v_sd, size=(n, 3)) if v_sd > 0 else np.zeros((n, 3))
    if random_orientation:
        q = rng.normal(size=(n, 4))
        q /= np.linalg.norm(q, axis=1, keepdims=True)
    else:
        q = np.tile(np.array([1.0, 0.0, 0.0, 0.0]), (n, 1))
    omega = np.zeros((n, 3))
    return dict(x=x, v=v, q=q, omega=omega)


def make_rigid_bodies(cfg: SPMConfig, seed: int, spacing_factor: float = 1.2, min_dist_factor: float = 1.05,
                      straddle: bool = False, max_tries: int = 20000) -> Dict[str, np.ndarray]:
    """Seeded bead positions of cfg.rigid's bodies, species after species and
    body after body (the order of Rigid_spec[] and Particle_RigidID): each
    body is a random walk of beads spacing_factor * A apart whose turns keep
    its inertia tensor free of equal eigenvalues.  The coordinates are not
    wrapped into the box (a body may reach over its edge, and with `straddle`
    the first body does), as user_specify inputs give them.  Beads of
    different bodies stay min_dist_factor * SIGMA apart (periodic images
    included).  Velocities and orientations are zero and the identity: the
    bodies' motion comes from Rigid_velocity / Rigid_omega."""
    rng = np.random.default_rng(seed)
    d = cfg.derived()
    L = np.array([d["LX"], d["LY"], d["LZ"]])
    step = spacing_factor * cfg.a
    rmin = min_dist_factor * d["SIGMA"]
    bodies = []
    tries = 0
    for beads, count, *_ in cfg.rigid:
        for _ in range(int(count)):
            while True:
                tries += 1
                if tries > max_tries:
                    raise ValueError(f"cannot place the rigid bodies in {cfg.shape}")
                pos = [rng.random(3) * L]
                if straddle and not bodies:
                    pos = [L * np.array([0.98, 0.5, 0.5])]
                u = rng.normal(size=3)
                u /= np.linalg.norm(u)
                for k in range(1, int(beads)):
                    # turn by 50-80 degrees about a random axis from the previous direction
                    w = np.cross(u, rng.normal(size=3))
                    w /= np.linalg.norm(w)
                    t = np.deg2rad(rng.uniform(50.0, 80.0))
                    u = np.cos(t) * u + np.sin(t) * w
                    pos.append(pos[-1] + step * u)
                body = np.array(pos)
                ok = True
                for other in bodies:
                    dd = body[:, None, :] - other[None, :, :]
                    dd -= np.rint(dd / L) * L
                    if np.sqrt((dd ** 2).sum(-1)).min() <= rmin:
                        ok = False
                        break
                if ok:
                    bodies.append(body)
                    break
    x = np.concatenate(bodies) if bodies else np.zeros((0, 3))
    n = len(x)
    return dict(x=x, v=np.zeros((n, 3)), q=np.tile(np.array([1.0, 0.0, 0.0, 0.0]), (n, 1)),
                omega=np.zeros((n, 3)))


def _fmt(v) -> str:
    if isinstance(v, bool):
        return "ON" if v else "OFF"
    if isinstance(v, float):
        return repr(v)
    return str(v)


def udf_keys(cfg: SPMConfig, particles: Dict[str, np.ndarray],
             out_dir: str = "/tmp/kapsel_avs") -> Dict[str, str]:
    """All UDF paths the reference reads for a spherical-particle spectral
    run, with this run's values."""
    eq = cfg.equation
    k: Dict[str, str] = {}
    k["resume.Calculation"] = "NEW"
    k["resume.CONTINUE.Saved_Data.jikan.ts"] = "0"
    k["constitutive_eq.type"] = eq
    base = f"constitutive_eq.{eq}"
    scalars = [("DX", cfg.dx), ("RHO", cfg.rho), ("ETA", cfg.eta), ("kBT", cfg.kbt)]
    if eq != EQ_EL:
        scalars += [("alpha_v", cfg.alpha_v), ("alpha_o", cfg.alpha_o)]
    for name, val in scalars:
        k[f"{base}.{name}"] = _fmt(float(val))
    if eq == EQ_EL:
        k[f"{base}.Dielectric_cst"] = _fmt(float(cfg.dielectric))
        k[f"{base}.INIT_profile"] = "Poisson_Boltzmann" if cfg.init_pb else "Uniform"
        if cfg.salt:
            k[f"{base}.Add_salt.type"] = "salt"
            s = f"{base}.Add_salt.salt"
            k[f"{s}.Valency_positive_ion"] = _fmt(float(cfg.valency[0]))
            k[f"{s}.Valency_negative_ion"] = _fmt(float(cfg.valency[1]))
            k[f"{s}.Onsager_coeff_positive_ion"] = _fmt(float(cfg.onsager[0]))
            k[f"{s}.Onsager_coeff_negative_ion"] = _fmt(float(cfg.onsager[1]))
            k[f"{s}.Debye_length"] = _fmt(float(cfg.debye_length))
        else:
            k[f"{base}.Add_salt.type"] = "saltfree"
            k[f"{base}.Add_salt.saltfree.Valency_counterion"] = _fmt(float(cfg.valency[0]))
            k[f"{base}.Add_salt.saltfree.Onsager_coeff_counterion"] = _fmt(float(cfg.onsager[0]))
        if cfg.e_field == "OFF":
            k[f"{base}.Electric_field.type"] = "OFF"
        else:
            k[f"{base}.Electric_field.type"] = "ON"
            k[f"{base}.Electric_field.ON.type"] = cfg.e_field
            f = f"{base}.Electric_field.ON.{cfg.e_field}"
            for c, v in zip(("Ex", "Ey", "Ez"), cfg.e_ext):
                k[f"{f}.{c}"] = _fmt(float(v))
            if cfg.e_field == "AC":
                k[f"{f}.Frequency"] = _fmt(float(cfg.e_frequency))
    if eq == EQ_LE:
        k[f"{base}.External_field.type"] = "DC"
        k[f"{base}.External_field.DC.Shear_rate"] = _fmt(float(cfg.shear_rate))
    if eq == EQ_SNS:
        ft = "AC" if cfg.shear_ac else "DC"
        k[f"{base}.External_field.type"] = ft
        k[f"{base}.External_field.{ft}.Shear_rate"] = _fmt(float(cfg.shear_rate))
        if cfg.shear_ac:
            k[f"{base}.External_field.AC.Frequency"] = _fmt(float(cfg.shear_frequency))
    k["object_type.type"] = "rigid" if cfg.rigid else "spherical_particle"
    for i, (beads, count, mr, motion, vel, om) in enumerate(cfg.rigid):
        ri = f"object_type.rigid.Rigid_spec[{i}]"
        k[f"{ri}.Beads_number"] = str(int(beads))
        k[f"{ri}.Chain_number"] = str(int(count))
        k[f"{ri}.MASS_RATIO"] = _fmt(float(mr))
        k[f"{ri}.Surface_charge"] = _fmt(0.0)
        k[f"{ri}.Rigid_motion"] = motion
        for c, v, w in zip("xyz", vel, om):
            k[f"{ri}.Rigid_velocity.{c}"] = _fmt(float(v))
            k[f"{ri}.Rigid_omega.{c}"] = _fmt(float(w))
    if cfg.rigid:
        k["switch.free_rigid.type"] = "YES" if cfg.rigid_dof else "NO"
        for i, (sid, vflags, wflags) in enumerate(cfg.rigid_dof):
            di = f"switch.free_rigid.YES.DOF[{i}]"
            k[f"{di}.spec_id"] = str(int(sid))
            for c, fv, fw in zip("xyz", vflags, wflags):
                k[f"{di}.vel.{c}"] = "YES" if fv else "NO"
                k[f"{di}.omega.{c}"] = "YES" if fw else "NO"
    ps = "object_type.spherical_particle.Particle_spec[0]"
    spec = cfg.species if len(cfg.species) > 1 else ((cfg.n_particles, cfg.mass_ratio, cfg.surface_charge),)
    for i, (cnt, mr, q) in enumerate(spec):
        pi = f"object_type.spherical_particle.Particle_spec[{i}]"
        k[f"{pi}.Particle_number"] = str(int(cnt))
        k[f"{pi}.MASS_RATIO"] = _fmt(float(mr))
        k[f"{pi}.Surface_charge"] = _fmt(float(q))
        if i > 0:
            k[f"{pi}.janus_axis"] = "NONE"
            k[f"{pi}.janus_propulsion"] = "OFF"
    k[f"{ps}.janus_axis"] = cfg.janus_axis
    k[f"{ps}.janus_propulsion"] = cfg.janus_propulsion
    if cfg.janus_propulsion == "TUMBLER":
        for c, f, t in zip("xyz", cfg.janus_force, cfg.janus_torque):
            k[f"{ps}.janus_force.{c}"] = _fmt(float(f))
            k[f"{ps}.janus_torque.{c}"] = _fmt(float(t))
    if cfg.janus_propulsion == "SQUIRMER":
        k[f"{ps}.janus_slip_vel"] = _fmt(float(cfg.slip_vel))
        k[f"{ps}.janus_slip_mode"] = _fmt(float(cfg.slip_mode))
        if cfg.rotlet_c1 or cfg.rotlet_c2:
            k[f"{ps}.janus_rotlet_C1"] = _fmt(float(cfg.rotlet_c1))
            k[f"{ps}.janus_rotlet_dipole_C2"] = _fmt(float(cfg.rotlet_c2))
    k["A_XI"] = _fmt(float(cfg.a_xi))
    k["A"] = _fmt(float(cfg.a))
    # Gravity is never used as such (MASS_RATIO=1); a nonzero G only makes the
    # reference call Add_f_gravity, where the oracle build injects body_force.
    has_bf = any(f != 0.0 for f in cfg.body_force)
    k["gravity.G"] = "1.0" if has_bf else "0.0"
    k["gravity.G_direction"] = "-X"
    if cfg.rigid and any(g != 0.0 for g in cfg.rigid_gravity):  # real gravity on the bodies
        d = next(i for i, g in enumerate(cfg.rigid_gravity) if g != 0.0)
        k["gravity.G"] = _fmt(float(cfg.rigid_gravity[d]))
        k["gravity.G_direction"] = "-" + "XYZ"[d]
    k["EPSILON"] = _fmt(float(cfg.epsilon))
    k["LJ_powers"] = cfg.lj_powers
    k["mesh.NPX"], k["mesh.NPY"], k["mesh.NPZ"] = str(cfg.npx), str(cfg.npy), str(cfg.npz)
    k["time_increment.type"] = "manual"
    k["time_increment.manual.delta_t"] = _fmt(float(cfg.dt))
    k["switch.ROTATION"] = _fmt(bool(cfg.rotation))
    k["switch.LJ_truncate"] = cfg.lj_truncate
    k["switch.INIT_distribution.type"] = "user_specify"
    k["switch.INIT_orientation"] = "user_specify"
    k["switch.SLIP_tol"] = _fmt(float(cfg.slip_tol))
    k["switch.SLIP_iter"] = str(int(cfg.slip_iter))
    for d, on in zip("xyz", cfg.fix_cell):
        k[f"switch.FIX_CELL.{d}"] = _fmt(bool(on))
    k["switch.pin.type"] = "NO"
    k["output.GTS"] = str(cfg.gts)
    k["output.Num_snap"] = str(cfg.num_snap)
    k["output.AVS"] = "ON"
    k["output.ON.Out_dir"] = out_dir
    k["output.ON.Out_name"] = "frame"
    k["output.ON.FileType"] = "BINARY"
    k["output.UDF"] = "OFF"
    up = "switch.INIT_distribution.user_specify.Particles"
    x, v, q, w = particles["x"], particles["v"], particles["q"], particles["omega"]
    for i in range(cfg.n_particles):
        t = f"{up}[{i}]"
        for j, c in enumerate("xyz"):
            k[f"{t}.R.{c}"] = repr(float(x[i, j]))
            k[f"{t}.v.{c}"] = repr(float(v[i, j]))
            k[f"{t}.omega.{c}"] = repr(float(w[i, j]))
        for j in range(4):
            k[f"{t}.q.q{j}"] = repr(float(q[i, j]))
    return k


def write_udf_keys(path: str, cfg: SPMConfig, particles: Dict[str, np.ndarray],
                   out_dir: Optional[str] = None) -> None:
    keys = udf_keys(cfg, particles, out_dir or "/tmp/kapsel_avs")
    with open(path, "w") as f:
        for kk, vv in keys.items():
            f.write(f"{kk} = {vv}\n")


def read_udf_keys(path: str) -> Dict[str, str]:
    out: Dict[str, str] = {}
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0]
            if "=" not in line:
                continue
            kk, vv = line.split("=", 1)
            out[kk.strip()] = vv.strip()
    return out


# ---------------------------------------------------------------------------
# UDF files in the OCTA format (the format KAPSEL's input.udf uses)
# ---------------------------------------------------------------------------
_INT = re.compile(r"[+-]?\d+$")


def _leaf_type(v: str) -> str:
    if _INT.match(v):
        return "int"
    try:
        float(v)
        return "double"
    except ValueError:
        return "string"


def _udf_tree(keys: Dict[str, str]) -> dict:
    """Nests flat UDF paths ("a.b[2].c") into dicts (structs) and lists
    (arrays), keeping the order in which fields first appear."""
    root: dict = {}
    for path, val in keys.items():
        segs = path.split(".")
        node = root
        for n, seg in enumerate(segs):
            name, *idx = seg.replace("]", "").split("[")
            last = n == len(segs) - 1
            if not idx:
                if last:
                    node[name] = val
                else:
                    node = node.setdefault(name, {})
                continue
            arr = node.setdefault(name, [])
            for m, i in enumerate(int(i) for i in idx):
                while len(arr) <= i:
                    arr.append(None)
                if m < len(idx) - 1:
                    arr[i] = arr[i] if arr[i] is not None else []
                    arr = arr[i]
                elif last:
                    arr[i] = val
                else:
                    arr[i] = arr[i] if arr[i] is not None else {}
                    node = arr[i]
    return root


def _udf_type(node) -> tuple:
    """(array depth, type text) of a tree node; arrays take their element
    type from element 0."""
    depth = 0
    while isinstance(node, list):
        depth += 1
        node = next((e for e in node if e is not None), "")
    if isinstance(node, dict):
        body = " ".join(f"{k}{'[]' * d}: {t}" for k, (d, t) in ((k, _udf_type(v)) for k, v in node.items()))
        return depth, "{" + body + "}"
    return depth, _leaf_type(node)


def _udf_value(node) -> str:
    if isinstance(node, list):
        return "[" + ", ".join(_udf_value(e) for e in node) + "]"
    if isinstance(node, dict):
        return "{" + ", ".join(_udf_value(v) for v in node.values()) + "}"
    return node if _leaf_type(node) != "string" else '"' + node + '"'


def udf_text(keys: Dict[str, str]) -> tuple:
    """(schema, data) text of a self-describing UDF file holding `keys`:
    a \\begin{def} block declaring every top-level field and a
    \\begin{data} block with the values in schema order."""
    tree = _udf_tree(keys)
    schema = ["\\begin{def}"]
    data = ["\\begin{data}"]
    for name, node in tree.items():
        d, t = _udf_type(node)
        schema.append(f"{name}{'[]' * d}: {t}")
        data.append(f"{name}: {_udf_value(node)}")
    schema.append("\\end{def}")
    data.append("\\end{data}")
    return "\n".join(schema) + "\n", "\n".join(data) + "\n"


def write_udf_from_keys(path: str, keys: Dict[str, str]) -> None:
    """Writes a key map (e.g. a restart key file of spm_save_restart, read
    with read_udf_keys) as a self-describing UDF file."""
    schema, data = udf_text(keys)
    with open(path, "w") as f:
        f.write("// written by kapsel3_b200.udf.write_udf_from_keys\n")
        f.write(schema)
        f.write(data)


def write_udf(path: str, cfg: SPMConfig, particles: Dict[str, np.ndarray],
              out_dir: Optional[str] = None, define_path: Optional[str] = None) -> None:
    """Writes the run as a UDF input file (the paths of `udf_keys`).  With
    `define_path` the schema goes to that file and the input file
    \\include's it, as KAPSEL's input.udf includes define.udf."""
    schema, data = udf_text(udf_keys(cfg, particles, out_dir or "/tmp/kapsel_avs"))
    with open(path, "w") as f:
        f.write("// SPM run written by kapsel3_b200.udf.write_udf\n")
        if define_path:
            with open(define_path, "w") as g:
                g.write(schema)
            rel = os.path.relpath(define_path, os.path.dirname(os.path.abspath(path)))
            f.write(f'\\include{{"{rel}"}}\n')
        else:
            f.write(schema)
        f.write(data)
