"""Python host mirror of the reference's SPM-step interface, over the C ABI.

`SPMRun` owns one device context.  Its methods carry the reference's names
and argument meaning (Time_evolution_hydro, NS_solver_slavedEuler,
Solenoidal_uk, Make_phi_particle_sum, Make_u_particle_sum, Make_phi_u_particle,
Make_f_particle_dt_sole, Calc_f_hydro_correct_precision, Calc_f_Lennard_Jones);
arrays are numpy float64 in the reference layout:
  * k-space field: complex128 [NX, NY, NZ//2+1] (== double[NX*NY*NZ_])
  * real field:    float64   [NX, NY, NZ]   (padded to NZ_ at the boundary)
  * particles:     dict of [Np, 3] / [Np, 4] arrays, or the packed
                   [Np, SPM_PARTICLE_WORDS] record array of the C ABI.
Errors raise `SpmError` with the library's message (the reference exits).
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional, Tuple

import numpy as np

from . import _native as N
from .udf import EQ_EL, EQ_LE, EQ_NS, EQ_SNS, SPMConfig, read_udf_keys

RECORD = [("x", 3), ("x_nopbc", 3), ("v", 3), ("v_old", 3), ("omega", 3), ("omega_old", 3),
          ("q", 4), ("q_old", 4), ("f_hydro", 3), ("f_hydro_previous", 3),
          ("torque_hydro", 3), ("torque_hydro_previous", 3), ("fr", 3), ("fr_previous", 3)]


def pack_particles(p: Dict[str, np.ndarray], n: int) -> np.ndarray:
    rec = np.zeros((n, N.SPM_PARTICLE_WORDS))
    c = 0
    for name, w in RECORD:
        if name in p:
            rec[:, c:c + w] = np.asarray(p[name], dtype=float).reshape(n, w)
        elif name == "x_nopbc" and "x" in p:
            rec[:, c:c + w] = np.asarray(p["x"], dtype=float)
        elif name == "q_old" and "q" in p:
            rec[:, c:c + w] = np.asarray(p["q"], dtype=float)
        elif name in ("q", "q_old"):
            rec[:, c] = 1.0
        c += w
    return rec


def unpack_particles(rec: np.ndarray) -> Dict[str, np.ndarray]:
    out, c = {}, 0
    for name, w in RECORD:
        out[name] = rec[:, c:c + w].copy()
        c += w
    return out


def params_from_config(cfg: SPMConfig, precision: int = N.SPM_PREC_FP64,
                       mt_seed: int = 0) -> N.SpmParams:
    L = N.lib()
    p = N.SpmParams()
    N.check(L.spm_params_default(C.byref(p)), "spm_params_default")
    p.npx, p.npy, p.npz = cfg.npx, cfg.npy, cfg.npz
    p.dx, p.rho, p.eta, p.kbt = cfg.dx, cfg.rho, cfg.eta, cfg.kbt
    p.alpha_v, p.alpha_o = cfg.alpha_v, cfg.alpha_o
    p.equation = {EQ_LE: N.SPM_EQ_LEES_EDWARDS, EQ_EL: N.SPM_EQ_ELECTROLYTE,
                  EQ_SNS: N.SPM_EQ_SHEAR_NAVIER_STOKES}.get(cfg.equation, N.SPM_EQ_NAVIER_STOKES)
    p.shear_ac, p.shear_frequency = int(cfg.shear_ac), float(cfg.shear_frequency)
    p.shear_rate = cfg.shear_rate
    p.n_particles = cfg.n_particles
    p.mass_ratio = cfg.mass_ratio
    p.a, p.a_xi = cfg.a, cfg.a_xi
    p.epsilon = cfg.epsilon
    p.lj_powers = {"12:6": 0, "24:12": 1, "36:18": 2}[cfg.lj_powers]
    p.lj_truncate = {"ON": 1, "OFF": 0, "NONE": -1}[cfg.lj_truncate]
    p.rotation = 1 if cfg.rotation else 0
    for d in range(3):
        p.fix_cell[d] = 1 if cfg.fix_cell[d] else 0
        p.body_force[d] = float(cfg.body_force[d])
    p.dt = cfg.dt
    p.precision = precision
    p.mt_seed = mt_seed
    p.dielectric, p.salt, p.init_pb = cfg.dielectric, int(cfg.salt), int(cfg.init_pb)
    for n in range(2):
        p.valency[n], p.onsager[n] = float(cfg.valency[n]), float(cfg.onsager[n])
    p.debye_length, p.surface_charge = cfg.debye_length, cfg.surface_charge
    p.e_field = {"OFF": 0, "DC": 1, "AC": 2}[cfg.e_field]
    for d in range(3):
        p.e_ext[d] = float(cfg.e_ext[d])
    p.e_frequency = cfg.e_frequency
    p.janus_axis = {"NONE": N.SPM_AXIS_NONE, "X": N.SPM_AXIS_X, "Y": N.SPM_AXIS_Y, "Z": N.SPM_AXIS_Z}[cfg.janus_axis]
    p.janus_propulsion = {"OFF": N.SPM_JANUS_OFF, "TUMBLER": N.SPM_JANUS_TUMBLER, "SQUIRMER": N.SPM_JANUS_SQUIRMER,
                          "OBSTACLE": N.SPM_JANUS_OBSTACLE}[cfg.janus_propulsion]
    for d in range(3):
        p.janus_force[d], p.janus_torque[d] = float(cfg.janus_force[d]), float(cfg.janus_torque[d])
    p.slip_vel, p.slip_mode = cfg.slip_vel, cfg.slip_mode
    p.rotlet_c1, p.rotlet_c2 = cfg.rotlet_c1, cfg.rotlet_c2
    p.slip_tol, p.slip_iter = cfg.slip_tol, int(cfg.slip_iter)
    if len(cfg.species) > 1:
        p.n_species = len(cfg.species)
        for i, (cnt, mr, q) in enumerate(cfg.species):
            p.species_count[i], p.species_mass_ratio[i], p.species_surface_charge[i] = int(cnt), float(mr), float(q)
    if cfg.rigid:
        p.rigid = 1
        if len(cfg.rigid) > 1:
            p.n_species = len(cfg.rigid)
        for i, (beads, count, mr, motion, vel, om) in enumerate(cfg.rigid):
            p.rigid_beads[i], p.rigid_count[i] = int(beads), int(count)
            if len(cfg.rigid) > 1:
                p.species_count[i], p.species_mass_ratio[i] = int(beads) * int(count), float(mr)
            for d in range(6):
                p.rigid_free[i][d] = 1 if motion == "free" else 0
            for d in range(3):
                p.rigid_velocity[i][d], p.rigid_omega[i][d] = float(vel[d]), float(om[d])
        p.mass_ratio = float(cfg.rigid[0][2])
        for d in range(3):
            p.rigid_gravity[d] = float(cfg.rigid_gravity[d])
        for sid, vflags, wflags in cfg.rigid_dof:
            for d in range(3):
                p.rigid_free[sid][d] = 1 if vflags[d] else 0
                p.rigid_free[sid][3 + d] = 1 if wflags[d] else 0
    return p


def read_udf(path: str) -> Dict[str, str]:
    """The data of a UDF input file (KAPSEL's input.udf format, schema from
    its \\include'd define.udf) flattened to {udf.path: value}."""
    L = N.lib()
    need = C.c_size_t()
    N.check(L.spm_udf_read_keys(path.encode(), None, 0, C.byref(need)), "spm_udf_read_keys")
    buf = C.create_string_buffer(need.value)
    N.check(L.spm_udf_read_keys(path.encode(), buf, need.value, C.byref(need)), "spm_udf_read_keys")
    return dict(line.split("=", 1) for line in buf.value.decode().splitlines())


def config_from_udf(path: str) -> Tuple[SPMConfig, Dict[str, np.ndarray]]:
    """Run parameters and initial particles of a UDF input file, as
    Gourmet_file_io and Init_Particle read them (user_specify or
    uniform_random placement; user_specify, random or space_align
    orientation).  A path ending in .keys is read as a key file
    ("udf.path = value" lines, kapsel3_b200.udf.write_udf_keys)."""
    L = N.lib()
    p = N.SpmParams()
    keys = path.endswith(".keys")
    parse = L.spm_params_from_udf_keys if keys else L.spm_params_from_udf
    N.check(parse(path.encode(), C.byref(p), None, 0), "spm_params_from_udf")
    rec = np.zeros((max(p.n_particles, 1), N.SPM_PARTICLE_WORDS))
    N.check(parse(path.encode(), C.byref(p), N.dptr(rec), p.n_particles), "spm_params_from_udf")
    kv = read_udf_keys(path) if keys else read_udf(path)
    cfg = SPMConfig(
        npx=p.npx, npy=p.npy, npz=p.npz, dx=p.dx, rho=p.rho, eta=p.eta, kbt=p.kbt,
        alpha_v=p.alpha_v, alpha_o=p.alpha_o,
        equation={N.SPM_EQ_LEES_EDWARDS: EQ_LE, N.SPM_EQ_ELECTROLYTE: EQ_EL,
                  N.SPM_EQ_SHEAR_NAVIER_STOKES: EQ_SNS}.get(p.equation, EQ_NS),
        shear_ac=bool(p.shear_ac), shear_frequency=p.shear_frequency,
        shear_rate=p.shear_rate, n_particles=p.n_particles, mass_ratio=p.mass_ratio, a=p.a, a_xi=p.a_xi,
        epsilon=p.epsilon, lj_powers=("12:6", "24:12", "36:18")[p.lj_powers],
        lj_truncate={1: "ON", 0: "OFF", -1: "NONE"}[p.lj_truncate], rotation=bool(p.rotation),
        fix_cell=tuple(bool(p.fix_cell[d]) for d in range(3)), dt=p.dt,
        gts=int(kv.get("output.GTS", 1)), num_snap=int(kv.get("output.Num_snap", 1)),
        body_force=tuple(float(p.body_force[d]) for d in range(3)),
        dielectric=p.dielectric, salt=bool(p.salt), init_pb=bool(p.init_pb), valency=tuple(p.valency),
        onsager=tuple(p.onsager), debye_length=p.debye_length, surface_charge=p.surface_charge,
        e_field=("OFF", "DC", "AC")[p.e_field], e_ext=tuple(p.e_ext), e_frequency=p.e_frequency,
        janus_axis=("NONE", "X", "Y", "Z")[p.janus_axis],
        janus_propulsion=("OFF", "TUMBLER", "SQUIRMER", "OBSTACLE")[p.janus_propulsion],
        janus_force=tuple(p.janus_force), janus_torque=tuple(p.janus_torque), slip_vel=p.slip_vel,
        slip_mode=p.slip_mode, rotlet_c1=p.rotlet_c1, rotlet_c2=p.rotlet_c2, slip_tol=p.slip_tol,
        slip_iter=p.slip_iter,
        species=tuple((p.species_count[i], p.species_mass_ratio[i], p.species_surface_charge[i])
                      for i in range(p.n_species)) if p.n_species > 1 and not p.rigid else ())
    if p.rigid:  # Rigid_spec[] and switch.free_rigid as the library parsed them
        nsp = max(p.n_species, 1)
        mr = [p.species_mass_ratio[s] if nsp > 1 else p.mass_ratio for s in range(nsp)]
        cfg.rigid = tuple((p.rigid_beads[s], p.rigid_count[s], mr[s],
                           kv[f"object_type.rigid.Rigid_spec[{s}].Rigid_motion"],
                           tuple(p.rigid_velocity[s]), tuple(p.rigid_omega[s])) for s in range(nsp))
        if kv.get("switch.free_rigid.type") == "YES":
            cfg.rigid_dof = tuple((s, tuple(bool(p.rigid_free[s][d]) for d in range(3)),
                                   tuple(bool(p.rigid_free[s][3 + d]) for d in range(3))) for s in range(nsp))
        cfg.rigid_gravity = tuple(p.rigid_gravity)
    return cfg, unpack_particles(rec[:p.n_particles])


class SPMRun:
    """One SPM run resident on the GPU."""

    def __init__(self, cfg: SPMConfig, precision: int = N.SPM_PREC_FP64, stream: Optional[int] = None,
                 mt_seed: int = 0):
        self.cfg = cfg
        self.L = N.lib()
        self.params = params_from_config(cfg, precision, mt_seed)
        self.precision = precision
        self.shape = cfg.shape
        nx, ny, nz = self.shape
        self.hnz = nz // 2 + 1
        self.nfield = nx * ny * 2 * self.hnz
        h = C.c_void_p()
        N.check(self.L.spm_create(C.byref(self.params), C.c_void_p(stream) if stream else None, C.byref(h)),
                "spm_create")
        self.h = h

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if self.h:
            self.L.spm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- helpers ---------------------------------------------------------
    def _kfield(self):
        return np.zeros(self.nfield)

    def _as_k(self, a: np.ndarray) -> np.ndarray:
        nx, ny, _ = self.shape
        return a.view(np.complex128).reshape(nx, ny, self.hnz)

    def _real_out(self, a: np.ndarray) -> np.ndarray:
        nx, ny, nz = self.shape
        return a.reshape(nx, ny, 2 * self.hnz)[:, :, :nz].copy()

    def _real_in(self, r: np.ndarray) -> np.ndarray:
        nx, ny, nz = self.shape
        a = np.zeros((nx, ny, 2 * self.hnz))
        a[:, :, :nz] = r
        return a.ravel()

    def _k_in(self, k: np.ndarray) -> np.ndarray:
        return np.ascontiguousarray(k, dtype=np.complex128).view(np.float64).ravel().copy()

    # -- whole run -------------------------------------------------------
    def initialize(self, particles):
        rec = particles if isinstance(particles, np.ndarray) else pack_particles(particles, self.cfg.n_particles)
        rec = np.ascontiguousarray(rec, dtype=float)
        N.check(self.L.spm_initialize(self.h, N.dptr(rec)), "spm_initialize")

    def step(self, n: int = 1):
        """Time_evolution_hydro / Time_evolution_hydro_OBL, n times."""
        N.check(self.L.spm_step(self.h, n), "spm_step")

    def synchronize(self):
        N.check(self.L.spm_synchronize(self.h), "spm_synchronize")

    def rigid_bodies(self) -> Dict[str, np.ndarray]:
        """The rigid bodies' state: xG, xG_nopbc, vG, wG ([nb, 3]), mass [nb]
        and the body-frame principal moments Ibody [nb, 3]."""
        n = C.c_int()
        N.check(self.L.spm_rigid_count(self.h, C.byref(n)), "spm_rigid_count")
        out = np.zeros((max(n.value, 1), N.SPM_RIGID_WORDS))
        N.check(self.L.spm_get_rigid(self.h, N.dptr(out)), "spm_get_rigid")
        out = out[:n.value]
        return dict(xg=out[:, 0:3], xg_nopbc=out[:, 3:6], vg=out[:, 6:9], wg=out[:, 9:12], mass=out[:, 12],
                    ibody=out[:, 13:16])

    def time_steps(self, n: int) -> float:
        ms = C.c_float()
        N.check(self.L.spm_time_steps(self.h, n, C.byref(ms)), "spm_time_steps")
        return float(ms.value)

    def particles_record(self) -> np.ndarray:
        rec = np.zeros((self.cfg.n_particles, N.SPM_PARTICLE_WORDS))
        N.check(self.L.spm_get_particles(self.h, N.dptr(rec)), "spm_get_particles")
        return rec

    def particles(self) -> Dict[str, np.ndarray]:
        return unpack_particles(self.particles_record())

    def set_particles(self, particles):
        rec = particles if isinstance(particles, np.ndarray) else pack_particles(particles, self.cfg.n_particles)
        rec = np.ascontiguousarray(rec, dtype=float)
        N.check(self.L.spm_set_particles(self.h, N.dptr(rec)), "spm_set_particles")

    def zeta(self):
        z0, z1, dc = self._kfield(), self._kfield(), np.zeros(3)
        N.check(self.L.spm_get_zeta(self.h, N.dptr(z0), N.dptr(z1), N.dptr(dc)), "spm_get_zeta")
        return np.stack([self._as_k(z0), self._as_k(z1)]), dc

    def set_zeta(self, zeta: np.ndarray, uk_dc):
        z0, z1 = self._k_in(zeta[0]), self._k_in(zeta[1])
        dc = np.ascontiguousarray(uk_dc, dtype=float)
        N.check(self.L.spm_set_zeta(self.h, N.dptr(z0), N.dptr(z1), N.dptr(dc)), "spm_set_zeta")

    def velocity(self) -> np.ndarray:
        u = [self._kfield() for _ in range(3)]
        N.check(self.L.spm_get_velocity(self.h, *[N.dptr(a) for a in u]), "spm_get_velocity")
        return np.stack([self._real_out(a) for a in u])

    def phi(self) -> np.ndarray:
        a = self._kfield()
        N.check(self.L.spm_get_phi(self.h, N.dptr(a)), "spm_get_phi")
        return self._real_out(a)

    def time(self):
        ts, t = C.c_int(), C.c_double()
        N.check(self.L.spm_get_time(self.h, C.byref(ts), C.byref(t)), "spm_get_time")
        return ts.value, t.value

    def set_time(self, ts: int, time: float, degree_oblique: float = 0.0):
        """Sets the step counter, the time and (Lees-Edwards) degree_oblique
        of the run, e.g. to continue a run whose state was set by hand."""
        N.check(self.L.spm_set_time(self.h, int(ts), float(time), float(degree_oblique)), "spm_set_time")

    def concentration(self, species: int = 0) -> np.ndarray:
        """k-space concentration of one ion species of an Electrolyte run."""
        a = self._kfield()
        N.check(self.L.spm_get_concentration(self.h, int(species), N.dptr(a)), "spm_get_concentration")
        return self._as_k(a)

    def shear_state(self):
        deg, st = C.c_double(), np.zeros(8)
        N.check(self.L.spm_get_shear_state(self.h, C.byref(deg), N.dptr(st)), "spm_get_shear_state")
        return deg.value, st

    def save_state(self, path: str):
        """Checkpoint of the device state (spm_save_state)."""
        N.check(self.L.spm_save_state(self.h, path.encode()), "spm_save_state")

    def load_state(self, path: str):
        """Restores a checkpoint written by a run with the same parameters."""
        N.check(self.L.spm_load_state(self.h, path.encode()), "spm_load_state")

    def load_restart(self, path: str):
        """Restores the saved section of a restart file of the reference
        program (spm_load_restart; UDF or key file)."""
        N.check(self.L.spm_load_restart(self.h, path.encode()), "spm_load_restart")

    def save_restart(self, path: str, input_path: Optional[str] = None):
        """Writes a restart key file the reference program resumes from
        (spm_save_restart): the keys of `input_path`, then the saved state."""
        N.check(self.L.spm_save_restart(self.h, input_path.encode() if input_path else None, path.encode()),
                "spm_save_restart")

    def udf_out_open(self, path: str):
        """Opens the per-frame UDF particle records (spm_udf_out_open)."""
        N.check(self.L.spm_udf_out_open(self.h, path.encode()), "spm_udf_out_open")

    def udf_out_record(self):
        """Appends one record of the current state (Output_udf)."""
        N.check(self.L.spm_udf_out_record(self.h), "spm_udf_out_record")

    def udf_out_close(self):
        N.check(self.L.spm_udf_out_close(self.h), "spm_udf_out_close")

    def avs_open(self, out_dir: str, out_name: str, num_snap: int):
        """Legacy AVS output of this run (spm_avs_open): headers now, one
        frame per avs_frame() call."""
        N.check(self.L.spm_avs_open(self.h, out_dir.encode(), out_name.encode(), int(num_snap)), "spm_avs_open")

    def avs_frame(self):
        """Enqueues the frame of the current step (spm_avs_frame); the files
        are written while the run goes on."""
        N.check(self.L.spm_avs_frame(self.h), "spm_avs_frame")

    def avs_close(self):
        """Waits for the enqueued frames and closes the output (spm_avs_close)."""
        N.check(self.L.spm_avs_close(self.h), "spm_avs_close")

    def kernel_launches(self, reset: bool = False) -> int:
        n = C.c_longlong()
        N.check(self.L.spm_kernel_launches(self.h, C.byref(n), 1 if reset else 0), "spm_kernel_launches")
        return n.value

    # -- reference solver boundaries (host arrays) -----------------------
    def NS_solver_slavedEuler(self, zeta: np.ndarray, uk_dc: np.ndarray):
        z0, z1 = self._k_in(zeta[0]), self._k_in(zeta[1])
        dc = np.ascontiguousarray(uk_dc, dtype=float).copy()
        N.check(self.L.spm_ns_solver_slaved_euler_host(self.h, N.dptr(z0), N.dptr(z1), N.dptr(dc)),
                "NS_solver_slavedEuler")
        return np.stack([self._as_k(z0), self._as_k(z1)])

    def Solenoidal_uk(self, uk: np.ndarray) -> np.ndarray:
        a = [self._k_in(uk[d]) for d in range(3)]
        N.check(self.L.spm_solenoidal_uk_host(self.h, *[N.dptr(x) for x in a]), "Solenoidal_uk")
        return np.stack([self._as_k(x) for x in a])

    def Zeta_k2u_k(self, zeta: np.ndarray, uk_dc) -> np.ndarray:
        z0, z1 = self._k_in(zeta[0]), self._k_in(zeta[1])
        dc = np.ascontiguousarray(uk_dc, dtype=float)
        u = [self._kfield() for _ in range(3)]
        N.check(self.L.spm_zeta_k2u_k_host(self.h, N.dptr(z0), N.dptr(z1), N.dptr(dc), *[N.dptr(x) for x in u]),
                "Zeta_k2u_k")
        return np.stack([self._as_k(x) for x in u])

    def U_k2zeta_k(self, uk: np.ndarray):
        a = [self._k_in(uk[d]) for d in range(3)]
        z0, z1, dc = self._kfield(), self._kfield(), np.zeros(3)
        N.check(self.L.spm_u_k2zeta_k_host(self.h, *[N.dptr(x) for x in a], N.dptr(z0), N.dptr(z1), N.dptr(dc)),
                "U_k2zeta_k")
        return np.stack([self._as_k(z0), self._as_k(z1)]), dc

    def A2a_k(self, a_real: np.ndarray) -> np.ndarray:
        a = self._real_in(a_real)
        N.check(self.L.spm_a2a_k_host(self.h, N.dptr(a)), "A2a_k")
        return self._as_k(a)

    def A_k2a(self, ak: np.ndarray) -> np.ndarray:
        a = self._k_in(ak)
        N.check(self.L.spm_a_k2a_host(self.h, N.dptr(a)), "A_k2a")
        return self._real_out(a)

    def Make_phi_particle_sum(self, particles):
        rec = np.ascontiguousarray(particles if isinstance(particles, np.ndarray)
                                   else pack_particles(particles, self.cfg.n_particles), dtype=float)
        phi, phs = self._kfield(), self._kfield()
        N.check(self.L.spm_make_phi_particle_sum_host(self.h, N.dptr(rec), N.dptr(phi), N.dptr(phs)),
                "Make_phi_particle_sum")
        return self._real_out(phi), self._real_out(phs)

    def Make_u_particle_sum(self, particles, phi_sum: np.ndarray) -> np.ndarray:
        rec = np.ascontiguousarray(particles if isinstance(particles, np.ndarray)
                                   else pack_particles(particles, self.cfg.n_particles), dtype=float)
        ps = self._real_in(phi_sum)
        up = [self._kfield() for _ in range(3)]
        N.check(self.L.spm_make_u_particle_sum_host(self.h, N.dptr(rec), N.dptr(ps), *[N.dptr(x) for x in up]),
                "Make_u_particle_sum")
        return np.stack([self._real_out(x) for x in up])

    def Make_phi_u_particle(self, particles):
        rec = np.ascontiguousarray(particles if isinstance(particles, np.ndarray)
                                   else pack_particles(particles, self.cfg.n_particles), dtype=float)
        phi = self._kfield()
        up = [self._kfield() for _ in range(3)]
        N.check(self.L.spm_make_phi_u_particle_host(self.h, N.dptr(rec), N.dptr(phi), *[N.dptr(x) for x in up]),
                "Make_phi_u_particle")
        return self._real_out(phi), np.stack([self._real_out(x) for x in up])

    def Make_f_particle_dt_sole(self, u: np.ndarray, up: np.ndarray, phi: np.ndarray) -> np.ndarray:
        ua = [self._real_in(u[d]) for d in range(3)]
        upa = [self._real_in(up[d]) for d in range(3)]
        ph = self._real_in(phi)
        f = [self._kfield() for _ in range(3)]
        N.check(self.L.spm_make_f_particle_dt_sole_host(self.h, *[N.dptr(x) for x in ua], *[N.dptr(x) for x in upa],
                                                        N.dptr(ph), *[N.dptr(x) for x in f]),
                "Make_f_particle_dt_sole")
        return np.stack([self._real_out(x) for x in f])

    def Calc_f_hydro_correct_precision(self, particles, phi_sum: np.ndarray, u: np.ndarray) -> np.ndarray:
        rec = np.ascontiguousarray(particles if isinstance(particles, np.ndarray)
                                   else pack_particles(particles, self.cfg.n_particles), dtype=float).copy()
        ps = self._real_in(phi_sum)
        ua = [self._real_in(u[d]) for d in range(3)]
        N.check(self.L.spm_calc_f_hydro_correct_precision_host(self.h, N.dptr(rec), N.dptr(ps),
                                                               *[N.dptr(x) for x in ua]),
                "Calc_f_hydro_correct_precision")
        return rec

    def Calc_f_Lennard_Jones(self, particles) -> np.ndarray:
        rec = np.ascontiguousarray(particles if isinstance(particles, np.ndarray)
                                   else pack_particles(particles, self.cfg.n_particles), dtype=float).copy()
        N.check(self.L.spm_calc_f_lennard_jones_host(self.h, N.dptr(rec)), "Calc_f_Lennard_Jones")
        return rec


def resume_run(path: str, precision: int = N.SPM_PREC_FP64, mt_seed: int = 0,
               config: Optional[SPMConfig] = None) -> "SPMRun":
    """A run resumed from a restart file of the reference program (UDF file,
    or a key file ending in .keys), as its main loop resumes one
    (sp_3d_ns.cxx:856-1005): the run is set up from the file's parameters and
    initial particles, takes one step (the reference's first pass, whose
    result the restore overwrites; it draws that step's thermostat noise),
    and then restores the saved section (Force_restore_parameters).
    `config` replaces the file's parameters where the file cannot hold them
    all (a constant body force has no UDF key)."""
    cfg, parts = config_from_udf(path)
    cfg = config or cfg
    run = SPMRun(cfg, precision=precision, mt_seed=mt_seed)
    try:
        run.initialize(parts)
        run.step(1)
        run.load_restart(path)
    except Exception:
        run.close()
        raise
    return run


def device_count() -> int:
    n = C.c_int()
    N.check(N.lib().spm_device_count(C.byref(n)), "spm_device_count")
    return n.value
