"""CPU restatement (numpy, FP64) of KAPSEL's spectral SPM time step.

TEST INFRASTRUCTURE ONLY -- this is the parity oracle.  Only tests, fixture
generation, `__graft_entry__.smoke()` and the CPU-baseline legs of bench.py may
import it; the product path never calls it and never falls back to it.

Every function restates the reference algorithm it names (file:line in the
KAPSEL tree).  Layout conventions:
  * real fields: float64 [NX, NY, NZ]  (the reference pads rows to NZ_=NZ+2)
  * k-space fields: complex128 [NX, NY, NZ//2+1]; viewed as float64 this is
    exactly the reference's in-place r2c layout [NX][NY][NZ_]
  * forward FFT = numpy.fft.rfftn (unnormalised, e^{-ikx}), inverse =
    irfftn (1/N^3): the conventions A2a_k / A_k2a realise with Ooura's rdft3d
    + rdft3dsort + conjugation (fft_wrapper.h:641-681).
Parity is pinned against the reference program itself (oracle/_ref, built
from the unmodified sources) by tests/test_oracle_vs_reference.py and by the
fixtures in tests/golden/.
"""
from __future__ import annotations

import math
from typing import Dict, Optional

import numpy as np

DBL_MAX = np.finfo(np.float64).max
KT_SNAP_V = 1.439   # input.cxx:309
KT_SNAP_O = 1.22    # input.cxx:311
CELL_LENGTH = 16    # md_force.cxx:14


# ----------------------------------------------------------------------------
# MT19937 (Matsumoto & Nishimura 1998), as the reference's mt19937ar.c is used
# through init_genrand / genrand_real3 (mt19937ar.c:65-192, fluct.h:35-60).
# ----------------------------------------------------------------------------
class MT19937:
    N, M = 624, 397

    def __init__(self, seed: int = 0):
        self.mt = [0] * self.N
        self.mt[0] = seed & 0xFFFFFFFF
        for i in range(1, self.N):
            prev = self.mt[i - 1]
            self.mt[i] = (1812433253 * (prev ^ (prev >> 30)) + i) & 0xFFFFFFFF
        self.mti = self.N

    def _twist(self):
        mt, N, M = self.mt, self.N, self.M
        for i in range(N):
            y = (mt[i] & 0x80000000) | (mt[(i + 1) % N] & 0x7FFFFFFF)
            v = mt[(i + M) % N] ^ (y >> 1)
            if y & 1:
                v ^= 0x9908B0DF
            mt[i] = v
        self.mti = 0

    def genrand_int32(self) -> int:
        if self.mti >= self.N:
            self._twist()
        y = self.mt[self.mti]
        self.mti += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & 0xFFFFFFFF

    def genrand_real3(self) -> float:
        """(0,1) open interval, 32-bit resolution."""
        return (float(self.genrand_int32()) + 0.5) * (1.0 / 4294967296.0)

    def gauss2(self):
        """Polar Box-Muller pair (fluct.h:48-60)."""
        while True:
            x1 = 2.0 * self.genrand_real3() - 1.0
            x2 = 2.0 * self.genrand_real3() - 1.0
            rsq = x1 * x1 + x2 * x2
            if not (rsq >= 1.0 or rsq == 0.0):
                break
        factor = math.sqrt(-2.0 * math.log(rsq) / rsq)
        return factor * x1, factor * x2


def nint(a: np.ndarray) -> np.ndarray:
    """macro.h:44-52: round half away from zero via int truncation."""
    return np.where(a >= 0.0, np.trunc(a + 0.5), np.trunc(a - 0.5))


def qtn_prod(qa: np.ndarray, qb: np.ndarray, alpha: float) -> np.ndarray:
    """quaternion.h:151-160 (rows are (s, v0, v1, v2))."""
    s = alpha * (qa[:, 0] * qb[:, 0] - (qa[:, 1] * qb[:, 1] + qa[:, 2] * qb[:, 2] + qa[:, 3] * qb[:, 3]))
    v0 = alpha * (qa[:, 0] * qb[:, 1] + qb[:, 0] * qa[:, 1] + qa[:, 2] * qb[:, 3] - qa[:, 3] * qb[:, 2])
    v1 = alpha * (qa[:, 0] * qb[:, 2] + qb[:, 0] * qa[:, 2] + qa[:, 3] * qb[:, 1] - qa[:, 1] * qb[:, 3])
    v2 = alpha * (qa[:, 0] * qb[:, 3] + qb[:, 0] * qa[:, 3] + qa[:, 1] * qb[:, 2] - qa[:, 2] * qb[:, 1])
    return np.stack([s, v0, v1, v2], axis=1)


def qdot_space(q: np.ndarray, omega: np.ndarray) -> np.ndarray:
    """rigid_body.cxx:157-168 with SPACE_FRAME: dq/dt = 0.5 (0,w) o q."""
    qw = np.concatenate([np.zeros((len(q), 1)), omega], axis=1)
    return qtn_prod(qw, q, 0.5)


def qtn_normalize(q: np.ndarray) -> np.ndarray:
    """quaternion.h:260-268."""
    norm = np.sqrt(q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1] + q[:, 2] * q[:, 2] + q[:, 3] * q[:, 3])
    return q * (1.0 / norm)[:, None]


class OracleSPM:
    """One SPM run: state plus the reference's step, restated in numpy."""

    def __init__(self, cfg, particles: Dict[str, np.ndarray]):
        self.cfg = cfg
        d = cfg.derived()
        self.d = d
        self.NX, self.NY, self.NZ = d["NX"], d["NY"], d["NZ"]
        self.HNZ = self.NZ // 2 + 1
        self.DX = cfg.dx
        self.dt = cfg.dt
        self.hdt = 0.5 * cfg.dt
        self.L = np.array([d["LX"], d["LY"], d["LZ"]])
        self.N3 = np.array([self.NX, self.NY, self.NZ])
        # Integer wavenumbers (fft_wrapper.h:719-729): index > N/2 maps negative.
        i = np.arange(self.NX)
        j = np.arange(self.NY)
        k = np.arange(self.HNZ)
        self.KX = np.where(i > self.NX // 2, i - self.NX, i)[:, None, None]
        self.KY = np.where(j > self.NY // 2, j - self.NY, j)[None, :, None]
        self.KZ = k[None, None, :]
        self.kx = d["WAVE_X"] * self.KX.astype(float)
        self.ky = d["WAVE_Y"] * self.KY.astype(float)
        self.kz = d["WAVE_Z"] * self.KZ.astype(float)
        # K2 / IK2 tables (fft_wrapper.cxx:45-76).
        self.K2 = self.kx ** 2 + self.ky ** 2 + self.kz ** 2
        with np.errstate(divide="ignore"):
            self.IK2 = np.where(self.K2 > 0.0, 1.0 / np.where(self.K2 > 0, self.K2, 1.0), 0.0)
        # 2/3 rule: retained modes (fft_wrapper.h:754-796 zeroes the rest;
        # fft_wrapper.cxx:172-184 lists the retained boxes).
        self.keep = (np.abs(self.KX) < d["TRN_X"]) & (np.abs(self.KY) < d["TRN_Y"]) & (self.KZ < d["TRN_Z"])
        self._sekibun()
        # particles
        n = cfg.n_particles
        self.np = n
        z3 = lambda: np.zeros((n, 3))
        self.x = np.array(particles["x"], dtype=float).copy()
        self.x_nopbc = self.x.copy()
        self.x_previous = self.x.copy()
        self.v = np.array(particles["v"], dtype=float).copy()
        self.v_old = z3()
        self.omega = np.array(particles["omega"], dtype=float).copy()
        self.omega_old = z3()
        q = np.array(particles["q"], dtype=float).copy()
        self.q = qtn_normalize(q)          # ORIENTATION=user_dir (init_particle.cxx:308-312)
        self.q_old = self.q.copy()
        self.f_hydro, self.f_hydro_previous = z3(), z3()
        self.torque_hydro, self.torque_hydro_previous = z3(), z3()
        self.fr, self.fr_previous = z3(), z3()
        self.torque_r, self.torque_r_previous = z3(), z3()
        self.mt = MT19937(0)               # MT_seed(GIVEN_SEED, 0), sp_3d_ns.cxx:767
        self.ts = 0
        self.time = 0.0
        self.zeta = np.zeros((2, self.NX, self.NY, self.HNZ), dtype=complex)
        self.uk_dc = np.zeros(3)
        self.phi = np.zeros((self.NX, self.NY, self.NZ))
        self.phi_sum = np.zeros_like(self.phi)
        self.u = np.zeros((3, self.NX, self.NY, self.NZ))
        self.dev_shear_stress_lj = 0.0
        self._initial_projection()

    # ------------------------------------------------------------------ FFT
    def fft(self, a: np.ndarray) -> np.ndarray:
        """A2a_k (fft_wrapper.h:641-654)."""
        return np.fft.rfftn(a, axes=(-3, -2, -1))

    def ifft(self, ak: np.ndarray) -> np.ndarray:
        """A_k2a (fft_wrapper.h:662-681)."""
        return np.fft.irfftn(ak, s=(self.NX, self.NY, self.NZ), axes=(-3, -2, -1))

    def truncate(self, ak: np.ndarray) -> np.ndarray:
        return np.where(self.keep, ak, 0.0)

    # --------------------------------------------------------- k-space maps
    def zeta_k2u_k(self, zeta: np.ndarray, uk_dc: np.ndarray) -> np.ndarray:
        """Zeta_k2u_k (fft_wrapper.cxx:591-688)."""
        kx, ky, kz, ik2 = self.kx, self.ky, self.kz, self.IK2
        z0, z1 = zeta[0], zeta[1]
        cx = self.KX != 0
        cy = (self.KX == 0) & (self.KY != 0)
        with np.errstate(divide="ignore", invalid="ignore"):
            inv_kx = np.where(cx, 1.0 / np.where(cx, kx, 1.0), 0.0)
            dmy = np.where(self.KY != 0, -(kz / np.where(self.KY != 0, ky, 1.0)), 0.0)
        om0 = np.where(cx, -inv_kx * (ky * z0 + kz * z1), np.where(cy, z1, z0))
        om1 = np.where(cx, z0, np.where(cy, dmy * z0, z1))
        om2 = np.where(cx, z1, np.where(cy, z0, 0.0))
        kx, ky, kz = kx * ik2, ky * ik2, kz * ik2
        u = np.empty((3,) + z0.shape, dtype=complex)
        u[0] = 1j * (ky * om2 - kz * om1)
        u[1] = 1j * (kz * om0 - kx * om2)
        u[2] = 1j * (kx * om1 - ky * om0)
        for dd in range(3):
            u[dd, 0, 0, 0] = complex(uk_dc[dd], u[dd, 0, 0, 0].imag)
        return u

    def _omega_to_zeta(self, om: np.ndarray) -> np.ndarray:
        """Component choice of Omega_k2zeta_k (fft_wrapper.cxx:227-263)."""
        cx = self.KX != 0
        cy = (self.KX == 0) & (self.KY != 0)
        z0 = np.where(cx, om[1], np.where(cy, om[2], om[0]))
        z1 = np.where(cx, om[2], np.where(cy, om[0], om[1]))
        return np.stack([z0, z1])

    def u_k2zeta_k(self, uk: np.ndarray):
        """U_k2zeta_k (fft_wrapper.cxx:407-476): zeta = reduced i k x u."""
        kx, ky, kz = self.kx, self.ky, self.kz
        uk_dc = np.array([uk[0, 0, 0, 0].real, uk[1, 0, 0, 0].real, uk[2, 0, 0, 0].real])
        om = np.empty_like(uk)
        om[0] = 1j * (ky * uk[2] - kz * uk[1])
        om[1] = 1j * (kz * uk[0] - kx * uk[2])
        om[2] = 1j * (kx * uk[1] - ky * uk[0])
        return self._omega_to_zeta(om), uk_dc

    def solenoidal_uk(self, uk: np.ndarray) -> np.ndarray:
        """Solenoidal_uk (operate_omega.cxx:171-195)."""
        kx, ky, kz = self.kx, self.ky, self.kz
        dmy = self.IK2 * (uk[0] * kx + uk[1] * ky + uk[2] * kz)
        return np.stack([uk[0] - dmy * kx, uk[1] - dmy * ky, uk[2] - dmy * kz])

    def solenoidal_u(self, u: np.ndarray) -> np.ndarray:
        """Solenoidal_u (operate_omega.h:105-112)."""
        uk = self.truncate(self.fft(u))
        return self.ifft(self.solenoidal_uk(uk))

    def u2advection_k(self, u: np.ndarray) -> np.ndarray:
        """U2advection_k (operate_omega.cxx:12-85): the curl of the advection
        term (with a minus sign), reduced to two components."""
        u1, u2, u3 = u[0], u[1], u[2]
        prod = np.stack([u2 * u3, u3 * u1, u1 * u2, (u2 - u3) * (u2 + u3), (u3 - u1) * (u3 + u1)])
        pk = self.fft(prod)
        u2u3, u3u1, u1u2, u22_u32, u32_u12 = pk
        u12_u22 = -u32_u12 - u22_u32
        k1, k2, k3 = self.kx, self.ky, self.kz
        k1k2, k2k3, k3k1 = k1 * k2, k2 * k3, k3 * k1
        om = np.empty((3,) + u2u3.shape, dtype=complex)
        om[0] = -(k2k3 * u22_u32 + (k3 - k2) * (k3 + k2) * u2u3 + k3k1 * u1u2 - k1k2 * u3u1)
        om[1] = -(k3k1 * u32_u12 + (k1 - k3) * (k1 + k3) * u3u1 + k1k2 * u2u3 - k2k3 * u1u2)
        om[2] = -(k1k2 * u12_u22 + (k2 - k1) * (k2 + k1) * u1u2 + k2k3 * u3u1 - k3k1 * u2u3)
        return self._omega_to_zeta(om)

    def ns_solver_slaved_euler(self):
        """NS_solver_slavedEuler (fluid_solver.cxx:348-374) with
        Zeta_k2advection_k (operate_omega.cxx:87-98)."""
        self.zeta = self.truncate(self.zeta)
        u = self.ifft(self.zeta_k2u_k(self.zeta, self.uk_dc))
        f_ns0 = self.u2advection_k(u)
        nu = self.cfg.eta / self.cfg.rho
        dmy0 = -nu * self.dt
        dmy1 = 1.0 / nu
        dmy = np.exp(dmy0 * self.K2) - 1.0
        upd = self.zeta + dmy * (self.zeta - (dmy1 * self.IK2) * f_ns0)
        self.zeta = np.where(self.keep, upd, self.zeta)

    # ------------------------------------------------------------ stencils
    def _sekibun(self):
        """Particle_domain (profile.cxx:22-65)."""
        d = self.d
        nh = int(self.cfg.a) + int(self.cfg.a_xi) + 2
        max_radius = d["RADIUS"] + d["HXI"] + 1.7321 * self.DX
        r = np.arange(-nh, nh + 1)
        I, J, K = np.meshgrid(r, r, r, indexing="ij")
        dist = np.sqrt((I * self.DX) ** 2 + (J * self.DX) ** 2 + (K * self.DX) ** 2)
        m = dist < max_radius
        self.cells = np.stack([I[m], J[m], K[m]], axis=1)  # i-major order, as the reference
        self.np_domain = len(self.cells)

    def profile(self, x: np.ndarray) -> np.ndarray:
        """Phi (profile.h:30-50): H(a+xi/2-x)/(H(a+xi/2-x)+H(x-a+xi/2))."""
        dx = self.DX
        R, hxi = self.d["RADIUS"], self.d["HXI"]

        def H(y):
            out = np.zeros_like(y)
            pos = y > 0
            out[pos] = np.exp(-((dx / y[pos]) ** 2))
            return out
        h1 = H(R + hxi - x)
        return h1 / (h1 + H(x - R + hxi))

    def stencil_geometry(self, x: np.ndarray):
        """Particle_cell + Relative_coord + Distance (make_phi.h:114-170,
        interaction.h:113-132) for every particle and Sekibun cell.
        Returns flat grid indices, r vectors and distances [Np, NP_domain]."""
        dx = self.DX
        idx = 1.0 / dx
        dmy = x * idx
        x_int = np.trunc(dmy).astype(np.int64)
        residue = (dmy - x_int) * dx
        cell = self.cells[None, :, :]
        r_mesh = (x_int[:, None, :] + cell + self.N3) % self.N3
        r = cell * dx - residue[:, None, :]
        xm = r_mesh * dx
        x12 = x[:, None, :] - xm
        x12 = x12 - nint(x12 / self.L) * self.L
        dist = np.sqrt(x12[..., 0] ** 2 + x12[..., 1] ** 2 + x12[..., 2] ** 2)
        flat = (r_mesh[..., 0] * self.NY + r_mesh[..., 1]) * self.NZ + r_mesh[..., 2]
        return flat, r, dist

    def make_phi_particle_sum(self):
        """Make_phi_particle_sum (make_phi.cxx:214-260)."""
        flat, r, dist = self.stencil_geometry(self.x)
        ph = self.profile(dist)
        phi_sum = np.zeros(self.NX * self.NY * self.NZ)
        np.add.at(phi_sum, flat.ravel(), ph.ravel())
        self.phi_sum = phi_sum.reshape(self.NX, self.NY, self.NZ)
        self.phi = np.minimum(self.phi_sum, 1.0)

    def _v_surface(self, v, omega, r):
        if self.cfg.rotation:   # Angular2v_rot_on (make_phi.h:403-407)
            w = omega[:, None, :]
            vr = np.stack([w[..., 1] * r[..., 2] - w[..., 2] * r[..., 1],
                           w[..., 2] * r[..., 0] - w[..., 0] * r[..., 2],
                           w[..., 0] * r[..., 1] - w[..., 1] * r[..., 0]], axis=-1)
        else:
            vr = np.zeros_like(r)
        return v[:, None, :] + vr

    def calc_f_hydro(self):
        """Calc_f_hydro_correct_precision (md_force.cxx:383-506)."""
        flat, r, dist = self.stencil_geometry(self.x)
        w = self.profile(dist) / np.maximum(self.phi_sum.ravel()[flat], 1.0)
        ug = self.u.reshape(3, -1)[:, flat]                      # [3, Np, M]
        vs = self._v_surface(self.v, self.omega, r)             # [Np, M, 3]
        dmy_fp = (vs - np.moveaxis(ug, 0, -1)) * w[..., None]
        force = dmy_fp.sum(axis=1)
        torque = np.stack([r[..., 1] * dmy_fp[..., 2] - r[..., 2] * dmy_fp[..., 1],
                           r[..., 2] * dmy_fp[..., 0] - r[..., 0] * dmy_fp[..., 2],
                           r[..., 0] * dmy_fp[..., 1] - r[..., 1] * dmy_fp[..., 0]], axis=-1).sum(axis=1)
        dmy = -self.d["DX3"] * self.cfg.rho / self.dt
        self.f_hydro = dmy * force
        if self.cfg.rotation:
            self.torque_hydro = dmy * torque

    def make_u_particle_sum(self) -> np.ndarray:
        """Make_u_particle_sum (make_phi.cxx:313-354)."""
        flat, r, dist = self.stencil_geometry(self.x)
        w = self.profile(dist) / np.maximum(self.phi_sum.ravel()[flat], 1.0)
        vs = self._v_surface(self.v, self.omega, r) * w[..., None]
        up = np.zeros((3, self.NX * self.NY * self.NZ))
        for dd in range(3):
            np.add.at(up[dd], flat.ravel(), vs[..., dd].ravel())
        return up.reshape(3, self.NX, self.NY, self.NZ)

    # ----------------------------------------------------------- particles
    def lj_multiplicity(self):
        """Pair multiplicity of the reference cell list (md_force.cxx:56-101):
        Cell_length 16, neighbour cells wrapped so that with fewer than three
        cells per axis a neighbour is visited more than once."""
        lc = np.array([self.NX // CELL_LENGTH, self.NY // CELL_LENGTH, self.NZ // CELL_LENGTH])
        mc = (self.x / (CELL_LENGTH * self.DX)).astype(np.int64)
        n = self.np
        mult = np.ones((n, n), dtype=np.int64)
        for dd in range(3):
            a = mc[:, dd][:, None]
            b = mc[:, dd][None, :]
            cnt = np.zeros((n, n), dtype=np.int64)
            for off in (-1, 0, 1):
                c = a + off
                c = np.where(c < 0, lc[dd] - 1, c)
                c = np.where(c > lc[dd] - 1, 0, c)
                cnt += (c == b)
            mult *= cnt
        return mult

    def calc_f_lennard_jones(self):
        """Calc_f_Lennard_Jones_shear_cap_primitive_lnk (md_force.cxx:34-196)
        with Lennard_Jones_f (interaction.h:160-199); 12:6 powers."""
        d = self.d
        sigma = d["LJ_dia"]
        cutoff = d["A_R_cutoff"] * sigma
        eps = self.cfg.epsilon
        mult = self.lj_multiplicity()
        n = self.np
        for i in range(n):
            for j in range(i):
                m = int(mult[i, j])
                if m == 0:
                    continue
                x12 = self.x[j] - self.x[i]
                x12 = x12 - nint(x12 / self.L) * self.L
                rij = math.sqrt(x12[0] ** 2 + x12[1] ** 2 + x12[2] ** 2)
                if rij < cutoff:
                    s = sigma / rij
                    s6 = (s * s) * (s * s) * (s * s)
                    lj = 24.0 * eps / (rij * rij) * (2.0 * s6 * s6 - s6)
                    dmy_r = min(DBL_MAX / rij, lj)
                    for _ in range(m):
                        fi = dmy_r * (-x12)
                        self.fr[i] += fi
                        self.fr[j] -= fi
                        self.dev_shear_stress_lj += fi[0] * x12[1]

    def force(self):
        """Force (particle_solver.h:88-111): LJ, then the constant body force
        in the place of Add_f_gravity."""
        if self.cfg.lj_truncate in ("ON", "OFF"):
            self.calc_f_lennard_jones()
        if any(f != 0.0 for f in self.cfg.body_force):
            self.fr += np.array(self.cfg.body_force)[None, :]

    def reset_forces(self):
        """reset_Forces (particle_solver.cxx:11-37)."""
        self.fr_previous, self.fr = self.fr, np.zeros_like(self.fr)
        self.f_hydro_previous, self.f_hydro = self.f_hydro, np.zeros_like(self.f_hydro)
        self.torque_r_previous, self.torque_r = self.torque_r, np.zeros_like(self.torque_r)
        self.torque_hydro_previous, self.torque_hydro = self.torque_hydro, np.zeros_like(self.torque_hydro)

    def pbc(self, x):
        """PBC (periodic_boundary.h:9-16)."""
        return np.fmod(x + self.L, self.L)

    def position_euler(self):
        """MD_solver_position_Euler (particle_solver.cxx:39-61) and
        MD_solver_orientation_Euler (particle_rotation_solver.h:23-29)."""
        self.x_previous = self.x.copy()
        dx = self.dt * self.v
        self.x_nopbc = self.x_nopbc + dx
        self.x = self.pbc(self.x + dx)
        if self.cfg.rotation:
            self.q_old = self.q.copy()
            dq = qdot_space(self.q, self.omega)
            self.q = qtn_normalize(self.q + dq * self.dt)

    def position_ab2(self):
        """MD_solver_position_AB2 (particle_solver.cxx:63-85) and
        MD_solver_orientation_AB2 (particle_rotation_solver.h:72-81)."""
        self.x_previous = self.x.copy()
        dx = self.hdt * (3.0 * self.v - self.v_old)
        self.x_nopbc = self.x_nopbc + dx
        self.x = self.pbc(self.x + dx)
        if self.cfg.rotation:
            dq = qdot_space(self.q, self.omega)
            dq_old = qdot_space(self.q_old, self.omega_old)
            self.q_old = self.q.copy()
            q = self.q + dq * (3.0 * self.hdt)
            q = q + dq_old * (-self.hdt)
            self.q = qtn_normalize(q)

    def velocity_euler(self):
        """MD_solver_velocity_Euler (particle_solver.cxx:103-142)."""
        self.force()
        imass, imoi = self.d["IMASS"], self.d["IMOI"]
        dmy, dmy_rot = self.dt * imass, self.dt * imoi
        self.v_old, self.omega_old = self.v.copy(), self.omega.copy()
        self.v = self.v + dmy * (self.f_hydro + self.fr)
        self.omega = self.omega + dmy_rot * (self.torque_hydro + self.torque_r)
        self.reset_forces()

    def velocity_ab2(self):
        """MD_solver_velocity_AB2_hydro (particle_solver.cxx:239-281)."""
        self.force()
        imass, imoi = self.d["IMASS"], self.d["IMOI"]
        dmy, dmy_rot = self.hdt * imass, self.hdt * imoi
        self.v_old, self.omega_old = self.v.copy(), self.omega.copy()
        self.v = self.v + dmy * (2.0 * self.f_hydro + self.fr + self.fr_previous)
        self.omega = self.omega + dmy_rot * (2.0 * self.torque_hydro + self.torque_r + self.torque_r_previous)
        self.reset_forces()

    def thermostat(self):
        """Add_random_force_thermostat (fluct.cxx:10-37), serial draw order."""
        cfg, d = self.cfg, self.d
        zeta_drag = 6.0 * math.pi * cfg.eta * d["RADIUS"]
        zeta_drag_rot = 8.0 * math.pi * cfg.eta * d["RADIUS"] ** 3
        sdv_v = math.sqrt(zeta_drag * self.dt * cfg.kbt * cfg.alpha_v)
        sdv_o = math.sqrt(zeta_drag_rot * self.dt * cfg.kbt * cfg.alpha_o)
        nv, no = KT_SNAP_V * sdv_v, KT_SNAP_O * sdv_o
        for n in range(self.np):
            g = []
            for _ in range(3):
                g.extend(self.mt.gauss2())
            for dd in range(3):
                self.v[n, dd] += g[dd] * nv * d["IMASS"]
                if cfg.rotation:
                    self.omega[n, dd] += g[dd + 3] * no * d["IMOI"]

    # ---------------------------------------------------------------- step
    def _initial_projection(self):
        """main()'s initial rigidity projection (sp_3d_ns.cxx:809-826) after
        Init_zeta_k (init_fluid.cxx:10-25) leaves zeta = 0."""
        self.make_phi_particle_sum()
        up = self.make_u_particle_sum()
        u = self.ifft(self.zeta_k2u_k(self.zeta, self.uk_dc))
        f = self.solenoidal_u(up - self.phi[None] * u)
        u = u + f
        self.zeta, self.uk_dc = self.u_k2zeta_k(self.fft(u))
        self.uk_dc = np.zeros(3)
        self.u = u

    def step(self):
        """Time_evolution_hydro (sp_3d_ns.cxx:41-194) for Navier_Stokes with
        free spherical particles, no walls or slip."""
        cfg = self.cfg
        self.ns_solver_slaved_euler()
        for dd in range(3):
            if cfg.fix_cell[dd]:
                self.uk_dc[dd] = 0.0
        self.zeta = self.truncate(self.zeta)
        self.u = self.ifft(self.zeta_k2u_k(self.zeta, self.uk_dc))
        if self.ts == 0:
            self.position_euler()
        else:
            self.position_ab2()
        self.make_phi_particle_sum()
        self.calc_f_hydro()
        if self.ts == 0:
            self.velocity_euler()
        else:
            self.velocity_ab2()
        if cfg.kbt > 0.0:
            self.thermostat()
        up = self.make_u_particle_sum()
        f = self.solenoidal_u(up - self.phi[None] * self.u)
        self.u = self.u + f
        self.zeta, self.uk_dc = self.u_k2zeta_k(self.fft(self.u))
        self.ts += 1
        self.time += self.dt

    def _phi_of_positions(self) -> np.ndarray:
        """phi_sum of the current particle positions (Make_phi_particle_sum)."""
        flat, r, dist = self.stencil_geometry(self.x)
        phi_sum = np.zeros(self.NX * self.NY * self.NZ)
        np.add.at(phi_sum, flat.ravel(), self.profile(dist).ravel())
        return phi_sum.reshape(self.NX, self.NY, self.NZ)

    def velocity_field(self) -> np.ndarray:
        """Real-space velocity of the current state, as rebuilt from zeta
        (Zeta_k2u_k + U_k2u)."""
        return self.ifft(self.zeta_k2u_k(self.zeta, self.uk_dc))
