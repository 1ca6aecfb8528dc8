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


def ooura_packed_planes(ak: np.ndarray) -> np.ndarray:
    """The kz = 0 and kz = NZ/2 planes of a k-space field [..., NX, NY, NZ/2+1]
    as A_k2a's inverse reads them.  rdft3dsort(-1) (fftsg3d.c:632-655) packs
    both planes into one half spectrum before rdft3d: it keeps, on kz = 0, the
    rows 0 < j < NY/2 and the entries i <= NX/2 of the rows j = 0, NY/2; on
    kz = NZ/2, the rows j > NY/2 and the entries i > NX/2 of the rows j = 0,
    NY/2; at the four self-conjugate points (i in {0, NX/2}, j in {0, NY/2})
    the real part only.  Every other entry is implied as the conjugate of its
    partner (-i, -j).  The result is Hermitian on both planes, so irfftn of it
    equals the reference's inverse also for a field that is not (a gradient
    i k a keeps +N/2 at the Nyquist wavenumber on both partners)."""
    out = np.array(ak, dtype=np.complex128, copy=True)
    nx, ny = out.shape[-3], out.shape[-2]
    h1, h2 = nx // 2, ny // 2
    i = np.arange(nx)[:, None]
    j = np.arange(ny)[None, :]
    edge = (j == 0) | (j == h2)
    selfc = edge & ((i == 0) | (i == h1))
    drops = ((j > h2) | (edge & (i > h1)), ((j > 0) & (j < h2)) | (edge & (i > 0) & (i < h1)))
    pi, pj = (nx - i) % nx, (ny - j) % ny
    for kz, drop in ((0, drops[0]), (out.shape[-1] - 1, drops[1])):
        plane = out[..., kz]
        partner = np.conj(plane[..., pi, pj])
        fixed = np.where(drop, partner, np.where(selfc, plane.real + 0j, plane))
        out[..., kz] = fixed
    return out


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
        """A_k2a (fft_wrapper.h:662-681).  Exact for a field that is Hermitian
        on the kz = 0 and kz = NZ/2 planes; any other goes through
        ooura_packed_planes first."""
        return np.fft.irfftn(ooura_packed_planes(ak), s=(self.NX, self.NY, self.NZ), axes=(-3, -2, -1))

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


# ============================================================================
# Lees-Edwards (oblique coordinates) step: Time_evolution_hydro_OBL
# (sp_3d_ns.cxx:328-433) for Shear_Navier_Stokes_Lees_Edwards with DC shear.
# ============================================================================
class OracleSPMLE(OracleSPM):
    """Sheared suspension: the velocity field is held in oblique (sheared)
    coordinates with contravariant components; degree_oblique grows by
    Shear_rate * dt per step."""

    def __init__(self, cfg, particles):
        self.gamma = 0.0            # degree_oblique (zero-initialised global)
        self.srate_eff = 0.0        # Shear_rate_eff (zero until the first step)
        self.strain = 0.0           # Shear_strain_realized (input.cxx:808)
        self.stress = {}
        super().__init__(cfg, particles)
        self.xy_aspect = self.NX / self.NY
        # Show_parameter zeroes v_x and omega_z of every particle of a sheared
        # run after the initial projection (init_particle.cxx:767-781).
        self.v[:, 0] = 0.0
        self.v_old[:, 0] = 0.0
        self.omega[:, 2] = 0.0
        self.omega_old[:, 2] = 0.0

    # ---- metric helpers -------------------------------------------------
    def contra2co(self, v):
        """contra2co_single (fft_wrapper.h:613-622)."""
        g = self.gamma
        return np.stack([v[0] + g * v[1], g * v[0] + (1.0 + g * g) * v[1], v[2]])

    def update_k2_obl(self):
        """Update_K2_OBL (fluid_solver.h:342-361)."""
        self.K2 = self.kx ** 2 + (self.ky - self.kx * self.gamma) ** 2 + self.kz ** 2
        with np.errstate(divide="ignore"):
            self.IK2 = np.where(self.K2 > 0.0, 1.0 / np.where(self.K2 > 0, self.K2, 1.0), 0.0)

    def zeta_k2u_k_obl(self, zeta, uk_dc):
        """Zeta_k2u_k_OBL (fft_wrapper.cxx:690-768): case split on KX / KZ,
        omega contra -> co, u = i k x omega_co / K2."""
        kx, ky, kz, ik2 = self.kx, self.ky, self.kz, self.IK2
        z0, z1 = zeta[0], zeta[1]
        cx = self.KX != 0
        cz = (self.KX == 0) & (self.KZ != 0)
        with np.errstate(divide="ignore", invalid="ignore"):
            inv_kx = np.where(cx, 1.0 / np.where(cx, kx, 1.0), 0.0)
            dmy = np.where(self.KZ != 0, -(ky / np.where(self.KZ != 0, kz, 1.0)), 0.0)
        om = np.stack([np.where(cx, -inv_kx * (ky * z0 + kz * z1), np.where(cz, z1, z0)),
                       np.where(cx, z0, np.where(cz, z0, 0.0)),
                       np.where(cx, z1, np.where(cz, dmy * z0, z1))])
        om = self.contra2co(om)
        kx, ky, kz = kx * ik2, ky * ik2, kz * ik2
        u = np.stack([1j * (ky * om[2] - kz * om[1]), 1j * (kz * om[0] - kx * om[2]),
                      1j * (kx * om[1] - ky * om[0])])
        for d in range(3):
            u[d, 0, 0, 0] = complex(uk_dc[d], u[d, 0, 0, 0].imag)
        return u

    def zeta_k2omega_k_obl(self, zeta):
        """Zeta_k2omega_k_OBL (fft_wrapper.cxx:806-845)."""
        kx, ky, kz = self.kx, self.ky, self.kz
        z0, z1 = zeta[0], zeta[1]
        cx = self.KX != 0
        cz = (self.KX == 0) & (self.KZ != 0)
        with np.errstate(divide="ignore", invalid="ignore"):
            inv_kx = np.where(cx, 1.0 / np.where(cx, kx, 1.0), 0.0)
            dmy = np.where(self.KZ != 0, -(ky / np.where(self.KZ != 0, kz, 1.0)), 0.0)
        om = np.stack([np.where(cx, -inv_kx * (ky * z0 + kz * z1), np.where(cz, z1, z0)),
                       np.where(cx, z0, np.where(cz, z0, 0.0)),
                       np.where(cx, z1, np.where(cz, dmy * z0, z1))])
        om[:, 0, 0, 0] = 1j * om[:, 0, 0, 0].imag   # omega[d][0] = 0 (real part only)
        return om

    def omega_to_zeta_obl(self, om):
        """Omega_k2zeta_k_OBL (fft_wrapper.cxx:265-292)."""
        cx = self.KX != 0
        cz = (self.KX == 0) & (self.KZ != 0)
        return np.stack([np.where(cx, om[1], np.where(cz, om[1], om[0])),
                         np.where(cx, om[2], np.where(cz, om[0], om[2]))])

    def u_k2zeta_k_obl(self, uk):
        """U_k2zeta_k_OBL (fft_wrapper.cxx:528-589)."""
        uk_dc = np.array([uk[d, 0, 0, 0].real for d in range(3)])
        uc = self.contra2co(uk)
        kx, ky, kz = self.kx, self.ky, self.kz
        om = np.stack([1j * (ky * uc[2] - kz * uc[1]), 1j * (kz * uc[0] - kx * uc[2]),
                       1j * (kx * uc[1] - ky * uc[0])])
        return self.omega_to_zeta_obl(om), uk_dc

    def solenoidal_uk_obl(self, uk):
        """Solenoidal_uk_OBL (operate_omega.cxx:197-227)."""
        g = self.gamma
        kx, ky, kz = self.kx, self.ky, self.kz
        kxc = (1.0 + g * g) * kx - g * ky
        kyc = -g * kx + ky
        dmy = self.IK2 * (uk[0] * kx + uk[1] * ky + uk[2] * kz)
        return np.stack([uk[0] - dmy * kxc, uk[1] - dmy * kyc, uk[2] - dmy * kz])

    # ---- oblique <-> Cartesian grids ------------------------------------
    def _shift_params(self, j, to_oblique):
        g = self.gamma
        dj = j - self.NY // 2
        sign = float(dj) if g >= 0.0 else float(-dj)
        if dj != 0:
            sign = sign / abs(sign)
        base = float(int(sign * g * dj))
        if to_oblique:   # orth2obl (fft_wrapper.h:315-327)
            io = base * sign
            alpha = (g * dj - io) * sign
        else:            # obl2orth (fft_wrapper.h:328-340)
            io = base * sign + sign
            alpha = (io - g * dj) * sign
        return io, alpha, sign

    def u_oblique2u(self, uu):
        """U_oblique2u (fft_wrapper.h:515-546), mean flow added."""
        NX, NY = self.NX, self.NY
        out = np.empty_like(uu)
        i = np.arange(NX)
        for j in range(NY):
            io, alpha, sign = self._shift_params(j, False)
            beta = 1.0 - alpha
            i_ob = np.fmod(i + io + 4.0 * NX, NX).astype(int)
            i_p = np.fmod(i + sign + 2.0 * NX, NX).astype(int)
            for d in range(3):
                out[d, i_ob, j, :] = beta * uu[d, i, j, :] + alpha * uu[d, i_p, j, :]
            out[0, i_ob, j, :] += self.gamma * out[1, i_ob, j, :]
            out[0, i_ob, j, :] += self.srate_eff * (j - NY / 2.0)
        return out

    def u2u_oblique(self, uu):
        """U2u_oblique (fft_wrapper.h:486-512), mean flow not removed."""
        NX, NY = self.NX, self.NY
        out = np.empty_like(uu)
        i = np.arange(NX)
        for j in range(NY):
            io, alpha, sign = self._shift_params(j, True)
            beta = 1.0 - alpha
            i_o = np.fmod(i + io + 4.0 * NX, NX).astype(int)
            i_op = np.fmod(i_o + sign + 4.0 * NX, NX).astype(int)
            for d in range(3):
                out[d, :, j, :] = beta * uu[d, i_o, j, :] + alpha * uu[d, i_op, j, :]
            out[0, :, j, :] -= self.gamma * out[1, :, j, :]
        return out

    def reset_u_obl(self, u, flg):
        """Reset_U_OBL (fluid_solver.h:312-337)."""
        NX, NY = self.NX, self.NY
        delta = self.xy_aspect if flg == 0 else -self.xy_aspect
        out = np.empty_like(u)
        i = np.arange(NX)
        for j in range(NY):
            s = float(j - NY // 2)
            if s != 0:
                s = s / abs(s)
            io = float(int(s * (j - NY // 2)) * s)
            i_obl = np.fmod(i + delta * io + 4.0 * NX, NX).astype(int)
            out[0, i_obl, j, :] = u[0, i, j, :] + delta * u[1, i, j, :]
            out[1, i_obl, j, :] = u[1, i, j, :]
            out[2, i_obl, j, :] = u[2, i, j, :]
        return out

    # ---- stencil geometry with the Lees-Edwards image ---------------------
    def stencil_geometry_obl(self, x):
        """Particle_cell + Relative_coord_check_stepover_Y + Distance_OBL
        (make_phi.h:114-139, 229-265; interaction.h:50-72)."""
        dx = self.DX
        NX, NY, NZ = self.NX, self.NY, self.NZ
        Lx, Ly, Lz = self.L
        g = self.gamma
        dmy = x * (1.0 / dx)
        x_int = np.trunc(dmy).astype(np.int64)
        residue = (dmy - x_int) * dx
        cell = self.cells[None, :, :]
        yy = x_int[:, None, 1] + cell[..., 1]
        rm1 = (yy + NY) % NY
        sgn = np.sign(yy - rm1).astype(np.int64)
        fx = np.fmod(x_int[:, None, 0] - sgn * g * NY + residue[:, None, 0] / dx + cell[..., 0] + 4 * NX, NX)
        rm0 = fx.astype(np.int64)
        xres = fx - rm0
        rm2 = (x_int[:, None, 2] + cell[..., 2] + NZ) % NZ
        r = np.stack([cell[..., 0] * dx - xres * dx, cell[..., 1] * dx - residue[:, None, 1],
                      cell[..., 2] * dx - residue[:, None, 2]], axis=-1)
        # Distance_OBL(x_mesh, x_p)
        xm = np.stack([rm0, rm1, rm2], axis=-1) * dx
        y12 = x[:, None, 1] - xm[..., 1]
        sy = y12.copy()
        y12 = y12 - nint(y12 / Ly) * Ly
        sy = sy - y12
        s = np.trunc(sy).astype(np.int64)
        s = np.sign(s)
        x12 = x[:, None, 0] - (xm[..., 0] + s * g * Ly)
        x12 = x12 - nint(x12 / Lx) * Lx
        z12 = x[:, None, 2] - xm[..., 2]
        z12 = z12 - nint(z12 / Lz) * Lz
        dist = np.sqrt(y12 ** 2 + x12 ** 2 + z12 ** 2)
        flat = (rm0 * NY + rm1) * NZ + rm2
        return flat, r, dist, sgn, rm1

    def make_phi_particle_sum_obl(self):
        """Make_phi_particle_sum_OBL (make_phi.cxx:262-311)."""
        flat, r, dist, sgn, rm1 = self.stencil_geometry_obl(self.x)
        ph = self.profile(dist)
        phi_sum = np.zeros(self.NX * self.NY * self.NZ)
        np.add.at(phi_sum, flat.ravel(), ph.ravel())
        self.phi_sum = phi_sum.reshape(self.NX, self.NY, self.NZ)
        self.phi = np.minimum(self.phi_sum, 1.0)

    def calc_f_hydro_obl(self, ucp):
        """Calc_f_hydro_correct_precision_OBL (md_force.cxx:508-745), with the
        sums of the Hydro_force / Hydro_force_new fields that
        Mean_shear_stress reduces (fluid_solver.h:253-279)."""
        flat, r, dist, sgn, rm1 = self.stencil_geometry_obl(self.x)
        Ly = self.L[1]
        rr = np.sqrt(r[..., 0] ** 2 + r[..., 1] ** 2 + r[..., 2] ** 2)
        w = self.profile(rr) / np.maximum(self.phi_sum.ravel()[flat], 1.0)
        ug = ucp.reshape(3, -1)[:, flat]
        vs = self._v_surface(self.v, self.omega, r)
        vs[..., 0] = vs[..., 0] - sgn * self.srate_eff * Ly
        dmy_fp = (vs - np.moveaxis(ug, 0, -1)) * w[..., None]
        force = dmy_fp.sum(axis=1)
        torque = np.stack([r[..., 1] * dmy_fp[..., 2] - r[..., 2] * dmy_fp[..., 1],
                           r[..., 2] * dmy_fp[..., 0] - r[..., 0] * dmy_fp[..., 2],
                           r[..., 0] * dmy_fp[..., 1] - r[..., 1] * dmy_fp[..., 0]], axis=-1).sum(axis=1)
        volume = w.sum(axis=1)
        itrace = (w * rr ** 2).sum(axis=1) * (2.0 / 3.0)
        dmy_ry = rm1 + sgn * Ly
        rho_p = self.cfg.mass_ratio * self.cfg.rho
        A = (dmy_fp[..., 0] * dmy_ry * rho_p).sum(axis=1)
        Y = (dmy_ry * w).sum(axis=1)
        mdf = self.momentum_depend_fr[:, 0]
        sv = -self.cfg.rho * force[:, 0] / volume
        swz = -self.cfg.rho * (torque[:, 1][:, None] * r[..., 2] - torque[:, 2][:, None] * r[..., 1]) / itrace[:, None]
        hf_new = A.sum() + (sv * Y).sum() + (swz * dmy_ry * w).sum()
        sum_force = force[:, 0].sum()
        sum_volume = volume.sum() / self.cfg.rho
        hf_old = A.sum() - ((mdf / volume) * Y).sum() - (sum_force / sum_volume) * Y.sum()
        dmy = -self.d["DX3"] * self.cfg.rho / self.dt
        self.f_hydro = dmy * force
        if self.cfg.rotation:
            self.torque_hydro = dmy * torque
        ivol = self.d["Ivolume"] * self.DX ** 3
        self.stress["hydro_old"] = -hf_old * ivol / self.dt
        self.stress["hydro_new"] = -hf_new * ivol / self.dt

    def make_u_particle_sum_obl(self):
        """Make_u_particle_sum_OBL (make_phi.cxx:356-402)."""
        flat, r, dist, sgn, rm1 = self.stencil_geometry_obl(self.x)
        w = self.profile(dist) / np.maximum(self.phi_sum.ravel()[flat], 1.0)
        vs = self._v_surface(self.v, self.omega, r)
        vs[..., 0] = vs[..., 0] - sgn * self.srate_eff * self.L[1]
        vs = vs * w[..., None]
        up = np.zeros((3, self.NX * self.NY * self.NZ))
        for dd in range(3):
            np.add.at(up[dd], flat.ravel(), vs[..., dd].ravel())
        return up.reshape(3, self.NX, self.NY, self.NZ)

    def pbc_obl(self):
        """MD_solver_position_*_OBL wrap: PBC_OBL (periodic_boundary.h:26-45)."""
        Lx, Ly, Lz = self.L
        for n in range(self.np):
            sy = self.x[n, 1]
            self.x[n, 1] = math.fmod(self.x[n, 1] + Ly, Ly)
            s = int(sy - self.x[n, 1])
            if s != 0:
                s = s // abs(s)
            self.x[n, 0] -= s * self.gamma * Ly
            self.x[n, 0] = math.fmod(self.x[n, 0] + Lx, Lx)
            self.x[n, 2] = math.fmod(self.x[n, 2] + Lz, Lz)
            dvx = -s * self.srate_eff * Ly
            self.v[n, 0] += dvx
            self.v_old[n, 0] += dvx

    def calc_f_lennard_jones_obl(self):
        """Calc_f_Lennard_Jones_shear_cap_primitive with Distance0_OBL
        (md_force.cxx:198-304, interaction.h:50-72)."""
        d = self.d
        sigma, cutoff, eps = d["LJ_dia"], d["A_R_cutoff"] * d["LJ_dia"], self.cfg.epsilon
        Lx, Ly, Lz = self.L
        ss0 = 0.0
        for n in range(self.np):
            for m in range(n + 1, self.np):
                x1, x2 = self.x[n], self.x[m]
                y12 = x2[1] - x1[1]
                sy = y12
                y12 -= nint(np.array(y12 / Ly)) * Ly
                sy -= y12
                s = int(sy)
                if s != 0:
                    s = s // abs(s)
                x12 = x2[0] - (x1[0] + s * self.gamma * Ly)
                x12 -= nint(np.array(x12 / Lx)) * Lx
                z12 = x2[2] - x1[2]
                z12 -= nint(np.array(z12 / Lz)) * Lz
                rij = math.sqrt(y12 * y12 + x12 * x12 + z12 * z12)
                if rij < cutoff:
                    sg = sigma / rij
                    s6 = (sg * sg) * (sg * sg) * (sg * sg)
                    lj = 24.0 * eps / (rij * rij) * (2.0 * s6 * s6 - s6)
                    dmy_r = min(DBL_MAX / rij, lj)
                    fn = dmy_r * -np.array([float(x12), float(y12), float(z12)])
                    self.fr[m] -= fn
                    self.fr[n] += fn
                    ss0 += fn[0] * float(y12)
        self.dev_shear_stress_lj = ss0

    def velocity_obl(self, euler):
        """MD_solver_velocity_*_OBL (particle_solver.cxx:336-432) with Force_OBL
        (particle_solver.h:113-128)."""
        self.dev_shear_stress_lj = 0.0
        if self.cfg.lj_truncate in ("ON", "OFF"):
            self.calc_f_lennard_jones_obl()
        if any(f != 0.0 for f in self.cfg.body_force):
            self.fr += np.array(self.cfg.body_force)[None, :]
        self.dev_shear_stress_lj *= self.d["Ivolume"]
        imass, imoi = self.d["IMASS"], self.d["IMOI"]
        h = self.dt if euler else self.hdt
        self.v_old, self.omega_old = self.v.copy(), self.omega.copy()
        if euler:
            self.v = self.v + h * imass * (self.f_hydro + self.fr)
            self.omega = self.omega + h * imoi * (self.torque_hydro + self.torque_r)
            self.momentum_depend_fr = self.dt * self.fr
        else:
            self.v = self.v + h * imass * (2.0 * self.f_hydro + self.fr + self.fr_previous)
            self.omega = self.omega + h * imoi * (2.0 * self.torque_hydro + self.torque_r + self.torque_r_previous)
            self.momentum_depend_fr = self.hdt * (self.fr + self.fr_previous)
        self.reset_forces()

    def reynolds_stress(self, ucp):
        """Calc_Reynolds_shear_stress (fluid_solver.h:165-183)."""
        j = np.arange(self.NY)[None, :, None]
        dy = (j - self.NY // 2) * self.DX
        s = np.sum((ucp[0] - self.srate_eff * dy) * ucp[1])
        return -(self.d["Ivolume"] * self.DX ** 3) * self.cfg.rho * s

    def shear_rate_correction(self, u0):
        """Calc_shear_rate_eff (sp_3d_ns.h:166-203)."""
        g = self.gamma
        ip = np.roll(u0, -1, axis=0)
        im = np.roll(u0, 1, axis=0)
        f_p1 = 0.5 * ((1 - g) * np.roll(ip, -1, axis=1) + (1 + g) * np.roll(im, -1, axis=1))
        f_m1 = 0.5 * ((1 - g) * np.roll(im, 1, axis=1) + (1 + g) * np.roll(ip, 1, axis=1))
        s = np.sum((f_p1 - f_m1) * (1.0 / (2.0 * self.DX)))
        return s * self.d["Ivolume"] * self.DX ** 3

    def step(self):
        if self.cfg.equation != "Shear_Navier_Stokes_Lees_Edwards":
            return super().step()
        cfg = self.cfg
        if not hasattr(self, "momentum_depend_fr"):
            self.momentum_depend_fr = np.zeros((self.np, 3))
        # NS_solver_slavedEuler_Shear_OBL with Zeta_k2advection_k_OBL
        # (fluid_solver.cxx:411-437, operate_omega.cxx:100-155)
        self.zeta = self.truncate(self.zeta)
        uk = self.zeta_k2u_k_obl(self.zeta, self.uk_dc)
        uky = uk[1].copy()
        u = self.ifft(uk)
        w = self.ifft(self.zeta_k2omega_k_obl(self.zeta))
        a = np.stack([u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]])
        ak = self.fft(a)
        ak[0] = ak[0] - 2.0 * self.srate_eff * uky
        ak[1] = ak[1] - 2.0 * self.srate_eff * self.gamma * uky
        kx, ky, kz = self.kx, self.ky, self.kz
        rot = np.stack([1j * (ky * ak[2] - kz * ak[1]), 1j * (kz * ak[0] - kx * ak[2]), 1j * (kx * ak[1] - ky * ak[0])])
        f_ns0 = self.omega_to_zeta_obl(rot)
        nu = cfg.eta / cfg.rho
        dmy = np.exp((-nu * self.dt) * self.K2) - 1.0
        upd = self.zeta + dmy * (self.zeta - ((1.0 / nu) * self.IK2) * f_ns0)
        self.zeta = np.where(self.keep, upd, self.zeta)
        # FIX_CELL (y always fixed under Lees-Edwards, input.cxx:1893-1896)
        for dd in range(3):
            if cfg.fix_cell[dd] or dd == 1:
                self.uk_dc[dd] = 0.0
        u = self.ifft(self.zeta_k2u_k_obl(self.zeta, self.uk_dc))
        self.srate_eff = cfg.shear_rate
        self.gamma += self.srate_eff * self.dt
        if self.gamma >= self.xy_aspect:
            u = self.reset_u_obl(u, 0)
            self.gamma -= self.xy_aspect
        elif self.gamma <= -self.xy_aspect:
            u = self.reset_u_obl(u, 1)
            self.gamma += self.xy_aspect
        self.update_k2_obl()
        ucp = self.u_oblique2u(u)
        self.srate_eff += self.shear_rate_correction(u[0])
        # particles
        euler = self.ts == 0
        self.x_previous = self.x.copy()
        dxp = self.dt * self.v if euler else self.hdt * (3.0 * self.v - self.v_old)
        self.x_nopbc = self.x_nopbc + dxp
        self.x = self.x + dxp
        self.pbc_obl()
        if cfg.rotation:
            if euler:
                self.q_old = self.q.copy()
                self.q = qtn_normalize(self.q + qdot_space(self.q, self.omega) * self.dt)
            else:
                dq = qdot_space(self.q, self.omega)
                dq_old = qdot_space(self.q_old, self.omega_old)
                self.q_old = self.q.copy()
                self.q = qtn_normalize((self.q + dq * (3.0 * self.hdt)) + dq_old * (-self.hdt))
        self.make_phi_particle_sum_obl()
        self.calc_f_hydro_obl(ucp)
        self.stress["reynolds"] = self.reynolds_stress(ucp)
        self.velocity_obl(euler)
        if cfg.kbt > 0.0:
            self.thermostat()
        up = self.make_u_particle_sum_obl()
        f = up - self.phi[None] * ucp
        u = u + self.u2u_oblique(f)
        uk = self.solenoidal_uk_obl(self.fft(u))
        self.zeta, self.uk_dc = self.u_k2zeta_k_obl(uk)
        self.u = u
        self.ts += 1
        self.time += self.dt
        # main loop bookkeeping and Mean_shear_stress (sp_3d_ns.cxx:960-965,
        # sp_3d_ns.h:296-339)
        self.strain += self.srate_eff * self.dt
        fluid = cfg.eta * self.srate_eff
        self.stress.update(dict(time=self.time, shear_rate=self.srate_eff, degree_oblique=self.gamma,
                                strain=self.strain, lj=self.dev_shear_stress_lj, fluid=fluid))
        self.stress["apparent"] = self.stress["hydro_new"] + self.stress["reynolds"] + self.dev_shear_stress_lj + fluid

    def velocity_field_obl(self):
        """Oblique (contravariant) real-space velocity rebuilt from zeta."""
        return self.ifft(self.zeta_k2u_k_obl(self.zeta, self.uk_dc))
