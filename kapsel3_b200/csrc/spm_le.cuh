// Lees-Edwards (sheared) step: kernels in oblique coordinates.
//
// The velocity field is held on the sheared grid with contravariant
// components; degree_oblique (gamma) grows by Shear_rate*dt per step
// (Time_evolution_hydro_OBL, sp_3d_ns.cxx:328-433).  gamma is tracked on the
// host and passed by value; Shear_rate_eff (which the reference corrects by a
// field average every step, sp_3d_ns.h:189-203) lives on the device.
#pragma once

#include "spm_common.cuh"
#include "spm_kernels.cuh"

namespace spm {

// Field slots the Lees-Edwards step needs beyond the common arena: the
// Cartesian velocity ucp (3) and one spare.
constexpr int LE_EXTRA_SLOTS = 4;

// Device-side scalars of the sheared run.
struct LEDev {
    double srate_eff;   // Shear_rate_eff
    double strain;      // Shear_strain_realized
    double correction;  // field-average part of Calc_shear_rate_eff
    double reynolds;    // Inertia_stress (Calc_Reynolds_shear_stress)
    double hydro_old;   // hydro_stress[1][0] from Hydro_force
    double hydro_new;   // hydro_stress[1][0] from Hydro_force_new
    double lj;          // dev_shear_stress_lj * Ivolume
    double time;
};

struct LEState {
    int     enabled        = 0;
    double  shear_rate     = 0.0;
    double  degree_oblique = 0.0;
    double  xy_aspect      = 1.0;
    LEDev  *dev            = nullptr;  // device scalars
    double *ppart          = nullptr;  // per-particle stress partials [Np][kLePart]
    double *partial        = nullptr;  // per-CTA partial sums of the field reductions
    double  stress_host[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

// ---------------------------------------------------------------------------
// k-space helpers (oblique metric)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double ik2_obl(const KPoint &p, double gam) {
    const double a  = p.ky - p.kx * gam;
    const double k2 = p.kx * p.kx + a * a + p.kz * p.kz;  // Update_K2_OBL (fluid_solver.h:342-361)
    return k2 > 0.0 ? 1.0 / k2 : 0.0;
}
__device__ __forceinline__ double k2_obl(const KPoint &p, double gam) {
    const double a = p.ky - p.kx * gam;
    return p.kx * p.kx + a * a + p.kz * p.kz;
}

// reduced contravariant vorticity -> full (case split on KX, then KZ:
// Zeta_k2u_k_OBL / Zeta_k2omega_k_OBL, fft_wrapper.cxx:714-745, 806-845)
template <typename T>
__device__ __forceinline__ void zeta_to_omega_obl(const KPoint &p, cplx<T> z0, cplx<T> z1, cplx<T> om[3]) {
    if (p.KX != 0) {
        const T a  = -(T)(1.0 / p.kx);
        const T ky = (T)p.ky, kz = (T)p.kz;
        om[0]      = cplx<T>{a * (ky * z0.re + kz * z1.re), a * (ky * z0.im + kz * z1.im)};
        om[1]      = z0;
        om[2]      = z1;
    } else if (p.KZ != 0) {
        const T dmy = (T)(-(p.ky / p.kz));
        om[0]       = z1;
        om[1]       = z0;
        om[2]       = cplx<T>{dmy * z0.re, dmy * z0.im};
    } else {
        om[0] = z0;
        om[1] = cplx<T>{0, 0};
        om[2] = z1;
    }
}
// Omega_k2zeta_k_OBL (fft_wrapper.cxx:265-292)
template <typename T>
__device__ __forceinline__ void omega_to_zeta_obl(const KPoint &p, const cplx<T> om[3], cplx<T> &z0, cplx<T> &z1) {
    if (p.KX != 0) {
        z0 = om[1];
        z1 = om[2];
    } else if (p.KZ != 0) {
        z0 = om[1];
        z1 = om[0];
    } else {
        z0 = om[0];
        z1 = om[2];
    }
}
// contra2co_single (fft_wrapper.h:613-622)
template <typename T>
__device__ __forceinline__ void contra2co(cplx<T> v[3], T g) {
    const cplx<T> a = v[0], b = v[1];
    v[0]            = cplx<T>{a.re + g * b.re, a.im + g * b.im};
    v[1]            = cplx<T>{g * a.re + ((T)1 + g * g) * b.re, g * a.im + ((T)1 + g * g) * b.im};
}

// u_hat (contravariant) from zeta: Zeta_k2u_k_OBL (fft_wrapper.cxx:690-768)
template <typename T>
__device__ __forceinline__ void zeta_to_u_obl(const KPoint &p, cplx<T> z0, cplx<T> z1, double gam, cplx<T> u[3]) {
    cplx<T> om[3];
    zeta_to_omega_obl<T>(p, z0, z1, om);
    contra2co<T>(om, (T)gam);
    const T ik2 = (T)ik2_obl(p, gam);
    i_cross<T>((T)p.kx * ik2, (T)p.ky * ik2, (T)p.kz * ik2, om, u);
}

// ---------------------------------------------------------------------------
// zeta -> u_hat (contra) [+ omega_hat] of the oblique advection term
// (Zeta_k2u_cpuky + Zeta_k2omega_OBL, operate_omega.h:150-185).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_le_zeta_to_u(Grid g, const cplx<T> *__restrict__ z0p, const cplx<T> *__restrict__ z1p,
                               const double *__restrict__ uk_dc, double gam, int truncate, cplx<T> *__restrict__ u0,
                               cplx<T> *__restrict__ u1, cplx<T> *__restrict__ u2, cplx<T> *__restrict__ w0,
                               cplx<T> *__restrict__ w1, cplx<T> *__restrict__ w2) {
    const size_t n = g.field_elems_c();
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        KPoint p;
        size_t row;
        cplx<T> u[3] = {{0, 0}, {0, 0}, {0, 0}}, om[3] = {{0, 0}, {0, 0}, {0, 0}};
        const bool in = k_point(g, idx, p, row);
        if (in && (p.keep || !truncate)) {
            const cplx<T> z0 = z0p[idx], z1 = z1p[idx];
            zeta_to_u_obl<T>(p, z0, z1, gam, u);
            if (w0) zeta_to_omega_obl<T>(p, z0, z1, om);
        }
        if (idx == 0) {
            u[0].re = (T)uk_dc[0];
            u[1].re = (T)uk_dc[1];
            u[2].re = (T)uk_dc[2];
            om[0].re = om[1].re = om[2].re = (T)0;  // omega[d][0] = 0 (fft_wrapper.cxx:841-843)
        }
        u0[idx] = u[0];
        u1[idx] = u[1];
        u2[idx] = u[2];
        if (w0) {
            w0[idx] = om[0];
            w1[idx] = om[1];
            w2[idx] = om[2];
        }
    }
}

// a = u x omega (real space, operate_omega.cxx:113-136), in place over u.
template <typename T>
__global__ void r_le_cross(Grid g, T *__restrict__ u0, T *__restrict__ u1, T *__restrict__ u2,
                           const T *__restrict__ w0, const T *__restrict__ w1, const T *__restrict__ w2) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= g.nz) continue;
        const T a = u0[idx], b = u1[idx], c = u2[idx];
        const T x = w0[idx], y = w1[idx], z = w2[idx];
        u0[idx] = b * z - c * y;
        u1[idx] = c * x - a * z;
        u2[idx] = a * y - b * x;
    }
}

// Oblique advection closure and slaved-Euler update
// (operate_omega.cxx:138-154, fluid_solver.cxx:411-437): a_hat -= 2 srate
// (1, gamma, 0) u_hat_y; f = reduced (i k x a_hat); zeta += (e^{-nu dt K2}-1)
// (zeta - IK2 f / nu) on the retained modes with the oblique K2.
template <typename T>
__global__ void k_le_ns_update(Grid g, cplx<T> *__restrict__ z0p, cplx<T> *__restrict__ z1p,
                               const cplx<T> *__restrict__ a0p, const cplx<T> *__restrict__ a1p,
                               const cplx<T> *__restrict__ a2p, const double *__restrict__ uk_dc,
                               const LEDev *__restrict__ le, double gam, double nu, double dt) {
    const size_t n     = g.field_elems_c();
    const double srate = le->srate_eff;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        KPoint p;
        size_t row;
        if (!k_point(g, idx, p, row)) continue;
        if (!p.keep) {
            z0p[idx] = z1p[idx] = cplx<T>{0, 0};
            continue;
        }
        const cplx<T> z0 = z0p[idx], z1 = z1p[idx];
        cplx<T>       u[3];
        zeta_to_u_obl<T>(p, z0, z1, gam, u);
        if (idx == 0) u[1].re = (T)uk_dc[1];
        cplx<T>  a[3] = {a0p[idx], a1p[idx], a2p[idx]};
        const T  c0   = (T)(2.0 * srate);
        const T  c1   = (T)(2.0 * srate * gam);
        a[0].re -= c0 * u[1].re;
        a[0].im -= c0 * u[1].im;
        a[1].re -= c1 * u[1].re;
        a[1].im -= c1 * u[1].im;
        cplx<T> rot[3];
        i_cross<T>((T)p.kx, (T)p.ky, (T)p.kz, a, rot);
        cplx<T> f0, f1;
        omega_to_zeta_obl<T>(p, rot, f0, f1);
        const double k2 = k2_obl(p, gam);
        T            dmy;
        if (sizeof(T) == 8)
            dmy = (T)(exp(-nu * dt * k2) - 1.0);
        else
            dmy = (T)expm1(-nu * dt * k2);
        const T c = (T)((1.0 / nu) * (k2 > 0.0 ? 1.0 / k2 : 0.0));
        cplx<T> n0 = z0, n1 = z1;
        n0.re += dmy * (z0.re - c * f0.re);
        n0.im += dmy * (z0.im - c * f0.im);
        n1.re += dmy * (z1.re - c * f1.re);
        n1.im += dmy * (z1.im - c * f1.im);
        z0p[idx] = n0;
        z1p[idx] = n1;
    }
}

// Solenoidal_uk_OBL + U_k2zeta_k_OBL (operate_omega.cxx:197-227,
// fft_wrapper.cxx:528-589).
template <typename T>
__global__ void k_le_project_to_zeta(Grid g, const cplx<T> *__restrict__ u0p, const cplx<T> *__restrict__ u1p,
                                     const cplx<T> *__restrict__ u2p, cplx<T> *__restrict__ z0p,
                                     cplx<T> *__restrict__ z1p, double *__restrict__ uk_dc, double gam) {
    const size_t n = g.field_elems_c();
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        KPoint p;
        size_t row;
        if (!k_point(g, idx, p, row)) {
            z0p[idx] = z1p[idx] = cplx<T>{0, 0};
            continue;
        }
        cplx<T>  u[3] = {u0p[idx], u1p[idx], u2p[idx]};
        const T  kx = (T)p.kx, ky = (T)p.ky, kz = (T)p.kz;
        const T  ik2 = (T)ik2_obl(p, gam);
        const T  g1  = (T)gam;
        const T  kxc = ((T)1 + g1 * g1) * kx - g1 * ky;
        const T  kyc = -g1 * kx + ky;
        const T  dr  = ik2 * (u[0].re * kx + u[1].re * ky + u[2].re * kz);
        const T  di  = ik2 * (u[0].im * kx + u[1].im * ky + u[2].im * kz);
        u[0].re -= dr * kxc;
        u[0].im -= di * kxc;
        u[1].re -= dr * kyc;
        u[1].im -= di * kyc;
        u[2].re -= dr * kz;
        u[2].im -= di * kz;
        if (idx == 0) {
            uk_dc[0] = (double)u[0].re;
            uk_dc[1] = (double)u[1].re;
            uk_dc[2] = (double)u[2].re;
        }
        contra2co<T>(u, g1);
        cplx<T> om[3];
        i_cross<T>(kx, ky, kz, u, om);
        cplx<T> a, b;
        omega_to_zeta_obl<T>(p, om, a, b);
        z0p[idx] = a;
        z1p[idx] = b;
    }
}

// ---------------------------------------------------------------------------
// Oblique <-> Cartesian grid transfers (linear interpolation along x).
// ---------------------------------------------------------------------------
struct ShiftRow {
    int    io;     // integer x shift of the row
    int    sign;   // +-1, 0 on the middle row
    double alpha;  // interpolation weight of the neighbour
};
// orth2obl (to_oblique) / obl2orth (fft_wrapper.h:315-340)
__device__ __forceinline__ ShiftRow shift_row(int j, int ny, double gam, bool to_oblique) {
    const int dj  = j - ny / 2;
    double    sgn = gam >= 0.0 ? (double)dj : -(double)dj;
    if (dj != 0) sgn = sgn / fabs(sgn);
    const double base = (double)(int)(sgn * gam * dj);
    ShiftRow     s;
    if (to_oblique) {
        const double io = base * sgn;
        s.io            = (int)io;
        s.alpha         = (gam * dj - io) * sgn;
    } else {
        const double io = base * sgn + sgn;
        s.io            = (int)io;
        s.alpha         = (io - gam * dj) * sgn;
    }
    s.sign = (int)sgn;
    return s;
}
__device__ __forceinline__ int wrap_x(double v, int nx) { return (int)fmod(v, (double)nx); }

// ucp = U_oblique2u(u) (fft_wrapper.h:515-546): Cartesian velocity on the
// Cartesian grid, mean shear flow srate*(j - NY/2) added.  Written as a
// gather over the output points.
template <typename T>
__global__ void r_le_obl2cart(Grid g, const T *__restrict__ u0, const T *__restrict__ u1, const T *__restrict__ u2,
                              T *__restrict__ c0, T *__restrict__ c1, T *__restrict__ c2, double gam,
                              double srate) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * g.nz;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int      k  = (int)(t % g.nz);
        const int      j  = (int)((t / g.nz) % g.ny);
        const int      io = (int)(t / ((size_t)g.nz * g.ny));  // output x index (i_oblique)
        const ShiftRow s  = shift_row(j, g.ny, gam, false);
        // i_oblique = fmod(i + io_shift + 4 NX, NX)  =>  i = (io - io_shift) mod NX
        int i = (io - s.io) % g.nx;
        if (i < 0) i += g.nx;
        const int    ip   = wrap_x((double)i + s.sign + 2.0 * g.nx, g.nx);
        const double beta = 1.0 - s.alpha;
        const size_t a    = ((size_t)i * g.ny + j) * rowlen + k;
        const size_t b    = ((size_t)ip * g.ny + j) * rowlen + k;
        const size_t o    = ((size_t)io * g.ny + j) * rowlen + k;
        const T      vy   = (T)(beta * (double)u1[a] + s.alpha * (double)u1[b]);
        T            vx   = (T)(beta * (double)u0[a] + s.alpha * (double)u0[b]);
        vx += (T)gam * vy;
        vx += (T)(srate * (j - g.ny / 2.0));
        c0[o] = vx;
        c1[o] = vy;
        c2[o] = (T)(beta * (double)u2[a] + s.alpha * (double)u2[b]);
    }
}

// u += U2u_oblique(up - min(phi_sum, 1) ucp)  (Make_f_particle_dt_nonsole,
// Transform_obl_u cartesian2oblique, Add_f_particle; fft_wrapper.h:486-512).
template <typename T>
__global__ void r_le_force_add(Grid g, const T *__restrict__ up0, const T *__restrict__ up1,
                               const T *__restrict__ up2, const T *__restrict__ phis, const T *__restrict__ c0,
                               const T *__restrict__ c1, const T *__restrict__ c2, T *__restrict__ u0,
                               T *__restrict__ u1, T *__restrict__ u2, double gam) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * g.nz;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int      k  = (int)(t % g.nz);
        const int      j  = (int)((t / g.nz) % g.ny);
        const int      i  = (int)(t / ((size_t)g.nz * g.ny));
        const ShiftRow s  = shift_row(j, g.ny, gam, true);
        const int      i0 = wrap_x((double)i + s.io + 4.0 * g.nx, g.nx);
        const int      i1 = wrap_x((double)i0 + s.sign + 4.0 * g.nx, g.nx);
        const size_t   a  = ((size_t)i0 * g.ny + j) * rowlen + k;
        const size_t   b  = ((size_t)i1 * g.ny + j) * rowlen + k;
        const size_t   o  = ((size_t)i * g.ny + j) * rowlen + k;
        auto f = [&](const T *up, const T *c, size_t m) {
            const T ph = phis[m] < (T)1 ? phis[m] : (T)1;
            return (double)(up[m] - ph * c[m]);
        };
        const double beta = 1.0 - s.alpha;
        const double fx   = beta * f(up0, c0, a) + s.alpha * f(up0, c0, b);
        const double fy   = beta * f(up1, c1, a) + s.alpha * f(up1, c1, b);
        const double fz   = beta * f(up2, c2, a) + s.alpha * f(up2, c2, b);
        const T      fyT  = (T)fy;
        u0[o] += (T)fx - (T)gam * fyT;
        u1[o] += fyT;
        u2[o] += (T)fz;
    }
}

// Reset_U_OBL (fluid_solver.h:312-337): remap when |gamma| reaches XYaspect.
template <typename T>
__global__ void r_le_reset(Grid g, const T *__restrict__ u0, const T *__restrict__ u1, const T *__restrict__ u2,
                           T *__restrict__ o0, T *__restrict__ o1, T *__restrict__ o2, double delta) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * g.nz;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int k  = (int)(t % g.nz);
        const int j  = (int)((t / g.nz) % g.ny);
        const int i  = (int)(t / ((size_t)g.nz * g.ny));
        double    sg = (double)(j - g.ny / 2);
        if (sg != 0.0) sg = sg / fabs(sg);
        const double io  = (double)(int)(sg * (j - g.ny / 2)) * sg;
        const int    iob = (int)fmod(i + delta * io + 4.0 * g.nx, (double)g.nx);
        const size_t a   = ((size_t)i * g.ny + j) * rowlen + k;
        const size_t o   = ((size_t)iob * g.ny + j) * rowlen + k;
        o0[o]            = u0[a] + (T)delta * u1[a];
        o1[o]            = u1[a];
        o2[o]            = u2[a];
    }
}

// Field reductions of the step: Calc_shear_rate_eff's average gradient of the
// oblique x velocity (sp_3d_ns.h:166-203) and the Reynolds stress of the
// Cartesian velocity (fluid_solver.h:165-183).  One block-level partial per
// CTA, summed in a fixed order by k_le_finish_reduction.
template <typename T>
__global__ void r_le_reductions(Grid g, const T *__restrict__ u0, const T *__restrict__ c0,
                                const T *__restrict__ c1, double gam, const LEDev *__restrict__ le, int which,
                                double *__restrict__ partial) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * g.nz;
    double       acc    = 0.0;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % g.nz);
        const int j = (int)((t / g.nz) % g.ny);
        const int i = (int)(t / ((size_t)g.nz * g.ny));
        if (which == 0) {
            const int    ip = (i + 1) % g.nx, im = (i + g.nx - 1) % g.nx;
            const int    jp = (j + 1) % g.ny, jm = (j + g.ny - 1) % g.ny;
            auto         at = [&](int a, int b) { return (double)u0[((size_t)a * g.ny + b) * rowlen + k]; };
            const double p1 = 0.5 * ((1 - gam) * at(ip, jp) + (1 + gam) * at(im, jp));
            const double m1 = 0.5 * ((1 - gam) * at(im, jm) + (1 + gam) * at(ip, jm));
            acc += (p1 - m1) * (1.0 / (2.0 * g.dx));
        } else {
            const size_t m = ((size_t)i * g.ny + j) * rowlen + k;
            acc += ((double)c0[m] - le->srate_eff * ((j - g.ny / 2) * g.dx)) * (double)c1[m];
        }
    }
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double a = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = a;
    }
}

// which = 0: Shear_rate_eff = shear_rate + ivol * sum (set once per step)
// which = 1: Inertia_stress = -ivol * RHO * sum
__global__ void k_le_finish_reduction(LEDev *le, const double *partial, int nparts, int which, double ivol,
                                      double rho, double shear_rate) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int i = 0; i < nparts; i++) s += partial[i];
    if (which == 0) {
        le->correction = s * ivol;
        le->srate_eff  = shear_rate + le->correction;
    } else {
        le->reynolds = -ivol * rho * s;
    }
}

// ---------------------------------------------------------------------------
// Stencil with the Lees-Edwards image (Relative_coord_check_stepover_Y,
// make_phi.h:229-265; Distance0_OBL, interaction.h:50-72).
// ---------------------------------------------------------------------------
struct StencilPointLE {
    size_t idx;
    double r[3];
    double dist;   // Distance_OBL(grid point, particle)
    double rnorm;  // |r| (used by Calc_f_hydro_correct_precision_OBL)
    int    sign;   // y stepover (+-1, 0)
    int    rm1;    // grid y index
};

__device__ __forceinline__ void stencil_point_le(const Grid &g, const Phys &ph, const double xp[3], int cell_packed,
                                                 double gam, StencilPointLE &s) {
    const int    c[3] = {(int)(int8_t)(cell_packed & 0xff), (int)(int8_t)((cell_packed >> 8) & 0xff),
                         (int)(int8_t)((cell_packed >> 16) & 0xff)};
    const double idx  = 1.0 / g.dx;
    int          xi[3];
    double       res[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double dmy = xp[d] * idx;
        xi[d]            = (int)dmy;
        res[d]           = (dmy - (double)xi[d]) * g.dx;
    }
    const int yy = xi[1] + c[1];
    const int r1 = (yy + g.ny) % g.ny;
    int       sg = yy - r1;
    if (sg != 0) sg = sg / abs(sg);
    const double fx = fmod((double)xi[0] - sg * gam * g.ny + res[0] / g.dx + c[0] + 4 * g.nx, (double)g.nx);
    const int    r0 = (int)fx;
    const double xr = fx - r0;
    const int    r2 = (xi[2] + c[2] + g.nz) % g.nz;
    s.r[0]          = c[0] * g.dx - xr * g.dx;
    s.r[1]          = c[1] * g.dx - res[1];
    s.r[2]          = c[2] * g.dx - res[2];
    s.rnorm         = sqrt(s.r[0] * s.r[0] + s.r[1] * s.r[1] + s.r[2] * s.r[2]);
    s.sign          = sg;
    s.rm1           = r1;
    // Distance0_OBL(x_mesh, x_p)
    const double xm[3] = {r0 * g.dx, r1 * g.dx, r2 * g.dx};
    double       y12   = xp[1] - xm[1];
    double       sy    = y12;
    y12 -= (double)nint_d(y12 / ph.L[1]) * ph.L[1];
    sy -= y12;
    int sd = (int)sy;
    if (sd != 0) sd = sd / abs(sd);
    double x12 = xp[0] - (xm[0] + (double)sd * gam * ph.L[1]);
    x12 -= (double)nint_d(x12 / ph.L[0]) * ph.L[0];
    double z12 = xp[2] - xm[2];
    z12 -= (double)nint_d(z12 / ph.L[2]) * ph.L[2];
    double d2 = 0.0;
    d2 += y12 * y12;
    d2 += x12 * x12;
    d2 += z12 * z12;
    s.dist = sqrt(d2);
    s.idx  = ((size_t)r0 * g.ny + r1) * (2 * (size_t)g.hnzp) + r2;
}

// Make_phi_particle_sum_OBL (make_phi.cxx:262-311)
template <typename T>
__global__ void s_le_phi_scatter(Grid g, Phys ph, const double *__restrict__ x, const int *__restrict__ cells,
                                 int ncells, double gam, T *__restrict__ phi_sum, unsigned int *err) {
    const int p = blockIdx.y;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ph.np || m >= ncells) return;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    if (!particle_in_box(ph, xp)) {
        if (m == 0) atomicOr(err, (unsigned)SPM_DEVERR_PARTICLE_OUT_OF_BOX);
        return;
    }
    StencilPointLE s;
    stencil_point_le(g, ph, xp, cells[m], gam, s);
    const double v = phi_prof(s.dist, ph.radius, ph.hxi, g.dx);
    if (v != 0.0) atomicAdd(&phi_sum[s.idx], (T)v);
}

// Make_u_particle_sum_OBL (make_phi.cxx:356-402)
template <typename T>
__global__ void s_le_up_scatter(Grid g, Phys ph, const double *__restrict__ x, const double *__restrict__ v,
                                const double *__restrict__ w, const int *__restrict__ cells, int ncells, double gam,
                                const LEDev *__restrict__ le, const T *__restrict__ phi_sum, T *__restrict__ up0,
                                T *__restrict__ up1, T *__restrict__ up2) {
    const int p = blockIdx.y;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ph.np || m >= ncells) return;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    if (!particle_in_box(ph, xp)) return;
    StencilPointLE s;
    stencil_point_le(g, ph, xp, cells[m], gam, s);
    double wgt = phi_prof(s.dist, ph.radius, ph.hxi, g.dx);
    if (wgt == 0.0) return;
    const double ps = (double)phi_sum[s.idx];
    wgt /= (ps > 1.0 ? ps : 1.0);
    double vs[3] = {v[3 * p] - s.sign * le->srate_eff * ph.L[1], v[3 * p + 1], v[3 * p + 2]};
    if (ph.rotation) {
        const double *o = w + 3 * p;
        vs[0] += o[1] * s.r[2] - o[2] * s.r[1];
        vs[1] += o[2] * s.r[0] - o[0] * s.r[2];
        vs[2] += o[0] * s.r[1] - o[1] * s.r[0];
    }
    atomicAdd(&up0[s.idx], (T)(vs[0] * wgt));
    atomicAdd(&up1[s.idx], (T)(vs[1] * wgt));
    atomicAdd(&up2[s.idx], (T)(vs[2] * wgt));
}

// Block-wide sum of K doubles (blockDim.x a multiple of 32, <= 1024); the
// result is valid in thread 0.
template <int K>
__device__ __forceinline__ void block_sumK(double v[K]) {
    __shared__ double red[32][K];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; k++) red[wid][k] = v[k];
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < K; k++) {
            double a = lane < nw ? red[lane][k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
            v[k] = a;
        }
    }
}

// Calc_f_hydro_correct_precision_OBL (md_force.cxx:508-745): force and torque
// of each particle, and per-particle partial sums of the Hydro_force and
// Hydro_force_new fields' totals (all that Mean_shear_stress reads of them).
// ppart[p] = {A, Y, force0, volume, new_p, mdf0/volume * Y, Yy, Yz} with
// Y = sum w dry, Yy = sum w dry r_y, Yz = sum w dry r_z over the particle's
// stencil (dry the cell's y with its image).  Rigid beads (rigid != 0) leave
// the spheres' extra term out of new_p: r_le_stress_new adds the bodies' one
// from Yy and Yz once their forces are summed.
constexpr int kLePart = 8;
struct LeRhoP {
    double v[4];  // RHO_particle of each species
};
template <typename T>
__global__ void s_le_hydro_force(Grid g, Phys ph, const double *__restrict__ x, const double *__restrict__ v,
                                 const double *__restrict__ w, const double *__restrict__ mdf,
                                 const int *__restrict__ cells, int ncells, double gam, const LEDev *__restrict__ le,
                                 LeRhoP rho_s, const T *__restrict__ phi_sum, const T *__restrict__ c0,
                                 const T *__restrict__ c1, const T *__restrict__ c2, double *__restrict__ f_hydro,
                                 double *__restrict__ torque_hydro, double *__restrict__ ppart, int rigid) {
    const int p = blockIdx.x;
    if (p >= ph.np) return;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    const double vp[3] = {v[3 * p], v[3 * p + 1], v[3 * p + 2]};
    const double op[3] = {w[3 * p], w[3 * p + 1], w[3 * p + 2]};
    const double srate = le->srate_eff;
    const double rho_p = rho_s.v[spec_of(ph, p)];
    double       acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // force 3, torque 3, volume, itrace, A
    for (int m = threadIdx.x; m < ncells; m += blockDim.x) {
        StencilPointLE s;
        stencil_point_le(g, ph, xp, cells[m], gam, s);
        double wgt = phi_prof(s.rnorm, ph.radius, ph.hxi, g.dx);
        const double ps = (double)phi_sum[s.idx];
        wgt /= (ps > 1.0 ? ps : 1.0);
        double vs[3] = {vp[0] - s.sign * srate * ph.L[1], vp[1], vp[2]};
        if (ph.rotation) {
            vs[0] += op[1] * s.r[2] - op[2] * s.r[1];
            vs[1] += op[2] * s.r[0] - op[0] * s.r[2];
            vs[2] += op[0] * s.r[1] - op[1] * s.r[0];
        }
        const double fp0 = (vs[0] - (double)c0[s.idx]) * wgt;
        const double fp1 = (vs[1] - (double)c1[s.idx]) * wgt;
        const double fp2 = (vs[2] - (double)c2[s.idx]) * wgt;
        acc[0] += fp0;
        acc[1] += fp1;
        acc[2] += fp2;
        acc[3] += s.r[1] * fp2 - s.r[2] * fp1;
        acc[4] += s.r[2] * fp0 - s.r[0] * fp2;
        acc[5] += s.r[0] * fp1 - s.r[1] * fp0;
        acc[6] += wgt;
        acc[7] += wgt * s.rnorm * s.rnorm;
        acc[8] += fp0 * (s.rm1 + s.sign * ph.L[1]) * rho_p;
    }
    block_sumK<9>(acc);
    __shared__ double tot[9];
    if (threadIdx.x == 0)
        for (int k = 0; k < 9; k++) tot[k] = acc[k];
    __syncthreads();
    const double volume = tot[6], itrace = tot[7] * (2.0 / 3.0);
    const double sv = -ph.rho * tot[0] / volume;
    double       acc2[4] = {0.0, 0.0, 0.0, 0.0};  // Y, new-stress extra term, Yy, Yz
    for (int m = threadIdx.x; m < ncells; m += blockDim.x) {
        StencilPointLE s;
        stencil_point_le(g, ph, xp, cells[m], gam, s);
        double wgt = phi_prof(s.rnorm, ph.radius, ph.hxi, g.dx);
        const double ps = (double)phi_sum[s.idx];
        wgt /= (ps > 1.0 ? ps : 1.0);
        const double dry = s.rm1 + s.sign * ph.L[1];
        const double sw  = -ph.rho * (tot[4] * s.r[2] - tot[5] * s.r[1]) / itrace;
        acc2[0] += dry * wgt;
        acc2[1] += (sv + sw) * dry * wgt;
        acc2[2] += dry * wgt * s.r[1];
        acc2[3] += dry * wgt * s.r[2];
    }
    block_sumK<4>(acc2);
    if (threadIdx.x == 0) {
        const double dmy = -ph.dx3 * ph.rho / ph.dt;
        for (int d = 0; d < 3; d++) f_hydro[3 * p + d] = dmy * tot[d];
        if (ph.rotation)
            for (int d = 0; d < 3; d++) torque_hydro[3 * p + d] = dmy * tot[3 + d];
        double *pp = ppart + kLePart * p;
        pp[0]      = tot[8];
        pp[1]      = acc2[0];
        pp[2]      = tot[0];
        pp[3]      = volume;
        pp[4]      = rigid ? tot[8] : tot[8] + acc2[1];
        pp[5]      = mdf[3 * p] / volume * acc2[0];
        pp[6]      = acc2[2];
        pp[7]      = acc2[3];
    }
}

// Totals of the hydrodynamic stress fields and the LJ stress
// (Calc_hydro_stress, fluid_solver.h:253-279; Force_OBL, particle_solver.h:113-128).
__global__ void k_le_stress_finish(LEDev *le, const double *ppart, const double *lj_stress, int np, double ivol,
                                   double ivolume_lj, double dt, double rho) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double A = 0, Y = 0, F = 0, V = 0, Nw = 0, M = 0, L = 0;
    for (int p = 0; p < np; p++) {
        const double *pp = ppart + kLePart * p;
        A += pp[0];
        Y += pp[1];
        F += pp[2];
        V += pp[3];
        Nw += pp[4];
        M += pp[5];
        L += lj_stress[p];
    }
    const double sum_volume = V / rho;
    const double hf_old     = A - M - (F / sum_volume) * Y;
    le->hydro_old           = -hf_old * ivol / dt;
    le->hydro_new           = -Nw * ivol / dt;
    le->lj                  = L * ivolume_lj;
}

// PBC_OBL wrap after the position update (particle_solver.cxx:283-334,
// periodic_boundary.h:26-45): crossing the y boundary shifts x by the
// oblique image and v_x by -+ Shear_rate_eff * LY.  Obstacles stay where
// they are (the wrap sits inside the non-obstacle branch there).
__global__ void p_le_wrap(Phys ph, PState s, double gam, const LEDev *__restrict__ le) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ph.np || ph.janus_prop == 3) return;
    const double dvx = pbc_obl(ph, s.x + 3 * n, gam, le->srate_eff);
    s.v[3 * n] += dvx;
    s.v_old[3 * n] += dvx;
}

// Show_parameter zeroes v_x and omega_z of a sheared run after the initial
// projection (init_particle.cxx:767-781).
__global__ void p_le_zero_vx(Phys ph, PState s) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ph.np) return;
    s.v[3 * n] = s.v_old[3 * n] = 0.0;
    s.omega[3 * n + 2] = s.omega_old[3 * n + 2] = 0.0;
}

__global__ void k_le_advance(LEDev *le, double dt, double time) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        le->strain += le->srate_eff * dt;
        le->time = time;
    }
}

inline void le_init(LEState &le, const Grid &g, const Phys &, const spm_params &p) {
    le.enabled    = p.equation == SPM_EQ_LEES_EDWARDS;
    le.shear_rate = p.shear_rate;
    le.xy_aspect  = (double)g.nx / (double)g.ny;
}
inline void le_reset(LEState &le) {
    le.degree_oblique = 0.0;
    if (le.dev) cudaMemset(le.dev, 0, sizeof(LEDev));
}

}  // namespace spm
