// Pointwise k-space / real-space kernels, smoothed-profile stencils and the
// particle integrators of the SPM step.  Field element type T is double (FP64
// path) or float (FP32-mixed path); particle state, stencil reductions and
// integrators are always double.
#pragma once

#include "spm_common.cuh"

namespace spm {

// Small per-run device words: uk_dc (the k = 0 velocity, FP64), the step
// counter (0 selects the Euler start of the integrators), the FIX_CELLxyz
// mask and the run's device error word.  Runs of a pool keep theirs in one
// array, run-consecutive, so one copy reads every run's counter and errors.
struct RunWords {
    double       uk_dc[4];
    int          ts;
    int          fix_mask;
    unsigned int err;
    int          pad;
};
constexpr int kRunWordStride = sizeof(RunWords) / sizeof(double);

// ---------------------------------------------------------------------------
// Physical constants of one run, passed by value to every kernel.
// ---------------------------------------------------------------------------
struct Phys {
    double dt, hdt;
    double nu;          // ETA / RHO
    double rho;
    double dx3;
    double radius, hxi;  // RADIUS, XI/2
    double L[3];
    double imass, imoi;
    double lj_sigma, lj_cutoff, lj_eps;
    int    lj_powers;   // 0: 12:6, 1: 24:12, 2: 36:18
    int    lj_on;       // LJ_truncate >= 0
    int    rotation;
    int    fix_cell[3];
    double body_force[3];
    double noise_v, noise_o;  // thermostat intensities (fluct.cxx:14-18)
    int    np;
    int    lc[3];       // reference cell-list cells per axis (md_force.cxx:56-58)
    double cell_len;    // Cell_length * DX (md_force.cxx:14, 59-61)
    // Janus particles (one species): propulsion 0 OFF, 1 TUMBLER, 2 SQUIRMER,
    // 3 OBSTACLE; axis 0 none, 1 x, 2 y, 3 z
    int    janus_prop, janus_axis;
    double janus_force[3], janus_torque[3];  // TUMBLER, body frame
    double slip_b1, slip_mode;               // SQUIRMER: B1, alpha/2
    double slip_c1, slip_c2;                 // SQUIRMER: rotlet C1, rotlet dipole C2
    double xi;                               // XI = A_XI DX
    // particle species: particles [spec_end[s-1], spec_end[s]) are species s
    int    nsp;
    int    spec_end[4];
    double imass_s[4], imoi_s[4];
    double qe_s[4];  // Surface_charge_e per species (Electrolyte)
};

// Mean-shear sustaining force of Shear_Navier_Stokes on the real-space u_x
// (Mean_shear_sustaining_yforce_PBC / _kforce_PBC, fluid_solver.cxx:41-119).
// DC: u_x = -/+ Shear_rate (LY/4) DX on the planes j = NY/4, 3NY/4.  AC:
// u_x = zigzag(j) cos(omega t) everywhere, zigzag = -rate j DX for j < LY/4,
// rate (LY - j DX) in the last quarter, rate (j DX - LY/2) between.
template <typename T>
// fs (optional) receives the change made to u_x, the reference's Shear_force
// (fluid_solver.cxx:71-72, 112), zero off the planes under DC.
__global__ void r_shear_sustain(Grid g, T *__restrict__ u0, int ac, double rate, double ly, double amp,
                                T *__restrict__ fs) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    const double qly = ly / 4., hly = ly / 2.;
    const int    j1 = g.ny / 4, j2 = 3 * g.ny / 4;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= g.nz) continue;
        const int j   = (int)((idx / rowlen) % (size_t)g.ny);
        const T   old = u0[idx];
        if (!ac) {
            if (j == j1) u0[idx] = (T)(-(rate * qly * g.dx));
            if (j == j2) u0[idx] = (T)(rate * qly * g.dx);
        } else {
            const int    q = (int)(j / qly);
            const double v = q == 0 ? -rate * j * g.dx : (q == 3 ? rate * ly - rate * j * g.dx : -rate * hly + rate * j * g.dx);
            u0[idx]        = (T)(v * amp);
        }
        if (fs) fs[idx] = u0[idx] - old;
    }
}

// p[n].spec: the species of particle n (consecutive blocks, species 0 first)
__device__ __forceinline__ int spec_of(const Phys &ph, int n) {
    int s = 0;
    while (s + 1 < ph.nsp && n >= ph.spec_end[s]) s++;
    return s;
}

// k index decomposition: element (i, j, kz) of a k-space field.
struct KPoint {
    int    KX, KY, KZ;
    double kx, ky, kz;
    bool   keep;  // inside the 2/3-rule retained box
};

__device__ __forceinline__ void k_point_ijk(const Grid &g, int i, int j, int kz, KPoint &p) {
    p.KX   = i > g.nx / 2 ? i - g.nx : i;  // Calc_KX_Ooura (fft_wrapper.h:719)
    p.KY   = j > g.ny / 2 ? j - g.ny : j;
    p.KZ   = kz;
    p.kx   = g.wave[0] * (double)p.KX;
    p.ky   = g.wave[1] * (double)p.KY;
    p.kz   = g.wave[2] * (double)p.KZ;
    p.keep = (abs(p.KX) < g.trn[0]) && (abs(p.KY) < g.trn[1]) && (p.KZ < g.trn[2]);
}

__device__ __forceinline__ bool k_point(const Grid &g, size_t idx, KPoint &p, size_t &row) {
    const int kz = (int)(idx % (size_t)g.hnzp);
    row          = idx / (size_t)g.hnzp;
    const int j  = (int)(row % (size_t)g.ny);
    const int i  = (int)(row / (size_t)g.ny);
    if (kz >= g.hnz) return false;
    k_point_ijk(g, i, j, kz, p);
    return true;
}

// The kz = 0 and kz = NZ/2 planes as the reference's inverse transform reads
// them (A_k2a, fft_wrapper.h:662-681).  Its Ooura rdft3d takes a packed half
// spectrum: rdft3dsort(-1) (fftsg3d.c:632-655) keeps, on kz = 0, the rows
// 0 < j < NY/2 and i <= NX/2 of the rows j = 0, NY/2; on kz = NZ/2, the rows
// j > NY/2 and i > NX/2 of the rows j = 0, NY/2; at the four self-conjugate
// points only the real part.  Every other entry of the two planes is implied
// as the conjugate of its partner (-i, -j).  A field that is not Hermitian
// there (a gradient i k a, or u from zeta, at the Nyquist wavenumbers whose
// partner keeps the same +N/2; an oblique Lees-Edwards zeta) is rewritten
// that way, after which any inverse real transform gives the reference's
// result.  Discarded entries read only kept partners, so one pass is
// race-free.  Thread per (plane, i, j); blockIdx.y = field, fields
// fstride_c complex values apart.
template <typename T>
__global__ void k_packed_planes(Grid g, cplx<T> *__restrict__ f, size_t fstride_c) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * g.nx * g.ny) return;
    cplx<T>   *a     = f + (size_t)blockIdx.y * fstride_c;
    const int  plane = t / (g.nx * g.ny);
    const int  i     = (t / g.ny) % g.nx;
    const int  j     = t % g.ny;
    const int  h1 = g.nx / 2, h2 = g.ny / 2;
    const int  kz      = plane ? g.hnz - 1 : 0;
    const bool edge_j  = (j == 0 || j == h2);
    const bool self_cj = edge_j && (i == 0 || i == h1);
    const bool drop    = plane == 0 ? (j > h2 || (edge_j && i > h1)) : ((j > 0 && j < h2) || (edge_j && i > 0 && i < h1));
    const size_t idx   = ((size_t)i * g.ny + j) * g.hnzp + kz;
    if (drop) {
        const cplx<T> v = a[((size_t)((g.nx - i) % g.nx) * g.ny + (g.ny - j) % g.ny) * g.hnzp + kz];
        a[idx]          = cplx<T>{v.re, -v.im};
    } else if (self_cj) {
        a[idx].im = (T)0;
    }
}

// Calls f(idx, p, valid) for the modes a k-space kernel visits.  BOX == 1:
// only the retained 2/3 box; a warp walks one (kx, ky) row at a time with its
// lanes on consecutive kz, so there is no per-element index division.
// BOX == 2: the retained box, one mode per thread.
// BOX == 0: every element of the field (valid = false on row padding).
template <int BOX, class F>
__device__ __forceinline__ void for_modes(const Grid &g, F f) {
    if constexpr (BOX == 2) {
        // retained box, one element per thread (heavier per-mode work: more
        // independent modes in flight than the row walk)
        const int    nyb = 2 * g.trn[1] - 1;
        const size_t n   = g.box_elems();
        for (size_t b = blockIdx.x * (size_t)blockDim.x + threadIdx.x; b < n; b += (size_t)gridDim.x * blockDim.x) {
            const int kz = (int)(b % (size_t)g.trn[2]);
            const int rr = (int)(b / (size_t)g.trn[2]);
            const int iy = rr % nyb, ix = rr / nyb;
            const int i  = ix < g.trn[0] ? ix : ix + g.nx - (2 * g.trn[0] - 1);
            const int j  = iy < g.trn[1] ? iy : iy + g.ny - nyb;
            KPoint    p;
            k_point_ijk(g, i, j, kz, p);
            f(((size_t)i * g.ny + j) * g.hnzp + kz, p, true);
        }
    } else if constexpr (BOX == 1) {
        const int nyb    = 2 * g.trn[1] - 1;
        const int nrows  = (2 * g.trn[0] - 1) * nyb;
        const int lane   = threadIdx.x & 31;
        const int warp   = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
        const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
        for (int rr = warp; rr < nrows; rr += nwarps) {
            const int    iy   = rr % nyb, ix = rr / nyb;
            const int    i    = ix < g.trn[0] ? ix : ix + g.nx - (2 * g.trn[0] - 1);
            const int    j    = iy < g.trn[1] ? iy : iy + g.ny - nyb;
            const size_t base = ((size_t)i * g.ny + j) * g.hnzp;
            for (int kz = lane; kz < g.trn[2]; kz += 32) {
                KPoint p;
                k_point_ijk(g, i, j, kz, p);
                f(base + kz, p, true);
            }
        }
    } else {
        const size_t n = g.field_elems_c();
        for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n;
             idx += (size_t)gridDim.x * blockDim.x) {
            KPoint p;
            size_t row;
            const bool v = k_point(g, idx, p, row);
            f(idx, p, v);
        }
    }
}

template <typename T>
__device__ __forceinline__ T ik2_of(const KPoint &p) {
    const double k2 = p.kx * p.kx + p.ky * p.ky + p.kz * p.kz;
    return k2 > 0.0 ? (T)(1.0 / k2) : (T)0;
}

// reduced vorticity -> full vorticity (Zeta_k2u_k case analysis,
// fft_wrapper.cxx:617-655)
template <typename T>
__device__ __forceinline__ void zeta_to_omega(const KPoint &p, cplx<T> z0, cplx<T> z1, cplx<T> om[3]) {
    if (p.KX != 0) {
        const T a = -(T)(1.0 / p.kx);
        const T ky = (T)p.ky, kz = (T)p.kz;
        om[0] = cplx<T>{a * (ky * z0.re + kz * z1.re), a * (ky * z0.im + kz * z1.im)};
        om[1] = z0;
        om[2] = z1;
    } else if (p.KY != 0) {
        const T dmy = (T)(-(p.kz / p.ky));
        om[0] = z1;
        om[1] = cplx<T>{dmy * z0.re, dmy * z0.im};
        om[2] = z0;
    } else {
        om[0] = z0;
        om[1] = z1;
        om[2] = cplx<T>{0, 0};
    }
}

// full vorticity -> reduced pair (Omega_k2zeta_k, fft_wrapper.cxx:227-263)
template <typename T>
__device__ __forceinline__ void omega_to_zeta(const KPoint &p, const cplx<T> om[3], cplx<T> &z0, cplx<T> &z1) {
    if (p.KX != 0) {
        z0 = om[1];
        z1 = om[2];
    } else if (p.KY != 0) {
        z0 = om[2];
        z1 = om[0];
    } else {
        z0 = om[0];
        z1 = om[1];
    }
}

// i (k x a)
template <typename T>
__device__ __forceinline__ void i_cross(T kx, T ky, T kz, const cplx<T> a[3], cplx<T> out[3]) {
    out[0] = cplx<T>{-(ky * a[2].im - kz * a[1].im), ky * a[2].re - kz * a[1].re};
    out[1] = cplx<T>{-(kz * a[0].im - kx * a[2].im), kz * a[0].re - kx * a[2].re};
    out[2] = cplx<T>{-(kx * a[1].im - ky * a[0].im), kx * a[1].re - ky * a[0].re};
}

// Compensated accumulation (hi, lo) += d by TwoSum (Knuth): hi + lo carries
// the value to about twice the working precision, so the rounding of many
// small FP32 increments does not accumulate in the state.
template <typename T>
__device__ __forceinline__ void comp_add(T &hi, T &lo, T d) {
    const T t  = d + lo;
    const T s  = hi + t;
    const T bp = s - hi;
    lo         = (hi - (s - bp)) + (t - bp);
    hi         = s;
}
template <typename T>
__device__ __forceinline__ void comp_add(cplx<T> &hi, cplx<T> &lo, cplx<T> d) {
    comp_add<T>(hi.re, lo.re, d.re);
    comp_add<T>(hi.im, lo.im, d.im);
}

// ---------------------------------------------------------------------------
// zeta (2/3-truncated on the fly) -> u_hat (3 fields).  Zeta_k2u_k with the
// preceding Truncate_two_third_rule (fft_wrapper.cxx:591-688,
// fft_wrapper.h:754-796).  uk_dc is inserted into the real part of k = 0.
// With `box` only the retained 2/3 box is visited (the pruned inverse passes
// read everything outside it as zero); k_ns_update and k_project_add_curl
// take the same flag and then leave modes outside the box untouched (zero).
// ---------------------------------------------------------------------------
template <typename T, int BOX>
__global__ void k_zeta_to_u(Grid g, const cplx<T> *__restrict__ z0p, const cplx<T> *__restrict__ z1p,
                            const double *__restrict__ uk_dc, cplx<T> *__restrict__ u0, cplx<T> *__restrict__ u1,
                            cplx<T> *__restrict__ u2, int truncate, size_t run_stride_c) {
    const size_t ro = blockIdx.y * run_stride_c;
    z0p += ro, z1p += ro, u0 += ro, u1 += ro, u2 += ro;
    uk_dc += blockIdx.y * kRunWordStride;
    for_modes<BOX>(g, [&](size_t idx, const KPoint &p, bool valid) {
        if (!valid) {
            u0[idx] = u1[idx] = u2[idx] = cplx<T>{0, 0};
            return;
        }
        cplx<T> u[3] = {{0, 0}, {0, 0}, {0, 0}};
        if (p.keep || !truncate) {
            cplx<T> om[3];
            zeta_to_omega<T>(p, z0p[idx], z1p[idx], om);
            const T ik2 = ik2_of<T>(p);
            i_cross<T>((T)p.kx * ik2, (T)p.ky * ik2, (T)p.kz * ik2, om, u);
        }
        if (idx == 0) {
            u[0].re = (T)uk_dc[0];
            u[1].re = (T)uk_dc[1];
            u[2].re = (T)uk_dc[2];
        }
        u0[idx] = u[0];
        u1[idx] = u[1];
        u2[idx] = u[2];
    });
}

// ---------------------------------------------------------------------------
// Real-space quadratic products of U2advection_k (operate_omega.cxx:31-47):
//   u0 <- u2 u3, u1 <- u3 u1, u2 <- u1 u2, a0 <- (u2-u3)(u2+u3), a1 <- (u3-u1)(u3+u1)
// (u1,u2,u3 = x,y,z components).  Rows of 2*hnzp reals, NZ used.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void r_advection_products(Grid g, T *__restrict__ u0, T *__restrict__ u1, T *__restrict__ u2,
                                     T *__restrict__ a0, T *__restrict__ a1) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= g.nz) continue;
        const T x = u0[idx], y = u1[idx], z = u2[idx];
        u0[idx] = y * z;
        u1[idx] = z * x;
        u2[idx] = x * y;
        a0[idx] = (y - z) * (y + z);
        a1[idx] = (z - x) * (z + x);
    }
}

// ---------------------------------------------------------------------------
// Curl of the advection term from the FFT'd products, reduction to two
// components and the slaved-Euler update of zeta on the retained modes
// (U2advection_k k-part operate_omega.cxx:57-83, Omega_k2zeta_k,
// NS_solver_slavedEuler fluid_solver.cxx:357-373).  Modes outside the
// retained box are written as zero (the reference truncates zeta in place at
// the start of Zeta_k2advection_k and never updates those modes).
// ---------------------------------------------------------------------------
template <typename T, int BOX>
__global__ void k_ns_update(Grid g, cplx<T> *__restrict__ z0p, cplx<T> *__restrict__ z1p,
                            cplx<T> *__restrict__ p_u2u3, cplx<T> *__restrict__ p_u3u1,
                            cplx<T> *__restrict__ p_u1u2, const cplx<T> *__restrict__ p_a0,
                            const cplx<T> *__restrict__ p_a1, double nu, double dt, size_t run_stride_c,
                            cplx<T> *__restrict__ zl0, cplx<T> *__restrict__ zl1,
                            const RunWords *__restrict__ rw) {
    const size_t ro = blockIdx.y * run_stride_c;
    z0p += ro, z1p += ro, p_u2u3 += ro, p_u3u1 += ro, p_u1u2 += ro, p_a0 += ro, p_a1 += ro;
    if (zl0) zl0 += ro, zl1 += ro;
    if (rw) rw += blockIdx.y;
    for_modes<BOX>(g, [&](size_t idx, const KPoint &p, bool valid) {
        if (!valid) return;
        if (!p.keep) {
            z0p[idx] = z1p[idx] = cplx<T>{0, 0};
            if (zl0) zl0[idx] = zl1[idx] = cplx<T>{0, 0};
            return;
        }
        const T k1 = (T)p.kx, k2 = (T)p.ky, k3 = (T)p.kz;
        const T k1k2 = k1 * k2, k2k3 = k2 * k3, k3k1 = k3 * k1;
        const T c0 = (k3 - k2) * (k3 + k2), c1 = (k1 - k3) * (k1 + k3), c2 = (k2 - k1) * (k2 + k1);
        const cplx<T> u2u3 = p_u2u3[idx], u3u1 = p_u3u1[idx], u1u2 = p_u1u2[idx];
        const cplx<T> a0 = p_a0[idx], a1 = p_a1[idx];
        const cplx<T> a2 = {-a1.re - a0.re, -a1.im - a0.im};
        cplx<T> om[3];
        om[0] = {-(k2k3 * a0.re + c0 * u2u3.re + k3k1 * u1u2.re - k1k2 * u3u1.re),
                 -(k2k3 * a0.im + c0 * u2u3.im + k3k1 * u1u2.im - k1k2 * u3u1.im)};
        om[1] = {-(k3k1 * a1.re + c1 * u3u1.re + k1k2 * u2u3.re - k2k3 * u1u2.re),
                 -(k3k1 * a1.im + c1 * u3u1.im + k1k2 * u2u3.im - k2k3 * u1u2.im)};
        om[2] = {-(k1k2 * a2.re + c2 * u1u2.re + k2k3 * u3u1.re - k3k1 * u2u3.re),
                 -(k1k2 * a2.im + c2 * u1u2.im + k2k3 * u3u1.im - k3k1 * u2u3.im)};
        cplx<T> f0, f1;
        omega_to_zeta<T>(p, om, f0, f1);
        const double k2sum = p.kx * p.kx + p.ky * p.ky + p.kz * p.kz;
        T            dmy, c;
        if (sizeof(T) == 8) {
            dmy = (T)(exp(-nu * dt * k2sum) - 1.0);
        } else {
            dmy = (T)expm1(-nu * dt * k2sum);
        }
        c = (T)((1.0 / nu) * (k2sum > 0.0 ? 1.0 / k2sum : 0.0));
        cplx<T> z0 = z0p[idx], z1 = z1p[idx];
        if (zl0) {
            // compensated state: increment from (hi - c f) + lo, added by TwoSum
            cplx<T> l0 = zl0[idx], l1 = zl1[idx];
            const cplx<T> d0 = {dmy * ((z0.re - c * f0.re) + l0.re), dmy * ((z0.im - c * f0.im) + l0.im)};
            const cplx<T> d1 = {dmy * ((z1.re - c * f1.re) + l1.re), dmy * ((z1.im - c * f1.im) + l1.im)};
            comp_add<T>(z0, l0, d0);
            comp_add<T>(z1, l1, d1);
            zl0[idx] = l0;
            zl1[idx] = l1;
        } else {
            z0.re += dmy * (z0.re - c * f0.re);
            z0.im += dmy * (z0.im - c * f0.im);
            z1.re += dmy * (z1.re - c * f1.re);
            z1.im += dmy * (z1.im - c * f1.im);
        }
        z0p[idx] = z0;
        z1p[idx] = z1;
        if (rw) {
            // Zeta_k2u_k of the new zeta (k_zeta_to_u of the retained box) into the
            // three product slots this mode has just consumed; k = 0 takes uk_dc
            // with the FIX_CELL components zeroed, as k_fix_cell then leaves it
            cplx<T> om[3], u[3] = {{0, 0}, {0, 0}, {0, 0}};
            zeta_to_omega<T>(p, z0, z1, om);
            const T ik2 = ik2_of<T>(p);
            i_cross<T>((T)p.kx * ik2, (T)p.ky * ik2, (T)p.kz * ik2, om, u);
            if (idx == 0)
                for (int d = 0; d < 3; d++) u[d].re = (rw->fix_mask & (1 << d)) ? (T)0 : (T)rw->uk_dc[d];
            p_u2u3[idx] = u[0];
            p_u3u1[idx] = u[1];
            p_u1u2[idx] = u[2];
        }
    });
}

// ---------------------------------------------------------------------------
// Truncate_two_third_rule (fft_wrapper.h:754-796) of the two zeta fields, in
// place over the whole grid: zeta uploaded by the host may carry modes the
// step's retained-box kernels never visit.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_truncate2(Grid g, cplx<T> *__restrict__ z0, cplx<T> *__restrict__ z1) {
    const size_t n = g.field_elems_c();
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        KPoint p;
        size_t row;
        if (k_point(g, idx, p, row) && p.keep) continue;
        z0[idx] = z1[idx] = cplx<T>{0, 0};
    }
}

// ---------------------------------------------------------------------------
// 2/3 truncation + solenoidal projection of three k-space fields
// (Solenoidal_u's k-space part: Truncate_two_third_rule + Solenoidal_uk,
// operate_omega.h:105-112, operate_omega.cxx:171-195).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_truncate_project(Grid g, cplx<T> *__restrict__ f0, cplx<T> *__restrict__ f1,
                                   cplx<T> *__restrict__ f2, int truncate) {
    const size_t n = g.field_elems_c();
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        KPoint p;
        size_t row;
        if (!k_point(g, idx, p, row)) continue;
        if (truncate && !p.keep) {
            f0[idx] = f1[idx] = f2[idx] = cplx<T>{0, 0};
            continue;
        }
        const T kx = (T)p.kx, ky = (T)p.ky, kz = (T)p.kz, ik2 = ik2_of<T>(p);
        cplx<T> a = f0[idx], b = f1[idx], c = f2[idx];
        const T dr = ik2 * (a.re * kx + b.re * ky + c.re * kz);
        const T di = ik2 * (a.im * kx + b.im * ky + c.im * kz);
        a.re -= dr * kx;
        a.im -= di * kx;
        b.re -= dr * ky;
        b.im -= di * ky;
        c.re -= dr * kz;
        c.im -= di * kz;
        f0[idx] = a;
        f1[idx] = b;
        f2[idx] = c;
    }
}

// ---------------------------------------------------------------------------
// u_hat -> zeta and uk_dc (U_k2zeta_k, fft_wrapper.cxx:407-476).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_u_to_zeta(Grid g, const cplx<T> *__restrict__ u0, const cplx<T> *__restrict__ u1,
                            const cplx<T> *__restrict__ u2, cplx<T> *__restrict__ z0p, cplx<T> *__restrict__ z1p,
                            double *__restrict__ uk_dc) {
    const size_t n = g.field_elems_c();
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        KPoint p;
        size_t row;
        if (!k_point(g, idx, p, row)) {
            z0p[idx] = z1p[idx] = cplx<T>{0, 0};
            continue;
        }
        const cplx<T> u[3] = {u0[idx], u1[idx], u2[idx]};
        if (idx == 0) {
            uk_dc[0] = (double)u[0].re;
            uk_dc[1] = (double)u[1].re;
            uk_dc[2] = (double)u[2].re;
        }
        cplx<T> om[3];
        i_cross<T>((T)p.kx, (T)p.ky, (T)p.kz, u, om);
        cplx<T> a, b;
        omega_to_zeta<T>(p, om, a, b);
        z0p[idx] = a;
        z1p[idx] = b;
    }
}

// ---------------------------------------------------------------------------
// Rigidity projection closed in k space.  The reference forms u_real + f_sole
// in real space and transforms it (Make_f_particle_dt_sole, Add_f_particle,
// U2zeta_k; sp_3d_ns.cxx:172-192, f_particle.h:60-84, operate_omega.h:208).
// Because u_real is the inverse transform of the truncated u_hat rebuilt from
// zeta, the same zeta follows pointwise from
//   u_hat_new = Zeta_k2u_k(zeta) + P T f_hat,  zeta_new = U_k2zeta_k(u_hat_new)
// which skips three inverse and three forward transforms.  uk_dc (the k = 0
// mode, not touched by the projection) is updated in FP64:
//   uk_dc += Re f_hat(0).
// Modes outside the 2/3 box come out exactly zero (the reference leaves
// round-off there, which its next step truncates before use).
// ---------------------------------------------------------------------------
template <typename T, int BOX>
__global__ void k_project_add_curl(Grid g, const cplx<T> *__restrict__ f0p, const cplx<T> *__restrict__ f1p,
                                   const cplx<T> *__restrict__ f2p, cplx<T> *__restrict__ z0p,
                                   cplx<T> *__restrict__ z1p, double *__restrict__ uk_dc, size_t run_stride_c,
                                   cplx<T> *__restrict__ zl0, cplx<T> *__restrict__ zl1) {
    const size_t ro = blockIdx.y * run_stride_c;
    f0p += ro, f1p += ro, f2p += ro, z0p += ro, z1p += ro;
    if (zl0) zl0 += ro, zl1 += ro;
    uk_dc += blockIdx.y * kRunWordStride;
    for_modes<BOX>(g, [&](size_t idx, const KPoint &p, bool valid) {
        if (!valid || !p.keep || idx == 0) {
            if (idx == 0) {
                uk_dc[0] += (double)f0p[0].re;
                uk_dc[1] += (double)f1p[0].re;
                uk_dc[2] += (double)f2p[0].re;
            }
            z0p[idx] = z1p[idx] = cplx<T>{0, 0};
            if (zl0) zl0[idx] = zl1[idx] = cplx<T>{0, 0};
            return;
        }
        const T kx = (T)p.kx, ky = (T)p.ky, kz = (T)p.kz, ik2 = ik2_of<T>(p);
        cplx<T> f[3] = {f0p[idx], f1p[idx], f2p[idx]};
        const T dr = ik2 * (f[0].re * kx + f[1].re * ky + f[2].re * kz);
        const T di = ik2 * (f[0].im * kx + f[1].im * ky + f[2].im * kz);
        f[0].re -= dr * kx;
        f[0].im -= di * kx;
        f[1].re -= dr * ky;
        f[1].im -= di * ky;
        f[2].re -= dr * kz;
        f[2].im -= di * kz;
        cplx<T> om[3], u[3];
        if (zl0) {
            // compensated state: curl(i k x omega(zeta) / k^2) = omega exactly
            // for a solenoidal omega, so zeta_new = zeta + zeta(i k x P f);
            // only that increment is formed and added by TwoSum
            i_cross<T>(kx, ky, kz, f, om);
            cplx<T> a, b;
            omega_to_zeta<T>(p, om, a, b);
            cplx<T> z0 = z0p[idx], z1 = z1p[idx], l0 = zl0[idx], l1 = zl1[idx];
            comp_add<T>(z0, l0, a);
            comp_add<T>(z1, l1, b);
            z0p[idx] = z0;
            z1p[idx] = z1;
            zl0[idx] = l0;
            zl1[idx] = l1;
            return;
        }
        zeta_to_omega<T>(p, z0p[idx], z1p[idx], om);
        i_cross<T>(kx * ik2, ky * ik2, kz * ik2, om, u);
#pragma unroll
        for (int d = 0; d < 3; d++) u[d] = cadd(u[d], f[d]);
        i_cross<T>(kx, ky, kz, u, om);
        cplx<T> a, b;
        omega_to_zeta<T>(p, om, a, b);
        z0p[idx] = a;
        z1p[idx] = b;
    });
}

// ---------------------------------------------------------------------------
// Real-space field updates.
// f = up - min(phi_sum, 1) u   (Make_f_particle_dt_nonsole, f_particle.h:35-54)
// written in place over up.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void r_make_f(Grid g, T *__restrict__ up0, T *__restrict__ up1, T *__restrict__ up2,
                         const T *__restrict__ u0, const T *__restrict__ u1, const T *__restrict__ u2,
                         const T *__restrict__ phi_sum) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= g.nz) continue;
        const T ph = phi_sum[idx] < (T)1 ? phi_sum[idx] : (T)1;
        up0[idx]   = up0[idx] - ph * u0[idx];
        up1[idx]   = up1[idx] - ph * u1[idx];
        up2[idx]   = up2[idx] - ph * u2[idx];
    }
}

// u += f  (Add_f_particle, f_particle.h:68-84)
template <typename T>
__global__ void r_add3(Grid g, T *__restrict__ u0, T *__restrict__ u1, T *__restrict__ u2, const T *__restrict__ f0,
                       const T *__restrict__ f1, const T *__restrict__ f2) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= g.nz) continue;
        u0[idx] += f0[idx];
        u1[idx] += f1[idx];
        u2[idx] += f2[idx];
    }
}

// phi = min(phi_sum, 1) over the whole field (Make_phi_particle_sum tail,
// make_phi.cxx:248-259) -- only materialised for the per-function API.
template <typename T>
__global__ void r_phi_clamp(Grid g, const T *__restrict__ phi_sum, T *__restrict__ phi) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= g.nz) continue;
        phi[idx] = phi_sum[idx] < (T)1 ? phi_sum[idx] : (T)1;
    }
}

// ---------------------------------------------------------------------------
// Smoothed profile (profile.h:30-50) and stencil geometry (make_phi.h:114-170,
// interaction.h:113-132).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double H_prof(double x, double dx) {
    if (!(x > 0.0)) return 0.0;
    const double r = dx / x;
    return exp(-(r * r));
}
__device__ __forceinline__ double phi_prof(double x, double radius, double hxi, double dx) {
    const double h1 = H_prof(radius + hxi - x, dx);
    return h1 / (h1 + H_prof(x - radius + hxi, dx));
}
__device__ __forceinline__ int nint_d(double a) { return a >= 0.0 ? (int)(a + 0.5) : (int)(a - 0.5); }

struct StencilPoint {
    size_t idx;   // real-field element index (padded rows)
    double r[3];  // cell * dx - residue
    double dist;  // minimum-image distance grid point <-> particle centre
};

__device__ __forceinline__ void stencil_point(const Grid &g, const Phys &ph, const double xp[3], int cell_packed,
                                              StencilPoint &s) {
    const int    c[3] = {(int)(int8_t)(cell_packed & 0xff), (int)(int8_t)((cell_packed >> 8) & 0xff),
                         (int)(int8_t)((cell_packed >> 16) & 0xff)};
    const int    n[3] = {g.nx, g.ny, g.nz};
    const double idx  = 1.0 / g.dx;
    int          rm[3];
    double       d2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double dmy     = xp[d] * idx;
        const int    x_int   = (int)dmy;
        const double residue = (dmy - (double)x_int) * g.dx;
        rm[d]                = (x_int + c[d] + n[d]) % n[d];
        s.r[d]               = (double)c[d] * g.dx - residue;
        double x12           = xp[d] - (double)rm[d] * g.dx;
        x12 -= (double)nint_d(x12 / ph.L[d]) * ph.L[d];
        d2 += x12 * x12;
    }
    s.dist = sqrt(d2);
    s.idx  = ((size_t)rm[0] * g.ny + rm[1]) * (2 * (size_t)g.hnzp) + rm[2];
}

__device__ __forceinline__ bool particle_in_box(const Phys &ph, const double xp[3]) {
    return xp[0] >= 0.0 && xp[0] < ph.L[0] && xp[1] >= 0.0 && xp[1] < ph.L[1] && xp[2] >= 0.0 && xp[2] < ph.L[2];
}

// phi_sum += Phi over every (particle, Sekibun cell)  (make_phi.cxx:214-247)
template <typename T>
__global__ void s_phi_scatter(Grid g, Phys ph, const double *__restrict__ x, const int *__restrict__ cells,
                              int ncells, T *__restrict__ phi_sum, unsigned int *err) {
    const int p = blockIdx.y;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ph.np || m >= ncells) return;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    if (!particle_in_box(ph, xp)) {
        if (m == 0) atomicOr(err, (unsigned)SPM_DEVERR_PARTICLE_OUT_OF_BOX);
        return;
    }
    StencilPoint s;
    stencil_point(g, ph, xp, cells[m], s);
    const double v = phi_prof(s.dist, ph.radius, ph.hxi, g.dx);
    if (v != 0.0) atomicAdd(&phi_sum[s.idx], (T)v);
}

// up += (v + w x r) Phi / max(phi_sum, 1)   (make_phi.cxx:313-354)
template <typename T>
__global__ void s_up_scatter(Grid g, Phys ph, const double *__restrict__ x, const double *__restrict__ v,
                             const double *__restrict__ w, const int *__restrict__ cells, int ncells,
                             const T *__restrict__ phi_sum, T *__restrict__ up0, T *__restrict__ up1,
                             T *__restrict__ up2) {
    const int p = blockIdx.y;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ph.np || m >= ncells) return;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    if (!particle_in_box(ph, xp)) return;
    StencilPoint s;
    stencil_point(g, ph, xp, cells[m], s);
    double wgt = phi_prof(s.dist, ph.radius, ph.hxi, g.dx);
    if (wgt == 0.0) return;
    const double ps = (double)phi_sum[s.idx];
    wgt /= (ps > 1.0 ? ps : 1.0);
    double vs[3] = {v[3 * p], v[3 * p + 1], v[3 * p + 2]};
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



// Block-wide sum of 6 doubles (blockDim.x a multiple of 32, <= 1024).
__device__ __forceinline__ void block_sum6(double v[6]) {
    __shared__ double red[32][6];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 6; k++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 6; k++) red[wid][k] = v[k];
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            double a = lane < nw ? red[lane][k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
            v[k] = a;
        }
    }
}

// Hydrodynamic force and torque (Calc_f_hydro_correct_precision,
// md_force.cxx:383-506): one CTA per particle, FP64 accumulation.
template <typename T>
__global__ void s_hydro_force(Grid g, Phys ph, const double *__restrict__ x, const double *__restrict__ v,
                              const double *__restrict__ w, const int *__restrict__ cells, int ncells,
                              const T *__restrict__ phi_sum, const T *__restrict__ u0, const T *__restrict__ u1,
                              const T *__restrict__ u2, double *__restrict__ f_hydro,
                              double *__restrict__ torque_hydro) {
    const int p = blockIdx.x;
    if (p >= ph.np) return;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    const double vp[3] = {v[3 * p], v[3 * p + 1], v[3 * p + 2]};
    const double op[3] = {w[3 * p], w[3 * p + 1], w[3 * p + 2]};
    const bool   inbox = particle_in_box(ph, xp);
    double       acc[6] = {0, 0, 0, 0, 0, 0};
    if (inbox) {
        for (int m = threadIdx.x; m < ncells; m += blockDim.x) {
            StencilPoint s;
            stencil_point(g, ph, xp, cells[m], s);
            double wgt = phi_prof(s.dist, ph.radius, ph.hxi, g.dx);
            if (wgt == 0.0) continue;
            const double ps = (double)phi_sum[s.idx];
            wgt /= (ps > 1.0 ? ps : 1.0);
            double vs[3] = {vp[0], vp[1], vp[2]};
            if (ph.rotation) {
                vs[0] += op[1] * s.r[2] - op[2] * s.r[1];
                vs[1] += op[2] * s.r[0] - op[0] * s.r[2];
                vs[2] += op[0] * s.r[1] - op[1] * s.r[0];
            }
            const double fp0 = (vs[0] - (double)u0[s.idx]) * wgt;
            const double fp1 = (vs[1] - (double)u1[s.idx]) * wgt;
            const double fp2 = (vs[2] - (double)u2[s.idx]) * wgt;
            acc[0] += fp0;
            acc[1] += fp1;
            acc[2] += fp2;
            acc[3] += s.r[1] * fp2 - s.r[2] * fp1;
            acc[4] += s.r[2] * fp0 - s.r[0] * fp2;
            acc[5] += s.r[0] * fp1 - s.r[1] * fp0;
        }
    }
    block_sum6(acc);
    if (threadIdx.x == 0) {
        const double dmy = -ph.dx3 * ph.rho / ph.dt;
        for (int d = 0; d < 3; d++) f_hydro[3 * p + d] = dmy * acc[d];
        if (ph.rotation)
            for (int d = 0; d < 3; d++) torque_hydro[3 * p + d] = dmy * acc[3 + d];
    }
}

// ---------------------------------------------------------------------------
// Stencil cache of the step.  The phi scatter evaluates, for every (particle,
// Sekibun cell), the grid index and the profile weight Phi; the hydrodynamic
// force and the phi*v_p scatter of the same step (same positions) read them
// back instead of recomputing the minimum-image distance and the profile.
// sc_idx[p * ncells + m] = -1 where Phi is zero (or the particle is outside
// the box).  Offsets r = cell * dx - residue are rebuilt from the cell.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void particle_residue(const Grid &g, const double xp[3], double res[3]) {
    const double idx = 1.0 / g.dx;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double dmy = xp[d] * idx;
        res[d]           = (dmy - (double)(int)dmy) * g.dx;
    }
}
__device__ __forceinline__ void cell_offset(const Grid &g, int cell_packed, const double res[3], double r[3]) {
    const int c[3] = {(int)(int8_t)(cell_packed & 0xff), (int)(int8_t)((cell_packed >> 8) & 0xff),
                      (int)(int8_t)((cell_packed >> 16) & 0xff)};
#pragma unroll
    for (int d = 0; d < 3; d++) r[d] = (double)c[d] * g.dx - res[d];
}

template <typename T>
__global__ void s_phi_scatter_cache(Grid g, Phys ph, const double *__restrict__ x, const int *__restrict__ cells,
                                    int ncells, T *__restrict__ phi_sum, unsigned int *err, int *__restrict__ sc_idx,
                                    double *__restrict__ sc_w) {
    const int p = blockIdx.y;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ph.np || m >= ncells) return;
    const size_t o     = (size_t)p * ncells + m;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    if (!particle_in_box(ph, xp)) {
        if (m == 0) atomicOr(err, (unsigned)SPM_DEVERR_PARTICLE_OUT_OF_BOX);
        sc_idx[o] = -1;
        return;
    }
    StencilPoint s;
    stencil_point(g, ph, xp, cells[m], s);
    const double v = phi_prof(s.dist, ph.radius, ph.hxi, g.dx);
    sc_idx[o]      = v != 0.0 ? (int)s.idx : -1;
    sc_w[o]        = v;
    if (v != 0.0) atomicAdd(&phi_sum[s.idx], (T)v);
}

// Calc_f_hydro_correct_precision from the stencil cache (same sums as
// s_hydro_force).
template <typename T>
__global__ void s_hydro_force_cached(Grid g, Phys ph, const double *__restrict__ x, const double *__restrict__ v,
                                     const double *__restrict__ w, const int *__restrict__ cells, int ncells,
                                     const int *__restrict__ sc_idx, const double *__restrict__ sc_w,
                                     const T *__restrict__ phi_sum, const T *__restrict__ u0,
                                     const T *__restrict__ u1, const T *__restrict__ u2, double *__restrict__ f_hydro,
                                     double *__restrict__ torque_hydro) {
    const int p = blockIdx.x;
    if (p >= ph.np) return;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    const double vp[3] = {v[3 * p], v[3 * p + 1], v[3 * p + 2]};
    const double op[3] = {w[3 * p], w[3 * p + 1], w[3 * p + 2]};
    double       res[3];
    particle_residue(g, xp, res);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    // U cells per thread per round: their cache entries first, then every
    // gather, then the sums, in the order m = t, t + B, t + 2B, ... of a
    // one-cell loop (the gathers of a round are in flight together)
    constexpr int U = 4;
    for (int m0 = threadIdx.x; m0 < ncells; m0 += U * blockDim.x) {
        int    id[U], cm[U];
        double sw[U];
#pragma unroll
        for (int k = 0; k < U; k++) {
            const int    m = m0 + k * blockDim.x;
            const size_t o = (size_t)p * ncells + m;
            id[k]          = m < ncells ? sc_idx[o] : -1;
            sw[k]          = m < ncells ? sc_w[o] : 0.0;
            cm[k]          = m < ncells ? cells[m] : 0;
        }
        T ps[U], a0[U], a1[U], a2[U];
#pragma unroll
        for (int k = 0; k < U; k++) {
            const int j = id[k] < 0 ? 0 : id[k];
            ps[k]       = phi_sum[j];
            a0[k]       = u0[j];
            a1[k]       = u1[j];
            a2[k]       = u2[j];
        }
#pragma unroll
        for (int k = 0; k < U; k++) {
            if (id[k] < 0) continue;
            double r[3];
            cell_offset(g, cm[k], res, r);
            const double psd = (double)ps[k];
            const double wgt = sw[k] / (psd > 1.0 ? psd : 1.0);
            double       vs[3] = {vp[0], vp[1], vp[2]};
            if (ph.rotation) {
                vs[0] += op[1] * r[2] - op[2] * r[1];
                vs[1] += op[2] * r[0] - op[0] * r[2];
                vs[2] += op[0] * r[1] - op[1] * r[0];
            }
            const double fp0 = (vs[0] - (double)a0[k]) * wgt;
            const double fp1 = (vs[1] - (double)a1[k]) * wgt;
            const double fp2 = (vs[2] - (double)a2[k]) * wgt;
            acc[0] += fp0;
            acc[1] += fp1;
            acc[2] += fp2;
            acc[3] += r[1] * fp2 - r[2] * fp1;
            acc[4] += r[2] * fp0 - r[0] * fp2;
            acc[5] += r[0] * fp1 - r[1] * fp0;
        }
    }
    block_sum6(acc);
    if (threadIdx.x == 0) {
        const double dmy = -ph.dx3 * ph.rho / ph.dt;
        for (int d = 0; d < 3; d++) f_hydro[3 * p + d] = dmy * acc[d];
        if (ph.rotation)
            for (int d = 0; d < 3; d++) torque_hydro[3 * p + d] = dmy * acc[3 + d];
    }
}

// The rigidity force f = up - min(phi_sum, 1) u (Make_f_particle_dt_nonsole,
// f_particle.h:35-54) scattered directly from the stencil cache.  With w_p =
// Phi_p / max(phi_sum, 1): up = sum_p w_p (v_p + omega_p x r) and
// min(phi_sum, 1) = sum_p w_p, so f = sum_p w_p (v_p + omega_p x r - u), the
// integrand of the hydrodynamic force.  f is zero wherever no profile
// reaches, so the forward z pass of f reads three fields instead of the
// seven (up, u, phi) of forming f on the fly.
template <typename T>
__global__ void s_f_scatter_cached(Grid g, Phys ph, const double *__restrict__ x, const double *__restrict__ v,
                                   const double *__restrict__ w, const int *__restrict__ cells, int ncells,
                                   const int *__restrict__ sc_idx, const double *__restrict__ sc_w,
                                   const T *__restrict__ phi_sum, const T *__restrict__ u0, const T *__restrict__ u1,
                                   const T *__restrict__ u2, T *__restrict__ f0, T *__restrict__ f1,
                                   T *__restrict__ f2) {
    const int p = blockIdx.y;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ph.np || m >= ncells) return;
    const size_t o  = (size_t)p * ncells + m;
    const int    id = sc_idx[o];
    if (id < 0) return;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    double       res[3], r[3];
    particle_residue(g, xp, res);
    cell_offset(g, cells[m], res, r);
    const double ps  = (double)phi_sum[id];
    const double wgt = sc_w[o] / (ps > 1.0 ? ps : 1.0);
    double       vs[3] = {v[3 * p], v[3 * p + 1], v[3 * p + 2]};
    if (ph.rotation) {
        const double *om = w + 3 * p;
        vs[0] += om[1] * r[2] - om[2] * r[1];
        vs[1] += om[2] * r[0] - om[0] * r[2];
        vs[2] += om[0] * r[1] - om[1] * r[0];
    }
    atomicAdd(&f0[id], (T)((vs[0] - (double)u0[id]) * wgt));
    atomicAdd(&f1[id], (T)((vs[1] - (double)u1[id]) * wgt));
    atomicAdd(&f2[id], (T)((vs[2] - (double)u2[id]) * wgt));
}

// ---------------------------------------------------------------------------
// Particle state (FP64, [Np][3] / [Np][4] arrays).
// ---------------------------------------------------------------------------
struct PState {
    double *x, *x_nopbc, *x_previous, *v, *v_old, *omega, *omega_old;
    double *q, *q_old;  // [Np][4]: s, v0, v1, v2
    double *f_hydro, *f_hydro_previous, *torque_hydro, *torque_hydro_previous;
    double *fr, *fr_previous, *torque_r, *torque_r_previous;
    double *mdf;        // momentum_depend_fr [Np][3] (particle_solver.cxx:336-432)
    double *lj_stress;  // [Np] per-particle share of sum f_x r_y (LE stress)
};

__device__ __forceinline__ void qtn_prod_d(const double *qa, const double *qb, double alpha, double *q) {
    q[0] = alpha * (qa[0] * qb[0] - (qa[1] * qb[1] + qa[2] * qb[2] + qa[3] * qb[3]));
    q[1] = alpha * (qa[0] * qb[1] + qb[0] * qa[1] + qa[2] * qb[3] - qa[3] * qb[2]);
    q[2] = alpha * (qa[0] * qb[2] + qb[0] * qa[2] + qa[3] * qb[1] - qa[1] * qb[3]);
    q[3] = alpha * (qa[0] * qb[3] + qb[0] * qa[3] + qa[1] * qb[2] - qa[2] * qb[1]);
}
// dq/dt = 0.5 (0, w) o q  (qdot SPACE_FRAME, rigid_body.cxx:157-168)
__device__ __forceinline__ void qdot_space_d(const double *q, const double *w, double *dq) {
    const double qw[4] = {0.0, w[0], w[1], w[2]};
    qtn_prod_d(qw, q, 0.5, dq);
}
__device__ __forceinline__ void qtn_normalize_d(double *q) {
    const double n = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const double s = 1.0 / n;
    for (int k = 0; k < 4; k++) q[k] *= s;
}

// MD_solver_position_Euler / _AB2 (particle_solver.cxx:39-85) with the
// orientation updates (particle_rotation_solver.h:23-29, 72-81) and PBC
// (periodic_boundary.h:9-16).
// wrap = 0 leaves the periodic wrap to p_le_wrap (Lees-Edwards image).
// The Euler start (ts == 0) is read from the run's device step counter, so a
// captured step graph serves every step.
__global__ void p_position(Phys ph, PState s, const int *__restrict__ ts_dev, int wrap) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ph.np || ph.janus_prop == 3) return;  // OBSTACLE: fixed (particle_solver.cxx:44)
    const int euler = *ts_dev == 0;
    for (int d = 0; d < 3; d++) {
        const int i       = 3 * n + d;
        s.x_previous[i]   = s.x[i];
        const double dlt  = euler ? ph.dt * s.v[i] : ph.hdt * (3.0 * s.v[i] - s.v_old[i]);
        s.x_nopbc[i] += dlt;
        s.x[i] = wrap ? fmod(s.x[i] + dlt + ph.L[d], ph.L[d]) : s.x[i] + dlt;
    }
    if (ph.rotation) {
        double *q = s.q + 4 * n, *qo = s.q_old + 4 * n;
        double  dq[4];
        if (euler) {
            for (int k = 0; k < 4; k++) qo[k] = q[k];
            qdot_space_d(q, s.omega + 3 * n, dq);
            for (int k = 0; k < 4; k++) q[k] += dq[k] * ph.dt;
        } else {
            double dqo[4];
            qdot_space_d(q, s.omega + 3 * n, dq);
            qdot_space_d(qo, s.omega_old + 3 * n, dqo);
            for (int k = 0; k < 4; k++) qo[k] = q[k];
            for (int k = 0; k < 4; k++) q[k] += dq[k] * (3.0 * ph.hdt);
            for (int k = 0; k < 4; k++) q[k] += dqo[k] * (-ph.hdt);
        }
        qtn_normalize_d(q);
    }
}

// Lennard-Jones magnitude / r (Lennard_Jones_f, interaction.h:160-199).
__device__ __forceinline__ double lj_f(double r, const Phys &ph) {
    double s = ph.lj_sigma / r;
    double p = (s * s) * (s * s) * (s * s);
    double coeff = 24.0 * ph.lj_eps;
    if (ph.lj_powers == 1) {
        p = p * p;
        coeff = 48.0 * ph.lj_eps;
    } else if (ph.lj_powers == 2) {
        p = p * p * p;
        coeff = 72.0 * ph.lj_eps;
    }
    return coeff / (r * r) * (2.0 * p * p - p);
}

// Number of times the reference cell list visits a pair (md_force.cxx:56-101):
// cells of Cell_length*DX = 16*DX, per axis the neighbour scan ic-1, ic, ic+1
// wraps -1 -> lc-1 and lc -> 0, so with lc < 3 cells per axis a neighbour
// cell is visited more than once (and with lc = 1 three times).
__device__ __forceinline__ int lj_multiplicity(const Phys &ph, const double *xa, const double *xb) {
    int mult = 1;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const int ma = (int)(xa[d] / ph.cell_len);
        const int mb = (int)(xb[d] / ph.cell_len);
        int       cnt = 0;
#pragma unroll
        for (int o = -1; o <= 1; o++) {
            int c = ma + o;
            if (c < 0) c = ph.lc[d] - 1;
            if (c > ph.lc[d] - 1) c = 0;
            cnt += (c == mb);
        }
        mult *= cnt;
    }
    return mult;
}

// Minimum-image x_b - x_a (Distance0, interaction.h:113-122).
__device__ __forceinline__ double min_image(const Phys &ph, const double *xa, const double *xb, double r[3]) {
    double d2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double x12 = xb[d] - xa[d];
        x12 -= (double)nint_d(x12 / ph.L[d]) * ph.L[d];
        r[d] = x12;
        d2 += x12 * x12;
    }
    return sqrt(d2);
}

// PBC_OBL (periodic_boundary.h:26-45): the periodic wrap of x with the
// Lees-Edwards image (crossing the y boundary shifts x by -+ gam LY) and the
// x-velocity change -sign Shear_rate_eff LY of that crossing.
__device__ __forceinline__ double pbc_obl(const Phys &ph, double *x, double gam, double srate) {
    double sy = x[1];
    x[1]      = fmod(x[1] + ph.L[1], ph.L[1]);
    sy -= x[1];
    int sign = (int)sy;
    if (sign != 0) sign = sign / abs(sign);
    x[0] -= (double)sign * gam * ph.L[1];
    x[0] = fmod(x[0] + ph.L[0], ph.L[0]);
    x[2] = fmod(x[2] + ph.L[2], ph.L[2]);
    return -(double)sign * srate * ph.L[1];
}

// LJ pair forces plus the constant body force (Force, particle_solver.h:88-111;
// Calc_f_Lennard_Jones_shear_cap_primitive_lnk, md_force.cxx:34-196).  Thread
// n gathers every pair term acting on particle n with the reference's pair
// multiplicity, so no atomics are needed.  lj_stress[n] receives particle n's
// share of sum f_x r_y over the pairs where it is the higher index, as the
// reference accumulates dev_shear_stress_lj.
// Rigid bodies (rid != nullptr): pairs of beads of one body are skipped
// (rigid_chain), f_lo[n] receives the pair forces on n where it is the lower
// index (for the bodies' torques), and under Lees-Edwards lj_stress[n] takes
// the bodies' term sum f_x R_y instead, R the image distance of the two
// bodies' centres xg (rigid_dev_shear_stress_lj, md_force.cxx:252-258).
// Pairs of two obstacles are skipped (obstacle_chain, interaction.h:29-35);
// the janus propulsion is the run's, so obstacle runs have no LJ pairs.
// One warp per particle: lanes stride over the partners, then a warp sum.
__global__ void p_forces(Phys ph, PState s, int all_pairs_le, double le_shift, const int *__restrict__ rid,
                         double *__restrict__ f_lo, const double *__restrict__ xg) {
    const int lane = threadIdx.x & 31;
    const int n    = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (n >= ph.np) return;
    double f[3]   = {0.0, 0.0, 0.0};
    double fl[3]  = {0.0, 0.0, 0.0};
    double stress = 0.0;
    if (ph.lj_on && ph.janus_prop != 3) {
        for (int m = lane; m < ph.np; m += 32) {
            if (m == n || (rid && rid[m] == rid[n])) continue;
            const int hi = n > m ? n : m, lo = n > m ? m : n;
            double    r[3], rr;  // r = x_other - x_n (with the periodic image rule)
            int       mult = 1;
            double    ry_body = 0.0;  // rigid, Lees-Edwards: y image distance of the bodies' centres
            if (all_pairs_le) {
                // O(N^2) loop with Distance0_OBL(x_lo, x_hi) (md_force.cxx:198-304,
                // interaction.h:50-72): y image first, then the x shift of the
                // Lees-Edwards image.
                const double *x1 = s.x + 3 * lo, *x2 = s.x + 3 * hi;
                double        y12 = x2[1] - x1[1];
                double        sy  = y12;
                y12 -= (double)nint_d(y12 / ph.L[1]) * ph.L[1];
                sy -= y12;
                int sign = (int)sy;
                if (sign != 0) sign = sign / abs(sign);
                double x12 = x2[0] - (x1[0] + (double)sign * le_shift);
                x12 -= (double)nint_d(x12 / ph.L[0]) * ph.L[0];
                double z12 = x2[2] - x1[2];
                z12 -= (double)nint_d(z12 / ph.L[2]) * ph.L[2];
                rr              = sqrt(y12 * y12 + x12 * x12 + z12 * z12);
                const double sg = (n == lo) ? 1.0 : -1.0;
                r[0]            = sg * x12;
                r[1]            = sg * y12;
                r[2]            = sg * z12;
                if (rid && xg) {
                    ry_body = xg[3 * rid[hi] + 1] - xg[3 * rid[lo] + 1];
                    ry_body -= (double)nint_d(ry_body / ph.L[1]) * ph.L[1];
                }
            } else {
                // cell-list pairs (i > j) with Distance0(x_i, x_j)
                mult = lj_multiplicity(ph, s.x + 3 * hi, s.x + 3 * lo);
                if (mult == 0) continue;
                double rij[3];
                rr              = min_image(ph, s.x + 3 * hi, s.x + 3 * lo, rij);
                const double sg = (n == hi) ? 1.0 : -1.0;
                r[0]            = sg * rij[0];
                r[1]            = sg * rij[1];
                r[2]            = sg * rij[2];
            }
            if (!(rr < ph.lj_cutoff)) continue;
            const double dmy_r = lj_f(rr, ph);
            for (int d = 0; d < 3; d++) f[d] += (double)mult * (-dmy_r * r[d]);
            if (n == hi) {
                // f_x of the lower-index partner (dmy_fn[0] = dmy_r r[0] here) times r_y, or the bodies' R_y
                stress += (rid && xg) ? (double)mult * (dmy_r * r[0]) * ry_body
                                      : (double)mult * (-dmy_r * r[0]) * r[1];
            } else {
                for (int d = 0; d < 3; d++) fl[d] += (double)mult * (-dmy_r * r[d]);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        f[0] += __shfl_xor_sync(0xffffffffu, f[0], o);
        f[1] += __shfl_xor_sync(0xffffffffu, f[1], o);
        f[2] += __shfl_xor_sync(0xffffffffu, f[2], o);
        stress += __shfl_xor_sync(0xffffffffu, stress, o);
        if (f_lo) {
            fl[0] += __shfl_xor_sync(0xffffffffu, fl[0], o);
            fl[1] += __shfl_xor_sync(0xffffffffu, fl[1], o);
            fl[2] += __shfl_xor_sync(0xffffffffu, fl[2], o);
        }
    }
    if (lane == 0) {
        for (int d = 0; d < 3; d++) s.fr[3 * n + d] += f[d] + ph.body_force[d];
        s.lj_stress[n] = stress;
        if (f_lo)
            for (int d = 0; d < 3; d++) f_lo[3 * n + d] = fl[d];
    }
}

// ---------------------------------------------------------------------------
// Cell list of the Lennard-Jones forces (Calc_f_Lennard_Jones_shear_cap_
// primitive_lnk, md_force.cxx:34-196): cells of Cell_length DX = 16 DX per
// axis, lc[d] = N[d] / 16 of them (md_force.cxx:14, 56-61), a particle in the
// cell (int)(x / 16 DX) of each axis (md_force.cxx:68-75).
// Layout: count[ncell], cell_of[np], bins[ncell][kLjBin].  A cell holding
// more than kLjBin particles keeps its count; its scans then go over all
// particles with cell_of == cell instead of the bin.
// ---------------------------------------------------------------------------
constexpr int kLjBin = 32;

__device__ __forceinline__ int lj_cell_axis(const Phys &ph, double x, int d, bool &bad) {
    int m = (int)(x / ph.cell_len);
    if (m < 0 || m >= ph.lc[d]) {
        bad = true;
        m   = m < 0 ? 0 : ph.lc[d] - 1;
    }
    return m;
}

// One thread per particle: its cell, and a slot in the cell's bin (count[]
// zeroed before the launch).
__global__ void p_cells_bin(Phys ph, const double *__restrict__ x, int *__restrict__ count,
                            int *__restrict__ cell_of, int *__restrict__ bins, unsigned int *err) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ph.np) return;
    bool      bad = false;
    const int c   = (lj_cell_axis(ph, x[3 * n], 0, bad) * ph.lc[1] + lj_cell_axis(ph, x[3 * n + 1], 1, bad)) *
                      ph.lc[2] +
                  lj_cell_axis(ph, x[3 * n + 2], 2, bad);
    if (bad && err) atomicOr(err, SPM_DEVERR_PARTICLE_OUT_OF_BOX);
    cell_of[n]       = c;
    const int slot   = atomicAdd(&count[c], 1);
    if (slot < kLjBin) bins[(size_t)c * kLjBin + slot] = n;
}

// The next particle index above `last` in cell c (np when none): the bin's
// entries, or every particle of the cell when the bin overflowed.  Visiting a
// cell in increasing particle index keeps every sum in a fixed order.
__device__ __forceinline__ int lj_next_in_cell(const Phys &ph, int c, int last, const int *__restrict__ count,
                                               const int *__restrict__ cell_of, const int *__restrict__ bins) {
    const int k    = count[c];
    int       best = ph.np;
    if (k <= kLjBin) {
        for (int i = 0; i < k; i++) {
            const int m = bins[(size_t)c * kLjBin + i];
            if (m > last && m < best) best = m;
        }
    } else {
        for (int m = last + 1; m < ph.np; m++)
            if (cell_of[m] == c) return m;
    }
    return best;
}

// LJ pair forces from the cell list plus the constant body force (Force,
// particle_solver.h:88-111).  One warp per particle n: lane l < 27 takes the
// l-th neighbour cell of n's cell in the reference's scan order with its wrap
// (-1 -> lc-1, lc -> 0, md_force.cxx:86-101), so with fewer than three cells
// on an axis a neighbour cell comes up more than once and its pairs count as
// often, as in the reference; a warp sum in a fixed order follows.  Every
// pair term is the one the reference forms for i > j with Distance0(x_i,
// x_j); lj_stress[n] receives particle n's share of sum f_x r_y over the
// pairs where it is the higher index.  Pairs of two obstacles exert no force
// (obstacle_chain, interaction.h:29-35; Janus particles are one species here).
// Beads of rigid bodies (rid != null): pairs within one body are skipped
// (rigid_chain, interaction.h:18-24), and f_lo[n] receives the force on n
// from the pairs where n is the lower index (the bodies' torques need it).
__global__ void p_forces_cells(Phys ph, PState s, const int *__restrict__ count, const int *__restrict__ cell_of,
                               const int *__restrict__ bins, const int *__restrict__ rid, double *__restrict__ f_lo) {
    const int lane = threadIdx.x & 31;
    const int n    = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (n >= ph.np) return;
    double f[3]   = {0.0, 0.0, 0.0};
    double fl[3]  = {0.0, 0.0, 0.0};
    double stress = 0.0;
    if (ph.lj_on && ph.janus_prop != 3 && lane < 27) {
        const int mc[3] = {cell_of[n] / (ph.lc[1] * ph.lc[2]), (cell_of[n] / ph.lc[2]) % ph.lc[1],
                           cell_of[n] % ph.lc[2]};
        const int o[3]  = {lane / 9 - 1, (lane / 3) % 3 - 1, lane % 3 - 1};
        int       cl[3];
        for (int d = 0; d < 3; d++) {
            int c = mc[d] + o[d];
            if (c < 0) c = ph.lc[d] - 1;
            if (c > ph.lc[d] - 1) c = 0;
            cl[d] = c;
        }
        const int cell = (cl[0] * ph.lc[1] + cl[1]) * ph.lc[2] + cl[2];
        for (int m = lj_next_in_cell(ph, cell, -1, count, cell_of, bins); m < ph.np;
             m     = lj_next_in_cell(ph, cell, m, count, cell_of, bins)) {
            if (m == n || (rid && rid[m] == rid[n])) continue;
            const int    hi = n > m ? n : m, lo = n > m ? m : n;
            double       rij[3];
            const double rr = min_image(ph, s.x + 3 * hi, s.x + 3 * lo, rij);
            if (!(rr < ph.lj_cutoff)) continue;
            const double sg    = (n == hi) ? 1.0 : -1.0;
            const double dmy_r = lj_f(rr, ph);
            for (int d = 0; d < 3; d++) f[d] += -dmy_r * (sg * rij[d]);
            if (n == hi) {
                stress += (-dmy_r * rij[0]) * rij[1];
            } else {
                for (int d = 0; d < 3; d++) fl[d] += -dmy_r * (sg * rij[d]);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        f[0] += __shfl_xor_sync(0xffffffffu, f[0], o);
        f[1] += __shfl_xor_sync(0xffffffffu, f[1], o);
        f[2] += __shfl_xor_sync(0xffffffffu, f[2], o);
        stress += __shfl_xor_sync(0xffffffffu, stress, o);
        if (f_lo) {
            fl[0] += __shfl_xor_sync(0xffffffffu, fl[0], o);
            fl[1] += __shfl_xor_sync(0xffffffffu, fl[1], o);
            fl[2] += __shfl_xor_sync(0xffffffffu, fl[2], o);
        }
    }
    if (lane == 0) {
        for (int d = 0; d < 3; d++) s.fr[3 * n + d] += f[d] + ph.body_force[d];
        s.lj_stress[n] = stress;
        if (f_lo)
            for (int d = 0; d < 3; d++) f_lo[3 * n + d] = fl[d];
    }
}

// MD_solver_velocity_Euler / _AB2_hydro (particle_solver.cxx:103-142,
// 239-281) followed by reset_Forces (particle_solver.cxx:11-37).
// Velocity / angular-velocity update of particle n (Euler at step 0, AB2
// after) and the shift of the current forces to the previous ones.
// qvq = q (0, v) q* (qtn_qvq_prod, quaternion.h:189-196); conj: with q*.
__device__ __forceinline__ void qtn_rotate_d(const double *q, const double *v, double *out, bool conj) {
    const double s = q[0], a = conj ? -q[1] : q[1], b = conj ? -q[2] : q[2], c = conj ? -q[3] : q[3];
    const double qs2 = s * s - (a * a + b * b + c * c);
    const double dot = a * v[0] + b * v[1] + c * v[2];
    out[0] = qs2 * v[0] + 2.0 * (dot * a + s * (b * v[2] - c * v[1]));
    out[1] = qs2 * v[1] + 2.0 * (dot * b + s * (c * v[0] - a * v[2]));
    out[2] = qs2 * v[2] + 2.0 * (dot * c + s * (a * v[1] - b * v[0]));
}

// self_propulsion (particle_solver.cxx:88-101): a TUMBLER's body-frame force
// and torque in the space frame (rigid_body_rotation BODY2SPACE).
__device__ __forceinline__ void self_propulsion_d(const Phys &ph, const double *q, double *f, double *t) {
    if (ph.janus_prop == 1) {
        qtn_rotate_d(q, ph.janus_force, f, false);
        qtn_rotate_d(q, ph.janus_torque, t, false);
    } else {
        f[0] = f[1] = f[2] = t[0] = t[1] = t[2] = 0.0;
    }
}

__device__ __forceinline__ void velocity_update_one(const Phys &ph, const PState &s, int n, int euler) {
    const int    sp  = spec_of(ph, n);
    const double dmy = (euler ? ph.dt : ph.hdt) * ph.imass_s[sp];
    const double dmr = (euler ? ph.dt : ph.hdt) * ph.imoi_s[sp];
    double       sf[3], st[3];
    self_propulsion_d(ph, s.q + 4 * n, sf, st);
    for (int d = 0; d < 3; d++) {
        const int i      = 3 * n + d;
        s.v_old[i]       = s.v[i];
        s.omega_old[i]   = s.omega[i];
        if (ph.janus_prop == 3) {  // OBSTACLE
            s.v[i]     = 0.0;
            s.omega[i] = 0.0;
        } else if (euler) {
            s.v[i] += dmy * (s.f_hydro[i] + s.fr[i] + sf[d]);
            s.omega[i] += dmr * (s.torque_hydro[i] + s.torque_r[i] + st[d]);
        } else {
            s.v[i] += dmy * (2.0 * (s.f_hydro[i] + sf[d]) + s.fr[i] + s.fr_previous[i]);
            s.omega[i] += dmr * (2.0 * (s.torque_hydro[i] + st[d]) + s.torque_r[i] + s.torque_r_previous[i]);
        }
        s.fr_previous[i]           = s.fr[i];
        s.fr[i]                    = 0.0;
        s.f_hydro_previous[i]      = s.f_hydro[i];
        s.f_hydro[i]               = 0.0;
        s.torque_r_previous[i]     = s.torque_r[i];
        s.torque_r[i]              = 0.0;
        s.torque_hydro_previous[i] = s.torque_hydro[i];
        s.torque_hydro[i]          = 0.0;
    }
}

__global__ void p_velocity(Phys ph, PState s, const int *__restrict__ ts_dev) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ph.np) return;
    velocity_update_one(ph, s, n, *ts_dev == 0);
}

// The Lees-Edwards velocity update also records momentum_depend_fr, the LJ
// and body-force impulse used by the next step's hydrodynamic stress
// (MD_solver_velocity_*_OBL, particle_solver.cxx:336-432).
__global__ void p_velocity_mdf(Phys ph, PState s, const int *__restrict__ ts_dev) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ph.np) return;
    const int euler = *ts_dev == 0;
    for (int d = 0; d < 3; d++) {
        const int i = 3 * n + d;
        s.mdf[i]    = euler ? ph.dt * s.fr[i] : ph.hdt * (s.fr[i] + s.fr_previous[i]);
    }
    // then the same update as Navier_Stokes runs, obstacles held at rest (the
    // obstacle branch of the _OBL solvers); tumblers and squirmers are
    // refused under Lees-Edwards, so the self-propulsion term is zero here
    velocity_update_one(ph, s, n, euler);
}

// Advances the device step counters of `nr` consecutive runs (end of every
// step).
__global__ void k_ts_advance(RunWords *rw, int nr) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nr) rw[r].ts += 1;
}

// FIX_CELLxyz (sp_3d_ns.cxx:45-51): zero the selected uk_dc components of
// `nr` consecutive runs, each with its own mask (bit d = axis d).
__global__ void k_fix_cell(RunWords *rw, int nr) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nr) return;
    const int m = rw[r].fix_mask;
    for (int d = 0; d < 3; d++)
        if (m & (1 << d)) rw[r].uk_dc[d] = 0.0;
}

// ---------------------------------------------------------------------------
// Thermostat: MT19937 (Matsumoto & Nishimura 1998; init_genrand/genrand_real3
// as used by the reference, mt19937ar.c:65-192) and polar Box-Muller
// (Gauss2, fluct.h:48-60), drawn in the reference's serial order: per
// particle three pairs, v gets the first three normals, omega the last three
// (Add_random_force_thermostat, fluct.cxx:10-37).
// State layout: mt[0..623], mt[624] = mti.
// ---------------------------------------------------------------------------
// The draws are made by one block of 1024 threads, with the generator state
// in shared memory, and reproduce the serial stream exactly:
//  - the MT19937 twist runs in four phases [0,227) [227,454) [454,623)
//    [623], each reading only words the serial loop has already updated or
//    not yet touched, then the outputs are tempered in parallel;
//  - Gauss2 consumes uniforms in consecutive pairs (x1, x2) from the
//    stream, so the pairs are fixed by the stream; each is accepted when
//    0 < x1^2 + x2^2 < 1, and a block prefix sum over the accept flags
//    hands accepted pair a to particle a / 3, pair a % 3 (normals 2(a%3),
//    2(a%3)+1 of that particle: v for normals 0-2, omega for 3-5);
//  - the state advances by exactly the uniforms the serial loop consumes
//    (up to the second uniform of the last accepted pair).
constexpr int kThermoThreads = 1024;
__device__ __forceinline__ unsigned int mt_temper(unsigned int y) {
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= (y >> 18);
    return y;
}
__device__ __forceinline__ unsigned int mt_twist_word(const unsigned int *mt, int i) {
    const unsigned int y = (mt[i] & 0x80000000u) | (mt[(i + 1) % 624] & 0x7fffffffu);
    unsigned int       v = mt[(i + 397) % 624] ^ (y >> 1);
    if (y & 1u) v ^= 0x9908b0dfu;
    return v;
}
// noise != null (rigid bodies): the six normals of particle n go to
// noise[6 n ..], nothing is applied (r_thermostat applies them per body).
__global__ void __launch_bounds__(kThermoThreads) p_thermostat(Phys ph, PState s, unsigned int *mt_g,
                                                               double *noise) {
    __shared__ unsigned int mt[624];
    __shared__ double       uni[624 + 1];  // the carried uniform, then this round's outputs
    __shared__ int          wsum[kThermoThreads / 32];
    __shared__ int          sh_mti, sh_carry, sh_done, sh_taken, sh_used;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int i = tid; i < 624; i += blockDim.x) mt[i] = mt_g[i];
    if (tid == 0) {
        sh_mti   = (int)mt_g[624];
        sh_carry = 0;
        sh_done  = 0;
        sh_taken = 0;
    }
    __syncthreads();
    const int need = 3 * ph.np;  // accepted pairs
    if (need == 0) return;
    // a round accepts about 245 pairs; the cap only bounds the loop
    for (int round = 0; !sh_done && round < need + 64; round++) {
        if (sh_mti >= 624) {  // twist, in four dependency-ordered phases
            const int lo[4] = {0, 227, 454, 623}, hi[4] = {227, 454, 623, 624};
            for (int ph4 = 0; ph4 < 4; ph4++) {
                const int    i = lo[ph4] + tid;
                unsigned int v = 0;
                if (i < hi[ph4]) v = mt_twist_word(mt, i);
                __syncthreads();
                if (i < hi[ph4]) mt[i] = v;
                __syncthreads();
            }
            if (tid == 0) sh_mti = 0;
            __syncthreads();
        }
        const int mti = sh_mti, carry = sh_carry, avail = 624 - mti;
        for (int j = tid; j < avail; j += blockDim.x)
            uni[carry + j] = ((double)mt_temper(mt[mti + j]) + 0.5) * (1.0 / 4294967296.0);
        __syncthreads();
        const int npairs = (carry + avail) / 2;
        // accept flags and their exclusive prefix sum (one pair per thread)
        bool   acc = false;
        double x1 = 0, x2 = 0, rsq = 0;
        if (tid < npairs) {
            x1  = 2.0 * uni[2 * tid] - 1.0;
            x2  = 2.0 * uni[2 * tid + 1] - 1.0;
            rsq = x1 * x1 + x2 * x2;
            acc = !(rsq >= 1.0 || rsq == 0.0);
        }
        const unsigned ball = __ballot_sync(0xffffffffu, acc);
        if (lane == 0) wsum[wid] = __popc(ball);
        __syncthreads();
        if (wid == 0) {
            int v = lane < kThermoThreads / 32 ? wsum[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += t;
            }
            if (lane < kThermoThreads / 32) wsum[lane] = v;  // inclusive per warp
        }
        __syncthreads();
        const int before = sh_taken + (wid ? wsum[wid - 1] : 0) + __popc(ball & ((1u << lane) - 1u));
        const int total  = sh_taken + wsum[kThermoThreads / 32 - 1];
        if (acc && before < need) {
            const double factor = sqrt(-2.0 * log(rsq) / rsq);
            const double g[2]   = {factor * x1, factor * x2};
            const int    n = before / 3, k = before % 3;
            for (int e = 0; e < 2; e++) {
                const int q = 2 * k + e;  // normal index of particle n
                if (noise)
                    noise[6 * n + q] = g[e];
                else if (q < 3)
                    s.v[3 * n + q] += g[e] * ph.noise_v * ph.imass_s[spec_of(ph, n)];
                else if (ph.rotation)
                    s.omega[3 * n + q - 3] += g[e] * ph.noise_o * ph.imoi_s[spec_of(ph, n)];
            }
            if (before == need - 1) sh_used = 2 * (tid + 1);  // uniforms consumed this round
        }
        __syncthreads();
        if (tid == 0) {
            if (total >= need) {
                sh_mti += sh_used - carry;  // state words consumed this round
                sh_done = 1;
            } else {
                sh_taken = total;
                if ((carry + avail) & 1) {  // odd output left: it starts the next pair
                    uni[0]   = uni[carry + avail - 1];
                    sh_carry = 1;
                } else {
                    sh_carry = 0;
                }
                sh_mti = 624;
            }
        }
        __syncthreads();
    }
    for (int i = tid; i < 624; i += blockDim.x) mt_g[i] = mt[i];
    if (tid == 0) mt_g[624] = (unsigned int)sh_mti;
}


}  // namespace spm
