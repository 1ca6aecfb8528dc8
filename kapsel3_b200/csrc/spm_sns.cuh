// Shear_Navier_Stokes diagnostics of the main loop (sp_3d_ns.cxx:958-960):
// Update_strain (sp_3d_ns.h:143-164, 205-214) and the shear-stress line of
// Mean_shear_stress (sp_3d_ns.h:319-340) with Calc_shear_stress
// (fluid_solver.h:185-247) and Make_rho_field (make_phi.cxx:60-112).
//
// After the step's rigidity force f is scattered (u + f, the field the
// reference's U2zeta_k takes), two sums per y row j of the grid give the
// rate and the stress:
//   F_j = sum_{x,z} (u + f)_x             -> the instantaneous shear rate,
//   P_j = sum_{x,z} fs rho                -> the shear stress,
// with fs the sustaining force of the step (the change NS_solver_slavedEuler_
// Shear_PBC made to u_x, fluid_solver.cxx:41-119) and rho = RHO + sum_p
// Phi_p (RHO_p - RHO) the density of the particles' current positions.
// Under AC a third one follows the step's new zeta:
//   Q_j = sum_{x,z} rho u_x, u from the new zeta -> the inertia stress.
//
//   * The shear rate averages d(u+f)_x/dy over NY/4 <= j < 3NY/4 as the
//     reference's spectral derivative of u from the step's zeta does; only the
//     modes (0, KY, 0) survive the average over x and z, and for them u_x
//     from zeta is (u + f)_x itself (the projection acts along y), so the
//     derivative is taken spectrally on the profile F_j in one dimension,
//     over the retained |KY| < TRN_Y that zeta carries.
//   * Calc_shear_stress: stress_yx = sum y (fs rho - mean) = sum_j y_j P_j -
//     mean sum_j y_j NX NZ, mean = sum_j P_j / N; printed as -stress_yx / (N dt).
//   * AC: Inertia_stress = (sum_j y_j Q_j - the previous step's sum) / (L^3 dt)
//     (the reference's rhop keeps the previous rho u_x; its u_x is that of the
//     step's final, projected velocity, i.e. of the new zeta).
#pragma once

#include "spm_kernels.cuh"

namespace spm {

// Device words of the diagnostics (double): the last step's shear rate,
// the strain accumulated from initialisation, -stress_yx, the viscosity
// -stress_yx / rate, the inertia stress, -stress_yx + inertia, and the
// previous step's sum_y y rho u_x.  rows[3 NY] follow (F, P, Q per row).
enum SnsWord { kSnsRate = 0, kSnsStrain, kSnsStress, kSnsVisc, kSnsInertia, kSnsApparent, kSnsPrevQ, kSnsWords = 8 };

struct RhoWeights {
    double drho[4];  // RHO_particle[spec] - RHO per species
};

// Make_rho_field's particle part: rho_d += Phi (RHO_p - RHO) over every
// (particle, Sekibun cell).
template <typename T>
__global__ void s_rho_scatter(Grid g, Phys ph, const double *__restrict__ x, const int *__restrict__ cells,
                              int ncells, T *__restrict__ rho_d, RhoWeights w) {
    const int p = blockIdx.y;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ph.np || m >= ncells) return;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    if (!particle_in_box(ph, xp)) return;
    StencilPoint s;
    stencil_point(g, ph, xp, cells[m], s);
    const double v = phi_prof(s.dist, ph.radius, ph.hxi, g.dx) * w.drho[spec_of(ph, p)];
    if (v != 0.0) atomicAdd(&rho_d[s.idx], (T)v);
}

// One block per y row j, summed in a fixed order (runs repeat bit for bit):
// mode 0: F_j = sum (a + b), P_j = sum fs rho into rows[3 j], rows[3 j + 1];
// mode 1: Q_j = sum rho a into rows[3 j + 2] (b and fs unused).
template <typename T>
__global__ void __launch_bounds__(256) r_sns_rows(Grid g, const T *__restrict__ a, const T *__restrict__ b,
                                                  const T *__restrict__ fs, const T *__restrict__ rho_d, double rho,
                                                  double *__restrict__ rows, int mode) {
    const int    j      = blockIdx.x;
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const int    nxz    = g.nx * g.nz;
    double       acc[2] = {0.0, 0.0};
    for (int t = threadIdx.x; t < nxz; t += blockDim.x) {
        const int    i = t / g.nz, k = t % g.nz;
        const size_t e = ((size_t)i * g.ny + j) * rowlen + k;
        const double r = rho + (double)rho_d[e];
        if (mode == 0) {
            acc[0] += (double)a[e] + (double)b[e];
            acc[1] += (double)fs[e] * r;
        } else {
            acc[0] += r * (double)a[e];
        }
    }
    __shared__ double red[2][256];
    for (int q = 0; q < 2; q++) red[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < 2; q++) red[q][threadIdx.x] += red[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (mode == 0) {
            rows[3 * j]     = red[0][0];
            rows[3 * j + 1] = red[1][0];
        } else {
            rows[3 * j + 2] = red[0][0];
        }
    }
}

// One block of 512 threads (NY <= 512).  mode 0: the shear rate from the
// spectral derivative of F, the strain and the stress; mode 1 (AC): the
// inertia stress from Q.
__global__ void __launch_bounds__(512) k_sns_finish(Grid g, const double *__restrict__ rows, double *__restrict__ w,
                                                    double dt, int mode) {
    const int    ny = g.ny, t = threadIdx.x;
    const double n  = (double)g.nx * g.ny * g.nz;
    __shared__ double red[3][512];
    double            part[3] = {0.0, 0.0, 0.0};
    if (t < ny && mode == 0) {
        // KY of index t (Nyquist +NY/2 contributes 0), the derivative's
        // coefficient i KY WAVE_Y F^(KY) and its sum over NY/4 <= j < 3 NY/4
        const int KY = t > ny / 2 ? t - ny : t;
        if (KY != 0 && abs(KY) < g.trn[1]) {
            double fr = 0.0, fi = 0.0;
            for (int j = 0; j < ny; j++) {
                double s, c;
                sincospi(-2.0 * (double)KY * j / ny, &s, &c);
                fr += rows[3 * j] * c;
                fi += rows[3 * j] * s;
            }
            const double wy = 2.0 * M_PI / (ny * g.dx) * KY;  // WAVE_Y KY
            const double gr = -wy * fi, gi = wy * fr;            // i KY WAVE_Y F^
            double       sr = 0.0;
            for (int j = ny / 4; j < 3 * ny / 4; j++) {
                double s, c;
                sincospi(2.0 * (double)KY * j / ny, &s, &c);
                sr += gr * c - gi * s;
            }
            part[0] = sr / ny;
        }
        part[1] = (double)t * g.dx * rows[3 * t + 1];  // y_j P_j
    }
    if (t < ny && mode == 1) part[2] = (double)t * g.dx * rows[3 * t + 2];  // y_j Q_j
    for (int q = 0; q < 3; q++) red[q][t] = part[q];
    __syncthreads();
    for (int s = 256; s > 0; s >>= 1) {
        if (t < s && t + s < (int)blockDim.x)
            for (int q = 0; q < 3; q++) red[q][t] += red[q][t + s];
        __syncthreads();
    }
    if (t == 0 && mode == 1) {
        const double vol = n * g.dx * g.dx * g.dx;
        w[kSnsInertia]   = (red[2][0] - w[kSnsPrevQ]) / (vol * dt);
        w[kSnsPrevQ]     = red[2][0];
        w[kSnsApparent]  = w[kSnsStress] + w[kSnsInertia];
    }
    if (t == 0 && mode == 0) {
        double p1 = 0.0;  // sum_j P_j in row order
        for (int j = 0; j < ny; j++) p1 += rows[3 * j + 1];
        const double rate   = -(2.0 / n) * red[0][0];
        const double sum_y  = g.dx * (double)g.nx * g.nz * (0.5 * (double)ny * (ny - 1));
        const double syx    = red[1][0] - (p1 / n) * sum_y;
        const double stress = -(syx / (n * dt));
        w[kSnsRate]   = rate;
        w[kSnsStrain] += rate * dt;
        w[kSnsStress] = stress;
        w[kSnsVisc]   = stress / rate;
    }
}

}  // namespace spm
