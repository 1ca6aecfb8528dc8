// Electrolyte (charged colloids in a solution of mobile ions): the device
// kernels of the reference's spectral Electrolyte step
// (NSsolute_solver_Euler and Rhs_NS_Nernst_Planck, fluid_solver.cxx:171-346;
// operate_electrolyte.cxx; solute_rhs.cxx; the Electrolyte branch of
// Time_evolution_hydro, sp_3d_ns.cxx:75-100).  Fields are FP64 rows of
// 2*hnzp reals (real space) or hnzp complex (k space), as for the
// Navier_Stokes step.
#pragma once

#include "spm_kernels.cuh"

namespace spm {

// Run constants of an Electrolyte context (Init_rho_ion,
// operate_electrolyte.cxx:667-791; input.cxx:834-930).
struct ELState {
    int     enabled = 0;
    int     nspec   = 0;           // 1: saltfree counterions, 2: positive and negative ions
    double  val_e[2] = {0, 0};     // Valency_e = Valency * Elementary_charge
    double  ons[2]   = {0, 0};     // Onsager coefficients
    double  iepsilon = 0.0;        // 1 / Dielectric_cst
    double  qe       = 0.0;        // Surface_charge_e of the particle species
    double  abs_q    = 0.0;        // sum over particles of |Surface_charge_e|
    double  counterion_number = 0; // saltfree: Surface_ion_number / Valency_counterion
    double  ion_number[2] = {0, 0};// salt: positive / negative ion numbers from the surface charge
    double  rho_inf[2]    = {0, 0};// salt: Rho_inf of each species
    int     e_on    = 0;           // External_field
    int     e_ac    = 0;           // AC field
    double  e_ext[3] = {0, 0, 0};  // E_ext
    double  e_omega = 0.0;         // Angular_Frequency = 2 pi Frequency
    int     init_pb = 0;           // INIT_profile Poisson_Boltzmann
    double  surface_ion_number = 0;// -sum over particles of Surface_charge
    int     init_iters = 0;        // iterations of the last initial-profile loop
    int     conc_in_box = 0;       // the ion fields are zero outside the 2/3 box (pruned inverses apply)
    int     time_known = 0;        // the device's time word holds time_dev
    double  time_dev   = 0.0;
    double *dev     = nullptr;     // device scalars (kEl*)
    double *partial = nullptr;     // per-CTA partial sums of the field reductions
};
// device scalars
constexpr int kElTotal  = 0;  // [0, 1]: Total_solute of each species
constexpr int kElQSum   = 2;  // sum of |surface charge field|
constexpr int kElCSum   = 3;  // [3, 4]: (1 - phi) c sums of each species
constexpr int kElVolume = 5;  // sum of (1 - phi)
constexpr int kElScratch = 6;  // [6, 8]: sums read by the host in the initial-profile loops
constexpr int kElTime    = 9;  // the run's time (advanced on the device every step)
constexpr int kElField   = 10; // [10, 15]: this step's external field: the k = 0 mode of grad psi (3), the Coulomb force's (3)
constexpr int kElScalars = 16;
constexpr double kElTol = 1.e-4;  // TOL of the initial-profile loops (operate_electrolyte.h:21)

// The step's external field from the time on the device, so that a captured
// step replays with the field of its own time: E_ext NX NY NZ sin(omega t)
// for the k = 0 mode of the potential's gradient (Add_constant_field_k,
// fluid_solver.cxx:221-231) and E_ext sin(omega t) for the Coulomb force
// (Make_Coulomb_force_x_on_fluid, operate_electrolyte.cxx:83-171); sin -> 1
// under a DC field.
__global__ void k_el_field(double *dev, double e0, double e1, double e2, int ac, double omega, double nxyz) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const double s   = ac ? sin(omega * dev[kElTime]) : 1.0;
    double       amp = nxyz;
    if (ac) amp *= s;
    const double e[3] = {e0, e1, e2};
    for (int d = 0; d < 3; d++) {
        dev[kElField + d]     = e[d] * amp;
        dev[kElField + 3 + d] = e[d] * s;
    }
}
// time += dt at the end of a step (the host's time advances the same way);
// k_el_set_time: the host's time after it was set outside a step
__global__ void k_el_time_advance(double *dev, double dt) {
    if (blockIdx.x == 0 && threadIdx.x == 0) dev[kElTime] += dt;
}
__global__ void k_el_set_time(double *dev, double t) {
    if (blockIdx.x == 0 && threadIdx.x == 0) dev[kElTime] = t;
}

// Total_solute[n] = (1 - phi) c sum * DX3 (Count_single_solute)
__global__ void k_el_total(double *dev, int n, double dx3) {
    if (blockIdx.x == 0 && threadIdx.x == 0) dev[kElTotal + n] = dev[kElCSum + n] * dx3;
}

// |phi_s'(x)| of the compact sine profile (DPhi_compact_sin, profile.h:164-173)
__device__ __forceinline__ double dphi_compact_sin(double x, double radius, double xi) {
    const double hxi   = xi * .5;
    const double ixi   = 1. / xi;
    const double dmy_x = radius - x;
    if (fabs(dmy_x) < hxi) return M_PI * .5 * ixi * cos(M_PI * dmy_x * ixi);
    return 0.;
}

// Make_phi_qq_particle (operate_electrolyte.cxx:173-208): phi += Phi and
// surface += Surface_charge_e[p.spec] * |phi_s'| over each particle's stencil.
template <typename T>
__global__ void s_el_phi_qq(Grid g, Phys ph, const double *__restrict__ x, const int *__restrict__ cells, int ncells,
                            T *__restrict__ phi, T *__restrict__ surface, unsigned int *err) {
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
    const double v  = phi_prof(s.dist, ph.radius, ph.hxi, g.dx);
    const double dq = ph.qe_s[spec_of(ph, p)] * dphi_compact_sin(s.dist, ph.radius, 2.0 * ph.hxi);  // Surface_charge_e[p.spec]
    if (v != 0.0) atomicAdd(&phi[s.idx], (T)v);
    if (dq != 0.0) atomicAdd(&surface[s.idx], (T)dq);
}

// Make_surface_normal (make_phi.cxx:17-55): sum of r / |r| over the stencil
// cells with ||r| - RADIUS| < XI / 2, r the cell offset from the particle.
template <typename T>
__global__ void s_el_surface_normal(Grid g, Phys ph, const double *__restrict__ x, const int *__restrict__ cells,
                                    int ncells, T *__restrict__ n0, T *__restrict__ n1, T *__restrict__ n2) {
    const int p = blockIdx.y;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ph.np || m >= ncells) return;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    if (!particle_in_box(ph, xp)) return;
    StencilPoint s;
    stencil_point(g, ph, xp, cells[m], s);
    const double dmy_r = sqrt(s.r[0] * s.r[0] + s.r[1] * s.r[1] + s.r[2] * s.r[2]);
    const double dmy   = fabs(dmy_r - ph.radius);
    if (dmy < ph.hxi) {
        const double ir = 1. / dmy_r;
        atomicAdd(&n0[s.idx], (T)(s.r[0] * ir));
        atomicAdd(&n1[s.idx], (T)(s.r[1] * ir));
        atomicAdd(&n2[s.idx], (T)(s.r[2] * ir));
    }
}

// Sums over the real cells (i < NX, j < NY, k < NZ), one partial per CTA,
// of (b = phi for the modes that use it):
//   0: (1 - phi) a (Count_single_solute)     1: |a|       2: (1 - phi)
//   3: (1 - phi) exp(-coef a)  (the Poisson-Boltzmann normalisations,
//      operate_electrolyte.cxx:445-455, 597-606)
//   4: (1 - phi) a (log a - 1)  (ideal-gas free energy, :306-316)
//   5: a (coef b - (e . (i, j, k)) DX)  (electrostatic free energy with the
//      external field's potential, :325-352, Add_external_electric_field_x)
struct ElSumArgs {
    int    mode;
    double coef, e[3];
};
template <typename T>
__global__ void __launch_bounds__(256) r_el_sum(Grid g, const T *__restrict__ a, const T *__restrict__ b,
                                                ElSumArgs m, double *__restrict__ partial) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    double       acc    = 0.0;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(idx % rowlen);
        if (k >= g.nz) continue;
        switch (m.mode) {
            case 0: acc += (1. - (double)b[idx]) * (double)a[idx]; break;
            case 1: acc += fabs((double)a[idx]); break;
            case 2: acc += (1. - (double)b[idx]); break;
            case 3: acc += (1. - (double)b[idx]) * exp(-m.coef * (double)a[idx]); break;
            case 4: {
                const double c = (double)a[idx];
                acc += (1. - (double)b[idx]) * c * (log(c) - 1.);
            } break;
            default: {
                const size_t row = idx / rowlen;
                const int    j = (int)(row % (size_t)g.ny), i = (int)(row / (size_t)g.ny);
                const double ext = (m.e[0] * (double)i + m.e[1] * (double)j + m.e[2] * (double)k) * g.dx;
                acc += (double)a[idx] * (m.coef * (double)b[idx] - ext);
            }
        }
    }
    __shared__ double red[8];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        partial[blockIdx.x] = t;
    }
}
// out = sum of the nb partials by one block of kElFinishThreads: thread t
// adds partials t, t + T, ... in order, then a fixed tree over the threads,
// so the result does not depend on scheduling.
constexpr int kElFinishThreads = 256;
__global__ void __launch_bounds__(kElFinishThreads) k_el_sum_finish(const double *__restrict__ partial, int nb,
                                                                     double *__restrict__ out) {
    __shared__ double red[kElFinishThreads];
    double            t = 0.0;
    for (int b = threadIdx.x; b < nb; b += kElFinishThreads) t += partial[b];
    red[threadIdx.x] = t;
    __syncthreads();
    for (int w = kElFinishThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// a *= s over the real cells, s = num / (den * dx3) from device scalars
// (the surface-charge normalisation of Make_phi_qq_particle and the solute
// rescale of Rescale_solute, solute_rhs.cxx:91-116; the latter on every
// element of a k-space field: scale_all).
template <typename T>
__global__ void r_el_scale(Grid g, T *__restrict__ a, double num, const double *__restrict__ num_dev,
                           const double *__restrict__ den_dev, double dx3, int scale_all) {
    const double s      = (num_dev ? *num_dev : num) / (*den_dev * dx3);
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if (!scale_all && (int)(idx % rowlen) >= g.nz) continue;
        a[idx] = (T)((double)a[idx] * s);
    }
}

// charge += Valency_e c (1 - phi) over the real cells (Conc_k2charge_field)
template <typename T>
__global__ void r_el_charge_add(Grid g, T *__restrict__ charge, const T *__restrict__ c, const T *__restrict__ phi,
                                double val_e) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= g.nz) continue;
        charge[idx] = (T)((double)charge[idx] + val_e * (double)c[idx] * (1. - (double)phi[idx]));
    }
}

// Counterions, Poisson-Boltzmann (Set_Poisson_Boltzmann_ion_charge_density_
// nosalt, operate_electrolyte.cxx:456-478): with rho_0 = num / (dev[s] DX^3)
// and dmy = rho_0 exp(-coef psi), c = (1 - alp) c + alp dmy; w0 = |dmy|,
// w1 = |c - dmy| for the convergence sums.  Real fields.
template <typename T>
__global__ void r_el_pb_mix(Grid g, T *__restrict__ c, const T *__restrict__ psi, double num,
                            const double *__restrict__ dev_sum, double dx3, double coef, double alp,
                            T *__restrict__ w0, T *__restrict__ w1) {
    const double rho0   = num / (*dev_sum * dx3);
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= g.nz) continue;
        const double dmy = rho0 * exp(-coef * (double)psi[idx]);
        const double cn  = (1. - alp) * (double)c[idx] + alp * dmy;
        c[idx]           = (T)cn;
        w0[idx]          = (T)fabs(dmy);
        w1[idx]          = (T)fabs(cn - dmy);
    }
}

// Salt, Poisson-Boltzmann (Set_Poisson_Boltzmann_ion_charge_density_salt,
// operate_electrolyte.cxx:595-630): nu from the quadratic a nu^2 + b nu + c
// = 0 with a = z+ rho+ I+, b = -Surface_ion_number, c = z- rho- I-, I the
// sums in dev[sp], dev[sn] (times DX^3); c+ = rho+ exp(-d0 psi) nu, c- =
// rho- exp(-d1 psi) / nu.  Real fields.
template <typename T>
__global__ void r_el_pb_salt(Grid g, T *__restrict__ c0, T *__restrict__ c1, const T *__restrict__ psi,
                             const double *__restrict__ dev, int sp, int sn, double dx3, double z0, double z1,
                             double rho_p, double rho_n, double surface_ion_number, double d0, double d1) {
    const double a  = z0 * rho_p * (dev[sp] * dx3);
    const double b  = -surface_ion_number;
    const double cq = z1 * rho_n * (dev[sn] * dx3);
    const double nu = (-b + sqrt(b * b - 4. * a * cq)) / (2. * a);
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= g.nz) {
            c0[idx] = c1[idx] = (T)0;
            continue;
        }
        const double pot = (double)psi[idx];
        c0[idx]          = (T)(rho_p * exp(-d0 * pot) * nu);
        c1[idx]          = (T)(rho_n * exp(-d1 * pot) / nu);
    }
}

// psi += alp (psi_new - psi); w0 = |psi|, w1 = |alp (psi_new - psi)|
// (operate_electrolyte.cxx:640-655).  Real fields.
template <typename T>
__global__ void r_el_pb_relax(Grid g, T *__restrict__ psi, const T *__restrict__ psi_new, double alp,
                              T *__restrict__ w0, T *__restrict__ w1) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= g.nz) continue;
        const double dmy = alp * ((double)psi_new[idx] - (double)psi[idx]);
        const double p   = (double)psi[idx] + dmy;
        psi[idx]         = (T)p;
        w0[idx]          = (T)fabs(p);
        w1[idx]          = (T)fabs(dmy);
    }
}

// c_n += dt rhs_n inside the 2/3 box (Field_solver_Euler of the ions alone,
// Ion_diffusion_solver_Euler, fluid_solver.cxx:262-296).
template <typename T>
__global__ void k_el_conc_update(Grid g, double dt, cplx<T> *__restrict__ c0, const cplx<T> *__restrict__ r0,
                                 cplx<T> *__restrict__ c1, const cplx<T> *__restrict__ r1, int nspec) {
    const size_t n = g.field_elems_c();
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        KPoint p;
        size_t row;
        if (!k_point(g, idx, p, row) || !p.keep) continue;
        cplx<T> c = c0[idx];
        c.re += (T)dt * r0[idx].re, c.im += (T)dt * r0[idx].im;
        c0[idx] = c;
        if (nspec > 1) {
            c = c1[idx];
            c.re += (T)dt * r1[idx].re, c.im += (T)dt * r1[idx].im;
            c1[idx] = c;
        }
    }
}

// out = a + b over the real cells
template <typename T>
__global__ void r_el_sum2(Grid g, T *__restrict__ out, const T *__restrict__ a, const T *__restrict__ b) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x)
        out[idx] = (int)(idx % rowlen) < g.nz ? a[idx] + b[idx] : (T)0;
}

// a = value on the real cells (the uniform initial ion density)
template <typename T>
__global__ void r_el_fill(Grid g, T *__restrict__ a, double value) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x)
        a[idx] = (int)(idx % rowlen) < g.nz ? (T)value : (T)0;
}

// Coulomb potential of a charge field in k space
// (Charge_field_k2Coulomb_potential_k_PBC, operate_electrolyte.cxx:69-81):
// a *= IK2 / Dielectric_cst; with `truncate` modes outside the 2/3 box are
// zeroed (Truncate_two_third_rule).
template <typename T>
__global__ void k_el_poisson(Grid g, cplx<T> *__restrict__ a, double iepsilon, int truncate) {
    const size_t n = g.field_elems_c();
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        KPoint p;
        size_t row;
        if (!k_point(g, idx, p, row)) continue;
        const double k2sum = p.kx * p.kx + p.ky * p.ky + p.kz * p.kz;
        const double f     = (k2sum > 0.0 ? 1.0 / k2sum : 0.0) * iepsilon;
        cplx<T>      v     = a[idx];
        v.re               = (T)((double)v.re * f);
        v.im               = (T)((double)v.im * f);
        if (truncate && !p.keep) v = cplx<T>{0, 0};
        a[idx] = v;
    }
}

// Gradient in k space of s a (A_k2da_k, fft_wrapper.cxx:200-225): g_d =
// (-k_d s a.im, k_d s a.re); at k = 0 the real parts get -e_d
// (Add_constant_field_k, fluid_solver.cxx:221-231, e = the step's field
// words of k_el_field; nullptr: no field).
template <typename T>
__global__ void k_el_grad(Grid g, const cplx<T> *__restrict__ a, cplx<T> *__restrict__ g0, cplx<T> *__restrict__ g1,
                          cplx<T> *__restrict__ g2, double s, int scaled, const double *__restrict__ e) {
    const size_t n = g.field_elems_c();
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        KPoint p;
        size_t row;
        if (!k_point(g, idx, p, row)) {
            g0[idx] = g1[idx] = g2[idx] = cplx<T>{0, 0};
            continue;
        }
        double re = (double)a[idx].re, im = (double)a[idx].im;
        if (scaled) re = s * re, im = s * im;
        cplx<T> d0 = {(T)(-p.kx * im), (T)(p.kx * re)};
        cplx<T> d1 = {(T)(-p.ky * im), (T)(p.ky * re)};
        cplx<T> d2 = {(T)(-p.kz * im), (T)(p.kz * re)};
        if (idx == 0 && e) {
            d0.re = (T)((double)d0.re - e[0]);
            d1.re = (T)((double)d1.re - e[1]);
            d2.re = (T)((double)d2.re - e[2]);
        }
        g0[idx] = d0, g1[idx] = d1, g2[idx] = d2;
    }
}

// Solute flux of one species in real space (Rhs_NS_solute,
// fluid_solver.cxx:190-206): on entry f = diffusion flux; adds the
// electro-migration term c Onsager (grad psi Valency_e)
// (Solute_solver_rhs_nonlinear_x_single), removes the component along the
// surface normal (Solute_impermeability; applying it once per cell is the
// same projection the reference applies once per particle whose stencil
// holds the cell), then adds the advection flux -c u (Add_advection_flux).
template <typename T>
__global__ void r_el_flux(Grid g, T *__restrict__ f0, T *__restrict__ f1, T *__restrict__ f2, const T *__restrict__ c,
                          const T *__restrict__ gp0, const T *__restrict__ gp1, const T *__restrict__ gp2,
                          const T *__restrict__ n0, const T *__restrict__ n1, const T *__restrict__ n2,
                          const T *__restrict__ u0, const T *__restrict__ u1, const T *__restrict__ u2, double ons,
                          double val_e) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= g.nz) continue;
        const double cc   = (double)c[idx];
        double       f[3] = {(double)f0[idx], (double)f1[idx], (double)f2[idx]};
        const double gp[3] = {(double)gp0[idx], (double)gp1[idx], (double)gp2[idx]};
        for (int d = 0; d < 3; d++) f[d] += cc * (ons * (gp[d] * val_e));
        const double nn[3] = {(double)n0[idx], (double)n1[idx], (double)n2[idx]};
        double       norm2 = 0.;
        for (int d = 0; d < 3; d++) norm2 += nn[d] * nn[d];
        if (norm2 > 0.) {
            double dmy = 0.;
            for (int d = 0; d < 3; d++) dmy += f[d] * nn[d];
            dmy /= norm2;
            for (int d = 0; d < 3; d++) f[d] -= nn[d] * dmy;
        }
        const double uu[3] = {(double)u0[idx], (double)u1[idx], (double)u2[idx]};
        for (int d = 0; d < 3; d++) f[d] += cc * -uu[d];
        f0[idx] = (T)f[0], f1[idx] = (T)f[1], f2[idx] = (T)f[2];
    }
}

// Divergence in k space (U_k2divergence_k, fft_wrapper.cxx:867-891)
template <typename T>
__global__ void k_el_div(Grid g, const cplx<T> *__restrict__ f0, const cplx<T> *__restrict__ f1,
                         const cplx<T> *__restrict__ f2, cplx<T> *__restrict__ div) {
    const size_t n = g.field_elems_c();
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        KPoint p;
        size_t row;
        if (!k_point(g, idx, p, row)) {
            div[idx] = cplx<T>{0, 0};
            continue;
        }
        const cplx<T> a = f0[idx], b = f1[idx], c = f2[idx];
        div[idx] = cplx<T>{(T)(-(p.kx * (double)a.im + p.ky * (double)b.im + p.kz * (double)c.im)),
                           (T)(p.kx * (double)a.re + p.ky * (double)b.re + p.kz * (double)c.re)};
    }
}

// Explicit Euler of NSsolute_solver_Euler over the retained modes
// (Field_solver_Euler, fluid_solver.cxx:120-136): zeta += dt (f_ns -
// nu K2 zeta) with f_ns the zeta form of the advection products
// (U2advection_k, operate_omega.cxx:12-98; Add_zeta_viscous_term,
// operate_omega.cxx:157-169), and c_n += dt rhs_n for each species.
template <typename T>
__global__ void k_el_update(Grid g, cplx<T> *__restrict__ z0p, cplx<T> *__restrict__ z1p,
                            const cplx<T> *__restrict__ p_u2u3, const cplx<T> *__restrict__ p_u3u1,
                            const cplx<T> *__restrict__ p_u1u2, const cplx<T> *__restrict__ p_a0,
                            const cplx<T> *__restrict__ p_a1, double nu, double dt, cplx<T> *__restrict__ c0,
                            const cplx<T> *__restrict__ r0, cplx<T> *__restrict__ c1, const cplx<T> *__restrict__ r1,
                            int nspec) {
    const size_t n = g.field_elems_c();
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        KPoint p;
        size_t row;
        if (!k_point(g, idx, p, row) || !p.keep) continue;
        const T k1 = (T)p.kx, k2 = (T)p.ky, k3 = (T)p.kz;
        const T k1k2 = k1 * k2, k2k3 = k2 * k3, k3k1 = k3 * k1;
        const T c0k = (k3 - k2) * (k3 + k2), c1k = (k1 - k3) * (k1 + k3), c2k = (k2 - k1) * (k2 + k1);
        const cplx<T> u2u3 = p_u2u3[idx], u3u1 = p_u3u1[idx], u1u2 = p_u1u2[idx];
        const cplx<T> a0 = p_a0[idx], a1 = p_a1[idx];
        const cplx<T> a2 = {-a1.re - a0.re, -a1.im - a0.im};
        cplx<T> om[3];
        om[0] = {-(k2k3 * a0.re + c0k * u2u3.re + k3k1 * u1u2.re - k1k2 * u3u1.re),
                 -(k2k3 * a0.im + c0k * u2u3.im + k3k1 * u1u2.im - k1k2 * u3u1.im)};
        om[1] = {-(k3k1 * a1.re + c1k * u3u1.re + k1k2 * u2u3.re - k2k3 * u1u2.re),
                 -(k3k1 * a1.im + c1k * u3u1.im + k1k2 * u2u3.im - k2k3 * u1u2.im)};
        om[2] = {-(k1k2 * a2.re + c2k * u1u2.re + k2k3 * u3u1.re - k3k1 * u2u3.re),
                 -(k1k2 * a2.im + c2k * u1u2.im + k2k3 * u3u1.im - k3k1 * u2u3.im)};
        cplx<T> f0, f1;
        omega_to_zeta<T>(p, om, f0, f1);
        const T       nk2 = (T)(nu * (p.kx * p.kx + p.ky * p.ky + p.kz * p.kz));
        cplx<T>       z0 = z0p[idx], z1 = z1p[idx];
        const cplx<T> r0z = {f0.re + -(nk2 * z0.re), f0.im + -(nk2 * z0.im)};
        const cplx<T> r1z = {f1.re + -(nk2 * z1.re), f1.im + -(nk2 * z1.im)};
        z0.re += (T)dt * r0z.re, z0.im += (T)dt * r0z.im;
        z1.re += (T)dt * r1z.re, z1.im += (T)dt * r1z.im;
        z0p[idx] = z0, z1p[idx] = z1;
        cplx<T> c = c0[idx];
        c.re += (T)dt * r0[idx].re, c.im += (T)dt * r0[idx].im;
        c0[idx] = c;
        if (nspec > 1) {
            c = c1[idx];
            c.re += (T)dt * r1[idx].re, c.im += (T)dt * r1[idx].im;
            c1[idx] = c;
        }
    }
}

// Coulomb body force on the fluid and its velocity kick
// (Make_Coulomb_force_x_on_fluid, operate_electrolyte.cxx:83-171, then
// u += f dt / RHO, sp_3d_ns.cxx:85-96): f_d = charge (-grad_d psi + E_d),
// E the step's field words of k_el_field.
template <typename T>
__global__ void r_el_coulomb(Grid g, const T *__restrict__ charge, const T *__restrict__ gp0, const T *__restrict__ gp1,
                             const T *__restrict__ gp2, T *__restrict__ u0, T *__restrict__ u1, T *__restrict__ u2,
                             int e_on, const double *__restrict__ e, double dmy) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    const double e0 = e_on ? e[0] : 0.0, e1 = e_on ? e[1] : 0.0, e2 = e_on ? e[2] : 0.0;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= g.nz) continue;
        const double q  = (double)charge[idx];
        double       ef = -(double)gp0[idx];
        if (e_on) ef += e0;
        u0[idx] = (T)((double)u0[idx] + q * ef * dmy);
        ef = -(double)gp1[idx];
        if (e_on) ef += e1;
        u1[idx] = (T)((double)u1[idx] + q * ef * dmy);
        ef = -(double)gp2[idx];
        if (e_on) ef += e2;
        u2[idx] = (T)((double)u2[idx] + q * ef * dmy);
    }
}

// f = up - phi u with the raw (unclamped) phi sum: on the Electrolyte step
// the phi array handed to Make_f_particle_dt_sole is the one Rescale_solute
// last filled by Make_phi_particle (solute_rhs.cxx:98-99).
template <typename T>
__global__ void r_el_make_f(Grid g, T *__restrict__ up0, T *__restrict__ up1, T *__restrict__ up2,
                            const T *__restrict__ u0, const T *__restrict__ u1, const T *__restrict__ u2,
                            const T *__restrict__ phi) {
    const size_t rowlen = 2 * (size_t)g.hnzp;
    const size_t n      = (size_t)g.nx * g.ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= g.nz) continue;
        const T ph = phi[idx];
        up0[idx]   = up0[idx] - ph * u0[idx];
        up1[idx]   = up1[idx] - ph * u1[idx];
        up2[idx]   = up2[idx] - ph * u2[idx];
    }
}

}  // namespace spm
