// Link-time drop-in of the B200 SPM boundary functions into KAPSEL.
//
// Compiled against KAPSEL's own headers and linked into the unmodified
// `kapsel` program with `-Wl,--wrap=<mangled name>` for each function below:
// every call the reference makes across object files to one of these
// functions then runs on the GPU through the C ABI of libkapsel_spm.so
// (include/kapsel_spm.h), with the reference's argument meaning, array layout
// (double[NX*NY*NZ_], FFTW r2c convention) and error convention (a failure
// prints the library's message and calls exit_job(EXIT_FAILURE), macro.h:178).
//
//   wrapped (mangled)                                   reference definition
//   NS_solver_slavedEuler                               fluid_solver.h:77-82, fluid_solver.cxx:348-374
//   Zeta_k2u_k / U_k2zeta_k                             fft_wrapper.h:162 / :150
//   Solenoidal_uk                                       operate_omega.h:72, operate_omega.cxx:171-195
//   Make_phi_particle_sum / Make_u_particle_sum         make_phi.h:50 / :55
//   Make_phi_u_particle                                 make_phi.h:70
//   Calc_f_hydro_correct_precision                      md_force.h:53, md_force.cxx:383-506
//   Calc_f_Lennard_Jones_shear_cap_primitive_lnk        md_force.h:60-63 (via Calc_f_Lennard_Jones, md_force.h:78-81)
//
// One device context serves the process; it is created at the first wrapped
// call from the reference's globals (set by Gourmet_file_io and
// Set_global_parameters, input.cxx) and serves Navier_Stokes runs of one
// particle species.  Each call copies its host arrays to the device and back
// (the _host entry points); header-inline reference code between the calls
// (A2a_k / A_k2a FFTs, the particle integrators) keeps running on the CPU.
// Keeping state resident across a whole step is the job of spm_step, which a
// maintainer calls from Time_evolution_hydro itself.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "kapsel_b200_common.h"

namespace {

using kapsel_b200::check;

spm_ctx            *g_ctx = nullptr;
std::vector<double> g_rec;

spm_ctx *ctx() {
    if (g_ctx) return g_ctx;
    if (SW_EQ != Navier_Stokes || Component_Number != 1) {
        fprintf(stderr, "kapsel_b200: the GPU boundary serves Navier_Stokes runs with one particle species\n");
        exit_job(EXIT_FAILURE);
    }
    spm_params p = kapsel_b200::params_from_globals(SPM_EQ_NAVIER_STOKES);
    check(spm_create(&p, nullptr, &g_ctx), "spm_create");
    return g_ctx;
}

double *records(const Particle *p) { return kapsel_b200::records(p, g_rec); }

}  // namespace

extern "C" {

void __wrap__Z21NS_solver_slavedEulerPPdRK5CTimeS_PK11Index_rangeRKiP8Particle(double **zeta, const CTime &jikan,
                                                                               double *uk_dc, const Index_range *,
                                                                               const int &, Particle *) {
    if (jikan.dt_fluid != DT) {
        fprintf(stderr, "kapsel_b200: dt changed during the run (%g != %g)\n", jikan.dt_fluid, DT);
        exit_job(EXIT_FAILURE);
    }
    check(spm_ns_solver_slaved_euler_host(ctx(), zeta[0], zeta[1], uk_dc), "NS_solver_slavedEuler");
}

void __wrap__Z10Zeta_k2u_kPPdS_S0_(double **zeta, double *uk_dc, double **u) {
    check(spm_zeta_k2u_k_host(ctx(), zeta[0], zeta[1], uk_dc, u[0], u[1], u[2]), "Zeta_k2u_k");
}

void __wrap__Z10U_k2zeta_kPPdS0_S_(double **u, double **zeta, double *uk_dc) {
    check(spm_u_k2zeta_k_host(ctx(), u[0], u[1], u[2], zeta[0], zeta[1], uk_dc), "U_k2zeta_k");
}

void __wrap__Z13Solenoidal_ukPPd(double **u) { check(spm_solenoidal_uk_host(ctx(), u[0], u[1], u[2]), "Solenoidal_uk"); }

void __wrap__Z21Make_phi_particle_sumPdS_P8Particled(double *phi, double *phi_sum, Particle *p, double radius) {
    if (radius != RADIUS) {
        fprintf(stderr, "kapsel_b200: Make_phi_particle_sum with radius %g != RADIUS\n", radius);
        exit_job(EXIT_FAILURE);
    }
    check(spm_make_phi_particle_sum_host(ctx(), records(p), phi, phi_sum), "Make_phi_particle_sum");
}

void __wrap__Z19Make_u_particle_sumPPdPKdP8Particled(double **up, const double *phi_sum, Particle *p,
                                                      double radius) {
    if (radius != RADIUS) {
        fprintf(stderr, "kapsel_b200: Make_u_particle_sum with radius %g != RADIUS\n", radius);
        exit_job(EXIT_FAILURE);
    }
    check(spm_make_u_particle_sum_host(ctx(), records(p), phi_sum, up[0], up[1], up[2]), "Make_u_particle_sum");
}

void __wrap__Z19Make_phi_u_particlePdPS_P8Particle(double *phi, double **up, Particle *p) {
    check(spm_make_phi_u_particle_host(ctx(), records(p), phi, up[0], up[1], up[2]), "Make_phi_u_particle");
}

void __wrap__Z30Calc_f_hydro_correct_precisionP8ParticlePKdPKS2_RK5CTime(Particle *p, const double *phi_sum,
                                                                          const double *const *u, const CTime &) {
    double *rec = records(p);
    check(spm_calc_f_hydro_correct_precision_host(ctx(), rec, phi_sum, u[0], u[1], u[2]),
          "Calc_f_hydro_correct_precision");
    for (int n = 0; n < Particle_Number; n++)
        for (int d = 0; d < 3; d++) {
            p[n].f_hydro[d]      = rec[(size_t)n * SPM_PARTICLE_WORDS + 26 + d];
            p[n].torque_hydro[d] = rec[(size_t)n * SPM_PARTICLE_WORDS + 32 + d];
        }
}

void __wrap__Z44Calc_f_Lennard_Jones_shear_cap_primitive_lnkP8ParticlePFvPKdS2_RdPdEd(
    Particle *p, void (*)(const double *, const double *, double &, double *), double cap) {
    if (cap != DBL_MAX) {
        fprintf(stderr, "kapsel_b200: capped Lennard-Jones forces are not served\n");
        exit_job(EXIT_FAILURE);
    }
    double *rec = records(p);
    check(spm_calc_f_lennard_jones_host(ctx(), rec), "Calc_f_Lennard_Jones");
    for (int n = 0; n < Particle_Number; n++)
        for (int d = 0; d < 3; d++) p[n].fr[d] = rec[(size_t)n * SPM_PARTICLE_WORDS + 38 + d];
}

}  // extern "C"
