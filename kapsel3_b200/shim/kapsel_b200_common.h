// Shared by the link-time shim and the resident time evolution: the device
// context's parameters from the reference's globals (set by Gourmet_file_io
// and Set_global_parameters, input.cxx), the Particle (variable.h:27-77) <->
// SPM_PARTICLE_WORDS record conversion, and the reference's error convention
// (print, then exit_job(EXIT_FAILURE), macro.h:178).
#pragma once

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "input.h"
#include "macro.h"
#include "variable.h"

#include "kapsel_spm.h"

namespace kapsel_b200 {

inline void check(int rc, const char *what) {
    if (rc != SPM_OK) {
        fprintf(stderr, "kapsel_b200: %s failed: %s\n", what, spm_last_error());
        exit_job(EXIT_FAILURE);
    }
}

inline int log2_exact(int n, const char *axis) {
    int k = 0;
    while ((1 << k) < n) k++;
    if ((1 << k) != n) {
        fprintf(stderr, "kapsel_b200: N%s = %d is not a power of two\n", axis, n);
        exit_job(EXIT_FAILURE);
    }
    return k;
}

// spm_params of the run the reference's globals describe, for `equation`
// (the SPM_EQ_* the program's SW_EQ maps to), FP64.
inline spm_params params_from_globals(int equation) {
    if (spm_params_size() != sizeof(spm_params)) {
        fprintf(stderr, "kapsel_b200: libkapsel_spm was built from another kapsel_spm.h (spm_params %zu bytes, "
                        "this program %zu): rebuild the program\n",
                spm_params_size(), sizeof(spm_params));
        exit_job(EXIT_FAILURE);
    }
    spm_params p;
    check(spm_params_default(&p), "spm_params_default");
    p.npx         = log2_exact(NX, "X");
    p.npy         = log2_exact(NY, "Y");
    p.npz         = log2_exact(NZ, "Z");
    p.dx          = DX;
    p.rho         = RHO;
    p.eta         = ETA;
    p.kbt         = kBT;
    p.alpha_v     = alpha_v;
    p.alpha_o     = alpha_o;
    p.equation    = equation;
    p.n_particles = Particle_Number;
    p.mass_ratio  = MASS_RATIOS[0];
    p.a           = A;
    p.a_xi        = A_XI;
    p.epsilon     = EPSILON;
    p.lj_powers   = LJ_powers;
    p.lj_truncate = LJ_truncate;
    p.rotation    = ROTATION;
    for (int d = 0; d < DIM; d++) p.fix_cell[d] = FIX_CELLxyz[d];
    if (equation == SPM_EQ_LEES_EDWARDS) p.shear_rate = Shear_rate;
    if (equation == SPM_EQ_SHEAR_NAVIER_STOKES) {
        p.shear_rate      = Shear_rate;
        p.shear_ac        = Shear_AC ? 1 : 0;
        p.shear_frequency = Shear_frequency;
    }
    if (equation == SPM_EQ_ELECTROLYTE) {  // constitutive_eq.Electrolyte (input.cxx:834-930)
        p.dielectric     = Dielectric_cst;
        p.init_pb        = Poisson_Boltzmann ? 1 : 0;
        p.salt           = N_spec == 2 ? 1 : 0;
        p.surface_charge = Surface_charge ? Surface_charge[0] : 0.0;
        if (p.salt) {
            p.valency[0]   = Valency_positive_ion;
            p.valency[1]   = Valency_negative_ion;
            p.onsager[0]   = Onsager_coeff_positive_ion;
            p.onsager[1]   = Onsager_coeff_negative_ion;
            p.debye_length = Debye_length;
        } else {
            p.valency[0] = Valency_counterion;
            p.onsager[0] = Onsager_coeff_counterion;
        }
        p.e_field = External_field ? (AC ? 2 : 1) : 0;
        for (int d = 0; d < DIM; d++) p.e_ext[d] = E_ext[d];
        p.e_frequency = AC ? Frequency : 0.0;
    }
    if (SW_PT == rigid) {  // Rigid_spec[0..] (input.cxx:1583-1700) and switch.free_rigid (:1961-2008)
        p.rigid = 1;
        for (int s = 0; s < Component_Number && s < SPM_MAX_SPECIES; s++) {
            p.rigid_beads[s] = Beads_Numbers[s];
            p.rigid_count[s] = Chain_Numbers[s];
            for (int d = 0; d < DIM; d++) {
                p.rigid_free[s][d]     = Rigid_Motions_vel[s][d];
                p.rigid_free[s][3 + d] = Rigid_Motions_omega[s][d];
                p.rigid_velocity[s][d] = Rigid_Velocities[s][d];
                p.rigid_omega[s][d]    = Rigid_Omegas[s][d];
            }
        }
    }
    if (G != 0.0) {  // Add_f_gravity (md_force.cxx:306-324): on the bodies, or a constant force on the spheres
        if (SW_PT == rigid) {
            p.rigid_gravity[G_direction] = G;
        } else {
            const double R = A * DX;
            p.body_force[G_direction] = -(G * RHO * 4.0 / 3.0 * M_PI * R * R * R) * (MASS_RATIOS[0] - 1.0);
        }
    }
    if (Component_Number > 1) {  // species: Particle_spec[0..] (Rigid_spec[0..]) in particle order
        p.n_species = Component_Number;
        for (int s = 0; s < Component_Number && s < SPM_MAX_SPECIES; s++) {
            p.species_count[s]          = Particle_Numbers[s];
            p.species_mass_ratio[s]     = MASS_RATIOS[s];
            p.species_surface_charge[s] = Surface_charge ? Surface_charge[s] : 0.0;
        }
    }
    if (SW_JANUS) {  // Particle_spec[0]'s propulsion (input.cxx:1403-1470; the slip mode is kept halved, :583)
        const JP  jp = janus_propulsion[0];
        const JAX ja = janus_axis[0];
        p.janus_propulsion = jp == motor ? SPM_JANUS_TUMBLER : jp == slip ? SPM_JANUS_SQUIRMER
                           : jp == obstacle ? SPM_JANUS_OBSTACLE : SPM_JANUS_OFF;
        p.janus_axis = ja == x_axis ? SPM_AXIS_X : ja == y_axis ? SPM_AXIS_Y : ja == z_axis ? SPM_AXIS_Z : SPM_AXIS_NONE;
        for (int d = 0; d < DIM; d++) {
            p.janus_force[d]  = janus_force[0][d];
            p.janus_torque[d] = janus_torque[0][d];
        }
        p.slip_vel  = janus_slip_vel[0];
        p.slip_mode = 2.0 * janus_slip_mode[0];
        p.rotlet_c1 = janus_rotlet_C1[0];
        p.rotlet_c2 = janus_rotlet_dipole_C2[0];
        p.slip_tol  = MAX_SLIP_TOL;
        p.slip_iter = MAX_SLIP_ITER;
    }
    p.dt        = DT;
    p.precision = SPM_PREC_FP64;
    return p;
}

// Particle -> records (SPM_PARTICLE_WORDS doubles each, header layout).
inline double *records(const Particle *p, std::vector<double> &rec) {
    rec.assign((size_t)Particle_Number * SPM_PARTICLE_WORDS, 0.0);
    for (int n = 0; n < Particle_Number; n++) {
        double         *r   = rec.data() + (size_t)n * SPM_PARTICLE_WORDS;
        const Particle &q   = p[n];
        const double   *a[] = {q.x, q.x_nopbc, q.v, q.v_old, q.omega, q.omega_old};
        for (int i = 0; i < 6; i++)
            for (int d = 0; d < 3; d++) r[3 * i + d] = a[i][d];
        r[18] = q.q.s;
        r[22] = q.q_old.s;
        for (int d = 0; d < 3; d++) {
            r[19 + d] = q.q.v[d];
            r[23 + d] = q.q_old.v[d];
        }
        const double *b[] = {q.f_hydro, q.f_hydro_previous, q.torque_hydro, q.torque_hydro_previous, q.fr,
                             q.fr_previous};
        for (int i = 0; i < 6; i++)
            for (int d = 0; d < 3; d++) r[26 + 3 * i + d] = b[i][d];
    }
    return rec.data();
}

// records -> Particle (the members the records carry).
inline void unpack_records(const double *rec, Particle *p) {
    for (int n = 0; n < Particle_Number; n++) {
        const double *r   = rec + (size_t)n * SPM_PARTICLE_WORDS;
        Particle     &q   = p[n];
        double       *a[] = {q.x, q.x_nopbc, q.v, q.v_old, q.omega, q.omega_old};
        for (int i = 0; i < 6; i++)
            for (int d = 0; d < 3; d++) a[i][d] = r[3 * i + d];
        q.q.s     = r[18];
        q.q_old.s = r[22];
        for (int d = 0; d < 3; d++) {
            q.q.v[d]     = r[19 + d];
            q.q_old.v[d] = r[23 + d];
        }
        double *b[] = {q.f_hydro, q.f_hydro_previous, q.torque_hydro, q.torque_hydro_previous, q.fr,
                       q.fr_previous};
        for (int i = 0; i < 6; i++)
            for (int d = 0; d < 3; d++) b[i][d] = r[26 + 3 * i + d];
    }
}

}  // namespace kapsel_b200
