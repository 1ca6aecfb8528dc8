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
// (SPM_EQ_NAVIER_STOKES or SPM_EQ_LEES_EDWARDS), FP64, one particle species.
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
