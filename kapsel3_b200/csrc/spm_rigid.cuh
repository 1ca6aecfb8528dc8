// Rigid bodies built from spherical beads (SW_PT == rigid; rigid.h,
// rigid_body.cxx, make_phi.cxx:589-801, md_force.cxx:383-506, fluct.cxx:40-95).
//
// A body is the beads [first[b], first[b+1]) of the particle arrays.  Its
// state: centre of mass xG (with and without the periodic wrap), velocity vG
// and angular velocity wG (space frame) with their previous values, the
// hydrodynamic force and torque (fG, tG) and the bead-bead (Lennard-Jones)
// ones (fGr, tGr) with their previous values, the mass, the space-frame
// inertia tensor I and its inverse, and the body-frame tensor Ibody (diagonal
// by construction).  Every bead keeps its offset from the centre in the body
// frame (gr_body) and in space (gr = R(q) gr_body, q the orientation of the
// body's first bead, which all its beads share).
//
// One block per body: thread 0 advances the body, then the block updates its
// beads.
#pragma once

#include "spm_janus.cuh"  // block_sum_n

namespace spm {

struct RigidDev {
    int     nb = 0;
    int    *first = nullptr;  // [nb + 1]
    int    *spec  = nullptr;  // [nb]
    int    *rid   = nullptr;  // [np] body of each bead
    double *xg = nullptr, *xg_nopbc = nullptr, *xg_prev = nullptr;           // [nb][3]
    double *vg = nullptr, *vg_old = nullptr, *wg = nullptr, *wg_old = nullptr;  // [nb][3]
    double *fg = nullptr, *fgr = nullptr, *tg = nullptr, *tgr = nullptr;        // [nb][3]
    double *fg_prev = nullptr, *fgr_prev = nullptr, *tg_prev = nullptr, *tgr_prev = nullptr;
    double *mass = nullptr, *imass = nullptr;              // [nb]
    double *I = nullptr, *Iinv = nullptr, *Ibody = nullptr;  // [nb][9], row-major
    double *gr = nullptr, *gr_body = nullptr;              // [np][3]
    double *f_lo  = nullptr;  // [np][3] LJ force on a bead from the pairs where it is the lower index
    double *noise = nullptr;  // [np][6] the thermostat's normal draws of each bead
    double *red   = nullptr;  // [nb][12] reductions of the set-up (mass, centre, inertia)
};
// Degrees of freedom per species (Rigid_Motions_vel / _omega, 1 free, 0 fixed).
struct RigidFree {
    int    v[4][3];
    int    w[4][3];
    double grav[3];  // G along G_direction
    double mr[4];    // the species' MASS_RATIO
};

__device__ __forceinline__ void cross3(const double *a, const double *b, double *c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// A' = R A R^T for BODY2SPACE (conj = false) and R^T A R for SPACE2BODY, in
// the reference's order of operations (rigid_body_matrix_rotation,
// rigid_body.cxx:26-62): the columns rotated, transposed, the rows rotated.
__device__ __forceinline__ void matrix_rotation_d(const double *q, const double *A, double *out, bool conj) {
    double c[3][3], t[9];
    for (int j = 0; j < 3; j++) {
        const double col[3] = {A[j], A[3 + j], A[6 + j]};
        qtn_rotate_d(q, col, c[j], conj);
    }
    for (int j = 0; j < 3; j++)
        for (int i = 0; i < 3; i++) t[3 * i + j] = c[j][i];
    for (int i = 0; i < 3; i++) qtn_rotate_d(q, t + 3 * i, out + 3 * i, conj);
}

// Inverse of a 3x3 matrix by its adjugate (the inverse of the inertia tensor,
// Matrix_Inverse of rigid.h:282).
__device__ __host__ __forceinline__ void inverse3(const double *A, double *B) {
    const double c00 = A[4] * A[8] - A[5] * A[7], c01 = A[5] * A[6] - A[3] * A[8], c02 = A[3] * A[7] - A[4] * A[6];
    const double det = A[0] * c00 + A[1] * c01 + A[2] * c02;
    const double id  = 1.0 / det;
    B[0]             = c00 * id;
    B[1]             = (A[2] * A[7] - A[1] * A[8]) * id;
    B[2]             = (A[1] * A[5] - A[2] * A[4]) * id;
    B[3]             = c01 * id;
    B[4]             = (A[0] * A[8] - A[2] * A[6]) * id;
    B[5]             = (A[2] * A[3] - A[0] * A[5]) * id;
    B[6]             = c02 * id;
    B[7]             = (A[1] * A[6] - A[0] * A[7]) * id;
    B[8]             = (A[0] * A[4] - A[1] * A[3]) * id;
}

// solver_Rigid_Position (Euler / AB2, rigid.h:333-404) followed by
// update_Orientation (rigid.h:252-276) and update_Particle_Configuration
// (rigid.h:171-188).  Euler when the run's step counter is 0.
// Lees-Edwards (le != 0; solver_Rigid_Position_OBL, rigid.h:400-463, and
// update_Particle_Configuration_OBL, rigid.h:190-210): the centre and every
// bead take the oblique wrap PBC_OBL of degree_oblique gam, and a crossing of
// the y boundary shifts vG, vG_old (the centre's) or the bead's v, v_old by
// -+ Shear_rate_eff LY (*srate).
__global__ void r_position(Phys ph, PState s, RigidDev R, const int *__restrict__ ts_dev, int le, double gam,
                           const double *__restrict__ srate) {
    const int b = blockIdx.x;
    if (b >= R.nb) return;
    const int f0 = R.first[b], f1 = R.first[b + 1];
    __shared__ double q[4], qo[4], xg[3], vg[3], wg[3];
    if (threadIdx.x == 0) {
        const int euler = *ts_dev == 0;
        for (int d = 0; d < 3; d++) {
            const int i     = 3 * b + d;
            R.xg_prev[i]    = R.xg[i];
            const double dl = euler ? ph.dt * R.vg[i] : ph.hdt * (3.0 * R.vg[i] - R.vg_old[i]);
            R.xg[i] += dl;
            R.xg_nopbc[i] += dl;
            if (!le) R.xg[i] = fmod(R.xg[i] + ph.L[d], ph.L[d]);
        }
        if (le) {
            const double dvx = pbc_obl(ph, R.xg + 3 * b, gam, *srate);
            R.vg[3 * b] += dvx;
            R.vg_old[3 * b] += dvx;
        }
        for (int d = 0; d < 3; d++) {
            xg[d] = R.xg[3 * b + d];
            vg[d] = R.vg[3 * b + d];
            wg[d] = R.wg[3 * b + d];
        }
        // MD_solver_orientation_Euler / _AB2 on the first bead
        double *qb = s.q + 4 * f0, *qob = s.q_old + 4 * f0;
        double  dq[4];
        if (euler) {
            for (int k = 0; k < 4; k++) qob[k] = qb[k];
            qdot_space_d(qb, s.omega + 3 * f0, dq);
            for (int k = 0; k < 4; k++) qb[k] += dq[k] * ph.dt;
        } else {
            double dqo[4];
            qdot_space_d(qb, s.omega + 3 * f0, dq);
            qdot_space_d(qob, s.omega_old + 3 * f0, dqo);
            for (int k = 0; k < 4; k++) qob[k] = qb[k];
            for (int k = 0; k < 4; k++) qb[k] += dq[k] * (3.0 * ph.hdt);
            for (int k = 0; k < 4; k++) qb[k] += dqo[k] * (-ph.hdt);
        }
        qtn_normalize_d(qb);
        for (int k = 0; k < 4; k++) {
            q[k]  = qb[k];
            qo[k] = qob[k];
        }
        // the space-frame inertia tensor of the new orientation and its inverse
        matrix_rotation_d(q, R.Ibody + 9 * b, R.I + 9 * b, false);
        inverse3(R.I + 9 * b, R.Iinv + 9 * b);
    }
    __syncthreads();
    for (int n = f0 + threadIdx.x; n < f1; n += blockDim.x) {
        if (n != f0)
            for (int k = 0; k < 4; k++) {
                s.q[4 * n + k]     = q[k];
                s.q_old[4 * n + k] = qo[k];
            }
        double gr[3];
        qtn_rotate_d(q, R.gr_body + 3 * n, gr, false);
        double vr[3];
        cross3(wg, gr, vr);
        for (int d = 0; d < 3; d++) {
            const int i       = 3 * n + d;
            R.gr[i]           = gr[d];
            s.x_previous[i]   = s.x[i];
            s.x[i]            = le ? xg[d] + gr[d] : fmod(xg[d] + gr[d] + ph.L[d], ph.L[d]);
            s.omega_old[i]    = s.omega[i];
            s.v_old[i]        = s.v[i];
            s.omega[i]        = wg[d];
            s.v[i]            = vg[d] + vr[d];
        }
        if (le) {
            const double dvx = pbc_obl(ph, s.x + 3 * n, gam, *srate);
            s.v_old[3 * n] += dvx;
            s.v[3 * n] += dvx;
        }
    }
}

// Per body: the hydrodynamic force and torque about the centre of mass from
// its beads' (Calc_f_hydro_correct_precision, md_force.cxx:457-501: forceGs =
// sum f_hydro, torqueGs = sum (GR + r) x f = sum GR x f_hydro + torque_hydro),
// and the Lennard-Jones ones (md_force.cxx:123-143): forceGrs = sum fr,
// torqueGrs = sum GR x (f_hi - f_lo), where a bead's pair forces as the higher
// index of a pair enter with their sign and those as the lower index with the
// opposite sign, as the reference adds GRvecs[j] x dmy_fi for both partners.
// Lees-Edwards (obl != 0; Calc_f_Lennard_Jones_shear_cap_primitive,
// md_force.cxx:244-258): the reference adds GRvecs x dmy_fn, the force on
// the lower index, for both partners, so there torqueGrs = sum GR x (f_lo -
// f_hi).
__global__ void r_collect(PState s, RigidDev R, RigidFree fr, int obl) {
    const int b = blockIdx.x;
    if (b >= R.nb) return;
    double acc[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int n = R.first[b] + threadIdx.x; n < R.first[b + 1]; n += blockDim.x) {
        const double *gr = R.gr + 3 * n, *fh = s.f_hydro + 3 * n, *th = s.torque_hydro + 3 * n;
        const double *fr = s.fr + 3 * n, *fl = R.f_lo + 3 * n;
        double        c[3], fs[3];
        cross3(gr, fh, c);
        for (int d = 0; d < 3; d++) {
            acc[d] += fh[d];
            acc[3 + d] += c[d] + th[d];
            acc[6 + d] += fr[d];
            fs[d] = obl ? 2.0 * fl[d] - fr[d] : fr[d] - 2.0 * fl[d];
        }
        cross3(gr, fs, c);
        for (int d = 0; d < 3; d++) acc[9 + d] += c[d];
    }
    block_sum_n<12>(acc);
    if (threadIdx.x == 0) {
        // gravity after the pair forces (Force, particle_solver.h:88-96): -G RHO V (MASS_RATIO - 1)
        // with RHO V = mass / MASS_RATIO
        const double mr = fr.mr[R.spec[b]];
        for (int d = 0; d < 3; d++) {
            R.fg[3 * b + d]  = acc[d];
            R.tg[3 * b + d]  = acc[3 + d];
            R.fgr[3 * b + d] = acc[6 + d];
            if (fr.grav[d] != 0.0) R.fgr[3 * b + d] -= fr.grav[d] * (R.mass[b] / mr) * (mr - 1.0);
            R.tgr[3 * b + d] = acc[9 + d];
        }
    }
}

// Euler's equations in the body frame (MD_solver_omega_Euler / _AB2,
// particle_rotation_solver.h:106-182): only the free components change.
__device__ __forceinline__ void omega_update_body(double *wg, const double *torque, const double *torque_old,
                                                  const double *Ib, const double *q, const double *q_old,
                                                  const int *freew, double dt, bool ab2) {
    double wb[3], tb[3], tbo[3] = {0, 0, 0};
    qtn_rotate_d(q, wg, wb, true);
    qtn_rotate_d(q, torque, tb, true);
    if (ab2) qtn_rotate_d(q_old, torque_old, tbo, true);
    double nw[3]   = {wb[0], wb[1], wb[2]};
    const double k = ab2 ? 2.0 : 1.0;
    for (int d = 0; d < 3; d++) {
        if (!freew[d]) continue;
        const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
        const double t = ab2 ? (tb[d] + tbo[d]) : tb[d];
        nw[d] += (dt / Ib[d]) * (t + k * (Ib[d1] - Ib[d2]) * wb[d1] * wb[d2]);
    }
    qtn_rotate_d(q, nw, wg, false);
}

// calc_Rigid_VOGs (rigid.h:409-527) and set_Particle_Velocities
// (rigid.h:213-225), then reset_Forces on the beads (particle_solver.cxx:11-37).
// Euler when the run's step counter is 0.  Lees-Edwards (le != 0;
// set_Particle_Velocities_OBL, rigid.h:232-250): a bead whose position
// xG + GR lies across the y boundary gets the v_x shift of that image.
__global__ void r_velocity(Phys ph, PState s, RigidDev R, RigidFree fr, const int *__restrict__ ts_dev, int le,
                           double gam, const double *__restrict__ srate) {
    const int b = blockIdx.x;
    if (b >= R.nb) return;
    const int f0 = R.first[b], f1 = R.first[b + 1];
    __shared__ double vg[3], wg[3];
    if (threadIdx.x == 0) {
        const int  sp    = R.spec[b];
        const bool euler = *ts_dev == 0;
        double    *v = R.vg + 3 * b, *w = R.wg + 3 * b;
        for (int d = 0; d < 3; d++) {
            R.vg_old[3 * b + d] = v[d];
            R.wg_old[3 * b + d] = w[d];
        }
        const double *fg = R.fg + 3 * b, *fgr = R.fgr + 3 * b, *fgrp = R.fgr_prev + 3 * b;
        const double *tg = R.tg + 3 * b, *tgr = R.tgr + 3 * b, *tgrp = R.tgr_prev + 3 * b;
        const double  Ib[3] = {R.Ibody[9 * b + 0], R.Ibody[9 * b + 4], R.Ibody[9 * b + 8]};
        if (euler) {
            const double dmy = ph.dt * R.imass[b];
            for (int d = 0; d < 3; d++)
                if (fr.v[sp][d]) v[d] += dmy * (fg[d] + fgr[d]);
            const double t[3] = {tg[0] + tgr[0], tg[1] + tgr[1], tg[2] + tgr[2]};
            omega_update_body(w, t, nullptr, Ib, s.q + 4 * f0, nullptr, fr.w[sp], ph.dt, false);
        } else {
            const double dmy = ph.hdt * R.imass[b];
            for (int d = 0; d < 3; d++)
                if (fr.v[sp][d]) v[d] += dmy * (2.0 * fg[d] + fgr[d] + fgrp[d]);
            const double t[3]  = {2.0 * tg[0] + tgr[0], 2.0 * tg[1] + tgr[1], 2.0 * tg[2] + tgr[2]};
            const double tp[3] = {tgrp[0], tgrp[1], tgrp[2]};
            omega_update_body(w, t, tp, Ib, s.q + 4 * f0, s.q_old + 4 * f0, fr.w[sp], ph.hdt, true);
        }
        for (int d = 0; d < 3; d++) {
            const int i   = 3 * b + d;
            R.fg_prev[i]  = R.fg[i];
            R.fgr_prev[i] = R.fgr[i];
            R.tg_prev[i]  = R.tg[i];
            R.tgr_prev[i] = R.tgr[i];
            R.fg[i] = R.fgr[i] = R.tg[i] = R.tgr[i] = 0.0;
            vg[d]                                    = v[d];
            wg[d]                                    = w[d];
        }
    }
    __syncthreads();
    for (int n = f0 + threadIdx.x; n < f1; n += blockDim.x) {
        double vr[3];
        cross3(wg, R.gr + 3 * n, vr);
        double dvx = 0.0;
        if (le) {
            double r[3] = {R.xg[3 * b] + R.gr[3 * n], R.xg[3 * b + 1] + R.gr[3 * n + 1],
                           R.xg[3 * b + 2] + R.gr[3 * n + 2]};
            dvx = pbc_obl(ph, r, gam, *srate);
        }
        for (int d = 0; d < 3; d++) {
            const int i               = 3 * n + d;
            s.omega[i]                = wg[d];
            s.v[i]                    = vg[d] + vr[d] + (d == 0 ? dvx : 0.0);
            s.fr_previous[i]          = s.fr[i];
            s.fr[i]                   = 0.0;
            s.f_hydro_previous[i]     = s.f_hydro[i];
            s.f_hydro[i]              = 0.0;
            s.torque_r_previous[i]    = s.torque_r[i];
            s.torque_r[i]             = 0.0;
            s.torque_hydro_previous[i] = s.torque_hydro[i];
            s.torque_hydro[i]         = 0.0;
        }
    }
}

// Lees-Edwards: the bodies' term of the new hydrodynamic stress
// (Calc_f_hydro_correct_precision_OBL, md_force.cxx:690-716).  With the
// body's hydrodynamic force and torque of this step (r_collect), dVg = dt
// IMass forceGs and dWg the Euler change of wG under torqueGs in the body
// frame (MD_solver_omega_Euler_update, particle_rotation_solver.h:129-145);
// each bead's new_p (ppart[4]) gains
//   RHO_p sum_mesh (dVg_x + dWg_y (GR_z + r_z) - dWg_z (GR_y + r_y)) dry w
// = RHO_p (Y (dVg_x + dWg_y GR_z - dWg_z GR_y) + dWg_y Yz - dWg_z Yy)
// from the bead's stencil moments Y, Yy, Yz (ppart[1], [6], [7]).
__global__ void r_le_stress_new(Phys ph, PState s, RigidDev R, RigidFree fr, double *__restrict__ ppart, int stride) {
    const int b = blockIdx.x;
    if (b >= R.nb) return;
    const int f0 = R.first[b], f1 = R.first[b + 1];
    __shared__ double dv, dw[3];
    if (threadIdx.x == 0) {
        dv = ph.dt * R.imass[b] * R.fg[3 * b];
        const double *q = s.q + 4 * f0;
        double        wb[3], tb[3], d[3];
        qtn_rotate_d(q, R.wg + 3 * b, wb, true);
        qtn_rotate_d(q, R.tg + 3 * b, tb, true);
        const double Ib[3] = {R.Ibody[9 * b + 0], R.Ibody[9 * b + 4], R.Ibody[9 * b + 8]};
        d[0] = (ph.dt / Ib[0]) * (tb[0] + (Ib[1] - Ib[2]) * wb[1] * wb[2]);
        d[1] = (ph.dt / Ib[1]) * (tb[1] + (Ib[2] - Ib[0]) * wb[2] * wb[0]);
        d[2] = (ph.dt / Ib[2]) * (tb[2] + (Ib[0] - Ib[1]) * wb[0] * wb[1]);
        qtn_rotate_d(q, d, dw, false);
    }
    __syncthreads();
    const double rho_p = fr.mr[R.spec[b]] * ph.rho;
    for (int n = f0 + threadIdx.x; n < f1; n += blockDim.x) {
        double       *pp = ppart + (size_t)stride * n;
        const double *gr = R.gr + 3 * n;
        pp[4] += rho_p * (pp[1] * (dv + dw[1] * gr[2] - dw[2] * gr[1]) + dw[1] * pp[7] - dw[2] * pp[6]);
    }
}

// The thermostat of rigid bodies (Add_random_force_thermostat, fluct.cxx:40-95):
// every bead's six normals (drawn in the reference's order into R.noise) give
// a force and torque kick; per body their sum, with the torque of the forces
// about the centre, changes the free components of vG (by the inverse mass)
// and of wG (by the inverse space-frame inertia tensor), and the beads'
// velocities follow (their angular velocities are left as they are, as in
// the reference).
__global__ void r_thermostat(Phys ph, PState s, RigidDev R, RigidFree fr) {
    const int b = blockIdx.x;
    if (b >= R.nb) return;
    const int f0 = R.first[b], f1 = R.first[b + 1];
    double    acc[6] = {0, 0, 0, 0, 0, 0};
    for (int n = f0 + threadIdx.x; n < f1; n += blockDim.x) {
        double fdt[3], c[3];
        for (int d = 0; d < 3; d++) {
            fdt[d] = R.noise[6 * n + d] * ph.noise_v;
            acc[d] += fdt[d];
            acc[3 + d] += R.noise[6 * n + 3 + d] * ph.noise_o;
        }
        cross3(R.gr + 3 * n, fdt, c);
        for (int d = 0; d < 3; d++) acc[3 + d] += c[d];
    }
    block_sum_n<6>(acc);
    __shared__ double vg[3], wg[3];
    if (threadIdx.x == 0) {
        const int sp = R.spec[b];
        double   *v = R.vg + 3 * b, *w = R.wg + 3 * b;
        for (int d = 0; d < 3; d++)
            if (fr.v[sp][d]) v[d] += acc[d] * R.imass[b];
        for (int d1 = 0; d1 < 3; d1++) {
            if (!fr.w[sp][d1]) continue;
            for (int d2 = 0; d2 < 3; d2++) w[d1] += R.Iinv[9 * b + 3 * d1 + d2] * acc[3 + d2];
        }
        for (int d = 0; d < 3; d++) {
            vg[d] = v[d];
            wg[d] = w[d];
        }
    }
    __syncthreads();
    for (int n = f0 + threadIdx.x; n < f1; n += blockDim.x) {
        double vr[3];
        cross3(wg, R.gr + 3 * n, vr);
        for (int d = 0; d < 3; d++) s.v[3 * n + d] = vg[d] + vr[d];
    }
}

// Set-up reductions over the beads' profiles with the overlap weight
// Phi / max(phi_sum, 1) (Make_phi_rigid_mass, make_phi.cxx:589-629, mode 0:
// sum w and sum w (GR + r); Make_phi_rigid_inertia, make_phi.cxx:678-735,
// mode 1: the nine sums w I(GR + r)).  red[b] receives the sums.
template <typename T>
__global__ void r_setup_sums(Grid g, Phys ph, const double *__restrict__ x, const int *__restrict__ cells, int ncells,
                             const T *__restrict__ phi_sum, RigidDev R, int mode) {
    const int b = blockIdx.x;
    if (b >= R.nb) return;
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int n = R.first[b]; n < R.first[b + 1]; n++) {
        const double xp[3] = {x[3 * n], x[3 * n + 1], x[3 * n + 2]};
        const double *gr   = R.gr + 3 * n;
        for (int m = threadIdx.x; m < ncells; m += blockDim.x) {
            StencilPoint sp;
            stencil_point(g, ph, xp, cells[m], sp);
            const double ps  = (double)phi_sum[sp.idx];
            const double wgt = phi_prof(sp.dist, ph.radius, ph.hxi, g.dx) / (ps > 1.0 ? ps : 1.0);
            const double ri[3] = {gr[0] + sp.r[0], gr[1] + sp.r[1], gr[2] + sp.r[2]};
            if (mode == 0) {
                acc[0] += wgt;
                for (int d = 0; d < 3; d++) acc[1 + d] += wgt * ri[d];
            } else {
                acc[0] += wgt * (ri[1] * ri[1] + ri[2] * ri[2]);
                acc[1] += wgt * (-ri[0] * ri[1]);
                acc[2] += wgt * (-ri[0] * ri[2]);
                acc[3] += wgt * (-ri[1] * ri[0]);
                acc[4] += wgt * (ri[0] * ri[0] + ri[2] * ri[2]);
                acc[5] += wgt * (-ri[1] * ri[2]);
                acc[6] += wgt * (-ri[2] * ri[0]);
                acc[7] += wgt * (-ri[2] * ri[1]);
                acc[8] += wgt * (ri[0] * ri[0] + ri[1] * ri[1]);
            }
        }
    }
    block_sum_n<9>(acc);
    if (threadIdx.x == 0)
        for (int k = 0; k < 9; k++) R.red[12 * b + k] = acc[k];
}

}  // namespace spm
