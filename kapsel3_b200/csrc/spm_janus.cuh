// Squirmers: spherical particles with a prescribed surface slip velocity,
// driven by the reference's self-consistent slip iteration (the SW_JANUS_SLIP
// branch of Time_evolution_hydro, sp_3d_ns.cxx:121-161; operate_surface.cxx;
// operate_surface.h:64-120; Calc_f_slip_correct_precision, md_force.cxx:
// 325-382; MD_solver_velocity_slip_*, particle_solver.cxx:144-237).
// Particle reductions are FP64 block sums over the stencil, one CTA per
// particle; field scatters use atomics, as the Navier_Stokes kernels do.
#pragma once

#include "spm_kernels.cuh"

namespace spm {

// Per-particle slip state, kSlipWords doubles per particle.
constexpr int kSlipV      = 0;   // v_slip[3]
constexpr int kSlipW      = 3;   // omega_slip[3]
constexpr int kSlipF      = 6;   // f_slip[3]
constexpr int kSlipT      = 9;   // torque_slip[3]
constexpr int kSlipMass   = 12;  // mass (sum of phi)
constexpr int kSlipSMass  = 13;  // surface_mass
constexpr int kSlipMC     = 14;  // mass_center[3]
constexpr int kSlipSMC    = 17;  // surface_mass_center[3]
constexpr int kSlipDV     = 20;  // surface_dv[3]
constexpr int kSlipDW     = 23;  // surface_dw[3]
constexpr int kSlipI      = 26;  // inertia[3][3]
constexpr int kSlipSI     = 35;  // surface_inertia[3][3]
constexpr int kSlipDeltaV = 44;  // delta_v[3] (droplet counter-flow)
constexpr int kSlipDeltaW = 47;  // delta_w[3]
constexpr int kSlipFPrev  = 50;  // f_slip_previous[3]
constexpr int kSlipTPrev  = 53;  // torque_slip_previous[3]
constexpr int kSlipWords  = 56;

constexpr double kEpsMP = 2.220446049250313e-16;  // DBL_EPSILON (macro.h:36)
constexpr double kTolMP = 10.0 * kEpsMP;          // TOL_MP (macro.h:37)

// less_than_mp (macro.h:164-167)
__device__ __forceinline__ bool less_than_mp_d(double a, double b) {
    const double eps = (fmax(fabs(a), fabs(b)) + 10.0) * kEpsMP;
    return (b - a) > eps;
}

// DPhi_compact_sin_norm (profile.h:175-184): cos(pi (R - x) / XI) inside the
// interface, else 0.
__device__ __forceinline__ double dphi_sin_norm(double x, double radius, double xi) {
    const double dmy_x = radius - x;
    if (fabs(dmy_x) < xi * 0.5) return cos(M_PI * dmy_x * (1.0 / xi));
    return 0.0;
}

// Squirmer_coord (make_phi.h:282-375): unit vectors n_r, n_theta, n_tau of a
// surface point at relative position x in the space frame, and the polar
// angle theta from the janus axis e3 of the body frame.
__device__ __forceinline__ void squirmer_coord(const double *x, const double *q, int axis, double *nr, double *nth,
                                               double *ntau, double &theta) {
    // e3: the body frame's janus axis (z, y or x)
    double e3[3] = {0, 0, 0};
    e3[axis == 3 ? 2 : axis == 2 ? 1 : 0] = 1.0;
    double r[3];
    qtn_rotate_d(q, x, r, true);  // SPACE2BODY
    double norm_r = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    double inv    = 1.0 / norm_r;
    for (int d = 0; d < 3; d++) r[d] *= inv;
    double ph[3] = {e3[1] * r[2] - e3[2] * r[1], e3[2] * r[0] - e3[0] * r[2], e3[0] * r[1] - e3[1] * r[0]};
    const double dot   = e3[0] * r[0] + e3[1] * r[1] + e3[2] * r[2];
    const double pnorm = sqrt(ph[0] * ph[0] + ph[1] * ph[1] + ph[2] * ph[2]);
    if ((pnorm > kTolMP || -kTolMP > pnorm) && less_than_mp_d(fabs(dot), 1.0)) {
        inv = 1.0 / pnorm;
        for (int d = 0; d < 3; d++) ph[d] *= inv;
        theta = acos(dot);
        double th[3] = {ph[1] * r[2] - ph[2] * r[1], ph[2] * r[0] - ph[0] * r[2], ph[0] * r[1] - ph[1] * r[0]};
        inv = 1.0 / sqrt(th[0] * th[0] + th[1] * th[1] + th[2] * th[2]);
        for (int d = 0; d < 3; d++) th[d] *= inv;
        qtn_rotate_d(q, r, nr, false);  // BODY2SPACE
        qtn_rotate_d(q, th, nth, false);
        qtn_rotate_d(q, ph, ntau, false);
    } else {  // r along the janus axis: no tangent vectors
        norm_r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        inv    = 1.0 / norm_r;
        for (int d = 0; d < 3; d++) nr[d] = x[d] * inv, nth[d] = 0.0, ntau[d] = 0.0;
        theta = dot > 0.0 ? 0.0 : M_PI;
    }
}

// Block-wide sum of N doubles (blockDim.x a multiple of 32, <= 1024); the
// result is valid in thread 0.  Fixed reduction order.
template <int N>
__device__ __forceinline__ void block_sum_n(double v[N]) {
    __shared__ double red[32][N];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < N; k++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < N; k++) red[wid][k] = v[k];
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < N; k++) {
            double a = lane < nw ? red[lane][k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
            v[k] = a;
        }
    }
}

// Make_particle_momentum_factor (operate_surface.cxx:12-153): the particle's
// phi moments (mass, centre, inertia) and, over its slip interface, the
// surface moments and the momentum change dv_s, dw_s of the slip profile
// relative to the fluid u.  One CTA per particle.
template <typename T>
__global__ void __launch_bounds__(256) s_slip_moments(Grid g, Phys ph, const double *__restrict__ x,
                                                      const double *__restrict__ q, const int *__restrict__ cells,
                                                      int ncells, const T *__restrict__ u0,
                                                      const T *__restrict__ u1, const T *__restrict__ u2,
                                                      double *__restrict__ slip) {
    const int p = blockIdx.x;
    if (p >= ph.np) return;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    const double qp[4] = {q[4 * p], q[4 * p + 1], q[4 * p + 2], q[4 * p + 3]};
    // acc: M0, SM0, M1[3], SM1[3], M2[9], SM2[9], dv[3], dw[3]
    double acc[32];
#pragma unroll
    for (int k = 0; k < 32; k++) acc[k] = 0.0;
    if (particle_in_box(ph, xp)) {
        for (int m = threadIdx.x; m < ncells; m += blockDim.x) {
            StencilPoint s;
            stencil_point(g, ph, xp, cells[m], s);
            const double r2  = s.dist * s.dist;
            const double phi = phi_prof(s.dist, ph.radius, ph.hxi, g.dx);
            acc[0] += phi;
            for (int d = 0; d < 3; d++) {
                acc[2 + d] += phi * s.r[d];
                acc[8 + 4 * d] += phi * r2;
                for (int l = 0; l < 3; l++) acc[8 + 3 * d + l] -= phi * s.r[d] * s.r[l];
            }
            if (ph.janus_prop == 2 && less_than_mp_d(fabs(s.dist - ph.radius), ph.hxi)) {
                const double phs = (1.0 - phi) * dphi_sin_norm(s.dist, ph.radius, ph.xi);
                acc[1] += phs;
                double nr[3], nth[3], ntau[3], th;
                squirmer_coord(s.r, qp, ph.janus_axis, nr, nth, ntau, th);
                const double mag = ph.slip_b1 * (sin(th) + ph.slip_mode * sin(2.0 * th));
                const double azi = ph.slip_c1 * sin(th) + ph.slip_c2 * 1.5 * sin(2.0 * th);
                const double uf[3] = {(double)u0[s.idx], (double)u1[s.idx], (double)u2[s.idx]};
                double       us[3];
                for (int d = 0; d < 3; d++) us[d] = nth[d] * mag + ntau[d] * azi - uf[d];
                const double rxu[3] = {s.r[1] * us[2] - s.r[2] * us[1], s.r[2] * us[0] - s.r[0] * us[2],
                                       s.r[0] * us[1] - s.r[1] * us[0]};
                for (int d = 0; d < 3; d++) {
                    acc[26 + d] += phs * us[d];
                    acc[29 + d] += phs * rxu[d];
                    acc[5 + d] += phs * s.r[d];
                    acc[17 + 4 * d] += phs * r2;
                    for (int l = 0; l < 3; l++) acc[17 + 3 * d + l] -= phs * s.r[d] * s.r[l];
                }
            }
        }
    }
    block_sum_n<32>(acc);
    if (threadIdx.x == 0) {
        double *sp        = slip + (size_t)p * kSlipWords;
        sp[kSlipMass]     = acc[0];
        sp[kSlipSMass]    = acc[1];
        for (int d = 0; d < 3; d++) {
            sp[kSlipMC + d]  = acc[2 + d];
            sp[kSlipSMC + d] = acc[5 + d];
            sp[kSlipDV + d]  = acc[26 + d];
            sp[kSlipDW + d]  = acc[29 + d];
        }
        for (int k = 0; k < 9; k++) sp[kSlipI + k] = acc[8 + k], sp[kSlipSI + k] = acc[17 + k];
    }
}

// slip_droplet (operate_surface.cxx:155-195): the velocity delta_v, delta_w
// of the counter-flow inside the particle that keeps the momentum change of
// the enforced slip (taken w.r.t. v_slip, omega_slip) at zero.  The 3 x 3
// inverse is the cofactor form of M_inv (lad3.h:219-236).  Thread per
// particle.
__global__ void p_slip_droplet(Phys ph, double *__restrict__ slip) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ph.np || ph.janus_prop != 2) return;
    double      *sp = slip + (size_t)n * kSlipWords;
    const double *vp = sp + kSlipV, *wp = sp + kSlipW, *mc = sp + kSlipMC, *smc = sp + kSlipSMC;
    const double *I = sp + kSlipI, *SI = sp + kSlipSI;
    const double imass = 1.0 / sp[kSlipMass];
    const double w_x_r[3] = {wp[1] * smc[2] - wp[2] * smc[1], wp[2] * smc[0] - wp[0] * smc[2],
                             wp[0] * smc[1] - wp[1] * smc[0]};
    const double r_x_v[3] = {smc[1] * vp[2] - smc[2] * vp[1], smc[2] * vp[0] - smc[0] * vp[2],
                             smc[0] * vp[1] - smc[1] * vp[0]};
    double dP[3], dL[3];
    for (int d = 0; d < 3; d++) {
        dP[d] = -(sp[kSlipSMass] * vp[d] + w_x_r[d] + sp[kSlipDV + d]);
        dL[d] = -(r_x_v[d] + SI[3 * d] * wp[0] + SI[3 * d + 1] * wp[1] + SI[3 * d + 2] * wp[2] + sp[kSlipDW + d]);
    }
    double L0[3] = {imass * (mc[1] * dP[2] - mc[2] * dP[1]), imass * (mc[2] * dP[0] - mc[0] * dP[2]),
                    imass * (mc[0] * dP[1] - mc[1] * dP[0])};
    const double mc2 = -(mc[0] * mc[0] + mc[1] * mc[1] + mc[2] * mc[2]) * imass;
    double       A[3][3];
    for (int d = 0; d < 3; d++) {
        L0[d] = dL[d] - L0[d];
        for (int l = 0; l < 3; l++) A[d][l] = (d == l ? mc2 : 0.0) + (I[3 * d + l] + imass * mc[d] * mc[l]);
    }
    const double det = -A[0][2] * A[1][1] * A[2][0] + A[0][1] * A[1][2] * A[2][0] + A[0][2] * A[1][0] * A[2][1] -
                       A[0][0] * A[1][2] * A[2][1] - A[0][1] * A[1][0] * A[2][2] + A[0][0] * A[1][1] * A[2][2];
    const double id = 1.0 / det;
    double       B[3][3];
    B[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) * id;
    B[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * id;
    B[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id;
    B[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) * id;
    B[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id;
    B[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * id;
    B[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) * id;
    B[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * id;
    B[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id;
    double dw[3];
    for (int d = 0; d < 3; d++) {
        double a = 0.0;
        for (int l = 0; l < 3; l++) a += B[d][l] * L0[l];
        dw[d] = a;
    }
    const double wxm[3] = {dw[1] * mc[2] - dw[2] * mc[1], dw[2] * mc[0] - dw[0] * mc[2], dw[0] * mc[1] - dw[1] * mc[0]};
    for (int d = 0; d < 3; d++) {
        sp[kSlipDeltaW + d] = dw[d];
        sp[kSlipDeltaV + d] = imass * (dP[d] - wxm[d]);
    }
}

// Make_force_u_slip_particle (operate_surface.cxx:197-360): up += phi
// (delta_v + delta_w x r) over the particle domain and, on the interface
// (|r| - RADIUS| < XI/2), phi_s (v_slip + omega_slip x r + u_s - u) with
// phi_s = (1 - phi) DPhi_compact_sin_norm and the squirmer slip u_s.
// Grid (cells, particles).
template <typename T>
__global__ void s_slip_scatter(Grid g, Phys ph, const double *__restrict__ x, const double *__restrict__ q,
                               const int *__restrict__ cells, int ncells, const double *__restrict__ slip,
                               const T *__restrict__ u0, const T *__restrict__ u1, const T *__restrict__ u2,
                               T *__restrict__ up0, T *__restrict__ up1, T *__restrict__ up2) {
    const int p = blockIdx.y;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ph.np || m >= ncells || ph.janus_prop != 2) return;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    if (!particle_in_box(ph, xp)) return;
    const double *sp = slip + (size_t)p * kSlipWords;
    StencilPoint  s;
    stencil_point(g, ph, xp, cells[m], s);
    const double phi = phi_prof(s.dist, ph.radius, ph.hxi, g.dx);
    const double *dv = sp + kSlipDeltaV, *dw = sp + kSlipDeltaW;
    double        fv[3];
    double        rot[3] = {0.0, 0.0, 0.0};
    if (ph.rotation) rot[0] = dw[1] * s.r[2] - dw[2] * s.r[1], rot[1] = dw[2] * s.r[0] - dw[0] * s.r[2],
                     rot[2] = dw[0] * s.r[1] - dw[1] * s.r[0];
    for (int d = 0; d < 3; d++) fv[d] = phi * (dv[d] + rot[d]);
    const double phs = (1.0 - phi) * dphi_sin_norm(s.dist, ph.radius, ph.xi);
    if (less_than_mp_d(fabs(s.dist - ph.radius), ph.hxi)) {
        const double *vp = sp + kSlipV, *wp = sp + kSlipW;
        double        vr[3] = {0.0, 0.0, 0.0};
        if (ph.rotation) vr[0] = wp[1] * s.r[2] - wp[2] * s.r[1], vr[1] = wp[2] * s.r[0] - wp[0] * s.r[2],
                         vr[2] = wp[0] * s.r[1] - wp[1] * s.r[0];
        const double qp[4] = {q[4 * p], q[4 * p + 1], q[4 * p + 2], q[4 * p + 3]};
        double       nr[3], nth[3], ntau[3], th;
        squirmer_coord(s.r, qp, ph.janus_axis, nr, nth, ntau, th);
        const double vs1 = ph.slip_b1 * (sin(th) + ph.slip_mode * sin(2.0 * th));
        const double vs2 = ph.slip_c1 * sin(th) + ph.slip_c2 * 1.5 * sin(2.0 * th);
        const double uf[3] = {(double)u0[s.idx], (double)u1[s.idx], (double)u2[s.idx]};
        // the two contributions are separate atomic adds in the reference
        for (int d = 0; d < 3; d++) {
            const double fs = phs * (vp[d] + vr[d] + nth[d] * vs1 + ntau[d] * vs2 - uf[d]);
            T *dst = d == 0 ? up0 : (d == 1 ? up1 : up2);
            if (fv[d] != 0.0) atomicAdd(&dst[s.idx], (T)fv[d]);
            atomicAdd(&dst[s.idx], (T)fs);
        }
    } else {
        if (fv[0] != 0.0) atomicAdd(&up0[s.idx], (T)fv[0]);
        if (fv[1] != 0.0) atomicAdd(&up1[s.idx], (T)fv[1]);
        if (fv[2] != 0.0) atomicAdd(&up2[s.idx], (T)fv[2]);
    }
}

// Calc_f_slip_correct_precision (md_force.cxx:325-382): f_slip = DX^3 RHO /
// dt sum phi up, torque_slip = DX^3 RHO / dt sum r x (phi up).  One CTA per
// particle.
template <typename T>
__global__ void __launch_bounds__(256) s_slip_force(Grid g, Phys ph, const double *__restrict__ x,
                                                    const int *__restrict__ cells, int ncells,
                                                    const T *__restrict__ up0, const T *__restrict__ up1,
                                                    const T *__restrict__ up2, double *__restrict__ slip) {
    const int p = blockIdx.x;
    if (p >= ph.np) return;
    const double xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    double       acc[6] = {0, 0, 0, 0, 0, 0};
    if (particle_in_box(ph, xp)) {
        for (int m = threadIdx.x; m < ncells; m += blockDim.x) {
            StencilPoint s;
            stencil_point(g, ph, xp, cells[m], s);
            const double phi = phi_prof(s.dist, ph.radius, ph.hxi, g.dx);
            if (phi == 0.0) continue;
            const double fp0 = (double)up0[s.idx] * phi, fp1 = (double)up1[s.idx] * phi, fp2 = (double)up2[s.idx] * phi;
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
        const double dmy = ph.dx3 * ph.rho / ph.dt;
        double      *sp  = slip + (size_t)p * kSlipWords;
        for (int d = 0; d < 6; d++) sp[kSlipF + d] = dmy * acc[d];
    }
}

// MD_solver_velocity_slip_iter (particle_solver.cxx:209-237) without its
// Force() call (the step computes the LJ and body forces beforehand).
// mode 0 (start / new): the Euler or AB2 update with f_hydro + f_slip (slip
// Euler / AB2, particle_solver.cxx:144-207); 1 (reset): v, omega back to
// v_old, omega_old; 2 (end): reset_Forces (particle_solver.cxx:11-37).
__global__ void p_velocity_slip(Phys ph, PState s, double *__restrict__ slip, const int *__restrict__ ts_dev,
                                int mode) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ph.np) return;
    double *sp = slip + (size_t)n * kSlipWords;
    if (mode == 0) {
        const int    euler = *ts_dev == 0;
        const double dmy   = (euler ? ph.dt : ph.hdt) * ph.imass_s[spec_of(ph, n)];
        const double dmr   = (euler ? ph.dt : ph.hdt) * ph.imoi_s[spec_of(ph, n)];
        double       sf[3], st[3];
        self_propulsion_d(ph, s.q + 4 * n, sf, st);
        for (int d = 0; d < 3; d++) {
            const int i    = 3 * n + d;
            s.v_old[i]     = s.v[i];
            s.omega_old[i] = s.omega[i];
            if (ph.janus_prop == 3) {
                s.v[i] = 0.0, s.omega[i] = 0.0;
            } else if (euler) {
                s.v[i] += dmy * (s.f_hydro[i] + sp[kSlipF + d] + s.fr[i] + sf[d]);
                s.omega[i] += dmr * (s.torque_hydro[i] + sp[kSlipT + d] + s.torque_r[i] + st[d]);
            } else {
                s.v[i] += dmy * (2.0 * (s.f_hydro[i] + sp[kSlipF + d] + sf[d]) + s.fr[i] + s.fr_previous[i]);
                s.omega[i] += dmr * (2.0 * (s.torque_hydro[i] + sp[kSlipT + d] + st[d]) + s.torque_r[i] +
                                     s.torque_r_previous[i]);
            }
        }
    } else if (mode == 1) {
        for (int d = 0; d < 3; d++) {
            const int i = 3 * n + d;
            s.v[i]      = s.v_old[i];
            s.omega[i]  = s.omega_old[i];
        }
    } else {
        for (int d = 0; d < 3; d++) {
            const int i                = 3 * n + d;
            s.fr_previous[i]           = s.fr[i];
            s.fr[i]                    = 0.0;
            s.f_hydro_previous[i]      = s.f_hydro[i];
            s.f_hydro[i]               = 0.0;
            sp[kSlipFPrev + d]         = sp[kSlipF + d];
            sp[kSlipF + d]             = 0.0;
            s.torque_r_previous[i]     = s.torque_r[i];
            s.torque_r[i]              = 0.0;
            s.torque_hydro_previous[i] = s.torque_hydro[i];
            s.torque_hydro[i]          = 0.0;
            sp[kSlipTPrev + d]         = sp[kSlipT + d];
            sp[kSlipT + d]             = 0.0;
        }
    }
}

// Update_slip_particle_velocity (operate_surface.h:95-116): iter 0 copies
// v, omega; later iterations relax with weight 0.7 on the new velocity.
__global__ void p_slip_relax(Phys ph, const PState s, double *__restrict__ slip, int iter) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ph.np) return;
    double      *sp      = slip + (size_t)n * kSlipWords;
    const double dmy_new = 0.7;
    const double dmy_old = 1.0 - dmy_new;
    for (int d = 0; d < 3; d++) {
        if (iter == 0) {
            sp[kSlipV + d] = s.v[3 * n + d];
            sp[kSlipW + d] = s.omega[3 * n + d];
        } else {
            sp[kSlipV + d] = dmy_old * sp[kSlipV + d] + dmy_new * s.v[3 * n + d];
            sp[kSlipW + d] = dmy_old * sp[kSlipW + d] + dmy_new * s.omega[3 * n + d];
        }
    }
}

// Slip_particle_convergence (operate_surface.h:64-94): sqrt of the largest
// over particles of |v_slip - v|^2 / |v|^2 + |w_slip - w|^2 / |w|^2 (a
// norm below TOL_MP leaves its term unscaled).  One block of 256 threads;
// *eps receives the value.
__global__ void __launch_bounds__(256) k_slip_converge(Phys ph, const PState s, const double *__restrict__ slip,
                                                       double *__restrict__ eps) {
    __shared__ double red[256];
    double            e = 0.0;
    if (ph.janus_prop == 2) {
        for (int n = threadIdx.x; n < ph.np; n += blockDim.x) {
            const double *sp = slip + (size_t)n * kSlipWords;
            double        dv = 0.0, dw = 0.0, nv = 0.0, nw = 0.0;
            for (int d = 0; d < 3; d++) {
                const double v = s.v[3 * n + d], w = s.omega[3 * n + d];
                nv += v * v;
                nw += w * w;
                dv += (sp[kSlipV + d] - v) * (sp[kSlipV + d] - v);
                dw += (sp[kSlipW + d] - w) * (sp[kSlipW + d] - w);
            }
            if (nv > kTolMP) dv /= nv;
            if (nw > kTolMP) dw /= nw;
            e = fmax(e, dv + dw);
        }
    }
    red[threadIdx.x] = e;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *eps = sqrt(red[0]);
}

}  // namespace spm
