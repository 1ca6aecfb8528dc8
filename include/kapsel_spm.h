/*
 * kapsel_spm.h -- C ABI of the B200 (sm_100a) smoothed-profile-method step.
 *
 * Drop-in boundary for KAPSEL's spectral SPM step (tsuyoshimaruyama/kapsel3).
 * Plain C types only: pointers, sizes, doubles.  Every entry point returns an
 * int status (SPM_OK = 0); on failure the context keeps its last good state
 * and spm_last_error() describes the failure.  The reference's own error
 * convention is exit_job(EXIT_FAILURE) (macro.h:178); the C++ shim that binds
 * the reference-named symbols turns a nonzero status into
 * exactly that.
 *
 * Field layout.  A k-space field is complex [NX][NY][NZ/2+1] stored as
 * interleaved doubles, i.e. the reference's in-place r2c array
 * double[NX*NY*NZ_], NZ_ = 2*(NZ/2+1) (input.cxx:444-445); a real-space field
 * uses the same array with data in z < NZ of each row.  Host-side entry points
 * (suffix _host) take such arrays in host memory, exactly as the reference's
 * functions receive them; device-resident state lives in the context.
 *
 * Particle record.  Host particle arrays are Np records of SPM_PARTICLE_WORDS
 * doubles laid out as
 *   x[3] x_nopbc[3] v[3] v_old[3] omega[3] omega_old[3] q[4] q_old[4]
 *   f_hydro[3] f_hydro_previous[3] torque_hydro[3] torque_hydro_previous[3]
 *   fr[3] fr_previous[3]
 * (the members of the reference's `Particle` that the step reads or writes,
 * variable.h:27-77; quaternions as (s, v0, v1, v2), quaternion.h:24-27).
 *
 * Threading: a context is used by one host thread at a time; different
 * contexts are independent (one GPU stream each).
 */
#ifndef KAPSEL_SPM_H
#define KAPSEL_SPM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPM_OK 0
#define SPM_ERR_ARG 1         /* invalid argument / unsupported size */
#define SPM_ERR_CUDA 2        /* CUDA runtime error (message in spm_last_error) */
#define SPM_ERR_NOMEM 3       /* device allocation failed */
#define SPM_ERR_DEVICE 4      /* kernel-reported error (particle left box, ...) */
#define SPM_ERR_NO_DEVICE 5   /* no CUDA device visible */

#define SPM_PARTICLE_WORDS 44

#define SPM_EQ_NAVIER_STOKES 0  /* constitutive_eq.type = Navier_Stokes */
#define SPM_EQ_LEES_EDWARDS 1   /* Shear_Navier_Stokes_Lees_Edwards */

#define SPM_PREC_FP64 0        /* every field and reduction in FP64 */
#define SPM_PREC_FP32_MIXED 1  /* fields/FFT/projection FP32, particle reductions and updates FP64 */

/* Physical and numerical parameters of one run: the UDF fields the step
 * reads (Gourmet_file_io, input.cxx:677-2556) and nothing derived.  Derived
 * globals (NU, IMASS, IMOI, TRN, WAVE, LJ_dia, ...) are computed inside, as
 * Set_global_parameters (input.cxx:425-604) does. */
typedef struct spm_params {
    int    npx, npy, npz;        /* mesh.NPX/Y/Z: N = 1 << NP (3 <= NP <= 9) */
    double dx, rho, eta, kbt;    /* constitutive_eq.<type>.DX, RHO, ETA, kBT */
    double alpha_v, alpha_o;     /* thermostat factors */
    int    equation;             /* SPM_EQ_* */
    double shear_rate;           /* Lees-Edwards DC shear rate (gradient along y) */
    int    n_particles;          /* Particle_spec[0].Particle_number (one species) */
    double mass_ratio;           /* Particle_spec[0].MASS_RATIO */
    double a, a_xi;              /* A, A_XI (radius and interface width / DX) */
    double epsilon;              /* EPSILON */
    int    lj_powers;            /* 0: 12:6, 1: 24:12, 2: 36:18 */
    int    lj_truncate;          /* 1: ON (repulsive), 0: OFF, -1: NONE */
    int    rotation;             /* switch.ROTATION */
    int    fix_cell[3];          /* switch.FIX_CELL.x/y/z */
    double dt;                   /* time_increment.manual.delta_t */
    double body_force[3];        /* constant force added to every particle's fr */
    int    precision;            /* SPM_PREC_* */
    unsigned int mt_seed;        /* MT19937 seed of the thermostat (reference: 0) */
} spm_params;

typedef struct spm_ctx spm_ctx;

/* ---- context ----------------------------------------------------------- */
const char *spm_last_error(void);
int spm_device_count(int *count);
/* Fills p with the reference's defaults for a Navier_Stokes run. */
int spm_params_default(spm_params *p);
/* Reads a UDF key file (lines "<udf.path> = <value>", the UDF paths of
 * Gourmet_file_io) into p; particle initial state goes to the optional
 * host record array (n_particles records, may be NULL). */
int spm_params_from_udf_keys(const char *path, spm_params *p, double *particles_out, int max_particles);
/* Allocates all device state for one run on the current device.
 * `stream` is a cudaStream_t (NULL: a new non-blocking stream). */
int spm_create(const spm_params *p, void *stream, spm_ctx **out);
int spm_destroy(spm_ctx *ctx);
/* Bytes of device memory one context with these parameters allocates. */
int spm_device_bytes(const spm_params *p, size_t *bytes);

/* ---- whole-run state ---------------------------------------------------- */
/* Uploads particle records and runs the reference's initialisation: zeta = 0
 * (Init_zeta_k, init_fluid.cxx:10-25), the initial rigidity projection and
 * uk_dc = 0 (sp_3d_ns.cxx:809-826).  Resets ts and time to 0. */
int spm_initialize(spm_ctx *ctx, const double *particles_host);
/* Runs n steps of Time_evolution_hydro (sp_3d_ns.cxx:41-194) or
 * Time_evolution_hydro_OBL (sp_3d_ns.cxx:328-433) on device-resident state.
 * Asynchronous on the context stream; errors raised by kernels surface at the
 * next synchronising call. */
int spm_step(spm_ctx *ctx, int nsteps);
int spm_synchronize(spm_ctx *ctx);
/* Copies state to / from host memory (blocking). */
int spm_get_particles(spm_ctx *ctx, double *particles_host);
int spm_set_particles(spm_ctx *ctx, const double *particles_host);
int spm_get_zeta(spm_ctx *ctx, double *zeta0, double *zeta1, double uk_dc[3]);
int spm_set_zeta(spm_ctx *ctx, const double *zeta0, const double *zeta1, const double uk_dc[3]);
/* Real-space velocity rebuilt from zeta (Zeta_k2u_k + U_k2u), three arrays
 * of NX*NY*NZ_ doubles. */
int spm_get_velocity(spm_ctx *ctx, double *u0, double *u1, double *u2);
/* phi = min(phi_sum, 1) of the current particle positions (NX*NY*NZ_). */
int spm_get_phi(spm_ctx *ctx, double *phi);
int spm_get_time(spm_ctx *ctx, int *ts, double *time);
/* Lees-Edwards bookkeeping: degree_oblique and the last step's shear-stress
 * line of Mean_shear_stress (sp_3d_ns.h:296-339): stress[0..7] =
 * {Shear_rate_eff, strain, lj, hydro_old, hydro_new, reynolds, fluid,
 * apparent}.  For a Lees-Edwards run spm_get_velocity returns the oblique
 * (contravariant) velocity on the sheared grid. */
int spm_get_shear_state(spm_ctx *ctx, double *degree_oblique, double stress[8]);

/* ---- reference solver boundaries (host arrays, reference layout) -------- */
/* NS_solver_slavedEuler (fluid_solver.h:77-82, fluid_solver.cxx:348-374):
 * zeta truncated and advanced by one slaved-Euler step in place. */
int spm_ns_solver_slaved_euler_host(spm_ctx *ctx, double *zeta0, double *zeta1, double uk_dc[3]);
/* Solenoidal_uk (operate_omega.h:72, operate_omega.cxx:171-195), in place on
 * three k-space fields. */
int spm_solenoidal_uk_host(spm_ctx *ctx, double *u0, double *u1, double *u2);
/* Zeta_k2u_k (fft_wrapper.h:162) and U_k2zeta_k (fft_wrapper.h:150). */
int spm_zeta_k2u_k_host(spm_ctx *ctx, const double *zeta0, const double *zeta1, const double uk_dc[3],
                        double *u0, double *u1, double *u2);
int spm_u_k2zeta_k_host(spm_ctx *ctx, const double *u0, const double *u1, const double *u2, double *zeta0,
                        double *zeta1, double uk_dc[3]);
/* A2a_k / A_k2a (fft_wrapper.h:641-681): in-place 3D real FFT of n fields. */
int spm_a2a_k_host(spm_ctx *ctx, double *a);
int spm_a_k2a_host(spm_ctx *ctx, double *a);
/* Make_phi_particle_sum (make_phi.h:50, make_phi.cxx:214-260): phi and
 * phi_sum of the given particle records. */
int spm_make_phi_particle_sum_host(spm_ctx *ctx, const double *particles_host, double *phi, double *phi_sum);
/* Make_u_particle_sum (make_phi.h:55, make_phi.cxx:313-354). */
int spm_make_u_particle_sum_host(spm_ctx *ctx, const double *particles_host, const double *phi_sum, double *up0,
                                 double *up1, double *up2);
/* Make_phi_u_particle (make_phi.h:70, make_phi.cxx:136-212): phi and
 * phi*v_p with the overlap normalisation. */
int spm_make_phi_u_particle_host(spm_ctx *ctx, const double *particles_host, double *phi, double *up0,
                                 double *up1, double *up2);
/* Make_f_particle_dt_sole (f_particle.h:60-67): f = P(up - phi u). */
int spm_make_f_particle_dt_sole_host(spm_ctx *ctx, const double *u0, const double *u1, const double *u2,
                                     const double *up0, const double *up1, const double *up2, const double *phi,
                                     double *f0, double *f1, double *f2);
/* Calc_f_hydro_correct_precision (md_force.h:53, md_force.cxx:383-506):
 * writes f_hydro / torque_hydro into the particle records. */
int spm_calc_f_hydro_correct_precision_host(spm_ctx *ctx, double *particles_host, const double *phi_sum,
                                            const double *u0, const double *u1, const double *u2);
/* Calc_f_Lennard_Jones (md_force.h:78-81): adds LJ forces to fr of the
 * particle records (cell-list pair multiplicity of the reference). */
int spm_calc_f_lennard_jones_host(spm_ctx *ctx, double *particles_host);

/* Allocation-free Make_f_particle_dt_sole on caller-owned DEVICE buffers.
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc (their device memory comes from their own pool or another
 * runtime, or their steady-state loop must stay free of allocator calls).
 * All ten pointers are device arrays in the reference layout
 * (double[NX*NY*NZ_]); the result f = P(up - min(phi,1) u) is written to
 * f0..f2.  FP64 only; grids of 8..64 points per axis (npx/npy/npz in 3..6),
 * larger grids are rejected with SPM_ERR_ARG.  Working memory is one
 * file-scope device array of about 6.5 MB that every GPU loading this
 * library keeps until the process exits; the first call on a device looks
 * up its address (make that call before any stream capture).  Every call
 * shares that array: calls that overlap on the GPU race.  `stream` is a
 * cudaStream_t (NULL: the legacy default stream). */
int spm_make_f_particle_dt_sole_noalloc(const double *u0, const double *u1, const double *u2, const double *up0,
                                        const double *up1, const double *up2, const double *phi, double *f0,
                                        double *f1, double *f2, int npx, int npy, int npz, void *stream);

/* ---- 3D FFT on device buffers ------------------------------------------- */
/* In-place transforms of nfields device fields of the context's precision,
 * consecutive fields `field_stride` complex elements apart. */
int spm_fft_forward_dev(spm_ctx *ctx, void *data, int nfields, size_t field_stride);
int spm_fft_inverse_dev(spm_ctx *ctx, void *data, int nfields, size_t field_stride);
/* Complex elements per allocated field row (NZ/2+1 for FP64; FP32 rows may
 * carry one extra complex of padding). */
int spm_row_complex(spm_ctx *ctx, int *hnzp);

/* ---- measurement -------------------------------------------------------- */
/* Times n steps with CUDA events on the context stream (ms total). */
int spm_time_steps(spm_ctx *ctx, int nsteps, float *ms);
/* Runs n steps with CUDA events around every strided (Y/X) FFT pass, the
 * dominant kernel; returns its average duration (us), algorithmic bytes per
 * launch (one read + one write of every transformed element) and count. */
int spm_profile_pass(spm_ctx *ctx, int nsteps, double *avg_us, double *bytes_per_launch, long long *count);
/* Launches of this library's kernels since the last reset. */
int spm_kernel_launches(spm_ctx *ctx, long long *count, int reset);

#ifdef __cplusplus
}
#endif
#endif /* KAPSEL_SPM_H */
