/*
 * kapsel_spm.h -- C ABI of the B200 (sm_100a) smoothed-profile-method step.
 *
 * Drop-in boundary for KAPSEL's spectral SPM step (tsuyoshimaruyama/kapsel3).
 * Plain C types only: pointers, sizes, doubles.  Every entry point returns an
 * int status (SPM_OK = 0); on failure the context keeps its last good state
 * and spm_last_error() describes the failure.  The reference's own error
 * convention is exit_job(EXIT_FAILURE) (macro.h:178); the C++ shim that binds
 * the reference-named symbols (kapsel3_b200/shim) turns a nonzero status into
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
/* Per rigid body: xGs[3], xGs without the periodic wrap[3], velocityGs[3],
 * omegaGs[3] (space frame), Rigid_Masses, the diagonal of Rigid_Moments_body[3] */
#define SPM_RIGID_WORDS 16
/* The whole state of a rigid body (spm_get_rigid_state): xGs, xGs_nopbc,
 * xGs_previous, velocityGs, velocityGs_old, omegaGs, omegaGs_old, forceGs,
 * forceGrs, torqueGs, torqueGrs, forceGs_previous, forceGrs_previous,
 * torqueGs_previous, torqueGrs_previous (3 each, space frame), then
 * Rigid_Moments and Rigid_IMoments (9 each, row-major). */
#define SPM_RIGID_STATE_WORDS 63

#define SPM_EQ_NAVIER_STOKES 0  /* constitutive_eq.type = Navier_Stokes */
#define SPM_EQ_LEES_EDWARDS 1   /* Shear_Navier_Stokes_Lees_Edwards */
#define SPM_EQ_ELECTROLYTE 2    /* Electrolyte: charged colloids with mobile ions */
#define SPM_EQ_SHEAR_NAVIER_STOKES 3 /* Shear_Navier_Stokes: periodic box, mean shear sustained on fluid planes */

/* Particle_spec[0].janus_propulsion (input.cxx:1427-1441) and janus_axis (1410-1425) */
#define SPM_JANUS_OFF 0       /* "OFF": passive colloids */
#define SPM_JANUS_TUMBLER 1   /* "TUMBLER": body-frame self force / torque */
#define SPM_JANUS_SQUIRMER 2  /* "SQUIRMER": surface slip velocity, self-consistent slip iteration */
#define SPM_JANUS_OBSTACLE 3  /* "OBSTACLE": fixed particles */
#define SPM_AXIS_NONE 0
#define SPM_AXIS_X 1
#define SPM_AXIS_Y 2
#define SPM_AXIS_Z 3

#define SPM_MAX_SPECIES 4  /* particle species (Particle_spec[0..3]) */

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
    /* Electrolyte (constitutive_eq.Electrolyte, input.cxx:834-930; read when
     * equation == SPM_EQ_ELECTROLYTE) */
    double dielectric;           /* Dielectric_cst */
    int    salt;                 /* Add_salt: 0 saltfree (one counterion species), 1 salt (two species) */
    int    init_pb;              /* INIT_profile: 0 Uniform, 1 Poisson_Boltzmann */
    double valency[2];           /* saltfree: Valency_counterion; salt: positive, negative ion */
    double onsager[2];           /* Onsager coefficients in the same order */
    double debye_length;         /* salt: Debye_length */
    double surface_charge;       /* Particle_spec[0].Surface_charge */
    int    e_field;              /* Electric_field: 0 OFF, 1 DC, 2 AC */
    double e_ext[3];             /* Ex, Ey, Ez */
    double e_frequency;          /* AC: Frequency */
    /* Janus particles (Particle_spec[0].janus_*, input.cxx:1403-1470): tumblers and squirmers in
     * Navier_Stokes and Shear_Navier_Stokes runs, obstacles with every equation (input.cxx:1509-1512) */
    int    janus_axis;           /* SPM_AXIS_*: the body axis e3 of the slip profile */
    int    janus_propulsion;     /* SPM_JANUS_* */
    double janus_force[3];       /* TUMBLER: janus_force, body frame */
    double janus_torque[3];      /* TUMBLER: janus_torque, body frame */
    double slip_vel;             /* SQUIRMER: janus_slip_vel (B1) */
    double slip_mode;            /* SQUIRMER: janus_slip_mode (alpha = B2/B1) */
    double rotlet_c1;            /* SQUIRMER: janus_rotlet_C1 */
    double rotlet_c2;            /* SQUIRMER: janus_rotlet_dipole_C2 */
    double slip_tol;             /* switch.SLIP_tol */
    int    slip_iter;            /* switch.SLIP_iter */
    /* Several particle species (Particle_spec[0..n_species-1], input.cxx:1403-1441).  n_species <= 1:
     * one species, described by n_particles, mass_ratio and surface_charge above.  n_species > 1: the
     * n_particles records are consecutive blocks of species_count[s] particles, species 0 first (the
     * reference's p[n].spec order); each species has its own MASS_RATIO and Surface_charge, all share
     * A, A_XI and the janus settings (which must be OFF). */
    int    n_species;
    int    species_count[SPM_MAX_SPECIES];
    double species_mass_ratio[SPM_MAX_SPECIES];
    double species_surface_charge[SPM_MAX_SPECIES];
    /* Shear_Navier_Stokes (constitutive_eq.Shear_Navier_Stokes.External_field, input.cxx:770-793): the
     * shear rate is shear_rate above; shear_ac = 0 DC, 1 AC with angular frequency shear_frequency */
    int    shear_ac;
    double shear_frequency;
    /* Rigid bodies of spherical beads (object_type.type = rigid, object_type.rigid.Rigid_spec[s],
     * input.cxx:1583-1700, 2468-2550; rigid.h).  rigid = 1: species s (n_species of them, one when
     * n_species <= 1) holds rigid_count[s] bodies (Chain_number) of rigid_beads[s] beads
     * (Beads_number); the n_particles records list the beads body after body, species 0 first, with
     * coordinates as given (no periodic wrap, as the reference reads them).  The beads' MASS_RATIO is
     * species_mass_ratio[s] (mass_ratio for one species).  rigid_free[s] = vx vy vz wx wy wz degrees
     * of freedom, 1 free, 0 fixed (Rigid_motion "free" / "fix", switch.free_rigid); rigid_velocity[s]
     * and rigid_omega[s] are the initial body velocity and body-frame angular velocity
     * (Rigid_velocity, Rigid_omega).  Navier_Stokes runs with ROTATION ON, lone contexts (no pool). */
    int    rigid;
    int    rigid_beads[SPM_MAX_SPECIES];
    int    rigid_count[SPM_MAX_SPECIES];
    int    rigid_free[SPM_MAX_SPECIES][6];
    double rigid_velocity[SPM_MAX_SPECIES][3];
    double rigid_omega[SPM_MAX_SPECIES][3];
    /* gravity.G along gravity.G_direction for rigid bodies: each body feels -G RHO V (MASS_RATIO - 1)
     * along that axis, V its mass over its density (Add_f_gravity, md_force.cxx:317-322) */
    double rigid_gravity[3];
} spm_params;

typedef struct spm_ctx spm_ctx;
typedef struct spm_pool spm_pool;

/* ---- context ----------------------------------------------------------- */
const char *spm_last_error(void);
int spm_device_count(int *count);
/* sizeof(spm_params) in the library.  A binding compiled against another
 * version of this header compares it with its own sizeof(spm_params) and
 * refuses to run on a mismatch (the struct grows at its end). */
size_t spm_params_size(void);
/* Fills p with the reference's defaults for a Navier_Stokes run. */
int spm_params_default(spm_params *p);
/* Reads a UDF key file (lines "<udf.path> = <value>", the UDF paths of
 * Gourmet_file_io) into p; particle initial state goes to the optional
 * host record array (n_particles records, may be NULL). */
int spm_params_from_udf_keys(const char *path, spm_params *p, double *particles_out, int max_particles);
/* Reads a UDF input file in the OCTA UDF format the reference reads
 * through UDFManager (Gourmet_file_io, input.cxx:677-2556): the schema from
 * its \begin{def}/\begin{global_def} blocks and \include'd files (the
 * reference's define.udf), the values from its \begin{data} block.  Same
 * parameters, particle records and errors as spm_params_from_udf_keys. */
int spm_params_from_udf(const char *path, spm_params *p, double *particles_out, int max_particles);
/* The \begin{data} values of a UDF file flattened to "<udf.path>=<value>\n"
 * lines (paths as the reference's Location strings name them, e.g.
 * "object_type.spherical_particle.Particle_spec[0].Particle_number").
 * *needed receives the text size including the terminating NUL; out is
 * filled only when capacity >= *needed (out may be NULL to query). */
int spm_udf_read_keys(const char *path, char *out, size_t capacity, size_t *needed);
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
 * next synchronising call.  Navier_Stokes steps, and Electrolyte steps after
 * the first, replay a CUDA graph of the step captured on first use (the
 * environment variable SPM_NO_GRAPH=1 at spm_create keeps direct launches). */
int spm_step(spm_ctx *ctx, int nsteps);
int spm_synchronize(spm_ctx *ctx);
/* Copies state to / from host memory (blocking). */
int spm_get_particles(spm_ctx *ctx, double *particles_host);
/* Rigid bodies of a run (SW_PT == rigid): their number, and their state
 * (SPM_RIGID_WORDS doubles per body; synchronising). */
int spm_rigid_count(spm_ctx *ctx, int *n);
int spm_get_rigid(spm_ctx *ctx, double *bodies);
/* The whole rigid state (SPM_RIGID_STATE_WORDS doubles per body) and every
 * bead's offset from its body's centre (6 doubles per bead: GRvecs, then
 * GRvecs_body), to and from host memory (synchronising).  A host that keeps
 * the reference's rigid globals (rigid.h; the resident time evolution)
 * reads them back for its output frames and restart file, and hands over a
 * state it set itself after spm_initialize. */
int spm_get_rigid_state(spm_ctx *ctx, double *bodies, double *offsets);
int spm_set_rigid_state(spm_ctx *ctx, const double *bodies, const double *offsets);
int spm_set_particles(spm_ctx *ctx, const double *particles_host);
int spm_get_zeta(spm_ctx *ctx, double *zeta0, double *zeta1, double uk_dc[3]);
int spm_set_zeta(spm_ctx *ctx, const double *zeta0, const double *zeta1, const double uk_dc[3]);
/* Real-space velocity rebuilt from zeta (Zeta_k2u_k + U_k2u), three arrays
 * of NX*NY*NZ_ doubles. */
int spm_get_velocity(spm_ctx *ctx, double *u0, double *u1, double *u2);
/* phi = min(phi_sum, 1) of the current particle positions (NX*NY*NZ_). */
int spm_get_phi(spm_ctx *ctx, double *phi);
int spm_get_time(spm_ctx *ctx, int *ts, double *time);
/* Sets the completed-step count, the time and (Lees-Edwards) degree_oblique,
 * as Force_restore_parameters restores jikan and degree_oblique
 * (resume.cxx:555-570) after the state was uploaded with spm_set_zeta and
 * spm_set_particles.  The step counter selects Euler (0) or Adams-Bashforth. */
int spm_set_time(spm_ctx *ctx, int ts, double time, double degree_oblique);
/* Lees-Edwards bookkeeping: degree_oblique and the last step's shear-stress
 * line of Mean_shear_stress (sp_3d_ns.h:296-339): stress[0..7] =
 * {Shear_rate_eff, strain, lj, hydro_old, hydro_new, reynolds, fluid,
 * apparent}.  For a Lees-Edwards run spm_get_velocity returns the oblique
 * (contravariant) velocity on the sheared grid.  A Shear_Navier_Stokes run
 * gives its line (Update_strain, sp_3d_ns.h:205-214; Mean_shear_stress,
 * :319-340): degree_oblique = 0, stress[0..5] = {the instantaneous shear
 * rate, the strain since initialisation, the shear stress -stress_yx, the
 * viscosity -stress_yx / rate, the inertia stress (AC), -stress_yx + inertia
 * (AC)}. */
int spm_get_shear_state(spm_ctx *ctx, double *degree_oblique, double stress[8]);
/* Electrolyte runs: the k-space concentration of ion species `species`
 * (0: the counterion of a saltfree run or the positive ion; 1: the negative
 * ion of a salt run), in the reference's r2c layout (Concentration[n]). */
int spm_get_concentration(spm_ctx *ctx, int species, double *conc_k);
/* Electrolyte runs: sets the k-space concentration of ion species `species`
 * (the reference's Concentration[n], r2c layout) and its Total_solute, the
 * amount Rescale_solute keeps outside the particles (solute_rhs.cxx:91-116;
 * Count_solute_each of the initial profile, solute_rhs.h:124-137): the state
 * a host that initialised the ions itself hands over. */
int spm_set_solute(spm_ctx *ctx, int species, const double *conc_k, double total_solute);
/* Checkpoint / restart (the reference's restart files, resume.cxx:10-74,
 * 381-588): writes, or reads back into a context created with the same
 * parameters, every piece of device state the next steps read (zeta with its
 * FP32 compensation words, uk_dc, the step counter, the particle buffer, the
 * MT19937 state, Lees-Edwards scalars) plus ts, time and degree_oblique, so
 * a restored run continues as the saved one would have.  The file format is
 * this library's own (binary, host byte order). */
int spm_save_state(spm_ctx *ctx, const char *path);
int spm_load_state(spm_ctx *ctx, const char *path);
/* The reference's own restart files, so that a run moves between the
 * reference program and this library in both directions.
 * spm_load_restart = Force_restore_parameters (resume.cxx:507-588): reads the
 * section resume.CONTINUE.Saved_Data of a restart file (a UDF file, or a key
 * file of "udf.path = value" lines) into an initialised context: zeta of every
 * mode, uk_dc, the particles (orientations normalised as Read_Particle_udf
 * does, :757-869), jikan and degree_oblique, and an Electrolyte run's k-space
 * concentrations.  The file's jikan.ts is the reference's index of the step
 * just completed; the context then counts jikan.ts + 1 steps.  The reference's
 * resumed program takes one step of its initial state before it restores (the
 * first pass of its main loop, sp_3d_ns.cxx:856-1005), which advances its
 * thermostat's generator; a caller that must follow it exactly does the same
 * (kapsel3_b200.spm.resume_run).
 * spm_save_restart = Save_Restart_udf (resume.cxx:10-74, 381-506): writes a key
 * file with the keys of input_path (the run's input, UDF or key file; NULL for
 * the resume section alone), resume.Calculation = CONTINUE and the section
 * above for the context's state.  In a rigid run Particles[] holds the bodies,
 * followed by GR_body, GR_masses and GR_moments_body (resume.cxx:253-379,
 * 925-1100); loading it needs the bodies' layout of spm_initialize.
 * Squirmers are refused. */
int spm_load_restart(spm_ctx *ctx, const char *path);
/* Per-frame particle records of the reference's UDF output (output.UDF = ON;
 * Output_udf, output.cxx:268-375): spm_udf_out_record appends one record of
 * the context's current state (E, t = the completed steps, and per particle
 * R, R_raw, v, q, omega and the previous step's f_hydro, torque_hydro, f_r,
 * torque_r, f_slip, torque_slip; rigid runs add RigidParticles[]) to the file
 * opened by spm_udf_out_open, as "record[<n>].<udf.path> = <value>" lines. */
int spm_udf_out_open(spm_ctx *ctx, const char *path);
int spm_udf_out_record(spm_ctx *ctx);
int spm_udf_out_close(spm_ctx *ctx);
int spm_save_restart(spm_ctx *ctx, const char *input_path, const char *path);
/* ---- output in the reference's legacy AVS format -----------------------
 * (output.AVS = ON, FileType = BINARY; Init_avs / Output_avs,
 * avs_output.cxx:45-143, 261-285; Init_avs_p / Output_avs_p,
 * avs_output_p.cxx; frame content of Output_field_data, output.cxx:129-191).
 * spm_avs_open writes <out_dir>/<out_name>.fld, <out_name>.cod and, with
 * particles, <out_name>p.fld, and creates <out_dir>/avs.  spm_avs_frame
 * writes the frame of the run's current (ts, time): avs/<out_name>_<ts>.dat
 * (ux uy uz phi pressure tau_xy tau_yz tau_zx tau_xx tau_yy as float, x
 * fastest) and avs/<out_name>p_<ts>.cod / .dat, appending the frame's
 * description to the .fld files.  It returns once the frame is enqueued on
 * the run's stream: the copy to host memory and the file writes overlap the
 * following steps.  spm_avs_flush waits until every enqueued frame is on
 * disk and reports the first write error; spm_avs_close flushes and releases
 * the staging buffers (spm_destroy does too).  Navier_Stokes runs only (not
 * Lees-Edwards, not pooled runs). */
int spm_avs_open(spm_ctx *ctx, const char *out_dir, const char *out_name, int num_snap);
int spm_avs_frame(spm_ctx *ctx);
int spm_avs_flush(spm_ctx *ctx);
int spm_avs_close(spm_ctx *ctx);

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
 * up its address and uploads the transform tables of every supported size
 * into it (make that call before any stream capture); later calls only
 * enqueue kernels and memsets on `stream` and return without waiting.  The
 * transforms have no device-side waits, so there is no device error to
 * report.  Every call shares that array: calls that overlap on the GPU
 * race.  `stream` is a cudaStream_t (NULL: the legacy default stream). */
int spm_make_f_particle_dt_sole_noalloc(const double *u0, const double *u1, const double *u2, const double *up0,
                                        const double *up1, const double *up2, const double *phi, double *f0,
                                        double *f1, double *f2, int npx, int npy, int npz, void *stream);

/* ---- 3D FFT on device buffers ------------------------------------------- */
/* In-place transforms of nfields device fields of the context's precision,
 * consecutive fields `field_stride` complex elements apart.  `data` and the
 * field stride in bytes must be multiples of 16 (SPM_ERR_ARG otherwise). */
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
/* Runs n steps (direct launches) with CUDA events around every launch of the
 * step's transform, k-space and stencil kernels on the stream it runs on, and
 * writes a JSON summary to json[cap]: per kernel family its launches, total
 * and per-launch device time (us) and algorithmic bytes per launch, plus the
 * device time of the n steps. */
int spm_profile_kernels(spm_ctx *ctx, int nsteps, char *json, size_t cap);
/* Launches of this library's kernels since the last reset. */
int spm_kernel_launches(spm_ctx *ctx, long long *count, int reset);

/* ---- serving pool (no reference counterpart) ----------------------------
 * A pool holds independent Navier_Stokes runs of one grid size, DX and
 * precision.  Their fields share one slot-major device arena so each FFT
 * stage and each k-space pointwise kernel of a pool step is one launch over
 * all runs; particle kernels run per run on the pool's stream.  The pool step
 * can be replayed from a CUDA graph captured once per membership.  A run of
 * a pool is an spm_ctx: the whole-run getters above work on it (between
 * steps); spm_destroy refuses it (use spm_pool_release).  Releasing a run
 * moves the pool's last run into its slot; run handles stay valid. */
/* Device bytes of a pool arena of `capacity` runs of this grid, and of the
 * per-run particle buffers for grid->n_particles particles. */
int spm_pool_device_bytes(const spm_params *grid, int capacity, size_t *arena_bytes, size_t *run_bytes);
/* `stream`: cudaStream_t of the pool (NULL: a new non-blocking stream). */
int spm_pool_create(const spm_params *grid, int capacity, void *stream, spm_pool **out);
int spm_pool_destroy(spm_pool *pool);
/* Adds a run and runs its initialisation (as spm_initialize).  The pool
 * doubles its arena when full. */
int spm_pool_admit(spm_pool *pool, const spm_params *p, const double *particles_host, spm_ctx **run);
int spm_pool_release(spm_pool *pool, spm_ctx *run);
int spm_pool_size(spm_pool *pool, int *runs, int *capacity);
int spm_pool_run(spm_pool *pool, int index, spm_ctx **run);
int spm_pool_stream(spm_pool *pool, void **stream);
/* Enqueues nsteps steps of every run (asynchronous); use_graph != 0 replays
 * a graph of the step captured for the current membership. */
int spm_pool_step(spm_pool *pool, int nsteps, int use_graph);
/* done = 1 when the steps enqueued last have finished. */
int spm_pool_query(spm_pool *pool, int *done);
/* Waits for the pool; last_ms = device time of the last spm_pool_step call;
 * errors[r] (optional, one per run slot) = run r's device error bits. */
int spm_pool_synchronize(spm_pool *pool, float *last_ms, unsigned int *errors);
int spm_pool_stats(spm_pool *pool, long long *graph_kernels, int *captures);
/* Host-side fault injection: the next `count` device allocations of contexts
 * and pools fail with SPM_ERR_NOMEM (0 switches it off). */
int spm_debug_fail_allocations(int count);
/* Bound of every device-side wait of the context's TMA transform passes, in
 * seconds of the GPU's global timer (default 1 s, at most 60).  A wait that
 * runs out sets the device error bit that the next synchronising call reports
 * as SPM_ERR_DEVICE ("TMA pipeline wait timed out"); the pass stops and the
 * context stays usable.  No reference counterpart. */
int spm_set_wait_limit(spm_ctx *ctx, double seconds);
/* Test switch for the bounded waits: the context's next `launches` TMA
 * transform passes issue no tile loads, so their first waits run out with
 * nothing in flight (0 switches it off).  The steps taken meanwhile run
 * without graph replay.  No reference counterpart. */
int spm_debug_skip_tma_loads(spm_ctx *ctx, int launches);
/* Device memory of contexts and pools comes from a stream-ordered memory pool
 * per device that keeps freed blocks mapped for reuse, because cudaFree waits
 * for the whole device and unmaps (up to 0.8 s for a pool arena on B200).
 * This returns the unused part to the driver; bytes = what was held unused. */
int spm_release_cached_memory(size_t *bytes);

/* ---- serving loop (no reference counterpart) -----------------------------
 * A persistent worker thread admits submitted Navier_Stokes runs by device-
 * memory budget into per-grid pools, steps every pool continuously (pools of
 * different grids on their own streams, overlapping on the GPU), retires runs
 * at their step count and records per-step latency: for every run step, the
 * host time between the completion of the run's previous step (or its
 * admission) and this one. */
#define SPM_REQ_QUEUED 0
#define SPM_REQ_RUNNING 1
#define SPM_REQ_DONE 2
#define SPM_REQ_FAILED 3
#define SPM_REQ_CANCELLED 4
#define SPM_REQ_KEEP_VELOCITY 1 /* submit flag: keep the final velocity field */

typedef struct spm_server spm_server;
typedef struct spm_server_config {
    size_t budget_bytes;        /* device bytes the server may hold (pools + runs) */
    int    pool_initial_capacity; /* run slots of a new pool's arena */
    int    use_graph;           /* replay each pool step from a captured CUDA graph */
    int    steps_per_launch;    /* steps enqueued per pool launch (1: per-step latency) */
    int    poll_us;             /* worker sleep when nothing progressed */
    int    device;              /* CUDA device index */
    double pool_idle_s;         /* an empty pool keeps its arena this long, unless a request waits */
} spm_server_config;
typedef struct spm_server_stats {
    long long submitted, rejected, admitted, completed, failed, cancelled, queued;
    long long run_steps;        /* steps summed over runs */
    long long graph_captures;
    int       max_active;       /* most runs resident at once */
    size_t    used_bytes, peak_bytes;
    double    busy_s;           /* first admission to last retirement */
    double    step_latency_p50_ms, step_latency_p99_ms, step_latency_max_ms;
    double    pool_step_device_p50_ms, pool_step_device_p99_ms;
    /* longest single host phase of the worker (ms): creating a pool, admitting
     * one run into a pool (arena growth and the run's initialisation included),
     * destroying a pool, launching one pool step (graph capture included when
     * the pool's membership changed), accounting one finished pool step
     * (result downloads included).  While the worker is in one of these, no
     * other pool's finished step is accounted, so they bound step latency. */
    double    pool_create_max_ms, admit_max_ms, pool_destroy_max_ms, launch_max_ms, finish_max_ms;
} spm_server_stats;

int spm_server_config_default(spm_server_config *cfg);
int spm_server_create(const spm_server_config *cfg, spm_server **out);
/* Stops the worker: cancels queued and running requests, frees all pools. */
int spm_server_destroy(spm_server *server);
/* Queues a run of nsteps steps (particle records as spm_initialize).
 * Rejected at once (nonzero status): bad parameters, Lees-Edwards runs,
 * particles outside the box, or a run larger than the whole budget. */
int spm_server_submit(spm_server *server, const spm_params *p, const double *particles_host, int nsteps, int flags,
                      long long *request_id);
int spm_server_cancel(spm_server *server, long long request_id);
/* Waits until the request is DONE, FAILED or CANCELLED (timeout_s < 0:
 * no limit); state = its state on return. */
int spm_server_wait(spm_server *server, long long request_id, double timeout_s, int *state);
int spm_server_status(spm_server *server, long long request_id, int *state, int *status, int *steps_done,
                      char *message, size_t message_len);
/* Final particle records, optional velocity (SPM_REQ_KEEP_VELOCITY), time,
 * and submission-to-completion latency of a DONE request. */
int spm_server_result(spm_server *server, long long request_id, double *particles_host, double *u0, double *u1,
                      double *u2, double *time, double *latency_s);
int spm_server_forget(spm_server *server, long long request_id);
int spm_server_get_stats(spm_server *server, spm_server_stats *stats);
/* Per-step latency samples in ms (up to cap; n = number recorded). */
int spm_server_latencies(spm_server *server, float *out, size_t cap, size_t *n);

#ifdef __cplusplus
}
#endif
#endif /* KAPSEL_SPM_H */
