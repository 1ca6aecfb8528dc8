// Device-resident time evolution inside the unmodified KAPSEL program.
//
// The reference's main loop advances the run through the function pointer
// Time_evolution (sp_3d_ns.cxx:10, set to Time_evolution_hydro or
// Time_evolution_hydro_OBL at sp_3d_ns.cxx:690-707, called at :954).  Once
// the reference has finished its own initialisation (the initial projection,
// sp_3d_ns.cxx:809-826), kapsel_b200_go_resident() points it at
// resident_time_evolution below, which keeps zeta, uk_dc and the particles on
// the GPU and advances them with spm_step.  The host copies are refreshed only
// where the main loop reads them: before an output frame (ts % GTS == 0,
// sp_3d_ns.cxx:863-874) and before the restart file written after the last
// step (sp_3d_ns.cxx:974-982).
//
// Served: Navier_Stokes, Shear_Navier_Stokes, Shear_Navier_Stokes_Lees_
// Edwards and Electrolyte runs of spherical particles (several species, or
// Janus particles of one species) and rigid bodies, new or resumed; an
// Electrolyte run hands over its ion concentrations and Total_solute with the
// rest, and gets the concentrations back at frames (Output_charge_field_data,
// Electrolyte_free_energy) and for its restart file; a rigid run hands over
// and gets back its bodies' state (the rigid.h globals: xGs, velocityGs,
// omegaGs, their forces and torques, Rigid_Moments, GRvecs) the same way.  A resumed run's first pass of the main loop
// steps its input state and then restores the saved one on the host
// (sp_3d_ns.cxx:856-1005); the next call uploads the restored state and its
// time, the generator keeping the draws of that first step as the
// reference's does.  For any other run the pointer is left alone and the
// reference steps on the CPU.  In a sheared run the main loop's per-step
// stress print (Update_strain, Mean_shear_stress, sp_3d_ns.h:205-339) reads
// CPU-side arrays this path updates only at frames; spm_get_shear_state
// returns that line from the device.
#include <vector>

#include "kapsel_b200_common.h"

extern void (*Time_evolution)(double **zeta, double uk_dc[DIM], double **f, Particle *p, CTime &jikan);
extern double  *phi;
extern double **Concentration;  // solute_rhs.cxx:16
extern double  *Total_solute;   // solute_rhs.h:17

namespace {

using kapsel_b200::check;

spm_ctx            *g_run = nullptr;
int                 g_eq  = SPM_EQ_NAVIER_STOKES;
std::vector<double> g_rec;
bool                g_restored = false;
double              g_body_force[3] = {0.0, 0.0, 0.0};

void rigid_globals(bool to_globals);

// Host copies of the state the main loop reads: zeta, uk_dc, the particles,
// phi (output frames) and, for Lees-Edwards, degree_oblique.
void download(double **zeta, double uk_dc[DIM], Particle *p) {
    check(spm_get_zeta(g_run, zeta[0], zeta[1], uk_dc), "spm_get_zeta");
    g_rec.assign((size_t)Particle_Number * SPM_PARTICLE_WORDS, 0.0);
    check(spm_get_particles(g_run, g_rec.data()), "spm_get_particles");
    kapsel_b200::unpack_records(g_rec.data(), p);
    if (phi) check(spm_get_phi(g_run, phi), "spm_get_phi");
    if (g_eq == SPM_EQ_ELECTROLYTE)
        for (int n = 0; n < N_spec; n++) check(spm_get_concentration(g_run, n, Concentration[n]), "spm_get_concentration");
    rigid_globals(true);
    if (g_eq == SPM_EQ_LEES_EDWARDS) {
        double stress[8];
        check(spm_get_shear_state(g_run, &degree_oblique, stress), "spm_get_shear_state");
    }
}

// Rigid bodies: the body state in the reference's rigid globals <->
// SPM_RIGID_STATE_WORDS per body and the beads' offsets.
std::vector<double> g_bodies, g_offsets;
void rigid_globals(bool to_globals) {
    if (SW_PT != rigid) return;
    double **vec[15] = {xGs,      xGs_nopbc, xGs_previous, velocityGs, velocityGs_old,    omegaGs,           omegaGs_old,
                        forceGs,  forceGrs,  torqueGs,     torqueGrs,  forceGs_previous,  forceGrs_previous, torqueGs_previous,
                        torqueGrs_previous};
    const int W = SPM_RIGID_STATE_WORDS;
    g_bodies.resize((size_t)Rigid_Number * W);
    g_offsets.resize((size_t)Particle_Number * 6);
    if (to_globals) check(spm_get_rigid_state(g_run, g_bodies.data(), g_offsets.data()), "spm_get_rigid_state");
    for (int b = 0; b < Rigid_Number; b++) {
        double *o = g_bodies.data() + (size_t)b * W;
        for (int v = 0; v < 15; v++)
            for (int d = 0; d < DIM; d++) {
                if (to_globals) vec[v][b][d] = o[3 * v + d];
                else o[3 * v + d] = vec[v][b][d];
            }
        for (int i = 0; i < DIM; i++)
            for (int j = 0; j < DIM; j++) {
                if (to_globals) {
                    Rigid_Moments[b][i][j]  = o[45 + 3 * i + j];
                    Rigid_IMoments[b][i][j] = o[54 + 3 * i + j];
                } else {
                    o[45 + 3 * i + j] = Rigid_Moments[b][i][j];
                    o[54 + 3 * i + j] = Rigid_IMoments[b][i][j];
                }
            }
    }
    for (int n = 0; n < Particle_Number; n++)
        for (int d = 0; d < DIM; d++) {
            if (to_globals) {
                GRvecs[n][d]      = g_offsets[(size_t)n * 6 + d];
                GRvecs_body[n][d] = g_offsets[(size_t)n * 6 + 3 + d];
            } else {
                g_offsets[(size_t)n * 6 + d]     = GRvecs[n][d];
                g_offsets[(size_t)n * 6 + 3 + d] = GRvecs_body[n][d];
            }
        }
    if (!to_globals) check(spm_set_rigid_state(g_run, g_bodies.data(), g_offsets.data()), "spm_set_rigid_state");
}

// Electrolyte: the ions as the reference initialised (or restored) them
void upload_solute() {
    if (g_eq != SPM_EQ_ELECTROLYTE) return;
    for (int n = 0; n < N_spec; n++)
        check(spm_set_solute(g_run, n, Concentration[n], Total_solute[n]), "spm_set_solute");
}

void resident_time_evolution(double **zeta, double uk_dc[DIM], double **f, Particle *p, CTime &jikan) {
    (void)f;
    if (g_run && RESUMED && !g_restored && jikan.ts == last_ts + 1) {  // the state Force_restore_parameters set
        check(spm_set_zeta(g_run, zeta[0], zeta[1], uk_dc), "spm_set_zeta");
        check(spm_set_particles(g_run, kapsel_b200::records(p, g_rec)), "spm_set_particles");
        upload_solute();
        rigid_globals(false);
        check(spm_set_time(g_run, jikan.ts, jikan.time, degree_oblique), "spm_set_time");
        g_restored = true;
    }
    if (!g_run) {  // the reference's state after its initial projection
        spm_params prm = kapsel_b200::params_from_globals(g_eq);
        // a body force set by the host replaces gravity, as it does on the CPU
        if (g_body_force[0] != 0.0 || g_body_force[1] != 0.0 || g_body_force[2] != 0.0)
            for (int d = 0; d < DIM; d++) prm.body_force[d] = g_body_force[d];
        check(spm_create(&prm, nullptr, &g_run), "spm_create");
        if (SW_PT == rigid) {
            // the bodies' layout, masses and frames from the beads' unwrapped
            // positions, as Init_Particle's rigid branch builds them; the
            // reference's own body state is handed over below
            kapsel_b200::records(p, g_rec);
            for (int n = 0; n < Particle_Number; n++)
                for (int d = 0; d < DIM; d++)
                    g_rec[(size_t)n * SPM_PARTICLE_WORDS + d] = g_rec[(size_t)n * SPM_PARTICLE_WORDS + 3 + d];
            check(spm_initialize(g_run, g_rec.data()), "spm_initialize");
        }
        check(spm_set_zeta(g_run, zeta[0], zeta[1], uk_dc), "spm_set_zeta");
        check(spm_set_particles(g_run, kapsel_b200::records(p, g_rec)), "spm_set_particles");
        upload_solute();
        rigid_globals(false);
    }
    if (jikan.dt_fluid != DT) {
        fprintf(stderr, "kapsel_b200: dt changed during the run (%g != %g)\n", jikan.dt_fluid, DT);
        exit_job(EXIT_FAILURE);
    }
    check(spm_step(g_run, 1), "spm_step");
    const int next = jikan.ts + 1;
    if (jikan.ts == MSTEP || (next <= MSTEP && next % GTS == 0)) download(zeta, uk_dc, p);
}

}  // namespace

// A constant force on every particle, added where Force() adds gravity
// (particle_solver.h:88-111); for a host that applies one on the CPU side
// (the reference has no input for it at density 1).  Call before
// kapsel_b200_go_resident.
extern "C" void kapsel_b200_set_body_force(double fx, double fy, double fz) {
    g_body_force[0] = fx;
    g_body_force[1] = fy;
    g_body_force[2] = fz;
}

// Called by the program once its initialisation is complete and before its
// main loop (see the build's Show_output_parameter hook).
extern "C" void kapsel_b200_go_resident() {
    if ((SW_PT != spherical_particle && SW_PT != rigid) || SW_WALL != NO_WALL || PINNING ||
        Component_Number > SPM_MAX_SPECIES || (SW_JANUS && Component_Number != 1))
        return;
    if (SW_EQ == Navier_Stokes) {
        g_eq = SPM_EQ_NAVIER_STOKES;
    } else if (SW_EQ == Shear_Navier_Stokes) {
        g_eq = SPM_EQ_SHEAR_NAVIER_STOKES;
    } else if (SW_EQ == Shear_Navier_Stokes_Lees_Edwards) {
        g_eq = SPM_EQ_LEES_EDWARDS;
    } else if (SW_EQ == Electrolyte) {
        g_eq = SPM_EQ_ELECTROLYTE;
    } else {
        return;
    }
    // a run the library refuses stays on the CPU
    spm_params prm = kapsel_b200::params_from_globals(g_eq);
    size_t     bytes = 0;
    if (spm_device_bytes(&prm, &bytes) != SPM_OK) {
        fprintf(stderr, "# kapsel_b200: time evolution stays on the CPU: %s\n", spm_last_error());
        return;
    }
    Time_evolution = resident_time_evolution;
    fprintf(stderr, "# kapsel_b200: time evolution resident on the GPU (host copies at output frames)\n");
}
