// Link-time stand-ins for the symbols that the reference's FDM phase-separation
// and HDF5 writer translation units (fdm_phase_separation.cxx,
// output_writer.cxx) would provide.  Those units need the HDF5 C/C++ API,
// which is not installed here, and they are never reached by the spectral
// Navier-Stokes / Lees-Edwards step (they belong to the FDM solver family,
// SW_EQ = *_FDM).  Every function aborts if it is ever called, so a run that
// strays into the FDM path fails loudly instead of computing nonsense.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "variable.h"  // CTime, Particle (reference types)

namespace {
[[noreturn]] void fdm_unavailable(const char *what) {
    std::fprintf(stderr, "reference oracle: FDM/HDF5 routine '%s' is not built into the oracle\n", what);
    std::abort();
}
}  // namespace

double * cp;
double * psi;
double * psi_o;
double * psicp;
double * psicp_o;
double * phi_obl;
double **stress;
double **stress_o;

void Calc_cp(double *, double *, double *) { fdm_unavailable("Calc_cp"); }
void Calc_cp_OBL(double *, double *, double *, double) { fdm_unavailable("Calc_cp_OBL"); }
void Cp2stress(double *, double *, double **) { fdm_unavailable("Cp2stress"); }
void Cp2stress_OBL(double *, double *, double **, double) { fdm_unavailable("Cp2stress_OBL"); }
void Init_phase_separation(double *, double *) { fdm_unavailable("Init_phase_separation"); }
void Psi2eta(double *, double *) { fdm_unavailable("Psi2eta"); }
void Set_poisson_rhs_ps(double **, double **, double **, double **, double *, CTime &) {
    fdm_unavailable("Set_poisson_rhs_ps");
}
void Set_poisson_rhs_viscosity(double **, double **, double **, double **, double **, double *, double *, CTime &) {
    fdm_unavailable("Set_poisson_rhs_viscosity");
}
void Set_poisson_rhs_viscosity_OBL(double **, double **, double **, double **, double **, double *, double *, CTime &) {
    fdm_unavailable("Set_poisson_rhs_viscosity_OBL");
}
void Update_psi_euler(double *, double **, double *, double *, CTime &) { fdm_unavailable("Update_psi_euler"); }
void Update_psi_euler_OBL(double *, double **, double *, CTime &, double) { fdm_unavailable("Update_psi_euler_OBL"); }
void Update_u_stress_ab2(double **, double **, double **, CTime &) { fdm_unavailable("Update_u_stress_ab2"); }
void Update_u_stress_euler(double **, double **, CTime &) { fdm_unavailable("Update_u_stress_euler"); }
void Output_hdf5_particle(std::string, Particle *, int) { fdm_unavailable("Output_hdf5_particle"); }
void Output_hdf5_particle_single(std::string, Particle *, int) { fdm_unavailable("Output_hdf5_particle_single"); }
void Output_hdf5_sca(std::string, std::string, double *, int) { fdm_unavailable("Output_hdf5_sca"); }
void Output_hdf5_vec(std::string, std::string, std::string, std::string, double **, int) {
    fdm_unavailable("Output_hdf5_vec");
}
void xdmf_output(CTime) { fdm_unavailable("xdmf_output"); }
