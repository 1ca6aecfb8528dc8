// Lees-Edwards (sheared) step: oblique-coordinate state and kernels.
#pragma once

#include "spm_common.cuh"
#include "spm_kernels.cuh"

namespace spm {

// Extra field slots the Lees-Edwards step needs beyond the common arena.
constexpr int LE_EXTRA_SLOTS = 4;

struct LEState {
    int    enabled        = 0;
    double shear_rate     = 0.0;
    double degree_oblique = 0.0;
    double stress[4]      = {0, 0, 0, 0};
};

inline void le_init(LEState &le, const Grid &, const Phys &, const spm_params &p) {
    le.enabled    = p.equation == SPM_EQ_LEES_EDWARDS;
    le.shear_rate = p.shear_rate;
}
inline void le_reset(LEState &le) {
    le.degree_oblique = 0.0;
    for (double &s : le.stress) s = 0.0;
}
inline int le_get_state(const LEState &le, double *deg, double stress[4]) {
    if (deg) *deg = le.degree_oblique;
    if (stress)
        for (int i = 0; i < 4; i++) stress[i] = le.stress[i];
    return SPM_OK;
}

}  // namespace spm

template <typename T, typename C>
int step_le(C *c) {
    (void)c;
    return -1;  // not available
}
