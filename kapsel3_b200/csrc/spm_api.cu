// C ABI of the B200 SPM step: context management, the whole step on
// device-resident state, and the reference-boundary entry points.
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/kapsel_spm.h"
#include "spm_fft_plan.cuh"
#include "spm_kernels.cuh"
#include "spm_le.cuh"

using namespace spm;

namespace {
thread_local std::string g_last_error;
int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}
}  // namespace

// Error reporting for the other translation units of the library.
int spm_internal_fail(int code, const char *msg) { return fail(code, msg); }

#undef SPM_CUDA_CHECK
#define SPM_CUDA_CHECK(expr)                                                                             \
    do {                                                                                                 \
        cudaError_t _e = (expr);                                                                         \
        if (_e != cudaSuccess)                                                                           \
            return fail(_e == cudaErrorMemoryAllocation ? SPM_ERR_NOMEM : SPM_ERR_CUDA,                  \
                        std::string(#expr) + ": " + cudaGetErrorName(_e) + " " + cudaGetErrorString(_e)); \
    } while (0)

// Doubles per particle in the device particle buffer: 12 three-vectors and
// two quaternions of the record, x_previous, torque_r, torque_r_previous,
// momentum_depend_fr and lj_stress.
constexpr int kPWords = 12 * 3 + 2 * 4 + 4 * 3 + 1;

// Field slots of the context arena (consecutive, fstride complex apart).
enum Slot { Z0 = 0, Z1, U0, U1, U2, A0, A1, UP0, UP1, UP2, PHIS, NSLOT };

struct spm_ctx {
    spm_params   P{};
    Grid         g{};
    Phys         ph{};
    cudaStream_t st         = nullptr;
    bool         own_stream = false;
    void *       arena      = nullptr;  // NSLOT fields
    size_t       fstride_c  = 0;        // complex elements per field
    FFTPlan<double> plan64;
    FFTPlan<float>  plan32;
    int *        cells   = nullptr;
    int          ncells  = 0;
    double *     uk_dc   = nullptr;  // device [3]
    double *     pbuf    = nullptr;  // particle state arrays
    PState       ps{};
    unsigned int *mt  = nullptr;  // 625 words
    unsigned int *err = nullptr;  // device error word
    int          ts   = 0;
    double       time = 0.0;
    long long    launches = 0;
    int          sm_count = 148;
    LEState      le{};
    // optional CUDA-event timing of the strided FFT passes inside real steps
    bool                     prof_on = false;
    std::vector<cudaEvent_t> prof_ev;
    double                   prof_bytes = 0.0;
    bool                     use_tma    = true;  // SPM_NO_TMA=1 selects the direct-load passes

    bool fp64() const { return P.precision == SPM_PREC_FP64; }
    template <typename T>
    T *real(int slot) const {
        return reinterpret_cast<T *>(static_cast<char *>(arena) + (size_t)slot * fstride_c * 2 * sizeof(T));
    }
    template <typename T>
    cplx<T> *cx(int slot) const {
        return reinterpret_cast<cplx<T> *>(real<T>(slot));
    }
    size_t elem_bytes() const { return fp64() ? sizeof(double) : sizeof(float); }
    size_t field_bytes() const { return fstride_c * 2 * elem_bytes(); }
    int    grid_blocks() const { return sm_count * 16; }
};

#define LAUNCH(ctx, kern, grid, block, smem, ...)                                           \
    do {                                                                                    \
        kern<<<(grid), (block), (smem), (ctx)->st>>>(__VA_ARGS__);                          \
        (ctx)->launches++;                                                                  \
        cudaError_t _le = cudaGetLastError();                                               \
        if (_le != cudaSuccess) return fail(SPM_ERR_CUDA, std::string("launch " #kern ": ") + \
                                                              cudaGetErrorString(_le));     \
    } while (0)

namespace {

// ---------------------------------------------------------------------------
// Parameter derivation (Set_global_parameters, input.cxx:425-604; particle
// section of Gourmet_file_io, input.cxx:1701-1707, 1807-1827).
// ---------------------------------------------------------------------------
int derive(const spm_params &p, Grid &g, Phys &ph) {
    if (p.npx < 3 || p.npx > 9 || p.npy < 3 || p.npy > 9 || p.npz < 3 || p.npz > 9)
        return fail(SPM_ERR_ARG, "mesh.NPX/NPY/NPZ must be in [3, 9] (grid 8..512 per axis)");
    if (p.n_particles < 0) return fail(SPM_ERR_ARG, "negative particle count");
    if (!(p.dx > 0) || !(p.rho > 0) || !(p.eta > 0) || !(p.dt > 0)) return fail(SPM_ERR_ARG, "DX, RHO, ETA, dt must be > 0");
    if (p.precision != SPM_PREC_FP64 && p.precision != SPM_PREC_FP32_MIXED) return fail(SPM_ERR_ARG, "bad precision");
    if (p.equation != SPM_EQ_NAVIER_STOKES && p.equation != SPM_EQ_LEES_EDWARDS) return fail(SPM_ERR_ARG, "bad equation");
    if (p.lj_powers < 0 || p.lj_powers > 2) return fail(SPM_ERR_ARG, "LJ_powers must be 12:6, 24:12 or 36:18");
    g.nx  = 1 << p.npx;
    g.ny  = 1 << p.npy;
    g.nz  = 1 << p.npz;
    g.hnz = g.nz / 2 + 1;
    g.hnzp = (p.precision == SPM_PREC_FP64) ? g.hnz : ((g.hnz + 1) & ~1);
    const int n[3] = {g.nx, g.ny, g.nz};
    for (int d = 0; d < 3; d++) {
        g.trn[d]  = (n[d] + 2) / 3;
        g.wave[d] = 2.0 * 3.14159265358979323846 / ((double)n[d] * p.dx);
    }
    g.dx = p.dx;

    const double radius = p.a * p.dx;
    const double xi     = p.a_xi * p.dx;
    const double sigma  = 2.0 * radius;
    const double mass   = p.mass_ratio * p.rho * 4.0 / 3.0 * M_PI * radius * radius * radius;
    const double moi    = 2.0 / 5.0 * mass * radius * radius;
    const double pw     = p.lj_powers == 0 ? 6.0 : (p.lj_powers == 1 ? 12.0 : 18.0);
    double a_r_cutoff   = 0.0;
    if (p.lj_truncate > 0) {
        a_r_cutoff = pow(2.0, 1.0 / pw);
    } else if (p.lj_truncate == 0) {
        const int nmin = std::min(g.nx, std::min(g.ny, g.nz));
        a_r_cutoff     = std::min(nmin * p.dx * 0.5 / sigma, 2.5);
    }
    double lj_dia = sigma;
    if (p.equation == SPM_EQ_LEES_EDWARDS) lj_dia = std::min((sigma + xi) / pow(2.0, 1.0 / pw), sigma);

    ph.dt     = p.dt;
    ph.hdt    = p.dt * 0.5;
    ph.nu     = p.eta / p.rho;
    ph.rho    = p.rho;
    ph.dx3    = p.dx * p.dx * p.dx;
    ph.radius = radius;
    ph.hxi    = xi * 0.5;
    for (int d = 0; d < 3; d++) ph.L[d] = n[d] * p.dx;
    ph.imass     = 1.0 / mass;
    ph.imoi      = 1.0 / moi;
    ph.lj_sigma  = lj_dia;
    ph.lj_cutoff = a_r_cutoff * lj_dia;
    ph.lj_eps    = p.epsilon;
    ph.lj_powers = p.lj_powers;
    ph.lj_on     = p.lj_truncate >= 0 ? 1 : 0;
    ph.rotation  = p.rotation ? 1 : 0;
    for (int d = 0; d < 3; d++) {
        ph.fix_cell[d]   = p.fix_cell[d] ? 1 : 0;
        ph.body_force[d] = p.body_force[d];
        ph.lc[d]         = n[d] / 16;
    }
    ph.cell_len = 16.0 * p.dx;
    if (ph.lj_on && p.equation == SPM_EQ_NAVIER_STOKES && (ph.lc[0] < 1 || ph.lc[1] < 1 || ph.lc[2] < 1))
        return fail(SPM_ERR_ARG, "the reference LJ cell list needs N >= 16 on every axis");
    // Thermostat intensities (fluct.cxx:11-18).
    const double zeta_drag     = 6.0 * M_PI * p.eta * radius;
    const double zeta_drag_rot = 8.0 * M_PI * p.eta * radius * radius * radius;
    ph.noise_v = 1.439 * sqrt(zeta_drag * p.dt * p.kbt * p.alpha_v);
    ph.noise_o = 1.22 * sqrt(zeta_drag_rot * p.dt * p.kbt * p.alpha_o);
    ph.np      = p.n_particles;
    return SPM_OK;
}

// Sekibun stencil (Particle_domain, profile.cxx:22-65): offsets with
// |r| < RADIUS + XI/2 + 1.7321 DX, i-major order; packed as 3 signed bytes.
std::vector<int> sekibun(const spm_params &p) {
    const int    nh         = (int)p.a + (int)p.a_xi + 2;
    const double dx         = p.dx;
    const double max_radius = p.a * dx + 0.5 * p.a_xi * dx + 1.7321 * dx;
    std::vector<int> cells;
    for (int i = -nh; i <= nh; i++)
        for (int j = -nh; j <= nh; j++)
            for (int k = -nh; k <= nh; k++) {
                const double r = sqrt((i * dx) * (i * dx) + (j * dx) * (j * dx) + (k * dx) * (k * dx));
                if (r < max_radius) cells.push_back((i & 0xff) | ((j & 0xff) << 8) | ((k & 0xff) << 16));
            }
    return cells;
}

void mt_init(unsigned int seed, unsigned int *mt) {
    mt[0] = seed;
    for (int i = 1; i < 624; i++) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (unsigned)i;
    mt[624] = 624;
}


int check_device_error(spm_ctx *c) {
    unsigned int e = 0;
    SPM_CUDA_CHECK(cudaMemcpyAsync(&e, c->err, sizeof(e), cudaMemcpyDeviceToHost, c->st));
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    if (e) {
        SPM_CUDA_CHECK(cudaMemsetAsync(c->err, 0, sizeof(unsigned int), c->st));
        std::string m = "device error:";
        if (e & SPM_DEVERR_PARTICLE_OUT_OF_BOX) m += " particle outside the periodic box;";
        if (e & SPM_DEVERR_LJ_CELL_OVERFLOW) m += " LJ cell overflow;";
        if (e & SPM_DEVERR_NAN) m += " non-finite value;";
        return fail(SPM_ERR_DEVICE, m);
    }
    return SPM_OK;
}

template <typename T>
FFTPlan<T> &plan_of(spm_ctx *c);
template <>
FFTPlan<double> &plan_of<double>(spm_ctx *c) {
    return c->plan64;
}
template <>
FFTPlan<float> &plan_of<float>(spm_ctx *c) {
    return c->plan32;
}

// Strided (Y/X) FFT pass: the persistent TMA kernel when it applies, else the
// direct-load kernel.
template <typename T, int DIR>
cudaError_t strided_dispatch(spm_ctx *c, int slot, int nf, int axis) {
    if (c->use_tma) {
        cudaError_t e = plan_of<T>(c).template strided_tma<DIR>(c->cx<T>(slot), nf, c->fstride_c, axis, c->st);
        if (e != cudaErrorNotSupported) return e;
    }
    return plan_of<T>(c).template strided<DIR>(c->cx<T>(slot), nf, c->fstride_c, axis, c->st);
}

// Strided (Y/X) FFT pass, bracketed by CUDA events when profiling is on.
template <typename T, int DIR>
int fft_strided_pass(spm_ctx *c, int slot, int nf, int axis) {
    if (c->prof_on) {
        cudaEvent_t a, b;
        SPM_CUDA_CHECK(cudaEventCreate(&a));
        SPM_CUDA_CHECK(cudaEventCreate(&b));
        SPM_CUDA_CHECK(cudaEventRecord(a, c->st));
        SPM_CUDA_CHECK((strided_dispatch<T, DIR>(c, slot, nf, axis)));
        SPM_CUDA_CHECK(cudaEventRecord(b, c->st));
        c->prof_ev.push_back(a);
        c->prof_ev.push_back(b);
        c->prof_bytes += 2.0 * nf * (double)c->g.nx * c->g.ny * c->g.hnz * sizeof(cplx<T>);
    } else {
        SPM_CUDA_CHECK((strided_dispatch<T, DIR>(c, slot, nf, axis)));
    }
    c->launches++;
    return SPM_OK;
}
template <typename T>
int fft_fwd(spm_ctx *c, int slot, int nf) {
    SPM_CUDA_CHECK(plan_of<T>(c).z_r2c(c->real<T>(slot), c->cx<T>(slot), nf, 2 * c->fstride_c, c->fstride_c, c->st));
    c->launches++;
    int rc;
    if ((rc = fft_strided_pass<T, -1>(c, slot, nf, 1)) != SPM_OK) return rc;
    return fft_strided_pass<T, -1>(c, slot, nf, 0);
}
template <typename T>
int fft_inv(spm_ctx *c, int slot, int nf) {
    int rc;
    if ((rc = fft_strided_pass<T, +1>(c, slot, nf, 0)) != SPM_OK) return rc;
    if ((rc = fft_strided_pass<T, +1>(c, slot, nf, 1)) != SPM_OK) return rc;
    SPM_CUDA_CHECK(plan_of<T>(c).z_c2r(c->cx<T>(slot), c->real<T>(slot), nf, c->fstride_c, 2 * c->fstride_c,
                                       (T)(1.0 / ((double)c->g.nx * c->g.ny * c->g.nz)), c->st));
    c->launches++;
    return SPM_OK;
}

__global__ void k_fix_cell(double *uk_dc, int fx, int fy, int fz) {
    if (threadIdx.x == 0) {
        if (fx) uk_dc[0] = 0.0;
        if (fy) uk_dc[1] = 0.0;
        if (fz) uk_dc[2] = 0.0;
    }
}
__global__ void k_zero3(double *uk_dc) {
    if (threadIdx.x < 3) uk_dc[threadIdx.x] = 0.0;
}

// ---------------------------------------------------------------------------
// Building blocks of the step (templated on the field type).
// ---------------------------------------------------------------------------
template <typename T>
int zeta_to_velocity(spm_ctx *c, int truncate) {
    LAUNCH(c, k_zeta_to_u<T>, c->grid_blocks(), 256, 0, c->g, c->cx<T>(Z0), c->cx<T>(Z1), c->uk_dc, c->cx<T>(U0),
           c->cx<T>(U1), c->cx<T>(U2), truncate);
    return fft_inv<T>(c, U0, 3);
}

// NS_solver_slavedEuler on the context's zeta (fluid_solver.cxx:348-374).
template <typename T>
int ns_solver(spm_ctx *c) {
    int rc;
    // zeta -> u_hat (truncated) -> inverse x, y passes
    LAUNCH(c, k_zeta_to_u<T>, c->grid_blocks(), 256, 0, c->g, c->cx<T>(Z0), c->cx<T>(Z1), c->uk_dc, c->cx<T>(U0),
           c->cx<T>(U1), c->cx<T>(U2), 1);
    if ((rc = fft_strided_pass<T, +1>(c, U0, 3, 0)) != SPM_OK) return rc;
    if ((rc = fft_strided_pass<T, +1>(c, U0, 3, 1)) != SPM_OK) return rc;
    // inverse z + products + forward z in one pass, then forward y, x passes
    SPM_CUDA_CHECK(plan_of<T>(c).z_products(c->cx<T>(U0), c->fstride_c, c->st));
    c->launches++;
    if ((rc = fft_strided_pass<T, -1>(c, U0, 5, 1)) != SPM_OK) return rc;
    if ((rc = fft_strided_pass<T, -1>(c, U0, 5, 0)) != SPM_OK) return rc;
    LAUNCH(c, k_ns_update<T>, c->grid_blocks(), 256, 0, c->g, c->cx<T>(Z0), c->cx<T>(Z1), c->cx<T>(U0),
           c->cx<T>(U1), c->cx<T>(U2), c->cx<T>(A0), c->cx<T>(A1), c->ph.nu, c->ph.dt);
    return SPM_OK;
}

template <typename T>
int phi_sum_scatter(spm_ctx *c) {
    SPM_CUDA_CHECK(cudaMemsetAsync(c->real<T>(PHIS), 0, c->field_bytes(), c->st));
    if (c->ph.np == 0) return SPM_OK;
    dim3 grid((c->ncells + 127) / 128, c->ph.np);
    LAUNCH(c, s_phi_scatter<T>, grid, 128, 0, c->g, c->ph, c->ps.x, c->cells, c->ncells, c->real<T>(PHIS), c->err);
    return SPM_OK;
}

template <typename T>
int up_scatter(spm_ctx *c) {
    SPM_CUDA_CHECK(cudaMemsetAsync(c->real<T>(UP0), 0, 3 * c->field_bytes(), c->st));
    if (c->ph.np == 0) return SPM_OK;
    dim3 grid((c->ncells + 127) / 128, c->ph.np);
    LAUNCH(c, s_up_scatter<T>, grid, 128, 0, c->g, c->ph, c->ps.x, c->ps.v, c->ps.omega, c->cells, c->ncells,
           c->real<T>(PHIS), c->real<T>(UP0), c->real<T>(UP1), c->real<T>(UP2));
    return SPM_OK;
}

// Rigidity projection of the step: f = up - phi u formed inside the forward z
// pass, forward y, x passes, then the projection and the update of zeta and
// uk_dc closed in k space (k_project_add_curl).
template <typename T>
int rigidity_projection(spm_ctx *c) {
    int rc;
    SPM_CUDA_CHECK(plan_of<T>(c).z_makef(c->real<T>(UP0), c->real<T>(U0), c->real<T>(PHIS), c->fstride_c, c->st));
    c->launches++;
    if ((rc = fft_strided_pass<T, -1>(c, UP0, 3, 1)) != SPM_OK) return rc;
    if ((rc = fft_strided_pass<T, -1>(c, UP0, 3, 0)) != SPM_OK) return rc;
    LAUNCH(c, k_project_add_curl<T>, c->grid_blocks(), 256, 0, c->g, c->cx<T>(UP0), c->cx<T>(UP1), c->cx<T>(UP2),
           c->cx<T>(Z0), c->cx<T>(Z1), c->uk_dc);
    return SPM_OK;
}

// The same projection in the reference's order (real-space f_sole, u += f,
// forward transform of u, U_k2zeta_k); kept as the unfused reference path.
template <typename T>
int rigidity_projection_unfused(spm_ctx *c) {
    int rc;
    LAUNCH(c, r_make_f<T>, c->grid_blocks(), 256, 0, c->g, c->real<T>(UP0), c->real<T>(UP1), c->real<T>(UP2),
           c->real<T>(U0), c->real<T>(U1), c->real<T>(U2), c->real<T>(PHIS));
    if ((rc = fft_fwd<T>(c, UP0, 3)) != SPM_OK) return rc;
    LAUNCH(c, k_truncate_project<T>, c->grid_blocks(), 256, 0, c->g, c->cx<T>(UP0), c->cx<T>(UP1), c->cx<T>(UP2), 1);
    if ((rc = fft_inv<T>(c, UP0, 3)) != SPM_OK) return rc;
    LAUNCH(c, r_add3<T>, c->grid_blocks(), 256, 0, c->g, c->real<T>(U0), c->real<T>(U1), c->real<T>(U2),
           c->real<T>(UP0), c->real<T>(UP1), c->real<T>(UP2));
    if ((rc = fft_fwd<T>(c, U0, 3)) != SPM_OK) return rc;
    LAUNCH(c, k_u_to_zeta<T>, c->grid_blocks(), 256, 0, c->g, c->cx<T>(U0), c->cx<T>(U1), c->cx<T>(U2),
           c->cx<T>(Z0), c->cx<T>(Z1), c->uk_dc);
    return SPM_OK;
}

int particle_blocks(spm_ctx *c) { return (c->ph.np + 127) / 128; }

// Time_evolution_hydro (sp_3d_ns.cxx:41-194), Navier_Stokes with free spheres.
template <typename T>
int step_ns(spm_ctx *c) {
    int rc;
    if ((rc = ns_solver<T>(c)) != SPM_OK) return rc;
    LAUNCH(c, k_fix_cell, 1, 32, 0, c->uk_dc, c->ph.fix_cell[0], c->ph.fix_cell[1], c->ph.fix_cell[2]);
    if ((rc = zeta_to_velocity<T>(c, 1)) != SPM_OK) return rc;
    const int euler = c->ts == 0 ? 1 : 0;
    if (c->ph.np > 0) LAUNCH(c, p_position, particle_blocks(c), 128, 0, c->ph, c->ps, euler, 1);
    if ((rc = phi_sum_scatter<T>(c)) != SPM_OK) return rc;
    if (c->ph.np > 0) {
        LAUNCH(c, s_hydro_force<T>, c->ph.np, 256, 0, c->g, c->ph, c->ps.x, c->ps.v, c->ps.omega, c->cells,
               c->ncells, c->real<T>(PHIS), c->real<T>(U0), c->real<T>(U1), c->real<T>(U2), c->ps.f_hydro,
               c->ps.torque_hydro);
        LAUNCH(c, p_forces, (c->ph.np + 3) / 4, 128, 0, c->ph, c->ps, 0, 0.0);
        LAUNCH(c, p_velocity, particle_blocks(c), 128, 0, c->ph, c->ps, euler);
        if (c->P.kbt > 0.0) LAUNCH(c, p_thermostat_serial, 1, 32, 0, c->ph, c->ps, c->mt);
    }
    if ((rc = up_scatter<T>(c)) != SPM_OK) return rc;
    if ((rc = rigidity_projection<T>(c)) != SPM_OK) return rc;
    c->ts++;
    c->time += c->ph.dt;
    return SPM_OK;
}

template <typename T>
int initialize_impl(spm_ctx *c) {
    int rc;
    SPM_CUDA_CHECK(cudaMemsetAsync(c->arena, 0, NSLOT * c->field_bytes(), c->st));
    LAUNCH(c, k_zero3, 1, 32, 0, c->uk_dc);
    if ((rc = phi_sum_scatter<T>(c)) != SPM_OK) return rc;
    if ((rc = up_scatter<T>(c)) != SPM_OK) return rc;
    // u = Zeta_k2u(zeta = 0) = 0
    if ((rc = zeta_to_velocity<T>(c, 1)) != SPM_OK) return rc;
    if ((rc = rigidity_projection<T>(c)) != SPM_OK) return rc;
    LAUNCH(c, k_zero3, 1, 32, 0, c->uk_dc);
    if (c->le.enabled && c->ph.np > 0) LAUNCH(c, p_le_zero_vx, particle_blocks(c), 128, 0, c->ph, c->ps);
    c->ts   = 0;
    c->time = 0.0;
    return SPM_OK;
}

}  // namespace
#include "spm_le_step.inc"
namespace {

template <typename T>
int step_impl(spm_ctx *c) {
    if (c->P.equation == SPM_EQ_LEES_EDWARDS) return step_le_impl<T>(c);
    return step_ns<T>(c);
}

// host <-> device field transfer with precision conversion
int upload_field(spm_ctx *c, int slot, const double *h) {
    const size_t nd = (size_t)c->g.nx * c->g.ny * 2 * c->g.hnz;  // reference layout
    if (c->fp64()) {
        SPM_CUDA_CHECK(cudaMemcpyAsync(c->real<double>(slot), h, nd * sizeof(double), cudaMemcpyHostToDevice, c->st));
        return SPM_OK;
    }
    std::vector<float> tmp(c->fstride_c * 2, 0.0f);
    const size_t rows = (size_t)c->g.nx * c->g.ny;
    for (size_t r = 0; r < rows; r++)
        for (int k = 0; k < 2 * c->g.hnz; k++) tmp[r * 2 * c->g.hnzp + k] = (float)h[r * 2 * c->g.hnz + k];
    SPM_CUDA_CHECK(cudaMemcpyAsync(c->real<float>(slot), tmp.data(), tmp.size() * sizeof(float),
                                   cudaMemcpyHostToDevice, c->st));
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    return SPM_OK;
}
int download_field(spm_ctx *c, int slot, double *h) {
    const size_t nd = (size_t)c->g.nx * c->g.ny * 2 * c->g.hnz;
    if (c->fp64()) {
        SPM_CUDA_CHECK(cudaMemcpyAsync(h, c->real<double>(slot), nd * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
        return SPM_OK;
    }
    std::vector<float> tmp(c->fstride_c * 2);
    SPM_CUDA_CHECK(cudaMemcpyAsync(tmp.data(), c->real<float>(slot), tmp.size() * sizeof(float),
                                   cudaMemcpyDeviceToHost, c->st));
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    const size_t rows = (size_t)c->g.nx * c->g.ny;
    for (size_t r = 0; r < rows; r++)
        for (int k = 0; k < 2 * c->g.hnz; k++) h[r * 2 * c->g.hnz + k] = (double)tmp[r * 2 * c->g.hnzp + k];
    return SPM_OK;
}

int upload_particles(spm_ctx *c, const double *rec, bool normalize_q) {
    const int np = c->ph.np;
    if (np == 0) return SPM_OK;
    std::vector<double> h((size_t)np * 44, 0.0);
    // host staging in the same order as the device arrays (see spm_create)
    for (int n = 0; n < np; n++) {
        const double *r = rec + (size_t)n * SPM_PARTICLE_WORDS;
        double        q[4], qo[4];
        for (int k = 0; k < 4; k++) {
            q[k]  = r[18 + k];
            qo[k] = r[22 + k];
        }
        if (normalize_q) {
            const double nn = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
            for (int k = 0; k < 4; k++) q[k] *= 1.0 / nn;
            for (int k = 0; k < 4; k++) qo[k] = q[k];
        }
        // 3-vectors: record offsets -> device array index
        const int voff[12] = {0, 3, 6, 9, 12, 15, 26, 29, 32, 35, 38, 41};
        for (int a = 0; a < 12; a++)
            for (int d = 0; d < 3; d++) h[(size_t)a * np * 3 + 3 * n + d] = r[voff[a] + d];
        for (int k = 0; k < 4; k++) {
            h[(size_t)12 * np * 3 + 4 * n + k] = q[k];
            h[(size_t)12 * np * 3 + (size_t)np * 4 + 4 * n + k] = qo[k];
        }
    }
    SPM_CUDA_CHECK(cudaMemcpyAsync(c->pbuf, h.data(), (size_t)np * 44 * sizeof(double), cudaMemcpyHostToDevice, c->st));
    // x_previous, torque_r, torque_r_previous, lj_stress start at zero / x
    SPM_CUDA_CHECK(cudaMemcpyAsync(c->ps.x_previous, c->ps.x, (size_t)np * 3 * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
    SPM_CUDA_CHECK(cudaMemsetAsync(c->ps.torque_r, 0, (size_t)np * 3 * sizeof(double), c->st));
    SPM_CUDA_CHECK(cudaMemsetAsync(c->ps.torque_r_previous, 0, (size_t)np * 3 * sizeof(double), c->st));
    SPM_CUDA_CHECK(cudaMemsetAsync(c->ps.lj_stress, 0, (size_t)np * sizeof(double), c->st));
    SPM_CUDA_CHECK(cudaMemsetAsync(c->ps.mdf, 0, (size_t)np * 3 * sizeof(double), c->st));
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    return SPM_OK;
}

int download_particles(spm_ctx *c, double *rec) {
    const int np = c->ph.np;
    if (np == 0) return SPM_OK;
    std::vector<double> h((size_t)np * 44);
    SPM_CUDA_CHECK(cudaMemcpyAsync(h.data(), c->pbuf, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    const int voff[12] = {0, 3, 6, 9, 12, 15, 26, 29, 32, 35, 38, 41};
    for (int n = 0; n < np; n++) {
        double *r = rec + (size_t)n * SPM_PARTICLE_WORDS;
        for (int a = 0; a < 12; a++)
            for (int d = 0; d < 3; d++) r[voff[a] + d] = h[(size_t)a * np * 3 + 3 * n + d];
        for (int k = 0; k < 4; k++) {
            r[18 + k] = h[(size_t)12 * np * 3 + 4 * n + k];
            r[22 + k] = h[(size_t)12 * np * 3 + (size_t)np * 4 + 4 * n + k];
        }
    }
    return SPM_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char *spm_last_error(void) { return g_last_error.c_str(); }

int spm_device_count(int *count) {
    if (!count) return fail(SPM_ERR_ARG, "null count");
    int         n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) n = 0;
    *count = n;
    return SPM_OK;
}

int spm_params_default(spm_params *p) {
    if (!p) return fail(SPM_ERR_ARG, "null params");
    std::memset(p, 0, sizeof(*p));
    p->npx = p->npy = p->npz = 5;
    p->dx = p->rho = p->eta = 1.0;
    p->alpha_v = p->alpha_o = 1.0;
    p->equation    = SPM_EQ_NAVIER_STOKES;
    p->n_particles = 0;
    p->mass_ratio  = 1.0;
    p->a           = 4.0;
    p->a_xi        = 2.0;
    p->epsilon     = 1.0;
    p->lj_powers   = 0;
    p->lj_truncate = 1;
    p->rotation    = 1;
    p->fix_cell[0] = p->fix_cell[1] = p->fix_cell[2] = 1;
    p->dt        = 0.05;
    p->precision = SPM_PREC_FP64;
    p->mt_seed   = 0;
    return SPM_OK;
}

int spm_device_bytes(const spm_params *p, size_t *bytes) {
    if (!p || !bytes) return fail(SPM_ERR_ARG, "null argument");
    Grid g;
    Phys ph;
    int  rc = derive(*p, g, ph);
    if (rc != SPM_OK) return rc;
    const size_t es  = p->precision == SPM_PREC_FP64 ? 8 : 4;
    const size_t fld = (size_t)g.nx * g.ny * g.hnzp * 2 * es;
    const size_t nslot = (p->equation == SPM_EQ_LEES_EDWARDS) ? (size_t)NSLOT + LE_EXTRA_SLOTS : (size_t)NSLOT;
    *bytes = nslot * fld + (size_t)std::max(p->n_particles, 1) * kPWords * 8 + 64 * 1024;
    return SPM_OK;
}

int spm_create(const spm_params *p, void *stream, spm_ctx **out) {
    if (!p || !out) return fail(SPM_ERR_ARG, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SPM_ERR_NO_DEVICE, "no CUDA device visible");
    spm_ctx *c = new spm_ctx();
    c->P       = *p;
    int rc     = derive(*p, c->g, c->ph);
    if (rc != SPM_OK) {
        delete c;
        return rc;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (stream) {
        c->st = static_cast<cudaStream_t>(stream);
    } else {
        if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return fail(SPM_ERR_CUDA, "stream creation failed");
        }
        c->own_stream = true;
    }
    c->fstride_c      = (size_t)c->g.nx * c->g.ny * c->g.hnzp;
    const int nslot   = (p->equation == SPM_EQ_LEES_EDWARDS) ? NSLOT + LE_EXTRA_SLOTS : NSLOT;
    cudaError_t e     = cudaMalloc(&c->arena, (size_t)nslot * c->field_bytes());
    if (e != cudaSuccess) {
        spm_destroy(c);
        return fail(SPM_ERR_NOMEM, std::string("field arena: ") + cudaGetErrorString(e));
    }
    e = c->fp64() ? c->plan64.create(c->g) : c->plan32.create(c->g);
    c->plan64.sm_count = c->plan32.sm_count = c->sm_count;
    {
        const char *nt = getenv("SPM_NO_TMA");
        c->use_tma     = !(nt && nt[0] == '1');
    }
    if (e != cudaSuccess) {
        spm_destroy(c);
        return fail(SPM_ERR_CUDA, std::string("FFT plan: ") + cudaGetErrorString(e));
    }
    std::vector<int> cells = sekibun(*p);
    c->ncells              = (int)cells.size();
    const int np           = std::max(p->n_particles, 1);
    if (cudaMalloc(&c->cells, cells.size() * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->uk_dc, 4 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->pbuf, (size_t)np * kPWords * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->mt, 625 * sizeof(unsigned int)) != cudaSuccess ||
        cudaMalloc(&c->err, sizeof(unsigned int)) != cudaSuccess) {
        spm_destroy(c);
        return fail(SPM_ERR_NOMEM, "small device buffers");
    }
    c->plan64.err = c->plan32.err = c->err;
    cudaMemcpy(c->cells, cells.data(), cells.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemset(c->err, 0, sizeof(unsigned int));
    cudaMemset(c->pbuf, 0, (size_t)np * kPWords * sizeof(double));
    cudaMemset(c->uk_dc, 0, 4 * sizeof(double));
    unsigned int mt[625];
    mt_init(p->mt_seed, mt);
    cudaMemcpy(c->mt, mt, sizeof(mt), cudaMemcpyHostToDevice);
    // particle arrays: 12 three-vectors in record order, then q, q_old, then
    // x_previous, torque_r, torque_r_previous (3-vectors) and lj_stress
    double *b = c->pbuf;
    auto    v3 = [&](int i) { return b + (size_t)i * np * 3; };
    c->ps.x                     = v3(0);
    c->ps.x_nopbc               = v3(1);
    c->ps.v                     = v3(2);
    c->ps.v_old                 = v3(3);
    c->ps.omega                 = v3(4);
    c->ps.omega_old             = v3(5);
    c->ps.f_hydro               = v3(6);
    c->ps.f_hydro_previous      = v3(7);
    c->ps.torque_hydro          = v3(8);
    c->ps.torque_hydro_previous = v3(9);
    c->ps.fr                    = v3(10);
    c->ps.fr_previous           = v3(11);
    c->ps.q                     = b + (size_t)12 * np * 3;
    c->ps.q_old                 = c->ps.q + (size_t)np * 4;
    c->ps.x_previous            = c->ps.q_old + (size_t)np * 4;
    c->ps.torque_r              = c->ps.x_previous + (size_t)np * 3;
    c->ps.torque_r_previous     = c->ps.torque_r + (size_t)np * 3;
    c->ps.mdf                   = c->ps.torque_r_previous + (size_t)np * 3;
    c->ps.lj_stress             = c->ps.mdf + (size_t)np * 3;
    le_init(c->le, c->g, c->ph, *p);
    if (c->le.enabled) {
        if (cudaMalloc(&c->le.dev, sizeof(LEDev)) != cudaSuccess ||
            cudaMalloc(&c->le.ppart, (size_t)np * 6 * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&c->le.partial, (size_t)c->grid_blocks() * sizeof(double)) != cudaSuccess) {
            spm_destroy(c);
            return fail(SPM_ERR_NOMEM, "Lees-Edwards buffers");
        }
        cudaMemset(c->le.dev, 0, sizeof(LEDev));
    }
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        spm_destroy(c);
        return fail(SPM_ERR_CUDA, std::string("create: ") + cudaGetErrorString(e));
    }
    *out = c;
    return SPM_OK;
}

int spm_destroy(spm_ctx *c) {
    if (!c) return SPM_OK;
    if (c->st) cudaStreamSynchronize(c->st);
    c->plan64.destroy();
    c->plan32.destroy();
    cudaFree(c->arena);
    cudaFree(c->cells);
    cudaFree(c->uk_dc);
    cudaFree(c->pbuf);
    cudaFree(c->mt);
    cudaFree(c->err);
    cudaFree(c->le.dev);
    cudaFree(c->le.ppart);
    cudaFree(c->le.partial);
    if (c->own_stream && c->st) cudaStreamDestroy(c->st);
    delete c;
    return SPM_OK;
}

int spm_initialize(spm_ctx *c, const double *particles_host) {
    if (!c) return fail(SPM_ERR_ARG, "null context");
    if (c->ph.np > 0 && !particles_host) return fail(SPM_ERR_ARG, "particle records required");
    int rc = upload_particles(c, particles_host, true);
    if (rc != SPM_OK) return rc;
    le_reset(c->le);
    rc = c->fp64() ? initialize_impl<double>(c) : initialize_impl<float>(c);
    if (rc != SPM_OK) return rc;
    return check_device_error(c);
}

int spm_step(spm_ctx *c, int nsteps) {
    if (!c || nsteps < 0) return fail(SPM_ERR_ARG, "bad argument");
    for (int i = 0; i < nsteps; i++) {
        int rc = c->fp64() ? step_impl<double>(c) : step_impl<float>(c);
        if (rc != SPM_OK) return rc;
    }
    return SPM_OK;
}

int spm_synchronize(spm_ctx *c) {
    if (!c) return fail(SPM_ERR_ARG, "null context");
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    return check_device_error(c);
}

int spm_get_particles(spm_ctx *c, double *rec) {
    if (!c || (!rec && c->ph.np > 0)) return fail(SPM_ERR_ARG, "bad argument");
    int rc = spm_synchronize(c);
    if (rc != SPM_OK) return rc;
    return download_particles(c, rec);
}

int spm_set_particles(spm_ctx *c, const double *rec) {
    if (!c || (!rec && c->ph.np > 0)) return fail(SPM_ERR_ARG, "bad argument");
    return upload_particles(c, rec, false);
}

int spm_get_zeta(spm_ctx *c, double *z0, double *z1, double uk_dc[3]) {
    if (!c || !z0 || !z1 || !uk_dc) return fail(SPM_ERR_ARG, "bad argument");
    int rc;
    if ((rc = spm_synchronize(c)) != SPM_OK) return rc;
    if ((rc = download_field(c, Z0, z0)) != SPM_OK) return rc;
    if ((rc = download_field(c, Z1, z1)) != SPM_OK) return rc;
    SPM_CUDA_CHECK(cudaMemcpy(uk_dc, c->uk_dc, 3 * sizeof(double), cudaMemcpyDeviceToHost));
    return SPM_OK;
}

int spm_set_zeta(spm_ctx *c, const double *z0, const double *z1, const double uk_dc[3]) {
    if (!c || !z0 || !z1 || !uk_dc) return fail(SPM_ERR_ARG, "bad argument");
    int rc;
    if ((rc = upload_field(c, Z0, z0)) != SPM_OK) return rc;
    if ((rc = upload_field(c, Z1, z1)) != SPM_OK) return rc;
    SPM_CUDA_CHECK(cudaMemcpyAsync(c->uk_dc, uk_dc, 3 * sizeof(double), cudaMemcpyHostToDevice, c->st));
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    return SPM_OK;
}

int spm_get_velocity(spm_ctx *c, double *u0, double *u1, double *u2) {
    if (!c || !u0 || !u1 || !u2) return fail(SPM_ERR_ARG, "bad argument");
    int rc = c->le.enabled ? (c->fp64() ? le_velocity<double>(c) : le_velocity<float>(c))
                           : (c->fp64() ? zeta_to_velocity<double>(c, 0) : zeta_to_velocity<float>(c, 0));
    if (rc != SPM_OK) return rc;
    if ((rc = spm_synchronize(c)) != SPM_OK) return rc;
    if ((rc = download_field(c, U0, u0)) != SPM_OK) return rc;
    if ((rc = download_field(c, U1, u1)) != SPM_OK) return rc;
    return download_field(c, U2, u2);
}

int spm_get_phi(spm_ctx *c, double *phi) {
    if (!c || !phi) return fail(SPM_ERR_ARG, "bad argument");
    int rc = c->le.enabled ? (c->fp64() ? le_phi_sum<double>(c) : le_phi_sum<float>(c))
                           : (c->fp64() ? phi_sum_scatter<double>(c) : phi_sum_scatter<float>(c));
    if (rc != SPM_OK) return rc;
    if (c->fp64())
        LAUNCH(c, r_phi_clamp<double>, c->grid_blocks(), 256, 0, c->g, c->real<double>(PHIS), c->real<double>(A0));
    else
        LAUNCH(c, r_phi_clamp<float>, c->grid_blocks(), 256, 0, c->g, c->real<float>(PHIS), c->real<float>(A0));
    if ((rc = spm_synchronize(c)) != SPM_OK) return rc;
    return download_field(c, A0, phi);
}

int spm_get_time(spm_ctx *c, int *ts, double *time) {
    if (!c) return fail(SPM_ERR_ARG, "null context");
    if (ts) *ts = c->ts;
    if (time) *time = c->time;
    return SPM_OK;
}

int spm_get_shear_state(spm_ctx *c, double *degree_oblique, double stress[8]) {
    if (!c) return fail(SPM_ERR_ARG, "null context");
    int rc = spm_synchronize(c);
    if (rc != SPM_OK) return rc;
    return le_get_state(c, degree_oblique, stress);
}

int spm_fft_forward_dev(spm_ctx *c, void *data, int nfields, size_t field_stride) {
    if (!c || !data || nfields < 1) return fail(SPM_ERR_ARG, "bad argument");
    cudaError_t e = c->fp64() ? c->plan64.forward((double *)data, nfields, field_stride, c->st)
                              : c->plan32.forward((float *)data, nfields, field_stride, c->st);
    c->launches += 3;
    SPM_CUDA_CHECK(e);
    return SPM_OK;
}

int spm_fft_inverse_dev(spm_ctx *c, void *data, int nfields, size_t field_stride) {
    if (!c || !data || nfields < 1) return fail(SPM_ERR_ARG, "bad argument");
    cudaError_t e = c->fp64() ? c->plan64.inverse((cplx<double> *)data, nfields, field_stride, c->st)
                              : c->plan32.inverse((cplx<float> *)data, nfields, field_stride, c->st);
    c->launches += 3;
    SPM_CUDA_CHECK(e);
    return SPM_OK;
}

int spm_row_complex(spm_ctx *c, int *hnzp) {
    if (!c || !hnzp) return fail(SPM_ERR_ARG, "bad argument");
    *hnzp = c->g.hnzp;
    return SPM_OK;
}

int spm_time_steps(spm_ctx *c, int nsteps, float *ms) {
    if (!c || !ms || nsteps < 1) return fail(SPM_ERR_ARG, "bad argument");
    cudaEvent_t a, b;
    SPM_CUDA_CHECK(cudaEventCreate(&a));
    SPM_CUDA_CHECK(cudaEventCreate(&b));
    SPM_CUDA_CHECK(cudaEventRecord(a, c->st));
    int rc = spm_step(c, nsteps);
    SPM_CUDA_CHECK(cudaEventRecord(b, c->st));
    SPM_CUDA_CHECK(cudaEventSynchronize(b));
    SPM_CUDA_CHECK(cudaEventElapsedTime(ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc != SPM_OK) return rc;
    return check_device_error(c);
}

int spm_profile_pass(spm_ctx *c, int nsteps, double *avg_us, double *bytes_per_launch, long long *count) {
    if (!c || nsteps < 1 || !avg_us || !bytes_per_launch || !count) return fail(SPM_ERR_ARG, "bad argument");
    c->prof_on    = true;
    c->prof_bytes = 0.0;
    int rc        = spm_step(c, nsteps);
    c->prof_on    = false;
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    double total = 0.0;
    const size_t n = c->prof_ev.size() / 2;
    for (size_t i = 0; i < n; i++) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->prof_ev[2 * i], c->prof_ev[2 * i + 1]);
        total += ms;
    }
    for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
    c->prof_ev.clear();
    if (rc != SPM_OK) return rc;
    *count            = (long long)n;
    *avg_us           = n ? 1000.0 * total / (double)n : 0.0;
    *bytes_per_launch = n ? c->prof_bytes / (double)n : 0.0;
    return check_device_error(c);
}

int spm_kernel_launches(spm_ctx *c, long long *count, int reset) {
    if (!c || !count) return fail(SPM_ERR_ARG, "bad argument");
    *count = c->launches;
    if (reset) c->launches = 0;
    return SPM_OK;
}

}  // extern "C"

#include "spm_api_boundary.inc"
