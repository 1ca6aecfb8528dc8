// C ABI of the B200 SPM step: context management, the whole step on
// device-resident state, and the reference-boundary entry points.
#include <atomic>
#include <cerrno>
#include <condition_variable>
#include <deque>
#include <thread>
#include <cctype>
#include <cstdlib>
#include <mutex>
#include <unordered_map>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include <sys/stat.h>

#include "../../include/kapsel_spm.h"
#include "spm_fft_plan.cuh"
#include "spm_kernels.cuh"
#include "spm_rigid.cuh"
#include "spm_le.cuh"
#include "spm_electrolyte.cuh"
#include "spm_janus.cuh"
#include "spm_sns.cuh"

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

namespace {
// Device allocations of contexts and pools go through dev_alloc, which can be
// told to fail the next n calls (host-side fault injection for the serving
// tests; spm_debug_fail_allocations).
std::atomic<int> g_fail_allocs{0};

// Device memory comes from a stream-ordered memory pool per device whose
// release threshold is unbounded: a freed block goes back to the pool, still
// mapped, and the next allocation reuses it.  cudaFree of a large block waits
// for the whole device and then unmaps it; on B200 a pool arena's cudaFree
// took up to 0.8 s inside a serving loop, a stall for every run in flight.
// Allocations are ordered on the pool's own stream and completed before
// dev_alloc returns, so any stream may use the block; a block is freed only
// after its owner's stream was synchronised (destroy_ctx, pool growth), so no
// work still uses it when the pool hands it out again.
struct DevMemPool {
    cudaMemPool_t pool = nullptr;
    cudaStream_t  st   = nullptr;
};
struct DevMem {
    std::mutex                        mu;
    std::unordered_map<int, DevMemPool> pools;  // device -> pool
    std::unordered_map<void *, int>     live;   // block -> device
};
DevMem &dev_mem() {
    static DevMem m;
    return m;
}
// The pool of device `dev` (created on first use; caller holds mu).
cudaError_t dev_pool(DevMem &m, int dev, DevMemPool **out) {
    auto it = m.pools.find(dev);
    if (it != m.pools.end()) {
        *out = &it->second;
        return cudaSuccess;
    }
    cudaMemPoolProps props{};
    props.allocType     = cudaMemAllocationTypePinned;
    props.handleTypes   = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id   = dev;
    DevMemPool dp;
    cudaError_t e = cudaMemPoolCreate(&dp.pool, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = ~0ull;
    if ((e = cudaMemPoolSetAttribute(dp.pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&dp.st, cudaStreamNonBlocking)) != cudaSuccess) {
        cudaMemPoolDestroy(dp.pool);
        return e;
    }
    *out = &(m.pools[dev] = dp);
    return cudaSuccess;
}

cudaError_t dev_alloc(void **p, size_t bytes) {
    for (int n = g_fail_allocs.load(); n > 0; n = g_fail_allocs.load())
        if (g_fail_allocs.compare_exchange_weak(n, n - 1)) {
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
    int dev = 0;
    cudaGetDevice(&dev);
    DevMem                     &m = dev_mem();
    std::lock_guard<std::mutex> lk(m.mu);
    DevMemPool                 *dp = nullptr;
    cudaError_t                 e  = dev_pool(m, dev, &dp);
    if (e != cudaSuccess) return e;
    if ((e = cudaMallocFromPoolAsync(p, bytes, dp->pool, dp->st)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(dp->st)) != cudaSuccess) return e;
    m.live[*p] = dev;
    return cudaSuccess;
}
void dev_free(void *p) {
    if (!p) return;
    DevMem                     &m = dev_mem();
    std::lock_guard<std::mutex> lk(m.mu);
    auto it = m.live.find(p);
    if (it == m.live.end()) return;
    auto pit = m.pools.find(it->second);
    if (pit != m.pools.end()) cudaFreeAsync(p, pit->second.st);
    m.live.erase(it);
}
}  // namespace

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
// FP32-mixed Navier_Stokes runs keep zeta as an unevaluated sum hi + lo of two
// FP32 fields: Z0/Z1 hold hi (the value every transform reads) and ZL0/ZL1
// the compensation term of the Kahan-style (TwoSum) updates.
constexpr int ZL0 = NSLOT, ZL1 = NSLOT + 1;

// Field slots a run needs.
// Electrolyte runs: concentrations, solute right-hand sides, grad psi,
// solute flux, surface normal, charge, raw phi, work, solute velocity
constexpr int EL_EXTRA_SLOTS = 19;
int slots_for(const spm_params &p) {
    if (p.equation == SPM_EQ_LEES_EDWARDS) return NSLOT + LE_EXTRA_SLOTS;
    if (p.equation == SPM_EQ_ELECTROLYTE) return NSLOT + EL_EXTRA_SLOTS;
    return p.precision == SPM_PREC_FP32_MIXED ? NSLOT + 2 : NSLOT;
}

struct spm_pool;
struct AvsOut;
struct UdfOut;

struct spm_ctx {
    spm_params   P{};
    Grid         g{};
    Phys         ph{};
    cudaStream_t st         = nullptr;
    bool         own_stream = false;
    // second stream of the step: the particle work that only needs the
    // previous step's state (position update, phi scatter, Lennard-Jones
    // forces, clearing the scatter slots) runs on it beside the fluid solver
    cudaStream_t side     = nullptr;
    cudaEvent_t  ev_fork  = nullptr;
    cudaEvent_t  ev_join  = nullptr;
    void *       arena      = nullptr;  // slot 0 of this run's fields
    size_t       fstride_c  = 0;        // complex elements per field
    size_t       slot_stride_c = 0;     // complex elements between two slots of this run
    bool         owns_arena = true;     // false for runs living in a pool's arena
    int          fft_runs   = 1;        // runs batched by this context's FFT stages (pool lead)
    RunWords *   rw         = nullptr;  // uk_dc, step counter, FIX_CELL mask (device)
    bool         owns_rw    = true;     // false for runs of a pool
    int *        ts_dev     = nullptr;  // &rw->ts
    FFTPlan<double> plan64;
    FFTPlan<float>  plan32;
    FFTPlan<double> *pp64 = &plan64;  // the plans in use (a pool's runs use the lead's)
    FFTPlan<float>  *pp32 = &plan32;
    spm_pool        *pool = nullptr;  // pool this run belongs to (null for a lone run)
    int *        cells   = nullptr;
    int *        lj_list = nullptr;  // LJ cell list: count[ncell], cell_of[np], bins[ncell][kLjBin]
    int *        sc_idx  = nullptr;  // stencil cache of the NS step: grid index per (particle, cell)
    double *     sc_w    = nullptr;  // ... and its profile weight
    int          ncells  = 0;
    double *     uk_dc   = nullptr;  // rw->uk_dc
    double *     pbuf    = nullptr;  // particle state arrays
    double *     rec_stage = nullptr;  // particle records in transit (SPM_PARTICLE_WORDS per particle)
    PState       ps{};
    unsigned int *mt  = nullptr;  // 625 words
    unsigned int *err = nullptr;  // device error word (&rw->err)
    int          ts   = 0;
    double       time = 0.0;
    long long    launches = 0;
    int          sm_count = 148;
    LEState      le{};
    ELState      el{};
    // squirmers: per-particle slip state (kSlipWords each) and the
    // convergence value of the last slip iteration
    double      *slip     = nullptr;
    double      *slip_eps = nullptr;
    // Shear_Navier_Stokes runs: the diagnostics' words and row sums (spm_sns.cuh)
    double      *sns      = nullptr;
    // rigid bodies (spm_rigid.cuh): device state and the species' free degrees of freedom
    RigidDev     rg{};
    RigidFree    rfree{};
    int         *rg_ibuf = nullptr;
    double      *rg_dbuf = nullptr;
    bool         rigid() const { return P.rigid != 0; }
    int          slip_iters = 0;  // iterations of the last step's slip loop
    // optional CUDA-event timing of the step's kernels inside real steps:
    // one record per launch (kernel family, algorithmic bytes, events on the
    // launching stream)
    struct ProfRec {
        const char *name;
        double      bytes;
        cudaEvent_t a, b;
    };
    bool                 prof_on = false;
    std::vector<ProfRec> prof;
    bool                     use_tma    = true;  // SPM_NO_TMA=1 selects the direct-load passes
    bool                     overlap    = true;  // SPM_NO_OVERLAP=1 keeps the particle work on the main stream
    bool                     zeta_dirty = false;  // zeta set by the host since the last NS step
    int                      nslots     = NSLOT;  // field slots of this run (slots_for)
    AvsOut                  *avs        = nullptr;  // AVS field/particle output (spm_avs_open)
    UdfOut                  *udf_out    = nullptr;  // UDF particle records (spm_udf_out_open)
    // one Navier_Stokes step of a lone run captured as a CUDA graph and
    // replayed by spm_step (SPM_NO_GRAPH=1 keeps the direct launches)
    bool                     use_graph    = true;
    cudaGraph_t              step_graph   = nullptr;
    cudaGraphExec_t          step_exec    = nullptr;
    long long                step_kernels = 0;

    bool fp64() const { return P.precision == SPM_PREC_FP64; }
    // zeta kept as a compensated FP32 pair (FP32-mixed Navier_Stokes)
    bool compensated() const {
        return !fp64() && (P.equation == SPM_EQ_NAVIER_STOKES || P.equation == SPM_EQ_SHEAR_NAVIER_STOKES);
    }
    template <typename T>
    cplx<T> *zl(int d) const {
        return compensated() ? cx<T>(ZL0 + d) : nullptr;
    }
    template <typename T>
    T *real(int slot) const {
        return reinterpret_cast<T *>(static_cast<char *>(arena) + (size_t)slot * slot_stride_c * 2 * sizeof(T));
    }
    template <typename T>
    cplx<T> *cx(int slot) const {
        return reinterpret_cast<cplx<T> *>(real<T>(slot));
    }
    size_t elem_bytes() const { return fp64() ? sizeof(double) : sizeof(float); }
    size_t field_bytes() const { return fstride_c * 2 * elem_bytes(); }
    int    grid_blocks() const { return sm_count * 16; }
    // blocks of 256 threads per run for the run-batched k-space kernels
    int pw_blocks() const {
        const size_t need = (fstride_c + 255) / 256;
        const int    cap  = std::max(1, grid_blocks() / std::max(1, fft_runs));
        return (int)std::min<size_t>(need, (size_t)cap);
    }
    dim3 pw_grid() const { return dim3(pw_blocks(), fft_runs); }
    // the same for kernels that visit the retained 2/3 box only
    dim3 box_grid() const {
        const size_t need = (g.box_elems() + 255) / 256;
        const int    cap  = std::max(1, grid_blocks() / std::max(1, fft_runs));
        return dim3((unsigned)std::min<size_t>(need, (size_t)cap), fft_runs);
    }
};

#define SPM_TRY(expr)                   \
    do {                                \
        int _rc = (expr);               \
        if (_rc != SPM_OK) return _rc;  \
    } while (0)

#define LAUNCH(ctx, kern, grid, block, smem, ...)                                           \
    do {                                                                                    \
        kern<<<(grid), (block), (smem), (ctx)->st>>>(__VA_ARGS__);                          \
        (ctx)->launches++;                                                                  \
        cudaError_t _le = cudaGetLastError();                                               \
        if (_le != cudaSuccess) return fail(SPM_ERR_CUDA, std::string("launch " #kern ": ") + \
                                                              cudaGetErrorString(_le));     \
    } while (0)

// Kernel timing inside real steps (spm_profile_kernels): prof_mark records
// an event on the context's current stream before a launch, prof_done one
// after it and files the pair under the kernel family with its algorithmic
// bytes.  Both do nothing unless profiling is on.
inline cudaEvent_t prof_mark(spm_ctx *c) {
    if (!c->prof_on) return nullptr;
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    cudaEventRecord(e, c->st);
    return e;
}
inline void prof_done(spm_ctx *c, cudaEvent_t a, const char *name, double bytes) {
    if (!a) return;
    cudaEvent_t b = nullptr;
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return;
    }
    cudaEventRecord(b, c->st);
    c->prof.push_back({name, bytes, a, b});
}
// LAUNCH, timed under `name` with `bytes` algorithmic bytes when profiling.
#define PLAUNCH(ctx, name, bytes, kern, grid, block, smem, ...)  \
    do {                                                        \
        cudaEvent_t _pa = prof_mark(ctx);                       \
        LAUNCH(ctx, kern, grid, block, smem, __VA_ARGS__);      \
        prof_done(ctx, _pa, name, (bytes));                     \
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
    // particle species (input.cxx:1403-1441)
    const int nsp = p.n_species > 1 ? p.n_species : 1;
    if (nsp > SPM_MAX_SPECIES) return fail(SPM_ERR_ARG, "at most SPM_MAX_SPECIES particle species");
    if (nsp > 1) {
        int sum = 0;
        for (int s = 0; s < nsp; s++) {
            if (p.species_count[s] < 0) return fail(SPM_ERR_ARG, "negative species_count");
            if (!(p.species_mass_ratio[s] > 0.0)) return fail(SPM_ERR_ARG, "species_mass_ratio must be > 0");
            sum += p.species_count[s];
        }
        if (sum != p.n_particles) return fail(SPM_ERR_ARG, "species_count must add up to n_particles");
        if (p.janus_propulsion != SPM_JANUS_OFF) return fail(SPM_ERR_ARG, "janus particles need a single species");
    }
    auto charge_of = [&](int s) { return nsp > 1 ? p.species_surface_charge[s] : p.surface_charge; };
    if (!(p.dx > 0) || !(p.rho > 0) || !(p.eta > 0) || !(p.dt > 0)) return fail(SPM_ERR_ARG, "DX, RHO, ETA, dt must be > 0");
    if (p.precision != SPM_PREC_FP64 && p.precision != SPM_PREC_FP32_MIXED) return fail(SPM_ERR_ARG, "bad precision");
    if (p.equation != SPM_EQ_NAVIER_STOKES && p.equation != SPM_EQ_LEES_EDWARDS && p.equation != SPM_EQ_ELECTROLYTE &&
        p.equation != SPM_EQ_SHEAR_NAVIER_STOKES)
        return fail(SPM_ERR_ARG, "bad equation");
    if (p.rigid && p.equation != SPM_EQ_NAVIER_STOKES && p.equation != SPM_EQ_SHEAR_NAVIER_STOKES &&
        p.equation != SPM_EQ_LEES_EDWARDS)
        return fail(SPM_ERR_ARG, "rigid bodies are served in Navier_Stokes, Shear_Navier_Stokes and Lees-Edwards runs");
    if (p.equation == SPM_EQ_SHEAR_NAVIER_STOKES && (p.shear_ac < 0 || p.shear_ac > 1))
        return fail(SPM_ERR_ARG, "shear_ac must be 0 (DC) or 1 (AC)");
    if (p.equation == SPM_EQ_ELECTROLYTE) {
        // Init_rho_ion's checks (operate_electrolyte.cxx:668-720)
        for (int s = 0; s < nsp; s++)
            if (charge_of(s) == 0.0) return fail(SPM_ERR_ARG, "Electrolyte needs a nonzero Surface_charge");
        for (int s = 1; s < nsp && p.salt == 0; s++)  // saltfree: colloids of one sign (operate_electrolyte.cxx:712-723)
            if (charge_of(0) * charge_of(s) <= 0.0)
                return fail(SPM_ERR_ARG, "saltfree runs need colloids of one sign; select salt in Add_salt");
        if (!(p.dielectric > 0.0)) return fail(SPM_ERR_ARG, "Dielectric_cst must be > 0");
        if (p.init_pb && p.salt == 1 && p.n_particles == 1 && p.valency[0] != -p.valency[1])
            return fail(SPM_ERR_ARG, "Poisson_Boltzmann with salt needs Valency_positive_ion = -Valency_negative_ion");
        if (p.salt == 0 && nsp == 1 && !(p.valency[0] * p.surface_charge < 0.0))
            return fail(SPM_ERR_ARG, "Valency_counterion must have the opposite sign of Surface_charge");
        if (p.salt == 1 && !(p.valency[0] > 0.0 && p.valency[1] < 0.0))
            return fail(SPM_ERR_ARG, "salt needs Valency_positive_ion > 0 and Valency_negative_ion < 0");
        if (p.salt == 1 && !(p.debye_length > 0.0)) return fail(SPM_ERR_ARG, "Debye_length must be > 0");
        if (p.e_field < 0 || p.e_field > 2) return fail(SPM_ERR_ARG, "bad Electric_field");
    }
    if (p.lj_powers < 0 || p.lj_powers > 2) return fail(SPM_ERR_ARG, "LJ_powers must be 12:6, 24:12 or 36:18");
    // Janus particles (input.cxx:1403-1470, 1868-1872)
    if (p.janus_propulsion < SPM_JANUS_OFF || p.janus_propulsion > SPM_JANUS_OBSTACLE)
        return fail(SPM_ERR_ARG, "bad janus_propulsion");
    if (p.janus_axis < SPM_AXIS_NONE || p.janus_axis > SPM_AXIS_Z) return fail(SPM_ERR_ARG, "bad janus_axis");
    // tumblers and squirmers only with the Navier-Stokes solvers; obstacles
    // with every equation (input.cxx:1509-1512)
    if ((p.janus_propulsion == SPM_JANUS_TUMBLER || p.janus_propulsion == SPM_JANUS_SQUIRMER) &&
        p.equation != SPM_EQ_NAVIER_STOKES && p.equation != SPM_EQ_SHEAR_NAVIER_STOKES)
        return fail(SPM_ERR_ARG, "janus tumblers and squirmers are served in Navier_Stokes and Shear_Navier_Stokes "
                                 "runs only");
    if (p.janus_propulsion == SPM_JANUS_SQUIRMER) {
        if (p.janus_axis == SPM_AXIS_NONE) return fail(SPM_ERR_ARG, "a SQUIRMER needs a janus_axis (X, Y or Z)");
        if (!(p.slip_vel > 0.0)) return fail(SPM_ERR_ARG, "a SQUIRMER needs janus_slip_vel (B1) > 0");
        if (p.slip_iter < 1 || !(p.slip_tol >= 0.0)) return fail(SPM_ERR_ARG, "SLIP_iter >= 1 and SLIP_tol >= 0");
    }
    // rigid bodies (object_type.rigid, input.cxx:1583-1700)
    if (p.rigid) {
        if (p.janus_propulsion != SPM_JANUS_OFF) return fail(SPM_ERR_ARG, "rigid bodies have no janus propulsion");
        if (!p.rotation) return fail(SPM_ERR_ARG, "rigid bodies need ROTATION ON");
        if (p.body_force[0] != 0.0 || p.body_force[1] != 0.0 || p.body_force[2] != 0.0)
            return fail(SPM_ERR_ARG, "rigid bodies take no constant body force");
        int beads = 0;
        for (int s = 0; s < nsp; s++) {
            if (p.rigid_beads[s] < 1 || p.rigid_count[s] < 0)
                return fail(SPM_ERR_ARG, "rigid species need Beads_number >= 1 and Chain_number >= 0");
            if (nsp > 1 && p.species_count[s] != p.rigid_beads[s] * p.rigid_count[s])
                return fail(SPM_ERR_ARG, "species_count must be Beads_number * Chain_number for rigid species");
            beads += p.rigid_beads[s] * p.rigid_count[s];
        }
        if (beads != p.n_particles) return fail(SPM_ERR_ARG, "the rigid bodies' beads must add up to n_particles");
        if ((p.rigid_gravity[0] != 0.0) + (p.rigid_gravity[1] != 0.0) + (p.rigid_gravity[2] != 0.0) > 1)
            return fail(SPM_ERR_ARG, "gravity acts along one axis (G_direction)");
    } else if (p.rigid_gravity[0] != 0.0 || p.rigid_gravity[1] != 0.0 || p.rigid_gravity[2] != 0.0) {
        return fail(SPM_ERR_ARG, "rigid_gravity is for rigid bodies; spherical particles take body_force");
    }
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
    if (ph.lj_on && (p.equation == SPM_EQ_NAVIER_STOKES || p.equation == SPM_EQ_SHEAR_NAVIER_STOKES) &&
        (ph.lc[0] < 1 || ph.lc[1] < 1 || ph.lc[2] < 1))
        return fail(SPM_ERR_ARG, "the reference LJ cell list needs N >= 16 on every axis");
    // Thermostat intensities (fluct.cxx:11-18).
    const double zeta_drag     = 6.0 * M_PI * p.eta * radius;
    const double zeta_drag_rot = 8.0 * M_PI * p.eta * radius * radius * radius;
    ph.noise_v = 1.439 * sqrt(zeta_drag * p.dt * p.kbt * p.alpha_v);
    ph.noise_o = 1.22 * sqrt(zeta_drag_rot * p.dt * p.kbt * p.alpha_o);
    ph.np      = p.n_particles;
    ph.nsp     = nsp;
    for (int s = 0, end = 0; s < SPM_MAX_SPECIES; s++) {
        const double mr = nsp > 1 ? p.species_mass_ratio[s < nsp ? s : 0] : p.mass_ratio;
        const double ms = mr * p.rho * 4.0 / 3.0 * M_PI * radius * radius * radius;
        end += s < nsp ? (nsp > 1 ? p.species_count[s] : p.n_particles) : 0;
        ph.spec_end[s] = end;
        ph.imass_s[s]  = 1.0 / ms;
        ph.imoi_s[s]   = 1.0 / (2.0 / 5.0 * ms * radius * radius);
        ph.qe_s[s]     = s < nsp ? charge_of(s) : 0.0;  // Elementary_charge = 1
    }
    ph.janus_prop = p.janus_propulsion;
    ph.janus_axis = p.janus_axis;
    for (int d = 0; d < 3; d++) {
        ph.janus_force[d]  = p.janus_propulsion == SPM_JANUS_TUMBLER ? p.janus_force[d] : 0.0;
        ph.janus_torque[d] = p.janus_propulsion == SPM_JANUS_TUMBLER ? p.janus_torque[d] : 0.0;
    }
    const bool squirm = p.janus_propulsion == SPM_JANUS_SQUIRMER;
    ph.slip_b1   = squirm ? p.slip_vel : 0.0;
    ph.slip_mode = squirm ? p.slip_mode / 2.0 : 0.0;  // alpha/2 = B2/(2 B1) (input.cxx:581-585)
    ph.slip_c1   = squirm ? p.rotlet_c1 : 0.0;
    ph.slip_c2   = squirm ? p.rotlet_c2 : 0.0;
    ph.xi        = xi;
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


// Point uk_dc / ts_dev into the run's RunWords and write its initial words.
void set_run_words(spm_ctx *c) {
    c->uk_dc  = c->rw->uk_dc;
    c->ts_dev = &c->rw->ts;
    c->err    = &c->rw->err;
    RunWords h{};
    const bool le = c->P.equation == SPM_EQ_LEES_EDWARDS;
    h.fix_mask    = (c->ph.fix_cell[0] ? 1 : 0) | ((c->ph.fix_cell[1] || le) ? 2 : 0) | (c->ph.fix_cell[2] ? 4 : 0);
    cudaMemcpy(c->rw, &h, sizeof(h), cudaMemcpyHostToDevice);
}

// Cells of the reference's LJ cell list (lc[d] = N[d] / 16 per axis).
int  lj_ncell(const Phys &ph) { return ph.lc[0] * ph.lc[1] * ph.lc[2]; }
bool lj_cell_list_applies(const Phys &ph) { return ph.lc[0] >= 1 && ph.lc[1] >= 1 && ph.lc[2] >= 1; }

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
        if (e & SPM_DEVERR_SCRATCH_TOO_SMALL) m += " scratch buffer too small;";
        if (e & SPM_DEVERR_TIMEOUT) m += " TMA pipeline wait timed out;";
        const unsigned known = SPM_DEVERR_PARTICLE_OUT_OF_BOX | SPM_DEVERR_LJ_CELL_OVERFLOW | SPM_DEVERR_NAN |
                               SPM_DEVERR_SCRATCH_TOO_SMALL | SPM_DEVERR_TIMEOUT;
        if (e & ~known) m += " unknown error bits 0x" + [](unsigned v) {
            char b[16];
            std::snprintf(b, sizeof(b), "%x", v);
            return std::string(b);
        }(e & ~known) + ";";
        return fail(SPM_ERR_DEVICE, m);
    }
    return SPM_OK;
}

template <typename T>
FFTPlan<T> &plan_of(spm_ctx *c);
template <>
FFTPlan<double> &plan_of<double>(spm_ctx *c) {
    return *c->pp64;
}
template <>
FFTPlan<float> &plan_of<float>(spm_ctx *c) {
    return *c->pp32;
}

// Strided (Y/X) FFT pass over `nf` slots of this context: the persistent TMA
// kernel when it applies, else the direct-load kernel.  A pool lead batches
// the same slots of all its runs (run-consecutive within a slot) into one
// launch per slot.
template <typename T, int DIR>
cudaError_t strided_dispatch(spm_ctx *c, int slot, int nf, int axis, PassPrune pr) {
    auto one = [&](cplx<T> *base, int nfields, size_t stride) {
        if (c->use_tma) {
            cudaError_t e = plan_of<T>(c).template strided_tma<DIR>(base, nfields, stride, axis, c->st, pr);
            if (e != cudaErrorNotSupported) return e;
        }
        return plan_of<T>(c).template strided<DIR>(base, nfields, stride, axis, c->st, pr);
    };
    if (c->fft_runs == 1) return one(c->cx<T>(slot), nf, c->slot_stride_c);
    for (int k = 0; k < nf; k++) {
        cudaError_t e = one(c->cx<T>(slot + k), c->fft_runs, c->fstride_c);
        if (e != cudaSuccess) return e;
        c->launches += k > 0;
    }
    return cudaSuccess;
}

// Pruning of the step's strided passes to the retained 2/3 box (PassPrune):
// inverse passes read modes outside it as zero, forward passes only produce
// the column tiles (and on the X pass the ky lines) the box needs.
PassPrune prune_inverse(const Grid &g, int axis) {
    return axis == 0 ? PassPrune{g.trn[2], g.trn[1], g.trn[0], g.trn[2], 0}
                     : PassPrune{g.trn[2], 0, g.trn[1], g.trn[2], 0};
}
PassPrune prune_forward(const Grid &g, int axis) {
    return axis == 0 ? PassPrune{g.trn[2], g.trn[1], 0, g.hnz, g.trn[0]} : PassPrune{g.trn[2], 0, 0, g.hnz, g.trn[1]};
}

// Complex elements a strided pass must read plus those it must write: the
// visited lines x columns x fields, reads limited to the lines that can be
// nonzero (|K| < line_trn) and writes to the lines that are needed (|K| <
// out_trn) on pruned passes.
template <typename T>
double pass_elems_rw(spm_ctx *c, int nf, int axis, const PassPrune &pr) {
    const Grid &g     = c->g;
    const int   n     = axis == 1 ? g.ny : g.nx;
    const int   outer = axis == 1 ? g.nx : g.ny;
    const int   wk    = (c->use_tma && n <= 256) ? FFTPlan<T>::W_T : FFTPlan<T>::W;
    const int   cols  = std::min(g.hnz, (std::min(pr.kz_cols, g.hnz) + wk - 1) / wk * wk);
    const int   hl    = pruned_box_lines(n, pr.line_trn);
    const int   hs    = pruned_box_lines(n, pr.out_trn);
    const int   lines = (hl == n ? n : 2 * hl) + (hs == n ? n : 2 * hs);
    return (double)nf * c->fft_runs * outer_count(outer, pr.outer_trn) * (double)lines * cols;
}

// Strided (Y/X) FFT pass, bracketed by CUDA events when profiling is on (the
// algorithmic bytes of a pass: pass_elems_rw complex elements).
template <typename T, int DIR>
int fft_strided_pass(spm_ctx *c, int slot, int nf, int axis, PassPrune pr) {
    cudaEvent_t a = prof_mark(c);
    SPM_CUDA_CHECK((strided_dispatch<T, DIR>(c, slot, nf, axis, pr)));
    prof_done(c, a, DIR > 0 ? "strided_pass_inverse" : "strided_pass_forward",
              pass_elems_rw<T>(c, nf, axis, pr) * sizeof(cplx<T>));
    c->launches++;
    return SPM_OK;
}
template <typename T, int DIR>
int fft_strided_pass(spm_ctx *c, int slot, int nf, int axis) {
    return fft_strided_pass<T, DIR>(c, slot, nf, axis, PassPrune::full(c->g.hnz));
}
// z passes over `nf` slots (one launch per slot when batching runs).
// kz_keep: inverse inputs kz >= kz_keep read as zero; kz_span: forward
// outputs kz >= kz_span left unwritten (both: pruned transforms).
template <typename T>
int z_pass_launch(spm_ctx *c, int slot, int nf, bool forward, int kz_keep, int kz_span) {
    const T scale = (T)(1.0 / ((double)c->g.nx * c->g.ny * c->g.nz));
    auto    one   = [&](int s, int nfields, size_t stride) {
        return forward ? plan_of<T>(c).z_r2c(c->real<T>(s), c->cx<T>(s), nfields, 2 * stride, stride, c->st,
                                             kz_span)
                       : plan_of<T>(c).z_c2r(c->cx<T>(s), c->real<T>(s), nfields, stride, 2 * stride, scale, c->st,
                                             kz_keep);
    };
    if (c->fft_runs == 1) {
        SPM_CUDA_CHECK(one(slot, nf, c->slot_stride_c));
        c->launches++;
        return SPM_OK;
    }
    for (int k = 0; k < nf; k++) {
        SPM_CUDA_CHECK(one(slot + k, c->fft_runs, c->fstride_c));
        c->launches++;
    }
    return SPM_OK;
}
template <typename T>
int z_pass(spm_ctx *c, int slot, int nf, bool forward, int kz_keep = 1 << 30, int kz_span = 1 << 30) {
    // algorithmic bytes: the real rows (NZ values) and the complex values
    // read (kz < kz_keep) or written (kz < kz_span)
    const double rows = (double)nf * c->fft_runs * c->g.nx * c->g.ny;
    const double kz   = std::min(forward ? kz_span : kz_keep, c->g.hnz);
    cudaEvent_t  pa   = prof_mark(c);
    const int    rc   = z_pass_launch<T>(c, slot, nf, forward, kz_keep, kz_span);
    prof_done(c, pa, forward ? "z_r2c" : "z_c2r", rows * (c->g.nz * sizeof(T) + kz * sizeof(cplx<T>)));
    return rc;
}
template <typename T>
int fft_fwd(spm_ctx *c, int slot, int nf) {
    int rc;
    if ((rc = z_pass<T>(c, slot, nf, true)) != SPM_OK) return rc;
    if ((rc = fft_strided_pass<T, -1>(c, slot, nf, 1)) != SPM_OK) return rc;
    return fft_strided_pass<T, -1>(c, slot, nf, 0);
}
template <typename T>
int fft_inv(spm_ctx *c, int slot, int nf) {
    int rc;
    if ((rc = fft_strided_pass<T, +1>(c, slot, nf, 0)) != SPM_OK) return rc;
    if ((rc = fft_strided_pass<T, +1>(c, slot, nf, 1)) != SPM_OK) return rc;
    return z_pass<T>(c, slot, nf, false);
}

// Inverse transform of fields that may carry entries outside the 2/3 box
// (state getters, output frames, the Coulomb force path): the packed-plane
// reading of the reference's A_k2a first (k_packed_planes), then fft_inv.
template <typename T>
int fft_inv_packed(spm_ctx *c, int slot, int nf) {
    LAUNCH(c, k_packed_planes<T>, dim3((2 * c->g.nx * c->g.ny + 255) / 256, nf), 256, 0, c->g, c->cx<T>(slot),
           c->slot_stride_c);
    return fft_inv<T>(c, slot, nf);
}

// Transforms of fields that are zero outside the 2/3 box, or whose modes
// outside it are never used: the pruned passes of the Navier_Stokes step.
// fft_inv_box = truncate, then inverse (only lines |K| < TRN and kz < TRN_Z
// are read); fft_fwd_box = forward, valid inside the box only (rows kz >=
// kz_span and lines outside it are not written).
template <typename T>
int fft_inv_box(spm_ctx *c, int slot, int nf) {
    SPM_TRY((fft_strided_pass<T, +1>(c, slot, nf, 0, prune_inverse(c->g, 0))));
    SPM_TRY((fft_strided_pass<T, +1>(c, slot, nf, 1, prune_inverse(c->g, 1))));
    return z_pass<T>(c, slot, nf, false, c->g.trn[2]);
}
template <typename T>
int fft_fwd_box(spm_ctx *c, int slot, int nf) {
    SPM_TRY(z_pass<T>(c, slot, nf, true, 1 << 30, c->g.kz_span()));
    SPM_TRY((fft_strided_pass<T, -1>(c, slot, nf, 1, prune_forward(c->g, 1))));
    return fft_strided_pass<T, -1>(c, slot, nf, 0, prune_forward(c->g, 0));
}

__global__ void k_zero3(double *uk_dc) {
    if (threadIdx.x < 3) uk_dc[threadIdx.x] = 0.0;
}

// Algorithmic bytes of a k-space kernel over the retained 2/3 box: `words`
// complex values read or written per retained mode, for every batched run.
template <typename T>
double box_bytes(const spm_ctx *L, int words) {
    return (double)L->fft_runs * (double)L->g.box_elems() * words * sizeof(cplx<T>);
}
// Algorithmic bytes of a stencil kernel over Np x NP_domain cells: the
// cached grid index (4 B) and weight (8 B) of every cell plus the field
// words it touches: kind 0 (phi scatter) a read-modify-write of phi; kind 1
// (hydrodynamic force) reads of u (3) and phi; kind 2 (f scatter) reads of u
// (3) and phi and read-modify-writes of the three f components.
template <typename T>
double stencil_bytes(const spm_ctx *c, int kind) {
    const int words = kind == 0 ? 2 : kind == 1 ? 4 : 10;
    return (double)c->ph.np * c->ncells * (12.0 + words * sizeof(T));
}

// ---------------------------------------------------------------------------
// Building blocks of the step (templated on the field type).  The `_runs`
// forms advance runs R[0..nr) that share one grid: per-run kernels go to each
// run, FFT stages to L, which is either the run itself or a pool lead whose
// FFT launches cover the same slots of every run of the pool.
// ---------------------------------------------------------------------------
// u (real space) from zeta.  truncate = 1 is the step's Zeta_k2u (2/3 rule
// applied, pruned passes); truncate = 0 keeps every mode (state getters).
template <typename T>
int zeta_to_velocity(spm_ctx *L, int truncate, bool have_u_hat = false) {
    if (!truncate) {
        LAUNCH(L, (k_zeta_to_u<T, 0>), L->pw_grid(), 256, 0, L->g, L->cx<T>(Z0), L->cx<T>(Z1), L->uk_dc, L->cx<T>(U0),
               L->cx<T>(U1), L->cx<T>(U2), 0, L->fstride_c);
        return fft_inv_packed<T>(L, U0, 3);
    }
    int rc;
    if (!have_u_hat)
        PLAUNCH(L, "k_zeta_to_u", box_bytes<T>(L, 5), (k_zeta_to_u<T, 1>), L->box_grid(), 256, 0, L->g,
                L->cx<T>(Z0), L->cx<T>(Z1), L->uk_dc, L->cx<T>(U0), L->cx<T>(U1), L->cx<T>(U2), 1, L->fstride_c);
    if ((rc = fft_strided_pass<T, +1>(L, U0, 3, 0, prune_inverse(L->g, 0))) != SPM_OK) return rc;
    if ((rc = fft_strided_pass<T, +1>(L, U0, 3, 1, prune_inverse(L->g, 1))) != SPM_OK) return rc;
    return z_pass<T>(L, U0, 3, false, L->g.trn[2]);
}

// NS_solver_slavedEuler (fluid_solver.cxx:348-374).  with_u: the update also
// writes the velocity of the new zeta (the k_zeta_to_u that Zeta_k2u of the
// step would run next) into U0..U2, k = 0 with FIX_CELL applied.
template <typename T>
int ns_solver(spm_ctx *L, bool with_u = false) {
    int rc;
    // zeta -> u_hat (truncated) -> inverse x, y passes
    PLAUNCH(L, "k_zeta_to_u", box_bytes<T>(L, 5), (k_zeta_to_u<T, 1>), L->box_grid(), 256, 0, L->g, L->cx<T>(Z0),
            L->cx<T>(Z1), L->uk_dc, L->cx<T>(U0), L->cx<T>(U1), L->cx<T>(U2), 1, L->fstride_c);
    if ((rc = fft_strided_pass<T, +1>(L, U0, 3, 0, prune_inverse(L->g, 0))) != SPM_OK) return rc;
    if ((rc = fft_strided_pass<T, +1>(L, U0, 3, 1, prune_inverse(L->g, 1))) != SPM_OK) return rc;
    // inverse z + products + forward z in one pass, then forward y, x passes
    {
        const double rows = (double)L->fft_runs * L->g.nx * L->g.ny;
        cudaEvent_t  pa   = prof_mark(L);
        SPM_CUDA_CHECK(plan_of<T>(L).z_products(L->cx<T>(U0), L->slot_stride_c, L->fft_runs, L->fstride_c, L->st,
                                                L->g.trn[2], L->g.kz_span()));
        prof_done(L, pa, "z_products", rows * (3.0 * L->g.trn[2] + 5.0 * L->g.kz_span()) * sizeof(cplx<T>));
    }
    L->launches++;
    if ((rc = fft_strided_pass<T, -1>(L, U0, 5, 1, prune_forward(L->g, 1))) != SPM_OK) return rc;
    if ((rc = fft_strided_pass<T, -1>(L, U0, 5, 0, prune_forward(L->g, 0))) != SPM_OK) return rc;
    PLAUNCH(L, "k_ns_update", box_bytes<T>(L, (L->compensated() ? 13 : 9) + (with_u ? 3 : 0)), (k_ns_update<T, 2>),
            L->box_grid(), 256, 0, L->g, L->cx<T>(Z0), L->cx<T>(Z1), L->cx<T>(U0), L->cx<T>(U1), L->cx<T>(U2),
            L->cx<T>(A0), L->cx<T>(A1), L->ph.nu, L->ph.dt, L->fstride_c, L->zl<T>(0), L->zl<T>(1),
            with_u ? L->rw : (const RunWords *)nullptr);
    return SPM_OK;
}

// Shared-profile scatters (Make_phi_particle_sum, make_phi.cxx:226-247;
// Make_phi_u_particle, make_phi.cxx:335-379 with phi taken from PHIS).
// `clear` zeroes the target slots first; the step clears them all at once.
template <typename T>
int phi_sum_scatter(spm_ctx *c, bool clear = true) {
    if (clear) SPM_CUDA_CHECK(cudaMemsetAsync(c->real<T>(PHIS), 0, c->field_bytes(), c->st));
    if (c->ph.np == 0) return SPM_OK;
    dim3 grid((c->ncells + 127) / 128, c->ph.np);
    LAUNCH(c, s_phi_scatter<T>, grid, 128, 0, c->g, c->ph, c->ps.x, c->cells, c->ncells, c->real<T>(PHIS), c->err);
    return SPM_OK;
}

template <typename T>
int up_scatter(spm_ctx *c, bool clear = true) {
    if (clear)
        for (int d = 0; d < 3; d++) SPM_CUDA_CHECK(cudaMemsetAsync(c->real<T>(UP0 + d), 0, c->field_bytes(), c->st));
    if (c->ph.np == 0) return SPM_OK;
    dim3 grid((c->ncells + 127) / 128, c->ph.np);
    LAUNCH(c, s_up_scatter<T>, grid, 128, 0, c->g, c->ph, c->ps.x, c->ps.v, c->ps.omega, c->cells, c->ncells,
           c->real<T>(PHIS), c->real<T>(UP0), c->real<T>(UP1), c->real<T>(UP2));
    return SPM_OK;
}

// The self-consistent slip iteration of squirmers (the SW_JANUS_SLIP branch
// of Time_evolution_hydro, sp_3d_ns.cxx:121-161), after the hydrodynamic
// force: the particle and surface moments, then until convergence the slip
// force field (droplet counter-flow + surface slip) in UP, its solenoidal
// projection, the slip force and the velocity update; between iterations
// v_slip relaxes and v returns to v_old.  At the end u += UP (Swap_mem of
// u and up + u) and UP keeps the slip field, to which the rigidity force f
// is added.  The convergence value is read on the host every iteration.
template <typename T>
int slip_loop(spm_ctx *c) {
    const int  pb = (c->ph.np + 127) / 128;
    const dim3 sgrid((c->ncells + 127) / 128, c->ph.np);
    LAUNCH(c, s_slip_moments<T>, c->ph.np, 256, 0, c->g, c->ph, c->ps.x, c->ps.q, c->cells, c->ncells,
           c->real<T>(U0), c->real<T>(U1), c->real<T>(U2), c->slip);
    LAUNCH(c, p_slip_relax, pb, 128, 0, c->ph, c->ps, c->slip, 0);
    for (int iter = 0;;) {
        for (int d = 0; d < 3; d++) SPM_CUDA_CHECK(cudaMemsetAsync(c->real<T>(UP0 + d), 0, c->field_bytes(), c->st));
        LAUNCH(c, p_slip_droplet, pb, 128, 0, c->ph, c->slip);
        LAUNCH(c, s_slip_scatter<T>, sgrid, 128, 0, c->g, c->ph, c->ps.x, c->ps.q, c->cells, c->ncells, c->slip,
               c->real<T>(U0), c->real<T>(U1), c->real<T>(U2), c->real<T>(UP0), c->real<T>(UP1), c->real<T>(UP2));
        SPM_TRY(fft_fwd_box<T>(c, UP0, 3));
        LAUNCH(c, k_truncate_project<T>, c->grid_blocks(), 256, 0, c->g, c->cx<T>(UP0), c->cx<T>(UP1), c->cx<T>(UP2),
               1);
        SPM_TRY(fft_inv_box<T>(c, UP0, 3));
        LAUNCH(c, s_slip_force<T>, c->ph.np, 256, 0, c->g, c->ph, c->ps.x, c->cells, c->ncells, c->real<T>(UP0),
               c->real<T>(UP1), c->real<T>(UP2), c->slip);
        LAUNCH(c, p_velocity_slip, pb, 128, 0, c->ph, c->ps, c->slip, c->ts_dev, 0);
        iter++;
        LAUNCH(c, k_slip_converge, 1, 256, 0, c->ph, c->ps, c->slip, c->slip_eps);
        double eps = 0.0;
        SPM_CUDA_CHECK(cudaMemcpyAsync(&eps, c->slip_eps, sizeof(double), cudaMemcpyDeviceToHost, c->st));
        SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
        if (eps < c->P.slip_tol || iter == c->P.slip_iter) {
            LAUNCH(c, p_velocity_slip, pb, 128, 0, c->ph, c->ps, c->slip, c->ts_dev, 2);
            c->slip_iters = iter;
            break;
        }
        LAUNCH(c, p_slip_relax, pb, 128, 0, c->ph, c->ps, c->slip, iter);
        LAUNCH(c, p_velocity_slip, pb, 128, 0, c->ph, c->ps, c->slip, c->ts_dev, 1);
    }
    LAUNCH(c, r_add3<T>, c->grid_blocks(), 256, 0, c->g, c->real<T>(U0), c->real<T>(U1), c->real<T>(U2),
           c->real<T>(UP0), c->real<T>(UP1), c->real<T>(UP2));
    return SPM_OK;
}

// Mean-shear sustaining step of NS_solver_slavedEuler_Shear_PBC (fluid_solver.
// cxx:377-409): u of the updated zeta (every mode), u_x set on the shear
// planes (DC) or to the oscillating profile at t = ts dt (AC), zeta and uk_dc
// from it (U2zeta_k), then zeta truncated in place as Time_evolution_hydro
// does next (sp_3d_ns.cxx:54-56); a fresh zeta has no compensation residue.
template <typename T>
int shear_sustain(spm_ctx *c) {
    SPM_TRY(zeta_to_velocity<T>(c, 0));
    const double t   = (double)c->ts * c->ph.dt;
    const double amp = c->P.shear_ac ? cos(c->P.shear_frequency * t) : 1.0;
    LAUNCH(c, r_shear_sustain<T>, c->grid_blocks(), 256, 0, c->g, c->real<T>(U0), c->P.shear_ac, c->P.shear_rate,
           c->ph.L[1], amp, c->sns ? c->real<T>(A0) : (T *)nullptr);
    SPM_TRY(fft_fwd<T>(c, U0, 3));
    LAUNCH(c, k_u_to_zeta<T>, c->grid_blocks(), 256, 0, c->g, c->cx<T>(U0), c->cx<T>(U1), c->cx<T>(U2),
           c->cx<T>(Z0), c->cx<T>(Z1), c->uk_dc);
    LAUNCH(c, k_truncate2<T>, c->grid_blocks(), 256, 0, c->g, c->cx<T>(Z0), c->cx<T>(Z1));
    if (c->compensated()) {
        SPM_CUDA_CHECK(cudaMemsetAsync(c->real<T>(ZL0), 0, c->field_bytes(), c->st));
        SPM_CUDA_CHECK(cudaMemsetAsync(c->real<T>(ZL1), 0, c->field_bytes(), c->st));
    }
    return SPM_OK;
}

// The Shear_Navier_Stokes diagnostics of the step (spm_sns.cuh), after the
// rigidity force f is scattered into UP and before its projection: the
// density of the particles' current positions into A1, the row sums of
// u + f (U0 + UP0), fs rho (A0 holds the step's sustaining force) and
// rho (u + f), then the rate, strain and stresses.
template <typename T>
int shear_diagnostics(spm_ctx *c) {
    SPM_CUDA_CHECK(cudaMemsetAsync(c->real<T>(A1), 0, c->field_bytes(), c->st));
    if (c->ph.np > 0) {
        RhoWeights w{};
        const int  nsp = std::max(c->P.n_species, 1);
        for (int s = 0; s < 4; s++) {
            const double mr = s < nsp ? (nsp > 1 ? c->P.species_mass_ratio[s] : c->P.mass_ratio) : 1.0;
            w.drho[s]       = mr * c->P.rho - c->P.rho;
        }
        const dim3 sgrid((c->ncells + 127) / 128, c->ph.np);
        LAUNCH(c, s_rho_scatter<T>, sgrid, 128, 0, c->g, c->ph, c->ps.x, c->cells, c->ncells, c->real<T>(A1), w);
    }
    double *rows = c->sns + kSnsWords;
    LAUNCH(c, r_sns_rows<T>, c->g.ny, 256, 0, c->g, c->real<T>(U0), c->real<T>(UP0), c->real<T>(A0), c->real<T>(A1),
           c->P.rho, rows, 0);
    LAUNCH(c, k_sns_finish, 1, 512, 0, c->g, rows, c->sns, c->ph.dt, 0);
    return SPM_OK;
}

// AC: the inertia stress from u_x of the step's new zeta (U0 is free at the
// end of the step; A1 still holds the density).
template <typename T>
int shear_inertia(spm_ctx *c) {
    LAUNCH(c, (k_zeta_to_u<T, 0>), c->pw_grid(), 256, 0, c->g, c->cx<T>(Z0), c->cx<T>(Z1), c->uk_dc, c->cx<T>(U0),
           c->cx<T>(U1), c->cx<T>(U2), 0, c->fstride_c);
    SPM_TRY(fft_inv_packed<T>(c, U0, 1));
    double *rows = c->sns + kSnsWords;
    LAUNCH(c, r_sns_rows<T>, c->g.ny, 256, 0, c->g, c->real<T>(U0), c->real<T>(U0), c->real<T>(A0), c->real<T>(A1),
           c->P.rho, rows, 1);
    LAUNCH(c, k_sns_finish, 1, 512, 0, c->g, rows, c->sns, c->ph.dt, 1);
    return SPM_OK;
}

// Zero UP0, UP1, UP2 and PHIS of every run of L in one memset (the slots are
// consecutive; in a pool the span also covers free run slots).
template <typename T>
int clear_scatter_slots(spm_ctx *L) {
    const size_t nc = (size_t)(PHIS - UP0) * L->slot_stride_c + (size_t)L->fft_runs * L->fstride_c;
    SPM_CUDA_CHECK(cudaMemsetAsync(L->real<T>(UP0), 0, nc * 2 * sizeof(T), L->st));
    return SPM_OK;
}

// Rigidity projection of the step: the forward transform of f (scattered by
// s_f_scatter_cached, or up itself when u = 0 at initialisation), then the
// projection and the update of zeta and uk_dc closed in k space
// (k_project_add_curl).
template <typename T>
int rigidity_projection(spm_ctx *L) {
    int rc;
    if ((rc = z_pass<T>(L, UP0, 3, true, 1 << 30, L->g.kz_span())) != SPM_OK) return rc;
    if ((rc = fft_strided_pass<T, -1>(L, UP0, 3, 1, prune_forward(L->g, 1))) != SPM_OK) return rc;
    if ((rc = fft_strided_pass<T, -1>(L, UP0, 3, 0, prune_forward(L->g, 0))) != SPM_OK) return rc;
    PLAUNCH(L, "k_project_add_curl", box_bytes<T>(L, L->compensated() ? 11 : 7), (k_project_add_curl<T, 2>),
            L->box_grid(), 256, 0, L->g, L->cx<T>(UP0), L->cx<T>(UP1), L->cx<T>(UP2), L->cx<T>(Z0), L->cx<T>(Z1),
            L->uk_dc, L->fstride_c, L->zl<T>(0), L->zl<T>(1));
    return SPM_OK;
}

int particle_blocks(spm_ctx *c) { return (c->ph.np + 127) / 128; }

// The LJ forces of Force() (particle_solver.h:88-111) with the constant
// body force: through the cell list (particles binned per 16-DX cell, one warp
// per particle over the 27 neighbour cells) when the grid has at least one
// such cell per axis, as the reference's cell list needs; else the scan over
// all partners with the reference's pair multiplicity (p_forces).
int lj_forces(spm_ctx *c, const Phys &ph) {
    if (ph.np == 0) return SPM_OK;
    if (!c->lj_list || !lj_cell_list_applies(ph)) {
        PLAUNCH(c, "p_forces", 0.0, p_forces, (ph.np + 3) / 4, 128, 0, ph, c->ps, 0, 0.0,
                c->rigid() ? c->rg.rid : nullptr, c->rigid() ? c->rg.f_lo : nullptr, (const double *)nullptr);
        return SPM_OK;
    }
    const int ncell   = lj_ncell(ph);
    int      *count   = c->lj_list;
    int      *cell_of = count + ncell;
    int      *bins    = cell_of + ph.np;
    if (ph.lj_on && ph.janus_prop != 3) {
        SPM_CUDA_CHECK(cudaMemsetAsync(count, 0, (size_t)ncell * sizeof(int), c->st));
        PLAUNCH(c, "p_cells_bin", 0.0, p_cells_bin, (ph.np + 127) / 128, 128, 0, ph, c->ps.x, count, cell_of, bins,
                c->err);
    }
    PLAUNCH(c, "p_forces_cells", 0.0, p_forces_cells, (ph.np + 3) / 4, 128, 0, ph, c->ps, count, cell_of, bins,
            c->rigid() ? c->rg.rid : nullptr, c->rigid() ? c->rg.f_lo : nullptr);
    return SPM_OK;
}

// Zeta uploaded by the host: truncate it once (the reference truncates zeta in
// place at the start of NS_solver_slavedEuler; the step's retained-box
// kernels leave the other modes as they are).
template <typename T>
int truncate_if_dirty(spm_ctx *c) {
    if (!c->zeta_dirty) return SPM_OK;
    LAUNCH(c, k_truncate2<T>, c->grid_blocks(), 256, 0, c->g, c->cx<T>(Z0), c->cx<T>(Z1));
    if (c->compensated()) LAUNCH(c, k_truncate2<T>, c->grid_blocks(), 256, 0, c->g, c->cx<T>(ZL0), c->cx<T>(ZL1));
    c->zeta_dirty = false;
    return SPM_OK;
}

// Time_evolution_hydro (sp_3d_ns.cxx:41-194), Navier_Stokes with free
// spheres.  L batches the grid stages of runs R[0..nr), which are L's runs in
// order (L is the run itself for a single context); particle kernels go to
// each run on the shared stream.
template <typename T>
int step_ns_runs(spm_ctx *L, spm_ctx *const *R, int nr) {
    int rc;
    for (int r = 0; r < nr; r++)
        if ((rc = truncate_if_dirty<T>(R[r])) != SPM_OK) return rc;
    // fork: position update (Euler/AB2 from the previous velocities), phi
    // scatter and Lennard-Jones forces need nothing from this step's fluid
    // solve; they run on the side stream while the main stream advances zeta.
    // The scatter slots are free here (the previous step consumed them).
    const cudaStream_t side = L->overlap ? L->side : L->st;
    if (L->overlap) {
        SPM_CUDA_CHECK(cudaEventRecord(L->ev_fork, L->st));
        SPM_CUDA_CHECK(cudaStreamWaitEvent(side, L->ev_fork, 0));
    }
    {
        const cudaStream_t main_st = L->st;
        L->st                      = side;
        for (int r = 0; r < nr; r++) R[r]->st = side;
        rc = clear_scatter_slots<T>(L);
        for (int r = 0; r < nr && rc == SPM_OK; r++) {
            spm_ctx *c = R[r];
            if (c->ph.np == 0) continue;
            auto side_work = [&]() -> int {
                if (c->rigid())
                    PLAUNCH(c, "r_position", 0.0, r_position, c->rg.nb, 128, 0, c->ph, c->ps, c->rg, c->ts_dev, 0, 0.0,
                            (const double *)nullptr);
                else
                    PLAUNCH(c, "p_position", 0.0, p_position, particle_blocks(c), 128, 0, c->ph, c->ps, c->ts_dev, 1);
                const dim3 sgrid((c->ncells + 127) / 128, c->ph.np);
                PLAUNCH(c, "s_phi_scatter_cache", stencil_bytes<T>(c, 0), s_phi_scatter_cache<T>, sgrid, 128, 0, c->g,
                        c->ph, c->ps.x, c->cells, c->ncells, c->real<T>(PHIS), c->err, c->sc_idx, c->sc_w);
                SPM_TRY(lj_forces(c, c->ph));
                return SPM_OK;
            };
            rc = side_work();
        }
        L->st = main_st;
        for (int r = 0; r < nr; r++) R[r]->st = main_st;
        if (rc != SPM_OK) return rc;
    }
    if (L->overlap) SPM_CUDA_CHECK(cudaEventRecord(L->ev_join, side));
    // FP64: the update writes u_hat of the new zeta as well (unless the shear
    // sustaining step changes zeta in between), one k_zeta_to_u fewer.  Measured
    // on B200 at 256^3 the fused update took 82 us against 60 + 37 us; in FP32 it
    // took 73 us against 44 + 25 us, so FP32 keeps the two kernels.
    const bool fuse_u = L->P.equation != SPM_EQ_SHEAR_NAVIER_STOKES && L->fp64();
    if ((rc = ns_solver<T>(L, fuse_u)) != SPM_OK) return rc;
    if (L->P.equation == SPM_EQ_SHEAR_NAVIER_STOKES) SPM_TRY(shear_sustain<T>(L));  // lone runs only
    LAUNCH(L, k_fix_cell, (nr + 127) / 128, 128, 0, L->rw, nr);
    if ((rc = zeta_to_velocity<T>(L, 1, fuse_u)) != SPM_OK) return rc;
    if (L->overlap) SPM_CUDA_CHECK(cudaStreamWaitEvent(L->st, L->ev_join, 0));  // join
    for (int r = 0; r < nr; r++) {
        spm_ctx *c = R[r];
        if (c->ph.np == 0) continue;
        PLAUNCH(c, "s_hydro_force_cached", stencil_bytes<T>(c, 1), s_hydro_force_cached<T>, c->ph.np, 256, 0, c->g,
                c->ph, c->ps.x, c->ps.v, c->ps.omega, c->cells, c->ncells, c->sc_idx, c->sc_w, c->real<T>(PHIS),
                c->real<T>(U0), c->real<T>(U1), c->real<T>(U2), c->ps.f_hydro, c->ps.torque_hydro);
        if (c->rigid()) {
            LAUNCH(c, r_collect, c->rg.nb, 128, 0, c->ps, c->rg, c->rfree, 0);
            LAUNCH(c, r_velocity, c->rg.nb, 128, 0, c->ph, c->ps, c->rg, c->rfree, c->ts_dev, 0, 0.0,
                   (const double *)nullptr);
        } else if (c->ph.janus_prop == SPM_JANUS_SQUIRMER) {
            SPM_TRY(slip_loop<T>(c));  // lone runs only; leaves the slip field in UP
        } else {
            PLAUNCH(c, "p_velocity", 0.0, p_velocity, particle_blocks(c), 128, 0, c->ph, c->ps, c->ts_dev);
        }
        // obstacles draw no noise (fluct.cxx:23)
        if (c->P.kbt > 0.0 && c->ph.janus_prop != SPM_JANUS_OBSTACLE) {
            LAUNCH(c, p_thermostat, 1, kThermoThreads, 0, c->ph, c->ps, c->mt, c->rigid() ? c->rg.noise : nullptr);
            if (c->rigid()) LAUNCH(c, r_thermostat, c->rg.nb, 128, 0, c->ph, c->ps, c->rg, c->rfree);
        }
        const dim3 sgrid((c->ncells + 127) / 128, c->ph.np);
        PLAUNCH(c, "s_f_scatter_cached", stencil_bytes<T>(c, 2), s_f_scatter_cached<T>, sgrid, 128, 0, c->g, c->ph,
                c->ps.x, c->ps.v, c->ps.omega, c->cells, c->ncells, c->sc_idx, c->sc_w, c->real<T>(PHIS),
                c->real<T>(U0), c->real<T>(U1), c->real<T>(U2), c->real<T>(UP0), c->real<T>(UP1), c->real<T>(UP2));
    }
    if (L->sns) SPM_TRY(shear_diagnostics<T>(L));  // lone Shear_Navier_Stokes runs
    if ((rc = rigidity_projection<T>(L)) != SPM_OK) return rc;
    if (L->sns && L->P.shear_ac) SPM_TRY(shear_inertia<T>(L));
    LAUNCH(L, k_ts_advance, (nr + 127) / 128, 128, 0, L->rw, nr);
    for (int r = 0; r < nr; r++) {
        R[r]->ts++;
        R[r]->time += R[r]->ph.dt;
    }
    return SPM_OK;
}
template <typename T>
int step_ns(spm_ctx *c) {
    return step_ns_runs<T>(c, &c, 1);
}

template <typename T>
int initialize_impl(spm_ctx *c) {
    int rc;
    for (int sl = 0; sl < c->nslots; sl++) SPM_CUDA_CHECK(cudaMemsetAsync(c->real<T>(sl), 0, c->field_bytes(), c->st));
    SPM_CUDA_CHECK(cudaMemsetAsync(c->ts_dev, 0, sizeof(int), c->st));
    LAUNCH(c, k_zero3, 1, 32, 0, c->uk_dc);
    if ((rc = phi_sum_scatter<T>(c)) != SPM_OK) return rc;
    if ((rc = up_scatter<T>(c)) != SPM_OK) return rc;
    // u = Zeta_k2u(zeta = 0) = 0
    if ((rc = zeta_to_velocity<T>(c, 1)) != SPM_OK) return rc;
    if ((rc = rigidity_projection<T>(c)) != SPM_OK) return rc;
    LAUNCH(c, k_zero3, 1, 32, 0, c->uk_dc);
    if (c->sns) SPM_CUDA_CHECK(cudaMemsetAsync(c->sns, 0, kSnsWords * sizeof(double), c->st));
    // shear runs start with v_x = omega_z = 0 (init_particle.cxx:768-781)
    if ((c->le.enabled || c->P.equation == SPM_EQ_SHEAR_NAVIER_STOKES) && c->ph.np > 0)
        LAUNCH(c, p_le_zero_vx, particle_blocks(c), 128, 0, c->ph, c->ps);
    c->ts   = 0;
    c->time = 0.0;
    return SPM_OK;
}

}  // namespace
#include "spm_le_step.inc"
#include "spm_electrolyte.inc"
namespace {

template <typename T>
int step_impl(spm_ctx *c) {
    if (c->P.equation == SPM_EQ_LEES_EDWARDS) return step_le_impl<T>(c);
    if (c->P.equation == SPM_EQ_ELECTROLYTE) {
        const int rc = step_el<T>(c);
        if (rc != SPM_OK) return rc;
        c->ts++;
        c->time += c->ph.dt;
        return SPM_OK;
    }
    return step_ns<T>(c);
}

// One Navier_Stokes step from the run's captured graph.  The first call
// captures step_ns (the side-stream fork and join included) and restores the
// host counters the capture advanced; every call replays the graph and
// advances them.  Host-set zeta is truncated before, outside the graph.
template <typename T>
int step_graphed(spm_ctx *c) {
    int rc;
    if ((rc = truncate_if_dirty<T>(c)) != SPM_OK) return rc;
    if (!c->step_exec) {
        const int       ts = c->ts;
        const double    tm = c->time;
        const long long ln = c->launches;
        SPM_CUDA_CHECK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
        rc              = c->el.enabled ? step_el<T>(c) : step_ns<T>(c);
        cudaGraph_t g   = nullptr;
        cudaError_t e   = cudaStreamEndCapture(c->st, &g);
        c->step_kernels = c->launches - ln;
        c->ts           = ts;
        c->time         = tm;
        c->launches     = ln;
        if (rc != SPM_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return rc != SPM_OK ? rc : fail(SPM_ERR_CUDA, std::string("step capture: ") + cudaGetErrorString(e));
        }
        if ((e = cudaGraphInstantiate(&c->step_exec, g, 0)) != cudaSuccess) {
            cudaGraphDestroy(g);
            return fail(SPM_ERR_CUDA, std::string("step graph instantiate: ") + cudaGetErrorString(e));
        }
        c->step_graph = g;
    }
    SPM_CUDA_CHECK(cudaGraphLaunch(c->step_exec, c->st));
    c->launches += c->step_kernels;
    c->ts++;
    c->time += c->ph.dt;
    return SPM_OK;
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

// Compensated zeta of an FP32-mixed run: upload x as hi = (float)x and
// lo = (float)(x - hi); download hi + lo.
int upload_field_split(spm_ctx *c, int slot_hi, int slot_lo, const double *h) {
    std::vector<float> hi(c->fstride_c * 2, 0.0f), lo(c->fstride_c * 2, 0.0f);
    const size_t rows = (size_t)c->g.nx * c->g.ny;
    for (size_t r = 0; r < rows; r++)
        for (int k = 0; k < 2 * c->g.hnz; k++) {
            const double x = h[r * 2 * c->g.hnz + k];
            const float  a = (float)x;
            hi[r * 2 * c->g.hnzp + k] = a;
            lo[r * 2 * c->g.hnzp + k] = (float)(x - (double)a);
        }
    SPM_CUDA_CHECK(cudaMemcpyAsync(c->real<float>(slot_hi), hi.data(), hi.size() * sizeof(float),
                                   cudaMemcpyHostToDevice, c->st));
    SPM_CUDA_CHECK(cudaMemcpyAsync(c->real<float>(slot_lo), lo.data(), lo.size() * sizeof(float),
                                   cudaMemcpyHostToDevice, c->st));
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    return SPM_OK;
}
int download_field_sum(spm_ctx *c, int slot_hi, int slot_lo, double *h) {
    std::vector<float> hi(c->fstride_c * 2), lo(c->fstride_c * 2);
    SPM_CUDA_CHECK(cudaMemcpyAsync(hi.data(), c->real<float>(slot_hi), hi.size() * sizeof(float),
                                   cudaMemcpyDeviceToHost, c->st));
    SPM_CUDA_CHECK(cudaMemcpyAsync(lo.data(), c->real<float>(slot_lo), lo.size() * sizeof(float),
                                   cudaMemcpyDeviceToHost, c->st));
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    const size_t rows = (size_t)c->g.nx * c->g.ny;
    for (size_t r = 0; r < rows; r++)
        for (int k = 0; k < 2 * c->g.hnz; k++)
            h[r * 2 * c->g.hnz + k] = (double)hi[r * 2 * c->g.hnzp + k] + (double)lo[r * 2 * c->g.hnzp + k];
    return SPM_OK;
}

// Particle records <-> device state.  The records (SPM_PARTICLE_WORDS doubles
// each) travel as one block between the caller's buffer and a device staging
// buffer; the AoS <-> SoA reordering runs on the device.  Record offsets of
// the twelve 3-vectors in the order of the device arrays (see spm_create),
// then q (18) and q_old (22).
__constant__ int kRecVec[12] = {0, 3, 6, 9, 12, 15, 26, 29, 32, 35, 38, 41};

__global__ void k_records_in(const double *__restrict__ rec, double *__restrict__ pbuf, PState s, int np,
                             int normalize_q) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= np) return;
    const double *r = rec + (size_t)n * SPM_PARTICLE_WORDS;
    double        q[4], qo[4];
    for (int k = 0; k < 4; k++) q[k] = r[18 + k], qo[k] = r[22 + k];
    if (normalize_q) {
        const double nn = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        for (int k = 0; k < 4; k++) q[k] *= 1.0 / nn;
        for (int k = 0; k < 4; k++) qo[k] = q[k];
    }
    for (int a = 0; a < 12; a++)
        for (int d = 0; d < 3; d++) pbuf[(size_t)a * np * 3 + 3 * n + d] = r[kRecVec[a] + d];
    for (int k = 0; k < 4; k++) {
        pbuf[(size_t)12 * np * 3 + 4 * n + k]                    = q[k];
        pbuf[(size_t)12 * np * 3 + (size_t)np * 4 + 4 * n + k] = qo[k];
    }
    // x_previous, torque_r, torque_r_previous, lj_stress, mdf start at x / zero
    for (int d = 0; d < 3; d++) {
        s.x_previous[3 * n + d]        = r[d];
        s.torque_r[3 * n + d]          = 0.0;
        s.torque_r_previous[3 * n + d] = 0.0;
        s.mdf[3 * n + d]               = 0.0;
    }
    s.lj_stress[n] = 0.0;
}

__global__ void k_records_out(const double *__restrict__ pbuf, double *__restrict__ rec, int np) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= np) return;
    double *r = rec + (size_t)n * SPM_PARTICLE_WORDS;
    for (int a = 0; a < 12; a++)
        for (int d = 0; d < 3; d++) r[kRecVec[a] + d] = pbuf[(size_t)a * np * 3 + 3 * n + d];
    for (int k = 0; k < 4; k++) {
        r[18 + k] = pbuf[(size_t)12 * np * 3 + 4 * n + k];
        r[22 + k] = pbuf[(size_t)12 * np * 3 + (size_t)np * 4 + 4 * n + k];
    }
}

// Returns once the records have been read from `rec` (the caller may reuse
// the buffer); the reordering kernel stays queued ahead of the next step.
int upload_particles(spm_ctx *c, const double *rec, bool normalize_q) {
    const int np = c->ph.np;
    if (np == 0) return SPM_OK;
    SPM_CUDA_CHECK(cudaMemcpyAsync(c->rec_stage, rec, (size_t)np * SPM_PARTICLE_WORDS * sizeof(double),
                                   cudaMemcpyHostToDevice, c->st));
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    LAUNCH(c, k_records_in, (np + 127) / 128, 128, 0, c->rec_stage, c->pbuf, c->ps, np, normalize_q ? 1 : 0);
    return SPM_OK;
}

int download_particles(spm_ctx *c, double *rec) {
    const int np = c->ph.np;
    if (np == 0) return SPM_OK;
    LAUNCH(c, k_records_out, (np + 127) / 128, 128, 0, c->pbuf, c->rec_stage, np);
    SPM_CUDA_CHECK(cudaMemcpyAsync(rec, c->rec_stage, (size_t)np * SPM_PARTICLE_WORDS * sizeof(double),
                                   cudaMemcpyDeviceToHost, c->st));
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    return SPM_OK;
}

#include "spm_rigid.inc"

void avs_release(spm_ctx *c);
void udf_out_release(spm_ctx *c);

// Electrolyte run constants from the parameters (Init_rho_ion,
// operate_electrolyte.cxx:667-720, 490-520; Elementary_charge = 1,
// input.cxx:293; Angular_Frequency = PI2 Frequency, input.cxx:514).
void el_init_state(ELState &el, const spm_params &p) {
    const double e = 1.0;
    el.enabled     = 1;
    el.nspec       = p.salt ? 2 : 1;
    el.iepsilon    = 1.0 / p.dielectric;
    const int nsp  = p.n_species > 1 ? p.n_species : 1;
    auto      cnt  = [&](int s) { return nsp > 1 ? p.species_count[s] : p.n_particles; };
    auto      chg  = [&](int s) { return nsp > 1 ? p.species_surface_charge[s] : p.surface_charge; };
    el.qe          = chg(0) * e;
    el.abs_q       = 0.0;
    double surface_ion_number = 0.0;
    for (int s = 0; s < nsp; s++) {
        for (int n = 0; n < cnt(s); n++) el.abs_q += fabs(chg(s) * e);
        surface_ion_number -= chg(s) * cnt(s);
    }
    el.surface_ion_number           = surface_ion_number;
    el.init_pb                      = p.init_pb;
    for (int n = 0; n < el.nspec; n++) {
        el.val_e[n] = p.valency[n] * e;
        el.ons[n]   = p.onsager[n];
    }
    if (el.nspec == 1) {
        el.counterion_number = surface_ion_number / p.valency[0];
    } else {
        // counterions of every species by the sign of its charge (Set_uniform_ion_charge_density_salt,
        // operate_electrolyte.cxx:498-507)
        el.ion_number[0] = el.ion_number[1] = 0.0;
        for (int s = 0; s < nsp; s++) {
            const double qn = chg(s) * (double)cnt(s);
            if (chg(s) < 0.)
                el.ion_number[0] += fabs(qn / p.valency[0]);
            else if (chg(s) > 0.)
                el.ion_number[1] += fabs(qn / p.valency[1]);
        }
        const double rho_inf = p.kbt * p.dielectric / ((e * p.debye_length) * (e * p.debye_length));
        el.rho_inf[0]        = rho_inf / (p.valency[0] * (p.valency[0] - p.valency[1]));
        el.rho_inf[1]        = -rho_inf / (p.valency[1] * (p.valency[0] - p.valency[1]));
    }
    el.e_on  = p.e_field != 0;
    el.e_ac  = p.e_field == 2;
    for (int d = 0; d < 3; d++) el.e_ext[d] = el.e_on ? p.e_ext[d] : 0.0;
    el.e_omega = 2. * M_PI * p.e_frequency;
}

void destroy_ctx(spm_ctx *c) {
    if (!c) return;
    avs_release(c);
    udf_out_release(c);
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->step_exec) cudaGraphExecDestroy(c->step_exec);
    if (c->step_graph) cudaGraphDestroy(c->step_graph);
    c->plan64.destroy();
    c->plan32.destroy();
    if (c->owns_arena) dev_free(c->arena);
    if (c->owns_rw) dev_free(c->rw);
    dev_free(c->cells);
    dev_free(c->lj_list);
    dev_free(c->sc_idx);
    dev_free(c->sc_w);
    dev_free(c->pbuf);
    dev_free(c->rec_stage);
    dev_free(c->mt);
    dev_free(c->le.dev);
    dev_free(c->le.ppart);
    dev_free(c->le.partial);
    dev_free(c->el.dev);
    dev_free(c->el.partial);
    dev_free(c->slip);
    dev_free(c->slip_eps);
    dev_free(c->sns);
    dev_free(c->rg_ibuf);
    dev_free(c->rg_dbuf);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->own_stream && c->st) cudaStreamDestroy(c->st);
    delete c;
}

// Creates a context of one of three kinds:
//  - a lone run (pool_cap == 0, lead == nullptr): own arena of NSLOT fields,
//    own RunWords and FFT plan;
//  - a pool lead (pool_cap > 0, lead == nullptr): no particles; arena of
//    NSLOT x pool_cap fields, slot-major, RunWords[pool_cap + 1] (the last one
//    holds the lead's own error word) and the FFT plan the pool's runs share;
//  - a pool run (lead != nullptr) at run slot `slot` of the lead's arena.
int create_ctx(const spm_params &p, cudaStream_t stream, int pool_cap, spm_ctx *lead, int slot, spm_ctx **out) {
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SPM_ERR_NO_DEVICE, "no CUDA device visible");
    spm_ctx *c = new spm_ctx();
    c->P       = p;
    if (pool_cap > 0) c->P.n_particles = 0;
    int rc = derive(c->P, c->g, c->ph);
    if (rc != SPM_OK) {
        delete c;
        return rc;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (stream) {
        c->st = stream;
    } else {
        if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return fail(SPM_ERR_CUDA, "stream creation failed");
        }
        c->own_stream = true;
    }
    if (!lead && (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
                  cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
                  cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess)) {
        destroy_ctx(c);
        return fail(SPM_ERR_CUDA, "side stream / events");
    }
    c->fstride_c    = (size_t)c->g.nx * c->g.ny * c->g.hnzp;
    const int nslot = slots_for(p);
    c->nslots       = nslot;
    {
        const char *nt = getenv("SPM_NO_TMA");
        c->use_tma     = !(nt && nt[0] == '1');
        const char *no = getenv("SPM_NO_OVERLAP");
        c->overlap     = !(no && no[0] == '1');
        const char *ng = getenv("SPM_NO_GRAPH");
        c->use_graph   = !(ng && ng[0] == '1');
    }
    cudaError_t e = cudaSuccess;
    if (lead) {
        c->owns_arena    = false;
        c->owns_rw       = false;
        c->slot_stride_c = lead->slot_stride_c;
        const size_t es  = c->elem_bytes();
        c->arena         = static_cast<char *>(lead->arena) + (size_t)slot * c->fstride_c * 2 * es;
        c->rw            = lead->rw + slot;
        c->pp64          = lead->pp64;
        c->pp32          = lead->pp32;
        c->use_tma       = lead->use_tma;
    } else {
        const int nruns  = pool_cap > 0 ? pool_cap : 1;
        c->slot_stride_c = (size_t)nruns * c->fstride_c;
        e                = dev_alloc(&c->arena, (size_t)nslot * nruns * c->field_bytes());
        if (e != cudaSuccess) {
            destroy_ctx(c);
            return fail(SPM_ERR_NOMEM, std::string("field arena: ") + cudaGetErrorString(e));
        }
        e = dev_alloc((void **)&c->rw, (size_t)(pool_cap > 0 ? pool_cap + 1 : 1) * sizeof(RunWords));
        if (e != cudaSuccess) {
            destroy_ctx(c);
            return fail(SPM_ERR_NOMEM, "run words");
        }
        e = c->fp64() ? c->plan64.create(c->g) : c->plan32.create(c->g);
        c->plan64.sm_count = c->plan32.sm_count = c->sm_count;
        if (e != cudaSuccess) {
            destroy_ctx(c);
            return fail(SPM_ERR_CUDA, std::string("FFT plan: ") + cudaGetErrorString(e));
        }
        if (pool_cap > 0) {
            cudaMemset(c->rw, 0, (size_t)(pool_cap + 1) * sizeof(RunWords));
            c->uk_dc  = c->rw->uk_dc;
            c->ts_dev = &c->rw->ts;
            c->err    = &c->rw[pool_cap].err;
            c->plan64.err = c->plan32.err = c->err;
            if (cudaDeviceSynchronize() != cudaSuccess) {
                destroy_ctx(c);
                return fail(SPM_ERR_CUDA, "pool lead setup");
            }
            *out = c;
            return SPM_OK;
        }
    }
    set_run_words(c);
    if (!lead) c->plan64.err = c->plan32.err = c->err;
    std::vector<int> cells = sekibun(p);
    c->ncells              = (int)cells.size();
    const int np           = std::max(p.n_particles, 1);
    if (dev_alloc((void **)&c->cells, cells.size() * sizeof(int)) != cudaSuccess ||
        dev_alloc((void **)&c->pbuf, (size_t)np * kPWords * sizeof(double)) != cudaSuccess ||
        dev_alloc((void **)&c->rec_stage, (size_t)std::max(np, 1) * SPM_PARTICLE_WORDS * sizeof(double)) != cudaSuccess ||
        dev_alloc((void **)&c->mt, 625 * sizeof(unsigned int)) != cudaSuccess ||
        (lj_cell_list_applies(c->ph) &&
         dev_alloc((void **)&c->lj_list, ((size_t)lj_ncell(c->ph) * (1 + kLjBin) + np) * sizeof(int)) != cudaSuccess)) {
        destroy_ctx(c);
        return fail(SPM_ERR_NOMEM, "small device buffers");
    }
    if ((p.equation == SPM_EQ_NAVIER_STOKES || p.equation == SPM_EQ_SHEAR_NAVIER_STOKES) && p.n_particles > 0) {
        const size_t nsc = (size_t)p.n_particles * cells.size();
        if (dev_alloc((void **)&c->sc_idx, nsc * sizeof(int)) != cudaSuccess ||
            dev_alloc((void **)&c->sc_w, nsc * sizeof(double)) != cudaSuccess) {
            destroy_ctx(c);
            return fail(SPM_ERR_NOMEM, "stencil cache");
        }
    }
    cudaMemcpy(c->cells, cells.data(), cells.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemset(c->pbuf, 0, (size_t)np * kPWords * sizeof(double));
    if (c->rigid() && (rc = rigid_alloc(c)) != SPM_OK) {
        destroy_ctx(c);
        return rc;
    }
    unsigned int mt[625];
    mt_init(p.mt_seed, mt);
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
    le_init(c->le, c->g, c->ph, p);
    if (p.equation == SPM_EQ_SHEAR_NAVIER_STOKES && pool_cap == 0 && !lead &&
        dev_alloc((void **)&c->sns, ((size_t)kSnsWords + 3 * (size_t)c->g.ny) * sizeof(double)) != cudaSuccess) {
        destroy_ctx(c);
        return fail(SPM_ERR_NOMEM, "shear diagnostics buffer");
    }
    if (p.janus_propulsion == SPM_JANUS_SQUIRMER) {
        if (dev_alloc((void **)&c->slip, (size_t)std::max(np, 1) * kSlipWords * sizeof(double)) != cudaSuccess ||
            dev_alloc((void **)&c->slip_eps, sizeof(double)) != cudaSuccess) {
            destroy_ctx(c);
            return fail(SPM_ERR_NOMEM, "slip buffers");
        }
        cudaMemset(c->slip, 0, (size_t)std::max(np, 1) * kSlipWords * sizeof(double));
    }
    if (p.equation == SPM_EQ_ELECTROLYTE) {
        el_init_state(c->el, p);
        if (dev_alloc((void **)&c->el.dev, kElScalars * sizeof(double)) != cudaSuccess ||
            dev_alloc((void **)&c->el.partial, (size_t)c->grid_blocks() * sizeof(double)) != cudaSuccess) {
            destroy_ctx(c);
            return fail(SPM_ERR_NOMEM, "Electrolyte buffers");
        }
        cudaMemset(c->el.dev, 0, kElScalars * sizeof(double));
    }
    if (c->le.enabled) {
        if (dev_alloc((void **)&c->le.dev, sizeof(LEDev)) != cudaSuccess ||
            dev_alloc((void **)&c->le.ppart, (size_t)np * kLePart * sizeof(double)) != cudaSuccess ||
            dev_alloc((void **)&c->le.partial, (size_t)c->grid_blocks() * sizeof(double)) != cudaSuccess) {
            destroy_ctx(c);
            return fail(SPM_ERR_NOMEM, "Lees-Edwards buffers");
        }
        cudaMemset(c->le.dev, 0, sizeof(LEDev));
    }
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        destroy_ctx(c);
        return fail(SPM_ERR_CUDA, std::string("create: ") + cudaGetErrorString(e));
    }
    *out = c;
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
    p->slip_tol  = 1e-5;
    p->slip_iter = 100;
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
    const size_t nslot = (size_t)slots_for(*p);
    const bool   ns = p->equation == SPM_EQ_NAVIER_STOKES || p->equation == SPM_EQ_SHEAR_NAVIER_STOKES;
    const size_t sc = ns ? (size_t)p->n_particles * sekibun(*p).size() * 12 : 0;
    *bytes = nslot * fld + (size_t)std::max(p->n_particles, 1) * kPWords * 8 + sc + 64 * 1024;
    return SPM_OK;
}

size_t spm_params_size(void) { return sizeof(spm_params); }

int spm_create(const spm_params *p, void *stream, spm_ctx **out) {
    if (!p || !out) return fail(SPM_ERR_ARG, "null argument");
    return create_ctx(*p, static_cast<cudaStream_t>(stream), 0, nullptr, 0, out);
}

int spm_destroy(spm_ctx *c) {
    if (!c) return SPM_OK;
    if (c->pool) return fail(SPM_ERR_ARG, "the run belongs to a pool: release it with spm_pool_release");
    destroy_ctx(c);
    return SPM_OK;
}

int spm_initialize(spm_ctx *c, const double *particles_host) {
    if (!c) return fail(SPM_ERR_ARG, "null context");
    if (c->ph.np > 0 && !particles_host) return fail(SPM_ERR_ARG, "particle records required");
    int rc;
    if (c->rigid()) {  // bodies set up from the beads as given (Init_Particle's rigid branch)
        std::vector<double> rec(particles_host, particles_host + (size_t)c->ph.np * SPM_PARTICLE_WORDS);
        rc = c->fp64() ? rigid_setup<double>(c, rec) : rigid_setup<float>(c, rec);
    } else {
        rc = upload_particles(c, particles_host, true);
    }
    if (rc != SPM_OK) return rc;
    le_reset(c->le);
    rc = c->fp64() ? initialize_impl<double>(c) : initialize_impl<float>(c);
    if (rc != SPM_OK) return rc;
    if (c->el.enabled && (rc = c->fp64() ? el_init_profile<double>(c) : el_init_profile<float>(c)) != SPM_OK)
        return rc;
    return check_device_error(c);
}

int spm_step(spm_ctx *c, int nsteps) {
    if (!c || nsteps < 0) return fail(SPM_ERR_ARG, "bad argument");
    // graph replay: lone Navier_Stokes runs (the slip loop of squirmers reads
    // its convergence on the host) and Electrolyte runs once their ion fields
    // are inside the 2/3 box (after the first step), not while a test switch
    // is armed
    const bool graphable = c->use_graph && !c->pool && !c->prof_on && c->P.janus_propulsion != SPM_JANUS_SQUIRMER &&
                           c->pp64->skip_loads == 0 && c->pp32->skip_loads == 0;
    for (int i = 0; i < nsteps; i++) {
        const bool el    = c->P.equation == SPM_EQ_ELECTROLYTE;
        const bool graph = graphable && (c->P.equation == SPM_EQ_NAVIER_STOKES || (el && c->el.conc_in_box));
        if (el) SPM_TRY(el_sync_time(c));
        int rc = graph ? (c->fp64() ? step_graphed<double>(c) : step_graphed<float>(c))
                       : (c->fp64() ? step_impl<double>(c) : step_impl<float>(c));
        if (rc != SPM_OK) return rc;
        if (el) c->el.time_dev = c->time;  // the step advanced the device's time word alike
    }
    return SPM_OK;
}

// Drops the captured step graph (its kernels hold launch parameters that
// changed); the next graphed step captures a new one.
static int drop_step_graph(spm_ctx *c) {
    if (!c->step_exec) return SPM_OK;
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    cudaGraphExecDestroy(c->step_exec);
    if (c->step_graph) cudaGraphDestroy(c->step_graph);
    c->step_exec  = nullptr;
    c->step_graph = nullptr;
    return SPM_OK;
}

int spm_set_wait_limit(spm_ctx *c, double seconds) {
    if (!c || !(seconds > 0.0) || seconds > 60.0) return fail(SPM_ERR_ARG, "wait limit must be in (0, 60] s");
    const unsigned long long ns = (unsigned long long)(seconds * 1e9) > 0 ? (unsigned long long)(seconds * 1e9) : 1;
    c->pp64->wait_ns = c->pp32->wait_ns = ns;
    return drop_step_graph(c);
}

int spm_debug_skip_tma_loads(spm_ctx *c, int launches) {
    if (!c || launches < 0) return fail(SPM_ERR_ARG, "bad argument");
    c->pp64->skip_loads = c->pp32->skip_loads = launches;
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

int spm_rigid_count(spm_ctx *c, int *n) {
    if (!c || !n) return fail(SPM_ERR_ARG, "bad argument");
    *n = c->rigid() ? c->rg.nb : 0;
    return SPM_OK;
}

int spm_get_rigid(spm_ctx *c, double *bodies) {
    if (!c || !c->rigid() || (!bodies && c->rg.nb > 0)) return fail(SPM_ERR_ARG, "bad argument (no rigid bodies)");
    int rc = spm_synchronize(c);
    if (rc != SPM_OK) return rc;
    return rigid_download(c, bodies);
}

int spm_get_rigid_state(spm_ctx *c, double *bodies, double *offsets) {
    if (!c || !c->rigid() || !bodies || !offsets) return fail(SPM_ERR_ARG, "bad argument (no rigid bodies)");
    int rc = spm_synchronize(c);
    if (rc != SPM_OK) return rc;
    return rigid_state_io(c, bodies, offsets, true);
}

int spm_set_rigid_state(spm_ctx *c, const double *bodies, const double *offsets) {
    if (!c || !c->rigid() || !bodies || !offsets) return fail(SPM_ERR_ARG, "bad argument (no rigid bodies)");
    int rc = spm_synchronize(c);
    if (rc != SPM_OK) return rc;
    return rigid_state_io(c, const_cast<double *>(bodies), const_cast<double *>(offsets), false);
}

int spm_set_particles(spm_ctx *c, const double *rec) {
    if (!c || (!rec && c->ph.np > 0)) return fail(SPM_ERR_ARG, "bad argument");
    return upload_particles(c, rec, false);
}

int spm_get_zeta(spm_ctx *c, double *z0, double *z1, double uk_dc[3]) {
    if (!c || !z0 || !z1 || !uk_dc) return fail(SPM_ERR_ARG, "bad argument");
    int rc;
    if ((rc = spm_synchronize(c)) != SPM_OK) return rc;
    if (c->compensated()) {
        if ((rc = download_field_sum(c, Z0, ZL0, z0)) != SPM_OK) return rc;
        if ((rc = download_field_sum(c, Z1, ZL1, z1)) != SPM_OK) return rc;
    } else {
        if ((rc = download_field(c, Z0, z0)) != SPM_OK) return rc;
        if ((rc = download_field(c, Z1, z1)) != SPM_OK) return rc;
    }
    SPM_CUDA_CHECK(cudaMemcpy(uk_dc, c->uk_dc, 3 * sizeof(double), cudaMemcpyDeviceToHost));
    return SPM_OK;
}

int spm_set_zeta(spm_ctx *c, const double *z0, const double *z1, const double uk_dc[3]) {
    if (!c || !z0 || !z1 || !uk_dc) return fail(SPM_ERR_ARG, "bad argument");
    int rc;
    if (c->compensated()) {
        if ((rc = upload_field_split(c, Z0, ZL0, z0)) != SPM_OK) return rc;
        if ((rc = upload_field_split(c, Z1, ZL1, z1)) != SPM_OK) return rc;
    } else {
        if ((rc = upload_field(c, Z0, z0)) != SPM_OK) return rc;
        if ((rc = upload_field(c, Z1, z1)) != SPM_OK) return rc;
    }
    c->zeta_dirty = !c->le.enabled;
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

int spm_set_time(spm_ctx *c, int ts, double time, double degree_oblique) {
    if (!c || ts < 0) return fail(SPM_ERR_ARG, "bad argument");
    int rc = spm_synchronize(c);
    if (rc != SPM_OK) return rc;
    c->ts              = ts;
    c->time            = time;
    c->el.time_known   = 0;  // the next Electrolyte step writes the time to the device
    SPM_CUDA_CHECK(cudaMemcpy(c->ts_dev, &c->ts, sizeof(int), cudaMemcpyHostToDevice));
    if (c->le.enabled) c->le.degree_oblique = degree_oblique;
    return SPM_OK;
}

int spm_get_shear_state(spm_ctx *c, double *degree_oblique, double stress[8]) {
    if (!c) return fail(SPM_ERR_ARG, "null context");
    int rc = spm_synchronize(c);
    if (rc != SPM_OK) return rc;
    if (c->sns) {
        double w[kSnsWords];
        SPM_CUDA_CHECK(cudaMemcpy(w, c->sns, sizeof(w), cudaMemcpyDeviceToHost));
        if (degree_oblique) *degree_oblique = 0.0;
        if (stress) {
            const int map[8] = {kSnsRate, kSnsStrain, kSnsStress, kSnsVisc, kSnsInertia, kSnsApparent, -1, -1};
            for (int i = 0; i < 8; i++) stress[i] = map[i] >= 0 ? w[map[i]] : 0.0;
        }
        return SPM_OK;
    }
    return le_get_state(c, degree_oblique, stress);
}

// A device field array for the transforms: complex values (and so the base
// and the field stride) 16-byte aligned, as the kernels' vector accesses and
// tensor maps need.
static bool fft_dev_aligned(const spm_ctx *c, const void *data, size_t field_stride) {
    const size_t cbytes = c->fp64() ? 16 : 8;
    return ((uintptr_t)data % 16) == 0 && (field_stride * cbytes) % 16 == 0;
}

int spm_fft_forward_dev(spm_ctx *c, void *data, int nfields, size_t field_stride) {
    if (!c || !data || nfields < 1) return fail(SPM_ERR_ARG, "bad argument");
    if (!fft_dev_aligned(c, data, field_stride))
        return fail(SPM_ERR_ARG, "field array and field stride must be 16-byte aligned");
    cudaError_t e = c->fp64() ? c->pp64->forward((double *)data, nfields, field_stride, c->st)
                              : c->pp32->forward((float *)data, nfields, field_stride, c->st);
    c->launches += 3;
    SPM_CUDA_CHECK(e);
    return SPM_OK;
}

int spm_fft_inverse_dev(spm_ctx *c, void *data, int nfields, size_t field_stride) {
    if (!c || !data || nfields < 1) return fail(SPM_ERR_ARG, "bad argument");
    if (!fft_dev_aligned(c, data, field_stride))
        return fail(SPM_ERR_ARG, "field array and field stride must be 16-byte aligned");
    cudaError_t e = c->fp64() ? c->pp64->inverse((cplx<double> *)data, nfields, field_stride, c->st)
                              : c->pp32->inverse((cplx<float> *)data, nfields, field_stride, c->st);
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

// nsteps steps with every profiled launch bracketed by CUDA events on its
// own stream (direct launches, no graph replay); `prof` collects the records.
static void profile_clear(spm_ctx *c) {
    for (const auto &r : c->prof) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    c->prof.clear();
}
static int profile_steps(spm_ctx *c, int nsteps, float *total_ms) {
    profile_clear(c);
    cudaEvent_t t0, t1;
    SPM_CUDA_CHECK(cudaEventCreate(&t0));
    SPM_CUDA_CHECK(cudaEventCreate(&t1));
    SPM_CUDA_CHECK(cudaEventRecord(t0, c->st));
    c->prof_on = true;
    int rc     = spm_step(c, nsteps);
    c->prof_on = false;
    cudaEventRecord(t1, c->st);
    SPM_CUDA_CHECK(cudaStreamSynchronize(c->st));
    SPM_CUDA_CHECK(cudaDeviceSynchronize());  // the side stream's records too
    if (total_ms) cudaEventElapsedTime(total_ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return rc;
}

int spm_profile_pass(spm_ctx *c, int nsteps, double *avg_us, double *bytes_per_launch, long long *count) {
    if (!c || nsteps < 1 || !avg_us || !bytes_per_launch || !count) return fail(SPM_ERR_ARG, "bad argument");
    const int rc    = profile_steps(c, nsteps, nullptr);
    double    total = 0.0, bytes = 0.0;
    long long n     = 0;
    for (const auto &r : c->prof) {
        if (std::strncmp(r.name, "strided_pass", 12) != 0) continue;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        total += ms;
        bytes += r.bytes;
        n++;
    }
    profile_clear(c);
    if (rc != SPM_OK) return rc;
    *count            = n;
    *avg_us           = n ? 1000.0 * total / (double)n : 0.0;
    *bytes_per_launch = n ? bytes / (double)n : 0.0;
    return check_device_error(c);
}

int spm_profile_kernels(spm_ctx *c, int nsteps, char *json, size_t cap) {
    if (!c || nsteps < 1 || !json || cap < 64) return fail(SPM_ERR_ARG, "bad argument");
    float     step_ms = 0.f;
    const int rc      = profile_steps(c, nsteps, &step_ms);
    struct Agg {
        long long n     = 0;
        double    ms    = 0.0;
        double    bytes = 0.0;
    };
    std::vector<std::pair<std::string, Agg>> agg;
    for (const auto &r : c->prof) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        auto it = std::find_if(agg.begin(), agg.end(), [&](const std::pair<std::string, Agg> &p) { return p.first == r.name; });
        if (it == agg.end()) {
            agg.push_back({r.name, Agg{}});
            it = agg.end() - 1;
        }
        it->second.n++;
        it->second.ms += ms;
        it->second.bytes += r.bytes;
    }
    profile_clear(c);
    if (rc != SPM_OK) return rc;
    std::string out = "{\"steps\": " + std::to_string(nsteps) + ", \"step_ms_total\": " + std::to_string(step_ms) +
                      ", \"kernels\": [";
    for (size_t i = 0; i < agg.size(); i++) {
        const Agg &a = agg[i].second;
        char       b[320];
        std::snprintf(b, sizeof(b),
                      "%s{\"name\": \"%s\", \"launches\": %lld, \"us_total\": %.3f, \"us_per_launch\": %.3f, "
                      "\"bytes_per_launch\": %.1f}",
                      i ? ", " : "", agg[i].first.c_str(), a.n, 1000.0 * a.ms, 1000.0 * a.ms / (double)a.n,
                      a.bytes / (double)a.n);
        out += b;
    }
    out += "]}";
    if (out.size() + 1 > cap) return fail(SPM_ERR_ARG, "profile buffer too small");
    std::memcpy(json, out.c_str(), out.size() + 1);
    return check_device_error(c);
}

int spm_kernel_launches(spm_ctx *c, long long *count, int reset) {
    if (!c || !count) return fail(SPM_ERR_ARG, "bad argument");
    *count = c->launches;
    if (reset) c->launches = 0;
    return SPM_OK;
}

}  // extern "C"

#include "spm_udf.inc"
#include "spm_api_boundary.inc"
#include "spm_pool.inc"
#include "spm_checkpoint.inc"
#include "spm_output.inc"
#include "spm_restart.inc"
#include "spm_udf_out.inc"
