// Allocation-free variant of Make_f_particle_dt_sole for callers that may not
// allocate device memory.
//
// Some hosts of this library cannot call cudaMalloc: a simulation code that
// hands out all device memory from its own pre-reserved pool, a process
// whose GPU memory is owned by another runtime, or a service that must keep
// its steady-state loop free of allocator calls (which can stall the device
// and fail under memory pressure long after start-up).  Such callers own the
// input and output buffers; everything else this entry point needs lives in
// one file-scope device array, g_noalloc_scratch, that every GPU which loads
// the library holds until the process exits (about 6.5 MB).
//
// Limits and rules (also in include/kapsel_spm.h):
//   * FP64, grids of 8..64 points per axis (NX*NY*(NZ/2+1) complex values
//     per field at most 64*64*33);
//   * the first call on a device resolves the array's device address with
//     cudaGetSymbolAddress and uploads the FFT twiddle tables of every
//     supported size into it; make that first call before any stream
//     capture.  Later calls issue only kernels and memsets on `stream`;
//   * the transforms use the passes without device-side waits, so a call has
//     no device error to report and stays asynchronous;
//   * every call shares the one array: calls that overlap on the GPU (two
//     streams, two host threads) race and give wrong results.
#include <mutex>

#include "../../include/kapsel_spm.h"
#include "spm_fft_plan.cuh"

using namespace spm;

int spm_internal_fail(int code, const char *msg);

namespace {

constexpr int    kNoAllocMaxN     = 64;
constexpr size_t kNoAllocField    = (size_t)kNoAllocMaxN * kNoAllocMaxN * (kNoAllocMaxN + 2);  // doubles
// twiddle tables of the sizes n = 8, 16, 32, 64: for each n the length-n
// table of the X and Y passes, then the z tables of NZ = n (n/2 and n/2 + 1
// values), 2n + 1 complex values in all
constexpr int    kNoAllocTwiddles = 2 * (8 + 16 + 32 + 64) + 4;                                // complex
constexpr size_t kNoAllocDoubles  = 3 * kNoAllocField + 2 * (size_t)kNoAllocTwiddles;

// offset (complex values) of the tables of size n = 2^lg (lg = 3..6)
constexpr int tw_offset(int lg) {
    int o = 0;
    for (int l = 3; l < lg; l++) o += 2 * (1 << l) + 1;
    return o;
}

// The scratch: three padded FP64 fields and the twiddle tables.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

struct NoAllocDevice {
    bool    ready = false;
    double *base  = nullptr;  // device address of g_noalloc_scratch
};
NoAllocDevice g_dev[64];
std::mutex    g_setup_mutex;

// f = up - min(phi, 1) u into the scratch rows (z < NZ).
__global__ void na_make_f(int nx, int ny, int nz, int hnzp, const double *__restrict__ u0,
                          const double *__restrict__ u1, const double *__restrict__ u2,
                          const double *__restrict__ up0, const double *__restrict__ up1,
                          const double *__restrict__ up2, const double *__restrict__ phi, double *__restrict__ f) {
    const size_t rowlen = 2 * (size_t)hnzp;
    const size_t n      = (size_t)nx * ny * rowlen;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        if ((int)(idx % rowlen) >= nz) continue;
        const double ph = phi[idx] < 1.0 ? phi[idx] : 1.0;
        f[idx]          = up0[idx] - ph * u0[idx];
        f[n + idx]      = up1[idx] - ph * u1[idx];
        f[2 * n + idx]  = up2[idx] - ph * u2[idx];
    }
}

// 2/3 truncation and solenoidal projection (Truncate_two_third_rule +
// Solenoidal_uk) of the three k-space fields in the scratch.
__global__ void na_project(Grid g, cplx<double> *__restrict__ f) {
    const size_t n = g.field_elems_c();
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        const int kz  = (int)(idx % (size_t)g.hnzp);
        const size_t row = idx / (size_t)g.hnzp;
        const int j   = (int)(row % (size_t)g.ny);
        const int i   = (int)(row / (size_t)g.ny);
        if (kz >= g.hnz) continue;
        const int KX = i > g.nx / 2 ? i - g.nx : i, KY = j > g.ny / 2 ? j - g.ny : j;
        const bool keep = (abs(KX) < g.trn[0]) && (abs(KY) < g.trn[1]) && (kz < g.trn[2]);
        cplx<double> a = f[idx], b = f[n + idx], c = f[2 * n + idx];
        if (!keep) {
            a = b = c = cplx<double>{0, 0};
        } else {
            const double kx = g.wave[0] * KX, ky = g.wave[1] * KY, kz2 = g.wave[2] * kz;
            const double k2 = kx * kx + ky * ky + kz2 * kz2;
            const double ik2 = k2 > 0.0 ? 1.0 / k2 : 0.0;
            const double dr  = ik2 * (a.re * kx + b.re * ky + c.re * kz2);
            const double di  = ik2 * (a.im * kx + b.im * ky + c.im * kz2);
            a.re -= dr * kx;
            a.im -= di * kx;
            b.re -= dr * ky;
            b.im -= di * ky;
            c.re -= dr * kz2;
            c.im -= di * kz2;
        }
        f[idx]         = a;
        f[n + idx]     = b;
        f[2 * n + idx] = c;
    }
}

void fill_table(cplx<double> *dst, int n, int count) {
    for (int j = 0; j < count; j++) {
        const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)j / (long double)n;
        dst[j]              = cplx<double>{(double)std::cos(a), (double)std::sin(a)};
    }
}

// Once per device, with that device current: resolve the scratch's device
// address, configure the FFT kernels and upload the twiddle tables of every
// supported size (a synchronous copy into the array).  No allocation.
int setup_device(int dev, NoAllocDevice *&out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    NoAllocDevice              &d = g_dev[dev];
    if (!d.ready) {
        void       *ptr = nullptr;
        cudaError_t e   = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || ptr == nullptr)
            return spm_internal_fail(SPM_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch) failed");
        if (FFTPlan<double>::configure_kernels() != cudaSuccess)
            return spm_internal_fail(SPM_ERR_CUDA, "FFT kernel configuration failed");
        static cplx<double> htw[kNoAllocTwiddles];
        for (int lg = 3; lg <= 6; lg++) {
            const int     n = 1 << lg;
            cplx<double> *t = htw + tw_offset(lg);
            fill_table(t, n, n);
            fill_table(t + n, n / 2, n / 2);
            fill_table(t + n + n / 2, n, n / 2 + 1);
        }
        double *base = static_cast<double *>(ptr);
        if (cudaMemcpy(base + 3 * kNoAllocField, htw, sizeof(htw), cudaMemcpyHostToDevice) != cudaSuccess)
            return spm_internal_fail(SPM_ERR_CUDA, "twiddle table upload failed");
        d.base  = base;
        d.ready = true;
    }
    out = &d;
    return SPM_OK;
}

}  // namespace

extern "C" int spm_make_f_particle_dt_sole_noalloc(const double *u0, const double *u1, const double *u2,
                                                   const double *up0, const double *up1, const double *up2,
                                                   const double *phi, double *f0, double *f1, double *f2, int npx,
                                                   int npy, int npz, void *stream) {
    if (!u0 || !u1 || !u2 || !up0 || !up1 || !up2 || !phi || !f0 || !f1 || !f2)
        return spm_internal_fail(SPM_ERR_ARG, "spm_make_f_particle_dt_sole_noalloc: null buffer");
    if (npx < 3 || npy < 3 || npz < 3 || npx > 6 || npy > 6 || npz > 6)
        return spm_internal_fail(SPM_ERR_ARG,
                                 "spm_make_f_particle_dt_sole_noalloc: grid must be 8..64 points per axis "
                                 "(its fixed scratch holds three 64^3 FP64 fields)");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return spm_internal_fail(SPM_ERR_NO_DEVICE, "no current CUDA device");
    NoAllocDevice *d  = nullptr;
    int            rc = setup_device(dev, d);
    if (rc != SPM_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    Grid g{};
    g.nx = 1 << npx;
    g.ny = 1 << npy;
    g.nz = 1 << npz;
    g.hnz = g.hnzp = g.nz / 2 + 1;
    const int n3[3] = {g.nx, g.ny, g.nz};
    for (int k = 0; k < 3; k++) {
        g.trn[k]  = (n3[k] + 2) / 3;
        g.wave[k] = 2.0 * 3.14159265358979323846 / (double)n3[k];  // DX = 1 grid units
    }
    g.dx = 1.0;
    const size_t  fc     = g.field_elems_c();  // complex per field
    double       *fields = d->base;
    cplx<double> *tw     = reinterpret_cast<cplx<double> *>(d->base + 3 * kNoAllocField);
    auto          table  = [&](int n) { return tw + tw_offset(__builtin_ctz((unsigned)n)); };

    // Cleared fields: the padding of a row is never written by na_make_f and
    // must read as zero.
    if (cudaMemsetAsync(fields, 0, 3 * fc * sizeof(cplx<double>), st) != cudaSuccess)
        return spm_internal_fail(SPM_ERR_CUDA, "spm_make_f_particle_dt_sole_noalloc: scratch set-up failed");

    FFTPlan<double> plan;
    plan.g     = g;
    plan.tw_x  = table(g.nx);
    plan.tw_y  = table(g.ny);
    plan.tw_zm = table(g.nz) + g.nz;
    plan.tw_zn = table(g.nz) + g.nz + g.nz / 2;
    int sms    = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    plan.sm_count = sms;

    na_make_f<<<sms * 8, 256, 0, st>>>(g.nx, g.ny, g.nz, g.hnzp, u0, u1, u2, up0, up1, up2, phi, fields);
    cudaError_t e = cudaGetLastError();
    cplx<double> *fk = reinterpret_cast<cplx<double> *>(fields);
    auto strided = [&](int dir, int axis) {
        return dir < 0 ? plan.strided<-1>(fk, 3, fc, axis, st) : plan.strided<+1>(fk, 3, fc, axis, st);
    };
    if (e == cudaSuccess) e = plan.z_r2c(fields, fk, 3, 2 * fc, fc, st);
    if (e == cudaSuccess) e = strided(-1, 1);
    if (e == cudaSuccess) e = strided(-1, 0);
    if (e == cudaSuccess) {
        na_project<<<sms * 8, 256, 0, st>>>(g, fk);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = strided(+1, 0);
    if (e == cudaSuccess) e = strided(+1, 1);
    double *outs[3] = {f0, f1, f2};
    for (int k = 0; k < 3 && e == cudaSuccess; k++)
        e = plan.z_c2r(fk + k * fc, outs[k], 1, fc, 2 * fc, 1.0 / ((double)g.nx * g.ny * g.nz), st);
    if (e != cudaSuccess) return spm_internal_fail(SPM_ERR_CUDA, cudaGetErrorString(e));
    return SPM_OK;
}
