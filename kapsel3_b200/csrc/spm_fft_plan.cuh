// Host-side plan for the hand-written 3D real FFT: twiddle tables and the
// dispatch from runtime sizes to the compile-time kernels of spm_fft.cuh.
#pragma once

#include <algorithm>
#include <vector>

#include "spm_fft.cuh"

namespace spm {

template <typename T>
struct FFTPlan {
    Grid     g{};
    cplx<T> *tw_x  = nullptr;  // e^{-2 pi i j/NX}, j < NX
    cplx<T> *tw_y  = nullptr;  // e^{-2 pi i j/NY}
    cplx<T> *tw_zm = nullptr;  // e^{-2 pi i j/(NZ/2)}, j < NZ/2
    cplx<T> *tw_zn = nullptr;  // e^{-2 pi i k/NZ}, k <= NZ/2

    static constexpr int W = sizeof(T) == 8 ? 16 : 32;  // kz columns per strided tile

    static bool size_ok(int n) { return n >= 8 && n <= 512 && (n & (n - 1)) == 0; }

    // The fused z pass of the advection term keeps the three velocity rows in
    // registers for FP32 rows of up to 256 reals, else in shared memory (one
    // warp of rows per CTA).
    template <int MM>
    static constexpr bool ureg() {
        return sizeof(T) == 4 && MM <= 128;
    }
    template <int MM>
    static constexpr int prows() {
        return ureg<MM>() ? zr_rows<T, MM>() : 32 / ZR<MM>::P;
    }
    // Resident CTAs the compiler must allow for: at M = 128 the register-held
    // rows fill 255 registers, two CTAs per SM; capping at 168 (three CTAs)
    // costs a few spilled values and measured 4% faster on B200.
    template <int MM>
    static constexpr int pminb() {
        return ureg<MM>() && MM == 128 ? 3 : 1;
    }
    // The FP64 inverse pass at M = 128 wants 132 registers, three CTAs of 128
    // threads per SM; capped at 128 a fourth fits, for a pass bound by load
    // latency (FP64 step at 256^3: 1.649 -> 1.623 ms).  Every other
    // instance keeps the compiler's own allocation (0: no cap).
    template <int MM>
    static constexpr int c2r_minb() {
        return sizeof(T) == 8 && MM == 128 ? 4 : 0;
    }

    // Fused inverse-z / advection products / forward-z pass over five slots.
    cudaError_t z_products(cplx<T> *io, size_t fs_c, int nruns, size_t run_stride_c, cudaStream_t st, int kz_keep,
                           int kz_span) const {
        const int nrows = g.nx * g.ny;
        const T   scale = (T)(1.0 / ((double)g.nx * g.ny * g.nz));
        switch (g.nz / 2) {
#define SPM_ZP(MM)                                                                                              \
    case MM: {                                                                                                  \
        constexpr int RR = prows<MM>();                                                                         \
        zr_products_kernel<T, MM, RR, ureg<MM>(), pminb<MM>()>                                                  \
            <<<dim3((nrows + RR - 1) / RR, nruns), RR * ZR<MM>::P, zr_products_smem<T, MM, RR, ureg<MM>()>(), st>>>( \
                io, fs_c, run_stride_c, nrows, g.hnzp, tw_zm, tw_zn, scale, kz_keep, kz_span);                 \
    } break;
            SPM_ZP(4) SPM_ZP(8) SPM_ZP(16) SPM_ZP(32) SPM_ZP(64) SPM_ZP(128) SPM_ZP(256)
#undef SPM_ZP
            default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }

    cudaError_t create(const Grid &grid) {
        g = grid;
        cudaError_t e;
        if ((e = make_table(&tw_x, g.nx, g.nx)) != cudaSuccess) return e;
        if ((e = make_table(&tw_y, g.ny, g.ny)) != cudaSuccess) return e;
        if ((e = make_table(&tw_zm, g.nz / 2, g.nz / 2)) != cudaSuccess) return e;
        if ((e = make_table(&tw_zn, g.nz, g.nz / 2 + 1)) != cudaSuccess) return e;
        return set_smem_attrs();
    }
    void destroy() {
        cudaFree(tw_x);
        cudaFree(tw_y);
        cudaFree(tw_zm);
        cudaFree(tw_zn);
        tw_x = tw_y = tw_zm = tw_zn = nullptr;
    }

    // In-place forward transform of nfields real fields (padded rows).
    cudaError_t forward(T *data, int nfields, size_t fstride_c, cudaStream_t st) const {
        cudaError_t e = z_r2c(data, reinterpret_cast<cplx<T> *>(data), nfields, 2 * fstride_c, fstride_c, st);
        if (e != cudaSuccess) return e;
        if ((e = strided<-1>(reinterpret_cast<cplx<T> *>(data), nfields, fstride_c, 1, st)) != cudaSuccess) return e;
        return strided<-1>(reinterpret_cast<cplx<T> *>(data), nfields, fstride_c, 0, st);
    }
    // In-place normalised inverse transform.
    cudaError_t inverse(cplx<T> *data, int nfields, size_t fstride_c, cudaStream_t st) const {
        cudaError_t e = strided<+1>(data, nfields, fstride_c, 0, st);
        if (e != cudaSuccess) return e;
        if ((e = strided<+1>(data, nfields, fstride_c, 1, st)) != cudaSuccess) return e;
        return z_c2r(data, reinterpret_cast<T *>(data), nfields, fstride_c, 2 * fstride_c,
                     (T)(1.0 / ((double)g.nx * g.ny * g.nz)), st);
    }

    // Individual passes (exposed for the fused step).
    cudaError_t z_r2c(const T *in, cplx<T> *out, int nfields, size_t fs_real, size_t fs_c, cudaStream_t st,
                      int kz_span = 1 << 30) const {
        const int nrows = g.nx * g.ny;
        switch (g.nz / 2) {
#define SPM_ZR2C(MM)                                                                                          \
    case MM: {                                                                                                \
        constexpr int RR = zr_rows<T, MM>();                                                                  \
        zr_r2c_kernel<T, MM, RR><<<dim3((nrows + RR - 1) / RR, nfields), RR * ZR<MM>::P, 0, st>>>(            \
            in, out, fs_real, fs_c, nrows, g.hnzp, tw_zm, tw_zn, kz_span);                                    \
    } break;
            SPM_ZR2C(4) SPM_ZR2C(8) SPM_ZR2C(16) SPM_ZR2C(32) SPM_ZR2C(64) SPM_ZR2C(128) SPM_ZR2C(256)
#undef SPM_ZR2C
            default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
    cudaError_t z_c2r(const cplx<T> *in, T *out, int nfields, size_t fs_c, size_t fs_real, T scale,
                      cudaStream_t st, int kz_keep = 1 << 30) const {
        const int nrows = g.nx * g.ny;
        switch (g.nz / 2) {
#define SPM_ZC2R(MM)                                                                                          \
    case MM: {                                                                                                \
        constexpr int RR = zr_rows<T, MM>();                                                                  \
        const dim3    grid((nrows + RR - 1) / RR, nfields);                                                   \
        if constexpr (c2r_minb<MM>() > 1)                                                                     \
            zr_c2r_kernel_capped<T, MM, RR, c2r_minb<MM>()><<<grid, RR * ZR<MM>::P, 0, st>>>(                 \
                in, out, fs_c, fs_real, nrows, g.hnzp, tw_zm, tw_zn, scale, kz_keep);                         \
        else                                                                                                  \
            zr_c2r_kernel<T, MM, RR><<<grid, RR * ZR<MM>::P, 0, st>>>(in, out, fs_c, fs_real, nrows, g.hnzp,  \
                                                                      tw_zm, tw_zn, scale, kz_keep);          \
    } break;
            SPM_ZC2R(4) SPM_ZC2R(8) SPM_ZC2R(16) SPM_ZC2R(32) SPM_ZC2R(64) SPM_ZC2R(128) SPM_ZC2R(256)
#undef SPM_ZC2R
            default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
    // Persistent TMA-pipelined strided pass (N <= 256): tile W_T columns,
    // S_T-deep buffer ring.  Returns cudaErrorNotSupported when it cannot run
    // (size or missing driver entry point); the caller then uses strided().
    static constexpr int W_T = sizeof(T) == 8 ? 16 : 32;
    static constexpr int S_T = 3;
    unsigned int *err = nullptr;  // device error word (set by the owner)
    // bound of every TMA ring wait, global-timer nanoseconds
    unsigned long long wait_ns = kWaitLimitNs;
    // test switch: the next skip_loads TMA pass launches issue no loads, so
    // their waits run out (see fft_strided_tma_kernel)
    mutable int skip_loads = 0;
    int           ctas_per_sm = 1;
    int           sm_count    = 148;

    template <int DIR>
    cudaError_t strided_tma(cplx<T> *data, int nfields, size_t fs_c, int axis, cudaStream_t st,
                            PassPrune pr) const {
        const int n = axis == 1 ? g.ny : g.nx;
        if (n > 256 || !encode_tiled_fn()) return cudaErrorNotSupported;
        const int outer   = axis == 1 ? g.nx : g.ny;
        const int ct_used = (std::min(pr.kz_cols, g.hnz) + W_T - 1) / W_T;
        const int ntiles  = nfields * outer_count(outer, pr.outer_trn) * ct_used;
        if (ntiles == 0) return cudaSuccess;
        const uint64_t dims[4] = {(uint64_t)2 * g.hnz, (uint64_t)g.ny, (uint64_t)g.nx, (uint64_t)nfields};
        const uint64_t strides[3] = {(uint64_t)2 * g.hnzp * sizeof(T), (uint64_t)g.ny * 2 * g.hnzp * sizeof(T),
                                     (uint64_t)fs_c * sizeof(cplx<T>)};
        // load and store maps: boxes of N lines, or of the pruned line count
        // (two boxes per tile, pruned_box_lines)
        CUtensorMap lmap, smap;
        auto        make = [&](CUtensorMap *m, int lines) {
            const uint32_t box[4] = {(uint32_t)(2 * W_T), axis == 1 ? (uint32_t)lines : 1u,
                                     axis == 1 ? 1u : (uint32_t)lines, 1u};
            return make_map_4d<T>(m, data, dims, strides, box);
        };
        if (!make(&lmap, pruned_box_lines(n, pr.line_trn)) || !make(&smap, pruned_box_lines(n, pr.out_trn)))
            return cudaErrorNotSupported;
        const cplx<T> *tw   = axis == 1 ? tw_y : tw_x;
        const int      grid = std::min(ntiles, sm_count * ctas_per_sm);
        const int      skip = skip_loads > 0 ? 1 : 0;
        if (skip) skip_loads--;
        switch (n) {
#define SPM_TMA(NN)                                                                                            \
    case NN:                                                                                                   \
        fft_strided_tma_kernel<T, NN, W_T, DIR, S_T>                                                           \
            <<<grid, W_T * Split<NN>::N1, (size_t)S_T * NN * W_T * sizeof(cplx<T>), st>>>(                     \
                lmap, smap, axis, outer, ct_used, ntiles, tw, err, pr, wait_ns, skip);                         \
        break;
            SPM_TMA(8) SPM_TMA(16) SPM_TMA(32) SPM_TMA(64) SPM_TMA(128) SPM_TMA(256)
#undef SPM_TMA
            default: return cudaErrorNotSupported;
        }
        return cudaGetLastError();
    }
    template <int DIR>
    cudaError_t strided_tma(cplx<T> *data, int nfields, size_t fs_c, int axis, cudaStream_t st) const {
        return strided_tma<DIR>(data, nfields, fs_c, axis, st, PassPrune::full(g.hnz));
    }

    // axis 1 = Y, axis 0 = X
    template <int DIR>
    cudaError_t strided(cplx<T> *data, int nfields, size_t fs_c, int axis, cudaStream_t st, PassPrune pr) const {
        const int    n            = axis == 1 ? g.ny : g.nx;
        const int    outer        = axis == 1 ? g.nx : g.ny;
        const size_t outer_stride = axis == 1 ? (size_t)g.ny * g.hnzp : (size_t)g.hnzp;
        const size_t axis_stride  = axis == 1 ? (size_t)g.hnzp : (size_t)g.ny * g.hnzp;
        const cplx<T> *tw         = axis == 1 ? tw_y : tw_x;
        const int    ct_used      = (std::min(pr.kz_cols, g.hnz) + W - 1) / W;
        const int    nblocks      = outer_count(outer, pr.outer_trn) * ct_used;
        if (nblocks == 0 || nfields == 0) return cudaSuccess;
        const dim3   grid(nblocks, nfields);
        switch (n) {
#define SPM_STR(NN)                                                                                              \
    case NN:                                                                                                     \
        fft_strided_kernel<T, NN, W, DIR><<<grid, W * Split<NN>::N1, (size_t)NN * W * sizeof(cplx<T>), st>>>( \
            data, fs_c, g.hnz, ct_used, outer, outer_stride, axis_stride, tw, pr);                              \
        break;
            SPM_STR(8) SPM_STR(16) SPM_STR(32) SPM_STR(64) SPM_STR(128) SPM_STR(256) SPM_STR(512)
#undef SPM_STR
            default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
    template <int DIR>
    cudaError_t strided(cplx<T> *data, int nfields, size_t fs_c, int axis, cudaStream_t st) const {
        return strided<DIR>(data, nfields, fs_c, axis, st, PassPrune::full(g.hnz));
    }

    // Sets the shared-memory limits of every FFT kernel (process-wide
    // function attributes; no allocation).
    static cudaError_t configure_kernels() { return set_smem_attrs(); }

  private:
    static cudaError_t make_table(cplx<T> **dst, int n, int count) {
        std::vector<cplx<T>> h(count);
        for (int j = 0; j < count; j++) {
            const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)j / (long double)n;
            h[j] = cplx<T>{(T)std::cos(a), (T)std::sin(a)};
        }
        cudaError_t e = cudaMalloc(dst, sizeof(cplx<T>) * count);
        if (e != cudaSuccess) return e;
        return cudaMemcpy(*dst, h.data(), sizeof(cplx<T>) * count, cudaMemcpyHostToDevice);
    }
    template <int NN, int DIR>
    static cudaError_t attr_one() {
        return cudaFuncSetAttribute(fft_strided_kernel<T, NN, W, DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(NN * W * sizeof(cplx<T>)));
    }
    template <int NN, int DIR>
    static cudaError_t attr_tma() {
        return cudaFuncSetAttribute(fft_strided_tma_kernel<T, NN, W_T, DIR, S_T>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)((size_t)S_T * NN * W_T * sizeof(cplx<T>)));
    }
    template <int MM>
    static cudaError_t attr_products() {
        return cudaFuncSetAttribute(zr_products_kernel<T, MM, prows<MM>(), ureg<MM>(), pminb<MM>()>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)zr_products_smem<T, MM, prows<MM>(), ureg<MM>()>());
    }
    static cudaError_t set_smem_attrs() {
        cudaError_t e = cudaSuccess;
#define SPM_TATTR(NN)                                         \
    if ((e = attr_tma<NN, -1>()) != cudaSuccess) return e;      \
    if ((e = attr_tma<NN, +1>()) != cudaSuccess) return e;
        SPM_TATTR(8) SPM_TATTR(16) SPM_TATTR(32) SPM_TATTR(64) SPM_TATTR(128) SPM_TATTR(256)
#undef SPM_TATTR
#define SPM_PATTR(MM) \
    if ((e = attr_products<MM>()) != cudaSuccess) return e;
        SPM_PATTR(4) SPM_PATTR(8) SPM_PATTR(16) SPM_PATTR(32) SPM_PATTR(64) SPM_PATTR(128) SPM_PATTR(256)
#undef SPM_PATTR
#define SPM_ATTR(NN)                                               \
    if ((e = attr_one<NN, -1>()) != cudaSuccess) return e;          \
    if ((e = attr_one<NN, +1>()) != cudaSuccess) return e;
        SPM_ATTR(8) SPM_ATTR(16) SPM_ATTR(32) SPM_ATTR(64) SPM_ATTR(128) SPM_ATTR(256) SPM_ATTR(512)
#undef SPM_ATTR
        return e;
    }
};

}  // namespace spm
