// Common device/host definitions for the B200 SPM step.
//
// Field layout in HBM (both precisions):
//   k-space field  : complex<T> [NX][NY][HNZP]        (HNZP >= NZ/2+1)
//   real field     : T          [NX][NY][2*HNZP]      (rows padded, in place)
// For T = double HNZP = NZ/2+1, which is exactly the reference's in-place r2c
// array [NX][NY][NZ_] (input.cxx:444-445, fft_wrapper.cxx:104-112), so FP64
// fields cross the C ABI without any reshuffle.  For T = float one extra
// complex is appended when NZ/2+1 is odd so every row starts on a 16-byte
// boundary.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>

namespace spm {

// A complex value aligned to its full size, so that a value in shared or
// global memory moves as one 8-byte (FP32) or 16-byte (FP64) access.
template <typename T>
struct alignas(2 * sizeof(T)) cplx {
    T re, im;
};

template <typename T>
struct vec2_of;
template <>
struct vec2_of<double> {
    using type = double2;
};
template <>
struct vec2_of<float> {
    using type = float2;
};

template <typename T>
__host__ __device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T>
__host__ __device__ __forceinline__ cplx<T> cadd(cplx<T> a, cplx<T> b) {
    return {a.re + b.re, a.im + b.im};
}
template <typename T>
__host__ __device__ __forceinline__ cplx<T> csub(cplx<T> a, cplx<T> b) {
    return {a.re - b.re, a.im - b.im};
}

// FP32 complex addition and subtraction as one paired instruction
// (add/sub.rn.f32x2 of sm_100): each lane rounds as the scalar operation
// does, with half the floating-point instructions in the transforms'
// butterflies.  (A product feeding the sum is no longer contracted into a
// fused multiply-add, so a result may differ from the scalar code's in the
// last bit.)
#if !defined(SPM_NO_F32X2)
#define SPM_F32X2_ASM(op)                                                                         \
    unsigned long long ua, ub, ur;                                                                \
    asm("mov.b64 %0, {%1, %2};" : "=l"(ua) : "f"(a.re), "f"(a.im));                               \
    asm("mov.b64 %0, {%1, %2};" : "=l"(ub) : "f"(b.re), "f"(b.im));                               \
    asm(op " %0, %1, %2;" : "=l"(ur) : "l"(ua), "l"(ub));                                         \
    cplx<float> r;                                                                                \
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.re), "=f"(r.im) : "l"(ur));                              \
    return r;
template <>
__host__ __device__ __forceinline__ cplx<float> cadd<float>(cplx<float> a, cplx<float> b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    SPM_F32X2_ASM("add.rn.f32x2")
#else
    return {a.re + b.re, a.im + b.im};
#endif
}
template <>
__host__ __device__ __forceinline__ cplx<float> csub<float>(cplx<float> a, cplx<float> b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    SPM_F32X2_ASM("sub.rn.f32x2")
#else
    return {a.re - b.re, a.im - b.im};
#endif
}
#undef SPM_F32X2_ASM
#endif

// Grid geometry shared by every kernel.
struct Grid {
    int nx, ny, nz;
    int hnz;     // NZ/2+1 complex values per row that carry data
    int hnzp;    // allocated complex values per row (>= hnz)
    int trn[3];  // 2/3-rule limits TRN = (N+2)/3 (input.cxx:448)
    double wave[3];
    double dx;
    __host__ __device__ size_t field_elems_c() const { return (size_t)nx * ny * hnzp; }  // complex elements

    // The retained 2/3 box |KX| < TRN_X, |KY| < TRN_Y, KZ < TRN_Z: the only
    // modes the step's k-space updates read or write.  box_index maps a
    // dense box index (kz fastest) to the field's complex element index.
    __host__ __device__ size_t box_elems() const {
        return (size_t)(2 * trn[0] - 1) * (size_t)(2 * trn[1] - 1) * (size_t)trn[2];
    }
    __host__ __device__ size_t box_index(size_t b) const {
        const int    kz = (int)(b % (size_t)trn[2]);
        const size_t r  = b / (size_t)trn[2];
        const int    ny_box = 2 * trn[1] - 1;
        const int    iy = (int)(r % (size_t)ny_box);
        const int    ix = (int)(r / (size_t)ny_box);
        const int    i  = ix < trn[0] ? ix : ix + nx - (2 * trn[0] - 1);
        const int    j  = iy < trn[1] ? iy : iy + ny - ny_box;
        return ((size_t)i * ny + j) * hnzp + kz;
    }
    // Complex values per z row that a pruned forward z pass must produce so
    // that every strided column tile covering KZ < TRN_Z reads written data
    // (tiles are 8, 16 or 32 columns wide).
    __host__ __device__ int kz_span() const {
        const int r = (trn[2] + 31) / 32 * 32;
        return r < hnz ? r : hnz;
    }
};

// Device-side error word: kernels that detect a violated precondition (a
// particle outside the box, a bounded wait that ran out) set a bit here and
// skip the offending work; the host checks it after the step.
enum SpmDeviceError : unsigned int {
    SPM_DEVERR_PARTICLE_OUT_OF_BOX = 1u << 0,
    SPM_DEVERR_LJ_CELL_OVERFLOW    = 1u << 1,
    SPM_DEVERR_NAN                 = 1u << 2,
    SPM_DEVERR_SCRATCH_TOO_SMALL   = 1u << 3,
};

}  // namespace spm

#define SPM_CUDA_CHECK(expr)                                                                         \
    do {                                                                                             \
        cudaError_t _e = (expr);                                                                     \
        if (_e != cudaSuccess) {                                                                     \
            std::fprintf(stderr, "kapsel_spm: CUDA error %s at %s:%d: %s\n", cudaGetErrorName(_e), \
                         __FILE__, __LINE__, cudaGetErrorString(_e));                                \
            return SPM_ERR_CUDA;                                                                     \
        }                                                                                            \
    } while (0)
