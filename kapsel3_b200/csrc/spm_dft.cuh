// Register-resident small DFTs (N = 2..32) used as the butterflies of the
// hand-written 3D FFT.  Everything is unrolled at compile time; twiddles are
// the exact values cos(2*pi*j/32) written as literals, so they fold into
// immediates and multiplications by 1 and by +-i are skipped.
#pragma once

#include "spm_common.cuh"

namespace spm {

// cos(2*pi*j/32) for j = 0..8 (mathematical constants, correctly rounded).
__host__ __device__ constexpr double cos32_base(int j) {
    return j == 0   ? 1.0
           : j == 1 ? 0.98078528040323044912618223613424
           : j == 2 ? 0.92387953251128675612818318939679
           : j == 3 ? 0.83146961230254523707878837761791
           : j == 4 ? 0.70710678118654752440084436210485
           : j == 5 ? 0.55557023301960222474283081394853
           : j == 6 ? 0.38268343236508977172845998403040
           : j == 7 ? 0.19509032201612826784828486847702
                    : 0.0;
}

// cos(2*pi*j/32) for any j (compile-time when j is).
__host__ __device__ constexpr double cos32(int j) {
    return (j & 31) <= 8    ? cos32_base(j & 31)
           : (j & 31) <= 16 ? -cos32_base(16 - (j & 31))
           : (j & 31) <= 24 ? -cos32_base((j & 31) - 16)
                            : cos32_base(32 - (j & 31));
}
__host__ __device__ constexpr double sin32(int j) { return cos32(j - 8); }

// e^{DIR * 2 pi i * k / N} for N | 32.  DIR = -1: forward (e^{-ikx}).
template <typename T, int N, int DIR>
__device__ __forceinline__ cplx<T> twiddle_c(int k) {
    const int j = k * (32 / N);
    return {(T)cos32(j), (T)(DIR * sin32(j))};
}

template <typename T, int N, int DIR>
__device__ __forceinline__ void twiddle_mul(cplx<T> &v, int k) {
    // k is a compile-time constant after unrolling; special cases fold away.
    const int j = (k * (32 / N)) & 31;
    if (j == 0) return;
    if (j == 8) {  // multiply by DIR * i
        T re = v.re;
        v.re = -(T)DIR * v.im;
        v.im = (T)DIR * re;
        return;
    }
    if (j == 16) {
        v.re = -v.re;
        v.im = -v.im;
        return;
    }
    if (j == 24) {  // multiply by -DIR * i
        T re = v.re;
        v.re = (T)DIR * v.im;
        v.im = -(T)DIR * re;
        return;
    }
    v = cmul(v, twiddle_c<T, N, DIR>(k));
}

__host__ __device__ constexpr int bitrev_c(int i, int n) {
    int r = 0;
    for (int b = 1; b < n; b <<= 1) {
        r = (r << 1) | (i & 1);
        i >>= 1;
    }
    return r;
}

// In-place length-N DFT of v[0..N): X[k] = sum_n v[n] e^{DIR 2 pi i n k / N}.
template <typename T, int N, int DIR>
__device__ __forceinline__ void dft_reg(cplx<T> (&v)[N]) {
#pragma unroll
    for (int i = 0; i < N; i++) {
        const int j = bitrev_c(i, N);
        if (j > i) {
            cplx<T> t = v[i];
            v[i]      = v[j];
            v[j]      = t;
        }
    }
#pragma unroll
    for (int len = 2; len <= N; len <<= 1) {
#pragma unroll
        for (int i = 0; i < N; i += len) {
#pragma unroll
            for (int k = 0; k < len / 2; k++) {
                cplx<T> b = v[i + k + len / 2];
                // twiddle e^{DIR 2 pi i k / len} expressed on the 32-grid
                const int j = (k * (32 / len)) & 31;
                if (j == 0) {
                } else if (j == 8) {
                    T re = b.re;
                    b.re = -(T)DIR * b.im;
                    b.im = (T)DIR * re;
                } else {
                    b = cmul(b, cplx<T>{(T)cos32(j), (T)(DIR * sin32(j))});
                }
                cplx<T> a        = v[i + k];
                v[i + k]         = cadd(a, b);
                v[i + k + len / 2] = csub(a, b);
            }
        }
    }
}

// Compile-time split N = N1 * N2 used by the four-step kernels
// (N1 threads per line in step 1, each doing an N2-point DFT).
template <int N>
struct Split;
template <>
struct Split<4> {
    static constexpr int N1 = 2, N2 = 2;
};
template <>
struct Split<8> {
    static constexpr int N1 = 2, N2 = 4;
};
template <>
struct Split<16> {
    static constexpr int N1 = 4, N2 = 4;
};
template <>
struct Split<32> {
    static constexpr int N1 = 4, N2 = 8;
};
template <>
struct Split<64> {
    static constexpr int N1 = 8, N2 = 8;
};
template <>
struct Split<128> {
    static constexpr int N1 = 8, N2 = 16;
};
template <>
struct Split<256> {
    static constexpr int N1 = 16, N2 = 16;
};
template <>
struct Split<512> {
    static constexpr int N1 = 16, N2 = 32;
};

}  // namespace spm
