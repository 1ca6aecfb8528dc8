// Z-row transforms of the 3D real FFT: one row of NZ = 2M reals <-> M+1
// complex values (the z part of A2a_k / A_k2a, fft_wrapper.h:641-681, done by
// Ooura's rdft3d as a real transform per z row).
//
// A row is owned by P threads of one warp.  The length-M complex transform of
// the packed row z[n] = (x[2n], x[2n+1]) is split as
//     k = a + Q j  (a < Q = 2P residues, j < J = M/Q),
//     n = b + J c  (b < J, c < Q),
// so that
//   * thread t owns the two residues a0 = t, a1 = Q - t (t = 0: 0 and Q/2),
//     i.e. the k-side values X[a + Q j] of both residues.  The set is closed
//     under k -> M - k, so the real <-> half-complex split, which pairs X[k]
//     with X[M-k], runs on the thread's own registers;
//   * thread t owns b = t + P s (s < BPT = J/P) on the n side, all c.
// The J-point DFTs over j (per residue) and the Q-point DFTs over c (per b) run
// in registers; the one transpose between them goes through a per-row block
// of shared memory, so a transform costs one write and one read of the row
// and only warp-level synchronisation.
#pragma once

#include "spm_dft.cuh"

namespace spm {

// The even/odd split of a length-2M real transform packed as M complex
// values, w = e^{-2 pi i k / (2M)}:
//   forward  X[k] = E + w O,  E = (Z[k] + conj Z[M-k]) / 2,
//            O = -i (Z[k] - conj Z[M-k]) / 2; hw = w / 2 is passed;
//   inverse  Z'[k] = c (X[k] + conj X[M-k]) + i c (X[k] - conj X[M-k]) conj(w),
//            the output scaled by c; cw = c w is passed.
// Folding the factors 1/2 and c into the twiddle leaves ten floating-point
// operations per value.
template <typename T>
__device__ __forceinline__ cplx<T> r2c_split(const cplx<T> &zk, const cplx<T> &zmk, const cplx<T> &hw) {
    const T sr = zk.re + zmk.re, di = zk.im - zmk.im;
    const T si = zk.im + zmk.im, dr = zk.re - zmk.re;
    return cplx<T>{(T)0.5 * sr + (hw.re * si + hw.im * dr), (T)0.5 * di + (hw.im * si - hw.re * dr)};
}
template <typename T>
__device__ __forceinline__ cplx<T> c2r_split(const cplx<T> &xk, const cplx<T> &xmk, const cplx<T> &cw, T c) {
    const T sr = xk.re + xmk.re, di = xk.im - xmk.im;
    const T dr = xk.re - xmk.re, si = xk.im + xmk.im;
    const T orr = dr * cw.re + si * cw.im;
    const T oi  = si * cw.re - dr * cw.im;
    return cplx<T>{c * sr - oi, c * di + orr};
}

template <int M>
struct ZR {
    // largest power of two P with 2 P^2 <= M (so that BPT >= 1)
    static constexpr int P   = (2 * 8 * 8 <= M) ? 8 : (2 * 4 * 4 <= M) ? 4 : (2 * 2 * 2 <= M) ? 2 : 1;
    static constexpr int Q   = 2 * P;
    static constexpr int J   = M / Q;
    static constexpr int BPT = J / P;
    static constexpr int V   = 2 * J;  // complex values per thread
    static_assert(BPT >= 1 && BPT * P == J && J <= 16 && Q <= 16, "unsupported z-row length");
};

// Per-row shared block: J lines of Q complex values.  The line pitch is an
// odd number of 16-byte units, so the P threads reading one line each (16-byte
// vectors) hit distinct banks; the block size is congruent to the bytes one
// row's threads store at once (P complex values) modulo 128, so the rows that
// one wavefront serves do not share banks.
template <typename T, int M>
struct ZRSmem {
    static constexpr int cb      = (int)sizeof(cplx<T>);
    static constexpr int pitch_b = (ZR<M>::Q * cb / 16) % 2 == 1 ? ZR<M>::Q * cb : ZR<M>::Q * cb + 16;
    static constexpr int raw     = ZR<M>::J * pitch_b;
    static constexpr int spread  = (ZR<M>::P * cb) % 128;
    static constexpr int want    = spread == 0 ? 0 : spread < 16 ? 16 : spread;  // 16-byte aligned blocks
    static constexpr int blk     = raw + ((want - raw % 128) + 128) % 128;  // bytes per row block
    static constexpr int pitch   = pitch_b / cb;                           // line pitch, complex units
};

// A line of Q consecutive complex values of a row block, moved as 16-byte
// vectors (two FP32 or one FP64 complex value per access).
template <typename T, int Q>
__device__ __forceinline__ void zr_line_load(const cplx<T> *src, cplx<T> (&v)[Q]) {
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int q = 0; q < Q; q += 2) {
            const float4 f = *reinterpret_cast<const float4 *>(src + q);
            v[q]           = cplx<T>{f.x, f.y};
            v[q + 1]       = cplx<T>{f.z, f.w};
        }
    } else {
#pragma unroll
        for (int q = 0; q < Q; q++) v[q] = src[q];
    }
}
template <typename T, int Q>
__device__ __forceinline__ void zr_line_store(cplx<T> *dst, const cplx<T> (&v)[Q]) {
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int q = 0; q < Q; q += 2)
            *reinterpret_cast<float4 *>(dst + q) = make_float4(v[q].re, v[q].im, v[q + 1].re, v[q + 1].im);
    } else {
#pragma unroll
        for (int q = 0; q < Q; q++) dst[q] = v[q];
    }
}

// Twiddle-table read that the compiler keeps where it is written: hoisting
// the tables' loads out of the products kernel's loop over transforms would
// hold every twiddle in registers for the whole kernel.
template <typename T>
__device__ __forceinline__ cplx<T> zr_tw(const cplx<T> *p) {
    cplx<T> w;
    if constexpr (sizeof(T) == 4) {
        asm volatile("ld.global.nc.v2.f32 {%0, %1}, [%2];" : "=f"(w.re), "=f"(w.im) : "l"(p));
    } else {
        asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2];" : "=d"(w.re), "=d"(w.im) : "l"(p));
    }
    return w;
}

// Mirror of the k-side value (r, j), i.e. of k = a_r + Q j, among the
// thread's own values: M - k = a_{r'} + Q j'.  t = 0 owns residues 0 and
// Q/2, which are their own mirrors; the mirror of k = 0 is k = M (xn).
template <typename T, int J>
__device__ __forceinline__ cplx<T> zr_mirror(const cplx<T> (&kv)[2][J], const cplx<T> &xn, bool t0, int r, int j) {
    if (r == 0) {
        const cplx<T> own = (j == 0) ? xn : kv[0][(J - j) % J];
        return t0 ? own : kv[1][J - 1 - j];
    }
    return t0 ? kv[1][J - 1 - j] : kv[0][J - 1 - j];
}

// The residues of thread t and the split twiddles e^{-2 pi i a / (2M)}.
template <typename T, int M>
__device__ __forceinline__ void zr_residues(int t, int (&a)[2], cplx<T> (&wb)[2], const cplx<T> *__restrict__ twN) {
    constexpr int Q = ZR<M>::Q;
    a[0] = t;
    a[1] = t == 0 ? Q / 2 : Q - t;
    wb[0] = twN[a[0]];
    wb[1] = twN[a[1]];
}

// Load the k-side values of one row (kz >= kz_keep read as zero).
template <typename T, int M>
__device__ __forceinline__ void zr_load_k(const cplx<T> *row, bool ok, const int (&a)[2], int kz_keep,
                                          cplx<T> (&kv)[2][ZR<M>::J], cplx<T> &xn) {
    constexpr int Q = ZR<M>::Q, J = ZR<M>::J;
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
        for (int j = 0; j < J; j++) {
            const int k = a[r] + Q * j;
            kv[r][j]    = (ok && k < kz_keep) ? row[k] : cplx<T>{0, 0};
        }
    xn = (ok && a[0] == 0 && M < kz_keep) ? row[M] : cplx<T>{0, 0};
}

// Store the k-side values of one row for kz < kz_span; the padding values
// kz = M+1 .. hnzp-1 are zeroed when kz_span reaches past M.
template <typename T, int M>
__device__ __forceinline__ void zr_store_k(cplx<T> *row, bool ok, int t, const int (&a)[2], int kz_span, int hnzp,
                                           const cplx<T> (&kv)[2][ZR<M>::J], const cplx<T> &xn) {
    constexpr int Q = ZR<M>::Q, J = ZR<M>::J, P = ZR<M>::P;
    if (!ok) return;
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
        for (int j = 0; j < J; j++) {
            const int k = a[r] + Q * j;
            if (k < kz_span) row[k] = kv[r][j];
        }
    if (t == 0 && M < kz_span) row[M] = xn;
    if (kz_span > M)
        for (int k = M + 1 + t; k < hnzp; k += P) row[k] = cplx<T>{0, 0};
}

// Inverse: X[k] (k-side values, X[M] in xn; imaginary parts of X[0] and X[M]
// discarded) -> out[s][c] = z[(t + P s) + J c] = (x[2n], x[2n+1]) * scale'
// where the full normalisation `scale` is applied in the split.
// S is the row's shared block; the call ends with the block free again.
template <typename T, int M>
__device__ __forceinline__ void zr_c2r(int t, const int (&a)[2], const cplx<T> (&wb)[2], cplx<T> (&kv)[2][ZR<M>::J],
                                       cplx<T> xn, cplx<T> *S, const cplx<T> *__restrict__ twM, T scale,
                                       cplx<T> (&out)[ZR<M>::BPT][ZR<M>::Q]) {
    constexpr int Q = ZR<M>::Q, J = ZR<M>::J, P = ZR<M>::P, BPT = ZR<M>::BPT;
    constexpr int pitch = ZRSmem<T, M>::pitch;
    const bool    t0    = t == 0;
    // Z'[k] = E' + i O' (see c2r_split) for the thread's k, all in registers
    cplx<T> zp[2][J];
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
        for (int j = 0; j < J; j++) {
            cplx<T> xk = kv[r][j], xm = zr_mirror<T, J>(kv, xn, t0, r, j);
            if (r == 0 && j == 0 && t0) xk.im = xm.im = 0;
            cplx<T> w = cplx<T>{scale * wb[r].re, scale * wb[r].im};
            twiddle_mul<T, 2 * J, -1>(w, j);  // c e^{-2 pi i (a + Q j) / (2M)}
            zp[r][j] = c2r_split<T>(xk, xm, w, scale);
        }
    // step 1: J-point DFTs over j, twiddle e^{+2 pi i a b / M}, to shared
#pragma unroll
    for (int r = 0; r < 2; r++) {
        dft_reg<T, J, +1>(zp[r]);
#pragma unroll
        for (int b = 1; b < J; b++) {
            cplx<T> w = zr_tw<T>(twM + ((a[r] * b) & (M - 1)));
            w.im      = -w.im;
            zp[r][b]  = cmul(zp[r][b], w);
        }
#pragma unroll
        for (int b = 0; b < J; b++) S[b * pitch + a[r]] = zp[r][b];
    }
    __syncwarp();
    // step 2: Q-point DFTs over the residues for b = t + P s
#pragma unroll
    for (int s = 0; s < BPT; s++) {
        const int b = t + P * s;
        zr_line_load<T, Q>(S + b * pitch, out[s]);
        dft_reg<T, Q, +1>(out[s]);
    }
    __syncwarp();
}

// Forward: in[s][c] = z[(t + P s) + J c] -> the k-side values X[k] of the
// thread's residues and, for t = 0, X[M] in xn.
template <typename T, int M>
__device__ __forceinline__ void zr_r2c(int t, const int (&a)[2], const cplx<T> (&wb)[2],
                                       cplx<T> (&in)[ZR<M>::BPT][ZR<M>::Q], cplx<T> *S, const cplx<T> *__restrict__ twM,
                                       cplx<T> (&kv)[2][ZR<M>::J], cplx<T> &xn) {
    constexpr int Q = ZR<M>::Q, J = ZR<M>::J, P = ZR<M>::P, BPT = ZR<M>::BPT;
    constexpr int pitch = ZRSmem<T, M>::pitch;
    const bool    t0    = t == 0;
    // step 1: Q-point DFTs over c for b = t + P s, to shared
#pragma unroll
    for (int s = 0; s < BPT; s++) {
        const int b = t + P * s;
        dft_reg<T, Q, -1>(in[s]);
        zr_line_store<T, Q>(S + b * pitch, in[s]);
    }
    __syncwarp();
    // step 2: twiddle e^{-2 pi i a b / M}, J-point DFTs over b per residue
    cplx<T> z[2][J];
#pragma unroll
    for (int r = 0; r < 2; r++) {
#pragma unroll
        for (int b = 0; b < J; b++) z[r][b] = S[b * pitch + a[r]];
#pragma unroll
        for (int b = 1; b < J; b++) z[r][b] = cmul(z[r][b], zr_tw<T>(twM + ((a[r] * b) & (M - 1))));
        dft_reg<T, J, -1>(z[r]);
    }
    __syncwarp();
    // X[k] = E + W_2M^k O with the mirror Z[M-k] from the thread's own values
    // (for k = 0 the mirror is Z[0] itself)
    const cplx<T> z0 = z[0][0];
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
        for (int j = 0; j < J; j++) {
            const cplx<T> zm = zr_mirror<T, J>(z, z0, t0, r, j);
            cplx<T>       w  = cplx<T>{(T)0.5 * wb[r].re, (T)0.5 * wb[r].im};
            twiddle_mul<T, 2 * J, -1>(w, j);  // e^{-2 pi i (a + Q j) / (2M)} / 2
            kv[r][j] = r2c_split<T>(z[r][j], zm, w);
        }
    xn = cplx<T>{z0.re - z0.im, (T)0};  // X[M] (used by t = 0 only)
}

// ---------------------------------------------------------------------------
// Kernels.  R rows per CTA (R * P a multiple of 32); blockIdx.y selects the
// field (c2r / r2c) or the run of a batched pool (products).
// ---------------------------------------------------------------------------
template <typename T, int M>
constexpr int zr_rows() {
    // 16 rows (32 for P < 2), fewer while the row blocks pass 40 KB; R * P
    // stays a multiple of 32
    constexpr int base = ZR<M>::P >= 2 ? 16 : 32;
    constexpr int minr = 32 / ZR<M>::P;
    int r = base;
    while (r > minr && r * ZRSmem<T, M>::blk > 40960) r /= 2;
    return r;
}

// Inverse z pass: complex rows -> real rows scaled by `scale` (in place
// allowed); inputs kz >= kz_keep read as zero.
template <typename T, int M, int R>
__device__ __forceinline__ void zr_c2r_rows(unsigned char *smem, const cplx<T> *in, T *out, size_t field_stride_c,
                                            size_t field_stride_real, int nrows, int hnzp,
                                            const cplx<T> *__restrict__ twM, const cplx<T> *__restrict__ twN, T scale,
                                            int kz_keep) {
    constexpr int P = ZR<M>::P, Q = ZR<M>::Q, J = ZR<M>::J, BPT = ZR<M>::BPT;
    const int  r   = threadIdx.x / P;
    const int  t   = threadIdx.x % P;
    const int  row = blockIdx.x * R + r;
    const bool ok  = row < nrows;
    const cplx<T> *rin = in + (size_t)blockIdx.y * field_stride_c + (size_t)(ok ? row : 0) * hnzp;
    T *rout            = out + (size_t)blockIdx.y * field_stride_real + (size_t)(ok ? row : 0) * 2 * hnzp;
    cplx<T>       *S   = reinterpret_cast<cplx<T> *>(smem + r * ZRSmem<T, M>::blk);
    int     a[2];
    cplx<T> wb[2], kv[2][J], xn, z[BPT][Q];
    zr_residues<T, M>(t, a, wb, twN);
    zr_load_k<T, M>(rin, ok, a, kz_keep, kv, xn);
    zr_c2r<T, M>(t, a, wb, kv, xn, S, twM, scale, z);
    if (!ok) return;
    using V2 = typename vec2_of<T>::type;
#pragma unroll
    for (int s = 0; s < BPT; s++)
#pragma unroll
        for (int c = 0; c < Q; c++) {
            V2 p;
            p.x = z[s][c].re;
            p.y = z[s][c].im;
            reinterpret_cast<V2 *>(rout)[(t + P * s) + J * c] = p;
        }
    if (t == 0)
        for (int k = 2 * M; k < 2 * hnzp; k++) rout[k] = (T)0;
}
template <typename T, int M, int R>
__global__ void __launch_bounds__(R *ZR<M>::P)
    zr_c2r_kernel(const cplx<T> *in, T *out, size_t field_stride_c, size_t field_stride_real, int nrows, int hnzp,
                  const cplx<T> *__restrict__ twM, const cplx<T> *__restrict__ twN, T scale, int kz_keep) {
    __shared__ __align__(16) unsigned char smem[R * ZRSmem<T, M>::blk];
    zr_c2r_rows<T, M, R>(smem, in, out, field_stride_c, field_stride_real, nrows, hnzp, twM, twN, scale, kz_keep);
}
// The same pass with the registers capped for MINB resident CTAs per SM.
template <typename T, int M, int R, int MINB>
__global__ void __launch_bounds__(R *ZR<M>::P, MINB)
    zr_c2r_kernel_capped(const cplx<T> *in, T *out, size_t field_stride_c, size_t field_stride_real, int nrows,
                         int hnzp, const cplx<T> *__restrict__ twM, const cplx<T> *__restrict__ twN, T scale,
                         int kz_keep) {
    __shared__ __align__(16) unsigned char smem[R * ZRSmem<T, M>::blk];
    zr_c2r_rows<T, M, R>(smem, in, out, field_stride_c, field_stride_real, nrows, hnzp, twM, twN, scale, kz_keep);
}

// Forward z pass: real rows -> complex rows (in place allowed); outputs kz >=
// kz_span are not written.
template <typename T, int M, int R>
__global__ void __launch_bounds__(R *ZR<M>::P)
    zr_r2c_kernel(const T *in, cplx<T> *out, size_t field_stride_real, size_t field_stride_c, int nrows, int hnzp,
                  const cplx<T> *__restrict__ twM, const cplx<T> *__restrict__ twN, int kz_span) {
    constexpr int P = ZR<M>::P, Q = ZR<M>::Q, J = ZR<M>::J, BPT = ZR<M>::BPT;
    __shared__ __align__(16) unsigned char smem[R * ZRSmem<T, M>::blk];
    const int  r   = threadIdx.x / P;
    const int  t   = threadIdx.x % P;
    const int  row = blockIdx.x * R + r;
    const bool ok  = row < nrows;
    const T   *rin  = in + (size_t)blockIdx.y * field_stride_real + (size_t)(ok ? row : 0) * 2 * hnzp;
    cplx<T>   *rout = out + (size_t)blockIdx.y * field_stride_c + (size_t)(ok ? row : 0) * hnzp;
    cplx<T>   *S    = reinterpret_cast<cplx<T> *>(smem + r * ZRSmem<T, M>::blk);
    using V2        = typename vec2_of<T>::type;
    int     a[2];
    cplx<T> wb[2], kv[2][J], xn, z[BPT][Q];
    zr_residues<T, M>(t, a, wb, twN);
#pragma unroll
    for (int s = 0; s < BPT; s++)
#pragma unroll
        for (int c = 0; c < Q; c++) {
            if (ok) {
                const V2 p = reinterpret_cast<const V2 *>(rin)[(t + P * s) + J * c];
                z[s][c]    = cplx<T>{p.x, p.y};
            } else {
                z[s][c] = cplx<T>{0, 0};
            }
        }
    zr_r2c<T, M>(t, a, wb, z, S, twM, kv, xn);
    zr_store_k<T, M>(rout, ok, t, a, kz_span, hnzp, kv, xn);
}

// The five advection products (U2advection_k, operate_omega.cxx:40-44) as
// A * B with A, B linear in (u1, u2, u3):  u2 u3, u3 u1, u1 u2,
// (u2 - u3)(u2 + u3), (u3 - u1)(u3 + u1).  With coefficients 0 and +-1 every
// factor is formed exactly as the direct sums and differences are, so the
// result is the same to the last bit, and a product index known only at run
// time costs a few fused multiply-adds instead of a chain of selects (which
// kept every candidate product alive in registers).
struct AdvCoef {
    float c[6];  // A = c0 u1 + c1 u2 + c2 u3,  B = c3 u1 + c4 u2 + c5 u3
};
__device__ __forceinline__ AdvCoef advection_coef(int p) {
    AdvCoef k;
    const float tab[5][6] = {{0, 1, 0, 0, 0, 1}, {0, 0, 1, 1, 0, 0}, {1, 0, 0, 0, 1, 0}, {0, 1, -1, 0, 1, 1},
                             {-1, 0, 1, 1, 0, 1}};
#pragma unroll
    for (int i = 0; i < 6; i++)
        k.c[i] = p == 0 ? tab[0][i] : p == 1 ? tab[1][i] : p == 2 ? tab[2][i] : p == 3 ? tab[3][i] : tab[4][i];
    return k;
}
template <typename T>
__device__ __forceinline__ cplx<T> advection_product(const AdvCoef &k, const cplx<T> &x, const cplx<T> &y,
                                                     const cplx<T> &z) {
    const T a0 = k.c[0], a1 = k.c[1], a2 = k.c[2], b0 = k.c[3], b1 = k.c[4], b2 = k.c[5];
    const T are = a0 * x.re + a1 * y.re + a2 * z.re, bre = b0 * x.re + b1 * y.re + b2 * z.re;
    const T aim = a0 * x.im + a1 * y.im + a2 * z.im, bim = b0 * x.im + b1 * y.im + b2 * z.im;
    return cplx<T>{are * bre, aim * bim};
}

// Fused z pass of the advection term: inverse z of the three velocity rows
// (io fields 0..2), the five products, forward z of the products into io
// fields 0..4.  Inputs kz >= kz_keep read as zero; outputs kz >= kz_span not
// written.  UREG: the velocity rows stay in registers (3 V complex values per
// thread); otherwise each thread parks u_x and u_y in its own slots of
// dynamic shared memory (laid out thread-fastest, conflict-free) and keeps
// u_z in registers, so that more rows fit an SM.
template <typename T, int M, int R, bool UREG, int MINB = 1>
__global__ void __launch_bounds__(R *ZR<M>::P, MINB)
    zr_products_kernel(cplx<T> *io, size_t field_stride_c, size_t run_stride_c, int nrows, int hnzp,
                       const cplx<T> *__restrict__ twM, const cplx<T> *__restrict__ twN, T scale, int kz_keep,
                       int kz_span) {
    constexpr int P = ZR<M>::P, Q = ZR<M>::Q, J = ZR<M>::J, BPT = ZR<M>::BPT;
    constexpr int NT = R * P;
    extern __shared__ __align__(16) unsigned char zsmem[];
    io += (size_t)blockIdx.y * run_stride_c;  // run of a batched pool
    const int    r    = threadIdx.x / P;
    const int    t    = threadIdx.x % P;
    const int    row  = blockIdx.x * R + r;
    const bool   ok   = row < nrows;
    const size_t roff = (size_t)(ok ? row : 0) * hnzp;
    cplx<T>     *S    = reinterpret_cast<cplx<T> *>(zsmem + r * ZRSmem<T, M>::blk);
    cplx<T>     *Upark = reinterpret_cast<cplx<T> *>(zsmem + R * ZRSmem<T, M>::blk) + threadIdx.x;
    int     a[2];
    cplx<T> wb[2];
    zr_residues<T, M>(t, a, wb, twN);
    constexpr int UD = UREG ? 3 : 1;
    cplx<T>       u[UD][BPT][Q];
    if constexpr (UREG) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            cplx<T> kv[2][J], xn;
            zr_load_k<T, M>(io + d * field_stride_c + roff, ok, a, kz_keep, kv, xn);
            zr_c2r<T, M>(t, a, wb, kv, xn, S, twM, scale, u[d]);
        }
    } else {
        // u_x and u_y wait in shared memory, u_z stays in the registers it
        // was transformed into
#pragma unroll 1
        for (int d = 0; d < 3; d++) {
            cplx<T> kv[2][J], xn;
            zr_load_k<T, M>(io + d * field_stride_c + roff, ok, a, kz_keep, kv, xn);
            zr_c2r<T, M>(t, a, wb, kv, xn, S, twM, scale, u[0]);
            if (d == 2) break;
#pragma unroll
            for (int s = 0; s < BPT; s++)
#pragma unroll
                for (int c = 0; c < Q; c++) Upark[((d * BPT + s) * Q + c) * NT] = u[0][s][c];
        }
    }
#pragma unroll 1
    for (int p = 0; p < 5; p++) {
        const AdvCoef k = advection_coef(p);
        cplx<T>       in[BPT][Q];
#pragma unroll
        for (int s = 0; s < BPT; s++)
#pragma unroll
            for (int c = 0; c < Q; c++) {
                if constexpr (UREG) {
                    in[s][c] = advection_product<T>(k, u[0][s][c], u[1][s][c], u[2][s][c]);
                } else {
                    // only the two components product p needs
                    const cplx<T> zero{0, 0};
                    const cplx<T> ux = (p != 0 && p != 3) ? Upark[((0 * BPT + s) * Q + c) * NT] : zero;
                    const cplx<T> uy = (p != 1 && p != 4) ? Upark[((1 * BPT + s) * Q + c) * NT] : zero;
                    const cplx<T> uz = (p != 2) ? u[0][s][c] : zero;
                    in[s][c]         = advection_product<T>(k, ux, uy, uz);
                }
            }
        cplx<T> kv[2][J], xn;
        zr_r2c<T, M>(t, a, wb, in, S, twM, kv, xn);
        zr_store_k<T, M>(io + p * field_stride_c + roff, ok, t, a, kz_span, hnzp, kv, xn);
    }
}

// Dynamic shared memory of zr_products_kernel.
template <typename T, int M, int R, bool UREG>
constexpr size_t zr_products_smem() {
    return (size_t)R * ZRSmem<T, M>::blk + (UREG ? 0 : (size_t)2 * ZR<M>::V * R * ZR<M>::P * sizeof(cplx<T>));
}

}  // namespace spm
