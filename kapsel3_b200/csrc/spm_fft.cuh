// Hand-written 3D real FFT for sm_100a (FP64 and FP32), replacing Ooura's
// rdft3d / rdft3dsort + conjugation behind A2a_k / A_k2a
// (fft_wrapper.h:641-681, fftsg3d.c:554-709).
//
// Convention (FFTW r2c, as the reference produces after its conjugation):
//   forward  X[kx][ky][kz] = sum_xyz a(x,y,z) e^{-2 pi i (kx x/NX + ky y/NY + kz z/NZ)}
//            kz = 0..NZ/2, unnormalised
//   inverse  a = (1/(NX NY NZ)) sum_k X e^{+...}, imaginary parts of the kz=0
//            and kz=NZ/2 planes are discarded (c2r semantics)
//
// Three in-place passes over HBM, each a single kernel:
//   Z pass: real rows (contiguous) <-> complex rows; length-NZ real transform
//           done as an NZ/2-point complex four-step FFT in registers + shared
//           memory, with the even/odd split post-/pre-processing.
//   Y pass, X pass: length-N complex transforms along a strided axis; a CTA
//           owns W adjacent kz columns of N lines (W*16 B contiguous per
//           line) and runs a four-step N = N1*N2 FFT: step 1 loads straight
//           from HBM into registers (N2-point DFT per thread), twiddles,
//           transposes through shared memory, step 2 (N1-point DFTs) writes
//           straight back to HBM.
// Each pass reads and writes every element exactly once.
#pragma once

#include "spm_dft.cuh"
#include "spm_tma.cuh"

namespace spm {

// ---------------------------------------------------------------------------
// Pruning of a strided pass to the 2/3-retained modes.  The step's k-space
// updates only read and write |KX| < TRN_X, |KY| < TRN_Y, KZ < TRN_Z, so
//   * a pass only visits column tiles that cover kz < kz_cols,
//   * the X pass only visits outer lines (ky) with |KY| < outer_trn,
//   * an inverse pass reads input lines with |K| >= line_trn and columns
//     kz >= col_keep as zero (those modes are never written upstream).
// Every retained output is computed by exactly the same arithmetic as in the
// full pass.  PassPrune::full(hnz) is the unpruned pass.
// ---------------------------------------------------------------------------
struct PassPrune {
    int kz_cols;    // columns [0, kz_cols) are needed
    int outer_trn;  // > 0: only outer lines o with |K(o)| < outer_trn
    int line_trn;   // > 0: input lines with |K(n)| >= line_trn read as zero
    int col_keep;   // input columns kz >= col_keep read as zero
    int out_trn;    // > 0: only output lines with |K(n)| < out_trn are needed
    static PassPrune full(int hnz) { return PassPrune{hnz, 0, 0, hnz, 0}; }
};
// Lines a TMA box of a pruned pass covers: two boxes of h lines at 0 and
// N - h hold every line with |K| < trn (h = trn), one box of N lines
// otherwise.
__host__ __device__ __forceinline__ int pruned_box_lines(int n, int trn) { return (trn > 0 && 2 * trn < n) ? trn : n; }

__host__ __device__ __forceinline__ int signed_mode(int n, int len) { return n > len / 2 ? n - len : n; }
__host__ __device__ __forceinline__ int outer_count(int n_outer, int outer_trn) {
    return outer_trn > 0 ? 2 * outer_trn - 1 : n_outer;
}
// index oi of the visited outer lines -> outer line o
__host__ __device__ __forceinline__ int outer_line(int oi, int n_outer, int outer_trn) {
    return (outer_trn > 0 && oi >= outer_trn) ? oi + n_outer - (2 * outer_trn - 1) : oi;
}

// ---------------------------------------------------------------------------
// Strided complex pass (Y or X axis).
// Block b visits column tile ct = b % ct_used of outer line
// o = outer_line(b / ct_used); element n of column c lives at
//   base + o * outer_stride + ct * W + c + n * axis_stride
// ---------------------------------------------------------------------------
template <typename T, int N, int W, int DIR>
__global__ void __launch_bounds__(W *Split<N>::N1)
    fft_strided_kernel(cplx<T> *__restrict__ data, size_t field_stride, int ncols, int ct_used, int n_outer,
                       size_t outer_stride, size_t axis_stride, const cplx<T> *__restrict__ twN, PassPrune pr) {
    constexpr int N1 = Split<N>::N1;
    constexpr int N2 = Split<N>::N2;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cplx<T> *s = reinterpret_cast<cplx<T> *>(smem_raw);

    const int c   = threadIdx.x % W;
    const int g   = threadIdx.x / W;  // n1 in step 1, k1 base in step 2
    const int b   = blockIdx.x;
    const int col = (b % ct_used) * W + c;
    const int o   = outer_line(b / ct_used, n_outer, pr.outer_trn);
    const bool ok = col < ncols;
    const bool col_in = ok && col < pr.col_keep;
    cplx<T> *base = data + (size_t)blockIdx.y * field_stride + (size_t)o * outer_stride + col;

    // Step 1: N2-point DFTs over n2 for fixed n1 = g, input index n1 + N1*n2.
    cplx<T> v[N2];
#pragma unroll
    for (int m = 0; m < N2; m++) {
        const int n = g + N1 * m;
        const bool in = col_in && (pr.line_trn == 0 || abs(signed_mode(n, N)) < pr.line_trn);
        if (in) {
            v[m] = base[(size_t)n * axis_stride];
        } else {
            v[m] = cplx<T>{0, 0};
        }
    }
    dft_reg<T, N2, DIR>(v);
#pragma unroll
    for (int k1 = 1; k1 < N2; k1++) {
        cplx<T> w = twN[(g * k1) & (N - 1)];
        if (DIR > 0) w.im = -w.im;
        v[k1] = cmul(v[k1], w);
    }
#pragma unroll
    for (int k1 = 0; k1 < N2; k1++) s[(g + N1 * k1) * W + c] = v[k1];
    __syncthreads();

    // Step 2: N1-point DFTs over n1 for each k1 owned by this thread.
#pragma unroll
    for (int i = 0; i < N2 / N1; i++) {
        const int k1 = g + N1 * i;
        cplx<T>   u[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) u[n1] = s[(n1 + N1 * k1) * W + c];
        dft_reg<T, N1, DIR>(u);
        if (ok) {
#pragma unroll
            for (int k2 = 0; k2 < N1; k2++) base[(size_t)(k1 + N2 * k2) * axis_stride] = u[k2];
        }
    }
}

// ---------------------------------------------------------------------------
// Strided complex pass, persistent and TMA-pipelined.
// The field is a 4D tensor of T: {2*hnz (kz re/im), NY, NX, nfields}.  A tile
// is W kz-columns x N lines (box {2W, N, 1, 1} on the Y pass, {2W, 1, N, 1}
// on the X pass); in shared memory both arrive as [n][W] complex.  Each CTA
// walks its tiles through an S-deep ring of buffers: TMA loads run S-1 tiles
// ahead of the four-step FFT, results go back with TMA stores from the same
// buffer.  Columns >= hnz are outside the tensor: loads zero-fill them and
// stores clip them.
// ---------------------------------------------------------------------------
template <typename T, int N, int W, int DIR, int S>
__global__ void __launch_bounds__(W *Split<N>::N1)
    fft_strided_tma_kernel(const __grid_constant__ CUtensorMap lmap, const __grid_constant__ CUtensorMap smap,
                           int axis, int n_outer, int ct_used, int ntiles, const cplx<T> *__restrict__ twN,
                           unsigned int *err, PassPrune pr) {
    constexpr int  N1         = Split<N>::N1;
    constexpr int  N2         = Split<N>::N2;
    // lines per load / store box (lmap / smap): N, or two boxes of the
    // pruned line count (inputs outside them are zero, outputs outside them
    // are not needed)
    const int      hl         = pruned_box_lines(N, pr.line_trn);
    const int      hs         = pruned_box_lines(N, pr.out_trn);
    const unsigned load_bytes = (unsigned)((hl == N ? N : 2 * hl) * W * sizeof(cplx<T>));
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cplx<T>           *buf = reinterpret_cast<cplx<T> *>(smem_raw);
    __shared__ __align__(8) uint64_t full[S];

    const int tid = threadIdx.x;
    const int c   = tid % W;
    const int g   = tid / W;
    const int n_used = outer_count(n_outer, pr.outer_trn);
    auto coords = [&](int t, int &c0, int &c1, int &c2, int &c3) {
        const int ct = t % ct_used, rest = t / ct_used;
        const int o = outer_line(rest % n_used, n_outer, pr.outer_trn), f = rest / n_used;
        c0 = 2 * ct * W;
        c3 = f;
        if (axis == 1) {
            c1 = 0;
            c2 = o;
        } else {
            c1 = o;
            c2 = 0;
        }
    };
    if (tid == 0) {
        for (int b = 0; b < S; b++) mbar_init(&full[b], 1);
        fence_mbar_init();
    }
    __syncthreads();
    // tile t into ring buffer b: lines [0, hl) and, when pruned, [N - hl, N)
    auto load_tile = [&](int t, int b) {
        int c0, c1, c2, c3;
        coords(t, c0, c1, c2, c3);
        cplx<T> *dst = buf + (size_t)b * N * W;
        mbar_expect_tx(&full[b], load_bytes);
        tma_load_4d(dst, &lmap, c0, c1, c2, c3, &full[b]);
        if (hl < N) {
            const int sh = N - hl;
            tma_load_4d(dst + (size_t)sh * W, &lmap, c0, c1 + (axis == 1 ? sh : 0), c2 + (axis == 1 ? 0 : sh), c3,
                        &full[b]);
        }
    };
    if (tid == 0) {
        for (int b = 0; b < S; b++) {
            const int t = blockIdx.x + b * gridDim.x;
            if (t < ntiles) load_tile(t, b);
        }
    }
    // the step-1 twiddles of this thread's n1 = g are the same for every tile
    cplx<T> tw1[N2];
#pragma unroll
    for (int k1 = 1; k1 < N2; k1++) {
        tw1[k1] = twN[(g * k1) & (N - 1)];
        if (DIR > 0) tw1[k1].im = -tw1[k1].im;
    }
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
        const int b  = it % S;
        cplx<T>  *B  = buf + (size_t)b * N * W;
        const bool w = mbar_wait(&full[b], (unsigned)((it / S) & 1), err);
        if (!__syncthreads_and(w)) break;
        // step 1: N2-point DFTs over n2 for n1 = g, in place (pruned inputs
        // read as zero)
        const bool col_in = (t % ct_used) * W + c < pr.col_keep;
        cplx<T> v[N2];
#pragma unroll
        for (int m = 0; m < N2; m++) {
            const int n = g + N1 * m;
            v[m] = (col_in && (pr.line_trn == 0 || abs(signed_mode(n, N)) < pr.line_trn)) ? B[n * W + c]
                                                                                           : cplx<T>{0, 0};
        }
        dft_reg<T, N2, DIR>(v);
#pragma unroll
        for (int k1 = 1; k1 < N2; k1++) v[k1] = cmul(v[k1], tw1[k1]);
#pragma unroll
        for (int k1 = 0; k1 < N2; k1++) B[(g + N1 * k1) * W + c] = v[k1];
        __syncthreads();
        // step 2: N1-point DFTs over n1, results back in natural order
        cplx<T> out[N2 / N1][N1];
#pragma unroll
        for (int i = 0; i < N2 / N1; i++) {
            const int k1 = g + N1 * i;
#pragma unroll
            for (int n1 = 0; n1 < N1; n1++) out[i][n1] = B[(n1 + N1 * k1) * W + c];
            dft_reg<T, N1, DIR>(out[i]);
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < N2 / N1; i++) {
            const int k1 = g + N1 * i;
#pragma unroll
            for (int k2 = 0; k2 < N1; k2++) B[(k1 + N2 * k2) * W + c] = out[i][k2];
        }
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            int c0, c1, c2, c3;
            coords(t, c0, c1, c2, c3);
            tma_store_4d(&smap, c0, c1, c2, c3, B);
            if (hs < N) {
                const int sh = N - hs;
                tma_store_4d(&smap, c0, c1 + (axis == 1 ? sh : 0), c2 + (axis == 1 ? 0 : sh), c3, B + (size_t)sh * W);
            }
            bulk_commit();
            // refill the buffer of the previous iteration with the tile S
            // iterations after it, once its store has read shared memory
            if (it >= 1) {
                const int tn = t + (S - 1) * (int)gridDim.x;
                if (tn < ntiles) {
                    bulk_wait_read<1>();
                    load_tile(tn, (it - 1) % S);
                }
            }
        }
    }
    if (tid == 0) bulk_wait_all();
}

// ---------------------------------------------------------------------------
// Z pass building blocks: one row of NZ = 2M reals <-> M+1 complex, handled
// by P = Split<M>::N1 threads (t = 0..P-1) with a shared workspace row `s`.
// Every thread of the CTA must call these together (they synchronise).
//
// r2c_row: ld(n) returns the packed pair (x[2n], x[2n+1]) for n < M;
//          st(k, X) receives X[k] for k = 0..M.
// c2r_row: ld(k) returns X[k] for k = 0..M (imaginary parts of X[0] and X[M]
//          are discarded); st(n, z) receives z = (x[2n], x[2n+1]) * scale-
//          normalised output.
// ---------------------------------------------------------------------------
// Workspace index of a z-row transform: one complex of padding after every
// N1 values, so the step-2 reads of the four-step FFT (stride N1) hit
// distinct shared-memory banks.  ws_len<M> complex per row.
template <int M>
__device__ __forceinline__ int wsi(int i) {
    return i + i / Split<M>::N1;
}
// Row strides of the per-row shared buffers, in complex (pair) units: at
// least `need`, and congruent to the P = N1 threads of a row modulo the pairs
// per 128 bytes, so the rows that one shared-memory wavefront serves (a
// half-warp of 8-byte or a quarter-warp of 16-byte accesses) fall on
// disjoint banks.
template <typename T, int M>
constexpr int row_stride(int need) {
    constexpr int mod = 128 / (int)sizeof(cplx<T>);
    constexpr int p   = Split<M>::N1 % mod;
    const int     r   = need % mod;
    return need + ((p - r + mod) % mod);
}
template <typename T, int M>
constexpr int ws_len() {
    return row_stride<T, M>(M + 2 + (M + 1) / Split<M>::N1);
}

// The even/odd split of a length-2M real transform packed as M complex
// values: X[k] from Z[k], Z[M-k] (forward) and Z'[k] from X[k], X[M-k]
// (inverse, scaled by c).  w = e^{-2 pi i k / (2M)}.
template <typename T>
__device__ __forceinline__ cplx<T> r2c_split(const cplx<T> &zk, const cplx<T> &zmk, const cplx<T> &w) {
    const T er  = (T)0.5 * (zk.re + zmk.re);
    const T ei  = (T)0.5 * (zk.im - zmk.im);
    const T orr = (T)0.5 * (zk.im + zmk.im);
    const T oi  = (T)-0.5 * (zk.re - zmk.re);
    return cplx<T>{er + (w.re * orr - w.im * oi), ei + (w.re * oi + w.im * orr)};
}
template <typename T>
__device__ __forceinline__ cplx<T> c2r_split(const cplx<T> &xk, const cplx<T> &xmk, const cplx<T> &w, T c) {
    const T er  = c * (xk.re + xmk.re);
    const T ei  = c * (xk.im - xmk.im);
    const T dr  = c * (xk.re - xmk.re);
    const T di  = c * (xk.im + xmk.im);
    const T orr = dr * w.re + di * w.im;
    const T oi  = di * w.re - dr * w.im;
    return cplx<T>{er - oi, ei + orr};
}

// r2c_row_m: as r2c_row, with ldm(m) returning the input of element
// t + M1 m (m = 0..M2-1, a compile-time index after unrolling), so the row
// may come from registers.
template <typename T, int M, class LdM, class St>
__device__ __forceinline__ void r2c_row_m(int t, LdM ldm, cplx<T> *s, const cplx<T> *__restrict__ twM,
                                          const cplx<T> *__restrict__ twN, St st) {
    constexpr int M1 = Split<M>::N1;
    constexpr int M2 = Split<M>::N2;
    constexpr int P  = M1;
    cplx<T>       v[M2];
#pragma unroll
    for (int m = 0; m < M2; m++) v[m] = ldm(m);
    dft_reg<T, M2, -1>(v);
#pragma unroll
    for (int k1 = 1; k1 < M2; k1++) v[k1] = cmul(v[k1], twM[(t * k1) & (M - 1)]);
#pragma unroll
    for (int k1 = 0; k1 < M2; k1++) s[wsi<M>(t + M1 * k1)] = v[k1];
    __syncthreads();
    cplx<T> z[M2 / M1][M1];
#pragma unroll
    for (int i = 0; i < M2 / M1; i++) {
        const int k1 = t + M1 * i;
#pragma unroll
        for (int n1 = 0; n1 < M1; n1++) z[i][n1] = s[wsi<M>(n1 + M1 * k1)];
        dft_reg<T, M1, -1>(z[i]);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < M2 / M1; i++) {
        const int k1 = t + M1 * i;
#pragma unroll
        for (int k2 = 0; k2 < M1; k2++) s[wsi<M>(k1 + M2 * k2)] = z[i][k2];
    }
    __syncthreads();
    // X[k] = E[k] + W_N^k O[k],  E = (Z[k] + conj Z[M-k]) / 2,
    // O = -i (Z[k] - conj Z[M-k]) / 2,  k = 0..M.  A thread reads the pair
    // Z[k], Z[M-k] (k = t + P i <= M/2) once and forms X[k] and X[M-k].
    constexpr int H = M / 2;
#pragma unroll
    for (int i = 0; i <= H / P; i++) {
        const int k = t + P * i;
        if (k <= H) {
            const cplx<T> zk  = s[wsi<M>(k)];
            const cplx<T> zmk = s[wsi<M>((M - k) & (M - 1))];
            st(k, r2c_split<T>(zk, zmk, twN[k]));  // twN: e^{-2 pi i k / (2M)}, k = 0..M
            if (k != H) st(M - k, r2c_split<T>(zmk, zk, twN[M - k]));
        }
    }
    __syncthreads();
}

template <typename T, int M, class Ld, class St>
__device__ __forceinline__ void r2c_row(int t, Ld ld, cplx<T> *s, const cplx<T> *__restrict__ twM,
                                        const cplx<T> *__restrict__ twN, St st) {
    r2c_row_m<T, M>(t, [&](int m) { return ld(t + Split<M>::N1 * m); }, s, twM, twN, st);
}

// c2r_row_m: as c2r_row, with stm(m, z) receiving output element t + M1 m
// (m = 0..M2-1, compile-time after unrolling), so the row may stay in
// registers.
template <typename T, int M, class Ld, class StM>
__device__ __forceinline__ void c2r_row_m(int t, Ld ld, cplx<T> *s, const cplx<T> *__restrict__ twM,
                                          const cplx<T> *__restrict__ twN, T scale, StM stm) {
    constexpr int M1 = Split<M>::N1;
    constexpr int M2 = Split<M>::N2;
    constexpr int P  = M1;
    // Z'[k] = E' + i O',  E' = c (X[k] + conj X[M-k]),
    // O' = c (X[k] - conj X[M-k]) W_N^{-k},  k = 0..M-1.  A thread loads
    // the pair X[k], X[M-k] (k = t + P i <= M/2; all loads first, in flight
    // together) and writes Z'[k] and Z'[M-k]; the imaginary parts of X[0]
    // and X[M] are discarded.
    constexpr int H  = M / 2;
    constexpr int NI = H / P + 1;
    cplx<T>       xa[NI], xb[NI];
#pragma unroll
    for (int i = 0; i < NI; i++) {
        const int k = t + P * i;
        if (k <= H) {
            xa[i] = ld(k);
            xb[i] = k == H ? xa[i] : ld(M - k);
        }
    }
#pragma unroll
    for (int i = 0; i < NI; i++) {
        const int k = t + P * i;
        if (k <= H) {
            cplx<T> a = xa[i], b = xb[i];
            if (k == 0) a.im = b.im = 0;
            s[wsi<M>(k)] = c2r_split<T>(a, b, twN[k], scale);
            if (k != 0 && k != H) s[wsi<M>(M - k)] = c2r_split<T>(b, a, twN[M - k], scale);
        }
    }
    __syncthreads();
    cplx<T> v[M2];
#pragma unroll
    for (int m = 0; m < M2; m++) v[m] = s[wsi<M>(t + M1 * m)];
    dft_reg<T, M2, +1>(v);
#pragma unroll
    for (int k1 = 1; k1 < M2; k1++) {
        cplx<T> w = twM[(t * k1) & (M - 1)];
        w.im      = -w.im;
        v[k1]     = cmul(v[k1], w);
    }
#pragma unroll
    for (int k1 = 0; k1 < M2; k1++) s[wsi<M>(t + M1 * k1)] = v[k1];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < M2 / M1; i++) {
        const int k1 = t + M1 * i;
        cplx<T>   u[M1];
#pragma unroll
        for (int n1 = 0; n1 < M1; n1++) u[n1] = s[wsi<M>(n1 + M1 * k1)];
        dft_reg<T, M1, +1>(u);
#pragma unroll
        for (int k2 = 0; k2 < M1; k2++) stm(i + (M2 / M1) * k2, u[k2]);  // element k1 + M2 k2 = t + M1 m
    }
    __syncthreads();
}

template <typename T, int M, class Ld, class St>
__device__ __forceinline__ void c2r_row(int t, Ld ld, cplx<T> *s, const cplx<T> *__restrict__ twM,
                                        const cplx<T> *__restrict__ twN, T scale, St st) {
    c2r_row_m<T, M>(t, ld, s, twM, twN, scale,
                    [&](int m, const cplx<T> &z) { st(t + Split<M>::N1 * m, z); });
}

template <typename T>
__device__ __forceinline__ cplx<T> load_pair(const T *row, int n) {
    using V2   = typename vec2_of<T>::type;
    const V2 p = reinterpret_cast<const V2 *>(row)[n];
    return cplx<T>{p.x, p.y};
}
template <typename T>
__device__ __forceinline__ void store_pair(T *row, int n, cplx<T> z) {
    using V2 = typename vec2_of<T>::type;
    V2 p;
    p.x                             = z.re;
    p.y                             = z.im;
    reinterpret_cast<V2 *>(row)[n] = p;
}

// ---------------------------------------------------------------------------
// Z pass, forward: real rows -> complex rows (in and out may alias).
// in:  real row r at in + r*2*hnzp (2M reals used),   M = NZ/2
// out: complex row r at out + r*hnzp (M+1 values, padding zeroed); outputs
//      kz >= kz_span are not written (pruned transforms downstream read none)
// ---------------------------------------------------------------------------
template <typename T, int M, int R>
__global__ void __launch_bounds__(R *Split<M>::N1)
    fft_z_r2c_kernel(const T *in, cplx<T> *out, size_t field_stride_real, size_t field_stride_c, int nrows,
                     int hnzp, const cplx<T> *__restrict__ twM, const cplx<T> *__restrict__ twN, int kz_span) {
    constexpr int P = Split<M>::N1;
    __shared__ __align__(16) cplx<T> s[R][ws_len<T, M>()];
    const int r   = threadIdx.x / P;
    const int t   = threadIdx.x % P;
    const int row = blockIdx.x * R + r;
    const bool ok = row < nrows;
    const T *rin  = in + (size_t)blockIdx.y * field_stride_real + (size_t)(ok ? row : 0) * 2 * hnzp;
    cplx<T> *rout = out + (size_t)blockIdx.y * field_stride_c + (size_t)(ok ? row : 0) * hnzp;
    r2c_row<T, M>(
        t, [&](int n) { return ok ? load_pair<T>(rin, n) : cplx<T>{0, 0}; }, s[r], twM, twN,
        [&](int k, cplx<T> X) {
            if (ok && k < kz_span) rout[k] = X;
        });
    if (ok && kz_span > M)
        for (int k = M + 1 + t; k < hnzp; k += P) rout[k] = cplx<T>{0, 0};
}

// ---------------------------------------------------------------------------
// Z pass, inverse: complex rows -> real rows, output scaled by `scale`.
// Inputs kz >= kz_keep are read as zero (pruned transforms; hnz: none).
// ---------------------------------------------------------------------------
template <typename T, int M, int R>
__global__ void __launch_bounds__(R *Split<M>::N1)
    fft_z_c2r_kernel(const cplx<T> *in, T *out, size_t field_stride_c, size_t field_stride_real, int nrows,
                     int hnzp, const cplx<T> *__restrict__ twM, const cplx<T> *__restrict__ twN, T scale,
                     int kz_keep) {
    constexpr int P = Split<M>::N1;
    __shared__ __align__(16) cplx<T> s[R][ws_len<T, M>()];
    const int r   = threadIdx.x / P;
    const int t   = threadIdx.x % P;
    const int row = blockIdx.x * R + r;
    const bool ok = row < nrows;
    const cplx<T> *rin = in + (size_t)blockIdx.y * field_stride_c + (size_t)(ok ? row : 0) * hnzp;
    T *rout            = out + (size_t)blockIdx.y * field_stride_real + (size_t)(ok ? row : 0) * 2 * hnzp;
    c2r_row<T, M>(
        t, [&](int k) { return (ok && k < kz_keep) ? rin[k] : cplx<T>{0, 0}; }, s[r], twM, twN, scale,
        [&](int n, cplx<T> z) {
            if (ok) store_pair<T>(rout, n, z);
        });
    if (ok && t == 0)
        for (int k = 2 * M; k < 2 * hnzp; k++) rout[k] = (T)0;
}

// ---------------------------------------------------------------------------
// Fused Z pass of the advection term (U2advection_k, operate_omega.cxx:12-55):
// inverse z transform of the three velocity components, the five quadratic
// products in registers/shared memory, forward z transform of the products.
// io[0..2] hold u_hat (z-complex rows) on input; io[0..4] receive the
// z-transformed products u2u3, u3u1, u1u2, (u2-u3)(u2+u3), (u3-u1)(u3+u1).
// Inputs kz >= kz_keep are read as zero; outputs are written for kz <
// kz_span only (the pruned passes downstream read no further).
// ---------------------------------------------------------------------------
template <typename T, int M, int R>
__global__ void __launch_bounds__(R *Split<M>::N1)
    fft_z_products_kernel(cplx<T> *io, size_t field_stride_c, size_t run_stride_c, int nrows, int hnzp,
                          const cplx<T> *__restrict__ twM, const cplx<T> *__restrict__ twN, T scale, int kz_keep,
                          int kz_span) {
    constexpr int P     = Split<M>::N1;
    constexpr int PITCH = 2 * row_stride<T, M>(M + 2);  // reals per staged row (>= 2 * hnzp)
    io += (size_t)blockIdx.y * run_stride_c;  // run of a batched pool
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T       *U  = reinterpret_cast<T *>(smem_raw);                 // [3][R][PITCH]
    cplx<T> *ws = reinterpret_cast<cplx<T> *>(U + 3 * R * PITCH);   // [R][ws_len<M>]
    const int r   = threadIdx.x / P;
    const int t   = threadIdx.x % P;
    const int row = blockIdx.x * R + r;
    const bool ok = row < nrows;
    const size_t roff = (size_t)(ok ? row : 0) * hnzp;
    T *Ur[3] = {U + (0 * R + r) * PITCH, U + (1 * R + r) * PITCH, U + (2 * R + r) * PITCH};
    // Inverse z of the three velocity rows: each thread loads its pairs
    // X[k], X[M-k] straight from global memory (all in flight together) and
    // the real row lands in U[d].
#pragma unroll 1
    for (int d = 0; d < 3; d++) {
        const cplx<T> *rin = io + d * field_stride_c + roff;
        T             *ur  = Ur[d];
        c2r_row<T, M>(
            t, [&](int k) { return (ok && k < kz_keep) ? rin[k] : cplx<T>{0, 0}; }, ws + r * ws_len<T, M>(), twM, twN,
            scale, [&](int n, cplx<T> z) { store_pair<T>(ur, n, z); });
    }
#pragma unroll 1
    for (int p = 0; p < 5; p++) {
        cplx<T> *rout = io + p * field_stride_c + roff;
        r2c_row<T, M>(
            t,
            [&](int n) {
                const cplx<T> a = load_pair<T>(Ur[0], n), b = load_pair<T>(Ur[1], n), c = load_pair<T>(Ur[2], n);
                const T       xs[2] = {a.re, a.im}, ys[2] = {b.re, b.im}, zs[2] = {c.re, c.im};
                T             o[2];
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const T x = xs[e], y = ys[e], z = zs[e];
                    o[e] = p == 0 ? y * z : p == 1 ? z * x : p == 2 ? x * y : p == 3 ? (y - z) * (y + z)
                                                                                     : (z - x) * (z + x);
                }
                return cplx<T>{o[0], o[1]};
            },
            ws + r * ws_len<T, M>(), twM, twN,
            [&](int k, cplx<T> X) {
                if (ok && k < kz_span) rout[k] = X;
            });
        if (ok && kz_span > M)
            for (int k = M + 1 + t; k < hnzp; k += P) rout[k] = cplx<T>{0, 0};
    }
}

// ---------------------------------------------------------------------------
// The same fused Z pass with the three velocity rows kept in registers: the
// inverse transform leaves element t + M1 m of its row in slot m of thread
// t, which is the slot the forward transform of a product reads it from, so
// the products are formed in registers and only the transform workspace is
// in shared memory (for FP32 rows: 3 x M2 complex values per thread).
// ---------------------------------------------------------------------------
template <typename T, int M, int R>
__global__ void __launch_bounds__(R *Split<M>::N1)
    fft_z_products_reg_kernel(cplx<T> *io, size_t field_stride_c, size_t run_stride_c, int nrows, int hnzp,
                              const cplx<T> *__restrict__ twM, const cplx<T> *__restrict__ twN, T scale,
                              int kz_keep, int kz_span) {
    constexpr int P  = Split<M>::N1;
    constexpr int M2 = Split<M>::N2;
    __shared__ __align__(16) cplx<T> ws[R][ws_len<T, M>()];
    io += (size_t)blockIdx.y * run_stride_c;  // run of a batched pool
    const int    r    = threadIdx.x / P;
    const int    t    = threadIdx.x % P;
    const int    row  = blockIdx.x * R + r;
    const bool   ok   = row < nrows;
    const size_t roff = (size_t)(ok ? row : 0) * hnzp;
    cplx<T>      u[3][M2];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const cplx<T> *rin = io + d * field_stride_c + roff;
        c2r_row_m<T, M>(
            t, [&](int k) { return (ok && k < kz_keep) ? rin[k] : cplx<T>{0, 0}; }, ws[r], twM, twN, scale,
            [&](int m, const cplx<T> &z) { u[d][m] = z; });
    }
#pragma unroll 1
    for (int p = 0; p < 5; p++) {
        cplx<T> *rout = io + p * field_stride_c + roff;
        r2c_row_m<T, M>(
            t,
            [&](int m) {
                const T xs[2] = {u[0][m].re, u[0][m].im}, ys[2] = {u[1][m].re, u[1][m].im},
                        zs[2] = {u[2][m].re, u[2][m].im};
                T o[2];
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const T x = xs[e], y = ys[e], z = zs[e];
                    o[e] = p == 0 ? y * z : p == 1 ? z * x : p == 2 ? x * y : p == 3 ? (y - z) * (y + z)
                                                                                     : (z - x) * (z + x);
                }
                return cplx<T>{o[0], o[1]};
            },
            ws[r], twM, twN,
            [&](int k, cplx<T> X) {
                if (ok && k < kz_span) rout[k] = X;
            });
        if (ok && kz_span > M)
            for (int k = M + 1 + t; k < hnzp; k += P) rout[k] = cplx<T>{0, 0};
    }
}

}  // namespace spm
