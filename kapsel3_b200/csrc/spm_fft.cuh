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
//   Z pass: real rows (contiguous) <-> complex rows (spm_zrow.cuh);
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
#include "spm_zrow.cuh"

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
// Every wait on a ring buffer is bounded by wait_ns of the global timer.  A
// CTA whose wait runs out records SPM_DEVERR_TIMEOUT, stops, waits (bounded
// again) for the loads it has issued and not consumed, and returns.
// skip_loads != 0 is a test switch: the CTAs issue no load at all, so every
// first wait runs out with nothing in flight.
// ---------------------------------------------------------------------------
template <typename T, int N, int W, int DIR, int S>
__global__ void __launch_bounds__(W *Split<N>::N1)
    fft_strided_tma_kernel(const __grid_constant__ CUtensorMap lmap, const __grid_constant__ CUtensorMap smap,
                           int axis, int n_outer, int ct_used, int ntiles, const cplx<T> *__restrict__ twN,
                           unsigned int *err, PassPrune pr, unsigned long long wait_ns, int skip_loads) {
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
    // tile t into ring buffer b: lines [0, hl) and, when pruned, [N - hl, N).
    // last_issued (thread 0): the last iteration whose tile load was issued.
    int  last_issued = -1;
    auto load_tile   = [&](int t, int b) {
        if (skip_loads) return;
        last_issued = (t - (int)blockIdx.x) / (int)gridDim.x;
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
    int  it      = 0;
    bool stopped = false;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
        const int b  = it % S;
        cplx<T>  *B  = buf + (size_t)b * N * W;
        const bool w = mbar_wait(&full[b], (unsigned)((it / S) & 1), err, wait_ns);
        if (!__syncthreads_and(w)) {
            stopped = true;
            break;
        }
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
    if (tid == 0) {
        // after a timeout: the loads issued for iterations it.. are still
        // owed to this CTA's shared memory; wait for them (bounded) first
        if (stopped)
            for (int j = it; j <= last_issued; j++) mbar_wait(&full[j % S], (unsigned)((j / S) & 1), nullptr, wait_ns);
        bulk_wait_all();
    }
}

}  // namespace spm
