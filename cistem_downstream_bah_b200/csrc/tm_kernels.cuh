// tm_kernels.cuh -- the search kernels for one batch of orientations.
//
// Data flow per orientation (o) of a batch, T = template box, X x Y = padded
// micrograph, XP = row pitch of half-spectra in complex values (X/2+1 rounded
// up to a multiple of the pass-B column chunk):
//
//   k_slice_colfft   Fourier slice of the 3-D template (trilinear, Hermitian
//                    mirror; image.cpp:2450-2607, 2899-3020) x (-1)^(i+j)
//                    (SwapRealSpaceQuadrants) x projection filter, then the
//                    inverse FFT along y of each of the T/2+1 columns
//   k_row_c2r        inverse c2r FFT of each row -> real T x T projection,
//                    plus per-row sums for the edge mean and variance
//   k_norm           per-orientation edge mean e and 1/sigma
//                    (match_template.cpp:1060-1068)
//   k_pass_a         (p - e)/sigma, placed at the origin of an X-wide row and
//                    forward FFT along x using only its T non-zero samples
//                    (X/T twiddled T-point FFTs) -> A[o][row][kx]
//   k_pass_b         per column kx: pruned forward FFT along y of the T rows
//                    of A, multiply by the prepared micrograph spectrum
//                    I'[ky][kx] (whitened spectrum x conj(placement phase) / N,
//                    DC zero), inverse FFT along y -> C[o][y][kx]
//   k_pass_c         per row y: c2r FFT along x of C[o][y][:] and, in
//                    registers, the MIP / argmax / sum / sum-of-squares /
//                    histogram update of match_template.cpp:1102-1149 over the
//                    batch; per-pixel state is read and written once per batch
//
// The placement of the projection at (X/2 - T/2, Y/2 - T/2)
// (ClipIntoLargerRealSpace2D, image.cpp:8398-8465), the forward-FFT scaling
// 1/N and the zeroed central pixel are folded into I' once per micrograph.
#pragma once
#include <cuda_fp16.h>
#include <float.h>
#include "tm_fft.cuh"
#include "tm_ptx.cuh"

namespace tmk {

using tmfft::cmul;
using tmfft::cmul_conj;
using tmfft::Twiddles;

__host__ __device__ constexpr int round_up16(int v) { return (v + 15) / 16 * 16; }
// region stride >= len whose value mod 16 equals `rem` (bank skew between regions)
__host__ __device__ constexpr int skewed(int len, int rem) { return round_up16(len) + rem; }

// Length of the pruned forward transform of T non-zero samples inside an
// N-point transform: the smallest L >= T that divides N and that the radix-V
// plan can split.  The N-point spectrum is then N/L twiddled L-point
// transforms of the zero-padded samples.
__host__ __device__ constexpr int prune_len(int T, int N, int V) {
    for (int L = T; L <= N; L++)
        if (N % L == 0 && tmfft::plannable(L, V)) return L;
    return -1;
}
// values per thread of the column transforms: 16 for powers of two, 18 for
// heights with a factor 3
__host__ __device__ constexpr int col_radix(int Y) { return Y % 3 == 0 ? 18 : 16; }

struct BatchArgs {
    int nb;                       // orientations in this batch
    int orient0;                  // index of the batch's first orientation within the plane
    long long gidx0;              // global orientation index of the batch's first orientation
    const float* rot;             // plane rotation table: 6 floats per orientation (m00 m01 m10 m11 m20 m21)
    const float2* tmpl;           // T*T*(T/2+1) template spectrum
    const float* filter;          // T*(T/2+1) projection filter
    float2* S;                    // nb * T * (T/2+1)
    float* P;                     // nb * T * T
    double* rowstat;              // nb * T * 4
    float2* norm;                 // nb: (edge mean, 1/sigma)
    float2* A;                    // nb * T * XP
    float2* C;                    // nb * Y * XP
    const float2* Ip;             // Y * XP prepared micrograph spectrum
    float* mip;                   // Y * X
    int* best;                    // Y * X
    double* sum;                  // Y * X
    double* sumsq;                // Y * X
    unsigned long long* hist;     // hist_bins
    float hist_min, hist_inv_step;
    int hist_bins;
    int* err;                     // device error flag (a bounded wait ran out)
    int half_scale_exp;           // FP16 form: the correlation spectra are stored times 2^half_scale_exp
    int tc_iexp, tc_zexp;         // FP16 column pass: I' held times 2^tc_iexp, stage-1 operand Z times 2^tc_zexp
    long long norm_pixels;        // pixel count of the projection variance (0: X*Y, the box;
                                  // a window of a larger micrograph passes the micrograph's)
    int XP;                       // row pitch (complex values) of A, C and Ip: X/2+1 rounded
                                  // up to a multiple of the pass-B column chunk
    Twiddles tw;                  // x axis (passes A and C): every length divides X
    Twiddles twy;                 // y axis (pass B): every length divides Y
    Twiddles twt;                 // template box (slice and projection kernels): lengths divide T
};

// --------------------------------------------------------------------------------------
// Trilinear Fourier interpolation with the reference's bounds and Hermitian rules
// (Image::ReturnLinearInterpolatedFourier, image.cpp:2899-3020), even T.
template <int T>
__device__ __forceinline__ float2 interp3(const float2* __restrict__ vol, float x, float y, float z) {
    constexpr int TP = T / 2 + 1;
    const int lb = -(T / 2), ub = T / 2 - 1;
    float2 acc = make_float2(0.f, 0.f);
    if (x >= 0.f) {
        int i0 = (int)floorf(x);
        if (i0 + 1 > T / 2) return acc;
        int j0 = (int)floorf(y);
        if (j0 < lb || j0 + 1 > ub) return acc;
        int k0 = (int)floorf(z);
        if (k0 < lb || k0 + 1 > ub) return acc;
        const float wx1 = x - (float)i0, wx0 = 1.f - wx1;
#pragma unroll
        for (int dk = 0; dk < 2; dk++) {
            const int k = k0 + dk;
            const int pz = k >= 0 ? k : T + k;
            const float wz = 1.f - fabsf(z - (float)k);
#pragma unroll
            for (int dj = 0; dj < 2; dj++) {
                const int j = j0 + dj;
                const int py = j >= 0 ? j : T + j;
                const float w = wz * (1.f - fabsf(y - (float)j));
                const float2* row = vol + ((size_t)pz * T + py) * TP;
                const float2 a = __ldg(row + i0), b = __ldg(row + i0 + 1);
                acc.x = fmaf(a.x, w * wx0, acc.x);
                acc.y = fmaf(a.y, w * wx0, acc.y);
                acc.x = fmaf(b.x, w * wx1, acc.x);
                acc.y = fmaf(b.y, w * wx1, acc.y);
            }
        }
    } else {
        int i0 = (int)floorf(x);
        if (i0 < -(T / 2)) return acc;
        int j0 = (int)floorf(y);
        if (j0 < lb || j0 + 1 > ub) return acc;
        int k0 = (int)floorf(z);
        if (k0 < lb || k0 + 1 > ub) return acc;
        const float wx1 = x - (float)i0, wx0 = 1.f - wx1;
#pragma unroll
        for (int dk = 0; dk < 2; dk++) {
            const int k = k0 + dk;
            const int pz = k > 0 ? T - k : -k;
            const float wz = 1.f - fabsf(z - (float)k);
#pragma unroll
            for (int dj = 0; dj < 2; dj++) {
                const int j = j0 + dj;
                const int py = j > 0 ? T - j : -j;
                const float w = wz * (1.f - fabsf(y - (float)j));
                const float2* row = vol + ((size_t)pz * T + py) * TP;
                // mirrored samples at x indices -i0 and -(i0+1), conjugated
                const float2 a = __ldg(row - i0), b = __ldg(row - i0 - 1);
                acc.x = fmaf(a.x, w * wx0, acc.x);
                acc.y = fmaf(-a.y, w * wx0, acc.y);
                acc.x = fmaf(b.x, w * wx1, acc.x);
                acc.y = fmaf(-b.y, w * wx1, acc.y);
            }
        }
    }
    return acc;
}

// --------------------------------------------------------------------------------------
// k_slice_colfft: block = CB columns x (T/V) threads (column fastest);
// grid = (ceil((T/2+1)/CB), nb)
template <int T>
struct SliceCol {
    static constexpr int V = T % 3 == 0 ? 24 : 16;   // values per thread
    static constexpr int PT = T / V;                 // threads per column
    static constexpr int RS = skewed(tmfft::padded_len(T), 1);
    static constexpr int CB = (16 * RS * 8 <= 48 * 1024) ? 16 : (8 * RS * 8 <= 48 * 1024) ? 8 : 4;   // columns per block
    static constexpr int NT = CB * PT;
};

template <int T>
__global__ void __launch_bounds__(SliceCol<T>::NT)
k_slice_colfft(BatchArgs a) {
    using SC = SliceCol<T>;
    constexpr int TP = T / 2 + 1;
    constexpr int PT = SC::PT, V = SC::V, CB = SC::CB, RS = SC::RS;
    __shared__ float2 sm[CB * RS];
    const int il = threadIdx.x % CB, tp = threadIdx.x / CB;
    const int i = blockIdx.x * CB + il;
    const int o = blockIdx.y;
    const bool valid = i <= T / 2;
    const float* m = a.rot + 6 * (size_t)(a.orient0 + o);
    const float m00 = __ldg(m), m01 = __ldg(m + 1), m10 = __ldg(m + 2), m11 = __ldg(m + 3), m20 = __ldg(m + 4), m21 = __ldg(m + 5);
    float2 v[V];
#pragma unroll
    for (int r = 0; r < V; r++) {
        const int y = tp + PT * r;
        const int j = y < T / 2 ? y : y - T;
        float2 val = make_float2(0.f, 0.f);
        if (valid) {
            if (i == 0) {
                if (j != 0) {
                    // j > 0 and j = -T/2 interpolate at (0, j); other j < 0 mirror (0, -j)
                    const int jj = (j > 0 || j == -(T / 2)) ? j : -j;
                    const float fy = (float)jj;
                    val = interp3<T>(a.tmpl, __fmul_rn(m01, fy), __fmul_rn(m11, fy), __fmul_rn(m21, fy));
                    if (jj != j) val.y = -val.y;
                }
            } else {
                // RotateCoords (matrix.h:32-37) in float without fused multiply-add,
                // so that samples on the box boundary are kept or dropped exactly
                // as the reference does
                const float fx = (float)i, fy = (float)j;
                val = interp3<T>(a.tmpl, __fadd_rn(__fmul_rn(m00, fx), __fmul_rn(m01, fy)),
                                 __fadd_rn(__fmul_rn(m10, fx), __fmul_rn(m11, fy)),
                                 __fadd_rn(__fmul_rn(m20, fx), __fmul_rn(m21, fy)));
            }
            float f = __ldg(a.filter + (size_t)y * TP + i);
            if ((i + j) & 1) f = -f;
            val.x *= f;
            val.y *= f;
        }
        v[r] = val;
    }
    tmfft::fft<T, V, +1>(v, tp, sm + il * RS, a.twt, [] __device__() { __syncthreads(); });
    if (valid) {
        float2* out = a.S + (size_t)o * T * TP;
#pragma unroll
        for (int r = 0; r < V; r++) out[(size_t)(tp + PT * r) * TP + i] = v[r];
    }
}

// --------------------------------------------------------------------------------------
// k_row_c2r: each row of T/2+1 complex -> T reals via a T/2-point inverse FFT
// (even/odd packing; imaginary parts of the DC and Nyquist terms ignored as in
// FFTW's c2r).  block = ROWS rows x PH threads; grid = (T/ROWS, nb).
template <int T>
struct RowC2R {
    static constexpr int H = T / 2;
    static constexpr int V = H % 3 == 0 ? 24 : 16;              // values per thread
    static constexpr int PH = H / V;                            // threads per row
    static constexpr int RS = skewed(tmfft::padded_len(H), PH % 16);
    static constexpr int ROWS0 = (256 / PH) < T ? (256 / PH) : T;
    static constexpr int ROWS = (ROWS0 * RS * 8 <= 48 * 1024) ? ROWS0 : ROWS0 / 2;   // rows per block
    static constexpr int NT = ROWS * PH;
    static_assert(32 % PH == 0 || PH % 32 == 0, "row reductions use warp shuffles");
};

template <int T>
__global__ void __launch_bounds__(RowC2R<T>::NT)
k_row_c2r(BatchArgs a) {
    using RC = RowC2R<T>;
    constexpr int TP = T / 2 + 1, H = RC::H, PH = RC::PH, ROWS = RC::ROWS, V = RC::V;
    constexpr int RS = RC::RS;
    __shared__ float2 sm[ROWS * RS];
    const int t = threadIdx.x % PH, rl = threadIdx.x / PH;
    const int y = blockIdx.x * ROWS + rl;
    const int o = blockIdx.y;
    const float2* Hrow = a.S + ((size_t)o * T + y) * TP;
    float2 v[V];
#pragma unroll
    for (int r = 0; r < V; r++) {
        const int k = t + PH * r;
        float2 hk = Hrow[k];
        float2 hm = Hrow[H - k];
        if (k == 0) { hk.y = 0.f; hm.y = 0.f; }
        const float2 e = make_float2(hk.x + hm.x, hk.y - hm.y);
        const float2 d = make_float2(hk.x - hm.x, hk.y + hm.y);
        const float2 od = cmul(d, a.twt.template w<+1>(k, T));
        v[r] = make_float2(e.x - od.y, e.y + od.x);
    }
    tmfft::fft<H, V, +1>(v, t, sm + rl * RS, a.twt, [] __device__() { __syncthreads(); });
    float* prow = a.P + ((size_t)o * T + y) * T;
    float s = 0.f, q = 0.f;
#pragma unroll
    for (int r = 0; r < V; r++) {
        const int mm = t + PH * r;
        reinterpret_cast<float2*>(prow)[mm] = v[r];
        s += v[r].x + v[r].y;
        q = fmaf(v[r].x, v[r].x, fmaf(v[r].y, v[r].y, q));
    }
    double ds = s, dq = q;
#pragma unroll
    for (int off = PH / 2; off > 0; off >>= 1) {
        ds += __shfl_xor_sync(0xffffffffu, ds, off);
        dq += __shfl_xor_sync(0xffffffffu, dq, off);
    }
    // edge sum: full first and last rows, else the first and last pixel
    float e0 = 0.f, e1 = 0.f;
    if (t == 0) e0 = v[0].x;                                   // pixel 0 = z[0].x
    if (t == (H - 1) % PH) e1 = v[(H - 1) / PH].y;            // pixel T-1 = z[H-1].y
    float ee = e0 + e1;
#pragma unroll
    for (int off = PH / 2; off > 0; off >>= 1) ee += __shfl_xor_sync(0xffffffffu, ee, off);
    const double edge = (y == 0 || y == T - 1) ? ds : (double)ee;
    if (t == 0) {
        double* st = a.rowstat + ((size_t)o * T + y) * 4;
        st[0] = ds;
        st[1] = dq;
        st[2] = edge;
        st[3] = 0.0;
    }
}

// --------------------------------------------------------------------------------------
// k_norm: one warp per orientation.  e = edge mean (ReturnAverageOfRealValuesOnEdges,
// image.cpp:5907-5945); variance as match_template.cpp:1066-1067 with the
// mean of squares and the mean of the edge-subtracted projection.
template <int T>
__global__ void __launch_bounds__(256)
k_norm(BatchArgs a, long long n_image) {
    const int lane = threadIdx.x & 31;
    const int o = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (o >= a.nb) return;
    double s = 0, q = 0, e = 0;
    for (int y = lane; y < T; y += 32) {
        const double* st = a.rowstat + ((size_t)o * T + y) * 4;
        s += st[0];
        q += st[1];
        e += st[2];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, off);
        q += __shfl_xor_sync(0xffffffffu, q, off);
        e += __shfl_xor_sync(0xffffffffu, e, off);
    }
    if (lane == 0) {
        const double n = (double)T * T;
        const float edge_mean = (float)(e / (double)(4 * T - 4));
        const double em = edge_mean;
        const double s1 = s - n * em;                 // sum of (p - e)
        const double s2 = q - 2.0 * em * s + n * em * em;  // sum of (p - e)^2
        const double ratio = n / (double)n_image;
        const double var = (s2 / n) * ratio - ((s1 / n) * ratio) * ((s1 / n) * ratio);
        a.norm[o] = make_float2(edge_mean, (float)(1.0 / sqrt(var)));
    }
}

// --------------------------------------------------------------------------------------
// k_pass_a: one block per (row, orientation); X/16 threads, thread j = s + MX*t'.
// The T samples are the first T of an LA-point zero-padded input (LA = T when T
// divides X).
template <int T, int X>
__global__ void __launch_bounds__(X / 16)
k_pass_a(BatchArgs a) {
    const int XP = a.XP;
    constexpr int LA = prune_len(T, X, 16);
    constexpr int MX = X / LA, PT = LA / 16;
    constexpr int RS = skewed(tmfft::padded_len(LA), 1);
    static_assert(LA > 0, "no pruned row transform for this template and width");
    __shared__ float2 sm[MX * RS];
    __shared__ float q[T];
    const int j = threadIdx.x;
    const int s = j % MX, tp = j / MX;
    const int row = blockIdx.x, o = blockIdx.y;
    const float2 nrm = a.norm[o];
    const float* prow = a.P + ((size_t)o * T + row) * T;
    for (int m = j; m < T; m += X / 16) q[m] = (prow[m] - nrm.x) * nrm.y;
    __syncthreads();
    float2 v[16];
    const float2 w0 = a.tw.template w<-1>(s * tp, X);
    const float2 w1 = a.tw.template w<-1>(s * PT, X);
    float2 w = w0;
#pragma unroll
    for (int r = 0; r < 16; r++) {
        const int n = tp + PT * r;
        const float qv = (LA == T || n < T) ? q[n] : 0.f;
        v[r] = make_float2(qv * w.x, qv * w.y);
        w = cmul(w, w1);
    }
    tmfft::fft<LA, 16, -1>(v, tp, sm + s * RS, a.tw, [] __device__() { __syncthreads(); });
    float2* out = a.A + ((size_t)o * T + row) * XP;
#pragma unroll
    for (int r = 0; r < 16; r++) {
        const int kx = j + (X / 16) * r;
        if (kx <= X / 2) out[kx] = v[r];
    }
}

// --------------------------------------------------------------------------------------
// Work items of the column passes: (column group, orientation).  A block owns
// whole column groups, every orientation of a group in turn (its micrograph
// values stay in TMEM), and the blocks take adjacent groups in rounds: block b
// has groups b, b + nblk, b + 2 nblk, ...  All blocks then write rows of the
// same orientation at about the same time, into adjacent 32-byte sectors of
// each row, which the L2 merges into whole lines before writing them back.
// (With each block on a contiguous run of items, the blocks wrote rows of
// unrelated orientations one sector at a time, and the 4096 x 4096 column pass
// took 2.3 times as long as with its stores going to L2-resident addresses.)
// Groups left over after the whole rounds are split by orientation ranges over
// the blocks that would otherwise idle.
struct ColSchedule {
    int nb, nblk, b, rounds, tail_g, o_lo, n;
    __host__ __device__ ColSchedule(int ngroups, int nbatch, int blk, int nblocks) : nb(nbatch), nblk(nblocks), b(blk) {
        rounds = ngroups / nblk;
        const int rem = ngroups % nblk;
        const int parts = rem ? min(nb, nblk / rem) : 1;
        int o_hi = 0;
        tail_g = -1;
        o_lo = 0;
        if (rem && b < rem * parts) {
            const int p = b / rem;
            tail_g = rounds * nblk + b % rem;
            o_lo = p * nb / parts;
            o_hi = (p + 1) * nb / parts;
        }
        n = rounds * nb + (o_hi - o_lo);
    }
    // most items a block gets
    __host__ __device__ static int max_items(int ngroups, int nbatch, int nblocks) {
        return (ngroups + nblocks - 1) / nblocks * nbatch;
    }
    // (group, orientation) of the block's idx-th item.  k_pass_b keeps the schedule
    // in shared memory (its fields cost no registers across the item loop);
    // k_pass_b_rg expands it into a list of items there.
    __host__ __device__ void locate(int idx, int& g, int& o) const {
        if (idx < rounds * nb) {
            g = (idx / nb) * nblk + b;
            o = idx % nb;
        } else {
            g = tail_g;
            o = o_lo + idx - rounds * nb;
        }
    }
    // the same from the block's shared-memory copy, read afresh on every call
    __device__ static void locate(const volatile ColSchedule* s, int idx, int& g, int& o) {
        const int nb = s->nb, rounds = s->rounds;
        if (idx < rounds * nb) {
            g = (idx / nb) * s->nblk + s->b;
            o = idx % nb;
        } else {
            g = s->tail_g;
            o = s->o_lo + idx - rounds * nb;
        }
    }
};
static_assert(sizeof(ColSchedule) <= 48, "the schedule sits in the last 48 bytes of a column pass's shared memory");

// --------------------------------------------------------------------------------------
// k_pass_b: persistent; block = W columns x P threads (thread = c + W*j,
// P = Y/V); work item = (group of G column chunks, orientation), orientation
// fastest.  With 2-column chunks (tall micrographs, where 4 columns would need
// more than 1024 threads) an item covers two chunks one after the other and
// writes its 4 columns from shared memory, so every store fills whole 32-byte
// row sectors (16-byte partial-sector stores cost DRAM read-modify-writes).
// Each thread parks the V values of the prepared micrograph spectrum I' it
// multiplies with in tensor memory (TMEM, 2V columns of its lane) for all
// orientations of the chunk, which leaves shared memory to full complex
// exchange buffers; a trailing partial warp (when W*P is not a multiple of 32)
// reads its I' values from global memory instead, since tcgen05 loads are
// whole-warp operations.  The rows of A for the next item stream in with
// cp.async while the current item is transformed.  The forward transform
// along y is pruned: MY = Y/L twiddled L-point transforms of the T rows of A
// zero-padded to L (L = T for power-of-two heights).
template <int T, int Y>
struct PassB {
    // values per thread: the column radix.  (32 values -- two radix-16
    // butterflies per thread and stage, 512 threads -- compiles and passes the
    // same tests but measured no faster on 4096 x 4096.)
    static constexpr int V = col_radix(Y);
    static constexpr int P = Y / V;                                 // threads per column
    // columns per block; 32 values per thread need 128 registers: 512 threads
    static constexpr int W = V == 32 ? 4 : (16 * P <= 1024) ? 16 : (8 * P <= 1024) ? 8 : (4 * P <= 1024) ? 4 : 2;
    static constexpr int NT = W * P;                                // threads per block
    static constexpr int L = prune_len(T, Y, V);                    // pruned forward length
    static constexpr int MY = Y / L, PT = L / V;
    static constexpr int FULL_WARPS = NT / 32;
    // chunks written back to back for one orientation, so that together they
    // cover whole 32-byte sectors of a row (G > 1 only for 2-column chunks)
    static constexpr int G = W >= 4 ? 1 : 4 / W;
    static constexpr int WG = W * G;                                // columns per work item
    // A 1024-thread block of at least 8 columns runs as NH = 2 independent
    // halves of 512 threads (W/2 columns each, own named barrier), so that one
    // half's transforms issue while the other waits at a barrier.  A warp then
    // covers W/2 >= 4 adjacent columns, whole 32-byte sectors of each row.  (With
    // 4 columns each half would write 16-byte halves of the sectors; measured at
    // 4096 x 4096, the L2 did not merge them and the DRAM traffic of the pass
    // rose from 11 to 30 GB per 128 orientations, so 4-column blocks stay whole.)
    static constexpr int NH = (NT == 1024 && G == 1 && W >= 8) ? 2 : 1;
    static constexpr int WL = W / NH;                               // columns interleaved in a warp
    static constexpr int NTH = NT / NH;                             // threads per half
    // bank skews (float2 units, half-warp = 16 lanes = (16/WL) values of j x WL columns)
    static constexpr int RST = (tmfft::padded_len(L) + 15) / 16 * 16 + 1;       // == 1 (mod 16)
    static constexpr int CS0 = (MY * RST > tmfft::padded_len(Y)) ? MY * RST : tmfft::padded_len(Y);
    static constexpr int CS = (CS0 + 15) / 16 * 16 + 16 / WL;                 // == 16/WL (mod 16)
    static constexpr size_t EXCH = (sizeof(float2) * WG * CS + 15) / 16 * 16;
    static constexpr size_t ASZ = sizeof(float2) * T * WG;          // one A staging buffer
    static constexpr int ABUFS = (EXCH + 2 * ASZ + 64 <= 232448) ? 2 : 1;
    static constexpr size_t SMEM = EXCH + ABUFS * ASZ + 64;         // + TMEM address slot
    // TMEM: 2V columns per thread; the warps of one lane quadrant sit side by side
    static constexpr int TCOLS = 2 * V;
    static constexpr uint32_t TMEM_COLS = [] {
        const int need = ((FULL_WARPS + 3) / 4) * TCOLS * G;
        uint32_t n = 32;
        while ((int)n < need) n *= 2;
        return n;
    }();
    static_assert(L > 0 && Y % V == 0 && P % PT == 0, "no pruned plan for this template and height");
    static_assert(NT <= 1024 && SMEM <= 232448, "pass B block exceeds the per-block limits");
    static_assert(TMEM_COLS <= 512, "pass B TMEM layout exceeds 512 columns");
    static_assert(V == 16 || V == 18 || V == 32, "TMEM load sequence covers 16, 18 or 32 values");
    static_assert(NH == 1 || (NTH % 32 == 0 && W % NH == 0), "halves must be whole warps and whole columns");
};

// I' values of one thread (V complex, 2V floats) into its TMEM columns
template <int V>
__device__ __forceinline__ void tmem_put_values(uint32_t taddr, const float* f) {
    tmptx::tmem_st16(taddr, f);
    tmptx::tmem_st16(taddr + 16, f + 16);
    if constexpr (V == 18) tmptx::tmem_st4(taddr + 32, f + 32);
    if constexpr (V == 32) {
        tmptx::tmem_st16(taddr + 32, f + 32);
        tmptx::tmem_st16(taddr + 48, f + 48);
    }
}

// RB = 0: C[o][y][kx] in FP32 complex.  RB > 0 (the FP16 form): C in FP16
// complex times 2^half_scale_exp, rows interleaved in blocks of RB,
// C16[o][y / RB][kx][y % RB], so that a warp's stores (8 consecutive rows of 4
// columns) fill whole 32-byte sectors and the tensor-core row pass reads a
// block of RB rows with one bulk copy.
template <int T, int Y, int RB = 0>
__global__ void __launch_bounds__(PassB<T, Y>::NT, 1)
k_pass_b(BatchArgs a, int ngroups) {
    using PB = PassB<T, Y>;
    constexpr int W = PB::W, MY = PB::MY, PT = PB::PT, NT = PB::NT, V = PB::V, P = PB::P, L = PB::L;
    const int XP = a.XP;
    extern __shared__ __align__(16) unsigned char smem_b[];
    float2* exch = reinterpret_cast<float2*>(smem_b);
    float2* abuf = reinterpret_cast<float2*>(smem_b + PB::EXCH);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem_b + PB::EXCH + PB::ABUFS * PB::ASZ);
    volatile ColSchedule* sch = reinterpret_cast<volatile ColSchedule*>(smem_b + PB::EXCH + PB::ABUFS * PB::ASZ + 16);
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const bool tmem_warp = warp < PB::FULL_WARPS;   // uniform per warp
    constexpr int NH = PB::NH, WL = PB::WL, NTH = PB::NTH;
    // half h owns columns h*WL .. h*WL + WL - 1; within it thread = c' + WL*j
    const int h = tid / NTH, loc = tid % NTH;
    const int c = h * WL + loc % WL, j = loc / WL;
    const int s = j % MY, tp = j / MY;
    constexpr int G = PB::G, WG = PB::WG;
    // the barrier over the threads that share this thread's columns
    auto sync = [h]() {
        if constexpr (NH == 1) __syncthreads();
        else asm volatile("bar.sync %0, %1;" ::"r"(1 + h), "n"(NTH) : "memory");
    };
    if (tid == 0) {
        const ColSchedule cs(ngroups, a.nb, blockIdx.x, gridDim.x);
        sch->nb = cs.nb; sch->nblk = cs.nblk; sch->b = cs.b; sch->rounds = cs.rounds;
        sch->tail_g = cs.tail_g; sch->o_lo = cs.o_lo; sch->n = cs.n;
    }
    __syncthreads();
    const int n_items = sch->n;
    if (n_items == 0) return;
    if (warp == 0) {
        tmptx::tmem_alloc(tmem_slot, PB::TMEM_COLS);
        tmptx::tmem_relinquish();
    }
    tmptx::tmem_fence_before_sync();
    __syncthreads();
    tmptx::tmem_fence_after_sync();
    const uint32_t tmem = *tmem_slot + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(PB::TCOLS * G * (warp >> 2));
    // the item's T rows of A into dst[row][WG]: each half copies (and later
    // reads) only its own columns
    constexpr int WGH = WG / NH;   // the item's columns per half
    auto issue_rows = [&](int it, float2* dst) {
        int grp, oo;
        ColSchedule::locate(sch, it, grp, oo);
        const float2* src = a.A + (size_t)oo * T * XP + grp * WG + h * WGH;
        for (int e = loc; e < T * WGH; e += NTH) {
            const int row = e / WGH, cc = e % WGH;
            tmptx::cp_async8(dst + row * WG + h * WGH + cc, src + (size_t)row * XP + cc);
        }
    };
    if (PB::ABUFS == 2) {
        issue_rows(0, abuf);
        tmptx::cp_async_commit();
    }
    int cur_group = -1;
    for (int it = 0; it < n_items; it++) {
        const int kk = it;
        const float2* acur = abuf + (PB::ABUFS == 2 ? (kk & 1) : 0) * (T * WG);
        float2* anext = abuf + (PB::ABUFS == 2 ? ((kk + 1) & 1) : 0) * (T * WG);
        int group, o;
        ColSchedule::locate(sch, it, group, o);
        const int kx0 = group * WG;
        // twiddles of the pruned forward, W_Y^(s * (tp + PT*r)) = w0 * w1^r, loaded early
        // (with 32 values, from the table again every 8 values)
        const float2 w0 = a.twy.template w<-1>(s * tp, Y);
        const float2 w1 = a.twy.template w<-1>(s * PT, Y);
        // The buffer the next rows go into was last read at the start of the
        // previous item's forward transform, whose barriers every thread has
        // passed; the exchange buffers are guarded by the transforms' own barriers.
        // With a single staging buffer the rows are reloaded in place, after a barrier.
        // (Each half copies and reads only its own columns, so its own barrier suffices.)
        if (PB::ABUFS == 1) sync();
        if (PB::ABUFS == 2) {
            if (it + 1 < n_items) issue_rows(it + 1, anext);
            tmptx::cp_async_commit();
            tmptx::cp_async_wait<1>();
        } else {
            issue_rows(it, anext);
            tmptx::cp_async_commit();
            tmptx::cp_async_wait<0>();
        }
        sync();  // this item's rows of A are visible to every thread of the half
        if (group != cur_group && tmem_warp) {
            // the V I' values this thread multiplies with in each chunk of the
            // group, into its TMEM columns
#pragma unroll 1
            for (int g = 0; g < G; g++) {
                const float2* Ig = a.Ip + kx0 + g * W + c;
                float buf[2 * V];
#pragma unroll
                for (int r = 0; r < V; r++) {
                    const float2 iv = __ldg(Ig + (size_t)(j + P * r) * XP);
                    buf[2 * r] = iv.x;
                    buf[2 * r + 1] = iv.y;
                }
                tmem_put_values<V>(tmem + g * PB::TCOLS, buf);
            }
            tmptx::tmem_wait_st();
        }
        cur_group = group;
#pragma unroll 1
        for (int g = 0; g < G; g++) {
            const int col = g * W + c;   // column within the item
            float2* colbuf = exch + col * PB::CS;
            float2* fwdbuf = colbuf + s * PB::RST;
            const uint32_t tslot = tmem + g * PB::TCOLS;
            float2 v[V];
            {
                float2 w = w0;
#pragma unroll
                for (int r = 0; r < V; r++) {
                    if (V == 32 && r % 8 == 0 && r > 0) w = a.twy.template w<-1>(s * (tp + PT * r), Y);
                    const int n = tp + PT * r;   // rows n >= T of the L-point input are zero
                    v[r] = (L == T || n < T) ? cmul(acur[n * WG + col], w) : make_float2(0.f, 0.f);
                    w = cmul(w, w1);
                }
            }
            // every thread passed the item barrier since the buffers were last read
            tmfft::fft<L, V, -1, false>(v, tp, fwdbuf, a.twy, sync);
            // thread (s, tp) holds F[k], k = s + MY*(tp + PT*r) = j + P*r
            if (tmem_warp) {
                float iv[16];
                tmptx::tmem_ld16(tslot, iv);
                tmptx::tmem_wait_ld();
                float iw[16], ix[4];
                tmptx::tmem_ld16(tslot + 16, iw);   // in flight while the first values are multiplied
                if constexpr (V == 18) tmptx::tmem_ld4(tslot + 32, ix);
#pragma unroll
                for (int r = 0; r < 8; r++) v[r] = cmul_conj(make_float2(iv[2 * r], iv[2 * r + 1]), v[r]);
                tmptx::tmem_wait_ld();
                if constexpr (V == 32) tmptx::tmem_ld16(tslot + 32, iv);
#pragma unroll
                for (int r = 0; r < 8; r++) v[8 + r] = cmul_conj(make_float2(iw[2 * r], iw[2 * r + 1]), v[8 + r]);
                if constexpr (V == 18) {
                    v[16] = cmul_conj(make_float2(ix[0], ix[1]), v[16]);
                    v[17] = cmul_conj(make_float2(ix[2], ix[3]), v[17]);
                }
                if constexpr (V == 32) {
                    tmptx::tmem_wait_ld16(iv);
                    tmptx::tmem_ld16(tslot + 48, iw);
#pragma unroll
                    for (int r = 0; r < 8; r++) v[16 + r] = cmul_conj(make_float2(iv[2 * r], iv[2 * r + 1]), v[16 + r]);
                    tmptx::tmem_wait_ld16(iw);
#pragma unroll
                    for (int r = 0; r < 8; r++) v[24 + r] = cmul_conj(make_float2(iw[2 * r], iw[2 * r + 1]), v[24 + r]);
                }
            } else {
                const float2* Ic = a.Ip + kx0 + col;
#pragma unroll
                for (int r = 0; r < V; r++) v[r] = cmul_conj(__ldg(Ic + (size_t)(j + P * r) * XP), v[r]);
            }
            tmfft::fft<Y, V, +1>(v, j, colbuf, a.twy, sync);
            if constexpr (RB > 0) {
                static_assert(G == 1 && Y % RB == 0 && (P % RB == 0), "FP16 output needs whole-column chunks");
                // row j + P r sits in block j / RB + r P / RB at position j % RB (RB divides P)
                const float sc = __int_as_float((127 + a.half_scale_exp) << 23);   // 2^e
                __half2* Co = reinterpret_cast<__half2*>(a.C) + (size_t)o * Y * XP +
                              ((size_t)(j / RB) * XP + kx0 + col) * RB + (j % RB);
#pragma unroll
                for (int r = 0; r < V; r++) {   // streaming stores, as the FP32 output
                    const __half2 hv = __floats2half2_rn(v[r].x * sc, v[r].y * sc);
                    __stcs(reinterpret_cast<unsigned int*>(Co + (size_t)r * P * XP), *reinterpret_cast<const unsigned int*>(&hv));
                }
            } else if constexpr (G == 1) {
                float2* Co = a.C + (size_t)o * Y * XP + kx0 + col;
#pragma unroll
                for (int r = 0; r < V; r++) __stcs(Co + (size_t)(j + P * r) * XP, v[r]);   // streaming
            } else {
                sync();   // every thread has read its last-stage inputs from colbuf
#pragma unroll
                for (int r = 0; r < V; r++) colbuf[tmfft::pad16(j + P * r)] = v[r];
            }
        }
        if constexpr (G > 1) {
            // the item's WG columns, row by row: whole 32-byte sectors per row
            sync();
            float2* Co = a.C + (size_t)o * Y * XP + kx0;
            for (int e = tid; e < Y * WG; e += NT) {
                const int row = e / WG, cc = e % WG;
                __stcs(Co + (size_t)row * XP + cc, exch[cc * PB::CS + tmfft::pad16(row)]);   // streaming
            }
        }
    }
    tmptx::cp_async_wait<0>();
    tmptx::tmem_fence_before_sync();
    __syncthreads();
    tmptx::tmem_fence_after_sync();
    if (warp == 0) tmptx::tmem_dealloc(*tmem_slot, PB::TMEM_COLS);
}

// --------------------------------------------------------------------------------------
// k_pass_b_rg: the column pass of 4096-high micrographs with 256-row pruned
// transforms (T = 256), arranged so that two of its three exchanges stay
// inside a warp.  Write the column spectrum index k = s + 16 k1 + 256 k2 and
// the output row m = m' + 256 M (s, k1, k2, M in 0..15, m' in 0..255).  Both
// transforms split by the residue s = k mod 16:
//   F[s + 16 k'] = sum_{n<256} (a[n] W4096^(-n s)) W256^(-n k')
//   y[m' + 256 M] = sum_s (W4096^(m' s) G_s[m']) W16^(M s),
//   G_s[m'] = sum_{k'} Z[s + 16 k'] W256^(m' k'),   Z = I' conj(F)
// (W_N^e = exp(2 pi i e / N)).  A residue's 256 values live in the 16 lanes of
// one half-warp from the forward 256-point transform through the multiply by
// I' to G_s: each 256-point transform is 16 x 16 with one transpose through
// the warp's own shared memory (__syncwarp only).  One block-wide exchange
// then gathers the 16 residues of each output row m' for the last 16-point
// DFT.  Per item (4 columns of one orientation) that is two block barriers
// instead of the six of k_pass_b's Stockham stages.
//
// Roles: residue phases -- warp w holds residue s = w >> 1 of columns
// 2 (w & 1) + (lane >> 4), lane q = lane & 15; final phase -- thread t holds
// row m' = t >> 2 of column t & 3 (a warp stores 8 rows x 4 columns, whole
// 32-byte row sectors).  The block buffer is blk[c][m'][s] (row stride 17,
// column stride CS = 4 mod 16: conflict-free 8-byte accesses in every phase).
// A warp's transposes use the block-buffer ranges that the same warp reads in
// the final phase, so they need no barrier of their own: nobody else touches
// those ranges between the warp's final read and the next block-wide write.
struct PassBRg {
    static constexpr int T = 256, Y = 4096, W = 4, NT = 1024;
    static constexpr int RS = 17;                       // row stride of blk (float2)
    static constexpr int CS = 256 * RS + 4;             // column stride, == 4 (mod 16)
    static constexpr int APITCH = 260;                  // A staging: [c][row], 4 columns
    static constexpr size_t EXCH = sizeof(float2) * W * CS;
    static constexpr size_t ASZ = sizeof(float2) * W * APITCH;
    static constexpr int ABUFS = 3;                     // rows of A prefetched two items ahead
    static constexpr size_t TWB = sizeof(float2) * NT;   // per-thread twiddle W256^(-q)
    static constexpr int MAX_ITEMS = 2048;              // a block's item list (group << 16 | orientation)
    static constexpr size_t LIST = sizeof(int) * MAX_ITEMS;
    static constexpr size_t SMEM = EXCH + ABUFS * ASZ + TWB + LIST + 64;
    // 8 warps per lane quadrant x 32 columns of I' (columns 0-255), and x 32 columns of
    // the thread's twiddles W4096^(-(q + 16 r) s) (columns 256-511)
    static constexpr uint32_t TMEM_COLS = 512;
    static_assert(SMEM <= 232448, "pass B block exceeds shared memory");
};

__global__ void __launch_bounds__(PassBRg::NT, 1)
k_pass_b_rg(BatchArgs a, int ngroups) {
    using PB = PassBRg;
    constexpr int T = PB::T, Y = PB::Y, RS = PB::RS, CS = PB::CS, AP = PB::APITCH;
    extern __shared__ __align__(16) unsigned char smem_b[];
    float2* const blk = reinterpret_cast<float2*>(smem_b);
    float2* const abuf = reinterpret_cast<float2*>(smem_b + PB::EXCH);
    float2* const twt = reinterpret_cast<float2*>(smem_b + PB::EXCH + PB::ABUFS * PB::ASZ);
    int* const items = reinterpret_cast<int*>(smem_b + PB::EXCH + PB::ABUFS * PB::ASZ + PB::TWB);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem_b + PB::EXCH + PB::ABUFS * PB::ASZ + PB::TWB + PB::LIST);
    const int tid = threadIdx.x;
    // this block's items (the launcher checks that they fit the list)
    int n_items;
    {
        const ColSchedule sch(ngroups, a.nb, blockIdx.x, gridDim.x);
        n_items = sch.n;
        for (int i = tid; i < sch.n; i += PB::NT) {
            int g, o;
            sch.locate(i, g, o);
            items[i] = (g << 16) | o;
        }
    }
    if (n_items == 0) return;
    if ((tid >> 5) == 0) {
        tmptx::tmem_alloc(tmem_slot, PB::TMEM_COLS);
        tmptx::tmem_relinquish();
    }
    // the item's 256 rows of A, column-major into the staging buffer [c][row]
    // (thread: row tid / 4, column tid % 4); items are (column group, orientation),
    // orientation fastest
    const float2* const Asrc = a.A + (size_t)(tid >> 2) * a.XP + (tid & 3);
    const uint32_t adst = tmptx::smem_u32(abuf + (tid & 3) * AP + (tid >> 2));
    auto issue_rows = [&](int grp, int oo, int buf) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(adst + buf * (uint32_t)(PB::ASZ)),
                     "l"(Asrc + (size_t)oo * T * a.XP + grp * 4)
                     : "memory");
    };
    // this thread's W256^(-q) in shared memory, indexed by thread (conflict-free reads)
    twt[tid] = a.twy.template w<-1>(16 * (tid & 15), Y);
    __syncthreads();   // the item list
    issue_rows(items[0] >> 16, items[0] & 0xffff, 0);
    tmptx::cp_async_commit();
    if (n_items > 1) issue_rows(items[1] >> 16, items[1] & 0xffff, 1);
    tmptx::cp_async_commit();
    tmptx::cp_async_wait<1>();
    tmptx::tmem_fence_before_sync();
    __syncthreads();
    tmptx::tmem_fence_after_sync();
    const uint32_t tmem = *tmem_slot + ((uint32_t)(32 * ((tid >> 5) & 3)) << 16) + (uint32_t)(32 * (tid >> 7));
    const uint32_t tmw = tmem + 256;   // the twiddles W4096^(-(q + 16 r) s) of the residue phases
    {
        const int s = tid >> 6, q = tid & 15;
#pragma unroll 1
        for (int h = 0; h < 2; h++) {
            float wb[16];
#pragma unroll
            for (int r = 0; r < 8; r++) {
                const float2 w = a.twy.template w<-1>((q + 16 * (8 * h + r)) * s, Y);
                wb[2 * r] = w.x;
                wb[2 * r + 1] = w.y;
            }
            tmptx::tmem_st16(tmw + 16 * h, wb);
        }
        tmptx::tmem_wait_st();
    }
    int cur_group = -1;
    int buf = 0;
#pragma unroll 1
    for (int it = 0; it < n_items; it++) {
        const int group = items[it] >> 16, o = items[it] & 0xffff;
        // residue phases: residue s = warp / 2, column c = 2 (warp % 2) + lane / 16, lane q = lane % 16
        const int s = tid >> 6, q = tid & 15, c = (tid >> 4) & 3;
        {
            // rows of item it + 2 into the buffer that item it - 1 used
            if (it + 2 < n_items) issue_rows(items[it + 2] >> 16, items[it + 2] & 0xffff, buf == 0 ? 2 : buf - 1);
            tmptx::cp_async_commit();
        }
        if (group != cur_group) {
            // this thread's 16 I' values, k = s + 16 q + 256 r, into its TMEM columns
            const float2* Ig = a.Ip + (size_t)(s + 16 * q) * a.XP + group * 4 + c;
#pragma unroll 1
            for (int h = 0; h < 2; h++) {
                float ib[16];
#pragma unroll
                for (int r = 0; r < 8; r++) {
                    const float2 iv = __ldg(Ig + (size_t)(256 * (8 * h + r)) * a.XP);
                    ib[2 * r] = iv.x;
                    ib[2 * r + 1] = iv.y;
                }
                tmptx::tmem_st16(tmem + 16 * h, ib);
            }
            tmptx::tmem_wait_st();
            cur_group = group;
        }
        // transposes: row rho (0..15) of this half-warp's 16 x 16 block sits in the
        // final-phase ranges of this warp (columns c % 2 and c % 2 + 2, 8 rows of m' each)
        float2* const scr = blk + (c & 1) * CS + 136 * (tid >> 5);
#define TM_RG_ROW(rho) (scr + ((rho) >> 3) * (2 * CS) + ((rho) & 7) * RS)
        float2 v[16];
        // forward: b[n] = a[n] W4096^(-n s) for n = q + 16 r, 16-point DFT over r (-> k1)
        {
            const float2* ac = abuf + buf * (PB::W * AP) + c * AP + q;
            float wb[16];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                tmptx::tmem_ld16(tmw + 16 * h, wb);
                tmptx::tmem_wait_ld16(wb);
#pragma unroll
                for (int r = 0; r < 8; r++) v[8 * h + r] = cmul(ac[16 * (8 * h + r)], make_float2(wb[2 * r], wb[2 * r + 1]));
            }
        }
        tmfft::dft16<-1>(v);
        tmfft::apply_twiddles<16>(v, twt[tid]);                         // W256^(-q k1)
        __syncwarp();   // the warp's final-phase reads of the previous item are done
#pragma unroll
        for (int r = 0; r < 16; r++) TM_RG_ROW(q)[r] = v[r];           // row n1 = q, column k1 = r
        __syncwarp();
#pragma unroll
        for (int r = 0; r < 16; r++) v[r] = TM_RG_ROW(r)[q];           // thread k1 = q holds n1 = r
        __syncwarp();
        tmfft::dft16<-1>(v);                                           // -> k2: F[s + 16 q + 256 r]
        // Z = I' conj(F)
        {
            float iv[16];
            tmptx::tmem_ld16(tmem, iv);
            tmptx::tmem_wait_ld16(iv);
#pragma unroll
            for (int r = 0; r < 8; r++) v[r] = cmul_conj(make_float2(iv[2 * r], iv[2 * r + 1]), v[r]);
            tmptx::tmem_ld16(tmem + 16, iv);
            tmptx::tmem_wait_ld16(iv);
#pragma unroll
            for (int r = 0; r < 8; r++) v[8 + r] = cmul_conj(make_float2(iv[2 * r], iv[2 * r + 1]), v[8 + r]);
        }
        // inverse, residue part: 16-point DFT over k2 (-> m1), W256^(m1 q), transpose,
        // 16-point DFT over k1 (-> m2), then W4096^(s (m1 + 16 m2))
        tmfft::dft16<+1>(v);
        tmfft::apply_twiddles<16>(v, tmfft::conjf2(twt[tid]));
#pragma unroll
        for (int r = 0; r < 16; r++) TM_RG_ROW(q)[r] = v[r];           // row k1 = q, column m1 = r
        __syncwarp();
#pragma unroll
        for (int r = 0; r < 16; r++) v[r] = TM_RG_ROW(r)[q];           // thread m1 = q holds k1 = r
#undef TM_RG_ROW
        tmfft::dft16<+1>(v);                                           // -> m2
        {
            float wb[16];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                tmptx::tmem_ld16(tmw + 16 * h, wb);
                tmptx::tmem_wait_ld16(wb);
#pragma unroll
                for (int r = 0; r < 8; r++) v[8 * h + r] = cmul_conj(v[8 * h + r], make_float2(wb[2 * r], wb[2 * r + 1]));
            }
        }
        // every warp is done with its transposes (which overlap other warps' final ranges)
        __syncthreads();
        {
            float2* bw = blk + c * CS + q * RS + s;
#pragma unroll
            for (int r = 0; r < 16; r++) bw[16 * RS * r] = v[r];         // G_s[m' = q + 16 r]
        }
        tmptx::cp_async_wait<1>();   // the next item's rows (issued at the top of the previous item)
        __syncthreads();
        // final phase: thread holds row m' = tid / 4 of column tid % 4
        {
            const float2* br = blk + (tid & 3) * CS + (tid >> 2) * RS;
#pragma unroll
            for (int r = 0; r < 16; r++) v[r] = br[r];                  // residues s = r of row m'
        }
        tmfft::dft16<+1>(v);                                           // -> M
        {
            // streaming stores (evict first): pass C reads the intermediate only after the
            // whole launch, far more than L2 holds (4.17 -> 4.02 ms per 128 orientations)
            float2* Co = a.C + ((size_t)o * Y + (tid >> 2)) * a.XP + group * 4 + (tid & 3);
            const size_t rstep = (size_t)256 * a.XP;
#pragma unroll
            for (int r = 0; r < 16; r++) {
                __stcs(Co, v[r]);
                Co += rstep;
            }
        }
        buf = buf == 2 ? 0 : buf + 1;
    }
    tmptx::cp_async_wait<0>();
    tmptx::tmem_fence_before_sync();
    __syncthreads();
    tmptx::tmem_fence_after_sync();
    if ((tid >> 5) == 0) tmptx::tmem_dealloc(*tmem_slot, PB::TMEM_COLS);
}

// --------------------------------------------------------------------------------------
// k_pass_c: one block per row y; X/16 threads each own 16 pixels
// (x = 2*(t + P*r) + h); loops over the batch keeping the per-pixel state in
// registers.  The per-pixel sum and sum of squares are compensated (Kahan)
// FP32 sums over the batch, added to the FP64 running sums once per batch.  At
// X = 4096 and 2048 (128 registers, two or four blocks per SM) a thread keeps plain
// FP32 partial sums over at most 8 orientations in registers and adds them
// (Kahan) into compensated sums parked in its TMEM lane (columns 0-63 of its
// 128), beside its twiddle multipliers (columns 64-127).
// Copies of a block's shared-memory histogram: lane l counts into copy
// l % n, bin b of copy c at word b * n + c, so that lanes of one warp whose
// values fall in the same bin (the bins near zero take most of them) rarely
// update the same word or bank.  n is the largest power of two up to
// max_copies whose copies fit in 32 KB.
__host__ __device__ inline int hist_copies(int bins, int max_copies) {
    int n = max_copies;
    while (n > 1 && (long long)bins * n * 4 > 32768) n >>= 1;
    return n;
}

template <int X>
struct PassC {
    static constexpr int H = X / 2;
    static constexpr int R = 8;
    static constexpr int P = H / R;                 // X/16 threads
    static constexpr int RSF = tmfft::padded_len(H);
    // X = 4096 (256 threads, two blocks per SM) and X = 2048 (128 threads, four
    // blocks per SM): every block's warps cover the four TMEM lane quadrants, and
    // the blocks of an SM together take its 512 columns
    static constexpr bool COMP_IN_TMEM = (X == 4096 || X == 2048) && P % 32 == 0;
    static constexpr int MIN_BLOCKS = X == 2048 ? 4 : 2;
    // with the compensation terms in TMEM, a thread also keeps its twiddle
    // multipliers there (the c2r packing's 8 and the transform's stages 1-3):
    // 128 columns per warp, columns 0-47 sums, 48-63 packing, 64 + 16 (s - 1) stage s
    static constexpr int WCOLS = COMP_IN_TMEM ? 128 : 64;
    static constexpr uint32_t TMEM_COLS = WCOLS * ((P / 32 + 3) / 4);   // warps of a lane quadrant side by side
    // one histogram copy: measured at X = 4096, 16 lane-striped copies (32 KB
    // more shared memory per block, less L1) made this pass 5 % slower
    static constexpr int HIST_COPIES = 1;
    // dynamic shared memory for a row pitch XP and `bins` histogram bins
    static size_t smem_bytes(int XP, int bins) {
        return 128 + sizeof(float2) * (2 * (size_t)XP + RSF) + 4 * (size_t)bins * hist_copies(bins, HIST_COPIES);
    }
};

// Stage multipliers of pass C's H-point inverse transform (8 values per thread),
// parked in the thread's TMEM columns 64 + 16 (s - 1) for stage s: the R/RS
// butterflies' RS - 1 powers each, as float pairs (tmfft::fft_pre's source).
template <int H>
struct PassCStageTw {
    using PL = tmfft::Plan<H, 8>;
    static_assert(PL::stages <= 4, "three twiddled stages fit columns 64-111");
    uint32_t col64;
    float tb[16];
    template <int s>
    __device__ __forceinline__ void issue() { tmptx::tmem_ld16(col64 + 16 * (s - 1), tb); }
    template <int s>
    __device__ __forceinline__ void get(int u, float2* p) {
        constexpr int RS = PL::radix(s);
        if (u == 0) tmptx::tmem_wait_ld16(tb);
#pragma unroll
        for (int r = 1; r < RS; r++) p[r] = make_float2(tb[2 * (u * (RS - 1) + r - 1)], tb[2 * (u * (RS - 1) + r - 1) + 1]);
    }
    // the multipliers of thread t, from the twiddle table, into its columns
    __device__ static void fill(uint32_t col64, int t, const tmfft::Twiddles& tw) {
        tmfft::sfor<PL::stages>([&](auto sc) {
            constexpr int s = decltype(sc)::value;
            if constexpr (s > 0) {
                constexpr int RS = PL::radix(s), Ns = PL::ns(s), R = 8, P = PL::P;
                float g[16];
#pragma unroll
                for (int i = 0; i < 16; i++) g[i] = 0.f;
#pragma unroll
                for (int u = 0; u < R / RS; u++) {
                    const int jm = (t + P * u) % Ns;
#pragma unroll
                    for (int r = 1; r < RS; r++) {
                        const float2 w = tw.template w<+1>(jm * (H / (Ns * RS)) * r, H);
                        g[2 * (u * (RS - 1) + r - 1)] = w.x;
                        g[2 * (u * (RS - 1) + r - 1) + 1] = w.y;
                    }
                }
                tmptx::tmem_st16(col64 + 16 * (s - 1), g);
            }
        });
    }
};

template <int X>
__global__ void __launch_bounds__(X / 16, PassC<X>::MIN_BLOCKS)
k_pass_c(BatchArgs a, int Y) {
    using PC = PassC<X>;
    constexpr int H = PC::H, P = PC::P;
    constexpr bool kTm = PC::COMP_IN_TMEM;
    static_assert(!kTm || PC::TMEM_COLS <= 256, "pass C TMEM columns");
    constexpr uint32_t kWaitLimit = 1u << 24;
    const int XP = a.XP;
    // rows of C stream in through 1-D bulk copies, double buffered: the copy
    // of orientation o+1 runs while orientation o is transformed.
    // dynamic shared memory: mbarriers | row buffer 0 | row buffer 1 | FFT buffer | histogram
    extern __shared__ __align__(128) unsigned char smem_c[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_c);
    float2* const rows = reinterpret_cast<float2*>(smem_c + 128);   // two buffers of XP
    float2* fbuf = rows + 2 * XP;
    unsigned int* shist = reinterpret_cast<unsigned int*>(fbuf + PC::RSF);
    const int t = threadIdx.x;
    const int y = blockIdx.x;
    const uint32_t row_bytes = (uint32_t)XP * (uint32_t)sizeof(float2);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem_c + 64);
    const int warp = t >> 5;
    if (t == 0) {
        tmptx::mbar_init(&mbar[0], 1);
        tmptx::mbar_init(&mbar[1], 1);
    }
    if constexpr (kTm) {
        if (warp == 0) {
            tmptx::tmem_alloc(tmem_slot, PC::TMEM_COLS);
            tmptx::tmem_relinquish();
        }
    }
    const int hcopies = hist_copies(a.hist_bins, PC::HIST_COPIES);
    const int hcopy = t & (hcopies - 1);
    for (int b = t; b < a.hist_bins * hcopies; b += P) shist[b] = 0u;
    if constexpr (kTm) tmptx::tmem_fence_before_sync();
    __syncthreads();
    if constexpr (kTm) tmptx::tmem_fence_after_sync();
    // this thread's TMEM columns (lane quadrant warp % 4)
    const uint32_t tcomp = kTm ? *tmem_slot + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(PC::WCOLS * (warp >> 2)) : 0u;
    if (t == 0 && a.nb > 0) {
        tmptx::mbar_arrive_expect_tx(&mbar[0], row_bytes);
        tmptx::bulk_g2s(rows, a.C + (size_t)y * XP, row_bytes, &mbar[0]);
    }
    float mip[16];
    int best[16];
    // per-pixel sum and sum of squares over the batch: compensated (Kahan) FP32,
    // added to the FP64 running sums once per batch.  Without TMEM: fs, fq_regs
    // and the compensation terms comp_regs[0..15] / [16..31] in registers, updated
    // per orientation.  With TMEM (X = 4096): fs and pq are plain FP32 partial sums
    // over at most 8 orientations, added every 8 orientations (Kahan) into the
    // compensated sums held in TMEM columns 0-15 (sum), 16-31 (its compensation),
    // 32-47 (sum of squares), 48-63 (its compensation).
    float fs[16];
    float fq_regs[kTm ? 1 : 16];
    float pq[kTm ? 16 : 1];
    const size_t rowoff = (size_t)y * X;
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const int x = 2 * (t + P * r);
        const float2 mv = *reinterpret_cast<const float2*>(a.mip + rowoff + x);
        const int2 bv = *reinterpret_cast<const int2*>(a.best + rowoff + x);
        mip[2 * r] = mv.x; mip[2 * r + 1] = mv.y;
        best[2 * r] = bv.x; best[2 * r + 1] = bv.y;
        fs[2 * r] = 0.f; fs[2 * r + 1] = 0.f;
        if constexpr (kTm) { pq[2 * r] = 0.f; pq[2 * r + 1] = 0.f; }
    }
    // the compensation terms: in registers, or parked in TMEM between orientations
    float comp_regs[kTm ? 1 : 32];
    if constexpr (kTm) {
        float z[16];
#pragma unroll
        for (int i = 0; i < 16; i++) z[i] = 0.f;
        tmptx::tmem_st16(tcomp, z);
        tmptx::tmem_st16(tcomp + 16, z);
        tmptx::tmem_st16(tcomp + 32, z);
        tmptx::tmem_st16(tcomp + 48, z);
        // the packing's multipliers W_X^k, k = t + P r (columns 112-127), and the
        // transform's stage multipliers (64-111)
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const float2 w = a.tw.template w<+1>(t + P * r, X);
            z[2 * r] = w.x;
            z[2 * r + 1] = w.y;
        }
        tmptx::tmem_st16(tcomp + 112, z);
        PassCStageTw<H>::fill(tcomp + 64, t, a.tw);
        tmptx::tmem_wait_st();
    } else {
#pragma unroll
        for (int i = 0; i < (kTm ? 1 : 32); i++) comp_regs[i] = 0.f;
#pragma unroll
        for (int i = 0; i < (kTm ? 1 : 16); i++) fq_regs[i] = 0.f;
    }
    auto sync = [] __device__() { __syncthreads(); };
    // histogram bin int((v - min) / step) as one multiply-add: (v - min) / step = v / step + hoff
    const float hoff = -a.hist_min * a.hist_inv_step;
    // Copy o goes to buffer o & 1 and completes phase o >> 1 of that buffer's
    // mbarrier.  After a wait runs out the block stops issuing copies and, before
    // it exits, waits for the copies still in flight at the parity of the phase
    // each one completes (bounded again).
    auto drain = [&](int o) {
        tmptx::mbar_wait_bounded(&mbar[(o - 1) & 1], ((o - 1) >> 1) & 1, kWaitLimit);   // the wait that ran out
        if (o < a.nb) tmptx::mbar_wait_bounded(&mbar[o & 1], (o >> 1) & 1, kWaitLimit);   // issued at o - 1
    };
    bool timed_out = false;
    int o = 0;
    for (; o < a.nb; o++) {
        const int buf = o & 1;
        // iteration o-1 is done with row buffer buf ^ 1; every thread learns whether a wait ran out
        if (__syncthreads_or(timed_out)) break;
        if (t == 0 && o + 1 < a.nb) {
            tmptx::mbar_arrive_expect_tx(&mbar[buf ^ 1], row_bytes);
            tmptx::bulk_g2s(rows + (buf ^ 1) * XP, a.C + ((size_t)(o + 1) * Y + y) * XP, row_bytes, &mbar[buf ^ 1]);
        }
        float pk[kTm ? 16 : 1];   // the packing's multipliers, from TMEM
        if constexpr (kTm) tmptx::tmem_ld16(tcomp + 112, pk);
        if (!tmptx::mbar_wait_bounded(&mbar[buf], (o >> 1) & 1, kWaitLimit)) {
            timed_out = true;
            atomicExch(a.err, 1);
        }
        if constexpr (kTm) tmptx::tmem_wait_ld16(pk);
        const float2* rb = rows + buf * XP;
        float2 v[8];
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const int k = t + P * r;
            float2 hk = rb[k];
            float2 hm = rb[H - k];
            if (k == 0) { hk.y = 0.f; hm.y = 0.f; }
            const float2 e = make_float2(hk.x + hm.x, hk.y - hm.y);
            const float2 d = make_float2(hk.x - hm.x, hk.y + hm.y);
            const float2 od = cmul(d, kTm ? make_float2(pk[2 * r], pk[2 * r + 1]) : a.tw.template w<+1>(k, X));
            v[r] = make_float2(e.x - od.y, e.y + od.x);
        }
        // the barrier at the top of the iteration follows the last reads of fbuf
        if constexpr (kTm) {
            PassCStageTw<H> stw{tcomp + 64, {}};
            tmfft::fft_pre<H, 8, +1, false>(v, t, fbuf, stw, sync);
        } else {
            tmfft::fft<H, 8, +1, false>(v, t, fbuf, a.tw, sync);
        }
        const int g = (int)(a.gidx0 + o);
        if constexpr (kTm) {
            // MIP / argmax, histogram and the plain partial sums of this orientation
#pragma unroll
            for (int r = 0; r < 8; r++) {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const float val = h ? v[r].y : v[r].x;
                    const int pi = 2 * r + h;
                    if (val > mip[pi]) { mip[pi] = val; best[pi] = g; }
                    fs[pi] += val;
                    pq[pi] = fmaf(val, val, pq[pi]);
                    const int bin = __float2int_rz(fmaf(val, a.hist_inv_step, hoff));
                    if ((unsigned)bin < (unsigned)a.hist_bins) atomicAdd(&shist[bin * hcopies + hcopy], 1u);
                }
            }
            if ((o & 7) == 7 || o == a.nb - 1) {
                // Kahan: the compensation holds what the last addition added beyond its input
#pragma unroll
                for (int sweep = 0; sweep < 4; sweep++) {   // 8 pixels of one sum at a time
                    float* part = ((sweep >> 1) ? pq : fs) + 8 * (sweep & 1);
                    const uint32_t col = tcomp + 32 * (sweep >> 1) + 8 * (sweep & 1);
                    float sm[8], cm[8];   // sum, compensation
                    tmptx::tmem_ld8(col, sm);
                    tmptx::tmem_ld8(col + 16, cm);
                    tmptx::tmem_wait_ld8x2(sm, cm);
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const float yv = part[i] - cm[i];
                        const float tv = sm[i] + yv;
                        cm[i] = (tv - sm[i]) - yv;
                        sm[i] = tv;
                        part[i] = 0.f;
                    }
                    tmptx::tmem_st8(col, sm);
                    tmptx::tmem_st8(col + 16, cm);
                }
                tmptx::tmem_wait_st();
            }
        } else {
            // epilogue in two sweeps over the 16 values, so that only one sum's 16
            // compensation terms are live at a time: (1) MIP / argmax, histogram and
            // the sum, (2) the sum of squares
#pragma unroll
            for (int sweep = 0; sweep < 2; sweep++) {
                float* comp = comp_regs + 16 * sweep;
#pragma unroll
                for (int r = 0; r < 8; r++) {
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const float val = h ? v[r].y : v[r].x;
                        const int pi = 2 * r + h;
                        // Kahan: the compensation holds what the last addition added beyond its input
                        if (sweep == 0) {
                            if (val > mip[pi]) { mip[pi] = val; best[pi] = g; }
                            const float ys = val - comp[pi];
                            const float ts = fs[pi] + ys;
                            comp[pi] = (ts - fs[pi]) - ys;
                            fs[pi] = ts;
                            const int bin = __float2int_rz(fmaf(val, a.hist_inv_step, hoff));
                            if ((unsigned)bin < (unsigned)a.hist_bins) atomicAdd(&shist[bin * hcopies + hcopy], 1u);
                        } else {
                            const float yq = fmaf(val, val, -comp[pi]);
                            const float tq = fq_regs[pi] + yq;
                            comp[pi] = (tq - fq_regs[pi]) - yq;
                            fq_regs[pi] = tq;
                        }
                    }
                }
            }
        }
    }
    // the sums and their compensation terms for the FP64 flush
    float send[kTm ? 64 : 1];
    const float* fsend = fs;
    const float* cend = comp_regs;
    const float* fqend = fq_regs;
    const float* cqend = comp_regs + (kTm ? 0 : 16);
    if constexpr (kTm) {
        tmptx::tmem_ld16(tcomp, send);
        tmptx::tmem_ld16(tcomp + 16, send + 16);
        tmptx::tmem_wait_ld32(send);
        tmptx::tmem_ld16(tcomp + 32, send + 32);
        tmptx::tmem_ld16(tcomp + 48, send + 48);
        tmptx::tmem_wait_ld32(send + 32);
        fsend = send;
        cend = send + 16;
        fqend = send + 32;
        cqend = send + 48;
        tmptx::tmem_fence_before_sync();
    }
    const bool failed = __syncthreads_or(timed_out);
    if constexpr (kTm) {
        // every warp has finished with its TMEM columns (the barrier above)
        tmptx::tmem_fence_after_sync();
        if (warp == 0) tmptx::tmem_dealloc(*tmem_slot, PC::TMEM_COLS);
    }
    if (failed) {
        // results of this block are discarded (the host reports the timeout)
        drain(o);
        return;
    }
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const int x = 2 * (t + P * r);
        *reinterpret_cast<float2*>(a.mip + rowoff + x) = make_float2(mip[2 * r], mip[2 * r + 1]);
        *reinterpret_cast<int2*>(a.best + rowoff + x) = make_int2(best[2 * r], best[2 * r + 1]);
        double2 sv = *reinterpret_cast<const double2*>(a.sum + rowoff + x);
        double2 qv = *reinterpret_cast<const double2*>(a.sumsq + rowoff + x);
        sv.x += (double)fsend[2 * r] - (double)cend[2 * r];
        sv.y += (double)fsend[2 * r + 1] - (double)cend[2 * r + 1];
        qv.x += (double)fqend[2 * r] - (double)cqend[2 * r];
        qv.y += (double)fqend[2 * r + 1] - (double)cqend[2 * r + 1];
        *reinterpret_cast<double2*>(a.sum + rowoff + x) = sv;
        *reinterpret_cast<double2*>(a.sumsq + rowoff + x) = qv;
    }
    __syncthreads();
    for (int b = t; b < a.hist_bins; b += P) {
        unsigned int cnt = 0;
        for (int k = 0; k < hcopies; k++) cnt += shist[b * hcopies + k];
        if (cnt) atomicAdd(a.hist + b, (unsigned long long)cnt);
    }
}

// --------------------------------------------------------------------------------------
// Prepared micrograph spectrum I'[ky][kx] = I[ky][kx] * exp(+2 pi i (kx*x0/X + ky*y0/Y)) / N
// with the projection placed at (x0, y0) = (X/2 - T/2, Y/2 - T/2), I'[0][0] = 0, and zero
// pitch padding (kx > X/2).  spec: Y*(X/2+1) complex; phases in double.
__global__ void k_prepare_image(const float2* __restrict__ spec, float2* __restrict__ ip, int X, int Y, int XP, int T) {
    const int kx = blockIdx.x * blockDim.x + threadIdx.x;
    const int ky = blockIdx.y;
    if (kx >= XP) return;
    const int hc = X / 2 + 1;
    float2 out = make_float2(0.f, 0.f);
    if (kx < hc && !(kx == 0 && ky == 0)) {
        const long long x0 = X / 2 - T / 2, y0 = Y / 2 - T / 2;
        double sx, cx, sy, cy;
        sincospi(2.0 * (double)((kx * x0) % X) / (double)X, &sx, &cx);
        sincospi(2.0 * (double)((ky * y0) % Y) / (double)Y, &sy, &cy);
        const double pr = cx * cy - sx * sy, pi = cx * sy + sx * cy;
        const float2 v = spec[(size_t)ky * hc + kx];
        const double invn = 1.0 / ((double)X * (double)Y);
        out = make_float2((float)(((double)v.x * pr - (double)v.y * pi) * invn),
                          (float)(((double)v.x * pi + (double)v.y * pr) * invn));
    }
    ip[(size_t)ky * XP + kx] = out;
}

// --------------------------------------------------------------------------------------
__global__ void k_reset_state(float* mip, int* best, double* sum, double* sumsq, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        mip[i] = -FLT_MAX;
        best[i] = -1;
        sum[i] = 0.0;
        sumsq[i] = 0.0;
    }
}

// --------------------------------------------------------------------------------------
// Launch shapes of one geometry, shared by every entry point.
template <int T, int X, int Y>
struct Launch {
    using PB = PassB<T, Y>;
    using PC = PassC<X>;
    using SC = SliceCol<T>;
    using RC = RowC2R<T>;
    static constexpr int pass_b_width = PB::WG;   // row pitch alignment (columns)
    // 4096-high micrographs with 256-row pruned transforms: the residue-grouped column pass
    static constexpr bool RG = (T == 256 && Y == 4096);
    static cudaError_t configure(int XP, int bins) {
        cudaError_t e = cudaFuncSetAttribute(k_pass_b<T, Y>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PB::SMEM);
        if (e != cudaSuccess) return e;
        if constexpr (RG) {
            e = cudaFuncSetAttribute(k_pass_b_rg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PassBRg::SMEM);
            if (e != cudaSuccess) return e;
        }
        return cudaFuncSetAttribute(k_pass_c<X>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PC::smem_bytes(XP, bins));
    }
    // slice, projection, normalisation and row transforms
    static void prep(BatchArgs& a, cudaStream_t s) {
        k_slice_colfft<T><<<dim3((T / 2 + 1 + SC::CB - 1) / SC::CB, a.nb), SC::NT, 0, s>>>(a);
        k_row_c2r<T><<<dim3(T / RC::ROWS, a.nb), RC::NT, 0, s>>>(a);
        k_norm<T><<<(a.nb + 7) / 8, 256, 0, s>>>(a, a.norm_pixels > 0 ? a.norm_pixels : (long long)X * Y);
        k_pass_a<T, X><<<dim3(T, a.nb), X / 16, 0, s>>>(a);
    }
    static void pass_b(BatchArgs& a, cudaStream_t s, int nsm) {
        const int ngroups = a.XP / PB::WG;
        if (RG && ColSchedule::max_items(ngroups, a.nb, nsm) <= PassBRg::MAX_ITEMS)
            k_pass_b_rg<<<nsm, PassBRg::NT, PassBRg::SMEM, s>>>(a, ngroups);
        else
            k_pass_b<T, Y><<<nsm, PB::NT, PB::SMEM, s>>>(a, ngroups);
    }
    static void pass_c(BatchArgs& a, cudaStream_t s) {
        k_pass_c<X><<<Y, X / 16, PC::smem_bytes(a.XP, a.hist_bins), s>>>(a, Y);
    }
};

}  // namespace tmk

#include "tm_tensor.cuh"

namespace tmk {

// Launch shapes of the FP16 tensor-core form of one geometry (row lengths X of
// 1024, 2048 or 4096): k_pass_b with FP16 output in blocks of R rows, and the
// tensor-core row pass.
template <int T, int X, int Y>
struct LaunchTc {
    using PB = PassB<T, Y>;
    using PCT = PassCTc<X>;
    static constexpr int R = PCT::R;
    // height 4096: the tensor-core column pass; other heights: the FP32 column FFTs with FP16 output
    static constexpr bool COL_TC = (Y == 4096);
    using PBT = PassBTc<T, R>;
    static constexpr size_t rows_tab_bytes = (size_t)PCT::B1_BYTES + PCT::B2_BYTES;
    static cudaError_t configure(int XP, int bins) {
        cudaError_t e;
        if constexpr (COL_TC) {
            e = cudaFuncSetAttribute(k_pass_b_tc<T, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, PBT::SMEM);
            // two CTAs of a pair per SM need the largest shared-memory carveout
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_pass_b_tc<T, R>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared);
        } else
            e = cudaFuncSetAttribute(k_pass_b<T, Y, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PB::SMEM);
        if (e != cudaSuccess) return e;
        return cudaFuncSetAttribute(k_pass_c_tc<X>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PCT::smem_bytes(XP, bins));
    }
    static void pass_b(BatchArgs& a, cudaStream_t s, int nsm, const uint4* tabs) {
        if constexpr (COL_TC) {
            // items = (group of 4 columns, orientation); two blocks per SM
            k_pass_b_tc<T, R><<<2 * nsm, PBT::NT, PBT::SMEM, s>>>(a, a.XP / 4, tabs + rows_tab_bytes / 16);
        } else {
            k_pass_b<T, Y, R><<<nsm, PB::NT, PB::SMEM, s>>>(a, a.XP / PB::WG);
        }
    }
    static void pass_c(BatchArgs& a, cudaStream_t s, const uint4* dft) {
        k_pass_c_tc<X><<<Y / R, PCT::NT, PCT::smem_bytes(a.XP, a.hist_bins), s>>>(a, Y, dft);
    }
    // the row pass's DFT operands, then (height 4096) the column pass's
    static constexpr size_t dft_bytes = rows_tab_bytes + (COL_TC ? PBT::dft_bytes : 0);
    static void fill_dft(uint16_t* host) {
        fill_tc_dft<X>(host);
        if constexpr (COL_TC) fill_tc_cols<T, R>(host + rows_tab_bytes / 2);
    }
};

}  // namespace tmk
