// tm_refine.cu -- batched TemplateScore of refine_template on the GPU (C ABI in
// include/tm_b200.h).
//
// One candidate = (Euler angles, particle window, projection filter,
// pixel-size operator).  Per batch of candidates (refine_template.cpp:24-80):
//
//   k_slice_colfft<TP>   Fourier slice of the TP^3 template (trilinear,
//                        Hermitian mirror) x (-1)^(i+j), inverse FFT of
//                        each column (shared with the search)
//   k_row_c2r<TP>        inverse c2r of each row -> TP x TP projection
//   [pixel-size change]  k_disc_sum / k_disc_mean + three batched GEMMs: the
//                        ChangePixelSize chain as out = Ar U Brt - Ai U Bit + pv,
//                        U = projection - pv (operators built on the host)
//   k_score_row_r2c<T>   r2c of each row of the T x T projection (or of the
//                        centred T x T crop of the TP x TP one)
//   k_score_col<T>       per column: forward FFT along y, x projection
//                        filter, zeroed DC, Hermitian-weighted sum of squares
//                        (ReturnSumOfSquares), x conj into the particle
//                        spectrum, inverse FFT along y
//   k_score_row_c2r_max<T> c2r of each row and the row's first maximum
//   k_score_peak         first maximum in scan order
//                        (FindPeakWithIntegerCoordinates), divided by the
//                        square root of the sum of squares (the reference
//                        normalises the projection before the product; the
//                        correlation is linear in it)
//
// Transforms are unnormalised: the score is invariant to the scale of the
// projection spectrum, so the reference's 1/N factors cancel.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <chrono>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/tm_b200.h"

// The slice and projection kernels of the search, instantiated in their own
// namespace so that this translation unit links beside tm_capi.cu.
namespace tmrk {
#include "tm_kernels.cuh"
}  // namespace tmrk

namespace tmr {

using tmrk::tmfft::cmul;
using tmrk::tmfft::cmul_conj;
using tmrk::tmfft::Twiddles;
using tmrk::tmk::skewed;
namespace tmfft = tmrk::tmfft;
namespace tmk = tmrk::tmk;
namespace tmptx = tmrk::tmptx;

struct ScoreArgs {
    int nb;
    const int* particle;       // nb
    const int* filter;         // nb
    const int* op;             // nb, -1 = no pixel-size change
    const float2* particles;   // slots * T*(T/2+1)
    const float* filters;      // slots * T*(T/2+1)
    const float* P;            // nb * TP*TP projections
    const float* Q;            // nb * T*T resampled projections
    const float* pv;           // nb pad values (resampled candidates)
    float2* R;                 // nb * T*(T/2+1)
    double* sumsq;             // nb
    float* rowmax;             // nb * T
    int* rowarg;               // nb * T
    float* out;                // nb * 3
    int TPbox;                 // projection box
    Twiddles tw;               // lengths dividing T
};

// ---------------------------------------------------------------------------------------------
// r2c of each row: T reals -> T/2+1 complex via a T/2-point FFT of the even /
// odd pairs.  The source is the resampled projection (+ pad value), the
// projection itself (TP == T) or its centred T x T crop (TP > T).
template <int T>
struct RowR2C {
    static constexpr int H = T / 2;
    static constexpr int V = H % 3 == 0 ? 24 : 16;
    static constexpr int PH = H / V;
    static constexpr int RS = skewed(tmfft::padded_len(H), PH % 16);
    static constexpr int ROWS0 = (256 / PH) < T ? (256 / PH) : T;
    static constexpr int ROWS = (ROWS0 * RS * 8 <= 40 * 1024) ? ROWS0 : ROWS0 / 2;
    static constexpr int NT = ROWS * PH;
};

template <int T>
__global__ void __launch_bounds__(RowR2C<T>::NT) k_score_row_r2c(ScoreArgs a) {
    using RC = RowR2C<T>;
    constexpr int H = RC::H, PH = RC::PH, ROWS = RC::ROWS, V = RC::V, RS = RC::RS, HC = T / 2 + 1;
    __shared__ float2 sm[ROWS * RS];
    const int t = threadIdx.x % PH, rl = threadIdx.x / PH;
    const int y = blockIdx.x * ROWS + rl;
    const int b = blockIdx.y;
    const float* src;
    float add = 0.f;
    if (a.op[b] >= 0) {
        src = a.Q + ((size_t)b * T + y) * T;
        add = a.pv[b];
    } else {
        const int TPb = a.TPbox;
        const int off = TPb / 2 - T / 2;   // centred ClipInto
        src = a.P + ((size_t)b * TPb + (y + off)) * TPb + off;
    }
    float2 v[V];
#pragma unroll
    for (int r = 0; r < V; r++) {
        const int n = t + PH * r;
        v[r] = make_float2(src[2 * n] + add, src[2 * n + 1] + add);
    }
    float2* buf = sm + rl * RS;
    tmfft::fft<H, V, -1>(v, t, buf, a.tw, [] __device__() { __syncthreads(); });
    __syncthreads();
#pragma unroll
    for (int r = 0; r < V; r++) buf[tmfft::pad16(t + PH * r)] = v[r];
    __syncthreads();
    float2* row = a.R + ((size_t)b * T + y) * HC;
#pragma unroll
    for (int r = 0; r < V; r++) {
        const int k = t + PH * r;
        const float2 zk = v[r];
        const float2 zm = buf[tmfft::pad16(k == 0 ? 0 : H - k)];
        // E = (Z[k] + conj Z[H-k]) / 2, O = (Z[k] - conj Z[H-k]) / 2i
        const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
        const float2 wo = cmul(o, a.tw.template w<-1>(k, T));
        row[k] = make_float2(e.x + wo.x, e.y + wo.y);
        if (k == 0) row[H] = make_float2(e.x - o.x, e.y - o.y);
    }
}

// ---------------------------------------------------------------------------------------------
// per column of the half spectrum: forward FFT along y, filter, DC, sum of
// squares, product with the particle, inverse FFT along y
template <int T>
struct ColS {
    static constexpr int V = T % 3 == 0 ? 24 : 16;
    static constexpr int PT = T / V;
    static constexpr int RS = skewed(tmfft::padded_len(T), 1);
    static constexpr int CB = (16 * RS * 8 <= 40 * 1024) ? 16 : (8 * RS * 8 <= 40 * 1024) ? 8 : 4;
    static constexpr int NT = CB * PT;
};

template <int T>
__global__ void __launch_bounds__(ColS<T>::NT) k_score_col(ScoreArgs a) {
    using CS = ColS<T>;
    constexpr int HC = T / 2 + 1, PT = CS::PT, V = CS::V, CB = CS::CB, RS = CS::RS;
    __shared__ float2 sm[CB * RS];
    __shared__ double red[CS::NT / 32 + 1];
    const int il = threadIdx.x % CB, tp = threadIdx.x / CB;
    const int i = blockIdx.x * CB + il;
    const int b = blockIdx.y;
    const bool valid = i < HC;
    float2* col = a.R + (size_t)b * T * HC + i;
    float2 v[V];
#pragma unroll
    for (int r = 0; r < V; r++) v[r] = valid ? col[(size_t)(tp + PT * r) * HC] : make_float2(0.f, 0.f);
    tmfft::fft<T, V, -1>(v, tp, sm + il * RS, a.tw, [] __device__() { __syncthreads(); });
    const float* flt = a.filters + (size_t)a.filter[b] * T * HC + i;
    const float2* w = a.particles + (size_t)a.particle[b] * T * HC + i;
    double ss = 0.0;
#pragma unroll
    for (int r = 0; r < V; r++) {
        const int y = tp + PT * r;
        float2 s = make_float2(0.f, 0.f);
        if (valid) {
            const float f = __ldg(flt + (size_t)y * HC);
            s = make_float2(v[r].x * f, v[r].y * f);
            if (i == 0 && y == 0) s = make_float2(0.f, 0.f);
            // ReturnSumOfSquares, Fourier space (image.cpp:300-313), even T:
            // weight 1/2 on the DC / Nyquist corners, the x = 0 and x = T/2
            // columns counted for y >= 0 only
            const int jj = y < T / 2 ? y : y - T;
            const bool xedge = (i == 0 || i == T / 2);
            const bool yedge = (jj == 0 || jj == -(T / 2));
            const double p = (double)s.x * s.x + (double)s.y * s.y;
            if (xedge && yedge) ss += 0.5 * p;
            else if (!xedge || jj >= 0) ss += p;
            s = cmul_conj(__ldg(w + (size_t)y * HC), s);
        }
        v[r] = s;
    }
    // block sum of the squares
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
    tmfft::fft<T, V, +1>(v, tp, sm + il * RS, a.tw, [] __device__() { __syncthreads(); });
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int k = 0; k < CS::NT / 32; k++) tot += red[k];
        atomicAdd(a.sumsq + b, tot);
    }
    if (valid) {
#pragma unroll
        for (int r = 0; r < V; r++) col[(size_t)(tp + PT * r) * HC] = v[r];
    }
}

// ---------------------------------------------------------------------------------------------
// c2r of each row and its first maximum
template <int T>
struct RowC2RMax {
    static constexpr int H = T / 2;
    static constexpr int V = H % 3 == 0 ? 24 : 16;
    static constexpr int PH = H / V;
    static constexpr int RS = skewed(tmfft::padded_len(H), PH % 16);
    static constexpr int ROWS0 = (256 / PH) < T ? (256 / PH) : T;
    static constexpr int ROWS = (ROWS0 * RS * 8 <= 40 * 1024) ? ROWS0 : ROWS0 / 2;
    static constexpr int NT = ROWS * PH;
    static_assert(32 % PH == 0, "row reductions use warp shuffles");
};

__device__ __forceinline__ bool better(float v, int x, float bv, int bx) {
    // larger value first, then the smaller index; NaN never wins (the
    // reference's strict '>' is false for it)
    if (v != v) return false;
    if (bv != bv) return true;
    return v > bv || (v == bv && x < bx);
}

template <int T>
__global__ void __launch_bounds__(RowC2RMax<T>::NT) k_score_row_c2r_max(ScoreArgs a) {
    using RC = RowC2RMax<T>;
    constexpr int H = RC::H, PH = RC::PH, ROWS = RC::ROWS, V = RC::V, RS = RC::RS, HC = T / 2 + 1;
    __shared__ float2 sm[ROWS * RS];
    const int t = threadIdx.x % PH, rl = threadIdx.x / PH;
    const int y = blockIdx.x * ROWS + rl;
    const int b = blockIdx.y;
    const float2* Hrow = a.R + ((size_t)b * T + y) * HC;
    float2 v[V];
#pragma unroll
    for (int r = 0; r < V; r++) {
        const int k = t + PH * r;
        float2 hk = Hrow[k];
        float2 hm = Hrow[H - k];
        if (k == 0) { hk.y = 0.f; hm.y = 0.f; }
        const float2 e = make_float2(hk.x + hm.x, hk.y - hm.y);
        const float2 d = make_float2(hk.x - hm.x, hk.y + hm.y);
        const float2 od = cmul(d, a.tw.template w<+1>(k, T));
        v[r] = make_float2(e.x - od.y, e.y + od.x);
    }
    tmfft::fft<H, V, +1>(v, t, sm + rl * RS, a.tw, [] __device__() { __syncthreads(); });
    // v[r] = (x[2m], x[2m+1]), m = t + PH r
    float bv = -FLT_MAX;
    int bx = T;
#pragma unroll
    for (int r = 0; r < V; r++) {
        const int m = t + PH * r;
        if (better(v[r].x, 2 * m, bv, bx)) { bv = v[r].x; bx = 2 * m; }
        if (better(v[r].y, 2 * m + 1, bv, bx)) { bv = v[r].y; bx = 2 * m + 1; }
    }
#pragma unroll
    for (int off = PH / 2; off > 0; off >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, bv, off);
        const int ox = __shfl_xor_sync(0xffffffffu, bx, off);
        if (better(ov, ox, bv, bx)) { bv = ov; bx = ox; }
    }
    if (t == 0) {
        a.rowmax[(size_t)b * T + y] = bv;
        a.rowarg[(size_t)b * T + y] = bx;
    }
}

// first maximum in scan order, one warp per candidate
template <int T>
__global__ void __launch_bounds__(256) k_score_peak(ScoreArgs a) {
    const int lane = threadIdx.x & 31;
    const int b = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (b >= a.nb) return;
    float bv = -FLT_MAX;
    int bi = T * T;   // y * T + x
    for (int y = lane; y < T; y += 32) {
        const float v = a.rowmax[(size_t)b * T + y];
        const int x = a.rowarg[(size_t)b * T + y];
        if (x < T && better(v, y * T + x, bv, bi)) { bv = v; bi = y * T + x; }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, bv, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
    }
    if (lane == 0) {
        float* o = a.out + 3 * (size_t)b;
        const double ss = 2.0 * a.sumsq[b];
        o[0] = (bi < T * T) ? (float)((double)bv / sqrt(ss)) : -FLT_MAX;
        o[1] = (float)(bi % T - T / 2);
        o[2] = (float)(bi / T - T / 2);
    }
}

// ---------------------------------------------------------------------------------------------
// pixel-size change
//
// pad value: mean of the projection within 0.45 TP of its centre
// (ReturnAverageOfRealValues, image.cpp:6263-6300).  The squared distances
// are sums of squared integers, exact in float, so the disc is the set the
// reference's powf test selects; its pixel count is fixed per box.  Grid
// (jobs, DISC_SPLIT): each block sums a band of rows into pvsum (double).
constexpr int DISC_SPLIT = 8;

__global__ void __launch_bounds__(256) k_disc_sum(const float* __restrict__ P, const int* __restrict__ jobs,
                                                  const int* __restrict__ has_pad, double* pvsum, int TP) {
    if (!has_pad[blockIdx.x]) return;
    const int b = jobs[blockIdx.x];
    __shared__ double rs[8];
    const float r2 = powf(0.45f * (float)TP, 2);
    const int c = TP / 2;
    const int rows = (TP + DISC_SPLIT - 1) / DISC_SPLIT;
    const int j0 = blockIdx.y * rows, j1 = min(TP, j0 + rows);
    const float* p = P + (size_t)b * TP * TP;
    double s = 0.0;
    for (int idx = j0 * TP + threadIdx.x; idx < j1 * TP; idx += blockDim.x) {
        const int j = idx / TP, i = idx % TP;
        const float d = (float)((i - c) * (i - c) + (j - c) * (j - c));
        if (d <= r2) s += p[idx];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) rs[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double ts = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) ts += rs[k];
        atomicAdd(pvsum + b, ts);
    }
}

__global__ void k_disc_mean(const int* __restrict__ jobs, const int* __restrict__ has_pad,
                            const double* __restrict__ pvsum, float* pv, int n_jobs, double inv_count) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_jobs) return;
    const int b = jobs[j];
    pv[b] = has_pad[j] ? (float)(pvsum[b] * inv_count) : 0.0f;
}

#include "tm_gemm.cuh"

}  // namespace tmr

// ---------------------------------------------------------------------------------------------
struct tm_refine_ctx {
    int device = 0, T = 0, TP = 0;
    int max_batch = 0, max_particles = 0, max_filters = 0, max_ops = 0;
    cudaStream_t stream = nullptr;
    float2 *tmpl = nullptr, *particles = nullptr, *S = nullptr, *R = nullptr, *tw_tp = nullptr, *tw_t = nullptr;
    float *filters = nullptr, *ops = nullptr, *ones = nullptr, *rot = nullptr, *P = nullptr, *Z = nullptr, *Q = nullptr;
    float *pv = nullptr, *rowmax = nullptr, *out = nullptr;
    double *rowstat = nullptr, *sumsq = nullptr, *pvsum = nullptr;
    long long disc_count = 1;
    int *cand = nullptr, *rowarg = nullptr, *jobs = nullptr, *has_pad = nullptr;
    int* gemm_err = nullptr;   // set by a tensor-core GEMM whose completion wait ran out
    tmr::GemmJob* gjobs = nullptr;
    int* op_has_pad_host = nullptr;
    // page-locked staging of the per-batch inputs and outputs
    float* h_rot = nullptr;
    int* h_cand = nullptr;
    int* h_jobs = nullptr;
    tmr::GemmJob* h_gjobs = nullptr;
    float* h_out = nullptr;
    int* h_gemm_err = nullptr;
    std::vector<char> op_set;
    int (*run)(tm_refine_ctx*, int n, int n_jobs) = nullptr;
    std::string err;
};

namespace {

int rset_err(tm_refine_ctx* c, int code, const char* fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return code;
}

#define TR_CUDA(ctx, call)                                                                                     \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess)                                                                                 \
            return rset_err((ctx), e_ == cudaErrorMemoryAllocation ? TM_ERR_OOM : TM_ERR_CUDA, "%s: %s (%s:%d)", \
                            #call, cudaGetErrorString(e_), __FILE__, __LINE__);                               \
    } while (0)

size_t hc_size(int T) { return (size_t)T * (T / 2 + 1); }
size_t op_floats(int T, int TP) { return (size_t)4 * T * TP; }   // ar, -ai (T x TP); brt | bit (TP x 2T)

template <int T, int TP>
int run_batch(tm_refine_ctx* c, int n, int n_jobs) {
    cudaStream_t s = c->stream;
    tmrk::tmk::BatchArgs a{};
    a.nb = n;
    a.orient0 = 0;
    a.rot = c->rot;
    a.tmpl = c->tmpl;
    a.filter = c->ones;
    a.S = c->S;
    a.P = c->P;
    a.rowstat = c->rowstat;
    a.twt.tab = c->tw_tp;
    a.twt.lmax = TP;
    using SC = tmrk::tmk::SliceCol<TP>;
    using RC = tmrk::tmk::RowC2R<TP>;
#define TR_LAUNCHED(name)                                                                                   \
    do {                                                                                                    \
        cudaError_t e_ = cudaGetLastError();                                                                \
        if (e_ != cudaSuccess) return rset_err(c, TM_ERR_CUDA, "%s launch failed: %s", name, cudaGetErrorString(e_)); \
    } while (0)
    tmrk::tmk::k_slice_colfft<TP><<<dim3((TP / 2 + 1 + SC::CB - 1) / SC::CB, n), SC::NT, 0, s>>>(a);
    TR_LAUNCHED("k_slice_colfft");
    tmrk::tmk::k_row_c2r<TP><<<dim3(TP / RC::ROWS, n), RC::NT, 0, s>>>(a);
    TR_LAUNCHED("k_row_c2r");
    if (n_jobs > 0) {
        TR_CUDA(c, cudaMemsetAsync(c->pvsum, 0, sizeof(double) * n, s));
        tmr::k_disc_sum<<<dim3(n_jobs, tmr::DISC_SPLIT), 256, 0, s>>>(c->P, c->jobs, c->has_pad, c->pvsum, TP);
        TR_LAUNCHED("k_disc_sum");
        tmr::k_disc_mean<<<(n_jobs + 127) / 128, 128, 0, s>>>(c->jobs, c->has_pad, c->pvsum, c->pv, n_jobs,
                                                              1.0 / (double)c->disc_count);
        TR_LAUNCHED("k_disc_mean");
        // on the tensor cores (split TF32, FP32 accumulation):
        // Z = (P - pv) [brt | bit]            (TP x 2T)
        TR_CUDA(c, tmr::gemm_tc(c->gjobs, n_jobs, TP, 2 * T, TP, TP, 2 * T, 2 * T, 0, c->gemm_err, s));
        // Q = Ar Z[:, :T] + (-Ai) Z[:, T:]     (T x T)
        TR_CUDA(c, tmr::gemm_tc(c->gjobs + n_jobs, n_jobs, T, T, TP, 2 * TP, 2 * T, T, 0, c->gemm_err, s));
        TR_CUDA(c, tmr::gemm_tc(c->gjobs + 2 * n_jobs, n_jobs, T, T, TP, 2 * TP, 2 * T, T, 1, c->gemm_err, s));
    }
    TR_CUDA(c, cudaMemsetAsync(c->sumsq, 0, sizeof(double) * n, s));
    tmr::ScoreArgs sa{};
    sa.nb = n;
    sa.particle = c->cand;
    sa.filter = c->cand + c->max_batch;
    sa.op = c->cand + 2 * c->max_batch;
    sa.particles = c->particles;
    sa.filters = c->filters;
    sa.P = c->P;
    sa.Q = c->Q;
    sa.pv = c->pv;
    sa.R = c->R;
    sa.sumsq = c->sumsq;
    sa.rowmax = c->rowmax;
    sa.rowarg = c->rowarg;
    sa.out = c->out;
    sa.TPbox = TP;
    sa.tw.tab = c->tw_t;
    sa.tw.lmax = T;
    using R1 = tmr::RowR2C<T>;
    using CS = tmr::ColS<T>;
    using R2 = tmr::RowC2RMax<T>;
    tmr::k_score_row_r2c<T><<<dim3(T / R1::ROWS, n), R1::NT, 0, s>>>(sa);
    TR_LAUNCHED("k_score_row_r2c");
    tmr::k_score_col<T><<<dim3((T / 2 + 1 + CS::CB - 1) / CS::CB, n), CS::NT, 0, s>>>(sa);
    TR_LAUNCHED("k_score_col");
    tmr::k_score_row_c2r_max<T><<<dim3(T / R2::ROWS, n), R2::NT, 0, s>>>(sa);
    TR_LAUNCHED("k_score_row_c2r_max");
    tmr::k_score_peak<T><<<(n + 7) / 8, 256, 0, s>>>(sa);
    TR_LAUNCHED("k_score_peak");
#undef TR_LAUNCHED
    return TM_OK;
}

struct RefineVariant {
    int T, TP;
    int (*run)(tm_refine_ctx*, int, int);
};

const RefineVariant kRefineVariants[] = {
    {32, 32, run_batch<32, 32>},       {32, 64, run_batch<32, 64>},       {48, 48, run_batch<48, 48>},
    {48, 96, run_batch<48, 96>},       {64, 64, run_batch<64, 64>},       {64, 128, run_batch<64, 128>},
    {128, 128, run_batch<128, 128>},   {128, 256, run_batch<128, 256>},   {256, 256, run_batch<256, 256>},
    {256, 512, run_batch<256, 512>},   {384, 384, run_batch<384, 384>},   {384, 768, run_batch<384, 768>},
};

void rfree(tm_refine_ctx* c) {
    void* d[] = {c->tmpl, c->particles, c->S, c->R, c->tw_tp, c->tw_t, c->filters, c->ops, c->ones, c->rot, c->P,
                 c->Z, c->Q, c->pv, c->rowmax, c->out, c->rowstat, c->sumsq, c->pvsum, c->cand, c->rowarg,
                 c->jobs, c->gjobs, c->gemm_err};   // has_pad lives inside jobs
    for (void* p : d)
        if (p) cudaFree(p);
    void* h[] = {c->h_rot, c->h_cand, c->h_jobs, c->h_gjobs, c->h_out, c->op_has_pad_host, c->h_gemm_err};
    for (void* p : h)
        if (p) cudaFreeHost(p);
    if (c->stream) cudaStreamDestroy(c->stream);
}

int wait_refine(tm_refine_ctx* c, double limit_s) {
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaStreamQuery(c->stream);
        if (e == cudaSuccess) return TM_OK;
        if (e != cudaErrorNotReady) return rset_err(c, TM_ERR_CUDA, "device error: %s", cudaGetErrorString(e));
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit_s)
            return rset_err(c, TM_ERR_TIMEOUT, "stream did not finish within %.0f s", limit_s);
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

template <class Tp>
int dalloc(tm_refine_ctx* c, Tp** p, size_t n) {
    TR_CUDA(c, cudaMalloc((void**)p, sizeof(Tp) * (n ? n : 1)));
    return TM_OK;
}

// RotationMatrix::SetToEulerRotation (matrix.cpp:490-510), the two used columns, float
void euler_rows1(float phi, float theta, float psi, float* m) {
    const float pif = 3.14159265359f;
    auto d2r = [pif](float deg) { return (float)((double)(deg * pif) / 180.); };
    const float cphi = cosf(d2r(phi)), sphi = sinf(d2r(phi));
    const float cth = cosf(d2r(theta)), sth = sinf(d2r(theta));
    const float cpsi = cosf(d2r(psi)), spsi = sinf(d2r(psi));
    m[0] = cphi * cth * cpsi - sphi * spsi;
    m[1] = -cphi * cth * spsi - sphi * cpsi;
    m[2] = sphi * cth * cpsi + cphi * spsi;
    m[3] = -sphi * cth * spsi + cphi * cpsi;
    m[4] = -sth * cpsi;
    m[5] = sth * spsi;
}

}  // namespace

extern "C" {

int tm_refine_create(int device, int template_box, int projection_box, const float* template_spectrum, int max_batch,
                     int max_particles, int max_filters, int max_operators, tm_refine_ctx** out) {
    if (!out || !template_spectrum || max_batch <= 0 || max_particles <= 0 || max_filters <= 0 || max_operators < 0)
        return TM_ERR_INVALID;
    *out = nullptr;
    const RefineVariant* var = nullptr;
    for (const RefineVariant& v : kRefineVariants)
        if (v.T == template_box && v.TP == projection_box) var = &v;
    if (!var) return TM_ERR_UNSUPPORTED;
    tm_refine_ctx* c = new tm_refine_ctx();
    *out = c;
    c->device = device;
    c->T = template_box;
    c->TP = projection_box;
    c->max_batch = max_batch;
    c->max_particles = max_particles;
    c->max_filters = max_filters;
    c->max_ops = max_operators;
    c->run = var->run;
    TR_CUDA(c, cudaSetDevice(device));
    TR_CUDA(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    const int T = c->T, TP = c->TP;
    const size_t tsz = (size_t)TP * TP * (TP / 2 + 1);
#define TRY(x)                       \
    do {                             \
        int rc_ = (x);               \
        if (rc_ != TM_OK) return rc_; \
    } while (0)
    TRY(dalloc(c, &c->tmpl, tsz));
    TRY(dalloc(c, &c->particles, hc_size(T) * max_particles));
    TRY(dalloc(c, &c->filters, hc_size(T) * max_filters));
    TRY(dalloc(c, &c->ops, op_floats(T, TP) * (max_operators ? max_operators : 1)));
    TRY(dalloc(c, &c->ones, hc_size(TP)));
    TRY(dalloc(c, &c->rot, (size_t)6 * max_batch));
    TRY(dalloc(c, &c->S, hc_size(TP) * max_batch));
    TRY(dalloc(c, &c->P, (size_t)TP * TP * max_batch));
    TRY(dalloc(c, &c->rowstat, (size_t)TP * 4 * max_batch));
    TRY(dalloc(c, &c->Z, (size_t)TP * 2 * T * max_batch));
    TRY(dalloc(c, &c->Q, (size_t)T * T * max_batch));
    TRY(dalloc(c, &c->pv, (size_t)max_batch));
    TRY(dalloc(c, &c->pvsum, (size_t)max_batch));
    {
        // pixels of the pad-value disc (0.45 TP around the centre)
        const float r2 = powf(0.45f * (float)TP, 2);
        long long cnt = 0;
        for (int j = 0; j < TP; j++)
            for (int i = 0; i < TP; i++)
                if ((float)((i - TP / 2) * (i - TP / 2) + (j - TP / 2) * (j - TP / 2)) <= r2) cnt++;
        c->disc_count = cnt > 0 ? cnt : 1;
    }
    TRY(dalloc(c, &c->R, hc_size(T) * max_batch));
    TRY(dalloc(c, &c->sumsq, (size_t)max_batch));
    TRY(dalloc(c, &c->rowmax, (size_t)T * max_batch));
    TRY(dalloc(c, &c->rowarg, (size_t)T * max_batch));
    TRY(dalloc(c, &c->out, (size_t)3 * max_batch));
    TRY(dalloc(c, &c->cand, (size_t)3 * max_batch));
    TRY(dalloc(c, &c->jobs, (size_t)2 * max_batch));
    TRY(dalloc(c, &c->gjobs, (size_t)3 * max_batch));
    TRY(dalloc(c, &c->gemm_err, 1));
    c->has_pad = c->jobs + max_batch;
    TR_CUDA(c, cudaMallocHost((void**)&c->h_rot, sizeof(float) * 6 * max_batch));
    TR_CUDA(c, cudaMallocHost((void**)&c->h_cand, sizeof(int) * 3 * max_batch));
    TR_CUDA(c, cudaMallocHost((void**)&c->h_jobs, sizeof(int) * 2 * max_batch));
    TR_CUDA(c, cudaMallocHost((void**)&c->h_gjobs, sizeof(tmr::GemmJob) * 3 * max_batch));
    TR_CUDA(c, cudaMallocHost((void**)&c->h_out, sizeof(float) * 3 * max_batch));
    TR_CUDA(c, cudaMallocHost((void**)&c->h_gemm_err, sizeof(int)));
    TR_CUDA(c, cudaMallocHost((void**)&c->op_has_pad_host, sizeof(int) * (max_operators ? max_operators : 1)));
    c->op_set.assign(max_operators, 0);
    // twiddle tables for the projection box and the template box
    for (int k = 0; k < 2; k++) {
        const int L = k == 0 ? TP : T;
        float2** tab = k == 0 ? &c->tw_tp : &c->tw_t;
        TRY(dalloc(c, tab, (size_t)L));
        std::vector<float2> tw(L);
        for (int m = 0; m < L; m++) {
            const double ang = -2.0 * M_PI * (double)m / (double)L;
            tw[m] = make_float2((float)cos(ang), (float)sin(ang));
        }
        TR_CUDA(c, cudaMemcpy(*tab, tw.data(), sizeof(float2) * L, cudaMemcpyHostToDevice));
    }
    {
        std::vector<float> ones(hc_size(TP), 1.0f);
        TR_CUDA(c, cudaMemcpy(c->ones, ones.data(), sizeof(float) * ones.size(), cudaMemcpyHostToDevice));
    }
    TR_CUDA(c, cudaMemcpy(c->tmpl, template_spectrum, sizeof(float2) * tsz, cudaMemcpyHostToDevice));
#undef TRY
    return TM_OK;
}

int tm_refine_set_particle(tm_refine_ctx* c, int slot, const float* spectrum) {
    if (!c || !spectrum || slot < 0 || slot >= c->max_particles) return TM_ERR_INVALID;
    TR_CUDA(c, cudaSetDevice(c->device));
    TR_CUDA(c, cudaMemcpyAsync(c->particles + hc_size(c->T) * slot, spectrum, sizeof(float2) * hc_size(c->T),
                               cudaMemcpyHostToDevice, c->stream));
    return wait_refine(c, 60.0);
}

int tm_refine_set_filter(tm_refine_ctx* c, int slot, const float* filter) {
    if (!c || !filter || slot < 0 || slot >= c->max_filters) return TM_ERR_INVALID;
    TR_CUDA(c, cudaSetDevice(c->device));
    TR_CUDA(c, cudaMemcpyAsync(c->filters + hc_size(c->T) * slot, filter, sizeof(float) * hc_size(c->T),
                               cudaMemcpyHostToDevice, c->stream));
    return wait_refine(c, 60.0);
}

int tm_refine_set_operator(tm_refine_ctx* c, int slot, const float* ar, const float* ai, const float* brt,
                           const float* bit, int has_pad_value) {
    if (!c || !ar || !ai || !brt || !bit || slot < 0 || slot >= c->max_ops) return TM_ERR_INVALID;
    TR_CUDA(c, cudaSetDevice(c->device));
    const int T = c->T, TP = c->TP;
    // layout: [ar | -ai] (T x 2TP), then [brt | bit] (TP x 2T)
    std::vector<float> buf(op_floats(T, TP));
    for (int t = 0; t < T; t++)
        for (int i = 0; i < TP; i++) {
            buf[(size_t)t * 2 * TP + i] = ar[(size_t)t * TP + i];
            buf[(size_t)t * 2 * TP + TP + i] = -ai[(size_t)t * TP + i];
        }
    float* bb = buf.data() + (size_t)2 * T * TP;
    for (int i = 0; i < TP; i++)
        for (int t = 0; t < T; t++) {
            bb[(size_t)i * 2 * T + t] = brt[(size_t)i * T + t];
            bb[(size_t)i * 2 * T + T + t] = bit[(size_t)i * T + t];
        }
    TR_CUDA(c, cudaMemcpyAsync(c->ops + op_floats(T, TP) * slot, buf.data(), sizeof(float) * buf.size(),
                               cudaMemcpyHostToDevice, c->stream));
    c->op_has_pad_host[slot] = has_pad_value ? 1 : 0;
    c->op_set[slot] = 1;
    return wait_refine(c, 60.0);
}

int tm_refine_score(tm_refine_ctx* c, int n, const float* euler, const int* particle, const int* filter,
                    const int* op, float* out) {
    if (!c || n < 0 || (n > 0 && (!euler || !particle || !filter || !op || !out))) return TM_ERR_INVALID;
    if (n == 0) return TM_OK;
    TR_CUDA(c, cudaSetDevice(c->device));
    const int T = c->T, TP = c->TP;
    for (int base = 0; base < n; base += c->max_batch) {
        const int m = n - base < c->max_batch ? n - base : c->max_batch;
        int n_jobs = 0;
        for (int k = 0; k < m; k++) {
            const int g = base + k;
            if (particle[g] < 0 || particle[g] >= c->max_particles || filter[g] < 0 || filter[g] >= c->max_filters ||
                op[g] < -1 || op[g] >= c->max_ops || (op[g] >= 0 && !c->op_set[op[g]]))
                return rset_err(c, TM_ERR_INVALID, "candidate %d: slot out of range", g);
            euler_rows1(euler[3 * g], euler[3 * g + 1], euler[3 * g + 2], c->h_rot + 6 * k);
            c->h_cand[k] = particle[g];
            c->h_cand[c->max_batch + k] = filter[g];
            c->h_cand[2 * c->max_batch + k] = op[g];
            if (op[g] >= 0) {
                const float* bcat = c->ops + op_floats(T, TP) * op[g] + (size_t)2 * T * TP;   // TP x 2T
                float* Z = c->Z + (size_t)TP * 2 * T * k;
                c->h_jobs[n_jobs] = k;
                c->h_jobs[c->max_batch + n_jobs] = c->op_has_pad_host[op[g]];
                c->h_gjobs[n_jobs] = tmr::GemmJob{c->P + (size_t)TP * TP * k, bcat, Z, c->pv + k};
                n_jobs++;
            }
        }
        // second and third GEMM jobs follow the first n_jobs entries
        for (int j = 0; j < n_jobs; j++) {
            const int k = c->h_jobs[j];
            const int g = base + k;
            const float* acat = c->ops + op_floats(T, TP) * op[g];
            float* Z = c->Z + (size_t)TP * 2 * T * k;
            float* Q = c->Q + (size_t)T * T * k;
            c->h_gjobs[n_jobs + j] = tmr::GemmJob{acat, Z, Q, nullptr};
            c->h_gjobs[2 * n_jobs + j] = tmr::GemmJob{acat + TP, Z + T, Q, nullptr};
        }
        cudaStream_t s = c->stream;
        TR_CUDA(c, cudaMemcpyAsync(c->rot, c->h_rot, sizeof(float) * 6 * m, cudaMemcpyHostToDevice, s));
        TR_CUDA(c, cudaMemcpyAsync(c->cand, c->h_cand, sizeof(int) * 3 * c->max_batch, cudaMemcpyHostToDevice, s));
        if (n_jobs > 0) {
            // jobs[0:n_jobs] and has_pad[0:n_jobs] (has_pad = jobs + max_batch)
            TR_CUDA(c, cudaMemcpyAsync(c->jobs, c->h_jobs, sizeof(int) * 2 * c->max_batch, cudaMemcpyHostToDevice, s));
            TR_CUDA(c, cudaMemcpyAsync(c->gjobs, c->h_gjobs, sizeof(tmr::GemmJob) * 3 * n_jobs, cudaMemcpyHostToDevice, s));
            TR_CUDA(c, cudaMemsetAsync(c->gemm_err, 0, sizeof(int), s));
        }
        int rc = c->run(c, m, n_jobs);
        if (rc != TM_OK) return rc;
        TR_CUDA(c, cudaMemcpyAsync(c->h_out, c->out, sizeof(float) * 3 * m, cudaMemcpyDeviceToHost, s));
        *c->h_gemm_err = 0;
        if (n_jobs > 0) TR_CUDA(c, cudaMemcpyAsync(c->h_gemm_err, c->gemm_err, sizeof(int), cudaMemcpyDeviceToHost, s));
        rc = wait_refine(c, 120.0);
        if (rc != TM_OK) return rc;
        if (*c->h_gemm_err) return rset_err(c, TM_ERR_TIMEOUT, "a tensor-core GEMM of the pixel-size change timed out");
        memcpy(out + 3 * (size_t)base, c->h_out, sizeof(float) * 3 * m);
    }
    return TM_OK;
}

const char* tm_refine_last_error(const tm_refine_ctx* c) { return c ? c->err.c_str() : "null context"; }

int tm_refine_destroy(tm_refine_ctx* c) {
    if (!c) return TM_ERR_INVALID;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    rfree(c);
    delete c;
    return TM_OK;
}

}  // extern "C"
