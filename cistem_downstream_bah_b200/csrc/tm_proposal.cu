// tm_proposal.cu -- the learned proposal network of the search (C ABI in
// include/tm_b200.h): a 5-layer CNN that reads tiles of the coarse search's
// maps and scores them for the fine search.  The reference has no counterpart;
// its outputs are checked against the FP64 restatement oracle/proposal.py.
//
//   layer 1  conv 3x3, cin -> 32, ReLU, max-pool 2     (tile      -> tile/2)
//   layer 2  conv 3x3, 32 -> 64, ReLU, max-pool 2      (tile/2    -> tile/4)
//   layer 3  conv 3x3, 64 -> 128, ReLU, max-pool 2     (tile/4    -> tile/8)
//   layer 4  conv 3x3, 128 -> 128, ReLU, global max    (tile/8    -> 128)
//   layer 5  fully connected 128 -> 4: objectness logit and a direction
//
// Weights are kept as FP32 master values (Adam state beside them) and used as
// BF16 copies by the forward and the backward-data kernels; activations,
// accumulation and weight gradients are FP32.  The weight gradient is taken
// with respect to the BF16 values the forward used.
//
// Loss of a batch of n tiles with labels (y, t) (y in {0,1}, t a unit vector):
//   L = 1/n sum_i [ w_i BCE(o_i, y_i) + lambda y_i (1 - cos(d_i, t_i)) ]
// with w_i = pos_weight for y_i = 1, else 1, o_i the objectness logit and d_i
// the direction output (only its direction matters: the angular bins are
// ranked by c_b . d).
//
// Every kernel is a bounded loop nest; nothing waits on another block.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>

#include <string>
#include <vector>

#include "../../include/tm_b200.h"

namespace tmp {

constexpr int kC1 = 32, kC2 = 64, kC3 = 128, kC4 = 128, kOut = 4;
constexpr int kThreads = 256;
constexpr int kMaxGroups = 4;   // output-channel groups of a conv block (COB <= 32)

// ----------------------------------------------------------------------------------------------
// 3x3 convolution, zero padding 1, NCHW.  out[n][o][y][x] = b[o] + sum_i sum_k
// in[n][i][y+ky-1][x+kx-1] * W(o, i, ky, kx), optionally ReLU.  With FLIP the
// kernel is the backward-data pass of a forward conv whose weights are
// Wf[co][ci][3][3]: W(o, i, ky, kx) = Wf[i][o][2-ky][2-kx] (o runs over the
// forward conv's input channels, i over its output channels), no bias, no ReLU.
//
// Block: a TH x TW tile of output pixels (TH = TW = min(16, H)) times COB output
// channels (COB = 8 x groups, groups = min(256 / P, 4)); thread t < P x groups
// computes pixel t % P for COT = 8 channels.  Input channels go through shared
// memory CIB = 8 at a time with their halo.
template <bool FLIP>
__global__ void __launch_bounds__(kThreads)
k_conv3x3(const float* __restrict__ in, const __nv_bfloat16* __restrict__ w, const float* __restrict__ bias,
          float* __restrict__ out, int Ci, int Co, int H, int W, int relu) {
    constexpr int CIB = 8, COT = 8;
    const int TH = H < 16 ? H : 16, TW = W < 16 ? W : 16;
    const int P = TH * TW;
    const int groups = kThreads / P < kMaxGroups ? kThreads / P : kMaxGroups;   // P divides 256
    const int COB = groups * COT;
    const int tiles_x = W / TW;
    const int ty0 = (blockIdx.x / tiles_x) * TH, tx0 = (blockIdx.x % tiles_x) * TW;
    const int co0 = blockIdx.y * COB;
    const int n = blockIdx.z;
    const int t = threadIdx.x;
    const int pix = t % P, grp = t / P;
    const int py = pix / TW, px = pix % TW;
    __shared__ float s_in[CIB][18 * 18];
    __shared__ float s_w[kMaxGroups * COT * CIB * 9];
    const bool active = grp < groups;
    float acc[COT];
#pragma unroll
    for (int j = 0; j < COT; j++) acc[j] = 0.0f;
    const int HW = (TH + 2) * (TW + 2);
    for (int ci0 = 0; ci0 < Ci; ci0 += CIB) {
        // input tile with halo
        for (int e = t; e < CIB * HW; e += kThreads) {
            const int c = e / HW, r = e % HW;
            const int yy = ty0 + r / (TW + 2) - 1, xx = tx0 + r % (TW + 2) - 1;
            const int ci = ci0 + c;
            float v = 0.0f;
            if (ci < Ci && yy >= 0 && yy < H && xx >= 0 && xx < W) v = in[(((size_t)n * Ci + ci) * H + yy) * W + xx];
            s_in[c][r] = v;
        }
        // weights of COB output channels x CIB input channels
        for (int e = t; e < COB * CIB * 9; e += kThreads) {
            const int o = e / (CIB * 9), r = e % (CIB * 9);
            const int c = r / 9, k = r % 9;
            const int co = co0 + o, ci = ci0 + c;
            float v = 0.0f;
            if (co < Co && ci < Ci) {
                if (!FLIP) v = __bfloat162float(w[((size_t)co * Ci + ci) * 9 + k]);
                else v = __bfloat162float(w[((size_t)ci * Co + co) * 9 + (8 - k)]);
            }
            s_w[e] = v;
        }
        __syncthreads();
        for (int c = 0; c < CIB && active; c++) {
#pragma unroll
            for (int k = 0; k < 9; k++) {
                const float v = s_in[c][(py + k / 3) * (TW + 2) + px + k % 3];
#pragma unroll
                for (int j = 0; j < COT; j++) acc[j] = fmaf(v, s_w[((grp * COT + j) * CIB + c) * 9 + k], acc[j]);
            }
        }
        __syncthreads();
    }
    if (!active) return;
    const int y = ty0 + py, x = tx0 + px;
#pragma unroll
    for (int j = 0; j < COT; j++) {
        const int co = co0 + grp * COT + j;
        if (co >= Co) continue;
        float v = acc[j] + (bias ? bias[co] : 0.0f);
        if (relu) v = fmaxf(v, 0.0f);
        out[(((size_t)n * Co + co) * H + y) * W + x] = v;
    }
}

// Weight and bias gradients of a 3x3 conv: dW[o][i][k] = sum_n sum_p g[n][o][p] *
// in[n][i][p + k - (1,1)], db[o] = sum_n sum_p g[n][o][p].  One block per
// (o, i) pair and image chunk; the nine sums are reduced in the block and added
// to dW with atomics (dW and db are zeroed before the backward pass).
__global__ void __launch_bounds__(kThreads)
k_conv3x3_wgrad(const float* __restrict__ in, const float* __restrict__ g, float* dW, float* db, int N, int Ci, int Co,
                int H, int W, int n_chunk) {
    const int o = blockIdx.x / Ci, i = blockIdx.x % Ci;
    const int n0 = blockIdx.y * n_chunk, n1 = min(N, n0 + n_chunk);
    const int HWp = H * W;
    float s[10];
#pragma unroll
    for (int k = 0; k < 10; k++) s[k] = 0.0f;
    // threads run over (image, pixel) pairs of the chunk, so that small maps keep them busy
    const long long e1 = (long long)(n1 - n0) * HWp;
    for (long long e = threadIdx.x; e < e1; e += kThreads) {
        const int n = n0 + (int)(e / HWp), p = (int)(e % HWp);
        const float gv = g[((size_t)n * Co + o) * HWp + p];
        if (gv == 0.0f) continue;
        const float* ip = in + ((size_t)n * Ci + i) * HWp;
        const int y = p / W, x = p % W;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const int yy = y + k / 3 - 1, xx = x + k % 3 - 1;
            if (yy >= 0 && yy < H && xx >= 0 && xx < W) s[k] = fmaf(gv, ip[yy * W + xx], s[k]);
        }
        s[9] += gv;
    }
    __shared__ float red[kThreads / 32][10];
#pragma unroll
    for (int k = 0; k < 10; k++) {
        float v = s[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 10) {
        float v = 0.0f;
        for (int w8 = 0; w8 < kThreads / 32; w8++) v += red[w8][threadIdx.x];
        if (threadIdx.x < 9) atomicAdd(&dW[((size_t)o * Ci + i) * 9 + threadIdx.x], v);
        else if (i == 0) atomicAdd(&db[o], v);
    }
}

// 2 x 2 max pool (first maximum in row-major order on ties) with its argmax
__global__ void k_maxpool2(const float* __restrict__ in, float* __restrict__ out, unsigned char* __restrict__ arg,
                           long long planes, int H, int W) {
    const int Ho = H / 2, Wo = W / 2;
    const long long total = planes * Ho * Wo;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long pl = e / (Ho * Wo);
        const int r = (int)(e % (Ho * Wo)), y = r / Wo, x = r % Wo;
        const float* ip = in + pl * H * W + (2 * y) * W + 2 * x;
        float m = ip[0];
        int a = 0;
        if (ip[1] > m) { m = ip[1]; a = 1; }
        if (ip[W] > m) { m = ip[W]; a = 2; }
        if (ip[W + 1] > m) { m = ip[W + 1]; a = 3; }
        out[e] = m;
        arg[e] = (unsigned char)a;
    }
}

// gradient through the max pool and the ReLU before it: the selected input of
// each window receives the output gradient when that input was positive
__global__ void k_maxpool2_bwd(const float* __restrict__ gout, const unsigned char* __restrict__ arg,
                               const float* __restrict__ act, float* __restrict__ gin, long long planes, int H, int W) {
    const int Ho = H / 2, Wo = W / 2;
    const long long total = planes * Ho * Wo;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long pl = e / (Ho * Wo);
        const int r = (int)(e % (Ho * Wo)), y = r / Wo, x = r % Wo;
        const long long base = pl * H * W + (2 * y) * W + 2 * x;
        const int a = arg[e];
        const float gv = gout[e];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const long long idx = base + (q / 2) * W + q % 2;
            gin[idx] = (q == a && act[idx] > 0.0f) ? gv : 0.0f;
        }
    }
}

// global max over the H*W pixels of each plane (first maximum) with its argmax
__global__ void k_global_max(const float* __restrict__ in, float* __restrict__ out, int* __restrict__ arg,
                             long long planes, int HW) {
    for (long long pl = blockIdx.x * (long long)blockDim.x + threadIdx.x; pl < planes;
         pl += (long long)gridDim.x * blockDim.x) {
        const float* ip = in + pl * HW;
        float m = ip[0];
        int a = 0;
        for (int p = 1; p < HW; p++)
            if (ip[p] > m) {
                m = ip[p];
                a = p;
            }
        out[pl] = m;
        arg[pl] = a;
    }
}

__global__ void k_global_max_bwd(const float* __restrict__ gout, const int* __restrict__ arg,
                                 const float* __restrict__ act, float* __restrict__ gin, long long planes, int HW) {
    const long long total = planes * HW;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long pl = e / HW;
        const int p = (int)(e % HW);
        gin[e] = (p == arg[pl] && act[e] > 0.0f) ? gout[pl] : 0.0f;
    }
}

// fully connected 128 -> 4
__global__ void k_fc(const float* __restrict__ g, const __nv_bfloat16* __restrict__ w, const float* __restrict__ b,
                     float* __restrict__ out, int n) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * kOut) return;
    const int i = e / kOut, j = e % kOut;
    float s = b[j];
    for (int c = 0; c < kC4; c++) s = fmaf(g[(size_t)i * kC4 + c], __bfloat162float(w[j * kC4 + c]), s);
    out[e] = s;
}

// loss terms and the gradient of the outputs; one thread per tile
__global__ void k_loss(const float* __restrict__ out, const float* __restrict__ labels, float* __restrict__ dout,
                       double* loss, int n, float pos_weight, float dir_weight) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* o = out + (size_t)i * kOut;
    const float* l = labels + (size_t)i * 4;
    const float y = l[0];
    const float wgt = y > 0.5f ? pos_weight : 1.0f;
    const float inv_n = 1.0f / (float)n;
    // BCE with logits: max(o, 0) - o y + log(1 + exp(-|o|))
    const float z = o[0];
    const float bce = fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z)));
    const float sig = 1.0f / (1.0f + expf(-z));
    float li = wgt * bce;
    float* d = dout + (size_t)i * kOut;
    d[0] = inv_n * wgt * (sig - y);
    d[1] = d[2] = d[3] = 0.0f;
    if (y > 0.5f) {
        const float dx = o[1], dy = o[2], dz = o[3];
        const float nn = dx * dx + dy * dy + dz * dz + 1e-12f;
        const float inv = rsqrtf(nn);
        const float dot = dx * l[1] + dy * l[2] + dz * l[3];
        li += dir_weight * (1.0f - dot * inv);
        const float c = -dir_weight * inv_n * inv;
        const float f = dot / nn;
        d[1] = c * (l[1] - f * dx);
        d[2] = c * (l[2] - f * dy);
        d[3] = c * (l[3] - f * dz);
    }
    atomicAdd(loss, (double)(li * inv_n));
}

// FC backward: dW5, db5 (one thread per weight) and dg
__global__ void k_fc_wgrad(const float* __restrict__ g, const float* __restrict__ dout, float* dW, float* db, int n) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= kOut * (kC4 + 1)) return;
    const int j = e / (kC4 + 1), c = e % (kC4 + 1);
    float s = 0.0f;
    for (int i = 0; i < n; i++) s = fmaf(dout[(size_t)i * kOut + j], c < kC4 ? g[(size_t)i * kC4 + c] : 1.0f, s);
    if (c < kC4) dW[j * kC4 + c] = s;
    else db[j] = s;
}

__global__ void k_fc_dgrad(const float* __restrict__ dout, const __nv_bfloat16* __restrict__ w, float* __restrict__ dg,
                           int n) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * kC4) return;
    const int i = e / kC4, c = e % kC4;
    float s = 0.0f;
#pragma unroll
    for (int j = 0; j < kOut; j++) s = fmaf(dout[(size_t)i * kOut + j], __bfloat162float(w[j * kC4 + c]), s);
    dg[e] = s;
}

__global__ void k_to_bf16(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst, long long n) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        dst[e] = __float2bfloat16_rn(src[e]);
}

// Adam (Kingma & Ba 2015) on the FP32 master values, then the BF16 copies
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       __nv_bfloat16* __restrict__ p16, long long n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const float ge = g[e];
        const float me = b1 * m[e] + (1.0f - b1) * ge;
        const float ve = b2 * v[e] + (1.0f - b2) * ge * ge;
        m[e] = me;
        v[e] = ve;
        const float pe = p[e] - lr * (me / c1) / (sqrtf(ve / c2) + eps);
        p[e] = pe;
        p16[e] = __float2bfloat16_rn(pe);
    }
}

// ----------------------------------------------------------------------------------------------
struct Layer {
    int ci, co, h;       // input channels, output channels, input height (= width)
    long long w, b;      // offsets of the weights and the bias in the parameter array
};

}  // namespace tmp

struct tm_pnet {
    int device = 0, cin = 0, tile = 0, max_batch = 0, nsm = 148;
    long long nparam = 0;
    tmp::Layer L[5];
    cudaStream_t stream = nullptr;
    float *p = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    __nv_bfloat16* p16 = nullptr;
    int step = 0;
    // activations (max_batch tiles) and their gradients
    float *x = nullptr, *a1 = nullptr, *q1 = nullptr, *a2 = nullptr, *q2 = nullptr, *a3 = nullptr, *q3 = nullptr,
          *a4 = nullptr, *g = nullptr, *out = nullptr, *lab = nullptr;
    unsigned char *i1 = nullptr, *i2 = nullptr, *i3 = nullptr;
    int* i4 = nullptr;
    float *d_a1 = nullptr, *d_q1 = nullptr, *d_a2 = nullptr, *d_q2 = nullptr, *d_a3 = nullptr, *d_q3 = nullptr,
          *d_a4 = nullptr, *d_g = nullptr, *d_out = nullptr;
    double* d_loss = nullptr;
    std::vector<void*> owned;
    std::string err;
};

namespace {

int pset_err(tm_pnet* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define PN_CUDA(c, expr)                                                                                     \
    do {                                                                                                     \
        cudaError_t e_ = (expr);                                                                             \
        if (e_ != cudaSuccess) return pset_err(c, TM_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_));    \
    } while (0)

template <typename T>
int palloc(tm_pnet* c, T** ptr, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 16);
    if (e != cudaSuccess) return pset_err(c, TM_ERR_CUDA, "cudaMalloc(%zu): %s", count * sizeof(T), cudaGetErrorString(e));
    c->owned.push_back(q);
    *ptr = (T*)q;
    return TM_OK;
}

int grid_for(long long n) {
    long long b = (n + 255) / 256;
    return (int)(b < 148LL * 16 ? (b > 0 ? b : 1) : 148LL * 16);
}

// launch of one conv: grid (spatial tiles, output-channel groups, images)
int conv(tm_pnet* c, bool flip, const float* in, const float* bias, float* out, const tmp::Layer& l, int n, int relu) {
    const int H = l.h;
    const int TH = H < 16 ? H : 16;
    const int P = TH * TH;
    const int COB = (tmp::kThreads / P < tmp::kMaxGroups ? tmp::kThreads / P : tmp::kMaxGroups) * 8;
    const int ci = flip ? l.co : l.ci, co = flip ? l.ci : l.co;
    dim3 grid((H / TH) * (H / TH), (co + COB - 1) / COB, n);
    if (flip)
        tmp::k_conv3x3<true><<<grid, tmp::kThreads, 0, c->stream>>>(in, c->p16 + l.w, nullptr, out, ci, co, H, H, 0);
    else
        tmp::k_conv3x3<false><<<grid, tmp::kThreads, 0, c->stream>>>(in, c->p16 + l.w, bias, out, ci, co, H, H, relu);
    PN_CUDA(c, cudaGetLastError());
    return TM_OK;
}

int forward(tm_pnet* c, int n) {
    using namespace tmp;
    const int h1 = c->tile, h2 = h1 / 2, h3 = h1 / 4, h4 = h1 / 8;
    int rc;
    if ((rc = conv(c, false, c->x, c->p + c->L[0].b, c->a1, c->L[0], n, 1))) return rc;
    k_maxpool2<<<grid_for((long long)n * kC1 * h2 * h2), 256, 0, c->stream>>>(c->a1, c->q1, c->i1, (long long)n * kC1, h1, h1);
    if ((rc = conv(c, false, c->q1, c->p + c->L[1].b, c->a2, c->L[1], n, 1))) return rc;
    k_maxpool2<<<grid_for((long long)n * kC2 * h3 * h3), 256, 0, c->stream>>>(c->a2, c->q2, c->i2, (long long)n * kC2, h2, h2);
    if ((rc = conv(c, false, c->q2, c->p + c->L[2].b, c->a3, c->L[2], n, 1))) return rc;
    k_maxpool2<<<grid_for((long long)n * kC3 * h4 * h4), 256, 0, c->stream>>>(c->a3, c->q3, c->i3, (long long)n * kC3, h3, h3);
    if ((rc = conv(c, false, c->q3, c->p + c->L[3].b, c->a4, c->L[3], n, 1))) return rc;
    k_global_max<<<grid_for((long long)n * kC4), 256, 0, c->stream>>>(c->a4, c->g, c->i4, (long long)n * kC4, h4 * h4);
    k_fc<<<(n * kOut + 127) / 128, 128, 0, c->stream>>>(c->g, c->p16 + c->L[4].w, c->p + c->L[4].b, c->out, n);
    PN_CUDA(c, cudaGetLastError());
    return TM_OK;
}

int wgrad(tm_pnet* c, const float* in, const float* g, const tmp::Layer& l, int n) {
    const int pairs = l.ci * l.co;
    int chunks = (148 * 8 + pairs - 1) / pairs;
    if (chunks > n) chunks = n;
    if (chunks < 1) chunks = 1;
    const int n_chunk = (n + chunks - 1) / chunks;
    dim3 grid(pairs, (n + n_chunk - 1) / n_chunk);
    tmp::k_conv3x3_wgrad<<<grid, tmp::kThreads, 0, c->stream>>>(in, g, c->grad + l.w, c->grad + l.b, n, l.ci, l.co, l.h,
                                                                l.h, n_chunk);
    PN_CUDA(c, cudaGetLastError());
    return TM_OK;
}

// forward + loss + backward into c->grad; the loss sum into c->d_loss
int backward(tm_pnet* c, int n, float pos_weight, float dir_weight) {
    using namespace tmp;
    const int h1 = c->tile, h2 = h1 / 2, h3 = h1 / 4, h4 = h1 / 8;
    int rc;
    if ((rc = forward(c, n))) return rc;
    PN_CUDA(c, cudaMemsetAsync(c->grad, 0, sizeof(float) * c->nparam, c->stream));
    PN_CUDA(c, cudaMemsetAsync(c->d_loss, 0, sizeof(double), c->stream));
    k_loss<<<(n + 127) / 128, 128, 0, c->stream>>>(c->out, c->lab, c->d_out, c->d_loss, n, pos_weight, dir_weight);
    k_fc_wgrad<<<(kOut * (kC4 + 1) + 127) / 128, 128, 0, c->stream>>>(c->g, c->d_out, c->grad + c->L[4].w,
                                                                        c->grad + c->L[4].b, n);
    k_fc_dgrad<<<(n * kC4 + 255) / 256, 256, 0, c->stream>>>(c->d_out, c->p16 + c->L[4].w, c->d_g, n);
    k_global_max_bwd<<<grid_for((long long)n * kC4 * h4 * h4), 256, 0, c->stream>>>(c->d_g, c->i4, c->a4, c->d_a4,
                                                                                    (long long)n * kC4, h4 * h4);
    PN_CUDA(c, cudaGetLastError());
    // layer 4
    if ((rc = wgrad(c, c->q3, c->d_a4, c->L[3], n))) return rc;
    if ((rc = conv(c, true, c->d_a4, nullptr, c->d_q3, c->L[3], n, 0))) return rc;
    k_maxpool2_bwd<<<grid_for((long long)n * kC3 * h4 * h4), 256, 0, c->stream>>>(c->d_q3, c->i3, c->a3, c->d_a3,
                                                                                  (long long)n * kC3, h3, h3);
    // layer 3
    if ((rc = wgrad(c, c->q2, c->d_a3, c->L[2], n))) return rc;
    if ((rc = conv(c, true, c->d_a3, nullptr, c->d_q2, c->L[2], n, 0))) return rc;
    k_maxpool2_bwd<<<grid_for((long long)n * kC2 * h3 * h3), 256, 0, c->stream>>>(c->d_q2, c->i2, c->a2, c->d_a2,
                                                                                  (long long)n * kC2, h2, h2);
    // layer 2
    if ((rc = wgrad(c, c->q1, c->d_a2, c->L[1], n))) return rc;
    if ((rc = conv(c, true, c->d_a2, nullptr, c->d_q1, c->L[1], n, 0))) return rc;
    k_maxpool2_bwd<<<grid_for((long long)n * kC1 * h2 * h2), 256, 0, c->stream>>>(c->d_q1, c->i1, c->a1, c->d_a1,
                                                                                  (long long)n * kC1, h1, h1);
    // layer 1 (no gradient of the input)
    if ((rc = wgrad(c, c->x, c->d_a1, c->L[0], n))) return rc;
    PN_CUDA(c, cudaGetLastError());
    return TM_OK;
}

int upload(tm_pnet* c, const float* tiles, const float* labels, int n) {
    if (n < 1 || n > c->max_batch) return pset_err(c, TM_ERR_INVALID, "batch %d outside 1..%d", n, c->max_batch);
    if (!tiles) return pset_err(c, TM_ERR_INVALID, "null tiles");
    const size_t per = (size_t)c->cin * c->tile * c->tile;
    PN_CUDA(c, cudaMemcpyAsync(c->x, tiles, sizeof(float) * per * n, cudaMemcpyHostToDevice, c->stream));
    if (labels) PN_CUDA(c, cudaMemcpyAsync(c->lab, labels, sizeof(float) * 4 * n, cudaMemcpyHostToDevice, c->stream));
    return TM_OK;
}

}  // namespace

extern "C" {

int tm_pnet_create(int device, int in_channels, int tile, int max_batch, tm_pnet** out) {
    if (!out) return TM_ERR_INVALID;
    *out = nullptr;
    if (in_channels < 1 || in_channels > 64 || max_batch < 1 || max_batch > 4096) return TM_ERR_INVALID;
    if (tile != 16 && tile != 32 && tile != 64 && tile != 128) return TM_ERR_UNSUPPORTED;
    tm_pnet* c = new tm_pnet();
    c->device = device;
    c->cin = in_channels;
    c->tile = tile;
    c->max_batch = max_batch;
    const int chans[5] = {in_channels, tmp::kC1, tmp::kC2, tmp::kC3, tmp::kC4};
    long long off = 0;
    for (int l = 0; l < 4; l++) {
        c->L[l].ci = chans[l];
        c->L[l].co = chans[l + 1];
        c->L[l].h = tile >> l;
        c->L[l].w = off;
        off += (long long)chans[l] * chans[l + 1] * 9;
        c->L[l].b = off;
        off += chans[l + 1];
    }
    c->L[4].ci = tmp::kC4;
    c->L[4].co = tmp::kOut;
    c->L[4].h = 1;
    c->L[4].w = off;
    off += tmp::kC4 * tmp::kOut;
    c->L[4].b = off;
    off += tmp::kOut;
    c->nparam = off;
    auto fail = [&](int rc) {
        tm_pnet_destroy(c);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return fail(TM_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(TM_ERR_CUDA);
    const long long B = max_batch, h = tile;
    int rc = TM_OK;
    rc = rc ? rc : palloc(c, &c->p, c->nparam);
    rc = rc ? rc : palloc(c, &c->grad, c->nparam);
    rc = rc ? rc : palloc(c, &c->m, c->nparam);
    rc = rc ? rc : palloc(c, &c->v, c->nparam);
    rc = rc ? rc : palloc(c, &c->p16, c->nparam);
    rc = rc ? rc : palloc(c, &c->x, B * in_channels * h * h);
    rc = rc ? rc : palloc(c, &c->a1, B * tmp::kC1 * h * h);
    rc = rc ? rc : palloc(c, &c->q1, B * tmp::kC1 * h * h / 4);
    rc = rc ? rc : palloc(c, &c->i1, B * tmp::kC1 * h * h / 4);
    rc = rc ? rc : palloc(c, &c->a2, B * tmp::kC2 * h * h / 4);
    rc = rc ? rc : palloc(c, &c->q2, B * tmp::kC2 * h * h / 16);
    rc = rc ? rc : palloc(c, &c->i2, B * tmp::kC2 * h * h / 16);
    rc = rc ? rc : palloc(c, &c->a3, B * tmp::kC3 * h * h / 16);
    rc = rc ? rc : palloc(c, &c->q3, B * tmp::kC3 * h * h / 64);
    rc = rc ? rc : palloc(c, &c->i3, B * tmp::kC3 * h * h / 64);
    rc = rc ? rc : palloc(c, &c->a4, B * tmp::kC4 * h * h / 64);
    rc = rc ? rc : palloc(c, &c->g, B * tmp::kC4);
    rc = rc ? rc : palloc(c, &c->i4, B * tmp::kC4);
    rc = rc ? rc : palloc(c, &c->out, B * tmp::kOut);
    rc = rc ? rc : palloc(c, &c->lab, B * 4);
    rc = rc ? rc : palloc(c, &c->d_a1, B * tmp::kC1 * h * h);
    rc = rc ? rc : palloc(c, &c->d_q1, B * tmp::kC1 * h * h / 4);
    rc = rc ? rc : palloc(c, &c->d_a2, B * tmp::kC2 * h * h / 4);
    rc = rc ? rc : palloc(c, &c->d_q2, B * tmp::kC2 * h * h / 16);
    rc = rc ? rc : palloc(c, &c->d_a3, B * tmp::kC3 * h * h / 16);
    rc = rc ? rc : palloc(c, &c->d_q3, B * tmp::kC3 * h * h / 64);
    rc = rc ? rc : palloc(c, &c->d_a4, B * tmp::kC4 * h * h / 64);
    rc = rc ? rc : palloc(c, &c->d_g, B * tmp::kC4);
    rc = rc ? rc : palloc(c, &c->d_out, B * tmp::kOut);
    rc = rc ? rc : palloc(c, &c->d_loss, 1);
    if (rc) return fail(rc);
    if (cudaMemset(c->p, 0, sizeof(float) * c->nparam) != cudaSuccess ||
        cudaMemset(c->m, 0, sizeof(float) * c->nparam) != cudaSuccess ||
        cudaMemset(c->v, 0, sizeof(float) * c->nparam) != cudaSuccess ||
        cudaMemset(c->p16, 0, sizeof(__nv_bfloat16) * c->nparam) != cudaSuccess)
        return fail(TM_ERR_CUDA);
    *out = c;
    return TM_OK;
}

long long tm_pnet_param_count(const tm_pnet* c) { return c ? c->nparam : -1; }

int tm_pnet_set_params(tm_pnet* c, const float* params) {
    if (!c || !params) return TM_ERR_INVALID;
    PN_CUDA(c, cudaSetDevice(c->device));
    PN_CUDA(c, cudaMemcpyAsync(c->p, params, sizeof(float) * c->nparam, cudaMemcpyHostToDevice, c->stream));
    PN_CUDA(c, cudaMemsetAsync(c->m, 0, sizeof(float) * c->nparam, c->stream));
    PN_CUDA(c, cudaMemsetAsync(c->v, 0, sizeof(float) * c->nparam, c->stream));
    tmp::k_to_bf16<<<grid_for(c->nparam), 256, 0, c->stream>>>(c->p, c->p16, c->nparam);
    PN_CUDA(c, cudaGetLastError());
    PN_CUDA(c, cudaStreamSynchronize(c->stream));
    c->step = 0;
    return TM_OK;
}

int tm_pnet_get_params(tm_pnet* c, float* params) {
    if (!c || !params) return TM_ERR_INVALID;
    PN_CUDA(c, cudaSetDevice(c->device));
    PN_CUDA(c, cudaMemcpyAsync(params, c->p, sizeof(float) * c->nparam, cudaMemcpyDeviceToHost, c->stream));
    PN_CUDA(c, cudaStreamSynchronize(c->stream));
    return TM_OK;
}

int tm_pnet_forward(tm_pnet* c, const float* tiles, int n, float* outputs) {
    if (!c || !outputs) return TM_ERR_INVALID;
    PN_CUDA(c, cudaSetDevice(c->device));
    int rc = upload(c, tiles, nullptr, n);
    if (rc) return rc;
    if ((rc = forward(c, n))) return rc;
    PN_CUDA(c, cudaMemcpyAsync(outputs, c->out, sizeof(float) * tmp::kOut * n, cudaMemcpyDeviceToHost, c->stream));
    PN_CUDA(c, cudaStreamSynchronize(c->stream));
    return TM_OK;
}

int tm_pnet_gradients(tm_pnet* c, const float* tiles, const float* labels, int n, float pos_weight, float dir_weight,
                      double* loss, float* grads) {
    if (!c || !labels || !loss || !grads) return TM_ERR_INVALID;
    PN_CUDA(c, cudaSetDevice(c->device));
    int rc = upload(c, tiles, labels, n);
    if (rc) return rc;
    if ((rc = backward(c, n, pos_weight, dir_weight))) return rc;
    PN_CUDA(c, cudaMemcpyAsync(grads, c->grad, sizeof(float) * c->nparam, cudaMemcpyDeviceToHost, c->stream));
    PN_CUDA(c, cudaMemcpyAsync(loss, c->d_loss, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PN_CUDA(c, cudaStreamSynchronize(c->stream));
    return TM_OK;
}

int tm_pnet_train_step(tm_pnet* c, const float* tiles, const float* labels, int n, float pos_weight, float dir_weight,
                       float lr, double* loss) {
    if (!c || !labels) return TM_ERR_INVALID;
    PN_CUDA(c, cudaSetDevice(c->device));
    int rc = upload(c, tiles, labels, n);
    if (rc) return rc;
    if ((rc = backward(c, n, pos_weight, dir_weight))) return rc;
    c->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)c->step), c2 = 1.0f - powf(b2, (float)c->step);
    tmp::k_adam<<<grid_for(c->nparam), 256, 0, c->stream>>>(c->p, c->grad, c->m, c->v, c->p16, c->nparam, lr, b1, b2,
                                                           1e-8f, c1, c2);
    PN_CUDA(c, cudaGetLastError());
    if (loss) PN_CUDA(c, cudaMemcpyAsync(loss, c->d_loss, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PN_CUDA(c, cudaStreamSynchronize(c->stream));
    return TM_OK;
}

const char* tm_pnet_last_error(const tm_pnet* c) { return c ? c->err.c_str() : "null network"; }

int tm_pnet_destroy(tm_pnet* c) {
    if (!c) return TM_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (void* q : c->owned) cudaFree(q);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return TM_OK;
}

}  // extern "C"
