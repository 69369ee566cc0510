// tm_whiten.cuh -- the micrograph whitening of match_template on the device
// (match_template.cpp:699-724, the same steps as the host restatement in
// host/prep.cpp, whiten()):
//
//   k_w_stats      sum and sum of squares (ReplaceOutliersWithMean(5), image.cpp:986-1007)
//   k_w_rows<X>    outliers replaced by the mean, r2c FFT of each row
//   k_w_cols<Y>    FFT of each column, SwapRealSpaceQuadrants (float phase
//                  shift as Image::PhaseShift forms it), zeroed central pixel
//   k_w_curve      Compute1DPowerSpectrumCurve: |F|^2 and counts accumulated
//                  into the radial curve with linear interpolation
//                  (Curve::AddValueAtXUsingLinearInterpolation), per-block
//                  shared bins then global double atomics
//   (host)         SquareRoot, Reciprocal, MultiplyByConstant(1 / max)
//   k_w_apply      ApplyCurveFilter, zeroed central pixel, the Hermitian-
//                  weighted sum of squares (ReturnSumOfSquares)
//   k_w_scale      division by sqrt(2 x sum)
//
// The forward transform is left unscaled: the curve is normalised by its
// maximum and the spectrum by its norm, so the reference's 1/N cancels.
#pragma once
#include "tm_fft.cuh"

namespace tmw {

using tmfft::cmul;
using tmfft::Twiddles;

__host__ __device__ constexpr int round_up16(int v) { return (v + 15) / 16 * 16; }
__host__ __device__ constexpr int skewed(int len, int rem) { return round_up16(len) + rem; }

__device__ __forceinline__ int logical(int phys, int n) { return phys >= (n % 2 == 0 ? n / 2 : n / 2 + 1) ? phys - n : phys; }

// ----------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_w_stats(const float* __restrict__ img, long long n, double* stats) {
    double s = 0.0, q = 0.0;
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
        const double v = img[i];
        s += v;
        q += v * v;
    }
    __shared__ double rs[8], rq[8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, off);
        q += __shfl_xor_sync(0xffffffffu, q, off);
    }
    if ((threadIdx.x & 31) == 0) {
        rs[threadIdx.x >> 5] = s;
        rq[threadIdx.x >> 5] = q;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ts = 0.0, tq = 0.0;
        for (int k = 0; k < 8; k++) {
            ts += rs[k];
            tq += rq[k];
        }
        atomicAdd(stats, ts);
        atomicAdd(stats + 1, tq);
    }
}

// ----------------------------------------------------------------------------------------------
// rows: X reals -> X/2+1 complex through an X/2-point FFT of the even/odd pairs
template <int X>
struct WRows {
    static constexpr int H = X / 2;
    static constexpr int V = 16;
    static constexpr int PH = H / V;
    static constexpr int RS = skewed(tmfft::padded_len(H), PH % 16);
    static constexpr int ROWS = PH >= 256 ? 1 : 256 / PH;
    static constexpr int NT = ROWS * PH;
};

template <int X>
__global__ void __launch_bounds__(WRows<X>::NT) k_w_rows(const float* __restrict__ img, float2* spec, int Y,
                                                          float mean, float vmin, float vmax, Twiddles tw) {
    using R = WRows<X>;
    constexpr int H = R::H, PH = R::PH, V = R::V, RS = R::RS, HC = X / 2 + 1;
    __shared__ float2 sm[R::ROWS * RS];
    const int t = threadIdx.x % PH, rl = threadIdx.x / PH;
    const int y = blockIdx.x * R::ROWS + rl;
    const bool valid = y < Y;
    const float* src = img + (size_t)(valid ? y : 0) * X;
    float2 v[V];
#pragma unroll
    for (int r = 0; r < V; r++) {
        const int n = t + PH * r;
        float a = src[2 * n], b = src[2 * n + 1];
        if (a > vmax || a < vmin) a = mean;
        if (b > vmax || b < vmin) b = mean;
        v[r] = make_float2(a, b);
    }
    float2* buf = sm + rl * RS;
    tmfft::fft<H, V, -1>(v, t, buf, tw, [] __device__() { __syncthreads(); });
    __syncthreads();
#pragma unroll
    for (int r = 0; r < V; r++) buf[tmfft::pad16(t + PH * r)] = v[r];
    __syncthreads();
    if (!valid) return;
    float2* row = spec + (size_t)y * HC;
#pragma unroll
    for (int r = 0; r < V; r++) {
        const int k = t + PH * r;
        const float2 zk = v[r];
        const float2 zm = buf[tmfft::pad16(k == 0 ? 0 : H - k)];
        const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
        const float2 wo = cmul(o, tw.template w<-1>(k, X));
        row[k] = make_float2(e.x + wo.x, e.y + wo.y);
        if (k == 0) row[H] = make_float2(e.x - o.x, e.y - o.y);
    }
}

// ----------------------------------------------------------------------------------------------
// columns: Y-point FFT, quadrant swap, zeroed DC; one column per PT threads
template <int Y>
struct WCols {
    static constexpr int V = Y % 3 == 0 ? 18 : 16;
    static constexpr int PT = Y / V;
    static constexpr int RS = skewed(tmfft::padded_len(Y), 1);
    static constexpr int CB = PT >= 128 ? 1 : 128 / PT;
    static constexpr int NT = CB * PT;
    static constexpr int SMEM = CB * RS * 8;
};

template <int Y>
__global__ void __launch_bounds__(WCols<Y>::NT) k_w_cols(float2* spec, int X, Twiddles tw) {
    using C = WCols<Y>;
    constexpr int V = C::V, PT = C::PT, CB = C::CB, RS = C::RS;
    extern __shared__ float2 wsm[];
    const int HC = X / 2 + 1;
    const int il = threadIdx.x % CB, tp = threadIdx.x / CB;
    const int i = blockIdx.x * CB + il;
    const bool valid = i < HC;
    float2* col = spec + (valid ? i : 0);
    float2 v[V];
#pragma unroll
    for (int r = 0; r < V; r++) v[r] = col[(size_t)(tp + PT * r) * HC];
    tmfft::fft<Y, V, -1>(v, tp, wsm + il * RS, tw, [] __device__() { __syncthreads(); });
    if (!valid) return;
    // SwapRealSpaceQuadrants: phase shift by (X/2, Y/2), phase formed in float
    // as Image::PhaseShift does (image.cpp:9221-9265)
    const double kPi = 3.14159265359;
    const float sx = (float)(X / 2), sy = (float)(Y / 2);
    const float px = (float)(sx * (float)i * 2.0 * kPi / X);
#pragma unroll
    for (int r = 0; r < V; r++) {
        const int y = tp + PT * r;
        const float py = (float)(sy * (float)logical(y, Y) * 2.0 * kPi / Y);
        const float th = -px - py;
        const float c = cosf(th), s = sinf(th);
        float2 a = v[r];
        a = make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
        if (i == 0 && y == 0) a = make_float2(0.f, 0.f);
        col[(size_t)y * HC] = a;
    }
}

// ----------------------------------------------------------------------------------------------
// the radial curve: n points on [0, hi], x[k] as Curve::SetupXAxis forms them (float)
struct CurveArgs {
    const float* x;   // n abscissae
    int n;
    float x0, x1;     // x[0], x[1]
};

// Curve::AddValueAtXUsingLinearInterpolation into shared bins
__device__ __forceinline__ void curve_add(const CurveArgs& c, double* bins, float f, double v) {
    int i = (c.x0 == c.x1) ? c.n - 2 : (int)((f - c.x0) / (c.x1 - c.x0));
    if (i > c.n - 1) i = c.n - 1;
    if (i < 0) i = 0;
    if (i == c.n - 1) {
        atomicAdd(bins + i, v);
        return;
    }
    const float d = (f - c.x[i]) / (c.x[i + 1] - c.x[i]);
    atomicAdd(bins + i, v * (1.0 - d));
    atomicAdd(bins + i + 1, v * (double)d);
}

// Compute1DPowerSpectrumCurve (image.cpp:7135-7201): |F|^2 into pw, 1 into cnt,
// skipping the x = 0 column's negative frequencies; smem = 2 n doubles
__global__ void __launch_bounds__(256) k_w_curve(const float2* __restrict__ spec, int X, int Y, CurveArgs c,
                                                 double* pw, double* cnt) {
    extern __shared__ double bins[];
    double* spw = bins;
    double* scnt = bins + c.n;
    for (int k = threadIdx.x; k < 2 * c.n; k += blockDim.x) bins[k] = 0.0;
    __syncthreads();
    const int HC = X / 2 + 1;
    const float vx = (float)(1.0 / (double)X), vy = (float)(1.0 / (double)Y);
    const int first_neg = Y % 2 == 0 ? Y / 2 : Y / 2 + 1;
    const long long n = (long long)Y * HC;
    for (long long p = blockIdx.x * 256LL + threadIdx.x; p < n; p += (long long)gridDim.x * 256) {
        const int y = (int)(p / HC), x = (int)(p % HC);
        if (x == 0 && y >= first_neg) continue;
        const float sy = powf(logical(y, Y) * vy, 2);
        const float f = sqrtf(powf(x * vx, 2) + sy);
        const float2 a = spec[p];
        curve_add(c, spw, f, (double)a.x * a.x + (double)a.y * a.y);
        curve_add(c, scnt, f, 1.0);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < c.n; k += blockDim.x) {
        if (spw[k] != 0.0) atomicAdd(pw + k, spw[k]);
        if (scnt[k] != 0.0) atomicAdd(cnt + k, scnt[k]);
    }
}

// Curve::ReturnLinearInterpolationFromX (curve.cpp:377-397) on the filter curve:
// the interval [x[k], x[k+1]) holding f (found from an estimate and checked
// against the stored abscissae), else the last point; below x[0] the first
__device__ __forceinline__ double curve_at(const CurveArgs& c, const double* y, float f) {
    int i = c.n - 1;
    if (f == f) {
        int k = (int)((f - c.x0) / (c.x1 - c.x0));
        if (k < 0) k = 0;
        if (k > c.n - 2) k = c.n - 2;
        while (k > 0 && f < c.x[k]) k--;
        while (k < c.n - 2 && f >= c.x[k + 1]) k++;
        if (f >= c.x[k] && f < c.x[k + 1]) i = k;
    }
    if (f < c.x[0]) i = 0;
    if (i == c.n - 1) return y[c.n - 1];
    const float d = (f - c.x[i]) / (c.x[i + 1] - c.x[i]);
    return y[i] * (1.0 - d) + y[i + 1] * (double)d;
}

// ApplyCurveFilter (image.cpp:7284-7310), zeroed DC, Hermitian-weighted sum of squares
__global__ void __launch_bounds__(256) k_w_apply(float2* spec, int X, int Y, CurveArgs c, const double* __restrict__ wf,
                                                 double* sumsq) {
    const int HC = X / 2 + 1;
    const float vx = (float)(1.0 / (double)X), vy = (float)(1.0 / (double)Y);
    const long long n = (long long)Y * HC;
    double ss = 0.0;
    for (long long p = blockIdx.x * 256LL + threadIdx.x; p < n; p += (long long)gridDim.x * 256) {
        const int y = (int)(p / HC), x = (int)(p % HC);
        const int jj = logical(y, Y);
        const double sy = pow((double)(jj * vy), 2.0);
        const float f = (float)sqrt(pow((double)(x * vx), 2.0) + sy);
        float2 a = spec[p];
        if (f <= 1.0f) {
            const double w = curve_at(c, wf, f);
            a = make_float2((float)(a.x * w), (float)(a.y * w));
        } else {
            a = make_float2(0.f, 0.f);
        }
        if (p == 0) a = make_float2(0.f, 0.f);
        spec[p] = a;
        const double q = (double)a.x * a.x + (double)a.y * a.y;
        const bool ex = x == 0 || (x == X / 2 && X % 2 == 0);
        const bool ey = jj == 0 || (jj == -(Y / 2) && X % 2 == 0);
        if (ex && ey) ss += 0.5 * q;
        else if ((x != 0 && (x != X / 2 || X % 2 != 0)) || jj >= 0) ss += q;
    }
    __shared__ double rs[8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, off);
    if ((threadIdx.x & 31) == 0) rs[threadIdx.x >> 5] = ss;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < 8; k++) t += rs[k];
        atomicAdd(sumsq, t);
    }
}

__global__ void __launch_bounds__(256) k_w_scale(float2* spec, long long n, const double* __restrict__ sumsq) {
    const double inv = 1.0 / sqrt(2.0 * sumsq[0]);
    for (long long p = blockIdx.x * 256LL + threadIdx.x; p < n; p += (long long)gridDim.x * 256) {
        const float2 a = spec[p];
        spec[p] = make_float2((float)(a.x * inv), (float)(a.y * inv));
    }
}

}  // namespace tmw
