// tm_template.cuh -- the template spectrum of match_template on the device
// (match_template.cpp:842-845: ChangePixelSize(..., return_fft = true),
// ZeroCentralPixel, SwapRealSpaceQuadrants; the steps of the host
// restatement host/prep.cpp, template_spectrum()):
//
//   [factor outside the 0.001 tolerance] k_t_disc_sum: the pad value (mean
//     within 0.45 T of the centre, ReturnAverageOfRealValues); then the
//     ChangePixelSize chain (pad to P^3, FFT, Fourier crop or grow to N^3,
//     inverse FFT, clip) as three axis operators (complex T x T, built on the
//     host) applied by batched GEMMs to vol - pad, real part, / P^3 + pad
//   k_t_rows<T>   r2c of each x row (T reals -> T/2+1)
//   k_t_cols<T>   complex FFT along y, then along z; the z pass scales by
//                 1/T^3, zeroes the central pixel and applies the quadrant
//                 swap (a phase shift by T/2 per axis, formed in float as
//                 Image::PhaseShift does)
#pragma once
#include "tm_fft.cuh"

namespace tmt {

using tmfft::cmul;
using tmfft::Twiddles;

__host__ __device__ constexpr int round_up16(int v) { return (v + 15) / 16 * 16; }
__host__ __device__ constexpr int skewed(int len, int rem) { return round_up16(len) + rem; }
__device__ __forceinline__ int logical(int phys, int n) { return phys >= (n % 2 == 0 ? n / 2 : n / 2 + 1) ? phys - n : phys; }

// mean of the voxels with powf distances^2 <= (0.45 T)^2 (integers: exact in float)
__global__ void __launch_bounds__(256) k_t_disc_sum(const float* __restrict__ vol, int T, double* acc) {
    const float r2 = powf(0.45f * (float)T, 2);
    const int c = T / 2;
    const long long n = (long long)T * T * T;
    double s = 0.0, k = 0.0;
    for (long long p = blockIdx.x * 256LL + threadIdx.x; p < n; p += (long long)gridDim.x * 256) {
        const int z = (int)(p / ((long long)T * T)), y = (int)((p / T) % T), x = (int)(p % T);
        const float d = powf((float)(z - c), 2) + powf((float)(y - c), 2) + powf((float)(x - c), 2);
        if (d <= r2) {
            s += vol[p];
            k += 1.0;
        }
    }
    __shared__ double rs[8], rk[8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, off);
        k += __shfl_xor_sync(0xffffffffu, k, off);
    }
    if ((threadIdx.x & 31) == 0) {
        rs[threadIdx.x >> 5] = s;
        rk[threadIdx.x >> 5] = k;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ts = 0.0, tk = 0.0;
        for (int w = 0; w < 8; w++) {
            ts += rs[w];
            tk += rk[w];
        }
        atomicAdd(acc, ts);
        atomicAdd(acc + 1, tk);
    }
}

// ----------------------------------------------------------------------------------------------
template <int T>
struct TRows {
    static constexpr int H = T / 2;
    static constexpr int V = H % 3 == 0 ? 24 : 16;
    static constexpr int PH = H / V;
    static constexpr int RS = skewed(tmfft::padded_len(H), PH % 16);
    static constexpr int rows_fit() {
        int r = PH >= 256 ? 1 : 256 / PH;
        while (r > 1 && r * RS * 8 > 40 * 1024) r /= 2;
        return r;
    }
    static constexpr int ROWS = rows_fit();
    static constexpr int NT = ROWS * PH;
};

// r2c of the T*T x rows of a real volume (+ add), into the half spectrum
template <int T>
__global__ void __launch_bounds__(TRows<T>::NT) k_t_rows(const float* __restrict__ vol, float add, float2* spec,
                                                          Twiddles tw) {
    using R = TRows<T>;
    constexpr int H = R::H, PH = R::PH, V = R::V, RS = R::RS, HC = T / 2 + 1;
    __shared__ float2 sm[R::ROWS * RS];
    const int t = threadIdx.x % PH, rl = threadIdx.x / PH;
    const int row = blockIdx.x * R::ROWS + rl;
    const bool valid = row < T * T;
    const float* src = vol + (size_t)(valid ? row : 0) * T;
    float2 v[V];
#pragma unroll
    for (int r = 0; r < V; r++) {
        const int n = t + PH * r;
        v[r] = make_float2(src[2 * n] + add, src[2 * n + 1] + add);
    }
    float2* buf = sm + rl * RS;
    tmfft::fft<H, V, -1>(v, t, buf, tw, [] __device__() { __syncthreads(); });
    __syncthreads();
#pragma unroll
    for (int r = 0; r < V; r++) buf[tmfft::pad16(t + PH * r)] = v[r];
    __syncthreads();
    if (!valid) return;
    float2* out = spec + (size_t)row * HC;
#pragma unroll
    for (int r = 0; r < V; r++) {
        const int k = t + PH * r;
        const float2 zk = v[r];
        const float2 zm = buf[tmfft::pad16(k == 0 ? 0 : H - k)];
        const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
        const float2 wo = cmul(o, tw.template w<-1>(k, T));
        out[k] = make_float2(e.x + wo.x, e.y + wo.y);
        if (k == 0) out[H] = make_float2(e.x - o.x, e.y - o.y);
    }
}

// ----------------------------------------------------------------------------------------------
template <int T>
struct TCols {
    static constexpr int V = T % 3 == 0 ? 24 : 16;
    static constexpr int PT = T / V;
    static constexpr int RS = skewed(tmfft::padded_len(T), 1);
    static constexpr int CB = (16 * RS * 8 <= 40 * 1024) ? 16 : (8 * RS * 8 <= 40 * 1024) ? 8 : 4;
    static constexpr int NT = CB * PT;
};

// Complex FFT of T-point columns of the half spectrum: column c starts at
// (c / inner) * outer + c % inner, element k at start + k * stride.  With
// `last`, the z pass: scale 1/T^3, zeroed DC, quadrant swap.
template <int T>
__global__ void __launch_bounds__(TCols<T>::NT) k_t_cols(float2* spec, long long ncols, long long inner,
                                                          long long outer, long long stride, int last, Twiddles tw) {
    using C = TCols<T>;
    constexpr int V = C::V, PT = C::PT, CB = C::CB, RS = C::RS, HC = T / 2 + 1;
    __shared__ float2 sm[CB * RS];
    const int il = threadIdx.x % CB, tp = threadIdx.x / CB;
    const long long c = (long long)blockIdx.x * CB + il;
    const bool valid = c < ncols;
    const long long cc = valid ? c : 0;
    float2* col = spec + (cc / inner) * outer + cc % inner;
    float2 v[V];
#pragma unroll
    for (int r = 0; r < V; r++) v[r] = col[(size_t)(tp + PT * r) * stride];
    tmfft::fft<T, V, -1>(v, tp, sm + il * RS, tw, [] __device__() { __syncthreads(); });
    if (!valid) return;
    if (last) {
        // z pass: the column is (y, x) = (cc / HC, cc % HC), element r is z
        const int x = (int)(cc % HC), y = (int)(cc / HC);
        const double kPi = 3.14159265359;
        const float s = (float)(T / 2);
        const float px = (float)(s * (float)x * 2.0 * kPi / T);
        const float py = (float)(s * (float)logical(y, T) * 2.0 * kPi / T);
        const double inv = 1.0 / ((double)T * T * T);
#pragma unroll
        for (int r = 0; r < V; r++) {
            const int z = tp + PT * r;
            const float pz = (float)(s * (float)logical(z, T) * 2.0 * kPi / T);
            const float th = -px - py - pz;
            const double cs = cosf(th), sn = sinf(th);
            double re = (double)v[r].x * inv, im = (double)v[r].y * inv;
            if (x == 0 && y == 0 && z == 0) re = im = 0.0;
            v[r] = make_float2((float)(re * cs - im * sn), (float)(re * sn + im * cs));
        }
    }
#pragma unroll
    for (int r = 0; r < V; r++) col[(size_t)(tp + PT * r) * stride] = v[r];
}

}  // namespace tmt
