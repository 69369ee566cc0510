// tm_generic.cuh -- run-time-length transforms for micrograph sizes without
// compiled kernels.
//
// The reference pads a micrograph side to the nearest size whose prime factors
// are small (match_template.cpp:527-575 with ReturnClosestFactorizedUpper,
// functions.cpp:529-577: largest factor 2, then 3, 5, 7, 9, 13, each within
// 10 % growth and a multiple of 4), so a side can carry the primes 2, 3, 5, 7,
// 11 and 13.  The compiled kernels cover the power-of-two widths and the
// 2^a 3^b heights of the common camera formats; every other padded size runs
// on the kernels here, whose FFT lengths are arguments:
//
//   fft_gen        a Stockham transform of a line of length L held in shared
//                  memory (two buffers, ping-pong), radix plan (16, 8, 4, 2,
//                  9, 3, 5, 7, 11, 13) chosen on the host
//   k_pass_a_gen   forward FFT along x of each normalised projection row
//   k_pass_b_gen   per column: forward FFT along y, conjugate multiply with
//                  I', inverse FFT along y
//   k_pass_c_gen   per row: the c2r packing, inverse X/2-point FFT and the
//                  MIP / argmax / compensated sums / histogram update
//   k_w_rows_gen,  the whitening's row r2c and column FFT (with the quadrant
//   k_w_cols_gen   swap and zeroed central pixel)
//
// The arithmetic is the compiled path's (FP32, the same packing, twiddle
// tables and epilogue); only the FFT organisation differs.  Lines up to
// kGenMaxLen = 8192 points.
#pragma once
#include "tm_fft.cuh"
#include "tm_whiten.cuh"

namespace tmk {

constexpr int kGenMaxStages = 24;
constexpr int kGenNT = 512;
constexpr int kGenMaxLen = 8192;

struct GenPlan {
    int L;                    // transform length
    int n;                    // stages
    int r[kGenMaxStages];     // radices, product L
};

// Radix plan of L; false when L has a prime factor above 13 or is too long.
inline bool gen_plan(int L, GenPlan& p) {
    p.L = L;
    p.n = 0;
    if (L < 2 || L > kGenMaxLen) return false;
    int m = L;
    const int order[] = {16, 8, 4, 2, 9, 3, 5, 7, 11, 13};
    for (int r : order)
        while (m % r == 0 && p.n < kGenMaxStages) {
            p.r[p.n++] = r;
            m /= r;
        }
    return m == 1;
}

// R-point DFT of prime length as R^2 multiplications by compile-time constants
template <int R, int DIR>
__device__ __forceinline__ void dft_naive(float2* e) {
    float2 o[R];
    tmfft::sfor<R>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        float2 acc = e[0];
        tmfft::sfor<R - 1>([&](auto ic) {
            constexpr int i = decltype(ic)::value + 1;
            acc = tmfft::cadd(acc, tmfft::twc<R, (i * k) % R, DIR>(e[i]));
        });
        o[k] = acc;
    });
#pragma unroll
    for (int i = 0; i < R; i++) e[i] = o[i];
}

template <int R, int DIR>
__device__ __forceinline__ void dft_any(float2* e) {
    if constexpr (R == 5 || R == 7 || R == 11 || R == 13) dft_naive<R, DIR>(e);
    else tmfft::dft<R, DIR>(e);
}

// One Stockham stage of radix R over `lines` lines (line stride `stride`), from
// `in` to `out`: butterfly b reads elements b + i L/R, twiddles them by
// W_{Ns R}^{(b mod Ns) i} and writes (b / Ns) Ns R + b mod Ns + i Ns -- the
// pattern of tmfft::fft.
template <int R, int DIR>
__device__ __forceinline__ void gen_stage(const float2* in, float2* out, int stride, int lines, int L, int Ns,
                                          const tmfft::Twiddles& tw) {
    const int nbf = L / R, total = lines * nbf;
    for (int g = threadIdx.x; g < total; g += kGenNT) {
        const int line = g / nbf, b = g - line * nbf;
        const float2* src = in + (size_t)line * stride;
        float2* dst = out + (size_t)line * stride;
        const int jm = b % Ns;
        const float2 w = tw.template w<DIR>(jm * (L / (Ns * R)), L);
        float2 e[R];
#pragma unroll
        for (int i = 0; i < R; i++) e[i] = src[b + i * nbf];
        float2 wp = w;
#pragma unroll
        for (int i = 1; i < R; i++) {
            e[i] = tmfft::cmul(e[i], wp);
            wp = tmfft::cmul(wp, w);
        }
        dft_any<R, DIR>(e);
        const int base = (b / Ns) * Ns * R + jm;
#pragma unroll
        for (int i = 0; i < R; i++) dst[base + i * Ns] = e[i];
    }
    __syncthreads();
}

// Transform of `lines` lines held in shared memory, ping-ponging between buf
// and tmp (both lines x stride); returns the buffer that holds the result.  The
// caller has passed a barrier since buf was filled.  DIR = -1 forward, +1
// inverse, unnormalised.  The twiddle table's length is a multiple of L.
template <int DIR>
__device__ float2* fft_gen(float2* buf, float2* tmp, int stride, int lines, const GenPlan& p, const tmfft::Twiddles& tw) {
    int Ns = 1;
    float2 *in = buf, *out = tmp;
    for (int s = 0; s < p.n; s++) {
        const int R = p.r[s];
        switch (R) {
            case 16: gen_stage<16, DIR>(in, out, stride, lines, p.L, Ns, tw); break;
            case 8: gen_stage<8, DIR>(in, out, stride, lines, p.L, Ns, tw); break;
            case 4: gen_stage<4, DIR>(in, out, stride, lines, p.L, Ns, tw); break;
            case 2: gen_stage<2, DIR>(in, out, stride, lines, p.L, Ns, tw); break;
            case 9: gen_stage<9, DIR>(in, out, stride, lines, p.L, Ns, tw); break;
            case 3: gen_stage<3, DIR>(in, out, stride, lines, p.L, Ns, tw); break;
            case 5: gen_stage<5, DIR>(in, out, stride, lines, p.L, Ns, tw); break;
            case 7: gen_stage<7, DIR>(in, out, stride, lines, p.L, Ns, tw); break;
            case 11: gen_stage<11, DIR>(in, out, stride, lines, p.L, Ns, tw); break;
            default: gen_stage<13, DIR>(in, out, stride, lines, p.L, Ns, tw); break;
        }
        Ns *= R;
        float2* sw = in;
        in = out;
        out = sw;
    }
    return in;
}

// ---------------------------------------------------------------------------------------
// k_pass_a_gen: block per (row, orientation); the T normalised samples at the
// start of an X-point line, forward FFT, kx = 0 .. X/2 into A.
template <int T>
__global__ void __launch_bounds__(kGenNT) k_pass_a_gen(BatchArgs a, int X, GenPlan px) {
    extern __shared__ float2 gbuf[];   // 2 x X
    const int row = blockIdx.x, o = blockIdx.y;
    const float2 nrm = a.norm[o];
    const float* prow = a.P + ((size_t)o * T + row) * T;
    for (int i = threadIdx.x; i < X; i += kGenNT)
        gbuf[i] = make_float2(i < T ? (prow[i] - nrm.x) * nrm.y : 0.f, 0.f);
    __syncthreads();
    const float2* f = fft_gen<-1>(gbuf, gbuf + X, X, 1, px, a.tw);
    float2* out = a.A + ((size_t)o * T + row) * a.XP;
    for (int k = threadIdx.x; k <= X / 2; k += kGenNT) out[k] = f[k];
}

// k_pass_b_gen: block per (group of LW adjacent columns, orientation), the LW
// columns transformed together (LW lines per Stockham stage, so that a stage
// has LW times the butterflies for the block's threads) and written as whole
// row segments (LW = 4: 32-byte sectors).  Streaming stores, as the compiled
// column passes.
template <int LW>
__global__ void __launch_bounds__(kGenNT) k_pass_b_gen(BatchArgs a, int T, int Y, GenPlan py) {
    extern __shared__ float2 gbuf[];   // 2 x LW x Y, line c at c * Y
    const int kx0 = blockIdx.x * LW, o = blockIdx.y;
    const int XP = a.XP;
    const float2* Ao = a.A + (size_t)o * T * XP + kx0;
    for (int e = threadIdx.x; e < LW * Y; e += kGenNT) {
        const int n = e / LW, c = e - n * LW;
        gbuf[c * Y + n] = n < T ? Ao[(size_t)n * XP + c] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* f = fft_gen<-1>(gbuf, gbuf + LW * Y, Y, LW, py, a.twy);
    for (int e = threadIdx.x; e < LW * Y; e += kGenNT) {
        const int k = e / LW, c = e - k * LW;
        f[c * Y + k] = cmul_conj(__ldg(a.Ip + (size_t)k * XP + kx0 + c), f[c * Y + k]);
    }
    __syncthreads();
    const float2* z = fft_gen<+1>(f, f == gbuf ? gbuf + LW * Y : gbuf, Y, LW, py, a.twy);
    float2* Co = a.C + (size_t)o * Y * XP + kx0;
    for (int e = threadIdx.x; e < LW * Y; e += kGenNT) {
        const int yy = e / LW, c = e - yy * LW;
        __stcs(Co + (size_t)yy * XP + c, z[c * Y + yy]);
    }
}
// columns per block of k_pass_b_gen for a height Y (two buffers of LW x Y in shared memory)
inline int gen_pass_b_lines(int Y) {
    if (2 * 4 * (size_t)Y * sizeof(float2) <= 232448) return 4;
    if (2 * 2 * (size_t)Y * sizeof(float2) <= 232448) return 2;
    return 1;
}

// k_pass_c_gen: block per row y; thread t owns the pixels x = t + kGenNT j and
// keeps their state in registers over the batch, as k_pass_c does.  An even
// width uses the c2r packing of k_pass_c (an X/2-point inverse FFT whose
// outputs hold pixel pairs); an odd width (the reference's factorisation can
// give one, e.g. 3^8) the full X-point inverse of the Hermitian extension,
// the imaginary part of the DC term ignored as FFTW's c2r does.
// MAXP pixels per thread (kGenNT * MAXP >= X): 4, 8 or 16, the smaller the
// fewer registers and the more blocks per SM.
template <bool ODD, int MAXP>
__global__ void __launch_bounds__(kGenNT, MAXP == 4 ? 3 : MAXP == 8 ? 2 : 1)
k_pass_c_gen(BatchArgs a, int X, int Y, GenPlan ph) {
    static_assert(kGenNT * 16 >= kGenMaxLen, "16 pixels per thread cover the longest rows");
    extern __shared__ float2 gbuf[];             // 2 x L (L = X/2 or X), then the histogram
    const int L = ODD ? X : X / 2, HC = X / 2 + 1, XP = a.XP, y = blockIdx.x, t = threadIdx.x;
    unsigned int* shist = reinterpret_cast<unsigned int*>(gbuf + 2 * L);
    for (int b = t; b < a.hist_bins; b += kGenNT) shist[b] = 0u;
    float mip[MAXP], fs[MAXP], fq[MAXP], cs[MAXP], cq[MAXP];
    int best[MAXP];
    const size_t rowoff = (size_t)y * X;
#pragma unroll
    for (int j = 0; j < MAXP; j++) {
        const int x = t + kGenNT * j;
        if (x < X) {
            mip[j] = a.mip[rowoff + x];
            best[j] = a.best[rowoff + x];
        }
        fs[j] = fq[j] = cs[j] = cq[j] = 0.f;
    }
    for (int o = 0; o < a.nb; o++) {
        const float2* row = a.C + ((size_t)o * Y + y) * XP;
        if constexpr (ODD) {
            for (int k = t; k < X; k += kGenNT) {
                float2 v = k < HC ? __ldg(row + k) : tmfft::conjf2(__ldg(row + (X - k)));
                if (k == 0) v.y = 0.f;
                gbuf[k] = v;
            }
        } else {
            const int H = L;
            for (int k = t; k < H; k += kGenNT) {
                float2 hk = __ldg(row + k);
                float2 hm = __ldg(row + H - k);
                if (k == 0) { hk.y = 0.f; hm.y = 0.f; }
                const float2 e = make_float2(hk.x + hm.x, hk.y - hm.y);
                const float2 d = make_float2(hk.x - hm.x, hk.y + hm.y);
                const float2 od = cmul(d, a.tw.template w<+1>(k, X));
                gbuf[k] = make_float2(e.x - od.y, e.y + od.x);
            }
        }
        __syncthreads();
        const float2* zb = fft_gen<+1>(gbuf, gbuf + L, L, 1, ph, a.tw);
        const int g = (int)(a.gidx0 + o);
#pragma unroll
        for (int j = 0; j < MAXP; j++) {
            const int x = t + kGenNT * j;
            if (x < X) {
                float val;
                if constexpr (ODD) val = zb[x].x;
                else val = (x & 1) ? zb[x >> 1].y : zb[x >> 1].x;
                if (val > mip[j]) { mip[j] = val; best[j] = g; }
                const float ys = val - cs[j];
                const float ts = fs[j] + ys;
                cs[j] = (ts - fs[j]) - ys;
                fs[j] = ts;
                const float yq = fmaf(val, val, -cq[j]);
                const float tq = fq[j] + yq;
                cq[j] = (tq - fq[j]) - yq;
                fq[j] = tq;
                const int bin = __float2int_rz((val - a.hist_min) * a.hist_inv_step);
                if (bin >= 0 && bin < a.hist_bins) atomicAdd(&shist[bin], 1u);
            }
        }
        __syncthreads();   // every output is read before the next orientation's row
    }
#pragma unroll
    for (int j = 0; j < MAXP; j++) {
        const int x = t + kGenNT * j;
        if (x < X) {
            a.mip[rowoff + x] = mip[j];
            a.best[rowoff + x] = best[j];
            a.sum[rowoff + x] += (double)fs[j] - (double)cs[j];
            a.sumsq[rowoff + x] += (double)fq[j] - (double)cq[j];
        }
    }
    __syncthreads();
    for (int b = t; b < a.hist_bins; b += kGenNT) {
        const unsigned int cnt = shist[b];
        if (cnt) atomicAdd(a.hist + b, (unsigned long long)cnt);
    }
}

// ---------------------------------------------------------------------------------------
// Whitening transforms of any size (the steps of tmw::k_w_rows / k_w_cols).
template <bool ODD>
__global__ void __launch_bounds__(kGenNT) k_w_rows_gen(const float* __restrict__ img, float2* spec, int X, float mean,
                                                       float vmin, float vmax, tmfft::Twiddles tw, GenPlan ph) {
    extern __shared__ float2 gbuf[];   // 2 x L (L = X/2, or X when X is odd)
    const int HC = X / 2 + 1, y = blockIdx.x;
    const float* src = img + (size_t)y * X;
    float2* row = spec + (size_t)y * HC;
    auto clean = [&](float v) { return (v > vmax || v < vmin) ? mean : v; };
    if constexpr (ODD) {
        // an odd width: the full X-point transform of the real row
        for (int x = threadIdx.x; x < X; x += kGenNT) gbuf[x] = make_float2(clean(src[x]), 0.f);
        __syncthreads();
        const float2* zb = fft_gen<-1>(gbuf, gbuf + X, X, 1, ph, tw);
        for (int k = threadIdx.x; k < HC; k += kGenNT) row[k] = zb[k];
    } else {
        const int H = X / 2;
        for (int n = threadIdx.x; n < H; n += kGenNT) gbuf[n] = make_float2(clean(src[2 * n]), clean(src[2 * n + 1]));
        __syncthreads();
        const float2* zb = fft_gen<-1>(gbuf, gbuf + H, H, 1, ph, tw);
        for (int k = threadIdx.x; k < H; k += kGenNT) {
            const float2 zk = zb[k];
            const float2 zm = zb[k == 0 ? 0 : H - k];
            const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
            const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
            const float2 wo = cmul(o, tw.template w<-1>(k, X));
            row[k] = make_float2(e.x + wo.x, e.y + wo.y);
            if (k == 0) row[H] = make_float2(e.x - o.x, e.y - o.y);
        }
    }
}

__global__ void __launch_bounds__(kGenNT) k_w_cols_gen(float2* spec, int X, int Y, tmfft::Twiddles tw, GenPlan py) {
    extern __shared__ float2 gbuf[];   // 2 x Y: one column
    const int HC = X / 2 + 1, col = blockIdx.x;
    for (int yy = threadIdx.x; yy < Y; yy += kGenNT) gbuf[yy] = spec[(size_t)yy * HC + col];
    __syncthreads();
    const float2* f = fft_gen<-1>(gbuf, gbuf + Y, Y, 1, py, tw);
    // SwapRealSpaceQuadrants as a float phase (Image::PhaseShift, image.cpp:9221-9265), zeroed DC
    const double kPi = 3.14159265359;
    const float sx = (float)(X / 2), sy = (float)(Y / 2);
    const float px = (float)(sx * (float)col * 2.0 * kPi / X);
    for (int yy = threadIdx.x; yy < Y; yy += kGenNT) {
        const float py_ = (float)(sy * (float)tmw::logical(yy, Y) * 2.0 * kPi / Y);
        const float th = -px - py_;
        const float cth = cosf(th), sth = sinf(th);
        float2 v = f[yy];
        v = make_float2(v.x * cth - v.y * sth, v.x * sth + v.y * cth);
        if (col == 0 && yy == 0) v = make_float2(0.f, 0.f);
        spec[(size_t)yy * HC + col] = v;
    }
}

}  // namespace tmk
