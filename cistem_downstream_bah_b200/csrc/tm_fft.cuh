// tm_fft.cuh -- register-resident Stockham FFT building blocks for sm_100a.
//
// An L-point complex transform is spread over P = L / R threads that each hold
// R values in registers.  On entry thread t holds x[t + P*r] (r = 0..R-1); on
// exit it holds X[t + P*r] (natural order, same stride).  Stages use radix R
// except the last, which may use a smaller radix RL (RL divides R); between
// stages the values go through a padded shared-memory buffer (Stockham
// autosort: stage s reads element b + r*L/Rs and writes (b/Ns)*Ns*Rs + b%Ns +
// r*Ns, with Ns the product of the earlier radices).
//
// Direction: DIR = -1 forward (exp(-2 pi i k n / L)), +1 inverse
// (unnormalised), matching the reference's FFTW conventions
// (src/core/image.cpp:5085-5113).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tmfft {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmul_conj(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// multiply by -i (DIR=-1) or +i (DIR=+1)
template <int DIR>
__device__ __forceinline__ float2 mul_i(float2 a) {
    return DIR < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

// padded shared-memory index: one spare float2 per 16
__device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded_len(int L) { return L + L / 16; }

// pad16(t + P*r) as a base plus a compile-time offset per r (0 <= t < P, P a
// multiple or a divisor of 16), so the 16 addresses need one register
template <int P>
__device__ __forceinline__ int rd_base(int t) { return (P % 16 == 0) ? t + (t >> 4) : t; }
template <int P>
__host__ __device__ constexpr int rd_off(int r) { return (P % 16 == 0) ? r * (P + P / 16) : P * r + ((P * r) >> 4); }

// pad16(idxD + r*Ns) for the Stockham write of a stage with one radix-R
// butterfly per thread (b = t): idxD = (t/Ns)*Ns*R + t%Ns; Ns == 1 or a multiple of 16
template <int R>
__device__ __forceinline__ int wr_base(int t, int Ns) {
    return Ns == 1 ? pad16(R * t) : pad16((t / Ns) * Ns * R + (t % Ns));
}
__host__ __device__ constexpr int wr_off(int r, int Ns) { return Ns == 1 ? r : r * (Ns + Ns / 16); }

template <int DIR>
__device__ __forceinline__ void dft2(float2& a, float2& b) {
    float2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int DIR>
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
    float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
    float2 s13 = cadd(a1, a3), d13 = mul_i<DIR>(csub(a1, a3));
    a0 = cadd(s02, s13);
    a2 = csub(s02, s13);
    a1 = cadd(d02, d13);
    a3 = csub(d02, d13);
}

// radix-8 in natural order: r = 2*r1 + r2, q = q1 + 4*q2
template <int DIR>
__device__ __forceinline__ void dft8(float2* v) {
    const float h = 0.70710678118654752440f;
    dft4<DIR>(v[0], v[2], v[4], v[6]);   // r2 = 0 -> q1 at v[0,2,4,6]
    dft4<DIR>(v[1], v[3], v[5], v[7]);   // r2 = 1 -> q1 at v[1,3,5,7]
    // twiddle W8^(q1 * r2) on r2 = 1
    v[3] = make_float2((v[3].x + (DIR < 0 ? v[3].y : -v[3].y)) * h, (v[3].y + (DIR < 0 ? -v[3].x : v[3].x)) * h);
    v[5] = mul_i<DIR>(v[5]);
    v[7] = make_float2((-v[7].x + (DIR < 0 ? v[7].y : -v[7].y)) * h, (-v[7].y + (DIR < 0 ? -v[7].x : v[7].x)) * h);
    float2 o[8];
#pragma unroll
    for (int q1 = 0; q1 < 4; q1++) {
        float2 a = v[2 * q1], b = v[2 * q1 + 1];
        o[q1] = cadd(a, b);
        o[q1 + 4] = csub(a, b);
    }
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = o[i];
}

// radix-16 in natural order: r = 4*r1 + r2, q = q1 + 4*q2
template <int DIR>
__device__ __forceinline__ void dft16(float2* v) {
#pragma unroll
    for (int r2 = 0; r2 < 4; r2++) dft4<DIR>(v[r2], v[4 + r2], v[8 + r2], v[12 + r2]);
    // v[r2 + 4*q1] now holds u_{r2}[q1]; twiddle by W16^(q1*r2)
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f, h = 0.70710678118654752440f;
    const float sg = DIR < 0 ? -1.f : 1.f;
    // (q1, r2) = (1,1): W^1, (1,2): W^2, (1,3): W^3, (2,1): W^2, (2,2): W^4, (2,3): W^6, (3,1): W^3, (3,2): W^6, (3,3): W^9
    const float2 w1 = make_float2(c1, sg * s1), w2 = make_float2(h, sg * h), w3 = make_float2(s1, sg * c1);
    const float2 w6 = make_float2(-h, sg * h), w9 = make_float2(-c1, -sg * s1);
    v[5] = cmul(v[5], w1);
    v[6] = cmul(v[6], w2);
    v[7] = cmul(v[7], w3);
    v[9] = cmul(v[9], w2);
    v[10] = mul_i<DIR>(v[10]);
    v[11] = cmul(v[11], w6);
    v[13] = cmul(v[13], w3);
    v[14] = cmul(v[14], w6);
    v[15] = cmul(v[15], w9);
    float2 o[16];
#pragma unroll
    for (int q1 = 0; q1 < 4; q1++) {
        float2 a0 = v[4 * q1], a1 = v[4 * q1 + 1], a2 = v[4 * q1 + 2], a3 = v[4 * q1 + 3];
        dft4<DIR>(a0, a1, a2, a3);
        o[q1] = a0;
        o[q1 + 4] = a1;
        o[q1 + 8] = a2;
        o[q1 + 12] = a3;
    }
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = o[i];
}

template <int RS, int DIR>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (RS == 16) dft16<DIR>(v);
    else if constexpr (RS == 8) dft8<DIR>(v);
    else if constexpr (RS == 4) dft4<DIR>(v[0], v[1], v[2], v[3]);
    else if constexpr (RS == 2) dft2<DIR>(v[0], v[1]);
}

// powers w^0 .. w^(n-1) by a shallow multiplication tree (depth <= 4)
template <int N>
__device__ __forceinline__ void powers(float2 w, float2* p) {
    p[0] = make_float2(1.f, 0.f);
    if constexpr (N > 1) p[1] = w;
    if constexpr (N > 2) p[2] = cmul(w, w);
    if constexpr (N > 3) p[3] = cmul(p[2], w);
    if constexpr (N > 4) {
        p[4] = cmul(p[2], p[2]);
#pragma unroll
        for (int i = 5; i < 8 && i < N; i++) p[i] = cmul(p[4], p[i - 4]);
    }
    if constexpr (N > 8) {
        p[8] = cmul(p[4], p[4]);
#pragma unroll
        for (int i = 9; i < 16 && i < N; i++) p[i] = cmul(p[8], p[i - 8]);
    }
}

// e[r] *= w^r for r = 1..RS-1.  The powers come from a shallow product tree
// (depth <= 4) computed next to their use, so few of them are live at once.
template <int RS>
__device__ __forceinline__ void apply_twiddles(float2* e, float2 w) {
    if constexpr (RS == 2) {
        e[1] = cmul(e[1], w);
    } else if constexpr (RS == 4) {
        const float2 w2 = cmul(w, w);
        e[1] = cmul(e[1], w);
        e[2] = cmul(e[2], w2);
        e[3] = cmul(e[3], cmul(w2, w));
    } else {
        const float2 w2 = cmul(w, w);
        const float2 w3 = cmul(w2, w);
        const float2 w4 = cmul(w2, w2);
        e[1] = cmul(e[1], w);
        e[2] = cmul(e[2], w2);
        e[3] = cmul(e[3], w3);
        e[4] = cmul(e[4], w4);
        e[5] = cmul(e[5], cmul(w4, w));
        e[6] = cmul(e[6], cmul(w4, w2));
        e[7] = cmul(e[7], cmul(w4, w3));
        if constexpr (RS == 16) {
            const float2 w8 = cmul(w4, w4);
            e[8] = cmul(e[8], w8);
            e[9] = cmul(e[9], cmul(w8, w));
            e[10] = cmul(e[10], cmul(w8, w2));
            e[11] = cmul(e[11], cmul(w8, w3));
            const float2 w12 = cmul(w8, w4);
            e[12] = cmul(e[12], w12);
            e[13] = cmul(e[13], cmul(w12, w));
            e[14] = cmul(e[14], cmul(w12, w2));
            e[15] = cmul(e[15], cmul(w12, w3));
        }
    }
}

// Twiddle source: a table of W_LMAX^m = exp(-2 pi i m / LMAX), m = 0..LMAX-1,
// for one power-of-two LMAX; W_L^m = table[m * (LMAX / L)].
struct Twiddles {
    const float2* __restrict__ tab;
    int lmax;
    template <int DIR>
    __device__ __forceinline__ float2 w(int m, int L) const {
        float2 t = __ldg(tab + (size_t)(m & (L - 1)) * (lmax / L));
        return DIR < 0 ? t : conjf2(t);
    }
};

// Number of stages and radix of stage s for L = R^k * RL.
template <int L, int R>
struct Plan {
    static constexpr int full = [] { int n = 0, m = L; while (m % R == 0 && m > 1) { m /= R; n++; } return n; }();
    static constexpr int RL = [] { int m = L; while (m % R == 0 && m > 1) m /= R; return m; }();
    static constexpr int stages = full + (RL > 1 ? 1 : 0);
    static constexpr int P = L / R;
    static_assert(RL == 1 || R % RL == 0, "last radix must divide R");
    __host__ __device__ static constexpr int radix(int s) { return s < full ? R : RL; }
};

// One cooperative FFT.  `sync` is a callable barrier over all threads that
// use `buf`.  buf has padded_len(L) float2 entries.  The caller must ensure no
// other thread still reads buf from a previous use before calling (the first
// exchange begins with a barrier).
template <int L, int R, int DIR, class Sync>
__device__ __forceinline__ void fft(float2 (&v)[R], int t, float2* buf, const Twiddles& tw, Sync sync) {
    using PL = Plan<L, R>;
    constexpr int P = PL::P;
    int Ns = 1;
#pragma unroll
    for (int s = 0; s < PL::stages; s++) {
        const int RS = PL::radix(s);
        const bool last = (s == PL::stages - 1);
        // twiddle base of this stage for the first butterfly, loaded before the
        // exchange so its latency hides behind the barrier and shared loads
        float2 w_first = make_float2(1.f, 0.f);
        if (s > 0) w_first = tw.template w<DIR>((t % Ns) * (L / (Ns * RS)), L);
        if (s > 0) {
            // load stage input: x[t + P*r]
            sync();
            const float2* rb = buf + rd_base<P>(t);
#pragma unroll
            for (int r = 0; r < R; r++) v[r] = rb[rd_off<P>(r)];
        }
        // butterflies: thread does R/RS of them, b = t + P*u, elements v[u + r*(R/RS)]
#pragma unroll
        for (int u = 0; u < R / (RS > 0 ? RS : 1); u++) {
            const int b = t + P * u;
            float2 e[16];
#pragma unroll
            for (int r = 0; r < RS; r++) e[r] = v[u + r * (R / RS)];
            if (s > 0) {
                const int jm = b % Ns;
                const float2 w = (u == 0) ? w_first : tw.template w<DIR>(jm * (L / (Ns * RS)), L);
                if (RS == 16) apply_twiddles<16>(e, w);
                else if (RS == 8) apply_twiddles<8>(e, w);
                else if (RS == 4) apply_twiddles<4>(e, w);
                else if (RS == 2) apply_twiddles<2>(e, w);
            }
            if (RS == 16) dft16<DIR>(e);
            else if (RS == 8) dft8<DIR>(e);
            else if (RS == 4) dft4<DIR>(e[0], e[1], e[2], e[3]);
            else if (RS == 2) dft2<DIR>(e[0], e[1]);
            if (last) {
#pragma unroll
                for (int r = 0; r < RS; r++) v[u + r * (R / RS)] = e[r];
            } else {
                if (u == 0) sync();  // previous readers of buf are done
                if (RS == R && (Ns == 1 || Ns % 16 == 0)) {
                    float2* wb = buf + wr_base<R>(b, Ns);
#pragma unroll
                    for (int r = 0; r < RS; r++) wb[wr_off(r, Ns)] = e[r];
                } else {
                    const int idxD = (b / Ns) * Ns * RS + (b % Ns);
#pragma unroll
                    for (int r = 0; r < RS; r++) buf[pad16(idxD + r * Ns)] = e[r];
                }
            }
        }
        Ns *= RS;
    }
}

// Same transform as fft(), with the exchanges done through a float buffer of
// padded_len(L) entries: real parts first, then imaginary parts.  Uses half
// the shared memory of fft() at the cost of two extra barriers per exchange.
template <int L, int R, int DIR, class Sync>
__device__ __forceinline__ void fft_split(float2 (&v)[R], int t, float* buf, const Twiddles& tw, Sync sync) {
    using PL = Plan<L, R>;
    constexpr int P = PL::P;
    int Ns = 1;
#pragma unroll
    for (int s = 0; s < PL::stages; s++) {
        const int RS = PL::radix(s);
        const bool last = (s == PL::stages - 1);
#pragma unroll
        for (int u = 0; u < R / (RS > 0 ? RS : 1); u++) {
            const int b = t + P * u;
            float2 e[16];
#pragma unroll
            for (int r = 0; r < RS; r++) e[r] = v[u + r * (R / RS)];
            if (s > 0) {
                const int jm = b % Ns;
                const float2 w = tw.template w<DIR>(jm * (L / (Ns * RS)), L);
                if (RS == 16) apply_twiddles<16>(e, w);
                else if (RS == 8) apply_twiddles<8>(e, w);
                else if (RS == 4) apply_twiddles<4>(e, w);
                else if (RS == 2) apply_twiddles<2>(e, w);
            }
            if (RS == 16) dft16<DIR>(e);
            else if (RS == 8) dft8<DIR>(e);
            else if (RS == 4) dft4<DIR>(e[0], e[1], e[2], e[3]);
            else if (RS == 2) dft2<DIR>(e[0], e[1]);
#pragma unroll
            for (int r = 0; r < RS; r++) v[u + r * (R / RS)] = e[r];
        }
        if (!last) {
            // the next stage reads x[t + P*r]; this stage wrote (b/Ns)*Ns*Rs + b%Ns + r*Ns
            // (non-last stages use RS == R, one butterfly per thread, b = t)
            float* wb = buf + wr_base<R>(t, Ns);
            const float* rb = buf + rd_base<P>(t);
            float nre[R];
            sync();
#pragma unroll
            for (int r = 0; r < R; r++) wb[wr_off(r, Ns)] = v[r].x;
            sync();
#pragma unroll
            for (int r = 0; r < R; r++) nre[r] = rb[rd_off<P>(r)];
            sync();
#pragma unroll
            for (int r = 0; r < R; r++) wb[wr_off(r, Ns)] = v[r].y;
            sync();
#pragma unroll
            for (int r = 0; r < R; r++) v[r] = make_float2(nre[r], rb[rd_off<P>(r)]);
        }
        Ns *= RS;
    }
}

}  // namespace tmfft
