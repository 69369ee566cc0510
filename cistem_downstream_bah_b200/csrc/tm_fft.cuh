// tm_fft.cuh -- register-resident Stockham FFT building blocks for sm_100a.
//
// An L-point complex transform is spread over P = L / R threads that each hold
// R values in registers.  On entry thread t holds x[t + P*r] (r = 0..R-1); on
// exit it holds X[t + P*r] (natural order, same stride).  Stages use radix R
// while R divides what is left of L, then the largest divisors of R that do
// (a thread then does R/Rs butterflies of radix Rs); between stages the values
// go through a padded shared-memory buffer (Stockham autosort: stage s reads
// element b + r*L/Rs and writes (b/Ns)*Ns*Rs + b%Ns + r*Ns, with Ns the
// product of the earlier radices).  Radices 2, 3, 4, 6, 8, 9, 12, 16, 18 and
// 24 are available, which covers the 2^a 3^b sizes the micrograph
// factorisation produces (match_template.cpp:527-583).
//
// Direction: DIR = -1 forward (exp(-2 pi i k n / L)), +1 inverse
// (unnormalised), matching the reference's FFTW conventions
// (src/core/image.cpp:5085-5113).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

namespace tmfft {

// compile-time loop: f(std::integral_constant<int, i>) for i = 0..N-1
template <class F, int... Is>
__device__ __forceinline__ void sfor_impl(F&& f, std::integer_sequence<int, Is...>) {
    (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void sfor(F&& f) {
    sfor_impl(f, std::make_integer_sequence<int, N>{});
}

// exp(2 pi i k / n) evaluated at compile time (Taylor series after reducing
// the angle to [-pi, pi]); used for the constants inside the small DFTs
__host__ __device__ constexpr double ct_angle(int k, int n) {
    int m = ((k % n) + n) % n;
    if (2 * m > n) m -= n;
    return 2.0 * 3.14159265358979323846 * (double)m / (double)n;
}
__host__ __device__ constexpr double ct_sin(double x) {
    double term = x, sum = x;
    for (int i = 1; i < 30; i++) {
        term *= -x * x / ((2.0 * i) * (2.0 * i + 1.0));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double ct_cos(double x) {
    double term = 1.0, sum = 1.0;
    for (int i = 1; i < 30; i++) {
        term *= -x * x / ((2.0 * i - 1.0) * (2.0 * i));
        sum += term;
    }
    return sum;
}

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
// butterfly per thread (b = t): idxD = (t/Ns)*Ns*R + t%Ns; valid for Ns == 1
// with R dividing 16, and for Ns a multiple of 16
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

template <int DIR>
__device__ __forceinline__ void dft3(float2& a, float2& b, float2& c) {
    // X1,2 = a - (b+c)/2 +- DIR i (sqrt(3)/2) (b-c)
    constexpr float h = 0.86602540378443864676f;
    const float2 sm = cadd(b, c), df = csub(b, c);
    const float2 m = make_float2(fmaf(-0.5f, sm.x, a.x), fmaf(-0.5f, sm.y, a.y));
    const float2 r = mul_i<DIR>(make_float2(h * df.x, h * df.y));
    a = cadd(a, sm);
    b = cadd(m, r);
    c = csub(m, r);
}

// x * W_R^K with W_R = exp(DIR 2 pi i / R), K a compile-time constant
template <int R, int K, int DIR>
__device__ __forceinline__ float2 twc(float2 x) {
    constexpr int k = ((K % R) + R) % R;
    if constexpr (k == 0) return x;
    else if constexpr (4 * k == R) return mul_i<DIR>(x);
    else if constexpr (2 * k == R) return make_float2(-x.x, -x.y);
    else if constexpr (4 * k == 3 * R) return mul_i<-DIR>(x);
    else {
        constexpr float c = (float)ct_cos(ct_angle(k, R));
        constexpr float sn = (float)(DIR * ct_sin(ct_angle(k, R)));
        return cmul(x, make_float2(c, sn));
    }
}

template <int RS, int DIR>
__device__ __forceinline__ void dft(float2* v);

// R1*R2-point DFT in natural order: r = R2*r1 + r2, q = q1 + R1*q2
// (R2 inner transforms of length R1, twiddles W_R^(r2 q1), R1 of length R2)
template <int R1, int R2, int DIR>
__device__ __forceinline__ void dft_pq(float2* v) {
    constexpr int R = R1 * R2;
    float2 u[R];
    sfor<R2>([&](auto r2c) {
        constexpr int r2 = decltype(r2c)::value;
        float2 t[R1];
#pragma unroll
        for (int r1 = 0; r1 < R1; r1++) t[r1] = v[R2 * r1 + r2];
        dft<R1, DIR>(t);
        sfor<R1>([&](auto q1c) {
            constexpr int q1 = decltype(q1c)::value;
            u[r2 * R1 + q1] = twc<R, r2 * q1, DIR>(t[q1]);
        });
    });
#pragma unroll
    for (int q1 = 0; q1 < R1; q1++) {
        float2 t[R2];
#pragma unroll
        for (int r2 = 0; r2 < R2; r2++) t[r2] = u[r2 * R1 + q1];
        dft<R2, DIR>(t);
#pragma unroll
        for (int q2 = 0; q2 < R2; q2++) v[q1 + R1 * q2] = t[q2];
    }
}

template <int RS, int DIR>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (RS == 16) dft16<DIR>(v);
    else if constexpr (RS == 8) dft8<DIR>(v);
    else if constexpr (RS == 4) dft4<DIR>(v[0], v[1], v[2], v[3]);
    else if constexpr (RS == 2) dft2<DIR>(v[0], v[1]);
    else if constexpr (RS == 3) dft3<DIR>(v[0], v[1], v[2]);
    else if constexpr (RS == 6) dft_pq<3, 2, DIR>(v);
    else if constexpr (RS == 9) dft_pq<3, 3, DIR>(v);
    else if constexpr (RS == 12) dft_pq<4, 3, DIR>(v);
    else if constexpr (RS == 18) dft_pq<9, 2, DIR>(v);
    else if constexpr (RS == 24) dft_pq<8, 3, DIR>(v);
    else static_assert(RS == 1, "unsupported radix");
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
    if constexpr (RS != 2 && RS != 4 && RS != 8 && RS != 16) {
        // w^k by a product tree of depth log2(RS)
        float2 p[RS];
        p[1] = w;
#pragma unroll
        for (int k = 2; k < RS; k++) p[k] = cmul(p[k >> 1], p[k - (k >> 1)]);
#pragma unroll
        for (int k = 1; k < RS; k++) e[k] = cmul(e[k], p[k]);
    } else if constexpr (RS == 2) {
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

// Twiddle source: a table of W_LMAX^m = exp(-2 pi i m / LMAX), m = 0..LMAX-1;
// W_L^m = table[(m mod L) * (LMAX / L)] for every L that divides LMAX.
struct Twiddles {
    const float2* __restrict__ tab;
    int lmax;
    template <int DIR>
    __device__ __forceinline__ float2 w(int m, int L) const {
        const int mm = (L & (L - 1)) == 0 ? (m & (L - 1)) : (m % L);
        float2 t = __ldg(tab + (size_t)mm * (lmax / L));
        return DIR < 0 ? t : conjf2(t);
    }
};

// Radix plan of an L-point transform with R values per thread: R while R
// divides what is left, then the largest divisors of R that divide the rest.
// Butterflies are at most radix 24: with R = 32 every stage is a divisor
// (16, ...) and a thread does R / radix butterflies per stage.
constexpr int kMaxRadix = 24;
struct RadixSeq {
    int n;        // stages, -1 if L cannot be split this way
    int r[24];
};
__host__ __device__ constexpr RadixSeq radix_seq(int L, int R) {
    RadixSeq q{0, {}};
    int m = L;
    while (R <= kMaxRadix && m > 1 && m % R == 0 && q.n < 24) {
        q.r[q.n++] = R;
        m /= R;
    }
    while (m > 1) {
        int d = R > kMaxRadix ? kMaxRadix : R;
        while (d > 1 && !(R % d == 0 && m % d == 0)) d--;
        if (d <= 1 || q.n >= 24) return RadixSeq{-1, {}};
        q.r[q.n++] = d;
        m /= d;
    }
    return q;
}
__host__ __device__ constexpr bool plannable(int L, int R) { return L % R == 0 && radix_seq(L, R).n > 0; }

template <int L, int R>
struct Plan {
    static constexpr RadixSeq seq = radix_seq(L, R);
    static_assert(L % R == 0 && seq.n > 0, "transform length cannot be planned with this radix");
    static constexpr int stages = seq.n;
    static constexpr int P = L / R;
    __host__ __device__ static constexpr int radix(int s) { return seq.r[s]; }
    // product of the radices of the stages before s
    __host__ __device__ static constexpr int ns(int s) {
        int n = 1;
        for (int i = 0; i < s; i++) n *= seq.r[i];
        return n;
    }
};

// One cooperative FFT.  `sync` is a callable barrier over all threads that
// use `buf`.  buf has padded_len(L) float2 entries.  The first exchange begins
// with a barrier so that no thread still reads buf from a previous use; a
// caller whose threads have all passed a barrier since buf was last read
// passes FIRST_SYNC = false to skip it.
template <int L, int R, int DIR, bool FIRST_SYNC = true, class Sync>
__device__ __forceinline__ void fft(float2 (&v)[R], int t, float2* buf, const Twiddles& tw, Sync sync) {
    using PL = Plan<L, R>;
    constexpr int P = PL::P;
    sfor<PL::stages>([&](auto sc) {
        constexpr int s = decltype(sc)::value;
        constexpr int RS = PL::radix(s);
        constexpr int Ns = PL::ns(s);
        constexpr bool last = (s == PL::stages - 1);
        // twiddle base of this stage for the first butterfly, loaded before the
        // exchange so its latency hides behind the barrier and shared loads
        float2 w_first = make_float2(1.f, 0.f);
        if constexpr (s > 0) w_first = tw.template w<DIR>((t % Ns) * (L / (Ns * RS)), L);
        if constexpr (s > 0) {
            // load stage input: x[t + P*r]
            sync();
            if constexpr (P % 16 == 0 || 16 % P == 0) {
                const float2* rb = buf + rd_base<P>(t);
#pragma unroll
                for (int r = 0; r < R; r++) v[r] = rb[rd_off<P>(r)];
            } else {
#pragma unroll
                for (int r = 0; r < R; r++) v[r] = buf[pad16(t + P * r)];
            }
        }
        // butterflies: thread does R/RS of them, b = t + P*u, elements v[u + r*(R/RS)]
#pragma unroll
        for (int u = 0; u < R / RS; u++) {
            const int b = t + P * u;
            float2 e[RS];
#pragma unroll
            for (int r = 0; r < RS; r++) e[r] = v[u + r * (R / RS)];
            if constexpr (s > 0) {
                const int jm = b % Ns;
                const float2 w = (u == 0) ? w_first : tw.template w<DIR>(jm * (L / (Ns * RS)), L);
                apply_twiddles<RS>(e, w);
            }
            dft<RS, DIR>(e);
            if constexpr (last) {
#pragma unroll
                for (int r = 0; r < RS; r++) v[u + r * (R / RS)] = e[r];
            } else {
                if (u == 0 && (FIRST_SYNC || s > 0)) sync();  // previous readers of buf are done
                // base + compile-time offsets equal pad16(idxD + r*Ns) when no
                // 16-element boundary falls inside a butterfly (Ns == 1, R | 16)
                // or every stride is a whole number of 16-blocks (16 | Ns)
                if constexpr (RS == R && ((Ns == 1 && 16 % R == 0) || Ns % 16 == 0)) {
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
    });
}

// The same transform with the twiddle multipliers of every stage supplied by
// the caller instead of a table lookup and a power tree:
// src.template issue<s>() starts fetching stage s's multipliers and is called
// before the stage's barrier, so that the fetch overlaps the barrier and the
// shared-memory loads; src.template get<s>(u, p) then fills p[1 .. RS-1] with
// w^1 .. w^(RS-1) of the thread's butterfly u (w as in fft above, DIR applied).
// Used where the multipliers are per-thread constants held in tensor memory.
template <int L, int R, int DIR, bool FIRST_SYNC = true, class Src, class Sync>
__device__ __forceinline__ void fft_pre(float2 (&v)[R], int t, float2* buf, Src& src, Sync sync) {
    using PL = Plan<L, R>;
    constexpr int P = PL::P;
    sfor<PL::stages>([&](auto sc) {
        constexpr int s = decltype(sc)::value;
        constexpr int RS = PL::radix(s);
        constexpr int Ns = PL::ns(s);
        constexpr bool last = (s == PL::stages - 1);
        if constexpr (s > 0) {
            src.template issue<s>();
            sync();
            if constexpr (P % 16 == 0 || 16 % P == 0) {
                const float2* rb = buf + rd_base<P>(t);
#pragma unroll
                for (int r = 0; r < R; r++) v[r] = rb[rd_off<P>(r)];
            } else {
#pragma unroll
                for (int r = 0; r < R; r++) v[r] = buf[pad16(t + P * r)];
            }
        }
#pragma unroll
        for (int u = 0; u < R / RS; u++) {
            const int b = t + P * u;
            float2 e[RS];
#pragma unroll
            for (int r = 0; r < RS; r++) e[r] = v[u + r * (R / RS)];
            if constexpr (s > 0) {
                float2 pw[RS];
                src.template get<s>(u, pw);
#pragma unroll
                for (int r = 1; r < RS; r++) e[r] = cmul(e[r], pw[r]);
            }
            dft<RS, DIR>(e);
            if constexpr (last) {
#pragma unroll
                for (int r = 0; r < RS; r++) v[u + r * (R / RS)] = e[r];
            } else {
                if (u == 0 && (FIRST_SYNC || s > 0)) sync();
                if constexpr (RS == R && ((Ns == 1 && 16 % R == 0) || Ns % 16 == 0)) {
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
    });
}

}  // namespace tmfft
