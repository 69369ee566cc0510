// prep.cpp -- host-side preparation of the search inputs (see prep.hpp).
#include "prep.hpp"

#include <cfloat>
#include <cmath>

#include "host_fft.hpp"

namespace tmhost {

namespace {
constexpr double kPi = 3.14159265359;       // the reference's PI (src/core/defines.h:6)
constexpr float kPif = 3.14159265359f;      // PIf (defines.h:7)

float deg2rad(float d) { return (float)((double)(d * kPif) / 180.); }
int logical(int phys, int n) { return phys >= (n % 2 == 0 ? n / 2 : n / 2 + 1) ? phys - n : phys; }

struct Curve {
    std::vector<float> x;
    std::vector<double> y;
    Curve(float lo, float hi, int n) : x(n), y(n, 0.0) {
        for (int i = 0; i < n; i++) x[i] = i * (hi - lo) / (float)(n - 1) + lo;
    }
    // Curve::ReturnLinearInterpolationFromX (curve.cpp:377-397)
    double at(float f) const {
        const int n = (int)x.size();
        int i = n - 1;
        for (int k = 0; k < n - 1; k++)
            if (f >= x[k] && f < x[k + 1]) { i = k; break; }
        if (f < x[0]) i = 0;
        if (i == n - 1) return y[n - 1];
        const float d = (f - x[i]) / (x[i + 1] - x[i]);
        return y[i] * (1.0 - d) + y[i + 1] * (double)d;
    }
    // AddValueAtXUsingLinearInterpolation with a linear axis (curve.cpp:500-560)
    void add(float f, double v) {
        const int n = (int)x.size();
        int i = (x[0] == x[1]) ? n - 2 : (int)((f - x[0]) / (x[1] - x[0]));
        if (i == n - 1) { y[i] += v; return; }
        const float d = (f - x[i]) / (x[i + 1] - x[i]);
        y[i] += v * (1.0 - d);
        y[i + 1] += v * (double)d;
    }
};

int curve_points(int nx) { return (int)((nx / 2.0 + 1.0) * sqrtf(2.0f) + 1.0); }

bool small_factors(int n, int largest) {
    for (int f = 2; f <= largest && n != 1; f++)
        while (n % f == 0) n /= f;
    return n == 1;
}

// Image::SwapRealSpaceQuadrants for an object centred in the box: a phase
// shift by (nx/2, ny/2, nz/2), with the phase formed in float and cosf/sinf
// as Image::PhaseShift does it (image.cpp:9221-9265, 9757-9824).
void swap_quadrants_centred(int nx, int ny, int nz, cplx* spec) {
    const int hc = nx / 2 + 1;
    const float sx = (float)(nx / 2), sy = (float)(ny / 2), sz = nz > 1 ? (float)(nz / 2) : 0.0f;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++) {
        const float pz = (float)(sz * (float)logical(k, nz) * 2.0 * kPi / nz);
        for (int j = 0; j < ny; j++) {
            const float py = (float)(sy * (float)logical(j, ny) * 2.0 * kPi / ny);
            cplx* row = spec + ((size_t)k * ny + j) * hc;
            for (int i = 0; i < hc; i++) {
                const float px = (float)(sx * (float)i * 2.0 * kPi / nx);
                const float t = -px - py - pz;
                const double c = cosf(t), s = sinf(t);
                const double re = row[i].real(), im = row[i].imag();
                row[i] = cplx(re * c - im * s, re * s + im * c);
            }
        }
    }
}

// centre-aligned real-space copy of an n^3 volume into m^3 (Image::ClipInto, image.cpp:8554-8590)
std::vector<double> clip3(const std::vector<double>& in, int n, int m, double pad) {
    std::vector<double> out((size_t)m * m * m);
    for (int kk = 0; kk < m; kk++) {
        const int k = n / 2 + (kk - m / 2);
        for (int jj = 0; jj < m; jj++) {
            const int j = n / 2 + (jj - m / 2);
            for (int ii = 0; ii < m; ii++) {
                const int i = n / 2 + (ii - m / 2);
                out[((size_t)kk * m + jj) * m + ii] =
                    (i < 0 || i >= n || j < 0 || j >= n || k < 0 || k >= n) ? pad : in[((size_t)k * n + j) * n + i];
            }
        }
    }
    return out;
}

// Fourier-space Image::ClipInto of an n^3 half spectrum into m^3 with zero
// padding, including the Nyquist fill when growing (image.cpp:8592-8700)
std::vector<cplx> fclip3(const std::vector<cplx>& in, int n, int m) {
    const int hn = n / 2 + 1, hm = m / 2 + 1;
    const int ub_x = n % 2 == 0 ? n / 2 : (n - 1) / 2;
    const int lb = n % 2 == 0 ? -(n / 2) : -((n - 1) / 2), ub = n % 2 == 0 ? n / 2 - 1 : (n - 1) / 2;
    auto src = [&](int lx, int ly, int lz) -> cplx {
        if (lx > ub_x || ly < lb || ly > ub || lz < lb || lz > ub) return cplx(0, 0);
        const int py = ly >= 0 ? ly : n + ly, pz = lz >= 0 ? lz : n + lz;
        return in[((size_t)pz * n + py) * hn + lx];
    };
    std::vector<cplx> out((size_t)m * m * hm);
    auto oat = [&](int px, int py, int pz) -> cplx& { return out[((size_t)pz * m + py) * hm + px]; };
    for (int kk = 0; kk < m; kk++)
        for (int jj = 0; jj < m; jj++)
            for (int ii = 0; ii < hm; ii++) oat(ii, jj, kk) = src(ii, logical(jj, m), logical(kk, m));
    if (n < m) {
        const int first_neg = n % 2 == 0 ? n / 2 : n / 2 + 1;
        // positive Nyquist of the second dimension: output logical y = first_neg from input y = lb
        for (int lz = lb; lz <= ub; lz++) {
            const int pz = lz >= 0 ? lz : m + lz;
            for (int ii = 0; ii < hn && ii < hm; ii++) oat(ii, first_neg, pz) = src(ii, lb, lz);
        }
        // positive Nyquist of the third dimension, mirrored from logical -n/2
        const int kk = first_neg, kk_mirror = m - first_neg;
        for (int jj = 1; jj <= first_neg; jj++)
            for (int ii = 0; ii < hn; ii++) oat(ii, jj, kk) = oat(ii, jj, kk_mirror);
        for (int jj = m - first_neg; jj <= m - 1; jj++)
            for (int ii = 0; ii < hn; ii++) oat(ii, jj, kk) = oat(ii, jj, kk_mirror);
        for (int ii = 0; ii < hn; ii++) oat(ii, 0, kk) = oat(ii, 0, kk_mirror);
    }
    return out;
}

// ChangePixelSize's pad -> forward FFT (scaled 1/P^3) -> Fourier crop or
// grow to N^3 -> inverse FFT -> centred real-space clip back to T^3, for a
// T^3 volume padded with `pad_value` to P^3 (image.cpp:8785-8817).  The chain
// is linear and separable, so it is evaluated as three T x T complex operators
// (one per axis) on the T^3 support instead of transforms of the P^3 box
// (P is about 1000 for every template the tolerance of 0.001 applies to):
//   out(q) = Re[ sum_k w(kx) F(k) e^{+2 pi i k.q/N} ],  F(k) = (1/P^3) sum_p u(p) e^{-2 pi i k.p/P} + pad delta_k
// with u = volume - pad on its support.  The frequencies kept are those the
// Fourier ClipInto keeps: cropping (N <= P) kx in [0, N/2], ky, kz in
// [-N/2, N/2-1]; growing (N > P) kx in [0, P/2] and ky, kz in [-P/2, P/2],
// the positive Nyquist planes being the copies ClipInto fills in (F is
// P-periodic).  w(kx) is the half-spectrum weight of the inverse real
// transform: 1 at kx = 0 and at kx = N/2, 2 elsewhere.
std::vector<double> resample_through_padding(const std::vector<double>& vol, int T, int P, int N, double pad_value) {
    const bool grow = N > P;
    const int kx_hi = grow ? P / 2 : N / 2;
    const int k_lo = grow ? -(P / 2) : -(N / 2), k_hi = grow ? P / 2 : N / 2 - 1;
    auto phase = [](long a, long n) { return 2.0 * M_PI * (double)(((a % n) + n) % n) / (double)n; };
    // operators [t][i]: input voxel i sits at P-grid position P/2 + i - T/2,
    // output voxel t reads N-grid position N/2 + t - T/2
    std::vector<cplx> mx((size_t)T * T), my((size_t)T * T);
    std::vector<char> inside(T);
    for (int t = 0; t < T; t++) {
        const long q = N / 2 + t - T / 2;
        inside[t] = q >= 0 && q < N;
        for (int i = 0; i < T; i++) {
            const long pp = P / 2 + i - T / 2;
            cplx ax = 0, ay = 0;
            for (int k = 0; k <= kx_hi; k++) {
                const double w = (k == 0 || (!grow && k == N / 2)) ? 1.0 : 2.0;
                ax += w * std::polar(1.0, phase((long)k * q, N) - phase((long)k * pp, P));
            }
            for (int k = k_lo; k <= k_hi; k++) ay += std::polar(1.0, phase((long)k * q, N) - phase((long)k * pp, P));
            mx[(size_t)t * T + i] = ax;
            my[(size_t)t * T + i] = ay;
        }
    }
    const size_t n3 = (size_t)T * T * T;
    std::vector<cplx> a(n3), b(n3);
    // x: a[z][y][t] = sum_i mx[t][i] u[z][y][i]
#pragma omp parallel for schedule(static)
    for (long r = 0; r < (long)T * T; r++) {
        const double* u = vol.data() + (size_t)r * T;
        for (int t = 0; t < T; t++) {
            cplx acc = 0;
            const cplx* m = &mx[(size_t)t * T];
            for (int i = 0; i < T; i++) acc += m[i] * (u[i] - pad_value);
            a[(size_t)r * T + t] = acc;
        }
    }
    // y: b[z][t][x] = sum_j my[t][j] a[z][j][x]
#pragma omp parallel for schedule(static)
    for (long zt = 0; zt < (long)T * T; zt++) {
        const long z = zt / T, t = zt % T;
        cplx* dst = &b[((size_t)z * T + t) * T];
        for (int x = 0; x < T; x++) dst[x] = 0;
        for (int j = 0; j < T; j++) {
            const cplx m = my[(size_t)t * T + j];
            const cplx* src = &a[((size_t)z * T + j) * T];
            for (int x = 0; x < T; x++) dst[x] += m * src[x];
        }
    }
    // z: out[t][y][x] = Re sum_k my[t][k] b[k][y][x] / P^3 + pad
    const double inv = 1.0 / ((double)P * P * P);
    std::vector<double> out(n3);
#pragma omp parallel for schedule(static)
    for (long ty = 0; ty < (long)T * T; ty++) {
        const long t = ty / T, y = ty % T;
        std::vector<cplx> acc(T, cplx(0, 0));
        for (int k = 0; k < T; k++) {
            const cplx m = my[(size_t)t * T + k];
            const cplx* src = &b[((size_t)k * T + y) * T];
            for (int x = 0; x < T; x++) acc[x] += m * src[x];
        }
        double* o = &out[((size_t)t * T + y) * T];
        for (int x = 0; x < T; x++)
            o[x] = (inside[t] && inside[y] && inside[x]) ? acc[x].real() * inv + pad_value : pad_value;
    }
    return out;
}

}  // namespace

float edge_mean(const Image2& im) {
    double s = 0;
    long n = 0;
    for (int x = 0; x < im.nx; x++) s += im.at(x, 0);
    n += im.nx;
    for (int y = 1; y < im.ny - 1; y++) { s += im.at(0, y); s += im.at(im.nx - 1, y); n += 2; }
    for (int x = 0; x < im.nx; x++) s += im.at(x, im.ny - 1);
    n += im.nx;
    return (float)(s / (float)n);
}

Image2 clip_into(const Image2& im, int ox, int oy, float pad) {
    Image2 o;
    o.nx = ox;
    o.ny = oy;
    o.v.resize((size_t)ox * oy);
    for (int jj = 0; jj < oy; jj++) {
        const int j = im.ny / 2 + (jj - oy / 2);
        for (int ii = 0; ii < ox; ii++) {
            const int i = im.nx / 2 + (ii - ox / 2);
            o.at(ii, jj) = (i < 0 || i >= im.nx || j < 0 || j >= im.ny) ? pad : im.at(i, j);
        }
    }
    return o;
}

Image2 rotate90(const Image2& im, bool positive) {
    Image2 o;
    o.nx = im.ny;
    o.ny = im.nx;
    o.v.resize(im.v.size());
    for (int yo = 0; yo < im.ny; yo++)
        for (int xo = 0; xo < im.nx; xo++) {
            const int xn = positive ? im.ny - yo - 1 : yo;
            const int yn = positive ? xo : im.nx - xo - 1;
            o.at(xn, yn) = im.at(xo, yo);
        }
    return o;
}

bool is_power_of_two(int n) {
    if (n == 0) return false;
    return std::ceil(std::log2((float)n)) == std::floor(std::log2((float)n));
}

int factorize_dimension(int original, int template_size) {
    static const int primes[6] = {2, 3, 5, 7, 9, 13};
    for (int p : primes) {
        // MUST_BE_FACTOR_OF_FOUR is passed as the int enforce_factor (= 1)
        int neg = original % 2 ? original - 1 : original;
        while (neg >= 2 && !small_factors(neg, p)) neg -= 1;
        int pos = original % 2 ? original + 1 : original;
        while (pos < 10000 * original && !small_factors(pos, p)) pos += 1;
        if ((float)(original - neg) < (float)template_size * 0.000001f) return neg;
        if ((float)(pos - original) < (float)original * 0.1f) return pos;
    }
    return original;
}

Whitened whiten(const Image2& micrograph, bool swap) {
    const int nx = micrograph.nx, ny = micrograph.ny, hc = nx / 2 + 1;
    const long n = (long)nx * ny;
    std::vector<double> img(micrograph.v.begin(), micrograph.v.end());
    // ReplaceOutliersWithMean(5) (image.cpp:986-1007)
    double s = 0, s2 = 0;
    for (double v : img) { s += v; s2 += v * v; }
    const float mean = (float)(s / n);
    const float sigma = sqrtf(fabsf((float)(s2 / n - (s / n) * (s / n))));
    const float vmax = mean + 5.0f * sigma, vmin = mean - 5.0f * sigma;
    for (double& v : img)
        if (v > vmax || v < vmin) v = mean;
    std::vector<cplx> spec((size_t)hc * ny);
    rfft2(nx, ny, img.data(), spec.data());
    const double inv = 1.0 / (double)n;
    for (cplx& c : spec) c *= inv;
    if (swap) swap_quadrants_centred(nx, ny, 1, spec.data());
    spec[0] = 0;
    // Compute1DPowerSpectrumCurve (image.cpp:7135-7201)
    const int npts = curve_points(nx);
    const float hi = 0.5f * sqrtf(2.0f);
    Curve pw(0.0f, hi, npts), cnt(0.0f, hi, npts);
    const float vx = (float)(1.0 / (double)nx), vy = (float)(1.0 / (double)ny);
    const int first_neg = ny % 2 == 0 ? ny / 2 : ny / 2 + 1;
    for (int y = 0; y < ny; y++) {
        const float sy = powf(logical(y, ny) * vy, 2);
        for (int x = 0; x < hc; x++) {
            if (x == 0 && y >= first_neg) continue;
            const float f = sqrtf(powf(x * vx, 2) + sy);
            pw.add(f, std::norm(spec[(size_t)y * hc + x]));
            cnt.add(f, 1.0);
        }
    }
    Curve wf(0.0f, hi, npts);
    double mx = -DBL_MAX;
    for (int i = 0; i < npts; i++) {
        double v = cnt.y[i] > 0 ? pw.y[i] / cnt.y[i] : 0.0;
        v = std::sqrt(v);
        if (v != 0.0) v = 1.0 / v;
        wf.y[i] = v;
        mx = std::max(mx, v);
    }
    for (double& v : wf.y) v *= 1.0 / mx;
    // ApplyCurveFilter (image.cpp:7284-7310)
    for (int y = 0; y < ny; y++) {
        const double sy = std::pow(logical(y, ny) * vy, 2);
        for (int x = 0; x < hc; x++) {
            const float f = (float)std::sqrt(std::pow(x * vx, 2) + sy);
            cplx& c = spec[(size_t)y * hc + x];
            c = f <= 1.0f ? c * wf.at(f) : cplx(0, 0);
        }
    }
    spec[0] = 0;
    // / sqrt(ReturnSumOfSquares), Fourier branch with Hermitian weights (image.cpp:307-330)
    double sum = 0;
    for (int y = 0; y < ny; y++) {
        const int jj = logical(y, ny);
        for (int x = 0; x < hc; x++) {
            const double p = std::norm(spec[(size_t)y * hc + x]);
            const bool ex = x == 0 || (x == nx / 2 && nx % 2 == 0);
            const bool ey = jj == 0 || (jj == -(ny / 2) && nx % 2 == 0);
            if (ex && ey) sum += 0.5 * p;
            else if ((x != 0 && (x != nx / 2 || nx % 2 != 0)) || jj >= 0) sum += p;
        }
    }
    const double norm = std::sqrt(2.0 * sum);
    Whitened out;
    out.spectrum.resize(spec.size());
    for (size_t i = 0; i < spec.size(); i++) out.spectrum[i] = std::complex<float>(spec[i] / norm);
    out.curve = wf.y;
    return out;
}

std::vector<std::complex<float>> template_spectrum(const std::vector<float>& volume, int T, float factor) {
    const int hc = T / 2 + 1;
    std::vector<double> vol(volume.begin(), volume.end());
    std::vector<cplx> spec;
    const float tol = 0.001f;
    if (fabsf(factor - 1.0f) < tol) {
        spec.resize((size_t)T * T * hc);
        rfft3(T, T, T, vol.data(), spec.data());
        const double inv = 1.0 / ((double)T * T * T);
        for (cplx& c : spec) c *= inv;
    } else {
        // ChangePixelSize (image.cpp:8705-8822), cubic volume
        const int old = T, min_dim = T;
        int pad, nw;
        if (tol < 1.0f / (min_dim * factor)) {
            const float inter = 1.0f / (tol * min_dim);
            pad = (int)(old * inter);
            if ((old % 2 == 0) != (pad % 2 == 0)) pad++;
            nw = (int)(pad / factor);
            if ((old % 2 == 0) != (nw % 2 == 0)) nw++;
        } else {
            pad = (int)(old * factor);
            if ((old % 2 == 0) != (pad % 2 == 0)) pad++;
            nw = old;
        }
        double padding_value = 0.0;
        if (pad > old) {
            // ReturnAverageOfRealValues within 0.45 * min_dim of the box centre (image.cpp:6263-6300)
            const float r2 = powf(0.45f * min_dim, 2);
            double s = 0;
            long cnt = 0;
            for (int k = 0; k < T; k++)
                for (int j = 0; j < T; j++)
                    for (int i = 0; i < T; i++) {
                        const float d = powf((float)(k - T / 2), 2) + powf((float)(j - T / 2), 2) + powf((float)(i - T / 2), 2);
                        if (d <= r2) { s += vol[((size_t)k * T + j) * T + i]; cnt++; }
                    }
            padding_value = cnt ? (float)(s / cnt) : 0.0;
        }
        if (nw == T) {
            // the cropped spectrum is the result (image.cpp:8805-8810)
            std::vector<double> big = clip3(vol, old, pad, padding_value);
            std::vector<cplx> bs((size_t)pad * pad * (pad / 2 + 1));
            rfft3(pad, pad, pad, big.data(), bs.data());
            const double inv = 1.0 / ((double)pad * pad * pad);
            for (cplx& c : bs) c *= inv;
            spec = fclip3(bs, pad, nw);
        } else {
            std::vector<double> back = resample_through_padding(vol, T, pad, nw, padding_value);
            spec.resize((size_t)T * T * hc);
            rfft3(T, T, T, back.data(), spec.data());
            const double inv2 = 1.0 / ((double)T * T * T);
            for (cplx& c : spec) c *= inv2;
        }
    }
    spec[0] = 0;
    swap_quadrants_centred(T, T, T, spec.data());
    std::vector<std::complex<float>> out(spec.size());
    for (size_t i = 0; i < spec.size(); i++) out[i] = std::complex<float>(spec[i]);
    return out;
}

std::vector<float> projection_filter(int T, const std::vector<double>& curve, const CtfParams& p, float defocus_offset) {
    const int hc = T / 2 + 1;
    // CTF::Init (ctf.cpp:95-130) and SetDefocus as match_template.cpp:895
    const float lam = (float)(12.2639f / sqrtf((float)(1000.0f * p.kv + 0.97845e-6 * powf(1000.0f * p.kv, 2)))) / p.pixel_size;
    const float lam2 = powf(lam, 2);
    const float cs = (float)(p.cs_mm * 10000000.0 / p.pixel_size);
    const float act = fabs(p.amplitude_contrast - 1.0) < 1e-3 ? (float)(kPi / 2.0f)
                                                              : atanf(p.amplitude_contrast / sqrtf((float)(1.0 - powf(p.amplitude_contrast, 2))));
    const float phase = deg2rad(p.phase_shift_deg);
    const float df1 = (p.defocus1 + defocus_offset) / p.pixel_size;
    const float df2 = (p.defocus2 + defocus_offset) / p.pixel_size;
    const float az0 = deg2rad(p.astigmatism_angle_deg);
    const float v = (float)(1.0 / (double)T);
    Curve wf(0.0f, 0.5f * sqrtf(2.0f), (int)curve.size());
    wf.y = curve;
    std::vector<float> out((size_t)T * hc);
    for (int j = 0; j < T; j++) {
        const float y = logical(j, T) * v;
        const float y2 = powf(y, 2);
        for (int i = 0; i < hc; i++) {
            const float x = i * v;
            const float az = (i == 0 && j == 0) ? 0.0f : atan2f(y, x);
            const float g2 = powf(x, 2) + y2;
            float ctf;
            if (df1 == 0.0f && df2 == 0.0f) ctf = -0.7f;
            else {
                const float df = 0.5f * (df1 + df2 + cosf(2.0f * (az - az0)) * (df1 - df2));
                ctf = -sinf(kPif * lam * g2 * (df - 0.5f * lam2 * g2 * cs) + phase + act);
            }
            const float f = (float)std::sqrt(std::pow(i * v, 2) + std::pow(logical(j, T) * v, 2));
            out[(size_t)j * hc + i] = f <= 1.0f ? (float)(ctf * wf.at(f)) : 0.0f;
        }
    }
    return out;
}

std::vector<std::pair<float, float>> search_grid(float angular_step, const std::string& symmetry) {
    std::vector<std::pair<float, float>> out;
    if (symmetry.empty()) return out;
    const char t = (char)toupper(symmetry[0]);
    int num = 0;
    if (symmetry.size() > 1) num = std::atoi(symmetry.c_str() + 1);
    float phi_max, theta_max;
    switch (t) {
        case 'C': if (num <= 0) return out; phi_max = 360.0f / num; theta_max = 90.0f; break;
        case 'D': if (num <= 0) return out; phi_max = 360.0f / num; theta_max = 90.0f; break;
        case 'T': phi_max = 180.0f; theta_max = 54.7f; break;
        case 'O': phi_max = 90.0f; theta_max = 54.7f; break;
        case 'I': phi_max = 180.0f; theta_max = 31.7f; break;
        default: return out;
    }
    if (t == 'C' && num == 1) theta_max = 180.0f;
    const float theta_step = theta_max / (int)(theta_max / angular_step + 0.5f);
    for (float theta = 0.0f; theta < theta_max + theta_step / 2.0; theta += theta_step) {
        float phi_step;
        if (theta == 0.0f || theta == 180.0f) phi_step = phi_max;
        else {
            phi_step = fabsf(angular_step / sinf(deg2rad(theta)));
            if (phi_step > phi_max) phi_step = phi_max;
            phi_step = phi_max / (int)(phi_max / phi_step + 0.5f);
        }
        for (float phi = 0.0f; phi < phi_max; phi += phi_step) out.emplace_back(phi, theta);
    }
    return out;
}

std::vector<float> psi_list(float psi_start, float psi_step, float psi_max) {
    std::vector<float> out;
    for (float psi = psi_start; psi <= psi_max; psi += psi_step) out.push_back(psi);
    return out;
}

float angular_step_for(float resolution, float radius) { return (float)(360.0 * resolution / kPi / radius); }

double erfcinv_approx(double x) {
    const double y = 1.0 - x;
    const double sgn = y < 0 ? -1.0 : 1.0;
    const double lnx = std::log((1 - y) * (1 + y));
    const double tt1 = 2 / (kPi * 0.147) + 0.5 * lnx;
    const double tt2 = 1 / 0.147 * lnx;
    return sgn * std::sqrt(-tt1 + std::sqrt(tt1 * tt1 - tt2));
}

void swap_quadrants(int nx, int ny, int nz, std::complex<double>* spec) { swap_quadrants_centred(nx, ny, nz, spec); }

std::vector<std::complex<float>> padded_template_spectrum(const std::vector<float>& volume, int T, int TP) {
    if (TP == T) return template_spectrum(volume, T, 1.0f);
    // ReturnAverageOfRealValuesOnEdges, 3-D (image.cpp:5951-6004): first and
    // last planes whole, the other planes' first and last rows and the first
    // and last pixel of their other rows
    double sum = 0.0;
    long n = 0;
    auto at = [&](int i, int j, int k) { return (double)volume[((size_t)k * T + j) * T + i]; };
    for (int k : {0, T - 1})
        for (int j = 0; j < T; j++)
            for (int i = 0; i < T; i++) sum += at(i, j, k);
    n += 2L * T * T;
    for (int k = 1; k < T - 1; k++)
        for (int j = 0; j < T; j++) {
            if (j == 0 || j == T - 1) {
                for (int i = 0; i < T; i++) sum += at(i, j, k);
                n += T;
            } else {
                sum += at(0, j, k) + at(T - 1, j, k);
                n += 2;
            }
        }
    const float edge = (float)(sum / (float)n);
    std::vector<double> vol(volume.begin(), volume.end());
    std::vector<double> big = clip3(vol, T, TP, edge);
    const int hc = TP / 2 + 1;
    std::vector<cplx> spec((size_t)TP * TP * hc);
    rfft3(TP, TP, TP, big.data(), spec.data());
    const double inv = 1.0 / ((double)TP * TP * TP);
    for (cplx& c : spec) c *= inv;
    spec[0] = 0;
    swap_quadrants_centred(TP, TP, TP, spec.data());
    std::vector<std::complex<float>> out(spec.size());
    for (size_t i = 0; i < spec.size(); i++) out[i] = std::complex<float>(spec[i]);
    return out;
}

}  // namespace tmhost
