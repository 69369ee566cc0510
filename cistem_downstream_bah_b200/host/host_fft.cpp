// host_fft.cpp -- mixed-radix (2, 3, 5, any odd prime) Stockham FFT in double,
// with multi-dimensional real transforms built from it.  Used once per
// micrograph / template plane; the search itself runs on the GPU.
#include "host_fft.hpp"

#include <cmath>
#include <map>
#include <mutex>

namespace tmhost {
namespace {

struct Plan {
    int n = 0;
    std::vector<int> radix;
    std::vector<cplx> w;   // exp(-2 pi i m / n)
};

const Plan& plan_for(int n) {
    static std::map<int, Plan> cache;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(n);
    if (it != cache.end()) return it->second;
    Plan p;
    p.n = n;
    int m = n;
    while (m % 4 == 0 && m > 4) { p.radix.push_back(4); m /= 4; }
    while (m % 2 == 0) { p.radix.push_back(2); m /= 2; }
    for (int f = 3; m > 1; f += 2)
        while (m % f == 0) { p.radix.push_back(f); m /= f; }
    p.w.resize(n);
    for (int i = 0; i < n; i++) p.w[i] = std::polar(1.0, -2.0 * M_PI * i / n);
    return cache.emplace(n, std::move(p)).first->second;
}

void stockham(const Plan& p, cplx* x, cplx* work, int sign) {
    const int n = p.n;
    cplx* a = x;
    cplx* b = work;
    int ns = 1;
    std::vector<cplx> u(64), o(64);
    for (int R : p.radix) {
        const int nr = n / R;
        if ((int)u.size() < R) { u.resize(R); o.resize(R); }
        for (int j = 0; j < nr; j++) {
            const int jm = j % ns;
            const int step = jm * (n / (ns * R));
            for (int r = 0; r < R; r++) {
                cplx tw = p.w[(size_t)(step * r) % n];
                if (sign > 0) tw = std::conj(tw);
                u[r] = a[j + r * nr] * tw;
            }
            for (int q = 0; q < R; q++) {
                cplx s = 0;
                for (int r = 0; r < R; r++) {
                    cplx tw = p.w[(size_t)((q * r) % R) * (n / R)];
                    if (sign > 0) tw = std::conj(tw);
                    s += u[r] * tw;
                }
                o[q] = s;
            }
            const int idxD = (j / ns) * ns * R + jm;
            for (int q = 0; q < R; q++) b[idxD + q * ns] = o[q];
        }
        std::swap(a, b);
        ns *= R;
    }
    if (a != x)
        for (int i = 0; i < n; i++) x[i] = a[i];
}

// real row -> half spectrum
void rfft_row(int n, const double* in, cplx* out) {
    std::vector<cplx> z(n), w(n);
    for (int i = 0; i < n; i++) z[i] = in[i];
    stockham(plan_for(n), z.data(), w.data(), -1);
    for (int k = 0; k <= n / 2; k++) out[k] = z[k];
}

// half spectrum -> real row; imaginary parts of DC and Nyquist ignored
void irfft_row(int n, const cplx* in, double* out) {
    std::vector<cplx> z(n), w(n);
    for (int k = 0; k <= n / 2; k++) z[k] = in[k];
    z[0] = z[0].real();
    if (n % 2 == 0) z[n / 2] = z[n / 2].real();
    for (int k = n / 2 + 1; k < n; k++) z[k] = std::conj(z[n - k]);
    stockham(plan_for(n), z.data(), w.data(), +1);
    for (int i = 0; i < n; i++) out[i] = z[i].real();
}

// transform `count` strided lines of length n
void lines(int n, cplx* data, long stride, long count, long line_step, int sign) {
    const Plan& p = plan_for(n);
#pragma omp parallel
    {
        std::vector<cplx> buf(n), w(n);
#pragma omp for schedule(static)
        for (long c = 0; c < count; c++) {
            cplx* base = data + c * line_step;
            for (int i = 0; i < n; i++) buf[i] = base[i * stride];
            stockham(p, buf.data(), w.data(), sign);
            for (int i = 0; i < n; i++) base[i * stride] = buf[i];
        }
    }
}

}  // namespace

void fft1(std::vector<cplx>& x, int sign) {
    std::vector<cplx> w(x.size());
    stockham(plan_for((int)x.size()), x.data(), w.data(), sign);
}

void rfft2(int nx, int ny, const double* in, cplx* out) {
    const int hc = nx / 2 + 1;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < ny; y++) rfft_row(nx, in + (size_t)y * nx, out + (size_t)y * hc);
    lines(ny, out, hc, hc, 1, -1);
}

void irfft2(int nx, int ny, const cplx* in, double* out) {
    const int hc = nx / 2 + 1;
    std::vector<cplx> tmp(in, in + (size_t)hc * ny);
    lines(ny, tmp.data(), hc, hc, 1, +1);
#pragma omp parallel for schedule(static)
    for (int y = 0; y < ny; y++) irfft_row(nx, tmp.data() + (size_t)y * hc, out + (size_t)y * nx);
}

void rfft3(int nx, int ny, int nz, const double* in, cplx* out) {
    const int hc = nx / 2 + 1;
#pragma omp parallel for schedule(static)
    for (long r = 0; r < (long)ny * nz; r++) rfft_row(nx, in + (size_t)r * nx, out + (size_t)r * hc);
    for (int z = 0; z < nz; z++) lines(ny, out + (size_t)z * ny * hc, hc, hc, 1, -1);
    lines(nz, out, (long)ny * hc, (long)ny * hc, 1, -1);
}

void irfft3(int nx, int ny, int nz, const cplx* in, double* out) {
    const int hc = nx / 2 + 1;
    std::vector<cplx> tmp(in, in + (size_t)hc * ny * nz);
    lines(nz, tmp.data(), (long)ny * hc, (long)ny * hc, 1, +1);
    for (int z = 0; z < nz; z++) lines(ny, tmp.data() + (size_t)z * ny * hc, hc, hc, 1, +1);
#pragma omp parallel for schedule(static)
    for (long r = 0; r < (long)ny * nz; r++) irfft_row(nx, tmp.data() + (size_t)r * hc, out + (size_t)r * nx);
}

}  // namespace tmhost
