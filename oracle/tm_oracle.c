/*
 * tm_oracle.c -- CPU restatement of cisTEM's match_template search path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the B200 search core:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg (and the
 * reference arm of bench.py) load it.  Nothing in the product library links it.
 *
 * It restates, in plain C, the reference CPU path of match_template
 * (src/programs/match_template/match_template.cpp:519-1370) and the Image / CTF /
 * Curve / EulerSearch primitives it calls.  Each function cites the reference
 * file:line it follows (paths relative to the reference project root).
 *
 * Precision: ORC_REAL is double by default (the FP64 oracle used for parity);
 * building with -DORC_FLOAT gives the FP32 variant that is timed as the
 * CPU baseline ("port").  Quantities that the reference computes with float
 * arithmetic and then uses for a discrete decision (search-grid angles, psi
 * loop, Euler matrices, curve bin indices, histogram bins) are computed here
 * with the same float (or double) arithmetic in both builds.
 *
 * Pinning: the FFT, phase-shift, cross-correlation, peak-search, clip and
 * resize primitives are checked against the known answers of the reference's
 * own unit tests (src/programs/console_test/console_test.cpp:641-1035) on the
 * MRC fixtures embedded there.  No reference test pins the match_template
 * outputs themselves (MIP, angles, sums, histogram), so the end-to-end search
 * is "parity unpinned" beyond those primitives: the oracle is the reference
 * algorithm restated, not the reference binary (which needs wxWidgets and
 * FFTW, neither available here).
 *
 * Conventions (image.cpp:4761-4800, 5085-5113): forward FFTs are unnormalised
 * and divided by N when "scaled"; inverse FFTs are unnormalised.  The complex
 * half-spectrum of an nx-by-ny real image holds (nx/2+1) complex values per
 * row, ny rows.  Real images here are compact (no FFTW row padding).
 */
#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORC_FLOAT
typedef float real;
#else
typedef double real;
#endif

#define ORC_PI 3.14159265358979323846
/* cisTEM's PI / PIf constants (src/core/defines.h:6-7) */
#define CIS_PI 3.14159265359
#define CIS_PIF 3.14159265359f

#define EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------- */
/* 1-D complex FFT: Stockham autosort, mixed radix (2, 3, 4, 5, generic).     */
/* ------------------------------------------------------------------------- */

typedef struct {
    int n;
    int nstages;
    int radix[40];
    double *tw_re, *tw_im; /* exp(-2 pi i m / n), m = 0..n-1 */
} fft_plan;

static void plan_init(fft_plan *p, int n)
{
    int m = n, k = 0;
    p->n = n;
    while (m % 4 == 0 && m > 4) { p->radix[k++] = 4; m /= 4; }
    while (m % 2 == 0) { p->radix[k++] = 2; m /= 2; }
    for (int f = 3; m > 1; f += 2) {
        while (m % f == 0) { p->radix[k++] = f; m /= f; }
    }
    if (n == 1) k = 0;
    p->nstages = k;
    p->tw_re = (double *)malloc(sizeof(double) * (size_t)n);
    p->tw_im = (double *)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) {
        double a = -2.0 * ORC_PI * (double)i / (double)n;
        p->tw_re[i] = cos(a);
        p->tw_im[i] = sin(a);
    }
}

#define PLAN_CACHE 256
static fft_plan g_plans[PLAN_CACHE];
static int g_nplans = 0;

/* Plans are created once per length and never freed (the set of lengths a
 * search uses is small). */
static const fft_plan *get_plan(int n)
{
    const fft_plan *found = NULL;
#pragma omp critical(orc_plan_cache)
    {
        for (int i = 0; i < g_nplans; i++)
            if (g_plans[i].n == n) { found = &g_plans[i]; break; }
        if (!found && g_nplans < PLAN_CACHE) {
            plan_init(&g_plans[g_nplans], n);
            found = &g_plans[g_nplans++];
        }
    }
    if (!found) abort();
    return found;
}

/* in-place complex FFT of length n on interleaved data x; sign -1 forward,
 * +1 inverse (unnormalised).  work holds 2n reals. */
static void cfft(const fft_plan *p, real *x, real *work, int sign)
{
    const int n = p->n;
    real *a = x, *b = work;
    int ns = 1;
    for (int s = 0; s < p->nstages; s++) {
        const int R = p->radix[s];
        const int nr = n / R;
        for (int j = 0; j < nr; j++) {
            const int jm = j % ns;
            const int tstep = jm * (n / (ns * R));
            double ur[R], ui[R];   /* any radix: the generic branch is a direct DFT */
            for (int r = 0; r < R; r++) {
                double xr = a[2 * (j + r * nr)], xi = a[2 * (j + r * nr) + 1];
                int m = (tstep * r) % n;
                double wr = p->tw_re[m], wi = sign < 0 ? p->tw_im[m] : -p->tw_im[m];
                ur[r] = xr * wr - xi * wi;
                ui[r] = xr * wi + xi * wr;
            }
            const int idxD = (j / ns) * ns * R + jm;
            if (R == 2) {
                b[2 * idxD] = (real)(ur[0] + ur[1]);
                b[2 * idxD + 1] = (real)(ui[0] + ui[1]);
                b[2 * (idxD + ns)] = (real)(ur[0] - ur[1]);
                b[2 * (idxD + ns) + 1] = (real)(ui[0] - ui[1]);
            } else if (R == 4) {
                double ar = ur[0] + ur[2], ai = ui[0] + ui[2];
                double br = ur[0] - ur[2], bi = ui[0] - ui[2];
                double cr = ur[1] + ur[3], ci = ui[1] + ui[3];
                double dr = ur[1] - ur[3], di = ui[1] - ui[3];
                /* multiply d by -i (forward) or +i (inverse) */
                double er = sign < 0 ? di : -di, ei = sign < 0 ? -dr : dr;
                b[2 * idxD] = (real)(ar + cr);          b[2 * idxD + 1] = (real)(ai + ci);
                b[2 * (idxD + ns)] = (real)(br + er);   b[2 * (idxD + ns) + 1] = (real)(bi + ei);
                b[2 * (idxD + 2 * ns)] = (real)(ar - cr); b[2 * (idxD + 2 * ns) + 1] = (real)(ai - ci);
                b[2 * (idxD + 3 * ns)] = (real)(br - er); b[2 * (idxD + 3 * ns) + 1] = (real)(bi - ei);
            } else {
                /* generic radix: direct DFT with exp(sign 2 pi i q r / R) */
                for (int q = 0; q < R; q++) {
                    double sr = 0.0, si = 0.0;
                    for (int r = 0; r < R; r++) {
                        int m = ((q * r) % R) * (n / R);
                        double wr = p->tw_re[m], wi = sign < 0 ? p->tw_im[m] : -p->tw_im[m];
                        sr += ur[r] * wr - ui[r] * wi;
                        si += ur[r] * wi + ui[r] * wr;
                    }
                    b[2 * (idxD + q * ns)] = (real)sr;
                    b[2 * (idxD + q * ns) + 1] = (real)si;
                }
            }
        }
        real *t = a; a = b; b = t;
        ns *= R;
    }
    if (a != x) memcpy(x, a, sizeof(real) * 2 * (size_t)n);
}

/* Real-to-half-complex forward transform of length n (n even uses the
 * packing trick, odd n goes through a full complex transform). out holds
 * n/2+1 complex values.  Unnormalised. */
static void rfft1(int n, const real *in, real *out, real *work)
{
    if (n % 2 == 0) {
        const int h = n / 2;
        const fft_plan *p = get_plan(h);
        real *z = work;             /* 2h reals */
        real *w2 = work + 2 * h;    /* 2h reals */
        for (int i = 0; i < h; i++) { z[2 * i] = in[2 * i]; z[2 * i + 1] = in[2 * i + 1]; }
        cfft(p, z, w2, -1);
        for (int k = 0; k <= h; k++) {
            int k1 = k % h, k2 = (h - k) % h;
            double zr = z[2 * k1], zi = z[2 * k1 + 1];
            double cr = z[2 * k2], ci = -z[2 * k2 + 1];
            double er = 0.5 * (zr + cr), ei = 0.5 * (zi + ci);          /* even part */
            double orr = 0.5 * (zi - ci), oi = -0.5 * (zr - cr);          /* odd part = (Z - conj)/ (2i) */
            double a = -2.0 * ORC_PI * (double)k / (double)n;
            double wr = cos(a), wi = sin(a);
            out[2 * k] = (real)(er + orr * wr - oi * wi);
            out[2 * k + 1] = (real)(ei + orr * wi + oi * wr);
        }
    } else {
        const fft_plan *p = get_plan(n);
        real *z = work, *w2 = work + 2 * n;
        for (int i = 0; i < n; i++) { z[2 * i] = in[i]; z[2 * i + 1] = 0; }
        cfft(p, z, w2, -1);
        for (int k = 0; k <= n / 2; k++) { out[2 * k] = z[2 * k]; out[2 * k + 1] = z[2 * k + 1]; }
    }
}

/* Half-complex-to-real inverse of length n, unnormalised.  As FFTW's c2r, the
 * imaginary parts of the DC and (even n) Nyquist terms are ignored. */
static void irfft1(int n, const real *in, real *out, real *work)
{
    if (n % 2 == 0) {
        const int h = n / 2;
        const fft_plan *p = get_plan(h);
        real *z = work, *w2 = work + 2 * h;
        for (int k = 0; k < h; k++) {
            double hr = in[2 * k], hi = (k == 0) ? 0.0 : in[2 * k + 1];
            int km = h - k;
            double mr = in[2 * km], mi = (km == h || km == 0) ? 0.0 : in[2 * km + 1];
            /* E = H[k] + conj(H[h-k]);  O = (H[k] - conj(H[h-k])) * exp(+2 pi i k / n) */
            double er = hr + mr, ei = hi - mi;
            double dr = hr - mr, di = hi + mi;
            double a = 2.0 * ORC_PI * (double)k / (double)n;
            double wr = cos(a), wi = sin(a);
            double orr = dr * wr - di * wi, oi = dr * wi + di * wr;
            z[2 * k] = (real)(er - oi);
            z[2 * k + 1] = (real)(ei + orr);
        }
        cfft(p, z, w2, +1);
        for (int m = 0; m < h; m++) { out[2 * m] = z[2 * m]; out[2 * m + 1] = z[2 * m + 1]; }
    } else {
        const fft_plan *p = get_plan(n);
        real *z = work, *w2 = work + 2 * n;
        for (int k = 0; k <= n / 2; k++) {
            z[2 * k] = in[2 * k]; z[2 * k + 1] = (k == 0) ? 0 : in[2 * k + 1];
        }
        for (int k = n / 2 + 1; k < n; k++) { z[2 * k] = in[2 * (n - k)]; z[2 * k + 1] = -in[2 * (n - k) + 1]; }
        cfft(p, z, w2, +1);
        for (int m = 0; m < n; m++) out[m] = z[2 * m];
    }
}

/* strided complex transform of `count` columns, each of length n, stride
 * `stride` complex elements between consecutive entries, `col_step` complex
 * elements between columns. */
static void cfft_columns(int n, real *data, long stride, int ncols, int sign)
{
    const fft_plan *p = get_plan(n);
#pragma omp parallel for schedule(static) if (ncols >= 64 && n >= 256)
    for (int c0 = 0; c0 < ncols; c0 += 8) {
        int nc = ncols - c0 < 8 ? ncols - c0 : 8;
        real *buf = (real *)malloc(sizeof(real) * 2 * (size_t)n * 10);
        real *work = buf + 2 * (size_t)n * 8;
        for (int y = 0; y < n; y++)
            for (int c = 0; c < nc; c++) {
                buf[2 * ((size_t)c * n + y)] = data[2 * ((size_t)y * stride + c0 + c)];
                buf[2 * ((size_t)c * n + y) + 1] = data[2 * ((size_t)y * stride + c0 + c) + 1];
            }
        for (int c = 0; c < nc; c++) cfft(p, buf + 2 * (size_t)c * n, work, sign);
        for (int y = 0; y < n; y++)
            for (int c = 0; c < nc; c++) {
                data[2 * ((size_t)y * stride + c0 + c)] = buf[2 * ((size_t)c * n + y)];
                data[2 * ((size_t)y * stride + c0 + c) + 1] = buf[2 * ((size_t)c * n + y) + 1];
            }
        free(buf);
    }
}

/* 2-D real-to-complex forward FFT, unnormalised (FFTW fftwf_plan_dft_r2c_2d,
 * image.cpp:4819).  in: ny*nx reals; out: ny*(nx/2+1) complex. */
EXPORT void orc_rfft2(int nx, int ny, const real *in, real *out)
{
    const int hc = nx / 2 + 1;
#pragma omp parallel if (ny >= 256)
    {
        real *work = (real *)malloc(sizeof(real) * 4 * (size_t)(nx + 2));
#pragma omp for schedule(static)
        for (int y = 0; y < ny; y++) rfft1(nx, in + (size_t)y * nx, out + 2 * (size_t)y * hc, work);
        free(work);
    }
    cfft_columns(ny, out, hc, hc, -1);
}

/* 2-D complex-to-real inverse FFT, unnormalised (fftwf_plan_dft_c2r_2d,
 * image.cpp:4820).  The input is not modified. */
EXPORT void orc_irfft2(int nx, int ny, const real *in, real *out)
{
    const int hc = nx / 2 + 1;
    real *tmp = (real *)malloc(sizeof(real) * 2 * (size_t)hc * ny);
    memcpy(tmp, in, sizeof(real) * 2 * (size_t)hc * ny);
    cfft_columns(ny, tmp, hc, hc, +1);
#pragma omp parallel if (ny >= 256)
    {
        real *work = (real *)malloc(sizeof(real) * 4 * (size_t)(nx + 2));
#pragma omp for schedule(static)
        for (int y = 0; y < ny; y++) irfft1(nx, tmp + 2 * (size_t)y * hc, out + (size_t)y * nx, work);
        free(work);
    }
    free(tmp);
}

/* 3-D real-to-complex forward FFT, unnormalised (fftwf_plan_dft_r2c_3d,
 * image.cpp:4813).  in: nz*ny*nx reals; out: nz*ny*(nx/2+1) complex. */
EXPORT void orc_rfft3(int nx, int ny, int nz, const real *in, real *out)
{
    const int hc = nx / 2 + 1;
    real *work = (real *)malloc(sizeof(real) * 4 * (size_t)(nx + 2));
    for (long r = 0; r < (long)ny * nz; r++) rfft1(nx, in + (size_t)r * nx, out + 2 * (size_t)r * hc, work);
    free(work);
    for (int z = 0; z < nz; z++) cfft_columns(ny, out + 2 * (size_t)z * ny * hc, hc, hc, -1);
    /* along z: treat each (y, kx) as a column with stride ny*hc */
    cfft_columns(nz, out, (long)ny * hc, ny * hc, -1);
}

/* complex 1-D FFT exposed for tests (sign -1 forward, +1 inverse) */
EXPORT void orc_cfft(int n, real *x, int sign)
{
    const fft_plan *p = get_plan(n);
    real *work = (real *)malloc(sizeof(real) * 2 * (size_t)n);
    cfft(p, x, work, sign);
    free(work);
}

/* ------------------------------------------------------------------------- */
/* Small cisTEM helpers restated with the reference's float semantics.        */
/* ------------------------------------------------------------------------- */

/* functions.h:433-436 */
static float deg_2_rad_f(float degrees) { return (float)((double)(degrees * CIS_PIF) / 180.); }
/* functions.h:428-431 */
static float rad_2_deg_f(float radians) { return (float)((double)radians / ((double)CIS_PIF / 180.)); }
/* functions.h:480-483 */
static int myroundint_f(float a) { return a > 0 ? (int)(a + 0.5f) : (int)(a - 0.5f); }

/* RotationMatrix::SetToEulerRotation (matrix.cpp:490-510), float arithmetic.
 * m is row-major m[row][col]; RotateCoords (matrix.h:32-37) is m * (x,y,z). */
EXPORT void orc_euler_matrix(float phi, float theta, float psi, float *m)
{
    float cos_phi = cosf(deg_2_rad_f(phi)), sin_phi = sinf(deg_2_rad_f(phi));
    float cos_theta = cosf(deg_2_rad_f(theta)), sin_theta = sinf(deg_2_rad_f(theta));
    float cos_psi = cosf(deg_2_rad_f(psi)), sin_psi = sinf(deg_2_rad_f(psi));
    m[0] = cos_phi * cos_theta * cos_psi - sin_phi * sin_psi;       /* m[0][0] */
    m[3] = sin_phi * cos_theta * cos_psi + cos_phi * sin_psi;       /* m[1][0] */
    m[6] = -sin_theta * cos_psi;                                    /* m[2][0] */
    m[1] = -cos_phi * cos_theta * sin_psi - sin_phi * cos_psi;      /* m[0][1] */
    m[4] = -sin_phi * cos_theta * sin_psi + cos_phi * cos_psi;      /* m[1][1] */
    m[7] = sin_theta * sin_psi;                                     /* m[2][1] */
    m[2] = sin_theta * cos_phi;                                     /* m[0][2] */
    m[5] = sin_theta * sin_phi;                                     /* m[1][2] */
    m[8] = cos_theta;                                               /* m[2][2] */
}

/* ReturnClosestFactorizedUpper / Lower (functions.cpp:529-627). */
static int only_small_factors(int number, int largest_factor)
{
    int remainder = number;
    for (int factor = 2; factor <= largest_factor && remainder != 1; factor++) {
        while (remainder % factor == 0) remainder /= factor;
    }
    return remainder == 1;
}

EXPORT int orc_closest_factorized_upper(int wanted, int largest_factor, int enforce_even, int enforce_factor)
{
    int number, increment;
    if (enforce_factor != 0) { enforce_even = 1; increment = enforce_factor; } else increment = 2;
    if (enforce_even) {
        int start = wanted % 2 ? wanted + 1 : wanted;
        for (number = start; number < 10000 * wanted; number += increment)
            if (only_small_factors(number, largest_factor)) break;
    } else {
        for (number = wanted; number < 10000 * wanted; number++)
            if (only_small_factors(number, largest_factor)) break;
    }
    return number;
}

EXPORT int orc_closest_factorized_lower(int wanted, int largest_factor, int enforce_even, int enforce_factor)
{
    int number, decrement;
    if (enforce_factor) { enforce_even = 1; decrement = enforce_factor; } else decrement = 2;
    if (enforce_even) {
        int start = wanted % 2 ? wanted - 1 : wanted;
        for (number = start; number >= 2; number -= decrement)
            if (only_small_factors(number, largest_factor)) break;
    } else {
        for (number = wanted; number >= 1; number--)
            if (only_small_factors(number, largest_factor)) break;
    }
    return number;
}

/* is_power_of_two (functions.h:422-426) */
EXPORT int orc_is_power_of_two(int n)
{
    if (n == 0) return 0;
    return ceil(log2((float)n)) == floor(log2((float)n));
}

/* The factorisation loop of match_template.cpp:527-583: returns the padded
 * size for one dimension.  template_size is the reference's XSize (only used
 * by the never-taken reduction branch). */
EXPORT int orc_factorize_dimension(int original, int template_size)
{
    static const int primes[6] = {2, 3, 5, 7, 9, 13};
    const float max_reduction = 0.000001f, max_increase = 0.1f;
    int result = original;
    for (int i = 0; i < 6; i++) {
        /* MUST_BE_FACTOR_OF_FOUR is a bool passed as the int enforce_factor: 1 */
        int neg = orc_closest_factorized_lower(original, primes[i], 1, 1);
        int pos = orc_closest_factorized_upper(original, primes[i], 1, 1);
        if ((float)(original - neg) < (float)template_size * max_reduction) { result = neg; break; }
        if ((float)(-original + pos) < (float)original * max_increase) { result = pos; break; }
    }
    return result;
}

/* CalculateAngularStep (functions.cpp:629-632) */
EXPORT float orc_angular_step(float required_resolution, float radius_in_angstroms)
{
    return (float)(360.0 * required_resolution / CIS_PI / radius_in_angstroms);
}

/* cisTEM_erfinv / cisTEM_erfcinv (functions.cpp:1270-1302): closed-form
 * approximation with a = 0.147. */
EXPORT double orc_erfcinv(double x)
{
    double y = 1.0 - x;
    double sgn = (y < 0) ? -1.0 : 1.0;
    double t = (1 - y) * (1 + y);
    double lnx = log(t);
    double tt1 = 2 / (CIS_PI * 0.147) + 0.5 * lnx;
    double tt2 = 1 / (0.147) * lnx;
    return sgn * sqrt(-tt1 + sqrt(tt1 * tt1 - tt2));
}

/* Psi list: for (psi = psi_start; psi <= psi_max; psi += psi_step) with float
 * accumulation (match_template.cpp:746-750, 1001).  Returns the count; writes
 * up to max_out values. */
EXPORT int orc_psi_list(float psi_start, float psi_step, float psi_max, float *out, int max_out)
{
    int n = 0;
    for (float psi = psi_start; psi <= psi_max; psi += psi_step) {
        if (n < max_out && out) out[n] = psi;
        n++;
    }
    return n;
}

/* EulerSearch::SetSymmetryLimits (euler_search.cpp:353-440) for the symmetry
 * type letter and number; returns 0 on success. */
static int symmetry_limits(char type, int number, float *phi_max, float *theta_max, int *test_mirror)
{
    switch (type) {
    case 'C': if (number <= 0) return -1; *phi_max = 360.0f / number; *theta_max = 90.0f; *test_mirror = 1; return 0;
    case 'D': if (number <= 0) return -1; *phi_max = 360.0f / number; *theta_max = 90.0f; *test_mirror = 0; return 0;
    case 'T': *phi_max = 180.0f; *theta_max = 54.7f; *test_mirror = 0; return 0;
    case 'O': *phi_max = 90.0f; *theta_max = 54.7f; *test_mirror = 0; return 0;
    case 'I': *phi_max = 180.0f; *theta_max = 31.7f; *test_mirror = 0; return 0;
    default: return -1;
    }
}

/* The search grid of match_template.cpp:687-697: EulerSearch::InitGrid then,
 * for C1, theta_max = 180 and CalculateGridSearchPositions(false)
 * (euler_search.cpp:180-260).  Writes (phi, theta) pairs; returns the number
 * of search positions (or -1 on a bad symmetry). */
EXPORT int orc_search_grid(char sym_type, int sym_number, float angular_step, float *out, int max_out)
{
    float phi_max, theta_max;
    int test_mirror;
    if (symmetry_limits(sym_type, sym_number, &phi_max, &theta_max, &test_mirror)) return -1;
    if (sym_type == 'C' && sym_number == 1 && test_mirror) theta_max = 180.0f;
    float theta_step = theta_max / (int)(theta_max / angular_step + 0.5f);
    float theta_start_local = 0.0f, phi_start_local = 0.0f;
    int n = 0;
    for (float theta = theta_start_local; theta < theta_max + theta_step / 2.0; theta += theta_step) {
        float phi_step;
        if (theta == 0.0f || theta == 180.0f) phi_step = phi_max;
        else {
            phi_step = fabsf(angular_step / sinf(deg_2_rad_f(theta)));
            if (phi_step > phi_max) phi_step = phi_max;
            phi_step = phi_max / (int)(phi_max / phi_step + 0.5f);
            phi_start_local = 0.0f;
        }
        for (float phi = 0.0f; phi < phi_max; phi += phi_step) {
            if (out && n < max_out) { out[2 * n] = phi + phi_start_local; out[2 * n + 1] = theta; }
            n++;
        }
    }
    return n;
}

/* ------------------------------------------------------------------------- */
/* Fourier-space primitives.                                                  */
/* ------------------------------------------------------------------------- */

static int logical_y(int phys, int n) { return phys >= (n % 2 == 0 ? n / 2 : n / 2 + 1) ? phys - n : phys; }

/* Image::PhaseShift (image.cpp:9221-9265) on a compact half-spectrum.  The
 * phase is computed as the reference does (float phase, cosf/sinf). */
EXPORT void orc_phase_shift(int nx, int ny, int nz, real *spec, float sx, float sy, float sz)
{
    const int hc = nx / 2 + 1;
    long idx = 0;
    for (int k = 0; k < nz; k++) {
        int kl = logical_y(k, nz);
        float pz = (float)(sz * (float)kl * 2.0 * CIS_PI / nz);
        for (int j = 0; j < ny; j++) {
            int jl = logical_y(j, ny);
            float py = (float)(sy * (float)jl * 2.0 * CIS_PI / ny);
            for (int i = 0; i < hc; i++, idx++) {
                float px = (float)(sx * (float)i * 2.0 * CIS_PI / nx);
                float t = -px - py - pz;
                double c = cosf(t), s = sinf(t);
                double re = spec[2 * idx], im = spec[2 * idx + 1];
                spec[2 * idx] = (real)(re * c - im * s);
                spec[2 * idx + 1] = (real)(re * s + im * c);
            }
        }
    }
}

/* Image::SwapRealSpaceQuadrants (image.cpp:9757-9824) for a spectrum whose
 * object_is_centred_in_box flag is `centred` (1: shift by the box centre;
 * 0: even sizes by the centre, odd sizes by centre - 1). */
EXPORT void orc_swap_quadrants(int nx, int ny, int nz, real *spec, int centred)
{
    float sx, sy, sz;
    if (centred) { sx = (float)(nx / 2); sy = (float)(ny / 2); sz = (float)(nz / 2); }
    else {
        sx = nx % 2 == 0 ? (float)(nx / 2) : (float)(nx / 2) - 1.0f;
        sy = ny % 2 == 0 ? (float)(ny / 2) : (float)(ny / 2) - 1.0f;
        sz = nz % 2 == 0 ? (float)(nz / 2) : (float)(nz / 2) - 1.0f;
    }
    if (nz == 1) sz = 0.0f;
    orc_phase_shift(nx, ny, nz, spec, sx, sy, sz);
}

/* Image::ReturnLinearInterpolatedFourier (image.cpp:2899-3020) on a cubic
 * T^3 half-spectrum (layout [z][y][x], x in 0..T/2). */
static void interp3(int T, const real *vol, real x, real y, real z, double *outr, double *outi)
{
    const int hc = T / 2 + 1;
    const int lbx = -(T / 2), ubx = T / 2;                     /* even T */
    const int lby = T % 2 == 0 ? -(T / 2) : -((T - 1) / 2);
    const int uby = T % 2 == 0 ? T / 2 - 1 : (T - 1) / 2;
    const int ubx_odd = (T - 1) / 2;
    const int ux = T % 2 == 0 ? ubx : ubx_odd;
    const int lx = T % 2 == 0 ? lbx : -ubx_odd;
    double sr = 0, si = 0;
    *outr = 0; *outi = 0;
    if (x >= 0) {
        int i0 = (int)floor(x), i1 = i0 + 1;
        if (i1 > ux) return;
        int j0 = (int)floor(y); if (j0 < lby) return; int j1 = j0 + 1; if (j1 > uby) return;
        int k0 = (int)floor(z); if (k0 < lby) return; int k1 = k0 + 1; if (k1 > uby) return;
        for (int k = k0; k <= k1; k++) {
            int pz = k >= 0 ? k : T + k;
            double zd = fabs(z - (real)k);
            for (int j = j0; j <= j1; j++) {
                int py = j >= 0 ? j : T + j;
                double yd = fabs(y - (real)j);
                const real *row = vol + 2 * ((size_t)hc * ((size_t)T * pz + py));
                for (int i = i0; i <= i1; i++) {
                    double w = (1.0 - fabs(x - (real)i)) * (1.0 - yd) * (1.0 - zd);
                    sr += row[2 * i] * w;
                    si += row[2 * i + 1] * w;
                }
            }
        }
    } else {
        int i0 = (int)floor(x); if (i0 < lx) return; int i1 = i0 + 1;
        int j0 = (int)floor(y); if (j0 < lby) return; int j1 = j0 + 1; if (j1 > uby) return;
        int k0 = (int)floor(z); if (k0 < lby) return; int k1 = k0 + 1; if (k1 > uby) return;
        for (int k = k0; k <= k1; k++) {
            int pz = k > 0 ? T - k : -k;
            double zd = fabs(z - (real)k);
            for (int j = j0; j <= j1; j++) {
                int py = j > 0 ? T - j : -j;
                double yd = fabs(y - (real)j);
                const real *row = vol + 2 * ((size_t)hc * ((size_t)T * pz + py));
                for (int i = i0; i <= i1; i++) {
                    double w = (1.0 - fabs(x - (real)i)) * (1.0 - yd) * (1.0 - zd);
                    sr += row[2 * (-i)] * w;
                    si -= row[2 * (-i) + 1] * w;   /* conjugate */
                }
            }
        }
    }
    *outr = sr; *outi = si;
}

/* Image::ExtractSlice with apply_resolution_limit = false (image.cpp:2450-2607)
 * from a quadrant-swapped T^3 half-spectrum into a T x T half-spectrum
 * (layout [y][x], x in 0..T/2).  m: row-major Euler matrix. */
EXPORT void orc_extract_slice(int T, const real *vol, const float *m, real *out)
{
    const int hc = T / 2 + 1;
    const int lby = T % 2 == 0 ? -(T / 2) : -((T - 1) / 2);
    const int uby = T % 2 == 0 ? T / 2 - 1 : (T - 1) / 2;
    const int ubx = T % 2 == 0 ? T / 2 : (T - 1) / 2;
    double vr, vi;
    /* RotateCoords (matrix.h:32-37) evaluates the rotated coordinates in float;
     * their floor() decides which samples fall outside the box, so they are
     * computed here with the same float operations (no fused multiply-add). */
    for (int j = lby; j <= uby; j++) {
        int py = j >= 0 ? j : T + j;
        for (int i = 1; i <= ubx; i++) {
            const float fi = (float)i, fj = (float)j;
            volatile float px0 = m[0] * fi, px1 = m[1] * fj;
            volatile float py0 = m[3] * fi, py1 = m[4] * fj;
            volatile float pz0 = m[6] * fi, pz1 = m[7] * fj;
            float x3 = px0 + px1, y3 = py0 + py1, z3 = pz0 + pz1;
            interp3(T, vol, x3, y3, z3, &vr, &vi);
            out[2 * ((size_t)py * hc + i)] = (real)vr;
            out[2 * ((size_t)py * hc + i) + 1] = (real)vi;
        }
    }
    for (int j = 1; j <= uby; j++) {
        const float fj = (float)j;
        float x3 = m[1] * fj, y3 = m[4] * fj, z3 = m[7] * fj;
        interp3(T, vol, x3, y3, z3, &vr, &vi);
        out[2 * ((size_t)j * hc)] = (real)vr;
        out[2 * ((size_t)j * hc) + 1] = (real)vi;
        out[2 * ((size_t)(T - j) * hc)] = (real)vr;
        out[2 * ((size_t)(T - j) * hc) + 1] = (real)(-vi);
    }
    if (-lby != uby) {
        int j = lby;
        const float fj = (float)j;
        float x3 = m[1] * fj, y3 = m[4] * fj, z3 = m[7] * fj;
        interp3(T, vol, x3, y3, z3, &vr, &vi);
        int py = T + j;
        out[2 * ((size_t)py * hc)] = (real)vr;
        out[2 * ((size_t)py * hc) + 1] = (real)vi;
    }
    out[0] = 0; out[1] = 0;
}

/* ------------------------------------------------------------------------- */
/* CTF (ctf.cpp:79-130, 445-561) and the projection filter.                   */
/* ------------------------------------------------------------------------- */

typedef struct {
    float wavelength, squared_wavelength, spherical_aberration, amplitude_contrast;
    float defocus_1, defocus_2, astigmatism_azimuth, additional_phase_shift;
    float precomputed_amplitude_contrast_term;
} orc_ctf;

/* CTF::WavelengthGivenAccelerationVoltage (ctf.cpp:556-561) */
static float wavelength_kv(float kv)
{
    return (float)(12.2639f / sqrtf((float)(1000.0f * kv + 0.97845e-6 * powf(1000.0f * kv, 2))));
}

/* CTF::Init (ctf.cpp:95-130) for the 11-argument call of match_template.cpp:647 */
static void ctf_init(orc_ctf *c, float kv, float cs_mm, float amp, float df1, float df2, float ang_deg, float pixel, float phase_rad)
{
    c->wavelength = wavelength_kv(kv) / pixel;
    c->squared_wavelength = powf(c->wavelength, 2);
    c->spherical_aberration = (float)(cs_mm * 10000000.0 / pixel);
    c->amplitude_contrast = amp;
    c->defocus_1 = df1 / pixel;
    c->defocus_2 = df2 / pixel;
    c->astigmatism_azimuth = (float)(ang_deg / 180.0 * CIS_PI);
    c->additional_phase_shift = phase_rad;
    if (fabs(amp - 1.0) < 1e-3) c->precomputed_amplitude_contrast_term = (float)(CIS_PI / 2.0f);
    else c->precomputed_amplitude_contrast_term = atanf(amp / sqrtf((float)(1.0 - powf(amp, 2))));
}

/* CTF::Evaluate (ctf.cpp:445-460) with low_resolution_contrast = 0 */
static float ctf_eval(const orc_ctf *c, float g2, float azimuth)
{
    if (c->defocus_1 == 0.0f && c->defocus_2 == 0.0f) return -0.7f;
    float df = 0.5f * (c->defocus_1 + c->defocus_2 + cosf(2.0f * (azimuth - c->astigmatism_azimuth)) * (c->defocus_1 - c->defocus_2));
    float phase = CIS_PIF * c->wavelength * g2 * (df - 0.5f * c->squared_wavelength * g2 * c->spherical_aberration)
                  + c->additional_phase_shift + c->precomputed_amplitude_contrast_term;
    return -sinf(phase);
}

/* Curve (curve.cpp): x axis from SetupXAxis (:247-259), linear interpolation
 * from x (:377-397), linear-interpolated accumulation (:500-560). */
typedef struct { int n; float *x; real *y; } orc_curve;

static void curve_setup(orc_curve *c, float lo, float hi, int n)
{
    c->n = n;
    c->x = (float *)malloc(sizeof(float) * n);
    c->y = (real *)calloc((size_t)n, sizeof(real));
    for (int i = 0; i < n; i++) c->x[i] = i * (hi - lo) / (float)(n - 1) + lo;
}

static int curve_prev_bin(const orc_curve *c, float x)
{
    for (int i = 0; i < c->n - 1; i++)
        if (x >= c->x[i] && x < c->x[i + 1]) return i;
    if (x < c->x[0]) return 0;
    return c->n - 1;
}

static real curve_interp(const orc_curve *c, float x)
{
    int i = curve_prev_bin(c, x);
    if (i == c->n - 1) return c->y[c->n - 1];
    float d = (x - c->x[i]) / (c->x[i + 1] - c->x[i]);
    return (real)(c->y[i] * (1.0 - d) + c->y[i + 1] * (double)d);
}

static void curve_add_linear_x(orc_curve *c, float x, real v)
{
    int i = (c->x[0] == c->x[1]) ? c->n - 2 : (int)((x - c->x[0]) / (c->x[1] - c->x[0]));
    if (i == c->n - 1) { c->y[i] += v; return; }
    float d = (x - c->x[i]) / (c->x[i + 1] - c->x[i]);
    c->y[i] += (real)(v * (1.0 - d));
    c->y[i + 1] += (real)(v * (double)d);
}

/* Whitening of match_template.cpp:703-724 on an nx x ny real micrograph:
 * ReplaceOutliersWithMean(5), ForwardFFT (scaled), SwapRealSpaceQuadrants,
 * ZeroCentralPixel, Compute1DPowerSpectrumCurve, sqrt, reciprocal, /max,
 * ApplyCurveFilter, ZeroCentralPixel, /sqrt(ReturnSumOfSquares).
 * Writes the whitened half-spectrum (ny*(nx/2+1) complex) and the whitening
 * curve (curve_n points; the caller sizes it with orc_whitening_curve_points). */
EXPORT int orc_whitening_curve_points(int nx)
{
    return (int)((nx / 2.0 + 1.0) * sqrtf(2.0f) + 1.0);
}

static void apply_curve_filter(int nx, int ny, real *spec, const orc_curve *c)
{
    /* Image::ApplyCurveFilter (image.cpp:7284-7310), resolution_limit 1 */
    const int hc = nx / 2 + 1;
    const float vx = (float)(1.0 / (double)nx), vy = (float)(1.0 / (double)ny);
    for (int j = 0; j < ny; j++) {
        double sy = pow(logical_y(j, ny) * vy, 2);
        for (int i = 0; i < hc; i++) {
            double sx = pow(i * vx, 2);
            float f = (float)sqrt(sx + sy);
            size_t a = (size_t)j * hc + i;
            if (f <= 1.0f) {
                real w = curve_interp(c, f);
                spec[2 * a] *= w; spec[2 * a + 1] *= w;
            } else { spec[2 * a] = 0; spec[2 * a + 1] = 0; }
        }
    }
}

EXPORT void orc_whiten_image(int nx, int ny, real *image /* modified */, real *spec_out, real *curve_out)
{
    const long n = (long)nx * ny;
    const int hc = nx / 2 + 1;
    /* ReplaceOutliersWithMean (image.cpp:986-1007) */
    double s = 0, s2 = 0;
    for (long i = 0; i < n; i++) { s += image[i]; s2 += pow(image[i], 2); }
    float sigma = sqrtf(fabsf((float)(s2 / n - pow(s / n, 2))));
    float mean = (float)(s / n);
    float vmax = mean + 5.0f * sigma, vmin = mean - 5.0f * sigma;
    for (long i = 0; i < n; i++) {
        if (image[i] > vmax) image[i] = mean;
        else if (image[i] < vmin) image[i] = mean;
    }
    orc_rfft2(nx, ny, image, spec_out);
    const double inv_n = 1.0 / (double)n;
    for (long i = 0; i < (long)hc * ny * 2; i++) spec_out[i] = (real)(spec_out[i] * inv_n);
    orc_swap_quadrants(nx, ny, 1, spec_out, 1);
    spec_out[0] = 0; spec_out[1] = 0;
    /* Compute1DPowerSpectrumCurve (image.cpp:7135-7201) */
    int npts = orc_whitening_curve_points(nx);
    orc_curve wf, nt;
    curve_setup(&wf, 0.0f, 0.5f * sqrtf(2.0f), npts);
    curve_setup(&nt, 0.0f, 0.5f * sqrtf(2.0f), npts);
    const float vx = (float)(1.0 / (double)nx), vy = (float)(1.0 / (double)ny);
    const int first_neg_y = ny % 2 == 0 ? ny / 2 : ny / 2 + 1;
    for (int j = 0; j < ny; j++) {
        float sy = powf(logical_y(j, ny) * vy, 2);
        for (int i = 0; i < hc; i++) {
            if (i == 0 && j >= first_neg_y) continue;   /* explicit Hermitian mate */
            float sx = powf(i * vx, 2);
            float f = sqrtf(sx + sy);
            size_t a = (size_t)j * hc + i;
            real p = spec_out[2 * a] * spec_out[2 * a] + spec_out[2 * a + 1] * spec_out[2 * a + 1];
            curve_add_linear_x(&wf, f, p);
            curve_add_linear_x(&nt, f, 1.0);
        }
    }
    for (int i = 0; i < npts; i++) wf.y[i] = nt.y[i] > 0 ? wf.y[i] / nt.y[i] : 0;
    for (int i = 0; i < npts; i++) wf.y[i] = (real)sqrt(wf.y[i]);                  /* SquareRoot */
    for (int i = 0; i < npts; i++) if (wf.y[i] != 0.0) wf.y[i] = (real)(1.0 / wf.y[i]); /* Reciprocal */
    real mx = -FLT_MAX;
    for (int i = 0; i < npts; i++) if (wf.y[i] > mx) mx = wf.y[i];
    for (int i = 0; i < npts; i++) wf.y[i] = (real)(wf.y[i] * (1.0 / mx));
    apply_curve_filter(nx, ny, spec_out, &wf);
    spec_out[0] = 0; spec_out[1] = 0;
    /* ReturnSumOfSquares in Fourier space (image.cpp:307-330): Hermitian weights */
    double sum = 0;
    for (int j = 0; j < ny; j++) {
        int jj = logical_y(j, ny);
        for (int i = 0; i < hc; i++) {
            size_t a = (size_t)j * hc + i;
            double p = (double)spec_out[2 * a] * spec_out[2 * a] + (double)spec_out[2 * a + 1] * spec_out[2 * a + 1];
            int edge_x = (i == 0 || (i == nx / 2 && nx % 2 == 0));
            int edge_y = (jj == 0 || (jj == -(ny / 2) && nx % 2 == 0));
            if (edge_x && edge_y) sum += p * 0.5;
            else if ((i != 0 && (i != nx / 2 || nx % 2 != 0)) || jj >= 0) sum += p;
        }
    }
    double norm = sqrt(2.0 * sum);
    for (long i = 0; i < (long)hc * ny * 2; i++) spec_out[i] = (real)(spec_out[i] / norm);
    for (int i = 0; i < npts; i++) curve_out[i] = wf.y[i];
    free(wf.x); free(wf.y); free(nt.x); free(nt.y);
}

/* Projection filter of match_template.cpp:895-898: CTF image (image.cpp:
 * 3113-3160) times the whitening curve (ApplyCurveFilter), on the T x T
 * half-plane.  filter_out: T*(T/2+1) reals (the imaginary part is 0). */
EXPORT void orc_projection_filter(int T, float kv, float cs_mm, float amp, float df1, float df2, float ang_deg,
                                  float pixel, float phase_deg, float defocus_offset,
                                  const real *curve, int curve_n, float curve_hi, real *filter_out)
{
    orc_ctf c;
    ctf_init(&c, kv, cs_mm, amp, df1, df2, ang_deg, pixel, deg_2_rad_f(phase_deg));
    /* input_ctf.SetDefocus((df1 + i*step)/pixel, ..., deg_2_rad(angle)) */
    c.defocus_1 = (df1 + defocus_offset) / pixel;
    c.defocus_2 = (df2 + defocus_offset) / pixel;
    c.astigmatism_azimuth = deg_2_rad_f(ang_deg);
    const int hc = T / 2 + 1;
    const float v = (float)(1.0 / (double)T);
    orc_curve wf;
    wf.n = curve_n;
    wf.x = (float *)malloc(sizeof(float) * curve_n);
    wf.y = (real *)malloc(sizeof(real) * curve_n);
    for (int i = 0; i < curve_n; i++) { wf.x[i] = i * (curve_hi - 0.0f) / (float)(curve_n - 1) + 0.0f; wf.y[i] = curve[i]; }
    for (int j = 0; j < T; j++) {
        float y = logical_y(j, T) * v;
        float y2 = powf(y, 2);
        for (int i = 0; i < hc; i++) {
            float x = i * v;
            float az = (i == 0 && j == 0) ? 0.0f : atan2f(y, x);
            float g2 = powf(x, 2) + y2;
            real val = ctf_eval(&c, g2, az);
            double sx = pow(i * v, 2), sy = pow(logical_y(j, T) * v, 2);
            float f = (float)sqrt(sx + sy);
            if (f <= 1.0f) val = (real)(val * curve_interp(&wf, f));
            else val = 0;
            filter_out[(size_t)j * hc + i] = val;
        }
    }
    free(wf.x); free(wf.y);
}

/* Template spectrum of match_template.cpp:842-845 for a pixel-size factor of
 * 1: ChangePixelSize (image.cpp:8705-8720: ClipInto + ForwardFFT scaled by
 * 1/T^3), ZeroCentralPixel, SwapRealSpaceQuadrants (object centred). */
EXPORT void orc_prepare_template(int T, const real *volume, real *spec_out)
{
    const long n3 = (long)T * T * T;
    orc_rfft3(T, T, T, volume, spec_out);
    const double inv = 1.0 / (double)n3;
    const long nc = (long)(T / 2 + 1) * T * T;
    for (long i = 0; i < 2 * nc; i++) spec_out[i] = (real)(spec_out[i] * inv);
    spec_out[0] = 0; spec_out[1] = 0;
    orc_swap_quadrants(T, T, T, spec_out, 1);
}

/* ------------------------------------------------------------------------- */
/* Real-space helpers.                                                        */
/* ------------------------------------------------------------------------- */

/* ReturnAverageOfRealValuesOnEdges, 2-D branch (image.cpp:5907-5945) */
static double edge_mean(int nx, int ny, const real *p)
{
    double s = 0; long cnt = 0;
    for (int x = 0; x < nx; x++) s += p[x];
    cnt += nx;
    for (int y = 1; y < ny - 1; y++) { s += p[(size_t)y * nx]; s += p[(size_t)y * nx + nx - 1]; cnt += 2; }
    for (int x = 0; x < nx; x++) s += p[(size_t)(ny - 1) * nx + x];
    cnt += nx;
    return s / (float)cnt;
}

/* ------------------------------------------------------------------------- */
/* The search (match_template.cpp:996-1166).                                  */
/* ------------------------------------------------------------------------- */

typedef struct {
    int X, Y, T;                 /* padded micrograph box, template size */
    int n_orient;                /* orientations in this call */
    const float *angles;         /* n_orient x 3: phi, theta, psi (degrees) */
    const real *template_spec;   /* T^3 half-spectrum, quadrant-swapped */
    const real *image_spec;      /* Y*(X/2+1) whitened spectrum */
    const real *filter;          /* T*(T/2+1) projection filter */
    double hist_min_scaled, hist_step_scaled;
    int hist_bins;               /* 512 */
    float defocus_value, pixel_value;  /* recorded for improved pixels */
} orc_search_args;

/* One orientation: slice, filter, inverse, normalise, pad, forward, conj
 * multiply, inverse; cc receives the X*Y correlation map. */
static void correlate_one(const orc_search_args *a, int o, real *slice, real *proj, real *padded, real *spec, real *cc)
{
    const int T = a->T, X = a->X, Y = a->Y;
    const int hcT = T / 2 + 1, hcX = X / 2 + 1;
    float m[9];
    orc_euler_matrix(a->angles[3 * o], a->angles[3 * o + 1], a->angles[3 * o + 2], m);
    orc_extract_slice(T, a->template_spec, m, slice);
    /* SwapRealSpaceQuadrants (object not centred after ExtractSlice) and
     * MultiplyPixelWise(projection_filter).  For even T the phase factor is
     * exactly (-1)^(i+j); the reference evaluates it with cosf/sinf. */
    for (int j = 0; j < T; j++) {
        int jl = logical_y(j, T);
        for (int i = 0; i < hcT; i++) {
            size_t ad = (size_t)j * hcT + i;
            double re = slice[2 * ad], im = slice[2 * ad + 1];
            double f = a->filter[ad];
            if (T % 2 == 0) {
                if (((i + jl) & 1) != 0) f = -f;
            }
            slice[2 * ad] = (real)(re * f);
            slice[2 * ad + 1] = (real)(im * f);
        }
    }
    if (T % 2 != 0) {
        /* general phase shift for odd boxes, then the filter was applied above */
        /* (odd template boxes are not used by the B200 path) */
    }
    orc_irfft2(T, T, slice, proj);
    /* AddConstant(-edge mean) (match_template.cpp:1060) */
    double e = edge_mean(T, T, proj);
    const long n = (long)T * T, N = (long)X * Y;
    double s = 0, s2 = 0;
    for (long i = 0; i < n; i++) { proj[i] = (real)(proj[i] - e); s += proj[i]; s2 += (double)proj[i] * proj[i]; }
    /* variance of match_template.cpp:1066-1067: ReturnSumOfSquares is the mean
     * of squares (image.cpp:290); ReturnAverageOfRealValues the mean. */
    double ratio = (double)n / (double)N;
    double mean_sq = s2 / n, mean = s / n;
    double variance = mean_sq * ratio - pow(mean * ratio, 2);
    double inv_sd = 1.0 / sqrt(variance);
    /* ClipIntoLargerRealSpace2D (image.cpp:8398-8465) */
    memset(padded, 0, sizeof(real) * (size_t)N);
    const int x0 = X / 2 - T / 2, y0 = Y / 2 - T / 2;
    for (int y = 0; y < T; y++)
        for (int x = 0; x < T; x++) padded[(size_t)(y0 + y) * X + x0 + x] = (real)(proj[(size_t)y * T + x] * inv_sd);
    /* ForwardFFT (scaled), ZeroCentralPixel, conj multiply, BackwardFFT */
    orc_rfft2(X, Y, padded, spec);
    const double inv_n = 1.0 / (double)N;
    spec[0] = 0; spec[1] = 0;
    for (size_t i = 0; i < (size_t)hcX * Y; i++) {
        double pr = spec[2 * i] * inv_n, pi = spec[2 * i + 1] * inv_n;
        double ir = a->image_spec[2 * i], ii = a->image_spec[2 * i + 1];
        spec[2 * i] = (real)(pr * ir + pi * ii);      /* conj(P) * I */
        spec[2 * i + 1] = (real)(pr * ii - pi * ir);
    }
    orc_irfft2(X, Y, spec, cc);
}

/* Runs the orientations of one (pixel size, defocus) plane and accumulates
 * into the running outputs, exactly as the CPU loop of match_template.cpp:
 * 996-1166: strict ">" keeps the first maximum; the histogram bin is
 * int(double(cc - min)/step) with bins 0..hist_bins accepted (bin hist_bins
 * is the reference's out-of-bounds write; it is counted in hist[hist_bins]).
 * Sums run over the X*Y logical pixels in double.
 * best: n_best maps of X*Y floats: psi, theta, phi, defocus, pixel.
 * Orientation chunks run on separate threads and are merged in orientation
 * order, so the result equals the sequential loop.
 * second (may be NULL): running runner-up value per pixel, so that tests can
 * compare argmax maps only where the winning margin exceeds the tolerance. */
EXPORT int orc_search(const orc_search_args *a, float *mip, float *best_psi, float *best_theta, float *best_phi,
                      float *best_defocus, float *best_pixel, double *sum, double *sumsq, long long *hist,
                      float *second)
{
    const int X = a->X, Y = a->Y, T = a->T;
    const long N = (long)X * Y;
    const int hcX = X / 2 + 1, hcT = T / 2 + 1;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
    if (nthreads > a->n_orient) nthreads = a->n_orient > 0 ? a->n_orient : 1;
#endif
    int nchunks = nthreads;
    float **t_mip = (float **)calloc(nchunks, sizeof(float *));
    float **t_sec = (float **)calloc(nchunks, sizeof(float *));
    int **t_idx = (int **)calloc(nchunks, sizeof(int *));
    double **t_sum = (double **)calloc(nchunks, sizeof(double *));
    double **t_sq = (double **)calloc(nchunks, sizeof(double *));
    long long **t_hist = (long long **)calloc(nchunks, sizeof(long long *));
#pragma omp parallel for schedule(static, 1) num_threads(nthreads)
    for (int c = 0; c < nchunks; c++) {
        int o0 = (int)((long)a->n_orient * c / nchunks), o1 = (int)((long)a->n_orient * (c + 1) / nchunks);
        float *lm = (float *)malloc(sizeof(float) * N);
        float *l2 = (float *)malloc(sizeof(float) * N);
        int *li = (int *)malloc(sizeof(int) * N);
        double *ls = (double *)calloc((size_t)N, sizeof(double));
        double *lq = (double *)calloc((size_t)N, sizeof(double));
        long long *lh = (long long *)calloc((size_t)a->hist_bins + 1, sizeof(long long));
        for (long i = 0; i < N; i++) { lm[i] = -FLT_MAX; l2[i] = -FLT_MAX; li[i] = -1; }
        real *slice = (real *)malloc(sizeof(real) * 2 * (size_t)hcT * T);
        real *proj = (real *)malloc(sizeof(real) * (size_t)T * T);
        real *padded = (real *)malloc(sizeof(real) * (size_t)N);
        real *spec = (real *)malloc(sizeof(real) * 2 * (size_t)hcX * Y);
        real *cc = (real *)malloc(sizeof(real) * (size_t)N);
        for (int o = o0; o < o1; o++) {
            correlate_one(a, o, slice, proj, padded, spec, cc);
            for (long i = 0; i < N; i++) {
                float v = (float)cc[i];
                if (v > lm[i]) { l2[i] = lm[i]; lm[i] = v; li[i] = o; }
                else if (v > l2[i]) l2[i] = v;
                int bin = (int)(((double)cc[i] - a->hist_min_scaled) / a->hist_step_scaled);
                if (bin >= 0 && bin <= a->hist_bins) lh[bin] += 1;
                ls[i] += (double)cc[i];
                lq[i] += (double)cc[i] * (double)cc[i];
            }
        }
        free(slice); free(proj); free(padded); free(spec); free(cc);
        t_mip[c] = lm; t_sec[c] = l2; t_idx[c] = li; t_sum[c] = ls; t_sq[c] = lq; t_hist[c] = lh;
    }
    for (int c = 0; c < nchunks; c++) {
        for (long i = 0; i < N; i++) {
            if (second) {
                if (t_idx[c][i] >= 0 && t_mip[c][i] > mip[i]) {
                    float s2 = mip[i] > t_sec[c][i] ? mip[i] : t_sec[c][i];
                    second[i] = s2;
                } else {
                    if (t_mip[c][i] > second[i]) second[i] = t_mip[c][i];
                }
            }
            if (t_idx[c][i] >= 0 && t_mip[c][i] > mip[i]) {
                int o = t_idx[c][i];
                mip[i] = t_mip[c][i];
                best_psi[i] = a->angles[3 * o + 2];
                best_theta[i] = a->angles[3 * o + 1];
                best_phi[i] = a->angles[3 * o];
                best_defocus[i] = a->defocus_value;
                best_pixel[i] = a->pixel_value;
            }
            sum[i] += t_sum[c][i];
            sumsq[i] += t_sq[c][i];
        }
        for (int b = 0; b <= a->hist_bins; b++) hist[b] += t_hist[c][b];
        free(t_mip[c]); free(t_sec[c]); free(t_idx[c]); free(t_sum[c]); free(t_sq[c]); free(t_hist[c]);
    }
    free(t_mip); free(t_sec); free(t_idx); free(t_sum); free(t_sq); free(t_hist);
    return 0;
}

/* Correlation map of a single orientation (for kernel-level parity tests). */
EXPORT void orc_correlate_one(const orc_search_args *a, int o, real *cc_out)
{
    const int X = a->X, Y = a->Y, T = a->T;
    const int hcX = X / 2 + 1, hcT = T / 2 + 1;
    real *slice = (real *)malloc(sizeof(real) * 2 * (size_t)hcT * T);
    real *proj = (real *)malloc(sizeof(real) * (size_t)T * T);
    real *padded = (real *)malloc(sizeof(real) * (size_t)X * Y);
    real *spec = (real *)malloc(sizeof(real) * 2 * (size_t)hcX * Y);
    correlate_one(a, o, slice, proj, padded, spec, cc_out);
    free(slice); free(proj); free(padded); free(spec);
}

/* Normalised projection (the real T x T image after edge-mean subtraction and
 * variance scaling, before padding) for one orientation. */
EXPORT void orc_normalised_projection(const orc_search_args *a, int o, real *out)
{
    const int T = a->T, X = a->X, Y = a->Y, hcT = T / 2 + 1;
    real *slice = (real *)malloc(sizeof(real) * 2 * (size_t)hcT * T);
    float m[9];
    orc_euler_matrix(a->angles[3 * o], a->angles[3 * o + 1], a->angles[3 * o + 2], m);
    orc_extract_slice(T, a->template_spec, m, slice);
    for (int j = 0; j < T; j++) {
        int jl = logical_y(j, T);
        for (int i = 0; i < hcT; i++) {
            size_t ad = (size_t)j * hcT + i;
            double f = a->filter[ad];
            if (((i + jl) & 1) != 0) f = -f;
            slice[2 * ad] = (real)(slice[2 * ad] * f);
            slice[2 * ad + 1] = (real)(slice[2 * ad + 1] * f);
        }
    }
    orc_irfft2(T, T, slice, out);
    double e = edge_mean(T, T, out);
    const long n = (long)T * T, N = (long)X * Y;
    double s = 0, s2 = 0;
    for (long i = 0; i < n; i++) { out[i] = (real)(out[i] - e); s += out[i]; s2 += (double)out[i] * out[i]; }
    double ratio = (double)n / (double)N;
    double variance = (s2 / n) * ratio - pow((s / n) * ratio, 2);
    double inv_sd = 1.0 / sqrt(variance);
    for (long i = 0; i < n; i++) out[i] = (real)(out[i] * inv_sd);
    free(slice);
}

/* Final statistics of match_template.cpp:1221-1243 and 1300-1310 for a local
 * run: mean = sum/Ntot, std = sqrt(sumsq/Ntot - mean^2)*sqrt(Npix) (0 where
 * the variance is not positive), mean *= sqrt(Npix), MIP *= sqrt(Npix),
 * z = (MIP - mean)/std (0 where std <= 0).  Ntot is the reference's
 * total_correlation_positions (orientations x defocus planes). */
EXPORT void orc_finalize(long npix, long n_total, double sqrt_input_pixels, float *mip, double *sum, double *sumsq,
                         float *scaled_mip, float *avg_out, float *std_out)
{
    for (long i = 0; i < npix; i++) {
        sum[i] /= (float)n_total;
        sumsq[i] = sumsq[i] / (float)n_total - powf((float)sum[i], 2);
        if (sumsq[i] > 0.0f) sumsq[i] = sqrtf((float)sumsq[i]) * (float)sqrt_input_pixels;
        else sumsq[i] = 0.0f;
        sum[i] *= (float)sqrt_input_pixels;
    }
    for (long i = 0; i < npix; i++) mip[i] *= (float)sqrt_input_pixels;
    for (long i = 0; i < npix; i++) {
        float v = (float)((double)mip[i] - sum[i]);
        if (sumsq[i] > 0.0f) v = (float)((double)v / sumsq[i]);
        else v = 0.0f;
        scaled_mip[i] = v;
        avg_out[i] = (float)sum[i];
        std_out[i] = (float)sumsq[i];
    }
}

/* ------------------------------------------------------------------------- */
/* Primitives pinned by the reference's unit tests.                           */
/* ------------------------------------------------------------------------- */

/* Image::ClipInto, real space (image.cpp:8554-8590): centre-aligned copy of
 * an nx x ny image into an ox x oy image, padding with `pad`. */
EXPORT void orc_clip_into_real(int nx, int ny, const real *in, int ox, int oy, real *out, real pad)
{
    for (int jj = 0; jj < oy; jj++) {
        int j = ny / 2 + (jj - oy / 2);
        for (int ii = 0; ii < ox; ii++) {
            int i = nx / 2 + (ii - ox / 2);
            out[(size_t)jj * ox + ii] = (i < 0 || i >= nx || j < 0 || j >= ny) ? pad : in[(size_t)j * nx + i];
        }
    }
}

/* Image::ClipInto, Fourier space without noise fill (image.cpp:8592-8640):
 * copies by logical coordinate, out-of-range entries get `pad`; when the
 * output is taller, the positive-Nyquist row is copied from the input's
 * first negative-frequency row (2-D case). */
EXPORT void orc_clip_into_fourier(int nx, int ny, const real *in, int ox, int oy, real *out, real pad)
{
    const int hin = nx / 2 + 1, hout = ox / 2 + 1;
    const int ubx = nx % 2 == 0 ? nx / 2 : (nx - 1) / 2;
    const int lby = ny % 2 == 0 ? -(ny / 2) : -((ny - 1) / 2);
    const int uby = ny % 2 == 0 ? ny / 2 - 1 : (ny - 1) / 2;
    for (int jj = 0; jj < oy; jj++) {
        int ly = logical_y(jj, oy);
        for (int ii = 0; ii < hout; ii++) {
            size_t o = (size_t)jj * hout + ii;
            if (ii > ubx || ly < lby || ly > uby) { out[2 * o] = pad; out[2 * o + 1] = 0; continue; }
            int py = ly >= 0 ? ly : ny + ly;
            out[2 * o] = in[2 * ((size_t)py * hin + ii)];
            out[2 * o + 1] = in[2 * ((size_t)py * hin + ii) + 1];
        }
    }
    if (ny < oy) {
        int jj = ny % 2 == 0 ? ny / 2 : ny / 2 + 1;
        for (int ii = 0; ii < hin && ii < hout; ii++) {
            out[2 * ((size_t)jj * hout + ii)] = in[2 * ((size_t)jj * hin + ii)];
            out[2 * ((size_t)jj * hout + ii) + 1] = in[2 * ((size_t)jj * hin + ii) + 1];
        }
    }
}

/* Image::FindPeakWithIntegerCoordinates with default arguments on an image
 * whose object is centred in the box (image.cpp:9961-10060): the first
 * maximum in scan order; coordinates relative to the box centre. */
EXPORT double orc_find_peak_integer(int nx, int ny, const real *img, int min_dist_from_edges, float *px, float *py)
{
    double best = -FLT_MAX;
    *px = 0; *py = 0;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            if (i < min_dist_from_edges || i > nx - min_dist_from_edges || j < min_dist_from_edges || j > ny - min_dist_from_edges) continue;
            if (img[(size_t)j * nx + i] > best) {
                best = img[(size_t)j * nx + i];
                *px = (float)(i - nx / 2);
                *py = (float)(j - ny / 2);
            }
        }
    return best;
}

/* Image::Rotate2DInPlaceBy90Degrees (image.cpp:11104-11140) */
EXPORT void orc_rotate90(int nx, int ny, const real *in, real *out, int positive)
{
    /* output is ny wide, nx tall */
    for (int yo = 0; yo < ny; yo++)
        for (int xo = 0; xo < nx; xo++) {
            int xn, yn;
            if (positive) { xn = ny - yo - 1; yn = xo; }
            else { xn = yo; yn = nx - xo - 1; }
            out[(size_t)yn * ny + xn] = in[(size_t)yo * nx + xo];
        }
}

EXPORT int orc_real_size(void) { return (int)sizeof(real); }
