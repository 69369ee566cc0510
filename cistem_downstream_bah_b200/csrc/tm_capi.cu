// tm_capi.cu -- C ABI of the B200 search core (declared in include/tm_b200.h).
//
// Owns all device memory of a search context, prepares the micrograph spectrum
// once, and drives one (pixel size, defocus) plane as a sequence of
// orientation batches: six kernels per batch on one stream, no host
// synchronisation inside a plane.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <thread>
#include <vector>

#include "../../include/tm_b200.h"
#include "tm_kernels.cuh"
#include "tm_whiten.cuh"
#include "tm_template.cuh"
#include "tm_generic.cuh"

namespace tmcg {
#include "tm_gemm.cuh"
}  // namespace tmcg

#define TM_VERSION "tm_b200 0.1 (sm_100a, fp32 search path)"

namespace {

struct Plane {
    long long base;       // global index of the plane's first orientation
    int n;                // orientations in the plane
    int angles_id;        // index into angle_lists
    float defocus, pixel;
};

struct Variant;

}  // namespace

struct tm_ctx {
    tm_dims d{};
    int X = 0, Y = 0, T = 0, XP = 0, TP = 0, B = 0;
    int Bcap = 0;   // orientation capacity of the batch buffers (B <= Bcap)
    int device = 0, nsm = 0;
    const Variant* var = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_prep = nullptr, ev_b = nullptr, ev_c = nullptr, ev_end = nullptr;
    cudaEvent_t ev_batch[2][4] = {};   // first / last batch of a plane: begin, after prep, pass B, pass C
    // device buffers
    float2 *tmpl = nullptr, *Ip = nullptr, *S = nullptr, *A = nullptr, *C = nullptr, *norm = nullptr;
    float2 *twx = nullptr, *twy = nullptr, *twt = nullptr;   // twiddle tables of the x, y and template lengths
    float *P = nullptr, *filter = nullptr, *rot = nullptr;
    double* rowstat = nullptr;
    float* mip = nullptr;
    int* best = nullptr;
    double *sum = nullptr, *sumsq = nullptr;
    unsigned long long* hist = nullptr;
    int* err_flag = nullptr;
    int* best_host = nullptr;   // page-locked copy of the best-orientation map (tm_get_results)
    int precision = TM_PRECISION_FP32;
    tmk::GenPlan gen_px{}, gen_py{}, gen_ph{};   // radix plans of X, Y and X/2 (sizes without compiled kernels)
    uint4* dft = nullptr;       // DFT operands of the tensor-core row pass (FP16 form)
    long long rot_capacity = 0;
    bool has_template = false, has_image = false;
    // bookkeeping for decoding the argmax
    std::vector<Plane> planes;
    std::vector<std::vector<float>> angle_lists;
    long long next_gidx = 0;
    long long n_ccs = 0;
    long long norm_pixels = 0;   // projection variance pixel count override (0: X*Y)
    // image set (tm_set_image_set): per image its prepared spectrum and running results
    struct Slot {
        float2* Ip = nullptr;
        float* mip = nullptr;
        int* best = nullptr;
        double *sum = nullptr, *sumsq = nullptr;
        unsigned long long* hist = nullptr;
    };
    std::vector<Slot> slots;
    double last_total_ms = 0, last_b_ms = 0, last_c_ms = 0, last_prep_ms = 0;
    std::string err;
};

namespace {

int set_err(tm_ctx* c, int code, const char* fmt, ...) {
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

#define TM_CUDA(ctx, call)                                                                              \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return set_err((ctx), e_ == cudaErrorMemoryAllocation ? TM_ERR_OOM : TM_ERR_CUDA, "%s: %s (%s:%d)", \
                           #call, cudaGetErrorString(e_), __FILE__, __LINE__);                         \
    } while (0)

// ---------------------------------------------------------------------------------------------
// Kernel variants per geometry.

// Device whitening of an X x Y micrograph into its half spectrum (tm_whiten.cuh).
struct WhitenBuffers {
    const float* img;     // X * Y reals
    float2* spec;         // Y * (X/2+1)
    double* scratch;      // 3 + 3 * npts doubles
    float* xs;            // npts abscissae
    tmfft::Twiddles twx, twy;
    int X, Y;             // sizes (read by the run-time-length whitening)
};
using WhitenFn = int (*)(cudaStream_t, int nsm, const WhitenBuffers&, std::vector<double>& curve, std::string& err);

// The FP16 tensor-core form of a geometry (tm_set_precision).
struct TensorForm {
    int (*configure)(tm_ctx*);
    int (*run_batch)(tm_ctx*, tmk::BatchArgs&, cudaEvent_t* ev);
    size_t dft_bytes;                 // the row pass's DFT operands
    void (*fill_dft)(uint16_t*);
};

struct Variant {
    int T, X, Y;
    int W;   // row pitch alignment of the pass-B column chunks (columns)
    int (*run_batch)(tm_ctx*, tmk::BatchArgs&, cudaEvent_t* ev);   // ev: 4 events to record (or null)
    int (*configure)(tm_ctx*);
    int (*run_stages)(tm_ctx*, tmk::BatchArgs&);   // every kernel before the MIP epilogue
    WhitenFn whiten;
    int (*run_batch_images)(tm_ctx*, tmk::BatchArgs&, const int* ids, int n_ids);   // image-set batch
    const TensorForm* tc;   // null where the FP16 tensor-core form has no kernels
};

// number of points of the whitening curve (match_template.cpp:702)
int curve_points(int X) { return (int)((X / 2.0 + 1.0) * sqrtf(2.0f) + 1.0); }

#define TW_CHECK(call)                                                               \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);                \
            return e_ == cudaErrorMemoryAllocation ? TM_ERR_OOM : TM_ERR_CUDA;      \
        }                                                                            \
    } while (0)

// The whitening steps around the two transforms; `transforms(mean, vmin, vmax)`
// launches the row r2c and the column FFT with the quadrant swap.
template <class Transforms>
int whiten_steps(cudaStream_t s, int nsm, const WhitenBuffers& b, int X, int Y, std::vector<double>& curve,
                 std::string& err, Transforms transforms) {
    const int hc = X / 2 + 1;
    const long long n = (long long)X * Y;
    const int npts = curve_points(X);
    double* stats = b.scratch;                 // sum, sum of squares, whitened sum of squares
    double* pw = b.scratch + 3;
    double* cnt = pw + npts;
    double* wf = cnt + npts;
    TW_CHECK(cudaMemsetAsync(b.scratch, 0, sizeof(double) * (3 + 2 * (size_t)npts), s));
    tmw::k_w_stats<<<nsm * 4, 256, 0, s>>>(b.img, n, stats);
    TW_CHECK(cudaGetLastError());
    double st[2];
    TW_CHECK(cudaMemcpyAsync(st, stats, sizeof st, cudaMemcpyDeviceToHost, s));
    TW_CHECK(cudaStreamSynchronize(s));
    // ReplaceOutliersWithMean(5) (image.cpp:986-1007), float as the host restatement forms it
    const float mean = (float)(st[0] / n);
    const float sigma = sqrtf(fabsf((float)(st[1] / n - (st[0] / n) * (st[0] / n))));
    const float vmax = mean + 5.0f * sigma, vmin = mean - 5.0f * sigma;
    TW_CHECK(transforms(mean, vmin, vmax));
    // the curve's abscissae (Curve::SetupXAxis(0, sqrt(2)/2, npts)), float
    const float hi = 0.5f * sqrtf(2.0f);
    std::vector<float> xs(npts);
    for (int i = 0; i < npts; i++) xs[i] = i * (hi - 0.0f) / (float)(npts - 1) + 0.0f;
    TW_CHECK(cudaMemcpyAsync(b.xs, xs.data(), sizeof(float) * npts, cudaMemcpyHostToDevice, s));
    tmw::CurveArgs ca{b.xs, npts, xs[0], xs[1]};
    const int curve_smem = (int)(2 * sizeof(double) * npts);
    if (curve_smem > 48 * 1024)
        TW_CHECK(cudaFuncSetAttribute(tmw::k_w_curve, cudaFuncAttributeMaxDynamicSharedMemorySize, curve_smem));
    tmw::k_w_curve<<<nsm * 2, 256, curve_smem, s>>>(b.spec, X, Y, ca, pw, cnt);
    TW_CHECK(cudaGetLastError());
    std::vector<double> hpw(npts), hcnt(npts);
    TW_CHECK(cudaMemcpyAsync(hpw.data(), pw, sizeof(double) * npts, cudaMemcpyDeviceToHost, s));
    TW_CHECK(cudaMemcpyAsync(hcnt.data(), cnt, sizeof(double) * npts, cudaMemcpyDeviceToHost, s));
    TW_CHECK(cudaStreamSynchronize(s));
    // SquareRoot, Reciprocal, MultiplyByConstant(1 / max) (match_template.cpp:716-718)
    curve.assign(npts, 0.0);
    double mx = -DBL_MAX;
    for (int i = 0; i < npts; i++) {
        double v = hcnt[i] > 0 ? hpw[i] / hcnt[i] : 0.0;
        v = sqrt(v);
        if (v != 0.0) v = 1.0 / v;
        curve[i] = v;
        mx = std::max(mx, v);
    }
    for (double& v : curve) v *= 1.0 / mx;
    TW_CHECK(cudaMemcpyAsync(wf, curve.data(), sizeof(double) * npts, cudaMemcpyHostToDevice, s));
    tmw::k_w_apply<<<nsm * 4, 256, 0, s>>>(b.spec, X, Y, ca, wf, stats + 2);
    TW_CHECK(cudaGetLastError());
    tmw::k_w_scale<<<nsm * 4, 256, 0, s>>>(b.spec, (long long)Y * hc, stats + 2);
    TW_CHECK(cudaGetLastError());
    TW_CHECK(cudaStreamSynchronize(s));
    return TM_OK;
}

template <int X, int Y>
int whiten_on_device(cudaStream_t s, int nsm, const WhitenBuffers& b, std::vector<double>& curve, std::string& err) {
    return whiten_steps(s, nsm, b, X, Y, curve, err, [&](float mean, float vmin, float vmax) {
        using R = tmw::WRows<X>;
        using C = tmw::WCols<Y>;
        constexpr int hc = X / 2 + 1;
        tmw::k_w_rows<X><<<(Y + R::ROWS - 1) / R::ROWS, R::NT, 0, s>>>(b.img, b.spec, Y, mean, vmin, vmax, b.twx);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (C::SMEM > 48 * 1024) {
            e = cudaFuncSetAttribute(tmw::k_w_cols<Y>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
            if (e != cudaSuccess) return e;
        }
        tmw::k_w_cols<Y><<<(hc + C::CB - 1) / C::CB, C::NT, C::SMEM, s>>>(b.spec, X, b.twy);
        return cudaGetLastError();
    });
}

// any size whose sides have radix plans (tm_generic.cuh)
int whiten_generic(cudaStream_t s, int nsm, const WhitenBuffers& b, std::vector<double>& curve, std::string& err) {
    const int X = b.X, Y = b.Y;
    const bool odd = X % 2 != 0;
    tmk::GenPlan ph, py;
    if (!tmk::gen_plan(odd ? X : X / 2, ph) || !tmk::gen_plan(Y, py)) {
        err = "no radix plan for the micrograph size";
        return TM_ERR_UNSUPPORTED;
    }
    return whiten_steps(s, nsm, b, X, Y, curve, err, [&](float mean, float vmin, float vmax) {
        const int smem_r = (int)sizeof(float2) * 2 * ph.L, smem_c = (int)sizeof(float2) * 2 * Y;
        auto rows = odd ? tmk::k_w_rows_gen<true> : tmk::k_w_rows_gen<false>;
        cudaError_t e = cudaFuncSetAttribute(rows, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_r);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(tmk::k_w_cols_gen, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_c);
        if (e != cudaSuccess) return e;
        rows<<<Y, tmk::kGenNT, smem_r, s>>>(b.img, b.spec, X, mean, vmin, vmax, b.twx, ph);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        tmk::k_w_cols_gen<<<X / 2 + 1, tmk::kGenNT, smem_c, s>>>(b.spec, X, Y, b.twy, py);
        return cudaGetLastError();
    });
}

template <int T, int X, int Y>
struct Impl {
    using LN = tmk::Launch<T, X, Y>;

    static int configure(tm_ctx* c) {
        TM_CUDA(c, LN::configure(c->XP, c->d.histogram_bins));
        return TM_OK;
    }

    static int run_stages(tm_ctx* c, tmk::BatchArgs& a) {
        LN::prep(a, c->stream);
        LN::pass_b(a, c->stream, c->nsm);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return set_err(c, TM_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
        return TM_OK;
    }

    // one orientation batch over several images of the image set: the slice,
    // projection, normalisation and row transforms once, then passes B and C
    // per image (they reuse the correlation buffer in stream order)
    static int run_batch_images(tm_ctx* c, tmk::BatchArgs& a, const int* ids, int n_ids) {
        cudaStream_t s = c->stream;
        LN::prep(a, s);
        for (int k = 0; k < n_ids; k++) {
            const tm_ctx::Slot& sl = c->slots[ids[k]];
            a.Ip = sl.Ip;
            a.mip = sl.mip;
            a.best = sl.best;
            a.sum = sl.sum;
            a.sumsq = sl.sumsq;
            a.hist = sl.hist;
            LN::pass_b(a, s, c->nsm);
            LN::pass_c(a, s);
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return set_err(c, TM_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
        return TM_OK;
    }

    static int run_batch(tm_ctx* c, tmk::BatchArgs& a, cudaEvent_t* ev) {
        cudaStream_t s = c->stream;
        if (ev) cudaEventRecord(ev[0], s);
        LN::prep(a, s);
        if (ev) cudaEventRecord(ev[1], s);
        LN::pass_b(a, s, c->nsm);
        if (ev) cudaEventRecord(ev[2], s);
        LN::pass_c(a, s);
        if (ev) cudaEventRecord(ev[3], s);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return set_err(c, TM_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
        return TM_OK;
    }
};

template <int T, int X, int Y>
struct TcImpl {
    using LT = tmk::LaunchTc<T, X, Y>;
    static int configure(tm_ctx* c) {
        TM_CUDA(c, LT::configure(c->XP, c->d.histogram_bins));
        return TM_OK;
    }
    // the FP16 form of a batch: the same slice and projection kernels, pass B
    // with FP16 output, the tensor-core row pass
    static int run_batch(tm_ctx* c, tmk::BatchArgs& a, cudaEvent_t* ev) {
        using LN = tmk::Launch<T, X, Y>;
        cudaStream_t s = c->stream;
        if (ev) cudaEventRecord(ev[0], s);
        LN::prep(a, s);
        if (ev) cudaEventRecord(ev[1], s);
        LT::pass_b(a, s, c->nsm, c->dft);
        if (ev) cudaEventRecord(ev[2], s);
        LT::pass_c(a, s, c->dft);
        if (ev) cudaEventRecord(ev[3], s);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return set_err(c, TM_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
        return TM_OK;
    }
    static constexpr TensorForm form = {&TcImpl::configure, &TcImpl::run_batch, LT::dft_bytes, &LT::fill_dft};
};

// Sizes without compiled kernels: the slice and projection kernels of the
// template box T and the run-time-length passes of tm_generic.cuh.
template <int T>
struct GenImpl {
    static int configure(tm_ctx* c) {
        TM_CUDA(c, cudaFuncSetAttribute(tmk::k_pass_a_gen<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sizeof(float2) * 2 * c->X));
        const int lw = tmk::gen_pass_b_lines(c->Y);
        TM_CUDA(c, cudaFuncSetAttribute(lw == 4 ? tmk::k_pass_b_gen<4> : lw == 2 ? tmk::k_pass_b_gen<2> : tmk::k_pass_b_gen<1>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(float2) * 2 * lw * c->Y));
        const int smem_c = (int)sizeof(float2) * (c->X % 2 ? 2 * c->X : c->X) + 4 * c->d.histogram_bins;
        TM_CUDA(c, cudaFuncSetAttribute(pass_c_kernel(c->X), cudaFuncAttributeMaxDynamicSharedMemorySize, smem_c));
        return TM_OK;
    }
    // the row pass for a width X: odd or even rows, 4, 8 or 16 pixels per thread
    static auto pass_c_kernel(int X) -> void (*)(tmk::BatchArgs, int, int, tmk::GenPlan) {
        const int mp = X <= 4 * tmk::kGenNT ? 4 : X <= 8 * tmk::kGenNT ? 8 : 16;
        if (X % 2) return mp == 4 ? tmk::k_pass_c_gen<true, 4> : mp == 8 ? tmk::k_pass_c_gen<true, 8> : tmk::k_pass_c_gen<true, 16>;
        return mp == 4 ? tmk::k_pass_c_gen<false, 4> : mp == 8 ? tmk::k_pass_c_gen<false, 8> : tmk::k_pass_c_gen<false, 16>;
    }
    static void prep(tm_ctx* c, tmk::BatchArgs& a, cudaStream_t s) {
        using SC = tmk::SliceCol<T>;
        using RC = tmk::RowC2R<T>;
        tmk::k_slice_colfft<T><<<dim3((T / 2 + 1 + SC::CB - 1) / SC::CB, a.nb), SC::NT, 0, s>>>(a);
        tmk::k_row_c2r<T><<<dim3(T / RC::ROWS, a.nb), RC::NT, 0, s>>>(a);
        tmk::k_norm<T><<<(a.nb + 7) / 8, 256, 0, s>>>(a, a.norm_pixels > 0 ? a.norm_pixels : (long long)c->X * c->Y);
        tmk::k_pass_a_gen<T><<<dim3(T, a.nb), tmk::kGenNT, sizeof(float2) * 2 * c->X, s>>>(a, c->X, c->gen_px);
    }
    static void pass_b(tm_ctx* c, tmk::BatchArgs& a, cudaStream_t s) {
        // the row pitch XP is a multiple of 4 columns (the variant's pass-B width)
        const int lw = tmk::gen_pass_b_lines(c->Y);
        const size_t smem = sizeof(float2) * 2 * lw * c->Y;
        if (lw == 4) tmk::k_pass_b_gen<4><<<dim3(a.XP / 4, a.nb), tmk::kGenNT, smem, s>>>(a, T, c->Y, c->gen_py);
        else if (lw == 2) tmk::k_pass_b_gen<2><<<dim3(a.XP / 2, a.nb), tmk::kGenNT, smem, s>>>(a, T, c->Y, c->gen_py);
        else tmk::k_pass_b_gen<1><<<dim3(a.XP, a.nb), tmk::kGenNT, smem, s>>>(a, T, c->Y, c->gen_py);
    }
    static void pass_c(tm_ctx* c, tmk::BatchArgs& a, cudaStream_t s) {
        const size_t smem = sizeof(float2) * (c->X % 2 ? 2 * c->X : c->X) + 4 * a.hist_bins;
        pass_c_kernel(c->X)<<<c->Y, tmk::kGenNT, smem, s>>>(a, c->X, c->Y, c->gen_ph);
    }
    static int done(tm_ctx* c) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return set_err(c, TM_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
        return TM_OK;
    }
    static int run_stages(tm_ctx* c, tmk::BatchArgs& a) {
        prep(c, a, c->stream);
        pass_b(c, a, c->stream);
        return done(c);
    }
    static int run_batch(tm_ctx* c, tmk::BatchArgs& a, cudaEvent_t* ev) {
        cudaStream_t s = c->stream;
        if (ev) cudaEventRecord(ev[0], s);
        prep(c, a, s);
        if (ev) cudaEventRecord(ev[1], s);
        pass_b(c, a, s);
        if (ev) cudaEventRecord(ev[2], s);
        pass_c(c, a, s);
        if (ev) cudaEventRecord(ev[3], s);
        return done(c);
    }
    static int run_batch_images(tm_ctx* c, tmk::BatchArgs& a, const int* ids, int n_ids) {
        prep(c, a, c->stream);
        for (int k = 0; k < n_ids; k++) {
            const tm_ctx::Slot& sl = c->slots[ids[k]];
            a.Ip = sl.Ip;
            a.mip = sl.mip;
            a.best = sl.best;
            a.sum = sl.sum;
            a.sumsq = sl.sumsq;
            a.hist = sl.hist;
            pass_b(c, a, c->stream);
            pass_c(c, a, c->stream);
        }
        return done(c);
    }
};

#define TM_VARIANT(T, X, Y)                                                                                 \
    {T, X, Y, tmk::Launch<T, X, Y>::pass_b_width, &Impl<T, X, Y>::run_batch, &Impl<T, X, Y>::configure,          \
     &Impl<T, X, Y>::run_stages, &whiten_on_device<X, Y>, &Impl<T, X, Y>::run_batch_images, nullptr}
// a geometry that also has the FP16 tensor-core form
#define TM_VARIANT_TC(T, X, Y)                                                                              \
    {T, X, Y, tmk::Launch<T, X, Y>::pass_b_width, &Impl<T, X, Y>::run_batch, &Impl<T, X, Y>::configure,          \
     &Impl<T, X, Y>::run_stages, &whiten_on_device<X, Y>, &Impl<T, X, Y>::run_batch_images, &TcImpl<T, X, Y>::form}

// Geometries with compiled kernels: template box T on a padded X x Y
// micrograph.  X is a power of two (the reference turns a micrograph whose
// padded width is not a power of two but whose height is by 90 degrees,
// match_template.cpp:587-596); Y may carry factors of 3 (3888 = 2^4 3^5 and
// 5832 = 2^3 3^6 are what its factorisation gives for 3710- and 5760-pixel
// sides).  The small 288- and 48-sized geometries exercise the same code paths
// for tests.
const Variant kVariants[] = {
    TM_VARIANT(32, 256, 256),
    TM_VARIANT(32, 512, 256),
    TM_VARIANT(32, 256, 512),
    TM_VARIANT(32, 512, 512),
    TM_VARIANT(64, 512, 512),
    TM_VARIANT_TC(64, 1024, 1024),
    TM_VARIANT_TC(128, 1024, 1024),
    TM_VARIANT_TC(128, 2048, 2048),
    TM_VARIANT_TC(256, 2048, 2048),
    TM_VARIANT_TC(256, 4096, 4096),
    TM_VARIANT_TC(64, 4096, 4096),
    TM_VARIANT(32, 256, 288),
    TM_VARIANT(48, 256, 256),
    TM_VARIANT(48, 256, 288),
    TM_VARIANT_TC(256, 4096, 3888),
    TM_VARIANT(256, 4096, 5832),
    TM_VARIANT_TC(384, 4096, 4096),
    TM_VARIANT(384, 4096, 5832),
    // the same camera formats with smaller and larger templates
    TM_VARIANT_TC(128, 4096, 4096),
    TM_VARIANT_TC(128, 4096, 3888),
    TM_VARIANT(128, 4096, 5832),
    TM_VARIANT_TC(64, 4096, 3888),
    TM_VARIANT(64, 4096, 5832),
    TM_VARIANT_TC(384, 4096, 3888),
    // binned camera formats: K3 at 2x (2880 x 2046 -> 2048 x 2916 rotated), K2 at 2x
    // (1919 x 1855 -> 2048 x 1944), 2560 x 1920 (-> 2048 x 2592), 5120 x 3840 (-> 4096 x 5184)
    TM_VARIANT(256, 2048, 2916),
    TM_VARIANT(128, 2048, 2916),
    TM_VARIANT(256, 2048, 1944),
    TM_VARIANT(256, 2048, 2592),
    TM_VARIANT(256, 4096, 5184),
    // windows of the learned proposal's fine search (edge max(2T, 256))
    TM_VARIANT(64, 256, 256),
    TM_VARIANT(128, 256, 256),
    TM_VARIANT(256, 512, 512),
};

const Variant* find_variant(int T, int X, int Y) {
    for (const Variant& v : kVariants)
        if (v.T == T && v.X == X && v.Y == Y) return &v;
    return nullptr;
}

// the run-time-length variants, one per template box (X = Y = 0: any size with radix plans)
#define TM_GENERIC(T)                                                                                  \
    {T, 0, 0, 4, &GenImpl<T>::run_batch, &GenImpl<T>::configure, &GenImpl<T>::run_stages, &whiten_generic, \
     &GenImpl<T>::run_batch_images, nullptr}
const Variant kGenericVariants[] = {TM_GENERIC(32), TM_GENERIC(48), TM_GENERIC(64), TM_GENERIC(128), TM_GENERIC(256),
                                    TM_GENERIC(384)};

// a size the run-time-length kernels take: sides 64..8192 whose lengths (and the
// half width, when the width is even) have radix plans (prime factors 2, 3, 5,
// 7, 11, 13); ph receives the row pass's plan (X/2, or X when X is odd)
bool generic_size(int X, int Y, tmk::GenPlan* px, tmk::GenPlan* py, tmk::GenPlan* ph) {
    tmk::GenPlan a, b, h;
    if (X < 64 || Y < 64) return false;
    if (!tmk::gen_plan(X, a) || !tmk::gen_plan(Y, b) || !tmk::gen_plan(X % 2 ? X : X / 2, h)) return false;
    if (px) *px = a;
    if (py) *py = b;
    if (ph) *ph = h;
    return true;
}

const Variant* find_generic_variant(int T, int X, int Y) {
    if (!generic_size(X, Y, nullptr, nullptr, nullptr)) return nullptr;
    for (const Variant& v : kGenericVariants)
        if (v.T == T) return &v;
    return nullptr;
}

template <class Tp>
int dalloc(tm_ctx* c, Tp** p, size_t count) {
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(Tp));
    if (e != cudaSuccess) {
        *p = nullptr;
        return set_err(c, e == cudaErrorMemoryAllocation ? TM_ERR_OOM : TM_ERR_CUDA, "cudaMalloc(%zu bytes): %s",
                       count * sizeof(Tp), cudaGetErrorString(e));
    }
    return TM_OK;
}

// Waits for the stream with a time limit; polling keeps the host responsive.
int wait_stream(tm_ctx* c, double limit_s) {
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaStreamQuery(c->stream);
        if (e == cudaSuccess) return TM_OK;
        if (e != cudaErrorNotReady) return set_err(c, TM_ERR_CUDA, "device error: %s", cudaGetErrorString(e));
        double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > limit_s) return set_err(c, TM_ERR_TIMEOUT, "stream did not finish within %.0f s", limit_s);
        // yield for the first milliseconds (a plane's tail), then poll every 20 us
        if (el < 2e-3) std::this_thread::yield();
        else std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

void free_all(tm_ctx* c) {
    void* ptrs[] = {c->tmpl, c->Ip, c->S, c->A, c->C, c->norm, c->twx, c->twy, c->twt, c->P, c->filter, c->rot,
                    c->rowstat, c->mip, c->best, c->sum, c->sumsq, c->hist, c->err_flag, c->dft};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (tm_ctx::Slot& sl : c->slots) {
        void* sp[] = {sl.Ip, sl.mip, sl.best, sl.sum, sl.sumsq, sl.hist};
        for (void* p : sp)
            if (p) cudaFree(p);
    }
    c->slots.clear();
    if (c->best_host) cudaFreeHost(c->best_host);
    if (c->stream) cudaStreamDestroy(c->stream);
    cudaEvent_t evs[] = {c->ev_start, c->ev_prep, c->ev_b, c->ev_c, c->ev_end};
    for (cudaEvent_t e : evs)
        if (e) cudaEventDestroy(e);
    for (auto& set : c->ev_batch)
        for (cudaEvent_t e : set)
            if (e) cudaEventDestroy(e);
}

// The two used columns of RotationMatrix::SetToEulerRotation (matrix.cpp:490-510)
// in float arithmetic, 6 floats per orientation: m00 m01 m10 m11 m20 m21.
void euler_rows(const float* euler_angles, int n, float* rot) {
    const float pif = 3.14159265359f;
    auto d2r = [pif](float deg) { return (float)((double)(deg * pif) / 180.); };
    for (int o = 0; o < n; o++) {
        const float phi = euler_angles[3 * o], theta = euler_angles[3 * o + 1], psi = euler_angles[3 * o + 2];
        const float cphi = cosf(d2r(phi)), sphi = sinf(d2r(phi));
        const float cth = cosf(d2r(theta)), sth = sinf(d2r(theta));
        const float cpsi = cosf(d2r(psi)), spsi = sinf(d2r(psi));
        float* m = rot + 6 * (size_t)o;
        m[0] = cphi * cth * cpsi - sphi * spsi;    // m[0][0]
        m[1] = -cphi * cth * spsi - sphi * cpsi;   // m[0][1]
        m[2] = sphi * cth * cpsi + cphi * spsi;    // m[1][0]
        m[3] = -sphi * cth * spsi + cphi * cpsi;   // m[1][1]
        m[4] = -sth * cpsi;                        // m[2][0]
        m[5] = sth * spsi;                         // m[2][1]
    }
}

tmk::BatchArgs make_args(tm_ctx* c) {
    tmk::BatchArgs a{};
    a.tmpl = c->tmpl;
    a.filter = c->filter;
    a.rot = c->rot;
    a.S = c->S;
    a.P = c->P;
    a.rowstat = c->rowstat;
    a.norm = c->norm;
    a.A = c->A;
    a.C = c->C;
    a.Ip = c->Ip;
    a.mip = c->mip;
    a.best = c->best;
    a.sum = c->sum;
    a.sumsq = c->sumsq;
    a.hist = c->hist;
    a.hist_min = (float)c->d.histogram_min_scaled;
    a.hist_inv_step = (float)(1.0 / c->d.histogram_step_scaled);
    a.hist_bins = c->d.histogram_bins;
    a.XP = c->XP;
    a.norm_pixels = c->norm_pixels;
    a.err = c->err_flag;
    a.tw.tab = c->twx;
    a.tw.lmax = c->X;
    a.twy.tab = c->twy;
    a.twy.lmax = c->Y;
    a.twt.tab = c->twt;
    a.twt.lmax = c->T;
    // FP16 form (powers of two): the correlation values are ~ 1/sqrt(N), N = X Y,
    // and the column-transformed spectra ~ 1/sqrt(N X); they are stored times
    // 2^e ~ sqrt(N X) so that the FP16 values are O(1).  The column pass holds I'
    // (~ N^-1.5) times 2^iexp ~ N^1.5 and its stage-1 operand Z (~ 1/N) times N.
    {
        const double l2n = log2((double)c->X * (double)c->Y);
        a.half_scale_exp = (int)lround(0.5 * (l2n + log2((double)c->X)));
        a.tc_iexp = (int)lround(1.5 * l2n);
        a.tc_zexp = (int)lround(l2n);
    }
    return a;
}

}  // namespace

namespace {

// ---------------------------------------------------------------------------------------------
// Template spectrum on the device (tm_template.cuh).

// The axis operators of the pixel-size change (image.cpp:8741-8822) for a
// T^3 volume padded to P^3 and resampled to N^3: m[t][i] = sum_k w(k)
// exp(2 pi i k (q/N - p/P)), q = N/2 + t - T/2, p = P/2 + i - T/2, as closed
// geometric sums (x axis: half-spectrum weights; y and z: the full axis).
void axis_operators(int T, int P, int N, std::vector<double>& mxr, std::vector<double>& mxi, std::vector<double>& myr,
                    std::vector<double>& myi) {
    const bool grow = N > P;
    const long kx_hi = grow ? P / 2 : N / 2;
    const long k_lo = grow ? -(P / 2) : -(N / 2), k_hi = grow ? P / 2 : N / 2 - 1;
    const long NP = (long)N * P;
    auto geo = [NP](long num, long a, long b, double& re, double& im) {
        num %= NP;
        if (num < 0) num += NP;
        const long cnt = b - a + 1;
        if (cnt <= 0) { re = im = 0.0; return; }
        if (num == 0) { re = (double)cnt; im = 0.0; return; }
        const double th = 2.0 * M_PI * (double)num / (double)NP;
        // e^{i th a} (1 - e^{i th cnt}) / (1 - e^{i th})
        const double ar = cos(th * a), ai = sin(th * a);
        const double nr = 1.0 - cos(th * cnt), ni = -sin(th * cnt);
        const double dr = 1.0 - cos(th), di = -sin(th);
        const double qr = (nr * dr + ni * di) / (dr * dr + di * di), qi = (ni * dr - nr * di) / (dr * dr + di * di);
        re = ar * qr - ai * qi;
        im = ar * qi + ai * qr;
    };
    mxr.assign((size_t)T * T, 0.0); mxi.assign((size_t)T * T, 0.0);
    myr.assign((size_t)T * T, 0.0); myi.assign((size_t)T * T, 0.0);
    for (int t = 0; t < T; t++) {
        const long q = N / 2 + t - T / 2;
        for (int i = 0; i < T; i++) {
            const long pp = P / 2 + i - T / 2;
            const long num = q * P - pp * N;
            double r0, i0, r1, i1;
            geo(num, 0, kx_hi, r0, i0);
            double xr = 2.0 * r0 - 1.0, xi = 2.0 * i0;
            if (!grow) {
                geo(num, N / 2, N / 2, r1, i1);
                xr -= r1;
                xi -= i1;
            }
            geo(num, k_lo, k_hi, r1, i1);
            mxr[(size_t)t * T + i] = xr;
            mxi[(size_t)t * T + i] = xi;
            myr[(size_t)t * T + i] = r1;
            myi[(size_t)t * T + i] = i1;
        }
    }
}

struct TemplateBuffers {
    const float* vol;     // T^3 reals
    float2* spec;         // T*T*(T/2+1)
    float* work;          // 5 T^3 floats (pixel-size change only)
    float* ops;           // 6 T*T floats
    double* acc;          // 2 doubles
    float* pad;           // 1 float
    tmcg::GemmJob* jobs;  // 4 + 4 T jobs
    tmfft::Twiddles tw;   // lmax = T
    int* gemm_err;        // 1 int: set by a tensor-core GEMM whose completion wait ran out
};
using TemplateFn = int (*)(cudaStream_t, int nsm, const TemplateBuffers&, float factor, std::string& err);

template <int T>
int template_on_device(cudaStream_t s, int nsm, const TemplateBuffers& b, float factor, std::string& err) {
    constexpr int HC = T / 2 + 1;
    const size_t n3 = (size_t)T * T * T;
    const float tol = 0.001f;
    const float* rows_src = b.vol;
    float add = 0.0f;
    if (!(fabsf(factor - 1.0f) < tol)) {
        // sizes (image.cpp:8741-8775), cubic volume
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
        if (nw <= T) {
            err = "pixel-size change to a resampled box not larger than the template is not supported";
            return TM_ERR_UNSUPPORTED;
        }
        float padding_value = 0.0f;
        if (pad > old) {
            TW_CHECK(cudaMemsetAsync(b.acc, 0, 2 * sizeof(double), s));
            tmt::k_t_disc_sum<<<nsm * 4, 256, 0, s>>>(b.vol, T, b.acc);
            TW_CHECK(cudaGetLastError());
            double acc[2];
            TW_CHECK(cudaMemcpyAsync(acc, b.acc, sizeof acc, cudaMemcpyDeviceToHost, s));
            TW_CHECK(cudaStreamSynchronize(s));
            padding_value = acc[1] > 0 ? (float)(acc[0] / acc[1]) : 0.0f;
        }
        std::vector<double> mxr, mxi, myr, myi;
        axis_operators(T, pad, nw, mxr, mxi, myr, myi);
        // ops: mxr^T, mxi^T (B operands of the x pass), myr, -myi, myi (y pass),
        // myr / P^3 and -myi / P^3 (z pass)
        const size_t t2 = (size_t)T * T;
        std::vector<float> ops(7 * t2);
        const double inv = 1.0 / ((double)pad * pad * pad);
        for (int t = 0; t < T; t++)
            for (int i = 0; i < T; i++) {
                const size_t ti = (size_t)t * T + i, it = (size_t)i * T + t;
                ops[0 * t2 + it] = (float)mxr[ti];
                ops[1 * t2 + it] = (float)mxi[ti];
                ops[2 * t2 + ti] = (float)myr[ti];
                ops[3 * t2 + ti] = (float)-myi[ti];
                ops[4 * t2 + ti] = (float)myi[ti];
                ops[5 * t2 + ti] = (float)(myr[ti] * inv);
                ops[6 * t2 + ti] = (float)(-myi[ti] * inv);
            }
        TW_CHECK(cudaMemcpyAsync(b.ops, ops.data(), sizeof(float) * ops.size(), cudaMemcpyHostToDevice, s));
        TW_CHECK(cudaMemcpyAsync(b.pad, &padding_value, sizeof(float), cudaMemcpyHostToDevice, s));
        float *Ar = b.work, *Ai = Ar + n3, *Br = Ai + n3, *Bi = Br + n3, *out = Bi + n3;
        const float* op = b.ops;
        std::vector<tmcg::GemmJob> jobs;
        // x pass: A = (vol - pad) mx^T (T^2 x T)
        jobs.push_back({b.vol, op + 0 * t2, Ar, b.pad});
        jobs.push_back({b.vol, op + 1 * t2, Ai, b.pad});
        // z pass: out = myr/P^3 Br - myi/P^3 Bi (T x T^2)
        jobs.push_back({op + 5 * t2, Br, out, nullptr});
        jobs.push_back({op + 6 * t2, Bi, out, nullptr});
        // y pass per z plane: Br = myr Ar - myi Ai, Bi = myr Ai + myi Ar
        for (int pass = 0; pass < 4; pass++)
            for (int z = 0; z < T; z++) {
                const size_t o = (size_t)z * t2;
                const float* A = op + (pass == 0 || pass == 2 ? 2 : pass == 1 ? 3 : 4) * t2;
                const float* Bm = (pass == 0 || pass == 3) ? Ar + o : Ai + o;
                float* Cm = (pass < 2) ? Br + o : Bi + o;
                jobs.push_back({A, Bm, Cm, nullptr});
            }
        TW_CHECK(cudaMemcpyAsync(b.jobs, jobs.data(), sizeof(tmcg::GemmJob) * jobs.size(), cudaMemcpyHostToDevice, s));
        TW_CHECK(cudaMemsetAsync(b.gemm_err, 0, sizeof(int), s));
        // the separable operators on the tensor cores (split TF32, FP32 accumulation)
        const int TT = T * T;
        TW_CHECK(tmcg::gemm_tc(b.jobs, 2, TT, T, T, T, T, T, 0, b.gemm_err, s));
        for (int pass = 0; pass < 4; pass++)
            TW_CHECK(tmcg::gemm_tc(b.jobs + 4 + pass * T, T, T, T, T, T, T, T, pass % 2, b.gemm_err, s));
        TW_CHECK(tmcg::gemm_tc(b.jobs + 2, 1, T, TT, T, T, TT, TT, 0, b.gemm_err, s));
        TW_CHECK(tmcg::gemm_tc(b.jobs + 3, 1, T, TT, T, T, TT, TT, 1, b.gemm_err, s));
        rows_src = out;
        add = padding_value;
    }
    using R = tmt::TRows<T>;
    using C = tmt::TCols<T>;
    tmt::k_t_rows<T><<<(T * T + R::ROWS - 1) / R::ROWS, R::NT, 0, s>>>(rows_src, add, b.spec, b.tw);
    TW_CHECK(cudaGetLastError());
    const long long ncols = (long long)T * HC;
    tmt::k_t_cols<T><<<(unsigned)((ncols + C::CB - 1) / C::CB), C::NT, 0, s>>>(b.spec, ncols, HC, (long long)T * HC, HC, 0,
                                                                              b.tw);
    TW_CHECK(cudaGetLastError());
    tmt::k_t_cols<T><<<(unsigned)((ncols + C::CB - 1) / C::CB), C::NT, 0, s>>>(b.spec, ncols, ncols, 0, ncols, 1, b.tw);
    TW_CHECK(cudaGetLastError());
    int gemm_failed = 0;
    if (rows_src != b.vol) TW_CHECK(cudaMemcpyAsync(&gemm_failed, b.gemm_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    TW_CHECK(cudaStreamSynchronize(s));
    if (gemm_failed) {
        err = "a tensor-core GEMM of the pixel-size change timed out";
        return TM_ERR_TIMEOUT;
    }
    return TM_OK;
}

struct TemplateVariant {
    int T;
    TemplateFn fn;
};
const TemplateVariant kTemplateVariants[] = {
    {32, template_on_device<32>},   {48, template_on_device<48>},   {64, template_on_device<64>},
    {128, template_on_device<128>}, {256, template_on_device<256>}, {384, template_on_device<384>},
};

TemplateFn find_template_fn(int T) {
    for (const TemplateVariant& v : kTemplateVariants)
        if (v.T == T) return v.fn;
    return nullptr;
}

// device buffers of one template preparation (freed by the caller)
struct TemplateScratch {
    float* vol = nullptr;
    float* work = nullptr;
    float* ops = nullptr;
    double* acc = nullptr;
    float* pad = nullptr;
    tmcg::GemmJob* jobs = nullptr;
    int* gemm_err = nullptr;
    void release() {
        void* p[] = {vol, work, ops, acc, pad, jobs, gemm_err};
        for (void* q : p)
            if (q) cudaFree(q);
        *this = TemplateScratch{};
    }
    cudaError_t alloc(int T, bool resample) {
        const size_t n3 = (size_t)T * T * T;
        cudaError_t e = cudaMalloc((void**)&vol, sizeof(float) * n3);
        if (e == cudaSuccess) e = cudaMalloc((void**)&acc, 2 * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc((void**)&pad, sizeof(float));
        if (e == cudaSuccess && resample) e = cudaMalloc((void**)&work, sizeof(float) * 5 * n3);
        if (e == cudaSuccess && resample) e = cudaMalloc((void**)&ops, sizeof(float) * 7 * (size_t)T * T);
        if (e == cudaSuccess && resample) e = cudaMalloc((void**)&jobs, sizeof(tmcg::GemmJob) * (4 + 4 * (size_t)T));
        if (e == cudaSuccess && resample) e = cudaMalloc((void**)&gemm_err, sizeof(int));
        return e;
    }
};

}  // namespace

extern "C" {

const char* tm_version(void) { return TM_VERSION; }

const char* tm_last_error(const tm_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int tm_create(const tm_dims* dims, tm_ctx** out) {
    if (!dims || !out) return TM_ERR_INVALID;
    *out = nullptr;
    tm_ctx* c = new tm_ctx();
    c->d = *dims;
    c->X = dims->image_x;
    c->Y = dims->image_y;
    c->T = dims->template_size;
    c->TP = c->T / 2 + 1;
    c->B = dims->orientation_batch > 0 ? dims->orientation_batch : 32;
    c->Bcap = dims->orientation_batch > 0 ? dims->orientation_batch : 128;   // 0 = automatic: room to tune up to 128
    if (dims->histogram_bins <= 0 || dims->histogram_bins > 1024 || !(dims->histogram_step_scaled > 0)) {
        *out = c;
        return set_err(c, TM_ERR_INVALID, "histogram_bins must be 1..1024 and the step positive");
    }
    c->var = find_variant(c->T, c->X, c->Y);
    if (!c->var && (c->var = find_generic_variant(c->T, c->X, c->Y)) != nullptr)
        generic_size(c->X, c->Y, &c->gen_px, &c->gen_py, &c->gen_ph);
    if (!c->var) {
        *out = c;
        return set_err(c, TM_ERR_UNSUPPORTED, "no kernel variant for template %d and image %d x %d", c->T, c->X, c->Y);
    }
    // the row pitch covers kx = 0 .. X/2 in whole pass-B chunks (and stays
    // even for the 16-byte loads of pass C)
    c->XP = (c->X / 2 + 1 + c->var->W - 1) / c->var->W * c->var->W;
    if (c->XP % 2) c->XP += c->var->W;
    c->device = dims->device;
    int rc;
#define TRY(x) if ((rc = (x)) != TM_OK) { *out = c; return rc; }
    {
        cudaError_t e = cudaSetDevice(c->device);
        if (e != cudaSuccess) { *out = c; return set_err(c, TM_ERR_CUDA, "cudaSetDevice(%d): %s", c->device, cudaGetErrorString(e)); }
        e = cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device);
        if (e != cudaSuccess) { *out = c; return set_err(c, TM_ERR_CUDA, "device query: %s", cudaGetErrorString(e)); }
    }
    {
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreate(&c->ev_start);
        if (e == cudaSuccess) e = cudaEventCreate(&c->ev_prep);
        if (e == cudaSuccess) e = cudaEventCreate(&c->ev_b);
        if (e == cudaSuccess) e = cudaEventCreate(&c->ev_c);
        if (e == cudaSuccess) e = cudaEventCreate(&c->ev_end);
        for (auto& set : c->ev_batch)
            for (cudaEvent_t& ev : set)
                if (e == cudaSuccess) e = cudaEventCreate(&ev);
        if (e != cudaSuccess) { *out = c; return set_err(c, TM_ERR_CUDA, "stream/event creation: %s", cudaGetErrorString(e)); }
    }
    if (dims->orientation_batch <= 0) {
        // automatic batch: keep the capacity for 128 (else 64, else 32) orientations
        // only if their correlation spectra fit in a quarter of the free device memory
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
            while (c->Bcap > 32 && (size_t)c->Bcap * c->Y * c->XP * sizeof(float2) > free_b / 4) c->Bcap /= 2;
    }
    const size_t T = c->T, X = c->X, Y = c->Y, XP = c->XP, TP = c->TP, B = c->Bcap;
    TRY(dalloc(c, &c->tmpl, T * T * TP));
    TRY(dalloc(c, &c->Ip, Y * XP));
    TRY(dalloc(c, &c->S, B * T * TP));
    TRY(dalloc(c, &c->P, B * T * T));
    TRY(dalloc(c, &c->rowstat, B * T * 4));
    TRY(dalloc(c, &c->norm, B));
    TRY(dalloc(c, &c->A, B * T * XP));
    TRY(dalloc(c, &c->C, B * Y * XP));
    TRY(dalloc(c, &c->filter, T * TP));
    TRY(dalloc(c, &c->mip, X * Y));
    TRY(dalloc(c, &c->best, X * Y));
    TRY(dalloc(c, &c->sum, X * Y));
    TRY(dalloc(c, &c->sumsq, X * Y));
    TRY(dalloc(c, &c->hist, (size_t)1024));
    TRY(dalloc(c, &c->err_flag, (size_t)1));
    {
        cudaError_t e = cudaMemset(c->err_flag, 0, sizeof(int));
        if (e != cudaSuccess) { *out = c; return set_err(c, TM_ERR_CUDA, "memset: %s", cudaGetErrorString(e)); }
    }
    // A's columns beyond X/2 are never written by the kernels and must read as zero
    {
        cudaError_t e = cudaMemsetAsync(c->A, 0, B * T * XP * sizeof(float2), c->stream);
        if (e != cudaSuccess) { *out = c; return set_err(c, TM_ERR_CUDA, "memset: %s", cudaGetErrorString(e)); }
    }
    // twiddle tables W_L^m = exp(-2 pi i m / L) for L = X, Y and T: every
    // transform length of a kernel divides the length of the table it uses
    {
        float2** tabs[3] = {&c->twx, &c->twy, &c->twt};
        const int lens[3] = {c->X, c->Y, c->T};
        for (int k = 0; k < 3; k++) {
            TRY(dalloc(c, tabs[k], (size_t)lens[k]));
            std::vector<float2> tw(lens[k]);
            for (int m = 0; m < lens[k]; m++) {
                double ang = -2.0 * M_PI * (double)m / (double)lens[k];
                tw[m] = make_float2((float)cos(ang), (float)sin(ang));
            }
            cudaError_t e = cudaMemcpy(*tabs[k], tw.data(), sizeof(float2) * lens[k], cudaMemcpyHostToDevice);
            if (e != cudaSuccess) { *out = c; return set_err(c, TM_ERR_CUDA, "twiddle upload: %s", cudaGetErrorString(e)); }
        }
    }
    TRY(c->var->configure(c));
#undef TRY
    *out = c;
    return tm_reset_results(c);
}

int tm_set_template(tm_ctx* c, const float* spectrum, int template_size) {
    if (!c || !spectrum) return TM_ERR_INVALID;
    if (template_size != c->T) return set_err(c, TM_ERR_INVALID, "template size %d differs from the context's %d", template_size, c->T);
    TM_CUDA(c, cudaSetDevice(c->device));
    TM_CUDA(c, cudaMemcpy(c->tmpl, spectrum, sizeof(float2) * (size_t)c->T * c->T * c->TP, cudaMemcpyHostToDevice));
    c->has_template = true;
    return TM_OK;
}

int tm_set_image(tm_ctx* c, const float* spectrum, int image_x, int image_y) {
    if (!c || !spectrum) return TM_ERR_INVALID;
    if (image_x != c->X || image_y != c->Y)
        return set_err(c, TM_ERR_INVALID, "image %d x %d differs from the context's %d x %d", image_x, image_y, c->X, c->Y);
    TM_CUDA(c, cudaSetDevice(c->device));
    // I'[ky][kx] = I[ky][kx] * exp(+2 pi i (kx*x0/X + ky*y0/Y)) / N, with the
    // projection placed at (x0, y0) = (X/2 - T/2, Y/2 - T/2); I'[0][0] = 0.
    // Computed on the device; the raw spectrum is staged in the correlation
    // buffer C, which holds nothing between planes.
    const int X = c->X, Y = c->Y, hc = X / 2 + 1, XP = c->XP;
    float2* staging = c->C;
    TM_CUDA(c, cudaMemcpyAsync(staging, spectrum, sizeof(float2) * (size_t)Y * hc, cudaMemcpyHostToDevice, c->stream));
    tmk::k_prepare_image<<<dim3((XP + 127) / 128, Y), 128, 0, c->stream>>>(staging, c->Ip, X, Y, XP, c->T);
    TM_CUDA(c, cudaGetLastError());
    int rc = wait_stream(c, 600.0);
    if (rc != TM_OK) return rc;
    c->has_image = true;
    return TM_OK;
}

int tm_set_micrograph(tm_ctx* c, const float* image, int image_x, int image_y, double* curve, int curve_capacity,
                      int* curve_points_out) {
    if (!c || !image) return TM_ERR_INVALID;
    if (image_x != c->X || image_y != c->Y)
        return set_err(c, TM_ERR_INVALID, "image %d x %d differs from the context's %d x %d", image_x, image_y, c->X, c->Y);
    TM_CUDA(c, cudaSetDevice(c->device));
    const int X = c->X, Y = c->Y, XP = c->XP;
    const int npts = curve_points(X);
    if (curve && curve_capacity < npts)
        return set_err(c, TM_ERR_INVALID, "curve capacity %d below the %d points of the whitening filter", curve_capacity, npts);
    float* d_img = nullptr;
    double* d_scratch = nullptr;
    float* d_xs = nullptr;
    int rc = dalloc(c, &d_img, (size_t)X * Y);
    if (rc == TM_OK) rc = dalloc(c, &d_scratch, (size_t)3 + 3 * npts);
    if (rc == TM_OK) rc = dalloc(c, &d_xs, (size_t)npts);
    std::vector<double> h_curve;
    if (rc == TM_OK) {
        cudaError_t e = cudaMemcpyAsync(d_img, image, sizeof(float) * (size_t)X * Y, cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) rc = set_err(c, TM_ERR_CUDA, "micrograph upload: %s", cudaGetErrorString(e));
    }
    if (rc == TM_OK) {
        // the whitened spectrum is staged in the correlation buffer C, as tm_set_image stages its input
        WhitenBuffers wb{d_img, c->C, d_scratch, d_xs, make_args(c).tw, make_args(c).twy, c->X, c->Y};
        std::string err;
        rc = c->var->whiten(c->stream, c->nsm, wb, h_curve, err);
        if (rc != TM_OK) set_err(c, rc, "whitening: %s", err.c_str());
    }
    if (rc == TM_OK) {
        tmk::k_prepare_image<<<dim3((XP + 127) / 128, Y), 128, 0, c->stream>>>(c->C, c->Ip, X, Y, XP, c->T);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = set_err(c, TM_ERR_CUDA, "k_prepare_image: %s", cudaGetErrorString(e));
        if (rc == TM_OK) rc = wait_stream(c, 600.0);
    }
    if (d_img) cudaFree(d_img);
    if (d_scratch) cudaFree(d_scratch);
    if (d_xs) cudaFree(d_xs);
    if (rc != TM_OK) return rc;
    if (curve) memcpy(curve, h_curve.data(), sizeof(double) * npts);
    if (curve_points_out) *curve_points_out = npts;
    c->has_image = true;
    return TM_OK;
}

int tm_whiten_micrograph(int device, const float* image, int image_x, int image_y, float* spectrum, double* curve,
                         int curve_capacity, int* curve_points_out) {
    if (!image || !spectrum || image_x <= 0 || image_y <= 0) return TM_ERR_INVALID;
    const Variant* var = nullptr;
    for (const Variant& v : kVariants)
        if (v.X == image_x && v.Y == image_y) var = &v;
    if (!var) var = find_generic_variant(64, image_x, image_y);   // the whitening does not depend on T
    if (!var) return TM_ERR_UNSUPPORTED;
    const int X = image_x, Y = image_y, hc = X / 2 + 1;
    const int npts = curve_points(X);
    if (curve && curve_capacity < npts) return TM_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return TM_ERR_CUDA;
    int dev_sms = 0;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device);
    cudaStream_t s = nullptr;
    float *d_img = nullptr, *d_xs = nullptr;
    float2 *d_spec = nullptr, *d_twx = nullptr, *d_twy = nullptr;
    double* d_scratch = nullptr;
    int rc = TM_OK;
    auto fail = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == TM_OK) rc = e == cudaErrorMemoryAllocation ? TM_ERR_OOM : TM_ERR_CUDA;
    };
    fail(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    if (rc == TM_OK) fail(cudaMalloc((void**)&d_img, sizeof(float) * (size_t)X * Y));
    if (rc == TM_OK) fail(cudaMalloc((void**)&d_spec, sizeof(float2) * (size_t)Y * hc));
    if (rc == TM_OK) fail(cudaMalloc((void**)&d_scratch, sizeof(double) * (3 + 3 * (size_t)npts)));
    if (rc == TM_OK) fail(cudaMalloc((void**)&d_xs, sizeof(float) * npts));
    if (rc == TM_OK) fail(cudaMalloc((void**)&d_twx, sizeof(float2) * X));
    if (rc == TM_OK) fail(cudaMalloc((void**)&d_twy, sizeof(float2) * Y));
    if (rc == TM_OK) {
        for (int k = 0; k < 2 && rc == TM_OK; k++) {
            const int L = k == 0 ? X : Y;
            std::vector<float2> tw(L);
            for (int m = 0; m < L; m++) {
                const double ang = -2.0 * M_PI * (double)m / (double)L;
                tw[m] = make_float2((float)cos(ang), (float)sin(ang));
            }
            fail(cudaMemcpy(k == 0 ? d_twx : d_twy, tw.data(), sizeof(float2) * L, cudaMemcpyHostToDevice));
        }
    }
    if (rc == TM_OK) fail(cudaMemcpyAsync(d_img, image, sizeof(float) * (size_t)X * Y, cudaMemcpyHostToDevice, s));
    std::vector<double> h_curve;
    if (rc == TM_OK) {
        tmfft::Twiddles twx{d_twx, X}, twy{d_twy, Y};
        WhitenBuffers wb{d_img, d_spec, d_scratch, d_xs, twx, twy, X, Y};
        std::string err;
        rc = var->whiten(s, dev_sms > 0 ? dev_sms : 148, wb, h_curve, err);
    }
    if (rc == TM_OK) {
        fail(cudaMemcpyAsync(spectrum, d_spec, sizeof(float2) * (size_t)Y * hc, cudaMemcpyDeviceToHost, s));
        if (rc == TM_OK) fail(cudaStreamSynchronize(s));
    }
    void* ptrs[] = {d_img, d_xs, d_spec, d_twx, d_twy, d_scratch};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s) cudaStreamDestroy(s);
    if (rc != TM_OK) return rc;
    if (curve) memcpy(curve, h_curve.data(), sizeof(double) * npts);
    if (curve_points_out) *curve_points_out = npts;
    return TM_OK;
}

int tm_set_template_volume(tm_ctx* c, const float* volume, int template_size, float pixel_size_factor) {
    if (!c || !volume) return TM_ERR_INVALID;
    if (template_size != c->T) return set_err(c, TM_ERR_INVALID, "template size %d differs from the context's %d", template_size, c->T);
    TemplateFn fn = find_template_fn(c->T);
    if (!fn) return set_err(c, TM_ERR_UNSUPPORTED, "no template kernels for box %d", c->T);
    TM_CUDA(c, cudaSetDevice(c->device));
    const bool resample = !(fabsf(pixel_size_factor - 1.0f) < 0.001f);
    TemplateScratch sc;
    cudaError_t e = sc.alloc(c->T, resample);
    if (e != cudaSuccess) {
        sc.release();
        return set_err(c, e == cudaErrorMemoryAllocation ? TM_ERR_OOM : TM_ERR_CUDA, "template buffers: %s", cudaGetErrorString(e));
    }
    int rc = TM_OK;
    e = cudaMemcpyAsync(sc.vol, volume, sizeof(float) * (size_t)c->T * c->T * c->T, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) rc = set_err(c, TM_ERR_CUDA, "template upload: %s", cudaGetErrorString(e));
    if (rc == TM_OK) {
        TemplateBuffers tb{sc.vol, c->tmpl, sc.work, sc.ops, sc.acc, sc.pad, sc.jobs, make_args(c).twt, sc.gemm_err};
        std::string err;
        rc = fn(c->stream, c->nsm, tb, pixel_size_factor, err);
        if (rc != TM_OK) set_err(c, rc, "template preparation: %s", err.c_str());
    }
    sc.release();
    if (rc == TM_OK) c->has_template = true;
    return rc;
}

int tm_template_spectrum(int device, const float* volume, int template_size, float pixel_size_factor, float* spectrum) {
    if (!volume || !spectrum) return TM_ERR_INVALID;
    const int T = template_size;
    TemplateFn fn = find_template_fn(T);
    if (!fn) return TM_ERR_UNSUPPORTED;
    if (cudaSetDevice(device) != cudaSuccess) return TM_ERR_CUDA;
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    const bool resample = !(fabsf(pixel_size_factor - 1.0f) < 0.001f);
    const size_t nspec = (size_t)T * T * (T / 2 + 1);
    TemplateScratch sc;
    cudaStream_t s = nullptr;
    float2 *d_spec = nullptr, *d_tw = nullptr;
    int rc = TM_OK;
    auto fail = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == TM_OK) rc = e == cudaErrorMemoryAllocation ? TM_ERR_OOM : TM_ERR_CUDA;
    };
    fail(sc.alloc(T, resample));
    if (rc == TM_OK) fail(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    if (rc == TM_OK) fail(cudaMalloc((void**)&d_spec, sizeof(float2) * nspec));
    if (rc == TM_OK) fail(cudaMalloc((void**)&d_tw, sizeof(float2) * T));
    if (rc == TM_OK) {
        std::vector<float2> tw(T);
        for (int m = 0; m < T; m++) {
            const double ang = -2.0 * M_PI * (double)m / (double)T;
            tw[m] = make_float2((float)cos(ang), (float)sin(ang));
        }
        fail(cudaMemcpy(d_tw, tw.data(), sizeof(float2) * T, cudaMemcpyHostToDevice));
    }
    if (rc == TM_OK) fail(cudaMemcpyAsync(sc.vol, volume, sizeof(float) * (size_t)T * T * T, cudaMemcpyHostToDevice, s));
    if (rc == TM_OK) {
        TemplateBuffers tb{sc.vol, d_spec, sc.work, sc.ops, sc.acc, sc.pad, sc.jobs, tmfft::Twiddles{d_tw, T}, sc.gemm_err};
        std::string err;
        rc = fn(s, nsm > 0 ? nsm : 148, tb, pixel_size_factor, err);
    }
    if (rc == TM_OK) fail(cudaMemcpyAsync(spectrum, d_spec, sizeof(float2) * nspec, cudaMemcpyDeviceToHost, s));
    if (rc == TM_OK) fail(cudaStreamSynchronize(s));
    sc.release();
    if (d_spec) cudaFree(d_spec);
    if (d_tw) cudaFree(d_tw);
    if (s) cudaStreamDestroy(s);
    return rc;
}

int tm_debug_gemm(int device, int M, int N, int K, const float* A, const float* B, float* C, float s, int accumulate,
                  int tensor) {
    if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0) return TM_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return TM_ERR_CUDA;
    float *dA = nullptr, *dB = nullptr, *dC = nullptr, *ds = nullptr;
    int* derr = nullptr;
    tmcg::GemmJob* dj = nullptr;
    cudaStream_t st = nullptr;
    int rc = TM_OK;
    auto fail = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == TM_OK) rc = e == cudaErrorMemoryAllocation ? TM_ERR_OOM : TM_ERR_CUDA;
    };
    fail(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (rc == TM_OK) fail(cudaMalloc((void**)&dA, sizeof(float) * (size_t)M * K));
    if (rc == TM_OK) fail(cudaMalloc((void**)&dB, sizeof(float) * (size_t)K * N));
    if (rc == TM_OK) fail(cudaMalloc((void**)&dC, sizeof(float) * (size_t)M * N));
    if (rc == TM_OK) fail(cudaMalloc((void**)&ds, sizeof(float)));
    if (rc == TM_OK) fail(cudaMalloc((void**)&derr, sizeof(int)));
    if (rc == TM_OK) fail(cudaMalloc((void**)&dj, sizeof(tmcg::GemmJob)));
    if (rc == TM_OK) fail(cudaMemcpy(dA, A, sizeof(float) * (size_t)M * K, cudaMemcpyHostToDevice));
    if (rc == TM_OK) fail(cudaMemcpy(dB, B, sizeof(float) * (size_t)K * N, cudaMemcpyHostToDevice));
    if (rc == TM_OK) fail(cudaMemcpy(dC, C, sizeof(float) * (size_t)M * N, cudaMemcpyHostToDevice));
    if (rc == TM_OK) fail(cudaMemcpy(ds, &s, sizeof(float), cudaMemcpyHostToDevice));
    if (rc == TM_OK) fail(cudaMemset(derr, 0, sizeof(int)));
    if (rc == TM_OK) {
        const tmcg::GemmJob job{dA, dB, dC, ds};
        fail(cudaMemcpy(dj, &job, sizeof job, cudaMemcpyHostToDevice));
    }
    if (rc == TM_OK) {
        if (tensor) {
            fail(tmcg::gemm_tc(dj, 1, M, N, K, K, N, N, accumulate, derr, st));
        } else {
            tmcg::k_gemm<<<dim3((N + 127) / 128, (M + 127) / 128, 1), 256, 0, st>>>(dj, M, N, K, K, N, N, accumulate);
            fail(cudaGetLastError());
        }
    }
    int failed = 0;
    if (rc == TM_OK) fail(cudaStreamSynchronize(st));
    if (rc == TM_OK) fail(cudaMemcpy(&failed, derr, sizeof(int), cudaMemcpyDeviceToHost));
    if (rc == TM_OK && failed) rc = TM_ERR_TIMEOUT;
    if (rc == TM_OK) fail(cudaMemcpy(C, dC, sizeof(float) * (size_t)M * N, cudaMemcpyDeviceToHost));
    void* p[] = {dA, dB, dC, ds, derr, dj};
    for (void* q : p)
        if (q) cudaFree(q);
    if (st) cudaStreamDestroy(st);
    return rc;
}

int tm_set_normalization_pixels(tm_ctx* c, long long n_pixels) {
    if (!c) return TM_ERR_INVALID;
    if (n_pixels < 0) return set_err(c, TM_ERR_INVALID, "normalisation pixel count %lld < 0", n_pixels);
    c->norm_pixels = n_pixels;
    return TM_OK;
}

int tm_set_precision(tm_ctx* c, int precision) {
    if (!c) return TM_ERR_INVALID;
    if (precision == TM_PRECISION_FP32) {
        c->precision = precision;
        return TM_OK;
    }
    if (precision != TM_PRECISION_FP16_TENSOR) return set_err(c, TM_ERR_INVALID, "unknown precision %d", precision);
    if (!c->var->tc)
        return set_err(c, TM_ERR_UNSUPPORTED, "no FP16 tensor-core form for template %d and image %d x %d", c->T, c->X, c->Y);
    TM_CUDA(c, cudaSetDevice(c->device));
    if (!c->dft) {
        const size_t bytes = c->var->tc->dft_bytes;
        std::vector<uint16_t> host(bytes / 2);
        c->var->tc->fill_dft(host.data());
        int rc = dalloc(c, &c->dft, bytes / sizeof(uint4));
        if (rc != TM_OK) return rc;
        TM_CUDA(c, cudaMemcpy(c->dft, host.data(), bytes, cudaMemcpyHostToDevice));
        rc = c->var->tc->configure(c);
        if (rc != TM_OK) return rc;
    }
    c->precision = precision;
    return TM_OK;
}

int tm_get_precision(const tm_ctx* c) { return c ? c->precision : TM_ERR_INVALID; }

int tm_reset_results(tm_ctx* c) {
    if (!c) return TM_ERR_INVALID;
    TM_CUDA(c, cudaSetDevice(c->device));
    const size_t n = (size_t)c->X * c->Y;
    tmk::k_reset_state<<<c->nsm * 4, 256, 0, c->stream>>>(c->mip, c->best, c->sum, c->sumsq, n);
    TM_CUDA(c, cudaGetLastError());
    TM_CUDA(c, cudaMemsetAsync(c->hist, 0, sizeof(unsigned long long) * 1024, c->stream));
    for (tm_ctx::Slot& sl : c->slots) {   // the image set's results too (their indices refer to the planes)
        tmk::k_reset_state<<<c->nsm * 4, 256, 0, c->stream>>>(sl.mip, sl.best, sl.sum, sl.sumsq, n);
        TM_CUDA(c, cudaGetLastError());
        TM_CUDA(c, cudaMemsetAsync(sl.hist, 0, sizeof(unsigned long long) * 1024, c->stream));
    }
    int rc = wait_stream(c, 60.0);
    if (rc != TM_OK) return rc;
    c->planes.clear();
    c->angle_lists.clear();
    c->next_gidx = 0;
    c->n_ccs = 0;
    return TM_OK;
}

int tm_run_plane(tm_ctx* c, const float* projection_filter, const float* euler_angles, int n, float defocus_offset,
                 float pixel_size_offset, tm_progress_fn progress, void* user) {
    if (!c || !projection_filter || (!euler_angles && n > 0) || n < 0) return TM_ERR_INVALID;
    if (!c->has_template || !c->has_image) return set_err(c, TM_ERR_INVALID, "template and image must be set before tm_run_plane");
    if (c->next_gidx + n > 2147483647LL) return set_err(c, TM_ERR_INVALID, "more than 2^31 orientations since the last reset");
    if (n == 0) return TM_OK;
    TM_CUDA(c, cudaSetDevice(c->device));
    // rotation table, float Euler matrices as RotationMatrix::SetToEulerRotation (matrix.cpp:490-510)
    if (n > c->rot_capacity) {
        if (c->rot) cudaFree(c->rot);
        c->rot = nullptr;
        int rc = dalloc(c, &c->rot, (size_t)6 * n);
        if (rc != TM_OK) return rc;
        c->rot_capacity = n;
    }
    std::vector<float> rot((size_t)6 * n);
    euler_rows(euler_angles, n, rot.data());
    TM_CUDA(c, cudaMemcpyAsync(c->rot, rot.data(), sizeof(float) * rot.size(), cudaMemcpyHostToDevice, c->stream));
    TM_CUDA(c, cudaMemcpyAsync(c->filter, projection_filter, sizeof(float) * (size_t)c->T * c->TP, cudaMemcpyHostToDevice, c->stream));
    // bookkeeping for decoding (reuse the previous angle list when identical)
    Plane pl;
    pl.base = c->next_gidx;
    pl.n = n;
    pl.defocus = defocus_offset;
    pl.pixel = pixel_size_offset;
    if (!c->angle_lists.empty() && (int)c->angle_lists.back().size() == 3 * n &&
        memcmp(c->angle_lists.back().data(), euler_angles, sizeof(float) * 3 * (size_t)n) == 0) {
        pl.angles_id = (int)c->angle_lists.size() - 1;
    } else {
        c->angle_lists.emplace_back(euler_angles, euler_angles + 3 * (size_t)n);
        pl.angles_id = (int)c->angle_lists.size() - 1;
    }
    c->planes.push_back(pl);

    tmk::BatchArgs a = make_args(c);
    a.rot = c->rot;
    TM_CUDA(c, cudaEventRecord(c->ev_start, c->stream));
    double b_ms = 0, c_ms = 0, prep_ms = 0;
    const int nbatch = (n + c->B - 1) / c->B;
    int timed_nb[2] = {0, 0};
    for (int bi = 0; bi < nbatch; bi++) {
        a.orient0 = bi * c->B;
        a.nb = n - a.orient0 < c->B ? n - a.orient0 : c->B;
        a.gidx0 = pl.base + a.orient0;
        // the kernel families are timed on the first and last batch (events
        // read after the plane, so the stream never stalls for them)
        const int set = bi == 0 ? 0 : (bi == nbatch - 1 ? 1 : -1);
        if (set >= 0) timed_nb[set] = a.nb;
        int rc = c->precision == TM_PRECISION_FP16_TENSOR
                     ? c->var->tc->run_batch(c, a, set >= 0 ? c->ev_batch[set] : nullptr)
                     : c->var->run_batch(c, a, set >= 0 ? c->ev_batch[set] : nullptr);
        if (rc != TM_OK) return rc;
        if (progress) {
            if (progress((long long)(a.orient0 + a.nb), (long long)n, user) != 0) {
                int w = wait_stream(c, 600.0);
                c->next_gidx += n;
                return w != TM_OK ? w : set_err(c, TM_ERR_CANCELLED, "cancelled by the progress callback");
            }
        }
    }
    TM_CUDA(c, cudaEventRecord(c->ev_c, c->stream));
    int w = wait_stream(c, 3600.0);
    if (w != TM_OK) return w;
    {
        int flag = 0;
        TM_CUDA(c, cudaMemcpy(&flag, c->err_flag, sizeof(int), cudaMemcpyDeviceToHost));
        if (flag) {
            cudaMemset(c->err_flag, 0, sizeof(int));
            return set_err(c, TM_ERR_TIMEOUT, "a bulk copy did not complete within its wait limit; results of this plane are invalid");
        }
    }
    float tot = 0;
    cudaEventElapsedTime(&tot, c->ev_start, c->ev_c);
    for (int set = 0; set < (nbatch > 1 ? 2 : 1); set++) {
        float t_prep = 0, t_b = 0, t_c = 0;
        cudaEvent_t* ev = c->ev_batch[set];
        cudaEventElapsedTime(&t_prep, ev[0], ev[1]);
        cudaEventElapsedTime(&t_b, ev[1], ev[2]);
        cudaEventElapsedTime(&t_c, ev[2], ev[3]);
        const double scale = (double)timed_nb[set];
        prep_ms += t_prep / scale;
        b_ms += t_b / scale;
        c_ms += t_c / scale;
    }
    // per-orientation averages of the sampled batches, scaled to the plane
    const int sampled = nbatch > 1 ? 2 : 1;
    c->last_total_ms = tot;
    c->last_prep_ms = prep_ms / sampled * n;
    c->last_b_ms = b_ms / sampled * n;
    c->last_c_ms = c_ms / sampled * n;
    c->next_gidx += n;
    c->n_ccs += n;
    return TM_OK;
}

int tm_get_results(tm_ctx* c, float* mip, float* best_psi, float* best_theta, float* best_phi, float* best_defocus,
                   float* best_pixel_size, double* sum, double* sum_of_squares, long long* histogram) {
    if (!c) return TM_ERR_INVALID;
    TM_CUDA(c, cudaSetDevice(c->device));
    const size_t n = (size_t)c->X * c->Y;
    int rc = wait_stream(c, 3600.0);
    if (rc != TM_OK) return rc;
    // the best-orientation map first: host threads decode it while this
    // thread copies the other maps
    std::vector<std::thread> pool;
    const bool want_angles = best_psi || best_theta || best_phi || best_defocus || best_pixel_size;
    if (want_angles) {
        if (!c->best_host) TM_CUDA(c, cudaMallocHost((void**)&c->best_host, sizeof(int) * n));
        TM_CUDA(c, cudaMemcpy(c->best_host, c->best, sizeof(int) * n, cudaMemcpyDeviceToHost));
        const int* best = c->best_host;
        // decode global orientation indices into angles and plane offsets, in parallel
        auto decode = [c, best, best_psi, best_theta, best_phi, best_defocus, best_pixel_size](size_t i0, size_t i1) {
            for (size_t i = i0; i < i1; i++) {
                const int g = best[i];
                float psi = 0, th = 0, ph = 0, df = 0, px = 0;
                if (g >= 0) {
                    // planes are few: linear scan from the back (most recent first)
                    for (size_t k = c->planes.size(); k-- > 0;) {
                        const Plane& p = c->planes[k];
                        if (g >= p.base && g < p.base + p.n) {
                            const float* ang = c->angle_lists[p.angles_id].data() + 3 * (size_t)(g - p.base);
                            ph = ang[0];
                            th = ang[1];
                            psi = ang[2];
                            df = p.defocus;
                            px = p.pixel;
                            break;
                        }
                    }
                }
                if (best_psi) best_psi[i] = psi;
                if (best_theta) best_theta[i] = th;
                if (best_phi) best_phi[i] = ph;
                if (best_defocus) best_defocus[i] = df;
                if (best_pixel_size) best_pixel_size[i] = px;
            }
        };
        unsigned nt = std::thread::hardware_concurrency();
        nt = nt < 1 ? 1 : (nt > 32 ? 32 : nt);
        if (n < ((size_t)1 << 16)) nt = 1;
        const size_t chunk = (n + nt - 1) / nt;
        for (unsigned k = 0; k < nt; k++) {
            const size_t i0 = k * chunk, i1 = std::min(n, i0 + chunk);
            if (i0 < i1) pool.emplace_back(decode, i0, i1);
        }
    }
    auto join = [&pool] {
        for (auto& th : pool) th.join();
        pool.clear();
    };
    cudaError_t e = cudaSuccess;
    if (mip && e == cudaSuccess) e = cudaMemcpy(mip, c->mip, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (sum && e == cudaSuccess) e = cudaMemcpy(sum, c->sum, sizeof(double) * n, cudaMemcpyDeviceToHost);
    if (sum_of_squares && e == cudaSuccess)
        e = cudaMemcpy(sum_of_squares, c->sumsq, sizeof(double) * n, cudaMemcpyDeviceToHost);
    if (histogram && e == cudaSuccess) {
        std::vector<unsigned long long> h(c->d.histogram_bins);
        e = cudaMemcpy(h.data(), c->hist, sizeof(unsigned long long) * h.size(), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            for (size_t i = 0; i < h.size(); i++) histogram[i] = (long long)h[i];
    }
    join();
    if (e != cudaSuccess) return set_err(c, TM_ERR_CUDA, "result copy: %s", cudaGetErrorString(e));
    return TM_OK;
}

long long tm_correlations_computed(const tm_ctx* c) { return c ? c->n_ccs : 0; }

int tm_last_timing(const tm_ctx* c, double* total_ms, double* pass_b_ms, double* pass_c_ms, double* prep_ms) {
    if (!c) return TM_ERR_INVALID;
    if (total_ms) *total_ms = c->last_total_ms;
    if (pass_b_ms) *pass_b_ms = c->last_b_ms;
    if (pass_c_ms) *pass_c_ms = c->last_c_ms;
    if (prep_ms) *prep_ms = c->last_prep_ms;
    return TM_OK;
}

int tm_debug_stage_buffers(tm_ctx* c, const float* projection_filter, const float* euler_angle, float* slice,
                           float* projection, float* normalisation, float* rows, float* columns) {
    if (!c || !projection_filter || !euler_angle) return TM_ERR_INVALID;
    if (!c->has_template || !c->has_image) return set_err(c, TM_ERR_INVALID, "template and image must be set first");
    TM_CUDA(c, cudaSetDevice(c->device));
    if (c->rot_capacity < 1) {
        int rc = dalloc(c, &c->rot, (size_t)6);
        if (rc != TM_OK) return rc;
        c->rot_capacity = 1;
    }
    float rot[6];
    euler_rows(euler_angle, 1, rot);
    TM_CUDA(c, cudaMemcpyAsync(c->rot, rot, sizeof rot, cudaMemcpyHostToDevice, c->stream));
    TM_CUDA(c, cudaMemcpyAsync(c->filter, projection_filter, sizeof(float) * (size_t)c->T * c->TP, cudaMemcpyHostToDevice, c->stream));
    tmk::BatchArgs a = make_args(c);
    a.nb = 1;
    a.orient0 = 0;
    a.gidx0 = 0;
    int rc = c->var->run_stages(c, a);
    if (rc != TM_OK) return rc;
    rc = wait_stream(c, 60.0);
    if (rc != TM_OK) return rc;
    const size_t T = c->T, TP = c->TP, XP = c->XP, hc = c->X / 2 + 1;
    if (slice) TM_CUDA(c, cudaMemcpy(slice, c->S, sizeof(float2) * T * TP, cudaMemcpyDeviceToHost));
    if (projection) TM_CUDA(c, cudaMemcpy(projection, c->P, sizeof(float) * T * T, cudaMemcpyDeviceToHost));
    if (normalisation) TM_CUDA(c, cudaMemcpy(normalisation, c->norm, sizeof(float2), cudaMemcpyDeviceToHost));
    if (rows) TM_CUDA(c, cudaMemcpy2D(rows, hc * sizeof(float2), c->A, XP * sizeof(float2), hc * sizeof(float2), T, cudaMemcpyDeviceToHost));
    if (columns) TM_CUDA(c, cudaMemcpy2D(columns, hc * sizeof(float2), c->C, XP * sizeof(float2), hc * sizeof(float2), (size_t)c->Y, cudaMemcpyDeviceToHost));
    return TM_OK;
}

int tm_autotune_batch(tm_ctx* c, const float* projection_filter, const float* euler_angles, int n, int* chosen) {
    if (!c || !projection_filter || !euler_angles || n <= 0) return TM_ERR_INVALID;
    const int cands[4] = {16, 32, 64, 128};
    int best_b = c->B;
    double best = 1e30;
    bool warmed = false;
    for (int b : cands) {
        if (b > c->Bcap) continue;
        c->B = b;
        int rc = tm_reset_results(c);
        if (rc != TM_OK) return rc;
        if (!warmed) {   // first launches of a context pay one-time costs
            rc = tm_run_plane(c, projection_filter, euler_angles, n < b ? n : b, 0.f, 0.f, nullptr, nullptr);
            if (rc != TM_OK) return rc;
            warmed = true;
        }
        rc = tm_run_plane(c, projection_filter, euler_angles, n, 0.f, 0.f, nullptr, nullptr);
        if (rc != TM_OK) return rc;
        const double per = c->last_total_ms / n;
        if (per < best) {
            best = per;
            best_b = b;
        }
    }
    c->B = best_b;
    if (chosen) *chosen = best_b;
    return tm_reset_results(c);
}

int tm_orientation_batch(const tm_ctx* c) { return c ? c->B : 0; }

int tm_set_image_set(tm_ctx* c, int n_images, const float* spectra) {
    if (!c || !spectra || n_images < 1 || n_images > 4096) return TM_ERR_INVALID;
    TM_CUDA(c, cudaSetDevice(c->device));
    int rc = tm_reset_results(c);   // a new set starts a new search: planes and main state cleared
    if (rc != TM_OK) return rc;
    const size_t X = c->X, Y = c->Y, XP = c->XP, hc = X / 2 + 1, n = X * Y;
    if ((int)c->slots.size() != n_images) {
        for (tm_ctx::Slot& sl : c->slots) {
            void* sp[] = {sl.Ip, sl.mip, sl.best, sl.sum, sl.sumsq, sl.hist};
            for (void* q : sp)
                if (q) cudaFree(q);
        }
        c->slots.assign((size_t)n_images, tm_ctx::Slot{});
        for (tm_ctx::Slot& sl : c->slots) {
            if ((rc = dalloc(c, &sl.Ip, Y * XP)) != TM_OK) return rc;
            if ((rc = dalloc(c, &sl.mip, n)) != TM_OK) return rc;
            if ((rc = dalloc(c, &sl.best, n)) != TM_OK) return rc;
            if ((rc = dalloc(c, &sl.sum, n)) != TM_OK) return rc;
            if ((rc = dalloc(c, &sl.sumsq, n)) != TM_OK) return rc;
            if ((rc = dalloc(c, &sl.hist, (size_t)1024)) != TM_OK) return rc;
            TM_CUDA(c, cudaMemsetAsync(sl.Ip, 0, sizeof(float2) * Y * XP, c->stream));
        }
    }
    // each spectrum is staged in the correlation buffer and prepared as tm_set_image does
    for (int k = 0; k < n_images; k++) {
        tm_ctx::Slot& sl = c->slots[k];
        TM_CUDA(c, cudaMemcpyAsync(c->C, spectra + (size_t)k * Y * hc * 2, sizeof(float2) * Y * hc,
                                   cudaMemcpyHostToDevice, c->stream));
        tmk::k_prepare_image<<<dim3((unsigned)((XP + 127) / 128), (unsigned)Y), 128, 0, c->stream>>>(c->C, sl.Ip, c->X, c->Y,
                                                                                                    c->XP, c->T);
        tmk::k_reset_state<<<c->nsm * 4, 256, 0, c->stream>>>(sl.mip, sl.best, sl.sum, sl.sumsq, n);
        TM_CUDA(c, cudaMemsetAsync(sl.hist, 0, sizeof(unsigned long long) * 1024, c->stream));
        TM_CUDA(c, cudaGetLastError());
        // the staging buffer is reused by the next image: keep the copies in order
        if ((rc = wait_stream(c, 600.0)) != TM_OK) return rc;
    }
    return TM_OK;
}

int tm_run_plane_images(tm_ctx* c, const float* projection_filter, const float* euler_angles, int n,
                        const int* images, int n_images, float defocus_offset, float pixel_size_offset) {
    if (!c || !projection_filter || (!euler_angles && n > 0) || n < 0 || !images || n_images < 1) return TM_ERR_INVALID;
    if (!c->has_template) return set_err(c, TM_ERR_INVALID, "template must be set before tm_run_plane_images");
    if (c->slots.empty()) return set_err(c, TM_ERR_INVALID, "no image set (tm_set_image_set)");
    for (int k = 0; k < n_images; k++)
        if (images[k] < 0 || images[k] >= (int)c->slots.size())
            return set_err(c, TM_ERR_INVALID, "image %d outside the set of %d", images[k], (int)c->slots.size());
    if (c->next_gidx + n > 2147483647LL) return set_err(c, TM_ERR_INVALID, "more than 2^31 orientations since the last reset");
    if (n == 0) return TM_OK;
    TM_CUDA(c, cudaSetDevice(c->device));
    if (n > c->rot_capacity) {
        if (c->rot) cudaFree(c->rot);
        c->rot = nullptr;
        int rc = dalloc(c, &c->rot, (size_t)6 * n);
        if (rc != TM_OK) return rc;
        c->rot_capacity = n;
    }
    std::vector<float> rot((size_t)6 * n);
    euler_rows(euler_angles, n, rot.data());
    TM_CUDA(c, cudaMemcpyAsync(c->rot, rot.data(), sizeof(float) * rot.size(), cudaMemcpyHostToDevice, c->stream));
    TM_CUDA(c, cudaMemcpyAsync(c->filter, projection_filter, sizeof(float) * (size_t)c->T * c->TP, cudaMemcpyHostToDevice, c->stream));
    Plane pl;
    pl.base = c->next_gidx;
    pl.n = n;
    pl.defocus = defocus_offset;
    pl.pixel = pixel_size_offset;
    c->angle_lists.emplace_back(euler_angles, euler_angles + 3 * (size_t)n);
    pl.angles_id = (int)c->angle_lists.size() - 1;
    c->planes.push_back(pl);
    tmk::BatchArgs a = make_args(c);
    a.rot = c->rot;
    TM_CUDA(c, cudaEventRecord(c->ev_start, c->stream));
    for (int o0 = 0; o0 < n; o0 += c->B) {
        a.orient0 = o0;
        a.nb = n - o0 < c->B ? n - o0 : c->B;
        a.gidx0 = pl.base + o0;
        int rc = c->var->run_batch_images(c, a, images, n_images);
        if (rc != TM_OK) return rc;
    }
    TM_CUDA(c, cudaEventRecord(c->ev_c, c->stream));
    int w = wait_stream(c, 3600.0);
    if (w != TM_OK) return w;
    int flag = 0;
    TM_CUDA(c, cudaMemcpy(&flag, c->err_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        cudaMemset(c->err_flag, 0, sizeof(int));
        return set_err(c, TM_ERR_TIMEOUT, "a bulk copy did not complete within its wait limit; results of this plane are invalid");
    }
    float tot = 0;
    cudaEventElapsedTime(&tot, c->ev_start, c->ev_c);
    c->last_total_ms = tot;
    c->last_prep_ms = c->last_b_ms = c->last_c_ms = 0;
    c->next_gidx += n;
    c->n_ccs += (long long)n * n_images;
    return TM_OK;
}

int tm_get_image_results(tm_ctx* c, int image, float* mip, float* best_psi, float* best_theta, float* best_phi) {
    if (!c || image < 0 || image >= (int)c->slots.size()) return TM_ERR_INVALID;
    TM_CUDA(c, cudaSetDevice(c->device));
    int rc = wait_stream(c, 3600.0);
    if (rc != TM_OK) return rc;
    const size_t n = (size_t)c->X * c->Y;
    const tm_ctx::Slot& sl = c->slots[image];
    if (mip) TM_CUDA(c, cudaMemcpy(mip, sl.mip, sizeof(float) * n, cudaMemcpyDeviceToHost));
    if (best_psi || best_theta || best_phi) {
        std::vector<int> best(n);
        TM_CUDA(c, cudaMemcpy(best.data(), sl.best, sizeof(int) * n, cudaMemcpyDeviceToHost));
        // planes are in increasing base order: binary search for the plane of each index
        std::vector<long long> bases(c->planes.size());
        for (size_t k = 0; k < bases.size(); k++) bases[k] = c->planes[k].base;
        for (size_t i = 0; i < n; i++) {
            const int g = best[i];
            float psi = 0, th = 0, ph = 0;
            const auto it = std::upper_bound(bases.begin(), bases.end(), (long long)g);
            if (g >= 0 && it != bases.begin()) {
                const Plane& p = c->planes[(size_t)(it - bases.begin()) - 1];
                const long long o = g - p.base;
                if (o >= 0 && o < p.n) {
                    const float* e = c->angle_lists[p.angles_id].data() + 3 * o;
                    ph = e[0];
                    th = e[1];
                    psi = e[2];
                }
            }
            if (best_psi) best_psi[i] = psi;
            if (best_theta) best_theta[i] = th;
            if (best_phi) best_phi[i] = ph;
        }
    }
    return TM_OK;
}

int tm_destroy(tm_ctx* c) {
    if (!c) return TM_ERR_INVALID;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_all(c);
    delete c;
    return TM_OK;
}

}  // extern "C"
