// tm_noalloc.cu -- plane search that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code running inside a host framework
// that owns every device allocation through its own pool (and forbids or
// cannot see outside allocations), plugins whose host only hands them
// pre-allocated buffers, and code that must not allocate while a stream is
// being captured into a CUDA graph.  tm_run_plane_noalloc serves them: the
// caller passes its own device buffers for the inputs and the running
// results, and every intermediate of the search lives in one file-scope
// device array of fixed size (kScratchBytes), which each GPU that loads this
// library keeps until the process exits.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "../../include/tm_b200.h"

// The search kernels, instantiated in their own namespace so that this
// translation unit's instantiations stay separate from the context path's.
namespace tmna {
#include "tm_kernels.cuh"
}

namespace {

constexpr size_t kScratchBytes = (size_t)16 << 20;   // 16 MiB per device
constexpr int kBatch = 8;                             // orientations per device pass
constexpr int kMaxDevices = 64;

// All intermediates of tm_run_plane_noalloc: twiddle table, prepared
// micrograph spectrum, rotation rows, slice spectra, projections, row sums,
// normalisation, row spectra, correlation spectra and the error flag.
static __device__ __align__(256) unsigned char tm_noalloc_scratch[kScratchBytes];

struct DeviceSetup {
    bool ready = false;
    unsigned char* scratch = nullptr;   // device address of tm_noalloc_scratch on this device
    int nsm = 0;
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

template <int T, int X, int Y>
struct NoAllocImpl {
    using LN = tmna::tmk::Launch<T, X, Y>;
    static cudaError_t configure(int XP, int bins) { return LN::configure(XP, bins); }
    static void run_batch(tmna::tmk::BatchArgs& a, cudaStream_t s, int nsm) {
        LN::prep(a, s);
        LN::pass_b(a, s, nsm);
        LN::pass_c(a, s);
    }
    static int pass_b_width() { return LN::pass_b_width; }
};

struct NoAllocVariant {
    int T, X, Y;
    cudaError_t (*configure)(int XP, int bins);
    void (*run_batch)(tmna::tmk::BatchArgs&, cudaStream_t, int);
    int (*pass_b_width)();
};

#define TM_NOALLOC_VARIANT(T, X, Y) \
    {T, X, Y, &NoAllocImpl<T, X, Y>::configure, &NoAllocImpl<T, X, Y>::run_batch, &NoAllocImpl<T, X, Y>::pass_b_width}

const NoAllocVariant kNoAllocVariants[] = {
    TM_NOALLOC_VARIANT(32, 256, 256),
    TM_NOALLOC_VARIANT(32, 512, 512),
    TM_NOALLOC_VARIANT(64, 512, 512),
};

// twiddle table W_L^m = exp(-2 pi i m / L), as the context path builds on the host
__global__ void k_noalloc_twiddles(float2* tab, int L) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < L) {
        double s, c;
        sincospi(-2.0 * (double)m / (double)L, &s, &c);
        tab[m] = make_float2((float)c, (float)s);
    }
}

// I'[ky][kx] = I[ky][kx] * exp(+2 pi i (kx*x0/X + ky*y0/Y)) / N, I'[0][0] = 0 and
// zero pitch padding: the preparation of tm_set_image, on the device
__global__ void k_noalloc_prepare(const float2* __restrict__ spec, float2* __restrict__ ip, int X, int Y, int XP, int T) {
    const int kx = blockIdx.x * blockDim.x + threadIdx.x;
    const int ky = blockIdx.y;
    if (kx >= XP) return;
    const int hc = X / 2 + 1;
    float2 out = make_float2(0.f, 0.f);
    if (kx < hc && !(kx == 0 && ky == 0)) {
        const long long x0 = X / 2 - T / 2, y0 = Y / 2 - T / 2;
        double sx, cx, sy, cy;
        sincospi(2.0 * (double)((kx * x0) % X) / (double)X, &sx, &cx);
        sincospi(2.0 * (double)((ky * y0) % Y) / (double)Y, &sy, &cy);
        const double pr = cx * cy - sx * sy, pi = cx * sy + sx * cy;
        const float2 v = spec[(size_t)ky * hc + kx];
        const double invn = 1.0 / ((double)X * (double)Y);
        out = make_float2((float)(((double)v.x * pr - (double)v.y * pi) * invn),
                          (float)(((double)v.x * pi + (double)v.y * pr) * invn));
    }
    ip[(size_t)ky * XP + kx] = out;
}

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

// Euler rows in float as RotationMatrix::SetToEulerRotation (matrix.cpp:490-510)
void euler_rows_noalloc(const float* ang, int n, float* rot) {
    const float pif = 3.14159265359f;
    auto d2r = [pif](float deg) { return (float)((double)(deg * pif) / 180.); };
    for (int o = 0; o < n; o++) {
        const float cphi = cosf(d2r(ang[3 * o])), sphi = sinf(d2r(ang[3 * o]));
        const float cth = cosf(d2r(ang[3 * o + 1])), sth = sinf(d2r(ang[3 * o + 1]));
        const float cpsi = cosf(d2r(ang[3 * o + 2])), spsi = sinf(d2r(ang[3 * o + 2]));
        float* m = rot + 6 * (size_t)o;
        m[0] = cphi * cth * cpsi - sphi * spsi;
        m[1] = -cphi * cth * spsi - sphi * cpsi;
        m[2] = sphi * cth * cpsi + cphi * spsi;
        m[3] = -sphi * cth * spsi + cphi * cpsi;
        m[4] = -sth * cpsi;
        m[5] = sth * spsi;
    }
}

}  // namespace

extern "C" int tm_run_plane_noalloc(int device, const tm_dims* dims, const float* d_template_spectrum,
                                    const float* d_image_spectrum, const float* d_projection_filter,
                                    const float* euler_angles, int n_orientations, int first_orientation_index,
                                    float* d_mip, int* d_best, double* d_sum, double* d_sum_of_squares,
                                    unsigned long long* d_histogram, void* stream) {
    if (!dims || !d_template_spectrum || !d_image_spectrum || !d_projection_filter || !d_mip || !d_best || !d_sum ||
        !d_sum_of_squares || !d_histogram || n_orientations < 0 || (n_orientations > 0 && !euler_angles))
        return TM_ERR_INVALID;
    if (device < 0 || device >= kMaxDevices) return TM_ERR_INVALID;
    if (dims->histogram_bins <= 0 || dims->histogram_bins > 1024 || !(dims->histogram_step_scaled > 0))
        return TM_ERR_INVALID;
    if ((long long)first_orientation_index + n_orientations > 2147483647LL || first_orientation_index < 0)
        return TM_ERR_INVALID;
    const int T = dims->template_size, X = dims->image_x, Y = dims->image_y;
    const NoAllocVariant* var = nullptr;
    for (const NoAllocVariant& v : kNoAllocVariants)
        if (v.T == T && v.X == X && v.Y == Y) var = &v;
    if (!var) return TM_ERR_UNSUPPORTED;
    const int W = var->pass_b_width();
    const int XP = (X / 2 + 1 + W - 1) / W * W;
    const int TP = T / 2 + 1;
    // scratch layout
    const int lmax = X > Y ? X : Y;
    size_t off = 0;
    const size_t o_tw = off;      off = align256(off + sizeof(float2) * lmax);
    const size_t o_ip = off;      off = align256(off + sizeof(float2) * (size_t)Y * XP);
    const size_t o_rot = off;     off = align256(off + sizeof(float) * 6 * kBatch);
    const size_t o_S = off;       off = align256(off + sizeof(float2) * (size_t)kBatch * T * TP);
    const size_t o_P = off;       off = align256(off + sizeof(float) * (size_t)kBatch * T * T);
    const size_t o_rs = off;      off = align256(off + sizeof(double) * (size_t)kBatch * T * 4);
    const size_t o_norm = off;    off = align256(off + sizeof(float2) * kBatch);
    const size_t o_A = off;       off = align256(off + sizeof(float2) * (size_t)kBatch * T * XP);
    const size_t o_C = off;       off = align256(off + sizeof(float2) * (size_t)kBatch * Y * XP);
    const size_t o_err = off;     off = align256(off + sizeof(int));
    if (off > kScratchBytes) return TM_ERR_UNSUPPORTED;   // exceeds the fixed scratch size

    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return TM_ERR_CUDA;
    {
        // once per device, with that device current: the device address of the
        // scratch array and the kernels' shared-memory limits
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        DeviceSetup& su = g_setup[device];
        if (!su.ready) {
            void* ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, tm_noalloc_scratch);
            if (e != cudaSuccess || !ptr) return TM_ERR_CUDA;
            e = cudaDeviceGetAttribute(&su.nsm, cudaDevAttrMultiProcessorCount, device);
            if (e != cudaSuccess) return TM_ERR_CUDA;
            for (const NoAllocVariant& v : kNoAllocVariants) {
                const int w = v.pass_b_width();
                const int xp = (v.X / 2 + 1 + w - 1) / w * w;
                e = v.configure(xp, 1024);
                if (e != cudaSuccess) return TM_ERR_CUDA;
            }
            su.scratch = static_cast<unsigned char*>(ptr);
            su.ready = true;
        }
    }
    unsigned char* base = g_setup[device].scratch;
    const int nsm = g_setup[device].nsm;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    tmna::tmk::BatchArgs a{};
    a.tmpl = reinterpret_cast<const float2*>(d_template_spectrum);
    a.filter = d_projection_filter;
    a.rot = reinterpret_cast<const float*>(base + o_rot);
    a.S = reinterpret_cast<float2*>(base + o_S);
    a.P = reinterpret_cast<float*>(base + o_P);
    a.rowstat = reinterpret_cast<double*>(base + o_rs);
    a.norm = reinterpret_cast<float2*>(base + o_norm);
    a.A = reinterpret_cast<float2*>(base + o_A);
    a.C = reinterpret_cast<float2*>(base + o_C);
    a.Ip = reinterpret_cast<const float2*>(base + o_ip);
    a.mip = d_mip;
    a.best = d_best;
    a.sum = d_sum;
    a.sumsq = d_sum_of_squares;
    a.hist = d_histogram;
    a.hist_min = (float)dims->histogram_min_scaled;
    a.hist_inv_step = (float)(1.0 / dims->histogram_step_scaled);
    a.hist_bins = dims->histogram_bins;
    a.XP = XP;
    a.err = reinterpret_cast<int*>(base + o_err);
    a.tw.tab = reinterpret_cast<const float2*>(base + o_tw);
    a.tw.lmax = lmax;
    a.twy = a.tw;   // the geometries here are powers of two: X, Y and T divide lmax
    a.twt = a.tw;

    // The array keeps the previous call's contents: rebuild the tables, clear
    // the error flag and the row spectra (their columns beyond X/2 are read as zero).
    k_noalloc_twiddles<<<(lmax + 255) / 256, 256, 0, s>>>(reinterpret_cast<float2*>(base + o_tw), lmax);
    k_noalloc_prepare<<<dim3((XP + 127) / 128, Y), 128, 0, s>>>(reinterpret_cast<const float2*>(d_image_spectrum),
                                                                reinterpret_cast<float2*>(base + o_ip), X, Y, XP, T);
    if ((e = cudaMemsetAsync(base + o_err, 0, sizeof(int), s)) != cudaSuccess) return TM_ERR_CUDA;
    if ((e = cudaMemsetAsync(base + o_A, 0, sizeof(float2) * (size_t)kBatch * T * XP, s)) != cudaSuccess) return TM_ERR_CUDA;
    float rot[6 * kBatch];
    for (int b0 = 0; b0 < n_orientations; b0 += kBatch) {
        const int nb = n_orientations - b0 < kBatch ? n_orientations - b0 : kBatch;
        euler_rows_noalloc(euler_angles + 3 * (size_t)b0, nb, rot);
        // the rows of the previous batch may still be in use: order the copy on the stream
        if ((e = cudaMemcpyAsync(base + o_rot, rot, sizeof(float) * 6 * nb, cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return TM_ERR_CUDA;
        // the host array is reused next iteration: wait until the copy has consumed it
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return TM_ERR_CUDA;
        a.nb = nb;
        a.orient0 = 0;
        a.gidx0 = (long long)first_orientation_index + b0;
        var->run_batch(a, s, nsm);
        if ((e = cudaGetLastError()) != cudaSuccess) return TM_ERR_CUDA;
    }
    int flag = 0;
    if ((e = cudaMemcpyAsync(&flag, base + o_err, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return TM_ERR_CUDA;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return TM_ERR_CUDA;
    return flag ? TM_ERR_TIMEOUT : TM_OK;
}
