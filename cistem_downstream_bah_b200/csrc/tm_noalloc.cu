// tm_noalloc.cu -- plane search that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code running inside a host framework
// that owns every device allocation through its own pool (and forbids or
// cannot see outside allocations), and plugins whose host only hands them
// pre-allocated buffers.  tm_run_plane_noalloc serves them: the caller passes
// its own device buffers for the inputs and the running results, and every
// intermediate of the search lives in one file-scope device array of fixed
// size (kScratchBytes), which each GPU that loads this library keeps until
// the process exits.
#include <cuda_fp16.h>
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

// Offsets of the intermediates inside the scratch array for one geometry
// (256-byte aligned), and the bytes they need.
struct ScratchLayout {
    size_t tw, ip, rot, S, P, rs, norm, A, C, err, total;
    int XP, lmax;
};
__host__ __device__ constexpr size_t align256(size_t v) { return (v + 255) / 256 * 256; }
__host__ __device__ constexpr ScratchLayout scratch_layout(int T, int X, int Y, int W) {
    ScratchLayout L{};
    // the row pitch of the context path: X/2+1 in whole pass-B chunks, even
    L.XP = (X / 2 + 1 + W - 1) / W * W;
    if (L.XP % 2) L.XP += W;
    L.lmax = X > Y ? X : Y;
    const size_t TP = (size_t)T / 2 + 1;
    size_t off = 0;
    L.tw = off;   off = align256(off + sizeof(float2) * (size_t)L.lmax);
    L.ip = off;   off = align256(off + sizeof(float2) * (size_t)Y * L.XP);
    L.rot = off;  off = align256(off + sizeof(float) * 6 * kBatch);
    L.S = off;    off = align256(off + sizeof(float2) * (size_t)kBatch * T * TP);
    L.P = off;    off = align256(off + sizeof(float) * (size_t)kBatch * T * T);
    L.rs = off;   off = align256(off + sizeof(double) * (size_t)kBatch * T * 4);
    L.norm = off; off = align256(off + sizeof(float2) * kBatch);
    L.A = off;    off = align256(off + sizeof(float2) * (size_t)kBatch * T * L.XP);
    L.C = off;    off = align256(off + sizeof(float2) * (size_t)kBatch * Y * L.XP);
    L.err = off;  off = align256(off + sizeof(int));
    L.total = off;
    return L;
}

template <int T, int X, int Y>
struct NoAllocImpl {
    using LN = tmna::tmk::Launch<T, X, Y>;
    static constexpr ScratchLayout layout = scratch_layout(T, X, Y, LN::pass_b_width);
    // every compiled geometry fits the fixed array (checked when this file compiles)
    static_assert(layout.total <= kScratchBytes, "a no-alloc geometry exceeds the fixed scratch array");
    static cudaError_t configure(int XP, int bins) { return LN::configure(XP, bins); }
    static void run_batch(tmna::tmk::BatchArgs& a, cudaStream_t s, int nsm) {
        LN::prep(a, s);
        LN::pass_b(a, s, nsm);
        LN::pass_c(a, s);
    }
};

struct NoAllocVariant {
    int T, X, Y;
    ScratchLayout layout;
    cudaError_t (*configure)(int XP, int bins);
    void (*run_batch)(tmna::tmk::BatchArgs&, cudaStream_t, int);
};

#define TM_NOALLOC_VARIANT(T, X, Y) \
    {T, X, Y, NoAllocImpl<T, X, Y>::layout, &NoAllocImpl<T, X, Y>::configure, &NoAllocImpl<T, X, Y>::run_batch}

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

// The rotation rows of one batch travel as a kernel argument, so the host
// needs no staging buffer and no synchronisation between batches.
struct BatchRows {
    float m[6 * kBatch];
};
__global__ void k_noalloc_rows(BatchRows rows, float* dst, int n) {
    const int i = threadIdx.x;
    if (i < 6 * n) dst[i] = rows.m[i];
}

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

int run_noalloc(int device, const NoAllocVariant& var, const tm_dims* dims, const float* d_template_spectrum,
                const float* d_image_spectrum, const float* d_projection_filter, const float* euler_angles,
                int n_orientations, int first_orientation_index, float* d_mip, int* d_best, double* d_sum,
                double* d_sum_of_squares, unsigned long long* d_histogram, cudaStream_t s) {
    const int T = var.T, X = var.X, Y = var.Y;
    const ScratchLayout& L = var.layout;
    if (L.total > kScratchBytes) return TM_ERR_UNSUPPORTED;   // cannot happen: checked at compile time
    cudaError_t e;
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
                e = v.configure(v.layout.XP, 1024);
                if (e != cudaSuccess) return TM_ERR_CUDA;
            }
            su.scratch = static_cast<unsigned char*>(ptr);
            su.ready = true;
        }
    }
    unsigned char* base = g_setup[device].scratch;
    const int nsm = g_setup[device].nsm;

    tmna::tmk::BatchArgs a{};
    a.tmpl = reinterpret_cast<const float2*>(d_template_spectrum);
    a.filter = d_projection_filter;
    a.rot = reinterpret_cast<const float*>(base + L.rot);
    a.S = reinterpret_cast<float2*>(base + L.S);
    a.P = reinterpret_cast<float*>(base + L.P);
    a.rowstat = reinterpret_cast<double*>(base + L.rs);
    a.norm = reinterpret_cast<float2*>(base + L.norm);
    a.A = reinterpret_cast<float2*>(base + L.A);
    a.C = reinterpret_cast<float2*>(base + L.C);
    a.Ip = reinterpret_cast<const float2*>(base + L.ip);
    a.mip = d_mip;
    a.best = d_best;
    a.sum = d_sum;
    a.sumsq = d_sum_of_squares;
    a.hist = d_histogram;
    a.hist_min = (float)dims->histogram_min_scaled;
    a.hist_inv_step = (float)(1.0 / dims->histogram_step_scaled);
    a.hist_bins = dims->histogram_bins;
    a.XP = L.XP;
    a.err = reinterpret_cast<int*>(base + L.err);
    a.tw.tab = reinterpret_cast<const float2*>(base + L.tw);
    a.tw.lmax = L.lmax;
    a.twy = a.tw;   // the geometries here are powers of two: X, Y and T divide lmax
    a.twt = a.tw;

    // The array keeps the previous call's contents: rebuild the tables, clear
    // the error flag and the row spectra (their columns beyond X/2 are read as zero).
    k_noalloc_twiddles<<<(L.lmax + 255) / 256, 256, 0, s>>>(reinterpret_cast<float2*>(base + L.tw), L.lmax);
    tmna::tmk::k_prepare_image<<<dim3((L.XP + 127) / 128, Y), 128, 0, s>>>(
        reinterpret_cast<const float2*>(d_image_spectrum), reinterpret_cast<float2*>(base + L.ip), X, Y, L.XP, T);
    if (cudaMemsetAsync(base + L.err, 0, sizeof(int), s) != cudaSuccess) return TM_ERR_CUDA;
    if (cudaMemsetAsync(base + L.A, 0, sizeof(float2) * (size_t)kBatch * T * L.XP, s) != cudaSuccess) return TM_ERR_CUDA;
    BatchRows rows;
    for (int b0 = 0; b0 < n_orientations; b0 += kBatch) {
        const int nb = n_orientations - b0 < kBatch ? n_orientations - b0 : kBatch;
        euler_rows_noalloc(euler_angles + 3 * (size_t)b0, nb, rows.m);
        // stream order puts this after the previous batch's kernels have read the rows
        k_noalloc_rows<<<1, 6 * kBatch, 0, s>>>(rows, reinterpret_cast<float*>(base + L.rot), nb);
        a.nb = nb;
        a.orient0 = 0;
        a.gidx0 = (long long)first_orientation_index + b0;
        var.run_batch(a, s, nsm);
        if (cudaGetLastError() != cudaSuccess) return TM_ERR_CUDA;
    }
    int flag = 0;
    if (cudaMemcpyAsync(&flag, base + L.err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return TM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return TM_ERR_CUDA;
    return flag ? TM_ERR_TIMEOUT : TM_OK;
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
    const NoAllocVariant* var = nullptr;
    for (const NoAllocVariant& v : kNoAllocVariants)
        if (v.T == dims->template_size && v.X == dims->image_x && v.Y == dims->image_y) var = &v;
    if (!var) return TM_ERR_UNSUPPORTED;   // no compiled variant, or its intermediates exceed the array
    // the caller's current device is put back on every return path
    int caller_device = -1;
    if (cudaGetDevice(&caller_device) != cudaSuccess) return TM_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return TM_ERR_CUDA;
    const int rc = run_noalloc(device, *var, dims, d_template_spectrum, d_image_spectrum, d_projection_filter,
                               euler_angles, n_orientations, first_orientation_index, d_mip, d_best, d_sum,
                               d_sum_of_squares, d_histogram, static_cast<cudaStream_t>(stream));
    if (cudaSetDevice(caller_device) != cudaSuccess && rc == TM_OK) return TM_ERR_CUDA;
    return rc;
}
