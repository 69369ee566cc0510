// tm_gemm.cuh -- batched FP32 GEMMs for the small dense operators of the
// host-side preparation moved to the device (the pixel-size change of the
// projections in refine_template and of the template volume): k_gemm on the
// CUDA cores and k_gemm_tc on the tensor cores (split TF32, below).  Included
// inside a namespace by each translation unit that uses it.
//
// C = (A - s) B (+ C), row-major, one job per blockIdx.z with its own
// pointers.  128 x 128 tiles, 8-deep k slices double-buffered through shared
// memory (the next slice is loaded into registers while the current one is
// multiplied), 8 x 8 outputs per thread as four 4 x 4 quadrants so that the
// shared-memory reads of a warp are conflict-free.
struct GemmJob {
    const float* A;
    const float* B;
    float* C;
    const float* s;   // scalar subtracted from A, or null
};

__global__ void __launch_bounds__(256) k_gemm(const GemmJob* __restrict__ jobs, int M, int N, int K, int lda, int ldb,
                                              int ldc, int accumulate) {
    constexpr int BM = 128, BN = 128, BK = 8;
    __shared__ __align__(16) float As[2][BK][BM];
    __shared__ __align__(16) float Bs[2][BK][BN];
    const GemmJob g = jobs[blockIdx.z];
    const float sub = g.s ? *g.s : 0.0f;
    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;   // output quadrant rows ty*4 (+64), cols tx*4 (+64)
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    // loader mapping: A slice 128 x 8 (4 per thread: rows am + 32 q, column ak);
    // B slice 8 x 128 (4 per thread: row bk, columns bn + 32 q)
    const int am = tid / BK, ak = tid % BK;
    const int bk = tid / 32, bn = tid % 32;
    float ra[4], rb[4];
    auto load = [&](int k0) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int gm = m0 + am + 32 * q, gk = k0 + ak;
            ra[q] = (gm < M && gk < K) ? g.A[(size_t)gm * lda + gk] - sub : 0.0f;
            const int hk = k0 + bk, hn = n0 + bn + 32 * q;
            rb[q] = (hk < K && hn < N) ? g.B[(size_t)hk * ldb + hn] : 0.0f;
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            As[buf][ak][am + 32 * q] = ra[q];
            Bs[buf][bk][bn + 32 * q] = rb[q];
        }
    };
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.0f;
    load(0);
    store(0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < K; k0 += BK) {
        const bool more = k0 + BK < K;
        if (more) load(k0 + BK);
#pragma unroll
        for (int k = 0; k < BK; k++) {
            float a[8], b[8];
            const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][k][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][k][64 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][k][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][k][64 + tx * 4]);
            a[0] = a0.x; a[1] = a0.y; a[2] = a0.z; a[3] = a0.w;
            a[4] = a1.x; a[5] = a1.y; a[6] = a1.z; a[7] = a1.w;
            b[0] = b0.x; b[1] = b0.y; b[2] = b0.z; b[3] = b0.w;
            b[4] = b1.x; b[5] = b1.y; b[6] = b1.z; b[7] = b1.w;
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        if (more) {
            store(buf ^ 1);
            __syncthreads();
            buf ^= 1;
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int gm = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int gn = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
            if (gn >= N) continue;
            float* c = g.C + (size_t)gm * ldc + gn;
            *c = accumulate ? *c + acc[i][j] : acc[i][j];
        }
    }
}

// --------------------------------------------------------------------------------------
// k_gemm_tc: the same product on the tensor cores.  Each FP32 operand value is
// split as x = hi + lo, hi = x with its 13 low mantissa bits cleared (exactly a
// TF32 value) and lo = x - hi (exact in FP32), and every K step issues three
// kind::tf32 MMAs, hi*hi + hi*lo + lo*hi, accumulating in FP32 in tensor
// memory; the dropped lo*lo term and the TF32 part of lo leave about 2^-20 of
// each product.  Block: 256 threads, a 128 x 128 tile of C (one TMEM lane per
// row, 128 columns), K in slices of 32.  The threads load slice c + 1 into
// registers while the tensor core multiplies slice c, then split it into the
// other shared-memory stage once the MMAs of slice c - 1 are done with it: the
// A slice one K index per lane (each warp load is one 128-byte row segment),
// the B slice one N index per thread and four K values per 16-byte store.
//
// Operand layout (both K-major, no swizzle): element (r, k) of a 128 x 32
// slice at (r % 8) * 16 + (k % 4) * 4 + (r / 8) * 128 + (k / 4) * GEMM_TC_LBO;
// the K groups are 16 bytes further apart than a dense layout, so that the 32
// lanes' 4-byte A stores fall in 32 different banks.
constexpr int GEMM_TC_BK = 32;
constexpr int GEMM_TC_NT = 256;
constexpr int GEMM_TC_SBO = 128;
constexpr int GEMM_TC_LBO = 16 * 128 + 16;
constexpr int GEMM_TC_TILE = (GEMM_TC_BK / 4) * GEMM_TC_LBO;   // one 128 x 32 operand slice
constexpr int GEMM_TC_STAGE = 4 * GEMM_TC_TILE;                // A hi, A lo, B hi, B lo
constexpr int GEMM_TC_SMEM = 128 + 2 * GEMM_TC_STAGE;
// values of one slice per thread: A 128 x 32 and B 32 x 128 over 256 threads
constexpr int GEMM_TC_PA = 128 * GEMM_TC_BK / GEMM_TC_NT;
constexpr int GEMM_TC_PB = 128 * GEMM_TC_BK / GEMM_TC_NT;

__device__ __forceinline__ uint32_t gemm_tc_off(int r, int k) {
    return (uint32_t)((r % 8) * 16 + (k % 4) * 4 + (r / 8) * GEMM_TC_SBO + (k / 4) * GEMM_TC_LBO);
}

__global__ void __launch_bounds__(GEMM_TC_NT, 1)
k_gemm_tc(const GemmJob* __restrict__ jobs, int M, int N, int K, int lda, int ldb, int ldc, int accumulate, int* err) {
    constexpr uint32_t kWaitLimit = 1u << 24;
    constexpr int PA = GEMM_TC_PA, PB = GEMM_TC_PB;
    extern __shared__ __align__(128) unsigned char smem_g[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_g);   // [0], [1]: MMAs of slices in stage 0 / 1
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem_g + 64);
    unsigned char* stage0 = smem_g + 128;
    const GemmJob g = jobs[blockIdx.z];
    const float sub = g.s ? *g.s : 0.0f;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int m0 = blockIdx.y * 128, n0 = blockIdx.x * 128;
    const int nk = (K + GEMM_TC_BK - 1) / GEMM_TC_BK;
    if (t == 0) {
        tmptx::mbar_init(&mbar[0], 1);
        tmptx::mbar_init(&mbar[1], 1);
    }
    if (warp == 0) {
        tmptx::tmem_alloc(tmem_slot, 128);
        tmptx::tmem_relinquish();
    }
    // this thread's share of a slice: A rows warp + 8 i at K index lane; B column
    // n0 + (t % 128) at the K groups (t / 128) + 2 j
    const int bn = t % 128, bq0 = t / 128;
    float ra[PA], rb[PB];
    auto load = [&](int c) {
        const int k0 = c * GEMM_TC_BK;
        const int ka = k0 + lane;
#pragma unroll
        for (int i = 0; i < PA; i++) {
            const int gm = m0 + warp + 8 * i;
            ra[i] = (gm < M && ka < K) ? g.A[(size_t)gm * lda + ka] - sub : 0.0f;
        }
        const int gn = n0 + bn;
#pragma unroll
        for (int j = 0; j < PB / 4; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int hk = k0 + 4 * (bq0 + 2 * j) + e;
                rb[4 * j + e] = (gn < N && hk < K) ? g.B[(size_t)hk * ldb + gn] : 0.0f;
            }
    };
    auto split = [](float x, float& hi, float& lo) {
        hi = __uint_as_float(__float_as_uint(x) & 0xffffe000u);
        lo = x - hi;
    };
    // the registers of a slice, split, into stage buffer `buf`
    auto store = [&](int buf) {
        unsigned char* base = stage0 + buf * GEMM_TC_STAGE;
        unsigned char *ahi = base, *alo = base + GEMM_TC_TILE, *bhi = base + 2 * GEMM_TC_TILE, *blo = base + 3 * GEMM_TC_TILE;
#pragma unroll
        for (int i = 0; i < PA; i++) {
            float hi, lo;
            split(ra[i], hi, lo);
            const uint32_t o = gemm_tc_off(warp + 8 * i, lane);
            *reinterpret_cast<float*>(ahi + o) = hi;
            *reinterpret_cast<float*>(alo + o) = lo;
        }
#pragma unroll
        for (int j = 0; j < PB / 4; j++) {
            float h[4], l[4];
#pragma unroll
            for (int e = 0; e < 4; e++) split(rb[4 * j + e], h[e], l[e]);
            const uint32_t o = gemm_tc_off(bn, 4 * (bq0 + 2 * j));
            *reinterpret_cast<float4*>(bhi + o) = make_float4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<float4*>(blo + o) = make_float4(l[0], l[1], l[2], l[3]);
        }
        tmptx::fence_proxy_async_smem();
    };
    bool timed_out = false;
    auto wait_slice = [&](int c) {   // slice c's commit completes phase c >> 1 of mbar[c & 1]
        if (!tmptx::mbar_wait_bounded(&mbar[c & 1], (c >> 1) & 1, kWaitLimit)) timed_out = true;
    };
    load(0);
    store(0);
    if (nk > 1) load(1);
    tmptx::tmem_fence_before_sync();
    __syncthreads();
    tmptx::tmem_fence_after_sync();
    const uint32_t tbase = *tmem_slot;
    const uint32_t idesc = tmptx::idesc_tf32_f32(128, 128);
    const uint32_t s_addr = tmptx::smem_u32(stage0);
    int issued = 0;
    for (int c = 0; c < nk; c++) {
        const int buf = c & 1;
        if (t == 0) {
            tmptx::tmem_fence_after_sync();
            const uint32_t a_hi = s_addr + buf * GEMM_TC_STAGE, a_lo = a_hi + GEMM_TC_TILE;
            const uint32_t b_hi = a_hi + 2 * GEMM_TC_TILE, b_lo = a_hi + 3 * GEMM_TC_TILE;
#pragma unroll
            for (int kk = 0; kk < GEMM_TC_BK / 8; kk++) {
                const uint32_t ko = kk * 2 * GEMM_TC_LBO;
                const uint64_t dah = tmptx::smem_desc_noswizzle(a_hi + ko, GEMM_TC_LBO, GEMM_TC_SBO);
                const uint64_t dal = tmptx::smem_desc_noswizzle(a_lo + ko, GEMM_TC_LBO, GEMM_TC_SBO);
                const uint64_t dbh = tmptx::smem_desc_noswizzle(b_hi + ko, GEMM_TC_LBO, GEMM_TC_SBO);
                const uint64_t dbl = tmptx::smem_desc_noswizzle(b_lo + ko, GEMM_TC_LBO, GEMM_TC_SBO);
                tmptx::mma_tf32_ss(tbase, dah, dbh, idesc, c > 0 || kk > 0);
                tmptx::mma_tf32_ss(tbase, dah, dbl, idesc, true);
                tmptx::mma_tf32_ss(tbase, dal, dbh, idesc, true);
            }
            tmptx::mma_commit(&mbar[buf]);
        }
        issued = c + 1;
        if (c + 1 < nk) {
            if (c >= 1) wait_slice(c - 1);   // the other buffer was read by slice c - 1
            store(buf ^ 1);                  // slice c + 1, loaded during slice c
            if (c + 2 < nk) load(c + 2);     // in flight during the MMAs of slice c + 1
            tmptx::tmem_fence_before_sync();
            if (__syncthreads_or(timed_out)) break;
            tmptx::tmem_fence_after_sync();
        }
    }
    // the last commit covers every MMA issued before it
    wait_slice(issued - 1);
    tmptx::tmem_fence_after_sync();
    const bool failed = __syncthreads_or(timed_out);
    if (failed) {
        if (t == 0 && err) atomicExch(err, 1);
    } else {
        // row m0 + 32 (warp % 4) + lane of the tile, columns 64 (warp / 4) .. + 63, 16 at a time
        const int gm = m0 + 32 * (warp & 3) + lane;
        const uint32_t trow = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + 64 * (warp >> 2);
#pragma unroll 1
        for (int j = 0; j < 4; j++) {
            float v[16];
            tmptx::tmem_ld16(trow + 16 * j, v);
            tmptx::tmem_wait_ld16(v);
            const int nc = n0 + 64 * (warp >> 2) + 16 * j;
            if (gm < M) {
                float* crow = g.C + (size_t)gm * ldc + nc;
                if (nc + 16 <= N && ((reinterpret_cast<uintptr_t>(crow) & 15) == 0)) {
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        float4 o = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                        if (accumulate) {
                            const float4 p = reinterpret_cast<const float4*>(crow)[q];
                            o.x += p.x; o.y += p.y; o.z += p.z; o.w += p.w;
                        }
                        reinterpret_cast<float4*>(crow)[q] = o;
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 16; i++)
                        if (nc + i < N) crow[i] = accumulate ? crow[i] + v[i] : v[i];
                }
            }
        }
    }
    tmptx::tmem_fence_before_sync();
    __syncthreads();
    tmptx::tmem_fence_after_sync();
    if (warp == 0) tmptx::tmem_dealloc(tbase, 128);
}

// Launch of k_gemm_tc over n_jobs jobs on the current device; err (may be
// null) is set to 1 if an MMA completion wait ran out (C is then not written).
inline cudaError_t gemm_tc(const GemmJob* jobs, int n_jobs, int M, int N, int K, int lda, int ldb, int ldc,
                           int accumulate, int* err, cudaStream_t s) {
    const cudaError_t e = cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_TC_SMEM);
    if (e != cudaSuccess) return e;
    k_gemm_tc<<<dim3((N + 127) / 128, (M + 127) / 128, n_jobs), GEMM_TC_NT, GEMM_TC_SMEM, s>>>(jobs, M, N, K, lda, ldb, ldc,
                                                                                    accumulate, err);
    return cudaGetLastError();
}
