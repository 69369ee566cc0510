// tm_gemm.cuh -- a batched FP32 GEMM for the small dense operators of the
// host-side preparation moved to the device (the pixel-size change of the
// projections in refine_template and of the template volume).  Included
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
