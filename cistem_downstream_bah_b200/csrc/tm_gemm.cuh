// tm_gemm.cuh -- a batched FP32 GEMM for the small dense operators of the
// host-side preparation moved to the device (the pixel-size change of the
// projections in refine_template and of the template volume).  Included
// inside a namespace by each translation unit that uses it.
// C = (A - s) B (+ C): row-major, per job pointers; 64 x 64 tiles, 4 x 4 per thread
struct GemmJob {
    const float* A;
    const float* B;
    float* C;
    const float* s;   // scalar subtracted from A, or null
};

__global__ void __launch_bounds__(256) k_gemm(const GemmJob* __restrict__ jobs, int M, int N, int K, int lda, int ldb,
                                              int ldc, int accumulate) {
    constexpr int BM = 64, BN = 64, BK = 16;
    __shared__ float As[BK][BM + 4];
    __shared__ float Bs[BK][BN + 4];
    const GemmJob g = jobs[blockIdx.z];
    const float sub = g.s ? *g.s : 0.0f;
    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += BK) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int e = tid + 256 * q;          // 0..1023
            const int am = e / BK, ak = e % BK;   // A tile: BM x BK
            const int gm = m0 + am, gk = k0 + ak;
            As[ak][am] = (gm < M && gk < K) ? g.A[(size_t)gm * lda + gk] - sub : 0.0f;
            const int bk = e / BN, bn = e % BN;   // B tile: BK x BN
            const int hk = k0 + bk, hn = n0 + bn;
            Bs[bk][bn] = (hk < K && hn < N) ? g.B[(size_t)hk * ldb + hn] : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < BK; k++) {
            float av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; i++) av[i] = As[k][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) bv[j] = Bs[k][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int gm = m0 + ty * 4 + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int gn = n0 + tx * 4 + j;
            if (gn >= N) continue;
            float* c = g.C + (size_t)gm * ldc + gn;
            *c = accumulate ? *c + acc[i][j] : acc[i][j];
        }
    }
}
