// tm_tensor.cuh -- FP16 tensor-core form of the row pass (pass C).
//
// The FP16 form of the search keeps the slice, projection and column kernels
// (k_pass_b stores its correlation spectra as FP16 complex, scaled by 2^e so
// that the row outputs are O(1), rows interleaved in blocks of R) and replaces
// k_pass_c by k_pass_c_tc: per block of R rows, for one orientation at a time,
//
//   pre-processing   the half-complex row Z[k] (k = 0..X/2) becomes the
//                    H = X/2-point complex sequence v[k] whose inverse FFT packs
//                    the real row (pixels 2n, 2n+1 = Re, Im of z[n]) -- the same
//                    packing as k_pass_c -- and is written, FP16, as the A
//                    operand of stage 1
//   stage 1 (MMA)    H = N1 x 64: for every k1 the 64-point inverse DFT over
//                    k2 of v[k1 + N1 k2], as one 128 x 128 x 64 tcgen05.mma
//                    (A = data, M = (row, k1, re/im); B = [cos | sin] of the
//                    64-point DFT, K = k2), FP32 accumulators in TMEM
//   epilogue 1       TMEM -> registers, re/im parts combined across lane
//                    pairs, twiddle exp(+2 pi i k1 n2 / H), FP16 A operand of
//                    stage 2 for each row
//   stage 2 (MMA)    for every n2 the N1-point inverse DFT over k1, one
//                    128 x 2N1 x N1 tcgen05.mma per row (K padded to 16)
//   epilogue 2       TMEM -> registers, re/im combined, z[n2 + 64 n1] scaled
//                    by 2^-e, and the MIP / argmax / compensated sums /
//                    histogram update of k_pass_c (match_template.cpp:1102-1149)
//
// R = 64 / N1 = 8192 / X rows, so that stage 1 is always M = 128 and every
// block holds 8192 pixels: 512 threads, 16 pixels each, their MIP, argmax and
// sum in registers and their sum of squares and the two compensation terms in
// TMEM.  The operands use the tensor core's no-swizzle layout of 8 x 8 core
// matrices (tmptx::smem_desc_noswizzle); the A operands are MN-major with their
// M groups 144 bytes apart, so that the epilogue's 16-byte stores of
// neighbouring lanes fall in different banks.
#pragma once
#include <cuda_fp16.h>

#include "tm_ptx.cuh"

namespace tmk {

template <int X>
struct PassCTc {
    static constexpr int H = X / 2;
    static constexpr int N2 = 64;                    // stage-1 DFT length
    static constexpr int N1 = H / N2;                // stage-2 DFT length
    static constexpr int R = N2 / N1;                // rows per block (8192 / X)
    static constexpr int K2 = N1 < 16 ? 16 : N1;     // stage-2 K, padded to the MMA's K step
    static constexpr int NT = 512;
    static constexpr int SBO_A = 144;                // A operands: M groups (16 B rows of 8 elements)
    static constexpr int LBO_A = 16 * SBO_A;         // K groups (M = 128: 16 M groups)
    static constexpr int A1_BYTES = (64 / 8) * LBO_A;
    static constexpr int A2_BYTES = (K2 / 8) * LBO_A;   // per row
    static constexpr int B1_N = 128, B1_K = 64;      // [cos | sin] of the 64-point DFT
    static constexpr int B2_N = 2 * N1, B2_K = K2;   // [cos | sin] of the N1-point DFT
    static constexpr int SBO_B = 128;                // B operands (K-major): N groups
    static constexpr int LBO_B1 = (B1_N / 8) * 128;  // K groups
    static constexpr int LBO_B2 = (B2_N / 8) * 128;
    static constexpr int B1_BYTES = (B1_K / 8) * LBO_B1;
    static constexpr int B2_BYTES = (B2_K / 8) * LBO_B2;
    static constexpr int TM_D1 = 0;                  // TMEM columns: stage-1 accumulator
    static constexpr int TM_D2 = 128;                // stage-2 accumulators, 2 N1 per row
    static constexpr int TM_STATE = 256;             // 48 per warp of a lane quadrant
    static constexpr uint32_t TMEM_COLS = 512;
    static constexpr int OFF_B1 = 128;
    static constexpr int OFF_B2 = OFF_B1 + B1_BYTES;
    static constexpr int OFF_A1 = OFF_B2 + B2_BYTES;
    static constexpr int OFF_A2 = OFF_A1 + A1_BYTES;
    static constexpr int OFF_ROWS = OFF_A2 + R * A2_BYTES;
    static_assert(N1 >= 2 && N1 * N2 == H && R * N1 == 64, "row length must be 2 * 64 * N1");
    static_assert(B2_N % 16 == 0 && B2_N <= 256, "stage-2 N must be a multiple of 16");
    static_assert(OFF_ROWS % 16 == 0, "operand regions 16-byte aligned");
    // bytes of one staged row block: R rows x XP FP16 complex values
    __host__ __device__ static size_t block_bytes(int XP) { return (size_t)XP * R * 4; }
    static constexpr int HIST_COPIES = 16;           // copies of the shared histogram (hist_copies)
    static size_t smem_bytes(int XP, int bins) {
        return OFF_ROWS + 2 * block_bytes(XP) + 4 * (size_t)bins * hist_copies(bins, HIST_COPIES);
    }
};

// The DFT matrices of the two stages as FP16 B operands, in the byte layout the
// kernel copies into shared memory: B1 (K = k2, N = [cos n2 | sin n2]) then B2
// (K = k1 padded to K2 with zero rows, N = [cos n1 | sin n1]).  Filled on the
// host; entry (n, k) of a K-major operand with N groups `sbo` and K groups `lbo`
// apart sits at (n % 8) * 16 + (k % 8) * 2 + (n / 8) * sbo + (k / 8) * lbo.
template <int X>
void fill_tc_dft(uint16_t* out) {
    using PC = PassCTc<X>;
    auto put = [](uint16_t* base, int n, int k, int sbo, int lbo, double v) {
        const __half h = __double2half(v);
        base[((n % 8) * 16 + (k % 8) * 2 + (n / 8) * sbo + (k / 8) * lbo) / 2] = *reinterpret_cast<const uint16_t*>(&h);
    };
    uint16_t* b1 = out;
    uint16_t* b2 = out + PC::B1_BYTES / 2;
    for (int i = 0; i < (PC::B1_BYTES + PC::B2_BYTES) / 2; i++) out[i] = 0;
    for (int k = 0; k < 64; k++)
        for (int n = 0; n < 64; n++) {
            const double th = 2.0 * M_PI * (double)((k * n) % 64) / 64.0;
            put(b1, n, k, PC::SBO_B, PC::LBO_B1, cos(th));
            put(b1, 64 + n, k, PC::SBO_B, PC::LBO_B1, sin(th));
        }
    for (int k = 0; k < PC::N1; k++)
        for (int n = 0; n < PC::N1; n++) {
            const double th = 2.0 * M_PI * (double)((k * n) % PC::N1) / (double)PC::N1;
            put(b2, n, k, PC::SBO_B, PC::LBO_B2, cos(th));
            put(b2, PC::N1 + n, k, PC::SBO_B, PC::LBO_B2, sin(th));
        }
}

// byte offset of element (m, k) in an MN-major A operand (M = 128)
template <int X>
__device__ __forceinline__ uint32_t a_off(int m, int k) {
    using PC = PassCTc<X>;
    return (uint32_t)((m % 8) * 2 + (k % 8) * 16 + (m / 8) * PC::SBO_A + (k / 8) * PC::LBO_A);
}

__device__ __forceinline__ uint32_t h2_bits(float a, float b) {
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

template <int X>
__global__ void __launch_bounds__(512, 1)
k_pass_c_tc(BatchArgs a, int Y, const uint4* __restrict__ dft) {
    using PC = PassCTc<X>;
    constexpr int H = PC::H, N1 = PC::N1, R = PC::R, K2 = PC::K2;
    constexpr uint32_t kWaitLimit = 1u << 24;
    const int XP = a.XP;
    extern __shared__ __align__(128) unsigned char smem_t[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_t);   // [0], [1]: row blocks; [2], [3]: stage-1 / stage-2 MMAs
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem_t + 64);
    unsigned char* sB1 = smem_t + PC::OFF_B1;
    unsigned char* sB2 = smem_t + PC::OFF_B2;
    unsigned char* sA1 = smem_t + PC::OFF_A1;
    unsigned char* sA2 = smem_t + PC::OFF_A2;
    unsigned char* rows = smem_t + PC::OFF_ROWS;
    const size_t blk = PC::block_bytes(XP);
    unsigned int* shist = reinterpret_cast<unsigned int*>(rows + 2 * blk);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int q = warp & 3, sub = warp >> 2;              // TMEM lane quadrant, column share
    const int m = 32 * q + lane;                          // this thread's TMEM lane (accumulator row)
    const int y0 = blockIdx.x * R;
    const uint32_t blk_bytes = (uint32_t)blk;
    const __half2* C16 = reinterpret_cast<const __half2*>(a.C);
    const float out_scale = exp2f(-(float)a.half_scale_exp);

    if (t == 0) {
        tmptx::mbar_init(&mbar[0], 1);
        tmptx::mbar_init(&mbar[1], 1);
        tmptx::mbar_init(&mbar[2], 1);
        tmptx::mbar_init(&mbar[3], 1);
    }
    if (warp == 0) {
        tmptx::tmem_alloc(tmem_slot, PC::TMEM_COLS);
        tmptx::tmem_relinquish();
    }
    // DFT matrices into shared memory; the stage-2 A operands start at zero
    // (their K rows beyond N1 are never written and multiply zero B rows)
    for (int i = t; i < (PC::B1_BYTES + PC::B2_BYTES) / 16; i += PC::NT)
        reinterpret_cast<uint4*>(sB1)[i] = __ldg(dft + i);
    for (int i = t; i < R * PC::A2_BYTES / 16; i += PC::NT) reinterpret_cast<uint4*>(sA2)[i] = make_uint4(0, 0, 0, 0);
    const int hcopies = hist_copies(a.hist_bins, PC::HIST_COPIES);
    const int hcopy = t & (hcopies - 1);
    for (int b = t; b < a.hist_bins * hcopies; b += PC::NT) shist[b] = 0u;
    tmptx::fence_proxy_async_smem();
    tmptx::tmem_fence_before_sync();
    __syncthreads();
    tmptx::tmem_fence_after_sync();
    const uint32_t tbase = *tmem_slot;
    const uint32_t tlane = (uint32_t)(32 * q) << 16;
    const uint32_t tstate = tbase + tlane + (uint32_t)(PC::TM_STATE + 48 * sub);
    if (t == 0 && a.nb > 0) {
        tmptx::mbar_arrive_expect_tx(&mbar[0], blk_bytes);
        tmptx::bulk_g2s(rows, C16 + (size_t)blockIdx.x * XP * R, blk_bytes, &mbar[0]);
    }   // copy 0 (counted in the pipeline below)

    // ---- this thread's 16 pixels: items u = 8 * (2 sub + p) + i of the lane pair
    // (n2 = m / 2), item = (row r, n1); pixel x = 2 (n2 + 64 n1) + h
    const int n2_own = m >> 1, p_own = m & 1;
    const int item0 = 8 * (2 * sub + p_own);
    float mip[16], fs[16];
    int best[16];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int it = item0 + i, r = it / N1, n1 = it % N1;
        const size_t off = (size_t)(y0 + r) * X + 2 * (n2_own + 64 * n1);
        const float2 mv = *reinterpret_cast<const float2*>(a.mip + off);
        const int2 bv = *reinterpret_cast<const int2*>(a.best + off);
        mip[2 * i] = mv.x; mip[2 * i + 1] = mv.y;
        best[2 * i] = bv.x; best[2 * i + 1] = bv.y;
        fs[2 * i] = 0.f; fs[2 * i + 1] = 0.f;
    }
    {
        float z[16];
#pragma unroll
        for (int i = 0; i < 16; i++) z[i] = 0.f;
        tmptx::tmem_st16(tstate, z);
        tmptx::tmem_st16(tstate + 16, z);
        tmptx::tmem_st16(tstate + 32, z);
        tmptx::tmem_wait_st();
    }

    const uint32_t id1 = tmptx::idesc_f16_f32(128, PC::B1_N, true, false);
    const uint32_t id2 = tmptx::idesc_f16_f32(128, PC::B2_N, true, false);
    const uint32_t a1_addr = tmptx::smem_u32(sA1), a2_addr = tmptx::smem_u32(sA2);
    const uint32_t b1_addr = tmptx::smem_u32(sB1), b2_addr = tmptx::smem_u32(sB2);
    // mbar[2]: stage-1 MMAs (one commit per orientation), mbar[3]: stage-2 MMAs.
    // The orientations are software-pipelined: the stage-1 MMAs of orientation
    // o + 1 run while the threads finish orientation o (epilogue 2), and the
    // stage-2 MMAs of o while they prepare o + 1, so the tensor core works
    // behind the CUDA-core stages.
    bool timed_out = false;
    int issued1 = 0, issued2 = 0, waited1 = 0, waited2 = 0;   // commits (uniform across the block)
    int copies = a.nb > 0 ? 1 : 0, copies_waited = 0;         // row-block copies issued / waited for
    auto fail = [&]() {
        timed_out = true;
        atomicExch(a.err, 1);
    };
    auto issue_copy = [&](int oo) {   // row block of orientation oo into buffer oo & 1
        if (t == 0) {
            tmptx::mbar_arrive_expect_tx(&mbar[oo & 1], blk_bytes);
            tmptx::bulk_g2s(rows + (oo & 1) * blk, C16 + ((size_t)oo * (Y / R) + blockIdx.x) * XP * R, blk_bytes,
                            &mbar[oo & 1]);
        }
        copies++;
    };
    // a wait that runs out leaves its counter behind, so the drain below waits for it again
    auto wait_copy = [&](int oo) {
        if (tmptx::mbar_wait_bounded(&mbar[oo & 1], (oo >> 1) & 1, kWaitLimit)) copies_waited++;
        else fail();
    };
    // pre-processing of orientation oo: v[r][k] -> A1[(r, k1, re/im)][k2], k = k1 + N1 k2
    auto pre = [&](int oo) {
        const __half2* zb = reinterpret_cast<const __half2*>(rows + (oo & 1) * blk);
#pragma unroll
        for (int i = 0; i < (R * H) / PC::NT; i++) {
            const int idx = t + PC::NT * i;
            const int r = idx / H, k = idx % H;
            float2 hk = __half22float2(zb[k * R + r]);
            float2 hm = __half22float2(zb[(H - k) * R + r]);
            if (k == 0) { hk.y = 0.f; hm.y = 0.f; }
            const float2 e = make_float2(hk.x + hm.x, hk.y - hm.y);
            const float2 d = make_float2(hk.x - hm.x, hk.y + hm.y);
            const float2 od = cmul(d, a.tw.template w<+1>(k, X));
            const int k1 = k % N1, k2 = k / N1;
            *reinterpret_cast<uint32_t*>(sA1 + a_off<X>(2 * (k1 + N1 * r), k2)) = h2_bits(e.x - od.y, e.y + od.x);
        }
        tmptx::fence_proxy_async_smem();
    };
    auto issue1 = [&]() {   // D1 = A1 (128 x 64) x B1 (64 x 128)
        if (t == 0) {
            tmptx::tmem_fence_after_sync();
#pragma unroll
            for (int kk = 0; kk < 4; kk++)
                tmptx::mma_f16_ss(tbase + PC::TM_D1,
                                  tmptx::smem_desc_noswizzle(a1_addr + kk * 2 * PC::LBO_A, PC::LBO_A, PC::SBO_A),
                                  tmptx::smem_desc_noswizzle(b1_addr + kk * 2 * PC::LBO_B1, PC::LBO_B1, PC::SBO_B), id1,
                                  kk > 0);
            tmptx::mma_commit(&mbar[2]);
        }
        issued1++;
    };
    auto issue2 = [&]() {   // per row, D2_r = A2_r (128 x K2) x B2 (K2 x 2 N1)
        if (t == 0) {
            tmptx::tmem_fence_after_sync();
#pragma unroll
            for (int r = 0; r < R; r++)
#pragma unroll
                for (int kk = 0; kk < K2 / 16; kk++)
                    tmptx::mma_f16_ss(tbase + PC::TM_D2 + r * PC::B2_N,
                                      tmptx::smem_desc_noswizzle(a2_addr + r * PC::A2_BYTES + kk * 2 * PC::LBO_A, PC::LBO_A,
                                                                 PC::SBO_A),
                                      tmptx::smem_desc_noswizzle(b2_addr + kk * 2 * PC::LBO_B2, PC::LBO_B2, PC::SBO_B), id2,
                                      kk > 0);
            tmptx::mma_commit(&mbar[3]);
        }
        issued2++;
    };
    auto wait1 = [&]() {
        if (tmptx::mbar_wait_bounded(&mbar[2], waited1 & 1, kWaitLimit)) waited1++;
        else fail();
        tmptx::tmem_fence_after_sync();
    };
    auto wait2 = [&]() {
        if (tmptx::mbar_wait_bounded(&mbar[3], waited2 & 1, kWaitLimit)) waited2++;
        else fail();
        tmptx::tmem_fence_after_sync();
    };
    // epilogue 1: lane m = (r, k1, p); columns n2 in [16 sub, 16 sub + 16) of the cos and sin halves
    auto epi1 = [&]() {
        const int p = m & 1, k1 = (m >> 1) % N1, r = (m >> 1) / N1;
        float c[16], sn[16];
        tmptx::tmem_ld16(tbase + tlane + PC::TM_D1 + 16 * sub, c);
        tmptx::tmem_ld16(tbase + tlane + PC::TM_D1 + 64 + 16 * sub, sn);
        tmptx::tmem_wait_ld16(c);
        tmptx::tmem_wait_ld16(sn);
        // the pair (p = 0, 1) splits the 16 n2: p = 0 takes the first 8, p = 1 the last 8;
        // each sends the partner the products it needs
        float rc[8], rs[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            rc[i] = __shfl_xor_sync(0xffffffffu, p ? c[i] : c[8 + i], 1);
            rs[i] = __shfl_xor_sync(0xffffffffu, p ? sn[i] : sn[8 + i], 1);
        }
        const int n2_0 = 16 * sub + 8 * p;
        // twiddles exp(+2 pi i k1 n2 / H) for n2 = n2_0 .. n2_0 + 7 by recurrence
        const float2 wstep = a.tw.template w<+1>(k1, H);
        float2 w = a.tw.template w<+1>(k1 * n2_0, H);
        uint32_t packed[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            // Y = (P_re,c - P_im,s) + i (P_re,s + P_im,c)
            const float yr = p ? rc[i] - sn[8 + i] : c[i] - rs[i];
            const float yi = p ? rs[i] + c[8 + i] : sn[i] + rc[i];
            const float2 yv = cmul(make_float2(yr, yi), w);
            w = cmul(w, wstep);
            packed[i] = h2_bits(yv.x, yv.y);
        }
        // A2_r[(n2, re/im)][k1]: two 16-byte rows (4 n2 each) of two M groups
        unsigned char* dst = sA2 + r * PC::A2_BYTES;
        *reinterpret_cast<uint4*>(dst + a_off<X>(2 * n2_0, k1)) = make_uint4(packed[0], packed[1], packed[2], packed[3]);
        *reinterpret_cast<uint4*>(dst + a_off<X>(2 * n2_0 + 8, k1)) = make_uint4(packed[4], packed[5], packed[6], packed[7]);
        tmptx::fence_proxy_async_smem();
        tmptx::tmem_fence_before_sync();
    };
    // epilogue 2: lane m = (n2, p); the 16 items [16 sub, 16 sub + 16) of the lane pair
    auto epi2 = [&](int oo) {
        const int p = p_own;
        float c[16], sn[16];
        const int it0 = 16 * sub;
        if constexpr (N1 >= 16) {
            const int r = it0 / N1, n1_0 = it0 % N1;
            const uint32_t col = tbase + tlane + PC::TM_D2 + r * PC::B2_N + n1_0;
            tmptx::tmem_ld16(col, c);
            tmptx::tmem_ld16(col + N1, sn);
        } else {
            // N1 = 8: the 16 items are two whole rows, [cos 8 | sin 8] each
            const uint32_t col = tbase + tlane + PC::TM_D2 + (it0 / N1) * PC::B2_N;
            float w[32];
            tmptx::tmem_ld16(col, w);
            tmptx::tmem_ld16(col + 16, w + 16);
            tmptx::tmem_wait_ld32(w);
#pragma unroll
            for (int i = 0; i < 8; i++) {
                c[i] = w[i]; sn[i] = w[8 + i];
                c[8 + i] = w[16 + i]; sn[8 + i] = w[24 + i];
            }
        }
        tmptx::tmem_wait_ld16(c);
        tmptx::tmem_wait_ld16(sn);
        float rc[8], rs[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            rc[i] = __shfl_xor_sync(0xffffffffu, p ? c[i] : c[8 + i], 1);
            rs[i] = __shfl_xor_sync(0xffffffffu, p ? sn[i] : sn[8 + i], 1);
        }
        const int g = (int)(a.gidx0 + oo);
        float val[16];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            val[2 * i] = (p ? rc[i] - sn[8 + i] : c[i] - rs[i]) * out_scale;
            val[2 * i + 1] = (p ? rs[i] + c[8 + i] : sn[i] + rc[i]) * out_scale;
        }
        // every read of D2 is done before the next stage-2 MMA (after the next barrier)
        tmptx::tmem_fence_before_sync();
        float st[32];
        // sweep 0: MIP / argmax, histogram and the sum (compensation in TMEM columns 0-15)
        tmptx::tmem_ld16(tstate, st);
        tmptx::tmem_wait_ld16(st);
#pragma unroll
        for (int pi = 0; pi < 16; pi++) {
            const float v = val[pi];
            if (v > mip[pi]) { mip[pi] = v; best[pi] = g; }
            const float ys = v - st[pi];
            const float ts = fs[pi] + ys;
            st[pi] = (ts - fs[pi]) - ys;
            fs[pi] = ts;
            const int bin = __float2int_rz((v - a.hist_min) * a.hist_inv_step);
            if (bin >= 0 && bin < a.hist_bins) atomicAdd(&shist[bin * hcopies + hcopy], 1u);
        }
        tmptx::tmem_st16(tstate, st);
        // sweep 1: the sum of squares (columns 32-47) and its compensation (16-31)
        tmptx::tmem_ld16(tstate + 16, st);
        tmptx::tmem_ld16(tstate + 32, st + 16);
        tmptx::tmem_wait_ld32(st);
#pragma unroll
        for (int pi = 0; pi < 16; pi++) {
            const float v = val[pi];
            const float yq = fmaf(v, v, -st[pi]);
            const float tq = st[16 + pi] + yq;
            st[pi] = (tq - st[16 + pi]) - yq;
            st[16 + pi] = tq;
        }
        tmptx::tmem_st16(tstate + 16, st);
        tmptx::tmem_st16(tstate + 32, st + 16);
        tmptx::tmem_wait_st();
    };

    // ---- prologue: orientation 0 prepared and its stage 1 issued; the row block of 1 in flight
    int o = 0;
    bool stop = __syncthreads_or(timed_out);
    if (!stop && a.nb > 1) issue_copy(1);
    if (!stop) {
        wait_copy(0);
        pre(0);
    }
    if (!(stop = __syncthreads_or(timed_out))) issue1();
    for (; !stop && o < a.nb; o++) {
        wait1();
        epi1();                                       // D1(o) -> A2 (stage 2 of o - 1 is complete)
        if ((stop = __syncthreads_or(timed_out))) break;
        issue2();                                     // stage 2 of o
        if (o + 1 < a.nb) {
            wait_copy(o + 1);
            if (o + 2 < a.nb) issue_copy(o + 2);      // into the buffer pre(o) has finished with
            pre(o + 1);                               // A1 is free: stage 1 of o is complete
        }
        if ((stop = __syncthreads_or(timed_out))) break;
        if (o + 1 < a.nb) issue1();                   // stage 1 of o + 1 runs during epilogue 2 of o
        wait2();
        epi2(o);
    }
    // ---- end of the batch: the FP64 flush, or the drain after a wait ran out
    float st[48];
    tmptx::tmem_ld16(tstate, st);
    tmptx::tmem_ld16(tstate + 16, st + 16);
    tmptx::tmem_wait_ld32(st);
    tmptx::tmem_ld16(tstate + 32, st + 32);
    tmptx::tmem_wait_ld16(st + 32);
    tmptx::tmem_fence_before_sync();
    const bool failed = __syncthreads_or(timed_out);
    if (failed) {
        // no MMA or bulk copy may still be writing TMEM or shared memory when the block exits:
        // wait (bounded) for every commit and copy issued and not yet waited for
        for (int k = waited1; k < issued1; k++) tmptx::mbar_wait_bounded(&mbar[2], k & 1, kWaitLimit);
        for (int k = waited2; k < issued2; k++) tmptx::mbar_wait_bounded(&mbar[3], k & 1, kWaitLimit);
        for (int k = copies_waited; k < copies; k++) tmptx::mbar_wait_bounded(&mbar[k & 1], (k >> 1) & 1, kWaitLimit);
    }
    tmptx::tmem_fence_before_sync();
    __syncthreads();
    tmptx::tmem_fence_after_sync();
    if (warp == 0) tmptx::tmem_dealloc(tbase, PC::TMEM_COLS);
    if (failed) return;   // results of this block are discarded (the host reports the timeout)
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int it = item0 + i, r = it / N1, n1 = it % N1;
        const size_t off = (size_t)(y0 + r) * X + 2 * (n2_own + 64 * n1);
        *reinterpret_cast<float2*>(a.mip + off) = make_float2(mip[2 * i], mip[2 * i + 1]);
        *reinterpret_cast<int2*>(a.best + off) = make_int2(best[2 * i], best[2 * i + 1]);
        double2 sv = *reinterpret_cast<const double2*>(a.sum + off);
        double2 qv = *reinterpret_cast<const double2*>(a.sumsq + off);
        sv.x += (double)fs[2 * i] - (double)st[2 * i];
        sv.y += (double)fs[2 * i + 1] - (double)st[2 * i + 1];
        qv.x += (double)st[32 + 2 * i] - (double)st[16 + 2 * i];
        qv.y += (double)st[32 + 2 * i + 1] - (double)st[16 + 2 * i + 1];
        *reinterpret_cast<double2*>(a.sum + off) = sv;
        *reinterpret_cast<double2*>(a.sumsq + off) = qv;
    }
    __syncthreads();
    for (int b = t; b < a.hist_bins; b += PC::NT) {
        unsigned int cnt = 0;
        for (int k = 0; k < hcopies; k++) cnt += shist[b * hcopies + k];
        if (cnt) atomicAdd(a.hist + b, (unsigned long long)cnt);
    }
}

// ======================================================================================
// k_pass_b_tc: the column pass on the tensor cores (FP16 form, height Y = 4096).
//
// Work item = 4 adjacent columns kx0..kx0+3 of one orientation (items ordered
// orientation-fastest, so a block keeps the prepared micrograph spectrum I' of
// its column group in shared memory, FP16, across orientations).  Per column
// (a "vector"), with n = n1 + 64 n2 (n < T, the non-zero rows of A),
// ky = a + 64 b and y = n2' + 64 n1':
//
//   stage H (MMA)  h[a][n1] = sum_n2 A[n1 + 64 n2] exp(-2 pi i n2 a / 64):
//                  one 128 x 256 x 16 MMA for the 4 columns, A = the sparse
//                  DFT E[(a, re/im)][(n2, re/im)], B = the data, N = (column, n1)
//   epilogue H     lane pairs (a, re), (a, im) combine; g = h exp(-2 pi i n1 a / Y)
//   stage F (MMA)  F[a + 64 b] = sum_n1 g[a][n1] exp(-2 pi i n1 b / 64), two
//                  128 x 128 x 128 MMAs (M = (column of the pair, a))
//   epilogue F     Z = I' conj(F) (the conjugate multiply of pass B), written
//                  conjugated as the A operand of stage 1
//   stage 1 (MMA)  conj(sum_k2 conj(Z[k1 + 64 k2]) exp(-2 pi i k2 n2 / 64))
//   epilogue 1     twiddle exp(+2 pi i k1 n2 / Y), conjugated, MN-major A of stage 2
//   stage 2 (MMA)  z[n2 + 64 n1] = conj(sum_k1 ... exp(-2 pi i k1 n1 / 64))
//   epilogue 2     FP16 into a shared staging tile, then the item's 4 columns go
//                  to C16[o][y / RB][kx][y % RB] in whole 32-byte sectors
//
// Complex values are 2 x 2 real blocks along K and N, so every TMEM lane holds
// whole complex outputs (stage H excepted: its lanes hold real or imaginary
// parts and pair up by shuffles).  One FP16 DFT matrix (the forward 64-point
// DFT) serves stages F, 1 and 2; the inverse stages apply it to conjugates.
// Scales (powers of two): the data enter stage H times 2^-6, I' is held
// times 2^iexp (~ N^1.5), the stage-1 operand is Z N, and the stored spectra
// are C 2^half_scale_exp, as k_pass_c_tc expects.
template <int T, int RB>
struct PassBTc {
    static constexpr int Y = 4096;
    static constexpr int NB = (T + 63) / 64;            // non-zero residues n2
    static constexpr int NT = 512;
    static constexpr int E_SBO = 128, E_LBO = 16 * 128;          // stage-H A: K-major, M 128, K 16
    static constexpr int BH_SBO = 128, BH_LBO = 32 * 128;        // stage-H B: MN-major, N 256, K 16
    static constexpr int BF_SBO = 128, BF_LBO = 16 * 128;        // DFT B: K-major, N 128, K 128
    static constexpr int AK_SBO = 128, AK_LBO = 16 * 128;        // K-major A (stages F, 1)
    static constexpr int AM_SBO = 128, AM_LBO = 16 * 128 + 16;   // MN-major A (stage 2), K groups skewed
    static constexpr int E_BYTES = 2 * E_LBO;
    static constexpr int BF_BYTES = 16 * BF_LBO;
    static constexpr int BH_BYTES = 2 * BH_LBO;
    static constexpr int OP_TILE = 16 * AM_LBO;                  // >= 16 * AK_LBO
    static constexpr int OFF_E = 128;
    static constexpr int OFF_BF = OFF_E + E_BYTES;
    static constexpr int OFF_BH = OFF_BF + BF_BYTES;
    static constexpr int OFF_OP = OFF_BH + BH_BYTES;
    static constexpr int OFF_I = OFF_OP + 2 * OP_TILE;
    static constexpr int SMEM = OFF_I + 4 * Y * 4;
    static constexpr uint32_t TMEM_COLS = 256;
    static_assert(2 * NB <= 16, "stage H takes at most 8 residues (T <= 512)");
    static_assert(2 * OP_TILE >= 4 * Y * 4, "the operand buffer doubles as the output staging tile");
    static_assert(SMEM <= 232448, "pass B tensor block exceeds shared memory");
    static constexpr size_t dft_bytes = (size_t)E_BYTES + BF_BYTES;
};

__host__ __device__ constexpr int kmaj_off(int m, int k, int sbo, int lbo) {
    return (m % 8) * 16 + (k % 8) * 2 + (m / 8) * sbo + (k / 8) * lbo;
}
__host__ __device__ constexpr int mnmaj_off(int m, int k, int sbo, int lbo) {
    return (m % 8) * 2 + (k % 8) * 16 + (m / 8) * sbo + (k / 8) * lbo;
}

// E (stage-H A operand) then the forward 64-point DFT (B operand of stages F,
// 1 and 2), FP16, in the kernel's shared-memory byte layout.
template <int T, int RB>
void fill_tc_cols(uint16_t* out) {
    using PB = PassBTc<T, RB>;
    auto put = [](uint16_t* base, int off, double v) {
        const __half h = __double2half(v);
        base[off / 2] = *reinterpret_cast<const uint16_t*>(&h);
    };
    for (size_t i = 0; i < PB::dft_bytes / 2; i++) out[i] = 0;
    uint16_t* e = out;
    uint16_t* bf = out + PB::E_BYTES / 2;
    for (int a = 0; a < 64; a++)
        for (int n2 = 0; n2 < PB::NB; n2++) {
            const double th = 2.0 * M_PI * (double)((n2 * a) % 64) / 64.0, c = cos(th), s = sin(th);
            // h = sum A exp(-i th): re = Ar c + Ai s, im = Ai c - Ar s
            put(e, kmaj_off(2 * a, 2 * n2, PB::E_SBO, PB::E_LBO), c);
            put(e, kmaj_off(2 * a, 2 * n2 + 1, PB::E_SBO, PB::E_LBO), s);
            put(e, kmaj_off(2 * a + 1, 2 * n2, PB::E_SBO, PB::E_LBO), -s);
            put(e, kmaj_off(2 * a + 1, 2 * n2 + 1, PB::E_SBO, PB::E_LBO), c);
        }
    for (int n1 = 0; n1 < 64; n1++)
        for (int b = 0; b < 64; b++) {
            const double th = 2.0 * M_PI * (double)((n1 * b) % 64) / 64.0, c = cos(th), s = sin(th);
            put(bf, kmaj_off(2 * b, 2 * n1, PB::BF_SBO, PB::BF_LBO), c);
            put(bf, kmaj_off(2 * b, 2 * n1 + 1, PB::BF_SBO, PB::BF_LBO), s);
            put(bf, kmaj_off(2 * b + 1, 2 * n1, PB::BF_SBO, PB::BF_LBO), -s);
            put(bf, kmaj_off(2 * b + 1, 2 * n1 + 1, PB::BF_SBO, PB::BF_LBO), c);
        }
}

__device__ __forceinline__ float2 h2f(uint32_t bits) {
    __half2 h = *reinterpret_cast<const __half2*>(&bits);
    return __half22float2(h);
}

template <int T, int RB>
__global__ void __launch_bounds__(512, 1)
k_pass_b_tc(BatchArgs a, int ngroups, const uint4* __restrict__ tabs) {
    using PB = PassBTc<T, RB>;
    constexpr int Y = PB::Y;
    constexpr uint32_t kWaitLimit = 1u << 24;
    const int XP = a.XP;
    extern __shared__ __align__(128) unsigned char smem_b16[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_b16);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem_b16 + 64);
    unsigned char* sE = smem_b16 + PB::OFF_E;
    unsigned char* sBF = smem_b16 + PB::OFF_BF;
    unsigned char* sBH = smem_b16 + PB::OFF_BH;
    unsigned char* sOP = smem_b16 + PB::OFF_OP;
    uint32_t* sI = reinterpret_cast<uint32_t*>(smem_b16 + PB::OFF_I);   // I' as FP16 complex, [column][ky]
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int q = warp & 3, sub = warp >> 2;
    const int m = 32 * q + lane;            // TMEM lane of this thread
    // the items of this block, as in k_pass_b (adjacent column groups per round)
    const ColSchedule sch(ngroups, a.nb, blockIdx.x, gridDim.x);
    const int it1 = sch.n;
    if (it1 == 0) return;
    if (t == 0) {
        tmptx::mbar_init(&mbar[0], 1);
        tmptx::mbar_init(&mbar[1], 1);
        tmptx::mbar_init(&mbar[2], 1);
    }
    if (warp == 0) {
        tmptx::tmem_alloc(tmem_slot, PB::TMEM_COLS);
        tmptx::tmem_relinquish();
    }
    for (int i = t; i < (PB::E_BYTES + PB::BF_BYTES) / 16; i += PB::NT) reinterpret_cast<uint4*>(sE)[i] = __ldg(tabs + i);
    // stage-H data rows beyond 2 NB multiply zero columns of E and must be finite
    for (int i = t; i < PB::BH_BYTES / 16; i += PB::NT) reinterpret_cast<uint4*>(sBH)[i] = make_uint4(0, 0, 0, 0);
    tmptx::fence_proxy_async_smem();
    tmptx::tmem_fence_before_sync();
    __syncthreads();
    tmptx::tmem_fence_after_sync();
    const uint32_t tbase = *tmem_slot;
    const uint32_t tlane = (uint32_t)(32 * q) << 16;
    const float sA = 1.0f / 64.0f;
    const float sI_scale = exp2f((float)a.tc_iexp);
    const float sZ = exp2f((float)(a.tc_zexp - a.tc_iexp + 6));     // Z N = I'_held conj(F_held) 2^(6 - iexp + zexp)
    const float sOut = exp2f((float)(a.half_scale_exp - a.tc_zexp));
    const uint32_t idH = tmptx::idesc_f16_f32(128, 256, false, true);
    const uint32_t idK = tmptx::idesc_f16_f32(128, 128, false, false);
    const uint32_t idM = tmptx::idesc_f16_f32(128, 128, true, false);
    const uint32_t e_addr = tmptx::smem_u32(sE), bf_addr = tmptx::smem_u32(sBF), bh_addr = tmptx::smem_u32(sBH);
    const uint32_t op_addr = tmptx::smem_u32(sOP);
    // mbar[0]: stage H (one commit per item, the whole block waits); mbar[1 + h]:
    // stages F, 1 and 2 of tile h.  After stage H the two tiles (columns 2h, 2h + 1)
    // are independent chains run by the two halves of the block (warps 8h .. 8h + 7,
    // named barrier 1 + h), so one half's MMAs run during the other half's epilogues.
    const int h = sub >> 1;                      // this thread's tile
    const int lead = 256 * h;                    // the thread that issues the tile's MMAs
    bool timed_out = false;
    int issuedH = 0, waitedH = 0, issuedT = 0, waitedT = 0;   // commits of stage H and of this thread's tile
    int cur_group = -1;
    auto fail = [&]() {
        timed_out = true;
        atomicExch(a.err, 1);
    };
    auto half_sync = [h]() { asm volatile("bar.sync %0, 256;" ::"r"(1 + h) : "memory"); };
    unsigned char* tile = sOP + h * PB::OP_TILE;
    const uint32_t tile_addr = op_addr + h * PB::OP_TILE;
    const uint32_t tcol = tbase + tlane + 128 * h;
    // D_tile = A_tile (128 x 128) x DFT (128 x 128), issued by the half's lead thread
    auto issue_tile = [&](int a_lbo, int a_sbo, uint32_t idesc) {
        if (t == lead) {
            tmptx::tmem_fence_after_sync();
#pragma unroll
            for (int kk = 0; kk < 8; kk++)
                tmptx::mma_f16_ss(tbase + 128 * h, tmptx::smem_desc_noswizzle(tile_addr + kk * 2 * a_lbo, a_lbo, a_sbo),
                                  tmptx::smem_desc_noswizzle(bf_addr + kk * 2 * PB::BF_LBO, PB::BF_LBO, PB::BF_SBO), idesc,
                                  kk > 0);
            tmptx::mma_commit(&mbar[1 + h]);
        }
        issuedT++;
    };
    auto wait_tile = [&]() {
        if (tmptx::mbar_wait_bounded(&mbar[1 + h], waitedT & 1, kWaitLimit)) waitedT++;
        else fail();
        tmptx::tmem_fence_after_sync();
    };
    // the item's stage-H data (4 T values, at most NPF per thread) are loaded one item
    // ahead, so that their latency hides behind the previous item's epilogues
    constexpr int NPF = (4 * T + PB::NT - 1) / PB::NT;
    float2 pf[NPF];
    auto prefetch = [&](int itn) {
        int gn, on;
        sch.locate(itn, gn, on);
        const float2* Ao = a.A + (size_t)on * T * XP + gn * 4;
#pragma unroll
        for (int q = 0; q < NPF; q++) {
            const int i = t + PB::NT * q;
            pf[q] = i < 4 * T ? __ldg(Ao + (size_t)(i >> 2) * XP + (i & 3)) : make_float2(0.f, 0.f);
        }
    };
    prefetch(0);
    for (int it = 0; it < it1; it++) {
        int group, o;
        sch.locate(it, group, o);
        const int kx0 = group * 4;
        // every thread is done with the previous item's staging tile and I'
        if (__syncthreads_or(timed_out)) break;
        if (group != cur_group) {
            // I' of the 4 columns, FP16 times 2^iexp, [column][ky]
#pragma unroll 4
            for (int i = t; i < 4 * Y; i += PB::NT) {
                const int c = i & 3, ky = i >> 2;
                const float2 v = __ldg(a.Ip + (size_t)ky * XP + kx0 + c);
                sI[c * Y + ky] = h2_bits(v.x * sI_scale, v.y * sI_scale);
            }
            cur_group = group;
        }
        // stage-H data: A[o][n][kx0 + c] times 2^-6 -> BH[(n2, re/im)][(c, n1)]
#pragma unroll
        for (int q = 0; q < NPF; q++) {
            const int i = t + PB::NT * q;
            if (i < 4 * T) {
                const int c = i & 3, n = i >> 2;
                const int nn = 64 * c + (n & 63), n2 = n >> 6;
                *reinterpret_cast<__half*>(sBH + mnmaj_off(nn, 2 * n2, PB::BH_SBO, PB::BH_LBO)) = __float2half_rn(pf[q].x * sA);
                *reinterpret_cast<__half*>(sBH + mnmaj_off(nn, 2 * n2 + 1, PB::BH_SBO, PB::BH_LBO)) =
                    __float2half_rn(pf[q].y * sA);
            }
        }
        if (it + 1 < it1) prefetch(it + 1);
        tmptx::fence_proxy_async_smem();
        tmptx::tmem_fence_before_sync();
        if (__syncthreads_or(timed_out)) break;
        if (t == 0) {
            tmptx::tmem_fence_after_sync();
            tmptx::mma_f16_ss(tbase, tmptx::smem_desc_noswizzle(e_addr, PB::E_LBO, PB::E_SBO),
                              tmptx::smem_desc_noswizzle(bh_addr, PB::BH_LBO, PB::BH_SBO), idH, false);
            tmptx::mma_commit(&mbar[0]);
        }
        issuedH++;
        if (tmptx::mbar_wait_bounded(&mbar[0], waitedH & 1, kWaitLimit)) waitedH++;
        else fail();
        tmptx::tmem_fence_after_sync();
        // ---- epilogue H: lane m = (a, p); columns (v = sub, n1); p = 0 keeps n1 < 32, p = 1 the rest
        {
            const int p = m & 1, av = m >> 1, v = sub, vl = v & 1;
#pragma unroll 1
            for (int j = 0; j < 2; j++) {
                float lo[16], hi[16];
                tmptx::tmem_ld16(tbase + tlane + 64 * v + 16 * j, lo);        // n1 = 16 j + i
                tmptx::tmem_ld16(tbase + tlane + 64 * v + 32 + 16 * j, hi);   // n1 = 32 + 16 j + i
                tmptx::tmem_wait_ld16(lo);
                tmptx::tmem_wait_ld16(hi);
                const int n1_0 = 32 * p + 16 * j;
                // exp(-2 pi i n1 a / Y) for n1 = n1_0 .. n1_0 + 15 by recurrence
                const float2 wstep = a.twy.template w<-1>(av, Y);
                float2 w = a.twy.template w<-1>(n1_0 * av, Y);
                uint32_t packed[16];
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const float r = __shfl_xor_sync(0xffffffffu, p ? lo[i] : hi[i], 1);
                    const float2 hv = p ? make_float2(r, hi[i]) : make_float2(lo[i], r);
                    const float2 g = cmul(hv, w);
                    w = cmul(w, wstep);
                    packed[i] = h2_bits(g.x, g.y);
                }
                const int mF = 64 * vl + av;
#pragma unroll
                for (int r = 0; r < 4; r++)
                    *reinterpret_cast<uint4*>(tile + kmaj_off(mF, 2 * n1_0 + 8 * r, PB::AK_SBO, PB::AK_LBO)) =
                        make_uint4(packed[4 * r], packed[4 * r + 1], packed[4 * r + 2], packed[4 * r + 3]);
            }
        }
        tmptx::fence_proxy_async_smem();
        tmptx::tmem_fence_before_sync();
        half_sync();
        issue_tile(PB::AK_LBO, PB::AK_SBO, idK);
        wait_tile();
        // ---- epilogue F: lane m = (vl, a); b in [32 (sub & 1), +32)
        const int vl = m >> 6, av = m & 63;
        const int v = 2 * h + vl;
#pragma unroll 1
        for (int j = 0; j < 2; j++) {
            const int b0 = 32 * (sub & 1) + 16 * j;
            float d[32];
            tmptx::tmem_ld16(tcol + 2 * b0, d);
            tmptx::tmem_ld16(tcol + 2 * b0 + 16, d + 16);
            tmptx::tmem_wait_ld32(d);
            uint32_t packed[16];
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const float2 iv = h2f(sI[v * Y + av + 64 * (b0 + i)]);
                const float2 z = cmul_conj(iv, make_float2(d[2 * i], d[2 * i + 1]));
                packed[i] = h2_bits(z.x * sZ, -z.y * sZ);      // conj(Z) for the inverse stages
            }
#pragma unroll
            for (int r = 0; r < 4; r++)
                *reinterpret_cast<uint4*>(tile + kmaj_off(m, 2 * b0 + 8 * r, PB::AK_SBO, PB::AK_LBO)) =
                    make_uint4(packed[4 * r], packed[4 * r + 1], packed[4 * r + 2], packed[4 * r + 3]);
        }
        tmptx::fence_proxy_async_smem();
        tmptx::tmem_fence_before_sync();
        half_sync();
        issue_tile(PB::AK_LBO, PB::AK_SBO, idK);
        wait_tile();
        // ---- epilogue 1: lane m = (vl, k1); Y = conj(D1), Y' = Y exp(+2 pi i k1 n2 / Y), A2 = conj(Y') MN-major
#pragma unroll 1
        for (int j = 0; j < 2; j++) {
            const int n2_0 = 32 * (sub & 1) + 16 * j;
            float d[32];
            tmptx::tmem_ld16(tcol + 2 * n2_0, d);
            tmptx::tmem_ld16(tcol + 2 * n2_0 + 16, d + 16);
            tmptx::tmem_wait_ld32(d);
            const float2 wstep = a.twy.template w<+1>(av, Y);
            float2 w = a.twy.template w<+1>(av * n2_0, Y);
            float re[16], im[16];
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const float2 yv = cmul(make_float2(d[2 * i], -d[2 * i + 1]), w);
                w = cmul(w, wstep);
                re[i] = yv.x;
                im[i] = -yv.y;
            }
            // K index 2 k1 (re) and 2 k1 + 1 (im); M = 64 vl + n2, 8 per 16-byte row
#pragma unroll
            for (int g = 0; g < 2; g++) {
                const int m2 = 64 * vl + n2_0 + 8 * g;
                *reinterpret_cast<uint4*>(tile + mnmaj_off(m2, 2 * av, PB::AM_SBO, PB::AM_LBO)) =
                    make_uint4(h2_bits(re[8 * g], re[8 * g + 1]), h2_bits(re[8 * g + 2], re[8 * g + 3]),
                               h2_bits(re[8 * g + 4], re[8 * g + 5]), h2_bits(re[8 * g + 6], re[8 * g + 7]));
                *reinterpret_cast<uint4*>(tile + mnmaj_off(m2, 2 * av + 1, PB::AM_SBO, PB::AM_LBO)) =
                    make_uint4(h2_bits(im[8 * g], im[8 * g + 1]), h2_bits(im[8 * g + 2], im[8 * g + 3]),
                               h2_bits(im[8 * g + 4], im[8 * g + 5]), h2_bits(im[8 * g + 6], im[8 * g + 7]));
            }
        }
        tmptx::fence_proxy_async_smem();
        tmptx::tmem_fence_before_sync();
        half_sync();
        issue_tile(PB::AM_LBO, PB::AM_SBO, idM);
        wait_tile();
        // ---- epilogue 2 (stage 2 has read A2: the tile becomes its columns' staging area):
        // lane m = (vl, n2); z[n2 + 64 n1] = conj(D2) -> staging [column vl][y], FP16
        uint32_t* stage = reinterpret_cast<uint32_t*>(tile) + vl * Y;
#pragma unroll 1
        for (int j = 0; j < 2; j++) {
            const int n1_0 = 32 * (sub & 1) + 16 * j;
            float d[32];
            tmptx::tmem_ld16(tcol + 2 * n1_0, d);
            tmptx::tmem_ld16(tcol + 2 * n1_0 + 16, d + 16);
            tmptx::tmem_wait_ld32(d);
#pragma unroll
            for (int i = 0; i < 16; i++) stage[av + 64 * (n1_0 + i)] = h2_bits(d[2 * i] * sOut, -d[2 * i + 1] * sOut);
        }
        tmptx::tmem_fence_before_sync();
        if (__syncthreads_or(timed_out)) break;
        // ---- the item's columns to C16[o][y / RB][kx][y % RB]: 16-byte chunks of 4 (column, row) values
        {
            __half2* C16 = reinterpret_cast<__half2*>(a.C) + (size_t)o * Y * XP;
            const uint32_t* st0 = reinterpret_cast<const uint32_t*>(sOP);
            const uint32_t* st1 = reinterpret_cast<const uint32_t*>(sOP + PB::OP_TILE);
            for (int ch = t; ch < Y; ch += PB::NT) {
                // chunk ch: row block rb, elements e = 4 (ch % RB) .. + 3 of its 4 RB (column, row) values
                const int rb = ch / RB, e0 = 4 * (ch % RB);
                uint32_t w4[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int c = (e0 + e) / RB, r = (e0 + e) % RB;
                    w4[e] = ((c >> 1) ? st1 : st0)[(c & 1) * Y + rb * RB + r];
                }
                // streaming store: the row pass reads the intermediate only after the whole launch
                __stcs(reinterpret_cast<uint4*>(C16 + ((size_t)rb * XP + kx0) * RB + e0), make_uint4(w4[0], w4[1], w4[2], w4[3]));
            }
        }
    }
    const bool failed = __syncthreads_or(timed_out);
    if (failed) {
        // no MMA may still be writing TMEM when the block exits
        for (int k = waitedH; k < issuedH; k++) tmptx::mbar_wait_bounded(&mbar[0], k & 1, kWaitLimit);
        for (int k = waitedT; k < issuedT; k++) tmptx::mbar_wait_bounded(&mbar[1 + h], k & 1, kWaitLimit);
    }
    tmptx::tmem_fence_before_sync();
    __syncthreads();
    tmptx::tmem_fence_after_sync();
    if (warp == 0) tmptx::tmem_dealloc(tbase, PB::TMEM_COLS);
}

}  // namespace tmk
