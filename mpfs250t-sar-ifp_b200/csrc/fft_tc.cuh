// Split-precision tensor-core FFT of one line of N = 128 * N2 complex points (N2 = 16, 32, 64), the
// float path's mixed-precision mode.  Four-step factorisation, both steps as tcgen05 MMAs:
//
//   n = n1 + 128 n2,  k = k2 + N2 k1
//   D1[n1][k2] = sum_n2 x[n1 + 128 n2] F_N2[n2][k2]                      (stage 1: A = data in TMEM,
//                                                                          B = F_N2 in shared memory)
//   T[n1][k2]  = D1[n1][k2] W_N^(n1 k2)                                  (FP32, CUDA cores)
//   X[k2 + N2 k1] = sum_n1 F_128[k1][n1] T[n1][k2]                       (stage 2: A = F_128 in TMEM,
//                                                                          B = T in shared memory)
// Every real product P Q runs as Ph Qh + Ph Ql + Pl Qh with fp16 hi/lo parts (v = hi + lo, 22
// significant bits) and fp32 accumulation; complex products are spelled out in real parts, the
// subtracted ones with the B operand negated by the instruction descriptor.  The line
// is scaled by a power of two s1 so that its largest component lies in [2^14, 2^15) (fp16 range with
// headroom); after stage 1 the scale becomes s1 / N2, which bounds |T| by the same range.
//
// CTA: 128 * NG threads (NG = N2 / 16); warp w serves TMEM lanes 32 (w % 4) .. +31 and the column
// group g = w / 4, so every thread owns 16 consecutive n2 (stage-1 input) or k2 (outputs) of its lane.
//
// TMEM (512 columns, one CTA per SM):
//   [0, 256)                 F_128 as the stage-2 A operand: Frh, Frl, Fih, Fil (64 columns each,
//                            two fp16 of consecutive n1 per 32-bit column)
//   [256, 256 + 2 N2)        stage-1 A operand: Arh, Arl, Aih, Ail (N2/2 columns each); free while
//                            stage 2 runs, so the next line's input can be written meanwhile
//   [256 + 2 N2, 256 + 4 N2) accumulators Re, Im: stage 1's D1, then stage 2's X (the products with
//                            a minus sign negate their B operand through the instruction descriptor)
// Shared memory: F_N2 image (4 arrays: Frh, Frl, Fih, Fil; MN-major N2 x N2) and the stage-2 B operand
// (4 arrays Trh, Trl, Tih, Til; MN-major, K = 128 rows n1, N = N2 columns k2).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "tc_sm100.cuh"

namespace pfa {
namespace tcfft {

template <int L>
struct Geo {
    static constexpr int N = 1 << L;
    static constexpr int N2 = N / 128;
    static_assert(N2 == 16 || N2 == 32 || N2 == 64, "tensor-core FFT lines are 2048, 4096 or 8192 points");
    static constexpr int NG = N2 / 16;
    static constexpr int THREADS = 128 * NG;
    static constexpr uint32_t COL_F = 0, COL_A = 256, COL_D = 256 + 2 * N2, TMEM_COLS = 512;
    static constexpr uint32_t FN2_ARR = (uint32_t)N2 * N2 * 2;
    static constexpr uint32_t FN2_BYTES = 4 * FN2_ARR;
    static constexpr uint32_t B2_ARR = 128u * N2 * 2;
    static constexpr uint32_t B2_BYTES = 4 * B2_ARR;           // = 8 N: also holds one complex line
};

// fp16 hi/lo split of v (|v| < 65504): v ~ hi + lo to 22 significant bits
__device__ __forceinline__ void split(float v, __half &hi, __half &lo) {
    hi = __float2half_rn(v);
    lo = __float2half_rn(v - __half2float(hi));
}
__device__ __forceinline__ uint32_t pack2(__half a, __half b) {
    return (uint32_t)__half_as_ushort(a) | ((uint32_t)__half_as_ushort(b) << 16);
}

// 16-byte-chunk swizzle of a staging buffer written by lanes with rows of 2^rowbits chunks: XOR of the
// chunk's low 3 bits with 3 bits of its row index (a bijection: the XORed bits lie below the source bits)
template <int ROWBITS>
__device__ __forceinline__ int swz_chunk(int ch) {
    constexpr int S = ROWBITS < 3 ? 3 : ROWBITS;
    return ch ^ ((ch >> S) & 7);
}

template <int L>
struct TcFft {
    using G = Geo<L>;
    static constexpr int N = G::N, N2 = G::N2, NG = G::NG;

    __device__ static __forceinline__ uint32_t lane_base(uint32_t tm, int q) { return tm + ((uint32_t)(32 * q) << 16); }

    // F_N2 image (global, prepared on the host in the shared-memory layout) -> shared memory
    __device__ static void load_fn2(const uint4 *src, unsigned char *dst, int tid) {
        uint4 *d = reinterpret_cast<uint4 *>(dst);
        for (int i = tid; i < (int)(G::FN2_BYTES / 16); i += G::THREADS) d[i] = __ldg(src + i);
    }

    // F_128 image (global [128 lanes][256 columns] of packed fp16 pairs) -> TMEM columns [0, 256)
    __device__ static void load_f128(const uint4 *src, uint32_t tm, int q, int g, int lane) {
        const int row = 32 * q + lane;
        constexpr int COLS = 256 / NG;
#pragma unroll 1
        for (int c0 = g * COLS; c0 < (g + 1) * COLS; c0 += 16) {
            uint32_t r[16];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const uint4 v = __ldg(src + (row * 256 + c0) / 4 + i);
                r[4 * i] = v.x; r[4 * i + 1] = v.y; r[4 * i + 2] = v.z; r[4 * i + 3] = v.w;
            }
            tc::tmem_st16(lane_base(tm, q) + G::COL_F + c0, r);
        }
        tc::tmem_wait_st();
    }

    // Power-of-two line scale from the per-thread max |component|: s1 puts the line max in [2^14, 2^15).
    // Uses red[0 .. warps) and two barriers.
    __device__ static float line_scale(float mx, float *red, int warp, int lane) {
        const unsigned b = __reduce_max_sync(0xffffffffu, __float_as_uint(mx));
        if (lane == 0) red[warp] = __uint_as_float(b);
        __syncthreads();
        float m = 0.f;
#pragma unroll
        for (int w = 0; w < G::THREADS / 32; ++w) m = fmaxf(m, red[w]);
        __syncthreads();
        if (!(m > 0.f) || !isfinite(m)) return 1.f;
        int e;
        frexpf(m, &e);                        // m in [2^(e-1), 2^e)
        return ldexpf(1.f, min(15 - e, 126));
    }

    // Stage-1 input: x[c] = x[n1 + 128 (16 g + c)] of lane n1 = 32 q + lane, scaled by s1, into TMEM.
    __device__ static void put_input(const float2 (&x)[16], float s1, uint32_t tm, int q, int g) {
        uint32_t rh[8], rl[8], ih[8], il[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            __half a0, a1, b0, b1, c0, c1, d0, d1;
            split(x[2 * c].x * s1, a0, b0);
            split(x[2 * c + 1].x * s1, a1, b1);
            split(x[2 * c].y * s1, c0, d0);
            split(x[2 * c + 1].y * s1, c1, d1);
            rh[c] = pack2(a0, a1);
            rl[c] = pack2(b0, b1);
            ih[c] = pack2(c0, c1);
            il[c] = pack2(d0, d1);
        }
        const uint32_t base = lane_base(tm, q) + G::COL_A + 8 * g;
        tc::tmem_st8(base + 0 * (N2 / 2), rh);
        tc::tmem_st8(base + 1 * (N2 / 2), rl);
        tc::tmem_st8(base + 2 * (N2 / 2), ih);
        tc::tmem_st8(base + 3 * (N2 / 2), il);
        tc::tmem_wait_st();
    }

    // Stage 1 (one thread): D1r = Ar Fr - Ai Fi, D1i = Ar Fi + Ai Fr, each real product split three ways.
    __device__ static void issue_stage1(uint32_t tm, uint32_t fn2) {
        constexpr uint32_t idesc = tc::idesc_f16(128, N2, false, true);
        constexpr uint32_t idesc_neg = tc::idesc_f16(128, N2, false, true, false, true);   // -B
        // {A array (Arh, Arl, Aih, Ail), F_N2 array (Frh, Frl, Fih, Fil), accumulator (re, im), negate B}
        constexpr int8_t terms[12][4] = {{0, 0, 0, 0}, {0, 1, 0, 0}, {1, 0, 0, 0}, {2, 2, 0, 1}, {2, 3, 0, 1},
                                         {3, 2, 0, 1}, {0, 2, 1, 0}, {0, 3, 1, 0}, {1, 2, 1, 0}, {2, 0, 1, 0},
                                         {2, 1, 1, 0}, {3, 0, 1, 0}};
#pragma unroll
        for (int t = 0; t < 12; ++t) {
#pragma unroll
            for (int s = 0; s < N2 / 16; ++s) {
                const uint32_t a = tm + G::COL_A + terms[t][0] * (N2 / 2) + 8 * s;
                const uint64_t b = tc::smem_desc(fn2 + terms[t][1] * G::FN2_ARR + s * 2 * N2 * 16, N2 * 16, 128);
                const uint32_t d = tm + G::COL_D + terms[t][2] * N2;
                tc::mma_ts(d, a, b, terms[t][3] ? idesc_neg : idesc, !((t == 0 || t == 6) && s == 0));
            }
        }
    }

    // This thread's inter-stage twiddles W_N^(n1 k2), k2 = 16 g + c, from the full W_N table (fixed per
    // thread, so a persistent kernel loads them once).
    __device__ static void twiddles(float2 (&w)[16], const float2 *tw, int n1, int g) {
#pragma unroll
        for (int c = 0; c < 16; ++c) w[c] = __ldg(tw + ((n1 * (16 * g + c)) & (N - 1)));
    }

    // Epilogue 1: D1 (scaled by s1) -> T = D1 W_N^(n1 k2) / N2 -> fp16 hi/lo stage-2 B operand in smem.
    __device__ static void epilogue1(uint32_t tm, unsigned char *b2, const float2 (&tw)[16], int q, int g, int lane) {
        const int n1 = 32 * q + lane;
        uint32_t re[16], im[16];
        tc::tmem_ld16(lane_base(tm, q) + G::COL_D + 16 * g, re);
        tc::tmem_ld16(lane_base(tm, q) + G::COL_D + N2 + 16 * g, im);
        tc::tmem_wait_ld();
        constexpr float inv = 1.0f / (float)N2;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                __half x0h[2], x0l[2], y0h[2], y0l[2];
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int cc = 8 * h + 2 * c + e;
                    const float2 w = tw[cc];
                    const float a = __uint_as_float(re[cc]) * inv, b = __uint_as_float(im[cc]) * inv;
                    split(fmaf(a, w.x, -b * w.y), x0h[e], x0l[e]);
                    split(fmaf(a, w.y, b * w.x), y0h[e], y0l[e]);
                }
                rh[c] = pack2(x0h[0], x0h[1]);
                rl[c] = pack2(x0l[0], x0l[1]);
                ih[c] = pack2(y0h[0], y0h[1]);
                il[c] = pack2(y0l[0], y0l[1]);
            }
            const uint32_t off = tc::mnmajor_off(n1, 16 * g + 8 * h, N2);
            *reinterpret_cast<uint4 *>(b2 + 0 * G::B2_ARR + off) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
            *reinterpret_cast<uint4 *>(b2 + 1 * G::B2_ARR + off) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
            *reinterpret_cast<uint4 *>(b2 + 2 * G::B2_ARR + off) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
            *reinterpret_cast<uint4 *>(b2 + 3 * G::B2_ARR + off) = make_uint4(il[0], il[1], il[2], il[3]);
        }
    }

    // Stage 2 (one thread): Re = Fr Tr - Fi Ti, Im = Fr Ti + Fi Tr (each real product split three ways),
    // into the accumulator columns stage 1 used (read by epilogue 1 before this is issued).
    __device__ static void issue_stage2(uint32_t tm, uint32_t b2) {
        constexpr uint32_t idesc = tc::idesc_f16(128, N2, false, true);
        constexpr uint32_t idesc_neg = tc::idesc_f16(128, N2, false, true, false, true);   // -B
        // {F_128 array (Frh, Frl, Fih, Fil), T array (Trh, Trl, Tih, Til), accumulator (re, im), negate B}
        constexpr int8_t terms[12][4] = {{0, 0, 0, 0}, {0, 1, 0, 0}, {1, 0, 0, 0}, {2, 2, 0, 1}, {2, 3, 0, 1},
                                         {3, 2, 0, 1}, {0, 2, 1, 0}, {0, 3, 1, 0}, {1, 2, 1, 0}, {2, 0, 1, 0},
                                         {2, 1, 1, 0}, {3, 0, 1, 0}};
#pragma unroll
        for (int t = 0; t < 12; ++t) {
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                const uint32_t a = tm + G::COL_F + terms[t][0] * 64 + 8 * s;
                const uint64_t b = tc::smem_desc(b2 + terms[t][1] * G::B2_ARR + s * 2 * N2 * 16, N2 * 16, 128);
                const uint32_t d = tm + G::COL_D + terms[t][2] * N2;
                tc::mma_ts(d, a, b, terms[t][3] ? idesc_neg : idesc, !((t == 0 || t == 6) && s == 0));
            }
        }
    }

    // Stage-2 result of lane k1 = 32 q + lane: y[c] = X[16 g + c + N2 k1] * s1 / N2 (unscaled by the caller).
    __device__ static void get_output(float2 (&y)[16], uint32_t tm, int q, int g) {
        uint32_t re[16], im[16];
        tc::tmem_ld16(lane_base(tm, q) + G::COL_D + 16 * g, re);
        tc::tmem_ld16(lane_base(tm, q) + G::COL_D + N2 + 16 * g, im);
        tc::tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < 16; ++c) y[c] = make_float2(__uint_as_float(re[c]), __uint_as_float(im[c]));
    }
};

}  // namespace tcfft
}  // namespace pfa
