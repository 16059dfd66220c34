// Split-precision (mixed) float mode: the FFTs of form_image_pfa.focus (src/form_image_pfa.py:225-240,
// transform2d :144-147) as fp16 hi/lo DFT-matrix products on the tcgen05 tensor cores with fp32
// accumulation (fft_tc.cuh); resampling, window and detection stay FP32 with FP64 coordinates.
//
//   k_mx_pass2<L,SINC>  persistent 4-CTA clusters: per range bin the pass-2 gather (as k_fl_pass2_fft),
//                       the cross FFT on the tensor cores, and corner turn #2 through distributed shared
//                       memory into the transposed buffer y1t [cross bin][npad]
//   k_mx_fft2<L>        persistent CTAs: per cross bin the range FFT on the tensor cores and the
//                       detection store (|z|, |z|^2 or complex with the (-1)^(u+v) centring sign)
//
// Both hold 512 TMEM columns, so they request enough shared memory that no two CTAs share an SM (a
// second CTA would block in tcgen05.alloc; in a cluster that could deadlock with its own peer).  Every
// completion wait is bounded; a timeout sets wait_err and the kernel finishes the line loop without
// issuing further MMAs (cluster barriers stay matched) and releases its TMEM.
#include <cooperative_groups.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "fft_tc.cuh"
#include "interp_f32.cuh"
#include "pfa_internal.h"

namespace pfa {
namespace {

using tcfft::Geo;
using tcfft::TcFft;

constexpr int kMxCT = 4;                      // cluster size of the mixed pass 2 (divides 8: npad holds whole clusters)
constexpr size_t kMxMinSmem = 118 * 1024;     // > half of the SM's shared memory: one CTA per SM

__host__ __device__ constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v >> 1); }

// The CTA agrees on a bounded completion wait (all threads poll; a barrier ANDs the outcomes).
__device__ __forceinline__ bool cta_wait(uint64_t *bar, uint32_t parity, bool ok) {
    const bool mine = ok ? tc::mbar_wait(bar, parity) : false;
    return __syncthreads_and(mine) != 0;
}

// ------------------------------------------------------------------------------------------ range FFT
struct MxFft2Args {
    const float2 *y1t;
    const float2 *tw;
    const uint4 *fn2, *f128;
    void *out;
    int *err;
    int n, npad, rows, centred, detect, inverse;
    float scale;
    int probe;            // test hook: > 0 = polls of a wait on a barrier nothing arrives on
};

template <int L>
__global__ void __launch_bounds__(Geo<L>::THREADS, 1) k_mx_fft2(MxFft2Args a) {
    using G = Geo<L>;
    using F = TcFft<L>;
    constexpr int N = G::N, N2 = G::N2, T = G::THREADS;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *fn2 = smem;
    unsigned char *b2 = smem + G::FN2_BYTES;                 // stage-2 operand, then the output staging
    float *red = reinterpret_cast<float *>(b2 + G::B2_BYTES);
    __shared__ __align__(8) uint64_t bar;
    __shared__ __align__(8) uint64_t unarmed;                 // test hook: nothing ever arrives here
    __shared__ uint32_t tbase;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, q = warp & 3, g = warp >> 2;
    if (warp == 0) tc::tmem_alloc(&tbase, G::TMEM_COLS);
    if (tid == 0) {
        tc::mbar_init(&bar, 1);
        tc::mbar_init(&unarmed, 1);
        tc::mbar_fence_init();
    }
    F::load_fn2(a.fn2, fn2, tid);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = tbase;
    F::load_f128(a.f128, tm, q, g, lane);
    const uint32_t fn2_s = tc::smem_u32(fn2), b2_s = tc::smem_u32(b2);
    uint32_t phase = 0;
    bool ok = true;
    const int ln = 32 * q + lane;                            // TMEM lane: n1 on input, k1 on output
    float2 twr[16];
    F::twiddles(twr, a.tw, ln, g);
    // Software pipeline over this CTA's lines: while the tensor core runs stage 1 of line r the CUDA
    // cores detect and store line r - step; while it runs stage 2 of line r they scale, split and stage
    // line r + step into the (then free) stage-1 operand columns.
    float2 xn[16];
    auto load_row = [&](int r) {
        // the cross-FFT rows are already conjugated for the inverse (pass 2 conjugates its input)
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            const int j = ln + 128 * (16 * g + c);            // range bins j >= n are the zero pad
            xn[c] = j < a.n ? __ldcs(a.y1t + (size_t)r * a.npad + j) : make_float2(0.f, 0.f);
        }
    };
    // scale and stage the line held in xn into the stage-1 operand; returns its scale
    auto stage_input = [&]() {
        float mx = 0.f;
#pragma unroll
        for (int c = 0; c < 16; ++c) mx = fmaxf(mx, fmaxf(fabsf(xn[c].x), fabsf(xn[c].y)));
        const float s1 = F::line_scale(mx, red, warp, lane);
        if (ok) {
            tc::fence_after_sync();
            F::put_input(xn, s1, tm, q, g);
        }
        return s1;
    };
    auto emit = [&](const float2 (&y)[16], float s1, int r) {
        const float sc = a.scale * ((float)N2 / s1);
        const float cs = a.inverse ? -sc : sc;                // inverse: conj(FFT(conj(x)))
        const int v0 = N2 * ln + 16 * g;                      // first output column of this thread
        float4 *stg = reinterpret_cast<float4 *>(b2);
        if (a.detect == PFA_DETECT_COMPLEX) {
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                float2 z0 = make_float2(y[2 * c].x * sc, y[2 * c].y * cs);
                float2 z1 = make_float2(y[2 * c + 1].x * sc, y[2 * c + 1].y * cs);
                if (a.centred && ((r + v0) & 1)) { z0.x = -z0.x; z0.y = -z0.y; }   // v0 + 2c has v0's parity
                if (a.centred && !((r + v0) & 1)) { z1.x = -z1.x; z1.y = -z1.y; }
                stg[tcfft::swz_chunk<ilog2c(N2 / 2)>((v0 >> 1) + c)] = make_float4(z0.x, z0.y, z1.x, z1.y);
            }
        } else {
            const bool mag = a.detect == PFA_DETECT_MAG;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                float o[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float zr = y[4 * c + e].x * sc, zi = y[4 * c + e].y * cs;
                    const float p = fmaf(zr, zr, zi * zi);
                    o[e] = mag ? sqrtf(p) : p;
                }
                stg[tcfft::swz_chunk<ilog2c(N2 / 4)>((v0 >> 2) + c)] = make_float4(o[0], o[1], o[2], o[3]);
            }
        }
        __syncthreads();
        if (a.detect == PFA_DETECT_COMPLEX) {
            float4 *dst = reinterpret_cast<float4 *>(static_cast<float2 *>(a.out) + (size_t)r * N);
            for (int ch = tid; ch < N / 2; ch += T) __stcs(dst + ch, stg[tcfft::swz_chunk<ilog2c(N2 / 2)>(ch)]);
        } else {
            float4 *dst = reinterpret_cast<float4 *>(static_cast<float *>(a.out) + (size_t)r * N);
            for (int ch = tid; ch < N / 4; ch += T) __stcs(dst + ch, stg[tcfft::swz_chunk<ilog2c(N2 / 4)>(ch)]);
        }
    };
    const int step = gridDim.x;
    int r = blockIdx.x;                                       // < rows: the grid is min(rows, SMs)
    load_row(r);
    float s_cur = stage_input();
    if (r + step < a.rows) load_row(r + step);
    tc::fence_before_sync();
    __syncthreads();
    if (a.probe > 0) {                                        // the bounded-wait path, before any MMA
        const bool mine = tc::mbar_wait(&unarmed, 0, (uint32_t)a.probe);
        ok = __syncthreads_and(mine) != 0;
    }
    if (tid == 0 && ok) {
        tc::fence_after_sync();
        F::issue_stage1(tm, fn2_s);
        tc::commit(&bar);
    }
    float2 yprev[16];
    float s_prev = 1.f;
    int r_prev = -1;
    for (; r < a.rows; r += step) {
        const int rn = r + step;
        if (r_prev >= 0) emit(yprev, s_prev, r_prev);         // overlaps stage 1 of line r
        ok = cta_wait(&bar, phase, ok);
        phase ^= 1u;
        tc::fence_after_sync();
        if (ok) F::epilogue1(tm, b2, twr, q, g, lane);
        tc::fence_smem_to_async();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0 && ok) {
            tc::fence_after_sync();
            F::issue_stage2(tm, b2_s);
            tc::commit(&bar);
        }
        float s_next = 1.f;
        if (rn < a.rows) {                                    // overlaps stage 2 of line r
            s_next = stage_input();
            if (rn + step < a.rows) load_row(rn + step);
        }
        ok = cta_wait(&bar, phase, ok);
        phase ^= 1u;
        tc::fence_after_sync();
        if (ok) {
            F::get_output(yprev, tm, q, g);
        } else {
#pragma unroll
            for (int c = 0; c < 16; ++c) yprev[c] = make_float2(0.f, 0.f);
        }
        s_prev = s_cur;
        r_prev = r;
        s_cur = s_next;
        tc::fence_before_sync();
        __syncthreads();
        if (rn < a.rows && tid == 0 && ok) {
            tc::fence_after_sync();
            F::issue_stage1(tm, fn2_s);
            tc::commit(&bar);
        }
    }
    if (r_prev >= 0) emit(yprev, s_prev, r_prev);
    if (!ok && tid == 0) atomicExch(a.err, 1);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tm, G::TMEM_COLS);
}

// ------------------------------------------------------------------------------------------ pass 2
struct MxPass2Args {
    const float2 *p1;
    const double *tan_s, *kr_grid, *kc_grid, *ham_m, *ham_n;
    const int16_t *tabq;
    const float2 *tw;
    const uint4 *fn2, *f128;
    float2 *y1t;
    int *err;
    int m, n, mpad, npad, centred, window, inverse, ngroups;
};

template <int L, bool SINC>
__global__ void __cluster_dims__(kMxCT, 1, 1) __launch_bounds__(Geo<L>::THREADS, 1) k_mx_pass2(MxPass2Args a) {
    using G = Geo<L>;
    using F = TcFft<L>;
    constexpr int N = G::N, N2 = G::N2, T = G::THREADS;
    extern __shared__ __align__(128) unsigned char smem[];
    const int m = a.m;
    const size_t row_bytes = ((size_t)8 * m + 15) & ~(size_t)15;
    unsigned char *fn2 = smem;
    unsigned char *b2 = smem + G::FN2_BYTES;                 // stage-2 operand, then the exchange line
    float2 *row = reinterpret_cast<float2 *>(b2 + G::B2_BYTES);
    int16_t *tab = reinterpret_cast<int16_t *>(b2 + G::B2_BYTES + row_bytes);
    float *red = reinterpret_cast<float *>(b2 + G::B2_BYTES + row_bytes + (SINC ? 2 * kTabShorts : 0));
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tbase;
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int cid = blockIdx.x / kMxCT, ncl = gridDim.x / kMxCT;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, q = warp & 3, g = warp >> 2;
    if (warp == 0) tc::tmem_alloc(&tbase, G::TMEM_COLS);
    if (tid == 0) {
        tc::mbar_init(&bar, 1);
        tc::mbar_fence_init();
    }
    F::load_fn2(a.fn2, fn2, tid);
    if (SINC)
        for (int i = tid; i < kTabShorts / 8; i += T)
            reinterpret_cast<uint4 *>(tab)[i] = __ldg(reinterpret_cast<const uint4 *>(a.tabq) + i);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = tbase;
    F::load_f128(a.f128, tm, q, g, lane);
    const uint32_t fn2_s = tc::smem_u32(fn2), b2_s = tc::smem_u32(b2);
    uint32_t phase = 0;
    bool ok = true;
    const int ln = 32 * q + lane;
    float2 twr[16];
    F::twiddles(twr, a.tw, ln, g);
    // p1 rows stream into shared memory one line ahead: issued once the previous gather is done
    auto fetch_row = [&](int grp) {
        const int jr = grp * kMxCT + rank;
        if (grp >= a.ngroups || jr >= a.n) return;
        const float2 *src = a.p1 + (size_t)jr * a.mpad;          // 256-byte aligned rows
        for (int c = tid; c < ((m + 1) >> 1); c += T) cp_async16(row + 2 * c, src + 2 * c);
        cp_async_commit();
    };
    // The pass-2 line of group grp (this CTA's range bin): gather, window, centring sign, conj for the
    // inverse; returns the line's max |component|.  Reads the p1 row fetched into shared memory.
    auto gather_line = [&](int grp, float2 (&x)[16]) {
        const int j = grp * kMxCT + rank;
        float mx = 0.f;
        if (j < a.n) {
            const double krj = a.kr_grid[j];
            const double e0 = krj * a.tan_s[0], e1 = krj * a.tan_s[m - 1];
            const bool asc = e1 >= e0;
            auto xa = [&](int t) { return krj * __ldg(a.tan_s + (asc ? t : m - 1 - t)); };
            const double lo_v = asc ? e0 : e1, hi_v = asc ? e1 : e0;
            const double inv_span = (double)(m - 1) / (hi_v - lo_v);
            const double hn = a.window ? a.ham_n[j] : 1.0;
            int bl[16];
            float bf[16];
            constexpr int CH = 4;
#pragma unroll
            for (int u0 = 0; u0 < 16; u0 += CH) {
                double qv[CH];
                bool okq[CH];
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    const int k = ln + 128 * (16 * g + u0 + c);
                    okq[c] = k < m;
                    qv[c] = okq[c] ? __ldg(a.kc_grid + k) : 0.0;
                }
                int ja[CH];
                Frac fr[CH];
                interp_brackets<SINC, CH>(xa, m, lo_v, hi_v, inv_span, qv, okq, ja, fr);
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    bl[u0 + c] = -1;
                    bf[u0 + c] = 0.f;
                    if (ja[c] >= 0) {
                        int lowi = ja[c];
                        if (!asc) { lowi = m - 2 - ja[c]; mirror_frac(fr[c]); }
                        bl[u0 + c] = lowi | (fr[c].ph << 16) | (fr[c].rev << 24);
                        bf[u0 + c] = fr[c].f;
                    }
                }
            }
            cp_async_wait_all();
            __syncthreads();
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                const int k = ln + 128 * (16 * g + c);
                float2 val = make_float2(0.f, 0.f);
                if (k < m && bl[c] >= 0) {
                    const Frac fr{bf[c], (bl[c] >> 16) & 0xff, (bl[c] >> 24) & 1};
                    val = gather_f32<SINC>(row, 0, m, bl[c] & 0xffff, fr, tab);
                    // np.outer(hamming(m), hamming(n)).astype(float32)[k, j]
                    const float wgt = a.window ? (float)(a.ham_m[k] * hn) : 1.0f;
                    const float sg = (a.centred && ((j + k) & 1)) ? -wgt : wgt;
                    val.x *= sg;
                    val.y *= sg;
                }
                x[c] = a.inverse ? make_float2(val.x, -val.y) : val;
                mx = fmaxf(mx, fmaxf(fabsf(x[c].x), fabsf(x[c].y)));
            }
        } else {
#pragma unroll
            for (int c = 0; c < 16; ++c) x[c] = make_float2(0.f, 0.f);
        }
        return mx;
    };
    // gather line grp, prefetch the row of the line after it, stage it into the stage-1 operand
    auto stage_line = [&](int grp) {
        float2 x[16];
        const float mx = gather_line(grp, x);
        const float s1 = F::line_scale(mx, red, warp, lane);   // its barriers end this line's gather
        fetch_row(grp + ncl);
        if (ok) {
            tc::fence_after_sync();
            F::put_input(x, s1, tm, q, g);
        }
        return s1;
    };
    // line grp in natural frequency order (stays conjugated for the inverse) -> exchange buffer, then
    // corner turn #2: this CTA writes cross bins [rank N/8, (rank+1) N/8) of the cluster's 8 range bins
    auto exchange = [&](const float2 (&y)[16], float s1, int grp) {
        const float sc = (float)N2 / s1;
        const int v0 = N2 * ln + 16 * g;
        float4 *xch = reinterpret_cast<float4 *>(b2);
#pragma unroll
        for (int c = 0; c < 8; ++c)
            xch[tcfft::swz_chunk<ilog2c(N2 / 2)>((v0 >> 1) + c)] =
                make_float4(y[2 * c].x * sc, y[2 * c].y * sc, y[2 * c + 1].x * sc, y[2 * c + 1].y * sc);
        cluster.sync();
#pragma unroll 4
        for (int s2 = 0; s2 < N / T; ++s2) {
            const int item = tid + T * s2;
            const int r8 = item & (kMxCT - 1);
            const int k = rank * (N / kMxCT) + item / kMxCT;
            const float2 *remote = cluster.map_shared_rank(reinterpret_cast<float2 *>(b2), r8);
            const int pos = 2 * tcfft::swz_chunk<ilog2c(N2 / 2)>(k >> 1) + (k & 1);
            a.y1t[(size_t)k * a.npad + grp * kMxCT + r8] = remote[pos];
        }
        cluster.sync();                                       // the peers are done with this buffer
    };
    // Software pipeline over the cluster's groups (every CTA of a cluster runs the same groups, so the
    // cluster barriers stay matched): the previous line's exchange runs while the tensor core computes
    // stage 1 of this line, the next line's gather and staging while it computes stage 2.
    fetch_row(cid);
    int grp = cid;                                            // < ngroups: the grid has at most ngroups clusters
    float s_cur = stage_line(grp);
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0 && ok) {
        tc::fence_after_sync();
        F::issue_stage1(tm, fn2_s);
        tc::commit(&bar);
    }
    float2 yprev[16];
    float s_prev = 1.f;
    int grp_prev = -1;
    for (; grp < a.ngroups; grp += ncl) {
        const int gn = grp + ncl;
        if (grp_prev >= 0) exchange(yprev, s_prev, grp_prev); // overlaps stage 1 of this line
        ok = cta_wait(&bar, phase, ok);
        phase ^= 1u;
        tc::fence_after_sync();
        if (ok) F::epilogue1(tm, b2, twr, q, g, lane);
        tc::fence_smem_to_async();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0 && ok) {
            tc::fence_after_sync();
            F::issue_stage2(tm, b2_s);
            tc::commit(&bar);
        }
        const float s_next = gn < a.ngroups ? stage_line(gn) : 1.f;   // overlaps stage 2 of this line
        ok = cta_wait(&bar, phase, ok);
        phase ^= 1u;
        tc::fence_after_sync();
        if (ok) {
            F::get_output(yprev, tm, q, g);
        } else {
#pragma unroll
            for (int c = 0; c < 16; ++c) yprev[c] = make_float2(0.f, 0.f);
        }
        s_prev = s_cur;
        grp_prev = grp;
        s_cur = s_next;
        tc::fence_before_sync();
        __syncthreads();
        if (gn < a.ngroups && tid == 0 && ok) {
            tc::fence_after_sync();
            F::issue_stage1(tm, fn2_s);
            tc::commit(&bar);
        }
    }
    if (grp_prev >= 0) exchange(yprev, s_prev, grp_prev);
    if (!ok && tid == 0) atomicExch(a.err, 1);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tm, G::TMEM_COLS);
}

// ------------------------------------------------------------------------------------------ launch
template <int L>
size_t fft2_smem() {
    return std::max(kMxMinSmem, (size_t)Geo<L>::FN2_BYTES + Geo<L>::B2_BYTES + 64 * 4);
}
template <int L, bool SINC>
size_t pass2_smem(int m) {
    return std::max(kMxMinSmem, (size_t)Geo<L>::FN2_BYTES + Geo<L>::B2_BYTES + (((size_t)8 * m + 15) & ~(size_t)15) +
                                    (SINC ? kTabShorts * 2 : 0) + 64 * 4);
}

template <int L>
cudaError_t launch_mx_fft2(const FloatDev &d, void *out, int detect, float scale, cudaStream_t st) {
    MxFft2Args p{d.y1, d.twn, d.mx_fn2n, d.mx_f128, out, d.wait_err, d.n, d.npad, d.m2,
                 d.layout == PFA_LAYOUT_CENTRED, detect, d.sgn > 0, scale, d.mx_probe};
    const size_t sm = fft2_smem<L>();
    auto fn = k_mx_fft2<L>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    fn<<<std::min(d.m2, d.sms), Geo<L>::THREADS, sm, st>>>(p);
    return cudaGetLastError();
}

template <int L, bool SINC>
cudaError_t launch_mx_pass2(const FloatDev &d, cudaStream_t st) {
    const int ngroups = d.npad / kMxCT;
    MxPass2Args p{d.p1, d.tan_s, d.kr, d.kc, d.ham_m64, d.ham_n64, d.tabq, d.twm, d.mx_fn2m, d.mx_f128, d.y1,
                  d.wait_err, d.m, d.n, d.mpad, d.npad, d.layout == PFA_LAYOUT_CENTRED, d.window, d.sgn > 0, ngroups};
    const size_t sm = pass2_smem<L, SINC>(d.m);
    auto fn = k_mx_pass2<L, SINC>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    const int ncl = std::max(1, std::min(ngroups, d.mx_clusters));
    fn<<<ncl * kMxCT, Geo<L>::THREADS, sm, st>>>(p);
    return cudaGetLastError();
}

template <int L, bool SINC>
int clusters_of(const FloatDev &d) {
    const size_t sm = pass2_smem<L, SINC>(d.m);
    auto fn = k_mx_pass2<L, SINC>;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kMxCT * d.sms);
    cfg.blockDim = dim3(Geo<L>::THREADS);
    cfg.dynamicSmemBytes = sm;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, (void *)fn, &cfg) != cudaSuccess) return 0;
    return n;
}

// host fp16 of a float64 value and of the remainder
void split_host(double v, uint16_t &hi, uint16_t &lo) {
    const __half h = __float2half_rn((float)v);
    const __half l = __float2half_rn((float)(v - (double)__half2float(h)));
    hi = __half_raw(h).x;
    lo = __half_raw(l).x;
}

// F_N2 shared-memory image: arrays Frh, Frl, Fih, Fil, element (n2, k2) MN-major
std::vector<uint16_t> fn2_image(int N2) {
    std::vector<uint16_t> img(4 * (size_t)N2 * N2);
    const size_t arr = (size_t)N2 * N2;
    for (int a = 0; a < N2; ++a)
        for (int b = 0; b < N2; ++b) {
            const double th = -2.0 * M_PI * (double)((a * b) % N2) / (double)N2;
            uint16_t rh, rl, ih, il;
            split_host(std::cos(th), rh, rl);
            split_host(std::sin(th), ih, il);
            const size_t o = tc::mnmajor_off(a, b, N2) / 2;
            img[0 * arr + o] = rh;
            img[1 * arr + o] = rl;
            img[2 * arr + o] = ih;
            img[3 * arr + o] = il;
        }
    return img;
}

// F_128 TMEM image: lane k1, column c = array * 64 + p holds F_128[k1][2p], F_128[k1][2p+1]
std::vector<uint32_t> f128_image() {
    std::vector<uint32_t> img(128 * 256);
    for (int k1 = 0; k1 < 128; ++k1)
        for (int p = 0; p < 64; ++p) {
            uint16_t v[4][2];
            for (int e = 0; e < 2; ++e) {
                const int n1 = 2 * p + e;
                const double th = -2.0 * M_PI * (double)((k1 * n1) % 128) / 128.0;
                split_host(std::cos(th), v[0][e], v[1][e]);
                split_host(std::sin(th), v[2][e], v[3][e]);
            }
            for (int a = 0; a < 4; ++a) img[k1 * 256 + a * 64 + p] = (uint32_t)v[a][0] | ((uint32_t)v[a][1] << 16);
        }
    return img;
}

template <class T>
cudaError_t upload(T **dst, const void *src, size_t bytes) {
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(dst), bytes);
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
}

}  // namespace

bool mixed_axis(int L) { return L >= 11 && L <= 13; }

cudaError_t mixed_prepare(FloatDev &d) {
    cudaError_t e;
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const std::vector<uint32_t> f128 = f128_image();
    if ((e = upload(&d.mx_f128, f128.data(), f128.size() * 4)) != cudaSuccess) return e;
    if (mixed_axis(d.Lm)) {
        const std::vector<uint16_t> im = fn2_image(d.m2 / 128);
        if ((e = upload(&d.mx_fn2m, im.data(), im.size() * 2)) != cudaSuccess) return e;
        switch (d.Lm) {
            case 11: d.mx_clusters = d.az_sinc ? clusters_of<11, true>(d) : clusters_of<11, false>(d); break;
            case 12: d.mx_clusters = d.az_sinc ? clusters_of<12, true>(d) : clusters_of<12, false>(d); break;
            default: d.mx_clusters = d.az_sinc ? clusters_of<13, true>(d) : clusters_of<13, false>(d); break;
        }
        if (d.mx_clusters < 1) d.mx_clusters = std::max(1, d.sms / kMxCT);   // grid size only: clusters are independent
    }
    if (mixed_axis(d.Ln)) {
        const std::vector<uint16_t> im = fn2_image(d.n2 / 128);
        if ((e = upload(&d.mx_fn2n, im.data(), im.size() * 2)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void mixed_free(FloatDev &d) {
    if (d.mx_f128) cudaFree(d.mx_f128);
    if (d.mx_fn2m) cudaFree(d.mx_fn2m);
    if (d.mx_fn2n) cudaFree(d.mx_fn2n);
    d.mx_f128 = nullptr;
    d.mx_fn2m = d.mx_fn2n = nullptr;
}

cudaError_t mixed_pass2(const FloatDev &d, cudaStream_t st) {
    switch (d.Lm) {
        case 11: return d.az_sinc ? launch_mx_pass2<11, true>(d, st) : launch_mx_pass2<11, false>(d, st);
        case 12: return d.az_sinc ? launch_mx_pass2<12, true>(d, st) : launch_mx_pass2<12, false>(d, st);
        case 13: return d.az_sinc ? launch_mx_pass2<13, true>(d, st) : launch_mx_pass2<13, false>(d, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t mixed_fft2(const FloatDev &d, void *out, int detect, float scale, cudaStream_t st) {
    switch (d.Ln) {
        case 11: return launch_mx_fft2<11>(d, out, detect, scale, st);
        case 12: return launch_mx_fft2<12>(d, out, detect, scale, st);
        case 13: return launch_mx_fft2<13>(d, out, detect, scale, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace pfa
