// Fixed-point PFA datapath on sm_100a, bit-exact to the reference emulator
// (mpfs/host/silicon_emulator.py:226-249).
//
// Kernels (one stream, stream-ordered):
//   k_q0max        block max of |re|,|im| over the complex64 signal (fixedpoint.fit_scale, :19-26)
//   k_fx_pass1     Q0 quantise + pass-1 bracket search (FP64) + 32-tap sinc / 2-tap lerp gather per
//                  pulse; a 32-slot x 128-bin shared tile turns the pulse-major output into range-bin
//                  rows (corner turn #1, silicon_emulator.py:142-148)
//   k_fx_pass2_fft pass-2 bracket search + gather + Q15 window + 13-stage per-row BFP FFT along the
//                  cross axis (silicon_emulator.py:150-156, 165-195, 198-205 with fixedpoint.py:266-289)
//   k_fx_fft2      renormalise FFT-1 rows by (emax - e_row) on load, BFP FFT along range
//                  (corner turn #2 by strided column reads, silicon_emulator.py:241-245)
//   k_fx_detect    renormalise FFT-2 rows, integer |z|, transpose to [range][cross] (:247-249, :208-213)
//
// Exactness notes.  Every floating step the emulator takes is reproduced with the same IEEE
// operation: __dmul_rn/__dadd_rn/__ddiv_rn (no FMA contraction) for the float64 coordinates and
// fractions, __fmul_rn/__fdiv_rn where NumPy 2 computes in float32 (pass-1 source scale, pass-2
// source coordinates, the Q0 division, the pass-1 lerp product), rint() for np.round.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "pfa_internal.h"

namespace pfa {
namespace {

constexpr int kSincTaps = 32;
constexpr int kSincFirst = -15;

__device__ __forceinline__ int sat16(int v) { return min(max(v, -32768), 32767); }
__device__ __forceinline__ long long sat16ll(long long v) { return v < -32768 ? -32768 : (v > 32767 ? 32767 : v); }
__device__ __forceinline__ uint32_t pack16(int re, int im) {
    return (uint32_t)(uint16_t)re | ((uint32_t)(uint16_t)im << 16);
}
__device__ __forceinline__ int lo16(uint32_t p) { return (int)(int16_t)(p & 0xffffu); }
__device__ __forceinline__ int hi16(uint32_t p) { return (int)(int16_t)(p >> 16); }
__device__ __forceinline__ int wrap16(int v) { return (int)(int16_t)(v & 0xffff); }

// Source samples are packed int16 I/Q words (pass-2 rows) or unpacked int32 pairs (pass-1 windows,
// one 8-byte shared load per tap instead of a load and two sign extensions).
__device__ __forceinline__ int re_of(uint32_t v) { return lo16(v); }
__device__ __forceinline__ int im_of(uint32_t v) { return hi16(v); }
__device__ __forceinline__ int re_of(int2 v) { return v.x; }
__device__ __forceinline__ int im_of(int2 v) { return v.y; }

// 16-byte global -> shared copies that complete asynchronously (both addresses 16-byte aligned)
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// Bulk prefetch of `bytes` (16-byte aligned, a multiple of 16) into L2, 16 KB per instruction by the first
// threads of the block: a line kernel prefetches the row of the block that starts when this one ends.
__device__ __forceinline__ void l2_prefetch(const void *p, size_t bytes, int tid) {
    constexpr size_t CH = 16384;
    const size_t off = (size_t)tid * CH;
    if (off < bytes) {
        const uint32_t sz = (uint32_t)(bytes - off < CH ? bytes - off : CH);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(static_cast<const char *>(p) + off), "r"(sz)
                     : "memory");
    }
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Smallest e with M <= 32767 * 2^e, i.e. ceil(log2(M / 32767)) of fixedpoint.fit_scale for a float32
// maximum M (exact: M/32767 is either an exact power of two or at least 2^-24 away from one).
__device__ __forceinline__ int q0_exponent(uint32_t bits) {
    float M = __uint_as_float(bits);
    if (!(M > 0.0f)) return 0;
    double md = (double)M;
    int e = ilogb(md) - 15;
    while (md > ldexp(32767.0, e)) ++e;
    return e;
}

// floor(x / lsb) in float32 (the emulator divides float32 planes by a weak float scalar), sat16.
__device__ __forceinline__ int q0_quantise(float x, float lsb) {
    return sat16((int)fmaxf(fminf(floorf(__fdiv_rn(x, lsb)), 32767.0f), -32768.0f));
}

// lower_bound over a non-decreasing sequence xa(0..n-1): first t with xa(t) >= q (n if none).
// Starts from a guess and walks; falls back to bisection after a few steps.
template <class F>
__device__ __forceinline__ int lower_bound_from(const F &xa, int n, double q, int g) {
    int t = min(max(g, 0), n);
    int steps = 0;
    while (t < n && xa(t) < q) {
        ++t;
        if (++steps > 6) {
            int lo = t, hi = n;
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (xa(mid) < q) lo = mid + 1; else hi = mid;
            }
            return lo;
        }
    }
    while (t > 0 && xa(t - 1) >= q) {
        --t;
        if (++steps > 6) {
            int lo = 0, hi = t;
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (xa(mid) < q) lo = mid + 1; else hi = mid;
            }
            return lo;
        }
    }
    return t;
}

struct Bracket {
    int idx;   // natural-order lower index, -1 = out of span
    int wq;    // Q15 weight
};

// interp_coeffs (serialize_inputs.py:67-94) for one query, given the count of ascending-view
// source coordinates below q and an accessor of the ascending view.
template <class F>
__device__ __forceinline__ Bracket bracket_from_count(const F &xa, int n, bool asc, double q, int cnt) {
    Bracket b{-1, 0};
    int k = cnt - 1;
    if (k < 0 || k >= n - 1) return b;
    double x0 = xa(k), x1 = xa(k + 1);
    double fa = __ddiv_rn(__dsub_rn(q, x0), __dsub_rn(x1, x0));
    double w = asc ? fa : __dsub_rn(1.0, fa);
    double r = rint(__dmul_rn(w, 32768.0));
    r = fmin(fmax(r, 0.0), 32767.0);
    b.idx = asc ? k : (n - 2 - k);
    b.wq = (int)r;
    return b;
}

// 32-tap sinc / edge lerp / zero of apply_sinc (silicon_emulator.py:88-122) on a window of packed
// int16x2 samples; `win` is indexed by (source index - base).
template <class W>
__device__ __forceinline__ uint32_t sinc_gather(const W *win, int base, int sn, Bracket b, const int16_t *tab) {
    if (b.idx < 0) return 0u;
    if (b.idx >= -kSincFirst && b.idx <= sn - (kSincTaps + kSincFirst)) {
        const int16_t *c = tab + (b.wq >> 7);           // table stored [tap][phase] (the global layout)
        const W *x = win + (b.idx + kSincFirst - base);
        // Two int32 half sums (taps 0-15, 16-31): the table is checked on upload to have
        // sum |tap| <= 65535 over each half of every phase, so |half sum| <= 32768 * 65535 < 2^31.
        int ar0 = 0, ai0 = 0, ar1 = 0, ai1 = 0;
#pragma unroll
        for (int t = 0; t < kSincTaps / 2; ++t) {
            const int ct = c[t * 256];
            const W v = x[t];
            ar0 += ct * re_of(v);
            ai0 += ct * im_of(v);
        }
#pragma unroll
        for (int t = kSincTaps / 2; t < kSincTaps; ++t) {
            const int ct = c[t * 256];
            const W v = x[t];
            ar1 += ct * re_of(v);
            ai1 += ct * im_of(v);
        }
        const long long ar = (long long)ar0 + ar1, ai = (long long)ai0 + ai1;
        return pack16((int)sat16ll((ar + (1 << 14)) >> 15), (int)sat16ll((ai + (1 << 14)) >> 15));
    }
    const W va = win[b.idx - base], vb = win[b.idx + 1 - base];
    const int ar = re_of(va), ai = im_of(va), br = re_of(vb), bi = im_of(vb);
    return pack16(sat16(ar + (((br - ar) * b.wq) >> 15)), sat16(ai + (((bi - ai) * b.wq) >> 15)));
}

// The same gather with the table in shared memory as phase-major rows of kSincRow int16 (taps 0..31,
// then padding): a lane reads its phase's 32 taps as four 16-byte loads, and the 80-byte row stride
// puts the rows of eight consecutive phases on distinct 16-byte bank groups.
constexpr int kSincRow = 40;
template <class W>
__device__ __forceinline__ uint32_t sinc_gather_pm(const W *win, int base, int sn, Bracket b, const int16_t *tab_pm) {
    if (b.idx < 0) return 0u;
    if (b.idx >= -kSincFirst && b.idx <= sn - (kSincTaps + kSincFirst)) {
        const uint4 *c4 = reinterpret_cast<const uint4 *>(tab_pm + (b.wq >> 7) * kSincRow);
        const W *x = win + (b.idx + kSincFirst - base);
        // the int32 half sums of sinc_gather (same bound, same exact integer result)
        int ar0 = 0, ai0 = 0, ar1 = 0, ai1 = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint4 u = c4[q];
            const uint32_t wd[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int t = 8 * q + e;                  // tap 2k in the low half of word k
                const int ct = (e & 1) ? ((int)wd[e >> 1] >> 16) : (int)(int16_t)(wd[e >> 1] & 0xffffu);
                const W v = x[t];
                if (t < kSincTaps / 2) {
                    ar0 += ct * re_of(v);
                    ai0 += ct * im_of(v);
                } else {
                    ar1 += ct * re_of(v);
                    ai1 += ct * im_of(v);
                }
            }
        }
        const long long ar = (long long)ar0 + ar1, ai = (long long)ai0 + ai1;
        return pack16((int)sat16ll((ar + (1 << 14)) >> 15), (int)sat16ll((ai + (1 << 14)) >> 15));
    }
    const W va = win[b.idx - base], vb = win[b.idx + 1 - base];
    const int ar = re_of(va), ai = im_of(va), br = re_of(vb), bi = im_of(vb);
    return pack16(sat16(ar + (((br - ar) * b.wq) >> 15)), sat16(ai + (((bi - ai) * b.wq) >> 15)));
}

// apply_fixed (silicon_emulator.py:60-71).  F32PROD: the product (b-a)*wq rounded to float32, as in
// pass 1 where the emulator's quantised signal is complex64.
template <bool F32PROD, class W>
__device__ __forceinline__ uint32_t lerp_gather(const W *win, int base, Bracket b) {
    if (b.idx < 0) return 0u;
    const W va = win[b.idx - base], vb = win[b.idx + 1 - base];
    const int ar = re_of(va), ai = im_of(va), br = re_of(vb), bi = im_of(vb);
    int sr, si;
    if (F32PROD) {
        const float w = (float)b.wq;
        sr = (int)floorf(__fmul_rn(__fmul_rn((float)(br - ar), w), 1.0f / 32768.0f));
        si = (int)floorf(__fmul_rn(__fmul_rn((float)(bi - ai), w), 1.0f / 32768.0f));
    } else {
        sr = ((br - ar) * b.wq) >> 15;
        si = ((bi - ai) * b.wq) >> 15;
    }
    return pack16(sat16(ar + sr), sat16(ai + si));
}

// floor(a / b) for b > 0 (C division truncates toward zero)
__device__ __forceinline__ int floordiv64(long long a, long long b) {
    const long long q = a / b;
    return (int)((a % b != 0 && a < 0) ? q - 1 : q);
}

// 4-point cubic Lagrange taps at mu = w / 2^15 in Q15 (gen_resample_vectors.lagrange_taps_q15,
// mpfs/fpga/tb/gen_resample_vectors.py:177-195): each tap's exact value x 2^15 is N / D with integer
// N (|N| < 2^48) and D, rounded half up once: floor((2 N + D) / (2 D)).
__device__ __forceinline__ void lagrange_q15(int w, int (&c)[4]) {
    const long long W = w, A = W + 32768, B = W - 32768, C = W - 65536;
    const long long d6 = 6LL << 30, d2 = 1LL << 31;
    c[0] = floordiv64(2 * (-(W * B * C)) + d6, 2 * d6);
    c[1] = floordiv64(2 * (A * B * C) + d2, 2 * d2);
    c[2] = floordiv64(2 * (-(A * W * C)) + d2, 2 * d2);
    c[3] = floordiv64(2 * (A * W * B) + d6, 2 * d6);
}

// gen_resample_vectors.gather_cubic (:298-325): taps at idx-1..idx+2 where 1 <= idx <= sn-3, sum >> 15
// (floor), sat16; other live brackets take the integer 2-tap lerp; idx < 0 gives 0.
template <class W>
__device__ __forceinline__ uint32_t cubic_gather(const W *win, int base, int sn, Bracket b) {
    if (b.idx < 0) return 0u;
    if (b.idx >= 1 && b.idx <= sn - 3) {
        int c[4];
        lagrange_q15(b.wq, c);
        const W *x = win + (b.idx - 1 - base);
        long long ar = 0, ai = 0;
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            ar += (long long)c[t] * re_of(x[t]);
            ai += (long long)c[t] * im_of(x[t]);
        }
        return pack16((int)sat16ll(ar >> 15), (int)sat16ll(ai >> 15));
    }
    return lerp_gather<false>(win, base, b);
}

// ------------------------------------------------------------------------------------------ K0
__global__ void k_q0max(const float4 *__restrict__ sig4, long long n4, const float *__restrict__ tail,
                        int ntail, uint32_t *__restrict__ out_bits) {
    float mx = 0.0f;
    const long long stride = (long long)gridDim.x * blockDim.x;
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n4; i += 4 * stride) {      // four independent loads in flight
        float4 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = __ldcs(sig4 + i + u * stride);
#pragma unroll
        for (int u = 0; u < 4; ++u)
            mx = fmaxf(mx, fmaxf(fmaxf(fabsf(v[u].x), fabsf(v[u].y)), fmaxf(fabsf(v[u].z), fabsf(v[u].w))));
    }
    for (; i < n4; i += stride) {
        const float4 v = __ldcs(sig4 + i);
        mx = fmaxf(mx, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
    }
    if (blockIdx.x == 0 && threadIdx.x < ntail) mx = fmaxf(mx, fabsf(tail[threadIdx.x]));
    uint32_t b = __reduce_max_sync(0xffffffffu, __float_as_uint(mx));
    if ((threadIdx.x & 31) == 0) atomicMax(out_bits, b);
}

__global__ void k_q0exp(int32_t *ctrl) { ctrl[3] = q0_exponent((uint32_t)ctrl[0]); }

// ------------------------------------------------------------------------------------------ K1
constexpr int P1_SLOTS = 32;          // sorted pulse slots per CTA
constexpr int P1_BINS = 128;          // range bins per CTA
constexpr int P1_WARPS = 8;
constexpr int P1_WMAX = 256;          // per-warp source window (samples); wider windows gather from global

struct Pass1Args {
    const float2 *sig;                // complex64 input (or nullptr)
    const uint32_t *sig_iq;           // packed int16 I/Q input (or nullptr)
    const float *f0, *df, *fac, *krp;
    const int32_t *order;
    const int16_t *sinc;
    const int32_t *ctrl;
    uint32_t *p1;
    int m, n, mpad;
    int cubic;                        // 4-tap Lagrange instead of the lerp (SINC off)
};

// per-slot pulse constants, computed once per CTA
struct P1Pulse {
    double fac, f0, df, inv_step, c0;
    int i;                            // source pulse, -1 for a slot past the last pulse
    int asc;
};

constexpr size_t P1_SMEM_TILE = (size_t)P1_BINS * (P1_SLOTS + 1) * 4;
constexpr size_t P1_SMEM_WIN = (size_t)P1_WARPS * P1_WMAX * 8;   // int32 I/Q pairs
constexpr size_t p1_smem(bool sinc) { return P1_SMEM_TILE + P1_SMEM_WIN + (sinc ? 2 * 256 * kSincRow : 0); }

template <bool SINC>
__global__ void __launch_bounds__(256, 4) k_fx_pass1(Pass1Args a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t(*tile)[P1_SLOTS + 1] = reinterpret_cast<uint32_t(*)[P1_SLOTS + 1]>(smem);
    int2(*win)[P1_WMAX] = reinterpret_cast<int2(*)[P1_WMAX]>(smem + P1_SMEM_TILE);
    int16_t *tab = reinterpret_cast<int16_t *>(smem + P1_SMEM_TILE + P1_SMEM_WIN);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = blockIdx.x * P1_SLOTS;
    const int j0 = blockIdx.y * P1_BINS;
    const int n = a.n;
    if (SINC) {
        // [tap][phase] in global memory -> phase-major rows of kSincRow in shared memory
        for (int i = tid; i < 256 * kSincTaps; i += blockDim.x) tab[(i & 255) * kSincRow + (i >> 8)] = a.sinc[i];
    }
    __shared__ P1Pulse prm[P1_SLOTS];
    if (tid < P1_SLOTS) {
        P1Pulse p{};
        p.i = -1;
        const int r = r0 + tid;
        if (r < a.m) {
            const int i = a.order[r];
            p.i = i;
            p.fac = (double)a.fac[i];
            p.f0 = (double)a.f0[i];
            p.df = (double)a.df[i];
            // kr_i[k] = f64(fac) * (f64(f0) + f64(k) * f64(df))   (silicon_emulator.py:144)
            auto kr = [&](int k) { return __dmul_rn(p.fac, __dadd_rn(p.f0, __dmul_rn((double)k, p.df))); };
            p.asc = kr(n - 1) >= kr(0);
            p.inv_step = 1.0 / (p.fac * p.df);      // affine-estimate coefficients (guess only)
            p.c0 = p.f0 / p.df;
        }
        prm[tid] = p;
    }
    // the query wavenumbers of this CTA's bins are the same for every pulse
    double qv[P1_BINS / 32];
#pragma unroll
    for (int t = 0; t < P1_BINS / 32; ++t) {
        const int j = j0 + lane + 32 * t;
        qv[t] = j < n ? (double)a.krp[j] : 0.0;
    }
    const float lsb = a.sig ? (float)ldexp(1.0, a.ctrl[3]) : 1.0f;
    __syncthreads();

    for (int s = 0; s < P1_SLOTS / P1_WARPS; ++s) {
        const int slot = warp + P1_WARPS * s;
        const P1Pulse &p = prm[slot];
        if (p.i < 0) {
            for (int t = lane; t < P1_BINS; t += 32) tile[t][slot] = 0u;
            continue;
        }
        const int i = p.i;
        const double fac = p.fac, f0 = p.f0, df = p.df;
        auto kr = [&](int k) { return __dmul_rn(fac, __dadd_rn(f0, __dmul_rn((double)k, df))); };
        const bool asc = p.asc;
        auto xa = [&](int t) { return asc ? kr(t) : kr(n - 1 - t); };
        const double inv_step = p.inv_step, c0 = p.c0;
        Bracket br[P1_BINS / 32];
        int lo_i = 1 << 30, hi_i = -1;
#pragma unroll
        for (int t = 0; t < P1_BINS / 32; ++t) {
            const int j = j0 + lane + 32 * t;
            br[t] = Bracket{-1, 0};
            if (j < n) {
                const double q = qv[t];
                const double kest = q * inv_step - c0;     // affine estimate of the source index
                int g = 0;
                if (isfinite(kest) && isfinite(inv_step)) {
                    const double tt = asc ? ceil(kest) : ceil((double)(n - 1) - kest);
                    g = (int)fmin(fmax(tt, -1.0), (double)n + 1.0);
                }
                const int cnt = lower_bound_from(xa, n, q, g);
                br[t] = bracket_from_count(xa, n, asc, q, cnt);
                if (br[t].idx >= 0) {
                    lo_i = min(lo_i, br[t].idx);
                    hi_i = max(hi_i, br[t].idx);
                }
            }
        }
        lo_i = __reduce_min_sync(0xffffffffu, lo_i);
        hi_i = __reduce_max_sync(0xffffffffu, hi_i);
        int wlo = 0, whi = 0;
        if (hi_i >= 0) {
            wlo = max(0, lo_i + (SINC ? kSincFirst : (a.cubic ? -1 : 0)));
            whi = min(n, hi_i + (SINC ? kSincTaps + kSincFirst : (a.cubic ? 3 : 2)));
        }
        const bool fits = (whi - wlo) <= P1_WMAX;
        int2 *w = win[warp];
        if (fits) {
            for (int k = wlo + lane; k < whi; k += 32) {
                const size_t off = (size_t)i * n + k;
                int2 v;
                if (a.sig) {
                    const float2 z = a.sig[off];
                    v = make_int2(q0_quantise(z.x, lsb), q0_quantise(z.y, lsb));
                } else {
                    const uint32_t q = a.sig_iq[off];
                    v = make_int2(lo16(q), hi16(q));
                }
                w[k - wlo] = v;
            }
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < P1_BINS / 32; ++t) {
            const int jj = lane + 32 * t;
            uint32_t out = 0u;
            if (j0 + jj < n && br[t].idx >= 0) {
                if (fits) {
                    out = SINC ? sinc_gather_pm(w, wlo, n, br[t], tab)
                               : (a.cubic ? cubic_gather(w, wlo, n, br[t]) : lerp_gather<true>(w, wlo, br[t]));
                } else {
                    // Window wider than the staging buffer: gather straight from global memory.
                    uint32_t tmp[kSincTaps + 1];
                    const int base = SINC ? max(0, br[t].idx + kSincFirst) : (a.cubic ? max(0, br[t].idx - 1) : br[t].idx);
                    const int cnt = SINC ? min(n, br[t].idx + kSincTaps + kSincFirst) - base
                                         : (a.cubic ? min(n, br[t].idx + 3) - base : 2);
                    for (int u = 0; u < cnt; ++u) {
                        const size_t off = (size_t)i * n + base + u;
                        if (a.sig) {
                            const float2 z = a.sig[off];
                            tmp[u] = pack16(q0_quantise(z.x, lsb), q0_quantise(z.y, lsb));
                        } else {
                            tmp[u] = a.sig_iq[off];
                        }
                    }
                    out = SINC ? sinc_gather_pm(tmp, base, n, br[t], tab)
                               : (a.cubic ? cubic_gather(tmp, base, n, br[t]) : lerp_gather<true>(tmp, base, br[t]));
                }
            }
            tile[jj][slot] = out;
        }
        __syncwarp();
    }
    __syncthreads();
    // corner turn #1: range-bin rows, sorted-slot columns, 128 B per row segment; four slots per lane,
    // four bins per warp store (mpad is a multiple of 32: every slot of the CTA exists)
    const int quarter = lane >> 3, l4 = 4 * (lane & 7);
    for (int jj = 4 * warp + quarter; jj < P1_BINS; jj += 4 * P1_WARPS) {
        const int j = j0 + jj;
        if (j >= n) break;
        *reinterpret_cast<uint4 *>(a.p1 + (size_t)j * a.mpad + r0 + l4) =
            make_uint4(tile[jj][l4], tile[jj][l4 + 1], tile[jj][l4 + 2], tile[jj][l4 + 3]);
    }
}

// ------------------------------------------------------------------------------------------ BFP FFT
// Per-row block-floating-point radix-2 DIT FFT of fixedpoint.fft1d_bfp_hw_perrow (fixedpoint.py:266-289)
// held in registers: E values per thread, T = N/E threads.  Stages whose butterfly bit lies in a
// thread's register bits run in registers; between bit groups the row is exchanged through shared
// memory.  After every stage the row max of |re|,|im| sets the conditional shift (the same for every
// layout, so the per-stage arithmetic is identical to the reference).
//
// Positions p are those of the bit-reversed working array.  Group g with bit range [lo, lo+LE):
// element v of logical thread t sits at p = (t & (2^lo - 1)) | v << lo | (t >> lo) << (lo + LE).
// Group 0 uses logical t = bitrev(tid), so its element v holds natural input index tid + T*bitrev(v).
template <int L, int E>
struct BfpFft {
    static constexpr int N = 1 << L;
    static constexpr int LE = (E == 32) ? 5 : (E == 16) ? 4 : (E == 8) ? 3 : (E == 4) ? 2 : 1;
    static constexpr int T = N / E;
    static constexpr int TB = L - LE;        // thread bits
    static constexpr int WARPS = T / 32;
    static constexpr int NG = (L + LE - 1) / LE;
    static_assert(T >= 32, "at least one warp");

    __device__ static __forceinline__ int group_lo(int g) {
        return (g * LE + LE <= L) ? g * LE : (L - LE);
    }
    __device__ static __forceinline__ int pos(int lo, int t, int v) {
        return (t & ((1 << lo) - 1)) | (v << lo) | ((t >> lo) << (lo + LE));
    }
    __device__ static __forceinline__ int swz(int p) { return p + (p >> 5); }
    __device__ static __forceinline__ int logical(int g, int tid) {
        return g == 0 ? (int)(__brev((unsigned)tid) >> (32 - TB)) : tid;
    }

    // Runs the full transform on xr/xi (group-0 layout in, last-group layout out).  Returns e_row.
    __device__ static int run(int (&xr)[E], int (&xi)[E], uint32_t *xbuf, const uint32_t *tw,
                              int (*red)[32], int tid) {
        int e_row = 0;
        int done = 0;
        int rbuf = 0;
        int cur_max = 32768;                    // bound on |re|, |im| of the stage input (CTA-uniform)
        const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
        for (int g = 0; g < NG; ++g) {
            const int lo = group_lo(g);
            const int t = logical(g, tid);
            if (g > 0) {
                // exchange: write in group g-1 layout, read in group g layout
                const int plo = group_lo(g - 1);
                const int pt = logical(g - 1, tid);
#pragma unroll
                for (int v = 0; v < E; ++v) xbuf[swz(pos(plo, pt, v))] = pack16(xr[v], xi[v]);
                __syncthreads();
#pragma unroll
                for (int v = 0; v < E; ++v) {
                    const uint32_t u = xbuf[swz(pos(lo, t, v))];
                    xr[v] = lo16(u);
                    xi[v] = hi16(u);
                }
            }
            const int tlow = t & ((1 << lo) - 1);
#pragma unroll
            for (int rb = 0; rb < LE; ++rb) {
                const int b = lo + rb;
                if (b < done) continue;
                // stage s = b + 1: pairs (p, p + 2^b); twiddle k = p mod 2^b from the stage table
                const uint32_t *tws = tw + ((1 << b) - 1);
                // row max of |re|, |im| as max(largest, -smallest): no |.| per value
                int hi = 0, lo_ = 0;
                auto butterflies = [&](auto sat_tag) {
                    constexpr bool SAT = decltype(sat_tag)::value;
#pragma unroll
                    for (int v = 0; v < E; ++v) {
                        if (v & (1 << rb)) continue;
                        const int v2 = v | (1 << rb);
                        const int k = tlow | ((v & ((1 << rb) - 1)) << lo);
                        const uint32_t w = tws[k];
                        const int wr = lo16(w), wi = hi16(w);
                        const int br = xr[v2], bi = xi[v2];
                        int tr = (wr * br - wi * bi) >> 15;
                        int ti = (wr * bi + wi * br) >> 15;
                        if constexpr (SAT) {
                            tr = sat16(tr);
                            ti = sat16(ti);
                        }
                        const int ar = xr[v], ai = xi[v];
                        xr[v] = ar + tr;
                        xi[v] = ai + ti;
                        xr[v2] = ar - tr;
                        xi[v2] = ai - ti;
                        hi = __vimax3_s32(hi, __vimax3_s32(xr[v], xi[v], xr[v2]), xi[v2]);
                        lo_ = __vimin3_s32(lo_, __vimin3_s32(xr[v], xi[v], xr[v2]), xi[v2]);
                    }
                };
                // |t| <= |w| |b| / 2^15 + 1 <= 1.4143 cur_max + 1 (|w| <= 32770, |b| <= sqrt(2) cur_max):
                // with cur_max <= 23000 the twiddle product cannot leave int16, so its saturation is skipped
                if (cur_max <= 23000) butterflies(std::false_type{});
                else butterflies(std::true_type{});
                const unsigned mx = __reduce_max_sync(0xffffffffu, (unsigned)max(hi, -lo_));
                if (lane == 0) red[rbuf][warp] = (int)mx;
                __syncthreads();
                int rowmax = 0;
                if constexpr (WARPS % 4 == 0) {
                    const int4 *r4 = reinterpret_cast<const int4 *>(red[rbuf]);   // 128-byte rows, 16-byte aligned
#pragma unroll
                    for (int q = 0; q < WARPS / 4; ++q) {
                        const int4 v4 = r4[q];
                        rowmax = max(rowmax, max(max(v4.x, v4.y), max(v4.z, v4.w)));
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < WARPS; ++q) rowmax = max(rowmax, red[rbuf][q]);
                }
                rbuf ^= 1;
                // max(0, ceil(log2((mx + 1) / 32767))) on integers
                int sh = 0;
                while ((long long)rowmax + 1 > (32767LL << sh)) ++sh;
                // |x| <= rowmax < 32767 * 2^sh, so x >> sh lies in [-32767, 32766]: no saturation needed
                if (sh) {
#pragma unroll
                    for (int v = 0; v < E; ++v) {
                        xr[v] >>= sh;
                        xi[v] >>= sh;
                    }
                }
                cur_max = sh ? (rowmax >> sh) + 1 : rowmax;   // bound on |re|, |im| entering the next stage
                e_row += sh;
            }
            done = lo + LE;
        }
        return e_row;
    }
    // Output position of element v after run(): p = tid | v << (L - LE)
};

// ------------------------------------------------------------------------------------------ K2
struct Pass2Args {
    const uint32_t *p1;
    const float *tan_s, *krp, *kcp;
    const int32_t *hamr, *hamc;
    const uint32_t *tw;
    const int16_t *sinc;
    uint32_t *y1;
    int32_t *e1, *ctrl;
    int m, n, mpad;
    int cubic;                        // 4-tap Lagrange instead of the lerp (SINC off)
    int pf;                           // L2 prefetch distance in rows (resident blocks of the grid), 0 = none
};

template <int L, int E, bool SINC>
__global__ void __launch_bounds__((1 << L) / E) k_fx_pass2_fft(Pass2Args a) {
    using F = BfpFft<L, E>;
    constexpr int N = F::N, T = F::T;
    extern __shared__ __align__(16) unsigned char smem[];
    // layout: [region A: row as int32 I/Q pairs | exchange buffer] [tw N] [sinc] [red]
    const int m = a.m;
    const size_t rowb = (size_t)32 * ((m + 3) >> 2);
    const size_t regA = (max(rowb, (size_t)4 * (N + N / 32)) + 15) & ~(size_t)15;
    int2 *row = reinterpret_cast<int2 *>(smem);
    uint32_t *xbuf = reinterpret_cast<uint32_t *>(smem);
    uint32_t *tw = reinterpret_cast<uint32_t *>(smem + regA);
    int16_t *tab = reinterpret_cast<int16_t *>(smem + regA + 4 * (size_t)N);
    int(*red)[32] = reinterpret_cast<int(*)[32]>(smem + regA + 4 * (size_t)N + (SINC ? 2 * 256 * kSincTaps : 0));

    const int tid = threadIdx.x;
    const int j = blockIdx.x;                       // range bin (< n)
    // the twiddles and the sinc table stream in while the p1 row is unpacked into int32 I/Q pairs (one
    // 8-byte shared load per sinc tap, no sign extension in the gather)
    {
        if (a.pf && j + a.pf < a.n) l2_prefetch(a.p1 + (size_t)(j + a.pf) * a.mpad, (size_t)4 * a.mpad, tid);
        for (int c = tid; c < N / 4; c += T) cp_async16(tw + 4 * c, a.tw + 4 * c);
        if (SINC)
            for (int c = tid; c < 256 * kSincTaps / 8; c += T) cp_async16(tab + 8 * c, a.sinc + 8 * c);
        cp_async_commit();
        const uint4 *src = reinterpret_cast<const uint4 *>(a.p1 + (size_t)j * a.mpad);   // 128-byte aligned, mpad >= m
        int4 *dst = reinterpret_cast<int4 *>(row);
        for (int c = tid; c < (m + 3) >> 2; c += T) {
            const uint4 v = __ldg(src + c);
            dst[2 * c] = make_int4(lo16(v.x), hi16(v.x), lo16(v.y), hi16(v.y));
            dst[2 * c + 1] = make_int4(lo16(v.z), hi16(v.z), lo16(v.w), hi16(v.w));
        }
    }
    cp_async_wait_all();
    __syncthreads();

    // source coordinates KRp[j] * tan_s in float32 (silicon_emulator.py:152), from the L1-resident tan_s
    const float krj = a.krp[j];
    const bool asc = __fmul_rn(krj, a.tan_s[m - 1]) >= __fmul_rn(krj, a.tan_s[0]);
    auto xa = [&](int t) { return (double)__fmul_rn(krj, __ldg(a.tan_s + (asc ? t : m - 1 - t))); };
    const double lo_v = xa(0), hi_v = xa(m - 1);
    const double inv_span = (double)(m - 1) / (hi_v - lo_v);
    const int hr = a.hamr[j];

    int xr[E], xi[E];
#pragma unroll
    for (int u = 0; u < E; ++u) {
        const int k = tid + T * u;                  // natural cross index
        const double q = (double)a.kcp[k];
        Bracket b{-1, 0};
        if (q > lo_v && q <= hi_v) {
            const int g = (int)((q - lo_v) * inv_span) + 1;
            const int cnt = lower_bound_from(xa, m, q, g);
            b = bracket_from_count(xa, m, asc, q, cnt);
        }
        const uint32_t v = SINC ? sinc_gather(row, 0, m, b, tab)
                                : (a.cubic ? cubic_gather(row, 0, m, b) : lerp_gather<false>(row, 0, b));
        // window_fixed: cw = (int16)((hr * hc) >> 15); out = (int16)((x * cw) >> 15)
        const int cw = wrap16((hr * a.hamc[k]) >> 15);
        const int wr = wrap16((lo16(v) * cw) >> 15);
        const int wi = wrap16((hi16(v) * cw) >> 15);
        const int vv = (int)(__brev((unsigned)u) >> (32 - F::LE));
        xr[vv] = wr;
        xi[vv] = wi;
    }
    __syncthreads();                                // region A becomes the exchange buffer
    const int e_row = F::run(xr, xi, xbuf, tw, red, tid);
    uint32_t *out = a.y1 + (size_t)j * N;
#pragma unroll
    for (int v = 0; v < E; ++v) out[tid + T * v] = pack16(xr[v], xi[v]);
    if (tid == 0) {
        a.e1[j] = e_row;
        atomicMax(a.ctrl + 1, e_row);
    }
}

// ------------------------------------------------------------------------------------------ K3
struct Fft2Args {
    const uint32_t *y1;
    const int32_t *e1;
    const uint32_t *tw;
    uint32_t *y2;
    int32_t *e2, *ctrl;
    int n;
};

template <int L, int E>
__global__ void __launch_bounds__((1 << L) / E) k_fx_fft2(Fft2Args a) {
    using F = BfpFft<L, E>;
    constexpr int N = F::N, T = F::T;
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr size_t XB = ((size_t)4 * (N + N / 32) + 15) & ~(size_t)15;   // exchange buffer, 16-byte multiple
    uint32_t *xbuf = reinterpret_cast<uint32_t *>(smem);
    uint32_t *tw = reinterpret_cast<uint32_t *>(smem + XB);
    int(*red)[32] = reinterpret_cast<int(*)[32]>(smem + XB + 4 * (size_t)N);
    const int tid = threadIdx.x;
    const int k = blockIdx.x;                       // cross bin
    for (int c = tid; c < N / 4; c += T) cp_async16(tw + 4 * c, a.tw + 4 * c);
    cp_async_commit();
    const int emax1 = a.ctrl[1];
    int xr[E], xi[E];
#pragma unroll
    for (int u = 0; u < E; ++u) {
        const int jr = tid + T * u;                 // natural range index
        int r = 0, i = 0;
        if (jr < a.n) {
            const uint32_t v = __ldg(a.y1 + (size_t)jr * N + k);
            const int s = min(emax1 - __ldg(a.e1 + jr), 31);   // >= 0: the shifted int16 stays in range
            r = lo16(v) >> s;
            i = hi16(v) >> s;
        }
        const int vv = (int)(__brev((unsigned)u) >> (32 - F::LE));
        xr[vv] = r;
        xi[vv] = i;
    }
    cp_async_wait_all();
    __syncthreads();
    const int e_row = F::run(xr, xi, xbuf, tw, red, tid);
    uint32_t *out = a.y2 + (size_t)k * N;
#pragma unroll
    for (int v = 0; v < E; ++v) out[tid + T * v] = pack16(xr[v], xi[v]);
    if (tid == 0) {
        a.e2[k] = e_row;
        atomicMax(a.ctrl + 2, e_row);
    }
}

// ------------------------------------------------------------------------------------------ K4
// img[j][k] = floor(sqrt(re^2 + im^2)) of sat16(y2[k][j] >> (emax2 - e2[k])); 64 (k) x 128 (j) tiles,
// two adjacent columns per thread (8-byte loads), two adjacent k per thread on the transposed store.
__device__ __forceinline__ uint16_t detect_one(uint32_t v, int sh, int fused) {
    // emulator order: renormalise the pair, then |z|; fused (silicon) order: |z| of the row at its own
    // exponent, then the magnitude shifted (model_detect_fusion.order_B_fused)
    const int ps = fused ? 0 : sh;
    const int r = lo16(v) >> ps, i = hi16(v) >> ps;          // an arithmetic shift keeps int16 range
    const unsigned p = (unsigned)(r * r) + (unsigned)(i * i);
    // p <= 2^31 rounds to 24 bits in float and the hardware square-root approximation (sqrt.approx.f32,
    // relative error well below 2^-20) keeps the estimate within 0.05 of sqrt(p) <= 46341, so its
    // truncation is within one of floor(sqrt(p)): one exact integer correction each way makes q exact
    // (checked on the CPU around every perfect square of the range with a 2^-21 relative error)
    float est;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(est) : "f"((float)p));
    unsigned q = (unsigned)est;
    q -= (q * q > p) ? 1u : 0u;
    q += ((q + 1) * (q + 1) <= p) ? 1u : 0u;
    if (fused) q >>= sh;
    return (uint16_t)min(q, 65535u);
}

__global__ void __launch_bounds__(256) k_fx_detect(const uint32_t *__restrict__ y2, const int32_t *__restrict__ e2,
                                                   const int32_t *__restrict__ ctrl, uint16_t *__restrict__ img, int G,
                                                   int fused) {
    __shared__ uint16_t t[128][65];
    // k tiles in reverse: FFT-2 wrote its rows in increasing k just before, so the first tiles read the
    // rows most likely still in L2
    const int k0 = (gridDim.y - 1 - blockIdx.y) * 64, j0 = blockIdx.x * 128;
    const int emax2 = ctrl[2];
    const int tx = threadIdx.x & 63, ty = threadIdx.x >> 6;   // 64 column pairs x 4 rows
    // all 16 loads of this thread in flight before any arithmetic
    const bool live = j0 + 2 * tx < G;                        // G = 64: half a tile
    uint2 v[16];
    int s[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const int k = k0 + ty + 4 * u;
        v[u] = live ? __ldcs(reinterpret_cast<const uint2 *>(y2 + (size_t)k * G + j0) + tx) : make_uint2(0u, 0u);
        s[u] = __ldg(e2 + k);
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const int sh = min(emax2 - s[u], 31);
        t[2 * tx][ty + 4 * u] = detect_one(v[u].x, sh, fused);
        t[2 * tx + 1][ty + 4 * u] = detect_one(v[u].y, sh, fused);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll 4
    for (int jj = w; jj < 128; jj += 8) {
        if (j0 + jj >= G) break;
        const uint32_t pair = (uint32_t)t[jj][2 * lane] | ((uint32_t)t[jj][2 * lane + 1] << 16);
        reinterpret_cast<uint32_t *>(img + (size_t)(j0 + jj) * G + k0)[lane] = pair;
    }
}

// ------------------------------------------------------------------------------------------ launch
// Blocks of `fn` resident on the whole device at once (the L2 prefetch distance of the line kernels).
template <class K>
int resident_blocks(K fn, int threads, size_t smem) {
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem) != cudaSuccess) {
        (void)cudaGetLastError();           // no prefetch; leave no error behind for the launch check
        return 0;
    }
    return sms * per;
}

template <int L>
struct FixedLaunch {
    static constexpr int N = 1 << L;
    static constexpr int E = (N >= 512) ? 16 : (N / 32);
    static constexpr int T = N / E;
    // FFT-2 tile: 32 values per thread for lines of 8192 points and more (two shared-memory exchanges
    // instead of three, half the warps in each stage's row-max reduction; 0.60 -> 0.58 ms at 8192^2)
    static constexpr int E2 = (L >= 13) ? 32 : E;
    static constexpr int T2 = N / E2;

    static size_t pass2_smem(int m, bool sinc) {
        size_t regA = (size_t)32 * ((m + 3) >> 2);
        const size_t xb = (size_t)4 * (N + N / 32);
        if (xb > regA) regA = xb;
        regA = (regA + 15) & ~(size_t)15;
        return regA + 4 * (size_t)N + (sinc ? 2 * 256 * kSincTaps : 0) + 2 * 32 * 4;
    }
    static size_t fft2_smem() { return (((size_t)4 * (N + N / 32) + 15) & ~(size_t)15) + 4 * (size_t)N + 2 * 32 * 4; }

    static cudaError_t run(const FixedDev &d, const float *sig, const uint32_t *sig_iq, uint16_t *img,
                           cudaStream_t st, StageProf &pf) {
        cudaError_t e;
        // K0: Q0 block exponent
        if (sig) {
            const long long nf = 2LL * d.m * d.n;
            const long long n4 = nf / 4;
            const int ntail = (int)(nf - 4 * n4);
            k_q0max<<<148 * 8, 256, 0, st>>>(reinterpret_cast<const float4 *>(sig), n4, sig + 4 * n4, ntail,
                                             reinterpret_cast<uint32_t *>(d.ctrl));
            k_q0exp<<<1, 1, 0, st>>>(d.ctrl);
        }
        if ((e = pf.mark(st, "q0max")) != cudaSuccess) return e;
        // K1: pass 1
        Pass1Args p1{reinterpret_cast<const float2 *>(sig), sig_iq, d.f0, d.df, d.fac, d.krp, d.order, d.sinc,
                     d.ctrl, d.p1, d.m, d.n, d.mpad, d.range_cubic};
        dim3 g1((d.m + P1_SLOTS - 1) / P1_SLOTS, (d.n + P1_BINS - 1) / P1_BINS);
        if (d.range_sinc) {
            e = cudaFuncSetAttribute(k_fx_pass1<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p1_smem(true));
            if (e != cudaSuccess) return e;
            k_fx_pass1<true><<<g1, 256, p1_smem(true), st>>>(p1);
        } else {
            e = cudaFuncSetAttribute(k_fx_pass1<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p1_smem(false));
            if (e != cudaSuccess) return e;
            k_fx_pass1<false><<<g1, 256, p1_smem(false), st>>>(p1);
        }
        if ((e = pf.mark(st, "pass1")) != cudaSuccess) return e;
        // K2: pass 2 + window + FFT-1
        Pass2Args p2{d.p1, d.tan_s, d.krp, d.kcp, d.hamr, d.hamc, d.tw, d.sinc, d.y1, d.e1, d.ctrl, d.m, d.n, d.mpad,
                     d.az_cubic, 0};
        const size_t s2 = pass2_smem(d.m, d.az_sinc != 0);
        if (d.az_sinc) {
            e = cudaFuncSetAttribute(k_fx_pass2_fft<L, E, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s2);
            if (e != cudaSuccess) return e;
            p2.pf = resident_blocks(k_fx_pass2_fft<L, E, true>, T, s2);
            k_fx_pass2_fft<L, E, true><<<d.n, T, s2, st>>>(p2);
        } else {
            e = cudaFuncSetAttribute(k_fx_pass2_fft<L, E, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s2);
            if (e != cudaSuccess) return e;
            p2.pf = resident_blocks(k_fx_pass2_fft<L, E, false>, T, s2);
            k_fx_pass2_fft<L, E, false><<<d.n, T, s2, st>>>(p2);
        }
        if ((e = pf.mark(st, "pass2_win_fft1")) != cudaSuccess) return e;
        // K3: FFT-2 along range
        Fft2Args f2{d.y1, d.e1, d.tw, d.y2, d.e2, d.ctrl, d.n};
        const size_t s3 = fft2_smem();
        e = cudaFuncSetAttribute(k_fx_fft2<L, E2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s3);
        if (e != cudaSuccess) return e;
        k_fx_fft2<L, E2><<<N, T2, s3, st>>>(f2);
        if ((e = pf.mark(st, "fft2")) != cudaSuccess) return e;
        // K4: renorm + detect + transpose
        dim3 g4((N + 127) / 128, N / 64);
        k_fx_detect<<<g4, 256, 0, st>>>(d.y2, d.e2, d.ctrl, img, N, d.fused_detect);
        if ((e = pf.mark(st, "renorm_detect")) != cudaSuccess) return e;
        return cudaGetLastError();
    }
};

}  // namespace

cudaError_t fixed_form(const FixedDev &d, const float *sig_c64, const uint32_t *sig_iq, uint16_t *img,
                       cudaStream_t st, StageProf *prof) {
    StageProf none;
    StageProf &pf = prof ? *prof : none;
    pf.count = 0;
    cudaError_t e = pf.mark(st, "start");
    if (e != cudaSuccess) return e;
    // reset the reduction words: q0 max, emax1, emax2
    e = cudaMemsetAsync(d.ctrl, 0, 4 * sizeof(int32_t), st);
    if (e != cudaSuccess) return e;
    switch (d.L) {
        case 6: return FixedLaunch<6>::run(d, sig_c64, sig_iq, img, st, pf);
        case 7: return FixedLaunch<7>::run(d, sig_c64, sig_iq, img, st, pf);
        case 8: return FixedLaunch<8>::run(d, sig_c64, sig_iq, img, st, pf);
        case 9: return FixedLaunch<9>::run(d, sig_c64, sig_iq, img, st, pf);
        case 10: return FixedLaunch<10>::run(d, sig_c64, sig_iq, img, st, pf);
        case 11: return FixedLaunch<11>::run(d, sig_c64, sig_iq, img, st, pf);
        case 12: return FixedLaunch<12>::run(d, sig_c64, sig_iq, img, st, pf);
        case 13: return FixedLaunch<13>::run(d, sig_c64, sig_iq, img, st, pf);
        case 14: return FixedLaunch<14>::run(d, sig_c64, sig_iq, img, st, pf);
        default: return cudaErrorInvalidValue;
    }
}

size_t fixed_workspace_bytes(int m, int n, int G) {
    const int mpad = (m + 31) / 32 * 32;
    return (size_t)4 * n * mpad + (size_t)4 * n * G + (size_t)4 * G * G + 8 * (size_t)G + 64;
}

}  // namespace pfa
