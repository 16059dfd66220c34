// Float resampling helpers shared by the FP32 and the split-precision kernels: np.interp brackets with
// the reference's exact end-point semantics (src/form_image_pfa.py:165-222), the FP32 lerp / float sinc
// gather, and cp.async row staging.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

namespace pfa {
namespace {

// ------------------------------------------------------------------------------------------ async copies
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem_dst, const void *gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
// all but the N most recent groups of this thread have landed
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Bulk prefetch of `bytes` (16-byte aligned address, size a multiple of 16) into L2, 16 KB per instruction,
// issued by the first threads of the block: a line kernel prefetches the line of the block that will start
// when this one ends, so that block's loads find it in L2.
__device__ __forceinline__ void l2_prefetch(const void *p, size_t bytes, int tid) {
    constexpr size_t CH = 16384;
    const size_t off = (size_t)tid * CH;
    if (off < bytes) {
        const uint32_t sz = (uint32_t)(bytes - off < CH ? bytes - off : CH);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(static_cast<const char *>(p) + off), "r"(sz)
                     : "memory");
    }
}

// ------------------------------------------------------------------------------------------ brackets
// np.interp bracket on an ascending accessor xa(0..n-1): returns j with xa(j) <= x < xa(j+1) and the
// fraction, or -1 when x is outside [xa(0), xa(n-1)]; x == xa(n-1) gives j = n-2, frac = 1.
struct Frac {
    float f;     // fraction toward the upper natural-order sample (lerp weight)
    int ph;      // sinc phase round(frac * 32768) >> 7, taken from the float64 ascending fraction
    int rev;     // descending source axis: taps run in reverse natural order
};

// phase of the float sinc from a float64 fraction (same rounding as the oracle's np.round)
__device__ __forceinline__ int sinc_phase(double fd) {
    return (int)fmin(fmax(rint(fd * 32768.0), 0.0), 32767.0) >> 7;
}

// Fraction of x in [a, b].  EXACT: float64 fraction (the sinc phase depends on it); else a float32 division.
template <bool EXACT>
__device__ __forceinline__ void make_frac(double x, double a, double b, Frac &frac) {
    if (EXACT) {
        const double fd = __ddiv_rn(__dsub_rn(x, a), __dsub_rn(b, a));
        frac.f = (float)fd;
        frac.ph = sinc_phase(fd);
    } else {
        frac.f = __fdiv_rn((float)(x - a), (float)(b - a));
        frac.ph = 0;
    }
    frac.rev = 0;
}

// Walks from the guess carrying both end values (two loads when the guess is right); bisection after a
// few steps.
template <bool EXACT, class F>
__device__ __forceinline__ int interp_bracket(const F &xa, int n, double x0, double x1, double x, int guess, Frac &frac) {
    if (!(x >= x0) || !(x <= x1)) return -1;
    // largest j in [0, n-2] with xa(j) <= x  (xa(0) = x0 <= x <= x1 = xa(n-1))
    int j = min(max(guess, 0), n - 2);
    double a = xa(j), b = xa(j + 1);
    int steps = 0;
    while (b <= x && j < n - 2) {
        if (++steps > 8) {
            int lo = j + 1, hi = n - 2;      // xa(j+1) <= x
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (xa(mid) <= x) lo = mid; else hi = mid - 1;
            }
            j = lo;
            a = xa(j);
            b = xa(j + 1);
            break;
        }
        ++j;
        a = b;
        b = xa(j + 1);
    }
    while (a > x && j > 0) {
        if (++steps > 16) {
            int lo = 0, hi = j - 1;          // xa(0) <= x < xa(j)
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (xa(mid) <= x) lo = mid; else hi = mid - 1;
            }
            j = lo;
            a = xa(j);
            b = xa(j + 1);
            break;
        }
        --j;
        b = a;
        a = xa(j);
    }
    make_frac<EXACT>(x, a, b, frac);
    return j;
}

// The same bracket for CH queries at once: the source values at guess - 1 .. guess + 2 are loaded for every
// query before any is tested, so the loads of the CH queries overlap and a guess that is off by one (the
// common miss of the affine guess on a tan(phi) axis) resolves without another round trip; a query that
// misses by more walks from the guess.
template <bool EXACT, int CH, class F>
__device__ __forceinline__ void interp_brackets(const F &xa, int n, double x0, double x1, double inv_span,
                                                const double (&x)[CH], const bool (&valid)[CH], int (&j)[CH],
                                                Frac (&frac)[CH]) {
    int g[CH];
    double v0[CH], v1[CH], v2[CH], v3[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        g[c] = (valid[c] && isfinite(inv_span)) ? min(max((int)((x[c] - x0) * inv_span), 0), n - 2) : 0;
        v0[c] = xa(max(g[c] - 1, 0));
        v1[c] = xa(g[c]);
        v2[c] = xa(g[c] + 1);
        v3[c] = xa(min(g[c] + 2, n - 1));
    }
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        j[c] = -1;
        frac[c] = Frac{0.f, 0, 0};
        if (!valid[c] || !(x[c] >= x0) || !(x[c] <= x1)) continue;
        // j is the unique index in [0, n-2] with xa(j) <= x < xa(j+1) (x == xa(n-1) takes j = n-2)
        const int gc = g[c];
        if (v1[c] <= x[c] && (x[c] < v2[c] || gc == n - 2)) {
            j[c] = gc;
            make_frac<EXACT>(x[c], v1[c], v2[c], frac[c]);
        } else if (gc + 1 <= n - 2 && v2[c] <= x[c] && (x[c] < v3[c] || gc + 1 == n - 2)) {
            j[c] = gc + 1;
            make_frac<EXACT>(x[c], v2[c], v3[c], frac[c]);
        } else if (gc >= 1 && v0[c] <= x[c] && x[c] < v1[c]) {
            j[c] = gc - 1;
            make_frac<EXACT>(x[c], v0[c], v1[c], frac[c]);
        } else {
            j[c] = interp_bracket<EXACT>(xa, n, x0, x1, x[c], gc, frac[c]);
        }
    }
}

// the same bracket seen from the descending side: lower natural index n-2-j, weights mirrored
__device__ __forceinline__ void mirror_frac(Frac &fr) {
    fr.f = 1.0f - fr.f;
    fr.rev = 1;
}

// Float sinc table: the Q15 taps as int16, 256 phases x 32 taps, one phase per row of kTabRow int16 (taps
// 0..31, then padding).  A lane reads its phase's taps eight at a time (four 16-byte loads; half the
// shared-memory wavefronts of a float table, whose random-phase loads conflict the same way).
constexpr int kTabRow = 40;
constexpr int kTabShorts = 256 * kTabRow;

// exact float of a sign-extended int16 without the conversion unit: the bit pattern of 1.5 * 2^23 plus
// v is the float 1.5 * 2^23 + v for |v| < 2^22
__device__ __forceinline__ float s16f(int v) { return __int_as_float(0x4B400000 + v) - 12582912.0f; }

// lerp or float sinc of complex64 samples `src` (indexed from `base`) at bracket (j, frac).  The sinc sums
// the taps in natural order (t = 0..31) with fused multiply-adds on the integer tap values and scales the
// sums by 2^-15 at the end: every partial sum is exactly 2^15 times the one a table of tap / 32768 gives
// (scaling by a power of two commutes with rounding), so the result is the same float.
template <bool SINC>
__device__ __forceinline__ float2 gather_f32(const float2 *src, int base, int sn, int j, Frac fr,
                                             const int16_t *tab) {
    if (j < 0) return make_float2(0.f, 0.f);
    const float frac = fr.f;
    if (SINC && j >= 15 && j <= sn - 17) {
        const uint4 *c4 = reinterpret_cast<const uint4 *>(tab + fr.ph * kTabRow);
        const float2 *x = src + (j - 15 - base);
        float ar = 0.f, ai = 0.f;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            // taps 8g .. 8g+7 of group g (tap 2k in the low half of word k); descending axis: tap 31 - t
            // at sample t, so sample group q takes tap group 3 - q in reverse
            const uint4 u = c4[fr.rev ? 3 - q : q];
            const uint32_t wd[4] = {u.x, u.y, u.z, u.w};
            float c[8];
#pragma unroll
            for (int e = 0; e < 8; ++e)
                c[e] = s16f((e & 1) ? ((int)wd[e >> 1] >> 16) : ((int)(wd[e >> 1] << 16) >> 16));
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const float ce = fr.rev ? c[7 - e] : c[e];
                ar = fmaf(ce, x[8 * q + e].x, ar);
                ai = fmaf(ce, x[8 * q + e].y, ai);
            }
        }
        return make_float2(ar * (1.0f / 32768.0f), ai * (1.0f / 32768.0f));
    }
    const float2 a = src[j - base], b = src[j + 1 - base];
    return make_float2(fmaf(frac, b.x - a.x, a.x), fmaf(frac, b.y - a.y, a.y));
}

}  // namespace
}  // namespace pfa
