// Register Stockham FFT (FP32 complex) for one N-point line per thread block.
//
// T = N / E threads, each holding E complex values.  The transform runs as Stockham autosort passes
// of radix R (the first pass radix E, then E, then the remainder), pass p with Ns = product of the
// earlier radices:
//     j = tid + T q  (q < E / R),   k = j mod Ns
//     v[r] = in[j + r N / R] * W_{Ns R}^{r k}          (one table twiddle per element and pass)
//     v    = DFT_R(v)                                  (constant twiddles, in registers)
//     out[(j / Ns) Ns R + k + r Ns] = v[r]
// so the result is in natural order and the last pass writes element (q, r) to index tid + T (q + r E/R):
// callers store x[v] at frequency index tid + T v.  Pass 0 reads its operands straight from registers:
// callers load x[u] with natural input index tid + T u.  Passes exchange through a padded shared buffer
// of N + N/16 elements (N + N/32 for E = 32; index i stored at i + i/16, resp. i + i/32: the pass-0
// scatter with stride R is conflict free).
// The twiddle table holds W_N^k = exp(-2 pi i k / N) for k < N.  The inverse transform is
// conj(FFT(conj(x))) without scaling (callers conjugate on load and store).
#pragma once

#include <cuda_runtime.h>

namespace pfa {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// multiply by -i (forward W_4)
__device__ __forceinline__ float2 cmul_mi(float2 a) { return make_float2(a.y, -a.x); }

// exp(-2 pi i e / 16) for e = 0..15, from the exact values of cos and sin at multiples of pi/8
__device__ __forceinline__ float2 w16(int e) {
    constexpr float c1 = 0.92387953251128674f, s1 = 0.38268343236508978f, h = 0.70710678118654752f;
    switch (e & 15) {
        case 0: return make_float2(1.f, 0.f);
        case 1: return make_float2(c1, -s1);
        case 2: return make_float2(h, -h);
        case 3: return make_float2(s1, -c1);
        case 4: return make_float2(0.f, -1.f);
        case 5: return make_float2(-s1, -c1);
        case 6: return make_float2(-h, -h);
        case 7: return make_float2(-c1, -s1);
        case 8: return make_float2(-1.f, 0.f);
        case 9: return make_float2(-c1, s1);
        case 10: return make_float2(-h, h);
        case 11: return make_float2(-s1, c1);
        case 12: return make_float2(0.f, 1.f);
        case 13: return make_float2(s1, c1);
        case 14: return make_float2(h, h);
        default: return make_float2(c1, s1);
    }
}

// exp(-2 pi i e / 32) = cos(e pi / 16) - i sin(e pi / 16) for e = 0..31, from the cosines of the multiples
// of pi/16 in [0, pi/2] (sin(k pi/16) = cos((8 - k) pi/16)) and the quadrant of e
__device__ __forceinline__ float2 w32(int e) {
    constexpr float c[9] = {1.f, 0.98078528040323044913f, 0.92387953251128675613f, 0.83146961230254523708f,
                            0.70710678118654752440f, 0.55557023301960222474f, 0.38268343236508977173f,
                            0.19509032201612826785f, 0.f};
    e &= 31;
    const int k = e & 7;
    const float ck = c[k], sk = c[8 - k];
    float cs, sn;                                   // cos and sin of e pi / 16
    switch (e >> 3) {
        case 0: cs = ck; sn = sk; break;
        case 1: cs = -sk; sn = ck; break;
        case 2: cs = -ck; sn = -sk; break;
        default: cs = sk; sn = -ck; break;
    }
    return make_float2(cs, -sn);
}

// W_R^e for the radices used here (R divides 32)
template <int R>
__device__ __forceinline__ float2 wr(int e) {
    if constexpr (R == 32) return w32(e);
    else return w16(e * (16 / R));
}

// In-place DFT of size R on v (natural-order output), forward sign.
template <int R>
struct Dft;

template <>
struct Dft<1> {
    __device__ static __forceinline__ void run(float2 (&)[1]) {}
};

template <>
struct Dft<2> {
    __device__ static __forceinline__ void run(float2 (&v)[2]) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <>
struct Dft<4> {
    __device__ static __forceinline__ void run(float2 (&v)[4]) {
        const float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        const float2 s13 = cadd(v[1], v[3]), d13 = cmul_mi(csub(v[1], v[3]));
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        v[1] = cadd(d02, d13);
        v[3] = csub(d02, d13);
    }
};

// R = P * Q with X[Q k1 + k2] = sum_{n1} W_R^{n1 k2} W_P^{n1 k1} sum_{n2} x[n1 + P n2] W_Q^{n2 k2}
template <int R, int P, int Q>
__device__ __forceinline__ void dft_split(float2 (&v)[R]) {
    float2 y[P][Q];
#pragma unroll
    for (int n1 = 0; n1 < P; ++n1) {
        float2 t[Q];
#pragma unroll
        for (int n2 = 0; n2 < Q; ++n2) t[n2] = v[n1 + P * n2];
        Dft<Q>::run(t);
#pragma unroll
        for (int k2 = 0; k2 < Q; ++k2) y[n1][k2] = (n1 * k2 == 0) ? t[k2] : cmul(t[k2], wr<R>(n1 * k2));
    }
#pragma unroll
    for (int k2 = 0; k2 < Q; ++k2) {
        float2 t[P];
#pragma unroll
        for (int n1 = 0; n1 < P; ++n1) t[n1] = y[n1][k2];
        Dft<P>::run(t);
#pragma unroll
        for (int k1 = 0; k1 < P; ++k1) v[Q * k1 + k2] = t[k1];
    }
}

template <>
struct Dft<8> {
    __device__ static __forceinline__ void run(float2 (&v)[8]) { dft_split<8, 2, 4>(v); }
};

template <>
struct Dft<16> {
    __device__ static __forceinline__ void run(float2 (&v)[16]) { dft_split<16, 4, 4>(v); }
};

template <>
struct Dft<32> {
    __device__ static __forceinline__ void run(float2 (&v)[32]) { dft_split<32, 4, 8>(v); }
};

template <int L, int E>
struct StockhamFft {
    static constexpr int N = 1 << L;
    static constexpr int T = N / E;
    static_assert(T >= 32, "at least one warp per line");
    // one pad element per PADW: the pass-0 scatter (stride R = E) stays free of bank conflicts
    static constexpr int PADW = E >= 32 ? 32 : 16;
    static constexpr int xbuf_elems() { return N + N / PADW; }
    __device__ static __forceinline__ int pad(int i) { return i + i / PADW; }

    // radix of pass p: E while the remaining size allows, then the remainder
    static constexpr int radix(int p) {
        int rem = N, r = E;
        for (int i = 0; i <= p; ++i) {
            r = rem >= E ? E : rem;
            rem /= r;
        }
        return r;
    }
    static constexpr int npass() {
        int rem = N, c = 0;
        while (rem > 1) {
            rem /= (rem >= E ? E : rem);
            ++c;
        }
        return c;
    }
    static constexpr int ns(int p) {
        int s = 1;
        for (int i = 0; i < p; ++i) s *= radix(i);
        return s;
    }

    template <int P>
    __device__ static __forceinline__ void pass(float2 (&x)[E], float2 *buf, const float2 *__restrict__ tw, int tid) {
        constexpr int R = radix(P);
        constexpr int G = E / R;
        constexpr int NS = ns(P);
        constexpr bool LAST = (P == npass() - 1);
        float2 v[G][R];
        if (P == 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[0][r] = x[r];
        } else {
            __syncthreads();   // the previous pass's stores are visible
#pragma unroll
            for (int q = 0; q < G; ++q)
#pragma unroll
                for (int r = 0; r < R; ++r) v[q][r] = buf[pad(tid + T * q + r * (N / R))];
        }
#pragma unroll
        for (int q = 0; q < G; ++q) {
            const int j = tid + T * q;
            const int k = j % NS;
            if (P > 0) {
                // W^{r k} for r < R from the table entries W^{k}, W^{4k}, W^{8k}, W^{12k}: every factor is
                // at most three complex products deep (error of a few ulp)
                constexpr int S = N / (NS * R);
                if constexpr (R <= 4) {
#pragma unroll
                    for (int r = 1; r < R; ++r) v[q][r] = cmul(v[q][r], __ldg(tw + r * k * S));
                } else {
                    float2 lo[4], hi[R / 4];
                    lo[0] = make_float2(1.f, 0.f);
                    lo[1] = __ldg(tw + k * S);
                    lo[2] = cmul(lo[1], lo[1]);
                    lo[3] = cmul(lo[2], lo[1]);
                    hi[0] = make_float2(1.f, 0.f);
#pragma unroll
                    for (int h = 1; h < R / 4; ++h) hi[h] = __ldg(tw + 4 * h * k * S);
#pragma unroll
                    for (int r = 1; r < R; ++r) {
                        const float2 w = (r & 3) == 0 ? hi[r >> 2] : ((r >> 2) == 0 ? lo[r & 3] : cmul(hi[r >> 2], lo[r & 3]));
                        v[q][r] = cmul(v[q][r], w);
                    }
                }
            }
            Dft<R>::run(v[q]);
        }
        if (LAST) {
#pragma unroll
            for (int q = 0; q < G; ++q)
#pragma unroll
                for (int r = 0; r < R; ++r) x[q + r * G] = v[q][r];
        } else {
            __syncthreads();   // every thread has read its operands of this pass
#pragma unroll
            for (int q = 0; q < G; ++q) {
                const int j = tid + T * q;
                const int k = j % NS;
                const int base = (j / NS) * NS * R + k;
#pragma unroll
                for (int r = 0; r < R; ++r) buf[pad(base + r * NS)] = v[q][r];
            }
        }
    }

    template <int P>
    __device__ static __forceinline__ void passes(float2 (&x)[E], float2 *buf, const float2 *tw, int tid) {
        if constexpr (P < npass()) {
            pass<P>(x, buf, tw, tid);
            passes<P + 1>(x, buf, tw, tid);
        }
    }

    // x[u] = input at natural index tid + T u  ->  x[v] = output at frequency index tid + T v.
    // `buf` may alias memory the caller read before the call: the first exchange begins with a barrier.
    __device__ static __forceinline__ void run(float2 (&x)[E], float2 *buf, const float2 *__restrict__ tw, int tid) {
        passes<0>(x, buf, tw, tid);
    }
};

}  // namespace pfa
