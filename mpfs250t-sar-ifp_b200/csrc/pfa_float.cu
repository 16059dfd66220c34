// Float PFA datapath on sm_100a: the drop-in for form_image_pfa.pfa + detection
// (src/form_image_pfa.py:165-246, mpfs/host/accel.py:39-44).
//
//   k_fl_pass1      per pulse: FP64 source wavenumbers kr = (2 freq / c) pr, np.interp bracket
//                   (xp[j] <= x < xp[j+1], zero outside [xp0, xp_last]), FP32 lerp (or the float sinc
//                   variant); 32-slot x 128-bin shared tile -> range-bin rows of tan(phi)-sorted pulses
//   k_fl_pass2_fft  per range bin j: source KR[j] * tan_s (FP64), bracket, gather, float32 Hamming
//                   product window, (-1)^(j+k) centring modulation, FP32 FFT along cross (length m2)
//   k_fl_fft2       per cross bin: FP32 FFT along range (length n2, rows j >= n are the zero pad),
//                   fused detection store (|z|, |z|^2 or complex with the (-1)^(u+v) centring sign)
//
// Centring: fftshift(fft(ifftshift(x)))[v] = (-1)^v fft((-1)^a x[a])[v] for even N with N/2 even, so the
// shifts of form_image_pfa.transform2d (:144-147) cost one sign flip on load and one on store.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "fft_f32.cuh"
#include "interp_f32.cuh"
#include "pfa_internal.h"
#include "tc_sm100.cuh"
#include "tma_sm100.cuh"

namespace pfa {
const int16_t *builtin_sinc_table();

namespace {

constexpr double kC = 299792458.0;

// FFT: register Stockham radix-16 (fft_f32.cuh).
template <int L, int E>
using F32Fft = StockhamFft<L, E>;

// resident CTAs per SM the line kernels are compiled for: 64 registers a thread for tiles of up to 16
// values, 128 for the 32-value tile (its radix-32 passes hold 64 floats of data)
constexpr int fl_min_ctas(int L, int E) {
    return E >= 32 ? (((1 << L) / E >= 512) ? 1 : 2) : (((1 << L) / E >= 1024) ? 1 : (((1 << L) / E >= 512) ? 2 : 4));
}

// ------------------------------------------------------------------------------------------ K1f
// Each warp owns a double-buffered window of its pulse's samples: the window of the next pulse streams
// in (cp.async) while the current one is gathered.  The KR grid lies inside every pulse's own span, so
// F1_BINS consecutive bins cover at most F1_BINS + 1 source intervals; a wider window (not produced by
// prepare_tables) falls back to gathering from global memory.
constexpr int F1_SLOTS = 32, F1_WARPS = 8, F1_WMAX = 144;
// range bins per CTA: the sinc variant takes a narrower tile so three CTAs (with the 20 KB table) fit an SM
constexpr int f1_bins(bool sinc) { return sinc ? 64 : 128; }

struct FPass1Args {
    const float2 *sig;
    const double *f0, *df, *flast, *pr, *kr_grid;
    const int32_t *order;
    const int16_t *tabq;
    const float *theta;     // per-pulse phase correction exp(-j theta_i) (autofocus), or nullptr
    float2 *p1;
    int m, n, mpad;
};

// per-slot pulse constants, computed once per CTA
struct F1Pulse {
    double f0, df, sc, kfirst, klast, inv_dk;
    float2 rot;
    int i;          // source pulse, -1 for a slot past the last pulse
    int asc;
};

constexpr size_t f1_smem(bool sinc) {
    return (size_t)f1_bins(sinc) * (F1_SLOTS + 1) * 8 + (size_t)F1_WARPS * 2 * F1_WMAX * 8 + (sinc ? kTabShorts * 2 : 0);
}

template <bool SINC>
__global__ void __launch_bounds__(256, SINC ? 3 : 4) k_fl_pass1(FPass1Args a) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int F1_BINS = f1_bins(SINC), TB = F1_BINS / 32, SPW = F1_SLOTS / F1_WARPS;
    constexpr size_t TILE_BYTES = (size_t)F1_BINS * (F1_SLOTS + 1) * 8;
    float2(*tile)[F1_SLOTS + 1] = reinterpret_cast<float2(*)[F1_SLOTS + 1]>(smem);
    float2(*win)[2][F1_WMAX] = reinterpret_cast<float2(*)[2][F1_WMAX]>(smem + TILE_BYTES);
    int16_t *tab = reinterpret_cast<int16_t *>(smem + TILE_BYTES + (size_t)F1_WARPS * 2 * F1_WMAX * 8);
    __shared__ F1Pulse prm[F1_SLOTS];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = blockIdx.x * F1_SLOTS, j0 = blockIdx.y * F1_BINS;
    const int n = a.n;
    if (SINC) {
        const uint4 *src = reinterpret_cast<const uint4 *>(a.tabq);
        uint4 *dst = reinterpret_cast<uint4 *>(tab);
#pragma unroll
        for (int i = 0; i < kTabShorts / 8 / 256; ++i) dst[tid + 256 * i] = __ldg(src + tid + 256 * i);
    }
    if (tid < F1_SLOTS) {
        F1Pulse p{};
        p.i = -1;
        p.rot = make_float2(1.f, 0.f);
        const int r = r0 + tid;
        if (r < a.m) {
            const int i = a.order[r];
            const double f0 = a.f0[i], df = a.df[i], pri = a.pr[i];
            p.i = i;
            p.f0 = f0;
            p.df = df;
            p.sc = 2.0 * pri / kC;
            // kr[i, k] = (2 freq[i, k] / c) pr[i] (form_image_pfa.py:176-187).  The end points are evaluated
            // with the reference's exact IEEE operations (KR's first and last samples coincide with some
            // pulse's end points, where np.interp returns the end sample); interior samples use the affine
            // model freq = f0 + k df.
            p.kfirst = __dmul_rn(__ddiv_rn(__dmul_rn(2.0, f0), kC), pri);
            p.klast = __dmul_rn(__ddiv_rn(__dmul_rn(2.0, a.flast[i]), kC), pri);
            p.inv_dk = 1.0 / fabs(p.sc * df);               // the source axis is affine in the sample index
            // the phase correction commutes with the (linear, per-pulse) interpolation: rotate the output
            if (a.theta) {
                float sn, cs;
                sincosf(a.theta[i], &sn, &cs);
                p.rot = make_float2(cs, -sn);
            }
        }
        prm[tid] = p;
    }
    // the query wavenumbers of this CTA's bins are the same for every pulse
    double q[TB];
#pragma unroll
    for (int t = 0; t < TB; ++t) {
        const int j = j0 + lane + 32 * t;
        q[t] = j < n ? a.kr_grid[j] : 0.0;
    }
    __syncthreads();

    // start the copy of a window (every lane commits one group per slot, possibly empty)
    auto fetch = [&](const F1Pulse &p, int wlo, int whi, float2 *w) {
        if (p.i >= 0 && whi - wlo <= F1_WMAX) {
            const float2 *row = a.sig + (size_t)p.i * n;
            for (int k = wlo + lane; k < whi; k += 32) cp_async8(w + (k - wlo), row + k);
        }
        cp_async_commit();
    };

    // iteration s brackets slot s and starts its window, then gathers slot s - 1 while that copy flies
    int jj[TB], jn[TB];
    Frac fr[TB], fn[TB];
    int wlo = 0, whi = 0, wlo_n = 0, whi_n = 0;
#pragma unroll
    for (int s = 0; s <= SPW; ++s) {
        if (s < SPW) {
            // np.interp bracket of this warp's bins on pulse pn, and the sample window [wlo, whi) they read
            const F1Pulse &pn = prm[warp + F1_WARPS * s];
            wlo_n = whi_n = 0;
            if (pn.i >= 0) {
                auto kr = [&](int k) {
                    return k == 0 ? pn.kfirst : (k == n - 1 ? pn.klast : pn.sc * (pn.f0 + (double)k * pn.df));
                };
                const bool asc = kr(n - 1) >= kr(0);
                auto xa = [&](int t) { return asc ? kr(t) : kr(n - 1 - t); };
                const double xa0 = xa(0), xa1 = xa(n - 1);
                const bool fin = isfinite(pn.inv_dk);
                // xa(ja) for ja in [0, n-2]: xa0 at ja = 0 (the exact end point), the affine model inside
                auto xa_lo = [&](int ja) {
                    return ja == 0 ? xa0 : pn.sc * (pn.f0 + (double)(asc ? ja : n - 1 - ja) * pn.df);
                };
                int lo_i = 1 << 30, hi_i = -1;
#pragma unroll
                for (int t = 0; t < TB; ++t) {
                    jn[t] = -1;
                    fn[t] = Frac{0.f, 0, 0};
                    if (j0 + lane + 32 * t < n && q[t] >= xa0 && q[t] <= xa1) {
                        // closed-form bracket on the affine axis; the end points are exact
                        const double pos = (q[t] - xa0) * pn.inv_dk;
                        const int ja = fin ? min(max((int)floor(pos), 0), n - 2) : 0;
                        const double fd = (q[t] - xa_lo(ja)) * pn.inv_dk;
                        fn[t].f = (float)fd;
                        fn[t].ph = sinc_phase(fd);
                        // natural-order index of the lower sample and the weight toward the upper one
                        int lowi;
                        if (asc) { lowi = ja; } else { lowi = n - 2 - ja; mirror_frac(fn[t]); }
                        jn[t] = lowi;
                        lo_i = min(lo_i, lowi);
                        hi_i = max(hi_i, lowi);
                    }
                }
                lo_i = __reduce_min_sync(0xffffffffu, lo_i);
                hi_i = __reduce_max_sync(0xffffffffu, hi_i);
                if (hi_i >= 0) {
                    wlo_n = max(0, lo_i - (SINC ? 15 : 0));
                    whi_n = min(n, hi_i + (SINC ? 17 : 2));
                }
            } else {
#pragma unroll
                for (int t = 0; t < TB; ++t) jn[t] = -1;
            }
            fetch(pn, wlo_n, whi_n, win[warp][s & 1]);
        }
        if (s > 0) {
            if (s < SPW) cp_async_wait_group<1>(); else cp_async_wait_group<0>();
            __syncwarp();
            const int slot = warp + F1_WARPS * (s - 1);
            const F1Pulse &p = prm[slot];
            if (p.i < 0) {
#pragma unroll
                for (int t = 0; t < TB; ++t) tile[lane + 32 * t][slot] = make_float2(0.f, 0.f);
            } else {
                const bool fits = whi - wlo <= F1_WMAX;
                const float2 *w = win[warp][(s - 1) & 1];
                const float2 *row = a.sig + (size_t)p.i * n;
#pragma unroll
                for (int t = 0; t < TB; ++t) {
                    const int jb = lane + 32 * t;
                    float2 out = make_float2(0.f, 0.f);
                    if (jj[t] >= 0)
                        out = fits ? gather_f32<SINC>(w, wlo, n, jj[t], fr[t], tab)
                                   : gather_f32<SINC>(row, 0, n, jj[t], fr[t], tab);
                    tile[jb][slot] = a.theta ? cmul(out, p.rot) : out;
                }
            }
            __syncwarp();
        }
#pragma unroll
        for (int t = 0; t < TB; ++t) {
            jj[t] = jn[t];
            fr[t] = fn[t];
        }
        wlo = wlo_n;
        whi = whi_n;
    }
    __syncthreads();
    // two slots per lane, two bins per warp store (mpad is a multiple of 32: every slot of the CTA exists)
    const int half = lane >> 4, l2 = 2 * (lane & 15);
    for (int jb = 2 * warp + half; jb < F1_BINS; jb += 2 * F1_WARPS) {
        const int j = j0 + jb;
        if (j >= n) break;
        const float2 u0 = tile[jb][l2], u1 = tile[jb][l2 + 1];
        *reinterpret_cast<float4 *>(a.p1 + (size_t)j * a.mpad + r0 + l2) = make_float4(u0.x, u0.y, u1.x, u1.y);
    }
}

// packed pass-2 bracket (written by the forward pass 2 of an autofocus gradient for the adjoint), on the
// ascending view of the pass-2 sources: bit 31 = outside the span, bits 17..30 = lower index ja, bits 0..16 =
// the lerp weight toward ja + 1 (x 131071) or, for an interior bracket of the float sinc (15 <= ja <= m-17,
// where no lerp weight is needed), the sinc phase
__device__ __forceinline__ uint32_t pack_br(int dead, int lowi, float f) {
    const uint32_t q = (uint32_t)fminf(fmaxf(rintf(f * 131071.f), 0.f), 131071.f);
    return ((uint32_t)dead << 31) | ((uint32_t)lowi << 17) | q;
}
__device__ __forceinline__ uint32_t pack_br_phase(int lowi, int ph) { return ((uint32_t)lowi << 17) | (uint32_t)ph; }
__device__ __forceinline__ int br_low(uint32_t p) { return (int)((p >> 17) & 0x3fffu); }

// ------------------------------------------------------------------------------------------ K2f
struct FPass2Args {
    CUtensorMap p1_map;   // TMA map of the pass-1 output rows (boxes of 256 samples)
    const double *tan_s, *kr_grid, *kc_grid, *ham_m, *ham_n;
    const int16_t *tabq;
    const float2 *tw;
    float2 *y1t;          // [m2][npad] cross-FFT output, transposed: row = cross bin, col = range bin
    uint32_t *pk_out;     // packed brackets [j][k] for the autofocus adjoint, or nullptr
    float2 *rp_out;       // float sinc, autofocus forward: R2 p1 [j][k] before the window (the adjoint's
                          // W^2 R2 p1 term), or nullptr
    int *err;             // set when the row load's bounded wait runs out
    int m, n, mpad, npad, centred, window, inverse;
    int probe;            // test hook: > 0 = first wait this many polls on a barrier nothing arrives on
    double *ysum;         // PK (autofocus forward): += sum |y1|^2 over the frame (S / n2, by Parseval)
};

// Polls of the pass-2 row-load wait (each try_wait may suspend for a while): a TMA row load lands in
// microseconds, so running out means the copy is lost; the frame is then flagged, not waited for.
constexpr uint32_t kRowWaitPolls = 1u << 22;

// Shared-memory bytes of pass 2's region A: the row as whole 256-sample boxes, or the FFT exchange buffer.
__host__ __device__ constexpr size_t pass2_region_a(int m, size_t xbuf_elems) {
    return ((size_t)2048 * ((m + 255) / 256) > (size_t)8 * xbuf_elems ? (size_t)2048 * ((m + 255) / 256)
                                                                       : (size_t)8 * xbuf_elems);
}

// Corner turn #2 fused into the cross FFT: a cluster of kCT CTAs holds kCT adjacent range bins; after
// their FFTs each CTA writes a 1/kCT slice of cross bins for all kCT rows (kCT * 8-byte runs) into the
// transposed buffer, reading the other rows from the cluster's distributed shared memory.  Four CTAs:
// a run fills one 32-byte sector, and 4-CTA clusters pack a GPC's SMs more fully than 8-CTA ones
// (pass 2 at 8192^2: 0.87 ms with 4, 0.95 with 2, 0.99 with 8).
constexpr int kCT = 4;
static_assert(8 % kCT == 0, "npad (a multiple of 8) must hold whole clusters");

// PK: also store the packed brackets for the autofocus adjoint (lerp only; a separate instantiation so
// that the frame's pass 2 carries no extra register pressure)
template <int L, int E, bool SINC, bool PK = false>
__global__ void __cluster_dims__(kCT, 1, 1) __launch_bounds__((1 << L) / E, fl_min_ctas(L, E))
k_fl_pass2_fft(const __grid_constant__ FPass2Args a) {
    using F = F32Fft<L, E>;
    constexpr int N = F::N, T = F::T;
    extern __shared__ __align__(1024) unsigned char smem[];
    // layout: [region A: the row (whole TMA boxes) | exchange buffer] [sinc table] [row mbarrier, probe]
    // [PK: T / 32 doubles of the |y1|^2 reduction].  No static shared memory: region A starts the window.
    const int m = a.m;
    const size_t regA = pass2_region_a(m, F::xbuf_elems());
    float2 *row = reinterpret_cast<float2 *>(smem);
    float2 *xbuf = reinterpret_cast<float2 *>(smem);
    int16_t *tab = reinterpret_cast<int16_t *>(smem + regA);
    uint64_t *row_bar = reinterpret_cast<uint64_t *>(smem + regA + (SINC ? 2 * kTabShorts : 0));
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int tid = threadIdx.x;
    // clusters in reverse range-bin order (a cluster's CTAs stay adjacent, rank order kept): pass 1 wrote
    // the high range-bin rows of p1 last, so the first clusters find their rows in L2
    const int j = (int)(gridDim.x - kCT - (blockIdx.x & ~(kCT - 1)) + (blockIdx.x & (kCT - 1)));
    const bool live = j < a.n;                 // grid is padded to a multiple of the cluster size
    float2 x[E];
    bool landed = true, issued = false;
    if (live) {
    // The row (256-sample boxes of the p1 tensor map) and the sinc table stream into shared memory by TMA
    // while the brackets are computed; warp 0 issues the copies.
    issued = (tma::saddr(row) & 127) == 0;          // CTA-uniform; a misaligned box is never issued
    if (tid == 0) {
        tc::mbar_init(row_bar, 1);
        tc::mbar_init(row_bar + 1, 1);     // the test hook's barrier: never arrived on
        tc::mbar_fence_init();
        tc::fence_smem_to_async();
    }
    __syncthreads();
    if (tid < 32 && issued) {
        const int nbox = (m + 255) >> 8;
        if (tid == 0) tma::arrive_expect_tx(row_bar, 2048u * nbox + (SINC ? 2u * kTabShorts : 0u));
        __syncwarp();
        for (int b = tid; b < nbox; b += 32) tma::load_2d(row + 256 * b, &a.p1_map, 256 * b, j, row_bar);
        if (SINC && tid == 0) tma::bulk_load(tab, a.tabq, 2u * kTabShorts, row_bar);
    }
    const double krj = a.kr_grid[j];
    const double s0 = krj * a.tan_s[0], s1 = krj * a.tan_s[m - 1];
    const bool asc = s1 >= s0;
    auto xa = [&](int t) { return krj * __ldg(a.tan_s + (asc ? t : m - 1 - t)); };
    const double lo_v = asc ? s0 : s1, hi_v = asc ? s1 : s0;
    const double inv_span = (double)(m - 1) / (hi_v - lo_v);
    const double hn = a.window ? a.ham_n[j] : 1.0;
    int bl[E];      // packed bracket: lower natural index | phase << 16 | reversed << 24; -1 = outside
    float bf[E];    // lerp weight toward the upper sample
    constexpr int CH = 2;
#pragma unroll
    for (int u0 = 0; u0 < E; u0 += CH) {
        double q[CH];
        bool ok[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const int k = tid + T * (u0 + c);
            ok[c] = k < m;
            q[c] = ok[c] ? __ldg(a.kc_grid + k) : 0.0;
        }
        int ja[CH];
        Frac fr[CH];
        interp_brackets<SINC, CH>(xa, m, lo_v, hi_v, inv_span, q, ok, ja, fr);
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const int u = u0 + c;
            if constexpr (PK) {
                // the adjoint's brackets on the ascending view (fraction and phase before any mirroring)
                if (ok[c]) {
                    uint32_t pkv;
                    if (ja[c] < 0) pkv = pack_br(1, q[c] < lo_v ? 0 : m - 2, 0.f);
                    else if (SINC && ja[c] >= 15 && ja[c] <= m - 17) pkv = pack_br_phase(ja[c], fr[c].ph);
                    else pkv = pack_br(0, ja[c], fr[c].f);
                    a.pk_out[(size_t)j * m + tid + T * u] = pkv;
                }
            }
            bl[u] = -1;
            bf[u] = 0.f;
            if (ja[c] >= 0) {
                int lowi = ja[c];
                if (!asc) { lowi = m - 2 - ja[c]; mirror_frac(fr[c]); }
                bl[u] = lowi | (fr[c].ph << 16) | (fr[c].rev << 24);
                bf[u] = fr[c].f;
            }
        }
    }
    // sinc: warp 0 waits for the row and the block barrier passes its view of the landed bytes to the other
    // warps; lerp: every thread waits (each measured the faster of the two for its kernel, by ~1 %)
    const bool probe_ok = a.probe <= 0 || tc::mbar_wait(row_bar + 1, 0, (uint32_t)a.probe);
    if constexpr (SINC) {
        bool got = true;
        if (tid < 32) got = issued && probe_ok && tc::mbar_wait(row_bar, 0, kRowWaitPolls);
        landed = __syncthreads_and(got) != 0;
    } else {
        landed = issued && probe_ok && tc::mbar_wait(row_bar, 0, kRowWaitPolls);
        __syncthreads();
    }
    if (!landed) atomicExch(a.err, 1);      // any thread whose wait ran out: the frame is not valid
#pragma unroll
    for (int u = 0; u < E; ++u) {
        const int k = tid + T * u;
        float2 val = make_float2(0.f, 0.f);
        if (k < m && landed) {
            if (bl[u] >= 0) {
                const int lowi = bl[u] & 0xffff;
                const Frac fr{bf[u], (bl[u] >> 16) & 0xff, (bl[u] >> 24) & 1};
                val = gather_f32<SINC>(row, 0, m, lowi, fr, tab);
                if constexpr (PK && SINC) a.rp_out[(size_t)j * m + k] = val;   // R2 p1 for the adjoint
                // np.outer(hamming(m), hamming(n)).astype(float32)[k, j]
                const float wgt = a.window ? (float)(a.ham_m[k] * hn) : 1.0f;
                const float sg = (a.centred && ((j + k) & 1)) ? -wgt : wgt;
                val.x *= sg;
                val.y *= sg;
            } else if constexpr (PK && SINC) {
                a.rp_out[(size_t)j * m + k] = make_float2(0.f, 0.f);
            }
        }
        x[u] = a.inverse ? make_float2(val.x, -val.y) : val;
    }
    F::run(x, xbuf, a.tw, tid);
    if constexpr (PK) {
        // the autofocus needs S = sum |z|^2 before its range adjoint: z = F_range y1 along zero-padded lines
        // of n2, so S = n2 sum |y1|^2 (Parseval), summed here where y1 is formed
        double *ysum_red = reinterpret_cast<double *>(row_bar + 2);   // dynamic: static shared memory
        double sq = 0.0;                                              // would move region A off 128 bytes
#pragma unroll
        for (int v = 0; v < E; ++v) sq += (double)fmaf(x[v].x, x[v].x, x[v].y * x[v].y);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
        if ((tid & 31) == 0) ysum_red[tid >> 5] = sq;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < T / 32; ++w) t += ysum_red[w];
            atomicAdd(a.ysum, t);
        }
    }
    } else {
#pragma unroll
        for (int v = 0; v < E; ++v) x[v] = make_float2(0.f, 0.f);
    }
    // exchange buffer: this CTA's FFT row in natural frequency order (stays conjugated for the inverse)
    __syncthreads();
#pragma unroll
    for (int v = 0; v < E; ++v) xbuf[tid + T * v] = x[v];
    cluster.sync();
    const int rank = (int)cluster.block_rank();
    const int j0 = j - rank;
    constexpr int SLICE = N / kCT;
#pragma unroll
    for (int s2 = 0; s2 < E; ++s2) {
        const int item = tid + T * s2;         // item = kk * kCT + r
        const int r = item % kCT;
        const int k = rank * SLICE + item / kCT;
        const float2 *remote = cluster.map_shared_rank(xbuf, r);
        a.y1t[(size_t)k * a.npad + j0 + r] = remote[k];
    }
    cluster.sync();                            // keep this CTA's shared memory alive for the readers
    if (issued && !landed) (void)tc::mbar_wait(row_bar, 0, kRowWaitPolls);   // no copy left in flight at exit
}

// ------------------------------------------------------------------------------------------ K3f
struct FFft2Args {
    const float2 *y1t;
    const float2 *tw;
    void *out;
    int n, npad, centred, detect, inverse;
    float scale;
    int pf;               // L2 prefetch distance in lines (the resident blocks of the grid), 0 = none
    int nlines;
};

template <int L, int E>
__global__ void __launch_bounds__((1 << L) / E, fl_min_ctas(L, E)) k_fl_fft2(FFft2Args a) {
    using F = F32Fft<L, E>;
    constexpr int N = F::N, T = F::T;
    extern __shared__ __align__(16) unsigned char smem[];
    float2 *xbuf = reinterpret_cast<float2 *>(smem);
    const int tid = threadIdx.x;
    const int k = blockIdx.x;                  // cross bin (row of the output image)
    if (a.pf && k + a.pf < a.nlines) l2_prefetch(a.y1t + (size_t)(k + a.pf) * a.npad, (size_t)8 * a.npad, tid);
    float2 x[E];
    const float2 *rowk = a.y1t + (size_t)k * a.npad;
#pragma unroll
    for (int u = 0; u < E; ++u) {
        const int j = tid + T * u;
        x[u] = j < a.n ? __ldcs(rowk + j) : make_float2(0.f, 0.f);
    }
    F::run(x, xbuf, a.tw, tid);
    const size_t base = (size_t)k * N;
    const float cs = a.inverse ? -a.scale : a.scale;     // inverse: conj(FFT(conj(x))) / (m2 n2)
#pragma unroll
    for (int v = 0; v < E; ++v) {
        const int col = tid + T * v;
        float2 z = make_float2(x[v].x * a.scale, x[v].y * cs);
        if (a.detect == PFA_DETECT_MAG) {
            static_cast<float *>(a.out)[base + col] = sqrtf(fmaf(z.x, z.x, z.y * z.y));
        } else if (a.detect == PFA_DETECT_POWER) {
            static_cast<float *>(a.out)[base + col] = fmaf(z.x, z.x, z.y * z.y);
        } else {
            if (a.centred && ((k + col) & 1)) { z.x = -z.x; z.y = -z.y; }
            static_cast<float2 *>(a.out)[base + col] = z;
        }
    }
}

// ------------------------------------------------------------------------------------------ autofocus
// Image-entropy autofocus gradient.  With x = s exp(-j theta) (applied in pass 1), p1 = R1 x,
// z = F_range F_cross (W . R2 p1), I = |z|^2 and E = -sum p log p (p = I / S):
//   g_z  = dE/dconj(z) = -(1/S)(log(I/S) + E) z                     (0 where I = 0)
//   g_p1 = R2^H (W . F_cross^H F_range^H g_z)
//   dE/dtheta_i = 2 Im sum_j conj(g_p1[j, slot_i]) p1[j, slot_i]     (pass 1 is linear and per pulse,
//                 so its adjoint never has to be formed)
// The range FFT is recomputed from the cross-FFT buffer in the adjoint pass instead of storing z.  One
// pass over z suffices: S = n2 sum |y1|^2 comes from the forward pass 2 (Parseval), the range adjoint
// takes the part -(1/S) log(I/S) z of g_z and sums I log I on the way, and the part -(E/S) z, whose
// adjoint is -(E/S) n2 m2 R2^H (W^2 . R2 p1) (F^H F = N on the zero-padded lines), is added in the cross
// adjoint, when E is known.
struct AfRangeArgs {
    const float2 *y1t;      // [m2][npad] forward cross-FFT output, transposed
    const float2 *tw;       // range twiddles (n2)
    double *acc;            // [0] sum |y1|^2 (from the forward pass 2), [1] += sum I log I
    float2 *zadj_t;         // [n][m2] F_range^H (-(1/S) log(I/S) z), range-bin rows
    int n, npad, m2;
};

template <int L, int E>
__device__ __forceinline__ void af_load_range_row(float2 (&x)[E], const AfRangeArgs &a, int k) {
    constexpr int T = (1 << L) / E;
    const float2 *row = a.y1t + (size_t)k * a.npad;
#pragma unroll
    for (int u = 0; u < E; ++u) {
        const int j = threadIdx.x + T * u;
        x[u] = j < a.n ? __ldcs(row + j) : make_float2(0.f, 0.f);
    }
}

template <int L, int E>
__global__ void __cluster_dims__(kCT, 1, 1) __launch_bounds__((1 << L) / E, fl_min_ctas(L, E))
k_af_range_adjoint(AfRangeArgs a) {
    namespace cg = cooperative_groups;
    using F = F32Fft<L, E>;
    constexpr int N = F::N, T = F::T;
    extern __shared__ __align__(16) unsigned char smem[];
    float2 *xbuf = reinterpret_cast<float2 *>(smem);
    cg::cluster_group cluster = cg::this_cluster();
    const int tid = threadIdx.x;
    const int k = blockIdx.x;                         // cross bin
    const double S = a.acc[0] * (double)N;
    const float invS = (float)(1.0 / S), off = (float)(-log(S));
    __shared__ double hred[T / 32];
    float2 x[E];
    af_load_range_row<L, E>(x, a, k);
    F::run(x, xbuf, a.tw, tid);                       // recompute z along range
    float hf = 0.f;                                   // this thread's sum I log I (E values; double beyond)
#pragma unroll
    for (int v = 0; v < E; ++v) {
        const float in = fmaf(x[v].x, x[v].x, x[v].y * x[v].y);
        const float lg = in > 0.f ? logf(in) : 0.f;
        hf = fmaf(in, lg, hf);
        const float c = in > 0.f ? -invS * (lg + off) : 0.f;            // -(1/S) log(I/S)
        x[v] = make_float2(c * x[v].x, -c * x[v].y);                    // conj of that part of g_z
    }
    double h = (double)hf;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
    if ((tid & 31) == 0) hred[tid >> 5] = h;
    F::run(x, xbuf, a.tw, tid);                       // F^H g = conj(F conj(g))
    __syncthreads();                                  // hred complete
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < T / 32; ++w) t += hred[w];
        atomicAdd(a.acc + 1, t);
    }
    __syncthreads();
#pragma unroll
    for (int v = 0; v < E; ++v) xbuf[tid + T * v] = make_float2(x[v].x, -x[v].y);   // range index j
    cluster.sync();
    const int rank = (int)cluster.block_rank();
    const int k0 = k - rank;
    constexpr int SLICE = N / kCT;
#pragma unroll
    for (int s2 = 0; s2 < E; ++s2) {
        const int item = tid + T * s2;
        const int r = item % kCT;
        const int j = rank * SLICE + item / kCT;
        if (j < a.n) {
            const float2 *remote = cluster.map_shared_rank(xbuf, r);
            a.zadj_t[(size_t)j * a.m2 + k0 + r] = remote[j];
        }
    }
    cluster.sync();
}

struct AfCrossArgs {
    const float2 *zadj_t;   // [n][m2]
    const float2 *p1;       // [n][mpad] forward pass-1 output (phase corrected)
    const uint32_t *pk;     // [n][m] packed brackets of the forward pass 2 (ascending view)
    const float2 *rp;       // [n][m] float sinc: R2 p1 of the forward pass 2 (before the window)
    const double *ham_m, *ham_n;
    const double *kr_grid, *tan_s;   // the direction of range bin j's pass-2 source axis
    const int16_t *tabq;    // float sinc table (Q15 taps, [phase][kTabRow])
    const float2 *tw;       // cross twiddles (m2)
    float *dacc;            // [mpad] per-slot Im sum conj(g_p1) p1
    const double *acc;      // [0] sum |y1|^2, [1] sum I log I (complete once the range adjoint has run)
    int m, n, mpad, window, n2;
};

// Shared-memory positions of bracket k and of W . F^H g at cross index k in the cross adjoint.  Its
// segmented reduction has lane t walk indices near 16 t; XOR-ing the low four index bits with bits of
// the group index (a permutation inside each aligned group of 16) spreads those lanes over the banks
// (4-byte brackets: bits 5..8; 8-byte values: bits 4..7), and consecutive writers stay conflict free.
__device__ __forceinline__ int pk_at(int k) { return k ^ ((k >> 5) & 15); }
__device__ __forceinline__ int y_at(int k) { return k ^ ((k >> 4) & 15); }
__device__ __forceinline__ float br_w(uint32_t p) { return (float)(p & 0x1ffffu) * (1.0f / 131071.f); }

// R2^H as an atomics-free segmented reduction.  On the ascending view of the sources, bracket k (lower index
// l_k, monotone in k) touches slots l_k and l_k + 1 (lerp: weights 1 - f and f) or, for an interior float
// sinc bracket, slots l_k - 15 .. l_k + 16 (weight tab[phase][u - l_k + 15] / 2^15).  So slot u collects
// the contiguous run of k with l_k in [u - 16, u + 15] (sinc) or [u - 1, u] (lerp).  Each thread owns E
// consecutive slots: the lerp walks one run per slot; the sinc reads each bracket of the union of its
// slots' runs once and adds it to every slot it reaches.  A descending source axis maps ascending slot u to
// natural slot m - 1 - u (the forward mirrors the bracket and reverses the taps, which is the same map).
template <int L, int E, bool SINC>
__global__ void __launch_bounds__((1 << L) / E, fl_min_ctas(L, E)) k_af_cross_adjoint(AfCrossArgs a) {
    using F = F32Fft<L, E>;
    constexpr int N = F::N, T = F::T;
    constexpr int REACH_LO = SINC ? 16 : 1, REACH_HI = SINC ? 15 : 0;
    extern __shared__ __align__(16) unsigned char smem[];
    float2 *xbuf = reinterpret_cast<float2 *>(smem);
    uint32_t *pk = reinterpret_cast<uint32_t *>(smem + (size_t)8 * F::xbuf_elems());
    const int tid = threadIdx.x;
    const int j = blockIdx.x;                         // range bin (< n)
    const int m = a.m;
    int16_t *tab = reinterpret_cast<int16_t *>(smem + (size_t)8 * F::xbuf_elems() + (size_t)4 * ((m + 15) & ~15));
    // the forward pass-2 brackets of this range bin (stored by the forward pass 2 of this gradient)
    {
        const uint32_t *src = a.pk + (size_t)j * m;
        for (int k = tid; k < m; k += T) pk[pk_at(k)] = __ldcs(src + k);
        if (SINC) {
            const uint4 *t4 = reinterpret_cast<const uint4 *>(a.tabq);
            for (int c = tid; c < kTabShorts / 8; c += T) reinterpret_cast<uint4 *>(tab)[c] = __ldg(t4 + c);
        }
    }
    const double krj = a.kr_grid[j];
    const bool asc = krj * a.tan_s[m - 1] >= krj * a.tan_s[0];    // as the forward pass 2 decides
    // adjoint of the cross FFT
    const float2 *row = a.zadj_t + (size_t)j * N;
    float2 x[E];
#pragma unroll
    for (int u = 0; u < E; ++u) {
        const float2 v = __ldcs(row + tid + T * u);
        x[u] = make_float2(v.x, -v.y);
    }
    F::run(x, xbuf, a.tw, tid);
    const double hn = a.window ? a.ham_n[j] : 1.0;
    // the -(E/S) z part of g_z: -(E/S) n2 m2 W^2 . R2 p1 at cross index k, R2 p1 from the forward brackets
    const double S = a.acc[0] * (double)a.n2;
    const double Ent = log(S) - a.acc[1] / S;
    const float beta = (float)(-(Ent / S) * (double)a.n2 * (double)N);
    const float2 *p1row = a.p1 + (size_t)j * a.mpad;
    auto nat = [&](int t) { return asc ? t : m - 1 - t; };   // ascending-view source -> natural slot
    __syncthreads();
    // four cross indices at a time: their two lerp samples are loaded (clamped indices, so unconditionally)
    // before any is used, so the loads of the four overlap
    constexpr int QB = E >= 4 ? 4 : E;
    static_assert(E % QB == 0, "tile of whole load batches");
#pragma unroll
    for (int v0 = 0; v0 < E; v0 += QB) {
        uint32_t bb[QB];
        float2 s0[QB], s1[QB];
#pragma unroll
        for (int c = 0; c < QB; ++c) {
            const int k = tid + T * (v0 + c);
            bb[c] = k < m ? pk[pk_at(k)] : 0x80000000u;
            if constexpr (SINC) {
                // the forward pass 2 stored R2 p1 (its 32-tap gathers): one coalesced load per cross index
                s0[c] = k < m ? __ldcs(a.rp + (size_t)j * m + k) : make_float2(0.f, 0.f);
            } else {
                const int l = min(br_low(bb[c]), m - 2);
                s0[c] = __ldg(p1row + nat(l));
                s1[c] = __ldg(p1row + nat(l + 1));
            }
        }
#pragma unroll
        for (int c = 0; c < QB; ++c) {
            const int v = v0 + c;
            const int k = tid + T * v;
            const float w = k < m ? (a.window ? (float)(a.ham_m[k] * hn) : 1.0f) : 0.f;
            float2 fw = make_float2(0.f, 0.f);          // (R2 p1)[k]
            if constexpr (SINC) {
                fw = s0[c];
            } else if (!(bb[c] >> 31)) {
                const float f = br_w(bb[c]);
                fw = make_float2(fmaf(f, s1[c].x - s0[c].x, s0[c].x), fmaf(f, s1[c].y - s0[c].y, s0[c].y));
            }
            const float bw = beta * w * w;
            // W . F_cross^H g, cross index k
            xbuf[y_at(k)] = make_float2(fmaf(bw, fw.x, w * x[v].x), fmaf(bw, fw.y, -w * x[v].y));
        }
    }
    __syncthreads();
    const int r_lo = tid * E;
    float2 gs[E];
#pragma unroll
    for (int s2 = 0; s2 < E; ++s2) gs[s2] = make_float2(0.f, 0.f);
    if (r_lo < m) {
        // The brackets of queries outside the row's source span carry no weight.  They are a prefix of k
        // (packed with lower index 0) and a suffix (lower index m - 2), so they sit inside the runs of
        // the first and the last slots; walking them would cost those threads (and their CTA) one step per
        // dead bracket and slot.  The walks cover only the live range [k0, k1).
        int k0, k1;
        {
            int lo = 0, hi = m;                         // first k past the dead prefix
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                const uint32_t b = pk[pk_at(mid)];
                if ((b >> 31) && br_low(b) == 0) lo = mid + 1; else hi = mid;
            }
            k0 = lo;
            hi = m;                                     // first dead k at or after k0: the dead suffix
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (!(pk[pk_at(mid)] >> 31)) lo = mid + 1; else hi = mid;
            }
            k1 = lo;
        }
        int lo = k0, hi = k1;                           // first live k with lower index >= r_lo - REACH_LO
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (br_low(pk[pk_at(mid)]) < r_lo - REACH_LO) lo = mid + 1; else hi = mid;
        }
        int kp = lo;
        if constexpr (SINC) {
            // Bracket-outer: every live bracket whose taps reach one of this thread's E slots (lower index
            // l in [r_lo - 16, r_lo + E + 14]) is read once and added to each slot it reaches, in the same
            // increasing-k order per slot as a slot-by-slot walk.  Interior brackets add tap r - l + 15 of
            // their phase row as the integer Q15 value, edge brackets their lerp weights times 2^15; the
            // sums are scaled by 2^-15 at the end (a power of two commutes with every rounding, so each sum
            // is the one the float taps give).
            for (int kk = kp; kk < k1; ++kk) {
                const uint32_t b = pk[pk_at(kk)];
                const int l = br_low(b);
                if (l > r_lo + E - 1 + REACH_HI) break;
                const float2 y = xbuf[y_at(kk)];
                if (l >= 15 && l <= m - 17) {
                    const int16_t *row = tab + (b & 0xffu) * kTabRow;
                    const int t0 = r_lo - l + 15;          // tap of slot r_lo
#pragma unroll
                    for (int s2 = 0; s2 < E; ++s2) {
                        if ((unsigned)(t0 + s2) < 32u) {
                            const float w = s16f(row[t0 + s2]);
                            gs[s2].x = fmaf(w, y.x, gs[s2].x);
                            gs[s2].y = fmaf(w, y.y, gs[s2].y);
                        }
                    }
                } else if (!(b >> 31)) {
                    const float f = br_w(b);
                    const float w0 = (1.0f - f) * 32768.f, w1 = f * 32768.f;
#pragma unroll
                    for (int s2 = 0; s2 < E; ++s2) {
                        const int r = r_lo + s2;
                        if (r == l) {
                            gs[s2].x = fmaf(w0, y.x, gs[s2].x);
                            gs[s2].y = fmaf(w0, y.y, gs[s2].y);
                        } else if (r == l + 1) {
                            gs[s2].x = fmaf(w1, y.x, gs[s2].x);
                            gs[s2].y = fmaf(w1, y.y, gs[s2].y);
                        }
                    }
                }
            }
#pragma unroll
            for (int s2 = 0; s2 < E; ++s2) {
                gs[s2].x *= 1.0f / 32768.f;
                gs[s2].y *= 1.0f / 32768.f;
                if (r_lo + s2 >= m) gs[s2] = make_float2(0.f, 0.f);
            }
        } else {
#pragma unroll
            for (int s2 = 0; s2 < E; ++s2) {
                const int r = r_lo + s2;
                if (r < m) {
                    float2 gsum = make_float2(0.f, 0.f);
                    for (int kk = kp; kk < k1; ++kk) {
                        const uint32_t b = pk[pk_at(kk)];
                        const int l = br_low(b);
                        if (l > r + REACH_HI) break;
                        if (b >> 31) continue;
                        const float f = br_w(b);
                        const float wgt = (l == r) ? 1.0f - f : (l == r - 1 ? f : 0.f);
                        const float2 y = xbuf[y_at(kk)];
                        gsum.x = fmaf(wgt, y.x, gsum.x);
                        gsum.y = fmaf(wgt, y.y, gsum.y);
                    }
                    while (kp < k1 && br_low(pk[pk_at(kp)]) < r + 1 - REACH_LO) ++kp;
                    gs[s2] = gsum;
                }
            }
        }
    }
    // the slot sums go through shared memory (padded: a thread's E consecutive slots hit distinct banks)
    // so that the p1 loads and the accumulation run slot-coalesced, all of a thread's loads in flight
    __syncthreads();
#pragma unroll
    for (int s2 = 0; s2 < E; ++s2) xbuf[F::pad(r_lo + s2)] = gs[s2];
    __syncthreads();
    float2 pv[E];
#pragma unroll
    for (int v = 0; v < E; ++v) {
        const int r = tid + T * v;
        pv[v] = r < m ? __ldcs(p1row + r) : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int v = 0; v < E; ++v) {
        const int r = tid + T * v;                    // natural slot
        if (r < m) {
            const float2 g = xbuf[F::pad(asc ? r : m - 1 - r)];
            atomicAdd(a.dacc + r, g.x * pv[v].y - g.y * pv[v].x);   // Im(conj(g) p1)
        }
    }
}

__global__ void k_af_finish(const float *dacc, const int32_t *order, const double *acc, float *dtheta, double *ent, int m,
                            int n2) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < m && dtheta) dtheta[order[r]] = 2.0f * dacc[r];
    if (r == 0 && ent) {
        const double S = acc[0] * (double)n2;
        ent[0] = log(S) - acc[1] / S;
    }
}

// One step of the autofocus descent on the device: g = dE/dtheta (2 dacc in slot order), theta <- theta -
// step (g - mean g) / max |g - mean g| (a constant phase does not change the image).  One block.
__global__ void __launch_bounds__(1024) k_af_update(const float *dacc, const int32_t *order, float *theta, int m,
                                                    float step) {
    __shared__ double red[32];
    __shared__ float bc[2];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double s = 0.0;
    for (int r = tid; r < m; r += blockDim.x) s += 2.0 * (double)dacc[r];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        bc[0] = (float)(t / m);
    }
    __syncthreads();
    const float mean = bc[0];
    float mx = 0.f;
    for (int r = tid; r < m; r += blockDim.x) mx = fmaxf(mx, fabsf(2.0f * dacc[r] - mean));
    mx = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(mx)));   // non-negative floats
    if (lane == 0) red[warp] = mx;
    __syncthreads();
    if (tid == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmaxf(t, (float)red[w]);
        bc[1] = fmaxf(t, 1e-30f);
    }
    __syncthreads();
    const float scale = step / bc[1];
    for (int r = tid; r < m; r += blockDim.x) theta[order[r]] -= scale * (2.0f * dacc[r] - mean);
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
struct Cfg {
    static constexpr int N = 1 << L;
    static constexpr int E = (N >= 512) ? 16 : (N / 32);
    static constexpr int T = N / E;
};

template <int L, int E, bool SINC>
cudaError_t launch_pass2(const FloatDev &d, cudaStream_t st) {
    using F = F32Fft<L, E>;
    FPass2Args p{d.p1_map, d.tan_s, d.kr, d.kc, d.ham_m64, d.ham_n64, d.tabq, d.twm, d.y1, d.pk_out, d.rp_out, d.wait_err,
                 d.m, d.n, d.mpad, d.npad, d.layout == PFA_LAYOUT_CENTRED, d.window, d.sgn > 0,
                 d.mixed ? 0 : d.mx_probe, d.pk_out ? d.af_acc : nullptr};
    // + 2 mbarriers + the autofocus forward's reduction scratch
    const size_t sm = pass2_region_a(d.m, F::xbuf_elems()) + (SINC ? kTabShorts * 2 : 0) + 16 +
                      (d.pk_out ? (size_t)8 * std::max(1, F::T / 32) : 0);
    auto fn = k_fl_pass2_fft<L, E, SINC>;
    if (d.pk_out) fn = k_fl_pass2_fft<L, E, SINC, true>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    fn<<<d.npad, (1 << L) / E, sm, st>>>(p);
    return cudaGetLastError();
}

template <int L, int E>
cudaError_t launch_fft2(const FloatDev &d, void *out, int detect, float scale, cudaStream_t st) {
    using F = F32Fft<L, E>;
    FFft2Args p{d.y1, d.twn, out, d.n, d.npad, d.layout == PFA_LAYOUT_CENTRED, detect, d.sgn > 0, scale, 0, d.m2};
    size_t sm = (size_t)8 * F::xbuf_elems();
    auto fn = k_fl_fft2<L, E>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    p.pf = resident_blocks(fn, (1 << L) / E, sm);
    fn<<<d.m2, (1 << L) / E, sm, st>>>(p);
    return cudaGetLastError();
}

// FFT register tile: 16 complex values per thread; 8 on request (twice the CTA size) for lines of 256
// points and more; 32 (half the CTA size, radix-32 passes: one shared-memory exchange fewer) for lines
// of 8192 and 16384 points, on request and by default for the range FFT (0 = automatic).  The cross
// FFT of pass 2 stays at 16 by default: that kernel is latency bound and loses more to the halved
// CTA than it gains from the saved exchange.
template <int L, bool SINC>
cudaError_t pass2_tile(const FloatDev &d, cudaStream_t st) {
    if constexpr (L >= 8 && L <= 13) {      // 2^L / 8 threads must stay within a CTA's 1024
        if (d.ept_cross == 8) return launch_pass2<L, 8, SINC>(d, st);
    }
    if constexpr (L >= 13) {
        if (d.ept_cross == 32) return launch_pass2<L, 32, SINC>(d, st);
    }
    return launch_pass2<L, Cfg<L>::E, SINC>(d, st);
}

template <int L>
cudaError_t fft2_tile(const FloatDev &d, void *out, int detect, float scale, cudaStream_t st) {
    if constexpr (L >= 8 && L <= 13) {
        if (d.ept_range == 8) return launch_fft2<L, 8>(d, out, detect, scale, st);
    }
    if constexpr (L >= 13) {               // the automatic choice (0) for these lines: 32 (measured faster)
        if (d.ept_range == 32 || d.ept_range == 0) return launch_fft2<L, 32>(d, out, detect, scale, st);
    }
    return launch_fft2<L, Cfg<L>::E>(d, out, detect, scale, st);
}

template <bool SINC>
cudaError_t dispatch_pass2(const FloatDev &d, cudaStream_t st) {
    switch (d.Lm) {
        case 6: return pass2_tile<6, SINC>(d, st);
        case 7: return pass2_tile<7, SINC>(d, st);
        case 8: return pass2_tile<8, SINC>(d, st);
        case 9: return pass2_tile<9, SINC>(d, st);
        case 10: return pass2_tile<10, SINC>(d, st);
        case 11: return pass2_tile<11, SINC>(d, st);
        case 12: return pass2_tile<12, SINC>(d, st);
        case 13: return pass2_tile<13, SINC>(d, st);
        case 14: return pass2_tile<14, SINC>(d, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t dispatch_fft2(const FloatDev &d, void *out, int detect, float scale, cudaStream_t st) {
    switch (d.Ln) {
        case 6: return fft2_tile<6>(d, out, detect, scale, st);
        case 7: return fft2_tile<7>(d, out, detect, scale, st);
        case 8: return fft2_tile<8>(d, out, detect, scale, st);
        case 9: return fft2_tile<9>(d, out, detect, scale, st);
        case 10: return fft2_tile<10>(d, out, detect, scale, st);
        case 11: return fft2_tile<11>(d, out, detect, scale, st);
        case 12: return fft2_tile<12>(d, out, detect, scale, st);
        case 13: return fft2_tile<13>(d, out, detect, scale, st);
        case 14: return fft2_tile<14>(d, out, detect, scale, st);
        default: return cudaErrorInvalidValue;
    }
}

int ilog2i(int v) { int l = 0; while ((1 << l) < v) ++l; return l; }

template <class T>
cudaError_t dal(T **p, size_t cnt) { return cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(cnt, 1) * sizeof(T)); }
template <class T>
void dfr(T *&p) { if (p) cudaFree(p); p = nullptr; }

// W_N^k = exp(-2 pi i k / N), k < N (the inverse transform conjugates data, not twiddles)
void full_twiddles(int N, std::vector<float2> &out) {
    out.resize(N);
    for (int k = 0; k < N; ++k) {
        const double th = -2.0 * M_PI * (double)k / (double)N;
        out[k] = make_float2((float)std::cos(th), (float)std::sin(th));
    }
}

}  // namespace

size_t float_workspace_bytes(int m, int n) {
    const int m2 = 1 << ilog2i(m), mpad = (m + 31) / 32 * 32;
    const int npad = (n + 7) / 8 * 8;
    return (size_t)8 * n * mpad + (size_t)8 * npad * m2;
}

cudaError_t float_alloc(FloatDev &d, int m, int n) {
    d.m = m; d.n = n;
    d.Lm = ilog2i(m); d.Ln = ilog2i(n);
    d.m2 = 1 << d.Lm; d.n2 = 1 << d.Ln;
    d.mpad = (m + 31) / 32 * 32;
    d.npad = (n + 7) / 8 * 8;             // whole clusters of the FP32 (kCT) and mixed pass-2 kernels
    if (d.m2 < 64 || d.n2 < 64 || d.m2 > 16384 || d.n2 > 16384) return cudaErrorInvalidValue;
    cudaError_t e;
#define TRY(x) do { e = (x); if (e != cudaSuccess) return e; } while (0)
    TRY(dal(&d.f0, m)); TRY(dal(&d.df, m)); TRY(dal(&d.flast, m)); TRY(dal(&d.pr, m)); TRY(dal(&d.tan_s, m)); TRY(dal(&d.order, m));
    TRY(dal(&d.kr, n)); TRY(dal(&d.kc, m)); TRY(dal(&d.ham_m64, m)); TRY(dal(&d.ham_n64, n));
    TRY(dal(&d.twm, d.m2)); TRY(dal(&d.twn, d.n2));
    TRY(dal(&d.tabq, kTabShorts));
    TRY(dal(&d.p1, (size_t)n * d.mpad)); TRY(dal(&d.y1, (size_t)d.npad * d.m2));
    TRY(dal(&d.wait_err, 1)); TRY(cudaMemset(d.wait_err, 0, sizeof(int)));
    // pass 2 reads its range-bin row of p1 as 256-sample boxes (2 KB; the last one zero-filled past mpad)
    TRY(tma::encode_2d(&d.p1_map, d.p1, 8, (uint64_t)d.mpad, (uint64_t)n, (uint64_t)8 * d.mpad, 256, 1));
#undef TRY
    return cudaSuccess;
}

void float_free(FloatDev &d) {
    dfr(d.f0); dfr(d.df); dfr(d.flast); dfr(d.pr); dfr(d.tan_s); dfr(d.order); dfr(d.kr); dfr(d.kc); dfr(d.ham_m64);
    dfr(d.ham_n64); dfr(d.twm); dfr(d.twn); dfr(d.tabq); dfr(d.p1); dfr(d.y1); dfr(d.wait_err);
    dfr(d.af_zadj); dfr(d.af_acc); dfr(d.af_dacc); dfr(d.af_pk); dfr(d.af_rp);
    mixed_free(d);
}

cudaError_t float_form(const FloatDev &d, const float2 *sig, void *out, int detect, cudaStream_t st, StageProf *prof,
                       const float *theta) {
    StageProf none;
    StageProf &pf = prof ? *prof : none;
    pf.count = 0;
    cudaError_t e = pf.mark(st, "start");
    if (e != cudaSuccess) return e;
    FPass1Args p1{sig, d.f0, d.df, d.flast, d.pr, d.kr, d.order, d.tabq, theta, d.p1, d.m, d.n, d.mpad};
    dim3 g1((d.m + F1_SLOTS - 1) / F1_SLOTS, (d.n + f1_bins(d.range_sinc) - 1) / f1_bins(d.range_sinc));
    if (d.range_sinc) {
        e = cudaFuncSetAttribute(k_fl_pass1<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f1_smem(true));
        if (e != cudaSuccess) return e;
        k_fl_pass1<true><<<g1, 256, f1_smem(true), st>>>(p1);
    } else {
        e = cudaFuncSetAttribute(k_fl_pass1<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f1_smem(false));
        if (e != cudaSuccess) return e;
        k_fl_pass1<false><<<g1, 256, f1_smem(false), st>>>(p1);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = pf.mark(st, "pass1")) != cudaSuccess) return e;
    // mixed mode: tensor-core FFTs on the axes whose lines are 2048..8192 points, FP32 FFTs elsewhere
    if (d.mixed && mixed_axis(d.Lm)) e = mixed_pass2(d, st);
    else e = d.az_sinc ? dispatch_pass2<true>(d, st) : dispatch_pass2<false>(d, st);
    if (e != cudaSuccess) return e;
    if ((e = pf.mark(st, "pass2_win_fft1")) != cudaSuccess) return e;
    const float scale = d.sgn > 0 ? 1.0f / ((float)d.m2 * (float)d.n2) : 1.0f;
    if (d.mixed && mixed_axis(d.Ln)) e = mixed_fft2(d, out, detect, scale, st);
    else e = dispatch_fft2(d, out, detect, scale, st);
    if (e != cudaSuccess) return e;
    return pf.mark(st, "fft2_detect");
}

template <int L>
cudaError_t launch_af_range(const FloatDev &d, cudaStream_t st) {
    using F = F32Fft<L, Cfg<L>::E>;
    AfRangeArgs p{d.y1, d.twn, d.af_acc, d.af_zadj, d.n, d.npad, d.m2};
    const size_t sm = (size_t)8 * F::xbuf_elems();
    auto f2 = k_af_range_adjoint<L, Cfg<L>::E>;
    const cudaError_t e = cudaFuncSetAttribute(f2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    f2<<<d.m2, Cfg<L>::T, sm, st>>>(p);
    return cudaGetLastError();
}

template <int L>
cudaError_t launch_af_cross(const FloatDev &d, cudaStream_t st) {
    using F = F32Fft<L, Cfg<L>::E>;
    AfCrossArgs p{d.af_zadj, d.p1, d.af_pk, d.af_rp, d.ham_m64, d.ham_n64, d.kr, d.tan_s, d.tabq, d.twm, d.af_dacc, d.af_acc,
                  d.m, d.n, d.mpad, d.window, d.n2};
    // exchange buffer, packed brackets (whole groups of 16), sinc table
    const size_t sm = (size_t)8 * F::xbuf_elems() + (size_t)4 * ((d.m + 15) & ~15) + (d.az_sinc ? kTabShorts * 2 : 0);
    auto fn = d.az_sinc ? k_af_cross_adjoint<L, Cfg<L>::E, true> : k_af_cross_adjoint<L, Cfg<L>::E, false>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    fn<<<d.n, Cfg<L>::T, sm, st>>>(p);
    return cudaGetLastError();
}

#define PFA_DISPATCH_L(Lv, call)                                        \
    switch (Lv) {                                                       \
        case 6: return call<6>; case 7: return call<7>;                 \
        case 8: return call<8>; case 9: return call<9>;                 \
        case 10: return call<10>; case 11: return call<11>;             \
        case 12: return call<12>; case 13: return call<13>;             \
        default: return cudaErrorInvalidValue;                          \
    }

cudaError_t af_range(const FloatDev &d, cudaStream_t st) {
#define CALL(Lx) launch_af_range<Lx>(d, st)
    switch (d.Ln) {
        case 6: return CALL(6); case 7: return CALL(7); case 8: return CALL(8); case 9: return CALL(9);
        case 10: return CALL(10); case 11: return CALL(11); case 12: return CALL(12); case 13: return CALL(13);
        case 14: return CALL(14);
        default: return cudaErrorInvalidValue;
    }
#undef CALL
}

cudaError_t af_cross(const FloatDev &d, cudaStream_t st) {
#define CALL(Lx) launch_af_cross<Lx>(d, st)
    switch (d.Lm) {
        case 6: return CALL(6); case 7: return CALL(7); case 8: return CALL(8); case 9: return CALL(9);
        case 10: return CALL(10); case 11: return CALL(11); case 12: return CALL(12); case 13: return CALL(13);
        case 14: return CALL(14);
        default: return cudaErrorInvalidValue;
    }
#undef CALL
}
#undef PFA_DISPATCH_L

// Entropy and its gradient w.r.t. the per-pulse phase correction theta (float32; lerp or float sinc passes).
cudaError_t autofocus_grad(const FloatDev &d0, const float2 *sig, const float *theta, float *dtheta, double *ent,
                           cudaStream_t st, StageProf *prof) {
    StageProf none;
    StageProf &pf = prof ? *prof : none;
    pf.count = 0;
    cudaError_t e = pf.mark(st, "start");
    if (e != cudaSuccess) return e;
    FloatDev d = d0;
    d.layout = PFA_LAYOUT_NATURAL;      // |z| (so E) does not depend on the centring
    d.sgn = -1;
    d.pk_out = d.af_pk;                 // the forward pass 2 keeps its brackets for the cross adjoint
    d.rp_out = d.az_sinc ? d.af_rp : nullptr;   // and, float sinc, its resampled rows
    if ((e = cudaMemsetAsync(d.af_acc, 0, 2 * sizeof(double), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(d.af_dacc, 0, sizeof(float) * d.mpad, st)) != cudaSuccess) return e;
    FPass1Args p1{sig, d.f0, d.df, d.flast, d.pr, d.kr, d.order, d.tabq, theta, d.p1, d.m, d.n, d.mpad};
    const bool rs = d.range_sinc != 0;
    dim3 g1((d.m + F1_SLOTS - 1) / F1_SLOTS, (d.n + f1_bins(rs) - 1) / f1_bins(rs));
    auto k1 = rs ? k_fl_pass1<true> : k_fl_pass1<false>;
    e = cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f1_smem(rs));
    if (e != cudaSuccess) return e;
    k1<<<g1, 256, f1_smem(rs), st>>>(p1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = pf.mark(st, "pass1_phase")) != cudaSuccess) return e;
    if ((e = (d.az_sinc ? dispatch_pass2<true>(d, st) : dispatch_pass2<false>(d, st))) != cudaSuccess) return e;
    if ((e = pf.mark(st, "pass2_win_fft1")) != cudaSuccess) return e;
    if ((e = af_range(d, st)) != cudaSuccess) return e;
    if ((e = pf.mark(st, "range_entropy_adjoint")) != cudaSuccess) return e;
    if ((e = af_cross(d, st)) != cudaSuccess) return e;
    if ((e = pf.mark(st, "cross_adjoint_pass2T")) != cudaSuccess) return e;
    k_af_finish<<<(d.m + 255) / 256, 256, 0, st>>>(d.af_dacc, d.order, d.af_acc, dtheta, ent, d.m, d.n2);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return pf.mark(st, "finish");
}

}  // namespace pfa

// ------------------------------------------------------------------------------------------ C ABI
namespace {
pfa_status ffail(pfa_plan *p, pfa_status st, const char *msg) {
    if (p) p->err = msg;
    return st;
}
struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev) { if (cudaGetDevice(&prev) != cudaSuccess) prev = -1; if (prev != dev) cudaSetDevice(dev); }
    ~DevGuard() { int cur = -1; if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev); }
};
pfa_status fcuda(pfa_plan *p, cudaError_t e, const char *where) {
    if (p) p->err = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? PFA_ERR_ALLOC : PFA_ERR_CUDA;
}
}  // namespace

extern "C" {

pfa_status pfa_set_float_job(pfa_plan *p, const pfa_float_job *job) {
    if (!p || !job) return PFA_ERR_BAD_ARG;
    if (p->cfg.mode != PFA_MODE_FLOAT32 && p->cfg.mode != PFA_MODE_MIXED) return ffail(p, PFA_ERR_BAD_CONFIG, "plan is not float mode");
    if (!job->f0 || !job->df || !job->f_last || !job->pr || !job->tan_s || !job->order || !job->kr_grid || !job->kc_grid)
        return ffail(p, PFA_ERR_BAD_ARG, "missing job vector");
    if (job->layout != PFA_LAYOUT_CENTRED && job->layout != PFA_LAYOUT_NATURAL) return ffail(p, PFA_ERR_BAD_ARG, "bad layout");
    DevGuard dg(p->device);
    pfa::FloatDev &d = p->fl;
    const int m = d.m, n = d.n;
    std::vector<int> seen(m, 0);
    for (int i = 0; i < m; ++i) {
        const int r = job->order[i];
        if (r < 0 || r >= m || seen[r]++) return ffail(p, PFA_ERR_BAD_ARG, "order is not a permutation");
    }
    d.sgn = job->sgn < 0 ? -1 : 1;
    d.layout = job->layout;
    d.window = (job->ham_m && job->ham_n) ? 1 : 0;
    cudaError_t e;
#define CPY(dst, src, cnt) do { e = cudaMemcpy(dst, src, sizeof(*(dst)) * (cnt), cudaMemcpyHostToDevice); \
        if (e != cudaSuccess) return fcuda(p, e, "float job upload"); } while (0)
    if (!d.consts_ready) {      // twiddles and the sinc table depend on the plan's shape only
        std::vector<float2> twm, twn;
        pfa::full_twiddles(d.m2, twm);
        pfa::full_twiddles(d.n2, twn);
        std::vector<int16_t> tabq(pfa::kTabShorts, 0);
        const int16_t *tq = pfa::builtin_sinc_table();
        for (int i = 0; i < 256 * 32; ++i) tabq[(i >> 5) * pfa::kTabRow + (i & 31)] = tq[i];   // [phase][tap], padded rows
        CPY(d.twm, twm.data(), d.m2); CPY(d.twn, twn.data(), d.n2);
        CPY(d.tabq, tabq.data(), pfa::kTabShorts);
        d.consts_ready = true;
    }
    CPY(d.f0, job->f0, m); CPY(d.df, job->df, m); CPY(d.flast, job->f_last, m); CPY(d.pr, job->pr, m); CPY(d.tan_s, job->tan_s, m);
    CPY(d.order, job->order, m); CPY(d.kr, job->kr_grid, n); CPY(d.kc, job->kc_grid, m);
    if (d.window) { CPY(d.ham_m64, job->ham_m, m); CPY(d.ham_n64, job->ham_n, n); }
#undef CPY
    p->job_ready = true;
    return PFA_OK;
}

pfa_status pfa_form_float(pfa_plan *p, const float *sig_dev, void *out_dev, int32_t detect, void *stream) {
    if (!p || !sig_dev || !out_dev) return PFA_ERR_BAD_ARG;
    if (p->cfg.mode != PFA_MODE_FLOAT32 && p->cfg.mode != PFA_MODE_MIXED) return ffail(p, PFA_ERR_BAD_CONFIG, "plan is not float mode");
    if (!p->job_ready) return ffail(p, PFA_ERR_NOT_READY, "pfa_set_float_job not called");
    if (detect < PFA_DETECT_MAG || detect > PFA_DETECT_COMPLEX) return ffail(p, PFA_ERR_BAD_ARG, "bad detect mode");
    if (reinterpret_cast<uintptr_t>(sig_dev) & 7) return ffail(p, PFA_ERR_BAD_ARG, "signal must be 8-byte aligned");
    if (p->fl.mixed && (reinterpret_cast<uintptr_t>(out_dev) & 15))
        return ffail(p, PFA_ERR_BAD_ARG, "mixed mode: output must be 16-byte aligned");
    DevGuard dg(p->device);
    cudaError_t e = pfa::float_form(p->fl, reinterpret_cast<const float2 *>(sig_dev), out_dev, detect,
                                    reinterpret_cast<cudaStream_t>(stream), &p->prof);
    if (e != cudaSuccess) return fcuda(p, e, "float form");
    return PFA_OK;
}

static pfa_status wait_timeout_check(pfa_plan *p);

pfa_status pfa_form_float_host(pfa_plan *p, const float *sig_host, void *out_host, int32_t detect) {
    if (!p || !sig_host || !out_host) return PFA_ERR_BAD_ARG;
    if (p->cfg.mode != PFA_MODE_FLOAT32 && p->cfg.mode != PFA_MODE_MIXED) return ffail(p, PFA_ERR_BAD_CONFIG, "plan is not float mode");
    DevGuard dg(p->device);
    const size_t in_b = sizeof(float) * 2 * (size_t)p->fl.m * p->fl.n;
    const size_t out_b = (detect == PFA_DETECT_COMPLEX ? 8 : 4) * (size_t)p->fl.m2 * p->fl.n2;
    cudaError_t e;
    if (!p->host_stream && (e = cudaStreamCreateWithFlags(&p->host_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fcuda(p, e, "stream");
    if (p->staging_in_bytes < in_b) {
        if (p->staging_in) cudaFree(p->staging_in);
        p->staging_in = nullptr;
        if ((e = cudaMalloc(reinterpret_cast<void **>(&p->staging_in), in_b)) != cudaSuccess) { p->staging_in_bytes = 0; return fcuda(p, e, "staging"); }
        p->staging_in_bytes = in_b;
    }
    if (p->staging_out_bytes < out_b) {
        if (p->staging_out) cudaFree(p->staging_out);
        p->staging_out = nullptr;
        if ((e = cudaMalloc(&p->staging_out, out_b)) != cudaSuccess) { p->staging_out_bytes = 0; return fcuda(p, e, "staging"); }
        p->staging_out_bytes = out_b;
    }
    if ((e = cudaMemcpyAsync(p->staging_in, sig_host, in_b, cudaMemcpyHostToDevice, p->host_stream)) != cudaSuccess)
        return fcuda(p, e, "h2d");
    pfa_status st = pfa_form_float(p, p->staging_in, p->staging_out, detect, p->host_stream);
    if (st != PFA_OK) return st;
    if ((e = cudaMemcpyAsync(out_host, p->staging_out, out_b, cudaMemcpyDeviceToHost, p->host_stream)) != cudaSuccess)
        return fcuda(p, e, "d2h");
    if ((e = cudaStreamSynchronize(p->host_stream)) != cudaSuccess) return fcuda(p, e, "sync");
    return wait_timeout_check(p);
}

// A bounded wait that ran out (pass 2's TMA row load; in mixed mode also a tensor-core completion) sets a
// device flag; synchronous entry points read (and clear) it after their frames and report PFA_ERR_TIMEOUT.
static pfa_status wait_timeout_check(pfa_plan *p) {
    if (!p->fl.wait_err) return PFA_OK;
    int flag = 0;
    cudaError_t e = cudaMemcpy(&flag, p->fl.wait_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fcuda(p, e, "timeout flag");
    if (!flag) return PFA_OK;
    cudaMemset(p->fl.wait_err, 0, sizeof(int));
    return ffail(p, PFA_ERR_TIMEOUT, "a bounded wait on the device timed out (frame not valid)");
}

static pfa_status float_frame(pfa_plan *p, const void *in, void *out, cudaStream_t st, int32_t detect) {
    return pfa_form_float(p, static_cast<const float *>(in), out, detect, st);
}

pfa_status pfa_form_float_host_frames(pfa_plan *p, const float *const *sig_hosts, void *const *out_hosts,
                                      int32_t detect, int32_t nframes) {
    if (!p) return PFA_ERR_BAD_ARG;
    if (p->cfg.mode != PFA_MODE_FLOAT32 && p->cfg.mode != PFA_MODE_MIXED) return ffail(p, PFA_ERR_BAD_CONFIG, "plan is not float mode");
    if (detect < PFA_DETECT_MAG || detect > PFA_DETECT_COMPLEX) return ffail(p, PFA_ERR_BAD_ARG, "bad detect mode");
    DevGuard dg(p->device);
    const size_t in_b = sizeof(float) * 2 * (size_t)p->fl.m * p->fl.n;
    const size_t out_b = (detect == PFA_DETECT_COMPLEX ? 8 : 4) * (size_t)p->fl.m2 * p->fl.n2;
    const pfa_status st = pfa::run_host_frames(p, reinterpret_cast<const void *const *>(sig_hosts), out_hosts, nframes,
                                               in_b, out_b, float_frame, detect);
    return st != PFA_OK ? st : wait_timeout_check(p);
}

pfa_status pfa_form_float_phase(pfa_plan *p, const float *sig_dev, const float *theta_dev, void *out_dev, int32_t detect,
                                void *stream) {
    if (!p || !sig_dev || !theta_dev || !out_dev) return PFA_ERR_BAD_ARG;
    if (p->cfg.mode != PFA_MODE_FLOAT32 && p->cfg.mode != PFA_MODE_MIXED) return ffail(p, PFA_ERR_BAD_CONFIG, "plan is not float mode");
    if (!p->job_ready) return ffail(p, PFA_ERR_NOT_READY, "pfa_set_float_job not called");
    if (detect < PFA_DETECT_MAG || detect > PFA_DETECT_COMPLEX) return ffail(p, PFA_ERR_BAD_ARG, "bad detect mode");
    if (reinterpret_cast<uintptr_t>(sig_dev) & 7) return ffail(p, PFA_ERR_BAD_ARG, "signal must be 8-byte aligned");
    if (p->fl.mixed && (reinterpret_cast<uintptr_t>(out_dev) & 15))
        return ffail(p, PFA_ERR_BAD_ARG, "mixed mode: output must be 16-byte aligned");
    DevGuard dg(p->device);
    cudaError_t e = pfa::float_form(p->fl, reinterpret_cast<const float2 *>(sig_dev), out_dev, detect,
                                    reinterpret_cast<cudaStream_t>(stream), &p->prof, theta_dev);
    if (e != cudaSuccess) return fcuda(p, e, "float form");
    return PFA_OK;
}

static pfa_status autofocus_common(pfa_plan *p, const float *sig_dev, const float *theta_dev, float *dtheta_dev,
                                   double *entropy_dev, void *stream);

pfa_status pfa_autofocus_step(pfa_plan *p, const float *sig_dev, float *theta_dev, float step, double *entropy_dev,
                              void *stream) {
    if (!p || !sig_dev || !theta_dev) return PFA_ERR_BAD_ARG;
    pfa_status st = autofocus_common(p, sig_dev, theta_dev, nullptr, entropy_dev, stream);
    if (st != PFA_OK) return st;
    DevGuard dg(p->device);
    pfa::k_af_update<<<1, 1024, 0, reinterpret_cast<cudaStream_t>(stream)>>>(p->fl.af_dacc, p->fl.order, theta_dev,
                                                                               p->fl.m, step);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFA_OK : fcuda(p, e, "autofocus update");
}

pfa_status pfa_autofocus_grad(pfa_plan *p, const float *sig_dev, const float *theta_dev, float *dtheta_dev,
                              double *entropy_dev, void *stream) {
    if (!p || !sig_dev || !theta_dev || !dtheta_dev) return PFA_ERR_BAD_ARG;
    return autofocus_common(p, sig_dev, theta_dev, dtheta_dev, entropy_dev, stream);
}

static pfa_status autofocus_common(pfa_plan *p, const float *sig_dev, const float *theta_dev, float *dtheta_dev,
                                   double *entropy_dev, void *stream) {
    if (p->cfg.mode != PFA_MODE_FLOAT32 && p->cfg.mode != PFA_MODE_MIXED) return ffail(p, PFA_ERR_BAD_CONFIG, "plan is not float mode");
    if (!p->job_ready) return ffail(p, PFA_ERR_NOT_READY, "pfa_set_float_job not called");
    pfa::FloatDev &d = p->fl;
    if (reinterpret_cast<uintptr_t>(sig_dev) & 7) return ffail(p, PFA_ERR_BAD_ARG, "signal must be 8-byte aligned");
    DevGuard dg(p->device);
    cudaError_t e;
    if (!d.af_zadj) {
        if ((e = pfa::dal(&d.af_zadj, (size_t)d.n * d.m2)) != cudaSuccess ||
            (e = pfa::dal(&d.af_acc, 2)) != cudaSuccess || (e = pfa::dal(&d.af_dacc, d.mpad)) != cudaSuccess ||
            (e = pfa::dal(&d.af_pk, (size_t)d.n * d.m)) != cudaSuccess ||
            (d.az_sinc && (e = pfa::dal(&d.af_rp, (size_t)d.n * d.m)) != cudaSuccess)) {
            pfa::dfr(d.af_zadj); pfa::dfr(d.af_acc); pfa::dfr(d.af_dacc); pfa::dfr(d.af_pk); pfa::dfr(d.af_rp);
            return fcuda(p, e, "autofocus workspace");
        }
    }
    e = pfa::autofocus_grad(d, reinterpret_cast<const float2 *>(sig_dev), theta_dev, dtheta_dev, entropy_dev,
                            reinterpret_cast<cudaStream_t>(stream), &p->prof);
    if (e != cudaSuccess) return fcuda(p, e, "autofocus");
    return PFA_OK;
}

}  // extern "C"
