// Display scaling of the detected image, the quantiser of save_detected_geotiff
// (src/form_image_pfa.py:287-292):
//
//     amp  = |img| (float32)
//     hi   = np.percentile(amp, 99.7)
//     data = np.clip(amp / (hi + 1e-12) * 255.0, 0, 255).astype(np.uint8)
//
// bit-exact on the device, for non-negative magnitudes (the bit-pattern order below needs x >= 0).  np.percentile of a float32 array computes in float32 (NumPy 2 promotion):
// q = f32(99.7) / 100, virtual index v = f32(n - 1) * q, k = floor(v), gamma = v - k, and the lerp of the
// order statistics a = s[k], b = s[k + 1] is a + (b - a) gamma (gamma < 0.5) or b - (b - a)(1 - gamma),
// each a separate float32 operation.  The host evaluates k and gamma; the device finds the two order
// statistics by a three-pass radix select on the float bit patterns (|z| >= 0, so the uint32 patterns
// sort like the values): 11 + 11 + 10 bits, each pass one block-histogram sweep over the image (HBM
// bound) and a one-block bin pick, then one more sweep for s[k + 1] when it differs from s[k].  All of
// it is stream-ordered in a caller-provided workspace: no allocation, no host synchronisation.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "pfa_internal.h"

namespace pfa {
namespace {

constexpr int kBins = 2048;

struct DispCtrl {
    unsigned long long rank;     // rank of s[k] among the elements that match the prefix so far
    unsigned long long below;    // elements below the current prefix (all passes so far)
    unsigned int prefix;         // value bits fixed so far
    unsigned int cnt_eq;         // elements equal to s[k] (after the last pass)
    unsigned int next_bits;      // s[k + 1] when larger than s[k] (atomicMin target)
    float hi;                    // the percentile
    float h;                     // hi + 1e-12 in float32
    int pad;
};

struct DispWs {
    DispCtrl ctrl;
    unsigned int hist[kBins];
};

__global__ void k_disp_init(DispWs *ws, unsigned long long rank) {
    for (int i = threadIdx.x; i < kBins; i += blockDim.x) ws->hist[i] = 0u;
    if (threadIdx.x == 0) {
        DispCtrl c{};
        c.rank = rank;
        c.next_bits = 0xffffffffu;
        ws->ctrl = c;
    }
}

// pass p: bits [shift, shift + width) of the elements whose bits above shift + width equal the prefix
__global__ void __launch_bounds__(512) k_disp_hist(const float *__restrict__ v, long long n, DispWs *ws, int shift,
                                                   int width) {
    __shared__ unsigned int h[kBins];
    for (int i = threadIdx.x; i < kBins; i += blockDim.x) h[i] = 0u;
    __syncthreads();
    const unsigned int prefix = ws->ctrl.prefix;
    const int top = shift + width;
    const unsigned int mask = (1u << width) - 1u;
    auto add = [&](float x) {
        const unsigned int b = __float_as_uint(x);
        if (top >= 32 || (b >> top) == prefix) atomicAdd(&h[(b >> shift) & mask], 1u);
    };
    const long long n4 = n >> 2;
    const float4 *v4 = reinterpret_cast<const float4 *>(v);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride) {
        const float4 q = __ldcs(v4 + i);
        add(q.x); add(q.y); add(q.z); add(q.w);
    }
    if (blockIdx.x == 0)
        for (long long i = 4 * n4 + threadIdx.x; i < n; i += blockDim.x) add(v[i]);
    __syncthreads();
    for (int i = threadIdx.x; i < (1 << width); i += blockDim.x)
        if (h[i]) atomicAdd(&ws->hist[i], h[i]);
}

// the bin holding rank `rank`: fixes `width` more bits of the prefix, clears the histogram for the next pass.
// One block of 512 threads: each thread scans 4 consecutive bins, a block-wide exclusive scan of the thread
// sums locates the bin.
__global__ void __launch_bounds__(512) k_disp_pick(DispWs *ws, int width, int last) {
    __shared__ unsigned long long part[512];
    const int tid = threadIdx.x;
    const int nb = 1 << width;                          // 1024 or 2048 bins: at most 4 per thread
    unsigned int h[4];
    unsigned long long s = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int b = 4 * tid + i;
        h[i] = b < nb ? ws->hist[b] : 0u;
        s += h[i];
    }
    part[tid] = s;
    __syncthreads();
    for (int off = 1; off < 512; off <<= 1) {           // inclusive Hillis-Steele scan of the thread sums
        const unsigned long long v = tid >= off ? part[tid - off] : 0ull;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    const unsigned long long rank = ws->ctrl.rank;
    const unsigned long long before = tid ? part[tid - 1] : 0ull;
    if (before <= rank && rank < part[tid]) {           // exactly one thread holds the rank
        unsigned long long acc = before;
        int b = 4 * tid;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (acc + h[i] > rank) { b = 4 * tid + i; break; }
            acc += h[i];
        }
        DispCtrl &c = ws->ctrl;
        c.rank = rank - acc;
        c.below += acc;
        c.prefix = (c.prefix << width) | (unsigned int)b;
        if (last) {
            c.cnt_eq = ws->hist[b];
            c.next_bits = 0xffffffffu;
        }
    }
    __syncthreads();
    for (int i = tid; i < kBins; i += blockDim.x) ws->hist[i] = 0u;
}

// s[k + 1] when it is larger than s[k]: the smallest value above s[k]
__global__ void __launch_bounds__(512) k_disp_min_above(const float *__restrict__ v, long long n, DispWs *ws) {
    const DispCtrl &c = ws->ctrl;
    if (c.rank + 1 < c.cnt_eq) return;                  // s[k + 1] == s[k]
    const unsigned int p = c.prefix;
    unsigned int best = 0xffffffffu;
    const long long n4 = n >> 2;
    const float4 *v4 = reinterpret_cast<const float4 *>(v);
    const long long stride = (long long)gridDim.x * blockDim.x;
    auto take = [&](float x) {
        const unsigned int b = __float_as_uint(x);
        if (b > p && b < best) best = b;
    };
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride) {
        const float4 q = __ldcs(v4 + i);
        take(q.x); take(q.y); take(q.z); take(q.w);
    }
    if (blockIdx.x == 0)
        for (long long i = 4 * n4 + threadIdx.x; i < n; i += blockDim.x) take(v[i]);
    best = __reduce_min_sync(0xffffffffu, best);
    if ((threadIdx.x & 31) == 0 && best != 0xffffffffu) atomicMin(&ws->ctrl.next_bits, best);
}

// hi = lerp(s[k], s[k+1], gamma) in float32 as NumPy evaluates it, and h = hi + 1e-12 (float32)
__global__ void k_disp_hi(DispWs *ws, float gamma, int top_only, float *hi_out) {
    DispCtrl &c = ws->ctrl;
    const float a = __uint_as_float(c.prefix);
    const float b = (top_only || c.rank + 1 < c.cnt_eq) ? a : __uint_as_float(c.next_bits);
    const float d = __fsub_rn(b, a);
    const float r = gamma < 0.5f ? __fadd_rn(a, __fmul_rn(d, gamma)) : __fsub_rn(b, __fmul_rn(d, __fsub_rn(1.0f, gamma)));
    c.hi = r;
    c.h = __fadd_rn(r, 1e-12f);
    if (hi_out) *hi_out = r;
}

// data = uint8(clip(amp / h * 255, 0, 255)) (truncation toward zero; a NaN quotient gives 0)
__global__ void __launch_bounds__(256) k_disp_quant(const float *__restrict__ v, long long n, const DispWs *ws,
                                                    uint8_t *__restrict__ out) {
    const float h = ws->ctrl.h;
    auto q8 = [&](float x) -> uint32_t {
        const float y = __fmul_rn(__fdiv_rn(x, h), 255.0f);
        const float c = fminf(fmaxf(y, 0.0f), 255.0f);     // NaN -> 0 (fmaxf returns the number)
        return (uint32_t)c;
    };
    const long long n4 = n >> 2;
    const float4 *v4 = reinterpret_cast<const float4 *>(v);
    uint32_t *o4 = reinterpret_cast<uint32_t *>(out);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride) {
        const float4 q = __ldcs(v4 + i);
        o4[i] = q8(q.x) | (q8(q.y) << 8) | (q8(q.z) << 16) | (q8(q.w) << 24);
    }
    if (blockIdx.x == 0)
        for (long long i = 4 * n4 + threadIdx.x; i < n; i += blockDim.x) out[i] = (uint8_t)q8(v[i]);
}

}  // namespace
}  // namespace pfa

extern "C" {

size_t pfa_display_workspace_bytes(void) { return sizeof(pfa::DispWs); }

pfa_status pfa_display_u8(const float *mag_dev, int64_t count, float percentile, void *workspace_dev, uint8_t *out_dev,
                          float *hi_dev, void *stream) {
    using namespace pfa;
    if (!mag_dev || !workspace_dev || !out_dev || count < 1) return PFA_ERR_BAD_ARG;
    if ((reinterpret_cast<uintptr_t>(mag_dev) & 15) || (reinterpret_cast<uintptr_t>(out_dev) & 3) ||
        (reinterpret_cast<uintptr_t>(workspace_dev) & 7))
        return PFA_ERR_BAD_ARG;
    if (!(percentile >= 0.0f && percentile <= 100.0f)) return PFA_ERR_BAD_ARG;
    // np.percentile's index arithmetic, float32 throughout (q = f32(pct) / f32(100), v = f32(n - 1) * q)
    volatile float q = percentile / 100.0f;
    volatile float vi = (float)(count - 1) * q;
    const float prev = floorf(vi);
    const bool top = vi >= (float)(count - 1);          // at or above the last index: the maximum
    const unsigned long long rank = top ? (unsigned long long)(count - 1) : (unsigned long long)prev;
    const float gamma = top ? 0.0f : (float)(vi - prev);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    DispWs *ws = static_cast<DispWs *>(workspace_dev);
    k_disp_init<<<1, 512, 0, st>>>(ws, rank);
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 4;
    const int shifts[3] = {21, 10, 0}, widths[3] = {11, 11, 10};
    for (int p = 0; p < 3; ++p) {
        k_disp_hist<<<blocks, 512, 0, st>>>(mag_dev, count, ws, shifts[p], widths[p]);
        k_disp_pick<<<1, 512, 0, st>>>(ws, widths[p], p == 2);
    }
    if (!top) k_disp_min_above<<<blocks, 512, 0, st>>>(mag_dev, count, ws);
    k_disp_hi<<<1, 1, 0, st>>>(ws, gamma, top ? 1 : 0, hi_dev);
    k_disp_quant<<<blocks * 2, 256, 0, st>>>(mag_dev, count, ws, out_dev);
    return cudaGetLastError() == cudaSuccess ? PFA_OK : PFA_ERR_CUDA;
}

}  // extern "C"
