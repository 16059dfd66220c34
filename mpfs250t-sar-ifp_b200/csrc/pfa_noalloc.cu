// pfa_form_fixed_noalloc: the fixed-point frame former without any allocation.
//
// Some callers cannot allocate device memory: hosts that own every byte of device memory through their
// own pool, real-time loops that must never enter the allocator, processes whose allocator is already
// exhausted.  This entry point serves them.  Its scratch -- the uploaded job vectors, the derived
// tables and the three intermediate frames -- is one file-scope static __device__ array sized for the
// largest frame it accepts (grid 1024: 12.1 MB, held by every GPU that loads the library until exit).
//
// Host code must not pass the array's name to a kernel: on the host that name is only a stand-in
// symbol, not a device address.  Every call looks the device address up with cudaGetSymbolAddress (the
// call's device current).  The first lookup on a device loads the module there; later ones are cheap and
// never stale, also after a device reset reloaded the module.  The same kernels as the planned path
// (pfa_fixed.cu) run on a FixedDev view whose pointers point into the array.
//
// The job vectors are copied host-to-device with cudaMemcpyAsync on the caller's stream.  From pinned
// host memory those copies are truly asynchronous, so the job arrays (and sinc_q15) must stay valid and
// unchanged until the stream has reached this call's work, the contract of any asynchronous copy.
//
// All calls share the array and it keeps the previous call's contents.  What must start at zero (the
// reduction words) is cleared by every call; everything else is fully rewritten before it is read.
// Calls that overlap on the GPU race on the array.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "pfa_internal.h"

namespace pfa {
const int16_t *builtin_sinc_table();
}

namespace {

constexpr int kMaxGrid = 1024;

constexpr size_t align256(size_t v) { return (v + 255) / 256 * 256; }

// Fixed byte layout of the static scratch, sized for the maximum grid.
struct NoAllocLayout {
    static constexpr size_t G = kMaxGrid, M = kMaxGrid, N = kMaxGrid;
    static constexpr size_t f0 = 0;
    static constexpr size_t df = f0 + align256(4 * M);
    static constexpr size_t pr = df + align256(4 * M);
    static constexpr size_t fac = pr + align256(4 * M);
    static constexpr size_t tan_s = fac + align256(4 * M);
    static constexpr size_t inv_order = tan_s + align256(4 * M);
    static constexpr size_t order = inv_order + align256(4 * M);
    static constexpr size_t krp = order + align256(4 * M);
    static constexpr size_t kcp = krp + align256(4 * G);
    static constexpr size_t hamr = kcp + align256(4 * G);
    static constexpr size_t hamc = hamr + align256(4 * G);
    static constexpr size_t tw_raw = hamc + align256(4 * G);
    static constexpr size_t tw = tw_raw + align256(2 * G);
    static constexpr size_t sinc = tw + align256(4 * G);
    static constexpr size_t sinc_raw = sinc + align256(2 * 256 * 32);
    static constexpr size_t e1 = sinc_raw + align256(2 * 256 * 32);
    static constexpr size_t e2 = e1 + align256(4 * G);
    static constexpr size_t ctrl = e2 + align256(4 * G);
    static constexpr size_t p1 = ctrl + align256(4 * 16);
    static constexpr size_t y1 = p1 + align256(4 * N * M);
    static constexpr size_t y2 = y1 + align256(4 * N * G);
    static constexpr size_t total = y2 + align256(4 * G * G);
};

// The scratch itself.  Only device code may name it directly; host code uses the looked-up address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NoAllocLayout::total];

// Derived job vectors: the pass-1 source scale f32(f32(2 pr) / f32(c)), the slot -> pulse order and the
// stage-contiguous twiddle table (stage b at offset 2^b - 1, entry k = raw[k << (L-1-b)]).
__global__ void k_noalloc_prep(const float *__restrict__ pr, const int32_t *__restrict__ inv_order,
                               const int16_t *__restrict__ tw_raw, const int16_t *__restrict__ sinc_raw,
                               float *__restrict__ fac, int32_t *__restrict__ order, uint32_t *__restrict__ tw,
                               int16_t *__restrict__ sinc, int m, int G, int L) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 256 * 32) sinc[(i & 31) * 256 + (i >> 5)] = sinc_raw[i];    // [phase][tap] -> [tap][phase]
    if (i < m) {
        fac[i] = __fdiv_rn(__fmul_rn(2.0f, pr[i]), 299792458.0f);
        order[inv_order[i]] = i;   // inv_order was checked to be a permutation on the host
    }
    if (i < G - 1) {
        const int b = 31 - __clz(i + 1);
        const int k = i + 1 - (1 << b);
        const int src = k << (L - 1 - b);
        tw[i] = (uint32_t)(uint16_t)tw_raw[2 * src] | ((uint32_t)(uint16_t)tw_raw[2 * src + 1] << 16);
    }
}

bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

}  // namespace

extern "C" pfa_status pfa_form_fixed_noalloc(const pfa_config *cfg, const pfa_fixed_job *job, const float *sig_dev,
                                             uint16_t *img_dev, void *stream) {
    if (!cfg || !job || !sig_dev || !img_dev) return PFA_ERR_BAD_ARG;
    if ((reinterpret_cast<uintptr_t>(sig_dev) & 15) || (reinterpret_cast<uintptr_t>(img_dev) & 3)) return PFA_ERR_BAD_ARG;
    const pfa_config c = *cfg;
    if (c.mode != PFA_MODE_FIXED) return PFA_ERR_BAD_CONFIG;
    if ((c.range_interp != PFA_INTERP_LERP && c.range_interp != PFA_INTERP_SINC && c.range_interp != PFA_INTERP_CUBIC) ||
        (c.az_interp != PFA_INTERP_LERP && c.az_interp != PFA_INTERP_SINC && c.az_interp != PFA_INTERP_CUBIC) ||
        (c.detect_order != PFA_DETECT_ORDER_EMULATOR && c.detect_order != PFA_DETECT_ORDER_FUSED))
        return PFA_ERR_BAD_CONFIG;
    if (c.m < 2 || c.n < 2 || c.grid < c.m || c.grid < c.n) return PFA_ERR_BAD_DIMS;
    if (c.grid > kMaxGrid) {
        std::fprintf(stderr, "pfa_form_fixed_noalloc: grid %d exceeds the static scratch limit %d\n", c.grid, kMaxGrid);
        return PFA_ERR_TOO_LARGE;
    }
    if (!is_pow2(c.grid) || c.grid < 64) return PFA_ERR_BAD_CONFIG;
    if (!job->f0 || !job->df || !job->pr || !job->tan_s || !job->inv_order || !job->kr_grid || !job->kc_grid ||
        !job->ham_r || !job->ham_c || !job->twiddle)
        return PFA_ERR_BAD_ARG;
    // inv_order must be a permutation (it drives row indexing); checked with a stack bitmap
    uint32_t seen[kMaxGrid / 32] = {};
    for (int i = 0; i < c.m; ++i) {
        const int r = job->inv_order[i];
        if (r < 0 || r >= c.m || (seen[r >> 5] >> (r & 31)) & 1u) return PFA_ERR_BAD_ARG;
        seen[r >> 5] |= 1u << (r & 31);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || c.device < 0 || c.device >= ndev) return PFA_ERR_NO_DEVICE;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return PFA_ERR_NO_DEVICE;
    if (prev != c.device && cudaSetDevice(c.device) != cudaSuccess) return PFA_ERR_NO_DEVICE;
    struct Restore {
        int prev, dev;
        ~Restore() { if (prev != dev) cudaSetDevice(prev); }
    } restore{prev, c.device};

    // set-up, on every call with the device current: the device address of the static scratch
    void *addr = nullptr;
    const cudaError_t ea = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (ea != cudaSuccess || !addr) return PFA_ERR_CUDA;
    unsigned char *base = static_cast<unsigned char *>(addr);
    using Lt = NoAllocLayout;
    const int m = c.m, n = c.n, G = c.grid;
    int L = 0;
    while ((1 << L) < G) ++L;
    pfa::FixedDev d;
    d.m = m; d.n = n; d.G = G; d.L = L; d.mpad = (m + 31) / 32 * 32;
    d.range_sinc = c.range_interp == PFA_INTERP_SINC;
    d.az_sinc = c.az_interp == PFA_INTERP_SINC;
    d.range_cubic = c.range_interp == PFA_INTERP_CUBIC;
    d.az_cubic = c.az_interp == PFA_INTERP_CUBIC;
    d.fused_detect = c.detect_order == PFA_DETECT_ORDER_FUSED;
    d.f0 = reinterpret_cast<float *>(base + Lt::f0);
    d.df = reinterpret_cast<float *>(base + Lt::df);
    d.fac = reinterpret_cast<float *>(base + Lt::fac);
    d.tan_s = reinterpret_cast<float *>(base + Lt::tan_s);
    d.order = reinterpret_cast<int32_t *>(base + Lt::order);
    d.krp = reinterpret_cast<float *>(base + Lt::krp);
    d.kcp = reinterpret_cast<float *>(base + Lt::kcp);
    d.hamr = reinterpret_cast<int32_t *>(base + Lt::hamr);
    d.hamc = reinterpret_cast<int32_t *>(base + Lt::hamc);
    d.tw = reinterpret_cast<uint32_t *>(base + Lt::tw);
    d.sinc = reinterpret_cast<int16_t *>(base + Lt::sinc);
    d.p1 = reinterpret_cast<uint32_t *>(base + Lt::p1);
    d.y1 = reinterpret_cast<uint32_t *>(base + Lt::y1);
    d.y2 = reinterpret_cast<uint32_t *>(base + Lt::y2);
    d.e1 = reinterpret_cast<int32_t *>(base + Lt::e1);
    d.e2 = reinterpret_cast<int32_t *>(base + Lt::e2);
    d.ctrl = reinterpret_cast<int32_t *>(base + Lt::ctrl);
    float *pr = reinterpret_cast<float *>(base + Lt::pr);
    int32_t *inv = reinterpret_cast<int32_t *>(base + Lt::inv_order);
    int16_t *tw_raw = reinterpret_cast<int16_t *>(base + Lt::tw_raw);
    int16_t *sinc_raw = reinterpret_cast<int16_t *>(base + Lt::sinc_raw);

    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int16_t *sinc = job->sinc_q15 ? job->sinc_q15 : pfa::builtin_sinc_table();
    if (!pfa::sinc_table_fits_int32(sinc)) return PFA_ERR_BAD_ARG;
    struct Cp { void *dst; const void *src; size_t bytes; } cps[] = {
        {d.f0, job->f0, 4u * m}, {d.df, job->df, 4u * m}, {pr, job->pr, 4u * m}, {d.tan_s, job->tan_s, 4u * m},
        {inv, job->inv_order, 4u * m}, {d.krp, job->kr_grid, 4u * G}, {d.kcp, job->kc_grid, 4u * G},
        {d.hamr, job->ham_r, 4u * G}, {d.hamc, job->ham_c, 4u * G}, {tw_raw, job->twiddle, 2u * G},
        {sinc_raw, sinc, 2u * 256 * 32}};
    for (const Cp &cp : cps) {
        if (cudaMemcpyAsync(cp.dst, cp.src, cp.bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) return PFA_ERR_CUDA;
    }
    int nthreads = (G - 1 > m ? G - 1 : m);
    if (nthreads < 256 * 32) nthreads = 256 * 32;
    k_noalloc_prep<<<(nthreads + 255) / 256, 256, 0, st>>>(pr, inv, tw_raw, sinc_raw, d.fac, d.order, d.tw, d.sinc,
                                                           m, G, L);
    if (cudaGetLastError() != cudaSuccess) return PFA_ERR_CUDA;
    // fixed_form clears the reduction words (ctrl) itself before its first kernel
    if (pfa::fixed_form(d, sig_dev, nullptr, img_dev, st, nullptr) != cudaSuccess) return PFA_ERR_CUDA;
    return PFA_OK;
}
