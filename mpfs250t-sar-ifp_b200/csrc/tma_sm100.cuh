// TMA loads for sm_100a: 2-D tiled tensor copies and plain bulk copies from this GPU's global memory into
// the issuing CTA's shared memory, completing on an mbarrier by transaction bytes, and the host-side
// encoder of the tensor maps (cuTensorMapEncodeTiled reached through the runtime's driver entry point,
// so the library does not link against libcuda).
//
// Rules the callers keep: the global base is 16-byte aligned, row strides are multiples of 16 bytes, the
// innermost box extent times the element size is a multiple of 16 bytes, every inner coordinate x of a
// copy times the element size is a multiple of 16 bytes, and shared-memory destinations are 128-byte
// aligned.  Waits are bounded (tc::mbar_wait).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace pfa {
namespace tma {

__device__ __forceinline__ uint32_t saddr(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// One arrival on `bar` that also raises its expected transaction count by `bytes`.
__device__ __forceinline__ void arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}

// box of `map` at (x, y) -> shared memory `dst`; the box's bytes complete on `bar` (out-of-range elements
// arrive as zeros and count too)
__device__ __forceinline__ void load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
            saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(saddr(bar))
        : "memory");
}

// `bytes` (a multiple of 16, both addresses 16-byte aligned) from global `src` -> shared `dst`
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     saddr(dst)),
                 "l"(src), "r"(bytes), "r"(saddr(bar))
                 : "memory");
}

// Row-major 2-D tensor map over `rows` rows of `cols` elements of `elem_bytes` each, `pitch_bytes` apart;
// boxes of box_cols x box_rows elements, no swizzle, zero fill outside the tensor.
inline cudaError_t encode_2d(CUtensorMap *map, const void *base, int elem_bytes, uint64_t cols, uint64_t rows,
                             uint64_t pitch_bytes, uint32_t box_cols, uint32_t box_rows) {
    using Encode = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Encode encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        const cudaError_t e = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q);
        if (e != cudaSuccess) return e;
        if (q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;   // driver without TMA maps
        encode = reinterpret_cast<Encode>(fn);
    }
    CUtensorMapDataType dt;
    switch (elem_bytes) {
        case 2: dt = CU_TENSOR_MAP_DATA_TYPE_UINT16; break;
        case 4: dt = CU_TENSOR_MAP_DATA_TYPE_UINT32; break;
        case 8: dt = CU_TENSOR_MAP_DATA_TYPE_UINT64; break;
        default: return cudaErrorNotSupported;
    }
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (pitch_bytes & 15) || ((box_cols * (uint32_t)elem_bytes) & 15) ||
        box_cols == 0 || box_cols > 256 || box_rows == 0 || box_rows > 256)
        return cudaErrorNotSupported;
    const cuuint64_t dims[2] = {cols, rows};
    const cuuint64_t strides[1] = {pitch_bytes};
    const cuuint32_t box[2] = {box_cols, box_rows};
    const cuuint32_t estride[2] = {1, 1};
    const CUresult r = encode(map, dt, 2, const_cast<void *>(base), dims, strides, box, estride,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorNotSupported;
}

}  // namespace tma
}  // namespace pfa
