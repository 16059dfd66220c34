// Float PFA datapath (FP32 and split-precision) -- placeholder until the float kernels land.
#include <cuda_runtime.h>

#include "pfa_internal.h"

namespace pfa {
size_t float_workspace_bytes(int, int) { return 0; }
cudaError_t float_alloc(FloatDev &, int, int) { return cudaErrorInvalidValue; }
void float_free(FloatDev &) {}
cudaError_t float_form(const FloatDev &, const float2 *, void *, int, cudaStream_t, StageProf *) { return cudaErrorNotSupported; }
}  // namespace pfa

extern "C" {
pfa_status pfa_set_float_job(pfa_plan *p, const pfa_float_job *) { return p ? PFA_ERR_BAD_CONFIG : PFA_ERR_BAD_ARG; }
pfa_status pfa_form_float(pfa_plan *p, const float *, void *, int32_t, void *) { return p ? PFA_ERR_BAD_CONFIG : PFA_ERR_BAD_ARG; }
pfa_status pfa_form_float_host(pfa_plan *p, const float *, void *, int32_t) { return p ? PFA_ERR_BAD_CONFIG : PFA_ERR_BAD_ARG; }
}
