// Internal plan state shared by the C-ABI glue and the kernel launchers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/pfa_b200.h"

namespace pfa {

// Device-resident fixed-point job + workspace for one (m, n, G) frame.
struct FixedDev {
    int m = 0, n = 0, G = 0, L = 0, mpad = 0;
    int range_sinc = 0, az_sinc = 0;
    int range_cubic = 0, az_cubic = 0;      // 4-tap Lagrange variant (sinc flags off)
    int fused_detect = 0;                   // silicon detect order
    // job vectors (device)
    float *f0 = nullptr, *df = nullptr, *fac = nullptr, *tan_s = nullptr;
    float *krp = nullptr, *kcp = nullptr;
    int32_t *order = nullptr;          // sorted slot -> pulse index
    int32_t *hamr = nullptr, *hamc = nullptr;
    uint32_t *tw = nullptr;            // stage-contiguous twiddles, G-1 packed int16x2
    int16_t *sinc = nullptr;           // 256 x 32
    // workspace (device)
    uint32_t *p1 = nullptr;            // [n][mpad] pass-1 output, packed int16x2
    uint32_t *y1 = nullptr;            // [n][G] FFT-1 output (range-bin rows)
    uint32_t *y2 = nullptr;            // [G][G] FFT-2 output (cross-bin rows)
    int32_t *e1 = nullptr;             // [G]
    int32_t *e2 = nullptr;             // [G]
    int32_t *ctrl = nullptr;           // [0] q0 max bits, [1] emax1, [2] emax2, [3] q0 exponent
    void *job_block = nullptr;         // the job vectors above (f0 .. sinc) in one allocation
    size_t job_bytes = 0;
};

struct FloatDev {
    int m = 0, n = 0, m2 = 0, n2 = 0, Lm = 0, Ln = 0, mpad = 0, npad = 0;
    int range_sinc = 0, az_sinc = 0, sgn = -1, layout = 0;
    double *f0 = nullptr, *df = nullptr, *flast = nullptr, *pr = nullptr, *tan_s = nullptr, *kr = nullptr, *kc = nullptr;
    float *ham_m = nullptr, *ham_n = nullptr;   // unused when window is off
    double *ham_m64 = nullptr, *ham_n64 = nullptr;
    int32_t *order = nullptr;
    float2 *twm = nullptr, *twn = nullptr;      // stage-contiguous twiddles for m2 and n2
    int16_t *tabq = nullptr;                    // sinc table (Q15 taps), [phase][tap] rows of 40 int16
    bool consts_ready = false;                  // twm, twn and tabq (plan constants) uploaded
    int window = 1;
    float2 *p1 = nullptr;              // [n][mpad] pass-1 output (range-bin rows, sorted pulses)
    CUtensorMap p1_map;                // TMA map of p1: 8-byte elements, boxes of 256 x 1
    float2 *y1 = nullptr;              // [m2][npad] cross FFT output, transposed (cross-bin rows)
    int ept_cross = 0, ept_range = 0;    // FFT register tile (complex values per thread; 0 = automatic)
    float2 *af_zadj = nullptr;         // [n][m2] autofocus: adjoint of the range FFT (range-bin rows)
    double *af_acc = nullptr;          // [2] sum I, sum I log I
    float *af_dacc = nullptr;          // [mpad] per-slot gradient accumulators
    uint32_t *af_pk = nullptr;         // [n][m] autofocus: packed pass-2 brackets of the forward pass
    uint32_t *pk_out = nullptr;        // where pass 2 stores its packed brackets for the adjoint (or nullptr)
    float2 *af_rp = nullptr;           // [n][m] autofocus, float-sinc plans: the forward's resampled rows R2 p1
    float2 *rp_out = nullptr;          // where a float-sinc pass 2 stores R2 p1 for the adjoint (or nullptr)
    // split-precision (mixed) mode: tensor-core FFTs for lines of 2048..8192 points
    int mixed = 0;
    uint4 *mx_f128 = nullptr;          // F_128 TMEM image [128 lanes][256 columns] of fp16 pairs
    uint4 *mx_fn2m = nullptr, *mx_fn2n = nullptr;   // F_{m2/128}, F_{n2/128} shared-memory images
    int *wait_err = nullptr;           // device flag: a bounded wait ran out (TMA row load, tensor-core completion)
    int mx_clusters = 0;               // resident 4-CTA clusters of the mixed pass 2
    int mx_probe = 0;                  // test hook: polls of a wait on an unarmed barrier (FP32: pass 2's
                                       // row load; mixed: the tensor-core range FFT)
    int sms = 0;                       // SM count of the plan's device
};

}  // namespace pfa

namespace pfa {
// Stage events recorded between kernels when profiling is on.
struct StageProf {
    static constexpr int kMax = 12;
    bool on = false;
    int count = 0;                      // events recorded in the last frame
    cudaEvent_t ev[kMax] = {};
    const char *names[kMax] = {};
    cudaError_t mark(cudaStream_t st, const char *name) {
        if (!on || count >= kMax) return cudaSuccess;
        names[count] = name;
        return cudaEventRecord(ev[count++], st);
    }
};
}  // namespace pfa

struct pfa_plan {
    pfa_config cfg{};
    int device = 0;
    bool job_ready = false;
    size_t ws_bytes = 0;
    pfa::FixedDev fx;
    pfa::FloatDev fl;
    float *staging_in = nullptr;       // device copy of the host signal (host entry points)
    void *staging_out = nullptr;
    size_t staging_in_bytes = 0, staging_out_bytes = 0;
    cudaStream_t host_stream = nullptr;
    // pipelined host frames: upload / compute / download streams, double-buffered staging
    cudaStream_t pipe_up = nullptr, pipe_comp = nullptr, pipe_down = nullptr;
    void *pipe_in[2] = {nullptr, nullptr}, *pipe_out[2] = {nullptr, nullptr};
    size_t pipe_in_bytes = 0, pipe_out_bytes = 0;
    cudaEvent_t pipe_ev[6] = {};      // uploaded[2], computed[2], downloaded[2]
    // fixed job staging: the host image of FixedDev::job_block (one upload per job) and the inputs the
    // grid-dependent tables were last derived from (rebuilt only when those change)
    std::vector<unsigned char> job_host;
    std::vector<int16_t> last_tw_in, last_sinc_in;
    int last_tw_builtin = -1, last_sinc_builtin = -1;
    pfa::StageProf prof;
    std::string err;
};

namespace pfa {

// Kernel launchers (pfa_fixed.cu / pfa_float.cu). They return a cudaError_t from the launches.
cudaError_t fixed_form(const FixedDev &d, const float *sig_c64, const uint32_t *sig_iq, uint16_t *img,
                       cudaStream_t st, StageProf *prof);
size_t fixed_workspace_bytes(int m, int n, int G);
cudaError_t fixed_alloc(FixedDev &d, int m, int n, int G);
void fixed_free(FixedDev &d);

// theta (device, [m], or nullptr): per-pulse phase correction exp(-j theta_i) applied in pass 1
cudaError_t float_form(const FloatDev &d, const float2 *sig, void *out, int detect, cudaStream_t st,
                       StageProf *prof, const float *theta = nullptr);
size_t float_workspace_bytes(int m, int n);
cudaError_t float_alloc(FloatDev &d, int m, int n);
void float_free(FloatDev &d);

// Split-precision tensor-core FFT mode (pfa_mixed.cu).
bool mixed_axis(int L);                                  // 2^L-point lines run on the tensor cores
cudaError_t mixed_prepare(FloatDev &d);                  // tables, SM/cluster occupancy (plan creation)
void mixed_free(FloatDev &d);
cudaError_t mixed_pass2(const FloatDev &d, cudaStream_t st);
cudaError_t mixed_fft2(const FloatDev &d, void *out, int detect, float scale, cudaStream_t st);

// Pipelined host frames (pfa_capi.cu): form(plan, in_dev, out_dev, stream, arg) runs one frame.
typedef pfa_status (*FrameFn)(pfa_plan *p, const void *in_dev, void *out_dev, cudaStream_t st, int32_t arg);
pfa_status run_host_frames(pfa_plan *p, const void *const *ins, void *const *outs, int32_t nframes, size_t in_bytes,
                           size_t out_bytes, FrameFn form, int32_t arg);

// Host-side table builders used when the caller passes NULL for a table (libm based).
void build_sinc_table(int16_t *tab);   // table from the exact-rational recipe, [phase][tap]
// True when every phase of a [phase][tap] Q15 table has sum |tap| <= 65535 over taps 0-15 and over
// taps 16-31: the condition for the fixed-point sinc's int32 half-sum accumulation to be exact.
bool sinc_table_fits_int32(const int16_t *tab);
void build_twiddles_q15(int G, int16_t *tw2);   // [G/2][2]
void build_hamming_q15(int len, int size, int32_t *out);

}  // namespace pfa
