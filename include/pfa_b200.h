/*
 * pfa_b200.h -- C ABI of the B200 Polar Format Algorithm (PFA) focusing engine.
 *
 * The engine replaces the focusing datapath of the reference SAR image former:
 *
 *   fixed point  -> the body of silicon_emulator.form_image() after the CPHD read
 *                   (mpfs/host/silicon_emulator.py:226-249): Q0 int16 quantise, resample_fixed
 *                   (:125-156), window_fixed (:165-195), fft_pass_bfp x2 with corner turns
 *                   (:198-205, :241-247), detect_fixed (:208-213).  Bit-exact: same uint16 image,
 *                   same CRC-32.
 *   float        -> form_image_pfa.resample_kspace + focus + |.| (src/form_image_pfa.py:165-246,
 *                   mpfs/host/accel.py:39-44), i.e. AccelBackend.focus(signal, tables).
 *
 * It stands where the board ABI sar_form_image(spin_limit) -> sar_seq_status_t stands
 * (mpfs/fpga/libero_sar/softconsole/mpfs-hal-ddr-demo/src/sar/sar_sequencer.c:1432, status enum
 * sar_sequencer.h:19-27): the job vectors below are the board's staged job (the 10-role DDR format of
 * mpfs/host/serialize_inputs.py:1-30, with the emulator's floor tapers), and every call returns a
 * status code instead of raising.
 *
 * Conventions: plain pointers and sizes; "dev" pointers are CUDA device pointers, "host" pointers are
 * host memory; `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).  Calls on one
 * plan are not thread-safe; distinct plans are independent.  All launches are stream-ordered and
 * asynchronous unless the name ends in _host.
 */
#ifndef PFA_B200_H
#define PFA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes, modelled on sar_seq_status_t (sar_sequencer.h:19-27). */
typedef enum pfa_status {
    PFA_OK = 0,
    PFA_ERR_BAD_CONFIG = 1,   /* unsupported mode/grid/interp combination                       */
    PFA_ERR_BAD_DIMS = 2,     /* grid smaller than the scene (standalone_emulator_README.md:90-95) */
    PFA_ERR_BAD_ARG = 3,      /* NULL or misaligned pointer, bad size                            */
    PFA_ERR_NOT_READY = 4,    /* job vectors not set before a form call                          */
    PFA_ERR_CUDA = 5,         /* CUDA runtime error (message in pfa_last_error)                  */
    PFA_ERR_ALLOC = 6,        /* device allocation failed                                        */
    PFA_ERR_TIMEOUT = 7,      /* a bounded wait ran out                                          */
    PFA_ERR_NO_DEVICE = 8,    /* no usable sm_100 device                                         */
    PFA_ERR_TOO_LARGE = 9     /* frame larger than pfa_form_fixed_noalloc's static scratch allows */
} pfa_status;

enum pfa_mode { PFA_MODE_FIXED = 0, PFA_MODE_FLOAT32 = 1, PFA_MODE_MIXED = 2 };
/* Resampler of a pass.  CUBIC (fixed mode only) is the 4-tap Lagrange interpolator of the RTL vector
 * generator (gen_resample_vectors.gather_cubic, mpfs/fpga/tb/gen_resample_vectors.py:177-195, 298-325),
 * offered for A/B comparison with board captures; its edge brackets use the integer 2-tap lerp. */
enum pfa_interp { PFA_INTERP_LERP = 0, PFA_INTERP_SINC = 1, PFA_INTERP_CUBIC = 2 };

/* Fixed-mode detection order.  EMULATOR: global renorm (>> (emax - e_row), int16) then integer |z|, as
 * silicon_emulator.form_image (mpfs/host/silicon_emulator.py:247-249).  FUSED: |z| at the row's native
 * exponent, then the magnitude shifted (model_detect_fusion.order_B_fused, mpfs/host/
 * model_detect_fusion.py:56-71): the silicon order when detect is fused into the FFT unloader. */
enum pfa_detect_order { PFA_DETECT_ORDER_EMULATOR = 0, PFA_DETECT_ORDER_FUSED = 1 };

/* Output layout of the float path. */
enum pfa_layout {
    PFA_LAYOUT_CENTRED = 0,   /* fftshift(fft2(ifftshift(pad))): (m2 rows = cross, n2 cols = range), form_image_pfa */
    PFA_LAYOUT_NATURAL = 1    /* fft2(pad) without shifts                                            */
};

/* What the float path writes. */
enum pfa_detect {
    PFA_DETECT_MAG = 0,       /* float32 |z|   (accel.NumpyBackend.focus)  */
    PFA_DETECT_POWER = 1,     /* float32 |z|^2                            */
    PFA_DETECT_COMPLEX = 2    /* complex64 z                              */
};

typedef struct pfa_config {
    int32_t mode;          /* pfa_mode                                                      */
    int32_t m;             /* pulses after decimation                                       */
    int32_t n;             /* samples per pulse after decimation                            */
    int32_t grid;          /* fixed: square output grid G (pow2, 64..16384, >= m and n)      */
                           /* float: 0 = pow2(m) x pow2(n) as form_image_pfa.focus           */
    int32_t range_interp;  /* pfa_interp for pass 1 (--range-sinc)                          */
    int32_t az_interp;     /* pfa_interp for pass 2 (--az-sinc)                             */
    int32_t device;        /* CUDA device ordinal                                           */
    int32_t fft_ept_cross; /* float: complex values per thread in the cross FFT (8, 16 or 32;
                              0 = automatic: 16; 8 applies to lines of 256..8192 points and 32 to
                              lines of 8192 and 16384, other lines use 16), i.e. CTA size
                              pow2(m)/ept -- the tile shape the autotuner picks                 */
    int32_t fft_ept_range; /* float: same for the range FFT (pow2(n)/ept threads; 0 = automatic:
                              32 for lines of 8192 and 16384 points, else 16)                    */
    int32_t detect_order;  /* fixed: pfa_detect_order (0 = emulator order)                      */
    int32_t test_wait_polls; /* test hook, 0 in normal use.  > 0: a bounded wait first waits this many
                              polls on a barrier nothing arrives on, so its timeout path runs --
                              FP32 mode: the cross pass's TMA row load (rows are not used); mixed
                              mode: the tensor-core range FFT (no MMA is issued).  The frame is
                              zeros and the synchronous entry points return PFA_ERR_TIMEOUT      */
    int32_t reserved[5];
} pfa_config;

/* Fixed-point job: host pointers, copied at pfa_set_fixed_job.  Built exactly as
 * silicon_emulator.resample_fixed/window_fixed build them (silicon_emulator.py:131-141, 185-188). */
typedef struct pfa_fixed_job {
    const float *f0;          /* [m]   freq[:,0] as float32                                     */
    const float *df;          /* [m]   (freq[:,1]-freq[:,0]) as float32                          */
    const float *pr;          /* [m]   radial projection as float32                              */
    const float *tan_s;       /* [m]   tan(phi) sorted ascending, float32                        */
    const int32_t *inv_order; /* [m]   pass-1 destination slot of pulse i (argsort(argsort(tan_phi))) */
    const float *kr_grid;     /* [G]   KR padded with the out-of-span sentinel                   */
    const float *kc_grid;     /* [G]   KC padded with the out-of-span sentinel                   */
    const int32_t *ham_r;     /* [G]   floor(hamming(n)*32768), zero pad; NULL = built in        */
    const int32_t *ham_c;     /* [G]   floor(hamming(m)*32768), zero pad; NULL = built in        */
    const int16_t *twiddle;   /* [G/2][2] floor(exp(-2pi j k/G)*32768) clipped; NULL = built in  */
    const int16_t *sinc_q15;  /* [256][32] polyphase table; NULL = built in                     */
} pfa_fixed_job;

/* Float job: host pointers, copied at pfa_set_float_job.  Mirrors form_image_pfa.resample_kspace
 * (src/form_image_pfa.py:177-217); freq[i,k] = f0[i] + k*df[i]. */
typedef struct pfa_float_job {
    const double *f0;         /* [m] freq[:, 0]                                                   */
    const double *df;         /* [m] frequency step along the pulse                               */
    const double *f_last;     /* [m] freq[:, n-1]: the end points' wavenumbers (2 f / c) pr are
                                 evaluated exactly as the reference does, since the output grid
                                 KR starts and ends exactly on one pulse's end points               */
    const double *pr;         /* [m] radial projection                                          */
    const double *tan_s;      /* [m] tan(phi) sorted ascending                                   */
    const int32_t *order;     /* [m] argsort(tan_phi)                                            */
    const double *kr_grid;    /* [n] KR                                                          */
    const double *kc_grid;    /* [m] KC                                                          */
    const double *ham_m;      /* [m] hamming(m); NULL = no window                               */
    const double *ham_n;      /* [n] hamming(n); NULL = no window                               */
    int32_t sgn;              /* CPHD SGN: -1 forward FFT, +1 inverse (with 1/(m2 n2))            */
    int32_t layout;           /* pfa_layout                                                      */
} pfa_float_job;

typedef struct pfa_plan pfa_plan;

/* Plan lifetime.  Allocates the device workspace for one frame of the configured shape.
 * Replaces: allocation of the emulator's (grid x grid) intermediates (silicon_emulator.py:153, 233-247). */
pfa_status pfa_plan_create(const pfa_config *cfg, pfa_plan **out);
pfa_status pfa_plan_destroy(pfa_plan *plan);
/* Device bytes held by the plan's workspace. */
size_t pfa_plan_workspace_bytes(const pfa_plan *plan);

/* Job upload.  Replaces: the geometry block of resample_fixed (silicon_emulator.py:131-141) and the
 * taper build of window_fixed (:185-188) / serialize_inputs.serialize (:206-225). */
pfa_status pfa_set_fixed_job(pfa_plan *plan, const pfa_fixed_job *job);
/* Replaces: the geometry block of form_image_pfa.resample_kspace (src/form_image_pfa.py:177-211). */
pfa_status pfa_set_float_job(pfa_plan *plan, const pfa_float_job *job);

/* Fixed-point frame from the complex64 phase history (m x n, interleaved re/im float32, device).
 * Replaces: silicon_emulator.form_image lines :226-249 (Q0 quantise .. detect_fixed).
 * img_dev: uint16 [G][G], rows = range bins, cols = cross bins (the emulator's natural order).
 * sig_dev must be 16-byte aligned, img_dev 4-byte aligned (PFA_ERR_BAD_ARG otherwise). */
pfa_status pfa_form_fixed(pfa_plan *plan, const float *sig_dev, uint16_t *img_dev, void *stream);
/* Same, from an already quantised int16 I/Q signal (m x n x 2, device): the board's sig.bin
 * (serialize_inputs.py:1-30, ddr_layout.quantize_iq16).  Replaces :233-249. */
pfa_status pfa_form_fixed_iq16(pfa_plan *plan, const int16_t *sig_iq_dev, uint16_t *img_dev, void *stream);
/* End-to-end host variant: copies the host signal in, forms, copies the image out, synchronises. */
pfa_status pfa_form_fixed_host(pfa_plan *plan, const float *sig_host, uint16_t *img_host);

/* Pipelined end-to-end frames from host memory, the counterpart of the reference's scene queue
 * (sar_pipeline.watch -> process_scene, mpfs/host/sar_pipeline.py:118-163): nframes host signals in,
 * nframes host images out.  Device staging is double buffered and uploads, frames and downloads run on
 * three streams, so frame k+1's upload and frame k-1's download overlap frame k.  All frames share the
 * plan's job (geometry).  Host buffers should be pinned for full PCIe bandwidth.  Synchronises. */
pfa_status pfa_form_fixed_host_frames(pfa_plan *plan, const float *const *sig_hosts, uint16_t *const *img_hosts,
                                      int32_t nframes);
pfa_status pfa_form_float_host_frames(pfa_plan *plan, const float *const *sig_hosts, void *const *out_hosts,
                                      int32_t detect, int32_t nframes);

/* Allocation-free fixed-point frame, for callers that cannot allocate device memory: code running
 * where cudaMalloc is forbidden or unsafe (inside a host that owns all device memory through its own
 * pool, a real-time loop that must not hit the allocator, or a process whose allocator is already
 * exhausted).  No counterpart in the reference (its board code uses fixed DDR buffers and never
 * allocates; this mirrors that property rather than any one function).
 * Everything the frame needs besides the caller's signal and image -- the job vectors and the three
 * intermediate frames -- lives in one file-scope static __device__ array of 12.1 MB that every GPU
 * which loads the library holds until the process exits.  Limits: grid <= 1024, otherwise
 * PFA_ERR_TOO_LARGE; m or n > grid gives PFA_ERR_BAD_DIMS.  job must carry ham_r, ham_c and twiddle (no
 * host-side table building); sinc_q15 may be NULL (built-in table).  The job vectors are copied to the
 * device with cudaMemcpyAsync on `stream`: like any asynchronous copy from (possibly pinned) host memory,
 * the job arrays and sinc_q15 must stay valid and unchanged until the stream has reached this call's work.
 * Every call looks up the array's device address (cudaGetSymbolAddress, with that device current); the
 * first call on a device also loads the library's device code there, so make that first call before any
 * stream capture.  All calls share the one array and it keeps the last call's contents: calls that overlap
 * on the GPU (different streams, threads or processes sharing a context) race and corrupt each other;
 * serialise them.  Calls no allocating routine: no cudaMalloc/cudaFree, no host heap. */
pfa_status pfa_form_fixed_noalloc(const pfa_config *cfg, const pfa_fixed_job *job, const float *sig_dev,
                                  uint16_t *img_dev, void *stream);

/* Per-row BFP exponents of the last fixed frame (silicon_emulator.fft_pass_bfp's `e`, :198-205):
 * e_range[n] (FFT-1 rows = range bins < n; rows >= n are all-zero and have exponent 0),
 * e_az[G] (FFT-2 rows = cross bins), q0_exp = the Q0 block exponent.  Host pointers; synchronises. */
pfa_status pfa_get_fixed_exponents(pfa_plan *plan, int32_t *e_range, int32_t *e_az, int32_t *q0_exp);

/* Float frame from the complex64 phase history (device).  out_dev: float32 [m2][n2] for
 * PFA_DETECT_MAG/POWER, complex64 [m2][n2] for PFA_DETECT_COMPLEX.
 * Replaces: accel.NumpyBackend.focus (mpfs/host/accel.py:39-44) / form_image_pfa.pfa (:243-246). */
pfa_status pfa_form_float(pfa_plan *plan, const float *sig_dev, void *out_dev, int32_t detect, void *stream);
pfa_status pfa_form_float_host(pfa_plan *plan, const float *sig_host, void *out_host, int32_t detect);

/* Image-entropy autofocus.  For the per-pulse phase correction theta[m] (float32, device) the plan
 * forms the float image of s[i,k] exp(-j theta_i) (the plan's lerp or float-sinc passes, window as set,
 * natural layout), its
 * entropy E = -sum p log p with p = |z|^2 / sum |z|^2, and dE/dtheta[m] with hand-written adjoint
 * kernels (range FFT recomputed, adjoint FFTs, window, transposed pass-2 resample -- lerp or 32-tap sinc --
 * as an atomics-free segmented reduction; descending source axes included).  entropy_dev (double,
 * device) may be NULL.  The first call on a plan adds its gradient workspace to the plan (12 n pow2(m)
 * bytes at most: the range-FFT adjoint and the packed pass-2 brackets; a float-sinc plan adds 8 n m
 * bytes for the forward's resampled rows), held until pfa_plan_destroy and not counted by
 * pfa_plan_workspace_bytes.  The reference has no autofocus; the image it forms is form_image_pfa.pfa
 * (src/form_image_pfa.py:243-246). */
pfa_status pfa_autofocus_grad(pfa_plan *plan, const float *sig_dev, const float *theta_dev, float *dtheta_dev,
                              double *entropy_dev, void *stream);

/* Display scaling of the detected float image, the quantiser of save_detected_geotiff
 * (src/form_image_pfa.py:287-292): hi = np.percentile(amp, percentile) and
 * out = uint8(clip(amp / (hi + 1e-12) * 255, 0, 255)), bit-exact to NumPy's float32 arithmetic, for
 * non-negative magnitudes amp (PFA_DETECT_MAG output).  mag_dev: float32 [count], 16-byte aligned;
 * out_dev: uint8 [count], 4-byte aligned; hi_dev (float32, device) may be NULL.  workspace_dev: at least
 * pfa_display_workspace_bytes() device bytes, 8-byte aligned, owned by the caller (no allocation, no host
 * synchronisation; calls sharing a workspace must not overlap).  The percentile is found by a radix select
 * over the float bit patterns on the device (three histogram passes plus one for the next order statistic).
 * The reference writes these bytes to its GeoTIFF; pfa_b200.geocode adds the map affine and the file. */
size_t pfa_display_workspace_bytes(void);
pfa_status pfa_display_u8(const float *mag_dev, int64_t count, float percentile, void *workspace_dev, uint8_t *out_dev,
                          float *hi_dev, void *stream);

/* Float frame of the phase-corrected signal s[i,k] exp(-j theta_i) (theta: float32 [m], device): the
 * correction is applied in pass 1, where it commutes with the per-pulse resample, so no corrected copy
 * of the signal is made.  Same outputs and rules as pfa_form_float; the image autofocus converges to. */
pfa_status pfa_form_float_phase(pfa_plan *plan, const float *sig_dev, const float *theta_dev, void *out_dev,
                                int32_t detect, void *stream);

/* One autofocus descent step on the device: the entropy gradient g of pfa_autofocus_grad, then
 * theta <- theta - step (g - mean g) / max |g - mean g| in place (the update pfa_b200.autofocus.autofocus
 * applies; a constant phase does not change the image).  theta_dev: float32 [m], device; entropy_dev
 * (double, device) may be NULL.  Stream-ordered, no host synchronisation: a loop of steps can be
 * captured in one CUDA graph. */
pfa_status pfa_autofocus_step(pfa_plan *plan, const float *sig_dev, float *theta_dev, float step, double *entropy_dev,
                              void *stream);

/* Per-stage device timing, the counterpart of the board's per-stage timestamps sar_stage_ts[]
 * (sar_sequencer.c:235-238) and form_image_pfa.StepTimer (src/form_image_pfa.py:42-60).  When enabled,
 * every form call records CUDA events between its kernels on the launching stream.
 * pfa_get_stage_times synchronises and writes up to `cap` stage durations (ms) of the last frame and
 * their names (comma separated) into names[names_len]; *count receives the number of stages. */
pfa_status pfa_set_profiling(pfa_plan *plan, int32_t enable);
pfa_status pfa_get_stage_times(pfa_plan *plan, float *ms, int32_t cap, int32_t *count, char *names, size_t names_len);

/* Diagnostics. */
const char *pfa_status_string(pfa_status st);
pfa_status pfa_last_error(const pfa_plan *plan, char *buf, size_t len);
/* Library version string. */
const char *pfa_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PFA_B200_H */
