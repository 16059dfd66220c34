// C ABI of the PFA engine: plan lifecycle, job upload, frame entry points, diagnostics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "pfa_internal.h"

namespace pfa {
#include "gen/sinc_q15.inc"   // kSincQ15[256 * 32], generated at build time by the exact-rational recipe

void build_sinc_table(int16_t *tab) { std::memcpy(tab, kSincQ15, sizeof(kSincQ15)); }
const int16_t *builtin_sinc_table() { return kSincQ15; }
bool sinc_table_fits_int32(const int16_t *tab) {
    for (int ph = 0; ph < 256; ++ph)
        for (int h = 0; h < 2; ++h) {
            int s = 0;
            for (int t = 16 * h; t < 16 * h + 16; ++t) s += std::abs((int)tab[ph * 32 + t]);
            if (s > 65535) return false;
        }
    return true;
}

void build_twiddles_q15(int G, int16_t *tw2) {
    // floor(exp(-2 pi j k / G) * 32768) clipped to int16 (src/fixedpoint.py:277, quant mode 'trunc')
    for (int k = 0; k < G / 2; ++k) {
        const double th = (-2.0 * M_PI * (double)k) / (double)G;
        const double c = std::floor(std::cos(th) / std::ldexp(1.0, -15));
        const double s = std::floor(std::sin(th) / std::ldexp(1.0, -15));
        tw2[2 * k] = (int16_t)std::min(std::max(c, -32768.0), 32767.0);
        tw2[2 * k + 1] = (int16_t)std::min(std::max(s, -32768.0), 32767.0);
    }
}

void build_hamming_q15(int len, int size, int32_t *out) {
    for (int i = 0; i < size; ++i) out[i] = 0;
    if (len == 1) { out[0] = 32768; return; }
    for (int i = 0; i < len; ++i) {
        const double h = 0.54 + 0.46 * std::cos(M_PI * (double)(2 * i + 1 - len) / (double)(len - 1));
        out[i] = (int32_t)std::floor(h * 32768.0);
    }
}
}  // namespace pfa

namespace {

bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }
int ilog2(int v) { int l = 0; while ((1 << l) < v) ++l; return l; }

pfa_status fail(pfa_plan *p, pfa_status st, const std::string &msg) {
    if (p) p->err = msg;
    return st;
}

pfa_status cuda_fail(pfa_plan *p, cudaError_t e, const char *where) {
    if (p) p->err = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? PFA_ERR_ALLOC : PFA_ERR_CUDA;
}

template <class T>
cudaError_t dalloc(T **ptr, size_t count, size_t *acc) {
    *acc += count * sizeof(T);
    return cudaMalloc(reinterpret_cast<void **>(ptr), std::max<size_t>(count, 1) * sizeof(T));
}

template <class T>
void dfree(T *&ptr) {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

namespace pfa {

// Byte offsets of the fixed job vectors inside FixedDev::job_block (256-byte aligned each).
struct FixedJobLayout {
    size_t f0, df, fac, tan_s, order, krp, kcp, hamr, hamc, tw, sinc, total;
    FixedJobLayout(int m, int G) {
        size_t o = 0;
        auto take = [&](size_t bytes) { const size_t at = o; o += (bytes + 255) / 256 * 256; return at; };
        f0 = take(4u * m); df = take(4u * m); fac = take(4u * m); tan_s = take(4u * m); order = take(4u * m);
        krp = take(4u * G); kcp = take(4u * G); hamr = take(4u * G); hamc = take(4u * G); tw = take(4u * G);
        sinc = take(2u * 256 * 32);
        total = o;
    }
};

cudaError_t fixed_alloc(FixedDev &d, int m, int n, int G) {
    size_t acc = 0;
    cudaError_t e = cudaSuccess;
    d.m = m; d.n = n; d.G = G; d.L = ilog2(G); d.mpad = (m + 31) / 32 * 32;
#define TRY(x) do { e = (x); if (e != cudaSuccess) return e; } while (0)
    const FixedJobLayout lay(m, G);
    TRY(cudaMalloc(&d.job_block, lay.total));
    d.job_bytes = lay.total;
    acc += lay.total;
    unsigned char *jb = static_cast<unsigned char *>(d.job_block);
    d.f0 = reinterpret_cast<float *>(jb + lay.f0); d.df = reinterpret_cast<float *>(jb + lay.df);
    d.fac = reinterpret_cast<float *>(jb + lay.fac); d.tan_s = reinterpret_cast<float *>(jb + lay.tan_s);
    d.order = reinterpret_cast<int32_t *>(jb + lay.order);
    d.krp = reinterpret_cast<float *>(jb + lay.krp); d.kcp = reinterpret_cast<float *>(jb + lay.kcp);
    d.hamr = reinterpret_cast<int32_t *>(jb + lay.hamr); d.hamc = reinterpret_cast<int32_t *>(jb + lay.hamc);
    d.tw = reinterpret_cast<uint32_t *>(jb + lay.tw); d.sinc = reinterpret_cast<int16_t *>(jb + lay.sinc);
    TRY(dalloc(&d.p1, (size_t)n * d.mpad, &acc));
    TRY(dalloc(&d.y1, (size_t)n * G, &acc));
    TRY(dalloc(&d.y2, (size_t)G * G, &acc));
    TRY(dalloc(&d.e1, G, &acc)); TRY(dalloc(&d.e2, G, &acc));
    TRY(dalloc(&d.ctrl, 16, &acc));
#undef TRY
    return cudaSuccess;
}

void fixed_free(FixedDev &d) {
    if (d.job_block) cudaFree(d.job_block);
    d.job_block = nullptr;
    d.f0 = d.df = d.fac = d.tan_s = d.krp = d.kcp = nullptr;
    d.order = d.hamr = d.hamc = nullptr;
    d.tw = nullptr;
    d.sinc = nullptr;
    dfree(d.p1); dfree(d.y1); dfree(d.y2); dfree(d.e1); dfree(d.e2); dfree(d.ctrl);
}

}  // namespace pfa

extern "C" {

const char *pfa_version(void) { return "pfa_b200 0.1 (sm_100a)"; }

const char *pfa_status_string(pfa_status st) {
    switch (st) {
        case PFA_OK: return "ok";
        case PFA_ERR_BAD_CONFIG: return "bad config";
        case PFA_ERR_BAD_DIMS: return "grid smaller than scene dims";
        case PFA_ERR_BAD_ARG: return "bad argument";
        case PFA_ERR_NOT_READY: return "job not set";
        case PFA_ERR_CUDA: return "cuda error";
        case PFA_ERR_ALLOC: return "device allocation failed";
        case PFA_ERR_TIMEOUT: return "timeout";
        case PFA_ERR_NO_DEVICE: return "no usable device";
        case PFA_ERR_TOO_LARGE: return "frame exceeds the no-allocation entry point's static scratch (grid <= 1024)";
    }
    return "unknown status";
}

pfa_status pfa_last_error(const pfa_plan *plan, char *buf, size_t len) {
    if (!plan || !buf || len == 0) return PFA_ERR_BAD_ARG;
    std::snprintf(buf, len, "%s", plan->err.c_str());
    return PFA_OK;
}

pfa_status pfa_plan_create(const pfa_config *cfg, pfa_plan **out) {
    if (!cfg || !out) return PFA_ERR_BAD_ARG;
    *out = nullptr;
    const pfa_config c = *cfg;
    if (c.m < 2 || c.n < 2) return PFA_ERR_BAD_DIMS;
    auto interp_ok = [&](int v) {
        return v == PFA_INTERP_LERP || v == PFA_INTERP_SINC || (v == PFA_INTERP_CUBIC && c.mode == PFA_MODE_FIXED);
    };
    if (!interp_ok(c.range_interp) || !interp_ok(c.az_interp)) return PFA_ERR_BAD_CONFIG;
    if (c.detect_order != PFA_DETECT_ORDER_EMULATOR && !(c.detect_order == PFA_DETECT_ORDER_FUSED && c.mode == PFA_MODE_FIXED))
        return PFA_ERR_BAD_CONFIG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= c.device || c.device < 0) return PFA_ERR_NO_DEVICE;
    pfa_plan *p = new (std::nothrow) pfa_plan();
    if (!p) return PFA_ERR_ALLOC;
    p->cfg = c;
    p->device = c.device;
    DeviceGuard dg(c.device);
    cudaError_t e;
    if (c.mode == PFA_MODE_FIXED) {
        if (!is_pow2(c.grid) || c.grid < 64 || c.grid > 16384) { delete p; return PFA_ERR_BAD_CONFIG; }
        if (c.grid < c.m || c.grid < c.n) { delete p; return PFA_ERR_BAD_DIMS; }
        e = pfa::fixed_alloc(p->fx, c.m, c.n, c.grid);
        p->fx.range_sinc = c.range_interp == PFA_INTERP_SINC;
        p->fx.az_sinc = c.az_interp == PFA_INTERP_SINC;
        p->fx.range_cubic = c.range_interp == PFA_INTERP_CUBIC;
        p->fx.az_cubic = c.az_interp == PFA_INTERP_CUBIC;
        p->fx.fused_detect = c.detect_order == PFA_DETECT_ORDER_FUSED;
        p->ws_bytes = pfa::fixed_workspace_bytes(c.m, c.n, c.grid);
    } else if (c.mode == PFA_MODE_FLOAT32 || c.mode == PFA_MODE_MIXED) {
        e = pfa::float_alloc(p->fl, c.m, c.n);
        p->fl.range_sinc = c.range_interp == PFA_INTERP_SINC;
        p->fl.az_sinc = c.az_interp == PFA_INTERP_SINC;
        auto ept_ok = [](int v) { return v == 0 || v == 8 || v == 16 || v == 32; };
        if (!ept_ok(c.fft_ept_cross) || !ept_ok(c.fft_ept_range)) {
            pfa::float_free(p->fl);
            delete p;
            return PFA_ERR_BAD_CONFIG;
        }
        p->fl.ept_cross = c.fft_ept_cross;      // 0: the automatic choice of the dispatch
        p->fl.ept_range = c.fft_ept_range;
        p->fl.mx_probe = c.test_wait_polls > 0 ? c.test_wait_polls : 0;
        p->ws_bytes = pfa::float_workspace_bytes(c.m, c.n);
        if (e == cudaErrorInvalidValue) { pfa::float_free(p->fl); delete p; return PFA_ERR_BAD_CONFIG; }
        if (e == cudaSuccess && c.mode == PFA_MODE_MIXED) {
            p->fl.mixed = 1;
            e = pfa::mixed_prepare(p->fl);
        }
    } else {
        delete p;
        return PFA_ERR_BAD_CONFIG;
    }
    if (e != cudaSuccess) {
        pfa::fixed_free(p->fx);
        pfa::float_free(p->fl);
        pfa_status st = e == cudaErrorMemoryAllocation ? PFA_ERR_ALLOC : PFA_ERR_CUDA;
        delete p;
        return st;
    }
    *out = p;
    return PFA_OK;
}

pfa_status pfa_plan_destroy(pfa_plan *p) {
    if (!p) return PFA_ERR_BAD_ARG;
    {
        DeviceGuard dg(p->device);
        pfa::fixed_free(p->fx);
        pfa::float_free(p->fl);
        if (p->staging_in) cudaFree(p->staging_in);
        if (p->staging_out) cudaFree(p->staging_out);
        if (p->host_stream) cudaStreamDestroy(p->host_stream);
        for (cudaStream_t s : {p->pipe_up, p->pipe_comp, p->pipe_down}) if (s) cudaStreamDestroy(s);
        for (int b = 0; b < 2; ++b) {
            if (p->pipe_in[b]) cudaFree(p->pipe_in[b]);
            if (p->pipe_out[b]) cudaFree(p->pipe_out[b]);
        }
        for (auto &ev : p->pipe_ev) if (ev) cudaEventDestroy(ev);
        for (auto &ev : p->prof.ev) if (ev) cudaEventDestroy(ev);
    }
    delete p;
    return PFA_OK;
}

size_t pfa_plan_workspace_bytes(const pfa_plan *p) { return p ? p->ws_bytes : 0; }

pfa_status pfa_set_fixed_job(pfa_plan *p, const pfa_fixed_job *job) {
    if (!p || !job) return PFA_ERR_BAD_ARG;
    if (p->cfg.mode != PFA_MODE_FIXED) return fail(p, PFA_ERR_BAD_CONFIG, "plan is not fixed mode");
    if (!job->f0 || !job->df || !job->pr || !job->tan_s || !job->inv_order || !job->kr_grid || !job->kc_grid)
        return fail(p, PFA_ERR_BAD_ARG, "missing job vector");
    DeviceGuard dg(p->device);
    pfa::FixedDev &d = p->fx;
    const int m = d.m, G = d.G;
    // The whole job goes up as one copy of its host image; the grid-dependent tables (twiddles, sinc) are
    // re-derived only when their inputs differ from the previous job's.
    const pfa::FixedJobLayout lay(m, G);
    std::vector<unsigned char> &img = p->job_host;
    const bool first = img.size() != lay.total;
    if (first) img.assign(lay.total, 0);
    auto at = [&](size_t off) { return img.data() + off; };
    std::memcpy(at(lay.f0), job->f0, 4u * m);
    std::memcpy(at(lay.df), job->df, 4u * m);
    std::memcpy(at(lay.tan_s), job->tan_s, 4u * m);
    // pass-1 source scale f32(f32(2 pr) / f32(c)) (NumPy 2 float32 arithmetic, silicon_emulator.py:144)
    float *fac = reinterpret_cast<float *>(at(lay.fac));
    const float c32 = (float)299792458.0;
    for (int i = 0; i < m; ++i) {
        volatile float two_pr = 2.0f * job->pr[i];
        fac[i] = two_pr / c32;
    }
    // sorted slot -> pulse (inverse of inv_order); reject non-permutations
    int32_t *order = reinterpret_cast<int32_t *>(at(lay.order));
    for (int i = 0; i < m; ++i) order[i] = -1;
    for (int i = 0; i < m; ++i) {
        const int r = job->inv_order[i];
        if (r < 0 || r >= m || order[r] != -1) return fail(p, PFA_ERR_BAD_ARG, "inv_order is not a permutation");
        order[r] = i;
    }
    std::memcpy(at(lay.krp), job->kr_grid, 4u * G);
    std::memcpy(at(lay.kcp), job->kc_grid, 4u * G);
    int32_t *hr = reinterpret_cast<int32_t *>(at(lay.hamr));
    int32_t *hc = reinterpret_cast<int32_t *>(at(lay.hamc));
    if (job->ham_r) std::memcpy(hr, job->ham_r, 4u * G); else pfa::build_hamming_q15(d.n, G, hr);
    if (job->ham_c) std::memcpy(hc, job->ham_c, 4u * G); else pfa::build_hamming_q15(m, G, hc);
    // twiddles: stage-contiguous layout, stage s (span 2^s) entries k < 2^(s-1) at offset 2^(s-1)-1
    const bool tw_same = !first && (job->twiddle ? (p->last_tw_builtin == 0 && p->last_tw_in.size() == (size_t)G &&
                                                    std::memcmp(p->last_tw_in.data(), job->twiddle, 2u * G) == 0)
                                                 : p->last_tw_builtin == 1);
    if (!tw_same) {
        std::vector<int16_t> tw2(G);
        if (job->twiddle) std::memcpy(tw2.data(), job->twiddle, sizeof(int16_t) * G); else pfa::build_twiddles_q15(G, tw2.data());
        uint32_t *tws = reinterpret_cast<uint32_t *>(at(lay.tw));
        std::memset(tws, 0, 4u * G);
        const int L = d.L;
        for (int b = 0; b < L; ++b) {
            for (int k = 0; k < (1 << b); ++k) {
                const int src = k << (L - 1 - b);
                tws[(1 << b) - 1 + k] = (uint32_t)(uint16_t)tw2[2 * src] | ((uint32_t)(uint16_t)tw2[2 * src + 1] << 16);
            }
        }
        p->last_tw_builtin = job->twiddle ? 0 : 1;
        if (job->twiddle) p->last_tw_in.assign(job->twiddle, job->twiddle + G); else p->last_tw_in.clear();
    }
    const bool sinc_same = !first && (job->sinc_q15 ? (p->last_sinc_builtin == 0 &&
                                                       std::memcmp(p->last_sinc_in.data(), job->sinc_q15, 2u * 256 * 32) == 0)
                                                    : p->last_sinc_builtin == 1);
    if (!sinc_same) {
        std::vector<int16_t> sinc_pt(256 * 32);
        if (job->sinc_q15) std::memcpy(sinc_pt.data(), job->sinc_q15, sizeof(int16_t) * 256 * 32); else pfa::build_sinc_table(sinc_pt.data());
        if (!pfa::sinc_table_fits_int32(sinc_pt.data())) {
            p->last_sinc_builtin = -1;
            return fail(p, PFA_ERR_BAD_ARG, "sinc table: sum |tap| over a half of a phase exceeds 65535");
        }
        int16_t *sinc = reinterpret_cast<int16_t *>(at(lay.sinc));
        for (int ph = 0; ph < 256; ++ph)          // device layout [tap][phase]
            for (int t = 0; t < 32; ++t) sinc[t * 256 + ph] = sinc_pt[ph * 32 + t];
        p->last_sinc_builtin = job->sinc_q15 ? 0 : 1;
        if (job->sinc_q15) p->last_sinc_in.assign(job->sinc_q15, job->sinc_q15 + 256 * 32); else p->last_sinc_in.clear();
    }
    const cudaError_t e = cudaMemcpy(d.job_block, img.data(), lay.total, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(p, e, "job upload");
    p->job_ready = true;
    return PFA_OK;
}

static pfa_status fixed_common(pfa_plan *p, const float *sig, const int16_t *iq, uint16_t *img, void *stream) {
    if (!p || !img || (!sig && !iq)) return PFA_ERR_BAD_ARG;
    if (p->cfg.mode != PFA_MODE_FIXED) return fail(p, PFA_ERR_BAD_CONFIG, "plan is not fixed mode");
    if (!p->job_ready) return fail(p, PFA_ERR_NOT_READY, "pfa_set_fixed_job not called");
    if (sig && (reinterpret_cast<uintptr_t>(sig) & 15)) return fail(p, PFA_ERR_BAD_ARG, "signal must be 16-byte aligned");
    if (iq && (reinterpret_cast<uintptr_t>(iq) & 3)) return fail(p, PFA_ERR_BAD_ARG, "iq16 signal must be 4-byte aligned");
    if (reinterpret_cast<uintptr_t>(img) & 3) return fail(p, PFA_ERR_BAD_ARG, "image must be 4-byte aligned");
    DeviceGuard dg(p->device);
    cudaError_t e = pfa::fixed_form(p->fx, sig, reinterpret_cast<const uint32_t *>(iq), img,
                                    reinterpret_cast<cudaStream_t>(stream), &p->prof);
    if (e != cudaSuccess) return cuda_fail(p, e, "fixed form");
    return PFA_OK;
}

pfa_status pfa_form_fixed(pfa_plan *p, const float *sig_dev, uint16_t *img_dev, void *stream) {
    return fixed_common(p, sig_dev, nullptr, img_dev, stream);
}

pfa_status pfa_form_fixed_iq16(pfa_plan *p, const int16_t *sig_iq_dev, uint16_t *img_dev, void *stream) {
    return fixed_common(p, nullptr, sig_iq_dev, img_dev, stream);
}

static pfa_status ensure_staging(pfa_plan *p, size_t in_bytes, size_t out_bytes) {
    cudaError_t e;
    if (!p->host_stream) {
        e = cudaStreamCreateWithFlags(&p->host_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(p, e, "stream create");
    }
    if (p->staging_in_bytes < in_bytes) {
        if (p->staging_in) cudaFree(p->staging_in);
        p->staging_in = nullptr;
        e = cudaMalloc(reinterpret_cast<void **>(&p->staging_in), in_bytes);
        if (e != cudaSuccess) { p->staging_in_bytes = 0; return cuda_fail(p, e, "staging alloc"); }
        p->staging_in_bytes = in_bytes;
    }
    if (p->staging_out_bytes < out_bytes) {
        if (p->staging_out) cudaFree(p->staging_out);
        p->staging_out = nullptr;
        e = cudaMalloc(&p->staging_out, out_bytes);
        if (e != cudaSuccess) { p->staging_out_bytes = 0; return cuda_fail(p, e, "staging alloc"); }
        p->staging_out_bytes = out_bytes;
    }
    return PFA_OK;
}

pfa_status pfa_form_fixed_host(pfa_plan *p, const float *sig_host, uint16_t *img_host) {
    if (!p || !sig_host || !img_host) return PFA_ERR_BAD_ARG;
    if (p->cfg.mode != PFA_MODE_FIXED) return fail(p, PFA_ERR_BAD_CONFIG, "plan is not fixed mode");
    DeviceGuard dg(p->device);
    const size_t in_b = sizeof(float) * 2 * (size_t)p->fx.m * p->fx.n;
    const size_t out_b = sizeof(uint16_t) * (size_t)p->fx.G * p->fx.G;
    pfa_status st = ensure_staging(p, in_b, out_b);
    if (st != PFA_OK) return st;
    cudaError_t e = cudaMemcpyAsync(p->staging_in, sig_host, in_b, cudaMemcpyHostToDevice, p->host_stream);
    if (e != cudaSuccess) return cuda_fail(p, e, "h2d");
    st = fixed_common(p, p->staging_in, nullptr, static_cast<uint16_t *>(p->staging_out), p->host_stream);
    if (st != PFA_OK) return st;
    e = cudaMemcpyAsync(img_host, p->staging_out, out_b, cudaMemcpyDeviceToHost, p->host_stream);
    if (e != cudaSuccess) return cuda_fail(p, e, "d2h");
    e = cudaStreamSynchronize(p->host_stream);
    if (e != cudaSuccess) return cuda_fail(p, e, "sync");
    return PFA_OK;
}

}  // extern "C"

pfa_status pfa::run_host_frames(pfa_plan *p, const void *const *ins, void *const *outs, int32_t nframes,
                                size_t in_b, size_t out_b, FrameFn form, int32_t arg) {
    if (!ins || !outs || nframes < 0) return PFA_ERR_BAD_ARG;
    for (int k = 0; k < nframes; ++k)
        if (!ins[k] || !outs[k]) return PFA_ERR_BAD_ARG;
    cudaError_t e;
    for (cudaStream_t *s : {&p->pipe_up, &p->pipe_comp, &p->pipe_down})
        if (!*s && (e = cudaStreamCreateWithFlags(s, cudaStreamNonBlocking)) != cudaSuccess) return cuda_fail(p, e, "pipe stream");
    for (auto &ev : p->pipe_ev)
        if (!ev && (e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return cuda_fail(p, e, "pipe event");
    if (p->pipe_in_bytes < in_b || p->pipe_out_bytes < out_b) {
        for (int b = 0; b < 2; ++b) {
            if (p->pipe_in[b]) cudaFree(p->pipe_in[b]);
            if (p->pipe_out[b]) cudaFree(p->pipe_out[b]);
            p->pipe_in[b] = p->pipe_out[b] = nullptr;
        }
        p->pipe_in_bytes = p->pipe_out_bytes = 0;
        for (int b = 0; b < 2; ++b) {
            if ((e = cudaMalloc(&p->pipe_in[b], in_b)) != cudaSuccess) return cuda_fail(p, e, "pipe staging");
            if ((e = cudaMalloc(&p->pipe_out[b], out_b)) != cudaSuccess) return cuda_fail(p, e, "pipe staging");
        }
        p->pipe_in_bytes = in_b;
        p->pipe_out_bytes = out_b;
    }
    cudaEvent_t *uploaded = p->pipe_ev, *computed = p->pipe_ev + 2, *downloaded = p->pipe_ev + 4;
    // Once the first copy is enqueued, every return drains the three streams first: copies into and out of
    // the caller's host buffers and the staging buffers must not outlive the call, and the next call's
    // frames 0 and 1 reuse the staging buffers without waiting on this call's events.
    auto drain = [p](pfa_status st) {
        for (cudaStream_t s : {p->pipe_up, p->pipe_comp, p->pipe_down}) {
            cudaError_t es = cudaStreamSynchronize(s);
            if (es != cudaSuccess && st == PFA_OK) st = cuda_fail(p, es, "pipe sync");
        }
        return st;
    };
    for (int k = 0; k < nframes; ++k) {
        const int b = k & 1;
        // upload k once frame k-2 no longer reads this staging buffer
        if (k >= 2 && (e = cudaStreamWaitEvent(p->pipe_up, computed[b], 0)) != cudaSuccess) return drain(cuda_fail(p, e, "pipe"));
        if ((e = cudaMemcpyAsync(p->pipe_in[b], ins[k], in_b, cudaMemcpyHostToDevice, p->pipe_up)) != cudaSuccess)
            return drain(cuda_fail(p, e, "pipe h2d"));
        if ((e = cudaEventRecord(uploaded[b], p->pipe_up)) != cudaSuccess) return drain(cuda_fail(p, e, "pipe"));
        // frame k after its upload, and after frame k-2's image left this output buffer
        if ((e = cudaStreamWaitEvent(p->pipe_comp, uploaded[b], 0)) != cudaSuccess) return drain(cuda_fail(p, e, "pipe"));
        if (k >= 2 && (e = cudaStreamWaitEvent(p->pipe_comp, downloaded[b], 0)) != cudaSuccess)
            return drain(cuda_fail(p, e, "pipe"));
        pfa_status st = form(p, p->pipe_in[b], p->pipe_out[b], p->pipe_comp, arg);
        if (st != PFA_OK) return drain(st);
        if ((e = cudaEventRecord(computed[b], p->pipe_comp)) != cudaSuccess) return drain(cuda_fail(p, e, "pipe"));
        // download k
        if ((e = cudaStreamWaitEvent(p->pipe_down, computed[b], 0)) != cudaSuccess) return drain(cuda_fail(p, e, "pipe"));
        if ((e = cudaMemcpyAsync(outs[k], p->pipe_out[b], out_b, cudaMemcpyDeviceToHost, p->pipe_down)) != cudaSuccess)
            return drain(cuda_fail(p, e, "pipe d2h"));
        if ((e = cudaEventRecord(downloaded[b], p->pipe_down)) != cudaSuccess) return drain(cuda_fail(p, e, "pipe"));
    }
    return drain(PFA_OK);
}

extern "C" {

static pfa_status fixed_frame(pfa_plan *p, const void *in, void *out, cudaStream_t st, int32_t) {
    return fixed_common(p, static_cast<const float *>(in), nullptr, static_cast<uint16_t *>(out), st);
}

pfa_status pfa_form_fixed_host_frames(pfa_plan *p, const float *const *sig_hosts, uint16_t *const *img_hosts,
                                      int32_t nframes) {
    if (!p) return PFA_ERR_BAD_ARG;
    if (p->cfg.mode != PFA_MODE_FIXED) return fail(p, PFA_ERR_BAD_CONFIG, "plan is not fixed mode");
    DeviceGuard dg(p->device);
    const size_t in_b = sizeof(float) * 2 * (size_t)p->fx.m * p->fx.n;
    const size_t out_b = sizeof(uint16_t) * (size_t)p->fx.G * p->fx.G;
    return pfa::run_host_frames(p, reinterpret_cast<const void *const *>(sig_hosts),
                                reinterpret_cast<void *const *>(img_hosts), nframes, in_b, out_b, fixed_frame, 0);
}

pfa_status pfa_get_fixed_exponents(pfa_plan *p, int32_t *e_range, int32_t *e_az, int32_t *q0_exp) {
    if (!p) return PFA_ERR_BAD_ARG;
    if (p->cfg.mode != PFA_MODE_FIXED) return fail(p, PFA_ERR_BAD_CONFIG, "plan is not fixed mode");
    DeviceGuard dg(p->device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(p, e, "sync");
    if (e_range && (e = cudaMemcpy(e_range, p->fx.e1, sizeof(int32_t) * p->fx.n, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(p, e, "exponents");
    if (e_az && (e = cudaMemcpy(e_az, p->fx.e2, sizeof(int32_t) * p->fx.G, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(p, e, "exponents");
    if (q0_exp) {
        int32_t ctrl[4];
        if ((e = cudaMemcpy(ctrl, p->fx.ctrl, sizeof(ctrl), cudaMemcpyDeviceToHost)) != cudaSuccess)
            return cuda_fail(p, e, "exponents");
        *q0_exp = ctrl[3];
    }
    return PFA_OK;
}

pfa_status pfa_set_profiling(pfa_plan *p, int32_t enable) {
    if (!p) return PFA_ERR_BAD_ARG;
    DeviceGuard dg(p->device);
    if (enable) {
        for (auto &ev : p->prof.ev) {
            if (!ev) {
                cudaError_t e = cudaEventCreate(&ev);
                if (e != cudaSuccess) return cuda_fail(p, e, "event create");
            }
        }
    }
    p->prof.on = enable != 0;
    p->prof.count = 0;
    return PFA_OK;
}

pfa_status pfa_get_stage_times(pfa_plan *p, float *ms, int32_t cap, int32_t *count, char *names, size_t names_len) {
    if (!p || !count) return PFA_ERR_BAD_ARG;
    DeviceGuard dg(p->device);
    const int n = p->prof.count > 0 ? p->prof.count - 1 : 0;
    *count = n;
    std::string nm;
    for (int i = 0; i < n; ++i) {
        if (ms && i < cap) {
            cudaError_t e = cudaEventSynchronize(p->prof.ev[i + 1]);
            if (e != cudaSuccess) return cuda_fail(p, e, "event sync");
            e = cudaEventElapsedTime(ms + i, p->prof.ev[i], p->prof.ev[i + 1]);
            if (e != cudaSuccess) return cuda_fail(p, e, "event time");
        }
        if (i) nm += ",";
        nm += p->prof.names[i + 1];
    }
    if (names && names_len) std::snprintf(names, names_len, "%s", nm.c_str());
    return PFA_OK;
}

}  // extern "C"
