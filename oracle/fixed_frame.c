/*
 * ORACLE (test infrastructure, never shipped or measured as the product): a C restatement of the
 * reference's bit-accurate fixed-point PFA datapath, mpfs/host/silicon_emulator.py form_image
 * (:216-253), for timing whole frames on every host core (OpenMP) in bench.py's reference arm and
 * cpu_baseline leg.  It follows the vectorised NumPy oracle (oracle/fixed_emulator.py) step for step;
 * tests/test_oracle_pins.py checks that both give the same image CRC, and the reference emulator's own
 * CRC of the Centerfield-shaped frame is checked by the reference arm on every run.
 *
 *   Q0 quantiser          silicon_emulator.py:226-229, src/fixedpoint.py:19-26 (fit_scale)
 *   bracket + Q15 weight  mpfs/host/serialize_inputs.py:67-94 (interp_coeffs)
 *   2-tap lerp            silicon_emulator.py:60-71 (apply_fixed); the pass-1 lerp multiplies in float32
 *   32-tap sinc           silicon_emulator.py:88-122 (apply_sinc); its edge lerp is the integer one
 *   two-pass resample     silicon_emulator.py:125-156 (resample_fixed)
 *   Q15 2-D Hamming       silicon_emulator.py:165-195 (window_fixed)
 *   per-row BFP FFT       src/fixedpoint.py:266-289 (fft1d_bfp_hw_perrow), renorm :198-205
 *   detect                silicon_emulator.py:208-213 (detect_fixed)
 *
 * Float steps use the same IEEE operations as NumPy: float64 coordinates f64(fac) * (f64(f0) + k f64(df))
 * (compile with -ffp-contract=off: no fused multiply-add), float32 pass-2 source coordinates, float64
 * fractions rounded half to even (rint), float32 Q0 division.  Integer steps are exact in int32/int64.
 *
 * Build: gcc -O3 -fopenmp -ffp-contract=off -fPIC -shared fixed_frame.c -o lib/libfixed_oracle.so -lm
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline int32_t sat16(int64_t v) { return v < -32768 ? -32768 : (v > 32767 ? 32767 : (int32_t)v); }
static inline int32_t wrap16(int64_t v) { return (int32_t)(int16_t)(uint16_t)(v & 0xffff); }

/* bracket_q15(query, xp) of one query against an ascending view xa of n source coordinates.
 * cnt = number of xa values < q (searchsorted 'left').  Writes idx (natural order, -1 outside) and wq. */
static inline void bracket(const double *xa, int n, int asc, double q, int cnt, int *idx, int *wq) {
    const int k = cnt - 1;
    if (k < 0 || k >= n - 1) { *idx = -1; *wq = 0; return; }
    const double fa = (q - xa[k]) / (xa[k + 1] - xa[k]);
    const double w = asc ? fa : 1.0 - fa;
    double r = rint(w * 32768.0);
    if (r < 0.0) r = 0.0;
    if (r > 32767.0) r = 32767.0;
    *idx = asc ? k : (n - 2 - k);
    *wq = (int)r;
}

/* Brackets of an ascending query vector qv[nq] against source coordinates xp[n] (either direction):
 * a merge walk over the ascending view.  NaN queries (none occur) would count as above every source. */
static void brackets(const double *qv, int nq, const double *xp, int n, double *xa, int *idx, int *wq) {
    const int asc = xp[n - 1] >= xp[0];
    for (int t = 0; t < n; ++t) xa[t] = asc ? xp[t] : xp[n - 1 - t];
    int cnt = 0;
    for (int j = 0; j < nq; ++j) {
        const double q = qv[j];
        if (j > 0 && q < qv[j - 1]) cnt = 0;              /* not ascending: restart the walk */
        while (cnt < n && xa[cnt] < q) ++cnt;
        bracket(xa, n, asc, q, cnt, idx + j, wq + j);
    }
}

/* One resampled line: mode 0 lerp, 1 sinc; f32prod: the float32 lerp product of pass 1. */
static void gather(const int32_t *xr, const int32_t *xi, int sn, const int *idx, const int *wq, int nq, int mode,
                   int f32prod, const int16_t *tab, int32_t *outr, int32_t *outi) {
    for (int j = 0; j < nq; ++j) {
        const int b = idx[j];
        if (b < 0) { outr[j] = outi[j] = 0; continue; }
        if (mode == 1 && b >= 15 && b <= sn - 17) {
            const int16_t *c = tab + (wq[j] >> 7) * 32;
            const int32_t *pr = xr + b - 15, *pi = xi + b - 15;
            int64_t ar = 0, ai = 0;
            for (int t = 0; t < 32; ++t) {
                ar += (int64_t)c[t] * pr[t];
                ai += (int64_t)c[t] * pi[t];
            }
            outr[j] = sat16((ar + (1 << 14)) >> 15);
            outi[j] = sat16((ai + (1 << 14)) >> 15);
            continue;
        }
        const int k = b > sn - 2 ? sn - 2 : b;
        const int32_t dr = xr[k + 1] - xr[k], di = xi[k + 1] - xi[k];
        int32_t sr, si;
        if (mode == 0 && f32prod) {
            const float w = (float)wq[j];
            sr = (int32_t)floorf(((float)dr * w) / 32768.0f);
            si = (int32_t)floorf(((float)di * w) / 32768.0f);
        } else {
            sr = (int32_t)(((int64_t)dr * wq[j]) >> 15);
            si = (int32_t)(((int64_t)di * wq[j]) >> 15);
        }
        outr[j] = sat16((int64_t)xr[k] + sr);
        outi[j] = sat16((int64_t)xi[k] + si);
    }
}

static int stage_shift(int64_t mx) {
    int sh = 0;
    int64_t lim = 32767;
    while (mx + 1 > lim) { ++sh; lim *= 2; }
    return sh;
}

/* fft1d_bfp_hw_perrow on one row (in place, natural order in and out); returns the row exponent. */
static int fft_row(int32_t *xr, int32_t *xi, int L, const int32_t *wr, const int32_t *wi, int32_t *tr_, int32_t *ti_) {
    const int n = 1 << L;
    for (int p = 0; p < n; ++p) {
        unsigned r = 0;
        for (int b = 0; b < L; ++b) r |= (unsigned)((p >> b) & 1) << (L - 1 - b);
        tr_[p] = xr[r];
        ti_[p] = xi[r];
    }
    memcpy(xr, tr_, sizeof(int32_t) * n);
    memcpy(xi, ti_, sizeof(int32_t) * n);
    int e = 0;
    for (int s = 1; s <= L; ++s) {
        const int blk = 1 << s, half = blk >> 1, stride = n / blk;
        int32_t hi = 0;
        for (int g = 0; g < n; g += blk) {
            for (int k = 0; k < half; ++k) {
                const int64_t w_r = wr[k * stride], w_i = wi[k * stride];
                const int a = g + k, c = a + half;
                const int32_t t_r = sat16((w_r * xr[c] - w_i * xi[c]) >> 15);
                const int32_t t_i = sat16((w_r * xi[c] + w_i * xr[c]) >> 15);
                const int32_t ar = xr[a], ai = xi[a];
                xr[a] = ar + t_r; xi[a] = ai + t_i;
                xr[c] = ar - t_r; xi[c] = ai - t_i;
            }
        }
        for (int p = 0; p < n; ++p) {
            const int32_t u = abs(xr[p]), v = abs(xi[p]);
            if (u > hi) hi = u;
            if (v > hi) hi = v;
        }
        const int sh = stage_shift(hi);
        if (sh) {
            for (int p = 0; p < n; ++p) { xr[p] = sat16(xr[p] >> sh); xi[p] = sat16(xi[p] >> sh); }
        }
        e += sh;
    }
    return e;
}

/* One FFT pass over G rows of (re, im) int32 planes followed by the global renormalisation. */
static void fft_pass(int32_t *xr, int32_t *xi, int G, int L, const int32_t *wr, const int32_t *wi, int32_t *e) {
    #pragma omp parallel
    {
        int32_t *tr_ = (int32_t *)malloc(sizeof(int32_t) * G), *ti_ = (int32_t *)malloc(sizeof(int32_t) * G);
        #pragma omp for schedule(dynamic, 16)
        for (int r = 0; r < G; ++r) e[r] = fft_row(xr + (size_t)r * G, xi + (size_t)r * G, L, wr, wi, tr_, ti_);
        free(tr_);
        free(ti_);
    }
    int emax = 0;
    for (int r = 0; r < G; ++r) if (e[r] > emax) emax = e[r];
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < G; ++r) {
        const int sh = emax - e[r];
        if (!sh) continue;
        int32_t *pr = xr + (size_t)r * G, *pi = xi + (size_t)r * G;
        for (int k = 0; k < G; ++k) { pr[k] = sat16(pr[k] >> sh); pi[k] = sat16(pi[k] >> sh); }
    }
}

static void transpose(const int32_t *src, int32_t *dst, int G) {
    #pragma omp parallel for schedule(static)
    for (int rb = 0; rb < G; rb += 64)
        for (int cb = 0; cb < G; cb += 64)
            for (int r = rb; r < rb + 64 && r < G; ++r)
                for (int c = cb; c < cb + 64 && c < G; ++c) dst[(size_t)c * G + r] = src[(size_t)r * G + c];
}

/* The whole frame.  sig: m x n complex64 (interleaved).  Geometry as fixed_emulator.fixed_geometry:
 * f0, df, fac (float32 [m]), inv_order (int32 [m]), tan_s (float32 [m]), krp, kcp (float32 [G]);
 * hr, hc: floor(hamming * 32768) zero padded (int32 [G]); wr, wi: Q15 twiddles (int32 [G/2]);
 * tab: sinc table [256][32].  Modes: 0 lerp, 1 sinc.  img: uint16 [G][G] (rows = range bins).
 * e_range[G], e_az[G] and *q0e receive the exponents.  nthreads <= 0: OpenMP's default.
 * Returns 0, or -1 when an allocation fails. */
int pfa_oracle_fixed_frame(const float *sig, int m, int n, int G, const float *f0, const float *df, const float *fac,
                           const int32_t *inv_order, const float *tan_s, const float *krp, const float *kcp,
                           const int32_t *hr, const int32_t *hc, const int32_t *wr, const int32_t *wi,
                           const int16_t *tab, int range_mode, int az_mode, int nthreads, uint16_t *img,
                           int32_t *e_range, int32_t *e_az, int32_t *q0e) {
    int L = 0;
    while ((1 << L) < G) ++L;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const size_t GG = (size_t)G * G;
    int32_t *ar = (int32_t *)calloc(GG, sizeof(int32_t)), *ai = (int32_t *)calloc(GG, sizeof(int32_t));
    int32_t *br = (int32_t *)malloc(GG * sizeof(int32_t)), *bi = (int32_t *)malloc(GG * sizeof(int32_t));
    int32_t *qr = (int32_t *)malloc((size_t)m * n * sizeof(int32_t)), *qi = (int32_t *)malloc((size_t)m * n * sizeof(int32_t));
    if (!ar || !ai || !br || !bi || !qr || !qi) {
        free(ar); free(ai); free(br); free(bi); free(qr); free(qi);
        return -1;
    }
    /* Q0: exponent of fit_scale from the float32 maximum, floor(x / 2^e) in float32, saturated */
    float big = 0.0f;
    #pragma omp parallel for reduction(max : big) schedule(static)
    for (size_t t = 0; t < (size_t)2 * m * n; ++t) {
        const float v = fabsf(sig[t]);
        if (v > big) big = v;
    }
    const int e0 = big == 0.0f ? 0 : (int)ceil(log2((double)big / 32767.0));
    *q0e = e0;
    const float lsb = (float)ldexp(1.0, e0);
    #pragma omp parallel for schedule(static)
    for (size_t t = 0; t < (size_t)m * n; ++t) {
        float a = floorf(sig[2 * t] / lsb), b = floorf(sig[2 * t + 1] / lsb);
        a = a < -32768.0f ? -32768.0f : (a > 32767.0f ? 32767.0f : a);
        b = b < -32768.0f ? -32768.0f : (b > 32767.0f ? 32767.0f : b);
        qr[t] = (int32_t)a;
        qi[t] = (int32_t)b;
    }
    /* pass 1: pulse i -> row inv_order[i] of the G x G scratch (a), columns = range bins */
    #pragma omp parallel
    {
        double *qv = (double *)malloc(sizeof(double) * G), *xp = (double *)malloc(sizeof(double) * n);
        double *xa = (double *)malloc(sizeof(double) * n);
        int *idx = (int *)malloc(sizeof(int) * G), *wq = (int *)malloc(sizeof(int) * G);
        for (int j = 0; j < G; ++j) qv[j] = (double)krp[j];
        #pragma omp for schedule(dynamic, 8)
        for (int i = 0; i < m; ++i) {
            const double fc = (double)fac[i], a0 = (double)f0[i], d0 = (double)df[i];
            for (int k = 0; k < n; ++k) xp[k] = fc * (a0 + (double)k * d0);
            brackets(qv, G, xp, n, xa, idx, wq);
            const size_t row = (size_t)inv_order[i] * G;
            gather(qr + (size_t)i * n, qi + (size_t)i * n, n, idx, wq, G, range_mode, 1, tab, ar + row, ai + row);
        }
        free(qv); free(xp); free(xa); free(idx); free(wq);
    }
    /* corner turn: b[j][slot] = a[slot][j] */
    transpose(ar, br, G);
    transpose(ai, bi, G);
    /* pass 2 + window: range row j of b (its first m slots) -> row j of a */
    #pragma omp parallel
    {
        double *qv = (double *)malloc(sizeof(double) * G), *xp = (double *)malloc(sizeof(double) * m);
        double *xa = (double *)malloc(sizeof(double) * m);
        int *idx = (int *)malloc(sizeof(int) * G), *wq = (int *)malloc(sizeof(int) * G);
        for (int k = 0; k < G; ++k) qv[k] = (double)kcp[k];
        #pragma omp for schedule(dynamic, 8)
        for (int j = 0; j < G; ++j) {
            for (int s = 0; s < m; ++s) xp[s] = (double)(krp[j] * tan_s[s]);     /* float32 product */
            brackets(qv, G, xp, m, xa, idx, wq);
            int32_t *orow = ar + (size_t)j * G, *oim = ai + (size_t)j * G;
            gather(br + (size_t)j * G, bi + (size_t)j * G, m, idx, wq, G, az_mode, 0, tab, orow, oim);
            for (int k = 0; k < G; ++k) {
                const int32_t cw = wrap16(((int64_t)hr[j] * hc[k]) >> 15);
                orow[k] = sat16(wrap16(((int64_t)orow[k] * cw) >> 15));
                oim[k] = sat16(wrap16(((int64_t)oim[k] * cw) >> 15));
            }
        }
        free(qv); free(xp); free(xa); free(idx); free(wq);
    }
    /* FFT-1 along the cross axis (rows = range bins), corner turn, FFT-2 along range (rows = cross bins) */
    fft_pass(ar, ai, G, L, wr, wi, e_range);
    transpose(ar, br, G);
    transpose(ai, bi, G);
    fft_pass(br, bi, G, L, wr, wi, e_az);
    /* detect, transposed back to [range][cross] */
    #pragma omp parallel for schedule(static)
    for (int jb = 0; jb < G; jb += 64)
        for (int k = 0; k < G; ++k)
            for (int j = jb; j < jb + 64 && j < G; ++j) {
                const int64_t re = br[(size_t)k * G + j], im = bi[(size_t)k * G + j];
                double mag = floor(sqrt((double)(re * re + im * im)));
                img[(size_t)j * G + k] = (uint16_t)(mag > 65535.0 ? 65535.0 : mag);
            }
    free(ar); free(ai); free(br); free(bi); free(qr); free(qi);
    return 0;
}
