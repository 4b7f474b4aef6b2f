/*
 * bls_oracle.c -- CPU restatement of the reference's Box Least Squares hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the tests compare the
 * CUDA engine in astro_transit_gpu_b200/csrc against.  Only the test-suite, the smoke check and the
 * CPU-baseline leg of bench.py load it; the product path never does.
 *
 * Two families of functions live here.
 *
 * (A) orc_ref_* -- faithful FP64 restatement of the reference kernels as they
 *     run with SCALAR_T=double.  These are pinned against golden vectors that
 *     the reference's own kernels (compiled from source, run on a B200) wrote.
 *       - astropy-binned geometry, method="parity":
 *           kernel  search/kernels/vbls_v42_parity.cu:36-129 (bins, windows)
 *                   search/kernels/vbls_v42_parity.cu:132-181 (argmax, outputs)
 *           host    search/v42_parity.py:42-67 (dt, totals, launch)
 *       - fixed-bin geometry, method="fast":
 *           kernel  search/kernels/bls.cu:47-169
 *           host    search/gpu_bls.py:57-78 (weights, weighted-mean subtraction)
 *     Objective "likelihood" is not in the reference kernels; it is the
 *     Gaussian log-likelihood gain of the box model,
 *     0.5 * depth^2 * W_in*W_out/(W_in+W_out), evaluated on the V42 windows.
 *
 * (B) orc_eng_* -- the engine's own exact arithmetic: deterministic fixed-point
 *     staging of (w, w*(y-c)), integer histograms, the FP32 window search with
 *     an exact rational comparison, and the FP64 re-evaluation of the winning
 *     window.  The CUDA engine must agree with (B) bit for bit; (B) agrees with
 *     (A) to the stated tolerances (tests/test_oracle.py).
 *
 * Build with -ffp-contract=off: every fused multiply-add below is spelled out
 * with fma()/fmaf(), everything else is rounded operation by operation.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_EINVAL 1
#define ORC_ENOMEM 2

#define OBJ_FAST 0       /* two-sided score of bls.cu */
#define OBJ_SNR 1        /* V42 / Astropy objective="snr" */
#define OBJ_LIKELIHOOD 2 /* Astropy objective="likelihood" */

static void set_threads(int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

/* ------------------------------------------------------------------------- */
/* (A) reference-faithful FP64 restatements                                   */
/* ------------------------------------------------------------------------- */

typedef struct { double c, f; } bin2;

/* Window order used to break exact ties: lowest start, then lowest duration
 * index.  The reference kernels break exact ties by their reduction trees;
 * in FP64 exact ties essentially never occur, so tests treat near-ties
 * (runner-up within gap) as equivalent. */

/*
 * One period of the astropy-binned geometry.
 * vbls_v42_parity.cu:36-47   bin geometry and the max_bins cap
 * vbls_v42_parity.cu:59      dur_bins = round(dur / bin_dur)
 * vbls_v42_parity.cu:65-76   fold, ind = int(ph/bin_dur)+1, clamp to n_bins
 * vbls_v42_parity.cu:78-84   padding copy and serial prefix
 * vbls_v42_parity.cu:97-129  windows, dip-only, SNR
 */
/* Pairwise sum of w[i] (what = 0) or y[i] * w[i] (what = 1) over [0, n),
 * w NULL = unit weights: an error of O(log n) ulp. */
static double pairwise_sum(int64_t n, const double* y, const double* w, int what)
{
    if (n <= 16) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            const double wi = w ? w[i] : 1.0;
            s += what ? y[i] * wi : wi;
        }
        return s;
    }
    const int64_t h = n / 2;
    return pairwise_sum(h, y, w, what) +
           pairwise_sum(n - h, y + h, w ? w + h : NULL, what);
}

static void ref_binned_period(int64_t n, const double* dt, const double* y, const double* w,
                              double tot_w, double tot_y, double t_start, double period,
                              double bin_dur, double inv_bin_dur, int oversample, int max_bins,
                              int nd, const int* dur_bins, int objective, bin2* bins,
                              double* o_power, double* o_depth, double* o_derr, double* o_t0,
                              double* o_dur, int32_t* o_win, double* o_gap)
{
    const double inv_period = 1.0 / period;
    int n_bins = (int)ceil(period * inv_bin_dur) + oversample;
    if (max_bins > 0 && n_bins >= max_bins) n_bins = max_bins - 1;
    memset(bins, 0, sizeof(bin2) * (size_t)(n_bins + 1));

    for (int64_t i = 0; i < n; ++i) {
        const double t = dt[i];
        const double ph = fma(-period, floor(t * inv_period), t);
        int ind = (int)(ph * inv_bin_dur) + 1;
        if (ind > n_bins) ind = n_bins;
        if (ind < 0) ind = 0; /* unreachable for finite input; keeps the write in bounds */
        const double wi = w ? w[i] : 1.0;
        bins[ind].c += wi;
        bins[ind].f = fma(y[i], wi, bins[ind].f);
    }
    for (int j = 1, ind = n_bins - oversample; j <= oversample; ++j, ++ind) bins[ind] = bins[j];
    for (int j = 1; j <= n_bins; ++j) {
        bins[j].c += bins[j - 1].c;
        bins[j].f += bins[j - 1].f;
    }

    double best = -1.0, second = -1.0;
    double b_depth = 0.0, b_derr = 0.0, b_t0 = 0.0, b_dur = 0.0;
    int32_t b_win = -1;
    for (int s = 0; s < n_bins; ++s) {
        for (int k = 0; k < nd; ++k) {
            const int d = dur_bins[k];
            if (s + d > n_bins) continue;
            const double ivar_in = bins[s + d].c - bins[s].c;
            const double y_in_sum = bins[s + d].f - bins[s].f;
            const double ivar_out = tot_w - ivar_in;
            const double y_out_sum = tot_y - y_in_sum;
            if (ivar_in < 1e-15 || ivar_out < 1e-15) continue;
            const double y_in = y_in_sum / ivar_in;
            const double y_out = y_out_sum / ivar_out;
            if (!(y_out >= y_in)) continue;
            const double depth = y_out - y_in;
            const double derr = sqrt(1.0 / ivar_in + 1.0 / ivar_out);
            double obj;
            if (objective == OBJ_LIKELIHOOD)
                obj = 0.5 * depth * depth * (ivar_in * ivar_out) / (ivar_in + ivar_out);
            else
                obj = depth / derr;
            if (obj > best) {
                second = best;
                best = obj;
                b_depth = depth;
                b_derr = derr;
                b_dur = (double)d * bin_dur;
                b_t0 = fmod((double)s * bin_dur + 0.5 * b_dur + t_start, period);
                b_win = s * nd + k;
            } else if (obj > second) {
                second = obj;
            }
        }
    }
    *o_power = best > 0.0 ? best : 0.0;
    *o_depth = b_depth;
    *o_derr = b_derr;
    *o_t0 = b_t0;
    *o_dur = b_dur;
    *o_win = b_win;
    *o_gap = (best > 0.0 && second > -1.0) ? (best - second) / best : 1.0;
}

int orc_ref_binned(int64_t n, const double* t, const double* y, const double* w, int64_t np,
                   const double* periods, int32_t nd, const double* durations, int32_t oversample,
                   int32_t max_bins, int32_t objective, int32_t nthreads, double* power,
                   double* depth, double* depth_err, double* t0, double* duration, int32_t* window,
                   double* gap)
{
    if (n <= 0 || np <= 0 || nd <= 0 || oversample < 1) return ORC_EINVAL;
    if (max_bins > 0 && max_bins < oversample + 2) return ORC_EINVAL;
    if (objective != OBJ_SNR && objective != OBJ_LIKELIHOOD) return ORC_EINVAL;

    /* v42_parity.py:42-46 -- t_start = time[0], dt = time - t_start */
    const double t_start = t[0];
    double* dt = (double*)malloc(sizeof(double) * (size_t)n);
    if (!dt) return ORC_ENOMEM;
    for (int64_t i = 0; i < n; ++i) dt[i] = t[i] - t_start;
    /* v42_parity.py:66-67: cp.sum(weights) and cp.sum(flux * weights), parallel
     * tree reductions; pairwise sums stand in for them (a sequential sum of n
     * equal weights drifts by up to n/2 ulp, which the kernel's
     * y_out = (tot_y - y_in_sum) / (tot_w - ivar_in) turns into a relative
     * depth error of order n * ulp / depth for sums near n * w) */
    const double tot_w = pairwise_sum(n, y, w, 0);
    const double tot_y = pairwise_sum(n, y, w, 1);
    /* vbls_v42_parity.cu:36-41 */
    double min_dur = durations[0];
    for (int k = 1; k < nd; ++k)
        if (durations[k] < min_dur) min_dur = durations[k];
    const double bin_dur = min_dur / (double)oversample;
    const double inv_bin_dur = 1.0 / bin_dur;
    int* dur_bins = (int*)malloc(sizeof(int) * (size_t)nd);
    if (!dur_bins) { free(dt); return ORC_ENOMEM; }
    for (int k = 0; k < nd; ++k) dur_bins[k] = (int)round(durations[k] * inv_bin_dur);

    double pmax = periods[0];
    for (int64_t p = 1; p < np; ++p)
        if (periods[p] > pmax) pmax = periods[p];
    int64_t cap = (int64_t)ceil(pmax * inv_bin_dur) + oversample + 2;
    if (max_bins > 0 && cap > max_bins + 2) cap = max_bins + 2;

    int err = ORC_OK;
    set_threads(nthreads);
#pragma omp parallel
    {
        bin2* bins = (bin2*)malloc(sizeof(bin2) * (size_t)cap);
        if (!bins) {
#pragma omp atomic write
            err = ORC_ENOMEM;
        } else {
#pragma omp for schedule(dynamic, 4)
            for (int64_t p = 0; p < np; ++p)
                ref_binned_period(n, dt, y, w, tot_w, tot_y, t_start, periods[p], bin_dur,
                                  inv_bin_dur, oversample, max_bins, nd, dur_bins, objective, bins,
                                  &power[p], &depth[p], &depth_err[p], &t0[p], &duration[p],
                                  &window[p], &gap[p]);
            free(bins);
        }
    }
    free(dur_bins);
    free(dt);
    return err;
}

/*
 * One period of the fixed-bin geometry (bls.cu, SCALAR_T=double).
 * bls.cu:48-68    fold: phase = frac(t_rel*inv_p), bin = int(phase*n_bins), drop if out of range
 * bls.cu:81-98    inclusive prefix; totals = last prefix entry
 * bls.cu:105-142  circular windows, n_dur_bins = int(dur*inv_p*n_bins + 0.5), score s^2/(r(1-r))
 * bls.cu:165      power = sqrt(max(0, score))
 */
static void ref_fixed_period(int64_t n, const double* t_rel, const double* f, const double* w,
                             double t_start, double inv_p, int n_bins, int nd,
                             const double* durations, bin2* bins, double* o_power,
                             double* o_depth, double* o_derr, double* o_t0, double* o_dur,
                             int32_t* o_win, double* o_gap)
{
    memset(bins, 0, sizeof(bin2) * (size_t)n_bins);
    const double nbd = (double)n_bins;
    for (int64_t i = 0; i < n; ++i) {
        double phase = t_rel[i] * inv_p;
        phase -= floor(phase);
        const int b = (int)(phase * nbd);
        if (b >= 0 && b < n_bins) {
            bins[b].c += w[i];
            bins[b].f += f[i] * w[i];
        }
    }
    for (int j = 1; j < n_bins; ++j) {
        bins[j].c += bins[j - 1].c;
        bins[j].f += bins[j - 1].f;
    }
    const double tot_c = bins[n_bins - 1].c, tot_f = bins[n_bins - 1].f;
    const double p = 1.0 / inv_p;

    double best = -1.0, second = -1.0;
    double b_t0 = 0.0, b_dur = 0.0, b_depth = 0.0, b_derr = 0.0;
    int32_t b_win = -1;
    for (int s = 0; s < n_bins; ++s) {
        for (int k = 0; k < nd; ++k) {
            const double dur = durations[k];
            int ndb = (int)fma(dur * inv_p, nbd, 0.5);
            if (ndb < 1) ndb = 1;
            if (ndb >= n_bins) continue;
            const int e = s + ndb - 1;
            double cc, cf;
            const double pc = s > 0 ? bins[s - 1].c : 0.0;
            const double pf = s > 0 ? bins[s - 1].f : 0.0;
            if (e < n_bins) {
                cc = bins[e].c - pc;
                cf = bins[e].f - pf;
            } else {
                const int we = e % n_bins;
                cc = (tot_c - pc) + bins[we].c;
                cf = (tot_f - pf) + bins[we].f;
            }
            if (cc > 0.0 && cc < tot_c) {
                const double r = cc / tot_c;
                const double sv = fma(-r, tot_f, cf);
                const double score = (sv * sv) / (r * (1.0 - r));
                if (score > best) {
                    second = best;
                    best = score;
                    b_t0 = fma((double)s / nbd, p, t_start);
                    b_dur = dur;
                    const double in_mean = cf / cc;
                    const double out_mean = (tot_f - cf) / (tot_c - cc);
                    b_depth = out_mean - in_mean;
                    b_derr = sqrt(1.0 / cc + 1.0 / (tot_c - cc));
                    b_win = s * nd + k;
                } else if (score > second) {
                    second = score;
                }
            }
        }
    }
    *o_power = sqrt(best > 0.0 ? best : 0.0);
    *o_t0 = b_t0;
    *o_dur = b_dur;
    *o_depth = b_depth;
    *o_derr = b_derr;
    *o_win = b_win;
    *o_gap = (best > 0.0 && second > -1.0) ? (best - second) / best : 1.0;
}

int orc_ref_fixed(int64_t n, const double* t, const double* y, const double* w, int64_t np,
                  const double* periods, int32_t nd, const double* durations, int32_t n_bins,
                  int32_t nthreads, double* power, double* depth, double* depth_err, double* t0,
                  double* duration, int32_t* window, double* gap)
{
    if (n <= 0 || np <= 0 || nd <= 0 || n_bins < 2) return ORC_EINVAL;
    double* t_rel = (double*)malloc(sizeof(double) * (size_t)n);
    double* f = (double*)malloc(sizeof(double) * (size_t)n);
    double* ww = (double*)malloc(sizeof(double) * (size_t)n);
    if (!t_rel || !f || !ww) { free(t_rel); free(f); free(ww); return ORC_ENOMEM; }
    /* gpu_bls.py:60-69 -- weights, weighted-mean subtraction (cp.sum: tree
     * reductions, restated as pairwise sums) */
    for (int64_t i = 0; i < n; ++i) ww[i] = w ? w[i] : 1.0;
    const double w_sum = pairwise_sum(n, y, ww, 0);
    const double wy_sum = pairwise_sum(n, y, ww, 1);
    const double w_mean = wy_sum / w_sum;
    const double t_start = t[0]; /* gpu_bls.py:121 */
    for (int64_t i = 0; i < n; ++i) {
        f[i] = y[i] - w_mean;
        t_rel[i] = t[i] - t_start;
    }
    int err = ORC_OK;
    set_threads(nthreads);
#pragma omp parallel
    {
        bin2* bins = (bin2*)malloc(sizeof(bin2) * (size_t)n_bins);
        if (!bins) {
#pragma omp atomic write
            err = ORC_ENOMEM;
        } else {
#pragma omp for schedule(dynamic, 4)
            for (int64_t p = 0; p < np; ++p) {
                const double inv_p = 1.0 / periods[p]; /* gpu_bls.py:76-77 (host, FP64) */
                ref_fixed_period(n, t_rel, f, ww, t_start, inv_p, n_bins, nd, durations, bins,
                                 &power[p], &depth[p], &depth_err[p], &t0[p], &duration[p],
                                 &window[p], &gap[p]);
            }
            free(bins);
        }
    }
    free(t_rel);
    free(f);
    free(ww);
    return err;
}

/* ------------------------------------------------------------------------- */
/* (B) the engine's exact arithmetic                                          */
/* ------------------------------------------------------------------------- */

/* A window length in bins from its real value, as the engine forms it: at
 * least 1 (NaN: 1) and at most 2^28 (every bin count is below 2^27, so a
 * clamped window is skipped exactly as the unclamped one). */
static int eng_len(double v)
{
    if (v >= 268435456.0) return 268435456;
    return v >= 1.0 ? (int)v : 1;
}

/* Per-point fixed-point magnitude bound |q| <= 2^qbits with
 * qbits = min(27, 63 - 2*bitlen(n)), bitlen(n) = number of bits of the point
 * count n: the engine's 32-bit split histogram words cannot overflow. */
static int eng_qbits(int64_t n)
{
    const int bl = n > 0 ? 64 - __builtin_clzll((unsigned long long)n) : 0;
    const int b = 63 - 2 * bl;
    return b < 27 ? b : 27;
}

typedef struct {
    double t_start;
    double shift;
    int64_t qw_tot;
    int64_t qy_tot;
    int64_t qy_abs;
    int32_t s_w;
    int32_t s_y;
} orc_stage_stats;

/* Scale exponent s such that m * 2^s <= 2^qbits for m = max |value|. */
static int q_scale(double m, int qbits)
{
    if (!(m > 0.0)) return 0;
    int e;
    frexp(m, &e); /* m = f * 2^e, f in [0.5, 1) so m < 2^e */
    return qbits - e;
}

/*
 * Deterministic staging of one light curve:
 *   t_start = t[0], dt = t - t_start
 *   w (FP32, NULL = 1) quantised to q_w = rint(w * 2^s_w)
 *   shift c = weighted mean of y from exact integer sums
 *   q_y = rint(w*(y - c) * 2^s_y)
 * Every reduction is a max or an integer sum, so the result does not depend
 * on the order in which points are visited.
 */
int orc_eng_stage(int64_t n, const double* t, const double* y, const float* w, double* dt,
                  int32_t* qw, int32_t* qy, orc_stage_stats* st)
{
    if (n <= 0) return ORC_EINVAL;
    double wmax = 0.0, amax = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double wi = w ? (double)w[i] : 1.0;
        if (!(wi > 0.0) || !isfinite(wi) || !isfinite(y[i]) || !isfinite(t[i])) return ORC_EINVAL;
        if (wi > wmax) wmax = wi;
        const double a = fabs(wi * y[i]);
        if (a > amax) amax = a;
    }
    const int qbits = eng_qbits(n);
    const int s_w = q_scale(wmax, qbits);
    const int s_a = q_scale(amax, qbits);
    int64_t sum_qw = 0, sum_qa = 0;
    for (int64_t i = 0; i < n; ++i) {
        const double wi = w ? (double)w[i] : 1.0;
        sum_qw += (int64_t)llrint(ldexp(wi, s_w));
        sum_qa += (int64_t)llrint(ldexp(wi * y[i], s_a));
    }
    const double shift = ldexp((double)sum_qa / (double)sum_qw, s_w - s_a);
    double vmax = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double wi = w ? (double)w[i] : 1.0;
        const double v = fabs(wi * (y[i] - shift));
        if (v > vmax) vmax = v;
    }
    const int s_y = q_scale(vmax, qbits);
    int64_t qw_tot = 0, qy_tot = 0, qy_abs = 0;
    const double t_start = t[0];
    for (int64_t i = 0; i < n; ++i) {
        const double wi = w ? (double)w[i] : 1.0;
        const int32_t a = (int32_t)llrint(ldexp(wi, s_w));
        const int32_t b = (int32_t)llrint(ldexp(wi * (y[i] - shift), s_y));
        qw[i] = a;
        qy[i] = b;
        dt[i] = t[i] - t_start;
        qw_tot += a;
        qy_tot += b;
        qy_abs += b < 0 ? -(int64_t)b : (int64_t)b;
    }
    st->t_start = t_start;
    st->shift = shift;
    st->qw_tot = qw_tot;
    st->qy_tot = qy_tot;
    st->qy_abs = qy_abs;
    st->s_w = s_w;
    st->s_y = s_y;
    return ORC_OK;
}

/* astropy-binned fold, identical to the engine's: FP64, fma for ph. */
static inline int eng_fold_binned(double d, double period, double inv_period, double inv_bin_dur,
                                  int n_bins)
{
    const double ph = fma(-period, floor(d * inv_period), d);
    int ind = (int)(ph * inv_bin_dur) + 1;
    if (ind > n_bins) ind = n_bins;
    if (ind < 0) ind = 0;
    return ind;
}

/* fixed-bin fold; returns the histogram slot (bin + 1) or -1 when dropped. */
static inline int eng_fold_fixed(double d, double inv_p, double nbd, int n_bins)
{
    double phase = d * inv_p;
    phase = phase - floor(phase);
    const int b = (int)(phase * nbd);
    return (b >= 0 && b < n_bins) ? b + 1 : -1;
}

/*
 * Exact comparison of two non-negative-denominator rationals a = an/ad and
 * b = bn/bd given as floats: returns 1 when an*bd > bn*ad.  The two products
 * are split into rounded value plus exact fma residual, so the comparison is
 * exact (no overflow/underflow for the normalised magnitudes used here).
 */
static inline int eng_ratio_gt(float an, float ad, float bn, float bd, int* eq)
{
    const float p = an * bd;
    const float q = bn * ad;
    *eq = 0;
    if (p != q) return p > q;
    const float e1 = fmaf(an, bd, -p);
    const float e2 = fmaf(bn, ad, -q);
    if (e1 != e2) return e1 > e2;
    *eq = 1;
    return 0;
}

typedef struct {
    float num, den;
    int32_t key;
} eng_cand;

static inline void eng_consider(eng_cand* best, float num, float den, int32_t key)
{
    int eq;
    const int gt = eng_ratio_gt(num, den, best->num, best->den, &eq);
    if (gt || (eq && key < best->key)) {
        best->num = num;
        best->den = den;
        best->key = key;
    }
}

/* Window-search constants.  Prefix sums are exact FP64 values scaled by
 * 2^-ew (weights) and 2^-ey (flux) with W_total < 2^ew, sum|q_y| <= 2^ey. */
typedef struct {
    double wtot, ytot; /* scaled exact totals */
    float c1;          /* ytot / wtot */
    double thr;        /* 1e-15 in scaled weight units */
} eng_consts;

static int exp_above(double v)
{
    int e = 0;
    if (v > 0.0) frexp(v, &e);
    return e;
}

/* FP32 num/den of a window (score proportional to the objective):
 * sigma = (S/W) W_in - S_in, num = sigma^2, den = W_in W_out.  Returns 0 if
 * the window is skipped. */
static inline int eng_window_score(double dw, double dy, const eng_consts* kc, int dip_only,
                                   float* num, float* den)
{
    const double wo = kc->wtot - dw;
    const float fdw = (float)dw;
    const float fwo = (float)wo;
    const float sig = fmaf(kc->c1, fdw, -(float)dy);
    if (dip_only && !(sig >= 0.0f)) return 0;
    *num = sig * sig;
    *den = fdw * fwo;
    return 1;
}

/* The same score for curves whose weights are all equal (and n < 2^24):
 * the engine evaluates it on exact FP32 point counts, W_in = fdw points,
 * N points in the histogram, c1 = S/N (the score changes by the constant
 * factor qw0^2 only). */
static inline int eng_window_score_cnt(float fdw, double dy, float fN, float c1n, int dip_only,
                                       float* num, float* den)
{
    const float fwo = fN - fdw;
    const float sig = fmaf(c1n, fdw, -(float)dy);
    if (dip_only && !(sig >= 0.0f)) return 0;
    *num = sig * sig;
    *den = fdw * fwo;
    return 1;
}

/* Uniform weights with fewer than 2^24 points: windows are scored on counts. */
static int eng_counting(int64_t n, const int32_t* qw)
{
    if (n >= (1LL << 24)) return 0;
    for (int64_t i = 1; i < n; ++i)
        if (qw[i] != qw[0]) return 0;
    return 1;
}

/* FP64 statistics of the winning window; dw, dy scaled by 2^-ew, 2^-ey */
static void eng_finalize(double dw, double dy, double wtot, double ytot, int s_w, int s_y,
                         int objective, double* power, double* depth, double* derr)
{
    const double w_in = ldexp(dw, -s_w);
    const double w_out = ldexp(wtot - dw, -s_w);
    const double s_in = ldexp(dy, -s_y);
    const double s_out = ldexp(ytot - dy, -s_y);
    const double y_in = s_in / w_in;
    const double y_out = s_out / w_out;
    const double dep = y_out - y_in;
    const double de = sqrt(1.0 / w_in + 1.0 / w_out);
    double pw;
    if (objective == OBJ_FAST) {
        /* s^2/(r(1-r)) with r = W_in/W, s = S_in - r*S  ==  depth^2 * W_in*W_out */
        const double sc = dep * dep * (w_in * w_out);
        pw = sqrt(sc);
    } else if (objective == OBJ_LIKELIHOOD) {
        pw = 0.5 * dep * dep * (w_in * w_out) / (w_in + w_out);
    } else {
        pw = dep / de;
    }
    *power = pw > 0.0 ? pw : 0.0;
    *depth = dep;
    *derr = de;
}

int orc_eng_binned(int64_t n, const double* dt, const int32_t* qw, const int32_t* qy,
                   const orc_stage_stats* st, int64_t np, const double* periods, int32_t nd,
                   const double* durations, int32_t oversample, int32_t max_bins,
                   int32_t objective, int32_t nthreads, float* power, float* depth,
                   float* depth_err, double* t0, float* duration, int32_t* window,
                   int32_t* point_bins)
{
    if (n <= 0 || np <= 0 || nd <= 0 || oversample < 1) return ORC_EINVAL;
    if (max_bins > 0 && max_bins < oversample + 2) return ORC_EINVAL;
    if (objective != OBJ_SNR && objective != OBJ_LIKELIHOOD) return ORC_EINVAL;
    double min_dur = durations[0];
    for (int k = 1; k < nd; ++k)
        if (durations[k] < min_dur) min_dur = durations[k];
    const double bin_dur = min_dur / (double)oversample;
    const double inv_bin_dur = 1.0 / bin_dur;
    int dur_bins[64];
    if (nd > 64) return ORC_EINVAL;
    for (int k = 0; k < nd; ++k) dur_bins[k] = eng_len(round(durations[k] * inv_bin_dur));
    double pmax = periods[0];
    for (int64_t p = 1; p < np; ++p)
        if (periods[p] > pmax) pmax = periods[p];
    int64_t cap = (int64_t)ceil(pmax * inv_bin_dur) + oversample + 2;
    if (max_bins > 0 && cap > max_bins + 2) cap = max_bins + 2;
    const int ew = exp_above((double)st->qw_tot), ey = exp_above((double)st->qy_abs);
    const double w_tot = ldexp((double)st->qw_tot, -ew), y_tot = ldexp((double)st->qy_tot, -ey);
    eng_consts kc;
    kc.wtot = w_tot;
    kc.ytot = y_tot;
    kc.c1 = w_tot > 0.0 ? (float)(y_tot / w_tot) : 0.0f;
    kc.thr = ldexp(1e-15, st->s_w - ew);
    const int counting = eng_counting(n, qw);
    const float fN = (float)n;
    const float c1n = (float)(y_tot / (double)n);

    int err = ORC_OK;
    set_threads(nthreads);
#pragma omp parallel
    {
        int64_t* hw = (int64_t*)malloc(sizeof(int64_t) * 3 * (size_t)cap);
        double* cw = (double*)malloc(sizeof(double) * 2 * (size_t)cap);
        float* cc = (float*)malloc(sizeof(float) * (size_t)cap);
        if (!hw || !cw || !cc) {
#pragma omp atomic write
            err = ORC_ENOMEM;
        } else {
            int64_t* hy = hw + cap;
            int64_t* hc = hw + 2 * cap;
            double* cy = cw + cap;
#pragma omp for schedule(dynamic, 4)
            for (int64_t p = 0; p < np; ++p) {
                const double period = periods[p];
                const double inv_period = 1.0 / period;
                int n_bins = (int)ceil(period * inv_bin_dur) + oversample;
                if (max_bins > 0 && n_bins >= max_bins) n_bins = max_bins - 1;
                memset(hw, 0, sizeof(int64_t) * (size_t)(n_bins + 1));
                memset(hy, 0, sizeof(int64_t) * (size_t)(n_bins + 1));
                memset(hc, 0, sizeof(int64_t) * (size_t)(n_bins + 1));
                for (int64_t i = 0; i < n; ++i) {
                    const int ind = eng_fold_binned(dt[i], period, inv_period, inv_bin_dur, n_bins);
                    if (point_bins) point_bins[p * n + i] = ind;
                    hw[ind] += qw[i];
                    hy[ind] += qy[i];
                    hc[ind] += 1;
                }
                for (int j = 1, ind = n_bins - oversample; j <= oversample; ++j, ++ind) {
                    hw[ind] = hw[j];
                    hy[ind] = hy[j];
                    hc[ind] = hc[j];
                }
                int64_t aw = 0, ay = 0, ac = 0;
                for (int j = 0; j <= n_bins; ++j) {
                    aw += hw[j];
                    ay += hy[j];
                    ac += hc[j];
                    cw[j] = ldexp((double)aw, -ew);
                    cy[j] = ldexp((double)ay, -ey);
                    cc[j] = (float)ac;
                }
                eng_cand best = {-1.0f, 1.0f, INT32_MAX};
                for (int s = 0; s < n_bins; ++s) {
                    for (int k = 0; k < nd; ++k) {
                        const int d = dur_bins[k];
                        if (s + d > n_bins) continue;
                        const double dw = cw[s + d] - cw[s];
                        const double dy = cy[s + d] - cy[s];
                        if (dw < kc.thr || (w_tot - dw) < kc.thr) continue;
                        float num, den;
                        if (counting) {
                            if (!eng_window_score_cnt(cc[s + d] - cc[s], dy, fN, c1n, 1, &num,
                                                      &den))
                                continue;
                        } else if (!eng_window_score(dw, dy, &kc, 1, &num, &den)) {
                            continue;
                        }
                        eng_consider(&best, num, den, s * nd + k);
                    }
                }
                if (best.key == INT32_MAX) {
                    power[p] = 0.0f; depth[p] = 0.0f; depth_err[p] = 0.0f;
                    t0[p] = 0.0; duration[p] = 0.0f; window[p] = -1;
                } else {
                    const int s = best.key / nd, k = best.key % nd, d = dur_bins[k];
                    const double dw = cw[s + d] - cw[s];
                    const double dy = cy[s + d] - cy[s];
                    double pw, dep, de;
                    eng_finalize(dw, dy, w_tot, y_tot, st->s_w - ew, st->s_y - ey, objective, &pw,
                                 &dep, &de);
                    const double durv = (double)d * bin_dur;
                    power[p] = (float)pw;
                    depth[p] = (float)dep;
                    depth_err[p] = (float)de;
                    duration[p] = (float)durv;
                    t0[p] = fmod((double)s * bin_dur + 0.5 * durv + st->t_start, period);
                    window[p] = best.key;
                }
            }
        }
        free(hw);
        free(cw);
        free(cc);
    }
    return err;
}

int orc_eng_fixed(int64_t n, const double* dt, const int32_t* qw, const int32_t* qy,
                  const orc_stage_stats* st, int64_t np, const double* periods, int32_t nd,
                  const double* durations, int32_t n_bins, int32_t nthreads, float* power,
                  float* depth, float* depth_err, double* t0, float* duration, int32_t* window,
                  int32_t* point_bins)
{
    if (n <= 0 || np <= 0 || nd <= 0 || n_bins < 2) return ORC_EINVAL;
    int err = ORC_OK;
    const double nbd = (double)n_bins;
    const int ew = exp_above((double)st->qw_tot), ey = exp_above((double)st->qy_abs);
    const int counting = eng_counting(n, qw);
    set_threads(nthreads);
#pragma omp parallel
    {
        int64_t* hw = (int64_t*)malloc(sizeof(int64_t) * 3 * (size_t)(n_bins + 1));
        double* cw = (double*)malloc(sizeof(double) * 2 * (size_t)(n_bins + 1));
        float* cc = (float*)malloc(sizeof(float) * (size_t)(n_bins + 1));
        if (!hw || !cw || !cc) {
#pragma omp atomic write
            err = ORC_ENOMEM;
        } else {
            int64_t* hy = hw + (n_bins + 1);
            int64_t* hc = hw + 2 * (n_bins + 1);
            double* cy = cw + (n_bins + 1);
#pragma omp for schedule(dynamic, 4)
            for (int64_t p = 0; p < np; ++p) {
                const double inv_p = 1.0 / periods[p];
                memset(hw, 0, sizeof(int64_t) * (size_t)(n_bins + 1));
                memset(hy, 0, sizeof(int64_t) * (size_t)(n_bins + 1));
                memset(hc, 0, sizeof(int64_t) * (size_t)(n_bins + 1));
                for (int64_t i = 0; i < n; ++i) {
                    const int slot = eng_fold_fixed(dt[i], inv_p, nbd, n_bins);
                    if (point_bins) point_bins[p * n + i] = slot;
                    if (slot >= 0) {
                        hw[slot] += qw[i];
                        hy[slot] += qy[i];
                        hc[slot] += 1;
                    }
                }
                int64_t aw = 0, ay = 0, ac = 0;
                for (int j = 0; j <= n_bins; ++j) {
                    aw += hw[j];
                    ay += hy[j];
                    ac += hc[j];
                    cw[j] = ldexp((double)aw, -ew);
                    cy[j] = ldexp((double)ay, -ey);
                    cc[j] = (float)ac;
                }
                const double w_tot = cw[n_bins], y_tot = cy[n_bins];
                const float fN = cc[n_bins];
                const float c1n = fN > 0.0f ? (float)(y_tot / (double)fN) : 0.0f;
                eng_cand best = {-1.0f, 1.0f, INT32_MAX};
                if (w_tot > 0.0) {
                    eng_consts kc;
                    kc.wtot = w_tot;
                    kc.ytot = y_tot;
                    kc.c1 = (float)(y_tot / w_tot);
                    kc.thr = 0.0;
                    for (int s = 0; s < n_bins; ++s) {
                        for (int k = 0; k < nd; ++k) {
                            const int L = eng_len(fma(durations[k] * inv_p, nbd, 0.5));
                            if (L >= n_bins) continue;
                            double dw, dy;
                            float fdw;
                            if (s + L <= n_bins) {
                                dw = cw[s + L] - cw[s];
                                dy = cy[s + L] - cy[s];
                                fdw = cc[s + L] - cc[s];
                            } else {
                                dw = (w_tot - cw[s]) + cw[s + L - n_bins];
                                dy = (y_tot - cy[s]) + cy[s + L - n_bins];
                                fdw = (fN - cc[s]) + cc[s + L - n_bins];
                            }
                            if (!(dw > 0.0 && dw < w_tot)) continue;
                            float num, den;
                            if (counting)
                                eng_window_score_cnt(fdw, dy, fN, c1n, 0, &num, &den);
                            else
                                eng_window_score(dw, dy, &kc, 0, &num, &den);
                            eng_consider(&best, num, den, s * nd + k);
                        }
                    }
                }
                if (best.key == INT32_MAX) {
                    power[p] = 0.0f; depth[p] = 0.0f; depth_err[p] = 0.0f;
                    t0[p] = 0.0; duration[p] = 0.0f; window[p] = -1;
                } else {
                    const int s = best.key / nd, k = best.key % nd;
                    const int L = eng_len(fma(durations[k] * inv_p, nbd, 0.5));
                    double dw, dy;
                    if (s + L <= n_bins) {
                        dw = cw[s + L] - cw[s];
                        dy = cy[s + L] - cy[s];
                    } else {
                        dw = (w_tot - cw[s]) + cw[s + L - n_bins];
                        dy = (y_tot - cy[s]) + cy[s + L - n_bins];
                    }
                    double pw, dep, de;
                    eng_finalize(dw, dy, w_tot, y_tot, st->s_w - ew, st->s_y - ey, OBJ_FAST, &pw,
                                 &dep, &de);
                    const double p_ = 1.0 / inv_p;
                    power[p] = (float)pw;
                    depth[p] = (float)dep;
                    depth_err[p] = (float)de;
                    duration[p] = (float)durations[k];
                    t0[p] = fma((double)s / nbd, p_, st->t_start);
                    window[p] = best.key;
                }
            }
        }
        free(hw);
        free(cw);
        free(cc);
    }
    return err;
}
