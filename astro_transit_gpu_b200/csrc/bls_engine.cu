// bls_engine.cu -- B200 (sm_100a) Box Least Squares engine behind the C ABI of
// include/astrotransit_b200.h.
//
// Hot path (one astropy-style BLS per (light curve, period)):
//   stage kernel   one CTA per curve: t_start = t[0], dt = t - t_start (FP64),
//                  deterministic fixed-point staging q_w = rint(w*2^s_w),
//                  q_y = rint(w*(y-c)*2^s_y) (|q| <= 2^27), per-curve totals,
//                  the curve's histogram word layout (kPack*) and staged order.
//   search kernel  persistent; CTAs (512 threads, two per SM, or 256 threads,
//                  four per SM, chosen per plan) pop (curve, period-chunk)
//                  tiles from a device counter.  Periods of a tile are packed
//                  into groups whose histograms fit shared memory; each
//                  thread keeps kR = 4
//                  time-ordered points in registers and folds them into every
//                  period of the group (FP64 fold, identical to the reference's
//                  per-point formula), adding each point's exact integer sums
//                  to its bin with two to four 32-bit shared-memory reductions
//                  on split words.  Teams of warps then scan each histogram
//                  (exact int64 -> exact FP64), evaluate every (start,
//                  duration) window in FP32 with an exact rational
//                  comparison, and re-evaluate the winner in FP64.
//   best kernel    per-curve argmax over the period grid.
//
// Reference semantics followed (paths within ubunbun18/Astro_Transit_GPU):
//   astropy-binned geometry  search/kernels/vbls_v42_parity.cu:36-129
//   fixed-bin geometry       search/kernels/bls.cu:47-169
//   host prologues           search/v42_parity.py:42-67, search/gpu_bls.py:57-78
//
// Build: nvcc -gencode arch=compute_100a,code=sm_100a -fmad=false (every
// intended fused multiply-add is an explicit fma()), see build.py.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/astrotransit_b200.h"

#define ATB_VERSION "astrotransit-b200 0.1.0 sm_100a"

namespace {

#ifndef ATB_BLOCK
#define ATB_BLOCK 512
#endif
#ifndef ATB_MIN_BLOCKS
#define ATB_MIN_BLOCKS 2
#endif
#ifndef ATB_POINTS_PER_THREAD
#define ATB_POINTS_PER_THREAD 4
#endif
// Search-CTA shapes: kBlock threads with kMinBlocks CTAs per SM (the default
// for the astropy-binned geometry), or kBlockB threads with kMinBlocksB CTAs
// per SM (the fixed-bin default; atb_params.cta_threads selects either).  The
// device code takes the CTA size from blockDim.x; shared arrays are sized for
// the larger shape.
constexpr int kBlock = ATB_BLOCK;            // threads of a search CTA
constexpr int kMinBlocks = ATB_MIN_BLOCKS;   // resident search CTAs per SM
constexpr int kBlockB = 256;
constexpr int kMinBlocksB = 4;
constexpr int kMaxWarps = (kBlock > kBlockB ? kBlock : kBlockB) / 32;
// Teams of tw warps (tw a power of two) must tile the CTA exactly, so that
// every warp of a team reaches the team's named barrier.
static_assert(kBlock % 32 == 0 && kBlock / 32 >= 2 && kBlock / 32 <= 32 &&
                  ((kBlock / 32) & (kBlock / 32 - 1)) == 0 && kBlockB / 32 >= 2 &&
                  ((kBlockB / 32) & (kBlockB / 32 - 1)) == 0,
              "search CTA: a power-of-two number of warps, at most 1024 threads");
constexpr int kBenchBlock = 512;  // threads of the microbenchmark kernels
constexpr int kR = ATB_POINTS_PER_THREAD;    // consecutive points a thread holds in registers
constexpr int kTileP = 64;             // periods per work-queue tile
constexpr int kMaxG = 64;              // periods per shared-memory group
constexpr int kMaxDur = 32;            // durations per curve
// Window lengths in bins are clamped to kLenCap: every bin count is below 2^27,
// so a clamped window never fits a period (it is skipped exactly as the
// unclamped one) and start + length never overflows an int.
constexpr int kLenCap = 1 << 28;
constexpr int kStageAlign = 32;        // staged curves start at multiples of 32 points
constexpr int kStageBlock = 256;
constexpr double kDefaultMergeRun = 8.0;   // atb_params.merge_run = 0
// atb_params.cta_threads = 0 with fixed bins: four 256-thread CTAs per SM
// (measured faster than two 512-thread ones for fixed bins; slower for the
// binned geometry, whose larger histograms want the bigger shared-memory share)
constexpr int kDefaultFixedThreads = kBlockB;
constexpr int kChunk = 32 * kR;        // staged points of one warp's fold step
constexpr double kMagicSlot = 4503599627370497.0;   // 2^52 + 1: x + C (rz) = 2^52 + int(x) + 1, x in (-1, 2^31 - 1)
constexpr double kMagicFloor = 6755399441055744.0;  // 1.5*2^52: (m + C)(rd) - C = floor(m), |m| < 2^50

// Histogram word layouts (per curve):
//   kPackSplit  weights not uniform: words (x, y) = weight sums split at
//               `lobits`, (z, w) = flux sums split the same way
//   kPackCount  uniform weights: x = point count, (z, w) = flux sums split
//   kPackTight  uniform weights and at most M < 2^12 points can share a bin
//               (b = bits of M): x = count * 2^(32-b) + sum(q mod 2^(32-2b)),
//               z = sum(q >> (32-2b)); neither word can overflow, and a point
//               costs two shared-memory reductions instead of three.
//               M = (floor(T / P_min) + 3) * K, with T the curve's time span and
//               K the most points inside any time window one bin wide: points
//               of one bin in one cycle lie in such a window, and the rounded
//               cycle index takes at most floor(T / P) + 2 values.  High words
//               sum to < M * 2^(27 - lobits) <= 2^(3b - 5) <= 2^31.
//   Checked tight: uniform weights with no proven bound, but few points per bin
//               on average (below kCheckedTightAvg per real bin at the grid's
//               coarsest binning): the tight words with b = 12, and every
//               period's histogram checked before use -- a count field that
//               overflowed (a bin holding 2^12 points or more) makes the decoded
//               counts sum to less than n (each such bin loses at least
//               2^12 - 1 points while carries add at most 1), and that period
//               is folded again in the count layout (kPackCountT), whose words
//               are derived from the same staged tight words.
constexpr int kPackSplit = 0;
constexpr int kPackCount = 1;
constexpr int kPackTight = 2;
constexpr int kPackCountT = 3;  // count-layout words computed from staged tight words
constexpr int kTightMaxBits = 12;
constexpr double kCheckedTightAvg = 1024.0;

// Per-curve fixed-point layout.  Point values are quantised to |q| <= 2^qbits;
// histogram words hold the low `lobits` bits and the arithmetic-shifted high
// part of each value in separate 32-bit counters, sized so neither can
// overflow for the curve's point count n (bitlen = bits of n):
//   low sums  < n * 2^lobits            <= 2^32
//   high sums < n * 2^(qbits - lobits)  <= 2^31
// with lobits = 32 - bitlen and qbits = min(27, 63 - 2*bitlen) (27 is the most
// the two-word layouts hold with up to 2^12 - 1 points per bin).
struct CurveStat {
    double t_start;
    double shift;
    long long qw_tot;
    long long qy_tot;
    long long qy_abs;
    int s_w;
    int s_y;
    double bin_dur;      // BINNED: min(duration) / oversample
    double inv_bin_dur;  // BINNED: 1 / bin_dur
    double dt_absmax;    // max |t - t_start|
    int n_dur;
    int qbits;
    int lobits;
    int qw0;        // the common q_w when uniform_w
    int uniform_w;  // every q_w equal: the weight words count points
    int thr_unit;   // 1e-15 (the reference's empty-window threshold) is below one
                    // quantised weight unit: "W < 1e-15" is then "W == 0"
    int ew;         // prefix sums are stored as exact FP64 values scaled by 2^-ew (weights)
    int ey;         // and 2^-ey (flux), so that |W| < 1 and |S| <= 1
    int packmode;   // histogram word layout, see kPack*
    int cshift;     // kPackTight: bit position of the point count in word x
    int occ_bits;   // bits of the bin-occupancy bound M (64: none)
    int cnt_win;    // uniform weights and fewer than 2^24 points: the window search
                    // works on exact FP32 point counts instead of FP64 weight sums
    int n_cnt;      // number of points (cnt_win)
    int ilv;        // staged order interleaved within whole chunks (staged_pos)
    double density; // points per unit time, (n - 1) / (time span); 0 for n < 2
    int tcheck;     // kPackTight without a proven bound: each period's counts are checked
    int stage_lob;  // kPackTight: low flux bits of the staged word x (32 - 2b)
    int stage_csh;  // kPackTight: bit position of the count in the staged word x (32 - b)
};

struct StageArgs {
    const long long* pt_off;
    const long long* t_off;
    const long long* stage_off;
    const long long* dur_beg;
    const int* dur_cnt;
    const double* t;
    const void* y;
    const float* w;
    const double* durations;
    double* sdt;
    int* sqw;  // q_w per point, or the fold's first word (tight, count layouts)
    int* sqy;  // q_y per point, or the fold's flux word (tight layout)
    CurveStat* stats;
    int* dbins;  // [n_curves * kMaxDur]
    int oversample;
    int* status;
    // period grids, for the bin-occupancy bound of kPackTight (NULL: no bound)
    const double* periods;
    const long long* per_beg;
    const long long* per_cnt;
    int geometry;
    int n_bins_fixed;
    int max_bins;
};

struct SearchArgs {
    int objective;
    int n_bins_fixed;
    int oversample;
    int max_bins;
    int n_curves;
    int cap;  // shared-memory histogram entries
    long long n_tiles;
    const long long* pt_off;
    const long long* stage_off;
    const long long* per_beg;
    const long long* per_cnt;
    const long long* dur_beg;
    const int* dur_cnt;
    const long long* out_beg;
    const long long* tile_off;
    const int* order;
    const double* periods;
    const double* durations;
    const double* sdt;
    const int* sqw;  // as StageArgs
    const int* sqy;
    const CurveStat* stats;
    const int* dbins;
    float* power;
    float* depth;
    float* depth_err;
    double* t0;
    float* duration;
    int* window;
    longlong2* ghist;
    long long ghist_stride;
    unsigned long long* tile_counter;
    int* status;
    unsigned long long* best_key;  // winner-take-all per-curve records (or NULL)
    int tile_p;                    // periods per work-queue tile (1..kTileP)
    double merge_run;              // expected points per bin from which kFoldChunk is used
};

// ----------------------------------------------------------------------------
// shared device helpers
// ----------------------------------------------------------------------------

__device__ __forceinline__ int q_scale(double m, int qbits) {
    if (!(m > 0.0)) return 0;
    int e;
    frexp(m, &e);
    return qbits - e;
}

__device__ __forceinline__ int bitlen64(long long n) { return n <= 0 ? 0 : 64 - __clzll(n); }
__device__ __forceinline__ int curve_lobits(long long n) { return min(30, 32 - bitlen64(n)); }
__device__ __forceinline__ int curve_qbits(long long n) { return min(27, 63 - 2 * bitlen64(n)); }

// Staged order of a curve's points.  Interleaved (n_full > 0): in every
// whole chunk of kChunk points the kR staged values of lane l are points l,
// l + 32, l + 64, ... of the chunk, so that the lanes of a warp fold 32
// consecutive points at a time, while each thread's values stay
// time-ordered; points of the last, partial chunk keep their order.  n_full =
// the points in whole chunks, 0 for the plain order.
__device__ __forceinline__ long long staged_pos(long long i, long long n_full) {
    if (i >= n_full) return i;
    const int r = (int)(i % kChunk);
    return i - r + (r & 31) * kR + (r >> 5);
}

// the inverse: the point held at staged position q
__device__ __forceinline__ long long staged_point(long long q, long long n_full) {
    if (q >= n_full) return q;
    const int r = (int)(q % kChunk);
    return q - r + (r % kR) * 32 + r / kR;
}

// floor(m) for |m| < 2^50 with two full-rate FP64 additions (exact)
__device__ __forceinline__ double floor_magic(double m) {
    return __dadd_rn(__dadd_rd(m, kMagicFloor), -kMagicFloor);
}

// int(x) + 1 (C truncation toward zero) for x in (-1, 2^31 - 1), with one
// full-rate FP64 addition: the sum lies in [2^52, 2^53), where the spacing of
// doubles is 1, so rounding toward zero leaves 2^52 + int(x) + 1, whose low
// word is the result (0 for x in (-1, 0)).
__device__ __forceinline__ int trunc1_magic(double x) {
    return __double2loint(__dadd_rz(x, kMagicSlot));
}

__device__ __forceinline__ double ll_as_d(long long v) { return __longlong_as_double(v); }

// V42 bin count, vbls_v42_parity.cu:46-47 (cap only when max_bins > 0)
__device__ __forceinline__ int binned_nbins(double period, double inv_bin_dur, int oversample,
                                            int max_bins) {
    double x = ceil(period * inv_bin_dur);
    if (!(x < 1.0e9)) x = 1.0e9;
    int nb = (int)x + oversample;
    if (max_bins > 0 && nb >= max_bins) nb = max_bins - 1;
    return nb;
}

// Exact comparison of candidates a = an/ad and b = bn/bd (floats, positive
// denominators): products split into rounded value + exact fma residual.
// Equal ratios are ordered by the smaller window key.
__device__ __forceinline__ bool cand_better(float an, float ad, int ak, float bn, float bd,
                                            int bk) {
    const float p = __fmul_rn(an, bd);
    const float q = __fmul_rn(bn, ad);
    if (p != q) return p > q;
    const float e1 = __fmaf_rn(an, bd, -p);
    const float e2 = __fmaf_rn(bn, ad, -q);
    if (e1 != e2) return e1 > e2;
    return ak < bk;
}

struct Cand {
    float num, den;
    int key;
};

__device__ __forceinline__ Cand warp_best(Cand c) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float on = __shfl_down_sync(0xffffffffu, c.num, off);
        const float od = __shfl_down_sync(0xffffffffu, c.den, off);
        const int ok = __shfl_down_sync(0xffffffffu, c.key, off);
        if (cand_better(on, od, ok, c.num, c.den, c.key)) {
            c.num = on;
            c.den = od;
            c.key = ok;
        }
    }
    return c;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, off));
    return v;
}

__device__ __forceinline__ long long warp_sum(long long v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// block reductions for the stage kernel (kStageBlock threads)
__device__ double block_max_d(double v, double* sh) {
    v = warp_max(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = sh[0];
    for (int i = 1; i < kStageBlock / 32; ++i) r = max(r, sh[i]);
    return r;
}

__device__ long long block_sum_ll(long long v, long long* sh) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    long long r = 0;
    for (int i = 0; i < kStageBlock / 32; ++i) r += sh[i];
    return r;
}

// ----------------------------------------------------------------------------
// stage kernel: one CTA per light curve
// ----------------------------------------------------------------------------

// Bits of a bound M on the number of points of curve c that can share one
// histogram bin in any period of its grid (64 when no bound is available):
//   M = (floor(T / P_min) + 3) * K,
// T = time span, K = most points inside any closed time window of one bin width
// (astropy-binned: min(duration)/oversample; fixed: P_max/n_bins), widened by a
// relative 1e-6 for rounding.  Requires time-ordered points and, for
// astropy bins, a bin cap (max_bins) that no period of the grid reaches.
__device__ int occupancy_bits(const StageArgs& a, int c, const double* t, long long n, double* shd,
                              long long* shl) {
    // time order
    int unsorted = 0;
    for (long long i = threadIdx.x; i + 1 < n; i += kStageBlock) unsorted |= t[i] > t[i + 1];
    if (__syncthreads_or(unsorted)) return 64;
    // grid extremes
    const double* per = a.periods + a.per_beg[c];
    const long long np = a.per_cnt[c];
    double pmax = 0.0, pinv = 0.0;
    for (long long i = threadIdx.x; i < np; i += kStageBlock) {
        const double P = per[i];
        if (P > 0.0 && P < 1.0e300) {
            pmax = max(pmax, P);
            pinv = max(pinv, 1.0 / P);
        }
    }
    pmax = block_max_d(pmax, shd);
    pinv = block_max_d(pinv, shd);
    if (!(pinv > 0.0)) return 64;
    double width;
    if (a.geometry == ATB_GEOM_BINNED) {
        const double* dur = a.durations + a.dur_beg[c];
        double min_dur = dur[0];
        for (int k = 1; k < a.dur_cnt[c]; ++k) min_dur = min(min_dur, dur[k]);
        width = min_dur / (double)a.oversample;
        // a bin cap that some period reaches piles points into the last bin
        // (vbls_v42_parity.cu:70): no bound then.  Bin counts grow with the
        // period, so the largest period decides (same arithmetic as the search).
        if (a.max_bins > 0 &&
            binned_nbins(pmax, 1.0 / width, a.oversample, 0) >= a.max_bins)
            return 64;
    } else {
        width = pmax / (double)a.n_bins_fixed;
    }
    if (!(width > 0.0) || !isfinite(width)) return 64;
    width = width * (1.0 + 1e-6) + 1e-12;
    // K: each thread scans a contiguous range of window starts with a second pointer
    const long long per_thr = (n + kStageBlock - 1) / kStageBlock;
    const long long i0 = min(n, (long long)threadIdx.x * per_thr);
    const long long i1 = min(n, i0 + per_thr);
    long long kmax = 0;
    if (i0 < i1) {
        long long lo = i0, hi = n;  // first j with t[j] > t[i0] + width
        while (lo < hi) {
            const long long mid = (lo + hi) >> 1;
            if (t[mid] - t[i0] <= width) lo = mid + 1; else hi = mid;
        }
        long long j = lo;
        for (long long i = i0; i < i1; ++i) {
            while (j < n && t[j] - t[i] <= width) ++j;
            kmax = max(kmax, j - i);
        }
    }
    kmax = (long long)block_max_d((double)kmax, shd);
    const double span = n > 0 ? t[n - 1] - t[0] : 0.0;
    const double cycles = floor(span * pinv * (1.0 + 1e-9)) + 3.0;
    const double m = cycles * (double)kmax;
    if (!(m < 4096.0)) return 64;
    return bitlen64((long long)m);
}

// Whether curve c may use the checked tight layout: fewer than
// kCheckedTightAvg points per real bin on average at the grid's coarsest
// binning (fixed: n_bins; astropy-binned: the bins of the smallest period),
// and, for astropy bins, a bin cap (max_bins) that no period reaches (the cap
// piles points into the last bin).  Bins far fuller than the average only cost
// a second fold of their period.
__device__ bool checked_tight_ok(const StageArgs& a, int c, long long n, double* shd) {
    const double* per = a.periods + a.per_beg[c];
    const long long np = a.per_cnt[c];
    double pmax = 0.0, pinv = 0.0;
    for (long long i = threadIdx.x; i < np; i += kStageBlock) {
        const double P = per[i];
        if (P > 0.0 && P < 1.0e300) {
            pmax = max(pmax, P);
            pinv = max(pinv, 1.0 / P);
        }
    }
    pmax = block_max_d(pmax, shd);
    pinv = block_max_d(pinv, shd);
    if (!(pinv > 0.0)) return false;
    double real_bins = (double)a.n_bins_fixed;
    if (a.geometry == ATB_GEOM_BINNED) {
        const double* dur = a.durations + a.dur_beg[c];
        double min_dur = dur[0];
        for (int k = 1; k < a.dur_cnt[c]; ++k) min_dur = min(min_dur, dur[k]);
        const double ibd = 1.0 / (min_dur / (double)a.oversample);
        if (!(ibd > 0.0) || !isfinite(ibd)) return false;
        if (a.max_bins > 0 && binned_nbins(pmax, ibd, a.oversample, 0) >= a.max_bins)
            return false;
        real_bins = (double)(binned_nbins(1.0 / pinv, ibd, a.oversample, 0) - a.oversample);
    }
    return real_bins >= 1.0 && (double)n < kCheckedTightAvg * real_bins;
}

template <typename YT>
__global__ void __launch_bounds__(kStageBlock) stage_kernel(const StageArgs a) {
    __shared__ double shd[kStageBlock / 32];
    __shared__ long long shl[kStageBlock / 32];
    const int c = blockIdx.x;
    const long long p0 = a.pt_off[c];
    const long long n = a.pt_off[c + 1] - p0;
    const long long tb = a.t_off ? a.t_off[c] : p0;
    const double* t = a.t + tb;
    const YT* y = static_cast<const YT*>(a.y) + p0;
    const float* w = a.w ? a.w + p0 : nullptr;
    const long long so = a.stage_off[c];
    const long long n_pad = (n + kR - 1) / kR * kR;
    const int qbits = curve_qbits(n);
    const double t_start = n > 0 ? t[0] : 0.0;

    // pass 1: magnitudes and validity
    double wmax = 0.0, amax = 0.0, tmax = 0.0;
    int bad = 0;
    for (long long i = threadIdx.x; i < n; i += kStageBlock) {
        const double wi = w ? (double)w[i] : 1.0;
        const double yi = (double)y[i];
        if (!(wi > 0.0) || !isfinite(wi) || !isfinite(yi) || !isfinite(t[i])) bad = 1;
        wmax = max(wmax, wi);
        amax = max(amax, fabs(wi * yi));
        tmax = max(tmax, fabs(t[i] - t_start));
    }
    wmax = block_max_d(wmax, shd);
    amax = block_max_d(amax, shd);
    tmax = block_max_d(tmax, shd);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(a.status, 1);
    const int s_w = q_scale(wmax, qbits);
    const int s_a = q_scale(amax, qbits);

    // pass 2: exact integer sums -> the shift c (weighted mean of y); the
    // range of the quantised weights decides the histogram layout
    long long sqw = 0, sqa = 0;
    int qw_min = 0x7fffffff, qw_max = -1;
    for (long long i = threadIdx.x; i < n; i += kStageBlock) {
        const double wi = w ? (double)w[i] : 1.0;
        const double yi = (double)y[i];
        const long long qa = __double2ll_rn(ldexp(wi, s_w));
        sqw += qa;
        sqa += __double2ll_rn(ldexp(wi * yi, s_a));
        qw_min = min(qw_min, (int)qa);
        qw_max = max(qw_max, (int)qa);
    }
    sqw = block_sum_ll(sqw, shl);
    sqa = block_sum_ll(sqa, shl);
    qw_max = (int)block_max_d((double)qw_max, shd);
    qw_min = -(int)block_max_d(-(double)qw_min, shd);
    const bool uniform = n > 0 && qw_min == qw_max;
    int packmode = uniform ? kPackCount : kPackSplit;
    int tight_bits = 64;
    if (uniform && a.periods) tight_bits = occupancy_bits(a, c, t, n, shd, shl);
    if (uniform && tight_bits <= kTightMaxBits && qbits <= 27) packmode = kPackTight;
    // no proven bound: the checked tight layout where bins are sparse on average
    bool tcheck = false;
    if (uniform && packmode != kPackTight && a.periods && qbits <= 27 && n < (1LL << 24) &&
        checked_tight_ok(a, c, n, shd)) {
        packmode = kPackTight;
        tight_bits = kTightMaxBits;
        tcheck = true;
    }
    const int qbits_y = qbits;
    const double shift = sqw != 0 ? ldexp((double)sqa / (double)sqw, s_w - s_a) : 0.0;

    // pass 3: magnitude of w*(y - c)
    double vmax = 0.0;
    for (long long i = threadIdx.x; i < n; i += kStageBlock) {
        const double wi = w ? (double)w[i] : 1.0;
        vmax = max(vmax, fabs(wi * ((double)y[i] - shift)));
    }
    vmax = block_max_d(vmax, shd);
    const int s_y = q_scale(vmax, qbits_y);

    // pass 4: staged arrays (padded with zero-weight points) and totals.
    // Uniform-weight layouts stage the fold's words (see fold_group):
    //   tight  x = (q_w != 0) << cshift | (q_y & lomask), z = q_y >> lobits
    //   count  x = (q_w != 0), and q_y as is
    //   split  q_w and q_y as they are
    const int lob = packmode == kPackTight ? 32 - 2 * tight_bits : curve_lobits(n);
    const int csh = 32 - tight_bits;
    // Staged order: with astropy bins (one bin width for every period),
    // interleaved when the mean spacing of the points reaches the bin width
    // -- a warp's 32 consecutive points then fall in distinct bins, while
    // lanes kR points apart would fall kR bins apart and share banks.  Denser
    // curves keep the plain order: interleaved, up to 32 lanes would add to
    // the same few bins, which serialises.  Fixed bins (P / n_bins, mostly
    // far wider) keep it too; interleaved, an uneven batch of the fast
    // method measured 14 % slower.
    double width = 0.0;
    if (a.geometry == ATB_GEOM_BINNED) {
        const double* dur = a.durations + a.dur_beg[c];
        double md = dur[0];
        for (int k = 1; k < a.dur_cnt[c]; ++k) md = min(md, dur[k]);
        width = md / (double)a.oversample;
    }
    const bool ilv = n > 1 && width > 0.0 && tmax >= width * (double)(n - 1);
    const long long n_full = ilv ? n_pad / kChunk * kChunk : 0;
    long long qw_tot = 0, qy_tot = 0, qy_abs = 0;
    for (long long i = threadIdx.x; i < n_pad; i += kStageBlock) {
        double d = 0.0;
        int qa = 0, qb = 0;
        if (i < n) {
            const double wi = w ? (double)w[i] : 1.0;
            qa = (int)__double2ll_rn(ldexp(wi, s_w));
            qb = (int)__double2ll_rn(ldexp(wi * ((double)y[i] - shift), s_y));
            d = t[i] - t_start;
        }
        int sa = qa, sb = qb;
        if (packmode == kPackTight) {
            sa = (int)((qa != 0 ? (1u << csh) : 0u) + ((unsigned)qb & ((1u << lob) - 1u)));
            sb = qb >> lob;
        } else if (packmode == kPackCount) {
            sa = qa != 0 ? 1 : 0;
        }
        const long long q = so + staged_pos(i, n_full);
        a.sdt[q] = d;
        a.sqw[q] = sa;
        a.sqy[q] = sb;
        qw_tot += qa;
        qy_tot += qb;
        qy_abs += qb < 0 ? -(long long)qb : (long long)qb;
    }
    qw_tot = block_sum_ll(qw_tot, shl);
    qy_tot = block_sum_ll(qy_tot, shl);
    qy_abs = block_sum_ll(qy_abs, shl);

    if (threadIdx.x == 0) {
        const int nd = a.dur_cnt[c];
        const double* dur = a.durations + a.dur_beg[c];
        double min_dur = dur[0];
        for (int k = 1; k < nd; ++k) min_dur = min(min_dur, dur[k]);
        bool bad_dur = !(min_dur > 0.0) || !isfinite(min_dur);
        const double bin_dur = min_dur / (double)a.oversample;
        const double ibd = 1.0 / bin_dur;
        for (int k = 0; k < nd; ++k) {
            // a valid duration is >= min_dur, so its length is >= oversample >= 1
            const double v = round(dur[k] * ibd);
            bad_dur = bad_dur || !(dur[k] > 0.0) || !isfinite(dur[k]);
            a.dbins[c * kMaxDur + k] = v >= (double)kLenCap ? kLenCap : (v >= 1.0 ? (int)v : 1);
        }
        if (bad_dur) atomicOr(a.status, 2);
        CurveStat st;
        st.t_start = t_start;
        st.shift = shift;
        st.qw_tot = qw_tot;
        st.qy_tot = qy_tot;
        st.qy_abs = qy_abs;
        st.s_w = s_w;
        st.s_y = s_y;
        st.bin_dur = bin_dur;
        st.inv_bin_dur = ibd;
        st.dt_absmax = tmax;
        st.n_dur = nd;
        st.qbits = qbits_y;
        st.lobits = curve_lobits(n);
        st.uniform_w = uniform ? 1 : 0;
        st.qw0 = n > 0 ? qw_max : 0;
        st.thr_unit = ldexp(1e-15, s_w) < 1.0 ? 1 : 0;
        int ew = 0, ey = 0;
        if (qw_tot > 0) frexp((double)qw_tot, &ew);
        if (qy_abs > 0) frexp((double)qy_abs, &ey);
        st.ew = ew;
        st.ey = ey;
        st.packmode = packmode;
        if (packmode == kPackTight) {
            st.lobits = 32 - 2 * tight_bits;
            st.cshift = 32 - tight_bits;
        } else {
            st.cshift = 0;
        }
        st.occ_bits = tcheck ? 64 : tight_bits;
        st.tcheck = tcheck ? 1 : 0;
        st.stage_lob = packmode == kPackTight ? 32 - 2 * tight_bits : 0;
        st.stage_csh = packmode == kPackTight ? 32 - tight_bits : 0;
        st.cnt_win = (uniform && n < (1LL << 24)) ? 1 : 0;
        st.n_cnt = st.cnt_win ? (int)n : 0;
        st.ilv = ilv ? 1 : 0;
        st.density = (n > 1 && tmax > 0.0) ? (double)(n - 1) / tmax : 0.0;
        a.stats[c] = st;
    }
}

// ----------------------------------------------------------------------------
// search kernel
// ----------------------------------------------------------------------------

__device__ __forceinline__ void red_shared_u32(unsigned addr, unsigned v) {
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

// Histogram entry of slot s: four 32-bit words -- weight sums split at
// `lobits` (x, y; x = point count when weights are uniform) and flux sums
// split the same way (z, w).  Component c is stored in word c ^ rot(s),
// rot(s) = (s >> 3) & 3, so that for a fixed component consecutive slots
// cycle through all 32 banks (a plain 16-byte layout would use only 8).
__device__ __forceinline__ unsigned slot_rot(int s) { return ((unsigned)s >> 3) & 3u; }

__device__ __forceinline__ uint4 load_components(const uint4* H, int s) {
    uint4 e = H[s];
    const unsigned r = slot_rot(s);
    if (r & 1u) {
        const unsigned t0 = e.x, t1 = e.z;
        e.x = e.y; e.y = t0; e.z = e.w; e.w = t1;
    }
    if (r & 2u) {
        const unsigned t0 = e.x, t1 = e.y;
        e.x = e.z; e.y = e.w; e.z = t0; e.w = t1;
    }
    return e;
}

__device__ __forceinline__ uint4 add_words(uint4 u, uint4 v) {
    return make_uint4(u.x + v.x, u.y + v.y, u.z + v.z, u.w + v.w);
}

__device__ __forceinline__ void store_components(uint4* H, int s, uint4 e) {
    const unsigned r = slot_rot(s);  // the rotation is an involution per bit
    if (r & 1u) {
        const unsigned t0 = e.x, t1 = e.z;
        e.x = e.y; e.y = t0; e.z = e.w; e.w = t1;
    }
    if (r & 2u) {
        const unsigned t0 = e.x, t1 = e.y;
        e.x = e.z; e.y = e.w; e.z = t0; e.w = t1;
    }
    H[s] = e;
}

struct Team {
    int id;        // team index
    int nthreads;  // 32 * warps
    int nwarps;
    int tid;       // thread index within the team
    int warp0;     // first block-level warp of the team
};

__device__ __forceinline__ void team_sync(const Team& tm) {
    if (tm.nwarps == 1) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(tm.id + 1), "r"(tm.nthreads) : "memory");
    }
}

struct GroupSmem {
    double tP[kTileP];   // the tile's periods
    int tNB[kTileP];     // and their bin counts
    double2 PIP[kMaxG];  // (P, 1/P) of each period of the group
    int2 NBB[kMaxG];     // (bin count, histogram offset) of each period
    int fmode[kMaxG];    // fold mode of each period (kFold*)
    int redo[kMaxG];     // checked tight layout: the period's counts overflowed
    int n_redo;          // how many periods of the group are folded again
    int any_chunk;       // some period of the group uses kFoldChunk
    long long slot[kMaxG];
    int dbins[kMaxDur];
    double dur[kMaxDur];
    int L[kMaxWarps][kMaxDur];
    longlong2 scan[kMaxWarps];
    float num[kMaxWarps];
    float den[kMaxWarps];
    int key[kMaxWarps];
    long long tile;
    long long pb, pe, pn;
    int curve;
    int G;
    int total;
    int glob;        // 0 shared-memory group, 1 global histogram, 2 bin-range passes
    int safe_floor;  // fold_safe over the group: the fast fold form is exact
    // bin-range passes (one period whose bins exceed shared memory)
    uint4 pad_save[16];  // raw entries of bins 1..oversample (the V42 padding source)
    longlong2 carry;     // exact sums of every bin below the next pass
    longlong2 mp_e0, mp_e1;  // prefix entries of the best window so far
    float mp_num, mp_den;
    int mp_key;
};
constexpr int kMpPadMax = 16;  // oversample limit of the bin-range passes

// The fast fold form is exact when |d*IP| < 2^50 for every point (floor by
// magic additions) and, with astropy bins, the phase ph = fma(-P, floor(d*IP), d)
// -- negative by at most P*|d*IP|*2^-52 where d*IP rounded up past an
// integer -- stays above -bin_dur, so that int(ph*inv_bin_dur) >= 0 and the
// guard slot only ever holds points of slot 1: |d*IP| * max(1, P*inv_bin_dur)
// < 2^40 bounds that error by 2^-12 bins.  dtmax_ip = max |d| / min P,
// p_ibd = max P * inv_bin_dur.
template <int GEOM>
__device__ __forceinline__ bool fold_safe(double dtmax_ip, double p_ibd) {
    if (!(dtmax_ip < 1.0e15)) return false;
    return GEOM != ATB_GEOM_BINNED || dtmax_ip * fmax(1.0, p_ibd) < 1099511627776.0;  // 2^40
}

// Histogram slots of one thread's kR points for one period.
//   astropy-binned (vbls_v42_parity.cu:65-70): ph = fma(-P, floor(d*IP), d),
//     slot = min(int(ph*inv_bin_dur) + 1, n_bins).  int(x) of x in (-1, 0) is 0
//     (slot 1); the magic addition gives 0 there.  GUARD: that 0 is kept --
//     slot 0 is a guard entry that finalize_period adds into slot 1 -- and one
//     unsigned minimum bounds every other value, non-finite inputs (flagged
//     by the staging) included, by n_bins.  Without GUARD, slot 0 becomes 1.
//   fixed bins (bls.cu:52-62): ph = d*IP - floor(d*IP) in [0, 1), b = int(ph*n_bins)
//     in [0, n_bins]; slot = b + 1, where b = n_bins (a product rounded up to
//     n_bins) is the trash slot n_bins + 1 that no window reads.  The unsigned
//     minimum keeps non-finite inputs inside the period's entries.
// `safe` (see fold_safe) selects the fast form: floor by exact
// magic-constant additions, the guard slot, and, when the points are
// time-ordered and the first and last share the cycle index k = floor(d*IP),
// one k for all of them (rounded multiplication and floor are monotone).
// Without `safe`, every point takes floor() and the clamp to [1, n_bins].
template <int GEOM, bool GUARD>
__device__ __forceinline__ void fold_slots(const double (&d)[kR], bool sorted, bool safe, double P,
                                           double IP, double ibd, int NB, unsigned (&e)[kR]) {
    const double nbd = (double)NB;
    if (!safe) {
#pragma unroll
        for (int j = 0; j < kR; ++j) {
            const double m = d[j] * IP;
            const double k = floor(m);
            if (GEOM == ATB_GEOM_BINNED) {
                const int s1 = trunc1_magic(fma(-P, k, d[j]) * ibd);
                e[j] = (unsigned)min(max(s1, 1), NB);
            } else {
                e[j] = min((unsigned)trunc1_magic((m - k) * nbd), (unsigned)NB + 1u);
            }
        }
        return;
    }
    // sorted: m0 <= m7, so floor(m7) == k0 exactly when m7 < k0 + 1
    const double m0 = d[0] * IP, m7 = d[kR - 1] * IP;
    const double k0 = floor_magic(m0);
    if (sorted && m7 < k0 + 1.0) {
#pragma unroll
        for (int j = 0; j < kR; ++j) {
            if (GEOM == ATB_GEOM_BINNED) {
                const int s1 = trunc1_magic(fma(-P, k0, d[j]) * ibd);
                e[j] = GUARD ? min((unsigned)s1, (unsigned)NB) : (unsigned)min(max(s1, 1), NB);
            } else {
                const double m = (j == 0) ? m0 : (j == kR - 1 ? m7 : d[j] * IP);
                e[j] = min((unsigned)trunc1_magic((m - k0) * nbd), (unsigned)NB + 1u);
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < kR; ++j) {
            const double m = d[j] * IP;
            const double k = floor_magic(m);
            if (GEOM == ATB_GEOM_BINNED) {
                const int s1 = trunc1_magic(fma(-P, k, d[j]) * ibd);
                e[j] = GUARD ? min((unsigned)s1, (unsigned)NB) : (unsigned)min(max(s1, 1), NB);
            } else {
                e[j] = min((unsigned)trunc1_magic((m - k) * nbd), (unsigned)NB + 1u);
            }
        }
    }
}

// Add one point's words to histogram entry e (component c of the entry lives
// at word c ^ rot(e)); `base0` is the shared-memory address of entry 0 (H0
// the pointer to it for global histograms).  MODE selects the layout
// (kPack*); words a..d are the point's components x, y, z, w (unused ones are
// ignored).
template <bool GLOB, int MODE>
__device__ __forceinline__ void hist_add_point(unsigned base0, uint4* H0, unsigned e, unsigned a,
                                               unsigned b, unsigned c, unsigned d) {
    if (GLOB) {
        const unsigned r = (e >> 3) & 3u;
        unsigned* w = reinterpret_cast<unsigned*>(H0 + e);
        atomicAdd(w + (0u ^ r), a);
        if (MODE == kPackSplit) atomicAdd(w + (1u ^ r), b);
        atomicAdd(w + (2u ^ r), c);
        if (MODE != kPackTight) atomicAdd(w + (3u ^ r), d);
    } else {
        // base0 + 16 e has four low zero bits; rot(e) << 2 = (e >> 1) & 12
        const unsigned ad = (base0 + 16u * e) | ((e >> 1) & 12u);
        red_shared_u32(ad, a);
        if (MODE == kPackSplit) red_shared_u32(ad ^ 4u, b);
        red_shared_u32(ad ^ 8u, c);
        if (MODE != kPackTight) red_shared_u32(ad ^ 12u, d);
    }
}

// Fold modes, chosen per period from the expected number of time-ordered
// points that share a bin (bin width x the curve's mean point density):
//   kFoldPoint  one reduction per histogram word and point
//   kFoldChunk  a lane whose kR points provably share one slot (fold_ends)
//               adds their summed words once; other lanes as kFoldPoint
// The histogram words are integers added modulo 2^32, so both modes give the
// same sums, bit for bit; they differ only in how many reductions reach shared
// memory.  With few points per bin the per-point form is cheapest (the check
// costs issue slots and rarely saves a reduction); with several, neighbouring
// lanes add to the same address, and same-address reductions serialise.
// (Merging equal slots across the lanes of a warp as well, with a segmented
// shuffle scan, measured slower on every workload: the shuffles cost more of
// the shared-memory pipe than the reductions they save.)
constexpr int kFoldPoint = 0;
constexpr int kFoldChunk = 1;

// Slot of a lane's first point and whether all kR points share it, in the fast
// fold form of fold_slots (the caller checked `safe`): the points are
// time-ordered and lie in one cycle (the same k = floor(d*IP)), where the
// slot is a non-decreasing function of d (every rounded operation is
// monotone), so equal first and last slots mean every slot is equal.  The
// arithmetic of both slots is fold_slots' own.
template <int GEOM, bool GUARD>
__device__ __forceinline__ void fold_ends(const double (&d)[kR], bool sorted, double P, double IP,
                                          double ibd, int NB, unsigned& e0, bool& uni) {
    const double m0 = d[0] * IP, m7 = d[kR - 1] * IP;
    const double k0 = floor_magic(m0);
    unsigned a, b;
    if (GEOM == ATB_GEOM_BINNED) {
        const int s0 = trunc1_magic(fma(-P, k0, d[0]) * ibd);
        const int s7 = trunc1_magic(fma(-P, k0, d[kR - 1]) * ibd);
        a = GUARD ? min((unsigned)s0, (unsigned)NB) : (unsigned)min(max(s0, 1), NB);
        b = GUARD ? min((unsigned)s7, (unsigned)NB) : (unsigned)min(max(s7, 1), NB);
    } else {
        const double nbd = (double)NB;
        a = min((unsigned)trunc1_magic((m0 - k0) * nbd), (unsigned)NB + 1u);
        b = min((unsigned)trunc1_magic((m7 - k0) * nbd), (unsigned)NB + 1u);
    }
    e0 = a;
    uni = sorted && m7 < k0 + 1.0 && a == b;
}

// Fold every staged point of the curve into the group's histograms, each
// period in its fold mode (kFold*; bin-range passes and global histograms
// always fold point by point).
// WIN: bin-range pass -- only slots lo .. lo+W-1 are kept, at entries
// 0 .. W-1 of H (one period at offset 0).
// G: the number of the group's periods to fold (its first G).  CHUNK: some
// period of the group uses kFoldChunk (groups without one run the plain loop).
template <int GEOM, bool GLOB, int MODE, bool WIN = false, bool CHUNK = false>
__device__ void fold_group(const SearchArgs& a, const GroupSmem& gs, uint4* H, long long so,
                           long long n_pad, const CurveStat& st, int G, int lo = 0,
                           unsigned W = 0) {
    const bool safe = gs.safe_floor != 0;
    // split position of the layout's words (count layout for kPackCountT)
    const int L = MODE == kPackCountT ? curve_lobits(st.n_cnt) : st.lobits;
    const unsigned lomask = (1u << L) - 1u;
    const int nt = (int)blockDim.x;
    for (long long base = 0; base < n_pad; base += (long long)nt * kR) {
        const long long i0 = base + (long long)threadIdx.x * kR;
        if (i0 >= n_pad) continue;
        double d[kR];
        int qw[kR], qy[kR];
        const double2* dp = reinterpret_cast<const double2*>(a.sdt + so + i0);
#pragma unroll
        for (int q = 0; q < kR / 2; ++q) {
            const double2 v = __ldg(dp + q);
            d[2 * q] = v.x;
            d[2 * q + 1] = v.y;
        }
        const int4* wp = reinterpret_cast<const int4*>(a.sqw + so + i0);
        const int4* yp = reinterpret_cast<const int4*>(a.sqy + so + i0);
#pragma unroll
        for (int q = 0; q < kR / 4; ++q) {
            const int4 vw = __ldg(wp + q);
            const int4 vy = __ldg(yp + q);
            qw[4 * q] = vw.x; qw[4 * q + 1] = vw.y; qw[4 * q + 2] = vw.z; qw[4 * q + 3] = vw.w;
            qy[4 * q] = vy.x; qy[4 * q + 1] = vy.y; qy[4 * q + 2] = vy.z; qy[4 * q + 3] = vy.w;
        }
        bool sorted = true;
#pragma unroll
        for (int j = 0; j + 1 < kR; ++j) sorted = sorted && (d[j] <= d[j + 1]);
        // each point's histogram words (padding points have q_w = q_y = 0);
        // the stage kernel has already packed the tight words and the count
        unsigned wa[kR], wb[kR], wc[kR], wd[kR];
#pragma unroll
        for (int j = 0; j < kR; ++j) {
            if (MODE == kPackTight) {
                wa[j] = (unsigned)qw[j];
                wb[j] = 0u;
                wc[j] = (unsigned)qy[j];
                wd[j] = 0u;
            } else if (MODE == kPackCountT) {
                // staged tight words x = count << csh | (q mod 2^lob), z = q >> lob
                const unsigned x = (unsigned)qw[j];
                const int q = qy[j] * (1 << st.stage_lob) +
                              (int)(x & ((1u << st.stage_lob) - 1u));
                wa[j] = x >> st.stage_csh;
                wb[j] = 0u;
                wc[j] = (unsigned)q & lomask;
                wd[j] = (unsigned)(q >> L);
            } else {
                wa[j] = MODE == kPackCount ? (unsigned)qw[j] : ((unsigned)qw[j] & lomask);
                wb[j] = MODE == kPackCount ? 0u : (unsigned)(qw[j] >> L);
                wc[j] = (unsigned)qy[j] & lomask;
                wd[j] = (unsigned)(qy[j] >> L);
            }
        }
        for (int g = 0; g < G; ++g) {
            const double2 pip = gs.PIP[g];
            const int2 nbb = gs.NBB[g];
            uint4* H0 = H + nbb.y;
            const unsigned base0 = GLOB ? 0u : (unsigned)__cvta_generic_to_shared(H0);
            if (CHUNK && !GLOB && !WIN) {
                const int fm = gs.fmode[g];  // the same for every lane
                if (fm != kFoldPoint) {
                    unsigned e0;
                    bool uni;
                    fold_ends<GEOM, GEOM == ATB_GEOM_BINNED>(d, sorted, pip.x, pip.y,
                                                              st.inv_bin_dur, nbb.x, e0, uni);
                    unsigned sa = 0u, sb = 0u, sc = 0u, sd = 0u;
#pragma unroll
                    for (int j = 0; j < kR; ++j) {
                        sa += wa[j];
                        sb += wb[j];
                        sc += wc[j];
                        sd += wd[j];
                    }
                    if (uni) hist_add_point<false, MODE>(base0, H0, e0, sa, sb, sc, sd);
                    if (uni) continue;
                }
            }
            unsigned e[kR];
            fold_slots<GEOM, GEOM == ATB_GEOM_BINNED && !WIN>(d, sorted, safe, pip.x, pip.y,
                                                             st.inv_bin_dur, nbb.x, e);
#pragma unroll
            for (int j = 0; j < kR; ++j) {
                if (WIN) {
                    const unsigned ee = e[j] - (unsigned)lo;  // entry of the pass
                    if (ee < W) hist_add_point<GLOB, MODE>(base0, H0, ee, wa[j], wb[j], wc[j], wd[j]);
                } else {
                    hist_add_point<GLOB, MODE>(base0, H0, e[j], wa[j], wb[j], wc[j], wd[j]);
                }
            }
        }
    }
}

// FP64 statistics of the winning window from exact scaled sums: real units
// are W = dw * 2^-s_w, S = dy * 2^-s_y (s_w, s_y net of the prefix scaling)
__device__ void window_stats(double dw, double dy, double wtot, double ytot, int s_w, int s_y,
                             int objective, double* power, double* depth, double* derr) {
    const double w_in = ldexp(dw, -s_w);
    const double w_out = ldexp(wtot - dw, -s_w);
    const double s_in = ldexp(dy, -s_y);
    const double s_out = ldexp(ytot - dy, -s_y);
    const double y_in = s_in / w_in;
    const double y_out = s_out / w_out;
    const double dep = y_out - y_in;
    const double de = sqrt(1.0 / w_in + 1.0 / w_out);
    double pw;
    if (objective == ATB_OBJ_FAST) {
        pw = sqrt(dep * dep * (w_in * w_out));
    } else if (objective == ATB_OBJ_LIKELIHOOD) {
        pw = 0.5 * dep * dep * (w_in * w_out) / (w_in + w_out);
    } else {
        pw = dep / de;
    }
    *power = pw > 0.0 ? pw : 0.0;
    *depth = dep;
    *derr = de;
}

// Exact sums (W, Y) of raw histogram entry i in layout MODE: the words the
// layout uses are read directly (component c of entry i is word c ^ rot(i),
// at byte offset 4c ^ ((i >> 1) & 12) in the entry).
// `lob` is the split position of the count and split layouts' words.
template <int MODE>
__device__ __forceinline__ void entry_sums_m(const longlong2* E, int i, const CurveStat& st,
                                             int lob, long long& w, long long& y) {
    const unsigned* ent = reinterpret_cast<const unsigned*>(E + i);
    const unsigned r = slot_rot(i);
    const unsigned x = ent[0u ^ r];
    if (MODE == kPackTight) {
        const unsigned z = ent[2u ^ r];
        w = (long long)(x >> st.cshift);
        y = (long long)(int)z * (1LL << st.lobits) + (long long)(x & ((1u << st.cshift) - 1u));
    } else {
        const unsigned z = ent[2u ^ r], v = ent[3u ^ r];
        w = MODE == kPackCount ? (long long)x
                               : (long long)ent[1u ^ r] * (1LL << lob) + (long long)x;
        y = (long long)(int)v * (1LL << lob) + (long long)z;
    }
    if (MODE != kPackSplit && !st.cnt_win) w *= (long long)st.qw0;
}

// Pass 1 of the scan for layout MODE: decode entries [b, e) once, write
// their exact int64 sums back in place, return the segment's totals.
template <int MODE>
__device__ __forceinline__ void scan_decode(longlong2* E, int b, int e, const CurveStat& st,
                                            int lob, long long& sw, long long& sy) {
    sw = 0;
    sy = 0;
    for (int i = b; i < e; ++i) {
        long long w, y;
        entry_sums_m<MODE>(E, i, st, lob, w, y);
        E[i] = make_longlong2(w, y);
        sw += w;
        sy += y;
    }
}

// Inclusive scan of the raw histogram entries E[0..M) in place.  Pass 1
// decodes each entry's split 32-bit words once into exact int64 sums (W, Y)
// and writes them back; pass 2 adds the running sums and writes exact values:
// the flux sum as FP64 scaled by 2^-ey, and the weight sum as FP64 scaled by
// 2^-ew or, for counting curves (cnt_win), the point count as FP32 in the low
// word (|sum| < 2^53 and counts < 2^24, so every conversion is exact).
// Threads own contiguous segments of odd length, so the 16-byte entries a
// warp touches in one step fall in distinct bank groups.
// cw0, cy0: exact sums added to every prefix (the bins below E[0]); the
// thread holding entry carry_idx stores that entry's exact prefix in *carry.
// cview: a checked tight curve folded in the count layout (kPackCountT).
__device__ void team_scan(const Team& tm, GroupSmem& gs, longlong2* E, int M, const CurveStat& st,
                          bool cview, long long cw0 = 0, long long cy0 = 0, int carry_idx = -1,
                          longlong2* carry = nullptr) {
    int seg = (M + tm.nthreads - 1) / tm.nthreads;
    seg |= 1;
    const int b = min(M, tm.tid * seg);
    const int e = min(M, b + seg);
    long long sw, sy;
    if (cview)
        scan_decode<kPackCount>(E, b, e, st, curve_lobits(st.n_cnt), sw, sy);
    else if (st.packmode == kPackTight)
        scan_decode<kPackTight>(E, b, e, st, st.lobits, sw, sy);
    else if (st.packmode == kPackCount)
        scan_decode<kPackCount>(E, b, e, st, st.lobits, sw, sy);
    else
        scan_decode<kPackSplit>(E, b, e, st, st.lobits, sw, sy);
    const int lane = threadIdx.x & 31;
    long long iw = sw, iy = sy;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const long long tw = __shfl_up_sync(0xffffffffu, iw, off);
        const long long ty = __shfl_up_sync(0xffffffffu, iy, off);
        if (lane >= off) {
            iw += tw;
            iy += ty;
        }
    }
    if (tm.nwarps > 1) {
        const int wl = (threadIdx.x >> 5) - tm.warp0;
        if (lane == 31) gs.scan[tm.warp0 + wl] = make_longlong2(iw, iy);
        team_sync(tm);
        long long ow = 0, oy = 0;
        for (int k = 0; k < wl; ++k) {
            const longlong2 v = gs.scan[tm.warp0 + k];
            ow += v.x;
            oy += v.y;
        }
        iw += ow;
        iy += oy;
    }
    long long xw = iw - sw + cw0, xy = iy - sy + cy0;
    const double sy2 = ldexp(1.0, -st.ey);
    if (carry_idx >= b && carry_idx < e) {
        long long cw = xw, cy = xy;
        for (int i = b; i <= carry_idx; ++i) {
            cw += E[i].x;
            cy += E[i].y;
        }
        *carry = make_longlong2(cw, cy);
    }
    if (st.cnt_win) {
        for (int i = b; i < e; ++i) {
            const longlong2 v = E[i];
            xw += v.x;
            xy += v.y;
            E[i] = make_longlong2((long long)__float_as_uint((float)(int)xw),
                                  __double_as_longlong((double)xy * sy2));
        }
    } else {
        const double sw2 = ldexp(1.0, -st.ew);
        for (int i = b; i < e; ++i) {
            const longlong2 v = E[i];
            xw += v.x;
            xy += v.y;
            E[i] = make_longlong2(__double_as_longlong((double)xw * sw2),
                                  __double_as_longlong((double)xy * sy2));
        }
    }
    team_sync(tm);
}

__device__ Cand team_best(const Team& tm, GroupSmem& gs, Cand c) {
    c = warp_best(c);
    if (tm.nwarps > 1) {
        const int lane = threadIdx.x & 31;
        const int wg = threadIdx.x >> 5;
        if (lane == 0) {
            gs.num[wg] = c.num;
            gs.den[wg] = c.den;
            gs.key[wg] = c.key;
        }
        team_sync(tm);
        if (tm.tid == 0) {
            for (int k = 1; k < tm.nwarps; ++k) {
                const int j = tm.warp0 + k;
                if (cand_better(gs.num[j], gs.den[j], gs.key[j], c.num, c.den, c.key)) {
                    c.num = gs.num[j];
                    c.den = gs.den[j];
                    c.key = gs.key[j];
                }
            }
        }
        team_sync(tm);
    }
    return c;
}

struct WinConsts {
    double wtot, ytot;  // exact totals, scaled like the prefix sums
    float c1;           // ytot / wtot, or ytot / N for counting curves
    float fN;           // counting curves: N, the number of points in the histogram
    double thr;         // 1e-15 in scaled weight units
    double qw0s;        // counting curves: the scaled weight of one point
};

// One (start, duration) window: returns false when the window is skipped,
// else FP32 num/den of a score proportional to the objective within the
// period:
//   sigma = (S/W) W_in - S_in,  num = sigma^2,  den = W_in W_out
//   (num/den = depth^2 W_in W_out / W^2, the SNR^2 up to a per-period factor)
//   BINNED (vbls_v42_parity.cu:103-116): skip empty in/out windows, dip-only
//   FIXED  (bls.cu:128): skip unless 0 < W_in < W
// Weighted curves pass exact scaled FP64 weight sums (dw); counting curves
// pass the exact FP32 point count of the window (fdw) and use N and S/N in
// place of W and S/W (the same score up to the constant factor qw0s^2).
// The dip-only rule of the astropy-binned geometry is carried by the sign of
// num = sigma*|sigma|: a window with sigma < 0 has num < 0 and never passes
// the filter num >= lim*den (lim >= 0, den > 0), and for sigma >= 0 num is
// sigma^2.  den > 0 is exactly "W_in > 0 and W_out > 0" (both are
// non-negative).
template <int GEOM, bool UNIT>
__device__ __forceinline__ bool window_eval(double dw, double dy, const WinConsts& kc, float& num,
                                            float& den) {
    const double wo = kc.wtot - dw;
    const float fdw = __double2float_rn(dw);
    const float fwo = __double2float_rn(wo);
    const float sig = __fmaf_rn(kc.c1, fdw, -__double2float_rn(dy));
    num = __fmul_rn(sig, GEOM == ATB_GEOM_BINNED ? fabsf(sig) : sig);
    den = __fmul_rn(fdw, fwo);
    if (UNIT) return den > 0.0f;  // exact: dw, wo are scaled integers and thr < 1 unit
    return !(dw < kc.thr || wo < kc.thr);
}

template <int GEOM, bool UNIT>
__device__ __forceinline__ bool window_eval_cnt(float fdw, double dy, const WinConsts& kc,
                                                float& num, float& den) {
    const float fwo = __fsub_rn(kc.fN, fdw);  // exact: integers below 2^24
    const float sig = __fmaf_rn(kc.c1, fdw, -__double2float_rn(dy));
    num = __fmul_rn(sig, GEOM == ATB_GEOM_BINNED ? fabsf(sig) : sig);
    den = __fmul_rn(fdw, fwo);
    if (UNIT) return den > 0.0f;
    return !((double)fdw * kc.qw0s < kc.thr || (double)fwo * kc.qw0s < kc.thr);
}

// Running best with a division-free pre-filter: `lim` (>= 0) is a lower bound
// of a ratio some window of the period reaches (rounded down by 2^-20), so
// num < lim*den can never win the exact comparison and is skipped.  share()
// gives every lane of the warp the largest lim of the warp: a window below
// another lane's best cannot be the period's best, and exact ties still pass
// the filter, so the lowest-key rule is unaffected.
struct Best {
    Cand c;
    float lim;
    __device__ __forceinline__ void init() {
        c = Cand{-1.0f, 1.0f, 0x7fffffff};
        lim = 0.0f;
    }
    __device__ __forceinline__ void consider(float num, float den, int key) {
        if (num >= __fmul_rn(lim, den) && cand_better(num, den, key, c.num, c.den, c.key)) {
            c.num = num;
            c.den = den;
            c.key = key;
            lim = fmaxf(lim, __fmul_rn(__fdiv_rn(num, den), 0.99999904632568359375f));  // 1 - 2^-20
        }
    }
    // non-negative floats order like their bit patterns; every lane must call it
    __device__ __forceinline__ void share() {
        lim = __int_as_float(__reduce_max_sync(0xffffffffu, __float_as_int(lim)));
    }
};

__device__ __forceinline__ float cnt_of(long long x) { return __int_as_float((int)x); }

// The windows (s, len[k]) of KC durations at one start s.  CHECK = false is
// the interior, where every window ends at or before bin NB: no clamping, no
// wrap and no range test.  The KC end points are loaded before any is used.
// Start range of one window search: starts s in [s_lo, s_hi) of a prefix
// array whose entry i is held at E[i - off]; end points are clamped to idx_max
// where they are out of range (their windows are skipped).  The whole period
// in one array is {0, 0, NB, NB}.
struct WinRange {
    int off, s_lo, s_hi, idx_max;
};

template <int GEOM, bool UNIT, bool CNT, int KC, bool CHECK>
__device__ __forceinline__ void windows_at(const longlong2* E, int NB, int s, const int (&len)[KC],
                                           const WinConsts& kc, const WinRange& rg,
                                           float (&num)[KC], float (&den)[KC], bool (&ok)[KC]) {
    const longlong2 e0 = E[s - rg.off];
    longlong2 e1[KC];
#pragma unroll
    for (int k = 0; k < KC; ++k) {
        int idx = s + len[k];
        if (CHECK) {
            if (GEOM == ATB_GEOM_FIXED && idx > NB) idx -= NB;
            idx = min(idx, rg.idx_max);
        }
        e1[k] = E[idx - rg.off];
    }
#pragma unroll
    for (int k = 0; k < KC; ++k) {
        bool in_range = true;
        bool wrap = false;
        if (CHECK) {
            if (GEOM == ATB_GEOM_BINNED) {
                in_range = s + len[k] <= NB;
            } else {
                in_range = len[k] < NB;
                wrap = s + len[k] > NB;
            }
        }
        bool okk;
        if (CNT) {
            const float c0 = cnt_of(e0.x);
            float fdw;
            double dy;
            if (wrap) {
                fdw = __fadd_rn(__fsub_rn(kc.fN, c0), cnt_of(e1[k].x));
                dy = (kc.ytot - ll_as_d(e0.y)) + ll_as_d(e1[k].y);
            } else {
                fdw = __fsub_rn(cnt_of(e1[k].x), c0);
                dy = ll_as_d(e1[k].y) - ll_as_d(e0.y);
            }
            okk = window_eval_cnt<GEOM, UNIT>(fdw, dy, kc, num[k], den[k]);
        } else {
            double dw, dy;
            if (wrap) {
                dw = (kc.wtot - ll_as_d(e0.x)) + ll_as_d(e1[k].x);
                dy = (kc.ytot - ll_as_d(e0.y)) + ll_as_d(e1[k].y);
            } else {
                dw = ll_as_d(e1[k].x) - ll_as_d(e0.x);
                dy = ll_as_d(e1[k].y) - ll_as_d(e0.y);
            }
            okk = window_eval<GEOM, UNIT>(dw, dy, kc, num[k], den[k]);
        }
        ok[k] = in_range && okk;
    }
}

// The division-free filter for the KC windows of one step of the warp; the
// exact comparison runs only in the (rare) steps where some lane has a
// window passing it.  Every lane of the warp must call it.
template <int KC>
__device__ __forceinline__ void window_filter(const float (&num)[KC], const float (&den)[KC],
                                              const bool (&ok)[KC], int key0, Best& best) {
    bool pass[KC];
    bool any = false;
#pragma unroll
    for (int k = 0; k < KC; ++k) {
        pass[k] = ok[k] && num[k] >= __fmul_rn(best.lim, den[k]);
        any = any || pass[k];
    }
    if (__any_sync(0xffffffffu, any)) {
#pragma unroll
        for (int k = 0; k < KC; ++k)
            if (pass[k]) best.consider(num[k], den[k], key0 + k);
        best.share();
    }
}

template <int GEOM, bool UNIT, bool CNT, int KC>
__device__ __forceinline__ void window_chunk(const longlong2* E, int NB, int nd, int k0,
                                             const int* lens_smem, int tid, int nthreads,
                                             const WinConsts& kc, const WinRange& rg,
                                             Best& best) {
    int len[KC];
    int lmax = 0;
#pragma unroll
    for (int k = 0; k < KC; ++k) {
        len[k] = lens_smem[k0 + k];
        lmax = max(lmax, len[k]);
    }
    // interior starts: s + lmax <= NB (and, with fixed bins, every window
    // shorter than the period)
    const int s_end =
        min(rg.s_hi, (GEOM == ATB_GEOM_FIXED && lmax >= NB) ? 0 : NB - lmax + 1);
    // warp-uniform trip count (lanes past the range skip the body), so that
    // the warp can share its filter bound after every step
    const int lane = tid & 31;
    int s0 = rg.s_lo + tid - lane;
    // interior steps (every lane's start is interior): no divergence
    for (; s0 + 31 < s_end; s0 += nthreads) {
        const int s = s0 + lane;
        float num[KC], den[KC];
        bool ok[KC];
        windows_at<GEOM, UNIT, CNT, KC, false>(E, NB, s, len, kc, rg, num, den, ok);
        window_filter<KC>(num, den, ok, s * nd + k0, best);
    }
    // the remaining steps
    for (; s0 < rg.s_hi; s0 += nthreads) {
        const int s = s0 + lane;
        float num[KC], den[KC];
        bool ok[KC];
        if (s < s_end) {
            windows_at<GEOM, UNIT, CNT, KC, false>(E, NB, s, len, kc, rg, num, den, ok);
        } else if (s < rg.s_hi) {
            windows_at<GEOM, UNIT, CNT, KC, true>(E, NB, s, len, kc, rg, num, den, ok);
        } else {
#pragma unroll
            for (int k = 0; k < KC; ++k) {
                num[k] = 0.0f;
                den[k] = 1.0f;
                ok[k] = false;
            }
        }
        window_filter<KC>(num, den, ok, s * nd + k0, best);
    }
}

// All windows of one period over starts tid, tid+nthreads, ...  Durations are
// taken four at a time (then two, then one): the end points of a chunk are
// loaded together (instruction-level parallelism with few live registers).
// `lim0` (>= 0) starts the filter bound: a ratio some window is known to reach.
template <int GEOM, bool UNIT, bool CNT>
__device__ Cand window_search(const longlong2* E, int NB, int nd, const int* lens_smem, int tid,
                              int nthreads, const WinConsts& kc, const WinRange& rg,
                              float lim0 = 0.0f) {
    Best best;
    best.init();
    best.lim = lim0;
    int k0 = 0;
    for (; k0 + 4 <= nd; k0 += 4)
        window_chunk<GEOM, UNIT, CNT, 4>(E, NB, nd, k0, lens_smem, tid, nthreads, kc, rg, best);
    if (nd - k0 >= 2) {
        window_chunk<GEOM, UNIT, CNT, 2>(E, NB, nd, k0, lens_smem, tid, nthreads, kc, rg, best);
        k0 += 2;
    }
    if (nd - k0 >= 1)
        window_chunk<GEOM, UNIT, CNT, 1>(E, NB, nd, k0, lens_smem, tid, nthreads, kc, rg, best);
    return best.c;
}

template <int GEOM>
__device__ void finalize_period(const SearchArgs& a, GroupSmem& gs, const Team& tm, longlong2* H,
                                int g, const CurveStat& st, int nd, bool cview) {
    longlong2* E = H + gs.NBB[g].y;
    const int NB = gs.NBB[g].x;
    const double P = gs.PIP[g].x;
    const double IP = gs.PIP[g].y;

    if (st.tcheck && !cview) {
        // checked tight layout: the decoded counts of the raw entries (every
        // slot the fold can write) must add up to the curve's n points, else
        // a count field overflowed and the period is folded again
        const int n_ent = (GEOM == ATB_GEOM_BINNED) ? NB + 1 : NB + 2;
        unsigned cnt = 0u;
        for (int i = tm.tid; i < n_ent; i += tm.nthreads) {
            const unsigned* ent = reinterpret_cast<const unsigned*>(E + i);
            cnt += ent[slot_rot(i)] >> st.cshift;  // component 0 of entry i
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
        if (tm.nwarps > 1) {
            const int wg = threadIdx.x >> 5;
            if ((threadIdx.x & 31) == 0) gs.scan[wg].x = (long long)cnt;
            team_sync(tm);
            cnt = 0u;
            for (int k = 0; k < tm.nwarps; ++k) cnt += (unsigned)gs.scan[tm.warp0 + k].x;
            team_sync(tm);  // before the scan reuses gs.scan
        }
        if (cnt != (unsigned)st.n_cnt) {
            if (tm.tid == 0) gs.redo[g] = 1;
            return;  // every thread of the team returns: the same total
        }
    }

    if (GEOM == ATB_GEOM_BINNED) {
        // padding copy, vbls_v42_parity.cu:78-80: bins 1..os onto NB-os..NB-1
        // with sequential semantics; when the two ranges are disjoint
        // (NB > 2 os) the copies are independent and run in parallel
        // first the fold's guard slot 0 (points with int(ph*inv_bin_dur) = 0
        // from ph*inv_bin_dur in (-1, 0)) joins slot 1; the words are 32-bit
        // sums, so the entries add word by word
        const int os = a.oversample;
        uint4* R = reinterpret_cast<uint4*>(E);
        if (NB > 2 * os) {
            if (tm.tid < os) {
                uint4 v = load_components(R, 1 + tm.tid);
                if (tm.tid == 0) {
                    v = add_words(v, load_components(R, 0));
                    R[0] = make_uint4(0u, 0u, 0u, 0u);
                    store_components(R, 1, v);
                }
                store_components(R, NB - os + tm.tid, v);
            }
        } else if (tm.tid == 0) {
            store_components(R, 1, add_words(load_components(R, 1), load_components(R, 0)));
            R[0] = make_uint4(0u, 0u, 0u, 0u);
            for (int j = 1, ind = NB - os; j <= os; ++j, ++ind)
                store_components(R, ind, load_components(R, j));
        }
        team_sync(tm);
    } else {
        if (tm.tid < nd) {
            // truncation of dur/P * n_bins + 0.5, at least 1 (NaN: 1)
            const double Lf = fma(gs.dur[tm.tid] * IP, (double)NB, 0.5);
            gs.L[tm.id][tm.tid] = Lf >= (double)kLenCap ? kLenCap : (Lf >= 1.0 ? (int)Lf : 1);
        }
    }
    team_scan(tm, gs, E, NB + 1, st, cview);

    // scaled exact totals; counting curves: N points of weight qw0s each
    const bool cnt = st.cnt_win != 0;
    const double qw0s = ldexp((double)st.qw0, -st.ew);
    double wtot, ytot;
    float fN = 0.0f;
    if (GEOM == ATB_GEOM_BINNED) {
        wtot = ldexp((double)st.qw_tot, -st.ew);
        ytot = ldexp((double)st.qy_tot, -st.ey);
        fN = (float)st.n_cnt;
    } else {
        const longlong2 te = E[NB];
        if (cnt) {
            fN = cnt_of(te.x);
            wtot = (double)fN * qw0s;
        } else {
            wtot = ll_as_d(te.x);
        }
        ytot = ll_as_d(te.y);
    }
    // exact scaled weight sum of prefix entry i
    auto pw_at = [&](int i) { return cnt ? (double)cnt_of(E[i].x) * qw0s : ll_as_d(E[i].x); };
    Cand best{-1.0f, 1.0f, 0x7fffffff};
    if (wtot > 0.0) {
        WinConsts kc;
        kc.wtot = wtot;
        kc.ytot = ytot;
        kc.c1 = cnt ? (float)(ytot / (double)fN) : (float)(ytot / wtot);
        kc.fN = fN;
        kc.thr = ldexp(1e-15, st.s_w - st.ew);
        kc.qw0s = qw0s;
        const int* lens = (GEOM == ATB_GEOM_BINNED) ? gs.dbins : gs.L[tm.id];
        const bool unit = GEOM == ATB_GEOM_FIXED || st.thr_unit;
        const WinRange rg{0, 0, NB, NB};
        if (cnt)
            best = unit ? window_search<GEOM, true, true>(E, NB, nd, lens, tm.tid, tm.nthreads, kc, rg)
                        : window_search<GEOM, false, true>(E, NB, nd, lens, tm.tid, tm.nthreads, kc, rg);
        else
            best = unit ? window_search<GEOM, true, false>(E, NB, nd, lens, tm.tid, tm.nthreads, kc, rg)
                        : window_search<GEOM, false, false>(E, NB, nd, lens, tm.tid, tm.nthreads, kc, rg);
    }
    best = team_best(tm, gs, best);

    if (tm.tid == 0) {
        const long long slot = gs.slot[g];
        float o_pw = 0.0f, o_dep = 0.0f, o_de = 0.0f, o_dur = 0.0f;
        double o_t0 = 0.0;
        int o_win = -1;
        if (best.key != 0x7fffffff) {
            const int s = best.key / nd, k = best.key % nd;
            double dw, dy;
            if (GEOM == ATB_GEOM_BINNED) {
                const int dd = gs.dbins[k];
                dw = pw_at(s + dd) - pw_at(s);
                dy = ll_as_d(E[s + dd].y) - ll_as_d(E[s].y);
                const double durv = (double)dd * st.bin_dur;
                o_dur = (float)durv;
                o_t0 = fmod((double)s * st.bin_dur + 0.5 * durv + st.t_start, P);
            } else {
                const int L = gs.L[tm.id][k];
                if (s + L <= NB) {
                    dw = pw_at(s + L) - pw_at(s);
                    dy = ll_as_d(E[s + L].y) - ll_as_d(E[s].y);
                } else {
                    dw = (wtot - pw_at(s)) + pw_at(s + L - NB);
                    dy = (ytot - ll_as_d(E[s].y)) + ll_as_d(E[s + L - NB].y);
                }
                o_dur = (float)gs.dur[k];
                o_t0 = fma((double)s / (double)NB, 1.0 / IP, st.t_start);
            }
            double pw, dep, de;
            window_stats(dw, dy, wtot, ytot, st.s_w - st.ew, st.s_y - st.ey, a.objective, &pw, &dep,
                         &de);
            o_pw = (float)pw;
            o_dep = (float)dep;
            o_de = (float)de;
            o_win = best.key;
        }
        if (a.best_key && o_win >= 0) {
            // (power bits << 32 | ~period index): non-negative floats order
            // like their bits, and among equal powers the lowest index wins
            const unsigned long long key =
                ((unsigned long long)__float_as_uint(o_pw) << 32) |
                (unsigned long long)(0xffffffffu - (unsigned)(slot - a.out_beg[gs.curve]));
            atomicMax(a.best_key + gs.curve, key);
        }
        if (a.power) a.power[slot] = o_pw;
        if (a.depth) a.depth[slot] = o_dep;
        if (a.depth_err) a.depth_err[slot] = o_de;
        if (a.t0) a.t0[slot] = o_t0;
        if (a.duration) a.duration[slot] = o_dur;
        if (a.window) a.window[slot] = o_win;
    }
    team_sync(tm);  // per-team scratch (window lengths, scan totals) is reused by the next period
}

// One astropy-binned period whose NB+1 prefix entries exceed the shared
// histogram area, searched in bin-range passes through shared memory: pass r
// folds every point but keeps only slots [lo, lo+W) (lo = r*S, S = W - Lmax,
// Lmax the longest window), applies the V42 padding copy to the slots it
// holds, scans them on top of the exact sums of every slot below lo (carried
// from the previous pass), and searches the windows that start in [lo, lo+S)
// -- each ends inside the pass.  The prefix values, and therefore every
// window's score, are the ones the single-pass path computes; the best window
// over the passes is kept with the same exact comparison, together with its
// two prefix entries for the final FP64 statistics.  The whole CTA is one team.
__device__ void run_period_binned_passes(const SearchArgs& a, GroupSmem& gs, longlong2* H,
                                         const CurveStat& st, long long so, long long n_pad,
                                         int nd) {
    // a checked tight curve is folded here in the count layout (no check)
    const bool cview = st.tcheck != 0;
    const int NB = gs.NBB[0].x;
    const double P = gs.PIP[0].x;
    const int os = a.oversample;
    int Lmax = 0;
    for (int k = 0; k < nd; ++k) Lmax = max(Lmax, gs.dbins[k]);
    const int W = a.cap - 2;
    const int S = W - Lmax;  // >= 1: checked when the group was formed
    Team tm;
    tm.id = 0;
    tm.nwarps = (int)(blockDim.x >> 5);
    tm.nthreads = (int)blockDim.x;
    tm.warp0 = 0;
    tm.tid = threadIdx.x;
    const bool cnt = st.cnt_win != 0;
    const double qw0s = ldexp((double)st.qw0, -st.ew);
    const double wtot = ldexp((double)st.qw_tot, -st.ew);
    const double ytot = ldexp((double)st.qy_tot, -st.ey);
    const float fN = (float)st.n_cnt;
    WinConsts kc;
    kc.wtot = wtot;
    kc.ytot = ytot;
    kc.c1 = cnt ? (float)(ytot / (double)fN) : (float)(ytot / wtot);
    kc.fN = fN;
    kc.thr = ldexp(1e-15, st.s_w - st.ew);
    kc.qw0s = qw0s;
    const bool unit = st.thr_unit != 0;
    if (threadIdx.x == 0) {
        gs.mp_num = -1.0f;
        gs.mp_den = 1.0f;
        gs.mp_key = 0x7fffffff;
        gs.carry = make_longlong2(0, 0);
    }
    uint4* HU = reinterpret_cast<uint4*>(H);
    for (int lo = 0; lo < NB; lo += S) {
        for (int i = threadIdx.x; i < W; i += blockDim.x) H[i] = make_longlong2(0, 0);
        __syncthreads();
        if (cview)
            fold_group<ATB_GEOM_BINNED, false, kPackCountT, true>(a, gs, HU, so, n_pad, st, 1, lo, W);
        else if (st.packmode == kPackTight)
            fold_group<ATB_GEOM_BINNED, false, kPackTight, true>(a, gs, HU, so, n_pad, st, 1, lo, W);
        else if (st.packmode == kPackCount)
            fold_group<ATB_GEOM_BINNED, false, kPackCount, true>(a, gs, HU, so, n_pad, st, 1, lo, W);
        else
            fold_group<ATB_GEOM_BINNED, false, kPackSplit, true>(a, gs, HU, so, n_pad, st, 1, lo, W);
        __syncthreads();
        // padding copy, vbls_v42_parity.cu:78-80: bins 1..os (saved by the
        // first pass) replace bins NB-os..NB-1 wherever a pass holds them
        if (lo == 0 && threadIdx.x < os) gs.pad_save[threadIdx.x] = load_components(HU, 1 + threadIdx.x);
        __syncthreads();
        if (threadIdx.x < os) {
            const int j = NB - os + threadIdx.x - lo;
            if (j >= 0 && j < W) store_components(HU, j, gs.pad_save[threadIdx.x]);
        }
        __syncthreads();
        const int M = min(W, NB + 1 - lo);
        const longlong2 c0 = gs.carry;
        __syncthreads();
        team_scan(tm, gs, H, M, st, cview, c0.x, c0.y, S - 1 < M ? S - 1 : -1, &gs.carry);
        Cand best{-1.0f, 1.0f, 0x7fffffff};
        if (wtot > 0.0) {
            const WinRange rg{lo, lo, min(lo + S, NB), min(NB, lo + W - 1)};
            const float lim0 = gs.mp_key != 0x7fffffff
                                   ? __fmul_rn(__fdiv_rn(gs.mp_num, gs.mp_den), 0.99999904632568359375f)
                                   : 0.0f;
            if (cnt)
                best = unit ? window_search<ATB_GEOM_BINNED, true, true>(H, NB, nd, gs.dbins, tm.tid,
                                                                         tm.nthreads, kc, rg, lim0)
                            : window_search<ATB_GEOM_BINNED, false, true>(H, NB, nd, gs.dbins, tm.tid,
                                                                          tm.nthreads, kc, rg, lim0);
            else
                best = unit ? window_search<ATB_GEOM_BINNED, true, false>(H, NB, nd, gs.dbins, tm.tid,
                                                                          tm.nthreads, kc, rg, lim0)
                            : window_search<ATB_GEOM_BINNED, false, false>(H, NB, nd, gs.dbins, tm.tid,
                                                                           tm.nthreads, kc, rg, lim0);
        }
        best = team_best(tm, gs, best);
        if (threadIdx.x == 0 && best.key != 0x7fffffff &&
            cand_better(best.num, best.den, best.key, gs.mp_num, gs.mp_den, gs.mp_key)) {
            const int s = best.key / nd, k = best.key % nd;
            gs.mp_num = best.num;
            gs.mp_den = best.den;
            gs.mp_key = best.key;
            gs.mp_e0 = H[s - lo];
            gs.mp_e1 = H[s + gs.dbins[k] - lo];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const long long slot = gs.slot[0];
        float o_pw = 0.0f, o_dep = 0.0f, o_de = 0.0f, o_dur = 0.0f;
        double o_t0 = 0.0;
        int o_win = -1;
        if (gs.mp_key != 0x7fffffff) {
            const int s = gs.mp_key / nd, k = gs.mp_key % nd;
            const int dd = gs.dbins[k];
            auto pw_of = [&](const longlong2 e) {
                return cnt ? (double)cnt_of(e.x) * qw0s : ll_as_d(e.x);
            };
            const double dw = pw_of(gs.mp_e1) - pw_of(gs.mp_e0);
            const double dy = ll_as_d(gs.mp_e1.y) - ll_as_d(gs.mp_e0.y);
            const double durv = (double)dd * st.bin_dur;
            o_dur = (float)durv;
            o_t0 = fmod((double)s * st.bin_dur + 0.5 * durv + st.t_start, P);
            double pw, dep, de;
            window_stats(dw, dy, wtot, ytot, st.s_w - st.ew, st.s_y - st.ey, a.objective, &pw, &dep,
                         &de);
            o_pw = (float)pw;
            o_dep = (float)dep;
            o_de = (float)de;
            o_win = gs.mp_key;
        }
        if (a.best_key && o_win >= 0) {
            const unsigned long long key =
                ((unsigned long long)__float_as_uint(o_pw) << 32) |
                (unsigned long long)(0xffffffffu - (unsigned)(slot - a.out_beg[gs.curve]));
            atomicMax(a.best_key + gs.curve, key);
        }
        if (a.power) a.power[slot] = o_pw;
        if (a.depth) a.depth[slot] = o_dep;
        if (a.depth_err) a.depth_err[slot] = o_de;
        if (a.t0) a.t0[slot] = o_t0;
        if (a.duration) a.duration[slot] = o_dur;
        if (a.window) a.window[slot] = o_win;
    }
    __syncthreads();
}

// Teams of warps finalise the group's first G periods.
template <int GEOM>
__device__ void finalize_group(const SearchArgs& a, GroupSmem& gs, longlong2* H,
                               const CurveStat& st, int nd, int G, bool cview) {
    // teams of tw warps (a power of two; teams as wide as 1/G of the CTA
    // measured slower); multi-warp teams synchronise on named barriers 1..15,
    // so at most 15 of them may exist
    int tw = 1;
    const int nw = (int)(blockDim.x >> 5);
    while (tw * 2 * G <= nw) tw *= 2;
    while (tw > 1 && nw / tw > 15) tw *= 2;
    const int n_teams = nw / tw;
    const int warp = threadIdx.x >> 5;
    Team tm;
    tm.id = warp / tw;
    tm.nwarps = tw;
    tm.nthreads = tw * 32;
    tm.warp0 = tm.id * tw;
    tm.tid = threadIdx.x - tm.warp0 * 32;
    for (int g = tm.id; g < G; g += n_teams) finalize_period<GEOM>(a, gs, tm, H, g, st, nd, cview);
    __syncthreads();
}

// The group's fold in the curve's own layout (shared-memory histograms when
// CHUNK, GLOB otherwise: CHUNK is only used with shared memory).
template <int GEOM, bool CHUNK, bool GLOB = false>
__device__ __forceinline__ void fold_layout(const SearchArgs& a, const GroupSmem& gs, uint4* HU,
                                            long long so, long long n_pad, const CurveStat& st,
                                            int G) {
    if (st.packmode == kPackTight)
        fold_group<GEOM, GLOB, kPackTight, false, CHUNK>(a, gs, HU, so, n_pad, st, G);
    else if (st.packmode == kPackCount)
        fold_group<GEOM, GLOB, kPackCount, false, CHUNK>(a, gs, HU, so, n_pad, st, G);
    else
        fold_group<GEOM, GLOB, kPackSplit, false, CHUNK>(a, gs, HU, so, n_pad, st, G);
}

template <int GEOM, bool GLOB>
__device__ void run_group(const SearchArgs& a, GroupSmem& gs, longlong2* H, const CurveStat& st,
                          long long so, long long n_pad, int nd) {
    const int total = gs.total;
    for (int i = threadIdx.x; i < total; i += blockDim.x) H[i] = make_longlong2(0, 0);
    __syncthreads();
    uint4* HU = reinterpret_cast<uint4*>(H);
    // global histograms fold a checked tight curve in the count layout at once
    const bool cview = GLOB && st.tcheck;
    const int G = gs.G;
    if constexpr (GLOB) {
        if (cview)
            fold_group<GEOM, GLOB, kPackCountT>(a, gs, HU, so, n_pad, st, G);
        else
            fold_layout<GEOM, false, GLOB>(a, gs, HU, so, n_pad, st, G);
    } else {
        if (gs.any_chunk)
            fold_layout<GEOM, true>(a, gs, HU, so, n_pad, st, G);
        else
            fold_layout<GEOM, false>(a, gs, HU, so, n_pad, st, G);
    }
    __syncthreads();
    finalize_group<GEOM>(a, gs, H, st, nd, G, cview);
    if (!GLOB && st.tcheck) {
        // periods whose counts overflowed the tight words: fold them again in
        // the count layout (their entries only) and finalise them.  The
        // group's arrays are compacted to those periods (only the first r
        // are used from here on; the caller advances by G, which no thread
        // writes here).
        if (threadIdx.x == 0) {
            int r = 0;
            for (int k = 0; k < G; ++k) {
                if (!gs.redo[k]) continue;
                gs.PIP[r] = gs.PIP[k];
                gs.NBB[r] = gs.NBB[k];
                gs.slot[r] = gs.slot[k];
                gs.fmode[r] = gs.fmode[k];
                ++r;
            }
            gs.n_redo = r;
        }
        __syncthreads();
        const int r = gs.n_redo;
        if (r > 0) {
            for (int k = 0; k < r; ++k) {
                const int off = gs.NBB[k].y, cnt = gs.NBB[k].x + 2;
                for (int i = threadIdx.x; i < cnt; i += blockDim.x) H[off + i] = make_longlong2(0, 0);
            }
            __syncthreads();
            if (gs.any_chunk)
                fold_group<GEOM, false, kPackCountT, false, true>(a, gs, HU, so, n_pad, st, r);
            else
                fold_group<GEOM, false, kPackCountT>(a, gs, HU, so, n_pad, st, r);
            __syncthreads();
            finalize_group<GEOM>(a, gs, H, st, nd, r, true);
        }
    }
}

template <int GEOM, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) search_kernel(const SearchArgs a) {
    extern __shared__ __align__(16) longlong2 s_hist[];
    __shared__ GroupSmem gs;

    for (;;) {
        if (threadIdx.x == 0) {
            const long long tile = (long long)atomicAdd(a.tile_counter, 1ULL);
            gs.tile = tile;
            if (tile < a.n_tiles) {
                int lo = 0, hi = a.n_curves;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (a.tile_off[mid] <= tile) lo = mid; else hi = mid;
                }
                const int c = a.order[lo];
                gs.curve = c;
                gs.pb = (tile - a.tile_off[lo]) * a.tile_p;
                gs.pe = min(gs.pb + a.tile_p, a.per_cnt[c]);
            }
        }
        __syncthreads();
        if (gs.tile >= a.n_tiles) break;

        const int c = gs.curve;
        const CurveStat st = a.stats[c];
        const int nd = a.dur_cnt[c];
        const long long n = a.pt_off[c + 1] - a.pt_off[c];
        const long long n_pad = (n + kR - 1) / kR * kR;
        const long long so = a.stage_off[c];
        const long long pbeg = a.per_beg[c];
        const long long obeg = a.out_beg[c];
        if (threadIdx.x < nd) {
            gs.dbins[threadIdx.x] = a.dbins[c * kMaxDur + threadIdx.x];
            gs.dur[threadIdx.x] = a.durations[a.dur_beg[c] + threadIdx.x];
        }
        long long pn = gs.pb;
        const long long pe = gs.pe;
        // the tile's periods and bin counts, loaded in parallel
        for (int i = threadIdx.x; i < (int)(pe - pn); i += NT) {
            double P = a.periods[pbeg + pn + i];
            if (!(P > 0.0) || !(P < 1.0e300)) {
                atomicOr(a.status, 4);
                P = 1.0;
            }
            gs.tP[i] = P;
            gs.tNB[i] = (GEOM == ATB_GEOM_BINNED)
                            ? binned_nbins(P, st.inv_bin_dur, a.oversample, a.max_bins)
                            : a.n_bins_fixed;
        }
        __syncthreads();
        while (pn < pe) {
            if (threadIdx.x == 0) {
                int g = 0, base = 0;
                long long p = pn;
                double ipmax = 0.0, pmax = 0.0;
                while (p < pe && g < kMaxG) {
                    const int li = (int)(p - gs.pb);
                    const double P = gs.tP[li];
                    const int NB = gs.tNB[li];
                    const int need = NB + 2;
                    if (g > 0 && base + need > a.cap) break;
                    const double IP = 1.0 / P;
                    ipmax = max(ipmax, IP);
                    pmax = max(pmax, P);
                    gs.PIP[g] = make_double2(P, IP);
                    gs.NBB[g] = make_int2(NB, base);
                    gs.slot[g] = obeg + p;
                    base += need;
                    ++g;
                    ++p;
                    if (base > a.cap) break;  // a lone oversized period: global histogram
                }
                gs.G = g;
                gs.total = base;
                gs.glob = base > a.cap ? 1 : 0;
                if (gs.glob && GEOM == ATB_GEOM_BINNED && a.oversample <= kMpPadMax) {
                    int lmax = 0;
                    for (int k = 0; k < nd; ++k) lmax = max(lmax, gs.dbins[k]);
                    // a pass must hold the windows of at least 64 starts
                    if (a.cap - 2 - lmax >= 64) gs.glob = 2;
                }
                gs.safe_floor =
                    fold_safe<GEOM>(st.dt_absmax * ipmax, pmax * st.inv_bin_dur) ? 1 : 0;
                // fold mode per period: expected time-ordered points per bin
                // (the plain staged order holds consecutive points per lane)
                const bool dense_ok = gs.safe_floor && !gs.glob && !st.ilv;
                int any_chunk = 0;
                for (int k = 0; k < g; ++k) {
                    const double bw = (GEOM == ATB_GEOM_BINNED)
                                          ? st.bin_dur
                                          : gs.PIP[k].x / (double)gs.NBB[k].x;
                    const double run = bw * st.density;
                    gs.fmode[k] = dense_ok && run >= a.merge_run ? kFoldChunk : kFoldPoint;
                    any_chunk |= gs.fmode[k];
                    gs.redo[k] = 0;
                }
                gs.any_chunk = any_chunk;
            }
            __syncthreads();
            if (gs.glob == 2) {
                run_period_binned_passes(a, gs, s_hist, st, so, n_pad, nd);
            } else if (gs.glob) {
                run_group<GEOM, true>(a, gs, a.ghist + (long long)blockIdx.x * a.ghist_stride, st,
                                      so, n_pad, nd);
            } else {
                run_group<GEOM, false>(a, gs, s_hist, st, so, n_pad, nd);
            }
            pn += gs.G;
            __syncthreads();
        }
    }
}

// per-curve argmax over the grid (first maximum, as cupy.argmax)
__global__ void best_kernel(int n_curves, const long long* per_cnt, const long long* out_beg,
                            const float* power, const unsigned long long* best_key, int* best) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n_curves) return;
    if (!power) {  // winner-take-all: the packed record holds the index
        if (lane == 0) {
            const unsigned long long k = best_key[warp];
            best[warp] = k ? (int)(0xffffffffu - (unsigned)(k & 0xffffffffu)) : -1;
        }
        return;
    }
    const long long cnt = per_cnt[warp];
    const float* pw = power + out_beg[warp];
    float bv = -INFINITY;
    long long bi = 0x7fffffffffffffffLL;
    for (long long i = lane; i < cnt; i += 32) {
        const float v = pw[i];
        if (v > bv) { bv = v; bi = i; }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, bv, off);
        const long long oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    if (lane == 0) best[warp] = cnt > 0 ? (int)bi : -1;
}

// ----------------------------------------------------------------------------
// top-k peaks of each curve's power spectrum (replaces the host
// scipy.signal.find_peaks(power, distance) + sort of gpu_bls.py:146-174)
// ----------------------------------------------------------------------------

constexpr int kTopKMax = 32;
constexpr int kTopKBlock = 256;

// Block-wide argmax of (value, index): larger value, then higher index (the
// order of a stable ascending sort read from the end, as the reference's
// argsort(...)[::-1]); index -1 marks "none".
__device__ void block_argmax(float& v, long long& i, float* sv, long long* si) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, v, off);
        const long long oi = __shfl_xor_sync(0xffffffffu, i, off);
        if (ov > v || (ov == v && oi > i)) { v = ov; i = oi; }
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { sv[w] = v; si[w] = i; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kTopKBlock / 32; ++k)
            if (sv[k] > v || (sv[k] == v && si[k] > i)) { v = sv[k]; i = si[k]; }
        sv[0] = v;
        si[0] = i;
    }
    __syncthreads();
    v = sv[0];
    i = si[0];
    __syncthreads();
}

// One CTA per curve.  A peak is the midpoint (l + r) / 2 of a maximal run
// x[l..r] of equal values with x[l-1] < x[l] and x[r+1] < x[r], 1 <= l,
// r <= n-2 (scipy's _local_maxima_1d); only the run's first index scans it,
// so a round costs O(n).  Rounds pick the largest peak at least `distance`
// samples away from every peak already picked -- the order in which scipy's
// distance filter keeps peaks -- so the first k picks are scipy's top k.
// Without any peak, the k largest values are returned (the reference's
// fallback).  Equal values go to the higher index.
__global__ void __launch_bounds__(kTopKBlock) topk_peaks_kernel(
    int n_curves, const long long* per_cnt, const long long* out_beg, const float* power, int k,
    int distance, int* out_idx) {
    __shared__ float sv[kTopKBlock / 32];
    __shared__ long long si[kTopKBlock / 32];
    __shared__ long long kept[kTopKMax];
    const int c = blockIdx.x;
    if (c >= n_curves) return;
    const long long n = per_cnt[c];
    const float* x = power + out_beg[c];
    int nk = 0;
    bool fallback = false;
    for (int round = 0; round < k; ++round) {
        float bv = -INFINITY;
        long long bi = -1;
        for (long long l = threadIdx.x; l < n; l += kTopKBlock) {
            long long m = l;
            const float v = x[l];
            if (!fallback) {
                if (l < 1 || l > n - 2 || !(x[l - 1] < v)) continue;
                long long r = l;
                while (r < n - 1 && x[r + 1] == v) ++r;
                if (r > n - 2 || !(x[r + 1] < v)) continue;
                m = (l + r) / 2;
            }
            bool alive = true;
            for (int q = 0; q < nk; ++q) {
                const long long dd = m > kept[q] ? m - kept[q] : kept[q] - m;
                if (fallback ? dd == 0 : dd < distance) alive = false;
            }
            if (alive && (v > bv || (v == bv && m > bi))) {
                bv = v;
                bi = m;
            }
        }
        block_argmax(bv, bi, sv, si);
        if (bi < 0) {
            if (round == 0 && !fallback && n > 0) {  // no peak at all
                fallback = true;
                --round;
                continue;
            }
            break;
        }
        if (threadIdx.x == 0) kept[nk] = bi;
        __syncthreads();
        ++nk;
    }
    for (int q = threadIdx.x; q < k; q += kTopKBlock)
        out_idx[(long long)c * k + q] = q < nk ? (int)kept[q] : -1;
}

// per-point histogram slots of curve 0 for every period (verification only):
// the same staged points, chunking and fold_slots code as the search kernel
template <int GEOM>
__global__ void debug_fold_kernel(const double* sdt, long long n, const CurveStat* stats,
                                  const double* periods, long long n_periods, int oversample,
                                  int max_bins, int n_bins_fixed, int* out) {
    const long long n_pad = (n + kR - 1) / kR * kR;
    const long long chunks = n_pad / kR;
    const CurveStat st = stats[0];
    const long long n_full = st.ilv ? n_pad / kChunk * kChunk : 0;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < chunks * n_periods;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long p = idx / chunks, ch = idx % chunks;
        const double P = periods[p];
        const int NB = (GEOM == ATB_GEOM_BINNED)
                           ? binned_nbins(P, st.inv_bin_dur, oversample, max_bins)
                           : n_bins_fixed;
        double d[kR];
        bool sorted = true;
#pragma unroll
        for (int j = 0; j < kR; ++j) d[j] = sdt[ch * kR + j];
#pragma unroll
        for (int j = 0; j + 1 < kR; ++j) sorted = sorted && (d[j] <= d[j + 1]);
        const double IP = 1.0 / P;
        const bool safe = fold_safe<GEOM>(st.dt_absmax * IP, P * st.inv_bin_dur);
        unsigned e[kR];
        fold_slots<GEOM, GEOM == ATB_GEOM_BINNED>(d, sorted, safe, P, IP, st.inv_bin_dur, NB, e);
#pragma unroll
        for (int j = 0; j < kR; ++j) {  // the guard slot 0 is counted in slot 1
            const long long i = staged_point(ch * kR + j, n_full);
            if (i < n) out[p * n + i] = max((int)e[j], 1);
        }
    }
}

__global__ void nbins_max_kernel(int n_curves, const long long* per_beg, const long long* per_cnt,
                                 const long long* dur_beg, const int* dur_cnt,
                                 const double* periods, const double* durations, int oversample,
                                 int max_bins, int* out) {
    const int c = blockIdx.x;
    if (c >= n_curves) return;
    // same bin duration as the stage kernel
    const double* dur = durations + dur_beg[c];
    double min_dur = dur[0];
    for (int k = 1; k < dur_cnt[c]; ++k) min_dur = min(min_dur, dur[k]);
    const double ibd = 1.0 / (min_dur / (double)oversample);
    int m = 0;
    for (long long i = threadIdx.x; i < per_cnt[c]; i += blockDim.x) {
        double P = periods[per_beg[c] + i];
        if (!(P > 0.0) || !(P < 1.0e300)) P = 1.0;  // the search kernel's substitute
        m = max(m, binned_nbins(P, ibd, oversample, max_bins));
    }
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// ----------------------------------------------------------------------------
// microbenchmarks for the roofline denominators
// ----------------------------------------------------------------------------

constexpr int kBenchSlots = 4096;  // counters of the reduction benchmark

// Shared-memory reductions of 64-bit (WIDE) or 32-bit counters: pattern 0 =
// each warp's lanes hit 32 consecutive counters (conflict-free), pattern 1 =
// pseudo-random counters.
template <bool WIDE>
__global__ void __launch_bounds__(kBenchBlock) bench_smem_red_kernel(int iters, int pattern,
                                                                unsigned long long* sink) {
    __shared__ unsigned long long h[kBenchSlots];
    for (int i = threadIdx.x; i < kBenchSlots; i += blockDim.x) h[i] = 0;
    __syncthreads();
    unsigned x = threadIdx.x * 2654435761u + blockIdx.x * 97u + 1u;
    const unsigned base = (unsigned)__cvta_generic_to_shared(h);
    for (int i = 0; i < iters; ++i) {
        unsigned slot;
        if (pattern == 0) {
            slot = (threadIdx.x + (unsigned)i * 64u) & (kBenchSlots - 1);
        } else {
            x = x * 1664525u + 1013904223u;
            slot = (x >> 9) & (kBenchSlots - 1);
        }
        if (WIDE)
            asm volatile("red.shared.add.u64 [%0], %1;" ::"r"(base + slot * 8u), "l"(1ULL) : "memory");
        else
            asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(base + slot * 4u), "r"(1u) : "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(sink, h[blockIdx.x & (kBenchSlots - 1)]);
}

// FP64 fused multiply-add throughput: 8 independent chains per thread
__global__ void __launch_bounds__(kBenchBlock) bench_dfma_kernel(int iters, double* sink) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = 1.0 + 1e-9 * (threadIdx.x + k);
    const double m = 0.9999999, c = 1e-7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], m, c);
    }
    double r = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) r += a[k];
    if (r == 12345.678) sink[0] = r;  // keeps the chains alive
}

}  // namespace

// ============================================================================
// host side
// ============================================================================

struct atb_handle {
    int device = 0;
    int n_sm = 0;
    int smem_optin = 0;
    int smem_per_sm = 0;
    // the stream-ordered scratch of asynchronous plans; it keeps up to
    // kPoolKeepBytes mapped across synchronisations, so that a plan made for
    // each call of a loop does not map and unmap device memory every time
    cudaMemPool_t pool = nullptr;
    std::string err;
};
constexpr unsigned long long kPoolKeepBytes = 1ull << 30;

struct atb_plan {
    atb_handle* h = nullptr;
    atb_params prm{};
    int n_curves = 0;
    int y_is_f64 = 0;
    int grid = 0;
    int smem_bytes = 0;
    int nt = kBlock;        // threads per search CTA
    int minb = kMinBlocks;  // resident search CTAs per SM
    long long n_tiles = 0;
    std::vector<void*> allocs;
    long long scratch_bytes = 0;
    StageArgs sa{};
    SearchArgs qa{};
    int* best = nullptr;
    int* status = nullptr;
    unsigned long long* counter = nullptr;
    // plans made by atb_plan_create_async: scratch comes from the stream-ordered
    // allocator and every set-up copy, the status read-back and the release run
    // on `stream`, so that no call waits for other streams' work
    cudaStream_t stream = nullptr;
    bool async = false;
};

namespace {

int fail(atb_handle* h, int code, const char* fmt, ...) {
    if (h) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        h->err = buf;
    }
    return code;
}

#define ATB_CUDA(h, call)                                                                      \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail((h), e_ == cudaErrorMemoryAllocation ? ATB_ENOMEM : ATB_ECUDA,         \
                        "%s: %s", #call, cudaGetErrorString(e_));                              \
    } while (0)

template <typename T>
int plan_alloc(atb_plan* p, T** out, size_t count) {
    void* ptr = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = !p->async     ? cudaMalloc(&ptr, bytes)
                    : p->h->pool ? cudaMallocFromPoolAsync(&ptr, bytes, p->h->pool, p->stream)
                                 : cudaMallocAsync(&ptr, bytes, p->stream);
    if (e != cudaSuccess)
        return fail(p->h, ATB_ENOMEM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    p->allocs.push_back(ptr);
    p->scratch_bytes += (long long)bytes;
    *out = static_cast<T*>(ptr);
    return ATB_OK;
}

template <typename T>
int plan_upload(atb_plan* p, T** out, const std::vector<T>& host) {
    int rc = plan_alloc(p, out, host.size());
    if (rc) return rc;
    if (!host.empty()) {
        // from pageable memory: returns once the data are staged, so `host` may go
        ATB_CUDA(p->h, p->async ? cudaMemcpyAsync(*out, host.data(), host.size() * sizeof(T),
                                                  cudaMemcpyHostToDevice, p->stream)
                                : cudaMemcpy(*out, host.data(), host.size() * sizeof(T),
                                             cudaMemcpyHostToDevice));
    }
    return ATB_OK;
}

void plan_free(atb_plan* p) {
    for (void* q : p->allocs) {
        if (p->async)
            cudaFreeAsync(q, p->stream);
        else
            cudaFree(q);
    }
    p->allocs.clear();
}

// Device-to-host read of one small value: on the plan's stream for
// asynchronous plans (waits for that stream only), else synchronous.
cudaError_t plan_read(atb_plan* p, void* dst, const void* src, size_t bytes) {
    if (!p->async) return cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, p->stream);
    return e == cudaSuccess ? cudaStreamSynchronize(p->stream) : e;
}

// Fold-mode threshold from its atb_params field: 0 = the default, < 0 = never.
double fold_threshold(int32_t v, double dflt) {
    return v == 0 ? dflt : (v < 0 ? 1.0e300 : (double)v);
}

// The search kernel's instance for a geometry and CTA size.
using SearchFn = void (*)(const SearchArgs);
SearchFn search_fn(int geom, int nt) {
    if (geom == ATB_GEOM_BINNED)
        return nt == kBlockB ? search_kernel<ATB_GEOM_BINNED, kBlockB, kMinBlocksB>
                             : search_kernel<ATB_GEOM_BINNED, kBlock, kMinBlocks>;
    return nt == kBlockB ? search_kernel<ATB_GEOM_FIXED, kBlockB, kMinBlocksB>
                         : search_kernel<ATB_GEOM_FIXED, kBlock, kMinBlocks>;
}

// CTA shape from atb_params.cta_threads (0 = the geometry's default);
// false for an unsupported size.
bool plan_shape(const atb_params* prm, int* nt, int* minb) {
    int v = prm->cta_threads;
    if (v == 0) v = prm->geometry == ATB_GEOM_FIXED ? kDefaultFixedThreads : kBlock;
    if (v == kBlock) {
        *nt = kBlock;
        *minb = kMinBlocks;
        return true;
    }
    if (v == kBlockB) {
        *nt = kBlockB;
        *minb = kMinBlocksB;
        return true;
    }
    return false;
}

int launch_stage(atb_plan* p, cudaStream_t s) {
    if (p->y_is_f64)
        stage_kernel<double><<<p->n_curves, kStageBlock, 0, s>>>(p->sa);
    else
        stage_kernel<float><<<p->n_curves, kStageBlock, 0, s>>>(p->sa);
    ATB_CUDA(p->h, cudaGetLastError());
    return ATB_OK;
}

template <bool WIDE>
int bench_smem_red(atb_handle* h, int pattern, double* reductions_per_s) {
    if (!h || !reductions_per_s) return ATB_EINVAL;
    ATB_CUDA(h, cudaSetDevice(h->device));
    unsigned long long* sink = nullptr;
    ATB_CUDA(h, cudaMalloc(&sink, sizeof(unsigned long long)));
    const int iters = 4096, grid = h->n_sm * 2;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    bench_smem_red_kernel<WIDE><<<grid, kBenchBlock>>>(iters, pattern, sink);  // warm-up
    cudaEventRecord(a);
    for (int r = 0; r < 5; ++r) bench_smem_red_kernel<WIDE><<<grid, kBenchBlock>>>(iters, pattern, sink);
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess) return fail(h, ATB_ECUDA, "bench: %s", cudaGetErrorString(e));
    *reductions_per_s = 5.0 * grid * kBenchBlock * (double)iters / (ms * 1e-3);
    return ATB_OK;
}

}  // namespace

extern "C" {

const char* atb_version(void) { return ATB_VERSION; }

int atb_create(int device, atb_handle** out) {
    if (!out) return ATB_EINVAL;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return ATB_ECUDA;
    atb_handle* h = new atb_handle();
    h->device = device;
    cudaSetDevice(device);
    cudaDeviceGetAttribute(&h->n_sm, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&h->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    cudaDeviceGetAttribute(&h->smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&h->pool, &props) == cudaSuccess) {
        unsigned long long keep = kPoolKeepBytes;
        cudaMemPoolSetAttribute(h->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        // memory freed on one stream goes to another only once that free has
        // completed: the pool never makes a plan wait for another stream's
        // batch (a server's small request behind a large one)
        int no = 0;
        cudaMemPoolSetAttribute(h->pool, cudaMemPoolReuseAllowInternalDependencies, &no);
    } else {
        h->pool = nullptr;  // the device's default pool serves instead
        cudaGetLastError();
    }
    *out = h;
    return ATB_OK;
}

void atb_destroy(atb_handle* h) {
    // allocations still outstanding keep the pool alive until they are freed
    if (h && h->pool) cudaMemPoolDestroy(h->pool);
    delete h;
}

int atb_last_error(const atb_handle* h, char* buf, size_t len) {
    if (!h) return 0;
    if (buf && len) {
        std::strncpy(buf, h->err.c_str(), len - 1);
        buf[len - 1] = '\0';
    }
    return (int)h->err.size();
}

namespace {
int plan_create(atb_handle* h, const atb_params* prm, const atb_batch* b, const atb_outputs* o,
                cudaStream_t stream, bool async, atb_plan** out);
}  // namespace

int atb_plan_create(atb_handle* h, const atb_params* prm, const atb_batch* b,
                    const atb_outputs* o, atb_plan** out) {
    return plan_create(h, prm, b, o, nullptr, false, out);
}

int atb_plan_create_async(atb_handle* h, const atb_params* prm, const atb_batch* b,
                          const atb_outputs* o, void* stream, atb_plan** out) {
    return plan_create(h, prm, b, o, static_cast<cudaStream_t>(stream), true, out);
}

namespace {
int plan_create(atb_handle* h, const atb_params* prm, const atb_batch* b, const atb_outputs* o,
                cudaStream_t stream, bool async, atb_plan** out) {
    if (!h) return ATB_EINVAL;
    if (!prm || !b || !o || !out) return fail(h, ATB_EINVAL, "null argument");
    *out = nullptr;
    h->err.clear();
    const int nc = b->n_curves;
    if (nc < 1) return fail(h, ATB_EINVAL, "n_curves must be >= 1");
    if (prm->geometry == ATB_GEOM_FIXED) {
        if (prm->objective != ATB_OBJ_FAST)
            return fail(h, ATB_EINVAL, "the fixed-bin geometry uses the fast objective");
        if (prm->n_bins < 2 || prm->n_bins > (1 << 24))
            return fail(h, ATB_EINVAL, "n_bins=%d out of range [2, 2^24]", prm->n_bins);
    } else if (prm->geometry == ATB_GEOM_BINNED) {
        if (prm->objective != ATB_OBJ_SNR && prm->objective != ATB_OBJ_LIKELIHOOD)
            return fail(h, ATB_EINVAL, "the binned geometry uses the snr or likelihood objective");
        if (prm->oversample < 1 || prm->oversample > 1000)
            return fail(h, ATB_EINVAL, "oversample=%d out of range [1, 1000]", prm->oversample);
        if (prm->max_bins != 0 && prm->max_bins < prm->oversample + 2)
            return fail(h, ATB_EINVAL, "max_bins=%d must be 0 or >= oversample+2", prm->max_bins);
    } else {
        return fail(h, ATB_EINVAL, "unknown geometry %d", prm->geometry);
    }
    int cta_nt = kBlock, cta_minb = kMinBlocks;
    if (!plan_shape(prm, &cta_nt, &cta_minb))
        return fail(h, ATB_EINVAL, "cta_threads=%d: 0, %d or %d expected", prm->cta_threads,
                    kBlock, kBlockB);
    if (!b->point_offset || !b->period_begin || !b->period_count || !b->dur_begin ||
        !b->dur_count || !b->out_begin)
        return fail(h, ATB_EINVAL, "batch index arrays must not be NULL");
    if (!b->t || !b->y || !b->periods || !b->durations)
        return fail(h, ATB_EINVAL, "batch data pointers must not be NULL");
    if (!o->power && !o->best_key)
        return fail(h, ATB_EINVAL, "outputs.power and outputs.best_key must not both be NULL");

    std::vector<long long> pt_off(nc + 1), t_off(nc), per_beg(nc), per_cnt(nc), dur_beg(nc),
        out_beg(nc), stage_off(nc), tile_off(nc + 1);
    std::vector<int> dur_cnt(nc), order(nc);
    long long staged = 0, n_out_max = 0;
    for (int c = 0; c <= nc; ++c) pt_off[c] = b->point_offset[c];
    for (int c = 0; c < nc; ++c) {
        const long long n = pt_off[c + 1] - pt_off[c];
        if (n < 0) return fail(h, ATB_EINVAL, "curve %d: decreasing point_offset", c);
        if (n > (1LL << 26)) return fail(h, ATB_EINVAL, "curve %d: more than 2^26 points", c);
        t_off[c] = b->time_offset ? b->time_offset[c] : pt_off[c];
        per_beg[c] = b->period_begin[c];
        per_cnt[c] = b->period_count[c];
        dur_beg[c] = b->dur_begin[c];
        dur_cnt[c] = b->dur_count[c];
        out_beg[c] = b->out_begin[c];
        if (per_cnt[c] < 0 || per_beg[c] < 0 || out_beg[c] < 0 || dur_beg[c] < 0)
            return fail(h, ATB_EINVAL, "curve %d: negative grid index", c);
        if (per_cnt[c] > (1LL << 30)) return fail(h, ATB_EINVAL, "curve %d: too many periods", c);
        if (dur_cnt[c] < 1 || dur_cnt[c] > kMaxDur)
            return fail(h, ATB_EINVAL, "curve %d: dur_count=%d outside [1, %d]", c, dur_cnt[c],
                        kMaxDur);
        stage_off[c] = staged;
        staged += (n + kR - 1) / kR * kR;
        staged = (staged + kStageAlign - 1) / kStageAlign * kStageAlign;
        n_out_max = std::max(n_out_max, out_beg[c] + per_cnt[c]);
    }
    // largest-first schedule of curves (cost ~ points x periods)
    for (int c = 0; c < nc; ++c) order[c] = c;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const double cx = (double)(pt_off[x + 1] - pt_off[x] + 64) * (double)per_cnt[x];
        const double cy = (double)(pt_off[y + 1] - pt_off[y] + 64) * (double)per_cnt[y];
        return cx > cy;
    });
    // periods per tile: as requested, else the largest power of two up to
    // kTileP that still gives every resident CTA about four tiles (a small
    // batch -- one curve of a few thousand periods -- otherwise leaves most
    // SMs idle)
    int tile_p = prm->tile_periods;
    if (tile_p < 1 || tile_p > kTileP) {
        const long long slots = 4LL * h->n_sm * cta_minb;
        tile_p = kTileP;
        while (tile_p > 8) {
            long long tiles = 0;
            for (int c = 0; c < nc; ++c) tiles += (per_cnt[c] + tile_p - 1) / tile_p;
            if (tiles >= slots) break;
            tile_p /= 2;
        }
    }
    tile_off[0] = 0;
    for (int j = 0; j < nc; ++j)
        tile_off[j + 1] = tile_off[j] + (per_cnt[order[j]] + tile_p - 1) / tile_p;

    ATB_CUDA(h, cudaSetDevice(h->device));
    atb_plan* p = new atb_plan();
    p->h = h;
    p->stream = stream;
    p->async = async;
    p->prm = *prm;
    p->n_curves = nc;
    p->y_is_f64 = b->y_is_f64 ? 1 : 0;
    p->n_tiles = tile_off[nc];
    p->nt = cta_nt;
    p->minb = cta_minb;

    int rc = ATB_OK;
    long long *d_pt, *d_toff, *d_pbeg, *d_pcnt, *d_dbeg, *d_obeg, *d_soff, *d_tiles;
    int *d_dcnt, *d_order, *d_dbins;
    double* d_sdt;
    int *d_sqw, *d_sqy;
    CurveStat* d_stats;
    if ((rc = plan_upload(p, &d_pt, pt_off)) || (rc = plan_upload(p, &d_toff, t_off)) ||
        (rc = plan_upload(p, &d_pbeg, per_beg)) || (rc = plan_upload(p, &d_pcnt, per_cnt)) ||
        (rc = plan_upload(p, &d_dbeg, dur_beg)) || (rc = plan_upload(p, &d_obeg, out_beg)) ||
        (rc = plan_upload(p, &d_soff, stage_off)) || (rc = plan_upload(p, &d_tiles, tile_off)) ||
        (rc = plan_upload(p, &d_dcnt, dur_cnt)) || (rc = plan_upload(p, &d_order, order)) ||
        (rc = plan_alloc(p, &d_dbins, (size_t)nc * kMaxDur)) ||
        (rc = plan_alloc(p, &d_sdt, (size_t)staged)) || (rc = plan_alloc(p, &d_sqw, (size_t)staged)) ||
        (rc = plan_alloc(p, &d_sqy, (size_t)staged)) || (rc = plan_alloc(p, &d_stats, (size_t)nc)) ||
        (rc = plan_alloc(p, &p->status, 1)) || (rc = plan_alloc(p, &p->counter, 1))) {
        plan_free(p);
        delete p;
        return rc;
    }

    StageArgs& sa = p->sa;
    sa.pt_off = d_pt;
    sa.t_off = d_toff;
    sa.stage_off = d_soff;
    sa.dur_beg = d_dbeg;
    sa.dur_cnt = d_dcnt;
    sa.t = b->t;
    sa.y = b->y;
    sa.w = b->w;
    sa.durations = b->durations;
    sa.sdt = d_sdt;
    sa.sqw = d_sqw;
    sa.sqy = d_sqy;
    sa.stats = d_stats;
    sa.dbins = d_dbins;
    sa.oversample = prm->geometry == ATB_GEOM_BINNED ? prm->oversample : 1;
    sa.status = p->status;
    sa.periods = b->periods;
    sa.per_beg = d_pbeg;
    sa.per_cnt = d_pcnt;
    sa.geometry = prm->geometry;
    sa.n_bins_fixed = prm->n_bins;
    sa.max_bins = prm->max_bins;

    // shared-memory histogram capacity and the global fallback size
    const int static_smem = (int)sizeof(GroupSmem) + 64;
    // cta_minb CTAs share the SM's shared memory (1 KiB per CTA is reserved)
    int dyn = std::min(h->smem_optin, h->smem_per_sm / cta_minb - 1024) - static_smem;
    dyn = dyn / 16 * 16;
    const int cap = dyn / 16;
    int nb_max = prm->n_bins;
    if (prm->geometry == ATB_GEOM_BINNED) {
        // largest bin count over the batch sizes the global-histogram fallback
        int* d_nb = nullptr;
        if ((rc = plan_alloc(p, &d_nb, 1))) { plan_free(p); delete p; return rc; }
        cudaMemsetAsync(d_nb, 0, sizeof(int), stream);
        nbins_max_kernel<<<nc, 256, 0, stream>>>(nc, d_pbeg, d_pcnt, d_dbeg, d_dcnt, b->periods,
                                                 b->durations, prm->oversample, prm->max_bins,
                                                 d_nb);
        cudaError_t e = plan_read(p, &nb_max, d_nb, sizeof(int));
        if (e != cudaSuccess) {
            plan_free(p);
            delete p;
            return fail(h, ATB_ECUDA, "n_bins reduction: %s", cudaGetErrorString(e));
        }
        int nd_max = 1;
        for (int c = 0; c < nc; ++c) nd_max = std::max(nd_max, dur_cnt[c]);
        if (nb_max >= (1 << 27) || (long long)nb_max * nd_max >= (1LL << 31)) {
            plan_free(p);
            delete p;
            return fail(h, ATB_EINVAL, "a period needs %d bins (limit 2^27 and bins x durations < 2^31)",
                        nb_max);
        }
    }
    int occ = 1;
    const SearchFn sfn = search_fn(prm->geometry, cta_nt);
    cudaError_t e0 = cudaFuncSetAttribute(sfn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    if (e0 != cudaSuccess) {
        plan_free(p);
        delete p;
        return fail(h, ATB_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e0));
    }
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, sfn, cta_nt, dyn);
    occ = std::max(occ, 1);
    long long grid = (long long)h->n_sm * occ;
    grid = std::max(1LL, std::min(grid, p->n_tiles));
    p->grid = (int)grid;
    p->smem_bytes = dyn;

    longlong2* d_ghist = nullptr;
    long long gstride = 0;
    if (nb_max + 2 > cap) {
        gstride = ((long long)nb_max + 2 + 15) / 16 * 16;
        const long long bytes = gstride * 16 * grid;
        if (bytes > (16LL << 30)) {
            plan_free(p);
            delete p;
            return fail(h, ATB_EINVAL, "global histograms would need %lld bytes", bytes);
        }
        if ((rc = plan_alloc(p, &d_ghist, (size_t)(gstride * grid)))) {
            plan_free(p);
            delete p;
            return rc;
        }
    }

    SearchArgs& qa = p->qa;
    qa.objective = prm->objective;
    qa.n_bins_fixed = prm->n_bins;
    qa.oversample = sa.oversample;
    qa.max_bins = prm->max_bins;
    qa.n_curves = nc;
    qa.cap = cap;
    qa.n_tiles = p->n_tiles;
    qa.pt_off = d_pt;
    qa.stage_off = d_soff;
    qa.per_beg = d_pbeg;
    qa.per_cnt = d_pcnt;
    qa.dur_beg = d_dbeg;
    qa.dur_cnt = d_dcnt;
    qa.out_beg = d_obeg;
    qa.tile_off = d_tiles;
    qa.order = d_order;
    qa.periods = b->periods;
    qa.durations = b->durations;
    qa.sdt = d_sdt;
    qa.sqw = d_sqw;
    qa.sqy = d_sqy;
    qa.stats = d_stats;
    qa.dbins = d_dbins;
    qa.power = o->power;
    qa.best_key = reinterpret_cast<unsigned long long*>(o->best_key);
    qa.tile_p = tile_p;
    qa.merge_run = fold_threshold(prm->merge_run, kDefaultMergeRun);
    qa.depth = o->depth;
    qa.depth_err = o->depth_err;
    qa.t0 = o->t0;
    qa.duration = o->duration;
    qa.window = o->window;
    qa.ghist = d_ghist;
    qa.ghist_stride = gstride;
    qa.tile_counter = p->counter;
    qa.status = p->status;
    p->best = o->best_period;
    // every set-up copy has completed (or, for asynchronous plans, is ordered
    // before the plan's kernels on its stream)
    if (!async) ATB_CUDA(h, cudaDeviceSynchronize());
    *out = p;
    return ATB_OK;
}
}  // namespace

int atb_plan_execute(atb_plan* p, void* stream) {
    if (!p) return ATB_EINVAL;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    atb_handle* h = p->h;
    ATB_CUDA(h, cudaMemsetAsync(p->counter, 0, sizeof(unsigned long long), s));
    ATB_CUDA(h, cudaMemsetAsync(p->status, 0, sizeof(int), s));
    int rc = launch_stage(p, s);
    if (rc) return rc;
    if (p->n_tiles > 0) {
        search_fn(p->prm.geometry, p->nt)<<<p->grid, p->nt, p->smem_bytes, s>>>(p->qa);
        ATB_CUDA(h, cudaGetLastError());
    }
    if (p->best) {
        const int threads = 256;
        const int blocks = (p->n_curves * 32 + threads - 1) / threads;
        best_kernel<<<blocks, threads, 0, s>>>(p->n_curves, p->qa.per_cnt, p->qa.out_beg,
                                               p->qa.power, p->qa.best_key, p->best);
        ATB_CUDA(h, cudaGetLastError());
    }
    return ATB_OK;
}

int atb_plan_kernel_count(const atb_plan* p) {
    if (!p) return 0;
    return 1 + (p->n_tiles > 0 ? 1 : 0) + (p->best ? 1 : 0);
}

int64_t atb_plan_scratch_bytes(const atb_plan* p) { return p ? p->scratch_bytes : 0; }

int atb_plan_curve_layout(atb_plan* p, int32_t* layout, int32_t* occupancy_bits) {
    if (!p || !layout || !occupancy_bits) return ATB_EINVAL;
    ATB_CUDA(p->h, cudaSetDevice(p->h->device));
    std::vector<CurveStat> st(p->n_curves);
    ATB_CUDA(p->h, plan_read(p, st.data(), p->sa.stats, sizeof(CurveStat) * st.size()));
    for (int c = 0; c < p->n_curves; ++c) {
        layout[c] = st[c].tcheck ? ATB_LAYOUT_TIGHT_CHECKED : st[c].packmode;
        occupancy_bits[c] = st[c].occ_bits;
    }
    return ATB_OK;
}

int atb_plan_check(atb_plan* p) {
    if (!p) return ATB_EINVAL;
    int st = 0;
    ATB_CUDA(p->h, plan_read(p, &st, p->status, sizeof(int)));
    if (st & 1) return fail(p->h, ATB_EDATA, "input contains non-finite values or weights <= 0");
    if (st & 2) return fail(p->h, ATB_EDATA, "durations must be positive and finite");
    if (st & 4) return fail(p->h, ATB_EDATA, "periods must be positive and finite");
    return ATB_OK;
}

void atb_plan_destroy(atb_plan* p) {
    if (!p) return;
    cudaSetDevice(p->h->device);
    plan_free(p);
    delete p;
}

int atb_search(atb_handle* h, const atb_params* prm, const atb_batch* b, const atb_outputs* o,
               void* stream) {
    atb_plan* p = nullptr;
    int rc = atb_plan_create(h, prm, b, o, &p);
    if (rc) return rc;
    rc = atb_plan_execute(p, stream);
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
        if (e != cudaSuccess) rc = fail(h, ATB_ECUDA, "search: %s", cudaGetErrorString(e));
    }
    if (!rc) rc = atb_plan_check(p);
    atb_plan_destroy(p);
    return rc;
}

int atb_run_gpu_bls(atb_handle* h, const double* t, const float* y, const float* w, int64_t n,
                    const double* periods, int64_t n_periods, const double* durations,
                    int32_t n_durations, int32_t n_bins, float* power, double* t0,
                    float* duration, float* depth, int32_t* best_index, void* stream) {
    if (!h) return ATB_EINVAL;
    atb_params prm{ATB_GEOM_FIXED, ATB_OBJ_FAST, n_bins, 10, 0, 0};
    const int64_t pt[2] = {0, n};
    const int64_t zero = 0;
    const int64_t pc = n_periods;
    const int32_t dc = n_durations;
    atb_batch b{};
    b.n_curves = 1;
    b.point_offset = pt;
    b.period_begin = &zero;
    b.period_count = &pc;
    b.dur_begin = &zero;
    b.dur_count = &dc;
    b.out_begin = &zero;
    b.t = t;
    b.y = y;
    b.w = w;
    b.periods = periods;
    b.durations = durations;
    int32_t* d_best = nullptr;
    if (best_index) {
        ATB_CUDA(h, cudaMalloc(&d_best, sizeof(int32_t)));
    }
    atb_outputs o{};
    o.power = power;
    o.t0 = t0;
    o.duration = duration;
    o.depth = depth;
    o.best_period = d_best;
    int rc = atb_search(h, &prm, &b, &o, stream);
    if (!rc && best_index) {
        cudaError_t e = cudaMemcpy(best_index, d_best, sizeof(int32_t), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = fail(h, ATB_ECUDA, "best index: %s", cudaGetErrorString(e));
    }
    if (d_best) cudaFree(d_best);
    return rc;
}

int atb_run_vbls_exact_parity(atb_handle* h, const double* time, const float* flux,
                              const float* weights, int64_t n_targets, int64_t n_data,
                              const double* periods, int64_t n_periods, const double* durations,
                              int32_t n_durations, int32_t oversample, int32_t max_bins,
                              int32_t objective, float* power, double* t0, float* duration,
                              float* depth, int32_t* best_index, void* stream) {
    if (!h) return ATB_EINVAL;
    if (n_targets < 1 || n_targets > (1 << 30)) return fail(h, ATB_EINVAL, "n_targets out of range");
    atb_params prm{ATB_GEOM_BINNED, objective, 0, oversample, max_bins, 0};
    const int nc = (int)n_targets;
    std::vector<int64_t> pt(nc + 1), toff(nc, 0), pbeg(nc, 0), pcnt(nc, n_periods), dbeg(nc, 0),
        obeg(nc);
    std::vector<int32_t> dcnt(nc, n_durations);
    for (int c = 0; c <= nc; ++c) pt[c] = (int64_t)c * n_data;
    for (int c = 0; c < nc; ++c) obeg[c] = (int64_t)c * n_periods;
    atb_batch b{};
    b.n_curves = nc;
    b.point_offset = pt.data();
    b.time_offset = toff.data();
    b.period_begin = pbeg.data();
    b.period_count = pcnt.data();
    b.dur_begin = dbeg.data();
    b.dur_count = dcnt.data();
    b.out_begin = obeg.data();
    b.t = time;
    b.y = flux;
    b.w = weights;
    b.periods = periods;
    b.durations = durations;
    atb_outputs o{};
    o.power = power;
    o.t0 = t0;
    o.duration = duration;
    o.depth = depth;
    o.best_period = best_index;
    return atb_search(h, &prm, &b, &o, stream);
}

int atb_debug_fold(atb_handle* h, const atb_params* prm, const double* t, const float* y,
                   const float* w, int64_t n, const double* periods, int64_t n_periods,
                   const double* durations, int32_t n_durations, int32_t* out_slots,
                   void* stream) {
    if (!h) return ATB_EINVAL;
    if (!prm || !out_slots || n < 1 || n_periods < 1) return fail(h, ATB_EINVAL, "bad arguments");
    const int64_t pt[2] = {0, n};
    const int64_t zero = 0;
    const int64_t pc = n_periods;
    const int32_t dc = n_durations;
    atb_batch b{};
    b.n_curves = 1;
    b.point_offset = pt;
    b.period_begin = &zero;
    b.period_count = &pc;
    b.dur_begin = &zero;
    b.dur_count = &dc;
    b.out_begin = &zero;
    b.t = t;
    b.y = y;
    b.w = w;
    b.periods = periods;
    b.durations = durations;
    float* tmp = nullptr;
    ATB_CUDA(h, cudaMalloc(&tmp, sizeof(float) * (size_t)n_periods));
    atb_outputs o{};
    o.power = tmp;
    atb_plan* p = nullptr;
    int rc = atb_plan_create(h, prm, &b, &o, &p);
    if (!rc) {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        rc = launch_stage(p, s);
        if (!rc) {
            const long long total = (long long)n * n_periods;
            const int blocks = (int)std::min<long long>((total + 255) / 256, 65535);
            if (prm->geometry == ATB_GEOM_BINNED)
                debug_fold_kernel<ATB_GEOM_BINNED><<<blocks, 256, 0, s>>>(
                    p->sa.sdt, n, p->sa.stats, periods, n_periods, prm->oversample,
                    prm->max_bins, prm->n_bins, out_slots);
            else
                debug_fold_kernel<ATB_GEOM_FIXED><<<blocks, 256, 0, s>>>(
                    p->sa.sdt, n, p->sa.stats, periods, n_periods, prm->oversample,
                    prm->max_bins, prm->n_bins, out_slots);
            cudaError_t e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) rc = fail(h, ATB_ECUDA, "debug fold: %s", cudaGetErrorString(e));
        }
        atb_plan_destroy(p);
    }
    cudaFree(tmp);
    return rc;
}


int atb_plan_top_k(atb_plan* p, int32_t k, int32_t distance, int32_t* out_idx, void* stream) {
    if (!p || !out_idx) return ATB_EINVAL;
    if (k < 1 || k > kTopKMax) return fail(p->h, ATB_EINVAL, "k=%d outside [1, %d]", k, kTopKMax);
    if (distance < 1) return fail(p->h, ATB_EINVAL, "distance=%d must be >= 1", distance);
    if (!p->qa.power) return fail(p->h, ATB_EINVAL, "the plan has no per-period power output");
    ATB_CUDA(p->h, cudaSetDevice(p->h->device));
    topk_peaks_kernel<<<p->n_curves, kTopKBlock, 0, static_cast<cudaStream_t>(stream)>>>(
        p->n_curves, p->qa.per_cnt, p->qa.out_beg, p->qa.power, k, distance, out_idx);
    ATB_CUDA(p->h, cudaGetLastError());
    return ATB_OK;
}

int atb_plan_profile(atb_plan* p, void* stream, float* ms_stage, float* ms_search,
                     float* ms_best) {
    if (!p) return ATB_EINVAL;
    atb_handle* h = p->h;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaEvent_t ev[4];
    for (auto& e : ev) ATB_CUDA(h, cudaEventCreate(&e));
    ATB_CUDA(h, cudaMemsetAsync(p->counter, 0, sizeof(unsigned long long), s));
    ATB_CUDA(h, cudaMemsetAsync(p->status, 0, sizeof(int), s));
    ATB_CUDA(h, cudaEventRecord(ev[0], s));
    int rc = launch_stage(p, s);
    ATB_CUDA(h, cudaEventRecord(ev[1], s));
    if (!rc && p->n_tiles > 0) {
        search_fn(p->prm.geometry, p->nt)<<<p->grid, p->nt, p->smem_bytes, s>>>(p->qa);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(h, ATB_ECUDA, "search launch: %s", cudaGetErrorString(e));
    }
    ATB_CUDA(h, cudaEventRecord(ev[2], s));
    if (!rc && p->best) {
        const int blocks = (p->n_curves * 32 + 255) / 256;
        best_kernel<<<blocks, 256, 0, s>>>(p->n_curves, p->qa.per_cnt, p->qa.out_beg,
                                           p->qa.power, p->qa.best_key, p->best);
    }
    ATB_CUDA(h, cudaEventRecord(ev[3], s));
    ATB_CUDA(h, cudaEventSynchronize(ev[3]));
    float m[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) cudaEventElapsedTime(&m[k], ev[k], ev[k + 1]);
    for (auto& e : ev) cudaEventDestroy(e);
    if (ms_stage) *ms_stage = m[0];
    if (ms_search) *ms_search = m[1];
    if (ms_best) *ms_best = m[2];
    return rc;
}


int atb_bench_smem_red_u64(atb_handle* h, int pattern, double* reductions_per_s) {
    return bench_smem_red<true>(h, pattern, reductions_per_s);
}

int atb_bench_smem_red_u32(atb_handle* h, int pattern, double* reductions_per_s) {
    return bench_smem_red<false>(h, pattern, reductions_per_s);
}

int atb_bench_dfma(atb_handle* h, double* fma_per_s) {
    if (!h || !fma_per_s) return ATB_EINVAL;
    ATB_CUDA(h, cudaSetDevice(h->device));
    double* sink = nullptr;
    ATB_CUDA(h, cudaMalloc(&sink, sizeof(double)));
    const int iters = 8192, grid = h->n_sm * 4;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    bench_dfma_kernel<<<grid, kBenchBlock>>>(iters, sink);
    cudaEventRecord(a);
    for (int r = 0; r < 5; ++r) bench_dfma_kernel<<<grid, kBenchBlock>>>(iters, sink);
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess) return fail(h, ATB_ECUDA, "bench: %s", cudaGetErrorString(e));
    *fma_per_s = 5.0 * grid * kBenchBlock * 8.0 * (double)iters / (ms * 1e-3);
    return ATB_OK;
}

}  // extern "C"

// ============================================================================
// Single-curve search that allocates nothing
// ============================================================================
//
// Every buffer the search needs beyond the caller's inputs and outputs lives in
// one file-scope device array: the staged points of the curve, its constants,
// the one-curve index arrays, the work-queue counter and the status word.  The
// array exists once per device that loads this library and stays resident
// until the process exits.

namespace {

constexpr long long kStaticPoints = ATB_STATIC_MAX_POINTS;
constexpr size_t kStaticMetaBytes = 4096;
constexpr size_t kStaticBytes = (size_t)kStaticPoints * 16 + kStaticMetaBytes;
static_assert(kStaticPoints % kStageAlign == 0, "whole staging chunks");

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

// byte offsets inside g_static_scratch
constexpr size_t kOffDt = 0;
constexpr size_t kOffQw = (size_t)kStaticPoints * 8;
constexpr size_t kOffQy = (size_t)kStaticPoints * 12;
constexpr size_t kOffMeta = (size_t)kStaticPoints * 16;

struct StaticMeta {
    long long pt_off[2];
    long long t_off[1];
    long long stage_off[1];
    long long per_beg[1];
    long long per_cnt[1];
    long long dur_beg[1];
    long long out_beg[1];
    long long tile_off[2];
    unsigned long long tile_counter;
    int dur_cnt[1];
    int order[1];
    int status;
    int nb_max;
    int dbins[kMaxDur];
    CurveStat stats[1];
};
static_assert(sizeof(StaticMeta) <= kStaticMetaBytes, "static metadata fits its slot");

// one-curve index arrays and the counters that must start at zero
__global__ void static_meta_init(StaticMeta* m, long long n, long long n_periods, int nd,
                                 long long n_tiles) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    m->pt_off[0] = 0;
    m->pt_off[1] = n;
    m->t_off[0] = 0;
    m->stage_off[0] = 0;
    m->per_beg[0] = 0;
    m->per_cnt[0] = n_periods;
    m->dur_beg[0] = 0;
    m->out_beg[0] = 0;
    m->tile_off[0] = 0;
    m->tile_off[1] = n_tiles;
    m->tile_counter = 0ULL;
    m->dur_cnt[0] = nd;
    m->order[0] = 0;
    m->status = 0;
    m->nb_max = 0;
}

int static_fail(char* err, size_t err_len, int code, const char* fmt, ...) {
    if (err && err_len) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(err, err_len, fmt, ap);
        va_end(ap);
    }
    return code;
}

}  // namespace

extern "C" int atb_search_curve_static(const atb_params* prm, const double* t, const void* y,
                                       int32_t y_is_f64, const float* w, int64_t n,
                                       const double* periods, int64_t n_periods,
                                       const double* durations, int32_t n_durations,
                                       float* power, float* depth, float* depth_err, double* t0,
                                       float* duration, int32_t* window, int32_t* best_index,
                                       void* stream, char* err, size_t err_len) {
    if (err && err_len) err[0] = '\0';
    if (!prm || !t || !y || !periods || !durations || !power)
        return static_fail(err, err_len, ATB_EINVAL, "null argument");
    if (n < 1 || n > kStaticPoints)
        return static_fail(err, err_len, ATB_EINVAL,
                           "n=%lld points outside [1, %lld] (the static scratch limit)",
                           (long long)n, (long long)kStaticPoints);
    if (n_periods < 1 || n_periods > (1LL << 30))
        return static_fail(err, err_len, ATB_EINVAL, "n_periods=%lld out of range",
                           (long long)n_periods);
    if (n_durations < 1 || n_durations > kMaxDur)
        return static_fail(err, err_len, ATB_EINVAL, "n_durations=%d outside [1, %d]",
                           n_durations, kMaxDur);
    if (prm->geometry == ATB_GEOM_FIXED) {
        if (prm->objective != ATB_OBJ_FAST)
            return static_fail(err, err_len, ATB_EINVAL, "the fixed-bin geometry uses the fast objective");
        if (prm->n_bins < 2 || prm->n_bins > (1 << 24))
            return static_fail(err, err_len, ATB_EINVAL, "n_bins=%d out of range", prm->n_bins);
    } else if (prm->geometry == ATB_GEOM_BINNED) {
        if (prm->objective != ATB_OBJ_SNR && prm->objective != ATB_OBJ_LIKELIHOOD)
            return static_fail(err, err_len, ATB_EINVAL,
                               "the binned geometry uses the snr or likelihood objective");
        if (prm->oversample < 1 || prm->oversample > 1000)
            return static_fail(err, err_len, ATB_EINVAL, "oversample=%d out of range", prm->oversample);
        if (prm->max_bins != 0 && prm->max_bins < prm->oversample + 2)
            return static_fail(err, err_len, ATB_EINVAL, "max_bins=%d must be 0 or >= oversample+2",
                               prm->max_bins);
    } else {
        return static_fail(err, err_len, ATB_EINVAL, "unknown geometry %d", prm->geometry);
    }
    // one CTA shape here: its shared-memory size bounds the bin counts accepted
    if (prm->cta_threads != 0 && prm->cta_threads != kBlock)
        return static_fail(err, err_len, ATB_EINVAL, "cta_threads=%d: 0 or %d expected",
                           prm->cta_threads, kBlock);

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return static_fail(err, err_len, ATB_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    int n_sm = 0, smem_optin = 0, smem_per_sm = 0;
    e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    if (e != cudaSuccess)
        return static_fail(err, err_len, ATB_ECUDA, "cudaDeviceGetAttribute: %s",
                           cudaGetErrorString(e));
    const int static_smem = (int)sizeof(GroupSmem) + 64;
    int dyn = std::min(smem_optin, smem_per_sm / kMinBlocks - 1024) - static_smem;
    dyn = dyn / 16 * 16;
    const int cap = dyn / 16;

    // Set-up, with the device current: the scratch array's device address and
    // the search kernels' shared-memory limit.  Both are taken again on every
    // call (neither allocates), so a cudaDeviceReset or a recreated primary
    // context between calls cannot leave a stale address or a lost limit.  The
    // first call on a device also makes the runtime load this library's
    // kernels and its scratch array onto that device.
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_static_scratch);
    if (e != cudaSuccess || !ptr)
        return static_fail(err, err_len, ATB_ECUDA, "cudaGetSymbolAddress: %s",
                           cudaGetErrorString(e));
    e = cudaFuncSetAttribute(search_kernel<ATB_GEOM_BINNED, kBlock, kMinBlocks>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(search_kernel<ATB_GEOM_FIXED, kBlock, kMinBlocks>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    if (e != cudaSuccess)
        return static_fail(err, err_len, ATB_ECUDA, "cudaFuncSetAttribute: %s",
                           cudaGetErrorString(e));
    unsigned char* base = static_cast<unsigned char*>(ptr);
    double* sdt = reinterpret_cast<double*>(base + kOffDt);
    int* sqw = reinterpret_cast<int*>(base + kOffQw);
    int* sqy = reinterpret_cast<int*>(base + kOffQy);
    StaticMeta* m = reinterpret_cast<StaticMeta*>(base + kOffMeta);

    // fixed bins: one histogram of n_bins per period must fit shared memory
    // (checked before the first launch, so that a rejected call leaves no work
    // in flight on the shared array)
    if (prm->geometry == ATB_GEOM_FIXED && prm->n_bins + 2 > cap)
        return static_fail(err, err_len, ATB_EINVAL,
                           "n_bins=%d; this entry point holds at most %d bins per period "
                           "(use the plan API)", prm->n_bins, cap - 2);
    const long long n_tiles = (n_periods + kTileP - 1) / kTileP;
    static_meta_init<<<1, 32, 0, s>>>(m, n, n_periods, n_durations, n_tiles);

    if (prm->geometry == ATB_GEOM_BINNED)
        nbins_max_kernel<<<1, 256, 0, s>>>(1, m->per_beg, m->per_cnt, m->dur_beg, m->dur_cnt,
                                           periods, durations, prm->oversample, prm->max_bins,
                                           &m->nb_max);

    StageArgs sa{};
    sa.pt_off = m->pt_off;
    sa.t_off = m->t_off;
    sa.stage_off = m->stage_off;
    sa.dur_beg = m->dur_beg;
    sa.dur_cnt = m->dur_cnt;
    sa.t = t;
    sa.y = y;
    sa.w = w;
    sa.durations = durations;
    sa.sdt = sdt;
    sa.sqw = sqw;
    sa.sqy = sqy;
    sa.stats = m->stats;
    sa.dbins = m->dbins;
    sa.oversample = prm->geometry == ATB_GEOM_BINNED ? prm->oversample : 1;
    sa.status = &m->status;
    sa.periods = periods;
    sa.per_beg = m->per_beg;
    sa.per_cnt = m->per_cnt;
    sa.geometry = prm->geometry;
    sa.n_bins_fixed = prm->n_bins;
    sa.max_bins = prm->max_bins;
    if (y_is_f64)
        stage_kernel<double><<<1, kStageBlock, 0, s>>>(sa);
    else
        stage_kernel<float><<<1, kStageBlock, 0, s>>>(sa);

    // Astropy bins: the largest period's bin count and the durations' window
    // lengths in bins (written by the stage kernel).  A period whose
    // histogram does not fit shared memory is searched in bin-range passes
    // through shared memory when the search kernel takes that path for it
    // (oversample <= kMpPadMax and a pass holds >= 64 window starts); the
    // global-histogram path, which needs allocated memory, is rejected here.
    int nb_max = prm->n_bins;
    if (prm->geometry == ATB_GEOM_BINNED) {
        int dbins[kMaxDur];
        e = cudaMemcpyAsync(&nb_max, &m->nb_max, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dbins, m->dbins, sizeof(int) * n_durations,
                                cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess)
            return static_fail(err, err_len, ATB_ECUDA, "bin count: %s", cudaGetErrorString(e));
        int lmax = 0;
        for (int k = 0; k < n_durations; ++k) lmax = std::max(lmax, dbins[k]);
        const bool passes = prm->oversample <= kMpPadMax && cap - 2 - lmax >= 64;
        if (nb_max + 2 > cap && !passes)
            return static_fail(err, err_len, ATB_EINVAL,
                               "a period needs %d bins and windows of %d bins; this entry point "
                               "holds at most %d per period (use the plan API)",
                               nb_max, lmax, cap - 2);
        if (nb_max >= (1 << 27))
            return static_fail(err, err_len, ATB_EINVAL, "a period needs %d bins (limit 2^27)",
                               nb_max);
    }
    if ((long long)nb_max * n_durations >= (1LL << 31))
        return static_fail(err, err_len, ATB_EINVAL, "bins x durations too large");

    SearchArgs qa{};
    qa.objective = prm->objective;
    qa.n_bins_fixed = prm->n_bins;
    qa.oversample = sa.oversample;
    qa.max_bins = prm->max_bins;
    qa.n_curves = 1;
    qa.cap = cap;
    qa.n_tiles = n_tiles;
    qa.pt_off = m->pt_off;
    qa.stage_off = m->stage_off;
    qa.per_beg = m->per_beg;
    qa.per_cnt = m->per_cnt;
    qa.dur_beg = m->dur_beg;
    qa.dur_cnt = m->dur_cnt;
    qa.out_beg = m->out_beg;
    qa.tile_off = m->tile_off;
    qa.order = m->order;
    qa.periods = periods;
    qa.durations = durations;
    qa.sdt = sdt;
    qa.sqw = sqw;
    qa.sqy = sqy;
    qa.stats = m->stats;
    qa.dbins = m->dbins;
    qa.power = power;
    qa.depth = depth;
    qa.depth_err = depth_err;
    qa.t0 = t0;
    qa.duration = duration;
    qa.window = window;
    qa.ghist = nullptr;  // never reached: oversized periods take the passes (checked above)
    qa.ghist_stride = 0;
    qa.tile_counter = &m->tile_counter;
    qa.tile_p = kTileP;
    qa.merge_run = fold_threshold(prm->merge_run, kDefaultMergeRun);
    qa.status = &m->status;
    int occ = 1;
    if (prm->geometry == ATB_GEOM_BINNED)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &occ, search_kernel<ATB_GEOM_BINNED, kBlock, kMinBlocks>, kBlock, dyn);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &occ, search_kernel<ATB_GEOM_FIXED, kBlock, kMinBlocks>, kBlock, dyn);
    const int grid = (int)std::max(1LL, std::min((long long)n_sm * std::max(occ, 1), n_tiles));
    if (prm->geometry == ATB_GEOM_BINNED)
        search_kernel<ATB_GEOM_BINNED, kBlock, kMinBlocks><<<grid, kBlock, dyn, s>>>(qa);
    else
        search_kernel<ATB_GEOM_FIXED, kBlock, kMinBlocks><<<grid, kBlock, dyn, s>>>(qa);
    if (best_index)
        best_kernel<<<1, 32, 0, s>>>(1, m->per_cnt, m->out_beg, power, nullptr, best_index);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return static_fail(err, err_len, ATB_ECUDA, "launch: %s", cudaGetErrorString(e));
    int status = 0;
    e = cudaMemcpyAsync(&status, &m->status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return static_fail(err, err_len, ATB_ECUDA, "search: %s", cudaGetErrorString(e));
    if (status & 1)
        return static_fail(err, err_len, ATB_EDATA, "input contains non-finite values or weights <= 0");
    if (status & 2)
        return static_fail(err, err_len, ATB_EDATA, "durations must be positive and finite");
    if (status & 4)
        return static_fail(err, err_len, ATB_EDATA, "periods must be positive and finite");
    return ATB_OK;
}
