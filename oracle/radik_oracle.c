/*
 * radik_oracle.c -- CPU restatement of RadiK.jl's exact Float32 radix top-k.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * engine in radik.jl_b200/csrc.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it; the product path never does.
 *
 * Every function cites the reference file:line it restates (paths are relative
 * to the RadiK.jl project root).  The reference is Julia (KernelAbstractions
 * kernels JIT-compiled by CUDA.jl); no Julia toolchain exists on this machine,
 * so the reference cannot be executed here.  Parity of this restatement is
 * pinned against the known-answer tests in the reference's test/ directory,
 * transcribed into tests/golden/reference_known_answers.json.
 *
 * Stage primitives (ro_count_bin_ex, ro_count_bin, ro_select_bin,
 * ro_select_candidate*, ro_filter) reproduce the reference kernels' semantics
 * literally, including their quirks (NaN skipped by the pass-1 histogram,
 * float compares in the filter).  The full pipeline ro_topk follows the
 * reference orchestrator's pass structure with three documented changes that
 * only matter where the reference result is ill-defined:
 *   1. NaN is the substitute value (floatmin when selecting the largest,
 *      floatmax when selecting the smallest) in EVERY pass, histogram included
 *      (reference: skipped in count_bin.jl:110-116 but substituted in
 *      select_candidate.jl:308 and filter.jl:336, which can overrun outputs);
 *   2. the final filter compares order-preserving keys, not floats, so -0 < +0
 *      as in Julia's isless/partialsort used by test/test_algorithm.jl:18
 *      (reference filter.jl:111,115 compares floats, letting -0 and +0 compete
 *      for the same tie slots);
 *   3. ties at the k-th key are resolved by ascending position inside the task
 *      (reference filter.jl:115-118 takes whichever tied elements win an atomic
 *      race; lowest-position is one of its possible outcomes), and the output
 *      sort breaks value ties by ascending position.
 * Tasks shorter than k keep their values sorted in the first len slots and are
 * padded with value 0 / index -1 afterwards (algorithm.jl:358-365 states this
 * intent; its code pads after sorting stale slots).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

/* ------------------------------------------------------------------------ */
/* L1 utilities                                                              */
/* ------------------------------------------------------------------------ */

/* Order-preserving uint32 key of a Float32: src/utils.jl:29-33
 *   mask = ((~(bits >> 31)) + 1) | 0x80000000 ; key = bits ^ mask          */
uint32_t ro_key(float v) {
    uint32_t b = f2u(v);
    uint32_t mask = ((~(b >> 31)) + 1u) | 0x80000000u;
    return b ^ mask;
}

/* Digit of the key: (key << LEFT) >> RIGHT, src/utils.jl:29-33 */
uint32_t ro_get_bin_id(float v, int left, int right) {
    return (uint32_t)(ro_key(v) << left) >> right;
}

/* src/utils.jl:62-66: first element of the task, 0 when NaN/Inf or disabled */
float ro_sample_scaler(const float* data, int64_t pos, int withscale) {
    if (!withscale) return 0.0f;
    float s = data[pos];
    return (isnan(s) || isinf(s)) ? 0.0f : s;
}

/* src/utils.jl:68-71: NaN -> floatmin (largest) / floatmax (smallest), then
 * optional subtraction of the scaler (IEEE round-to-nearest, no contraction). */
float ro_apply_scaling(float v, float scaler, int withscale, int largest) {
    volatile float p = isnan(v) ? (largest ? FLT_MIN : FLT_MAX) : v;
    if (!withscale) return p;
    volatile float r = p - scaler;
    return r;
}

/* ------------------------------------------------------------------------ */
/* Stage primitives (literal reference semantics)                            */
/* ------------------------------------------------------------------------ */

/* count_bin_ex_kernel!, src/kernels/count_bin.jl:78-203: per-task histogram
 * of get_bin_id(apply_scaling(v)) over task_offsets; NaN inputs skipped
 * (:111).  hist is [T][hist_len] and is overwritten.                        */
void ro_count_bin_ex(const float* data, const int64_t* off, int64_t T, int left,
                     int right, int64_t hist_len, int withscale, int largest,
                     int32_t* hist) {
    for (int64_t t = 0; t < T; ++t) {
        int32_t* h = hist + t * hist_len;
        memset(h, 0, sizeof(int32_t) * (size_t)hist_len);
        int64_t a = off[t], b = off[t + 1];
        if (b <= a) continue;
        float sc = ro_sample_scaler(data, a, withscale);
        for (int64_t i = a; i < b; ++i) {
            float v = data[i];
            if (isnan(v)) continue;
            float s = ro_apply_scaling(v, sc, withscale, largest);
            h[ro_get_bin_id(s, left, right)] += 1;
        }
    }
}

/* count_bin_kernel!, src/kernels/count_bin.jl:20-59: padded layout
 * data[t*stride + i], i < task_lens[t]; no NaN skip, no scaling.            */
void ro_count_bin(const float* data, const int32_t* task_lens, int64_t stride,
                  int64_t T, int left, int right, int64_t hist_len,
                  int32_t* hist) {
    for (int64_t t = 0; t < T; ++t) {
        int32_t* h = hist + t * hist_len;
        memset(h, 0, sizeof(int32_t) * (size_t)hist_len);
        for (int64_t i = 0; i < task_lens[t]; ++i)
            h[ro_get_bin_id(data[t * stride + i], left, right)] += 1;
    }
}

/* select_bin_kernel! + find_bin_and_write!, src/kernels/select_bin.jl:125-159,
 * 268-348.  For each task find the (non-empty) bin b holding rank k counted
 * from the top bin (largest) or from bin 0 (smallest):
 *   before(b) < k <= before(b) + hist[b]
 * and write bin_ids[t] = b + 1 (1-based), k_values[t] = k - before(b),
 * counts[t] = hist[b].  Nothing is written when k is not in (0, total].     */
void ro_select_bin(const int32_t* hist, int64_t T, int64_t hist_len, int largest,
                   int32_t* bin_ids, int32_t* k_values, int32_t* counts) {
    for (int64_t t = 0; t < T; ++t) {
        const int32_t* h = hist + t * hist_len;
        int64_t k = k_values[t];
        int64_t before = 0;
        for (int64_t j = 0; j < hist_len; ++j) {
            int64_t b = largest ? (hist_len - 1 - j) : j;
            int64_t c = h[b];
            if (c > 0 && before < k && k <= before + c) {
                bin_ids[t] = (int32_t)(b + 1);
                k_values[t] = (int32_t)(k - before);
                counts[t] = (int32_t)c;
                break;
            }
            before += c;
        }
    }
}

/* select_candidate_kernel!, src/kernels/select_candidate.jl:67-137: copy the
 * values of task t (padded layout) whose 1-based bin equals bin_ids[t] into
 * out[t*stride ...] in position order; counts[t] receives the number copied. */
void ro_select_candidate(const float* data, const int32_t* task_lens, int64_t stride,
                         int64_t T, const int32_t* bin_ids, int left, int right,
                         float* out, int32_t* counts) {
    for (int64_t t = 0; t < T; ++t) {
        int32_t c = 0;
        for (int64_t i = 0; i < task_lens[t]; ++i) {
            float v = data[t * stride + i];
            if ((int64_t)ro_get_bin_id(v, left, right) + 1 == bin_ids[t])
                out[t * stride + c++] = v;
        }
        counts[t] = c;
    }
}

/* select_candidate_ex_kernel!, src/kernels/select_candidate.jl:233-375: same
 * over task_offsets, on scaled values (NaN substituted, :308).  Output row t
 * starts at out[t*stride].                                                   */
void ro_select_candidate_ex(const float* data, const int64_t* off, int64_t T,
                            const int32_t* bin_ids, int left, int right,
                            int withscale, int largest, int64_t stride,
                            float* out, int32_t* counts) {
    for (int64_t t = 0; t < T; ++t) {
        int32_t c = 0;
        int64_t a = off[t], b = off[t + 1];
        float sc = b > a ? ro_sample_scaler(data, a, withscale) : 0.0f;
        for (int64_t i = a; i < b; ++i) {
            float s = ro_apply_scaling(data[i], sc, withscale, largest);
            if ((int64_t)ro_get_bin_id(s, left, right) + 1 == bin_ids[t])
                out[t * stride + c++] = s;
        }
        counts[t] = c;
    }
}

static inline int64_t read_idx(const void* p, int bytes, int64_t i) {
    if (bytes == 8) return ((const int64_t*)p)[i];
    return ((const int32_t*)p)[i];
}
static inline void write_idx(void* p, int bytes, int64_t i, int64_t v) {
    if (bytes == 8) ((int64_t*)p)[i] = v;
    else ((int32_t*)p)[i] = (int32_t)v;
}

/* filter_kernel! / filter_general_kernel!, src/kernels/filter.jl:106-139,
 * 172-380, 397-621.  Per task: len <= k copies everything (:272-322);
 * otherwise emits (v, idx) when the scaled value is strictly better than
 * kth[t] (float compare, :111) and, for scaled == kth[t], while the boundary
 * counter stays >= 0 after decrement (:115-118).  idx = 1-based position in
 * the task (:76-77, :85-86) or idx_in[global position].  Emission order is
 * position order.  counts[t] receives the number emitted; out rows have
 * stride out_stride (>= max(k, len) so that the reference's possible overrun
 * stays visible).  boundary is updated in place like the reference's counter. */
void ro_filter(const float* data, const int64_t* off, int64_t T, const float* kth,
               int32_t* boundary, int64_t k, int64_t out_stride, int withscale, int largest,
               const void* idx_in, int idx_in_bytes, float* val_out, void* idx_out,
               int idx_out_bytes, int32_t* counts) {
    for (int64_t t = 0; t < T; ++t) {
        int64_t a = off[t], b = off[t + 1], len = b - a, c = 0;
        for (int64_t i = a; i < b; ++i) {
            float v = data[i];
            int emit = 0;
            if (len <= k) {
                emit = 1;
            } else {
                float sc = ro_sample_scaler(data, a, withscale);
                float s = ro_apply_scaling(v, sc, withscale, largest);
                if ((largest && s > kth[t]) || (!largest && s < kth[t])) emit = 1;
                if (s == kth[t]) {
                    boundary[t] -= 1;
                    if (boundary[t] > -1) emit = 1;
                }
            }
            if (emit) {
                int64_t idx = idx_in_bytes ? read_idx(idx_in, idx_in_bytes, i) : (i - a + 1);
                val_out[t * out_stride + c] = v;
                write_idx(idx_out, idx_out_bytes, t * out_stride + c, idx);
                ++c;
            }
        }
        counts[t] = (int32_t)c;
    }
}

/* ------------------------------------------------------------------------ */
/* Full pipeline: topk_radix_select!, src/algorithm.jl:162-368               */
/* ------------------------------------------------------------------------ */

typedef struct { uint32_t key; uint32_t pos; } ro_item;

/* Rank-k bin search of select_bin.jl:125-159 over a histogram of `bins`. */
static int64_t find_bin(const int64_t* h, int64_t bins, int largest, int64_t* k,
                        int64_t* cnt) {
    int64_t before = 0;
    for (int64_t j = 0; j < bins; ++j) {
        int64_t b = largest ? (bins - 1 - j) : j;
        if (h[b] > 0 && before < *k && *k <= before + h[b]) {
            *k -= before;
            *cnt = h[b];
            return b;
        }
        before += h[b];
    }
    return -1;
}

static int cmp_u64(const void* a, const void* b) {
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* One task.  Returns 0, or -1 on allocation failure. */
static int topk_one(const float* data, int64_t a, int64_t n, int64_t k, int largest,
                    int ascend, int withscale, const void* idx_in, int idx_in_bytes,
                    float* vo, void* io, int io_bytes, int64_t orow) {
    uint32_t* win = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n < k ? (n > 0 ? n : 1) : k));
    if (!win) return -1;
    int64_t nw = 0;

    if (n <= k) {
        /* filter.jl:272-322: copy all */
        for (int64_t i = 0; i < n; ++i) win[nw++] = (uint32_t)i;
    } else {
        float sc = ro_sample_scaler(data, a, withscale);
        ro_item* cand = (ro_item*)malloc(sizeof(ro_item) * (size_t)n);
        ro_item* next = (ro_item*)malloc(sizeof(ro_item) * (size_t)n);
        int64_t* h = (int64_t*)malloc(sizeof(int64_t) * 4096);
        if (!cand || !next || !h) { free(cand); free(next); free(h); free(win); return -1; }
        for (int64_t i = 0; i < n; ++i) {
            cand[i].key = ro_key(ro_apply_scaling(data[a + i], sc, withscale, largest));
            cand[i].pos = (uint32_t)i;
        }
        /* Three passes of 12/12/8 key bits: algorithm.jl:214-299.  Each pass:
         * histogram (count_bin), rank search (select_bin), compaction of the
         * selected bin (select_candidate).  Pass p+1 runs only while the
         * selected bin still holds more than one element (:247, :279).     */
        static const int L[3] = {0, 12, 24}, R[3] = {20, 20, 24};
        int64_t ncand = n, kk = k;
        uint32_t kth = 0;
        for (int p = 0; p < 3; ++p) {
            int64_t bins = (int64_t)1 << (32 - R[p]);
            memset(h, 0, sizeof(int64_t) * (size_t)bins);
            for (int64_t i = 0; i < ncand; ++i)
                h[(uint32_t)(cand[i].key << L[p]) >> R[p]] += 1;
            int64_t cnt = 0;
            int64_t b = find_bin(h, bins, largest, &kk, &cnt);
            int64_t m = 0;
            for (int64_t i = 0; i < ncand; ++i)
                if ((int64_t)((uint32_t)(cand[i].key << L[p]) >> R[p]) == b) next[m++] = cand[i];
            ro_item* tmp = cand; cand = next; next = tmp;
            ncand = m;
            kth = cand[0].key;
            if (ncand <= 1) break;
        }
        /* Final filter (filter.jl:106-139) on keys: strictly better than the
         * k-th key, then kk ties in ascending position.                     */
        int64_t ties = kk;
        for (int64_t i = 0; i < n; ++i) {
            uint32_t key = ro_key(ro_apply_scaling(data[a + i], sc, withscale, largest));
            int better = largest ? (key > kth) : (key < kth);
            if (better) win[nw++] = (uint32_t)i;
            else if (key == kth && ties > 0) { win[nw++] = (uint32_t)i; --ties; }
        }
        free(cand); free(next); free(h);
    }

    /* Final sort (algorithm.jl:340-352): by the key of the (NaN-substituted)
     * original value, ascending when ASCEND else descending; equal keys by
     * ascending position. */
    uint64_t* s = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(nw > 0 ? nw : 1));
    if (!s) { free(win); return -1; }
    for (int64_t j = 0; j < nw; ++j) {
        float v = data[a + win[j]];
        uint32_t ok = ro_key(ro_apply_scaling(v, 0.0f, 0, largest));
        if (!ascend) ok = ~ok;
        s[j] = ((uint64_t)ok << 32) | win[j];
    }
    qsort(s, (size_t)nw, sizeof(uint64_t), cmp_u64);
    for (int64_t j = 0; j < k; ++j) {
        if (j < nw) {
            int64_t pos = (int64_t)(uint32_t)s[j];
            vo[orow + j] = data[a + pos];
            int64_t idx = idx_in_bytes ? read_idx(idx_in, idx_in_bytes, a + pos) : pos + 1;
            write_idx(io, io_bytes, orow + j, idx);
        } else {
            /* algorithm.jl:358-365 */
            vo[orow + j] = 0.0f;
            write_idx(io, io_bytes, orow + j, -1);
        }
    }
    free(s);
    free(win);
    return 0;
}

/* Batched exact top-k.  off has T+1 entries (0-based prefix sums).  Output
 * rows have stride k (column-major [k, T] as in the Julia API).  Tasks run in
 * parallel on `threads` OpenMP threads (<= 0: all available).  Returns 0 on
 * success, -1 on allocation failure, -2 on invalid arguments. */
int ro_topk(const float* data, const int64_t* off, int64_t T, int64_t k, int largest,
            int ascend, int withscale, const void* idx_in, int idx_in_bytes,
            float* val_out, void* idx_out, int idx_out_bytes, int threads) {
    if (T < 0 || k < 0 || (idx_out_bytes != 4 && idx_out_bytes != 8)) return -2;
    if (idx_in_bytes != 0 && idx_in_bytes != 4 && idx_in_bytes != 8) return -2;
    int err = 0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads) reduction(| : err)
#endif
    for (int64_t t = 0; t < T; ++t) {
        int64_t a = off[t], n = off[t + 1] - off[t];
        if (k == 0) continue;
        if (topk_one(data, a, n, k, largest, ascend, withscale, idx_in, idx_in_bytes,
                     val_out, idx_out, idx_out_bytes, t * k) != 0)
            err |= 1;
    }
    return err ? -1 : 0;
}

int ro_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
