// fused.cuh -- single-read exact top-k for k up to a few thousand.
//
// One persistent kernel replaces the reference's whole per-call pipeline
// (src/algorithm.jl:214-365: count_bin_ex -> select_bin -> select_candidate_ex
// -> passes 2/3 -> filter -> sort -> pad, three full reads of the input).
//
// Work items are segments of tasks (a task shorter than the segment size is
// one segment), handed out through an atomic queue in the order the plan
// chose (longest first).  A CTA streams its segment once from HBM with
// 128-bit loads and keeps, in a shared-memory buffer, every element whose
// composite (score << 32 | ~pos, see common.cuh) beats the current threshold.
// When the buffer fills up, block_shrink (the histogram / rank search /
// narrowing cycle of count_bin.jl, select_bin.jl and select_candidate.jl on
// on-chip data) keeps a few more than the k best and raises the threshold to
// the lower edge of what it kept.  Segments of one task share a global
// threshold (atomicMax of the segments' thresholds, each a valid lower bound
// of the task's k-th composite).  For tasks split into many segments with a
// large k, a sampling kernel seeds that threshold from a sample of the task
// (sample.cuh); if the seeded threshold turns out too high (fewer than k
// elements above it), the task is flagged and a retry launch recomputes it
// from scratch, so results never depend on the sample.
// A single-segment task is finished by its CTA; for a multi-segment task every
// segment appends its surviving top-k to the task's candidate region and the
// last segment to finish (atomic counter, no waiting) merges them.
// Finishing = exact top-k, gather of the original values, sort (bitonic for
// <= 4096 entries, radix sort above), index mapping and padding.
//
// Each task carries its own k and flags (largest / ascend), and optionally its
// own input and output pointers, so one launch can serve a batch assembled
// from independent requests.
#pragma once

#include "block_ops.cuh"
#include "tma.cuh"

namespace radik {

// kTaskFlush: a sampled task split into segments whose candidates go straight
// to its candidate region (no per-segment selection); the merge kernel
// (merge.cuh) finishes it.
// kTaskDefer: a single-segment task whose streaming block leaves its
// candidates in the task's region (p.cap entries) and queues it, so that the
// block moves on to its next task at once; blocks with no streaming left
// finish queued tasks (fused_ws.cuh).
// kTaskFinishHere: a flush-mode task with a small k that the block flushing
// its last segment finishes (no merge kernel).
enum : uint32_t {
    kTaskLargest = 1u, kTaskAscend = 2u, kTaskSampled = 4u, kTaskFlush = 8u, kTaskDefer = 16u, kTaskFinishHere = 32u
};

struct FusedTask {
    int64_t start;   // global offset of the task in p.data (uniform-input mode)
    int64_t len;     // elements
    int64_t cbase;   // first entry of the task's candidate region (multi-segment tasks), else -1
    int32_t nseg;
    uint32_t k;      // results wanted for this task (<= FusedParams::kmax)
    uint32_t flags;  // kTaskLargest | kTaskAscend | kTaskSampled
    uint32_t pad_;
};

// Per-task pointers (request-batching mode); row outputs hold k entries.
struct FusedTaskIO {
    const float* data;
    float* val_out;
    void* idx_out;
    const void* idx_in;  // nullable, indexed by position inside the task
};

struct FusedSeg {
    int32_t pos;         // position (inside the task) of the segment's first element
    int32_t len;
    int32_t task;
    int32_t seg_in_task;
};

struct FusedParams {
    const float* data;       // uniform-input mode: concatenated tasks
    const FusedTask* tasks;
    const FusedSeg* segs;
    const FusedTaskIO* task_io;  // nullable: per-task pointers instead of data/val_out/...
    int32_t nsegs;
    uint32_t kmax;           // largest k of the launch
    uint32_t cap;            // shared buffer capacity in composites
    int retry;               // retry launch: only tasks flagged in `fail` run
    const void* idx_in;      // uniform mode, nullable: custom indices (idx_bytes wide)
    int idx_bytes;           // width of idx_out (and idx_in when present)
    float* val_out;          // uniform mode: [T][k]
    void* idx_out;           // uniform mode: [T][k]
    // workspace
    uint64_t* gthr;          // [T] exclusive thresholds (keep c > gthr)
    uint32_t* task_done;     // [T] finished segments
    uint32_t* task_cnt;      // [T] entries in the candidate region
    uint32_t* fail;          // [T] seeded threshold too high
    uint32_t* fail_any;      // [1] some task is flagged in `fail` (the retry launch exits at once otherwise)
    uint32_t sample_max;     // warp-specialised kernel: most elements of a single-segment task's sample
    uint32_t* work_counter;  // [1]
    uint64_t* cand;          // candidate regions
    uint64_t* sort_scratch;  // [gridDim.x * kmax] (kmax > 4096 only)
    uint32_t* rank_ready;    // [T] merge kernel left the k output keys for rank_write_kernel (nullable)
    uint32_t* defer_ctr;     // [2] deferred tasks queued / claimed by finishers
    uint32_t* defer_q;       // [ndefer] queued task + 1 (0: not yet); nullable: no deferral
    uint32_t ndefer;         // deferred tasks of the launch
    uint32_t* err;
};

constexpr uint32_t kBitonicMax = 4096;

__device__ __forceinline__ uint64_t load_volatile_u64(const uint64_t* p) {
    return *reinterpret_cast<const volatile uint64_t*>(p);
}

// Everything the kernel needs to know about one task.
struct TaskView {
    const float* data;
    float* vout;
    void* iout;
    const void* iin;
    int64_t len;
    uint32_t k;
    bool ascend;
    ScoreParams sp;
};

template <bool kScale>
__device__ __forceinline__ TaskView task_view(const FusedParams& p, int t, const FusedTask& td) {
    TaskView v;
    if (p.task_io) {
        const FusedTaskIO io = p.task_io[t];
        v.data = io.data;
        v.vout = io.val_out;
        v.iout = io.idx_out;
        v.iin = io.idx_in;
    } else {
        v.data = p.data + td.start;
        v.vout = p.val_out + static_cast<int64_t>(t) * td.k;
        v.iout = static_cast<char*>(p.idx_out) + static_cast<int64_t>(t) * td.k * p.idx_bytes;
        v.iin = p.idx_in ? static_cast<const char*>(p.idx_in) + td.start * p.idx_bytes : nullptr;
    }
    v.len = td.len;
    v.k = td.k;
    v.ascend = (td.flags & kTaskAscend) != 0;
    v.sp = make_score_params((td.flags & kTaskLargest) != 0, kScale);
    return v;
}

template <int THREADS>
struct FusedShared {
    BlockScratch<THREADS> bs;
    uint32_t cnt;
    int32_t work;
    uint32_t last;
    uint32_t base;
    uint32_t abort;  // a bounded wait gave up: the CTA stops
    uint32_t pad2_;
    uint32_t wc[THREADS / 32];  // per-warp region counts while gathering
    uint64_t gthr;
};


// Appends composite c (when pass) to the shared buffer with one shared atomic
// per warp (warp-aggregated).  All lanes of the warp must call.
__device__ __forceinline__ void warp_append(bool pass, uint64_t c, uint64_t* buf, uint32_t* cnt, uint32_t cap,
                                            uint32_t* err) {
    uint32_t m = __ballot_sync(kFullMask, pass);
    if (m == 0) return;
    const uint32_t lane = lane_id();
    const uint32_t leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(cnt, __popc(m));
    base = __shfl_sync(kFullMask, base, leader);
    if (pass) {
        uint32_t i = base + __popc(m & lanemask_lt());
        if (i < cap) buf[i] = c;
        else record_error(err, kErrCapacity);
    }
}

// Reserves room for n entries per lane (one shared atomic per warp) and
// returns this lane's first slot.  All lanes of the warp must call; the warp
// total must be non-zero.
__device__ __forceinline__ uint32_t warp_reserve(uint32_t n, uint32_t* cnt) {
    const uint32_t incl = warp_inclusive_scan<true>(n);
    const uint32_t total = __shfl_sync(kFullMask, incl, 31);
    uint32_t base = 0;
    if (lane_id() == 31) base = atomicAdd(cnt, total);
    base = __shfl_sync(kFullMask, base, 31);
    return base + incl - n;
}

// Write a task's output row from its m sorted output keys (low 32 bits =
// position): value, index (automatic 1-based or custom), padding.
template <int THREADS, bool kFromKey = false>
__device__ void write_row(const FusedParams& p, const TaskView& tv, const uint64_t* sorted, uint32_t m) {
    const int tid = threadIdx.x;
    const uint32_t nan_key = key_of_bits(tv.sp.nan_bits);
    for (uint32_t j = tid; j < tv.k; j += THREADS) {
        float v = 0.0f;
        int64_t idx = -1;
        if (j < m) {
            uint32_t pos = static_cast<uint32_t>(sorted[j]);
            if (pos >= static_cast<uint64_t>(tv.len)) pos = 0;  // bounded gather (error recorded earlier)
            if constexpr (kFromKey) {
                // The value is the key's preimage unless the key is the NaN
                // substitute's (then the element may be a NaN: read it).
                uint32_t key = static_cast<uint32_t>(sorted[j] >> 32);
                if (!tv.ascend) key = ~key;
                v = (key == nan_key) ? tv.data[pos] : __uint_as_float((key & 0x80000000u) ? (key ^ 0x80000000u) : ~key);
            } else {
                v = tv.data[pos];
            }
            if (tv.iin) {
                idx = (p.idx_bytes == 8) ? static_cast<const int64_t*>(tv.iin)[pos]
                                         : static_cast<int64_t>(static_cast<const int32_t*>(tv.iin)[pos]);
            } else {
                idx = static_cast<int64_t>(pos) + 1;  // 1-based position (filter.jl:76-77)
            }
        }
        tv.vout[j] = v;
        if (p.idx_bytes == 8) static_cast<int64_t*>(tv.iout)[j] = idx;
        else static_cast<int32_t*>(tv.iout)[j] = static_cast<int32_t>(idx);
    }
    block_sync<THREADS>();
}

// Sort the m finished composites of a task by the output order, map indices
// and write the task's output row (padding slots m..k-1 with 0 / -1,
// src/algorithm.jl:358-365).  buf has room for next_pow2(m) <= cap entries
// and, past m, for the radix sort's shared counters.
template <int THREADS, bool kFromScore = false>
__device__ void finish_task(const FusedParams& p, const TaskView& tv, uint64_t* buf, uint32_t m,
                            FusedShared<THREADS>& sh) {
    const int tid = threadIdx.x;
    for (uint32_t i = tid; i < m; i += THREADS) {
        const uint64_t c = buf[i];
        uint32_t pos = composite_pos(c);
        if (pos >= static_cast<uint64_t>(tv.len)) {  // never expected; keep the gather in bounds
            record_error(p.err, kErrBounds);
            pos = 0;
        }
        if constexpr (kFromScore) {
            // Unscaled scores are the keys of the NaN-substituted values.
            uint32_t key = static_cast<uint32_t>(c >> 32) ^ tv.sp.flip;
            if (!tv.ascend) key = ~key;
            buf[i] = (static_cast<uint64_t>(key) << 32) | pos;
        } else {
            uint32_t bits = __float_as_uint(tv.data[pos]);
            buf[i] = output_sort_key(bits, pos, tv.sp, tv.ascend);
        }
    }
    block_sync<THREADS>();
    uint64_t* sorted = buf;
    // Scratch past the entries for the register sorts: their n <= 8 THREADS
    // keys need 2 n slots after buf[0, n).
    if (m <= static_cast<uint32_t>(THREADS) && p.cap >= 2u * THREADS) {
        small_sort_u64<THREADS>(buf, m, buf + THREADS);
    } else if (m <= 2u * THREADS && p.cap >= 6u * THREADS) {
        regs_sort_u64<THREADS, 2>(buf, m, buf + 2 * THREADS);
    } else if (m <= 4u * THREADS && p.cap >= 12u * THREADS) {
        regs_sort_u64<THREADS, 4>(buf, m, buf + 4 * THREADS);
    } else if (m <= 8u * THREADS && p.cap >= 24u * THREADS) {
        regs_sort_u64<THREADS, 8>(buf, m, buf + 8 * THREADS);
    } else if (m <= kBitonicMax) {
        uint32_t P = 1;
        while (P < m) P <<= 1;
        for (uint32_t i = m + tid; i < P; i += THREADS) buf[i] = ~0ull;
        block_sync<THREADS>();
        bitonic_sort_u64<THREADS>(buf, P);
    } else {
        // Digit counters behind the keys; the second key buffer in shared
        // memory too when the buffer holds it (the merge kernel's does),
        // else the block's slice of the global sort scratch.
        uint32_t* wd = reinterpret_cast<uint32_t*>(buf + m);
        uint32_t* db = wd + (THREADS / 32) * 256;
        const size_t soff = (static_cast<size_t>(m) + ((THREADS / 32) * 256 + 256) / 2 + 2) & ~size_t(1);
        uint64_t* scratch = (soff + m <= p.cap) ? buf + soff
                                                : p.sort_scratch + static_cast<int64_t>(blockIdx.x) * p.kmax;
        sorted = radix_sort_u64<THREADS>(buf, scratch, m, sh.bs, wd, db);
    }
    block_sync<THREADS>();
    write_row<THREADS, kFromScore>(p, tv, sorted, m);
}

// Bucket finish (finish_by_buckets): largest k, and largest bin whose
// entries it orders by scanning the bin.
constexpr uint32_t kBucketMaxK = 512;
constexpr uint32_t kBucketScanMax = 64;

// Output row of a single-segment task from its candidates buf[0, cnt) (unique
// composites), with one histogram pass and no sorting network:
//   1. the candidates are counted in 256 bins of the (up to) 8 score bits
//      below their common prefix (bins follow the composite order and keep
//      equal scores together);
//   2. warp 0 scans the bins from the top: the bin b* holding rank
//      m = min(cnt, want), the entries above each bin (its bucket offset in
//      composite order) and how many of b*'s entries are in (need);
//   3. the entries of bins >= b* are scattered to their buckets;
//   4. an entry's rank inside its bin (by composite, then by output order)
//      comes from a scan of its bin's few entries; b*'s entries are in when
//      their rank is below need.  The row position follows: bins are in score
//      order, so a descending row (largest, !ascend / smallest, ascend) is the
//      composite order itself, and an ascending-score row is the bins in
//      reverse with each bin's entries by ascending (score, position).
// Returns false, having written nothing, when a bin at or above b* holds more
// than kBucketScanMax entries (many ties or clustered values) or the scratch
// behind the candidates is too small; the caller then finishes by radix
// selection.  Unscaled scores only (a value is its key's preimage; the element
// itself where the key is the NaN substitute's).  Slots m..k-1 are padded
// with 0 / -1 (src/algorithm.jl:358-365).  All threads must call.
template <int THREADS>
__device__ bool finish_by_buckets(const FusedParams& p, const TaskView& tv, uint64_t* buf, uint32_t cnt, uint32_t want,
                                  FusedShared<THREADS>& sh) {
    constexpr int NW = THREADS / 32;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t m = cnt < want ? cnt : want;
    // Scratch behind the candidates: the buckets, then bucket offsets and
    // scatter cursors (256 words each).
    const uint32_t boff = (cnt + 1u) & ~1u;
    const uint32_t words_off = boff + m + kBucketScanMax;
    if (static_cast<size_t>(words_off) + 256u > p.cap) return false;  // uniform: no barrier taken yet
    uint64_t* bucket = buf + boff;
    uint32_t* off = reinterpret_cast<uint32_t*>(buf + words_off);
    uint32_t* cur = off + 256;
    uint32_t* hist = sh.bs.hist;

    // OR and AND of the high and low words (one warp reduction each); the
    // bins and cursors are cleared before the same barrier.
    {
        uint32_t hor = 0u, hand = ~0u, lor = 0u, land = ~0u;
#pragma unroll 1
        for (uint32_t i = tid; i < cnt; i += THREADS) {
            const uint64_t c = buf[i];
            hor |= static_cast<uint32_t>(c >> 32);
            hand &= static_cast<uint32_t>(c >> 32);
            lor |= static_cast<uint32_t>(c);
            land &= static_cast<uint32_t>(c);
        }
        hor = __reduce_or_sync(kFullMask, hor);
        hand = __reduce_and_sync(kFullMask, hand);
        lor = __reduce_or_sync(kFullMask, lor);
        land = __reduce_and_sync(kFullMask, land);
        if (lane == 0) {
            sh.bs.warp_a[warp] = (static_cast<uint64_t>(hor) << 32) | lor;
            sh.bs.warp_b[warp] = (static_cast<uint64_t>(hand) << 32) | land;
        }
        for (uint32_t b = tid; b < 256u; b += THREADS) {
            hist[b] = 0;
            cur[b] = 0;
        }
    }
    block_sync<THREADS>();
    uint64_t vor = 0, vand = ~0ull;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        vor |= sh.bs.warp_a[w];
        vand &= sh.bs.warp_b[w];
    }
    const uint64_t diff = vor ^ vand;
    const int top = diff ? 63 - __clzll(static_cast<long long>(diff)) : 0;
    // Bins cut the scores only (a run of equal scores stays in one bin) unless
    // every candidate has the same score; then they cut the positions, and
    // either row order is the composite order (ascending positions).
    const bool one_score = top < 32;
    const int w = one_score ? (top + 1 < 8 ? top + 1 : 8) : (top - 31 < 8 ? top - 31 : 8);
    const int shift = top + 1 - w;
    const uint32_t nb = 1u << w, bmask = nb - 1u;
#pragma unroll 1
    for (uint32_t i = tid; i < cnt; i += THREADS) atomicAdd(hist + (static_cast<uint32_t>(buf[i] >> shift) & bmask), 1u);
    block_sync<THREADS>();
    if (warp == 0) {
        // Bins from the top: lane l takes bins nb-1-8l ... nb-8-8l (all
        // loads at once; bins past nb count 0).
        uint32_t h[8], sum = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t rb = lane * 8u + static_cast<uint32_t>(j);
            h[j] = rb < nb ? hist[nb - 1u - rb] : 0u;
            sum += h[j];
        }
        const uint32_t incl = warp_inclusive_scan<true>(sum);
        uint32_t run = incl - sum;  // entries in the bins above this lane's
        uint32_t bstar = 0xffffffffu, need = 0, big = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t rb = lane * 8u + static_cast<uint32_t>(j);
            if (rb < nb) {
                const uint32_t b = nb - 1u - rb;
                off[b] = run;
                if (run < m) {  // a bin that holds some of the m best
                    big = h[j] > big ? h[j] : big;
                    if (run + h[j] >= m) {
                        bstar = b;
                        need = m - run;
                    }
                }
            }
            run += h[j];
        }
        big = __reduce_max_sync(kFullMask, big);
        const uint32_t who = __ballot_sync(kFullMask, bstar != 0xffffffffu);
        if (who != 0u) {
            const uint32_t src = __ffs(who) - 1u;
            bstar = __shfl_sync(kFullMask, bstar, src);
            need = __shfl_sync(kFullMask, need, src);
        }
        if (lane == 0) {
            sh.bs.bc32[0] = bstar;  // 0xffffffff: m == 0
            sh.bs.bc32[1] = need;
            sh.bs.bc32[2] = big > kBucketScanMax ? 1u : 0u;
        }
    }
    block_sync<THREADS>();
    const uint32_t bstar = sh.bs.bc32[0], need = sh.bs.bc32[1];
    if (sh.bs.bc32[2] != 0u) return false;  // uniform; buf[0, cnt) is untouched
    const uint32_t nsel = bstar == 0xffffffffu ? 0u : off[bstar] + hist[bstar];  // entries of bins >= b*
    if (nsel != 0u) {
#pragma unroll 1
        for (uint32_t i = tid; i < cnt; i += THREADS) {
            const uint64_t c = buf[i];
            const uint32_t b = static_cast<uint32_t>(c >> shift) & bmask;
            if (b >= bstar) bucket[off[b] + atomicAdd(cur + b, 1u)] = c;
        }
    }
    block_sync<THREADS>();
    const bool same_order = one_score || (tv.sp.flip == 0u) != tv.ascend;
    const uint32_t nan_key = key_of_bits(tv.sp.nan_bits);
    // Writes the selected entry c to row slot o.
    auto emit = [&](uint64_t c, uint32_t o) {
        uint32_t pos = composite_pos(c);
        if (pos >= static_cast<uint64_t>(tv.len) || o >= m) {  // never expected; keep accesses in bounds
            record_error(p.err, pos >= static_cast<uint64_t>(tv.len) ? kErrBounds : kErrInternal);
            return;
        }
        const uint32_t key = static_cast<uint32_t>(c >> 32) ^ tv.sp.flip;
        const float val = (key == nan_key) ? tv.data[pos] : value_of_key(key);
        int64_t idx;
        if (tv.iin) {
            idx = (p.idx_bytes == 8) ? static_cast<const int64_t*>(tv.iin)[pos]
                                     : static_cast<int64_t>(static_cast<const int32_t*>(tv.iin)[pos]);
        } else {
            idx = static_cast<int64_t>(pos) + 1;  // 1-based position (filter.jl:76-77)
        }
        tv.vout[o] = val;
        if (p.idx_bytes == 8) static_cast<int64_t*>(tv.iout)[o] = idx;
        else static_cast<int32_t*>(tv.iout)[o] = static_cast<int32_t>(idx);
    };
    // Ranks inside the bins by composite (descending).  In composite order
    // (same_order) an entry's row slot is its bin's offset plus that rank and
    // b*'s entries are in when the rank is below need: written at once.
    // Otherwise the need-th of b* is the bound tau of the m best, found first.
    // (Loops kept rolled: this runs once per task and its code is fetched cold.)
#pragma unroll 1
    for (uint32_t s = tid; s < nsel; s += THREADS) {
        const uint64_t c = bucket[s];
        const uint32_t b = static_cast<uint32_t>(c >> shift) & bmask;
        const uint32_t lo = off[b], hi = lo + hist[b];
        uint32_t rd = 0;
#pragma unroll 1
        for (uint32_t j = lo; j < hi; ++j) rd += bucket[j] > c ? 1u : 0u;
        if (same_order) {
            if (b != bstar || rd < need) emit(c, off[b] + rd);
        } else if (b == bstar && rd == need - 1u) {
            sh.gthr = c;
        }
    }
    if (!same_order) {
        block_sync<THREADS>();
        const uint64_t tau = sh.gthr;
#pragma unroll 1
        for (uint32_t s = tid; s < nsel; s += THREADS) {
            const uint64_t c = bucket[s];
            const uint32_t b = static_cast<uint32_t>(c >> shift) & bmask;
            if (b == bstar && c < tau) continue;  // below the m best
            const uint32_t sel_b = b == bstar ? need : hist[b];
            // Ascending scores: the bins below this one come first, then this
            // bin's selected entries by ascending (score, position).
            const uint32_t lo = off[b], hi = lo + hist[b];
            const uint32_t sc = static_cast<uint32_t>(c >> 32), pc = composite_pos(c);
            uint32_t ra = 0;
#pragma unroll 1
            for (uint32_t j = lo; j < hi; ++j) {
                const uint64_t y = bucket[j];
                const uint32_t sy = static_cast<uint32_t>(y >> 32);
                const bool in = b != bstar || y >= tau;
                ra += (in && (sy < sc || (sy == sc && composite_pos(y) < pc))) ? 1u : 0u;
            }
            emit(c, m - off[b] - sel_b + ra);
        }
    }
    if (cnt < want && tid == 0) record_error(p.err, kErrInternal);  // the caller redoes a short count
    for (uint32_t j = m + tid; j < tv.k; j += THREADS) {
        tv.vout[j] = 0.0f;
        if (p.idx_bytes == 8) static_cast<int64_t*>(tv.iout)[j] = -1;
        else static_cast<int32_t*>(tv.iout)[j] = -1;
    }
    block_sync<THREADS>();  // buf and the block scratch are reused by the caller
    return true;
}

// Shared count, clamped to the buffer (appends past cap were dropped and
// recorded); all threads must call.
template <int THREADS>
__device__ __forceinline__ uint32_t buffer_count(const FusedParams& p, FusedShared<THREADS>& sh) {
    uint32_t cnt = sh.cnt;
    if (cnt > p.cap) {
        cnt = p.cap;
        block_sync<THREADS>();
        if (threadIdx.x == 0) sh.cnt = cnt;
        block_sync<THREADS>();
    }
    return cnt;
}

// Mid-stream reduction: keeps between k and max_keep entries, all of them
// >= the returned keep_from (0 when nothing was dropped).
template <int THREADS>
__device__ uint64_t shrink_mid(const FusedParams& p, uint32_t k, uint32_t max_keep, uint64_t* buf,
                               FusedShared<THREADS>& sh) {
    const uint32_t cnt = buffer_count<THREADS>(p, sh);
    uint64_t vor = 0, vand = ~0ull;
    for (uint32_t i = threadIdx.x; i < cnt; i += THREADS) { uint64_t c = buf[i]; vor |= c; vand &= c; }
    block_or_and<THREADS>(vor, vand, sh.bs);
    uint64_t kf = 0, mn = 0;
    const uint32_t kept = block_shrink<THREADS>(buf, cnt, k, max_keep, vand, vor, sh.bs, p.err, &kf, &mn);
    block_sync<THREADS>();
    if (threadIdx.x == 0) sh.cnt = kept;
    block_sync<THREADS>();
    return (kept >= k && kept < cnt) ? kf : 0ull;
}

// Exact reduction of the buffer to its best k (radix selection).  Returns
// the number kept and, through *kth, the k-th composite (0 if fewer than k).
template <int THREADS>
__device__ uint32_t shrink_final(const FusedParams& p, uint32_t k, uint64_t* buf, FusedShared<THREADS>& sh,
                                 uint64_t* kth) {
    const uint32_t cnt = buffer_count<THREADS>(p, sh);
    uint32_t m = block_select_topk<THREADS>(buf, cnt, k, sh.bs, p.err, kth);
    if (m < k) *kth = 0;
    block_sync<THREADS>();
    if (threadIdx.x == 0) sh.cnt = m;
    block_sync<THREADS>();
    return m;
}

// Finishes a single-segment task whose candidates are buf[0, sh.cnt) (a
// superset of its best min(len, k)): for k <= 512 by one histogram pass and
// buckets (finish_by_buckets) when no bin is crowded, else by exact radix
// selection (shrink_final) then finish_task.  All threads must call.
template <int THREADS, bool kScale>
__device__ void finish_candidates(const FusedParams& p, const TaskView& tv, uint64_t* buf, FusedShared<THREADS>& sh) {
    const uint32_t k = tv.k;
    const uint32_t want = tv.len < static_cast<int64_t>(k) ? static_cast<uint32_t>(tv.len) : k;
    const uint32_t cnt = buffer_count<THREADS>(p, sh);
    if constexpr (!kScale) {
        if (want <= kBucketMaxK && finish_by_buckets<THREADS>(p, tv, buf, cnt, want, sh)) return;
    }
    uint64_t kth = 0;
    const uint32_t m = shrink_final<THREADS>(p, k, buf, sh, &kth);
    if (m != want && threadIdx.x == 0) record_error(p.err, kErrInternal);
    finish_task<THREADS, !kScale>(p, tv, buf, m < want ? m : want, sh);
}

// Starting threshold of a single-segment task from a sample of `S` of its
// elements (16 chunks of S/16 consecutive elements): one below the composite
// of sample rank r.  With lam = k S / len sampled elements expected among the
// task's k best, r = lam + 5 sqrt(lam) + 12 puts the threshold five standard
// deviations of that count below the k-th (too high only with probability
// ~1e-7; the task is then redone without it).  Up to r = S / 2, so a k that
// is a quarter of the row (lam = S / 4) still gets a threshold near the
// sample's 66th percentile instead of none.  0 (no pruning) when the sample
// is too small.
template <int THREADS, bool kScale>
__device__ uint64_t sampled_threshold(const TaskView& tv, float scaler, uint32_t k, uint64_t* buf,
                                      FusedShared<THREADS>& sh, uint32_t* err) {
    constexpr uint32_t S = 1024, CH = S / 16;
    const int64_t len = tv.len;
    if (len < 8 * static_cast<int64_t>(S)) return 0ull;
    const float lam = static_cast<float>(k) * S / static_cast<float>(len);
    const uint32_t r = static_cast<uint32_t>(ceilf(lam + 5.0f * sqrtf(lam) + 12.0f));
    if (r > S / 2) return 0ull;
    const int64_t cstride = len / 16;
    uint64_t vor = 0, vand = ~0ull;
    for (uint32_t i = threadIdx.x; i < S; i += THREADS) {
        const int64_t q = static_cast<int64_t>(i / CH) * cstride + (i % CH);
        const uint32_t bits = __float_as_uint(tv.data[q]);
        const uint64_t c = make_composite(score_of<kScale>(bits, scaler, tv.sp), static_cast<uint32_t>(q));
        buf[i] = c;
        vor |= c;
        vand &= c;
    }
    block_or_and<THREADS>(vor, vand, sh.bs);  // barriers: the sample is in buf
    const uint64_t kf = block_rank_threshold<THREADS>(buf, S, r, 4 * r, vand, vor, sh.bs);
    block_sync<THREADS>();
    return kf > 0 ? kf - 1 : 0ull;
}

// Candidate appends go to one region per warp (kRegionEntries in total, after
// the settled region of the shared buffer) so that a warp counts its own
// entries in a register.  gather_regions moves every warp's entries behind the
// settled ones, leaving the candidates in [0, sh.cnt); all threads must call.
constexpr uint32_t kRegionEntries = 2048;

template <int THREADS, uint32_t R>
__device__ void gather_regions(uint64_t* s_buf, uint32_t cap_s, uint32_t& wcnt, FusedShared<THREADS>& sh) {
    constexpr int NW = THREADS / 32;
    constexpr uint32_t PER = (R + 31) / 32;  // region entries per lane
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t wc = wcnt < R ? wcnt : R;
    if (lane == 0) sh.wc[warp] = wc;
    block_sync<THREADS>();
    uint32_t off = sh.cnt, total = sh.cnt;
#pragma unroll
    for (int i = 0; i < NW; ++i) {
        off += (i < warp) ? sh.wc[i] : 0u;
        total += sh.wc[i];
    }
    // Every warp takes its entries into registers first; a warp's destination
    // may cover another warp's region, so nothing is written before all reads.
    const uint64_t* region = s_buf + cap_s + warp * R;
    uint64_t x[PER];
#pragma unroll
    for (uint32_t j = 0; j < PER; ++j) {
        const uint32_t idx = j * 32 + lane;
        x[j] = idx < wc ? region[idx] : 0ull;
    }
    block_sync<THREADS>();
#pragma unroll
    for (uint32_t j = 0; j < PER; ++j) {
        const uint32_t idx = j * 32 + lane;
        if (idx < wc) s_buf[off + idx] = x[j];
    }
    if (threadIdx.x == 0) sh.cnt = total;
    block_sync<THREADS>();
    wcnt = 0;
}

// Cheap superset test of "composite > thr" on raw float values.  An element
// whose composite exceeds thr has a score >= thr's score; in value terms that
// is x >= t (largest) or x <= t (smallest) for the value t whose key is that
// score, and a float compare accepts at least those values (it only adds
// +-0 ties, which the exact test on candidates settles).  NaN elements score
// as the reference's substitute, so they may pass only when that substitute
// does (nan_pass).  Values are compared sign-flipped for the smallest, so
// one compare covers both directions.
struct FastFilter {
    float t;          // compare x * dir >= t (after the sign flip)
    float tr;         // the same threshold unflipped: x <= tr (smallest)
    uint32_t dir;     // 0 (largest) or 0x80000000 (smallest): sign flip of x
    bool nan_pass;
    float4 pad4;      // value that never passes (fills past the end of a segment)
};

template <bool kScale>
__device__ __forceinline__ FastFilter make_fast_filter(uint64_t thr, const ScoreParams& sp, float scaler) {
    constexpr uint32_t kNegInf = 0x007fffffu, kPosInf = 0xff800000u;  // keys of -inf, +inf
    FastFilter f;
    const uint32_t s = static_cast<uint32_t>(thr >> 32);
    const bool largest = sp.flip == 0;
    f.dir = largest ? 0u : 0x80000000u;
    float t;
    if (largest) {  // pass iff key >= s
        t = (s <= kNegInf) ? -INFINITY : (s > kPosInf ? __uint_as_float(0x7fc00000u) : value_of_key(s));
    } else {        // pass iff key <= ~s
        const uint32_t K = ~s;
        t = (K >= kPosInf) ? INFINITY : (K < kNegInf ? __uint_as_float(0x7fc00000u) : value_of_key(K));
    }
    f.t = __uint_as_float(__float_as_uint(t) ^ f.dir);
    f.tr = t;
    const float never = largest ? -INFINITY : INFINITY;  // fails unless everything passes
    f.pad4 = make_float4(never, never, never, never);
    uint32_t nan_score = sp.nan_score;
    if constexpr (kScale)
        nan_score = key_of_bits(__float_as_uint(__fsub_rn(__uint_as_float(sp.nan_bits), scaler))) ^ sp.flip;
    f.nan_pass = nan_score >= s;
    return f;
}

constexpr uint32_t kWaitPolls = 1u << 22;

// Geometry of one work item, identical in every thread of the CTA.
struct SegGeom {
    FusedSeg sg;
    FusedTask td;
    int64_t s0, s1, a0, a1, nvec;
    uint32_t ntiles;
    bool skip;  // retry launch and the task was not flagged
};

template <int TILE, bool kScale>
__device__ __forceinline__ SegGeom seg_geom(const FusedParams& p, int w, TaskView* tv) {
    SegGeom g;
    g.sg = p.segs[w];
    g.td = p.tasks[g.sg.task];
    g.skip = p.retry && p.fail[g.sg.task] == 0;
    *tv = task_view<kScale>(p, g.sg.task, g.td);
    g.s0 = g.sg.pos;
    g.s1 = static_cast<int64_t>(g.sg.pos) + g.sg.len;
    // Position q sits on a 16-byte boundary iff (q + mis) % 4 == 0.
    const int64_t mis = static_cast<int64_t>((reinterpret_cast<uintptr_t>(tv->data) >> 2) & 3);
    g.a0 = ((g.s0 + mis + 3) & ~int64_t(3)) - mis;
    g.a1 = ((g.s1 + mis) & ~int64_t(3)) - mis;
    if (g.a0 > g.a1) { g.a0 = g.s1; g.a1 = g.s1; }  // no aligned body: everything is head
    g.nvec = (g.a1 - g.a0) >> 2;
    g.ntiles = static_cast<uint32_t>((g.nvec * 4 + TILE - 1) / TILE);
    return g;
}

// Thread 0: start the bulk copy of tile i of a segment into ring stage
// (first + i) % STAGES.
template <int TILE, int STAGES>
__device__ __forceinline__ void issue_tile(float* ring, uint64_t* bars, const TaskView& tv, const SegGeom& g,
                                           uint32_t i, uint32_t first) {
    const uint32_t st = (first + i) % STAGES;
    const int64_t e0 = static_cast<int64_t>(i) * TILE;
    const uint32_t bytes = static_cast<uint32_t>(min(static_cast<int64_t>(TILE), g.nvec * 4 - e0)) * 4u;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bars + st, bytes);
    bulk_load(ring + static_cast<size_t>(st) * TILE, tv.data + g.a0 + e0, bytes, bars + st);
}

template <int TILE, int STAGES>
__device__ __forceinline__ void issue_prologue(float* ring, uint64_t* bars, const TaskView& tv, const SegGeom& g,
                                               uint32_t first) {
    for (uint32_t i = 0; i < g.ntiles && i < static_cast<uint32_t>(STAGES); ++i)
        issue_tile<TILE, STAGES>(ring, bars, tv, g, i, first);
}

template <int THREADS, int VEC, int STAGES, bool kScale>
__global__ void __launch_bounds__(THREADS, (THREADS >= 512 ? 1 : 3)) fused_topk_kernel(FusedParams p) {
    grid_dep_wait();  // launched after the previous kernel of the call
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ FusedShared<THREADS> sh;
    constexpr int U = VEC / 4;                      // float4 per thread per tile
    constexpr uint32_t TILE = THREADS * VEC;        // elements per tile (one ring stage)
    constexpr int NW = THREADS / 32;
    constexpr uint32_t R = kRegionEntries / NW;     // append region of each warp
    constexpr uint32_t RSLACK = 2 * U * 4;           // refill the regions before they run short
    float* ring = reinterpret_cast<float*>(smem_raw);
    uint64_t* s_buf = reinterpret_cast<uint64_t*>(smem_raw + static_cast<size_t>(STAGES) * TILE * 4);
    uint64_t* bars = s_buf + p.cap;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const uint32_t lt = lanemask_lt();
    const uint32_t cap = p.cap;
    const uint32_t cap_s = p.cap - kRegionEntries;  // settled region [0, cap_s), then the warp regions
    uint64_t* region = s_buf + cap_s + warp * R;
    // Merge path (contiguous buffer): shrink once fewer than this many slots are free.
    const uint32_t compact_at = cap - max(cap / 8, static_cast<uint32_t>(THREADS) + 8u);

    if (p.retry && *reinterpret_cast<volatile const uint32_t*>(p.fail_any) == 0u) return;  // nothing to redo
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(bars + s, 1);
        fence_mbar_init();
        sh.abort = 0;
        sh.work = static_cast<int32_t>(atomicAdd(p.work_counter, 1u));
    }
    block_sync<THREADS>();
    uint32_t gtile = 0;      // tiles this CTA consumed so far: ring stage and mbarrier phase
    int w = sh.work;
    bool prefetched = false;  // the current item's first tiles are already in flight

    while (w < p.nsegs) {
        TaskView tv;
        const SegGeom G = seg_geom<TILE, kScale>(p, w, &tv);
        const int t = G.sg.task;
        int nw = p.nsegs;  // next work item, fetched once this one's tiles are consumed
        if (G.skip) {      // retry launch: only flagged tasks run
            block_sync<THREADS>();
            if (tid == 0) sh.work = static_cast<int32_t>(atomicAdd(p.work_counter, 1u));
            block_sync<THREADS>();
            w = sh.work;
            prefetched = false;
            continue;
        }
        const FusedTask& td = G.td;
        const uint32_t k = tv.k;
        const uint32_t mid_keep = k + (cap_s - k) / 2;
        const bool multi = td.nseg > 1;
        const float scaler = kScale ? task_scaler(tv.data, 0, tv.len, 1) : 0.0f;
        bool next_prefetched = false;

        for (int attempt = 0; attempt < 2; ++attempt) {
            if (!prefetched && tid == 0) issue_prologue<TILE, STAGES>(ring, bars, tv, G, gtile);
            prefetched = false;
            uint64_t thr = 0;
            bool sampled_local = false;
            if (multi) {
                if (tid == 0) sh.gthr = load_volatile_u64(p.gthr + t);
                block_sync<THREADS>();
                thr = sh.gthr;
            } else if (attempt == 0) {
                // Overlaps with the tile copies already in flight.
                thr = sampled_threshold<THREADS, kScale>(tv, scaler, k, s_buf, sh, p.err);
                sampled_local = thr != 0;
            }
            block_sync<THREADS>();
            if (tid == 0) { sh.cnt = 0; sh.gthr = thr; }
            block_sync<THREADS>();
            uint32_t wcnt = 0;  // entries in this warp's region (same in all its lanes)

            // Head [s0, a0) and tail [a1, s1): fewer than 4 elements each (warp 0).
            if (warp == 0) {
                const int nh = static_cast<int>(G.a0 - G.s0), nt = static_cast<int>(G.s1 - G.a1);
                bool pass = false;
                uint64_t c = 0;
                int64_t q = -1;
                if (tid < nh) q = G.s0 + tid;
                else if (tid >= 8 && tid - 8 < nt) q = G.a1 + (tid - 8);
                if (q >= 0) {
                    uint32_t bits = __float_as_uint(tv.data[q]);
                    c = make_composite(score_of<kScale>(bits, scaler, tv.sp), static_cast<uint32_t>(q));
                    pass = c > thr;
                }
                const uint32_t m = __ballot_sync(kFullMask, pass);
                if (pass) region[__popc(m & lt)] = c;
                wcnt = __popc(m);
            }
            const uint32_t pos0 = static_cast<uint32_t>(G.a0);
            FastFilter ff = make_fast_filter<kScale>(thr, tv.sp, scaler);
            const int64_t nvec = G.nvec;
            const uint32_t ntiles = G.ntiles;
            uint64_t gnext = 0;  // thread 0: latest global threshold, read a few tiles ahead
            for (uint32_t it = 0; it < ntiles; ++it) {
                const uint32_t g = gtile + it;
                const uint32_t st = g % STAGES;
                bool flag = false;  // this thread needs the slow path after the tile
                if (!mbar_wait_bounded(bars + st, (g / STAGES) & 1u, kWaitPolls)) {
                    record_error(p.err, kErrTimeout);
                    sh.abort = 1;
                    flag = true;
                }
                if (multi && tid == 0 && (it & 7) == 0) gnext = load_volatile_u64(p.gthr + t);
                const float4* t4 = reinterpret_cast<const float4*>(ring + static_cast<size_t>(st) * TILE);
                const int64_t qb = static_cast<int64_t>(it) * (TILE / 4);
                // Fast superset filter: one compare per element, and only
                // "does any element of this thread pass" is kept.
                float4 v[U];
                const bool full = qb + static_cast<int64_t>(U) * THREADS <= nvec;
                bool anyp = false;
                if (full) {
#pragma unroll
                    for (int j = 0; j < U; ++j) v[j] = t4[j * THREADS + tid];
                } else {
#pragma unroll
                    for (int j = 0; j < U; ++j) {
                        const int64_t q = qb + j * THREADS + tid;
                        v[j] = (q < nvec) ? t4[j * THREADS + tid] : ff.pad4;
                    }
                }
                if constexpr (kScale) {
#pragma unroll
                    for (int j = 0; j < U; ++j) {
                        v[j].x = __fsub_rn(v[j].x, scaler); v[j].y = __fsub_rn(v[j].y, scaler);
                        v[j].z = __fsub_rn(v[j].z, scaler); v[j].w = __fsub_rn(v[j].w, scaler);
                    }
                }
                if (ff.dir == 0u && !ff.nan_pass) {
#pragma unroll
                    for (int j = 0; j < U; ++j)
                        anyp |= (v[j].x >= ff.t) | (v[j].y >= ff.t) | (v[j].z >= ff.t) | (v[j].w >= ff.t);
                } else if (!ff.nan_pass) {
#pragma unroll
                    for (int j = 0; j < U; ++j)
                        anyp |= (v[j].x <= ff.tr) | (v[j].y <= ff.tr) | (v[j].z <= ff.tr) | (v[j].w <= ff.tr);
                } else if (ff.dir == 0u) {
#pragma unroll
                    for (int j = 0; j < U; ++j)
                        anyp |= !(v[j].x < ff.t) | !(v[j].y < ff.t) | !(v[j].z < ff.t) | !(v[j].w < ff.t);
                } else {
#pragma unroll
                    for (int j = 0; j < U; ++j)
                        anyp |= !(v[j].x > ff.tr) | !(v[j].y > ff.tr) | !(v[j].z > ff.tr) | !(v[j].w > ff.tr);
                }
                // Candidates (a superset of the passing elements, kept with
                // their exact composites) go to this warp's region: one warp
                // scan of the per-lane counts, then each lane writes its own.
                uint32_t dm = 0;  // candidates that found no room (re-offered after a shrink)
                if (__any_sync(kFullMask, anyp)) {
                    uint32_t pm = 0;
                    if (anyp) {
#pragma unroll
                        for (int j = 0; j < U; ++j) {
                            const int64_t q = qb + j * THREADS + tid;
                            const float f4[4] = {v[j].x, v[j].y, v[j].z, v[j].w};
#pragma unroll
                            for (int e = 0; e < 4; ++e) {
                                const float x = __uint_as_float(__float_as_uint(f4[e]) ^ ff.dir);
                                const bool ps = (q < nvec) && (ff.nan_pass ? !(x < ff.t) : (x >= ff.t));
                                pm |= static_cast<uint32_t>(ps) << (j * 4 + e);
                            }
                        }
                    }
                    const uint32_t n = __popc(pm);
                    const uint32_t incl = warp_inclusive_scan<true>(n);
                    uint32_t slot = wcnt + incl - n;
                    wcnt += __shfl_sync(kFullMask, incl, 31);
                    const float* tile = ring + static_cast<size_t>(st) * TILE;
                    for (uint32_t m = pm; m; m &= m - 1) {
                        const int b = __ffs(m) - 1;
                        const uint32_t li = static_cast<uint32_t>((b >> 2) * THREADS + tid) * 4u + (b & 3);
                        const uint32_t pos = pos0 + static_cast<uint32_t>(qb) * 4u + li;
                        const uint64_t c = make_composite(score_of<kScale>(__float_as_uint(tile[li]), scaler, tv.sp), pos);
                        if (slot < R) region[slot] = c;
                        else dm |= 1u << b;
                        ++slot;
                    }
                    flag = flag || dm != 0 || wcnt + RSLACK > R;
                }
                const bool refresh = multi && (it & 7) == 7;
                if (refresh && tid == 0 && gnext > sh.gthr) sh.gthr = gnext;
                // One barrier per tile; it also tells every thread whether a
                // warp region runs short, candidates wait for room, or a wait
                // timed out.
                if (block_sync_or<THREADS>(flag ? 1 : 0)) {
                    if (sh.abort) {
                        // Drain the copies this CTA still has in flight (bounded).
                        if (tid == 0) {
                            for (uint32_t i = it + 1; i < ntiles && i < it + STAGES; ++i)
                                mbar_wait_bounded(bars + (gtile + i) % STAGES, ((gtile + i) / STAGES) & 1u,
                                                  kWaitPolls);
                        }
                        block_sync<THREADS>();
                        return;
                    }
                    // Gather the regions, shrink, raise the threshold, and
                    // re-offer the candidates that found no room; repeat until
                    // all of them are placed or no longer pass.
                    for (int round = 0; round < 16; ++round) {
                        gather_regions<THREADS, R>(s_buf, cap_s, wcnt, sh);
                        const uint64_t kf = shrink_mid<THREADS>(p, k, mid_keep, s_buf, sh);
                        if (kf != 0) {
                            thr = (kf - 1) > thr ? (kf - 1) : thr;
                            ff = make_fast_filter<kScale>(thr, tv.sp, scaler);
                            if (multi && tid == 0)
                                atomicMax(reinterpret_cast<unsigned long long*>(p.gthr + t), kf - 1);
                        }
                        const uint32_t rm_in = dm;
                        dm = 0;
                        bool again = false;
                        if (__any_sync(kFullMask, rm_in != 0)) {
                            const float* tile = ring + static_cast<size_t>(st) * TILE;
                            uint32_t rm = 0;
                            for (uint32_t m = rm_in; m; m &= m - 1) {
                                const int b = __ffs(m) - 1;
                                const uint32_t li = static_cast<uint32_t>((b >> 2) * THREADS + tid) * 4u + (b & 3);
                                const uint32_t pos = pos0 + static_cast<uint32_t>(qb) * 4u + li;
                                const uint64_t c =
                                    make_composite(score_of<kScale>(__float_as_uint(tile[li]), scaler, tv.sp), pos);
                                rm |= (c > thr) ? (1u << b) : 0u;
                            }
                            const uint32_t n = __popc(rm);
                            const uint32_t incl = warp_inclusive_scan<true>(n);
                            uint32_t slot = wcnt + incl - n;
                            wcnt += __shfl_sync(kFullMask, incl, 31);
                            for (uint32_t m = rm; m; m &= m - 1) {
                                const int b = __ffs(m) - 1;
                                const uint32_t li = static_cast<uint32_t>((b >> 2) * THREADS + tid) * 4u + (b & 3);
                                const uint32_t pos = pos0 + static_cast<uint32_t>(qb) * 4u + li;
                                const uint64_t c =
                                    make_composite(score_of<kScale>(__float_as_uint(tile[li]), scaler, tv.sp), pos);
                                if (slot < R) region[slot] = c;
                                else dm |= 1u << b;
                                ++slot;
                            }
                            again = dm != 0 || wcnt + RSLACK > R;
                        }
                        if (!block_sync_or<THREADS>(again ? 1 : 0)) break;
                    }
                    if (dm != 0) record_error(p.err, kErrCapacity);
                }
                if (refresh) {
                    const uint64_t g_now = sh.gthr;
                    if (g_now > thr) {
                        thr = g_now;
                        ff = make_fast_filter<kScale>(thr, tv.sp, scaler);
                    }
                }
                // The stage just read is free: refill it with tile it + STAGES.
                if (tid == 0 && it + STAGES < ntiles) issue_tile<TILE, STAGES>(ring, bars, tv, G, it + STAGES, gtile);
            }
            gtile += ntiles;
            gather_regions<THREADS, R>(s_buf, cap_s, wcnt, sh);  // all candidates now in [0, sh.cnt)

            if (!multi) {
                const uint32_t want = tv.len < static_cast<int64_t>(k) ? static_cast<uint32_t>(tv.len) : k;
                if (sh.cnt < want && sampled_local) continue;  // sample overestimated: redo without it
            }
            break;
        }

        // This item's tiles are all consumed: fetch the next item and start its
        // first tile copies, so they overlap the selection work below.
        if (tid == 0) sh.work = static_cast<int32_t>(atomicAdd(p.work_counter, 1u));
        block_sync<THREADS>();
        nw = sh.work;
        if (nw < p.nsegs) {
            TaskView ntv;
            const SegGeom NG = seg_geom<TILE, kScale>(p, nw, &ntv);
            if (!NG.skip) {
                if (tid == 0) issue_prologue<TILE, STAGES>(ring, bars, ntv, NG, gtile);
                next_prefetched = true;
            }
        }

        if (!multi) {
            finish_candidates<THREADS, kScale>(p, tv, s_buf, sh);
        } else {
            // Multi-segment task: publish this segment's k-th composite, append
            // the survivors to the task's candidate region, count the segment.
            uint64_t kth = 0;
            shrink_final<THREADS>(p, k, s_buf, sh, &kth);
            if (tid == 0) {
                if (kth != 0) atomicMax(reinterpret_cast<unsigned long long*>(p.gthr + t), kth - 1);
                sh.gthr = load_volatile_u64(p.gthr + t);
            }
            block_sync<THREADS>();
            {
                const uint64_t g = sh.gthr;
                const uint32_t cnt = sh.cnt;
                uint64_t* dst = p.cand + td.cbase;
                const uint32_t region = static_cast<uint32_t>(td.nseg) * p.kmax;
                for (uint32_t b0 = 0; b0 < cnt; b0 += THREADS) {
                    uint32_t i = b0 + tid;
                    uint64_t c = (i < cnt) ? s_buf[i] : 0ull;
                    bool keep = (i < cnt) && c > g;
                    uint32_t total;
                    uint32_t off = block_exclusive_scan<THREADS>(keep ? 1u : 0u, &total, sh.bs);
                    if (tid == 0 && total) sh.base = atomicAdd(p.task_cnt + t, total);
                    block_sync<THREADS>();
                    if (keep) {
                        uint32_t o = sh.base + off;
                        if (o < region) dst[o] = c;
                        else record_error(p.err, kErrCapacity);
                    }
                    block_sync<THREADS>();
                }
            }
            __threadfence();
            block_sync<THREADS>();
            if (tid == 0) {
                uint32_t done = atomicAdd(p.task_done + t, 1u);
                sh.last = (done == static_cast<uint32_t>(td.nseg - 1)) ? 1u : 0u;
            }
            block_sync<THREADS>();
            if (sh.last) {
                // Last segment of the task: merge all segments' survivors.
                __threadfence();
                if (tid == 0) {
                    sh.cnt = 0;
                    sh.gthr = load_volatile_u64(p.gthr + t);
                    sh.base = __ldcg(p.task_cnt + t);
                }
                block_sync<THREADS>();
                const uint64_t g = sh.gthr;
                const uint32_t region = static_cast<uint32_t>(td.nseg) * p.kmax;
                const uint32_t n = sh.base < region ? sh.base : region;
                const unsigned long long* src = reinterpret_cast<const unsigned long long*>(p.cand + td.cbase);
                for (uint32_t b0 = 0; b0 < n; b0 += THREADS) {
                    {
                        uint32_t i = b0 + tid;
                        uint64_t c = (i < n) ? __ldcg(src + i) : 0ull;
                        warp_append((i < n) && c > g, c, s_buf, &sh.cnt, cap, p.err);
                    }
                    block_sync<THREADS>();
                    const uint32_t cnt_now = sh.cnt;
                    block_sync<THREADS>();
                    if (cnt_now > compact_at) shrink_mid<THREADS>(p, k, mid_keep, s_buf, sh);
                }
                block_sync<THREADS>();
                const uint32_t m = shrink_final<THREADS>(p, k, s_buf, sh, &kth);
                if (m < k && (td.flags & kTaskSampled) && !p.retry) {
                    // The sampled threshold was above the task's k-th composite.
                    if (tid == 0) {
                        p.fail[t] = 1u;
                        atomicExch(p.fail_any, 1u);
                    }
                } else {
                    if (m != k && tid == 0) record_error(p.err, kErrInternal);
                    finish_task<THREADS, !kScale>(p, tv, s_buf, m < k ? m : k, sh);
                }
            }
        }
        block_sync<THREADS>();
        w = nw;
        prefetched = next_prefetched;
    }
}

}  // namespace radik
