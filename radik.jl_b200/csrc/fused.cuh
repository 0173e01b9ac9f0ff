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

enum : uint32_t { kTaskLargest = 1u, kTaskAscend = 2u, kTaskSampled = 4u };

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
    uint32_t* work_counter;  // [1]
    uint64_t* cand;          // candidate regions
    uint64_t* sort_scratch;  // [gridDim.x * kmax] (kmax > 4096 only)
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
    uint64_t gthr;
    uint64_t hi;     // upper bound of the buffer's composites
};

__device__ __forceinline__ uint64_t warp_max_u64(uint64_t v) {
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) {
        uint64_t o = __shfl_xor_sync(kFullMask, static_cast<unsigned long long>(v), m);
        v = o > v ? o : v;
    }
    return v;
}

// Appends composite c (when pass) to the shared buffer with one shared atomic
// per warp (warp-aggregated) and keeps the buffer's upper bound.  All lanes
// of the warp must call.
__device__ __forceinline__ void warp_append(bool pass, uint64_t c, uint64_t* buf, uint32_t* cnt, uint64_t* hi,
                                            uint32_t cap, uint32_t* err) {
    uint32_t m = __ballot_sync(kFullMask, pass);
    if (m == 0) return;
    const uint32_t lane = lane_id();
    const uint32_t leader = __ffs(m) - 1;
    const uint64_t mx = warp_max_u64(pass ? c : 0ull);
    uint32_t base = 0;
    if (lane == leader) {
        base = atomicAdd(cnt, __popc(m));
        atomicMax(reinterpret_cast<unsigned long long*>(hi), static_cast<unsigned long long>(mx));
    }
    base = __shfl_sync(kFullMask, base, leader);
    if (pass) {
        uint32_t i = base + __popc(m & lanemask_lt());
        if (i < cap) buf[i] = c;
        else record_error(err, kErrCapacity);
    }
}

// Write a task's output row from its m sorted output keys (low 32 bits =
// position): value, index (automatic 1-based or custom), padding.
template <int THREADS>
__device__ void write_row(const FusedParams& p, const TaskView& tv, const uint64_t* sorted, uint32_t m) {
    const int tid = threadIdx.x;
    for (uint32_t j = tid; j < tv.k; j += THREADS) {
        float v = 0.0f;
        int64_t idx = -1;
        if (j < m) {
            uint32_t pos = static_cast<uint32_t>(sorted[j]);
            if (pos >= static_cast<uint64_t>(tv.len)) pos = 0;  // bounded gather (error recorded earlier)
            v = tv.data[pos];
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
    __syncthreads();
}

// Sort the m finished composites of a task by the output order, map indices
// and write the task's output row (padding slots m..k-1 with 0 / -1,
// src/algorithm.jl:358-365).  buf has room for next_pow2(m) <= cap entries
// and, past m, for the radix sort's shared counters.
template <int THREADS>
__device__ void finish_task(const FusedParams& p, const TaskView& tv, uint64_t* buf, uint32_t m,
                            FusedShared<THREADS>& sh) {
    const int tid = threadIdx.x;
    for (uint32_t i = tid; i < m; i += THREADS) {
        uint32_t pos = composite_pos(buf[i]);
        if (pos >= static_cast<uint64_t>(tv.len)) {  // never expected; keep the gather in bounds
            record_error(p.err, kErrBounds);
            pos = 0;
        }
        uint32_t bits = __float_as_uint(tv.data[pos]);
        buf[i] = output_sort_key(bits, pos, tv.sp, tv.ascend);
    }
    __syncthreads();
    uint64_t* sorted = buf;
    if (m <= kBitonicMax) {
        uint32_t P = 1;
        while (P < m) P <<= 1;
        for (uint32_t i = m + tid; i < P; i += THREADS) buf[i] = ~0ull;
        __syncthreads();
        bitonic_sort_u64<THREADS>(buf, P);
    } else {
        uint64_t* scratch = p.sort_scratch + static_cast<int64_t>(blockIdx.x) * p.kmax;
        uint32_t* wd = reinterpret_cast<uint32_t*>(buf + m);
        uint32_t* db = wd + (THREADS / 32) * 256;
        sorted = radix_sort_u64<THREADS>(buf, scratch, m, sh.bs, wd, db);
    }
    __syncthreads();
    write_row<THREADS>(p, tv, sorted, m);
}

// Shared count, clamped to the buffer (appends past cap were dropped and
// recorded); all threads must call.
template <int THREADS>
__device__ __forceinline__ uint32_t buffer_count(const FusedParams& p, FusedShared<THREADS>& sh) {
    uint32_t cnt = sh.cnt;
    if (cnt > p.cap) {
        cnt = p.cap;
        __syncthreads();
        if (threadIdx.x == 0) sh.cnt = cnt;
        __syncthreads();
    }
    return cnt;
}

// Mid-stream reduction: keeps between k and max_keep entries (all of them
// >= the returned keep_from); lo must bound every entry from below.
// Returns keep_from, or 0 when nothing was dropped.
template <int THREADS>
__device__ uint64_t shrink_mid(const FusedParams& p, uint32_t k, uint32_t max_keep, uint64_t lo, uint64_t* buf,
                               FusedShared<THREADS>& sh) {
    const uint32_t cnt = buffer_count<THREADS>(p, sh);
    uint64_t kf = 0, mn = 0;
    const uint32_t kept = block_shrink<THREADS>(buf, cnt, k, max_keep, lo, sh.hi, sh.bs, p.err, &kf, &mn);
    __syncthreads();
    if (threadIdx.x == 0) sh.cnt = kept;
    __syncthreads();
    return (kept >= k && kept < cnt) ? kf : 0ull;
}

// Exact top-k of a small buffer (next_pow2(cnt) <= cap and <= 4096 entries):
// one descending bitonic sort puts the best min(cnt, k) composites first.
// Returns their number; *kth receives the k-th composite (0 if fewer than k).
template <int THREADS>
__device__ uint32_t select_small(uint64_t* buf, uint32_t cnt, uint32_t k, uint64_t* kth) {
    uint32_t P = 1;
    while (P < cnt) P <<= 1;
    for (uint32_t i = cnt + threadIdx.x; i < P; i += THREADS) buf[i] = 0ull;  // below every composite
    __syncthreads();
    bitonic_sort_u64<THREADS>(buf, P, true);
    const uint32_t m = cnt < k ? cnt : k;
    *kth = (m == k && m > 0) ? buf[m - 1] : 0ull;
    return m;
}

// Exact reduction of the buffer to its best k, by bitonic sort when small,
// else by radix selection.  Returns the number kept and the k-th composite.
template <int THREADS>
__device__ uint32_t shrink_final(const FusedParams& p, uint32_t k, uint64_t* buf, FusedShared<THREADS>& sh,
                                 uint64_t* kth) {
    const uint32_t cnt = buffer_count<THREADS>(p, sh);
    uint32_t P = 1;
    while (P < cnt) P <<= 1;
    uint32_t m;
    if (P <= kBitonicMax && P <= p.cap) {
        m = select_small<THREADS>(buf, cnt, k, kth);
    } else {
        m = block_select_topk<THREADS>(buf, cnt, k, sh.bs, p.err, kth);
        if (m < k) *kth = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) sh.cnt = m;
    __syncthreads();
    return m;
}

// Starting threshold of a single-segment task from a sample of `S` of its
// elements (16 chunks of S/16 consecutive elements): one below the composite
// of sample rank r, where r is chosen so that about 2k elements of the task
// are expected above it.  0 (no pruning) when the sample is too small.
template <int THREADS, bool kScale>
__device__ uint64_t sampled_threshold(const TaskView& tv, float scaler, uint32_t k, uint64_t* buf) {
    constexpr uint32_t S = 1024, CH = S / 16;
    const int64_t len = tv.len;
    if (len < 8 * static_cast<int64_t>(S)) return 0ull;
    const float lam = static_cast<float>(k) * S / static_cast<float>(len);
    const uint32_t r = static_cast<uint32_t>(ceilf(2.0f * lam + 4.0f * sqrtf(lam) + 12.0f));
    if (r > S / 4) return 0ull;
    const int64_t cstride = len / 16;
    for (uint32_t i = threadIdx.x; i < S; i += THREADS) {
        const int64_t q = static_cast<int64_t>(i / CH) * cstride + (i % CH);
        const uint32_t bits = __float_as_uint(tv.data[q]);
        buf[i] = make_composite(score_of<kScale>(bits, scaler, tv.sp), static_cast<uint32_t>(q));
    }
    __syncthreads();
    bitonic_sort_u64<THREADS>(buf, S, true);
    const uint64_t c = buf[r - 1];
    __syncthreads();
    return c - 1;
}

constexpr uint32_t kWaitPolls = 1u << 22;

template <int THREADS, int VEC, int STAGES, bool kScale>
__global__ void __launch_bounds__(THREADS, (THREADS >= 512 ? 1 : 3)) fused_topk_kernel(FusedParams p) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ FusedShared<THREADS> sh;
    constexpr int U = VEC / 4;                      // float4 per thread per tile
    constexpr uint32_t TILE = THREADS * VEC;        // elements per tile (one ring stage)
    float* ring = reinterpret_cast<float*>(smem_raw);
    uint64_t* s_buf = reinterpret_cast<uint64_t*>(smem_raw + static_cast<size_t>(STAGES) * TILE * 4);
    uint64_t* bars = s_buf + p.cap;
    const int tid = threadIdx.x;
    const uint32_t cap = p.cap;
    const uint32_t compact_at = cap - TILE - 8;     // host guarantees cap >= kmax + TILE + headroom

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(bars + s, 1);
        fence_mbar_init();
        sh.abort = 0;
    }
    __syncthreads();
    uint32_t gtile = 0;  // tiles this CTA consumed so far: ring stage and mbarrier phase

    for (;;) {
        if (tid == 0) sh.work = static_cast<int32_t>(atomicAdd(p.work_counter, 1u));
        __syncthreads();
        const int w = sh.work;
        if (w >= p.nsegs || sh.abort) break;
        const FusedSeg sg = p.segs[w];
        const int t = sg.task;
        if (p.retry && p.fail[t] == 0) {  // retry launch: only flagged tasks
            __syncthreads();
            continue;
        }
        const FusedTask td = p.tasks[t];
        const TaskView tv = task_view<kScale>(p, t, td);
        const uint32_t k = tv.k;
        const uint32_t mid_keep = k + (cap - k - TILE) / 4;
        const bool multi = td.nseg > 1;
        const float scaler = kScale ? task_scaler(tv.data, 0, tv.len, 1) : 0.0f;
        const int64_t s0 = sg.pos, s1 = static_cast<int64_t>(sg.pos) + sg.len;
        // Position q sits on a 16-byte boundary iff (q + mis) % 4 == 0.
        const int64_t mis = static_cast<int64_t>((reinterpret_cast<uintptr_t>(tv.data) >> 2) & 3);
        int64_t a0 = ((s0 + mis + 3) & ~int64_t(3)) - mis;
        int64_t a1 = ((s1 + mis) & ~int64_t(3)) - mis;
        if (a0 > a1) { a0 = s1; a1 = s1; }   // no aligned body: everything is head
        const int64_t nvec = (a1 - a0) >> 2;
        const uint32_t ntiles = static_cast<uint32_t>((nvec * 4 + TILE - 1) / TILE);

        bool done_task = false;
        for (int attempt = 0; attempt < 2 && !done_task; ++attempt) {
            uint64_t thr = 0;
            bool sampled_local = false;
            if (multi) {
                if (tid == 0) sh.gthr = load_volatile_u64(p.gthr + t);
                __syncthreads();
                thr = sh.gthr;
            } else if (attempt == 0) {
                thr = sampled_threshold<THREADS, kScale>(tv, scaler, k, s_buf);
                sampled_local = thr != 0;
            }
            if (tid == 0) { sh.cnt = 0; sh.hi = 0; sh.gthr = thr; }
            __syncthreads();
            uint64_t lo = thr;  // every buffered composite is >= lo

            // Prologue: start the first STAGES tile copies.
            if (tid == 0) {
                for (uint32_t i = 0; i < ntiles && i < static_cast<uint32_t>(STAGES); ++i) {
                    const uint32_t st = (gtile + i) % STAGES;
                    const int64_t e0 = static_cast<int64_t>(i) * TILE;
                    const uint32_t bytes = static_cast<uint32_t>(min(static_cast<int64_t>(TILE), nvec * 4 - e0)) * 4u;
                    fence_proxy_async_smem();
                    mbar_arrive_expect_tx(bars + st, bytes);
                    bulk_load(ring + static_cast<size_t>(st) * TILE, tv.data + a0 + e0, bytes, bars + st);
                }
            }
            // Head [s0, a0) and tail [a1, s1): fewer than 4 elements each.
            if (tid < 32) {
                const int nh = static_cast<int>(a0 - s0), nt = static_cast<int>(s1 - a1);
                bool pass = false;
                uint64_t c = 0;
                int64_t q = -1;
                if (tid < nh) q = s0 + tid;
                else if (tid >= 8 && tid - 8 < nt) q = a1 + (tid - 8);
                if (q >= 0) {
                    uint32_t bits = __float_as_uint(tv.data[q]);
                    c = make_composite(score_of<kScale>(bits, scaler, tv.sp), static_cast<uint32_t>(q));
                    pass = c > thr;
                }
                warp_append(pass, c, s_buf, &sh.cnt, &sh.hi, cap, p.err);
            }
            const uint32_t pos0 = static_cast<uint32_t>(a0);
            for (uint32_t it = 0; it < ntiles; ++it) {
                const uint32_t g = gtile + it;
                const uint32_t st = g % STAGES;
                if (!mbar_wait_bounded(bars + st, (g / STAGES) & 1u, kWaitPolls)) {
                    record_error(p.err, kErrTimeout);
                    sh.abort = 1;
                }
                const float4* t4 = reinterpret_cast<const float4*>(ring + static_cast<size_t>(st) * TILE);
                const int64_t qb = static_cast<int64_t>(it) * (TILE / 4);
                float4 v[U];
                uint32_t pm = 0;
#pragma unroll
                for (int j = 0; j < U; ++j) {
                    const int64_t q = qb + j * THREADS + tid;
                    v[j] = (q < nvec) ? t4[j * THREADS + tid] : make_float4(0.f, 0.f, 0.f, 0.f);
                    if (q < nvec) {
                        const uint32_t pb = pos0 + static_cast<uint32_t>(q) * 4u;
                        const float f[4] = {v[j].x, v[j].y, v[j].z, v[j].w};
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            uint64_t c = make_composite(score_of<kScale>(__float_as_uint(f[e]), scaler, tv.sp), pb + e);
                            pm |= (c > thr) ? (1u << (j * 4 + e)) : 0u;
                        }
                    }
                }
                if (__any_sync(kFullMask, pm != 0)) {
#pragma unroll
                    for (int j = 0; j < U; ++j) {
                        const int64_t q = qb + j * THREADS + tid;
                        const uint32_t pb = pos0 + static_cast<uint32_t>(q) * 4u;
                        const float f[4] = {v[j].x, v[j].y, v[j].z, v[j].w};
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const bool ps = (pm >> (j * 4 + e)) & 1u;
                            uint64_t c = ps ? make_composite(score_of<kScale>(__float_as_uint(f[e]), scaler, tv.sp), pb + e)
                                            : 0ull;
                            warp_append(ps, c, s_buf, &sh.cnt, &sh.hi, cap, p.err);
                        }
                    }
                }
                uint64_t gnew = 0;
                if (multi && tid == 0 && (it & 7) == 7) gnew = load_volatile_u64(p.gthr + t);
                if (multi && tid == 0 && gnew > sh.gthr) sh.gthr = gnew;
                // Snapshot shared state between two barriers: nobody may read
                // it after a faster thread started on the next tile.
                __syncthreads();
                const uint32_t cnt_now = sh.cnt;
                const uint64_t g_now = sh.gthr;
                const uint32_t ab = sh.abort;
                __syncthreads();
                if (ab) {
                    // Drain the copies this CTA still has in flight (bounded).
                    if (tid == 0) {
                        for (uint32_t i = it + 1; i < ntiles && i < it + STAGES; ++i)
                            mbar_wait_bounded(bars + (gtile + i) % STAGES, ((gtile + i) / STAGES) & 1u, kWaitPolls);
                    }
                    __syncthreads();
                    return;
                }
                // The stage just read is free: refill it with tile it + STAGES.
                if (tid == 0 && it + STAGES < ntiles) {
                    const int64_t e0 = static_cast<int64_t>(it + STAGES) * TILE;
                    const uint32_t bytes = static_cast<uint32_t>(min(static_cast<int64_t>(TILE), nvec * 4 - e0)) * 4u;
                    fence_proxy_async_smem();
                    mbar_arrive_expect_tx(bars + st, bytes);
                    bulk_load(ring + static_cast<size_t>(st) * TILE, tv.data + a0 + e0, bytes, bars + st);
                }
                if (cnt_now > compact_at) {
                    const uint64_t kf = shrink_mid<THREADS>(p, k, mid_keep, lo, s_buf, sh);
                    if (kf != 0) {
                        lo = kf;
                        thr = (kf - 1) > thr ? (kf - 1) : thr;
                        if (multi && tid == 0) atomicMax(reinterpret_cast<unsigned long long*>(p.gthr + t), kf - 1);
                    }
                }
                if (multi) thr = g_now > thr ? g_now : thr;
            }
            gtile += ntiles;
            __syncthreads();

            if (!multi) {
                uint64_t kth = 0;
                const uint32_t want = tv.len < static_cast<int64_t>(k) ? static_cast<uint32_t>(tv.len) : k;
                const uint32_t have = buffer_count<THREADS>(p, sh);
                if (have < want && sampled_local) continue;  // sample overestimated: redo without it
                const uint32_t m = shrink_final<THREADS>(p, k, s_buf, sh, &kth);
                if (m != want && tid == 0) record_error(p.err, kErrInternal);
                finish_task<THREADS>(p, tv, s_buf, m < want ? m : want, sh);
            }
            done_task = true;
        }
        if (!multi) continue;

        // Multi-segment task: publish this segment's k-th composite, append the
        // survivors to the task's candidate region, count the segment done.
        uint64_t kth = 0;
        shrink_final<THREADS>(p, k, s_buf, sh, &kth);
        if (tid == 0) {
            if (kth != 0) atomicMax(reinterpret_cast<unsigned long long*>(p.gthr + t), kth - 1);
            sh.gthr = load_volatile_u64(p.gthr + t);
        }
        __syncthreads();
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
                __syncthreads();
                if (keep) {
                    uint32_t o = sh.base + off;
                    if (o < region) dst[o] = c;
                    else record_error(p.err, kErrCapacity);
                }
                __syncthreads();
            }
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) {
            uint32_t done = atomicAdd(p.task_done + t, 1u);
            sh.last = (done == static_cast<uint32_t>(td.nseg - 1)) ? 1u : 0u;
        }
        __syncthreads();
        if (!sh.last) continue;

        // Last segment of the task: merge all segments' survivors.
        __threadfence();
        if (tid == 0) {
            sh.cnt = 0;
            sh.hi = 0;
            sh.gthr = load_volatile_u64(p.gthr + t);
            sh.base = __ldcg(p.task_cnt + t);
        }
        __syncthreads();
        const uint64_t g = sh.gthr;
        const uint32_t region = static_cast<uint32_t>(td.nseg) * p.kmax;
        const uint32_t n = sh.base < region ? sh.base : region;
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(p.cand + td.cbase);
        uint64_t mlo = g;
        for (uint32_t b0 = 0; b0 < n; b0 += 4 * THREADS) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                uint32_t i = b0 + j * THREADS + tid;
                uint64_t c = (i < n) ? __ldcg(src + i) : 0ull;
                warp_append((i < n) && c > g, c, s_buf, &sh.cnt, &sh.hi, cap, p.err);
            }
            __syncthreads();
            const uint32_t cnt_now = sh.cnt;
            __syncthreads();
            if (cnt_now > compact_at) {
                const uint64_t kf = shrink_mid<THREADS>(p, k, mid_keep, mlo, s_buf, sh);
                if (kf != 0) mlo = kf;
            }
        }
        __syncthreads();
        const uint32_t m = shrink_final<THREADS>(p, k, s_buf, sh, &kth);
        if (m < k && (td.flags & kTaskSampled) && !p.retry) {
            // The sampled threshold was above the task's k-th composite.
            if (tid == 0) p.fail[t] = 1u;
            __syncthreads();
            continue;
        }
        if (m != k && tid == 0) record_error(p.err, kErrInternal);
        finish_task<THREADS>(p, tv, s_buf, m < k ? m : k, sh);
    }
}

}  // namespace radik
