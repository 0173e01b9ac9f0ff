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
// When the buffer fills up, block_select_topk (the histogram / rank search /
// narrowing cycle of count_bin.jl, select_bin.jl and select_candidate.jl on
// on-chip data) keeps the top k and raises the threshold to the k-th
// composite.  Segments of one task share a global threshold (atomicMax of the
// segments' k-th composites, a valid lower bound of the task's k-th
// composite).  A single-segment task is finished by its CTA; for a
// multi-segment task every segment writes its surviving top-k to global
// candidate slots and the last segment to finish (atomic counter, no waiting)
// merges them.  Finishing = exact top-k, gather of the original values,
// sort (bitonic <= 4096 entries, radix sort above), index mapping and padding.
#pragma once

#include "block_ops.cuh"

namespace radik {

struct FusedTask {
    int64_t start;   // global offset of the task
    int64_t len;     // elements
    int64_t slot0;   // first candidate slot (multi-segment tasks), else -1
    int32_t nseg;
    int32_t pad_;
};

struct FusedSeg {
    int64_t start;   // global offset of the first element of the segment
    int32_t len;
    int32_t task;
    int32_t seg_in_task;
    int32_t pad_;
};

struct FusedParams {
    const float* data;
    const FusedTask* tasks;
    const FusedSeg* segs;
    int32_t nsegs;
    uint32_t k;
    uint32_t cap;            // shared buffer capacity in composites
    int ascend;
    ScoreParams sp;
    const void* idx_in;      // nullable: custom indices (4 or 8 bytes wide)
    int idx_bytes;           // width of idx_out (and idx_in when present)
    float* val_out;          // [T][k]
    void* idx_out;           // [T][k]
    // workspace
    uint64_t* gthr;          // [T]
    uint32_t* task_done;     // [T]
    uint32_t* work_counter;  // [1]
    uint64_t* cand;          // [slots * k]
    uint32_t* slot_cnt;      // [slots]
    uint64_t* sort_scratch;  // [gridDim.x * k] (k > 4096 only)
    uint32_t* err;
};

constexpr uint32_t kBitonicMax = 4096;

__device__ __forceinline__ uint64_t load_volatile_u64(const uint64_t* p) {
    return *reinterpret_cast<const volatile uint64_t*>(p);
}

template <int THREADS>
struct FusedShared {
    BlockScratch<THREADS> bs;
    uint32_t cnt;
    int32_t work;
    uint32_t last;
    uint32_t pad_;
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

// Sort the m finished composites of task t by the output order, map indices
// and write the task's output row (padding slots m..k-1 with 0 / -1,
// src/algorithm.jl:358-365).  buf has room for max(next_pow2(m), m + 8K).
template <int THREADS>
__device__ void finish_task(const FusedParams& p, int t, const FusedTask& td, uint64_t* buf, uint32_t m,
                            FusedShared<THREADS>& sh) {
    const int tid = threadIdx.x;
    const uint32_t k = p.k;
    for (uint32_t i = tid; i < m; i += THREADS) {
        uint32_t pos = composite_pos(buf[i]);
        if (pos >= static_cast<uint64_t>(td.len)) {  // never expected; keep the gather in bounds
            record_error(p.err, kErrBounds);
            pos = 0;
        }
        uint32_t bits = __float_as_uint(p.data[td.start + pos]);
        buf[i] = output_sort_key(bits, pos, p.sp, p.ascend != 0);
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
        uint64_t* scratch = p.sort_scratch + static_cast<int64_t>(blockIdx.x) * k;
        uint32_t* wd = reinterpret_cast<uint32_t*>(buf + m);
        uint32_t* db = wd + (THREADS / 32) * 256;
        sorted = radix_sort_u64<THREADS>(buf, scratch, m, sh.bs, wd, db);
    }
    __syncthreads();
    float* vrow = p.val_out + static_cast<int64_t>(t) * k;
    for (uint32_t j = tid; j < k; j += THREADS) {
        float v = 0.0f;
        int64_t idx = -1;
        if (j < m) {
            uint32_t pos = static_cast<uint32_t>(sorted[j]);
            if (pos >= static_cast<uint64_t>(td.len)) pos = 0;  // bounded gather (error recorded above)
            int64_t g = td.start + pos;
            v = p.data[g];
            if (p.idx_in) {
                idx = (p.idx_bytes == 8) ? static_cast<const int64_t*>(p.idx_in)[g]
                                         : static_cast<int64_t>(static_cast<const int32_t*>(p.idx_in)[g]);
            } else {
                idx = static_cast<int64_t>(pos) + 1;  // 1-based position (filter.jl:76-77)
            }
        }
        vrow[j] = v;
        if (p.idx_bytes == 8) static_cast<int64_t*>(p.idx_out)[static_cast<int64_t>(t) * k + j] = idx;
        else static_cast<int32_t*>(p.idx_out)[static_cast<int64_t>(t) * k + j] = static_cast<int32_t>(idx);
    }
    __syncthreads();
}

// Reduce the shared buffer to its top k when it holds more; returns the k-th
// composite (0 when the buffer holds fewer than k entries).
template <int THREADS>
__device__ uint64_t shrink_to_k(const FusedParams& p, uint64_t* buf, FusedShared<THREADS>& sh) {
    uint32_t cnt = sh.cnt;
    if (cnt > p.cap) {  // entries beyond cap were dropped (error already recorded)
        cnt = p.cap;
        __syncthreads();
        if (threadIdx.x == 0) sh.cnt = cnt;
        __syncthreads();
    }
    uint64_t mn = 0;
    if (cnt > p.k) {
        mn = block_select_topk<THREADS>(buf, cnt, p.k, sh.bs, p.err);
        if (threadIdx.x == 0) sh.cnt = p.k;
        __syncthreads();
    } else if (cnt == p.k && cnt > 0) {
        uint64_t v = ~0ull;
        for (uint32_t i = threadIdx.x; i < cnt; i += THREADS) v = buf[i] < v ? buf[i] : v;
        mn = block_min_u64<THREADS>(v, sh.bs);
    }
    return mn;
}

template <int THREADS, int VEC, bool kScale>
__global__ void __launch_bounds__(THREADS, 2) fused_topk_kernel(FusedParams p) {
    extern __shared__ __align__(16) uint64_t s_buf[];
    __shared__ FusedShared<THREADS> sh;
    constexpr int U = VEC / 4;                      // float4 per thread per iteration
    constexpr uint32_t TILE = THREADS * VEC;        // elements per iteration
    const int tid = threadIdx.x;
    const uint32_t cap = p.cap;
    const uint32_t compact_at = cap - TILE - 8;     // host guarantees cap >= k + TILE + 8

    for (;;) {
        if (tid == 0) sh.work = static_cast<int32_t>(atomicAdd(p.work_counter, 1u));
        __syncthreads();
        const int w = sh.work;
        if (w >= p.nsegs) break;
        const FusedSeg sg = p.segs[w];
        const int t = sg.task;
        const FusedTask td = p.tasks[t];
        const bool multi = td.nseg > 1;
        const float scaler = kScale ? task_scaler(p.data, td.start, td.len, 1) : 0.0f;
        if (tid == 0) {
            sh.cnt = 0;
            sh.gthr = multi ? load_volatile_u64(p.gthr + t) : 0ull;
        }
        __syncthreads();
        uint64_t thr = sh.gthr;

        const int64_t s0 = sg.start, s1 = sg.start + sg.len;
        // Element g sits on a 16-byte boundary iff (g + mis) % 4 == 0.
        const int64_t mis = static_cast<int64_t>((reinterpret_cast<uintptr_t>(p.data) >> 2) & 3);
        int64_t a0 = ((s0 + mis + 3) & ~int64_t(3)) - mis;
        int64_t a1 = ((s1 + mis) & ~int64_t(3)) - mis;
        if (a0 > a1) { a0 = s1; a1 = s1; }   // no aligned body: everything is head
        // Head [s0, a0) and tail [a1, s1): fewer than 4 elements each.
        {
            const int nh = static_cast<int>(a0 - s0), nt = static_cast<int>(s1 - a1);
            bool pass = false;
            uint64_t c = 0;
            if (tid < 32) {
                int64_t g = -1;
                if (tid < nh) g = s0 + tid;
                else if (tid >= 8 && tid - 8 < nt) g = a1 + (tid - 8);
                if (g >= 0) {
                    uint32_t bits = __float_as_uint(p.data[g]);
                    c = make_composite(score_of<kScale>(bits, scaler, p.sp), static_cast<uint32_t>(g - td.start));
                    pass = c > thr;
                }
                warp_append(pass, c, s_buf, &sh.cnt, cap, p.err);
            }
        }
        // Aligned body with 128-bit loads, one iteration of prefetch.
        const int64_t nvec = (a1 - a0) >> 2;
        const float4* v4 = reinterpret_cast<const float4*>(p.data + a0);
        const uint32_t pos0 = static_cast<uint32_t>(a0 - td.start);
        const int64_t per_iter = static_cast<int64_t>(THREADS) * U;
        const int64_t niter = (nvec + per_iter - 1) / per_iter;
        float4 cur[U], nxt[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            int64_t q = static_cast<int64_t>(j) * THREADS + tid;
            cur[j] = (q < nvec) ? __ldcs(v4 + q) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        for (int64_t it = 0; it < niter; ++it) {
            const int64_t qb = it * per_iter;
            if (it + 1 < niter) {
#pragma unroll
                for (int j = 0; j < U; ++j) {
                    int64_t q = qb + per_iter + static_cast<int64_t>(j) * THREADS + tid;
                    nxt[j] = (q < nvec) ? __ldcs(v4 + q) : make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
            uint64_t gnew = 0;
            if (multi && tid == 0 && (it & 7) == 7) gnew = load_volatile_u64(p.gthr + t);
            // Filter this iteration's elements against the threshold.
            uint32_t pm = 0;
#pragma unroll
            for (int j = 0; j < U; ++j) {
                int64_t q = qb + static_cast<int64_t>(j) * THREADS + tid;
                if (q < nvec) {
                    const uint32_t pb = pos0 + static_cast<uint32_t>(q) * 4u;
                    const float f[4] = {cur[j].x, cur[j].y, cur[j].z, cur[j].w};
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        uint64_t c = make_composite(score_of<kScale>(__float_as_uint(f[e]), scaler, p.sp), pb + e);
                        pm |= (c > thr) ? (1u << (j * 4 + e)) : 0u;
                    }
                }
            }
            if (__any_sync(kFullMask, pm != 0)) {
#pragma unroll
                for (int j = 0; j < U; ++j) {
                    int64_t q = qb + static_cast<int64_t>(j) * THREADS + tid;
                    const uint32_t pb = pos0 + static_cast<uint32_t>(q) * 4u;
                    const float f[4] = {cur[j].x, cur[j].y, cur[j].z, cur[j].w};
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const bool ps = (pm >> (j * 4 + e)) & 1u;
                        uint64_t c = ps ? make_composite(score_of<kScale>(__float_as_uint(f[e]), scaler, p.sp), pb + e)
                                        : 0ull;
                        warp_append(ps, c, s_buf, &sh.cnt, cap, p.err);
                    }
                }
            }
            if (multi && tid == 0 && (it & 7) == 7 && gnew > sh.gthr) sh.gthr = gnew;
            // Snapshot the shared count between two barriers so that no thread
            // can read it after a faster one already appended to the next tile.
            __syncthreads();
            const uint32_t cnt_now = sh.cnt;
            const uint64_t g_now = sh.gthr;
            __syncthreads();
            if (cnt_now > compact_at) {
                uint64_t mn = shrink_to_k<THREADS>(p, s_buf, sh);
                if (multi && tid == 0 && mn != 0) atomicMax(reinterpret_cast<unsigned long long*>(p.gthr + t), mn);
                thr = mn > thr ? mn : thr;
            }
            if (multi) thr = g_now > thr ? g_now : thr;
#pragma unroll
            for (int j = 0; j < U; ++j) cur[j] = nxt[j];
        }
        __syncthreads();

        if (!multi) {
            shrink_to_k<THREADS>(p, s_buf, sh);
            const uint32_t m = sh.cnt;
            const uint32_t want = td.len < static_cast<int64_t>(p.k) ? static_cast<uint32_t>(td.len) : p.k;
            if (m != want && tid == 0) record_error(p.err, kErrInternal);
            finish_task<THREADS>(p, t, td, s_buf, m < want ? m : want, sh);
            continue;
        }

        // Multi-segment task: publish this segment's k-th composite, write the
        // survivors to the segment's candidate slot, count the segment done.
        uint64_t mn = shrink_to_k<THREADS>(p, s_buf, sh);
        if (tid == 0) {
            if (mn != 0) atomicMax(reinterpret_cast<unsigned long long*>(p.gthr + t), mn);
            sh.gthr = load_volatile_u64(p.gthr + t);
        }
        __syncthreads();
        {
            const uint64_t g = sh.gthr;
            const uint32_t cnt = sh.cnt;
            const int64_t slot = td.slot0 + sg.seg_in_task;
            uint64_t* dst = p.cand + slot * p.k;
            uint32_t out = 0;
            for (uint32_t base = 0; base < cnt; base += THREADS) {
                uint32_t i = base + tid;
                uint64_t c = (i < cnt) ? s_buf[i] : 0ull;
                bool keep = (i < cnt) && c >= g;
                uint32_t total;
                uint32_t off = block_exclusive_scan<THREADS>(keep ? 1u : 0u, &total, sh.bs);
                if (keep) {
                    if (out + off < p.k) dst[out + off] = c;
                    else record_error(p.err, kErrCapacity);
                }
                out += total;
            }
            if (tid == 0) p.slot_cnt[slot] = out < p.k ? out : p.k;
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
        if (tid == 0) { sh.cnt = 0; sh.gthr = load_volatile_u64(p.gthr + t); }
        __syncthreads();
        const uint64_t g = sh.gthr;
        for (int si = 0; si < td.nseg; ++si) {
            const int64_t slot = td.slot0 + si;
            const uint32_t n = __ldcg(p.slot_cnt + slot);
            const uint64_t* srcp = p.cand + slot * p.k;
            for (uint32_t base = 0; base < n; base += THREADS) {
                uint32_t i = base + tid;
                uint64_t c = (i < n) ? __ldcg(reinterpret_cast<const unsigned long long*>(srcp + i)) : 0ull;
                bool keep = (i < n) && c >= g;
                warp_append(keep, c, s_buf, &sh.cnt, cap, p.err);
                __syncthreads();
                const uint32_t cnt_now = sh.cnt;
                __syncthreads();
                if (cnt_now > compact_at) shrink_to_k<THREADS>(p, s_buf, sh);
            }
        }
        __syncthreads();
        shrink_to_k<THREADS>(p, s_buf, sh);
        const uint32_t m = sh.cnt;
        if (m != p.k && tid == 0) record_error(p.err, kErrInternal);
        finish_task<THREADS>(p, t, td, s_buf, m < p.k ? m : p.k, sh);
    }
}

}  // namespace radik
