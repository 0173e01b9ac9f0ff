// merge.cuh -- finish tasks whose segments ran in flush mode.
//
// In flush mode (fused_ws.cuh) every segment of a large sampled task wrote
// all its elements above the task's seeded threshold to the task's candidate
// region: a superset of the task's k best.  One block per such task selects
// the exact k best of the region:
//   * when the launch passes rank_ready (few tasks: the host's rank_pays),
//     the region fits in shared memory beside the select's scratch and
//     k <= kRankMaxK: the region is loaded at once and the k-th largest
//     composite is found with block_topk_bound (8-bit digit windows over
//     per-warp histograms narrow it to one bin, whose entries one warp then
//     bisects); the k selected entries are written back to the region as
//     output sort keys, and rank_write_kernel puts every one at its place in
//     the output row: its place is the number of the k keys below it,
//     counted by many blocks at once (k^2 compares spread over the GPU
//     instead of a sorting network on one SM);
//   * otherwise the region is loaded into shared memory (in chunks, keeping a
//     few more than k with block_shrink whenever the buffer fills), selected
//     with block_select_topk, sorted and written by this block.
// If fewer than k candidates exist (the sampled threshold was above the
// task's k-th composite) or the region overflowed, the task is flagged and
// the retry launch recomputes it without the sample.
#pragma once

#include "fused.cuh"

namespace radik {

constexpr uint32_t kRankMaxK = 8192;   // largest k whose row rank_write_kernel writes
constexpr int kRankThreads = 256;      // rank_write_kernel: threads per block
constexpr int kRankSplit = 16;         // threads counting for one output key
constexpr int kRankPerBlock = kRankThreads / kRankSplit;  // output keys placed per block

template <int THREADS, bool kScale>
__global__ void __launch_bounds__(THREADS) merge_topk_kernel(FusedParams p, const int32_t* merge_tasks) {
    grid_dep_wait();  // launched after the streaming kernel
    extern __shared__ __align__(16) uint64_t s_buf[];
    __shared__ FusedShared<THREADS> sh;
    __shared__ uint32_t s_spill_n;        // block_topk_bound: entries of the boundary bin
    __shared__ unsigned long long s_tau;  // ... and the bound warp 0 found
    const int tid = threadIdx.x;
    const int t = merge_tasks[blockIdx.x];
    // The task's flag, descriptor and candidate count, loaded together.
    const uint32_t failed = __ldcg(p.fail + t);
    const FusedTask td = p.tasks[t];
    const uint32_t have = __ldcg(p.task_cnt + t);
    if (failed != 0u) return;  // the retry launch redoes it
    const TaskView tv = task_view<kScale>(p, t, td);
    const uint32_t k = tv.k;
    const uint32_t cap = p.cap;
    const uint32_t region = static_cast<uint32_t>(td.nseg) * p.kmax;
    const uint32_t n = have < region ? have : region;
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(p.cand + td.cbase);
    // Room kept free while streaming chunks: a shrink keeps at most mid_keep.
    const uint32_t mid_keep = k + (cap - k) / 4;
    if (tid == 0) sh.cnt = 0;
    block_sync<THREADS>();
    // Shared memory of the usual case: the region, then per-warp histograms
    // (256 words per warp), then the boundary bin.
    const uint32_t hist_off = (n + 1) & ~1u;
    const uint32_t spill_off = hist_off + (THREADS / 32) * 256 / 2;
    if (p.rank_ready != nullptr && spill_off + kWarpBisect <= cap && hist_off + k <= cap && k <= kRankMaxK &&
        k <= region) {
        if (n < k) {  // fewer than k candidates: the sampled threshold was too high
            if (tid == 0) {
                p.fail[t] = 1u;
                atomicExch(p.fail_any, 1u);
            }
            return;
        }
        uint64_t vor = 0, vand = ~0ull;
#pragma unroll 8
        for (uint32_t i = tid; i < n; i += THREADS) {
            const uint64_t c = __ldcg(src + i);
            s_buf[i] = c;
            vor |= c;
            vand &= c;
        }
        block_or_and<THREADS>(vor, vand, sh.bs);  // barriers: the region is in s_buf
        const uint64_t tau = block_topk_bound<THREADS>(s_buf, n, k, vor, vand, sh.bs,
                                                       reinterpret_cast<uint32_t*>(s_buf + hist_off),
                                                       s_buf + spill_off, &s_spill_n, &s_tau, p.err);
        // The k selected entries go back to the region as output sort keys:
        // slots from a block-wide scan of every thread's count, staged in
        // shared memory (after the histograms) and copied out coalesced.
        uint64_t* dst = p.cand + td.cbase;
        uint64_t* stage = s_buf + hist_off;  // k <= cap - hist_off entries (checked below)
        uint32_t nsel = 0;
        for (uint32_t i = tid; i < n; i += THREADS) nsel += (s_buf[i] >= tau) ? 1u : 0u;
        uint32_t total = 0;
        uint32_t slot = block_exclusive_scan<THREADS>(nsel, &total, sh.bs);  // barriers: histograms no longer read
        for (uint32_t i = tid; i < n; i += THREADS) {
            const uint64_t c = s_buf[i];
            if (c < tau) continue;
            uint32_t pos = composite_pos(c);
            if (pos >= static_cast<uint64_t>(tv.len)) {  // never expected; keep the gather in bounds
                record_error(p.err, kErrBounds);
                pos = 0;
            }
            uint64_t okey;
            if constexpr (kScale) {
                okey = output_sort_key(__float_as_uint(tv.data[pos]), pos, tv.sp, tv.ascend);
            } else {
                uint32_t key = static_cast<uint32_t>(c >> 32) ^ tv.sp.flip;  // key of the substituted value
                if (!tv.ascend) key = ~key;
                okey = (static_cast<uint64_t>(key) << 32) | pos;
            }
            if (slot < k) stage[slot] = okey;
            else record_error(p.err, kErrInternal);
            ++slot;
        }
        block_sync<THREADS>();
        for (uint32_t i = tid; i < k; i += THREADS) dst[i] = stage[i];
        if (tid == 0) {
            if (total == k) p.rank_ready[t] = 1u;
            else record_error(p.err, kErrInternal);
        }
        return;
    }
    if (n >= k && spill_off + kWarpBisect <= cap && hist_off + k <= cap) {
        // The region fits beside the select's scratch: load it at once, find
        // the k-th largest composite (block_topk_bound), gather the k entries
        // at or above it in the staging area behind the histograms, move them
        // to the front and sort and write them (finish_task).
        uint64_t vor = 0, vand = ~0ull;
#pragma unroll 8
        for (uint32_t i = tid; i < n; i += THREADS) {
            const uint64_t c = __ldcg(src + i);
            s_buf[i] = c;
            vor |= c;
            vand &= c;
        }
        block_or_and<THREADS>(vor, vand, sh.bs);  // barriers: the region is in s_buf
        const uint64_t tau = block_topk_bound<THREADS>(s_buf, n, k, vor, vand, sh.bs,
                                                       reinterpret_cast<uint32_t*>(s_buf + hist_off),
                                                       s_buf + spill_off, &s_spill_n, &s_tau, p.err);
        uint64_t* stage = s_buf + hist_off;  // [hist_off, hist_off + k) does not meet [0, k): k <= n < hist_off
        uint32_t nsel = 0;
        for (uint32_t i = tid; i < n; i += THREADS) nsel += (s_buf[i] >= tau) ? 1u : 0u;
        uint32_t total = 0;
        uint32_t slot = block_exclusive_scan<THREADS>(nsel, &total, sh.bs);  // barriers: histograms no longer read
        for (uint32_t i = tid; i < n; i += THREADS) {
            const uint64_t c = s_buf[i];
            if (c < tau) continue;
            if (slot < k) stage[slot] = c;
            else record_error(p.err, kErrInternal);
            ++slot;
        }
        block_sync<THREADS>();
        for (uint32_t i = tid; i < k; i += THREADS) s_buf[i] = stage[i];
        if (tid == 0 && total != k) record_error(p.err, kErrInternal);
        block_sync<THREADS>();
        finish_task<THREADS, !kScale>(p, tv, s_buf, k, sh);
        return;
    }
    for (uint32_t b0 = 0; b0 < n;) {
        const uint32_t cnt = sh.cnt;
        const uint32_t take = min(n - b0, cap - cnt);  // > 0: cnt <= mid_keep < cap
        // Independent loads, several per thread in flight.
#pragma unroll 4
        for (uint32_t i = tid; i < take; i += THREADS) s_buf[cnt + i] = __ldcg(src + b0 + i);
        b0 += take;
        block_sync<THREADS>();
        if (tid == 0) sh.cnt = cnt + take;
        block_sync<THREADS>();
        if (b0 < n) shrink_mid<THREADS>(p, k, mid_keep, s_buf, sh);
    }
    uint64_t kth = 0;
    const uint32_t m = shrink_final<THREADS>(p, k, s_buf, sh, &kth);
    if (m < k) {
        if (tid == 0) {
            p.fail[t] = 1u;
            atomicExch(p.fail_any, 1u);
        }
        return;
    }
    finish_task<THREADS, !kScale>(p, tv, s_buf, k, sh);
}

// Output rows of the tasks whose k selected output keys merge_topk_kernel
// left in their candidate regions: block (x, y) places keys
// x * kRankPerBlock .. (x + 1) * kRankPerBlock - 1 of task merge_tasks[y].  A key's place in the row is the
// number of the task's k keys below it (keys are unique); kRankSplit threads
// count it over interleaved pairs of keys in shared memory and the first
// writes the value and index there.
template <bool kScale>
__global__ void __launch_bounds__(kRankThreads) rank_write_kernel(FusedParams p, const int32_t* merge_tasks) {
    grid_dep_wait();  // launched after the merge kernel
    extern __shared__ __align__(16) uint64_t s_keys[];
    const int tid = threadIdx.x;
    const int t = merge_tasks[blockIdx.y];
    const uint32_t ready = __ldcg(p.rank_ready + t);
    const FusedTask td = p.tasks[t];
    if (ready == 0u) return;
    const TaskView tv = task_view<kScale>(p, t, td);
    const uint32_t k = tv.k;
    const uint32_t q0 = blockIdx.x * kRankPerBlock;
    if (q0 >= k || k > kRankMaxK) return;
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(p.cand + td.cbase);
    const uint32_t k2 = (k + 1) & ~1u;  // an even count: a padding key ~0 ranks above every real key
    for (uint32_t i = tid; i < k2; i += kRankThreads) s_keys[i] = i < k ? __ldcg(src + i) : ~0ull;
    __syncthreads();
    const uint32_t q = q0 + static_cast<uint32_t>(tid) / kRankSplit;
    const uint32_t part = static_cast<uint32_t>(tid) % kRankSplit;
    const uint64_t x = q < k ? s_keys[q] : ~0ull;
    const ulonglong2* pairs = reinterpret_cast<const ulonglong2*>(s_keys);
    uint32_t c0 = 0, c1 = 0;
    // Pairs part, part + kRankSplit, ...: the threads of a key read
    // consecutive bytes, and the other key of the warp reads the same ones.
#pragma unroll 4
    for (uint32_t i = part; i < k2 / 2; i += kRankSplit) {
        const ulonglong2 y = pairs[i];
        c0 += (y.x < x) ? 1u : 0u;
        c1 += (y.y < x) ? 1u : 0u;
    }
    uint32_t c = c0 + c1;
#pragma unroll
    for (int m = 1; m < kRankSplit; m <<= 1) c += __shfl_xor_sync(kFullMask, c, m);
    if (part != 0u || q >= k) return;
    if (c >= k) {  // never expected: keys are unique
        record_error(p.err, kErrInternal);
        return;
    }
    const uint32_t pos = static_cast<uint32_t>(x);
    float val;
    if constexpr (kScale) {
        val = tv.data[pos];
    } else {
        uint32_t key = static_cast<uint32_t>(x >> 32);
        if (!tv.ascend) key = ~key;
        val = (key == key_of_bits(tv.sp.nan_bits)) ? tv.data[pos]
                                                   : __uint_as_float((key & 0x80000000u) ? (key ^ 0x80000000u) : ~key);
    }
    int64_t idx;
    if (tv.iin) {
        idx = (p.idx_bytes == 8) ? static_cast<const int64_t*>(tv.iin)[pos]
                                 : static_cast<int64_t>(static_cast<const int32_t*>(tv.iin)[pos]);
    } else {
        idx = static_cast<int64_t>(pos) + 1;  // 1-based position (filter.jl:76-77)
    }
    tv.vout[c] = val;
    if (p.idx_bytes == 8) static_cast<int64_t*>(tv.iout)[c] = idx;
    else static_cast<int32_t*>(tv.iout)[c] = static_cast<int32_t>(idx);
}

}  // namespace radik
