// merge.cuh -- finish tasks whose segments ran in flush mode.
//
// In flush mode (fused_ws.cuh) every segment of a large sampled task wrote
// all its elements above the task's seeded threshold to the task's candidate
// region: a superset of the task's k best.  One block per such task loads the
// region into shared memory (all of it when it fits, which the host sizes for;
// otherwise in chunks, keeping a few more than k with block_shrink whenever
// the buffer fills), selects the exact k best, sorts them and writes the
// task's row.  If fewer than k candidates exist (the sampled threshold was
// above the task's k-th composite) or the region overflowed, the task is
// flagged and the retry launch recomputes it without the sample.
#pragma once

#include "fused.cuh"

namespace radik {

template <int THREADS, bool kScale>
__global__ void __launch_bounds__(THREADS) merge_topk_kernel(FusedParams p, const int32_t* merge_tasks) {
    extern __shared__ __align__(16) uint64_t s_buf[];
    __shared__ FusedShared<THREADS> sh;
    const int tid = threadIdx.x;
    const int t = merge_tasks[blockIdx.x];
    if (*reinterpret_cast<volatile const uint32_t*>(p.fail + t) != 0u) return;  // the retry launch redoes it
    const FusedTask td = p.tasks[t];
    const TaskView tv = task_view<kScale>(p, t, td);
    const uint32_t k = tv.k;
    const uint32_t cap = p.cap;
    const uint32_t region = static_cast<uint32_t>(td.nseg) * p.kmax;
    const uint32_t have = *reinterpret_cast<volatile const uint32_t*>(p.task_cnt + t);
    const uint32_t n = have < region ? have : region;
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(p.cand + td.cbase);
    // Room kept free while streaming chunks: a shrink keeps at most mid_keep.
    const uint32_t mid_keep = k + (cap - k) / 4;
    if (tid == 0) sh.cnt = 0;
    block_sync<THREADS>();
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

}  // namespace radik
