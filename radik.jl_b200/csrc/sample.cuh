// sample.cuh -- seed the global threshold of a large task from a sample.
//
// A task split into many segments with a large k cannot be pruned by the
// segments' own k-th values: a segment's k-th best is far below the task's.
// Before the fused kernel runs, each such task is sampled by `njobs` CTAs:
// every CTA reads `nchunks` chunks of kSampleChunk contiguous elements spread
// over the task and keeps the exact top r of its sample (block_select_topk);
// the last CTA of the task (atomic counter, no waiting) takes the exact r-th
// best of the union and stores it, minus one, as the task's exclusive global
// threshold.  About r * len / sample_size elements of the task lie above it;
// r is chosen on the host so that this count exceeds k with a wide margin.
// The fused kernel verifies the count; a task whose seeded threshold was too
// high is recomputed without it (retry launch).
#pragma once

#include "fused.cuh"

namespace radik {

constexpr int kSampleChunk = 512;

struct SampleJob {
    int32_t task;
    int32_t job_in_task;
    int32_t njobs;       // CTAs sampling this task
    int32_t r;           // sample rank (from the best) of the threshold, <= 64
    int32_t nchunks;     // chunks per CTA
    int32_t pad_;
    int64_t pos0;        // position (inside the task) of this CTA's first chunk
    int64_t stride;      // distance between consecutive chunks
    int64_t out_base;    // first of the task's njobs * r slots in the sample buffer
};

template <int THREADS, bool kScale>
__global__ void __launch_bounds__(THREADS) sample_threshold_kernel(FusedParams p, const SampleJob* jobs,
                                                                    uint64_t* sample_out, uint32_t* sample_done) {
    extern __shared__ __align__(16) uint64_t s_buf[];
    __shared__ FusedShared<THREADS> sh;
    const int tid = threadIdx.x;
    const SampleJob job = jobs[blockIdx.x];
    const int t = job.task;
    const FusedTask td = p.tasks[t];
    const TaskView tv = task_view<kScale>(p, t, td);
    const float scaler = kScale ? task_scaler(tv.data, 0, tv.len, 1) : 0.0f;
    const uint32_t ns = static_cast<uint32_t>(job.nchunks) * kSampleChunk;
    for (uint32_t i = tid; i < ns; i += THREADS) {
        int64_t q = job.pos0 + static_cast<int64_t>(i / kSampleChunk) * job.stride + (i % kSampleChunk);
        if (q >= tv.len) {  // the host keeps chunks inside the task
            record_error(p.err, kErrBounds);
            q = 0;
        }
        uint32_t bits = __float_as_uint(tv.data[q]);
        s_buf[i] = make_composite(score_of<kScale>(bits, scaler, tv.sp), static_cast<uint32_t>(q));
    }
    __syncthreads();
    const uint32_t r = static_cast<uint32_t>(job.r);
    uint64_t kth = 0;
    uint32_t kept = block_select_topk<THREADS>(s_buf, ns, r, sh.bs, p.err, &kth);
    uint64_t* out = sample_out + job.out_base + static_cast<int64_t>(job.job_in_task) * r;
    for (uint32_t i = tid; i < r; i += THREADS) out[i] = (i < kept) ? s_buf[i] : 0ull;
    __threadfence();
    __syncthreads();
    if (tid == 0) sh.last = (atomicAdd(sample_done + t, 1u) == static_cast<uint32_t>(job.njobs - 1)) ? 1u : 0u;
    __syncthreads();
    if (!sh.last) return;
    __threadfence();
    const uint32_t nall = static_cast<uint32_t>(job.njobs) * r;
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(sample_out + job.out_base);
    for (uint32_t i = tid; i < nall; i += THREADS) s_buf[i] = __ldcg(src + i);
    __syncthreads();
    // Zero entries (sample CTAs with fewer than r values) never rank above a
    // real composite, which is always > 0.
    kept = block_select_topk<THREADS>(s_buf, nall, r, sh.bs, p.err, &kth);
    if (tid == 0 && kept >= r && kth > 1)
        atomicMax(reinterpret_cast<unsigned long long*>(p.gthr + t), static_cast<unsigned long long>(kth - 1));
}

}  // namespace radik
