// sample.cuh -- seed the global threshold of a large task from a sample.
//
// A task split into many segments with a large k cannot be pruned by the
// segments' own k-th values: a segment's k-th best is far below the task's.
// Before the fused kernel runs, each such task is sampled by `njobs` CTAs:
// every CTA reads `nchunks` chunks of kSampleChunk contiguous elements spread
// over the task (16-byte aligned, so as float4), reduces every 4 consecutive
// samples to their best score (a group maximum) and keeps the exact top r of
// its groups; the last CTA of the task (atomic counter, no waiting) takes the
// lower edge of the digit bin holding the r-th best of the union, rounded
// down to a whole score, and stores it, minus one, as the task's exclusive
// global threshold.  At least r groups, hence r sampled elements, score at
// or above it, so about r * len / samples elements of the task lie above it;
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
    int32_t r;           // sample rank (from the best) of the threshold, <= 256 (njobs * r <= 8192)
    int32_t nchunks;     // chunks per CTA (1 to 8)
    int32_t pad_;
    int64_t pos0;        // position (inside the task) of this CTA's first chunk
    int64_t stride;      // distance between consecutive chunks (a multiple of 4)
    int64_t out_base;    // first of the task's njobs * r slots in the sample buffer
};

template <int THREADS, bool kScale>
__global__ void __launch_bounds__(THREADS) sample_threshold_kernel(FusedParams p, const SampleJob* jobs,
                                                                    uint64_t* sample_out, uint32_t* sample_done) {
    grid_dep_wait();  // launched after the state is cleared
    grid_dep_launch();
    extern __shared__ __align__(16) uint64_t s_buf[];
    __shared__ FusedShared<THREADS> sh;
    constexpr uint32_t kChunk4 = kSampleChunk / 4;  // float4 per chunk
    const int tid = threadIdx.x;
    const SampleJob job = jobs[blockIdx.x];
    const int t = job.task;
    const FusedTask td = p.tasks[t];
    const TaskView tv = task_view<kScale>(p, t, td);
    const float scaler = kScale ? task_scaler(tv.data, 0, tv.len, 1) : 0.0f;
    // Chunks start at 16-byte boundaries: positions move up by the task
    // pointer's misalignment (the host leaves room for it).
    const int64_t mis = static_cast<int64_t>((reinterpret_cast<uintptr_t>(tv.data) >> 2) & 3);
    const int64_t shift = (4 - mis) & 3;
    const uint32_t ngroups = static_cast<uint32_t>(job.nchunks) * kChunk4;
    uint64_t vor = 0, vand = ~0ull;
    for (uint32_t gi = tid; gi < ngroups; gi += THREADS) {
        const uint32_t c = gi / kChunk4, e = gi % kChunk4;
        int64_t q = job.pos0 + static_cast<int64_t>(c) * job.stride + shift + 4 * static_cast<int64_t>(e);
        if (q + 4 > tv.len) {  // the host keeps chunks inside the task
            record_error(p.err, kErrBounds);
            q = shift;
        }
        const float4 f = *reinterpret_cast<const float4*>(tv.data + q);  // (q + mis) % 4 == 0
        const uint32_t a = score_of<kScale>(__float_as_uint(f.x), scaler, tv.sp);
        const uint32_t b = score_of<kScale>(__float_as_uint(f.y), scaler, tv.sp);
        const uint32_t cc = score_of<kScale>(__float_as_uint(f.z), scaler, tv.sp);
        const uint32_t d = score_of<kScale>(__float_as_uint(f.w), scaler, tv.sp);
        // Unique composite: best score of the group, then the group's number.
        const uint64_t g = (static_cast<uint64_t>(max(max(a, b), max(cc, d))) << 32) |
                           (static_cast<uint32_t>(job.job_in_task) * ngroups + gi);
        s_buf[gi] = g;
        vor |= g;
        vand &= g;
    }
    block_or_and<THREADS>(vor, vand, sh.bs);  // barriers: the groups are in s_buf
    const uint32_t r = static_cast<uint32_t>(job.r);
    uint64_t kf = 0, mn = 0;
    const uint32_t kept = block_shrink<THREADS>(s_buf, ngroups, r, r, vand, vor, sh.bs, p.err, &kf, &mn);
    uint64_t* out = sample_out + job.out_base + static_cast<int64_t>(job.job_in_task) * r;
    for (uint32_t i = tid; i < r; i += THREADS) out[i] = (i < kept) ? s_buf[i] : 0ull;
    __threadfence();
    block_sync<THREADS>();
    if (tid == 0) sh.last = (atomicAdd(sample_done + t, 1u) == static_cast<uint32_t>(job.njobs - 1)) ? 1u : 0u;
    block_sync<THREADS>();
    if (!sh.last) return;
    __threadfence();
    const uint32_t nall = static_cast<uint32_t>(job.njobs) * r;
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(sample_out + job.out_base);
    vor = 0;
    vand = ~0ull;
    for (uint32_t i = tid; i < nall; i += THREADS) {
        const uint64_t g = __ldcg(src + i);
        s_buf[i] = g;
        vor |= g;
        vand &= g;
    }
    block_or_and<THREADS>(vor, vand, sh.bs);
    // Zero entries (CTAs with fewer than r groups) never rank above a real
    // group, whose composite is > 0.  The lower edge of the bin of rank r is
    // rounded down to its score: every element at or above that score passes.
    const uint64_t edge = block_rank_threshold<THREADS>(s_buf, nall, r, 4 * r, vand, vor, sh.bs);
    const uint64_t score = edge >> 32;
    if (tid == 0 && score > 0)
        atomicMax(reinterpret_cast<unsigned long long*>(p.gthr + t), static_cast<unsigned long long>((score << 32) - 1));
}

// One block per sampled task when the whole sample fits one block (at most
// kSampleOneMaxChunks chunks, 8192 group maxima, 8 per thread): the block
// reads every chunk of the task (the same chunks as above, job.nchunks of
// them at job.stride), keeps the group maxima's scores in registers and finds
// the threshold with per-warp histograms of 8-bit windows below the scores'
// common prefix: the lower edge of the bin holding the r-th best score, once
// that bin and the bins above it hold at most r + r/2 maxima (or no bits are
// left).  At least r maxima score at or above it.  No sample buffer, no
// atomics between blocks, no last-block merge.
constexpr int kSampleOneThreads = 1024;
constexpr int kSampleOneMaxChunks = 64;

template <bool kScale>
__global__ void __launch_bounds__(kSampleOneThreads) sample_one_kernel(FusedParams p, const SampleJob* jobs) {
    grid_dep_wait();  // launched after the state is cleared
    grid_dep_launch();
    constexpr int THREADS = kSampleOneThreads;
    constexpr int NW = THREADS / 32;
    constexpr uint32_t kChunk4 = kSampleChunk / 4;                        // groups per chunk
    constexpr int G = kSampleOneMaxChunks * static_cast<int>(kChunk4) / THREADS;  // groups per thread
    __shared__ uint32_t whist[NW][256];
    __shared__ uint32_t tot[256];
    __shared__ uint32_t red[2][NW];
    __shared__ uint32_t res[3];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const SampleJob job = jobs[blockIdx.x];
    const int t = job.task;
    const FusedTask td = p.tasks[t];
    const TaskView tv = task_view<kScale>(p, t, td);
    const float scaler = kScale ? task_scaler(tv.data, 0, tv.len, 1) : 0.0f;
    const int64_t mis = static_cast<int64_t>((reinterpret_cast<uintptr_t>(tv.data) >> 2) & 3);
    const int64_t shift = (4 - mis) & 3;
    const uint32_t nchunks = job.nchunks < kSampleOneMaxChunks ? static_cast<uint32_t>(job.nchunks)
                                                               : static_cast<uint32_t>(kSampleOneMaxChunks);
    const uint32_t ngroups = nchunks * kChunk4;
    float4 f[G];
#pragma unroll
    for (int j = 0; j < G; ++j) {
        const uint32_t gi = static_cast<uint32_t>(j) * THREADS + tid;
        int64_t q = job.pos0 + static_cast<int64_t>(gi / kChunk4) * job.stride + shift + 4 * static_cast<int64_t>(gi % kChunk4);
        if (gi < ngroups && q + 4 > tv.len) {  // the host keeps chunks inside the task
            record_error(p.err, kErrBounds);
            q = shift;
        }
        f[j] = gi < ngroups ? *reinterpret_cast<const float4*>(tv.data + q) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    uint32_t g[G];
    uint32_t vor = 0u, vand = ~0u;
#pragma unroll
    for (int j = 0; j < G; ++j) {
        const uint32_t a = score_of<kScale>(__float_as_uint(f[j].x), scaler, tv.sp);
        const uint32_t b = score_of<kScale>(__float_as_uint(f[j].y), scaler, tv.sp);
        const uint32_t c = score_of<kScale>(__float_as_uint(f[j].z), scaler, tv.sp);
        const uint32_t d = score_of<kScale>(__float_as_uint(f[j].w), scaler, tv.sp);
        g[j] = max(max(a, b), max(c, d));
        if (static_cast<uint32_t>(j) * THREADS + tid < ngroups) {
            vor |= g[j];
            vand &= g[j];
        }
    }
    vor = __reduce_or_sync(kFullMask, vor);
    vand = __reduce_and_sync(kFullMask, vand);
    if (lane == 0) {
        red[0][warp] = vor;
        red[1][warp] = vand;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) (&whist[0][0])[i * THREADS + tid] = 0u;
    __syncthreads();
    vor = 0u;
    vand = ~0u;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        vor |= red[0][w];
        vand &= red[1][w];
    }
    const uint32_t r0 = static_cast<uint32_t>(job.r);
    const uint32_t slack = r0 / 2;
    uint32_t T = vand;  // every maximum is >= vand
    const uint32_t diff = vor ^ vand;
    if (diff != 0u && r0 >= 1u && r0 <= ngroups) {
        int top = 31 - __clz(diff);
        uint32_t prefix = top >= 31 ? 0u : (vand & ~((2u << top) - 1u));  // bits above top, shared by all
        uint32_t r = r0, above_total = 0;
        for (int pass = 0; pass < 4; ++pass) {
            const int w = top + 1 < 8 ? top + 1 : 8;
            const int sh = top + 1 - w;
            const uint32_t nb = 1u << w;
            const uint32_t hmask = (top >= 31) ? 0u : ~((2u << top) - 1u);
#pragma unroll
            for (int j = 0; j < G; ++j) {
                const bool in = static_cast<uint32_t>(j) * THREADS + tid < ngroups && (g[j] & hmask) == prefix;
                if (in) atomicAdd(&whist[warp][(g[j] >> sh) & (nb - 1u)], 1u);
            }
            __syncthreads();
            uint32_t sb = 0;
            if (tid < nb) {
#pragma unroll 8
                for (int ww = 0; ww < NW; ++ww) sb += whist[ww][tid];
            }
            __syncthreads();  // every warp histogram read: clear them for the next window
#pragma unroll
            for (int i = 0; i < 8; ++i) (&whist[0][0])[i * THREADS + tid] = 0u;
            if (tid < nb) tot[tid] = sb;
            __syncthreads();
            if (warp == 0) {
                // Bins from the top, 8 per lane: the bin holding rank r.
                uint32_t h[8], sum = 0;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const uint32_t rb = lane * 8u + static_cast<uint32_t>(j);
                    h[j] = rb < nb ? tot[nb - 1u - rb] : 0u;
                    sum += h[j];
                }
                uint32_t run = warp_inclusive_scan<true>(sum) - sum;
                uint32_t hit = 0u, hb = 0, habove = 0, hcnt = 0;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const uint32_t rb = lane * 8u + static_cast<uint32_t>(j);
                    if (rb < nb && run < r && run + h[j] >= r) {
                        hit = 1u;
                        hb = nb - 1u - rb;
                        habove = run;
                        hcnt = h[j];
                    }
                    run += h[j];
                }
                const uint32_t who = __ballot_sync(kFullMask, hit != 0u);
                if (who != 0u) {
                    const uint32_t src = __ffs(who) - 1u;
                    hb = __shfl_sync(kFullMask, hb, src);
                    habove = __shfl_sync(kFullMask, habove, src);
                    hcnt = __shfl_sync(kFullMask, hcnt, src);
                } else {
                    hb = 0xffffffffu;  // rank r beyond the entries in play: never expected
                }
                if (lane == 0) {
                    res[0] = hb;
                    res[1] = habove;
                    res[2] = hcnt;
                }
            }
            __syncthreads();
            const uint32_t hb = res[0], habove = res[1], hcnt = res[2];
            if (hb == 0xffffffffu) {
                if (tid == 0) record_error(p.err, kErrInternal);
                T = 0u;
                break;
            }
            prefix |= hb << sh;
            T = prefix;
            above_total += habove;
            if (above_total + hcnt <= r0 + slack || sh == 0) break;
            r -= habove;
            top = sh - 1;
        }
    }
    if (tid == 0 && T > 0u)
        atomicMax(reinterpret_cast<unsigned long long*>(p.gthr + t), (static_cast<unsigned long long>(T) << 32) - 1ull);
}

}  // namespace radik
