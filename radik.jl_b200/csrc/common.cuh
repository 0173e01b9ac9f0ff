// common.cuh -- shared device definitions for the RadiK B200 top-k engine.
//
// Ordering model.  Every Float32 maps to an order-preserving uint32 key
// (RadiK.jl src/utils.jl:29-33).  NaN is replaced by the reference's
// substitute before keying (src/utils.jl:68-71: floatmin when selecting the
// largest, floatmax when selecting the smallest) and optionally shifted by the
// task's scaler (WITHSCALE, src/utils.jl:62-71).  The engine always selects the
// LARGEST "score": score = key for largest=true, score = ~key otherwise, so
// every kernel runs in one direction.  Each element of a task also carries a
// unique 64-bit "composite" = score << 32 | ~pos (pos = 0-based position in
// the task): the top-k composites are the top-k scores with ties at the k-th
// score resolved towards the lowest positions, which makes the selection
// deterministic (the reference resolves those ties by an atomic race,
// src/kernels/filter.jl:115-118).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace radik {

constexpr uint32_t kFullMask = 0xffffffffu;

// Device-side error word bits (host reads them after a synchronous call).
enum : uint32_t {
    kErrCapacity = 1u << 0,   // a bounded buffer would have overflowed; write skipped
    kErrBounds = 1u << 1,     // an index fell outside its buffer; access skipped
    kErrTimeout = 1u << 2,    // a bounded wait gave up
    kErrInternal = 1u << 3,   // an invariant of the selection did not hold
};

__device__ __forceinline__ uint32_t key_of_bits(uint32_t b) {
    // src/utils.jl:29-33 -- sign set: ~b ; sign clear: b | 0x80000000
    return b ^ (static_cast<uint32_t>(static_cast<int32_t>(b) >> 31) | 0x80000000u);
}

// The Float32 whose key is `key` (inverse of key_of_bits).
__device__ __forceinline__ float value_of_key(uint32_t key) {
    return __uint_as_float((key & 0x80000000u) ? (key ^ 0x80000000u) : ~key);
}

__device__ __forceinline__ bool is_nan_bits(uint32_t b) { return (b & 0x7fffffffu) > 0x7f800000u; }

// Score parameters of one call (same for all tasks).
struct ScoreParams {
    uint32_t flip;      // 0 when selecting the largest, 0xffffffff for the smallest
    uint32_t nan_bits;  // bit pattern of the NaN substitute (floatmin or floatmax)
    uint32_t nan_score; // score of the NaN substitute without scaling
    int withscale;
};

__host__ __device__ inline ScoreParams make_score_params(bool largest, bool withscale) {
    ScoreParams p;
    p.flip = largest ? 0u : 0xffffffffu;
    p.nan_bits = largest ? 0x00800000u : 0x7f7fffffu;  // FLT_MIN / FLT_MAX
    uint32_t b = p.nan_bits;
    uint32_t key = b ^ ((b >> 31) ? 0xffffffffu : 0x80000000u);
    p.nan_score = key ^ p.flip;
    p.withscale = withscale ? 1 : 0;
    return p;
}

// Score of one element (no scaling).
__device__ __forceinline__ uint32_t score_noscale(uint32_t bits, const ScoreParams& p) {
    uint32_t s = key_of_bits(bits) ^ p.flip;
    return is_nan_bits(bits) ? p.nan_score : s;
}

// Score of one element with the task scaler (src/utils.jl:68-71).
__device__ __forceinline__ uint32_t score_scaled(uint32_t bits, float scaler, const ScoreParams& p) {
    uint32_t b = is_nan_bits(bits) ? p.nan_bits : bits;
    float v = __fsub_rn(__uint_as_float(b), scaler);
    return key_of_bits(__float_as_uint(v)) ^ p.flip;
}

template <bool kScale>
__device__ __forceinline__ uint32_t score_of(uint32_t bits, float scaler, const ScoreParams& p) {
    if constexpr (kScale) return score_scaled(bits, scaler, p);
    else return score_noscale(bits, p);
}

// Scaler of a task: its first element, 0 when NaN/Inf (src/utils.jl:62-66).
__device__ __forceinline__ float task_scaler(const float* data, int64_t start, int64_t len, int withscale) {
    if (!withscale || len <= 0) return 0.0f;
    float s = data[start];
    uint32_t b = __float_as_uint(s);
    return ((b & 0x7f800000u) == 0x7f800000u) ? 0.0f : s;
}

__device__ __forceinline__ uint64_t make_composite(uint32_t score, uint32_t pos) {
    return (static_cast<uint64_t>(score) << 32) | static_cast<uint32_t>(~pos);
}
__device__ __forceinline__ uint32_t composite_pos(uint64_t c) { return ~static_cast<uint32_t>(c); }

// Output sort key: ascending order of the (NaN-substituted) value key when
// ascend, descending otherwise; equal keys by ascending position
// (src/algorithm.jl:340-352 sorts val_out with rev = !ASCEND).
__device__ __forceinline__ uint64_t output_sort_key(uint32_t value_bits, uint32_t pos, const ScoreParams& p,
                                                    bool ascend) {
    uint32_t b = is_nan_bits(value_bits) ? p.nan_bits : value_bits;
    uint32_t k = key_of_bits(b);
    if (!ascend) k = ~k;
    return (static_cast<uint64_t>(k) << 32) | pos;
}

// ---------------------------------------------------------------------------
// Work descriptors (built on the host by a plan, read by the kernels)
// ---------------------------------------------------------------------------
struct TaskDesc {
    int64_t start;      // global offset of the task's first element
    int64_t len;        // number of elements
    int64_t cand_base;  // first candidate slot of the task (multi-segment tasks)
    int32_t nseg;       // number of segments
    int32_t first_seg;  // index of its first segment in the segment table
};

struct SegDesc {
    int64_t start;      // global offset of the segment's first element
    int32_t len;        // elements in the segment
    int32_t task;       // task index
    int32_t seg_in_task;
    int32_t pad_;
};

// ---------------------------------------------------------------------------
// Warp / block helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Inclusive warp scan (Hillis-Steele over shuffles, the role of @warpreduce in
// src/utils.jl:84-101).  kUp: prefix from lane 0; otherwise suffix from lane 31.
template <bool kUp, typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
    const uint32_t lane = lane_id();
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        T o = kUp ? __shfl_up_sync(kFullMask, v, off) : __shfl_down_sync(kFullMask, v, off);
        if (kUp ? (lane >= static_cast<uint32_t>(off)) : (lane + off < 32)) v += o;
    }
    return v;
}

// Barrier over the first THREADS threads of the CTA (hardware barrier 1).
// In a kernel whose block has exactly THREADS threads it is __syncthreads();
// the fused kernel's consumer warps use it without the producer warp that
// feeds them.  Same rules as __syncthreads: every participating warp reaches
// it, without divergence.
template <int THREADS>
__device__ __forceinline__ void block_sync() {
    asm volatile("bar.sync 1, %0;" ::"n"(THREADS) : "memory");
}

// block_sync that also returns whether `pred` holds in any participating thread.
template <int THREADS>
__device__ __forceinline__ bool block_sync_or(bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"(static_cast<uint32_t>(pred)), "n"(THREADS)
        : "memory");
    return r != 0;
}

// Programmatic dependent launch: a kernel launched with the programmatic
// stream serialization attribute may start while the previous kernel of its
// stream finishes; it waits here before it reads anything that kernel wrote.
// Without the attribute this returns at once.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Lets the stream's next kernel (launched programmatically) be scheduled now:
// its blocks take free SM slots and wait in grid_dep_wait, which still waits
// for this whole grid to complete and its writes to be visible.  Called once
// all of a grid's blocks are resident, it hides the next launch's latency.
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ void record_error(uint32_t* err, uint32_t bits) {
    if (err) atomicOr(err, bits);
}

}  // namespace radik
