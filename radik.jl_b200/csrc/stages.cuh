// stages.cuh -- the reference kernels' own contracts as standalone device
// stages (used by the stage entry points of radik.h and their parity tests):
//   count_bin_ex  src/kernels/count_bin.jl:78-203
//   count_bin     src/kernels/count_bin.jl:20-59
//   select_bin    src/kernels/select_bin.jl:268-348
//   filter        src/kernels/filter.jl:172-621
// Semantics are the reference's, quirks included (NaN skipped by count_bin_ex,
// float compares in filter); the engine's own pipeline (fused.cuh,
// general.cuh) uses key compares throughout.
#pragma once

#include "block_ops.cuh"

namespace radik {

__device__ __forceinline__ uint32_t ref_bin_id(float v, int left, int right) {
    return (key_of_bits(__float_as_uint(v)) << left) >> right;  // src/utils.jl:29-33
}

// src/utils.jl:68-71
__device__ __forceinline__ float ref_apply_scaling(float v, float scaler, int withscale, int largest) {
    float pv = isnan(v) ? (largest ? __uint_as_float(0x00800000u) : __uint_as_float(0x7f7fffffu)) : v;
    return withscale ? __fsub_rn(pv, scaler) : pv;
}

struct StageTask {
    int64_t start;
    int64_t len;
};

// grid: (x chunks, y task groups); shared histogram merged with global atomics
// like count_bin.jl:192-199.
__global__ void stage_count_bin_ex(int32_t* hist, const float* data, const StageTask* tasks, int64_t T,
                                   int left, int right, int hist_len, int withscale, int largest) {
    extern __shared__ int32_t h[];
    for (int64_t t = blockIdx.y; t < T; t += gridDim.y) {
        for (int i = threadIdx.x; i < hist_len; i += blockDim.x) h[i] = 0;
        __syncthreads();
        const StageTask td = tasks[t];
        float scaler = task_scaler(data, td.start, td.len, withscale);
        for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < td.len;
             i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
            float v = data[td.start + i];
            if (isnan(v)) continue;  // count_bin.jl:111
            atomicAdd(&h[ref_bin_id(ref_apply_scaling(v, scaler, withscale, largest), left, right)], 1);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < hist_len; i += blockDim.x)
            if (h[i]) atomicAdd(hist + t * hist_len + i, h[i]);
        __syncthreads();
    }
}

__global__ void stage_count_bin(int32_t* hist, const float* data, const StageTask* tasks, int64_t stride,
                                int64_t T, int left, int right, int hist_len) {
    extern __shared__ int32_t h[];
    for (int64_t t = blockIdx.y; t < T; t += gridDim.y) {
        for (int i = threadIdx.x; i < hist_len; i += blockDim.x) h[i] = 0;
        __syncthreads();
        const int64_t len = tasks[t].len;
        for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < len;
             i += static_cast<int64_t>(gridDim.x) * blockDim.x)
            atomicAdd(&h[ref_bin_id(data[t * stride + i], left, right)], 1);
        __syncthreads();
        for (int i = threadIdx.x; i < hist_len; i += blockDim.x)
            if (h[i]) atomicAdd(hist + t * hist_len + i, h[i]);
        __syncthreads();
    }
}

// One CTA per task.  Thread i owns hist_len/THREADS consecutive bins counted
// from the rank origin (top bin when largest), scans them, and the thread
// whose range holds rank k writes the 1-based bin, residual and count
// (find_bin_and_write!, select_bin.jl:125-159).
template <int THREADS>
__global__ void __launch_bounds__(THREADS) stage_select_bin(int32_t* bin_ids, int32_t* k_values, int32_t* counts,
                                                            const int32_t* hist, int64_t hist_len, int largest) {
    __shared__ BlockScratch<THREADS> s;
    const int64_t t = blockIdx.x;
    const int32_t* h = hist + t * hist_len;
    const int64_t per = (hist_len + THREADS - 1) / THREADS;
    auto bin_at = [&](int64_t j) { return largest ? hist_len - 1 - j : j; };
    int64_t sum = 0;
    for (int64_t j = 0; j < per; ++j) {
        int64_t rj = threadIdx.x * per + j;
        if (rj < hist_len) sum += h[bin_at(rj)];
    }
    uint32_t total;
    uint32_t before = block_exclusive_scan<THREADS>(static_cast<uint32_t>(sum), &total, s);
    const int64_t k = k_values[t];
    __syncthreads();
    if (k > 0 && before < k && k <= before + sum) {
        int64_t rr = k - before;
        for (int64_t j = 0; j < per; ++j) {
            int64_t rj = threadIdx.x * per + j;
            if (rj >= hist_len) break;
            int64_t b = bin_at(rj);
            int64_t c = h[b];
            if (c > 0 && c >= rr) {
                bin_ids[t] = static_cast<int32_t>(b + 1);
                k_values[t] = static_cast<int32_t>(rr);
                counts[t] = static_cast<int32_t>(c);
                break;
            }
            rr -= c;
        }
    }
}

// filter_stage_packed! / filter_stage_item!, filter.jl:106-139.
__global__ void stage_filter(float* val_out, void* idx_out, int idx_bytes, int32_t* counts, int32_t* boundary,
                             const float* data, const void* idx_in, const float* kth, const StageTask* tasks,
                             int64_t T, int64_t k, int withscale, int largest, uint32_t* err) {
    for (int64_t t = blockIdx.y; t < T; t += gridDim.y) {
        const StageTask td = tasks[t];
        const float scaler = task_scaler(data, td.start, td.len, withscale);
        const float kv = kth[t];
        for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < td.len;
             i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
            const int64_t g = td.start + i;
            const float v = data[g];
            bool emit = false;
            if (td.len <= k) {
                emit = true;  // filter.jl:272-322
            } else {
                float sv = ref_apply_scaling(v, scaler, withscale, largest);
                if ((largest && sv > kv) || (!largest && sv < kv)) emit = true;
                if (sv == kv && atomicSub(boundary + t, 1) - 1 > -1) emit = true;
            }
            if (!emit) continue;
            int32_t slot = atomicAdd(counts + t, 1);
            if (slot >= k) { record_error(err, kErrCapacity); continue; }
            int64_t idx = idx_in ? (idx_bytes == 8 ? static_cast<const int64_t*>(idx_in)[g]
                                                   : static_cast<int64_t>(static_cast<const int32_t*>(idx_in)[g]))
                                 : i + 1;
            val_out[t * k + slot] = v;
            if (idx_bytes == 8) static_cast<int64_t*>(idx_out)[t * k + slot] = idx;
            else static_cast<int32_t*>(idx_out)[t * k + slot] = static_cast<int32_t>(idx);
        }
    }
}

}  // namespace radik
