// block_ops.cuh -- CTA-wide building blocks of the top-k engine:
//   * reductions and an exclusive scan,
//   * block_select_topk: exact top-k of a buffer of unique 64-bit composites
//     by MSB-first radix selection (histogram -> rank search -> narrow), the
//     countBin / selectBin / selectCandidate cycle of RadiK.jl
//     (src/kernels/count_bin.jl, select_bin.jl, select_candidate.jl) run on
//     an on-chip buffer, with the digit window starting at the highest bit
//     where the buffer's composites differ,
//   * bitonic_sort_u64: ascending sort of a power-of-two array in shared
//     memory (replaces BitonicSort.jl's bitonic_sort!, src/algorithm.jl:343),
//   * radix_sort_u64: stable LSD radix sort with 8-bit digits (replaces
//     AcceleratedKernels.merge_sort_by_key!, src/algorithm.jl:345-351).
#pragma once

#include "common.cuh"

namespace radik {

template <int THREADS>
struct BlockScratch {
    static constexpr int kWarps = THREADS / 32;
    uint32_t hist[256];
    uint32_t warp_u32[kWarps];
    uint64_t warp_a[kWarps];
    uint64_t warp_b[kWarps];
    uint64_t bc64[2];
    uint32_t bc32[4];
};

__device__ __forceinline__ uint64_t shfl_xor_u64(uint64_t v, int m) {
    return __shfl_xor_sync(kFullMask, static_cast<unsigned long long>(v), m);
}

// OR and AND of v over the block; result visible to all threads.
template <int THREADS>
__device__ __forceinline__ void block_or_and(uint64_t& vor, uint64_t& vand, BlockScratch<THREADS>& s) {
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) {
        vor |= shfl_xor_u64(vor, m);
        vand &= shfl_xor_u64(vand, m);
    }
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0) { s.warp_a[w] = vor; s.warp_b[w] = vand; }
    __syncthreads();
    vor = 0; vand = ~0ull;
#pragma unroll
    for (int i = 0; i < BlockScratch<THREADS>::kWarps; ++i) { vor |= s.warp_a[i]; vand &= s.warp_b[i]; }
    __syncthreads();
}

template <int THREADS>
__device__ __forceinline__ uint64_t block_min_u64(uint64_t v, BlockScratch<THREADS>& s) {
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) { uint64_t o = shfl_xor_u64(v, m); v = o < v ? o : v; }
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0) s.warp_a[w] = v;
    __syncthreads();
    v = ~0ull;
#pragma unroll
    for (int i = 0; i < BlockScratch<THREADS>::kWarps; ++i) v = s.warp_a[i] < v ? s.warp_a[i] : v;
    __syncthreads();
    return v;
}

template <int THREADS>
__device__ __forceinline__ uint32_t block_sum_u32(uint32_t v, BlockScratch<THREADS>& s) {
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(kFullMask, v, m);
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0) s.warp_u32[w] = v;
    __syncthreads();
    v = 0;
#pragma unroll
    for (int i = 0; i < BlockScratch<THREADS>::kWarps; ++i) v += s.warp_u32[i];
    __syncthreads();
    return v;
}

// Exclusive scan of one u32 per thread in thread order; *total gets the sum.
template <int THREADS>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total, BlockScratch<THREADS>& s) {
    uint32_t inc = warp_inclusive_scan<true>(v);
    const int w = threadIdx.x >> 5;
    if (lane_id() == 31) s.warp_u32[w] = inc;
    __syncthreads();
    uint32_t before = 0, all = 0;
#pragma unroll
    for (int i = 0; i < BlockScratch<THREADS>::kWarps; ++i) {
        uint32_t x = s.warp_u32[i];
        before += (i < w) ? x : 0u;
        all += x;
    }
    __syncthreads();
    *total = all;
    return before + inc - v;
}

// Rank search over a 256-bin histogram from the top bin (select_bin.jl:
// warp scan + find_bin_and_write!, here one warp with 8 bins per lane):
// returns bin b with above(b) < r <= above(b) + hist[b]; writes residual rank
// and the bin count.  Executed by warp 0; result broadcast through s.bc32.
template <int THREADS>
__device__ __forceinline__ void block_rank_search(uint32_t r, uint32_t nbins, BlockScratch<THREADS>& s) {
    if (threadIdx.x < 32) {
        const uint32_t lane = lane_id();
        if (lane == 0) { s.bc32[0] = 0; s.bc32[1] = 0; s.bc32[2] = 0xffffffffu; }
        __syncwarp();
        const uint32_t per = (nbins + 31) / 32;
        uint32_t c[8];
        uint32_t sum = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            uint32_t b = lane * per + j;
            c[j] = (j < static_cast<int>(per) && b < nbins) ? s.hist[b] : 0u;
            sum += c[j];
        }
        uint32_t incl = warp_inclusive_scan<false>(sum);  // suffix sum from this lane up
        uint32_t above = incl - sum;
        if (above < r && r <= incl) {
            uint32_t rr = r - above;
#pragma unroll
            for (int j = 7; j >= 0; --j) {
                if (j < static_cast<int>(per) && c[j] > 0) {
                    if (c[j] >= rr) {
                        s.bc32[0] = lane * per + j;
                        s.bc32[1] = rr;
                        s.bc32[2] = c[j];
                        rr = 0;
                        break;
                    }
                    rr -= c[j];
                }
            }
        }
    }
    __syncthreads();
}

// Exact top-k of buf[0, cnt) (unique composites; cnt > k >= 1).  On return
// buf[0, k) holds the k largest composites in their previous relative order
// and the smallest of them is returned.  All threads must call.
template <int THREADS>
__device__ __forceinline__ uint64_t block_select_topk(uint64_t* buf, uint32_t cnt, uint32_t k, BlockScratch<THREADS>& s,
                                      uint32_t* err) {
    const int tid = threadIdx.x;
    // Highest bit where the composites differ.
    uint64_t vor = 0, vand = ~0ull;
    for (uint32_t i = tid; i < cnt; i += THREADS) { uint64_t c = buf[i]; vor |= c; vand &= c; }
    block_or_and<THREADS>(vor, vand, s);
    const uint64_t diff = vor ^ vand;
    int top = 63 - __clzll(static_cast<long long>(diff));  // diff != 0 since cnt >= 2
    uint64_t prefix = (top >= 63) ? 0ull : (vand >> (top + 1));
    int pbits = 63 - top;  // number of prefix bits (above `top`)
    uint32_t r = k;
    uint64_t keep_from = 0;
    for (int guard = 0; guard < 64; ++guard) {
        const int w = top + 1 < 8 ? top + 1 : 8;
        const int sh = top + 1 - w;
        for (int i = tid; i < 256; i += THREADS) s.hist[i] = 0;
        __syncthreads();
        const uint64_t dmask = (1ull << w) - 1;
        for (uint32_t i = tid; i < cnt; i += THREADS) {
            uint64_t c = buf[i];
            bool match = (pbits == 0) || ((c >> (sh + w)) == prefix);
            if (match) atomicAdd(&s.hist[(c >> sh) & dmask], 1u);
        }
        __syncthreads();
        block_rank_search<THREADS>(r, 1u << w, s);
        const uint32_t b = s.bc32[0], rr = s.bc32[1], cb = s.bc32[2];
        __syncthreads();
        prefix = (pbits == 0) ? b : ((prefix << w) | b);
        pbits += w;
        r = rr;
        if (cb == rr || sh == 0) {
            if (cb != rr && tid == 0) record_error(err, kErrInternal);
            keep_from = prefix << sh;
            break;
        }
        top = sh - 1;
    }
    // Ordered in-place compaction of the kept composites to the front.
    constexpr int E = 4;
    uint64_t mn = ~0ull;
    uint32_t out = 0;
    for (uint32_t base = 0; base < cnt; base += THREADS * E) {
        uint64_t v[E];
        uint32_t nk = 0, km = 0;
#pragma unroll
        for (int j = 0; j < E; ++j) {
            uint32_t i = base + tid * E + j;
            v[j] = (i < cnt) ? buf[i] : 0ull;
            bool kp = (i < cnt) && v[j] >= keep_from;
            nk += kp ? 1u : 0u;
            km |= kp ? (1u << j) : 0u;
        }
        uint32_t total;
        uint32_t off = block_exclusive_scan<THREADS>(nk, &total, s);  // has barriers: reads done
        uint32_t o = out + off;
#pragma unroll
        for (int j = 0; j < E; ++j) {
            if (km & (1u << j)) {
                if (o < cnt) buf[o] = v[j];
                mn = v[j] < mn ? v[j] : mn;
                ++o;
            }
        }
        out += total;
        __syncthreads();
    }
    if (out != k && tid == 0) record_error(err, kErrInternal);
    return block_min_u64<THREADS>(mn, s);
}

// Ascending bitonic sort of a[0, n) in shared memory, n a power of two.
template <int THREADS>
__device__ __forceinline__ void bitonic_sort_u64(uint64_t* a, uint32_t n) {
    for (uint32_t size = 2; size <= n; size <<= 1) {
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint32_t i = threadIdx.x; i < (n >> 1); i += THREADS) {
                uint32_t lo = 2 * i - (i & (stride - 1));
                uint32_t hi = lo + stride;
                bool asc = (lo & size) == 0;
                uint64_t x = a[lo], y = a[hi];
                if ((x > y) == asc) { a[lo] = y; a[hi] = x; }
            }
            __syncthreads();
        }
    }
}

// Stable ascending LSD radix sort (8-bit digits) of a[0, n) using b[0, n) as
// scratch; digits on which all keys agree are skipped.  Returns the buffer
// (a or b) that holds the sorted keys.  Buffers may live in shared or global
// memory (generic addressing).
template <int THREADS>
__device__ __forceinline__ uint64_t* radix_sort_u64(uint64_t* a, uint64_t* b, uint32_t n, BlockScratch<THREADS>& s,
                                    uint32_t* warp_digit /* [THREADS/32][256] shared */,
                                    uint32_t* digit_base /* [256] shared */) {
    constexpr int W = THREADS / 32;
    const int tid = threadIdx.x, w = tid >> 5;
    uint64_t vor = 0, vand = ~0ull;
    for (uint32_t i = tid; i < n; i += THREADS) { vor |= a[i]; vand &= a[i]; }
    block_or_and<THREADS>(vor, vand, s);
    const uint64_t diff = vor ^ vand;
    for (int sh = 0; sh < 64; sh += 8) {
        if (((diff >> sh) & 0xffull) == 0) continue;
        // digit histogram -> exclusive offsets
        for (int i = tid; i < 256; i += THREADS) s.hist[i] = 0;
        __syncthreads();
        for (uint32_t i = tid; i < n; i += THREADS) atomicAdd(&s.hist[(a[i] >> sh) & 0xff], 1u);
        __syncthreads();
        if (tid < 32) {
            uint32_t c[8], sum = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) { c[j] = s.hist[tid * 8 + j]; sum += c[j]; }
            uint32_t inc = warp_inclusive_scan<true>(sum);
            uint32_t run = inc - sum;
#pragma unroll
            for (int j = 0; j < 8; ++j) { digit_base[tid * 8 + j] = run; run += c[j]; }
        }
        __syncthreads();
        // stable scatter, one tile of THREADS keys at a time in order
        for (uint32_t base = 0; base < n; base += THREADS) {
            uint32_t i = base + tid;
            bool valid = i < n;
            uint64_t v = valid ? a[i] : 0ull;
            uint32_t d = valid ? static_cast<uint32_t>((v >> sh) & 0xff) : 256u + lane_id();
            uint32_t peers = __match_any_sync(kFullMask, d);
            uint32_t rank = __popc(peers & lanemask_lt());
            for (int j = tid; j < W * 256; j += THREADS) warp_digit[j] = 0;
            __syncthreads();
            if (valid && rank == 0) warp_digit[w * 256 + d] = __popc(peers);
            __syncthreads();
            // per digit: prefix over warps (thread d handles digit d)
            for (int dd = tid; dd < 256; dd += THREADS) {
                uint32_t run = digit_base[dd];
                for (int ww = 0; ww < W; ++ww) {
                    uint32_t c = warp_digit[ww * 256 + dd];
                    warp_digit[ww * 256 + dd] = run;
                    run += c;
                }
                digit_base[dd] = run;
            }
            __syncthreads();
            if (valid) b[warp_digit[w * 256 + d] + rank] = v;
            __syncthreads();
        }
        uint64_t* t = a; a = b; b = t;
    }
    return a;
}

}  // namespace radik
