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

// Histogram increment with the lanes of a warp that hit the same bin
// combined into one shared atomic (same-bin lanes would otherwise serialise).
// All lanes of the warp must call; lanes with valid == false add nothing.
__device__ __forceinline__ void warp_hist_add(uint32_t* hist, uint32_t bin, bool valid) {
    const uint32_t key = valid ? bin : 0xffffffffu;
    const uint32_t peers = __match_any_sync(kFullMask, key);
    if (valid && (lanemask_lt() & peers) == 0) atomicAdd(hist + bin, static_cast<uint32_t>(__popc(peers)));
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
    block_sync<THREADS>();
    vor = 0; vand = ~0ull;
#pragma unroll
    for (int i = 0; i < BlockScratch<THREADS>::kWarps; ++i) { vor |= s.warp_a[i]; vand &= s.warp_b[i]; }
    block_sync<THREADS>();
}

template <int THREADS>
__device__ __forceinline__ uint64_t block_min_u64(uint64_t v, BlockScratch<THREADS>& s) {
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) { uint64_t o = shfl_xor_u64(v, m); v = o < v ? o : v; }
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0) s.warp_a[w] = v;
    block_sync<THREADS>();
    v = ~0ull;
#pragma unroll
    for (int i = 0; i < BlockScratch<THREADS>::kWarps; ++i) v = s.warp_a[i] < v ? s.warp_a[i] : v;
    block_sync<THREADS>();
    return v;
}

template <int THREADS>
__device__ __forceinline__ uint32_t block_sum_u32(uint32_t v, BlockScratch<THREADS>& s) {
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(kFullMask, v, m);
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0) s.warp_u32[w] = v;
    block_sync<THREADS>();
    v = 0;
#pragma unroll
    for (int i = 0; i < BlockScratch<THREADS>::kWarps; ++i) v += s.warp_u32[i];
    block_sync<THREADS>();
    return v;
}

// Exclusive scan of one u32 per thread in thread order; *total gets the sum.
template <int THREADS>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total, BlockScratch<THREADS>& s) {
    uint32_t inc = warp_inclusive_scan<true>(v);
    const int w = threadIdx.x >> 5;
    if (lane_id() == 31) s.warp_u32[w] = inc;
    block_sync<THREADS>();
    uint32_t before = 0, all = 0;
#pragma unroll
    for (int i = 0; i < BlockScratch<THREADS>::kWarps; ++i) {
        uint32_t x = s.warp_u32[i];
        before += (i < w) ? x : 0u;
        all += x;
    }
    block_sync<THREADS>();
    *total = all;
    return before + inc - v;
}

// Rank search over a histogram of nb (<= 256) bins counted from the top bin
// (the role of select_bin_kernel!'s warp scan + find_bin_and_write!,
// select_bin.jl:125-159, 268-348).  Warp 0 does it: lane l owns bins
// nb-1-l*per .. nb-(l+1)*per, a suffix warp scan gives the count above each
// lane's range, and the owner of rank r writes (bin, residual rank, bin count,
// count above the bin) to s.bc32 (bin count 0xffffffff when r exceeds the
// total).  All threads must call (the result is published by a barrier).
template <int THREADS>
__device__ __forceinline__ void block_rank_search(uint32_t r, uint32_t nb, BlockScratch<THREADS>& s) {
    if (threadIdx.x < 32) {
        const uint32_t lane = lane_id();
        const uint32_t per = (nb + 31) / 32;  // <= 8
        uint32_t c[8];
        uint32_t sum = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t rb = lane * per + j;
            c[j] = (j < static_cast<int>(per) && rb < nb) ? s.hist[nb - 1 - rb] : 0u;
            sum += c[j];
        }
        const uint32_t incl = warp_inclusive_scan<true>(sum);  // count in lanes <= this one
        const uint32_t before = incl - sum;
        const uint32_t total = __shfl_sync(kFullMask, incl, 31);
        if (lane == 0 && r > total) { s.bc32[0] = 0; s.bc32[1] = 0; s.bc32[2] = 0xffffffffu; s.bc32[3] = 0; }
        if (before < r && r <= incl) {
            uint32_t rr = r - before;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (j < static_cast<int>(per) && c[j] > 0) {
                    if (c[j] >= rr) {
                        s.bc32[0] = nb - 1 - (lane * per + j);
                        s.bc32[1] = rr;
                        s.bc32[2] = c[j];
                        s.bc32[3] = r - rr;
                        break;
                    }
                    rr -= c[j];
                }
            }
        }
    }
    block_sync<THREADS>();
}

// Ordered in-place compaction: moves the entries of buf[0, cnt) that are
// >= keep_from to the front (previous order kept).  Returns their number;
// *mn receives their minimum (~0 when none).
template <int THREADS>
__device__ __forceinline__ uint32_t block_compact_ge(uint64_t* buf, uint32_t cnt, uint64_t keep_from,
                                                     BlockScratch<THREADS>& s, uint64_t* mn_out) {
    constexpr int E = 4;
    const int tid = threadIdx.x;
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
        block_sync<THREADS>();
    }
    *mn_out = block_min_u64<THREADS>(mn, s);
    return out;
}

// Narrows buf[0, cnt) (unique composites, all inside [lo, hi]) to the entries
// >= keep_from, the lower edge of the digit bin that holds rank k counted from
// the largest: the countBin -> selectBin -> selectCandidate cycle of
// count_bin.jl, select_bin.jl and select_candidate.jl run on on-chip data.
// Digits are 8-bit windows starting right below the common prefix of lo and
// hi; windows are refined until at most max_keep (>= k) entries would remain,
// so max_keep == k yields exactly the top k.  Between windows the buffer is
// compacted to the entries that can still be kept, so refinements scan only
// those.  Kept entries move to the front (previous order).  Returns their
// number (cnt when cnt <= k); *keep_from_out and *mn_out receive the
// threshold and the smallest kept composite.  All threads must call.
template <int THREADS>
__device__ uint32_t block_shrink(uint64_t* buf, uint32_t cnt, uint32_t k, uint32_t max_keep, uint64_t lo,
                                 uint64_t hi, BlockScratch<THREADS>& s, uint32_t* err, uint64_t* keep_from_out,
                                 uint64_t* mn_out) {
    constexpr int W = 8;
    const int tid = threadIdx.x;
    const uint64_t diff = lo ^ hi;
    if (cnt <= k || diff == 0) {
        *keep_from_out = lo;
        uint64_t mn = ~0ull;
        for (uint32_t i = tid; i < cnt; i += THREADS) mn = buf[i] < mn ? buf[i] : mn;
        *mn_out = block_min_u64<THREADS>(mn, s);
        return cnt;
    }
    int top = 63 - __clzll(static_cast<long long>(diff));
    uint64_t prefix = (top >= 63) ? 0ull : (hi >> (top + 1));
    int pbits = 63 - top;  // bits above `top` shared by the entries still in play
    uint32_t r = k, above_total = 0, n = cnt;
    uint64_t keep_from = lo;
    for (int guard = 0; guard < 9; ++guard) {
        const int w = top + 1 < W ? top + 1 : W;
        const int sh = top + 1 - w;
        const uint32_t nb = 1u << w;
        for (uint32_t i = tid; i < nb; i += THREADS) s.hist[i] = 0;
        block_sync<THREADS>();
        const uint64_t dmask = nb - 1;
        for (uint32_t base = 0; base < n; base += THREADS) {
            const uint32_t i = base + tid;
            const uint64_t c = i < n ? buf[i] : 0ull;
            const bool in = i < n && (pbits == 0 || (c >> (sh + w)) == prefix);
            warp_hist_add(s.hist, static_cast<uint32_t>((c >> sh) & dmask), in);
        }
        block_sync<THREADS>();
        block_rank_search<THREADS>(r, nb, s);
        const uint32_t b = s.bc32[0], rr = s.bc32[1], cb = s.bc32[2], ab = s.bc32[3];
        block_sync<THREADS>();
        if (cb == 0xffffffffu) {  // rank beyond the entries: inputs outside [lo, hi]
            if (tid == 0) record_error(err, kErrInternal);
            keep_from = lo;
            break;
        }
        prefix = (pbits == 0) ? b : ((prefix << w) | b);
        pbits += w;
        above_total += ab;
        r = rr;
        keep_from = prefix << sh;
        if (above_total + cb <= max_keep || sh == 0) break;
        if (2 * (above_total + cb) < n) {  // drop what can no longer be kept
            uint64_t mn;
            n = block_compact_ge<THREADS>(buf, n, keep_from, s, &mn);
        }
        top = sh - 1;
    }
    *keep_from_out = keep_from;
    return block_compact_ge<THREADS>(buf, n, keep_from, s, mn_out);
}

// Lower edge of the digit bin holding rank r (from the largest) among
// buf[0, n) (values inside [lo, hi]): at least r entries are >= it, and at
// most `slack` unless `max_windows` digit windows do not get there.  The
// buffer is left as it is.  All threads must call.
template <int THREADS>
__device__ uint64_t block_rank_threshold(const uint64_t* buf, uint32_t n, uint32_t r, uint32_t slack, uint64_t lo,
                                         uint64_t hi, BlockScratch<THREADS>& s, int max_windows = 2) {
    constexpr int W = 8;
    const int tid = threadIdx.x;
    const uint64_t diff = lo ^ hi;
    if (n <= r || diff == 0) return lo;
    int top = 63 - __clzll(static_cast<long long>(diff));
    uint64_t prefix = (top >= 63) ? 0ull : (hi >> (top + 1));
    int pbits = 63 - top;
    uint32_t above_total = 0;
    uint64_t keep_from = lo;
    for (int pass = 0; pass < max_windows; ++pass) {
        const int w = top + 1 < W ? top + 1 : W;
        const int sh = top + 1 - w;
        const uint32_t nb = 1u << w;
        for (uint32_t i = tid; i < nb; i += THREADS) s.hist[i] = 0;
        block_sync<THREADS>();
        const uint64_t dmask = nb - 1;
        for (uint32_t base = 0; base < n; base += THREADS) {
            const uint32_t i = base + tid;
            const uint64_t c = i < n ? buf[i] : 0ull;
            const bool in = i < n && (pbits == 0 || (c >> (sh + w)) == prefix);
            warp_hist_add(s.hist, static_cast<uint32_t>((c >> sh) & dmask), in);
        }
        block_sync<THREADS>();
        block_rank_search<THREADS>(r, nb, s);
        const uint32_t b = s.bc32[0], rr = s.bc32[1], cb = s.bc32[2], ab = s.bc32[3];
        block_sync<THREADS>();
        if (cb == 0xffffffffu) return keep_from;
        prefix = (pbits == 0) ? b : ((prefix << w) | b);
        pbits += w;
        above_total += ab;
        r = rr;
        keep_from = prefix << sh;
        if (above_total + cb <= slack || sh == 0) break;
        top = sh - 1;
    }
    return keep_from;
}

// Largest T such that at least r of the warp's values x[] (NV per lane,
// padding 0, 1 <= r <= number of real values) are >= T: the r-th largest
// value, built two bits at a time below the values' common prefix (three
// counts per step, one warp reduction each).  With kExact, the search also
// stops at the first T with exactly r values >= T (any such T separates the
// r largest from the rest).  Only the calling warp takes part.
template <int NV, bool kExact = false>
__device__ __forceinline__ uint32_t warp_rank_search(const uint32_t (&x)[NV], uint32_t r) {
    uint32_t vor = 0u, vand = ~0u;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        vor |= x[j];
        if (x[j] != 0u) vand &= x[j];
    }
    vor = __reduce_or_sync(kFullMask, vor);
    vand = __reduce_and_sync(kFullMask, vand);
    const uint32_t diff = vor ^ vand;
    if (diff == 0u) return vand;
    int b = 31 - __clz(diff);                 // highest bit where the values differ
    uint32_t T = vand & ~((2u << b) - 1u);    // their common prefix: every value is >= T
    for (; b >= 1; b -= 2) {
        const uint32_t c1 = T | (1u << (b - 1)), c2 = T | (2u << (b - 1)), c3 = T | (3u << (b - 1));
        uint32_t n1 = 0, n2 = 0, n3 = 0;
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            n1 += x[j] >= c1 ? 1u : 0u;
            n2 += x[j] >= c2 ? 1u : 0u;
            n3 += x[j] >= c3 ? 1u : 0u;
        }
        n1 = __reduce_add_sync(kFullMask, n1);
        n2 = __reduce_add_sync(kFullMask, n2);
        n3 = __reduce_add_sync(kFullMask, n3);
        const uint32_t nT = n3 >= r ? n3 : (n2 >= r ? n2 : (n1 >= r ? n1 : 0u));
        T = n3 >= r ? c3 : (n2 >= r ? c2 : (n1 >= r ? c1 : T));
        if (kExact && nT == r) return T;
    }
    if (b == 0) {
        const uint32_t c1 = T | 1u;
        uint32_t n1 = 0;
#pragma unroll
        for (int j = 0; j < NV; ++j) n1 += x[j] >= c1 ? 1u : 0u;
        if (__reduce_add_sync(kFullMask, n1) >= r) T = c1;
    }
    return T;
}

// The r-th largest (1-based, 1 <= r <= n) of the high words of gm[0, n)
// (n <= 32 * NV), found by the calling warp (warp_rank_search).
template <int NV>
__device__ __forceinline__ uint32_t warp_rank_value(const uint64_t* gm, uint32_t n, uint32_t r) {
    const uint32_t lane = lane_id();
    uint32_t x[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        const uint32_t i = static_cast<uint32_t>(j) * 32u + lane;
        x[j] = i < n ? static_cast<uint32_t>(gm[i] >> 32) : 0u;  // padding 0 is below every candidate T
    }
    return warp_rank_search<NV>(x, r);
}

constexpr uint32_t kWarpBisect = 512;  // boundary-bin entries one warp finishes (16 per lane)

// Bound of the k best among buf[0, n) (unique composites in shared memory,
// 1 <= k <= n; vor and vand span them).  8-bit digit windows below the
// common prefix narrow the entries in play to the bin holding rank k: every
// warp counts into its own histogram (whist, 256 words per warp: no
// contention between warps on the few bins that most entries fall into), the
// histograms are summed and searched for rank k.  Once that bin holds at
// most kWarpBisect entries they are copied to `spill` and warp 0 finds the
// exact bound by bisection over their bits.  Returns tau with exactly k
// entries >= tau.  All threads call.
template <int THREADS>
__device__ uint64_t block_topk_bound(const uint64_t* buf, uint32_t n, uint32_t k, uint64_t vor, uint64_t vand,
                                     BlockScratch<THREADS>& s, uint32_t* whist, uint64_t* spill, uint32_t* spill_n,
                                     unsigned long long* result, uint32_t* err) {
    constexpr int W = 8;
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    const uint64_t diff = vor ^ vand;
    if (diff == 0ull) return vand;  // a single entry
    int top = 63 - __clzll(static_cast<long long>(diff));
    uint64_t prefix = (top >= 63) ? 0ull : (vand >> (top + 1));
    int pbits = 63 - top;  // bits above `top` shared by the entries still in play
    uint32_t r = k;
    for (int guard = 0; guard < 9; ++guard) {
        const int w = top + 1 < W ? top + 1 : W;
        const int sh = top + 1 - w;
        const uint32_t nb = 1u << w;
        uint32_t* my = whist + (tid >> 5) * 256u;
        for (uint32_t i = lane; i < nb; i += 32) my[i] = 0;
        __syncwarp();
        for (uint32_t i = tid; i < n; i += THREADS) {
            const uint64_t c = buf[i];
            if (pbits == 0 || (c >> (sh + w)) == prefix) atomicAdd(my + (static_cast<uint32_t>(c >> sh) & (nb - 1)), 1u);
        }
        block_sync<THREADS>();
        for (uint32_t i = tid; i < nb; i += THREADS) {
            uint32_t sum = 0;
#pragma unroll 8
            for (int ww = 0; ww < THREADS / 32; ++ww) sum += whist[ww * 256 + i];
            s.hist[i] = sum;
        }
        block_sync<THREADS>();
        block_rank_search<THREADS>(r, nb, s);
        const uint32_t b = s.bc32[0], rr = s.bc32[1], cb = s.bc32[2];
        block_sync<THREADS>();  // hist and bc32 are rewritten by the next window
        if (cb == 0xffffffffu) {  // never expected: rank k lies beyond the entries
            if (tid == 0) record_error(err, kErrInternal);
            return vand;
        }
        const uint64_t bin_prefix = (pbits == 0) ? b : ((prefix << w) | b);
        if (cb == rr || sh == 0) return bin_prefix << sh;  // the whole bin is in: k entries >= its lower edge
        if (cb <= kWarpBisect) {
            // The boundary bin to `spill`; warp 0 finds its rr-th largest.
            if (tid == 0) *spill_n = 0;
            block_sync<THREADS>();
            const uint32_t lt = lanemask_lt();
            for (uint32_t base = 0; base < n; base += THREADS) {
                const uint32_t i = base + tid;
                const uint64_t c = i < n ? buf[i] : 0ull;
                const bool in = i < n && (c >> sh) == bin_prefix;
                const uint32_t m = __ballot_sync(kFullMask, in);
                if (m == 0u) continue;
                const uint32_t leader = __ffs(m) - 1;
                uint32_t o = 0;
                if (lane == leader) o = atomicAdd(spill_n, __popc(m));
                o = __shfl_sync(kFullMask, o, leader);
                if (in && o + __popc(m & lt) < kWarpBisect) spill[o + __popc(m & lt)] = c;
            }
            block_sync<THREADS>();
            if (tid < 32) {
                const uint32_t cnt = *spill_n < kWarpBisect ? *spill_n : kWarpBisect;
                uint64_t wor = 0, wand = ~0ull;
                for (uint32_t i = lane; i < cnt; i += 32) {
                    wor |= spill[i];
                    wand &= spill[i];
                }
#pragma unroll
                for (int m = 16; m > 0; m >>= 1) {
                    wor |= __shfl_xor_sync(kFullMask, wor, m);
                    wand &= __shfl_xor_sync(kFullMask, wand, m);
                }
                uint64_t tau = wand;
                const uint64_t d = wor ^ wand;
                if (d != 0ull && rr <= cnt) {
                    int bb = 63 - __clzll(static_cast<long long>(d));
                    tau = (bb == 63) ? 0ull : (wand & ~((2ull << bb) - 1));
                    uint32_t cge = cnt;
                    for (; bb >= 0 && cge != rr; --bb) {
                        const uint64_t cand = tau | (1ull << bb);
                        uint32_t c = 0;
                        for (uint32_t i = lane; i < cnt; i += 32) c += (spill[i] >= cand) ? 1u : 0u;
                        c = __reduce_add_sync(kFullMask, c);
                        if (c >= rr) {
                            tau = cand;
                            cge = c;
                        }
                    }
                }
                if (lane == 0) {
                    if (cnt != cb) record_error(err, kErrInternal);
                    *result = tau;
                }
            }
            block_sync<THREADS>();
            return *result;
        }
        prefix = bin_prefix;
        pbits += w;
        r = rr;
        top = sh - 1;
    }
    if (tid == 0) record_error(err, kErrInternal);
    return prefix;
}

// Exact top-k of buf[0, cnt) (unique composites): on return buf[0, min(cnt,k))
// holds the k largest in their previous order; returns their number and the
// smallest of them (the k-th composite) through *kth.
template <int THREADS>
__device__ uint32_t block_select_topk(uint64_t* buf, uint32_t cnt, uint32_t k, BlockScratch<THREADS>& s,
                                      uint32_t* err, uint64_t* kth) {
    uint64_t vor = 0, vand = ~0ull;
    for (uint32_t i = threadIdx.x; i < cnt; i += THREADS) { uint64_t c = buf[i]; vor |= c; vand &= c; }
    block_or_and<THREADS>(vor, vand, s);
    uint64_t kf;
    uint32_t kept = block_shrink<THREADS>(buf, cnt, k, k, vand, vor, s, err, &kf, kth);
    if (cnt > k && kept != k && threadIdx.x == 0) record_error(err, kErrInternal);
    return kept;
}

// Ascending sort of buf[0, m) for m <= THREADS (unique keys below ~0):
// every warp sorts 32 entries in registers (bitonic network over shuffles),
// then each entry's final place is its lane plus, for every other warp's
// sorted run, the number of entries below it (binary search).  Three
// barriers in all; `runs` is scratch for THREADS entries.
template <int THREADS>
__device__ void small_sort_u64(uint64_t* buf, uint32_t m, uint64_t* runs) {
    const int tid = threadIdx.x;
    const uint32_t lane = tid & 31, warp = tid >> 5;
    uint64_t v = static_cast<uint32_t>(tid) < m ? buf[tid] : ~0ull;
#pragma unroll
    for (uint32_t size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            const uint64_t o = __shfl_xor_sync(kFullMask, static_cast<unsigned long long>(v), stride);
            const bool up = (lane & size) == 0;      // this block of `size` lanes ascends
            const bool low = (lane & stride) == 0;   // lower lane of the pair
            const bool take_min = low == up;
            v = take_min ? (o < v ? o : v) : (o > v ? o : v);
        }
    }
    runs[tid] = v;
    block_sync<THREADS>();
    uint32_t pos = lane;
#pragma unroll
    for (uint32_t w2 = 0; w2 < static_cast<uint32_t>(THREADS / 32); ++w2) {
        if (w2 == warp) continue;
        const uint64_t* r = runs + w2 * 32;
        uint32_t c = 0;  // entries of run w2 below v
#pragma unroll
        for (uint32_t step = 16; step >= 1; step >>= 1)
            if (r[c + step - 1] < v) c += step;
        if (r[c] < v) ++c;
        pos += c;
    }
    block_sync<THREADS>();
    if (v != ~0ull && pos < m) buf[pos] = v;
    block_sync<THREADS>();
}

// Ascending bitonic sort of n = THREADS * PER keys held in registers: thread
// t holds elements t, t + THREADS, ...  A compare-exchange at stride s pairs
// lanes of one warp (s < 32: shuffles), threads of different warps (32 <= s
// < THREADS: through shared memory, two buffers `sm` of n entries each, one
// barrier per stage) or registers of one thread (s >= THREADS).
template <int THREADS, int PER>
__device__ void bitonic_sort_regs(uint64_t (&v)[PER], uint64_t* sm) {
    constexpr uint32_t N = THREADS * PER;
    const uint32_t tid = threadIdx.x;
    int buf = 0;
    for (uint32_t size = 2; size <= N; size <<= 1) {
        for (uint32_t s = size >> 1; s > 0; s >>= 1) {
            if (s >= static_cast<uint32_t>(THREADS)) {
                const uint32_t js = s / THREADS;
#pragma unroll
                for (int j = 0; j < PER; ++j) {
#pragma unroll
                    for (int jp = j + 1; jp < PER; ++jp) {
                        if (static_cast<uint32_t>(j ^ jp) == js) {
                            const uint32_t e = static_cast<uint32_t>(j) * THREADS + tid;  // lower of the pair
                            const bool up = (e & size) == 0;
                            const uint64_t a = v[j], b = v[jp];
                            const bool sw = up ? (a > b) : (a < b);
                            v[j] = sw ? b : a;
                            v[jp] = sw ? a : b;
                        }
                    }
                }
            } else if (s >= 32) {
                uint64_t* x = sm + buf * N;
#pragma unroll
                for (int j = 0; j < PER; ++j) x[j * THREADS + tid] = v[j];
                block_sync<THREADS>();
#pragma unroll
                for (int j = 0; j < PER; ++j) {
                    const uint32_t e = static_cast<uint32_t>(j) * THREADS + tid;
                    const uint64_t o = x[j * THREADS + (tid ^ s)];
                    const bool up = (e & size) == 0, low = (tid & s) == 0;
                    v[j] = (low == up) ? (o < v[j] ? o : v[j]) : (o > v[j] ? o : v[j]);
                }
                buf ^= 1;  // the next exchange writes the other buffer: no second barrier
            } else {
#pragma unroll
                for (int j = 0; j < PER; ++j) {
                    const uint32_t e = static_cast<uint32_t>(j) * THREADS + tid;
                    const uint64_t o = __shfl_xor_sync(kFullMask, static_cast<unsigned long long>(v[j]), s);
                    const bool up = (e & size) == 0, low = (tid & s) == 0;
                    v[j] = (low == up) ? (o < v[j] ? o : v[j]) : (o > v[j] ? o : v[j]);
                }
            }
        }
    }
    block_sync<THREADS>();  // the buffers may be reused
}

// Sorts buf[0, m) ascending with bitonic_sort_regs (n = THREADS * PER >= m,
// padding ~0); scratch holds 2 n entries.
template <int THREADS, int PER>
__device__ void regs_sort_u64(uint64_t* buf, uint32_t m, uint64_t* scratch) {
    uint64_t v[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const uint32_t e = static_cast<uint32_t>(j) * THREADS + threadIdx.x;
        v[j] = e < m ? buf[e] : ~0ull;
    }
    bitonic_sort_regs<THREADS, PER>(v, scratch);
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const uint32_t e = static_cast<uint32_t>(j) * THREADS + threadIdx.x;
        if (e < m) buf[e] = v[j];
    }
    block_sync<THREADS>();
}

// Bitonic sort of a[0, n) in shared memory (n a power of two), ascending or
// descending.
template <int THREADS>
__device__ __forceinline__ void bitonic_sort_u64(uint64_t* a, uint32_t n, bool descending = false) {
    for (uint32_t size = 2; size <= n; size <<= 1) {
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint32_t i = threadIdx.x; i < (n >> 1); i += THREADS) {
                uint32_t lo = 2 * i - (i & (stride - 1));
                uint32_t hi = lo + stride;
                bool asc = ((lo & size) == 0) != descending;
                uint64_t x = a[lo], y = a[hi];
                if ((x > y) == asc) { a[lo] = y; a[hi] = x; }
            }
            block_sync<THREADS>();
        }
    }
}

// Stable ascending LSD radix sort (8-bit digits) of a[0, n) using b[0, n) as
// scratch; digits on which all keys agree are skipped.  Returns the buffer
// (a or b) that holds the sorted keys.  Buffers may live in shared or global
// memory (generic addressing).  Every warp owns a contiguous chunk of the
// keys; a digit pass is: per-warp histograms of the chunk, the digit-major
// exclusive scan over (digit, warp) -- each warp's first slot per digit --
// and a scatter in which every warp walks its chunk in order, 32 keys at a
// time, ranking lanes of equal digits with one match: no block barrier
// inside the scatter, five per pass.
constexpr int kSortGroups = 4;  // radix_sort_u64: groups of 32 keys a warp handles at once

template <int THREADS>
__device__ __forceinline__ uint64_t* radix_sort_u64(uint64_t* a, uint64_t* b, uint32_t n, BlockScratch<THREADS>& s,
                                    uint32_t* warp_digit /* [THREADS/32][256] shared */,
                                    uint32_t* digit_base /* [256] shared */) {
    constexpr int W = THREADS / 32;
    const int tid = threadIdx.x, w = tid >> 5;
    const uint32_t lane = lane_id();
    uint64_t vor = 0, vand = ~0ull;
    for (uint32_t i = tid; i < n; i += THREADS) { vor |= a[i]; vand &= a[i]; }
    block_or_and<THREADS>(vor, vand, s);
    const uint64_t diff = vor ^ vand;
    const uint32_t chunk = (n + W - 1) / W;
    const uint32_t lo = static_cast<uint32_t>(w) * chunk < n ? static_cast<uint32_t>(w) * chunk : n;
    const uint32_t hi = lo + chunk < n ? lo + chunk : n;
    uint32_t* mine = warp_digit + w * 256;
    for (int sh = 0; sh < 64; sh += 8) {
        if (((diff >> sh) & 0xffull) == 0) continue;
        // 1. histogram of this warp's chunk, four groups of 32 keys at a time
        //    (their loads and matches in flight together)
        for (uint32_t j = lane; j < 256; j += 32) mine[j] = 0;
        __syncwarp();
        for (uint32_t base = lo; base < hi; base += 32u * kSortGroups) {
            uint32_t d[kSortGroups];
#pragma unroll
            for (int u = 0; u < kSortGroups; ++u) {
                const uint32_t i = base + static_cast<uint32_t>(u) * 32u + lane;
                d[u] = i < hi ? static_cast<uint32_t>((a[i] >> sh) & 0xff) : 256u + lane;
            }
#pragma unroll
            for (int u = 0; u < kSortGroups; ++u) {
                const uint32_t peers = __match_any_sync(kFullMask, d[u]);
                if (d[u] < 256u && (lanemask_lt() & peers) == 0u) atomicAdd(mine + d[u], static_cast<uint32_t>(__popc(peers)));
            }
        }
        block_sync<THREADS>();
        // 2. digit totals, their exclusive scan, then each warp's first slot
        for (int d = tid; d < 256; d += THREADS) {
            uint32_t tot = 0;
            for (int ww = 0; ww < W; ++ww) tot += warp_digit[ww * 256 + d];
            digit_base[d] = tot;
        }
        block_sync<THREADS>();
        if (tid < 32) {
            uint32_t c[8], sum = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) { c[j] = digit_base[tid * 8 + j]; sum += c[j]; }
            uint32_t run = warp_inclusive_scan<true>(sum) - sum;
#pragma unroll
            for (int j = 0; j < 8; ++j) { digit_base[tid * 8 + j] = run; run += c[j]; }
        }
        block_sync<THREADS>();
        for (int d = tid; d < 256; d += THREADS) {
            uint32_t run = digit_base[d];
            for (int ww = 0; ww < W; ++ww) {
                const uint32_t c = warp_digit[ww * 256 + d];
                warp_digit[ww * 256 + d] = run;
                run += c;
            }
        }
        block_sync<THREADS>();
        // 3. stable scatter: chunks in warp order, keys in order inside a
        //    chunk.  Per group of 32 keys the first lane of each digit takes
        //    the group's slots with one shared atomic on the warp's cursor and
        //    hands the base to its peers; a warp barrier after each group's
        //    atomics orders them before the next group's, so keys keep their
        //    order.  The groups' loads and matches are in flight together.
        for (uint32_t base = lo; base < hi; base += 32u * kSortGroups) {
            uint64_t v[kSortGroups];
            uint32_t d[kSortGroups];
#pragma unroll
            for (int u = 0; u < kSortGroups; ++u) {
                const uint32_t i = base + static_cast<uint32_t>(u) * 32u + lane;
                v[u] = i < hi ? a[i] : 0ull;
                d[u] = i < hi ? static_cast<uint32_t>((v[u] >> sh) & 0xff) : 256u + lane;
            }
#pragma unroll
            for (int u = 0; u < kSortGroups; ++u) {
                const uint32_t peers = __match_any_sync(kFullMask, d[u]);
                const uint32_t leader = static_cast<uint32_t>(__ffs(peers)) - 1u;
                uint32_t off = 0;
                if (d[u] < 256u && lane == leader) off = atomicAdd(mine + d[u], static_cast<uint32_t>(__popc(peers)));
                __syncwarp();
                off = __shfl_sync(kFullMask, off, static_cast<int>(leader));
                if (d[u] < 256u) b[off + __popc(peers & lanemask_lt())] = v[u];
            }
        }
        block_sync<THREADS>();
        uint64_t* t = a; a = b; b = t;
    }
    return a;
}

}  // namespace radik
