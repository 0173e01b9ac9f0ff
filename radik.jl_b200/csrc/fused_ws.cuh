// fused_ws.cuh -- warp-specialised form of the fused top-k kernel.
//
// Same work items, thresholds, candidate buffer, retry and finishing as
// fused_topk_kernel (fused.cuh); what differs is how tiles move and how warps
// coordinate:
//   * one producer warp pulls work items from the queue, hands them to the
//     consumer warps through a small ring of item slots, and streams every
//     item's tiles with 1-D bulk copies into a ring of shared-memory stages
//     ("full" mbarrier per stage, completed by the copy's byte count);
//   * every tile belongs to one consumer warp (tiles are dealt round-robin),
//     32 elements per lane, so the per-tile cost (wait, release, bookkeeping)
//     is paid once per 32 elements; the warp frees the stage ("empty"
//     mbarrier) as soon as it is done with it, and no barrier is shared
//     between warps while they stream;
//   * the fast test keeps one bit per element (the float compare against
//     the threshold's value, on the registers it loaded); one warp scan
//     places the warp's candidates in its own region, and their values are
//     read back from the stage the warp still holds;
//   * when a warp's region overflows it keeps the tile, raises a request and
//     every consumer warp joins a block-wide shrink (polling the request
//     between tiles and while waiting for one), after which the requester
//     places the rest of its tile with the raised threshold;
//   * a single-segment task's first two tiles are a sample of it (chunks
//     spread over the whole task), streamed like any tile so that its
//     latency overlaps the previous task; its group maxima give the starting
//     threshold (see ws_sample_rank).
// Consumer warps synchronise with hardware barrier 1 over THREADS consumer
// threads (block_sync), so the producer never takes part in their barriers.
// Every mbarrier wait is bounded; a wait that gives up records a timeout and
// sets the CTA's abort flag, after which all waits give up at once, the
// producer stops issuing and waits (bounded) for its copies in flight.
#pragma once

#include "fused.cuh"

namespace radik {

constexpr int kItemSlots = 4;

template <int THREADS>
struct WsShared {
    FusedShared<THREADS> f;
    uint64_t thr;               // threshold published by the last block-wide shrink
    int32_t items[kItemSlots];  // work items, producer -> consumers
    int32_t cur;                // the consumers' current item (written by thread 0)
    uint32_t req;               // a consumer warp needs room
    uint32_t arrived;           // consumer warps done with the current item's tiles
};

__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t* a) {
    return *reinterpret_cast<const volatile uint32_t*>(a);
}
__device__ __forceinline__ void st_volatile_u32(uint32_t* a, uint32_t v) {
    *reinterpret_cast<volatile uint32_t*>(a) = v;
}

// Bounded wait of one thread on one mbarrier phase; gives up early once the
// CTA aborts.  Returns false when it gave up (a timeout is recorded and the
// abort flag set).
__device__ __forceinline__ bool ws_wait(uint64_t* bar, uint32_t parity, uint32_t* abort, uint32_t* err) {
    for (uint32_t i = 0; i < kWaitPolls; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 63u) == 63u && ld_volatile_u32(abort)) return false;
    }
    record_error(err, kErrTimeout);
    st_volatile_u32(abort, 1u);
    return false;
}

// Appends a warp's region (its first min(wcnt, R) entries) to a task's
// candidate region in global memory: one atomic per warp reserves the slots.
// A region that would overflow flags the task (the retry launch recomputes
// it) and is dropped.  All lanes of the warp must call; wcnt becomes 0.
__device__ __forceinline__ void ws_flush(const uint64_t* region, uint32_t& wcnt, uint32_t R, uint64_t* dst,
                                         uint32_t* cnt, uint32_t cap, uint32_t* fail_t, uint32_t* fail_any,
                                         uint32_t lane) {
    const uint32_t n = wcnt < R ? wcnt : R;
    if (n != 0) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(cnt, n);
        base = __shfl_sync(kFullMask, base, 0);
        if (static_cast<uint64_t>(base) + n <= cap) {
            for (uint32_t i = lane; i < n; i += 32) dst[base + i] = region[i];
        } else if (lane == 0) {
            *fail_t = 1u;
            atomicExch(fail_any, 1u);
        }
        __syncwarp();
    }
    wcnt = 0;
}

// Bounded wait of a whole warp on one mbarrier phase.
__device__ __forceinline__ bool ws_warp_wait(uint64_t* bar, uint32_t parity, uint32_t* abort, uint32_t* err) {
    for (uint32_t polls = 1;; ++polls) {
        if (__all_sync(kFullMask, mbar_try_wait(bar, parity))) return true;
        if (__any_sync(kFullMask, polls >= kWaitPolls || ((polls & 63u) == 0u && ld_volatile_u32(abort) != 0u))) {
            if (lane_id() == 0) {
                record_error(err, kErrTimeout);
                st_volatile_u32(abort, 1u);
            }
            return false;
        }
    }
}

// Sample of a single-segment task: chunks of kSampleChunkLen consecutive
// elements spread evenly over the task (p.sample_max <= kSampleMax elements
// for tasks of at least 16 times that, half as many down to 8 times the
// half, none below; the first tiles of the task in the ring).  The consumers
// take the maximum score of every 4 consecutive sampled elements (a group)
// and keep every element scoring at least the r-th largest group maximum
// (found exactly by one warp, warp_rank_value): at least r groups, hence at
// least r sampled elements, score at or above it.
// With lam = k * samples / len sampled elements expected at or above the
// task's k-th score, the threshold is too high only when at least r of them
// fall in the sample: r = lam + 5 sqrt(lam) + 3 makes that a Poisson tail of
// about 4e-7 at lam = 8.  A task that fails is redone from global memory
// (attempt 1 from rank 2r + 8 of the same sample, then with no threshold),
// so results never depend on the sample; but one such redo delays its whole
// batch, so the tail must stay far below one per batch of a thousand tasks.
// 256-element chunks (1 KB copies): at a batch's start every block loads its
// sample at once, and 64-element chunks (256 B copies) took 8.7 us to arrive
// on the uniform batch; 1 KB copies cut the whole call by 4-6 %.
constexpr uint32_t kSampleChunkLen = 256;
constexpr uint32_t kSampleMax = 4096;

// Sampled elements of a task (0: no sample); the same in producer and
// consumers.  `most`: the sample tiles the block's consumer warps can take
// (one each), in elements.
__device__ __forceinline__ uint32_t ws_sample_len(const FusedParams& p, const FusedTask& td, uint32_t most) {
    if (p.retry || td.nseg != 1) return 0u;
    const uint32_t smax = p.sample_max < most ? p.sample_max : most;
    if (td.len >= 16 * static_cast<int64_t>(smax)) return smax;
    if (td.len >= 4 * static_cast<int64_t>(smax)) return smax / 2;
    return 0u;
}

// Rank r of the starting threshold among the sample's groups (0: none).
__device__ __forceinline__ uint32_t ws_sample_rank(const FusedTask& td, uint32_t slen) {
    if (slen == 0) return 0u;
    const float lam = static_cast<float>(td.k) * static_cast<float>(slen) / static_cast<float>(td.len);
    const uint32_t r = static_cast<uint32_t>(ceilf(lam + 5.0f * sqrtf(lam) + 3.0f));
    return r <= slen / 4 / 4 ? r : 0u;  // at most a quarter of the groups
}

// First element of sample chunk c of nch, 16-byte aligned in memory (mis: the
// task pointer's offset in elements from a 16-byte boundary).
__device__ __forceinline__ int64_t ws_sample_pos(int64_t len, int64_t mis, uint32_t c, uint32_t nch) {
    int64_t q = ((static_cast<int64_t>(c) * len / nch + mis) & ~int64_t(3)) - mis;
    if (q < 0) q += 4;
    const int64_t last = ((len - kSampleChunkLen + mis) & ~int64_t(3)) - mis;  // last aligned start that fits
    return q < last ? q : last;
}

// Producer (one thread): items to the item ring, tiles to the stage ring.
template <int THREADS, int J, int STAGES, bool kScale>
__device__ void ws_producer(const FusedParams& p, float* ring, uint64_t* full, uint64_t* empty, uint64_t* item_full,
                            uint64_t* item_empty, WsShared<THREADS>& sh) {
    constexpr uint32_t TW = 128u * J;  // elements per warp tile
    constexpr uint32_t kChunksPerTile = TW / kSampleChunkLen;
    static_assert((kSampleMax / 2) % TW == 0 && TW % kSampleChunkLen == 0, "sample tiles");
    const uint64_t pol = l2_evict_first_policy();  // the input is read once
    uint32_t g = 0;            // tiles issued
    uint32_t st = 0, eph = 1;  // stage of tile g; parity of the "empty" phase it must wait for
    for (uint32_t d = 0;; ++d) {
        const uint32_t slot = d % kItemSlots;
        if (d >= kItemSlots && !ws_wait(item_empty + slot, ((d / kItemSlots) - 1u) & 1u, &sh.f.abort, p.err)) break;
        const int32_t w =
            ld_volatile_u32(&sh.f.abort) ? p.nsegs : static_cast<int32_t>(atomicAdd(p.work_counter, 1u));
        sh.items[slot] = w;
        mbar_arrive(item_full + slot);  // release: the consumers read items[slot] after their wait
        if (w >= p.nsegs) break;
        TaskView tv;
        const SegGeom G = seg_geom<TW, kScale>(p, w, &tv);
        if (G.skip) continue;
        bool ok = true;
        const uint32_t slen = ws_sample_len(p, G.td, static_cast<uint32_t>(THREADS / 32) * TW);
        const uint32_t ns = ws_sample_rank(G.td, slen) != 0 ? slen / TW : 0u;
        const uint32_t nch = slen / kSampleChunkLen;
        const uint32_t nt = G.ntiles + ns;
        const int64_t mis = static_cast<int64_t>((reinterpret_cast<uintptr_t>(tv.data) >> 2) & 3);
        for (uint32_t i = 0; i < nt; ++i, ++g) {
            if (g >= static_cast<uint32_t>(STAGES) && !ws_wait(empty + st, eph, &sh.f.abort, p.err)) {
                ok = false;
                break;
            }
            float* dst = ring + static_cast<size_t>(st) * TW;
            if (i < ns) {
                mbar_arrive_expect_tx(full + st, TW * 4u);
                for (uint32_t c = 0; c < kChunksPerTile; ++c)
                    bulk_load_hint(dst + c * kSampleChunkLen,
                                   tv.data + ws_sample_pos(tv.len, mis, i * kChunksPerTile + c, nch), kSampleChunkLen * 4u,
                                   full + st, pol);
            } else {
                const int64_t e0 = static_cast<int64_t>(i - ns) * TW;
                const uint32_t bytes = static_cast<uint32_t>(min(static_cast<int64_t>(TW), G.nvec * 4 - e0)) * 4u;
                mbar_arrive_expect_tx(full + st, bytes);
                bulk_load_hint(dst, tv.data + G.a0 + e0, bytes, full + st, pol);
            }
            if (++st == static_cast<uint32_t>(STAGES)) { st = 0; eph ^= 1u; }
        }
        if (!ok) break;
    }
    // Copies still in flight must land before the CTA exits.
    for (uint32_t j = g > static_cast<uint32_t>(STAGES) ? g - STAGES : 0u; j < g; ++j)
        mbar_wait_bounded(full + j % STAGES, (j / STAGES) & 1u, kWaitPolls);
}

// Fast test of a warp tile: bit 4 j + e of the result is set when component
// e of this lane's float4 j passes the fast filter (the float compare against
// the threshold's value).  Float4 j of the lane is src[j * 32 + lane]; only
// the first nv float4 of the tile are elements: the others read as ff.pad4
// and their bits are cleared (pad4 passes when the threshold is -inf).
template <int J, bool kScale>
__device__ __forceinline__ uint32_t ws_elem_mask(const float4* src, uint32_t nv, uint32_t lane, const FastFilter& ff,
                                                 float scaler) {
    float4 x[J];
    uint32_t valid = 0xffffffffu;
    if (nv >= 32u * J) {
#pragma unroll
        for (int j = 0; j < J; ++j) x[j] = src[j * 32 + lane];
    } else {
        valid = 0;
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const bool in = j * 32 + lane < nv;
            x[j] = in ? src[j * 32 + lane] : ff.pad4;
            valid |= in ? (0xfu << (4 * j)) : 0u;
        }
    }
    if constexpr (kScale) {
#pragma unroll
        for (int j = 0; j < J; ++j) {
            x[j].x = __fsub_rn(x[j].x, scaler); x[j].y = __fsub_rn(x[j].y, scaler);
            x[j].z = __fsub_rn(x[j].z, scaler); x[j].w = __fsub_rn(x[j].w, scaler);
        }
    }
    uint32_t em = 0;
    if (ff.dir == 0u && !ff.nan_pass) {
#pragma unroll
        for (int j = 0; j < J; ++j)
            em |= (static_cast<uint32_t>(x[j].x >= ff.t) | (static_cast<uint32_t>(x[j].y >= ff.t) << 1) |
                   (static_cast<uint32_t>(x[j].z >= ff.t) << 2) | (static_cast<uint32_t>(x[j].w >= ff.t) << 3))
                  << (4 * j);
    } else if (!ff.nan_pass) {
#pragma unroll
        for (int j = 0; j < J; ++j)
            em |= (static_cast<uint32_t>(x[j].x <= ff.tr) | (static_cast<uint32_t>(x[j].y <= ff.tr) << 1) |
                   (static_cast<uint32_t>(x[j].z <= ff.tr) << 2) | (static_cast<uint32_t>(x[j].w <= ff.tr) << 3))
                  << (4 * j);
    } else if (ff.dir == 0u) {
#pragma unroll
        for (int j = 0; j < J; ++j)
            em |= (static_cast<uint32_t>(!(x[j].x < ff.t)) | (static_cast<uint32_t>(!(x[j].y < ff.t)) << 1) |
                   (static_cast<uint32_t>(!(x[j].z < ff.t)) << 2) | (static_cast<uint32_t>(!(x[j].w < ff.t)) << 3))
                  << (4 * j);
    } else {
#pragma unroll
        for (int j = 0; j < J; ++j)
            em |= (static_cast<uint32_t>(!(x[j].x > ff.tr)) | (static_cast<uint32_t>(!(x[j].y > ff.tr)) << 1) |
                   (static_cast<uint32_t>(!(x[j].z > ff.tr)) << 2) | (static_cast<uint32_t>(!(x[j].w > ff.tr)) << 3))
                  << (4 * j);
    }
    return em & valid;
}

// Places candidates of a warp tile in the warp's region.  Element bit
// b = 4 j + e of a lane is component e of its float4 j (src[j * 32 + lane]).
// `elems` lists this lane's elements: from the fast filter (exact == false,
// placed as they are) or offered again after a shrink (exact == true, kept
// only if their composite beats thr).  One warp scan gives every lane its
// slots; returns the element bits that found no room.
template <int J, bool kScale>
__device__ __forceinline__ uint32_t ws_place(const float4* src, uint32_t elems, bool exact, uint32_t qb, uint32_t pos0,
                                             uint64_t thr, float scaler, const ScoreParams& sp, uint64_t* region,
                                             uint32_t R, uint32_t& wcnt, uint32_t lane) {
    const float* srcf = reinterpret_cast<const float*>(src);
    uint32_t pm = elems;
    if (exact) {
        uint32_t keep = 0;
        for (uint32_t m = pm; m; m &= m - 1) {
            const int b = __ffs(m) - 1;
            const uint32_t q = static_cast<uint32_t>(b >> 2) * 32u + lane;
            const uint64_t c = make_composite(score_of<kScale>(__float_as_uint(srcf[q * 4 + (b & 3)]), scaler, sp),
                                              pos0 + (qb + q) * 4u + (b & 3));
            if (c > thr) keep |= 1u << b;
        }
        pm = keep;
    }
    const uint32_t n = __popc(pm);
    const uint32_t incl = warp_inclusive_scan<true>(n);
    uint32_t slot = wcnt + incl - n;
    wcnt += __shfl_sync(kFullMask, incl, 31);
    uint32_t om = 0;
    for (uint32_t m = pm; m; m &= m - 1) {
        const int b = __ffs(m) - 1;
        const uint32_t q = static_cast<uint32_t>(b >> 2) * 32u + lane;
        const uint64_t c = make_composite(score_of<kScale>(__float_as_uint(srcf[q * 4 + (b & 3)]), scaler, sp),
                                          pos0 + (qb + q) * 4u + (b & 3));
        if (slot < R) region[slot] = c;
        else om |= 1u << b;
        ++slot;
    }
    return om;
}

// Candidate append regions of the warp-specialised form, all consumer warps
// together: the narrow form (2 consumer warps, 7 blocks per SM) has half.
__host__ __device__ constexpr uint32_t ws_region_entries(int ncw) {
    return ncw == 2 ? kRegionEntries / 2 : kRegionEntries;
}
// Blocks per SM the form is compiled for (its register budget).
__host__ __device__ constexpr int ws_blocks_per_sm(int ncw) { return ncw == 2 ? 7 : (ncw >= 8 ? 3 : 4); }

template <int NCW, int J, int STAGES, bool kScale>
__global__ void __launch_bounds__((NCW + 1) * 32, ws_blocks_per_sm(NCW)) fused_ws_kernel(FusedParams p) {
    grid_dep_wait();  // launched after the previous kernel of the call (state clear or sampler)
    grid_dep_launch();  // every block of the grid is resident (grid <= resident blocks)
    constexpr int THREADS = NCW * 32;             // consumer threads
    constexpr uint32_t TW = 128u * J;             // elements per warp tile (one ring stage)
    constexpr uint32_t TW4 = TW / 4;              // float4 per warp tile
    constexpr uint32_t REG = ws_region_entries(NCW);
    constexpr uint32_t R = REG / NCW;  // append region of each consumer warp
    static_assert(J * 4 <= 32, "element bits of a lane fit in 32 bits");
    // Ring tile g sits in stage g % STAGES and belongs to warp g % NCW.  With
    // STAGES a multiple of NCW every stage belongs to one warp, so the tile a
    // warp waits for always follows, in its stage, a tile that warp has
    // already consumed: the stage's barrier is then never more than one phase
    // behind the awaited one, which a parity wait requires.  (With shared
    // stages a warp could wait on phase n while phase n - 1, another warp's
    // tile, was still in flight, and the parity test would pass at once.)
    static_assert(STAGES % NCW == 0, "every ring stage belongs to one consumer warp");
    // ws_sample_len keeps the sample to one tile per consumer warp; its group
    // maxima (redo path) fit in the candidate buffer.
    static_assert(static_cast<uint32_t>(NCW) * TW / 4 <= REG, "group maxima fit in the candidate buffer");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ WsShared<THREADS> sh;
    float* ring = reinterpret_cast<float*>(smem_raw);
    uint64_t* s_buf = reinterpret_cast<uint64_t*>(smem_raw + static_cast<size_t>(STAGES) * TW * 4);
    uint64_t* full = s_buf + p.cap;
    uint64_t* empty = full + STAGES;
    uint64_t* item_full = empty + STAGES;
    uint64_t* item_empty = item_full + kItemSlots;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const uint32_t lane = tid & 31;

    if (p.retry && *reinterpret_cast<volatile const uint32_t*>(p.fail_any) == 0u) return;  // nothing to redo
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        for (int s = 0; s < kItemSlots; ++s) {
            mbar_init(item_full + s, 1);
            mbar_init(item_empty + s, 1);
        }
        fence_mbar_init();
        sh.f.abort = 0;
        sh.req = 0;
        sh.arrived = 0;
    }
    __syncthreads();  // the only barrier the producer warp takes part in
    if (warp == NCW) {
        if (lane == 0) ws_producer<THREADS, J, STAGES, kScale>(p, ring, full, empty, item_full, item_empty, sh);
        return;
    }

    // ---- consumer warps ----------------------------------------------------
    const uint32_t lt = lanemask_lt();
    const uint32_t cap = p.cap;
    const uint32_t cap_s = p.cap - REG;  // settled region [0, cap_s), then the warp regions
    uint64_t* region = s_buf + cap_s + warp * R;
    const uint32_t compact_at = cap - max(cap / 8, static_cast<uint32_t>(THREADS) + 8u);
    const float4* ring4 = reinterpret_cast<const float4*>(ring);
    uint32_t gbase = 0;  // ring index of the current item's first tile (same in every consumer warp)

    for (uint32_t d = 0;; ++d) {
        const uint32_t slot = d % kItemSlots;
        if (tid == 0) {
            int32_t w = p.nsegs;
            if (ws_wait(item_full + slot, (d / kItemSlots) & 1u, &sh.f.abort, p.err)) w = sh.items[slot];
            if (ld_volatile_u32(&sh.f.abort)) w = p.nsegs;
            sh.cur = w;
        }
        block_sync<THREADS>();
        const int32_t w = sh.cur;
        if (w >= p.nsegs) break;
        TaskView tv;
        const SegGeom G = seg_geom<TW, kScale>(p, w, &tv);
        if (!G.skip) {
            const int t = G.sg.task;
            const FusedTask& td = G.td;
            const uint32_t k = tv.k;
            const uint32_t mid_keep = k + (cap_s - k) / 2;
            const bool multi = td.nseg > 1;
            // Flush mode: candidates above the seeded threshold go straight to the
            // task's candidate region; no per-segment selection (merge.cuh finishes).
            const bool flush = multi && (td.flags & kTaskFlush) != 0 && !p.retry;
            uint64_t* fdst = p.cand + (td.cbase >= 0 ? td.cbase : 0);
            const uint32_t fcap = static_cast<uint32_t>(td.nseg) * p.kmax;
            const float scaler = kScale ? task_scaler(tv.data, 0, tv.len, 1) : 0.0f;
            const uint32_t pos0 = static_cast<uint32_t>(G.a0);
            const uint32_t nvec = static_cast<uint32_t>(G.nvec);
            const uint32_t ntiles = G.ntiles;
            const uint32_t slen = ws_sample_len(p, td, static_cast<uint32_t>(NCW) * TW);
            const uint32_t sample_r = ws_sample_rank(td, slen);
            const uint32_t ns = sample_r != 0 ? slen / TW : 0u;
            const float4* gsrc = reinterpret_cast<const float4*>(tv.data + G.a0);
            uint32_t wcnt = 0;  // entries in this warp's region (same in all its lanes)

            bool thr_used = false;  // the last attempt started from a sampled threshold
            for (int attempt = 0; attempt < 3; ++attempt) {
                // attempt 0 streams the ring from the sample's threshold (rank
                // sample_r).  A single-segment task whose threshold turned out
                // too high re-reads the segment from global memory: attempt 1
                // from a far more conservative rank of the same sample (read
                // again from global memory), attempt 2 with no threshold.
                const bool from_ring = attempt == 0;
                uint64_t thr = 0;
                thr_used = false;
                if (multi) {
                    if (tid == 0) sh.thr = load_volatile_u64(p.gthr + t);
                    block_sync<THREADS>();
                    thr = sh.thr;
                } else if (ns != 0 && attempt < 2) {
                    // Group maxima of 4 consecutive samples, then the exact
                    // rr-th largest of them (warp 0): every element scoring at
                    // least that passes.
                    const uint32_t rr = attempt == 0 ? sample_r : 2 * sample_r + 8;
                    const uint32_t ngroups = slen / 4;
                    const uint32_t s = (static_cast<uint32_t>(warp) + NCW - gbase % NCW) % NCW;  // my sample tile
                    if (attempt == 1) {
                        const int64_t mis = static_cast<int64_t>((reinterpret_cast<uintptr_t>(tv.data) >> 2) & 3);
                        const uint32_t nch = slen / kSampleChunkLen;
                        for (uint32_t gi = tid; gi < ngroups; gi += THREADS) {
                            const uint32_t c = gi / (kSampleChunkLen / 4), e = gi % (kSampleChunkLen / 4);
                            const float4 f = *reinterpret_cast<const float4*>(
                                tv.data + ws_sample_pos(tv.len, mis, c, nch) + 4 * e);
                            const uint32_t a = score_of<kScale>(__float_as_uint(f.x), scaler, tv.sp);
                            const uint32_t b = score_of<kScale>(__float_as_uint(f.y), scaler, tv.sp);
                            const uint32_t cc = score_of<kScale>(__float_as_uint(f.z), scaler, tv.sp);
                            const uint32_t ee = score_of<kScale>(__float_as_uint(f.w), scaler, tv.sp);
                            s_buf[gi] = static_cast<uint64_t>(max(max(a, b), max(cc, ee))) << 32;
                        }
                    } else if (s < ns) {
                        const uint32_t gt = gbase + s;
                        const uint32_t st = gt % STAGES;
                        const bool ok = ws_warp_wait(full + st, (gt / STAGES) & 1u, &sh.f.abort, p.err);
                        const float4* src = ring4 + static_cast<size_t>(st) * TW4;
#pragma unroll
                        for (int j = 0; j < J; ++j) {
                            const float4 f = ok ? src[j * 32 + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
                            const uint32_t a = score_of<kScale>(__float_as_uint(f.x), scaler, tv.sp);
                            const uint32_t b = score_of<kScale>(__float_as_uint(f.y), scaler, tv.sp);
                            const uint32_t c = score_of<kScale>(__float_as_uint(f.z), scaler, tv.sp);
                            const uint32_t e = score_of<kScale>(__float_as_uint(f.w), scaler, tv.sp);
                            s_buf[s * TW4 + j * 32 + lane] = static_cast<uint64_t>(max(max(a, b), max(c, e))) << 32;
                        }
                        __syncwarp();
                        if (lane == 0) mbar_arrive(empty + st);
                    }
                    block_sync<THREADS>();  // the maxima are in s_buf
                    if (warp == 0 && rr <= ngroups / 2) {
                        const uint32_t sv = ngroups <= 512 ? warp_rank_value<16>(s_buf, ngroups, rr)
                                                           : warp_rank_value<32>(s_buf, ngroups, rr);
                        thr = sv != 0u ? (static_cast<uint64_t>(sv) << 32) - 1u : 0ull;
                    }
                    thr_used = true;  // when warp 0 found one (published below)
                }
                block_sync<THREADS>();
                if (tid == 0) {
                    sh.f.cnt = 0;
                    sh.thr = thr;
                    sh.req = 0;
                    sh.arrived = 0;
                }
                block_sync<THREADS>();
                thr = sh.thr;  // warp 0's sampled threshold reaches every warp
                thr_used = thr_used && thr != 0;
                wcnt = 0;

                // Head [s0, a0) and tail [a1, s1): fewer than 4 elements each (warp 0).
                if (warp == 0) {
                    const int nh = static_cast<int>(G.a0 - G.s0), nt = static_cast<int>(G.s1 - G.a1);
                    bool pass = false;
                    uint64_t c = 0;
                    int64_t q = -1;
                    if (tid < nh) q = G.s0 + tid;
                    else if (tid >= 8 && tid - 8 < nt) q = G.a1 + (tid - 8);
                    if (q >= 0) {
                        const uint32_t bits = __float_as_uint(tv.data[q]);
                        c = make_composite(score_of<kScale>(bits, scaler, tv.sp), static_cast<uint32_t>(q));
                        pass = c > thr;
                    }
                    const uint32_t m = __ballot_sync(kFullMask, pass);
                    if (pass) region[__popc(m & lt)] = c;
                    wcnt = __popc(m);
                }

                FastFilter ff = make_fast_filter<kScale>(thr, tv.sp, scaler);
                uint64_t gnext = 0;  // lane 0: latest global threshold, read a tile ahead of its use
                // My data tiles: i = i0, i0 + NCW, ... (tile i is ring tile gbase + ns + i).
                uint32_t i = (static_cast<uint32_t>(warp) + NCW - (gbase + ns) % NCW) % NCW;
                uint32_t om = 0;     // element bits of tile i that found no room (tile i is held)
                uint32_t mine = 0;   // my tiles done (threshold refresh cadence)
                uint32_t polls = 0;
                bool arrived_me = false;
                for (;;) {
                    if (__any_sync(kFullMask, ld_volatile_u32(&sh.req) != 0u)) {
                        // Block-wide shrink: gather the regions, keep a few more
                        // than k, raise the threshold; every consumer warp is here.
                        block_sync<THREADS>();
                        gather_regions<THREADS, R>(s_buf, cap_s, wcnt, sh.f);
                        const uint64_t kf = shrink_mid<THREADS>(p, k, mid_keep, s_buf, sh.f);
                        if (tid == 0) {
                            if (kf != 0 && kf - 1 > sh.thr) sh.thr = kf - 1;
                            if (multi && kf != 0)
                                atomicMax(reinterpret_cast<unsigned long long*>(p.gthr + t), kf - 1);
                            sh.req = 0;
                        }
                        block_sync<THREADS>();
                        if (sh.thr > thr) {
                            thr = sh.thr;
                            ff = make_fast_filter<kScale>(thr, tv.sp, scaler);
                        }
                        if (__any_sync(kFullMask, om != 0u)) {
                            // Place the rest of the held tile.
                            const uint32_t gt = gbase + ns + i;
                            const uint32_t st = gt % STAGES;
                            const float4* src = from_ring ? ring4 + static_cast<size_t>(st) * TW4 : gsrc + i * TW4;
                            const uint32_t qb = i * TW4;
                            om = ws_place<J, kScale>(src, om, true, qb, pos0, thr, scaler, tv.sp, region, R, wcnt,
                                                     lane);
                            if (__any_sync(kFullMask, om != 0u)) {
                                if (lane == 0) st_volatile_u32(&sh.req, 1u);
                            } else {
                                __syncwarp();
                                if (from_ring && lane == 0) mbar_arrive(empty + st);
                                i += NCW;
                                ++mine;
                            }
                        }
                        continue;
                    }
                    if (i < ntiles) {
                        const uint32_t gt = gbase + ns + i;
                        const uint32_t st = gt % STAGES;
                        const float4* src;
                        if (from_ring) {
                            if (!__all_sync(kFullMask, mbar_try_wait(full + st, (gt / STAGES) & 1u))) {
                                // Not there yet: poll again from the top of the loop,
                                // which serves shrink requests (a requester may hold
                                // the stage this tile needs).  Bounded.
                                ++polls;
                                if (__any_sync(kFullMask, polls >= kWaitPolls ||
                                                              ((polls & 63u) == 0u &&
                                                               ld_volatile_u32(&sh.f.abort) != 0u))) {
                                    // The tile never came: the CTA aborts (the host
                                    // reports the error word; results are void).
                                    if (lane == 0) {
                                        record_error(p.err, kErrTimeout);
                                        st_volatile_u32(&sh.f.abort, 1u);
                                    }
                                    polls = 0;
                                    i += NCW;
                                }
                                continue;
                            }
                            polls = 0;
                            src = ring4 + static_cast<size_t>(st) * TW4;
                        } else {
                            src = gsrc + i * TW4;
                        }
                        const uint32_t qb = i * TW4;
                        const uint32_t nv = nvec - qb < TW4 ? nvec - qb : TW4;
                        const uint32_t em = ws_elem_mask<J, kScale>(src, nv, lane, ff, scaler);
                        if (__any_sync(kFullMask, em != 0u)) {
                            om = ws_place<J, kScale>(src, em, false, qb, pos0, thr, scaler, tv.sp, region, R, wcnt,
                                                     lane);
                            if (flush) {
                                // Write the region out and place the rest (bounded:
                                // each round places up to R of at most 32 * 4 * J).
                                for (int rounds = 0; rounds < 64 && __any_sync(kFullMask, om != 0u); ++rounds) {
                                    ws_flush(region, wcnt, R, fdst, p.task_cnt + t, fcap, p.fail + t, p.fail_any,
                                             lane);
                                    om = ws_place<J, kScale>(src, om, true, qb, pos0, thr, scaler, tv.sp, region, R,
                                                             wcnt, lane);
                                }
                            } else if (__any_sync(kFullMask, om != 0u)) {
                                if (lane == 0) st_volatile_u32(&sh.req, 1u);
                                continue;  // tile i stays held until its candidates are placed
                            }
                        }
                        __syncwarp();
                        if (from_ring && lane == 0) mbar_arrive(empty + st);
                        i += NCW;
                        ++mine;
                        if (multi) {
                            // Segments of the task raise a shared threshold: read it
                            // every other tile and use it on the next one.
                            if ((mine & 1u) == 1u) {
                                if (lane == 0) gnext = load_volatile_u64(p.gthr + t);
                            } else {
                                const uint64_t gg = __shfl_sync(kFullMask, gnext, 0);
                                if (gg > thr) {
                                    thr = gg;
                                    ff = make_fast_filter<kScale>(thr, tv.sp, scaler);
                                }
                            }
                        }
                        continue;
                    }
                    // All my tiles are done: wait (serving shrink requests) until
                    // every consumer warp is done.
                    if (!arrived_me) {
                        if (flush) ws_flush(region, wcnt, R, fdst, p.task_cnt + t, fcap, p.fail + t, p.fail_any, lane);
                        arrived_me = true;
                        if (lane == 0) atomicAdd(&sh.arrived, 1u);
                    }
                    if (__any_sync(kFullMask, ld_volatile_u32(&sh.arrived) >= static_cast<uint32_t>(NCW))) break;
                    __nanosleep(32);
                }
                block_sync<THREADS>();
                if (flush) break;  // the candidates are in the task's region
                gather_regions<THREADS, R>(s_buf, cap_s, wcnt, sh.f);  // all candidates now in [0, sh.f.cnt)
                if (!multi) {
                    const uint32_t want = tv.len < static_cast<int64_t>(k) ? static_cast<uint32_t>(tv.len) : k;
                    if (sh.f.cnt < want && thr_used) continue;  // threshold too high: redo from a lower one
                }
                break;
            }
            gbase += ns + ntiles;  // the ring tiles of this item (the redo reads global memory)

            if (flush && (td.flags & kTaskFinishHere) != 0u) {
                // The block that flushes a task's last segment finishes it:
                // the region, filtered by the task's threshold (kept within
                // the buffer by shrinks), then the k best, sorted and written.
                __threadfence();  // this block's region writes before its arrival
                block_sync<THREADS>();
                if (tid == 0) {
                    const uint32_t done = atomicAdd(p.task_done + t, 1u);
                    sh.f.last = (done == static_cast<uint32_t>(td.nseg - 1)) ? 1u : 0u;
                }
                block_sync<THREADS>();
                if (sh.f.last) {
                    __threadfence();
                    if (tid == 0) {
                        sh.f.cnt = 0;
                        sh.f.gthr = load_volatile_u64(p.gthr + t);
                        sh.f.base = __ldcg(p.task_cnt + t);
                    }
                    block_sync<THREADS>();
                    const uint64_t gt = sh.f.gthr;
                    const uint32_t cregion = static_cast<uint32_t>(td.nseg) * p.kmax;
                    // A count above the region means a flush overflowed it and
                    // already flagged the task for the retry launch.
                    const uint32_t n = sh.f.base <= cregion ? sh.f.base : 0u;
                    const unsigned long long* csrc = reinterpret_cast<const unsigned long long*>(p.cand + td.cbase);
                    if (n <= cap) {
                        // The region fits the buffer: every load in flight at
                        // once, no shrinking, no barrier between the loads.
                        constexpr int U = 4;
                        for (uint32_t b0 = 0; b0 < n; b0 += U * THREADS) {
                            uint64_t c[U];
#pragma unroll
                            for (int u = 0; u < U; ++u) {
                                const uint32_t ii = b0 + static_cast<uint32_t>(u) * THREADS + tid;
                                c[u] = (ii < n) ? __ldcg(csrc + ii) : 0ull;
                            }
#pragma unroll
                            for (int u = 0; u < U; ++u) {
                                const uint32_t ii = b0 + static_cast<uint32_t>(u) * THREADS + tid;
                                warp_append((ii < n) && c[u] > gt, c[u], s_buf, &sh.f.cnt, cap, p.err);
                            }
                        }
                    } else {
                        for (uint32_t b0 = 0; b0 < n; b0 += THREADS) {
                            {
                                const uint32_t ii = b0 + tid;
                                const uint64_t c = (ii < n) ? __ldcg(csrc + ii) : 0ull;
                                warp_append((ii < n) && c > gt, c, s_buf, &sh.f.cnt, cap, p.err);
                            }
                            block_sync<THREADS>();
                            const uint32_t cnt_now = sh.f.cnt;
                            block_sync<THREADS>();
                            if (cnt_now > compact_at) shrink_mid<THREADS>(p, k, mid_keep, s_buf, sh.f);
                        }
                    }
                    block_sync<THREADS>();
                    const uint32_t want = tv.len < static_cast<int64_t>(k) ? static_cast<uint32_t>(tv.len) : k;
                    if (sh.f.base > cregion) {
                    } else if (sh.f.cnt < want) {
                        // The sampled threshold was above the task's k-th
                        // composite: the retry launch recomputes the task.
                        if (tid == 0) {
                            p.fail[t] = 1u;
                            atomicExch(p.fail_any, 1u);
                        }
                    } else {
                        finish_candidates<THREADS, kScale>(p, tv, s_buf, sh.f);
                    }
                }
            } else if (flush) {
                // merge.cuh selects the task's k best from its candidate region.
            } else if (!multi && (td.flags & kTaskDefer) != 0u && !p.retry && p.defer_q != nullptr) {
                // Deferred finish: the candidates (at least min(len, k), all in
                // [0, sh.f.cnt) after the gather) to the task's region, then the
                // task into the ready queue; a block with no streaming left
                // selects, sorts and writes the row (finisher loop below).
                const uint32_t cnt = buffer_count<THREADS>(p, sh.f);
                uint64_t* dst = p.cand + td.cbase;
                for (uint32_t i = tid; i < cnt; i += THREADS) dst[i] = s_buf[i];
                if (tid == 0) p.task_cnt[t] = cnt;
                __threadfence();  // the region and the count before the publication
                block_sync<THREADS>();
                if (tid == 0) {
                    const uint32_t j = atomicAdd(p.defer_ctr, 1u);
                    if (j < p.ndefer) atomicExch(p.defer_q + j, static_cast<uint32_t>(t) + 1u);
                    else record_error(p.err, kErrInternal);
                }
            } else if (!multi) {
                finish_candidates<THREADS, kScale>(p, tv, s_buf, sh.f);
            } else {
                // Multi-segment task: publish this segment's k-th composite, append
                // the survivors to the task's candidate region, count the segment.
                uint64_t kth = 0;
                shrink_final<THREADS>(p, k, s_buf, sh.f, &kth);
                if (tid == 0) {
                    if (kth != 0) atomicMax(reinterpret_cast<unsigned long long*>(p.gthr + t), kth - 1);
                    sh.f.gthr = load_volatile_u64(p.gthr + t);
                }
                block_sync<THREADS>();
                {
                    const uint64_t gt = sh.f.gthr;
                    const uint32_t cnt = sh.f.cnt;
                    uint64_t* dst = p.cand + td.cbase;
                    const uint32_t cregion = static_cast<uint32_t>(td.nseg) * p.kmax;
                    for (uint32_t b0 = 0; b0 < cnt; b0 += THREADS) {
                        const uint32_t ii = b0 + tid;
                        const uint64_t c = (ii < cnt) ? s_buf[ii] : 0ull;
                        const bool keep = (ii < cnt) && c > gt;
                        uint32_t total;
                        const uint32_t off = block_exclusive_scan<THREADS>(keep ? 1u : 0u, &total, sh.f.bs);
                        if (tid == 0 && total) sh.f.base = atomicAdd(p.task_cnt + t, total);
                        block_sync<THREADS>();
                        if (keep) {
                            const uint32_t o = sh.f.base + off;
                            if (o < cregion) dst[o] = c;
                            else record_error(p.err, kErrCapacity);
                        }
                        block_sync<THREADS>();
                    }
                }
                __threadfence();
                block_sync<THREADS>();
                if (tid == 0) {
                    const uint32_t done = atomicAdd(p.task_done + t, 1u);
                    sh.f.last = (done == static_cast<uint32_t>(td.nseg - 1)) ? 1u : 0u;
                }
                block_sync<THREADS>();
                if (sh.f.last) {
                    // Last segment of the task: merge all segments' survivors.
                    __threadfence();
                    if (tid == 0) {
                        sh.f.cnt = 0;
                        sh.f.gthr = load_volatile_u64(p.gthr + t);
                        sh.f.base = __ldcg(p.task_cnt + t);
                    }
                    block_sync<THREADS>();
                    const uint64_t gt = sh.f.gthr;
                    const uint32_t cregion = static_cast<uint32_t>(td.nseg) * p.kmax;
                    const uint32_t n = sh.f.base < cregion ? sh.f.base : cregion;
                    const unsigned long long* csrc = reinterpret_cast<const unsigned long long*>(p.cand + td.cbase);
                    for (uint32_t b0 = 0; b0 < n; b0 += THREADS) {
                        {
                            const uint32_t ii = b0 + tid;
                            const uint64_t c = (ii < n) ? __ldcg(csrc + ii) : 0ull;
                            warp_append((ii < n) && c > gt, c, s_buf, &sh.f.cnt, cap, p.err);
                        }
                        block_sync<THREADS>();
                        const uint32_t cnt_now = sh.f.cnt;
                        block_sync<THREADS>();
                        if (cnt_now > compact_at) shrink_mid<THREADS>(p, k, mid_keep, s_buf, sh.f);
                    }
                    block_sync<THREADS>();
                    const uint32_t m = shrink_final<THREADS>(p, k, s_buf, sh.f, &kth);
                    if (m < k && (td.flags & kTaskSampled) && !p.retry) {
                        // The sampled threshold was above the task's k-th composite.
                        if (tid == 0) {
                            p.fail[t] = 1u;
                            atomicExch(p.fail_any, 1u);
                        }
                    } else {
                        if (m != k && tid == 0) record_error(p.err, kErrInternal);
                        finish_task<THREADS, !kScale>(p, tv, s_buf, m < k ? m : k, sh.f);
                    }
                }
            }
        }
        block_sync<THREADS>();  // the item is finished: its slot may be reused
        if (tid == 0) mbar_arrive(item_empty + slot);
    }

    // Finisher loop: no streaming work is left for this block; finish the
    // deferred tasks that other blocks (or this one) queued, in queue order.
    // Every queued slot is filled exactly once by the block that streamed
    // the task, and all blocks of the grid are resident, so each wait ends;
    // it is bounded all the same.
    if (p.defer_q != nullptr && !p.retry) {
        for (;;) {
            if (tid == 0) {
                int32_t job = -1;
                if (!ld_volatile_u32(&sh.f.abort)) {
                    const uint32_t j = atomicAdd(p.defer_ctr + 1, 1u);
                    if (j < p.ndefer) job = static_cast<int32_t>(j);
                }
                uint32_t v = 0;
                if (job >= 0) {
                    for (uint32_t polls = 0; polls < kWaitPolls; ++polls) {
                        v = ld_volatile_u32(p.defer_q + job);
                        if (v != 0u) break;
                        __nanosleep(64);
                    }
                    if (v == 0u) {
                        record_error(p.err, kErrTimeout);
                        st_volatile_u32(&sh.f.abort, 1u);
                    }
                }
                sh.f.last = v;
            }
            block_sync<THREADS>();
            const uint32_t v = sh.f.last;
            block_sync<THREADS>();
            if (v == 0u) break;
            __threadfence();  // the region is read after its publication
            const int t = static_cast<int>(v - 1u);
            const FusedTask td = p.tasks[t];
            const TaskView tv = task_view<kScale>(p, t, td);
            uint32_t n = __ldcg(p.task_cnt + t);
            if (n > p.cap) {  // never expected: the streaming block kept at most cap
                if (tid == 0) record_error(p.err, kErrCapacity);
                n = p.cap;
            }
            const unsigned long long* src = reinterpret_cast<const unsigned long long*>(p.cand + td.cbase);
#pragma unroll 4
            for (uint32_t i = tid; i < n; i += THREADS) s_buf[i] = __ldcg(src + i);
            if (tid == 0) sh.f.cnt = n;
            block_sync<THREADS>();
            finish_candidates<THREADS, kScale>(p, tv, s_buf, sh.f);
        }
    }
}

}  // namespace radik
