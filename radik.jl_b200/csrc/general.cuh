// general.cuh -- multi-pass exact top-k: the reference's pass structure
// (src/algorithm.jl:214-352) as separate launches, used for any k (including
// k too large for an on-chip candidate buffer) and as the plain per-call path.
//
//   pass 0  hist over the input of digit = composite bits 63..52 (the 12-bit
//           first digit of count_bin_ex_kernel!, count_bin.jl:78-203)
//           -> rank search per task (select_bin.jl:268-348)
//           -> compaction over the input: composites in higher bins are
//              winners, members of the selected bin become candidates
//              (select_candidate_ex_kernel!, select_candidate.jl:233-375,
//              fused with the strict part of filter_kernel!, filter.jl:111)
//   pass p  the same over the candidate buffer with the next digit of the
//           64-bit composite (bits 51..40, 39..32 -- the 12/8-bit passes 2 and
//           3 of the reference -- then 31..20, 19..8, 7..0 of ~position, which
//           resolve ties at the k-th key by lowest position)
//   final   per task: sort of the k winners by output order, index mapping,
//           padding (src/algorithm.jl:340-365).
// A task finishes as soon as its selected bin holds exactly the residual
// rank: all of the bin's members are winners then.
#pragma once

#include "block_ops.cuh"
#include "fused.cuh"

namespace radik {

struct PlainState {
    uint32_t active;  // 1 while the task still needs passes
    uint32_t r;       // residual rank inside the current candidate set
    uint32_t ncand;   // candidates in the current ping buffer
    uint32_t nout;    // winners emitted
    uint32_t bin;     // selected bin of the current pass
    uint32_t bincnt;  // members of the selected bin
    uint32_t allwin;  // the selected bin's members are all winners
    uint32_t nnext;   // candidates written to the pong buffer by this pass
};

struct PlainParams {
    const float* data;
    const FusedTask* tasks;   // start/len of each task (slot0/nseg unused)
    const FusedSeg* segs;     // input segments (all tasks)
    int32_t nsegs;
    int32_t ntasks;
    uint32_t k;
    ScoreParams sp;
    uint32_t* hist;           // [T][4096]
    PlainState* st;           // [T]
    uint64_t* out_stage;      // [T][k]
    uint64_t* cand[2];        // [N] each, task t's region starts at tasks[t].start
    uint32_t* err;
};

// Pass-0 digit histogram over the input segments (persistent grid).
template <int THREADS, bool kScale>
__global__ void __launch_bounds__(THREADS) plain_hist_input(PlainParams p) {
    __shared__ uint32_t h[4096];
    for (int w = blockIdx.x; w < p.nsegs; w += gridDim.x) {
        const FusedSeg sg = p.segs[w];
        const FusedTask td = p.tasks[sg.task];
        if (td.len <= static_cast<int64_t>(p.k)) continue;  // copy-all task (filter.jl:272)
        for (int i = threadIdx.x; i < 4096; i += THREADS) h[i] = 0;
        __syncthreads();
        const float scaler = kScale ? task_scaler(p.data, td.start, td.len, 1) : 0.0f;
        const float* src = p.data + td.start + sg.pos;
        // Four independent loads per thread in flight, then their bins.
        for (int64_t i0 = 0; i0 < sg.len; i0 += 4 * THREADS) {
            uint32_t bits[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int64_t i = i0 + u * THREADS + threadIdx.x;
                bits[u] = i < sg.len ? __float_as_uint(src[i]) : 0u;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (i0 + u * THREADS + threadIdx.x < sg.len) atomicAdd(&h[score_of<kScale>(bits[u], scaler, p.sp) >> 20], 1u);
        }
        __syncthreads();
        uint32_t* gh = p.hist + static_cast<int64_t>(sg.task) * 4096;
        for (int i = threadIdx.x; i < 4096; i += THREADS)
            if (h[i]) atomicAdd(gh + i, h[i]);
        __syncthreads();
    }
}

// Rank search of one pass for every task with work; one CTA per task.
// pass 0 initialises the state from k and the task length.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) plain_select(PlainParams p, int pass, int width) {
    __shared__ BlockScratch<THREADS> s;
    const int t = blockIdx.x;
    PlainState* st = p.st + t;
    const FusedTask td = p.tasks[t];
    if (pass == 0) {
        if (td.len <= static_cast<int64_t>(p.k)) {
            if (threadIdx.x == 0) { st->active = 0; st->r = 0; st->ncand = 0; st->allwin = 0; }
            return;
        }
        if (threadIdx.x == 0) { st->active = 1; st->r = p.k; st->ncand = static_cast<uint32_t>(td.len); }
        __syncthreads();
    }
    if (!st->active) return;
    const uint32_t nb = 1u << width;
    uint32_t* gh = p.hist + static_cast<int64_t>(t) * 4096;
    const uint32_t per = (nb + THREADS - 1) / THREADS;
    // thread i owns bins (from the top) [i*per, (i+1)*per)
    uint32_t sum = 0;
    for (uint32_t j = 0; j < per; ++j) {
        uint32_t rb = threadIdx.x * per + j;
        if (rb < nb) sum += gh[nb - 1 - rb];
    }
    // Read the state before the scan: its barriers order every thread's reads
    // before the one thread that owns rank r rewrites r and the bin below.
    const uint32_t r = st->r;
    const uint32_t ncand = st->ncand;
    uint32_t total;
    uint32_t before = block_exclusive_scan<THREADS>(sum, &total, s);
    if (threadIdx.x == 0 && total != ncand) record_error(p.err, kErrInternal);
    if (before < r && r <= before + sum) {
        uint32_t rr = r - before;
        for (uint32_t j = 0; j < per; ++j) {
            uint32_t rb = threadIdx.x * per + j;
            if (rb >= nb) break;
            uint32_t b = nb - 1 - rb;
            uint32_t c = gh[b];
            if (c >= rr && c > 0) {
                st->bin = b;
                st->bincnt = c;
                st->r = rr;
                st->allwin = (c == rr) ? 1u : 0u;
                st->nnext = 0;
                break;
            }
            rr -= c;
        }
    }
    __syncthreads();  // every reader of the row is done
    // clear the histogram row for the next pass
    for (uint32_t i = threadIdx.x; i < nb; i += THREADS) gh[i] = 0;
}

__device__ __forceinline__ void emit_winner(const PlainParams& p, int t, uint64_t c) {
    uint32_t slot = atomicAdd(&p.st[t].nout, 1u);
    if (slot < p.k) p.out_stage[static_cast<int64_t>(t) * p.k + slot] = c;
    else record_error(p.err, kErrCapacity);
}

// Pass-0 compaction over the input segments.
template <int THREADS, bool kScale>
__global__ void __launch_bounds__(THREADS) plain_compact_input(PlainParams p) {
    for (int w = blockIdx.x; w < p.nsegs; w += gridDim.x) {
        const FusedSeg sg = p.segs[w];
        const int t = sg.task;
        const FusedTask td = p.tasks[t];
        const bool copy_all = td.len <= static_cast<int64_t>(p.k);
        const float scaler = kScale ? task_scaler(p.data, td.start, td.len, 1) : 0.0f;
        const uint32_t bin = copy_all ? 0u : p.st[t].bin;
        const bool allwin = copy_all ? true : (p.st[t].allwin != 0);
        uint32_t* nnext = &p.st[t].nnext;
        // Four independent loads per thread in flight, then their tests.
        for (int64_t i0 = 0; i0 < sg.len; i0 += 4 * THREADS) {
            uint32_t bits[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int64_t i = i0 + u * THREADS + threadIdx.x;
                bits[u] = i < sg.len ? __float_as_uint(p.data[td.start + sg.pos + i]) : 0u;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int64_t i = i0 + u * THREADS + threadIdx.x;
                if (i >= sg.len) continue;
                const uint32_t s = score_of<kScale>(bits[u], scaler, p.sp);
                const uint64_t c = make_composite(s, static_cast<uint32_t>(sg.pos + i));
                const uint32_t d = s >> 20;
                if (copy_all || d > bin || (d == bin && allwin)) {
                    emit_winner(p, t, c);
                } else if (d == bin) {
                    uint32_t slot = atomicAdd(nnext, 1u);
                    if (slot < static_cast<uint32_t>(td.len)) p.cand[0][td.start + slot] = c;
                    else record_error(p.err, kErrCapacity);
                }
            }
        }
    }
}

// Histogram of a candidate pass (digit = (c >> sh) & (2^width - 1)).
template <int THREADS>
__global__ void __launch_bounds__(THREADS) plain_hist_cand(PlainParams p, int t0, int src, int sh, int width) {
    __shared__ uint32_t h[4096];
    const int t = t0 + blockIdx.y;
    if (!p.st[t].active) return;
    const uint32_t n = p.st[t].ncand;
    const uint32_t nb = 1u << width;
    for (uint32_t i = threadIdx.x; i < nb; i += THREADS) h[i] = 0;
    __syncthreads();
    const uint64_t* c = p.cand[src] + p.tasks[t].start;
    const uint64_t mask = nb - 1;
    for (uint32_t i = blockIdx.x * THREADS + threadIdx.x; i < n; i += gridDim.x * THREADS)
        atomicAdd(&h[(c[i] >> sh) & mask], 1u);
    __syncthreads();
    uint32_t* gh = p.hist + static_cast<int64_t>(t) * 4096;
    for (uint32_t i = threadIdx.x; i < nb; i += THREADS)
        if (h[i]) atomicAdd(gh + i, h[i]);
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS) plain_compact_cand(PlainParams p, int t0, int src, int sh, int width) {
    const int t = t0 + blockIdx.y;
    if (!p.st[t].active) return;
    const uint32_t n = p.st[t].ncand;
    const uint32_t bin = p.st[t].bin;
    const bool allwin = p.st[t].allwin != 0;
    const uint64_t mask = (1ull << width) - 1;
    const int64_t base = p.tasks[t].start;
    const uint64_t* c = p.cand[src] + base;
    uint64_t* nx = p.cand[src ^ 1] + base;
    for (uint32_t i = blockIdx.x * THREADS + threadIdx.x; i < n; i += gridDim.x * THREADS) {
        uint64_t v = c[i];
        uint32_t d = static_cast<uint32_t>((v >> sh) & mask);
        if (d > bin || (d == bin && allwin)) {
            emit_winner(p, t, v);
        } else if (d == bin) {
            uint32_t slot = atomicAdd(&p.st[t].nnext, 1u);
            if (slot < n) nx[slot] = v;
            else record_error(p.err, kErrCapacity);
        }
    }
}

// After a compaction: the pong buffer becomes the candidate set; tasks whose
// bin members were all winners are done.  One thread per task.
__global__ void plain_advance(PlainParams p, uint32_t* any_active) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= p.ntasks) return;
    PlainState* st = p.st + t;
    if (!st->active) return;
    if (st->allwin) {
        st->active = 0;
        if (st->nout != p.k) record_error(p.err, kErrInternal);
        return;
    }
    uint32_t n = st->nnext;
    if (n != st->bincnt) record_error(p.err, kErrInternal);
    const uint32_t len = static_cast<uint32_t>(p.tasks[t].len);
    st->ncand = n < len ? n : len;  // candidates past the task's region were dropped
    st->nnext = 0;
    atomicOr(any_active, 1u);
}

// Sort the winners of each task, map indices, pad.  One CTA per task.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) plain_finalize(PlainParams p, FusedParams fp, uint64_t* scratch) {
    extern __shared__ __align__(16) uint64_t s_buf[];
    __shared__ FusedShared<THREADS> sh;
    const int t = blockIdx.x;
    const FusedTask td = p.tasks[t];
    const TaskView tv = task_view<false>(fp, t, td);
    const uint32_t m = td.len < static_cast<int64_t>(p.k) ? static_cast<uint32_t>(td.len) : p.k;
    if (threadIdx.x == 0 && p.st[t].nout != m) record_error(p.err, kErrInternal);
    const uint64_t* row = p.out_stage + static_cast<int64_t>(t) * p.k;
    if (m <= kBitonicMax) {
        for (uint32_t i = threadIdx.x; i < m; i += THREADS) s_buf[i] = row[i];
        __syncthreads();
        finish_task<THREADS>(fp, tv, s_buf, m, sh);
    } else {
        // Sort keys built in the task's staging row, radix-sorted with a
        // scratch row, then the shared row writer.
        uint64_t* a = p.out_stage + static_cast<int64_t>(t) * p.k;
        uint64_t* b = scratch + static_cast<int64_t>(t) * p.k;
        for (uint32_t i = threadIdx.x; i < m; i += THREADS) {
            uint32_t pos = composite_pos(a[i]);
            if (pos >= static_cast<uint64_t>(td.len)) { record_error(p.err, kErrBounds); pos = 0; }
            uint32_t bits = __float_as_uint(tv.data[pos]);
            a[i] = output_sort_key(bits, pos, tv.sp, tv.ascend);
        }
        __syncthreads();
        uint32_t* wd = reinterpret_cast<uint32_t*>(s_buf);
        uint32_t* db = wd + (THREADS / 32) * 256;
        uint64_t* sorted = radix_sort_u64<THREADS>(a, b, m, sh.bs, wd, db);
        __syncthreads();
        write_row<THREADS>(fp, tv, sorted, m);
    }
}

}  // namespace radik
