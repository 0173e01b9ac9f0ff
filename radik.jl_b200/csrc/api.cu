// api.cu -- C ABI of the engine (include/radik.h): workspace, launch plans,
// the fused single-read path, the multi-pass path and the stage entry points.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <utility>
#include <vector>

#include "../../include/radik.h"
#include "fused.cuh"
#include "fused_ws.cuh"
#include "general.cuh"
#include "merge.cuh"
#include "sample.cuh"
#include "stages.cuh"

using namespace radik;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define RADIK_CUDA(call)                                                                         \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) return fail(RADIK_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

// Every device and pinned-host allocation the library makes goes through
// these two, which count them (radik_alloc_count).
std::atomic<uint64_t> g_alloc_count{0};

cudaError_t counted_malloc(void** p, size_t n) {
    g_alloc_count.fetch_add(1, std::memory_order_relaxed);
    return cudaMalloc(p, n);
}

template <typename T>
cudaError_t counted_malloc_host(T** p, size_t n) {
    g_alloc_count.fetch_add(1, std::memory_order_relaxed);
    return cudaMallocHost(reinterpret_cast<void**>(p), n);
}

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    // Grows to at least b bytes; `grow` > 1 allocates that much more, so a
    // buffer that keeps growing (the request server's) reallocates -- and
    // synchronises the device -- only rarely.
    cudaError_t ensure(size_t b, double grow = 1.0) {
        if (b <= bytes) return cudaSuccess;
        if (p) { cudaFree(p); p = nullptr; bytes = 0; }
        size_t nb = b < 256 ? 256 : b;
        if (grow > 1.0) nb = std::max(nb, static_cast<size_t>(static_cast<double>(nb) * grow));
        cudaError_t e = counted_malloc(&p, nb);
        if (e == cudaSuccess) bytes = nb;
        return e;
    }
    void release() { if (p) cudaFree(p); p = nullptr; bytes = 0; }
    template <typename T> T* as(size_t byte_off = 0) const {
        return reinterpret_cast<T*>(static_cast<char*>(p) + byte_off);
    }
};

struct DeviceInfo {
    int sms = 148;
    int max_smem_optin = 227 * 1024;
};

DeviceInfo device_info() {
    static std::mutex mu;
    static int cached_dev = -1;
    static DeviceInfo cached;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if (dev != cached_dev) {
        DeviceInfo d;
        cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&d.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        cached = d;
        cached_dev = dev;
    }
    return cached;
}

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
size_t round_down_entries(size_t n) { return n / 64 * 64; }

// ---------------------------------------------------------------------------
// Fused kernel dispatch
// ---------------------------------------------------------------------------
using FusedKernel = void (*)(FusedParams);
constexpr int kStages = 6;  // TMA ring depth of the fused kernel

template <int T, int V, bool S>
FusedKernel fused_ptr() { return fused_topk_kernel<T, V, kStages, S>; }

FusedKernel pick_fused(int threads, int vec, bool scale) {
    if (threads == 256 && vec == 8) return scale ? fused_ptr<256, 8, true>() : fused_ptr<256, 8, false>();
    if (threads == 256 && vec == 16) return scale ? fused_ptr<256, 16, true>() : fused_ptr<256, 16, false>();
    if (threads == 512 && vec == 8) return scale ? fused_ptr<512, 8, true>() : fused_ptr<512, 8, false>();
    return nullptr;
}

// Warp-specialised form: `threads` consumer threads plus one producer warp;
// a ring of `stages` warp tiles of 128 * j elements (j float4 per lane).
template <int NCW, int J, int ST, bool S>
FusedKernel fused_ws_ptr() { return fused_ws_kernel<NCW, J, ST, S>; }

// Shapes: consumer threads, float4 per lane in a warp tile (j), ring stages.
FusedKernel pick_fused_ws(int threads, int j, int stages, bool scale) {
    if (threads == 256 && j == 8 && stages == 16) return scale ? fused_ws_ptr<8, 8, 16, true>() : fused_ws_ptr<8, 8, 16, false>();
    if (threads == 256 && j == 4 && stages == 24) return scale ? fused_ws_ptr<8, 4, 24, true>() : fused_ws_ptr<8, 4, 24, false>();
    if (threads == 128 && j == 8 && stages == 8) return scale ? fused_ws_ptr<4, 8, 8, true>() : fused_ws_ptr<4, 8, 8, false>();
    if (threads == 128 && j == 8 && stages == 12) return scale ? fused_ws_ptr<4, 8, 12, true>() : fused_ws_ptr<4, 8, 12, false>();
    if (threads == 64 && j == 8 && stages == 4) return scale ? fused_ws_ptr<2, 8, 4, true>() : fused_ws_ptr<2, 8, 4, false>();
    return nullptr;
}

// Dynamic shared memory of the fused kernel: TMA ring, candidate buffer,
// one mbarrier per ring stage.
size_t fused_smem(uint32_t cap, int threads, int vec) {
    return static_cast<size_t>(kStages) * threads * vec * sizeof(float) + static_cast<size_t>(cap) * 8 + kStages * 8;
}

// Warp-specialised form: ring, candidate buffer, "full" and "empty" mbarrier
// per stage, the item ring's barriers.
size_t fused_ws_smem(uint32_t cap, int j, int stages) {
    const size_t st = static_cast<size_t>(stages);
    return st * 128 * j * sizeof(float) + static_cast<size_t>(cap) * 8 + (2 * st + 2 * kItemSlots) * 8;
}

using MergeKernel = void (*)(FusedParams, const int32_t*);
constexpr int kMergeThreads = 1024;  // one block per flush-mode task

MergeKernel pick_merge(bool scale) {
    return scale ? merge_topk_kernel<kMergeThreads, true> : merge_topk_kernel<kMergeThreads, false>;
}
MergeKernel pick_rank(bool scale) { return scale ? rank_write_kernel<true> : rank_write_kernel<false>; }
constexpr size_t kRankSmem = sizeof(uint64_t) * (kRankMaxK + 2);

using SampleKernel = void (*)(FusedParams, const SampleJob*, uint64_t*, uint32_t*);

SampleKernel pick_sample(bool scale) {
    return scale ? sample_threshold_kernel<256, true> : sample_threshold_kernel<256, false>;
}

int env_int(const char* name, int dflt) {
    const char* v = std::getenv(name);
    return (v && *v) ? std::atoi(v) : dflt;
}

// Tunable shape of a plan.  Defaults are the measured best for the common
// cases; radik_ws_autotune picks another per batch shape; environment
// variables (RADIK_WS, RADIK_WST, RADIK_WSJ, RADIK_WSS, RADIK_WS_SAMPLE,
// RADIK_SEG_DIV, RADIK_DEFER, RADIK_SEG_MIN) override both, for experiments.
struct TuneConfig {
    int form = -1;          // -1 automatic, 0 barrier form, 1 warp-specialised form
    int ws_threads = 128;   // warp-specialised: consumer threads
    int ws_j = 8;           // float4 per lane in a warp tile
    int ws_stages = 8;      // ring stages (a multiple of the consumer warps)
    int sample_max = 2048;  // single-segment sample (elements)
    int seg_div = 3;        // work items per resident block when splitting tasks
    int defer = -1;         // deferred finish of single-segment tasks: -1 automatic, 0 no, 1 yes
    int seg_min_tiles = 0;  // shortest segment of a split task in 2048-element tiles; 0 automatic
    int plain_sched = 0;    // multi-pass path: digit schedule of the candidate passes (kPlainSchedules)
    int bar_threads = 0;    // barrier form's block: 256 or 512 threads; 0 automatic (512 for 4096 < k <= 8192)
    bool operator==(const TuneConfig& o) const {
        return form == o.form && ws_threads == o.ws_threads && ws_j == o.ws_j && ws_stages == o.ws_stages &&
               sample_max == o.sample_max && seg_div == o.seg_div && defer == o.defer &&
               seg_min_tiles == o.seg_min_tiles && plain_sched == o.plain_sched && bar_threads == o.bar_threads;
    }
};

// Digit schedules of the multi-pass path after its fixed 12-bit first digit
// (composite bits 63..52): the (shift, width) of each candidate pass over the
// remaining 52 bits, widths <= 12 (4096-bin histograms).  More bits per pass
// mean fewer passes (each a histogram, a bin search, a compaction and a host
// read of the "any task active" flag); fewer bits mean smaller histograms.
struct PlainPass {
    int sh, w;
};
constexpr int kPlainSchedules = 4;
constexpr int kPlainMaxPasses = 7;
struct PlainSchedule {
    int n;
    PlainPass pass[kPlainMaxPasses];
};
constexpr PlainSchedule kPlainSchedule[kPlainSchedules] = {
    {5, {{40, 12}, {32, 8}, {20, 12}, {8, 12}, {0, 8}}},                    // score 12+8, position 12+12+8
    {5, {{40, 12}, {28, 12}, {16, 12}, {4, 12}, {0, 4}}},                   // 12-bit digits
    {5, {{41, 11}, {30, 11}, {19, 11}, {8, 11}, {0, 8}}},                   // 11-bit digits
    {7, {{44, 8}, {36, 8}, {28, 8}, {20, 8}, {12, 8}, {4, 8}, {0, 4}}},    // 8-bit digits
};

TuneConfig with_env(TuneConfig c) {
    c.form = env_int("RADIK_WS", c.form);
    c.ws_threads = env_int("RADIK_WST", c.ws_threads);
    c.ws_j = env_int("RADIK_WSJ", c.ws_j);
    c.ws_stages = env_int("RADIK_WSS", c.ws_stages);
    c.sample_max = env_int("RADIK_WS_SAMPLE", c.sample_max);
    c.seg_div = std::max(1, env_int("RADIK_SEG_DIV", c.seg_div));
    c.defer = env_int("RADIK_DEFER", c.defer);
    c.seg_min_tiles = std::max(0, env_int("RADIK_SEG_MIN", c.seg_min_tiles));
    c.plain_sched = env_int("RADIK_PLAIN_SCHED", c.plain_sched);
    c.bar_threads = env_int("RADIK_THREADS", c.bar_threads);
    if (c.bar_threads != 256 && c.bar_threads != 512) c.bar_threads = 0;
    if (c.sample_max != 2048 && c.sample_max != 4096) c.sample_max = 2048;
    if (c.plain_sched < 0 || c.plain_sched >= kPlainSchedules) c.plain_sched = 0;
    return c;
}

}  // namespace

// ---------------------------------------------------------------------------
// Workspace and plan
// ---------------------------------------------------------------------------
struct PlanKey {
    std::vector<int64_t> lens;
    int64_t k = -1;
    uint32_t flags = 0;
    int idx_bytes = 0;
    TuneConfig tune;
    bool operator==(const PlanKey& o) const {
        return k == o.k && flags == o.flags && idx_bytes == o.idx_bytes && lens == o.lens && tune == o.tune;
    }
};

struct Plan {
    PlanKey key;
    bool valid = false;
    bool fused = false;
    bool ws_form = false;   // warp-specialised fused kernel
    int ws_stages = 16;     // its ring stages
    int ws_sample_max = 2048;    // its single-segment sample (elements)
    int threads = 256, vec = 16;
    int launch_threads = 256;  // threads plus the producer warp of the warp-specialised form
    uint32_t cap = 0;
    int grid = 0;
    size_t smem = 0;
    int64_t T = 0, N = 0, cand_entries = 0, sample_entries = 0;
    int32_t nsegs = 0;
    size_t tasks_off = 0, segs_off = 0, jobs_off = 0, merge_off = 0;
    // Retry launch (barrier form, full candidate buffer) for sampled tasks.
    uint32_t retry_cap = 0;
    size_t retry_smem = 0;
    int retry_grid = 0, retry_threads = 256, retry_vec = 8;
    // Merge kernel for flush-mode tasks.
    uint32_t merge_cap = 0;
    size_t merge_smem = 0;
    std::vector<FusedTask> tasks;
    std::vector<FusedSeg> segs;
    std::vector<SampleJob> jobs;
    // One sampling block per task (sample_one_kernel), every job's whole sample in it.
    bool sample_one = false;
    std::vector<int32_t> merge_tasks;
    // Deferred single-segment tasks (finished by blocks with no streaming left).
    std::vector<int32_t> defer_tasks;
};

struct radik_ws {
    int device = 0;
    int64_t n = 0;          // longest task served (RadiKWorkspace n)
    int64_t num_tasks = 0;  // largest batch (RadiKWorkspace num_tasks)
    int index_bytes = 4;
    double grow = 1.0;          // device buffers grow by this factor over a call's need (the server's: 1.5)
    cudaStream_t last_stream = nullptr;
    uint32_t* h_err = nullptr;  // pinned
    char* h_stage = nullptr;    // pinned staging of plan descriptors (stream-ordered uploads)
    size_t h_stage_bytes = 0;
    DevBuf state;     // StateLayout: per-call counters and thresholds
    DevBuf desc;      // tasks + segs + sample jobs of the plan
    DevBuf cand;      // fused: candidate regions of multi-segment tasks
    DevBuf samples;   // fused: sampled composites
    DevBuf scratch;   // sort scratch
    DevBuf hist;      // plain: [T][4096]
    DevBuf pstate;    // plain: [T] PlainState
    DevBuf stage;     // plain: [T][k]
    DevBuf pcand[2];  // plain: [N] each
    DevBuf io_in, io_idx, io_vout, io_iout;  // host-buffer entry point
    Plan plan;
    // Configurations chosen by radik_ws_autotune, by batch shape.
    std::vector<std::pair<PlanKey, TuneConfig>> tuned;
};

namespace {

// Device state of one workspace.  The header holds the sticky error word and
// the work counters; everything after `err` is zeroed before every call.
struct StateLayout {
    // kAny: multi-pass path: some task still active; fused path: some task failed.
    static constexpr size_t kErr = 0, kWork = 4, kWorkRetry = 8, kAny = 12, kHeader = 16;
    size_t gthr, gthr_r, done, done_r, cnt, cnt_r, fail, sdone, rk, dctr, dq, bytes;
    explicit StateLayout(int64_t T) {
        const size_t t8 = round_up(sizeof(uint64_t) * static_cast<size_t>(std::max<int64_t>(T, 1)), 16);
        const size_t t4 = round_up(sizeof(uint32_t) * static_cast<size_t>(std::max<int64_t>(T, 1)), 16);
        gthr = kHeader;
        gthr_r = gthr + t8;
        done = gthr_r + t8;
        done_r = done + t4;
        cnt = done_r + t4;
        cnt_r = cnt + t4;
        fail = cnt_r + t4;
        sdone = fail + t4;
        rk = sdone + t4;
        dctr = rk + t4;   // deferred tasks queued / claimed
        dq = dctr + 16;   // queue of deferred tasks
        bytes = dq + t4;
    }
};

uint32_t* err_ptr(radik_ws* ws) { return ws->state.as<uint32_t>(StateLayout::kErr); }

// Shared-buffer capacity of the fused kernel: a settled region that holds
// k entries plus the slack of a mid-stream shrink, followed by the per-warp
// candidate regions (kRegionEntries).  Candidates that find no room are
// re-offered after a shrink, so no region needs to hold a whole tile.
size_t fused_cap(size_t k, size_t tile, int threads, size_t regions = kRegionEntries) {
    (void)tile;
    size_t cap_s = round_up(k + std::max<size_t>(k / 4, 512), 64);
    size_t cap = cap_s + regions;
    size_t p2 = 1;
    while (p2 < std::min<size_t>(k, kBitonicMax)) p2 <<= 1;
    cap = std::max(cap, p2);
    cap = std::max(cap, k + (static_cast<size_t>(threads) / 32 * 256 + 256) / 2 + 8);
    return round_up(cap, 64);
}

// Segment length: about seg_div work items per resident block, at least
// min_tiles tiles (64 by default; a short single task runs faster on more,
// smaller, sampled segments), a multiple of the tile (env RADIK_SEG
// overrides).
int64_t pick_seg_len(int64_t N, int64_t resident, size_t tile, bool fused, int seg_div, int min_tiles) {
    int64_t seg_len = env_int("RADIK_SEG", 0);
    if (seg_len <= 0) {
        const int64_t target = N / std::max<int64_t>(1, seg_div * resident);
        seg_len = std::max<int64_t>(static_cast<int64_t>(min_tiles) * static_cast<int64_t>(tile), target);
    }
    seg_len = static_cast<int64_t>(round_up(static_cast<size_t>(seg_len), tile));
    if (!fused) seg_len = std::max<int64_t>(seg_len, 1 << 16);
    return seg_len;
}

// Splits the tasks into segments of seg_len (the fused path splits a task
// only when it is longer than seg_len and than k) and decides which split
// tasks are sampled: fills tasks, segs, jobs, cand_entries, sample_entries.
void segment_tasks(Plan& np, const int64_t* lens, int64_t T, int64_t k, uint32_t flags, int64_t seg_len,
                   bool fused) {
    const size_t kk = static_cast<size_t>(k);
    np.tasks.resize(T);
    np.segs.clear();
    np.jobs.clear();
    np.cand_entries = 0;
    np.sample_entries = 0;
    int64_t off = 0;
    const uint32_t tflags = ((flags & RADIK_LARGEST) ? kTaskLargest : 0u) | ((flags & RADIK_ASCEND) ? kTaskAscend : 0u);
    const bool allow_sample = env_int("RADIK_SAMPLE", 1) != 0;
    for (int64_t t = 0; t < T; ++t) {
        FusedTask& td = np.tasks[t];
        td.start = off;
        td.len = lens[t];
        td.k = static_cast<uint32_t>(k);
        td.flags = tflags;
        td.pad_ = 0;
        int64_t nseg = 1;
        if (fused && td.len > seg_len && td.len > k) nseg = (td.len + seg_len - 1) / seg_len;
        if (!fused) nseg = std::max<int64_t>(1, (td.len + seg_len - 1) / seg_len);
        td.nseg = static_cast<int32_t>(nseg);
        td.cbase = -1;
        if (fused && nseg > 1) {
            td.cbase = np.cand_entries;
            np.cand_entries += nseg * static_cast<int64_t>(kk);
            // Seed the global threshold from a sample when the segments' own
            // k-th values would leave a large merge (many segments, large k).
            // Sampling blocks and chunks per block: fewer of them when k is a
            // large share of the task, so that lam (and the rank r below) stays
            // within what a block ranks.
            int64_t njobs = std::min<int64_t>(128, std::max<int64_t>(8, td.len >> 21));
            int64_t nchunks = 8;
            auto lam_of = [&](int64_t jobs, int64_t ch) {
                return static_cast<double>(kk) * static_cast<double>(jobs * ch * kSampleChunk) /
                       static_cast<double>(td.len);
            };
            while (njobs > 1 && lam_of(njobs, nchunks) > 160.0) njobs = std::max<int64_t>(1, njobs / 2);
            while (nchunks > 1 && lam_of(njobs, nchunks) > 160.0) nchunks /= 2;
            const int64_t S = njobs * nchunks * kSampleChunk;
            const int64_t stride = (td.len / (njobs * nchunks)) & ~int64_t(3);
            const double lam = static_cast<double>(kk) * static_cast<double>(S) / static_cast<double>(td.len);
            // Rank of the threshold among the sample's group maxima: the
            // threshold is too high only when r or more sampled elements lie
            // above the task's k-th, a Poisson(lam) tail; lam + max(3 sqrt(lam)
            // + 6, 5 sqrt(lam)) keeps it below about 1e-5 for small lam and
            // 5 sigma for large lam (a large k on long rows: a served batch
            // holds hundreds of such tasks, each failure a recomputation).  Each
            // sampling block keeps its top r of its 1024 maxima and the last
            // one ranks the union in shared memory: r <= 256, at most a quarter
            // of a block's maxima, and njobs * r <= 8192.
            const double margin = std::max(3.0 * std::sqrt(lam) + 6.0, 5.0 * std::sqrt(lam));
            const int64_t r = static_cast<int64_t>(std::ceil(lam + margin));
            const bool r_fits = r <= 256 && r <= nchunks * (kSampleChunk / 4) / 4 && njobs * r <= 8192;
            if (allow_sample && nseg * static_cast<int64_t>(kk) >= 8192 && stride >= kSampleChunk + 4 && r_fits) {
                td.flags |= kTaskSampled;
                for (int64_t j = 0; j < njobs; ++j) {
                    SampleJob sj;
                    sj.task = static_cast<int32_t>(t);
                    sj.job_in_task = static_cast<int32_t>(j);
                    sj.njobs = static_cast<int32_t>(njobs);
                    sj.r = static_cast<int32_t>(r);
                    sj.nchunks = static_cast<int32_t>(nchunks);
                    sj.pad_ = 0;
                    sj.pos0 = j * nchunks * stride;
                    sj.stride = stride;
                    sj.out_base = np.sample_entries;
                    np.jobs.push_back(sj);
                }
                np.sample_entries += njobs * r;
            }
        }
        for (int64_t sgi = 0; sgi < nseg; ++sgi) {
            FusedSeg sg;
            sg.pos = static_cast<int32_t>(sgi * seg_len);
            const int64_t e = std::min(td.len, (sgi + 1) * seg_len);
            sg.len = static_cast<int32_t>(e - sgi * seg_len);
            sg.task = static_cast<int32_t>(t);
            sg.seg_in_task = static_cast<int32_t>(sgi);
            np.segs.push_back(sg);
        }
        off += td.len;
    }
    // When every sampled task's sample fits one block, one block per task
    // reads and ranks it (no sample buffer, no merge between blocks).
    np.sample_one = false;
    if (!np.jobs.empty() && env_int("RADIK_SAMPLE_ONE", 1) != 0) {
        bool fits = true;
        for (const SampleJob& sj : np.jobs)
            fits = fits && static_cast<int64_t>(sj.njobs) * sj.nchunks <= kSampleOneMaxChunks;
        if (fits) {
            std::vector<SampleJob> one;
            for (const SampleJob& sj : np.jobs)
                if (sj.job_in_task == 0) {
                    SampleJob o1 = sj;
                    o1.nchunks = sj.njobs * sj.nchunks;
                    o1.njobs = 1;
                    o1.pos0 = 0;
                    o1.out_base = 0;
                    one.push_back(o1);
                }
            np.jobs.swap(one);
            np.sample_entries = 0;
            np.sample_one = true;
        }
    }
    // Longest work first (uneven batches), stable on task order.
    std::stable_sort(np.segs.begin(), np.segs.end(),
                     [](const FusedSeg& a, const FusedSeg& b) { return a.len > b.len; });
    np.nsegs = static_cast<int32_t>(np.segs.size());
}

// Sets a kernel's dynamic shared memory limit and returns how many of its
// blocks fit on an SM (0 when it does not fit at all).
int set_smem_and_occupancy(const void* fn, int threads, size_t smem) {
    static std::mutex attr_mu;
    std::lock_guard<std::mutex> lock(attr_mu);
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return occ;
}

// Host half of a launch plan: kernel configuration, segment table, sample
// jobs and descriptor offsets.  Allocates no device memory.
int plan_shape(const int64_t* lens, int64_t T, int64_t k, uint32_t flags, Plan& np, const TuneConfig& tc) {
    const DeviceInfo di = device_info();
    np.T = T;
    np.N = 0;
    for (int64_t t = 0; t < T; ++t) np.N += lens[t];
    const bool scale = (flags & RADIK_WITHSCALE) != 0;
    const bool plain = (flags & RADIK_PLAIN) != 0;
    const size_t kk = static_cast<size_t>(k);
    const size_t smem_max = static_cast<size_t>(di.max_smem_optin) - 4096;

    // Shapes.  Barrier form (fused.cuh): bar_threads x RADIK_VEC tiles, 512
    // threads for 4096 < k <= 8192 (their final selection and sort of up to
    // 16 keys per thread: 256 x 32,768 at k = 8192 0.427 -> 0.390 ms,
    // 256 x 131,072 0.782 -> 0.682 ms, the served stream +18 %; at k = 4096
    // 256 threads stay faster, 0.160 against 0.200 ms; beyond 8192 the
    // 256-thread plan's choice of the multi-pass path is kept).
    // Warp-specialised form (fused_ws.cuh): RADIK_WST consumer threads, warp
    // tiles of 128 * RADIK_WSJ elements, RADIK_WSS ring stages.
    const int bar_threads = tc.bar_threads != 0 ? tc.bar_threads : ((kk > 4096 && kk <= 8192) ? 512 : 256);
    const int bar_vec = env_int("RADIK_VEC", 8);
    const int ws_env = tc.form;
    const int ws_j = tc.ws_j;
    const int ws_threads = tc.ws_threads;
    np.ws_stages = tc.ws_stages;
    np.ws_sample_max = tc.sample_max;
    const size_t seg_tile = 2048;  // segments are whole tiles of either form
    // Shortest segment.  A single task too short to give every SM a 64-tile
    // segment is cut into 4-tile segments, sampled, and merged: 2^20 to 2^24
    // elements ran up to 2x faster that way (k up to 1024; a larger k would
    // leave short segments unsampled, every element a candidate).
    const int min_tiles =
        tc.seg_min_tiles > 0 ? tc.seg_min_tiles
                             : ((T == 1 && k <= 1024 && np.N < static_cast<int64_t>(di.sms) * 64 * seg_tile) ? 4 : 64);

    // Segments and samples first, sized for the warp-specialised form's
    // residency (four blocks per SM).
    segment_tasks(np, lens, T, k, flags, pick_seg_len(np.N, 4LL * di.sms, seg_tile, !plain, tc.seg_div, min_tiles),
                  !plain);
    bool all_flush = T > 0;  // every non-empty task is split and sampled
    for (int64_t t = 0; t < T; ++t)
        if (lens[t] > 0 && (np.tasks[t].flags & kTaskSampled) == 0) all_flush = false;

    // Kernel form: the warp-specialised kernel when at least three of its
    // blocks fit on an SM, else the form that keeps more bytes in flight per
    // SM (a large k makes the candidate buffer the larger part of shared
    // memory).  In the warp-specialised form, sampled split tasks run in
    // flush mode and need no candidate buffer of k entries, so a batch made
    // only of them gets the minimum buffer.  RADIK_WS=0/1 forces a form.
    uint32_t cap_bar = static_cast<uint32_t>(fused_cap(kk, static_cast<size_t>(bar_threads) * bar_vec, bar_threads));
    if (kk > kBitonicMax) {
        // Room for the radix sort's second key buffer and digit counters in
        // shared memory too (finish_task); such a block has an SM to itself
        // either way.
        const size_t want = round_up(2 * kk + (static_cast<size_t>(bar_threads) / 32 * 256 + 256) / 2 + 64, 64);
        if (fused_smem(want, bar_threads, bar_vec) <= smem_max) cap_bar = std::max<uint32_t>(cap_bar, want);
    }
    const uint32_t cap_ws = static_cast<uint32_t>(fused_cap(all_flush ? 0 : kk, static_cast<size_t>(ws_threads) * ws_j,
                                                            ws_threads, ws_region_entries(ws_threads / 32)));
    {
        const size_t sm_bytes = static_cast<size_t>(di.max_smem_optin) + 1024;  // per SM, a block's reserve included
        const size_t ws_blk = fused_ws_smem(cap_ws, ws_j, np.ws_stages) + 2048;
        const size_t bar_blk = fused_smem(cap_bar, bar_threads, bar_vec) + 2048;
        const size_t ws_occ = std::min<size_t>(static_cast<size_t>(ws_blocks_per_sm(ws_threads / 32)), sm_bytes / ws_blk),
                     bar_occ = std::min<size_t>(3, sm_bytes / bar_blk);
        const size_t ws_ring = static_cast<size_t>(np.ws_stages) * 128 * ws_j * 4;
        const size_t bar_ring = static_cast<size_t>(kStages) * bar_threads * bar_vec * 4;
        const bool ws_auto = ws_occ >= 3 || (ws_occ >= 1 && ws_occ * ws_ring >= bar_occ * bar_ring);
        np.ws_form = ws_env >= 0 ? ws_env != 0 : ws_auto;
    }
    np.threads = np.ws_form ? ws_threads : bar_threads;
    np.vec = np.ws_form ? ws_j : bar_vec;
    np.cap = np.ws_form ? cap_ws : cap_bar;
    np.launch_threads = np.threads + (np.ws_form ? 32 : 0);
    FusedKernel fk = np.ws_form ? pick_fused_ws(np.threads, np.vec, np.ws_stages, scale)
                                : pick_fused(np.threads, np.vec, scale);
    if (!fk) return fail(RADIK_ERR_INVALID, "unsupported RADIK_THREADS/RADIK_VEC/RADIK_WS* combination");
    np.smem = np.ws_form ? fused_ws_smem(np.cap, np.vec, np.ws_stages) : fused_smem(np.cap, np.threads, np.vec);
    np.fused = !plain && np.smem <= smem_max;
    // Tasks that sample need the retry launch (barrier form, full buffer);
    // flush-mode tasks need the merge kernel.
    const bool sampled = !np.jobs.empty();
    np.retry_cap = cap_bar;
    np.retry_smem = fused_smem(cap_bar, bar_threads, bar_vec);
    // The merge block takes nearly all of an SM's shared memory so that a
    // task's whole candidate region (about 3k entries) usually fits at once.
    np.merge_cap = static_cast<uint32_t>(
        std::max(fused_cap(kk, 0, kMergeThreads), round_down_entries((smem_max - 8192) / 8)));
    np.merge_smem = static_cast<size_t>(np.merge_cap) * 8;
    if (np.fused && sampled && (np.retry_smem > smem_max || (np.ws_form && np.merge_smem > smem_max))) np.fused = false;

    int occ = 1;
    if (np.fused) {
        occ = set_smem_and_occupancy(reinterpret_cast<const void*>(fk), np.launch_threads, np.smem);
        if (occ < 1) np.fused = false;
    }
    if (!np.fused || !np.ws_form) {
        // Re-segment for the form that runs.
        occ = std::max(occ, 1);
        segment_tasks(np, lens, T, k, flags,
                      pick_seg_len(np.N, static_cast<int64_t>(occ) * di.sms, seg_tile, np.fused, tc.seg_div,
                                   min_tiles),
                      np.fused);
    }
    const int64_t resident = static_cast<int64_t>(occ) * di.sms;
    np.merge_tasks.clear();
    if (np.fused && np.ws_form)
        for (int64_t t = 0; t < T; ++t)
            if (np.tasks[t].flags & kTaskSampled) {
                np.tasks[t].flags |= kTaskFlush;
                // A small k is finished by the block that flushes the task's
                // last segment (one histogram pass over a few hundred
                // candidates); a large k goes to the merge and rank kernels,
                // which spread its k^2 placement over the GPU.
                if (kk <= kBucketMaxK && env_int("RADIK_FINISH_HERE", 1) != 0)
                    np.tasks[t].flags |= kTaskFinishHere;
                else
                    np.merge_tasks.push_back(static_cast<int32_t>(t));
            }
    // Deferred finish: when a batch has at least as many single-segment
    // tasks as resident blocks, their blocks leave the candidates in a
    // region of cap entries, queue the task and take the next one; blocks
    // with no streaming left finish queued tasks while the others stream.
    np.defer_tasks.clear();
    if (np.fused && np.ws_form && tc.defer != 0) {
        std::vector<int32_t> elig;
        for (int64_t t = 0; t < T; ++t) {
            const FusedTask& td = np.tasks[t];
            if (td.nseg == 1 && td.len > static_cast<int64_t>(kk) && td.len >= 4096 && (td.flags & kTaskSampled) == 0)
                elig.push_back(static_cast<int32_t>(t));
        }
        const bool want = tc.defer > 0 || static_cast<int64_t>(elig.size()) >= resident;
        if (want && !elig.empty()) {
            for (int32_t t : elig) {
                np.tasks[t].flags |= kTaskDefer;
                np.tasks[t].cbase = np.cand_entries;
                np.cand_entries += np.cap;
            }
            np.defer_tasks = std::move(elig);
        }
    }
    np.grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(np.nsegs, resident)));
    const int grid_cap = env_int("RADIK_GRID", 0);  // fewer CTAs than resident (tests: many items per CTA)
    if (grid_cap > 0 && np.fused) np.grid = std::min(np.grid, grid_cap);
    np.retry_grid = 0;
    if (np.fused && !np.jobs.empty()) {
        const int rocc = set_smem_and_occupancy(reinterpret_cast<const void*>(pick_fused(bar_threads, bar_vec, scale)),
                                                bar_threads, np.retry_smem);
        np.retry_grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(np.nsegs, std::max(rocc, 1) * di.sms)));
        if (grid_cap > 0) np.retry_grid = std::min(np.retry_grid, grid_cap);
        np.retry_threads = bar_threads;
        np.retry_vec = bar_vec;
    }
    if (np.fused && !np.merge_tasks.empty()) {
        set_smem_and_occupancy(reinterpret_cast<const void*>(pick_merge(scale)), kMergeThreads, np.merge_smem);
        set_smem_and_occupancy(reinterpret_cast<const void*>(pick_rank(scale)), kRankThreads, kRankSmem);
    }
    np.tasks_off = 0;
    np.segs_off = round_up(sizeof(FusedTask) * T, 256);
    np.jobs_off = np.segs_off + round_up(sizeof(FusedSeg) * np.segs.size(), 256);
    np.merge_off = np.jobs_off + round_up(sizeof(SampleJob) * np.jobs.size(), 256);
    np.valid = true;
    return RADIK_OK;
}

// Size of the descriptor block (tasks, segments, sample jobs, merge lists) of a plan.
size_t plan_desc_bytes(const Plan& pl) { return pl.merge_off + sizeof(int32_t) * pl.merge_tasks.size(); }

// Build the launch plan for a batch shape and size the workspace for it.
// Key of a call's plan: the batch shape and the configuration that applies
// to it (one chosen by radik_ws_autotune for this shape, else the defaults),
// with environment overrides on top.
constexpr uint32_t kPlanFlags = RADIK_LARGEST | RADIK_ASCEND | RADIK_WITHSCALE | RADIK_WITHIDXIN | RADIK_PLAIN;

// Whether a key describes this batch shape (its tuning aside); compares the
// task lengths in place (no copy: calls with a thousand tasks repeat this).
bool key_matches(const PlanKey& q, const int64_t* lens, int64_t T, int64_t k, uint32_t mflags, int idx_bytes) {
    return q.k == k && q.flags == mflags && q.idx_bytes == idx_bytes && static_cast<int64_t>(q.lens.size()) == T &&
           std::equal(q.lens.begin(), q.lens.end(), lens);
}

// Process-wide tuning table: the autotuner's choices for every batch shape it
// has seen (any workspace), keyed by the shape's digest; saved to and loaded
// from a text file (radik_tune_save / radik_tune_load, or the file named by
// RADIK_TUNE_FILE, read at first use and rewritten after each autotuning).
struct TuneEntry {
    uint64_t digest = 0;  // FNV-1a of the task lengths
    int64_t T = 0, N = 0, k = 0;
    uint32_t flags = 0;
    int idx_bytes = 0;
    TuneConfig cfg;
};
std::mutex g_tune_mu;
std::vector<TuneEntry> g_tune;
std::once_flag g_tune_env_once;

uint64_t lens_digest(const int64_t* lens, int64_t T) {
    uint64_t h = 1469598103934665603ull;
    for (int64_t t = 0; t < T; ++t) {
        uint64_t v = static_cast<uint64_t>(lens[t]);
        for (int b = 0; b < 8; ++b) {
            h ^= (v >> (8 * b)) & 0xffu;
            h *= 1099511628211ull;
        }
    }
    return h;
}

TuneEntry tune_entry(const int64_t* lens, int64_t T, int64_t k, uint32_t mflags, int idx_bytes) {
    TuneEntry e;
    e.digest = lens_digest(lens, T);
    e.T = T;
    e.N = std::accumulate(lens, lens + T, int64_t(0));
    e.k = k;
    e.flags = mflags;
    e.idx_bytes = idx_bytes;
    return e;
}

bool same_shape(const TuneEntry& a, const TuneEntry& b) {
    return a.digest == b.digest && a.T == b.T && a.N == b.N && a.k == b.k && a.flags == b.flags &&
           a.idx_bytes == b.idx_bytes;
}

// One line per entry: digest T N k flags idx_bytes, then the configuration.
int tune_write(const char* path) {
    std::FILE* fp = std::fopen(path, "w");
    if (!fp) return -1;
    std::fprintf(fp, "# radik tuning table v1: digest T N k flags idx_bytes form ws_threads ws_j ws_stages "
                     "sample_max seg_div defer seg_min_tiles plain_sched [bar_threads]\n");
    int n = 0;
    for (const TuneEntry& e : g_tune) {
        const TuneConfig& c = e.cfg;
        if (c.bar_threads != 0)
            std::fprintf(fp, "%llu %lld %lld %lld %u %d %d %d %d %d %d %d %d %d %d %d\n",
                         static_cast<unsigned long long>(e.digest), static_cast<long long>(e.T),
                         static_cast<long long>(e.N), static_cast<long long>(e.k), e.flags, e.idx_bytes, c.form,
                         c.ws_threads, c.ws_j, c.ws_stages, c.sample_max, c.seg_div, c.defer, c.seg_min_tiles,
                         c.plain_sched, c.bar_threads);
        else
            std::fprintf(fp, "%llu %lld %lld %lld %u %d %d %d %d %d %d %d %d %d %d\n",
                         static_cast<unsigned long long>(e.digest), static_cast<long long>(e.T),
                         static_cast<long long>(e.N), static_cast<long long>(e.k), e.flags, e.idx_bytes, c.form,
                         c.ws_threads, c.ws_j, c.ws_stages, c.sample_max, c.seg_div, c.defer, c.seg_min_tiles,
                         c.plain_sched);
        ++n;
    }
    return std::fclose(fp) == 0 ? n : -1;
}

void tune_put(const TuneEntry& e) {
    for (TuneEntry& x : g_tune)
        if (same_shape(x, e)) {
            x.cfg = e.cfg;
            return;
        }
    g_tune.push_back(e);
}

// Reads a table written by tune_write; malformed lines are skipped.  Returns
// the entries read, -1 when the file cannot be opened.
int tune_read(const char* path) {
    std::FILE* fp = std::fopen(path, "r");
    if (!fp) return -1;
    char line[512];
    int n = 0;
    while (std::fgets(line, sizeof(line), fp)) {
        if (line[0] == '#') continue;
        unsigned long long dg = 0;
        long long T = 0, N = 0, k = 0;
        unsigned flags = 0;
        TuneEntry e;
        TuneConfig& c = e.cfg;
        const int got = std::sscanf(line, "%llu %lld %lld %lld %u %d %d %d %d %d %d %d %d %d %d %d", &dg, &T, &N, &k,
                                    &flags, &e.idx_bytes, &c.form, &c.ws_threads, &c.ws_j, &c.ws_stages,
                                    &c.sample_max, &c.seg_div, &c.defer, &c.seg_min_tiles, &c.plain_sched,
                                    &c.bar_threads);
        if (got != 15 && got != 16) continue;
        if (got == 15) c.bar_threads = 0;
        if (c.plain_sched < 0 || c.plain_sched >= kPlainSchedules) continue;
        if (c.bar_threads != 0 && c.bar_threads != 256 && c.bar_threads != 512) continue;
        e.digest = dg;
        e.T = T;
        e.N = N;
        e.k = k;
        e.flags = flags;
        tune_put(e);
        ++n;
    }
    std::fclose(fp);
    return n;
}

void tune_env_load() {
    std::call_once(g_tune_env_once, [] {
        const char* path = std::getenv("RADIK_TUNE_FILE");
        if (path && *path) {
            std::lock_guard<std::mutex> lock(g_tune_mu);
            tune_read(path);
        }
    });
}

// The configuration for a batch shape: the one radik_ws_autotune chose for
// it in this workspace, else in any workspace of the process (or a loaded
// table), else the defaults; environment overrides on top.
TuneConfig shape_config(const radik_ws* ws, const int64_t* lens, int64_t T, int64_t k, uint32_t mflags,
                        int idx_bytes) {
    TuneConfig tc;
    bool found = false;
    for (const auto& e : ws->tuned)
        if (key_matches(e.first, lens, T, k, mflags, idx_bytes)) {
            tc = e.second;
            found = true;
            break;
        }
    if (!found) {
        tune_env_load();
        const TuneEntry q = tune_entry(lens, T, k, mflags, idx_bytes);
        std::lock_guard<std::mutex> lock(g_tune_mu);
        for (const TuneEntry& e : g_tune)
            if (same_shape(e, q)) {
                tc = e.cfg;
                break;
            }
    }
    return with_env(tc);
}

PlanKey plan_key(const radik_ws* ws, const int64_t* lens, int64_t T, int64_t k, uint32_t flags, int idx_bytes,
                 const TuneConfig* force = nullptr) {
    PlanKey key;
    key.lens.assign(lens, lens + T);
    key.k = k;
    key.flags = flags & kPlanFlags;
    key.idx_bytes = idx_bytes;
    key.tune = force ? with_env(*force) : shape_config(ws, lens, T, k, key.flags, idx_bytes);
    return key;
}

// With `upload` set, descriptors are uploaded with copies ordered on that
// stream from pinned staging memory (the request server: no host wait, no
// legacy-stream synchronisation); otherwise synchronously.
int build_plan(radik_ws* ws, const int64_t* lens, int64_t T, int64_t k, uint32_t flags, int idx_bytes,
               cudaStream_t upload = nullptr, bool use_upload = false) {
    Plan& pl = ws->plan;
    {
        // The plan of the last call usually fits: check it without building a key.
        const uint32_t mflags = flags & kPlanFlags;
        if (pl.valid && key_matches(pl.key, lens, T, k, mflags, idx_bytes) &&
            pl.key.tune == shape_config(ws, lens, T, k, mflags, idx_bytes))
            return RADIK_OK;
    }
    PlanKey key = plan_key(ws, lens, T, k, flags, idx_bytes);

    Plan np;
    np.key = key;
    int rc = plan_shape(lens, T, k, flags, np, key.tune);
    if (rc) return rc;
    const bool scale = (flags & RADIK_WITHSCALE) != 0;
    const size_t kk = static_cast<size_t>(k);

    // Device buffers.
    const StateLayout L(T);
    const size_t desc_bytes = plan_desc_bytes(np);
    const double g = ws->grow;
    cudaError_t e = ws->state.ensure(L.bytes, g);
    if (e == cudaSuccess) e = ws->desc.ensure(desc_bytes, g);
    if (e == cudaSuccess && np.fused) {
        e = ws->cand.ensure(sizeof(uint64_t) * static_cast<size_t>(np.cand_entries), g);
        if (e == cudaSuccess) e = ws->samples.ensure(sizeof(uint64_t) * static_cast<size_t>(np.sample_entries), g);
        const size_t sort_blocks = std::max<size_t>(
            {static_cast<size_t>(np.grid), static_cast<size_t>(np.retry_grid), np.merge_tasks.size()});
        if (e == cudaSuccess && kk > kBitonicMax)
            e = ws->scratch.ensure(sizeof(uint64_t) * sort_blocks * kk, g);
    }
    if (e == cudaSuccess && !np.fused) {
        e = ws->hist.ensure(sizeof(uint32_t) * 4096 * static_cast<size_t>(T));
        if (e == cudaSuccess) e = ws->pstate.ensure(sizeof(PlainState) * static_cast<size_t>(T));
        if (e == cudaSuccess) e = ws->stage.ensure(sizeof(uint64_t) * static_cast<size_t>(T) * kk);
        if (e == cudaSuccess) e = ws->pcand[0].ensure(sizeof(uint64_t) * static_cast<size_t>(np.N));
        if (e == cudaSuccess) e = ws->pcand[1].ensure(sizeof(uint64_t) * static_cast<size_t>(np.N));
        if (e == cudaSuccess && kk > kBitonicMax)
            e = ws->scratch.ensure(sizeof(uint64_t) * static_cast<size_t>(T) * kk);
    }
    if (e != cudaSuccess) {
        pl.valid = false;
        return fail(e == cudaErrorMemoryAllocation ? RADIK_ERR_OOM : RADIK_ERR_CUDA,
                    std::string("workspace allocation: ") + cudaGetErrorString(e));
    }
    if (use_upload) {
        // Stage the whole descriptor block in pinned memory, one async copy.
        if (ws->h_stage_bytes < desc_bytes) {
            if (ws->h_stage) cudaFreeHost(ws->h_stage);
            ws->h_stage = nullptr;
            ws->h_stage_bytes = 0;
            const size_t nb = ws->grow > 1.0 ? static_cast<size_t>(static_cast<double>(desc_bytes) * ws->grow)
                                             : desc_bytes;
            e = counted_malloc_host(&ws->h_stage, nb);
            if (e == cudaSuccess) ws->h_stage_bytes = nb;
        }
        if (e == cudaSuccess) {
            if (T) std::memcpy(ws->h_stage + np.tasks_off, np.tasks.data(), sizeof(FusedTask) * T);
            if (!np.segs.empty())
                std::memcpy(ws->h_stage + np.segs_off, np.segs.data(), sizeof(FusedSeg) * np.segs.size());
            if (!np.jobs.empty())
                std::memcpy(ws->h_stage + np.jobs_off, np.jobs.data(), sizeof(SampleJob) * np.jobs.size());
            if (!np.merge_tasks.empty())
                std::memcpy(ws->h_stage + np.merge_off, np.merge_tasks.data(),
                            sizeof(int32_t) * np.merge_tasks.size());
            e = cudaMemcpyAsync(ws->desc.p, ws->h_stage, desc_bytes, cudaMemcpyHostToDevice, upload);
        }
        if (e == cudaSuccess) e = cudaMemsetAsync(ws->state.p, 0, L.bytes, upload);
    } else {
        e = cudaMemcpy(ws->desc.as<char>(np.tasks_off), np.tasks.data(), sizeof(FusedTask) * T, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !np.segs.empty())
            e = cudaMemcpy(ws->desc.as<char>(np.segs_off), np.segs.data(), sizeof(FusedSeg) * np.segs.size(),
                           cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !np.jobs.empty())
            e = cudaMemcpy(ws->desc.as<char>(np.jobs_off), np.jobs.data(), sizeof(SampleJob) * np.jobs.size(),
                           cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !np.merge_tasks.empty())
            e = cudaMemcpy(ws->desc.as<char>(np.merge_off), np.merge_tasks.data(),
                           sizeof(int32_t) * np.merge_tasks.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(ws->state.p, 0, L.bytes);
    }
    if (e == cudaSuccess && np.fused && !np.jobs.empty()) {
        SampleKernel sk = pick_sample(scale);
        const size_t ssmem = sizeof(uint64_t) * std::max<size_t>(8 * kSampleChunk, 128 * 64);
        e = cudaFuncSetAttribute(reinterpret_cast<const void*>(sk), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(ssmem));
    }
    if (e != cudaSuccess) {
        pl.valid = false;
        return fail(RADIK_ERR_CUDA, std::string("plan upload: ") + cudaGetErrorString(e));
    }
    pl = std::move(np);
    return RADIK_OK;
}

FusedParams fused_params(radik_ws* ws, float* vout, void* iout, int idx_bytes, const float* vin, const void* iin,
                         int64_t k, uint32_t flags) {
    const Plan& pl = ws->plan;
    const StateLayout L(pl.T);
    FusedParams p;
    std::memset(&p, 0, sizeof(p));
    p.data = vin;
    p.tasks = ws->desc.as<FusedTask>(pl.tasks_off);
    p.segs = ws->desc.as<FusedSeg>(pl.segs_off);
    p.task_io = nullptr;
    p.nsegs = pl.nsegs;
    p.kmax = static_cast<uint32_t>(k);
    p.cap = pl.cap;
    p.retry = 0;
    p.idx_in = (flags & RADIK_WITHIDXIN) ? iin : nullptr;
    p.idx_bytes = idx_bytes;
    p.val_out = vout;
    p.idx_out = iout;
    p.err = err_ptr(ws);
    p.work_counter = ws->state.as<uint32_t>(StateLayout::kWork);
    p.gthr = ws->state.as<uint64_t>(L.gthr);
    p.task_done = ws->state.as<uint32_t>(L.done);
    p.task_cnt = ws->state.as<uint32_t>(L.cnt);
    p.fail = ws->state.as<uint32_t>(L.fail);
    p.fail_any = ws->state.as<uint32_t>(StateLayout::kAny);
    p.sample_max = static_cast<uint32_t>(pl.ws_sample_max);
    p.cand = ws->cand.as<uint64_t>();
    p.sort_scratch = ws->scratch.as<uint64_t>();
    p.rank_ready = ws->state.as<uint32_t>(L.rk);
    p.ndefer = static_cast<uint32_t>(pl.defer_tasks.size());
    p.defer_ctr = ws->state.as<uint32_t>(L.dctr);
    p.defer_q = pl.defer_tasks.empty() ? nullptr : ws->state.as<uint32_t>(L.dq);
    return p;
}

// The rank kernel places every output key by counting the keys below it:
// k^2 compares per task, spread over the GPU.  That pays off for a few tasks
// (one large task's merge runs on one SM otherwise); for many flush-mode
// tasks their merge blocks already fill the GPU and sort their rows
// themselves.
bool rank_pays(size_t ntasks, uint64_t k) {
    return k <= kRankMaxK && static_cast<uint64_t>(ntasks) * k * k <= (uint64_t(1) << 26);
}

// Clears the per-call state (n 32-bit words): a kernel rather than a memset,
// so that the call's first kernel can be launched programmatically after it.
__global__ void state_clear_kernel(uint32_t* p, uint32_t n) {
    grid_dep_wait();  // the stream's previous kernel (a previous call's) may still read the state
    grid_dep_launch();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = 0u;
}

// Launch of a kernel that follows another kernel on the stream: with
// programmatic stream serialization the launch overlaps the end of the
// previous kernel (the kernel waits in grid_dep_wait before reading its
// results).  `after_kernel` false: an ordinary launch.
template <typename... KArgs, typename... AArgs>
cudaError_t launch_after(bool after_kernel, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                         cudaStream_t s, AArgs&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = after_kernel ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<AArgs>(args)...);
}

int run_fused(radik_ws* ws, const FusedParams& p, uint32_t flags, cudaStream_t s) {
    const Plan& pl = ws->plan;
    const StateLayout L(pl.T);
    const bool scale = (flags & RADIK_WITHSCALE) != 0;
    // Reset the per-call state (the error word stays sticky until read).
    {
        const uint32_t nw = static_cast<uint32_t>((L.bytes - StateLayout::kWork) / 4);
        const unsigned cg = std::max(1u, std::min(148u * 4u, (nw + 255u) / 256u));
        RADIK_CUDA(launch_after(true, state_clear_kernel, dim3(cg), dim3(256), 0, s,
                                ws->state.as<uint32_t>(StateLayout::kWork), nw));
    }
    if (!pl.jobs.empty()) {
        if (pl.sample_one) {
            RADIK_CUDA(launch_after(true, scale ? sample_one_kernel<true> : sample_one_kernel<false>,
                                    dim3(static_cast<unsigned>(pl.jobs.size())), dim3(kSampleOneThreads), 0, s, p,
                                    static_cast<const SampleJob*>(ws->desc.as<SampleJob>(pl.jobs_off))));
        } else {
            SampleKernel sk = pick_sample(scale);
            const size_t ssmem = sizeof(uint64_t) * std::max<size_t>(8 * kSampleChunk, 128 * 64);
            RADIK_CUDA(launch_after(true, sk, dim3(static_cast<unsigned>(pl.jobs.size())), dim3(256), ssmem, s, p,
                                    static_cast<const SampleJob*>(ws->desc.as<SampleJob>(pl.jobs_off)),
                                    ws->samples.as<uint64_t>(), ws->state.as<uint32_t>(L.sdone)));
        }
    }
    FusedKernel fk = pl.ws_form ? pick_fused_ws(pl.threads, pl.vec, pl.ws_stages, scale)
                                : pick_fused(pl.threads, pl.vec, scale);
    RADIK_CUDA(launch_after(true, fk, dim3(pl.grid), dim3(pl.launch_threads), pl.smem, s, p));
    if (!pl.merge_tasks.empty()) {
        // Flush-mode tasks: exact selection from their candidate regions.
        FusedParams m = p;
        m.cap = pl.merge_cap;
        const bool use_rank = rank_pays(pl.merge_tasks.size(), p.kmax);
        if (!use_rank) m.rank_ready = nullptr;  // each merge block sorts and writes its row
        RADIK_CUDA(launch_after(true, pick_merge(scale), dim3(static_cast<unsigned>(pl.merge_tasks.size())),
                                dim3(kMergeThreads), pl.merge_smem, s, m,
                                static_cast<const int32_t*>(ws->desc.as<int32_t>(pl.merge_off))));
        // ... and the output rows of those it left to the rank kernel.
        if (use_rank) {
            const dim3 rgrid(static_cast<unsigned>((p.kmax + kRankPerBlock - 1) / kRankPerBlock),
                             static_cast<unsigned>(pl.merge_tasks.size()));
            const size_t rsmem = sizeof(uint64_t) * (std::min<size_t>(p.kmax, kRankMaxK) + 2);
            RADIK_CUDA(launch_after(true, pick_rank(scale), rgrid, dim3(kRankThreads), rsmem, s, m,
                                    static_cast<const int32_t*>(ws->desc.as<int32_t>(pl.merge_off))));
        }
    }
    if (!pl.jobs.empty()) {
        // Recompute, without the sampled threshold and with the full candidate
        // buffer, any task whose seeded threshold left fewer than k candidates
        // (or overflowed its region); exits at once otherwise.
        FusedParams r = p;
        r.retry = 1;
        r.cap = pl.retry_cap;
        r.work_counter = ws->state.as<uint32_t>(StateLayout::kWorkRetry);
        r.gthr = ws->state.as<uint64_t>(L.gthr_r);
        r.task_done = ws->state.as<uint32_t>(L.done_r);
        r.task_cnt = ws->state.as<uint32_t>(L.cnt_r);
        FusedKernel rk = pick_fused(pl.retry_threads, pl.retry_vec, scale);
        RADIK_CUDA(launch_after(true, rk, dim3(pl.retry_grid), dim3(pl.retry_threads), pl.retry_smem, s, r));
    }
    return RADIK_OK;
}

int run_plain(radik_ws* ws, const FusedParams& fp, uint32_t flags, cudaStream_t s) {
    const Plan& pl = ws->plan;
    const int64_t T = pl.T;
    const uint32_t k = fp.kmax;
    const bool scale = (flags & RADIK_WITHSCALE) != 0;
    PlainParams p;
    std::memset(&p, 0, sizeof(p));
    p.data = fp.data;
    p.tasks = fp.tasks;
    p.segs = fp.segs;
    p.nsegs = pl.nsegs;
    p.ntasks = static_cast<int32_t>(T);
    p.k = k;
    p.sp = make_score_params((flags & RADIK_LARGEST) != 0, scale);
    p.hist = ws->hist.as<uint32_t>();
    p.st = ws->pstate.as<PlainState>();
    p.out_stage = ws->stage.as<uint64_t>();
    p.cand[0] = ws->pcand[0].as<uint64_t>();
    p.cand[1] = ws->pcand[1].as<uint64_t>();
    p.err = fp.err;
    uint32_t* any = ws->state.as<uint32_t>(StateLayout::kAny);
    const DeviceInfo di = device_info();
    const int grid_in = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(pl.nsegs, 8LL * di.sms)));

    RADIK_CUDA(cudaMemsetAsync(p.hist, 0, sizeof(uint32_t) * 4096 * T, s));
    RADIK_CUDA(cudaMemsetAsync(p.st, 0, sizeof(PlainState) * T, s));
    if (scale) plain_hist_input<256, true><<<grid_in, 256, 0, s>>>(p);
    else plain_hist_input<256, false><<<grid_in, 256, 0, s>>>(p);
    plain_select<256><<<static_cast<unsigned>(T), 256, 0, s>>>(p, 0, 12);
    if (scale) plain_compact_input<256, true><<<grid_in, 256, 0, s>>>(p);
    else plain_compact_input<256, false><<<grid_in, 256, 0, s>>>(p);
    RADIK_CUDA(cudaMemsetAsync(any, 0, 4, s));
    plain_advance<<<static_cast<unsigned>((T + 255) / 256), 256, 0, s>>>(p, any);
    RADIK_CUDA(cudaGetLastError());

    // Candidate passes over the remaining composite bits; the host reads the
    // "any task active" flag after each pass (src/algorithm.jl:242-244,
    // :275-277 read back candidate counts the same way).
    const PlainSchedule& sched = kPlainSchedule[pl.key.tune.plain_sched];
    int src = 0;
    for (int ps = 0; ps < sched.n; ++ps) {
        const int sh = sched.pass[ps].sh, wd = sched.pass[ps].w;
        uint32_t h_any = 0;
        RADIK_CUDA(cudaMemcpyAsync(&h_any, any, 4, cudaMemcpyDeviceToHost, s));
        RADIK_CUDA(cudaStreamSynchronize(s));
        if (!h_any) break;
        int64_t maxlen = 0;
        for (int64_t t = 0; t < T; ++t) maxlen = std::max(maxlen, pl.tasks[t].len);
        const unsigned gx = static_cast<unsigned>(std::max<int64_t>(
            1, std::min<int64_t>((maxlen + 255) / 256, std::max<int64_t>(1, 4LL * di.sms / std::max<int64_t>(T, 1)))));
        for (int64_t t0 = 0; t0 < T; t0 += 65535) {
            unsigned gy = static_cast<unsigned>(std::min<int64_t>(65535, T - t0));
            plain_hist_cand<256><<<dim3(gx, gy), 256, 0, s>>>(p, static_cast<int>(t0), src, sh, wd);
        }
        plain_select<256><<<static_cast<unsigned>(T), 256, 0, s>>>(p, ps + 1, wd);
        for (int64_t t0 = 0; t0 < T; t0 += 65535) {
            unsigned gy = static_cast<unsigned>(std::min<int64_t>(65535, T - t0));
            plain_compact_cand<256><<<dim3(gx, gy), 256, 0, s>>>(p, static_cast<int>(t0), src, sh, wd);
        }
        RADIK_CUDA(cudaMemsetAsync(any, 0, 4, s));
        plain_advance<<<static_cast<unsigned>((T + 255) / 256), 256, 0, s>>>(p, any);
        RADIK_CUDA(cudaGetLastError());
        src ^= 1;
    }
    const size_t fsmem = std::max<size_t>(sizeof(uint64_t) * kBitonicMax, sizeof(uint32_t) * (8 * 256 + 256));
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(reinterpret_cast<const void*>(plain_finalize<256>),
                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(fsmem));
        attr_set = true;
    }
    if (T > 0) plain_finalize<256><<<static_cast<unsigned>(T), 256, fsmem, s>>>(p, fp, ws->scratch.as<uint64_t>());
    RADIK_CUDA(cudaGetLastError());
    return RADIK_OK;
}

int finish_sync(radik_ws* ws, cudaStream_t s) {
    RADIK_CUDA(cudaMemcpyAsync(ws->h_err, err_ptr(ws), 4, cudaMemcpyDeviceToHost, s));
    RADIK_CUDA(cudaStreamSynchronize(s));
    if (*ws->h_err) {
        uint32_t bits = *ws->h_err;
        cudaMemsetAsync(err_ptr(ws), 0, 4, s);
        cudaStreamSynchronize(s);
        char buf[128];
        std::snprintf(buf, sizeof(buf), "device error word 0x%x (capacity=1 bounds=2 timeout=4 internal=8)", bits);
        return fail((bits & kErrTimeout) ? RADIK_ERR_TIMEOUT : RADIK_ERR_DEVICE, buf);
    }
    return RADIK_OK;
}

// A workspace's buffers live on the device it was created on; the kernels
// run on the current device.
int check_ws_device(const radik_ws* ws) {
    int dev = 0;
    RADIK_CUDA(cudaGetDevice(&dev));
    if (dev != ws->device) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "the workspace belongs to cuda:%d but the current device is cuda:%d",
                      ws->device, dev);
        return fail(RADIK_ERR_INVALID, buf);
    }
    return RADIK_OK;
}

int validate_lens(const int64_t* lens, int64_t T, int64_t* maxlen) {
    *maxlen = 0;
    for (int64_t t = 0; t < T; ++t) {
        if (lens[t] < 0) return fail(RADIK_ERR_INVALID, "task_lens must be non-negative");
        if (lens[t] > INT32_MAX) return fail(RADIK_ERR_INVALID, "a task may hold at most 2^31-1 elements");
        *maxlen = std::max(*maxlen, lens[t]);
    }
    return RADIK_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Exported API
// ---------------------------------------------------------------------------
extern "C" {

const char* radik_version(void) { return "radik-b200 0.1.0 (sm_100a)"; }

const char* radik_last_error(void) { return g_last_error.c_str(); }

int radik_alloc_count(uint64_t* count) {
    if (!count) return fail(RADIK_ERR_INVALID, "NULL argument");
    *count = g_alloc_count.load(std::memory_order_relaxed);
    return RADIK_OK;
}

const char* radik_status_string(int st) {
    switch (st) {
        case RADIK_OK: return "ok";
        case RADIK_ERR_INVALID: return "invalid argument";
        case RADIK_ERR_OOM: return "out of memory";
        case RADIK_ERR_WS_TOO_SMALL: return "workspace too small";
        case RADIK_ERR_CUDA: return "CUDA error";
        case RADIK_ERR_DEVICE: return "device-side error";
        case RADIK_ERR_TIMEOUT: return "device wait timed out";
        case RADIK_ERR_CAPTURE: return "not allowed during stream capture";
        default: return "unknown status";
    }
}

int radik_ws_create(int64_t n, int64_t num_tasks, int index_bytes, radik_ws** out) {
    if (!out) return fail(RADIK_ERR_INVALID, "ws pointer is NULL");
    *out = nullptr;
    if (n < 0 || num_tasks < 0) return fail(RADIK_ERR_INVALID, "workspace sizes must be non-negative");
    if (index_bytes != 4 && index_bytes != 8) return fail(RADIK_ERR_INVALID, "workspace integer type must be 4 or 8 bytes");
    radik_ws* ws = new (std::nothrow) radik_ws();
    if (!ws) return fail(RADIK_ERR_OOM, "host allocation of the workspace failed");
    cudaGetDevice(&ws->device);
    ws->n = n;
    ws->num_tasks = num_tasks;
    ws->index_bytes = index_bytes;
    if (counted_malloc_host(&ws->h_err, sizeof(uint32_t)) != cudaSuccess) {
        delete ws;
        return fail(RADIK_ERR_OOM, "pinned allocation failed");
    }
    *ws->h_err = 0;
    const size_t sb = StateLayout(num_tasks).bytes;
    if (ws->state.ensure(sb) != cudaSuccess || cudaMemset(ws->state.p, 0, sb) != cudaSuccess) {
        cudaFreeHost(ws->h_err);
        delete ws;
        return fail(RADIK_ERR_OOM, "device allocation of the workspace failed");
    }
    *out = ws;
    return RADIK_OK;
}

int radik_ws_destroy(radik_ws* ws) {
    if (!ws) return RADIK_OK;
    for (DevBuf* b : {&ws->state, &ws->desc, &ws->cand, &ws->samples, &ws->scratch, &ws->hist, &ws->pstate,
                      &ws->stage, &ws->pcand[0], &ws->pcand[1], &ws->io_in, &ws->io_idx, &ws->io_vout, &ws->io_iout})
        b->release();
    if (ws->h_err) cudaFreeHost(ws->h_err);
    if (ws->h_stage) cudaFreeHost(ws->h_stage);
    delete ws;
    return RADIK_OK;
}

int radik_ws_bytes(const radik_ws* ws, size_t* bytes) {
    if (!ws || !bytes) return fail(RADIK_ERR_INVALID, "NULL argument");
    size_t b = 0;
    for (const DevBuf* d : {&ws->state, &ws->desc, &ws->cand, &ws->samples, &ws->scratch, &ws->hist, &ws->pstate,
                            &ws->stage, &ws->pcand[0], &ws->pcand[1], &ws->io_in, &ws->io_idx, &ws->io_vout,
                            &ws->io_iout})
        b += d->bytes;
    *bytes = b;
    return RADIK_OK;
}

int radik_ws_error(radik_ws* ws, uint32_t* bits) {
    if (!ws || !bits) return fail(RADIK_ERR_INVALID, "NULL argument");
    RADIK_CUDA(cudaMemcpyAsync(ws->h_err, err_ptr(ws), 4, cudaMemcpyDeviceToHost, ws->last_stream));
    RADIK_CUDA(cudaStreamSynchronize(ws->last_stream));
    *bits = *ws->h_err;
    RADIK_CUDA(cudaMemsetAsync(err_ptr(ws), 0, 4, ws->last_stream));
    RADIK_CUDA(cudaStreamSynchronize(ws->last_stream));
    return RADIK_OK;
}

int radik_tune_save(const char* path) {
    if (!path) return fail(RADIK_ERR_INVALID, "NULL path");
    tune_env_load();
    std::lock_guard<std::mutex> lock(g_tune_mu);
    if (tune_write(path) < 0) return fail(RADIK_ERR_INVALID, "cannot write the tuning file");
    return RADIK_OK;
}

int radik_tune_load(const char* path, int64_t* entries) {
    if (!path) return fail(RADIK_ERR_INVALID, "NULL path");
    tune_env_load();
    std::lock_guard<std::mutex> lock(g_tune_mu);
    const int n = tune_read(path);
    if (n < 0) return fail(RADIK_ERR_INVALID, "cannot read the tuning file");
    if (entries) *entries = n;
    return RADIK_OK;
}

int radik_tune_clear(void) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune.clear();
    return RADIK_OK;
}

int radik_ws_plan_info(const radik_ws* ws, radik_plan_info* info) {
    if (!ws || !info) return fail(RADIK_ERR_INVALID, "NULL argument");
    const Plan& pl = ws->plan;
    if (!pl.valid) return fail(RADIK_ERR_INVALID, "the workspace has no plan yet");
    info->path = !pl.fused ? 2 : (pl.ws_form ? 1 : 0);
    info->block_threads = pl.fused ? pl.launch_threads : 256;
    info->grid = pl.grid;
    info->smem_bytes = static_cast<int>(pl.smem);
    info->candidate_capacity = static_cast<int>(pl.cap);
    info->segments = pl.nsegs;
    info->sample_jobs = static_cast<int>(pl.jobs.size());
    // fused: sampling kernel + fused kernel (+ merge kernel for flush-mode
    // tasks) + retry launch when sampled;
    // multi-pass: histogram, select, compact, advance, finalize at least.
    // state clear + streaming kernel (+ sampler and retry) (+ merge and rank)
    info->kernels_per_call =
        pl.fused ? 2 + (pl.jobs.empty() ? 0 : 2) +
                       (pl.merge_tasks.empty() ? 0 : (rank_pays(pl.merge_tasks.size(), pl.key.k) ? 2 : 1))
                 : 5;
    return RADIK_OK;
}

int radik_ws_prepare(radik_ws* ws, const int64_t* h_task_lens, int64_t num_tasks, int64_t k, uint32_t flags,
                     int idx_bytes) {
    if (!ws || (!h_task_lens && num_tasks > 0)) return fail(RADIK_ERR_INVALID, "NULL argument");
    if (k < 0) return fail(RADIK_ERR_INVALID, "k must be non-negative");
    if (idx_bytes != 4 && idx_bytes != 8) return fail(RADIK_ERR_INVALID, "index width must be 4 or 8 bytes");
    int rc = check_ws_device(ws);
    if (rc) return rc;
    int64_t maxlen = 0;
    rc = validate_lens(h_task_lens, num_tasks, &maxlen);
    if (rc) return rc;
    if (maxlen > ws->n || num_tasks > ws->num_tasks)
        return fail(RADIK_ERR_WS_TOO_SMALL, "workspace requires n >= max(task_lens) and num_tasks <= its num_tasks");
    return build_plan(ws, h_task_lens, num_tasks, k, flags, idx_bytes);
}

int radik_topk_radix_select(float* d_val_out, void* d_idx_out, int idx_bytes, radik_ws* ws, const float* d_val_in,
                            const void* d_idx_in, const int64_t* h_task_lens, int64_t num_tasks, int64_t k,
                            uint32_t flags, void* stream) {
    if (!ws) return fail(RADIK_ERR_INVALID, "workspace is NULL");
    if (num_tasks < 0 || k < 0) return fail(RADIK_ERR_INVALID, "num_tasks and k must be non-negative");
    if (idx_bytes != 4 && idx_bytes != 8) return fail(RADIK_ERR_INVALID, "index width must be 4 or 8 bytes");
    if (k > INT32_MAX) return fail(RADIK_ERR_INVALID, "k must fit in 32 bits");
    if ((flags & RADIK_WITHIDXIN) && !d_idx_in) return fail(RADIK_ERR_INVALID, "WITHIDXIN needs idx_in");
    if (num_tasks == 0 || k == 0) return RADIK_OK;
    if (!d_val_out || !d_idx_out || !h_task_lens) return fail(RADIK_ERR_INVALID, "NULL output or task_lens");
    int rc = check_ws_device(ws);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ws->last_stream = s;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cap);
    int64_t maxlen = 0;
    rc = validate_lens(h_task_lens, num_tasks, &maxlen);
    if (rc) return rc;
    if (maxlen > ws->n || num_tasks > ws->num_tasks)
        return fail(RADIK_ERR_WS_TOO_SMALL, "workspace requires n >= max(task_lens) and num_tasks <= its num_tasks");
    if (maxlen > 0 && !d_val_in) return fail(RADIK_ERR_INVALID, "val_in is NULL");
    if ((reinterpret_cast<uintptr_t>(d_val_in) & 3) || (reinterpret_cast<uintptr_t>(d_val_out) & 3) ||
        (reinterpret_cast<uintptr_t>(d_idx_out) & (idx_bytes - 1)) ||
        ((flags & RADIK_WITHIDXIN) && (reinterpret_cast<uintptr_t>(d_idx_in) & (idx_bytes - 1))))
        return fail(RADIK_ERR_INVALID, "device arrays must be aligned to their element size");
    {
        const uint32_t mflags = flags & kPlanFlags;
        const bool have_plan = ws->plan.valid && key_matches(ws->plan.key, h_task_lens, num_tasks, k, mflags, idx_bytes) &&
                               ws->plan.key.tune == shape_config(ws, h_task_lens, num_tasks, k, mflags, idx_bytes);
        if (!have_plan) {
            if (cap != cudaStreamCaptureStatusNone)
                return fail(RADIK_ERR_CAPTURE, "no prepared plan for this shape: call radik_ws_prepare before capture");
            rc = build_plan(ws, h_task_lens, num_tasks, k, flags, idx_bytes);
            if (rc) return rc;
        }
    }
    FusedParams p = fused_params(ws, d_val_out, d_idx_out, idx_bytes, d_val_in, d_idx_in, k, flags);
    if (ws->plan.fused) {
        rc = run_fused(ws, p, flags, s);
    } else {
        if (cap != cudaStreamCaptureStatusNone)
            return fail(RADIK_ERR_CAPTURE, "the multi-pass path synchronises with the host and cannot be captured");
        rc = run_plain(ws, p, flags, s);
    }
    if (rc) return rc;
    if (flags & RADIK_ASYNC) return RADIK_OK;
    return finish_sync(ws, s);
}

int radik_ws_autotune(radik_ws* ws, float* d_val_out, void* d_idx_out, int idx_bytes, const float* d_val_in,
                      const void* d_idx_in, const int64_t* h_task_lens, int64_t num_tasks, int64_t k, uint32_t flags,
                      void* stream, int reps, radik_plan_info* chosen, double* best_ms) {
    if (!ws || !h_task_lens) return fail(RADIK_ERR_INVALID, "NULL argument");
    if (num_tasks <= 0 || k <= 0) return fail(RADIK_ERR_INVALID, "num_tasks and k must be positive");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus capst = cudaStreamCaptureStatusNone;
    RADIK_CUDA(cudaStreamIsCapturing(s, &capst));
    if (capst != cudaStreamCaptureStatusNone) return fail(RADIK_ERR_CAPTURE, "autotuning cannot run during capture");
    reps = std::max(1, std::min(reps, 100));
    // Candidate shapes: the defaults, other rings and block sizes of the
    // warp-specialised form, a larger sample, the barrier form, other
    // segment sizes for split tasks, and both fixed shortest segments (4
    // tiles spread a single task of a few million elements over the whole
    // GPU; 64 tiles keep it in fewer, unsampled segments).
    std::vector<TuneConfig> cands;
    TuneConfig d;
    cands.push_back(d);
    if (flags & RADIK_PLAIN) {
        // The multi-pass path: its digit schedules.
        for (int i = 1; i < kPlainSchedules; ++i) {
            TuneConfig c = d;
            c.plain_sched = i;
            cands.push_back(c);
        }
    } else {
    { TuneConfig c = d; c.form = 1; c.ws_stages = 12; cands.push_back(c); }
    { TuneConfig c = d; c.form = 1; c.ws_threads = 256; c.ws_stages = 16; cands.push_back(c); }
    { TuneConfig c = d; c.form = 1; c.sample_max = 4096; cands.push_back(c); }
    // The narrow form: 2 consumer warps, 7 blocks per SM -- one round for a
    // batch of up to 7 tasks per SM.
    { TuneConfig c = d; c.form = 1; c.ws_threads = 64; c.ws_stages = 4; cands.push_back(c); }
    { TuneConfig c = d; c.form = 0; cands.push_back(c); }
    { TuneConfig c = d; c.form = 0; c.bar_threads = (k > 4096 && k <= 8192) ? 256 : 512; cands.push_back(c); }
    { TuneConfig c = d; c.seg_div = 2; cands.push_back(c); }
    { TuneConfig c = d; c.seg_div = 6; cands.push_back(c); }
    { TuneConfig c = d; c.defer = 0; cands.push_back(c); }
    { TuneConfig c = d; c.defer = 1; cands.push_back(c); }
    { TuneConfig c = d; c.seg_min_tiles = 4; cands.push_back(c); }
    { TuneConfig c = d; c.seg_min_tiles = 64; cands.push_back(c); }
    }
    PlanKey base = plan_key(ws, h_task_lens, num_tasks, k, flags, idx_bytes);
    auto set_choice = [&](const TuneConfig& c) {
        for (auto& e : ws->tuned) {
            PlanKey kk = base;
            kk.tune = e.first.tune;
            if (e.first == kk) { e.second = c; return; }
        }
        ws->tuned.emplace_back(base, c);
    };
    // Timed calls run back to back on rotating copies of the input, as many
    // as keep the bytes read between two reads of one copy above three times
    // the L2 (none for an input that large already): a stream of calls on
    // fresh data, not one buffer left in L2.
    int dev = 0, l2 = 0;
    RADIK_CUDA(cudaGetDevice(&dev));
    RADIK_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
    const int64_t n_in = std::accumulate(h_task_lens, h_task_lens + num_tasks, int64_t(0));
    const size_t in_bytes = sizeof(float) * static_cast<size_t>(std::max<int64_t>(n_in, 1));
    const size_t l2x3 = 3 * static_cast<size_t>(std::max(l2, 1 << 20));
    const int ncopy =
        in_bytes >= l2x3 ? 0 : static_cast<int>(std::min<size_t>(128, (l2x3 + in_bytes - 1) / in_bytes + 1));
    float* copies = nullptr;
    if (ncopy > 0) {
        RADIK_CUDA(counted_malloc(reinterpret_cast<void**>(&copies), in_bytes * ncopy));
        for (int c = 0; c < ncopy; ++c) {
            const cudaError_t e = cudaMemcpyAsync(copies + static_cast<size_t>(c) * (in_bytes / sizeof(float)),
                                                  d_val_in, in_bytes, cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) {
                cudaFree(copies);
                return fail(RADIK_ERR_CUDA, "copy of the autotuning input failed");
            }
        }
    }
    int rot = 0;  // calls so far: every call reads the next copy
    auto next_input = [&]() -> const float* {
        return ncopy > 0 ? copies + static_cast<size_t>(rot++ % ncopy) * (in_bytes / sizeof(float)) : d_val_in;
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        if (copies) cudaFree(copies);
        return fail(RADIK_ERR_CUDA, "cudaEventCreate failed");
    }
    // Two rounds over the candidates (the second after every plan is built
    // and the clocks have settled); a candidate's time is its better round.
    std::vector<double> cand_ms(cands.size(), 1e30);
    int rc = RADIK_OK;
    for (int round = 0; round < 2; ++round) {
        for (size_t ci = 0; ci < cands.size(); ++ci) {
            if (round > 0 && cand_ms[ci] >= 1e30) continue;  // did not run in the first round
            set_choice(cands[ci]);
            const uint32_t af = flags | RADIK_ASYNC;
            rc = radik_topk_radix_select(d_val_out, d_idx_out, idx_bytes, ws, d_val_in, d_idx_in, h_task_lens,
                                         num_tasks, k, af, stream);  // builds the plan, warms up
            if (rc == RADIK_OK) rc = finish_sync(ws, s);
            if (rc != RADIK_OK) continue;  // this shape does not apply here
            cudaEventRecord(e0, s);
            for (int i = 0; i < reps && rc == RADIK_OK; ++i)
                rc = radik_topk_radix_select(d_val_out, d_idx_out, idx_bytes, ws, next_input(), d_idx_in, h_task_lens,
                                             num_tasks, k, af, stream);
            cudaEventRecord(e1, s);
            if (rc == RADIK_OK) rc = finish_sync(ws, s);
            if (rc != RADIK_OK) continue;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            cand_ms[ci] = std::min(cand_ms[ci], static_cast<double>(ms) / reps);
        }
    }
    double best = 1e30;
    TuneConfig best_c = d;
    for (size_t ci = 0; ci < cands.size(); ++ci)
        if (cand_ms[ci] < best) {
            best = cand_ms[ci];
            best_c = cands[ci];
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (copies) {
        cudaStreamSynchronize(s);
        cudaFree(copies);
    }
    if (best >= 1e30) return rc != RADIK_OK ? rc : fail(RADIK_ERR_INVALID, "no configuration ran");
    set_choice(best_c);
    {
        // Remember the choice for every workspace of the process (and the
        // tuning file, when one is named).
        tune_env_load();
        TuneEntry e = tune_entry(h_task_lens, num_tasks, k, base.flags, idx_bytes);
        e.cfg = best_c;
        std::lock_guard<std::mutex> lock(g_tune_mu);
        tune_put(e);
        const char* path = std::getenv("RADIK_TUNE_FILE");
        if (path && *path) tune_write(path);
    }
    rc = build_plan(ws, h_task_lens, num_tasks, k, flags, idx_bytes);
    if (rc) return rc;
    if (chosen) radik_ws_plan_info(ws, chosen);
    if (best_ms) *best_ms = best;
    return RADIK_OK;
}

int radik_topk(float* d_val_out, void* d_idx_out, int idx_bytes, const float* d_data, int64_t data_len,
               const void* d_indices, int64_t indices_len, const int64_t* h_task_lens, int64_t num_tasks, int64_t k,
               int largest, int rev, void* stream) {
    if (num_tasks < 0 || k < 0) return fail(RADIK_ERR_INVALID, "num_tasks and k must be non-negative");
    int64_t maxlen = 0, total = 0;
    int rc = validate_lens(h_task_lens, num_tasks, &maxlen);
    if (rc) return rc;
    for (int64_t t = 0; t < num_tasks; ++t) total += h_task_lens[t];
    if (total > data_len) return fail(RADIK_ERR_INVALID, "sum(task_lens) exceeds the data length");
    // src/algorithm.jl:506-510
    if (d_indices && indices_len > 0 && indices_len != data_len) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "indices length must equal data length. Got %lld vs %lld",
                      static_cast<long long>(indices_len), static_cast<long long>(data_len));
        return fail(RADIK_ERR_INVALID, buf);
    }
    radik_ws* ws = nullptr;
    rc = radik_ws_create(maxlen, num_tasks, 4, &ws);  // fresh workspace per call (:503)
    if (rc) return rc;
    uint32_t flags = (largest ? RADIK_LARGEST : 0u) | (rev ? 0u : RADIK_ASCEND) | RADIK_WITHPACKING;
    if (d_indices && indices_len > 0) flags |= RADIK_WITHIDXIN;
    rc = radik_topk_radix_select(d_val_out, d_idx_out, idx_bytes, ws, d_data, d_indices, h_task_lens, num_tasks, k,
                                 flags, stream);
    std::string keep = g_last_error;
    radik_ws_destroy(ws);
    g_last_error = keep;
    return rc;
}

int radik_topk_host(float* h_val_out, void* h_idx_out, int idx_bytes, const float* h_data, int64_t data_len,
                    const void* h_indices, int64_t indices_len, const int64_t* h_task_lens, int64_t num_tasks,
                    int64_t k, int largest, int rev, radik_ws* ws, void* stream) {
    if (!ws) return fail(RADIK_ERR_INVALID, "workspace is NULL");
    if (idx_bytes != 4 && idx_bytes != 8) return fail(RADIK_ERR_INVALID, "index width must be 4 or 8 bytes");
    if (h_indices && indices_len > 0 && indices_len != data_len) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "indices length must equal data length. Got %lld vs %lld",
                      static_cast<long long>(indices_len), static_cast<long long>(data_len));
        return fail(RADIK_ERR_INVALID, buf);
    }
    int rc = check_ws_device(ws);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool with_idx = h_indices && indices_len > 0;
    const size_t out_n = static_cast<size_t>(num_tasks) * static_cast<size_t>(k);
    cudaError_t e = ws->io_in.ensure(sizeof(float) * static_cast<size_t>(data_len));
    if (e == cudaSuccess && with_idx) e = ws->io_idx.ensure(static_cast<size_t>(idx_bytes) * data_len);
    if (e == cudaSuccess) e = ws->io_vout.ensure(sizeof(float) * out_n);
    if (e == cudaSuccess) e = ws->io_iout.ensure(static_cast<size_t>(idx_bytes) * out_n);
    if (e != cudaSuccess) return fail(RADIK_ERR_OOM, std::string("io buffers: ") + cudaGetErrorString(e));
    RADIK_CUDA(cudaMemcpyAsync(ws->io_in.p, h_data, sizeof(float) * data_len, cudaMemcpyHostToDevice, s));
    if (with_idx)
        RADIK_CUDA(cudaMemcpyAsync(ws->io_idx.p, h_indices, static_cast<size_t>(idx_bytes) * data_len,
                                   cudaMemcpyHostToDevice, s));
    uint32_t flags = (largest ? RADIK_LARGEST : 0u) | (rev ? 0u : RADIK_ASCEND) | RADIK_ASYNC;
    if (with_idx) flags |= RADIK_WITHIDXIN;
    rc = radik_topk_radix_select(ws->io_vout.as<float>(), ws->io_iout.p, idx_bytes, ws, ws->io_in.as<float>(),
                                     with_idx ? ws->io_idx.p : nullptr, h_task_lens, num_tasks, k, flags, stream);
    if (rc) return rc;
    if (out_n) {
        RADIK_CUDA(cudaMemcpyAsync(h_val_out, ws->io_vout.p, sizeof(float) * out_n, cudaMemcpyDeviceToHost, s));
        RADIK_CUDA(cudaMemcpyAsync(h_idx_out, ws->io_iout.p, static_cast<size_t>(idx_bytes) * out_n,
                                   cudaMemcpyDeviceToHost, s));
    }
    return finish_sync(ws, s);
}

}  // extern "C"

// ---- allocation-free entry point --------------------------------------------
//
// radik_topk_noalloc runs the fused kernel with its scratch (per-call state,
// plan descriptors, candidate regions of multi-segment tasks, sampled
// thresholds) in one statically sized device array instead of a workspace.
// It exists for callers that must not allocate device memory at the point
// of the call: code running inside a memory pool's out-of-memory handler or
// an allocator callback, processes with a hard device-memory cap, and
// latency-critical loops that cannot afford cudaMalloc's implicit device
// synchronisation.

namespace {
constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;  // 8 MiB per device
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

// Set-up of an allocation-free call on the current device: the device
// address of the static scratch (in host code the array's name is only a
// host-side stand-in, never a device address) and the sampling kernels'
// shared-memory attribute.  Redone on every call -- neither allocates -- so
// that a context reset between calls cannot leave a stale address behind.
int noalloc_setup(char** base) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return fail(RADIK_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    const size_t ssmem = sizeof(uint64_t) * std::max<size_t>(8 * kSampleChunk, 128 * 64);
    for (bool scale : {false, true}) {
        e = cudaFuncSetAttribute(reinterpret_cast<const void*>(pick_sample(scale)),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(ssmem));
        if (e != cudaSuccess) return fail(RADIK_ERR_CUDA, std::string("sampling kernel: ") + cudaGetErrorString(e));
    }
    *base = static_cast<char*>(p);
    return RADIK_OK;
}

}  // namespace

extern "C" {

int radik_topk_noalloc(float* d_val_out, void* d_idx_out, int idx_bytes, const float* d_val_in, const void* d_idx_in,
                       const int64_t* h_task_lens, int64_t num_tasks, int64_t k, uint32_t flags, void* stream) {
    if (num_tasks < 0 || k < 0) return fail(RADIK_ERR_INVALID, "num_tasks and k must be non-negative");
    if (idx_bytes != 4 && idx_bytes != 8) return fail(RADIK_ERR_INVALID, "index width must be 4 or 8 bytes");
    if (flags & (RADIK_PLAIN | RADIK_ASYNC))
        return fail(RADIK_ERR_INVALID, "radik_topk_noalloc runs the fused path synchronously; "
                                       "RADIK_PLAIN and RADIK_ASYNC are not accepted");
    if ((flags & RADIK_WITHIDXIN) && !d_idx_in) return fail(RADIK_ERR_INVALID, "WITHIDXIN needs idx_in");
    if (k > static_cast<int64_t>(kBitonicMax)) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "radik_topk_noalloc supports k <= %u (got k = %lld)", kBitonicMax,
                      static_cast<long long>(k));
        return fail(RADIK_ERR_WS_TOO_SMALL, buf);
    }
    if (num_tasks == 0 || k == 0) return RADIK_OK;
    if (!d_val_out || !d_idx_out || !h_task_lens) return fail(RADIK_ERR_INVALID, "NULL output or task_lens");
    int64_t maxlen = 0;
    int rc = validate_lens(h_task_lens, num_tasks, &maxlen);
    if (rc) return rc;
    if (maxlen > 0 && !d_val_in) return fail(RADIK_ERR_INVALID, "val_in is NULL");
    if ((reinterpret_cast<uintptr_t>(d_val_in) & 3) || (reinterpret_cast<uintptr_t>(d_val_out) & 3) ||
        (reinterpret_cast<uintptr_t>(d_idx_out) & (idx_bytes - 1)) ||
        ((flags & RADIK_WITHIDXIN) && (reinterpret_cast<uintptr_t>(d_idx_in) & (idx_bytes - 1))))
        return fail(RADIK_ERR_INVALID, "device arrays must be aligned to their element size");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    RADIK_CUDA(cudaStreamIsCapturing(s, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        return fail(RADIK_ERR_CAPTURE, "radik_topk_noalloc uploads its plan and waits for the stream; "
                                       "it cannot run while the stream captures");
    int dev = 0;
    RADIK_CUDA(cudaGetDevice(&dev));
    char* base = nullptr;
    rc = noalloc_setup(&base);
    if (rc) return rc;

    // A workspace view whose buffers all point into the static scratch; it
    // owns nothing and is never passed to radik_ws_destroy.
    radik_ws view;
    view.device = dev;
    view.n = maxlen;
    view.num_tasks = num_tasks;
    view.index_bytes = idx_bytes;
    TuneConfig tc = with_env(TuneConfig{});
    tc.defer = 0;  // deferred regions are sized for a workspace, not for the static scratch
    if (tc.seg_min_tiles == 0) tc.seg_min_tiles = 64;  // long segments: fewer candidate regions
    rc = plan_shape(h_task_lens, num_tasks, k, flags, view.plan, tc);
    if (rc) return rc;
    const Plan& pl = view.plan;
    if (!pl.fused) return fail(RADIK_ERR_WS_TOO_SMALL, "the fused kernel's candidate buffer does not fit for this k");
    const StateLayout L(num_tasks);
    const size_t desc_off = round_up(L.bytes, 256);
    const size_t cand_off = round_up(desc_off + plan_desc_bytes(pl), 256);
    const size_t samp_off = round_up(cand_off + sizeof(uint64_t) * static_cast<size_t>(pl.cand_entries), 256);
    const size_t need = samp_off + sizeof(uint64_t) * static_cast<size_t>(pl.sample_entries);
    if (need > kNoAllocScratchBytes) {
        char buf[200];
        std::snprintf(buf, sizeof(buf),
                      "radik_topk_noalloc needs %zu bytes of scratch for this batch; its static scratch holds %zu",
                      need, kNoAllocScratchBytes);
        return fail(RADIK_ERR_WS_TOO_SMALL, buf);
    }
    view.state.p = base;
    view.state.bytes = L.bytes;
    view.desc.p = base + desc_off;
    view.desc.bytes = plan_desc_bytes(pl);
    view.cand.p = base + cand_off;
    view.cand.bytes = sizeof(uint64_t) * static_cast<size_t>(pl.cand_entries);
    view.samples.p = base + samp_off;
    view.samples.bytes = sizeof(uint64_t) * static_cast<size_t>(pl.sample_entries);

    // Everything that must start at zero (error word, work counters, global
    // thresholds, done/candidate counters, retry flags) is cleared here; the
    // descriptors are uploaded from pageable host memory, which the runtime
    // stages before this call returns.
    RADIK_CUDA(cudaMemsetAsync(base, 0, L.bytes, s));
    RADIK_CUDA(cudaMemcpyAsync(view.desc.as<char>(pl.tasks_off), pl.tasks.data(), sizeof(FusedTask) * pl.T,
                               cudaMemcpyHostToDevice, s));
    if (!pl.segs.empty())
        RADIK_CUDA(cudaMemcpyAsync(view.desc.as<char>(pl.segs_off), pl.segs.data(), sizeof(FusedSeg) * pl.segs.size(),
                                   cudaMemcpyHostToDevice, s));
    if (!pl.jobs.empty())
        RADIK_CUDA(cudaMemcpyAsync(view.desc.as<char>(pl.jobs_off), pl.jobs.data(), sizeof(SampleJob) * pl.jobs.size(),
                                   cudaMemcpyHostToDevice, s));
    if (!pl.merge_tasks.empty())
        RADIK_CUDA(cudaMemcpyAsync(view.desc.as<char>(pl.merge_off), pl.merge_tasks.data(),
                                   sizeof(int32_t) * pl.merge_tasks.size(), cudaMemcpyHostToDevice, s));
    FusedParams p = fused_params(&view, d_val_out, d_idx_out, idx_bytes, d_val_in, d_idx_in, k, flags);
    rc = run_fused(&view, p, flags, s);
    if (rc) return rc;
    uint32_t h_err = 0;
    RADIK_CUDA(cudaMemcpyAsync(&h_err, err_ptr(&view), sizeof(h_err), cudaMemcpyDeviceToHost, s));
    RADIK_CUDA(cudaStreamSynchronize(s));
    if (h_err) {
        char buf[128];
        std::snprintf(buf, sizeof(buf), "device error word 0x%x (capacity=1 bounds=2 timeout=4 internal=8)", h_err);
        return fail((h_err & kErrTimeout) ? RADIK_ERR_TIMEOUT : RADIK_ERR_DEVICE, buf);
    }
    return RADIK_OK;
}

// ---- stage entry points ----------------------------------------------------

namespace {
int upload_stage_tasks(const int64_t* lens, int64_t T, DevBuf& buf, cudaStream_t s, int64_t stride = -1) {
    std::vector<StageTask> v(T);
    int64_t off = 0;
    for (int64_t t = 0; t < T; ++t) {
        v[t].start = stride >= 0 ? t * stride : off;
        v[t].len = lens[t];
        off += lens[t];
    }
    if (buf.ensure(sizeof(StageTask) * std::max<int64_t>(T, 1)) != cudaSuccess) return fail(RADIK_ERR_OOM, "stage tasks");
    RADIK_CUDA(cudaMemcpyAsync(buf.p, v.data(), sizeof(StageTask) * T, cudaMemcpyHostToDevice, s));
    RADIK_CUDA(cudaStreamSynchronize(s));
    return RADIK_OK;
}

int check_bits(int left, int right, int* hist_len) {
    if (left < 0 || left > 31 || right < 20 || right > 31)
        return fail(RADIK_ERR_INVALID, "LEFT must be in [0,31] and RIGHT in [20,31] (at most 4096 bins)");
    *hist_len = 1 << (32 - right);
    return RADIK_OK;
}
}  // namespace

int radik_count_bin_ex(int32_t* d_hist, const float* d_data, const int64_t* h_task_lens, int64_t num_tasks, int left,
                       int right, int withscale, int largest, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int hl = 0;
    int rc = check_bits(left, right, &hl);
    if (rc) return rc;
    if (num_tasks <= 0) return RADIK_OK;
    DevBuf tb;
    rc = upload_stage_tasks(h_task_lens, num_tasks, tb, s);
    if (rc) { tb.release(); return rc; }
    RADIK_CUDA(cudaMemsetAsync(d_hist, 0, sizeof(int32_t) * hl * num_tasks, s));
    const DeviceInfo di = device_info();
    dim3 grid(static_cast<unsigned>(std::max(1, 2 * di.sms / static_cast<int>(std::min<int64_t>(num_tasks, 2 * di.sms)))),
              static_cast<unsigned>(std::min<int64_t>(num_tasks, 65535)));
    stage_count_bin_ex<<<grid, 256, sizeof(int32_t) * hl, s>>>(d_hist, d_data, tb.as<StageTask>(), num_tasks, left,
                                                                 right, hl, withscale, largest);
    cudaError_t e = cudaStreamSynchronize(s);
    tb.release();
    if (e != cudaSuccess) return fail(RADIK_ERR_CUDA, cudaGetErrorString(e));
    return RADIK_OK;
}

int radik_count_bin(int32_t* d_hist, const float* d_data, const int64_t* h_task_lens, int64_t stride,
                    int64_t num_tasks, int left, int right, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int hl = 0;
    int rc = check_bits(left, right, &hl);
    if (rc) return rc;
    if (num_tasks <= 0) return RADIK_OK;
    for (int64_t t = 0; t < num_tasks; ++t)
        if (h_task_lens[t] > stride) return fail(RADIK_ERR_INVALID, "task_lens must not exceed stride");
    DevBuf tb;
    rc = upload_stage_tasks(h_task_lens, num_tasks, tb, s, stride);
    if (rc) { tb.release(); return rc; }
    RADIK_CUDA(cudaMemsetAsync(d_hist, 0, sizeof(int32_t) * hl * num_tasks, s));
    dim3 grid(8, static_cast<unsigned>(std::min<int64_t>(num_tasks, 65535)));
    stage_count_bin<<<grid, 256, sizeof(int32_t) * hl, s>>>(d_hist, d_data, tb.as<StageTask>(), stride, num_tasks,
                                                              left, right, hl);
    cudaError_t e = cudaStreamSynchronize(s);
    tb.release();
    if (e != cudaSuccess) return fail(RADIK_ERR_CUDA, cudaGetErrorString(e));
    return RADIK_OK;
}

int radik_select_bin(int32_t* d_bin_ids, int32_t* d_k_values, int32_t* d_counts, const int32_t* d_hist,
                     int64_t num_tasks, int64_t hist_len, int largest, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (hist_len <= 0 || hist_len > (1 << 20)) return fail(RADIK_ERR_INVALID, "hist_len out of range");
    if (num_tasks <= 0) return RADIK_OK;
    stage_select_bin<256><<<static_cast<unsigned>(num_tasks), 256, 0, s>>>(d_bin_ids, d_k_values, d_counts, d_hist,
                                                                           hist_len, largest);
    RADIK_CUDA(cudaGetLastError());
    RADIK_CUDA(cudaStreamSynchronize(s));
    return RADIK_OK;
}

int radik_filter(float* d_val_out, void* d_idx_out, int idx_bytes, int32_t* d_counts, int32_t* d_boundary,
                 const float* d_data, const void* d_idx_in, const float* d_kth, const int64_t* h_task_lens,
                 int64_t num_tasks, int64_t k, int withscale, int largest, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (idx_bytes != 4 && idx_bytes != 8) return fail(RADIK_ERR_INVALID, "index width must be 4 or 8 bytes");
    if (num_tasks <= 0) return RADIK_OK;
    DevBuf tb, eb;
    int rc = upload_stage_tasks(h_task_lens, num_tasks, tb, s);
    if (rc) { tb.release(); return rc; }
    if (eb.ensure(4) != cudaSuccess) { tb.release(); return fail(RADIK_ERR_OOM, "error word"); }
    cudaMemsetAsync(eb.p, 0, 4, s);
    RADIK_CUDA(cudaMemsetAsync(d_counts, 0, sizeof(int32_t) * num_tasks, s));
    dim3 grid(16, static_cast<unsigned>(std::min<int64_t>(num_tasks, 65535)));
    stage_filter<<<grid, 256, 0, s>>>(d_val_out, d_idx_out, idx_bytes, d_counts, d_boundary, d_data, d_idx_in, d_kth,
                                      tb.as<StageTask>(), num_tasks, k, withscale, largest, eb.as<uint32_t>());
    uint32_t h = 0;
    cudaMemcpyAsync(&h, eb.p, 4, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    tb.release();
    eb.release();
    if (e != cudaSuccess) return fail(RADIK_ERR_CUDA, cudaGetErrorString(e));
    if (h) return fail(RADIK_ERR_DEVICE, "filter emitted more than k elements for a task (output bounded)");
    return RADIK_OK;
}

}  // extern "C"

#include "server.inl"
