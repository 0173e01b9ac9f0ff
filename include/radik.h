/*
 * radik.h -- C ABI of the B200 (sm_100a) exact Float32 radix top-k engine.
 *
 * Drop-in boundary for RadiK.jl (WilliBee/RadiK.jl v0.1.3).  Each entry point
 * names the reference interface it replaces (paths relative to the RadiK.jl
 * project root).  All array arguments are raw pointers:
 *   d_*  device memory (CUDA global memory of the current device),
 *   h_*  host memory.
 * Layouts follow the Julia API: the input is the concatenation of all tasks
 * (Float32, task t occupies [off_t, off_t + task_lens[t])), outputs are
 * column-major [k, num_tasks] arrays, i.e. task t's k results are contiguous
 * at t*k.  Indices are 4- or 8-byte signed integers (Int32 / Int64);
 * automatic indices are 1-based positions inside each task, custom indices
 * are copied from indices[global position]; short tasks are padded with value
 * 0 and index -1.  `stream` is a cudaStream_t (NULL = legacy default stream).
 *
 * Every function returns a radik_status; radik_last_error() holds the message
 * of the last failure on the calling thread (the text of the reference's
 * error(...) where one exists).
 */
#ifndef RADIK_B200_H
#define RADIK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum radik_status {
    RADIK_OK = 0,
    RADIK_ERR_INVALID = 1,        /* bad argument (Julia: ErrorException)          */
    RADIK_ERR_OOM = 2,            /* device or host allocation failed              */
    RADIK_ERR_WS_TOO_SMALL = 3,   /* workspace cannot hold the call                */
    RADIK_ERR_CUDA = 4,           /* a CUDA runtime call failed                    */
    RADIK_ERR_DEVICE = 5,         /* a kernel reported an error (see radik_ws_error) */
    RADIK_ERR_TIMEOUT = 6,        /* a bounded device wait gave up                 */
    RADIK_ERR_CAPTURE = 7         /* operation not allowed while the stream captures */
} radik_status;

/* Flags of topk_radix_select! (src/algorithm.jl:170-175: Val(LARGEST),
 * Val(ASCEND), Val(WITHSCALE), Val(WITHIDXIN), Val(WITHPACKING)). */
#define RADIK_LARGEST     0x1u
#define RADIK_ASCEND      0x2u
#define RADIK_WITHSCALE   0x4u
#define RADIK_WITHIDXIN   0x8u
#define RADIK_WITHPACKING 0x10u   /* accepted for parity; loads are always 128-bit */
/* Engine flags (no reference counterpart). */
#define RADIK_ASYNC       0x100u  /* return after enqueueing; no host synchronisation */
#define RADIK_PLAIN       0x200u  /* use the multi-pass per-call path (reference shape) */

typedef struct radik_ws radik_ws;

/* RadiKWorkspace(backend, n, num_tasks, I=Int32), src/algorithm.jl:58-83.
 * n: longest task the workspace serves; num_tasks: largest batch;
 * index_bytes: width of the workspace integer type I (4 or 8).  Device
 * buffers grow on first use with a larger k; prepare before graph capture. */
int radik_ws_create(int64_t n, int64_t num_tasks, int index_bytes, radik_ws** ws);
int radik_ws_destroy(radik_ws* ws);
/* Device bytes currently held by the workspace. */
int radik_ws_bytes(const radik_ws* ws, size_t* bytes);
/* Synchronises the workspace's last stream, returns and clears the device
 * error word (bit 0 capacity, 1 bounds, 2 timeout, 3 internal). */
int radik_ws_error(radik_ws* ws, uint32_t* bits);

/* Builds (and caches in ws) the launch plan for this batch shape: segment
 * table, kernel choice, buffer sizes.  Calls with the same shape reuse it and
 * enqueue only kernels and memsets, so they can be captured in CUDA graphs. */
int radik_ws_prepare(radik_ws* ws, const int64_t* h_task_lens, int64_t num_tasks, int64_t k, uint32_t flags,
                     int idx_bytes);

/* Description of the plan a workspace holds (engine-specific, no reference
 * counterpart): which kernels a call launches and with what shape. */
typedef struct radik_plan_info {
    int path;               /* 0 fused single-read, 1 warp-specialised fused, 2 multi-pass */
    int block_threads;      /* threads per block of the fused kernel */
    int grid;               /* blocks of the fused kernel */
    int smem_bytes;         /* dynamic shared memory per block */
    int candidate_capacity; /* shared candidate buffer, composites */
    int segments;           /* work items (task segments) */
    int sample_jobs;        /* blocks of the sampling kernel (0: not launched) */
    int kernels_per_call;   /* kernels one call launches (multi-pass: lower bound) */
} radik_plan_info;

/* Fills *info from the plan built by the last prepare or call; fails with
 * RADIK_ERR_INVALID when the workspace has no plan yet. */
int radik_ws_plan_info(const radik_ws* ws, radik_plan_info* info);

/* Autotuner (engine-specific, no reference counterpart): runs the call
 * below on the caller's data with each candidate configuration -- of the
 * fused path (kernel form, block and ring shape, sample size, segment size),
 * or with RADIK_PLAIN of the multi-pass path (digit width and pass count of
 * its candidate passes) -- `reps` timed calls each, and keeps the fastest for
 * this batch shape (task_lens, k, flags, index width) in ws and in the
 * process-wide tuning table below; later calls with that shape, in any
 * workspace, use it.  The outputs hold a valid result afterwards.  *chosen
 * (nullable) describes the chosen plan, *best_ms (nullable) its time per
 * call.  Not during stream capture. */
int radik_ws_autotune(radik_ws* ws, float* d_val_out, void* d_idx_out, int idx_bytes, const float* d_val_in,
                      const void* d_idx_in, const int64_t* h_task_lens, int64_t num_tasks, int64_t k,
                      uint32_t flags, void* stream, int reps, radik_plan_info* chosen, double* best_ms);

/* Tuning table (engine-specific, no reference counterpart).  The autotuner's
 * choice for a batch shape (task lengths, k, flags, index width) is kept for
 * every workspace of the process: a workspace that meets a tuned shape uses
 * it without timing again.  radik_tune_save writes the table to a text file,
 * radik_tune_load merges one in (*entries, nullable: lines read),
 * radik_tune_clear empties it.  With RADIK_TUNE_FILE set, that file is loaded
 * at first use and rewritten after each autotuning.  No device work. */
int radik_tune_save(const char* path);
int radik_tune_load(const char* path, int64_t* entries);
int radik_tune_clear(void);

/* topk_radix_select!(val_out, idx_out, ws, val_in, idx_in, task_lens, k,
 *                    Val(LARGEST), Val(ASCEND), Val(WITHSCALE), Val(WITHIDXIN),
 *                    Val(WITHPACKING), Val(VLOAD_SIZE_BYTES))
 * src/algorithm.jl:162-368.  Requires max(task_lens) <= ws n and
 * num_tasks <= ws num_tasks (src/algorithm.jl:156-160).  d_idx_in is read only
 * with RADIK_WITHIDXIN.  Synchronous (like the reference, :353) unless
 * RADIK_ASYNC is set. */
int radik_topk_radix_select(float* d_val_out, void* d_idx_out, int idx_bytes, radik_ws* ws,
                            const float* d_val_in, const void* d_idx_in, const int64_t* h_task_lens,
                            int64_t num_tasks, int64_t k, uint32_t flags, void* stream);

/* topk!(val_out, idx_out, data, task_lens, k; indices, largest, rev),
 * src/algorithm.jl:477-522: validates the index length (:506-510), allocates a
 * fresh workspace for the call (:503), runs with ASCEND = !rev (:520) and
 * returns when the results are complete.  d_indices may be NULL
 * (indices_len 0) for automatic indices. */
int radik_topk(float* d_val_out, void* d_idx_out, int idx_bytes, const float* d_data, int64_t data_len,
               const void* d_indices, int64_t indices_len, const int64_t* h_task_lens, int64_t num_tasks,
               int64_t k, int largest, int rev, void* stream);

/* Same as radik_topk with HOST buffers: copies the input (and indices) to
 * the device, runs, copies the results back.  h_data may be pinned or
 * pageable. */
int radik_topk_host(float* h_val_out, void* h_idx_out, int idx_bytes, const float* h_data, int64_t data_len,
                    const void* h_indices, int64_t indices_len, const int64_t* h_task_lens, int64_t num_tasks,
                    int64_t k, int largest, int rev, radik_ws* ws, void* stream);

/* No counterpart in the reference (RadiK.jl always allocates a workspace).
 * Same arguments and results as radik_topk_radix_select without a workspace:
 * the fused kernel's scratch lives in one static 8 MiB device array per
 * device, so the call performs no device allocation or free.  It serves
 * callers that must not allocate device memory where they call: a memory
 * pool's out-of-memory handler or allocator callback, a process under a hard
 * device-memory cap, or a loop that cannot take cudaMalloc's implicit device
 * synchronisation.
 * Limits: k <= 4096, and the batch's scratch (about 40 bytes per task, 16
 * per segment, k * 8 bytes per segment of a task split across several
 * blocks) must fit in 8 MiB; larger calls fail with RADIK_ERR_WS_TOO_SMALL
 * and a message giving the bytes needed.  RADIK_PLAIN and RADIK_ASYNC are
 * rejected: the call clears the scratch state that must start at zero,
 * uploads the plan, launches, and waits for `stream` before returning.
 * Every call looks up the static array's address on the current device
 * (cudaGetSymbolAddress) and sets the kernel attributes it needs; neither
 * allocates, and a context that was reset and recreated between calls gets
 * the new address.  The first call on a device may load the library's
 * device code there: make it before any stream capture.  A capturing stream
 * is rejected with RADIK_ERR_CAPTURE.
 * All calls on one device share the array: calls that overlap in time (from
 * several host threads, or on streams that are not ordered with each other)
 * race and corrupt each other's results. */
int radik_topk_noalloc(float* d_val_out, void* d_idx_out, int idx_bytes, const float* d_val_in,
                       const void* d_idx_in, const int64_t* h_task_lens, int64_t num_tasks, int64_t k,
                       uint32_t flags, void* stream);

/* ---- Request server (engine-specific, no reference counterpart) ----------
 * Continuous batching of top-k requests: a worker thread packs pending
 * requests that share (k, flags, index width) into one fused launch (every
 * row of every request is a task with its own input and output pointers),
 * runs up to `slots` launches at once on their own streams and device-
 * resident workspaces, and admits a request only while the bytes of the
 * requests in flight (inputs and outputs) plus the workspace pool stay under
 * mem_cap_bytes.  Inputs and outputs are caller-owned device memory and must
 * stay valid until the request completes. */
typedef struct radik_server radik_server;

typedef struct radik_server_config {
    int slots;              /* concurrent launches (streams + workspaces), 1..64 */
    int device;             /* CUDA device ordinal */
    int64_t mem_cap_bytes;  /* admission cap: in-flight request bytes + workspace pool */
    int64_t max_batch_rows; /* most rows packed into one launch */
} radik_server_config;

typedef struct radik_server_stats {
    uint64_t submitted, completed, batches, rows;
    double elements;        /* input elements of the completed requests */
    double p50_us, p99_us, mean_us;  /* submit-to-completion latency of completed requests */
    int64_t mem_in_flight;  /* request bytes in flight now */
    int64_t mem_pool;       /* device bytes held by the slots' workspaces */
} radik_server_stats;

int radik_server_create(const radik_server_config* cfg, radik_server** server);
/* Waits for every submitted request, then releases the server. */
int radik_server_destroy(radik_server* server);
/* Queues a request: d_data [rows][row_len] Float32 (row-major), outputs
 * d_val_out [rows][k] and d_idx_out [rows][k] (idx_bytes wide, 1-based
 * positions inside the row), flags RADIK_LARGEST / RADIK_ASCEND /
 * RADIK_WITHSCALE as for radik_topk_radix_select.  *ticket identifies it. */
int radik_server_submit(radik_server* server, const float* d_data, int64_t rows, int64_t row_len, int64_t k,
                        uint32_t flags, float* d_val_out, void* d_idx_out, int idx_bytes, uint64_t* ticket);
/* Waits up to timeout_us (negative: no limit) for a request; RADIK_OK when
 * it completed (the ticket is then released), RADIK_ERR_TIMEOUT if not yet. */
int radik_server_wait(radik_server* server, uint64_t ticket, int64_t timeout_us);
int radik_server_get_stats(radik_server* server, radik_server_stats* stats);
/* Per-request latencies behind the statistics: for the requests completed
 * since the last reset, in completion order, tickets[i] and lat_us[i]
 * (submission to completion) for i < min(cap, *n); *n receives how many
 * there are.  Callers group them by request shape. */
int radik_server_get_latencies(radik_server* server, uint64_t* tickets, double* lat_us, int64_t cap, int64_t* n);
/* One launched batch: its k, rows (tasks), longest row, input elements, the
 * device time of its work on the slot's stream (plan upload to the last
 * kernel) and the host time the worker spent launching it. */
typedef struct radik_server_batch {
    int64_t k, rows, max_row_len;
    double elements, gpu_us, launch_us;
} radik_server_batch;
/* The batches completed since the last reset, in completion order:
 * out[i] for i < min(cap, *n); *n receives how many there are. */
int radik_server_get_batches(radik_server* server, radik_server_batch* out, int64_t cap, int64_t* n);
int radik_server_reset_stats(radik_server* server);

/* ---- Stage entry points: the reference kernels' own contracts ----------- */

/* count_bin_ex_kernel!, src/kernels/count_bin.jl:78-203: per-task histogram
 * of get_bin_id(apply_scaling(v), LEFT, RIGHT) over the concatenated tasks
 * (NaN skipped).  d_hist: int32 [num_tasks][2^(32-RIGHT)], overwritten. */
int radik_count_bin_ex(int32_t* d_hist, const float* d_data, const int64_t* h_task_lens, int64_t num_tasks,
                       int left, int right, int withscale, int largest, void* stream);

/* count_bin_kernel!, src/kernels/count_bin.jl:20-59: padded layout
 * d_data[t*stride + i], i < task_lens[t]. */
int radik_count_bin(int32_t* d_hist, const float* d_data, const int64_t* h_task_lens, int64_t stride,
                    int64_t num_tasks, int left, int right, void* stream);

/* select_bin_kernel!, src/kernels/select_bin.jl:268-348: per task, the
 * 1-based bin holding rank k_values[t] (from the top bin when largest),
 * the residual rank and the bin's count; entries are left unchanged when the
 * rank is out of range.  d_hist int32 [num_tasks][hist_len]. */
int radik_select_bin(int32_t* d_bin_ids, int32_t* d_k_values, int32_t* d_counts, const int32_t* d_hist,
                     int64_t num_tasks, int64_t hist_len, int largest, void* stream);

/* filter_kernel! / filter_general_kernel!, src/kernels/filter.jl:172-621:
 * emits (value, index) for elements strictly better than d_kth[t] and, for
 * elements equal to it, while the boundary counter d_boundary[t] stays >= 0
 * after decrement; tasks with len <= k copy everything.  Output rows have
 * stride k; d_counts[t] receives the number emitted (emission order is
 * unspecified, as in the reference). */
int radik_filter(float* d_val_out, void* d_idx_out, int idx_bytes, int32_t* d_counts, int32_t* d_boundary,
                 const float* d_data, const void* d_idx_in, const float* d_kth, const int64_t* h_task_lens,
                 int64_t num_tasks, int64_t k, int withscale, int largest, void* stream);

/* Engine diagnostics (no reference counterpart): the number of CUDA
 * allocations -- device memory and pinned host memory -- this library has
 * made in the process so far (workspace buffers, plan staging, the
 * host-buffer entry point's device copies, server slots).  Comparing it
 * before and after a call shows whether that call allocated. */
int radik_alloc_count(uint64_t* count);

/* Message of the last failure on this thread ("" when none). */
const char* radik_last_error(void);
const char* radik_status_string(int status);
/* Library version string. */
const char* radik_version(void);

#ifdef __cplusplus
}
#endif

#endif /* RADIK_B200_H */
