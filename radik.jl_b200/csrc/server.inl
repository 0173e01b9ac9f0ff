// server.inl -- request-batching top-k server (included by api.cu).
//
// Clients submit requests: a row-major [rows, row_len] Float32 matrix in
// device memory, k, flags and caller-owned output rows ([rows, k] values and
// indices).  A worker thread keeps a pool of slots -- each a CUDA stream, a
// device-resident workspace and a completion event -- and practises
// continuous batching: whenever a slot is free it packs the pending requests
// that share (k, flags, index width) into one fused launch (the kernels'
// per-task pointer mode: every row is a task with its own input and output
// pointers), up to max_batch_rows rows, admitting a request only while the
// bytes of the requests in flight plus the workspace pool stay under the
// memory cap.  Requests that arrive while batches run wait in the queue and
// join the next free slot, so work from different requests overlaps on the
// device across slots.  Completion is observed by polling the slots' events;
// a request's latency runs from its submission to the moment its batch is
// seen complete.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

namespace {

using ServerClock = std::chrono::steady_clock;

struct ServerReq {
    const float* data = nullptr;
    int64_t rows = 0, row_len = 0, k = 0;
    uint32_t flags = 0;
    float* vout = nullptr;
    void* iout = nullptr;
    int idx_bytes = 4;
    size_t bytes = 0;  // input + outputs, counted against the memory cap while in flight
    ServerClock::time_point t_submit, t_done;
    int status = RADIK_OK;
    bool done = false;
};

struct ServerSlot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done_ev = nullptr;
    cudaEvent_t t0_ev = nullptr, t1_ev = nullptr;  // the batch's device work, timed
    radik_server_batch info{};                     // the batch in flight (k, rows, elements, launch time)
    radik_ws* ws = nullptr;
    DevBuf io;                  // FusedTaskIO per row of the batch
    FusedTaskIO* h_io = nullptr;  // pinned staging
    size_t h_io_cap = 0;
    uint32_t* h_err = nullptr;  // pinned: the batch's device error word
    std::vector<uint64_t> reqs;
    size_t mem = 0;
    bool busy = false;
};

}  // namespace

struct radik_server {
    radik_server_config cfg{};
    int device = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> pending;
    std::unordered_map<uint64_t, ServerReq> reqs;
    std::vector<ServerSlot> slots;
    std::thread worker;
    bool stop = false;
    size_t in_flight = 0;
    uint64_t next_id = 1;
    uint64_t submitted = 0, completed = 0, batches = 0, rows = 0;
    double elements = 0;
    std::vector<double> lat_us;
    std::vector<uint64_t> lat_ticket;  // ticket of lat_us[i]
    std::vector<radik_server_batch> batch_log;  // completed batches since the last reset
    std::string worker_error;
    size_t pool_bytes = 0;  // device bytes of the slots' workspaces, updated by the worker under mu
};

namespace {

size_t server_pool_bytes(radik_server* sv) {
    size_t b = 0;
    for (auto& sl : sv->slots) {
        size_t x = 0;
        if (sl.ws && radik_ws_bytes(sl.ws, &x) == RADIK_OK) b += x;
        b += sl.io.bytes;
    }
    return b;
}

// Enqueues one batch (copies of its requests, all of one group) on a slot
// reserved for it.  Runs without the server's lock: it touches only the
// slot, which no other thread uses while it is reserved.
int server_launch(ServerSlot& sl, const std::vector<ServerReq>& batch) {
    const ServerReq& r0 = batch[0];
    int64_t T = 0, maxlen = 0;
    for (const ServerReq& r : batch) {
        T += r.rows;
        maxlen = std::max(maxlen, r.row_len);
    }
    std::vector<int64_t> lens;
    lens.reserve(T);
    if (sl.h_io_cap < static_cast<size_t>(T)) {
        if (sl.h_io) cudaFreeHost(sl.h_io);
        sl.h_io = nullptr;
        sl.h_io_cap = 0;
        const size_t cap = static_cast<size_t>(T) + static_cast<size_t>(T) / 2;  // headroom: reallocate rarely
        RADIK_CUDA(counted_malloc_host(&sl.h_io, sizeof(FusedTaskIO) * cap));
        sl.h_io_cap = cap;
    }
    int64_t row = 0;
    for (const ServerReq& r : batch) {
        for (int64_t i = 0; i < r.rows; ++i, ++row) {
            lens.push_back(r.row_len);
            FusedTaskIO& io = sl.h_io[row];
            io.data = r.data + i * r.row_len;
            io.val_out = r.vout + i * r.k;
            io.idx_out = static_cast<char*>(r.iout) + i * r.k * r.idx_bytes;
            io.idx_in = nullptr;
        }
    }
    radik_ws* ws = sl.ws;
    ws->num_tasks = std::max<int64_t>(ws->num_tasks, T);
    ws->n = std::max<int64_t>(ws->n, maxlen);
    sl.info.k = r0.k;
    sl.info.rows = T;
    sl.info.max_row_len = maxlen;
    sl.info.elements = 0;
    for (const ServerReq& r : batch) sl.info.elements += static_cast<double>(r.rows) * static_cast<double>(r.row_len);
    const uint32_t flags = r0.flags | RADIK_ASYNC;
    RADIK_CUDA(cudaEventRecord(sl.t0_ev, sl.stream));
    int rc = build_plan(ws, lens.data(), T, r0.k, flags, r0.idx_bytes, sl.stream, true);
    if (rc) return rc;
    if (!ws->plan.fused) return fail(RADIK_ERR_INVALID, "request shape has no fused plan (k too large to serve)");
    if (sl.io.ensure(sizeof(FusedTaskIO) * T, 1.5) != cudaSuccess) return fail(RADIK_ERR_OOM, "server io table");
    RADIK_CUDA(cudaMemcpyAsync(sl.io.p, sl.h_io, sizeof(FusedTaskIO) * T, cudaMemcpyHostToDevice, sl.stream));
    RADIK_CUDA(cudaMemsetAsync(err_ptr(ws), 0, 4, sl.stream));
    FusedParams p = fused_params(ws, nullptr, nullptr, r0.idx_bytes, nullptr, nullptr, r0.k, flags);
    p.task_io = sl.io.as<FusedTaskIO>();
    rc = run_fused(ws, p, flags, sl.stream);
    if (rc) return rc;
    RADIK_CUDA(cudaEventRecord(sl.t1_ev, sl.stream));
    RADIK_CUDA(cudaMemcpyAsync(sl.h_err, err_ptr(ws), 4, cudaMemcpyDeviceToHost, sl.stream));
    RADIK_CUDA(cudaEventRecord(sl.done_ev, sl.stream));
    return RADIK_OK;
}

void server_worker(radik_server* sv) {
    cudaSetDevice(sv->device);
    std::unique_lock<std::mutex> lk(sv->mu);
    for (;;) {
        bool progress = false;
        // Completions.
        for (auto& sl : sv->slots) {
            if (!sl.busy) continue;
            const cudaError_t q = cudaEventQuery(sl.done_ev);
            if (q == cudaErrorNotReady) continue;
            const auto now = ServerClock::now();
            const int st = (q != cudaSuccess) ? RADIK_ERR_CUDA : (*sl.h_err ? RADIK_ERR_DEVICE : RADIK_OK);
            if (q != cudaSuccess) cudaGetLastError();
            for (uint64_t id : sl.reqs) {
                ServerReq& r = sv->reqs[id];
                r.done = true;
                r.status = st;
                r.t_done = now;
                sv->completed += 1;
                sv->rows += static_cast<uint64_t>(r.rows);
                sv->elements += static_cast<double>(r.rows) * static_cast<double>(r.row_len);
                sv->lat_us.push_back(std::chrono::duration<double, std::micro>(r.t_done - r.t_submit).count());
                sv->lat_ticket.push_back(id);
            }
            if (q == cudaSuccess) {
                float ms = 0.0f;
                if (cudaEventElapsedTime(&ms, sl.t0_ev, sl.t1_ev) != cudaSuccess) cudaGetLastError();
                sl.info.gpu_us = 1e3 * static_cast<double>(ms);
                sv->batch_log.push_back(sl.info);
            }
            sv->in_flight -= sl.mem;
            sl.mem = 0;
            sl.reqs.clear();
            sl.busy = false;
            progress = true;
        }
        if (progress) sv->cv_done.notify_all();
        // Dispatch: fill free slots from the queue.
        for (auto& sl : sv->slots) {
            if (sl.busy || sv->pending.empty()) continue;
            const ServerReq& head = sv->reqs[sv->pending.front()];
            const int64_t k = head.k;
            const uint32_t fl = head.flags;
            const int ib = head.idx_bytes;
            const size_t pool = server_pool_bytes(sv);
            std::vector<uint64_t> ids;
            int64_t rows = 0;
            size_t mem = 0;
            for (auto it = sv->pending.begin(); it != sv->pending.end();) {
                const ServerReq& r = sv->reqs[*it];
                if (r.k != k || r.flags != fl || r.idx_bytes != ib) { ++it; continue; }
                if (!ids.empty() && rows + r.rows > sv->cfg.max_batch_rows) break;
                // Admission by memory; with nothing in flight the head request is
                // admitted anyway (the pool is already allocated), so the queue
                // always makes progress.
                const bool alone = sv->in_flight == 0 && ids.empty();
                if (!alone && pool + sv->in_flight + mem + r.bytes > static_cast<size_t>(sv->cfg.mem_cap_bytes)) break;
                ids.push_back(*it);
                rows += r.rows;
                mem += r.bytes;
                it = sv->pending.erase(it);
            }
            if (ids.empty()) break;  // admission: wait for memory to free up
            // Reserve the slot and its memory, then launch without the lock so
            // that submitters and waiters are not held up by the plan build,
            // the uploads or a workspace that grows.
            std::vector<ServerReq> batch;
            batch.reserve(ids.size());
            for (uint64_t id : ids) batch.push_back(sv->reqs[id]);
            sl.busy = true;
            sl.mem = mem;
            sv->in_flight += mem;
            lk.unlock();
            const auto l0 = ServerClock::now();
            const int rc = server_launch(sl, batch);
            sl.info.launch_us = std::chrono::duration<double, std::micro>(ServerClock::now() - l0).count();
            std::string err;
            if (rc != RADIK_OK) {
                err = g_last_error;
                // Kernels of the batch may already be enqueued: the callers'
                // buffers stay in use until they are done.
                cudaStreamSynchronize(sl.stream);
                cudaGetLastError();
            }
            lk.lock();
            sv->pool_bytes = server_pool_bytes(sv);
            if (rc != RADIK_OK) {
                const auto now = ServerClock::now();
                for (uint64_t id : ids) {
                    ServerReq& r = sv->reqs[id];
                    r.done = true;
                    r.status = rc;
                    r.t_done = now;
                }
                sv->worker_error = err;
                sl.busy = false;
                sv->in_flight -= sl.mem;
                sl.mem = 0;
                sv->cv_done.notify_all();
                continue;
            }
            sl.reqs = std::move(ids);
            sv->batches += 1;
            progress = true;
        }
        bool any_busy = false;
        for (auto& sl : sv->slots) any_busy = any_busy || sl.busy;
        if (sv->stop && sv->pending.empty() && !any_busy) break;
        if (!progress) {
            if (any_busy) {
                lk.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(5));
                lk.lock();
            } else {
                sv->cv_work.wait_for(lk, std::chrono::milliseconds(2));
            }
        }
    }
}

}  // namespace

extern "C" {

int radik_server_create(const radik_server_config* cfg, radik_server** out) {
    if (!cfg || !out) return fail(RADIK_ERR_INVALID, "NULL argument");
    *out = nullptr;
    if (cfg->slots < 1 || cfg->slots > 64) return fail(RADIK_ERR_INVALID, "slots must be in [1, 64]");
    if (cfg->mem_cap_bytes <= 0 || cfg->max_batch_rows < 1)
        return fail(RADIK_ERR_INVALID, "mem_cap_bytes and max_batch_rows must be positive");
    radik_server* sv = new (std::nothrow) radik_server();
    if (!sv) return fail(RADIK_ERR_OOM, "host allocation of the server failed");
    sv->cfg = *cfg;
    sv->device = cfg->device;
    RADIK_CUDA(cudaSetDevice(sv->device));
    sv->slots.resize(cfg->slots);
    for (auto& sl : sv->slots) {
        int rc = RADIK_OK;
        if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.done_ev, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreate(&sl.t0_ev) != cudaSuccess || cudaEventCreate(&sl.t1_ev) != cudaSuccess ||
            counted_malloc_host(&sl.h_err, sizeof(uint32_t)) != cudaSuccess)
            rc = fail(RADIK_ERR_CUDA, "server slot set-up failed");
        if (rc == RADIK_OK) rc = radik_ws_create(1, 1, 4, &sl.ws);
        if (rc == RADIK_OK) sl.ws->grow = 1.5;  // batches vary: grow with headroom, reallocate rarely
        if (rc != RADIK_OK) {
            radik_server_destroy(sv);
            return rc;
        }
        *sl.h_err = 0;
    }
    sv->worker = std::thread(server_worker, sv);
    *out = sv;
    return RADIK_OK;
}

int radik_server_destroy(radik_server* sv) {
    if (!sv) return RADIK_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    if (sv->worker.joinable()) sv->worker.join();
    for (auto& sl : sv->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        if (sl.ws) radik_ws_destroy(sl.ws);
        sl.io.release();
        if (sl.h_io) cudaFreeHost(sl.h_io);
        if (sl.h_err) cudaFreeHost(sl.h_err);
        if (sl.done_ev) cudaEventDestroy(sl.done_ev);
        if (sl.t0_ev) cudaEventDestroy(sl.t0_ev);
        if (sl.t1_ev) cudaEventDestroy(sl.t1_ev);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    delete sv;
    return RADIK_OK;
}

int radik_server_submit(radik_server* sv, const float* d_data, int64_t rows, int64_t row_len, int64_t k,
                        uint32_t flags, float* d_val_out, void* d_idx_out, int idx_bytes, uint64_t* ticket) {
    if (!sv || !ticket) return fail(RADIK_ERR_INVALID, "NULL argument");
    if (rows < 1 || row_len < 1 || k < 1) return fail(RADIK_ERR_INVALID, "rows, row_len and k must be positive");
    if (row_len > INT32_MAX) return fail(RADIK_ERR_INVALID, "a row may hold at most 2^31-1 elements");
    if (idx_bytes != 4 && idx_bytes != 8) return fail(RADIK_ERR_INVALID, "index width must be 4 or 8 bytes");
    if (!d_data || !d_val_out || !d_idx_out) return fail(RADIK_ERR_INVALID, "NULL data or output");
    if (flags & (RADIK_PLAIN | RADIK_WITHIDXIN))
        return fail(RADIK_ERR_INVALID, "served requests use the fused path with automatic indices");
    ServerReq r;
    r.data = d_data;
    r.rows = rows;
    r.row_len = row_len;
    r.k = k;
    r.flags = flags & (RADIK_LARGEST | RADIK_ASCEND | RADIK_WITHSCALE);
    r.vout = d_val_out;
    r.iout = d_idx_out;
    r.idx_bytes = idx_bytes;
    r.bytes = static_cast<size_t>(rows) * (static_cast<size_t>(row_len) * 4 + static_cast<size_t>(k) * (4 + idx_bytes));
    if (r.bytes > static_cast<size_t>(sv->cfg.mem_cap_bytes))
        return fail(RADIK_ERR_WS_TOO_SMALL, "request exceeds the server's memory cap");
    r.t_submit = ServerClock::now();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        const uint64_t id = sv->next_id++;
        sv->reqs.emplace(id, r);
        sv->pending.push_back(id);
        sv->submitted += 1;
        *ticket = id;
    }
    sv->cv_work.notify_one();
    return RADIK_OK;
}

int radik_server_wait(radik_server* sv, uint64_t ticket, int64_t timeout_us) {
    if (!sv) return fail(RADIK_ERR_INVALID, "NULL argument");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(ticket);
    if (it == sv->reqs.end()) return fail(RADIK_ERR_INVALID, "unknown or already collected ticket");
    const auto deadline = ServerClock::now() + std::chrono::microseconds(timeout_us < 0 ? 0 : timeout_us);
    while (!it->second.done) {
        if (timeout_us >= 0 && ServerClock::now() >= deadline) return RADIK_ERR_TIMEOUT;
        sv->cv_done.wait_for(lk, std::chrono::milliseconds(1));
        it = sv->reqs.find(ticket);
    }
    const int st = it->second.status;
    sv->reqs.erase(it);
    if (st != RADIK_OK) return fail(st, sv->worker_error.empty() ? "request failed on the device" : sv->worker_error);
    return RADIK_OK;
}

int radik_server_get_stats(radik_server* sv, radik_server_stats* out) {
    if (!sv || !out) return fail(RADIK_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    out->submitted = sv->submitted;
    out->completed = sv->completed;
    out->batches = sv->batches;
    out->rows = sv->rows;
    out->elements = sv->elements;
    std::vector<double> l = sv->lat_us;
    std::sort(l.begin(), l.end());
    auto pct = [&](double q) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, static_cast<size_t>(q * (l.size() - 1) + 0.5))]; };
    out->p50_us = pct(0.50);
    out->p99_us = pct(0.99);
    double sum = 0;
    for (double x : l) sum += x;
    out->mean_us = l.empty() ? 0.0 : sum / static_cast<double>(l.size());
    out->mem_in_flight = static_cast<int64_t>(sv->in_flight);
    out->mem_pool = static_cast<int64_t>(sv->pool_bytes);
    return RADIK_OK;
}

int radik_server_get_latencies(radik_server* sv, uint64_t* tickets, double* lat_us, int64_t cap, int64_t* n) {
    if (!sv || !n || cap < 0 || (cap > 0 && (!tickets || !lat_us))) return fail(RADIK_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    const int64_t have = static_cast<int64_t>(sv->lat_us.size());
    for (int64_t i = 0; i < std::min(cap, have); ++i) {
        tickets[i] = sv->lat_ticket[i];
        lat_us[i] = sv->lat_us[i];
    }
    *n = have;
    return RADIK_OK;
}

int radik_server_get_batches(radik_server* sv, radik_server_batch* out, int64_t cap, int64_t* n) {
    if (!sv || !n || cap < 0 || (cap > 0 && !out)) return fail(RADIK_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    const int64_t have = static_cast<int64_t>(sv->batch_log.size());
    for (int64_t i = 0; i < std::min(cap, have); ++i) out[i] = sv->batch_log[i];
    *n = have;
    return RADIK_OK;
}

int radik_server_reset_stats(radik_server* sv) {
    if (!sv) return fail(RADIK_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->completed = sv->batches = sv->rows = 0;
    sv->submitted = 0;
    sv->elements = 0;
    sv->lat_us.clear();
    sv->lat_ticket.clear();
    sv->batch_log.clear();
    return RADIK_OK;
}

}  // extern "C"
