// svo_server.cpp -- a request loop around the batched build (continuous
// batching under a device-memory budget).  No counterpart in the reference,
// which builds one mesh per process (main.cpp:8-14).
//
// Requests wait in a FIFO queue.  Each worker thread owns a CUDA stream and
// repeatedly takes the longest queue prefix that fits the budget (at most
// max_batch requests), builds it as one batch (svo_batch_create, then one
// svo_batch_emit for all of it) and publishes the results.  While one
// worker's batch is on the GPU the others admit what arrived meanwhile and
// launch on their own streams, so batches of different sizes overlap on the
// device.  Admission reserves svo_estimate_bytes() per request.  Once the
// batch's counting phase knows each result's exact size, the batch keeps the
// longest prefix whose exact needs fit the budget beside what other batches
// hold and sends the rest back to the front of the queue with their exact
// sizes; after emission a request holds the exact bytes of its result until
// the client releases it.  Queued requests can be cancelled.
#include <chrono>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <set>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "svo_b200.h"
#include "svo_host.h"

struct svo_server {
    struct Req {
        uint64_t ticket = 0;
        svo_mesh_desc desc{};
        uint64_t est = 0;   // bytes reserved at admission
        uint64_t base = 0;  // the inputs + scratch part of est
        uint64_t held = 0;  // bytes reserved now
        std::chrono::steady_clock::time_point t_submit, t_start, t_done;
        bool done = false;
        int status = SVO_OK;
        svo_result *result = nullptr;
    };
    svo_ctx *ctx = nullptr;
    svo_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_decide;
    uint64_t admitted_batches = 0;  // sequence number of the next batch admitted
    uint64_t decided_batches = 0;   // batches whose keep/requeue decision is made
    std::deque<Req *> queue;         // pending requests in ticket (arrival) order
    std::set<uint64_t> unkept;       // tickets neither kept by a batch nor finished nor cancelled
    std::deque<uint64_t> finished;  // tickets in completion order, not yet taken by svo_server_next
    std::unordered_map<uint64_t, Req *> reqs;
    uint64_t next_ticket = 1;
    uint64_t reserved = 0;
    uint64_t peak_reserved = 0;
    int busy = 0;  // workers with a batch on the device
    bool stop = false;
    std::vector<std::thread> workers;
    std::vector<cudaStream_t> streams;
    uint64_t batches = 0, built = 0, requeued = 0;
    double build_s = 0.0, queue_s = 0.0;  // summed over batches / requests
    void (*on_finish)(void *, uint64_t) = nullptr;  // called under mu for each finished request
    void *on_finish_arg = nullptr;
};

namespace {

using Clock = std::chrono::steady_clock;

// SVO_SERVER_TRACE=1 in the environment: admissions, keep/requeue decisions,
// publications and releases on stderr (for diagnosing admission under a tight
// budget).
bool trace_on() {
    static const bool on = [] {
        const char *v = std::getenv("SVO_SERVER_TRACE");
        return v && *v && *v != '0';
    }();
    return on;
}
#define SVO_TRACE(...)                          \
    do {                                        \
        if (trace_on()) {                       \
            std::fprintf(stderr, "[svo_server] " __VA_ARGS__); \
            std::fputc('\n', stderr);           \
        }                                       \
    } while (0)

int server_fail(int code, const char *msg) {
    svo::host::set_error(msg);
    return code;
}

int max_res(const int r[3]) { return std::max(r[0], std::max(r[1], r[2])); }

// Admission estimate: inputs + scratch of a res^3 grid (`base`) and the
// outputs of 16*res^2 nodes (a closed surface spanning the grid).
uint64_t estimate_parts(int64_t n_points, int64_t n_tris, const int res[3], uint32_t flags, uint64_t *base) {
    uint64_t side = 1;
    while (side < (uint64_t)max_res(res)) side *= 2;
    const uint64_t nt = n_tris > 0 ? (uint64_t)n_tris : (uint64_t)std::max<int64_t>(n_points, 0) / 3;
    const uint64_t inputs = 12 * (uint64_t)std::max<int64_t>(n_points, 0) + 12 * nt;
    // level bitmaps (side^3 / 7 bytes), triangle queues; with dedup its candidate bitmap (side^3 / 8)
    const uint64_t scratch = side * side * side / 7 + 32 * nt + (1u << 20) +
                             ((flags & SVO_FLAG_DEDUP) ? side * side * side / 8 : 0);
    const uint64_t nodes = 16 * side * side;
    uint64_t per_node = sizeof(svo_node);
    if (!(flags & SVO_FLAG_NO_VERT_EDGE)) per_node += 8 * sizeof(svo_vertex) + 12 * sizeof(svo_edge);
    if (flags & SVO_FLAG_DEDUP) per_node += 8 * 4;
    *base = inputs + scratch;
    return inputs + scratch + nodes * per_node;
}

void reserve(svo_server *s, uint64_t add, uint64_t remove) {
    s->reserved = s->reserved + add - remove;
    s->peak_reserved = std::max(s->peak_reserved, s->reserved);
}

// The longest FIFO prefix that fits the budget; a request larger than the
// whole budget runs alone when nothing else is reserved.
bool admissible(const svo_server *s) {
    if (s->queue.empty()) return false;
    const uint64_t e = s->queue.front()->est;
    return s->reserved + e <= s->cfg.mem_budget || s->reserved == 0;
}

void publish(svo_server *s, svo_server::Req *r, svo_result *res, int status, uint64_t bytes,
             Clock::time_point now) {
    reserve(s, bytes, r->held);
    r->held = bytes;
    r->result = res;
    r->status = status;
    r->t_done = now;
    r->done = true;
    s->finished.push_back(r->ticket);
    if (s->on_finish) s->on_finish(s->on_finish_arg, r->ticket);
}

// seq: the batch's admission sequence number.  Batches count concurrently but
// make their keep/requeue decisions in admission order, and a request is kept
// only when every older request is kept, finished or cancelled; requests sent
// back return to their arrival position.  Memory thus goes to requests first
// come, first served: a younger result never holds the memory an older
// request waits for (a client waiting for requests in arrival order, holding
// the younger result, would wait forever).
void run_batch(svo_server *s, cudaStream_t st, std::vector<svo_server::Req *> &take, uint64_t seq) {
    svo::host::TraceRange trace("svo_server: batch");
    const int n = (int)take.size();
    const auto t0 = Clock::now();
    std::vector<svo_mesh_desc> d(n);
    for (int i = 0; i < n; ++i) d[i] = take[i]->desc;
    std::vector<svo_result *> out(n, nullptr);
    std::vector<int> status(n, SVO_OK);
    std::vector<uint64_t> bytes(n, 0);
    svo_batch *b = nullptr;
    int keep = n;  // take[0, keep) is built by this batch; the rest is requeued
    int rc = svo_batch_create(s->ctx, d.data(), n, s->cfg.flags, st, &b);
    auto decided = [&]() {  // under s->mu
        ++s->decided_batches;
        s->cv_decide.notify_all();
    };
    if (rc == SVO_OK) {
        // Exact output sizes are known now.  Hold them instead of the
        // estimates for the prefix that fits beside what others hold; send
        // the rest back to the front of the queue with their exact sizes.
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_decide.wait(lk, [&] { return s->decided_batches == seq; });
            uint64_t mine = 0;
            for (svo_server::Req *r : take) mine += r->held;
            const uint64_t others = s->reserved - mine;
            uint64_t acc = 0, drop = 0;
            keep = 0;
            for (int i = 0; i < n; ++i) {
                const int64_t ob = svo_batch_mesh_output_bytes(b, i);  // -1: this mesh failed counting
                const uint64_t need = take[i]->base + (ob > 0 ? (uint64_t)ob : 0);
                const bool fits = others + acc + need <= s->cfg.mem_budget || (others == 0 && i == 0);
                // memory goes to requests in arrival order: a request is kept only
                // when every older one is kept, finished or cancelled
                const bool oldest = !s->unkept.empty() && *s->unkept.begin() == take[i]->ticket;
                drop += take[i]->held;
                if (keep == i && fits && oldest) {
                    acc += need;
                    take[i]->held = need;
                    s->unkept.erase(take[i]->ticket);
                    ++keep;
                } else {
                    take[i]->est = need;
                    take[i]->held = 0;
                }
            }
            reserve(s, acc, drop);
            for (int i = keep; i < n; ++i) {  // back into the queue at their arrival position
                auto at = std::lower_bound(s->queue.begin(), s->queue.end(), take[i]->ticket,
                                           [](const svo_server::Req *q, uint64_t t) { return q->ticket < t; });
                s->queue.insert(at, take[i]);
            }
            s->requeued += (uint64_t)(n - keep);
            SVO_TRACE("decide seq %llu: %d of %d kept (first ticket %llu), others %llu, reserved %llu",
                      (unsigned long long)seq, keep, n, (unsigned long long)take[0]->ticket,
                      (unsigned long long)others, (unsigned long long)s->reserved);
            decided();
        }
        if (keep < n) s->cv_work.notify_all();
        if (keep > 0) {
            rc = svo_batch_emit(b, 0, keep, out.data(), status.data());
            for (int i = 0; i < keep; ++i)
                if (status[i] == SVO_OK) bytes[i] = (uint64_t)svo_batch_mesh_output_bytes(b, i);
        }
        svo_batch_free(b);
    } else {
        for (int i = 0; i < n; ++i) status[i] = rc;
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_decide.wait(lk, [&] { return s->decided_batches == seq; });
        for (svo_server::Req *r : take) s->unkept.erase(r->ticket);  // finished, with the error
        decided();
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        const auto now = Clock::now();
        for (int i = 0; i < keep; ++i) publish(s, take[i], out[i], status[i], bytes[i], now);
        SVO_TRACE("seq %llu publishes %d (rc %d), reserved %llu, queued %zu", (unsigned long long)seq, keep, rc,
                  (unsigned long long)s->reserved, s->queue.size());
        if (keep > 0) s->batches += 1;
        s->built += (uint64_t)keep;
        s->build_s += std::chrono::duration<double>(now - t0).count();
        for (int i = 0; i < keep; ++i)
            s->queue_s += std::chrono::duration<double>(take[i]->t_start - take[i]->t_submit).count();
        --s->busy;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
}

void worker(svo_server *s, int w) {
    int dev = 0;
    svo_ctx_device(s->ctx, &dev);
    cudaSetDevice(dev);
    cudaStream_t st = s->streams[w];
    for (;;) {
        std::vector<svo_server::Req *> take;
        uint64_t seq = 0;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return admissible(s) || (s->stop && s->queue.empty()); });
            if (s->queue.empty()) return;  // stopping and drained
            const auto now = Clock::now();
            while (!s->queue.empty() && (int)take.size() < s->cfg.max_batch) {
                svo_server::Req *r = s->queue.front();
                if (s->reserved + r->est > s->cfg.mem_budget && !(s->reserved == 0 && take.empty())) break;
                reserve(s, r->est, 0);
                r->held = r->est;
                r->t_start = now;
                take.push_back(r);
                s->queue.pop_front();
            }
            ++s->busy;
            seq = s->admitted_batches++;
            SVO_TRACE("worker %d admits seq %llu: %zu requests from ticket %llu, reserved %llu, queued %zu", w,
                      (unsigned long long)seq, take.size(), (unsigned long long)take[0]->ticket,
                      (unsigned long long)s->reserved, s->queue.size());
        }
        run_batch(s, st, take, seq);
    }
}

}  // namespace

namespace svo::host {

void server_on_finish(svo_server *s, void (*fn)(void *, uint64_t), void *arg) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->on_finish = fn;
    s->on_finish_arg = arg;
}

}  // namespace svo::host

extern "C" {

uint64_t svo_estimate_bytes(int64_t n_points, int64_t n_tris, int res_x, int res_y, int res_z, uint32_t flags) {
    const int r[3] = {res_x, res_y, res_z};
    uint64_t base = 0;
    return estimate_parts(n_points, n_tris, r, flags, &base);
}

int svo_server_create(svo_ctx *ctx, const svo_server_config *cfg, svo_server **out) {
    if (!ctx || !cfg || !out) return server_fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (cfg->workers < 1 || cfg->workers > 64 || cfg->max_batch < 1 || cfg->mem_budget == 0)
        return server_fail(SVO_ERR_INVALID_ARGUMENT, "workers in [1, 64], max_batch >= 1, mem_budget > 0");
    int dev = 0;
    svo_ctx_device(ctx, &dev);
    if (cudaSetDevice(dev) != cudaSuccess) return server_fail(SVO_ERR_CUDA, "cudaSetDevice");
    svo_server *s = new svo_server();
    s->ctx = ctx;
    s->cfg = *cfg;
    for (int w = 0; w < cfg->workers; ++w) {
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            for (cudaStream_t x : s->streams) cudaStreamDestroy(x);
            delete s;
            return server_fail(SVO_ERR_CUDA, "worker stream");
        }
        s->streams.push_back(st);
    }
    // Map the budget's memory into the context's pools now, so that batches
    // carve cached memory instead of growing the pools while serving.
    svo_ctx_reserve(ctx, cfg->mem_budget, cfg->mem_budget / 4, s->streams[0]);
    for (int w = 0; w < cfg->workers; ++w) s->workers.emplace_back(worker, s, w);
    *out = s;
    return SVO_OK;
}

int svo_server_submit(svo_server *s, const svo_mesh_desc *desc, uint64_t *ticket) {
    if (!s || !desc || !ticket) return server_fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    auto *r = new svo_server::Req();
    r->desc = *desc;
    r->est = estimate_parts(desc->n_points, desc->n_tris, desc->res, s->cfg.flags, &r->base);
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            delete r;
            return server_fail(SVO_ERR_INVALID_ARGUMENT, "server is shutting down");
        }
        r->ticket = s->next_ticket++;
        s->reqs[r->ticket] = r;
        s->queue.push_back(r);
        s->unkept.insert(r->ticket);
        *ticket = r->ticket;
    }
    s->cv_work.notify_one();
    return SVO_OK;
}

int svo_server_wait(svo_server *s, uint64_t ticket, int64_t timeout_us, svo_result **result, int *status,
                    double *latency_s) {
    if (!s) return server_fail(SVO_ERR_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return server_fail(SVO_ERR_INVALID_ARGUMENT, "unknown ticket");
    svo_server::Req *r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_us < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), ready)) {
        return server_fail(SVO_ERR_TIMEOUT, "request not finished");
    }
    if (result) *result = r->result;
    if (status) *status = r->status;
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    return SVO_OK;
}

int svo_server_next(svo_server *s, int64_t timeout_us, uint64_t *ticket, svo_result **result, int *status,
                    double *latency_s) {
    if (!s || !ticket) return server_fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto ready = [&] { return !s->finished.empty(); };
    if (timeout_us < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), ready)) {
        return server_fail(SVO_ERR_TIMEOUT, "no finished request");
    }
    *ticket = s->finished.front();
    s->finished.pop_front();
    svo_server::Req *r = s->reqs.at(*ticket);
    if (result) *result = r->result;
    if (status) *status = r->status;
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    return SVO_OK;
}

int svo_server_release(svo_server *s, uint64_t ticket) {
    if (!s) return server_fail(SVO_ERR_INVALID_ARGUMENT, "null server");
    svo_result *res = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return server_fail(SVO_ERR_INVALID_ARGUMENT, "unknown ticket");
        svo_server::Req *r = it->second;
        if (!r->done) return server_fail(SVO_ERR_INVALID_ARGUMENT, "request not finished");
        for (auto f = s->finished.begin(); f != s->finished.end(); ++f)
            if (*f == ticket) {
                s->finished.erase(f);
                break;
            }
        reserve(s, 0, r->held);
        SVO_TRACE("release ticket %llu, reserved %llu, queued %zu", (unsigned long long)ticket,
                  (unsigned long long)s->reserved, s->queue.size());
        res = r->result;
        s->reqs.erase(it);
        delete r;
    }
    svo_result_free(res);
    s->cv_work.notify_all();
    return SVO_OK;
}

int svo_server_cancel(svo_server *s, uint64_t ticket) {
    if (!s) return server_fail(SVO_ERR_INVALID_ARGUMENT, "null server");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return server_fail(SVO_ERR_INVALID_ARGUMENT, "unknown ticket");
        svo_server::Req *r = it->second;
        auto q = std::find(s->queue.begin(), s->queue.end(), r);
        if (q == s->queue.end())
            return server_fail(SVO_ERR_INVALID_ARGUMENT, r->done ? "request already finished"
                                                               : "request already building");
        s->queue.erase(q);
        s->unkept.erase(ticket);
        publish(s, r, nullptr, SVO_ERR_CANCELLED, 0, Clock::now());
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
    return SVO_OK;
}

int svo_server_stats(const svo_server *s, svo_server_stats_t *out) {
    if (!s || !out) return server_fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    auto *m = const_cast<svo_server *>(s);
    std::lock_guard<std::mutex> lk(m->mu);
    out->queued = (int64_t)s->queue.size();
    out->busy_workers = s->busy;
    out->reserved_bytes = s->reserved;
    out->batches = s->batches;
    out->built = s->built;
    out->build_seconds = s->build_s;
    out->queue_seconds = s->queue_s;
    out->peak_reserved_bytes = s->peak_reserved;
    out->requeued = s->requeued;
    out->admitted_batches = s->admitted_batches;
    out->decided_batches = s->decided_batches;
    return SVO_OK;
}

void svo_server_destroy(svo_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        // finished results nobody can take any more: freed now, so that their
        // bytes admit what is still queued (the queue is built to the end)
        for (auto &kv : s->reqs) {
            svo_server::Req *r = kv.second;
            if (!r->done) continue;
            svo_result_free(r->result);
            r->result = nullptr;
            reserve(s, 0, r->held);
            r->held = 0;
        }
    }
    s->cv_work.notify_all();
    for (auto &t : s->workers) t.join();
    for (auto &kv : s->reqs) {
        svo_result_free(kv.second->result);
        delete kv.second;
    }
    for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
    delete s;
}

}  // extern "C"
