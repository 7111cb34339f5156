// svo_fleet.cpp -- served builds over several GPUs: one svo_server per
// context (one context per device) behind one ticket space.  No counterpart in
// the reference, which builds one mesh per process (main.cpp:8-14).
//
// A request is built whole by one member, so the members never exchange data
// (replicas, no collective).  Fleet ticket = member ticket * n + member index:
// the mapping is a function, so nothing has to be recorded before a member can
// finish a request.  Routing: the member with the fewest estimated bytes
// submitted and not yet released (ties: the lowest index), which spreads large
// and small requests alike.  Completion order across the members comes from a
// hook each member calls, under its own lock, when a request finishes; the
// fleet's lock is only ever taken inside a member's (the hook) or alone, never
// around a call into a member.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "svo_b200.h"
#include "svo_host.h"

struct svo_fleet {
    struct Member {
        svo_fleet *fleet = nullptr;
        int index = 0;
        svo_server *server = nullptr;
        uint64_t outstanding = 0;  // estimated bytes submitted and not yet released
    };
    std::vector<Member> members;  // sized once at creation: the hooks point into it
    svo_server_config cfg{};
    mutable std::mutex mu;
    std::condition_variable cv_done;
    std::deque<uint64_t> finished;             // fleet tickets in completion order, not yet reported
    std::unordered_map<uint64_t, uint64_t> est;  // live fleet tickets -> their estimates
};

namespace {

using Clock = std::chrono::steady_clock;

int fleet_fail(int code, const char *msg) {
    svo::host::set_error(msg);
    return code;
}

void on_member_finish(void *arg, uint64_t member_ticket) {
    auto *m = static_cast<svo_fleet::Member *>(arg);
    svo_fleet *f = m->fleet;
    {
        std::lock_guard<std::mutex> lk(f->mu);
        f->finished.push_back(member_ticket * f->members.size() + (uint64_t)m->index);
    }
    f->cv_done.notify_all();
}

// The member and its ticket for a fleet ticket; false when it cannot be one.
bool decode(const svo_fleet *f, uint64_t ticket, int *member, uint64_t *member_ticket) {
    const uint64_t n = f->members.size();
    *member = (int)(ticket % n);
    *member_ticket = ticket / n;
    return *member_ticket >= 1;
}

}  // namespace

extern "C" {

int svo_fleet_create(svo_ctx *const *ctxs, int n, const svo_server_config *cfg, svo_fleet **out) {
    if (!ctxs || !cfg || !out) return fleet_fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (n < 1 || n > 64) return fleet_fail(SVO_ERR_INVALID_ARGUMENT, "1 to 64 members");
    for (int i = 0; i < n; ++i)
        if (!ctxs[i]) return fleet_fail(SVO_ERR_INVALID_ARGUMENT, "null context");
    auto *f = new svo_fleet();
    f->cfg = *cfg;
    f->members.resize(n);
    for (int i = 0; i < n; ++i) {
        svo_fleet::Member &m = f->members[i];
        m.fleet = f;
        m.index = i;
        const int rc = svo_server_create(ctxs[i], cfg, &m.server);
        if (rc != SVO_OK) {
            for (int j = 0; j < i; ++j) svo_server_destroy(f->members[j].server);
            delete f;
            return rc;  // svo_server_create set the message
        }
        svo::host::server_on_finish(m.server, on_member_finish, &m);
    }
    *out = f;
    return SVO_OK;
}

int svo_fleet_submit(svo_fleet *f, const svo_mesh_desc *desc, uint64_t *ticket) {
    if (!f || !desc || !ticket) return fleet_fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    const uint64_t e = svo_estimate_bytes(desc->n_points, desc->n_tris, desc->res[0], desc->res[1], desc->res[2],
                                          f->cfg.flags);
    int pick = 0;
    {
        std::lock_guard<std::mutex> lk(f->mu);
        for (int i = 1; i < (int)f->members.size(); ++i)
            if (f->members[i].outstanding < f->members[pick].outstanding) pick = i;
        f->members[pick].outstanding += e;
    }
    uint64_t mt = 0;
    const int rc = svo_server_submit(f->members[pick].server, desc, &mt);
    std::lock_guard<std::mutex> lk(f->mu);
    if (rc != SVO_OK) {
        f->members[pick].outstanding -= e;
        return rc;
    }
    *ticket = mt * f->members.size() + (uint64_t)pick;
    f->est[*ticket] = e;
    return SVO_OK;
}

int svo_fleet_wait(svo_fleet *f, uint64_t ticket, int64_t timeout_us, svo_result **result, int *status,
                   double *latency_s) {
    if (!f) return fleet_fail(SVO_ERR_INVALID_ARGUMENT, "null fleet");
    int m = 0;
    uint64_t mt = 0;
    if (!decode(f, ticket, &m, &mt)) return fleet_fail(SVO_ERR_INVALID_ARGUMENT, "unknown ticket");
    return svo_server_wait(f->members[m].server, mt, timeout_us, result, status, latency_s);
}

int svo_fleet_next(svo_fleet *f, int64_t timeout_us, uint64_t *ticket, svo_result **result, int *status,
                   double *latency_s) {
    if (!f || !ticket) return fleet_fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    const auto deadline = Clock::now() + std::chrono::microseconds(std::max<int64_t>(timeout_us, 0));
    for (;;) {
        uint64_t t = 0;
        {
            std::unique_lock<std::mutex> lk(f->mu);
            auto ready = [&] { return !f->finished.empty(); };
            if (timeout_us < 0) {
                f->cv_done.wait(lk, ready);
            } else if (!f->cv_done.wait_until(lk, deadline, ready)) {
                return fleet_fail(SVO_ERR_TIMEOUT, "no finished request");
            }
            t = f->finished.front();
            f->finished.pop_front();
        }
        int m = 0;
        uint64_t mt = 0;
        decode(f, t, &m, &mt);
        // finished, so the member answers at once -- unless the client released
        // the ticket meanwhile, which drops it from the completion order
        if (svo_server_wait(f->members[m].server, mt, 0, result, status, latency_s) == SVO_OK) {
            *ticket = t;
            return SVO_OK;
        }
    }
}

int svo_fleet_release(svo_fleet *f, uint64_t ticket) {
    if (!f) return fleet_fail(SVO_ERR_INVALID_ARGUMENT, "null fleet");
    int m = 0;
    uint64_t mt = 0;
    if (!decode(f, ticket, &m, &mt)) return fleet_fail(SVO_ERR_INVALID_ARGUMENT, "unknown ticket");
    const int rc = svo_server_release(f->members[m].server, mt);
    if (rc != SVO_OK) return rc;
    std::lock_guard<std::mutex> lk(f->mu);
    auto it = std::find(f->finished.begin(), f->finished.end(), ticket);
    if (it != f->finished.end()) f->finished.erase(it);
    auto e = f->est.find(ticket);
    if (e != f->est.end()) {
        f->members[m].outstanding -= e->second;
        f->est.erase(e);
    }
    return SVO_OK;
}

int svo_fleet_cancel(svo_fleet *f, uint64_t ticket) {
    if (!f) return fleet_fail(SVO_ERR_INVALID_ARGUMENT, "null fleet");
    int m = 0;
    uint64_t mt = 0;
    if (!decode(f, ticket, &m, &mt)) return fleet_fail(SVO_ERR_INVALID_ARGUMENT, "unknown ticket");
    return svo_server_cancel(f->members[m].server, mt);
}

int svo_fleet_member(const svo_fleet *f, uint64_t ticket) {
    if (!f) return -1;
    std::lock_guard<std::mutex> lk(f->mu);
    return f->est.count(ticket) ? (int)(ticket % f->members.size()) : -1;
}

int svo_fleet_stats(const svo_fleet *f, int member, svo_server_stats_t *out) {
    if (!f || !out) return fleet_fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    if (member < 0 || member >= (int)f->members.size()) return fleet_fail(SVO_ERR_INVALID_ARGUMENT, "no such member");
    return svo_server_stats(f->members[member].server, out);
}

void svo_fleet_destroy(svo_fleet *f) {
    if (!f) return;
    for (svo_fleet::Member &m : f->members) svo_server_destroy(m.server);
    delete f;
}

}  // extern "C"
