// Serving replicas across GPUs: one request loop (pd_ctx) per device, and a
// router that sends each whole request to the replica with the least work
// still pending. Built on the public C ABI only.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "pd_plan.h"
#include "pd_tuning.h"
#include "pripps_debye.h"

namespace {

std::mutex g_router_err_mu;
std::string g_router_err;

int router_fail(int rc, const std::string &m) {
    std::lock_guard<std::mutex> g(g_router_err_mu);
    g_router_err = m;
    return rc;
}

constexpr int kReplicaShift = 56;  // router ticket = replica << 56 | context ticket

// Relative device time of a request: pair·q per frame, times the frames and
// the cost of its kernel form (FP64 sin per pair·q, two accumulators).
double request_work(const pd_request *req) {
    const double n = static_cast<double>(req->n_atoms);
    double w = n * (n - 1.0) / 2.0 * static_cast<double>(req->nq) *
               static_cast<double>(req->n_frames ? req->n_frames : 1);
    if (req->precision == PD_FP64) w *= 24.0;
    if (pd::request_mode(req, req->species, req->hyd_weights) == PD_MODE_WEIGHTED) w *= 1.5;
    return w;
}

}  // namespace

struct pd_router {
    std::vector<pd_ctx *> replicas;
    std::mutex mu;
    std::vector<double> pending;  // work submitted and not yet seen finished, per replica
    struct Entry {
        uint32_t replica;
        double work;
        bool settled;  // its work no longer counts as pending
    };
    std::map<uint64_t, Entry> tickets;

    // Polls the outstanding tickets so that finished work stops counting.
    void refresh_locked() {
        for (auto &kv : tickets) {
            Entry &e = kv.second;
            if (e.settled) continue;
            const uint64_t ct = kv.first & ((uint64_t{1} << kReplicaShift) - 1);
            if (pd_poll(replicas[e.replica], ct) != 0) settle_locked(e);
        }
    }
    void settle_locked(Entry &e) {
        if (e.settled) return;
        e.settled = true;
        pending[e.replica] = std::max(0.0, pending[e.replica] - e.work);
    }
};

extern "C" {

int pd_route_choose(const double *pending_work, uint32_t n, uint32_t *choice) {
    if (!pending_work || n == 0 || !choice) return PD_EINVAL;
    uint32_t best = 0;
    for (uint32_t i = 1; i < n; ++i)
        if (pending_work[i] < pending_work[best]) best = i;
    *choice = best;
    return PD_OK;
}

int pd_router_create(const int *devices, uint32_t n_devices, uint64_t mem_budget_bytes,
                     pd_router **out) {
    if (!devices || n_devices == 0 || n_devices > 64 || !out)
        return router_fail(PD_EINVAL, "pd_router_create: 1..64 devices are required");
    *out = nullptr;
    auto r = std::make_unique<pd_router>();
    for (uint32_t i = 0; i < n_devices; ++i) {
        pd_ctx *c = nullptr;
        const int rc = pd_ctx_create(devices[i], mem_budget_bytes, &c);
        if (rc != PD_OK) {
            const std::string m = pd_last_error(nullptr);
            for (pd_ctx *x : r->replicas) pd_ctx_destroy(x);
            return router_fail(rc, "pd_router_create: device " + std::to_string(devices[i]) +
                                       ": " + m);
        }
        r->replicas.push_back(c);
    }
    r->pending.assign(n_devices, 0.0);
    *out = r.release();
    return PD_OK;
}

void pd_router_destroy(pd_router *r) {
    if (!r) return;
    for (pd_ctx *c : r->replicas) pd_ctx_destroy(c);
    delete r;
}

int pd_router_submit(pd_router *r, const pd_request *req, uint64_t *ticket) {
    if (!r || !req || !ticket) return router_fail(PD_EINVAL, "pd_router_submit: bad arguments");
    std::string msg;
    int rc = pd::validate_request(req, false, msg);
    if (rc) return router_fail(rc, "pd_router_submit: " + msg);
    const double work = request_work(req);
    std::lock_guard<std::mutex> g(r->mu);
    r->refresh_locked();
    uint32_t k = 0;
    pd_route_choose(r->pending.data(), static_cast<uint32_t>(r->pending.size()), &k);
    uint64_t ct = 0;
    rc = pd_submit(r->replicas[k], req, &ct);
    if (rc) return router_fail(rc, std::string("pd_router_submit: ") + pd_last_error(r->replicas[k]));
    if (ct >> kReplicaShift) return router_fail(PD_ENOMEM, "pd_router_submit: ticket space exhausted");
    const uint64_t t = (static_cast<uint64_t>(k) << kReplicaShift) | ct;
    r->tickets[t] = pd_router::Entry{k, work, false};
    r->pending[k] += work;
    *ticket = t;
    return PD_OK;
}

int pd_router_wait(pd_router *r, uint64_t ticket, int timeout_ms, double *out_terms) {
    if (!r) return PD_EINVAL;
    pd_ctx *c = nullptr;
    {
        std::lock_guard<std::mutex> g(r->mu);
        auto it = r->tickets.find(ticket);
        if (it == r->tickets.end()) return router_fail(PD_ENOTFOUND, "pd_router_wait: unknown ticket");
        c = r->replicas[it->second.replica];
    }
    const uint64_t ct = ticket & ((uint64_t{1} << kReplicaShift) - 1);
    const int rc = pd_wait(c, ct, timeout_ms, out_terms);
    std::lock_guard<std::mutex> g(r->mu);
    auto it = r->tickets.find(ticket);
    if (rc != PD_ETIMEOUT || pd_poll(c, ct) != 0) {
        if (it != r->tickets.end()) r->settle_locked(it->second);
    }
    // a result handed out (or a final failure) ends the ticket on the router
    // too; a wait that only timed out keeps it
    if (it != r->tickets.end() && (rc == PD_OK || (rc != PD_ETIMEOUT && out_terms)))
        r->tickets.erase(it);
    if (rc != PD_OK) router_fail(rc, std::string("pd_router_wait: ") + pd_last_error(c));
    return rc;
}

int pd_router_poll(pd_router *r, uint64_t ticket) {
    if (!r) return PD_EINVAL;
    std::lock_guard<std::mutex> g(r->mu);
    auto it = r->tickets.find(ticket);
    if (it == r->tickets.end()) return PD_ENOTFOUND;
    const int p = pd_poll(r->replicas[it->second.replica],
                          ticket & ((uint64_t{1} << kReplicaShift) - 1));
    if (p != 0) r->settle_locked(it->second);
    return p;
}

int pd_router_cancel(pd_router *r, uint64_t ticket) {
    if (!r) return PD_EINVAL;
    std::lock_guard<std::mutex> g(r->mu);
    auto it = r->tickets.find(ticket);
    if (it == r->tickets.end()) return PD_ENOTFOUND;
    return pd_cancel(r->replicas[it->second.replica],
                     ticket & ((uint64_t{1} << kReplicaShift) - 1));
}

int pd_router_replica(pd_router *r, uint64_t ticket, uint32_t *replica, pd_ctx **ctx,
                      uint64_t *ctx_ticket) {
    if (!r) return PD_EINVAL;
    std::lock_guard<std::mutex> g(r->mu);
    auto it = r->tickets.find(ticket);
    if (it == r->tickets.end()) return PD_ENOTFOUND;
    if (replica) *replica = it->second.replica;
    if (ctx) *ctx = r->replicas[it->second.replica];
    if (ctx_ticket) *ctx_ticket = ticket & ((uint64_t{1} << kReplicaShift) - 1);
    return PD_OK;
}

const char *pd_router_last_error(void) {
    static thread_local std::string copy;
    std::lock_guard<std::mutex> g(g_router_err_mu);
    copy = g_router_err;
    return copy.c_str();
}

}  // extern "C"
