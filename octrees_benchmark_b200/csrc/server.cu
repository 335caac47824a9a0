// Serving scheduler (oct_server_* in include/octree_b200.h): continuous
// batching of radius and kNN requests over device-resident clouds.
//
// No reference counterpart: the reference answers queries inside its own
// benchmark loop (neighbor_benchmarks.hpp:502-568) and has no server.
//
// A server owns `slots` batched engines, each on its own stream.  Clients
// submit requests from any thread.  One scheduler thread loops over three
// steps: (1) batches whose stream has drained are completed - every request of
// the batch gets its completion record and stays readable in its slot until
// the client releases it; (2) slots whose requests are all released become
// free; (3) each free slot takes queued requests - first those queued longer
// than max_wait_ms, in arrival order, then the others smallest estimated work
// first (OCT_SERVER_FIFO: arrival order only) - while the batch stays within
// the request and centre limits and while the registered clouds, the admitted
// batches and this batch fit the HBM budget.  A request that does not fit
// waits for batches to finish (one admission stall per request), unless
// nothing is running, in which case it is admitted alone.
// Batches on different slots overlap on the device.  The budget counts each
// cloud's device bytes and, per admitted request, its engine arrays (44 B per
// centre, 12 B per kNN slot) and an estimate of its radius results (pi r^2
// times the cloud's points per m^2 of its box, with margin).
//
// OCT_SERVER_PLAIN runs one request per launch instead, first come first
// served, through the single-cloud path with the plain search configuration
// (the baseline the batched server is compared with).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cloud.h"

using namespace octb;
using Clock = std::chrono::steady_clock;

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr size_t kAdmitWindow = 4096;  // queued requests considered per admission

struct CloudEntry {
    uint64_t bytes = 0;
    bool owned = false;
    uint32_t refs = 0;      // queued and running requests on the cloud
    uint64_t last_use = 0;  // logical time of its last request
    double density = 0.0;   // points per m^2 of the box's xy extent
};

struct Ticket {
    oct_request req{};
    uint64_t id = 0;
    int slot = -1;
    oct_request_place place{};
    int status = OCT_OK;
    bool done = false;
    bool launched = false;
    uint64_t est = 0;
    Clock::time_point t_submit, t_launch, t_done;
};

enum SlotState { kFree = 0, kRunning = 1, kDone = 2 };

struct Slot {
    oct_engine eng = nullptr;
    SlotState state = kFree;
    std::vector<uint64_t> tickets;  // the batch's tickets, in batch order
    uint32_t outstanding = 0;       // tickets not yet released
    uint64_t est = 0;               // admission bytes of the running batch
    // plain mode: the one request's results
    DevBuf offs, idx, kidx, kd2, kcnt;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct oct_server_s {
    oct_server_params p{};
    bool plain = false;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv_work;  // the scheduler: new requests, releases
    std::condition_variable cv_done;  // clients: completions, clouds going idle
    std::deque<uint64_t> queue;       // queued ticket ids, arrival order
    std::unordered_map<uint64_t, Ticket> tickets;
    std::deque<oct_completion> done;
    std::unordered_map<oct_cloud, CloudEntry> clouds;
    uint64_t next_ticket = 1, clock = 0;
    uint64_t cloud_bytes = 0, inflight = 0;
    oct_server_stats st{};
    bool stop = false;
    bool fifo = false;
    bool head_stalled = false;
    std::thread worker;
    std::string last_error;
};

namespace {

int fail_s(oct_server s, int status, const std::string& msg) {
    s->last_error = msg;
    return status;
}

void note_peak(oct_server s) {
    s->st.peak_bytes = std::max<uint64_t>(s->st.peak_bytes, s->cloud_bytes + s->inflight);
}

// Lock held.
void complete_ticket(oct_server s, Ticket& t, int status) {
    t.done = true;
    t.status = status;
    t.t_done = Clock::now();
    oct_completion c{};
    c.ticket = t.id;
    c.status = status;
    c.type = t.req.type;
    c.nq = t.req.nq;
    c.n_results = t.place.n_results;
    c.queue_ms = ms_between(t.t_submit, t.launched ? t.t_launch : t.t_done);
    c.latency_ms = ms_between(t.t_submit, t.t_done);
    s->done.push_back(c);
    auto it = s->clouds.find(t.req.cloud);
    if (it != s->clouds.end() && it->second.refs) --it->second.refs;
    ++s->st.completed;
}

uint64_t estimate(oct_server s, const oct_request& r) {
    uint64_t b = 44ull * r.nq;
    if (r.type == OCT_REQ_KNN) {
        b += 12ull * r.k * r.nq;
    } else {
        const auto it = s->clouds.find(r.cloud);
        const double dens = it != s->clouds.end() ? it->second.density : 0.0;
        const double rr = r.radius > 0.0 ? r.radius : 1.0;
        const double per = 1.3 * kPi * rr * rr * dens + 16.0;
        b += (uint64_t)(4.0 * per * (double)r.nq);
    }
    return b;
}

// One request through the single-cloud path (plain mode).  Lock not held.
int run_plain(Slot& sl, Ticket& t) {
    const oct_request& r = t.req;
    oct_cloud h = r.cloud;
    const uint64_t nq = r.nq;
    cudaError_t e;
    t.place.q_begin = 0;
    t.place.out_begin = 0;
    t.place.nq = nq;
    t.place.n_results = 0;
    if (nq == 0) return OCT_OK;
    if (r.type == OCT_REQ_RADIUS) {
        if ((e = sl.offs.reserve(8 * (nq + 1))) != cudaSuccess) return OCT_ERR_OUT_OF_MEMORY;
        if (sl.idx.bytes < 4096 && (e = sl.idx.reserve(4 << 20)) != cudaSuccess) return OCT_ERR_OUT_OF_MEMORY;
        uint64_t total = 0;
        int st = oct_radius_search(h, r.kernel, r.algo, r.centers, nq, r.radii, r.radius, sl.offs.as<uint64_t>(),
                                   sl.idx.as<uint32_t>(), sl.idx.bytes / 4, &total, OCT_MEM_DEVICE);
        if (st == OCT_ERR_CAPACITY) {
            if ((e = sl.idx.reserve(4 * (total + total / 4 + 1024))) != cudaSuccess) return OCT_ERR_OUT_OF_MEMORY;
            st = oct_radius_search(h, r.kernel, r.algo, r.centers, nq, r.radii, r.radius, sl.offs.as<uint64_t>(),
                                   sl.idx.as<uint32_t>(), sl.idx.bytes / 4, &total, OCT_MEM_DEVICE);
        }
        if (st != OCT_OK) return st;
        t.place.n_results = total;
    } else {
        if ((e = sl.kidx.reserve(4ull * nq * r.k)) != cudaSuccess) return OCT_ERR_OUT_OF_MEMORY;
        if ((e = sl.kd2.reserve(8ull * nq * r.k)) != cudaSuccess) return OCT_ERR_OUT_OF_MEMORY;
        if ((e = sl.kcnt.reserve(4ull * nq)) != cudaSuccess) return OCT_ERR_OUT_OF_MEMORY;
        const int st = oct_knn(h, r.centers, nq, r.k, sl.kidx.as<uint32_t>(), sl.kd2.as<double>(),
                               sl.kcnt.as<uint32_t>(), OCT_MEM_DEVICE);
        if (st != OCT_OK) return st;
    }
    return oct_synchronize(h);
}

void worker_plain(oct_server s) {
    Slot& sl = s->slots[0];
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        if (sl.state == kDone && sl.outstanding == 0) {
            sl.state = kFree;
            sl.tickets.clear();
        }
        if (sl.state != kFree || s->queue.empty()) {
            s->cv_work.wait_for(lk, std::chrono::milliseconds(2));
            continue;
        }
        const uint64_t id = s->queue.front();
        s->queue.pop_front();
        Ticket& t = s->tickets[id];
        t.slot = 0;
        t.launched = true;
        t.t_launch = Clock::now();
        sl.tickets.assign(1, id);
        sl.outstanding = 1;
        sl.state = kRunning;
        ++s->st.batches;
        lk.unlock();
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev != s->p.device) cudaSetDevice(s->p.device);
        const int st = run_plain(sl, t);  // the ticket stays put: only its release erases it
        lk.lock();
        complete_ticket(s, t, st);
        sl.state = kDone;
        s->cv_done.notify_all();
    }
}

struct Cand {
    uint32_t cls;  // 0: waited longer than max_wait_ms, 1: the others
    uint64_t key;  // arrival position (class 0) or estimated work (class 1)
    uint32_t pos;  // position in the queue
};

void worker_batched(oct_server s) {
    std::vector<oct_request> reqs;
    std::vector<uint64_t> ids;
    std::vector<oct_request_place> places;
    std::vector<Cand> cand;
    std::vector<uint8_t> taken;
    cudaSetDevice(s->p.device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        bool progress = false;
        // (1) batches whose stream has drained (engine calls run without the lock: a
        // running slot is touched by this thread only)
        for (size_t i = 0; i < s->slots.size(); ++i) {
            Slot& sl = s->slots[i];
            if (sl.state != kRunning) continue;
            lk.unlock();
            int ready = 0;
            const int rs = oct_engine_ready(sl.eng, &ready);
            int st = rs;
            double wait_ms = 0.0;
            if (rs == OCT_OK && ready) {
                places.assign(sl.tickets.size(), oct_request_place{});
                const Clock::time_point w0 = Clock::now();
                st = oct_engine_wait(sl.eng, places.data(), nullptr);
                wait_ms = ms_between(w0, Clock::now());
            }
            lk.lock();
            s->st.max_finish_ms = std::max(s->st.max_finish_ms, wait_ms);
            if (rs == OCT_OK && !ready) continue;
            for (size_t j = 0; j < sl.tickets.size(); ++j) {
                Ticket& t = s->tickets[sl.tickets[j]];
                if (st == OCT_OK) t.place = places[j];
                complete_ticket(s, t, st);
            }
            s->inflight -= sl.est;
            sl.est = 0;
            sl.state = kDone;
            progress = true;
            s->cv_done.notify_all();
        }
        // (2) slots whose requests are all released
        for (Slot& sl : s->slots) {
            if (sl.state == kDone && sl.outstanding == 0) {
                sl.state = kFree;
                sl.tickets.clear();
            }
        }
        // (3) admission into free slots.  Candidates (the first kAdmitWindow queued requests) in order:
        // those queued longer than max_wait_ms in arrival order, then the rest smallest estimated work
        // first (FIFO mode: arrival order only), so that small requests do not wait behind large ones
        // and no request waits for ever.
        for (size_t i = 0; i < s->slots.size() && !s->queue.empty(); ++i) {
            Slot& sl = s->slots[i];
            if (sl.state != kFree) continue;
            reqs.clear();
            ids.clear();
            cand.clear();
            const Clock::time_point now = Clock::now();
            const size_t window = std::min<size_t>(s->queue.size(), kAdmitWindow);
            for (size_t pos = 0; pos < window; ++pos) {
                const Ticket& t = s->tickets[s->queue[pos]];
                const bool aged = s->fifo || ms_between(t.t_submit, now) > s->p.max_wait_ms;
                cand.push_back({aged ? 0u : 1u, aged ? (uint64_t)pos : t.est, (uint32_t)pos});
            }
            std::sort(cand.begin(), cand.end(), [](const Cand& a, const Cand& b) {
                return a.cls != b.cls ? a.cls < b.cls : (a.key != b.key ? a.key < b.key : a.pos < b.pos);
            });
            taken.assign(window, 0);
            uint64_t q = 0, est = 0;
            for (size_t ci = 0; ci < cand.size() && reqs.size() < s->p.max_batch_requests; ++ci) {
                Ticket& t = s->tickets[s->queue[cand[ci].pos]];
                if (!reqs.empty() && q + t.req.nq > s->p.max_batch_queries) {
                    if (s->fifo) break;
                    continue;  // a smaller one may still fit
                }
                const bool fits = s->cloud_bytes + s->inflight + est + t.est <= s->p.hbm_budget;
                const bool alone = reqs.empty() && s->inflight == 0;  // nothing to wait for: admit it alone
                if (!fits && !alone) {
                    if (reqs.empty() && !s->head_stalled) {
                        ++s->st.admission_stalls;
                        s->head_stalled = true;
                    }
                    break;
                }
                s->head_stalled = false;
                reqs.push_back(t.req);
                ids.push_back(t.id);
                q += t.req.nq;
                est += t.est;
                taken[cand[ci].pos] = 1;
                if (!fits) break;
            }
            if (reqs.empty()) break;
            {  // drop the admitted requests from the queue, keeping the others in arrival order
                std::deque<uint64_t> rest;
                for (size_t pos = 0; pos < s->queue.size(); ++pos)
                    if (pos >= window || !taken[pos]) rest.push_back(s->queue[pos]);
                s->queue.swap(rest);
            }
            sl.tickets = ids;
            sl.outstanding = (uint32_t)ids.size();
            sl.state = kRunning;  // claimed: clients do not touch it while the lock is dropped
            lk.unlock();
            const Clock::time_point s0 = Clock::now();
            const int st = oct_engine_submit(sl.eng, reqs.data(), (uint32_t)reqs.size(), nullptr);
            const double submit_ms = ms_between(s0, Clock::now());
            lk.lock();
            s->st.max_submit_ms = std::max(s->st.max_submit_ms, submit_ms);
            const Clock::time_point launched = Clock::now();
            for (uint64_t id : ids) {
                Ticket& t = s->tickets[id];
                t.slot = (int)i;
                t.launched = true;
                t.t_launch = launched;
            }
            if (st != OCT_OK) {
                char buf[512] = {0};
                oct_engine_last_error(sl.eng, buf, sizeof(buf));
                s->last_error = buf;
                for (uint64_t id : ids) complete_ticket(s, s->tickets[id], st);
                sl.state = kDone;
                s->cv_done.notify_all();
            } else {
                sl.state = kRunning;
                sl.est = est;
                s->inflight += est;
                note_peak(s);
                ++s->st.batches;
            }
            progress = true;
        }
        if (!progress) {
            bool running = false;
            for (const Slot& sl : s->slots) running = running || sl.state == kRunning;
            if (running) s->cv_work.wait_for(lk, std::chrono::microseconds(50));
            else s->cv_work.wait_for(lk, std::chrono::milliseconds(2));
        }
    }
}

}  // namespace

extern "C" {

int oct_server_create(const oct_server_params* p, oct_server* out) {
    if (!p || !out) return OCT_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return OCT_ERR_NO_DEVICE;
    }
    if (p->device < 0 || p->device >= ndev) return OCT_ERR_INVALID_ARG;
    oct_server s = new (std::nothrow) oct_server_s();
    if (!s) return OCT_ERR_OUT_OF_MEMORY;
    s->p = *p;
    s->plain = (p->flags & OCT_SERVER_PLAIN) != 0;
    s->fifo = (p->flags & OCT_SERVER_FIFO) != 0;
    if (s->p.slots == 0) s->p.slots = 3;
    if (s->plain) s->p.slots = 1;
    if (s->p.max_batch_requests == 0) s->p.max_batch_requests = 1024;
    if (s->p.max_batch_queries == 0) s->p.max_batch_queries = 512ull << 10;
    if (!(s->p.max_wait_ms > 0.0)) s->p.max_wait_ms = 40.0;
    if (s->p.hbm_budget == 0) s->p.hbm_budget = 120ull << 30;
    s->slots.resize(s->p.slots);
    if (!s->plain) {
        for (Slot& sl : s->slots) {
            oct_engine_params ep{};
            ep.device = p->device;
            if (p->flags & OCT_SERVER_NO_GRAPH) ep.flags |= OCT_ENGINE_NO_GRAPH;
            // results of a full batch at ~1024 neighbours per centre (2 GB per slot at 512K centres): batches
            // rarely outgrow it, and one that does is run again on the scheduler thread
            ep.reserve_results = std::max<uint64_t>(64ull << 20, 1024ull * s->p.max_batch_queries);
            ep.reserve_queries = s->p.max_batch_queries;  // the per-centre arrays of the largest batch
            const int st = oct_engine_create(&ep, &sl.eng);
            if (st != OCT_OK) {
                oct_server_destroy(s);
                return st;
            }
        }
    }
    s->worker = std::thread(s->plain ? worker_plain : worker_batched, s);
    *out = s;
    return OCT_OK;
}

int oct_server_destroy(oct_server s) {
    if (!s) return OCT_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    if (s->worker.joinable()) s->worker.join();
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(s->p.device);
    for (Slot& sl : s->slots) {
        if (sl.eng) {
            if (sl.state == kRunning) oct_engine_wait(sl.eng, nullptr, nullptr);
            oct_engine_destroy(sl.eng);
        }
        DevBuf* bufs[] = {&sl.offs, &sl.idx, &sl.kidx, &sl.kd2, &sl.kcnt};
        for (DevBuf* b : bufs) b->release();
    }
    for (auto& kv : s->clouds)
        if (kv.second.owned) oct_cloud_destroy(kv.first);
    if (prev >= 0) cudaSetDevice(prev);
    delete s;
    return OCT_OK;
}

int oct_server_last_error(oct_server s, char* buf, size_t len) {
    if (!s || !buf || len == 0) return OCT_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    const size_t k = std::min(len - 1, s->last_error.size());
    memcpy(buf, s->last_error.data(), k);
    buf[k] = '\0';
    return OCT_OK;
}

int oct_server_set_config(oct_server s, const oct_search_config* cfg) {
    if (!s || !cfg) return OCT_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    for (Slot& sl : s->slots)
        if (sl.state != kFree) return fail_s(s, OCT_ERR_STATE, "configuration change while batches are running");
    for (Slot& sl : s->slots) {
        if (!sl.eng) continue;
        const int st = oct_engine_set_config(sl.eng, cfg);
        if (st != OCT_OK) return fail_s(s, st, "engine rejected the configuration");
    }
    return OCT_OK;
}

int oct_server_add_cloud(oct_server s, oct_cloud h, uint32_t flags) {
    if (!s || !h) return OCT_ERR_INVALID_ARG;
    const Cloud& c = h->c;
    if (!c.built) return fail_s(s, OCT_ERR_STATE, "cloud is not built");
    if (c.device != s->p.device) return fail_s(s, OCT_ERR_INVALID_ARG, "cloud on another device");
    uint64_t bytes = 0;
    oct_cloud_memory(h, &bytes);
    std::vector<oct_cloud> evict;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->clouds.count(h)) return fail_s(s, OCT_ERR_INVALID_ARG, "cloud already registered");
        // evict idle owned clouds, least recently used first, until the new one fits
        while (s->cloud_bytes + s->inflight + bytes > s->p.hbm_budget) {
            oct_cloud victim = nullptr;
            uint64_t best = UINT64_MAX;
            for (auto& kv : s->clouds) {
                if (kv.second.owned && kv.second.refs == 0 && kv.second.last_use < best) {
                    best = kv.second.last_use;
                    victim = kv.first;
                }
            }
            if (!victim) return fail_s(s, OCT_ERR_OUT_OF_MEMORY, "cloud does not fit the HBM budget");
            s->cloud_bytes -= s->clouds[victim].bytes;
            s->clouds.erase(victim);
            ++s->st.evictions;
            evict.push_back(victim);
        }
        CloudEntry ce;
        ce.bytes = bytes;
        ce.owned = (flags & OCT_CLOUD_OWNED) != 0;
        ce.last_use = ++s->clock;
        const double area = 4.0 * c.box.radii[0] * c.box.radii[1];
        ce.density = area > 0.0 ? (double)c.n / area : 0.0;
        s->clouds[h] = ce;
        s->cloud_bytes += bytes;
        note_peak(s);
    }
    for (oct_cloud v : evict) oct_cloud_destroy(v);
    if (s->plain) {  // the baseline searches with the plain configuration
        oct_search_config cfg{};
        cfg.packet = 0;
        cfg.radius_lanes = 8;
        cfg.knn_bucket = 256;
        oct_set_search_config(h, &cfg);
    }
    return OCT_OK;
}

int oct_server_remove_cloud(oct_server s, oct_cloud h) {
    if (!s || !h) return OCT_ERR_INVALID_ARG;
    bool owned = false;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->clouds.find(h);
        if (it == s->clouds.end()) return fail_s(s, OCT_ERR_STATE, "cloud is not registered");
        s->cv_done.wait(lk, [&] { return s->stop || s->clouds[h].refs == 0; });
        it = s->clouds.find(h);
        owned = it->second.owned;
        s->cloud_bytes -= it->second.bytes;
        s->clouds.erase(it);
    }
    if (owned) oct_cloud_destroy(h);
    return OCT_OK;
}

int oct_server_submit(oct_server s, const oct_request* r, uint64_t* ticket) {
    if (!s || !r || !ticket) return OCT_ERR_INVALID_ARG;
    if (r->nq && !r->centers) return fail_s(s, OCT_ERR_INVALID_ARG, "centers is NULL");
    if (r->type == OCT_REQ_KNN && (r->k < 1 || r->k > 1024))
        return fail_s(s, OCT_ERR_INVALID_ARG, "kNN takes 1 <= k <= 1024");
    if (r->type == OCT_REQ_RADIUS &&
        ((r->kernel < OCT_KERNEL_CIRCLE || r->kernel > OCT_KERNEL_CUBE) ||
         (r->algo != OCT_NEIGHBORS && r->algo != OCT_NEIGHBORS_PRUNE)))
        return fail_s(s, OCT_ERR_INVALID_ARG, "bad kernel or algo");
    if (r->type != OCT_REQ_RADIUS && r->type != OCT_REQ_KNN) return fail_s(s, OCT_ERR_INVALID_ARG, "bad type");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->clouds.find(r->cloud);
        if (it == s->clouds.end()) return fail_s(s, OCT_ERR_STATE, "cloud is not registered (or was evicted)");
        ++it->second.refs;
        it->second.last_use = ++s->clock;
        const uint64_t id = s->next_ticket++;
        Ticket& t = s->tickets[id];
        t.req = *r;
        t.id = id;
        t.place.nq = r->nq;
        t.t_submit = Clock::now();
        t.est = estimate(s, *r);
        s->queue.push_back(id);
        ++s->st.submitted;
        s->st.queries += r->nq;
        *ticket = id;
    }
    s->cv_work.notify_one();
    return OCT_OK;
}

int oct_server_poll(oct_server s, oct_completion* out, uint32_t max, uint32_t* n, int32_t wait_ms) {
    if (!s || !n || (max && !out)) return OCT_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && wait_ms > 0)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return s->stop || !s->done.empty(); });
    uint32_t k = 0;
    while (k < max && !s->done.empty()) {
        out[k++] = s->done.front();
        s->done.pop_front();
    }
    *n = k;
    return OCT_OK;
}

int oct_server_copy_radius(oct_server s, uint64_t ticket, uint64_t* offsets, uint32_t* idx, uint64_t cap,
                           uint32_t flags) {
    if (!s) return OCT_ERR_INVALID_ARG;
    Slot* sl = nullptr;
    oct_request_place pl{};
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end() || !it->second.done || it->second.slot < 0)
            return fail_s(s, OCT_ERR_STATE, "no completed request with this ticket");
        if (it->second.req.type != OCT_REQ_RADIUS) return fail_s(s, OCT_ERR_INVALID_ARG, "not a radius request");
        if (it->second.status != OCT_OK) return it->second.status;
        sl = &s->slots[it->second.slot];
        pl = it->second.place;
    }
    cudaSetDevice(s->p.device);
    if (!s->plain) return oct_engine_copy_radius(sl->eng, &pl, offsets, idx, cap, flags);
    const cudaMemcpyKind kind = (flags & OCT_MEM_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (offsets && cudaMemcpy(offsets, sl->offs.ptr, 8 * (pl.nq + 1), kind) != cudaSuccess) return OCT_ERR_CUDA;
    if (idx && pl.n_results > cap) return fail_s(s, OCT_ERR_CAPACITY, "idx_capacity smaller than the results");
    if (idx && pl.n_results && cudaMemcpy(idx, sl->idx.ptr, 4 * pl.n_results, kind) != cudaSuccess)
        return OCT_ERR_CUDA;
    return OCT_OK;
}

int oct_server_copy_knn(oct_server s, uint64_t ticket, uint32_t* idx, double* d2, uint32_t* counts, uint32_t flags) {
    if (!s) return OCT_ERR_INVALID_ARG;
    Slot* sl = nullptr;
    oct_request_place pl{};
    uint32_t k = 0;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end() || !it->second.done || it->second.slot < 0)
            return fail_s(s, OCT_ERR_STATE, "no completed request with this ticket");
        if (it->second.req.type != OCT_REQ_KNN) return fail_s(s, OCT_ERR_INVALID_ARG, "not a kNN request");
        if (it->second.status != OCT_OK) return it->second.status;
        sl = &s->slots[it->second.slot];
        pl = it->second.place;
        k = it->second.req.k;
    }
    cudaSetDevice(s->p.device);
    if (!s->plain) return oct_engine_copy_knn(sl->eng, &pl, k, idx, d2, counts, flags);
    const cudaMemcpyKind kind = (flags & OCT_MEM_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    const uint64_t slots = pl.nq * k;
    if (idx && slots && cudaMemcpy(idx, sl->kidx.ptr, 4 * slots, kind) != cudaSuccess) return OCT_ERR_CUDA;
    if (d2 && slots && cudaMemcpy(d2, sl->kd2.ptr, 8 * slots, kind) != cudaSuccess) return OCT_ERR_CUDA;
    if (counts && pl.nq && cudaMemcpy(counts, sl->kcnt.ptr, 4 * pl.nq, kind) != cudaSuccess) return OCT_ERR_CUDA;
    return OCT_OK;
}

int oct_server_release(oct_server s, uint64_t ticket) {
    if (!s) return OCT_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end() || !it->second.done)
            return fail_s(s, OCT_ERR_STATE, "no completed request with this ticket");
        const int slot = it->second.slot;
        if (slot >= 0 && s->slots[slot].outstanding) --s->slots[slot].outstanding;
        s->tickets.erase(it);
    }
    s->cv_work.notify_one();
    return OCT_OK;
}

int oct_server_get_stats(oct_server s, oct_server_stats* out) {
    if (!s || !out) return OCT_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    out->cloud_bytes = s->cloud_bytes;
    out->inflight_bytes = s->inflight;
    out->queued = (uint32_t)s->queue.size();
    uint32_t running = 0;
    for (const Slot& sl : s->slots) running += sl.state == kRunning;
    out->in_flight = running;
    return OCT_OK;
}

}  // extern "C"
