// Served form of the engine: a request loop with continuous batching.
//
// Requests (a system spec + a sweep count) are queued by scmf_server_submit.
// Three threads keep the GPU busy:
//   admission   takes queued requests in arrival order while their device
//               memory fits the HBM budget (and the slot limit), creates each
//               system on its own stream, initialises it there (random walks,
//               grid, field) and marks it ready; this runs beside the rounds.
//   rounds      at each round boundary adds the ready systems, drops the
//               finished and cancelled ones, rebuilds the batched plan if the
//               set changed, and runs a fixed number of sweeps over every
//               active system on the server stream (one move and one field
//               launch per sweep for all of them).  A system stops at its own
//               sweep count inside the round: its SysDev stop_step makes the
//               kernels skip its tiles, so rounds are not cut short by the
//               request with the fewest sweeps left.
//   completion  reads finished systems back (energies, accepts, counts) on
//               their own streams and frees them while the next round runs.
// Systems stay resident between rounds; requests that arrive while others run
// join at the next round boundary.  No reference counterpart: the reference
// runs one system per process.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_set>
#include <vector>

#include "scmf_engine.h"

using namespace scmf;

namespace {

struct Request {
    uint64_t id = 0;
    scmf_spec spec;
    int n_sweeps = 0;
    uint32_t* counts_out = nullptr;
    double t_submit = 0;
    size_t bytes = 0;
};

struct Active {
    Request req;
    scmf_system* sys = nullptr;
    int remaining = 0;
    double t_admit = 0;
    scmf_status status = SCMF_OK;  // status to report when it reaches completion
};

}  // namespace

struct scmf_server {
    scmf_server_opts opts{};
    int device = 0;
    std::mutex mu;
    std::condition_variable cv_work;   // admission: queue changed or stop
    std::condition_variable cv_ready;  // rounds: a system is ready or stop
    std::condition_variable cv_fin;    // completion: a system finished or stop
    std::condition_variable cv_done;   // clients: a result was delivered
    std::deque<Request> queue;
    std::deque<Active> ready;          // initialised, waiting for the next round boundary
    std::deque<Active> finishing;      // handed to the completion thread
    std::deque<scmf_result> done;
    std::unordered_set<uint64_t> running;    // admitted and not yet delivered
    std::unordered_set<uint64_t> cancelled;  // running ids to drop
    uint64_t next_id = 1;
    size_t bytes_in_use = 0;
    int n_active = 0;  // systems in the current rounds (mirror for other threads)
    bool stop = false, admission_done = false, rounds_done = false;
    std::thread admitter, worker, completer;
    cudaStream_t stream = nullptr;  // the rounds' stream
    std::chrono::steady_clock::time_point t0;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    void admit_loop();
    void round_loop();
    void complete_loop();
    void hand_over(Active&& a) {
        std::lock_guard<std::mutex> g(mu);
        finishing.push_back(std::move(a));
        cv_fin.notify_all();
    }
};

// Reads a finished system back into its result and frees it (completion thread).
static void finish(scmf_server* s, Active& a) {
    scmf_result r{};
    r.id = a.req.id;
    r.status = a.status;
    r.n_sweeps = a.req.n_sweeps;
    r.sweeps_done = a.req.n_sweeps - std::max(0, a.remaining);
    r.n_beads = a.sys ? a.sys->n_beads : 0;
    r.t_submit = a.req.t_submit;
    r.t_admit = a.t_admit;
    if (a.sys && a.status == SCMF_OK) {
        scmf_stats stats{};
        scmf_status rc = scmf_get_stats(a.sys, &stats);
        if (!rc && a.req.counts_out)
            rc = scmf_get_counts(a.sys, a.req.counts_out, (size_t)a.sys->n_cells * a.sys->spec.n_types);
        r.status = rc;
        r.e_bond = stats.e_bond;
        r.e_field = stats.e_field;
        r.accepts = stats.total_accepts;
    }
    if (a.sys) scmf_system_destroy(a.sys);
    a.sys = nullptr;
    r.t_done = s->now();
    std::lock_guard<std::mutex> g(s->mu);
    s->bytes_in_use -= std::min(s->bytes_in_use, a.req.bytes);
    s->running.erase(r.id);
    s->cancelled.erase(r.id);
    s->done.push_back(r);
    s->cv_done.notify_all();
}

void scmf_server::admit_loop() {
    cudaSetDevice(device);
    for (;;) {
        Request r;
        {
            std::unique_lock<std::mutex> lk(mu);
            for (;;) {
                if (stop) {  // shutting down: queued requests are dropped
                    queue.clear();
                    admission_done = true;
                    cv_ready.notify_all();
                    return;
                }
                if (!queue.empty()) {
                    const Request& q = queue.front();
                    const bool slot = opts.max_active <= 0 || (int)running.size() < opts.max_active;
                    if (slot && bytes_in_use + q.bytes <= opts.hbm_budget_bytes) break;
                }
                // wait for a submission, a freed slot or memory, or shutdown
                cv_work.wait_for(lk, std::chrono::milliseconds(50));
            }
            r = std::move(queue.front());
            queue.pop_front();
            bytes_in_use += r.bytes;
            running.insert(r.id);
        }
        Active a;
        a.req = std::move(r);
        a.remaining = a.req.n_sweeps;
        a.t_admit = now();
        // a private stream: creation and initialisation overlap the rounds
        scmf_status rc = scmf_system_create(&a.req.spec, nullptr, &a.sys);
        if (!rc) rc = scmf_init_coords(a.sys);
        if (!rc) rc = set_stop_step(a.sys, (uint32_t)a.req.n_sweeps);
        bool drop;
        {
            std::lock_guard<std::mutex> g(mu);
            drop = cancelled.count(a.req.id) > 0;
        }
        if (rc || drop || a.remaining == 0) {
            a.status = rc ? rc : (drop ? SCMF_E_CANCELLED : SCMF_OK);
            hand_over(std::move(a));
            continue;
        }
        std::lock_guard<std::mutex> g(mu);
        ready.push_back(std::move(a));
        cv_ready.notify_all();
    }
}

void scmf_server::round_loop() {
    cudaSetDevice(device);
    DevPlan plan;
    bool plan_valid = false;
    const int per_round = opts.sweeps_per_round > 0 ? opts.sweeps_per_round : 25;
    scmf_tune tune = default_tune();
    tune.use_graph = opts.use_graph;
    tune.beads_per_tile = 4096;  // the active systems fill the GPU together: full-size tiles for all
    std::vector<Active> active;
    for (;;) {
        // round boundary: take ready systems, drop cancelled ones
        std::vector<uint64_t> drop;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (active.empty() && ready.empty()) {
                if (admission_done) break;
                cv_ready.wait_for(lk, std::chrono::milliseconds(50));
            }
            while (!ready.empty()) {
                active.push_back(std::move(ready.front()));
                ready.pop_front();
                plan_valid = false;
            }
            for (auto& a : active)
                if (stop || cancelled.count(a.req.id)) drop.push_back(a.req.id);
        }
        if (!drop.empty()) {
            std::vector<Active> keep;
            for (auto& a : active) {
                if (std::find(drop.begin(), drop.end(), a.req.id) != drop.end()) {
                    a.status = SCMF_E_CANCELLED;
                    hand_over(std::move(a));
                } else {
                    keep.push_back(std::move(a));
                }
            }
            active.swap(keep);
            plan_valid = false;
        }
        {
            std::lock_guard<std::mutex> g(mu);
            n_active = (int)active.size();
        }
        if (active.empty()) continue;
        int round = 0;
        for (auto& a : active) round = std::max(round, std::min(per_round, a.remaining));
        scmf_status rc = SCMF_OK;
        if (!plan_valid) {
            Plan p;
            for (auto& a : active) a.sys->append_plan(tune, &p);
            rc = plan.upload(p, tune, stream);
            plan_valid = rc == SCMF_OK;
        }
        if (!rc) rc = plan.run_sweeps(stream, round);
        if (!rc && cudaStreamSynchronize(stream) != cudaSuccess) rc = fail(SCMF_E_CUDA, "round failed");
        std::vector<Active> keep;
        for (auto& a : active) {
            a.remaining = std::max(0, a.remaining - round);
            if (rc || a.remaining == 0) {
                a.status = rc;
                hand_over(std::move(a));
                plan_valid = false;
            } else {
                keep.push_back(std::move(a));
            }
        }
        active.swap(keep);
    }
    plan.release();
    std::lock_guard<std::mutex> g(mu);
    n_active = 0;
    rounds_done = true;
    cv_fin.notify_all();
}

void scmf_server::complete_loop() {
    cudaSetDevice(device);
    for (;;) {
        Active a;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_fin.wait(lk, [this] { return !finishing.empty() || (rounds_done && admission_done); });
            if (finishing.empty()) return;
            a = std::move(finishing.front());
            finishing.pop_front();
        }
        finish(this, a);
        std::lock_guard<std::mutex> g(mu);
        cv_work.notify_all();  // memory and a slot came free
    }
}

extern "C" {

scmf_status scmf_server_create(const scmf_server_opts* opts, scmf_server** out) {
    if (!opts || !out) return fail(SCMF_E_INVALID, "NULL argument");
    if (opts->hbm_budget_bytes == 0) return fail(SCMF_E_INVALID, "hbm_budget_bytes must be > 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return fail(SCMF_E_CUDA, "no CUDA device available");
    }
    scmf_server* s = new scmf_server;
    s->opts = *opts;
    s->t0 = std::chrono::steady_clock::now();
    cudaGetDevice(&s->device);
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete s;
        return fail(SCMF_E_CUDA, "cudaStreamCreate failed");
    }
    s->admitter = std::thread([s] { s->admit_loop(); });
    s->worker = std::thread([s] { s->round_loop(); });
    s->completer = std::thread([s] { s->complete_loop(); });
    *out = s;
    return SCMF_OK;
}

scmf_status scmf_server_submit(scmf_server* s, const scmf_spec* spec, int32_t n_sweeps, uint32_t* counts_out,
                               uint64_t* id_out) {
    if (!s || !spec || n_sweeps < 0) return fail(SCMF_E_INVALID, "bad arguments");
    scmf_status rc = validate_spec(*spec);
    if (rc) return rc;
    Request r;
    r.spec = *spec;
    r.n_sweeps = n_sweeps;
    r.counts_out = counts_out;
    r.bytes = system_device_bytes(*spec);
    if (r.bytes > s->opts.hbm_budget_bytes)
        return fail(SCMF_E_NOMEM, "request needs %zu bytes, budget is %llu", r.bytes,
                    (unsigned long long)s->opts.hbm_budget_bytes);
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stop) return fail(SCMF_E_STATE, "server is shutting down");
    r.id = s->next_id++;
    r.t_submit = s->now();
    if (id_out) *id_out = r.id;
    s->queue.push_back(std::move(r));
    s->cv_work.notify_all();
    return SCMF_OK;
}

scmf_status scmf_server_poll(scmf_server* s, scmf_result* out, int32_t max, int32_t* n_out, int32_t wait_ms) {
    if (!s || !n_out || max < 0 || (max > 0 && !out)) return fail(SCMF_E_INVALID, "bad arguments");
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && wait_ms > 0)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [s] { return !s->done.empty(); });
    int n = 0;
    while (n < max && !s->done.empty()) {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    *n_out = n;
    return SCMF_OK;
}

scmf_status scmf_server_pending(scmf_server* s, int32_t* queued, int32_t* active, uint64_t* bytes) {
    if (!s) return fail(SCMF_E_INVALID, "NULL server");
    std::lock_guard<std::mutex> g(s->mu);
    if (queued) *queued = (int32_t)s->queue.size();
    if (active) *active = (int32_t)s->n_active;
    if (bytes) *bytes = s->bytes_in_use;
    return SCMF_OK;
}

scmf_status scmf_server_cancel(scmf_server* s, uint64_t id) {
    if (!s) return fail(SCMF_E_INVALID, "NULL server");
    std::lock_guard<std::mutex> g(s->mu);
    for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
        if (it->id != id) continue;
        scmf_result r{};
        r.id = id;
        r.status = SCMF_E_CANCELLED;
        r.n_sweeps = it->n_sweeps;
        r.t_submit = it->t_submit;
        r.t_done = s->now();
        s->queue.erase(it);
        s->done.push_back(r);
        s->cv_done.notify_all();
        return SCMF_OK;
    }
    if (s->running.count(id)) {
        s->cancelled.insert(id);
        return SCMF_OK;
    }
    return fail(SCMF_E_INVALID, "no queued or running request %llu", (unsigned long long)id);
}

scmf_status scmf_server_drain(scmf_server* s, int32_t timeout_ms) {
    if (!s || timeout_ms < 0) return fail(SCMF_E_INVALID, "bad arguments");
    std::unique_lock<std::mutex> lk(s->mu);
    const bool idle = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                          [s] { return s->queue.empty() && s->running.empty(); });
    if (!idle)
        return fail(SCMF_E_TIMEOUT, "%zu queued and %zu running requests after %d ms", s->queue.size(),
                    s->running.size(), (int)timeout_ms);
    return SCMF_OK;
}

double scmf_server_now(const scmf_server* s) { return s ? s->now() : 0.0; }

void scmf_server_destroy(scmf_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
        s->cv_ready.notify_all();
        s->cv_fin.notify_all();
    }
    if (s->admitter.joinable()) s->admitter.join();
    if (s->worker.joinable()) s->worker.join();
    if (s->completer.joinable()) s->completer.join();
    cudaStreamDestroy(s->stream);
    delete s;
}

}  // extern "C"
