// psb_server.cu -- a solve server with continuous batching (no counterpart in
// the reference, which solves one puzzle per call).
//
// Clients submit solve requests (puzzle, start state) from any thread without
// blocking.  Requests with more than large_states states go to the large
// lane: a second thread runs them one at a time as single two-bit searches
// (one reusable psb_bfs session per puzzle size, on its own stream), so a
// large search never sets the pace of the small ones.  The batch lane's
// server thread owns a psb_engine and loops:
//   1. admit queued requests while an instance slot and pool space for the
//      request's two-bit array are free (admission by HBM footprint: 2 bits x
//      states, padded).  The smallest requests go first; a request that does
//      not fit now waits without holding back the others, until it has been
//      passed over kMaxBypass times: then nothing else is admitted until it
//      fits, which the running searches guarantee as they finish.  A request
//      larger than the whole pool completes at once with PSB_ERR_NOMEM;
//   2. advance every resident search by one BFS level (psb_engine_step), so
//      requests that arrive while others are running overlap on the GPU;
//   3. collect finished searches: per-depth counts, eccentricity (the last
//      depth) and latency from submission to completion.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <tuple>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/psb200.h"
#include "psb_internal.h"

namespace {
using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket;
    int kind, a, b;
    uint64_t initial;
    Clock::time_point submitted;
    uint64_t footprint;   // engine pool bytes (0 if the puzzle is invalid: admission reports why)
    uint32_t bypassed;    // times a later request was admitted while this one did not fit
    uint64_t states;      // IndexesCount() (0 if the puzzle is invalid)
};

// A request passed over this many times stops later admissions until it fits.
constexpr uint32_t kMaxBypass = 64;

struct Done {
    uint64_t ticket;
    int status;  // PSB_OK or the admission/engine error
    std::vector<uint64_t> counts;
    double latency;
};
}  // namespace

struct psb_server {
    psb_engine* engine = nullptr;
    uint32_t max_depths = 0;
    uint32_t levels_per_step = 1;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request> queue;
    std::vector<Done> done;
    std::unordered_map<uint64_t, Request> running;
    std::atomic<bool> stop{false};
    std::atomic<uint64_t> next_ticket{1};
    // Large lane.
    uint64_t large_states = 0;
    std::deque<Request> large_queue;
    std::condition_variable large_cv;
    std::thread large_worker;
    uint32_t large_running = 0;
    int fatal = PSB_OK;
    std::string fatal_msg;
    uint64_t admitted = 0, completed = 0, steps = 0;
};

namespace {

// Admits queued requests, smallest footprint first (ties: oldest first), while
// the engine has a slot and pool space.  Called with s->mu held.
void admit_queued(psb_server* s) {
    std::vector<size_t> order(s->queue.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t x, size_t y) { return s->queue[x].footprint < s->queue[y].footprint; });
    // The oldest request that has been passed over too often goes first, alone.
    for (size_t i = 0; i < s->queue.size(); i++) {
        if (s->queue[i].bypassed >= kMaxBypass) {
            order.assign(1, i);
            break;
        }
    }
    std::vector<bool> gone(s->queue.size(), false);
    std::vector<size_t> waiting;  // did not fit this time
    for (size_t i : order) {
        Request& r = s->queue[i];
        uint32_t slot = 0;
        const int rc = psb_engine_add(s->engine, r.kind, r.a, r.b, r.initial, r.ticket, &slot);
        if (rc == PSB_ERR_CAPACITY) {  // no slot or pool space now: wait for running searches to finish
            waiting.push_back(i);
            continue;
        }
        gone[i] = true;
        if (rc != PSB_OK) {  // unsupported puzzle, bad start, larger than the pool: report at once
            s->done.push_back(Done{r.ticket, rc, {}, 0.0});
            continue;
        }
        s->running.emplace(r.ticket, r);
        s->admitted++;
        for (size_t w : waiting)  // admitted ahead of requests that were submitted earlier
            if (s->queue[w].ticket < r.ticket) s->queue[w].bypassed++;
    }
    std::deque<Request> rest;
    for (size_t i = 0; i < s->queue.size(); i++)
        if (!gone[i]) rest.push_back(s->queue[i]);
    s->queue.swap(rest);
}

void serve(psb_server* s) {
    std::vector<uint64_t> tags(1024), counts;
    std::vector<uint32_t> nd(1024);
    counts.resize(size_t(1024) * s->max_depths);
    for (;;) {
        std::vector<Request> admit;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            if (s->running.empty())
                s->cv.wait(lock, [&] { return s->stop.load() || !s->queue.empty(); });
            if (s->stop.load()) return;
            admit_queued(s);
            if (s->running.empty() && !s->queue.empty()) {
                // Nothing runs and nothing was admitted: only possible while the
                // engine is still releasing space.  Wait briefly instead of spinning.
                s->cv.wait_for(lock, std::chrono::milliseconds(1));
                continue;
            }
        }
        if (!s->running.empty()) {
            // Several levels per step while nothing waits for admission (fewer
            // host round trips); one level while requests wait, so they are
            // admitted as soon as a finished search frees its space.
            uint32_t levels = s->levels_per_step;
            {
                std::lock_guard<std::mutex> lock(s->mu);
                if (!s->queue.empty()) levels = 1;
            }
            int rc = psb_engine_step(s->engine, levels);
            uint32_t n = 0;
            if (rc == PSB_OK) rc = psb_engine_poll(s->engine, tags.data(), nd.data(), counts.data(), 1024, &n);
            const auto now = Clock::now();
            std::lock_guard<std::mutex> lock(s->mu);
            s->steps++;
            if (rc != PSB_OK) {
                char buf[512];
                psb_last_error(buf, sizeof buf);
                s->fatal = rc;
                s->fatal_msg = buf;
                for (auto& kv : s->running) s->done.push_back(Done{kv.first, rc, {}, 0.0});
                s->running.clear();
                s->stop = true;
                return;
            }
            for (uint32_t i = 0; i < n; i++) {
                auto it = s->running.find(tags[i]);
                if (it == s->running.end()) continue;
                const double lat = std::chrono::duration<double>(now - it->second.submitted).count();
                const uint64_t* row = counts.data() + size_t(i) * s->max_depths;
                s->done.push_back(Done{tags[i], PSB_OK, std::vector<uint64_t>(row, row + nd[i]), lat});
                s->running.erase(it);
                s->completed++;
            }
        }
    }
}

// The large lane: one request at a time, first come first served, each as a
// single two-bit search on this thread's stream.  Sessions are kept per
// puzzle size, so a size's arrays are allocated once.
void serve_large(psb_server* s) {
    struct Sess {
        psb_puzzle* puzzle = nullptr;
        psb_bfs_session* session = nullptr;
    };
    std::map<std::tuple<int, int, int>, Sess> sessions;
    cudaStream_t stream = nullptr;
    cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    std::vector<uint64_t> counts(s->max_depths);
    for (;;) {
        Request r;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            s->large_cv.wait(lock, [&] { return s->stop.load() || !s->large_queue.empty(); });
            if (s->stop.load()) break;
            r = s->large_queue.front();
            s->large_queue.pop_front();
            s->large_running = 1;
        }
        psb_bfs_opts o{};
        o.struct_size = sizeof(psb_bfs_opts);
        o.device = -1;
        o.stream = stream;
        int rc = PSB_OK;
        Sess& x = sessions[std::make_tuple(r.kind, r.a, r.b)];
        if (!x.puzzle) rc = psb_puzzle_create(r.kind, r.a, r.b, &x.puzzle);
        if (rc == PSB_OK && !x.session) rc = psb_bfs_session_create(x.puzzle, PSB_TWO_BIT, &o, &x.session);
        uint32_t nd = 0;
        if (rc == PSB_OK) rc = psb_bfs_session_run(x.session, r.initial, &o, counts.data(), s->max_depths, &nd, nullptr);
        const double lat = std::chrono::duration<double>(Clock::now() - r.submitted).count();
        std::lock_guard<std::mutex> lock(s->mu);
        if (rc == PSB_OK) {
            s->done.push_back(Done{r.ticket, PSB_OK, std::vector<uint64_t>(counts.begin(), counts.begin() + nd), lat});
            s->completed++;
        } else {
            s->done.push_back(Done{r.ticket, rc, {}, 0.0});
        }
        s->large_running = 0;
    }
    for (auto& kv : sessions) {
        if (kv.second.session) psb_bfs_session_destroy(kv.second.session);
        if (kv.second.puzzle) psb_puzzle_destroy(kv.second.puzzle);
    }
    cudaStreamSynchronize(stream);
    cudaStreamDestroy(stream);
}

}  // namespace

extern "C" {

int psb_server_start(const psb_server_opts* opts, psb_server** out) {
    if (!opts || !out || opts->struct_size != sizeof(psb_server_opts)) return psb_set_error(PSB_ERR_ARG, "bad options");
    auto* s = new psb_server();
    if (int rc = psb_engine_create(&opts->engine, &s->engine)) { delete s; return rc; }
    s->max_depths = opts->engine.max_depths;
    s->levels_per_step = opts->levels_per_step ? opts->levels_per_step : 1;
    s->large_states = opts->large_states ? opts->large_states : (uint64_t(1) << 26);
    int device = -1;
    cudaGetDevice(&device);
    s->worker = std::thread([s, device] {
        cudaSetDevice(device);
        serve(s);
    });
    s->large_worker = std::thread([s, device] {
        cudaSetDevice(device);
        serve_large(s);
    });
    *out = s;
    return PSB_OK;
}

int psb_server_submit(psb_server* s, int kind, int a, int b, uint64_t initial, uint64_t* ticket) {
    if (!s || !ticket) return psb_set_error(PSB_ERR_ARG, "bad argument");
    uint64_t footprint = 0, states = 0;
    if (psb_engine_footprint(kind, a, b, &footprint) != PSB_OK) footprint = 0;
    psb_puzzle* p = nullptr;
    if (psb_puzzle_create(kind, a, b, &p) == PSB_OK) {
        int ops = 0, br = 0, odd = 0;
        psb_puzzle_info(p, &states, &ops, &br, &odd);
        psb_puzzle_destroy(p);
    }
    Request r{s->next_ticket.fetch_add(1), kind, a, b, initial, Clock::now(), footprint, 0, states};
    const bool large = states > s->large_states;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->stop.load()) return psb_set_error(s->fatal ? s->fatal : PSB_ERR_ARG, "server stopped");
        (large ? s->large_queue : s->queue).push_back(r);
    }
    (large ? s->large_cv : s->cv).notify_one();
    *ticket = r.ticket;
    return PSB_OK;
}

int psb_server_poll(psb_server* s, uint64_t* tickets, int* status, uint32_t* n_depths, uint64_t* counts,
                    double* latency_s, uint32_t cap, uint32_t* n) {
    if (!s || !n || (cap && (!tickets || !status || !n_depths || !counts || !latency_s)))
        return psb_set_error(PSB_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> lock(s->mu);
    const uint32_t k = uint32_t(std::min<size_t>(cap, s->done.size()));
    for (uint32_t i = 0; i < k; i++) {
        const Done& d = s->done[i];
        tickets[i] = d.ticket;
        status[i] = d.status;
        n_depths[i] = uint32_t(d.counts.size());
        latency_s[i] = d.latency;
        std::memset(counts + size_t(i) * s->max_depths, 0, 8ull * s->max_depths);
        std::memcpy(counts + size_t(i) * s->max_depths, d.counts.data(), 8 * d.counts.size());
    }
    s->done.erase(s->done.begin(), s->done.begin() + k);
    *n = k;
    return PSB_OK;
}

int psb_server_info(psb_server* s, uint32_t* queued, uint32_t* running, uint64_t* completed, uint64_t* steps) {
    if (!s) return psb_set_error(PSB_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> lock(s->mu);
    if (queued) *queued = uint32_t(s->queue.size() + s->large_queue.size());
    if (running) *running = uint32_t(s->running.size()) + s->large_running;
    if (completed) *completed = s->completed;
    if (steps) *steps = s->steps;
    return s->fatal;
}

int psb_server_stop(psb_server* s) {
    if (!s) return PSB_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    s->large_cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    if (s->large_worker.joinable()) s->large_worker.join();
    psb_engine_destroy(s->engine);
    delete s;
    return PSB_OK;
}

}  // extern "C"
