// Serving loop: continuous batching of independent MPO solves on one GPU.
//
// Requests (an operator, chain options, a number of levels) are queued in
// arrival order.  A pool of worker threads, each with its own library
// context (CUDA stream and device arena), takes the request at the head of
// the queue as soon as a worker is free and the request's estimated device
// footprint (nc_chain_footprint_bytes) fits in the memory budget next to the
// requests already running; requests that arrive while others run are
// therefore admitted as slots and memory free up, and their kernels overlap
// on the device.  Each request builds its chain, keeps its MPS and
// environments resident on the device for all of its sweeps, solves its
// levels at its bond dimension (nc_chain_solve_levels_at_bandwidth) and
// frees everything (stream-ordered, so other requests are not stalled).
// A request's result depends only on its own inputs (its seed fixes the
// initial state and every kernel's reduction order is fixed), so it is the
// same alone and in the mix.
//
// There is no counterpart in the reference (which solves one chain per
// process); the C interface it mirrors for one request is
// Nutcracker_Operator_simpleSolveForLeastEigenvalues (operator.cpp:23-36).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "nc_abi_util.h"
#include "nc_common.cuh"
#include "nutcracker_b200.h"

using nc::g_status;

namespace {

using Clock = std::chrono::steady_clock;

double seconds(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

struct Request {
    int64_t id = 0;
    std::vector<std::vector<uint32_t>> idx;
    std::vector<std::vector<nc_complex>> W;
    std::vector<nc_operator_site> sites;
    nc_chain_options opt{};
    uint32_t levels = 1;
    uint64_t footprint = 0;
    Clock::time_point t_submit, t_start, t_done;
    bool done = false;
    nc_request_result res{};
};

}  // namespace

struct nc_server {
    int device = 0;
    uint32_t max_inflight = 1;
    uint64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::map<int64_t, std::unique_ptr<Request>> all;
    std::vector<std::thread> workers;
    uint64_t used = 0, peak = 0;
    uint32_t running = 0;
    int64_t next_id = 1;
    bool stop = false;
    bool any_submit = false;
    Clock::time_point first_submit, last_done;
    std::vector<double> latencies;
    uint64_t completed = 0, failed = 0, submitted = 0;

    void worker();
};

void nc_server::worker() {
    cudaSetDevice(device);
    // Many workers share the host's cores: their waits block instead of
    // spinning, so the threads that are launching work keep the cores.
    nc::Context::get().blocking_sync = true;
    for (;;) {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] {
                if (stop) return true;
                if (queue.empty()) return false;
                // admission of the head request by device footprint; with nothing
                // running, an oversized request still runs (alone)
                return used == 0 || used + queue.front()->footprint <= budget;
            });
            if (stop && queue.empty()) return;
            if (queue.empty()) continue;
            r = queue.front();
            queue.pop_front();
            used += r->footprint;
            peak = std::max(peak, used);
            ++running;
            r->t_start = Clock::now();
        }
        // run the request on this thread's context (its own stream and arena)
        int status = 0;
        std::string msg;
        nc_chain* ch = nc_chain_create((uint32_t)r->sites.size(), r->sites.data(), &r->opt);
        if (!ch) {
            status = nc_last_status() ? nc_last_status() : -1;
            msg = nc_last_error();
        } else {
            if (nc_chain_solve_levels_at_bandwidth(ch, r->levels, r->res.energies) != 0) {
                status = nc_last_status();
                msg = nc_last_error();
            } else {
                nc_chain_info info;
                if (nc_chain_get_info(ch, &info) == 0) {
                    r->res.sweeps = info.sweeps;
                    r->res.bandwidth_dimension = info.bandwidth_dimension;
                }
            }
            nc_chain_free(ch);
        }
        // the request's copy of its operator is not needed once its chain is
        // gone; only the (small) result stays with the request id
        std::vector<std::vector<uint32_t>>().swap(r->idx);
        std::vector<std::vector<nc_complex>>().swap(r->W);
        std::vector<nc_operator_site>().swap(r->sites);
        {
            std::lock_guard<std::mutex> lk(mu);
            r->t_done = Clock::now();
            r->res.status = status;
            r->res.levels = r->levels;
            r->res.footprint_bytes = r->footprint;
            r->res.seconds_queued = seconds(r->t_submit, r->t_start);
            r->res.seconds_run = seconds(r->t_start, r->t_done);
            r->res.seconds_total = seconds(r->t_submit, r->t_done);
            std::snprintf(r->res.message, sizeof(r->res.message), "%s", msg.c_str());
            r->done = true;
            used -= r->footprint;
            --running;
            last_done = r->t_done;
            if (status == 0) {
                ++completed;
                latencies.push_back(r->res.seconds_total);
            } else {
                ++failed;
            }
        }
        cv_done.notify_all();
        cv_work.notify_all();
    }
}

extern "C" {

void nc_server_options_init(nc_server_options* o) {
    std::memset(o, 0, sizeof(*o));
    o->max_inflight = 16;
    o->memory_budget_bytes = 0;
}

nc_server* nc_server_create(const nc_server_options* options) {
    NC_ABI_BEGIN
    nc_server_options o;
    nc_server_options_init(&o);
    if (options) o = *options;
    NC_ARG(o.max_inflight >= 1 && o.max_inflight <= 256, "max_inflight must be in [1, 256]");
    auto s = std::make_unique<nc_server>();
    NC_CUDA(cudaGetDevice(&s->device));
    s->max_inflight = o.max_inflight;
    s->budget = o.memory_budget_bytes;
    if (s->budget == 0) {
        size_t free_b = 0, total_b = 0;
        NC_CUDA(cudaMemGetInfo(&free_b, &total_b));
        s->budget = (uint64_t)(0.8 * (double)free_b);
    }
    for (uint32_t i = 0; i < s->max_inflight; ++i) s->workers.emplace_back([p = s.get()] { p->worker(); });
    return s.release();
    NC_ABI_END
    return nullptr;
}

int64_t nc_server_submit(nc_server* s, uint32_t number_of_sites, const nc_operator_site* sites,
                         const nc_chain_options* options, uint32_t levels) {
    NC_ABI_BEGIN
    NC_ARG(s && sites && number_of_sites >= 1 && levels >= 1 && levels <= NC_SERVER_MAX_LEVELS,
           "bad request (levels must be in [1, NC_SERVER_MAX_LEVELS])");
    auto r = std::make_unique<Request>();
    r->levels = levels;
    if (options) r->opt = *options;
    else nc_chain_options_init(&r->opt);
    r->idx.resize(number_of_sites);
    r->W.resize(number_of_sites);
    r->sites.resize(number_of_sites);
    for (uint32_t i = 0; i < number_of_sites; ++i) {
        const nc_operator_site& in = sites[i];
        const size_t nnz = in.number_of_matrices, dd = (size_t)in.physical_dimension * in.physical_dimension;
        r->idx[i].assign(in.indices, in.indices + 2 * nnz);
        r->W[i].assign(in.matrices, in.matrices + dd * nnz);
        r->sites[i] = in;
        r->sites[i].indices = r->idx[i].data();
        r->sites[i].matrices = r->W[i].data();
    }
    if (nc_chain_footprint_bytes(number_of_sites, r->sites.data(), &r->opt, levels, &r->footprint) != 0)
        throw nc::Error(nc_last_status(), nc_last_error());
    std::lock_guard<std::mutex> lk(s->mu);
    NC_ARG(!s->stop, "server is shutting down");
    r->id = s->next_id++;
    r->t_submit = Clock::now();
    if (!s->any_submit) {
        s->any_submit = true;
        s->first_submit = r->t_submit;
    }
    ++s->submitted;
    const int64_t id = r->id;
    s->queue.push_back(r.get());
    s->all[id] = std::move(r);
    s->cv_work.notify_one();
    return id;
    NC_ABI_END
    return -1;
}

int nc_server_poll(nc_server* s, int64_t id, nc_request_result* out) {
    NC_ABI_BEGIN
    NC_ARG(s, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    NC_ARG(it != s->all.end(), "unknown request id");
    if (!it->second->done) return 1;
    if (out) *out = it->second->res;
    NC_ABI_END
    return g_status;
}

int nc_server_wait(nc_server* s, int64_t id, nc_request_result* out) {
    NC_ABI_BEGIN
    NC_ARG(s, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    NC_ARG(it != s->all.end(), "unknown request id");
    Request* r = it->second.get();
    s->cv_done.wait(lk, [&] { return r->done; });
    if (out) *out = r->res;
    NC_ABI_END
    return g_status;
}

int nc_server_drain(nc_server* s) {
    NC_ABI_BEGIN
    NC_ARG(s, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] { return s->queue.empty() && s->running == 0; });
    NC_ABI_END
    return g_status;
}

int nc_server_get_stats(nc_server* s, nc_server_stats* out) {
    NC_ABI_BEGIN
    NC_ARG(s && out, "bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->failed = s->failed;
    out->in_flight = s->running;
    out->queued = s->queue.size();
    out->peak_bytes_in_flight = s->peak;
    out->memory_budget_bytes = s->budget;
    if (!s->latencies.empty()) {
        std::vector<double> l = s->latencies;
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) {
            const size_t k = (size_t)std::min<double>((double)l.size() - 1, std::ceil(q * l.size()) - 1);
            return l[k];
        };
        out->p50_seconds = pct(0.50);
        out->p99_seconds = pct(0.99);
        double sum = 0;
        for (double v : l) sum += v;
        out->mean_seconds = sum / l.size();
        out->window_seconds = seconds(s->first_submit, s->last_done);
        out->solves_per_second = out->window_seconds > 0 ? s->completed / out->window_seconds : 0;
    }
    NC_ABI_END
    return g_status;
}

void nc_server_free(nc_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    delete s;
}

}  // extern "C"
