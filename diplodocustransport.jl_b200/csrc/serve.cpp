// Serving loop: continuous batching of solve requests over batched (DTB_MIXED) contexts.
//
// Each registered grid is one batched context with its own stream, and each grid progresses
// on its own: a library-owned host thread polls the grids and, for every grid whose previous
// chunk has finished (an event on its stream), (1) reads back the f of every slot whose steps
// are done and frees the slot, (2) admits queued requests into free slots, (3) launches the
// next chunk of batched steps if the grid has running slots. Grids never wait for one another:
// a small grid's requests are admitted and finished at its own chunk boundaries while a large
// grid's chunk is still on the device. Requests that arrive meanwhile join at their grid's next
// admission point, so work of different requests and grids overlaps on the device. Device
// memory of all grids (operators and every slot's state, allocated with the grid's context) is
// checked against an HBM budget when a grid is registered.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "ctx.h"

// batch_api.cpp internals
int batch_launch(dtb_ctx* c, int64_t nsteps);
int batch_finish(dtb_ctx* c);
int batch_capacity(dtb_ctx* c);
long long batch_step(dtb_ctx* c);

namespace {

using clk = std::chrono::steady_clock;

struct Request {
    int64_t id = 0;
    int grid = 0;
    std::vector<double> f;  // f0 on submission, the result when done
    double dt_scale = 1.0;
    int64_t n_steps = 0;
    int state = 0;          // 0 queued, 1 running, 2 done, 3 failed, 4 cancelled
    bool cancel = false;    // cancellation asked while running: the slot is freed at its grid's next chunk boundary
    int slot = -1;
    double t_submit = 0, t_admit = 0, t_done = 0;
    double cr_max = 0;
    int finite = 1;
};

struct Grid {
    dtb_ctx* ctx = nullptr;
    int capacity = 0;
    // slot tables, written by the loop thread only (under the lock when they change)
    std::vector<int64_t> slot_req;     // request id per slot, -1 when free
    std::vector<long long> slot_stop;  // device step at which the slot's request is done
    std::deque<int64_t> queue;         // guarded by the server lock
    cudaEvent_t done_ev = nullptr;     // recorded after the grid's chunk in flight
    bool in_flight = false;
    double t_launch = 0;
    int64_t chunk = 0;
    double ema_step_ms = 0.1;
    int n_running = 0;
    int n_cancel = 0;                  // running requests cancelled since the last pass (server lock)
};

}  // namespace

struct dtb_server {
    dtb_serve_opts opts{};
    std::vector<Grid> grids;
    std::map<int64_t, Request> req;  // guarded by mu; done requests are erased when collected
    int64_t next_id = 1;
    int64_t bytes = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread th;
    bool running = false, stop = false;
    int error = DTB_OK;
    std::string error_msg;
    clk::time_point t0 = clk::now();
    // statistics
    int64_t steps_done = 0;      // instance-steps completed
    int64_t batched_steps = 0;   // batched steps launched, summed over grids
    int64_t completed = 0;
    double busy_s = 0;
    std::vector<double> tts;     // time to solution of every completed request (DTB_PROFILE summary)

    double now() const { return std::chrono::duration<double>(clk::now() - t0).count(); }
};

namespace {

void fail(dtb_server* s, int rc) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->error = rc;
    s->error_msg = dtb_last_error();
    s->stop = true;
    for (auto& kv : s->req)
        if (kv.second.state < 2) kv.second.state = 3;
    s->cv_done.notify_all();
}

// Reads back and frees every slot of `g` whose request is done at the grid's current step, and
// frees the slots of running requests that were cancelled.
int complete_slots(dtb_server* s, Grid& g) {
    const long long st = batch_step(g.ctx);
    bool any = false;
    for (int sl = 0; sl < g.capacity; ++sl) {
        const int64_t id = g.slot_req[(size_t)sl];
        if (id < 0) continue;
        Request* r;
        bool cancelled;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r = &s->req.at(id);  // not erased before it is done
            cancelled = r->cancel;
        }
        if (cancelled) {
            int rc = dtb_batch_release(g.ctx, sl);
            if (rc != DTB_OK) return rc;
            std::lock_guard<std::mutex> lk(s->mu);
            r->state = 4;
            r->t_done = s->now();
            g.slot_req[(size_t)sl] = -1;
            g.n_running--;
            any = true;
            continue;
        }
        if (st < g.slot_stop[(size_t)sl]) continue;
        int64_t done = 0, left = 0;
        double cr = 0;
        int32_t fin = 1;
        int rc = dtb_batch_get_f(g.ctx, sl, r->f.data());
        if (rc == DTB_OK) rc = dtb_batch_slot_info(g.ctx, sl, &done, &left, &cr, &fin);
        if (rc == DTB_OK) rc = dtb_batch_release(g.ctx, sl);
        if (rc != DTB_OK) return rc;
        std::lock_guard<std::mutex> lk(s->mu);
        r->cr_max = cr;
        r->finite = fin;
        r->t_done = s->now();
        r->state = 2;
        g.slot_req[(size_t)sl] = -1;
        g.n_running--;
        s->steps_done += r->n_steps;
        s->completed++;
        s->tts.push_back(r->t_done - r->t_submit);
        any = true;
    }
    if (any) s->cv_done.notify_all();
    return DTB_OK;
}

// Admits queued requests of `g` into its free slots (the grid has no chunk in flight).
int admit_slots(dtb_server* s, Grid& g) {
    std::vector<std::pair<int, Request*>> a;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (int sl = 0; sl < g.capacity && !g.queue.empty(); ++sl) {
            if (g.slot_req[(size_t)sl] >= 0) continue;
            const int64_t id = g.queue.front();
            g.queue.pop_front();
            Request& r = s->req.at(id);
            r.slot = sl;
            r.state = 1;
            g.slot_req[(size_t)sl] = id;
            g.n_running++;
            a.push_back({sl, &r});
        }
    }
    // uploads outside the lock: a running request is neither erased nor written by others, and
    // its f0 and dt are fixed at submission
    for (auto& sr : a) {
        Request& r = *sr.second;
        const long long stop = batch_step(g.ctx) + r.n_steps;
        int rc = dtb_batch_admit(g.ctx, sr.first, r.f.data(), r.dt_scale, r.n_steps);
        if (rc != DTB_OK) return rc;
        g.slot_stop[(size_t)sr.first] = stop;
        std::lock_guard<std::mutex> lk(s->mu);
        r.t_admit = s->now();
    }
    return DTB_OK;
}

// Launches the next chunk of `g`: up to the earliest finishing request, capped at the target
// device time per chunk so that arrivals are admitted promptly.
int launch_chunk(dtb_server* s, Grid& g, int max_chunk, double target_ms) {
    const long long st = batch_step(g.ctx);
    long long left = (long long)1 << 60;
    for (int sl = 0; sl < g.capacity; ++sl)
        if (g.slot_req[(size_t)sl] >= 0) left = std::min(left, g.slot_stop[(size_t)sl] - st);
    const int cap = std::max(1, std::min(max_chunk, (int)(target_ms / std::max(1e-3, g.ema_step_ms))));
    g.chunk = std::max<long long>(1, std::min<long long>(left, cap));
    DTB_TRY(batch_launch(g.ctx, g.chunk));
    {
        DeviceGuard dg(g.ctx->device);
        DTB_CUDA(cudaEventRecord(g.done_ev, g.ctx->stream));
    }
    g.in_flight = true;
    g.t_launch = s->now();
    std::lock_guard<std::mutex> lk(s->mu);
    s->batched_steps += g.chunk;
    return DTB_OK;
}

void loop(dtb_server* s) {
    const int max_chunk = s->opts.max_chunk_steps > 0 ? s->opts.max_chunk_steps : 256;
    const double target_ms = s->opts.chunk_ms > 0 ? s->opts.chunk_ms : 20.0;
    double t_prev = s->now();
    bool busy_prev = false;
    while (true) {
        {
            std::unique_lock<std::mutex> lk(s->mu);
            bool any = false;
            for (auto& g : s->grids) any = any || g.in_flight || g.n_running > 0 || !g.queue.empty();
            if (!any && !s->stop) s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
            if (s->stop) return;
        }
        bool progressed = false;
        for (auto& g : s->grids) {
            if (g.in_flight) {
                cudaError_t q;
                {
                    DeviceGuard dg(g.ctx->device);
                    q = cudaEventQuery(g.done_ev);
                }
                if (q == cudaErrorNotReady) continue;
                g.in_flight = false;
                int rc = batch_finish(g.ctx);  // the chunk is done: reads its error flag
                if (rc != DTB_OK) return fail(s, rc);
                // device time per batched step of this grid (an upper bound while grids overlap)
                g.ema_step_ms = 0.7 * g.ema_step_ms + 0.3 * (1e3 * (s->now() - g.t_launch) / (double)g.chunk);
                rc = complete_slots(s, g);
                if (rc != DTB_OK) return fail(s, rc);
                progressed = true;
            }
            bool queued, cancels;
            {
                std::lock_guard<std::mutex> lk(s->mu);
                queued = !g.queue.empty();
                cancels = g.n_cancel > 0;
                g.n_cancel = 0;
            }
            if (cancels) {  // running requests of this grid were cancelled: free their slots now
                int rc = complete_slots(s, g);
                if (rc != DTB_OK) return fail(s, rc);
            }
            if (queued && g.n_running < g.capacity) {
                int rc = admit_slots(s, g);
                if (rc != DTB_OK) return fail(s, rc);
            }
            if (g.n_running > 0) {
                int rc = launch_chunk(s, g, max_chunk, target_ms);
                if (rc != DTB_OK) return fail(s, rc);
                progressed = true;
            }
        }
        // busy time: intervals during which some grid had a chunk on the device
        bool busy = false;
        for (auto& g : s->grids) busy = busy || g.in_flight;
        const double t = s->now();
        if (busy_prev) {
            std::lock_guard<std::mutex> lk(s->mu);
            s->busy_s += t - t_prev;
        }
        t_prev = t;
        busy_prev = busy;
        // nothing finished: give the device a moment before polling the events again
        if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

}  // namespace

extern "C" {

int32_t dtb_serve_create(const dtb_serve_opts* opts, dtb_server** out) {
    DTB_CHECK(out, DTB_EINVAL, "dtb_serve_create: null output");
    auto* s = new dtb_server();
    if (opts) s->opts = *opts;
    *out = s;
    return DTB_OK;
}

int32_t dtb_serve_add_grid(dtb_server* s, dtb_ctx* ctx, int32_t* grid_id) {
    DTB_CHECK(s && ctx && grid_id, DTB_EINVAL, "dtb_serve_add_grid: null argument");
    DTB_CHECK(!s->running, DTB_ESTATE, "dtb_serve_add_grid: register grids before dtb_serve_start");
    DTB_CHECK(ctx->prec == DTB_MIXED, DTB_EINVAL, "dtb_serve_add_grid: the context must be batched (DTB_MIXED)");
    DTB_TRY(dtb_commit(ctx));
    int64_t b = 0;
    DTB_TRY(dtb_device_bytes(ctx, &b));
    if (s->opts.hbm_budget_bytes > 0 && s->bytes + b > s->opts.hbm_budget_bytes) {
        set_error("dtb_serve_add_grid: the grid needs " + std::to_string(b) + " device bytes; " +
                  std::to_string(s->opts.hbm_budget_bytes - s->bytes) + " of the HBM budget are left");
        return DTB_ENOMEM;
    }
    Grid g;
    g.ctx = ctx;
    g.capacity = batch_capacity(ctx);
    g.slot_req.assign((size_t)g.capacity, -1);
    g.slot_stop.assign((size_t)g.capacity, 0);
    {
        DeviceGuard dg(ctx->device);
        DTB_CUDA(cudaEventCreateWithFlags(&g.done_ev, cudaEventDisableTiming));
    }
    s->bytes += b;
    s->grids.push_back(std::move(g));
    *grid_id = (int32_t)s->grids.size() - 1;
    return DTB_OK;
}

int32_t dtb_serve_start(dtb_server* s) {
    DTB_CHECK(s, DTB_EINVAL, "dtb_serve_start: null server");
    DTB_CHECK(!s->running, DTB_ESTATE, "dtb_serve_start: already running");
    DTB_CHECK(!s->grids.empty(), DTB_ESTATE, "dtb_serve_start: no grid registered");
    s->t0 = clk::now();
    s->running = true;
    s->th = std::thread(loop, s);
    return DTB_OK;
}

int32_t dtb_serve_submit(dtb_server* s, int32_t grid_id, const double* f0, double dt_scale, int64_t n_steps,
                         int64_t* request_id) {
    DTB_CHECK(s && f0 && request_id, DTB_EINVAL, "dtb_serve_submit: null argument");
    DTB_CHECK(grid_id >= 0 && grid_id < (int32_t)s->grids.size(), DTB_ENOTFOUND, "dtb_serve_submit: unknown grid");
    DTB_CHECK(n_steps >= 1 && std::isfinite(dt_scale), DTB_EINVAL, "dtb_serve_submit: bad step count or dt");
    Grid& g = s->grids[(size_t)grid_id];
    const int64_t n = g.ctx->n_mom;
    std::lock_guard<std::mutex> lk(s->mu);
    DTB_CHECK(s->error == DTB_OK, s->error, "dtb_serve_submit: the server stopped after an error: " + s->error_msg);
    Request r;
    r.id = s->next_id++;
    r.grid = grid_id;
    r.f.assign(f0, f0 + n);
    r.dt_scale = dt_scale;
    r.n_steps = n_steps;
    r.t_submit = s->now();
    *request_id = r.id;
    g.queue.push_back(r.id);
    s->req.emplace(r.id, std::move(r));
    s->cv_work.notify_all();
    return DTB_OK;
}

int32_t dtb_serve_wait(dtb_server* s, int64_t request_id, double timeout_s, double* f_out, dtb_request_stats* st) {
    DTB_CHECK(s, DTB_EINVAL, "dtb_serve_wait: null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->req.find(request_id);
    DTB_CHECK(it != s->req.end(), DTB_ENOTFOUND, "dtb_serve_wait: unknown request");
    const auto deadline = clk::now() + std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9);
    while (it->second.state < 2) {
        if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && it->second.state < 2) {
            set_error("dtb_serve_wait: request " + std::to_string(request_id) + " not done within the timeout");
            return DTB_ETIMEOUT;
        }
    }
    Request& r = it->second;
    if (r.state == 4) {
        s->req.erase(it);
        set_error("dtb_serve_wait: request " + std::to_string(request_id) + " was cancelled");
        return DTB_ESTATE;
    }
    if (r.state == 3) {
        set_error("dtb_serve_wait: the server stopped after an error: " + s->error_msg);
        return s->error != DTB_OK ? s->error : DTB_ECUDA;
    }
    if (f_out) std::copy(r.f.begin(), r.f.end(), f_out);
    if (st) {
        st->t_submit = r.t_submit;
        st->t_admit = r.t_admit;
        st->t_done = r.t_done;
        st->steps = r.n_steps;
        st->cr_max = r.cr_max;
        st->finite = r.finite;
        st->grid = r.grid;
    }
    s->req.erase(it);  // collected: the id is unknown from now on
    return DTB_OK;
}

int32_t dtb_serve_cancel(dtb_server* s, int64_t request_id) {
    DTB_CHECK(s, DTB_EINVAL, "dtb_serve_cancel: null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->req.find(request_id);
    DTB_CHECK(it != s->req.end(), DTB_ENOTFOUND, "dtb_serve_cancel: unknown request");
    Request& r = it->second;
    if (r.state == 0) {  // queued: leaves the queue at once
        auto& q = s->grids[(size_t)r.grid].queue;
        q.erase(std::remove(q.begin(), q.end(), request_id), q.end());
        r.state = 4;
        r.t_done = s->now();
        s->cv_done.notify_all();
    } else if (r.state == 1 && !r.cancel) {  // running: its slot is freed at the grid's next chunk boundary
        r.cancel = true;
        s->grids[(size_t)r.grid].n_cancel++;
        s->cv_work.notify_all();
    }
    return DTB_OK;  // a request already done or failed is left as it is
}

int32_t dtb_serve_get_stats(dtb_server* s, dtb_serve_stats* st) {
    DTB_CHECK(s && st, DTB_EINVAL, "dtb_serve_get_stats: null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    st->completed = s->completed;
    st->instance_steps = s->steps_done;
    st->batched_steps = s->batched_steps;
    st->busy_s = s->busy_s;
    st->elapsed_s = s->now();
    int64_t q = 0, r = 0;
    for (auto& g : s->grids) {
        q += (int64_t)g.queue.size();
        r += g.n_running;
    }
    st->queued = q;
    st->running = r;
    st->device_bytes = s->bytes;
    return s->error;
}

int32_t dtb_serve_destroy(dtb_server* s) {
    if (!s) return DTB_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    if (s->th.joinable()) s->th.join();
    if (const char* path = profile_path()) {
        // one JSON line per server: requests served, instance-steps/s, busy time, p50/p99 time to solution
        std::vector<double> t = s->tts;
        std::sort(t.begin(), t.end());
        auto pct = [&](double q) { return t.empty() ? 0.0 : t[(size_t)std::min<double>(t.size() - 1, q * (t.size() - 1) + 0.5)]; };
        const double el = s->now();
        char b[512];
        std::snprintf(b, sizeof(b),
                      "{\"server\": 1, \"grids\": %zu, \"completed\": %lld, \"instance_steps\": %lld, "
                      "\"elapsed_s\": %.6g, \"busy_s\": %.6g, \"instance_steps_per_s\": %.6g, \"tts_p50_s\": %.6g, "
                      "\"tts_p99_s\": %.6g, \"device_bytes\": %lld}\n",
                      s->grids.size(), (long long)s->completed, (long long)s->steps_done, el, s->busy_s,
                      el > 0 ? (double)s->steps_done / el : 0.0, pct(0.5), pct(0.99), (long long)s->bytes);
        if (FILE* f = std::fopen(path, "a")) {
            std::fputs(b, f);
            std::fclose(f);
        }
    }
    for (auto& g : s->grids) {
        if (!g.done_ev) continue;
        DeviceGuard dg(g.ctx->device);
        if (g.in_flight) cudaEventSynchronize(g.done_ev);  // the caller may destroy the context next
        cudaEventDestroy(g.done_ev);
    }
    delete s;
    return DTB_OK;
}

}  // extern "C"
