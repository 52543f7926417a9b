// serve.cpp -- continuous-batching job server over independent contexts.
//
// Every submitted job (its own mesh, options and iteration count) waits in a
// FIFO until its arrival time has passed, a slot is free and its estimated
// HBM footprint fits the budget; it is then admitted: a worker thread builds
// its context on a stream of its own and runs its design iterations back to
// back, so the kernels of all admitted jobs overlap on the device.  A job
// that finishes frees its slot and memory at once and the scheduler admits
// the next ones: no step barrier couples the jobs.  Each job's state
// (densities, displacements, filter warm start, MMA history) stays resident
// in its context from admission to completion.
//
// Instance batching (topo_server_set_batching): admitted jobs up to a size
// limit run their first design iteration on a thread of their own (it
// allocates and tunes their context) and then join one batch worker, which
// keeps every job it holds going: each job's iterations are replayed from its
// step graphs (conditional nodes decide the solver loops on the device) and
// relaunched as soon as they are done, with no host thread per job and no
// host round trip inside an iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "ctx.h"

namespace topo {
void set_error(const char* fmt, ...);
const char* last_error();
}  // namespace topo

using namespace topo;

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
    int id = 0;
    topo_params p{};
    int nen = 8, nn = 0, ne = 0, ncases = 1, iterations = 0;
    std::vector<double> vertex, load_vals;
    std::vector<int32_t> element, fixed, case_ptr, load_dofs;
    double arrival_s = 0.0;
    size_t est_bytes = 0;
    std::shared_ptr<std::atomic<int>> cancel = std::make_shared<std::atomic<int>>(0);
    // results
    int state = 0;  // 0 queued, 1 running, 2 done, 3 failed, 4 cancelled
    int status = 0;
    std::string error;
    double admit_s = 0.0, finish_s = 0.0;
    std::vector<double> iter_ms, fx_hist;
    std::vector<double> xphys;
};

}  // namespace

struct topo_server {
    size_t budget = 0;
    int max_active = 1;
    int batch_max_elems = 0;      // batching: jobs of at most this many elements (0: off)
    std::vector<std::pair<Job*, topo_ctx*>> ready;  // prepared jobs waiting to join the batch
    int preparing = 0;            // batched jobs still in their first iteration
    bool batch_quit = false;
    std::vector<Job> jobs;
    std::mutex mu;
    std::condition_variable cv;
    size_t reserved = 0, peak_reserved = 0;
    int active = 0, max_seen = 0;
    double makespan = 0.0;
    bool ran = false;
};

extern "C" {

size_t topo_estimate_job_bytes(int nen, int n_nodes, int n_elems, int precision) {
    const double s = precision == TOPO_PREC_MIXED ? 4.0 : 8.0;  // AMG value size
    // per element: packed Ke in FP64 + FP32, connectivity, masks, element
    // pair slots, filter matrices, SIMP moduli, design and MMA vectors, and
    // the node-row copy of Ke for the level-0 assembly (nen x 3 x 3nen values)
    const double npk = nen == 8 ? 300 : 78, nkf = nen == 8 ? 36 : 10;
    const double per_elem = npk * 12 + 4.0 * nen + 4 + 2.0 * nen * nen + nkf * 8 + nen * 8 + 12 + 8 + 20 * 8 + 4.0 * nen +
                            9.0 * nen * nen * s;
    // per node: level-0 operator (BSR + sliced ELLPACK), prolongator (BSR and
    // packed), its smoothing temporary, A*P, restriction, the Galerkin
    // product plans (about 7 pairs of 8 bytes per stencil neighbour), Krylov
    // basis, vectors
    const double deg = nen == 8 ? 27.0 : 24.0;
    const double per_node = deg * (9 * s + 4) * 2 + 8 * 18 * s * 4 + deg * 18 * s + deg * 7 * 8 + 31 * 24 + 30 * 3 * s +
                            16 * 24 + 8 * 3 * s + 7 * 8;
    const double bytes = n_elems * per_elem + n_nodes * per_node * 1.25 + 96.0 * (1 << 20);
    return (size_t)bytes;
}

int topo_server_create(size_t hbm_budget_bytes, int max_active, topo_server** out) {
    if (!out || max_active < 1) { set_error("bad argument"); return TOPO_ERR_ARG; }
    try {
        topo_server* s = new topo_server();
        if (hbm_budget_bytes == 0) {
            size_t fr = 0, tot = 0;
            if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
                cudaGetLastError();
                delete s;
                set_error("no CUDA device: this library has no CPU fallback");
                return TOPO_ERR_CUDA;
            }
            hbm_budget_bytes = (size_t)(0.85 * fr);
        }
        s->budget = hbm_budget_bytes;
        s->max_active = max_active;
        *out = s;
        return 0;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return TOPO_ERR_OOM;
    }
}

int topo_server_destroy(topo_server* s) {
    delete s;
    return 0;
}

int topo_server_submit(topo_server* s, const topo_params* p, int nen, int n_nodes, const double* vertex, int n_elems,
                       const int32_t* element, int n_fixed, const int32_t* fixed_dofs, int n_cases,
                       const int32_t* case_ptr, const int32_t* load_dofs, const double* load_vals, int iterations,
                       double arrival_s, int* job_id) {
    if (!s || !vertex || !element || !case_ptr || (n_fixed > 0 && !fixed_dofs) || iterations < 1 || n_cases < 1) {
        set_error("bad argument");
        return TOPO_ERR_ARG;
    }
    if (s->ran) { set_error("the server already ran; create a new one"); return TOPO_ERR_ARG; }
    try {
        Job j;
        j.id = (int)s->jobs.size();
        if (p) j.p = *p;
        else topo_params_default(&j.p);
        j.nen = nen;
        j.nn = n_nodes;
        j.ne = n_elems;
        j.ncases = n_cases;
        j.iterations = iterations;
        j.arrival_s = arrival_s;
        j.vertex.assign(vertex, vertex + 3L * n_nodes);
        j.element.assign(element, element + (long)n_elems * nen);
        j.fixed.assign(fixed_dofs, fixed_dofs + n_fixed);
        j.case_ptr.assign(case_ptr, case_ptr + n_cases + 1);
        j.load_dofs.assign(load_dofs, load_dofs + case_ptr[n_cases]);
        j.load_vals.assign(load_vals, load_vals + case_ptr[n_cases]);
        j.est_bytes = topo_estimate_job_bytes(nen, n_nodes, n_elems, j.p.precision);
        if (j.est_bytes > s->budget) {
            set_error("job %d needs about %zu bytes, more than the whole budget %zu", j.id, j.est_bytes, s->budget);
            return TOPO_ERR_OOM;
        }
        if (job_id) *job_id = j.id;
        s->jobs.push_back(std::move(j));
        return 0;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return TOPO_ERR_OOM;
    }
}

// a finished, failed or cancelled job gives back its slot and memory
static void retire(topo_server* s, Job* j, int rc, Clock::time_point t0) {
    std::lock_guard<std::mutex> lk(s->mu);
    j->status = rc;
    j->state = rc == TOPO_ERR_CANCELLED ? 4 : rc < 0 ? 3 : 2;
    j->finish_s = std::chrono::duration<double>(Clock::now() - t0).count();
    s->reserved -= j->est_bytes;
    s->active--;
    s->cv.notify_all();
}

static void run_job(topo_server* s, Job* j, Clock::time_point t0) {
    topo_ctx* ctx = nullptr;
    int rc = topo_create(&j->p, j->nen, j->nn, j->vertex.data(), j->ne, j->element.data(), (int)j->fixed.size(),
                         j->fixed.data(), j->ncases, j->case_ptr.data(), j->load_dofs.data(), j->load_vals.data(),
                         nullptr, &ctx);
    try {  // an exception must not leave this thread
        if (rc >= 0) rc = topo_opt_init(ctx);
        j->iter_ms.reserve(j->iterations);
        j->fx_hist.reserve(j->iterations);
        for (int it = 0; rc >= 0 && it < j->iterations; it++) {
            // cancellation is honoured between design iterations, when none
            // of this job's work is in flight
            if (j->cancel->load()) {
                rc = TOPO_ERR_CANCELLED;
                j->error = "cancelled";
                break;
            }
            auto a = Clock::now();
            int itr = 0;
            double fx = 0.0, gx = 0.0, ch = 0.0;
            rc = topo_opt_step(ctx, &itr, &fx, &gx, &ch);
            auto b = Clock::now();
            j->iter_ms.push_back(std::chrono::duration<double, std::milli>(b - a).count());
            j->fx_hist.push_back(fx);
        }
        if (rc >= 0) {
            double* xp = nullptr;
            j->xphys.resize(j->ne);
            rc = topo_opt_vector(ctx, 1, &xp);
            if (rc >= 0) rc = topo_memcpy_d2h(j->xphys.data(), xp, sizeof(double) * j->ne, ctx);
        }
        if (rc < 0 && rc != TOPO_ERR_CANCELLED) j->error = topo::last_error();
    } catch (...) {
        rc = TOPO_ERR_OOM;
        j->error = "host allocation failed";
    }
    if (ctx) topo_destroy(ctx);
    retire(s, j, rc, t0);
}

// final design of a job, then its context goes
static int finish_ctx(Job* j, topo_ctx* ctx, int rc) {
    if (rc >= 0) {
        double* xp = nullptr;
        try {
            j->xphys.resize(j->ne);
        } catch (...) {
            j->error = "host allocation failed";
            topo_destroy(ctx);
            return TOPO_ERR_OOM;
        }
        rc = topo_opt_vector(ctx, 1, &xp);
        if (rc >= 0) rc = topo_memcpy_d2h(j->xphys.data(), xp, sizeof(double) * j->ne, ctx);
        if (rc < 0) j->error = topo::last_error();
    }
    topo_destroy(ctx);
    return rc;
}

// Batched job, first part: context, the first design iteration (direct: it
// allocates and tunes) and the second (it captures the step graphs), then
// the hand-over to the batch worker, so that no capture holds up the jobs
// the worker is running.
static void prepare_job(topo_server* s, Job* j, Clock::time_point t0) {
    topo_ctx* ctx = nullptr;
    j->p.step_graph = 1;
    // default launch shapes: timing candidate shapes on a device shared with
    // the batch would measure the neighbours, and hold them up
    j->p.autotune = 0;
    int rc = topo_create(&j->p, j->nen, j->nn, j->vertex.data(), j->ne, j->element.data(), (int)j->fixed.size(),
                         j->fixed.data(), j->ncases, j->case_ptr.data(), j->load_dofs.data(), j->load_vals.data(),
                         nullptr, &ctx);
    try {
        j->iter_ms.reserve(j->iterations);
        j->fx_hist.reserve(j->iterations);
        if (rc >= 0) rc = topo_opt_init(ctx);
        if (rc >= 0 && j->cancel->load()) {
            rc = TOPO_ERR_CANCELLED;
            j->error = "cancelled";
        }
        for (int it = 0; rc >= 0 && it < 2 && it < j->iterations; it++) {
            auto a = Clock::now();
            double fx = 0.0;
            rc = topo_opt_step(ctx, nullptr, &fx, nullptr, nullptr);
            j->iter_ms.push_back(std::chrono::duration<double, std::milli>(Clock::now() - a).count());
            j->fx_hist.push_back(fx);
        }
        if (rc < 0 && rc != TOPO_ERR_CANCELLED) j->error = topo::last_error();
    } catch (...) {
        rc = TOPO_ERR_OOM;
        j->error = "host allocation failed";
    }
    if (rc >= 0 && (int)j->iter_ms.size() < j->iterations) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->ready.push_back({j, ctx});
        s->preparing--;
        s->cv.notify_all();
        return;
    }
    if (ctx) rc = finish_ctx(j, ctx, rc);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->preparing--;
    }
    retire(s, j, rc, t0);
}

// A batched job that is done: its final design is read back and its context
// destroyed on a thread of its own, so that the frees (each of which waits
// for the device) hold up no job the batch worker is running.
static void finish_batched(topo_server* s, Job* j, topo_ctx* ctx, int rc, Clock::time_point t0) {
    if (rc == TOPO_ERR_CANCELLED) {
        topo_destroy(ctx);
    } else {
        rc = finish_ctx(j, ctx, rc);
    }
    retire(s, j, rc, t0);
}

// Batched jobs, the rest: one host thread keeps every held job going.  Each
// job's next design iteration is launched (topo_opt_step_async) as soon as its
// previous one is done; the thread polls (topo_opt_step_query, which never
// blocks and launches the second half of an iteration once its solve is
// done), so no job waits for another and the host never waits on the device.
static void batch_worker(topo_server* s, Clock::time_point t0) {
    std::vector<std::thread> reapers;
    auto finish = [&](Job* j, topo_ctx* ctx, int rc) {
        try {
            reapers.emplace_back(finish_batched, s, j, ctx, rc, t0);
        } catch (...) {
            finish_batched(s, j, ctx, rc, t0);  // no thread: finish here
        }
    };
    struct Held {
        Job* j;
        topo_ctx* ctx;
        Clock::time_point start;
        bool running;
    };
    std::vector<Held> held;
    while (true) {
        {
            std::unique_lock<std::mutex> lk(s->mu);
            while (s->ready.empty() && held.empty() && !(s->batch_quit && s->preparing == 0))
                s->cv.wait_for(lk, std::chrono::milliseconds(50));
            for (auto& r : s->ready) held.push_back({r.first, r.second, Clock::now(), false});
            s->ready.clear();
            if (held.empty() && s->batch_quit && s->preparing == 0) break;
        }
        bool progressed = false;
        for (size_t i = 0; i < held.size();) {
            Held& h = held[i];
            Job* j = h.j;
            int rc = 0;
            bool retire_now = false;
            if (!h.running) {
                if (j->cancel->load()) {  // cancellations take effect between iterations
                    j->error = "cancelled";
                    finish(j, h.ctx, TOPO_ERR_CANCELLED);
                    held.erase(held.begin() + i);
                    continue;
                }
                h.start = Clock::now();
                rc = topo_opt_step_async(h.ctx);
                if (rc < 0) {
                    j->error = topo::last_error();
                    retire_now = true;
                } else {
                    h.running = true;
                }
                progressed = true;
            } else {
                int done = 0;
                double fx = 0.0;
                rc = topo_opt_step_query(h.ctx, &done, nullptr, &fx, nullptr, nullptr);
                if (rc < 0 || done) {
                    j->iter_ms.push_back(std::chrono::duration<double, std::milli>(Clock::now() - h.start).count());
                    j->fx_hist.push_back(fx);
                    h.running = false;
                    progressed = true;
                    if (rc < 0) j->error = topo::last_error();
                    retire_now = rc < 0 || (int)j->iter_ms.size() >= j->iterations;
                }
            }
            if (retire_now) {
                finish(j, h.ctx, rc);
                held.erase(held.begin() + i);
            } else {
                i++;
            }
        }
        if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    for (auto& t : reapers) t.join();
}

int topo_server_set_batching(topo_server* s, int max_elems) {
    if (!s || max_elems < 0) { set_error("bad argument"); return TOPO_ERR_ARG; }
    if (s->ran) { set_error("the server already ran"); return TOPO_ERR_ARG; }
    s->batch_max_elems = max_elems;
    return 0;
}

int topo_server_run(topo_server* s) {
    if (!s) { set_error("null server"); return TOPO_ERR_ARG; }
    if (s->ran) { set_error("the server already ran"); return TOPO_ERR_ARG; }
    s->ran = true;
    std::vector<int> order;
    std::vector<std::thread> workers;
    try {  // before any worker starts; thread starts are guarded below
        order.resize(s->jobs.size());
        workers.reserve(s->jobs.size());
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return TOPO_ERR_OOM;
    }
    for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return s->jobs[a].arrival_s < s->jobs[b].arrival_s; });
    const auto t0 = Clock::now();
    size_t next = 0;
    std::thread batcher;
    if (s->batch_max_elems > 0) {
        try {
            batcher = std::thread(batch_worker, s, t0);
        } catch (...) {
            s->batch_max_elems = 0;  // no worker thread: every job runs on its own thread
        }
    }
    {
        std::unique_lock<std::mutex> lk(s->mu);
        while (true) {
            const double now = std::chrono::duration<double>(Clock::now() - t0).count();
            // FIFO admission: the head of the queue goes first once it has
            // arrived and fits (slot + estimated footprint)
            while (next < order.size()) {
                Job& j = s->jobs[order[next]];
                if (j.cancel->load()) {  // cancelled while queued: never admitted
                    j.status = TOPO_ERR_CANCELLED;
                    j.error = "cancelled";
                    j.state = 4;
                    j.admit_s = j.finish_s = now;
                    next++;
                    continue;
                }
                if (j.arrival_s > now || s->active >= s->max_active || s->reserved + j.est_bytes > s->budget) break;
                j.state = 1;
                j.admit_s = now;
                s->reserved += j.est_bytes;
                s->peak_reserved = std::max(s->peak_reserved, s->reserved);
                s->active++;
                s->max_seen = std::max(s->max_seen, s->active);
                const bool batched = s->batch_max_elems > 0 && j.ne <= s->batch_max_elems && j.ncases == 1;
                try {
                    if (batched) {
                        s->preparing++;
                        workers.emplace_back(prepare_job, s, &j, t0);
                    } else {
                        workers.emplace_back(run_job, s, &j, t0);
                    }
                } catch (...) {
                    if (batched) s->preparing--;
                    // no host thread for this job: it fails, the others go on
                    j.status = TOPO_ERR_OOM;
                    j.error = "could not start a host thread for the job";
                    j.state = 3;
                    j.finish_s = now;
                    s->reserved -= j.est_bytes;
                    s->active--;
                }
                next++;
            }
            if (next == order.size() && s->active == 0) break;
            if (next < order.size() && s->jobs[order[next]].arrival_s > now && s->active < s->max_active) {
                const double wait = s->jobs[order[next]].arrival_s - now;
                s->cv.wait_for(lk, std::chrono::duration<double>(wait));
            } else {
                s->cv.wait_for(lk, std::chrono::milliseconds(50));
            }
        }
    }
    for (auto& t : workers) t.join();
    if (batcher.joinable()) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->batch_quit = true;
            s->cv.notify_all();
        }
        batcher.join();
    }
    s->makespan = std::chrono::duration<double>(Clock::now() - t0).count();
    int failed = 0;
    for (auto& j : s->jobs) failed += j.state == 3;
    if (failed) {
        set_error("%d job(s) failed", failed);
        return TOPO_NOT_CONVERGED;
    }
    return 0;
}

int topo_server_cancel(topo_server* s, int job_id) {
    if (!s || job_id < 0 || job_id >= (int)s->jobs.size()) { set_error("no such job"); return TOPO_ERR_ARG; }
    s->jobs[job_id].cancel->store(1);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->cv.notify_all();
    }
    return 0;
}

int topo_server_job(topo_server* s, int job_id, int* status, int* n_iters, double* iter_ms, double* fx_hist,
                    double* xphys, double* admit_s, double* finish_s) {
    if (!s || job_id < 0 || job_id >= (int)s->jobs.size()) { set_error("no such job"); return TOPO_ERR_ARG; }
    const Job& j = s->jobs[job_id];
    if (status) *status = j.status;
    if (n_iters) *n_iters = (int)j.iter_ms.size();
    if (iter_ms) std::copy(j.iter_ms.begin(), j.iter_ms.end(), iter_ms);
    if (fx_hist) std::copy(j.fx_hist.begin(), j.fx_hist.end(), fx_hist);
    if (xphys && !j.xphys.empty()) std::copy(j.xphys.begin(), j.xphys.end(), xphys);
    if (admit_s) *admit_s = j.admit_s;
    if (finish_s) *finish_s = j.finish_s;
    if (j.state >= 3) set_error("%s", j.error.c_str());
    return j.state >= 3 ? j.status : 0;
}

int topo_server_stats_get(topo_server* s, topo_server_stats* st) {
    if (!s || !st) { set_error("null argument"); return TOPO_ERR_ARG; }
    try {
    std::vector<double> lat, wait;
    int done = 0, failed = 0;
    long iters = 0;
    for (const auto& j : s->jobs) {
        done += j.state == 2;
        failed += j.state == 3;
        iters += (long)j.iter_ms.size();
        lat.insert(lat.end(), j.iter_ms.begin(), j.iter_ms.end());
        if (j.state == 2 || j.state == 3) wait.push_back(j.admit_s - j.arrival_s);
    }
    auto pct = [](std::vector<double> v, double q) {
        if (v.empty()) return 0.0;
        std::sort(v.begin(), v.end());
        const double pos = q * (v.size() - 1);
        const size_t lo = (size_t)std::floor(pos), hi = std::min(v.size() - 1, lo + 1);
        return v[lo] + (pos - lo) * (v[hi] - v[lo]);
    };
    st->jobs_submitted = (int)s->jobs.size();
    st->jobs_done = done;
    st->jobs_failed = failed;
    st->max_active = s->max_seen;
    st->iterations = iters;
    st->p50_iter_ms = pct(lat, 0.5);
    st->p99_iter_ms = pct(lat, 0.99);
    double sum = 0.0;
    for (double x : lat) sum += x;
    st->mean_iter_ms = lat.empty() ? 0.0 : sum / lat.size();
    st->makespan_s = s->makespan;
    st->jobs_per_hour = s->makespan > 0 ? 3600.0 * done / s->makespan : 0.0;
    st->iters_per_s = s->makespan > 0 ? iters / s->makespan : 0.0;
    st->peak_reserved_bytes = (double)s->peak_reserved;
    st->p50_queue_s = pct(wait, 0.5);
    st->p99_queue_s = pct(wait, 0.99);
    return 0;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return TOPO_ERR_OOM;
    }
}

}  // extern "C"
