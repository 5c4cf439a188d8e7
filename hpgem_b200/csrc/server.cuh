// Serving loop (hgg_server_*): continuous batching of independent solves.
//
// Requests (a structured mesh description, order, physics, parameters,
// tableau, precision, initial condition, dt, step count) are admitted in
// arrival order by device-memory footprint: a set-up thread reserves the
// request's footprint against the budget (waiting while it does not fit),
// builds its handle and projects its initial condition.  The GPU thread owns
// one hgg_batch and keeps two chunks of steps in flight: it issues chunk k+1,
// then waits for chunk k and reads, from a pinned copy of the batch counters
// taken at the end of chunk k, which members have no steps left.  Those leave
// the batch (host bookkeeping and stream-ordered table updates, no wait for the
// device) and go to a retire thread, which copies their solution back on the
// handle's own stream into a pinned buffer and frees their device memory, which
// admits the next requests.  Requests that are ready join before the next chunk
// is issued.  A chunk is max_chunk steps (fewer when no member needs more);
// members that finish inside a chunk stay in it without work.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct ServerRequest {
    int64_t id = 0;
    std::string description, tableau;
    int order = 1, physics = 0, precision = 0;
    std::vector<double> params;
    std::vector<double> u0;  // initial coefficients, or empty (then init_fn)
    hgg_initial_fn init_fn = nullptr;
    void *user = nullptr;
    double dt = 0.0;
    int nsteps = 0;
    // life cycle
    int state = 0;  // 0 queued, 1 set-up, 2 ready, 3 running, 4 done, 5 failed
    int error = 0;
    std::string message;
    hgg_handle *h = nullptr;
    int slot = -1;
    int issued = 0;         // steps issued to the device
    int64_t join_seq = 0;   // sequence number of the first chunk issued after joining
    int64_t footprint = 0;
    int64_t dofs = 0;
    std::vector<double> result;
    double t_submit = 0, t_ready = 0, t_start = 0, t_done = 0;
};

}  // namespace

struct hgg_server {
    int device = 0;
    int64_t budget = 0;
    int max_chunk = 25;
    std::mutex mu;
    std::condition_variable cv_setup, cv_gpu, cv_done, cv_mem, cv_retire;
    std::deque<ServerRequest *> queued, ready, retiring;
    std::unordered_map<int64_t, std::unique_ptr<ServerRequest>> requests;
    int64_t next_id = 1;
    int64_t reserved = 0;
    bool stopping = false;
    bool gpu_done = false;  // the GPU thread has ended: the retire thread empties its queue and ends
    std::vector<std::thread> setup_threads;
    std::thread gpu_thread, retire_thread;
    std::vector<cudaStream_t> side_streams;  // set-up threads' and retire thread's (high priority)
    hgg_batch *batch = nullptr;
    std::string err = "no error";
    int gpu_error = 0;
    // counters
    int64_t completed = 0, dof_updates = 0, chunks = 0;
    // GPU thread: stepping (issuing graph launches, waiting for chunks), membership
    // work (joins, removals, tables, graph captures), waiting for work; retire thread
    // busy; device time of the chunks (CUDA events around each chunk on the batch stream)
    double t_step = 0, t_members = 0, t_idle = 0, t_retire = 0, t_device = 0;
    double t_join = 0, t_prepare = 0, t_copyback = 0;  // parts: joins, table uploads and captures, copies back
};

namespace {

thread_local std::string g_server_create_error = "no error";

// device bytes of a problem: both solution buffers, the stage vectors, the
// conversion scratch and the per-element geometry and operator tables
int64_t estimate_footprint(const hgg_problem_desc &d) {
    const int64_t N = d.n_elements * (int64_t)d.n_vars * d.n_basis;
    const int64_t kbytes = d.precision == HGG_PRECISION_FP32 ? 4 : 8;
    const int64_t ahead = d.physics == HGG_PHYSICS_ADVECTION ? 0 : 2 * 8;  // wave: stage inputs formed ahead
    return (3 * 8 + ahead + d.n_stages * kbytes) * (N + 64 * 64) + d.n_elements * 640 + (8 << 20);
}

void setup_loop(hgg_server *s, cudaStream_t stream) {
    cudaSetDevice(s->device);
    for (;;) {
        ServerRequest *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_setup.wait(lk, [&] { return s->stopping || !s->queued.empty(); });
            if (s->queued.empty()) return;  // stopping
            r = s->queued.front();
            s->queued.pop_front();
            r->state = 1;
        }
        // footprint from the host descriptor
        hgg_problem_desc d{};
        void *owner = nullptr;
        int rc = hgg_structured_descriptor(r->description.c_str(), r->order, r->physics, r->params.data(),
                                           r->tableau.c_str(), r->precision, &d, &owner);
        if (rc == 0) {
            r->footprint = estimate_footprint(d);
            r->dofs = d.n_elements * (int64_t)d.n_vars * d.n_basis;
            hgg_free_descriptor(owner);
        }
        bool holds = false;  // this request's footprint is counted in s->reserved
        if (rc == 0) {
            std::unique_lock<std::mutex> lk(s->mu);
            if (r->footprint > s->budget) {
                rc = HGG_ERR_NOMEM;
                r->message = "request needs more device memory than the server's budget";
            } else {
                // admission: wait until the footprint fits next to the requests already admitted
                s->cv_mem.wait(lk, [&] { return s->stopping || s->reserved + r->footprint <= s->budget; });
                if (s->stopping) {
                    rc = HGG_ERR_INVALID;
                    r->message = "server stopped";
                } else {
                    s->reserved += r->footprint;
                    holds = true;
                }
            }
        } else {
            r->message = hgg_last_error(nullptr);
        }
        if (rc == 0) {
            rc = hgg_create_structured(r->description.c_str(), r->order, r->physics, r->params.data(),
                                       r->tableau.c_str(), r->precision, &r->h);
            if (rc) r->message = hgg_last_error(nullptr);
            // the projection on this thread's high-priority stream: its kernels take SMs
            // ahead of the waiting CTAs of the running batch
            else if ((rc = hgg_set_stream(r->h, stream))) r->message = hgg_last_error(r->h);
        }
        if (rc == 0) {
            if (!r->u0.empty()) {
                if ((int64_t)r->u0.size() != hgg_vector_length(r->h)) {
                    rc = HGG_ERR_INVALID;
                    r->message = "initial coefficients have the wrong length";
                } else {
                    rc = hgg_set_state(r->h, 0, r->u0.data());
                }
            } else if (r->init_fn) {
                const int32_t nq = hgg_num_quadrature_points(r->h);
                const int64_t nE = hgg_vector_length(r->h) / ((int64_t)r->h->op.V * r->h->op.nB);
                const int dim = r->h->op.dim;
                std::vector<double> xyz((size_t)nE * nq * dim), vals((size_t)nE * nq * r->h->op.V);
                rc = hgg_quadrature_points(r->h, xyz.data());
                if (rc == 0) {
                    r->init_fn(xyz.data(), nE * nq, dim, vals.data(), r->user);
                    rc = hgg_project(r->h, vals.data(), 0);
                }
            }
            if (rc) r->message = hgg_last_error(r->h);
            else hgg_set_store_last_stage(r->h, 0);
            // the batch reads the handle's buffers on its own stream: the set-up work is
            // finished, and the handle goes back to its own (idle) stream
            if (rc == 0 && (cudaStreamSynchronize(r->h->stream) != cudaSuccess || hgg_set_stream(r->h, nullptr))) {
                rc = HGG_ERR_CUDA;
                r->message = "set-up copies failed";
            }
        }
        std::vector<double>().swap(r->u0);
        std::lock_guard<std::mutex> lk(s->mu);
        if (rc) {
            if (r->h) {
                hgg_destroy(r->h);
                r->h = nullptr;
            }
            if (holds) s->reserved -= r->footprint;
            r->error = rc;
            r->state = 5;
            r->t_done = now_s();
            s->cv_done.notify_all();
            s->cv_mem.notify_all();
        } else {
            r->state = 2;
            r->t_ready = now_s();
            s->ready.push_back(r);
            s->cv_gpu.notify_all();
        }
    }
}

// the batch counters after one chunk, copied into pinned memory on the batch stream
struct ChunkSnapshot {
    int *host = nullptr;  // parity[cap], remaining[cap], status
    cudaEvent_t start = nullptr, end = nullptr;
    int64_t seq = 0;
};

// a request finished or failed: bookkeeping under the lock
void finish_request(hgg_server *s, ServerRequest *r, int rc, const std::string &msg) {
    r->error = rc;
    if (rc) r->message = msg;
    r->state = rc ? 5 : 4;
    r->t_done = now_s();
    s->reserved -= r->footprint;
    if (rc == 0) {
        s->completed++;
        s->dof_updates += r->dofs * (int64_t)r->nsteps;
    }
    s->cv_mem.notify_all();
    s->cv_done.notify_all();
}

// every request not finished fails with the device error; the server stops
void fail_unfinished(hgg_server *s, int rc, const std::string &msg) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->gpu_error = rc;
    s->err = msg;
    for (auto &kv : s->requests) {
        ServerRequest *r = kv.second.get();
        if (r->state >= 4) continue;
        r->error = rc;
        r->message = msg;
        r->state = 5;
        r->t_done = now_s();
    }
    s->queued.clear();
    s->ready.clear();
    s->stopping = true;
    s->cv_done.notify_all();
    s->cv_setup.notify_all();
    s->cv_mem.notify_all();
}

void gpu_loop_body(hgg_server *s, ChunkSnapshot *snap) {
    hgg_batch *b = s->batch;
    const int cap = b->cap;
    std::vector<ServerRequest *> member(cap, nullptr);  // by batch slot
    int n_members = 0;
    std::deque<int> inflight;  // snapshots of the chunks issued and not yet waited for, oldest first
    int next_snap = 0;
    int64_t seq = 0;  // chunks issued
    for (;;) {
        // 1. the requests that are ready; block only with nothing in the batch
        std::vector<ServerRequest *> joining;
        const double t0 = now_s();
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (n_members == 0 && inflight.empty()) {
                s->cv_gpu.wait(lk, [&] {
                    return !s->ready.empty() || (s->stopping && s->queued.empty() && s->ready.empty());
                });
                if (s->ready.empty()) return;  // stopping
            }
            while (!s->ready.empty() && n_members + (int)joining.size() < cap) {
                joining.push_back(s->ready.front());
                s->ready.pop_front();
            }
            s->t_idle += now_s() - t0;
        }
        const double t1 = now_s();
        // 2. joins: stream-ordered after the chunks in flight
        for (ServerRequest *r : joining) {
            const double tj = now_s();
            int32_t slot = -1;
            int rc = hgg_batch_add(b, r->h, r->dt, r->nsteps, &slot);
            if (rc) {
                const std::string msg = hgg_batch_last_error(b);
                hgg_destroy(r->h);
                r->h = nullptr;
                std::lock_guard<std::mutex> lk(s->mu);
                finish_request(s, r, rc, msg);
                continue;
            }
            r->slot = slot;
            r->issued = 0;
            r->join_seq = seq;
            member[slot] = r;
            n_members++;
            std::lock_guard<std::mutex> lk(s->mu);
            r->state = 3;
            r->t_start = now_s();
            s->t_join += r->t_start - tj;
        }
        // 3. issue the next chunk: the most steps any member still needs, capped
        int chunk = 0;
        for (int i = 0; i < cap; ++i)
            if (member[i]) chunk = std::max(chunk, member[i]->nsteps - member[i]->issued);
        chunk = std::min(chunk, s->max_chunk);
        double t_issue = 0.0;  // graph launches: they block while the device's launch queue is full
        double t_prepare = 0.0;
        if (chunk > 0) {
            ChunkSnapshot &sn = snap[next_snap];
            cudaEventRecord(sn.start, b->stream);
            const double tp = now_s();
            int rc = prepare_batch(b);  // tables of the classes whose members changed, capture if needed
            if (rc) return fail_unfinished(s, rc, hgg_batch_last_error(b));
            const double ti = now_s();
            t_prepare = ti - tp;
            for (int k = 0; k < chunk; ++k)
                if (cudaGraphLaunch(b->graph, b->stream) != cudaSuccess)
                    return fail_unfinished(s, HGG_ERR_CUDA, "serving loop: graph launch failed");
            b->launches += (int64_t)chunk * launches_per_step(b);
            t_issue = now_s() - ti;
            cudaMemcpyAsync(sn.host, b->d_parity, sizeof(int) * cap, cudaMemcpyDeviceToHost, b->stream);
            cudaMemcpyAsync(sn.host + cap, b->d_remaining, sizeof(int) * cap, cudaMemcpyDeviceToHost, b->stream);
            cudaMemcpyAsync(sn.host + 2 * cap, b->d_status, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
            cudaEventRecord(sn.end, b->stream);
            sn.seq = seq++;
            inflight.push_back(next_snap);
            next_snap = (next_snap + 1) % 3;
            for (int i = 0; i < cap; ++i)
                if (member[i]) member[i]->issued = std::min(member[i]->nsteps, member[i]->issued + chunk);
        } else if (inflight.empty()) {
            // every member's steps are issued and waited for, yet a member remains
            return fail_unfinished(s, HGG_ERR_INVALID, "serving loop: a member has no steps left to issue");
        }
        const double t2 = now_s();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->t_members += t2 - t1 - t_issue;
            s->t_step += t_issue;
            s->t_prepare += t_prepare;
            if (chunk > 0) s->chunks++;
        }
        // 4. wait for the oldest chunk once two are in flight (or nothing more can be issued)
        if (inflight.size() < 2 && chunk > 0) continue;
        ChunkSnapshot &sn = snap[inflight.front()];
        inflight.pop_front();
        cudaError_t e = cudaEventSynchronize(sn.end);
        const double t3 = now_s();
        if (e != cudaSuccess) return fail_unfinished(s, HGG_ERR_CUDA, std::string("chunk: ") + cudaGetErrorString(e));
        const int status = sn.host[2 * cap];
        if (status) return fail_unfinished(s, HGG_ERR_DEVICE, hgg::status_message(status));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, sn.start, sn.end);
        // 5. members with no steps left after that chunk leave the batch for the retire thread
        std::vector<ServerRequest *> done;
        for (int i = 0; i < cap; ++i) {
            ServerRequest *r = member[i];
            if (!r || r->join_seq > sn.seq || sn.host[cap + i] != 0) continue;
            int rc = remove_member(b, i, sn.host[i]);
            if (rc) return fail_unfinished(s, rc, hgg_batch_last_error(b));
            member[i] = nullptr;
            n_members--;
            done.push_back(r);
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->t_step += t3 - t2;
        s->t_members += now_s() - t3;
        s->t_device += 1e-3 * ms;
        for (ServerRequest *r : done) s->retiring.push_back(r);
        if (!done.empty()) s->cv_retire.notify_one();
    }
}

void gpu_loop(hgg_server *s) {
    cudaSetDevice(s->device);
    ChunkSnapshot snap[3];
    bool ok = true;
    for (auto &sn : snap) {
        ok = ok && cudaHostAlloc((void **)&sn.host, sizeof(int) * (2 * s->batch->cap + 1), cudaHostAllocDefault) ==
                       cudaSuccess;
        ok = ok && cudaEventCreate(&sn.start) == cudaSuccess && cudaEventCreate(&sn.end) == cudaSuccess;
    }
    if (ok) gpu_loop_body(s, snap);
    else fail_unfinished(s, HGG_ERR_CUDA, "serving loop: pinned counters or events could not be created");
    cudaStreamSynchronize(s->batch->stream);
    for (auto &sn : snap) {
        if (sn.host) cudaFreeHost(sn.host);
        if (sn.start) cudaEventDestroy(sn.start);
        if (sn.end) cudaEventDestroy(sn.end);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->gpu_done = true;
    s->cv_retire.notify_all();
}

// copies finished solutions back (the handle's own stream, a pinned buffer) and frees
// their device memory, off the GPU thread
void retire_loop(hgg_server *s, cudaStream_t stream) {
    cudaSetDevice(s->device);
    double *pinned = nullptr;
    size_t pinned_n = 0;
    for (;;) {
        std::vector<ServerRequest *> work;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_retire.wait(lk, [&] { return !s->retiring.empty() || s->gpu_done; });
            if (s->retiring.empty()) break;
            work.assign(s->retiring.begin(), s->retiring.end());
            s->retiring.clear();
        }
        for (ServerRequest *r : work) {
            const double t0 = now_s();
            bool failed_already;
            {
                std::lock_guard<std::mutex> lk(s->mu);
                failed_already = r->state >= 4;
            }
            int rc = 0;
            std::string msg;
            if (!failed_already) rc = hgg_set_stream(r->h, stream);  // high priority, see setup_loop
            if (!failed_already && rc == 0) {
                // one copy engine transfer into pinned memory, the layout change on the host: a
                // kernel here would wait for SMs behind the batch's persistent kernels
                const size_t n = (size_t)r->h->N_alloc;
                if (n > pinned_n) {
                    if (pinned) cudaFreeHost(pinned);
                    pinned = nullptr;
                    pinned_n = 0;
                    if (cudaHostAlloc((void **)&pinned, sizeof(double) * n, cudaHostAllocDefault) == cudaSuccess)
                        pinned_n = n;
                }
                const double tc = now_s();
                if (!pinned) {
                    rc = HGG_ERR_NOMEM;
                    msg = "pinned staging buffer could not be allocated";
                } else {
                    r->result.resize((size_t)r->h->N);
                    rc = hgg::solution_to_host(r->h, pinned, r->result.data());
                    if (rc) msg = hgg_last_error(r->h);
                }
                std::lock_guard<std::mutex> lk(s->mu);
                s->t_copyback += now_s() - tc;
            }
            hgg_destroy(r->h);
            r->h = nullptr;
            std::lock_guard<std::mutex> lk(s->mu);
            if (!failed_already) finish_request(s, r, rc, msg);
            s->t_retire += now_s() - t0;
        }
    }
    if (pinned) cudaFreeHost(pinned);
}

int sfail(hgg_server *s, int code, const std::string &msg) {
    if (s) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->err = msg;
    } else {
        g_server_create_error = msg;
    }
    return code;
}

}  // namespace

extern "C" {

int hgg_server_start(int64_t budget_bytes, int32_t max_chunk, int32_t setup_threads, int32_t capacity,
                     hgg_server **out) {
    if (!out || budget_bytes <= 0 || max_chunk < 1 || setup_threads < 1 || capacity < 1)
        return sfail(nullptr, HGG_ERR_INVALID, "budget, chunk, set-up threads and capacity must be positive");
    *out = nullptr;
    auto *s = new hgg_server();
    if (cudaGetDevice(&s->device) != cudaSuccess) {
        delete s;
        return sfail(nullptr, HGG_ERR_NOT_LOADED, "no CUDA device available");
    }
    s->budget = budget_bytes;
    s->max_chunk = max_chunk;
    int rc = hgg_batch_create(capacity, &s->batch);
    if (rc) {
        g_server_create_error = hgg_batch_last_error(nullptr);
        delete s;
        return rc;
    }
    // fixed launch shapes: timing candidates would wait for the chunks in flight
    hgg_batch_set_autotune(s->batch, 0);
    // high-priority streams of the set-up threads and the retire thread
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    s->side_streams.assign(setup_threads + 1, nullptr);
    for (auto &st : s->side_streams)
        if (cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, hi) != cudaSuccess) {
            g_server_create_error = "cudaStreamCreateWithPriority failed";
            for (auto &t : s->side_streams)
                if (t) cudaStreamDestroy(t);
            hgg_batch_destroy(s->batch);
            delete s;
            return HGG_ERR_CUDA;
        }
    for (int i = 0; i < setup_threads; ++i) s->setup_threads.emplace_back(setup_loop, s, s->side_streams[i]);
    s->gpu_thread = std::thread(gpu_loop, s);
    s->retire_thread = std::thread(retire_loop, s, s->side_streams[setup_threads]);
    *out = s;
    return 0;
}

int hgg_server_submit(hgg_server *s, const char *description, int32_t order, int32_t physics, const double *params,
                      int32_t n_params, const char *tableau, int32_t precision, const double *u0, int64_t n_u0,
                      hgg_initial_fn init_fn, void *user, double dt, int32_t nsteps, int64_t *id) {
    if (!s || !description || !params || n_params < 1 || !tableau || !id || !(dt > 0.0) || nsteps < 1)
        return sfail(s, HGG_ERR_INVALID, "bad request");
    if (!u0 && !init_fn) return sfail(s, HGG_ERR_INVALID, "an initial condition is required");
    auto r = std::make_unique<ServerRequest>();
    r->description = description;
    r->tableau = tableau;
    r->order = order;
    r->physics = physics;
    r->precision = precision;
    r->params.assign(params, params + n_params);
    if (u0) r->u0.assign(u0, u0 + n_u0);
    r->init_fn = init_fn;
    r->user = user;
    r->dt = dt;
    r->nsteps = nsteps;
    r->t_submit = now_s();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) {
        s->err = "server is stopping";
        return HGG_ERR_INVALID;
    }
    r->id = s->next_id++;
    *id = r->id;
    s->queued.push_back(r.get());
    s->requests.emplace(r->id, std::move(r));
    s->cv_setup.notify_one();
    return 0;
}

// 1: done (solution copied to `out` if not null, latency in seconds), 0: not yet,
// < 0: the request failed (message via hgg_server_last_error) or the id is unknown.
// With wait != 0 it blocks until the request is finished.
int hgg_server_poll(hgg_server *s, int64_t id, int32_t wait, double *out, int64_t n_out, double *latency_s) {
    if (!s) return sfail(s, HGG_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) {
        s->err = "unknown request id";
        return HGG_ERR_INVALID;
    }
    ServerRequest *r = it->second.get();
    if (wait) s->cv_done.wait(lk, [&] { return r->state >= 4; });
    if (r->state < 4) return 0;
    if (latency_s) *latency_s = r->t_done - r->t_submit;
    if (r->state == 5) {
        s->err = r->message;
        return r->error ? r->error : HGG_ERR_INVALID;
    }
    if (out) {
        if (n_out != (int64_t)r->result.size()) {
            s->err = "output length " + std::to_string(n_out) + " != " + std::to_string(r->result.size());
            return HGG_ERR_INVALID;
        }
        std::copy(r->result.begin(), r->result.end(), out);
    }
    return 1;
}

// number of coefficients of a finished request's solution (0 while running)
int64_t hgg_server_result_length(hgg_server *s, int64_t id) {
    if (!s) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return -1;
    return it->second->state == 4 ? (int64_t)it->second->result.size() : 0;
}

// drops a finished request's record and result
int hgg_server_release(hgg_server *s, int64_t id) {
    if (!s) return sfail(s, HGG_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end() || it->second->state < 4) {
        s->err = "unknown or unfinished request";
        return HGG_ERR_INVALID;
    }
    s->requests.erase(it);
    return 0;
}

// timestamps (seconds, steady clock) of a request: submit, ready (set up), start (first step), done
int hgg_server_times(hgg_server *s, int64_t id, double *t4) {
    if (!s || !t4) return sfail(s, HGG_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) {
        s->err = "unknown request id";
        return HGG_ERR_INVALID;
    }
    const ServerRequest *r = it->second.get();
    t4[0] = r->t_submit;
    t4[1] = r->t_ready;
    t4[2] = r->t_start;
    t4[3] = r->t_done;
    return 0;
}

// completed requests, their DoF-updates, chunks stepped, bytes reserved now
int hgg_server_stats(hgg_server *s, int64_t *stats4) {
    if (!s || !stats4) return sfail(s, HGG_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    stats4[0] = s->completed;
    stats4[1] = s->dof_updates;
    stats4[2] = s->chunks;
    stats4[3] = s->reserved;
    return 0;
}

// seconds: GPU thread stepping (issuing launches, waiting for chunks), GPU thread
// membership work (joins, removals, tables, graph captures), GPU thread waiting for
// work, retire thread (copies back, frees), device time of the chunks
int hgg_server_timing(hgg_server *s, double *t8) {
    if (!s || !t8) return sfail(s, HGG_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    t8[0] = s->t_step;
    t8[1] = s->t_members;
    t8[2] = s->t_idle;
    t8[3] = s->t_retire;
    t8[4] = s->t_device;
    t8[5] = s->t_join;
    t8[6] = s->t_prepare;
    t8[7] = s->t_copyback;
    return 0;
}

const char *hgg_server_last_error(hgg_server *s) {
    if (!s) return g_server_create_error.c_str();
    std::lock_guard<std::mutex> lk(s->mu);
    thread_local std::string copy;
    copy = s->err;
    return copy.c_str();
}

// Finishes every submitted request, then stops the threads and frees the server.
int hgg_server_stop(hgg_server *s) {
    if (!s) return sfail(s, HGG_ERR_INVALID, "null server");
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_done.wait(lk, [&] {
            for (auto &kv : s->requests)
                if (kv.second->state < 4) return s->gpu_error != 0;
            return true;
        });
        s->stopping = true;
    }
    s->cv_setup.notify_all();
    s->cv_gpu.notify_all();
    s->cv_mem.notify_all();
    for (auto &t : s->setup_threads) t.join();
    s->gpu_thread.join();
    s->retire_thread.join();
    const int rc = s->gpu_error;
    hgg_batch_destroy(s->batch);
    for (auto &kv : s->requests)
        if (kv.second->h) hgg_destroy(kv.second->h);
    for (auto &t : s->side_streams) cudaStreamDestroy(t);
    delete s;
    return rc;
}

}  // extern "C"
