// Request server: continuous batching of independent propagations on one GPU.
//
// The reference runs one scene per Engine and leaves scheduling to its
// directors (solver/src/vk_engine.ixx:597-698; scenario/src/base_director.ixx);
// this server accepts solves as they arrive, admits them against a device
// memory budget, keeps every admitted field and its tables resident in HBM as
// a member of one ses_batch, and advances all members together in rounds.  A
// round ends at the earliest observation point or completion of any member,
// so new requests join (and finished ones leave) between rounds while the
// others keep stepping; two rounds are kept queued so that the device never
// waits for the host's bookkeeping.  Observations stream back as records;
// latency is submission to completion.
//
// Built on the public C ABI (ses_gpu_*, ses_batch_*) plus one CUDA stream and
// events of its own (the batch's stream, round boundaries): one worker thread
// owns the batch and every handle; callers only touch the queues under a mutex.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ses_gpu.h"

namespace sesk {
void set_last_error(const std::string& msg);  // ses_gpu.cu
}

namespace {

using Clock = std::chrono::steady_clock;

// Requests admitted (handles created) per round while other requests run.
constexpr int kAdmitPerRound = 4;

ses_status sfail(ses_status s, const std::string& msg) {
    sesk::set_last_error(msg);
    return s;
}

double ms_since(Clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

long long grid_points(const ses_grid_desc& g) { return (long long)g.x.n * g.y.n * g.z.n; }

// Device bytes a request will hold (ses_gpu_create: psi, scratch and the
// potential table at the field's element size, V in FP64, plus per-axis tables
// and allocation rounding), used for admission before the handle exists.
size_t estimate_bytes(const ses_grid_desc& g, ses_precision p) {
    const size_t N = (size_t)grid_points(g);
    const size_t E = p == SES_C128 ? 16 : 8;
    return N * (3 * E + 8) + ((size_t)12 << 20);
}

struct Request {
    int64_t id = 0;
    ses_grid_desc grid{};
    ses_precision prec = SES_C64;
    double dt = 0, mass = 1, xlo = 0, xhi = 0;
    std::vector<double> V, psi0, mx, my, mz;
    int nsteps = 0, every = 0;
    int state = SES_REQ_QUEUED;
    Clock::time_point t_submit;
    double latency_ms = -1.0;
    std::deque<ses_record> records;
    std::vector<double> result;
    bool result_ready = false;
    bool cancel = false;
    std::string error;
    // worker-owned while running
    ses_handle h = nullptr;
    size_t bytes = 0;
    int done = 0;
};

}  // namespace

struct ses_server_s {
    int dev = 0;
    size_t budget = 0;
    int max_round = 100;
    ses_batch batch = nullptr;

    std::mutex mu;
    std::condition_variable cv;    // wakes the worker (new request, cancel, close)
    std::condition_variable idle;  // signalled whenever nothing is queued or running
    bool stop = false;
    std::deque<std::shared_ptr<Request>> queue;
    std::map<int64_t, std::shared_ptr<Request>> all;
    int64_t next_id = 1;
    std::thread worker;

    // worker-owned
    std::vector<std::shared_ptr<Request>> active;
    size_t used = 0;
    cudaStream_t stream = nullptr;              // the batch's stream: rounds, joins, observations
    cudaEvent_t ev_start[2] = {nullptr, nullptr};  // per round parity: start and end of a queued round
    cudaEvent_t ev_end[2] = {nullptr, nullptr};
    ses_observables* obuf[2] = {nullptr, nullptr};  // pinned observable slots per round parity
    size_t ocap[2] = {0, 0};

    // statistics (under mu)
    int64_t submitted = 0, admitted = 0, completed = 0, cancelled = 0, failed = 0, rounds = 0;
    int64_t running = 0;
    size_t used_view = 0;
    double gridpt_steps = 0, busy_ms = 0;
    std::vector<double> latencies;
    Clock::time_point t_open;
};

namespace {

int next_event(const Request& r) {
    int e = r.nsteps;
    if (r.every > 0) e = std::min(e, (r.done / r.every + 1) * r.every);
    return e;
}

// Publish a request's final state (worker thread); its handle is released by the caller.
void publish(ses_server_s* s, const std::shared_ptr<Request>& r, int state, const std::string& err) {
    std::lock_guard<std::mutex> lk(s->mu);
    r->state = state;
    r->error = err;
    --s->running;
    if (state == SES_REQ_DONE) {
        r->latency_ms = ms_since(r->t_submit);
        s->latencies.push_back(r->latency_ms);
        ++s->completed;
    } else if (state == SES_REQ_CANCELLED) {
        ++s->cancelled;
    } else {
        ++s->failed;
    }
}

// Free a request's device memory (leaving the batch first if it is a member).
void release_handle(ses_server_s* s, const std::shared_ptr<Request>& r) {
    if (r->h) {
        ses_gpu_destroy(r->h);  // removes it from the batch when it is a member
        r->h = nullptr;
    }
    s->used -= std::min(s->used, r->bytes);
    std::lock_guard<std::mutex> lk(s->mu);
    s->used_view = s->used;
}

void retire(ses_server_s* s, const std::shared_ptr<Request>& r, int state, const std::string& err) {
    release_handle(s, r);
    publish(s, r, state, err);
}

// Create the handle of a queued request (worker thread); it joins the batch
// later, between rounds.  0: created; 1: out of device memory while other
// requests hold memory (retry later); 2: failed and published.
int create_one(ses_server_s* s, const std::shared_ptr<Request>& r, bool others_hold_memory) {
    ses_handle h = nullptr;
    ses_status st = ses_gpu_create(&r->grid, r->prec, r->dt, r->mass, r->V.data(), r->psi0.data(), &h);
    if (st == SES_OK && !r->mx.empty())
        st = ses_gpu_set_absorber_separable(h, r->mx.data(), r->my.data(), r->mz.data());
    if (st != SES_OK) {
        const std::string err = ses_last_error();
        if (h) ses_gpu_destroy(h);
        if (st == SES_ENOMEM && others_hold_memory) return 1;
        std::lock_guard<std::mutex> lk(s->mu);
        r->state = SES_REQ_FAILED;
        r->error = err;
        ++s->failed;
        return 2;
    }
    size_t b = 0;
    ses_gpu_footprint(h, &b);
    r->h = h;
    r->bytes = std::max(b, estimate_bytes(r->grid, r->prec));  // charge what admission assumed
    s->used += r->bytes;
    r->V = std::vector<double>();
    r->psi0 = std::vector<double>();
    std::lock_guard<std::mutex> lk(s->mu);
    r->state = SES_REQ_RUNNING;
    ++s->admitted;
    ++s->running;
    s->used_view = s->used;
    return 0;
}

// One queued round: every member advances R merged Strang steps; the listed
// observers are observed at its end (asynchronously, into pinned slots) and the
// finishers leave the batch there.
struct Round {
    int R = 0;
    int slot = 0;  // pinned observable buffer and event pair (round parity)
    double pts = 0;
    std::vector<std::shared_ptr<Request>> observers;
    std::vector<int> obs_step;
    std::vector<std::shared_ptr<Request>> finishers;
};

// The worker keeps up to two rounds queued on the server's stream, so the
// device steps round k+1 while the host publishes round k, admits new requests
// (creates their handles and tables) and reads back finished fields.  Joining,
// leaving, stepping and observing are all stream-ordered (no host wait); the host
// waits only for the oldest round's end event.  A round ends at the earliest
// observation point or completion of any member.
void worker_main(ses_server_s* s) {
    cudaSetDevice(s->dev);
    std::deque<Round> q;
    std::vector<std::shared_ptr<Request>> pending;  // created, join the batch at the next planned round
    long long round_no = 0;
    auto fail_everything = [&](const std::string& err) {
        for (const auto& r : s->active) retire(s, r, SES_REQ_FAILED, err);
        s->active.clear();
        for (Round& rd : q)
            for (const auto& r : rd.finishers) retire(s, r, SES_REQ_FAILED, err);
        q.clear();
    };
    auto cancelled = [&](const std::shared_ptr<Request>& r) {
        std::lock_guard<std::mutex> lk(s->mu);
        return r->cancel;
    };
    for (;;) {
        // A. the oldest queued round: wait for its end, publish its observations and results
        if (!q.empty()) {
            Round rd = std::move(q.front());
            q.pop_front();
            const cudaEvent_t e1 = s->ev_end[rd.slot];
            const auto t0 = Clock::now();
            cudaError_t qe;
            while ((qe = cudaEventQuery(e1)) == cudaErrorNotReady) {
                if (ms_since(t0) > 600000.0) break;
                std::this_thread::sleep_for(std::chrono::microseconds(20));
            }
            int derr = 0;
            ses_status st = qe == cudaSuccess ? SES_OK : (qe == cudaErrorNotReady ? SES_ETIMEDOUT : SES_EDEVICE);
            // the batch's error word (an expired bounded wait in a pipelined pass) is
            // read when nothing else is queued, so the check never drains the queue
            if (st == SES_OK && q.empty()) st = ses_batch_sync(s->batch, 600000);
            if (st != SES_OK) {
                derr = 1;
                const std::string err = qe == cudaSuccess ? ses_last_error() : "round did not complete";
                for (const auto& r : rd.finishers) retire(s, r, SES_REQ_FAILED, err);
                fail_everything(err);
                cudaGetLastError();
            }
            if (!derr) {
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, s->ev_start[rd.slot], e1);
                {
                    std::lock_guard<std::mutex> lk(s->mu);
                    ++s->rounds;
                    s->gridpt_steps += rd.pts;
                    s->busy_ms += ms;
                }
                const ses_observables* ob = s->obuf[rd.slot];
                for (size_t j = 0; j < rd.observers.size(); ++j) {
                    Request& r = *rd.observers[j];
                    const int step = rd.obs_step[j];
                    ses_record rec{};
                    rec.id = r.id;
                    rec.step = step;
                    rec.final_record = step >= r.nsteps ? 1 : 0;
                    rec.t_ms = ms_since(r.t_submit);
                    rec.obs = ob[j];
                    std::lock_guard<std::mutex> lk(s->mu);
                    r.records.push_back(rec);
                }
                for (const auto& r : rd.finishers) {  // off the batch since this round's end
                    std::vector<double> out((size_t)grid_points(r->grid) * 2);
                    const ses_status rs = ses_gpu_read_psi(r->h, out.data());
                    const std::string err = rs == SES_OK ? "" : ses_last_error();
                    {
                        std::lock_guard<std::mutex> lk(s->mu);
                        r->result.swap(out);
                        r->result_ready = rs == SES_OK;
                    }
                    retire(s, r, rs == SES_OK ? SES_REQ_DONE : SES_REQ_FAILED, err);
                }
            }
        }

        // B. cancellations of running requests: they leave the batch (stream-ordered) and are freed
        for (size_t i = 0; i < s->active.size();) {
            if (cancelled(s->active[i])) {
                ses_batch_remove(s->batch, s->active[i]->h);
                retire(s, s->active[i], SES_REQ_CANCELLED, "");
                s->active.erase(s->active.begin() + (long)i);
            } else {
                ++i;
            }
        }

        // C. plan and queue rounds until two are in flight
        while (q.size() < 2) {
            for (const auto& r : pending) {
                if (cancelled(r)) {
                    retire(s, r, SES_REQ_CANCELLED, "");
                    continue;
                }
                const ses_status st = ses_batch_add(s->batch, r->h);
                if (st != SES_OK) {
                    retire(s, r, SES_REQ_FAILED, ses_last_error());
                    continue;
                }
                s->active.push_back(r);
            }
            pending.clear();
            if (s->active.empty()) break;
            Round rd;
            rd.slot = (int)(round_no & 1);
            rd.R = s->max_round;
            for (const auto& r : s->active) rd.R = std::min(rd.R, next_event(*r) - r->done);
            rd.R = std::max(rd.R, 1);
            cudaEventRecord(s->ev_start[rd.slot], s->stream);
            ses_status st = ses_batch_step(s->batch, rd.R, 1);
            for (const auto& r : s->active) {
                r->done += rd.R;
                rd.pts += (double)grid_points(r->grid) * rd.R;
                if (r->done >= r->nsteps || (r->every > 0 && r->done % r->every == 0)) {
                    rd.observers.push_back(r);
                    rd.obs_step.push_back(r->done);
                }
            }
            if (st == SES_OK && rd.observers.size() > s->ocap[rd.slot]) {
                if (s->obuf[rd.slot]) cudaFreeHost(s->obuf[rd.slot]);
                s->obuf[rd.slot] = nullptr;
                s->ocap[rd.slot] = 0;
                const size_t want = rd.observers.size() * 2 + 16;
                if (cudaMallocHost(reinterpret_cast<void**>(&s->obuf[rd.slot]), want * sizeof(ses_observables)) ==
                    cudaSuccess)
                    s->ocap[rd.slot] = want;
                else
                    st = sfail(SES_ENOMEM, "pinned observable buffer allocation failed");
            }
            for (size_t j = 0; st == SES_OK && j < rd.observers.size(); ++j) {
                const Request& r = *rd.observers[j];
                st = ses_gpu_observe_async(r.h, r.xlo, r.xhi, &s->obuf[rd.slot][j]);
            }
            for (size_t i = 0; st == SES_OK && i < s->active.size();) {
                std::shared_ptr<Request> r = s->active[i];
                if (r->done >= r->nsteps) {
                    st = ses_batch_remove(s->batch, r->h);  // its own stream waits for this round
                    rd.finishers.push_back(r);
                    s->active.erase(s->active.begin() + (long)i);
                    continue;
                }
                ++i;
            }
            if (st == SES_OK && cudaEventRecord(s->ev_end[rd.slot], s->stream) != cudaSuccess)
                st = sfail(SES_EDEVICE, "event record failed");
            if (st != SES_OK) {
                const std::string err = ses_last_error();
                for (const auto& r : rd.finishers) retire(s, r, SES_REQ_FAILED, err);
                fail_everything(err);
                break;
            }
            q.push_back(std::move(rd));
            ++round_no;
        }

        // D. admission, first come first served while the estimate fits the budget:
        //    with rounds queued, a few requests per pass (their set-up overlaps the
        //    device's work); with nothing to run, one, which then starts stepping
        std::vector<std::shared_ptr<Request>> take;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (q.empty() && s->active.empty() && pending.empty() && s->queue.empty()) {
                s->idle.notify_all();
                s->cv.wait(lk, [&] { return s->stop || !s->queue.empty(); });
            }
            if (s->stop && s->queue.empty() && s->active.empty() && pending.empty() && q.empty()) break;
            size_t room = s->budget > s->used ? s->budget - s->used : 0;
            const size_t cap = q.empty() ? 1 : (size_t)kAdmitPerRound;
            while (!s->queue.empty() && take.size() < cap) {
                std::shared_ptr<Request> r = s->queue.front();
                if (r->cancel) {
                    r->state = SES_REQ_CANCELLED;
                    ++s->cancelled;
                    s->queue.pop_front();
                    continue;
                }
                const size_t est = estimate_bytes(r->grid, r->prec);
                if (est > room) break;
                room -= est;
                take.push_back(r);
                s->queue.pop_front();
            }
        }
        for (size_t i = 0; i < take.size(); ++i) {
            const bool others = !q.empty() || !s->active.empty() || !pending.empty();
            const int c = create_one(s, take[i], others);
            if (c == 0) pending.push_back(take[i]);
            if (c == 1) {  // out of device memory: back to the head of the queue
                std::lock_guard<std::mutex> lk(s->mu);
                for (size_t j = take.size(); j-- > i;) s->queue.push_front(take[j]);
                break;
            }
        }
        if (q.empty() && s->active.empty() && pending.empty()) {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->queue.empty()) s->idle.notify_all();
        }
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->idle.notify_all();
}

double percentile(std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = p * (double)(v.size() - 1);
    const size_t lo = (size_t)pos;
    const size_t hi = std::min(lo + 1, v.size() - 1);
    return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

}  // namespace

extern "C" {

ses_status ses_serve_open(size_t budget_bytes, int max_round_steps, ses_server* out) {
    if (!out) return sfail(SES_EINVAL, "null output");
    *out = nullptr;
    if (budget_bytes == 0) return sfail(SES_EINVAL, "budget must be > 0");
    if (max_round_steps < 0) return sfail(SES_EINVAL, "max_round_steps must be >= 0");
    auto* s = new ses_server_s();
    s->budget = budget_bytes;
    s->max_round = max_round_steps > 0 ? max_round_steps : 100;
    cudaGetDevice(&s->dev);
    ses_status st = ses_batch_create(&s->batch);
    if (st == SES_OK && cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
        st = sfail(SES_EDEVICE, "stream creation failed");
    for (int i = 0; st == SES_OK && i < 2; ++i)
        if (cudaEventCreate(&s->ev_start[i]) != cudaSuccess || cudaEventCreate(&s->ev_end[i]) != cudaSuccess)
            st = sfail(SES_EDEVICE, "event creation failed");
    if (st == SES_OK) st = ses_batch_set_stream(s->batch, s->stream);
    if (st != SES_OK) {
        if (s->batch) ses_batch_destroy(s->batch);
        if (s->stream) cudaStreamDestroy(s->stream);
        delete s;
        return st;
    }
    s->t_open = Clock::now();
    s->worker = std::thread(worker_main, s);
    *out = s;
    return SES_OK;
}

ses_status ses_serve_submit(ses_server s, const ses_request* r, int64_t* id) {
    if (!s || !r || !id) return sfail(SES_EINVAL, "null argument");
    const ses_axis ax[3] = {r->grid.x, r->grid.y, r->grid.z};
    for (const ses_axis& a : ax)
        if (a.n < 1 || !(a.xmax > a.xmin)) return sfail(SES_EINVAL, "axis needs n >= 1 and xmax > xmin");
    if (r->prec != SES_C128 && r->prec != SES_C64) return sfail(SES_EINVAL, "unknown precision");
    if (!r->V || !r->psi0) return sfail(SES_EINVAL, "request needs V and psi0");
    if (r->nsteps < 1 || r->observe_every < 0) return sfail(SES_EINVAL, "need nsteps >= 1 and observe_every >= 0");
    const bool any_mask = r->mask_x || r->mask_y || r->mask_z;
    if (any_mask && !(r->mask_x && r->mask_y && r->mask_z))
        return sfail(SES_EINVAL, "absorber profiles: give all three or none");
    if (estimate_bytes(r->grid, r->prec) > s->budget)
        return sfail(SES_ENOMEM, "request needs more device memory than the server's budget");
    auto q = std::make_shared<Request>();
    q->grid = r->grid;
    q->prec = r->prec;
    q->dt = r->dt;
    q->mass = r->mass > 0 ? r->mass : 1.0;
    q->xlo = r->xlo;
    q->xhi = r->xhi;
    const size_t N = (size_t)grid_points(r->grid);
    q->V.assign(r->V, r->V + N);
    q->psi0.assign(r->psi0, r->psi0 + 2 * N);
    if (any_mask) {
        q->mx.assign(r->mask_x, r->mask_x + r->grid.x.n);
        q->my.assign(r->mask_y, r->mask_y + r->grid.y.n);
        q->mz.assign(r->mask_z, r->mask_z + r->grid.z.n);
    }
    q->nsteps = r->nsteps;
    q->every = r->observe_every;
    q->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return sfail(SES_EBUSY, "server is closing");
        q->id = s->next_id++;
        s->all[q->id] = q;
        s->queue.push_back(q);
        ++s->submitted;
    }
    s->cv.notify_one();
    *id = q->id;
    return SES_OK;
}

ses_status ses_serve_poll(ses_server s, int64_t id, ses_record* recs, int cap, int* n, int* state) {
    if (!s) return sfail(SES_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return sfail(SES_ENOTFOUND, "unknown request id");
    Request& r = *it->second;
    int k = 0;
    while (recs && k < cap && !r.records.empty()) {
        recs[k++] = r.records.front();
        r.records.pop_front();
    }
    if (n) *n = k;
    if (state) *state = r.state;
    return SES_OK;
}

ses_status ses_serve_result(ses_server s, int64_t id, double* psi_out, double* latency_ms) {
    if (!s) return sfail(SES_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return sfail(SES_ENOTFOUND, "unknown request id");
    Request& r = *it->second;
    if (r.state == SES_REQ_FAILED) return sfail(SES_EDEVICE, "request failed: " + r.error);
    if (r.state != SES_REQ_DONE) return sfail(SES_EBUSY, "request has not completed");
    if (latency_ms) *latency_ms = r.latency_ms;
    if (psi_out) {
        if (!r.result_ready) return sfail(SES_ENOTFOUND, "result already taken");
        std::memcpy(psi_out, r.result.data(), r.result.size() * sizeof(double));
        r.result = std::vector<double>();
        r.result_ready = false;
    }
    return SES_OK;
}

ses_status ses_serve_cancel(ses_server s, int64_t id) {
    if (!s) return sfail(SES_EINVAL, "null server");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->all.find(id);
        if (it == s->all.end()) return sfail(SES_ENOTFOUND, "unknown request id");
        it->second->cancel = true;
    }
    s->cv.notify_one();
    return SES_OK;
}

ses_status ses_serve_wait_idle(ses_server s, int timeout_ms) {
    if (!s) return sfail(SES_EINVAL, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    const auto pred = [&] { return s->submitted == s->completed + s->cancelled + s->failed; };
    if (timeout_ms <= 0) timeout_ms = 600000;
    if (!s->idle.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred))
        return sfail(SES_ETIMEDOUT, "server still busy after " + std::to_string(timeout_ms) + " ms");
    return SES_OK;
}

ses_status ses_serve_stats(ses_server s, ses_serve_stats_t* out) {
    if (!s || !out) return sfail(SES_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = s->submitted;
    out->admitted = s->admitted;
    out->completed = s->completed;
    out->cancelled = s->cancelled;
    out->failed = s->failed;
    out->queued = (int64_t)s->queue.size();
    out->running = s->running;
    out->rounds = s->rounds;
    out->bytes_in_use = s->used_view;
    out->budget = s->budget;
    out->gridpt_steps = s->gridpt_steps;
    out->busy_ms = s->busy_ms;
    out->wall_ms = ms_since(s->t_open);
    out->latency_p50_ms = percentile(s->latencies, 0.50);
    out->latency_p99_ms = percentile(s->latencies, 0.99);
    return SES_OK;
}

ses_status ses_serve_close(ses_server s) {
    if (!s) return sfail(SES_EINVAL, "null server");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (auto& kv : s->all) kv.second->cancel = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto& r : s->active)
        if (r->h) ses_gpu_destroy(r->h);
    ses_batch_destroy(s->batch);
    cudaStreamSynchronize(s->stream);
    for (int i = 0; i < 2; ++i) {
        if (s->ev_start[i]) cudaEventDestroy(s->ev_start[i]);
        if (s->ev_end[i]) cudaEventDestroy(s->ev_end[i]);
        if (s->obuf[i]) cudaFreeHost(s->obuf[i]);
    }
    cudaStreamDestroy(s->stream);
    delete s;
    return SES_OK;
}

}  // extern "C"
