// Request server: continuous batching of independent propagations on one GPU.
//
// The reference runs one scene per Engine and leaves scheduling to its
// directors (solver/src/vk_engine.ixx:597-698; scenario/src/base_director.ixx);
// this server accepts solves as they arrive, admits them against a device
// memory budget, keeps every admitted field and its tables resident in HBM as
// a member of one ses_batch, and advances all members together in rounds.  A
// round ends at the earliest observation point or completion of any member,
// so new requests join (and finished ones leave) between rounds while the
// others keep stepping; rounds are queued ahead so that the device never waits
// for the host's bookkeeping.  Observations stream back as records;
// latency is submission to completion.
//
// Built on the public C ABI (ses_gpu_*, ses_batch_*) plus one CUDA stream and
// events of its own (the batch's stream, round boundaries): one worker thread
// owns the batch and every handle; callers only touch the queues under a mutex.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
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
    int final_state = SES_REQ_DONE;  // what the finisher publishes
    std::string final_err;
};

}  // namespace

struct ses_server_s {
    int dev = 0;
    size_t budget = 0;
    int max_round = 100;
    // SES_SERVE_ALIGN=1: requests join only on a grid of max_round steps of the
    // server's clock, so that members observing every max_round steps observe at
    // the same round ends (fewer, longer rounds; joins wait up to one round).
    // Off by default: on the mixed request stream it did not raise throughput.
    bool align = false;
    ses_batch batch = nullptr;
    cudaStream_t stream = nullptr;  // the batch's stream: rounds, joins, observations

    std::mutex mu;
    std::condition_variable cv_admit;   // admitter: new request, memory freed, close
    std::condition_variable cv_work;    // worker: handle created, cancel, close
    std::condition_variable cv_finish;  // finisher: request left the batch, close
    std::condition_variable idle;       // every submitted request has finished
    bool stop = false;
    bool worker_done = false;
    std::deque<std::shared_ptr<Request>> queue;     // submitted, waiting for admission
    std::deque<std::shared_ptr<Request>> created;   // handle built, joins the batch at the next round
    std::deque<std::shared_ptr<Request>> finished;  // left the batch: read back (if done) and free
    std::map<int64_t, std::shared_ptr<Request>> all;
    int64_t next_id = 1;
    int64_t releases = 0;  // handles freed so far (admission retries after out-of-memory)
    size_t used = 0;       // device bytes charged to admitted requests
    std::thread worker, admitter, finisher;

    // worker-owned
    std::vector<std::shared_ptr<Request>> active;

    // statistics (under mu)
    int64_t submitted = 0, admitted = 0, completed = 0, cancelled = 0, failed = 0, rounds = 0;
    int64_t running = 0;
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

bool cancelled(ses_server_s* s, const std::shared_ptr<Request>& r) {
    std::lock_guard<std::mutex> lk(s->mu);
    return r->cancel;
}

// Publish a request's final state (counters under the lock); `was_running`: it
// held a handle (counted in `running`).
void publish(ses_server_s* s, const std::shared_ptr<Request>& r, int state, const std::string& err,
             bool was_running) {
    std::lock_guard<std::mutex> lk(s->mu);
    r->state = state;
    r->error = err;
    if (was_running) --s->running;
    if (state == SES_REQ_DONE) {
        r->latency_ms = ms_since(r->t_submit);
        s->latencies.push_back(r->latency_ms);
        ++s->completed;
    } else if (state == SES_REQ_CANCELLED) {
        ++s->cancelled;
    } else {
        ++s->failed;
    }
    s->idle.notify_all();
}

// Hand a request that left the batch (or never joined it) to the finisher.
void to_finisher(ses_server_s* s, const std::shared_ptr<Request>& r, int state, const std::string& err) {
    std::lock_guard<std::mutex> lk(s->mu);
    r->final_state = state;
    r->final_err = err;
    s->finished.push_back(r);
    s->cv_finish.notify_one();
}

// ---------------------------------------------------------------------------
// Admitter thread: creates the handles of queued requests (device allocation,
// uploads, table builds on the handle's own stream) while the worker keeps the
// device stepping, first come first served while the estimate fits the budget.
// ---------------------------------------------------------------------------
void admitter_main(ses_server_s* s) {
    cudaSetDevice(s->dev);
    for (;;) {
        std::shared_ptr<Request> r;
        size_t est = 0;
        int64_t releases_seen = 0;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_admit.wait(lk, [&] {
                if (s->stop) return true;
                if (s->queue.empty()) return false;
                const auto& f = s->queue.front();
                return f->cancel || estimate_bytes(f->grid, f->prec) + s->used <= s->budget;
            });
            if (s->stop) break;
            r = s->queue.front();
            s->queue.pop_front();
            if (r->cancel) {
                r->state = SES_REQ_CANCELLED;
                ++s->cancelled;
                s->idle.notify_all();
                continue;
            }
            est = estimate_bytes(r->grid, r->prec);
            s->used += est;  // reserved while the handle is built
            releases_seen = s->releases;
        }
        ses_handle h = nullptr;
        ses_status st = ses_gpu_create(&r->grid, r->prec, r->dt, r->mass, r->V.data(), r->psi0.data(), &h);
        if (st == SES_OK && !r->mx.empty())
            st = ses_gpu_set_absorber_separable(h, r->mx.data(), r->my.data(), r->mz.data());
        if (st != SES_OK) {
            const std::string err = ses_last_error();
            if (h) ses_gpu_destroy(h);
            std::unique_lock<std::mutex> lk(s->mu);
            s->used -= std::min(s->used, est);
            if (st == SES_ENOMEM && (s->running > 0 || s->used > 0)) {
                // others hold device memory: retry once some of it is freed
                s->queue.push_front(r);
                s->cv_admit.wait(lk, [&] { return s->stop || s->releases != releases_seen; });
                continue;
            }
            r->state = SES_REQ_FAILED;
            r->error = err;
            ++s->failed;
            s->idle.notify_all();
            continue;
        }
        size_t b = 0;
        ses_gpu_footprint(h, &b);
        std::lock_guard<std::mutex> lk(s->mu);
        r->h = h;
        r->bytes = std::max(b, est);  // charge at least what admission assumed
        s->used += r->bytes - est;
        r->V = std::vector<double>();
        r->psi0 = std::vector<double>();
        r->state = SES_REQ_RUNNING;
        ++s->admitted;
        ++s->running;
        s->created.push_back(r);
        s->cv_work.notify_one();
    }
}

// ---------------------------------------------------------------------------
// Finisher thread: reads back the fields of requests that completed (their own
// stream waits for the round that finished them), publishes them and frees their
// handles -- freeing device memory waits for the device, which this thread can
// afford while the worker keeps rounds queued.
// ---------------------------------------------------------------------------
void finisher_main(ses_server_s* s) {
    cudaSetDevice(s->dev);
    for (;;) {
        std::shared_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_finish.wait(lk, [&] { return !s->finished.empty() || s->worker_done; });
            if (s->finished.empty()) break;  // the worker has exited and nothing is left
            r = s->finished.front();
            s->finished.pop_front();
        }
        int state = r->final_state;
        std::string err = r->final_err;
        if (state == SES_REQ_DONE) {
            std::vector<double> out((size_t)grid_points(r->grid) * 2);
            const ses_status rs = ses_gpu_read_psi(r->h, out.data());
            if (rs != SES_OK) {
                state = SES_REQ_FAILED;
                err = ses_last_error();
            }
            std::lock_guard<std::mutex> lk(s->mu);
            r->result.swap(out);
            r->result_ready = rs == SES_OK;
        }
        if (r->h) ses_gpu_destroy(r->h);
        r->h = nullptr;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->used -= std::min(s->used, r->bytes);
            ++s->releases;
            s->cv_admit.notify_one();
        }
        publish(s, r, state, err, true);
    }
}

// One queued round: every member advances R merged Strang steps; the listed
// observers are observed at its end (asynchronously, into a pinned buffer) and
// the finishers leave the batch there.
struct Round {
    int R = 0;
    double pts = 0;     // grid points x steps
    double est_ms = 0;  // estimated device time
    std::vector<std::shared_ptr<Request>> observers;
    std::vector<int> obs_step;
    std::vector<std::shared_ptr<Request>> finishers;
    ses_observables* obs = nullptr;  // pinned, from the worker's pool
    size_t ocap = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;  // start / end on the server stream, from the pool
};

// Queue rounds until about this much device time is queued: the host's work
// between rounds then never leaves the device idle, while a newly created
// request waits at most this long to join.
constexpr double kQueueMs = 40.0;
constexpr size_t kMaxQueued = 64;

// ---------------------------------------------------------------------------
// Worker thread: owns the batch.  Keeps rounds queued on the server's stream --
// joining, stepping, observing and leaving are all stream-ordered, so the host
// waits only for the oldest round's end event, then publishes its observations
// and hands the requests it finished to the finisher.  A round ends at the
// earliest observation point or completion of any member.
// ---------------------------------------------------------------------------
void worker_main(ses_server_s* s) {
    cudaSetDevice(s->dev);
    std::deque<Round> q;
    std::vector<std::pair<ses_observables*, size_t>> obs_pool;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
    double ms_per_ptstep = 1.0 / 4.0e7;  // device ms per grid point x step, refined from measured rounds
    double queued_ms = 0.0;
    long long clock = 0;  // steps planned since the server last ran empty
    auto give_back = [&](Round& rd) {
        if (rd.obs) obs_pool.emplace_back(rd.obs, rd.ocap);
        ev_pool.emplace_back(rd.e0, rd.e1);
        rd.obs = nullptr;
    };
    auto fail_everything = [&](const std::string& err) {
        cudaStreamSynchronize(s->stream);
        for (const auto& r : s->active) {
            ses_batch_remove(s->batch, r->h);
            to_finisher(s, r, SES_REQ_FAILED, err);
        }
        s->active.clear();
        for (Round& rd : q) {
            for (const auto& r : rd.finishers) to_finisher(s, r, SES_REQ_FAILED, err);
            give_back(rd);
        }
        q.clear();
        queued_ms = 0.0;
    };
    for (;;) {
        // A. the oldest queued round: wait for its end, publish its observations
        if (!q.empty()) {
            Round rd = std::move(q.front());
            q.pop_front();
            queued_ms = std::max(0.0, queued_ms - rd.est_ms);
            const auto t0 = Clock::now();
            cudaError_t qe;
            while ((qe = cudaEventQuery(rd.e1)) == cudaErrorNotReady) {
                if (ms_since(t0) > 600000.0) break;
                std::this_thread::sleep_for(std::chrono::microseconds(20));
            }
            ses_status st = qe == cudaSuccess ? SES_OK : (qe == cudaErrorNotReady ? SES_ETIMEDOUT : SES_EDEVICE);
            // the batch's error word (an expired bounded wait in a pipelined pass) is
            // read when nothing else is queued, so the check never drains the queue
            if (st == SES_OK && q.empty()) st = ses_batch_sync(s->batch, 600000);
            if (st != SES_OK) {
                const std::string err = qe == cudaSuccess ? ses_last_error() : "round did not complete";
                cudaGetLastError();
                for (const auto& r : rd.finishers) to_finisher(s, r, SES_REQ_FAILED, err);
                give_back(rd);
                fail_everything(err);
            } else {
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, rd.e0, rd.e1);
                if (rd.pts > 0 && ms > 0) ms_per_ptstep = 0.8 * ms_per_ptstep + 0.2 * (ms / rd.pts);
                {
                    std::lock_guard<std::mutex> lk(s->mu);
                    ++s->rounds;
                    s->gridpt_steps += rd.pts;
                    s->busy_ms += ms;
                    for (size_t j = 0; j < rd.observers.size(); ++j) {
                        Request& r = *rd.observers[j];
                        ses_record rec{};
                        rec.id = r.id;
                        rec.step = rd.obs_step[j];
                        rec.final_record = rec.step >= r.nsteps ? 1 : 0;
                        rec.t_ms = ms_since(r.t_submit);
                        rec.obs = rd.obs[j];
                        r.records.push_back(rec);
                    }
                }
                give_back(rd);
                for (const auto& r : rd.finishers) to_finisher(s, r, SES_REQ_DONE, "");
            }
        }

        // B. cancellations of running requests: they leave the batch (stream-ordered)
        for (size_t i = 0; i < s->active.size();) {
            if (cancelled(s, s->active[i])) {
                ses_batch_remove(s->batch, s->active[i]->h);
                to_finisher(s, s->active[i], SES_REQ_CANCELLED, "");
                s->active.erase(s->active.begin() + (long)i);
            } else {
                ++i;
            }
        }

        // C. new members join at the next alignment point; rounds are planned and
        //    queued until about kQueueMs of device work is queued
        auto join_created = [&]() {
            std::vector<std::shared_ptr<Request>> joining;
            {
                std::lock_guard<std::mutex> lk(s->mu);
                joining.assign(s->created.begin(), s->created.end());
                s->created.clear();
            }
            for (const auto& r : joining) {
                if (cancelled(s, r)) {
                    to_finisher(s, r, SES_REQ_CANCELLED, "");
                    continue;
                }
                const ses_status st = ses_batch_add(s->batch, r->h);
                if (st != SES_OK) {
                    to_finisher(s, r, SES_REQ_FAILED, ses_last_error());
                    continue;
                }
                s->active.push_back(r);
            }
        };
        if (s->active.empty()) clock = 0;  // an idle server starts new requests at once
        const int grid = s->align ? s->max_round : 1;
        if (clock % grid == 0) join_created();
        while (!s->active.empty() && q.size() < kMaxQueued && (q.empty() || queued_ms < kQueueMs)) {
            if (clock % grid == 0 && q.size() > 0) join_created();
            Round rd;
            // with alignment, rounds end on the grid of multiples of max_round steps of
            // the server's clock, where requests join: members that observe every
            // max_round steps (or a divisor of it) then observe at round ends, and
            // only completions and other cadences cut rounds short
            rd.R = s->align ? s->max_round - (int)(clock % s->max_round) : s->max_round;
            for (const auto& r : s->active) rd.R = std::min(rd.R, next_event(*r) - r->done);
            rd.R = std::max(rd.R, 1);
            clock += rd.R;
            if (ev_pool.empty()) {
                cudaEvent_t a = nullptr, b = nullptr;
                if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
                    fail_everything("event creation failed");
                    break;
                }
                ev_pool.emplace_back(a, b);
            }
            rd.e0 = ev_pool.back().first;
            rd.e1 = ev_pool.back().second;
            ev_pool.pop_back();
            cudaEventRecord(rd.e0, s->stream);
            ses_status st = ses_batch_step(s->batch, rd.R, 1);
            for (const auto& r : s->active) {
                r->done += rd.R;
                rd.pts += (double)grid_points(r->grid) * rd.R;
                if (r->done >= r->nsteps || (r->every > 0 && r->done % r->every == 0)) {
                    rd.observers.push_back(r);
                    rd.obs_step.push_back(r->done);
                }
            }
            if (st == SES_OK && !rd.observers.empty()) {
                for (size_t i = 0; i < obs_pool.size(); ++i)
                    if (obs_pool[i].second >= rd.observers.size()) {
                        rd.obs = obs_pool[i].first;
                        rd.ocap = obs_pool[i].second;
                        obs_pool.erase(obs_pool.begin() + (long)i);
                        break;
                    }
                if (!rd.obs) {
                    const size_t want = rd.observers.size() * 2 + 16;
                    if (cudaMallocHost(reinterpret_cast<void**>(&rd.obs), want * sizeof(ses_observables)) ==
                        cudaSuccess)
                        rd.ocap = want;
                    else
                        st = sfail(SES_ENOMEM, "pinned observable buffer allocation failed");
                }
            }
            for (size_t j = 0; st == SES_OK && j < rd.observers.size(); ++j) {
                const Request& r = *rd.observers[j];
                st = ses_gpu_observe_async(r.h, r.xlo, r.xhi, &rd.obs[j]);
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
            if (st == SES_OK && cudaEventRecord(rd.e1, s->stream) != cudaSuccess)
                st = sfail(SES_EDEVICE, "event record failed");
            if (st != SES_OK) {
                const std::string err = ses_last_error();
                for (const auto& r : rd.finishers) to_finisher(s, r, SES_REQ_FAILED, err);
                give_back(rd);
                fail_everything(err);
                break;
            }
            rd.est_ms = rd.pts * ms_per_ptstep;
            queued_ms += rd.est_ms;
            q.push_back(std::move(rd));
        }

        // D. nothing queued or running: sleep until a handle is created or the server closes
        if (q.empty() && s->active.empty()) {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !s->created.empty(); });
            if (s->stop && s->created.empty()) break;
        }
    }
    for (auto& o : obs_pool) cudaFreeHost(o.first);
    for (auto& e : ev_pool) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->worker_done = true;
    s->cv_finish.notify_all();
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
    if (const char* e = std::getenv("SES_SERVE_ALIGN")) s->align = std::atoi(e) != 0;
    cudaGetDevice(&s->dev);
    ses_status st = ses_batch_create(&s->batch);
    if (st == SES_OK && cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
        st = sfail(SES_EDEVICE, "stream creation failed");
    if (st == SES_OK) st = ses_batch_set_stream(s->batch, s->stream);
    if (st != SES_OK) {
        if (s->batch) ses_batch_destroy(s->batch);
        if (s->stream) cudaStreamDestroy(s->stream);
        delete s;
        return st;
    }
    s->t_open = Clock::now();
    s->worker = std::thread(worker_main, s);
    s->admitter = std::thread(admitter_main, s);
    s->finisher = std::thread(finisher_main, s);
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
    s->cv_admit.notify_one();
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
    s->cv_admit.notify_all();
    s->cv_work.notify_all();
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
    out->bytes_in_use = s->used;
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
    s->cv_admit.notify_all();
    s->cv_work.notify_all();
    if (s->admitter.joinable()) s->admitter.join();  // a handle being built lands in `created`
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->cv_work.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();      // cancels the running requests, drains its rounds
    if (s->finisher.joinable()) s->finisher.join();  // frees every handle
    ses_batch_destroy(s->batch);
    cudaStreamSynchronize(s->stream);
    cudaStreamDestroy(s->stream);
    delete s;
    return SES_OK;
}

}  // extern "C"
