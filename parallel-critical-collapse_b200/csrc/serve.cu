// serve.cu -- the serving loop behind pcc_serve_start / pcc_submit /
// pcc_poll / pcc_wait / pcc_serve_stop / pcc_serve_stats.
//
// A request is one whole Newton solve (NewtonSolver::run, NewtonSolver.cpp:
// 279-372) of its own SimulationConfig.  A scheduler thread owns the device
// side of serving:
//
//   admission  requests are admitted in arrival order while the device bytes
//              of the admitted solves (their buffers, allocated stream-ordered
//              so that admission never synchronises the device) fit the HBM
//              budget and, optionally, a cap on concurrent solves;
//   per solve  a high-priority stream carries the solve's own small kernels:
//              Newton reset and boundary data (prologue), and after its sweeps
//              the mismatches, the device-side convergence test, J, the Newton
//              solve and the damped update; a pinned copy of the solve's Newton
//              state tells the loop whether to start the next iteration;
//   sweeps     the sweeps of every solve whose boundary data are ready are
//              pooled, and batch march launches of about one wave each take
//              them shortest work first (the solve admitted longest ago gets
//              one CTA's worth, then the solves with the least work per Newton
//              iteration take all their remaining sweeps until the wave is
//              full); two launches are in flight on low-priority streams, so a
//              launch that drains leaves its SMs to the next one, and to the
//              high-priority per-solve kernels first.
//
// Threads.  pcc_submit / pcc_poll / pcc_wait / pcc_serve_stats may be called
// from any thread while serving runs.  Each holds the server as a "user" for
// its duration (ctx->serve_mu guards the pointer, Server::users counts the
// holders); pcc_serve_stop first lets the loop finish every submitted request,
// then unpublishes the server, wakes the waiters still blocked in pcc_wait
// (they return PCC_ERR_BUSY) and deletes it only once no user is left.  A
// finished result is handed out once: the pcc_poll or pcc_wait call that
// returns it with done = 1 erases the record, so a long-running service keeps
// no per-request memory for results already delivered.
//
// Newton state stays on the device for the whole solve; the host reads one
// small record per iteration.  A solve's result does not depend on the mix it
// ran in: every sweep is computed by one sweep slot with the same arithmetic,
// and its per-solve kernels are its own.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "pcc_objects.h"

namespace pcc {

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

int sweeps_per_cta(int ntau) { return ntau >= 1024 ? 1 : 1024 / ntau; }  // 2 stages, 128-thread CTAs

}  // namespace

struct ServeRequest {
    uint64_t ticket = 0;
    pcc_solve_desc desc{};
    std::vector<double> in0;
    pcc_precision prec = PCC_PREC_FP64;
    Clock::time_point t_submit;
};

struct ServeRecord {
    bool done = false;
    pcc_status status = PCC_OK;
    pcc_newton_state st{};
    std::vector<double> x;
    double ms_queued = -1.0, ms_latency = -1.0;
    size_t footprint = 0;
    std::string error;
};

struct Active {
    ServeRequest req;
    pcc_solve* s = nullptr;
    cudaStream_t st = nullptr;  // high priority: this solve's own kernels
    cudaEvent_t ev = nullptr;   // end of the work last enqueued on st
    NewtonDev* h_nd = nullptr;  // pinned slot written by the Newton tail
    int phase = 0;              // 0 boundary data in flight, 1 sweeps, 2 Newton tail in flight
    int next_item = 0, n_items = 0, outstanding = 0;
    int lu_steps = -1, lu_fb = 0;
    size_t footprint = 0;
    Clock::time_point t_admit;
};

struct Launch {
    BatchTables tab;
    cudaStream_t st = nullptr;
    bool busy = false;
    std::vector<std::pair<Active*, int>> parts;
};

struct Server {
    pcc_ctx* ctx = nullptr;
    size_t budget = 0;
    int max_active = 0;
    std::thread th;
    std::mutex mu;
    std::condition_variable cv_submit, cv_done;
    // guarded by mu
    std::deque<ServeRequest> queue;
    std::map<uint64_t, ServeRecord> records;
    uint64_t next_ticket = 1;
    std::atomic<bool> stop{false}, abort{false};
    int users = 0;          // API calls holding the server (pcc_submit/poll/wait/stats)
    bool closing = false;   // pcc_serve_stop has unpublished the server
    bool stop_claimed = false;  // a pcc_serve_stop call owns the shutdown (guarded by ctx->serve_mu)
    std::string fatal;
    long long submitted = 0, completed = 0, launches_done = 0, sweeps_done = 0;
    int n_active = 0, n_waiting = 0;
    size_t used_published = 0;
    // owned by the loop thread
    std::vector<std::unique_ptr<Active>> active;
    std::deque<ServeRequest> waiting;
    Launch launches[2];
    int next_launch = 0;
    size_t used = 0;
    NewtonDev* h_slots = nullptr;  // pinned Newton-state slots
    std::vector<int> free_slots;
    int lo_prio = 0, hi_prio = 0;

    void loop();
    bool admit();
    bool poll_active();
    bool poll_launches();
    bool start_launches();
    void finish(Active& a, pcc_status status, const std::string& why);
    void publish();
};

static constexpr int kServeSlots = 4096;

void Server::publish()
{
    std::lock_guard<std::mutex> lk(mu);
    n_active = (int)active.size();
    n_waiting = (int)waiting.size() + (int)queue.size();
    used_published = used;
}

void Server::finish(Active& a, pcc_status status, const std::string& why)
{
    ServeRecord rec;
    rec.done = true;
    rec.status = status;
    rec.error = why;
    rec.footprint = a.footprint;
    if (a.s) {
        const NewtonDev nd = *a.h_nd;
        rec.st.iterations = nd.its;
        rec.st.code = nd.state;
        rec.st.err = nd.err;
        rec.st.err_old = nd.err_old;
        rec.st.fail_column = rec.st.fail_side = rec.st.fail_grid_index = -1;
        rec.st.lu_refinement_steps = a.lu_steps;
        rec.st.lu_fell_back = a.lu_fb;
        rec.x.resize(a.s->nn);
        const double* src = nd.state == kNewtonStopped ? a.s->d_in0old : a.s->d_in0;
        if (cudaMemcpyAsync(rec.x.data(), src, a.s->nn * sizeof(double), cudaMemcpyDeviceToHost, a.st) != cudaSuccess ||
            cudaStreamSynchronize(a.st) != cudaSuccess) {
            rec.status = PCC_ERR_CUDA;
            rec.error = "result copy failed";
        }
        if (rec.status == PCC_OK && nd.state != kNewtonConverged && nd.state != kNewtonStopped) {
            rec.status = nd.state == kNewtonIrkFailed        ? PCC_ERR_IRK_NO_CONVERGENCE
                         : nd.state == kNewtonDeltaMismatch ? PCC_ERR_DELTA_MISMATCH
                         : nd.state == kNewtonSingular      ? PCC_ERR_LU_SINGULAR
                                                            : PCC_ERR_NEWTON_NO_CONVERGENCE;
        }
        solve_release(a.s);  // stream-ordered frees on a.st
        a.s = nullptr;
        used -= a.footprint;
    }
    rec.ms_queued = ms_between(a.req.t_submit, a.t_admit);
    rec.ms_latency = ms_between(a.req.t_submit, Clock::now());
    free_slots.push_back((int)(a.h_nd - h_slots));
    if (a.ev) cudaEventDestroy(a.ev);
    if (a.st) cudaStreamDestroy(a.st);  // released once its work has finished
    {
        std::lock_guard<std::mutex> lk(mu);
        records[a.req.ticket] = std::move(rec);
        completed += 1;
    }
    cv_done.notify_all();
}

bool Server::admit()
{
    bool progress = false;
    while (!waiting.empty() && !abort) {
        ServeRequest& req = waiting.front();
        const size_t fp = solve_footprint(req.desc, ctx->sms);
        if (max_active > 0 && (int)active.size() >= max_active) break;
        if (free_slots.empty()) break;
        if (used + fp > budget) {
            if (!active.empty()) break;  // wait for memory to free up
            Active a;
            a.req = std::move(req);
            a.t_admit = Clock::now();
            a.h_nd = h_slots + free_slots.back();
            free_slots.pop_back();
            waiting.pop_front();
            finish(a, PCC_ERR_OOM, "the solve alone exceeds the serving memory budget");
            progress = true;
            continue;
        }
        auto a = std::make_unique<Active>();
        a->req = std::move(req);
        waiting.pop_front();
        a->t_admit = Clock::now();
        a->footprint = fp;
        a->h_nd = h_slots + free_slots.back();
        free_slots.pop_back();
        std::memset(a->h_nd, 0, sizeof(NewtonDev));
        progress = true;
        if (cudaStreamCreateWithPriority(&a->st, cudaStreamNonBlocking, hi_prio) != cudaSuccess ||
            cudaEventCreateWithFlags(&a->ev, cudaEventDisableTiming) != cudaSuccess) {
            finish(*a, PCC_ERR_CUDA, "stream or event creation failed");
            continue;
        }
        pcc_status r = solve_create(ctx, &a->req.desc, a->st, false, &a->s);
        if (r != PCC_OK) {
            a->s = nullptr;
            finish(*a, r, pcc_last_error(ctx));
            continue;
        }
        used += fp;
        if ((int)a->req.in0.size() != a->s->nn) {
            finish(*a, PCC_ERR_INVALID_ARG, "in0 must hold Nnewton = 3 Ntau / 4 values");
            continue;
        }
        r = newton_reset(a->s, a->req.in0.data(), a->st);
        if (r == PCC_OK) r = newton_prologue(a->s, a->st);
        if (r != PCC_OK || cudaEventRecord(a->ev, a->st) != cudaSuccess) {
            finish(*a, r == PCC_OK ? PCC_ERR_CUDA : r, "enqueue failed");
            continue;
        }
        a->phase = 0;
        active.push_back(std::move(a));
    }
    return progress;
}

bool Server::poll_active()
{
    bool progress = false;
    for (auto it = active.begin(); it != active.end();) {
        Active& a = **it;
        if (abort && a.phase == 1 && a.outstanding == 0) {
            // stopping: sweeps not yet launched are dropped
            finish(a, PCC_ERR_BUSY, fatal.empty() ? "serving stopped" : fatal);
            it = active.erase(it);
            progress = true;
            continue;
        }
        if (a.phase == 0 || a.phase == 2) {
            const cudaError_t q = cudaEventQuery(a.ev);
            if (q == cudaErrorNotReady) {
                ++it;
                continue;
            }
            if (q != cudaSuccess) {
                std::lock_guard<std::mutex> lk(mu);
                fatal = cudaGetErrorString(q);
                abort = true;
                ++it;
                continue;
            }
            progress = true;
            if (a.phase == 0) {
                a.phase = 1;
                a.next_item = 0;
                a.n_items = (int)a.s->sweeps_build.size();
                a.outstanding = 0;
            } else if (a.h_nd->state == kNewtonRunning && !abort) {
                pcc_status r = newton_prologue(a.s, a.st);
                if (r != PCC_OK || cudaEventRecord(a.ev, a.st) != cudaSuccess) {
                    finish(a, PCC_ERR_CUDA, "enqueue failed");
                    it = active.erase(it);
                    continue;
                }
                a.phase = 0;
            } else {
                finish(a, abort ? PCC_ERR_BUSY : PCC_OK, abort ? "serving stopped" : "");
                it = active.erase(it);
                continue;
            }
        }
        ++it;
    }
    return progress;
}

bool Server::poll_launches()
{
    bool progress = false;
    for (Launch& L : launches) {
        if (!L.busy) continue;
        const cudaError_t q = cudaEventQuery(L.tab.ev[1]);
        if (q == cudaErrorNotReady) continue;
        if (q != cudaSuccess) {
            std::lock_guard<std::mutex> lk(mu);
            fatal = cudaGetErrorString(q);
            abort = true;
            continue;
        }
        progress = true;
        L.busy = false;
        long long n = 0;
        for (auto& part : L.parts) {
            Active& a = *part.first;
            n += part.second;
            a.outstanding -= part.second;
            if (a.outstanding == 0 && a.next_item == a.n_items && !abort) {
                // every sweep of this iteration is done: the Newton tail on the solve's own stream
                pcc_status r = newton_tail(a.s, a.req.prec, a.st, &a.lu_steps, &a.lu_fb);
                if (r == PCC_OK &&
                    cudaMemcpyAsync(a.h_nd, a.s->d_newton, sizeof(NewtonDev), cudaMemcpyDeviceToHost, a.st) ==
                        cudaSuccess &&
                    cudaEventRecord(a.ev, a.st) == cudaSuccess) {
                    a.phase = 2;
                } else {
                    std::lock_guard<std::mutex> lk(mu);
                    fatal = "Newton tail enqueue failed";
                    abort = true;
                }
            }
        }
        L.parts.clear();
        std::lock_guard<std::mutex> lk(mu);
        launches_done += 1;
        sweeps_done += n;
    }
    return progress;
}

bool Server::start_launches()
{
    bool progress = false;
    for (int k = 0; k < 2 && !abort; ++k) {
        Launch& L = launches[(next_launch + k) % 2];
        if (L.busy) continue;
        std::vector<Active*> ready;
        for (auto& a : active)
            if (a->phase == 1 && a->next_item < a->n_items) ready.push_back(a.get());
        if (ready.empty()) break;
        // About one wave of sweeps, shortest work first: the solve admitted
        // longest ago gets one CTA's worth first (no solve waits for ever),
        // then the wave fills with the solves whose Newton iteration is the
        // least work (sweeps x steps x Ntau log2 Ntau), each taking all of
        // its remaining sweeps, so that small solves finish early instead of
        // sharing every wave with large ones.  Throughput is the same; a
        // solve's results do not depend on the mix.
        const int capacity = 2 * ctx->sms;
        auto work = [](const Active* a) {
            const double n = a->s->d.ntau;
            return (double)a->n_items * (a->s->d.nl + a->s->d.nr) * n * std::log2(n);
        };
        std::stable_sort(ready.begin(), ready.end(),
                         [&](const Active* x, const Active* y) { return work(x) < work(y); });
        size_t oldest = 0;
        for (size_t i = 1; i < ready.size(); ++i)
            if (ready[i]->t_admit < ready[oldest]->t_admit) oldest = i;
        std::vector<BatchItem> items;
        std::vector<int> taken(ready.size(), 0);
        double ctas = 0.0;
        auto give = [&](size_t i, int limit) {
            Active& a = *ready[i];
            const int spc = sweeps_per_cta(a.s->d.ntau);
            const int take = std::min({limit, a.n_items - a.next_item,
                                       (int)std::ceil((capacity - ctas) * spc)});
            if (take <= 0) return;
            for (int j = 0; j < take; ++j) items.push_back({a.s, a.s->sweeps_build[a.next_item + j]});
            a.next_item += take;
            taken[i] += take;
            ctas += (double)take / spc;
        };
        give(oldest, sweeps_per_cta(ready[oldest]->s->d.ntau));
        for (size_t i = 0; i < ready.size() && ctas < capacity; ++i) give(i, ready[i]->n_items);
        L.parts.clear();
        for (size_t i = 0; i < ready.size(); ++i)
            if (taken[i]) {
                ready[i]->outstanding += taken[i];
                L.parts.push_back({ready[i], taken[i]});
            }
        const int max_ctas = std::max(1, (int)std::ceil(ctas));
        pcc_status r = batch_march_items(ctx, L.tab, items, L.st, max_ctas);
        if (r != PCC_OK) {
            std::lock_guard<std::mutex> lk(mu);
            fatal = pcc_last_error(ctx);
            abort = true;
            break;
        }
        L.busy = true;
        next_launch = (next_launch + k + 1) % 2;
        progress = true;
    }
    return progress;
}

void Server::loop()
{
    cudaSetDevice(ctx->device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu);
            while (!queue.empty()) {
                waiting.push_back(std::move(queue.front()));
                queue.pop_front();
            }
            const bool idle = active.empty() && !launches[0].busy && !launches[1].busy;
            if (abort) {
                // drop what has not started; in-flight work runs to its end below
                lk.unlock();
                while (!waiting.empty()) {
                    Active a;
                    a.req = std::move(waiting.front());
                    waiting.pop_front();
                    a.t_admit = Clock::now();
                    if (free_slots.empty()) break;
                    a.h_nd = h_slots + free_slots.back();
                    free_slots.pop_back();
                    finish(a, PCC_ERR_BUSY, fatal.empty() ? "serving stopped" : fatal);
                }
                lk.lock();
                if (idle) break;
            } else if (stop && idle && waiting.empty()) {
                break;
            } else if (idle && waiting.empty()) {
                cv_submit.wait_for(lk, std::chrono::milliseconds(50));
                continue;
            }
        }
        bool progress = admit();
        progress = poll_active() || progress;
        progress = poll_launches() || progress;
        progress = start_launches() || progress;
        publish();
        if (!progress) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    publish();
}

void server_shutdown(pcc_ctx* ctx)
{
    Server* sv = nullptr;
    if (ctx) {
        std::lock_guard<std::mutex> g(ctx->serve_mu);
        sv = ctx->server;
        ctx->server = nullptr;  // no new user can take it from here on
    }
    if (!sv) return;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
        sv->abort = true;
    }
    sv->cv_submit.notify_all();
    if (sv->th.joinable()) sv->th.join();
    {
        // wake the callers still blocked in pcc_wait (they return
        // PCC_ERR_BUSY) and wait until every user has left
        std::unique_lock<std::mutex> lk(sv->mu);
        sv->closing = true;
        sv->cv_done.notify_all();
        sv->cv_done.wait(lk, [&] { return sv->users == 0; });
    }
    for (Launch& L : sv->launches) {
        batch_tables_free(L.tab);
        if (L.st) cudaStreamDestroy(L.st);
    }
    if (sv->h_slots) cudaFreeHost(sv->h_slots);
    delete sv;
}

}  // namespace pcc

using namespace pcc;

namespace {

// Starts the loop; the caller holds ctx->serve_mu and has checked that no
// server runs.
pcc_status serve_start_locked(pcc_ctx* ctx, const pcc_serve_opts* opts)
{
    if (opts && opts->max_active < 0) return PCC_ERR_INVALID_ARG;
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    auto sv = std::make_unique<Server>();
    sv->ctx = ctx;
    size_t free_b = 0, total_b = 0;
    PCC_CUDA(ctx, cudaMemGetInfo(&free_b, &total_b));
    sv->budget = (opts && opts->hbm_budget_bytes) ? opts->hbm_budget_bytes : free_b / 4 * 3;
    sv->max_active = opts ? opts->max_active : 0;
    PCC_CUDA(ctx, cudaDeviceGetStreamPriorityRange(&sv->lo_prio, &sv->hi_prio));
    for (Launch& L : sv->launches) {
        PCC_CUDA(ctx, cudaStreamCreateWithPriority(&L.st, cudaStreamNonBlocking, sv->lo_prio));
        pcc_status r = batch_tables_reserve(ctx, L.tab, 1 << 20);
        if (r != PCC_OK) return r;
    }
    PCC_CUDA(ctx, cudaMallocHost(&sv->h_slots, kServeSlots * sizeof(NewtonDev)));
    for (int i = kServeSlots - 1; i >= 0; --i) sv->free_slots.push_back(i);
    Server* raw = sv.release();
    ctx->server = raw;
    raw->th = std::thread([raw] { raw->loop(); });
    return PCC_OK;
}

// The running server, held as a user until release(); null when none runs or
// it is being stopped.
Server* acquire(pcc_ctx* ctx)
{
    std::lock_guard<std::mutex> g(ctx->serve_mu);
    Server* sv = ctx->server;
    if (!sv) return nullptr;
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->users += 1;
    return sv;
}

void release(Server* sv)
{
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->users -= 1;
    if (sv->closing) sv->cv_done.notify_all();
}

struct UserGuard {
    Server* sv;
    ~UserGuard()
    {
        if (sv) release(sv);
    }
};

}  // namespace

extern "C" {

pcc_status pcc_serve_start(pcc_ctx* ctx, const pcc_serve_opts* opts)
{
    if (!ctx) return PCC_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->serve_mu);
    if (ctx->server) return fail(ctx, PCC_ERR_BUSY, "serving already started");
    return serve_start_locked(ctx, opts);
}

pcc_status pcc_submit(pcc_ctx* ctx, const pcc_request* req, uint64_t* ticket)
{
    if (!ctx || !req || !req->in0 || !ticket) return PCC_ERR_INVALID_ARG;
    if (req->precision != PCC_PREC_FP64 && req->precision != PCC_PREC_MIXED) return PCC_ERR_INVALID_ARG;
    if (req->desc.ntau < 128 || req->desc.ntau > 2048 || (req->desc.ntau & (req->desc.ntau - 1)))
        return fail(ctx, PCC_ERR_INVALID_ARG, "Ntau must be 128..2048, power of two");
    if (!march_batch_supported(req->desc.ntau, req->desc.scheme))
        return fail(ctx, PCC_ERR_UNSUPPORTED, "serving batches Ntau 128..1024 with 2 IRK stages");
    if (!all_finite(req->in0, 3 * req->desc.ntau / 4))
        return fail(ctx, PCC_ERR_NAN, "non-finite value in the free data");
    {
        // the lazy start: two first submits from different threads start one loop
        std::lock_guard<std::mutex> g(ctx->serve_mu);
        if (!ctx->server) {
            pcc_status r = serve_start_locked(ctx, nullptr);
            if (r != PCC_OK) return r;
        }
    }
    Server* sv = acquire(ctx);
    if (!sv) return fail(ctx, PCC_ERR_BUSY, "serving is stopping");
    UserGuard hold{sv};
    ServeRequest r;
    r.desc = req->desc;
    r.in0.assign(req->in0, req->in0 + 3 * req->desc.ntau / 4);
    r.prec = req->precision;
    r.t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        if (sv->stop) return fail(ctx, PCC_ERR_BUSY, "serving is stopping");
        r.ticket = sv->next_ticket++;
        *ticket = r.ticket;
        sv->records[r.ticket] = ServeRecord{};
        sv->queue.push_back(std::move(r));
        sv->submitted += 1;
    }
    sv->cv_submit.notify_all();
    return PCC_OK;
}

static void fill_result(const ServeRecord& rec, pcc_result* out, double* x_out)
{
    if (out) {
        std::memset(out, 0, sizeof(*out));
        out->done = rec.done ? 1 : 0;
        out->status = rec.status;
        out->newton = rec.st;
        out->ms_queued = rec.ms_queued;
        out->ms_latency = rec.ms_latency;
        out->footprint_bytes = rec.footprint;
    }
    if (rec.done && x_out && !rec.x.empty()) std::memcpy(x_out, rec.x.data(), rec.x.size() * sizeof(double));
}

pcc_status pcc_poll(pcc_ctx* ctx, uint64_t ticket, pcc_result* out, double* x_out)
{
    if (!ctx) return PCC_ERR_INVALID_ARG;
    Server* sv = acquire(ctx);
    if (!sv) return PCC_ERR_INVALID_ARG;
    UserGuard hold{sv};
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->records.find(ticket);
    if (it == sv->records.end()) return PCC_ERR_INVALID_ARG;
    fill_result(it->second, out, x_out);
    if (it->second.done) sv->records.erase(it);  // delivered: a result is handed out once
    return PCC_OK;
}

pcc_status pcc_wait(pcc_ctx* ctx, uint64_t ticket, double timeout_s, pcc_result* out, double* x_out)
{
    if (!ctx) return PCC_ERR_INVALID_ARG;
    Server* sv = acquire(ctx);
    if (!sv) return PCC_ERR_INVALID_ARG;
    UserGuard hold{sv};
    std::unique_lock<std::mutex> lk(sv->mu);
    if (sv->records.find(ticket) == sv->records.end()) return PCC_ERR_INVALID_ARG;
    const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                          std::chrono::duration<double>(timeout_s < 0 ? 0.0 : timeout_s));
    // records are erased only by the call that delivers them, so the ticket's
    // record stays while this call waits (unless another thread takes it)
    auto ready = [&] {
        auto it = sv->records.find(ticket);
        return it == sv->records.end() || it->second.done || sv->closing;
    };
    sv->cv_done.wait_until(lk, until, ready);
    auto it = sv->records.find(ticket);
    if (it == sv->records.end()) return PCC_ERR_INVALID_ARG;  // delivered to another caller meanwhile
    fill_result(it->second, out, x_out);
    if (it->second.done) {
        sv->records.erase(it);
        return PCC_OK;
    }
    return sv->closing ? PCC_ERR_BUSY : PCC_ERR_TIMEOUT;
}

pcc_status pcc_serve_stats(pcc_ctx* ctx, pcc_serve_info* out)
{
    if (!ctx || !out) return PCC_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    Server* sv = acquire(ctx);
    if (!sv) return PCC_OK;
    UserGuard hold{sv};
    std::lock_guard<std::mutex> lk(sv->mu);
    out->submitted = sv->submitted;
    out->completed = sv->completed;
    out->launches = sv->launches_done;
    out->sweeps = sv->sweeps_done;
    out->active = sv->n_active;
    out->waiting = sv->n_waiting;
    out->bytes_in_use = sv->used_published;
    out->budget_bytes = sv->budget;
    return PCC_OK;
}

pcc_status pcc_serve_stop(pcc_ctx* ctx)
{
    if (!ctx) return PCC_ERR_INVALID_ARG;
    Server* sv = nullptr;
    {
        std::lock_guard<std::mutex> g(ctx->serve_mu);
        sv = ctx->server;
        if (!sv || sv->stop_claimed) return PCC_OK;  // not running, or another call is stopping it
        sv->stop_claimed = true;
    }
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;  // finish everything submitted, then leave
    }
    sv->cv_submit.notify_all();
    if (sv->th.joinable()) sv->th.join();  // waiters keep receiving results meanwhile
    std::string fatal = sv->fatal;
    server_shutdown(ctx);
    if (!fatal.empty()) return fail(ctx, PCC_ERR_CUDA, "serving loop: " + fatal);
    return PCC_OK;
}

}  // extern "C"
