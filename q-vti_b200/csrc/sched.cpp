// Shot scheduler: batches of shots and a continuous serving loop on one GPU.
//
// The reference runs its shots one after another from a host loop
// (viscoelas_3D.cpp:355-405; each shot is one synchronous
// cuda_forward_acoustic_3D call, cuviscoelas_3D.cu:1163-1629).  Shots are
// independent, so here many of them -- grids of any supported size -- are in
// flight on one GPU at once:
//
//   * every shot runs on a pooled simulation (one stream each) whose time
//     loop is CUDA graphs of 16 steps (and of one step for a remainder),
//     launched in chunks of kChunk steps
//     with at most two chunks queued ahead, so a long shot never fills the
//     launch queue and the scheduler thread stays free;
//   * shots are admitted first in, first out (or smallest first, with a
//     bound on how often a shot is passed) when a slot and device memory
//     are free: an idle pooled simulation of the same grid is reused,
//     otherwise idle simulations are freed (least recently used first) until
//     the new one fits the budget;
//   * the number of shots in flight is fixed by the caller, taken from the
//     per-grid autotuner cache (plus one slot for a shot being set up), or
//     bounded by the cells in flight.
//
// One scheduler thread issues every engine call of a server; callers only
// touch the queue and the results under the server's mutex.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "qvti.h"

namespace {

constexpr int kChunk = 32;                      // steps per enqueued chunk
constexpr int kMaxBypass = 8;                   // smallest first: passes before the head goes next
constexpr long long kCellsInFlight = 1ll << 25;  // default bound: two 256^3 grids

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct GridKey {
    int ntx, nty, ntz, pml, vti;
    float dx, dy, dz, dt, f0;
    auto tie() const { return std::tie(ntx, nty, ntz, pml, vti, dx, dy, dz, dt, f0); }
    bool operator<(const GridKey& o) const { return tie() < o.tie(); }
    bool operator==(const GridKey& o) const { return tie() == o.tie(); }
};

GridKey key_of(const qvti_shot& s) { return {s.ntx, s.nty, s.ntz, s.pml, s.vti, s.dx, s.dy, s.dz, s.dt, s.f0}; }

// Grids that share the transform sizes share the tuning (pml, spacing and dt
// do not change the launch shapes).
struct ShapeKey {
    int ntx, nty, ntz, vti;
    bool operator<(const ShapeKey& o) const
    {
        return std::tie(ntx, nty, ntz, vti) < std::tie(o.ntx, o.nty, o.ntz, o.vti);
    }
};

struct Tuning {
    int active, kz_batch, form;
    int tiles[QVTI_NUM_TILES];
};
std::mutex g_tune_mu;
std::map<ShapeKey, Tuning> g_tune;

bool cached_tuning(const ShapeKey& k, Tuning* t)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(k);
    if (it == g_tune.end()) return false;
    *t = it->second;
    return true;
}

qvti_config config_of(const GridKey& k, int device)
{
    qvti_config c{};
    c.ntx = k.ntx; c.nty = k.nty; c.ntz = k.ntz; c.pml = k.pml;
    c.dx = k.dx; c.dy = k.dy; c.dz = k.dz; c.dt = k.dt; c.f0 = k.f0;
    c.vti = k.vti; c.device = device; c.w0 = 0.f;
    return c;
}

struct PoolSim {
    qvti_sim* sim = nullptr;
    GridKey key{};
    size_t bytes = 0;
    bool busy = false;
    double last_used = 0;
    int* nonfinite = nullptr;  // pinned host copy of the simulation's non-finite flag
    ~PoolSim()
    {
        if (nonfinite) cudaFreeHost(nonfinite);
    }
};

struct Job {
    long long ticket = 0;
    qvti_shot shot{};
    double t_submit = 0, t_start = 0;
    PoolSim* slot = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t chunk[2] = {nullptr, nullptr};
    int nchunk = 0;  // chunks queued and not known finished (0..2)
    int bypassed = 0;  // times a smaller shot was admitted ahead of it (smallest first)
    int enq = 0;     // steps enqueued
    bool finished = false;  // all steps queued (worker-owned)
    bool ready = false;     // result available (under the server mutex)
    qvti_shot_result res{};
};

size_t shot_bytes(const qvti_shot& s)
{
    return qvti_footprint_bytes(s.ntx, s.nty, s.ntz, s.pml, s.vti) + 3 * sizeof(float) * (size_t)s.nt * (size_t)s.rn;
}

}  // namespace

struct qvti_server {
    qvti_sched_opts opts{};
    size_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job*> queue;                               // waiting (under mu)
    std::map<long long, std::unique_ptr<Job>> jobs;       // every uncollected ticket (under mu)
    int n_active = 0;                                     // under mu
    size_t pool_bytes = 0;                                // under mu (written by the worker)
    long long next_ticket = 1;
    bool stopping = false;
    // worker-owned
    std::vector<std::unique_ptr<PoolSim>> pool;
    std::vector<Job*> active;
    std::thread worker;

    void loop();
    bool admit_one();
    int start(Job* j, PoolSim* ps);
    void top_up(Job* j);
    void finish(Job* j, int status);
    int cap_for(const Job* j, long long active_cells) const;
    Job* next_waiting() const;
    PoolSim* acquire(const Job* j, bool* blocked);
};

namespace {

void release_events(Job* j)
{
    if (j->ev0) cudaEventDestroy(j->ev0);
    if (j->ev1) cudaEventDestroy(j->ev1);
    for (auto& e : j->chunk)
        if (e) cudaEventDestroy(e);
    j->ev0 = j->ev1 = j->chunk[0] = j->chunk[1] = nullptr;
}

}  // namespace

// Shots in flight allowed while `j` is at the head of the queue.
int qvti_server::cap_for(const Job* j, long long active_cells) const
{
    if (opts.max_active > 0) return opts.max_active;
    // the autotuner measures steady-state stepping; one more slot lets the
    // next shot's host set-up (model upload, reset, graph build) overlap the
    // others' steps instead of leaving the GPU idle between shots
    Tuning t;
    if (cached_tuning({j->shot.ntx, j->shot.nty, j->shot.ntz, j->shot.vti}, &t)) return t.active + 1;
    // untuned grid: bound the cells in flight (always admit onto an idle GPU)
    const long long cells = (long long)j->shot.ntx * j->shot.nty * j->shot.ntz;
    return (active_cells == 0 || active_cells + cells <= kCellsInFlight) ? n_active + 1 : n_active;
}

// An idle pooled simulation for the job's grid, or a new one once idle
// simulations have been freed to make room.  A pooled simulation's bytes are
// its footprint plus the largest record buffers it has held (they only
// grow).  *blocked: the memory is held by shots in flight; retry after one
// finishes.  nullptr without *blocked: creation failed (qvti_last_error).
PoolSim* qvti_server::acquire(const Job* j, bool* blocked)
{
    *blocked = false;
    const GridKey key = key_of(j->shot);
    const size_t need = shot_bytes(j->shot);
    PoolSim* reuse = nullptr;
    for (auto& p : pool)
        if (!p->busy && p->key == key && (!reuse || p->bytes > reuse->bytes)) reuse = p.get();
    const size_t grow = reuse ? (need > reuse->bytes ? need - reuse->bytes : 0) : need;
    size_t held;
    {
        std::lock_guard<std::mutex> lk(mu);
        held = pool_bytes;
    }
    while (held + grow > budget) {
        auto victim = pool.end();
        for (auto it = pool.begin(); it != pool.end(); ++it)
            if (!(*it)->busy && it->get() != reuse &&
                (victim == pool.end() || (*it)->last_used < (*victim)->last_used))
                victim = it;
        if (victim == pool.end()) {
            *blocked = true;
            std::lock_guard<std::mutex> lk(mu);
            pool_bytes = held;  // what was freed so far stays freed
            return nullptr;
        }
        qvti_destroy((*victim)->sim);
        held -= (*victim)->bytes;
        pool.erase(victim);
    }
    if (reuse) {
        reuse->bytes += grow;
        std::lock_guard<std::mutex> lk(mu);
        pool_bytes = held + grow;
        return reuse;
    }
    auto ps = std::make_unique<PoolSim>();
    const qvti_config cfg = config_of(key, opts.device);
    if (cudaHostAlloc(reinterpret_cast<void**>(&ps->nonfinite), sizeof(int), cudaHostAllocDefault) != cudaSuccess ||
        qvti_create(&cfg, &ps->sim) != QVTI_OK) {
        std::lock_guard<std::mutex> lk(mu);
        pool_bytes = held;
        return nullptr;
    }
    ps->key = key;
    ps->bytes = need;
    pool.push_back(std::move(ps));
    {
        std::lock_guard<std::mutex> lk(mu);
        pool_bytes = held + need;
    }
    return pool.back().get();
}

// Upload the shot's model, source and receivers, then queue its first steps.
int qvti_server::start(Job* j, PoolSim* ps)
{
    const qvti_shot& s = j->shot;
    qvti_sim* sim = ps->sim;
    ps->busy = true;
    j->slot = ps;
    int rc;
    Tuning t;
    if (cached_tuning({s.ntx, s.nty, s.ntz, s.vti}, &t)) {
        if ((rc = qvti_set_kz_batch(sim, t.kz_batch))) return rc;
        if ((rc = qvti_set_form(sim, t.form))) return rc;
        if ((rc = qvti_set_tiles(sim, t.tiles))) return rc;
    }
    if ((rc = qvti_set_model(sim, s.velp, s.vels, s.rho, s.gama_p, s.gama_s, s.eps, s.delta, 0))) return rc;
    if ((rc = qvti_set_receivers(sim, s.r_iz, s.r_ix, s.r_iy, s.rn))) return rc;
    if ((rc = qvti_set_source(sim, s.src_type, s.s_ix, s.s_iy, s.s_iz, s.wavelet, s.nt))) return rc;
    if ((rc = qvti_reset(sim))) return rc;
    *ps->nonfinite = 0;
    void* stv = nullptr;
    if ((rc = qvti_get_stream(sim, &stv))) return rc;
    j->st = static_cast<cudaStream_t>(stv);
    if (cudaEventCreate(&j->ev0) != cudaSuccess || cudaEventCreate(&j->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&j->chunk[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&j->chunk[1], cudaEventDisableTiming) != cudaSuccess)
        return QVTI_ERR_CUDA;
    if (cudaEventRecord(j->ev0, j->st) != cudaSuccess) return QVTI_ERR_CUDA;
    j->t_start = now_s();
    j->res.queue_s = j->t_start - j->t_submit;
    top_up(j);
    return QVTI_OK;
}

// Keep at most two chunks of the job's steps queued on its stream.  Each
// chunk ends with the non-finite sentinel; once a finished chunk reports a
// NaN or Inf, no more steps are queued and the shot ends with
// QVTI_ERR_NONFINITE (the other shots in flight are not affected).
void qvti_server::top_up(Job* j)
{
    while (j->enq < j->shot.nt) {
        if (j->nchunk == 2) {
            if (cudaEventQuery(j->chunk[0]) == cudaErrorNotReady) return;
            std::swap(j->chunk[0], j->chunk[1]);
            j->nchunk = 1;
            if (*j->slot->nonfinite) {  // written in stream order before chunk[0]'s event
                j->res.status = QVTI_ERR_NONFINITE;
                j->enq = j->shot.nt;
                break;
            }
        }
        const int n = std::min(kChunk, j->shot.nt - j->enq);
        if (qvti_step(j->slot->sim, n) != QVTI_OK || qvti_check_finite_async(j->slot->sim, j->slot->nonfinite)) {
            j->res.status = qvti_last_error();
            j->enq = j->shot.nt;
            break;
        }
        j->enq += n;
        cudaEventRecord(j->chunk[j->nchunk++], j->st);
    }
    if (j->enq >= j->shot.nt && !j->finished) {
        cudaEventRecord(j->ev1, j->st);
        j->finished = true;  // all steps queued; done once ev1 completes
    }
}

void qvti_server::finish(Job* j, int status)
{
    if (status == QVTI_OK && j->res.status == QVTI_OK) {
        const cudaError_t e = cudaEventSynchronize(j->ev1);
        if (e != cudaSuccess) status = QVTI_ERR_CUDA;
        float ms = 0.f;
        if (status == QVTI_OK && cudaEventElapsedTime(&ms, j->ev0, j->ev1) == cudaSuccess) j->res.device_ms = ms;
        if (status == QVTI_OK && *j->slot->nonfinite) status = QVTI_ERR_NONFINITE;
        if (status == QVTI_OK)
            status = qvti_get_records(j->slot->sim, j->shot.rec_vx, j->shot.rec_vy, j->shot.rec_vz);
    }
    if (j->res.status == QVTI_OK) j->res.status = status;
    release_events(j);
    if (j->slot) {
        j->slot->busy = false;
        j->slot->last_used = now_s();
        if (j->res.status != QVTI_OK) {  // do not reuse a simulation left in an unknown state
            for (auto it = pool.begin(); it != pool.end(); ++it)
                if (it->get() == j->slot) {
                    qvti_destroy((*it)->sim);
                    std::lock_guard<std::mutex> lk(mu);
                    pool_bytes -= (*it)->bytes;
                    pool.erase(it);
                    break;
                }
        }
        j->slot = nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    j->res.latency_s = now_s() - j->t_submit;
    j->ready = true;
    --n_active;
    cv_done.notify_all();
}

// Admit the head of the queue if the slot cap and device memory allow.
// The waiting shot admission considers next (under mu): the head, or with
// QVTI_SCHED_SMALLEST_FIRST the one of fewest cell-steps unless the head
// has been passed kMaxBypass times.
Job* qvti_server::next_waiting() const
{
    Job* head = queue.front();
    if (opts.policy != QVTI_SCHED_SMALLEST_FIRST || head->bypassed >= kMaxBypass) return head;
    auto work = [](const Job* j) { return (double)j->shot.ntx * j->shot.nty * j->shot.ntz * j->shot.nt; };
    Job* best = head;
    for (Job* j : queue)
        if (work(j) < work(best)) best = j;  // strict: ties keep submission order
    return best;
}

bool qvti_server::admit_one()
{
    Job* j;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (queue.empty()) return false;
        j = next_waiting();
        long long cells = 0;
        for (Job* a : active) cells += (long long)a->shot.ntx * a->shot.nty * a->shot.ntz;
        if (n_active >= cap_for(j, cells)) return false;
    }
    bool blocked = false;
    PoolSim* ps = acquire(j, &blocked);
    if (!ps && blocked) return false;
    {
        // submissions only append: j is still queued, and the shots ahead of
        // it have been passed once more
        std::lock_guard<std::mutex> lk(mu);
        for (auto it = queue.begin(); it != queue.end(); ++it) {
            if (*it == j) {
                queue.erase(it);
                break;
            }
            ++(*it)->bypassed;
        }
        ++n_active;
    }
    active.push_back(j);
    int rc = QVTI_ERR_OOM;
    if (ps) rc = start(j, ps);
    else if (qvti_last_error() != QVTI_OK) rc = qvti_last_error();
    if (rc != QVTI_OK) {
        active.pop_back();
        j->res.status = rc;
        finish(j, rc);
    }
    return true;
}

void qvti_server::loop()
{
    cudaSetDevice(opts.device);
    for (;;) {
        // retire finished shots, keep the others fed
        for (size_t i = 0; i < active.size();) {
            Job* j = active[i];
            top_up(j);
            if (j->finished) {
                const cudaError_t q = cudaEventQuery(j->ev1);
                if (q != cudaErrorNotReady) {
                    active.erase(active.begin() + i);
                    finish(j, q == cudaSuccess ? QVTI_OK : QVTI_ERR_CUDA);
                    continue;
                }
            }
            ++i;
        }
        while (admit_one()) {
        }
        std::unique_lock<std::mutex> lk(mu);
        if (stopping && queue.empty() && active.empty()) break;
        if (active.empty() && (queue.empty() || n_active > 0))
            cv_work.wait_for(lk, std::chrono::milliseconds(50));
        else
            cv_work.wait_for(lk, std::chrono::microseconds(100));
    }
    for (auto& p : pool) qvti_destroy(p->sim);
    pool.clear();
    std::lock_guard<std::mutex> lk(mu);
    pool_bytes = 0;
}

extern "C" int qvti_server_create(const qvti_sched_opts* opts, qvti_server** out)
{
    if (!opts || !out || opts->max_active < 0 ||
        (opts->policy != QVTI_SCHED_FIFO && opts->policy != QVTI_SCHED_SMALLEST_FIRST))
        return QVTI_ERR_ARG;
    *out = nullptr;
    if (cudaSetDevice(opts->device) != cudaSuccess) return QVTI_ERR_CUDA;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return QVTI_ERR_CUDA;
    auto* s = new (std::nothrow) qvti_server();
    if (!s) return QVTI_ERR_OOM;
    s->opts = *opts;
    s->budget = opts->mem_budget ? opts->mem_budget : (size_t)(0.9 * (double)free_b);
    s->worker = std::thread([s] { s->loop(); });
    *out = s;
    return QVTI_OK;
}

extern "C" int qvti_server_submit(qvti_server* srv, const qvti_shot* shot, long long* ticket)
{
    if (!srv || !shot || !ticket || shot->nt <= 0 || !shot->wavelet || !shot->velp || !shot->vels || !shot->rho ||
        !shot->gama_p || !shot->gama_s || (shot->vti && (!shot->eps || !shot->delta)) || shot->rn < 0 ||
        (shot->rn > 0 && (!shot->r_ix || !shot->r_iy)))
        return QVTI_ERR_ARG;
    if (shot_bytes(*shot) > srv->budget) return QVTI_ERR_OOM;
    auto j = std::make_unique<Job>();
    j->shot = *shot;
    j->t_submit = now_s();
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->stopping) return QVTI_ERR_STATE;
    j->ticket = srv->next_ticket++;
    *ticket = j->ticket;
    srv->queue.push_back(j.get());
    srv->jobs.emplace(j->ticket, std::move(j));
    srv->cv_work.notify_one();
    return QVTI_OK;
}

extern "C" int qvti_server_wait(qvti_server* srv, long long ticket, double timeout_s, qvti_shot_result* res)
{
    if (!srv || !res) return QVTI_ERR_ARG;
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->jobs.find(ticket);
    if (it == srv->jobs.end()) return QVTI_ERR_ARG;
    Job* j = it->second.get();
    auto ready = [j] { return j->ready; };
    if (timeout_s < 0) {
        srv->cv_done.wait(lk, ready);
    } else if (!srv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
        return QVTI_ERR_TIMEOUT;
    }
    *res = j->res;
    srv->jobs.erase(it);
    return QVTI_OK;
}

extern "C" int qvti_server_load(qvti_server* srv, int* queued, int* active, size_t* pool_bytes)
{
    if (!srv) return QVTI_ERR_ARG;
    std::lock_guard<std::mutex> lk(srv->mu);
    if (queued) *queued = (int)srv->queue.size();
    if (active) *active = srv->n_active;
    if (pool_bytes) *pool_bytes = srv->pool_bytes;
    return QVTI_OK;
}

extern "C" int qvti_server_destroy(qvti_server* srv)
{
    if (!srv) return QVTI_ERR_ARG;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stopping = true;
        srv->cv_work.notify_one();
    }
    if (srv->worker.joinable()) srv->worker.join();
    delete srv;
    return QVTI_OK;
}

extern "C" int qvti_run_batch(const qvti_shot* shots, int n, const qvti_sched_opts* opts, qvti_shot_result* results,
                              double* wall_s)
{
    if (!shots || n < 0 || !opts || !results) return QVTI_ERR_ARG;
    if (opts->max_active == 0) {  // tune every grid of the batch once
        for (int i = 0; i < n; ++i) {
            const ShapeKey k{shots[i].ntx, shots[i].nty, shots[i].ntz, shots[i].vti};
            Tuning t;
            if (cached_tuning(k, &t)) continue;
            const qvti_config cfg = config_of(key_of(shots[i]), opts->device);
            int a = 0, b = 0;
            double g = 0;
            if (qvti_autotune(&cfg, 4, 8, &a, &b, &g) != QVTI_OK) {
                std::lock_guard<std::mutex> lk(g_tune_mu);
                g_tune[k] = {1, (cfg.ntz / 2 + 1), QVTI_FORM_PLAIN};
            }
        }
    }
    qvti_server* srv = nullptr;
    int rc = qvti_server_create(opts, &srv);
    if (rc) return rc;
    const double t0 = now_s();
    std::vector<long long> tickets(n, -1);
    for (int i = 0; i < n; ++i) {
        rc = qvti_server_submit(srv, &shots[i], &tickets[i]);
        if (rc) {
            results[i] = qvti_shot_result{};
            results[i].status = rc;
        }
    }
    for (int i = 0; i < n; ++i)
        if (tickets[i] >= 0) qvti_server_wait(srv, tickets[i], -1.0, &results[i]);
    if (wall_s) *wall_s = now_s() - t0;
    qvti_server_destroy(srv);
    for (int i = 0; i < n; ++i)
        if (results[i].status) return results[i].status;
    return QVTI_OK;
}

// ------------------------------------------------------------- autotuner --
// Probe one grid: first the form of the transforms (the FP32 Stockham stages,
// or the tensor-core DFT plan where the grid has one) with one shot in
// flight, then, in that form, 1..max_active shots in flight for each kz
// batch in {nz/2+1, (nz/2+2)/2}.  A setting must be 2 % faster than the
// simpler one (plain form, fewer shots) to be taken.
extern "C" int qvti_autotune_ex(const qvti_config* cfg, int max_active, int probe_steps, qvti_tuning* best_out)
{
    if (!cfg || max_active < 1 || probe_steps < 1 || !best_out) return QVTI_ERR_ARG;
    if (cudaSetDevice(cfg->device) != cudaSuccess) return QVTI_ERR_CUDA;
    const size_t ntp = (size_t)cfg->ntx * cfg->nty * cfg->ntz;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return QVTI_ERR_CUDA;
    const size_t per = qvti_footprint_bytes(cfg->ntx, cfg->nty, cfg->ntz, cfg->pml, cfg->vti);
    const int fit = (int)std::min<size_t>((size_t)max_active, std::max<size_t>(1, (size_t)(0.8 * free_b) / per));
    // homogeneous probe model (Vp 3000, Vs 1700, rho 2200, Qp 100, Qs 50)
    std::vector<float> vp(ntp, 3000.f), vs(ntp, 1700.f), rho(ntp, 2200.f);
    std::vector<float> gp(ntp, (float)(std::atan(1.0 / 100.0) / 3.1415926)), gs(ntp, (float)(std::atan(1.0 / 50.0) / 3.1415926));
    std::vector<float> eps(cfg->vti ? ntp : 0, 0.1f), dl(cfg->vti ? ntp : 0, 0.05f);
    const int warm = 2;
    const int nt = 2 * (warm + probe_steps);  // the form probe and the concurrency probes
    std::vector<float> wav(nt, 0.f);
    wav[0] = 1.f;
    std::vector<qvti_sim*> sims;
    int rc = QVTI_OK;
    for (int i = 0; i < fit && rc == QVTI_OK; ++i) {
        qvti_sim* s = nullptr;
        if ((rc = qvti_create(cfg, &s))) break;
        sims.push_back(s);
        rc = qvti_set_model(s, vp.data(), vs.data(), rho.data(), gp.data(), gs.data(), cfg->vti ? eps.data() : nullptr,
                            cfg->vti ? dl.data() : nullptr, 0);
        if (!rc) rc = qvti_set_source(s, QVTI_SRC_EXPLOSIVE, cfg->ntx / 2, cfg->nty / 2, cfg->ntz / 2, wav.data(), nt);
    }
    if (sims.empty()) return rc ? rc : QVTI_ERR_OOM;
    const int nkz = cfg->ntz / 2 + 1;
    // steps per second of `c` simulations, each running `steps` after a reset and `warm` steps
    auto probe = [&](int c, int b, int form, double* rate) -> int {
        for (int i = 0; i < c; ++i) {
            int r;
            if ((r = qvti_set_kz_batch(sims[i], b)) || (r = qvti_set_form(sims[i], form)) || (r = qvti_reset(sims[i])) ||
                (r = qvti_step(sims[i], warm)))
                return r;
        }
        if (cudaDeviceSynchronize() != cudaSuccess) return QVTI_ERR_CUDA;
        const double t0 = now_s();
        for (int i = 0; i < c; ++i)
            if (int r = qvti_step(sims[i], probe_steps)) return r;
        if (cudaDeviceSynchronize() != cudaSuccess) return QVTI_ERR_CUDA;
        *rate = (double)c * ntp * probe_steps / (now_s() - t0) / 1e9;
        return QVTI_OK;
    };
    double best = -1;
    int ba = 1, bb = nkz, bf = QVTI_FORM_PLAIN;
    int tiles[QVTI_NUM_TILES] = {};
    // 1. the form, one shot in flight, all kz planes at once
    double r_plain = 0, r_tc = 0;
    rc = probe(1, nkz, QVTI_FORM_PLAIN, &r_plain);
    if (!rc && qvti_set_form(sims[0], QVTI_FORM_TC) == QVTI_OK) {
        rc = probe(1, nkz, QVTI_FORM_TC, &r_tc);
        if (!rc && r_tc > r_plain * 1.02) bf = QVTI_FORM_TC;
    }
    // 2. per-kernel tiles in that form, applied to every probe simulation
    if (!rc && !(rc = qvti_set_form(sims[0], bf)) && !(rc = qvti_set_kz_batch(sims[0], nkz)))
        rc = qvti_autotune_tiles(sims[0], probe_steps, tiles, nullptr);
    for (size_t i = 0; i < sims.size() && rc == QVTI_OK; ++i) rc = qvti_set_tiles(sims[i], tiles);
    // 3. shots in flight and kz batching in that form
    const int kzb[2] = {nkz, (nkz + 1) / 2};
    for (int b : kzb) {
        for (int c = 1; c <= (int)sims.size() && rc == QVTI_OK; ++c) {
            double rate = 0;
            if ((rc = probe(c, b, bf, &rate))) break;
            if (rate > best * 1.02) {  // prefer fewer shots in flight unless clearly faster
                best = rate;
                ba = c;
                bb = b;
            }
        }
        if (rc || b == kzb[1] || kzb[0] == kzb[1]) break;
    }
    for (qvti_sim* s : sims) qvti_destroy(s);
    if (rc) return rc;
    best_out->active = ba;
    best_out->kz_batch = bb;
    best_out->form = bf;
    best_out->gcell_steps = best;
    Tuning t{ba, bb, bf, {}};
    for (int i = 0; i < QVTI_NUM_TILES; ++i) best_out->tiles[i] = t.tiles[i] = tiles[i];
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[{cfg->ntx, cfg->nty, cfg->ntz, cfg->vti}] = t;
    return QVTI_OK;
}

extern "C" int qvti_autotune(const qvti_config* cfg, int max_active, int probe_steps, int* best_active,
                             int* best_kz_batch, double* gcell_steps)
{
    if (!best_active || !best_kz_batch || !gcell_steps) return QVTI_ERR_ARG;
    qvti_tuning t{};
    const int rc = qvti_autotune_ex(cfg, max_active, probe_steps, &t);
    if (rc) return rc;
    *best_active = t.active;
    *best_kz_batch = t.kz_batch;
    *gcell_steps = t.gcell_steps;
    return QVTI_OK;
}
