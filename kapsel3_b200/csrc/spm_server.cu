// Serving loop: a persistent worker thread that admits independent SPM runs
// by device-memory budget, keeps their state resident in per-grid pools
// (spm_pool_*), advances every pool continuously (one graph replay per pool
// step, pools of different grids on their own streams so they overlap on the
// GPU), retires runs when they reach their step count and records per-step
// latency.  Host code only; it drives the GPU through the library's C ABI.
//
// Request life cycle: QUEUED -> RUNNING -> DONE | FAILED | CANCELLED.  A
// request is admitted when its pool has a free run slot (or can grow) and the
// bytes it adds fit the budget; requests that do not fit yet stay queued
// while later ones that fit are admitted.  A request that could not fit even
// on an idle GPU is rejected at submission.
#include <algorithm>
#include <atomic>
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

#include <cuda_runtime.h>

#include "../../include/kapsel_spm.h"

int spm_internal_fail(int code, const char *msg);

namespace {

using Clock = std::chrono::steady_clock;
double now_s() { return std::chrono::duration<double>(Clock::now().time_since_epoch()).count(); }

struct Request {
    long long           id = 0;
    spm_params          p{};
    std::vector<double> particles;
    int                 nsteps = 0;
    int                 flags  = 0;
    int                 state  = SPM_REQ_QUEUED;
    int                 status = SPM_OK;
    std::string         message;
    std::atomic<bool>   cancel{false};
    size_t              run_bytes = 0;
    // while running
    spm_ctx *run        = nullptr;
    int      pool_index = -1;
    int      steps_done = 0;
    double   t_submit = 0, t_admit = 0, t_last = 0, t_done = 0;
    // results
    std::vector<double> out_particles, out_u;
    double              out_time = 0.0;
};

struct PoolEntry {
    spm_params             key{};
    spm_pool              *pool  = nullptr;
    size_t                 arena = 0;  // bytes of the current arena
    std::vector<Request *> members;    // members[r] runs in run slot r
    bool                   inflight = false;
    int                    steps_inflight = 0;
    double                 t_launch = 0.0;
    double                 t_empty  = 0.0;  // when the pool last became empty (0: has members)
};

bool same_key(const spm_params &a, const spm_params &b) {
    return a.npx == b.npx && a.npy == b.npy && a.npz == b.npz && a.precision == b.precision && a.dx == b.dx &&
           a.equation == b.equation;
}

double percentile(std::vector<float> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i   = (size_t)pos;
    const double f   = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

struct spm_server {
    spm_server_config cfg{};
    int               device = 0;
    std::thread       worker;
    std::mutex        mu;
    std::condition_variable cv_done;  // request state changes
    std::condition_variable cv_work;  // new submissions / stop
    bool              stop = false;
    long long         next_id = 1;
    std::deque<Request *>                        queue;
    std::map<long long, std::unique_ptr<Request>> all;
    std::vector<std::unique_ptr<PoolEntry>>      pools;  // worker thread only
    size_t            used = 0, peak = 0;
    // statistics (under mu)
    std::vector<float> lat_ms;      // one sample per run step
    std::vector<float> pool_dev_ms; // device time per pool step
    long long submitted = 0, rejected = 0, admitted = 0, completed = 0, failed = 0, cancelled = 0;
    long long run_steps = 0, captures = 0;
    int       max_active = 0;
    double    t_first_admit = 0.0, t_last_done = 0.0;
    // longest host phases of the worker (ms)
    double    create_max = 0, admit_max = 0, destroy_max = 0, launch_max = 0, finish_max = 0;
    std::string worker_error;
    void phase(double &mx, double t0) {
        const double ms = (now_s() - t0) * 1e3;
        std::lock_guard<std::mutex> lk(mu);
        mx = std::max(mx, ms);
    }

    void set_state(Request *q, int state, int status, const std::string &msg) {
        q->state   = state;
        q->status  = status;
        q->message = msg;
        q->t_done  = now_s();
        cv_done.notify_all();
    }
    size_t arena_bytes(const spm_params &p, int cap) {
        size_t a = 0, r = 0;
        spm_pool_device_bytes(&p, cap, &a, &r);
        return a;
    }
    void loop();
    bool admit_some();
    void finish_pool_steps(PoolEntry *pe);
    void finish_pool_steps_impl(PoolEntry *pe);
    void retire(PoolEntry *pe, Request *q, int state, int status, const std::string &msg);
    void launch(PoolEntry *pe);
};

// Releases a member from its pool (the pool moves its last run into the
// freed slot, so the member list is permuted the same way).
void spm_server::retire(PoolEntry *pe, Request *q, int state, int status, const std::string &msg) {
    auto it = std::find(pe->members.begin(), pe->members.end(), q);
    if (it == pe->members.end()) return;
    const size_t r = (size_t)(it - pe->members.begin());
    spm_pool_release(pe->pool, q->run);
    pe->members[r] = pe->members.back();
    pe->members.pop_back();
    q->run = nullptr;
    std::lock_guard<std::mutex> lk(mu);
    used -= q->run_bytes;
    if (state == SPM_REQ_DONE) completed++;
    if (state == SPM_REQ_FAILED) failed++;
    if (state == SPM_REQ_CANCELLED) cancelled++;
    t_last_done = now_s();
    set_state(q, state, status, msg);
}

// Accounts the steps a pool just finished: per-step latency samples, errors,
// retirement of runs that reached their step count or were cancelled.
void spm_server::finish_pool_steps(PoolEntry *pe) {
    const double t_phase = now_s();
    finish_pool_steps_impl(pe);
    phase(finish_max, t_phase);
}
void spm_server::finish_pool_steps_impl(PoolEntry *pe) {
    const int n = (int)pe->members.size();
    std::vector<unsigned int> errs(n, 0u);
    float       dev_ms = 0.f;
    const int   rc     = spm_pool_synchronize(pe->pool, &dev_ms, errs.data());
    const double t     = now_s();
    const int   k      = pe->steps_inflight;
    pe->inflight       = false;
    pe->steps_inflight = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (k > 0) pool_dev_ms.push_back(dev_ms / (float)k);
        for (Request *q : pe->members) {
            const float per = (float)((t - q->t_last) * 1000.0 / std::max(k, 1));
            for (int i = 0; i < k; i++) lat_ms.push_back(per);
            q->t_last = t;
            q->steps_done += k;
            run_steps += k;
        }
    }
    std::vector<Request *> snapshot = pe->members;
    for (int r = 0; r < n; r++) {
        Request *q = snapshot[r];
        if (rc != SPM_OK) {
            retire(pe, q, SPM_REQ_FAILED, rc, std::string("pool step: ") + spm_last_error());
        } else if (errs[r]) {
            retire(pe, q, SPM_REQ_FAILED, SPM_ERR_DEVICE,
                   "device error bits " + std::to_string(errs[r]) + " (particle left the box / LJ overflow / NaN)");
        } else if (q->cancel) {
            retire(pe, q, SPM_REQ_CANCELLED, SPM_OK, "cancelled");
        } else if (q->steps_done >= q->nsteps) {
            int s = SPM_OK;
            q->out_particles.assign((size_t)std::max(q->p.n_particles, 0) * SPM_PARTICLE_WORDS, 0.0);
            if (q->p.n_particles > 0) s = spm_get_particles(q->run, q->out_particles.data());
            if (s == SPM_OK && (q->flags & SPM_REQ_KEEP_VELOCITY)) {
                const size_t nf = (size_t)(1 << q->p.npx) * (1 << q->p.npy) * 2 * ((1 << q->p.npz) / 2 + 1);
                q->out_u.assign(3 * nf, 0.0);
                s = spm_get_velocity(q->run, q->out_u.data(), q->out_u.data() + nf, q->out_u.data() + 2 * nf);
            }
            int ts = 0;
            spm_get_time(q->run, &ts, &q->out_time);
            if (s != SPM_OK)
                retire(pe, q, SPM_REQ_FAILED, s, std::string("result download: ") + spm_last_error());
            else
                retire(pe, q, SPM_REQ_DONE, SPM_OK, "");
        }
    }
}

void spm_server::launch(PoolEntry *pe) {
    if (pe->members.empty()) return;
    int k = cfg.steps_per_launch > 0 ? cfg.steps_per_launch : 1;
    for (Request *q : pe->members) k = std::min(k, q->nsteps - q->steps_done);
    if (k <= 0) k = 1;
    const double t_phase = now_s();
    const int    rc      = spm_pool_step(pe->pool, k, cfg.use_graph);
    phase(launch_max, t_phase);
    if (rc != SPM_OK) {
        const std::string msg = std::string("pool step launch: ") + spm_last_error();
        std::vector<Request *> snapshot = pe->members;
        for (Request *q : snapshot) retire(pe, q, SPM_REQ_FAILED, rc, msg);
        return;
    }
    pe->inflight       = true;
    pe->steps_inflight = k;
    pe->t_launch       = now_s();
}

// Admits queued requests that fit; returns true if any was admitted.
bool spm_server::admit_some() {
    bool any = false;
    for (;;) {
        Request   *q      = nullptr;
        PoolEntry *target = nullptr;
        int        grow_to = 0;
        {
            std::lock_guard<std::mutex> lk(mu);
            for (auto it = queue.begin(); it != queue.end();) {
                if ((*it)->cancel) {
                    cancelled++;
                    set_state(*it, SPM_REQ_CANCELLED, SPM_OK, "cancelled before admission");
                    it = queue.erase(it);
                } else {
                    ++it;
                }
            }
            for (auto it = queue.begin(); it != queue.end(); ++it) {
                Request   *c  = *it;
                PoolEntry *pe = nullptr;
                for (auto &p : pools)
                    if (same_key(p->key, c->p)) pe = p.get();
                int    cap = 0;
                size_t add = c->run_bytes;
                if (!pe) {
                    cap = std::max(cfg.pool_initial_capacity, 1);
                    add += arena_bytes(c->p, cap);
                } else {
                    if (pe->inflight) continue;  // membership changes only between steps
                    int runs = 0, pcap = 0;
                    spm_pool_size(pe->pool, &runs, &pcap);
                    if (runs == pcap) add += arena_bytes(c->p, 2 * pcap);  // old and new arena coexist while growing
                }
                if (used + add <= cfg.budget_bytes) {
                    q       = c;
                    target  = pe;
                    grow_to = cap;
                    queue.erase(it);
                    break;
                }
            }
        }
        if (!q) return any;
        // create the pool if needed
        int rc = SPM_OK;
        if (!target) {
            spm_pool    *pl = nullptr;
            const double t_phase = now_s();
            rc           = spm_pool_create(&q->p, grow_to, nullptr, &pl);
            phase(create_max, t_phase);
            if (rc == SPM_OK) {
                auto pe   = std::make_unique<PoolEntry>();
                pe->key   = q->p;
                pe->pool  = pl;
                pe->arena = arena_bytes(q->p, grow_to);
                target    = pe.get();
                pools.push_back(std::move(pe));
                std::lock_guard<std::mutex> lk(mu);
                used += target->arena;
            }
        }
        spm_ctx *run = nullptr;
        if (rc == SPM_OK) {
            int cap_before = 0, cap_after = 0;
            spm_pool_size(target->pool, nullptr, &cap_before);
            const double t_phase = now_s();
            rc = spm_pool_admit(target->pool, &q->p, q->particles.empty() ? nullptr : q->particles.data(), &run);
            phase(admit_max, t_phase);
            spm_pool_size(target->pool, nullptr, &cap_after);
            if (cap_after != cap_before) {
                std::lock_guard<std::mutex> lk(mu);
                const size_t a = arena_bytes(q->p, cap_after);
                used           = used - target->arena + a;
                target->arena  = a;
            }
        }
        std::lock_guard<std::mutex> lk(mu);
        if (rc != SPM_OK) {
            failed++;
            set_state(q, SPM_REQ_FAILED, rc, std::string("admission: ") + spm_last_error());
            continue;
        }
        used += q->run_bytes;
        peak = std::max(peak, used);
        q->run     = run;
        q->t_admit = q->t_last = now_s();
        if (admitted == 0) t_first_admit = q->t_admit;
        admitted++;
        q->state = SPM_REQ_RUNNING;
        target->members.push_back(q);
        int active = 0;
        for (auto &p : pools) active += (int)p->members.size();
        max_active = std::max(max_active, active);
        any        = true;
        cv_done.notify_all();
    }
}

void spm_server::loop() {
    cudaSetDevice(device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu);
            bool active = false;
            for (auto &p : pools) active = active || !p->members.empty();
            if (stop && !active) break;
            if (!active && queue.empty()) {
                cv_work.wait(lk, [&] { return stop || !queue.empty(); });
                if (stop && queue.empty()) break;
            }
        }
        // finished steps, retirements
        bool progressed = false;
        for (auto &pe : pools) {
            if (!pe->inflight) continue;
            int done = 0;
            if (spm_pool_query(pe->pool, &done) != SPM_OK) done = 1;
            if (done) {
                finish_pool_steps(pe.get());
                progressed = true;
            }
        }
        // stop requested: cancel everything still running or queued
        {
            std::lock_guard<std::mutex> lk(mu);
            if (stop)
                for (auto &pe : pools)
                    for (Request *q : pe->members) q->cancel = true;
            if (stop)
                for (Request *q : queue) q->cancel = true;
        }
        // idle pools with cancelled members: release them now
        for (auto &pe : pools) {
            if (pe->inflight) continue;
            std::vector<Request *> snapshot = pe->members;
            for (Request *q : snapshot)
                if (q->cancel) retire(pe.get(), q, SPM_REQ_CANCELLED, SPM_OK, "cancelled");
        }
        if (admit_some()) progressed = true;
        // Drop pools that stayed empty for pool_idle_s, or at once when a
        // queued request is waiting: freeing an arena waits for the whole
        // device, so a pool that empties and refills within a moment keeps it.
        bool waiting = false;
        {
            std::lock_guard<std::mutex> lk(mu);
            waiting = !queue.empty();
        }
        const double tnow = now_s();
        for (size_t i = 0; i < pools.size();) {
            PoolEntry *pe = pools[i].get();
            if (!pe->members.empty()) pe->t_empty = 0.0;
            if (pe->members.empty() && !pe->inflight && pe->t_empty == 0.0) pe->t_empty = tnow;
            const bool idle_long = pe->t_empty > 0.0 && tnow - pe->t_empty >= cfg.pool_idle_s;
            if (pe->members.empty() && !pe->inflight && (idle_long || waiting || stop)) {
                long long k = 0;
                int       cnt = 0;
                spm_pool_stats(pe->pool, &k, &cnt);
                const double t_phase = now_s();
                spm_pool_destroy(pe->pool);
                phase(destroy_max, t_phase);
                std::lock_guard<std::mutex> lk(mu);
                captures += cnt;
                used -= pe->arena;
                pools.erase(pools.begin() + (long)i);
            } else {
                i++;
            }
        }
        for (auto &pe : pools)
            if (!pe->inflight && !pe->members.empty()) {
                launch(pe.get());
                progressed = true;
            }
        if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(cfg.poll_us > 0 ? cfg.poll_us : 20));
    }
    for (auto &pe : pools) {
        long long k = 0;
        int       cnt = 0;
        spm_pool_stats(pe->pool, &k, &cnt);
        spm_pool_destroy(pe->pool);
        std::lock_guard<std::mutex> lk(mu);
        captures += cnt;
    }
    pools.clear();
    std::lock_guard<std::mutex> lk(mu);
    for (Request *q : queue) {
        cancelled++;
        set_state(q, SPM_REQ_CANCELLED, SPM_OK, "server stopped");
    }
    queue.clear();
}

extern "C" {

int spm_server_config_default(spm_server_config *c) {
    if (!c) return spm_internal_fail(SPM_ERR_ARG, "null config");
    std::memset(c, 0, sizeof(*c));
    c->budget_bytes          = (size_t)150 << 30;
    c->pool_initial_capacity = 8;
    c->use_graph             = 1;
    c->steps_per_launch      = 1;
    c->poll_us               = 20;
    c->pool_idle_s           = 2.0;
    c->device                = 0;
    return SPM_OK;
}

int spm_server_create(const spm_server_config *cfg, spm_server **out) {
    if (!out) return spm_internal_fail(SPM_ERR_ARG, "null argument");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return spm_internal_fail(SPM_ERR_NO_DEVICE, "no CUDA device visible");
    spm_server *s = new spm_server();
    if (cfg)
        s->cfg = *cfg;
    else
        spm_server_config_default(&s->cfg);
    if (s->cfg.device < 0 || s->cfg.device >= n) {
        delete s;
        return spm_internal_fail(SPM_ERR_ARG, "device index out of range");
    }
    s->device = s->cfg.device;
    s->worker = std::thread([s] { s->loop(); });
    *out      = s;
    return SPM_OK;
}

int spm_server_destroy(spm_server *s) {
    if (!s) return SPM_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    delete s;
    return SPM_OK;
}

int spm_server_submit(spm_server *s, const spm_params *p, const double *particles, int nsteps, int flags,
                      long long *id) {
    if (!s || !p || !id || nsteps < 1) return spm_internal_fail(SPM_ERR_ARG, "bad argument");
    *id = 0;
    if (p->equation != SPM_EQ_NAVIER_STOKES) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->rejected++;
        return spm_internal_fail(SPM_ERR_ARG, "the server runs Navier_Stokes requests");
    }
    size_t arena = 0, run = 0;
    int    rc    = spm_pool_device_bytes(p, 1, &arena, &run);
    if (rc != SPM_OK) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->rejected++;
        return rc;
    }
    if (arena + run > s->cfg.budget_bytes) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->rejected++;
        return spm_internal_fail(SPM_ERR_NOMEM, "request exceeds the device-memory budget");
    }
    auto q = std::make_unique<Request>();
    q->p         = *p;
    q->nsteps    = nsteps;
    q->flags     = flags;
    q->run_bytes = run;
    if (p->n_particles > 0) {
        if (!particles) return spm_internal_fail(SPM_ERR_ARG, "particle records required");
        q->particles.assign(particles, particles + (size_t)p->n_particles * SPM_PARTICLE_WORDS);
        const double L[3] = {(double)(1 << p->npx) * p->dx, (double)(1 << p->npy) * p->dx, (double)(1 << p->npz) * p->dx};
        for (int i = 0; i < p->n_particles; i++)
            for (int d = 0; d < 3; d++) {
                const double x = q->particles[(size_t)i * SPM_PARTICLE_WORDS + d];
                if (!(x >= 0.0 && x < L[d])) {
                    std::lock_guard<std::mutex> lk(s->mu);
                    s->rejected++;
                    return spm_internal_fail(SPM_ERR_ARG, "particle position outside the periodic box");
                }
            }
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return spm_internal_fail(SPM_ERR_ARG, "server is stopping");
    q->id       = s->next_id++;
    q->t_submit = now_s();
    *id         = q->id;
    s->queue.push_back(q.get());
    s->all[q->id] = std::move(q);
    s->submitted++;
    s->cv_work.notify_all();
    return SPM_OK;
}

int spm_server_cancel(spm_server *s, long long id) {
    if (!s) return spm_internal_fail(SPM_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return spm_internal_fail(SPM_ERR_ARG, "unknown request");
    it->second->cancel = true;
    s->cv_work.notify_all();
    return SPM_OK;
}

int spm_server_wait(spm_server *s, long long id, double timeout_s, int *state) {
    if (!s || !state) return spm_internal_fail(SPM_ERR_ARG, "bad argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return spm_internal_fail(SPM_ERR_ARG, "unknown request");
    Request *q    = it->second.get();
    auto     done = [&] { return q->state >= SPM_REQ_DONE; };
    if (timeout_s < 0)
        s->cv_done.wait(lk, done);
    else
        s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
    *state = q->state;
    return SPM_OK;
}

int spm_server_status(spm_server *s, long long id, int *state, int *status, int *steps_done, char *message,
                      size_t message_len) {
    if (!s) return spm_internal_fail(SPM_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return spm_internal_fail(SPM_ERR_ARG, "unknown request");
    Request *q = it->second.get();
    if (state) *state = q->state;
    if (status) *status = q->status;
    if (steps_done) *steps_done = q->steps_done;
    if (message && message_len) {
        std::strncpy(message, q->message.c_str(), message_len - 1);
        message[message_len - 1] = 0;
    }
    return SPM_OK;
}

int spm_server_result(spm_server *s, long long id, double *particles, double *u0, double *u1, double *u2,
                      double *time, double *latency_s) {
    if (!s) return spm_internal_fail(SPM_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return spm_internal_fail(SPM_ERR_ARG, "unknown request");
    Request *q = it->second.get();
    if (q->state != SPM_REQ_DONE) return spm_internal_fail(SPM_ERR_ARG, "request has no result");
    if (particles && !q->out_particles.empty())
        std::memcpy(particles, q->out_particles.data(), q->out_particles.size() * sizeof(double));
    if (u0 || u1 || u2) {
        if (q->out_u.empty()) return spm_internal_fail(SPM_ERR_ARG, "velocity was not kept (SPM_REQ_KEEP_VELOCITY)");
        const size_t nf = q->out_u.size() / 3;
        if (u0) std::memcpy(u0, q->out_u.data(), nf * sizeof(double));
        if (u1) std::memcpy(u1, q->out_u.data() + nf, nf * sizeof(double));
        if (u2) std::memcpy(u2, q->out_u.data() + 2 * nf, nf * sizeof(double));
    }
    if (time) *time = q->out_time;
    if (latency_s) *latency_s = q->t_done - q->t_submit;
    return SPM_OK;
}

int spm_server_forget(spm_server *s, long long id) {
    if (!s) return spm_internal_fail(SPM_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return spm_internal_fail(SPM_ERR_ARG, "unknown request");
    if (it->second->state < SPM_REQ_DONE) return spm_internal_fail(SPM_ERR_ARG, "request still active");
    s->all.erase(it);
    return SPM_OK;
}

int spm_server_get_stats(spm_server *s, spm_server_stats *st) {
    if (!s || !st) return spm_internal_fail(SPM_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(st, 0, sizeof(*st));
    st->submitted   = s->submitted;
    st->rejected    = s->rejected;
    st->admitted    = s->admitted;
    st->completed   = s->completed;
    st->failed      = s->failed;
    st->cancelled   = s->cancelled;
    st->queued      = (long long)s->queue.size();
    st->run_steps   = s->run_steps;
    st->max_active  = s->max_active;
    st->graph_captures = s->captures;
    st->used_bytes  = s->used;
    st->peak_bytes  = s->peak;
    st->busy_s      = s->t_last_done > s->t_first_admit ? s->t_last_done - s->t_first_admit : 0.0;
    st->step_latency_p50_ms = percentile(s->lat_ms, 0.50);
    st->step_latency_p99_ms = percentile(s->lat_ms, 0.99);
    st->step_latency_max_ms = s->lat_ms.empty() ? 0.0 : *std::max_element(s->lat_ms.begin(), s->lat_ms.end());
    st->pool_step_device_p50_ms = percentile(s->pool_dev_ms, 0.50);
    st->pool_step_device_p99_ms = percentile(s->pool_dev_ms, 0.99);
    st->pool_create_max_ms      = s->create_max;
    st->admit_max_ms            = s->admit_max;
    st->pool_destroy_max_ms     = s->destroy_max;
    st->launch_max_ms           = s->launch_max;
    st->finish_max_ms           = s->finish_max;
    return SPM_OK;
}

// Copies up to `cap` per-step latency samples (ms); n = total samples.
int spm_server_latencies(spm_server *s, float *out, size_t cap, size_t *n) {
    if (!s || !n) return spm_internal_fail(SPM_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *n = s->lat_ms.size();
    if (out) std::memcpy(out, s->lat_ms.data(), std::min(cap, s->lat_ms.size()) * sizeof(float));
    return SPM_OK;
}

}  // extern "C"
