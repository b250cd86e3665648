// server.cu — served mode: a request loop that admits simulation jobs as they
// arrive, keeps their state resident on the GPU and advances every resident
// job together through one soil_batch (continuous batching).
//
// One host thread (the loop) owns all GPU work of the server's context.  API
// calls from other threads only touch the queue and the job records, under
// one mutex.  Per loop iteration:
//   1. admit queued jobs, first come first served, while the HBM reservation
//      (a per-atom estimate plus a fixed part per job) fits the budget and a
//      slot is free; each admitted job becomes a set-up soil_sys in the batch;
//   2. advance the batch by q steps, q = min(quantum, fewest steps any
//      resident job still needs), so no job runs past its own step count (a
//      lone resident job steps through the single-system path instead);
//   3. retire finished (or cancelled) jobs: read back their final state, leave
//      the batch, free their memory and reservation, wake their waiters.
// A job's trajectory depends only on its own inputs and step count: the
// batch computes every member exactly as soil_step would alone.
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

#include "sys_internal.cuh"

namespace {

using Clock = std::chrono::steady_clock;

// SOIL_SERVE_SOLO=0 keeps a lone resident job in the batch engine.
bool solo_steps() {
    static const bool on = [] {
        const char* env = std::getenv("SOIL_SERVE_SOLO");
        return !(env && std::atoi(env) == 0);
    }();
    return on;
}

struct Job {
    uint64_t id = 0;
    int32_t state = SOIL_JOB_QUEUED;
    std::string error;
    // inputs (copied at submit)
    soil_box box{};
    soil_neigh_cfg cfg{};
    double dt = 0.0, harmonic_k = 0.0, shear_rate = 0.0;
    uint64_t natoms = 0, steps = 0, steps_done = 0;
    std::vector<uint32_t> tag;
    std::vector<double> pos, vel, mass, cutoff, radius;
    // while resident
    soil_sys* sys = nullptr;
    uint64_t reserved = 0;
    bool cancel = false;
    // results
    std::vector<uint32_t> out_tag;
    std::vector<double> out_pos, out_vel;
    std::vector<int32_t> out_img;
    double t_submit = 0.0, t_admit = -1.0, t_done = -1.0;
};

}  // namespace

struct soil_server {
    soil_ctx* ctx = nullptr;
    soil_server_cfg cfg{};
    soil_batch* batch = nullptr;
    Clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_loop, cv_done;
    std::deque<uint64_t> queue;
    std::map<uint64_t, std::unique_ptr<Job>> jobs;
    std::vector<Job*> active;  // loop thread only
    uint64_t next_id = 1;
    uint64_t reserved = 0;
    bool stop = false;
    std::thread loop;
    // statistics (under mu)
    uint64_t admitted = 0, completed = 0, failed = 0, atom_steps = 0, batch_steps = 0;
    double busy_s = 0.0;
    int32_t max_active_seen = 0;
};

namespace {

double now_s(const soil_server* sv) {
    return std::chrono::duration<double>(Clock::now() - sv->t0).count();
}

uint64_t reservation_of(const soil_server* sv, uint64_t natoms) {
    return natoms * (uint64_t)sv->cfg.bytes_per_atom + sv->cfg.bytes_per_job;
}

std::string last_error(soil_ctx* ctx) {
    const char* e = soil_last_error(ctx);
    return e ? std::string(e) : std::string();
}

// Builds the job's system and adds it to the batch (loop thread).
int create_system(soil_server* sv, Job* j) {
    soil_sys* s = nullptr;
    int st = soil_sys_create(sv->ctx, &j->box, &j->cfg, j->dt, &s);
    if (st != SOIL_OK) return st;
    int32_t rc = -1;
    const double* cols[1] = {j->radius.data()};
    if ((st = soil_sys_register_column(s, "radius", 1, SOIL_COL_FORWARD, &rc)) != SOIL_OK ||
        (st = soil_sys_add_atoms(s, j->natoms, j->tag.data(), nullptr, j->pos.data(),
                                 j->vel.data(), j->mass.data(), j->cutoff.data(), cols)) !=
            SOIL_OK ||
        (st = soil_sys_set_harmonic(s, j->harmonic_k, rc)) != SOIL_OK ||
        (j->shear_rate != 0.0 && (st = soil_sys_set_shear(s, j->shear_rate)) != SOIL_OK) ||
        (st = soil_sys_setup(s)) != SOIL_OK || (st = soil_batch_add(sv->batch, s)) != SOIL_OK) {
        soil_sys_destroy(s);
        return st;
    }
    j->sys = s;
    return SOIL_OK;
}

// Reads the final local state back, leaves the batch and frees the system.
int retire_system(soil_server* sv, Job* j, bool keep_results) {
    int st = SOIL_OK;
    if (keep_results) {
        soil_counts c;
        st = soil_sys_counts(j->sys, &c);
        if (st == SOIL_OK) {
            const uint64_t n = c.nlocal;
            j->out_tag.resize(n);
            j->out_pos.resize(3 * n);
            j->out_vel.resize(3 * n);
            j->out_img.resize(3 * n);
            st = soil_sys_get_atoms(j->sys, 0, n, j->out_tag.data(), j->out_pos.data(),
                                    j->out_vel.data(), nullptr, j->out_img.data(), nullptr);
        }
    }
    soil_batch_remove(sv->batch, j->sys);
    soil_sys_destroy(j->sys);
    j->sys = nullptr;
    return st;
}

void finish(soil_server* sv, Job* j, int32_t state, const std::string& err) {
    std::lock_guard<std::mutex> g(sv->mu);
    j->state = state;
    j->error = err;
    j->t_done = now_s(sv);
    sv->reserved -= j->reserved;
    j->reserved = 0;
    if (state == SOIL_JOB_DONE) sv->completed += 1;
    else sv->failed += 1;
    j->tag.clear();
    j->tag.shrink_to_fit();
    j->pos = std::vector<double>();
    j->vel = std::vector<double>();
    j->mass = std::vector<double>();
    j->cutoff = std::vector<double>();
    j->radius = std::vector<double>();
    sv->cv_done.notify_all();
}

void run_loop(soil_server* sv) {
    cudaSetDevice(sv->ctx->device);
    for (;;) {
        // ---- admission ----
        std::vector<Job*> admit;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            if (sv->active.empty())
                sv->cv_loop.wait(lk, [&] { return sv->stop || !sv->queue.empty(); });
            if (sv->stop) break;
            while (!sv->queue.empty()) {
                Job* j = sv->jobs[sv->queue.front()].get();
                if (j->cancel) {  // cancelled while queued
                    sv->queue.pop_front();
                    j->state = SOIL_JOB_CANCELLED;
                    j->t_done = now_s(sv);
                    sv->failed += 1;
                    sv->cv_done.notify_all();
                    continue;
                }
                const uint64_t need = reservation_of(sv, j->natoms);
                const bool room = sv->active.size() + admit.size() < sv->cfg.max_active;
                const bool fits = sv->reserved + need <= sv->cfg.hbm_budget_bytes;
                // a job larger than the whole budget is admitted alone
                const bool alone = sv->active.empty() && admit.empty();
                if (!room || !(fits || alone)) break;
                sv->queue.pop_front();
                sv->reserved += need;
                j->reserved = need;
                j->state = SOIL_JOB_RUNNING;
                j->t_admit = now_s(sv);
                sv->admitted += 1;
                admit.push_back(j);
            }
        }
        for (Job* j : admit) {
            const int st = create_system(sv, j);
            if (st != SOIL_OK) {
                finish(sv, j, SOIL_JOB_FAILED, last_error(sv->ctx));
                continue;
            }
            sv->active.push_back(j);
        }
        {
            std::lock_guard<std::mutex> g(sv->mu);
            sv->max_active_seen = std::max<int32_t>(sv->max_active_seen, (int32_t)sv->active.size());
        }
        if (sv->active.empty()) continue;

        // ---- advance every resident job ----
        uint64_t q = sv->cfg.quantum_steps;
        uint64_t natoms = 0;
        for (Job* j : sv->active) {
            q = std::min(q, j->steps - j->steps_done);
            natoms += j->natoms;
        }
        const auto tb = Clock::now();
        int st = SOIL_OK;
        if (q > 0 && sv->active.size() == 1 && solo_steps()) {
            // A lone job gains nothing from the batch (no launches to share)
            // and the single-system path is faster for one box: it leaves the
            // batch for these q steps and joins it again for the next
            // admission point.  The trajectory is the same either way.
            soil_sys* s = sv->active[0]->sys;
            st = soil_batch_remove(sv->batch, s);
            if (st == SOIL_OK) st = soil_step(s, q);
            if (st == SOIL_OK) st = soil_sys_sync(s);
            const int back = soil_batch_add(sv->batch, s);
            if (st == SOIL_OK) st = back;
        } else if (q > 0) {
            st = soil_batch_step(sv->batch, q);
        }
        if (st == SOIL_OK) st = soil_batch_sync(sv->batch);
        const double dtb = std::chrono::duration<double>(Clock::now() - tb).count();
        if (st != SOIL_OK) {
            const std::string err = last_error(sv->ctx);
            for (Job* j : sv->active) {
                retire_system(sv, j, false);
                finish(sv, j, SOIL_JOB_FAILED, err);
            }
            sv->active.clear();
            continue;
        }
        {
            std::lock_guard<std::mutex> g(sv->mu);
            sv->busy_s += dtb;
            sv->batch_steps += q;
            sv->atom_steps += natoms * q;
            for (Job* j : sv->active) j->steps_done += q;
        }

        // ---- retire finished and cancelled jobs ----
        std::vector<Job*> keep;
        for (Job* j : sv->active) {
            bool cancel;
            {
                std::lock_guard<std::mutex> g(sv->mu);
                cancel = j->cancel;
            }
            if (j->steps_done >= j->steps) {
                const int rs = retire_system(sv, j, true);
                finish(sv, j, rs == SOIL_OK ? SOIL_JOB_DONE : SOIL_JOB_FAILED,
                       rs == SOIL_OK ? std::string() : last_error(sv->ctx));
            } else if (cancel) {
                retire_system(sv, j, false);
                finish(sv, j, SOIL_JOB_CANCELLED, "cancelled");
            } else {
                keep.push_back(j);
            }
        }
        sv->active.swap(keep);
    }
    // shutdown: drop every resident system
    for (Job* j : sv->active) {
        retire_system(sv, j, false);
        finish(sv, j, SOIL_JOB_CANCELLED, "server stopped");
    }
    sv->active.clear();
}

Job* find(soil_server* sv, uint64_t id) {
    auto it = sv->jobs.find(id);
    return it == sv->jobs.end() ? nullptr : it->second.get();
}

void fill_info(const soil_server* sv, const Job* j, soil_job_info* out) {
    (void)sv;
    out->state = j->state;
    out->natoms = j->natoms;
    out->steps = j->steps;
    out->steps_done = j->steps_done;
    out->t_submit = j->t_submit;
    out->t_admit = j->t_admit;
    out->t_done = j->t_done;
}

bool terminal(int32_t st) {
    return st == SOIL_JOB_DONE || st == SOIL_JOB_FAILED || st == SOIL_JOB_CANCELLED;
}

}  // namespace

extern "C" {

int soil_server_create(soil_ctx* ctx, const soil_server_cfg* cfg, soil_server** out) {
    if (!ctx || !out) return SOIL_ERR_INVALID;
    *out = nullptr;
    soil_server* sv = new (std::nothrow) soil_server();
    if (!sv) return SOIL_ERR_OOM;
    sv->ctx = ctx;
    if (cfg) sv->cfg = *cfg;
    if (!sv->cfg.max_active) sv->cfg.max_active = 65536;
    if (!sv->cfg.quantum_steps) sv->cfg.quantum_steps = 50;
    if (!sv->cfg.bytes_per_atom) sv->cfg.bytes_per_atom = 1024;
    if (!sv->cfg.bytes_per_job) sv->cfg.bytes_per_job = 8u << 20;
    if (!sv->cfg.hbm_budget_bytes) sv->cfg.hbm_budget_bytes = ~0ull;
    const int st = soil_batch_create(ctx, &sv->batch);
    if (st != SOIL_OK) {
        delete sv;
        return st;
    }
    sv->t0 = Clock::now();
    sv->loop = std::thread(run_loop, sv);
    *out = sv;
    return SOIL_OK;
}

int soil_server_destroy(soil_server* sv) {
    if (!sv) return SOIL_OK;
    {
        std::lock_guard<std::mutex> g(sv->mu);
        sv->stop = true;
        for (uint64_t id : sv->queue) {
            Job* j = sv->jobs[id].get();
            j->state = SOIL_JOB_CANCELLED;
        }
        sv->queue.clear();
    }
    sv->cv_loop.notify_all();
    sv->loop.join();
    soil_batch_destroy(sv->batch);
    delete sv;
    return SOIL_OK;
}

int soil_server_submit(soil_server* sv, const soil_job_spec* js, uint64_t* id_out) {
    if (!sv || !js || !id_out) return SOIL_ERR_INVALID;
    const uint64_t n = js->natoms;
    if (!n || !js->tag || !js->pos3 || !js->vel3 || !js->mass || !js->cutoff_radius ||
        !js->radius || js->harmonic_k == 0.0)
        return SOIL_ERR_INVALID;
    std::unique_ptr<Job> j(new (std::nothrow) Job());
    if (!j) return SOIL_ERR_OOM;
    j->box = js->box;
    j->cfg = js->cfg;
    j->dt = js->dt;
    j->harmonic_k = js->harmonic_k;
    j->shear_rate = js->shear_rate;
    j->natoms = n;
    j->steps = js->steps;
    j->tag.assign(js->tag, js->tag + n);
    j->pos.assign(js->pos3, js->pos3 + 3 * n);
    j->vel.assign(js->vel3, js->vel3 + 3 * n);
    j->mass.assign(js->mass, js->mass + n);
    j->cutoff.assign(js->cutoff_radius, js->cutoff_radius + n);
    j->radius.assign(js->radius, js->radius + n);
    {
        std::lock_guard<std::mutex> g(sv->mu);
        if (sv->stop) return SOIL_ERR_STATE;
        j->id = sv->next_id++;
        j->t_submit = now_s(sv);
        *id_out = j->id;
        sv->queue.push_back(j->id);
        sv->jobs[j->id] = std::move(j);
    }
    sv->cv_loop.notify_all();
    return SOIL_OK;
}

int soil_server_poll(soil_server* sv, uint64_t id, soil_job_info* info) {
    if (!sv || !info) return SOIL_ERR_INVALID;
    std::lock_guard<std::mutex> g(sv->mu);
    Job* j = find(sv, id);
    if (!j) return SOIL_ERR_NOT_FOUND;
    fill_info(sv, j, info);
    return SOIL_OK;
}

int soil_server_wait(soil_server* sv, uint64_t id, double timeout_s, soil_job_info* info) {
    if (!sv) return SOIL_ERR_INVALID;
    std::unique_lock<std::mutex> lk(sv->mu);
    Job* j = find(sv, id);
    if (!j) return SOIL_ERR_NOT_FOUND;
    const auto pred = [&] { return terminal(j->state); };
    bool ok = true;
    if (timeout_s < 0) sv->cv_done.wait(lk, pred);
    else ok = sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred);
    if (info) fill_info(sv, j, info);
    return ok ? SOIL_OK : SOIL_ERR_TIMEOUT;
}

int soil_server_cancel(soil_server* sv, uint64_t id) {
    if (!sv) return SOIL_ERR_INVALID;
    {
        std::lock_guard<std::mutex> g(sv->mu);
        Job* j = find(sv, id);
        if (!j) return SOIL_ERR_INVALID;
        if (terminal(j->state)) return SOIL_OK;
        j->cancel = true;
    }
    sv->cv_loop.notify_all();
    return SOIL_OK;
}

int soil_server_result(soil_server* sv, uint64_t id, uint32_t* tag, double* pos3, double* vel3,
                       int32_t* image3) {
    if (!sv) return SOIL_ERR_INVALID;
    std::lock_guard<std::mutex> g(sv->mu);
    Job* j = find(sv, id);
    if (!j) return SOIL_ERR_NOT_FOUND;
    if (j->state != SOIL_JOB_DONE) return SOIL_ERR_STATE;
    const uint64_t n = j->out_tag.size();
    if (tag) std::memcpy(tag, j->out_tag.data(), n * 4);
    if (pos3) std::memcpy(pos3, j->out_pos.data(), n * 24);
    if (vel3) std::memcpy(vel3, j->out_vel.data(), n * 24);
    if (image3) std::memcpy(image3, j->out_img.data(), n * 12);
    return SOIL_OK;
}

int soil_server_release(soil_server* sv, uint64_t id) {
    if (!sv) return SOIL_ERR_INVALID;
    std::lock_guard<std::mutex> g(sv->mu);
    Job* j = find(sv, id);
    if (!j) return SOIL_ERR_NOT_FOUND;
    if (!terminal(j->state)) return SOIL_ERR_STATE;
    sv->jobs.erase(id);
    return SOIL_OK;
}

int soil_server_job_error(soil_server* sv, uint64_t id, char* buf, uint64_t len) {
    if (!sv || !buf || !len) return SOIL_ERR_INVALID;
    std::lock_guard<std::mutex> g(sv->mu);
    Job* j = find(sv, id);
    if (!j) return SOIL_ERR_NOT_FOUND;
    std::snprintf(buf, (size_t)len, "%s", j->error.c_str());
    return SOIL_OK;
}

int soil_server_get_stats(soil_server* sv, soil_server_stats* out) {
    if (!sv || !out) return SOIL_ERR_INVALID;
    std::lock_guard<std::mutex> g(sv->mu);
    out->queued = sv->queue.size();
    out->admitted = sv->admitted;
    out->completed = sv->completed;
    out->failed = sv->failed;
    out->atom_steps = sv->atom_steps;
    out->batch_steps = sv->batch_steps;
    out->busy_s = sv->busy_s;
    out->elapsed_s = now_s(sv);
    out->reserved_bytes = sv->reserved;
    out->max_active = sv->max_active_seen;
    return SOIL_OK;
}

}  // extern "C"
