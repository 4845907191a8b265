// Job server: simulation jobs admitted by HBM budget and advanced in batches by one worker thread.
//
// A client of the public C ABI only (img_create / img_set_state / img_batch_* / img_step /
// img_download_many / img_totals / img_progress).  img_batch_submit copies a job's settings and
// initial state and returns at once; the worker admits queued jobs in submission order while their
// device memory (img_bytes_required) fits the budget, creates each job's context and adds it to the
// running batch of its kind (precision, physics, time update mode, swept dimensions) -- a fresh member
// takes its first, edge-capturing iteration inside the batch -- and advances every batch one iteration
// per round.  Jobs whose settings cannot share batched launches (artificial viscosity, radiation, a
// treadmill) run as contexts of their own, stepped in the same rounds.  Every `check_every` rounds
// the finished members (TIMEMAX, ITERMAX or a device error) are retired: their result is copied to
// host memory, their context destroyed and their memory returned to the budget.  img_batch_poll and
// img_batch_cancel may be called from any thread at any time.
//
// No reference counterpart: the reference runs one simulation per MATLAB session.
#include <algorithm>
#include <chrono>
#include <atomic>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "imogen_b200.h"

namespace {

double mono_now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

constexpr int kResultVars = 11;   // IMG_VAR_MASS .. IMG_VAR_CMAGZ

struct Job {
    int id = 0;
    img_config cfg{};
    std::vector<double> mass, mom, ener, mag;   // initial state, released at admission
    size_t bytes = 0;
    int status = IMG_JOB_QUEUED;
    double submitted = 0, admitted = 0, completed = 0;
    double time = 0;
    int iterations = 0;
    int error_code = 0;
    std::string error;
    std::vector<double> result[kResultVars];
    double totals[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool cancel = false;
    // worker-side
    img_ctx* ctx = nullptr;
    img_batch* batch = nullptr;
    int steps = 0;   // iterations issued to a context of its own
};

using Kind = std::tuple<int, int, int, int, int, int, int>;

Kind kind_of(const img_config& c) {
    return Kind(c.precision, c.fluid_active, c.magnet_active, c.update_mode, c.grid[0] >= 3, c.grid[1] >= 3,
                c.grid[2] >= 3);
}

bool batchable(const img_config& c) {
    return c.viscosity_type == IMG_VISC_NONE && c.radiation_type == IMG_RAD_NONE && c.treadmill <= 0 &&
           !(c.fade_active & (IMG_FADE_MASS | IMG_FADE_MOM | IMG_FADE_ENER));
}

}  // namespace

struct img_server {
    size_t budget = 0, used = 0, peak = 0;
    int check_every = 4;
    int keep = IMG_KEEP_STATE;
    std::mutex mu;
    std::condition_variable cv;
    bool stop = false;
    std::deque<int> queue;
    std::map<int, Job> jobs;
    int next_id = 0;
    std::atomic<long long> rounds{0};
    // worker-side
    std::map<Kind, img_batch*> batches;
    std::vector<int> running;   // job ids on the device
    std::thread worker;
    std::string err;

    void run();
    void admit();
    void cancel_running();
    void step_all();
    void retire(bool all);
    void finish(Job& j, int status);
};

void img_server::finish(Job& j, int status) {
    // called by the worker without the lock: results first, then the record under the lock
    double t = 0;
    int it = 0, stopped = 0;
    if (status == IMG_JOB_DONE) {
        int rc = img_progress(j.ctx, &t, &it, &stopped);
        if (rc != IMG_OK) {
            status = IMG_JOB_FAILED;
            j.error_code = rc;
            j.error = img_last_error(j.ctx);
        } else if (keep == IMG_KEEP_TOTALS) {
            img_totals(j.ctx, j.totals);
        } else {
            const size_t n = (size_t)j.cfg.grid[0] * j.cfg.grid[1] * j.cfg.grid[2];
            int ids[kResultVars];
            double* hosts[kResultVars];
            for (int v = 0; v < kResultVars; ++v) {
                j.result[v].assign(n, 0.0);
                ids[v] = v;
                hosts[v] = j.result[v].data();
            }
            img_download_many(j.ctx, kResultVars, ids, hosts, n);
        }
    } else if (status == IMG_JOB_FAILED) {
        const int rc = img_progress(j.ctx, &t, &it, &stopped);   // the device error as a status and message
        j.error_code = rc != IMG_OK ? rc : IMG_ERR_CUDA;
        j.error = img_last_error(j.ctx);
    }
    if (j.batch) img_batch_remove(j.batch, j.ctx);
    img_destroy(j.ctx);
    j.ctx = nullptr;
    j.batch = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    j.time = t;
    j.iterations = it;
    j.status = status;
    j.completed = mono_now();
    used -= j.bytes;
    running.erase(std::find(running.begin(), running.end(), j.id));
}

void img_server::admit() {
    std::vector<int> take;
    {
        std::lock_guard<std::mutex> lock(mu);
        while (!queue.empty()) {
            Job& j = jobs[queue.front()];
            if (used + j.bytes > budget) break;   // first come, first served: wait for memory
            queue.pop_front();
            used += j.bytes;
            peak = std::max(peak, used);
            j.status = IMG_JOB_RUNNING;
            j.admitted = mono_now();
            take.push_back(j.id);
        }
    }
    for (int id : take) {
        Job* j;
        {
            std::lock_guard<std::mutex> lock(mu);
            j = &jobs[id];   // std::map nodes stay put
        }
        int rc = img_create(&j->ctx, &j->cfg);
        if (rc == IMG_OK) rc = img_set_state(j->ctx, j->mass.data(), j->mom.data(), j->ener.data(), j->mag.data());
        if (rc == IMG_OK && batchable(j->cfg)) {
            img_batch*& b = batches[kind_of(j->cfg)];
            if (!b) rc = img_batch_create(&b);
            if (rc == IMG_OK) rc = img_batch_add(b, j->ctx);
            if (rc == IMG_OK) j->batch = b;
        }
        std::lock_guard<std::mutex> lock(mu);
        j->mass.clear(); j->mass.shrink_to_fit();
        j->mom.clear(); j->mom.shrink_to_fit();
        j->ener.clear(); j->ener.shrink_to_fit();
        j->mag.clear(); j->mag.shrink_to_fit();
        if (rc != IMG_OK) {
            j->error_code = rc;
            j->error = img_last_error(j->ctx);
            if (j->ctx) img_destroy(j->ctx);
            j->ctx = nullptr;
            j->status = IMG_JOB_FAILED;
            j->completed = mono_now();
            used -= j->bytes;
            continue;
        }
        running.push_back(id);
    }
}

void img_server::cancel_running() {
    std::vector<int> victims;
    {
        std::lock_guard<std::mutex> lock(mu);
        for (int id : running)
            if (jobs[id].cancel) victims.push_back(id);
    }
    for (int id : victims) {
        Job* j;
        {
            std::lock_guard<std::mutex> lock(mu);
            j = &jobs[id];
        }
        if (j->batch) img_batch_remove(j->batch, j->ctx);
        img_destroy(j->ctx);
        j->ctx = nullptr;
        j->batch = nullptr;
        std::lock_guard<std::mutex> lock(mu);
        j->status = IMG_JOB_CANCELLED;
        j->completed = mono_now();
        used -= j->bytes;
        running.erase(std::find(running.begin(), running.end(), id));
    }
}

void img_server::step_all() {
    for (auto& kv : batches) {
        int n = 0;
        img_batch_size(kv.second, &n);
        if (n == 0 || img_batch_step(kv.second) == IMG_OK) continue;
        // a failed batch step (a CUDA error): its members fail with the batch's message
        const std::string why = img_batch_last_error(kv.second);
        std::vector<int> ids;
        {
            std::lock_guard<std::mutex> lock(mu);
            for (int id : running)
                if (jobs[id].batch == kv.second) ids.push_back(id);
        }
        for (int id : ids) {
            Job* j;
            {
                std::lock_guard<std::mutex> lock(mu);
                j = &jobs[id];
            }
            finish(*j, IMG_JOB_FAILED);
            std::lock_guard<std::mutex> lock(mu);
            if (j->error.empty()) j->error = why;
        }
    }
    std::vector<int> ids;
    {
        std::lock_guard<std::mutex> lock(mu);
        ids = running;
    }
    for (int id : ids) {
        Job* j;
        {
            std::lock_guard<std::mutex> lock(mu);
            j = &jobs[id];
        }
        if (j->batch || j->steps >= j->cfg.iter_max) continue;
        img_step(j->ctx);   // a context of its own: one iteration per round, ITERMAX counted here
        j->steps += 1;
    }
}

void img_server::retire(bool all) {
    std::vector<int> ids;
    {
        std::lock_guard<std::mutex> lock(mu);
        ids = running;
    }
    for (auto& kv : batches) {
        int n = 0;
        img_batch_size(kv.second, &n);
        if (n == 0) continue;
        std::vector<int> flags(n);
        img_batch_status(kv.second, flags.data(), n);   // synchronises the batch's stream
    }
    for (int id : ids) {
        Job* j;
        {
            std::lock_guard<std::mutex> lock(mu);
            j = &jobs[id];
            if (j->cancel) continue;   // a requested cancellation wins over a completion in the same round
        }
        double t;
        int it, stopped = 0;
        const int rc = img_progress(j->ctx, &t, &it, &stopped);
        const bool capped = !j->batch && j->steps >= j->cfg.iter_max;
        if (rc != IMG_OK) finish(*j, IMG_JOB_FAILED);
        else if (stopped || capped || all) finish(*j, IMG_JOB_DONE);
    }
}

void img_server::run() {
    for (;;) {
        {
            std::unique_lock<std::mutex> lock(mu);
            if (stop) break;
            if (queue.empty() && running.empty()) {
                cv.wait_for(lock, std::chrono::milliseconds(20));
                continue;
            }
        }
        admit();
        cancel_running();
        bool any;
        {
            std::lock_guard<std::mutex> lock(mu);
            any = !running.empty();
        }
        if (!any) {
            std::unique_lock<std::mutex> lock(mu);
            cv.wait_for(lock, std::chrono::milliseconds(1));   // waiting for memory or for submissions
            continue;
        }
        step_all();
        const long long r = ++rounds;
        if (r % check_every == 0) retire(false);
    }
}

extern "C" {

int img_server_create(img_server** out, size_t hbm_budget, int check_every, int keep) {
    if (!out || hbm_budget == 0 || (keep != IMG_KEEP_STATE && keep != IMG_KEEP_TOTALS)) return IMG_ERR_ARG;
    auto* s = new img_server();
    s->budget = hbm_budget;
    s->check_every = std::max(1, check_every);
    s->keep = keep;
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return IMG_OK;
}

int img_server_destroy(img_server* s) {
    if (!s) return IMG_ERR_ARG;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    s->worker.join();
    for (int id : s->running) {   // jobs still on the device are dropped
        Job& j = s->jobs[id];
        if (j.ctx) img_destroy(j.ctx);
    }
    for (auto& kv : s->batches) img_batch_destroy(kv.second);
    delete s;
    return IMG_OK;
}

int img_batch_submit(img_server* s, const img_config* cfg, const double* mass, const double* mom, const double* ener,
                     const double* mag, int* job_id) {
    if (!s || !cfg || !mass || !mom || !ener || !mag || !job_id) return IMG_ERR_ARG;
    const size_t n = (size_t)cfg->grid[0] * cfg->grid[1] * cfg->grid[2];
    const size_t bytes = img_bytes_required(cfg);
    if (n == 0 || bytes == 0) return IMG_ERR_ARG;
    if (bytes > s->budget) return IMG_ERR_NOMEM;   // could never be admitted
    Job j;
    j.cfg = *cfg;
    j.mass.assign(mass, mass + n);
    j.mom.assign(mom, mom + 3 * n);
    j.ener.assign(ener, ener + n);
    j.mag.assign(mag, mag + 3 * n);
    j.bytes = bytes;
    j.submitted = mono_now();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        j.id = s->next_id++;
        *job_id = j.id;
        s->queue.push_back(j.id);
        s->jobs.emplace(j.id, std::move(j));
    }
    s->cv.notify_all();
    return IMG_OK;
}

int img_batch_poll(img_server* s, int job_id, img_job_info* info) {
    if (!s || !info) return IMG_ERR_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return IMG_ERR_ARG;
    const Job& j = it->second;
    info->status = j.status;
    info->time = j.time;
    info->iterations = j.iterations;
    info->submitted = j.submitted;
    info->admitted = j.admitted;
    info->completed = j.completed;
    info->error_code = j.error_code;
    std::snprintf(info->error, sizeof info->error, "%s", j.error.c_str());
    return IMG_OK;
}

int img_batch_cancel(img_server* s, int job_id) {
    if (!s) return IMG_ERR_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return IMG_ERR_ARG;
    Job& j = it->second;
    if (j.status == IMG_JOB_QUEUED) {
        s->queue.erase(std::find(s->queue.begin(), s->queue.end(), job_id));
        j.status = IMG_JOB_CANCELLED;
        j.completed = mono_now();
        return IMG_OK;
    }
    if (j.status == IMG_JOB_RUNNING && !j.cancel) {
        j.cancel = true;   // the worker stops it before its next round
        return IMG_OK;
    }
    return IMG_ERR_STATE;   // already ended (or already being cancelled)
}

int img_batch_result(img_server* s, int job_id, int var_id, double* host, size_t n) {
    if (!s || !host) return IMG_ERR_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return IMG_ERR_ARG;
    const Job& j = it->second;
    if (j.status != IMG_JOB_DONE) return IMG_ERR_STATE;
    if (var_id == IMG_RESULT_TOTALS) {
        if (s->keep != IMG_KEEP_TOTALS || n < 8) return IMG_ERR_ARG;
        std::memcpy(host, j.totals, sizeof j.totals);
        return IMG_OK;
    }
    if (s->keep != IMG_KEEP_STATE || var_id < 0 || var_id >= kResultVars || n != j.result[var_id].size())
        return IMG_ERR_ARG;
    std::memcpy(host, j.result[var_id].data(), n * sizeof(double));
    return IMG_OK;
}

int img_server_stats(img_server* s, img_server_info* info) {
    if (!s || !info) return IMG_ERR_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    info->budget = s->budget;
    info->used = s->used;
    info->peak = s->peak;
    info->queued = (int)s->queue.size();
    info->running = (int)s->running.size();
    int done = 0;
    for (const auto& kv : s->jobs) done += kv.second.status >= IMG_JOB_DONE;
    info->finished = done;
    info->rounds = s->rounds.load();
    return IMG_OK;
}

double img_monotonic_seconds(void) { return mono_now(); }

}  // extern "C"
