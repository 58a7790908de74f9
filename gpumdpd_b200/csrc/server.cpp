// server.cpp -- continuous-batching job server over the packed engine.
//
// Jobs (a run.in text plus a system) are submitted at any time and queued.  At every
// scheduling point (dpd_server_step) the server
//   1. admits queued jobs, in submission order with backfilling, while the device
//      memory of the admitted set fits the budget; admitted jobs of similar length
//      (steps within a factor 2) become one cohort: one packed engine (one launch per
//      stage for all of them, the step captured in a CUDA graph) on its own CUDA stream;
//   2. keeps every cohort's stream fed with chunks of steps, two in flight: while one
//      runs, the next is queued behind it, and a completed chunk is checked from a copy
//      of the replicas' state words taken on the stream after it, so the stream never
//      waits for the host; the cohorts' kernels overlap on the device;
//   3. retires the jobs that reached their `run N`: their thermo rows, final state and
//      RDF are copied out, and a cohort's device memory returns to the budget when its
//      last job has finished.
// Each job keeps its own tags, seed, step counter and step limit inside its cohort, so
// its trajectory is the one it has alone, up to the FP32 summation order of forces.
// A job whose replica reports an error (its own status word) fails alone: the replica
// is frozen and its cohort mates run on.  Cancelling a job freezes it the same way.
// A server is used from one host thread at a time.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dpd_b200.h"
#include "engine.h"

namespace {

using Clock = std::chrono::steady_clock;

enum JobStatus { JOB_DONE = 0, JOB_QUEUED = 1, JOB_RUNNING = 2 };

struct Job {
    int64_t id = 0;
    dpd::Replica rep;  // parsed input; moved into the cohort's engine at admission
    int64_t n_atoms = 0;
    int64_t bytes = 0;  // device bytes of the job alone
    int64_t slots = 0;  // particle slots (warp-rounded)
    int nmax = 16, maxb = 0;
    uint32_t steps = 0;  // the run.in's `run N`
    int status = JOB_QUEUED;
    double submit_s = 0, start_s = -1, finish_s = -1;
    int rdf_nbins = 0;
    // results, kept after the cohort's engine is released
    std::vector<dpd_thermo> thermo;
    std::vector<double> x, v, rdf;
    int64_t rdf_samples = 0;
};

// A chunk of steps in flight: an event after it and the replicas' state words copied
// (pinned host memory) on the stream after it.
struct Chunk {
    cudaEvent_t ev = nullptr;
    RepState* rs = nullptr;
};

struct Cohort {
    std::unique_ptr<dpd::Engine> eng;
    std::vector<int64_t> jobs;  // job id of each replica
    std::vector<bool> finished;
    uint32_t max_steps = 0;     // longest job in the cohort
    uint32_t issued = 0;        // steps issued after the zero step
    bool started = false;
    Chunk slot[2];
    std::deque<int> pending;    // slots of the enqueued chunks not yet checked, oldest first
    int next_slot = 0;
    int64_t bytes = 0;
    ~Cohort()
    {
        if (eng) cudaStreamSynchronize(eng->stream());
        for (Chunk& k : slot) {
            if (k.ev) cudaEventDestroy(k.ev);
            if (k.rs) cudaFreeHost(k.rs);
        }
    }
};

// list capacity and bonds per atom of one job, as the engine's layout computes them
void job_shape(const dpd::Replica& R, int& nmax, int& maxb)
{
    const double cut = R.in.global_cut + R.in.skin;
    const double sphere = 4.0 / 3.0 * M_PI * std::pow(cut, 3.0);
    const int nm = (int)(R.in.max_rho * sphere) + 1;
    nmax = std::max(16, ((nm + 15) / 16) * 16);
    maxb = 0;
    if (R.sys.n_bonds > 0) {
        std::vector<int> deg(R.sys.n_atoms, 0);
        for (int b = 0; b < R.sys.n_bonds; b++) {
            deg[R.sys.bonds[3 * b + 1] - 1]++;
            deg[R.sys.bonds[3 * b + 2] - 1]++;
        }
        for (int d : deg) maxb = std::max(maxb, d);
    }
}

}  // namespace

struct dpd_server {
    double budget = 0;
    int chunk = 100;
    dpd_tuning tune{};
    std::map<int64_t, Job> jobs;
    std::deque<int64_t> queue;
    std::vector<std::unique_ptr<Cohort>> cohorts;
    int64_t next_id = 1;
    int64_t used_bytes = 0;
    double max_wait_s = 0.0;  // admission window (see dpd_server_set_policy)
    int min_jobs = 1;

    int64_t particle_steps = 0;
    double busy_s = 0;
    Clock::time_point t0 = Clock::now();
    std::string err;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
    int fail(int code, const std::string& msg)
    {
        err = msg;
        return code;
    }
    int admit();
    int make_cohort(const std::vector<int64_t>& ids);
    int advance();
    void retire_job(Cohort& c, int r, int64_t id);
    // end a running job of cohort c (replica r) with an error status; its cohort mates
    // run on
    void fail_job(Cohort& c, int r, int code, const std::string& msg);
};

void dpd_server::fail_job(Cohort& c, int r, int code, const std::string& msg)
{
    Job& j = jobs[c.jobs[r]];
    j.status = code;
    j.finish_s = now();
    c.finished[r] = true;
    err = "job " + std::to_string(j.id) + ": " + msg;
    if (c.eng->freeze_async(r) != DPD_OK) err += " (and its replica could not be frozen)";
}

// Admission: one new cohort from the queued jobs that fit the budget together.  The
// estimate of a set is the sum of the jobs' own estimates, corrected for the set's
// common list capacity and bonds per slot (the packed engine uses the maxima).
int dpd_server::admit()
{
    if (queue.empty()) return DPD_OK;
    // admission window: while cohorts are running, queued jobs are gathered until there
    // are min_jobs of them or the oldest has waited max_wait_s, so that jobs arriving
    // close together share one packed engine
    if (!cohorts.empty() && (int)queue.size() < min_jobs &&
        now() - jobs[queue.front()].submit_s < max_wait_s)
        return DPD_OK;
    std::vector<int64_t> pick;
    int64_t sum = 0, slots = 0, sum_list = 0, sum_bond = 0;
    int nmax_c = 16, maxb_c = 0;
    const int64_t room = (int64_t)budget - used_bytes;
    for (int64_t id : queue) {
        const Job& j = jobs[id];
        const int nm = std::max(nmax_c, j.nmax), mb = std::max(maxb_c, j.maxb);
        const int64_t s2 = slots + j.slots;
        const int64_t list2 = sum_list + j.slots * 4 * (int64_t)j.nmax;
        const int64_t bond2 = sum_bond + j.slots * 24 * (int64_t)std::max(j.maxb, 1);
        const int64_t est = sum + j.bytes + (s2 * 4 * (int64_t)nm - list2) +
                            (s2 * 24 * (int64_t)std::max(mb, 1) - bond2);
        if (est > room) continue;  // backfill: a later, smaller job may still fit
        if (s2 > (int64_t)((1 << 27) - 1) / 2) break;  // list entries hold 27 bits of slot index
        pick.push_back(id);
        sum += j.bytes;
        slots = s2;
        sum_list = list2;
        sum_bond = bond2;
        nmax_c = nm;
        maxb_c = mb;
    }
    if (pick.empty()) return DPD_OK;
    for (int64_t id : pick) queue.erase(std::find(queue.begin(), queue.end(), id));
    // Jobs of similar length share a cohort (steps in [2^k, 2^(k+1))): a cohort's step
    // costs as much as all its particles, finished jobs included, so a long job packed
    // with many short ones would crawl after they finish.
    std::map<int, std::vector<int64_t>> groups;
    for (int64_t id : pick) {
        int k = 0;
        while ((jobs[id].steps >> (k + 1)) != 0u) k++;
        groups[k].push_back(id);
    }
    int first_err = DPD_OK;
    for (auto& g : groups) {
        const int e = make_cohort(g.second);
        if (e && !first_err) first_err = e;
    }
    return first_err;
}

int dpd_server::make_cohort(const std::vector<int64_t>& ids)
{
    auto c = std::make_unique<Cohort>();
    std::vector<dpd::Replica> reps;
    std::vector<uint32_t> limits;
    for (int64_t id : ids) {
        Job& j = jobs[id];
        reps.push_back(std::move(j.rep));
        limits.push_back(j.steps);
        c->jobs.push_back(id);
        c->max_steps = std::max(c->max_steps, j.steps);
    }
    c->finished.assign(ids.size(), false);
    c->eng = std::make_unique<dpd::Engine>();
    // the longest jobs bound the makespan: their cohorts' streams get the highest
    // priority (one level per doubling of the step count), so their steps run at
    // nearly their alone speed while shorter cohorts fill the rest of the GPU
    {
        int least = 0, greatest = 0;
        if (cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess) {
            int k = 0;
            while ((c->max_steps >> (k + 1)) != 0u) k++;
            c->eng->set_stream_priority(std::max(greatest, least - std::max(0, k - 9)));
        }
    }
    int e = c->eng->init(std::move(reps), &tune);
    if (!e) e = c->eng->set_limits(limits);
    const double t = now();
    if (e) {
        // the jobs of a cohort that cannot be created fail with the engine's message
        const std::string msg = c->eng->err;
        for (int64_t id : ids) {
            jobs[id].status = e;
            jobs[id].finish_s = t;
        }
        return fail(e, "admitting " + std::to_string(ids.size()) + " job(s): " + msg);
    }
    for (Chunk& k : c->slot) {
        if (cudaEventCreateWithFlags(&k.ev, cudaEventDisableTiming) != cudaSuccess ||
            cudaMallocHost((void**)&k.rs, sizeof(RepState) * ids.size()) != cudaSuccess)
            return fail(DPD_E_CUDA, "cannot create a cohort's chunk events");
    }
    c->bytes = c->eng->device_bytes();
    used_bytes += c->bytes;
    for (int64_t id : ids) {
        jobs[id].status = JOB_RUNNING;
        jobs[id].start_s = t;
    }
    cohorts.push_back(std::move(c));
    return DPD_OK;
}

void dpd_server::retire_job(Cohort& c, int r, int64_t id)
{
    Job& j = jobs[id];
    dpd::Engine& eng = *c.eng;
    const int n = eng.rep(r).sys.n_atoms;
    j.x.resize(3 * (size_t)n);
    j.v.resize(3 * (size_t)n);
    int e = eng.get_state(r, j.x.data(), j.v.data(), nullptr, nullptr);
    if (!e) {
        j.thermo.resize(DPD_RING_ROWS);
        int nr = 0;
        e = eng.get_thermo(r, j.thermo.data(), DPD_RING_ROWS, &nr);
        j.thermo.resize(e ? 0 : nr);
    }
    if (!e && j.rdf_nbins > 0) {
        j.rdf.resize(j.rdf_nbins);
        e = eng.rdf_result(r, j.rdf.data(), &j.rdf_samples);
    }
    j.status = e ? e : JOB_DONE;
    j.finish_s = now();
    if (e) err = "job " + std::to_string(id) + ": " + eng.err;
    particle_steps += (int64_t)n * j.steps;
}

// One scheduling pass over the cohorts, without waiting for any of them: a cohort whose
// chunk has completed is checked, its finished jobs are retired and its next chunk is
// enqueued at once, so every cohort's stream stays fed while the others run and the
// cohorts' kernels overlap on the device.  When no cohort has completed a chunk the pass
// sleeps briefly instead of spinning.
int dpd_server::advance()
{
    if (cohorts.empty()) return DPD_OK;
    const double t_begin = now();
    int first_err = DPD_OK;
    bool progressed = false;
    auto fail_cohort = [&](Cohort& c, int rc) {
        const double t = now();
        for (size_t r = 0; r < c.jobs.size(); r++)
            if (!c.finished[r]) {
                jobs[c.jobs[r]].status = rc;
                jobs[c.jobs[r]].finish_s = t;
                c.finished[r] = true;
            }
        err = "cohort failed: " + c.eng->err;
        if (!first_err) first_err = rc;
    };
    auto all_done = [](const Cohort& c) {
        return std::all_of(c.finished.begin(), c.finished.end(), [](bool b) { return b; });
    };
    for (auto& cp : cohorts) {
        Cohort& c = *cp;
        // completed chunks, oldest first: errors from their status words, finished jobs
        bool failed = false;
        while (!c.pending.empty()) {
            const Chunk& k = c.slot[c.pending.front()];
            const cudaError_t q = cudaEventQuery(k.ev);
            if (q == cudaErrorNotReady) break;
            c.pending.pop_front();
            progressed = true;
            if (q != cudaSuccess) {
                // a CUDA error ends the whole cohort (it is sticky for the context)
                c.eng->err = std::string("CUDA error in a chunk: ") + cudaGetErrorString(q);
                fail_cohort(c, DPD_E_CUDA);
                cudaStreamSynchronize(c.eng->stream());
                c.pending.clear();
                failed = true;
                break;
            }
            // a replica's own status word fails its job alone
            for (size_t r = 0; r < c.jobs.size(); r++) {
                if (c.finished[r]) continue;
                const int rc = c.eng->status_error(k.rs[r].status, (int)r);
                if (rc) {
                    fail_job(c, (int)r, rc, c.eng->err);
                    if (!first_err) first_err = rc;
                }
            }
            for (size_t r = 0; r < c.jobs.size(); r++) {
                if (c.finished[r]) continue;
                if (k.rs[r].step > jobs[c.jobs[r]].steps) {
                    retire_job(c, (int)r, c.jobs[r]);
                    c.finished[r] = true;
                }
            }
        }
        if (failed) continue;
        // keep two chunks in flight until the longest job's steps are issued
        while (c.pending.size() < 2 && !all_done(c) && (!c.started || c.issued < c.max_steps)) {
            const uint32_t n = std::min<uint32_t>((uint32_t)chunk, c.max_steps - c.issued);
            Chunk& k = c.slot[c.next_slot];
            int rc = c.eng->run_async(n);  // the first call also runs the zero step
            if (!rc) rc = c.eng->rstate_async(k.rs);
            if (!rc && cudaEventRecord(k.ev, c.eng->stream()) != cudaSuccess) rc = DPD_E_CUDA;
            if (rc) {
                fail_cohort(c, rc);
                break;
            }
            c.pending.push_back(c.next_slot);
            c.next_slot ^= 1;
            c.started = true;
            c.issued += n;
            progressed = true;
        }
    }
    // release cohorts whose jobs have all finished
    for (size_t k = 0; k < cohorts.size();) {
        Cohort& c = *cohorts[k];
        if (c.pending.empty() && all_done(c)) {
            used_bytes -= c.bytes;
            cohorts.erase(cohorts.begin() + k);
        } else {
            k++;
        }
    }
    if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(100));
    busy_s += now() - t_begin;
    return first_err;
}

extern "C" {

int dpd_server_create(double hbm_budget_bytes, int chunk_steps, const dpd_tuning* tune, dpd_server** out)
{
    if (!out) return DPD_E_ARG;
    *out = nullptr;
    if (!(hbm_budget_bytes > 0) || chunk_steps < 1) return DPD_E_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return DPD_E_NODEV;
    auto* s = new (std::nothrow) dpd_server;
    if (!s) return DPD_E_NOMEM;
    s->budget = hbm_budget_bytes;
    s->chunk = chunk_steps;
    if (tune) {
        s->tune = *tune;
    } else {
        s->tune = dpd::engine_default_tuning();
    }
    // cohorts run side by side: no tiny-grid kernels (launch_mode 3 for 0)
    if (s->tune.launch_mode == 0) s->tune.launch_mode = 3;
    *out = s;
    return DPD_OK;
}

int dpd_server_submit(dpd_server* srv, const char* run_in_text, const dpd_system* sys, int64_t* job_id)
{
    if (!srv || !run_in_text || !sys) return DPD_E_ARG;
    Job j;
    std::string err;
    int e = dpd::make_replica_from_system(run_in_text, sys, j.rep, err);
    if (e) return srv->fail(e, err);
    if (j.rep.in.nsteps == 0) return srv->fail(DPD_E_ARG, "a job needs `run N` with N > 0");
    j.id = srv->next_id++;
    j.n_atoms = j.rep.sys.n_atoms;
    j.steps = j.rep.in.nsteps;
    j.slots = ((j.n_atoms + 31) / 32) * 32;
    job_shape(j.rep, j.nmax, j.maxb);
    j.bytes = dpd::Engine::estimate_bytes({&j.rep});
    j.rdf_nbins = j.rep.ff.rdfs.empty() ? 0 : j.rep.ff.rdfs[0].nbins;
    if (j.bytes > (int64_t)srv->budget)
        return srv->fail(DPD_E_NOMEM, "job needs " + std::to_string(j.bytes) + " device bytes, more than the budget");
    j.submit_s = srv->now();
    const int64_t id = j.id;
    srv->jobs.emplace(id, std::move(j));
    srv->queue.push_back(id);
    if (job_id) *job_id = id;
    return DPD_OK;
}

int dpd_server_set_policy(dpd_server* srv, double max_wait_s, int min_jobs)
{
    if (!srv || !(max_wait_s >= 0) || min_jobs < 1) return DPD_E_ARG;
    srv->max_wait_s = max_wait_s;
    srv->min_jobs = min_jobs;
    return DPD_OK;
}

int dpd_server_step(dpd_server* srv, int* n_active, int* n_queued)
{
    if (!srv) return DPD_E_ARG;
    int e = srv->admit();
    int e2 = srv->advance();
    int active = 0;
    for (auto& c : srv->cohorts)
        for (bool f : c->finished) active += f ? 0 : 1;
    if (n_active) *n_active = active;
    if (n_queued) *n_queued = (int)srv->queue.size();
    return e ? e : e2;
}

int dpd_server_result(dpd_server* srv, int64_t job_id, dpd_job_result* res)
{
    if (!srv || !res) return DPD_E_ARG;
    auto it = srv->jobs.find(job_id);
    if (it == srv->jobs.end()) return srv->fail(DPD_E_ARG, "unknown job id");
    const Job& j = it->second;
    std::memset(res, 0, sizeof(*res));
    res->job_id = j.id;
    res->status = j.status;
    res->steps = j.status == JOB_DONE ? j.steps : 0;
    res->submit_s = j.submit_s;
    res->start_s = j.start_s;
    res->finish_s = j.finish_s;
    double st = 0, sp = 0;
    int n = 0;
    for (size_t k = 1; k < j.thermo.size(); k++) {
        st += j.thermo[k].temp;
        sp += j.thermo[k].pressure;
        n++;
    }
    res->mean_temp = n ? st / n : (j.thermo.empty() ? 0.0 : j.thermo[0].temp);
    res->mean_pressure = n ? sp / n : (j.thermo.empty() ? 0.0 : j.thermo[0].pressure);
    // standard errors of the means from block averages (rows after the first, in up to
    // 10 consecutive blocks of equal length; the last rows that do not fill a block
    // are left out of this estimate)
    res->stderr_temp = res->stderr_pressure = NAN;
    if (n >= 4) {
        const int nb = std::min(10, n / 2), len = n / nb;
        double mt = 0, mp = 0, vt = 0, vp = 0;
        std::vector<double> bt(nb), bp(nb);
        for (int b = 0; b < nb; b++) {
            double a = 0, c = 0;
            for (int k = 0; k < len; k++) {
                a += j.thermo[1 + b * len + k].temp;
                c += j.thermo[1 + b * len + k].pressure;
            }
            bt[b] = a / len;
            bp[b] = c / len;
            mt += bt[b] / nb;
            mp += bp[b] / nb;
        }
        for (int b = 0; b < nb; b++) {
            vt += (bt[b] - mt) * (bt[b] - mt);
            vp += (bp[b] - mp) * (bp[b] - mp);
        }
        res->stderr_temp = std::sqrt(vt / (nb - 1) / nb);
        res->stderr_pressure = std::sqrt(vp / (nb - 1) / nb);
    }
    if (!j.thermo.empty()) res->last = j.thermo.back();
    return DPD_OK;
}

int dpd_server_cancel(dpd_server* srv, int64_t job_id)
{
    if (!srv) return DPD_E_ARG;
    auto it = srv->jobs.find(job_id);
    if (it == srv->jobs.end()) return srv->fail(DPD_E_ARG, "unknown job id");
    Job& j = it->second;
    if (j.status == JOB_QUEUED) {
        srv->queue.erase(std::find(srv->queue.begin(), srv->queue.end(), job_id));
        j.status = DPD_E_CANCELLED;
        j.finish_s = srv->now();
        return DPD_OK;
    }
    if (j.status != JOB_RUNNING) return srv->fail(DPD_E_STATE, "job " + std::to_string(job_id) + " has already ended");
    for (auto& c : srv->cohorts)
        for (size_t r = 0; r < c->jobs.size(); r++)
            if (c->jobs[r] == job_id && !c->finished[r]) {
                srv->fail_job(*c, (int)r, DPD_E_CANCELLED, "cancelled");
                return DPD_OK;
            }
    return srv->fail(DPD_E_STATE, "job " + std::to_string(job_id) + " is not in a running batch");
}

int dpd_server_job_state(dpd_server* srv, int64_t job_id, double* x, double* v)
{
    if (!srv) return DPD_E_ARG;
    auto it = srv->jobs.find(job_id);
    if (it == srv->jobs.end()) return srv->fail(DPD_E_ARG, "unknown job id");
    const Job& j = it->second;
    if (j.status != JOB_DONE) return srv->fail(DPD_E_STATE, "job has not finished");
    if (x) std::copy(j.x.begin(), j.x.end(), x);
    if (v) std::copy(j.v.begin(), j.v.end(), v);
    return DPD_OK;
}

int dpd_server_job_rdf(dpd_server* srv, int64_t job_id, double* g, int64_t* nsamples)
{
    if (!srv) return DPD_E_ARG;
    auto it = srv->jobs.find(job_id);
    if (it == srv->jobs.end()) return srv->fail(DPD_E_ARG, "unknown job id");
    const Job& j = it->second;
    if (j.status != JOB_DONE) return srv->fail(DPD_E_STATE, "job has not finished");
    if (j.rdf_nbins == 0) return srv->fail(DPD_E_STATE, "job has no rdf compute");
    if (g) std::copy(j.rdf.begin(), j.rdf.end(), g);
    if (nsamples) *nsamples = j.rdf_samples;
    return DPD_OK;
}

int dpd_server_stats(dpd_server* srv, int64_t* particle_steps, double* busy_s, int64_t* device_bytes)
{
    if (!srv) return DPD_E_ARG;
    if (particle_steps) *particle_steps = srv->particle_steps;
    if (busy_s) *busy_s = srv->busy_s;
    if (device_bytes) *device_bytes = srv->used_bytes;
    return DPD_OK;
}

const char* dpd_server_last_error(dpd_server* srv)
{
    return srv ? srv->err.c_str() : "null server";
}

int dpd_server_destroy(dpd_server* srv)
{
    delete srv;
    return DPD_OK;
}

}  // extern "C"
