// capi.cpp -- the extern "C" boundary of libdpd_b200.so (include/dpd_b200.h).
#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "../../include/dpd_b200.h"
#include "engine.h"
#include "fp64.h"

// One handle type for both engines: `f64` is set for the FP64 parity mode, which answers
// run, sync, thermo, state and info; every other call refuses it.
struct dpd_engine {
    dpd::Engine eng;
    std::unique_ptr<dpd::EngineF64> f64;
};

static thread_local std::string g_create_err;

static int set_create_err(const std::string& e, int code)
{
    g_create_err = e;
    return code;
}

extern "C" {

const char* dpd_version(void) { return "dpd_b200 1.0 (sm_100a)"; }

int dpd_create(const char* run_in_text, const char* data_path, const char* base_dir, dpd_engine** out)
{
    if (!run_in_text || !out) return set_create_err("null argument", DPD_E_ARG);
    *out = nullptr;
    std::vector<dpd::Replica> reps(1);
    std::string err;
    int e = dpd::make_replica(run_in_text, data_path ? data_path : "", base_dir ? base_dir : "", reps[0], err);
    if (e) return set_create_err(err, e);
    auto* h = new (std::nothrow) dpd_engine;
    if (!h) return set_create_err("out of host memory", DPD_E_NOMEM);
    e = h->eng.init(std::move(reps), nullptr);
    if (e) {
        g_create_err = h->eng.err;
        delete h;
        return e;
    }
    *out = h;
    return DPD_OK;
}

int dpd_create_from_system(const char* run_in_text, const dpd_system* sys, dpd_engine** out)
{
    if (!run_in_text || !sys || !out) return set_create_err("null argument", DPD_E_ARG);
    *out = nullptr;
    std::vector<dpd::Replica> reps(1);
    std::string err;
    int e = dpd::make_replica_from_system(run_in_text, sys, reps[0], err);
    if (e) return set_create_err(err, e);
    auto* h = new (std::nothrow) dpd_engine;
    if (!h) return set_create_err("out of host memory", DPD_E_NOMEM);
    e = h->eng.init(std::move(reps), nullptr);
    if (e) {
        g_create_err = h->eng.err;
        delete h;
        return e;
    }
    *out = h;
    return DPD_OK;
}

int dpd_batch_create(int n_rep, const char* const* run_in_texts, const dpd_system* systems,
                     const dpd_tuning* tune, dpd_engine** out)
{
    if (n_rep <= 0 || !run_in_texts || !systems || !out) return set_create_err("invalid argument", DPD_E_ARG);
    *out = nullptr;
    std::vector<dpd::Replica> reps(n_rep);
    for (int r = 0; r < n_rep; r++) {
        std::string err;
        int e = dpd::make_replica_from_system(run_in_texts[r] ? run_in_texts[r] : "", &systems[r], reps[r], err);
        if (e) return set_create_err("replica " + std::to_string(r) + ": " + err, e);
    }
    auto* h = new (std::nothrow) dpd_engine;
    if (!h) return set_create_err("out of host memory", DPD_E_NOMEM);
    int e = h->eng.init(std::move(reps), tune);
    if (e) {
        g_create_err = h->eng.err;
        delete h;
        return e;
    }
    *out = h;
    return DPD_OK;
}

#define ENG_CHECK_ANY(h)              \
    if (!(h)) {                       \
        g_create_err = "null engine"; \
        return DPD_E_ARG;             \
    }
#define ENG_CHECK(h)                                                    \
    ENG_CHECK_ANY(h)                                                    \
    if ((h)->f64) {                                                     \
        (h)->f64->err = "not available in the FP64 parity mode";        \
        return DPD_E_ARG;                                               \
    }

int dpd_create_fp64(const char* run_in_text, const char* data_path, const char* base_dir,
                    const dpd_system* sys, dpd_engine** out)
{
    if (!run_in_text || !out) return set_create_err("null argument", DPD_E_ARG);
    *out = nullptr;
    dpd::Replica rep;
    std::string err;
    int e = sys ? dpd::make_replica_from_system(run_in_text, sys, rep, err)
                : dpd::make_replica(run_in_text, data_path ? data_path : "", base_dir ? base_dir : "", rep, err);
    if (e) return set_create_err(err, e);
    // the engine first: a refused input makes no CUDA call
    std::unique_ptr<dpd::EngineF64> f(new (std::nothrow) dpd::EngineF64);
    if (!f) return set_create_err("out of host memory", DPD_E_NOMEM);
    e = f->init(std::move(rep));
    if (e) return set_create_err(f->err, e);
    auto* h = new (std::nothrow) dpd_engine;
    if (!h) return set_create_err("out of host memory", DPD_E_NOMEM);
    h->f64 = std::move(f);
    *out = h;
    return DPD_OK;
}

int dpd_run(dpd_engine* h, uint32_t nsteps)
{
    ENG_CHECK_ANY(h);
    if (h->f64) return h->f64->run(nsteps);
    return h->eng.run(nsteps);
}

int dpd_sync(dpd_engine* h)
{
    ENG_CHECK_ANY(h);
    if (h->f64) return DPD_OK;  // its runs are synchronous
    return h->eng.sync_and_check();
}

int dpd_get_thermo(dpd_engine* h, dpd_thermo* rows, int max_rows, int* n_rows)
{
    ENG_CHECK_ANY(h);
    if (!rows || max_rows < 0) return DPD_E_ARG;
    if (h->f64) return h->f64->get_thermo(rows, max_rows, n_rows);
    return h->eng.get_thermo(0, rows, max_rows, n_rows);
}

int dpd_dump_open(dpd_engine* h, const char* path, int64_t start, int64_t every, int flags)
{
    ENG_CHECK(h);
    if (!path) return DPD_E_ARG;
    const dpd::RunInput& in = h->eng.rep(0).in;
    if (every <= 0) {
        if (!in.dump) {
            h->eng.err = "no dump command in the run.in";
            return DPD_E_ARG;
        }
        return h->eng.dump_open(path, in.dump_start, in.dump_f, !in.dump_wrapped, in.dump_force, in.dump_vel);
    }
    if (start < 0 || start > 0xFFFFFFFFll || every > 0xFFFFFFFFll) return DPD_E_ARG;
    return h->eng.dump_open(path, (uint32_t)start, (uint32_t)every, (flags & DPD_DUMP_UNWRAPPED) != 0,
                            (flags & DPD_DUMP_FORCE) != 0, (flags & DPD_DUMP_VEL) != 0);
}

int dpd_get_compute(dpd_engine* h, const char* id, double* rows, int max_rows, int* n_cols, int* n_rows)
{
    ENG_CHECK(h);
    if (!id || !rows || max_rows < 0) return DPD_E_ARG;
    return h->eng.compute_rows(0, id, rows, max_rows, n_cols, n_rows);
}

int dpd_write_restart(dpd_engine* h, const char* path)
{
    ENG_CHECK(h);
    if (!path) return DPD_E_ARG;
    return h->eng.write_restart(path);
}

int dpd_read_restart(dpd_engine* h, const char* path)
{
    ENG_CHECK(h);
    if (!path) return DPD_E_ARG;
    return h->eng.read_restart(path);
}

int dpd_compute_dump_open(dpd_engine* h, const char* id, const char* path)
{
    ENG_CHECK(h);
    if (!id) return DPD_E_ARG;
    return h->eng.compute_dump_open(id, path ? path : "");
}

int dpd_dump_close(dpd_engine* h)
{
    ENG_CHECK(h);
    return h->eng.dump_close();
}

int dpd_bond_compute_aos(dpd_engine* h, const float* d_pos, const int* d_bondlist, int n_bonds, float* d_force,
                         float* d_bond_pe, float* d_virial)
{
    ENG_CHECK(h);
    return h->eng.bond_compute_aos(d_pos, d_bondlist, n_bonds, d_force, d_bond_pe, d_virial);
}

int dpd_nve_aos(dpd_engine* h, int phase, const int* d_group, int n_group, const int* d_type, float* d_pos,
                float* d_uwpos, float* d_vel, const float* d_force)
{
    ENG_CHECK(h);
    return h->eng.nve_aos(phase, d_group, n_group, d_type, d_pos, d_uwpos, d_vel, d_force);
}

int dpd_get_spring_records(dpd_engine* h, double* rows, int max_rows, int* n_rows)
{
    ENG_CHECK(h);
    if (!rows || max_rows < 0) return DPD_E_ARG;
    return h->eng.spring_records(0, rows, max_rows, n_rows);
}

int dpd_get_state(dpd_engine* h, double* x, double* v, int* image, double* f)
{
    ENG_CHECK_ANY(h);
    if (h->f64) return h->f64->get_state(x, v, image, f);
    return h->eng.get_state(0, x, v, image, f);
}

int dpd_set_state(dpd_engine* h, const double* x, const double* v)
{
    ENG_CHECK_ANY(h);
    if (h->f64) return h->f64->set_state(x, v);
    return h->eng.set_state(0, x, v);
}

int dpd_get_density(dpd_engine* h, double* rho)
{
    ENG_CHECK(h);
    if (!rho) return DPD_E_ARG;
    return h->eng.get_density(0, rho);
}

int dpd_get_cells(dpd_engine* h, int* cell, float* offset, int* nc, float* w, float* cut2)
{
    ENG_CHECK(h);
    return h->eng.get_cells(0, cell, offset, nc, w, cut2);
}

int dpd_get_neighbors(dpd_engine* h, int* pairs, int64_t cap, int64_t* n_pairs)
{
    ENG_CHECK(h);
    return h->eng.get_neighbors(0, pairs, cap, n_pairs);
}

int dpd_compute_rdf(dpd_engine* h, int ta, int tb, double rmax, int nbins, double* g)
{
    ENG_CHECK(h);
    return h->eng.compute_rdf_now(0, ta, tb, rmax, nbins, g);
}

int dpd_rdf_config(dpd_engine* h, int ta, int tb, double rmax, int nbins, int every)
{
    ENG_CHECK(h);
    return h->eng.rdf_config(0, ta, tb, rmax, nbins, every);
}

int dpd_rdf_result(dpd_engine* h, double* g, int64_t* nsamples)
{
    ENG_CHECK(h);
    if (!g) return DPD_E_ARG;
    return h->eng.rdf_result(0, g, nsamples);
}

int dpd_get_info(dpd_engine* h, int64_t* step, int64_t* n_builds, int64_t* n_atoms, int64_t* device_bytes)
{
    ENG_CHECK_ANY(h);
    if (h->f64) {  // cell grids are rebuilt every step: builds = steps
        if (step) *step = h->f64->steps_done();
        if (n_builds) *n_builds = h->f64->steps_done() + 1;
        if (n_atoms) *n_atoms = h->f64->n_atoms();
        if (device_bytes) *device_bytes = h->f64->device_bytes();
        return DPD_OK;
    }
    if (step) *step = h->eng.steps_done(0);
    if (n_builds) *n_builds = h->eng.n_builds();
    if (n_atoms) *n_atoms = h->eng.total_atoms();
    if (device_bytes) *device_bytes = h->eng.device_bytes();
    return DPD_OK;
}

int dpd_get_list_stats(dpd_engine* h, int64_t* n_pairs, int64_t* n_atoms, int64_t* n_builds)
{
    ENG_CHECK(h);
    return h->eng.list_stats(n_pairs, n_atoms, n_builds);
}

int dpd_set_tuning(dpd_engine* h, const dpd_tuning* t)
{
    ENG_CHECK(h);
    return h->eng.set_tuning(t);
}

int dpd_write_data(dpd_engine* h, const char* path)
{
    ENG_CHECK_ANY(h);
    if (h->f64) return path ? h->f64->write_data(path) : DPD_E_ARG;
    if (!path) return DPD_E_ARG;
    return h->eng.write_data(0, path);
}

int dpd_time_steps(dpd_engine* h, uint32_t nsteps, double* total_ms, double* pair_ms, int64_t* pair_launches)
{
    ENG_CHECK_ANY(h);
    if (h->f64) {  // no separate pair timing in the parity mode
        if (pair_ms) *pair_ms = 0.0;
        if (pair_launches) *pair_launches = 0;
        return h->f64->time_steps(nsteps, total_ms);
    }
    return h->eng.time_steps(nsteps, total_ms, pair_ms, pair_launches);
}

const char* dpd_last_error(dpd_engine* h)
{
    if (!h) return g_create_err.c_str();
    if (h->f64) return h->f64->err.c_str();
    return h->eng.err.c_str();
}

int dpd_destroy(dpd_engine* h)
{
    delete h;
    return DPD_OK;
}

int dpd_pair_compute_aos(dpd_engine* h, const float* d_pos, const float* d_vel, const int* d_id,
                         const int* d_type, int n, uint32_t step, float* d_force, float* d_pe,
                         float* d_virial)
{
    ENG_CHECK(h);
    return h->eng.pair_compute_aos(d_pos, d_vel, d_id, d_type, n, step, d_force, d_pe, d_virial);
}

int dpd_batch_n(dpd_engine* h, int* n_rep)
{
    ENG_CHECK(h);
    if (n_rep) *n_rep = h->eng.n_rep();
    return DPD_OK;
}

int dpd_batch_get_thermo(dpd_engine* h, int rep, dpd_thermo* rows, int max_rows, int* n_rows)
{
    ENG_CHECK(h);
    return h->eng.get_thermo(rep, rows, max_rows, n_rows);
}

int dpd_batch_get_state(dpd_engine* h, int rep, double* x, double* v, int* image, double* f)
{
    ENG_CHECK(h);
    return h->eng.get_state(rep, x, v, image, f);
}

int dpd_batch_rdf_result(dpd_engine* h, int rep, double* g, int64_t* nsamples)
{
    ENG_CHECK(h);
    return h->eng.rdf_result(rep, g, nsamples);
}

}  // extern "C"
