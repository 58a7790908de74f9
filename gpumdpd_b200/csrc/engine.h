// engine.h -- host side of the engine: one packed batch of replicas on one GPU.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dpd_b200.h"
#include "dpd_common.h"
#include "dpd_io.h"
#include "dump.h"

struct StepArgs;  // kernels_step.cuh

namespace dpd {

// Host loop over [0, n) split across hardware threads (state conversion of millions of
// particles on every upload/download).
template <class F>
inline void parallel_for(int64_t n, F fn)
{
    int nt = (int)std::min<int64_t>(std::max(1u, std::thread::hardware_concurrency()), 32);
    if (n < 65536) nt = 1;
    std::vector<std::thread> th;
    for (int t = 1; t < nt; t++) th.emplace_back([=] { fn(n * t / nt, n * (t + 1) / nt); });
    fn(0, n / nt);
    for (auto& x : th) x.join();
}

struct Replica {
    RunInput in;
    SystemData sys;
    ForceField ff;
    RepDesc desc{};
    int nmax = 16;
    int maxb = 0;
    std::vector<int> crank;  // linear cell -> position in this replica's cell order
    double box_len[3] = {0, 0, 0};  // engine box: nc * w (float w), see layout()
};

struct DeviceBuffers {
    RepDesc* reps = nullptr;
    RepState* rstate = nullptr;
    int* warp_rep = nullptr;
    int* crank = nullptr;
    float4* coeff = nullptr;
    float2* mass = nullptr;
    float4* bondc = nullptr;
    float4* pos[2] = {nullptr, nullptr};  // double-buffered by *parity
    float4* vel[2] = {nullptr, nullptr};
    int4* img = nullptr;  // [tags] image counters by tag index, not permuted
    int2* bonds[2] = {nullptr, nullptr};
    int* parity = nullptr;
    float4 *force4 = nullptr, *last4 = nullptr;
    float* rho = nullptr;
    int *cell_rep = nullptr, *cell_lin = nullptr;
    int *cnt = nullptr, *cstart = nullptr, *skey = nullptr, *srank = nullptr, *tag2idx = nullptr;
    int *ncount = nullptr, *nlist = nullptr, *blocksum = nullptr;
    unsigned int* ticket = nullptr;  // k_permute's last-block counter
    unsigned int* ticket2 = nullptr; // k_integrate_adv's last-block counter
    double *acc = nullptr, *ring = nullptr;
    unsigned long long* rdf_hist = nullptr;
    int* build_flag = nullptr;
    uint32_t* phase = nullptr;
    uint32_t* limit = nullptr;  // per replica: last step it may evaluate (job length)
    FixDesc* fix = nullptr;     // per replica group fixes (allocated when any replica has one)
    FixOut* fixo = nullptr;
    double* spring_ring = nullptr;  // spring records (allocated when a spring writes a file)
    GCDesc* gc = nullptr;           // group computes (allocated when any replica has one)
    float4* uw0 = nullptr;
    double* gc_ring = nullptr;
    int* gc_count = nullptr;
    int* wall_ext = nullptr;        // wall extents (fix two_wall, compute wall_contact)
    int* tile_rep = nullptr;        // pair schedule 11: replica and coordinates of each tile
    int* tile_code = nullptr;
};

// the knobs of an engine created without tuning: pair schedule 8, linear cells (z
// fastest), the list build over column ranges
inline dpd_tuning engine_default_tuning()
{
    dpd_tuning t{};
    t.pair_variant = 8;
    t.cell_order = 0;
    t.build_variant = 5;
    return t;
}

class Engine {
public:
    Engine() = default;
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // replicas must be fully parsed; builds the packed layout and uploads it
    int init(std::vector<Replica>&& reps, const dpd_tuning* tune);
    int run(uint32_t nsteps);
    // enqueue nsteps steps on the engine's stream and return without waiting
    int run_async(uint32_t nsteps);
    int sync_and_check();
    int time_steps(uint32_t nsteps, double* total_ms, double* pair_ms, int64_t* launches);
    int get_thermo(int rep, dpd_thermo* rows, int max_rows, int* n_rows);
    int get_state(int rep, double* x, double* v, int* image, double* f);
    int set_state(int rep, const double* x, const double* v);
    int get_density(int rep, double* rho);
    int get_cells(int rep, int* cell, float* off, int* nc, float* w, float* cut2);
    int get_neighbors(int rep, int* pairs, int64_t cap, int64_t* n_pairs);
    int compute_rdf_now(int rep, int ta, int tb, double rmax, int nbins, double* g);
    int rdf_config(int rep, int ta, int tb, double rmax, int nbins, int every);
    int rdf_result(int rep, double* g, int64_t* nsamples);
    int write_data(int rep, const std::string& path);
    int set_tuning(const dpd_tuning* t);
    int list_stats(int64_t* n_pairs, int64_t* n_atoms, int64_t* n_builds);
    // rows {step, value} (temp, rho, msd) or {step, fx, fy, fz} (tf) of a group compute
    // of a replica, by compute ID (newest DPD_RING_ROWS); *n_cols = 2 or 4
    int compute_rows(int rep, const std::string& id, double* rows, int max_rows, int* n_cols, int* n_rows);
    // spring records {step, Fx, Fy, Fz, +-|F|, energy} of a replica (newest DPD_RING_ROWS)
    int spring_records(int rep, double* rows, int max_rows, int* n_rows);
    // trajectory frames of replica 0 in the reference's all.trj format, written by a host
    // thread from snapshots while the device keeps stepping (dump.cu)
    int dump_open(const std::string& path, uint32_t start, uint32_t every, bool unwrapped, bool force,
                  bool vel);
    // the frames of a `compute ID group dump freq file` of replica 0 (to its file, or path)
    int compute_dump_open(const std::string& id, const std::string& path);
    int dump_close();  // every open trajectory
    // exact checkpoint of every replica's FP32 state, forces and step counters; resume
    // into an engine made from the same run.in and system (restart.cu)
    int write_restart(const std::string& path);
    int read_restart(const std::string& path);
    // FP32 slots of a replica (host copies; the image counters already in tag order) to
    // FP64 arrays in tag order; false on a bad tag
    bool slots_to_tags(int rep, const float4* pos, const float4* vel, const int4* img, const float4* frc,
                       const float* spring_a, double* x, double* v, int* image, double* f) const;
    int pair_compute_aos(const float* d_pos, const float* d_vel, const int* d_id, const int* d_type,
                         int n, uint32_t step, float* d_force, float* d_pe, float* d_virial);
    // the bond force and fix nve on the reference's AoS buffers (kernels_aos.cuh)
    int bond_compute_aos(const float* d_pos, const int* d_bondlist, int n_bonds, float* d_force,
                         float* d_bond_pe, float* d_virial);
    int nve_aos(int phase, const int* d_group, int n_group, const int* d_type, float* d_pos, float* d_uwpos,
                float* d_vel, const float* d_force);

    int n_rep() const { return (int)reps_.size(); }
    const Replica& rep(int r) const { return reps_[r]; }
    int64_t steps_done(int r) const;
    int64_t n_builds();
    int64_t device_bytes() const { return dev_bytes_; }
    // priority of the engine's stream (CUDA stream priority: lower is served first); set
    // before init().  A server gives its longest jobs the highest priority.
    void set_stream_priority(int p) { stream_priority_ = p; }
    int64_t total_atoms() const;
    std::string err;

    // per-replica step limits: replica r evaluates no step beyond limit[r]
    int set_limits(const std::vector<uint32_t>& limit);
    // stop replica r after the work already enqueued on the engine's stream: its limit
    // becomes 0, so the next run segment leaves it inactive (no host wait)
    int freeze_async(int rep);
    int read_rstate(std::vector<RepState>& st);
    // enqueue a copy of every replica's state word into host memory (pinned, n_rep entries)
    // on the engine's stream, after the work enqueued so far
    int rstate_async(RepState* host);
    // the error of a device status word of replica r (DPD_OK when clean)
    int status_error(int status, int r);
    cudaStream_t stream() const { return stream_; }
    // device bytes init() would allocate for these replicas (no CUDA calls)
    static int64_t estimate_bytes(const std::vector<const Replica*>& reps);

private:
    int layout();
    void rank_cells(Replica& R) const;
    int upload_ranks();
    int alloc_and_upload();
    int upload_particles();
    void enqueue_step(cudaStream_t s, cudaEvent_t ev0, cudaEvent_t ev1);
    void enqueue_build(cudaStream_t s, bool list = true, bool wide = false);
    void enqueue_integrate_initial(cudaStream_t s);
    int build_graph();
    // pair schedule 11 (the cell-tile kernel, DPD engines): the tile table and staging
    // capacity for the current tuning; refresh_list() builds the neighbour list of the
    // current state on demand (that schedule builds none in its steps)
    bool use_tile() const { return tune_.pair_variant == 11 && !any_mdpd_; }
    // list-build variant 4: the list built from the same tiles (DPD engines)
    bool tile_build() const { return tune_.build_variant == 4 && !any_mdpd_ && !use_tile(); }
    int prepare_tiles();
    int refresh_list();
    int dump_frame(DumpWriter* w, uint32_t step);
    int dump_start(std::unique_ptr<DumpWriter> w);
    static bool dump_due(const DumpWriter* w, uint32_t step);
    static uint32_t next_dump(const DumpWriter* w, uint32_t s);
    int cur_parity();
    int staging();
    int cuda_fail(cudaError_t e, const char* what);
    template <class T> int dalloc(T** p, size_t n);

    std::vector<Replica> reps_;
    DeviceBuffers b_;
    dpd_tuning tune_{};
    cudaStream_t stream_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;
    int P_ = 0, C_ = 0, nmax_ = 16, maxb_ = 0;
    bool any_mdpd_ = false, any_dpd_ = false, bonds_ = false, rdf_ = false;
    bool any_spring_ = false, any_eos_ = false;  // some replica has a spring / an rvcm or recenter
    bool any_gc_ = false;                         // some replica has a temp/rho/msd/tf/wall_contact compute
    bool any_motion_ = false, any_twowall_ = false, any_wallc_ = false;  // fix move/wall_reflect, two_wall, wall_contact
    // the integrate variant with group fixes and computes
    bool ext() const { return any_spring_ || any_eos_ || any_gc_ || any_motion_ || any_twowall_; }
    void enqueue_two_wall(cudaStream_t s, const ::StepArgs& sa);
    std::vector<int> gc_ring_base_;               // first compute ring of each replica
    bool zero_pending_ = true;
    bool force_build_ = false;  // the next run starts with a list build (after a restart)
    bool ranks_dirty_ = false;  // new cell ranks (a changed cell order) wait for the next run
    uint32_t next_step_ = 0;
    std::vector<void*> allocs_;
    float4 *h_pos_ = nullptr, *h_vel_ = nullptr, *h_frc_ = nullptr;  // pinned staging
    int4* h_img_ = nullptr;
    int2* bonds_tag_ = nullptr;  // bond partner table in tag order (device)
    int4* angle_tbl_ = nullptr;   // angles: {coef index or -1, global tags i, j, k}
    float4* angle_coef_ = nullptr;  // {k, theta0 in radians, cos, sin theta0} per replica and angle type
    int* angle_wrep_ = nullptr;   // replica of each warp of the angle table
    int nang_ = 0;                // angle table length (padded to whole warps per replica)
    float *pe_slot_ = nullptr, *vir_slot_ = nullptr;  // per-atom PE/virial of the AoS entry
    int* aos_status_ = nullptr;    // status bits of the AoS bond / nve kernels (device)
    float* aos_mass_ = nullptr;    // masses per type for the AoS nve kernel (device)
    int aos_check(const char* what);
    bool aos_built_ = false;
    int64_t dev_bytes_ = 0;
    std::vector<uint32_t> host_target_;
    int ntiles_ = 0, tile_edge_ = 0, tile_smax_ = 0, tile_hc_ = 32;
    int stream_priority_ = 0;
    std::vector<std::unique_ptr<DumpWriter>> dumps_;
};

int make_replica(const std::string& run_in, const std::string& data_path, const std::string& base_dir,
                 Replica& out, std::string& err);
int make_replica_from_system(const std::string& run_in, const dpd_system* sys, Replica& out,
                             std::string& err);

}  // namespace dpd
