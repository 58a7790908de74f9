/*
 * dpd_b200.h -- C ABI of libdpd_b200.so, a B200-native DPD timestep engine.
 *
 * The reference (xxin125/gpumdpd, "GPUDPD") is a monolithic CUDA executable whose
 * plugin boundary is a set of C++ classes registered at static-init time
 * (Pair, Bond, Fix, Compute; src/force/pair.cuh:8-15, src/force/bond.cuh:8-15,
 * src/fix/fix.cuh:7-26, src/compute/compute.cuh:7-22) sharing a `System&` of raw
 * device pointers, driven by src/main/utils.cuh:166-314.  It has no FFI of its own,
 * so every entry point below names the reference interface whose job it takes over.
 *
 * Conventions
 *  - Every function returns an int status: 0 on success, a negative DPD_E_* code on
 *    failure (the reference calls exit(1) instead: src/main/common.cuh:46-60,175-200).
 *    dpd_last_error() gives the message of the most recent failure on that handle
 *    (or of a failed create when the handle is NULL).
 *  - A dpd_engine owns all of its device memory and its CUDA stream; one engine is
 *    used from one host thread at a time.  Nothing here exits the process.
 *  - Particles are identified by their 1-based tag (the data file's atom id); arrays
 *    returned "by tag" have tag-1 as their row index.  Types are 1-based.
 *  - Host arrays are plain C arrays; no torch or CUDA types cross the boundary.
 */
#ifndef DPD_B200_H
#define DPD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DPD_OK 0
#define DPD_E_ARG -1       /* invalid argument or command (run.in grammar error) */
#define DPD_E_IO -2        /* file cannot be read or written                       */
#define DPD_E_CUDA -3      /* a CUDA call failed                                    */
#define DPD_E_NOMEM -4     /* device memory could not be allocated / over budget    */
#define DPD_E_OVERFLOW -5  /* neighbour list or cell capacity exceeded (max_rho)    */
#define DPD_E_STATE -6     /* call not valid in the engine's current state          */
#define DPD_E_NUMERIC -7   /* non-finite position/velocity, or a FENE bond broke    */
#define DPD_E_NODEV -8     /* no CUDA device: there is no CPU fallback               */
#define DPD_E_CANCELLED -9 /* a served job was cancelled before it finished          */

typedef struct dpd_engine dpd_engine;

/* One system given as arrays instead of a data file (same content as the data file
 * read by src/system/read_data.cu:201-343).  x and v are double[3*n_atoms] rows in
 * `tag` order of the arrays given (any order; tags must be 1..n_atoms).  v may be
 * NULL (zero velocities, as a data file without a Velocities section).            */
typedef struct dpd_system {
    int n_atoms;
    int n_atomtypes;
    int n_bonds;       /* 0 for atom_style atomic */
    int n_bondtypes;
    double lo[3];
    double hi[3];
    const double* masses; /* [n_atomtypes] */
    const int* tag;       /* [n_atoms], 1-based, a permutation of 1..n_atoms */
    const int* type;      /* [n_atoms], 1-based */
    const int* mol;       /* [n_atoms] or NULL */
    const double* x;      /* [3*n_atoms] */
    const double* v;      /* [3*n_atoms] or NULL */
    const int* bonds;     /* [3*n_bonds]: type, tag_i, tag_j */
    int n_angles;         /* atom_style angle: harmonic angles (src/force/angle_harmonic.cu) */
    int n_angletypes;
    const int* angles;    /* [4*n_angles]: type, tag_i, tag_j (apex), tag_k */
} dpd_system;

/* Thermo row, the columns of thermo.txt (src/compute/thermo.cu:39-62,122-214) in
 * FP64, plus total momentum and kinetic energy. */
typedef struct dpd_thermo {
    int64_t step;
    double temp;
    double pair_pe;
    double bond_pe;
    double pressure;
    double p[6];        /* pxx pxy pxz pyy pyz pzz */
    double ke;
    double momentum[3];
    double angle_pe;    /* atom_style angle: the angle_pe column */
} dpd_thermo;

/* Launch/tuning knobs chosen by the autotuner (gpumdpd_b200/tune.py).  An engine,
 * batch or server created without a dpd_tuning runs pair_variant 8, cell_order 0 and
 * build_variant 5, with every other field zero. */
typedef struct dpd_tuning {
    int pair_block;        /* pair_variant 11: 3 = the tile kernel compiled for 3
                              CTAs per SM (more registers), else 4                */
    int pair_variant;      /* 0 = thread per particle, 1-3 = warp pair-queue,
                              4-5 = flattened warp schedule (small skins),
                              6 = flattened with the list build fused (DPD),
                              7-8 = flattened, log and non-log steps split (8 is
                              the default), 9 = as 8 with the i-side forces summed
                              per owner in the warp before the reduction,
                              10 = one thread per list entry, 11 = no neighbour
                              list: a CTA per tile of cells stages the tile's
                              neighbourhood in shared memory and evaluates its
                              pairs straight from the cell ranges (DPD engines;
                              mDPD runs 8)                                        */
    int cell_order;        /* 0 = linear cells (z fastest), 1 = Morton-ordered cells,
                              2 = x-y columns in Morton order, the cells of a column
                              consecutive (z fastest).  A change between runs takes
                              effect at the next run, which starts with a list build */
    int build_variant;     /* list build: 0 = cell ranges in registers, 4
                              blocks/SM; 1, 2 = cell ranges in shared memory, 6 or
                              8 blocks/SM; 3 = a thread per (slot, stencil cell)
                              (grids up to 1184 blocks; larger ones use 0); 4 = a
                              CTA per tile of cells walking the candidates staged
                              in shared memory (DPD engines; mDPD runs 0); 5 = a
                              thread per slot walking five column ranges of slots
                              (cells z-1..z+1 of a column, contiguous under cell
                              order 0 or 2; cell by cell where they are not)      */
    int launch_mode;       /* 0 = small grids (up to 1184 blocks of 256 slots) run the
                              pair pass as one launch (schedule 4 in place of 8) and
                              the integrate as one, the step's bookkeeping in the
                              integrate's last block; tiny ones (up to 148 blocks)
                              also build the list with a thread per (slot, stencil
                              cell) (in place of build variant 0 or 5) and run the pair
                              pass with a thread per list entry (schedule 10);
                              1 = never; 2 = always; 3 = as 0 without the tiny-grid
                              kernels (the server's cohorts: engines that share
                              the GPU run better on fewer, fuller blocks)         */
    int tile;              /* pair_variant 11: home cells per tile edge, 1..6 (0 = the
                              engine's choice)                                    */
    int tile_capacity;     /* pair_variant 11: particles a CTA stages (0 = 1.5 times
                              the mean of a tile's neighbourhood, plus 64); a
                              neighbourhood beyond it is taken a home cell at a
                              time                                                */
    int reserved;
} dpd_tuning;

/* ---- plain engine: replaces main()/read_info/preprocess/zero_step/simulation
 *      (src/main/main.cu:15-72, src/main/utils.cuh:117-314) ---------------------- */

/* Create an engine from the text of a run.in file (the reference's command grammar,
 * src/main/read_in.cu:40-290 plus each plugin's isEnabled/validateParams) and either
 * the data file it names (data_path == NULL: use the read_data line, resolved
 * relative to base_dir when base_dir is not NULL) or an explicit data_path. */
int dpd_create(const char* run_in_text, const char* data_path, const char* base_dir,
               dpd_engine** out);

/* Same, with the system given as arrays (the read_data line is then ignored). */
int dpd_create_from_system(const char* run_in_text, const dpd_system* sys, dpd_engine** out);

/* Advance nsteps timesteps (the first call also performs the reference's zero step:
 * neighbour build, force evaluation and thermo at step 0).  Asynchronous on the
 * engine's stream except for error checking at the end. */
int dpd_run(dpd_engine* eng, uint32_t nsteps);

/* Wait for outstanding work and report any device-side error status. */
int dpd_sync(dpd_engine* eng);

/* Thermo rows logged so far (every `thermo` steps, as src/compute/thermo.cu:96-220).
 * Copies up to max_rows of the most recent rows; *n_rows receives the number copied. */
int dpd_get_thermo(dpd_engine* eng, dpd_thermo* rows, int max_rows, int* n_rows);

/* Trajectory frames in the reference's all.trj format (Dump::dump, src/system/dump.cu:23-201):
 * `ITEM:` headers, then `id type x y z [fx fy fz] [vx vy vz]` per atom in tag order with
 * nine decimals, at step 0 when start is 0 and at every step >= start with
 * (step - start) % every == 0 (src/main/utils.cuh:198-202,293-297).  every <= 0 takes
 * start, frequency and columns from the run.in's `dump` command (DPD_E_ARG without one).
 * flags: DPD_DUMP_UNWRAPPED (image-unwrapped positions), DPD_DUMP_FORCE, DPD_DUMP_VEL.
 * Frames are snapshotted on the device and written by a host thread while the run goes
 * on; dpd_dump_close (or dpd_destroy) waits for the last frame.  Velocities are written
 * whenever DPD_DUMP_VEL is set (the reference's dump refreshes them only with forces). */
#define DPD_DUMP_UNWRAPPED 1
#define DPD_DUMP_FORCE 2
#define DPD_DUMP_VEL 4
int dpd_dump_open(dpd_engine* eng, const char* path, int64_t start, int64_t every, int flags);
/* The frames of the run.in's `compute ID groupID dump frequency filename`
 * (src/compute/compute_dump.cu:40-130): the group's atoms, `id type x y z` (atom_style
 * atomic) or `id mol type x y z`, wrapped positions, every frequency steps from the zero
 * step on, to `path` (NULL: the compute's file name).  Written like dpd_dump_open's. */
int dpd_compute_dump_open(dpd_engine* eng, const char* id, const char* path);
/* Wait for the last frame of every open trajectory and close them. */
int dpd_dump_close(dpd_engine* eng);

/* Exact checkpoint and resume (new; the reference restarts from a write_data file at
 * step 0, which replays its random-force stream, src/force/pair_dpd.cu:213).  The file
 * holds the FP32 state as the engine keeps it (cell codes and offsets, velocities, image
 * counters), the forces of the last evaluated step, the step counter and the fix results
 * of every replica.  dpd_read_restart loads it into an engine created from the same run.in
 * and system (DPD_E_ARG when atom count, types or cell grid differ); the next dpd_run
 * continues with the following step.  Thermo rows, spring records and RDF sums restart
 * empty. */
int dpd_write_restart(dpd_engine* eng, const char* path);
int dpd_read_restart(dpd_engine* eng, const char* path);

/* Rows of a group compute by its ID (`compute ID group temp|rho|msd|tf freq ... file`,
 * src/compute/compute_temp.cu, compute_rho.cu, compute_msd.cu, compute_tf.cu), the values
 * the reference writes to its file every freq steps from the zero step on: {step, T} with
 * T = 2 KE / (3 Ng - 3); {step, count in the region / region volume} (wrapped positions);
 * {step, mean |x - x0|^2} over the group (unwrapped, x0 the data file's positions);
 * {step, Fx, Fy, Fz} summed over the group.  *n_cols = 2 or 4; rows row-major, up to
 * max_rows of the most recent (the device keeps 2048). */
int dpd_get_compute(dpd_engine* eng, const char* id, double* rows, int max_rows, int* n_cols, int* n_rows);

/* Bond::compute_force on the reference's own device buffers (Bond_harmonic, src/force/
 * bond_harmonic.cu:167-402): d_bondlist holds n_bonds entries {type, id_i, id_j} (1-based
 * ids, atom index = id - 1), d_pos the FP32 AoS positions, d_force the forces the bond
 * force is added to.  On log steps pass d_bond_pe (per bond, overwritten) and/or d_virial
 * (6 per atom, half of each bond's r_a F_b added to both atoms); NULL otherwise.  The bond
 * style and coefficients are the engine's run.in's (harmonic, or this engine's fene).
 * Runs on the legacy default stream, in order with the caller's kernels. */
int dpd_bond_compute_aos(dpd_engine* eng, const float* d_pos, const int* d_bondlist, int n_bonds,
                         float* d_force, float* d_bond_pe, float* d_virial);

/* Fix nve on the reference's own device buffers (src/fix/fix_nve.cu:30-152) for the atom
 * indices of a group (d_group, n_group): phase 0 the initial half kick and drift (positions
 * wrapped into the box, d_uwpos advanced when not NULL), phase 1 the final half kick.  dt,
 * masses and box are the engine's run.in and system's.  Legacy default stream, like
 * dpd_bond_compute_aos. */
int dpd_nve_aos(dpd_engine* eng, int phase, const int* d_group, int n_group, const int* d_type, float* d_pos,
                float* d_uwpos, float* d_vel, const float* d_force);

/* Records of `fix ... spring k x y z r0 file freq` (src/fix/fix_spring.cu:340-360, the
 * rows it writes to its file): 6 doubles per row {step, Fx, Fy, Fz, +-|F|, energy}, every
 * freq steps from the zero step on.  Copies up to max_rows of the most recent rows (the
 * device keeps the last 2048); *n_rows = 0 without such a fix. */
int dpd_get_spring_records(dpd_engine* eng, double* rows, int max_rows, int* n_rows);

/* Current state by tag: x wrapped into the box, v, image counters, forces of the
 * last evaluated step (any pointer may be NULL). Replaces Dump/write_data reads of
 * d_pos/d_vel/d_force (src/system/dump.cu:23-201). */
int dpd_get_state(dpd_engine* eng, double* x, double* v, int* image, double* f);

/* Overwrite positions/velocities by tag (x wrapped into the box on load). */
int dpd_set_state(dpd_engine* eng, const double* x, const double* v);

/* Local density of the last mDPD evaluation by tag (src/force/pair_mdpd.cu:219-300). */
int dpd_get_density(dpd_engine* eng, double* rho);

/* Engine's internal FP32 representation by tag: cell coordinates (3 ints) and
 * offsets within the cell (3 floats); plus the grid (nc[3], w[3]).  For parity
 * tests of the neighbour predicate. */
int dpd_get_cells(dpd_engine* eng, int* cell, float* offset, int* nc, float* w, float* cut2);

/* Current half neighbour list as unordered tag pairs (lo, hi), at most cap pairs;
 * *n_pairs receives the total (Neigh_list::build, src/force/neigh_list.cu:397-479). */
int dpd_get_neighbors(dpd_engine* eng, int* pairs, int64_t cap, int64_t* n_pairs);

/* Radial distribution function g(r) between types ta and tb, nbins bins on [0,rmax),
 * evaluated on the current state (new: the reference has no RDF). */
int dpd_compute_rdf(dpd_engine* eng, int ta, int tb, double rmax, int nbins, double* g);

/* Accumulated RDF over sampling steps configured with dpd_rdf_config. */
int dpd_rdf_config(dpd_engine* eng, int ta, int tb, double rmax, int nbins, int every);
int dpd_rdf_result(dpd_engine* eng, double* g, int64_t* nsamples);

/* Counters: steps done, neighbour-list builds, particles, bytes of device memory. */
int dpd_get_info(dpd_engine* eng, int64_t* step, int64_t* n_builds, int64_t* n_atoms,
                 int64_t* device_bytes);

/* Neighbour-list statistics of replica 0: pairs in the current half list, particles,
 * list builds so far (the mean half-list length is pairs/particles). */
int dpd_get_list_stats(dpd_engine* eng, int64_t* n_pairs, int64_t* n_atoms, int64_t* n_builds);

/* Apply tuning knobs (takes effect at the next run). */
int dpd_set_tuning(dpd_engine* eng, const dpd_tuning* t);

/* Write a data file in the reference's write_data format (src/system/read_data.cu:473-637). */
int dpd_write_data(dpd_engine* eng, const char* path);

/* Time `nsteps` steps on the device with CUDA events: total milliseconds of the
 * timed region and of the pair kernel alone (sum over launches). */
int dpd_time_steps(dpd_engine* eng, uint32_t nsteps, double* total_ms, double* pair_ms,
                   int64_t* pair_launches);

const char* dpd_last_error(dpd_engine* eng);
int dpd_destroy(dpd_engine* eng);

/* ---- in-loop drop-in for Pair::compute_force on the reference's own buffers ---
 * Computes the pair force of the enabled style into the reference's AoS device
 * arrays, from its AoS positions/velocities (d_pos/d_vel numtyp[3N] with numtyp =
 * float, d_id/d_type int[N]); same memset-then-accumulate contract as
 * Pair_dpd::compute_force (src/force/pair_dpd.cu:564-633) and Pair_mdpd's
 * (src/force/pair_mdpd.cu:689-779): d_force is overwritten; when d_pe/d_virial are
 * not NULL they are overwritten with per-atom PE and the 6-component per-atom virial
 * ((1/2) r (x) F per pair to each atom).  The engine keeps its own cell list and
 * rebuilds it when any particle moved more than skin/2 since the last build.  All
 * pointers are device pointers; runs on the engine's stream and synchronises.   */
int dpd_pair_compute_aos(dpd_engine* eng, const float* d_pos, const float* d_vel,
                         const int* d_id, const int* d_type, int n, uint32_t step,
                         float* d_force, float* d_pe, float* d_virial);

/* ---- batched replicas (one engine, many independent systems) --------------------
 * Replicas are packed into one offset-indexed particle array and advanced together
 * by the same kernels, one launch per stage; the timestep is captured in a CUDA
 * graph.  run_in_texts[r] / systems[r] describe replica r as for the plain engine. */
int dpd_batch_create(int n_rep, const char* const* run_in_texts, const dpd_system* systems,
                     const dpd_tuning* tune, dpd_engine** out);
int dpd_batch_n(dpd_engine* eng, int* n_rep);
int dpd_batch_get_thermo(dpd_engine* eng, int rep, dpd_thermo* rows, int max_rows,
                         int* n_rows);
int dpd_batch_get_state(dpd_engine* eng, int rep, double* x, double* v, int* image,
                        double* f);
int dpd_batch_rdf_result(dpd_engine* eng, int rep, double* g, int64_t* nsamples);

/* ---- FP64 parity mode: the reference's -DDOUBLE build (src/main/common.cuh:38-42,
 *      numtyp = double) ------------------------------------------------------------
 * An engine in double precision: wrapped FP64 positions in tag order, every pair taken
 * from both sides (no force atomics, runs repeat bit for bit), the Saru tail of the
 * -DDOUBLE build.  It separates precision effects from algorithm effects: against the
 * -DDOUBLE build it agrees step by step to FP64 rounding.  Covers pair_style dpd/mdpd,
 * bond_style harmonic/fene, angle_style harmonic, fix nve and thermo; other fixes,
 * computes and dumps are refused at creation.  The handle answers dpd_run, dpd_sync,
 * dpd_get_thermo, dpd_get_state, dpd_set_state, dpd_get_info, dpd_write_data,
 * dpd_time_steps (total time only), dpd_last_error and dpd_destroy; other calls return
 * DPD_E_ARG.  sys != NULL: the system from arrays (as
 * dpd_create_from_system), else the run.in's data file (as dpd_create). */
int dpd_create_fp64(const char* run_in_text, const char* data_path, const char* base_dir,
                    const dpd_system* sys, dpd_engine** out);

/* ---- serving: continuous batching of DPD jobs -----------------------------------
 * No counterpart in the reference (one run.in per process, src/main/main.cu:15-72).
 * A server owns a device-memory budget.  Jobs are submitted at any time; at each
 * scheduling point (every `chunk` steps) finished jobs are retired, their memory is
 * released, and queued jobs are admitted while they fit the budget; all admitted
 * jobs advance together in one packed batch.  Each job keeps its own tags, seed and
 * step counter, so its trajectory does not depend on which other jobs share the
 * batch.  A job that fails (a non-finite state, a broken bond, a list overflow) fails
 * alone: its replica is frozen and the other jobs of its batch run on (the reference
 * exits the process on any such error, src/main/common.cuh:46-60). */
typedef struct dpd_server dpd_server;

typedef struct dpd_job_result {
    int64_t job_id;
    int status;            /* 0 done, >0 still queued/running, <0 error code      */
    int64_t steps;
    double mean_temp;      /* mean over logged rows after the first               */
    double mean_pressure;
    double submit_s, start_s, finish_s; /* host clock seconds since server creation */
    dpd_thermo last;
    double stderr_temp;    /* standard errors of the two means: block averages over  */
    double stderr_pressure;/* up to 10 blocks of those rows (NaN with fewer than 4)   */
} dpd_job_result;

/* `tune` (NULL: the engine defaults) applies to every cohort; its launch_mode 0 runs
 * as 3, since the cohorts share the GPU. */
int dpd_server_create(double hbm_budget_bytes, int chunk_steps, const dpd_tuning* tune,
                      dpd_server** out);
/* Submit a job (copies the inputs); *job_id receives its id. */
int dpd_server_submit(dpd_server* srv, const char* run_in_text, const dpd_system* sys,
                      int64_t* job_id);
/* Admission window.  While jobs are running, queued jobs are admitted together once
 * min_jobs are waiting or the oldest has waited max_wait_s seconds (defaults 1 and 0:
 * admit at every scheduling point).  Jobs admitted together share one packed engine,
 * so a window trades a bounded extra wait for fewer, larger batches.  An idle server
 * admits at once. */
int dpd_server_set_policy(dpd_server* srv, double max_wait_s, int min_jobs);
/* One scheduling pass (admit; for every cohort whose chunk of steps has completed,
 * retire its finished jobs and enqueue its next chunk; never waits for a running chunk).
 * Call it in a loop; *n_active and *n_queued receive the running and queued job counts
 * after the pass. */
int dpd_server_step(dpd_server* srv, int* n_active, int* n_queued);
int dpd_server_result(dpd_server* srv, int64_t job_id, dpd_job_result* res);
/* Cancel a queued or running job: a queued job leaves the queue; a running job's replica
 * is frozen at the end of the chunks already in flight and the other jobs of its batch
 * run on; when it was the last running job of its batch, the batch's device memory
 * returns to the budget at the next scheduling point.  The job's status becomes
 * DPD_E_CANCELLED.  DPD_E_STATE for a job that has already finished or failed. */
int dpd_server_cancel(dpd_server* srv, int64_t job_id);
int dpd_server_job_state(dpd_server* srv, int64_t job_id, double* x, double* v);
int dpd_server_job_rdf(dpd_server* srv, int64_t job_id, double* g, int64_t* nsamples);
int dpd_server_stats(dpd_server* srv, int64_t* particle_steps, double* busy_s,
                     int64_t* device_bytes);
const char* dpd_server_last_error(dpd_server* srv);
int dpd_server_destroy(dpd_server* srv);

/* ---- pair force without device allocation ---------------------------------------
 * No counterpart in the reference.  For callers that may not allocate device memory:
 * a force plugin inside a host MD code or framework that owns all device memory
 * (its caching allocator or a fixed arena set up at start-up), and fixed-latency
 * loops, where cudaMalloc/cudaFree can synchronize the whole device and stall other
 * streams, or fail when the device is nearly full in the middle of a run.  Computes the
 * pair_style dpd force (Saru random force keyed on min/max id, seed + step) on AoS
 * device buffers, like dpd_pair_compute_aos, but needs no engine and calls no
 * cudaMalloc, cudaFree or allocating library routine: the cell binning lives in a
 * file-scope static device array of about 5 MB, which every device that loads the
 * library holds until exit.  Limits: n <= DPD_NOALLOC_MAX_ATOMS, at most
 * DPD_NOALLOC_MAX_CELLS cells of edge >= max rc with at least 3 per dimension,
 * ntypes <= DPD_NOALLOC_MAX_TYPES; larger inputs return DPD_E_ARG before any launch.
 * Positions must lie in [lo, hi): one more than a thousandth of a cell outside, an id
 * below 1 or a type out of range returns DPD_E_ARG (after the launches).  CUDA loads
 * device code lazily, so the first call on a device loads the library's kernels and
 * the array with them (the driver reserves the array's device memory at that moment)
 * and resolves the array's device address (cudaGetSymbolAddress, with that device
 * current; again whenever the device's CUDA context has changed).  Make that first call
 * at start-up, as a warm-up, and before any stream capture.  All calls share the array
 * and it keeps the last call's contents (each call clears what must start at zero), so
 * calls that overlap on the GPU -- other streams, other threads -- race and must be
 * serialized by the caller.  Work goes on `stream` (a cudaStream_t, NULL = legacy default
 * stream); the call waits for that work (it reads back a status word) and returns after
 * the forces are written; d_force is overwritten. */
#define DPD_NOALLOC_MAX_ATOMS 262144
#define DPD_NOALLOC_MAX_CELLS 262144
#define DPD_NOALLOC_MAX_TYPES 8

typedef struct dpd_pair_params {
    double lo[3];
    double hi[3];
    int ntypes;
    double coeff[DPD_NOALLOC_MAX_TYPES][DPD_NOALLOC_MAX_TYPES][3]; /* A, gamma, rc; symmetric */
    double kT;      /* pair_style dpd temp */
    double dt;      /* timestep */
    uint32_t seed;  /* pair_style dpd seed */
} dpd_pair_params;

int dpd_pair_forces_noalloc(const dpd_pair_params* params, const float* d_pos, const float* d_vel,
                            const int* d_id, const int* d_type, int n, uint32_t step, float* d_force,
                            void* stream);

/* Library version string. */
const char* dpd_version(void);

#ifdef __cplusplus
}
#endif
#endif /* DPD_B200_H */
