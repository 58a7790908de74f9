// fp64.h -- the FP64 parity engine: the timestep of the reference's -DDOUBLE build
// (src/main/common.cuh:38-42 with numtyp = double) on the GPU.
//
// The single-precision engine (engine.h) keeps cell-offset FP32 state; this one keeps
// wrapped FP64 positions in tag order and evaluates every pair from both sides, so its
// forces carry no FP32 rounding and no summation-order dependence beyond FP64's.  Its
// job is to separate precision effects from algorithm effects: against the reference's
// -DDOUBLE build it agrees step by step to FP64 rounding (dump print precision), where
// the FP32 engine agrees to FP32 rounding and then statistically.
//
// Scope: pair_style dpd and mdpd, bond_style harmonic and fene, angle_style harmonic,
// fix nve (on a group), thermo rows.  Any other fix, compute, dump or rdf command is
// refused at creation.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dpd_b200.h"
#include "engine.h"

namespace dpd {

class EngineF64 {
public:
    ~EngineF64();
    int init(Replica&& rep);
    int run(uint32_t nsteps);
    int get_thermo(dpd_thermo* rows, int max_rows, int* n_rows) const;
    int get_state(double* x, double* v, int* image, double* f);
    int set_state(const double* x, const double* v);
    int write_data(const std::string& path);
    int time_steps(uint32_t nsteps, double* total_ms);
    int64_t steps_done() const { return zero_pending_ && next_step_ == 0 ? 0 : (int64_t)next_step_ - 1; }
    int64_t n_atoms() const { return n_; }
    int64_t device_bytes() const { return bytes_; }
    std::string err;

private:
    int fail(cudaError_t e, const char* what);
    int upload_state(bool pos, bool vel);
    int eval_forces(uint32_t step, bool log);
    int check_status();
    int log_row(uint32_t step);

    Replica R_;
    int n_ = 0, ncell_ = 0, nc_[3] = {0, 0, 0};
    double L_[3] = {0, 0, 0};
    uint32_t next_step_ = 0;
    bool zero_pending_ = true;
    int64_t bytes_ = 0;
    cudaStream_t stream_ = nullptr;
    // device state, tag order
    double *x_ = nullptr, *v_ = nullptr, *f_ = nullptr, *rho_ = nullptr;
    double* q_ = nullptr;        // per-atom log terms: pair, bond, angle PE, virial[6]
    double* part_ = nullptr;     // per-block partial sums of the thermo reduction
    double* sums_ = nullptr;     // reduced thermo sums
    int *img_ = nullptr, *type_ = nullptr, *cnt_ = nullptr, *ccode_ = nullptr;
    int* status_ = nullptr;
    double4* crec_ = nullptr;    // cell records (position, atom index), cap_ per cell
    int *bstart_ = nullptr, *astart_ = nullptr;
    int2* bent_ = nullptr;       // bond partner index, bond type (1-based)
    int4* aent_ = nullptr;       // angle atoms i, j (apex), k as indices, angle type (1-based)
    double* tab_ = nullptr;      // coefficient tables: pair (5 per type pair), mass, bond (4), angle (2)
    int cap_ = 0;                // slots per cell
    std::vector<dpd_thermo> rows_;
};

}  // namespace dpd
