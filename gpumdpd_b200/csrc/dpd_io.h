// dpd_io.h -- the reference's command surface: run.in grammar, data files, thermo.txt.
#pragma once
#include <array>
#include <cstdint>
#include <functional>
#include <map>
#include <string>
#include <vector>

namespace dpd {

// Global commands of run.in, src/main/read_in.cu:40-290 (Read_in::read).
struct RunInput {
    int atom_style = -1;  // 0 atomic, 1 bond, 2 angle
    double global_cut = 0, skin = 0, max_rho = 0;
    int nl_f = 1;
    double dt = 0;
    unsigned log_f = 0;
    unsigned nsteps = 0;
    std::string read_data;
    bool write_data = false;
    std::string write_data_name;
    bool dump = false;
    unsigned dump_start = 0, dump_f = 1;
    bool dump_wrapped = false, dump_force = false, dump_vel = false;
    std::vector<std::vector<std::string>> lines;  // every command line, tokenized
    std::vector<std::string> raw;                 // the same lines as text
};

// Contents of a data file (src/system/read_data.cu:145-468), rows indexed by tag-1.
struct SystemData {
    int n_atoms = 0, n_atomtypes = 0, n_bonds = 0, n_bondtypes = 0, n_angles = 0, n_angletypes = 0;
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    std::vector<double> masses;
    std::vector<int> type, mol;
    std::vector<double> x, v;
    std::vector<int> bonds;  // type, tag_i, tag_j
    std::vector<int> angles;  // type, tag_i, tag_j (apex), tag_k
    bool has_velocities = false;
};

// Group computes written to a file every `frequency` steps (src/compute/compute_temp.cu,
// compute_rho.cu, compute_msd.cu, compute_tf.cu): the group's temperature, its number
// density inside a box region, its mean squared displacement from the initial unwrapped
// positions, and its total force.
enum { GC_TEMP = 1, GC_RHO = 2, GC_MSD = 3, GC_TF = 4, GC_WALL = 5 };
struct GroupCompute {
    std::string id, group, file;
    int kind = GC_TEMP;
    unsigned frequency = 1;
    uint32_t type_mask = 0;
    double region[6] = {0, 0, 0, 0, 0, 0};  // rho: xlo xhi ylo yhi zlo zhi
    // wall_contact (src/compute/compute_wall_contact.cu): group atoms within `cutoff` of
    // the wall group's extreme position along `dir` (side +1: its maximum, lo wall; -1:
    // its minimum, hi wall)
    uint32_t wall_mask = 0;
    int wall_side = 1, wall_dir = 2;
    double cutoff = 0;
};

// compute ID groupID dump frequency filename (src/compute/compute_dump.cu): wrapped
// positions of the group every `frequency` steps from the zero step on.
struct ComputeDump {
    std::string id, file;
    uint32_t mask = 0;
    unsigned frequency = 1;
};

// Wall fixes (src/fix/fix_move.cu, fix_wall_reflect.cu, fix_two_wall.cu); several of each.
struct FixMove {      // initial_integrate: v = V and x += V dt for the group
    uint32_t mask = 0;
    double v[3] = {0, 0, 0};
};
struct FixWallReflect { // post_integrate: mirror group atoms outside [lo, hi] along dir
    uint32_t mask = 0;
    int dir = 2;
    double lo = 0, hi = 0;
};
struct FixTwoWall {   // post_integrate: the same between max(lo-wall group) and min(hi-wall group)
    uint32_t mask = 0, lo_mask = 0, hi_mask = 0;
    int dir = 2;
};

struct ComputeRdf {
    std::string id, file;
    int ta = 1, tb = 1, nbins = 150, every = 100;
    double rmax = 3.0;
};

// Group fixes on the timestep (src/fix/fix_spring.cu, fix_rvcm.cu, fix_recenter.cu); at most
// one of each per system.  mask: the group's types (bit type-1).
struct FixSpring {   // post_force: F = -k (|r| - r0) r/|r| on the group's centre of mass
    bool on = false;
    uint32_t mask = 0;
    double k = 0, c[3] = {0, 0, 0}, r0 = 0;
    std::string file;    // optional record file: step Fx Fy Fz +-|F| energy every file_freq steps
    unsigned file_freq = 0;
};
struct FixRvcm {     // end_of_step every freq: remove the group's centre-of-mass velocity
    bool on = false;
    uint32_t mask = 0;
    unsigned freq = 1;
    int flag[3] = {0, 0, 0};
};
struct FixRecenter { // end_of_step every freq: move the group's centre of mass to c
    bool on = false;
    uint32_t mask = 0;
    unsigned freq = 1;
    double c[3] = {0, 0, 0};
};

// Pair/bond styles and their coefficients, groups, fixes and computes, parsed after
// the data file is known (as the reference's isEnabled/validateParams do).
struct ForceField {
    int pair_style = -1;  // 0 dpd (src/force/pair_dpd.cu:19-173), 1 mdpd (pair_mdpd.cu:21-192)
    double temp = 0, rc = 0, rd = 0;
    unsigned seed = 0;
    int ntypes = 0;
    std::vector<std::array<double, 5>> coeff;  // triangular index: A, B, gamma, rc, rd
    int bond_style = 0;                        // 0 none, 1 harmonic, 2 fene
    std::vector<std::array<double, 4>> bond_coeff;
    int angle_style = 0;                       // 0 none, 1 harmonic (src/force/angle_harmonic.cu)
    std::vector<std::array<double, 2>> angle_coeff;  // k, theta0 in degrees
    std::map<std::string, std::vector<int>> groups;
    uint32_t integ_mask = 0;  // types integrated by fix nve
    FixSpring spring;
    FixRvcm rvcm;
    FixRecenter recenter;
    std::vector<GroupCompute> gcs;
    std::vector<ComputeDump> cdumps;
    std::vector<FixMove> moves;
    std::vector<FixWallReflect> reflects;
    std::vector<FixTwoWall> twowalls;
    std::vector<ComputeRdf> rdfs;
};

int tri_index(int ti, int tj, int nt);  // src/force/pair_dpd.cu:134, 0-based

int parse_run_in(const std::string& text, RunInput& out, std::string& err);
int read_data_file(const std::string& path, int atom_style, SystemData& out, std::string& err);
int parse_force_field(const RunInput& in, const SystemData& sys, ForceField& ff, std::string& err);
int write_data_file(const std::string& path, int atom_style, const SystemData& sys,
                    std::string& err);

}  // namespace dpd
