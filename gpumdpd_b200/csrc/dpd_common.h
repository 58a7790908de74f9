// dpd_common.h -- types shared by the host engine and the sm_100a kernels.
#pragma once
#include <stdint.h>

#define DPD_MAX_TYPES 32
#define DPD_NACC 48          // FP64 accumulators per replica and slot
#define DPD_NACC_THERMO 20   // the first DPD_NACC_THERMO feed the thermo row
#define DPD_ACC_SLOTS 32     // atomic spreading slots per replica
#define DPD_THERMO_FIELDS 17 // doubles per logged thermo row
#define DPD_RING_ROWS 2048   // thermo rows kept per replica on the device
#define DPD_CELL_BITS 10     // bits per cell coordinate in the packed cell code
#define DPD_MAX_NC ((1 << DPD_CELL_BITS) - 1)
#define DPD_TYPE_BITS 5      // type-1 in the low bits of the packed tag word
#define DPD_MAX_TAG ((1 << (32 - DPD_TYPE_BITS)) - 1)

// accumulator slots
enum {
    ACC_KE = 0,      // sum 1/2 m v^2
    ACC_KIN = 1,     // 6: sum m v_a v_b
    ACC_PAIR_PE = 7,
    ACC_BOND_PE = 8,
    ACC_VIR = 9,     // 6: sum over pairs and bonds of r_a F_b
    ACC_MOM = 15,    // 3: sum m v
    ACC_NONFINITE = 18,
    ACC_ANGLE_PE = 19,
    // group-fix sums, consumed (and zeroed) by the fix reductions of the same step
    ACC_SPRING_COM = 20,  // 3: sum over the spring group of m x_unwrapped
    ACC_RVCM_P = 23,      // 3: sum over the rvcm group of m v
    ACC_RECENTER_COM = 26, // 3: sum over the recenter group of m x_unwrapped
    ACC_GC = 32            // 3 per group compute (DPD_MAX_GC of them), consumed by k_advance
};
#define DPD_MAX_GC 4

// status bits (per replica, device)
enum {
    ST_LIST_OVERFLOW = 1,
    ST_NONFINITE = 2,
    ST_BOND_MISSING = 4,
    ST_FENE_BROKEN = 8,
    ST_BOND_OVERFLOW = 16,
    ST_BAD_INPUT = 32,  // an AoS input carried an id or type outside the system
    ST_WALL_ORDER = 64, // fix two_wall: the high wall is not above the low wall
    ST_CONTACT_BOX = 128, // compute wall_contact: contact region outside the box
};

// Per-replica constant description (device copy, read through the L1 cache).
struct RepDesc {
    int p_begin;    // first particle slot (multiple of 32)
    int p_end;      // one past the last real particle
    int p_cap_end;  // one past the last slot (multiple of 32); [p_end, p_cap_end) are ghosts
    int n_real;
    int c_begin;    // first cell of this replica in the packed cell arrays
    int ncell;      // cells nc[0]*nc[1]*nc[2]; local cell `ncell` holds the ghosts
    int nc[3];
    int tag_base;   // offset of this replica's tags in tag2idx
    float w[3];     // cell widths (>= global_cut + skin)
    float inv_w[3];
    float L[3];
    float cut2;     // (global_cut + skin)^2 in float, list predicate
    float rcmax2;   // max over type pairs of rc^2
    float hskin2;   // (skin/2)^2
    int skin_zero;  // skin == 0: rebuild every nl_f steps unconditionally
    int ntypes;
    int coeff_off;  // in units of float4, 3 float4 per (ti,tj)
    int mass_off;   // float2 (mass, 1/mass) per type
    int style;      // 0 dpd, 1 mdpd
    uint32_t seed;
    float dt;
    int nl_f;
    int log_f;
    int bond_style; // 0 none, 1 harmonic, 2 fene
    int bond_off;   // float4 per bond type
    uint32_t integ_mask; // bit (type-1) set when the type is integrated (fix nve group)
    double lo[3];
    double volume;
    int rdf_every;  // 0 = off
    int rdf_ta, rdf_tb, rdf_nbins;
    float rdf_rmax;
    int rdf_off;    // offset into the RDF histogram array (nbins per replica)
    int gc_n;       // group computes of this replica (table at gc[r * DPD_MAX_GC])
};

// Per-replica group fixes (src/fix/fix_spring.cu, fix_rvcm.cu, fix_recenter.cu).
// A mask holds bit (type-1) of each type of the fix's group; 0 = fix absent.
struct FixDesc {
    uint32_t spring_mask, rvcm_mask, recenter_mask;
    uint32_t rvcm_freq, recenter_freq;
    int rvcm_flag[3];
    double spring_k, spring_c[3], spring_r0, spring_m;  // spring_m: group mass
    double rvcm_m, recenter_m, recenter_c[3];
    double L[3];           // box lengths of the cell grid (unwrapped = lo + c w + o + img L)
    uint32_t spring_file_f; // spring record every this many steps (0 = none)
    // wall fixes (src/fix/fix_move.cu, fix_wall_reflect.cu, fix_two_wall.cu)
    int n_move, n_reflect, n_twowall;
    uint32_t move_mask[4];
    float move_v[4][3];
    uint32_t refl_mask[4];
    int refl_dir[4];
    float refl_lo[4], refl_hi[4];
    uint32_t tw_mask[2], tw_lo[2], tw_hi[2];
    int tw_dir[2];
};

// Group computes (temp, rho, msd, tf), DPD_MAX_GC per replica (device).
struct GCDesc {
    int kind;         // 1 temp, 2 rho, 3 msd, 4 tf
    uint32_t mask;    // the group's types (bit type-1)
    uint32_t freq;
    int ring;         // row ring of this compute (global index)
    double norm;      // temp 1/(3 Ng - 3); rho 1/volume; msd 1/Ng
    double region[6]; // rho: xlo xhi ylo yhi zlo zhi
    double L[3];      // box lengths of the cell grid
    uint32_t wall_mask; // wall_contact: the wall group's types
    int wall_side;      // +1: lo wall (its maximum), -1: hi wall (its minimum)
    int wall_dir;
    float cutoff;
    float box_lo, box_hi;  // the box along wall_dir
};

// Per-replica results of the fix reductions of the current step (device).
struct FixOut {
    float spring_a[3];     // spring force over group mass: member i gets m_i * spring_a
    float vcm[3];          // flag * centre-of-mass velocity of a due rvcm
    float shift[3];        // position shift of a due recenter
    int nrec;              // spring records written
};

// Per-replica dynamic state (device).
struct RepState {
    uint32_t step;      // the step whose force evaluation comes next
    uint32_t target;    // last step to evaluate in the current run
    int zero_pending;   // next evaluation is the zero step (no final half kick)
    int status;
    int nlog;           // thermo rows written
    int nbuild;
    int64_t rdf_samples;
};

// Coefficient table entry per ordered type pair (3 float4):
//  c0 = {A, gamma, sigma = sqrt(gamma)*sqrt(2kT)/sqrt(dt), rc^2}
//  c1 = {1/rc, 0.5*A*rc, B, 1/rd}
//  c2 = {rd^2, 0.25*B*rd, 15/(2 pi rd^3), rc}
