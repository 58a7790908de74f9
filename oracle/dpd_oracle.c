/*
 * dpd_oracle.c -- FP64 single-threaded CPU restatement of the GPUDPD timestep.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine in
 * gpumdpd_b200/: only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * reference legs of bench.py load it.  The product never links or calls it.
 *
 * Every function states the reference lines (xxin125/gpumdpd, paths relative to
 * the project root) whose arithmetic it restates.  State is double precision
 * throughout except two places that deliberately reproduce single precision:
 *   - oracle_saru(): the integer mixing is bit-exact uint32 and the float tail
 *     is evaluated in float exactly as src/force/pair_dpd.cu:233-235 does, so the
 *     random numbers are identical to the reference's and to the CUDA engine's;
 *   - oracle_pairs_f32(): the neighbour predicate evaluated in the engine's own
 *     FP32 cell-offset representation with a fixed operation order, which is the
 *     definition of the "bit-exact" neighbour set the engine is tested against.
 * Compile with -ffp-contract=off so that no FMA is formed implicitly.
 *
 * Parity is pinned by golden vectors produced by the reference's own CUDA build
 * (oracle/build_ref.sh + tests/golden/gen_ref_fixtures.py), see tests/test_oracle.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define ORACLE_MAXT 32
#define M_PI 3.14159265358979323846 /* src/force/pair_mdpd.cu:3 */

/* ------------------------------------------------------------------------- */
/* Saru counter-based RNG: src/force/pair_dpd.cu:203-236 (same constants; the
 * stream must be identical, so the steps are kept as published).              */

/* 0: float tail of the -DSINGLE build (the engine's); 1: tail of the -DDOUBLE build,
 * where (float)s * 2^-32f is float and the rest is double (pair_dpd.cu:235 with
 * numtyp = double).  Only the golden-vector tests against the DOUBLE build set 1. */
static int g_saru_double_tail = 0;
void oracle_set_saru_double_tail(int on) { g_saru_double_tail = on; }

static double saru_value(uint32_t seed1, uint32_t seed2, uint32_t seed, int32_t timestep);

float oracle_saru(uint32_t seed1, uint32_t seed2, uint32_t seed, int32_t timestep)
{
    int keep = g_saru_double_tail;
    g_saru_double_tail = 0;
    float r = (float)saru_value(seed1, seed2, seed, timestep);
    g_saru_double_tail = keep;
    return r;
}

static double saru_value(uint32_t seed1, uint32_t seed2, uint32_t seed, int32_t timestep)
{
    uint32_t seed3 = seed + (uint32_t)timestep;
    seed3 ^= (seed1 << 7) ^ (seed2 >> 6);
    seed2 += (seed1 >> 4) ^ (seed3 >> 15);
    seed1 ^= (seed2 << 9) + (seed3 << 8);
    seed3 ^= 0xA5366B4Du * ((seed2 >> 11) ^ (seed1 << 1));
    seed2 += 0x72BE1579u * ((seed1 << 4) ^ (seed3 >> 16));
    seed1 ^= 0x3F38A6EDu * ((seed3 >> 5) ^ (uint32_t)(((int32_t)seed2) >> 22));
    seed2 += seed1 * seed3;
    seed1 += seed3 ^ (seed2 >> 2);
    seed2 ^= (uint32_t)(((int32_t)seed2) >> 17);
    uint32_t state = 0x79dedea3u * (seed1 ^ (uint32_t)(((int32_t)seed1) >> 14));
    uint32_t wstate = (state + seed2) ^ (uint32_t)(((int32_t)state) >> 8);
    state = state + (wstate * (wstate ^ 0xdddf97f5u));
    wstate = 0xABCB96F7u + (wstate >> 1);
    uint32_t sum = 0;
    for (int r = 0; r < 8; r++) {
        sum += 0x9e3779b9u;
        state += ((wstate << 4) + 0xA341316Cu) ^ (wstate + sum) ^ ((wstate >> 5) + 0xC8013EA4u);
        wstate += ((state << 4) + 0xAD90777Du) ^ (state + sum) ^ ((state >> 5) + 0x7E95761Eu);
    }
    uint32_t v = (state ^ (state >> 26)) + wstate;
    uint32_t s = (v ^ (v >> 20)) * 0x6957f5a7u;
    /* float tail, one rounding per operation as in the reference's -DSINGLE build:
       (float)s * 2^-32 * 2 is exact scaling, then -1 rounds, then *sqrt(3)f rounds */
    volatile float a = (float)s;
    if (g_saru_double_tail) {
        volatile float a32 = a * 2.3283064365386963e-10f; /* 2^-32, exact */
        return 1.7320508075688772935274463 * ((double)a32 * 2.0 - 1.0);
    }
    volatile float u = a * 4.6566128730773926e-10f - 1.0f; /* 2^-31 */
    volatile float th = 1.7320508075688772f * u;
    return (double)th;
}

void oracle_saru_batch(int n, const uint32_t* t1, const uint32_t* t2, uint32_t seed,
                       const int32_t* step, float* out)
{
    for (int k = 0; k < n; k++) out[k] = oracle_saru(t1[k], t2[k], seed, step[k]);
}

/* ------------------------------------------------------------------------- */
/* minimum image: src/force/neigh_list.cu:377-379 (d -= L*((d>=L/2)-(d<-L/2)))  */

static inline double min_image(double d, double L)
{
    double h = 0.5 * L;
    return d - L * (double)((d >= h) - (d < -h));
}

/* triangular type-pair index: src/force/pair_dpd.cu:134 (0-based result) */
static inline int tri_index(int ti, int tj, int nt)
{
    int a = ti < tj ? ti : tj, b = ti < tj ? tj : ti;
    return ((a - 1) * nt - (a - 1) * (a - 2) / 2 + b - a + 1) - 1;
}

/* ------------------------------------------------------------------------- */
/* Half pair enumeration over a cell grid (cells >= cutoff, >= 3 per dim) or
 * all pairs when the box is too small.  The callback receives every unordered
 * pair {i,j} whose minimum-image distance squared is <= cut2.                 */

typedef void (*pair_cb)(int i, int j, double dx, double dy, double dz, double r2, void* ctx);

static void for_each_pair(int n, const double* x, const double* lo, const double* L,
                          double cut, pair_cb cb, void* ctx)
{
    double cut2 = cut * cut;
    int nc[3];
    for (int d = 0; d < 3; d++) nc[d] = (int)floor(L[d] / cut);
    if (nc[0] < 3 || nc[1] < 3 || nc[2] < 3) {
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++) {
                double dx = min_image(x[3 * i] - x[3 * j], L[0]);
                double dy = min_image(x[3 * i + 1] - x[3 * j + 1], L[1]);
                double dz = min_image(x[3 * i + 2] - x[3 * j + 2], L[2]);
                double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 <= cut2) cb(i, j, dx, dy, dz, r2, ctx);
            }
        return;
    }
    long ncell = (long)nc[0] * nc[1] * nc[2];
    int* head = (int*)malloc(sizeof(int) * ncell);
    int* next = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
    int* cidx = (int*)malloc(sizeof(int) * 3 * (n > 0 ? n : 1));
    for (long c = 0; c < ncell; c++) head[c] = -1;
    for (int i = n - 1; i >= 0; i--) {
        int c3[3];
        for (int d = 0; d < 3; d++) {
            int k = (int)floor((x[3 * i + d] - lo[d]) / (L[d] / nc[d]));
            if (k < 0) k = 0;
            if (k >= nc[d]) k = nc[d] - 1;
            c3[d] = k;
            cidx[3 * i + d] = k;
        }
        long c = ((long)c3[0] * nc[1] + c3[1]) * nc[2] + c3[2];
        next[i] = head[c];
        head[c] = i;
    }
    for (int i = 0; i < n; i++) {
        for (int ox = -1; ox <= 1; ox++)
            for (int oy = -1; oy <= 1; oy++)
                for (int oz = -1; oz <= 1; oz++) {
                    int cx = (cidx[3 * i] + ox + nc[0]) % nc[0];
                    int cy = (cidx[3 * i + 1] + oy + nc[1]) % nc[1];
                    int cz = (cidx[3 * i + 2] + oz + nc[2]) % nc[2];
                    long c = ((long)cx * nc[1] + cy) * nc[2] + cz;
                    for (int j = head[c]; j >= 0; j = next[j]) {
                        if (j <= i) continue;
                        double dx = min_image(x[3 * i] - x[3 * j], L[0]);
                        double dy = min_image(x[3 * i + 1] - x[3 * j + 1], L[1]);
                        double dz = min_image(x[3 * i + 2] - x[3 * j + 2], L[2]);
                        double r2 = dx * dx + dy * dy + dz * dz;
                        if (r2 <= cut2) cb(i, j, dx, dy, dz, r2, ctx);
                    }
                }
    }
    free(head);
    free(next);
    free(cidx);
}

/* ------------------------------------------------------------------------- */
/* Neighbour pairs (tag pairs, tag_lo < tag_hi) within `cut`, FP64 predicate.  */

typedef struct {
    const int* tag;
    int* out;
    long cap, cnt;
} pairs_ctx;

static void pairs_collect(int i, int j, double dx, double dy, double dz, double r2, void* c)
{
    (void)dx; (void)dy; (void)dz; (void)r2;
    pairs_ctx* p = (pairs_ctx*)c;
    if (p->cnt < p->cap) {
        int a = p->tag[i], b = p->tag[j];
        p->out[2 * p->cnt] = a < b ? a : b;
        p->out[2 * p->cnt + 1] = a < b ? b : a;
    }
    p->cnt++;
}

long oracle_pairs_f64(int n, const int* tag, const double* x, const double* lo, const double* L,
                      double cut, int* out, long cap)
{
    pairs_ctx p = {tag, out, cap, 0};
    for_each_pair(n, x, lo, L, cut, pairs_collect, &p);
    return p.cnt;
}

/* The engine's neighbour predicate in its own FP32 representation: particle i is
 * in cell (cx,cy,cz) of an nc-grid of widths w (float) at float offset o within
 * the cell.  Displacement d = dc*w + (o_i - o_j) with dc the cell difference
 * wrapped to the nearest image; r2 = fma(dz,dz,fma(dy,dy,dx*dx)); kept when
 * r2 <= cut2 (float).  Same predicate as the engine's list builder; it restates
 * the reference's r2 <= (global_cut+skin)^2 test (src/force/neigh_list.cu:373-382)
 * on the cell-offset representation.  Returns unordered tag pairs.            */
static int pair_f32(int i, int j, const int* cell, const float* off, const int* nc, const float* w,
                    float cut2)
{
    float d[3];
    for (int k = 0; k < 3; k++) {
        int dc = cell[3 * i + k] - cell[3 * j + k];
        if (dc > nc[k] / 2) dc -= nc[k];
        if (dc < -(nc[k] / 2)) dc += nc[k];
        if (dc > 1 || dc < -1) return 0;
        volatile float diff = off[3 * i + k] - off[3 * j + k];
        d[k] = fmaf((float)dc, w[k], diff);
    }
    volatile float r2 = d[0] * d[0];
    r2 = fmaf(d[1], d[1], r2);
    r2 = fmaf(d[2], d[2], r2);
    return r2 <= cut2;
}

static long emit_pair(const int* tag, int i, int j, int* out, long cap, long cnt)
{
    if (cnt < cap) {
        int a = tag[i], b = tag[j];
        out[2 * cnt] = a < b ? a : b;
        out[2 * cnt + 1] = a < b ? b : a;
    }
    return cnt + 1;
}

/* With at least 3 cells per dimension the candidates of i are the particles of the 27
 * cells around its own (each visited once), taken once per pair (j > i); any pair whose
 * wrapped cell difference exceeds 1 fails the predicate anyway, so the set is the one
 * of the all-pairs loop used for smaller grids. */
long oracle_pairs_f32(int n, const int* tag, const int* cell /*3n*/, const float* off /*3n*/,
                      const int* nc, const float* w, float cut2, int* out, long cap)
{
    long cnt = 0;
    if (nc[0] < 3 || nc[1] < 3 || nc[2] < 3) {
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++)
                if (pair_f32(i, j, cell, off, nc, w, cut2)) cnt = emit_pair(tag, i, j, out, cap, cnt);
        return cnt;
    }
    long ncell = (long)nc[0] * nc[1] * nc[2];
    int* head = (int*)malloc(sizeof(int) * ncell);
    int* next = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
    for (long c = 0; c < ncell; c++) head[c] = -1;
    for (int i = n - 1; i >= 0; i--) {
        long c = ((long)cell[3 * i] * nc[1] + cell[3 * i + 1]) * nc[2] + cell[3 * i + 2];
        next[i] = head[c];
        head[c] = i;
    }
    for (int i = 0; i < n; i++)
        for (int ox = -1; ox <= 1; ox++)
            for (int oy = -1; oy <= 1; oy++)
                for (int oz = -1; oz <= 1; oz++) {
                    int cx = (cell[3 * i] + ox + nc[0]) % nc[0];
                    int cy = (cell[3 * i + 1] + oy + nc[1]) % nc[1];
                    int cz = (cell[3 * i + 2] + oz + nc[2]) % nc[2];
                    long c = ((long)cx * nc[1] + cy) * nc[2] + cz;
                    for (int j = head[c]; j >= 0; j = next[j])
                        if (j > i && pair_f32(i, j, cell, off, nc, w, cut2))
                            cnt = emit_pair(tag, i, j, out, cap, cnt);
                }
    free(head);
    free(next);
    return cnt;
}

/* ------------------------------------------------------------------------- */
/* Force field description passed from Python.                               */

typedef struct {
    int style;           /* 0 = dpd (src/force/pair_dpd.cu), 1 = mdpd (src/force/pair_mdpd.cu) */
    int ntypes;
    double kT;           /* pair_style temp */
    double dt;
    uint32_t seed;
    double coeff[ORACLE_MAXT * ORACLE_MAXT][5]; /* [type pair (triangular)] A, B, gamma, rc, rd */
    double mass[ORACLE_MAXT];
    int bond_style;      /* 0 none, 1 harmonic (src/force/bond_harmonic.cu), 2 fene (new) */
    int nbondtypes;
    double bond_coeff[ORACLE_MAXT][4]; /* harmonic: k, r0 ; fene: K, R0, eps, sigma */
    int angle_style;     /* 0 none, 1 harmonic (src/force/angle_harmonic.cu) */
    int nangletypes;
    double angle_coeff[ORACLE_MAXT][2]; /* k, theta0 in degrees */
    /* group fixes; masks are the group's types (bit type-1) */
    int spring_on;       /* src/fix/fix_spring.cu:281-370 (post_force) */
    uint32_t spring_mask;
    double spring_k, spring_c[3], spring_r0;
    int rvcm_on;         /* src/fix/fix_rvcm.cu:233-286 (end_of_step) */
    uint32_t rvcm_mask;
    uint32_t rvcm_freq;
    int rvcm_flag[3];
    int recenter_on;     /* src/fix/fix_recenter.cu:270-335 (end_of_step) */
    uint32_t recenter_mask;
    uint32_t recenter_freq;
    double recenter_c[3];
    uint32_t integ_mask; /* types integrated by fix nve; 0 = every type */
    int n_move;          /* src/fix/fix_move.cu:33-100 (initial_integrate) */
    uint32_t move_mask[4];
    double move_v[4][3];
    int n_reflect;       /* src/fix/fix_wall_reflect.cu:84-140 (post_integrate) */
    uint32_t refl_mask[4];
    int refl_dir[4];
    double refl_lo[4], refl_hi[4];
    int n_twowall;       /* src/fix/fix_two_wall.cu:84-200 (post_integrate) */
    uint32_t tw_mask[2], tw_lo[2], tw_hi[2];
    int tw_dir[2];
} oracle_ff;

/* The angle list (type, tag_i, tag_j, tag_k per angle; j is the apex) of the next
 * oracle_forces/oracle_run calls; set by the caller, NULL for none.                */
static const int* g_angles = 0;
static int g_nangles = 0;
void oracle_set_angles(int nangles, const int* angles)
{
    g_nangles = angles ? nangles : 0;
    g_angles = angles;
}

typedef struct {
    const oracle_ff* ff;
    const int* tag;
    const int* type;
    const double* v;
    const double* rho;
    uint32_t step;
    double* f;
    double* rho_out;
    double pe;
    double vir[6];
    double sig_scale; /* sqrt(2 kT) / sqrt(dt), src/force/pair_dpd.cu:577-578 */
} force_ctx;

/* mDPD local density: src/force/pair_mdpd.cu:253-297.  rho_i = sum over j != i of
 * 15/(2 pi rd^3) (1 - r/rd)^2 for r < rd, no self term.                        */
static void density_cb(int i, int j, double dx, double dy, double dz, double r2, void* c)
{
    (void)dx; (void)dy; (void)dz;
    force_ctx* k = (force_ctx*)c;
    int idx = tri_index(k->type[i], k->type[j], k->ff->ntypes);
    double rd = k->ff->coeff[idx][4];
    double r = sqrt(r2);
    double wd = 1.0 - r / rd;
    if (wd < 0.0) wd = 0.0;
    double factor = 15.0 / 2.0 / M_PI / (rd * rd * rd);
    double add = factor * wd * wd;
    k->rho_out[i] += add;
    k->rho_out[j] += add;
}

/* DPD pair force: src/force/pair_dpd.cu:292-403 (log variant: PE 0.5*A*rc*wc^2
 * per pair, virial r (x) F per pair).  mDPD: src/force/pair_mdpd.cu:399-521.   */
static void force_cb(int i, int j, double dx, double dy, double dz, double r2, void* c)
{
    force_ctx* k = (force_ctx*)c;
    const oracle_ff* ff = k->ff;
    int idx = tri_index(k->type[i], k->type[j], ff->ntypes);
    double A = ff->coeff[idx][0], B = ff->coeff[idx][1], gamma = ff->coeff[idx][2];
    double rc = ff->coeff[idx][3], rd = ff->coeff[idx][4];
    if (!(r2 <= rc * rc)) return;
    double r = sqrt(r2);
    if (r < 1.0e-10) return;
    double rinv = 1.0 / r;
    double dvx = k->v[3 * i] - k->v[3 * j];
    double dvy = k->v[3 * i + 1] - k->v[3 * j + 1];
    double dvz = k->v[3 * i + 2] - k->v[3 * j + 2];
    double dot = dx * dvx + dy * dvy + dz * dvz;
    double wc = 1.0 - r / rc;
    double wr = wc;
    int a = k->tag[i], b = k->tag[j];
    uint32_t t1 = (uint32_t)(a < b ? a : b), t2 = (uint32_t)(a < b ? b : a);
    double theta = saru_value(t1, t2, ff->seed, (int32_t)k->step);
    double sigma = sqrt(gamma) * k->sig_scale;
    double fpair;
    double pe;
    if (ff->style == 0) {
        fpair = A * wc - gamma * wr * wr * dot * rinv + sigma * wr * theta;
        pe = 0.5 * A * rc * wc * wc;
    } else {
        double wd = 1.0 - r / rd;
        if (wd < 0.0) wd = 0.0;
        double rhoi = k->rho[i], rhoj = k->rho[j];
        fpair = A * wc + B * (rhoi + rhoj) * wd - gamma * wr * wr * dot * rinv + sigma * wr * theta;
        pe = 0.5 * A * rc * wc * wc + 0.25 * B * rd * (rhoi + rhoj) * wd * wd;
    }
    fpair *= rinv;
    double fx = dx * fpair, fy = dy * fpair, fz = dz * fpair;
    k->f[3 * i] += fx;
    k->f[3 * i + 1] += fy;
    k->f[3 * i + 2] += fz;
    k->f[3 * j] -= fx;
    k->f[3 * j + 1] -= fy;
    k->f[3 * j + 2] -= fz;
    k->pe += pe;
    k->vir[0] += dx * fx;
    k->vir[1] += dx * fy;
    k->vir[2] += dx * fz;
    k->vir[3] += dy * fy;
    k->vir[4] += dy * fz;
    k->vir[5] += dz * fz;
}

static double max_rc(const oracle_ff* ff)
{
    double m = 0.0;
    int np = ff->ntypes * (ff->ntypes + 1) / 2;
    for (int p = 0; p < np; p++)
        if (ff->coeff[p][3] > m) m = ff->coeff[p][3];
    return m;
}

/* Bonds.  Harmonic: src/force/bond_harmonic.cu:208-268: E = k (r-r0)^2,
 * F_i = -2 k (r-r0)/r * d, d = x_i - x_j, virial d (x) F_i.
 * FENE (not in the reference): E = -0.5 K R0^2 ln(1-(r/R0)^2) plus the WCA
 * repulsion 4 eps[(s/r)^12-(s/r)^6]+eps for r < 2^(1/6) s.                    */
static int bond_forces(int n, const int* tag_to_idx, int ntag, const double* x, const double* lo,
                       const double* L, const oracle_ff* ff, int nbonds, const int* bonds,
                       double* f, double* pe_out, double* vir)
{
    (void)n; (void)lo;
    int status = 0;
    for (int b = 0; b < nbonds; b++) {
        int bt = bonds[3 * b], ta = bonds[3 * b + 1], tb = bonds[3 * b + 2];
        if (ta < 1 || ta > ntag || tb < 1 || tb > ntag) { status = -1; continue; }
        int i = tag_to_idx[ta - 1], j = tag_to_idx[tb - 1];
        double dx = min_image(x[3 * i] - x[3 * j], L[0]);
        double dy = min_image(x[3 * i + 1] - x[3 * j + 1], L[1]);
        double dz = min_image(x[3 * i + 2] - x[3 * j + 2], L[2]);
        double r2 = dx * dx + dy * dy + dz * dz;
        double r = sqrt(r2);
        double fbond = 0.0, e = 0.0;
        const double* bc = ff->bond_coeff[bt - 1];
        if (ff->bond_style == 1) {
            fbond = r > 0.0 ? -2.0 * bc[0] * (r - bc[1]) / r : 0.0;
            e = bc[0] * (r - bc[1]) * (r - bc[1]);
        } else if (ff->bond_style == 2) {
            double K = bc[0], R0 = bc[1], eps = bc[2], sg = bc[3];
            double rr = r2 / (R0 * R0);
            if (rr >= 1.0) { status = -2; rr = 0.999; }
            fbond = -K / (1.0 - rr);
            e = -0.5 * K * R0 * R0 * log(1.0 - rr);
            if (eps > 0.0 && r2 < pow(2.0, 1.0 / 3.0) * sg * sg) {
                double sr2 = sg * sg / r2, sr6 = sr2 * sr2 * sr2;
                fbond += 48.0 * eps * sr6 * (sr6 - 0.5) / r2;
                e += 4.0 * eps * sr6 * (sr6 - 1.0) + eps;
            }
        }
        double fx = dx * fbond, fy = dy * fbond, fz = dz * fbond;
        f[3 * i] += fx; f[3 * i + 1] += fy; f[3 * i + 2] += fz;
        f[3 * j] -= fx; f[3 * j + 1] -= fy; f[3 * j + 2] -= fz;
        *pe_out += e;
        vir[0] += dx * fx; vir[1] += dx * fy; vir[2] += dx * fz;
        vir[3] += dy * fy; vir[4] += dy * fz; vir[5] += dz * fz;
    }
    return status;
}

/* Harmonic angles: src/force/angle_harmonic.cu:187-270.  d1 = x_i - x_j, d2 = x_k - x_j
 * (minimum image), c = cos(theta) clamped to [-1, 1], s = sin(theta) >= 0.001,
 * E = k (theta - theta0)^2, a = -2 k (theta - theta0) / s, a11 = a c / |d1|^2,
 * a12 = -a / (|d1| |d2|), a22 = a c / |d2|^2, F_i = a11 d1 + a12 d2,
 * F_k = a22 d2 + a12 d1, F_j = -(F_i + F_k); virial d1 (x) F_i + d2 (x) F_k (the
 * reference gives a third of it to each atom).                                  */
static int angle_forces(const int* tag_to_idx, int ntag, const double* x, const double* L,
                        const oracle_ff* ff, int nangles, const int* angles, double* f, double* pe_out,
                        double* vir)
{
    int status = 0;
    for (int a = 0; a < nangles; a++) {
        const int at = angles[4 * a], ti = angles[4 * a + 1], tj = angles[4 * a + 2], tk = angles[4 * a + 3];
        if (ti < 1 || ti > ntag || tj < 1 || tj > ntag || tk < 1 || tk > ntag || at < 1 || at > ff->nangletypes) {
            status = -1;
            continue;
        }
        const int i = tag_to_idx[ti - 1], j = tag_to_idx[tj - 1], k = tag_to_idx[tk - 1];
        double d1[3], d2[3];
        for (int c = 0; c < 3; c++) {
            d1[c] = min_image(x[3 * i + c] - x[3 * j + c], L[c]);
            d2[c] = min_image(x[3 * k + c] - x[3 * j + c], L[c]);
        }
        const double rsq1 = d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2];
        const double rsq2 = d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2];
        const double r1 = sqrt(rsq1), r2 = sqrt(rsq2);
        double c = (d1[0] * d2[0] + d1[1] * d2[1] + d1[2] * d2[2]) / (r1 * r2);
        if (c > 1.0) c = 1.0;
        if (c < -1.0) c = -1.0;
        double s = sqrt(1.0 - c * c);
        if (s < 0.001) s = 0.001;
        const double kk = ff->angle_coeff[at - 1][0];
        const double theta0 = ff->angle_coeff[at - 1][1] * (M_PI / 180.0);
        const double dtheta = acos(c) - theta0;
        const double aa = -2.0 * kk * dtheta / s;
        const double a11 = aa * c / rsq1, a12 = -aa / (r1 * r2), a22 = aa * c / rsq2;
        double fi[3], fk[3];
        for (int q = 0; q < 3; q++) {
            fi[q] = a11 * d1[q] + a12 * d2[q];
            fk[q] = a22 * d2[q] + a12 * d1[q];
            f[3 * i + q] += fi[q];
            f[3 * k + q] += fk[q];
            f[3 * j + q] -= fi[q] + fk[q];
        }
        *pe_out += kk * dtheta * dtheta;
        vir[0] += d1[0] * fi[0] + d2[0] * fk[0];
        vir[1] += d1[0] * fi[1] + d2[0] * fk[1];
        vir[2] += d1[0] * fi[2] + d2[0] * fk[2];
        vir[3] += d1[1] * fi[1] + d2[1] * fk[1];
        vir[4] += d1[1] * fi[2] + d2[1] * fk[2];
        vir[5] += d1[2] * fi[2] + d2[2] * fk[2];
    }
    return status;
}

/* Forces at one state.  out: f[3n], rho[n] (mdpd, may be NULL), energy[3] = pair,
 * bond, angle; virial[6] = xx xy xz yy yz zz (pair + bond + angle).             */
int oracle_forces(int n, const int* tag, const int* type, const double* x, const double* v,
                  const double* lo, const double* L, const oracle_ff* ff, uint32_t step,
                  int nbonds, const int* bonds, double* f, double* rho, double* energy,
                  double* virial)
{
    memset(f, 0, sizeof(double) * 3 * n);
    double* rho_buf = rho ? rho : (double*)calloc(n > 0 ? n : 1, sizeof(double));
    force_ctx k;
    memset(&k, 0, sizeof(k));
    k.ff = ff; k.tag = tag; k.type = type; k.v = v; k.step = step; k.f = f;
    k.sig_scale = sqrt(2.0 * ff->kT) / sqrt(ff->dt);
    double cut = max_rc(ff);
    if (ff->style == 1) {
        memset(rho_buf, 0, sizeof(double) * n);
        k.rho_out = rho_buf;
        for_each_pair(n, x, lo, L, cut, density_cb, &k);
    }
    k.rho = rho_buf;
    for_each_pair(n, x, lo, L, cut, force_cb, &k);
    double bpe = 0.0, ape = 0.0, bvir[6] = {0, 0, 0, 0, 0, 0};
    int status = 0;
    const int want_angles = ff->angle_style != 0 && g_nangles > 0;
    if ((ff->bond_style != 0 && nbonds > 0) || want_angles) {
        int ntag = 0;
        for (int i = 0; i < n; i++) if (tag[i] > ntag) ntag = tag[i];
        int* t2i = (int*)malloc(sizeof(int) * (ntag > 0 ? ntag : 1));
        for (int t = 0; t < ntag; t++) t2i[t] = -1;
        for (int i = 0; i < n; i++) t2i[tag[i] - 1] = i;
        if (ff->bond_style != 0 && nbonds > 0)
            status = bond_forces(n, t2i, ntag, x, lo, L, ff, nbonds, bonds, f, &bpe, bvir);
        if (want_angles) status |= angle_forces(t2i, ntag, x, L, ff, g_nangles, g_angles, f, &ape, bvir);
        free(t2i);
    }
    if (energy) { energy[0] = k.pe; energy[1] = bpe; energy[2] = ape; }
    if (virial) for (int c = 0; c < 6; c++) virial[c] = k.vir[c] + bvir[c];
    if (!rho) free(rho_buf);
    return status;
}

/* ------------------------------------------------------------------------- */
/* Thermo: src/compute/thermo.cu:240-246 (KE), 301-303 (T = 2KE/(3N-3)),
 * 422-434 + 506-517 (P_ab = (sum m v_a v_b + W_ab)/V, P = trace/3).
 * out[12]: T, pair_pe, bond_pe, P, Pxx, Pxy, Pxz, Pyy, Pyz, Pzz, KE, angle_pe  */
static void thermo(int n, const int* type, const double* v, const double* L, const oracle_ff* ff,
                   const double* energy, const double* virial, double* out)
{
    double ke = 0.0, kin[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < n; i++) {
        double m = ff->mass[type[i] - 1];
        const double* vi = v + 3 * i;
        ke += 0.5 * m * (vi[0] * vi[0] + vi[1] * vi[1] + vi[2] * vi[2]);
        kin[0] += m * vi[0] * vi[0]; kin[1] += m * vi[0] * vi[1]; kin[2] += m * vi[0] * vi[2];
        kin[3] += m * vi[1] * vi[1]; kin[4] += m * vi[1] * vi[2]; kin[5] += m * vi[2] * vi[2];
    }
    double vol = L[0] * L[1] * L[2];
    out[0] = 2.0 * ke / (3.0 * n - 3.0);
    out[1] = energy[0];
    out[2] = energy[1];
    for (int c = 0; c < 6; c++) out[4 + c] = (kin[c] + virial[c]) / vol;
    out[3] = (out[4] + out[7] + out[9]) / 3.0;
    out[10] = ke;
    out[11] = energy[2];
}

/* ------------------------------------------------------------------------- */
/* Group fixes.  Unwrapped positions are x + img L (the reference's uwpos).          */
static double group_mass(int n, const int* type, const oracle_ff* ff, uint32_t mask)
{
    double m = 0.0;
    for (int i = 0; i < n; i++)
        if ((mask >> (type[i] - 1)) & 1u) m += ff->mass[type[i] - 1];
    return m;
}

/* The record of the last spring evaluation: Fx, Fy, Fz, +-|F|, energy (the row the
 * reference writes to the spring's file, src/fix/fix_spring.cu:340-360).              */
static double spring_last[5];

void oracle_spring_last(double* out)
{
    for (int k = 0; k < 5; k++) out[k] = spring_last[k];
}

/* fix spring, post_force: F = -k (r - r0) d / r with d = com - c (r = |d| > 1e-10) on the
 * group's centre of mass, a share m_i / M to each member; not part of the virial.     */
static void fix_spring(int n, const int* type, const double* x, const int* img, const double* L,
                       const oracle_ff* ff, double* f)
{
    const uint32_t mask = ff->spring_mask;
    const double M = group_mass(n, type, ff, mask);
    if (!(M > 0)) return;
    double com[3] = {0, 0, 0};
    for (int i = 0; i < n; i++) {
        if (!((mask >> (type[i] - 1)) & 1u)) continue;
        const double m = ff->mass[type[i] - 1];
        for (int d = 0; d < 3; d++) com[d] += m * (x[3 * i + d] + img[3 * i + d] * L[d]);
    }
    double dv[3], r2 = 0.0;
    for (int d = 0; d < 3; d++) {
        dv[d] = com[d] / M - ff->spring_c[d];
        r2 += dv[d] * dv[d];
    }
    const double r = sqrt(r2);
    for (int k = 0; k < 5; k++) spring_last[k] = 0.0;
    if (!(r > 1.0e-10)) return;
    const double dr = r - ff->spring_r0;
    for (int d = 0; d < 3; d++) spring_last[d] = -ff->spring_k * dr * dv[d] / r;
    spring_last[3] = sqrt(spring_last[0] * spring_last[0] + spring_last[1] * spring_last[1] +
                          spring_last[2] * spring_last[2]) * (dr < 0.0 ? -1.0 : 1.0);
    spring_last[4] = 0.5 * ff->spring_k * dr * dr;
    for (int i = 0; i < n; i++) {
        if (!((mask >> (type[i] - 1)) & 1u)) continue;
        const double share = ff->mass[type[i] - 1] / M;
        for (int d = 0; d < 3; d++) f[3 * i + d] += -ff->spring_k * dr * dv[d] / r * share;
    }
}

/* fix rvcm and fix recenter, end_of_step of a step that is a multiple of their frequency. */
static void fix_end_of_step(int n, const int* type, double* x, double* v, int* img, const double* lo,
                            const double* L, const oracle_ff* ff, uint32_t step)
{
    if (ff->rvcm_on && ff->rvcm_freq && step % ff->rvcm_freq == 0) {
        const uint32_t mask = ff->rvcm_mask;
        const double M = group_mass(n, type, ff, mask);
        double p[3] = {0, 0, 0};
        for (int i = 0; i < n; i++) {
            if (!((mask >> (type[i] - 1)) & 1u)) continue;
            for (int d = 0; d < 3; d++) p[d] += ff->mass[type[i] - 1] * v[3 * i + d];
        }
        if (M > 0)
            for (int i = 0; i < n; i++) {
                if (!((mask >> (type[i] - 1)) & 1u)) continue;
                for (int d = 0; d < 3; d++) v[3 * i + d] -= ff->rvcm_flag[d] * p[d] / M;
            }
    }
    if (ff->recenter_on && ff->recenter_freq && step % ff->recenter_freq == 0) {
        const uint32_t mask = ff->recenter_mask;
        const double M = group_mass(n, type, ff, mask);
        double com[3] = {0, 0, 0};
        for (int i = 0; i < n; i++) {
            if (!((mask >> (type[i] - 1)) & 1u)) continue;
            const double m = ff->mass[type[i] - 1];
            for (int d = 0; d < 3; d++) com[d] += m * (x[3 * i + d] + img[3 * i + d] * L[d]);
        }
        if (M > 0)
            for (int i = 0; i < n; i++) {
                if (!((mask >> (type[i] - 1)) & 1u)) continue;
                for (int d = 0; d < 3; d++) {
                    double q = x[3 * i + d] + (ff->recenter_c[d] - com[d] / M);
                    const double hi = lo[d] + L[d];
                    while (q >= hi || q < lo[d]) {
                        const int k = (q >= hi) - (q < lo[d]);
                        q -= L[d] * k;
                        img[3 * i + d] += k;
                    }
                    x[3 * i + d] = q;
                }
            }
    }
}

/* fix move (initial_integrate after fix nve's drift): v = V, x += V dt; then the
 * post_integrate walls: fix wall_reflect mirrors group atoms outside [lo, hi] along its
 * axis and reverses that velocity component; fix two_wall does the same between the
 * maximum position of its lo-wall group and the minimum of its hi-wall group.         */
static void wrap_coord(double* x, int* img, const double* lo, const double* L, int i, int d)
{
    double p = x[3 * i + d];
    const double hi = lo[d] + L[d];
    while (p >= hi || p < lo[d]) {
        const int k = (p >= hi) - (p < lo[d]);
        p -= L[d] * k;
        img[3 * i + d] += k;
    }
    x[3 * i + d] = p;
}

static void wall_fixes(int n, const int* type, double* x, double* v, int* img, const double* lo,
                       const double* L, const oracle_ff* ff)
{
    for (int k = 0; k < ff->n_move; k++)
        for (int i = 0; i < n; i++) {
            if (!((ff->move_mask[k] >> (type[i] - 1)) & 1u)) continue;
            for (int d = 0; d < 3; d++) {
                v[3 * i + d] = ff->move_v[k][d];
                x[3 * i + d] += ff->move_v[k][d] * ff->dt;
                wrap_coord(x, img, lo, L, i, d);
            }
        }
    for (int k = 0; k < ff->n_reflect; k++) {
        const int d = ff->refl_dir[k];
        for (int i = 0; i < n; i++) {
            if (!((ff->refl_mask[k] >> (type[i] - 1)) & 1u)) continue;
            const double p = x[3 * i + d];
            if (p < ff->refl_lo[k] || p > ff->refl_hi[k]) {
                x[3 * i + d] = p + 2.0 * ((p < ff->refl_lo[k] ? ff->refl_lo[k] : ff->refl_hi[k]) - p);
                v[3 * i + d] = -v[3 * i + d];
            }
        }
    }
    for (int k = 0; k < ff->n_twowall; k++) {
        const int d = ff->tw_dir[k];
        double wlo = -INFINITY, whi = INFINITY;
        for (int i = 0; i < n; i++) {
            const uint32_t bit = 1u << (type[i] - 1);
            if (ff->tw_lo[k] & bit) wlo = fmax(wlo, x[3 * i + d]);
            if (ff->tw_hi[k] & bit) whi = fmin(whi, x[3 * i + d]);
        }
        for (int i = 0; i < n; i++) {
            if (!((ff->tw_mask[k] >> (type[i] - 1)) & 1u)) continue;
            const double p = x[3 * i + d];
            if (p < wlo || p > whi) {
                x[3 * i + d] = p + 2.0 * ((p < wlo ? wlo : whi) - p);
                v[3 * i + d] = -v[3 * i + d];
            }
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Velocity-Verlet run with the reference's step order (src/main/utils.cuh:166-213
 * for step 0, :254-303 per step; src/fix/fix_nve.cu:42-86 and :131-149).
 * State in/out: x (wrapped into [lo, lo+L)), v, img (image counters, 3n ints).
 * Steps first_step .. first_step+nsteps-1 are run after an optional zero step
 * (do_zero_step != 0 computes forces and thermo at step first_step-1 first).
 * thermo_out receives 12 doubles per logged step (step % log_f == 0), the step
 * numbers go to log_steps; returns the number of logged rows (or <0 on error).
 * f_out holds the last computed forces.                                       */
int oracle_run(int n, const int* tag, const int* type, double* x, double* v, int* img,
               const double* lo, const double* L, const oracle_ff* ff, int nbonds,
               const int* bonds, uint32_t first_step, int nsteps, int do_zero_step,
               uint32_t log_f, double* thermo_out, int* log_steps, int max_log, double* f_out,
               double* rho_out)
{
    double* f = f_out;
    double energy[3], virial[6];
    int nlog = 0;
    int status = 0;
    double dt = ff->dt;
    if (do_zero_step) {
        uint32_t s0 = first_step - 1;
        status |= oracle_forces(n, tag, type, x, v, lo, L, ff, s0, nbonds, bonds, f, rho_out,
                                energy, virial);
        if (ff->spring_on) fix_spring(n, type, x, img, L, ff, f);
        if (log_f && s0 % log_f == 0 && nlog < max_log) {
            thermo(n, type, v, L, ff, energy, virial, thermo_out + 12 * nlog);
            log_steps[nlog++] = (int)s0;
        }
    }
    for (int s = 0; s < nsteps; s++) {
        uint32_t step = first_step + (uint32_t)s;
        for (int i = 0; i < n; i++) {
            double dtm = 0.5 * dt / ff->mass[type[i] - 1];
            const uint32_t bit = 1u << (type[i] - 1);
            if (ff->integ_mask && !(ff->integ_mask & bit)) continue;
            for (int d = 0; d < 3; d++) {
                v[3 * i + d] += dtm * f[3 * i + d];
                double p = x[3 * i + d] + dt * v[3 * i + d];
                double hi = lo[d] + L[d];
                while (p >= hi || p < lo[d]) {
                    int k = (p >= hi) - (p < lo[d]);
                    p -= L[d] * k;
                    img[3 * i + d] += k;
                }
                x[3 * i + d] = p;
            }
        }
        wall_fixes(n, type, x, v, img, lo, L, ff);
        status |= oracle_forces(n, tag, type, x, v, lo, L, ff, step, nbonds, bonds, f, rho_out,
                                energy, virial);
        if (ff->spring_on) fix_spring(n, type, x, img, L, ff, f);
        for (int i = 0; i < n; i++) {
            double dtm = 0.5 * dt / ff->mass[type[i] - 1];
            if (ff->integ_mask && !(ff->integ_mask & (1u << (type[i] - 1)))) continue;
            for (int d = 0; d < 3; d++) v[3 * i + d] += dtm * f[3 * i + d];
        }
        fix_end_of_step(n, type, x, v, img, lo, L, ff, step);
        if (log_f && step % log_f == 0 && nlog < max_log) {
            thermo(n, type, v, L, ff, energy, virial, thermo_out + 12 * nlog);
            log_steps[nlog++] = (int)step;
        }
    }
    return status < 0 ? status : nlog;
}

/* ------------------------------------------------------------------------- */
/* Radial distribution function between type sets (new: the reference has none).
 * g(r) for pairs (a in type ta, b in type tb), bins of width dr up to rmax:
 * g_k = count_k / (N_a N_b' 4/3 pi (r_{k+1}^3 - r_k^3) / V), where N_b' = N_b
 * (or N_a - 1 when ta == tb and pairs are counted both ways).                 */
typedef struct {
    const int* type;
    int ta, tb;
    double dr;
    int nbins;
    double* hist;
} rdf_ctx;

static void rdf_cb(int i, int j, double dx, double dy, double dz, double r2, void* c)
{
    (void)dx; (void)dy; (void)dz;
    rdf_ctx* k = (rdf_ctx*)c;
    int a = k->type[i], b = k->type[j];
    int match = (a == k->ta && b == k->tb) || (a == k->tb && b == k->ta);
    if (!match) return;
    int bin = (int)(sqrt(r2) / k->dr);
    if (bin < k->nbins) {
        double w = (k->ta == k->tb) ? 2.0 : 1.0;
        k->hist[bin] += w;
    }
}

int oracle_rdf(int n, const int* type, const double* x, const double* lo, const double* L,
               int ta, int tb, double rmax, int nbins, double* g_out)
{
    rdf_ctx k = {type, ta, tb, rmax / nbins, nbins, g_out};
    memset(g_out, 0, sizeof(double) * nbins);
    for_each_pair(n, x, lo, L, rmax, rdf_cb, &k);
    long na = 0, nb = 0;
    for (int i = 0; i < n; i++) {
        if (type[i] == ta) na++;
        if (type[i] == tb) nb++;
    }
    double vol = L[0] * L[1] * L[2];
    double npair = (ta == tb) ? (double)na * (double)(na - 1) : (double)na * (double)nb;
    for (int b = 0; b < nbins; b++) {
        double r0 = b * k.dr, r1 = (b + 1) * k.dr;
        double shell = 4.0 / 3.0 * M_PI * (r1 * r1 * r1 - r0 * r0 * r0);
        double ideal = npair * shell / vol;
        g_out[b] = ideal > 0 ? g_out[b] / ideal : 0.0;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* CPU baseline timing path: the reference's algorithm (half Verlet list with
 * skin, rebuilt on the reference's displacement criterion, src/force/neigh_list.cu
 * :322-393 and :483-514) over a DPD system, in FP64, split over nthreads POSIX
 * threads with thread-private force buffers, plus the bond forces
 * (src/force/bond_harmonic.cu:275-351) on one thread.  Advances nsteps after a
 * step-0 force evaluation and returns the number of list builds (-3 when a bond
 * names a tag outside 1..n).                                                    */
typedef struct {
    int i0, i1, n, nmax;
    const int *tag, *type, *nl, *nn;
    const double *x, *v, *L;
    const oracle_ff* ff;
    double* fl;
    uint32_t step;
    double sig_scale;
} bench_task;

static void* bench_force_range(void* arg)
{
    bench_task* t = (bench_task*)arg;
    const oracle_ff* ff = t->ff;
    const double *x = t->x, *v = t->v, *L = t->L;
    double* fl = t->fl;
    memset(fl, 0, sizeof(double) * 3 * (size_t)t->n);
    for (int i = t->i0; i < t->i1; i++) {
        for (int k = 0; k < t->nn[i]; k++) {
            int j = t->nl[(size_t)i * t->nmax + k];
            double dx = min_image(x[3 * i] - x[3 * j], L[0]);
            double dy = min_image(x[3 * i + 1] - x[3 * j + 1], L[1]);
            double dz = min_image(x[3 * i + 2] - x[3 * j + 2], L[2]);
            double r2 = dx * dx + dy * dy + dz * dz;
            int idx = tri_index(t->type[i], t->type[j], ff->ntypes);
            double A = ff->coeff[idx][0], gamma = ff->coeff[idx][2], rc = ff->coeff[idx][3];
            if (!(r2 <= rc * rc)) continue;
            double r = sqrt(r2);
            if (r < 1e-10) continue;
            double dvx = v[3 * i] - v[3 * j], dvy = v[3 * i + 1] - v[3 * j + 1],
                   dvz = v[3 * i + 2] - v[3 * j + 2];
            double dot = dx * dvx + dy * dvy + dz * dvz;
            double wc = 1.0 - r / rc;
            int a = t->tag[i], b = t->tag[j];
            double th = oracle_saru((uint32_t)(a < b ? a : b), (uint32_t)(a < b ? b : a),
                                    ff->seed, (int32_t)t->step);
            double fp = (A * wc - gamma * wc * wc * dot / r + sqrt(gamma) * t->sig_scale * wc * th) / r;
            fl[3 * i] += dx * fp; fl[3 * i + 1] += dy * fp; fl[3 * i + 2] += dz * fp;
            fl[3 * j] -= dx * fp; fl[3 * j + 1] -= dy * fp; fl[3 * j + 2] -= dz * fp;
        }
    }
    return NULL;
}

typedef struct {
    int i0, i1, n, nmax;
    const int *head, *next, *cid, *nc;
    const double *x, *L;
    double cut2;
    int* nl;
    int* nn;
    double* f;
    const double* fpriv;
    int nt;
} build_task;

static void* bench_build_range(void* arg)
{
    build_task* t = (build_task*)arg;
    const double *x = t->x, *L = t->L;
    const int* nc = t->nc;
    for (int i = t->i0; i < t->i1; i++) {
        int cnt = 0;
        for (int ox = -1; ox <= 1; ox++)
            for (int oy = -1; oy <= 1; oy++)
                for (int oz = -1; oz <= 1; oz++) {
                    int cx = (t->cid[3 * i] + ox + nc[0]) % nc[0];
                    int cy = (t->cid[3 * i + 1] + oy + nc[1]) % nc[1];
                    int cz = (t->cid[3 * i + 2] + oz + nc[2]) % nc[2];
                    long c = ((long)cx * nc[1] + cy) * nc[2] + cz;
                    for (int j = t->head[c]; j >= 0; j = t->next[j]) {
                        if (j <= i) continue;
                        double dx = min_image(x[3 * i] - x[3 * j], L[0]);
                        double dy = min_image(x[3 * i + 1] - x[3 * j + 1], L[1]);
                        double dz = min_image(x[3 * i + 2] - x[3 * j + 2], L[2]);
                        if (dx * dx + dy * dy + dz * dz <= t->cut2 && cnt < t->nmax)
                            t->nl[(size_t)i * t->nmax + cnt++] = j;
                    }
                }
        t->nn[i] = cnt;
    }
    return NULL;
}

static void* bench_reduce_range(void* arg)
{
    build_task* t = (build_task*)arg;
    for (long k = 3L * t->i0; k < 3L * t->i1; k++) {
        double acc = 0.0;
        for (int q = 0; q < t->nt; q++) acc += t->fpriv[(size_t)3 * t->n * q + k];
        t->f[k] = acc;
    }
    return NULL;
}

int oracle_bench_steps(int n, const int* tag, const int* type, double* x, double* v,
                       const double* lo, const double* L, const oracle_ff* ff, int nbonds,
                       const int* bonds, uint32_t first_step, int nsteps, double skin,
                       int nthreads)
{
    double cut = max_rc(ff) + skin;
    double cut2 = cut * cut;
    int nc[3];
    for (int d = 0; d < 3; d++) nc[d] = (int)floor(L[d] / cut);
    if (nc[0] < 3 || nc[1] < 3 || nc[2] < 3) return -1;
    int nt = nthreads > 0 ? nthreads : 1;
    if (nt > 256) nt = 256;
    long ncell = (long)nc[0] * nc[1] * nc[2];
    int nmax = 256;
    int* nl = (int*)malloc(sizeof(int) * (size_t)n * nmax);
    int* nn = (int*)malloc(sizeof(int) * n);
    double* xlast = (double*)malloc(sizeof(double) * 3 * n);
    double* f = (double*)calloc((size_t)3 * n, sizeof(double));
    int* head = (int*)malloc(sizeof(int) * ncell);
    int* next = (int*)malloc(sizeof(int) * n);
    int* cid = (int*)malloc(sizeof(int) * 3 * n);
    double* fpriv = (double*)malloc(sizeof(double) * 3 * (size_t)n * nt);
    pthread_t th[256];
    bench_task task[256];
    double sig_scale = sqrt(2.0 * ff->kT) / sqrt(ff->dt);
    int* tag_to_idx = NULL;
    if (nbonds > 0 && bonds) {
        tag_to_idx = (int*)malloc(sizeof(int) * n);
        for (int i = 0; i < n; i++) tag_to_idx[i] = 0;
        for (int i = 0; i < n; i++)
            if (tag[i] >= 1 && tag[i] <= n) tag_to_idx[tag[i] - 1] = i;
    }
    int builds = 0;
    int need = 1;
    for (int s = -1; s < nsteps; s++) {
        uint32_t step = first_step + (uint32_t)s;
        if (s >= 0) {
            for (int i = 0; i < n; i++) {
                double dtm = 0.5 * ff->dt / ff->mass[type[i] - 1];
                for (int d = 0; d < 3; d++) {
                    v[3 * i + d] += dtm * f[3 * i + d];
                    double p = x[3 * i + d] + ff->dt * v[3 * i + d];
                    double hi = lo[d] + L[d];
                    while (p >= hi || p < lo[d]) p -= L[d] * ((p >= hi) - (p < lo[d]));
                    x[3 * i + d] = p;
                }
            }
            double h2 = 0.25 * skin * skin;
            need = 0;
            for (int i = 0; i < n && !need; i++) {
                double dx = min_image(x[3 * i] - xlast[3 * i], L[0]);
                double dy = min_image(x[3 * i + 1] - xlast[3 * i + 1], L[1]);
                double dz = min_image(x[3 * i + 2] - xlast[3 * i + 2], L[2]);
                if (dx * dx + dy * dy + dz * dz >= h2) need = 1;
            }
        }
        if (need) {
            builds++;
            for (long c = 0; c < ncell; c++) head[c] = -1;
            for (int i = n - 1; i >= 0; i--) {
                for (int d = 0; d < 3; d++) {
                    int k = (int)floor((x[3 * i + d] - lo[d]) / (L[d] / nc[d]));
                    if (k < 0) k = 0;
                    if (k >= nc[d]) k = nc[d] - 1;
                    cid[3 * i + d] = k;
                }
                long c = ((long)cid[3 * i] * nc[1] + cid[3 * i + 1]) * nc[2] + cid[3 * i + 2];
                next[i] = head[c];
                head[c] = i;
            }
            build_task bt[256];
            for (int t = 0; t < nt; t++) {
                bt[t].i0 = (int)((long)n * t / nt);
                bt[t].i1 = (int)((long)n * (t + 1) / nt);
                bt[t].n = n; bt[t].nmax = nmax; bt[t].head = head; bt[t].next = next;
                bt[t].cid = cid; bt[t].nc = nc; bt[t].x = x; bt[t].L = L; bt[t].cut2 = cut2;
                bt[t].nl = nl; bt[t].nn = nn;
            }
            for (int t = 1; t < nt; t++) pthread_create(&th[t], NULL, bench_build_range, &bt[t]);
            bench_build_range(&bt[0]);
            for (int t = 1; t < nt; t++) pthread_join(th[t], NULL);
            memcpy(xlast, x, sizeof(double) * 3 * n);
        }
        for (int t = 0; t < nt; t++) {
            task[t].i0 = (int)((long)n * t / nt);
            task[t].i1 = (int)((long)n * (t + 1) / nt);
            task[t].n = n; task[t].nmax = nmax;
            task[t].tag = tag; task[t].type = type; task[t].nl = nl; task[t].nn = nn;
            task[t].x = x; task[t].v = v; task[t].L = L; task[t].ff = ff;
            task[t].fl = fpriv + (size_t)3 * n * t;
            task[t].step = step; task[t].sig_scale = sig_scale;
        }
        for (int t = 1; t < nt; t++) pthread_create(&th[t], NULL, bench_force_range, &task[t]);
        bench_force_range(&task[0]);
        for (int t = 1; t < nt; t++) pthread_join(th[t], NULL);
        {
            build_task rt[256];
            for (int t = 0; t < nt; t++) {
                rt[t].i0 = (int)((long)n * t / nt);
                rt[t].i1 = (int)((long)n * (t + 1) / nt);
                rt[t].n = n; rt[t].nt = nt; rt[t].f = f; rt[t].fpriv = fpriv;
            }
            for (int t = 1; t < nt; t++) pthread_create(&th[t], NULL, bench_reduce_range, &rt[t]);
            bench_reduce_range(&rt[0]);
            for (int t = 1; t < nt; t++) pthread_join(th[t], NULL);
        }
        if (tag_to_idx) {
            double pe = 0.0, vir[6] = {0, 0, 0, 0, 0, 0};
            if (bond_forces(n, tag_to_idx, n, x, lo, L, ff, nbonds, bonds, f, &pe, vir) == -1) builds = -3;
        }
        if (s >= 0) {
            for (int i = 0; i < n; i++) {
                double dtm = 0.5 * ff->dt / ff->mass[type[i] - 1];
                for (int d = 0; d < 3; d++) v[3 * i + d] += dtm * f[3 * i + d];
            }
        }
    }
    free(nl); free(nn); free(xlast); free(f); free(head); free(next); free(cid); free(fpriv);
    free(tag_to_idx);
    return builds;
}

int oracle_max_types(void) { return ORACLE_MAXT; }
int oracle_ff_size(void) { return (int)sizeof(oracle_ff); }
