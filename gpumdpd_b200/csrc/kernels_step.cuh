// kernels_step.cuh -- per-step kernels: mDPD density, pair forces (+bonds, fused),
// fused final/initial velocity-Verlet integration, per-replica bookkeeping, RDF.
#pragma once
#include "kernels.cuh"

struct StepArgs {
    const RepDesc* reps;
    const int* warp_rep;
    RepState* rstate;
    int P;
    int nmax;
    int maxb;
    const float4* coeff;   // 3 float4 per ordered type pair, per replica
    const float2* mass;    // (m, 1/m) per type, per replica
    const float4* bondc;   // per bond type, per replica: harmonic {k, r0}; fene {K, R0, eps, sigma}
    PBuf buf;
    const int* parity;
    float4* force4;
    float* rho;
    const float4* last4;
    const int* tag2idx;
    const int* ncount;
    const int* nlist;
    double* acc;           // [nrep][DPD_ACC_SLOTS][DPD_NACC]
    double* ring;          // [nrep][DPD_RING_ROWS][DPD_THERMO_FIELDS]
    unsigned long long* rdf_hist;
    const int* cstart;     // cell ranges of the last list build
    const int* crank;
    int* build_flag;       // [2]
    uint32_t* phase;
    int nrep;
    int mode;              // integrate kernel: 0 = per-step (final+initial), 1 = initial only
    const FixDesc* fix;    // [nrep] group fixes (null when no replica has one)
    FixOut* fixo;          // [nrep]
    double* spring_ring;   // [nrep][DPD_RING_ROWS][6] spring records (null: none)
    unsigned int* ticket;  // blocks of k_integrate_adv done (reset by the last one)
    const GCDesc* gc;      // [nrep][DPD_MAX_GC] group computes (null when none)
    const float4* uw0;     // [atoms of all replicas] initial unwrapped positions by global tag
    double* gc_ring;       // [computes][DPD_RING_ROWS][4] rows {step, values}
    int* gc_count;         // [computes] rows written
    int* wall_ext;         // [nrep][8] wall extents, order-preserving ints: two_wall k at
                           // 2k (max of its lo wall), 2k+1 (min of its hi wall); wall_contact
                           // compute k at 4+k
};

// order-preserving int image of a float (atomicMax / atomicMin on positions)
__device__ __forceinline__ int ford(float f)
{
    const int b = __float_as_int(f);
    return b >= 0 ? b : b ^ 0x7fffffff;
}
__device__ __forceinline__ float ford_inv(int b) { return __int_as_float(b >= 0 ? b : b ^ 0x7fffffff); }

// position of a slot along axis q wrapped into [lo, lo + L) (the reference's d_pos)
__device__ __forceinline__ float wrapped_coord(const RepDesc& d, double L, const float4& p, int q)
{
    const int code = __float_as_int(p.w);
    const float o = q == 0 ? p.x : (q == 1 ? p.y : p.z);
    double xa = (double)((code >> (q * DPD_CELL_BITS)) & DPD_MAX_NC) * (double)d.w[q] + (double)o;
    xa -= floor(xa / L) * L;
    if (xa >= L) xa -= L;
    return (float)(d.lo[q] + xa);
}

__device__ __forceinline__ void add_axis(float4& p, int q, float dx)
{
    if (q == 0) p.x += dx;
    else if (q == 1) p.y += dx;
    else p.z += dx;
}
__device__ __forceinline__ void flip_axis(float4& v, int q)
{
    if (q == 0) v.x = -v.x;
    else if (q == 1) v.y = -v.y;
    else v.z = -v.z;
}

// group computes due at the current step of a replica (bit k: compute k), evaluated with
// the end-of-step state after the thermo (src/main/utils.cuh:191-194, 290-291)
__device__ __forceinline__ int gc_due(const StepArgs& a, const RepDesc& d, const RepState& st, int r)
{
    int due = 0;
    for (int k = 0; k < d.gc_n; k++)
        if ((st.step % a.gc[r * DPD_MAX_GC + k].freq) == 0u) due |= 1 << k;
    return due;
}

// end-of-step fixes due at the current step of a replica: bit 0 rvcm, bit 1 recenter
// (src/main/utils.cuh:287: Fix_end_of_step after the final half kick of steps >= 1)
__device__ __forceinline__ int fix_eos_due(const FixDesc& f, const RepState& st, int mode)
{
    if (mode != 0 || st.zero_pending || !(st.step <= st.target)) return 0;
    int due = 0;
    if (f.rvcm_mask && (st.step % f.rvcm_freq) == 0u) due |= 1;
    if (f.recenter_mask && (st.step % f.recenter_freq) == 0u) due |= 2;
    return due;
}

__device__ __forceinline__ bool rep_active(const RepState& st) { return st.step <= st.target; }

// displacement between two arbitrary particles (bonds, RDF)
__device__ __forceinline__ void disp3(const RepDesc& d, int ci, float4 pi, float4 pj, float& dx,
                                      float& dy, float& dz)
{
    const int cj = __float_as_int(pj.w);
    dx = disp1(cell_x(ci), cell_x(cj), pi.x, pj.x, d.nc[0], d.w[0], d.L[0]);
    dy = disp1(cell_y(ci), cell_y(cj), pi.y, pj.y, d.nc[1], d.w[1], d.L[1]);
    dz = disp1(cell_z(ci), cell_z(cj), pi.z, pj.z, d.nc[2], d.w[2], d.L[2]);
}

// per-warp table of the 27 cell shifts (c_i - c_j) * w of a replica
__device__ __forceinline__ void fill_shift(float4* tab, const RepDesc& d, int lane)
{
    if (lane < 27) {
        const int dx = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dz = lane % 3 - 1;
        tab[lane] = make_float4(__int2float_rn(dx) * d.w[0], __int2float_rn(dy) * d.w[1],
                                __int2float_rn(dz) * d.w[2], 0.0f);
    }
}

// displacement of a listed pair: (o_i - o_j) + (c_i - c_j) w, bit-identical to the
// list predicate
__device__ __forceinline__ void pair_disp(const float4* tab, int ent, float4 pi, float4 pj, float& dx,
                                          float& dy, float& dz)
{
    const float4 sh = tab[(uint32_t)ent >> DPD_CODE_SHIFT];
    dx = __fadd_rn(__fsub_rn(pi.x, pj.x), sh.x);
    dy = __fadd_rn(__fsub_rn(pi.y, pj.y), sh.y);
    dz = __fadd_rn(__fsub_rn(pi.z, pj.z), sh.z);
}

// ---------------------------------------------------------------------------------
// mDPD local density, src/force/pair_mdpd.cu:219-300: rho_i = sum_j 15/(2 pi rd^3)
// max(0, 1-r/rd)^2 over the half list, both sides.
__global__ void __launch_bounds__(256) k_density(StepArgs a)
{
    griddep_wait();
    __shared__ float4 tab[8][27];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.P) return;
    const int r = a.warp_rep[s >> 5];
    const RepDesc& d = a.reps[r];
    if (!rep_active(a.rstate[r]) || d.style != 1) return;  // warp-uniform
    fill_shift(tab[warp], d, lane);
    __syncwarp();
    if (s >= d.p_end) return;
    const int par = *a.parity;
    const float4* pos = a.buf.pos[par];
    const float4* vel = a.buf.vel[par];
    const float4 pi = pos[s];
    const int ti = type0_of(vel[s].w);
    const float4* crow = a.coeff + d.coeff_off + ti * d.ntypes * 3;
    const int n = min(a.ncount[s], a.nmax);
    const int* lst = a.nlist + ((size_t)(s >> 5) * a.nmax) * 32 + lane;
    float rho_i = 0.0f;
    for (int k = 0; k < n; k++) {
        const int ent = __ldg(lst + (size_t)k * 32);
        const int j = ent & DPD_J_MASK;
        const float4 pj = __ldg(pos + j);
        float dx, dy, dz;
        pair_disp(tab[warp], ent, pi, pj, dx, dy, dz);
        const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
        const int tj = type0_of(__ldg(&vel[j].w));
        const float4 c2 = __ldg(crow + tj * 3 + 2);
        if (r2 < c2.x) {
            const float4 c1 = __ldg(crow + tj * 3 + 1);
            const float rr = r2 * rsqrtf(fmaxf(r2, 1e-30f));
            const float wd = fmaxf(1.0f - rr * c1.w, 0.0f);
            const float add = c2.z * wd * wd;
            rho_i += add;
            atomicAdd(&a.rho[j], add);
        }
    }
    atomicAdd(&a.rho[s], rho_i);
}

// Bond forces computed by both partners (each takes its own side; energy and virial
// halved), so bonds need no atomics.  Harmonic: src/force/bond_harmonic.cu:208-268
// (E = k (r-r0)^2, F_i = -2k(r-r0)/r d).  FENE: -0.5 K R0^2 ln(1-(r/R0)^2) + WCA.
template <bool LOG>
__device__ __forceinline__ void bond_loop(const StepArgs& a, const RepDesc& d, const float4* pos,
                                          const int2* bonds, const int r_idx, const int s,
                                          const float4 pi, float& fx, float& fy, float& fz,
                                          double (&accv)[8])
{
    const int ci = __float_as_int(pi.w);
    for (int b = 0; b < a.maxb; b++) {
        const int2 bp = bonds[(size_t)b * a.P + s];
        if (bp.x <= 0) break;
        if (bp.x > d.n_real) {
            atomicOr(&a.rstate[r_idx].status, ST_BOND_MISSING);
            continue;
        }
        const int j = a.tag2idx[d.tag_base + bp.x - 1];
        if (j < d.p_begin || j >= d.p_end) {
            atomicOr(&a.rstate[r_idx].status, ST_BOND_MISSING);
            continue;
        }
        const float4 pj = pos[j];
        float dx, dy, dz;
        disp3(d, ci, pi, pj, dx, dy, dz);
        const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
        const float4 bc = __ldg(a.bondc + d.bond_off + bp.y - 1);
        float fbond = 0.0f, e = 0.0f;
        if (d.bond_style == 1) {
            const float r = sqrtf(r2);
            const float dr = r - bc.y;
            fbond = r > 0.0f ? -2.0f * bc.x * dr / r : 0.0f;
            e = bc.x * dr * dr;
        } else if (d.bond_style == 2) {
            float rr = r2 / (bc.y * bc.y);
            if (rr >= 1.0f) {
                atomicOr(&a.rstate[r_idx].status, ST_FENE_BROKEN);
                rr = 0.999f;
            }
            fbond = -bc.x / (1.0f - rr);
            e = -0.5f * bc.x * bc.y * bc.y * logf(1.0f - rr);
            if (bc.z > 0.0f && r2 < 1.2599210498948732f * bc.w * bc.w) {
                const float sr2 = bc.w * bc.w / r2;
                const float sr6 = sr2 * sr2 * sr2;
                fbond += 48.0f * bc.z * sr6 * (sr6 - 0.5f) / r2;
                e += 4.0f * bc.z * sr6 * (sr6 - 1.0f) + bc.z;
            }
        }
        const float bx = dx * fbond, by = dy * fbond, bz = dz * fbond;
        fx += bx;
        fy += by;
        fz += bz;
        if (LOG) {
            accv[1] += 0.5 * (double)e;
            accv[2] += 0.5 * (double)dx * bx;
            accv[3] += 0.5 * (double)dx * by;
            accv[4] += 0.5 * (double)dx * bz;
            accv[5] += 0.5 * (double)dy * by;
            accv[6] += 0.5 * (double)dy * bz;
            accv[7] += 0.5 * (double)dz * bz;
        }
    }
}

// One DPD / mDPD pair (src/force/pair_dpd.cu:495-547, src/force/pair_mdpd.cu:616-672):
// F = [A w + B (rho_i+rho_j) w_d - gamma w^2 (r.v)/r + sigma w theta] r/r with
// w = 1 - r/rc, theta = Saru(min tag, max tag, seed + step).  Returns false when the
// pair is outside its cutoff.
template <int STYLE, bool LOG>
__device__ __forceinline__ bool pair_force(const float4* crow, float r2, float dx, float dy, float dz,
                                           float4 vi, float4 vj, float rho_i, float rho_j, uint32_t seed,
                                           uint32_t step, float& fx, float& fy, float& fz,
                                           double (&accv)[8])
{
    const int tj = type0_of(vj.w);
    const float4 c0 = __ldg(crow + tj * 3 + 0);
    if (!(r2 <= c0.w)) return false;
    const float rinv = rsqrtf(r2);
    const float r = r2 * rinv;
    if (r < 1.0e-10f) return false;
    const float4 c1 = __ldg(crow + tj * 3 + 1);
    const float dot = dx * (vi.x - vj.x) + dy * (vi.y - vj.y) + dz * (vi.z - vj.z);
    const float wc = 1.0f - r * c1.x;
    const int tagi = tag_of(vi.w), tagj = tag_of(vj.w);
    const float th = saru_theta((uint32_t)min(tagi, tagj), (uint32_t)max(tagi, tagj), seed, step);
    float fpair = c0.x * wc;
    float wd = 0.0f;
    float4 c2;
    if (STYLE == 1) {
        c2 = __ldg(crow + tj * 3 + 2);
        wd = fmaxf(1.0f - r * c1.w, 0.0f);
        fpair += c1.z * (rho_i + rho_j) * wd;
    }
    fpair -= c0.y * wc * wc * dot * rinv;
    fpair += c0.z * wc * th;
    fpair *= rinv;
    fx = dx * fpair;
    fy = dy * fpair;
    fz = dz * fpair;
    if (LOG) {
        double pe = (double)(c1.y * wc * wc);
        if (STYLE == 1) pe += (double)(c2.y * (rho_i + rho_j) * wd * wd);
        accv[0] += pe;
        accv[2] += (double)dx * fx;
        accv[3] += (double)dx * fy;
        accv[4] += (double)dx * fz;
        accv[5] += (double)dy * fy;
        accv[6] += (double)dy * fz;
        accv[7] += (double)dz * fz;
    }
    return true;
}

// ---------------------------------------------------------------------------------
// Pair force, thread-per-particle schedule (kept for comparison by the tuner).
template <int STYLE, bool BONDS>
__global__ void __launch_bounds__(256) k_pair(StepArgs a)
{
    griddep_wait();
    __shared__ float4 tab[8][27];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    int r = -1;
    bool work = false, log = false, wactive = false;
    uint32_t step = 0;
    if (s < a.P) {
        r = a.warp_rep[s >> 5];
        const RepState st = a.rstate[r];
        const RepDesc& d = a.reps[r];
        wactive = rep_active(st) && d.style == STYLE;
        work = wactive && s < d.p_end;
        step = st.step;
        log = wactive && (step % (uint32_t)d.log_f) == 0u;
        if (wactive) fill_shift(tab[warp], d, lane);
    }
    __syncwarp();
    double accv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (work) {
        const RepDesc& d = a.reps[r];
        const int par = *a.parity;
        const float4* pos = a.buf.pos[par];
        const float4* vel = a.buf.vel[par];
        const float4 pi = pos[s];
        const float4 vi = vel[s];
        const float rho_i = STYLE == 1 ? a.rho[s] : 0.0f;
        const float4* crow = a.coeff + d.coeff_off + type0_of(vi.w) * d.ntypes * 3;
        const int n = min(a.ncount[s], a.nmax);
        const int* lst = a.nlist + ((size_t)(s >> 5) * a.nmax) * 32 + lane;
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        for (int k = 0; k < n; k++) {
            const int ent = __ldg(lst + (size_t)k * 32);
            const int j = ent & DPD_J_MASK;
            const float4 pj = __ldg(pos + j);
            float dx, dy, dz;
            pair_disp(tab[warp], ent, pi, pj, dx, dy, dz);
            const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
            if (r2 > d.rcmax2) continue;
            const float4 vj = __ldg(vel + j);
            const float rho_j = STYLE == 1 ? __ldg(a.rho + j) : 0.0f;
            float gx, gy, gz;
            bool ok = log ? pair_force<STYLE, true>(crow, r2, dx, dy, dz, vi, vj, rho_i, rho_j, d.seed, step, gx, gy, gz, accv)
                          : pair_force<STYLE, false>(crow, r2, dx, dy, dz, vi, vj, rho_i, rho_j, d.seed, step, gx, gy, gz, accv);
            if (!ok) continue;
            fx += gx;
            fy += gy;
            fz += gz;
            atomicAdd(&a.force4[j], make_float4(-gx, -gy, -gz, 0.0f));
        }
        if (BONDS) {
            if (log) bond_loop<true>(a, d, pos, a.buf.bonds[par], r, s, pi, fx, fy, fz, accv);
            else bond_loop<false>(a, d, pos, a.buf.bonds[par], r, s, pi, fx, fy, fz, accv);
        }
        atomicAdd(&a.force4[s], make_float4(fx, fy, fz, 0.0f));
    }
    if (__syncthreads_or(log)) {
        const int fields[8] = {ACC_PAIR_PE, ACC_BOND_PE, ACC_VIR + 0, ACC_VIR + 1,
                               ACC_VIR + 2, ACC_VIR + 3, ACC_VIR + 4, ACC_VIR + 5};
        acc_flush<8>(accv, fields, log ? r : -1, a.acc);
    }
}

// ---------------------------------------------------------------------------------
// Pair force for small grids: one thread per list entry.  Warp w takes line k of the
// warp-interleaved list (the k-th entries of 32 slots) with k = w / (P/32), so the few
// pairs of a small system spread over the whole GPU instead of a few warps walking them
// in turn, and the warps past the longest list return at once.  Both sides of a pair are
// float4 reductions; the bonds of a slot are taken by its k = 0 thread.
template <int STYLE, bool BONDS>
__global__ void __launch_bounds__(256) k_pair_entry(StepArgs a)
{
    griddep_wait();
    __shared__ float4 tab[8][27];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nw = a.P >> 5;
    const int line = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int k = line / nw, wslot = line - k * nw;
    int r = -1;
    bool wactive = false, log = false;
    uint32_t step = 0;
    if (k < a.nmax) {
        r = a.warp_rep[wslot];
        const RepState st = a.rstate[r];
        const RepDesc& d = a.reps[r];
        wactive = rep_active(st) && d.style == STYLE;
        step = st.step;
        log = wactive && (step % (uint32_t)d.log_f) == 0u;
        if (wactive) fill_shift(tab[warp], d, lane);
    }
    __syncwarp();
    double accv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int s = wslot * 32 + lane;
    if (wactive && s < a.reps[r].p_end) {
        const RepDesc& d = a.reps[r];
        const int par = *a.parity;
        const float4* pos = a.buf.pos[par];
        if (k < min(a.ncount[s], a.nmax)) {
            const float4* vel = a.buf.vel[par];
            const int ent = __ldg(a.nlist + ((size_t)wslot * a.nmax + k) * 32 + lane);
            const int j = ent & DPD_J_MASK;
            const float4 pi = pos[s], pj = __ldg(pos + j);
            float dx, dy, dz;
            pair_disp(tab[warp], ent, pi, pj, dx, dy, dz);
            const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
            if (r2 <= d.rcmax2) {
                const float4 vi = vel[s], vj = __ldg(vel + j);
                const float rho_i = STYLE == 1 ? a.rho[s] : 0.0f, rho_j = STYLE == 1 ? __ldg(a.rho + j) : 0.0f;
                const float4* crow = a.coeff + d.coeff_off + type0_of(vi.w) * d.ntypes * 3;
                float gx, gy, gz;
                const bool ok = log ? pair_force<STYLE, true>(crow, r2, dx, dy, dz, vi, vj, rho_i, rho_j, d.seed, step, gx, gy, gz, accv)
                                    : pair_force<STYLE, false>(crow, r2, dx, dy, dz, vi, vj, rho_i, rho_j, d.seed, step, gx, gy, gz, accv);
                if (ok) {
                    atomicAdd(&a.force4[j], make_float4(-gx, -gy, -gz, 0.0f));
                    atomicAdd(&a.force4[s], make_float4(gx, gy, gz, 0.0f));
                }
            }
        }
        if (BONDS && k == 0) {
            float fx = 0.0f, fy = 0.0f, fz = 0.0f;
            const float4 pi = pos[s];
            if (log) bond_loop<true>(a, d, pos, a.buf.bonds[par], r, s, pi, fx, fy, fz, accv);
            else bond_loop<false>(a, d, pos, a.buf.bonds[par], r, s, pi, fx, fy, fz, accv);
            atomicAdd(&a.force4[s], make_float4(fx, fy, fz, 0.0f));
        }
    }
    if (__syncthreads_or(log)) {
        const int fields[8] = {ACC_PAIR_PE, ACC_BOND_PE, ACC_VIR + 0, ACC_VIR + 1,
                               ACC_VIR + 2, ACC_VIR + 3, ACC_VIR + 4, ACC_VIR + 5};
        acc_flush<8>(accv, fields, log ? r : -1, a.acc);
    }
}

// ---------------------------------------------------------------------------------
// Pair force, warp pair-queue schedule.  Thread-per-particle loops diverge on the
// ~130-instruction Saru evaluation (only the pairs inside rc need it), so each warp
// first filters its 32 particles' list candidates (DPD_U per lane per iteration, loads
// issued before use), compacts the pairs inside the cutoff into a shared-memory queue
// with a ballot, and evaluates 32 queued pairs at a time with every lane busy.  The
// i-side force is reduced through shared-memory atomics, the j-side with one float4
// atomic per pair.
#define DPD_U 4                 // candidates per lane per filter iteration
#define DPD_Q (32 + 32 * DPD_U)  // queue capacity per warp
template <int STYLE, bool BONDS, int MINB, bool ISMEM>
__global__ void __launch_bounds__(256, MINB) k_pair_q(StepArgs a)
{
    griddep_wait();
    __shared__ int sq_j[8][DPD_Q];
    __shared__ int sq_i[8][DPD_Q];
    __shared__ float4 sq_d[8][DPD_Q];
    __shared__ float4 s_vi[8][32];
    __shared__ float s_rho[8][32];
    __shared__ float s_f[8][32][3];
    __shared__ float4 tab[8][27];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    int r = -1;
    bool work = false, log = false, wactive = false;
    uint32_t step = 0;
    if (s < a.P) {
        r = a.warp_rep[s >> 5];
        const RepState st = a.rstate[r];
        const RepDesc& d = a.reps[r];
        wactive = rep_active(st) && d.style == STYLE;
        work = wactive && s < d.p_end;
        step = st.step;
        log = wactive && (step % (uint32_t)d.log_f) == 0u;
    }
    double accv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (wactive) {  // warp-uniform
        const RepDesc& d = a.reps[r];
        const int par = *a.parity;
        const float4* pos = a.buf.pos[par];
        const float4* vel = a.buf.vel[par];
        fill_shift(tab[warp], d, lane);
        float4 pi = make_float4(0, 0, 0, 0), vi = make_float4(0, 0, 0, 0);
        float rho_i = 0.0f;
        int n = 0;
        if (work) {
            pi = pos[s];
            vi = vel[s];
            if (STYLE == 1) rho_i = a.rho[s];
            n = min(a.ncount[s], a.nmax);
        }
        s_vi[warp][lane] = vi;
        s_rho[warp][lane] = rho_i;
        s_f[warp][lane][0] = 0.0f;
        s_f[warp][lane][1] = 0.0f;
        s_f[warp][lane][2] = 0.0f;
        const int nw = __reduce_max_sync(0xffffffffu, n);
        const int* lst = a.nlist + ((size_t)(s >> 5) * a.nmax) * 32 + lane;
        const float rcmax2 = d.rcmax2;
        const unsigned lt = (1u << lane) - 1u;
        const float4* cbase = a.coeff + d.coeff_off;
        const int nt = d.ntypes;
        const uint32_t seed = d.seed;
        // Queue invariant: entries [base, qn) are pending.  The filter runs only when
        // fewer than 32 are pending (they are first moved to the front), so before it
        // qn <= 31 and after it qn <= 31 + 32*DPD_U < DPD_Q.
        int k = 0, qn = 0, base = 0;
        __syncwarp();
        while (true) {
            if (k < nw && qn - base < 32) {
                if (base > 0) {
                    // source starts at base >= 32, destination ends below 32: no overlap
                    const int left = qn - base;
                    if (lane < left) {
                        sq_j[warp][lane] = sq_j[warp][base + lane];
                        sq_i[warp][lane] = sq_i[warp][base + lane];
                        sq_d[warp][lane] = sq_d[warp][base + lane];
                    }
                    qn = left;
                    base = 0;
                    __syncwarp();
                }
                // list entries carry the shift code in bits 27-31, so they may be negative
                // as ints: validity is k + u < n, not the sign
                int ee[DPD_U];
                float4 pp[DPD_U];
#pragma unroll
                for (int u = 0; u < DPD_U; u++) ee[u] = (k + u < n) ? __ldg(lst + (size_t)(k + u) * 32) : 0;
#pragma unroll
                for (int u = 0; u < DPD_U; u++)
                    if (k + u < n) pp[u] = __ldg(pos + (ee[u] & DPD_J_MASK));
#pragma unroll
                for (int u = 0; u < DPD_U; u++) {
                    bool hit = false;
                    float dx = 0, dy = 0, dz = 0, r2 = 0;
                    if (k + u < n) {
                        pair_disp(tab[warp], ee[u], pi, pp[u], dx, dy, dz);
                        r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
                        hit = r2 <= rcmax2;
                    }
                    const unsigned m = __ballot_sync(0xffffffffu, hit);
                    if (hit) {
                        const int pos_q = qn + __popc(m & lt);
                        sq_j[warp][pos_q] = ee[u] & DPD_J_MASK;
                        sq_i[warp][pos_q] = lane;
                        sq_d[warp][pos_q] = make_float4(dx, dy, dz, r2);
                    }
                    qn += __popc(m);
                }
                k += DPD_U;
            }
            const bool tail = k >= nw;
            const int avail = qn - base;
            if (avail < 32 && !(tail && avail > 0)) {
                if (tail) break;  // nothing pending and no candidates left
                continue;         // partial chunk: filter more candidates first
            }
            __syncwarp();
            const int cnt = min(avail, 32);
            if (lane < cnt) {
                const int j = sq_j[warp][base + lane];
                const int il = sq_i[warp][base + lane];
                const float4 dd = sq_d[warp][base + lane];
                const float4 vv = s_vi[warp][il];
                const float4 vj = __ldg(vel + j);
                const float4* crow = cbase + type0_of(vv.w) * nt * 3;
                const float rho_j = STYLE == 1 ? __ldg(a.rho + j) : 0.0f;
                float fx, fy, fz;
                bool ok = log ? pair_force<STYLE, true>(crow, dd.w, dd.x, dd.y, dd.z, vv, vj, s_rho[warp][il], rho_j, seed, step, fx, fy, fz, accv)
                              : pair_force<STYLE, false>(crow, dd.w, dd.x, dd.y, dd.z, vv, vj, s_rho[warp][il], rho_j, seed, step, fx, fy, fz, accv);
                if (ok) {
                    if (ISMEM) {
                        atomicAdd(&s_f[warp][il][0], fx);
                        atomicAdd(&s_f[warp][il][1], fy);
                        atomicAdd(&s_f[warp][il][2], fz);
                    } else {
                        atomicAdd(&a.force4[(s & ~31) + il], make_float4(fx, fy, fz, 0.0f));
                    }
                    atomicAdd(&a.force4[j], make_float4(-fx, -fy, -fz, 0.0f));
                }
            }
            __syncwarp();  // chunk entries are read before any compaction overwrites them
            base += cnt;
            if (base == qn) {
                qn = 0;
                base = 0;
            }
        }
        __syncwarp();
        float fx = s_f[warp][lane][0], fy = s_f[warp][lane][1], fz = s_f[warp][lane][2];
        if (work) {
            if (BONDS) {
                if (log) bond_loop<true>(a, d, pos, a.buf.bonds[par], r, s, pi, fx, fy, fz, accv);
                else bond_loop<false>(a, d, pos, a.buf.bonds[par], r, s, pi, fx, fy, fz, accv);
            }
            atomicAdd(&a.force4[s], make_float4(fx, fy, fz, 0.0f));
        }
    }
    if (__syncthreads_or(log)) {
        const int fields[8] = {ACC_PAIR_PE, ACC_BOND_PE, ACC_VIR + 0, ACC_VIR + 1,
                               ACC_VIR + 2, ACC_VIR + 3, ACC_VIR + 4, ACC_VIR + 5};
        acc_flush<8>(accv, fields, log ? r : -1, a.acc);
    }
}

// ---------------------------------------------------------------------------------
// Pair force, flattened warp schedule.  The list entries of a warp's 32 particles are
// taken as one sequence, particle by particle (lane-major); an exclusive scan of the
// counts gives each particle's start.  Every iteration evaluates 32 consecutive entries,
// one per lane, so all lanes are busy whatever the per-particle counts, with no
// compaction queue; the owner of entry t is found by a 5-step binary search over the
// starts.  The next chunk's entries are fetched while the current chunk is evaluated, and
// the pos/vel gathers of a chunk are issued together, so each chunk waits for one L2
// round trip.  Entries outside rc idle their lane for the Saru part, so this schedule
// suits small skins (at skin 0 every listed pair is inside rc).  Both the i-side and
// j-side forces go to L2 as float4 reductions.  FP64 log sums are flushed per warp, so
// no block barrier is needed on non-log steps.
// LOGM: 2 = any step; 0 = non-log steps only (no FP64 sums: fewer registers, more
// warps per SM); 1 = log steps only.  0 and 1 are launched together, each returning at
// once on the other kind of step.
// SEG: the i-side forces of an iteration are summed per owner in registers first (the flat
// entries of one owner sit in consecutive lanes: a segmented warp scan), so one float4
// reduction per owner and iteration reaches L2 instead of one per pair.
// Warp-level FP64 sums of a replica kept across several calls (grid-stride loops): added
// to `tot` while the replica stays the same, flushed to the spread accumulators (one
// atomic per field and warp) when it changes and at the end.
template <int NV>
struct WarpAcc {
    double tot[NV];
    int rep = -1;
    __device__ __forceinline__ WarpAcc()
    {
#pragma unroll
        for (int k = 0; k < NV; k++) tot[k] = 0.0;
    }
    // warp-uniform r
    __device__ __forceinline__ void add(const double (&v)[NV], int r, const int* fields, double* acc)
    {
        if (r != rep) {
            flush(fields, acc);
            rep = r;
        }
#pragma unroll
        for (int k = 0; k < NV; k++) tot[k] += v[k];
    }
    __device__ __forceinline__ void flush(const int* fields, double* acc)
    {
        if (rep >= 0) acc_flush_warp<NV>(tot, fields, rep, acc);
#pragma unroll
        for (int k = 0; k < NV; k++) tot[k] = 0.0;
        rep = -1;
    }
};

template <int STYLE, bool BONDS, int LOGM = 2, bool SEG = false>
__device__ __forceinline__ void pair_flat_warp(const StepArgs& a, const int s, WarpAcc<8>* keep = nullptr)
{
    __shared__ int s_start[8][33];
    __shared__ float4 s_pi[8][32];
    __shared__ float4 s_vi[8][32];
    __shared__ float s_rho[8][32];
    __shared__ float4 tab[8][27];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if ((s & ~31) >= a.P) return;  // whole warp beyond the slots
    const int r = a.warp_rep[s >> 5];
    const RepState st = a.rstate[r];
    const RepDesc& d = a.reps[r];
    if (!rep_active(st) || d.style != STYLE) return;  // warp-uniform
    const bool work = s < d.p_end;
    const uint32_t step = st.step;
    const bool log_step = (step % (uint32_t)d.log_f) == 0u;
    if ((LOGM == 0 && log_step) || (LOGM == 1 && !log_step)) return;  // warp-uniform
    const bool log = LOGM == 2 ? log_step : LOGM == 1;
    const int fields[8] = {ACC_PAIR_PE, ACC_BOND_PE, ACC_VIR + 0, ACC_VIR + 1,
                           ACC_VIR + 2, ACC_VIR + 3, ACC_VIR + 4, ACC_VIR + 5};
    // FP64 sums: with `keep` (grid-stride calls) straight into the warp's kept sums, which
    // are flushed when the warp moves to another replica; else this call's own
    double own[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (keep && keep->rep != r) {
        keep->flush(fields, a.acc);
        keep->rep = r;
    }
    double (&accv)[8] = keep ? keep->tot : own;
    const int par = *a.parity;
    const float4* pos = a.buf.pos[par];
    const float4* vel = a.buf.vel[par];
    fill_shift(tab[warp], d, lane);
    float4 pi = make_float4(0, 0, 0, 0), vi = make_float4(0, 0, 0, 0);
    float rho_i = 0.0f;
    int n = 0;
    if (work) {
        pi = pos[s];
        vi = vel[s];
        if (STYLE == 1) rho_i = a.rho[s];
        n = min(a.ncount[s], a.nmax);
    }
    s_pi[warp][lane] = pi;
    s_vi[warp][lane] = vi;
    s_rho[warp][lane] = rho_i;
    int incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    s_start[warp][lane] = incl - n;
    if (lane == 31) s_start[warp][32] = total;
    __syncwarp();
    const int* wl = a.nlist + (size_t)(s >> 5) * a.nmax * 32;
    const float rcmax2 = d.rcmax2;
    const float4* cbase = a.coeff + d.coeff_off;
    const int nt = d.ntypes;
    const uint32_t seed = d.seed;
    const int wbase = s & ~31;
    // owner lane and list entry of flat entry t (t < total)
    auto locate = [&](int t, int& l, int& ent) {
        int lo = 0;  // largest l with start[l] <= t (empty particles share a start)
#pragma unroll
        for (int stp = 16; stp >= 1; stp >>= 1)
            if (s_start[warp][lo + stp] <= t) lo += stp;
        l = lo;
        // a plain load: the fused kernel reads entries its own warp has just written
        ent = wl[(size_t)(t - s_start[warp][lo]) * 32 + lo];
    };
    int l_nx = 0, ent_nx = 0;
    if (lane < total) locate(lane, l_nx, ent_nx);
    for (int t0 = 0; t0 < total; t0 += 32) {
        const bool valid = t0 + lane < total;
        const int l = l_nx, ent = ent_nx;
        float4 pj = make_float4(0, 0, 0, 0), vj = make_float4(0, 0, 0, 0);
        float rho_j = 0.0f;
        const int j = ent & DPD_J_MASK;
        if (valid) {
            pj = __ldg(pos + j);
            vj = __ldg(vel + j);
            if (STYLE == 1) rho_j = __ldg(a.rho + j);
        }
        if (t0 + 32 + lane < total) locate(t0 + 32 + lane, l_nx, ent_nx);
        float ix = 0.0f, iy = 0.0f, iz = 0.0f;
        if (valid) {
            const float4 pil = s_pi[warp][l];
            float dx, dy, dz;
            pair_disp(tab[warp], ent, pil, pj, dx, dy, dz);
            const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
            if (r2 <= rcmax2) {
                const float4 vv = s_vi[warp][l];
                const float4* crow = cbase + type0_of(vv.w) * nt * 3;
                float fx, fy, fz;
                const bool ok = log ? pair_force<STYLE, true>(crow, r2, dx, dy, dz, vv, vj, s_rho[warp][l], rho_j, seed, step, fx, fy, fz, accv)
                                    : pair_force<STYLE, false>(crow, r2, dx, dy, dz, vv, vj, s_rho[warp][l], rho_j, seed, step, fx, fy, fz, accv);
                if (ok) {
                    atomicAdd(&a.force4[j], make_float4(-fx, -fy, -fz, 0.0f));
                    if (SEG) {
                        ix = fx;
                        iy = fy;
                        iz = fz;
                    } else {
                        atomicAdd(&a.force4[wbase + l], make_float4(fx, fy, fz, 0.0f));
                    }
                }
            }
        }
        if (SEG) {
            // lanes past the end get keys of their own: they never join a segment
            const int key = valid ? l : 32 + lane;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const float tx = __shfl_up_sync(0xffffffffu, ix, o);
                const float ty = __shfl_up_sync(0xffffffffu, iy, o);
                const float tz = __shfl_up_sync(0xffffffffu, iz, o);
                const int tk = __shfl_up_sync(0xffffffffu, key, o);
                if (lane >= o && tk == key) {
                    ix += tx;
                    iy += ty;
                    iz += tz;
                }
            }
            const int nk = __shfl_down_sync(0xffffffffu, key, 1);
            if (valid && (lane == 31 || nk != key) && (ix != 0.0f || iy != 0.0f || iz != 0.0f))
                atomicAdd(&a.force4[wbase + l], make_float4(ix, iy, iz, 0.0f));
        }
    }
    if (BONDS && work) {
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        if (log) bond_loop<true>(a, d, pos, a.buf.bonds[par], r, s, pi, fx, fy, fz, accv);
        else bond_loop<false>(a, d, pos, a.buf.bonds[par], r, s, pi, fx, fy, fz, accv);
        atomicAdd(&a.force4[s], make_float4(fx, fy, fz, 0.0f));
    }
    if (log && !keep) acc_flush_warp<8>(accv, fields, r, a.acc);
}

template <int STYLE, bool BONDS, int MINB>
__global__ void __launch_bounds__(256, MINB) k_pair_flat(StepArgs a)
{
    griddep_wait();
    pair_flat_warp<STYLE, BONDS>(a, blockIdx.x * blockDim.x + threadIdx.x);
}

template <int STYLE, bool BONDS, int LOGM, int MINB, bool SEG = false>
__global__ void __launch_bounds__(256, MINB) k_pair_flat_split(StepArgs a)
{
    griddep_wait();
    pair_flat_warp<STYLE, BONDS, LOGM, SEG>(a, blockIdx.x * blockDim.x + threadIdx.x);
}

// The log-step half of the split schedule as a small grid-stride launch: every block
// first checks whether any replica logs this step (the common answer is no, and then the
// launch costs one wave of tiny blocks instead of a full grid of early exits).
template <int STYLE, bool BONDS, bool SEG = false>
__global__ void __launch_bounds__(256, 4) k_pair_flat_logsteps(StepArgs a)
{
    griddep_wait();
    int any = 0;
    for (int r = threadIdx.x; r < a.nrep; r += blockDim.x) {
        const RepState st = a.rstate[r];
        any |= rep_active(st) && (st.step % (uint32_t)a.reps[r].log_f) == 0u;
    }
    if (!__syncthreads_or(any)) return;
    const int nvb = (a.P + 255) / 256;
    // the warp's sums over its virtual blocks, flushed once per replica
    WarpAcc<8> keep;
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
        pair_flat_warp<STYLE, BONDS, 1, SEG>(a, vb * 256 + threadIdx.x, &keep);
        __syncwarp();  // the warp's shared slots are reused by the next virtual block
    }
    const int fields[8] = {ACC_PAIR_PE, ACC_BOND_PE, ACC_VIR + 0, ACC_VIR + 1,
                           ACC_VIR + 2, ACC_VIR + 3, ACC_VIR + 4, ACC_VIR + 5};
    keep.flush(fields, a.acc);
}

// List build fused with the flattened pair force (DPD only: mDPD needs every density
// before any force).  On a build step each warp first builds its 32 particles' half list
// (the list of the build kernel, bit for bit), then evaluates those pairs at once, while
// the neighbours' positions are still in L1; on other steps it is the flattened pair
// kernel.  One launch instead of two, and the list is read back from L1/L2.
template <bool BONDS, int MINB>
__global__ void __launch_bounds__(256, MINB) k_build_pair(StepArgs a, BuildArgs b)
{
    griddep_wait();
    if (build_on(b)) {
        build_nlist_slot(b, blockIdx.x * blockDim.x + threadIdx.x);
        __syncwarp();
    }
    pair_flat_warp<0, BONDS>(a, blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------------
// Velocity Verlet, src/fix/fix_nve.cu:30-152, fused: final half kick of step n (and
// the thermo sums of step n), then initial half kick + drift of step n+1, the
// displacement check for the next list build (src/force/neigh_list.cu:483-514), and
// zeroing of the force accumulators.  Cells stay fixed between builds, so the drift
// only moves the offsets.
// LOGM: 2 = any step; 0 = every step except logged mode-0 steps (no FP64 sums: fewer
// registers); 1 = logged mode-0 steps only.  0 and 1 together cover every slot once.
// A step is logged when the thermo or (EXT) a group compute is due.  EXT adds the group
// fixes and the group computes.
template <int LOGM, bool EXT>
__device__ __forceinline__ void integrate_slot(const StepArgs& a, const int s, WarpAcc<10>* keep = nullptr)
{
    int r = -1;
    bool log = false;
    int gcd = 0;
    double accv[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    double gv[3 * DPD_MAX_GC];
    if (EXT && LOGM != 0)
        for (int k = 0; k < 3 * DPD_MAX_GC; k++) gv[k] = 0.0;
    if (s < a.P) {
        // the particle's three streams are requested first (every slot < P is valid
        // memory), so their latency overlaps the replica-state reads; on a logged step the
        // non-log kernel's loads are wasted, which costs less than putting the state read
        // before them on every other step
        const int par = *a.parity;
        float4* posp = a.buf.pos[par];
        float4* velp = a.buf.vel[par];
        float4 v = velp[s];
        const float4 f = a.force4[s];
        float4 p = posp[s];
        r = a.warp_rep[s >> 5];
        const RepState st = a.rstate[r];
        const RepDesc& d = a.reps[r];
        const bool active = rep_active(st);
        const bool work = active && s < d.p_end;
        const bool fin = a.mode == 0 && !st.zero_pending;
        log = a.mode == 0 && active && (st.step % (uint32_t)d.log_f) == 0u;
        if (EXT && a.mode == 0 && active && d.gc_n) gcd = gc_due(a, d, st, r);
        if ((LOGM == 0 && (log || gcd)) || (LOGM == 1 && !(log || gcd))) return;  // warp-uniform
        if (LOGM == 0) log = false;
        const bool init = a.mode == 1 ? true : st.step < st.target;
        const uint32_t next = a.mode == 1 ? st.step : st.step + 1u;
        const bool check = init && (next % (uint32_t)d.nl_f) == 0u;
        if (work) {
            const int t0 = type0_of(v.w);
            const float2 m = __ldg(a.mass + d.mass_off + t0);
            const bool integ = (d.integ_mask >> t0) & 1u;
            const float dt = d.dt;
            const float dtm = (0.5f * dt) * m.y;
            float4 fe = f;
            int eos = 0;
            bool shifted = false;
            if (EXT && a.fix) {
                // group fixes: the spring's share m_i F / M joins the force of both half
                // kicks (post_force); a due rvcm or recenter (end_of_step) has had its
                // final half kick in k_fix_sums<1> and acts here before the thermo sums
                const FixDesc& fd = a.fix[r];
                eos = fix_eos_due(fd, st, a.mode);
                if ((fd.spring_mask >> t0) & 1u) {
                    const FixOut& fo = a.fixo[r];
                    fe.x = __fmaf_rn(fo.spring_a[0], m.x, fe.x);
                    fe.y = __fmaf_rn(fo.spring_a[1], m.x, fe.y);
                    fe.z = __fmaf_rn(fo.spring_a[2], m.x, fe.z);
                }
                if (eos) {
                    const FixOut& fo = a.fixo[r];
                    if ((eos & 1) && ((fd.rvcm_mask >> t0) & 1u)) {
                        v.x -= fo.vcm[0];
                        v.y -= fo.vcm[1];
                        v.z -= fo.vcm[2];
                    }
                    if ((eos & 2) && ((fd.recenter_mask >> t0) & 1u)) {
                        p.x += fo.shift[0];
                        p.y += fo.shift[1];
                        p.z += fo.shift[2];
                        shifted = true;
                    }
                }
            }
            if (fin && integ && !eos) {
                v.x = __fmaf_rn(dtm, fe.x, v.x);
                v.y = __fmaf_rn(dtm, fe.y, v.y);
                v.z = __fmaf_rn(dtm, fe.z, v.z);
            }
            if (log) {
                const double vx = v.x, vy = v.y, vz = v.z, mm = m.x;
                accv[0] = 0.5 * mm * (vx * vx + vy * vy + vz * vz);
                accv[1] = mm * vx * vx;
                accv[2] = mm * vx * vy;
                accv[3] = mm * vx * vz;
                accv[4] = mm * vy * vy;
                accv[5] = mm * vy * vz;
                accv[6] = mm * vz * vz;
                accv[7] = mm * vx;
                accv[8] = mm * vy;
                accv[9] = mm * vz;
            }
            if (EXT && LOGM != 0 && gcd) {
                // group computes on the end-of-step state: src/compute/compute_temp.cu:74-173
                // (kinetic energy), compute_rho.cu:109-207 (count inside the region, wrapped
                // positions), compute_msd.cu:80-175 (|x_unwrapped - x0_unwrapped|^2),
                // compute_tf.cu:80-181 (force, the spring's share included)
#pragma unroll
                for (int k = 0; k < DPD_MAX_GC; k++) {
                    if (!((gcd >> k) & 1)) continue;
                    const GCDesc& g = a.gc[r * DPD_MAX_GC + k];
                    if (!((g.mask >> t0) & 1u)) continue;
                    if (g.kind == 1) {
                        gv[3 * k] = 0.5 * (double)m.x * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
                    } else if (g.kind == 5) {
                        // src/compute/compute_wall_contact.cu:60-100,186-290: atoms within the
                        // cutoff of the wall group's extreme position
                        const float bound = ford_inv(a.wall_ext[r * 8 + 4 + k]);
                        const float cb = g.wall_side > 0 ? bound + g.cutoff : bound - g.cutoff;
                        if (g.wall_side > 0 ? cb > g.box_hi : cb < g.box_lo)
                            atomicOr(&a.rstate[r].status, ST_CONTACT_BOX);
                        const float xw = wrapped_coord(d, g.L[g.wall_dir], p, g.wall_dir);
                        const bool in = g.wall_side > 0 ? (xw >= bound && xw < cb) : (xw >= cb && xw < bound);
                        gv[3 * k] = in ? 1.0 : 0.0;
                    } else if (g.kind == 4) {
                        gv[3 * k] = fe.x;
                        gv[3 * k + 1] = fe.y;
                        gv[3 * k + 2] = fe.z;
                    } else {
                        const int code = __float_as_int(p.w);
                        const float o[3] = {p.x, p.y, p.z};
                        double xa[3];
#pragma unroll
                        for (int q = 0; q < 3; q++)
                            xa[q] = (double)((code >> (q * DPD_CELL_BITS)) & DPD_MAX_NC) * (double)d.w[q] + (double)o[q];
                        if (g.kind == 2) {
                            bool in = true;
#pragma unroll
                            for (int q = 0; q < 3; q++) {
                                double w = xa[q] - floor(xa[q] / g.L[q]) * g.L[q];
                                if (w >= g.L[q]) w -= g.L[q];
                                w += d.lo[q];
                                in = in && w >= g.region[2 * q] && w < g.region[2 * q + 1];
                            }
                            gv[3 * k] = in ? 1.0 : 0.0;
                        } else {
                            const int ti = d.tag_base + (int)((uint32_t)__float_as_int(v.w) >> DPD_TYPE_BITS) - 1;
                            const int4 im = a.buf.img[ti];
                            const float4 x0 = a.uw0[ti];
                            const double dx = d.lo[0] + xa[0] + (double)im.x * g.L[0] - x0.x;
                            const double dy = d.lo[1] + xa[1] + (double)im.y * g.L[1] - x0.y;
                            const double dz = d.lo[2] + xa[2] + (double)im.z * g.L[2] - x0.z;
                            gv[3 * k] = dx * dx + dy * dy + dz * dz;
                        }
                    }
                }
            }
            if (EXT && shifted && !init) posp[s] = p;
            if (init) {
                if (integ) {
                    v.x = __fmaf_rn(dtm, fe.x, v.x);
                    v.y = __fmaf_rn(dtm, fe.y, v.y);
                    v.z = __fmaf_rn(dtm, fe.z, v.z);
                    p.x = __fmaf_rn(dt, v.x, p.x);
                    p.y = __fmaf_rn(dt, v.y, p.y);
                    p.z = __fmaf_rn(dt, v.z, p.z);
                }
                bool moved = integ || shifted;
                if (EXT && a.fix) {
                    // fix move (initial_integrate, src/fix/fix_move.cu:33-80): v = V, x += V dt;
                    // then fix wall_reflect (post_integrate, src/fix/fix_wall_reflect.cu:84-125):
                    // a group atom past a wall is mirrored back, its normal velocity reversed
                    const FixDesc& fd = a.fix[r];
                    for (int k = 0; k < fd.n_move; k++)
                        if ((fd.move_mask[k] >> t0) & 1u) {
                            v.x = fd.move_v[k][0];
                            v.y = fd.move_v[k][1];
                            v.z = fd.move_v[k][2];
                            p.x += fd.move_v[k][0] * dt;
                            p.y += fd.move_v[k][1] * dt;
                            p.z += fd.move_v[k][2] * dt;
                            moved = true;
                        }
                    for (int k = 0; k < fd.n_reflect; k++)
                        if ((fd.refl_mask[k] >> t0) & 1u) {
                            const int q = fd.refl_dir[k];
                            const float xw = wrapped_coord(d, fd.L[q], p, q);
                            if (xw < fd.refl_lo[k] || xw > fd.refl_hi[k]) {
                                add_axis(p, q, 2.0f * ((xw < fd.refl_lo[k] ? fd.refl_lo[k] : fd.refl_hi[k]) - xw));
                                flip_axis(v, q);
                                moved = true;
                            }
                        }
                }
                if (moved) {
                    if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z) || !isfinite(v.x) ||
                        !isfinite(v.y) || !isfinite(v.z))
                        atomicOr(&a.rstate[r].status, ST_NONFINITE);
                    posp[s] = p;
                }
                if (check) {
                    bool need = d.skin_zero != 0;
                    if (!need) {
                        // same cell as at the last build: the displacement is the offset change
                        const float4 q = a.last4[s];
                        const float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
                        const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
                        need = !(r2 < d.hskin2);
                    }
                    if (need) {
                        const uint32_t ph = *a.phase + (a.mode == 1 ? 0u : 1u);
                        a.build_flag[ph & 1] = 1;
                    }
                }
                a.force4[s] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (d.style == 1) a.rho[s] = 0.0f;
            }
            velp[s] = v;
        }
    }
    // `log` is warp-uniform (a warp holds one replica): a warp-level flush, no barrier
    if (a.mode == 0 && log) {
        const int fields[10] = {ACC_KE, ACC_KIN + 0, ACC_KIN + 1, ACC_KIN + 2, ACC_KIN + 3,
                                ACC_KIN + 4, ACC_KIN + 5, ACC_MOM + 0, ACC_MOM + 1, ACC_MOM + 2};
        if (keep) keep->add(accv, r, fields, a.acc);
        else acc_flush_warp<10>(accv, fields, r, a.acc);
    }
    if (EXT && LOGM != 0 && gcd) {
        int fields[3 * DPD_MAX_GC];
#pragma unroll
        for (int k = 0; k < 3 * DPD_MAX_GC; k++) fields[k] = ACC_GC + k;
        acc_flush_warp<3 * DPD_MAX_GC>(gv, fields, r, a.acc);
    }
}

template <bool EXT>
__global__ void __launch_bounds__(256) k_integrate(StepArgs a)
{
    griddep_wait();
    integrate_slot<2, EXT>(a, blockIdx.x * blockDim.x + threadIdx.x);
}

template <bool EXT>
__global__ void __launch_bounds__(256) k_integrate_nolog(StepArgs a)
{
    griddep_wait();
    integrate_slot<0, EXT>(a, blockIdx.x * blockDim.x + threadIdx.x);
}

// logged steps: a small grid-stride launch that returns at once when no replica logs
// (thermo or a group compute due)
template <bool EXT>
__global__ void __launch_bounds__(256) k_integrate_logsteps(StepArgs a)
{
    griddep_wait();
    int any = 0;
    for (int r = threadIdx.x; r < a.nrep; r += blockDim.x) {
        const RepState st = a.rstate[r];
        if (!rep_active(st)) continue;
        any |= (st.step % (uint32_t)a.reps[r].log_f) == 0u;
        if (EXT && a.reps[r].gc_n) any |= gc_due(a, a.reps[r], st, r);
    }
    if (!__syncthreads_or(any)) return;
    const int nvb = (a.P + 255) / 256;
    // the warp's sums over its virtual blocks, flushed once per replica
    WarpAcc<10> keep;
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) integrate_slot<1, EXT>(a, vb * 256 + threadIdx.x, &keep);
    const int fields[10] = {ACC_KE, ACC_KIN + 0, ACC_KIN + 1, ACC_KIN + 2, ACC_KIN + 3,
                            ACC_KIN + 4, ACC_KIN + 5, ACC_MOM + 0, ACC_MOM + 1, ACC_MOM + 2};
    keep.flush(fields, a.acc);
}

// ---------------------------------------------------------------------------------
// Wall extents: the maximum position of a lo-wall group and the minimum of a hi-wall
// group along the wall axis (src/fix/fix_two_wall.cu:145-180 and
// src/compute/compute_wall_contact.cu:186-225 take them with thrust max/min_element).
// PH 0: the two_wall groups, after the drift; PH 1: the wall groups of wall_contact
// computes due this step, before the integrate (the end-of-step positions).
template <int PH>
__global__ void k_wall_reset(StepArgs a)
{
    griddep_wait();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nrep) return;
    int* e = a.wall_ext + r * 8;
    if (PH == 0) {
        for (int k = 0; k < 2; k++) {
            e[2 * k] = ford(-INFINITY);
            e[2 * k + 1] = ford(INFINITY);
        }
    } else {
        for (int k = 0; k < DPD_MAX_GC; k++) {
            const bool lo = !a.gc || a.gc[r * DPD_MAX_GC + k].wall_side > 0;
            e[4 + k] = ford(lo ? -INFINITY : INFINITY);
        }
    }
}

template <int PH>
__global__ void __launch_bounds__(256) k_wall_extent(StepArgs a)
{
    griddep_wait();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.P) return;  // warp-uniform
    const int r = a.warp_rep[s >> 5];
    const RepState st = a.rstate[r];
    if (!rep_active(st)) return;
    const RepDesc& d = a.reps[r];
    const int lane = threadIdx.x & 31;
    const int par = *a.parity;
    const bool real = s < d.p_end;
    float4 p = make_float4(0, 0, 0, 0);
    int t0 = 0;
    if (real) {
        p = a.buf.pos[par][s];
        t0 = type0_of(a.buf.vel[par][s].w);
    }
    if (PH == 0) {
        if (!a.fix) return;
        const FixDesc& fd = a.fix[r];
        for (int k = 0; k < fd.n_twowall; k++) {
            const int q = fd.tw_dir[k];
            const bool inlo = real && ((fd.tw_lo[k] >> t0) & 1u), inhi = real && ((fd.tw_hi[k] >> t0) & 1u);
            const float xw = (inlo || inhi) ? wrapped_coord(d, fd.L[q], p, q) : 0.0f;
            const int mx = __reduce_max_sync(0xffffffffu, inlo ? ford(xw) : INT_MIN);
            const int mn = __reduce_min_sync(0xffffffffu, inhi ? ford(xw) : INT_MAX);
            if (lane == 0) {
                if (mx != INT_MIN) atomicMax(&a.wall_ext[r * 8 + 2 * k], mx);
                if (mn != INT_MAX) atomicMin(&a.wall_ext[r * 8 + 2 * k + 1], mn);
            }
        }
    } else {
        if (!a.gc || a.mode != 0 || !d.gc_n) return;
        const int due = gc_due(a, d, st, r);
        for (int k = 0; k < d.gc_n; k++) {
            const GCDesc& g = a.gc[r * DPD_MAX_GC + k];
            if (g.kind != 5 || !((due >> k) & 1)) continue;
            const bool in = real && ((g.wall_mask >> t0) & 1u);
            const float xw = in ? wrapped_coord(d, g.L[g.wall_dir], p, g.wall_dir) : 0.0f;
            if (g.wall_side > 0) {
                const int mx = __reduce_max_sync(0xffffffffu, in ? ford(xw) : INT_MIN);
                if (lane == 0 && mx != INT_MIN) atomicMax(&a.wall_ext[r * 8 + 4 + k], mx);
            } else {
                const int mn = __reduce_min_sync(0xffffffffu, in ? ford(xw) : INT_MAX);
                if (lane == 0 && mn != INT_MAX) atomicMin(&a.wall_ext[r * 8 + 4 + k], mn);
            }
        }
    }
}

// fix two_wall, post_integrate (src/fix/fix_two_wall.cu:84-125, 183-200): group atoms
// below the lo wall's maximum or above the hi wall's minimum are mirrored back with the
// normal velocity reversed; then the list-rebuild check of the moved atoms.
__global__ void __launch_bounds__(256) k_two_wall(StepArgs a)
{
    griddep_wait();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.P || !a.fix) return;
    const int r = a.warp_rep[s >> 5];
    const RepState st = a.rstate[r];
    const RepDesc& d = a.reps[r];
    if (!rep_active(st) || s >= d.p_end) return;
    const bool init = a.mode == 1 ? true : st.step < st.target;
    if (!init) return;  // no drift this launch: nothing to correct
    const FixDesc& fd = a.fix[r];
    if (!fd.n_twowall) return;
    const int par = *a.parity;
    float4 p = a.buf.pos[par][s];
    float4 v = a.buf.vel[par][s];
    const int t0 = type0_of(v.w);
    bool moved = false;
    for (int k = 0; k < fd.n_twowall; k++) {
        if (!((fd.tw_mask[k] >> t0) & 1u)) continue;
        const float lo = ford_inv(a.wall_ext[r * 8 + 2 * k]), hi = ford_inv(a.wall_ext[r * 8 + 2 * k + 1]);
        if (hi <= lo) atomicOr(&a.rstate[r].status, ST_WALL_ORDER);
        const int q = fd.tw_dir[k];
        const float xw = wrapped_coord(d, fd.L[q], p, q);
        if (xw < lo || xw > hi) {
            add_axis(p, q, 2.0f * ((xw < lo ? lo : hi) - xw));
            flip_axis(v, q);
            moved = true;
        }
    }
    if (!moved) return;
    a.buf.pos[par][s] = p;
    a.buf.vel[par][s] = v;
    const uint32_t next = a.mode == 1 ? st.step : st.step + 1u;
    if ((next % (uint32_t)d.nl_f) == 0u && !d.skin_zero) {
        const float4 q = a.last4[s];
        const float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
        if (!(__fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx))) < d.hskin2)) {
            const uint32_t ph = *a.phase + (a.mode == 1 ? 0u : 1u);
            a.build_flag[ph & 1] = 1;
        }
    }
}

// ---------------------------------------------------------------------------------
// Group fixes.  Sums over a group are warp-reduced into the spread FP64 accumulators
// (fields ACC_SPRING_COM, ACC_RVCM_P, ACC_RECENTER_COM) and reduced per replica by
// k_fix_reduce of the same phase, which zeroes them again.  Unwrapped positions are
// lo + c w + o + img L (the reference keeps them as uwpos, src/system/system.cuh:14).
//  PH 0 (every step, replicas with a spring): sum m x over the spring group, from the
//       positions the forces of this step were evaluated at (src/fix/fix_spring.cu:281-300).
//  PH 1 (replicas with an rvcm or recenter due this step): the final half kick (with the
//       spring share), then sum m v over the rvcm group (src/fix/fix_rvcm.cu:233-262) and
//       m x over the recenter group (src/fix/fix_recenter.cu:270-300).
__device__ __forceinline__ double unwrapped(const RepDesc& d, const FixDesc& fd, int code, float o,
                                            int img, int k)
{
    const int c = (code >> (k * DPD_CELL_BITS)) & DPD_MAX_NC;
    return d.lo[k] + (double)c * (double)d.w[k] + (double)o + (double)img * fd.L[k];
}

template <int PH>
__global__ void __launch_bounds__(256) k_fix_sums(StepArgs a)
{
    griddep_wait();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.P) return;  // P is a multiple of 32: warp-uniform
    const int r = a.warp_rep[s >> 5];
    const RepState st = a.rstate[r];
    const FixDesc& fd = a.fix[r];
    int eos = 0;
    if (PH == 0) {
        if (!rep_active(st) || !fd.spring_mask) return;
    } else {
        eos = fix_eos_due(fd, st, a.mode);
        if (!eos) return;
    }
    const RepDesc& d = a.reps[r];
    double accv[6] = {0, 0, 0, 0, 0, 0};
    if (s < d.p_end) {
        const int par = *a.parity;
        float4 v = a.buf.vel[par][s];
        const int t0 = type0_of(v.w);
        const float2 m = __ldg(a.mass + d.mass_off + t0);
        if (PH == 1) {
            if ((d.integ_mask >> t0) & 1u) {
                float4 f = a.force4[s];
                if ((fd.spring_mask >> t0) & 1u) {
                    const FixOut& fo = a.fixo[r];
                    f.x = __fmaf_rn(fo.spring_a[0], m.x, f.x);
                    f.y = __fmaf_rn(fo.spring_a[1], m.x, f.y);
                    f.z = __fmaf_rn(fo.spring_a[2], m.x, f.z);
                }
                const float dtm = (0.5f * d.dt) * m.y;
                v.x = __fmaf_rn(dtm, f.x, v.x);
                v.y = __fmaf_rn(dtm, f.y, v.y);
                v.z = __fmaf_rn(dtm, f.z, v.z);
                a.buf.vel[par][s] = v;
            }
            if ((eos & 1) && ((fd.rvcm_mask >> t0) & 1u)) {
                accv[0] = (double)m.x * v.x;
                accv[1] = (double)m.x * v.y;
                accv[2] = (double)m.x * v.z;
            }
        }
        const uint32_t gm = PH == 0 ? fd.spring_mask : ((eos & 2) ? fd.recenter_mask : 0u);
        if ((gm >> t0) & 1u) {
            const float4 p = a.buf.pos[par][s];
            const int4 im = a.buf.img[d.tag_base + tag_of(v.w) - 1];
            const int code = __float_as_int(p.w);
            const int base = PH == 0 ? 0 : 3;
            accv[base + 0] = (double)m.x * unwrapped(d, fd, code, p.x, im.x, 0);
            accv[base + 1] = (double)m.x * unwrapped(d, fd, code, p.y, im.y, 1);
            accv[base + 2] = (double)m.x * unwrapped(d, fd, code, p.z, im.z, 2);
        }
    }
    if (PH == 0) {
        double v3[3] = {accv[0], accv[1], accv[2]};
        const int fields[3] = {ACC_SPRING_COM + 0, ACC_SPRING_COM + 1, ACC_SPRING_COM + 2};
        acc_flush_warp<3>(v3, fields, r, a.acc);
    } else {
        const int fields[6] = {ACC_RVCM_P + 0, ACC_RVCM_P + 1, ACC_RVCM_P + 2,
                               ACC_RECENTER_COM + 0, ACC_RECENTER_COM + 1, ACC_RECENTER_COM + 2};
        acc_flush_warp<6>(accv, fields, r, a.acc);
    }
}

// sum and zero three fields of a replica's spread accumulators
__device__ __forceinline__ void acc_take3(double* acc, int r, int field, double out[3])
{
    double* base = acc + (size_t)r * DPD_ACC_SLOTS * DPD_NACC;
    out[0] = out[1] = out[2] = 0.0;
    for (int sl = 0; sl < DPD_ACC_SLOTS; sl++)
        for (int k = 0; k < 3; k++) {
            out[k] += base[sl * DPD_NACC + field + k];
            base[sl * DPD_NACC + field + k] = 0.0;
        }
}

// One thread per replica.  PH 0: the spring force F = -k (r - r0) d / r, d = com - c,
// when r > 1e-10 (src/fix/fix_spring.cu:300-340), kept as F / M, and the spring record
// {step, Fx, Fy, Fz, +-|F|, k (r - r0)^2 / 2} of file steps.  PH 1: flag * vcm of a due
// rvcm (src/fix/fix_rvcm.cu:262-286) and target - com of a due recenter
// (src/fix/fix_recenter.cu:300-335).
template <int PH>
__global__ void k_fix_reduce(StepArgs a)
{
    griddep_wait();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nrep) return;
    const RepState st = a.rstate[r];
    const FixDesc& fd = a.fix[r];
    FixOut& fo = a.fixo[r];
    if (PH == 0) {
        if (!rep_active(st) || !fd.spring_mask) return;
        double sum[3];
        acc_take3(a.acc, r, ACC_SPRING_COM, sum);
        double dv[3], r2 = 0.0;
        for (int k = 0; k < 3; k++) {
            dv[k] = (fd.spring_m > 0.0 ? sum[k] / fd.spring_m : 0.0) - fd.spring_c[k];
            r2 += dv[k] * dv[k];
        }
        const double rr = sqrt(r2), dr = rr - fd.spring_r0;
        double F[3] = {0.0, 0.0, 0.0}, fm = 0.0, e = 0.0;
        if (rr > 1.0e-10 && fd.spring_m > 0.0) {
            for (int k = 0; k < 3; k++) F[k] = -fd.spring_k * dr * dv[k] / rr;
            fm = sqrt(F[0] * F[0] + F[1] * F[1] + F[2] * F[2]);
            if (dr < 0.0) fm = -fm;
            e = 0.5 * fd.spring_k * dr * dr;
        }
        for (int k = 0; k < 3; k++) fo.spring_a[k] = fd.spring_m > 0.0 ? (float)(F[k] / fd.spring_m) : 0.0f;
        if (a.spring_ring && fd.spring_file_f && (st.step % fd.spring_file_f) == 0u) {
            double* row = a.spring_ring + ((size_t)r * DPD_RING_ROWS + (fo.nrec % DPD_RING_ROWS)) * 6;
            row[0] = (double)st.step;
            row[1] = F[0];
            row[2] = F[1];
            row[3] = F[2];
            row[4] = fm;
            row[5] = e;
            fo.nrec++;
        }
    } else {
        const int eos = fix_eos_due(fd, st, a.mode);
        if (!eos) return;
        if (eos & 1) {
            double P[3];
            acc_take3(a.acc, r, ACC_RVCM_P, P);
            for (int k = 0; k < 3; k++)
                fo.vcm[k] = fd.rvcm_flag[k] && fd.rvcm_m > 0.0 ? (float)(P[k] / fd.rvcm_m) : 0.0f;
        }
        if (eos & 2) {
            double c[3];
            acc_take3(a.acc, r, ACC_RECENTER_COM, c);
            for (int k = 0; k < 3; k++)
                fo.shift[k] = fd.recenter_m > 0.0 ? (float)(fd.recenter_c[k] - c[k] / fd.recenter_m) : 0.0f;
        }
    }
}

// ---------------------------------------------------------------------------------
// Harmonic angles, src/force/angle_harmonic.cu:187-270, one thread per angle, after the
// pair kernel: d1 = x_i - x_j, d2 = x_k - x_j (j the apex), c = cos(theta) clamped to
// [-1, 1], s = sin(theta) >= 0.001, E = k (theta - theta0)^2, a = -2 k dtheta / s,
// F_i = a c/|d1|^2 d1 - a/(|d1||d2|) d2, F_k likewise, F_j = -(F_i + F_k), added with
// float4 reductions.  The table is in global tag indices (it never moves); each
// replica's range is padded to whole warps (entries with coef < 0 are padding), so a
// warp's FP64 sums belong to one replica.
// a*b - c*d with about one rounding (Kahan's form with fma): the cross product of two
// nearly parallel vectors without cancellation
__device__ __forceinline__ float diff_of_products(float a, float b, float c, float d)
{
    const float w = c * d;
    const float e = __fmaf_rn(-c, d, w);
    const float f = __fmaf_rn(a, b, -w);
    return f + e;
}

__global__ void __launch_bounds__(256) k_angle(StepArgs a, const int4* __restrict__ tbl,
                                               const float4* __restrict__ coef, const int* awarp_rep, int nang)
{
    griddep_wait();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if ((q & ~31) >= nang) return;  // nang is a multiple of 32
    const int r = awarp_rep[q >> 5];
    const RepState st = a.rstate[r];
    if (!rep_active(st)) return;  // warp-uniform
    const RepDesc& d = a.reps[r];
    const bool log = (st.step % (uint32_t)d.log_f) == 0u;
    double accv[7] = {0, 0, 0, 0, 0, 0, 0};
    const int4 e = tbl[q];
    if (e.x >= 0) {
        const int i = a.tag2idx[e.y], j = a.tag2idx[e.z], k = a.tag2idx[e.w];
        if (i < d.p_begin || i >= d.p_end || j < d.p_begin || j >= d.p_end || k < d.p_begin || k >= d.p_end) {
            atomicOr(&a.rstate[r].status, ST_BOND_MISSING);
        } else {
            const float4* pos = a.buf.pos[*a.parity];
            const float4 pi = pos[i], pj = pos[j], pk = pos[k];
            float d1x, d1y, d1z, d2x, d2y, d2z;
            disp3(d, __float_as_int(pi.w), pi, pj, d1x, d1y, d1z);
            disp3(d, __float_as_int(pk.w), pk, pj, d2x, d2y, d2z);
            const float rsq1 = d1x * d1x + d1y * d1y + d1z * d1z;
            const float rsq2 = d2x * d2x + d2y * d2y + d2z * d2z;
            const float r1 = sqrtf(rsq1), r2 = sqrtf(rsq2), r12 = r1 * r2;
            float c = (d1x * d2x + d1y * d2y + d1z * d2z) / r12;
            c = fminf(fmaxf(c, -1.0f), 1.0f);
            // The reference's harmonic angle (src/force/angle_harmonic.cu), kept accurate in
            // FP32 near straight triples: sin(theta) from the cross product rather than
            // sqrt(1 - c^2), and theta - theta0 as atan2 of its sine and cosine (cos and sin
            // of theta0 precomputed in double) rather than acos(c) - theta0, which near
            // c = -1 resolves the angle only to about 3e-4 rad
            const float cpx = diff_of_products(d1y, d2z, d1z, d2y);
            const float cpy = diff_of_products(d1z, d2x, d1x, d2z);
            const float cpz = diff_of_products(d1x, d2y, d1y, d2x);
            const float st = sqrtf(cpx * cpx + cpy * cpy + cpz * cpz) / r12;
            const float sn = fmaxf(st, 0.001f);
            const float4 kc = coef[e.x];  // {k, theta0 in radians, cos theta0, sin theta0}
            const float dth = atan2f(st * kc.z - c * kc.w, c * kc.z + st * kc.w);
            const float aa = -2.0f * kc.x * dth / sn;
            const float a11 = aa * c / rsq1, a12 = -aa / (r1 * r2), a22 = aa * c / rsq2;
            const float fix = a11 * d1x + a12 * d2x, fiy = a11 * d1y + a12 * d2y, fiz = a11 * d1z + a12 * d2z;
            const float fkx = a22 * d2x + a12 * d1x, fky = a22 * d2y + a12 * d1y, fkz = a22 * d2z + a12 * d1z;
            atomicAdd(&a.force4[i], make_float4(fix, fiy, fiz, 0.0f));
            atomicAdd(&a.force4[k], make_float4(fkx, fky, fkz, 0.0f));
            atomicAdd(&a.force4[j], make_float4(-(fix + fkx), -(fiy + fky), -(fiz + fkz), 0.0f));
            if (log) {
                accv[0] = (double)kc.x * (double)dth * (double)dth;
                accv[1] = (double)d1x * fix + (double)d2x * fkx;
                accv[2] = (double)d1x * fiy + (double)d2x * fky;
                accv[3] = (double)d1x * fiz + (double)d2x * fkz;
                accv[4] = (double)d1y * fiy + (double)d2y * fky;
                accv[5] = (double)d1y * fiz + (double)d2y * fkz;
                accv[6] = (double)d1z * fiz + (double)d2z * fkz;
            }
        }
    }
    if (log) {
        const int fields[7] = {ACC_ANGLE_PE, ACC_VIR + 0, ACC_VIR + 1, ACC_VIR + 2,
                               ACC_VIR + 3, ACC_VIR + 4, ACC_VIR + 5};
        acc_flush_warp<7>(accv, fields, r, a.acc);
    }
}

// ---------------------------------------------------------------------------------
// End of step bookkeeping, one thread per replica: thermo row of a logged step
// (src/compute/thermo.cu:274-306, 479-520), step counter, build flag of this phase.
// The step's bookkeeping of replica r by one warp (lane = spread slot: DPD_ACC_SLOTS is
// 32): on a logged step the lanes take the 32 spread slots of the thermo sums and a fixed
// butterfly adds them (the row then repeats bit for bit); lane 0 writes the thermo row and
// does the rest.
static_assert(DPD_ACC_SLOTS == 32, "advance_rep gives each lane of a warp one spread slot");
__device__ __forceinline__ void advance_rep(const StepArgs& a, const int r, const int lane)
{
    {
        RepState st = a.rstate[r];
        const RepDesc& d = a.reps[r];
        if (rep_active(st)) {
            if ((st.step % (uint32_t)d.log_f) == 0u) {
                double sum[DPD_NACC_THERMO];
                double* base = a.acc + (size_t)r * DPD_ACC_SLOTS * DPD_NACC + (size_t)lane * DPD_NACC;
#pragma unroll
                for (int k = 0; k < DPD_NACC_THERMO; k++) sum[k] = base[k];
#pragma unroll
                for (int k = 0; k < DPD_NACC_THERMO; k++) base[k] = 0.0;
#pragma unroll
                for (int k = 0; k < DPD_NACC_THERMO; k++)
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) sum[k] += __shfl_xor_sync(0xffffffffu, sum[k], o);
                if (lane != 0) return;
                double* row = a.ring + ((size_t)r * DPD_RING_ROWS + (st.nlog % DPD_RING_ROWS)) *
                                           DPD_THERMO_FIELDS;
                const double vol = d.volume;
                const double ndof = 3.0 * d.n_real - 3.0;
                row[0] = (double)st.step;
                row[1] = ndof > 0 ? 2.0 * sum[ACC_KE] / ndof : 0.0;
                row[2] = sum[ACC_PAIR_PE];
                row[3] = sum[ACC_BOND_PE];
                for (int c = 0; c < 6; c++) row[5 + c] = (sum[ACC_KIN + c] + sum[ACC_VIR + c]) / vol;
                row[4] = (row[5] + row[8] + row[10]) / 3.0;
                row[11] = sum[ACC_KE];
                row[12] = sum[ACC_MOM + 0];
                row[13] = sum[ACC_MOM + 1];
                row[14] = sum[ACC_MOM + 2];
                row[15] = (double)st.status;
                row[16] = sum[ACC_ANGLE_PE];
                st.nlog++;
            }
            if (lane != 0) return;
            if (a.gc && d.gc_n) {
                const int due = gc_due(a, d, st, r);
                double* base = a.acc + (size_t)r * DPD_ACC_SLOTS * DPD_NACC;
                for (int k = 0; k < d.gc_n; k++) {
                    if (!((due >> k) & 1)) continue;
                    const GCDesc& g = a.gc[r * DPD_MAX_GC + k];
                    double s3[3] = {0.0, 0.0, 0.0};
                    for (int sl = 0; sl < DPD_ACC_SLOTS; sl++)
                        for (int q = 0; q < 3; q++) {
                            s3[q] += base[sl * DPD_NACC + ACC_GC + 3 * k + q];
                            base[sl * DPD_NACC + ACC_GC + 3 * k + q] = 0.0;
                        }
                    double* row = a.gc_ring + ((size_t)g.ring * DPD_RING_ROWS + (a.gc_count[g.ring] % DPD_RING_ROWS)) * 4;
                    row[0] = (double)st.step;
                    if (g.kind == 4) {
                        row[1] = s3[0];
                        row[2] = s3[1];
                        row[3] = s3[2];
                    } else {
                        row[1] = (g.kind == 1 ? 2.0 : 1.0) * s3[0] * g.norm;
                        row[2] = row[3] = 0.0;
                    }
                    a.gc_count[g.ring]++;
                }
            }
            st.step++;
            st.zero_pending = 0;
            a.rstate[r] = st;
        }
    }
}

// the step's phase: this phase's build flag cleared, the phase counter advanced
__device__ __forceinline__ void advance_phase(const StepArgs& a)
{
    const uint32_t ph = *a.phase;
    a.build_flag[ph & 1] = 0;
    *a.phase = ph + 1u;
}

// a warp per replica
__global__ void k_advance(StepArgs a)
{
    griddep_wait();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = g >> 5;
    if (r < a.nrep) advance_rep(a, r, threadIdx.x & 31);
    if (g == 0) advance_phase(a);
}

// Small grids, where a launch costs more than the work: the whole velocity-Verlet step
// (any step, logged or not) in one launch whose last block (a ticket counter) also does
// the step's bookkeeping of every replica.  Every block's writes and FP64 sums are done
// and fenced before it takes its ticket.
template <bool EXT>
__global__ void __launch_bounds__(256) k_integrate_adv(StepArgs a)
{
    griddep_wait();
    integrate_slot<2, EXT>(a, blockIdx.x * blockDim.x + threadIdx.x);
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(a.ticket, 1u) == gridDim.x - 1u;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int r = threadIdx.x >> 5; r < a.nrep; r += blockDim.x >> 5) advance_rep(a, r, threadIdx.x & 31);
    __syncthreads();
    if (threadIdx.x == 0) {
        advance_phase(a);
        *a.ticket = 0u;
    }
}

// ---------------------------------------------------------------------------------
// RDF sampling (new; no reference counterpart): histogram of minimum-image distances
// from particles of type ta to particles of type tb within rmax, sampled on steps that
// are multiples of rdf_every, from the end-of-step positions.  Candidate cells are the
// last build's cells within reach of the particle: rmax with a build this step (skin 0,
// nl_f 1: the sample sees the build's positions); rmax + skin when the displacement check
// runs every step (nl_f 1: no particle has moved skin/2 since the build); otherwise one
// more layer of cells.  In the first two cases cells farther than rmax (+ skin/2 for the
// candidate's drift) from the particle itself are skipped.  A warp takes its 32 slots one after the other; for each type-ta particle the
// lanes share out the stencil's cells (one cell per lane and turn), so the lanes stay busy
// whatever the cell sizes.  Each warp keeps its histogram and its stencil (the cell
// offsets, packed, when there are at most DPD_RDF_MAXCELLS) in shared memory.
#define DPD_RDF_MAXBINS 512
#define DPD_RDF_MAXCELLS 512
__global__ void __launch_bounds__(256) k_rdf(StepArgs a)
{
    griddep_wait();
    __shared__ unsigned int hs[8][DPD_RDF_MAXBINS];
    __shared__ int stab[8][DPD_RDF_MAXCELLS];
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if ((s & ~31) >= a.P) return;  // warp-uniform
    const int r = a.warp_rep[s >> 5];
    const RepDesc& d = a.reps[r];
    const RepState st = a.rstate[r];
    if (!(d.rdf_every > 0 && rep_active(st) && (st.step % (uint32_t)d.rdf_every) == 0u)) return;  // warp-uniform
    const int par = *a.parity;
    const float4* pos = a.buf.pos[par];
    const float4* vel = a.buf.vel[par];
    const int nb = min(d.rdf_nbins, DPD_RDF_MAXBINS);
    for (int b = lane; b < nb; b += 32) hs[warp][b] = 0u;
    __syncwarp();
    if (s == d.p_begin) atomicAdd((unsigned long long*)&a.rstate[r].rdf_samples, 1ull);
    const float rmax2 = d.rdf_rmax * d.rdf_rmax;
    const float inv_dr = (float)d.rdf_nbins / d.rdf_rmax;
    int lo3[3], n3[3];
    const bool fresh = d.skin_zero && d.nl_f == 1;
    const bool bounded = !d.skin_zero && d.nl_f == 1;
    const float hskin = bounded ? sqrtf(d.hskin2) : 0.0f;  // the drift bound, skin/2
    bool local = true;  // the searched cells are nearer than half the grid in every axis
    for (int k = 0; k < 3; k++) {
        // 1e-6: a ratio rounded down to an integer still covers the last layer
        const int nr = fresh || bounded ? (int)ceilf((d.rdf_rmax + 2.0f * hskin) * d.inv_w[k] * 1.000001f)
                                        : (int)ceilf(d.rdf_rmax * d.inv_w[k] * 1.000001f) + 1;
        if (2 * nr + 1 >= d.nc[k]) {
            lo3[k] = -(d.nc[k] / 2);
            n3[k] = d.nc[k];
            local = false;
        } else {
            lo3[k] = -nr;
            n3[k] = 2 * nr + 1;
        }
    }
    const bool prune = (fresh || bounded) && local;
    const float reach2 = (d.rdf_rmax + hskin) * (d.rdf_rmax + hskin);
    const int ncand = n3[0] * n3[1] * n3[2];
    const bool tabled = ncand <= DPD_RDF_MAXCELLS;
    // cell offset c of the stencil, packed as (ox+512) | (oy+512)<<10 | (oz+512)<<20
    auto decode = [&](int c) {
        return (lo3[0] + c / (n3[1] * n3[2]) + 512) | ((lo3[1] + (c / n3[2]) % n3[1] + 512) << 10) |
               ((lo3[2] + c % n3[2] + 512) << 20);
    };
    if (tabled)
        for (int c = lane; c < ncand; c += 32) stab[warp][c] = decode(c);
    __syncwarp();
    const int w0 = s & ~31;
    for (int q = 0; q < 32; q++) {
        const int si = w0 + q;
        if (si >= d.p_end) break;  // warp-uniform
        const float4 vi = vel[si];
        if (type0_of(vi.w) + 1 != d.rdf_ta) continue;  // warp-uniform
        const float4 pi = pos[si];
        const int ci = __float_as_int(pi.w);
        const int cx = cell_x(ci), cy = cell_y(ci), cz = cell_z(ci);
        // the stencil in chunks of 32 cells, one per lane; the chunk's candidates are
        // shared out over the lanes as one flat sequence (owner cell by a binary search
        // over the lanes' scanned counts)
        for (int c0 = 0; c0 < ncand; c0 += 32) {
            const int c = c0 + lane;
            int beg = 0, cnt = 0;
            float sx = 0.0f, sy = 0.0f, sz = 0.0f;
            if (c < ncand) {
                const int pk = tabled ? stab[warp][c] : decode(c);
                const int ox = (pk & 1023) - 512, oy = ((pk >> 10) & 1023) - 512, oz = ((pk >> 20) & 1023) - 512;
                bool keep = true;
                if (prune) {
                    // distance from the particle to the near face of that cell
                    const float gx = ox > 0 ? (float)ox * d.w[0] - pi.x : (ox < 0 ? pi.x - (float)(ox + 1) * d.w[0] : 0.0f);
                    const float gy = oy > 0 ? (float)oy * d.w[1] - pi.y : (oy < 0 ? pi.y - (float)(oy + 1) * d.w[1] : 0.0f);
                    const float gz = oz > 0 ? (float)oz * d.w[2] - pi.z : (oz < 0 ? pi.z - (float)(oz + 1) * d.w[2] : 0.0f);
                    keep = gx * gx + gy * gy + gz * gz < reach2;
                }
                if (keep) {
                    // |offset| < nc: one wrap at most
                    int nx = cx + ox; nx += nx < 0 ? d.nc[0] : 0; nx -= nx >= d.nc[0] ? d.nc[0] : 0;
                    int ny = cy + oy; ny += ny < 0 ? d.nc[1] : 0; ny -= ny >= d.nc[1] ? d.nc[1] : 0;
                    int nz = cz + oz; nz += nz < 0 ? d.nc[2] : 0; nz -= nz >= d.nc[2] ? d.nc[2] : 0;
                    const int key = d.c_begin + a.crank[d.c_begin + (nx * d.nc[1] + ny) * d.nc[2] + nz];
                    beg = a.cstart[key];
                    cnt = a.cstart[key + 1] - beg;
                    sx = __int2float_rn(-ox) * d.w[0];
                    sy = __int2float_rn(-oy) * d.w[1];
                    sz = __int2float_rn(-oz) * d.w[2];
                }
            }
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            const int start = incl - cnt;
            for (int t0 = 0; t0 < total; t0 += 32) {
                const int t = t0 + lane;
                int l = 0;  // the last lane whose start is <= t
#pragma unroll
                for (int stp = 16; stp >= 1; stp >>= 1) {
                    const int sv = __shfl_sync(0xffffffffu, start, l + stp);
                    if (sv <= t) l += stp;
                }
                const int j = __shfl_sync(0xffffffffu, beg, l) + (t - __shfl_sync(0xffffffffu, start, l));
                const float hx = __shfl_sync(0xffffffffu, sx, l), hy = __shfl_sync(0xffffffffu, sy, l),
                            hz = __shfl_sync(0xffffffffu, sz, l);
                if (t < total && j != si) {
                    const float4 pj = __ldg(pos + j);
                    float dx, dy, dz;
                    if (local) {
                        // (o_i - o_j) + (c_i - c_j) w with c_j = c_i + offset: the nearest
                        // image for every pair this search can reach
                        dx = __fadd_rn(__fsub_rn(pi.x, pj.x), hx);
                        dy = __fadd_rn(__fsub_rn(pi.y, pj.y), hy);
                        dz = __fadd_rn(__fsub_rn(pi.z, pj.z), hz);
                    } else {
                        disp3(d, ci, pi, pj, dx, dy, dz);
                    }
                    const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
                    if (r2 < rmax2 && type0_of(__ldg(&vel[j].w)) + 1 == d.rdf_tb) {
                        const int bin = (int)(sqrtf(r2) * inv_dr);
                        if (bin < nb) atomicAdd(&hs[warp][bin], 1u);
                    }
                }
            }
        }
    }
    __syncwarp();
    unsigned long long* hist = a.rdf_hist + d.rdf_off;
    for (int b = lane; b < nb; b += 32) {
        const unsigned int c = hs[warp][b];
        if (c) atomicAdd(hist + b, (unsigned long long)c);
    }
}
