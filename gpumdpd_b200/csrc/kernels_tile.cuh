// kernels_tile.cuh -- DPD pair forces straight from the cell ranges of the counting sort,
// with no neighbour list: the list build and the list-driven pair pass as one kernel.
//
// A CTA takes a tile of home cells (T x T x T, fewer at the grid's edge) of one replica
// and stages the particles of the cells its half stencil reaches -- x in [x0-1, x0+T],
// y in [y0-1, y0+T], z in [z0, z0+T] -- into shared memory, cell by cell with x fastest,
// so that the 13 forward cells of a home cell plus the rest of its own cell form five
// contiguous ranges of staged particles:
//   R0: own cell after i, then cell (x+1, y, z)        (offsets 0 and (1,0,0))
//   R1: cells (x-1..x+1, y+1, z)                       (the row dz = 0, dy = +1)
//   R2..R4: cells (x-1..x+1, y-1..y+1, z+1)             (the three rows dz = +1)
// -- the half stencil of src/force/neigh_list.cu:322-393 (every unordered cell pair
// once; at least 3 cells per dimension).  Its warps take home cells one at a time
// (a shared counter hands them out): the lanes take the home cell's candidates j, 32 at
// a time, and each lane tests its j against every particle i of the home cell in turn
// (i broadcast from shared memory), with the list predicate of the list build:
//   d = (o_i - o_j) + (c_i - c_j) w,  r2 = fma(dz,dz, fma(dy,dy, dx*dx)) <= rc_max^2,
// so the pairs evaluated are exactly the list path's.  Pairs inside the cutoff go to a
// per-warp ring queue; whenever 32 are pending, the lanes evaluate them together (Saru
// random force, src/force/pair_dpd.cu:468-558), each with the float4 reductions of both
// sides into the force array.  The home particles' bonds follow (bond_loop).  Log steps
// add the FP64 energy and virial sums, flushed per warp.
//
// When a tile's neighbourhood holds more particles than the staging capacity (a local
// density far above the mean), the CTA takes its home cells one at a time with the
// smaller neighbourhood of one cell; only if that does not fit either is the replica's
// ST_LIST_OVERFLOW raised (the pairs of that cell are then missing, and the run fails
// with DPD_E_OVERFLOW).
#pragma once
#include "kernels_step.cuh"

#define TILE_MAX_EDGE 6
#define TILE_MAX_REGION ((TILE_MAX_EDGE + 2) * (TILE_MAX_EDGE + 2) * (TILE_MAX_EDGE + 1))
#define TILE_Q 64  // per-warp ring queue of pairs (power of two, >= 63)

struct TileArgs {
    const int* tile_rep;   // [ntiles] replica of each tile
    const int* tile_code;  // [ntiles] tile coordinates ix | iy << 10 | iz << 20
    int ntiles;
    int edge;              // home cells per tile edge
    int smax;              // staging capacity (particles) of a CTA
};

// dynamic shared memory of a CTA: staged positions, velocities, slots; region cell
// starts (+1) and global starts; per-warp pair queues
__host__ __device__ inline size_t tile_smem_bytes(int smax)
{
    return (size_t)smax * (16 + 16 + 4) + (size_t)(2 * TILE_MAX_REGION + 32) * 4 +
           (size_t)8 * TILE_Q * (16 + 4);
}

struct TileSmem {
    float4* pos;   // [smax] {o.x, o.y, o.z, region cell code rx | ry << 8 | rz << 16}
    float4* vel;   // [smax] as in the particle arrays (tag and type in .w)
    int* slot;     // [smax] particle slot
    int* rstart;   // [TILE_MAX_REGION + 16] first staged index of each region cell, the
                   // total after the last one; [TILE_MAX_REGION + 8 + w]: warp totals
    int* gstart;   // [TILE_MAX_REGION] first slot of each region cell
    float4* qd;    // [8][TILE_Q] {dx, dy, dz, r2} of a queued pair
    uint32_t* qij; // [8][TILE_Q] i | j << 16 (staged indices)
};

__device__ __forceinline__ TileSmem tile_smem(unsigned char* base, int smax)
{
    TileSmem t;
    t.pos = (float4*)base;
    t.vel = t.pos + smax;
    t.slot = (int*)(t.vel + smax);
    t.rstart = t.slot + smax;
    t.gstart = t.rstart + TILE_MAX_REGION + 16;
    t.qd = (float4*)(t.gstart + TILE_MAX_REGION + 16);
    t.qij = (uint32_t*)(t.qd + 8 * TILE_Q);
    return t;
}

// Evaluate `cnt` (<= 32) queued pairs from the warp's ring position `head`.
template <bool LOG>
__device__ __forceinline__ void tile_eval(const StepArgs& a, const RepDesc& d, const TileSmem& sm, int warp,
                                          int lane, uint32_t head, int cnt, uint32_t step, double (&accv)[8])
{
    if (lane < cnt) {
        const uint32_t e = (head + lane) & (TILE_Q - 1);
        const float4 dd = sm.qd[warp * TILE_Q + e];
        const uint32_t ij = sm.qij[warp * TILE_Q + e];
        const int i = ij & 0xffff, j = ij >> 16;
        const float4 vi = sm.vel[i], vj = sm.vel[j];
        const float4* crow = a.coeff + d.coeff_off + type0_of(vi.w) * d.ntypes * 3;
        float fx, fy, fz;
        if (pair_force<0, LOG>(crow, dd.w, dd.x, dd.y, dd.z, vi, vj, 0.0f, 0.0f, d.seed, step, fx, fy, fz, accv)) {
            atomicAdd(&a.force4[sm.slot[i]], make_float4(fx, fy, fz, 0.0f));
            atomicAdd(&a.force4[sm.slot[j]], make_float4(-fx, -fy, -fz, 0.0f));
        }
    }
    __syncwarp();
}

// Stage the neighbourhood of the home box [hx0, hx0+ex) x [hy0, hy0+ey) x [hz0, hz0+ez)
// (global cell coordinates) of replica r and evaluate its pairs and its home particles'
// bonds.  Returns false (having done nothing) when the neighbourhood does not fit the
// staging capacity.  Called by the whole CTA; begins and ends with a barrier.
template <bool LOG, bool BONDS>
__device__ bool tile_box(const StepArgs& a, const TileArgs& ta, const TileSmem& sm, const RepDesc& d, int r,
                         int hx0, int hy0, int hz0, int ex, int ey, int ez, uint32_t step, double (&accv)[8])
{
    __shared__ int s_total, s_next;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int RX = ex + 2, RY = ey + 2, RZ = ez + 1, NR = RX * RY * RZ;
    const int ncx = d.nc[0], ncy = d.nc[1], ncz = d.nc[2];
    __syncthreads();  // the previous box's shared data is no longer read
    // 1. cell ranges of the region, and their exclusive scan (two region cells a thread)
    int cnt2[2] = {0, 0};
#pragma unroll
    for (int u = 0; u < 2; u++) {
        const int c = 2 * tid + u;
        if (c < NR) {
            const int lx = c % RX, ly = (c / RX) % RY, lz = c / (RX * RY);
            int gx = hx0 - 1 + lx, gy = hy0 - 1 + ly, gz = hz0 + lz;
            gx += gx < 0 ? ncx : 0; gx -= gx >= ncx ? ncx : 0;
            gy += gy < 0 ? ncy : 0; gy -= gy >= ncy ? ncy : 0;
            gz -= gz >= ncz ? ncz : 0;
            const int key = d.c_begin + __ldg(a.crank + d.c_begin + (gx * ncy + gy) * ncz + gz);
            const int g0 = __ldg(a.cstart + key);
            sm.gstart[c] = g0;
            cnt2[u] = __ldg(a.cstart + key + 1) - g0;
        }
    }
    {
        const int tot = cnt2[0] + cnt2[1];
        int incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) sm.rstart[TILE_MAX_REGION + 8 + warp] = incl;  // warp totals
        __syncthreads();
        int base = 0;
        for (int w = 0; w < warp; w++) base += sm.rstart[TILE_MAX_REGION + 8 + w];
        const int ex0 = base + incl - tot;
        __syncthreads();  // totals read before rstart entries are written
        if (2 * tid < NR) sm.rstart[2 * tid] = ex0;
        if (2 * tid + 1 < NR) sm.rstart[2 * tid + 1] = ex0 + cnt2[0];
        if (tid == blockDim.x - 1) {
            s_total = base + incl;
            s_next = 0;
        }
    }
    __syncthreads();
    const int S = s_total;
    if (S > ta.smax) return false;  // CTA-uniform
    if (tid == 0) sm.rstart[NR] = S;
    // 2. stage the region's particles, a thread per region cell
    {
        const int par = *a.parity;
        const float4* pos = a.buf.pos[par];
        const float4* vel = a.buf.vel[par];
        for (int c = tid; c < NR; c += blockDim.x) {
            const int lx = c % RX, ly = (c / RX) % RY, lz = c / (RX * RY);
            const float code = __int_as_float(lx | (ly << 8) | (lz << 16));
            const int k0 = sm.rstart[c], k1 = (c + 1 < NR) ? sm.rstart[c + 1] : S, g0 = sm.gstart[c];
            for (int k = k0; k < k1; k++) {
                const int s = g0 + (k - k0);
                const float4 p = pos[s];
                sm.pos[k] = make_float4(p.x, p.y, p.z, code);
                sm.vel[k] = vel[s];
                sm.slot[k] = s;
            }
        }
    }
    __syncthreads();
    // 3. home cells, handed out one at a time to the warps
    const float wx = d.w[0], wy = d.w[1], wz = d.w[2];
    const float rcmax2 = d.rcmax2;
    const int nhome = ex * ey * ez;
    const unsigned lt = (1u << lane) - 1u;
    uint32_t head = 0, tail = 0;
    auto rc_idx = [&](int x, int y, int z) { return (z * RY + y) * RX + x; };
    for (;;) {
        int h = 0;
        if (lane == 0) h = atomicAdd(&s_next, 1);
        h = __shfl_sync(0xffffffffu, h, 0);
        if (h >= nhome) break;
        const int hx = h % ex, hy = (h / ex) % ey, hz = h / (ex * ey);
        const int ch = rc_idx(hx + 1, hy + 1, hz);
        const int ia = sm.rstart[ch], ib = sm.rstart[ch + 1];
        if (ia == ib) continue;
        // lanes 0..4 hold the five candidate ranges {start, length}
        int rs = 0, rl = 0;
        if (lane < 5) {
            int c0, c1;
            if (lane == 0) {
                c0 = 0;  // unused: R0 starts at the home cell's first particle
                c1 = rc_idx(hx + 2, hy + 1, hz);
            } else if (lane == 1) {
                c0 = rc_idx(hx, hy + 2, hz);
                c1 = rc_idx(hx + 2, hy + 2, hz);
            } else {
                c0 = rc_idx(hx, hy + lane - 2, hz + 1);
                c1 = rc_idx(hx + 2, hy + lane - 2, hz + 1);
            }
            rs = lane == 0 ? ia : sm.rstart[c0];
            rl = sm.rstart[c1 + 1] - rs;
        }
        int rp = rl;  // inclusive prefix of the lengths over lanes 0..4
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, rp, o);
            if (lane >= o) rp += t;
        }
        const int M = __shfl_sync(0xffffffffu, rp, 4);
        const int p1 = __shfl_sync(0xffffffffu, rp, 0), p2 = __shfl_sync(0xffffffffu, rp, 1),
                  p3 = __shfl_sync(0xffffffffu, rp, 2), p4 = __shfl_sync(0xffffffffu, rp, 3);
        for (int cb = 0; cb < M; cb += 32) {
            const int t = cb + lane;
            const bool valid = t < M;
            const int k = (t >= p1) + (t >= p2) + (t >= p3) + (t >= p4);
            const int kstart = __shfl_sync(0xffffffffu, rs, k);
            const int kpre = __shfl_sync(0xffffffffu, rp - rl, k);  // exclusive prefix
            const int j = valid ? kstart + (t - kpre) : 0;
            const float4 pj = sm.pos[j];
            const int code = __float_as_int(pj.w);
            // (c_i - c_j) w: exact multiples of w (differences in {-1, 0, 1})
            const float sx = __int2float_rn(hx + 1 - (code & 0xff)) * wx;
            const float sy = __int2float_rn(hy + 1 - ((code >> 8) & 0xff)) * wy;
            const float sz = __int2float_rn(hz - (code >> 16)) * wz;
            for (int i = ia; i < ib; i++) {
                const float4 pi = sm.pos[i];
                const float dx = __fadd_rn(__fsub_rn(pi.x, pj.x), sx);
                const float dy = __fadd_rn(__fsub_rn(pi.y, pj.y), sy);
                const float dz = __fadd_rn(__fsub_rn(pi.z, pj.z), sz);
                const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
                const bool hit = valid && j > i && r2 <= rcmax2;
                const unsigned m = __ballot_sync(0xffffffffu, hit);
                if (m) {
                    if (hit) {
                        const uint32_t e = (tail + __popc(m & lt)) & (TILE_Q - 1);
                        sm.qd[warp * TILE_Q + e] = make_float4(dx, dy, dz, r2);
                        sm.qij[warp * TILE_Q + e] = (uint32_t)i | ((uint32_t)j << 16);
                    }
                    tail += __popc(m);
                    __syncwarp();
                    if (tail - head >= 32u) {
                        tile_eval<LOG>(a, d, sm, warp, lane, head, 32, step, accv);
                        head += 32;
                    }
                }
            }
        }
    }
    if (tail != head) tile_eval<LOG>(a, d, sm, warp, lane, head, (int)(tail - head), step, accv);
    // 4. bonds of the home particles (each takes its own side of its bonds)
    if (BONDS && d.bond_style) {
        const int par = *a.parity;
        const float4* pos = a.buf.pos[par];
        for (int k = tid; k < S; k += blockDim.x) {
            const int code = __float_as_int(sm.pos[k].w);
            const int rx = code & 0xff, ry = (code >> 8) & 0xff, rz = code >> 16;
            if (rx < 1 || rx > ex || ry < 1 || ry > ey || rz >= ez) continue;
            const int s = sm.slot[k];
            float fx = 0.0f, fy = 0.0f, fz = 0.0f;
            bond_loop<LOG>(a, d, pos, a.buf.bonds[par], r, s, pos[s], fx, fy, fz, accv);
            atomicAdd(&a.force4[s], make_float4(fx, fy, fz, 0.0f));
        }
    }
    return true;
}

// One tile: the whole home box, or (when its neighbourhood does not fit) its home cells
// one at a time.
template <bool LOG, bool BONDS>
__device__ __forceinline__ void tile_run(const StepArgs& a, const TileArgs& ta, const TileSmem& sm, int t,
                                         double (&accv)[8])
{
    const int r = ta.tile_rep[t];
    const RepDesc& d = a.reps[r];
    const RepState st = a.rstate[r];
    const int code = ta.tile_code[t];
    const int E = ta.edge;
    const int x0 = (code & 1023) * E, y0 = ((code >> 10) & 1023) * E, z0 = (code >> 20) * E;
    const int ex = min(E, d.nc[0] - x0), ey = min(E, d.nc[1] - y0), ez = min(E, d.nc[2] - z0);
    if (tile_box<LOG, BONDS>(a, ta, sm, d, r, x0, y0, z0, ex, ey, ez, st.step, accv)) return;
    for (int h = 0; h < ex * ey * ez; h++) {
        const int hx = x0 + h % ex, hy = y0 + (h / ex) % ey, hz = z0 + h / (ex * ey);
        if (!tile_box<LOG, BONDS>(a, ta, sm, d, r, hx, hy, hz, 1, 1, 1, st.step, accv) && threadIdx.x == 0)
            atomicOr(&a.rstate[r].status, ST_LIST_OVERFLOW);
    }
}

__device__ __forceinline__ bool tile_live(const StepArgs& a, const TileArgs& ta, int t, bool& log)
{
    const int r = ta.tile_rep[t];
    const RepState st = a.rstate[r];
    const RepDesc& d = a.reps[r];
    log = (st.step % (uint32_t)d.log_f) == 0u;
    return rep_active(st) && d.style == 0;
}

// Non-log steps: a CTA per tile.
template <bool BONDS, int MINB>
__global__ void __launch_bounds__(256, MINB) k_tile(StepArgs a, TileArgs ta)
{
    griddep_wait();
    extern __shared__ __align__(16) unsigned char tile_dyn[];
    const int t = blockIdx.x;
    bool log = false;
    if (t >= ta.ntiles || !tile_live(a, ta, t, log) || log) return;  // CTA-uniform
    const TileSmem sm = tile_smem(tile_dyn, ta.smax);
    double accv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    tile_run<false, BONDS>(a, ta, sm, t, accv);
}

// Log steps: a small grid-stride launch over the tiles of the replicas that log this
// step (the common answer is none, and then every block returns at once).
template <bool BONDS>
__global__ void __launch_bounds__(256, 2) k_tile_logsteps(StepArgs a, TileArgs ta)
{
    griddep_wait();
    extern __shared__ __align__(16) unsigned char tile_dyn[];
    int any = 0;
    for (int r = threadIdx.x; r < a.nrep; r += blockDim.x) {
        const RepState st = a.rstate[r];
        any |= rep_active(st) && (st.step % (uint32_t)a.reps[r].log_f) == 0u;
    }
    if (!__syncthreads_or(any)) return;
    const TileSmem sm = tile_smem(tile_dyn, ta.smax);
    for (int t = blockIdx.x; t < ta.ntiles; t += gridDim.x) {
        bool log = false;
        if (!tile_live(a, ta, t, log) || !log) continue;  // CTA-uniform
        double accv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        tile_run<true, BONDS>(a, ta, sm, t, accv);
        const int fields[8] = {ACC_PAIR_PE, ACC_BOND_PE, ACC_VIR + 0, ACC_VIR + 1,
                               ACC_VIR + 2, ACC_VIR + 3, ACC_VIR + 4, ACC_VIR + 5};
        acc_flush_warp<8>(accv, fields, ta.tile_rep[t], a.acc);
    }
}
