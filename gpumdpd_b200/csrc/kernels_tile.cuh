// kernels_tile.cuh -- DPD pair forces straight from the cell ranges of the counting sort,
// with no neighbour list: the list build and the list-driven pair pass as one kernel.
//
// A CTA takes a tile of home cells (T x T x T, fewer at the grid's edge) of one replica
// and stages the positions of the particles of the cells its half stencil reaches -- x in [x0-1, x0+T],
// y in [y0-1, y0+T], z in [z0, z0+T] -- into shared memory, cell by cell with x fastest,
// so that the 13 forward cells of a home cell plus the rest of its own cell form five
// contiguous ranges of staged particles:
//   R0: own cell after i, then cell (x+1, y, z)        (offsets 0 and (1,0,0))
//   R1: cells (x-1..x+1, y+1, z)                       (the row dz = 0, dy = +1)
//   R2..R4: cells (x-1..x+1, y-1..y+1, z+1)             (the three rows dz = +1)
// -- the half stencil of src/force/neigh_list.cu:322-393 (every unordered cell pair
// once; at least 3 cells per dimension).  The warps take the home particles 32 at a time
// (a shared counter hands them out); each lane walks its particle's five ranges as one
// sequence with the list predicate of the list build,
//   d = (o_i - o_j) + (c_i - c_j) w,  r2 = fma(dz,dz, fma(dy,dy, dx*dx)) <= rc_max^2,
// so the pairs evaluated are exactly the list path's, and keeps its hits in its own
// column of a shared buffer.  The warp then takes its 32 lanes' hits as one sequence,
// 32 pairs at a time (the owner lane of each found by a binary search over the scanned
// counts), and evaluates them with every lane busy (Saru random force,
// src/force/pair_dpd.cu:468-558), each with the float4 reductions of both sides into the
// force array.  The home particles' bonds follow (bond_loop).  Log steps add the FP64
// energy and virial sums, flushed per warp.
//
// When a tile's neighbourhood holds more particles than the staging capacity (a local
// density far above the mean), the CTA takes its home cells one at a time with the
// smaller neighbourhood of one cell; only if that does not fit either, or a particle has
// more pairs than the hit buffer holds (the list capacity of `neighbor ... max_rho`), is
// the replica's ST_LIST_OVERFLOW raised (pairs are then missing, and the run fails with
// DPD_E_OVERFLOW).
#pragma once
#include "kernels_step.cuh"

#define TILE_MAX_EDGE 6
#define TILE_MAX_REGION ((TILE_MAX_EDGE + 2) * (TILE_MAX_EDGE + 2) * (TILE_MAX_EDGE + 1))
#define TILE_THREADS 256

struct TileArgs {
    const int* tile_rep;   // [ntiles] replica of each tile
    const int* tile_code;  // [ntiles] tile coordinates ix | iy << 10 | iz << 20
    int ntiles;
    int edge;              // home cells per tile edge
    int smax;              // staging capacity (particles) of a CTA
    int hc;                // pairs a home particle may have (hit buffer column)
};

// dynamic shared memory of a CTA: staged positions and slots; region cell starts (+1)
// and global starts; home rows; the hit buffer
__host__ __device__ inline size_t tile_smem_bytes(int smax, int hc)
{
    return (size_t)smax * (16 + 4) + (size_t)(2 * TILE_MAX_REGION + 32) * 4 + 128 * 4 +
           (size_t)hc * TILE_THREADS * 2;
}

struct TileSmem {
    float4* pos;    // [smax] {o.x, o.y, o.z, region cell code rx | ry << 8 | rz << 16}
    int* slot;      // [smax] particle slot
    int* rstart;    // [TILE_MAX_REGION + 16] first staged index of each region cell, the
                    // total after the last one; [TILE_MAX_REGION + 8 + w]: warp totals
    int* gstart;    // [TILE_MAX_REGION] first slot of each region cell
    int* rowpre;    // [64] home particles before each home row (y, z), the total after
    int* rowbeg;    // [64] first staged index of each home row
    uint16_t* hits; // [hc][TILE_THREADS] staged index j of each pair found, a column a thread
};

__device__ __forceinline__ TileSmem tile_smem(unsigned char* base, int smax)
{
    TileSmem t;
    t.pos = (float4*)base;
    t.slot = (int*)(t.pos + smax);
    t.rstart = t.slot + smax;
    t.gstart = t.rstart + TILE_MAX_REGION + 16;
    t.rowpre = t.gstart + TILE_MAX_REGION + 16;
    t.rowbeg = t.rowpre + 64;
    t.hits = (uint16_t*)(t.rowbeg + 64);
    return t;
}

// One staged pair (i, j): the displacement again from the offsets and the region cells
// (bit for bit the walk's), the velocities (tag and type in .w) through L1, then the DPD
// force into both sides.
template <bool LOG>
__device__ __forceinline__ void tile_pair(const StepArgs& a, const RepDesc& d, const TileSmem& sm,
                                          const float4* vel, int i, int j, uint32_t step, double (&accv)[8])
{
    const int si = sm.slot[i], sj = sm.slot[j];
    const float4 pi = sm.pos[i], pj = sm.pos[j];
    const int ci = __float_as_int(pi.w), cj = __float_as_int(pj.w);
    const float sx = __int2float_rn((ci & 0xff) - (cj & 0xff)) * d.w[0];
    const float sy = __int2float_rn(((ci >> 8) & 0xff) - ((cj >> 8) & 0xff)) * d.w[1];
    const float sz = __int2float_rn((ci >> 16) - (cj >> 16)) * d.w[2];
    const float dx = __fadd_rn(__fsub_rn(pi.x, pj.x), sx);
    const float dy = __fadd_rn(__fsub_rn(pi.y, pj.y), sy);
    const float dz = __fadd_rn(__fsub_rn(pi.z, pj.z), sz);
    const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
    const float4 vi = __ldg(vel + si), vj = __ldg(vel + sj);
    const float4* crow = a.coeff + d.coeff_off + type0_of(vi.w) * d.ntypes * 3;
    float fx, fy, fz;
    if (pair_force<0, LOG>(crow, r2, dx, dy, dz, vi, vj, 0.0f, 0.0f, d.seed, step, fx, fy, fz, accv)) {
        atomicAdd(&a.force4[si], make_float4(fx, fy, fz, 0.0f));
        atomicAdd(&a.force4[sj], make_float4(-fx, -fy, -fz, 0.0f));
    }
}

// The candidates of staged home particle i: its five ranges walked as one sequence with
// the list predicate r2 <= cut2; hit(count, j, code) is called for each pair found, code =
// 9 (dcx+1) + 3 (dcy+1) + (dcz+1) of the cell difference c_i - c_j.  Returns the count.
template <class Hit>
__device__ __forceinline__ int tile_walk(const TileSmem& sm, int i, int RX, int RY, float wx, float wy, float wz,
                                         float cut2, Hit&& hit)
{
    const float4 pi = sm.pos[i];
    const int code = __float_as_int(pi.w);
    const int rx = code & 0xff, ry = (code >> 8) & 0xff, rz = code >> 16;
    int cnt = 0, k = 0;
    // range 0: the rest of the own cell (sx = 0), then cell x+1 (sx = -w); b1 = 0: no
    // cell x-1 part
    const int cr = (rz * RY + ry) * RX + rx + 1;
    int j = i + 1, b1 = 0, b2 = sm.rstart[cr], end = sm.rstart[cr + 1];
    float sy = 0.0f, sz = 0.0f;
    int cyz = 4;  // 3 (dcy+1) + (dcz+1) of the current range
    for (;;) {
        if (j >= end) {
            if (++k == 5) break;
            // ranges 1..4: the rows (x-1..x+1) at (y+1, z), (y-1, z+1), (y, z+1), (y+1, z+1)
            const int yy = k == 1 ? ry + 1 : ry + k - 3, zz = k == 1 ? rz : rz + 1;
            const int c0 = (zz * RY + yy) * RX + rx - 1;
            j = sm.rstart[c0];
            b1 = sm.rstart[c0 + 1];
            b2 = sm.rstart[c0 + 2];
            end = sm.rstart[c0 + 3];
            sy = __int2float_rn(ry - yy) * wy;
            sz = __int2float_rn(rz - zz) * wz;
            cyz = 3 * (ry - yy + 1) + (rz - zz + 1);
            continue;
        }
        const float4 pj = sm.pos[j];
        const float sx = j < b1 ? wx : (j < b2 ? 0.0f : -wx);
        const float dx = __fadd_rn(__fsub_rn(pi.x, pj.x), sx);
        const float dy = __fadd_rn(__fsub_rn(pi.y, pj.y), sy);
        const float dz = __fadd_rn(__fsub_rn(pi.z, pj.z), sz);
        const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
        if (r2 <= cut2) {
            hit(cnt, j, (j < b1 ? 18 : (j < b2 ? 9 : 0)) + cyz);
            cnt++;
        }
        j++;
    }
    return cnt;
}

// Stage the neighbourhood of the home box [hx0, hx0+ex) x [hy0, hy0+ey) x [hz0, hz0+ez)
// (global cell coordinates) of replica r and evaluate its pairs and its home particles'
// bonds.  Returns false (having done nothing) when the neighbourhood does not fit the
// staging capacity.  Called by the whole CTA; begins and ends with a barrier.
// LIST: instead of the forces, the half list of the list schedules: each home particle's
// pairs within (global_cut + skin) as entries j | code << 27 of its warp-interleaved list
// (the list build's entries, src/force/neigh_list.cu:322-393).
template <bool LOG, bool BONDS, bool LIST = false>
__device__ __forceinline__ bool tile_box(const StepArgs& a, const TileArgs& ta, const TileSmem& sm, const RepDesc& d, int r,
                         int hx0, int hy0, int hz0, int ex, int ey, int ez, uint32_t step, double (&accv)[8],
                         int* nlist = nullptr, int* ncount = nullptr)
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
        for (int c = tid; c < NR; c += blockDim.x) {
            const int lx = c % RX, ly = (c / RX) % RY, lz = c / (RX * RY);
            const float code = __int_as_float(lx | (ly << 8) | (lz << 16));
            const int k0 = sm.rstart[c], k1 = (c + 1 < NR) ? sm.rstart[c + 1] : S, g0 = sm.gstart[c];
            for (int k = k0; k < k1; k++) {
                const int s = g0 + (k - k0);
                const float4 p = pos[s];
                sm.pos[k] = make_float4(p.x, p.y, p.z, code);
                sm.slot[k] = s;
            }
        }
    }
    __syncthreads();
    // 3. home rows (the home cells of one (y, z), contiguous in staged order) and the
    //    count of home particles before each
    auto rc_idx = [&](int x, int y, int z) { return (z * RY + y) * RX + x; };
    const int NROW = ey * ez;  // <= 36
    if (warp == 0) {
        int sz0 = 0, sz1 = 0, bg0 = 0, bg1 = 0;
        if (lane < NROW) {
            bg0 = sm.rstart[rc_idx(1, lane % ey + 1, lane / ey)];
            sz0 = sm.rstart[rc_idx(ex, lane % ey + 1, lane / ey) + 1] - bg0;
        }
        if (lane + 32 < NROW) {
            const int r2w = lane + 32;
            bg1 = sm.rstart[rc_idx(1, r2w % ey + 1, r2w / ey)];
            sz1 = sm.rstart[rc_idx(ex, r2w % ey + 1, r2w / ey) + 1] - bg1;
        }
        int i0 = sz0, i1 = sz1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t0 = __shfl_up_sync(0xffffffffu, i0, o), t1 = __shfl_up_sync(0xffffffffu, i1, o);
            if (lane >= o) {
                i0 += t0;
                i1 += t1;
            }
        }
        const int tot0 = __shfl_sync(0xffffffffu, i0, 31), tot1 = __shfl_sync(0xffffffffu, i1, 31);
        if (lane < NROW) {
            sm.rowpre[lane] = i0 - sz0;
            sm.rowbeg[lane] = bg0;
        }
        if (lane + 32 < NROW) {
            sm.rowpre[lane + 32] = tot0 + i1 - sz1;
            sm.rowbeg[lane + 32] = bg1;
        }
        if (lane == 0) sm.rowpre[NROW] = tot0 + tot1;
    }
    __syncthreads();
    // 4. home particles, handed out 32 at a time to the warps: each lane walks its
    //    particle's candidates, then the warp evaluates the pairs its lanes found
    const float wx = d.w[0], wy = d.w[1], wz = d.w[2];
    const float rcmax2 = d.rcmax2;
    const int H = sm.rowpre[NROW];
    if (LIST) {
        for (int t = tid; t < H; t += blockDim.x) {
            int rr = 0;
#pragma unroll
            for (int stp = 32; stp >= 1; stp >>= 1)
                if (rr + stp < NROW && sm.rowpre[rr + stp] <= t) rr += stp;
            const int i = sm.rowbeg[rr] + (t - sm.rowpre[rr]);
            const int s = sm.slot[i];
            int* out = nlist + ((size_t)(s >> 5) * a.nmax) * 32 + (s & 31);
            const int nmax = a.nmax;
            int cnt = tile_walk(sm, i, RX, RY, wx, wy, wz, d.cut2, [&](int c, int j, int code) {
                if (c < nmax) out[(size_t)c * 32] = sm.slot[j] | (code << DPD_CODE_SHIFT);
            });
            if (cnt > nmax) {
                atomicOr(&a.rstate[r].status, ST_LIST_OVERFLOW);
                cnt = nmax;
            }
            ncount[s] = cnt;
        }
        return true;
    }
    const int hc = ta.hc;
    uint16_t* col = sm.hits + tid;
    const float4* vel = a.buf.vel[*a.parity];
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&s_next, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= H) break;
        const int t = base + lane;
        int cnt = 0, i = 0;
        if (t < H) {
            int rr = 0;  // the last row whose first home particle is at or before t
#pragma unroll
            for (int stp = 32; stp >= 1; stp >>= 1)
                if (rr + stp < NROW && sm.rowpre[rr + stp] <= t) rr += stp;
            i = sm.rowbeg[rr] + (t - sm.rowpre[rr]);
            cnt = tile_walk(sm, i, RX, RY, wx, wy, wz, rcmax2, [&](int c, int j, int) {
                if (c < hc) col[c * TILE_THREADS] = (uint16_t)j;
            });
        }
        if (__any_sync(0xffffffffu, cnt > hc) && lane == 0) atomicOr(&a.rstate[r].status, ST_LIST_OVERFLOW);
        const int c = min(cnt, hc);
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int excl = incl - c;
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        __syncwarp();  // the lanes' hits are written
        for (int b = 0; b < total; b += 32) {
            const int f = b + lane;
            int o = 0;  // owner lane: the last lane whose first hit is at or before f
#pragma unroll
            for (int stp = 16; stp >= 1; stp >>= 1)
                if (__shfl_sync(0xffffffffu, excl, o + stp) <= f) o += stp;
            const int io = __shfl_sync(0xffffffffu, i, o);
            const int q = f - __shfl_sync(0xffffffffu, excl, o);
            if (f < total) tile_pair<LOG>(a, d, sm, vel, io, sm.hits[q * TILE_THREADS + warp * 32 + o], step, accv);
        }
        __syncwarp();  // the hits are read before the next walk writes the columns again
    }
    // 5. bonds of the home particles (each takes its own side of its bonds)
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
// one at a time (a single call site, so that the box code is inlined once).
template <bool LOG, bool BONDS, bool LIST = false>
__device__ __forceinline__ void tile_run(const StepArgs& a, const TileArgs& ta, const TileSmem& sm, int t,
                                         double (&accv)[8], int* nlist = nullptr, int* ncount = nullptr)
{
    const int r = ta.tile_rep[t];
    const RepDesc& d = a.reps[r];
    const RepState st = a.rstate[r];
    const int code = ta.tile_code[t];
    const int E = ta.edge;
    const int x0 = (code & 1023) * E, y0 = ((code >> 10) & 1023) * E, z0 = (code >> 20) * E;
    const int ex = min(E, d.nc[0] - x0), ey = min(E, d.nc[1] - y0), ez = min(E, d.nc[2] - z0);
    bool whole = true;
    int nbox = 1;
    for (int b = 0; b < nbox; b++) {
        int bx = x0, by = y0, bz = z0, bex = ex, bey = ey, bez = ez;
        if (!whole) {
            bx = x0 + b % ex;
            by = y0 + (b / ex) % ey;
            bz = z0 + b / (ex * ey);
            bex = bey = bez = 1;
        }
        const bool ok = tile_box<LOG, BONDS, LIST>(a, ta, sm, d, r, bx, by, bz, bex, bey, bez, st.step, accv, nlist,
                                                   ncount);
        if (!ok && whole) {  // CTA-uniform: the home cells one at a time instead
            whole = false;
            nbox = ex * ey * ez;
            b = -1;
        } else if (!ok && threadIdx.x == 0) {
            atomicOr(&a.rstate[r].status, ST_LIST_OVERFLOW);
        }
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

// The half list of the list schedules built from the tiles (list-build variant 4): a CTA
// per tile stages its neighbourhood's positions and walks each home particle's candidates
// in shared memory, instead of a thread per particle gathering its 14 cell ranges from
// global memory.  The same entries as the list build; their order within a particle's list
// is the walk's.  Runs only when a list build is due.
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_tile_build(StepArgs a, TileArgs ta, BuildArgs b)
{
    griddep_wait();
    extern __shared__ __align__(16) unsigned char tile_dyn[];
    if (!build_on(b)) return;  // grid-uniform
    const int t = blockIdx.x;
    if (t >= ta.ntiles || !rep_active(a.rstate[ta.tile_rep[t]])) return;  // a finished replica gets no list
    const TileSmem sm = tile_smem(tile_dyn, ta.smax);
    double accv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    tile_run<false, false, true>(a, ta, sm, t, accv, b.nlist, b.ncount);
}
