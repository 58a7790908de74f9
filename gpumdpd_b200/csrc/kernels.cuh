// kernels.cuh -- sm_100a kernels of the neighbour-list build, plus shared helpers.
//
// Particle layout (packed over replicas; each replica owns a warp-aligned slot range),
// double-buffered by a device-side parity bit (the list build permutes into the other
// buffer and flips it):
//   pos[s]   = {ox, oy, oz, cell code}  offsets relative to cell (cx,cy,cz); the code
//              packs cx | cy<<10 | cz<<20 (replica-local).  Cells are assigned at a list
//              build and kept until the next one, so offsets may drift slightly outside
//              [0,w) in between; a build re-bins every particle.
//   vel[s]   = {vx, vy, vz, tag<<5 | (type-1)}
//   force4[s]= {fx, fy, fz, 0}           accumulated with vector atomics
//   img[t]   = image counters, by tag (tag_base + tag - 1), single-buffered: a build that
//              re-bins a particle across the box updates its counters in place, so the
//              permutation does not move them
// Slots are sorted by cell (counting sort at every build; cells in the engine's cell order:
// linear with z fastest, Morton, or x-y columns in Morton order with z fastest; within a
// cell in the order the counting pass's atomics drew).  The half neighbour list is
// warp-chunked,
//   nlist[((s>>5)*nmax + k)*32 + (s&31)] = j | code<<27,
// where code = 9(dcx+1)+3(dcy+1)+(dcz+1) encodes the cell difference c_i - c_j in
// {-1,0,1}^3 of the pair at build time; the displacement is (o_i - o_j) + code*w.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "dpd_common.h"
#include "saru.cuh"

#define DPD_J_MASK 0x07FFFFFF
#define DPD_CODE_SHIFT 27

// Kernels of the step are launched with programmatic dependent launch: the next kernel's
// launch overlaps the end of the previous one, and each kernel waits here (PTX
// griddepcontrol.wait) until its predecessor's memory is visible.  Without a programmatic
// predecessor the wait returns at once.
__device__ __forceinline__ void griddep_wait()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// ---------------------------------------------------------------------------------
__device__ __forceinline__ int cell_x(int code) { return code & DPD_MAX_NC; }
__device__ __forceinline__ int cell_y(int code) { return (code >> DPD_CELL_BITS) & DPD_MAX_NC; }
__device__ __forceinline__ int cell_z(int code) { return (code >> (2 * DPD_CELL_BITS)) & DPD_MAX_NC; }
__device__ __forceinline__ int cell_pack(int x, int y, int z)
{
    return x | (y << DPD_CELL_BITS) | (z << (2 * DPD_CELL_BITS));
}
__device__ __forceinline__ int tag_of(float w) { return (int)(((uint32_t)__float_as_int(w)) >> DPD_TYPE_BITS); }
__device__ __forceinline__ int type0_of(float w) { return __float_as_int(w) & ((1 << DPD_TYPE_BITS) - 1); }

// wrap a cell difference to the nearest image of the cell grid
__device__ __forceinline__ int wrap_dc(int dc, int nc)
{
    int h = nc >> 1;
    dc -= (dc > h) ? nc : 0;
    dc += (dc < -h) ? nc : 0;
    return dc;
}

// General displacement p_i - p_j between any two particles (bonds, RDF, skin check):
// cell difference wrapped to the grid, then a position-level minimum image.
__device__ __forceinline__ float disp1(int ci, int cj, float oi, float oj, int nc, float w, float L)
{
    int dc = wrap_dc(ci - cj, nc);
    float d = __fmaf_rn(__int2float_rn(dc), w, __fsub_rn(oi, oj));
    float h = 0.5f * L;
    d -= (d >= h) ? L : 0.0f;
    d += (d < -h) ? L : 0.0f;
    return d;
}

// ---------------------------------------------------------------------------------
// FP64 per-replica accumulation: warp reduce, then one atomic per (block, replica
// segment, field) into one of DPD_ACC_SLOTS spread copies.
template <int NV>
__device__ __forceinline__ void acc_flush(double (&val)[NV], const int* field, int rep, double* acc)
{
    __shared__ double sh[32][NV];
    __shared__ int shrep[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double x = val[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        val[k] = x;
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) sh[warp][k] = val[k];
        shrep[warp] = rep;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        const int k = threadIdx.x;
        const int nw = blockDim.x >> 5;
        const int slot = blockIdx.x & (DPD_ACC_SLOTS - 1);
        double s = 0.0;
        int cur = shrep[0];
        for (int w = 0; w < nw; w++) {
            int r = shrep[w];
            if (r != cur) {
                if (cur >= 0 && s != 0.0)
                    atomicAdd(&acc[((size_t)cur * DPD_ACC_SLOTS + slot) * DPD_NACC + field[k]], s);
                s = 0.0;
                cur = r;
            }
            s += sh[w][k];
        }
        if (cur >= 0 && s != 0.0)
            atomicAdd(&acc[((size_t)cur * DPD_ACC_SLOTS + slot) * DPD_NACC + field[k]], s);
    }
}

// The same per warp: warp reduce, then lane k adds field k into the spread slot of this
// warp.  Needs no block barrier; call it from warp-uniform code only.
template <int NV>
__device__ __forceinline__ void acc_flush_warp(double (&val)[NV], const int* field, int rep, double* acc)
{
    const int lane = threadIdx.x & 31;
    const int slot = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) & (DPD_ACC_SLOTS - 1);
    double mine = 0.0;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double x = val[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == k) mine = x;
    }
    if (lane < NV && mine != 0.0)
        atomicAdd(&acc[((size_t)rep * DPD_ACC_SLOTS + slot) * DPD_NACC + field[lane]], mine);
}

// ---------------------------------------------------------------------------------
// Double-buffered particle arrays; `par` selects the current buffer.  The image counters
// are indexed by tag and not permuted.
struct PBuf {
    float4* pos[2];
    float4* vel[2];
    int4* img;
    int2* bonds[2];
};

// Neighbour-list build: counting sort of slots by (re-binned) cell (in-cell order: the
// order the counting atomics drew), permutation into the other buffer with the parity
// flip by its last block, then the half list.  All kernels return at once unless the
// build flag of this phase is set.
struct BuildArgs {
    const RepDesc* reps;
    const int* warp_rep;
    const int* crank;       // [cells] linear cell -> position in the replica's cell order
    const int* cell_rep;    // [cells] replica of a cell key
    const int* cell_lin;    // [cells] linear index of a cell key (-1: ghost cell)
    int P;                  // total slots
    int C;                  // total cells (all replicas, ghost cells included)
    int nmax;               // neighbour list capacity per slot
    int maxb;               // bond partners per slot
    const int* build_flag;  // [2]
    const uint32_t* phase;
    int* parity;
    PBuf buf;
    float4* last4;
    int* cnt;
    int* cstart;            // [C+1]
    int* skey;              // [P] cell key of each slot at this build
    int* srank;             // [P] arrival rank of the slot in its cell
    int* tag2idx;
    int* ncount;
    int* nlist;
    RepState* rstate;
    int* blocksum;
    unsigned int* ticket;   // blocks of the permutation done (reset by the last one)
};

__device__ __forceinline__ bool build_on(const BuildArgs& a)
{
    return a.build_flag[(*a.phase) & 1] != 0;
}

// Re-bin a particle: move whole cell widths from the offset into the cell index,
// wrapping the cell grid and counting images.  Returns false for a non-finite offset
// and for a runaway one (a million cell widths or more since the last build, which no
// finite-temperature trajectory reaches: its offset is clamped into the new cell).
__device__ __forceinline__ bool rebin(const RepDesc& d, float4& p, int dimg[3])
{
    int code = __float_as_int(p.w);
    int c[3] = {cell_x(code), cell_y(code), cell_z(code)};
    float o[3] = {p.x, p.y, p.z};
    bool ok = true, moved = false;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        dimg[k] = 0;
        if (!(o[k] >= 0.0f && o[k] < d.w[k])) {
            if (!isfinite(o[k])) {
                ok = false;
                o[k] = 0.0f;
                continue;
            }
            float q = floorf(o[k] * d.inv_w[k]);
            if (!(fabsf(q) < 1.0e6f)) ok = false;
            q = fminf(fmaxf(q, -1.0e6f), 1.0e6f);
            o[k] = __fmaf_rn(-q, d.w[k], o[k]);
            int cc = c[k] + (int)q;
            const int nc = d.nc[k];
            const int wrap = cc >= 0 ? cc / nc : -((-cc + nc - 1) / nc);
            cc -= wrap * nc;
            dimg[k] = wrap;
            c[k] = cc;
            if (o[k] >= d.w[k]) o[k] = __int_as_float(__float_as_int(d.w[k]) - 1);
            if (o[k] < 0.0f) o[k] = 0.0f;
            moved = true;
        }
    }
    if (moved) code = cell_pack(c[0], c[1], c[2]);
    p = make_float4(o[0], o[1], o[2], __int_as_float(code));
    return ok;
}

__device__ __forceinline__ int cell_key(const BuildArgs& a, const RepDesc& d, int code, bool ghost)
{
    if (ghost) return d.c_begin + d.ncell;
    int lin = (cell_x(code) * d.nc[1] + cell_y(code)) * d.nc[2] + cell_z(code);
    return d.c_begin + a.crank[d.c_begin + lin];
}

__device__ __forceinline__ int slot_key(const BuildArgs& a, int s, int par)
{
    const RepDesc& d = a.reps[a.warp_rep[s >> 5]];
    if (s >= d.p_end) return d.c_begin + d.ncell;
    float4 p = a.buf.pos[par][s];
    int dimg[3];
    rebin(d, p, dimg);
    return cell_key(a, d, __float_as_int(p.w), false);
}

__global__ void k_bin_count(BuildArgs a)
{
    griddep_wait();
    if (!build_on(a)) return;
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.P) return;
    const int key = slot_key(a, s, *a.parity);
    a.skey[s] = key;
    a.srank[s] = atomicAdd(&a.cnt[key], 1);
}

// exclusive scan of cnt[0..C) into cstart[0..C], three passes (block scan of 4096
// elements, scan of block sums in one block, add back).
// SINGLE: the whole scan fits one block (C <= 4096): the block's scan is the result, and
// it writes the total, so the two passes over the block sums are not launched.
template <bool SINGLE>
__global__ void k_scan_blocks(BuildArgs a)
{
    griddep_wait();
    if (!build_on(a)) return;
    __shared__ int sh[1024];
    const int base = blockIdx.x * 4096;
    int v[4], tot = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        int idx = base + threadIdx.x * 4 + k;
        v[k] = idx < a.C ? a.cnt[idx] : 0;
        if (idx < a.C) a.cnt[idx] = 0;  // ready for the next build's counting pass
        tot += v[k];
    }
    sh[threadIdx.x] = tot;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += t;
        __syncthreads();
    }
    int run = sh[threadIdx.x] - tot;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        int idx = base + threadIdx.x * 4 + k;
        if (idx < a.C) a.cstart[idx] = run;
        run += v[k];
    }
    if (threadIdx.x == 1023) {
        if (SINGLE) a.cstart[a.C] = sh[1023];
        else a.blocksum[blockIdx.x] = sh[1023];
    }
}

__global__ void k_scan_sums(BuildArgs a, int nblocks)
{
    griddep_wait();
    if (!build_on(a)) return;
    __shared__ int sh[1024];
    int carry = 0;
    for (int base = 0; base < nblocks; base += 1024) {
        int idx = base + threadIdx.x;
        int v = idx < nblocks ? a.blocksum[idx] : 0;
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
            __syncthreads();
            sh[threadIdx.x] += t;
            __syncthreads();
        }
        if (idx < nblocks) a.blocksum[idx] = carry + sh[threadIdx.x] - v;
        int total = sh[1023];
        __syncthreads();
        carry += total;
    }
    if (threadIdx.x == 0) a.cstart[a.C] = carry;
}

__global__ void k_scan_add(BuildArgs a)
{
    griddep_wait();
    if (!build_on(a)) return;
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < a.C) a.cstart[idx] += a.blocksum[idx / 4096];
}

// scatter every slot to its place in the other buffer (cell start + the rank the counting
// pass drew), re-binning positions; the new positions are also the reference positions
// of the displacement check (last4).  Reads are coalesced; the writes of a warp land in
// a few neighbouring cells.
__device__ __forceinline__ void permute_slot(const BuildArgs& a, const int s)
{
    const int par = *a.parity, nxt = par ^ 1;
    const int r = a.warp_rep[s >> 5];
    const RepDesc& d = a.reps[r];
    // the slot's own records first: their loads do not wait on the destination, which takes
    // a dependent gather (the cell start of the slot's key)
    float4 p = a.buf.pos[par][s];
    const float4 v = a.buf.vel[par][s];
    int2 b01[2] = {make_int2(0, 0), make_int2(0, 0)};  // the first two bond records
#pragma unroll
    for (int k = 0; k < 2; k++)
        if (k < a.maxb) b01[k] = a.buf.bonds[par][(size_t)k * a.P + s];
    const int key = a.skey[s], rank = a.srank[s];
    int dimg[3] = {0, 0, 0};
    const bool real = s < d.p_end;
    if (real && !rebin(d, p, dimg)) atomicOr(&a.rstate[r].status, ST_NONFINITE);
    const int dst = a.cstart[key] + rank;
    if (dst < d.p_begin || dst >= d.p_cap_end) {  // cannot happen: keys stay in the replica
        atomicOr(&a.rstate[r].status, ST_BAD_INPUT);
        return;
    }
    if (real) {
        int t = tag_of(v.w);
        if (t >= 1 && t <= d.n_real) {
            a.tag2idx[d.tag_base + t - 1] = dst;
            // across the box: the particle's own counters (one slot per tag, no race)
            if (dimg[0] | dimg[1] | dimg[2]) {
                int4* ip = a.buf.img + d.tag_base + t - 1;
                int4 im = *ip;
                im.x += dimg[0];
                im.y += dimg[1];
                im.z += dimg[2];
                *ip = im;
            }
        }
    }
    a.buf.pos[nxt][dst] = p;
    a.buf.vel[nxt][dst] = v;
    if (!d.skin_zero) a.last4[dst] = p;  // skin 0 rebuilds unconditionally: no skin check
#pragma unroll
    for (int k = 0; k < 2; k++)
        if (k < a.maxb) a.buf.bonds[nxt][(size_t)k * a.P + dst] = b01[k];
    for (int k = 2; k < a.maxb; k++)
        a.buf.bonds[nxt][(size_t)k * a.P + dst] = a.buf.bonds[par][(size_t)k * a.P + s];
}

// The permutation.  FLIP (small grids, where a launch costs more than the work): the
// last block to finish (a ticket counter) also flips the parity, counts the build of
// every replica and resets the ticket.  Every block has read the parity before it takes
// its ticket, and the list build that follows waits for the whole grid.  Large grids
// leave the flip to k_flip: the ticket's fence in every block costs more than a launch.
template <bool FLIP>
__global__ void k_permute(BuildArgs a, int nrep)
{
    griddep_wait();
    if (!build_on(a)) return;  // grid-uniform
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < a.P) permute_slot(a, s);
    if (!FLIP) return;
    if (s < a.P) a.ncount[s] = 0;  // k_build_wide counts with atomics
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(a.ticket, 1u) == gridDim.x - 1u;
    }
    __syncthreads();
    if (last) {
        for (int r = threadIdx.x; r < nrep; r += blockDim.x) a.rstate[r].nbuild++;
        if (threadIdx.x == 0) {
            *a.parity ^= 1;
            *a.ticket = 0u;
        }
    }
}

__global__ void k_flip(BuildArgs a, int nrep)
{
    griddep_wait();
    if (!build_on(a)) return;
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nrep) a.rstate[r].nbuild++;
    if (r == 0) *a.parity ^= 1;
}

// half stencil: the 13 cell offsets with (oz>0) | (oz==0 & oy>0) | (oz==0 & oy==0 & ox>0)
__constant__ int8_t c_half[13][3] = {
    {1, 0, 0}, {-1, 1, 0}, {0, 1, 0}, {1, 1, 0}, {-1, -1, 1}, {0, -1, 1}, {1, -1, 1},
    {-1, 0, 1}, {0, 0, 1}, {1, 0, 1}, {-1, 1, 1}, {0, 1, 1}, {1, 1, 1}};

// Half list, one thread per particle (slots in cell order, so a warp's lanes share
// most stencil cells through L1).  Candidates are the own cell's later slots (j > i)
// and the 13 forward cells; all 14 cell ranges are loaded first and each cell's slots
// are read 4 at a time so several loads are in flight per thread.  The predicate is
// r2 = fma(dz,dz,fma(dy,dy,dx*dx)) <= (global_cut+skin)^2 in float with
// d = (o_i - o_j) + (c_i - c_j) w, the reference's test (src/force/neigh_list.cu:373-382)
// on the cell-offset representation.  Entries store j and the shift code of the pair.
template <bool ALL = false>
__device__ __forceinline__ void build_nlist_slot(const BuildArgs& a, const int s)
{
    if (s >= a.P) return;
    const int r = a.warp_rep[s >> 5];
    const RepDesc& d = a.reps[r];
    // ghosts, and replicas past their last step (a finished job of a server cohort),
    // get no list (ALL: every replica's list, for an on-demand build between runs)
    if (s >= d.p_end || (!ALL && a.rstate[r].step > a.rstate[r].target)) {
        a.ncount[s] = 0;
        return;
    }
    const float4* pos = a.buf.pos[*a.parity];
    const float4 pi = pos[s];
    const int code = __float_as_int(pi.w);
    const int cx = cell_x(code), cy = cell_y(code), cz = cell_z(code);
    const int ncx = d.nc[0], ncy = d.nc[1], ncz = d.nc[2];
    const float cut2 = d.cut2;
    const float wx = d.w[0], wy = d.w[1], wz = d.w[2];
    int* out = a.nlist + ((size_t)(s >> 5) * a.nmax) * 32 + (s & 31);
    int count = 0;
    int jb[14], je[14];
#pragma unroll
    for (int st = 0; st < 14; st++) {
        const int ox = st ? c_half[st - 1][0] : 0, oy = st ? c_half[st - 1][1] : 0, oz = st ? c_half[st - 1][2] : 0;
        int nx = cx + ox; nx += nx < 0 ? ncx : 0; nx -= nx >= ncx ? ncx : 0;
        int ny = cy + oy; ny += ny < 0 ? ncy : 0; ny -= ny >= ncy ? ncy : 0;
        int nz = cz + oz; nz += nz < 0 ? ncz : 0; nz -= nz >= ncz ? ncz : 0;
        jb[st] = d.c_begin + __ldg(a.crank + d.c_begin + (nx * ncy + ny) * ncz + nz);
    }
#pragma unroll
    for (int st = 0; st < 14; st++) {
        const int key = jb[st];
        jb[st] = __ldg(a.cstart + key);
        je[st] = __ldg(a.cstart + key + 1);
    }
    jb[0] = s + 1;
#pragma unroll
    for (int st = 0; st < 14; st++) {
        const int ox = st ? c_half[st - 1][0] : 0, oy = st ? c_half[st - 1][1] : 0, oz = st ? c_half[st - 1][2] : 0;
        // (c_i - c_j) w with c_j = c_i + (ox,oy,oz): exact multiples of w
        const float sx = __int2float_rn(-ox) * wx, sy = __int2float_rn(-oy) * wy, sz = __int2float_rn(-oz) * wz;
        const int tagbits = ((1 - ox) * 9 + (1 - oy) * 3 + (1 - oz)) << DPD_CODE_SHIFT;
        const int e = je[st];
        for (int j0 = jb[st]; j0 < e; j0 += 4) {
            float4 pj[4];
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (j0 + u < e) pj[u] = pos[j0 + u];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                if (j0 + u < e) {
                    const float dx = __fadd_rn(__fsub_rn(pi.x, pj[u].x), sx);
                    const float dy = __fadd_rn(__fsub_rn(pi.y, pj[u].y), sy);
                    const float dz = __fadd_rn(__fsub_rn(pi.z, pj[u].z), sz);
                    float r2 = __fmul_rn(dx, dx);
                    r2 = __fmaf_rn(dy, dy, r2);
                    r2 = __fmaf_rn(dz, dz, r2);
                    if (r2 <= cut2) {
                        if (count < a.nmax) out[(size_t)count * 32] = (j0 + u) | tagbits;
                        count++;
                    }
                }
            }
        }
    }
    if (count > a.nmax) {
        atomicOr(&a.rstate[r].status, ST_LIST_OVERFLOW);
        count = a.nmax;
    }
    a.ncount[s] = count;
}

__global__ void __launch_bounds__(256, 4) k_build_nlist(BuildArgs a)
{
    griddep_wait();
    if (!build_on(a)) return;
    build_nlist_slot(a, blockIdx.x * blockDim.x + threadIdx.x);
}

// the same list of the current state, whatever the build flag (on demand, for engines
// whose steps build no list)
__global__ void __launch_bounds__(256, 4) k_build_nlist_now(BuildArgs a)
{
    build_nlist_slot<true>(a, blockIdx.x * blockDim.x + threadIdx.x);
}

// Small grids, where one thread per particle leaves most of the GPU idle and each thread's
// 14 cell ranges form a long serial chain: the same half list with one thread per (slot,
// stencil cell), the 14 threads of a slot appending to its list through an atomic count
// (zeroed by k_permute<true>, which always precedes it).  The same entries and the same
// predicate; their order within a slot's list is the order the atomics drew, and a count
// above nmax is left in place (every reader clamps it) with the overflow flagged.
__global__ void __launch_bounds__(256) k_build_wide(BuildArgs a)
{
    griddep_wait();
    if (!build_on(a)) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 14 * a.P) return;
    const int st = t / a.P, s = t - st * a.P;  // consecutive threads: consecutive slots
    const int r = a.warp_rep[s >> 5];
    const RepDesc& d = a.reps[r];
    if (s >= d.p_end || a.rstate[r].step > a.rstate[r].target) return;  // no list
    const float4* pos = a.buf.pos[*a.parity];
    const float4 pi = pos[s];
    const int code = __float_as_int(pi.w);
    const int ox = st ? c_half[st - 1][0] : 0, oy = st ? c_half[st - 1][1] : 0, oz = st ? c_half[st - 1][2] : 0;
    int nx = cell_x(code) + ox; nx += nx < 0 ? d.nc[0] : 0; nx -= nx >= d.nc[0] ? d.nc[0] : 0;
    int ny = cell_y(code) + oy; ny += ny < 0 ? d.nc[1] : 0; ny -= ny >= d.nc[1] ? d.nc[1] : 0;
    int nz = cell_z(code) + oz; nz += nz < 0 ? d.nc[2] : 0; nz -= nz >= d.nc[2] ? d.nc[2] : 0;
    const int key = d.c_begin + __ldg(a.crank + d.c_begin + (nx * d.nc[1] + ny) * d.nc[2] + nz);
    const int jb = st ? __ldg(a.cstart + key) : s + 1, je = __ldg(a.cstart + key + 1);
    const float sx = __int2float_rn(-ox) * d.w[0], sy = __int2float_rn(-oy) * d.w[1], sz = __int2float_rn(-oz) * d.w[2];
    const int tagbits = ((1 - ox) * 9 + (1 - oy) * 3 + (1 - oz)) << DPD_CODE_SHIFT;
    const float cut2 = d.cut2;
    int* out = a.nlist + ((size_t)(s >> 5) * a.nmax) * 32 + (s & 31);
    for (int j0 = jb; j0 < je; j0 += 4) {
        float4 pj[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (j0 + u < je) pj[u] = pos[j0 + u];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (j0 + u < je) {
                const float dx = __fadd_rn(__fsub_rn(pi.x, pj[u].x), sx);
                const float dy = __fadd_rn(__fsub_rn(pi.y, pj[u].y), sy);
                const float dz = __fadd_rn(__fsub_rn(pi.z, pj[u].z), sz);
                float r2 = __fmul_rn(dx, dx);
                r2 = __fmaf_rn(dy, dy, r2);
                r2 = __fmaf_rn(dz, dz, r2);
                if (r2 <= cut2) {
                    const int k = atomicAdd(a.ncount + s, 1);
                    if (k < a.nmax) out[(size_t)k * 32] = (j0 + u) | tagbits;
                    else atomicOr(&a.rstate[r].status, ST_LIST_OVERFLOW);
                }
            }
        }
    }
}

// The same list with the 14 cell ranges kept in shared memory instead of registers
// ([stencil cell][thread], conflict-free): fewer registers per thread, so more warps per
// SM hide the candidate-gather latency.  Identical entries in identical order.
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_build_nlist_s(BuildArgs a)
{
    __shared__ int2 s_rng[14][256];
    griddep_wait();
    if (!build_on(a)) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int tid = threadIdx.x;
    if (s >= a.P) return;
    const int r = a.warp_rep[s >> 5];
    const RepDesc& d = a.reps[r];
    if (s >= d.p_end || a.rstate[r].step > a.rstate[r].target) {
        a.ncount[s] = 0;
        return;
    }
    const float4* pos = a.buf.pos[*a.parity];
    const float4 pi = pos[s];
    const int code = __float_as_int(pi.w);
    const int cx = cell_x(code), cy = cell_y(code), cz = cell_z(code);
    const int ncx = d.nc[0], ncy = d.nc[1], ncz = d.nc[2];
    for (int st = 0; st < 14; st++) {
        const int ox = st ? c_half[st - 1][0] : 0, oy = st ? c_half[st - 1][1] : 0, oz = st ? c_half[st - 1][2] : 0;
        int nx = cx + ox; nx += nx < 0 ? ncx : 0; nx -= nx >= ncx ? ncx : 0;
        int ny = cy + oy; ny += ny < 0 ? ncy : 0; ny -= ny >= ncy ? ncy : 0;
        int nz = cz + oz; nz += nz < 0 ? ncz : 0; nz -= nz >= ncz ? ncz : 0;
        const int key = d.c_begin + __ldg(a.crank + d.c_begin + (nx * ncy + ny) * ncz + nz);
        s_rng[st][tid] = make_int2(st ? __ldg(a.cstart + key) : s + 1, __ldg(a.cstart + key + 1));
    }
    const float cut2 = d.cut2;
    const float wx = d.w[0], wy = d.w[1], wz = d.w[2];
    int* out = a.nlist + ((size_t)(s >> 5) * a.nmax) * 32 + (s & 31);
    int count = 0;
    for (int st = 0; st < 14; st++) {
        const int ox = st ? c_half[st - 1][0] : 0, oy = st ? c_half[st - 1][1] : 0, oz = st ? c_half[st - 1][2] : 0;
        const float sx = __int2float_rn(-ox) * wx, sy = __int2float_rn(-oy) * wy, sz = __int2float_rn(-oz) * wz;
        const int tagbits = ((1 - ox) * 9 + (1 - oy) * 3 + (1 - oz)) << DPD_CODE_SHIFT;
        const int2 rg = s_rng[st][tid];
        for (int j0 = rg.x; j0 < rg.y; j0 += 4) {
            float4 pj[4];
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (j0 + u < rg.y) pj[u] = pos[j0 + u];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                if (j0 + u < rg.y) {
                    const float dx = __fadd_rn(__fsub_rn(pi.x, pj[u].x), sx);
                    const float dy = __fadd_rn(__fsub_rn(pi.y, pj[u].y), sy);
                    const float dz = __fadd_rn(__fsub_rn(pi.z, pj[u].z), sz);
                    float r2 = __fmul_rn(dx, dx);
                    r2 = __fmaf_rn(dy, dy, r2);
                    r2 = __fmaf_rn(dz, dz, r2);
                    if (r2 <= cut2) {
                        if (count < a.nmax) out[(size_t)count * 32] = (j0 + u) | tagbits;
                        count++;
                    }
                }
            }
        }
    }
    if (count > a.nmax) {
        atomicOr(&a.rstate[r].status, ST_LIST_OVERFLOW);
        count = a.nmax;
    }
    a.ncount[s] = count;
}

// ---------------------------------------------------------------------------------
// The list build over x-y columns (build variant 5).  The half stencil with x outermost,
// (ox > 0) | (ox == 0 & oy > 0) | (ox == 0 & oy == 0 & oz > 0), is the rest of the own
// cell, cell z+1 of the own column, and cells z-1..z+1 of the columns (x, y+1),
// (x+1, y-1), (x+1, y), (x+1, y+1).  When the cells of a column are consecutive in the
// cell order (cell order 0, linear with z fastest, or 2, columns in Morton order), each of
// these five groups is one contiguous slot range, walked 4 slots at a time with the z
// shift of each slot taken from the range's two cell boundaries: five ranges of about
// nine candidates in place of fourteen cells of about three, so fewer idle lanes at the
// ends of short ranges.  At the ends of a column (z = 0 or z = nc-1) the cell across the
// periodic boundary is not next to the other two: the group is its two contiguous cells
// plus that one cell, walked after the five ranges.  A particle whose groups are not
// contiguous otherwise (every particle under the Morton order) walks the same 13 cells one
// at a time.  The predicate and the pair set are those of the other builds (the half list
// of src/force/neigh_list.cu:322-393); which particle of a pair holds it follows this
// stencil's orientation.
__constant__ int8_t c_half_x[13][3] = {
    {0, 0, 1}, {0, 1, -1}, {0, 1, 0}, {0, 1, 1}, {1, -1, -1}, {1, -1, 0}, {1, -1, 1},
    {1, 0, -1}, {1, 0, 0}, {1, 0, 1}, {1, 1, -1}, {1, 1, 0}, {1, 1, 1}};

// slots [jb, je) of one column group: cell z-1 below b1, cell z in [b1, b2), cell z+1
// from b2; sx, sy the group's shifts (c_i - c_j) w in x and y, cxy its 9 (dcx+1) + 3 (dcy+1)
__device__ __forceinline__ void column_walk(const float4* __restrict__ pos, const float4 pi, const int jb,
                                            const int je, const int b1, const int b2, const float sx,
                                            const float sy, const float wz, const int cxy, const float cut2,
                                            int* out, const int nmax, int& count)
{
    for (int j0 = jb; j0 < je; j0 += 4) {
        float4 pj[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (j0 + u < je) pj[u] = pos[j0 + u];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int j = j0 + u;
            if (j < je) {
                const bool below = j < b1, mid = j < b2;
                const float sz = below ? wz : (mid ? 0.0f : -wz);
                const float dx = __fadd_rn(__fsub_rn(pi.x, pj[u].x), sx);
                const float dy = __fadd_rn(__fsub_rn(pi.y, pj[u].y), sy);
                const float dz = __fadd_rn(__fsub_rn(pi.z, pj[u].z), sz);
                float r2 = __fmul_rn(dx, dx);
                r2 = __fmaf_rn(dy, dy, r2);
                r2 = __fmaf_rn(dz, dz, r2);
                if (r2 <= cut2) {
                    if (count < nmax)
                        out[(size_t)count * 32] = j | ((cxy + (below ? 2 : (mid ? 1 : 0))) << DPD_CODE_SHIFT);
                    count++;
                }
            }
        }
    }
}

__global__ void __launch_bounds__(256, 4) k_build_cols(BuildArgs a)
{
    griddep_wait();
    if (!build_on(a)) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.P) return;
    const int r = a.warp_rep[s >> 5];
    const RepDesc& d = a.reps[r];
    if (s >= d.p_end || a.rstate[r].step > a.rstate[r].target) {
        a.ncount[s] = 0;
        return;
    }
    const float4* pos = a.buf.pos[*a.parity];
    const float4 pi = pos[s];
    const int code = __float_as_int(pi.w);
    const int cx = cell_x(code), cy = cell_y(code), cz = cell_z(code);
    const int ncx = d.nc[0], ncy = d.nc[1], ncz = d.nc[2];
    const float cut2 = d.cut2;
    const float wx = d.w[0], wy = d.w[1], wz = d.w[2];
    const int* crank = a.crank + d.c_begin;
    const int* cstart = a.cstart + d.c_begin;
    int* out = a.nlist + ((size_t)(s >> 5) * a.nmax) * 32 + (s & 31);
    int count = 0;
    // z = 0: cell z-1 lies across the periodic boundary; z = nc-1: cell z+1 does
    const bool wlo = cz == 0, whi = cz == ncz - 1;
    const int zm = wlo ? ncz - 1 : cz - 1, zp = whi ? 0 : cz + 1;
    // ranks of cells z-1, z, z+1 of the five columns (group 0: the own column, whose
    // z-1 cell is not in the stencil)
    int rl[5], rm[5], rh[5];
#pragma unroll
    for (int g = 0; g < 5; g++) {
        const int ox = g < 2 ? 0 : 1, oy = g == 0 ? 0 : (g == 1 ? 1 : g - 3);
        int nx = cx + ox; nx -= nx >= ncx ? ncx : 0;
        int ny = cy + oy; ny += ny < 0 ? ncy : 0; ny -= ny >= ncy ? ncy : 0;
        const int base = (nx * ncy + ny) * ncz;
        rl[g] = g ? __ldg(crank + base + zm) : 0;
        rm[g] = __ldg(crank + base + cz);
        rh[g] = __ldg(crank + base + zp);
    }
    // the cells of each group on this side of the periodic boundary are consecutive
    bool contiguous = true;
#pragma unroll
    for (int g = 0; g < 5; g++)
        contiguous &= (whi || rh[g] == rm[g] + 1) && (wlo || g == 0 || rm[g] == rl[g] + 1);
    if (contiguous) {
        // main range of a group: from cell z-1 (cell z at z = 0) to the end of cell z+1
        // (of cell z at z = nc-1); the end of cell z is the start of cell z+1 in between
        int jb[5], b1[5], b2[5], je[5];
#pragma unroll
        for (int g = 0; g < 5; g++) {
            jb[g] = g ? __ldg(cstart + (wlo ? rm[g] : rl[g])) : s + 1;
            b1[g] = g ? __ldg(cstart + rm[g]) : s + 1;
            b2[g] = __ldg(cstart + rm[g] + 1);
            je[g] = __ldg(cstart + (whi ? rm[g] : rh[g]) + 1);
        }
#pragma unroll
        for (int g = 0; g < 5; g++) {
            const int ox = g < 2 ? 0 : 1, oy = g == 0 ? 0 : (g == 1 ? 1 : g - 3);
            column_walk(pos, pi, jb[g], je[g], b1[g], b2[g], __int2float_rn(-ox) * wx, __int2float_rn(-oy) * wy,
                        wz, (1 - ox) * 9 + (1 - oy) * 3, cut2, out, a.nmax, count);
        }
        if (wlo || whi) {
            // the cell across the boundary of each group: z-1 below, z+1 above both bounds
#pragma unroll 1
            for (int g = wlo ? 1 : 0; g < 5; g++) {
                const int ox = g < 2 ? 0 : 1, oy = g == 0 ? 0 : (g == 1 ? 1 : g - 3);
                int nx = cx + ox; nx -= nx >= ncx ? ncx : 0;
                int ny = cy + oy; ny += ny < 0 ? ncy : 0; ny -= ny >= ncy ? ncy : 0;
                const int key = __ldg(crank + (nx * ncy + ny) * ncz + (wlo ? zm : zp));
                const int b = __ldg(cstart + key), e = __ldg(cstart + key + 1);
                column_walk(pos, pi, b, e, wlo ? e : b, wlo ? e : b, __int2float_rn(-ox) * wx,
                            __int2float_rn(-oy) * wy, wz, (1 - ox) * 9 + (1 - oy) * 3, cut2, out, a.nmax, count);
            }
        }
    } else {
#pragma unroll 1
        for (int st = 0; st < 14; st++) {
            const int ox = st ? c_half_x[st - 1][0] : 0, oy = st ? c_half_x[st - 1][1] : 0,
                      oz = st ? c_half_x[st - 1][2] : 0;
            int nx = cx + ox; nx -= nx >= ncx ? ncx : 0;
            int ny = cy + oy; ny += ny < 0 ? ncy : 0; ny -= ny >= ncy ? ncy : 0;
            int nz = cz + oz; nz += nz < 0 ? ncz : 0; nz -= nz >= ncz ? ncz : 0;
            const int key = __ldg(crank + (nx * ncy + ny) * ncz + nz);
            const int b = st ? __ldg(cstart + key) : s + 1, e = __ldg(cstart + key + 1);
            // the whole cell on one side of both boundaries: below b1 for z-1, in [b1, b2)
            // for z, from b2 for z+1
            column_walk(pos, pi, b, e, oz < 0 ? e : b, oz > 0 ? b : e, __int2float_rn(-ox) * wx,
                        __int2float_rn(-oy) * wy, wz, (1 - ox) * 9 + (1 - oy) * 3, cut2, out, a.nmax, count);
        }
    }
    if (count > a.nmax) {
        atomicOr(&a.rstate[r].status, ST_LIST_OVERFLOW);
        count = a.nmax;
    }
    a.ncount[s] = count;
}
