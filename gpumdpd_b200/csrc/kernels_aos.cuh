// kernels_aos.cuh -- the in-loop drop-in for Pair::compute_force on the reference's own
// device buffers (AoS numtyp[3N] positions/velocities/forces, int[N] ids and types, atom
// index = id - 1 as src/system/read_data.cu:265 lays them out).  The engine keeps its
// cell-sorted copy and half list; each call maps the AoS state into it by tag, rebuilds
// the list when a particle moved more than skin/2, evaluates the pair force and writes
// the result back in AoS order.
#pragma once
#include "kernels_step.cuh"

// AoS -> engine slots.  Positions become offsets relative to the slot's current cell
// (nearest periodic image of the cell), velocities and the tag/type word are replaced.
__global__ void k_aos_in(StepArgs a, const float* __restrict__ xin, const float* __restrict__ vin,
                         const int* __restrict__ id, const int* __restrict__ type, int n, uint32_t step,
                         int force_build)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const RepDesc& d = a.reps[0];
    if (i == 0) {
        RepState st = a.rstate[0];
        st.step = step;
        st.target = step;
        st.zero_pending = 1;
        a.rstate[0] = st;
        if (force_build) a.build_flag[(*a.phase) & 1] = 1;
    }
    if (i >= n) return;
    const int tag = id[i];
    const int ty = type[i];
    if (tag < 1 || tag > d.n_real || ty < 1 || ty > d.ntypes) {
        atomicOr(&a.rstate[0].status, ST_BAD_INPUT);
        return;
    }
    const int s = a.tag2idx[d.tag_base + tag - 1];
    if (s < d.p_begin || s >= d.p_end) {
        atomicOr(&a.rstate[0].status, ST_BAD_INPUT);
        return;
    }
    const int par = *a.parity;
    const float4 p = a.buf.pos[par][s];
    const int code = __float_as_int(p.w);
    const int c[3] = {cell_x(code), cell_y(code), cell_z(code)};
    float o[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float xa = xin[3 * i + k] - (float)d.lo[k];
        float q = xa - __int2float_rn(c[k]) * d.w[k];
        q -= d.L[k] * rintf((q - 0.5f * d.w[k]) / d.L[k]);
        o[k] = q;
    }
    const float4 pn = make_float4(o[0], o[1], o[2], p.w);
    a.buf.pos[par][s] = pn;
    a.buf.vel[par][s] = make_float4(vin[3 * i], vin[3 * i + 1], vin[3 * i + 2],
                                    __int_as_float((tag << DPD_TYPE_BITS) | (ty - 1)));
    a.force4[s] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (d.style == 1) a.rho[s] = 0.0f;
    // displacement since the last build (same cell): src/force/neigh_list.cu:483-514
    const float4 q = a.last4[s];
    const float dx = pn.x - q.x, dy = pn.y - q.y, dz = pn.z - q.z;
    const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
    if (d.skin_zero || !(r2 < d.hskin2)) a.build_flag[(*a.phase) & 1] = 1;
}

// Pair force with per-atom PE and virial (the reference's log variants,
// src/force/pair_dpd.cu:240-419 and src/force/pair_mdpd.cu:346-537): per pair, DPD adds
// 0.5*ppe to each atom (ppe = 0.5 A rc w^2); mDPD adds 0.5 u_c + u_d,i to i and
// 0.5 u_c + u_d,j to j; both atoms get 0.5 r (x) F.  Thread per particle, j-side atomics.
template <int STYLE>
__global__ void __launch_bounds__(256) k_pair_peratom(StepArgs a, float* pe_slot, float* vir_slot)
{
    __shared__ float4 tab[8][27];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.P) return;
    const RepDesc& d = a.reps[0];
    fill_shift(tab[warp], d, lane);
    __syncwarp();
    if (s >= d.p_end) return;
    const uint32_t step = a.rstate[0].step;
    const int par = *a.parity;
    const float4* pos = a.buf.pos[par];
    const float4* vel = a.buf.vel[par];
    const float4 pi = pos[s];
    const float4 vi = vel[s];
    const float rho_i = STYLE == 1 ? a.rho[s] : 0.0f;
    const float4* crow = a.coeff + d.coeff_off + type0_of(vi.w) * d.ntypes * 3;
    const int n = min(a.ncount[s], a.nmax);
    const int* lst = a.nlist + ((size_t)(s >> 5) * a.nmax) * 32 + lane;
    float fx = 0, fy = 0, fz = 0, pe = 0, v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0, v5 = 0;
    double unused[8];
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
        if (!pair_force<STYLE, false>(crow, r2, dx, dy, dz, vi, vj, rho_i, rho_j, d.seed, step, gx, gy, gz, unused))
            continue;
        const int tj = type0_of(vj.w);
        const float4 c1 = __ldg(crow + tj * 3 + 1);
        const float r = sqrtf(r2);
        const float wc = 1.0f - r * c1.x;
        float pei, pej;
        if (STYLE == 0) {
            pei = pej = 0.5f * (c1.y * wc * wc);
        } else {
            const float4 c2 = __ldg(crow + tj * 3 + 2);
            const float wd = fmaxf(1.0f - r * c1.w, 0.0f);
            const float uc = c1.y * wc * wc;
            pei = 0.5f * uc + c2.y * rho_i * wd * wd;
            pej = 0.5f * uc + c2.y * rho_j * wd * wd;
        }
        const float w0 = 0.5f * dx * gx, w1 = 0.5f * dx * gy, w2 = 0.5f * dx * gz;
        const float w3 = 0.5f * dy * gy, w4 = 0.5f * dy * gz, w5 = 0.5f * dz * gz;
        fx += gx; fy += gy; fz += gz;
        pe += pei;
        v0 += w0; v1 += w1; v2 += w2; v3 += w3; v4 += w4; v5 += w5;
        atomicAdd(&a.force4[j], make_float4(-gx, -gy, -gz, 0.0f));
        atomicAdd(&pe_slot[j], pej);
        atomicAdd(&vir_slot[6 * (size_t)j + 0], w0);
        atomicAdd(&vir_slot[6 * (size_t)j + 1], w1);
        atomicAdd(&vir_slot[6 * (size_t)j + 2], w2);
        atomicAdd(&vir_slot[6 * (size_t)j + 3], w3);
        atomicAdd(&vir_slot[6 * (size_t)j + 4], w4);
        atomicAdd(&vir_slot[6 * (size_t)j + 5], w5);
    }
    atomicAdd(&a.force4[s], make_float4(fx, fy, fz, 0.0f));
    atomicAdd(&pe_slot[s], pe);
    atomicAdd(&vir_slot[6 * (size_t)s + 0], v0);
    atomicAdd(&vir_slot[6 * (size_t)s + 1], v1);
    atomicAdd(&vir_slot[6 * (size_t)s + 2], v2);
    atomicAdd(&vir_slot[6 * (size_t)s + 3], v3);
    atomicAdd(&vir_slot[6 * (size_t)s + 4], v4);
    atomicAdd(&vir_slot[6 * (size_t)s + 5], v5);
}

// engine slots -> AoS (index = tag - 1); clears the slot accumulators for the next call
__global__ void k_aos_out(StepArgs a, float* fout, float* pe_out, float* vir_out, float* pe_slot,
                          float* vir_slot)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.P) return;
    const RepDesc& d = a.reps[0];
    if (s >= d.p_end) return;
    const float4 v = a.buf.vel[*a.parity][s];
    const int i = tag_of(v.w) - 1;
    if (i < 0 || i >= d.n_real) return;
    const float4 f = a.force4[s];
    fout[3 * (size_t)i] = f.x;
    fout[3 * (size_t)i + 1] = f.y;
    fout[3 * (size_t)i + 2] = f.z;
    if (pe_out && pe_slot) {
        pe_out[i] = pe_slot[s];
        pe_slot[s] = 0.0f;
    }
    if (vir_out && vir_slot) {
#pragma unroll
        for (int c = 0; c < 6; c++) {
            vir_out[6 * (size_t)i + c] = vir_slot[6 * (size_t)s + c];
            vir_slot[6 * (size_t)s + c] = 0.0f;
        }
    }
}

__global__ void k_aos_done(int* build_flag, const uint32_t* phase)
{
    build_flag[(*phase) & 1] = 0;
}

// ---------------------------------------------------------------------------------
// Bond::compute_force on the reference's AoS buffers (src/force/bond_harmonic.cu:167-402):
// one thread per entry of the bond list {type, id_i, id_j}; displacement x_i - x_j with
// the reference's minimum image (d -= L((d >= L/2) - (d < -L/2))), harmonic E = k(r-r0)^2,
// F_i = -2k(r-r0)/r d, or this engine's FENE; forces added to both atoms; on log steps the
// bond's energy (one value per bond, as the reference's d_bond_pe) and half the virial
// r_a F_b to each atom.
struct AosBondArgs {
    float L[3], hL[3];
    int style;       // 1 harmonic, 2 fene
    int ntypes;
    const float4* coef;  // per bond type: harmonic {k, r0}; fene {K, R0, eps, sigma}
    int n_atoms;
    int* status;     // device int: bit ST_BOND_MISSING (an id outside the system), ST_FENE_BROKEN
};

template <bool LOG>
__global__ void k_bond_aos(AosBondArgs b, const float* __restrict__ pos, const int* __restrict__ bl, int nb,
                           float* force, float* bond_pe, float* virial)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nb) return;
    const int ty = bl[3 * q], ia = bl[3 * q + 1] - 1, ja = bl[3 * q + 2] - 1;
    if (ty < 1 || ty > b.ntypes || ia < 0 || ia >= b.n_atoms || ja < 0 || ja >= b.n_atoms) {
        atomicOr(b.status, ST_BOND_MISSING);
        return;
    }
    float d[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float x = pos[3 * ia + k] - pos[3 * ja + k];
        x = x - b.L[k] * (float)((x >= b.hL[k]) - (x < -b.hL[k]));
        d[k] = x;
    }
    const float r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const float4 c = b.coef[ty - 1];
    float fbond = 0.0f, e = 0.0f;
    if (b.style == 1) {
        const float r = sqrtf(r2);
        fbond = r > 0.0f ? -2.0f * c.x * (r - c.y) / r : 0.0f;
        e = c.x * (r - c.y) * (r - c.y);
    } else {
        float rr = r2 / (c.y * c.y);
        if (rr >= 1.0f) {
            atomicOr(b.status, ST_FENE_BROKEN);
            rr = 0.999f;
        }
        fbond = -c.x / (1.0f - rr);
        e = -0.5f * c.x * c.y * c.y * logf(1.0f - rr);
        if (c.z > 0.0f && r2 < 1.2599210498948732f * c.w * c.w) {
            const float sr2 = c.w * c.w / r2;
            const float sr6 = sr2 * sr2 * sr2;
            fbond += 48.0f * c.z * sr6 * (sr6 - 0.5f) / r2;
            e += 4.0f * c.z * sr6 * (sr6 - 1.0f) + c.z;
        }
    }
    const float f[3] = {d[0] * fbond, d[1] * fbond, d[2] * fbond};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        atomicAdd(force + 3 * ia + k, f[k]);
        atomicAdd(force + 3 * ja + k, -f[k]);
    }
    if (LOG) {
        if (bond_pe) bond_pe[q] = e;
        if (virial) {
            const float v6[6] = {0.5f * d[0] * f[0], 0.5f * d[0] * f[1], 0.5f * d[0] * f[2],
                                 0.5f * d[1] * f[1], 0.5f * d[1] * f[2], 0.5f * d[2] * f[2]};
#pragma unroll
            for (int k = 0; k < 6; k++) {
                atomicAdd(virial + 6 * ia + k, v6[k]);
                atomicAdd(virial + 6 * ja + k, v6[k]);
            }
        }
    }
}

// fix nve on the reference's AoS buffers (src/fix/fix_nve.cu:30-152), one thread per atom
// of the group's index list: PHASE 0 the initial half kick v += dt/2 f/m, the drift
// x += dt v wrapped into [lo, hi) and the unwrapped position uw += dt v; PHASE 1 the
// final half kick.  The same FP32 operations as the reference's kernels.
struct AosNveArgs {
    float dt;
    float lo[3], hi[3], L[3];
    int ntypes;
    const float* mass;  // per type
    int n_atoms;
    int* status;        // device int: bit ST_BAD_INPUT (an index or type outside the system)
};

template <int PHASE>
__global__ void k_nve_aos(AosNveArgs b, const int* __restrict__ group, int ng, const int* __restrict__ type,
                          float* pos, float* uwpos, float* vel, const float* __restrict__ force)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ng) return;
    const int i = group[q];
    if (i < 0 || i >= b.n_atoms || type[i] < 1 || type[i] > b.ntypes) {
        atomicOr(b.status, ST_BAD_INPUT);
        return;
    }
    const float dtm = (0.5f * b.dt) * (1.0f / b.mass[type[i] - 1]);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float v = __fmaf_rn(dtm, force[3 * i + k], vel[3 * i + k]);
        vel[3 * i + k] = v;
        if (PHASE == 0) {
            float p = __fmaf_rn(b.dt, v, pos[3 * i + k]);
            for (int it = 0; it < 64 && (p >= b.hi[k] || p < b.lo[k]); it++)
                p -= b.L[k] * (float)((p >= b.hi[k]) - (p < b.lo[k]));
            pos[3 * i + k] = p;
            if (uwpos) uwpos[3 * i + k] = __fmaf_rn(b.dt, v, uwpos[3 * i + k]);
        }
    }
}
