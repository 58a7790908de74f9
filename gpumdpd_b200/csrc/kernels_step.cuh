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
    float4* pos4;
    float4* vel4;
    float4* force4;
    float* rho;
    int4* img;
    const float4* last4;
    const int2* bonds;
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
};

__device__ __forceinline__ bool rep_active(const RepState& st) { return st.step <= st.target; }

// ---------------------------------------------------------------------------------
// displacement between two slots (cell-offset representation)
template <bool SMALL>
__device__ __forceinline__ void disp3(const RepDesc& d, int ci, float4 pi, float4 pj, float& dx,
                                      float& dy, float& dz)
{
    const int cj = __float_as_int(pj.w);
    dx = disp1<SMALL>(cell_x(ci), cell_x(cj), pi.x, pj.x, d.nc[0], d.w[0], d.L[0]);
    dy = disp1<SMALL>(cell_y(ci), cell_y(cj), pi.y, pj.y, d.nc[1], d.w[1], d.L[1]);
    dz = disp1<SMALL>(cell_z(ci), cell_z(cj), pi.z, pj.z, d.nc[2], d.w[2], d.L[2]);
}

// ---------------------------------------------------------------------------------
// mDPD local density, src/force/pair_mdpd.cu:219-300: rho_i = sum_j 15/(2 pi rd^3)
// max(0, 1-r/rd)^2 over the half list, both sides.
template <bool SMALL>
__global__ void __launch_bounds__(256) k_density(StepArgs a)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.P) return;
    const int r = a.warp_rep[s >> 5];
    const RepDesc& d = a.reps[r];
    if (!rep_active(a.rstate[r]) || s >= d.p_end) return;
    const float4 pi = a.pos4[s];
    const int ci = __float_as_int(pi.w);
    const int ti = type0_of(a.vel4[s].w);
    const float4* crow = a.coeff + d.coeff_off + ti * d.ntypes * 3;
    const int n = min(a.ncount[s], a.nmax);
    const int* lst = a.nlist + ((size_t)(s >> 5) * a.nmax) * 32 + (s & 31);
    float rho_i = 0.0f;
    for (int k = 0; k < n; k++) {
        const int j = __ldg(lst + (size_t)k * 32);
        const float4 pj = __ldg(a.pos4 + j);
        float dx, dy, dz;
        disp3<SMALL>(d, ci, pi, pj, dx, dy, dz);
        const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
        const int tj = type0_of(__ldg(&a.vel4[j].w));
        const float4 c1 = __ldg(crow + tj * 3 + 1);
        const float4 c2 = __ldg(crow + tj * 3 + 2);
        if (r2 < c2.x) {
            const float rr = r2 * rsqrtf(fmaxf(r2, 1e-30f));
            const float wd = fmaxf(1.0f - rr * c1.w, 0.0f);
            const float add = c2.z * wd * wd;
            rho_i += add;
            atomicAdd(&a.rho[j], add);
        }
    }
    atomicAdd(&a.rho[s], rho_i);
}

// ---------------------------------------------------------------------------------
// Pair force over the half list with the Saru random force; j-side by vector atomics.
// DPD: src/force/pair_dpd.cu:468-558; mDPD: src/force/pair_mdpd.cu:587-682.
// LOG adds PE and the pair virial (src/force/pair_dpd.cu:366-383) in FP64.
template <bool LOG, int STYLE, bool SMALL>
__device__ __forceinline__ void pair_loop(const StepArgs& a, const RepDesc& d, const int s,
                                          const float4 pi, const float4 vi, const float rho_i,
                                          const uint32_t step, float& fx, float& fy, float& fz,
                                          double (&accv)[8])
{
    const int ci = __float_as_int(pi.w);
    const int tagi = tag_of(vi.w);
    const int ti = type0_of(vi.w);
    const float4* crow = a.coeff + d.coeff_off + ti * d.ntypes * 3;
    const int n = min(a.ncount[s], a.nmax);
    const int* lst = a.nlist + ((size_t)(s >> 5) * a.nmax) * 32 + (s & 31);
    const float rcmax2 = d.rcmax2;
    for (int k = 0; k < n; k++) {
        const int j = __ldg(lst + (size_t)k * 32);
        const float4 pj = __ldg(a.pos4 + j);
        float dx, dy, dz;
        disp3<SMALL>(d, ci, pi, pj, dx, dy, dz);
        const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
        if (r2 > rcmax2) continue;
        const float4 vj = __ldg(a.vel4 + j);
        const int tj = type0_of(vj.w);
        const float4 c0 = __ldg(crow + tj * 3 + 0);
        if (!(r2 <= c0.w)) continue;
        const float rinv = rsqrtf(r2);
        const float r = r2 * rinv;
        if (r < 1.0e-10f) continue;
        const float4 c1 = __ldg(crow + tj * 3 + 1);
        const float dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
        const float dot = dx * dvx + dy * dvy + dz * dvz;
        const float wc = 1.0f - r * c1.x;
        const int tagj = tag_of(vj.w);
        const float th = saru_theta((uint32_t)min(tagi, tagj), (uint32_t)max(tagi, tagj), d.seed, step);
        float fpair = c0.x * wc;
        float wd = 0.0f, rho_j = 0.0f;
        float4 c2;
        if (STYLE == 1) {
            c2 = __ldg(crow + tj * 3 + 2);
            wd = fmaxf(1.0f - r * c1.w, 0.0f);
            rho_j = __ldg(a.rho + j);
            fpair += c1.z * (rho_i + rho_j) * wd;
        }
        fpair -= c0.y * wc * wc * dot * rinv;
        fpair += c0.z * wc * th;
        fpair *= rinv;
        const float ffx = dx * fpair, ffy = dy * fpair, ffz = dz * fpair;
        fx += ffx;
        fy += ffy;
        fz += ffz;
        atomicAdd(&a.force4[j], make_float4(-ffx, -ffy, -ffz, 0.0f));
        if (LOG) {
            double pe = (double)(c1.y * wc * wc);
            if (STYLE == 1) pe += (double)(c2.y * (rho_i + rho_j) * wd * wd);
            accv[0] += pe;
            accv[2] += (double)dx * ffx;
            accv[3] += (double)dx * ffy;
            accv[4] += (double)dx * ffz;
            accv[5] += (double)dy * ffy;
            accv[6] += (double)dy * ffz;
            accv[7] += (double)dz * ffz;
        }
    }
}

// Bond forces computed by both partners (each takes its own side; energy and virial
// halved), so bonds need no atomics.  Harmonic: src/force/bond_harmonic.cu:208-268
// (E = k (r-r0)^2, F_i = -2k(r-r0)/r d).  FENE: -0.5 K R0^2 ln(1-(r/R0)^2) + WCA.
template <bool LOG, bool SMALL>
__device__ __forceinline__ void bond_loop(const StepArgs& a, const RepDesc& d, const int r_idx,
                                          const int s, const float4 pi, float& fx, float& fy,
                                          float& fz, double (&accv)[8])
{
    const int ci = __float_as_int(pi.w);
    for (int b = 0; b < a.maxb; b++) {
        const int2 bp = a.bonds[(size_t)b * a.P + s];
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
        const float4 pj = a.pos4[j];
        float dx, dy, dz;
        disp3<true>(d, ci, pi, pj, dx, dy, dz);
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

template <int STYLE, bool SMALL, bool BONDS>
__global__ void __launch_bounds__(256) k_pair(StepArgs a)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    int r = -1;
    bool work = false, log = false;
    uint32_t step = 0;
    if (s < a.P) {
        r = a.warp_rep[s >> 5];
        const RepState st = a.rstate[r];
        const RepDesc& d = a.reps[r];
        work = rep_active(st) && s < d.p_end;
        step = st.step;
        log = rep_active(st) && (step % (uint32_t)d.log_f) == 0u;
    }
    double accv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (work) {
        const RepDesc& d = a.reps[r];
        const float4 pi = a.pos4[s];
        const float4 vi = a.vel4[s];
        const float rho_i = STYLE == 1 ? a.rho[s] : 0.0f;
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        if (log) {
            pair_loop<true, STYLE, SMALL>(a, d, s, pi, vi, rho_i, step, fx, fy, fz, accv);
            if (BONDS) bond_loop<true, SMALL>(a, d, r, s, pi, fx, fy, fz, accv);
        } else {
            pair_loop<false, STYLE, SMALL>(a, d, s, pi, vi, rho_i, step, fx, fy, fz, accv);
            if (BONDS) bond_loop<false, SMALL>(a, d, r, s, pi, fx, fy, fz, accv);
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
// Velocity Verlet, src/fix/fix_nve.cu:30-152, fused: final half kick of step n (and
// the thermo sums of step n), then initial half kick + drift of step n+1, cell
// re-wrap with image counters, displacement check for the next list build
// (src/force/neigh_list.cu:483-514), and zeroing of the force accumulators.
__global__ void __launch_bounds__(256) k_integrate(StepArgs a)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    int r = -1;
    bool work = false, log = false;
    double accv[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (s < a.P) {
        r = a.warp_rep[s >> 5];
        const RepState st = a.rstate[r];
        const RepDesc& d = a.reps[r];
        const bool active = a.mode == 1 ? st.step <= st.target : rep_active(st);
        work = active && s < d.p_end;
        bool fin = a.mode == 0 && !st.zero_pending;
        log = a.mode == 0 && active && (st.step % (uint32_t)d.log_f) == 0u;
        bool init = a.mode == 1 ? true : st.step < st.target;
        uint32_t next = a.mode == 1 ? st.step : st.step + 1u;
        bool check = init && (next % (uint32_t)d.nl_f) == 0u;
        if (work) {
            float4 v = a.vel4[s];
            float4 f = a.force4[s];
            float4 p = a.pos4[s];
            const int t0 = type0_of(v.w);
            const float2 m = __ldg(a.mass + d.mass_off + t0);
            const bool integ = (d.integ_mask >> t0) & 1u;
            const float dtm = (0.5f * d.dt) * m.y;
            if (fin && integ) {
                v.x = __fmaf_rn(dtm, f.x, v.x);
                v.y = __fmaf_rn(dtm, f.y, v.y);
                v.z = __fmaf_rn(dtm, f.z, v.z);
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
            if (init) {
                int code = __float_as_int(p.w);
                if (integ) {
                    v.x = __fmaf_rn(dtm, f.x, v.x);
                    v.y = __fmaf_rn(dtm, f.y, v.y);
                    v.z = __fmaf_rn(dtm, f.z, v.z);
                    float o[3] = {__fmaf_rn(d.dt, v.x, p.x), __fmaf_rn(d.dt, v.y, p.y),
                                  __fmaf_rn(d.dt, v.z, p.z)};
                    int c[3] = {cell_x(code), cell_y(code), cell_z(code)};
                    int dimg[3] = {0, 0, 0};
                    bool moved = false;
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        if (!(o[k] >= 0.0f && o[k] < d.w[k])) {
                            if (!isfinite(o[k])) {
                                atomicOr(&a.rstate[r].status, ST_NONFINITE);
                                o[k] = 0.0f;
                                continue;
                            }
                            float q = floorf(o[k] * d.inv_w[k]);
                            q = fminf(fmaxf(q, -1.0e6f), 1.0e6f);
                            o[k] = __fmaf_rn(-q, d.w[k], o[k]);
                            int cc = c[k] + (int)q;
                            int nc = d.nc[k];
                            int wrap = cc >= 0 ? cc / nc : -((-cc + nc - 1) / nc);
                            cc -= wrap * nc;
                            dimg[k] = wrap;
                            c[k] = cc;
                            if (o[k] >= d.w[k]) o[k] = __int_as_float(__float_as_int(d.w[k]) - 1);
                            if (o[k] < 0.0f) o[k] = 0.0f;
                            moved = true;
                        }
                    }
                    if (!isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z))
                        atomicOr(&a.rstate[r].status, ST_NONFINITE);
                    if (moved) code = cell_pack(c[0], c[1], c[2]);
                    if (dimg[0] | dimg[1] | dimg[2]) {
                        int4 im = a.img[s];
                        im.x += dimg[0];
                        im.y += dimg[1];
                        im.z += dimg[2];
                        a.img[s] = im;
                    }
                    p = make_float4(o[0], o[1], o[2], __int_as_float(code));
                    a.pos4[s] = p;
                }
                if (check) {
                    bool need = d.skin_zero != 0;
                    if (!need) {
                        const float4 q = a.last4[s];
                        float dx, dy, dz;
                        disp3<true>(d, code, p, q, dx, dy, dz);
                        const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
                        need = r2 >= d.hskin2;
                    }
                    if (need) {
                        uint32_t ph = *a.phase + (a.mode == 1 ? 0u : 1u);
                        a.build_flag[ph & 1] = 1;
                    }
                }
                a.force4[s] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (d.style == 1) a.rho[s] = 0.0f;
            }
            a.vel4[s] = v;
        }
    }
    if (a.mode == 0 && __syncthreads_or(log)) {
        const int fields[10] = {ACC_KE, ACC_KIN + 0, ACC_KIN + 1, ACC_KIN + 2, ACC_KIN + 3,
                                ACC_KIN + 4, ACC_KIN + 5, ACC_MOM + 0, ACC_MOM + 1, ACC_MOM + 2};
        acc_flush<10>(accv, fields, log ? r : -1, a.acc);
    }
}

// ---------------------------------------------------------------------------------
// End of step bookkeeping, one thread per replica: thermo row of a logged step
// (src/compute/thermo.cu:274-306, 479-520), step counter, build flag of this phase.
__global__ void k_advance(StepArgs a)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < a.nrep) {
        RepState st = a.rstate[r];
        const RepDesc& d = a.reps[r];
        if (rep_active(st)) {
            if ((st.step % (uint32_t)d.log_f) == 0u) {
                double sum[DPD_NACC];
                for (int k = 0; k < DPD_NACC; k++) sum[k] = 0.0;
                double* base = a.acc + (size_t)r * DPD_ACC_SLOTS * DPD_NACC;
                for (int sl = 0; sl < DPD_ACC_SLOTS; sl++)
                    for (int k = 0; k < DPD_NACC; k++) {
                        sum[k] += base[sl * DPD_NACC + k];
                        base[sl * DPD_NACC + k] = 0.0;
                    }
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
                st.nlog++;
            }
            st.step++;
            st.zero_pending = 0;
            a.rstate[r] = st;
        }
    }
    if (r == 0) {
        uint32_t ph = *a.phase;
        a.build_flag[ph & 1] = 0;
        *a.phase = ph + 1u;
    }
}

// ---------------------------------------------------------------------------------
// RDF sampling (new; no reference counterpart): histogram of minimum-image distances
// from particles of type ta to particles of type tb within rmax, sampled on steps
// that are multiples of rdf_every, from the end-of-step positions.  Candidate cells
// are the last build's cells around the particle's cell plus one layer (particles
// drift by less than a cell between builds); each build cell is visited once.
#define DPD_RDF_MAXBINS 512
__global__ void __launch_bounds__(256) k_rdf(StepArgs a)
{
    __shared__ unsigned int hs[8][DPD_RDF_MAXBINS];
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int r = -1;
    bool on = false;
    if (s < a.P) {
        r = a.warp_rep[s >> 5];
        const RepDesc& d = a.reps[r];
        const RepState st = a.rstate[r];
        on = d.rdf_every > 0 && rep_active(st) && (st.step % (uint32_t)d.rdf_every) == 0u;
    }
    // every warp is single-replica, so `on` is warp-uniform
    if (!on) return;
    const RepDesc& d = a.reps[r];
    const int nb = min(d.rdf_nbins, DPD_RDF_MAXBINS);
    for (int b = lane; b < nb; b += 32) hs[warp][b] = 0u;
    __syncwarp();
    if (s == d.p_begin) atomicAdd((unsigned long long*)&a.rstate[r].rdf_samples, 1ull);
    if (s < d.p_end) {
        const float4 pi = a.pos4[s];
        const int ti = type0_of(a.vel4[s].w) + 1;
        if (ti == d.rdf_ta) {
            const int ci = __float_as_int(pi.w);
            const int cx = cell_x(ci), cy = cell_y(ci), cz = cell_z(ci);
            const float rmax2 = d.rdf_rmax * d.rdf_rmax;
            const float inv_dr = (float)d.rdf_nbins / d.rdf_rmax;
            int lo3[3], hi3[3];
            for (int k = 0; k < 3; k++) {
                int nr = (int)ceilf(d.rdf_rmax * d.inv_w[k]) + 1;
                if (2 * nr + 1 >= d.nc[k]) {
                    lo3[k] = -(d.nc[k] / 2);
                    hi3[k] = d.nc[k] - 1 - d.nc[k] / 2;
                } else {
                    lo3[k] = -nr;
                    hi3[k] = nr;
                }
            }
            for (int ox = lo3[0]; ox <= hi3[0]; ox++) {
                const int nx = ((cx + ox) % d.nc[0] + d.nc[0]) % d.nc[0];
                for (int oy = lo3[1]; oy <= hi3[1]; oy++) {
                    const int ny = ((cy + oy) % d.nc[1] + d.nc[1]) % d.nc[1];
                    for (int oz = lo3[2]; oz <= hi3[2]; oz++) {
                        const int nz = ((cz + oz) % d.nc[2] + d.nc[2]) % d.nc[2];
                        const int key = d.c_begin + a.crank[d.c_begin + (nx * d.nc[1] + ny) * d.nc[2] + nz];
                        const int jb = a.cstart[key], je = a.cstart[key + 1];
                        for (int j = jb; j < je; j++) {
                            if (j == s) continue;
                            const float4 vj = __ldg(a.vel4 + j);
                            if (type0_of(vj.w) + 1 != d.rdf_tb) continue;
                            const float4 pj = __ldg(a.pos4 + j);
                            float dx, dy, dz;
                            disp3<true>(d, ci, pi, pj, dx, dy, dz);
                            const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
                            if (r2 < rmax2) {
                                int bin = (int)(sqrtf(r2) * inv_dr);
                                if (bin < nb) atomicAdd(&hs[warp][bin], 1u);
                            }
                        }
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
