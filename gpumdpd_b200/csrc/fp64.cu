// fp64.cu -- the FP64 parity engine (fp64.h): the reference's -DDOUBLE timestep on the GPU.
//
// State lives in tag order as wrapped FP64 positions, velocities, forces and image counters.
// Each step: the initial half kick and drift with wrapping (src/fix/fix_nve.cu:42-86), a
// cell grid of fixed-capacity cells (atomic append, then each cell sorted by index so the
// summation order is fixed), the mDPD density pass (src/force/pair_mdpd.cu:253-297), the
// force pass, the final half kick (src/fix/fix_nve.cu:131-149) and on logged steps a
// fixed-order reduction of the thermo sums (src/compute/thermo.cu:240-246,301-303,422-434,
// 506-517).  The force pass gives one warp per atom all its pairs from both sides (the
// 27 cells' candidates filtered 32 at a time, the pairs inside the cutoff evaluated 32 at
// a time), its bonds and its angles, summed by a fixed butterfly, so no atomics touch the
// forces and runs repeat bit for bit.
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "dpd_common.h"
#include "fp64.h"
#include "saru.cuh"

namespace dpd {

namespace {

enum { F64_NONFINITE = 1, F64_FENE = 2, F64_CELL_OVERFLOW = 4, F64_FAR = 8 };
enum { NQ = 9, NSUM = 19, RED_BLOCKS = 256 };
// pair table per type pair: A, B, gamma, rc, rd, sigma = sqrt(gamma) sqrt(2 kT)/sqrt(dt),
// 1/rc, 1/rd, rc^2
enum { NC = 9 };

struct F64Args {
    int n, ntypes, style, bond_style, angle_style, cap;
    int nc[3];
    uint32_t seed, integ_mask;
    double lo[3], L[3], w[3], dt, maxrc2;
    const double *coeff, *mass, *bondc, *anglec;
    double *x, *v, *f, *rho, *q;
    int *img, *type, *cnt, *status;
    double4* crec;  // cell records: position and atom index (exact in a double), cap per cell
    int* ccode;  // each atom's cell as cx | cy << 10 | cz << 20, written by the binning
    const int *bstart, *astart;
    const int2* bent;
    const int4* aent;
};

// minimum image, src/force/neigh_list.cu:377-379: d -= L*((d >= L/2) - (d < -L/2))
__device__ __forceinline__ double min_image(double d, double L)
{
    const double h = 0.5 * L;
    return d - L * (double)((d >= h) - (d < -h));
}

// triangular type-pair index, src/force/pair_dpd.cu:134 (types 1-based, result 0-based)
__device__ __forceinline__ int tri(int ti, int tj, int nt)
{
    const int a = min(ti, tj), b = max(ti, tj);
    return ((a - 1) * nt - (a - 1) * (a - 2) / 2 + b - a + 1) - 1;
}

__device__ __forceinline__ int cell_of(const F64Args& a, const double* p, int c[3])
{
#pragma unroll
    for (int d = 0; d < 3; d++) {
        int k = (int)floor((p[d] - a.lo[d]) / a.w[d]);
        c[d] = min(max(k, 0), a.nc[d] - 1);
    }
    return (c[0] * a.nc[1] + c[1]) * a.nc[2] + c[2];
}

__global__ void k64_clear(int* p, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = 0;
}

// atoms into their cells (appended in the order the atomics draw)
__global__ void k64_bin(F64Args a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    int c[3];
    const int cell = cell_of(a, a.x + 3 * i, c);
    a.ccode[i] = c[0] | (c[1] << 10) | (c[2] << 20);
    const int k = atomicAdd(a.cnt + cell, 1);
    if (k < a.cap)
        a.crec[(size_t)cell * a.cap + k] = make_double4(a.x[3 * i], a.x[3 * i + 1], a.x[3 * i + 2], (double)i);
    else atomicOr(a.status, F64_CELL_OVERFLOW);
}

// each cell's records in atom-index order: the pair sums then run in a fixed order
__global__ void k64_sort_cells(F64Args a, int ncell)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    double4* l = a.crec + (size_t)c * a.cap;
    const int m = min(a.cnt[c], a.cap);
    for (int p = 1; p < m; p++) {
        const double4 v = l[p];
        int q = p - 1;
        while (q >= 0 && l[q].w > v.w) {
            l[q + 1] = l[q];
            q--;
        }
        l[q + 1] = v;
    }
}

// the c-th of the 27 cells around atom i (c = 9 (ox+1) + 3 (oy+1) + (oz+1); nc >= 3 per
// dimension, so no cell is visited twice); calls fn(j, dx, dy, dz, r2) for every other
// atom j there with r2 <= maxrc2, in index order
template <class F>
__device__ __forceinline__ void for_cell(const F64Args& a, int i, int c, F&& fn)
{
    const double xi = a.x[3 * i], yi = a.x[3 * i + 1], zi = a.x[3 * i + 2];
    const int code = a.ccode[i];
    int cx = (code & 1023) + c / 9 - 1, cy = ((code >> 10) & 1023) + (c / 3) % 3 - 1, cz = (code >> 20) + c % 3 - 1;
    cx += cx < 0 ? a.nc[0] : 0; cx -= cx >= a.nc[0] ? a.nc[0] : 0;
    cy += cy < 0 ? a.nc[1] : 0; cy -= cy >= a.nc[1] ? a.nc[1] : 0;
    cz += cz < 0 ? a.nc[2] : 0; cz -= cz >= a.nc[2] ? a.nc[2] : 0;
    const int cell = (cx * a.nc[1] + cy) * a.nc[2] + cz;
    const double4* l = a.crec + (size_t)cell * a.cap;
    const int m = min(a.cnt[cell], a.cap);
    for (int p = 0; p < m; p++) {
        const double4 rj = l[p];
        const int j = (int)rj.w;
        if (j == i) continue;
        const double dx = min_image(xi - rj.x, a.L[0]);
        const double dy = min_image(yi - rj.y, a.L[1]);
        const double dz = min_image(zi - rj.z, a.L[2]);
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 <= a.maxrc2) fn(j, dx, dy, dz, r2);
    }
}

// sum over the warp by a fixed butterfly: the same order on every run
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// mDPD local density, src/force/pair_mdpd.cu:253-297: rho_i = sum_{j != i}
// 15/(2 pi rd^3) max(0, 1 - r/rd)^2 (pairs within the largest cutoff).  One warp per
// atom, lane c takes the c-th of the 27 cells.
__global__ void __launch_bounds__(256) k64_density(F64Args a)
{
    const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (i >= a.n) return;  // warp-uniform
    const int ti = a.type[i];
    double rho = 0.0;
    if (lane < 27)
        for_cell(a, i, lane, [&](int j, double, double, double, double r2) {
            const double* c = a.coeff + NC * tri(ti, a.type[j], a.ntypes);
            const double rd = c[4];
            double wd = 1.0 - sqrt(r2) * c[7];
            if (wd < 0.0) wd = 0.0;
            rho += 15.0 / 2.0 / 3.14159265358979323846 / (rd * rd * rd) * wd * wd;
        });
    rho = warp_sum(rho);
    if (lane == 0) a.rho[i] = rho;
}

// Forces on atom i, one warp per atom.  The records of the 27 cells around the atom
// (src/force/pair_dpd.cu:292-403, pair_mdpd.cu:399-521) are taken 32 at a time as one
// sequence, cell by cell in a fixed order and each cell's records in index order: each
// lane tests one candidate, the pairs inside the largest cutoff are queued in the warp's
// shared ring in ballot order, and whenever 32 are queued every lane evaluates one (the
// Saru random force, the FP64 force) into its own partial sums -- a fixed assignment of
// pairs to lanes, so the sums repeat bit for bit.  The lanes also share out the atom's
// bonds (src/force/bond_harmonic.cu:208-268; FENE + WCA as the FP32 engine) and harmonic
// angles (src/force/angle_harmonic.cu:187-270), and a fixed butterfly sums the lanes.  On
// logged steps the atom's share of the energies and of the virial: half of each pair and
// bond, a third of each angle, as the reference splits them.
#define F64_Q 64  // per-warp ring of queued pairs (power of two, >= 63)

template <bool LOG>
__device__ __forceinline__ void f64_pairs(const F64Args& a, int i, int ti, double rho_i, uint32_t step,
                                          const double4* qd, const int* qj, uint32_t head, int cnt, int lane,
                                          double& fx, double& fy, double& fz, double& pe, double (&vir)[6])
{
    if (lane >= cnt) return;
    const uint32_t e = (head + lane) & (F64_Q - 1);
    const double4 d = qd[e];
    const int j = qj[e];
    const double dx = d.x, dy = d.y, dz = d.z, r2 = d.w;
    const double* c = a.coeff + NC * tri(ti, a.type[j], a.ntypes);
    if (!(r2 <= c[8])) return;
    const double A = c[0], B = c[1], gamma = c[2], rc = c[3], rd = c[4], sigma = c[5];
    // 1/r by rsqrt and r/rc as r * (1/rc): within an ulp of the divisions
    const double rinv = rsqrt(r2);
    const double r = r2 * rinv;
    if (r < 1.0e-10) return;
    const double dot = dx * (a.v[3 * i] - a.v[3 * j]) + dy * (a.v[3 * i + 1] - a.v[3 * j + 1]) +
                       dz * (a.v[3 * i + 2] - a.v[3 * j + 2]);
    const double wc = 1.0 - r * c[6];
    const uint32_t t1 = (uint32_t)min(i, j) + 1u, t2 = (uint32_t)max(i, j) + 1u;
    const double theta = saru_theta_f64(t1, t2, a.seed, step);
    double fpair, e2;
    if (a.style == 0) {
        fpair = A * wc - gamma * wc * wc * dot * rinv + sigma * wc * theta;
        e2 = 0.5 * A * rc * wc * wc;
    } else {
        double wd = 1.0 - r * c[7];
        if (wd < 0.0) wd = 0.0;
        const double rs = rho_i + a.rho[j];
        fpair = A * wc + B * rs * wd - gamma * wc * wc * dot * rinv + sigma * wc * theta;
        e2 = 0.5 * A * rc * wc * wc + 0.25 * B * rd * rs * wd * wd;
    }
    fpair *= rinv;
    const double gx = dx * fpair, gy = dy * fpair, gz = dz * fpair;
    fx += gx;
    fy += gy;
    fz += gz;
    if (LOG) {
        pe += 0.5 * e2;
        vir[0] += 0.5 * dx * gx; vir[1] += 0.5 * dx * gy; vir[2] += 0.5 * dx * gz;
        vir[3] += 0.5 * dy * gy; vir[4] += 0.5 * dy * gz; vir[5] += 0.5 * dz * gz;
    }
}

template <bool LOG>
__global__ void __launch_bounds__(256) k64_force(F64Args a, uint32_t step)
{
    __shared__ double4 s_qd[8][F64_Q];
    __shared__ int s_qj[8][F64_Q];
    const int warp = threadIdx.x >> 5;
    const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (i >= a.n) return;  // warp-uniform
    const int ti = a.type[i];
    double fx = 0.0, fy = 0.0, fz = 0.0, pe = 0.0, bpe = 0.0, ape = 0.0;
    double vir[6] = {0, 0, 0, 0, 0, 0};
    const double rho_i = a.style == 1 ? a.rho[i] : 0.0;
    const double xi = a.x[3 * i], yi = a.x[3 * i + 1], zi = a.x[3 * i + 2];
    // lane c < 27: the c-th cell around the atom (c = 9 (ox+1) + 3 (oy+1) + (oz+1); nc >= 3
    // per dimension, so no cell is visited twice) and its record count
    int cell = 0, m = 0;
    if (lane < 27) {
        const int code = a.ccode[i];
        int cx = (code & 1023) + lane / 9 - 1, cy = ((code >> 10) & 1023) + (lane / 3) % 3 - 1,
            cz = (code >> 20) + lane % 3 - 1;
        cx += cx < 0 ? a.nc[0] : 0; cx -= cx >= a.nc[0] ? a.nc[0] : 0;
        cy += cy < 0 ? a.nc[1] : 0; cy -= cy >= a.nc[1] ? a.nc[1] : 0;
        cz += cz < 0 ? a.nc[2] : 0; cz -= cz >= a.nc[2] ? a.nc[2] : 0;
        cell = (cx * a.nc[1] + cy) * a.nc[2] + cz;
        m = min(a.cnt[cell], a.cap);
    }
    int incl = m;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    const int excl = incl - m;
    const int M = __shfl_sync(0xffffffffu, incl, 31);
    const unsigned lt = (1u << lane) - 1u;
    uint32_t head = 0, tail = 0;
    for (int cb = 0; cb < M; cb += 32) {
        const int t = cb + lane;
        // the candidate's cell: the last of the 27 whose first record is at or before t
        // (an empty cell shares its start with the next one, which then wins)
        int c = 0;
#pragma unroll
        for (int stp = 16; stp >= 1; stp >>= 1) {
            const int probe = min(c + stp, 26);
            const int pstart = __shfl_sync(0xffffffffu, excl, probe);
            if (c + stp <= 26 && pstart <= t) c += stp;
        }
        const int cc = __shfl_sync(0xffffffffu, cell, c);
        const int c0 = __shfl_sync(0xffffffffu, excl, c);
        bool hit = false;
        double dx = 0.0, dy = 0.0, dz = 0.0, r2 = 0.0;
        int j = 0;
        if (t < M) {
            const double4 rj = a.crec[(size_t)cc * a.cap + (t - c0)];
            j = (int)rj.w;
            dx = min_image(xi - rj.x, a.L[0]);
            dy = min_image(yi - rj.y, a.L[1]);
            dz = min_image(zi - rj.z, a.L[2]);
            r2 = dx * dx + dy * dy + dz * dz;
            hit = j != i && r2 <= a.maxrc2;
        }
        const unsigned bm = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            const uint32_t e = (tail + __popc(bm & lt)) & (F64_Q - 1);
            s_qd[warp][e] = make_double4(dx, dy, dz, r2);
            s_qj[warp][e] = j;
        }
        tail += __popc(bm);
        __syncwarp();
        if (tail - head >= 32u) {
            f64_pairs<LOG>(a, i, ti, rho_i, step, s_qd[warp], s_qj[warp], head, 32, lane, fx, fy, fz, pe, vir);
            head += 32;
            __syncwarp();
        }
    }
    if (tail != head)
        f64_pairs<LOG>(a, i, ti, rho_i, step, s_qd[warp], s_qj[warp], head, (int)(tail - head), lane, fx, fy, fz,
                       pe, vir);
    for (int b = a.bstart[i] + lane; b < a.bstart[i + 1]; b += 32) {
        const int2 e2 = a.bent[b];
        const int j = e2.x;
        const double dx = min_image(a.x[3 * i] - a.x[3 * j], a.L[0]);
        const double dy = min_image(a.x[3 * i + 1] - a.x[3 * j + 1], a.L[1]);
        const double dz = min_image(a.x[3 * i + 2] - a.x[3 * j + 2], a.L[2]);
        const double r2 = dx * dx + dy * dy + dz * dz;
        const double r = sqrt(r2);
        const double* bc = a.bondc + 4 * (e2.y - 1);
        double fbond = 0.0, e = 0.0;
        if (a.bond_style == 1) {
            fbond = r > 0.0 ? -2.0 * bc[0] * (r - bc[1]) / r : 0.0;
            e = bc[0] * (r - bc[1]) * (r - bc[1]);
        } else if (a.bond_style == 2) {
            const double K = bc[0], R0 = bc[1], eps = bc[2], sg = bc[3];
            double rr = r2 / (R0 * R0);
            if (rr >= 1.0) {
                atomicOr(a.status, F64_FENE);
                rr = 0.999;
            }
            fbond = -K / (1.0 - rr);
            e = -0.5 * K * R0 * R0 * log(1.0 - rr);
            if (eps > 0.0 && r2 < 1.2599210498948731647672106 * sg * sg) {  // 2^(1/3) s^2
                const double sr2 = sg * sg / r2, sr6 = sr2 * sr2 * sr2;
                fbond += 48.0 * eps * sr6 * (sr6 - 0.5) / r2;
                e += 4.0 * eps * sr6 * (sr6 - 1.0) + eps;
            }
        }
        const double gx = dx * fbond, gy = dy * fbond, gz = dz * fbond;
        fx += gx;
        fy += gy;
        fz += gz;
        if (LOG) {
            bpe += 0.5 * e;
            vir[0] += 0.5 * dx * gx; vir[1] += 0.5 * dx * gy; vir[2] += 0.5 * dx * gz;
            vir[3] += 0.5 * dy * gy; vir[4] += 0.5 * dy * gz; vir[5] += 0.5 * dz * gz;
        }
    }
    for (int t = a.astart[i] + lane; t < a.astart[i + 1]; t += 32) {
        const int4 an = a.aent[t];
        double d1[3], d2[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            d1[c] = min_image(a.x[3 * an.x + c] - a.x[3 * an.y + c], a.L[c]);
            d2[c] = min_image(a.x[3 * an.z + c] - a.x[3 * an.y + c], a.L[c]);
        }
        const double rsq1 = d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2];
        const double rsq2 = d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2];
        const double r1 = sqrt(rsq1), r2 = sqrt(rsq2);
        double c = (d1[0] * d2[0] + d1[1] * d2[1] + d1[2] * d2[2]) / (r1 * r2);
        c = fmin(fmax(c, -1.0), 1.0);
        double s = sqrt(1.0 - c * c);
        if (s < 0.001) s = 0.001;
        const double kk = a.anglec[2 * (an.w - 1)];
        const double theta0 = a.anglec[2 * (an.w - 1) + 1] * (3.14159265358979323846 / 180.0);
        const double dth = acos(c) - theta0;
        const double aa = -2.0 * kk * dth / s;
        const double a11 = aa * c / rsq1, a12 = -aa / (r1 * r2), a22 = aa * c / rsq2;
        double fi[3], fk[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            fi[q] = a11 * d1[q] + a12 * d2[q];
            fk[q] = a22 * d2[q] + a12 * d1[q];
        }
        if (i == an.x) {
            fx += fi[0]; fy += fi[1]; fz += fi[2];
        } else if (i == an.z) {
            fx += fk[0]; fy += fk[1]; fz += fk[2];
        } else {
            fx -= fi[0] + fk[0]; fy -= fi[1] + fk[1]; fz -= fi[2] + fk[2];
        }
        if (LOG) {
            const double third = 1.0 / 3.0;
            ape += third * kk * dth * dth;
            vir[0] += third * (d1[0] * fi[0] + d2[0] * fk[0]);
            vir[1] += third * (d1[0] * fi[1] + d2[0] * fk[1]);
            vir[2] += third * (d1[0] * fi[2] + d2[0] * fk[2]);
            vir[3] += third * (d1[1] * fi[1] + d2[1] * fk[1]);
            vir[4] += third * (d1[1] * fi[2] + d2[1] * fk[2]);
            vir[5] += third * (d1[2] * fi[2] + d2[2] * fk[2]);
        }
    }
    fx = warp_sum(fx);
    fy = warp_sum(fy);
    fz = warp_sum(fz);
    if (lane == 0) {
        a.f[3 * i] = fx;
        a.f[3 * i + 1] = fy;
        a.f[3 * i + 2] = fz;
    }
    if (LOG) {
        pe = warp_sum(pe);
        bpe = warp_sum(bpe);
        ape = warp_sum(ape);
#pragma unroll
        for (int k = 0; k < 6; k++) vir[k] = warp_sum(vir[k]);
        if (lane == 0) {
            double* q = a.q + (size_t)NQ * i;
            q[0] = pe;
            q[1] = bpe;
            q[2] = ape;
#pragma unroll
            for (int k = 0; k < 6; k++) q[3 + k] = vir[k];
        }
    }
}

__device__ __forceinline__ bool integrated(const F64Args& a, int t)
{
    return !a.integ_mask || ((a.integ_mask >> (t - 1)) & 1u);
}

// half kick and drift with the reference's wrap (a while loop moving whole box lengths
// and counting images); a non-finite coordinate, or one more than 4 box lengths away
// after a step, is an error
__global__ void k64_initial(F64Args a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int t = a.type[i];
    if (!integrated(a, t)) return;
    const double dtm = 0.5 * a.dt / a.mass[t - 1];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        a.v[3 * i + d] += dtm * a.f[3 * i + d];
        double p = a.x[3 * i + d] + a.dt * a.v[3 * i + d];
        const double hi = a.lo[d] + a.L[d];
        if (!isfinite(p)) {
            atomicOr(a.status, F64_NONFINITE);
            p = a.lo[d];
        }
        int guard = 0;
        while ((p >= hi || p < a.lo[d]) && guard < 4) {
            const int k = (p >= hi) - (p < a.lo[d]);
            p -= a.L[d] * k;
            a.img[3 * i + d] += k;
            guard++;
        }
        if (p >= hi || p < a.lo[d]) {
            atomicOr(a.status, F64_FAR);
            p = a.lo[d];
        }
        a.x[3 * i + d] = p;
    }
}

__global__ void k64_final(F64Args a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int t = a.type[i];
    if (!integrated(a, t)) return;
    const double dtm = 0.5 * a.dt / a.mass[t - 1];
#pragma unroll
    for (int d = 0; d < 3; d++) a.v[3 * i + d] += dtm * a.f[3 * i + d];
}

// Thermo sums in a fixed order: block b takes a contiguous range of atoms, each thread a
// fixed stride of it, then a fixed tree over the block; the final pass adds the blocks'
// partial sums in block order.  Sums: KE, m v_a v_b (6), momentum (3), pair, bond and
// angle PE, virial (6).
__global__ void __launch_bounds__(256) k64_thermo_partial(F64Args a, double* part)
{
    __shared__ double sh[NSUM][256];
    double acc[NSUM];
#pragma unroll
    for (int k = 0; k < NSUM; k++) acc[k] = 0.0;
    const int per = (a.n + gridDim.x - 1) / gridDim.x;
    const int b0 = blockIdx.x * per, b1 = min(a.n, b0 + per);
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const double m = a.mass[a.type[i] - 1];
        const double vx = a.v[3 * i], vy = a.v[3 * i + 1], vz = a.v[3 * i + 2];
        acc[0] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
        acc[1] += m * vx * vx; acc[2] += m * vx * vy; acc[3] += m * vx * vz;
        acc[4] += m * vy * vy; acc[5] += m * vy * vz; acc[6] += m * vz * vz;
        acc[7] += m * vx; acc[8] += m * vy; acc[9] += m * vz;
        const double* q = a.q + (size_t)NQ * i;
#pragma unroll
        for (int k = 0; k < NQ; k++) acc[10 + k] += q[k];
    }
#pragma unroll
    for (int k = 0; k < NSUM; k++) sh[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int k = 0; k < NSUM; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x < NSUM) part[(size_t)blockIdx.x * NSUM + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void k64_thermo_final(const double* part, int nblocks, double* sums)
{
    const int k = threadIdx.x;
    if (k >= NSUM) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; b++) s += part[(size_t)b * NSUM + k];
    sums[k] = s;
}

}  // namespace

// ---------------------------------------------------------------------------------
#define F64_CK(call)                                  \
    do {                                              \
        cudaError_t e_ = (call);                      \
        if (e_ != cudaSuccess) return fail(e_, #call); \
    } while (0)

int EngineF64::fail(cudaError_t e, const char* what)
{
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return DPD_E_CUDA;
}

EngineF64::~EngineF64()
{
    void* ptrs[] = {x_, v_, f_, rho_, q_, part_, sums_, img_, type_, cnt_, ccode_, crec_, status_,
                    bstart_, astart_, bent_, aent_, tab_};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (stream_) cudaStreamDestroy(stream_);
}

template <class T>
static cudaError_t dalloc64(T** p, size_t n, int64_t& bytes)
{
    bytes += (int64_t)(sizeof(T) * (n ? n : 1));
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (n ? n : 1));
    if (e == cudaSuccess) e = cudaMemset(*p, 0, sizeof(T) * (n ? n : 1));
    return e;
}

int EngineF64::init(Replica&& rep)
{
    R_ = std::move(rep);
    const RunInput& in = R_.in;
    const ForceField& ff = R_.ff;
    // the parity mode covers the force field and NVE; every fix and compute other than
    // nve, and dumps, belong to the single-precision engine
    if (ff.spring.on || ff.rvcm.on || ff.recenter.on || !ff.moves.empty() || !ff.reflects.empty() ||
        !ff.twowalls.empty() || !ff.gcs.empty() || !ff.cdumps.empty() || !ff.rdfs.empty() || in.dump) {
        err = "the FP64 parity mode runs pair, bond and angle styles with fix nve only: "
              "remove the other fixes, computes and dumps";
        return DPD_E_ARG;
    }
    if (in.log_f == 0) {
        err = "thermo interval must be positive";
        return DPD_E_ARG;
    }
    n_ = R_.sys.n_atoms;
    if (n_ < 2) {
        err = "the FP64 parity mode needs at least 2 atoms";
        return DPD_E_ARG;
    }
    for (int d = 0; d < 3; d++) {
        L_[d] = R_.sys.hi[d] - R_.sys.lo[d];
        nc_[d] = (int)std::floor(L_[d] / in.global_cut);
        if (nc_[d] < 3) {
            err = "box too small: the cell grid needs at least 3 cells of size global_cut per dimension";
            return DPD_E_ARG;
        }
        if (nc_[d] > DPD_MAX_NC) {
            err = "box too large: at most 1023 cells per dimension";
            return DPD_E_ARG;
        }
    }
    ncell_ = nc_[0] * nc_[1] * nc_[2];
    const double wv = (L_[0] / nc_[0]) * (L_[1] / nc_[1]) * (L_[2] / nc_[2]);
    cap_ = std::max(32, (((int)(2.0 * in.max_rho * wv) + 1 + 15) / 16) * 16);
    // every table index the kernels take from the input is checked here
    const int ntyp = R_.sys.n_atomtypes;
    const int nbtyp = std::max(R_.sys.n_bondtypes, 1), natyp = std::max(R_.sys.n_angletypes, 1);
    if ((int)R_.sys.type.size() < n_ || (int)R_.sys.masses.size() < ntyp ||
        (int)ff.coeff.size() < ntyp * (ntyp + 1) / 2) {
        err = "incomplete system or pair coefficients";
        return DPD_E_ARG;
    }
    for (int i = 0; i < n_; i++)
        if (R_.sys.type[i] < 1 || R_.sys.type[i] > ntyp) {
            err = "atom type out of range";
            return DPD_E_ARG;
        }
    // bonds and angles in tag order, as adjacency lists of each atom
    const int nb = R_.sys.n_bonds, na = R_.ff.angle_style ? R_.sys.n_angles : 0;
    for (int b = 0; b < nb; b++)
        if (R_.sys.bonds[3 * b] < 1 || R_.sys.bonds[3 * b] > nbtyp) {
            err = "bond type out of range";
            return DPD_E_ARG;
        }
    for (int t = 0; t < na; t++)
        if (R_.sys.angles[4 * t] < 1 || R_.sys.angles[4 * t] > natyp) {
            err = "angle type out of range";
            return DPD_E_ARG;
        }
    std::vector<int> bstart(n_ + 1, 0), astart(n_ + 1, 0);
    auto tag_ok = [&](int t) { return t >= 1 && t <= n_; };
    for (int b = 0; b < nb; b++) {
        const int* e = &R_.sys.bonds[3 * b];
        if (!tag_ok(e[1]) || !tag_ok(e[2])) {
            err = "bond partner not found";
            return DPD_E_STATE;
        }
        bstart[e[1]]++;
        bstart[e[2]]++;
    }
    for (int t = 0; t < na; t++) {
        const int* e = &R_.sys.angles[4 * t];
        if (!tag_ok(e[1]) || !tag_ok(e[2]) || !tag_ok(e[3])) {
            err = "angle atom not found";
            return DPD_E_STATE;
        }
        astart[e[1]]++;
        astart[e[2]]++;
        astart[e[3]]++;
    }
    for (int i = 0; i < n_; i++) {
        bstart[i + 1] += bstart[i];
        astart[i + 1] += astart[i];
    }
    std::vector<int2> bent(std::max(2 * nb, 1));
    std::vector<int4> aent(std::max(3 * na, 1));
    {
        std::vector<int> fb(bstart.begin(), bstart.end() - 1), fa(astart.begin(), astart.end() - 1);
        for (int b = 0; b < nb; b++) {
            const int* e = &R_.sys.bonds[3 * b];
            const int i = e[1] - 1, j = e[2] - 1;
            bent[fb[i]++] = make_int2(j, e[0]);
            bent[fb[j]++] = make_int2(i, e[0]);
        }
        for (int t = 0; t < na; t++) {
            const int* e = &R_.sys.angles[4 * t];
            const int4 an = make_int4(e[1] - 1, e[2] - 1, e[3] - 1, e[0]);
            for (int k = 1; k <= 3; k++) aent[fa[e[k] - 1]++] = an;
        }
    }
    // coefficient tables
    const int nt = R_.sys.n_atomtypes, ntri = nt * (nt + 1) / 2;
    const int nbt = std::max(R_.sys.n_bondtypes, 1), nat = std::max(R_.sys.n_angletypes, 1);
    std::vector<double> tab((size_t)NC * ntri + nt + 4 * nbt + 2 * nat, 0.0);
    // sqrt(2 kT) / sqrt(dt), src/force/pair_dpd.cu:577-578
    const double sig_scale = std::sqrt(2.0 * ff.temp) / std::sqrt(in.dt);
    for (int p = 0; p < ntri && p < (int)ff.coeff.size(); p++) {
        double* c = &tab[(size_t)NC * p];
        for (int k = 0; k < 5; k++) c[k] = ff.coeff[p][k];
        c[5] = std::sqrt(c[2]) * sig_scale;
        c[6] = c[3] > 0.0 ? 1.0 / c[3] : 0.0;
        c[7] = c[4] > 0.0 ? 1.0 / c[4] : HUGE_VAL;  // no rd: w_d clamps to 0
        c[8] = c[3] * c[3];
    }
    for (int t = 0; t < nt; t++) tab[NC * ntri + t] = R_.sys.masses[t];
    for (int b = 0; b < (int)ff.bond_coeff.size() && b < nbt; b++)
        for (int k = 0; k < 4; k++) tab[NC * ntri + nt + 4 * b + k] = ff.bond_coeff[b][k];
    for (int b = 0; b < (int)ff.angle_coeff.size() && b < nat; b++)
        for (int k = 0; k < 2; k++) tab[NC * ntri + nt + 4 * nbt + 2 * b + k] = ff.angle_coeff[b][k];

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        err = "no CUDA device available (this engine has no CPU fallback)";
        return DPD_E_NODEV;
    }
    if (const char* dv = std::getenv("DPD_B200_DEVICE")) {  // as the single-precision engine
        const int dev = std::atoi(dv);
        if (dev < 0 || dev >= ndev) {
            err = "DPD_B200_DEVICE is not a device index";
            return DPD_E_NODEV;
        }
        F64_CK(cudaSetDevice(dev));
    }
    F64_CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    const size_t n = (size_t)n_;
    F64_CK(dalloc64(&x_, 3 * n, bytes_));
    F64_CK(dalloc64(&v_, 3 * n, bytes_));
    F64_CK(dalloc64(&f_, 3 * n, bytes_));
    F64_CK(dalloc64(&rho_, n, bytes_));
    F64_CK(dalloc64(&q_, (size_t)NQ * n, bytes_));
    F64_CK(dalloc64(&part_, (size_t)NSUM * RED_BLOCKS, bytes_));
    F64_CK(dalloc64(&sums_, (size_t)NSUM, bytes_));
    F64_CK(dalloc64(&img_, 3 * n, bytes_));
    F64_CK(dalloc64(&type_, n, bytes_));
    F64_CK(dalloc64(&cnt_, (size_t)ncell_, bytes_));
    F64_CK(dalloc64(&ccode_, n, bytes_));
    F64_CK(dalloc64(&crec_, (size_t)ncell_ * cap_, bytes_));
    F64_CK(dalloc64(&status_, 1, bytes_));
    F64_CK(dalloc64(&bstart_, n + 1, bytes_));
    F64_CK(dalloc64(&astart_, n + 1, bytes_));
    F64_CK(dalloc64(&bent_, bent.size(), bytes_));
    F64_CK(dalloc64(&aent_, aent.size(), bytes_));
    F64_CK(dalloc64(&tab_, tab.size(), bytes_));
    F64_CK(cudaMemcpy(type_, R_.sys.type.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    F64_CK(cudaMemcpy(bstart_, bstart.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    F64_CK(cudaMemcpy(astart_, astart.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    F64_CK(cudaMemcpy(bent_, bent.data(), sizeof(int2) * bent.size(), cudaMemcpyHostToDevice));
    F64_CK(cudaMemcpy(aent_, aent.data(), sizeof(int4) * aent.size(), cudaMemcpyHostToDevice));
    F64_CK(cudaMemcpy(tab_, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
    return upload_state(true, true);
}

// positions wrapped into [lo, lo + L) with image counts from zero (as a data file is
// read) and/or velocities; the next run starts with a zero step
int EngineF64::upload_state(bool pos, bool vel)
{
    const size_t n3 = 3 * (size_t)n_;
    zero_pending_ = true;
    if (vel) {
        std::vector<double> v(n3, 0.0);
        if (R_.sys.v.size() >= n3) std::copy(R_.sys.v.begin(), R_.sys.v.begin() + n3, v.begin());
        F64_CK(cudaMemcpyAsync(v_, v.data(), sizeof(double) * n3, cudaMemcpyHostToDevice, stream_));
        F64_CK(cudaStreamSynchronize(stream_));
    }
    if (!pos) return DPD_OK;
    std::vector<double> x(R_.sys.x.begin(), R_.sys.x.begin() + n3);
    std::vector<int> img(n3, 0);
    for (size_t k = 0; k < n3; k++) {
        const int d = (int)(k % 3);
        double p = x[k];
        if (!std::isfinite(p)) {
            err = "non-finite position in the input";
            return DPD_E_ARG;
        }
        const double lo = R_.sys.lo[d], hi = lo + L_[d];
        if (p >= hi || p < lo) {
            const double q = std::floor((p - lo) / L_[d]);
            p -= L_[d] * q;
            img[k] += (int)q;
            if (p >= hi) p = lo;
            if (p < lo) p = lo;
        }
        x[k] = p;
    }
    F64_CK(cudaMemcpyAsync(x_, x.data(), sizeof(double) * n3, cudaMemcpyHostToDevice, stream_));
    F64_CK(cudaMemcpyAsync(img_, img.data(), sizeof(int) * n3, cudaMemcpyHostToDevice, stream_));
    F64_CK(cudaStreamSynchronize(stream_));
    return DPD_OK;
}

static F64Args make_args(const Replica& R, int n, const int nc[3], const double L[3], int cap)
{
    F64Args a;
    memset(&a, 0, sizeof(a));
    a.n = n;
    a.ntypes = R.sys.n_atomtypes;
    a.style = R.ff.pair_style;
    a.bond_style = R.sys.n_bonds > 0 ? R.ff.bond_style : 0;
    a.angle_style = R.ff.angle_style;
    a.cap = cap;
    a.seed = R.ff.seed;
    a.integ_mask = R.ff.integ_mask;
    a.dt = R.in.dt;
    double rcm = 0.0;
    for (auto& c : R.ff.coeff) rcm = std::max(rcm, c[3]);
    a.maxrc2 = rcm * rcm;
    for (int d = 0; d < 3; d++) {
        a.nc[d] = nc[d];
        a.lo[d] = R.sys.lo[d];
        a.L[d] = L[d];
        a.w[d] = L[d] / nc[d];
    }
    return a;
}

int EngineF64::eval_forces(uint32_t step, bool log)
{
    F64Args a = make_args(R_, n_, nc_, L_, cap_);
    const int nt = R_.sys.n_atomtypes, ntri = nt * (nt + 1) / 2, nbt = std::max(R_.sys.n_bondtypes, 1);
    a.coeff = tab_;
    a.mass = tab_ + NC * ntri;
    a.bondc = tab_ + NC * ntri + nt;
    a.anglec = tab_ + NC * ntri + nt + 4 * nbt;
    a.x = x_; a.v = v_; a.f = f_; a.rho = rho_; a.q = q_;
    a.img = img_; a.type = type_; a.cnt = cnt_; a.crec = crec_; a.status = status_; a.ccode = ccode_;
    a.bstart = bstart_; a.astart = astart_; a.bent = bent_; a.aent = aent_;
    const int g = (n_ + 255) / 256, gc = (ncell_ + 255) / 256;
    const int gw = (int)(((size_t)n_ * 32 + 255) / 256);  // a warp per atom
    k64_clear<<<gc, 256, 0, stream_>>>(cnt_, ncell_);
    k64_bin<<<g, 256, 0, stream_>>>(a);
    k64_sort_cells<<<gc, 256, 0, stream_>>>(a, ncell_);
    if (a.style == 1) k64_density<<<gw, 256, 0, stream_>>>(a);
    if (log) k64_force<true><<<gw, 256, 0, stream_>>>(a, step);
    else k64_force<false><<<gw, 256, 0, stream_>>>(a, step);
    F64_CK(cudaGetLastError());
    return DPD_OK;
}

// the thermo row of a logged step (src/compute/thermo.cu): T = 2 KE / (3N - 3),
// P_ab = (sum m v_a v_b + W_ab) / V, P = trace / 3
int EngineF64::log_row(uint32_t step)
{
    F64Args a = make_args(R_, n_, nc_, L_, cap_);
    const int nt = R_.sys.n_atomtypes, ntri = nt * (nt + 1) / 2;
    a.mass = tab_ + NC * ntri;
    a.v = v_; a.q = q_; a.type = type_;
    const int nb = std::min((int)RED_BLOCKS, (n_ + 255) / 256);
    k64_thermo_partial<<<nb, 256, 0, stream_>>>(a, part_);
    k64_thermo_final<<<1, 32, 0, stream_>>>(part_, nb, sums_);
    double s[NSUM];
    F64_CK(cudaMemcpyAsync(s, sums_, sizeof(s), cudaMemcpyDeviceToHost, stream_));
    F64_CK(cudaStreamSynchronize(stream_));
    dpd_thermo t;
    memset(&t, 0, sizeof(t));
    const double vol = L_[0] * L_[1] * L_[2];
    t.step = step;
    t.ke = s[0];
    t.temp = 2.0 * s[0] / (3.0 * n_ - 3.0);
    t.pair_pe = s[10];
    t.bond_pe = s[11];
    t.angle_pe = s[12];
    for (int c = 0; c < 6; c++) t.p[c] = (s[1 + c] + s[13 + c]) / vol;
    t.pressure = (t.p[0] + t.p[3] + t.p[5]) / 3.0;
    for (int c = 0; c < 3; c++) t.momentum[c] = s[7 + c];
    rows_.push_back(t);
    return DPD_OK;
}

int EngineF64::check_status()
{
    int st = 0;
    F64_CK(cudaMemcpyAsync(&st, status_, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    F64_CK(cudaStreamSynchronize(stream_));
    if (st & F64_CELL_OVERFLOW) {
        err = "cell overflow in the FP64 parity mode: increase max_rho in the neighbor command";
        return DPD_E_OVERFLOW;
    }
    if (st & (F64_NONFINITE | F64_FAR)) {
        err = "non-finite position or velocity";
        return DPD_E_NUMERIC;
    }
    if (st & F64_FENE) {
        err = "FENE bond stretched beyond R0";
        return DPD_E_NUMERIC;
    }
    return DPD_OK;
}

// Steps in the order of the reference's loop (src/main/utils.cuh:166-213 for the zero
// step, :254-303 per step): the zero step evaluates forces at the current step and logs
// it when due; each step then kicks and drifts, evaluates forces, kicks, and logs.
int EngineF64::run(uint32_t nsteps)
{
    F64Args a = make_args(R_, n_, nc_, L_, cap_);
    const int nt = R_.sys.n_atomtypes, ntri = nt * (nt + 1) / 2;
    a.mass = tab_ + NC * ntri;
    a.x = x_; a.v = v_; a.f = f_; a.img = img_; a.type = type_; a.status = status_;
    const int g = (n_ + 255) / 256;
    const uint32_t log_f = R_.in.log_f;
    int e;
    if (zero_pending_) {
        const uint32_t s0 = next_step_;
        const bool log = s0 % log_f == 0;
        if ((e = eval_forces(s0, log))) return e;
        if ((e = check_status())) return e;
        if (log && (e = log_row(s0))) return e;
        zero_pending_ = false;
        next_step_ = s0 + 1;
    }
    for (uint32_t k = 0; k < nsteps; k++) {
        const uint32_t step = next_step_;
        const bool log = step % log_f == 0;
        k64_initial<<<g, 256, 0, stream_>>>(a);
        if ((e = eval_forces(step, log))) return e;
        k64_final<<<g, 256, 0, stream_>>>(a);
        F64_CK(cudaGetLastError());
        if (log) {
            if ((e = log_row(step))) return e;
            if ((e = check_status())) return e;
        }
        next_step_ = step + 1;
    }
    return check_status();
}

int EngineF64::get_thermo(dpd_thermo* rows, int max_rows, int* n_rows) const
{
    const int n = std::min((int)rows_.size(), std::max(max_rows, 0));
    for (int k = 0; k < n; k++) rows[k] = rows_[rows_.size() - n + k];
    if (n_rows) *n_rows = n;
    return DPD_OK;
}

int EngineF64::get_state(double* x, double* v, int* image, double* f)
{
    const size_t n3 = 3 * (size_t)n_;
    if (x) F64_CK(cudaMemcpyAsync(x, x_, sizeof(double) * n3, cudaMemcpyDeviceToHost, stream_));
    if (v) F64_CK(cudaMemcpyAsync(v, v_, sizeof(double) * n3, cudaMemcpyDeviceToHost, stream_));
    if (image) F64_CK(cudaMemcpyAsync(image, img_, sizeof(int) * n3, cudaMemcpyDeviceToHost, stream_));
    if (f) F64_CK(cudaMemcpyAsync(f, f_, sizeof(double) * n3, cudaMemcpyDeviceToHost, stream_));
    F64_CK(cudaStreamSynchronize(stream_));
    return DPD_OK;
}

// nsteps steps timed with CUDA events on the engine's stream
int EngineF64::time_steps(uint32_t nsteps, double* total_ms)
{
    if (zero_pending_) {
        int e = run(0);
        if (e) return e;
    }
    cudaEvent_t e0, e1;
    F64_CK(cudaEventCreate(&e0));
    F64_CK(cudaEventCreate(&e1));
    F64_CK(cudaEventRecord(e0, stream_));
    int e = run(nsteps);
    cudaEventRecord(e1, stream_);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e) return e;
    if (total_ms) *total_ms = ms;
    return DPD_OK;
}

// the reference's write_data file of the current state (as the single-precision engine)
int EngineF64::write_data(const std::string& path)
{
    SystemData s = R_.sys;
    s.v.resize(s.x.size());
    int e = get_state(s.x.data(), s.v.data(), nullptr, nullptr);
    if (e) return e;
    return write_data_file(path, R_.in.atom_style, s, err);
}

// new positions (image counts restart from zero) and/or velocities by tag; the next run
// starts with a zero step
int EngineF64::set_state(const double* x, const double* v)
{
    const size_t n3 = 3 * (size_t)n_;
    if (x) std::copy(x, x + n3, R_.sys.x.begin());
    if (v) {
        R_.sys.v.resize(n3);
        std::copy(v, v + n3, R_.sys.v.begin());
    }
    return upload_state(x != nullptr, v != nullptr);
}

}  // namespace dpd
