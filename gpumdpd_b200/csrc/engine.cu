// engine.cu -- host engine: packed replica layout, device buffers, the captured
// timestep, state I/O.  The timestep order is the reference's
// (src/main/utils.cuh:166-213 zero step, :254-303 per step):
//   [list build if flagged] [mDPD density] [pair + bonds] [RDF sample]
//   [final half kick n, thermo n, initial half kick + drift n+1, build check] [advance]
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <atomic>
#include <thread>

#include "dump.h"
#include "engine.h"
#include "kernels.cuh"
#include "kernels_aos.cuh"
#include "kernels_step.cuh"
#include "kernels_tile.cuh"

namespace dpd {

#define CK(call)                                               \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);    \
    } while (0)

int Engine::cuda_fail(cudaError_t e, const char* what)
{
    err = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? DPD_E_NOMEM : DPD_E_CUDA;
}

template <class T>
int Engine::dalloc(T** p, size_t n)
{
    size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    // stream-ordered: neither allocation nor release synchronizes the device, so engines
    // of the job server can come and go while other engines' kernels run
    cudaError_t e = cudaMallocAsync((void**)p, bytes, stream_);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    allocs_.push_back((void*)*p);
    dev_bytes_ += (int64_t)bytes;
    e = cudaMemsetAsync(*p, 0, bytes, stream_);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    return DPD_OK;
}

Engine::~Engine()
{
    dump_close();
    if (graph_) cudaGraphExecDestroy(graph_);
    if (stream_) cudaStreamSynchronize(stream_);
    for (void* p : allocs_) cudaFreeAsync(p, stream_);
    if (stream_) cudaStreamSynchronize(stream_);
    for (void* p : {(void*)h_pos_, (void*)h_vel_, (void*)h_frc_, (void*)h_img_})
        if (p) cudaFreeHost(p);
    if (stream_) cudaStreamDestroy(stream_);
}

// ---------------------------------------------------------------------------------
static uint32_t morton3(uint32_t x, uint32_t y, uint32_t z)
{
    auto spread = [](uint32_t v) {
        v &= 0x3ff;
        v = (v | (v << 16)) & 0x030000FF;
        v = (v | (v << 8)) & 0x0300F00F;
        v = (v | (v << 4)) & 0x030C30C3;
        v = (v | (v << 2)) & 0x09249249;
        return v;
    };
    return spread(x) | (spread(y) << 1) | (spread(z) << 2);
}

static uint32_t morton2(uint32_t x, uint32_t y)
{
    auto spread = [](uint32_t v) {
        v &= 0x3ff;
        v = (v | (v << 8)) & 0x00FF00FF;
        v = (v | (v << 4)) & 0x0F0F0F0F;
        v = (v | (v << 2)) & 0x33333333;
        v = (v | (v << 1)) & 0x55555555;
        return v;
    };
    return spread(x) | (spread(y) << 1);
}

// The order of a replica's cells in the slot array: 0 = linear (z fastest), 1 = Morton,
// 2 = the x-y columns in Morton order with the cells of a column consecutive (z
// fastest), so that cells z-1..z+1 of a column are one slot range (list build 5).
void Engine::rank_cells(Replica& R) const
{
    const RepDesc& d = R.desc;
    R.crank.resize(d.ncell);
    std::vector<std::pair<uint32_t, int>> order(d.ncell);
    for (int cx = 0; cx < d.nc[0]; cx++)
        for (int cy = 0; cy < d.nc[1]; cy++)
            for (int cz = 0; cz < d.nc[2]; cz++) {
                const int lin = (cx * d.nc[1] + cy) * d.nc[2] + cz;
                uint32_t key = (uint32_t)lin;
                if (tune_.cell_order == 1) key = morton3(cx, cy, cz);
                else if (tune_.cell_order == 2) key = morton2(cx, cy) * (uint32_t)d.nc[2] + (uint32_t)cz;
                order[lin] = {key, lin};
            }
    std::sort(order.begin(), order.end());
    for (int k = 0; k < d.ncell; k++) R.crank[order[k].second] = k;
}

// the device copies of the cell ranks and of their inverse
int Engine::upload_ranks()
{
    std::vector<int> crank(C_, 0), cell_lin(C_, -1);
    for (const Replica& R : reps_) {
        const RepDesc& d = R.desc;
        for (int c = 0; c < d.ncell; c++) {
            crank[d.c_begin + c] = R.crank[c];
            cell_lin[d.c_begin + R.crank[c]] = c;
        }
    }
    CK(cudaMemcpyAsync(b_.crank, crank.data(), sizeof(int) * C_, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(b_.cell_lin, cell_lin.data(), sizeof(int) * C_, cudaMemcpyHostToDevice, stream_));
    CK(cudaStreamSynchronize(stream_));
    return DPD_OK;
}

int Engine::layout()
{
    P_ = 0;
    C_ = 0;
    nmax_ = 16;
    maxb_ = 0;
    int tag_base = 0, coeff_off = 0, mass_off = 0, bond_off = 0, rdf_off = 0;
    any_mdpd_ = any_dpd_ = bonds_ = rdf_ = any_gc_ = false;
    for (size_t r = 0; r < reps_.size(); r++) {
        Replica& R = reps_[r];
        RepDesc& d = R.desc;
        memset(&d, 0, sizeof(d));
        const double cut = R.in.global_cut + R.in.skin;
        for (int k = 0; k < 3; k++) {
            const double L = R.sys.hi[k] - R.sys.lo[k];
            int nc = (int)std::floor(L / cut);
            if (nc < 3) {
                err = "box too small: the cell grid needs at least 3 cells of size global_cut+skin per dimension";
                return DPD_E_ARG;
            }
            if (nc > DPD_MAX_NC) {
                err = "box too large: at most 1023 cells per dimension";
                return DPD_E_ARG;
            }
            d.nc[k] = nc;
            d.w[k] = (float)(L / nc);
            d.inv_w[k] = 1.0f / d.w[k];
            R.box_len[k] = (double)nc * (double)d.w[k];
            d.L[k] = (float)R.box_len[k];
            d.lo[k] = R.sys.lo[k];
        }
        const int n = R.sys.n_atoms;
        if (n > DPD_MAX_TAG) {
            err = "too many atoms in one system";
            return DPD_E_ARG;
        }
        d.p_begin = P_;
        d.n_real = n;
        d.p_end = P_ + n;
        d.p_cap_end = P_ + ((n + 31) / 32) * 32;
        P_ = d.p_cap_end;
        d.c_begin = C_;
        d.ncell = d.nc[0] * d.nc[1] * d.nc[2];
        C_ += d.ncell + 1;
        d.tag_base = tag_base;
        tag_base += n;
        const float cutf = (float)cut;
        d.cut2 = cutf * cutf;
        double rcm = 0;
        for (auto& c : R.ff.coeff) rcm = std::max(rcm, c[3]);
        d.rcmax2 = (float)(rcm * rcm);
        const float hs = (float)(R.in.skin * 0.5);
        d.hskin2 = hs * hs;
        d.skin_zero = R.in.skin == 0.0;
        d.ntypes = R.sys.n_atomtypes;
        d.coeff_off = coeff_off;
        coeff_off += d.ntypes * d.ntypes * 3;
        d.mass_off = mass_off;
        mass_off += d.ntypes;
        d.style = R.ff.pair_style;
        if (d.style == 1) any_mdpd_ = true; else any_dpd_ = true;
        d.seed = R.ff.seed;
        d.dt = (float)R.in.dt;
        d.nl_f = R.in.nl_f;
        d.log_f = (int)R.in.log_f;
        d.bond_style = R.sys.n_bonds > 0 ? R.ff.bond_style : 0;
        if (d.bond_style) bonds_ = true;
        d.bond_off = bond_off;
        bond_off += std::max(R.sys.n_bondtypes, 1);
        d.integ_mask = R.ff.integ_mask;
        d.volume = R.box_len[0] * R.box_len[1] * R.box_len[2];
        if (!R.ff.rdfs.empty()) {
            const ComputeRdf& c = R.ff.rdfs[0];
            d.rdf_every = c.every;
            d.rdf_ta = c.ta;
            d.rdf_tb = c.tb;
            d.rdf_nbins = c.nbins;
            d.rdf_rmax = (float)c.rmax;
            rdf_ = true;
        }
        d.gc_n = (int)R.ff.gcs.size();
        if (d.gc_n) any_gc_ = true;
        d.rdf_off = rdf_off;
        rdf_off += R.ff.rdfs.empty() ? 0 : R.ff.rdfs[0].nbins;
        // neighbour capacity: src/force/neigh_list.cu:14-17
        const double sphere = 4.0 / 3.0 * M_PI * std::pow(cut, 3.0);
        int nm = (int)(R.in.max_rho * sphere) + 1;
        nm = ((nm + 15) / 16) * 16;
        R.nmax = nm;
        nmax_ = std::max(nmax_, nm);
        // bond partners per atom
        if (d.bond_style) {
            std::vector<int> deg(n, 0);
            for (int b = 0; b < R.sys.n_bonds; b++) {
                deg[R.sys.bonds[3 * b + 1] - 1]++;
                deg[R.sys.bonds[3 * b + 2] - 1]++;
            }
            for (int i = 0; i < n; i++) R.maxb = std::max(R.maxb, deg[i]);
            maxb_ = std::max(maxb_, R.maxb);
        }
        rank_cells(R);
    }
    if (maxb_ > 16) {
        err = "an atom has more than 16 bonds";
        return DPD_E_ARG;
    }
    if (P_ > DPD_J_MASK) {
        err = "too many particles in one engine (the list entry holds 27 bits of slot index)";
        return DPD_E_ARG;
    }
    return DPD_OK;
}

int Engine::init(std::vector<Replica>&& reps, const dpd_tuning* tune)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        err = "no CUDA device available (this engine has no CPU fallback)";
        return DPD_E_NODEV;
    }
    // one process per GPU: DPD_B200_DEVICE picks this process's device (the library's
    // own CUDA runtime does not see a device chosen through another runtime copy)
    if (const char* dv = std::getenv("DPD_B200_DEVICE")) {
        const int dev = std::atoi(dv);
        if (dev < 0 || dev >= ndev) {
            err = "DPD_B200_DEVICE is not a device index";
            return DPD_E_NODEV;
        }
        CK(cudaSetDevice(dev));
    }
    reps_ = std::move(reps);
    if (reps_.empty()) {
        err = "no replicas";
        return DPD_E_ARG;
    }
    tune_ = tune ? *tune : engine_default_tuning();
    int st = layout();
    if (st) return st;
    CK(cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, stream_priority_));
    st = alloc_and_upload();
    if (st) return st;
    host_target_.assign(reps_.size(), 0);
    return build_graph();
}

int Engine::alloc_and_upload()
{
    const int nrep = (int)reps_.size();
    int st;
#define DA(ptr, n) if ((st = dalloc(&ptr, (size_t)(n)))) return st
    DA(b_.reps, nrep);
    DA(b_.rstate, nrep);
    DA(b_.warp_rep, P_ / 32);
    DA(b_.crank, C_);
    int ncoeff = 0, nmass = 0, nbond = 0, nrdf = 0;
    for (auto& R : reps_) {
        ncoeff += R.desc.ntypes * R.desc.ntypes * 3;
        nmass += R.desc.ntypes;
        nbond += std::max(R.sys.n_bondtypes, 1);
        nrdf += R.ff.rdfs.empty() ? 0 : R.ff.rdfs[0].nbins;
    }
    DA(b_.coeff, ncoeff);
    DA(b_.mass, nmass);
    DA(b_.bondc, nbond);
    for (int q = 0; q < 2; q++) {
        DA(b_.pos[q], P_);
        DA(b_.vel[q], P_);
        DA(b_.bonds[q], (size_t)std::max(maxb_, 1) * P_);
    }
    DA(b_.parity, 1);
    DA(b_.force4, P_);
    DA(b_.last4, P_);
    DA(b_.rho, P_);
    DA(b_.cell_rep, C_);
    DA(b_.cell_lin, C_);
    DA(b_.cnt, C_);
    DA(b_.cstart, C_ + 1);
    DA(b_.ticket, 1);
    DA(b_.ticket2, 1);
    DA(b_.skey, P_);
    DA(b_.srank, P_);
    int64_t ntag = 0;
    for (auto& R : reps_) ntag += R.sys.n_atoms;
    DA(b_.tag2idx, ntag);
    DA(b_.img, ntag);
    DA(b_.ncount, P_);
    DA(b_.nlist, (size_t)P_ * nmax_);
    DA(b_.blocksum, (C_ + 4095) / 4096 + 1);
    DA(b_.acc, (size_t)nrep * DPD_ACC_SLOTS * DPD_NACC);
    DA(b_.ring, (size_t)nrep * DPD_RING_ROWS * DPD_THERMO_FIELDS);
    DA(b_.rdf_hist, nrdf);
    DA(b_.build_flag, 2);
    DA(b_.phase, 1);
    DA(b_.limit, nrep);
    if (!any_mdpd_) {  // pair schedule 11: at most one tile per cell
        DA(b_.tile_rep, C_);
        DA(b_.tile_code, C_);
    }
#undef DA
    {
        std::vector<uint32_t> lim(nrep, 0xFFFFFFFFu);
        CK(cudaMemcpyAsync(b_.limit, lim.data(), sizeof(uint32_t) * nrep, cudaMemcpyHostToDevice, stream_));
        CK(cudaStreamSynchronize(stream_));
    }
    // tables
    std::vector<RepDesc> hd(nrep);
    std::vector<int> wrep(P_ / 32), cell_rep(C_, 0);
    std::vector<float4> coeff(ncoeff);
    std::vector<float2> mass(nmass);
    std::vector<float4> bondc(nbond);
    for (int r = 0; r < nrep; r++) {
        const Replica& R = reps_[r];
        const RepDesc& d = R.desc;
        hd[r] = d;
        for (int wv = d.p_begin / 32; wv < d.p_cap_end / 32; wv++) wrep[wv] = r;
        for (int c = 0; c <= d.ncell; c++) cell_rep[d.c_begin + c] = r;
        const int nt = d.ntypes;
        const double sig_scale = std::sqrt(2.0 * R.ff.temp) / std::sqrt(R.in.dt);
        for (int ti = 0; ti < nt; ti++)
            for (int tj = 0; tj < nt; tj++) {
                const auto& c = R.ff.coeff[tri_index(ti + 1, tj + 1, nt)];
                const double A = c[0], B = c[1], gamma = c[2], rc = c[3], rd = c[4];
                const size_t o = d.coeff_off + (size_t)(ti * nt + tj) * 3;
                const float rcf = (float)rc;
                coeff[o] = make_float4((float)A, (float)gamma, (float)(std::sqrt(gamma) * sig_scale), rcf * rcf);
                coeff[o + 1] = make_float4((float)(1.0 / rc), (float)(0.5 * A * rc), (float)B,
                                           rd > 0 ? (float)(1.0 / rd) : 0.0f);
                const float rdf = (float)rd;
                coeff[o + 2] = make_float4(rdf * rdf, (float)(0.25 * B * rd),
                                           rd > 0 ? (float)(15.0 / (2.0 * M_PI * rd * rd * rd)) : 0.0f, rcf);
            }
        for (int t = 0; t < nt; t++) mass[d.mass_off + t] = make_float2((float)R.sys.masses[t], (float)(1.0 / R.sys.masses[t]));
        for (int b = 0; b < std::max(R.sys.n_bondtypes, 1); b++) {
            if (b < (int)R.ff.bond_coeff.size()) {
                const auto& c = R.ff.bond_coeff[b];
                bondc[d.bond_off + b] = make_float4((float)c[0], (float)c[1], (float)c[2], (float)c[3]);
            } else {
                bondc[d.bond_off + b] = make_float4(0, 0, 0, 0);
            }
        }
    }
    CK(cudaMemcpyAsync(b_.reps, hd.data(), sizeof(RepDesc) * nrep, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(b_.warp_rep, wrep.data(), sizeof(int) * wrep.size(), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(b_.cell_rep, cell_rep.data(), sizeof(int) * C_, cudaMemcpyHostToDevice, stream_));
    if ((st = upload_ranks())) return st;
    CK(cudaMemcpyAsync(b_.coeff, coeff.data(), sizeof(float4) * ncoeff, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(b_.mass, mass.data(), sizeof(float2) * nmass, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(b_.bondc, bondc.data(), sizeof(float4) * nbond, cudaMemcpyHostToDevice, stream_));
    // harmonic angles (atom_style angle): a static table in global tag indices
    {
        std::vector<int4> tbl;
        std::vector<float4> acoef;
        std::vector<int> awrep;
        for (int r = 0; r < nrep; r++) {
            const Replica& R = reps_[r];
            if (R.ff.angle_style != 1 || R.sys.angles.empty()) continue;
            const int off = (int)acoef.size();
            for (const auto& c : R.ff.angle_coeff) {
                const double th0 = c[1] * (M_PI / 180.0);
                acoef.push_back(make_float4((float)c[0], (float)th0, (float)std::cos(th0), (float)std::sin(th0)));
            }
            const int tb = R.desc.tag_base;
            for (size_t q = 0; q < R.sys.angles.size() / 4; q++) {
                const int* a = &R.sys.angles[4 * q];
                tbl.push_back(make_int4(off + a[0] - 1, tb + a[1] - 1, tb + a[2] - 1, tb + a[3] - 1));
            }
            while (tbl.size() % 32) tbl.push_back(make_int4(-1, 0, 0, 0));
            while (awrep.size() < tbl.size() / 32) awrep.push_back(r);
        }
        nang_ = (int)tbl.size();
        if (nang_ > 0) {
            if ((st = dalloc(&angle_tbl_, tbl.size()))) return st;
            if ((st = dalloc(&angle_coef_, acoef.size()))) return st;
            if ((st = dalloc(&angle_wrep_, awrep.size()))) return st;
            CK(cudaMemcpyAsync(angle_tbl_, tbl.data(), sizeof(int4) * tbl.size(), cudaMemcpyHostToDevice, stream_));
            CK(cudaMemcpyAsync(angle_coef_, acoef.data(), sizeof(float4) * acoef.size(), cudaMemcpyHostToDevice, stream_));
            CK(cudaMemcpyAsync(angle_wrep_, awrep.data(), sizeof(int) * awrep.size(), cudaMemcpyHostToDevice, stream_));
            CK(cudaStreamSynchronize(stream_));
        }
    }
    // group fixes (spring, rvcm, recenter): group masses in FP64 from the type counts
    {
        std::vector<FixDesc> fd(nrep);
        bool spring_file = false;
        any_spring_ = any_eos_ = any_motion_ = any_twowall_ = false;
        for (int r = 0; r < nrep; r++) {
            const Replica& R = reps_[r];
            FixDesc& f = fd[r];
            memset(&f, 0, sizeof(f));
            auto gmass = [&](uint32_t mask) {
                double m = 0.0;
                for (int i = 0; i < R.sys.n_atoms; i++) {
                    const int t = R.sys.type[i];
                    if ((mask >> (t - 1)) & 1u) m += R.sys.masses[t - 1];
                }
                return m;
            };
            for (int k = 0; k < 3; k++) f.L[k] = R.box_len[k];
            if (R.ff.spring.on && R.ff.spring.mask) {
                f.spring_mask = R.ff.spring.mask;
                f.spring_k = R.ff.spring.k;
                for (int k = 0; k < 3; k++) f.spring_c[k] = R.ff.spring.c[k];
                f.spring_r0 = R.ff.spring.r0;
                f.spring_m = gmass(f.spring_mask);
                f.spring_file_f = R.ff.spring.file_freq;
                spring_file |= f.spring_file_f != 0;
                any_spring_ = true;
            }
            if (R.ff.rvcm.on && R.ff.rvcm.mask) {
                f.rvcm_mask = R.ff.rvcm.mask;
                f.rvcm_freq = R.ff.rvcm.freq;
                for (int k = 0; k < 3; k++) f.rvcm_flag[k] = R.ff.rvcm.flag[k];
                f.rvcm_m = gmass(f.rvcm_mask);
                any_eos_ = true;
            }
            if (R.ff.recenter.on && R.ff.recenter.mask) {
                f.recenter_mask = R.ff.recenter.mask;
                f.recenter_freq = R.ff.recenter.freq;
                for (int k = 0; k < 3; k++) f.recenter_c[k] = R.ff.recenter.c[k];
                f.recenter_m = gmass(f.recenter_mask);
                any_eos_ = true;
            }
            f.n_move = (int)R.ff.moves.size();
            for (int k = 0; k < f.n_move; k++) {
                f.move_mask[k] = R.ff.moves[k].mask;
                for (int q = 0; q < 3; q++) f.move_v[k][q] = (float)R.ff.moves[k].v[q];
            }
            f.n_reflect = (int)R.ff.reflects.size();
            for (int k = 0; k < f.n_reflect; k++) {
                const FixWallReflect& w = R.ff.reflects[k];
                f.refl_mask[k] = w.mask;
                f.refl_dir[k] = w.dir;
                f.refl_lo[k] = (float)w.lo;
                f.refl_hi[k] = (float)w.hi;
            }
            f.n_twowall = (int)R.ff.twowalls.size();
            for (int k = 0; k < f.n_twowall; k++) {
                const FixTwoWall& w = R.ff.twowalls[k];
                f.tw_mask[k] = w.mask;
                f.tw_lo[k] = w.lo_mask;
                f.tw_hi[k] = w.hi_mask;
                f.tw_dir[k] = w.dir;
            }
            if (f.n_move || f.n_reflect) any_motion_ = true;
            if (f.n_twowall) any_twowall_ = true;
        }
        if (any_spring_ || any_eos_ || any_motion_ || any_twowall_) {
            if ((st = dalloc(&b_.fix, nrep))) return st;
            if ((st = dalloc(&b_.fixo, nrep))) return st;
            if (spring_file && (st = dalloc(&b_.spring_ring, (size_t)nrep * DPD_RING_ROWS * 6))) return st;
            CK(cudaMemcpyAsync(b_.fix, fd.data(), sizeof(FixDesc) * nrep, cudaMemcpyHostToDevice, stream_));
            CK(cudaStreamSynchronize(stream_));
        }
    }
    // group computes: descriptors, initial unwrapped positions by global tag, row rings
    gc_ring_base_.assign(nrep, 0);
    any_wallc_ = false;
    if (any_gc_) {
        std::vector<GCDesc> gd((size_t)nrep * DPD_MAX_GC);
        memset(gd.data(), 0, sizeof(GCDesc) * gd.size());
        std::vector<float4> uw0;
        int ring = 0;
        for (int r = 0; r < nrep; r++) {
            const Replica& R = reps_[r];
            gc_ring_base_[r] = ring;
            for (size_t k = 0; k < R.ff.gcs.size(); k++) {
                const GroupCompute& c = R.ff.gcs[k];
                GCDesc& g = gd[(size_t)r * DPD_MAX_GC + k];
                g.kind = c.kind;
                g.mask = c.type_mask;
                g.freq = c.frequency;
                g.ring = ring++;
                int64_t ng = 0;
                for (int i = 0; i < R.sys.n_atoms; i++) ng += (c.type_mask >> (R.sys.type[i] - 1)) & 1u;
                for (int q = 0; q < 6; q++) g.region[q] = c.region[q];
                for (int q = 0; q < 3; q++) g.L[q] = R.box_len[q];
                if (c.kind == GC_TEMP) g.norm = ng > 1 ? 1.0 / (3.0 * ng - 3.0) : 0.0;
                if (c.kind == GC_MSD) g.norm = ng > 0 ? 1.0 / ng : 0.0;
                if (c.kind == GC_RHO)
                    g.norm = 1.0 / ((c.region[1] - c.region[0]) * (c.region[3] - c.region[2]) * (c.region[5] - c.region[4]));
                if (c.kind == GC_WALL) {
                    g.norm = 1.0;
                    g.wall_mask = c.wall_mask;
                    g.wall_side = c.wall_side;
                    g.wall_dir = c.wall_dir;
                    g.cutoff = (float)c.cutoff;
                    g.box_lo = (float)R.sys.lo[c.wall_dir];
                    g.box_hi = (float)R.sys.hi[c.wall_dir];
                    any_wallc_ = true;
                }
            }
            // initial unwrapped positions: the data file's positions wrapped into the box
            for (int i = 0; i < R.sys.n_atoms; i++) {
                float q[3];
                for (int k = 0; k < 3; k++) {
                    double x = R.sys.x[3 * (size_t)i + k] - R.desc.lo[k];
                    x -= R.box_len[k] * std::floor(x / R.box_len[k]);
                    q[k] = (float)(R.desc.lo[k] + x);
                }
                uw0.push_back(make_float4(q[0], q[1], q[2], 0.0f));
            }
        }
        if ((st = dalloc(&b_.gc, gd.size()))) return st;
        if ((st = dalloc(&b_.uw0, uw0.size()))) return st;
        if ((st = dalloc(&b_.gc_ring, (size_t)ring * DPD_RING_ROWS * 4))) return st;
        if ((st = dalloc(&b_.gc_count, ring))) return st;
        CK(cudaMemcpyAsync(b_.gc, gd.data(), sizeof(GCDesc) * gd.size(), cudaMemcpyHostToDevice, stream_));
        CK(cudaMemcpyAsync(b_.uw0, uw0.data(), sizeof(float4) * uw0.size(), cudaMemcpyHostToDevice, stream_));
        CK(cudaStreamSynchronize(stream_));
    }
    if ((any_twowall_ || any_wallc_) && (st = dalloc(&b_.wall_ext, (size_t)nrep * 8))) return st;
    std::vector<RepState> rs(nrep);
    for (auto& s : rs) {
        memset(&s, 0, sizeof(s));
        s.zero_pending = 1;
    }
    CK(cudaMemcpyAsync(b_.rstate, rs.data(), sizeof(RepState) * nrep, cudaMemcpyHostToDevice, stream_));
    int st2 = upload_particles();
    if (st2) return st2;
    CK(cudaStreamSynchronize(stream_));
    return DPD_OK;
}

int Engine::staging()
{
    if (h_pos_) return DPD_OK;
    CK(cudaMallocHost((void**)&h_pos_, sizeof(float4) * P_));
    CK(cudaMallocHost((void**)&h_vel_, sizeof(float4) * P_));
    CK(cudaMallocHost((void**)&h_frc_, sizeof(float4) * P_));
    CK(cudaMallocHost((void**)&h_img_, sizeof(int4) * P_));
    return DPD_OK;
}

// Convert the FP64 state of every replica into the cell-offset representation and
// upload it (tag order) into buffer 0.  The bond partner table is built once, kept on
// the device in tag order, and copied on later uploads.
int Engine::upload_particles()
{
    int st = staging();
    if (st) return st;
    float4* pos = h_pos_;
    float4* vel = h_vel_;
    const bool first = !bonds_tag_;
    std::vector<int2> bonds;
    if (first) bonds.assign((size_t)std::max(maxb_, 1) * P_, make_int2(0, 0));
    for (auto& R : reps_) {
        const RepDesc& d = R.desc;
        const int n = R.sys.n_atoms;
        parallel_for(n, [&](int64_t i0, int64_t i1) {
        for (int64_t i = i0; i < i1; i++) {
            const int s = d.p_begin + i;
            int c[3];
            float o[3];
            for (int k = 0; k < 3; k++) {
                double x = R.sys.x[3 * (size_t)i + k] - d.lo[k];
                if (!std::isfinite(x)) {
                    // kept non-finite: the first list build flags the replica
                    // (DPD_E_NUMERIC) instead of binning garbage
                    c[k] = 0;
                    o[k] = NAN;
                    continue;
                }
                const double L = R.box_len[k];
                if (x >= L || x < 0) x -= L * std::floor(x / L);
                int cc = (int)std::floor(x / (double)d.w[k]);
                cc = std::min(std::max(cc, 0), d.nc[k] - 1);
                double off = x - (double)cc * (double)d.w[k];
                float of = (float)off;
                if (of >= d.w[k]) of = std::nextafter(d.w[k], 0.0f);
                if (of < 0.0f) of = 0.0f;
                c[k] = cc;
                o[k] = of;
            }
            int code = c[0] | (c[1] << DPD_CELL_BITS) | (c[2] << (2 * DPD_CELL_BITS));
            float codef;
            memcpy(&codef, &code, 4);
            pos[s] = make_float4(o[0], o[1], o[2], codef);
            const int tagw = ((i + 1) << DPD_TYPE_BITS) | (R.sys.type[i] - 1);
            float tagf;
            memcpy(&tagf, &tagw, 4);
            vel[s] = make_float4((float)R.sys.v[3 * (size_t)i], (float)R.sys.v[3 * (size_t)i + 1],
                                 (float)R.sys.v[3 * (size_t)i + 2], tagf);
        }
        });
        if (first && d.bond_style) {
            std::vector<int> deg(n, 0);
            for (int b = 0; b < R.sys.n_bonds; b++) {
                const int ty = R.sys.bonds[3 * b], ta = R.sys.bonds[3 * b + 1], tb = R.sys.bonds[3 * b + 2];
                const int ia = ta - 1, ib = tb - 1;
                bonds[(size_t)deg[ia] * P_ + d.p_begin + ia] = make_int2(tb, ty);
                deg[ia]++;
                bonds[(size_t)deg[ib] * P_ + d.p_begin + ib] = make_int2(ta, ty);
                deg[ib]++;
            }
        }
        for (int s = d.p_end; s < d.p_cap_end; s++) {
            pos[s] = make_float4(0, 0, 0, 0);
            vel[s] = make_float4(0, 0, 0, 0);
        }
    }
    // the state goes into buffer 0, which becomes the current one
    const size_t nb = (size_t)std::max(maxb_, 1) * P_;
    if (first) {
        if ((st = dalloc(&bonds_tag_, nb))) return st;
        CK(cudaMemcpyAsync(bonds_tag_, bonds.data(), sizeof(int2) * nb, cudaMemcpyHostToDevice, stream_));
    }
    CK(cudaMemcpyAsync(b_.pos[0], pos, sizeof(float4) * P_, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(b_.vel[0], vel, sizeof(float4) * P_, cudaMemcpyHostToDevice, stream_));
    {
        int64_t ntag = 0;
        for (auto& R : reps_) ntag += R.sys.n_atoms;
        CK(cudaMemsetAsync(b_.img, 0, sizeof(int4) * ntag, stream_));
    }
    CK(cudaMemcpyAsync(b_.bonds[0], bonds_tag_, sizeof(int2) * nb, cudaMemcpyDeviceToDevice, stream_));
    CK(cudaMemsetAsync(b_.parity, 0, sizeof(int), stream_));
    // slots are in tag order until the first build
    {
        std::vector<int> t2i;
        for (auto& R : reps_)
            for (int t = 0; t < R.sys.n_atoms; t++) t2i.push_back(R.desc.p_begin + t);
        CK(cudaMemcpyAsync(b_.tag2idx, t2i.data(), sizeof(int) * t2i.size(), cudaMemcpyHostToDevice, stream_));
        CK(cudaStreamSynchronize(stream_));
    }
    aos_built_ = false;
    CK(cudaMemsetAsync(b_.force4, 0, sizeof(float4) * P_, stream_));
    CK(cudaMemsetAsync(b_.rho, 0, sizeof(float) * P_, stream_));
    CK(cudaStreamSynchronize(stream_));
    return DPD_OK;
}

// ---------------------------------------------------------------------------------
static BuildArgs build_args(const DeviceBuffers& b, int P, int C, int nmax, int maxb)
{
    BuildArgs a;
    a.reps = b.reps;
    a.warp_rep = b.warp_rep;
    a.crank = b.crank;
    a.P = P;
    a.C = C;
    a.nmax = nmax;
    a.maxb = maxb;
    a.build_flag = b.build_flag;
    a.phase = b.phase;
    a.parity = b.parity;
    a.cell_rep = b.cell_rep;
    a.cell_lin = b.cell_lin;
    for (int q = 0; q < 2; q++) {
        a.buf.pos[q] = b.pos[q];
        a.buf.vel[q] = b.vel[q];
        a.buf.bonds[q] = b.bonds[q];
    }
    a.buf.img = b.img;
    a.last4 = b.last4;
    a.cnt = b.cnt;
    a.cstart = b.cstart;
    a.skey = b.skey;
    a.srank = b.srank;
    a.tag2idx = b.tag2idx;
    a.ncount = b.ncount;
    a.nlist = b.nlist;
    a.rstate = b.rstate;
    a.blocksum = b.blocksum;
    a.ticket = b.ticket;
    return a;
}

static StepArgs step_args(const DeviceBuffers& b, int P, int nmax, int maxb, int nrep)
{
    StepArgs a;
    a.reps = b.reps;
    a.warp_rep = b.warp_rep;
    a.rstate = b.rstate;
    a.P = P;
    a.nmax = nmax;
    a.maxb = maxb;
    a.coeff = b.coeff;
    a.mass = b.mass;
    a.bondc = b.bondc;
    for (int q = 0; q < 2; q++) {
        a.buf.pos[q] = b.pos[q];
        a.buf.vel[q] = b.vel[q];
        a.buf.bonds[q] = b.bonds[q];
    }
    a.buf.img = b.img;
    a.parity = b.parity;
    a.force4 = b.force4;
    a.rho = b.rho;
    a.last4 = b.last4;
    a.tag2idx = b.tag2idx;
    a.ncount = b.ncount;
    a.nlist = b.nlist;
    a.acc = b.acc;
    a.ring = b.ring;
    a.rdf_hist = b.rdf_hist;
    a.cstart = b.cstart;
    a.crank = b.crank;
    a.build_flag = b.build_flag;
    a.phase = b.phase;
    a.nrep = nrep;
    a.mode = 0;
    a.fix = b.fix;
    a.fixo = b.fixo;
    a.spring_ring = b.spring_ring;
    a.gc = b.gc;
    a.uw0 = b.uw0;
    a.gc_ring = b.gc_ring;
    a.gc_count = b.gc_count;
    a.wall_ext = b.wall_ext;
    a.ticket = b.ticket2;
    return a;
}

// Launch with programmatic dependent launch allowed: in a captured graph the kernel's
// launch overlaps the tail of its predecessor (every step kernel starts with
// griddep_wait(), which orders it after the predecessor's memory).
template <typename... KArgs, typename... Args>
static void pdl_launch(void (*kern)(KArgs...), int grid, int block, cudaStream_t s, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// the same with dynamic shared memory
template <typename... KArgs, typename... Args>
static void pdl_launch_smem(void (*kern)(KArgs...), int grid, int block, size_t smem, cudaStream_t s,
                            Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

template <int STYLE, bool BONDS>
static void launch_pair2(int variant, int grid, cudaStream_t s, const StepArgs& a)
{
    if (variant == 0) pdl_launch(k_pair<STYLE, BONDS>, grid, 256, s, a);
    else if (variant == 2) pdl_launch(k_pair_q<STYLE, BONDS, 4, true>, grid, 256, s, a);
    else if (variant == 3) pdl_launch(k_pair_q<STYLE, BONDS, 3, false>, grid, 256, s, a);
    else if (variant == 4) pdl_launch(k_pair_flat<STYLE, BONDS, 4>, grid, 256, s, a);
    else if (variant == 5) pdl_launch(k_pair_flat<STYLE, BONDS, 3>, grid, 256, s, a);
    else if (variant == 6) pdl_launch(k_pair_flat<STYLE, BONDS, 4>, grid, 256, s, a);
    else if (variant == 7) {
        pdl_launch(k_pair_flat_split<STYLE, BONDS, 0, 6>, grid, 256, s, a);
        pdl_launch(k_pair_flat_split<STYLE, BONDS, 1, 4>, grid, 256, s, a);
    } else if (variant == 8) {
        pdl_launch(k_pair_flat_split<STYLE, BONDS, 0, 5>, grid, 256, s, a);
        pdl_launch(k_pair_flat_logsteps<STYLE, BONDS>, std::min(grid, 148 * 4), 256, s, a);
    } else if (variant == 9) {
        pdl_launch(k_pair_flat_split<STYLE, BONDS, 0, 5, true>, grid, 256, s, a);
        pdl_launch(k_pair_flat_logsteps<STYLE, BONDS, true>, std::min(grid, 148 * 4), 256, s, a);
    } else if (variant == 10) {
        pdl_launch(k_pair_entry<STYLE, BONDS>, (a.nmax * (a.P >> 5) + 7) / 8, 256, s, a);
    }
    else pdl_launch(k_pair_q<STYLE, BONDS, 4, false>, grid, 256, s, a);
}

// pair_variant 0: thread per particle; 1: warp pair-queue, i-side and
// j-side forces by float4 reductions in L2, 4 blocks/SM; 2: warp pair-queue with the
// i-side reduced through shared-memory atomics; 3: as 1 with 3 blocks/SM; 4: flattened
// warp schedule, 4 blocks/SM; 5: flattened, 3 blocks/SM; 6: the flattened schedule with
// the list build fused into it (DPD; mDPD falls back to 4); 7 and 8 (the default): the
// flattened schedule as two launches, non-log steps without FP64 sums at 6 (7) or 5 (8)
// blocks/SM, log steps at 4; 9: as 8 with the i-side forces summed per owner in the warp;
// 10: one thread per list entry (small grids); 11 (DPD engines): no list, the cell-tile
// kernel (kernels_tile.cuh) after the counting sort
template <int STYLE>
static void launch_pair(int variant, bool bonds, int grid, cudaStream_t s, const StepArgs& a)
{
    if (bonds) launch_pair2<STYLE, true>(variant, grid, s, a);
    else launch_pair2<STYLE, false>(variant, grid, s, a);
}

// The list-build chain; every kernel returns at once unless this phase's flag is set.
void Engine::enqueue_build(cudaStream_t s, bool list, bool wide)
{
    const int nrep = (int)reps_.size();
    BuildArgs ba = build_args(b_, P_, C_, nmax_, maxb_);
    const int gp = (P_ + 255) / 256;
    const int gc = (C_ + 255) / 256;
    const int nsb = (C_ + 4095) / 4096;
    pdl_launch(k_bin_count, gp, 256, s, ba);
    if (nsb == 1) {
        pdl_launch(k_scan_blocks<true>, 1, 1024, s, ba);
    } else {
        pdl_launch(k_scan_blocks<false>, nsb, 1024, s, ba);
        pdl_launch(k_scan_sums, 1, 1024, s, ba, nsb);
        pdl_launch(k_scan_add, gc, 256, s, ba);
    }
    if (gp <= 148 * 8) {
        pdl_launch(k_permute<true>, gp, 256, s, ba, nrep);
    } else {
        pdl_launch(k_permute<false>, gp, 256, s, ba, nrep);
        pdl_launch(k_flip, (nrep + 255) / 256, 256, s, ba, nrep);
    }
    if (list) {
        if (tile_build()) {
            const StepArgs sa = step_args(b_, P_, nmax_, maxb_, nrep);
            const TileArgs ta{b_.tile_rep, b_.tile_code, ntiles_, tile_edge_, tile_smax_, 0};
            pdl_launch_smem(k_tile_build<5>, ntiles_, 256, tile_smem_bytes(tile_smax_, 0), s, sa, ta, ba);
        } else if (wide && gp <= 148 * 8) pdl_launch(k_build_wide, (14 * P_ + 255) / 256, 256, s, ba);
        else if (tune_.build_variant == 1) pdl_launch(k_build_nlist_s<6>, gp, 256, s, ba);
        else if (tune_.build_variant == 2) pdl_launch(k_build_nlist_s<8>, gp, 256, s, ba);
        else if (tune_.build_variant == 5) pdl_launch(k_build_cols, gp, 256, s, ba);
        else pdl_launch(k_build_nlist, gp, 256, s, ba);
    }
}

void Engine::enqueue_step(cudaStream_t s, cudaEvent_t ev0, cudaEvent_t ev1)
{
    const int nrep = (int)reps_.size();
    StepArgs sa = step_args(b_, P_, nmax_, maxb_, nrep);
    const int gp = (P_ + 255) / 256;
    // small grids: fewer, larger launches (the pair pass and the integrate each in one)
    const bool small = tune_.launch_mode == 2 || ((tune_.launch_mode == 0 || tune_.launch_mode == 3) && gp <= 148 * 8);
    // tiny grids (at most one block of 256 slots per SM): the list build with a thread per
    // (slot, stencil cell) and the pair pass with a thread per list entry; past that their
    // idle lanes cost more than the parallelism gains.  launch_mode 3 leaves them out: an
    // engine that shares the GPU with others (a server's cohorts) gains more from leaving
    // SMs to them than from spreading its own few pairs
    const bool tiny = small && gp <= 148 && tune_.launch_mode != 3;
    // schedule 11: no neighbour list, the cell-tile kernel after the counting sort
    const bool tile = use_tile();
    const int variant = tile ? 11 : (small && tune_.pair_variant == 8 ? (tiny ? 10 : 4) : tune_.pair_variant);
    // schedule 6: the DPD list build runs inside the pair kernel
    const bool fused = variant == 6 && !any_mdpd_;
    enqueue_build(s, !fused && !tile,
                  (tiny && (tune_.build_variant == 0 || tune_.build_variant == 5)) || tune_.build_variant == 3);
    if (any_mdpd_) pdl_launch(k_density, gp, 256, s, sa);
    if (ev0) cudaEventRecordWithFlags(ev0, s, cudaEventRecordExternal);
    if (tile) {
        const TileArgs ta{b_.tile_rep, b_.tile_code, ntiles_, tile_edge_, tile_smax_, tile_hc_};
        const size_t sm = tile_smem_bytes(tile_smax_, tile_hc_);
        const int glog = std::min(ntiles_, 148 * 2);
        // pair_block 3: the kernel compiled for 3 CTAs per SM (more registers), else 4
        const bool b3 = tune_.pair_block == 3;
        if (bonds_) {
            if (b3) pdl_launch_smem(k_tile<true, 3>, ntiles_, 256, sm, s, sa, ta);
            else pdl_launch_smem(k_tile<true, 4>, ntiles_, 256, sm, s, sa, ta);
            pdl_launch_smem(k_tile_logsteps<true>, glog, 256, sm, s, sa, ta);
        } else {
            if (b3) pdl_launch_smem(k_tile<false, 3>, ntiles_, 256, sm, s, sa, ta);
            else pdl_launch_smem(k_tile<false, 4>, ntiles_, 256, sm, s, sa, ta);
            pdl_launch_smem(k_tile_logsteps<false>, glog, 256, sm, s, sa, ta);
        }
    } else if (fused) {
        const BuildArgs ba = build_args(b_, P_, C_, nmax_, maxb_);
        if (bonds_) pdl_launch(k_build_pair<true, 4>, gp, 256, s, sa, ba);
        else pdl_launch(k_build_pair<false, 4>, gp, 256, s, sa, ba);
    } else if (any_dpd_) {
        launch_pair<0>(variant, bonds_, gp, s, sa);
    }
    if (any_mdpd_) launch_pair<1>(variant, bonds_, gp, s, sa);
    if (ev1) cudaEventRecordWithFlags(ev1, s, cudaEventRecordExternal);
    if (nang_ > 0) pdl_launch(k_angle, (nang_ + 255) / 256, 256, s, sa, angle_tbl_, angle_coef_, angle_wrep_, nang_);
    if (rdf_) pdl_launch(k_rdf, gp, 256, s, sa);
    const int gr = (nrep + 255) / 256;
    if (any_spring_) {
        // post_force: the spring acts on the forces of this step
        pdl_launch(k_fix_sums<0>, gp, 256, s, sa);
        pdl_launch(k_fix_reduce<0>, gr, 256, s, sa);
    }
    if (any_eos_) {
        // end_of_step: final half kick, group sums and the rvcm / recenter corrections
        pdl_launch(k_fix_sums<1>, gp, 256, s, sa);
        pdl_launch(k_fix_reduce<1>, gr, 256, s, sa);
    }
    if (any_wallc_) {
        // wall_contact computes: wall extents of the end-of-step positions
        pdl_launch(k_wall_reset<1>, gr, 256, s, sa);
        pdl_launch(k_wall_extent<1>, gp, 256, s, sa);
    }
    if (small && !any_twowall_) {
        // the step's bookkeeping runs in the integrate's last block
        if (ext()) pdl_launch(k_integrate_adv<true>, gp, 256, s, sa);
        else pdl_launch(k_integrate_adv<false>, gp, 256, s, sa);
        return;
    }
    if (ext()) {
        pdl_launch(k_integrate_nolog<true>, gp, 256, s, sa);
        pdl_launch(k_integrate_logsteps<true>, std::min(gp, 148 * 4), 256, s, sa);
    } else {
        pdl_launch(k_integrate_nolog<false>, gp, 256, s, sa);
        pdl_launch(k_integrate_logsteps<false>, std::min(gp, 148 * 4), 256, s, sa);
    }
    if (any_twowall_) enqueue_two_wall(s, sa);
    pdl_launch(k_advance, (nrep * 32 + 255) / 256, 256, s, sa);
}

// fix two_wall after a drift: wall extents, then the reflection of the group
void Engine::enqueue_two_wall(cudaStream_t s, const StepArgs& sa)
{
    const int gp = (P_ + 255) / 256, gr = ((int)reps_.size() + 255) / 256;
    pdl_launch(k_wall_reset<0>, gr, 256, s, sa);
    pdl_launch(k_wall_extent<0>, gp, 256, s, sa);
    pdl_launch(k_two_wall, gp, 256, s, sa);
}

void Engine::enqueue_integrate_initial(cudaStream_t s)
{
    StepArgs sa = step_args(b_, P_, nmax_, maxb_, (int)reps_.size());
    sa.mode = 1;
    if (ext()) k_integrate<true><<<(P_ + 255) / 256, 256, 0, s>>>(sa);
    else k_integrate<false><<<(P_ + 255) / 256, 256, 0, s>>>(sa);
    if (any_twowall_) enqueue_two_wall(s, sa);
}

// The tile table of pair schedule 11: the tiles of every replica (edge^3 home cells,
// fewer at a grid's edge), each replica's tiles in Morton order of their coordinates
// (neighbouring tiles run close in time, whatever the cell order of the slots), the staging capacity of a CTA: 1.5 times the mean particle
// count of a tile's neighbourhood (plus 64) in the densest replica, and the pairs a
// particle may have (the list capacity max_rho implies at the largest cutoff, 16..96).  Edge 0
// (the default) takes the largest edge up to 4 that still gives at least 8 tiles per
// SM, else 1.
int Engine::prepare_tiles()
{
    ntiles_ = 0;
    if (!use_tile() && !tile_build()) return DPD_OK;
    auto count = [&](int E) {
        int64_t n = 0;
        for (auto& R : reps_) {
            const RepDesc& d = R.desc;
            n += (int64_t)((d.nc[0] + E - 1) / E) * ((d.nc[1] + E - 1) / E) * ((d.nc[2] + E - 1) / E);
        }
        return n;
    };
    int E = tune_.tile;
    if (E <= 0) {
        E = 1;
        for (int e = 4; e >= 2; e--)
            if (count(e) >= 148 * 8) {
                E = e;
                break;
            }
    }
    E = std::min(E, TILE_MAX_EDGE);
    std::vector<int> trep, tcode;
    int smax = 128, hc = 0;
    for (int r = 0; r < (int)reps_.size(); r++) {
        const RepDesc& d = reps_[r].desc;
        const int nt[3] = {(d.nc[0] + E - 1) / E, (d.nc[1] + E - 1) / E, (d.nc[2] + E - 1) / E};
        std::vector<std::pair<uint32_t, int>> order;
        for (int x = 0; x < nt[0]; x++)
            for (int y = 0; y < nt[1]; y++)
                for (int z = 0; z < nt[2]; z++) order.push_back({morton3(x, y, z), x | (y << 10) | (z << 20)});
        std::sort(order.begin(), order.end());
        for (auto& o : order) {
            trep.push_back(r);
            tcode.push_back(o.second);
        }
        const double mean_cell = (double)d.n_real / std::max(d.ncell, 1);
        const int region = (std::min(E, d.nc[0]) + 2) * (std::min(E, d.nc[1]) + 2) * (std::min(E, d.nc[2]) + 1);
        smax = std::max(smax, (int)std::ceil(1.5 * mean_cell * region) + 64);
        // pairs a particle may have inside the largest cutoff: the reference's list
        // capacity rule (src/force/neigh_list.cu:14-17) at that cutoff
        const double rcm = std::sqrt((double)d.rcmax2);
        hc = std::max(hc, ((int)(reps_[r].in.max_rho * 4.0 / 3.0 * M_PI * rcm * rcm * rcm) + 1 + 15) / 16 * 16);
    }
    hc = std::min(96, std::max(16, hc));
    if (tune_.tile_capacity > 0) smax = tune_.tile_capacity;
    smax = (smax + 31) / 32 * 32;
    // at most 200 KB of shared memory a CTA (a neighbourhood beyond it takes its home
    // cells one at a time)
    while (smax > 32 && tile_smem_bytes(smax, hc) > 200 * 1024) smax -= 32;
    if ((int64_t)trep.size() > C_) {
        err = "tile table larger than the cell count";
        return DPD_E_STATE;
    }
    ntiles_ = (int)trep.size();
    tile_edge_ = E;
    tile_smax_ = smax;
    tile_hc_ = hc;
    CK(cudaMemcpyAsync(b_.tile_rep, trep.data(), sizeof(int) * trep.size(), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(b_.tile_code, tcode.data(), sizeof(int) * tcode.size(), cudaMemcpyHostToDevice, stream_));
    CK(cudaStreamSynchronize(stream_));
    const int bytes = (int)tile_smem_bytes(smax, hc);
    CK(cudaFuncSetAttribute(k_tile<true, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaFuncSetAttribute(k_tile<false, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaFuncSetAttribute(k_tile<true, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaFuncSetAttribute(k_tile<false, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaFuncSetAttribute(k_tile_build<5>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)tile_smem_bytes(smax, 0)));
    CK(cudaFuncSetAttribute(k_tile_logsteps<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaFuncSetAttribute(k_tile_logsteps<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    return DPD_OK;
}

// the half list of the current state (cells of the last build), for get_neighbors and
// list_stats of an engine whose steps build none
int Engine::refresh_list()
{
    if (!use_tile()) return DPD_OK;
    const BuildArgs ba = build_args(b_, P_, C_, nmax_, maxb_);
    k_build_nlist_now<<<(P_ + 255) / 256, 256, 0, stream_>>>(ba);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
    return DPD_OK;
}

int Engine::build_graph()
{
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    {
        const int e = prepare_tiles();
        if (e) return e;
    }
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    enqueue_step(stream_, nullptr, nullptr);
    cudaError_t e = cudaStreamEndCapture(stream_, &g);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&graph_, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    CK(cudaGraphUpload(graph_, stream_));
    return DPD_OK;
}

// set the run target of every replica (absolute step), optionally mark the next
// evaluation as a zero step and raise the list-build flag of the current phase
__global__ void k_set_target(RepState* st, const uint32_t* limit, int nrep, uint32_t target, int zero,
                             int set_build, int* build_flag, const uint32_t* phase)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nrep) {
        st[r].target = min(target, limit[r]);
        if (zero) st[r].zero_pending = 1;
    }
    if (r == 0 && set_build) build_flag[(*phase) & 1] = 1;
}

int Engine::run_async(uint32_t nsteps)
{
    const int nrep = (int)reps_.size();
    const int g = (nrep + 255) / 256;
    // steps first..last: the zero step at next_step_ then nsteps steps, or nsteps steps.
    // A trajectory frame needs the state at the end of its step, so a run with dumps is
    // split into segments that end on dump steps (each later segment starts with the
    // initial half kick and drift that the fused integrate leaves to the next step).
    bool zero = zero_pending_;
    const uint32_t first = next_step_;
    const uint32_t last = zero ? next_step_ + nsteps : next_step_ - 1 + nsteps;
    if (!zero && nsteps == 0) return DPD_OK;
    uint32_t s = first;
    for (;;) {
        uint32_t end = last;
        for (auto& w : dumps_) end = std::min(end, next_dump(w.get(), s));
        if (ranks_dirty_) {
            const int e = upload_ranks();
            if (e) return e;
            ranks_dirty_ = false;
        }
        k_set_target<<<g, 256, 0, stream_>>>(b_.rstate, b_.limit, nrep, end, zero ? 1 : 0,
                                             zero || force_build_ ? 1 : 0, b_.build_flag, b_.phase);
        force_build_ = false;
        if (!zero) enqueue_integrate_initial(stream_);
        CK(cudaGetLastError());
        for (uint32_t k = s; k <= end; k++) CK(cudaGraphLaunch(graph_, stream_));
        zero = false;
        // the host's step counter follows each segment, so a failed frame write leaves
        // it where the device stopped
        next_step_ = end + 1;
        zero_pending_ = false;
        for (auto& w : dumps_)
            if (dump_due(w.get(), end)) {
                int e = dump_frame(w.get(), end);
                if (e) return e;
            }
        if (end == last) break;
        s = end + 1;
    }
    return DPD_OK;
}

int Engine::run(uint32_t nsteps)
{
    int e = run_async(nsteps);
    if (e) return e;
    return sync_and_check();
}

int Engine::read_rstate(std::vector<RepState>& st)
{
    st.resize(reps_.size());
    CK(cudaMemcpyAsync(st.data(), b_.rstate, sizeof(RepState) * st.size(), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    return DPD_OK;
}

int Engine::rstate_async(RepState* host)
{
    CK(cudaMemcpyAsync(host, b_.rstate, sizeof(RepState) * reps_.size(), cudaMemcpyDeviceToHost, stream_));
    return DPD_OK;
}

int Engine::sync_and_check()
{
    CK(cudaStreamSynchronize(stream_));
    CK(cudaGetLastError());
    std::vector<RepState> st;
    int e = read_rstate(st);
    if (e) return e;
    for (size_t r = 0; r < st.size(); r++) {
        const int code = status_error(st[r].status, (int)r);
        if (code) return code;
    }
    return DPD_OK;
}

int Engine::status_error(int s, int r)
{
    if (s & ST_LIST_OVERFLOW) {
        err = "neighbour list overflow in replica " + std::to_string(r) + ": increase max_rho in the neighbor command";
        return DPD_E_OVERFLOW;
    }
    if (s & ST_NONFINITE) {
        err = "non-finite (or runaway) position or velocity in replica " + std::to_string(r);
        return DPD_E_NUMERIC;
    }
    if (s & ST_FENE_BROKEN) {
        err = "FENE bond stretched beyond R0 in replica " + std::to_string(r);
        return DPD_E_NUMERIC;
    }
    if (s & ST_BOND_MISSING) {
        err = "bond partner not found in replica " + std::to_string(r);
        return DPD_E_STATE;
    }
    if (s & ST_WALL_ORDER) {
        err = "The high wall is positioned lower than the low wall (fix two_wall, replica " + std::to_string(r) + ")";
        return DPD_E_STATE;
    }
    if (s & ST_CONTACT_BOX) {
        err = "contact region out of the box (compute wall_contact, replica " + std::to_string(r) + ")";
        return DPD_E_STATE;
    }
    if (s & ST_BAD_INPUT) {
        err = "an atom id or type in the AoS input is outside the engine's system";
        return DPD_E_ARG;
    }
    return DPD_OK;
}

int Engine::time_steps(uint32_t nsteps, double* total_ms, double* pair_ms, int64_t* launches)
{
    if (zero_pending_) {
        int e = run(0);
        if (e) return e;
    }
    if (nsteps == 0) return DPD_E_ARG;
    const int nrep = (int)reps_.size();
    std::vector<cudaEvent_t> ev(2 * (size_t)nsteps + 2);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    const uint32_t target = next_step_ - 1 + nsteps;
    if (ranks_dirty_) {
        const int e = upload_ranks();
        if (e) return e;
        ranks_dirty_ = false;
    }
    // a pending list build (new cell ranks, a restart) comes first, as in a run
    k_set_target<<<(nrep + 255) / 256, 256, 0, stream_>>>(b_.rstate, b_.limit, nrep, target, 0, force_build_ ? 1 : 0,
                                                          b_.build_flag, b_.phase);
    force_build_ = false;
    enqueue_integrate_initial(stream_);
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    for (uint32_t k = 0; k < nsteps; k++) enqueue_step(stream_, ev[2 * k + 2], ev[2 * k + 3]);
    cudaError_t ce = cudaStreamEndCapture(stream_, &g);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
    cudaGraphExec_t ge;
    ce = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
    // upload the executable graph before the timed region (a first launch would otherwise
    // include the upload)
    CK(cudaGraphUpload(ge, stream_));
    CK(cudaStreamSynchronize(stream_));
    CK(cudaEventRecord(ev[0], stream_));
    CK(cudaGraphLaunch(ge, stream_));
    CK(cudaEventRecord(ev[1], stream_));
    CK(cudaStreamSynchronize(stream_));
    next_step_ = target + 1;
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    double pair = 0;
    for (uint32_t k = 0; k < nsteps; k++) {
        float p = 0;
        CK(cudaEventElapsedTime(&p, ev[2 * k + 2], ev[2 * k + 3]));
        pair += p;
    }
    cudaGraphExecDestroy(ge);
    for (auto& e : ev) cudaEventDestroy(e);
    if (total_ms) *total_ms = ms;
    if (pair_ms) *pair_ms = pair;
    if (launches) *launches = (int64_t)nsteps * ((any_dpd_ ? 1 : 0) + (any_mdpd_ ? 1 : 0));
    return sync_and_check();
}

__global__ void k_freeze(uint32_t* limit, int r)
{
    if (threadIdx.x == 0) limit[r] = 0u;
}

int Engine::freeze_async(int rep)
{
    if (rep < 0 || rep >= (int)reps_.size()) return DPD_E_ARG;
    k_freeze<<<1, 32, 0, stream_>>>(b_.limit, rep);
    CK(cudaGetLastError());
    return DPD_OK;
}

int Engine::set_limits(const std::vector<uint32_t>& limit)
{
    if (limit.size() != reps_.size()) return DPD_E_ARG;
    CK(cudaMemcpyAsync(b_.limit, limit.data(), sizeof(uint32_t) * limit.size(), cudaMemcpyHostToDevice, stream_));
    CK(cudaStreamSynchronize(stream_));
    return DPD_OK;
}

// Device bytes that init() allocates for these replicas, from the same sizes as
// layout() and alloc_and_upload() (the server admits jobs against its budget with it).
int64_t Engine::estimate_bytes(const std::vector<const Replica*>& reps)
{
    int64_t P = 0, C = 0, ntag = 0, ncoeff = 0, nmass = 0, nbond = 0, nrdf = 0, nang = 0;
    int64_t nmax = 16, maxb = 0;
    const int64_t nrep = (int64_t)reps.size();
    for (const Replica* R : reps) nang += ((int64_t)(R->sys.angles.size() / 4) + 31) / 32 * 32;
    for (const Replica* R : reps) {
        const double cut = R->in.global_cut + R->in.skin;
        int64_t ncell = 1;
        for (int k = 0; k < 3; k++)
            ncell *= std::max(1, (int)std::floor((R->sys.hi[k] - R->sys.lo[k]) / cut));
        const int64_t n = R->sys.n_atoms;
        P += ((n + 31) / 32) * 32;
        C += ncell + 1;
        ntag += n;
        const int64_t nt = R->sys.n_atomtypes;
        ncoeff += nt * nt * 3;
        nmass += nt;
        nbond += std::max(R->sys.n_bondtypes, 1);
        nrdf += R->ff.rdfs.empty() ? 0 : R->ff.rdfs[0].nbins;
        const double sphere = 4.0 / 3.0 * M_PI * std::pow(cut, 3.0);
        const int64_t nm = (int64_t)(R->in.max_rho * sphere) + 1;
        nmax = std::max(nmax, ((nm + 15) / 16) * 16);
        if (R->sys.n_bonds > 0) {
            std::vector<int> deg(n, 0);
            for (int b = 0; b < R->sys.n_bonds; b++) {
                deg[R->sys.bonds[3 * b + 1] - 1]++;
                deg[R->sys.bonds[3 * b + 2] - 1]++;
            }
            for (int d : deg) maxb = std::max<int64_t>(maxb, d);
        }
    }
    const int64_t mb = std::max<int64_t>(maxb, 1);
    int64_t bytes = nrep * ((int64_t)sizeof(RepDesc) + (int64_t)sizeof(RepState) + 4);
    bytes += (P / 32) * 4 + ncoeff * 16 + nmass * 8 + nbond * 16 + nrdf * 8;
    bytes += P * (2 * (16 + 16 + 16) + 2 * mb * 8 + 16 + 16 + 4 + 4 + 8 + 4 * nmax + mb * 8);
    bytes += C * (4 * 5) + ntag * 4 + ((C + 4095) / 4096 + 1) * 4;
    bytes += nrep * ((int64_t)DPD_ACC_SLOTS * DPD_NACC * 8 + (int64_t)DPD_RING_ROWS * DPD_THERMO_FIELDS * 8);
    bytes += nang * 16 + (nang / 32) * 4 + nrep * 32 * 8;  // angle table, warp replicas, coefficients
    bytes += nrep * (int64_t)(sizeof(FixDesc) + sizeof(FixOut));  // group fixes (upper bound)
    for (const Replica* R : reps)  // group computes: descriptors, x0, rows
        if (!R->ff.gcs.empty())
            bytes += (int64_t)sizeof(GCDesc) * DPD_MAX_GC + 16 * (int64_t)R->sys.n_atoms +
                     (int64_t)R->ff.gcs.size() * (DPD_RING_ROWS * 32 + 4);
    for (const Replica* R : reps)
        if (R->ff.spring.on && R->ff.spring.file_freq) {
            bytes += nrep * (int64_t)DPD_RING_ROWS * 6 * 8;
            break;
        }
    return bytes + 64 * 1024 + nrep * 1024;  // arrays of size 0 still take one element
}

int64_t Engine::steps_done(int r) const
{
    (void)r;
    return zero_pending_ && next_step_ == 0 ? 0 : (int64_t)next_step_ - 1;
}

int64_t Engine::n_builds()
{
    std::vector<RepState> st;
    if (read_rstate(st)) return -1;
    return st.empty() ? 0 : st[0].nbuild;
}

int64_t Engine::total_atoms() const
{
    int64_t n = 0;
    for (auto& R : reps_) n += R.sys.n_atoms;
    return n;
}

// ---------------------------------------------------------------------------------
int Engine::get_thermo(int rep, dpd_thermo* rows, int max_rows, int* n_rows)
{
    if (rep < 0 || rep >= (int)reps_.size()) return DPD_E_ARG;
    std::vector<RepState> st;
    int e = read_rstate(st);
    if (e) return e;
    const int nlog = st[rep].nlog;
    const int avail = std::min(nlog, DPD_RING_ROWS);
    const int n = std::min(avail, max_rows);
    std::vector<double> ring((size_t)DPD_RING_ROWS * DPD_THERMO_FIELDS);
    CK(cudaMemcpyAsync(ring.data(), b_.ring + (size_t)rep * DPD_RING_ROWS * DPD_THERMO_FIELDS,
                       sizeof(double) * ring.size(), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    for (int k = 0; k < n; k++) {
        const int idx = (nlog - n + k) % DPD_RING_ROWS;
        const double* row = ring.data() + (size_t)idx * DPD_THERMO_FIELDS;
        dpd_thermo& t = rows[k];
        t.step = (int64_t)row[0];
        t.temp = row[1];
        t.pair_pe = row[2];
        t.bond_pe = row[3];
        t.pressure = row[4];
        for (int c = 0; c < 6; c++) t.p[c] = row[5 + c];
        t.ke = row[11];
        for (int c = 0; c < 3; c++) t.momentum[c] = row[12 + c];
        t.angle_pe = row[16];
    }
    if (n_rows) *n_rows = n;
    return DPD_OK;
}

int Engine::compute_rows(int rep, const std::string& id, double* rows, int max_rows, int* n_cols, int* n_rows)
{
    if (rep < 0 || rep >= (int)reps_.size() || max_rows < 0) return DPD_E_ARG;
    const Replica& R = reps_[rep];
    int k = -1;
    for (size_t q = 0; q < R.ff.gcs.size(); q++)
        if (R.ff.gcs[q].id == id) k = (int)q;
    if (k < 0) {
        err = "no temp/rho/msd/tf compute with ID " + id;
        return DPD_E_ARG;
    }
    const int ring = gc_ring_base_[rep] + k;
    int count = 0;
    CK(cudaMemcpyAsync(&count, b_.gc_count + ring, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    std::vector<double> buf((size_t)DPD_RING_ROWS * 4);
    CK(cudaMemcpyAsync(buf.data(), b_.gc_ring + (size_t)ring * DPD_RING_ROWS * 4, sizeof(double) * buf.size(),
                       cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    const int nc = R.ff.gcs[k].kind == GC_TF ? 4 : 2;
    const int n = std::min(std::min(count, DPD_RING_ROWS), max_rows);
    for (int q = 0; q < n; q++) {
        const double* src = buf.data() + 4 * (size_t)((count - n + q) % DPD_RING_ROWS);
        for (int c = 0; c < nc; c++) rows[(size_t)q * nc + c] = src[c];
    }
    if (n_cols) *n_cols = nc;
    if (n_rows) *n_rows = n;
    return DPD_OK;
}

int Engine::spring_records(int rep, double* rows, int max_rows, int* n_rows)
{
    if (rep < 0 || rep >= (int)reps_.size() || max_rows < 0) return DPD_E_ARG;
    if (n_rows) *n_rows = 0;
    if (!b_.spring_ring) return DPD_OK;
    FixOut fo;
    CK(cudaMemcpyAsync(&fo, b_.fixo + rep, sizeof(FixOut), cudaMemcpyDeviceToHost, stream_));
    std::vector<double> ring((size_t)DPD_RING_ROWS * 6);
    CK(cudaMemcpyAsync(ring.data(), b_.spring_ring + (size_t)rep * DPD_RING_ROWS * 6, sizeof(double) * ring.size(),
                       cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    const int n = std::min(std::min(fo.nrec, DPD_RING_ROWS), max_rows);
    for (int k = 0; k < n; k++) {
        const int idx = (fo.nrec - n + k) % DPD_RING_ROWS;
        memcpy(rows + 6 * (size_t)k, ring.data() + 6 * (size_t)idx, 6 * sizeof(double));
    }
    if (n_rows) *n_rows = n;
    return DPD_OK;
}

int Engine::cur_parity()
{
    int par = 0;
    if (cudaStreamSynchronize(stream_) != cudaSuccess) return -1;
    if (cudaMemcpy(&par, b_.parity, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return par & 1;
}

int Engine::get_state(int rep, double* x, double* v, int* image, double* f)
{
    if (rep < 0 || rep >= (int)reps_.size()) return DPD_E_ARG;
    const RepDesc& d = reps_[rep].desc;
    const Replica& R = reps_[rep];
    const int ns = d.p_cap_end - d.p_begin;
    int st = staging();
    if (st) return st;
    float4* pos = h_pos_;
    float4* vel = h_vel_;
    float4* frc = h_frc_;
    int4* img = h_img_;
    const int par = cur_parity();
    if (par < 0) return cuda_fail(cudaGetLastError(), "cudaMemcpy(parity)");
    CK(cudaMemcpyAsync(vel, b_.vel[par] + d.p_begin, sizeof(float4) * ns, cudaMemcpyDeviceToHost, stream_));
    if (x || image) {
        CK(cudaMemcpyAsync(pos, b_.pos[par] + d.p_begin, sizeof(float4) * ns, cudaMemcpyDeviceToHost, stream_));
        CK(cudaMemcpyAsync(img, b_.img + d.tag_base, sizeof(int4) * d.n_real, cudaMemcpyDeviceToHost, stream_));
    }
    if (f) CK(cudaMemcpyAsync(frc, b_.force4 + d.p_begin, sizeof(float4) * ns, cudaMemcpyDeviceToHost, stream_));
    // a spring's share of the force (post_force adds it to the force array the reference
    // dumps, src/fix/fix_spring.cu:350-370); the engine adds it inside the half kicks
    FixOut fo{};
    const bool spring = f && b_.fixo && R.ff.spring.on && R.ff.spring.mask;
    if (spring) CK(cudaMemcpyAsync(&fo, b_.fixo + rep, sizeof(FixOut), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    if (!slots_to_tags(rep, pos, vel, img, frc, spring ? fo.spring_a : nullptr, x, v, image, f)) {
        err = "corrupt tag in device state";
        return DPD_E_STATE;
    }
    return DPD_OK;
}

bool Engine::slots_to_tags(int rep, const float4* pos, const float4* vel, const int4* img, const float4* frc,
                           const float* spring_a, double* x, double* v, int* image, double* f) const
{
    const Replica& R = reps_[rep];
    const RepDesc& d = R.desc;
    std::atomic<int> bad{0};
    parallel_for(d.n_real, [&](int64_t k0, int64_t k1) {
    for (int64_t k = k0; k < k1; k++) {
        int tw;
        memcpy(&tw, &vel[k].w, 4);
        const int tag = (int)((uint32_t)tw >> DPD_TYPE_BITS);
        if (tag < 1 || tag > d.n_real) {
            bad = 1;
            continue;
        }
        const int t0 = tw & ((1 << DPD_TYPE_BITS) - 1);
        const size_t o = 3 * (size_t)(tag - 1);
        int code;
        memcpy(&code, &pos[k].w, 4);
        const int c[3] = {code & DPD_MAX_NC, (code >> DPD_CELL_BITS) & DPD_MAX_NC, (code >> (2 * DPD_CELL_BITS)) & DPD_MAX_NC};
        for (int q = 0; q < 3; q++) {
            // exact position of the FP32 state; offsets may have drifted past the cell
            // (and the box) since the last build, so wrap into [lo, lo + L)
            const float off = q == 0 ? pos[k].x : (q == 1 ? pos[k].y : pos[k].z);
            double xa = (double)c[q] * (double)d.w[q] + (double)off;
            const double L = R.box_len[q];
            const double wrap = std::floor(xa / L);
            xa -= wrap * L;
            if (xa >= L) xa -= L;
            if (x) x[o + q] = d.lo[q] + xa;
            if (v) v[o + q] = q == 0 ? vel[k].x : (q == 1 ? vel[k].y : vel[k].z);
            if (f) {
                f[o + q] = q == 0 ? frc[k].x : (q == 1 ? frc[k].y : frc[k].z);
                if (spring_a && ((R.ff.spring.mask >> t0) & 1u)) f[o + q] += (double)spring_a[q] * R.sys.masses[t0];
            }
            const int4& im = img[tag - 1];
            if (image) image[o + q] = (q == 0 ? im.x : (q == 1 ? im.y : im.z)) + (int)wrap;
        }
    }
    });
    return !bad;
}

int Engine::set_state(int rep, const double* x, const double* v)
{
    if (rep < 0 || rep >= (int)reps_.size()) return DPD_E_ARG;
    Replica& R = reps_[rep];
    const size_t n3 = 3 * (size_t)R.sys.n_atoms;
    int e = DPD_OK;
    if (!x || !v) {
        std::vector<double> xv(n3), vv(n3);
        e = get_state(rep, xv.data(), vv.data(), nullptr, nullptr);
        if (e) return e;
        R.sys.x = xv;
        R.sys.v = vv;
    }
    // host copies of a few hundred MB: one thread's memcpy would take tens of ms
    auto pcopy = [n3](double* dst, const double* src) {
        parallel_for((int64_t)n3, [&](int64_t i0, int64_t i1) { memcpy(dst + i0, src + i0, sizeof(double) * (i1 - i0)); });
    };
    if (x) pcopy(R.sys.x.data(), x);
    if (v) pcopy(R.sys.v.data(), v);
    // full re-upload of every replica's particles (the host copies of the others are
    // refreshed first); the next run starts with a zero step and a list build
    for (int r = 0; r < (int)reps_.size(); r++) {
        if (r == rep) continue;
        Replica& Q = reps_[r];
        e = get_state(r, Q.sys.x.data(), Q.sys.v.data(), nullptr, nullptr);
        if (e) return e;
    }
    e = upload_particles();
    if (e) return e;
    zero_pending_ = true;
    return sync_and_check();
}

int Engine::get_density(int rep, double* rho)
{
    if (rep < 0 || rep >= (int)reps_.size()) return DPD_E_ARG;
    const RepDesc& d = reps_[rep].desc;
    const int ns = d.p_cap_end - d.p_begin;
    std::vector<float> r(ns);
    std::vector<float4> vel(ns);
    const int par = cur_parity();
    if (par < 0) return cuda_fail(cudaGetLastError(), "cudaMemcpy(parity)");
    CK(cudaMemcpyAsync(r.data(), b_.rho + d.p_begin, sizeof(float) * ns, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(vel.data(), b_.vel[par] + d.p_begin, sizeof(float4) * ns, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    for (int k = 0; k < d.n_real; k++) {
        int tw;
        memcpy(&tw, &vel[k].w, 4);
        const int tag = (int)((uint32_t)tw >> DPD_TYPE_BITS);
        if (tag >= 1 && tag <= d.n_real) rho[tag - 1] = r[k];
    }
    return DPD_OK;
}

int Engine::get_cells(int rep, int* cell, float* off, int* nc, float* w, float* cut2)
{
    if (rep < 0 || rep >= (int)reps_.size()) return DPD_E_ARG;
    const RepDesc& d = reps_[rep].desc;
    const int ns = d.p_cap_end - d.p_begin;
    std::vector<float4> pos(ns), vel(ns);
    const int par = cur_parity();
    if (par < 0) return cuda_fail(cudaGetLastError(), "cudaMemcpy(parity)");
    CK(cudaMemcpyAsync(pos.data(), b_.pos[par] + d.p_begin, sizeof(float4) * ns, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(vel.data(), b_.vel[par] + d.p_begin, sizeof(float4) * ns, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    for (int k = 0; k < d.n_real; k++) {
        int tw, code;
        memcpy(&tw, &vel[k].w, 4);
        memcpy(&code, &pos[k].w, 4);
        const int tag = (int)((uint32_t)tw >> DPD_TYPE_BITS);
        if (tag < 1 || tag > d.n_real) continue;
        const size_t o = 3 * (size_t)(tag - 1);
        if (cell) {
            cell[o] = code & DPD_MAX_NC;
            cell[o + 1] = (code >> DPD_CELL_BITS) & DPD_MAX_NC;
            cell[o + 2] = (code >> (2 * DPD_CELL_BITS)) & DPD_MAX_NC;
        }
        if (off) {
            off[o] = pos[k].x;
            off[o + 1] = pos[k].y;
            off[o + 2] = pos[k].z;
        }
    }
    for (int q = 0; q < 3; q++) {
        if (nc) nc[q] = d.nc[q];
        if (w) w[q] = d.w[q];
    }
    if (cut2) *cut2 = d.cut2;
    return DPD_OK;
}

int Engine::get_neighbors(int rep, int* pairs, int64_t cap, int64_t* n_pairs)
{
    if (rep < 0 || rep >= (int)reps_.size()) return DPD_E_ARG;
    {
        const int e = refresh_list();
        if (e) return e;
    }
    const RepDesc& d = reps_[rep].desc;
    const int ns = d.p_cap_end - d.p_begin;
    std::vector<int> cnt(ns), lst((size_t)ns * nmax_);
    std::vector<float4> vel(P_);
    const int par = cur_parity();
    if (par < 0) return cuda_fail(cudaGetLastError(), "cudaMemcpy(parity)");
    CK(cudaMemcpyAsync(cnt.data(), b_.ncount + d.p_begin, sizeof(int) * ns, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(lst.data(), b_.nlist + (size_t)d.p_begin * nmax_, sizeof(int) * lst.size(), cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(vel.data(), b_.vel[par], sizeof(float4) * P_, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    auto tag_at = [&](int s) {
        int tw;
        memcpy(&tw, &vel[s].w, 4);
        return (int)((uint32_t)tw >> DPD_TYPE_BITS);
    };
    int64_t np = 0;
    for (int k = 0; k < d.n_real; k++) {
        const int s = d.p_begin + k;
        const int c = std::min(cnt[k], nmax_);
        for (int q = 0; q < c; q++) {
            const int j = lst[((size_t)(k >> 5) * nmax_ + q) * 32 + (k & 31)] & DPD_J_MASK;
            if (j < 0 || j >= P_) continue;
            int a = tag_at(s), bb = tag_at(j);
            if (np < cap && pairs) {
                pairs[2 * np] = std::min(a, bb);
                pairs[2 * np + 1] = std::max(a, bb);
            }
            np++;
        }
    }
    if (n_pairs) *n_pairs = np;
    return DPD_OK;
}

int Engine::rdf_result(int rep, double* g, int64_t* nsamples)
{
    if (rep < 0 || rep >= (int)reps_.size()) return DPD_E_ARG;
    const Replica& R = reps_[rep];
    if (R.ff.rdfs.empty()) {
        err = "no rdf compute configured for this system";
        return DPD_E_STATE;
    }
    const ComputeRdf& c = R.ff.rdfs[0];
    std::vector<unsigned long long> h(c.nbins);
    std::vector<RepState> st;
    int e = read_rstate(st);
    if (e) return e;
    CK(cudaMemcpyAsync(h.data(), b_.rdf_hist + R.desc.rdf_off, sizeof(unsigned long long) * c.nbins, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    const int64_t ns = st[rep].rdf_samples;
    if (nsamples) *nsamples = ns;
    int64_t na = 0, nb = 0;
    for (int i = 0; i < R.sys.n_atoms; i++) {
        na += R.sys.type[i] == c.ta;
        nb += R.sys.type[i] == c.tb;
    }
    const double vol = R.desc.volume;
    const double npair = c.ta == c.tb ? (double)na * (double)(na - 1) : (double)na * (double)nb;
    const double dr = c.rmax / c.nbins;
    for (int b = 0; b < c.nbins; b++) {
        const double r0 = b * dr, r1 = (b + 1) * dr;
        const double shell = 4.0 / 3.0 * M_PI * (r1 * r1 * r1 - r0 * r0 * r0);
        const double ideal = npair * shell / vol * (double)std::max<int64_t>(ns, 1);
        g[b] = ideal > 0 ? (double)h[b] / ideal : 0.0;
    }
    return DPD_OK;
}

int Engine::compute_rdf_now(int rep, int ta, int tb, double rmax, int nbins, double* g)
{
    (void)rep; (void)ta; (void)tb; (void)rmax; (void)nbins; (void)g;
    err = "use an rdf compute (compute ID group rdf ...) to sample the RDF";
    return DPD_E_STATE;
}

int Engine::rdf_config(int rep, int ta, int tb, double rmax, int nbins, int every)
{
    (void)rep; (void)ta; (void)tb; (void)rmax; (void)nbins; (void)every;
    err = "rdf sampling is configured by the compute rdf command";
    return DPD_E_STATE;
}

int Engine::write_data(int rep, const std::string& path)
{
    if (rep < 0 || rep >= (int)reps_.size()) return DPD_E_ARG;
    Replica& R = reps_[rep];
    SystemData s = R.sys;
    int e = get_state(rep, s.x.data(), s.v.data(), nullptr, nullptr);
    if (e) return e;
    return write_data_file(path, R.in.atom_style, s, err);
}

int Engine::list_stats(int64_t* n_pairs, int64_t* n_atoms, int64_t* n_builds)
{
    {
        const int e = refresh_list();
        if (e) return e;
    }
    const RepDesc& d = reps_[0].desc;
    const int ns = d.p_cap_end - d.p_begin;
    std::vector<int> cnt(ns);
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(cnt.data(), b_.ncount + d.p_begin, sizeof(int) * ns, cudaMemcpyDeviceToHost));
    int64_t tot = 0;
    for (int k = 0; k < d.n_real; k++) tot += std::min(cnt[k], nmax_);
    if (n_pairs) *n_pairs = tot;
    if (n_atoms) *n_atoms = d.n_real;
    if (n_builds) *n_builds = this->n_builds();
    return DPD_OK;
}

int Engine::set_tuning(const dpd_tuning* t)
{
    if (!t) return DPD_E_ARG;
    if (t->pair_variant < 0 || t->pair_variant > 11 || t->cell_order < 0 || t->cell_order > 2 ||
        t->pair_block < 0 || t->build_variant < 0 || t->build_variant > 5 || t->launch_mode < 0 ||
        t->launch_mode > 3 || t->tile < 0 || t->tile > TILE_MAX_EDGE || t->tile_capacity < 0 ||
        t->tile_capacity > 4096) {
        err = "dpd_set_tuning: pair_variant must be 0..11, build_variant 0..5, cell_order 0..2, "
              "launch_mode 0..3, tile edge 0..6, tile capacity 0..4096";
        return DPD_E_ARG;
    }
    const bool reorder = t->cell_order != tune_.cell_order;
    tune_ = *t;
    if (reorder) {
        // the slots stay sorted in the old order (and the device keeps the old ranks, so
        // that the list and cell ranges stay consistent) until the next run, which uploads
        // the new ranks and starts with a list build
        for (Replica& R : reps_) rank_cells(R);
        ranks_dirty_ = true;
        force_build_ = true;
    }
    return build_graph();
}

// Pair::compute_force on the reference's AoS device buffers (see kernels_aos.cuh).  Bonds
// are left to the caller's own bond style, as the reference computes them separately.
// status of the AoS bond / nve kernels: they run on the legacy default stream, in order
// with the caller's own kernels; the status is read back after each call
int Engine::aos_check(const char* what)
{
    CK(cudaGetLastError());
    int stt = 0;
    CK(cudaMemcpyAsync(&stt, aos_status_, sizeof(int), cudaMemcpyDeviceToHost, cudaStreamLegacy));
    CK(cudaStreamSynchronize(cudaStreamLegacy));
    if (stt) {
        CK(cudaMemsetAsync(aos_status_, 0, sizeof(int), cudaStreamLegacy));
        if (stt & ST_FENE_BROKEN) {
            err = std::string(what) + ": FENE bond stretched beyond R0";
            return DPD_E_NUMERIC;
        }
        err = std::string(what) + ": an atom id, index or type outside the engine's system";
        return DPD_E_ARG;
    }
    return DPD_OK;
}

int Engine::bond_compute_aos(const float* d_pos, const int* d_bondlist, int n_bonds, float* d_force,
                             float* d_bond_pe, float* d_virial)
{
    if (reps_.size() != 1) {
        err = "the AoS bond entry point works on a single-system engine";
        return DPD_E_STATE;
    }
    const Replica& R = reps_[0];
    if (R.ff.bond_style == 0 || R.ff.bond_coeff.empty()) {
        err = "the engine's run.in has no bond_style";
        return DPD_E_STATE;
    }
    if (n_bonds < 0 || (n_bonds > 0 && (!d_pos || !d_bondlist || !d_force))) {
        err = "null device pointer or negative bond count";
        return DPD_E_ARG;
    }
    int st;
    if (!aos_status_ && (st = dalloc(&aos_status_, 1))) return st;
    CK(cudaStreamSynchronize(stream_));  // the status word was zeroed on the engine's stream
    AosBondArgs b;
    for (int k = 0; k < 3; k++) {
        b.L[k] = (float)R.sys.hi[k] - (float)R.sys.lo[k];
        b.hL[k] = 0.5f * b.L[k];
    }
    b.style = R.ff.bond_style;
    b.ntypes = (int)R.ff.bond_coeff.size();
    b.coef = b_.bondc + R.desc.bond_off;
    b.n_atoms = R.sys.n_atoms;
    b.status = aos_status_;
    if (n_bonds > 0) {
        const int g = (n_bonds + 255) / 256;
        if (d_bond_pe || d_virial)
            k_bond_aos<true><<<g, 256, 0, cudaStreamLegacy>>>(b, d_pos, d_bondlist, n_bonds, d_force, d_bond_pe, d_virial);
        else
            k_bond_aos<false><<<g, 256, 0, cudaStreamLegacy>>>(b, d_pos, d_bondlist, n_bonds, d_force, nullptr, nullptr);
    }
    return aos_check("bond force");
}

int Engine::nve_aos(int phase, const int* d_group, int n_group, const int* d_type, float* d_pos, float* d_uwpos,
                    float* d_vel, const float* d_force)
{
    if (reps_.size() != 1) {
        err = "the AoS nve entry point works on a single-system engine";
        return DPD_E_STATE;
    }
    if ((phase != 0 && phase != 1) || n_group < 0 ||
        (n_group > 0 && (!d_group || !d_type || !d_pos || !d_vel || !d_force))) {
        err = "phase must be 0 (initial) or 1 (final); null device pointer or negative count";
        return DPD_E_ARG;
    }
    const Replica& R = reps_[0];
    int st;
    if (!aos_status_ && (st = dalloc(&aos_status_, 1))) return st;
    if (!aos_mass_) {
        if ((st = dalloc(&aos_mass_, R.sys.n_atomtypes))) return st;
        std::vector<float> m(R.sys.n_atomtypes);
        for (int t = 0; t < R.sys.n_atomtypes; t++) m[t] = (float)R.sys.masses[t];
        CK(cudaMemcpyAsync(aos_mass_, m.data(), sizeof(float) * m.size(), cudaMemcpyHostToDevice, stream_));
    }
    CK(cudaStreamSynchronize(stream_));
    AosNveArgs b;
    b.dt = (float)R.in.dt;
    for (int k = 0; k < 3; k++) {
        b.lo[k] = (float)R.sys.lo[k];
        b.hi[k] = (float)R.sys.hi[k];
        b.L[k] = b.hi[k] - b.lo[k];
    }
    b.ntypes = R.sys.n_atomtypes;
    b.mass = aos_mass_;
    b.n_atoms = R.sys.n_atoms;
    b.status = aos_status_;
    if (n_group > 0) {
        const int g = (n_group + 255) / 256;
        if (phase == 0)
            k_nve_aos<0><<<g, 256, 0, cudaStreamLegacy>>>(b, d_group, n_group, d_type, d_pos, d_uwpos, d_vel, d_force);
        else
            k_nve_aos<1><<<g, 256, 0, cudaStreamLegacy>>>(b, d_group, n_group, d_type, d_pos, d_uwpos, d_vel, d_force);
    }
    return aos_check("nve");
}

int Engine::pair_compute_aos(const float* d_pos, const float* d_vel, const int* d_id, const int* d_type,
                             int n, uint32_t step, float* d_force, float* d_pe, float* d_virial)
{
    if (reps_.size() != 1) {
        err = "the AoS pair entry point works on a single-system engine";
        return DPD_E_STATE;
    }
    const RepDesc& d = reps_[0].desc;
    if (!d_pos || !d_vel || !d_id || !d_type || !d_force) {
        err = "null device pointer";
        return DPD_E_ARG;
    }
    if (n != d.n_real) {
        err = "n does not match the number of atoms of the engine's system";
        return DPD_E_ARG;
    }
    int st;
    if ((d_pe || d_virial) && !pe_slot_) {
        if ((st = dalloc(&pe_slot_, P_))) return st;
        if ((st = dalloc(&vir_slot_, 6 * (size_t)P_))) return st;
    }
    // the caller's buffers were written on the legacy default stream (the reference's own
    // kernels): this engine's stream runs after that work
    CK(cudaStreamSynchronize(cudaStreamLegacy));
    StepArgs sa = step_args(b_, P_, nmax_, maxb_, 1);
    const int gp = (P_ + 255) / 256;
    k_aos_in<<<(n + 255) / 256, 256, 0, stream_>>>(sa, d_pos, d_vel, d_id, d_type, n, step, aos_built_ ? 0 : 1);
    enqueue_build(stream_, true, tune_.build_variant == 3);
    if (any_mdpd_) k_density<<<gp, 256, 0, stream_>>>(sa);
    const bool peratom = d_pe || d_virial;
    // this entry builds the list itself: schedule 11 (no list) runs as the default 8
    const int pv = tune_.pair_variant == 11 ? 8 : tune_.pair_variant;
    if (d.style == 0) {
        if (peratom) k_pair_peratom<0><<<gp, 256, 0, stream_>>>(sa, pe_slot_, vir_slot_);
        else launch_pair<0>(pv, false, gp, stream_, sa);
    } else {
        if (peratom) k_pair_peratom<1><<<gp, 256, 0, stream_>>>(sa, pe_slot_, vir_slot_);
        else launch_pair<1>(pv, false, gp, stream_, sa);
    }
    k_aos_out<<<gp, 256, 0, stream_>>>(sa, d_force, d_pe, d_virial, pe_slot_, vir_slot_);
    k_aos_done<<<1, 1, 0, stream_>>>(b_.build_flag, b_.phase);
    CK(cudaGetLastError());
    aos_built_ = true;
    return sync_and_check();
}

// ---------------------------------------------------------------------------------
int make_replica(const std::string& run_in, const std::string& data_path, const std::string& base_dir,
                 Replica& R, std::string& err)
{
    int e = parse_run_in(run_in, R.in, err);
    if (e) return e;
    std::string path = data_path.empty() ? R.in.read_data : data_path;
    if (data_path.empty() && !base_dir.empty() && !path.empty() && path[0] != '/') path = base_dir + "/" + path;
    e = read_data_file(path, R.in.atom_style, R.sys, err);
    if (e) return e;
    return parse_force_field(R.in, R.sys, R.ff, err);
}

int make_replica_from_system(const std::string& run_in, const dpd_system* s, Replica& R, std::string& err)
{
    int e = parse_run_in(run_in, R.in, err);
    if (e) return e;
    if (!s || s->n_atoms <= 0 || s->n_atomtypes <= 0 || !s->tag || !s->type || !s->x || !s->masses) {
        err = "incomplete dpd_system";
        return DPD_E_ARG;
    }
    SystemData& d = R.sys;
    d.n_atoms = s->n_atoms;
    d.n_atomtypes = s->n_atomtypes;
    d.n_bonds = R.in.atom_style >= 1 ? s->n_bonds : 0;
    d.n_bondtypes = s->n_bondtypes;
    for (int k = 0; k < 3; k++) {
        d.lo[k] = s->lo[k];
        d.hi[k] = s->hi[k];
        if (!(d.hi[k] > d.lo[k])) {
            err = "Invalid box dimensions.";
            return DPD_E_ARG;
        }
    }
    d.masses.assign(s->masses, s->masses + s->n_atomtypes);
    for (double m : d.masses)
        if (!(m > 0)) {
            err = "All the masses are not set.";
            return DPD_E_ARG;
        }
    const int n = s->n_atoms;
    d.type.assign(n, 0);
    d.mol.assign(n, 0);
    d.x.assign(3 * (size_t)n, 0.0);
    d.v.assign(3 * (size_t)n, 0.0);
    std::vector<char> seen(n, 0);
    for (int i = 0; i < n; i++) {
        const int t = s->tag[i];
        if (t < 1 || t > n || seen[t - 1]) {
            err = "tags must be a permutation of 1..n_atoms";
            return DPD_E_ARG;
        }
        seen[t - 1] = 1;
        if (s->type[i] < 1 || s->type[i] > s->n_atomtypes) {
            err = "atom type out of range";
            return DPD_E_ARG;
        }
        d.type[t - 1] = s->type[i];
        if (s->mol) d.mol[t - 1] = s->mol[i];
        for (int k = 0; k < 3; k++) {
            double c = s->x[3 * (size_t)i + k];
            const double L = d.hi[k] - d.lo[k];
            if (!std::isfinite(c)) {
                err = "non-finite position";
                return DPD_E_ARG;
            }
            if (c >= d.hi[k] || c < d.lo[k]) c -= L * std::floor((c - d.lo[k]) / L);
            if (c >= d.hi[k]) c = d.lo[k];
            d.x[3 * (size_t)(t - 1) + k] = c;
            d.v[3 * (size_t)(t - 1) + k] = s->v ? s->v[3 * (size_t)i + k] : 0.0;
        }
    }
    d.has_velocities = s->v != nullptr;
    if (d.n_bonds > 0) {
        if (!s->bonds) {
            err = "bonds missing";
            return DPD_E_ARG;
        }
        d.bonds.assign(s->bonds, s->bonds + 3 * (size_t)d.n_bonds);
        for (int b = 0; b < d.n_bonds; b++) {
            const int ty = d.bonds[3 * b], a = d.bonds[3 * b + 1], c = d.bonds[3 * b + 2];
            if (ty < 1 || ty > std::max(1, d.n_bondtypes) || a < 1 || a > n || c < 1 || c > n || a == c) {
                err = "invalid bond " + std::to_string(b + 1);
                return DPD_E_ARG;
            }
        }
    }
    if (R.in.atom_style == 2) {
        d.n_angles = s->n_angles;
        d.n_angletypes = s->n_angletypes;
        if (d.n_angles > 0) {
            if (!s->angles) {
                err = "angles missing";
                return DPD_E_ARG;
            }
            d.angles.assign(s->angles, s->angles + 4 * (size_t)d.n_angles);
            for (int q = 0; q < d.n_angles; q++) {
                const int* a = &d.angles[4 * q];
                if (a[0] < 1 || a[0] > std::max(1, d.n_angletypes) || a[1] < 1 || a[1] > n || a[2] < 1 ||
                    a[2] > n || a[3] < 1 || a[3] > n || a[1] == a[2] || a[2] == a[3] || a[1] == a[3]) {
                    err = "invalid angle " + std::to_string(q + 1);
                    return DPD_E_ARG;
                }
            }
        }
    }
    return parse_force_field(R.in, R.sys, R.ff, err);
}

}  // namespace dpd
