// restart.cu -- exact checkpoint and resume of an engine.  The reference restarts from a
// write_data file (src/system/read_data.cu:473-637): FP32 positions and velocities only,
// no image flags, and the run starts again at step 0, so the counter-based random force
// (seeded with seed + step, src/force/pair_dpd.cu:213) replays the first run's stream.
// A restart file here holds the engine's own FP32 state (cell codes and offsets,
// velocities, image counters, the forces of the last evaluated step) with the step
// counters and the fix results, so a resumed run continues the same step sequence: the
// first half kick uses the stored forces and the random force uses the next step.
//
// Layout (host byte order): magic "DPDB2RS1", u32 version, i32 replicas, u32 next step,
// i32 zero step pending; per replica: i32 atoms, i32 nc[3], f32 w[3], RepState, FixOut,
// then in tag order float4 pos[n], float4 vel[n], int4 img[n], float4 force[n].
#include <cstdio>
#include <cstring>
#include <vector>

#include "engine.h"

namespace dpd {

static const char kMagic[8] = {'D', 'P', 'D', 'B', '2', 'R', 'S', '1'};

// CUDA call check that closes the open file first
#define CK(call)                                               \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) {                               \
            if (fp) fclose(fp);                                \
            return cuda_fail(e_, #call);                       \
        }                                                      \
    } while (0)

int Engine::write_restart(const std::string& path)
{
    int st = sync_and_check();
    if (st) return st;
    std::vector<RepState> rs;
    if ((st = read_rstate(rs))) return st;
    const int par = cur_parity();
    if (par < 0) return cuda_fail(cudaGetLastError(), "cudaMemcpy(parity)");
    if ((st = staging())) return st;
    FILE* fp = fopen(path.c_str(), "wb");
    if (!fp) {
        err = "cannot open restart file " + path;
        return DPD_E_IO;
    }
    bool ok = true;
    auto put = [&](const void* p, size_t n) { ok = ok && fwrite(p, 1, n, fp) == n; };
    const uint32_t version = 1, next = next_step_;
    const int32_t nrep = (int32_t)reps_.size(), zero = zero_pending_ ? 1 : 0;
    put(kMagic, 8);
    put(&version, 4);
    put(&nrep, 4);
    put(&next, 4);
    put(&zero, 4);
    for (int r = 0; r < nrep && ok; r++) {
        const RepDesc& d = reps_[r].desc;
        const int n = d.n_real;
        FixOut fo{};
        if (b_.fixo) CK(cudaMemcpy(&fo, b_.fixo + r, sizeof(FixOut), cudaMemcpyDeviceToHost));
        CK(cudaMemcpyAsync(h_pos_, b_.pos[par] + d.p_begin, sizeof(float4) * n, cudaMemcpyDeviceToHost, stream_));
        CK(cudaMemcpyAsync(h_vel_, b_.vel[par] + d.p_begin, sizeof(float4) * n, cudaMemcpyDeviceToHost, stream_));
        CK(cudaMemcpyAsync(h_img_, b_.img + d.tag_base, sizeof(int4) * n, cudaMemcpyDeviceToHost, stream_));
        CK(cudaMemcpyAsync(h_frc_, b_.force4 + d.p_begin, sizeof(float4) * n, cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        // slots to tag order
        std::vector<float4> pos(n), vel(n), frc(n);
        std::vector<int4> img(n);
        for (int k = 0; k < n; k++) {
            int tw;
            memcpy(&tw, &h_vel_[k].w, 4);
            const int tag = (int)((uint32_t)tw >> DPD_TYPE_BITS);
            if (tag < 1 || tag > n) {
                fclose(fp);
                err = "corrupt tag in device state";
                return DPD_E_STATE;
            }
            pos[tag - 1] = h_pos_[k];
            vel[tag - 1] = h_vel_[k];
            img[k] = h_img_[k];  // already in tag order
            frc[tag - 1] = h_frc_[k];
        }
        const int32_t na = n;
        put(&na, 4);
        put(d.nc, sizeof(d.nc));
        put(d.w, sizeof(d.w));
        put(&rs[r], sizeof(RepState));
        put(&fo, sizeof(FixOut));
        put(pos.data(), sizeof(float4) * n);
        put(vel.data(), sizeof(float4) * n);
        put(img.data(), sizeof(int4) * n);
        put(frc.data(), sizeof(float4) * n);
    }
    if (fclose(fp) != 0) ok = false;
    fp = nullptr;
    if (!ok) {
        err = "cannot write restart file " + path;
        return DPD_E_IO;
    }
    return DPD_OK;
}

int Engine::read_restart(const std::string& path)
{
    int st = sync_and_check();
    if (st) return st;
    if ((st = staging())) return st;
    FILE* fp = fopen(path.c_str(), "rb");
    if (!fp) {
        err = "cannot open restart file " + path;
        return DPD_E_IO;
    }
    bool ok = true;
    auto get = [&](void* p, size_t n) { ok = ok && fread(p, 1, n, fp) == n; };
    char magic[8];
    uint32_t version = 0, next = 0;
    int32_t nrep = 0, zero = 0;
    get(magic, 8);
    get(&version, 4);
    get(&nrep, 4);
    get(&next, 4);
    get(&zero, 4);
    if (!ok || memcmp(magic, kMagic, 8) != 0 || version != 1) {
        fclose(fp);
        err = "not a restart file of this engine: " + path;
        return DPD_E_IO;
    }
    if (nrep != (int32_t)reps_.size()) {
        fclose(fp);
        err = "restart file holds " + std::to_string(nrep) + " replicas, the engine " + std::to_string(reps_.size());
        return DPD_E_ARG;
    }
    std::vector<RepState> rs(nrep);
    std::vector<FixOut> fos(nrep);
    std::vector<float4> frc_all(P_, make_float4(0, 0, 0, 0));
    for (int s = 0; s < P_; s++) {
        h_pos_[s] = make_float4(0, 0, 0, 0);
        h_vel_[s] = make_float4(0, 0, 0, 0);
        h_img_[s] = make_int4(0, 0, 0, 0);
    }
    for (int r = 0; r < nrep; r++) {
        const Replica& R = reps_[r];
        const RepDesc& d = R.desc;
        int32_t na = 0, nc[3];
        float w[3];
        get(&na, 4);
        get(nc, sizeof(nc));
        get(w, sizeof(w));
        if (!ok || na != d.n_real || memcmp(nc, d.nc, sizeof(nc)) != 0 || memcmp(w, d.w, sizeof(w)) != 0) {
            fclose(fp);
            err = "restart file does not match replica " + std::to_string(r) +
                  " (atom count or cell grid differ: same run.in and system required)";
            return DPD_E_ARG;
        }
        get(&rs[r], sizeof(RepState));
        get(&fos[r], sizeof(FixOut));
        get(h_pos_ + d.p_begin, sizeof(float4) * na);
        get(h_vel_ + d.p_begin, sizeof(float4) * na);
        get(h_img_ + d.p_begin, sizeof(int4) * na);
        get(frc_all.data() + d.p_begin, sizeof(float4) * na);
        if (!ok) break;
        for (int t = 0; t < na && ok; t++) {
            int tw;
            memcpy(&tw, &h_vel_[d.p_begin + t].w, 4);
            if ((int)((uint32_t)tw >> DPD_TYPE_BITS) != t + 1 || (tw & ((1 << DPD_TYPE_BITS) - 1)) != R.sys.type[t] - 1)
                ok = false;
        }
        if (!ok) {
            fclose(fp);
            err = "restart file does not match replica " + std::to_string(r) + " (tags or types differ)";
            return DPD_E_ARG;
        }
    }
    fclose(fp);
    fp = nullptr;
    if (!ok) {
        err = "truncated restart file " + path;
        return DPD_E_IO;
    }
    // the state goes into buffer 0 in tag order, as after upload_particles
    const size_t nb = (size_t)std::max(maxb_, 1) * P_;
    CK(cudaMemcpyAsync(b_.pos[0], h_pos_, sizeof(float4) * P_, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(b_.vel[0], h_vel_, sizeof(float4) * P_, cudaMemcpyHostToDevice, stream_));
    for (const auto& R : reps_)
        CK(cudaMemcpyAsync(b_.img + R.desc.tag_base, h_img_ + R.desc.p_begin, sizeof(int4) * R.desc.n_real,
                           cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(b_.force4, frc_all.data(), sizeof(float4) * P_, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(b_.bonds[0], bonds_tag_, sizeof(int2) * nb, cudaMemcpyDeviceToDevice, stream_));
    CK(cudaMemsetAsync(b_.parity, 0, sizeof(int), stream_));
    std::vector<int> t2i;
    for (auto& R : reps_)
        for (int t = 0; t < R.sys.n_atoms; t++) t2i.push_back(R.desc.p_begin + t);
    CK(cudaMemcpyAsync(b_.tag2idx, t2i.data(), sizeof(int) * t2i.size(), cudaMemcpyHostToDevice, stream_));
    int64_t nbins = 0;
    for (int r = 0; r < nrep; r++) {
        rs[r].nlog = 0;  // the thermo ring, the spring records and the RDF start empty
        rs[r].status = 0;
        rs[r].rdf_samples = 0;
        fos[r].nrec = 0;
        if (!reps_[r].ff.rdfs.empty()) nbins += reps_[r].ff.rdfs[0].nbins;
    }
    if (nbins > 0) CK(cudaMemsetAsync(b_.rdf_hist, 0, sizeof(unsigned long long) * nbins, stream_));
    int ngc = 0;
    for (auto& R : reps_) ngc += (int)R.ff.gcs.size();
    if (ngc > 0) CK(cudaMemsetAsync(b_.gc_count, 0, sizeof(int) * ngc, stream_));
    CK(cudaMemcpyAsync(b_.rstate, rs.data(), sizeof(RepState) * nrep, cudaMemcpyHostToDevice, stream_));
    if (b_.fixo) CK(cudaMemcpyAsync(b_.fixo, fos.data(), sizeof(FixOut) * nrep, cudaMemcpyHostToDevice, stream_));
    CK(cudaStreamSynchronize(stream_));
    next_step_ = next;
    zero_pending_ = zero != 0;
    force_build_ = true;  // slots are in tag order: the next step builds the list
    aos_built_ = false;
    return DPD_OK;
}

}  // namespace dpd
