// dump.cu -- trajectory frames of replica 0 in the reference's all.trj format
// (src/system/dump.cu:23-201), and the group frames of a dump compute
// (src/compute/compute_dump.cu): LAMMPS-style frames with id type x y z [fx fy fz]
// [vx vy vz], positions wrapped or unwrapped, nine decimals.  Frames are taken at the
// reference's dump steps (step 0 when start is 0, from src/main/utils.cuh:198-202; then
// step >= start with (step - start) % every == 0, :293-297).  Unlike the reference,
// velocities are written whenever vel_yes is given (its dump copies them from the device
// only when force_yes is also set, src/system/dump.cu:67-73).
#include <algorithm>
#include <cstring>
#include <vector>

#include "dump.h"
#include "engine.h"

namespace dpd {

// Copy replica 0's current slots (the parity buffer of this step), its image counters
// (kept by tag, copied in tag order) and the fix results into a snapshot slot.  One
// thread per particle slot.
__global__ void k_snapshot(const int* parity, const float4* pos0, const float4* pos1, const float4* vel0,
                           const float4* vel1, const int4* img, int nimg, const float4* force4,
                           const FixOut* fixo, int p0, int ns, float4* opos, float4* ovel, int4* oimg,
                           float4* ofrc, FixOut* ofo)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0 && fixo) *ofo = fixo[0];
    if (s >= ns) return;
    const int par = *parity & 1;
    opos[s] = (par ? pos1 : pos0)[p0 + s];
    ovel[s] = (par ? vel1 : vel0)[p0 + s];
    if (s < nimg) oimg[s] = img[s];  // in tag order
    ofrc[s] = force4[p0 + s];
}

bool Engine::dump_due(const DumpWriter* w, uint32_t step)
{
    if (step == 0) return w->start == 0;
    return step >= w->start && (step - w->start) % w->every == 0;
}

uint32_t Engine::next_dump(const DumpWriter* w, uint32_t s)
{
    if (s == 0 && w->start == 0) return 0;
    const uint64_t start = w->start, every = w->every;
    const uint64_t d0 = std::max<uint64_t>(std::max<uint64_t>(s, 1), start);
    const uint64_t d = start + (d0 - start + every - 1) / every * every;
    return d > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)d;
}

// Format one frame (tag order) and append it to the file.  Lines are formatted in
// parallel chunks and written in order.  A compute dump (w.group != 0) lists the group's
// atoms with wrapped positions (src/compute/compute_dump.cu:60-130).
static bool write_frame(FILE* fp, const Replica& R, const DumpWriter& w, uint32_t step, const double* x,
                        const int* img, const double* v, const double* f)
{
    const int n = R.sys.n_atoms;
    auto member = [&](int i) { return !w.group || ((w.group >> (R.sys.type[i] - 1)) & 1u); };
    int nout = n;
    if (w.group) {
        nout = 0;
        for (int i = 0; i < n; i++) nout += member(i);
    }
    fprintf(fp, "ITEM: TIMESTEP\n%u\n", step);
    fprintf(fp, "ITEM: NUMBER OF ATOMS\n%d\n", nout);
    fprintf(fp, "ITEM: BOX BOUNDS pp pp pp\n");
    for (int k = 0; k < 3; k++) fprintf(fp, "%.9f %.9f\n", R.sys.lo[k], R.sys.hi[k]);
    if (w.group)
        fprintf(fp, "ITEM: ATOMS id %stype x y z\n", w.mol ? "mol " : "");
    else
        fprintf(fp, "ITEM: ATOMS id type x y z%s%s\n", w.force ? " fx fy fz" : "", w.vel ? " vx vy vz" : "");
    const int nchunk = n < 65536 ? 1 : 64;
    std::vector<std::string> out(nchunk);
    parallel_for(nchunk, [&](int64_t c0, int64_t c1) {
        for (int64_t c = c0; c < c1; c++) {
            const int i0 = (int)((int64_t)n * c / nchunk), i1 = (int)((int64_t)n * (c + 1) / nchunk);
            std::string& s = out[c];
            s.reserve((size_t)(i1 - i0) * 128);
            char buf[320];
            for (int i = i0; i < i1; i++) {
                if (!member(i)) continue;
                double p[3];
                for (int q = 0; q < 3; q++)
                    p[q] = w.unwrapped ? x[3 * (size_t)i + q] + (double)img[3 * (size_t)i + q] * R.box_len[q]
                                       : x[3 * (size_t)i + q];
                int len;
                if (w.group && w.mol)
                    len = snprintf(buf, sizeof(buf), "%d %d %d %.9f %.9f %.9f", i + 1,
                                   R.sys.mol.empty() ? 0 : R.sys.mol[i], R.sys.type[i], p[0], p[1], p[2]);
                else
                    len = snprintf(buf, sizeof(buf), "%d %d %.9f %.9f %.9f", i + 1, R.sys.type[i], p[0], p[1], p[2]);
                if (w.force)
                    len += snprintf(buf + len, sizeof(buf) - len, " %.9f %.9f %.9f", f[3 * (size_t)i],
                                    f[3 * (size_t)i + 1], f[3 * (size_t)i + 2]);
                if (w.vel)
                    len += snprintf(buf + len, sizeof(buf) - len, " %.9f %.9f %.9f", v[3 * (size_t)i],
                                    v[3 * (size_t)i + 1], v[3 * (size_t)i + 2]);
                buf[len++] = '\n';
                s.append(buf, (size_t)len);
            }
        }
    });
    for (auto& s : out)
        if (fwrite(s.data(), 1, s.size(), fp) != s.size()) return false;
    return fflush(fp) == 0;
}

static void free_writer(DumpWriter* w)
{
    if (w->file) fclose(w->file);
    w->file = nullptr;
    if (w->copy) cudaStreamSynchronize(w->copy);
    for (int k = 0; k < 2; k++) {
        for (void* p : {(void*)w->dpos[k], (void*)w->dvel[k], (void*)w->dfrc[k], (void*)w->dimg[k], (void*)w->dfo[k]})
            if (p) cudaFree(p);
        for (void* p : {(void*)w->hpos[k], (void*)w->hvel[k], (void*)w->hfrc[k], (void*)w->himg[k], (void*)w->hfo[k]})
            if (p) cudaFreeHost(p);
        if (w->taken[k]) cudaEventDestroy(w->taken[k]);
        if (w->copied[k]) cudaEventDestroy(w->copied[k]);
    }
    if (w->copy) cudaStreamDestroy(w->copy);
}

int Engine::dump_open(const std::string& path, uint32_t start, uint32_t every, bool unwrapped, bool force,
                      bool vel)
{
    for (auto& w : dumps_)
        if (w->id.empty()) {
            err = "a trajectory dump is already open";
            return DPD_E_STATE;
        }
    std::unique_ptr<DumpWriter> w(new DumpWriter());
    w->path = path;
    w->start = start;
    w->every = every;
    w->unwrapped = unwrapped;
    w->force = force;
    w->vel = vel;
    return dump_start(std::move(w));
}

int Engine::compute_dump_open(const std::string& id, const std::string& path)
{
    if (reps_.empty()) return DPD_E_STATE;
    const Replica& R = reps_[0];
    const ComputeDump* c = nullptr;
    for (auto& q : R.ff.cdumps)
        if (q.id == id) c = &q;
    if (!c) {
        err = "no dump compute with ID " + id;
        return DPD_E_ARG;
    }
    for (auto& w : dumps_)
        if (w->id == id) {
            err = "the dump compute " + id + " is already open";
            return DPD_E_STATE;
        }
    std::unique_ptr<DumpWriter> w(new DumpWriter());
    w->path = path.empty() ? c->file : path;
    w->id = id;
    w->start = 0;
    w->every = c->frequency;
    w->group = c->mask ? c->mask : 0xFFFFFFFFu;
    w->mol = R.in.atom_style != 0;
    return dump_start(std::move(w));
}

// open the file, allocate the two snapshot slots and start the writer thread
int Engine::dump_start(std::unique_ptr<DumpWriter> w)
{
    if (w->every == 0 || reps_.empty()) {
        err = "dump frequency must be positive";
        return DPD_E_ARG;
    }
    w->file = fopen(w->path.c_str(), "w");
    if (!w->file) {
        err = "cannot open dump file " + w->path;
        return DPD_E_IO;
    }
    const RepDesc& d = reps_[0].desc;
    w->ns = d.p_cap_end - d.p_begin;
    const size_t n = (size_t)w->ns;
    auto fail = [&](cudaError_t e, const char* what) {
        free_writer(w.get());
        return cuda_fail(e, what);
    };
    cudaError_t e;
    for (int k = 0; k < 2; k++) {
        if ((e = cudaMalloc((void**)&w->dpos[k], sizeof(float4) * n)) != cudaSuccess) return fail(e, "cudaMalloc(dump)");
        if ((e = cudaMalloc((void**)&w->dvel[k], sizeof(float4) * n)) != cudaSuccess) return fail(e, "cudaMalloc(dump)");
        if ((e = cudaMalloc((void**)&w->dfrc[k], sizeof(float4) * n)) != cudaSuccess) return fail(e, "cudaMalloc(dump)");
        if ((e = cudaMalloc((void**)&w->dimg[k], sizeof(int4) * n)) != cudaSuccess) return fail(e, "cudaMalloc(dump)");
        if ((e = cudaMalloc((void**)&w->dfo[k], sizeof(FixOut))) != cudaSuccess) return fail(e, "cudaMalloc(dump)");
        if ((e = cudaMallocHost((void**)&w->hpos[k], sizeof(float4) * n)) != cudaSuccess) return fail(e, "cudaMallocHost(dump)");
        if ((e = cudaMallocHost((void**)&w->hvel[k], sizeof(float4) * n)) != cudaSuccess) return fail(e, "cudaMallocHost(dump)");
        if ((e = cudaMallocHost((void**)&w->hfrc[k], sizeof(float4) * n)) != cudaSuccess) return fail(e, "cudaMallocHost(dump)");
        if ((e = cudaMallocHost((void**)&w->himg[k], sizeof(int4) * n)) != cudaSuccess) return fail(e, "cudaMallocHost(dump)");
        if ((e = cudaMallocHost((void**)&w->hfo[k], sizeof(FixOut))) != cudaSuccess) return fail(e, "cudaMallocHost(dump)");
        if ((e = cudaEventCreateWithFlags(&w->taken[k], cudaEventDisableTiming)) != cudaSuccess) return fail(e, "cudaEventCreate");
        if ((e = cudaEventCreateWithFlags(&w->copied[k], cudaEventDisableTiming)) != cudaSuccess) return fail(e, "cudaEventCreate");
    }
    if ((e = cudaStreamCreateWithFlags(&w->copy, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "cudaStreamCreate");
    DumpWriter* wp = w.get();
    const Replica* R = &reps_[0];
    const bool spring = b_.fixo && R->ff.spring.on && R->ff.spring.mask;
    w->thread = std::thread([this, wp, R, spring] {
        const int n = R->sys.n_atoms;
        std::vector<double> x(3 * (size_t)n), v(3 * (size_t)n), f(3 * (size_t)n);
        std::vector<int> img(3 * (size_t)n);
        for (;;) {
            int slot;
            {
                std::unique_lock<std::mutex> lk(wp->mu);
                wp->cv.wait(lk, [&] { return wp->stop || !wp->queue.empty(); });
                if (wp->queue.empty()) break;
                slot = wp->queue.front();
                wp->queue.pop_front();
            }
            std::string error;
            const cudaError_t ce = cudaEventSynchronize(wp->copied[slot]);
            if (ce != cudaSuccess) {
                error = std::string("CUDA error in dump copy: ") + cudaGetErrorString(ce);
            } else if (!slots_to_tags(0, wp->hpos[slot], wp->hvel[slot], wp->himg[slot], wp->hfrc[slot],
                                      spring ? wp->hfo[slot]->spring_a : nullptr, x.data(), v.data(), img.data(),
                                      f.data())) {
                error = "corrupt tag in a dump snapshot";
            } else if (!write_frame(wp->file, *R, *wp, wp->step[slot], x.data(), img.data(), v.data(), f.data())) {
                error = "cannot write dump file " + wp->path;
            }
            {
                std::lock_guard<std::mutex> lk(wp->mu);
                if (!error.empty() && wp->error.empty()) wp->error = error;
                wp->busy[slot] = false;
            }
            wp->cv.notify_all();
        }
    });
    dumps_.push_back(std::move(w));
    return DPD_OK;
}

int Engine::dump_frame(DumpWriter* w, uint32_t step)
{
    const int slot = w->next_slot;
    {
        std::unique_lock<std::mutex> lk(w->mu);
        w->cv.wait(lk, [&] { return !w->busy[slot]; });
        if (!w->error.empty()) {
            err = w->error;
            return DPD_E_IO;
        }
        w->busy[slot] = true;
        w->step[slot] = step;
    }
    const int p0 = reps_[0].desc.p_begin;
    k_snapshot<<<(w->ns + 255) / 256, 256, 0, stream_>>>(b_.parity, b_.pos[0], b_.pos[1], b_.vel[0], b_.vel[1],
                                                        b_.img + reps_[0].desc.tag_base, reps_[0].desc.n_real,
                                                        b_.force4, b_.fixo, p0, w->ns,
                                                        w->dpos[slot], w->dvel[slot], w->dimg[slot],
                                                        w->dfrc[slot], w->dfo[slot]);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(w->taken[slot], stream_);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(w->copy, w->taken[slot], 0);
    const size_t n = (size_t)w->ns;
    if (e == cudaSuccess) e = cudaMemcpyAsync(w->hpos[slot], w->dpos[slot], sizeof(float4) * n, cudaMemcpyDeviceToHost, w->copy);
    if (e == cudaSuccess) e = cudaMemcpyAsync(w->hvel[slot], w->dvel[slot], sizeof(float4) * n, cudaMemcpyDeviceToHost, w->copy);
    if (e == cudaSuccess) e = cudaMemcpyAsync(w->himg[slot], w->dimg[slot], sizeof(int4) * n, cudaMemcpyDeviceToHost, w->copy);
    if (e == cudaSuccess) e = cudaMemcpyAsync(w->hfrc[slot], w->dfrc[slot], sizeof(float4) * n, cudaMemcpyDeviceToHost, w->copy);
    if (e == cudaSuccess) e = cudaMemcpyAsync(w->hfo[slot], w->dfo[slot], sizeof(FixOut), cudaMemcpyDeviceToHost, w->copy);
    if (e == cudaSuccess) e = cudaEventRecord(w->copied[slot], w->copy);
    if (e != cudaSuccess) {
        std::lock_guard<std::mutex> lk(w->mu);
        w->busy[slot] = false;
        return cuda_fail(e, "dump snapshot");
    }
    {
        std::lock_guard<std::mutex> lk(w->mu);
        w->queue.push_back(slot);
        w->frames++;
    }
    w->cv.notify_all();
    w->next_slot ^= 1;
    return DPD_OK;
}

int Engine::dump_close()
{
    int rc = DPD_OK;
    for (auto& wu : dumps_) {
        DumpWriter* w = wu.get();
        {
            std::lock_guard<std::mutex> lk(w->mu);
            w->stop = true;
        }
        w->cv.notify_all();
        if (w->thread.joinable()) w->thread.join();
        if (!w->error.empty() && rc == DPD_OK) {
            err = w->error;
            rc = DPD_E_IO;
        }
        if (w->file && fclose(w->file) != 0 && rc == DPD_OK) {
            err = "cannot close dump file " + w->path;
            rc = DPD_E_IO;
        }
        w->file = nullptr;
        free_writer(w);
    }
    dumps_.clear();
    return rc;
}

}  // namespace dpd
