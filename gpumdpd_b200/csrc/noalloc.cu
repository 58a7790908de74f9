// noalloc.cu -- dpd_pair_forces_noalloc: the DPD pair force on AoS device buffers with
// no device allocation at all.
//
// Who needs it: callers that may not allocate device memory -- a force plugin inside a
// host MD code or framework that owns all device memory (a caching allocator or an arena
// set up at start-up), and fixed-latency loops, where cudaMalloc/cudaFree can synchronize
// the whole device or fail when it is nearly full.  The engine entry points allocate
// their cell lists and neighbour lists at create time; this one instead bins the
// particles into a file-scope static device array of fixed size and calls no cudaMalloc,
// cudaFree or allocating library routine.
//
// Limits: at most DPD_NOALLOC_MAX_ATOMS atoms, DPD_NOALLOC_MAX_CELLS cells of edge
// >= max rc (at least 3 per dimension) and DPD_NOALLOC_MAX_TYPES types; larger inputs are
// rejected with DPD_E_ARG before anything is launched.  The scratch array is shared by
// every call in the process (each device that loads the library holds its own copy until
// exit) and keeps the last call's contents: each call clears what must start at zero.
// Calls that overlap on the GPU (different streams or threads) race on the array.
//
// Set-up: CUDA loads a library's device code lazily, so the first call on a device
// loads this module, and with it the array (the driver reserves its device memory then,
// not when the library is loaded).  That first call also resolves the array's device
// address with the device current; the address is kept per device and CUDA context, and
// resolved again when the context changes (after a cudaDeviceReset, for instance).  Make
// that first call at start-up, before any stream capture.  Every call waits for its own
// work on `stream` before it returns (it reads back a status word).
#include <algorithm>
#include <cmath>
#include <cuda.h>
#include <mutex>

#include "../../include/dpd_b200.h"
#include "saru.cuh"

namespace {

constexpr int kMaxAtoms = DPD_NOALLOC_MAX_ATOMS;
constexpr int kMaxCells = DPD_NOALLOC_MAX_CELLS;
constexpr int kMaxTypes = DPD_NOALLOC_MAX_TYPES;
// scratch layout in ints: status word (padded), per-cell count, start (+1), fill,
// per-atom cell and sorted atom index
constexpr size_t kOffStatus = 0;
constexpr size_t kOffCount = 64;
constexpr size_t kOffStart = kOffCount + kMaxCells;
constexpr size_t kOffFill = kOffStart + kMaxCells + 64;
constexpr size_t kOffCellOf = kOffFill + kMaxCells;
constexpr size_t kOffSorted = kOffCellOf + kMaxAtoms;
constexpr size_t kWords = kOffSorted + kMaxAtoms;

}  // namespace

// The scratch: ~5 MB per device.  Host code must not take its address directly (the host
// symbol is only a stand-in); the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) int g_noalloc_scratch[kWords];

namespace {

struct NaParams {
    float lo[3], L[3], inv_w[3];
    int nc[3];
    int ncell;
    int ntypes;
    uint32_t seed;
    float rcmax2;
    float4 coeff[kMaxTypes * kMaxTypes];  // {A, gamma, sigma, rc^2} of ordered type pairs
    float inv_rc[kMaxTypes * kMaxTypes];
};

__global__ void k_na_clear(int* scratch, int ncell)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) scratch[kOffStatus] = 0;
    if (c < ncell) {
        scratch[kOffCount + c] = 0;
        scratch[kOffFill + c] = 0;
    }
}

__device__ __forceinline__ int na_cell(const NaParams& p, const float* x, int i)
{
    int c[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        int q = (int)floorf((x[3 * i + k] - p.lo[k]) * p.inv_w[k]);
        c[k] = min(max(q, 0), p.nc[k] - 1);
    }
    return (c[0] * p.nc[1] + c[1]) * p.nc[2] + c[2];
}

// a position more than a thousandth of a cell outside [lo, hi) (or not finite): the
// cell stencil would miss some of its pairs
__device__ __forceinline__ bool na_outside(const NaParams& p, const float* x, int i)
{
    bool out = false;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float q = (x[3 * i + k] - p.lo[k]) * p.inv_w[k];
        out = out || !(q >= -1.0e-3f && q < (float)p.nc[k] + 1.0e-3f);
    }
    return out;
}

__global__ void k_na_count(NaParams p, int* scratch, const float* x, const int* id, const int* type, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (type[i] < 1 || type[i] > p.ntypes || id[i] < 1) atomicOr(&scratch[kOffStatus], 1);
    if (na_outside(p, x, i)) atomicOr(&scratch[kOffStatus], 2);
    const int c = na_cell(p, x, i);
    scratch[kOffCellOf + i] = c;
    atomicAdd(&scratch[kOffCount + c], 1);
}

// exclusive scan of the cell counts by one block of 1024 threads
__global__ void k_na_scan(int* scratch, int ncell)
{
    __shared__ int sh[1024];
    const int per = (ncell + 1023) / 1024;
    const int b = threadIdx.x * per, e = min(b + per, ncell);
    int tot = 0;
    for (int c = b; c < e; c++) tot += scratch[kOffCount + c];
    sh[threadIdx.x] = tot;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += t;
        __syncthreads();
    }
    int run = sh[threadIdx.x] - tot;
    for (int c = b; c < e; c++) {
        scratch[kOffStart + c] = run;
        run += scratch[kOffCount + c];
    }
    if (threadIdx.x == 1023) scratch[kOffStart + ncell] = sh[1023];
}

__global__ void k_na_scatter(int* scratch, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = scratch[kOffCellOf + i];
    const int slot = scratch[kOffStart + c] + atomicAdd(&scratch[kOffFill + c], 1);
    if (slot >= 0 && slot < n) scratch[kOffSorted + slot] = i;
}

__device__ __forceinline__ float na_min_image(float d, float L)
{
    const float h = 0.5f * L;
    return d - L * (float)((d >= h) - (d < -h));
}

// Full-stencil pair force per atom (each pair evaluated from both sides, no atomics),
// the reference's DPD force with the Saru random term (src/force/pair_dpd.cu:468-558).
__global__ void __launch_bounds__(256) k_na_force(NaParams p, const int* scratch, const float* x,
                                                  const float* v, const int* id, const int* type, int n,
                                                  uint32_t step, float* f)
{
    __shared__ float4 sc[kMaxTypes * kMaxTypes];
    __shared__ float sir[kMaxTypes * kMaxTypes];
    for (int k = threadIdx.x; k < p.ntypes * p.ntypes; k += blockDim.x) {
        sc[k] = p.coeff[k];
        sir[k] = p.inv_rc[k];
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int ti = min(max(type[i], 1), p.ntypes) - 1;
    const int tagi = id[i];
    const float xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
    const float vxi = v[3 * i], vyi = v[3 * i + 1], vzi = v[3 * i + 2];
    const int c = scratch[kOffCellOf + i];
    const int cz = c % p.nc[2], cy = (c / p.nc[2]) % p.nc[1], cx = c / (p.nc[2] * p.nc[1]);
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    for (int ox = -1; ox <= 1; ox++)
        for (int oy = -1; oy <= 1; oy++)
            for (int oz = -1; oz <= 1; oz++) {
                const int nx = (cx + ox + p.nc[0]) % p.nc[0];
                const int ny = (cy + oy + p.nc[1]) % p.nc[1];
                const int nz = (cz + oz + p.nc[2]) % p.nc[2];
                const int nb = (nx * p.nc[1] + ny) * p.nc[2] + nz;
                const int jb = scratch[kOffStart + nb], je = scratch[kOffStart + nb + 1];
                for (int q = jb; q < je; q++) {
                    const int j = scratch[kOffSorted + q];
                    if (j == i) continue;
                    const float dx = na_min_image(xi - x[3 * j], p.L[0]);
                    const float dy = na_min_image(yi - x[3 * j + 1], p.L[1]);
                    const float dz = na_min_image(zi - x[3 * j + 2], p.L[2]);
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 > p.rcmax2) continue;
                    const int tj = min(max(type[j], 1), p.ntypes) - 1;
                    const float4 cc = sc[ti * p.ntypes + tj];
                    if (!(r2 <= cc.w)) continue;
                    const float r = sqrtf(r2);
                    if (r < 1.0e-10f) continue;
                    const float rinv = 1.0f / r;
                    const float dot = dx * (vxi - v[3 * j]) + dy * (vyi - v[3 * j + 1]) + dz * (vzi - v[3 * j + 2]);
                    const float wc = 1.0f - r * sir[ti * p.ntypes + tj];
                    const int tagj = id[j];
                    const float th = saru_theta((uint32_t)min(tagi, tagj), (uint32_t)max(tagi, tagj), p.seed, step);
                    float fpair = cc.x * wc - cc.y * wc * wc * dot * rinv + cc.z * wc * th;
                    fpair *= rinv;
                    fx += dx * fpair;
                    fy += dy * fpair;
                    fz += dz * fpair;
                }
            }
    f[3 * i] = fx;
    f[3 * i + 1] = fy;
    f[3 * i + 2] = fz;
}

std::mutex g_mu;
struct ScratchAddr {
    unsigned long long ctx_id = 0;  // CUDA context the address belongs to (0: none yet)
    int* ptr = nullptr;
};
ScratchAddr g_addr[64];

// the unique id of the calling thread's current CUDA context (driver entry points looked
// up through the runtime, so the library needs no link to libcuda); 0 when unavailable
unsigned long long current_context_id()
{
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
            qb == cudaDriverEntryPointSuccess) {
            get_current = (GetCurrent)a;
            get_id = (GetId)b;
        }
        looked_up = true;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Set-up: the device address of the scratch array, resolved with the device current
// once per device and CUDA context (again after the context changes; on every call when
// the context id cannot be read).  cudaSetDevice makes the device's primary context
// current, so the context read here is the one the kernels will run in.
int scratch_ptr(int** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return DPD_E_NODEV;
    if (cudaSetDevice(dev) != cudaSuccess) return DPD_E_CUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    const unsigned long long ctx = current_context_id();
    ScratchAddr& a = g_addr[dev];
    if (!a.ptr || ctx == 0 || a.ctx_id != ctx) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return DPD_E_CUDA;
        a.ptr = (int*)p;
        a.ctx_id = ctx;
    }
    *out = a.ptr;
    return DPD_OK;
}

}  // namespace

extern "C" int dpd_pair_forces_noalloc(const dpd_pair_params* prm, const float* d_pos, const float* d_vel,
                                       const int* d_id, const int* d_type, int n, uint32_t step,
                                       float* d_force, void* stream)
{
    if (!prm || !d_pos || !d_vel || !d_id || !d_type || !d_force) return DPD_E_ARG;
    if (n < 1 || n > kMaxAtoms) return DPD_E_ARG;
    if (prm->ntypes < 1 || prm->ntypes > kMaxTypes) return DPD_E_ARG;
    if (!(prm->dt > 0) || !(prm->kT >= 0)) return DPD_E_ARG;
    NaParams p;
    double rcmax = 0.0;
    const double sig_scale = std::sqrt(2.0 * prm->kT) / std::sqrt(prm->dt);
    for (int a = 0; a < prm->ntypes; a++)
        for (int b = 0; b < prm->ntypes; b++) {
            const double A = prm->coeff[a][b][0], g = prm->coeff[a][b][1], rc = prm->coeff[a][b][2];
            if (!(rc > 0) || g < 0) return DPD_E_ARG;
            const float rcf = (float)rc;
            p.coeff[a * prm->ntypes + b] = make_float4((float)A, (float)g, (float)(std::sqrt(g) * sig_scale), rcf * rcf);
            p.inv_rc[a * prm->ntypes + b] = (float)(1.0 / rc);
            rcmax = std::max(rcmax, rc);
        }
    p.ncell = 1;
    for (int k = 0; k < 3; k++) {
        const double L = prm->hi[k] - prm->lo[k];
        if (!(L > 0)) return DPD_E_ARG;
        const int nc = (int)std::floor(L / rcmax);
        if (nc < 3) return DPD_E_ARG;
        p.nc[k] = nc;
        p.lo[k] = (float)prm->lo[k];
        p.L[k] = (float)L;
        p.inv_w[k] = (float)(nc / L);
        if ((long long)p.ncell * nc > kMaxCells) return DPD_E_ARG;
        p.ncell *= nc;
    }
    const float rcf = (float)rcmax;
    p.rcmax2 = rcf * rcf;
    p.ntypes = prm->ntypes;
    p.seed = prm->seed;
    int* scratch = nullptr;
    int st = scratch_ptr(&scratch);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    k_na_clear<<<(p.ncell + 255) / 256, 256, 0, s>>>(scratch, p.ncell);
    k_na_count<<<(n + 255) / 256, 256, 0, s>>>(p, scratch, d_pos, d_id, d_type, n);
    k_na_scan<<<1, 1024, 0, s>>>(scratch, p.ncell);
    k_na_scatter<<<(n + 255) / 256, 256, 0, s>>>(scratch, n);
    k_na_force<<<(n + 255) / 256, 256, 0, s>>>(p, scratch, d_pos, d_vel, d_id, d_type, n, step, d_force);
    if (cudaGetLastError() != cudaSuccess) return DPD_E_CUDA;
    int status = 0;
    if (cudaMemcpyAsync(&status, scratch + kOffStatus, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return DPD_E_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return DPD_E_CUDA;
    return status ? DPD_E_ARG : DPD_OK;
}
