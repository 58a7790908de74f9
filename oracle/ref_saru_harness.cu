// Test-infrastructure harness: compiles the reference's src/force/pair_dpd.cu in this
// translation unit (by #include from the reference tree, nothing copied) so that its
// file-static Saru generator (src/force/pair_dpd.cu:212-236) can be called on the GPU
// to produce known-answer vectors.  Built by oracle/build_ref.sh into oracle/_ref/.
//
// usage: ref_saru in.bin out.bin
//   in.bin : int32 n, then n records of {uint32 t1, uint32 t2, uint32 seed, int32 step}
//   out.bin: n float32 random numbers
#include "force/pair_dpd.cu"

__constant__ numtyp masses[256];
__constant__ numtyp gpu_pair_coeff[256];
__constant__ numtyp gpu_bond_coeff[256];
__constant__ numtyp gpu_angle_coeff[256];

__global__ void k_saru_kat(const unsigned* rec, float* out, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    numtyp r = 0;
    saru(rec[4 * i], rec[4 * i + 1], rec[4 * i + 2], (int)rec[4 * i + 3], r);
    out[i] = (float)r;
}

int main(int argc, char** argv)
{
    if (argc != 3) return 2;
    FILE* f = fopen(argv[1], "rb");
    if (!f) return 3;
    int n = 0;
    if (fread(&n, 4, 1, f) != 1 || n <= 0 || n > (1 << 24)) return 4;
    std::vector<unsigned> rec(4 * (size_t)n);
    if (fread(rec.data(), 4, rec.size(), f) != rec.size()) return 5;
    fclose(f);
    unsigned* d_rec = nullptr;
    float* d_out = nullptr;
    CUDA_CHECK(cudaMalloc(&d_rec, 4 * rec.size()));
    CUDA_CHECK(cudaMalloc(&d_out, 4 * (size_t)n));
    CUDA_CHECK(cudaMemcpy(d_rec, rec.data(), 4 * rec.size(), cudaMemcpyHostToDevice));
    k_saru_kat<<<(n + 255) / 256, 256>>>(d_rec, d_out, n);
    CUDA_CHECK(cudaGetLastError());
    std::vector<float> out(n);
    CUDA_CHECK(cudaMemcpy(out.data(), d_out, 4 * (size_t)n, cudaMemcpyDeviceToHost));
    FILE* g = fopen(argv[2], "wb");
    if (!g) return 6;
    fwrite(out.data(), 4, n, g);
    fclose(g);
    return 0;
}
