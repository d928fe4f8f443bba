// zmaps.cu -- z-column post-processing of FE volumes.
//
// Replaces the convolveZ and izoZ kernels (SPAMMM kernels/AFM.cl:666-723):
// a convolution of every (x,y) column of an FE volume along z with a weight
// vector, and the height at which each column's Fz first exceeds an
// iso-value.  The reference launches them on (nx*ny) columns with one
// work-item per column; here the convolution runs a thread per output texel
// (consecutive threads = consecutive heights of a column: coalesced float4
// rows, the column's inputs shared through L1) with the weights staged in
// shared memory, and the iso-height search a thread per column.
//
// This translation unit is compiled with -fmad=false: the convolution's sums
// are explicit fused multiply-adds in jz order (fe = fma(Fin, w, fe)), the
// order the CPU oracle repeats, so results are bit-identical to it.
#include "spm_internal.cuh"

namespace spm {
namespace {

constexpr int CZ_THREADS = 256;
constexpr int CZ_MAX_W = 1024;

__global__ void __launch_bounds__(CZ_THREADS)
convolve_z_kernel(const float4* __restrict__ Fin, long long n_out_total, int nz_in, int nz_out, const float* __restrict__ w,
                  int nzw, float4* __restrict__ Fout) {
    __shared__ float s_w[CZ_MAX_W];
    for (int i = threadIdx.x; i < nzw; i += CZ_THREADS) s_w[i] = w[i];
    __syncthreads();
    const long long t = (long long)blockIdx.x * CZ_THREADS + threadIdx.x;
    if (t >= n_out_total) return;
    const long long col = t / nz_out;
    const int izo = (int)(t - col * nz_out);
    const float4* f = Fin + col * nz_in + izo;
    float4 fe = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int jz = 0; jz < nzw; jz++) {
        const float4 a = __ldg(f + jz);
        const float wj = s_w[jz];
        fe.x = __fmaf_rn(a.x, wj, fe.x);
        fe.y = __fmaf_rn(a.y, wj, fe.y);
        fe.z = __fmaf_rn(a.z, wj, fe.z);
        fe.w = __fmaf_rn(a.w, wj, fe.w);
    }
    Fout[t] = fe;
}

__global__ void __launch_bounds__(CZ_THREADS)
izo_z_kernel(const float4* __restrict__ Fin, int n_col, int nz, float iso, float* __restrict__ zMap) {
    const int c = blockIdx.x * CZ_THREADS + threadIdx.x;
    if (c >= n_col) return;
    const float4* f = Fin + (long long)c * nz;
    float oz = __ldg(&f[0].z);
    for (int iz = 1; iz < nz; iz++) {
        const float fz = __ldg(&f[iz].z);
        if (fz > iso) {
            const float t = __fdiv_rn(iso - oz, fz - oz);
            zMap[c] = (float)iz + t;
            return;
        }
        oz = fz;
    }
    zMap[c] = -1.f;
}

}  // namespace
}  // namespace spm

extern "C" int spm_convolve_z(const float* Fin, int n_col, int nz_in, int nz_out, const float* w, float* Fout,
                              void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(n_col >= 0 && nz_in >= 0 && nz_out >= 0, "spm_convolve_z: negative sizes (%d,%d,%d)", n_col, nz_in,
                nz_out);
    const int nzw = nz_in - nz_out;
    SPM_REQUIRE(nzw >= 0 && nzw <= CZ_MAX_W, "spm_convolve_z: nz_in - nz_out = %d outside [0, %d]", nzw, CZ_MAX_W);
    const long long total = (long long)n_col * nz_out;
    if (total == 0) return SPM_OK;
    SPM_REQUIRE(Fin && Fout && (nzw == 0 || w), "spm_convolve_z: null pointer");
    SPM_REQUIRE(aligned16(Fin) && aligned16(Fout) && (reinterpret_cast<uintptr_t>(w) & 3u) == 0,
                "spm_convolve_z: misaligned buffers");
    const long long blocks = (total + CZ_THREADS - 1) / CZ_THREADS;
    SPM_REQUIRE(blocks < (1LL << 31), "spm_convolve_z: %lld outputs are too many", total);
    convolve_z_kernel<<<(unsigned)blocks, CZ_THREADS, 0, as_stream(stream)>>>(
        reinterpret_cast<const float4*>(Fin), total, nz_in, nz_out, w, nzw, reinterpret_cast<float4*>(Fout));
    return check_launch("spm_convolve_z");
}

extern "C" int spm_izo_z(const float* Fin, int n_col, int nz, float iso, float* zMap, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(n_col >= 0 && nz >= 0, "spm_izo_z: negative sizes (%d,%d)", n_col, nz);
    if (n_col == 0) return SPM_OK;
    SPM_REQUIRE(nz >= 1, "spm_izo_z: nz=%d < 1", nz);
    SPM_REQUIRE(Fin && zMap, "spm_izo_z: null pointer");
    SPM_REQUIRE(aligned16(Fin) && (reinterpret_cast<uintptr_t>(zMap) & 3u) == 0, "spm_izo_z: misaligned buffers");
    izo_z_kernel<<<(unsigned)((n_col + CZ_THREADS - 1) / CZ_THREADS), CZ_THREADS, 0, as_stream(stream)>>>(
        reinterpret_cast<const float4*>(Fin), n_col, nz, iso, zMap);
    return check_launch("spm_izo_z");
}
