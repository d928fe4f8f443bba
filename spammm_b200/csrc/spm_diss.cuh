// spm_diss.cuh -- the dissipation integral of one pixel, shared by
// spm_dissipation (df.cu) and the fused epilogue of the paired relaxation
// (relax.cu), so both compute the same bits.
//
// compute_dissipation (SPAMMM spammm/SPM/AFM.py:3238-3277):
// E_diss = |trapz over the heights idx[off[o]..off[o+1]) of (F_fwd - F_bwd).n|
// with abscissae h, in FP64, as sum_j (h[b]-h[a]) * (dF(a) + dF(b)) / 2.
// An index outside [0, nz) makes the value NaN (never read out of bounds).
// Compiled with -fmad=false in both translation units.
#pragma once
#include <cuda_runtime.h>

namespace spm {

struct DissRow {
    double x, y, z;
};

// F.n of row i of a float4 FE array (rows of 4 floats); LOAD: a functor
// float4 (const float4*) choosing the load path (read-only cache or coherent).
template <class LOAD>
__device__ __forceinline__ double diss_fn(const float4* v, size_t i, const double (&n)[3], const LOAD& ld) {
    const float4 f = ld(v + i);
    return ((double)f.x * n[0] + (double)f.y * n[1]) + (double)f.z * n[2];
}

template <class LOAD>
__device__ __forceinline__ float diss_value(const float4* Ff, const float4* Fb, size_t row0, int nz,
                                            const double (&n)[3], const double* __restrict__ h,
                                            const int* __restrict__ off, const int* __restrict__ idx, int o,
                                            const LOAD& ld) {
    double acc = 0.0;
    const int j0 = off[o], j1 = off[o + 1];
    for (int t = j0; t + 1 < j1; t++) {
        const int a = idx[t], b = idx[t + 1];
        if (a < 0 || a >= nz || b < 0 || b >= nz) {
            acc = __longlong_as_double(0x7ff8000000000000LL);
            break;
        }
        const double da = diss_fn(Ff, row0 + a, n, ld) - diss_fn(Fb, row0 + a, n, ld);
        const double db = diss_fn(Ff, row0 + b, n, ld) - diss_fn(Fb, row0 + b, n, ld);
        acc += (h[b] - h[a]) * (da + db) / 2.0;
    }
    return (float)fabs(acc);
}

struct LdgLoad {
    __device__ __forceinline__ float4 operator()(const float4* p) const { return __ldg(p); }
};
// Coherent L2 load: data written earlier in the same kernel by another thread (after a fence).
struct CgLoad {
    __device__ __forceinline__ float4 operator()(const float4* p) const {
        float4 r;
        asm volatile("ld.global.cg.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
                     : "l"(p));
        return r;
    }
};

}  // namespace spm
