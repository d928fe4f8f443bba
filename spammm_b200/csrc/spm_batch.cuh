// spm_batch.cuh -- helpers shared by the batched kernels.
//
// A batch is an array of spm_batch_mol descriptors in device memory.  Work
// items of every stage (grid tiles, relaxation slots, states, gather units,
// loss chunks, pixels, atoms) are numbered across the batch by a prefix field
// of the descriptor; the molecule that owns item x is the largest m with
// prefix(m) <= x, found by binary search (log2(n_mol) cached loads).
#pragma once
#include "spm_internal.cuh"
#include "spm_fire.cuh"

namespace spm {

template <typename T, T spm_batch_mol::*F>
__device__ __forceinline__ int find_mol(const spm_batch_mol* __restrict__ mols, int n_mol, long long x) {
    int lo = 0, hi = n_mol - 1;  // mols[0].*F == 0 <= x
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((long long)__ldg(&(mols[mid].*F)) <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

#define SPM_MOL_BY(field, mols, n, x) find_mol<decltype(spm_batch_mol::field), &spm_batch_mol::field>(mols, n, x)

// The molecule of item x, stepping forward from m, the molecule of an item <= x
// (a CTA that takes several consecutive items searches once, then steps).
template <typename T, T spm_batch_mol::*F>
__device__ __forceinline__ int step_mol(const spm_batch_mol* __restrict__ mols, int n_mol, int m, long long x) {
    while (m + 1 < n_mol && (long long)__ldg(&(mols[m + 1].*F)) <= x) m++;
    return m;
}

#define SPM_MOL_STEP(field, mols, n, m, x) \
    step_mol<decltype(spm_batch_mol::field), &spm_batch_mol::field>(mols, n, m, x)

__device__ __forceinline__ float4 ld4f(const float* a) { return make_float4(__ldg(a), __ldg(a + 1), __ldg(a + 2), __ldg(a + 3)); }

// Pixel k of relaxation slot lt (slot index within molecule D).  With a
// raster (raster_ny > 0) slots run over tiles of (32 >> th_log2) (ix) x
// (1 << th_log2) (iy) pixels, 32 slots per tile, tiles ordered iy-fastest;
// without one, slot lt is pixel lt.  false: the slot lies outside the raster
// (an edge tile) or past the last pixel.
__device__ __forceinline__ bool slot_pixel(const spm_batch_mol* D, unsigned lt, int th_log2, int& k) {
    const int ny = D->raster_ny, n_scan = D->n_scan;
    if (ny <= 0) {
        k = (int)lt;
        return k < n_scan;
    }
    const int nxr = n_scan / ny;
    const unsigned th = 1u << th_log2;
    const unsigned nty = ((unsigned)ny + th - 1u) >> th_log2;
    const unsigned tile = lt >> 5, r = lt & 31u;
    const int ix = (int)((tile / nty) * (32u >> th_log2) + (r >> th_log2));
    const int iy = (int)((tile % nty) * th + (r & (th - 1u)));
    k = ix * ny + iy;
    return ix < nxr && iy < ny;
}

// Sampling view of a molecule's slab (full-grid coordinates, the stored box
// only; stride float4 per stored node: 2 x-pairs, 4 xz-quads, value first).
__device__ __forceinline__ GridView slab_view(const spm_batch_mol& D, const float* grid, int stride = 2) {
    GridView G;
    G.g = reinterpret_cast<const float4*>(grid) + (long long)stride * D.grid_off;
    G.stride = stride;
    G.nx = D.nx; G.ny = D.ny; G.nz = D.nz;
    G.dA = ld4f(D.dinvA);
    G.dB = ld4f(D.dinvB);
    G.dC = ld4f(D.dinvC);
    G.x_lo = D.x_lo;
    G.nx_slab = D.nx_slab;
    G.y_lo = D.y_lo;
    G.ny_slab = D.ny_slab;
    G.z_lo = D.z_lo;
    G.nz_slab = D.nz_slab;
    return G;
}

}  // namespace spm
