// df.cu -- stage (c): frequency shift, dissipation and the df loss seed.
//
// Replaces the host NumPy/SciPy post-processing of SPAMMM:
//   compute_df_amp_dir  spammm/SPM/AFM.py:3203-3236 (9-point Gauss-Chebyshev,
//                       scipy.ndimage.map_coordinates(order=1, mode='nearest'),
//                       numpy.gradient with edge_order=1)
//   compute_df_dir      spammm/SPM/AFM.py:3105-3123
//   compute_dissipation spammm/SPM/AFM.py:3238-3277
//   df_loss_seed        spammm/SPM/AFM.py:3125-3200
// All arithmetic is FP64, as on the reference host.  The FEs volume is
// (nx,ny,nz,4) float32 with z fastest.  The amplitude df is FP64-arithmetic
// bound (9 quadrature nodes x 2 interpolations per output): the z-column
// kernels tabulate each interpolated sample once per column, and the finite
// differences multiply by 1/dr and 1/(2 dr) instead of dividing (within an
// FP64 ulp of numpy.gradient's division; the float32 results are unchanged at
// the reference fixtures' tolerance).  Compiled with -fmad=false so the FP64
// expression order otherwise matches NumPy's.
#include "spm_internal.cuh"
#include "spm_diss.cuh"
#include "spm_batch.cuh"
#include <cmath>
#include <vector>

namespace spm {
namespace {

constexpr int DF_THREADS = 256;
constexpr int NQ = 9;  // Gauss-Chebyshev nodes

struct DfGeom {
    int nx, ny, nz;
    double n[3];       // oscillation direction (unit)
    double dr[3];      // spacing
    double shift[3];   // amp * n / dr
    double idr[3];     // 1 / dr and 1 / (2 dr): the one-sided and central differences multiply by them
    double idr2[3];
    double uk[NQ];     // cos((2k+1) pi / 18)
    double wk;         // 1/9
    int act[3];        // active axes (|n| > 1e-15)
    int nact;
};

// One (Fx,Fy,Fz,E) row of an FP32 or FP64 volume, widened to double.
struct Row {
    double x, y, z, w;
};
__device__ __forceinline__ Row load_row(const float* __restrict__ v, size_t i) {
    const float4 f = __ldg(reinterpret_cast<const float4*>(v) + i);
    return Row{(double)f.x, (double)f.y, (double)f.z, (double)f.w};
}
__device__ __forceinline__ Row load_row(const double* __restrict__ v, size_t i) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(v) + 2 * i);
    const double2 b = __ldg(reinterpret_cast<const double2*>(v) + 2 * i + 1);
    return Row{a.x, a.y, b.x, b.y};
}

template <typename T>
__device__ __forceinline__ double fn_at(const T* __restrict__ FEs, const DfGeom& P, int ix, int iy, int iz) {
    const Row f = load_row(FEs, ((size_t)ix * P.ny + iy) * P.nz + iz);
    return (f.x * P.n[0] + f.y * P.n[1]) + f.z * P.n[2];
}

__device__ __forceinline__ int clampi(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

// map_coordinates(F_n, (ix,iy,iz) + u*shift, order=1, mode='nearest'):
// per-axis weights (1-t, t) at floor(c), clamped indices, corners summed with
// the last axis fastest and each term formed as ((f*w0)*w1)*w2.
template <typename T>
__device__ double shifted_fn(const T* __restrict__ FEs, const DfGeom& P, int ix, int iy, int iz, double u) {
    const int dims[3] = {P.nx, P.ny, P.nz};
    const int idx[3] = {ix, iy, iz};
    int i0[3];
    double w[3][2];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double c = (double)idx[d] + u * P.shift[d];
        const double fl = floor(c);
        const double t = c - fl;
        i0[d] = (int)fl;
        w[d][0] = 1.0 - t;
        w[d][1] = t;
    }
    double acc = 0.0;
#pragma unroll
    for (int a0 = 0; a0 < 2; a0++) {
        if (w[0][a0] == 0.0) continue;
#pragma unroll
        for (int a1 = 0; a1 < 2; a1++) {
            if (w[1][a1] == 0.0) continue;
#pragma unroll
            for (int a2 = 0; a2 < 2; a2++) {
                if (w[2][a2] == 0.0) continue;
                double coeff = fn_at(FEs, P, clampi(i0[0] + a0, dims[0]), clampi(i0[1] + a1, dims[1]),
                                     clampi(i0[2] + a2, dims[2]));
                coeff *= w[0][a0];
                coeff *= w[1][a1];
                coeff *= w[2][a2];
                acc += coeff;
            }
        }
    }
    return acc;
}

// numpy.gradient(S, dr, axis) at one point, uniform spacing, edge_order=1.
template <bool AMP, typename T>
__device__ double grad_at(const T* __restrict__ FEs, const DfGeom& P, int ax, int ix, int iy, int iz, double u) {
    const int dims[3] = {P.nx, P.ny, P.nz};
    int idx[3] = {ix, iy, iz};
    const int i = idx[ax], n = dims[ax];
    auto S = [&](int j) {
        int q[3] = {idx[0], idx[1], idx[2]};
        q[ax] = j;
        return AMP ? shifted_fn(FEs, P, q[0], q[1], q[2], u) : fn_at(FEs, P, q[0], q[1], q[2]);
    };
    if (i == 0) return (S(1) - S(0)) * P.idr[ax];
    if (i == n - 1) return (S(n - 1) - S(n - 2)) * P.idr[ax];
    return (S(i + 1) - S(i - 1)) * P.idr2[ax];
}

template <typename T>
__global__ void __launch_bounds__(DF_THREADS)
df_amp_dir_kernel(const T* __restrict__ FEs, DfGeom P, const int* __restrict__ out_iz, int n_out,
                  float* __restrict__ df) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)P.nx * P.ny * n_out;
    if (gid >= total) return;
    const int o = (int)(gid % n_out);
    const long long pix = gid / n_out;
    const int iy = (int)(pix % P.ny), ix = (int)(pix / P.ny);
    const int iz = out_iz ? out_iz[o] : o;
    if (iz < 0 || iz >= P.nz) {  // invalid selection: flag the element instead of reading out of bounds
        df[gid] = __int_as_float(0x7fc00000);
        return;
    }
    double acc = 0.0;
    for (int k = 0; k < NQ; k++) {
        for (int a = 0; a < P.nact; a++) {
            const int ax = P.act[a];
            const double g = grad_at<true>(FEs, P, ax, ix, iy, iz, P.uk[k]);
            acc -= (P.wk * P.n[ax]) * g;
        }
    }
    df[gid] = (float)acc;
}

// Oscillation along +-z only (the common case): one warp per pixel column.
// The column's F_n values are staged once in shared memory (coalesced reads of
// nz contiguous rows); each lane then evaluates its output heights with the
// same expression sequence as df_amp_dir_kernel (x/y weights are exactly 1
// there and the zero-weight corners are skipped), so results are identical.
constexpr int DFZ_WARPS = 8;
constexpr int DFZ_MAXNZ = 512;
constexpr int DFZ_TAB = 64;  // columns up to this height take each quadrature sample once (a table row)

// acc - wk * (central difference of the tabulated samples at height iz): the
// per-node step of the amplitude average, the one-sided difference at the
// column's ends (iz < 0 or >= nz: no output, acc unchanged).
__device__ __forceinline__ double df_accumulate(double acc, int iz, int nz, const double* row, double idr,
                                                double idr2, double wkn) {
    if (iz < 0 || iz >= nz) return acc;
    double g;
    if (iz == 0) g = (row[1] - row[0]) * idr;
    else if (iz == nz - 1) g = (row[nz - 1] - row[nz - 2]) * idr;
    else g = (row[iz + 1] - row[iz - 1]) * idr2;
    return acc - wkn * g;
}

template <typename T>
__global__ void __launch_bounds__(DFZ_WARPS * 32)
df_amp_z_kernel(const T* __restrict__ FEs, DfGeom P, const int* __restrict__ out_iz, int n_out,
                float* __restrict__ df) {
    __shared__ double s_fn[DFZ_WARPS][DFZ_MAXNZ];
    __shared__ double s_row[DFZ_WARPS][DFZ_TAB];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const long long pix = (long long)blockIdx.x * DFZ_WARPS + w;
    if (pix >= (long long)P.nx * P.ny) return;  // whole warp exits together: no CTA barrier below
    const int nz = P.nz;
    double* fn = s_fn[w];
    for (int z = l; z < nz; z += 32) {
        const Row f = load_row(FEs, (size_t)pix * nz + z);
        fn[z] = (f.x * P.n[0] + f.y * P.n[1]) + f.z * P.n[2];
    }
    __syncwarp();
    const double sh = P.shift[2], nzc = P.n[2];
    auto S = [&](int j, double u) {
        const double c = (double)j + u * sh;
        const double fl = floor(c);
        const double t = c - fl;
        const int i0 = (int)fl;
        const double w0 = 1.0 - t, w1 = t;
        double acc = 0.0;
        if (w0 != 0.0) acc += fn[clampi(i0, nz)] * w0;
        if (w1 != 0.0) acc += fn[clampi(i0 + 1, nz)] * w1;
        return acc;
    };
    if (nz >= 2 && nz <= DFZ_TAB && n_out <= DFZ_TAB) {
        // each S(j, u_k) once: per quadrature node the warp tabulates the column's nz samples, then
        // every output takes its central difference from the table (same values, same order)
        double* row = s_row[w];
        int izs[DFZ_TAB / 32];
        double acc[DFZ_TAB / 32];
#pragma unroll
        for (int m = 0; m < DFZ_TAB / 32; m++) {
            const int o = l + 32 * m;
            izs[m] = o < n_out ? (out_iz ? out_iz[o] : o) : -1;
            acc[m] = 0.0;
        }
        for (int k = 0; k < NQ; k++) {
            const double u = P.uk[k];
            for (int j = l; j < nz; j += 32) row[j] = S(j, u);
            __syncwarp();
#pragma unroll
            for (int m = 0; m < DFZ_TAB / 32; m++) acc[m] = df_accumulate(acc[m], izs[m], nz, row, P.idr[2], P.idr2[2], P.wk * nzc);
            __syncwarp();  // the row is rewritten for the next node
        }
#pragma unroll
        for (int m = 0; m < DFZ_TAB / 32; m++) {
            const int o = l + 32 * m;
            if (o < n_out)
                df[pix * n_out + o] = (izs[m] < 0 || izs[m] >= nz) ? __int_as_float(0x7fc00000) : (float)acc[m];
        }
        return;
    }
    for (int o = l; o < n_out; o += 32) {
        const int iz = out_iz ? out_iz[o] : o;
        float res;
        if (iz < 0 || iz >= nz) {
            res = __int_as_float(0x7fc00000);
        } else {
            double acc = 0.0;
            for (int k = 0; k < NQ; k++) {
                const double u = P.uk[k];
                double g;
                if (iz == 0) g = (S(1, u) - S(0, u)) * P.idr[2];
                else if (iz == nz - 1) g = (S(nz - 1, u) - S(nz - 2, u)) * P.idr[2];
                else g = (S(iz + 1, u) - S(iz - 1, u)) * P.idr2[2];
                acc -= (P.wk * nzc) * g;
            }
            res = (float)acc;
        }
        df[pix * n_out + o] = res;
    }
}

template <typename T>
__global__ void __launch_bounds__(DF_THREADS)
df_dir_kernel(const T* __restrict__ FEs, DfGeom P, double* __restrict__ df) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)P.nx * P.ny * P.nz;
    if (gid >= total) return;
    const int iz = (int)(gid % P.nz);
    const long long pix = gid / P.nz;
    const int iy = (int)(pix % P.ny), ix = (int)(pix / P.ny);
    double acc = 0.0;
    for (int a = 0; a < P.nact; a++) {
        const int ax = P.act[a];
        acc -= P.n[ax] * grad_at<false>(FEs, P, ax, ix, iy, iz, 0.0);
    }
    df[gid] = acc;
}

struct DissGeom {
    int nx, ny, nz, n_out;
    double n[3];
};

// |sum_j (x[j+1]-x[j]) * (y[j] + y[j+1]) / 2| over the masked heights.  Float
// volumes use spm_diss.cuh's diss_value (shared with the fused epilogue of the
// paired relaxation in relax.cu): the same operations, as written below.
__global__ void __launch_bounds__(DF_THREADS)
dissipation_f32_kernel(const float4* __restrict__ Ff, const float4* __restrict__ Fb, DissGeom P,
                       const double* __restrict__ h, const int* __restrict__ off, const int* __restrict__ idx,
                       float* __restrict__ E) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)P.nx * P.ny * P.n_out;
    if (gid >= total) return;
    const int o = (int)(gid % P.n_out);
    const long long pix = gid / P.n_out;
    const double n[3] = {P.n[0], P.n[1], P.n[2]};
    E[gid] = diss_value(Ff, Fb, (size_t)pix * P.nz, P.nz, n, h, off, idx, o, LdgLoad{});
}

template <typename T>
__global__ void __launch_bounds__(DF_THREADS)
dissipation_kernel(const T* __restrict__ Ff, const T* __restrict__ Fb, DissGeom P,
                   const double* __restrict__ h, const int* __restrict__ off, const int* __restrict__ idx,
                   float* __restrict__ E) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)P.nx * P.ny * P.n_out;
    if (gid >= total) return;
    const int o = (int)(gid % P.n_out);
    const long long pix = gid / P.n_out;
    auto dF = [&](int j) {
        const Row a = load_row(Ff, (size_t)pix * P.nz + j), b = load_row(Fb, (size_t)pix * P.nz + j);
        const double fa = (a.x * P.n[0] + a.y * P.n[1]) + a.z * P.n[2];
        const double fbv = (b.x * P.n[0] + b.y * P.n[1]) + b.z * P.n[2];
        return fa - fbv;
    };
    double acc = 0.0;
    const int j0 = off[o], j1 = off[o + 1];
    for (int t = j0; t + 1 < j1; t++) {
        const int a = idx[t], b = idx[t + 1];
        if (a < 0 || a >= P.nz || b < 0 || b >= P.nz) {  // invalid index list: flag, never read out of bounds
            acc = __longlong_as_double(0x7ff8000000000000LL);
            break;
        }
        acc += (h[b] - h[a]) * (dF(a) + dF(b)) / 2.0;
    }
    E[gid] = (float)fabs(acc);
}

// ---- df loss seed: df, per-block partial sums of w and w*(df-t)^2 ----------
constexpr int LS_THREADS = 256;

template <typename T>
__global__ void __launch_bounds__(LS_THREADS)
loss_partials_kernel(const T* __restrict__ FEs, const double* __restrict__ tgt, const double* __restrict__ wts,
                     int nx, int ny, int nz, double idz2, double* __restrict__ df_out, double* __restrict__ partial) {
    __shared__ double s_w[LS_THREADS], s_l[LS_THREADS];
    const long long total = (long long)nx * ny * nz;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double w = 0.0, l = 0.0;
    if (gid < total) {
        const int iz = (int)(gid % nz);
        double d = 0.0;
        if (iz > 0 && iz < nz - 1) {
            const double fp = load_row(FEs, gid + 1).z, fm = load_row(FEs, gid - 1).z;
            d = -(fp - fm) * idz2;
        }
        df_out[gid] = d;
        w = wts ? wts[gid] : ((iz > 0 && iz < nz - 1) ? 1.0 : 0.0);
        const double diff = d - tgt[gid];
        l = w * (diff * diff);
    }
    s_w[threadIdx.x] = w;
    s_l[threadIdx.x] = l;
    __syncthreads();
    for (int s = LS_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            s_w[threadIdx.x] += s_w[threadIdx.x + s];
            s_l[threadIdx.x] += s_l[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = s_w[0];
        partial[2 * blockIdx.x + 1] = s_l[0];
    }
}

// One CTA folds the per-block partials in a fixed order: (wsum, loss).
__global__ void __launch_bounds__(LS_THREADS)
loss_final_kernel(const double* __restrict__ partial, int nblk, double* __restrict__ sums, double* __restrict__ loss) {
    __shared__ double s_w[LS_THREADS], s_l[LS_THREADS];
    double w = 0.0, l = 0.0;
    for (int i = threadIdx.x; i < nblk; i += LS_THREADS) {
        w += partial[2 * i];
        l += partial[2 * i + 1];
    }
    s_w[threadIdx.x] = w;
    s_l[threadIdx.x] = l;
    __syncthreads();
    for (int s = LS_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            s_w[threadIdx.x] += s_w[threadIdx.x + s];
            s_l[threadIdx.x] += s_l[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        sums[0] = s_w[0];
        sums[1] = s_l[0];
        loss[0] = 0.5 * s_l[0] / s_w[0];
    }
}

// dL/dFz = transpose of the central-difference stencil applied to w*(df-t)/wsum (df and the
// gradient multiply by the reciprocals 1/(2 dz) and 1/wsum, computed once: within an ulp of the
// divisions, which cost the loss kernels a divergent FP64 division per state).
__global__ void __launch_bounds__(LS_THREADS)
loss_grad_kernel(const double* __restrict__ df, const double* __restrict__ tgt, const double* __restrict__ wts,
                 const double* __restrict__ sums, int nx, int ny, int nz, double coeff, float4* __restrict__ dL) {
    const long long total = (long long)nx * ny * nz;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= total) return;
    const int iz = (int)(gid % nz);
    const double iwsum = 1.0 / sums[0];  // one division per thread, the same for every thread
    auto g = [&](long long j) {
        const int jz = (int)(j % nz);
        const double w = wts ? wts[j] : ((jz > 0 && jz < nz - 1) ? 1.0 : 0.0);
        return w * (df[j] - tgt[j]) * iwsum;
    };
    double v;
    if (iz == 0) v = g(gid + 1) * coeff;
    else if (iz == nz - 1) v = -g(gid - 1) * coeff;
    else v = (g(gid + 1) - g(gid - 1)) * coeff;
    dL[gid] = make_float4(0.f, 0.f, (float)v, 0.f);
}

int fill_geom(DfGeom& P, int nx, int ny, int nz, const double* n, const double* dr, double amp) {
    P.nx = nx; P.ny = ny; P.nz = nz;
    P.nact = 0;
    for (int d = 0; d < 3; d++) {
        P.n[d] = n[d];
        P.dr[d] = dr[d];
        P.shift[d] = (amp * n[d]) / dr[d];
        P.idr[d] = 1.0 / dr[d];
        P.idr2[d] = 1.0 / (2.0 * dr[d]);
        if (fabs(n[d]) > 1e-15) P.act[P.nact++] = d;
    }
    for (int k = 0; k < NQ; k++) P.uk[k] = cos((double)(2 * k + 1) / (double)(2 * NQ) * M_PI);
    P.wk = 1.0 / NQ;
    const int dims[3] = {nx, ny, nz};
    for (int a = 0; a < P.nact; a++)
        if (dims[P.act[a]] < 2)
            return set_error(SPM_ERR_ARG, "df: FEs axis %d needs at least 2 samples for this oscillation direction",
                             P.act[a]);
    return SPM_OK;
}

}  // namespace
}  // namespace spm

extern "C" int spm_df_amp_dir(const void* FEs, int fes_dtype, int nx, int ny, int nz, const double* n,
                              const double* dr, double amp, const int* out_iz, int n_out, float* df, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(FEs && df && n && dr, "spm_df_amp_dir: null pointer");
    SPM_REQUIRE(fes_dtype == SPM_F32 || fes_dtype == SPM_F64, "spm_df_amp_dir: fes_dtype=%d", fes_dtype);
    SPM_REQUIRE(nx > 0 && ny > 0 && nz > 0, "spm_df_amp_dir: dims (%d,%d,%d) must be positive", nx, ny, nz);
    SPM_REQUIRE(aligned16(FEs), "spm_df_amp_dir: FEs not 16-byte aligned");
    for (int d = 0; d < 3; d++)
        SPM_REQUIRE(std::isfinite(n[d]) && std::isfinite(dr[d]) && dr[d] > 0.0,
                    "spm_df_amp_dir: n/dr must be finite with dr > 0");
    SPM_REQUIRE(std::isfinite(amp), "spm_df_amp_dir: amp must be finite");
    DfGeom P;
    int rc = fill_geom(P, nx, ny, nz, n, dr, amp);
    if (rc) return rc;
    if (out_iz == nullptr) n_out = nz;
    SPM_REQUIRE(n_out >= 0, "spm_df_amp_dir: n_out=%d < 0", n_out);
    const long long total = (long long)nx * ny * n_out;
    if (total == 0) return SPM_OK;
    if (n[0] == 0.0 && n[1] == 0.0 && nz <= DFZ_MAXNZ) {  // z-only oscillation: column kernel
        const long long npix = (long long)nx * ny;
        const unsigned nb = (unsigned)((npix + DFZ_WARPS - 1) / DFZ_WARPS);
        if (fes_dtype == SPM_F32)
            df_amp_z_kernel<<<nb, DFZ_WARPS * 32, 0, as_stream(stream)>>>(static_cast<const float*>(FEs), P, out_iz,
                                                                           n_out, df);
        else
            df_amp_z_kernel<<<nb, DFZ_WARPS * 32, 0, as_stream(stream)>>>(static_cast<const double*>(FEs), P, out_iz,
                                                                           n_out, df);
        return check_launch("spm_df_amp_dir");
    }
    const unsigned nb = (unsigned)((total + DF_THREADS - 1) / DF_THREADS);
    if (fes_dtype == SPM_F32)
        df_amp_dir_kernel<<<nb, DF_THREADS, 0, as_stream(stream)>>>(static_cast<const float*>(FEs), P, out_iz, n_out, df);
    else
        df_amp_dir_kernel<<<nb, DF_THREADS, 0, as_stream(stream)>>>(static_cast<const double*>(FEs), P, out_iz, n_out, df);
    return check_launch("spm_df_amp_dir");
}

extern "C" int spm_df_dir(const void* FEs, int fes_dtype, int nx, int ny, int nz, const double* n, const double* dr,
                          double* df, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(FEs && df && n && dr, "spm_df_dir: null pointer");
    SPM_REQUIRE(fes_dtype == SPM_F32 || fes_dtype == SPM_F64, "spm_df_dir: fes_dtype=%d", fes_dtype);
    SPM_REQUIRE(nx > 0 && ny > 0 && nz > 0, "spm_df_dir: dims (%d,%d,%d) must be positive", nx, ny, nz);
    SPM_REQUIRE(aligned16(FEs), "spm_df_dir: FEs not 16-byte aligned");
    for (int d = 0; d < 3; d++)
        SPM_REQUIRE(std::isfinite(n[d]) && std::isfinite(dr[d]) && dr[d] > 0.0, "spm_df_dir: n/dr must be finite, dr > 0");
    DfGeom P;
    int rc = fill_geom(P, nx, ny, nz, n, dr, 0.0);
    if (rc) return rc;
    const long long total = (long long)nx * ny * nz;
    const unsigned nb = (unsigned)((total + DF_THREADS - 1) / DF_THREADS);
    if (fes_dtype == SPM_F32)
        df_dir_kernel<<<nb, DF_THREADS, 0, as_stream(stream)>>>(static_cast<const float*>(FEs), P, df);
    else
        df_dir_kernel<<<nb, DF_THREADS, 0, as_stream(stream)>>>(static_cast<const double*>(FEs), P, df);
    return check_launch("spm_df_dir");
}

extern "C" int spm_dissipation(const void* FEs_fwd, const void* FEs_bwd, int fes_dtype, int nx, int ny, int nz,
                               const double* n, const double* h_scan, const int* off, const int* idx, int n_out,
                               float* E_diss, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(FEs_fwd && FEs_bwd && n && h_scan && off && idx && E_diss, "spm_dissipation: null pointer");
    SPM_REQUIRE(fes_dtype == SPM_F32 || fes_dtype == SPM_F64, "spm_dissipation: fes_dtype=%d", fes_dtype);
    SPM_REQUIRE(nx > 0 && ny > 0 && nz > 0 && n_out >= 0, "spm_dissipation: bad dims (%d,%d,%d) n_out=%d", nx, ny, nz,
                n_out);
    SPM_REQUIRE(aligned16(FEs_fwd) && aligned16(FEs_bwd), "spm_dissipation: FEs not 16-byte aligned");
    DissGeom P;
    P.nx = nx; P.ny = ny; P.nz = nz; P.n_out = n_out;
    for (int d = 0; d < 3; d++) P.n[d] = n[d];
    const long long total = (long long)nx * ny * n_out;
    if (total == 0) return SPM_OK;
    const unsigned nb = (unsigned)((total + DF_THREADS - 1) / DF_THREADS);
    if (fes_dtype == SPM_F32)
        dissipation_f32_kernel<<<nb, DF_THREADS, 0, as_stream(stream)>>>(
            static_cast<const float4*>(FEs_fwd), static_cast<const float4*>(FEs_bwd), P, h_scan, off, idx, E_diss);
    else
        dissipation_kernel<<<nb, DF_THREADS, 0, as_stream(stream)>>>(static_cast<const double*>(FEs_fwd),
                                                                     static_cast<const double*>(FEs_bwd), P, h_scan,
                                                                     off, idx, E_diss);
    return check_launch("spm_dissipation");
}

extern "C" long long spm_df_loss_scratch_bytes(int nx, int ny, int nz) {
    const long long total = (long long)nx * ny * nz;
    if (nx <= 0 || ny <= 0 || nz <= 0) return 0;
    const long long nblk = (total + spm::LS_THREADS - 1) / spm::LS_THREADS;
    return (2 * nblk + 2) * (long long)sizeof(double);
}

extern "C" int spm_df_loss_seed(const void* FEs, int fes_dtype, const double* target, const double* weights, int nx,
                                int ny, int nz, double dtip, double* df_out, float* dL_dFEs, double* loss_out,
                                void* scratch, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(FEs && target && df_out && dL_dFEs && loss_out && scratch, "spm_df_loss_seed: null pointer");
    SPM_REQUIRE(fes_dtype == SPM_F32 || fes_dtype == SPM_F64, "spm_df_loss_seed: fes_dtype=%d", fes_dtype);
    SPM_REQUIRE(nx > 0 && ny > 0, "spm_df_loss_seed: nx=%d ny=%d must be positive", nx, ny);
    SPM_REQUIRE(nz >= 3, "spm_df_loss_seed: need nz>=3 for central difference, got nz=%d", nz);
    SPM_REQUIRE(dtip < 0.0, "spm_df_loss_seed: dtip must be <0, got dtip=%g", dtip);
    SPM_REQUIRE(aligned16(FEs) && aligned16(dL_dFEs), "spm_df_loss_seed: FEs/dL_dFEs not 16-byte aligned");
    SPM_REQUIRE((reinterpret_cast<uintptr_t>(scratch) & 7u) == 0, "spm_df_loss_seed: scratch not 8-byte aligned");
    const long long total = (long long)nx * ny * nz;
    const long long nblk = (total + LS_THREADS - 1) / LS_THREADS;
    SPM_REQUIRE(nblk < (1LL << 31), "spm_df_loss_seed: volume too large");
    double* partial = reinterpret_cast<double*>(scratch);
    double* sums = partial + 2 * nblk;
    const double dz = fabs(dtip);
    cudaStream_t st = as_stream(stream);
    if (fes_dtype == SPM_F32)
        loss_partials_kernel<<<(unsigned)nblk, LS_THREADS, 0, st>>>(static_cast<const float*>(FEs), target, weights,
                                                                    nx, ny, nz, 1.0 / (2.0 * dz), df_out, partial);
    else
        loss_partials_kernel<<<(unsigned)nblk, LS_THREADS, 0, st>>>(static_cast<const double*>(FEs), target, weights,
                                                                    nx, ny, nz, 1.0 / (2.0 * dz), df_out, partial);
    loss_final_kernel<<<1, LS_THREADS, 0, st>>>(partial, (int)nblk, sums, loss_out);
    loss_grad_kernel<<<(unsigned)nblk, LS_THREADS, 0, st>>>(df_out, target, weights, sums, nx, ny, nz,
                                                            1.0 / (2.0 * dz), reinterpret_cast<float4*>(dL_dFEs));
    return check_launch("spm_df_loss_seed");
}

// ---------------------------------------------------------------------------
// Batched df and df loss: each molecule's states are its (n_scan,1,nz_steps)
// volume (z-step fastest, the first z-step highest).  Work items find their
// molecule through the descriptor prefixes (pix_off, chunk_off); every
// per-element expression and every reduction order is the single-volume
// kernel's, so each molecule's results are bit-identical to those calls.
// ---------------------------------------------------------------------------
namespace spm {
namespace {

// Warp per stroke.  The stroke is staged lowest z-step first, so the column
// is the ascending volume spm_df_amp_dir expects (dr = |dtip| > 0); results
// are written back in stroke order.
__global__ void __launch_bounds__(DFZ_WARPS * 32)
batch_df_amp_kernel(int n_mol, const spm_batch_mol* __restrict__ mols, long long n_pix,
                    const float* __restrict__ FEs, DfGeom P, float* __restrict__ df) {
    __shared__ double s_fn[DFZ_WARPS][DFZ_MAXNZ];
    __shared__ double s_row[DFZ_WARPS][DFZ_TAB];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const long long pix = (long long)blockIdx.x * DFZ_WARPS + w;
    if (pix >= n_pix) return;  // whole warp exits together: no CTA barrier below
    const spm_batch_mol* D = mols + SPM_MOL_BY(pix_off, mols, n_mol, pix);
    const int nz = D->nz_steps;
    const long long s0 = D->state_off + (pix - D->pix_off) * (long long)nz;
    if (nz < 2 || nz > DFZ_MAXNZ) {  // no central difference (or no room): flag the stroke
        for (int o = l; o < nz; o += 32) df[s0 + o] = __int_as_float(0x7fc00000);
        return;
    }
    double* fn = s_fn[w];
    for (int z = l; z < nz; z += 32) {
        const Row f = load_row(FEs, (size_t)(s0 + (nz - 1 - z)));
        fn[z] = (f.x * P.n[0] + f.y * P.n[1]) + f.z * P.n[2];
    }
    __syncwarp();
    const double sh = P.shift[2], nzc = P.n[2];
    auto S = [&](int j, double u) {
        const double c = (double)j + u * sh;
        const double fl = floor(c);
        const double t = c - fl;
        const int i0 = (int)fl;
        const double w0 = 1.0 - t, w1 = t;
        double acc = 0.0;
        if (w0 != 0.0) acc += fn[clampi(i0, nz)] * w0;
        if (w1 != 0.0) acc += fn[clampi(i0 + 1, nz)] * w1;
        return acc;
    };
    if (nz <= DFZ_TAB) {  // each S(j, u_k) once, as df_amp_z_kernel
        double* row = s_row[w];
        double acc[DFZ_TAB / 32];
#pragma unroll
        for (int m = 0; m < DFZ_TAB / 32; m++) acc[m] = 0.0;
        for (int k = 0; k < NQ; k++) {
            const double u = P.uk[k];
            for (int j = l; j < nz; j += 32) row[j] = S(j, u);
            __syncwarp();
#pragma unroll
            for (int m = 0; m < DFZ_TAB / 32; m++) acc[m] = df_accumulate(acc[m], l + 32 * m, nz, row, P.idr[2], P.idr2[2], P.wk * nzc);
            __syncwarp();  // the row is rewritten for the next node
        }
#pragma unroll
        for (int m = 0; m < DFZ_TAB / 32; m++) {
            const int iz = l + 32 * m;
            if (iz < nz) df[s0 + (nz - 1 - iz)] = (float)acc[m];
        }
        return;
    }
    for (int iz = l; iz < nz; iz += 32) {
        double acc = 0.0;
        for (int k = 0; k < NQ; k++) {
            const double u = P.uk[k];
            double g;
            if (iz == 0) g = (S(1, u) - S(0, u)) * P.idr[2];
            else if (iz == nz - 1) g = (S(nz - 1, u) - S(nz - 2, u)) * P.idr[2];
            else g = (S(iz + 1, u) - S(iz - 1, u)) * P.idr2[2];
            acc -= (P.wk * nzc) * g;
        }
        df[s0 + (nz - 1 - iz)] = (float)acc;
    }
}

// Loss chunks per CTA of the partials and gradient kernels.  The first
// chunk's molecule is found by binary search, the next ones by stepping
// forward from it, so the search's dependent descriptor loads are paid once
// per LS_CHUNKS chunks; every chunk is computed and reduced exactly as alone.
constexpr int LS_CHUNKS = 4;

// The chunk's single-volume tree (v[t] += v[t+s], s = 128 .. 1) of its threads' (w, l):
// levels >= 32 through shared memory, the last five in warp 0 by shuffles -- the same
// additions in the same order.  Ends with a barrier, so s_w / s_l can be reused.
__device__ __forceinline__ void chunk_partials(double w, double l, double* s_w, double* s_l, double* out) {
    s_w[threadIdx.x] = w;
    s_l[threadIdx.x] = l;
    __syncthreads();
    for (int s = LS_THREADS / 2; s >= 32; s >>= 1) {
        if (threadIdx.x < s) {
            s_w[threadIdx.x] += s_w[threadIdx.x + s];
            s_l[threadIdx.x] += s_l[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x < 32) {
        double vw = s_w[threadIdx.x], vl = s_l[threadIdx.x];
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            vw += __shfl_down_sync(0xffffffffu, vw, s);
            vl += __shfl_down_sync(0xffffffffu, vl, s);
        }
        if (threadIdx.x == 0) {
            out[0] = vw;
            out[1] = vl;
        }
    }
    __syncthreads();
}

// LS_CHUNKS consecutive 256-state chunks per CTA: df and each chunk's (w, w*diff^2) sums.
__global__ void __launch_bounds__(LS_THREADS)
batch_loss_partials_kernel(int n_mol, long long n_chunks, const spm_batch_mol* __restrict__ mols,
                           const float* __restrict__ FEs, const double* __restrict__ tgt,
                           const double* __restrict__ wts, double idz2, double* __restrict__ df_out,
                           double* __restrict__ partial) {
    __shared__ double s_w[LS_THREADS], s_l[LS_THREADS];
    const long long c0 = (long long)blockIdx.x * LS_CHUNKS;
    int m = SPM_MOL_BY(chunk_off, mols, n_mol, c0);
    // every state's terms first (independent loads of all chunks in flight), then the reductions
    double wv[LS_CHUNKS], lv[LS_CHUNKS];
#pragma unroll
    for (int k = 0; k < LS_CHUNKS; k++) {
        const long long ch = c0 + k;
        wv[k] = 0.0;
        lv[k] = 0.0;
        if (ch >= n_chunks) continue;
        m = SPM_MOL_STEP(chunk_off, mols, n_mol, m, ch);
        const spm_batch_mol* D = mols + m;
        const int nz = D->nz_steps;
        const long long nst = (long long)D->n_scan * nz;
        const long long ls = (ch - D->chunk_off) * LS_THREADS + threadIdx.x;
        if (ls < nst) {
            const long long gid = D->state_off + ls;
            const int iz = ls < (1LL << 32) ? (int)((unsigned)ls % (unsigned)nz) : (int)(ls % nz);  // 32-bit when it fits
            double d = 0.0;
            if (iz > 0 && iz < nz - 1) {
                const double fp = load_row(FEs, gid + 1).z, fm = load_row(FEs, gid - 1).z;
                d = -(fp - fm) * idz2;
            }
            df_out[gid] = d;
            wv[k] = wts ? wts[gid] : ((iz > 0 && iz < nz - 1) ? 1.0 : 0.0);
            const double diff = d - tgt[gid];
            lv[k] = wv[k] * (diff * diff);
        }
    }
#pragma unroll
    for (int k = 0; k < LS_CHUNKS; k++)
        if (c0 + k < n_chunks) chunk_partials(wv[k], lv[k], s_w, s_l, partial + 2 * (c0 + k));  // uniform over the CTA
}

// CTA per molecule: fold its chunk partials in the fixed single-volume order.
__global__ void __launch_bounds__(LS_THREADS)
batch_loss_final_kernel(const spm_batch_mol* __restrict__ mols, const double* __restrict__ partial,
                        double* __restrict__ sums, double* __restrict__ loss) {
    __shared__ double s_w[LS_THREADS], s_l[LS_THREADS];
    const int m = blockIdx.x;
    const spm_batch_mol* D = mols + m;
    const long long nst = (long long)D->n_scan * D->nz_steps;
    const long long nblk = (nst + LS_THREADS - 1) / LS_THREADS;
    const double* pm = partial + 2 * D->chunk_off;
    double w = 0.0, l = 0.0;
    for (long long i = threadIdx.x; i < nblk; i += LS_THREADS) {
        w += pm[2 * i];
        l += pm[2 * i + 1];
    }
    s_w[threadIdx.x] = w;
    s_l[threadIdx.x] = l;
    __syncthreads();
    for (int s = LS_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            s_w[threadIdx.x] += s_w[threadIdx.x + s];
            s_l[threadIdx.x] += s_l[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        sums[2 * m] = s_w[0];
        sums[2 * m + 1] = s_l[0];
        // zero total weight (no pixels, or every state masked): the molecule contributes nothing,
        // where the single-volume formula would give 0/0
        loss[m] = s_w[0] > 0.0 ? 0.5 * s_l[0] / s_w[0] : 0.0;
    }
}

__global__ void __launch_bounds__(LS_THREADS)
batch_loss_grad_kernel(int n_mol, long long n_chunks, const spm_batch_mol* __restrict__ mols,
                       const double* __restrict__ df, const double* __restrict__ tgt, const double* __restrict__ wts,
                       const double* __restrict__ sums, double coeff, float4* __restrict__ dL) {
    const long long c0 = (long long)blockIdx.x * LS_CHUNKS;
    int m = SPM_MOL_BY(chunk_off, mols, n_mol, c0);
#pragma unroll
    for (int k = 0; k < LS_CHUNKS; k++) {
        const long long ch = c0 + k;
        if (ch >= n_chunks) return;
        m = SPM_MOL_STEP(chunk_off, mols, n_mol, m, ch);
        const spm_batch_mol* D = mols + m;
        const int nz = D->nz_steps;
        const long long nst = (long long)D->n_scan * nz;
        const long long ls = (ch - D->chunk_off) * LS_THREADS + threadIdx.x;
        if (ls >= nst) continue;
        const long long gid = D->state_off + ls;
        const int iz = ls < (1LL << 32) ? (int)((unsigned)ls % (unsigned)nz) : (int)(ls % nz);  // 32-bit when it fits
        const double wsum = sums[2 * m];
        // no central difference (nz < 3: the stencil would leave the stroke) or zero total
        // weight (no loss): no gradient
        if (nz < 3 || !(wsum > 0.0)) {
            dL[gid] = make_float4(0.f, 0.f, 0.f, 0.f);
            continue;
        }
        const double iwsum = 1.0 / wsum;  // one division per thread, uniform over the molecule's chunk
        auto g = [&](long long j, int jz) {  // jz: the z-step of state j
            const double w = wts ? wts[j] : ((jz > 0 && jz < nz - 1) ? 1.0 : 0.0);
            return w * (df[j] - tgt[j]) * iwsum;
        };
        double v;
        if (iz == 0) v = g(gid + 1, 1) * coeff;
        else if (iz == nz - 1) v = -g(gid - 1, iz - 1) * coeff;
        else v = (g(gid + 1, iz + 1) - g(gid - 1, iz - 1)) * coeff;
        dL[gid] = make_float4(0.f, 0.f, (float)v, 0.f);
    }
}

}  // namespace
}  // namespace spm

extern "C" int spm_batch_df_amp(int n_mol, const spm_batch_mol* mols, long long n_pixels, const float* FEs,
                                double dtip, double amp, float* df, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(n_mol >= 0 && n_pixels >= 0, "spm_batch_df_amp: negative sizes");
    if (n_mol == 0 || n_pixels == 0) return SPM_OK;
    SPM_REQUIRE(mols && FEs && df, "spm_batch_df_amp: null pointer");
    SPM_REQUIRE(aligned16(FEs), "spm_batch_df_amp: FEs not 16-byte aligned");
    SPM_REQUIRE(std::isfinite(dtip) && dtip != 0.0 && std::isfinite(amp), "spm_batch_df_amp: dtip=%g amp=%g", dtip, amp);
    const double n[3] = {0.0, 0.0, 1.0}, dr[3] = {1.0, 1.0, fabs(dtip)};
    DfGeom P;
    int rc = fill_geom(P, 1, 1, 2, n, dr, amp);
    if (rc) return rc;
    const long long nb = (n_pixels + DFZ_WARPS - 1) / DFZ_WARPS;
    SPM_REQUIRE(nb < (1LL << 31), "spm_batch_df_amp: too many pixels");
    batch_df_amp_kernel<<<(unsigned)nb, DFZ_WARPS * 32, 0, as_stream(stream)>>>(n_mol, mols, n_pixels, FEs, P, df);
    return check_launch("spm_batch_df_amp");
}

extern "C" long long spm_batch_loss_scratch_bytes(long long n_chunks, int n_mol) {
    if (n_chunks < 0 || n_mol < 0) return 0;
    return (2 * n_chunks + 2 * (long long)n_mol) * (long long)sizeof(double);
}

namespace spm {
namespace {
// weights[s] = w_base[s] * (status[s-1] == 0 && status[s] == 0 && status[s+1] == 0), neighbours
// taken cyclically over the whole state array, status = diag[.].w.
__global__ void __launch_bounds__(256)
failure_mask_kernel(long long n, const float4* __restrict__ diag, const double* __restrict__ w_base,
                    double* __restrict__ weights) {
    const long long s = (long long)blockIdx.x * 256 + threadIdx.x;
    if (s >= n) return;
    const long long sm = s > 0 ? s - 1 : n - 1, sp = s + 1 < n ? s + 1 : 0;
    const bool ok = diag[s].w == 0.f && diag[sm].w == 0.f && diag[sp].w == 0.f;
    weights[s] = w_base[s] * (ok ? 1.0 : 0.0);
}
}  // namespace
}  // namespace spm

extern "C" int spm_batch_failure_mask(long long n_states, const float* diag, const double* w_base, double* weights,
                                      void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(n_states >= 0, "spm_batch_failure_mask: n_states=%lld", n_states);
    if (n_states == 0) return SPM_OK;
    SPM_REQUIRE(diag && w_base && weights && aligned16(diag), "spm_batch_failure_mask: null or misaligned buffers");
    const long long nb = (n_states + 255) / 256;
    SPM_REQUIRE(nb < (1LL << 31), "spm_batch_failure_mask: too many states");
    failure_mask_kernel<<<(unsigned)nb, 256, 0, as_stream(stream)>>>(n_states, reinterpret_cast<const float4*>(diag),
                                                                     w_base, weights);
    return check_launch("spm_batch_failure_mask");
}

extern "C" int spm_batch_df_loss_seed(int n_mol, const spm_batch_mol* mols, long long n_chunks, const float* FEs,
                                      const double* target, const double* weights, double dtip, double* df_out,
                                      float* dL_dFEs, double* loss_out, void* scratch, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(n_mol >= 0 && n_chunks >= 0, "spm_batch_df_loss_seed: negative sizes");
    if (n_mol == 0) return SPM_OK;
    SPM_REQUIRE(mols && loss_out && scratch, "spm_batch_df_loss_seed: null pointer");
    SPM_REQUIRE(dtip < 0.0, "spm_batch_df_loss_seed: dtip must be <0, got dtip=%g", dtip);
    SPM_REQUIRE(n_chunks < (1LL << 31), "spm_batch_df_loss_seed: too many states");
    SPM_REQUIRE((reinterpret_cast<uintptr_t>(scratch) & 7u) == 0, "spm_batch_df_loss_seed: scratch not 8-byte aligned");
    if (n_chunks > 0)
        SPM_REQUIRE(FEs && target && df_out && dL_dFEs && aligned16(FEs) && aligned16(dL_dFEs),
                    "spm_batch_df_loss_seed: null or misaligned state buffers");
    double* partial = static_cast<double*>(scratch);
    double* sums = partial + 2 * n_chunks;
    const double dz = fabs(dtip);
    cudaStream_t st = as_stream(stream);
    const unsigned nblk = (unsigned)((n_chunks + LS_CHUNKS - 1) / LS_CHUNKS);
    if (n_chunks > 0)
        batch_loss_partials_kernel<<<nblk, LS_THREADS, 0, st>>>(n_mol, n_chunks, mols, FEs, target, weights,
                                                                1.0 / (2.0 * dz), df_out, partial);
    batch_loss_final_kernel<<<(unsigned)n_mol, LS_THREADS, 0, st>>>(mols, partial, sums, loss_out);
    if (n_chunks > 0)
        batch_loss_grad_kernel<<<nblk, LS_THREADS, 0, st>>>(n_mol, n_chunks, mols, df_out, target, weights, sums,
                                                            1.0 / (2.0 * dz), reinterpret_cast<float4*>(dL_dFEs));
    return check_launch("spm_batch_df_loss_seed");
}

// ---------------------------------------------------------------------------
// Allocation-free df loss seed.
//
// Some callers cannot allocate device memory around this call: code that runs
// inside a host framework whose allocator owns all device memory (and may not
// be re-entered from the loss callback), callers that must never trigger an
// implicit device synchronisation from cudaMalloc/cudaFree in a latency-bound
// fitting loop, or callers that hold device memory budgets fixed up front.
// For them spm_df_loss_seed_noalloc takes no scratch argument: its per-block
// partial sums live in a fixed file-scope device array of
// SPM_DF_LOSS_NOALLOC_MAX_ELEMS / 256 (w, w*diff^2) pairs (1 MiB) that every
// GPU loading this library holds until the process exits.
// ---------------------------------------------------------------------------
#include <mutex>

namespace spm {
namespace {

constexpr long long NOALLOC_MAX_BLOCKS = SPM_DF_LOSS_NOALLOC_MAX_ELEMS / LS_THREADS;
// Shared by every call on a device: partials of block b at [2b, 2b+1], the
// final (wsum, sum) pair after them.  Each call overwrites every slot it later
// reads, so nothing has to be cleared between calls.
static __device__ __align__(256) double g_loss_scratch[2 * NOALLOC_MAX_BLOCKS + 2];

constexpr int MAX_DEVICES = 64;
std::mutex g_scratch_mutex;
double* g_scratch_addr[MAX_DEVICES] = {nullptr};

// Device address of g_loss_scratch on the current device (resolved once per
// device with that device current; the host-side symbol is not a device address).
int loss_scratch_address(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(SPM_ERR_CUDA, "spm_df_loss_seed_noalloc: cudaGetDevice: %s",
                                           cudaGetErrorString(e));
    if (dev < 0 || dev >= MAX_DEVICES)
        return set_error(SPM_ERR_UNSUPPORTED, "spm_df_loss_seed_noalloc: device ordinal %d >= %d", dev, MAX_DEVICES);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (g_scratch_addr[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_loss_scratch);
        if (e != cudaSuccess || p == nullptr)
            return set_error(SPM_ERR_CUDA, "spm_df_loss_seed_noalloc: cudaGetSymbolAddress: %s",
                             cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return SPM_OK;
}

}  // namespace
}  // namespace spm

extern "C" int spm_df_loss_seed_noalloc(const void* FEs, int fes_dtype, const double* target, const double* weights,
                                        int nx, int ny, int nz, double dtip, double* df_out, float* dL_dFEs,
                                        double* loss_out, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(FEs && target && df_out && dL_dFEs && loss_out, "spm_df_loss_seed_noalloc: null pointer");
    SPM_REQUIRE(fes_dtype == SPM_F32 || fes_dtype == SPM_F64, "spm_df_loss_seed_noalloc: fes_dtype=%d", fes_dtype);
    SPM_REQUIRE(nx > 0 && ny > 0, "spm_df_loss_seed_noalloc: nx=%d ny=%d must be positive", nx, ny);
    SPM_REQUIRE(nz >= 3, "spm_df_loss_seed_noalloc: need nz>=3 for central difference, got nz=%d", nz);
    SPM_REQUIRE(dtip < 0.0, "spm_df_loss_seed_noalloc: dtip must be <0, got dtip=%g", dtip);
    SPM_REQUIRE(aligned16(FEs) && aligned16(dL_dFEs), "spm_df_loss_seed_noalloc: FEs/dL_dFEs not 16-byte aligned");
    const long long total = (long long)nx * ny * nz;
    if (total > SPM_DF_LOSS_NOALLOC_MAX_ELEMS)
        return set_error(SPM_ERR_UNSUPPORTED,
                         "spm_df_loss_seed_noalloc: volume of %lld elements exceeds the fixed scratch limit of %lld "
                         "(use spm_df_loss_seed with caller scratch)", total, (long long)SPM_DF_LOSS_NOALLOC_MAX_ELEMS);
    double* partial = nullptr;
    int rc = loss_scratch_address(&partial);
    if (rc) return rc;
    const long long nblk = (total + LS_THREADS - 1) / LS_THREADS;
    double* sums = partial + 2 * nblk;
    const double dz = fabs(dtip);
    cudaStream_t st = as_stream(stream);
    if (fes_dtype == SPM_F32)
        loss_partials_kernel<<<(unsigned)nblk, LS_THREADS, 0, st>>>(static_cast<const float*>(FEs), target, weights,
                                                                    nx, ny, nz, 1.0 / (2.0 * dz), df_out, partial);
    else
        loss_partials_kernel<<<(unsigned)nblk, LS_THREADS, 0, st>>>(static_cast<const double*>(FEs), target, weights,
                                                                    nx, ny, nz, 1.0 / (2.0 * dz), df_out, partial);
    loss_final_kernel<<<1, LS_THREADS, 0, st>>>(partial, (int)nblk, sums, loss_out);
    loss_grad_kernel<<<(unsigned)nblk, LS_THREADS, 0, st>>>(df_out, target, weights, sums, nx, ny, nz,
                                                            1.0 / (2.0 * dz), reinterpret_cast<float4*>(dL_dFEs));
    return check_launch("spm_df_loss_seed_noalloc");
}
