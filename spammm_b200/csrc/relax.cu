// relax.cu -- stage (b): probe-particle relaxation on the force grid.
//
// Replaces relaxStrokes (SPAMMM kernels/AFM.cl:345-394, launched by
// AFMulator.scan_fdbm, spammm/SPM/AFM.py:607-617), relaxStrokesTilted
// (AFM.cl:478-562, AFMulator.run_scan, AFM.py:995-1004) and the raw sampler
// getFEinStrokesTilted (AFM.cl:210-233, AFMulator.get_raw_FE, AFM.py:2565-2574).
//
// The reference launches one work-item per work-group (local size 1).  Here a
// CTA of 128 threads covers an 8 (ix) x 16 (iy) pixel block and each warp a
// compact 4 x 8 block, so the eight texel rows a warp reads per step overlap in
// L1.  The stroke state (pos, v, dt, damp, tipPos) lives in registers.  Each
// lane runs its own (z-step, iteration) sequence as one flattened loop: a lane
// that converges moves straight on to its next z-step instead of waiting for
// the slowest lane of the warp, so a warp costs max over lanes of the TOTAL
// iterations rather than the sum over z of per-step maxima.  Per-pixel
// arithmetic is exactly the reference's sequence (see spm_fire.cuh), so the
// flattening changes no result bit.
//
// This translation unit is compiled with -fmad=false: the only fused
// multiply-adds are the explicit __fmaf_rn calls shared with the CPU oracle.
#include "spm_internal.cuh"
#include "spm_fire.cuh"

namespace spm {
namespace {

constexpr int RX_THREADS = 128;

// Pixel owned by this thread (ix-major raster index k) or -1.
__device__ __forceinline__ int pixel_of_thread(int n_scan, int raster_ny) {
    if (raster_ny > 0) {
        const int nxr = n_scan / raster_ny;
        const int nby = (raster_ny + 15) / 16;
        const int bx = blockIdx.x / nby, by = blockIdx.x % nby;
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        const int ix = bx * 8 + (w >> 1) * 4 + (l >> 3);
        const int iy = by * 16 + (w & 1) * 8 + (l & 7);
        if (ix >= nxr || iy >= raster_ny) return -1;
        return ix * raster_ny + iy;
    }
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    return k < n_scan ? k : -1;
}

__device__ __forceinline__ float4 ld4(const float* a) { return make_float4(a[0], a[1], a[2], a[3]); }

// MODE 0: relaxStrokes; MODE 1: relaxStrokesTilted.
template <int MODE>
__global__ void __launch_bounds__(RX_THREADS)
relax_kernel(GridView G, const float4* __restrict__ pts, int n_scan, spm_scan_params P,
             float4* __restrict__ FEs, float4* __restrict__ disps, int* __restrict__ iter_count) {
    const int k = pixel_of_thread(n_scan, P.raster_ny);
    if (k < 0) return;
    const bool fire = (P.flags & SPM_FLAG_FIRE) != 0;
    const bool flip = (P.flags & SPM_FLAG_FLIP_Z) != 0;
    const int nzs = P.nz;
    const float4 kk = ld4(P.stiffness), d0 = ld4(P.dpos0);
    const float4 tc = ld4(P.tipC);
    const V3 a = mk3(P.tipA[0], P.tipA[1], P.tipA[2]);
    const V3 b = mk3(P.tipB[0], P.tipB[1], P.tipB[2]);
    const V3 c = mk3(tc.x, tc.y, tc.z);
    const float surf = P.surfFF[0];

    const float4 p4 = pts[k];
    V3 tip = mk3(p4.x, p4.y, p4.z);
    V3 pos, dTip;
    if (MODE == 0) {
        pos = mk3(tip.x + d0.x, tip.y + d0.y, tip.z + d0.z);
        dTip = mk3(P.dTip[0], P.dTip[1], P.dTip[2]);
    } else {
        pos = add3(tip, rotmatT(mk3(d0.x, d0.y, d0.z), a, b, c));
        dTip = mk3(__fmul_rn(c.x, tc.w), __fmul_rn(c.y, tc.w), __fmul_rn(c.z, tc.w));
    }
    Integrator I;
    I.dt = P.relax_params[0];
    I.damp = P.relax_params[1];
    I.dtmax = I.dt;
    I.dtmin = __fmul_rn(I.dtmax, 0.1f);
    I.damp0 = I.damp;

    float4* fe_out = FEs + (size_t)k * nzs;
    float4* dp_out = (MODE == 0) ? disps + (size_t)k * nzs : nullptr;
    V3 v = mk3(0.f, 0.f, 0.f);
    float4 fe = make_float4(0.f, 0.f, 0.f, 0.f);
    int iz = 0, it = 0, total_it = 0;
    const int max_iter = P.max_iter;
    while (iz < nzs) {
        bool done = max_iter <= 0;
        if (!done) {
            fe = interp_fe(G, pos);
            V3 f;
            if (MODE == 0) {
                V3 ft = tip_force(sub3(pos, tip), kk, d0);
                f = mk3(fe.x + ft.x, fe.y + ft.y, fe.z + ft.z);
            } else {
                V3 ft = rotmatT(tip_force(rotmat(sub3(pos, tip), a, b, c), kk, d0), a, b, c);
                f = mk3(fe.x + ft.x, fe.y + ft.y, fe.z + ft.z);
                f.x = __fmaf_rn(c.x, surf, f.x);
                f.y = __fmaf_rn(c.y, surf, f.y);
                f.z = __fmaf_rn(c.z, surf, f.z);
            }
            md_step(f, v, pos, I, fire);
            ++it;
            ++total_it;
            done = (dot3(f, f) < P.f2conv) || (it >= max_iter);
        }
        if (done) {
            const int oz = flip ? (nzs - 1 - iz) : iz;
            if (MODE == 0) {
                fe_out[oz] = fe;
                const V3 ref = mk3(tip.x + d0.x, tip.y + d0.y, tip.z + d0.z);
                dp_out[oz] = make_float4(pos.x - ref.x, pos.y - ref.y, pos.z - ref.z, 0.f);
            } else {
                const float4 g = interp_fe(G, pos);
                const V3 r = rotmat(mk3(g.x, g.y, g.z), a, b, c);
                fe_out[oz] = make_float4(r.x, r.y, r.z, g.w);
            }
            tip = add3(tip, dTip);
            pos = add3(pos, dTip);
            v = mk3(0.f, 0.f, 0.f);
            fe = make_float4(0.f, 0.f, 0.f, 0.f);
            it = 0;
            ++iz;
        }
    }
    if (iter_count) iter_count[k] = total_it;
}

__global__ void __launch_bounds__(RX_THREADS)
raw_kernel(GridView G, const float4* __restrict__ pts, int n_scan, spm_scan_params P, float4* __restrict__ FEs) {
    const int k = pixel_of_thread(n_scan, P.raster_ny);
    if (k < 0) return;
    const V3 a = mk3(P.tipA[0], P.tipA[1], P.tipA[2]);
    const V3 b = mk3(P.tipB[0], P.tipB[1], P.tipB[2]);
    const V3 c = mk3(P.tipC[0], P.tipC[1], P.tipC[2]);
    const float4 p4 = pts[k];
    V3 pos = mk3(p4.x + P.dpos0[0], p4.y + P.dpos0[1], p4.z + P.dpos0[2]);
    const V3 dTip = mk3(P.dTip[0], P.dTip[1], P.dTip[2]);
    const bool flip = (P.flags & SPM_FLAG_FLIP_Z) != 0;
    float4* out = FEs + (size_t)k * P.nz;
    for (int iz = 0; iz < P.nz; iz++) {
        const float4 g = interp_fe(G, pos);
        const V3 r = rotmat(mk3(g.x, g.y, g.z), a, b, c);
        out[flip ? (P.nz - 1 - iz) : iz] = make_float4(r.x, r.y, r.z, g.w);
        pos = add3(pos, dTip);
    }
}

int check_scan_args(const char* who, const float* grid, int nx, int ny, int nz, const float* points, int n_scan,
                    const spm_scan_params* p, const float* out0) {
    SPM_REQUIRE(p != nullptr, "%s: null params", who);
    SPM_REQUIRE(nx > 0 && ny > 0 && nz > 0, "%s: grid dims (%d,%d,%d) must be positive", who, nx, ny, nz);
    SPM_REQUIRE(n_scan >= 0, "%s: n_scan=%d < 0", who, n_scan);
    SPM_REQUIRE(p->nz >= 0, "%s: nz=%d < 0", who, p->nz);
    SPM_REQUIRE(grid != nullptr, "%s: null grid", who);
    if (n_scan > 0 && p->nz > 0)  // empty scans may pass null point/output buffers
        SPM_REQUIRE(points && out0, "%s: null points/output pointer", who);
    SPM_REQUIRE(aligned16(grid) && aligned16(points) && aligned16(out0), "%s: buffers must be 16-byte aligned", who);
    long long t = 0;
    SPM_REQUIRE(mul_ok((long long)nx * ny, nz, &t), "%s: grid size overflows", who);
    SPM_REQUIRE(mul_ok(n_scan, (long long)p->nz * 4, &t), "%s: output size overflows", who);
    SPM_REQUIRE(p->raster_ny >= 0, "%s: raster_ny=%d < 0", who, p->raster_ny);
    SPM_REQUIRE((p->flags & ~(SPM_FLAG_FIRE | SPM_FLAG_FLIP_Z)) == 0, "%s: unknown flags 0x%x", who, p->flags);
    return SPM_OK;
}

GridView make_view(const float* grid, int nx, int ny, int nz, const spm_scan_params* p) {
    GridView G;
    G.g = reinterpret_cast<const float4*>(grid);
    G.nx = nx; G.ny = ny; G.nz = nz;
    G.dA = make_float4(p->dinvA[0], p->dinvA[1], p->dinvA[2], p->dinvA[3]);
    G.dB = make_float4(p->dinvB[0], p->dinvB[1], p->dinvB[2], p->dinvB[3]);
    G.dC = make_float4(p->dinvC[0], p->dinvC[1], p->dinvC[2], p->dinvC[3]);
    return G;
}

int blocks_for(int n_scan, const spm_scan_params& P) {
    if (P.raster_ny > 0) {
        const int nxr = n_scan / P.raster_ny;
        return ((nxr + 7) / 8) * ((P.raster_ny + 15) / 16);
    }
    return (n_scan + RX_THREADS - 1) / RX_THREADS;
}

spm_scan_params normalized(const spm_scan_params* p, int n_scan) {
    spm_scan_params P = *p;
    if (P.raster_ny > 0 && (n_scan % P.raster_ny) != 0) P.raster_ny = 0;  // not a full raster: 1D map
    return P;
}

}  // namespace
}  // namespace spm

extern "C" int spm_relax_strokes(const float* grid, int nx, int ny, int nz, const float* points, int n_scan,
                                 const spm_scan_params* p, float* FEs, float* disps, void* stream) {
    return spm_relax_strokes_counted(grid, nx, ny, nz, points, n_scan, p, FEs, disps, nullptr, stream);
}

extern "C" int spm_relax_strokes_counted(const float* grid, int nx, int ny, int nz, const float* points, int n_scan,
                                         const spm_scan_params* p, float* FEs, float* disps, int* iter_count,
                                         void* stream) {
    using namespace spm;
    clear_error();
    int rc = check_scan_args("spm_relax_strokes", grid, nx, ny, nz, points, n_scan, p, FEs);
    if (rc) return rc;
    if (n_scan == 0 || p->nz == 0) return SPM_OK;
    SPM_REQUIRE(disps != nullptr && aligned16(disps), "spm_relax_strokes: disps null or misaligned");
    spm_scan_params P = normalized(p, n_scan);
    relax_kernel<0><<<blocks_for(n_scan, P), RX_THREADS, 0, as_stream(stream)>>>(
        make_view(grid, nx, ny, nz, p), reinterpret_cast<const float4*>(points), n_scan, P,
        reinterpret_cast<float4*>(FEs), reinterpret_cast<float4*>(disps), iter_count);
    return check_launch("spm_relax_strokes");
}

extern "C" int spm_relax_strokes_tilted(const float* grid, int nx, int ny, int nz, const float* points, int n_scan,
                                        const spm_scan_params* p, float* FEs, void* stream) {
    using namespace spm;
    clear_error();
    int rc = check_scan_args("spm_relax_strokes_tilted", grid, nx, ny, nz, points, n_scan, p, FEs);
    if (rc) return rc;
    if (n_scan == 0 || p->nz == 0) return SPM_OK;
    spm_scan_params P = normalized(p, n_scan);
    relax_kernel<1><<<blocks_for(n_scan, P), RX_THREADS, 0, as_stream(stream)>>>(
        make_view(grid, nx, ny, nz, p), reinterpret_cast<const float4*>(points), n_scan, P,
        reinterpret_cast<float4*>(FEs), nullptr, nullptr);
    return check_launch("spm_relax_strokes_tilted");
}

extern "C" int spm_fe_in_strokes_tilted(const float* grid, int nx, int ny, int nz, const float* points, int n_scan,
                                        const spm_scan_params* p, float* FEs, void* stream) {
    using namespace spm;
    clear_error();
    int rc = check_scan_args("spm_fe_in_strokes_tilted", grid, nx, ny, nz, points, n_scan, p, FEs);
    if (rc) return rc;
    if (n_scan == 0 || p->nz == 0) return SPM_OK;
    spm_scan_params P = normalized(p, n_scan);
    raw_kernel<<<blocks_for(n_scan, P), RX_THREADS, 0, as_stream(stream)>>>(
        make_view(grid, nx, ny, nz, p), reinterpret_cast<const float4*>(points), n_scan, P,
        reinterpret_cast<float4*>(FEs));
    return check_launch("spm_fe_in_strokes_tilted");
}
