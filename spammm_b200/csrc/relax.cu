// relax.cu -- stage (b): probe-particle relaxation on the force grid.
//
// Replaces relaxStrokes (SPAMMM kernels/AFM.cl:345-394, launched by
// AFMulator.scan_fdbm, spammm/SPM/AFM.py:607-617), relaxStrokesTilted
// (AFM.cl:478-562, AFMulator.run_scan, AFM.py:995-1004), relaxStrokes2D
// (AFM.cl:410-450, AFMulator.scan_fdbm_2d, AFM.py:644-704) and the raw sampler
// getFEinStrokesTilted (AFM.cl:210-233, AFMulator.get_raw_FE, AFM.py:2565-2574).
//
// The reference launches one work-item per work-group (local size 1).  Here
// every lane relaxes whole strokes with the stroke state (pos, v, dt, damp,
// tipPos) and the eight texels of its current cell in registers:
//   * with a device-side pixel counter (the workspace of spm_relax_ex), a
//     persistent warp draws a 4 (ix) x 8 (iy) pixel tile at a time and its
//     lanes step down the z-steps together (relax_tile_kernel), so the texel
//     rows they read overlap in L1 and they run the sampling, FIRE and
//     per-z-step code as one (the flattened per-lane loop below, where lanes
//     drift to their own pixel, z-step and phase, kept 49% of the lanes of a
//     warp busy on the 480x480-pixel scan and took 1.65x as long);
//   * without one, relax_kernel's flattened (pixel, z-step, integrator step)
//     loop runs one pixel per lane; relaxStrokes2D always uses it;
//   * node offsets are 32-bit when the grid has fewer than 2^32 nodes.
// Per-pixel arithmetic is exactly the reference's sequence (spm_fire.cuh), so
// neither the scheduling nor the flattening changes a result bit.
//
// This translation unit is compiled with -fmad=false: the only fused
// multiply-adds are the explicit __fmaf_rn calls shared with the CPU oracle.
#include <climits>
#include "spm_internal.cuh"
#include "spm_fire.cuh"
#include "spm_batch.cuh"
#include "spm_diss.cuh"

namespace spm {
namespace {

constexpr int RX_THREADS = 128;

// Pixel of this thread under the static schedule (one pixel per lane), or -1.
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

// Next pixel from the device counter (dynamic schedule), or -1 when drained.
// Counter slot t maps to tile t/32 (4x8 pixels, tiles ordered iy-fastest).
__device__ __forceinline__ int next_pixel(unsigned* counter, int n_scan, int raster_ny) {
    const unsigned lane = threadIdx.x & 31u;
    const int ny = raster_ny;
    const int nxr = ny > 0 ? n_scan / ny : 0;
    const unsigned nty = ny > 0 ? (unsigned)(ny + 7) / 8 : 0u;
    const unsigned nslots = ny > 0 ? ((unsigned)(nxr + 3) / 4) * nty * 32u : (unsigned)n_scan;
    while (true) {
        const unsigned m = __activemask();
        const int leader = __ffs(m) - 1;
        const unsigned rank = __popc(m & ((1u << lane) - 1u));
        unsigned base = 0;
        if ((int)lane == leader) base = atomicAdd(counter, (unsigned)__popc(m));
        base = __shfl_sync(m, base, leader);
        const unsigned t = base + rank;
        if (t >= nslots) return -1;
        if (ny <= 0) return (int)t;
        const unsigned tile = t >> 5, r = t & 31u;
        const int ix = (int)((tile / nty) * 4 + (r >> 3));
        const int iy = (int)((tile % nty) * 8 + (r & 7));
        if (ix < nxr && iy < ny) return ix * ny + iy;
        // an edge tile's slot outside the raster: draw again (t only grows: bounded)
    }
}

__device__ __forceinline__ float4 ld4(const float* a) { return make_float4(a[0], a[1], a[2], a[3]); }

// Probe frame, spring and integrator settings of an SPM_RELAX_PP scan.
struct PPFrame {
    V3 a, b, c, dTip, d0r;
    float4 kk, d0;
    float surf, f2conv;
    int max_iter;
    bool fire;
};

__device__ __forceinline__ PPFrame pp_frame(const spm_scan_params& P) {
    PPFrame F;
    const float4 tc = ld4(P.tipC);
    F.a = mk3(P.tipA[0], P.tipA[1], P.tipA[2]);
    F.b = mk3(P.tipB[0], P.tipB[1], P.tipB[2]);
    F.c = mk3(tc.x, tc.y, tc.z);
    F.kk = ld4(P.stiffness);
    F.d0 = ld4(P.dpos0);
    F.surf = P.surfFF[0];
    F.f2conv = P.f2conv;
    F.max_iter = P.max_iter;
    F.fire = (P.flags & SPM_FLAG_FIRE) != 0;
    F.dTip = mk3(__fmul_rn(F.c.x, tc.w), __fmul_rn(F.c.y, tc.w), __fmul_rn(F.c.z, tc.w));
    F.d0r = rotmatT(mk3(F.d0.x, F.d0.y, F.d0.z), F.a, F.b, F.c);
    return F;
}

__device__ __forceinline__ PolishSpring pp_spring(const PPFrame& F) {
    PolishSpring S;
    S.a = F.a; S.b = F.b; S.c = F.c;
    S.kk = F.kk; S.d0 = F.d0;
    S.surf = F.surf;
    S.frame = true;
    return S;
}

// The polished output of a relaxStrokes (MODE 0: plain spring) or relaxStrokesTilted (MODE 1:
// tip frame) z-step: q and fe in, the polished position and the sample there out.
template <int MODE, typename IDX>
__device__ __forceinline__ void polish_state(const GridView& G, V3 a, V3 b, V3 c, float4 kk, float4 d0, float surf,
                                             V3 tip, V3& q, float4& fe) {
    PolishSpring S;
    S.a = a; S.b = b; S.c = c;
    S.kk = kk; S.d0 = d0;
    S.surf = surf;
    S.frame = MODE != 0;
    float T[3][3];
    polish_coefs(G, T);
    newton_polish(FullCellFetch<IDX>{G}, T, S, tip, q, fe);
}

// One SPM_RELAX_PP iteration (the direct path's bookkeeping: the convergence
// test comes before the update).  Returns true when the z-step is finished;
// conv tells whether it converged.  CACHE: sample through the texel cache T
// (fnx, fny, fnz the dimensions as floats).
template <typename IDX, bool CACHE>
__device__ __forceinline__ bool pp_iter(const GridView& G, const PPFrame& F, V3 tip, V3& pos, V3& v, Integrator& I,
                                        float4& fe, int& it, int& total_it, bool& conv, TexelCache& T, float fnx,
                                        float fny, float fnz) {
    conv = false;
    if (it >= F.max_iter) return true;
    ++it;
    ++total_it;
    if constexpr (CACHE) fe = interp_fe_cached_full<IDX>(G, fnx, fny, fnz, pos, T);
    else fe = interp_fe<IDX>(G, pos);
    const V3 ft = rotmatT(tip_force(rotmat(sub3(pos, tip), F.a, F.b, F.c), F.kk, F.d0), F.a, F.b, F.c);
    V3 f = mk3(fe.x + ft.x, fe.y + ft.y, fe.z + ft.z);
    f.x = __fmaf_rn(F.c.x, F.surf, f.x);
    f.y = __fmaf_rn(F.c.y, F.surf, f.y);
    f.z = __fmaf_rn(F.c.z, F.surf, f.z);
    if (dot3(f, f) < F.f2conv) {
        conv = true;
        return true;
    }
    md_step(f, v, pos, I, F.fire);
    return it >= F.max_iter;
}

// Outputs of a finished SPM_RELAX_PP z-step: tip-frame FE at the final
// position and PP = (pos, +iterations if converged and finite, else -iterations).
// POLISH: the state is Newton-polished first (newton_polish); FE is then the sample at the
// polished position, which PP reports.
template <typename IDX, bool POLISH>
__device__ __forceinline__ void pp_emit(const GridView& G, const PPFrame& F, V3 tip, V3 pos, float4 fe, int it,
                                        bool conv, float4* fe_out, float4* pp_out) {
    if (!conv) fe = interp_fe<IDX>(G, pos);  // the position moved after the last sample
    if constexpr (POLISH) {
        float T[3][3];
        polish_coefs(G, T);
        newton_polish(FullCellFetch<IDX>{G}, T, pp_spring(F), tip, pos, fe);
    }
    const V3 r = rotmat(mk3(fe.x, fe.y, fe.z), F.a, F.b, F.c);
    *fe_out = make_float4(r.x, r.y, r.z, fe.w);
    const bool finite = isfinite(fe.x) && isfinite(fe.y) && isfinite(fe.z) && isfinite(fe.w) && isfinite(pos.x) &&
                        isfinite(pos.y) && isfinite(pos.z);
    *pp_out = make_float4(pos.x, pos.y, pos.z, (float)((conv && finite) ? it : -it));
}

// MODE 0: relaxStrokes; MODE 1: relaxStrokesTilted; MODE 2: PP (differentiable
// path); MODE 3: relaxStrokes2D.
// CACHE (MODE 0-2): the FIRE loop samples through a register TexelCache (the
// cell's eight texels reloaded only when the cell changes; same values; all
// strokes share the grid, so a lane keeps its cache from pixel to pixel).
template <int MODE, typename IDX, bool CACHE, bool POLISH>
__global__ void __launch_bounds__(RX_THREADS)
relax_kernel(GridView G, const float4* __restrict__ pts, int n_scan, spm_scan_params P,
             float4* __restrict__ FEs, float4* __restrict__ disps, int* __restrict__ iter_count,
             unsigned* __restrict__ counter) {
    const float fnx = (float)G.nx, fny = (float)G.ny, fnz = (float)G.nz;
    TexelCache T;
    T.kx = __int_as_float(0x7fc00000);  // NaN matches no cell
    const bool fire = (P.flags & SPM_FLAG_FIRE) != 0;
    const bool flip = (P.flags & SPM_FLAG_FLIP_Z) != 0;
    const int nzs = P.nz;
    const int max_iter = P.max_iter;
    const float4 kk = ld4(P.stiffness), d0 = ld4(P.dpos0);
    const float4 tc = ld4(P.tipC);
    const V3 a = mk3(P.tipA[0], P.tipA[1], P.tipA[2]);
    const V3 b = mk3(P.tipB[0], P.tipB[1], P.tipB[2]);
    const V3 c = mk3(tc.x, tc.y, tc.z);
    const float surf = P.surfFF[0];
    const V3 dTip = (MODE == 0) ? mk3(P.dTip[0], P.dTip[1], P.dTip[2])
                                : mk3(__fmul_rn(c.x, tc.w), __fmul_rn(c.y, tc.w), __fmul_rn(c.z, tc.w));
    const V3 d0r = (MODE == 0) ? mk3(d0.x, d0.y, d0.z) : rotmatT(mk3(d0.x, d0.y, d0.z), a, b, c);
    const float dh2 = -P.dTip[2];                  // MODE 3: descent per slice (dTip.z = -dh)
    const float cv2 = 1.f - P.relax_params[1];     // MODE 3: velocity retention 1 - damp

    // SPM_FLAG_PAIRED (MODE 0): strokes of the second half go backward
    const int half = (MODE == 0 && (P.flags & SPM_FLAG_PAIRED)) ? n_scan / 2 : n_scan;

    int k = counter ? next_pixel(counter, n_scan, P.raster_ny) : pixel_of_thread(n_scan, P.raster_ny);
    V3 tip, pos, v;
    V3 dTipS = dTip;  // this stroke's step and z order
    bool flipS = flip;
    Integrator I;
    float4 fe;
    int iz = 0, it = 0, total_it = 0;
    auto start = [&](int kp) {
        const float4 p4 = pts[kp];
        const bool bwd = kp >= half;
        dTipS = bwd ? mk3(-dTip.x, -dTip.y, -dTip.z) : dTip;
        flipS = flip != bwd;
        tip = mk3(p4.x, p4.y, p4.z);
        pos = (MODE == 0) ? mk3(tip.x + d0r.x, tip.y + d0r.y, tip.z + d0r.z) : (MODE == 3 ? tip : add3(tip, d0r));
        I.dt = P.relax_params[0];
        I.damp = P.relax_params[1];
        I.dtmax = I.dt;
        I.dtmin = __fmul_rn(I.dtmax, 0.1f);
        I.damp0 = I.damp;
        v = mk3(0.f, 0.f, 0.f);
        fe = make_float4(0.f, 0.f, 0.f, 0.f);
        iz = 0;
        it = 0;
        total_it = 0;
    };
    if (k >= 0) start(k);
    PPFrame F;
    if (MODE == 2) F = pp_frame(P);
    while (k >= 0) {
        if (MODE == 2) {
            bool conv;
            if (pp_iter<IDX, CACHE>(G, F, tip, pos, v, I, fe, it, total_it, conv, T, fnx, fny, fnz)) {
                const size_t o = (size_t)k * nzs + iz;
                pp_emit<IDX, POLISH>(G, F, tip, pos, fe, it, conv, FEs + o, disps + o);
                tip = add3(tip, dTip);
                pos = add3(pos, dTip);
                v = mk3(0.f, 0.f, 0.f);
                fe = make_float4(0.f, 0.f, 0.f, 0.f);
                it = 0;
                if (++iz == nzs) {
                    if (iter_count) iter_count[k] = total_it;
                    k = counter ? next_pixel(counter, n_scan, P.raster_ny) : -1;
                    if (k >= 0) start(k);
                }
            }
            continue;
        }
        if (MODE == 3) {
            // relaxStrokes2D: z fixed per slice, x,y relaxed by damped MD from the anchor
            const float pz = tip.z - __fmul_rn((float)iz, dh2);
            bool done = max_iter <= 0;
            if (!done) {
                fe = interp_fe<IDX>(G, mk3(pos.x, pos.y, pz));
                const float fx = fe.x - __fmul_rn(kk.x, pos.x - tip.x);
                const float fy = fe.y - __fmul_rn(kk.x, pos.y - tip.y);
                v.x = __fmaf_rn(fx, P.relax_params[0], __fmul_rn(v.x, cv2));
                v.y = __fmaf_rn(fy, P.relax_params[0], __fmul_rn(v.y, cv2));
                pos.x = __fmaf_rn(v.x, P.relax_params[0], pos.x);
                pos.y = __fmaf_rn(v.y, P.relax_params[0], pos.y);
                ++it;
                ++total_it;
                done = (__fmaf_rn(fy, fy, __fmul_rn(fx, fx)) < P.f2conv) || (it >= max_iter);
            }
            if (done) {
                const int oz = flip ? (nzs - 1 - iz) : iz;
                const size_t o = (size_t)k * nzs + oz;
                FEs[o] = interp_fe<IDX>(G, mk3(pos.x, pos.y, pz));
                disps[o] = make_float4(pos.x - tip.x, pos.y - tip.y, 0.f, 0.f);
                pos = tip;
                v = mk3(0.f, 0.f, 0.f);
                it = 0;
                if (++iz == nzs) {
                    if (iter_count) iter_count[k] = total_it;
                    k = counter ? next_pixel(counter, n_scan, P.raster_ny) : -1;
                    if (k >= 0) start(k);
                }
            }
            continue;
        }
        bool done = max_iter <= 0;
        if (!done) {
            if constexpr (CACHE) fe = interp_fe_cached_full<IDX>(G, fnx, fny, fnz, pos, T);
            else fe = interp_fe<IDX>(G, pos);
            V3 f;
            if (MODE == 0) {
                const V3 ft = tip_force(sub3(pos, tip), kk, d0);
                f = mk3(fe.x + ft.x, fe.y + ft.y, fe.z + ft.z);
            } else {
                const V3 ft = rotmatT(tip_force(rotmat(sub3(pos, tip), a, b, c), kk, d0), a, b, c);
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
            const int oz = flipS ? (nzs - 1 - iz) : iz;
            const size_t o = (size_t)k * nzs + oz;
            V3 q = pos;  // the output position (polished or not); the next z-step starts from pos
            if (MODE == 0) {
                float4 fo = fe;
                if constexpr (POLISH) polish_state<MODE, IDX>(G, a, b, c, kk, d0, surf, tip, q, fo);
                FEs[o] = fo;
                const V3 ref = mk3(tip.x + d0.x, tip.y + d0.y, tip.z + d0.z);
                disps[o] = make_float4(q.x - ref.x, q.y - ref.y, q.z - ref.z, 0.f);
            } else {
                float4 g = interp_fe<IDX>(G, pos);
                if constexpr (POLISH) polish_state<MODE, IDX>(G, a, b, c, kk, d0, surf, tip, q, g);
                const V3 r = rotmat(mk3(g.x, g.y, g.z), a, b, c);
                FEs[o] = make_float4(r.x, r.y, r.z, g.w);
            }
            tip = add3(tip, dTipS);
            pos = add3(pos, dTipS);
            v = mk3(0.f, 0.f, 0.f);
            fe = make_float4(0.f, 0.f, 0.f, 0.f);
            it = 0;
            if (++iz == nzs) {
                if (iter_count) iter_count[k] = total_it;
                k = counter ? next_pixel(counter, n_scan, P.raster_ny) : -1;
                if (k >= 0) start(k);
            }
        }
    }
}

// The dissipation integral fused into the paired relaxation (spm_relax_pair_dissipation): the
// strokes of pixel p are p (forward) and p + n_scan/2 (backward); the lane that finishes the
// second of the two (a per-pixel atomic counter decides, no lane waits) integrates E_diss of the
// pixel from both strokes' FEs as spm_dissipation does (spm_diss.cuh: the same bits).
struct DissArgs {
    const double* h;     // abscissae of the stored z order (DEVICE double[nz])
    const int* off;      // per output: idx[off[o]..off[o+1]) (DEVICE int[n_out+1])
    const int* idx;      // height indices (DEVICE)
    float* E;            // (n_scan/2, n_out)
    int* pair;           // per pixel: strokes finished (zeroed by the launch)
    int n_out;
    double n[3];         // oscillation direction (normalised)
};

// MODE 0-2 (relaxStrokes, relaxStrokesTilted, PP) under the z-synchronised
// tile schedule: a warp draws the 32 pixels of one 4 (ix) x 8 (iy) raster tile
// (32 consecutive pixels without a raster) from the device counter, and its
// lanes relax their strokes one z-step at a time, meeting after each (their
// FIRE loops reconverge there anyway).  Against relax_kernel's flattened loop,
// where every lane is at its own pixel, z-step and phase and the warp runs the
// sampling miss path and the per-z-step epilogue for a few lanes at a time
// (49% of the lanes active per instruction on the 480x480-pixel scan), the
// lanes of a warp run that code together: 3.81 -> 2.30 ms on that scan.  The
// per-lane sequence is relax_kernel's (the same iteration, emit and texel
// cache), so the results are the same bits.
template <int MODE, typename IDX, bool POLISH, bool DISS = false>
__global__ void __launch_bounds__(RX_THREADS)
relax_tile_kernel(GridView G, const float4* __restrict__ pts, int n_scan, spm_scan_params P,
                  float4* __restrict__ FEs, float4* __restrict__ disps, int* __restrict__ iter_count,
                  unsigned* __restrict__ counter, DissArgs DA = DissArgs{}) {
    static_assert(!DISS || MODE == 0, "the fused dissipation is for relaxStrokes pairs");
    static_assert(MODE >= 0 && MODE <= 2, "relaxStrokes2D keeps the flattened loop");
    const unsigned lane = threadIdx.x & 31u;
    const float fnx = (float)G.nx, fny = (float)G.ny, fnz = (float)G.nz;
    TexelCache T;
    T.kx = __int_as_float(0x7fc00000);  // NaN matches no cell
    const bool fire = (P.flags & SPM_FLAG_FIRE) != 0;
    const bool flip = (P.flags & SPM_FLAG_FLIP_Z) != 0;
    const int nzs = P.nz, max_iter = P.max_iter;
    const float4 kk = ld4(P.stiffness), d0 = ld4(P.dpos0);
    const float4 tc = ld4(P.tipC);
    const V3 a = mk3(P.tipA[0], P.tipA[1], P.tipA[2]);
    const V3 b = mk3(P.tipB[0], P.tipB[1], P.tipB[2]);
    const V3 c = mk3(tc.x, tc.y, tc.z);
    const float surf = P.surfFF[0];
    const V3 dTip = (MODE == 0) ? mk3(P.dTip[0], P.dTip[1], P.dTip[2])
                                : mk3(__fmul_rn(c.x, tc.w), __fmul_rn(c.y, tc.w), __fmul_rn(c.z, tc.w));
    const V3 d0r = (MODE == 0) ? mk3(d0.x, d0.y, d0.z) : rotmatT(mk3(d0.x, d0.y, d0.z), a, b, c);
    PPFrame F;
    if (MODE == 2) F = pp_frame(P);
    // SPM_FLAG_PAIRED (MODE 0): strokes of the second half go backward
    const int half = (MODE == 0 && (P.flags & SPM_FLAG_PAIRED)) ? n_scan / 2 : n_scan;
    const int ny = P.raster_ny;
    const int nxr = ny > 0 ? n_scan / ny : 0;
    const unsigned nty = ny > 0 ? (unsigned)(ny + 7) / 8 : 0u;
    const unsigned nslots = ny > 0 ? ((unsigned)(nxr + 3) / 4) * nty * 32u : ((unsigned)n_scan + 31u) / 32u * 32u;
    while (true) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(counter, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= nslots) return;  // warp-uniform
        const unsigned t = base + lane;
        int k = -1;
        if (ny > 0) {
            const unsigned tile = t >> 5, r = t & 31u;
            const int ix = (int)((tile / nty) * 4 + (r >> 3));
            const int iy = (int)((tile % nty) * 8 + (r & 7));
            if (ix < nxr && iy < ny) k = ix * ny + iy;
        } else if (t < (unsigned)n_scan) {
            k = (int)t;
        }
        const unsigned members = __ballot_sync(0xffffffffu, k >= 0);
        if (k >= 0) {
            const float4 p4 = pts[k];
            const bool bwd = k >= half;
            const V3 dTipS = bwd ? mk3(-dTip.x, -dTip.y, -dTip.z) : dTip;
            const bool flipS = flip != bwd;
            V3 tip = mk3(p4.x, p4.y, p4.z);
            V3 pos = (MODE == 0) ? mk3(tip.x + d0r.x, tip.y + d0r.y, tip.z + d0r.z) : add3(tip, d0r);
            Integrator I;
            I.dt = P.relax_params[0];
            I.damp = P.relax_params[1];
            I.dtmax = I.dt;
            I.dtmin = __fmul_rn(I.dtmax, 0.1f);
            I.damp0 = I.damp;
            V3 v = mk3(0.f, 0.f, 0.f);
            int total_it = 0;
            for (int iz = 0; iz < nzs; ++iz) {
                float4 fe = make_float4(0.f, 0.f, 0.f, 0.f);
                int it = 0;
                if (MODE == 2) {
                    bool conv;
                    while (!pp_iter<IDX, true>(G, F, tip, pos, v, I, fe, it, total_it, conv, T, fnx, fny, fnz)) {
                    }
                    const size_t o = (size_t)k * nzs + iz;
                    pp_emit<IDX, POLISH>(G, F, tip, pos, fe, it, conv, FEs + o, disps + o);
                } else {
                    bool done = max_iter <= 0;
                    while (!done) {
                        fe = interp_fe_cached_full<IDX>(G, fnx, fny, fnz, pos, T);
                        V3 f;
                        if (MODE == 0) {
                            const V3 ft = tip_force(sub3(pos, tip), kk, d0);
                            f = mk3(fe.x + ft.x, fe.y + ft.y, fe.z + ft.z);
                        } else {
                            const V3 ft = rotmatT(tip_force(rotmat(sub3(pos, tip), a, b, c), kk, d0), a, b, c);
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
                    const int oz = flipS ? (nzs - 1 - iz) : iz;
                    const size_t o = (size_t)k * nzs + oz;
                    V3 q = pos;  // the output position; the next z-step starts from pos
                    if (MODE == 0) {
                        float4 fo = fe;
                        if constexpr (POLISH) polish_state<MODE, IDX>(G, a, b, c, kk, d0, surf, tip, q, fo);
                        FEs[o] = fo;
                        const V3 ref = mk3(tip.x + d0.x, tip.y + d0.y, tip.z + d0.z);
                        disps[o] = make_float4(q.x - ref.x, q.y - ref.y, q.z - ref.z, 0.f);
                    } else {
                        float4 g = interp_fe<IDX>(G, pos);
                        if constexpr (POLISH) polish_state<MODE, IDX>(G, a, b, c, kk, d0, surf, tip, q, g);
                        const V3 r = rotmat(mk3(g.x, g.y, g.z), a, b, c);
                        FEs[o] = make_float4(r.x, r.y, r.z, g.w);
                    }
                }
                tip = add3(tip, dTipS);
                pos = add3(pos, dTipS);
                v = mk3(0.f, 0.f, 0.f);
                __syncwarp(members);  // the tile's lanes start the next z-step together
            }
            if (iter_count) iter_count[k] = total_it;
            if constexpr (DISS) {
                // publish this stroke's FEs, then count it; the second stroke of the pixel integrates
                const int pix = k < half ? k : k - half;
                __threadfence();
                if (atomicAdd(DA.pair + pix, 1) == 1) {
                    __threadfence();
                    const float4* Ff = FEs;
                    const float4* Fb = FEs + (size_t)half * nzs;
                    for (int o = 0; o < DA.n_out; o++)
                        DA.E[(size_t)pix * DA.n_out + o] =
                            diss_value(Ff, Fb, (size_t)pix * nzs, nzs, DA.n, DA.h, DA.off, DA.idx, o, CgLoad{});
                }
            }
        }
        __syncwarp();  // the whole warp draws the next tile
    }
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
        const float4 g = interp_fe<size_t>(G, pos);
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
    SPM_REQUIRE((p->flags & ~(SPM_FLAG_FIRE | SPM_FLAG_FLIP_Z | SPM_FLAG_PAIRED | SPM_FLAG_POLISH)) == 0,
                "%s: unknown flags 0x%x", who, p->flags);
    return SPM_OK;
}

GridView make_view(const float* grid, int nx, int ny, int nz, const spm_scan_params* p) {
    GridView G;
    G.g = reinterpret_cast<const float4*>(grid);
    G.nx = nx; G.ny = ny; G.nz = nz;
    G.x_lo = 0; G.nx_slab = nx; G.y_lo = 0; G.ny_slab = ny; G.z_lo = 0; G.nz_slab = nz; G.stride = 1;
    G.dA = make_float4(p->dinvA[0], p->dinvA[1], p->dinvA[2], p->dinvA[3]);
    G.dB = make_float4(p->dinvB[0], p->dinvB[1], p->dinvB[2], p->dinvB[3]);
    G.dC = make_float4(p->dinvC[0], p->dinvC[1], p->dinvC[2], p->dinvC[3]);
    return G;
}

int static_blocks(int n_scan, const spm_scan_params& P) {
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

// Persistent grid size of a counter-scheduled relaxation kernel: as many CTAs as are co-resident
// (the counter balances the rest).
template <class K>
int persistent_blocks(K kern, int n_scan, int& blocks) {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, RX_THREADS, 0) != cudaSuccess)
        return set_error(SPM_ERR_CUDA, "relax: cannot query the device occupancy");
    const int cap = sms * (per_sm > 0 ? per_sm : 1);
    const int need = (n_scan + RX_THREADS - 1) / RX_THREADS;
    blocks = need < cap ? need : cap;
    return SPM_OK;
}

template <int MODE, typename IDX, bool POLISH>
int launch_relax(const GridView& G, const float4* pts, int n_scan, const spm_scan_params& P, float4* FEs,
                 float4* disps, int* iter_count, unsigned* counter, cudaStream_t st) {
    if (counter) {
        if (cudaMemsetAsync(counter, 0, sizeof(unsigned), st) != cudaSuccess)
            return set_error(SPM_ERR_CUDA, "relax: cannot reset the pixel counter");
        if constexpr (MODE <= 2) {  // z-synchronised tiles from the counter
            auto kern = relax_tile_kernel<MODE, IDX, POLISH, false>;
            int blocks = 0;
            if (int rc = persistent_blocks(kern, n_scan, blocks)) return rc;
            kern<<<blocks, RX_THREADS, 0, st>>>(G, pts, n_scan, P, FEs, disps, iter_count, counter, DissArgs{});
            return check_launch("relax");
        }
        auto kern = relax_kernel<MODE, IDX, (MODE <= 2), POLISH>;
        int blocks = 0;
        if (int rc = persistent_blocks(kern, n_scan, blocks)) return rc;
        kern<<<blocks, RX_THREADS, 0, st>>>(G, pts, n_scan, P, FEs, disps, iter_count, counter);
        return check_launch("relax");
    }
    relax_kernel<MODE, IDX, (MODE <= 2), POLISH><<<static_blocks(n_scan, P), RX_THREADS, 0, st>>>(
        G, pts, n_scan, P, FEs, disps, iter_count, counter);
    return check_launch("relax");
}

template <int MODE>
int launch_mode(const GridView& G, long long nodes, const float4* pts, int n_scan, const spm_scan_params& P,
                float4* FEs, float4* disps, int* iter_count, unsigned* counter, cudaStream_t st) {
    if constexpr (MODE <= 2) {
        if (P.flags & SPM_FLAG_POLISH) {
            if (nodes < (1LL << 32))
                return launch_relax<MODE, unsigned, true>(G, pts, n_scan, P, FEs, disps, iter_count, counter, st);
            return launch_relax<MODE, size_t, true>(G, pts, n_scan, P, FEs, disps, iter_count, counter, st);
        }
    }
    if (nodes < (1LL << 32))
        return launch_relax<MODE, unsigned, false>(G, pts, n_scan, P, FEs, disps, iter_count, counter, st);
    return launch_relax<MODE, size_t, false>(G, pts, n_scan, P, FEs, disps, iter_count, counter, st);
}

// ---- batched SPM_RELAX_PP ---------------------------------------------------
// Slot t of the batch -> (molecule, pixel): the molecule owning t by its
// slot_off prefix; inside a raster molecule slots run over tiles of
// (32 >> th_log2) (ix) x (1 << th_log2) (iy) pixels, tiles ordered iy-fastest.
__device__ __forceinline__ bool next_batch_pixel(unsigned* counter, unsigned n_slots, const spm_batch_mol* mols,
                                                 int n_mol, int th_log2, int& m, int& k) {
    const unsigned lane = threadIdx.x & 31u;
    while (true) {
        const unsigned msk = __activemask();
        const int leader = __ffs(msk) - 1;
        const unsigned rank = __popc(msk & ((1u << lane) - 1u));
        unsigned base = 0;
        if ((int)lane == leader) base = atomicAdd(counter, (unsigned)__popc(msk));
        base = __shfl_sync(msk, base, leader);
        const unsigned t = base + rank;
        if (t >= n_slots) return false;
        m = SPM_MOL_BY(slot_off, mols, n_mol, (long long)t);
        const spm_batch_mol* D = mols + m;
        if (slot_pixel(D, t - (unsigned)D->slot_off, th_log2, k)) return true;
        // a slot outside the raster (edge tile) or past the last pixel: draw again (t only grows: bounded)
    }
}

// One SPM_RELAX_PP iteration of a z-stroke (probe frame = identity, tipC =
// (0,0,1,dz)) on an axis-aligned slab: pp_iter with the frame rotations
// dropped -- with an identity frame they change no value (the sign of an exact
// zero aside) -- and c*surf reduced to its z part.
template <typename IDX, bool CACHE, int LAYOUT>
__device__ __forceinline__ float4 sample_z(const AxisView& G, V3 p, TexelCache& T) {
    if constexpr (CACHE) return interp_fe_cached<IDX, LAYOUT>(G, p, T);
    else return interp_fe_cell<IDX, LAYOUT>(G, p);
}

template <typename IDX, bool CACHE, int LAYOUT>
__device__ __forceinline__ bool pp_iter_z(const AxisView& G, TexelCache& T, const spm_scan_params& P, V3 tip,
                                          V3& pos, V3& v, float& dt, float& damp, float4& fe, int& it, int& total_it,
                                          bool& conv) {
    conv = false;
    if (it >= P.max_iter) return true;
    ++it;
    ++total_it;
    fe = sample_z<IDX, CACHE, LAYOUT>(G, pos, T);
    if (fe.w != fe.w) return true;  // outside the slab (or a NaN grid): not converged
    const V3 ft = tip_force(sub3(pos, tip), ld4(P.stiffness), ld4(P.dpos0));
    V3 f = mk3(fe.x + ft.x, fe.y + ft.y, fe.z + ft.z);
    f.z = __fadd_rn(f.z, P.surfFF[0]);
    if (dot3(f, f) < P.f2conv) {
        conv = true;
        return true;
    }
    // the stroke's integrator constants straight from the launch parameters (dtmin = dtmax * 0.1)
    md_step_c(f, v, pos, dt, damp, __fmul_rn(P.relax_params[0], 0.1f), P.relax_params[0], P.relax_params[1],
              (P.flags & SPM_FLAG_FIRE) != 0);
    return it >= P.max_iter;
}

template <int LAYOUT>
__device__ __forceinline__ AxisView axis_view(const spm_batch_mol* D, const float* grid) {
    AxisView G;
    G.g = reinterpret_cast<const float4*>(grid) + LAYOUT * D->grid_off;
    G.nx = D->nx; G.ny = D->ny; G.nz = D->nz;
    G.x_lo = D->x_lo; G.nx_slab = D->nx_slab;
    G.y_lo = D->y_lo; G.ny_slab = D->ny_slab;
    G.z_lo = D->z_lo; G.nz_slab = D->nz_slab;
    G.fnx = (float)G.nx; G.fny = (float)G.ny; G.fnz = (float)G.nz;
    G.ax = D->dinvA[0]; G.aw = D->dinvA[3];
    G.by = D->dinvB[1]; G.bw = D->dinvB[3];
    G.cz = D->dinvC[2]; G.cw = D->dinvC[3];
    return G;
}

// Variants (spm_batch_shape.rx_regs): MINB = 3: up to 80 registers per thread
// (768 resident threads per SM); MINB = 4: 64 registers (1024 threads, a few
// spilled values); CACHE: texels kept in registers across iterations (112
// registers, MINB = 2); MINB = 5: CTAs of at most 128 threads at up to 102
// registers (640 threads per SM).
template <int MINB, bool CACHE, int LAYOUT>
__global__ void __launch_bounds__(MINB == 5 ? 128 : 256, MINB)
batch_relax_kernel(int n_mol, const spm_batch_mol* __restrict__ mols, unsigned n_slots, int th_log2,
                   const float* __restrict__ grid, const float4* __restrict__ pts, spm_scan_params P,
                   float4* __restrict__ FEs, float4* __restrict__ PPs, int* __restrict__ iter_count,
                   unsigned* __restrict__ counter) {
    const float dz = P.tipC[3];
    int m = 0, k = 0;
    bool have = next_batch_pixel(counter, n_slots, mols, n_mol, th_log2, m, k);
    AxisView G;
    TexelCache T;
    long long sbase = 0;
    int nzs = 0, pix = 0;
    V3 tip, pos, v;
    float dt = 0.f, damp = 0.f;
    float4 fe;
    int iz = 0, it = 0, total_it = 0;
    auto start = [&]() {
        const spm_batch_mol* D = mols + m;
        G = axis_view<LAYOUT>(D, grid);
        T.kx = __int_as_float(0x7fc00000);  // new slab: nothing cached (NaN matches no cell)
        nzs = D->nz_steps;
        pix = D->pix_off + k;
        sbase = D->state_off + (long long)k * nzs;
        const float4 p4 = pts[pix];
        tip = mk3(p4.x, p4.y, p4.z);
        pos = mk3(tip.x + P.dpos0[0], tip.y + P.dpos0[1], tip.z + P.dpos0[2]);
        dt = P.relax_params[0];
        damp = P.relax_params[1];
        v = mk3(0.f, 0.f, 0.f);
        fe = make_float4(0.f, 0.f, 0.f, 0.f);
        iz = 0;
        it = 0;
        total_it = 0;
    };
    if (have) start();
    while (have) {
        bool conv;
        if (pp_iter_z<unsigned, CACHE, LAYOUT>(G, T, P, tip, pos, v, dt, damp, fe, it, total_it, conv)) {
            if (!conv) fe = sample_z<unsigned, CACHE, LAYOUT>(G, pos, T);  // the position moved after the last sample
            const long long o = sbase + iz;
            FEs[o] = fe;
            // all seven values finite <=> the sum of their products with zero is zero
            // (x*0 is NaN for x = +-inf or NaN, +-0 otherwise)
            float z0 = __fmul_rn(fe.x, 0.f);
            z0 = __fmaf_rn(fe.y, 0.f, z0);
            z0 = __fmaf_rn(fe.z, 0.f, z0);
            z0 = __fmaf_rn(fe.w, 0.f, z0);
            z0 = __fmaf_rn(pos.x, 0.f, z0);
            z0 = __fmaf_rn(pos.y, 0.f, z0);
            z0 = __fmaf_rn(pos.z, 0.f, z0);
            const bool finite = (z0 == 0.f);
            PPs[o] = make_float4(pos.x, pos.y, pos.z, (float)((conv && finite) ? it : -it));
            tip.z = __fadd_rn(tip.z, dz);
            pos.z = __fadd_rn(pos.z, dz);
            v = mk3(0.f, 0.f, 0.f);
            it = 0;
            if (++iz == nzs) {
                if (iter_count) iter_count[pix] = total_it;
                have = next_batch_pixel(counter, n_slots, mols, n_mol, th_log2, m, k);
                if (have) start();
            }
        }
    }
}

// z-synchronised schedule (spm_batch_shape.rx_sync = 1): a warp draws 32
// slots at once -- one pixel tile of one molecule, slot numbering being
// 32-aligned per molecule -- and its lanes relax their strokes one z-step at a
// time, waiting for each other at the end of every z-step.  Every texel load
// of the warp then reads the same z-layers around neighbouring pixels; the
// cost is the lanes idling while the tile's slowest pixel of that z-step
// converges.  Each lane runs exactly the FIRE sequence of the other schedule
// (pp_iter_z), so the results are the same bits.
//
// Cell fetcher of an axis-aligned batch slab for newton_polish: the same
// addressing as interp_fe_cell, the eight texels unpacked to float4.
template <int LAYOUT>
struct SlabCellFetch {
    const AxisView& G;
    __device__ __forceinline__ bool operator()(V3 p, float& ax, float& ay, float& az, float4 (&t)[8]) const {
        const float u = __fmaf_rn(p.x, G.ax, G.aw);
        const float v = __fmaf_rn(p.y, G.by, G.bw);
        const float w = __fmaf_rn(p.z, G.cz, G.cw);
        int x0, x1, y0, y1, z0, z1;
        bool ok = tex_axis(u, G.nx, G.fnx, x0, x1, ax);
        ok = tex_axis(v, G.ny, G.fny, y0, y1, ay) && ok;
        ok = tex_axis(w, G.nz, G.fnz, z0, z1, az) && ok;
        ok = ok && to_slab(x0, x1, G.x_lo, G.nx_slab) && to_slab(y0, y1, G.y_lo, G.ny_slab) &&
             to_slab(z0, z1, G.z_lo, G.nz_slab);
        if (!ok) return false;
        ulonglong2 c[8];
        load_cell<LAYOUT, unsigned>(G, x0, y0, y1, z0, z1, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7]);
#pragma unroll
        for (int i = 0; i < 8; i++) {
            upk(c[i].x, t[i].x, t[i].y);
            upk(c[i].y, t[i].z, t[i].w);
        }
        return true;
    }
};

// SlabCellFetch through the lane's TexelCache: a cell already cached (the one FIRE ended in, or the
// previous Newton evaluation's) needs no loads; a new cell is loaded and cached.  The same texel
// values either way.
template <int LAYOUT>
struct SlabCellFetchCached {
    const AxisView& G;
    TexelCache& T;
    __device__ __forceinline__ bool operator()(V3 p, float& ax, float& ay, float& az, float4 (&t)[8]) const {
        const float u = __fmaf_rn(p.x, G.ax, G.aw);
        const float v = __fmaf_rn(p.y, G.by, G.bw);
        const float w = __fmaf_rn(p.z, G.cz, G.cw);
        float fx, fy, fz;
        ax = tex_coord(u, G.fnx, fx);
        ay = tex_coord(v, G.fny, fy);
        az = tex_coord(w, G.fnz, fz);
        if (!(fx == T.kx && fy == T.ky && fz == T.kz)) {
            int x0, x1, y0, y1, z0, z1;
            bool ok = tex_index(fx, G.nx, G.fnx, x0, x1);
            ok = tex_index(fy, G.ny, G.fny, y0, y1) && ok;
            ok = tex_index(fz, G.nz, G.fnz, z0, z1) && ok;
            ok = ok && to_slab(x0, x1, G.x_lo, G.nx_slab) && to_slab(y0, y1, G.y_lo, G.ny_slab) &&
                 to_slab(z0, z1, G.z_lo, G.nz_slab);
            if (!ok) return false;
            load_cell<LAYOUT, unsigned>(G, x0, y0, y1, z0, z1, T.f000, T.f100, T.f010, T.f110, T.f001, T.f101,
                                        T.f011, T.f111);
            T.kx = fx;
            T.ky = fy;
            T.kz = fz;
        }
        const ulonglong2 c[8] = {T.f000, T.f100, T.f010, T.f110, T.f001, T.f101, T.f011, T.f111};
#pragma unroll
        for (int i = 0; i < 8; i++) {
            upk(c[i].x, t[i].x, t[i].y);
            upk(c[i].y, t[i].z, t[i].w);
        }
        return true;
    }
};

// newton_core on a batch slab, kept out of line for the kernels that also run FIRE: the FIRE loop
// keeps its registers, and every argument goes by value so that no caller variable (the lane's
// texel cache above all) has its address taken and moves to local memory.  The callee fetches its
// cells itself.  q: the start; ok false (q, fe not set) when its cell is not available.
struct NewtonResult {
    V3 q;
    float4 fe;
    float g2;
    int evals;
    bool ok;
};

template <int LAYOUT>
__device__ __noinline__ NewtonResult slab_newton(const AxisView G, const PolishSpring S, float t00, float t11,
                                                 float t22, V3 tip, V3 q, bool early, float f2stop) {
    const float Tc[3][3] = {{t00, 0.f, 0.f}, {0.f, t11, 0.f}, {0.f, 0.f, t22}};
    NewtonResult r;
    r.q = q;
    r.fe = make_float4(0.f, 0.f, 0.f, 0.f);
    r.g2 = 0.f;
    r.evals = 0;
    r.ok = newton_core(SlabCellFetch<LAYOUT>{G}, Tc, S, tip, r.q, r.fe, r.g2, r.evals, early, f2stop,
                       early ? WARM_NEWTON_STEPS : POLISH_STEPS);
    return r;
}

// Warm start (SPM_FLAG_WARM): a z-step starts from the equilibrium the state
// had in the previous call (PPs in) when that one converged and the stroke
// arrives at this z-step where it arrived in the previous call: its
// continuation start (the previous z-step's end position, shifted with the
// tip) within WARM_MAX_JUMP per axis of the previous call's (the previous
// call's equilibrium of the previous z-step, shifted the same way; at the
// first z-step both are the tip's start).  Otherwise -- the probe jumped on
// the way down in one of the two calls, or there is no previous equilibrium --
// it starts from the continuation as a cold call does, so every state stays on
// its stroke's branch.
// An optimiser step that moves every atom by 0.01 A and every charge by 0.01 e moves 99% of the
// equilibria -- and so of the continuation starts -- by less than 0.35 A (the soft lateral
// spring); a bound of 0.1 A sent 3% of the strokes back to FIRE after such a step.
constexpr float WARM_MAX_JUMP = 0.3f;

// A lane's stroke state between z-steps: the tip, the continuation position,
// the FIRE velocity and integrator state (carried down the stroke), the last
// sample and the iteration total.
struct StrokeLane {
    V3 tip, pos, v;
    V3 prev;  // SPM_FLAG_WARM: the previous call's continuation start of this z-step (x NaN: none)
    float dt, damp;
    float4 fe;
    int total_it;
};

// The polish's spring and texel-coordinate transform of an axis-aligned batch slab.
__device__ __forceinline__ void batch_polish_setup(const AxisView& G, const spm_scan_params& P, PolishSpring& S,
                                                   float (&Tc)[3][3]) {
    S.a = mk3(1.f, 0.f, 0.f); S.b = mk3(0.f, 1.f, 0.f); S.c = mk3(0.f, 0.f, 1.f);
    S.kk = ld4(P.stiffness); S.d0 = ld4(P.dpos0);
    S.surf = P.surfFF[0];
    S.frame = true;
    S.ident = true;  // batches scan z-strokes (a, b, c = x, y, z; checked at launch) on axis-aligned slabs
    Tc[0][0] = __fmul_rn(G.fnx, G.ax); Tc[0][1] = 0.f; Tc[0][2] = 0.f;
    Tc[1][0] = 0.f; Tc[1][1] = __fmul_rn(G.fny, G.by); Tc[1][2] = 0.f;
    Tc[2][0] = 0.f; Tc[2][1] = 0.f; Tc[2][2] = __fmul_rn(G.fnz, G.cz);
}

// One z-step of a lane's stroke (state o): the warm start, Newton-first with
// POLISH, FIRE, the polish, the outputs, and the step to the next z-step.
// PREFIX (two-pass schedule, POLISH and SPM_FLAG_WARM): only a z-step that
// Newton's method finishes from the previous equilibrium is done; any other
// returns false with nothing stored and L unchanged, for the FIRE pass to
// redo from the same state.
template <bool CACHE, int LAYOUT, bool POLISH, bool PREFIX>
__device__ __forceinline__ bool stroke_zstep(const AxisView& G, TexelCache& T, const spm_scan_params& P,
                                             const PolishSpring& S, const float (&Tc)[3][3], StrokeLane& L,
                                             long long o, float dz, float4* __restrict__ FEs,
                                             float4* __restrict__ PPs) {
    V3 pos = L.pos;
    bool warm_start = false;
    V3 next_prev = mk3(__int_as_float(0x7fc00000), 0.f, 0.f);
    if (P.flags & SPM_FLAG_WARM) {
        const float4 pw = PPs[o];
        if (pw.w > 0.f) {  // false for NaN
            if (fabsf(pos.x - L.prev.x) <= WARM_MAX_JUMP && fabsf(pos.y - L.prev.y) <= WARM_MAX_JUMP &&
                fabsf(pos.z - L.prev.z) <= WARM_MAX_JUMP) {  // false for NaN
                pos = mk3(pw.x, pw.y, pw.z);
                warm_start = true;
            }
            next_prev = mk3(pw.x, pw.y, __fadd_rn(pw.z, dz));
        }
    }
    int it = 0;
    bool conv = false, newton_done = false;
    float4 fe = L.fe;
    if constexpr (POLISH) {
        // from a previous equilibrium Newton's method converges in a few steps: FIRE only if it does not
        if (warm_start) {
            NewtonResult r;
            if constexpr (PREFIX) {  // no FIRE in this kernel: inline, through the lane's texel cache
                r.q = pos;
                r.ok = newton_core(SlabCellFetchCached<LAYOUT>{G, T}, Tc, S, L.tip, r.q, r.fe, r.g2, r.evals, true,
                                   P.f2conv, WARM_NEWTON_STEPS);
            } else {
                r = slab_newton<LAYOUT>(G, S, Tc[0][0], Tc[1][1], Tc[2][2], L.tip, pos, true, P.f2conv);
            }
            if (r.ok) {
                pos = r.q;
                if (r.g2 < P.f2conv) {
                    fe = r.fe;
                    it = r.evals;
                    conv = true;
                    newton_done = true;
                }
            }
        }
    }
    if constexpr (PREFIX) {
        if (!newton_done) return false;
    }
    L.total_it += it;
    if (!newton_done) {
        while (!pp_iter_z<unsigned, CACHE, LAYOUT>(G, T, P, L.tip, pos, L.v, L.dt, L.damp, fe, it, L.total_it,
                                                   conv)) {
        }
        if (!conv) fe = sample_z<unsigned, CACHE, LAYOUT>(G, pos, T);  // the position moved after the last sample
    }
    V3 q = pos;
    if constexpr (POLISH) {
        if (!newton_done && fe.w == fe.w) {
            const NewtonResult r = slab_newton<LAYOUT>(G, S, Tc[0][0], Tc[1][1], Tc[2][2], L.tip, q, false, 0.f);
            if (r.ok) {
                q = r.q;
                fe = r.fe;
            }
        }
    }
    FEs[o] = fe;
    // all seven values finite <=> the sum of their products with zero is zero
    float z0 = __fmul_rn(fe.x, 0.f);
    z0 = __fmaf_rn(fe.y, 0.f, z0);
    z0 = __fmaf_rn(fe.z, 0.f, z0);
    z0 = __fmaf_rn(fe.w, 0.f, z0);
    z0 = __fmaf_rn(q.x, 0.f, z0);
    z0 = __fmaf_rn(q.y, 0.f, z0);
    z0 = __fmaf_rn(q.z, 0.f, z0);
    const bool finite = (z0 == 0.f);
    PPs[o] = make_float4(q.x, q.y, q.z, (float)((conv && finite) ? it : -it));
    L.fe = fe;
    L.tip.z = __fadd_rn(L.tip.z, dz);
    L.pos = mk3(pos.x, pos.y, __fadd_rn(pos.z, dz));
    L.prev = next_prev;
    L.v = mk3(0.f, 0.f, 0.f);
    return true;
}

// A lane's stroke state at its first z-step.
__device__ __forceinline__ StrokeLane stroke_start(const float4* __restrict__ pts, int pix, const spm_scan_params& P) {
    const float4 p4 = pts[pix];
    StrokeLane L;
    L.tip = mk3(p4.x, p4.y, p4.z);
    L.pos = mk3(L.tip.x + P.dpos0[0], L.tip.y + P.dpos0[1], L.tip.z + P.dpos0[2]);
    L.prev = L.pos;  // the first z-step starts where it started in every call
    L.v = mk3(0.f, 0.f, 0.f);
    L.dt = P.relax_params[0];
    L.damp = P.relax_params[1];
    L.fe = make_float4(0.f, 0.f, 0.f, 0.f);
    L.total_it = 0;
    return L;
}

// One lane's stroke of pixel k; every lane of `members` runs the same number
// of z-steps (the molecule's nz_steps) and meets the others after each.
// POLISH: each z-step's equilibrium Newton-polished before it is stored (the
// stroke continues from the unpolished position, as relax_pp_pixel and the
// per-image kernels do).
template <bool CACHE, int LAYOUT, bool POLISH>
__device__ __forceinline__ void relax_tile_stroke(const spm_batch_mol* D, const float* __restrict__ grid,
                                                  const float4* __restrict__ pts, const spm_scan_params& P,
                                                  float4* __restrict__ FEs, float4* __restrict__ PPs,
                                                  int* __restrict__ iter_count, int k, float dz, unsigned members) {
    const AxisView G = axis_view<LAYOUT>(D, grid);
    TexelCache T;
    T.kx = __int_as_float(0x7fc00000);  // nothing cached (NaN matches no cell)
    const int nzs = D->nz_steps;
    const int pix = D->pix_off + k;
    const long long sbase = D->state_off + (long long)k * nzs;
    StrokeLane L = stroke_start(pts, pix, P);
    PolishSpring S;
    float Tc[3][3];
    if constexpr (POLISH) batch_polish_setup(G, P, S, Tc);
    for (int iz = 0; iz < nzs; ++iz) {
        stroke_zstep<CACHE, LAYOUT, POLISH, false>(G, T, P, S, Tc, L, sbase + iz, dz, FEs, PPs);
        __syncwarp(members);  // the tile's lanes start the next z-step together
    }
    if (iter_count) iter_count[pix] = L.total_it;
}

// ---- two-pass schedule (spm_batch_shape.rx_sync = 2, POLISH and WARM) ----
// In a fit's later calls most z-steps finish with Newton's method from their
// previous equilibrium, and a few need FIRE; in one z-synchronised tile the
// few hold the whole warp at every z-step.  The prefix pass runs the tiles
// with Newton only: a lane's stroke goes as far as its z-steps finish that
// way, and at its first z-step that needs FIRE the lane stores its stroke
// state (before that z-step) in the tail list and stops.  The tail pass runs
// the listed strokes from there with the full z-step, 32 entries per warp
// stepping together.  Each z-step does exactly the computation of the
// one-pass schedule from the same state, so the results are the same bits.
struct TailEntry {
    int m, k, iz, total_it;
    float tip_z, px, py, pz;
    float qx, qy, qz, pad;  // StrokeLane::prev
};
static_assert(sizeof(TailEntry) == 48, "tail entries are 48 bytes");

// Workspace of the two-pass schedule: words 0-1 as the one-pass kernels (slot
// counter, staged-variant flag), word 2 the tail count, word 3 the tail pass's
// draw counter, then the tail list from byte 16.
constexpr long long TAIL_OFF = 16;

template <int MINB, bool CACHE, int LAYOUT>
__global__ void __launch_bounds__(MINB == 5 ? 128 : 256, MINB)
batch_relax_prefix_kernel(int n_mol, const spm_batch_mol* __restrict__ mols, unsigned n_slots, int th_log2,
                          const float* __restrict__ grid, const float4* __restrict__ pts, spm_scan_params P,
                          float4* __restrict__ FEs, float4* __restrict__ PPs, int* __restrict__ iter_count,
                          unsigned* __restrict__ ws) {
    const float dz = P.tipC[3];
    const unsigned lane = threadIdx.x & 31u;
    TailEntry* tail = reinterpret_cast<TailEntry*>(reinterpret_cast<char*>(ws) + TAIL_OFF);
    while (true) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(ws, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n_slots) return;  // warp-uniform
        const int m = SPM_MOL_BY(slot_off, mols, n_mol, (long long)base);
        const spm_batch_mol* D = mols + m;
        int k;
        const bool valid = slot_pixel(D, base + lane - (unsigned)D->slot_off, th_log2, k);
        const unsigned members = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const AxisView G = axis_view<LAYOUT>(D, grid);
            TexelCache T;
            T.kx = __int_as_float(0x7fc00000);
            const int nzs = D->nz_steps;
            const int pix = D->pix_off + k;
            const long long sbase = D->state_off + (long long)k * nzs;
            StrokeLane L = stroke_start(pts, pix, P);
            PolishSpring S;
            float Tc[3][3];
            batch_polish_setup(G, P, S, Tc);
            bool active = true;
            for (int iz = 0; iz < nzs; ++iz) {  // every member runs every z-step: the ballots stay uniform
                const bool fail = active && !stroke_zstep<CACHE, LAYOUT, true, true>(G, T, P, S, Tc, L, sbase + iz,
                                                                                      dz, FEs, PPs);
                const unsigned fm = __ballot_sync(members, fail);
                if (fm) {
                    const int leader = __ffs(fm) - 1;
                    unsigned at = 0;
                    if ((int)lane == leader) at = atomicAdd(ws + 2, (unsigned)__popc(fm));
                    at = __shfl_sync(members, at, leader);
                    if (fail) {  // L is the state before this z-step (a failed prefix z-step leaves it)
                        TailEntry e;
                        e.m = m; e.k = k; e.iz = iz; e.total_it = L.total_it;
                        e.tip_z = L.tip.z; e.px = L.pos.x; e.py = L.pos.y; e.pz = L.pos.z;
                        e.qx = L.prev.x; e.qy = L.prev.y; e.qz = L.prev.z; e.pad = 0.f;
                        tail[at + (unsigned)__popc(fm & ((1u << lane) - 1u))] = e;  // < n_slots: one per stroke
                        active = false;
                    }
                }
                __syncwarp(members);
            }
            if (active && iter_count) iter_count[pix] = L.total_it;
        }
        __syncwarp();  // the whole warp draws the next tile
    }
}

template <int MINB, bool CACHE, int LAYOUT>
__global__ void __launch_bounds__(MINB == 5 ? 128 : 256, MINB)
batch_relax_tail_kernel(const spm_batch_mol* __restrict__ mols, const float* __restrict__ grid,
                        const float4* __restrict__ pts, spm_scan_params P, float4* __restrict__ FEs,
                        float4* __restrict__ PPs, int* __restrict__ iter_count, unsigned* __restrict__ ws) {
    const float dz = P.tipC[3];
    const unsigned lane = threadIdx.x & 31u;
    const TailEntry* tail = reinterpret_cast<const TailEntry*>(reinterpret_cast<const char*>(ws) + TAIL_OFF);
    const unsigned n_tail = ws[2];  // written by the prefix pass, which ran before this launch
    // entries per draw: 32 while the list fills every launched warp; a shorter list is spread over
    // all of them (a warp's time is the sum over its rounds of its slowest lane's FIRE steps, so
    // strokes sharing a warp wait for one another while whole warps would sit idle)
    const unsigned warps = gridDim.x * (blockDim.x >> 5);
    const unsigned per = min(32u, max(1u, (n_tail + warps - 1u) / warps));
    while (true) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(ws + 3, per);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n_tail) return;  // warp-uniform
        const bool valid = lane < per && base + lane < n_tail;
        const unsigned members = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const TailEntry e = tail[base + lane];
            const spm_batch_mol* D = mols + e.m;
            const AxisView G = axis_view<LAYOUT>(D, grid);
            TexelCache T;
            T.kx = __int_as_float(0x7fc00000);
            const int nzs = D->nz_steps;
            const int pix = D->pix_off + e.k;
            const long long sbase = D->state_off + (long long)e.k * nzs;
            StrokeLane L = stroke_start(pts, pix, P);  // tip x, y and the integrator's start values
            L.tip.z = e.tip_z;
            L.pos = mk3(e.px, e.py, e.pz);
            L.prev = mk3(e.qx, e.qy, e.qz);
            L.total_it = e.total_it;
            PolishSpring S;
            float Tc[3][3];
            batch_polish_setup(G, P, S, Tc);
            const int steps = nzs - e.iz;
            const int rounds = __reduce_max_sync(members, steps);
            for (int r = 0; r < rounds; ++r) {  // the same count on every member
                if (r < steps) stroke_zstep<CACHE, LAYOUT, true, false>(G, T, P, S, Tc, L, sbase + e.iz + r, dz, FEs, PPs);
                __syncwarp(members);
            }
            if (iter_count) iter_count[pix] = L.total_it;
        }
        __syncwarp();
    }
}

template <int MINB, bool CACHE, int LAYOUT, bool POLISH>
__global__ void __launch_bounds__(MINB == 5 ? 128 : 256, MINB)
batch_relax_sync_kernel(int n_mol, const spm_batch_mol* __restrict__ mols, unsigned n_slots, int th_log2,
                        const float* __restrict__ grid, const float4* __restrict__ pts, spm_scan_params P,
                        float4* __restrict__ FEs, float4* __restrict__ PPs, int* __restrict__ iter_count,
                        unsigned* __restrict__ counter) {
    const float dz = P.tipC[3];
    const unsigned lane = threadIdx.x & 31u;
    while (true) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(counter, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n_slots) return;  // warp-uniform
        const int m = SPM_MOL_BY(slot_off, mols, n_mol, (long long)base);
        const spm_batch_mol* D = mols + m;
        int k;
        const bool valid = slot_pixel(D, base + lane - (unsigned)D->slot_off, th_log2, k);
        const unsigned members = __ballot_sync(0xffffffffu, valid);
        if (valid) relax_tile_stroke<CACHE, LAYOUT, POLISH>(D, grid, pts, P, FEs, PPs, iter_count, k, dz, members);
        __syncwarp();  // the whole warp draws the next tile
    }
}

// ---- z-slab staging in shared memory through the bulk-copy (TMA) engine ----
// spm_batch_shape.rx_regs = 5 (x-pair slabs, 128-thread CTAs, rx_sync = 1).  At
// every z-step each warp computes the box of slab nodes around its lanes'
// current cells (the cells' x range -1..+1, y and z ranges -1..+2: room for the
// probe to move a cell) and copies its (z, y) rows -- contiguous runs of
// x-pair nodes, 32 bytes each -- into the warp's shared-memory slice with
// cp.async.bulk (one row per lane at a time, completion on the warp's
// mbarrier).  A texel-cache miss then reads a cell inside the box from shared
// memory, else from global memory as the default kernel does; a box larger
// than STAGE_CAP nodes is not staged (all misses go to global memory).  The
// wait is bounded: after STAGE_SPIN polls the warp records the timeout in the
// workspace (word 1), waits once more (bounded) for its copies and stops
// staging.  Results are the default kernel's bits (the same texel values).
// Loads are plain bulk copies from this GPU's own memory (no multicast).
constexpr int STAGE_WARPS = 4;
constexpr int STAGE_CAP = 320;  // nodes per warp (10 KB)
constexpr unsigned STAGE_SPIN = 1u << 20;

struct StageBox {
    const ulonglong2* s;  // the warp's slice: node (x, y, z) of the box at 2 * ((z * ny + y) * nx + x)
    int x0, y0, z0, nx, ny, nz;
    bool ok;
};

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}" : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}

// interp_fe_cached's miss path with the staged box first (x-pair slabs).
__device__ __forceinline__ float4 interp_fe_staged(const AxisView& G, V3 p, TexelCache& T, const StageBox& B) {
    const float u = __fmaf_rn(p.x, G.ax, G.aw);
    const float v = __fmaf_rn(p.y, G.by, G.bw);
    const float w = __fmaf_rn(p.z, G.cz, G.cw);
    float fx, fy, fz;
    const float ax = tex_coord(u, G.fnx, fx);
    const float ay = tex_coord(v, G.fny, fy);
    const float az = tex_coord(w, G.fnz, fz);
    if (!(fx == T.kx && fy == T.ky && fz == T.kz)) {
        int x0, x1, y0, y1, z0, z1;
        bool ok = tex_index(fx, G.nx, G.fnx, x0, x1);
        ok = tex_index(fy, G.ny, G.fny, y0, y1) && ok;
        ok = tex_index(fz, G.nz, G.fnz, z0, z1) && ok;
        ok = ok && to_slab(x0, x1, G.x_lo, G.nx_slab) && to_slab(y0, y1, G.y_lo, G.ny_slab) &&
             to_slab(z0, z1, G.z_lo, G.nz_slab);
        if (!ok) {
            float nan = __int_as_float(0x7fc00000);
            return make_float4(nan, nan, nan, nan);
        }
        const int bx = x0 - B.x0, by0 = y0 - B.y0, by1 = y1 - B.y0, bz0 = z0 - B.z0, bz1 = z1 - B.z0;
        if (B.ok && (unsigned)bx < (unsigned)B.nx && (unsigned)by0 < (unsigned)B.ny && (unsigned)by1 < (unsigned)B.ny &&
            (unsigned)bz0 < (unsigned)B.nz && (unsigned)bz1 < (unsigned)B.nz) {
            const ulonglong2* q00 = B.s + 2 * ((bz0 * B.ny + by0) * B.nx + bx);
            const ulonglong2* q10 = B.s + 2 * ((bz0 * B.ny + by1) * B.nx + bx);
            const ulonglong2* q01 = B.s + 2 * ((bz1 * B.ny + by0) * B.nx + bx);
            const ulonglong2* q11 = B.s + 2 * ((bz1 * B.ny + by1) * B.nx + bx);
            T.f000 = q00[0]; T.f100 = q00[1];
            T.f010 = q10[0]; T.f110 = q10[1];
            T.f001 = q01[0]; T.f101 = q01[1];
            T.f011 = q11[0]; T.f111 = q11[1];
        } else {
            load_cell<2, unsigned>(G, x0, y0, y1, z0, z1, T.f000, T.f100, T.f010, T.f110, T.f001, T.f101, T.f011,
                                   T.f111);
        }
        T.kx = fx;
        T.ky = fy;
        T.kz = fz;
    }
    return blend_cached(T, ax, ay, az);
}

// The staged counterpart of relax_tile_stroke (no polish, no warm start).
__device__ __forceinline__ void relax_tile_stroke_staged(const spm_batch_mol* D, const float* __restrict__ grid,
                                                         const float4* __restrict__ pts, const spm_scan_params& P,
                                                         float4* __restrict__ FEs, float4* __restrict__ PPs,
                                                         int* __restrict__ iter_count, int k, float dz,
                                                         unsigned members, ulonglong2* slice, unsigned bar,
                                                         unsigned& parity, bool& staging, unsigned* status) {
    const AxisView G = axis_view<2>(D, grid);
    TexelCache T;
    T.kx = __int_as_float(0x7fc00000);
    const int nzs = D->nz_steps;
    const int pix = D->pix_off + k;
    const long long sbase = D->state_off + (long long)k * nzs;
    const float4 p4 = pts[pix];
    V3 tip = mk3(p4.x, p4.y, p4.z);
    V3 pos = mk3(tip.x + P.dpos0[0], tip.y + P.dpos0[1], tip.z + P.dpos0[2]);
    V3 v = mk3(0.f, 0.f, 0.f);
    float dt = P.relax_params[0], damp = P.relax_params[1];
    float4 fe = make_float4(0.f, 0.f, 0.f, 0.f);
    int total_it = 0;
    const unsigned lane = threadIdx.x & 31u;
    const int leader = __ffs(members) - 1;
    for (int iz = 0; iz < nzs; ++iz) {
        StageBox B;
        B.s = slice;
        B.ok = false;
        if (staging) {
            // this lane's cell (slab indices), -1 if it is not an interior, stored cell
            float fx, fy, fz;
            tex_coord(__fmaf_rn(pos.x, G.ax, G.aw), G.fnx, fx);
            tex_coord(__fmaf_rn(pos.y, G.by, G.bw), G.fny, fy);
            tex_coord(__fmaf_rn(pos.z, G.cz, G.cw), G.fnz, fz);
            const int cx = (int)fx - G.x_lo, cy = (int)fy - G.y_lo, cz = (int)fz - G.z_lo;
            const bool in = fx == fx && fy == fy && fz == fz && cx >= 0 && cy >= 0 && cz >= 0 &&
                            cx < G.nx_slab && cy + 1 < G.ny_slab && cz + 1 < G.nz_slab;
            // warp min / max over the members (redux.sync: defined for any member mask); lanes without a
            // stored interior cell contribute the neutral values
            int mn[3], mx[3];
            mn[0] = __reduce_min_sync(members, in ? cx : INT_MAX);
            mn[1] = __reduce_min_sync(members, in ? cy : INT_MAX);
            mn[2] = __reduce_min_sync(members, in ? cz : INT_MAX);
            mx[0] = __reduce_max_sync(members, in ? cx : -1);
            mx[1] = __reduce_max_sync(members, in ? cy : -1);
            mx[2] = __reduce_max_sync(members, in ? cz : -1);
            if (mn[0] != INT_MAX) {  // then every mn/mx is a cell index in [0, n_slab)
                const int bx0 = max(mn[0] - 1, 0), bx1 = min(mx[0] + 1, G.nx_slab - 1);
                const int by0 = max(mn[1] - 1, 0), by1 = min(mx[1] + 2, G.ny_slab - 1);
                const int bz0 = max(mn[2] - 1, 0), bz1 = min(mx[2] + 2, G.nz_slab - 1);
                B.x0 = bx0; B.y0 = by0; B.z0 = bz0;
                B.nx = bx1 - bx0 + 1; B.ny = by1 - by0 + 1; B.nz = bz1 - bz0 + 1;
                if (B.nx >= 1 && B.ny >= 1 && B.nz >= 1 && B.nx <= STAGE_CAP && B.ny <= STAGE_CAP &&
                    B.nz <= STAGE_CAP && B.nx * B.ny * B.nz <= STAGE_CAP) {
                    const int rows = B.ny * B.nz;
                    const unsigned row_bytes = (unsigned)B.nx * 32u;
                    if ((int)lane == leader) {
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                                     :: "r"(bar), "r"(row_bytes * (unsigned)rows) : "memory");
                    }
                    __syncwarp(members);
                    const int rank = __popc(members & ((1u << lane) - 1u)), nmem = __popc(members);
                    for (int r = rank; r < rows; r += nmem) {
                        const int y = r % B.ny, z = r / B.ny;
                        const float4* src = G.g + 2 * (((size_t)(bz0 + z) * G.ny_slab + (by0 + y)) * G.nx_slab + bx0);
                        const unsigned dst = smem_addr(slice + 2 * (size_t)r * B.nx);
                        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                                     "[%0], [%1], %2, [%3];" :: "r"(dst), "l"(src), "r"(row_bytes), "r"(bar)
                                     : "memory");
                    }
                    unsigned spins = 0;
                    bool done = mbar_try_wait(bar, parity);
                    while (!done && ++spins < STAGE_SPIN) done = mbar_try_wait(bar, parity);
                    if (!done) {
                        // record it, give the copies a last bounded chance, and stop staging for good
                        atomicOr(status, 1u);
                        spins = 0;
                        while (!done && ++spins < STAGE_SPIN) done = mbar_try_wait(bar, parity);
                        staging = false;
                    } else {
                        B.ok = true;
                    }
                    parity ^= 1u;
                    __syncwarp(members);
                }
            }
        }
        int it = 0;
        bool conv = false;
        while (true) {
            if (it >= P.max_iter) break;
            ++it;
            ++total_it;
            fe = interp_fe_staged(G, pos, T, B);
            if (fe.w != fe.w) break;
            const V3 ft = tip_force(sub3(pos, tip), ld4(P.stiffness), ld4(P.dpos0));
            V3 f = mk3(fe.x + ft.x, fe.y + ft.y, fe.z + ft.z);
            f.z = __fadd_rn(f.z, P.surfFF[0]);
            if (dot3(f, f) < P.f2conv) {
                conv = true;
                break;
            }
            md_step_c(f, v, pos, dt, damp, __fmul_rn(P.relax_params[0], 0.1f), P.relax_params[0], P.relax_params[1],
                      (P.flags & SPM_FLAG_FIRE) != 0);
        }
        if (!conv) fe = interp_fe_staged(G, pos, T, B);  // the position moved after the last sample
        const long long o = sbase + iz;
        FEs[o] = fe;
        float z0 = __fmul_rn(fe.x, 0.f);
        z0 = __fmaf_rn(fe.y, 0.f, z0);
        z0 = __fmaf_rn(fe.z, 0.f, z0);
        z0 = __fmaf_rn(fe.w, 0.f, z0);
        z0 = __fmaf_rn(pos.x, 0.f, z0);
        z0 = __fmaf_rn(pos.y, 0.f, z0);
        z0 = __fmaf_rn(pos.z, 0.f, z0);
        const bool finite = (z0 == 0.f);
        PPs[o] = make_float4(pos.x, pos.y, pos.z, (float)((conv && finite) ? it : -it));
        tip.z = __fadd_rn(tip.z, dz);
        pos.z = __fadd_rn(pos.z, dz);
        v = mk3(0.f, 0.f, 0.f);
        __syncwarp(members);  // the tile's lanes start the next z-step (and its staging) together
    }
    if (iter_count) iter_count[pix] = total_it;
}

__global__ void __launch_bounds__(STAGE_WARPS * 32, 4)
batch_relax_staged_kernel(int n_mol, const spm_batch_mol* __restrict__ mols, unsigned n_slots, int th_log2,
                          const float* __restrict__ grid, const float4* __restrict__ pts, spm_scan_params P,
                          float4* __restrict__ FEs, float4* __restrict__ PPs, int* __restrict__ iter_count,
                          unsigned* __restrict__ counter) {
    __shared__ __align__(128) ulonglong2 s_box[STAGE_WARPS][2 * STAGE_CAP];
    __shared__ __align__(8) unsigned long long s_bar[STAGE_WARPS];
    const float dz = P.tipC[3];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned bar = smem_addr(&s_bar[warp]);
    if (lane == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    unsigned parity = 0;
    bool staging = true;
    while (true) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(counter, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n_slots) return;  // warp-uniform
        const int m = SPM_MOL_BY(slot_off, mols, n_mol, (long long)base);
        const spm_batch_mol* D = mols + m;
        int k;
        const bool valid = slot_pixel(D, base + lane - (unsigned)D->slot_off, th_log2, k);
        const unsigned members = __ballot_sync(0xffffffffu, valid);
        if (valid)
            relax_tile_stroke_staged(D, grid, pts, P, FEs, PPs, iter_count, k, dz, members, s_box[warp], bar, parity,
                                     staging, counter + 1);
        // lanes outside the tile keep the warp's staging state in step with the members'
        parity = __shfl_sync(0xffffffffu, parity, __ffs(members) - 1);
        staging = __shfl_sync(0xffffffffu, staging, __ffs(members) - 1);
        __syncwarp();  // the whole warp draws the next tile
    }
}

}  // namespace
}  // namespace spm

extern "C" long long spm_batch_relax_workspace_bytes(long long n_slots, const spm_batch_shape* shape) {
    if (n_slots < 0 || !shape) return -1;
    return spm::TAIL_OFF + (shape->rx_sync == 2 ? (long long)sizeof(spm::TailEntry) * n_slots : 0);
}

extern "C" int spm_batch_relax(int n_mol, const spm_batch_mol* mols, long long n_slots, const spm_batch_shape* shape,
                               const float* grid, const float* points, const spm_scan_params* p, float* FEs,
                               float* PPs, int* iter_count, void* workspace, long long workspace_bytes,
                               void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(shape && p, "spm_batch_relax: null shape/params");
    SPM_REQUIRE(n_mol >= 0 && n_slots >= 0, "spm_batch_relax: negative sizes");
    if (n_mol == 0 || n_slots == 0) return SPM_OK;
    SPM_REQUIRE(n_slots < (1LL << 31), "spm_batch_relax: %lld slots exceed the 31-bit counter", n_slots);
    SPM_REQUIRE(mols && grid && points && FEs && PPs && workspace, "spm_batch_relax: null device pointer");
    SPM_REQUIRE(aligned16(grid) && aligned16(points) && aligned16(FEs) && aligned16(PPs) &&
                (reinterpret_cast<uintptr_t>(workspace) & 3u) == 0 && (reinterpret_cast<uintptr_t>(mols) & 7u) == 0,
                "spm_batch_relax: misaligned buffers");
    SPM_REQUIRE((p->flags & ~(SPM_FLAG_FIRE | SPM_FLAG_FLIP_Z | SPM_FLAG_POLISH | SPM_FLAG_WARM)) == 0,
                "spm_batch_relax: unknown flags 0x%x", p->flags);
    if (!(p->tipA[0] == 1.f && p->tipA[1] == 0.f && p->tipA[2] == 0.f && p->tipB[0] == 0.f && p->tipB[1] == 1.f &&
          p->tipB[2] == 0.f && p->tipC[0] == 0.f && p->tipC[1] == 0.f && p->tipC[2] == 1.f))
        return set_error(SPM_ERR_UNSUPPORTED, "spm_batch_relax: batches scan z-strokes: tipA,tipB,tipC must be x,y,z");
    const int thr = shape->rx_threads, h = shape->rx_tile_h;
    SPM_REQUIRE(thr == 64 || thr == 128 || thr == 256, "spm_batch_relax: rx_threads=%d", thr);
    SPM_REQUIRE(h >= 1 && h <= 32 && (h & (h - 1)) == 0, "spm_batch_relax: rx_tile_h=%d", h);
    SPM_REQUIRE(shape->rx_ctas_per_sm >= 0, "spm_batch_relax: rx_ctas_per_sm=%d", shape->rx_ctas_per_sm);
    int th_log2 = 0;
    while ((1 << th_log2) < h) th_log2++;
    SPM_REQUIRE(shape->rx_regs >= 0 && shape->rx_regs <= 5, "spm_batch_relax: rx_regs=%d", shape->rx_regs);
    if (shape->rx_regs == 5)
        SPM_REQUIRE(thr == 128 && shape->grid_layout == 0 && shape->rx_sync == 1 &&
                    !(p->flags & (SPM_FLAG_POLISH | SPM_FLAG_WARM)),
                    "spm_batch_relax: rx_regs=5 (shared-memory slab staging) takes 128-thread CTAs, x-pair slabs, "
                    "rx_sync = 1 and neither SPM_FLAG_POLISH nor SPM_FLAG_WARM");
    SPM_REQUIRE(shape->rx_regs != 4 || thr <= 128, "spm_batch_relax: rx_regs=4 takes CTAs of at most 128 threads, "
                "rx_threads=%d", thr);
    SPM_REQUIRE(shape->grid_layout == 0 || shape->grid_layout == 1, "spm_batch_relax: grid_layout=%d",
                shape->grid_layout);
    SPM_REQUIRE(shape->rx_sync >= 0 && shape->rx_sync <= 2, "spm_batch_relax: rx_sync=%d", shape->rx_sync);
    if (p->flags & (SPM_FLAG_POLISH | SPM_FLAG_WARM))
        SPM_REQUIRE(shape->rx_sync >= 1, "spm_batch_relax: SPM_FLAG_POLISH / SPM_FLAG_WARM need the z-synchronised "
                    "schedules (rx_sync = 1 or 2)");
    SPM_REQUIRE(shape->rx_regs != 5 || shape->rx_sync == 1, "spm_batch_relax: rx_regs=5 takes rx_sync = 1");
    const long long ws_need = spm_batch_relax_workspace_bytes(n_slots, shape);
    SPM_REQUIRE(workspace_bytes >= ws_need, "spm_batch_relax: workspace of %lld bytes, %lld needed", workspace_bytes,
                ws_need);
    // rx_sync = 2 runs the two-pass schedule when a warm polished call can use it, else rx_sync = 1's
    const bool two_pass = shape->rx_sync == 2 && (p->flags & SPM_FLAG_POLISH) && (p->flags & SPM_FLAG_WARM);
    const int sync = shape->rx_sync == 2 ? 1 : shape->rx_sync;
    using Kern = decltype(&batch_relax_kernel<3, false, 2>);
    // [rx_sync][grid_layout][rx_regs]: 0 = 80 registers, 1 = 64, 2 = texel cache at up to 128,
    // 3 = texel cache squeezed to 80 (some values spilled, 50% more warps), 4 = texel cache at up to 102
    // (128-thread CTAs)
    static const Kern table[2][2][5] = {
        {{batch_relax_kernel<3, false, 2>, batch_relax_kernel<4, false, 2>, batch_relax_kernel<2, true, 2>,
          batch_relax_kernel<3, true, 2>, batch_relax_kernel<5, true, 2>},
         {batch_relax_kernel<3, false, 4>, batch_relax_kernel<4, false, 4>, batch_relax_kernel<2, true, 4>,
          batch_relax_kernel<3, true, 4>, batch_relax_kernel<5, true, 4>}},
        {{batch_relax_sync_kernel<3, false, 2, false>, batch_relax_sync_kernel<4, false, 2, false>,
          batch_relax_sync_kernel<2, true, 2, false>, batch_relax_sync_kernel<3, true, 2, false>,
          batch_relax_sync_kernel<5, true, 2, false>},
         {batch_relax_sync_kernel<3, false, 4, false>, batch_relax_sync_kernel<4, false, 4, false>,
          batch_relax_sync_kernel<2, true, 4, false>, batch_relax_sync_kernel<3, true, 4, false>,
          batch_relax_sync_kernel<5, true, 4, false>}}};
    // the polished z-synchronised variants, [grid_layout][rx_regs]
    static const Kern polished[2][5] = {
        {batch_relax_sync_kernel<3, false, 2, true>, batch_relax_sync_kernel<4, false, 2, true>,
         batch_relax_sync_kernel<2, true, 2, true>, batch_relax_sync_kernel<3, true, 2, true>,
         batch_relax_sync_kernel<5, true, 2, true>},
        {batch_relax_sync_kernel<3, false, 4, true>, batch_relax_sync_kernel<4, false, 4, true>,
         batch_relax_sync_kernel<2, true, 4, true>, batch_relax_sync_kernel<3, true, 4, true>,
         batch_relax_sync_kernel<5, true, 4, true>}};
    // the two-pass schedule's passes, [grid_layout][rx_regs]
    static const Kern prefix[2][5] = {
        {batch_relax_prefix_kernel<3, false, 2>, batch_relax_prefix_kernel<4, false, 2>,
         batch_relax_prefix_kernel<2, true, 2>, batch_relax_prefix_kernel<3, true, 2>,
         batch_relax_prefix_kernel<5, true, 2>},
        {batch_relax_prefix_kernel<3, false, 4>, batch_relax_prefix_kernel<4, false, 4>,
         batch_relax_prefix_kernel<2, true, 4>, batch_relax_prefix_kernel<3, true, 4>,
         batch_relax_prefix_kernel<5, true, 4>}};
    using TailKern = decltype(&batch_relax_tail_kernel<3, false, 2>);
    static const TailKern tails[2][5] = {
        {batch_relax_tail_kernel<3, false, 2>, batch_relax_tail_kernel<4, false, 2>,
         batch_relax_tail_kernel<2, true, 2>, batch_relax_tail_kernel<3, true, 2>, batch_relax_tail_kernel<5, true, 2>},
        {batch_relax_tail_kernel<3, false, 4>, batch_relax_tail_kernel<4, false, 4>,
         batch_relax_tail_kernel<2, true, 4>, batch_relax_tail_kernel<3, true, 4>, batch_relax_tail_kernel<5, true, 4>}};
    const Kern kern = shape->rx_regs == 5 ? batch_relax_staged_kernel
                      : two_pass ? prefix[shape->grid_layout][shape->rx_regs]
                      : (p->flags & SPM_FLAG_POLISH) ? polished[shape->grid_layout][shape->rx_regs]
                                                      : table[sync][shape->grid_layout][shape->rx_regs];
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, thr, 0) != cudaSuccess)
        return set_error(SPM_ERR_CUDA, "spm_batch_relax: cannot query the device occupancy");
    if (per_sm < 1) per_sm = 1;
    if (shape->rx_ctas_per_sm > 0 && shape->rx_ctas_per_sm < per_sm) per_sm = shape->rx_ctas_per_sm;
    const long long need = (n_slots + thr - 1) / thr;
    const long long cap = (long long)sms * per_sm;
    const unsigned blocks = (unsigned)(need < cap ? need : cap);
    cudaStream_t st = as_stream(stream);
    unsigned* ctr = static_cast<unsigned*>(workspace);
    // word 0: the slot counter; word 1: the staged variant's wait-timeout flag; words 2-3: the two-pass
    // schedule's tail count and tail draw counter
    if (cudaMemsetAsync(ctr, 0, 4 * sizeof(unsigned), st) != cudaSuccess)
        return set_error(SPM_ERR_CUDA, "spm_batch_relax: cannot reset the slot counter");
    kern<<<blocks, thr, 0, st>>>(n_mol, mols, (unsigned)n_slots, th_log2, grid,
                                               reinterpret_cast<const float4*>(points), *p,
                                               reinterpret_cast<float4*>(FEs), reinterpret_cast<float4*>(PPs),
                                               iter_count, ctr);
    if (two_pass) {
        int rc = check_launch("spm_batch_relax (prefix pass)");
        if (rc) return rc;
        // the tail list is drawn up to 32 entries per warp until the count the prefix pass left is used up
        const TailKern tk = tails[shape->grid_layout][shape->rx_regs];
        int per_sm_t = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_t, tk, thr, 0) != cudaSuccess)
            return set_error(SPM_ERR_CUDA, "spm_batch_relax: cannot query the device occupancy");
        if (per_sm_t < 1) per_sm_t = 1;
        if (shape->rx_ctas_per_sm > 0 && shape->rx_ctas_per_sm < per_sm_t) per_sm_t = shape->rx_ctas_per_sm;
        const long long cap_t = (long long)sms * per_sm_t;
        tk<<<(unsigned)(need < cap_t ? need : cap_t), thr, 0, st>>>(mols, grid, reinterpret_cast<const float4*>(points),
                                                                     *p, reinterpret_cast<float4*>(FEs),
                                                                     reinterpret_cast<float4*>(PPs), iter_count, ctr);
        return check_launch("spm_batch_relax (tail pass)");
    }
    return check_launch("spm_batch_relax");
}

extern "C" long long spm_relax_workspace_bytes(void) { return 16; }

extern "C" int spm_relax_ex(int mode, const float* grid, int nx, int ny, int nz, const float* points, int n_scan,
                            const spm_scan_params* p, float* FEs, float* disps, int* iter_count, void* workspace,
                            void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(mode == SPM_RELAX_STROKES || mode == SPM_RELAX_TILTED || mode == SPM_RELAX_PP ||
                mode == SPM_RELAX_2D, "spm_relax_ex: mode=%d", mode);
    int rc = check_scan_args("spm_relax_ex", grid, nx, ny, nz, points, n_scan, p, FEs);
    if (rc) return rc;
    if (p->flags & SPM_FLAG_PAIRED)
        SPM_REQUIRE(mode == SPM_RELAX_STROKES && n_scan % 2 == 0,
                    "spm_relax_ex: SPM_FLAG_PAIRED needs mode SPM_RELAX_STROKES and an even n_scan (mode=%d, n_scan=%d)",
                    mode, n_scan);
    if (p->flags & SPM_FLAG_POLISH)
        SPM_REQUIRE(mode != SPM_RELAX_2D, "spm_relax_ex: SPM_FLAG_POLISH is not defined for SPM_RELAX_2D");
    if (n_scan == 0 || p->nz == 0) return SPM_OK;
    if (mode != SPM_RELAX_TILTED)
        SPM_REQUIRE(disps != nullptr && aligned16(disps), "spm_relax_ex: disps/PPs null or misaligned");
    SPM_REQUIRE(workspace == nullptr || (reinterpret_cast<uintptr_t>(workspace) & 3u) == 0,
                "spm_relax_ex: workspace not 4-byte aligned");
    spm_scan_params P = normalized(p, n_scan);
    const GridView G = make_view(grid, nx, ny, nz, p);
    const long long nodes = (long long)nx * ny * nz;
    const float4* pt = reinterpret_cast<const float4*>(points);
    unsigned* ctr = static_cast<unsigned*>(workspace);
    cudaStream_t st = as_stream(stream);
    if (mode == SPM_RELAX_STROKES)
        return launch_mode<0>(G, nodes, pt, n_scan, P, reinterpret_cast<float4*>(FEs),
                              reinterpret_cast<float4*>(disps), iter_count, ctr, st);
    if (mode == SPM_RELAX_PP)
        return launch_mode<2>(G, nodes, pt, n_scan, P, reinterpret_cast<float4*>(FEs),
                              reinterpret_cast<float4*>(disps), iter_count, ctr, st);
    if (mode == SPM_RELAX_2D)
        return launch_mode<3>(G, nodes, pt, n_scan, P, reinterpret_cast<float4*>(FEs),
                              reinterpret_cast<float4*>(disps), iter_count, ctr, st);
    return launch_mode<1>(G, nodes, pt, n_scan, P, reinterpret_cast<float4*>(FEs), nullptr, iter_count, ctr, st);
}

extern "C" int spm_relax_strokes(const float* grid, int nx, int ny, int nz, const float* points, int n_scan,
                                 const spm_scan_params* p, float* FEs, float* disps, void* stream) {
    return spm_relax_ex(SPM_RELAX_STROKES, grid, nx, ny, nz, points, n_scan, p, FEs, disps, nullptr, nullptr, stream);
}

extern "C" int spm_relax_strokes_tilted(const float* grid, int nx, int ny, int nz, const float* points, int n_scan,
                                        const spm_scan_params* p, float* FEs, void* stream) {
    return spm_relax_ex(SPM_RELAX_TILTED, grid, nx, ny, nz, points, n_scan, p, FEs, nullptr, nullptr, nullptr, stream);
}

extern "C" int spm_fe_in_strokes_tilted(const float* grid, int nx, int ny, int nz, const float* points, int n_scan,
                                        const spm_scan_params* p, float* FEs, void* stream) {
    using namespace spm;
    clear_error();
    int rc = check_scan_args("spm_fe_in_strokes_tilted", grid, nx, ny, nz, points, n_scan, p, FEs);
    if (rc) return rc;
    SPM_REQUIRE(!(p->flags & (SPM_FLAG_PAIRED | SPM_FLAG_POLISH)),
                "spm_fe_in_strokes_tilted: SPM_FLAG_PAIRED / SPM_FLAG_POLISH are for the relaxations only");
    if (n_scan == 0 || p->nz == 0) return SPM_OK;
    spm_scan_params P = normalized(p, n_scan);
    raw_kernel<<<static_blocks(n_scan, P), RX_THREADS, 0, as_stream(stream)>>>(
        make_view(grid, nx, ny, nz, p), reinterpret_cast<const float4*>(points), n_scan, P,
        reinterpret_cast<float4*>(FEs));
    return check_launch("spm_fe_in_strokes_tilted");
}

extern "C" long long spm_relax_pair_workspace_bytes(int n_scan) {
    if (n_scan < 0) return 0;
    return 16 + 4LL * (n_scan / 2);
}

extern "C" int spm_relax_pair_dissipation(const float* grid, int nx, int ny, int nz, const float* points, int n_scan,
                                          const spm_scan_params* p, float* FEs, float* disps, int* iter_count,
                                          const double* n, const double* h_scan, const int* off, const int* idx,
                                          int n_out, float* E_diss, void* workspace, void* stream) {
    using namespace spm;
    clear_error();
    int rc = check_scan_args("spm_relax_pair_dissipation", grid, nx, ny, nz, points, n_scan, p, FEs);
    if (rc) return rc;
    SPM_REQUIRE((p->flags & SPM_FLAG_PAIRED) && n_scan % 2 == 0,
                "spm_relax_pair_dissipation: needs SPM_FLAG_PAIRED and an even n_scan (n_scan=%d)", n_scan);
    SPM_REQUIRE(n && workspace && n_out >= 0, "spm_relax_pair_dissipation: null direction/workspace or n_out < 0");
    if (n_scan == 0 || p->nz == 0) return SPM_OK;
    SPM_REQUIRE(disps && aligned16(disps), "spm_relax_pair_dissipation: disps null or misaligned");
    SPM_REQUIRE(n_out == 0 || (h_scan && off && idx && E_diss), "spm_relax_pair_dissipation: null dissipation array");
    SPM_REQUIRE((reinterpret_cast<uintptr_t>(workspace) & 15u) == 0,
                "spm_relax_pair_dissipation: workspace not 16-byte aligned");
    const double nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    SPM_REQUIRE(nn > 0.0 && isfinite(nn), "spm_relax_pair_dissipation: oscillation direction must be non-zero");
    spm_scan_params P = normalized(p, n_scan);
    const GridView G = make_view(grid, nx, ny, nz, p);
    DissArgs DA;
    DA.h = h_scan; DA.off = off; DA.idx = idx; DA.E = E_diss; DA.n_out = n_out;
    // the oscillation direction as compute_dissipation takes it: n = osc_dir / |osc_dir|
    for (int d = 0; d < 3; d++) DA.n[d] = n[d] / nn;
    unsigned* ctr = static_cast<unsigned*>(workspace);
    DA.pair = reinterpret_cast<int*>(static_cast<char*>(workspace) + 16);
    cudaStream_t st = as_stream(stream);
    if (cudaMemsetAsync(DA.pair, 0, sizeof(int) * (size_t)(n_scan / 2), st) != cudaSuccess)
        return set_error(SPM_ERR_CUDA, "spm_relax_pair_dissipation: cannot reset the pair counters");
    const bool big = (long long)nx * ny * nz >= (1LL << 32);
    const bool pol = (P.flags & SPM_FLAG_POLISH) != 0;
    auto kern = big ? (pol ? relax_tile_kernel<0, size_t, true, true> : relax_tile_kernel<0, size_t, false, true>)
                    : (pol ? relax_tile_kernel<0, unsigned, true, true> : relax_tile_kernel<0, unsigned, false, true>);
    int blocks = 0;
    if (int rc2 = persistent_blocks(kern, n_scan, blocks)) return rc2;
    if (cudaMemsetAsync(ctr, 0, sizeof(unsigned), st) != cudaSuccess)
        return set_error(SPM_ERR_CUDA, "spm_relax_pair_dissipation: cannot reset the pixel counter");
    kern<<<blocks, RX_THREADS, 0, st>>>(G, reinterpret_cast<const float4*>(points), n_scan, P,
                                        reinterpret_cast<float4*>(FEs), reinterpret_cast<float4*>(disps), iter_count,
                                        ctr, DA);
    return check_launch("spm_relax_pair_dissipation");
}
