// spm_fire.cuh -- device helpers of the probe-relaxation kernels.
//
// The operation order here is the canonical FP32 order of this library:
// every fused multiply-add is an explicit __fmaf_rn and the translation units
// that include this header are compiled with -fmad=false, IEEE sqrt and IEEE
// division.  The relaxation results are therefore a pure function of the
// inputs, independent of compiler contraction choices.
//
// Semantics follow SPAMMM kernels/AFM.cl: tipForce :53-58, interpFE :100-105
// (REPEAT + LINEAR sampler with normalized coordinates, :49), update_FIRE
// :136-157, rotMat/rotMatT kernels/common.cl:43-44.
#pragma once
#include <cuda_runtime.h>
#include "spm_f32x2.cuh"

namespace spm {

struct V3 {
    float x, y, z;
};

__device__ __forceinline__ V3 mk3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 add3(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ float dot3(V3 a, V3 b) {
    return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, __fmul_rn(a.x, b.x)));
}
__device__ __forceinline__ V3 rotmat(V3 v, V3 a, V3 b, V3 c) { return V3{dot3(v, a), dot3(v, b), dot3(v, c)}; }
__device__ __forceinline__ V3 rotmatT(V3 v, V3 a, V3 b, V3 c) {
    return V3{__fmaf_rn(c.x, v.z, __fmaf_rn(b.x, v.y, __fmul_rn(a.x, v.x))),
              __fmaf_rn(c.y, v.z, __fmaf_rn(b.y, v.y, __fmul_rn(a.y, v.x))),
              __fmaf_rn(c.z, v.z, __fmaf_rn(b.z, v.y, __fmul_rn(a.z, v.x)))};
}

// Harmonic 3D spring + radial bond: (d - d0.xyz)*k.xyz + d*(k.w*(r - d0.w)/r).
// With k.w == 0 the radial term is exactly +-0 and is skipped (only the sign of
// an all-zero component can differ from adding it; the oracle does the same).
__device__ __forceinline__ V3 tip_force(V3 d, float4 k, float4 d0) {
    if (k.w == 0.f)
        return V3{__fmul_rn(d.x - d0.x, k.x), __fmul_rn(d.y - d0.y, k.y), __fmul_rn(d.z - d0.z, k.z)};
    float r = __fsqrt_rn(dot3(d, d));
    r = fmaxf(r, 1e-10f);
    float s = __fdiv_rn(__fmul_rn(k.w, r - d0.w), r);
    return V3{__fmaf_rn(d.x, s, __fmul_rn(d.x - d0.x, k.x)),
              __fmaf_rn(d.y, s, __fmul_rn(d.y - d0.y, k.y)),
              __fmaf_rn(d.z, s, __fmul_rn(d.z - d0.z, k.z))};
}

struct Integrator {
    float dt, damp, dtmin, dtmax, damp0;
};

// FIRE velocity mixing (Bitzek et al., PRL 97, 170201 (2006)) or plain damping,
// followed by v += f*dt, pos += v*dt.  dt and damp evolve; dtmin, dtmax and
// damp0 are the stroke's constants.
__device__ __forceinline__ void md_step_c(V3 f, V3& v, V3& pos, float& dt, float& damp, float dtmin, float dtmax,
                                          float damp0, bool use_fire) {
    if (use_fire) {
        float ff = dot3(f, f);
        float vv = dot3(v, v);
        float vf = dot3(v, f);
        if (vf < 0.f) {
            v.x = __fmul_rn(v.x, 0.f); v.y = __fmul_rn(v.y, 0.f); v.z = __fmul_rn(v.z, 0.f);
            dt = fmaxf(dtmin, __fmul_rn(dt, 0.5f));
            damp = damp0;
        } else {
            float cf = __fmul_rn(damp, __fsqrt_rn(__fdiv_rn(vv, ff + 1e-8f)));
            float cv = 1.f - damp;
            v.x = __fmaf_rn(f.x, cf, __fmul_rn(v.x, cv));
            v.y = __fmaf_rn(f.y, cf, __fmul_rn(v.y, cv));
            v.z = __fmaf_rn(f.z, cf, __fmul_rn(v.z, cv));
            dt = fminf(dtmax, __fmul_rn(dt, 1.1f));
            damp = __fmul_rn(damp, 0.99f);
        }
    } else {
        float cv = 1.f - damp;
        v.x = __fmul_rn(v.x, cv); v.y = __fmul_rn(v.y, cv); v.z = __fmul_rn(v.z, cv);
    }
    v.x = __fmaf_rn(f.x, dt, v.x);
    v.y = __fmaf_rn(f.y, dt, v.y);
    v.z = __fmaf_rn(f.z, dt, v.z);
    pos.x = __fmaf_rn(v.x, dt, pos.x);
    pos.y = __fmaf_rn(v.y, dt, pos.y);
    pos.z = __fmaf_rn(v.z, dt, pos.z);
}

__device__ __forceinline__ void md_step(V3 f, V3& v, V3& pos, Integrator& I, bool use_fire) {
    md_step_c(f, v, pos, I.dt, I.damp, I.dtmin, I.dtmax, I.damp0, use_fire);
}

// REPEAT addressing + linear filter along one axis (OpenCL 1.2 sec. 8.2);
// fn = (float)n.
__device__ __forceinline__ bool tex_axis(float u, int n, float fn, int& i0, int& i1, float& a) {
    float s = u - floorf(u);
    float t = __fmaf_rn(s, fn, -0.5f);
    if (!(t >= -1.f && t < fn)) return false;
    float fi = floorf(t);
    a = t - fi;
    int i = (int)fi;
    if (i < 0) i += n;
    int j = i + 1;
    if (j >= n) j -= n;
    i0 = i;
    i1 = j;
    return true;
}
__device__ __forceinline__ bool tex_axis(float u, int n, int& i0, int& i1, float& a) {
    return tex_axis(u, n, (float)n, i0, i1, a);
}

__device__ __forceinline__ float lerp_c(float a, float ma, float f0, float f1) {
    return __fmaf_rn(a, f1, __fmul_rn(ma, f0));
}

__device__ __forceinline__ float4 lerp4(float a, float ma, float4 f0, float4 f1) {
    return make_float4(lerp_c(a, ma, f0.x, f1.x), lerp_c(a, ma, f0.y, f1.y), lerp_c(a, ma, f0.z, f1.z),
                       lerp_c(a, ma, f0.w, f1.w));
}

struct GridView {
    const float4* __restrict__ g;
    int nx, ny, nz;
    float4 dA, dB, dC;  // normalized-coordinate transform rows
    // slab views: only the box [x_lo, x_lo + nx_slab) x [y_lo, y_lo + ny_slab) x [z_lo, z_lo + nz_slab)
    // of the full grid is stored (full views: the whole grid)
    int x_lo, nx_slab, y_lo, ny_slab, z_lo, nz_slab;
    int stride;         // slab views: float4 per stored node (2 x-pairs, 4 xz-quads); node value first
};

// The texels i0, i1 of a cell along one axis as indices of a stored range
// [lo, lo + n): false when either lies outside it.
__device__ __forceinline__ bool to_slab(int& i0, int& i1, int lo, int n) {
    i0 -= lo;
    i1 -= lo;
    return (unsigned)i0 < (unsigned)n && (unsigned)i1 < (unsigned)n;
}

// interpFE: exact FP32 trilinear sample with periodic wrap on a full
// (nz,ny,nx) grid.  IDX is the type of the node offsets (unsigned for grids
// below 2^32 nodes, size_t above).
template <typename IDX = size_t>
__device__ __forceinline__ float4 interp_fe(const GridView& G, V3 p) {
    float u = __fmaf_rn(p.x, G.dA.x, __fmaf_rn(p.y, G.dA.y, __fmaf_rn(p.z, G.dA.z, G.dA.w)));
    float v = __fmaf_rn(p.x, G.dB.x, __fmaf_rn(p.y, G.dB.y, __fmaf_rn(p.z, G.dB.z, G.dB.w)));
    float w = __fmaf_rn(p.x, G.dC.x, __fmaf_rn(p.y, G.dC.y, __fmaf_rn(p.z, G.dC.z, G.dC.w)));
    int x0, x1, y0, y1, z0, z1;
    float ax, ay, az;
    bool ok = tex_axis(u, G.nx, x0, x1, ax);
    ok = tex_axis(v, G.ny, y0, y1, ay) && ok;
    ok = tex_axis(w, G.nz, z0, z1, az) && ok;
    if (!ok) {
        float nan = __int_as_float(0x7fc00000);
        return make_float4(nan, nan, nan, nan);
    }
    float mx = 1.f - ax, my = 1.f - ay, mz = 1.f - az;
    const IDX r00 = ((IDX)z0 * G.ny + y0) * G.nx, r10 = ((IDX)z0 * G.ny + y1) * G.nx;
    const IDX r01 = ((IDX)z1 * G.ny + y0) * G.nx, r11 = ((IDX)z1 * G.ny + y1) * G.nx;
    float4 f000 = __ldg(G.g + r00 + x0), f100 = __ldg(G.g + r00 + x1);
    float4 f010 = __ldg(G.g + r10 + x0), f110 = __ldg(G.g + r10 + x1);
    float4 f001 = __ldg(G.g + r01 + x0), f101 = __ldg(G.g + r01 + x1);
    float4 f011 = __ldg(G.g + r11 + x0), f111 = __ldg(G.g + r11 + x1);
    float4 c00 = lerp4(ax, mx, f000, f100);
    float4 c10 = lerp4(ax, mx, f010, f110);
    float4 c01 = lerp4(ax, mx, f001, f101);
    float4 c11 = lerp4(ax, mx, f011, f111);
    float4 c0 = lerp4(ay, my, c00, c10);
    float4 c1 = lerp4(ay, my, c01, c11);
    return lerp4(az, mz, c0, c1);
}

// Axis-aligned grids: dinvA = (ax,0,0,aw), dinvB = (0,by,0,bw), dinvC =
// (0,0,cz,cw).  The zero terms of interp_fe's coordinate FMAs are exact, so
// u = fma(p.x, ax, aw) is interp_fe's u for every finite p (up to the sign of
// an exact zero), and the samplers on an AxisView return interp_fe's sample.
struct AxisView {
    const float4* __restrict__ g;
    int nx, ny, nz;                                  // full grid
    int x_lo, nx_slab, y_lo, ny_slab, z_lo, nz_slab;  // the stored box (batch slab)
    float fnx, fny, fnz;  // the dimensions as floats (converted once per pixel, not per sample)
    float ax, aw, by, bw, cz, cw;
};

// lerp_c on two packed channel pairs: fma(a, f1, ma*f0) per lane.
__device__ __forceinline__ ulonglong2 lerp_pk(f2 a, f2 ma, ulonglong2 f0, ulonglong2 f1) {
    return make_ulonglong2(fma2(a, f1.x, mul2(ma, f0.x)), fma2(a, f1.y, mul2(ma, f0.y)));
}

// 256-bit read-only load of an x-pair: (value(x), value(x+1)) as packed
// channel pairs lo = {(Fx,Fy), (Fz,E)} of x and hi = the same of x+1.
__device__ __forceinline__ void ld_pair(const float4* p, ulonglong2& lo, ulonglong2& hi) {
    unsigned long long a, b, c, d;
    asm("ld.global.nc.v4.b64 {%0, %1, %2, %3}, [%4];" : "=l"(a), "=l"(b), "=l"(c), "=l"(d) : "l"(p));
    lo = make_ulonglong2(a, b);
    hi = make_ulonglong2(c, d);
}

// The eight texels of cell (x0, y0..y1, z0..z1) (slab indices) of a slab in
// the x-pair (LAYOUT 2: node idx at G.g[2*idx], its +x neighbour after it) or
// xz-quad (LAYOUT 4: G.g[4*idx + 2*dz + dx]) layout, as packed channel pairs.
// With xz-quads the cell's 8 texels are two 64-byte chunks (rows y0 and y1).
template <int LAYOUT, typename IDX>
__device__ __forceinline__ void load_cell(const AxisView& G, int x0, int y0, int y1, int z0, int z1,
                                          ulonglong2& f000, ulonglong2& f100, ulonglong2& f010, ulonglong2& f110,
                                          ulonglong2& f001, ulonglong2& f101, ulonglong2& f011, ulonglong2& f111) {
    if (LAYOUT == 4) {
        const IDX q0 = ((IDX)z0 * G.ny_slab + y0) * G.nx_slab + x0, q1 = ((IDX)z0 * G.ny_slab + y1) * G.nx_slab + x0;
        ld_pair(G.g + 4 * q0, f000, f100);
        ld_pair(G.g + 4 * q0 + 2, f001, f101);
        ld_pair(G.g + 4 * q1, f010, f110);
        ld_pair(G.g + 4 * q1 + 2, f011, f111);
    } else {
        const IDX r00 = ((IDX)z0 * G.ny_slab + y0) * G.nx_slab + x0, r10 = ((IDX)z0 * G.ny_slab + y1) * G.nx_slab + x0;
        const IDX r01 = ((IDX)z1 * G.ny_slab + y0) * G.nx_slab + x0, r11 = ((IDX)z1 * G.ny_slab + y1) * G.nx_slab + x0;
        ld_pair(G.g + 2 * r00, f000, f100);
        ld_pair(G.g + 2 * r10, f010, f110);
        ld_pair(G.g + 2 * r01, f001, f101);
        ld_pair(G.g + 2 * r11, f011, f111);
    }
}

// interp_fe on an AxisView over an x-paired (LAYOUT 2) or xz-quad (LAYOUT 4)
// slab: the same texel addressing and the same lerps on the same values, so
// the same sample, with the channel pairs (x,y) and (z,w) of a texel lerped
// by one packed f32x2 instruction each; NaN when the cell is not stored.  (The
// cell's +x and +z texels are x0+1 and z0+1, or 0 when a slab spanning that
// axis wraps; both layouts store exactly those.)
template <typename IDX, int LAYOUT>
__device__ __forceinline__ float4 interp_fe_cell(const AxisView& G, V3 p) {
    const float u = __fmaf_rn(p.x, G.ax, G.aw);
    const float v = __fmaf_rn(p.y, G.by, G.bw);
    const float w = __fmaf_rn(p.z, G.cz, G.cw);
    int x0, x1, y0, y1, z0, z1;
    float ax, ay, az;
    bool ok = tex_axis(u, G.nx, G.fnx, x0, x1, ax);
    ok = tex_axis(v, G.ny, G.fny, y0, y1, ay) && ok;
    ok = tex_axis(w, G.nz, G.fnz, z0, z1, az) && ok;
    ok = ok && to_slab(x0, x1, G.x_lo, G.nx_slab) && to_slab(y0, y1, G.y_lo, G.ny_slab) &&
         to_slab(z0, z1, G.z_lo, G.nz_slab);
    if (!ok) {
        float nan = __int_as_float(0x7fc00000);
        return make_float4(nan, nan, nan, nan);
    }
    const f2 AX = bc(ax), MX = bc(1.f - ax), AY = bc(ay), MY = bc(1.f - ay), AZ = bc(az), MZ = bc(1.f - az);
    ulonglong2 f000, f100, f010, f110, f001, f101, f011, f111;
    load_cell<LAYOUT, IDX>(G, x0, y0, y1, z0, z1, f000, f100, f010, f110, f001, f101, f011, f111);
    const ulonglong2 c00 = lerp_pk(AX, MX, f000, f100);
    const ulonglong2 c10 = lerp_pk(AX, MX, f010, f110);
    const ulonglong2 c01 = lerp_pk(AX, MX, f001, f101);
    const ulonglong2 c11 = lerp_pk(AX, MX, f011, f111);
    const ulonglong2 c0 = lerp_pk(AY, MY, c00, c10);
    const ulonglong2 c1 = lerp_pk(AY, MY, c01, c11);
    const ulonglong2 c = lerp_pk(AZ, MZ, c0, c1);
    float4 r;
    upk(c.x, r.x, r.y);
    upk(c.y, r.z, r.w);
    return r;
}

// The eight texels of the last sampled cell, kept in registers across FIRE
// iterations: the probe moves ~1e-3..1e-2 A per iteration inside a 0.1 A
// cell, so the cell rarely changes and most samples need no load at all.
struct TexelCache {
    float kx, ky, kz;  // floor of the cached cell's texel coordinates (NaN: empty)
    ulonglong2 f000, f100, f010, f110, f001, f101, f011, f111;
};

// tex_axis's first half: the texel coordinate t of u and its floor fi (the
// lerp weight is t - fi).  The cell's indices, the wrap and the range test
// are functions of fi alone.
__device__ __forceinline__ float tex_coord(float u, float fn, float& fi) {
    const float s = u - floorf(u);
    const float t = __fmaf_rn(s, fn, -0.5f);
    fi = floorf(t);
    return t - fi;
}

// tex_axis's second half for a given floor fi: false outside the sampler's
// range [-1, n), else the wrapped indices i0, i1.
__device__ __forceinline__ bool tex_index(float fi, int n, float fn, int& i0, int& i1) {
    if (!(fi >= -1.f && fi < fn)) return false;  // <=> t in [-1, fn) for t in [fi, fi + 1)
    int i = (int)fi;
    if (i < 0) i += n;
    int j = i + 1;
    if (j >= n) j -= n;
    i0 = i;
    i1 = j;
    return true;
}

// The packed trilinear blend of a cached cell (interp_fe's lerp order).
__device__ __forceinline__ float4 blend_cached(const TexelCache& T, float ax, float ay, float az) {
    const f2 AX = bc(ax), MX = bc(1.f - ax), AY = bc(ay), MY = bc(1.f - ay), AZ = bc(az), MZ = bc(1.f - az);
    const ulonglong2 c00 = lerp_pk(AX, MX, T.f000, T.f100);
    const ulonglong2 c10 = lerp_pk(AX, MX, T.f010, T.f110);
    const ulonglong2 c01 = lerp_pk(AX, MX, T.f001, T.f101);
    const ulonglong2 c11 = lerp_pk(AX, MX, T.f011, T.f111);
    const ulonglong2 c0 = lerp_pk(AY, MY, c00, c10);
    const ulonglong2 c1 = lerp_pk(AY, MY, c01, c11);
    const ulonglong2 c = lerp_pk(AZ, MZ, c0, c1);
    float4 r;
    upk(c.x, r.x, r.y);
    upk(c.y, r.z, r.w);
    return r;
}

// interp_fe on a full (nz,ny,nx) grid with any sampling transform, with a
// TexelCache: the same texels and lerps, so the same sample; the eight
// texels are loaded only when the cell (the floors of the three texel
// coordinates) changes.  fnx, fny, fnz: the dimensions as floats.
template <typename IDX>
__device__ __forceinline__ float4 interp_fe_cached_full(const GridView& G, float fnx, float fny, float fnz, V3 p,
                                                        TexelCache& T) {
    const float u = __fmaf_rn(p.x, G.dA.x, __fmaf_rn(p.y, G.dA.y, __fmaf_rn(p.z, G.dA.z, G.dA.w)));
    const float v = __fmaf_rn(p.x, G.dB.x, __fmaf_rn(p.y, G.dB.y, __fmaf_rn(p.z, G.dB.z, G.dB.w)));
    const float w = __fmaf_rn(p.x, G.dC.x, __fmaf_rn(p.y, G.dC.y, __fmaf_rn(p.z, G.dC.z, G.dC.w)));
    float fx, fy, fz;
    const float ax = tex_coord(u, fnx, fx);
    const float ay = tex_coord(v, fny, fy);
    const float az = tex_coord(w, fnz, fz);
    if (!(fx == T.kx && fy == T.ky && fz == T.kz)) {
        int x0, x1, y0, y1, z0, z1;
        bool ok = tex_index(fx, G.nx, fnx, x0, x1);
        ok = tex_index(fy, G.ny, fny, y0, y1) && ok;
        ok = tex_index(fz, G.nz, fnz, z0, z1) && ok;
        if (!ok) {
            float nan = __int_as_float(0x7fc00000);
            return make_float4(nan, nan, nan, nan);
        }
        const IDX r00 = ((IDX)z0 * G.ny + y0) * G.nx, r10 = ((IDX)z0 * G.ny + y1) * G.nx;
        const IDX r01 = ((IDX)z1 * G.ny + y0) * G.nx, r11 = ((IDX)z1 * G.ny + y1) * G.nx;
        const ulonglong2* g = reinterpret_cast<const ulonglong2*>(G.g);
        T.f000 = __ldg(g + r00 + x0); T.f100 = __ldg(g + r00 + x1);
        T.f010 = __ldg(g + r10 + x0); T.f110 = __ldg(g + r10 + x1);
        T.f001 = __ldg(g + r01 + x0); T.f101 = __ldg(g + r01 + x1);
        T.f011 = __ldg(g + r11 + x0); T.f111 = __ldg(g + r11 + x1);
        T.kx = fx;
        T.ky = fy;
        T.kz = fz;
    }
    return blend_cached(T, ax, ay, az);
}

// interp_fe_cell with a TexelCache: identical values (the same texels, the
// same lerps); loads only when the cell differs from the cached one.  The
// cell is identified by the floors of its three texel coordinates, so a
// sample inside the cached cell needs no index arithmetic, wrap or range test
// (a cached cell passed them; equal floors give the same indices).
template <typename IDX, int LAYOUT>
__device__ __forceinline__ float4 interp_fe_cached(const AxisView& G, V3 p, TexelCache& T) {
    const float u = __fmaf_rn(p.x, G.ax, G.aw);
    const float v = __fmaf_rn(p.y, G.by, G.bw);
    const float w = __fmaf_rn(p.z, G.cz, G.cw);
    float fx, fy, fz;
    const float ax = tex_coord(u, G.fnx, fx);
    const float ay = tex_coord(v, G.fny, fy);
    const float az = tex_coord(w, G.fnz, fz);
    if (!(fx == T.kx && fy == T.ky && fz == T.kz)) {  // NaN never equals: an empty cache or a NaN position
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
        load_cell<LAYOUT, IDX>(G, x0, y0, y1, z0, z1, T.f000, T.f100, T.f010, T.f110, T.f001, T.f101, T.f011,
                               T.f111);
        T.kx = fx;
        T.ky = fy;
        T.kz = fz;
    }
    return blend_cached(T, ax, ay, az);
}

// ---- Newton polish of a relaxed state (SPM_FLAG_POLISH; not in the reference) --------------
// FIRE stops once |G|^2 < f2conv, where G(q) = F_grid(q) + spring(q) [+ c*surf] is the total
// force on the probe; with k_xy = 0.0156 eV/A^2 a 1e-5 eV/A stop leaves the probe up to ~5e-3 A
// from the equilibrium of the interpolated field.  The polish takes that equilibrium directly:
// G and its Jacobian J = dG/dq are exact functions of the sampled cell -- the trilinear
// interpolant's texel-coordinate derivatives times dt/dq = n * dinv, plus the spring's
// Jacobian -- and up to POLISH_STEPS Newton steps q <- q - J^-1 G are taken, each kept only if
// |dq|_inf <= POLISH_MAX_STEP and it lowers |G|^2.  The oracle (ora_core.h, newton_polish)
// repeats every operation in the same order, so results are bit-identical to it.
constexpr int POLISH_STEPS = 4;
constexpr float NEWTON_FLOOR_STEP = 1e-5f;  // A; the early stop of the warm starts' Newton-first
constexpr int WARM_NEWTON_STEPS = 8;         // steps of the warm starts' Newton-first
constexpr float POLISH_MAX_STEP = 0.1f;
// The warm starts' Newton-first steps up to WARM_MAX_STEP per axis: on the soft lateral spring
// (k_xy = 0.0156 eV/A^2) a 1.6 meV/A change of the grid force moves an equilibrium by 0.1 A, and
// an optimiser step that moves every atom by 0.01 A and every charge by 0.01 e moves half of them
// by more than 0.075 A.
constexpr float WARM_MAX_STEP = 0.3f;

// Spring and frame of a polished state: frame = false is relaxStrokes' spring (tip_force on
// q - tip, no rotation, no surface bias); frame = true the tip frame a,b,c with surf along c.
struct PolishSpring {
    V3 a, b, c;
    float4 kk, d0;
    float surf;
    bool frame;
    // frame with a, b, c = x, y, z and a diagonal texel transform T (batch slabs): the rotations
    // and the zero terms of T are left out -- the same values, up to the sign of a zero
    bool ident = false;
};

// One evaluation at q from the cell's texels t[4*k + 2*j + i] (corner x_i, y_j, z_k) and
// weights (ax, ay, az): fe = the trilinear sample (interp_fe's lerps, so the same value), G,
// and J (row = force component, column = coordinate).  T[a][m] = n_a * dinv_a[m].
__device__ __forceinline__ void polish_eval(const float4 (&t)[8], float ax, float ay, float az,
                                            const float (&T)[3][3], const PolishSpring& S, V3 tip, V3 q,
                                            float4& fe, V3& Gv, float (&J)[3][3]) {
    const float mx = 1.f - ax, my = 1.f - ay, mz = 1.f - az;
    float val[4];
#pragma unroll
    for (int ch = 0; ch < 4; ch++) {
        const float f000 = (&t[0].x)[ch], f100 = (&t[1].x)[ch], f010 = (&t[2].x)[ch], f110 = (&t[3].x)[ch];
        const float f001 = (&t[4].x)[ch], f101 = (&t[5].x)[ch], f011 = (&t[6].x)[ch], f111 = (&t[7].x)[ch];
        const float c00 = lerp_c(ax, mx, f000, f100), c10 = lerp_c(ax, mx, f010, f110);
        const float c01 = lerp_c(ax, mx, f001, f101), c11 = lerp_c(ax, mx, f011, f111);
        const float c0 = lerp_c(ay, my, c00, c10), c1 = lerp_c(ay, my, c01, c11);
        val[ch] = lerp_c(az, mz, c0, c1);
        if (ch < 3) {
            const float e0 = lerp_c(ay, my, f100 - f000, f110 - f010);
            const float e1 = lerp_c(ay, my, f101 - f001, f111 - f011);
            const float dX = lerp_c(az, mz, e0, e1);
            const float dY = lerp_c(az, mz, c10 - c00, c11 - c01);
            const float dZ = c1 - c0;
            if (S.ident) {
                J[ch][0] = __fmul_rn(dX, T[0][0]);
                J[ch][1] = __fmul_rn(dY, T[1][1]);
                J[ch][2] = __fmul_rn(dZ, T[2][2]);
            } else {
#pragma unroll
                for (int m = 0; m < 3; m++)
                    J[ch][m] = __fmaf_rn(dZ, T[2][m], __fmaf_rn(dY, T[1][m], __fmul_rn(dX, T[0][m])));
            }
        }
    }
    fe = make_float4(val[0], val[1], val[2], val[3]);
    const bool rot = S.frame && !S.ident;
    const V3 d = rot ? rotmat(sub3(q, tip), S.a, S.b, S.c) : sub3(q, tip);
    const V3 fs = tip_force(d, S.kk, S.d0);
    const V3 ft = rot ? rotmatT(fs, S.a, S.b, S.c) : fs;
    Gv = mk3(val[0] + ft.x, val[1] + ft.y, val[2] + ft.z);
    if (S.ident) {
        Gv.z = __fadd_rn(S.surf, Gv.z);  // surf along c = z
    } else if (S.frame) {
        Gv.x = __fmaf_rn(S.c.x, S.surf, Gv.x);
        Gv.y = __fmaf_rn(S.c.y, S.surf, Gv.y);
        Gv.z = __fmaf_rn(S.c.z, S.surf, Gv.z);
    }
    // spring Jacobian in the tip frame: diag(k) [+ s I + beta d d^T for the radial bond]
    float Jd[3][3] = {{S.kk.x, 0.f, 0.f}, {0.f, S.kk.y, 0.f}, {0.f, 0.f, S.kk.z}};
    if (S.kk.w != 0.f) {
        float r = __fsqrt_rn(dot3(d, d));
        r = fmaxf(r, 1e-10f);
        const float s = __fdiv_rn(__fmul_rn(S.kk.w, r - S.d0.w), r);
        const float beta = __fdiv_rn(__fmul_rn(S.kk.w, S.d0.w), __fmul_rn(__fmul_rn(r, r), r));
        const float dv[3] = {d.x, d.y, d.z};
        Jd[0][0] = S.kk.x + s;
        Jd[1][1] = S.kk.y + s;
        Jd[2][2] = S.kk.z + s;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const float bd = __fmul_rn(beta, dv[i]);
#pragma unroll
            for (int j = 0; j < 3; j++) Jd[i][j] = __fmaf_rn(bd, dv[j], Jd[i][j]);
        }
    }
    if (rot) {
        const float R[3][3] = {{S.a.x, S.a.y, S.a.z}, {S.b.x, S.b.y, S.b.z}, {S.c.x, S.c.y, S.c.z}};
        float M[3][3];
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int j = 0; j < 3; j++)
                M[m][j] = __fmaf_rn(Jd[m][2], R[2][j], __fmaf_rn(Jd[m][1], R[1][j], __fmul_rn(Jd[m][0], R[0][j])));
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
                J[i][j] = J[i][j] + __fmaf_rn(R[2][i], M[2][j], __fmaf_rn(R[1][i], M[1][j], __fmul_rn(R[0][i], M[0][j])));
    } else {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) J[i][j] = J[i][j] + Jd[i][j];
    }
}

// Newton step dq = -J^-1 G (adjugate / determinant); false when J is singular or the step is
// not finite or longer than max_step along an axis.
__device__ __forceinline__ bool polish_step(const float (&J)[3][3], V3 Gv, V3& dq, float max_step = POLISH_MAX_STEP) {
    float A[3][3];
    A[0][0] = __fmul_rn(J[1][1], J[2][2]) - __fmul_rn(J[1][2], J[2][1]);
    A[0][1] = __fmul_rn(J[0][2], J[2][1]) - __fmul_rn(J[0][1], J[2][2]);
    A[0][2] = __fmul_rn(J[0][1], J[1][2]) - __fmul_rn(J[0][2], J[1][1]);
    A[1][0] = __fmul_rn(J[1][2], J[2][0]) - __fmul_rn(J[1][0], J[2][2]);
    A[1][1] = __fmul_rn(J[0][0], J[2][2]) - __fmul_rn(J[0][2], J[2][0]);
    A[1][2] = __fmul_rn(J[0][2], J[1][0]) - __fmul_rn(J[0][0], J[1][2]);
    A[2][0] = __fmul_rn(J[1][0], J[2][1]) - __fmul_rn(J[1][1], J[2][0]);
    A[2][1] = __fmul_rn(J[0][1], J[2][0]) - __fmul_rn(J[0][0], J[2][1]);
    A[2][2] = __fmul_rn(J[0][0], J[1][1]) - __fmul_rn(J[0][1], J[1][0]);
    const float det = (__fmul_rn(J[0][0], A[0][0]) + __fmul_rn(J[0][1], A[1][0])) + __fmul_rn(J[0][2], A[2][0]);
    if (!(det != 0.f)) return false;  // also NaN
    float r[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const float tq = (__fmul_rn(A[i][0], Gv.x) + __fmul_rn(A[i][1], Gv.y)) + __fmul_rn(A[i][2], Gv.z);
        r[i] = __fdiv_rn(-tq, det);
    }
    if (!(fabsf(r[0]) <= max_step && fabsf(r[1]) <= max_step && fabsf(r[2]) <= max_step))
        return false;  // also NaN
    dq = mk3(r[0], r[1], r[2]);
    return true;
}

// The Newton loop over any cell fetcher: fetch(q, ax, ay, az, t) -> false when q's cell is
// not available (outside the sampler's range or the stored slab).  On return q is the polished
// position, fe the sample there, g2 = |G(q)|^2 and evals the cells evaluated; false (q and fe
// unchanged) when the first fetch fails.
// early (the warm starts' Newton-first, not the polish): steps of up to WARM_MAX_STEP per axis
// (the polish's: POLISH_MAX_STEP), and also stop
//  - before a step whose every component is at most NEWTON_FLOOR_STEP: the predicted distance to
//    the root is at the float32 floor of the positions' noise (the spread of polished equilibria
//    reached from different starts is ~1e-6 A), so the step would change nothing measurable and
//    its cell evaluation is saved -- the previous equilibrium of an unmoved state is kept after one
//    evaluation, a state that moved ~1e-3 A after one step;
//  - after a kept step that lowered |G|^2 by less than 4x to below f2stop (the caller's convergence
//    bound) -- quadratic convergence has ended, |G| is at the float32 floor, and the next step
//    would most likely be refused; above f2stop (a step that crossed into a cell with another
//    Jacobian) the iteration goes on, up to max_steps steps.
template <class Fetch>
__device__ __forceinline__ bool newton_core(const Fetch& fetch, const float (&T)[3][3], const PolishSpring& S,
                                            V3 tip, V3& q, float4& fe, float& g2_out, int& evals,
                                            bool early = false, float f2stop = 0.f, int max_steps = POLISH_STEPS) {
    float4 t[8];
    float ax, ay, az;
    evals = 0;
    if (!fetch(q, ax, ay, az, t)) return false;
    float J[3][3];
    V3 Gv;
    float4 fe0;
    polish_eval(t, ax, ay, az, T, S, tip, q, fe0, Gv, J);
    evals = 1;
    float g2 = dot3(Gv, Gv);
    for (int it = 0; it < max_steps; it++) {
        V3 dq;
        if (!polish_step(J, Gv, dq, early ? WARM_MAX_STEP : POLISH_MAX_STEP)) break;
        if (early && fabsf(dq.x) <= NEWTON_FLOOR_STEP && fabsf(dq.y) <= NEWTON_FLOOR_STEP &&
            fabsf(dq.z) <= NEWTON_FLOOR_STEP)
            break;
        const V3 q1 = add3(q, dq);
        if (!fetch(q1, ax, ay, az, t)) break;
        float J1[3][3];
        V3 G1;
        float4 fe1;
        polish_eval(t, ax, ay, az, T, S, tip, q1, fe1, G1, J1);
        ++evals;
        const float g21 = dot3(G1, G1);
        if (!(g21 < g2)) break;
        const bool slow = !(g21 < 0.25f * g2);
        q = q1;
        fe0 = fe1;
        Gv = G1;
        g2 = g21;
        if (early && slow && g21 < f2stop) break;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) J[i][j] = J1[i][j];
    }
    fe = fe0;
    g2_out = g2;
    return true;
}

// Newton polish of a relaxed state (see above): q, fe in and out.
template <class Fetch>
__device__ __forceinline__ void newton_polish(const Fetch& fetch, const float (&T)[3][3], const PolishSpring& S,
                                              V3 tip, V3& q, float4& fe) {
    float g2;
    int evals;
    newton_core(fetch, T, S, tip, q, fe, g2, evals);
}

// Cell fetcher of a full (nz,ny,nx) grid with any sampling transform (interp_fe's addressing).
template <typename IDX>
struct FullCellFetch {
    const GridView& G;
    __device__ __forceinline__ bool operator()(V3 p, float& ax, float& ay, float& az, float4 (&t)[8]) const {
        const float u = __fmaf_rn(p.x, G.dA.x, __fmaf_rn(p.y, G.dA.y, __fmaf_rn(p.z, G.dA.z, G.dA.w)));
        const float v = __fmaf_rn(p.x, G.dB.x, __fmaf_rn(p.y, G.dB.y, __fmaf_rn(p.z, G.dB.z, G.dB.w)));
        const float w = __fmaf_rn(p.x, G.dC.x, __fmaf_rn(p.y, G.dC.y, __fmaf_rn(p.z, G.dC.z, G.dC.w)));
        int x0, x1, y0, y1, z0, z1;
        bool ok = tex_axis(u, G.nx, x0, x1, ax);
        ok = tex_axis(v, G.ny, y0, y1, ay) && ok;
        ok = tex_axis(w, G.nz, z0, z1, az) && ok;
        if (!ok) return false;
        const IDX r00 = ((IDX)z0 * G.ny + y0) * G.nx, r10 = ((IDX)z0 * G.ny + y1) * G.nx;
        const IDX r01 = ((IDX)z1 * G.ny + y0) * G.nx, r11 = ((IDX)z1 * G.ny + y1) * G.nx;
        t[0] = __ldg(G.g + r00 + x0); t[1] = __ldg(G.g + r00 + x1);
        t[2] = __ldg(G.g + r10 + x0); t[3] = __ldg(G.g + r10 + x1);
        t[4] = __ldg(G.g + r01 + x0); t[5] = __ldg(G.g + r01 + x1);
        t[6] = __ldg(G.g + r11 + x0); t[7] = __ldg(G.g + r11 + x1);
        return true;
    }
};

// T[a][m] = n_a * dinv_a[m] of a full-grid view.
__device__ __forceinline__ void polish_coefs(const GridView& G, float (&T)[3][3]) {
    const float fx = (float)G.nx, fy = (float)G.ny, fz = (float)G.nz;
    T[0][0] = __fmul_rn(fx, G.dA.x); T[0][1] = __fmul_rn(fx, G.dA.y); T[0][2] = __fmul_rn(fx, G.dA.z);
    T[1][0] = __fmul_rn(fy, G.dB.x); T[1][1] = __fmul_rn(fy, G.dB.y); T[1][2] = __fmul_rn(fy, G.dB.z);
    T[2][0] = __fmul_rn(fz, G.dC.x); T[2][1] = __fmul_rn(fz, G.dC.y); T[2][2] = __fmul_rn(fz, G.dC.z);
}

}  // namespace spm
