// adjoint_grid.cu -- implicit-function adjoint of the grid path: d(loss)/d(atom
// positions, charges, LJ or Morse parameters, tip stiffness) through
// (a) the force-grid build and (b) the relaxation on that grid.
//
// The reference differentiates only its grid-free direct path
// (kernels/AFM.cl:1711-2029); this extends the same implicit-function
// construction to the grid path.  At a converged state q* (forward:
// SPM_RELAX_PP) the total force G(q) = F_grid(q) + R^T g(R(q - tip)) + c*surf
// vanishes; F_grid is the trilinear interpolant of the grid's force channels.
//   J  = dF_grid/dq + R^T (dg/dd) R          (F_grid is not a gradient field:
//                                             J is not symmetric)
//   b  = (dF_grid/dq)^T R^T u_xyz + grad(E_grid) u_w
//   J^T lambda = b,   ubar = (R^T u_xyz - lambda, u_w)
// and for any parameter theta of the grid values g(node) or of the spring,
//   dL/dtheta = sum_states sum_corners w * ubar . dg(node)/dtheta  -  lambda . dG_tip/dtheta.
//
// Kernels:
//   adjoint_grid_state_kernel  one thread per state: the 3x3 solve in registers,
//                              status gates (non-converged / non-finite /
//                              unstable / singular / touches a |E|>100-capped
//                              node, where the cap makes g non-differentiable),
//                              ubar and the per-state spring-gradient terms.
//   adjoint_grid_atoms_kernel  CTA per (atom, chunk of 1024 states): each state's
//                              eight trilinear corner nodes are revisited and the
//                              pair-law derivatives evaluated there (a
//                              state-major gather: no scatter onto the grid, no
//                              atomics), FP64 accumulation, fixed-order CTA
//                              tree, then a fixed-order fold over chunks.
// Batched (spm_batch_*, many molecules per launch), node-major instead:
//   batch_ubar_max_kernel      per-molecule max |ubar| (fixed-point scale)
//   batch_scatter_kernel       w * ubar onto each state's 8 corner nodes of an
//                              adjoint grid, 64-bit fixed point: exact,
//                              order-independent integer sums
//   batch_adjoint_nodes_kernel atomics-free scatter by atom tiles: non-zero
//                              adjoint-grid nodes staged in shared memory, one
//                              thread per (atom, phase), pair-law derivatives
//                              at each node once (not once per touching state)
//   batch_fold_rows_kernel     fixed-order fold of the per-unit partials
#include "spm_internal.cuh"
#include "spm_fire.cuh"
#include "spm_batch.cuh"

namespace spm {
namespace {

constexpr int AG_THREADS = 128;
constexpr int AG_PER_THREAD = 8;
constexpr int AG_CHUNK = AG_THREADS * AG_PER_THREAD;
constexpr float R2SAFE = 1e-4f;
constexpr float COULOMB_CONST = 14.3996448915f;

struct Corners {
    int x[2], y[2], z[2];
    float ax, ay, az;
    bool ok;
};

// Both texels i[0], i[1] of a cell along one axis lie in the stored range [lo, lo + n).
__device__ __forceinline__ bool in_slab(const int* i, int lo, int n) {
    return (unsigned)(i[0] - lo) < (unsigned)n && (unsigned)(i[1] - lo) < (unsigned)n;
}

// Texel cell of a point (the same REPEAT/LINEAR addressing as interp_fe).
// Indices are the full grid's; SLAB: ok only if all eight texels are stored.
template <bool SLAB>
__device__ __forceinline__ Corners corners_of(const GridView& G, V3 p) {
    Corners C;
    const float u = __fmaf_rn(p.x, G.dA.x, __fmaf_rn(p.y, G.dA.y, __fmaf_rn(p.z, G.dA.z, G.dA.w)));
    const float v = __fmaf_rn(p.x, G.dB.x, __fmaf_rn(p.y, G.dB.y, __fmaf_rn(p.z, G.dB.z, G.dB.w)));
    const float w = __fmaf_rn(p.x, G.dC.x, __fmaf_rn(p.y, G.dC.y, __fmaf_rn(p.z, G.dC.z, G.dC.w)));
    C.ok = tex_axis(u, G.nx, C.x[0], C.x[1], C.ax);
    C.ok = tex_axis(v, G.ny, C.y[0], C.y[1], C.ay) && C.ok;
    C.ok = tex_axis(w, G.nz, C.z[0], C.z[1], C.az) && C.ok;
    if (SLAB)
        C.ok = C.ok && in_slab(C.x, G.x_lo, G.nx_slab) && in_slab(C.y, G.y_lo, G.ny_slab) &&
               in_slab(C.z, G.z_lo, G.nz_slab);
    return C;
}

// Stored node (x, y, z) (full-grid indices) of a full grid or of a batch slab
// (batch slabs hold G.stride float4 per node, its value first).
template <bool SLAB>
__device__ __forceinline__ float4 node_at(const GridView& G, int x, int y, int z) {
    if (!SLAB) return __ldg(G.g + ((size_t)z * G.ny + y) * G.nx + x);
    const size_t idx = ((size_t)(z - G.z_lo) * G.ny_slab + (y - G.y_lo)) * G.nx_slab + (x - G.x_lo);
    return __ldg(G.g + (size_t)G.stride * idx);
}

struct Sites {
    float qs[4];  // Qs[k]*COULOMB_CONST
    float qz[4];
};

__device__ __forceinline__ float4 add4(float4 p, float4 q) { return make_float4(p.x + q.x, p.y + q.y, p.z + q.z, p.w + q.w); }
__device__ __forceinline__ float4 sub4(float4 p, float4 q) { return make_float4(p.x - q.x, p.y - q.y, p.z - q.z, p.w - q.w); }
__device__ __forceinline__ float4 scale4(float4 p, float s) { return make_float4(p.x * s, p.y * s, p.z * s, p.w * s); }

// Two float4 texels from one 32-byte read-only load (p 32-byte aligned).
__device__ __forceinline__ void ld_texel_pair(const float4* p, float4& lo, float4& hi) {
    unsigned long long a0, a1, b0, b1;
    asm("ld.global.nc.v4.b64 {%0, %1, %2, %3}, [%4];" : "=l"(a0), "=l"(a1), "=l"(b0), "=l"(b1) : "l"(p));
    upk(a0, lo.x, lo.y);
    upk(a1, lo.z, lo.w);
    upk(b0, hi.x, hi.y);
    upk(b1, hi.z, hi.w);
}

// The eight texels f[k][j][i] of cell C (corner (x_i, y_j, z_k)).  Batch slabs
// in the x-pair layout (stride 2) hold a node's +x neighbour after it, so each
// (y, z) row of the cell is one 32-byte load; xz-quads (stride 4) hold the
// (x, z), (x+1, z), (x, z+1), (x+1, z+1) texels of a node together, two
// 32-byte loads per y row.  Full grids read the eight texels one by one.
template <bool SLAB>
__device__ __forceinline__ void load_cell_texels(const GridView& G, const Corners& C, float4 (&f)[2][2][2]) {
    if (SLAB && G.stride == 2) {
#pragma unroll
        for (int k = 0; k < 2; k++)
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const size_t idx = ((size_t)(C.z[k] - G.z_lo) * G.ny_slab + (C.y[j] - G.y_lo)) * G.nx_slab +
                                   (C.x[0] - G.x_lo);
                ld_texel_pair(G.g + 2 * idx, f[k][j][0], f[k][j][1]);
            }
    } else if (SLAB && G.stride == 4) {
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const size_t idx = ((size_t)(C.z[0] - G.z_lo) * G.ny_slab + (C.y[j] - G.y_lo)) * G.nx_slab +
                               (C.x[0] - G.x_lo);
            ld_texel_pair(G.g + 4 * idx, f[0][j][0], f[0][j][1]);
            ld_texel_pair(G.g + 4 * idx + 2, f[1][j][0], f[1][j][1]);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 2; k++)
#pragma unroll
            for (int j = 0; j < 2; j++)
#pragma unroll
                for (int i = 0; i < 2; i++) f[k][j][i] = node_at<SLAB>(G, C.x[i], C.y[j], C.z[k]);
    }
}

// Adjoint of one state: p4 = the stroke's start point, iz = its z-step,
// pp = stored PP, u = dL/dFEs of the state; writes ubar, dk (unless dk_o is null), diag.
template <bool SLAB>
__device__ __forceinline__ void state_adjoint(const GridView& G, const spm_scan_params& P, float4 p4, int iz,
                                              float4 pp, float4 u, float4* ubar_o, float4* dk_o, float4* diag_o) {
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    auto fail = [&](float res, float lmin, float cond, float status) {
        *ubar_o = zero;
        if (dk_o) *dk_o = zero;
        *diag_o = make_float4(res, lmin, cond, status);
    };
    if (!(isfinite(pp.x) && isfinite(pp.y) && isfinite(pp.z) && isfinite(pp.w) && isfinite(u.x) && isfinite(u.y) &&
          isfinite(u.z) && isfinite(u.w))) { fail(0.f, 0.f, 0.f, 2.f); return; }
    if (pp.w <= 0.f) { fail(0.f, 0.f, 0.f, 1.f); return; }
    const V3 a = mk3(P.tipA[0], P.tipA[1], P.tipA[2]);
    const V3 b = mk3(P.tipB[0], P.tipB[1], P.tipB[2]);
    const V3 c = mk3(P.tipC[0], P.tipC[1], P.tipC[2]);
    const V3 tip = mk3(p4.x + c.x * P.tipC[3] * (float)iz, p4.y + c.y * P.tipC[3] * (float)iz,
                       p4.z + c.z * P.tipC[3] * (float)iz);
    const V3 q = mk3(pp.x, pp.y, pp.z);
    const Corners C = corners_of<SLAB>(G, q);
    if (!C.ok) { fail(0.f, 0.f, 0.f, 2.f); return; }
    // the identity probe frame of z-strokes and axis-aligned grids drop the rotations and the zero
    // terms of the coordinate derivatives (exact: only the sign of a zero can differ)
    const bool ident = a.x == 1.f && a.y == 0.f && a.z == 0.f && b.x == 0.f && b.y == 1.f && b.z == 0.f &&
                       c.x == 0.f && c.y == 0.f && c.z == 1.f;
    const bool axis = G.dA.y == 0.f && G.dA.z == 0.f && G.dB.x == 0.f && G.dB.z == 0.f && G.dC.x == 0.f &&
                      G.dC.y == 0.f;
    // the cell's texels f[k][j][i] (x-pair / xz-quad slabs: one 32-byte load per x-pair)
    float4 f[2][2][2];
    load_cell_texels<SLAB>(G, C, f);
    bool capped = false;
#pragma unroll
    for (int k = 0; k < 2; k++)
#pragma unroll
        for (int j = 0; j < 2; j++)
            capped |= fabsf(f[k][j][0].w) >= 99.9999f || fabsf(f[k][j][1].w) >= 99.9999f;
    // value and texel-coordinate derivatives of the 4 channels, separably: lerps along x, then y,
    // then z, carrying the differences along the axes already passed
    const float ax = C.ax, ay = C.ay, az = C.az, mx = 1.f - ax, my = 1.f - ay, mz = 1.f - az;
    float4 cx[2][2], ex[2][2];
#pragma unroll
    for (int k = 0; k < 2; k++)
#pragma unroll
        for (int j = 0; j < 2; j++) {
            cx[k][j] = add4(scale4(f[k][j][0], mx), scale4(f[k][j][1], ax));
            ex[k][j] = sub4(f[k][j][1], f[k][j][0]);
        }
    float4 cy[2], exy[2], ey[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        cy[k] = add4(scale4(cx[k][0], my), scale4(cx[k][1], ay));
        exy[k] = add4(scale4(ex[k][0], my), scale4(ex[k][1], ay));
        ey[k] = sub4(cx[k][1], cx[k][0]);
    }
    const float4 v4 = add4(scale4(cy[0], mz), scale4(cy[1], az));
    const float4 dx4 = add4(scale4(exy[0], mz), scale4(exy[1], az));
    const float4 dy4 = add4(scale4(ey[0], mz), scale4(ey[1], az));
    const float4 dz4 = sub4(cy[1], cy[0]);
    const float val[4] = {v4.x, v4.y, v4.z, v4.w}, dx[4] = {dx4.x, dx4.y, dx4.z, dx4.w};
    const float dy[4] = {dy4.x, dy4.y, dy4.z, dy4.w}, dz[4] = {dz4.x, dz4.y, dz4.z, dz4.w};
    // dt_axis/dq_m = n_axis * dinv_axis[m]
    const float ta[3] = {G.nx * G.dA.x, G.nx * G.dA.y, G.nx * G.dA.z};
    const float tb[3] = {G.ny * G.dB.x, G.ny * G.dB.y, G.ny * G.dB.z};
    const float tc[3] = {G.nz * G.dC.x, G.nz * G.dC.y, G.nz * G.dC.z};
    float Jg[3][3], gE[3];
    if (axis) {
#pragma unroll
        for (int ch = 0; ch < 3; ch++) {
            Jg[ch][0] = dx[ch] * ta[0];
            Jg[ch][1] = dy[ch] * tb[1];
            Jg[ch][2] = dz[ch] * tc[2];
        }
        gE[0] = dx[3] * ta[0];
        gE[1] = dy[3] * tb[1];
        gE[2] = dz[3] * tc[2];
    } else {
        for (int m = 0; m < 3; m++) {
            for (int ch = 0; ch < 3; ch++) Jg[ch][m] = dx[ch] * ta[m] + dy[ch] * tb[m] + dz[ch] * tc[m];
            gE[m] = dx[3] * ta[m] + dy[3] * tb[m] + dz[3] * tc[m];
        }
    }
    // tip spring in the tip frame
    const float4 kk = make_float4(P.stiffness[0], P.stiffness[1], P.stiffness[2], P.stiffness[3]);
    const float4 d0 = make_float4(P.dpos0[0], P.dpos0[1], P.dpos0[2], P.dpos0[3]);
    const V3 dl = ident ? sub3(q, tip) : rotmat(sub3(q, tip), a, b, c);
    const V3 ft = ident ? tip_force(dl, kk, d0) : rotmatT(tip_force(dl, kk, d0), a, b, c);
    const float surf = P.surfFF[0];
    const V3 Gv = mk3(val[0] + ft.x + c.x * surf, val[1] + ft.y + c.y * surf, val[2] + ft.z + c.z * surf);
    const float resid = sqrtf(Gv.x * Gv.x + Gv.y * Gv.y + Gv.z * Gv.z);
    if (resid >= 5e-4f) { fail(resid, 0.f, 0.f, 1.f); return; }
    if (capped) { fail(resid, 0.f, 0.f, 5.f); return; }
    float r = sqrtf(dl.x * dl.x + dl.y * dl.y + dl.z * dl.z);
    r = fmaxf(r, 1e-10f);
    const float phi = (kk.w == 0.f) ? 0.f : kk.w * (1.f - d0.w / r);
    const float beta = (kk.w == 0.f) ? 0.f : kk.w * d0.w / (r * r * r);
    const float Jt[3][3] = {{kk.x + phi + beta * dl.x * dl.x, beta * dl.x * dl.y, beta * dl.x * dl.z},
                            {beta * dl.y * dl.x, kk.y + phi + beta * dl.y * dl.y, beta * dl.y * dl.z},
                            {beta * dl.z * dl.x, beta * dl.z * dl.y, kk.z + phi + beta * dl.z * dl.z}};
    const float R[3][3] = {{a.x, a.y, a.z}, {b.x, b.y, b.z}, {c.x, c.y, c.z}};
    float J[3][3];
    if (ident) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) J[i][j] = Jg[i][j] + Jt[i][j];
    } else {
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                float s = Jg[i][j];
                for (int m = 0; m < 3; m++)
                    for (int n = 0; n < 3; n++) s += R[m][i] * Jt[m][n] * R[n][j];
                J[i][j] = s;
            }
    }
    // b = Jg^T R^T u_xyz + gE u_w
    const V3 uw = ident ? mk3(u.x, u.y, u.z) : rotmatT(mk3(u.x, u.y, u.z), a, b, c);
    const float uv[3] = {uw.x, uw.y, uw.z};
    float bv[3];
    for (int m = 0; m < 3; m++) bv[m] = Jg[0][m] * uv[0] + Jg[1][m] * uv[1] + Jg[2][m] * uv[2] + gE[m] * u.w;
    // J^T lambda = b via the adjugate: (J^T)^-1 = adj(J)^T / det(J)
    float A[3][3];  // A = adj(J): A[i][j] = cofactor(J)[j][i]
    A[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    A[0][1] = J[0][2] * J[2][1] - J[0][1] * J[2][2];
    A[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
    A[1][0] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    A[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
    A[1][2] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
    A[2][0] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    A[2][1] = J[0][1] * J[2][0] - J[0][0] * J[2][1];
    A[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    const float det = J[0][0] * A[0][0] + J[0][1] * A[1][0] + J[0][2] * A[2][0];
    const float scale = fmaxf(fmaxf(fabsf(J[0][0]), fmaxf(fabsf(J[1][1]), fabsf(J[2][2]))), 1e-20f);
    if (!(fabsf(det) >= 1e-18f * scale * scale * scale)) { fail(resid, 0.f, 0.f, 4.f); return; }
    const float id = 1.f / det;
    float lam[3];
    for (int i = 0; i < 3; i++) lam[i] = (A[0][i] * bv[0] + A[1][i] * bv[1] + A[2][i] * bv[2]) * id;
    if (!(isfinite(lam[0]) && isfinite(lam[1]) && isfinite(lam[2]))) { fail(resid, 0.f, 0.f, 2.f); return; }
    // stability: smallest eigenvalue of the symmetric part of -J (closed form for 3x3)
    const float s00 = -J[0][0], s11 = -J[1][1], s22 = -J[2][2];
    const float s01 = -0.5f * (J[0][1] + J[1][0]), s02 = -0.5f * (J[0][2] + J[2][0]), s12 = -0.5f * (J[1][2] + J[2][1]);
    float lmin;
    {
        // (one reciprocal of p and one sincos: cos(phi + 2pi/3) = -cos(phi)/2 - sin(phi) sqrt(3)/2)
        const float third = 1.f / 3.f;
        const float p1 = s01 * s01 + s02 * s02 + s12 * s12;
        const float qm = (s00 + s11 + s22) * third;
        const float p2 = (s00 - qm) * (s00 - qm) + (s11 - qm) * (s11 - qm) + (s22 - qm) * (s22 - qm) + 2.f * p1;
        const float pp2 = sqrtf(p2 * (1.f / 6.f));
        if (pp2 < 1e-20f) {
            lmin = qm;
        } else {
            const float ip = 1.f / pp2;
            const float b00 = (s00 - qm) * ip, b11 = (s11 - qm) * ip, b22 = (s22 - qm) * ip;
            const float b01 = s01 * ip, b02 = s02 * ip, b12 = s12 * ip;
            const float detB = b00 * (b11 * b22 - b12 * b12) - b01 * (b01 * b22 - b12 * b02) +
                               b02 * (b01 * b12 - b11 * b02);
            const float phi3 = acosf(fmaxf(-1.f, fminf(1.f, 0.5f * detB))) * third;
            float sn, cs;
            sincosf(phi3, &sn, &cs);
            const float e1 = qm + 2.f * pp2 * cs;
            const float e3 = qm + 2.f * pp2 * (-0.5f * cs - 0.8660254037844386f * sn);
            lmin = fminf(e1, fminf(3.f * qm - e1 - e3, e3));
        }
    }
    if (lmin <= 1e-5f) { fail(resid, lmin, 0.f, 3.f); return; }
    float jinf = 0.f, ainf = 0.f;
    for (int i = 0; i < 3; i++) {
        jinf = fmaxf(jinf, fabsf(J[i][0]) + fabsf(J[i][1]) + fabsf(J[i][2]));
        ainf = fmaxf(ainf, fabsf(A[i][0]) + fabsf(A[i][1]) + fabsf(A[i][2]));
    }
    const float cond = jinf * ainf / fabsf(det);
    if (!(cond < 1e6f)) { fail(resid, lmin, cond, 4.f); return; }
    *ubar_o = make_float4(uv[0] - lam[0], uv[1] - lam[1], uv[2] - lam[2], u.w);
    // spring-parameter terms  -lambda . R^T dg/dk   (lambda in the tip frame: R lambda)
    const V3 lt = ident ? mk3(lam[0], lam[1], lam[2]) : rotmat(mk3(lam[0], lam[1], lam[2]), a, b, c);
    const float rw = (r - d0.w) / r;
    if (dk_o)
        *dk_o = make_float4(-lt.x * (dl.x - d0.x), -lt.y * (dl.y - d0.y), -lt.z * (dl.z - d0.z),
                            -(lt.x * dl.x + lt.y * dl.y + lt.z * dl.z) * rw);
    *diag_o = make_float4(resid, lmin, cond, 0.f);
}

__global__ void __launch_bounds__(AG_THREADS)
adjoint_grid_state_kernel(GridView G, const float4* __restrict__ pts, int n_scan, spm_scan_params P,
                          const float4* __restrict__ PPs, const float4* __restrict__ dL, float4* __restrict__ ubar,
                          float4* __restrict__ dk, float4* __restrict__ diag) {
    const long long st = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (st >= (long long)n_scan * P.nz) return;
    const int iscan = (int)(st / P.nz), iz = (int)(st % P.nz);
    state_adjoint<false>(G, P, pts[iscan], iz, PPs[st], dL[st], ubar + st, dk + st, diag + st);
}

struct NodeGeom {
    float4 p0, dA, dB, dC;
};

// Pair-law parameter derivatives at one grid node, contracted with the
// node's adjoint weights (uF: force channels, uE: energy channel).
template <int KIND>
__device__ __forceinline__ void pair_grad(V3 node, float4 at, float p1, float p2, float p3, const Sites& S, V3 uF,
                                          float uE, double* acc) {
    const V3 dp = mk3(node.x - at.x, node.y - at.y, node.z - at.z);
    const float r2 = dp.x * dp.x + dp.y * dp.y + dp.z * dp.z + R2SAFE;
    const float du = dp.x * uF.x + dp.y * uF.y + dp.z * uF.z;
    float s, dsdr2, E_dummy;
    float g_p1, g_p2;
    if (KIND == SPM_KIND_LJ) {
        const float c6 = p1, c12 = p2;
        const float ir2 = 1.f / r2;
        const float ir6 = ir2 * ir2 * ir2;
        const float ir8 = ir6 * ir2;
        const float ir14 = ir8 * ir6;
        s = 12.f * c12 * ir14 - 6.f * c6 * ir8;
        dsdr2 = -84.f * c12 * ir14 * ir2 + 24.f * c6 * ir8 * ir2;
        g_p1 = du * (-6.f * ir8) + uE * (-ir6);           // c6
        g_p2 = du * (12.f * ir14) + uE * (ir6 * ir6);     // c12
        E_dummy = 0.f;
    } else {
        const float R0 = p1, E0 = p2, K = p3;
        const float r = sqrtf(r2);
        const float e = expf(K * (r - R0));
        const float Ep = 2.f * K * E0 * e * (e - 1.f);
        const float Epp = 2.f * K * K * E0 * e * (2.f * e - 1.f);
        s = -Ep / r;
        dsdr2 = -(Epp / r - Ep / (r * r)) / (2.f * r);
        g_p1 = du * (Epp / r) + uE * (-Ep);                                  // R0
        g_p2 = du * (-2.f * K * e * (e - 1.f) / r) + uE * (e * (e - 2.f));    // E0
        E_dummy = 0.f;
    }
    (void)E_dummy;
    // d/da of (uF.F + uE E) = -(s uF + 2 s' (dp.uF) dp) + uE F,   F = s dp
    float gx = -(s * uF.x + 2.f * dsdr2 * du * dp.x) + uE * s * dp.x;
    float gy = -(s * uF.y + 2.f * dsdr2 * du * dp.y) + uE * s * dp.y;
    float gz = -(s * uF.z + 2.f * dsdr2 * du * dp.z) + uE * s * dp.z;
    float gq = 0.f;
    for (int k = 0; k < 4; k++) {
        if (S.qs[k] == 0.f) continue;
        const V3 dk = mk3(dp.x, dp.y, dp.z + S.qz[k]);
        const float rk2 = dk.x * dk.x + dk.y * dk.y + dk.z * dk.z + R2SAFE;
        const float irk = rsqrtf(rk2);
        const float irk3 = irk * irk * irk;
        const float sk = S.qs[k] * at.w * irk3;
        const float dsk = -1.5f * sk / rk2;
        const float duk = dk.x * uF.x + dk.y * uF.y + dk.z * uF.z;
        gx += -(sk * uF.x + 2.f * dsk * duk * dk.x) + uE * sk * dk.x;
        gy += -(sk * uF.y + 2.f * dsk * duk * dk.y) + uE * sk * dk.y;
        gz += -(sk * uF.z + 2.f * dsk * duk * dk.z) + uE * sk * dk.z;
        gq += duk * (S.qs[k] * irk3) + uE * (S.qs[k] * irk);
    }
    acc[0] += gx;
    acc[1] += gy;
    acc[2] += gz;
    acc[3] += g_p1;
    acc[4] += g_p2;
    acc[5] += gq;
}

// Sum over states [s_begin, s_end) (thread-strided) of one atom's pair-law
// derivatives at each state's eight corner nodes, weighted by w * ubar.
template <int KIND, bool SLAB>
__device__ __forceinline__ void gather_atom(float4 at, float p1, float p2, float p3, const Sites& S,
                                            const NodeGeom& NG, const GridView& G, const float4* __restrict__ PPs,
                                            const float4* __restrict__ ubar, long long s_begin, long long s_end,
                                            double* acc) {
    for (long long st = s_begin + threadIdx.x; st < s_end; st += blockDim.x) {
        const float4 ub = __ldg(ubar + st);
        if (ub.x == 0.f && ub.y == 0.f && ub.z == 0.f && ub.w == 0.f) continue;
        const float4 pp = __ldg(PPs + st);
        const Corners C = corners_of<SLAB>(G, mk3(pp.x, pp.y, pp.z));
        if (!C.ok) continue;
        for (int k = 0; k < 2; k++)
            for (int j = 0; j < 2; j++)
                for (int i = 0; i < 2; i++) {
                    const float w = (i ? C.ax : 1.f - C.ax) * (j ? C.ay : 1.f - C.ay) * (k ? C.az : 1.f - C.az);
                    if (w == 0.f) continue;
                    const int ix = C.x[i], iy = C.y[j], iz = C.z[k];
                    const V3 node = mk3(NG.p0.x + NG.dA.x * ix + NG.dB.x * iy + NG.dC.x * iz,
                                        NG.p0.y + NG.dA.y * ix + NG.dB.y * iy + NG.dC.y * iz,
                                        NG.p0.z + NG.dA.z * ix + NG.dB.z * iy + NG.dC.z * iz);
                    pair_grad<KIND>(node, at, p1, p2, p3, S, mk3(w * ub.x, w * ub.y, w * ub.z), w * ub.w, acc);
                }
    }
}

// Fixed-order CTA tree of the six accumulators; thread 0..5 write out[0..5].
__device__ __forceinline__ void cta_sum6(double* acc, double (*red)[AG_THREADS], double* out) {
#pragma unroll
    for (int c6 = 0; c6 < 6; c6++) red[c6][threadIdx.x] = acc[c6];
    __syncthreads();
    for (int s = AG_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
#pragma unroll
            for (int c6 = 0; c6 < 6; c6++) red[c6][threadIdx.x] += red[c6][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 6) out[threadIdx.x] = red[threadIdx.x][0];
}

template <int KIND>
__global__ void __launch_bounds__(AG_THREADS)
adjoint_grid_atoms_kernel(int na, const float4* __restrict__ atoms, const float* __restrict__ params, int pstride,
                          Sites S, NodeGeom NG, GridView G, const float4* __restrict__ PPs,
                          const float4* __restrict__ ubar, long long n_state, double* __restrict__ partial) {
    __shared__ double red[6][AG_THREADS];
    const int ia = blockIdx.y;
    const float4 at = __ldg(atoms + ia);
    const float* pr = params + (size_t)ia * pstride;
    const float p1 = __ldg(pr + 0), p2 = __ldg(pr + 1), p3 = (pstride > 2) ? __ldg(pr + 2) : 0.f;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const long long s0 = (long long)blockIdx.x * AG_CHUNK;
    const long long s1 = s0 + AG_CHUNK < n_state ? s0 + AG_CHUNK : n_state;
    gather_atom<KIND, false>(at, p1, p2, p3, S, NG, G, PPs, ubar, s0, s1, acc);
    cta_sum6(acc, red, partial + ((size_t)ia * gridDim.x + blockIdx.x) * 6);
}

// out[r*cols + c] = sum over chunks of in[(r*chunks + ch)*cols + c], fixed order.
__global__ void __launch_bounds__(256)
fold_chunks_kernel(const double* __restrict__ in, int chunks, int cols, double* __restrict__ out) {
    __shared__ double red[256];
    const int r = blockIdx.x, c = blockIdx.y;
    double acc = 0.0;
    for (int ch = threadIdx.x; ch < chunks; ch += 256) acc += in[((size_t)r * chunks + ch) * cols + c];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[(size_t)r * cols + c] = red[0];
}

// Per-chunk sums of float4 rows (spring-gradient terms) in FP64.
__global__ void __launch_bounds__(256)
sum_rows_kernel(const float4* __restrict__ rows, long long n, double* __restrict__ partial) {
    __shared__ double red[4][256];
    double acc[4] = {0, 0, 0, 0};
    const long long base = (long long)blockIdx.x * 256 * 8;
    for (int t = 0; t < 8; t++) {
        const long long i = base + (long long)t * 256 + threadIdx.x;
        if (i < n) {
            const float4 v = __ldg(rows + i);
            acc[0] += v.x; acc[1] += v.y; acc[2] += v.z; acc[3] += v.w;
        }
    }
    for (int c = 0; c < 4; c++) red[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int c = 0; c < 4; c++) red[c][threadIdx.x] += red[c][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 4) partial[(size_t)blockIdx.x * 4 + threadIdx.x] = red[threadIdx.x][0];
}

GridView view_of(const float* grid, int nx, int ny, int nz, const spm_scan_params* p) {
    GridView G;
    G.g = reinterpret_cast<const float4*>(grid);
    G.nx = nx; G.ny = ny; G.nz = nz;
    G.x_lo = 0; G.nx_slab = nx; G.y_lo = 0; G.ny_slab = ny; G.z_lo = 0; G.nz_slab = nz; G.stride = 1;
    G.dA = make_float4(p->dinvA[0], p->dinvA[1], p->dinvA[2], p->dinvA[3]);
    G.dB = make_float4(p->dinvB[0], p->dinvB[1], p->dinvB[2], p->dinvB[3]);
    G.dC = make_float4(p->dinvC[0], p->dinvC[1], p->dinvC[2], p->dinvC[3]);
    return G;
}

long long n_chunks(long long n_state) { return n_state > 0 ? (n_state + AG_CHUNK - 1) / AG_CHUNK : 1; }
long long n_rowblocks(long long n_state) { return n_state > 0 ? (n_state + 2047) / 2048 : 1; }

// ---- batched ----------------------------------------------------------------
// At most 85 registers (72 used, 7 CTAs per SM): the kernel waits on its
// texel loads, so resident warps pay, but the separable cell arithmetic keeps
// all eight texels live and spilled at 64 registers (3.41 -> 3.00 ms on the
// 64-molecule fit; 4.14 ms before the x-pair loads, the separable lerps and the
// identity-frame path).
//
// umax, box (optional, zeroed before the launch): the per-molecule max |ubar| and touched box of
// batch_ubar_max_kernel, from each state's ubar as it is written -- warp maxima (redux) into the
// molecule's atomics, per lane where a warp spans two molecules.  Maxima are order-free.
__global__ void __launch_bounds__(AG_THREADS, 6)
batch_adjoint_state_kernel(int n_mol, const spm_batch_mol* __restrict__ mols, long long n_states, int stride,
                           const float* __restrict__ grid, const float4* __restrict__ pts, spm_scan_params P,
                           const float4* __restrict__ PPs, const float4* __restrict__ dL, float4* __restrict__ ubar,
                           float4* __restrict__ dk, float4* __restrict__ diag, unsigned* __restrict__ umax,
                           int* __restrict__ box) {
    const long long st = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = st < n_states;
    int m = 0;
    float v = 0.f;
    int b[4] = {0, 0, 0, 0};
    if (in) {
        m = SPM_MOL_BY(state_off, mols, n_mol, st);
        const spm_batch_mol* D = mols + m;
        const long long ls = st - D->state_off;
        const int nz = D->nz_steps;
        int iscan, iz;
        if (ls < (1LL << 32)) {  // 32-bit division when it fits
            iscan = (int)((unsigned)ls / (unsigned)nz);
            iz = (int)((unsigned)ls - (unsigned)iscan * (unsigned)nz);
        } else {
            iscan = (int)(ls / nz);
            iz = (int)(ls % nz);
        }
        const float4 pp = PPs[st];
        state_adjoint<true>(slab_view(*D, grid, stride), P, pts[D->pix_off + iscan], iz, pp, dL[st], ubar + st,
                            dk ? dk + st : nullptr, diag + st);
        if (umax) {
            const float4 u = ubar[st];  // this thread's own store
            v = fmaxf(fmaxf(fabsf(u.x), fabsf(u.y)), fmaxf(fabsf(u.z), fabsf(u.w)));
            if (!(u.x == 0.f && u.y == 0.f && u.z == 0.f && u.w == 0.f)) {  // the scatter's test
                const GridView G = slab_view(*D, nullptr);
                const Corners C = corners_of<true>(G, mk3(pp.x, pp.y, pp.z));
                if (C.ok) {
#pragma unroll
                    for (int k = 0; k < 2; k++) {
                        b[0] = max(b[0], G.ny_slab - 1 - (C.y[k] - G.y_lo));
                        b[1] = max(b[1], C.y[k] - G.y_lo + 1);
                        b[2] = max(b[2], G.nz_slab - 1 - (C.z[k] - G.z_lo));
                        b[3] = max(b[3], C.z[k] - G.z_lo + 1);
                    }
                }
            }
        }
    }
    if (umax) {  // launch-uniform: CTA maxima, one atomic per value and CTA when the CTA has one molecule
        __shared__ int s_red[AG_THREADS / 32][5];
        __shared__ int s_m[AG_THREADS / 32];
        const unsigned FULL = 0xffffffffu;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const int m0 = __shfl_sync(FULL, m, 0);
        const bool one = __all_sync(FULL, !in || m == m0);
        const int wv = (int)__reduce_max_sync(FULL, __float_as_uint(v));  // v >= 0: bit order = value order
        int wb[4];
#pragma unroll
        for (int k = 0; k < 4; k++) wb[k] = __reduce_max_sync(FULL, b[k]);
        if (lane == 0) {
            s_m[warp] = one ? m0 : -1;  // -1: the warp spans two molecules
            s_red[warp][0] = wv;
#pragma unroll
            for (int k = 0; k < 4; k++) s_red[warp][k + 1] = wb[k];
        }
        __syncthreads();
        bool cta_one = true;
#pragma unroll
        for (int w = 0; w < AG_THREADS / 32; w++) cta_one = cta_one && s_m[w] == s_m[0] && s_m[w] >= 0;
        if (cta_one) {
            if (threadIdx.x < 5) {
                int val = 0;
#pragma unroll
                for (int w = 0; w < AG_THREADS / 32; w++) val = max(val, s_red[w][threadIdx.x]);
                // the umax word holds a finite non-negative float's bits (< 2^31): int order = value order
                int* dst = threadIdx.x == 0 ? reinterpret_cast<int*>(umax + s_m[0]) : box + 4 * s_m[0] + (threadIdx.x - 1);
                if (val > 0) atomicMax(dst, val);
            }
        } else if (in) {  // the CTA at a molecule boundary: per lane
            if (v > 0.f) atomicMax(umax + m, __float_as_uint(v));
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (b[k] > 0) atomicMax(box + 4 * m + k, b[k]);
        }
    }
}

// ---- node-major adjoint through the grid build (batched) -------------------
// Adjoint grid: per slab node four int64 fixed-point sums (Fx, Fy, Fz, E
// weights) at the grid's float4 offsets x 4.  A molecule's scale is 2^(42-e)
// with max|ubar| < 2^e: every contribution |w*ubar| <= 2^42 units and up to
// 2^20 contributions per node stay below 2^62.
__device__ __forceinline__ int scale_exp(unsigned umax_bits) {
    const int eb = (int)((umax_bits >> 23) & 0xffu);
    return (eb > 0 ? eb : 1) - 126;  // max|ubar| < 2^e
}
__device__ __forceinline__ double pow2(int k) { return __longlong_as_double((long long)(1023 + k) << 52); }

constexpr unsigned long long ADJ_CLEAN = 0x4e41454c434d5053ull;  // marker base: the adjoint grid is all zero
constexpr unsigned long long ADJ_DIRTY = 1ull;

// The clear marker of one scratch buffer and layout: ADJ_CLEAN mixed with the buffer's address and
// the layout's size and molecule count, so that memory which held a scratch of another address or
// layout -- whose marker slot may sit exactly where this layout's does -- does not carry it.
unsigned long long adj_clean_token(const void* scratch, long long total, int n_mol) {
    const unsigned long long t = ADJ_CLEAN ^ (reinterpret_cast<uintptr_t>(scratch) * 0x9E3779B97F4A7C15ull) ^
                                 ((unsigned long long)total * 0xC2B2AE3D27D4EB4Full) ^
                                 ((unsigned long long)n_mol << 40);
    return t == ADJ_DIRTY ? t ^ 2ull : t;
}

// Zeroes the fixed-point adjoint grid (n2 16-byte pairs) unless its marker
// says it is clear.  The node kernel zeroes every node it reads, so after a
// completed call the grid is clear again; only a first use, or a call that
// stopped between the scatter and the node kernel, leaves work here.
__global__ void __launch_bounds__(256)
adj_clear_kernel(ulonglong2* __restrict__ gq, long long n2, const unsigned long long* __restrict__ mark,
                 unsigned long long clean) {
    if (*mark == clean) return;
    for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < n2; i += (long long)gridDim.x * 256)
        gq[i] = make_ulonglong2(0ull, 0ull);
}

// UM_CHUNKS consecutive 256-state chunks per CTA: per-molecule max |ubar| (as
// float bits; order-free) and the bounding box of the slab rows and layers the
// scatter will touch, box[4m..4m+3] = max of (ny_slab-1-yl, yl+1,
// nz_slab-1-zl, zl+1) over the cell corners of every state with a non-zero
// ubar (all zero: none); yl, zl are slab rows and layers.  The CTA searches
// the first chunk's molecule once and steps to the next ones; its maxima are
// flushed to the molecule's atomics whenever the molecule changes.
constexpr int UM_CHUNKS = 4;

__global__ void __launch_bounds__(256)
batch_ubar_max_kernel(int n_mol, long long n_chunks, const spm_batch_mol* __restrict__ mols,
                      const float4* __restrict__ ubar, const float4* __restrict__ PPs, unsigned* __restrict__ umax,
                      int* __restrict__ box) {
    __shared__ float s_m[8];
    __shared__ int s_b[4][8];
    float v = 0.f;
    int b[4] = {0, 0, 0, 0};
    // CTA-uniform: the block's maxima of molecule m into its atomics; v and b restart at zero
    auto flush = [&](int m) {
        for (int o = 16; o > 0; o >>= 1) {
            v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
#pragma unroll
            for (int k = 0; k < 4; k++) b[k] = max(b[k], __shfl_xor_sync(0xffffffffu, b[k], o));
        }
        if ((threadIdx.x & 31) == 0) {
            s_m[threadIdx.x >> 5] = v;
#pragma unroll
            for (int k = 0; k < 4; k++) s_b[k][threadIdx.x >> 5] = b[k];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            float w = s_m[0];
            for (int k = 1; k < 8; k++) w = fmaxf(w, s_m[k]);
            if (w > 0.f) atomicMax(umax + m, __float_as_uint(w));
        }
        if (threadIdx.x < 4) {
            int w = s_b[threadIdx.x][0];
            for (int k = 1; k < 8; k++) w = max(w, s_b[threadIdx.x][k]);
            if (w > 0) atomicMax(box + 4 * m + threadIdx.x, w);
        }
        __syncthreads();
        v = 0.f;
#pragma unroll
        for (int k = 0; k < 4; k++) b[k] = 0;
    };
    const long long c0 = (long long)blockIdx.x * UM_CHUNKS;
    int m = SPM_MOL_BY(chunk_off, mols, n_mol, c0);
    for (int q = 0; q < UM_CHUNKS; q++) {
        const long long ch = c0 + q;
        if (ch >= n_chunks) break;
        const int mq = SPM_MOL_STEP(chunk_off, mols, n_mol, m, ch);
        if (mq != m) {
            flush(m);
            m = mq;
        }
        const spm_batch_mol* D = mols + m;
        const long long nst = (long long)D->n_scan * D->nz_steps;
        const long long ls = (ch - D->chunk_off) * 256 + threadIdx.x;
        if (ls < nst) {
            const float4 u = __ldg(ubar + D->state_off + ls);
            v = fmaxf(v, fmaxf(fmaxf(fabsf(u.x), fabsf(u.y)), fmaxf(fabsf(u.z), fabsf(u.w))));
            if (!(u.x == 0.f && u.y == 0.f && u.z == 0.f && u.w == 0.f)) {  // the scatter's test
                const GridView G = slab_view(*D, nullptr);
                const float4 pp = __ldg(PPs + D->state_off + ls);
                const Corners C = corners_of<true>(G, mk3(pp.x, pp.y, pp.z));
                if (C.ok) {
#pragma unroll
                    for (int k = 0; k < 2; k++) {
                        b[0] = max(b[0], G.ny_slab - 1 - (C.y[k] - G.y_lo));
                        b[1] = max(b[1], C.y[k] - G.y_lo + 1);
                        b[2] = max(b[2], G.nz_slab - 1 - (C.z[k] - G.z_lo));
                        b[3] = max(b[3], C.z[k] - G.z_lo + 1);
                    }
                }
            }
        }
    }
    flush(m);
}

// Thread per state: w * ubar onto the eight corner nodes (exact integer sums).  Block 0 marks the
// adjoint grid dirty until the node kernel has cleared it again.
// Consecutive lanes are consecutive z-steps of a stroke; when lane l+1's cell
// sits one layer below lane l's in the same (x,y) cell, lane l+1's upper
// layer is lane l's lower layer: lane l adds those four corners' sums to its
// own (integers: exact) and lane l+1 skips them, halving the atomics of a
// stroke.
//
// AGG (spm_batch_shape.adj_agg = 1): the CTA's 256 states -- a few neighbouring strokes -- first add
// their corner sums into a shared-memory table keyed by the adjoint-grid offset (open addressing,
// AGG_PROBES probes; a corner that finds no slot goes to global memory directly), then each table
// entry is added to the global grid once per channel.  Integer sums: the same bits either way.
constexpr int AGG_SLOTS = 2048;
constexpr int AGG_PROBES = 8;
constexpr unsigned long long AGG_EMPTY = ~0ull;

template <bool AGG>
__global__ void __launch_bounds__(256)
batch_scatter_kernel(int n_mol, const spm_batch_mol* __restrict__ mols, long long n_states,
                     const float4* __restrict__ PPs, const float4* __restrict__ ubar, const unsigned* __restrict__ umax,
                     unsigned long long* __restrict__ gq, unsigned long long* __restrict__ mark) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *mark = ADJ_DIRTY;  // the adjoint grid is written from here on
    extern __shared__ unsigned long long s_agg[];  // AGG: keys[AGG_SLOTS], then values[AGG_SLOTS][4]
    unsigned long long* s_key = s_agg;
    unsigned long long* s_val = s_agg + AGG_SLOTS;
    if constexpr (AGG) {
        for (int i = threadIdx.x; i < AGG_SLOTS; i += blockDim.x) s_key[i] = AGG_EMPTY;
        for (int i = threadIdx.x; i < 4 * AGG_SLOTS; i += blockDim.x) s_val[i] = 0ull;
        __syncthreads();
    }
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long st = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float4 ub = make_float4(0.f, 0.f, 0.f, 0.f);
    if (st < n_states) ub = __ldg(ubar + st);
    bool valid = !(ub.x == 0.f && ub.y == 0.f && ub.z == 0.f && ub.w == 0.f);
    Corners C = {{0, 0}, {0, 0}, {0, 0}, 0.f, 0.f, 0.f, false};
    long long stroke = -1;
    int nxs = 0, nys = 0, x_lo = 0, y_lo = 0, z_lo = 0;
    unsigned long long* base = gq;
    double scale = 0.0;
    if (valid) {
        const int m = SPM_MOL_BY(state_off, mols, n_mol, st);
        const spm_batch_mol* D = mols + m;
        const GridView G = slab_view(*D, nullptr);
        const float4 pp = __ldg(PPs + st);
        C = corners_of<true>(G, mk3(pp.x, pp.y, pp.z));
        valid = C.ok;
        const long long ls = st - D->state_off;
        stroke = D->pix_off + (ls < (1LL << 32) ? (long long)((unsigned)ls / (unsigned)D->nz_steps)
                                                : ls / D->nz_steps);
        nxs = G.nx_slab; nys = G.ny_slab;
        x_lo = G.x_lo; y_lo = G.y_lo; z_lo = G.z_lo;
        base = gq + (size_t)D->grid_off * 4;
        scale = pow2(42 - scale_exp(__ldg(umax + m)));
    }
    // merge tests against the next lane (it gives me its upper layer) and the previous one (I give mine)
    const bool nb_valid = __shfl_down_sync(FULL, valid, 1);
    const long long nb_stroke = __shfl_down_sync(FULL, stroke, 1);
    const int nb_x0 = __shfl_down_sync(FULL, C.x[0], 1), nb_y0 = __shfl_down_sync(FULL, C.y[0], 1);
    const int nb_z1 = __shfl_down_sync(FULL, C.z[1], 1);
    const bool take = valid && lane < 31 && nb_valid && nb_stroke == stroke && nb_x0 == C.x[0] && nb_y0 == C.y[0] &&
                      nb_z1 == C.z[0];
    const bool pv_valid = __shfl_up_sync(FULL, valid, 1);
    const long long pv_stroke = __shfl_up_sync(FULL, stroke, 1);
    const int pv_x0 = __shfl_up_sync(FULL, C.x[0], 1), pv_y0 = __shfl_up_sync(FULL, C.y[0], 1);
    const int pv_z0 = __shfl_up_sync(FULL, C.z[0], 1);
    const bool given = valid && lane > 0 && pv_valid && pv_stroke == stroke && pv_x0 == C.x[0] && pv_y0 == C.y[0] &&
                       C.z[1] == pv_z0;
    float w[8];
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const int i = c & 1, j = (c >> 1) & 1, k = c >> 2;
        w[c] = valid ? (i ? C.ax : 1.f - C.ax) * (j ? C.ay : 1.f - C.ay) * (k ? C.az : 1.f - C.az) : 0.f;
    }
    const float ubc[4] = {ub.x, ub.y, ub.z, ub.w};
    int slot[8];
    if constexpr (AGG) {
        // the table slot of each corner this state adds to (-1: none found, the corner goes to global memory)
#pragma unroll
        for (int c = 0; c < 8; c++) {
            slot[c] = -1;
            if (!valid || (c >= 4 && given) || w[c] == 0.f) continue;
            const int i = c & 1, j = (c >> 1) & 1, k = c >> 2;
            const size_t node = ((size_t)(C.z[k] - z_lo) * nys + (C.y[j] - y_lo)) * nxs + (C.x[i] - x_lo);
            const unsigned long long key = (unsigned long long)((base - gq) + node * 4);
            unsigned h = (unsigned)((key * 0x9E3779B97F4A7C15ull) >> 53) & (AGG_SLOTS - 1);
            for (int probe = 0; probe < AGG_PROBES; probe++) {
                const unsigned long long prev = atomicCAS(s_key + h, AGG_EMPTY, key);
                if (prev == AGG_EMPTY || prev == key) {
                    slot[c] = (int)h;
                    break;
                }
                h = (h + 1) & (AGG_SLOTS - 1);
            }
        }
    }
#pragma unroll
    for (int ch = 0; ch < 4; ch++) {
        long long q[8];
#pragma unroll
        for (int c = 0; c < 8; c++) q[c] = (w[c] == 0.f) ? 0ll : __double2ll_rn((double)(w[c] * ubc[ch]) * scale);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const long long up = __shfl_down_sync(FULL, q[4 + c], 1);
            if (take) q[c] += up;
        }
        if (valid) {
#pragma unroll
            for (int c = 0; c < 8; c++) {
                if (c >= 4 && given) continue;
                if (q[c] == 0) continue;
                if (AGG && slot[c] >= 0) {
                    atomicAdd(s_val + 4 * slot[c] + ch, (unsigned long long)q[c]);
                    continue;
                }
                const int i = c & 1, j = (c >> 1) & 1, k = c >> 2;
                const size_t node = ((size_t)(C.z[k] - z_lo) * nys + (C.y[j] - y_lo)) * nxs + (C.x[i] - x_lo);
                atomicAdd(base + node * 4 + ch, (unsigned long long)q[c]);
            }
        }
    }
    if constexpr (AGG) {
        __syncthreads();
        for (int t = threadIdx.x; t < AGG_SLOTS; t += blockDim.x) {
            const unsigned long long key = s_key[t];
            if (key == AGG_EMPTY) continue;
#pragma unroll
            for (int ch = 0; ch < 4; ch++) {
                const unsigned long long v = s_val[4 * t + ch];
                if (v != 0ull) atomicAdd(gq + key + ch, v);
            }
        }
    }
}

// Tile scatter (spm_batch_shape.adj_agg = 2): a warp takes one relaxation slot tile -- 32 pixels of
// one molecule, (32/h) x h of the raster -- and its lanes walk their strokes down together, one
// z-step at a time.  A state's upper corner layer is its stroke predecessor's lower layer when the
// cell column is the same: the lane adds the carried lower-layer sums there (as the default
// kernel's lane pairs do).  Then the pixel one row up the raster (the next lane of the tile column)
// hands over the nodes its upper layer shares with this lane's: all four when its cell is the same,
// the two of its lower row when its cell is the next one in y; it drops them from its own atomics.
// Then the same across the tile's columns (lane + h, the next raster column): all four nodes, or
// the two of its first column when its cell is the next one in x.  In each round a lane gives only
// to one neighbour and takes only from the other, moving sums between lanes that hold the same node,
// so the integer sums are the default kernel's bits.  A carried layer whose column moved goes to the
// grid on its own.
// Eight CTAs of four warps per SM (64 registers, no spills): the walk waits on its loads and
// shuffles, so resident warps pay (11.8 -> 11.6 ms for the 64-molecule fit's adjoint against 96
// registers at five CTAs).
constexpr int SCT_WARPS = 4;

__global__ void __launch_bounds__(SCT_WARPS * 32, 8)
batch_scatter_tile_kernel(int n_mol, const spm_batch_mol* __restrict__ mols, unsigned n_slots, int th_log2,
                          const float4* __restrict__ PPs, const float4* __restrict__ ubar,
                          const unsigned* __restrict__ umax, unsigned long long* __restrict__ gq,
                          unsigned long long* __restrict__ mark, unsigned* __restrict__ counter) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *mark = ADJ_DIRTY;  // the adjoint grid is written from here on
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int th = 1 << th_log2;
    const bool has_above = (lane & (th - 1)) < th - 1;  // the next lane is the next raster row, same column
    const bool has_below = (lane & (th - 1)) > 0;
    while (true) {
        unsigned tb = 0;
        if (lane == 0) tb = atomicAdd(counter, 32u);
        tb = __shfl_sync(FULL, tb, 0);
        if (tb >= n_slots) return;  // warp-uniform
        const int m = SPM_MOL_BY(slot_off, mols, n_mol, (long long)tb);
        const spm_batch_mol* D = mols + m;
        int k = 0;
        const bool lv = slot_pixel(D, tb + lane - (unsigned)D->slot_off, th_log2, k);
        const int nz = D->nz_steps;
        const GridView G = slab_view(*D, nullptr);
        const long long sbase = D->state_off + (long long)(lv ? k : 0) * nz;
        unsigned long long* base = gq + (size_t)D->grid_off * 4;
        const double scale = pow2(42 - scale_exp(__ldg(umax + m)));
        const int nxs = G.nx_slab, nys = G.ny_slab, x_lo = G.x_lo, y_lo = G.y_lo, z_lo = G.z_lo;
        auto add = [&](int x, int y, int z, int ch, long long v) {
            if (v == 0) return;
            const size_t node = ((size_t)(z - z_lo) * nys + (y - y_lo)) * nxs + (x - x_lo);
            atomicAdd(base + node * 4 + ch, (unsigned long long)v);
        };
        // the default kernel's fixed-point term (its w == 0 test is redundant: ubar is finite, so a zero
        // weight gives a zero product and the integer 0 either way)
        auto fixq = [&](float w, float u) { return __double2ll_rn((double)(w * u) * scale); };
        // the carried lower layer of the previous z-step (weights and ubar)
        bool cv = false;
        int cx0 = 0, cy0 = 0, cz0 = 0, cx1 = 0, cy1 = 0;
        float cw[4] = {0.f, 0.f, 0.f, 0.f};
        float4 cub = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int iz = 0; iz <= nz; ++iz) {  // iz == nz: flush the last carried layer only
            bool valid = false;
            Corners C = {{0, 0}, {0, 0}, {0, 0}, 0.f, 0.f, 0.f, false};
            float4 ub = make_float4(0.f, 0.f, 0.f, 0.f);
            if (lv && iz < nz) {
                ub = __ldg(ubar + sbase + iz);
                valid = !(ub.x == 0.f && ub.y == 0.f && ub.z == 0.f && ub.w == 0.f);
                if (valid) {
                    const float4 pp = __ldg(PPs + sbase + iz);
                    C = corners_of<true>(G, mk3(pp.x, pp.y, pp.z));
                    valid = C.ok;
                }
            }
            // upper-layer weights (k = 1) and lower-layer weights (k = 0) of corner c = i + 2 j
            float wu[4], wl[4];
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int i = c & 1, j = c >> 1;
                const float wxy = (i ? C.ax : 1.f - C.ax) * (j ? C.ay : 1.f - C.ay);
                wu[c] = valid ? wxy * C.az : 0.f;
                wl[c] = valid ? wxy * (1.f - C.az) : 0.f;
            }
            const bool merge = valid && cv && C.x[0] == cx0 && C.y[0] == cy0 && C.z[1] == cz0;
            if (cv && !merge) {  // the carried layer's column moved: its own atomics
                const float c4[4] = {cub.x, cub.y, cub.z, cub.w};
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int i = c & 1, j = c >> 1;
#pragma unroll
                    for (int ch = 0; ch < 4; ch++) add(i ? cx1 : cx0, j ? cy1 : cy0, cz0, ch, fixq(cw[c], c4[ch]));
                }
            }
            // the lane above (next raster row): same cell (A) or the next cell in y (B), same x and layer
            const int ax0 = __shfl_down_sync(FULL, C.x[0], 1), ay0 = __shfl_down_sync(FULL, C.y[0], 1);
            const int az1 = __shfl_down_sync(FULL, C.z[1], 1);
            const bool av = __shfl_down_sync(FULL, valid, 1);
            const bool col = valid && av && has_above && ax0 == C.x[0] && az1 == C.z[1];
            const bool take_all = col && ay0 == C.y[0];
            const bool take_row = col && !take_all && ay0 == C.y[1];
            const bool give_all = __shfl_up_sync(FULL, take_all, 1) && has_below;
            const bool give_row = __shfl_up_sync(FULL, take_row, 1) && has_below;
            // then the lane one tile column over (next raster column, same row): same cell, or the next
            // cell in x (its column i = 0 is this lane's i = 1), same y row and layer
            const int bx0 = __shfl_down_sync(FULL, C.x[0], th), by0 = __shfl_down_sync(FULL, C.y[0], th);
            const int bz1 = __shfl_down_sync(FULL, C.z[1], th);
            const bool bv = __shfl_down_sync(FULL, valid, th);
            const bool colx = valid && bv && lane + th < 32 && by0 == C.y[0] && bz1 == C.z[1];
            const bool takex_all = colx && bx0 == C.x[0];
            const bool takex_col = colx && !takex_all && bx0 == C.x[1];
            const bool givex_all = __shfl_up_sync(FULL, takex_all, th) && lane >= th;
            const bool givex_col = __shfl_up_sync(FULL, takex_col, th) && lane >= th;
            const float u4[4] = {ub.x, ub.y, ub.z, ub.w}, c4[4] = {cub.x, cub.y, cub.z, cub.w};
            unsigned nd[4];  // the upper layer's slab nodes, once for the four channels
#pragma unroll
            for (int c = 0; c < 4; c++)
                nd[c] = ((unsigned)(C.z[1] - z_lo) * (unsigned)nys + (unsigned)(C.y[c >> 1] - y_lo)) * (unsigned)nxs +
                        (unsigned)(C.x[c & 1] - x_lo);
#pragma unroll
            for (int ch = 0; ch < 4; ch++) {
                if (__all_sync(FULL, u4[ch] == 0.f && (!merge || c4[ch] == 0.f))) continue;  // warp-uniform
                long long v[4];
#pragma unroll
                for (int c = 0; c < 4; c++) v[c] = fixq(wu[c], u4[ch]) + (merge ? fixq(cw[c], c4[ch]) : 0ll);
                long long up[4];
#pragma unroll
                for (int c = 0; c < 4; c++) up[c] = __shfl_down_sync(FULL, v[c], 1);  // the lane above's, as computed
                if (give_all) {
#pragma unroll
                    for (int c = 0; c < 4; c++) v[c] = 0;
                } else if (give_row) {
                    v[0] = 0;
                    v[1] = 0;
                }
                if (take_all) {
#pragma unroll
                    for (int c = 0; c < 4; c++) v[c] += up[c];
                } else if (take_row) {
                    v[2] += up[0];  // its row j = 0 is this lane's row j = 1
                    v[3] += up[1];
                }
                long long rt[4];
#pragma unroll
                for (int c = 0; c < 4; c++) rt[c] = __shfl_down_sync(FULL, v[c], th);  // after the row merge
                if (givex_all) {
#pragma unroll
                    for (int c = 0; c < 4; c++) v[c] = 0;
                } else if (givex_col) {
                    v[0] = 0;
                    v[2] = 0;
                }
                if (takex_all) {
#pragma unroll
                    for (int c = 0; c < 4; c++) v[c] += rt[c];
                } else if (takex_col) {
                    v[1] += rt[0];  // its column i = 0 is this lane's column i = 1
                    v[3] += rt[2];
                }
                if (valid) {
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        if (v[c] != 0) atomicAdd(base + (size_t)nd[c] * 4 + ch, (unsigned long long)v[c]);
                }
            }
            // carry this state's lower layer
            cv = valid;
            cx0 = C.x[0]; cx1 = C.x[1]; cy0 = C.y[0]; cy1 = C.y[1]; cz0 = C.z[0];
#pragma unroll
            for (int c = 0; c < 4; c++) cw[c] = wl[c];
            cub = ub;
        }
        __syncwarp();  // the whole warp draws the next tile
    }
}

constexpr int NM_THREADS = 256;
constexpr int NM_PER_THREAD = 2;
constexpr int NM_STAGE = NM_THREADS * NM_PER_THREAD;  // nodes examined per staging pass
constexpr int NM_FLUSH = 64;                          // FP32 partial sums folded into FP64 every 64 pairs
constexpr float LOG2E = 1.4426950408889634f;

__device__ __forceinline__ float mufu_rsqrt(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float mufu_ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Tip-charge sites of the node-major adjoint: sites with a zero z-offset sit on
// the node and share the pair law's 1/r; the others get their own rsqrt.
struct NodeSites {
    float qon;           // sum of Qs[k]*COULOMB_CONST over sites with QZs[k] == 0
    int noff;
    float qs[4], qz[4];  // off-node sites
};

NodeSites make_node_sites(const float* Qs, const float* QZs) {
    NodeSites S = {};
    for (int k = 0; k < 4; k++) {
        if (Qs[k] == 0.f) continue;
        if (QZs[k] == 0.f) {
            S.qon += Qs[k] * COULOMB_CONST;
        } else {
            S.qs[S.noff] = Qs[k] * COULOMB_CONST;
            S.qz[S.noff] = QZs[k];
            S.noff++;
        }
    }
    return S;
}

__device__ __forceinline__ f2 rsqrt2(f2 x) {
    float a, b;
    upk(x, a, b);
    return pk(mufu_rsqrt(a), mufu_rsqrt(b));
}
__device__ __forceinline__ f2 ex2_2(f2 x) {
    float a, b;
    upk(x, a, b);
    return pk(mufu_ex2(a), mufu_ex2(b));
}

// Per-atom constants of the packed pair derivatives (both lanes equal).
struct AtomC {
    f2 x, y, z;      // position
    f2 c0, c1, c2, c3;  // LJ: 12 c12, -6 c6, 168 c12, -48 c6; Morse: K log2e, -K R0 log2e, -2 K E0, 2 K^2 E0
    f2 c4;           // Morse: -2 K
    f2 qw, qw3;      // Q * qon and 3 Q * qon (on-node tip charges)
    float q;         // Q
};

// Derivatives of the pair laws of the grid build (LJ / Morse + point-charge
// Coulomb, R2SAFE-softened, as pair_grad) at two nodes per call, contracted
// with the nodes' adjoint vectors g = (gx,gy,gz,gw):
//   acc[0..2] += dF/d(atom position)^T g   acc[3], acc[4] += dF/d(pair params)^T g (PAR)
//   acc[5]    += dF/d(atom charge)^T g
// with Blackwell's packed FP32 (two nodes per instruction), one MUFU rsqrt per
// node for the pair law and the on-node charges together, MUFU ex2 for Morse.
// The radial factors s = -E'(r)/r and sp2 = -2 s'(r)/r of the pair law and of
// the on-node charges (Q qon / r) are summed before the powers of 1/r they
// share are applied.  LJ's acc[3] is accumulated negated (the sign is applied
// when it is folded).
template <int KIND, bool ON, bool PAR>
__device__ __forceinline__ void pair_adj2(f2 nx, f2 ny, f2 nz, f2 gx, f2 gy, f2 gz, f2 gw, const AtomC& C,
                                          const NodeSites& S, f2* acc) {
    const f2 dx = sub2(nx, C.x), dy = sub2(ny, C.y), dz = sub2(nz, C.z);
    const f2 r2 = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, bc(R2SAFE))));
    const f2 rs = rsqrt2(r2);
    const f2 ir2 = mul2(rs, rs);
    const f2 du = fma2(dx, gx, fma2(dy, gy, mul2(dz, gz)));
    f2 s, sp2;
    if (KIND == SPM_KIND_LJ) {
        const f2 ir4 = mul2(ir2, ir2);
        const f2 ir6 = mul2(ir4, ir2);
        const f2 a1 = fma2(C.c0, ir6, C.c1);  // 12 c12 ir6 - 6 c6:   s = a1 ir8
        const f2 a2 = fma2(C.c2, ir6, C.c3);  // 168 c12 ir6 - 48 c6: sp2 = a2 ir10
        if (ON) {
            s = mul2(fma2(a1, ir6, mul2(C.qw, rs)), ir2);     // + Q qon / r^3
            sp2 = mul2(fma2(a2, ir6, mul2(C.qw3, rs)), ir4);  // + 3 Q qon / r^5
        } else {
            s = mul2(mul2(a1, ir6), ir2);
            sp2 = mul2(mul2(a2, ir6), ir4);
        }
        if (PAR) {
            const f2 h6 = mul2(bc(6.f), ir2);
            const f2 t6 = fma2(du, h6, gw);                // gw + 6 du / r^2
            const f2 t12 = fma2(du, h6, t6);               // gw + 12 du / r^2
            acc[3] = fma2(t6, ir6, acc[3]);                // -(d/dc6):  gw ir6 + 6 du ir8
            acc[4] = fma2(t12, mul2(ir6, ir6), acc[4]);    //   d/dc12:  gw ir12 + 12 du ir14
        }
    } else {
        const f2 r = mul2(r2, rs);
        const f2 e = ex2_2(fma2(C.c0, r, C.c1));              // exp(K (r - R0))
        const f2 em1 = sub2(e, bc(1.f));
        const f2 nEp = mul2(mul2(C.c2, e), em1);              // -E'
        const f2 Epp = mul2(mul2(C.c3, e), fma2(bc(2.f), e, bc(-1.f)));
        if (ON) {
            s = mul2(fma2(C.qw, ir2, nEp), rs);                                   // + Q qon / r^3
            sp2 = mul2(fma2(Epp, rs, mul2(fma2(C.qw3, ir2, nEp), ir2)), rs);     // + 3 Q qon / r^5
        } else {
            s = mul2(nEp, rs);
            sp2 = mul2(fma2(Epp, rs, mul2(nEp, ir2)), rs);
        }
        if (PAR) {
            acc[3] = fma2(gw, nEp, fma2(mul2(du, Epp), rs, acc[3]));
            acc[4] = fma2(mul2(gw, e), sub2(e, bc(2.f)), fma2(mul2(du, mul2(mul2(C.c4, e), em1)), rs, acc[4]));
        }
    }
    if (ON) {
        const f2 qr = mul2(bc(S.qon), rs);
        acc[5] = fma2(qr, fma2(du, ir2, gw), acc[5]);  // qon / r (gw + du / r^2)
    }
    const f2 A = fma2(gw, s, mul2(sp2, du));
    const f2 ns = mul2(s, bc(-1.f));
    acc[0] = fma2(A, dx, fma2(ns, gx, acc[0]));
    acc[1] = fma2(A, dy, fma2(ns, gy, acc[1]));
    acc[2] = fma2(A, dz, fma2(ns, gz, acc[2]));
    for (int k = 0; k < S.noff; k++) {
        const f2 dk = add2(dz, bc(S.qz[k]));
        const f2 rk = rsqrt2(fma2(dx, dx, fma2(dy, dy, fma2(dk, dk, bc(R2SAFE)))));
        const f2 irk2 = mul2(rk, rk);
        const f2 qr = mul2(bc(S.qs[k]), rk);
        const f2 sk = mul2(mul2(qr, bc(C.q)), irk2);
        const f2 duk = fma2(dx, gx, fma2(dy, gy, mul2(dk, gz)));
        const f2 Ak = fma2(gw, sk, mul2(mul2(bc(3.f), sk), mul2(irk2, duk)));
        const f2 nsk = mul2(sk, bc(-1.f));
        acc[0] = fma2(Ak, dx, fma2(nsk, gx, acc[0]));
        acc[1] = fma2(Ak, dy, fma2(nsk, gy, acc[1]));
        acc[2] = fma2(Ak, dk, fma2(nsk, gz, acc[2]));
        acc[5] = fma2(gw, qr, fma2(duk, mul2(qr, irk2), acc[5]));
    }
}


__device__ __forceinline__ f2 lds2(const float* p) { return *reinterpret_cast<const f2*>(p); }

// acc[c * stride] += the two lanes of sums[c] (FP64), sums[c] = 0; the
// pair-parameter columns only with PAR.
template <bool PAR>
__device__ __forceinline__ void fold_sums(f2* sums, double* acc, int stride) {
#pragma unroll
    for (int c = 0; c < 6; c++) {
        if (!PAR && (c == 3 || c == 4)) continue;
        float lo, hi;
        upk(sums[c], lo, hi);
        acc[c * stride] += (double)lo + (double)hi;
        sums[c] = bc(0.f);
    }
}

// Dynamic shared memory of batch_adjoint_nodes_kernel: x, y, z, gx, gy, gz, gw
// of up to 2*NM_STAGE staged nodes (+1 zero-weight pad node), the phase
// partials and the double-buffered warp counts of the compaction scan.
constexpr int NM_BUF = 2 * NM_STAGE + 2;
constexpr size_t NM_SMEM = 7 * NM_BUF * sizeof(float) + 6 * NM_THREADS * sizeof(double) + 2 * (NM_THREADS / 32) * sizeof(int);
// BULK (spm_batch_shape.adj_stage = 1): a block of NM_THREADS adjoint-grid nodes (32 bytes each) is
// fetched by one bulk copy into shared memory while the previous block is examined and computed,
// completion on an mbarrier: 8 KB more per CTA (four still fit per SM)
constexpr size_t NM_RAW = (size_t)NM_THREADS * 32;
constexpr size_t NM_SMEM_BULK = (NM_SMEM + 15) / 16 * 16 + NM_RAW + 16;
constexpr unsigned NM_SPIN = 1u << 22;  // bounded mbarrier polls before a block is read with plain loads
// ILP = 3 (two atoms per thread): the second atom's FP64 sums after the first's
constexpr size_t NM_SMEM_2ATOM = (NM_SMEM + 15) / 16 * 16 + 6 * NM_THREADS * sizeof(double);

__device__ __forceinline__ bool nm_try_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}" : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}

// CTA per node unit (molecule, `chunk` consecutive slab nodes).  Non-zero
// adjoint-grid nodes are compacted into shared memory (one float array per
// component, so nodes 2i and 2i+1 load as one packed pair); thread t owns atom
// a0 + t % nag and every P-th staged node pair (P = 256 / nag phases), so the
// atom's derivative sums stay in its registers: no atomics, no cross-thread
// reduction until the phases are folded once per unit.
//   * NM_STAGE-node passes outside the molecule's box of touched rows and slab
//     layers (box, from the ubar-maximum kernel) are skipped without being read;
//   * the non-zero nodes of consecutive blocks accumulate in shared memory
//     until at least NM_STAGE are staged, so every compute phase between two
//     barriers is dense;
//   * every non-zero node is zeroed after it is staged (by the last atom
//     group), so the adjoint grid is left cleared for the next call.
// Four CTAs per SM (64 registers, a few bytes spilled, 4 x 41 KB of shared
// memory with 512-node passes): the loop is bound by its dependency chains,
// so resident warps pay (64-molecule fit: two CTAs at 128 registers 12.2 ms,
// three at 80 registers 10.7 ms, four at 64 registers 2% less than three;
// five at 48 registers spill too much).  ILP = 2: two independent node pairs
// per step at two CTAs per SM (up to 128 registers).  PAR: also the
// pair-parameter columns 3-4 (else written as 0).
template <int KIND, bool ON, bool PAR, int ILP, bool BULK = false>
__global__ void __launch_bounds__(NM_THREADS, ILP == 1 ? 4 : 2)
batch_adjoint_nodes_kernel(int n_mol, const spm_batch_mol* __restrict__ mols, int chunk,
                           const float4* __restrict__ atoms, const float* __restrict__ params, int pstride,
                           NodeSites S, unsigned long long* __restrict__ gq, const int* __restrict__ box,
                           const unsigned* __restrict__ umax, double* __restrict__ partial,
                           unsigned* __restrict__ status) {
    static_assert(!BULK || ILP == 1, "bulk-copy staging with one node pair per step");
    constexpr int APT = ILP == 3 ? 2 : 1;  // atoms per thread
    extern __shared__ __align__(16) unsigned char nm_smem[];
    float(*s_n)[NM_BUF] = reinterpret_cast<float(*)[NM_BUF]>(nm_smem);
    double(*red)[NM_THREADS] = reinterpret_cast<double(*)[NM_THREADS]>(nm_smem + 7 * NM_BUF * sizeof(float));
    int(*s_wsum)[NM_THREADS / 32] = reinterpret_cast<int(*)[NM_THREADS / 32]>(
        nm_smem + 7 * NM_BUF * sizeof(float) + 6 * NM_THREADS * sizeof(double));
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    // BULK: the raw block (node i of the block at s_raw[2i], s_raw[2i+1]) and its mbarrier
    ulonglong2* s_raw = reinterpret_cast<ulonglong2*>(nm_smem + (NM_SMEM + 15) / 16 * 16);
    const unsigned bar = (unsigned)__cvta_generic_to_shared(nm_smem + (NM_SMEM + 15) / 16 * 16 + NM_RAW);
    unsigned parity = 0;
    bool bulk = BULK;  // false after a wait ran out: plain loads from then on
    if (BULK) {
        if (t == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bar) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
    }
    const long long unit = blockIdx.x;
    const int m = SPM_MOL_BY(unit_off, mols, n_mol, unit);
    const spm_batch_mol* D = mols + m;
    const long long lc = unit - D->unit_off;
    // slab pitches (stored columns, rows) and the stored box's corner in the full grid
    const int nx = D->nx_slab, ny = D->ny_slab, x_lo = D->x_lo, y_lo = D->y_lo, z_lo = D->z_lo;
    const long long slab = (long long)nx * ny * D->nz_slab;
    const long long n0 = lc * chunk;
    const long long n1 = n0 + chunk < slab ? n0 + chunk : slab;
    const int na = D->n_atoms;
    NodeGeom NG;
    NG.p0 = ld4f(D->p0);
    NG.dA = ld4f(D->dA);
    NG.dB = ld4f(D->dB);
    NG.dC = ld4f(D->dC);
    const double inv_scale = pow2(scale_exp(__ldg(umax + m)) - 42);
    ulonglong2* q2 = reinterpret_cast<ulonglong2*>(gq + (size_t)D->grid_off * 4);
    // touched slab rows in [ylo, yhi] and slab layers in [zlo, zhi] (empty: yhi < 0)
    const int ylo = ny - 1 - box[4 * m], yhi = box[4 * m + 1] - 1;
    const int zlo = D->nz_slab - 1 - box[4 * m + 2], zhi = box[4 * m + 3] - 1;
    auto touched = [&](long long b0, long long b1) {  // may nodes [b0, b1) be non-zero?
        const unsigned r0 = (unsigned)b0 / (unsigned)nx, r1 = (unsigned)(b1 - 1) / (unsigned)nx;  // rows zl*ny + y
        const int za = (int)(r0 / (unsigned)ny), zb = (int)(r1 / (unsigned)ny);
        if (yhi < 0 || zb < zlo || za > zhi) return false;
        if (za != zb) return true;  // spans a layer boundary: keep
        const int ya = (int)(r0 - (unsigned)za * ny), yb = (int)(r1 - (unsigned)za * ny);
        return !(yb < ylo || ya > yhi);
    };
    // ILP = 3: the second atom's FP64 sums (red2[c][t]), after the shared arrays
    double(*red2)[NM_THREADS] = reinterpret_cast<double(*)[NM_THREADS]>(nm_smem + (NM_SMEM + 15) / 16 * 16);
    auto atom_consts = [&](int ga) {
        const float4 at = __ldg(atoms + ga);
        const float* pr = params + (size_t)ga * pstride;
        const float p1 = __ldg(pr + 0), p2 = __ldg(pr + 1), p3 = (pstride > 2) ? __ldg(pr + 2) : 0.f;
        AtomC C;
        C.x = bc(at.x);
        C.y = bc(at.y);
        C.z = bc(at.z);
        C.q = at.w;
        C.qw = bc(at.w * S.qon);
        C.qw3 = bc(3.f * (at.w * S.qon));
        if (KIND == SPM_KIND_LJ) {  // p1 = c6, p2 = c12
            C.c0 = bc(12.f * p2);
            C.c1 = bc(-6.f * p1);
            C.c2 = bc(168.f * p2);
            C.c3 = bc(-48.f * p1);
            C.c4 = bc(0.f);
        } else {  // p1 = R0, p2 = E0, p3 = K
            C.c0 = bc(p3 * LOG2E);
            C.c1 = bc(-p3 * p1 * LOG2E);
            C.c2 = bc(-2.f * p3 * p2);
            C.c3 = bc(2.f * p3 * p3 * p2);
            C.c4 = bc(-2.f * p3);
        }
        return C;
    };
    for (int a0 = 0, nag = 0; a0 < na; a0 += nag) {
        // atom group: nslot thread slots x P phases <= 256 threads, APT atoms per slot (slot s takes atoms
        // a0 + s and a0 + nslot + s).  The remaining atoms go in one group when that keeps >= 85% of the
        // threads busy, else a group of 256/P slots with P = ceil(256/slots needed) and the rest after it
        // (65 atoms, one per thread: 64 at 4 phases + 1 at 256 instead of 65 at 3)
        const int rem = na - a0;
        int nslot;
        if (rem >= APT * NM_THREADS) {
            nslot = NM_THREADS;
        } else {
            const int rs = (rem + APT - 1) / APT;
            nslot = (NM_THREADS / rs) * rs * 100 >= 85 * NM_THREADS ? rs : NM_THREADS / ((NM_THREADS + rs - 1) / rs);
        }
        nag = min(rem, APT * nslot);
        const int P = NM_THREADS / nslot;
        const bool last_group = a0 + nag >= na;
        const bool act = t < nslot * P;
        const int a = a0 + (act ? t % nslot : 0), ph = act ? t / nslot : 0;
        const AtomC C = atom_consts(D->atom_off + a);
        // ILP = 3: the slot's second atom, or an inert one (zero constants; its sums are not written)
        const bool has_b = APT == 2 && act && (t % nslot) + nslot < nag;
        AtomC CB;
        if (APT == 2) {
            if (has_b) {
                CB = atom_consts(D->atom_off + a + nslot);
            } else {
                const f2 z = bc(0.f);
                CB.x = z; CB.y = z; CB.z = z; CB.c0 = z; CB.c1 = z; CB.c2 = z; CB.c3 = z; CB.c4 = z;
                CB.qw = z; CB.qw3 = z; CB.q = 0.f;
            }
        }
        // the atom's FP64 sums, in shared memory (red[c][t]) to keep registers for the pair loop
        double* acc = &red[0][t];
        double* acc2 = &red2[0][t];
#pragma unroll
        for (int c = 0; c < 6; c++) {
            acc[c * NM_THREADS] = 0.0;
            if (APT == 2) acc2[c * NM_THREADS] = 0.0;
        }
        // the staged nodes' derivative sums: FP32 over NM_FLUSH pairs, then FP64
        auto compute = [&](int L) {
            if (t == 0 && (L & 1)) {  // pad to whole pairs: a distant node of zero weight adds +-0
#pragma unroll
                for (int c = 0; c < 3; c++) s_n[c][L] = 1e4f;
#pragma unroll
                for (int c = 3; c < 7; c++) s_n[c][L] = 0.f;
            }
            __syncthreads();
            if (act) {
                const f2 zero = bc(0.f);
                f2 a32[6] = {zero, zero, zero, zero, zero, zero};
                int n32 = 0;
                const int Lp = (L + 1) >> 1;
                auto pair_at = [&](int jp, f2* sums) {
                    const int j = 2 * jp;
                    pair_adj2<KIND, ON, PAR>(lds2(&s_n[0][j]), lds2(&s_n[1][j]), lds2(&s_n[2][j]), lds2(&s_n[3][j]),
                                             lds2(&s_n[4][j]), lds2(&s_n[5][j]), lds2(&s_n[6][j]), C, S, sums);
                };
                int jp = ph;
                if (ILP == 3) {
                    // each staged node pair loaded once for the slot's two atoms
                    f2 b32[6] = {zero, zero, zero, zero, zero, zero};
                    for (; jp < Lp; jp += P) {
                        const int j = 2 * jp;
                        const f2 nx = lds2(&s_n[0][j]), ny = lds2(&s_n[1][j]), nz = lds2(&s_n[2][j]);
                        const f2 gx = lds2(&s_n[3][j]), gy = lds2(&s_n[4][j]), gz = lds2(&s_n[5][j]);
                        const f2 gw = lds2(&s_n[6][j]);
                        pair_adj2<KIND, ON, PAR>(nx, ny, nz, gx, gy, gz, gw, C, S, a32);
                        pair_adj2<KIND, ON, PAR>(nx, ny, nz, gx, gy, gz, gw, CB, S, b32);
                        if (++n32 == NM_FLUSH / 2) {
                            fold_sums<PAR>(a32, acc, NM_THREADS);
                            fold_sums<PAR>(b32, acc2, NM_THREADS);
                            n32 = 0;
                        }
                    }
                    fold_sums<PAR>(b32, acc2, NM_THREADS);
                } else if (ILP == 2) {
                    // two independent node pairs per step, each into its own FP32 sums
                    f2 b32[6] = {zero, zero, zero, zero, zero, zero};
                    for (; jp + P < Lp; jp += 2 * P) {
                        pair_at(jp, a32);
                        pair_at(jp + P, b32);
                        if (++n32 == NM_FLUSH / 2) {
                            fold_sums<PAR>(a32, acc, NM_THREADS);
                            fold_sums<PAR>(b32, acc, NM_THREADS);
                            n32 = 0;
                        }
                    }
                    fold_sums<PAR>(b32, acc, NM_THREADS);
                    for (; jp < Lp; jp += P) pair_at(jp, a32);
                } else {
                    // blocks of NM_FLUSH / 2 pairs between folds (the last one shorter), walking one
                    // pointer through the staged arrays (the seven components at fixed offsets from it)
                    const float* sp = &s_n[0][2 * jp];
                    const int sstep = 2 * P;
                    int left = jp < Lp ? (Lp - jp + P - 1) / P : 0;  // pairs of this thread
                    while (left > 0) {
                        const int nb = min(NM_FLUSH / 2, left);
#pragma unroll 4
                        for (int k = 0; k < nb; k++, sp += sstep)
                            pair_adj2<KIND, ON, PAR>(lds2(sp), lds2(sp + NM_BUF), lds2(sp + 2 * NM_BUF),
                                                     lds2(sp + 3 * NM_BUF), lds2(sp + 4 * NM_BUF),
                                                     lds2(sp + 5 * NM_BUF), lds2(sp + 6 * NM_BUF), C, S, a32);
                        left -= nb;
                        if (left > 0) fold_sums<PAR>(a32, acc, NM_THREADS);
                    }
                }
                fold_sums<PAR>(a32, acc, NM_THREADS);
            }
            __syncthreads();  // the buffer is restaged next
        };
        int staged = 0, pass = 0;  // block-uniform
        if (BULK) {
            // blocks of NM_THREADS nodes; the next touched block is fetched while this one is examined
            // and while the staged nodes are computed
            auto next_touched = [&](long long b) {
                while (b < n1 && !touched(b, b + NM_THREADS < n1 ? b + NM_THREADS : n1)) b += NM_THREADS;
                return b;
            };
            auto issue = [&](long long b) {  // thread 0; b < n1
                const long long e = b + NM_THREADS < n1 ? b + NM_THREADS : n1;
                const unsigned bytes = (unsigned)(e - b) * 32u;
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
                asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                             :: "r"((unsigned)__cvta_generic_to_shared(s_raw)), "l"(q2 + 2 * b), "r"(bytes), "r"(bar)
                             : "memory");
            };
            long long b0 = next_touched(n0);
            if (bulk && t == 0 && b0 < n1) issue(b0);
            while (true) {
                const bool more = b0 < n1;
                if (more) {
                    const long long b1 = b0 + NM_THREADS < n1 ? b0 + NM_THREADS : n1;
                    bool from_smem = bulk;
                    if (bulk) {  // every thread polls: bounded, then a second bounded wait for the copy in flight
                        unsigned spins = 0;
                        bool done = nm_try_wait(bar, parity);
                        while (!done && ++spins < NM_SPIN) done = nm_try_wait(bar, parity);
                        if (!done) {
                            if (t == 0) atomicOr(status, 1u);
                            spins = 0;
                            while (!done && ++spins < NM_SPIN) done = nm_try_wait(bar, parity);
                        }
                        from_smem = __syncthreads_and(done);
                        parity ^= 1u;
                        if (!from_smem) bulk = false;  // block-uniform: plain loads from here on
                    }
                    const long long node = b0 + t;
                    ulonglong2 lo = make_ulonglong2(0ull, 0ull), hi = lo;
                    if (node < b1) {
                        if (from_smem) {
                            lo = s_raw[2 * t];
                            hi = s_raw[2 * t + 1];
                        } else {
                            lo = q2[2 * node];
                            hi = q2[2 * node + 1];
                        }
                    }
                    const bool nzr = (lo.x | lo.y | hi.x | hi.y) != 0ull;
                    int x = nzr ? 1 : 0;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(0xffffffffu, x, o);
                        if (lane >= o) x += y;
                    }
                    int* ws = s_wsum[pass & 1];
                    if (lane == 31) ws[warp] = x;
                    __syncthreads();  // also: every thread has read its raw node
                    int off = staged + x - (nzr ? 1 : 0), L = 0;
#pragma unroll
                    for (int w = 0; w < NM_THREADS / 32; w++) {
                        const int c = ws[w];
                        if (w < warp) off += c;
                        L += c;
                    }
                    const long long bn = next_touched(b0 + NM_THREADS);
                    if (bulk && t == 0 && bn < n1) issue(bn);  // the raw block is free: fetch the next one
                    if (nzr) {
                        if (last_group) {
                            q2[2 * node] = make_ulonglong2(0ull, 0ull);
                            q2[2 * node + 1] = make_ulonglong2(0ull, 0ull);
                        }
                        const unsigned l32 = (unsigned)node, yz = l32 / (unsigned)nx;
                        const int ix = (int)(l32 - yz * (unsigned)nx) + x_lo;
                        const int iy = (int)(yz % (unsigned)ny) + y_lo, iz = (int)(yz / (unsigned)ny) + z_lo;
                        s_n[0][off] = NG.p0.x + NG.dA.x * ix + NG.dB.x * iy + NG.dC.x * iz;
                        s_n[1][off] = NG.p0.y + NG.dA.y * ix + NG.dB.y * iy + NG.dC.y * iz;
                        s_n[2][off] = NG.p0.z + NG.dA.z * ix + NG.dB.z * iy + NG.dC.z * iz;
                        s_n[3][off] = (float)((double)(long long)lo.x * inv_scale);
                        s_n[4][off] = (float)((double)(long long)lo.y * inv_scale);
                        s_n[5][off] = (float)((double)(long long)hi.x * inv_scale);
                        s_n[6][off] = (float)((double)(long long)hi.y * inv_scale);
                    }
                    staged += L;
                    ++pass;
                    b0 = bn;
                }
                if (staged >= NM_STAGE || (!more && staged > 0)) {
                    compute(staged);
                    staged = 0;
                }
                if (!more) break;
            }
        }
        for (long long b0 = BULK ? n1 : n0; !BULK; b0 += NM_STAGE) {
            const bool more = b0 < n1;
            const long long b1 = b0 + NM_STAGE < n1 ? b0 + NM_STAGE : n1;
            if (more && touched(b0, b1)) {
            // stage: each thread examines NM_PER_THREAD nodes, compaction by a block scan of counts;
            // the non-zero nodes are read again (an L1 hit) when they are written to shared memory
            bool nz[NM_PER_THREAD];
            int cnt = 0;
#pragma unroll
            for (int r = 0; r < NM_PER_THREAD; r++) {
                const long long node = b0 + r * NM_THREADS + t;
                nz[r] = false;
                if (node < b1) {
                    const ulonglong2 lo = q2[2 * node], hi = q2[2 * node + 1];
                    nz[r] = (lo.x | lo.y | hi.x | hi.y) != 0ull;
                }
                cnt += nz[r] ? 1 : 0;
            }
            int x = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            int* ws = s_wsum[pass & 1];  // alternating: no barrier needed before the next pass writes
            if (lane == 31) ws[warp] = x;
            __syncthreads();
            int off = staged + x - cnt, L = 0;
#pragma unroll
            for (int w = 0; w < NM_THREADS / 32; w++) {
                const int c = ws[w];
                if (w < warp) off += c;
                L += c;
            }
#pragma unroll
            for (int r = 0; r < NM_PER_THREAD; r++) {
                if (!nz[r]) continue;
                const long long li = b0 + r * NM_THREADS + t;  // node index in the slab
                const ulonglong2 lo = q2[2 * li], hi = q2[2 * li + 1];
                if (last_group) {
                    q2[2 * li] = make_ulonglong2(0ull, 0ull);
                    q2[2 * li + 1] = make_ulonglong2(0ull, 0ull);
                }
                const unsigned l32 = (unsigned)li, yz = l32 / (unsigned)nx;  // slabs hold < 2^32 nodes
                const int ix = (int)(l32 - yz * (unsigned)nx) + x_lo;
                const int iy = (int)(yz % (unsigned)ny) + y_lo, iz = (int)(yz / (unsigned)ny) + z_lo;
                s_n[0][off] = NG.p0.x + NG.dA.x * ix + NG.dB.x * iy + NG.dC.x * iz;
                s_n[1][off] = NG.p0.y + NG.dA.y * ix + NG.dB.y * iy + NG.dC.y * iz;
                s_n[2][off] = NG.p0.z + NG.dA.z * ix + NG.dB.z * iy + NG.dC.z * iz;
                s_n[3][off] = (float)((double)(long long)lo.x * inv_scale);
                s_n[4][off] = (float)((double)(long long)lo.y * inv_scale);
                s_n[5][off] = (float)((double)(long long)hi.x * inv_scale);
                s_n[6][off] = (float)((double)(long long)hi.y * inv_scale);
                off++;
            }
            staged += L;
            ++pass;
            }
            // compute once at least NM_STAGE nodes are staged (< 2 * NM_STAGE: a pass adds at most
            // NM_STAGE), and at the end of the unit; one call site, so the body is inlined
            if (staged >= NM_STAGE || (!more && staged > 0)) {
                compute(staged);
                staged = 0;
            }
            if (!more) break;
        }
#pragma unroll
        for (int c = 0; c < 6; c++) {
            red[c][t] = act ? red[c][t] : 0.0;
            if (APT == 2) red2[c][t] = act ? red2[c][t] : 0.0;
        }
        if (KIND == SPM_KIND_LJ && PAR) {  // accumulated negated
            red[3][t] = -red[3][t];
            if (APT == 2) red2[3][t] = -red2[3][t];
        }
        __syncthreads();
        if (t < nslot) {
            double* out = partial + ((size_t)D->row_off + (size_t)lc * na + a0 + t) * 6;
#pragma unroll
            for (int c = 0; c < 6; c++) {
                double s6 = 0.0;
                for (int q = 0; q < P; q++) s6 += red[c][t + q * nslot];
                out[c] = s6;
            }
            if (APT == 2 && t + nslot < nag) {
                double* out2 = partial + ((size_t)D->row_off + (size_t)lc * na + a0 + nslot + t) * 6;
#pragma unroll
                for (int c = 0; c < 6; c++) {
                    double s6 = 0.0;
                    for (int q = 0; q < P; q++) s6 += red2[c][t + q * nslot];
                    out2[c] = s6;
                }
            }
        }
        __syncthreads();
    }
}

// grad[ga*6 + c] = sum over the molecule's node units, fixed order.  When the
// node kernel ran before it (mark != null), block 0 marks the adjoint grid clear.
__global__ void __launch_bounds__(256)
batch_fold_rows_kernel(int n_mol, const spm_batch_mol* __restrict__ mols, int chunk, const double* __restrict__ partial,
                       double* __restrict__ grad, unsigned long long* __restrict__ mark, unsigned long long clean) {
    if (mark && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *mark = clean;
    __shared__ double red[256];
    const long long ga = blockIdx.x;
    const int c = blockIdx.y;
    const spm_batch_mol* D = mols + SPM_MOL_BY(atom_off, mols, n_mol, ga);
    const long long nst = (long long)D->n_scan * D->nz_steps;
    const long long slab = (long long)D->nx_slab * D->ny_slab * D->nz_slab;
    const long long nu = nst > 0 ? (slab + chunk - 1) / chunk : 0;
    const long long a = ga - D->atom_off;
    double acc = 0.0;
    for (long long u = threadIdx.x; u < nu; u += 256) acc += partial[((size_t)D->row_off + u * D->n_atoms + a) * 6 + c];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) grad[ga * 6 + c] = red[0];
}

using NodeKern = decltype(&batch_adjoint_nodes_kernel<SPM_KIND_LJ, true, true, 1>);

template <bool PAR, int ILP, bool BULK>
NodeKern node_kernel(int kind, bool on) {
    if (kind == SPM_KIND_MORSE)
        return on ? batch_adjoint_nodes_kernel<SPM_KIND_MORSE, true, PAR, ILP, BULK>
                  : batch_adjoint_nodes_kernel<SPM_KIND_MORSE, false, PAR, ILP, BULK>;
    return on ? batch_adjoint_nodes_kernel<SPM_KIND_LJ, true, PAR, ILP, BULK>
              : batch_adjoint_nodes_kernel<SPM_KIND_LJ, false, PAR, ILP, BULK>;
}

// The node kernel for a pair law, on-node charges or not, pair-parameter
// columns or not, 1 or 2 node pairs per step, and node blocks read with plain
// loads or fetched by bulk copies (stage = 1, with one node pair per step).
NodeKern node_kernel(int kind, bool on, bool par, int ilp, int stage) {
    if (stage == 1) return par ? node_kernel<true, 1, true>(kind, on) : node_kernel<false, 1, true>(kind, on);
    if (ilp == 3) return par ? node_kernel<true, 3, false>(kind, on) : node_kernel<false, 3, false>(kind, on);
    if (ilp == 2) return par ? node_kernel<true, 2, false>(kind, on) : node_kernel<false, 2, false>(kind, on);
    return par ? node_kernel<true, 1, false>(kind, on) : node_kernel<false, 1, false>(kind, on);
}

// Scratch layout of spm_batch_adjoint_params (byte offsets, 16-byte aligned):
// the fixed-point adjoint grid, per-unit partials, dk row sums, then the
// per-molecule |ubar| maxima and touched boxes (cleared together), and the
// adjoint grid's clean marker.
struct AdjScratch {
    long long gq, part, dk, umax, box, mark, total;
};
AdjScratch adj_scratch_layout(const long long* totals, int n_mol) {
    AdjScratch L;
    auto up16 = [](long long v) { return (v + 15) / 16 * 16; };
    L.gq = 0;
    L.part = up16(L.gq + totals[7] * 32);
    L.dk = up16(L.part + totals[8] * 48);
    L.umax = up16(L.dk + n_rowblocks(totals[4]) * 32);
    L.box = L.umax + (long long)n_mol * 4;
    L.mark = up16(L.box + (long long)n_mol * 16);
    L.total = L.mark + 16;
    return L;
}

}  // namespace
}  // namespace spm

extern "C" int spm_batch_adjoint_state(int n_mol, const spm_batch_mol* mols, long long n_states,
                                       const spm_batch_shape* shape, const float* grid, const float* points,
                                       const spm_scan_params* p, const float* PPs, const float* dL_dFEs, float* ubar,
                                       float* dk, float* diag, const long long* totals, void* adj_scratch,
                                       void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(p && shape, "spm_batch_adjoint_state: null params/shape");
    SPM_REQUIRE(shape->grid_layout == 0 || shape->grid_layout == 1, "spm_batch_adjoint_state: grid_layout=%d",
                shape->grid_layout);
    SPM_REQUIRE(n_mol >= 0 && n_states >= 0, "spm_batch_adjoint_state: negative sizes");
    if (n_mol == 0 || n_states == 0) return SPM_OK;
    SPM_REQUIRE(mols && grid && points && PPs && dL_dFEs && ubar && diag, "spm_batch_adjoint_state: null pointer");
    SPM_REQUIRE(aligned16(grid) && aligned16(points) && aligned16(PPs) && aligned16(dL_dFEs) && aligned16(ubar) &&
                aligned16(dk) && aligned16(diag), "spm_batch_adjoint_state: buffers not 16-byte aligned");
    const long long nb = (n_states + AG_THREADS - 1) / AG_THREADS;
    SPM_REQUIRE(nb < (1LL << 31), "spm_batch_adjoint_state: too many states");
    cudaStream_t st = as_stream(stream);
    unsigned* umax = nullptr;
    int* box = nullptr;
    if (adj_scratch) {  // the maxima and touched boxes of spm_batch_adjoint_params, from the ubar written here
        SPM_REQUIRE(totals && (reinterpret_cast<uintptr_t>(adj_scratch) & 15u) == 0,
                    "spm_batch_adjoint_state: adj_scratch needs totals and 16-byte alignment");
        const AdjScratch SL = adj_scratch_layout(totals, n_mol);
        char* base = static_cast<char*>(adj_scratch);
        umax = reinterpret_cast<unsigned*>(base + SL.umax);
        box = reinterpret_cast<int*>(base + SL.box);
        if (cudaMemsetAsync(umax, 0, (size_t)(SL.mark - SL.umax), st) != cudaSuccess)
            return set_error(SPM_ERR_CUDA, "spm_batch_adjoint_state: memset failed");
    }
    batch_adjoint_state_kernel<<<(unsigned)nb, AG_THREADS, 0, st>>>(
        n_mol, mols, n_states, shape->grid_layout ? 4 : 2, grid, reinterpret_cast<const float4*>(points), *p,
        reinterpret_cast<const float4*>(PPs),
        reinterpret_cast<const float4*>(dL_dFEs), reinterpret_cast<float4*>(ubar), reinterpret_cast<float4*>(dk),
        reinterpret_cast<float4*>(diag), umax, box);
    return check_launch("spm_batch_adjoint_state");
}

extern "C" long long spm_batch_adjoint_scratch_bytes(const long long* totals, int n_mol) {
    using namespace spm;
    if (!totals || n_mol < 0) return 0;
    return adj_scratch_layout(totals, n_mol).total;
}

extern "C" int spm_batch_adjoint_params(int kind, int n_mol, const spm_batch_mol* mols, const long long* totals,
                                        const spm_batch_shape* shape, const float* atoms, const float* params,
                                        const float* Qs, const float* QZs, const float* PPs, const float* ubar,
                                        const float* dk, double* grad, double* dk_sum, int adj_flags, void* scratch,
                                        void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(kind == SPM_KIND_LJ || kind == SPM_KIND_MORSE, "spm_batch_adjoint_params: kind=%d", kind);
    SPM_REQUIRE((adj_flags & ~(SPM_ADJ_PAIR_PARAMS | SPM_ADJ_STATE_MAXIMA)) == 0,
                "spm_batch_adjoint_params: unknown flags 0x%x", adj_flags);
    SPM_REQUIRE(shape && totals && Qs && QZs && dk_sum && scratch, "spm_batch_adjoint_params: null pointer");
    SPM_REQUIRE(n_mol >= 0, "spm_batch_adjoint_params: n_mol=%d", n_mol);
    const long long n_units = totals[2], n_chunks = totals[3], n_states = totals[4], n_atoms = totals[5];
    SPM_REQUIRE(n_units >= 0 && n_chunks >= 0 && n_states >= 0 && n_atoms >= 0 && totals[7] >= 0 && totals[8] >= 0,
                "spm_batch_adjoint_params: negative totals");
    const int chunk = shape->adj_chunk;
    SPM_REQUIRE(chunk >= 1024 && chunk <= (1 << 20) && chunk % 1024 == 0, "spm_batch_adjoint_params: adj_chunk=%d",
                chunk);
    SPM_REQUIRE(shape->adj_ilp >= 1 && shape->adj_ilp <= 3, "spm_batch_adjoint_params: adj_ilp=%d", shape->adj_ilp);
    SPM_REQUIRE(shape->adj_agg >= 0 && shape->adj_agg <= 2, "spm_batch_adjoint_params: adj_agg=%d", shape->adj_agg);
    SPM_REQUIRE(totals[1] >= 0 && totals[1] < (1LL << 31), "spm_batch_adjoint_params: slots=%lld", totals[1]);
    SPM_REQUIRE(shape->adj_stage == 0 || (shape->adj_stage == 1 && shape->adj_ilp == 1),
                "spm_batch_adjoint_params: adj_stage=%d (1 takes adj_ilp = 1)", shape->adj_stage);
    SPM_REQUIRE((reinterpret_cast<uintptr_t>(scratch) & 15u) == 0, "spm_batch_adjoint_params: scratch not 16-byte aligned");
    SPM_REQUIRE(n_units < (1LL << 31) && n_chunks < (1LL << 31) && n_atoms < (1LL << 30) &&
                (n_states + 255) / 256 < (1LL << 31), "spm_batch_adjoint_params: batch too large");
    cudaStream_t st = as_stream(stream);
    const AdjScratch SL = adj_scratch_layout(totals, n_mol);
    char* base = static_cast<char*>(scratch);
    unsigned long long* gq = reinterpret_cast<unsigned long long*>(base + SL.gq);
    double* part = reinterpret_cast<double*>(base + SL.part);
    double* dkpart = reinterpret_cast<double*>(base + SL.dk);
    unsigned* umax = reinterpret_cast<unsigned*>(base + SL.umax);
    int* box = reinterpret_cast<int*>(base + SL.box);
    unsigned long long* mark = reinterpret_cast<unsigned long long*>(base + SL.mark);
    const unsigned long long clean = adj_clean_token(scratch, SL.total, n_mol);
    bool nodes_ran = false;
    if (n_mol > 0 && n_atoms > 0) {
        SPM_REQUIRE(mols && atoms && params && grad && aligned16(atoms), "spm_batch_adjoint_params: null atoms/grad");
        if (n_states > 0 && n_units > 0) {
            SPM_REQUIRE(PPs && ubar && aligned16(PPs) && aligned16(ubar),
                        "spm_batch_adjoint_params: state buffers null or misaligned");
            static bool smem_set[64] = {};  // the node kernels' dynamic shared memory (> 48 KB), once per device
            int dev = 0;
            if (cudaGetDevice(&dev) != cudaSuccess)
                return set_error(SPM_ERR_CUDA, "spm_batch_adjoint_params: no current device");
            if (dev < 0 || dev >= 64 || !smem_set[dev]) {
                for (int v = 0; v < 32; v++) {
                    const int stage = (v >> 3) == 2 ? 1 : 0, ilp = (v >> 3) == 1 ? 2 : (v >> 3) == 3 ? 3 : 1;
                    const auto k = node_kernel(v & 1 ? SPM_KIND_MORSE : SPM_KIND_LJ, (v & 2) != 0, (v & 4) != 0,
                                               ilp, stage);
                    const size_t bytes = stage ? NM_SMEM_BULK : ilp == 3 ? NM_SMEM_2ATOM : NM_SMEM;
                    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
                        return set_error(SPM_ERR_CUDA, "spm_batch_adjoint_params: cannot set shared memory size");
                }
                if (dev >= 0 && dev < 64) smem_set[dev] = true;
            }
            const bool given = (adj_flags & SPM_ADJ_STATE_MAXIMA) != 0;  // from spm_batch_adjoint_state
            if (!given && cudaMemsetAsync(umax, 0, (size_t)(SL.mark - SL.umax), st) != cudaSuccess)  // maxima + boxes
                return set_error(SPM_ERR_CUDA, "spm_batch_adjoint_params: memset failed");
            adj_clear_kernel<<<1184, 256, 0, st>>>(reinterpret_cast<ulonglong2*>(gq), totals[7] * 2, mark, clean);
            if (!given)
                batch_ubar_max_kernel<<<(unsigned)((n_chunks + UM_CHUNKS - 1) / UM_CHUNKS), 256, 0, st>>>(
                    n_mol, n_chunks, mols, reinterpret_cast<const float4*>(ubar), reinterpret_cast<const float4*>(PPs),
                    umax, box);
            if (shape->adj_agg == 2) {
                int th_log2 = 0;
                while ((1 << th_log2) < shape->rx_tile_h) th_log2++;
                unsigned* counter = reinterpret_cast<unsigned*>(mark + 1) + 1;  // the marker slot's last word
                if (cudaMemsetAsync(counter, 0, sizeof(unsigned), st) != cudaSuccess)
                    return set_error(SPM_ERR_CUDA, "spm_batch_adjoint_params: memset failed");
                int dev_t = 0, sms = 0, per_sm = 0;
                if (cudaGetDevice(&dev_t) != cudaSuccess ||
                    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_t) != cudaSuccess ||
                    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_scatter_tile_kernel, SCT_WARPS * 32,
                                                                  0) != cudaSuccess)
                    return set_error(SPM_ERR_CUDA, "spm_batch_adjoint_params: cannot query the device occupancy");
                const long long need = (totals[1] + SCT_WARPS * 32 - 1) / (SCT_WARPS * 32);
                const long long cap = (long long)sms * (per_sm > 0 ? per_sm : 1);
                batch_scatter_tile_kernel<<<(unsigned)(need < cap ? need : cap), SCT_WARPS * 32, 0, st>>>(
                    n_mol, mols, (unsigned)totals[1], th_log2, reinterpret_cast<const float4*>(PPs),
                    reinterpret_cast<const float4*>(ubar), umax, gq, mark, counter);
            } else if (shape->adj_agg) {
                const size_t agg_smem = sizeof(unsigned long long) * 5 * AGG_SLOTS;
                if (cudaFuncSetAttribute(batch_scatter_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)agg_smem) != cudaSuccess)
                    return set_error(SPM_ERR_CUDA, "spm_batch_adjoint_params: cannot enable %zu B of shared memory",
                                     agg_smem);
                batch_scatter_kernel<true><<<(unsigned)((n_states + 255) / 256), 256, agg_smem, st>>>(
                    n_mol, mols, n_states, reinterpret_cast<const float4*>(PPs), reinterpret_cast<const float4*>(ubar),
                    umax, gq, mark);
            } else {
                batch_scatter_kernel<false><<<(unsigned)((n_states + 255) / 256), 256, 0, st>>>(
                    n_mol, mols, n_states, reinterpret_cast<const float4*>(PPs), reinterpret_cast<const float4*>(ubar),
                    umax, gq, mark);
            }
            const NodeSites S = make_node_sites(Qs, QZs);
            const int pstride = kind == SPM_KIND_MORSE ? 4 : 2;
            const bool on = S.qon != 0.f;
            const auto kern = node_kernel(kind, on, (adj_flags & SPM_ADJ_PAIR_PARAMS) != 0, shape->adj_ilp,
                                          shape->adj_stage);
            // status: the second word of the marker slot (bit 0: a bulk copy's wait ran out)
            unsigned* status = reinterpret_cast<unsigned*>(mark + 1);
            const size_t nm_bytes = shape->adj_stage ? NM_SMEM_BULK : shape->adj_ilp == 3 ? NM_SMEM_2ATOM : NM_SMEM;
            kern<<<(unsigned)n_units, NM_THREADS, nm_bytes, st>>>(
                n_mol, mols, chunk, reinterpret_cast<const float4*>(atoms), params, pstride, S, gq, box, umax, part,
                status);
            nodes_ran = true;
        }
        batch_fold_rows_kernel<<<dim3((unsigned)n_atoms, 6), 256, 0, st>>>(n_mol, mols, chunk, part, grad,
                                                                           nodes_ran ? mark : nullptr, clean);
    }
    if (n_states > 0 && !dk) {  // no spring-parameter terms: dk_sum = 0
        if (cudaMemsetAsync(dk_sum, 0, 4 * sizeof(double), st) != cudaSuccess)
            return set_error(SPM_ERR_CUDA, "spm_batch_adjoint_params: memset failed");
    } else if (n_states > 0) {
        SPM_REQUIRE(aligned16(dk), "spm_batch_adjoint_params: dk not 16-byte aligned");
        const long long rb = n_rowblocks(n_states);
        sum_rows_kernel<<<(unsigned)rb, 256, 0, st>>>(reinterpret_cast<const float4*>(dk), n_states, dkpart);
        fold_chunks_kernel<<<dim3(1, 4), 256, 0, st>>>(dkpart, (int)rb, 4, dk_sum);
    } else if (cudaMemsetAsync(dk_sum, 0, 4 * sizeof(double), st) != cudaSuccess) {
        return set_error(SPM_ERR_CUDA, "spm_batch_adjoint_params: memset failed");
    }
    return check_launch("spm_batch_adjoint_params");
}

extern "C" int spm_adjoint_grid_state(const float* grid, int nx, int ny, int nz, const float* points, int n_scan,
                                      const spm_scan_params* p, const float* PPs, const float* dL_dFEs, float* ubar,
                                      float* dk, float* diag, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(p && grid, "spm_adjoint_grid_state: null grid/params");
    SPM_REQUIRE(nx > 0 && ny > 0 && nz > 0 && n_scan >= 0 && p->nz >= 0, "spm_adjoint_grid_state: bad sizes");
    const long long n_state = (long long)n_scan * p->nz;
    if (n_state == 0) return SPM_OK;
    SPM_REQUIRE(points && PPs && dL_dFEs && ubar && dk && diag, "spm_adjoint_grid_state: null pointer");
    SPM_REQUIRE(aligned16(grid) && aligned16(points) && aligned16(PPs) && aligned16(dL_dFEs) && aligned16(ubar) &&
                aligned16(dk) && aligned16(diag), "spm_adjoint_grid_state: buffers not 16-byte aligned");
    adjoint_grid_state_kernel<<<(unsigned)((n_state + AG_THREADS - 1) / AG_THREADS), AG_THREADS, 0,
                                as_stream(stream)>>>(
        view_of(grid, nx, ny, nz, p), reinterpret_cast<const float4*>(points), n_scan, *p,
        reinterpret_cast<const float4*>(PPs), reinterpret_cast<const float4*>(dL_dFEs),
        reinterpret_cast<float4*>(ubar), reinterpret_cast<float4*>(dk), reinterpret_cast<float4*>(diag));
    return check_launch("spm_adjoint_grid_state");
}

extern "C" long long spm_adjoint_grid_scratch_bytes(int n_atoms, long long n_state) {
    using namespace spm;
    if (n_atoms < 0 || n_state < 0) return 0;
    return ((long long)n_atoms * n_chunks(n_state) * 6 + n_rowblocks(n_state) * 4) * (long long)sizeof(double);
}

extern "C" int spm_adjoint_grid_params(int kind, int n_atoms, const float* atoms, const float* params,
                                       const float* p0, const float* dA, const float* dB, const float* dC,
                                       const float* Qs, const float* QZs, const float* grid, int nx, int ny, int nz,
                                       const spm_scan_params* p, const float* PPs, const float* ubar,
                                       const float* dk, long long n_state, double* grad, double* dk_sum,
                                       void* scratch, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(kind == SPM_KIND_LJ || kind == SPM_KIND_MORSE, "spm_adjoint_grid_params: kind=%d", kind);
    SPM_REQUIRE(n_atoms >= 0 && n_atoms <= 65535, "spm_adjoint_grid_params: n_atoms=%d outside [0,65535]", n_atoms);
    SPM_REQUIRE(p && p0 && dA && dB && dC && Qs && QZs && grid && grad && dk_sum && scratch,
                "spm_adjoint_grid_params: null pointer");
    SPM_REQUIRE(n_state >= 0 && nx > 0 && ny > 0 && nz > 0, "spm_adjoint_grid_params: bad sizes");
    if (n_state > 0)
        SPM_REQUIRE(PPs && ubar && dk && aligned16(PPs) && aligned16(ubar) && aligned16(dk),
                    "spm_adjoint_grid_params: state buffers null or misaligned");
    if (n_atoms > 0) SPM_REQUIRE(atoms && params && aligned16(atoms), "spm_adjoint_grid_params: null atoms/params");
    SPM_REQUIRE((reinterpret_cast<uintptr_t>(scratch) & 7u) == 0, "spm_adjoint_grid_params: scratch not 8-byte aligned");
    Sites S = {};
    for (int k = 0; k < 4; k++) { S.qs[k] = Qs[k] * COULOMB_CONST; S.qz[k] = QZs[k]; }
    NodeGeom NG;
    NG.p0 = make_float4(p0[0], p0[1], p0[2], p0[3]);
    NG.dA = make_float4(dA[0], dA[1], dA[2], dA[3]);
    NG.dB = make_float4(dB[0], dB[1], dB[2], dB[3]);
    NG.dC = make_float4(dC[0], dC[1], dC[2], dC[3]);
    const long long chunks = n_chunks(n_state);
    const long long rb = n_rowblocks(n_state);
    SPM_REQUIRE(chunks < (1LL << 31), "spm_adjoint_grid_params: too many states");
    double* part = static_cast<double*>(scratch);
    double* dkpart = part + (size_t)n_atoms * chunks * 6;
    cudaStream_t st = as_stream(stream);
    const GridView G = view_of(grid, nx, ny, nz, p);
    const int pstride = kind == SPM_KIND_MORSE ? 4 : 2;
    if (n_atoms > 0) {
        if (n_state > 0) {
            dim3 grd((unsigned)chunks, (unsigned)n_atoms);
            if (kind == SPM_KIND_LJ)
                adjoint_grid_atoms_kernel<SPM_KIND_LJ><<<grd, AG_THREADS, 0, st>>>(
                    n_atoms, reinterpret_cast<const float4*>(atoms), params, pstride, S, NG, G,
                    reinterpret_cast<const float4*>(PPs), reinterpret_cast<const float4*>(ubar), n_state, part);
            else
                adjoint_grid_atoms_kernel<SPM_KIND_MORSE><<<grd, AG_THREADS, 0, st>>>(
                    n_atoms, reinterpret_cast<const float4*>(atoms), params, pstride, S, NG, G,
                    reinterpret_cast<const float4*>(PPs), reinterpret_cast<const float4*>(ubar), n_state, part);
        } else if (cudaMemsetAsync(part, 0, (size_t)n_atoms * 6 * sizeof(double), st) != cudaSuccess) {
            return set_error(SPM_ERR_CUDA, "spm_adjoint_grid_params: memset failed");
        }
        fold_chunks_kernel<<<dim3((unsigned)n_atoms, 6), 256, 0, st>>>(part, n_state > 0 ? (int)chunks : 1, 6, grad);
    }
    if (n_state > 0) {
        sum_rows_kernel<<<(unsigned)rb, 256, 0, st>>>(reinterpret_cast<const float4*>(dk), n_state, dkpart);
        fold_chunks_kernel<<<dim3(1, 4), 256, 0, st>>>(dkpart, (int)rb, 4, dk_sum);
    } else if (cudaMemsetAsync(dk_sum, 0, 4 * sizeof(double), st) != cudaSuccess) {
        return set_error(SPM_ERR_CUDA, "spm_adjoint_grid_params: memset failed");
    }
    return check_launch("spm_adjoint_grid_params");
}
