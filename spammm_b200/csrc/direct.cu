// direct.cu -- grid-free Morse + point-charge Coulomb probe relaxation and its
// implicit-function adjoint.
//
// Replaces SPAMMM's differentiable direct path (kernels/AFM.cl:1391-2029,
// host AFMulator.run_scan_morse_direct / vjp_scan_morse_direct,
// spammm/SPM/AFM.py:2063-2519):
//   relax_direct_kernel     <- relaxStrokesTiltedMorseDirect (AFM.cl:1419-1511)
//   adjoint_state_kernel    <- morseDirectStateAdjoint       (AFM.cl:1711-1845)
//   adjoint_partials_kernel <- morseDirectParamPartials      (AFM.cl:1850-1992)
//   adjoint_reduce_kernel   <- reduceMorseDirectParamPartials (AFM.cl:1996-2029)
//
// B200 shape.  The forward keeps every atom of the molecule in shared memory
// in the pre-transformed form of the grid builder (MUFU rsqrt/ex2 inner loop)
// and gives each pixel a group of 4-32 lanes that split the atoms of every
// force evaluation and sum them by a butterfly, each lane then holding the same
// stroke state in registers -- a scan of 10^4 pixels fills the GPU, and a FIRE
// step costs the latency of na/LPP pair terms instead of na.  The adjoint solves one symmetric
// 3x3 system per state in registers (cofactors, as the reference) and forms
// the per-atom parameter partials with a CTA per (atom, 128-scan chunk) that
// reduces in shared memory in a fixed order; a second pass folds the chunks in
// a fixed order.  No floating-point atomics: the gradient is bit-reproducible.
#include "spm_internal.cuh"
#include "spm_fire.cuh"

namespace spm {
namespace {

constexpr int DX_THREADS = 128;
constexpr float R2SAFE = 1e-4f;
constexpr float COULOMB_CONST = 14.3996448915f;
constexpr float LOG2E = 1.4426950408889634f;

__device__ __forceinline__ float fast_rsqrt(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float fast_ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

struct Sites {
    float qs[4];  // Qs[k]*COULOMB_CONST (all four sites, zero allowed)
    float qz[4];
    double qs64[4];  // the same sites in FP64 (Qs[k] * COULOMB_CONST in double), for the convergence check
    double qz64[4];
    int ns;
};

__device__ __forceinline__ void stage_atoms(int na, const float4* __restrict__ atoms, const float4* __restrict__ cMs,
                                            const float* qs_nz, int ns, float4* s_pos, float4* s_m, float* s_q) {
    for (int j = threadIdx.x; j < na; j += blockDim.x) {
        const float4 a = __ldg(atoms + j);
        const float4 c = __ldg(cMs + j);
        s_pos[j] = make_float4(a.x, a.y, a.z, a.w);
        s_m[j] = make_float4(c.z * LOG2E, -c.z * c.x * LOG2E, c.y, -2.f * c.z * c.y);
        for (int k = 0; k < ns; k++) s_q[k * na + j] = a.w * qs_nz[k];
    }
}

// LPP lanes per pixel: the group's lanes split the atoms (lane `sub` takes atoms sub, sub + LPP, ...)
// and sum their partial forces by an xor butterfly over the group, so every lane of the group ends
// with the same bits (each level adds the same two values, in either order) and runs the same FIRE
// update: the group stays converged without a broadcast.  gmask: the group's lanes.
template <int LPP>
__device__ __forceinline__ float group_sum(float v, unsigned gmask) {
#pragma unroll
    for (int o = 1; o < LPP; o <<= 1) v += __shfl_xor_sync(gmask, v, o);
    return v;
}
template <int LPP>
__device__ __forceinline__ double group_sum(double v, unsigned gmask) {
#pragma unroll
    for (int o = 1; o < LPP; o <<= 1) v += __shfl_xor_sync(gmask, v, o);
    return v;
}

template <int NS, int LPP>
__device__ __forceinline__ float4 group_pair_sum(V3 p, int na, int sub, unsigned gmask, const float4* s_pos,
                                                 const float4* s_m, const float* s_q, const float* qz) {
    float fx = 0.f, fy = 0.f, fz = 0.f, fe = 0.f;
    for (int j = sub; j < na; j += LPP) {
        const float4 a = s_pos[j];
        const float4 m = s_m[j];
        const float dx = p.x - a.x, dy = p.y - a.y, dz = p.z - a.z;
        const float dxy2 = fmaf(dx, dx, fmaf(dy, dy, R2SAFE));
        const float r2 = fmaf(dz, dz, dxy2);
        const float rs = fast_rsqrt(r2);
        const float r = r2 * rs;
        const float e = fast_ex2(fmaf(m.x, r, m.y));
        fe = fmaf(m.z * e, e - 2.f, fe);
        const float sg = (m.w * e) * (e - 1.f) * rs;
        fx = fmaf(dx, sg, fx);
        fy = fmaf(dy, sg, fy);
        fz = fmaf(dz, sg, fz);
#pragma unroll
        for (int k = 0; k < NS; k++) {
            const float dzk = dz + qz[k];
            const float rsk = fast_rsqrt(fmaf(dzk, dzk, dxy2));
            const float Ek = s_q[k * na + j] * rsk;
            fe += Ek;
            const float sk = Ek * rsk * rsk;
            fx = fmaf(dx, sk, fx);
            fy = fmaf(dy, sk, fy);
            fz = fmaf(dzk, sk, fz);
        }
    }
    return make_float4(group_sum<LPP>(fx, gmask), group_sum<LPP>(fy, gmask), group_sum<LPP>(fz, gmask),
                       group_sum<LPP>(fe, gmask));
}

// |total force|^2 at p in FP64 -- the Morse + Coulomb sums from the atoms' float32 inputs with IEEE
// double exp/sqrt (the reference's FP64 pair law, kernels/AFM.cl:730-757 in double), the spring and the
// surface bias -- to confirm a convergence the FP32 sums report: near |F|^2 = f2conv their rounding
// (MUFU rsqrt/ex2, and the radial spring's r - d0 of a 4 A bond at float32 resolution) can put the
// FP32 test on the converged side of a state whose force is not.  The atoms are split over the
// group and the FP64 sums reduced by the same butterfly.
template <int LPP>
__device__ __noinline__ double group_force2_f64(V3 p, V3 tip, int na, int sub, unsigned gmask,
                                                const float4* __restrict__ atoms, const float4* __restrict__ cMs,
                                                const Sites& S, V3 a, V3 b, V3 c, float4 kk, float4 d0, float surf) {
    const double px = p.x, py = p.y, pz = p.z;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int j = sub; j < na; j += LPP) {
        const float4 at = __ldg(atoms + j);
        const float4 cm = __ldg(cMs + j);
        const double dx = px - at.x, dy = py - at.y, dz = pz - at.z;
        const double dxy2 = dx * dx + dy * dy;
        const double r = sqrt(dxy2 + dz * dz + 1e-4);
        const double K = cm.z, R0 = cm.x, E0 = cm.y;
        const double e = exp(K * (r - R0));
        const double sr = (-E0 * e * (e - 1.0) * 2.0 * K) / r;
        fx += dx * sr;
        fy += dy * sr;
        fz += dz * sr;
        for (int k = 0; k < S.ns; k++) {
            if (S.qs64[k] == 0.0) continue;
            const double dzk = dz + S.qz64[k];
            const double ir2 = 1.0 / (dxy2 + dzk * dzk + 1e-4);
            const double sk = S.qs64[k] * (double)at.w * sqrt(ir2) * ir2;
            fx += dx * sk;
            fy += dy * sk;
            fz += dzk * sk;
        }
    }
    fx = group_sum<LPP>(fx, gmask);
    fy = group_sum<LPP>(fy, gmask);
    fz = group_sum<LPP>(fz, gmask);
    const double ex = (double)p.x - tip.x, ey = (double)p.y - tip.y, ez = (double)p.z - tip.z;
    const double dl[3] = {ex * a.x + ey * a.y + ez * a.z, ex * b.x + ey * b.y + ez * b.z, ex * c.x + ey * c.y + ez * c.z};
    double ft[3] = {(dl[0] - d0.x) * kk.x, (dl[1] - d0.y) * kk.y, (dl[2] - d0.z) * kk.z};
    if (kk.w != 0.f) {
        double r = sqrt(dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2]);
        r = r > 1e-10 ? r : 1e-10;
        const double sr = kk.w * (r - d0.w) / r;
        for (int i = 0; i < 3; i++) ft[i] += dl[i] * sr;
    }
    fx += a.x * ft[0] + b.x * ft[1] + c.x * ft[2] + c.x * (double)surf;
    fy += a.y * ft[0] + b.y * ft[1] + c.y * ft[2] + c.y * (double)surf;
    fz += a.z * ft[0] + b.z * ft[1] + c.z * ft[2] + c.z * (double)surf;
    return fx * fx + fy * fy + fz * fz;
}

// Groups of LPP lanes, one pixel per group (DX_THREADS / LPP pixels per CTA, in raster order); the
// whole molecule staged in shared memory; each group runs its pixel's (z-step, FIRE step) sequence
// with the stroke state held identically by every lane of the group.  Convergence is tested before
// the update, and an FP32 "converged" is confirmed in FP64.
template <int NS, int LPP>
__global__ void __launch_bounds__(DX_THREADS)
relax_direct_kernel(int na, const float4* __restrict__ atoms, const float4* __restrict__ cMs,
                    const float4* __restrict__ pts, int n_scan, spm_scan_params P, Sites S,
                    float4* __restrict__ FEs, float4* __restrict__ PPs) {
    extern __shared__ float4 smem[];
    float4* s_pos = smem;
    float4* s_m = smem + na;
    float* s_q = reinterpret_cast<float*>(smem + 2 * na);
    stage_atoms(na, atoms, cMs, S.qs, NS, s_pos, s_m, s_q);
    __syncthreads();
    const int lane = threadIdx.x & 31, sub = lane & (LPP - 1);
    const unsigned gmask = (LPP == 32) ? 0xffffffffu : (((1u << LPP) - 1u) << (lane & ~(LPP - 1)));
    const int k = blockIdx.x * (DX_THREADS / LPP) + threadIdx.x / LPP;
    if (k >= n_scan) return;  // the whole group

    const float4 kk = make_float4(P.stiffness[0], P.stiffness[1], P.stiffness[2], P.stiffness[3]);
    const float4 d0 = make_float4(P.dpos0[0], P.dpos0[1], P.dpos0[2], P.dpos0[3]);
    const V3 a = mk3(P.tipA[0], P.tipA[1], P.tipA[2]);
    const V3 b = mk3(P.tipB[0], P.tipB[1], P.tipB[2]);
    const V3 c = mk3(P.tipC[0], P.tipC[1], P.tipC[2]);
    const V3 dTip = mk3(c.x * P.tipC[3], c.y * P.tipC[3], c.z * P.tipC[3]);
    const float surf = P.surfFF[0];
    const float4 p4 = pts[k];
    V3 tip = mk3(p4.x, p4.y, p4.z);
    V3 pos = add3(tip, rotmatT(mk3(d0.x, d0.y, d0.z), a, b, c));
    Integrator I;
    I.dt = P.relax_params[0];
    I.damp = P.relax_params[1];
    I.dtmax = I.dt;
    I.dtmin = I.dtmax * 0.1f;
    I.damp0 = I.damp;

    float4* fe_out = FEs + (size_t)k * P.nz;
    float4* pp_out = PPs + (size_t)k * P.nz;
    V3 v = mk3(0.f, 0.f, 0.f);
    int iz = 0, it = 0;
    while (iz < P.nz) {
        bool done = false, conv = false;
        float4 fe = make_float4(0.f, 0.f, 0.f, 0.f);
        if (it < P.max_iter) {
            ++it;
            fe = group_pair_sum<NS, LPP>(pos, na, sub, gmask, s_pos, s_m, s_q, S.qz);
            const V3 ft = rotmatT(tip_force(rotmat(sub3(pos, tip), a, b, c), kk, d0), a, b, c);
            V3 f = mk3(fe.x + ft.x, fe.y + ft.y, fe.z + ft.z);
            f.x = fmaf(c.x, surf, f.x);
            f.y = fmaf(c.y, surf, f.y);
            f.z = fmaf(c.z, surf, f.z);
            if (dot3(f, f) < P.f2conv &&
                group_force2_f64<LPP>(pos, tip, na, sub, gmask, atoms, cMs, S, a, b, c, kk, d0, surf) <
                    (double)P.f2conv) {
                done = conv = true;
            } else {
                md_step(f, v, pos, I, true);
                done = (it >= P.max_iter);
            }
        } else {
            done = true;  // max_iter == 0
        }
        if (done) {
            if (!conv) fe = group_pair_sum<NS, LPP>(pos, na, sub, gmask, s_pos, s_m, s_q, S.qz);  // moved since
            if (sub == 0) {
                const V3 r = rotmat(mk3(fe.x, fe.y, fe.z), a, b, c);
                fe_out[iz] = make_float4(r.x, r.y, r.z, fe.w);
                const bool finite = isfinite(fe.x) && isfinite(fe.y) && isfinite(fe.z) && isfinite(fe.w) &&
                                    isfinite(pos.x) && isfinite(pos.y) && isfinite(pos.z);
                pp_out[iz] = make_float4(pos.x, pos.y, pos.z, (float)((conv && finite) ? it : -it));
            }
            tip = add3(tip, dTip);
            pos = add3(pos, dTip);
            v = mk3(0.f, 0.f, 0.f);
            it = 0;
            ++iz;
        }
    }
}

// ---------------------------------------------------------------- adjoint
struct Sym3 {
    float xx, xy, xz, yy, yz, zz;
};

__device__ __forceinline__ void add_outer(Sym3& H, V3 d, float co, float cd) {
    H.xx += co * d.x * d.x + cd;
    H.xy += co * d.x * d.y;
    H.xz += co * d.x * d.z;
    H.yy += co * d.y * d.y + cd;
    H.yz += co * d.y * d.z;
    H.zz += co * d.z * d.z + cd;
}

__device__ __forceinline__ V3 sym_mul(const Sym3& H, V3 u) {
    return mk3(H.xx * u.x + H.xy * u.y + H.xz * u.z, H.xy * u.x + H.yy * u.y + H.yz * u.z,
               H.xz * u.x + H.yz * u.y + H.zz * u.z);
}

// Sample FE and energy Hessian at q (AFM.cl:1549-1622), accurate FP32 math.
__device__ void fe_hessian(V3 q, int na, const float4* s_pos, const float4* s_c, const Sites& S, float4& fe, Sym3& H) {
    fe = make_float4(0.f, 0.f, 0.f, 0.f);
    H = Sym3{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int j = 0; j < na; j++) {
        const float4 at = s_pos[j];
        const float4 cm = s_c[j];
        const V3 d = mk3(q.x - at.x, q.y - at.y, q.z - at.z);
        const float r2 = d.x * d.x + d.y * d.y + d.z * d.z + R2SAFE;
        const float r = sqrtf(r2);
        const float R0 = cm.x, E0 = cm.y, K = cm.z;
        const float s = expf(K * (r - R0));
        const float Ep = 2.f * K * E0 * s * (s - 1.f);
        const float Epp = 2.f * K * K * E0 * s * (2.f * s - 1.f);
        const float fr = -Ep / r;
        fe.x += d.x * fr; fe.y += d.y * fr; fe.z += d.z * fr;
        fe.w += E0 * s * (s - 2.f);
        add_outer(H, d, (Epp - Ep / r) / r2, Ep / r);
        for (int k = 0; k < 4; k++) {
            if (S.qs[k] == 0.f) continue;
            const V3 dk = mk3(d.x, d.y, d.z + S.qz[k]);
            const float rk2 = dk.x * dk.x + dk.y * dk.y + dk.z * dk.z + R2SAFE;
            const float rk = sqrtf(rk2);
            const float rk3 = rk * rk2, rk5 = rk3 * rk2;
            const float C = at.w * S.qs[k];
            fe.x += dk.x * (C / rk3); fe.y += dk.y * (C / rk3); fe.z += dk.z * (C / rk3);
            fe.w += C / rk;
            add_outer(H, dk, 3.f * C / rk5, -C / rk3);
        }
    }
}

__device__ float eigmin_sym(const Sym3& A) {
    // Smallest eigenvalue of a symmetric 3x3 (trigonometric closed form, AFM.cl:1652-1672).
    const float p1 = A.xy * A.xy + A.xz * A.xz + A.yz * A.yz;
    const float q = (A.xx + A.yy + A.zz) / 3.f;
    const float p2 = (A.xx - q) * (A.xx - q) + (A.yy - q) * (A.yy - q) + (A.zz - q) * (A.zz - q) + 2.f * p1;
    const float p = sqrtf(p2 / 6.f);
    if (p < 1e-20f) return q;
    const float b00 = (A.xx - q) / p, b11 = (A.yy - q) / p, b22 = (A.zz - q) / p;
    const float b01 = A.xy / p, b02 = A.xz / p, b12 = A.yz / p;
    const float detB = b00 * (b11 * b22 - b12 * b12) - b01 * (b01 * b22 - b12 * b02) + b02 * (b01 * b12 - b11 * b02);
    const float rr = fmaxf(-1.f, fminf(1.f, detB * 0.5f));
    const float phi = acosf(rr) / 3.f;
    const float e1 = q + 2.f * p * cosf(phi);
    const float e3 = q + 2.f * p * cosf(phi + 2.0943951023931953f);
    const float e2 = 3.f * q - e1 - e3;
    return fminf(e1, fminf(e2, e3));
}

__global__ void __launch_bounds__(DX_THREADS)
adjoint_state_kernel(int na, const float4* __restrict__ atoms, const float4* __restrict__ cMs,
                     const float4* __restrict__ pts, int n_scan, spm_scan_params P, Sites S,
                     const float4* __restrict__ PPs, const float4* __restrict__ dL, float4* __restrict__ lam,
                     float4* __restrict__ diag) {
    extern __shared__ float4 smem[];
    float4* s_pos = smem;
    float4* s_c = smem + na;
    for (int j = threadIdx.x; j < na; j += blockDim.x) {
        s_pos[j] = __ldg(atoms + j);
        s_c[j] = __ldg(cMs + j);
    }
    __syncthreads();
    const long long st = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (st >= (long long)n_scan * P.nz) return;
    const int iscan = (int)(st / P.nz), iz = (int)(st % P.nz);
    const float4 pp = PPs[st];
    const float4 u = dL[st];
    const bool fin = isfinite(pp.x) && isfinite(pp.y) && isfinite(pp.z) && isfinite(pp.w) && isfinite(u.x) &&
                     isfinite(u.y) && isfinite(u.z) && isfinite(u.w);
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!fin) { lam[st] = zero; diag[st] = make_float4(0.f, 0.f, 0.f, 2.f); return; }
    if (pp.w <= 0.f) { lam[st] = zero; diag[st] = make_float4(0.f, 0.f, 0.f, 1.f); return; }
    const V3 a = mk3(P.tipA[0], P.tipA[1], P.tipA[2]);
    const V3 b = mk3(P.tipB[0], P.tipB[1], P.tipB[2]);
    const V3 c = mk3(P.tipC[0], P.tipC[1], P.tipC[2]);
    const float4 p4 = pts[iscan];
    const V3 tip = mk3(p4.x + c.x * P.tipC[3] * (float)iz, p4.y + c.y * P.tipC[3] * (float)iz,
                       p4.z + c.z * P.tipC[3] * (float)iz);
    const V3 q = mk3(pp.x, pp.y, pp.z);
    float4 fe;
    Sym3 H;
    fe_hessian(q, na, s_pos, s_c, S, fe, H);
    const float4 kk = make_float4(P.stiffness[0], P.stiffness[1], P.stiffness[2], P.stiffness[3]);
    const float4 d0 = make_float4(P.dpos0[0], P.dpos0[1], P.dpos0[2], P.dpos0[3]);
    const V3 dl = rotmat(sub3(q, tip), a, b, c);
    const V3 ft = rotmatT(tip_force(dl, kk, d0), a, b, c);
    const V3 G = mk3(fe.x + ft.x + c.x * P.surfFF[0], fe.y + ft.y + c.y * P.surfFF[0], fe.z + ft.z + c.z * P.surfFF[0]);
    const float resid = sqrtf(G.x * G.x + G.y * G.y + G.z * G.z);
    if (resid >= 5e-4f) { lam[st] = zero; diag[st] = make_float4(resid, 0.f, 0.f, 1.f); return; }
    if (!(isfinite(H.xx) && isfinite(H.xy) && isfinite(H.xz) && isfinite(H.yy) && isfinite(H.yz) && isfinite(H.zz))) {
        lam[st] = zero; diag[st] = make_float4(resid, 0.f, 0.f, 2.f); return;
    }
    // tip-force Jacobian in tip coordinates (AFM.cl:1627-1639)
    float r = sqrtf(dl.x * dl.x + dl.y * dl.y + dl.z * dl.z);
    r = fmaxf(r, 1e-10f);
    const float phi = kk.w * (1.f - d0.w / r);
    const float beta = kk.w * d0.w / (r * r * r);
    const float Jt[3][3] = {{kk.x + phi + beta * dl.x * dl.x, beta * dl.x * dl.y, beta * dl.x * dl.z},
                            {beta * dl.y * dl.x, kk.y + phi + beta * dl.y * dl.y, beta * dl.y * dl.z},
                            {beta * dl.z * dl.x, beta * dl.z * dl.y, kk.z + phi + beta * dl.z * dl.z}};
    const float R[3][3] = {{a.x, a.y, a.z}, {b.x, b.y, b.z}, {c.x, c.y, c.z}};
    float Jw[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            float s = 0.f;
            for (int m = 0; m < 3; m++)
                for (int n = 0; n < 3; n++) s += R[m][i] * Jt[m][n] * R[n][j];
            Jw[i][j] = s;
        }
    const float j00 = Jw[0][0] - H.xx, j01 = Jw[0][1] - H.xy, j02 = Jw[0][2] - H.xz;
    const float j11 = Jw[1][1] - H.yy, j12 = Jw[1][2] - H.yz, j22 = Jw[2][2] - H.zz;
    const V3 uw = rotmatT(mk3(u.x, u.y, u.z), a, b, c);
    const V3 Hu = sym_mul(H, uw);
    const V3 bv = mk3(-Hu.x - fe.x * u.w, -Hu.y - fe.y * u.w, -Hu.z - fe.z * u.w);
    const float a00 = j11 * j22 - j12 * j12, a01 = j02 * j12 - j01 * j22, a02 = j01 * j12 - j02 * j11;
    const float a11 = j00 * j22 - j02 * j02, a12 = j01 * j02 - j00 * j12, a22 = j00 * j11 - j01 * j01;
    const float det = j00 * a00 + j01 * a01 + j02 * a02;
    const float scale = fmaxf(fmaxf(fabsf(j00), fmaxf(fabsf(j11), fabsf(j22))), 1e-20f);
    if (fabsf(det) < 1e-18f * scale * scale * scale) {
        lam[st] = zero; diag[st] = make_float4(resid, 0.f, 0.f, 4.f); return;
    }
    const float id = 1.f / det;
    const V3 l = mk3((a00 * bv.x + a01 * bv.y + a02 * bv.z) * id, (a01 * bv.x + a11 * bv.y + a12 * bv.z) * id,
                     (a02 * bv.x + a12 * bv.y + a22 * bv.z) * id);
    if (!(isfinite(l.x) && isfinite(l.y) && isfinite(l.z))) {
        lam[st] = zero; diag[st] = make_float4(resid, 0.f, 0.f, 2.f); return;
    }
    const Sym3 negJ{-j00, -j01, -j02, -j11, -j12, -j22};
    const float lmin = eigmin_sym(negJ);
    if (lmin <= 1e-5f) { lam[st] = zero; diag[st] = make_float4(resid, lmin, 0.f, 3.f); return; }
    const float jinf = fmaxf(fabsf(j00) + fabsf(j01) + fabsf(j02),
                             fmaxf(fabsf(j01) + fabsf(j11) + fabsf(j12), fabsf(j02) + fabsf(j12) + fabsf(j22)));
    const float ainf = fmaxf(fabsf(a00) + fabsf(a01) + fabsf(a02),
                             fmaxf(fabsf(a01) + fabsf(a11) + fabsf(a12), fabsf(a02) + fabsf(a12) + fabsf(a22)));
    const float cond = jinf * (ainf / fmaxf(fabsf(det), 1e-30f));
    if (!(cond < 1e6f)) { lam[st] = zero; diag[st] = make_float4(resid, lmin, cond, 4.f); return; }
    lam[st] = make_float4(l.x, l.y, l.z, 0.f);
    diag[st] = make_float4(resid, lmin, cond, 0.f);
}

constexpr int PART_THREADS = 128;

// grid (n_chunks, n_atoms): thread = one scan; partial over z; CTA tree-reduce.
__global__ void __launch_bounds__(PART_THREADS)
adjoint_partials_kernel(int na, const float4* __restrict__ atoms, const float4* __restrict__ cMs,
                        const float4* __restrict__ pts, int n_scan, spm_scan_params P, Sites S,
                        const float4* __restrict__ PPs, const float4* __restrict__ dL,
                        const float4* __restrict__ lam, float* __restrict__ partial) {
    __shared__ float red[6][PART_THREADS];
    const int ia = blockIdx.y;
    const int is = blockIdx.x * PART_THREADS + threadIdx.x;
    float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (is < n_scan) {
        const float4 at = __ldg(atoms + ia);
        const float4 cm = __ldg(cMs + ia);
        const V3 a = mk3(P.tipA[0], P.tipA[1], P.tipA[2]);
        const V3 b = mk3(P.tipB[0], P.tipB[1], P.tipB[2]);
        const V3 c = mk3(P.tipC[0], P.tipC[1], P.tipC[2]);
        for (int iz = 0; iz < P.nz; iz++) {
            const size_t st = (size_t)is * P.nz + iz;
            const float4 pp = PPs[st], u = dL[st], lm = lam[st];
            const bool fin = isfinite(pp.x) && isfinite(pp.y) && isfinite(pp.z) && isfinite(pp.w) && isfinite(u.x) &&
                             isfinite(u.y) && isfinite(u.z) && isfinite(u.w) && isfinite(lm.x) && isfinite(lm.y) &&
                             isfinite(lm.z);
            if (pp.w <= 0.f || !fin) continue;
            if (u.x * u.x + u.y * u.y + u.z * u.z + u.w * u.w == 0.f && lm.x * lm.x + lm.y * lm.y + lm.z * lm.z == 0.f)
                continue;
            const V3 uw = rotmatT(mk3(u.x, u.y, u.z), a, b, c);
            const V3 w = mk3(uw.x - lm.x, uw.y - lm.y, uw.z - lm.z);
            const float uE = u.w;
            const V3 d = mk3(pp.x - at.x, pp.y - at.y, pp.z - at.z);
            const float r2 = d.x * d.x + d.y * d.y + d.z * d.z + R2SAFE;
            const float r = sqrtf(r2);
            const float R0 = cm.x, E0 = cm.y, K = cm.z;
            const float s = expf(K * (r - R0));
            const float Ep = 2.f * K * E0 * s * (s - 1.f);
            const float Epp = 2.f * K * K * E0 * s * (2.f * s - 1.f);
            V3 F = mk3(d.x * (-Ep / r), d.y * (-Ep / r), d.z * (-Ep / r));
            Sym3 Hi{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            add_outer(Hi, d, (Epp - Ep / r) / r2, Ep / r);
            const float dFdR0 = 2.f * K * K * E0 * s * (2.f * s - 1.f) / r;  // times d
            const float dFdE0 = -2.f * K * s * (s - 1.f) / r;                // times d
            const float dEdR0 = -2.f * K * E0 * s * (s - 1.f);
            const float dEdE0 = s * (s - 2.f);
            V3 dFdQ = mk3(0.f, 0.f, 0.f);
            float dEdQ = 0.f;
            for (int k = 0; k < 4; k++) {
                if (S.qs[k] == 0.f) continue;
                const V3 dk = mk3(d.x, d.y, d.z + S.qz[k]);
                const float rk2 = dk.x * dk.x + dk.y * dk.y + dk.z * dk.z + R2SAFE;
                const float rk = sqrtf(rk2);
                const float rk3 = rk * rk2, rk5 = rk3 * rk2;
                const float C = at.w * S.qs[k];
                F = add3(F, mk3(dk.x * (C / rk3), dk.y * (C / rk3), dk.z * (C / rk3)));
                dFdQ = add3(dFdQ, mk3(dk.x * (S.qs[k] / rk3), dk.y * (S.qs[k] / rk3), dk.z * (S.qs[k] / rk3)));
                dEdQ += S.qs[k] / rk;
                add_outer(Hi, dk, 3.f * C / rk5, -C / rk3);
            }
            const V3 Hw = sym_mul(Hi, w);
            acc[0] += Hw.x + F.x * uE;
            acc[1] += Hw.y + F.y * uE;
            acc[2] += Hw.z + F.z * uE;
            acc[3] += (w.x * d.x + w.y * d.y + w.z * d.z) * dFdR0 + uE * dEdR0;
            acc[4] += (w.x * d.x + w.y * d.y + w.z * d.z) * dFdE0 + uE * dEdE0;
            acc[5] += (w.x * dFdQ.x + w.y * dFdQ.y + w.z * dFdQ.z) + uE * dEdQ;
        }
    }
#pragma unroll
    for (int c6 = 0; c6 < 6; c6++) red[c6][threadIdx.x] = acc[c6];
    __syncthreads();
    for (int s = PART_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
#pragma unroll
            for (int c6 = 0; c6 < 6; c6++) red[c6][threadIdx.x] += red[c6][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x < 6) partial[((size_t)ia * gridDim.x + blockIdx.x) * 6 + threadIdx.x] = red[threadIdx.x][0];
}

// One CTA per atom folds its chunk partials in a fixed order.
__global__ void __launch_bounds__(256)
adjoint_reduce_kernel(const float* __restrict__ partial, int n_chunks, float* __restrict__ grad) {
    __shared__ float red[6][256];
    const int ia = blockIdx.x;
    float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int ch = threadIdx.x; ch < n_chunks; ch += 256)
#pragma unroll
        for (int c6 = 0; c6 < 6; c6++) acc[c6] += partial[((size_t)ia * n_chunks + ch) * 6 + c6];
#pragma unroll
    for (int c6 = 0; c6 < 6; c6++) red[c6][threadIdx.x] = acc[c6];
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
#pragma unroll
            for (int c6 = 0; c6 < 6; c6++) red[c6][threadIdx.x] += red[c6][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x < 6) grad[(size_t)ia * 6 + threadIdx.x] = red[threadIdx.x][0];
}

int common_checks(const char* who, int na, const float* atoms, const float* cMs, const float* points, int n_scan,
                  const spm_scan_params* p) {
    SPM_REQUIRE(p != nullptr && atoms && cMs, "%s: null pointer", who);
    SPM_REQUIRE(points || n_scan == 0, "%s: null points", who);
    if (na < 1 || na > SPM_DIRECT_MAX_ATOMS)
        return set_error(SPM_ERR_UNSUPPORTED, "%s: n_atoms=%d out of range [1,%d]", who, na, SPM_DIRECT_MAX_ATOMS);
    SPM_REQUIRE(n_scan >= 0 && p->nz >= 0, "%s: n_scan=%d nz=%d must be >= 0", who, n_scan, p->nz);
    SPM_REQUIRE(aligned16(atoms) && aligned16(cMs) && aligned16(points), "%s: buffers not 16-byte aligned", who);
    long long t = 0;
    SPM_REQUIRE(mul_ok(n_scan, (long long)p->nz * 4, &t), "%s: state count overflows", who);
    return SPM_OK;
}

Sites make_sites(const float* Qs, const float* QZs, bool compact, int* ns) {
    Sites S = {};
    int n = 0;
    for (int k = 0; k < 4; k++) {
        if (compact) {
            if (Qs[k] != 0.f) {
                S.qs[n] = Qs[k] * COULOMB_CONST; S.qz[n] = QZs[k];
                S.qs64[n] = (double)Qs[k] * 14.3996448915; S.qz64[n] = QZs[k];
                n++;
            }
        } else {
            S.qs[k] = Qs[k] * COULOMB_CONST;
            S.qz[k] = QZs[k];
            S.qs64[k] = (double)Qs[k] * 14.3996448915;
            S.qz64[k] = QZs[k];
        }
    }
    S.ns = compact ? n : 4;
    if (ns) *ns = S.ns;
    return S;
}

// Lanes per pixel: about four atoms per lane, at least 4 and at most 32 lanes, more while the scan
// leaves the GPU short of warps (fewer than ~8 warps per SM of a 148-SM part).
int direct_lpp(int na, int n_scan) {
    int lpp = 4;
    while (lpp < 32 && lpp * 4 < na) lpp *= 2;
    while (lpp < 32 && (long long)n_scan * lpp < 148LL * 8 * 32) lpp *= 2;
    return lpp;
}

template <int NS>
int launch_direct(int na, const float* atoms, const float* cMs, const float* points, int n_scan,
                  const spm_scan_params& P, const Sites& S, float* FEs, float* PPs, cudaStream_t st) {
    const size_t smem = (size_t)na * (2 * sizeof(float4) + NS * sizeof(float));
    const int lpp = direct_lpp(na, n_scan);
    auto kern = lpp == 4 ? relax_direct_kernel<NS, 4> : lpp == 8 ? relax_direct_kernel<NS, 8>
              : lpp == 16 ? relax_direct_kernel<NS, 16> : relax_direct_kernel<NS, 32>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return set_error(SPM_ERR_CUDA, "spm_relax_direct_morse: smem %zu B: %s", smem,
                                               cudaGetErrorString(e));
    }
    const int per_cta = DX_THREADS / lpp;
    const int blocks = (n_scan + per_cta - 1) / per_cta;
    kern<<<blocks, DX_THREADS, smem, st>>>(na, reinterpret_cast<const float4*>(atoms),
                                           reinterpret_cast<const float4*>(cMs),
                                           reinterpret_cast<const float4*>(points), n_scan, P, S,
                                           reinterpret_cast<float4*>(FEs), reinterpret_cast<float4*>(PPs));
    return check_launch("spm_relax_direct_morse");
}

}  // namespace
}  // namespace spm

extern "C" int spm_relax_direct_morse(int n_atoms, const float* atoms, const float* cMs, const float* points,
                                      int n_scan, const spm_scan_params* p, const float* Qs, const float* QZs,
                                      float* FEs, float* PPs, void* stream) {
    using namespace spm;
    clear_error();
    int rc = common_checks("spm_relax_direct_morse", n_atoms, atoms, cMs, points, n_scan, p);
    if (rc) return rc;
    SPM_REQUIRE(Qs && QZs && FEs && PPs, "spm_relax_direct_morse: null Qs/QZs/FEs/PPs");
    SPM_REQUIRE(aligned16(FEs) && aligned16(PPs), "spm_relax_direct_morse: outputs not 16-byte aligned");
    if (n_scan == 0 || p->nz == 0) return SPM_OK;
    spm_scan_params P = *p;
    if (P.raster_ny > 0 && n_scan % P.raster_ny != 0) P.raster_ny = 0;
    int ns = 0;
    Sites S = make_sites(Qs, QZs, true, &ns);
    cudaStream_t st = as_stream(stream);
    switch (ns) {
        case 0: return launch_direct<0>(n_atoms, atoms, cMs, points, n_scan, P, S, FEs, PPs, st);
        case 1: return launch_direct<1>(n_atoms, atoms, cMs, points, n_scan, P, S, FEs, PPs, st);
        case 2: return launch_direct<2>(n_atoms, atoms, cMs, points, n_scan, P, S, FEs, PPs, st);
        case 3: return launch_direct<3>(n_atoms, atoms, cMs, points, n_scan, P, S, FEs, PPs, st);
        default: return launch_direct<4>(n_atoms, atoms, cMs, points, n_scan, P, S, FEs, PPs, st);
    }
}

extern "C" int spm_adjoint_direct_state(int n_atoms, const float* atoms, const float* cMs, const float* points,
                                        int n_scan, const spm_scan_params* p, const float* Qs, const float* QZs,
                                        const float* PPs, const float* dL_dFEs, float* lambdas, float* diag,
                                        void* stream) {
    using namespace spm;
    clear_error();
    int rc = common_checks("spm_adjoint_direct_state", n_atoms, atoms, cMs, points, n_scan, p);
    if (rc) return rc;
    SPM_REQUIRE(Qs && QZs && PPs && dL_dFEs && lambdas && diag, "spm_adjoint_direct_state: null pointer");
    SPM_REQUIRE(aligned16(PPs) && aligned16(dL_dFEs) && aligned16(lambdas) && aligned16(diag),
                "spm_adjoint_direct_state: buffers not 16-byte aligned");
    const long long n_state = (long long)n_scan * p->nz;
    if (n_state == 0) return SPM_OK;
    Sites S = make_sites(Qs, QZs, false, nullptr);
    const size_t smem = (size_t)n_atoms * 2 * sizeof(float4);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(adjoint_state_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return set_error(SPM_ERR_CUDA, "spm_adjoint_direct_state: %s", cudaGetErrorString(e));
    }
    adjoint_state_kernel<<<(unsigned)((n_state + DX_THREADS - 1) / DX_THREADS), DX_THREADS, smem, as_stream(stream)>>>(
        n_atoms, reinterpret_cast<const float4*>(atoms), reinterpret_cast<const float4*>(cMs),
        reinterpret_cast<const float4*>(points), n_scan, *p, S, reinterpret_cast<const float4*>(PPs),
        reinterpret_cast<const float4*>(dL_dFEs), reinterpret_cast<float4*>(lambdas), reinterpret_cast<float4*>(diag));
    return check_launch("spm_adjoint_direct_state");
}

extern "C" long long spm_adjoint_direct_scratch_bytes(int n_atoms, int n_scan) {
    if (n_atoms <= 0 || n_scan < 0) return 0;
    const long long chunks = ((long long)n_scan + spm::PART_THREADS - 1) / spm::PART_THREADS;
    return (long long)n_atoms * (chunks > 0 ? chunks : 1) * 6 * (long long)sizeof(float);
}

extern "C" int spm_adjoint_direct_params(int n_atoms, const float* atoms, const float* cMs, const float* points,
                                         int n_scan, const spm_scan_params* p, const float* Qs, const float* QZs,
                                         const float* PPs, const float* dL_dFEs, const float* lambdas, float* grad,
                                         void* scratch, void* stream) {
    using namespace spm;
    clear_error();
    int rc = common_checks("spm_adjoint_direct_params", n_atoms, atoms, cMs, points, n_scan, p);
    if (rc) return rc;
    SPM_REQUIRE(Qs && QZs && PPs && dL_dFEs && lambdas && grad && scratch, "spm_adjoint_direct_params: null pointer");
    SPM_REQUIRE(aligned16(PPs) && aligned16(dL_dFEs) && aligned16(lambdas),
                "spm_adjoint_direct_params: buffers not 16-byte aligned");
    SPM_REQUIRE(n_atoms <= 65535, "spm_adjoint_direct_params: n_atoms=%d exceeds the launch limit", n_atoms);
    Sites S = make_sites(Qs, QZs, false, nullptr);
    const int chunks = n_scan > 0 ? (n_scan + PART_THREADS - 1) / PART_THREADS : 1;
    float* part = static_cast<float*>(scratch);
    cudaStream_t st = as_stream(stream);
    adjoint_partials_kernel<<<dim3(chunks, n_atoms), PART_THREADS, 0, st>>>(
        n_atoms, reinterpret_cast<const float4*>(atoms), reinterpret_cast<const float4*>(cMs),
        reinterpret_cast<const float4*>(points), n_scan, *p, S, reinterpret_cast<const float4*>(PPs),
        reinterpret_cast<const float4*>(dL_dFEs), reinterpret_cast<const float4*>(lambdas), part);
    adjoint_reduce_kernel<<<n_atoms, 256, 0, st>>>(part, chunks, grad);
    return check_launch("spm_adjoint_direct_params");
}
