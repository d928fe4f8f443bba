/*
 * spm_oracle.c -- TEST INFRASTRUCTURE ONLY: the CPU oracle for the
 * probe-particle AFM hot path.  It is the checker, never the thing measured or
 * shipped: the product library (spammm_b200/libspmb200.so) does not link it,
 * and only tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke()
 * load it.
 *
 * It restates SPAMMM's OpenCL kernels (kernels/AFM.cl, kernels/common.cl) on
 * the CPU in two precisions (see ora_core.h for the per-function citations):
 *   *_f : canonical FP32 op order, bit-identical to the CUDA relaxation paths
 *   *_d : FP64 (the FP64 oracle)
 * OpenMP parallelises over grid nodes / scan pixels; results do not depend on
 * the thread count (every node and pixel is computed independently).
 *
 * Build: oracle/Makefile (gcc -O3 -mavx2 -mfma -ffp-contract=off -fopenmp).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define COULOMB_CONST 14.3996448915

/* ---- FP32 instantiation ---- */
#define REAL float
#define GRID_T float
#define SFX(n) n##_f
#define FMA fmaf
#define SQRT sqrtf
#define FLOOR floorf
#define FMAX fmaxf
#define FMIN fminf
#define EXP expf
#define FABS fabsf
#include "ora_core.h"
#undef REAL
#undef GRID_T
#undef SFX
#undef FMA
#undef SQRT
#undef FLOOR
#undef FMAX
#undef FMIN
#undef EXP
#undef FABS

/* ---- FP64 instantiation ---- */
#define REAL double
#define GRID_T double
#define SFX(n) n##_d
#define FMA fma
#define SQRT sqrt
#define FLOOR floor
#define FMAX fmax
#define FMIN fmin
#define EXP exp
#define FABS fabs
#include "ora_core.h"

static void cvt4_f(const float* s, float* d) { d[0] = s[0]; d[1] = s[1]; d[2] = s[2]; d[3] = s[3]; }
static void cvt4_d(const float* s, double* d) { d[0] = s[0]; d[1] = s[1]; d[2] = s[2]; d[3] = s[3]; }

int ora_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void ora_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------ */
/* Stage (a): force-grid build  (evalLJC_QZs_toImg / evalMorseC_QZs_toImg)   */
/*   kind 0 = LJ   prm (na,2) = (c6,c12)                                      */
/*   kind 1 = Morse prm (na,4) = (R0,E0,K,0)                                  */
/* Output layout (nz,ny,nx,4) x fastest, exactly the OpenCL image layout.     */
/* Nodes with |E|>100 are rescaled by 100/|E| (AFM.cl:984-985, :1053-1054).   */
/* node0/nnodes select a contiguous slice of the flattened node index (used    */
/* to time a bounded sample); pass node0=0,nnodes=nx*ny*nz for the full grid. */
/* ------------------------------------------------------------------------ */
#define GRID_BUILD_BODY(REALT, SF, OUT_T)                                                        \
    REALT* at = (REALT*)malloc(sizeof(REALT) * 4 * (size_t)(na > 0 ? na : 1));                    \
    REALT* pr = (REALT*)malloc(sizeof(REALT) * 4 * (size_t)(na > 0 ? na : 1));                    \
    for (int j = 0; j < na; j++) {                                                                \
        for (int c = 0; c < 4; c++) at[4 * j + c] = (REALT)atoms[4 * j + c];                     \
        for (int c = 0; c < 4; c++) pr[4 * j + c] = c < pstride ? (REALT)prm[pstride * j + c] : 0; \
    }                                                                                             \
    REALT qs[4], qz[4];                                                                           \
    for (int s = 0; s < 4; s++) { qs[s] = (REALT)Qs[s] * (REALT)COULOMB_CONST; qz[s] = (REALT)QZs[s]; } \
    long long nab = (long long)nx * ny;                                                           \
    long long total = nab * nz;                                                                   \
    long long n1 = node0 + nnodes; if (n1 > total) n1 = total;                                    \
    _Pragma("omp parallel for schedule(dynamic, 256)")                                            \
    for (long long iG = node0; iG < n1; iG++) {                                                   \
        int ia = (int)(iG % nx), ib = (int)((iG % nab) / nx), ic = (int)(iG / nab);               \
        SF##v3 pos;                                                                               \
        pos.x = (REALT)p0[0] + (REALT)dA[0] * ia + (REALT)dB[0] * ib + (REALT)dC[0] * ic;          \
        pos.y = (REALT)p0[1] + (REALT)dA[1] * ia + (REALT)dB[1] * ib + (REALT)dC[1] * ic;          \
        pos.z = (REALT)p0[2] + (REALT)dA[2] * ia + (REALT)dB[2] * ib + (REALT)dC[2] * ic;          \
        REALT fe[4];                                                                              \
        SF##pair_fe(kind, na, at, pr, 4, pos, qs, qz, fe);                                        \
        REALT renorm = (REALT)100 / (REALT)fabs((double)fe[3]);                                   \
        if (renorm < (REALT)1) { fe[0] *= renorm; fe[1] *= renorm; fe[2] *= renorm; fe[3] *= renorm; } \
        OUT_T* o = out + (size_t)(iG - node0) * 4;                                                \
        o[0] = (OUT_T)fe[0]; o[1] = (OUT_T)fe[1]; o[2] = (OUT_T)fe[2]; o[3] = (OUT_T)fe[3];       \
    }                                                                                             \
    free(at); free(pr);

/* pair_fe with the _f / _d suffix expects the v3 type name prefix */
typedef v3_f f_v3;
typedef v3_d d_v3;
#define f_pair_fe pair_fe_f
#define d_pair_fe pair_fe_d

void ora_grid_build_d(int kind, int na, const float* atoms, const float* prm, int pstride,
                      int nx, int ny, int nz, const float* p0, const float* dA, const float* dB,
                      const float* dC, const float* Qs, const float* QZs,
                      long long node0, long long nnodes, double* out) {
    GRID_BUILD_BODY(double, d_, double)
}

/* FP64 grid build from FP64 inputs (finite-difference checks perturb atoms by
 * less than float32 resolves). */
void ora_grid_build_d64(int kind, int na, const double* atoms, const double* prm, int pstride,
                        int nx, int ny, int nz, const double* p0, const double* dA, const double* dB,
                        const double* dC, const double* Qs, const double* QZs,
                        long long node0, long long nnodes, double* out) {
    GRID_BUILD_BODY(double, d_, double)
}

void ora_grid_build_f(int kind, int na, const float* atoms, const float* prm, int pstride,
                      int nx, int ny, int nz, const float* p0, const float* dA, const float* dB,
                      const float* dC, const float* Qs, const float* QZs,
                      long long node0, long long nnodes, float* out) {
    GRID_BUILD_BODY(float, f_, float)
}

/* Direct pair FE at arbitrary query points (FP64), uncapped                  */
/* (cs_brute_afm_morse_c_points semantics, contact_surface.cl:1341-1390).     */
void ora_pair_fe_d(int kind, int na, const double* atoms, const double* prm, int pstride,
                   const double* q, int nq, const double* Qs, const double* QZs, double* out) {
    double qs[4], pr4[4];
    (void)pr4;
    for (int s = 0; s < 4; s++) qs[s] = Qs[s] * COULOMB_CONST;
    double* pr = (double*)malloc(sizeof(double) * 4 * (size_t)(na > 0 ? na : 1));
    for (int j = 0; j < na; j++)
        for (int c = 0; c < 4; c++) pr[4 * j + c] = c < pstride ? prm[pstride * j + c] : 0;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nq; i++) {
        v3_d p = mk3_d(q[3 * i], q[3 * i + 1], q[3 * i + 2]);
        pair_fe_d(kind, na, atoms, pr, 4, p, qs, QZs, out + 4 * (size_t)i);
    }
    free(pr);
}

/* Sum over atoms (and tip-charge sites) of the ABSOLUTE value of each atom's
 * contribution, per channel, at arbitrary query points, FP64: the scale of the
 * cancellation in a grid value.  A floating-point sum of the contributions
 * has an error proportional to this sum, not to |sum|; the grid-build tests
 * state their FP32 tolerance against it. */
void ora_pair_fe_abs_d(int kind, int na, const double* atoms, const double* prm, int pstride,
                       const double* q, int nq, const double* Qs, const double* QZs, double* out) {
    double qs[4];
    for (int s = 0; s < 4; s++) qs[s] = Qs[s] * COULOMB_CONST;
    double* pr = (double*)malloc(sizeof(double) * 4 * (size_t)(na > 0 ? na : 1));
    for (int j = 0; j < na; j++)
        for (int c = 0; c < 4; c++) pr[4 * j + c] = c < pstride ? prm[pstride * j + c] : 0;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nq; i++) {
        v3_d p = mk3_d(q[3 * i], q[3 * i + 1], q[3 * i + 2]);
        double acc[4] = {0, 0, 0, 0};
        for (int j = 0; j < na; j++) {
            const double* at = atoms + 4 * j;
            double fe[4] = {0, 0, 0, 0};
            if (kind == 0) acc_lj_d(fe, at, pr[4 * j], pr[4 * j + 1], p);
            else acc_morse_d(fe, mk3_d(p.x - at[0], p.y - at[1], p.z - at[2]), pr[4 * j], pr[4 * j + 1], pr[4 * j + 2]);
            for (int c = 0; c < 4; c++) acc[c] += fabs(fe[c]);
            for (int s = 0; s < 4; s++) {
                if (qs[s] == 0) continue;
                double fc[4] = {0, 0, 0, 0};
                acc_coulomb_d(fc, at, mk3_d(p.x, p.y, p.z + QZs[s]), qs[s]);
                for (int c = 0; c < 4; c++) acc[c] += fabs(fc[c]);
            }
        }
        for (int c = 0; c < 4; c++) out[4 * (size_t)i + c] = acc[c];
    }
    free(pr);
}

/* ------------------------------------------------------------------------ */
/* Stage (b): relaxation over strokes                                         */
/* ------------------------------------------------------------------------ */
void ora_relax_strokes_f(const float* grid, int nx, int ny, int nz, const float* dinvA,
                         const float* dinvB, const float* dinvC, const float* pts, int nscan, int nzs,
                         const float* dTip, const float* k, const float* d0, const float* relax,
                         int max_iter, float f2conv, int use_fire, int flip, int polish, float* FEs,
                         float* disps) {
    gridref_f G; G.nx = nx; G.ny = ny; G.nz = nz;
    cvt4_f(dinvA, G.dA); cvt4_f(dinvB, G.dB); cvt4_f(dinvC, G.dC);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < nscan; i++)
        relax_strokes_pixel_f(grid, &G, pts + 4 * (size_t)i, nzs, dTip, k, d0, relax, max_iter, f2conv,
                              use_fire, flip, polish, FEs + (size_t)i * nzs * 4, disps + (size_t)i * nzs * 4);
}

void ora_relax_strokes_d(const double* grid, int nx, int ny, int nz, const float* dinvA,
                         const float* dinvB, const float* dinvC, const float* pts, int nscan, int nzs,
                         const float* dTip, const float* k, const float* d0, const float* relax,
                         int max_iter, double f2conv, int use_fire, int flip, int polish, double* FEs,
                         double* disps) {
    gridref_d G; G.nx = nx; G.ny = ny; G.nz = nz;
    cvt4_d(dinvA, G.dA); cvt4_d(dinvB, G.dB); cvt4_d(dinvC, G.dC);
    double t[4], kk[4], dd[4], rr[4];
    cvt4_d(dTip, t); cvt4_d(k, kk); cvt4_d(d0, dd); cvt4_d(relax, rr);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < nscan; i++)
        relax_strokes_pixel_d(grid, &G, pts + 4 * (size_t)i, nzs, t, kk, dd, rr, max_iter, f2conv,
                              use_fire, flip, polish, FEs + (size_t)i * nzs * 4, disps + (size_t)i * nzs * 4);
}

void ora_relax_2d_f(const float* grid, int nx, int ny, int nz, const float* dinvA, const float* dinvB,
                    const float* dinvC, const float* pts, int nscan, int nzs, float K, float dh, float dt, float damp,
                    int max_iter, float f2conv, int flip, float* FEs, float* disps) {
    gridref_f G; G.nx = nx; G.ny = ny; G.nz = nz;
    cvt4_f(dinvA, G.dA); cvt4_f(dinvB, G.dB); cvt4_f(dinvC, G.dC);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < nscan; i++)
        relax_2d_pixel_f(grid, &G, pts + 4 * (size_t)i, nzs, K, dh, dt, damp, max_iter, f2conv, flip,
                         FEs + (size_t)i * nzs * 4, disps + (size_t)i * nzs * 4);
}

void ora_relax_tilted_f(const float* grid, int nx, int ny, int nz, const float* dinvA,
                        const float* dinvB, const float* dinvC, const float* pts, int nscan, int nzs,
                        const float* tA, const float* tB, const float* tC, const float* k, const float* d0,
                        const float* relax, const float* surf, int max_iter, float f2conv, int use_fire,
                        int polish, float* FEs) {
    gridref_f G; G.nx = nx; G.ny = ny; G.nz = nz;
    cvt4_f(dinvA, G.dA); cvt4_f(dinvB, G.dB); cvt4_f(dinvC, G.dC);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < nscan; i++)
        relax_tilted_pixel_f(grid, &G, pts + 4 * (size_t)i, nzs, tA, tB, tC, k, d0, relax, surf, max_iter,
                             f2conv, use_fire, polish, FEs + (size_t)i * nzs * 4);
}

void ora_relax_tilted_d(const double* grid, int nx, int ny, int nz, const float* dinvA,
                        const float* dinvB, const float* dinvC, const float* pts, int nscan, int nzs,
                        const float* tA, const float* tB, const float* tC, const float* k, const float* d0,
                        const float* relax, const float* surf, int max_iter, double f2conv, int use_fire,
                        int polish, double* FEs) {
    gridref_d G; G.nx = nx; G.ny = ny; G.nz = nz;
    cvt4_d(dinvA, G.dA); cvt4_d(dinvB, G.dB); cvt4_d(dinvC, G.dC);
    double a[4], b[4], c[4], kk[4], dd[4], rr[4], ss[4];
    cvt4_d(tA, a); cvt4_d(tB, b); cvt4_d(tC, c); cvt4_d(k, kk); cvt4_d(d0, dd); cvt4_d(relax, rr); cvt4_d(surf, ss);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < nscan; i++)
        relax_tilted_pixel_d(grid, &G, pts + 4 * (size_t)i, nzs, a, b, c, kk, dd, rr, ss, max_iter, f2conv,
                             use_fire, polish, FEs + (size_t)i * nzs * 4);
}

void ora_raw_tilted_f(const float* grid, int nx, int ny, int nz, const float* dinvA, const float* dinvB,
                      const float* dinvC, const float* pts, int nscan, int nzs, const float* tA,
                      const float* tB, const float* tC, const float* dTip, const float* d0, float* FEs) {
    gridref_f G; G.nx = nx; G.ny = ny; G.nz = nz;
    cvt4_f(dinvA, G.dA); cvt4_f(dinvB, G.dB); cvt4_f(dinvC, G.dC);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nscan; i++)
        raw_tilted_pixel_f(grid, &G, pts + 4 * (size_t)i, nzs, tA, tB, tC, dTip, d0, FEs + (size_t)i * nzs * 4);
}

void ora_raw_tilted_d(const double* grid, int nx, int ny, int nz, const float* dinvA, const float* dinvB,
                      const float* dinvC, const float* pts, int nscan, int nzs, const float* tA,
                      const float* tB, const float* tC, const float* dTip, const float* d0, double* FEs) {
    gridref_d G; G.nx = nx; G.ny = ny; G.nz = nz;
    cvt4_d(dinvA, G.dA); cvt4_d(dinvB, G.dB); cvt4_d(dinvC, G.dC);
    double a[4], b[4], c[4], t[4], dd[4];
    cvt4_d(tA, a); cvt4_d(tB, b); cvt4_d(tC, c); cvt4_d(dTip, t); cvt4_d(d0, dd);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nscan; i++)
        raw_tilted_pixel_d(grid, &G, pts + 4 * (size_t)i, nzs, a, b, c, t, dd, FEs + (size_t)i * nzs * 4);
}

/* Direct (grid-free) Morse+Coulomb relaxation, FP64.  atoms/cMs in FP64. */
void ora_relax_direct_d(int na, const double* atoms, const double* cMs, const float* pts, int nscan, int nzs,
                        const float* tA, const float* tB, const float* tC, const float* k, const float* d0,
                        const float* relax, const float* surf, const float* Qs, const float* QZs, int max_iter,
                        double f2conv, int quirks, double* FEs, double* PPs) {
    double a[4], b[4], c[4], kk[4], dd[4], rr[4], ss[4], qs[4], qz[4];
    cvt4_d(tA, a); cvt4_d(tB, b); cvt4_d(tC, c); cvt4_d(k, kk); cvt4_d(d0, dd); cvt4_d(relax, rr);
    cvt4_d(surf, ss); cvt4_d(QZs, qz);
    for (int s = 0; s < 4; s++) qs[s] = (double)Qs[s] * COULOMB_CONST;
    if (quirks & 2) {  /* integrator state threads through the pixels: serial */
        double carry[2] = {rr[0], rr[1]};
        for (int i = 0; i < nscan; i++)
            relax_direct_pixel_d(na, atoms, cMs, pts + 4 * (size_t)i, nzs, a, b, c, kk, dd, rr, ss, qs, qz,
                                 max_iter, f2conv, FEs + (size_t)i * nzs * 4, PPs + (size_t)i * nzs * 4, quirks,
                                 carry);
        return;
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < nscan; i++)
        relax_direct_pixel_d(na, atoms, cMs, pts + 4 * (size_t)i, nzs, a, b, c, kk, dd, rr, ss, qs, qz,
                             max_iter, f2conv, FEs + (size_t)i * nzs * 4, PPs + (size_t)i * nzs * 4, quirks, NULL);
}

/* Grid relaxation with converged-position telemetry (see relax_pp_pixel). */
void ora_relax_pp_f(const float* grid, int nx, int ny, int nz, const float* dinvA, const float* dinvB,
                    const float* dinvC, const float* pts, int nscan, int nzs, const float* tA, const float* tB,
                    const float* tC, const float* k, const float* d0, const float* relax, const float* surf,
                    int max_iter, float f2conv, int use_fire, int polish, float* FEs, float* PPs) {
    gridref_f G; G.nx = nx; G.ny = ny; G.nz = nz;
    cvt4_f(dinvA, G.dA); cvt4_f(dinvB, G.dB); cvt4_f(dinvC, G.dC);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < nscan; i++)
        relax_pp_pixel_f(grid, &G, pts + 4 * (size_t)i, nzs, tA, tB, tC, k, d0, relax, surf, max_iter, f2conv,
                         use_fire, polish, FEs + (size_t)i * nzs * 4, PPs + (size_t)i * nzs * 4);
}

/* FP64 variant: every parameter vector is double (used by finite-difference
 * checks, whose perturbations are below float32 resolution). */
void ora_relax_pp_d(const double* grid, int nx, int ny, int nz, const double* dinvA, const double* dinvB,
                    const double* dinvC, const float* pts, int nscan, int nzs, const double* tA, const double* tB,
                    const double* tC, const double* k, const double* d0, const double* relax, const double* surf,
                    int max_iter, double f2conv, int use_fire, int polish, double* FEs, double* PPs) {
    gridref_d G; G.nx = nx; G.ny = ny; G.nz = nz;
    for (int c = 0; c < 4; c++) { G.dA[c] = dinvA[c]; G.dB[c] = dinvB[c]; G.dC[c] = dinvC[c]; }
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < nscan; i++)
        relax_pp_pixel_d(grid, &G, pts + 4 * (size_t)i, nzs, tA, tB, tC, k, d0, relax, surf, max_iter, f2conv, use_fire,
                         polish, FEs + (size_t)i * nzs * 4, PPs + (size_t)i * nzs * 4);
}

/* convolveZ (kernels/AFM.cl:666-701): per z-column c,
 * Fout[c,izo] = sum over jz < nzin-nzout of Fin[c,izo+jz] * w[jz] on all four
 * channels, accumulated in jz order from zero (fe += Fin*w, the fused
 * multiply-add the OpenCL compiler contracts it to). */
void ora_convolve_z_f(const float* Fin, int ncol, int nzin, int nzout, const float* w, float* Fout) {
    const int nzw = nzin - nzout;
#pragma omp parallel for schedule(static)
    for (int c = 0; c < ncol; c++)
        for (int izo = 0; izo < nzout; izo++) {
            float fe[4] = {0.f, 0.f, 0.f, 0.f};
            for (int jz = 0; jz < nzw; jz++) {
                const float* a = Fin + ((size_t)c * nzin + izo + jz) * 4;
                for (int k = 0; k < 4; k++) fe[k] = fmaf(a[k], w[jz], fe[k]);
            }
            memcpy(Fout + ((size_t)c * nzout + izo) * 4, fe, sizeof fe);
        }
}

/* izoZ (kernels/AFM.cl:705-723): per column the first iz >= 1 whose Fz
 * exceeds iso gives iz + (iso - Fz[iz-1]) / (Fz[iz] - Fz[iz-1]); else -1. */
void ora_izo_z_f(const float* Fin, int ncol, int nz, float iso, float* zMap) {
#pragma omp parallel for schedule(static)
    for (int c = 0; c < ncol; c++) {
        const float* f = Fin + (size_t)c * nz * 4;
        float oz = f[2], res = -1.f;
        for (int iz = 1; iz < nz; iz++) {
            const float fz = f[(size_t)iz * 4 + 2];
            if (fz > iso) {
                const float t = (iso - oz) / (fz - oz);
                res = (float)iz + t;
                break;
            }
            oz = fz;
        }
        zMap[c] = res;
    }
}
