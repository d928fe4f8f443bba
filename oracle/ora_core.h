/*
 * ora_core.h -- TEST INFRASTRUCTURE ONLY (the oracle). Never linked into the
 * product library; only tests/, bench.py's CPU-baseline leg and
 * __graft_entry__.smoke() load the oracle, and only as the checker.
 *
 * CPU restatement of the probe-particle AFM kernels of SPAMMM
 * (kernels/AFM.cl, kernels/common.cl), written once and instantiated twice by
 * spm_oracle.c:
 *   REAL=float  (suffix _f): the canonical FP32 operation order.  Every
 *               product/sum that the CUDA kernels fuse is an explicit FMA here
 *               and the file is compiled with -ffp-contract=off, so the FP32
 *               relaxation paths are bit-identical to the sm_100a kernels
 *               (which are compiled with -fmad=false and the same explicit
 *               fmaf calls).
 *   REAL=double (suffix _d): the same algorithm in FP64 (the FP64 oracle).
 *
 * Reference semantics followed (file:line in the SPAMMM tree):
 *   tipForce            kernels/AFM.cl:53-58
 *   interpFE            kernels/AFM.cl:100-105 (+ OpenCL REPEAT/LINEAR sampler,
 *                       kernels/AFM.cl:49, normalized coordinates)
 *   update_FIRE         kernels/AFM.cl:136-157 (FTDEC/FTINC/FDAMP/F2SAFE :124-132)
 *   relaxStrokes        kernels/AFM.cl:345-394
 *   relaxStrokesTilted  kernels/AFM.cl:478-562
 *   relaxStrokes2D      kernels/AFM.cl:410-450
 *   getFEinStrokesTilted kernels/AFM.cl:210-233
 *   rotMat / rotMatT    kernels/common.cl:43-44
 *   getCoulombAFM/getLJ/getMorse kernels/AFM.cl:730-757
 *   evalLJC_QZs_toImg   kernels/AFM.cl:916-991, evalMorseC_QZs_toImg :996-1056
 *   relaxStrokesTiltedMorseDirect kernels/AFM.cl:1419-1511
 *
 * Required macros: REAL, SFX(name), FMA, SQRT, FLOOR, FMAX, FMIN, EXP, FABS.
 */

typedef struct { REAL x, y, z; } SFX(v3);

static inline SFX(v3) SFX(mk3)(REAL x, REAL y, REAL z) { SFX(v3) r; r.x = x; r.y = y; r.z = z; return r; }
static inline SFX(v3) SFX(sub3)(SFX(v3) a, SFX(v3) b) { return SFX(mk3)(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline SFX(v3) SFX(add3)(SFX(v3) a, SFX(v3) b) { return SFX(mk3)(a.x + b.x, a.y + b.y, a.z + b.z); }
/* dot(a,b) in the canonical order x*x, then fma y, then fma z */
static inline REAL SFX(dot3)(SFX(v3) a, SFX(v3) b) { return FMA(a.z, b.z, FMA(a.y, b.y, a.x * b.x)); }
/* rotMat(v,a,b,c) = (dot(v,a), dot(v,b), dot(v,c))      common.cl:43 */
static inline SFX(v3) SFX(rotmat)(SFX(v3) v, SFX(v3) a, SFX(v3) b, SFX(v3) c) {
    return SFX(mk3)(SFX(dot3)(v, a), SFX(dot3)(v, b), SFX(dot3)(v, c));
}
/* rotMatT(v,a,b,c) = a*v.x + b*v.y + c*v.z              common.cl:44 */
static inline SFX(v3) SFX(rotmatT)(SFX(v3) v, SFX(v3) a, SFX(v3) b, SFX(v3) c) {
    return SFX(mk3)(FMA(c.x, v.z, FMA(b.x, v.y, a.x * v.x)),
                    FMA(c.y, v.z, FMA(b.y, v.y, a.y * v.x)),
                    FMA(c.z, v.z, FMA(b.z, v.y, a.z * v.x)));
}

/* tipForce                                               AFM.cl:53-58
 * (dpos-dpos0.xyz)*k.xyz + dpos*(k.w*(r-dpos0.w)/r), r = max(|dpos|,1e-10) */
static inline SFX(v3) SFX(tip_force)(SFX(v3) d, const REAL* k, const REAL* d0) {
    /* k.w == 0: the radial term is exactly +-0 and is skipped (the CUDA kernels
     * skip it too; only the sign of an all-zero component can differ). */
    if (k[3] == (REAL)0)
        return SFX(mk3)((d.x - d0[0]) * k[0], (d.y - d0[1]) * k[1], (d.z - d0[2]) * k[2]);
    REAL r = SQRT(SFX(dot3)(d, d));
    r = FMAX(r, (REAL)1e-10);
    REAL s = (k[3] * (r - d0[3])) / r;
    return SFX(mk3)(FMA(d.x, s, (d.x - d0[0]) * k[0]),
                    FMA(d.y, s, (d.y - d0[1]) * k[1]),
                    FMA(d.z, s, (d.z - d0[2]) * k[2]));
}

/* update_FIRE (Bitzek et al. 2006)                       AFM.cl:136-157 */
static inline void SFX(fire_update)(SFX(v3) f, SFX(v3)* v, REAL* dt, REAL* damp,
                                    REAL dtmin, REAL dtmax, REAL damp0) {
    REAL ff = SFX(dot3)(f, f);
    REAL vv = SFX(dot3)(*v, *v);
    REAL vf = SFX(dot3)(*v, f);
    if (vf < (REAL)0) {
        v->x = v->x * (REAL)0; v->y = v->y * (REAL)0; v->z = v->z * (REAL)0;
        *dt = FMAX(dtmin, (*dt) * (REAL)0.5);
        *damp = damp0;
    } else {
        REAL cf = (*damp) * SQRT(vv / (ff + (REAL)1e-8));
        REAL cv = (REAL)1 - (*damp);
        v->x = FMA(f.x, cf, v->x * cv);
        v->y = FMA(f.y, cf, v->y * cv);
        v->z = FMA(f.z, cf, v->z * cv);
        *dt = FMIN(dtmax, (*dt) * (REAL)1.1);
        *damp = (*damp) * (REAL)0.99;
    }
}

/* One integrator step after the force f is known: FIRE (use_fire) or plain
 * damping (OPT_FIRE=0 branch, AFM.cl:383-386), then v += f*dt, pos += v*dt. */
static inline void SFX(md_step)(SFX(v3) f, SFX(v3)* v, SFX(v3)* pos, REAL* dt, REAL* damp,
                                REAL dtmin, REAL dtmax, REAL damp0, int use_fire) {
    if (use_fire) {
        SFX(fire_update)(f, v, dt, damp, dtmin, dtmax, damp0);
    } else {
        REAL cv = (REAL)1 - (*damp);
        v->x = v->x * cv; v->y = v->y * cv; v->z = v->z * cv;
    }
    v->x = FMA(f.x, *dt, v->x);
    v->y = FMA(f.y, *dt, v->y);
    v->z = FMA(f.z, *dt, v->z);
    pos->x = FMA(v->x, *dt, pos->x);
    pos->y = FMA(v->y, *dt, pos->y);
    pos->z = FMA(v->z, *dt, pos->z);
}

/* OpenCL normalized-coordinate REPEAT + LINEAR addressing (OpenCL 1.2 spec
 * sec. 8.2): s = frac(u); t = s*n - 0.5; i0 = floor(t) wrapped; a = t - floor(t).
 * Exact FP32 weights (the hardware filter's 8-bit weight quantisation is not
 * reproduced).  Returns 0 for non-finite coordinates. */
static inline int SFX(tex_axis)(REAL u, int n, int* i0, int* i1, REAL* a) {
    REAL s = u - FLOOR(u);
    REAL t = FMA(s, (REAL)n, (REAL)-0.5);
    if (!(t >= (REAL)-1 && t < (REAL)n)) return 0;
    REAL fi = FLOOR(t);
    *a = t - fi;
    int i = (int)fi;
    if (i < 0) i += n;
    int j = i + 1;
    if (j >= n) j -= n;
    *i0 = i; *i1 = j;
    return 1;
}

/* interpFE: trilinear sample of the (nz,ny,nx,4) force grid    AFM.cl:100-105 */
static inline void SFX(interp_fe)(const GRID_T* g, int nx, int ny, int nz,
                                  const REAL* dA, const REAL* dB, const REAL* dC,
                                  SFX(v3) p, REAL* out) {
    REAL u = FMA(p.x, dA[0], FMA(p.y, dA[1], FMA(p.z, dA[2], dA[3])));
    REAL v = FMA(p.x, dB[0], FMA(p.y, dB[1], FMA(p.z, dB[2], dB[3])));
    REAL w = FMA(p.x, dC[0], FMA(p.y, dC[1], FMA(p.z, dC[2], dC[3])));
    int x0, x1, y0, y1, z0, z1; REAL ax, ay, az;
    if (!SFX(tex_axis)(u, nx, &x0, &x1, &ax) || !SFX(tex_axis)(v, ny, &y0, &y1, &ay) ||
        !SFX(tex_axis)(w, nz, &z0, &z1, &az)) {
        REAL nan = (REAL)NAN;
        out[0] = nan; out[1] = nan; out[2] = nan; out[3] = nan;
        return;
    }
    REAL mx = (REAL)1 - ax, my = (REAL)1 - ay, mz = (REAL)1 - az;
    size_t r00 = ((size_t)z0 * ny + y0) * nx, r10 = ((size_t)z0 * ny + y1) * nx;
    size_t r01 = ((size_t)z1 * ny + y0) * nx, r11 = ((size_t)z1 * ny + y1) * nx;
    const GRID_T* f000 = g + (r00 + x0) * 4; const GRID_T* f100 = g + (r00 + x1) * 4;
    const GRID_T* f010 = g + (r10 + x0) * 4; const GRID_T* f110 = g + (r10 + x1) * 4;
    const GRID_T* f001 = g + (r01 + x0) * 4; const GRID_T* f101 = g + (r01 + x1) * 4;
    const GRID_T* f011 = g + (r11 + x0) * 4; const GRID_T* f111 = g + (r11 + x1) * 4;
    for (int c = 0; c < 4; c++) {
        REAL c00 = FMA(ax, (REAL)f100[c], mx * (REAL)f000[c]);
        REAL c10 = FMA(ax, (REAL)f110[c], mx * (REAL)f010[c]);
        REAL c01 = FMA(ax, (REAL)f101[c], mx * (REAL)f001[c]);
        REAL c11 = FMA(ax, (REAL)f111[c], mx * (REAL)f011[c]);
        REAL c0 = FMA(ay, c10, my * c00);
        REAL c1 = FMA(ay, c11, my * c01);
        out[c] = FMA(az, c1, mz * c0);
    }
}

typedef struct {
    int nx, ny, nz;
    REAL dA[4], dB[4], dC[4];
} SFX(gridref);

/* ---- Newton polish (opt-in SPM_FLAG_POLISH; not in the reference) ----------
 * After FIRE stops, up to POLISH_STEPS Newton steps q <- q - J^-1 G on the
 * total force G(q) = F_grid(q) + spring(q) [+ c*surf], F_grid the trilinear
 * sample of the force channels and J = dG/dq exact for that interpolant (its
 * texel-coordinate derivatives times n*dinv, plus the spring's Jacobian); a
 * step is kept only if it moves q by at most POLISH_MAX_STEP per axis and
 * lowers |G|^2.  Same operations in the same order as the CUDA kernels
 * (spm_fire.cuh: polish_eval / polish_step / newton_polish), so the FP32
 * instantiation is bit-identical to them.  frame=0: relaxStrokes' spring
 * (tip_force on q - tip); frame=1: tip frame a,b,c with surf along c. */
#define POLISH_STEPS 4
#define POLISH_MAX_STEP 0.1

typedef struct {
    SFX(v3) a, b, c;
    REAL k[4], d0[4];
    REAL surf;
    int frame;
} SFX(pspring);

/* fetch the cell of q: texels t[4*k+2*j+i] (corner x_i,y_j,z_k) and weights */
static inline int SFX(polish_fetch)(const GRID_T* g, const SFX(gridref)* G, SFX(v3) p, REAL t[8][4],
                                    REAL* ax, REAL* ay, REAL* az) {
    REAL u = FMA(p.x, G->dA[0], FMA(p.y, G->dA[1], FMA(p.z, G->dA[2], G->dA[3])));
    REAL v = FMA(p.x, G->dB[0], FMA(p.y, G->dB[1], FMA(p.z, G->dB[2], G->dB[3])));
    REAL w = FMA(p.x, G->dC[0], FMA(p.y, G->dC[1], FMA(p.z, G->dC[2], G->dC[3])));
    int x[2] = {0, 0}, y[2] = {0, 0}, z[2] = {0, 0};
    int ok = SFX(tex_axis)(u, G->nx, &x[0], &x[1], ax);
    ok = SFX(tex_axis)(v, G->ny, &y[0], &y[1], ay) && ok;
    ok = SFX(tex_axis)(w, G->nz, &z[0], &z[1], az) && ok;
    if (!ok) return 0;
    for (int k = 0; k < 2; k++)
        for (int j = 0; j < 2; j++)
            for (int i = 0; i < 2; i++) {
                const GRID_T* f = g + (((size_t)z[k] * G->ny + y[j]) * G->nx + x[i]) * 4;
                for (int c = 0; c < 4; c++) t[4 * k + 2 * j + i][c] = (REAL)f[c];
            }
    return 1;
}

static inline REAL SFX(lerp_c)(REAL a, REAL ma, REAL f0, REAL f1) { return FMA(a, f1, ma * f0); }

static void SFX(polish_eval)(REAL t[8][4], REAL ax, REAL ay, REAL az, REAL T[3][3], const SFX(pspring)* S,
                             SFX(v3) tip, SFX(v3) q, REAL* fe, SFX(v3)* Gv, REAL J[3][3]) {
    const REAL mx = (REAL)1 - ax, my = (REAL)1 - ay, mz = (REAL)1 - az;
    for (int ch = 0; ch < 4; ch++) {
        const REAL f000 = t[0][ch], f100 = t[1][ch], f010 = t[2][ch], f110 = t[3][ch];
        const REAL f001 = t[4][ch], f101 = t[5][ch], f011 = t[6][ch], f111 = t[7][ch];
        const REAL c00 = SFX(lerp_c)(ax, mx, f000, f100), c10 = SFX(lerp_c)(ax, mx, f010, f110);
        const REAL c01 = SFX(lerp_c)(ax, mx, f001, f101), c11 = SFX(lerp_c)(ax, mx, f011, f111);
        const REAL c0 = SFX(lerp_c)(ay, my, c00, c10), c1 = SFX(lerp_c)(ay, my, c01, c11);
        fe[ch] = SFX(lerp_c)(az, mz, c0, c1);
        if (ch < 3) {
            const REAL e0 = SFX(lerp_c)(ay, my, f100 - f000, f110 - f010);
            const REAL e1 = SFX(lerp_c)(ay, my, f101 - f001, f111 - f011);
            const REAL dX = SFX(lerp_c)(az, mz, e0, e1);
            const REAL dY = SFX(lerp_c)(az, mz, c10 - c00, c11 - c01);
            const REAL dZ = c1 - c0;
            for (int m = 0; m < 3; m++) J[ch][m] = FMA(dZ, T[2][m], FMA(dY, T[1][m], dX * T[0][m]));
        }
    }
    SFX(v3) d = S->frame ? SFX(rotmat)(SFX(sub3)(q, tip), S->a, S->b, S->c) : SFX(sub3)(q, tip);
    SFX(v3) fs = SFX(tip_force)(d, S->k, S->d0);
    SFX(v3) ft = S->frame ? SFX(rotmatT)(fs, S->a, S->b, S->c) : fs;
    *Gv = SFX(mk3)(fe[0] + ft.x, fe[1] + ft.y, fe[2] + ft.z);
    if (S->frame) {
        Gv->x = FMA(S->c.x, S->surf, Gv->x);
        Gv->y = FMA(S->c.y, S->surf, Gv->y);
        Gv->z = FMA(S->c.z, S->surf, Gv->z);
    }
    REAL Jd[3][3] = {{S->k[0], 0, 0}, {0, S->k[1], 0}, {0, 0, S->k[2]}};
    if (S->k[3] != (REAL)0) {
        REAL r = SQRT(SFX(dot3)(d, d));
        r = FMAX(r, (REAL)1e-10);
        const REAL s = (S->k[3] * (r - S->d0[3])) / r;
        const REAL beta = (S->k[3] * S->d0[3]) / ((r * r) * r);
        const REAL dv[3] = {d.x, d.y, d.z};
        Jd[0][0] = S->k[0] + s;
        Jd[1][1] = S->k[1] + s;
        Jd[2][2] = S->k[2] + s;
        for (int i = 0; i < 3; i++) {
            const REAL bd = beta * dv[i];
            for (int j = 0; j < 3; j++) Jd[i][j] = FMA(bd, dv[j], Jd[i][j]);
        }
    }
    if (S->frame) {
        const REAL R[3][3] = {{S->a.x, S->a.y, S->a.z}, {S->b.x, S->b.y, S->b.z}, {S->c.x, S->c.y, S->c.z}};
        REAL M[3][3];
        for (int m = 0; m < 3; m++)
            for (int j = 0; j < 3; j++) M[m][j] = FMA(Jd[m][2], R[2][j], FMA(Jd[m][1], R[1][j], Jd[m][0] * R[0][j]));
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                J[i][j] = J[i][j] + FMA(R[2][i], M[2][j], FMA(R[1][i], M[1][j], R[0][i] * M[0][j]));
    } else {
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) J[i][j] = J[i][j] + Jd[i][j];
    }
}

static int SFX(polish_step)(REAL J[3][3], SFX(v3) Gv, SFX(v3)* dq) {
    REAL A[3][3];
    A[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    A[0][1] = J[0][2] * J[2][1] - J[0][1] * J[2][2];
    A[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
    A[1][0] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    A[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
    A[1][2] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
    A[2][0] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    A[2][1] = J[0][1] * J[2][0] - J[0][0] * J[2][1];
    A[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    const REAL det = (J[0][0] * A[0][0] + J[0][1] * A[1][0]) + J[0][2] * A[2][0];
    if (!(det != (REAL)0)) return 0;
    REAL r[3];
    for (int i = 0; i < 3; i++) {
        const REAL tq = (A[i][0] * Gv.x + A[i][1] * Gv.y) + A[i][2] * Gv.z;
        r[i] = (-tq) / det;
    }
    if (!(FABS(r[0]) <= (REAL)POLISH_MAX_STEP && FABS(r[1]) <= (REAL)POLISH_MAX_STEP &&
          FABS(r[2]) <= (REAL)POLISH_MAX_STEP))
        return 0;
    *dq = SFX(mk3)(r[0], r[1], r[2]);
    return 1;
}

/* q in/out; fe: the sample at the final q (left unchanged with q if q's cell
 * is outside the sampler's range). */
static void SFX(newton_polish)(const GRID_T* g, const SFX(gridref)* G, const SFX(pspring)* S, SFX(v3) tip,
                               SFX(v3)* q, REAL* fe) {
    REAL T[3][3];
    const REAL fx = (REAL)G->nx, fy = (REAL)G->ny, fz = (REAL)G->nz;
    for (int m = 0; m < 3; m++) { T[0][m] = fx * G->dA[m]; T[1][m] = fy * G->dB[m]; T[2][m] = fz * G->dC[m]; }
    REAL t[8][4], ax = 0, ay = 0, az = 0;
    if (!SFX(polish_fetch)(g, G, *q, t, &ax, &ay, &az)) return;
    REAL J[3][3], fe0[4];
    SFX(v3) Gv;
    SFX(polish_eval)(t, ax, ay, az, T, S, tip, *q, fe0, &Gv, J);
    REAL g2 = SFX(dot3)(Gv, Gv);
    for (int it = 0; it < POLISH_STEPS; it++) {
        SFX(v3) dq;
        if (!SFX(polish_step)(J, Gv, &dq)) break;
        const SFX(v3) q1 = SFX(add3)(*q, dq);
        if (!SFX(polish_fetch)(g, G, q1, t, &ax, &ay, &az)) break;
        REAL J1[3][3], fe1[4];
        SFX(v3) G1;
        SFX(polish_eval)(t, ax, ay, az, T, S, tip, q1, fe1, &G1, J1);
        const REAL g21 = SFX(dot3)(G1, G1);
        if (!(g21 < g2)) break;
        *q = q1;
        for (int c = 0; c < 4; c++) fe0[c] = fe1[c];
        Gv = G1;
        g2 = g21;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) J[i][j] = J1[i][j];
    }
    for (int c = 0; c < 4; c++) fe[c] = fe0[c];
}

/* relaxStrokes: one pixel, all z-steps                    AFM.cl:345-394
 * FEs/disps are (nzs,4) rows for this pixel in stroke order (iz=0 highest),
 * or reversed when flip!=0 (the z flip scan_fdbm applies on the host). */
static void SFX(relax_strokes_pixel)(const GRID_T* g, const SFX(gridref)* G, const float* pt,
                                     int nzs, const REAL* dTip, const REAL* k, const REAL* d0,
                                     const REAL* relax, int max_iter, REAL f2conv, int use_fire,
                                     int flip, int polish, REAL* FEs, REAL* disps) {
    SFX(pspring) S;
    S.a = S.b = S.c = SFX(mk3)(0, 0, 0);
    for (int i = 0; i < 4; i++) { S.k[i] = k[i]; S.d0[i] = d0[i]; }
    S.surf = 0;
    S.frame = 0;
    SFX(v3) tip = SFX(mk3)((REAL)pt[0], (REAL)pt[1], (REAL)pt[2]);
    SFX(v3) pos = SFX(mk3)(tip.x + d0[0], tip.y + d0[1], tip.z + d0[2]);
    REAL dt = relax[0], damp = relax[1];
    REAL dtmax = dt, dtmin = dtmax * (REAL)0.1, damp0 = damp;
    for (int iz = 0; iz < nzs; iz++) {
        SFX(v3) v = SFX(mk3)(0, 0, 0);
        REAL fe[4] = {0, 0, 0, 0};
        for (int i = 0; i < max_iter; i++) {
            SFX(interp_fe)(g, G->nx, G->ny, G->nz, G->dA, G->dB, G->dC, pos, fe);
            SFX(v3) ft = SFX(tip_force)(SFX(sub3)(pos, tip), k, d0);
            SFX(v3) f = SFX(mk3)(fe[0] + ft.x, fe[1] + ft.y, fe[2] + ft.z);
            SFX(md_step)(f, &v, &pos, &dt, &damp, dtmin, dtmax, damp0, use_fire);
            if (SFX(dot3)(f, f) < f2conv) break;
        }
        int oz = flip ? (nzs - 1 - iz) : iz;
        SFX(v3) q = pos;  /* output position; the next z-step starts from pos */
        if (polish) SFX(newton_polish)(g, G, &S, tip, &q, fe);
        SFX(v3) ref = SFX(mk3)(tip.x + d0[0], tip.y + d0[1], tip.z + d0[2]);
        FEs[oz * 4 + 0] = fe[0]; FEs[oz * 4 + 1] = fe[1];
        FEs[oz * 4 + 2] = fe[2]; FEs[oz * 4 + 3] = fe[3];
        disps[oz * 4 + 0] = q.x - ref.x; disps[oz * 4 + 1] = q.y - ref.y;
        disps[oz * 4 + 2] = q.z - ref.z; disps[oz * 4 + 3] = 0;
        tip.x = tip.x + dTip[0]; tip.y = tip.y + dTip[1]; tip.z = tip.z + dTip[2];
        pos.x = pos.x + dTip[0]; pos.y = pos.y + dTip[1]; pos.z = pos.z + dTip[2];
    }
}

/* relaxStrokes2D: one pixel                                AFM.cl:410-450
 * z fixed per slice (pz = az - iz*dh), x,y relaxed by damped MD from the anchor
 * (reset per slice): f = F_grid.xy - K (p - anchor), v = v*(1-damp) + f*dt,
 * p += v*dt, stop after the update once |f|^2 < f2conv or after max_iter
 * steps; FE re-sampled at the final position, disps = (p - anchor, 0, 0). */
static void SFX(relax_2d_pixel)(const GRID_T* g, const SFX(gridref)* G, const float* pt, int nzs, REAL K,
                                REAL dh, REAL dt, REAL damp, int max_iter, REAL f2conv, int flip, REAL* FEs,
                                REAL* disps) {
    const REAL ax = (REAL)pt[0], ay = (REAL)pt[1], az = (REAL)pt[2];
    const REAL cv = (REAL)1 - damp;
    for (int iz = 0; iz < nzs; iz++) {
        const REAL pz = az - (REAL)iz * dh;
        REAL px = ax, py = ay, vx = 0, vy = 0;
        REAL fe[4];
        for (int i = 0; i < max_iter; i++) {
            SFX(interp_fe)(g, G->nx, G->ny, G->nz, G->dA, G->dB, G->dC, SFX(mk3)(px, py, pz), fe);
            const REAL fx = fe[0] - K * (px - ax);
            const REAL fy = fe[1] - K * (py - ay);
            vx = FMA(fx, dt, vx * cv);
            vy = FMA(fy, dt, vy * cv);
            px = FMA(vx, dt, px);
            py = FMA(vy, dt, py);
            if (FMA(fy, fy, fx * fx) < f2conv) break;
        }
        SFX(interp_fe)(g, G->nx, G->ny, G->nz, G->dA, G->dB, G->dC, SFX(mk3)(px, py, pz), fe);
        const int oz = flip ? (nzs - 1 - iz) : iz;
        FEs[oz * 4 + 0] = fe[0]; FEs[oz * 4 + 1] = fe[1];
        FEs[oz * 4 + 2] = fe[2]; FEs[oz * 4 + 3] = fe[3];
        disps[oz * 4 + 0] = px - ax; disps[oz * 4 + 1] = py - ay;
        disps[oz * 4 + 2] = 0; disps[oz * 4 + 3] = 0;
    }
}

/* relaxStrokesTilted: one pixel                            AFM.cl:478-562 */
static void SFX(relax_tilted_pixel)(const GRID_T* g, const SFX(gridref)* G, const float* pt, int nzs,
                                    const REAL* tA, const REAL* tB, const REAL* tC, const REAL* k,
                                    const REAL* d0, const REAL* relax, const REAL* surf, int max_iter,
                                    REAL f2conv, int use_fire, int polish, REAL* FEs) {
    SFX(v3) a = SFX(mk3)(tA[0], tA[1], tA[2]);
    SFX(v3) b = SFX(mk3)(tB[0], tB[1], tB[2]);
    SFX(v3) c = SFX(mk3)(tC[0], tC[1], tC[2]);
    SFX(v3) dTip = SFX(mk3)(c.x * tC[3], c.y * tC[3], c.z * tC[3]);
    SFX(v3) d0r = SFX(rotmatT)(SFX(mk3)(d0[0], d0[1], d0[2]), a, b, c);
    SFX(v3) tip = SFX(mk3)((REAL)pt[0], (REAL)pt[1], (REAL)pt[2]);
    SFX(v3) pos = SFX(add3)(tip, d0r);
    REAL dt = relax[0], damp = relax[1];
    REAL dtmax = dt, dtmin = dtmax * (REAL)0.1, damp0 = damp;
    for (int iz = 0; iz < nzs; iz++) {
        SFX(v3) v = SFX(mk3)(0, 0, 0);
        REAL fe[4];
        for (int i = 0; i < max_iter; i++) {
            SFX(interp_fe)(g, G->nx, G->ny, G->nz, G->dA, G->dB, G->dC, pos, fe);
            SFX(v3) dl = SFX(rotmat)(SFX(sub3)(pos, tip), a, b, c);
            SFX(v3) ft = SFX(rotmatT)(SFX(tip_force)(dl, k, d0), a, b, c);
            SFX(v3) f = SFX(mk3)(fe[0] + ft.x, fe[1] + ft.y, fe[2] + ft.z);
            f.x = FMA(c.x, surf[0], f.x); f.y = FMA(c.y, surf[0], f.y); f.z = FMA(c.z, surf[0], f.z);
            SFX(md_step)(f, &v, &pos, &dt, &damp, dtmin, dtmax, damp0, use_fire);
            if (SFX(dot3)(f, f) < f2conv) break;
        }
        SFX(interp_fe)(g, G->nx, G->ny, G->nz, G->dA, G->dB, G->dC, pos, fe);
        if (polish) {
            SFX(pspring) S;
            S.a = a; S.b = b; S.c = c;
            for (int i = 0; i < 4; i++) { S.k[i] = k[i]; S.d0[i] = d0[i]; }
            S.surf = surf[0];
            S.frame = 1;
            SFX(v3) q = pos;
            SFX(newton_polish)(g, G, &S, tip, &q, fe);
        }
        SFX(v3) fr = SFX(rotmat)(SFX(mk3)(fe[0], fe[1], fe[2]), a, b, c);
        FEs[iz * 4 + 0] = fr.x; FEs[iz * 4 + 1] = fr.y; FEs[iz * 4 + 2] = fr.z; FEs[iz * 4 + 3] = fe[3];
        tip = SFX(add3)(tip, dTip);
        pos = SFX(add3)(pos, dTip);
    }
}

/* getFEinStrokesTilted: raw (unrelaxed) sampling          AFM.cl:210-233 */
static void SFX(raw_tilted_pixel)(const GRID_T* g, const SFX(gridref)* G, const float* pt, int nzs,
                                  const REAL* tA, const REAL* tB, const REAL* tC, const REAL* dTip,
                                  const REAL* d0, REAL* FEs) {
    SFX(v3) a = SFX(mk3)(tA[0], tA[1], tA[2]);
    SFX(v3) b = SFX(mk3)(tB[0], tB[1], tB[2]);
    SFX(v3) c = SFX(mk3)(tC[0], tC[1], tC[2]);
    SFX(v3) pos = SFX(mk3)((REAL)pt[0] + d0[0], (REAL)pt[1] + d0[1], (REAL)pt[2] + d0[2]);
    REAL fe[4];
    for (int iz = 0; iz < nzs; iz++) {
        SFX(interp_fe)(g, G->nx, G->ny, G->nz, G->dA, G->dB, G->dC, pos, fe);
        SFX(v3) fr = SFX(rotmat)(SFX(mk3)(fe[0], fe[1], fe[2]), a, b, c);
        FEs[iz * 4 + 0] = fr.x; FEs[iz * 4 + 1] = fr.y; FEs[iz * 4 + 2] = fr.z; FEs[iz * 4 + 3] = fe[3];
        pos.x = pos.x + dTip[0]; pos.y = pos.y + dTip[1]; pos.z = pos.z + dTip[2];
    }
}

/* ---- pair laws ------------------------------------------------------------ */

/* getCoulombAFM(atom,pos)*Qs accumulated into fe        AFM.cl:730-736 */
static inline void SFX(acc_coulomb)(REAL* fe, const REAL* atom, SFX(v3) pos, REAL qs) {
    SFX(v3) dp = SFX(mk3)(pos.x - atom[0], pos.y - atom[1], pos.z - atom[2]);
    REAL ir2 = (REAL)1 / (SFX(dot3)(dp, dp) + (REAL)1e-4);
    REAL E = atom[3] * SQRT(ir2);
    REAL s = E * ir2;
    fe[0] += dp.x * s * qs; fe[1] += dp.y * s * qs; fe[2] += dp.z * s * qs; fe[3] += E * qs;
}

/* getLJ                                                 AFM.cl:738-745 */
static inline void SFX(acc_lj)(REAL* fe, const REAL* atom, REAL c6, REAL c12, SFX(v3) pos) {
    SFX(v3) dp = SFX(mk3)(pos.x - atom[0], pos.y - atom[1], pos.z - atom[2]);
    REAL ir2 = (REAL)1 / (SFX(dot3)(dp, dp) + (REAL)1e-4);
    REAL ir6 = ir2 * ir2 * ir2;
    REAL E = (c12 * ir6 - c6) * ir6;
    REAL fr = ((REAL)12 * c12 * ir6 - (REAL)6 * c6) * ir6 * ir2;
    fe[0] += dp.x * fr; fe[1] += dp.y * fr; fe[2] += dp.z * fr; fe[3] += E;
}

/* getMorse                                              AFM.cl:747-757 */
static inline void SFX(acc_morse)(REAL* fe, SFX(v3) dp, REAL R0, REAL E0, REAL K) {
    REAL r = SQRT(SFX(dot3)(dp, dp) + (REAL)1e-4);
    REAL e = EXP(K * (r - R0));
    REAL E = E0 * e * (e - (REAL)2);
    REAL fr = -E0 * e * (e - (REAL)1) * (REAL)2 * K;
    REAL s = fr / r;
    fe[0] += dp.x * s; fe[1] += dp.y * s; fe[2] += dp.z * s; fe[3] += E;
}

/* Sum of the pair law over all atoms at one query point (4 tip-charge sites at
 * world-z offsets QZs, Qs pre-scaled by COULOMB_CONST). kind: 0=LJ, 1=Morse. */
static inline void SFX(pair_fe)(int kind, int na, const REAL* atoms, const REAL* prm, int pstride,
                                SFX(v3) pos, const REAL* Qs, const REAL* QZs, REAL* fe) {
    fe[0] = fe[1] = fe[2] = fe[3] = 0;
    for (int j = 0; j < na; j++) {
        const REAL* at = atoms + 4 * j;
        const REAL* pj = prm + pstride * j;
        if (kind == 0) {
            SFX(acc_lj)(fe, at, pj[0], pj[1], pos);
        } else {
            SFX(acc_morse)(fe, SFX(mk3)(pos.x - at[0], pos.y - at[1], pos.z - at[2]), pj[0], pj[1], pj[2]);
        }
        for (int s = 0; s < 4; s++) {
            if (Qs[s] == (REAL)0) continue;   /* exact: a zero-charge site adds only zeros */
            SFX(acc_coulomb)(fe, at, SFX(mk3)(pos.x, pos.y, pos.z + QZs[s]), Qs[s]);
        }
    }
}

/* relaxStrokesTiltedMorseDirect: one pixel (convergence tested BEFORE the
 * update; PPs.w = +iters converged / -iters not)        AFM.cl:1419-1511 */
/* quirks (0 = kernel semantics): bit0 keeps v across z-steps and bit1 takes
 * the integrator state (dt, damp) from *carry and leaves it there, which is how
 * the reference's FP64 test oracle _cpu_relax_direct
 * (tests/SPM/test_afm_morse.py:548-604) loops; used only to pin this
 * restatement against that oracle's golden output. */
static void SFX(relax_direct_pixel)(int na, const REAL* atoms, const REAL* cMs, const float* pt, int nzs,
                                    const REAL* tA, const REAL* tB, const REAL* tC, const REAL* k,
                                    const REAL* d0, const REAL* relax, const REAL* surf,
                                    const REAL* Qs, const REAL* QZs, int max_iter, REAL f2conv,
                                    REAL* FEs, REAL* PPs, int quirks, REAL* carry) {
    SFX(v3) a = SFX(mk3)(tA[0], tA[1], tA[2]);
    SFX(v3) b = SFX(mk3)(tB[0], tB[1], tB[2]);
    SFX(v3) c = SFX(mk3)(tC[0], tC[1], tC[2]);
    SFX(v3) dTip = SFX(mk3)(c.x * tC[3], c.y * tC[3], c.z * tC[3]);
    SFX(v3) d0r = SFX(rotmatT)(SFX(mk3)(d0[0], d0[1], d0[2]), a, b, c);
    SFX(v3) tip = SFX(mk3)((REAL)pt[0], (REAL)pt[1], (REAL)pt[2]);
    SFX(v3) pos = SFX(add3)(tip, d0r);
    REAL dt = relax[0], damp = relax[1];
    REAL dtmax = dt, dtmin = dtmax * (REAL)0.1, damp0 = damp;
    if (quirks & 2) { dt = carry[0]; damp = carry[1]; }
    SFX(v3) v = SFX(mk3)(0, 0, 0);
    for (int iz = 0; iz < nzs; iz++) {
        if (!(quirks & 1)) v = SFX(mk3)(0, 0, 0);
        REAL fe[4];
        int itr = 0, conv = 0;
        for (int i = 0; i < max_iter; i++) {
            itr = i + 1;
            SFX(pair_fe)(1, na, atoms, cMs, 4, pos, Qs, QZs, fe);
            SFX(v3) dl = SFX(rotmat)(SFX(sub3)(pos, tip), a, b, c);
            SFX(v3) ft = SFX(rotmatT)(SFX(tip_force)(dl, k, d0), a, b, c);
            SFX(v3) f = SFX(mk3)(fe[0] + ft.x, fe[1] + ft.y, fe[2] + ft.z);
            f.x = FMA(c.x, surf[0], f.x); f.y = FMA(c.y, surf[0], f.y); f.z = FMA(c.z, surf[0], f.z);
            if (SFX(dot3)(f, f) < f2conv) { conv = 1; break; }
            SFX(md_step)(f, &v, &pos, &dt, &damp, dtmin, dtmax, damp0, 1);
        }
        SFX(pair_fe)(1, na, atoms, cMs, 4, pos, Qs, QZs, fe);
        SFX(v3) fr = SFX(rotmat)(SFX(mk3)(fe[0], fe[1], fe[2]), a, b, c);
        FEs[iz * 4 + 0] = fr.x; FEs[iz * 4 + 1] = fr.y; FEs[iz * 4 + 2] = fr.z; FEs[iz * 4 + 3] = fe[3];
        int finite = isfinite(fe[0]) && isfinite(fe[1]) && isfinite(fe[2]) && isfinite(fe[3]) &&
                     isfinite(pos.x) && isfinite(pos.y) && isfinite(pos.z);
        int itw = (conv && finite) ? itr : -itr;
        PPs[iz * 4 + 0] = pos.x; PPs[iz * 4 + 1] = pos.y; PPs[iz * 4 + 2] = pos.z; PPs[iz * 4 + 3] = (REAL)itw;
        tip = SFX(add3)(tip, dTip);
        pos = SFX(add3)(pos, dTip);
    }
    if (quirks & 2) { carry[0] = dt; carry[1] = damp; }
}

/* Grid relaxation with the direct path's bookkeeping (convergence tested
 * before each update, PPs = (pos, +iters / -iters), FE re-sampled only when
 * the position moved after the last sample): relaxStrokesTilted's tip frame,
 * spring and surface bias (AFM.cl:478-562) with the control flow of
 * relaxStrokesTiltedMorseDirect (AFM.cl:1441-1505).  Used by the
 * differentiable grid path, whose implicit adjoint needs the equilibrium. */
static void SFX(relax_pp_pixel)(const GRID_T* g, const SFX(gridref)* G, const float* pt, int nzs,
                                const REAL* tA, const REAL* tB, const REAL* tC, const REAL* k,
                                const REAL* d0, const REAL* relax, const REAL* surf, int max_iter,
                                REAL f2conv, int use_fire, int polish, REAL* FEs, REAL* PPs) {
    SFX(v3) a = SFX(mk3)(tA[0], tA[1], tA[2]);
    SFX(v3) b = SFX(mk3)(tB[0], tB[1], tB[2]);
    SFX(v3) c = SFX(mk3)(tC[0], tC[1], tC[2]);
    SFX(v3) dTip = SFX(mk3)(c.x * tC[3], c.y * tC[3], c.z * tC[3]);
    SFX(v3) d0r = SFX(rotmatT)(SFX(mk3)(d0[0], d0[1], d0[2]), a, b, c);
    SFX(v3) tip = SFX(mk3)((REAL)pt[0], (REAL)pt[1], (REAL)pt[2]);
    SFX(v3) pos = SFX(add3)(tip, d0r);
    REAL dt = relax[0], damp = relax[1];
    REAL dtmax = dt, dtmin = dtmax * (REAL)0.1, damp0 = damp;
    for (int iz = 0; iz < nzs; iz++) {
        SFX(v3) v = SFX(mk3)(0, 0, 0);
        REAL fe[4] = {0, 0, 0, 0};
        int itr = 0, conv = 0;
        for (int i = 0; i < max_iter; i++) {
            itr = i + 1;
            SFX(interp_fe)(g, G->nx, G->ny, G->nz, G->dA, G->dB, G->dC, pos, fe);
            SFX(v3) dl = SFX(rotmat)(SFX(sub3)(pos, tip), a, b, c);
            SFX(v3) ft = SFX(rotmatT)(SFX(tip_force)(dl, k, d0), a, b, c);
            SFX(v3) f = SFX(mk3)(fe[0] + ft.x, fe[1] + ft.y, fe[2] + ft.z);
            f.x = FMA(c.x, surf[0], f.x); f.y = FMA(c.y, surf[0], f.y); f.z = FMA(c.z, surf[0], f.z);
            if (SFX(dot3)(f, f) < f2conv) { conv = 1; break; }
            SFX(md_step)(f, &v, &pos, &dt, &damp, dtmin, dtmax, damp0, use_fire);
        }
        if (!conv) SFX(interp_fe)(g, G->nx, G->ny, G->nz, G->dA, G->dB, G->dC, pos, fe);
        SFX(v3) q = pos;  /* output position; the next z-step starts from pos */
        if (polish) {
            SFX(pspring) S;
            S.a = a; S.b = b; S.c = c;
            for (int i = 0; i < 4; i++) { S.k[i] = k[i]; S.d0[i] = d0[i]; }
            S.surf = surf[0];
            S.frame = 1;
            SFX(newton_polish)(g, G, &S, tip, &q, fe);
        }
        SFX(v3) fr = SFX(rotmat)(SFX(mk3)(fe[0], fe[1], fe[2]), a, b, c);
        FEs[iz * 4 + 0] = fr.x; FEs[iz * 4 + 1] = fr.y; FEs[iz * 4 + 2] = fr.z; FEs[iz * 4 + 3] = fe[3];
        int finite = isfinite(fe[0]) && isfinite(fe[1]) && isfinite(fe[2]) && isfinite(fe[3]) &&
                     isfinite(q.x) && isfinite(q.y) && isfinite(q.z);
        PPs[iz * 4 + 0] = q.x; PPs[iz * 4 + 1] = q.y; PPs[iz * 4 + 2] = q.z;
        PPs[iz * 4 + 3] = (REAL)((conv && finite) ? itr : -itr);
        tip = SFX(add3)(tip, dTip);
        pos = SFX(add3)(pos, dTip);
    }
}
