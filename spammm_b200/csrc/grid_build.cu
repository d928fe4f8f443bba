// grid_build.cu -- stage (a): LJ/Morse + point-charge Coulomb force grid.
//
// Replaces evalLJC_QZs_toImg / evalMorseC_QZs_toImg (SPAMMM kernels/AFM.cl:
// 916-1056) behind AFMulator.make_forcefield (spammm/SPM/AFM.py:897-946).
//
// B200 shape.  One thread owns a z-column of GB_ZB (16) nodes at fixed (ia,ib); a
// CTA is 32 (x) x 4 (y) threads, so stores of the (nz,ny,nx,4) grid are
// 512-byte coalesced rows.  Atoms are staged GB_TILE at a time in shared
// memory already transformed for the inner loop, read back as warp-uniform
// broadcasts.  The work per (node, atom) pair is FP32 FMA + MUFU bound, so the
// inner loop is written to minimise issued instructions:
//   * every reference grid has dC = (0,0,dz): dx^2+dy^2+R2SAFE of a pair is
//     computed once per (thread, atom) and shared by the column's nodes;
//   * nodes are evaluated two at a time with Blackwell's packed FP32
//     instructions (fma/mul/add/sub .f32x2), halving the FP32 issue count;
//   * tip-charge sites with a zero z-offset sit on the node itself; their
//     charges are merged into one term that reuses the pair law's 1/r (one
//     MUFU rsqrt per pair in total for LJ + on-node Coulomb); sites with a
//     non-zero offset get their own rsqrt.
// Transcendentals use MUFU approximations (rsqrt.approx, ex2.approx).
#include "spm_internal.cuh"
#include "spm_batch.cuh"
#include "spm_f32x2.cuh"

namespace spm {
namespace {

constexpr int GB_TX = 32;     // threads along x
constexpr int GB_TY = 4;      // threads along y
constexpr int GB_ZB = 16;     // nodes along z per thread (8 packed pairs: the per-atom overhead
                              // of the tile loop amortised over 16 nodes; 7% faster than 8 on a
                              // 1200-atom 480x480x240 grid)
constexpr int GB_TILE = 256;  // atoms per shared-memory tile
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
__device__ __forceinline__ f2 rsqrt2(f2 x) {
    float a, b;
    upk(x, a, b);
    return pk(fast_rsqrt(a), fast_rsqrt(b));
}
__device__ __forceinline__ f2 ex2_2(f2 x) {
    float a, b;
    upk(x, a, b);
    return pk(fast_ex2(a), fast_ex2(b));
}
struct GridGeom {
    int nx, ny, nz;
    float4 p0, dA, dB, dC;
};

struct TipSites {
    float qs_on;   // sum of Qs[k]*COULOMB_CONST over sites with QZs[k] == 0
    float qs[4];   // Qs[k]*COULOMB_CONST of the non-zero sites with QZs[k] != 0
    float qz[4];   // their z-offsets
};

// Node coordinate along one axis: p0 + dA*ia + dB*ib (+ dC*ic), in this
// fixed operation order in every kernel, so a batched slab node gets the same
// bits as the same node of a full per-molecule grid.
__device__ __forceinline__ float node_xy(float p0, float da, float db, int ia, int ib) {
    return __fmaf_rn(db, (float)ib, __fmaf_rn(da, (float)ia, p0));
}

// The stored box of a build: columns [x_lo, x_lo + nxs), rows [y_lo, y_lo +
// nys) and layers [zst_lo, zst_hi) of the full grid.
struct StoreBox {
    int x_lo, nxs, y_lo, nys, zst_lo, zst_hi;
};

// One CTA tile: a (blockDim.x x blockDim.y) patch of z-columns (full-grid
// column ia, row ib), ZB nodes each starting at global layer ic0; nodes
// outside the box B are not stored, the rest go to out[idx], idx = (zl*nys +
// yl)*nxs + xl with (xl, yl, zl) = (ia - x_lo, ib - y_lo, ic - zst_lo)
// (LAYOUT 1).  LAYOUT 2, x-pairs: out[2*idx + dx] = value(x_lo + (xl + dx) mod
// nxs), so a node's value is also written to its x-1 neighbour's second slot.
// LAYOUT 4, xz-quads: out[4*idx + 2*dz + dx] = value(x_lo + (xl + dx) mod nxs,
// zst_lo + (zl + dz) mod (zst_hi - zst_lo)), written to the four nodes whose
// quads contain it.
// KIND: SPM_KIND_LJ / SPM_KIND_MORSE; ON: an on-node charge term exists;
// NOFF: number of off-node sites.
template <int KIND, bool ON, int NOFF, int ZB, int LAYOUT = 1>
__device__ __forceinline__ void build_tile(int na, const float4* __restrict__ atoms, const float* __restrict__ params,
                                           int pstride, float4* __restrict__ out, const GridGeom& G,
                                           const TipSites& S, const StoreBox& B, int ia, int ib, int ic0) {
    constexpr int ZP = ZB / 2;
    __shared__ float4 s_pos[GB_TILE];                   // (x, y, z, Q*qs_on)
    __shared__ float4 s_prm[GB_TILE];                   // transformed pair parameters
    __shared__ float s_q[NOFF > 0 ? NOFF : 1][GB_TILE];  // Q*Qs[k]*C per off-node site

    const int nthr = blockDim.x * blockDim.y;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int xl = ia - B.x_lo, yl = ib - B.y_lo;
    const bool active = (unsigned)xl < (unsigned)B.nxs && (unsigned)yl < (unsigned)B.nys;

    const float px = node_xy(G.p0.x, G.dA.x, G.dB.x, ia, ib);
    const float py = node_xy(G.p0.y, G.dA.y, G.dB.y, ia, ib);
    const float pzb = node_xy(G.p0.z, G.dA.z, G.dB.z, ia, ib);
    f2 pz[ZP];
#pragma unroll
    for (int p = 0; p < ZP; p++)
        pz[p] = pk(__fmaf_rn(G.dC.z, (float)(ic0 + 2 * p), pzb), __fmaf_rn(G.dC.z, (float)(ic0 + 2 * p + 1), pzb));

    const f2 zero = pk(0.f, 0.f);
    f2 fx[ZP], fy[ZP], fz[ZP], fe[ZP];
#pragma unroll
    for (int p = 0; p < ZP; p++) { fx[p] = zero; fy[p] = zero; fz[p] = zero; fe[p] = zero; }
    const f2 one = bc(1.f);

    for (int t0 = 0; t0 < na; t0 += GB_TILE) {
        const int nt = min(GB_TILE, na - t0);
        for (int j = tid; j < nt; j += nthr) {
            float4 a = __ldg(atoms + t0 + j);
            const float* pr = params + (size_t)(t0 + j) * pstride;
            s_pos[j] = make_float4(a.x, a.y, a.z, a.w * S.qs_on);
            if (KIND == SPM_KIND_MORSE) {
                float R0 = __ldg(pr + 0), E0 = __ldg(pr + 1), K = __ldg(pr + 2);
                s_prm[j] = make_float4(K * LOG2E, -K * R0 * LOG2E, E0, -2.f * K * E0);
            } else {
                float c6 = __ldg(pr + 0), c12 = __ldg(pr + 1);
                s_prm[j] = make_float4(-c6, c12, -6.f * c6, 12.f * c12);
            }
#pragma unroll
            for (int k = 0; k < NOFF; k++) s_q[k][j] = a.w * S.qs[k];
        }
        __syncthreads();
        if (active) {
#pragma unroll 1
            for (int j = 0; j < nt; j++) {
                const float4 a = s_pos[j];
                const float4 c = s_prm[j];
                const float dxs = px - a.x;
                const float dys = py - a.y;
                const float dxy2s = fmaf(dxs, dxs, fmaf(dys, dys, R2SAFE));
                const f2 dx = bc(dxs), dy = bc(dys), dxy2 = bc(dxy2s), az = bc(a.z);
                const f2 c0 = bc(c.x), c1 = bc(c.y), c2 = bc(c.z), c3 = bc(c.w);
                const f2 qon = bc(a.w);
#pragma unroll
                for (int p = 0; p < ZP; p++) {
                    const f2 dz = sub2(pz[p], az);
                    const f2 r2 = fma2(dz, dz, dxy2);
                    const f2 rs = rsqrt2(r2);
                    // s = |F|/r of the pair law plus the on-node charges; the charges' Q/r^3 is
                    // added before the last factor 1/r (Morse) or 1/r^2 (LJ) the two terms share
                    f2 s;
                    if (KIND == SPM_KIND_MORSE) {
                        // E = E0 e (e-2) = E0 (w - e), F = dp * (-2 K E0) w / r, w = e (e-1), e = exp(K (r-R0))
                        const f2 r = mul2(r2, rs);
                        const f2 e = ex2_2(fma2(c0, r, c1));
                        const f2 w = mul2(e, sub2(e, one));
                        fe[p] = fma2(c2, sub2(w, e), fe[p]);
                        const f2 m = mul2(c3, w);
                        if (ON) {
                            const f2 Ek = mul2(qon, rs);
                            fe[p] = add2(fe[p], Ek);
                            s = mul2(fma2(Ek, rs, m), rs);
                        } else {
                            s = mul2(m, rs);
                        }
                    } else {
                        // E = (c12 ir6 - c6) ir6, F = dp * (12 c12 ir6 - 6 c6) ir6 ir2
                        const f2 ir2 = mul2(rs, rs);
                        const f2 ir6 = mul2(mul2(ir2, ir2), ir2);
                        fe[p] = fma2(fma2(c1, ir6, c0), ir6, fe[p]);
                        if (ON) {
                            const f2 Ek = mul2(qon, rs);
                            fe[p] = add2(fe[p], Ek);
                            s = mul2(fma2(fma2(c3, ir6, c2), ir6, Ek), ir2);
                        } else {
                            s = mul2(mul2(fma2(c3, ir6, c2), ir6), ir2);
                        }
                    }
                    fx[p] = fma2(dx, s, fx[p]);
                    fy[p] = fma2(dy, s, fy[p]);
                    fz[p] = fma2(dz, s, fz[p]);
#pragma unroll
                    for (int k = 0; k < NOFF; k++) {
                        // Coulomb at the tip-charge site node + zhat*QZs[k]
                        const f2 dzk = add2(dz, bc(S.qz[k]));
                        const f2 rsk = rsqrt2(fma2(dzk, dzk, dxy2));
                        const f2 Ek = mul2(bc(s_q[k][j]), rsk);
                        fe[p] = add2(fe[p], Ek);
                        const f2 sk = mul2(mul2(Ek, rsk), rsk);
                        fx[p] = fma2(dx, sk, fx[p]);
                        fy[p] = fma2(dy, sk, fy[p]);
                        fz[p] = fma2(dzk, sk, fz[p]);
                    }
                }
            }
        }
        __syncthreads();
    }
    if (!active) return;
#pragma unroll
    for (int p = 0; p < ZP; p++) {
        float x[2], y[2], z[2], e[2];
        upk(fx[p], x[0], x[1]);
        upk(fy[p], y[0], y[1]);
        upk(fz[p], z[0], z[1]);
        upk(fe[p], e[0], e[1]);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int ic = ic0 + 2 * p + h;
            if (ic >= B.zst_hi) break;
            float4 o = make_float4(x[h], y[h], z[h], e[h]);
            // |E| > 100 cap of the reference builders (AFM.cl:1053-1054)
            // (the division only where it can scale: 100/|E| < 1 needs |E| > 100; NaN compares false)
            if (fabsf(o.w) > 100.f) {
                const float renorm = __fdiv_rn(100.f, fabsf(o.w));
                if (renorm < 1.f) { o.x *= renorm; o.y *= renorm; o.z *= renorm; o.w *= renorm; }
            }
            const int zl = ic - B.zst_lo;
            const size_t row = ((size_t)zl * B.nys + yl) * B.nxs;
            const int il = xl > 0 ? xl - 1 : B.nxs - 1;
            if (LAYOUT == 2) {
                out[2 * (row + xl)] = o;
                out[2 * (row + il) + 1] = o;
            } else if (LAYOUT == 4) {
                const int nzs = B.zst_hi - B.zst_lo;
                const size_t rowb = ((size_t)(zl > 0 ? zl - 1 : nzs - 1) * B.nys + yl) * B.nxs;
                out[4 * (row + xl) + 0] = o;
                out[4 * (row + il) + 1] = o;
                out[4 * (rowb + xl) + 2] = o;
                out[4 * (rowb + il) + 3] = o;
            } else {
                out[row + xl] = o;
            }
        }
    }
}

template <int KIND, bool ON, int NOFF>
__global__ void __launch_bounds__(GB_TX * GB_TY)
grid_build_kernel(int na, const float4* __restrict__ atoms, const float* __restrict__ params, int pstride,
                  float4* __restrict__ grid, GridGeom G, TipSites S) {
    const StoreBox B = {0, G.nx, 0, G.ny, 0, G.nz};
    build_tile<KIND, ON, NOFF, GB_ZB>(na, atoms, params, pstride, grid, G, S, B, blockIdx.x * GB_TX + threadIdx.x,
                                      blockIdx.y * GB_TY + threadIdx.y, blockIdx.z * GB_ZB);
}

template <int KIND, bool ON>
int launch_noff(int noff, dim3 grd, dim3 block, cudaStream_t st, int na, const float4* atoms, const float* params,
                int pstride, float4* out, const GridGeom& G, const TipSites& S) {
    switch (noff) {
        case 0: grid_build_kernel<KIND, ON, 0><<<grd, block, 0, st>>>(na, atoms, params, pstride, out, G, S); break;
        case 1: grid_build_kernel<KIND, ON, 1><<<grd, block, 0, st>>>(na, atoms, params, pstride, out, G, S); break;
        case 2: grid_build_kernel<KIND, ON, 2><<<grd, block, 0, st>>>(na, atoms, params, pstride, out, G, S); break;
        case 3: grid_build_kernel<KIND, ON, 3><<<grd, block, 0, st>>>(na, atoms, params, pstride, out, G, S); break;
        default: grid_build_kernel<KIND, ON, 4><<<grd, block, 0, st>>>(na, atoms, params, pstride, out, G, S); break;
    }
    return check_launch("spm_grid_build");
}

template <int KIND>
int launch_kind(bool on, int noff, dim3 grd, dim3 block, cudaStream_t st, int na, const float4* atoms,
                const float* params, int pstride, float4* out, const GridGeom& G, const TipSites& S) {
    if (on) return launch_noff<KIND, true>(noff, grd, block, st, na, atoms, params, pstride, out, G, S);
    return launch_noff<KIND, false>(noff, grd, block, st, na, atoms, params, pstride, out, G, S);
}

// Tip-charge sites: zero-offset charges merged into the on-node term.
TipSites make_sites(const float* Qs, const float* QZs, bool& on, int& noff) {
    TipSites S = {};
    noff = 0;
    on = false;
    for (int k = 0; k < 4; k++) {
        if (Qs[k] == 0.f) continue;  // a zero-charge site only adds zeros
        if (QZs[k] == 0.f) {
            S.qs_on += Qs[k] * COULOMB_CONST;
            on = true;
        } else {
            S.qs[noff] = Qs[k] * COULOMB_CONST;
            S.qz[noff] = QZs[k];
            noff++;
        }
    }
    return S;
}

// ---- batched slabs ----------------------------------------------------------
// One CTA per tile of the batch: 32*TY consecutive (x fastest) of the slab's
// nx_slab*ny_slab columns, ZB layers; tiles of a molecule are numbered columns
// first, then z, over ceil(nx_slab*ny_slab / (32*TY)) x ceil(nz_slab/ZB).
// (Column tiles need not fit the slab's rows: a 32 x TY box of rows would
// leave a quarter of the node-atom pairs idle on the batch distribution.)
template <int KIND, bool ON, int NOFF, int ZB, int LAYOUT>
__global__ void __launch_bounds__(256)
batch_grid_build_kernel(int n_mol, const spm_batch_mol* __restrict__ mols, const float4* __restrict__ atoms,
                        const float* __restrict__ params, int pstride, float4* __restrict__ grid, TipSites S) {
    const long long tile = blockIdx.x;
    const spm_batch_mol* D = mols + SPM_MOL_BY(tile_off, mols, n_mol, tile);
    const int ty = blockDim.y;
    const int z_lo = D->z_lo, nzs = D->nz_slab;
    const StoreBox B = {D->x_lo, D->nx_slab, D->y_lo, D->ny_slab, z_lo, z_lo + nzs};
    const long long lt = tile - D->tile_off;
    const long long ncol = (long long)B.nxs * B.nys;
    const int cpt = GB_TX * ty;  // columns per tile
    const long long ntc = (ncol + cpt - 1) / cpt;
    const long long bc = lt % ntc, bz = lt / ntc;
    if (bz * ZB >= nzs) return;  // whole CTA: outside the slab (prefix of another shape)
    const long long col = bc * cpt + threadIdx.y * GB_TX + threadIdx.x;
    // a column past the slab's last gets a row outside the box: computed by nobody, stored nowhere
    const int yl = col < ncol ? (int)(col / B.nxs) : B.nys, xl = col < ncol ? (int)(col - (long long)yl * B.nxs) : 0;
    GridGeom G;
    G.nx = D->nx; G.ny = D->ny; G.nz = D->nz;
    G.p0 = ld4f(D->p0);
    G.dA = ld4f(D->dA);
    G.dB = ld4f(D->dB);
    G.dC = ld4f(D->dC);
    const int ao = D->atom_off;
    build_tile<KIND, ON, NOFF, ZB, LAYOUT>(D->n_atoms, atoms + ao, params + (size_t)ao * pstride, pstride,
                                           grid + LAYOUT * D->grid_off, G, S, B, B.x_lo + xl, B.y_lo + yl,
                                           z_lo + (int)bz * ZB);
}

struct BatchLaunch {
    unsigned blocks;
    dim3 block;
    cudaStream_t st;
    int n_mol;
    const spm_batch_mol* mols;
    const float4* atoms;
    const float* params;
    int pstride;
    float4* grid;
    int layout;  // float4 per node: 2 (x-pairs) or 4 (xz-quads)
};

template <int KIND, bool ON, int NOFF, int LAYOUT>
void launch_batch_zl(int zb, const BatchLaunch& L, const TipSites& S) {
    if (zb == 16)
        batch_grid_build_kernel<KIND, ON, NOFF, 16, LAYOUT><<<L.blocks, L.block, 0, L.st>>>(
            L.n_mol, L.mols, L.atoms, L.params, L.pstride, L.grid, S);
    else
        batch_grid_build_kernel<KIND, ON, NOFF, 8, LAYOUT><<<L.blocks, L.block, 0, L.st>>>(
            L.n_mol, L.mols, L.atoms, L.params, L.pstride, L.grid, S);
}

template <int KIND, bool ON, int NOFF>
void launch_batch_zb(int zb, const BatchLaunch& L, const TipSites& S) {
    if (L.layout == 4) launch_batch_zl<KIND, ON, NOFF, 4>(zb, L, S);
    else launch_batch_zl<KIND, ON, NOFF, 2>(zb, L, S);
}

template <int KIND, bool ON>
void launch_batch_noff(int noff, int zb, const BatchLaunch& L, const TipSites& S) {
    switch (noff) {
        case 0: launch_batch_zb<KIND, ON, 0>(zb, L, S); break;
        case 1: launch_batch_zb<KIND, ON, 1>(zb, L, S); break;
        case 2: launch_batch_zb<KIND, ON, 2>(zb, L, S); break;
        case 3: launch_batch_zb<KIND, ON, 3>(zb, L, S); break;
        default: launch_batch_zb<KIND, ON, 4>(zb, L, S); break;
    }
}

template <int KIND>
void launch_batch_kind(bool on, int noff, int zb, const BatchLaunch& L, const TipSites& S) {
    if (on) launch_batch_noff<KIND, true>(noff, zb, L, S);
    else launch_batch_noff<KIND, false>(noff, zb, L, S);
}

}  // namespace
}  // namespace spm

extern "C" int spm_batch_grid_build(int kind, int n_mol, const spm_batch_mol* mols, long long n_tiles,
                                    const spm_batch_shape* shape, const float* atoms, const float* params,
                                    const float* Qs, const float* QZs, float* grid, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(kind == SPM_KIND_LJ || kind == SPM_KIND_MORSE, "spm_batch_grid_build: kind=%d", kind);
    SPM_REQUIRE(shape && Qs && QZs, "spm_batch_grid_build: null shape or host vector");
    SPM_REQUIRE(n_mol >= 0 && n_tiles >= 0, "spm_batch_grid_build: negative sizes");
    if (n_mol == 0 || n_tiles == 0) return SPM_OK;
    SPM_REQUIRE(mols && grid && atoms && params, "spm_batch_grid_build: null device pointer");
    SPM_REQUIRE(aligned16(grid) && aligned16(atoms) && (reinterpret_cast<uintptr_t>(mols) & 7u) == 0,
                "spm_batch_grid_build: misaligned buffers");
    SPM_REQUIRE(shape->gb_ty == 2 || shape->gb_ty == 4 || shape->gb_ty == 8, "spm_batch_grid_build: gb_ty=%d",
                shape->gb_ty);
    SPM_REQUIRE(shape->gb_zb == 8 || shape->gb_zb == 16, "spm_batch_grid_build: gb_zb=%d", shape->gb_zb);
    SPM_REQUIRE(shape->grid_layout == 0 || shape->grid_layout == 1, "spm_batch_grid_build: grid_layout=%d",
                shape->grid_layout);
    SPM_REQUIRE(n_tiles <= 0x7fffffffLL, "spm_batch_grid_build: %lld tiles exceed one launch", n_tiles);
    int noff = 0;
    bool on = false;
    const TipSites S = make_sites(Qs, QZs, on, noff);
    BatchLaunch L;
    L.blocks = (unsigned)n_tiles;
    L.block = dim3(GB_TX, shape->gb_ty, 1);
    L.st = as_stream(stream);
    L.n_mol = n_mol;
    L.mols = mols;
    L.atoms = reinterpret_cast<const float4*>(atoms);
    L.params = params;
    L.pstride = (kind == SPM_KIND_MORSE) ? 4 : 2;
    L.grid = reinterpret_cast<float4*>(grid);
    L.layout = shape->grid_layout ? 4 : 2;
    if (kind == SPM_KIND_MORSE) launch_batch_kind<SPM_KIND_MORSE>(on, noff, shape->gb_zb, L, S);
    else launch_batch_kind<SPM_KIND_LJ>(on, noff, shape->gb_zb, L, S);
    return check_launch("spm_batch_grid_build");
}

extern "C" int spm_grid_build(int kind, int n_atoms, const float* atoms, const float* params, float* grid,
                              int nx, int ny, int nz, const float* p0, const float* dA, const float* dB,
                              const float* dC, const float* Qs, const float* QZs, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(kind == SPM_KIND_LJ || kind == SPM_KIND_MORSE, "spm_grid_build: kind=%d is not LJ(0)/Morse(1)", kind);
    SPM_REQUIRE(n_atoms >= 0, "spm_grid_build: n_atoms=%d < 0", n_atoms);
    SPM_REQUIRE(nx > 0 && ny > 0 && nz > 0, "spm_grid_build: grid dims (%d,%d,%d) must be positive", nx, ny, nz);
    SPM_REQUIRE(grid && p0 && dA && dB && dC && Qs && QZs, "spm_grid_build: null grid or host vector");
    SPM_REQUIRE(n_atoms == 0 || (atoms && params), "spm_grid_build: null atoms/params with n_atoms=%d", n_atoms);
    SPM_REQUIRE(aligned16(grid) && (n_atoms == 0 || aligned16(atoms)), "spm_grid_build: grid/atoms not 16-byte aligned");
    long long nab = 0, total = 0;
    SPM_REQUIRE(mul_ok(nx, ny, &nab) && mul_ok(nab, nz, &total), "spm_grid_build: node count overflows");
    if (dC[0] != 0.f || dC[1] != 0.f)
        return set_error(SPM_ERR_UNSUPPORTED, "spm_grid_build: dC=(%g,%g,%g) must be (0,0,dz)", dC[0], dC[1], dC[2]);
    if ((long long)ny > 65535LL * GB_TY || ((long long)nz + GB_ZB - 1) / GB_ZB > 65535LL)
        return set_error(SPM_ERR_UNSUPPORTED, "spm_grid_build: ny=%d or nz=%d exceeds the launch limits", ny, nz);
    GridGeom G;
    G.nx = nx; G.ny = ny; G.nz = nz;
    G.p0 = make_float4(p0[0], p0[1], p0[2], p0[3]);
    G.dA = make_float4(dA[0], dA[1], dA[2], dA[3]);
    G.dB = make_float4(dB[0], dB[1], dB[2], dB[3]);
    G.dC = make_float4(dC[0], dC[1], dC[2], dC[3]);
    int noff = 0;
    bool on = false;
    const TipSites S = make_sites(Qs, QZs, on, noff);
    dim3 block(GB_TX, GB_TY, 1);
    dim3 grd((nx + GB_TX - 1) / GB_TX, (ny + GB_TY - 1) / GB_TY, (nz + GB_ZB - 1) / GB_ZB);
    const int pstride = (kind == SPM_KIND_MORSE) ? 4 : 2;
    cudaStream_t st = as_stream(stream);
    const float4* a4 = reinterpret_cast<const float4*>(atoms);
    float4* g4 = reinterpret_cast<float4*>(grid);
    if (kind == SPM_KIND_MORSE) return launch_kind<SPM_KIND_MORSE>(on, noff, grd, block, st, n_atoms, a4, params, pstride, g4, G, S);
    return launch_kind<SPM_KIND_LJ>(on, noff, grd, block, st, n_atoms, a4, params, pstride, g4, G, S);
}

// ---- the uncapped pair sums at arbitrary points ----------------------------
// Replaces cs_brute_afm_morse_c_points (kernels/contact_surface.cl:1341-1390,
// called by AFMulator._brute_afm_morse_c_queries, spammm/SPM/AFM.py:1051-1067):
// per query point the LJ or Morse law plus the Coulomb law at the four
// tip-charge sites (point + zhat*QZs[k], weighted by Qs[k]*COULOMB_CONST) summed
// over all atoms, with no |E| > 100 cap.  One thread per point, atoms staged in
// shared memory; FP32 with IEEE division, sqrt and exp.
namespace spm {
namespace {
constexpr int PQ_THREADS = 128;

template <int KIND>
__global__ void __launch_bounds__(PQ_THREADS)
pair_points_kernel(int na, const float4* __restrict__ atoms, const float* __restrict__ params, int pstride,
                   const float* __restrict__ q, int nq, float4 qs, float4 qz, float4* __restrict__ out) {
    __shared__ float4 s_a[PQ_THREADS];
    __shared__ float4 s_p[PQ_THREADS];
    const int iq = blockIdx.x * PQ_THREADS + threadIdx.x;
    const bool act = iq < nq;
    const float px = act ? q[3 * (size_t)iq] : 0.f, py = act ? q[3 * (size_t)iq + 1] : 0.f,
                pz = act ? q[3 * (size_t)iq + 2] : 0.f;
    const float sq[4] = {qs.x, qs.y, qs.z, qs.w}, sz[4] = {qz.x, qz.y, qz.z, qz.w};
    float fx = 0.f, fy = 0.f, fz = 0.f, fe = 0.f;
    for (int t0 = 0; t0 < na; t0 += PQ_THREADS) {
        const int j = t0 + threadIdx.x;
        if (j < na) {
            s_a[threadIdx.x] = __ldg(atoms + j);
            const float* pr = params + (size_t)j * pstride;
            s_p[threadIdx.x] = make_float4(__ldg(pr), __ldg(pr + 1), KIND == SPM_KIND_MORSE ? __ldg(pr + 2) : 0.f, 0.f);
        }
        __syncthreads();
        const int nt = min(PQ_THREADS, na - t0);
        for (int jj = 0; jj < nt; jj++) {
            const float4 a = s_a[jj];
            const float4 c = s_p[jj];
            const float dx = px - a.x, dy = py - a.y, dz = pz - a.z;
            const float r2 = dx * dx + dy * dy + dz * dz + R2SAFE;
            float s;
            if (KIND == SPM_KIND_MORSE) {  // getMorse: E0 e (e - 2), F = dp * (-2 K E0 e (e-1)) / r
                const float r = sqrtf(r2);
                const float e = expf(c.z * (r - c.x));
                fe += c.y * e * (e - 2.f);
                s = __fdiv_rn(-c.y * e * (e - 1.f) * 2.f * c.z, r);
            } else {  // getLJ: (c12 ir6 - c6) ir6, F = dp * (12 c12 ir6 - 6 c6) ir6 ir2
                const float ir2 = __fdiv_rn(1.f, r2);
                const float ir6 = ir2 * ir2 * ir2;
                fe += (c.y * ir6 - c.x) * ir6;
                s = (12.f * c.y * ir6 - 6.f * c.x) * ir6 * ir2;
            }
            fx += dx * s;
            fy += dy * s;
            fz += dz * s;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (sq[k] == 0.f) continue;
                const float dzk = dz + sz[k];
                const float ir2 = __fdiv_rn(1.f, dx * dx + dy * dy + dzk * dzk + R2SAFE);
                const float E = a.w * sqrtf(ir2) * sq[k];
                fe += E;
                const float sk = E * ir2;
                fx += dx * sk;
                fy += dy * sk;
                fz += dzk * sk;
            }
        }
        __syncthreads();
    }
    if (act) out[iq] = make_float4(fx, fy, fz, fe);
}
}  // namespace
}  // namespace spm

extern "C" int spm_pair_fe_points(int kind, int n_atoms, const float* atoms, const float* params, const float* queries,
                                  int n_q, const float* Qs, const float* QZs, float* out, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(kind == SPM_KIND_LJ || kind == SPM_KIND_MORSE, "spm_pair_fe_points: kind=%d", kind);
    SPM_REQUIRE(n_atoms >= 0 && n_q >= 0, "spm_pair_fe_points: negative sizes");
    SPM_REQUIRE(Qs && QZs, "spm_pair_fe_points: null host vectors");
    if (n_q == 0) return SPM_OK;
    SPM_REQUIRE(queries && out && (n_atoms == 0 || (atoms && params)), "spm_pair_fe_points: null device pointer");
    SPM_REQUIRE(aligned16(out) && (n_atoms == 0 || aligned16(atoms)), "spm_pair_fe_points: out/atoms not aligned");
    const float4 qs = make_float4(Qs[0] * COULOMB_CONST, Qs[1] * COULOMB_CONST, Qs[2] * COULOMB_CONST,
                                  Qs[3] * COULOMB_CONST);
    const float4 qz = make_float4(QZs[0], QZs[1], QZs[2], QZs[3]);
    const unsigned nb = (unsigned)((n_q + PQ_THREADS - 1) / PQ_THREADS);
    cudaStream_t st = as_stream(stream);
    const float4* a4 = reinterpret_cast<const float4*>(atoms);
    float4* o4 = reinterpret_cast<float4*>(out);
    if (kind == SPM_KIND_MORSE)
        pair_points_kernel<SPM_KIND_MORSE><<<nb, PQ_THREADS, 0, st>>>(n_atoms, a4, params, 4, queries, n_q, qs, qz, o4);
    else
        pair_points_kernel<SPM_KIND_LJ><<<nb, PQ_THREADS, 0, st>>>(n_atoms, a4, params, 2, queries, n_q, qs, qz, o4);
    return check_launch("spm_pair_fe_points");
}
