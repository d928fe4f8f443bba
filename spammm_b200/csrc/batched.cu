// batched.cu -- host-side planning of a batch of molecules.
//
// spm_batch_prepare validates a descriptor array and numbers the work items of
// every batched stage across the batch for one launch shape:
//   tile_off   grid-build CTA tiles  ceil(nx_slab*ny_slab / (32*gb_ty)) x ceil(nz_slab/gb_zb)
//   slot_off   relaxation slots      raster: 32 per (32/h) x h pixel tile, else one per pixel
//                                    rounded up to 32 (a warp's 32 slots never span molecules)
//   unit_off   adjoint node units    ceil(slab nodes/adj_chunk) (0 without states)
//   chunk_off  loss chunks           ceil(states/256)
//   row_off    adjoint partial rows  units x n_atoms
// The kernels find the molecule of a work item by binary search over these
// prefixes, so one launch per stage covers any mix of molecule sizes.
#include "spm_internal.cuh"
#include <cmath>

extern "C" spm_batch_shape spm_batch_default_shape(void) {
    spm_batch_shape s;
    s.gb_ty = 4;
    s.gb_zb = 8;
    s.rx_threads = 128;
    s.rx_tile_h = 8;
    s.rx_ctas_per_sm = 0;
    s.adj_chunk = 16384;
    s.rx_regs = 4;
    s.grid_layout = 0;
    s.rx_sync = 2;  // as 1 unless the call is warm and polished
    s.adj_ilp = 1;
    s.adj_agg = 2;  // the tile walk with neighbour merges: 14.1 -> 11.8 ms on the 64-molecule fit's adjoint
    s.adj_stage = 0;
    return s;
}

extern "C" int spm_batch_prepare(spm_batch_mol* mols, int n_mol, const spm_batch_shape* shape, long long* totals_out) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(shape && totals_out, "spm_batch_prepare: null shape/totals");
    SPM_REQUIRE(n_mol >= 0, "spm_batch_prepare: n_mol=%d < 0", n_mol);
    SPM_REQUIRE(n_mol == 0 || mols, "spm_batch_prepare: null descriptors");
    const spm_batch_shape& S = *shape;
    SPM_REQUIRE(S.gb_ty == 2 || S.gb_ty == 4 || S.gb_ty == 8, "spm_batch_prepare: gb_ty=%d", S.gb_ty);
    SPM_REQUIRE(S.gb_zb == 8 || S.gb_zb == 16, "spm_batch_prepare: gb_zb=%d", S.gb_zb);
    SPM_REQUIRE(S.rx_threads == 64 || S.rx_threads == 128 || S.rx_threads == 256, "spm_batch_prepare: rx_threads=%d",
                S.rx_threads);
    SPM_REQUIRE(S.rx_tile_h >= 1 && S.rx_tile_h <= 32 && (S.rx_tile_h & (S.rx_tile_h - 1)) == 0,
                "spm_batch_prepare: rx_tile_h=%d", S.rx_tile_h);
    SPM_REQUIRE(S.rx_ctas_per_sm >= 0, "spm_batch_prepare: rx_ctas_per_sm=%d", S.rx_ctas_per_sm);
    SPM_REQUIRE(S.adj_chunk >= 1024 && S.adj_chunk <= (1 << 20) && S.adj_chunk % 1024 == 0,
                "spm_batch_prepare: adj_chunk=%d", S.adj_chunk);
    SPM_REQUIRE(S.rx_regs >= 0 && S.rx_regs <= 5, "spm_batch_prepare: rx_regs=%d", S.rx_regs);
    SPM_REQUIRE(S.grid_layout == 0 || S.grid_layout == 1, "spm_batch_prepare: grid_layout=%d", S.grid_layout);
    SPM_REQUIRE(S.rx_sync >= 0 && S.rx_sync <= 2, "spm_batch_prepare: rx_sync=%d", S.rx_sync);
    SPM_REQUIRE(S.adj_ilp >= 1 && S.adj_ilp <= 3, "spm_batch_prepare: adj_ilp=%d", S.adj_ilp);
    SPM_REQUIRE(S.adj_agg >= 0 && S.adj_agg <= 2, "spm_batch_prepare: adj_agg=%d", S.adj_agg);
    SPM_REQUIRE(S.adj_stage == 0 || (S.adj_stage == 1 && S.adj_ilp == 1), "spm_batch_prepare: adj_stage=%d",
                S.adj_stage);
    const long long th = S.rx_tile_h, tw = 32 / S.rx_tile_h;
    long long tiles = 0, slots = 0, units = 0, chunks = 0, states = 0, atoms = 0, pixels = 0, grid_end = 0, rows = 0;
    for (int m = 0; m < n_mol; m++) {
        spm_batch_mol& D = mols[m];
        SPM_REQUIRE(D.n_atoms >= 0 && D.n_scan >= 0 && D.nz_steps >= 0, "spm_batch_prepare: molecule %d: negative counts",
                    m);
        SPM_REQUIRE(D.atom_off == atoms && D.pix_off == pixels && D.state_off == states,
                    "spm_batch_prepare: molecule %d: atom/pixel/state rows must follow the previous molecule's "
                    "(atom_off=%d pix_off=%d state_off=%lld, expected %lld %lld %lld)",
                    m, D.atom_off, D.pix_off, D.state_off, atoms, pixels, states);
        SPM_REQUIRE(D.nx > 0 && D.ny > 0 && D.nz > 0, "spm_batch_prepare: molecule %d: grid (%d,%d,%d)", m, D.nx, D.ny,
                    D.nz);
        SPM_REQUIRE(D.z_lo >= 0 && D.nz_slab >= 1 && (long long)D.z_lo + D.nz_slab <= D.nz,
                    "spm_batch_prepare: molecule %d: slab [%d,%d) outside [0,%d)", m, D.z_lo, D.z_lo + D.nz_slab, D.nz);
        SPM_REQUIRE(D.x_lo >= 0 && D.nx_slab >= 1 && (long long)D.x_lo + D.nx_slab <= D.nx && D.y_lo >= 0 &&
                    D.ny_slab >= 1 && (long long)D.y_lo + D.ny_slab <= D.ny,
                    "spm_batch_prepare: molecule %d: slab columns [%d,%d) / rows [%d,%d) outside the (%d,%d) grid", m,
                    D.x_lo, D.x_lo + D.nx_slab, D.y_lo, D.y_lo + D.ny_slab, D.nx, D.ny);
        const long long slab = (long long)D.nx_slab * D.ny_slab * D.nz_slab;
        SPM_REQUIRE(slab < (1LL << 32), "spm_batch_prepare: molecule %d: slab of %lld nodes >= 2^32", m, slab);
        SPM_REQUIRE(D.grid_off >= grid_end, "spm_batch_prepare: molecule %d: grid_off=%lld overlaps the previous slab "
                    "(ends at %lld)", m, D.grid_off, grid_end);
        SPM_REQUIRE(D.dC[0] == 0.f && D.dC[1] == 0.f, "spm_batch_prepare: molecule %d: dC must be (0,0,dz)", m);
        SPM_REQUIRE(D.dinvA[1] == 0.f && D.dinvA[2] == 0.f && D.dinvB[0] == 0.f && D.dinvB[2] == 0.f &&
                    D.dinvC[0] == 0.f && D.dinvC[1] == 0.f,
                    "spm_batch_prepare: molecule %d: the sampling transform must be axis-aligned", m);
        SPM_REQUIRE(D.raster_ny >= 0, "spm_batch_prepare: molecule %d: raster_ny=%d", m, D.raster_ny);
        if (D.raster_ny > 0 && D.n_scan % D.raster_ny != 0) D.raster_ny = 0;  // not a full raster: 1D order
        const long long nst = (long long)D.n_scan * D.nz_steps;
        D.tile_off = tiles;
        D.slot_off = slots;
        D.unit_off = units;
        D.chunk_off = chunks;
        D.row_off = rows;
        tiles += (((long long)D.nx_slab * D.ny_slab + 32LL * S.gb_ty - 1) / (32LL * S.gb_ty)) *
                 ((D.nz_slab + S.gb_zb - 1LL) / S.gb_zb);
        if (nst > 0) {
            if (D.raster_ny > 0) {
                const long long nxr = D.n_scan / D.raster_ny;
                slots += ((nxr + tw - 1) / tw) * ((D.raster_ny + th - 1) / th) * 32;
            } else {
                slots += (D.n_scan + 31LL) / 32 * 32;
            }
            const long long u = (slab + S.adj_chunk - 1) / S.adj_chunk;
            units += u;
            rows += u * D.n_atoms;
            chunks += (nst + 255) / 256;
        }
        states += nst;
        atoms += D.n_atoms;
        pixels += D.n_scan;
        grid_end = D.grid_off + slab;
        SPM_REQUIRE(atoms < (1LL << 30) && pixels < (1LL << 31), "spm_batch_prepare: batch too large");
    }
    SPM_REQUIRE(tiles < (1LL << 31) && slots < (1LL << 31) && units < (1LL << 31) && chunks < (1LL << 31) &&
                rows < (1LL << 40), "spm_batch_prepare: batch too large for one launch per stage");
    totals_out[0] = tiles;
    totals_out[1] = slots;
    totals_out[2] = units;
    totals_out[3] = chunks;
    totals_out[4] = states;
    totals_out[5] = atoms;
    totals_out[6] = pixels;
    totals_out[7] = grid_end;
    totals_out[8] = rows;
    return SPM_OK;
}

// ---- fitting update -----------------------------------------------------------
namespace spm {
namespace {
constexpr int ADAM_THREADS = 1024;

// One Adam step over every (atom, column) of the column mask, in FP32.  A single CTA strides over
// the atoms (a fit's batch holds thousands of atoms: one launch of a few microseconds), reads the
// step count before the barrier and writes the incremented count after it, so every thread uses
// the same step and the count stays on the device for graph replays.
__global__ void __launch_bounds__(ADAM_THREADS)
batch_adam_kernel(long long n_atoms, const double* __restrict__ grad, float4* __restrict__ atoms,
                  float4* __restrict__ m, float4* __restrict__ v, float* __restrict__ t, double lr_, double b1_,
                  double b2_, double eps_, int cols) {
    const float t1 = *t + 1.f;
    // the coefficients in FP64, then rounded once: 1 - b in FP32 would lose 1e-5 of (1 - 0.999)
    const float b1 = (float)b1_, b2 = (float)b2_, c1 = (float)(1.0 - b1_), c2 = (float)(1.0 - b2_);
    const float bc1 = (float)(1.0 - pow(b1_, (double)t1)), bc2 = (float)(1.0 - pow(b2_, (double)t1));
    const float lr = (float)lr_, eps = (float)eps_;
    for (long long i = threadIdx.x; i < n_atoms; i += ADAM_THREADS) {
        float4 a = atoms[i], mi = m[i], vi = v[i];
        const double* gr = grad + 6 * i;
        float* ac = &a.x;
        float* mc = &mi.x;
        float* vc = &vi.x;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (!((cols >> c) & 1)) continue;
            const float g = (float)gr[c < 3 ? c : 5];  // x, y, z, then the charge column
            mc[c] = mc[c] * b1 + c1 * g;
            vc[c] = vc[c] * b2 + c2 * (g * g);
            ac[c] -= lr * ((mc[c] / bc1) / (sqrtf(vc[c] / bc2) + eps));
        }
        atoms[i] = a;
        m[i] = mi;
        v[i] = vi;
    }
    __syncthreads();
    if (threadIdx.x == 0) *t = t1;
}
}  // namespace
}  // namespace spm

extern "C" int spm_batch_adam_step(long long n_atoms, const double* grad, float* atoms, float* m, float* v, float* t,
                                   double lr, double beta1, double beta2, double eps, int cols, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(n_atoms >= 0, "spm_batch_adam_step: n_atoms=%lld", n_atoms);
    SPM_REQUIRE(grad && atoms && m && v && t, "spm_batch_adam_step: null pointer");
    SPM_REQUIRE(aligned16(atoms) && aligned16(m) && aligned16(v), "spm_batch_adam_step: buffers not 16-byte aligned");
    SPM_REQUIRE(std::isfinite(lr) && beta1 >= 0.0 && beta1 < 1.0 && beta2 >= 0.0 && beta2 < 1.0 && eps > 0.0,
                "spm_batch_adam_step: lr=%g beta1=%g beta2=%g eps=%g", lr, beta1, beta2, eps);
    SPM_REQUIRE((cols & ~15) == 0, "spm_batch_adam_step: cols=%d (bits 0-3: x, y, z, charge)", cols);
    batch_adam_kernel<<<1, ADAM_THREADS, 0, as_stream(stream)>>>(n_atoms, grad, reinterpret_cast<float4*>(atoms),
                                                                 reinterpret_cast<float4*>(m),
                                                                 reinterpret_cast<float4*>(v), t, lr, beta1, beta2,
                                                                 eps, cols);
    return check_launch("spm_batch_adam_step");
}
