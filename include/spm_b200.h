/*
 * spm_b200.h -- C ABI of libspmb200.so, the sm_100a implementation of
 * SPAMMM's probe-particle AFM hot path:
 *   (a) force-grid build, (b) FIRE probe relaxation down z-strokes,
 *   (c) Fz -> df conversion, plus the grid-free direct Morse path and its
 *   implicit-function adjoint.
 *
 * Conventions (identical to the reference's OpenCL buffers/images):
 *   - every pointer argument is a DEVICE pointer unless the comment says
 *     "host"; float4 arrays are (n,4) float32 rows, C order;
 *   - the force grid is (nz,ny,nx,4) float32, x fastest, channels
 *     (Fx,Fy,Fz,E): the layout of the reference's RGBA float image3d_t;
 *   - scan points are (n_scan,4) float32 rows (x,y,z,0), raster ix-major
 *     (spammm/SPM/AFM.py:82-95); per-state outputs are (n_scan,nz,4), iz=0 at
 *     the first (highest) tip position unless SPM_FLAG_FLIP_Z is set;
 *   - `stream` is a cudaStream_t (NULL = legacy default stream); every call
 *     is asynchronous on that stream and allocates no device memory unless a
 *     comment says otherwise;
 *   - every function returns SPM_OK (0) or an SPM_ERR_* code and leaves a
 *     message for spm_last_error() (thread-local).
 */
#ifndef SPM_B200_H
#define SPM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define SPM_ABI_VERSION 4

enum spm_status {
    SPM_OK = 0,
    SPM_ERR_ARG = 1,          /* null pointer, non-positive size, size overflow, bad flag */
    SPM_ERR_CUDA = 2,         /* CUDA launch or runtime error (text in spm_last_error) */
    SPM_ERR_UNSUPPORTED = 3,  /* input outside a kernel's stated limits (e.g. atom count) */
    SPM_ERR_TIMEOUT = 4       /* a bounded device-side wait gave up */
};

/* Potential kinds for the grid build / pair law. */
#define SPM_KIND_LJ    0      /* params (na,2) = (c6, c12)          AFM.cl:738-745 */
#define SPM_KIND_MORSE 1      /* params (na,4) = (R0, E0, K<0, 0)    AFM.cl:747-757 */

/* Element type of (n,4) FE volumes accepted by the df functions. */
#define SPM_F32 0
#define SPM_F64 1

/* spm_scan_params.flags */
#define SPM_FLAG_FIRE   1     /* FIRE integrator (OPT_FIRE=1); else plain damping (OPT_FIRE=0) */
#define SPM_FLAG_FLIP_Z 2     /* store iz reversed: the z flip AFMulator.scan_fdbm applies (AFM.py:627-633) */
#define SPM_FLAG_PAIRED 4     /* relaxStrokes only: the first n_scan/2 points start forward strokes, the
                                 rest backward strokes, which step by -dTip and store iz in the order
                                 opposite to the forward ones (SPM_FLAG_FLIP_Z inverted): the forward
                                 and reverse=True scans of AFMulator.scan_fdbm (AFM.py:584-633) in one
                                 launch; n_scan even */
#define SPM_FLAG_WARM   16    /* spm_batch_relax only, with rx_sync = 1 or 2: PPs is read as well as written;
                                 a z-step starts from the state's equilibrium in PPs (the previous
                                 call's) when that converged and the stroke arrives at the z-step
                                 where it did in the previous call (its continuation start within
                                 0.1 A per axis of the previous call's equilibrium of the z-step
                                 before, shifted by the z-step), else from the continuation as
                                 without the flag (the probe jumped on the way, or no previous
                                 equilibrium).  For fits whose atoms move a little per call.
                                 With SPM_FLAG_POLISH a warm-started z-step first takes the polish's
                                 Newton steps from the previous equilibrium and runs FIRE only if they
                                 do not reach |F|^2 < f2conv (PPs.w then counts the Newton
                                 evaluations); both starts reach the same equilibrium */
#define SPM_FLAG_POLISH 8     /* relaxations (not SPM_RELAX_2D): after FIRE stops, up to 4 Newton steps
                                 q <- q - J^-1 G on the total force G(q) of the interpolated grid and the
                                 spring (J = dG/dq, exact for the trilinear interpolant), each kept only
                                 if it moves q by at most 0.1 A per axis and lowers |G|; outputs (FE,
                                 disp / PP) are then taken at the polished position, the sample there.
                                 The FIRE trajectory is unchanged (the next z-step starts from the
                                 unpolished position).  Not in the reference: it removes FIRE's stopping
                                 slack (~|F|/k_xy) from the equilibria */

/* Scan/tip parameters shared by the relaxation and sampling kernels.  Field
 * names follow the reference's kernel arguments (kernels/AFM.cl:345-562). */
typedef struct spm_scan_params {
    float dinvA[4], dinvB[4], dinvC[4];  /* world -> normalized grid coordinate (.w = -o/L + 0.5/n) */
    float tipA[4], tipB[4], tipC[4];     /* tip frame rows; tipC[3] = dtip for the tilted kernels */
    float dTip[4];                       /* per-z tip step for relaxStrokes / raw sampling */
    float stiffness[4];                  /* (kx,ky,kz,k_radial) eV/A^2, negative = restoring */
    float dpos0[4];                      /* probe rest offset (xyz) and radial bond length (w) */
    float relax_params[4];               /* (dt, damp, -, -) */
    float surfFF[4];                     /* surface bias along tipC (x) */
    int   nz;                            /* z-steps per stroke */
    int   max_iter;                      /* integrator steps per z-step (reference: N_RELAX_STEP_MAX=128) */
    float f2conv;                        /* |F|^2 convergence threshold (reference: F2CONV=1e-8) */
    int   flags;                         /* SPM_FLAG_* */
    int   raster_ny;                     /* >0: points form an ix-major (n_scan/raster_ny, raster_ny)
                                            raster; lets the kernels give each warp a compact
                                            4x8 pixel block (results do not depend on it) */
} spm_scan_params;

/* Library/ABI identification. */
int spm_abi_version(void);
/* Last error message of the calling thread ("" if none). */
const char* spm_last_error(void);

/* ------------------------------------------------------------------------
 * (a) Force-grid build.
 * Replaces AFMulator.make_forcefield (spammm/SPM/AFM.py:897-946) ->
 * evalLJC_QZs_toImg (kernels/AFM.cl:916-991) / evalMorseC_QZs_toImg
 * (kernels/AFM.cl:996-1056).  Node (ia,ib,ic) sits at p0 + dA*ia + dB*ib +
 * dC*ic; value = sum over atoms of the LJ or Morse pair law plus the Coulomb
 * law at the four tip-charge sites node + zhat*QZs[k] weighted by
 * Qs[k]*14.3996448915; nodes with |E| > 100 are rescaled by 100/|E|.
 *   atoms  (n_atoms,4) = (x,y,z,Q);  params per SPM_KIND_*;
 *   p0,dA,dB,dC,Qs,QZs: HOST float[4];  grid out (nz,ny,nx,4).
 * Requires dC = (0,0,dz) (true for every reference grid constructor). */
int spm_grid_build(int kind, int n_atoms, const float* atoms, const float* params,
                   float* grid, int nx, int ny, int nz,
                   const float* p0, const float* dA, const float* dB, const float* dC,
                   const float* Qs, const float* QZs, void* stream);

/* The same pair sums at arbitrary points, uncapped: replaces
 * cs_brute_afm_morse_c_points (kernels/contact_surface.cl:1341-1390) behind
 * AFMulator._brute_afm_morse_c_queries (spammm/SPM/AFM.py:1051-1067), the
 * direct reference of the grid builder.  queries (n_q,3) float32, out (n_q,4)
 * = (Fx,Fy,Fz,E); atoms/params/Qs/QZs as spm_grid_build. */
int spm_pair_fe_points(int kind, int n_atoms, const float* atoms, const float* params, const float* queries,
                       int n_q, const float* Qs, const float* QZs, float* out, void* stream);

/* ------------------------------------------------------------------------
 * (b) Probe relaxation on the grid.
 * spm_relax_strokes replaces AFMulator.scan_fdbm's launch of relaxStrokes
 * (spammm/SPM/AFM.py:607-617 -> kernels/AFM.cl:345-394): per pixel and z-step,
 * up to max_iter integrator steps on the trilinearly sampled grid force plus
 * tipForce; stores the last in-loop sample FE and the displacement
 * pos - (tipPos + dpos0).  Uses p->dTip, ignores the tip frame.
 *   FEs, disps out: (n_scan, p->nz, 4). */
int spm_relax_strokes(const float* grid, int nx, int ny, int nz,
                      const float* points, int n_scan, const spm_scan_params* p,
                      float* FEs, float* disps, void* stream);

/* Extended form of spm_relax_strokes (mode SPM_RELAX_STROKES) and
 * spm_relax_strokes_tilted (mode SPM_RELAX_TILTED, disps unused); no
 * counterpart in the reference, results identical to those two calls.
 *   iter_count: DEVICE int[n_scan] or NULL -- each pixel's integrator steps
 *               summed over its z-steps (telemetry);
 *   workspace:  DEVICE buffer of spm_relax_workspace_bytes() bytes or NULL.
 *               With a workspace, lanes take pixels from a device-side counter
 *               (dynamic load balance across lanes, warps and CTA waves); the
 *               call resets it on `stream`.  Calls that overlap on the device
 *               must not share a workspace. */
#define SPM_RELAX_STROKES 0
#define SPM_RELAX_TILTED  1
/* SPM_RELAX_PP: the tilted relaxation with the direct path's equilibrium
 * bookkeeping (kernels/AFM.cl:1441-1505) on the grid -- convergence tested
 * before each update, FEs sampled at the stored position, and `disps`
 * receiving PPs = (pos, +iters converged / -iters not).  The forward of the
 * differentiable grid path (spm_adjoint_grid_*). */
#define SPM_RELAX_PP      2
/* SPM_RELAX_2D: relaxStrokes2D (kernels/AFM.cl:410-450, AFMulator.scan_fdbm_2d
 * spammm/SPM/AFM.py:644-704): per slice iz the probe z is fixed at
 * point.z - iz*dh with dh = -p->dTip[2]; x,y start at the anchor and follow
 * damped MD (v = v*(1-damp) + f*dt, p += v*dt, f = F_grid.xy - K_lat (p -
 * anchor)) for at most max_iter steps, stopping after the update once
 * |f|^2 < f2conv; FEs = the grid sample at the final position, disps =
 * (dx, dy, 0, 0).  K_lat = p->stiffness[0] (> 0), (dt, damp) =
 * p->relax_params[0..1]; SPM_FLAG_FLIP_Z honoured, the tip frame ignored. */
#define SPM_RELAX_2D      3
long long spm_relax_workspace_bytes(void);
int spm_relax_ex(int mode, const float* grid, int nx, int ny, int nz,
                 const float* points, int n_scan, const spm_scan_params* p,
                 float* FEs, float* disps, int* iter_count, void* workspace, void* stream);

/* The forward + reverse=True scan_fdbm pair and compute_dissipation in ONE
 * launch (spammm/SPM/AFM.py:584-633 twice, then AFM.py:3238-3277; no single
 * counterpart in the reference): spm_relax_ex(SPM_RELAX_STROKES) with
 * SPM_FLAG_PAIRED (required; n_scan even, pixel p's strokes are points p and
 * p + n_scan/2), and per pixel E_diss[p, o] = |trapz over the stored heights
 * idx[off[o]..off[o+1]) of (FE_fwd - FE_bwd).n| with abscissae h_scan
 * (DEVICE double[p->nz], in the stored z order) -- the arithmetic of
 * spm_dissipation, bit for bit.  The lane that finishes the second stroke of
 * a pixel integrates it, reading both strokes' FEs back from L2; no lane
 * waits.  n: HOST double[3] (normalised here); off (DEVICE int[n_out+1]), idx
 * (DEVICE int[]); E_diss out (n_scan/2, n_out) float32; FEs, disps, iter_count
 * as spm_relax_ex.  workspace: DEVICE, 16-byte aligned, >=
 * spm_relax_pair_workspace_bytes(n_scan) bytes (reset by the call). */
int spm_relax_pair_dissipation(const float* grid, int nx, int ny, int nz, const float* points, int n_scan,
                               const spm_scan_params* p, float* FEs, float* disps, int* iter_count,
                               const double* n, const double* h_scan, const int* off, const int* idx,
                               int n_out, float* E_diss, void* workspace, void* stream);
long long spm_relax_pair_workspace_bytes(int n_scan);

/* Replaces AFMulator.run_scan -> relaxStrokesTilted (spammm/SPM/AFM.py:950-1010,
 * kernels/AFM.cl:478-562): tip-frame spring, surface bias, re-sampled FE after
 * the loop, output rotated into the tip frame.  dtip = p->tipC[3]. */
int spm_relax_strokes_tilted(const float* grid, int nx, int ny, int nz,
                             const float* points, int n_scan, const spm_scan_params* p,
                             float* FEs, void* stream);

/* Replaces AFMulator.get_raw_FE -> getFEinStrokesTilted (spammm/SPM/AFM.py:2523-2580,
 * kernels/AFM.cl:210-233): unrelaxed samples at point + dpos0 + iz*dTip,
 * rotated into the tip frame. */
int spm_fe_in_strokes_tilted(const float* grid, int nx, int ny, int nz,
                             const float* points, int n_scan, const spm_scan_params* p,
                             float* FEs, void* stream);

/* ------------------------------------------------------------------------
 * (c) Frequency shift.  FE volumes are (nx,ny,nz,4) float32 or float64
 * (fes_dtype = SPM_F32 / SPM_F64), as the reference's NumPy functions accept
 * either.
 * spm_df_amp_dir replaces compute_df_amp_dir (spammm/SPM/AFM.py:3203-3236):
 * F_n = F.n on the (nx,ny,nz,4) volume FEs (iz=0 lowest), 9-point
 * Gauss-Chebyshev average of -d(F_n)/ds over the oscillation s in [-amp,amp]
 * (linear interpolation with clamped indices, numpy.gradient differences),
 * evaluated in FP64.  n, dr: HOST double[3] (n normalised by the caller,
 * dr = grid spacing).  out_iz: DEVICE int[n_out] list of z indices to emit
 * (NULL = all nz, n_out ignored; an index outside [0,nz) yields NaN).
 * df out: (nx,ny,n_out) float32. */
int spm_df_amp_dir(const void* FEs, int fes_dtype, int nx, int ny, int nz, const double* n,
                   const double* dr, double amp, const int* out_iz, int n_out, float* df, void* stream);

/* Replaces compute_df_dir (spammm/SPM/AFM.py:3105-3123): df = -n.grad(F.n)
 * without amplitude averaging; df out (nx,ny,nz) float64. */
int spm_df_dir(const void* FEs, int fes_dtype, int nx, int ny, int nz, const double* n,
               const double* dr, double* df, void* stream);

/* Replaces compute_dissipation (spammm/SPM/AFM.py:3238-3277): for each output
 * height i, |trapz over the index list idx[off[i]..off[i+1]) of
 * (F_fwd - F_bwd).n dz| with abscissae h_scan.  n: HOST double[3];
 * h_scan (DEVICE double[nz]), off (DEVICE int[n_out+1]), idx (DEVICE int[]);
 * an index outside [0,nz) yields NaN.  E out (nx,ny,n_out) float32. */
int spm_dissipation(const void* FEs_fwd, const void* FEs_bwd, int fes_dtype, int nx, int ny, int nz,
                    const double* n, const double* h_scan, const int* off, const int* idx,
                    int n_out, float* E_diss, void* stream);

/* Replaces the convolveZ kernel (kernels/AFM.cl:666-701): for each of n_col
 * z-columns and izo < nz_out, Fout[c,izo] = sum over jz < nzw of
 * Fin[c,izo+jz] * w[jz], nzw = nz_in - nz_out (0..1024; the reference holds
 * up to 64 weights), all four channels, accumulated in jz order with fused
 * multiply-adds.  Fin (n_col,nz_in,4), Fout (n_col,nz_out,4) float32; w
 * (DEVICE float[nzw]). */
int spm_convolve_z(const float* Fin, int n_col, int nz_in, int nz_out, const float* w, float* Fout,
                   void* stream);

/* Replaces the izoZ kernel (kernels/AFM.cl:705-723): per column the first
 * iz >= 1 with Fin[c,iz].z > iso gives zMap[c] = iz + (iso - Fin[c,iz-1].z) /
 * (Fin[c,iz].z - Fin[c,iz-1].z); no such iz gives -1.  Fin (n_col,nz,4)
 * float32, zMap (n_col) float32. */
int spm_izo_z(const float* Fin, int n_col, int nz, float iso, float* zMap, void* stream);

/* spm_df_loss_seed for callers that cannot allocate device memory around the
 * call (their allocator owns all device memory, or a cudaMalloc/cudaFree and
 * its implicit synchronisation is not allowed in their loop).  No counterpart
 * in the reference.  It takes no scratch: the per-block partial sums live in a
 * fixed 1 MiB device array inside the library, which every GPU that loads the
 * library holds until the process exits.  Limits and rules:
 *   - nx*ny*nz <= SPM_DF_LOSS_NOALLOC_MAX_ELEMS, else SPM_ERR_UNSUPPORTED;
 *   - the first call on each device looks up that array's device address
 *     (cudaGetSymbolAddress, with the device current); make that first call
 *     before any stream capture;
 *   - all calls on a device share the array: calls that overlap on the GPU
 *     (e.g. on two streams at once) race and give wrong results; serialise them;
 *   - every slot a call reads is written earlier by the same call, so no state
 *     carries over from the previous call;
 *   - the device address found by that first call is kept for the life of
 *     the process: after cudaDeviceReset (or anything else that destroys the
 *     device's primary context) the kept address is stale; do not call this
 *     entry point on that device again in the same process;
 *   - allocates nothing (no cudaMalloc/cudaFree or allocating library call). */
#define SPM_DF_LOSS_NOALLOC_MAX_ELEMS 16777216LL
int spm_df_loss_seed_noalloc(const void* FEs, int fes_dtype, const double* target, const double* weights,
                             int nx, int ny, int nz, double dtip, double* df_out, float* dL_dFEs,
                             double* loss_out, void* stream);

/* Replaces df_loss_seed (spammm/SPM/AFM.py:3125-3200): central-difference df of
 * Fz = FEs[...,2] with |dtip|, L = 0.5*sum(w (df - target)^2)/sum(w) and the
 * exact transpose dL/dFEs (only the z channel non-zero).  target, weights
 * (nx,ny,nz) float64 (weights NULL = 1 inside, 0 on the two boundary slices);
 * df_out (nx,ny,nz) f64, dL_dFEs (nx,ny,nz,4) f32, loss_out: device double[1].
 * Uses `scratch` (device, >= spm_df_loss_scratch_bytes(nx,ny,nz) bytes). */
int spm_df_loss_seed(const void* FEs, int fes_dtype, const double* target, const double* weights,
                     int nx, int ny, int nz, double dtip, double* df_out, float* dL_dFEs,
                     double* loss_out, void* scratch, void* stream);
long long spm_df_loss_scratch_bytes(int nx, int ny, int nz);

/* ------------------------------------------------------------------------
 * Differentiable grid-free Morse+Coulomb path.
 * spm_relax_direct_morse replaces AFMulator.run_scan_morse_direct
 * (spammm/SPM/AFM.py:2063-2233) -> relaxStrokesTiltedMorseDirect
 * (kernels/AFM.cl:1419-1511): uncapped direct pair sum, convergence tested
 * before each update, PPs = (pos, +iters converged / -iters not).
 * atoms (n_atoms,4), cMs (n_atoms,4) = (R0,E0,K,0); Qs,QZs HOST float[4];
 * FEs, PPs out (n_scan,nz,4).  1 <= n_atoms <= SPM_DIRECT_MAX_ATOMS. */
#define SPM_DIRECT_MAX_ATOMS 4096
int spm_relax_direct_morse(int n_atoms, const float* atoms, const float* cMs,
                           const float* points, int n_scan, const spm_scan_params* p,
                           const float* Qs, const float* QZs,
                           float* FEs, float* PPs, void* stream);

/* Replaces morseDirectStateAdjoint (kernels/AFM.cl:1711-1845): per state the
 * implicit-function adjoint J lambda = b at the stored PP; lambdas (n_state,4),
 * diag (n_state,4) = (residual, lambda_min, cond, status 0..4). */
int spm_adjoint_direct_state(int n_atoms, const float* atoms, const float* cMs,
                             const float* points, int n_scan, const spm_scan_params* p,
                             const float* Qs, const float* QZs, const float* PPs,
                             const float* dL_dFEs, float* lambdas, float* diag, void* stream);

/* Replaces morseDirectParamPartials + reduceMorseDirectParamPartials
 * (kernels/AFM.cl:1850-2029): grad (n_atoms,6) float32 = per-atom
 * d(loss)/d(x,y,z,R0,E0,Q), reduced deterministically (no atomics) through
 * `scratch` (device, >= spm_adjoint_direct_scratch_bytes(...) bytes). */
int spm_adjoint_direct_params(int n_atoms, const float* atoms, const float* cMs,
                              const float* points, int n_scan, const spm_scan_params* p,
                              const float* Qs, const float* QZs, const float* PPs,
                              const float* dL_dFEs, const float* lambdas,
                              float* grad, void* scratch, void* stream);
long long spm_adjoint_direct_scratch_bytes(int n_atoms, int n_scan);

/* ------------------------------------------------------------------------
 * Differentiable grid path (no counterpart in the reference, which
 * differentiates only its grid-free direct path, kernels/AFM.cl:1711-2029).
 * Forward: spm_grid_build + spm_relax_ex(SPM_RELAX_PP) -> FEs, PPs.
 *
 * spm_adjoint_grid_state: per state, at the stored equilibrium PPs, solves
 * J^T lambda = b with J = dF_grid/dq + R^T (dg/dd) R (F_grid = trilinear
 * interpolant of the grid forces, g = tip spring) and
 * b = (dF_grid/dq)^T R^T u_xyz + grad(E_grid) u_w, u = dL_dFEs[state].
 * Writes ubar = (R^T u_xyz - lambda, u_w), dk = the state's d(loss)/d(stiffness)
 * terms, diag = (residual, lambda_min, cond, status) with status 0 ok,
 * 1 not converged / residual >= 5e-4, 2 non-finite, 3 unstable, 4 singular or
 * ill-conditioned, 5 touches a node rescaled by the |E|>100 cap (masked:
 * ubar = dk = 0).  All (n_scan*nz,4) float32. */
int spm_adjoint_grid_state(const float* grid, int nx, int ny, int nz,
                           const float* points, int n_scan, const spm_scan_params* p,
                           const float* PPs, const float* dL_dFEs,
                           float* ubar, float* dk, float* diag, void* stream);

/* spm_adjoint_grid_params: d(loss)/d(atom parameters) through the grid build
 * (atomics-free: each state's 8 trilinear corner nodes are revisited per atom
 * and the pair-law derivatives contracted with ubar; FP64 accumulation, fixed
 * reduction order) and d(loss)/d(stiffness).  kind/atoms/params/p0/dA/dB/dC/
 * Qs/QZs as spm_grid_build (HOST float[4] vectors); grid, nx, ny, nz, p as the
 * forward.  grad out (n_atoms,6) double = (x, y, z, P1, P2, Q) with
 * (P1,P2) = (c6,c12) for LJ, (R0,E0) for Morse; dk_sum out double[4] =
 * d(loss)/d(stiffness.xyzw).  scratch >= spm_adjoint_grid_scratch_bytes. */
int spm_adjoint_grid_params(int kind, int n_atoms, const float* atoms, const float* params,
                            const float* p0, const float* dA, const float* dB, const float* dC,
                            const float* Qs, const float* QZs, const float* grid, int nx, int ny, int nz,
                            const spm_scan_params* p, const float* PPs, const float* ubar,
                            const float* dk, long long n_state, double* grad, double* dk_sum,
                            void* scratch, void* stream);
long long spm_adjoint_grid_scratch_bytes(int n_atoms, long long n_state);

/* ------------------------------------------------------------------------
 * Batched grid path: many molecules of uneven atom count, grid size and scan
 * window, each stage ONE launch over the whole batch (no counterpart in the
 * reference, whose AFMulator (spammm/SPM/AFM.py) handles one molecule per
 * call).  Per molecule the results equal the per-molecule calls
 * spm_grid_build -> spm_relax_ex(SPM_RELAX_PP) -> spm_adjoint_grid_state on
 * the same inputs: forward values bit for bit, gradients up to the order of
 * the FP64 sums.  Scans are z-strokes: one probe frame and spring shared by
 * the batch (spm_scan_params), per-molecule grids, rasters and z-step counts.
 *
 * SLABS.  A molecule stores only the box of nodes [x_lo, x_lo + nx_slab) x
 * [y_lo, y_lo + ny_slab) x [z_lo, z_lo + nz_slab) of its full (nx,ny,nz) grid
 * (the nodes its probe can reach: the scan window and the tip's z-range, each
 * widened by a margin).  Nodes are built and sampled in the full grid's
 * coordinates, so stored values and samples are bit-identical to the full
 * grid's; a probe that needs a node outside the box stops at once and its
 * state reports "not converged" (FEs NaN, PPs.w = -iterations).  A box that
 * spans an axis completely keeps that axis' periodic wrap.
 *
 * DESCRIPTORS.  One spm_batch_mol per molecule, in the order work is handed
 * out; every *_off field is non-decreasing in that order (kernels locate a
 * work item's molecule by binary search).  The caller fills the geometry
 * fields and the buffer offsets: atom_off, pix_off and state_off contiguous
 * from 0 (each molecule's rows right after the previous molecule's), grid_off
 * increasing with non-overlapping slabs;
 * spm_batch_prepare fills tile_off, slot_off, unit_off and chunk_off for a
 * given spm_batch_shape, which every launch on these descriptors must then
 * be given unchanged.  The descriptor array is copied to device memory by the
 * caller; launches take the DEVICE copy.  Layouts:
 *   atoms  (total_atoms,4) x,y,z,Q;  params (total_atoms,2) LJ c6,c12 or
 *          (total_atoms,4) Morse R0,E0,K,-
 *   grid   slabs in one of two layouts (spm_batch_shape.grid_layout), node
 *          idx = (zl*ny_slab + yl)*nx_slab + xl of a molecule, (xl, yl, zl) =
 *          (x - x_lo, y - y_lo, z - z_lo):
 *          0 x-pairs: grid[2*(grid_off + idx) + dx] = value(x_lo + (xl+dx) mod
 *            nx_slab, y, z), a trilinear cell row is one 32-byte load (the
 *            wrapped second value of the last stored column is a real
 *            neighbour only when nx_slab = nx); 2*totals[7] float4;
 *          1 xz-quads: grid[4*(grid_off + idx) + 2*dz + dx] = value(x_lo +
 *            (xl+dx) mod nx_slab, y, z_lo + (zl+dz) mod nz_slab), a cell's
 *            two (y) rows are two 64-byte chunks; 4*totals[7] float4
 *   points (total_pixels,4) tip start positions (raster ix-major when
 *          raster_ny > 0, as spm_relax_ex)
 *   states (total_states,4) per molecule n_scan x nz_steps, z-step fastest */
typedef struct spm_batch_mol {
    long long grid_off;   /* float4 index of the slab */
    long long state_off;  /* first state */
    long long tile_off;   /* first grid-build tile              (spm_batch_prepare) */
    long long slot_off;   /* first relaxation slot              (spm_batch_prepare) */
    long long unit_off;   /* first adjoint node-chunk unit      (spm_batch_prepare) */
    long long chunk_off;  /* first 256-state loss chunk         (spm_batch_prepare) */
    long long row_off;    /* first (unit, atom) adjoint partial (spm_batch_prepare) */
    int atom_off, n_atoms;
    int pix_off, n_scan;
    int nx, ny, nz;       /* full grid */
    int z_lo, nz_slab;    /* stored layers */
    int nz_steps;         /* z-steps of every stroke */
    int raster_ny;        /* > 0: points form an (n_scan/raster_ny) x raster_ny raster */
    int x_lo, nx_slab;    /* stored columns */
    int y_lo, ny_slab;    /* stored rows */
    int reserved;
    float p0[4], dA[4], dB[4], dC[4];   /* node geometry (dA,dB,dC as spm_grid_build) */
    float dinvA[4], dinvB[4], dinvC[4]; /* sampling transform (as spm_scan_params) */
} spm_batch_mol;

/* Launch shapes; spm_batch_default_shape() gives a valid default, the
 * autotuner in the Python package searches the rest. */
typedef struct spm_batch_shape {
    int gb_ty;          /* grid build: CTA = 32 x gb_ty threads, gb_ty in {2,4,8} */
    int gb_zb;          /* grid build: nodes along z per thread, 8 or 16 */
    int rx_threads;     /* relaxation CTA size: 64, 128 or 256 */
    int rx_tile_h;      /* relaxation pixel tile: (32/rx_tile_h) x rx_tile_h pixels, power of two <= 32 */
    int rx_ctas_per_sm; /* persistent relaxation CTAs per SM, 0 = occupancy maximum */
    int adj_chunk;      /* slab nodes per adjoint unit: multiple of 1024 in [1024, 1048576] */
    int rx_regs;        /* relaxation kernel variant: 0 = 80 registers per thread, 1 = 64 (more warps,
                           some spills), 2 = the cell's 8 texels kept in registers across FIRE
                           iterations (up to 128 registers, loads only when the cell changes),
                           3 = the texel cache at 80 registers (some spills, more warps), 4 = the
                           texel cache at up to 102 registers in CTAs of at most 128 threads, 5 = the
                           texel cache with each warp's z-slab box staged in shared memory by bulk copies
                           (128-thread CTAs, x-pair slabs, rx_sync = 1, no SPM_FLAG_POLISH / WARM) */
    int grid_layout;    /* slab layout: 0 = x-pairs (2 float4 per node), 1 = xz-quads (4 float4 per
                           node: half the cache lines per sample, twice the memory) */
    int rx_sync;        /* relaxation schedule: 0 = every lane draws its next pixel when its stroke ends,
                           1 = a warp draws a pixel tile and its lanes step down the z-steps together
                           (all lanes sample the same z-layer of neighbouring pixels), 2 = with
                           SPM_FLAG_POLISH and SPM_FLAG_WARM two passes: the tiles of 1 with Newton's
                           method from the previous equilibria only, each stroke stopping at its first
                           z-step that needs FIRE, then those strokes' remaining z-steps, 32 strokes
                           per warp stepping together (without both flags: as 1).  Same results */
    int adj_ilp;        /* adjoint node kernel: 1 = one atom and one node pair per step (4 CTAs per SM),
                           2 = two independent node pairs per step (2 CTAs per SM, more registers),
                           3 = two atoms per thread sharing each node pair's loads (2 CTAs per SM) */
    int adj_agg;        /* adjoint scatter: 0 = every state's corner sums straight to the global adjoint
                           grid (64-bit atomics), 1 = first merged per CTA in a shared-memory table
                           (the strokes of one CTA share nodes), one global atomic per distinct node,
                           2 = a warp walks a relaxation pixel tile (rx_tile_h) down its strokes; each
                           lane carries its lower corner layer down the stroke and takes over the
                           nodes its raster neighbours (next row, next column) share with it before
                           the atomics (the default).  Same sums */
    int adj_stage;      /* adjoint node kernel: 0 = each block of adjoint-grid nodes read with plain
                           loads, 1 = fetched into shared memory by a bulk copy while the previous
                           block is examined and computed (with adj_ilp = 1) */
} spm_batch_shape;

spm_batch_shape spm_batch_default_shape(void);

/* Validates the descriptors (HOST array) and fills tile_off, slot_off,
 * unit_off, chunk_off and row_off for `shape`.  totals_out (HOST
 * long long[SPM_BATCH_TOTALS]) = (tiles, slots, units, chunks, states, atoms,
 * pixels, grid float4s, rows). */
#define SPM_BATCH_TOTALS 9
int spm_batch_prepare(spm_batch_mol* mols, int n_mol, const spm_batch_shape* shape, long long* totals_out);

/* Force-grid slabs of every molecule (pair laws, tip sites and the |E|>100
 * cap as spm_grid_build), written in the x-paired layout.
 * n_tiles = totals_out[0]. */
int spm_batch_grid_build(int kind, int n_mol, const spm_batch_mol* mols, long long n_tiles,
                         const spm_batch_shape* shape, const float* atoms, const float* params,
                         const float* Qs, const float* QZs, float* grid, void* stream);

/* SPM_RELAX_PP relaxation of every stroke of every molecule in one persistent
 * launch (two with shape->rx_sync = 2): lanes draw (molecule, pixel) slots
 * from a device counter in `workspace` (workspace_bytes >=
 * spm_batch_relax_workspace_bytes(n_slots, shape) bytes, device memory, its
 * counters reset by the call; rx_sync = 2 also keeps its list of strokes
 * for the second pass there, 48 bytes per slot).
 * p: probe frame, spring, FIRE settings, flags, tipC[3] = z-step; its dinv*,
 * nz and raster_ny are ignored (per-molecule values come from mols).
 * flags: SPM_FLAG_FIRE, SPM_FLAG_POLISH and SPM_FLAG_WARM (the last two with
 * shape->rx_sync = 1 or 2).
 * FEs, PPs out (total_states,4); iter_count (total_pixels) or NULL. */
long long spm_batch_relax_workspace_bytes(long long n_slots, const spm_batch_shape* shape);
int spm_batch_relax(int n_mol, const spm_batch_mol* mols, long long n_slots, const spm_batch_shape* shape,
                    const float* grid, const float* points, const spm_scan_params* p,
                    float* FEs, float* PPs, int* iter_count, void* workspace, long long workspace_bytes,
                    void* stream);

/* Frequency shift of every stroke, as spm_df_amp_dir with n = z and
 * dr = |dtip| on the stroke taken in ascending z (the stroke reversed), the
 * result written back in stroke order: df out (total_states) float32.
 * Strokes with nz_steps < 2 or > 512 get NaN. */
int spm_batch_df_amp(int n_mol, const spm_batch_mol* mols, long long n_pixels, const float* FEs,
                     double dtip, double amp, float* df, void* stream);

/* df loss of every molecule, as spm_df_loss_seed on its (n_scan,1,nz_steps)
 * volume: target, weights (total_states) float64 (weights NULL = 1 inside,
 * 0 on each stroke's first and last z-step); df_out (total_states) f64;
 * dL_dFEs (total_states,4) f32; loss_out (n_mol) f64 in descriptor order.
 * A molecule whose weights sum to zero (no pixels, nz_steps < 3 with the
 * default weights, every state masked) gets loss 0 and dL_dFEs = 0, where
 * the single-volume formula's 0/0 is NaN: it adds nothing to a batch loss.
 * With nz_steps < 3 dL_dFEs is 0 (no central difference).
 * scratch >= spm_batch_loss_scratch_bytes(n_chunks, n_mol). */
int spm_batch_df_loss_seed(int n_mol, const spm_batch_mol* mols, long long n_chunks, const float* FEs,
                           const double* target, const double* weights, double dtip, double* df_out,
                           float* dL_dFEs, double* loss_out, void* scratch, void* stream);
long long spm_batch_loss_scratch_bytes(long long n_chunks, int n_mol);

/* Loss weights of a fitting step from the previous step's adjoint status:
 * weights[s] = w_base[s] if states s-1, s and s+1 (cyclic over the n_states
 * array) all passed the adjoint gates (diag[.].w == 0), else 0 -- a failed
 * state and the z-neighbours whose central-difference df sees it leave the
 * loss.  diag (n_states,4) f32; w_base, weights (n_states) f64. */
int spm_batch_failure_mask(long long n_states, const float* diag, const double* w_base, double* weights,
                           void* stream);

/* One Adam step (Kingma & Ba, 2015) of a fit over the batch's atoms, in place, FP32: for every atom i
 * and every column c set in `cols` (bit 0-3: x, y, z, charge), g = grad[6 i + (c < 3 ? c : 5)],
 * m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2, atoms -= lr (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps)
 * with t = *t_steps + 1, which is stored back (a device float, so graph replays count the steps);
 * 1 - b1, 1 - b2 and the bias corrections are formed in FP64 and rounded once.
 * grad (n_atoms,6) f64 as spm_batch_adjoint_params writes it; atoms, m, v (n_atoms,4) f32, 16-byte
 * aligned.  One launch of one CTA.  Replaces the in-place tensor updates of a fitting loop (the
 * reference fits with host-side optimisers; this has no reference counterpart). */
int spm_batch_adam_step(long long n_atoms, const double* grad, float* atoms, float* m, float* v, float* t_steps,
                        double lr, double beta1, double beta2, double eps, int cols, void* stream);

/* spm_adjoint_grid_state over the batch (same outputs per state).
 * adj_scratch (optional, with totals: the scratch of spm_batch_adjoint_params
 * for this batch): the call also leaves there each molecule's max |ubar| and
 * box of touched slab rows and layers, which spm_batch_adjoint_params then
 * takes with SPM_ADJ_STATE_MAXIMA instead of a pass over ubar of its own.
 * NULL: no maxima (totals may be NULL).  dk may be NULL: the spring-parameter
 * terms are not written (fits that do not move the spring; pass NULL to
 * spm_batch_adjoint_params too). */
int spm_batch_adjoint_state(int n_mol, const spm_batch_mol* mols, long long n_states,
                            const spm_batch_shape* shape, const float* grid, const float* points,
                            const spm_scan_params* p, const float* PPs, const float* dL_dFEs, float* ubar,
                            float* dk, float* diag, const long long* totals, void* adj_scratch, void* stream);

/* spm_adjoint_grid_params over the batch, node-major: grad (total_atoms,6)
 * double as spm_adjoint_grid_params, dk_sum double[4] summed over the whole
 * batch (one probe; 0 when dk is NULL).
 *   1. the states' w*ubar are scattered onto an adjoint grid over each slab
 *      (the transpose of the trilinear sample) in 64-bit fixed point with a
 *      per-molecule power-of-two scale (2^42 / max|ubar|), so the integer
 *      sums are exact and order-independent: bit-reproducible;
 *   2. an atomics-free scatter by atom tiles: each CTA stages a chunk of
 *      non-zero adjoint-grid nodes in shared memory and every thread owns one
 *      atom (and a phase of the chunk), evaluating the pair-law derivatives of
 *      its atom at each staged node; per-(chunk, atom) FP64 partials are folded
 *      per atom in a fixed order.  Nodes outside each molecule's box of
 *      touched rows and layers are not read, and every node read is zeroed
 *      again.
 * totals: the HOST array of spm_batch_prepare; scratch (device) >=
 * spm_batch_adjoint_scratch_bytes(totals, n_mol).  The scratch keeps the
 * cleared adjoint grid between calls, with a marker that says it is clear
 * (tied to the buffer's address and the layout): reuse one scratch buffer
 * call after call, and zero-fill a newly allocated one before its first call
 * (memory that held an earlier scratch of the same layout at the same
 * address can still carry its marker over content written since); other
 * content -- a zero-filled buffer, a call that failed half-way -- is cleared
 * by the next call.
 * adj_flags: SPM_ADJ_PAIR_PARAMS computes grad columns 3-4 (the pair
 * parameters); without it they are written as 0 and the node kernel skips
 * their terms (fits of positions and charges only).  SPM_ADJ_STATE_MAXIMA:
 * the scratch holds the maxima and boxes of this ubar from
 * spm_batch_adjoint_state (called with this scratch after the last change
 * of ubar); without it the call computes them. */
#define SPM_ADJ_PAIR_PARAMS 1
#define SPM_ADJ_STATE_MAXIMA 2
int spm_batch_adjoint_params(int kind, int n_mol, const spm_batch_mol* mols, const long long* totals,
                             const spm_batch_shape* shape, const float* atoms, const float* params,
                             const float* Qs, const float* QZs, const float* PPs, const float* ubar,
                             const float* dk, double* grad, double* dk_sum, int adj_flags, void* scratch,
                             void* stream);
long long spm_batch_adjoint_scratch_bytes(const long long* totals, int n_mol);

/* ------------------------------------------------------------------------
 * Measurement helper (not part of the reference interface): runs a dependent
 * FFMA chain on every SM and writes the achieved FP32 FLOP/s to *out_flops
 * (host double).  Blocking. */
int spm_fp32_peak_probe(int iters, double* out_flops, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SPM_B200_H */
