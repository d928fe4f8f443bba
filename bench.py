"""Benchmark of the probe-particle AFM hot path on B200.

Step = one pass of the plain path over one synthetic system: (a) LJ + Coulomb
force-grid build, (b) FIRE relaxation of every pixel down its z-stroke
(relaxStrokes semantics, <= 1000 steps, |F| < 1e-5 eV/A), (c) 9-point
finite-amplitude df at every height.  Workload: 1140-ion NaCl(100) slab +
60-atom molecule (1200 atoms), grid 480x480x240 (48x48x24 A at 0.1 A), 480x480
pixels x 60 z-steps (synthetic, seeded; see spammm_b200/synthetic.py).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` = px*z per second of the whole step
with inputs resident in HBM (CUDA events around the K timed steps, max over
ranks); `e2e` = the same through the drop-in AFMulator API with host buffers
(uploads and downloads inside the timed region).  Under torchrun each rank runs
its own replica of the workload (the path has no exchange step).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "probe relax px·z/s; batched fwd+adjoint images/s vs plain, Δf err≤1e-3"
UNIT = "px·z/s"
# algorithmic work per (node, atom) pair with every law counted in full, FMA = 2 flops: LJ 26, Morse 28, +23 per
# non-zero tip-charge site (the on-node charge's Coulomb law included, although the kernel shares its rsqrt)
FLOPS_PAIR = {0: 26, 1: 28}
FLOPS_SITE = 23
# work the grid-build kernel executes per (node, atom) pair (csrc/grid_build.cu, build_tile's packed
# f32x2 loop; two nodes per instruction): FP32-pipe lane instructions and flops (FMA = 2), besides one
# MUFU rsqrt (and one ex2 for Morse).  Pair law with the on-node charge merged (ON): LJ 15 instructions /
# 23 flops, Morse 16 / 23; without charges: LJ 13 / 20, Morse 13 / 19; each off-node charge site adds
# 8 / 13 (+1 MUFU).
EXEC_PAIR = {(0, True): (15, 23), (0, False): (13, 20), (1, True): (16, 23), (1, False): (13, 19)}
EXEC_SITE = (8, 13)
# DRAM bytes of one grid_build_kernel launch on the 1200-atom / 480x480x240 workload, from the ncu
# capture in profiles/grid_build_plain_large.md (dram__bytes_read.sum + dram__bytes_write.sum)
GRID_BUILD_DRAM_BYTES = 6017024 + 826515456


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="plain_large", choices=["plain_large", "plain_small"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the many-molecule workloads")
    ap.add_argument("--batch-mols", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=3)
    ap.add_argument("--fit-mols", type=int, default=64)
    ap.add_argument("--fit-steps", type=int, default=100)
    ap.add_argument("--fit-lr", type=float, default=0.01, help="Adam learning rate of the fit (A, e)")
    ap.add_argument("--fit-groups", type=int, default=4,
                    help="fit molecules dealt into this many batches, each on its own stream in one graph")
    ap.add_argument("--fit-z-end", type=float, default=3.0,
                    help="lowest tip height of the fit's scans above the molecule plane (A)")
    ap.add_argument("--batch-only", action="store_true",
                    help="run only the many-molecule workloads (small sizes make profiling cases)")
    ap.add_argument("--no-tune", action="store_true", help="library default launch shapes, no autotuning")
    ap.add_argument("--fit-cold", action="store_true",
                    help="fit without the Newton polish and warm starts (every step relaxes from the strokes)")
    return ap.parse_args()


def make_config(name):
    from spammm_b200 import synthetic
    return synthetic.plain_large() if name == "plain_large" else synthetic.plain_small()


def config_dict(cfg, l2_note):
    return {"workload": f"{cfg.name}: {len(cfg.atoms)} atoms, grid {'x'.join(map(str, cfg.ngrid))} at "
                        f"{cfg.step} A, {len(cfg.scan_xs)}x{len(cfg.scan_ys)} px x {cfg.nz} z, FIRE<= {cfg.max_iter}, "
                        f"|F|<{np.sqrt(cfg.f2conv):.0e} eV/A, df amp {cfg.amp} A",
            "atoms": int(len(cfg.atoms)), "grid": list(cfg.ngrid), "pixels": [len(cfg.scan_xs), len(cfg.scan_ys)],
            "nz": cfg.nz, "potential": "LJ" if cfg.kind == 0 else "Morse", "l2": l2_note}


def grid_vectors(cfg):
    o = cfg.origin
    p0 = np.array([o[0], o[1], o[2], 0], np.float32)
    s = cfg.step
    return p0, np.array([s, 0, 0, 0], np.float32), np.array([0, s, 0, 0], np.float32), np.array([0, 0, s, 0],
                                                                                                np.float32)


def scan_points(cfg):
    gx, gy = np.meshgrid(cfg.scan_xs, cfg.scan_ys, indexing="ij")
    pts = np.zeros((cfg.n_pix, 4), np.float32)
    pts[:, 0] = gx.ravel()
    pts[:, 1] = gy.ravel()
    pts[:, 2] = np.float32(cfg.z_top)
    return pts


def scan_params(cfg, dinv):
    from spammm_b200 import _lib
    return _lib.make_scan_params(dinv=dinv, dTip=[0, 0, -cfg.dz, 0], stiffness=cfg.stiffness, dpos0=cfg.dpos0,
                                 relax_params=[0.5, 0.1, 0.02, 0.5], nz=cfg.nz, max_iter=cfg.max_iter,
                                 f2conv=cfg.f2conv, fire=True, flip_z=True, raster_ny=len(cfg.scan_ys))


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(ms, world, device=None):
    """The largest per-rank duration over all ranks (every rank receives it); the timed region of a
    replica run ends when its slowest rank ends."""
    if world <= 1:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank, ms_per_step, world):
    """Whole-job throughput of `world` replicas, each processing units_per_rank per step."""
    return world * units_per_rank / (ms_per_step * 1e-3)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


# ---------------------------------------------------------------------------- CPU (oracle) sample
class CpuSample:
    """A bounded, proportional sample of the step for the CPU (the oracle's C/OpenMP
    restatement of the reference kernels, all host threads): a patch x patch pixel window
    at the centre of the scan with its whole z-strokes, and the grid nodes under that window
    (the patch's columns x every z-layer), so the sample holds the same grid nodes per px*z as
    the full step.  One timed step = build those nodes + relax the window's strokes (on a
    sub-grid around the window with a lateral margin, built once before timing: the same
    values, see below) + df of the window.  Nothing is extrapolated: the reported rate is the
    sample's px*z over its measured time."""

    def __init__(self, cfg, patch=96, threads=None):
        from oracle import oracle as O
        self.O = O
        if threads:
            O.set_num_threads(threads)
        self.threads = O.num_threads()
        self.cfg = cfg
        nx, ny, nzg = cfg.ngrid
        patch = min(patch, len(cfg.scan_xs), len(cfg.scan_ys))
        self.patch = patch
        cx, cy = len(cfg.scan_xs) // 2, len(cfg.scan_ys) // 2
        self.xs = cfg.scan_xs[cx - patch // 2: cx - patch // 2 + patch]
        self.ys = cfg.scan_ys[cy - patch // 2: cy - patch // 2 + patch]
        p0, self.dA, self.dB, self.dC = grid_vectors(cfg)
        # grid-build part: the block of columns under the window, all z-layers (nodes per px*z of the full step)
        nodes_per_pxz = nx * ny * nzg / cfg.pxz
        self.n_cols = int(round(nodes_per_pxz * patch * patch * cfg.nz / nzg))
        side = int(round(np.sqrt(self.n_cols)))
        self.bx, self.by = side, max(1, self.n_cols // side)
        ix0 = int(round((float(self.xs[0]) - cfg.origin[0]) / cfg.step))
        iy0 = int(round((float(self.ys[0]) - cfg.origin[1]) / cfg.step))
        self.bp0 = np.array([cfg.origin[0] + ix0 * cfg.step, cfg.origin[1] + iy0 * cfg.step, cfg.origin[2], 0],
                            np.float32)
        # relaxation part: sub-grid with a lateral margin around the window (the node values are the full
        # grid's: same positions, same pair sums); periodic wrap is never reached inside it
        margin = 3.0
        sx0 = cfg.origin[0] + np.floor((float(self.xs[0]) - margin - cfg.origin[0]) / cfg.step) * cfg.step
        sy0 = cfg.origin[1] + np.floor((float(self.ys[0]) - margin - cfg.origin[1]) / cfg.step) * cfg.step
        sz0 = cfg.origin[2] + np.floor((cfg.z_top - cfg.dz * cfg.nz - 1.5 - cfg.origin[2]) / cfg.step) * cfg.step
        snx = int(np.ceil((float(self.xs[-1]) + margin - sx0) / cfg.step)) + 1
        sny = int(np.ceil((float(self.ys[-1]) + margin - sy0) / cfg.step)) + 1
        snz = int(np.ceil((cfg.z_top + 1.5 - sz0) / cfg.step)) + 1
        self.sub_n = (snx, sny, snz)
        sp0 = np.array([sx0, sy0, sz0, 0], np.float32)
        self.sub = O.grid_build(cfg.kind, cfg.atoms, cfg.params, self.sub_n, sp0, self.dA, self.dB, self.dC,
                                cfg.tipQs, cfg.tipQZs, prec="f32")
        self.dinv = O.dinv_axis_aligned(np.array(self.sub_n) * cfg.step, sp0[:3], self.sub_n)
        gx, gy = np.meshgrid(self.xs, self.ys, indexing="ij")
        self.pts = np.zeros((gx.size, 4), np.float32)
        self.pts[:, 0], self.pts[:, 1], self.pts[:, 2] = gx.ravel(), gy.ravel(), cfg.z_top
        self.pxz = self.pts.shape[0] * cfg.nz
        self.stage_s = np.zeros(3)
        self.steps = 0

    def step(self):
        cfg, O = self.cfg, self.O
        t0 = time.perf_counter()
        O.grid_build(cfg.kind, cfg.atoms, cfg.params, (self.bx, self.by, cfg.ngrid[2]), self.bp0, self.dA, self.dB,
                     self.dC, cfg.tipQs, cfg.tipQZs, prec="f32")
        t1 = time.perf_counter()
        FEs, _ = O.relax_strokes(self.sub, self.dinv, self.pts, cfg.nz, [0, 0, -cfg.dz, 0], cfg.stiffness, cfg.dpos0,
                                 [0.5, 0.1, 0.02, 0.5], cfg.max_iter, cfg.f2conv, True, True)
        t2 = time.perf_counter()
        O.compute_df_amp_dir(FEs.reshape(len(self.xs), len(self.ys), cfg.nz, 4), (cfg.step, cfg.step, cfg.dz),
                             (0, 0, 1), cfg.amp)
        t3 = time.perf_counter()
        self.stage_s += (t1 - t0, t2 - t1, t3 - t2)
        self.steps += 1
        return t3 - t0

    def describe(self):
        cfg = self.cfg
        n = max(self.steps, 1)
        return {"kind": "port", "cores": int(self.threads),
                "sample": f"oracle C/OpenMP FP32 on all host threads; per step: grid build of {self.bx}x{self.by}"
                          f"x{cfg.ngrid[2]} nodes ({self.bx * self.by * cfg.ngrid[2] / np.prod(cfg.ngrid):.2%} of the "
                          f"grid: the nodes per px*z of the full step) + FIRE relaxation of the central "
                          f"{len(self.xs)}x{len(self.ys)}-pixel window x {cfg.nz} z-steps ({self.pxz} px*z, "
                          f"{self.pxz / cfg.pxz:.2%} of the scan; on a {'x'.join(map(str, self.sub_n))} sub-grid built "
                          f"once before timing) + numpy df of the window; value = sample px*z / measured step time, "
                          f"nothing extrapolated",
                "stage_s_per_step": {"grid": self.stage_s[0] / n, "relax": self.stage_s[1] / n,
                                     "df": self.stage_s[2] / n}}


def cpu_sample(cfg, steps=3, threads=None):
    """cpu_baseline leg of our arm: a few steps of CpuSample.  Returns (px*z/s, details)."""
    cs = CpuSample(cfg, threads=threads)
    cs.step()  # warm-up
    cs.stage_s[:] = 0
    cs.steps = 0
    t = sum(cs.step() for _ in range(steps))
    det = cs.describe()
    det["ms_per_step"] = t / steps * 1e3
    return cs.pxz * steps / t, det


# ---------------------------------------------------------------------------- GPU arm
def run_ours(args, rank, world, local_rank):
    import torch
    from spammm_b200 import gpu, _lib, AFM
    from spammm_b200.AFM import AFMulator

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    cfg = make_config(args.config)
    nx, ny, nz = cfg.ngrid
    p0, dA, dB, dC = grid_vectors(cfg)
    L = np.array(cfg.ngrid) * cfg.step
    dinv = AFMulator._make_dinv_axis_aligned(L, cfg.origin.astype(np.float32), cfg.ngrid)
    P = scan_params(cfg, dinv)
    atoms_d = torch.from_numpy(cfg.atoms).to(dev)
    prm_d = torch.from_numpy(cfg.params).to(dev)
    pts_d = torch.from_numpy(scan_points(cfg)).to(dev)
    grid = torch.empty((nz, ny, nx, 4), dtype=torch.float32, device=dev)
    FEs = torch.empty((cfg.n_pix, cfg.nz, 4), dtype=torch.float32, device=dev)
    disps = torch.empty_like(FEs)
    npx, npy = len(cfg.scan_xs), len(cfg.scan_ys)
    spacing = (cfg.step, cfg.step, cfg.dz)
    stream = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    stage = np.zeros(3)

    def step(record):
        if record:
            ev[0].record(stream)
        gpu.grid_build(cfg.kind, atoms_d, prm_d, cfg.ngrid, p0, dA, dB, dC, cfg.tipQs, cfg.tipQZs, out=grid)
        if record:
            ev[1].record(stream)
        gpu.relax_strokes(grid, P, pts_d, FEs=FEs, disps=disps)
        if record:
            ev[2].record(stream)
        df = gpu.df_amp_dir(FEs.view(npx, npy, cfg.nz, 4), spacing, (0, 0, 1), cfg.amp)
        if record:
            ev[3].record(stream)
        return df

    for _ in range(args.warmup):
        step(False)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    for _ in range(args.steps):
        step(True)
        stream.synchronize()
        stage += [ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]), ev[2].elapsed_time(ev[3])]
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_total = max_over_ranks(t0.elapsed_time(t1), world, dev)
    stage /= args.steps
    ms_step = ms_total / args.steps
    # the events above wrap each stage; the sum of stages is the kernel time of a step (host syncs excluded)
    value = replica_value(cfg.pxz, ms_step, world)
    out = {}
    # FIRE telemetry (outside the timed region): integrator steps per px*z
    cnt = torch.empty(cfg.n_pix, dtype=torch.int32, device=dev)
    gpu.relax_strokes(grid, P, pts_d, FEs=FEs, disps=disps, iter_count=cnt)
    steps_total = float(cnt.double().sum().item())
    out["fire"] = {"steps_per_pxz": steps_total / cfg.pxz, "max_steps_pixel": int(cnt.max().item()),
                   "sampled_bytes_per_launch": steps_total * 8 * 16}

    # ---- e2e through the drop-in API (host buffers)
    e2e = None
    if not args.no_e2e:
        afm = AFMulator(use_morse=(cfg.kind == 1))
        afm.n_relax_max, afm.f2conv = cfg.max_iter, cfg.f2conv
        afm.tipQs, afm.tipQZs = cfg.tipQs, cfg.tipQZs

        def e2e_step():
            afm.atoms_arr = cfg.atoms.copy()
            afm.cLJs_arr = cfg.params.copy()
            afm.setup_grid_world(cfg.origin, L, cfg.ngrid)
            afm.make_forcefield()
            afm.setup_fdbm_grid_from_img(afm.img_FF, cfg.ngrid, cfg.origin, cfg.step)
            hs = (cfg.z_top - cfg.dz * np.arange(cfg.nz)[::-1]).astype(np.float32)
            F, disp = afm.scan_fdbm(cfg.scan_xs, cfg.scan_ys, hs, mol_z=0.0, bond_length=0.0,
                                    stiffness=cfg.stiffness, dpos0=cfg.dpos0)
            df = AFM.compute_df_amp_dir(F, spacing, (0., 0., 1.), cfg.amp)
            return F, disp, df

        # warm-up holds each result until the next step returns, as the timed loop does: the pinned host
        # buffers of two live results are then allocated (cudaHostAlloc) before the timed region
        held = None
        for _ in range(max(3, args.warmup)):
            held = e2e_step()
        del held
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ke = max(1, min(args.steps, 3))
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(ke):
            F, disp, df_h = e2e_step()
        a1.record(stream)
        torch.cuda.synchronize()
        ms_e = max_over_ranks(a0.elapsed_time(a1), world, dev)
        h2d = cfg.atoms.nbytes + cfg.params.nbytes + cfg.n_pix * 16 + F.nbytes  # atoms, params, points, FEs for df
        d2h = F.nbytes + 3 * F[..., 0].nbytes + df_h.nbytes  # FEs, tip displacement, df
        e2e = {"value": replica_value(cfg.pxz, ms_e / ke, world), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e / ke,
               "path": "AFMulator.setup_grid_world/make_forcefield/scan_fdbm + compute_df_amp_dir (numpy in/out)"}

    # ---- roofline of the dominant kernel
    peaks = measured_peaks()
    fp32_peak = gpu.fp32_peak_flops(1 << 15)
    ns = int(np.count_nonzero(cfg.tipQs))
    on = bool(cfg.tipQs[0] != 0 and cfg.tipQZs[0] == 0)  # the kernel merges an on-node site into the pair law
    n_off = ns - (1 if on else 0)
    inst_pair = EXEC_PAIR[(cfg.kind, on)][0] + EXEC_SITE[0] * n_off
    xflops_pair = EXEC_PAIR[(cfg.kind, on)][1] + EXEC_SITE[1] * n_off
    flops = cfg.pairs * (FLOPS_PAIR[cfg.kind] + FLOPS_SITE * ns)
    ach_fp32 = flops / (stage[0] * 1e-3)
    # FP32-pipe issue: lane instructions per second against the pipe's peak (the FFMA probe's FLOP/s / 2);
    # reported as FMA-equivalent TFLOP/s (2 flops per lane instruction) against the probe's peak
    ach_pipe = cfg.pairs * inst_pair * 2 / (stage[0] * 1e-3)
    ach_exec = cfg.pairs * xflops_pair / (stage[0] * 1e-3)
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    slab_nodes = nx * ny * (int(np.ceil((cfg.dz * cfg.nz + 2.0) / cfg.step)) + 2)
    relax_bytes = cfg.pxz * 32 + slab_nodes * 16
    ach_relax = relax_bytes / (stage[1] * 1e-3) / 1e9
    df_bytes = cfg.pxz * (16 + 4)
    names = ["grid_build_kernel", "relax_tile_kernel<0>", "df_amp_dir_kernel"]
    dom = int(np.argmax(stage))
    if dom == 0:
        roof = {"kernel": names[0], "bound": "fp32 pipe issue", "achieved": ach_pipe / 1e12,
                "peak": fp32_peak / 1e12, "unit": "TFLOP/s", "frac": ach_pipe / fp32_peak,
                "traffic": GRID_BUILD_DRAM_BYTES if cfg.name == "plain_large" else None,
                "traffic_note": "ncu dram__bytes_read.sum + write.sum of one launch (profiles/grid_build_plain_large.md); "
                                "the grid it writes is 884.7 MB",
                "peak_source": "measured live: FFMA-chain probe (spm_fp32_peak_probe) on this GPU",
                "algorithmic": f"{cfg.pairs:.3e} (node,atom) pairs x {inst_pair} FP32 lane instructions as "
                               f"executed (FMA-equivalent: x2 flops)",
                "executed_flops": {"per_pair": xflops_pair, "tflops": ach_exec / 1e12, "frac": ach_exec / fp32_peak,
                                   "note": "FMA = 2, mul/add = 1: the kernel's 15 lane instructions per pair hold "
                                           "8 FMAs and 7 mul/add"},
                "laws_counted_in_full": {"per_pair": FLOPS_PAIR[cfg.kind] + FLOPS_SITE * ns,
                                      "tflops": ach_fp32 / 1e12, "frac": ach_fp32 / fp32_peak,
                                      "note": "counts the on-node Coulomb law in full; the kernel shares its "
                                              "rsqrt and radial factor with the pair law, so this exceeds 1"}}
    else:
        roof = {"kernel": names[dom], "bound": "hbm", "achieved": ach_relax if dom == 1 else
                df_bytes / (stage[2] * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s", "traffic": None,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks else "fallback"}
        roof["frac"] = roof["achieved"] / hbm_peak
    out.update(stage_ms={"grid_build": stage[0], "relax": stage[1], "df": stage[2]},
               stage_roofline={"grid_build_pipe_frac": ach_pipe / fp32_peak, "fp32_peak_tflops": fp32_peak / 1e12,
                               "relax": {"bound": "issue / FIRE dependency chain (latency)",
                                         "fire_steps_per_s": steps_total / (stage[1] * 1e-3),
                                         "alg_gbs": ach_relax, "alg_bytes": relax_bytes,
                                         "alg_hbm_frac": ach_relax / hbm_peak},
                               "df_alg_gbs": df_bytes / (stage[2] * 1e-3) / 1e9})
    if rank != 0:
        return None
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded NaCl slab + planar molecule)",
            "config": config_dict(cfg, "inputs larger than L2 (grid 885 MB) -- no flush needed"),
            "roofline": roof, "gpu_launches": 3 * args.steps, "clocks": clk, "e2e": e2e}
    line.update(out)
    line["parallelism"] = f"replicas x{world}" if world > 1 else "single GPU"
    if not args.no_batch and world == 1:
        line["batched"] = run_batched(args, local_rank)
    if world == 1:
        line["direct"] = run_direct(args, local_rank)
    if not args.no_cpu and world == 1:
        v, det = cpu_sample(cfg)
        det["value"] = v
        det["unit"] = UNIT
        line["cpu_baseline"] = det
    return line


# ---------------------------------------------------------------------------- direct path
# per (FIRE step, atom) of relax_direct_kernel's pair loop: Morse 18 FP32 lane instructions + 2 MUFU
# (rsqrt, ex2), each non-zero tip-charge site 9 + 1 (the loop as written in csrc/direct.cu)
DIRECT_PAIR = (18, 2)
DIRECT_SITE = (9, 1)


def run_direct(args, dev_index):
    """The grid-free Morse path (run_scan_morse_direct / vjp_scan_morse_direct): the config-0 molecule
    with Morse parameters, 100x100 pixels x 40 z-steps, the AFMulator's default probe (radial 4 A
    bond) and FIRE settings; forward and the implicit VJP of a df-like seed, device-resident inputs,
    CUDA events."""
    import torch
    from spammm_b200 import _lib, gpu, synthetic
    from spammm_b200.AFM import AFMulator, N_RELAX_STEP_MAX, F2CONV
    cfg = synthetic.plain_small(kind=1)
    n = len(cfg.scan_xs)
    gx, gy = np.meshgrid(cfg.scan_xs, cfg.scan_ys, indexing="ij")
    dpos0 = AFMulator.DEFAULT_dpos0
    pts = np.zeros((n * n, 4), np.float32)
    pts[:, 0], pts[:, 1], pts[:, 2] = gx.ravel(), gy.ravel(), cfg.z_top - dpos0[2]  # the probe starts at z_top
    tipC = AFMulator.DEFAULT_tipC.copy()
    tipC[3] = -cfg.dz
    P = _lib.make_scan_params(tipA=AFMulator.DEFAULT_tipA, tipB=AFMulator.DEFAULT_tipB, tipC=tipC,
                              stiffness=AFMulator.DEFAULT_stiffness, dpos0=dpos0, relax_params=AFMulator.DEFAULT_relax_pars,
                              surfFF=AFMulator.DEFAULT_surfFF, nz=cfg.nz, raster_ny=n, max_iter=N_RELAX_STEP_MAX,
                              f2conv=F2CONV, fire=True)
    dev = torch.device("cuda", dev_index)
    atoms = torch.from_numpy(cfg.atoms).to(dev)
    cMs = torch.from_numpy(cfg.params).to(dev)
    pts_d = torch.from_numpy(pts).to(dev)
    Qs, QZs = AFMulator.DEFAULT_tipQs, AFMulator.DEFAULT_tipQZs
    for _ in range(max(3, args.warmup)):
        FEs, PPs = gpu.relax_direct_morse(atoms, cMs, pts_d, P, Qs, QZs)
    torch.cuda.synchronize()
    steps = max(3, args.steps)
    e0, e1 = _events()
    e0.record()
    for _ in range(steps):
        FEs, PPs = gpu.relax_direct_morse(atoms, cMs, pts_d, P, Qs, QZs)
    e1.record()
    torch.cuda.synchronize()
    ms_fwd = e0.elapsed_time(e1) / steps
    fire_steps = float(PPs[..., 3].abs().double().sum())
    converged = float((PPs[..., 3] > 0).float().mean())
    # the VJP of a df-like seed (dL/dFz only), the reference's two adjoint passes
    dL = torch.zeros_like(FEs)
    dL[..., 2] = torch.randn(FEs.shape[:2], generator=torch.Generator(device=dev).manual_seed(3), device=dev) * 1e-3
    ok = PPs[..., 3] > 0
    dL[~ok] = 0.0
    PPv = PPs.clone()
    PPv[..., 3] = PPv[..., 3].abs()  # the VJP takes converged states; the few that are not carry a zero seed
    for _ in range(3):
        lam, diag = gpu.adjoint_direct_state(atoms, cMs, pts_d, P, Qs, QZs, PPv, dL)
        grad = gpu.adjoint_direct_params(atoms, cMs, pts_d, P, Qs, QZs, PPv, dL, lam)
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for _ in range(steps):
        lam, diag = gpu.adjoint_direct_state(atoms, cMs, pts_d, P, Qs, QZs, PPv, dL)
        grad = gpu.adjoint_direct_params(atoms, cMs, pts_d, P, Qs, QZs, PPv, dL, lam)
    e1.record()
    torch.cuda.synchronize()
    ms_vjp = e0.elapsed_time(e1) / steps
    na = cfg.atoms.shape[0]
    sites = int(sum(1 for q in Qs if q != 0.0))
    fp32_per, mufu_per = DIRECT_PAIR[0] + sites * DIRECT_SITE[0], DIRECT_PAIR[1] + sites * DIRECT_SITE[1]
    pair_steps = fire_steps * na
    fp32_peak = gpu.fp32_peak_flops(1 << 15)
    lane_rate = pair_steps * fp32_per / (ms_fwd * 1e-3)  # FP32 lane instructions per second
    pxz = n * n * cfg.nz
    return {"workload": f"config-0 molecule ({na} atoms, Morse + {sites} tip-charge sites), {n}x{n} px x {cfg.nz} "
                        "z-steps, the AFMulator's default probe and FIRE (<= 128 steps, |F|^2 < 1e-8), no grid",
            "forward_ms": ms_fwd, "px_z_per_s": pxz / (ms_fwd * 1e-3), "fire_steps_per_state": fire_steps / pxz,
            "converged_frac": converged, "vjp_ms": ms_vjp, "vjp_states_per_s": pxz / (ms_vjp * 1e-3),
            "roofline": {"bound": "fp32 pipe issue (+ MUFU)", "unit": "TFLOP/s",
                         "achieved": 2.0 * lane_rate / 1e12, "peak": fp32_peak / 1e12,
                         "frac": 2.0 * lane_rate / fp32_peak,
                         "algorithmic": f"{pair_steps:.3e} (FIRE step, atom) pairs x {fp32_per} FP32 lane instructions "
                                        f"(+{mufu_per} MUFU) as written; FMA-equivalent x2"}}


# ---------------------------------------------------------------------------- batched path
def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _replay_ms(graph, reps):
    import torch
    e0, e1 = _events()
    e0.record()
    for _ in range(reps):
        graph.replay()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _plain_images_per_s(items, probe):
    """The per-image drop-in path (AFMulator: setup_grid_world, make_forcefield,
    scan_fdbm, compute_df_amp_dir; numpy in/out) on every molecule of the
    batch, one after another, wall clock."""
    import torch
    from spammm_b200 import AFM
    from spammm_b200.AFM import AFMulator

    def one(it):
        afm = AFMulator(use_morse=False)
        afm.n_relax_max, afm.f2conv = probe.max_iter, probe.f2conv
        afm.tipQs, afm.tipQZs = probe.tipQs, probe.tipQZs
        afm.atoms_arr = it.atoms.copy()
        afm.cLJs_arr = it.params.copy()
        afm.setup_grid_world(it.origin, np.array(it.ngrid) * it.step, it.ngrid)
        afm.make_forcefield()
        afm.setup_fdbm_grid_from_img(afm.img_FF, it.ngrid, it.origin, it.step)
        hs = (it.z_top - 0.1 * np.arange(it.nz)[::-1]).astype(np.float32)
        F, _ = afm.scan_fdbm(it.xs, it.ys, hs, mol_z=0.0, bond_length=0.0, stiffness=probe.stiffness,
                             dpos0=probe.dpos0)
        return AFM.compute_df_amp_dir(F, 0.1, (0., 0., 1.), 1.0)

    one(items[0])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for it in items:
        one(it)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return {"images_per_s": len(items) / dt, "ms_per_image": dt / len(items) * 1e3, "molecules": len(items),
            "path": "AFMulator.setup_grid_world/make_forcefield/scan_fdbm + compute_df_amp_dir per molecule "
                    "(numpy in/out), the same molecules as the fit, wall clock"}


def _plain_gpu_ms_per_image(items, probe):
    """GPU time of the per-image path's kernels alone: for every molecule, with its inputs resident on the
    device, the full-grid build, the relaxation (relaxStrokes, the per-image kernels) and the amplitude df,
    back to back on one stream, timed with CUDA events (no host work, no copies)."""
    import torch
    from spammm_b200 import _lib, gpu
    from spammm_b200.AFM import AFMulator
    dev = torch.device("cuda", torch.cuda.current_device())
    work = []
    for it in items:
        L = np.array(it.ngrid) * it.step
        dinv = AFMulator._make_dinv_axis_aligned(L, np.asarray(it.origin, np.float32), it.ngrid)
        P = _lib.make_scan_params(dinv=dinv, dTip=[0, 0, -0.1, 0], stiffness=probe.stiffness, dpos0=probe.dpos0,
                                  relax_params=probe.relax_params, nz=it.nz, max_iter=probe.max_iter,
                                  f2conv=probe.f2conv, flip_z=True, raster_ny=len(it.ys))
        gx, gy = np.meshgrid(it.xs, it.ys, indexing="ij")
        pts = np.zeros((gx.size, 4), np.float32)
        pts[:, 0], pts[:, 1], pts[:, 2] = gx.ravel(), gy.ravel(), it.z_top
        s = it.step
        vec = (np.array([*it.origin, 0], np.float32), np.array([s, 0, 0, 0], np.float32),
               np.array([0, s, 0, 0], np.float32), np.array([0, 0, s, 0], np.float32))
        work.append((it, P, torch.from_numpy(pts).to(dev), torch.from_numpy(it.atoms).to(dev),
                     torch.from_numpy(it.params).to(dev), vec))

    def run():
        for it, P, pts, atoms, prm, (p0, dA, dB, dC) in work:
            grid = gpu.grid_build(0, atoms, prm, it.ngrid, p0, dA, dB, dC, probe.tipQs, probe.tipQZs)
            FEs, _ = gpu.relax_strokes(grid, P, pts)
            gpu.df_amp_dir(FEs.view(len(it.xs), len(it.ys), it.nz, 4), (it.step, it.step, 0.1), (0., 0., 1.), 1.0)

    run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / len(items)


def run_batched(args, dev_index):
    """Many-molecule workloads: (3) forward images of a 512-molecule batch,
    (4) 100 Adam steps of batched forward+adjoint fitting on 64 molecules."""
    import torch
    from spammm_b200 import autotune, synthetic
    from spammm_b200.batch import AFMBatch, BatchAdam
    out = {}
    # ---- (4) fitting: target df from N(0,0.1 A)-perturbed positions; fit starts at the unperturbed structures
    items = synthetic.batch_molecules(args.fit_mols, seed=5, z_end=args.fit_z_end)
    # the per-image drop-in path on the same molecules first, on a device that holds no batch
    from spammm_b200.batch import ProbeSpec
    plain = _plain_images_per_s(items, ProbeSpec())
    plain["gpu_kernel_ms_per_image"] = _plain_gpu_ms_per_image(items, ProbeSpec())
    torch.cuda.empty_cache()
    polish, warm = not args.fit_cold, not args.fit_cold
    if args.no_tune:
        from spammm_b200 import _lib
        shape, tune_rep = _lib.lib().spm_batch_default_shape(), None
    else:
        # the fit (BatchAdam) reads the position and charge gradients only
        shape, tune_rep = autotune.tuned_shape(items, max_molecules=args.fit_mols, reps=2, pair_param_grads=False,
                                               polish=polish, warm=warm)
    rng = np.random.default_rng(11)
    pert = []
    for it in items:
        a = it.atoms.copy()
        a[:, :3] += rng.normal(0.0, 0.1, (len(a), 3)).astype(np.float32)
        pert.append(a)
    from spammm_b200.batch import StreamGroup, molecule_groups
    groups = molecule_groups(len(items), args.fit_groups)
    bs, opts, starts, truths = [], [], [], []
    loss0 = 0.0
    for idx in groups:
        b = AFMBatch([items[i] for i in idx], shape=shape).set_relax_options(polish=polish)
        for j, i in enumerate(idx):
            b.set_atoms(j, pert[i])
        b.forward_adjoint()  # target 0: df_c is the perturbed structures' df
        target = b.df_c.clone()
        b.set_relax_options(warm=warm)
        b.reset_warm_start()
        start = torch.as_tensor(b.plan.atoms, device=b.atoms.device)
        truths.append(b.atoms.clone())
        b.atoms.copy_(start)
        b.set_target_states(target)
        b.enable_failure_mask()
        opt = BatchAdam(b, lr=args.fit_lr, cols=(0, 1, 2, 3))
        b.forward_adjoint()
        loss0 += float(b.loss.sum())
        bs.append(b)
        opts.append(opt)
        starts.append(start)
    sg = StreamGroup([opt.step for opt in opts])
    g = sg.capture()
    for b, opt, start in zip(bs, opts, starts):
        b.atoms.copy_(start)
        opt.reset()
        b.enable_failure_mask()
        b.reset_warm_start()
    clk = ClockSampler(dev_index)
    clk.start()
    e0, e1 = _events()
    e0.record()
    for _ in range(args.fit_steps):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / args.fit_steps
    for b in bs:
        b.forward_adjoint()
    torch.cuda.synchronize()
    atoms = torch.cat([b.atoms for b in bs])
    start, truth = torch.cat(starts), torch.cat(truths)
    n_states = sum(b.total_states for b in bs)

    def rmse(x, y):
        return float(((x[:, :3] - y[:, :3]) ** 2).sum(1).mean().sqrt())
    st = torch.stack([torch.bincount(b.diag[:, 3].long(), minlength=6)[:6] for b in bs]).sum(0).tolist()
    out["fit"] = {
        "workload": f"{args.fit_mols} molecules of the batch distribution, target df from N(0,0.1 A)-perturbed "
                    f"positions, {args.fit_steps} Adam steps (lr {args.fit_lr}) on positions and charges from the "
                    "unperturbed structures, one CUDA-graph replay per step (forward + df loss + adjoint + update)",
        "groups": f"{len(bs)} batches of {'/'.join(str(len(i)) for i in groups)} molecules (dealt round-robin), "
                  "each on its own stream, forked and joined inside the one graph",
        "relax_options": {"newton_polish": polish, "warm_start": warm},
        "ms_per_step": ms, "images_per_s": args.fit_mols / (ms * 1e-3), "states_per_step": n_states,
        "loss_start": loss0, "loss_final": float(sum(float(b.loss.sum()) for b in bs)),
        "rmse_vs_unperturbed_A": rmse(atoms, start), "rmse_vs_target_structure_A": rmse(atoms, truth),
        "rmse_start_vs_target_structure_A": rmse(start, truth), "adjoint_status_counts": st,
        "shape": dict(zip([f for f, _ in type(shape)._fields_], shape.key())), "autotune": tune_rep,
        "clocks": clocks}
    # where a step goes: eager fit steps, the groups one after another on one stream, each stage bracketed by
    # CUDA events and summed over the groups; the first step repeats the final forward's atoms and is not
    # counted, so every counted step relaxes atoms the update moved
    stages = (("grid", "build_grids"), ("relax", "relax"), ("loss", "loss_seed"), ("adjoint_state", "adjoint_state"),
              ("adjoint_params", "adjoint_params"), ("failure_mask", "_update_mask"))
    ev = {k: [] for k, _ in stages + (("step", None),)}

    def timed(key, fn):
        def run():
            e0, e1 = _events()
            e0.record()
            fn()
            e1.record()
            ev[key].append((e0, e1))
        return run

    def eager_step():
        for opt in opts:
            opt.step()
    for b in bs:
        for key, meth in stages:
            setattr(b, meth, timed(key, getattr(b, meth)))  # instance attributes shadow the methods
    try:
        for _ in range(4):
            timed("step", eager_step)()
    finally:
        for b in bs:
            for _, meth in stages:
                delattr(b, meth)
    torch.cuda.synchronize()
    sr = {}
    for k, v in ev.items():
        per = len(v) // 4  # calls per step: one per group, one for the whole step
        ts = [e0.elapsed_time(e1) for e0, e1 in v]
        sr[k] = float(np.median([sum(ts[i * per:(i + 1) * per]) for i in range(1, 4)]))
    # the failure mask runs on a side stream beside adjoint_params: not part of the critical path's sum
    sr["update_and_rest"] = sr["step"] - sum(sr[k] for k, _ in stages if k != "failure_mask")
    out["fit"]["stage_ms"] = sr
    out["fit"]["stage_ms_note"] = ("eager fit steps after an Adam update (median of 3), the groups one after "
                                   "another, each stage between CUDA events and summed over the groups; the failure "
                                   "mask runs on a side stream beside adjoint_params; the graph replay above runs "
                                   "the groups' launches concurrently and without host gaps")
    out["plain_per_image"] = plain
    out["fit"]["vs_plain_per_image"] = out["fit"]["images_per_s"] / out["plain_per_image"]["images_per_s"]
    out["fit"]["vs_plain_gpu_kernels"] = plain["gpu_kernel_ms_per_image"] / (ms / args.fit_mols)
    out["fit"]["fire_steps_per_state_last_step"] = float(sum(float(b.iter_count.double().sum()) for b in bs)) / n_states
    del g, sg, bs, opts, b, opt
    torch.cuda.empty_cache()
    # ---- (3) forward images of a large batch in one graph
    items = synthetic.batch_molecules(args.batch_mols, seed=3)
    from spammm_b200 import _lib
    from spammm_b200.batch import BatchPlan
    plan = BatchPlan(items)
    if tune_rep is not None:  # a cold unpolished relaxation: the tuner's fastest cold shape, not the fit's warm one
        shape = autotune._with(shape, **tune_rep["relax"]["best"])
    need = (4 if shape.grid_layout else 2) * plan.grid_float4 * 16 + plan.total_states * 36
    layout_note = None
    if shape.grid_layout and need > 0.85 * torch.cuda.mem_get_info()[0]:
        shape = _lib.BatchShape(*shape.key())
        shape.grid_layout = 0  # xz-quad slabs would not fit: x-pairs (half the grid memory)
        layout_note = "x-pair slabs (xz-quads exceed the free memory)"
    del plan
    b = AFMBatch(items, shape=shape)
    gf = b.capture(lambda: b.forward(amp=1.0))
    clk = ClockSampler(dev_index)
    clk.start()
    ms = _replay_ms(gf, args.batch_steps)
    clocks = clk.stop()
    out["forward"] = {
        "workload": f"{args.batch_mols} molecules: U{{10..120}} atoms, grids 12-32 A per side at 0.1 A (slabs "
                    f"of the reachable nodes built), 64^2-256^2 px, 30-60 z-steps; grid slabs + relaxation + "
                    "df in one CUDA graph",
        "ms_per_step": ms, "images_per_s": args.batch_mols / (ms * 1e-3), "states": b.total_states,
        "px_z_per_s": b.total_states / (ms * 1e-3), "slab_gb": b.grid_float4 * 16 / 1e9,
        "iters_per_state": float(b.iter_count.double().sum()) / b.total_states,
        "converged_frac": float((b.PPs[:, 3] > 0).float().mean()), "clocks": clocks,
        "gpu_launches_per_step": 3, "grid_layout": "xz-quads" if b.shape.grid_layout else "x-pairs",
        "layout_note": layout_note}
    del gf, b
    torch.cuda.empty_cache()
    return out


def run_reference(args, rank, world):
    """The reference's CPU implementation of the path on the host cores: the reference itself is
    PyOpenCL and neither this image nor the GPU boxes have an OpenCL platform (clGetPlatformIDs
    returns -1001, no ICD under /etc/OpenCL/vendors, no pyopencl), so the arm times the oracle's
    C/OpenMP restatement of its kernels, on every host thread, one bounded proportional sample
    (CpuSample) per step.  Under torchrun only rank 0 runs."""
    if rank != 0:
        return None
    cfg = make_config(args.config)
    cs = CpuSample(cfg)
    for _ in range(args.warmup):
        cs.step()
    cs.stage_s[:] = 0
    cs.steps = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cs.step()
    wall = time.perf_counter() - t0
    value = cs.pxz * args.steps / wall
    det = cs.describe()
    det["value"] = value
    det["unit"] = UNIT
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded NaCl slab + planar molecule)",
            "config": dict(config_dict(cfg, "CPU"), sample=det["sample"]), "impl": "reference",
            "cpu_baseline": det,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's path is PyOpenCL and no OpenCL platform exists on this image or the GPU box "
                    "(probed: no pyopencl, clGetPlatformIDs -1001); this arm times the C/OpenMP restatement of "
                    "its kernels on the host cores, per step a bounded proportional sample of the workload"}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    elif args.batch_only:
        line = None
        if rank == 0:
            line = {"metric": "batched fwd+adjoint images/s", "batched": run_batched(args, local_rank)}
    else:
        if world > 1:
            import datetime
            import torch
            torch.cuda.set_device(local_rank)
            torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        line = run_ours(args, rank, world, local_rank)
        if world > 1:
            import torch
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
