"""Launch-shape autotuner of the batched path.

Every batched stage reads only its own fields of ``spm_batch_shape``:

  grid build   gb_ty (CTA rows: 32 x gb_ty threads), gb_zb (z-nodes per thread)
  relaxation   rx_sync (z-synchronised warp tiles, independent lanes, or -- warm polished fits --
               a Newton-only pass in tiles and a FIRE pass over the strokes it stopped),
               rx_threads (CTA size), rx_tile_h (pixel tile (32/h) x h per warp
               draw), rx_regs (80 / 64 registers, or the register texel cache
               at up to 128, 80 or 102 registers),
               grid_layout (x-pair or xz-quad slabs: the grid is rebuilt in the
               candidate's layout before the relaxation is timed)
  adjoint      adj_chunk (slab nodes per node-major unit), adj_ilp (node pairs
               per step of the node kernel: 1 at 4 CTAs per SM, 2 at 2), adj_agg
               (the scatter: per state, a CTA table, or a tile walk merging the
               nodes neighbouring pixels share), adj_stage (node blocks by bulk
               copies)

so the stages are tuned one after another, each over its own candidates with
the others held fixed, by timing the stage's launch with CUDA events on a
representative sub-batch (every k-th molecule of the work order, so the mix
of sizes is kept).  Results are cached per (device, workload signature) for
the process, and optionally in a JSON file.
"""
import json
import os

import numpy as np
import torch

from . import _lib
from .batch import AFMBatch

GRID_CANDIDATES = [dict(gb_ty=ty, gb_zb=zb) for ty in (2, 4, 8) for zb in (8, 16)]
# z-synchronised warp tiles ran 3x faster than lanes drawing pixels independently on the
# 64-molecule fit (the CTA size made no difference); one independent-lane shape stays as a check
# rx_regs = 5: the z-slab of each warp staged in shared memory by bulk copies (x-pair slabs only)
RELAX_CANDIDATES = [dict(rx_sync=1, rx_threads=128, rx_tile_h=h, rx_regs=r, grid_layout=g) for g in (0, 1)
                    for h in (2, 4, 8, 16) for r in (0, 1, 2, 3, 4)] + \
                   [dict(rx_sync=1, rx_threads=128, rx_tile_h=h, rx_regs=5, grid_layout=0) for h in (2, 4, 8, 16)] + \
                   [dict(rx_sync=0, rx_threads=128, rx_tile_h=8, rx_regs=0, grid_layout=0)]
ADJOINT_CANDIDATES = [dict(adj_chunk=c, adj_ilp=i, adj_agg=a, adj_stage=0) for c in (4096, 16384, 65536)
                      for i in (1, 2, 3) for a in (0, 1, 2)] + \
                     [dict(adj_chunk=c, adj_ilp=1, adj_agg=0, adj_stage=1) for c in (4096, 16384)]

_CACHE = {}


def _with(shape, **kw):
    s = _lib.BatchShape(*shape.key())
    for k, v in kw.items():
        setattr(s, k, int(v))
    return s


def _time(fn, reps):
    fn()
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def _warm_step_ms(batch, reps, sigma=5e-3, seed=0):
    """Time of a warm-started relaxation after the atoms moved by N(0, sigma) A per coordinate (a fit
    step's size): the equilibria of the unmoved atoms are restored before every timed call.  The atoms
    and the previous equilibria are put back afterwards."""
    atoms0 = batch.atoms.clone()
    batch.PPs.fill_(float("nan"))
    batch.build_grids()
    batch.relax()
    pps0 = batch.PPs.clone()
    g = torch.Generator(device=batch.atoms.device).manual_seed(seed)
    batch.atoms[:, :3] += sigma * torch.randn(batch.atoms[:, :3].shape, generator=g, device=batch.atoms.device,
                                              dtype=batch.atoms.dtype)
    batch.build_grids()
    best = float("inf")
    for _ in range(reps + 1):  # the first call warms up
        batch.PPs.copy_(pps0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        batch.relax()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    batch.atoms.copy_(atoms0)
    batch.PPs.fill_(float("nan"))
    batch.build_grids()
    return best


def signature(items, kind):
    """Workload key: molecule count, kind, total atoms / pixels / states."""
    return (len(items), int(kind), int(sum(len(it.atoms) for it in items)), int(sum(it.n_scan for it in items)),
            int(sum(it.n_scan * it.nz for it in items)))


def sub_batch(items, max_molecules):
    """Every k-th molecule in order of relaxation work (the batch's own order)."""
    if len(items) <= max_molecules:
        return list(items)
    cost = np.array([it.n_scan * it.nz for it in items])
    order = np.argsort(-cost, kind="stable")
    pick = order[np.linspace(0, len(items) - 1, max_molecules).round().astype(int)]
    return [items[i] for i in sorted(set(pick.tolist()))]


def tune(batch, reps=2, adjoint=True, log=None, max_grid_bytes=None):
    """Tune batch.shape in place, stage by stage; returns (shape, timings).
    max_grid_bytes: leave out slab layouts whose grid buffer would exceed it.  A batch relaxing
    with the polish or warm starts (set_relax_options) is tuned over the z-synchronised schedules
    only, the ones that support them; the relaxation shapes are timed cold, and with the polish and
    warm starts both the fastest of them are also timed warm after the atoms moved by a fit step's
    size, in the one-pass and the two-pass schedules (rx_sync = 1, 2), which then decides."""
    report = {}
    warm = batch.warm
    batch.set_relax_options(warm=False)
    shape = batch.shape

    def pick(name, cands, run, prepare=None):
        nonlocal shape
        res = []
        for kw in cands:
            s = _with(shape, **kw)
            batch.set_shape(s)
            if prepare is not None:
                prepare()
            ms = _time(run, reps)
            res.append((ms, kw))
            if log:
                log(f"autotune {name} {kw}: {ms:.3f} ms")
        res.sort(key=lambda r: r[0])
        shape = _with(shape, **res[0][1])
        report[name] = {"best": res[0][1], "ms": res[0][0], "worst_ms": res[-1][0], "tried": len(res),
                        "all": [[ms, kw] for ms, kw in res]}

    pick("grid", GRID_CANDIDATES, batch.build_grids)
    batch.set_shape(shape)
    batch.build_grids()
    cands = [c for c in RELAX_CANDIDATES if (c["rx_sync"] == 1 and c["rx_regs"] != 5) or not (batch.polish or warm)]
    if max_grid_bytes is not None:
        cands = [c for c in cands if (4 if c["grid_layout"] else 2) * batch.grid_float4 * 16 <= max_grid_bytes]
    pick("relax", cands, batch.relax, prepare=batch.build_grids)
    warm_pick = {}
    if warm and batch.polish:
        # a fit's later calls: the fastest cold shapes timed warm, each in the one-pass (rx_sync = 1) and the
        # two-pass (rx_sync = 2) schedule; the best shape per slab layout is kept for the layout choice below
        batch.set_relax_options(warm=True)
        tried = []
        first = {}  # the fastest cold shape of each (register variant, slab layout): the warm step weighs
        for ms_cold, kw in report["relax"]["all"]:  # the Newton evaluations, not FIRE, so its order differs
            first.setdefault((kw["rx_regs"], kw["grid_layout"]), (ms_cold, kw))
        for ms_cold, kw in first.values():
            for sync in (1, 2):
                k2 = dict(kw, rx_sync=sync)
                batch.set_shape(_with(shape, **k2))
                ms = _warm_step_ms(batch, reps)
                tried.append((ms, k2))
                if log:
                    log(f"autotune relax (warm step) {k2}: {ms:.3f} ms")
        batch.set_relax_options(warm=False)
        tried.sort(key=lambda r: r[0])
        for ms, kw in tried:
            warm_pick.setdefault(kw["grid_layout"], (ms, kw))
        shape = _with(shape, **tried[0][1])
        report["relax_warm"] = {"best": tried[0][1], "ms": tried[0][0], "all": [[ms, kw] for ms, kw in tried]}
    if adjoint:
        # the slab layout also sets the adjoint's cost: between the best relaxation shape of each layout,
        # keep the one whose relaxation + state adjoint + adjoint through the grid is faster
        best_by_layout = {}
        for ms, kw in report["relax"]["all"]:
            best_by_layout.setdefault(kw["grid_layout"], kw)
        if warm_pick:  # the warm-step timings stand for the relaxation
            best_by_layout = {lay: kw for lay, (ms, kw) in warm_pick.items()}
        if len(best_by_layout) > 1:
            def step():
                batch.relax()
                batch.loss_seed()
                batch.adjoint_state()
                batch.adjoint_params()

            def adjoint_stages():
                batch.loss_seed()
                batch.adjoint_state()
                batch.adjoint_params()
            joint = []
            for lay, kw in sorted(best_by_layout.items()):
                s = _with(shape, **kw)
                batch.set_shape(s)
                batch.build_grids()
                if warm_pick:
                    batch.relax()
                    joint.append((warm_pick[lay][0] + _time(adjoint_stages, reps), kw))
                else:
                    joint.append((_time(step, reps), kw))
                if log:
                    log(f"autotune relax+adjoint, layout {lay} {kw}: {joint[-1][0]:.3f} ms")
            joint.sort(key=lambda r: r[0])
            shape = _with(shape, **joint[0][1])
            report["relax_adjoint_layout"] = {"best": joint[0][1], "all": [[ms, kw] for ms, kw in joint]}
        batch.set_shape(shape)
        batch.build_grids()
        batch.relax()
        batch.loss_seed()
        batch.adjoint_state()
        # the state adjoint before each candidate: a launch shape with another scratch size starts without the
        # maxima the state call leaves there
        pick("adjoint", ADJOINT_CANDIDATES, batch.adjoint_params, prepare=batch.adjoint_state)
    batch.set_shape(shape)
    batch.set_relax_options(warm=warm)
    return shape, report


def tuned_shape(items, kind=0, probe=None, dtip=-0.1, max_molecules=24, reps=2, adjoint=True, cache_file=None,
                log=None, pair_param_grads=True, polish=False, warm=False):
    """Best BatchShape for a workload, tuned on a sub-batch of at most
    max_molecules molecules (cached per device and workload signature).
    pair_param_grads: whether the adjoint is timed with the pair-parameter
    columns (False for fits that read positions and charges only); polish,
    warm: the relaxation options the batch will run with (set_relax_options)."""
    dev = torch.cuda.get_device_name()
    key = json.dumps([dev, signature(items, kind), bool(adjoint), bool(pair_param_grads), bool(polish), bool(warm)])
    if key not in _CACHE and cache_file and os.path.exists(cache_file):
        with open(cache_file) as f:
            _CACHE.update(json.load(f))
    if key in _CACHE:
        return _lib.BatchShape(*_CACHE[key]["shape"]), _CACHE[key]["report"]
    sub = AFMBatch(sub_batch(items, max_molecules), kind=kind, probe=probe, dtip=dtip)
    sub.pair_param_grads = bool(pair_param_grads)
    sub.set_relax_options(polish=polish, warm=warm)
    shape, report = tune(sub, reps=reps, adjoint=adjoint, log=log)
    del sub
    torch.cuda.empty_cache()
    _CACHE[key] = {"shape": list(shape.key()), "report": report}
    if cache_file:
        with open(cache_file, "w") as f:
            json.dump(_CACHE, f, indent=1)
    return shape, report


def _parse_shape(text, base):
    """'rx_regs=5,rx_tile_h=4' -> a BatchShape from base with those fields set."""
    kw = {}
    for part in filter(None, text.split(",")):
        k, _, v = part.partition("=")
        if not hasattr(base, k):
            raise ValueError(f"unknown spm_batch_shape field {k!r}")
        kw[k] = int(v)
    return _with(base, **kw)


def main(argv=None):
    """Time one stage of the batched path under given launch shapes on a
    synthetic batch, or run the tuner:

        python -m spammm_b200.autotune --mols 16 --stage relax \\
            --shape rx_regs=4,rx_tile_h=4 --shape rx_regs=5,rx_tile_h=4

    Each --shape (fields of spm_batch_shape over the library default) builds
    the slabs in its own layout, runs the stage --warmup times untimed and
    --reps times timed with CUDA events, and prints the best time.  Without
    --shape the tuner runs on the batch and prints its report."""
    import argparse
    from . import synthetic
    ap = argparse.ArgumentParser(prog="python -m spammm_b200.autotune")
    ap.add_argument("--mols", type=int, default=16)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--stage", choices=("grid", "relax", "adjoint"), default="relax")
    ap.add_argument("--shape", action="append", default=[])
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--polish", action="store_true")
    ap.add_argument("--positions-charges", action="store_true",
                    help="adjoint stage: gradient columns of positions and charges only (as a fit's steps)")
    ap.add_argument("--warm", action="store_true",
                    help="relax stage: time a warm-started call after the atoms moved by 5e-3 A (implies --polish)")
    args = ap.parse_args(argv)
    if args.warm:
        args.polish = True
    items = synthetic.batch_molecules(args.mols, seed=args.seed)
    base = _lib.lib().spm_batch_default_shape()
    if not args.shape:
        shape, report = tuned_shape(items, max_molecules=args.mols, reps=args.reps, polish=args.polish,
                                    log=lambda s: print(s, flush=True))
        print(json.dumps({"shape": {f[0]: v for f, v in zip(_lib.BatchShape._fields_, shape.key())}, "report": report}))
        return
    rng = np.random.default_rng(args.seed)
    for text in args.shape:
        b = AFMBatch(items, shape=_parse_shape(text, base)).set_relax_options(polish=args.polish)
        b.pair_param_grads = not args.positions_charges
        b.build_grids()
        if args.stage == "relax" and args.warm:
            b.set_relax_options(warm=True)
            ms = _warm_step_ms(b, args.reps)
            n_tail = int(b.workspace[2]) if b.shape.rx_sync == 2 else None
            print(json.dumps({"shape": text, "stage": "relax (warm step)", "ms": ms, "states": int(b.total_states),
                              "strokes": int(b.total_pixels), "second_pass_strokes": n_tail}), flush=True)
            del b
            torch.cuda.empty_cache()
            continue
        if args.stage == "grid":
            run = b.build_grids
        elif args.stage == "relax":
            run = b.relax
        else:
            for i, it in enumerate(b.items):
                b.set_target(i, rng.normal(0.0, 0.05, (len(it.xs), len(it.ys), it.nz)))
            b.relax()
            b.loss_seed()
            b.adjoint_state()
            run = b.adjoint_params
        for _ in range(args.warmup):
            run()
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(args.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            run()
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        print(json.dumps({"shape": text, "stage": args.stage, "ms": best, "states": int(b.total_states),
                          "slab_bytes": int(b.grid.numel()) * 4}), flush=True)
        del b
        torch.cuda.empty_cache()


if __name__ == "__main__":
    main()
