"""Batched grid path on the GPU: every molecule of a batch against the
per-molecule calls (bit-exact forward, loss and state adjoint; gradients to
FP64 summation order), the CPU oracle, CUDA-graph replay and launch shapes."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as O
from spammm_b200 import _lib, gpu, synthetic
from spammm_b200.batch import AFMBatch, BatchAdam, ProbeSpec

pytestmark = pytest.mark.gpu


def _items(kind=0, n=6, seed=21):
    return synthetic.batch_molecules(n, seed=seed, kind=kind, natoms=(10, 40), side=(5, 9), zside=(8, 14),
                                     npx=(6, 22), nzs=(8, 16))


def _per_molecule(batch, i):
    """The unbatched path for molecule i: full grid, relax_pp."""
    it = batch.items[i]
    spec = it.spec(batch.kind, batch.probe, batch.dtip)
    p0, dA, dB, dC = spec.vectors()
    grid = gpu.grid_build(batch.kind, it.atoms.astype(np.float32), it.params.astype(np.float32), spec.ngrid, p0, dA,
                          dB, dC, spec.tipQs, spec.tipQZs)
    P = spec.scan_params(batch.probe.stiffness)
    pts = torch.as_tensor(spec.points, device="cuda")
    FEs, PPs = gpu.relax_pp(grid, P, pts)
    return spec, grid, P, pts, FEs, PPs


def _target(batch, seed=4):
    rng = np.random.default_rng(seed)
    for i, it in enumerate(batch.items):
        batch.set_target(i, rng.normal(0.0, 0.05, (len(it.xs), len(it.ys), it.nz)))


@pytest.mark.parametrize("kind", [0, 1])
def test_batch_forward_matches_per_molecule(cuda, kind):
    b = AFMBatch(_items(kind), kind=kind)
    b.forward(amp=1.0)
    torch.cuda.synchronize()
    for i, it in enumerate(b.items):
        spec, grid, P, pts, FEs, PPs = _per_molecule(b, i)
        D = b.desc(i)
        full = b.slab_of_full(i, grid)
        assert torch.equal(b.slab(i), full), f"molecule {i}: slab differs from full grid"
        assert torch.equal(b.slab(i, 1), torch.roll(full, -1, dims=2)), f"molecule {i}: x-pair halves differ"
        assert (b.pps(i)[..., 3] > 0).all(), f"molecule {i}: a stroke left the slab or did not converge"
        assert torch.equal(b.fes(i), FEs) and torch.equal(b.pps(i), PPs), f"molecule {i}: relaxation differs"
        # df of the stroke, ascending z (dr = |dtip|), as the single-volume call
        vol = FEs.view(it.n_scan, 1, it.nz, 4).flip(2).contiguous()
        df = gpu.df_amp_dir(vol, abs(b.dtip), (0., 0., 1.), 1.0).flip(2).reshape(len(it.xs), len(it.ys), it.nz)
        assert torch.equal(b.df_image(i), df), f"molecule {i}: df differs"


def test_batch_slab_box_spanning_an_axis(cuda):
    """A box that spans an axis keeps that axis' periodic wrap (the x-pair
    neighbour of the last column is column 0); a box cut to the window on
    another axis stores only those rows.  Both give the full grid's nodes and
    relaxation bit for bit."""
    import dataclasses
    items = _items(0, n=3, seed=95)
    it = items[0]
    cell = it.ngrid[0] * it.step
    xs = (float(it.origin[0]) + (np.arange(24) + 0.5) * cell / 24).astype(np.float32)  # the whole cell in x
    items[0] = dataclasses.replace(it, xs=xs, ys=it.ys[:max(2, len(it.ys) // 3)])
    b = AFMBatch(items)
    D = b.desc(0)
    assert (D.x_lo, D.nx_slab) == (0, D.nx) and D.ny_slab < D.ny
    b.forward()
    torch.cuda.synchronize()
    for i in range(len(items)):
        spec, grid, P, pts, FEs, PPs = _per_molecule(b, i)
        full = b.slab_of_full(i, grid)
        assert torch.equal(b.slab(i), full) and torch.equal(b.slab(i, 1), torch.roll(full, -1, dims=2)), i
        assert torch.equal(b.fes(i), FEs) and torch.equal(b.pps(i), PPs), i
    assert torch.equal(b.slab(0, 1)[:, :, -1], b.slab(0)[:, :, 0])  # the wrap across the periodic seam


def test_batch_relax_matches_oracle(cuda):
    b = AFMBatch(_items(0, n=3, seed=8))
    b.forward()
    torch.cuda.synchronize()
    for i, it in enumerate(b.items):
        spec, grid, P, pts, FEs, PPs = _per_molecule(b, i)
        oFE, oPP = O.relax_pp(grid.cpu().numpy(), spec.dinv(), spec.points, spec.nz, [1, 0, 0, 0], [0, 1, 0, 0],
                              [0, 0, 1, spec.dtip], b.probe.stiffness, spec.dpos0, spec.relax_params, [0, 0, 0, 0],
                              spec.max_iter, spec.f2conv, True)
        assert np.array_equal(b.fes(i).cpu().numpy(), oFE) and np.array_equal(b.pps(i).cpu().numpy(), oPP)


@pytest.mark.parametrize("kind", [0, 1])
def test_batch_loss_and_adjoint_match_per_molecule(cuda, kind):
    b = AFMBatch(_items(kind, seed=33 + kind), kind=kind)
    _target(b)
    b.forward_adjoint()
    torch.cuda.synchronize()
    dk_total = torch.zeros(4, dtype=torch.float64, device="cuda")
    for i, it in enumerate(b.items):
        spec, grid, P, pts, FEs, PPs = _per_molecule(b, i)
        a, c = b._rows(i, "state")
        tgt = b.target[a:c].view(it.n_scan, 1, it.nz)
        loss, df, dL = gpu.df_loss_seed(FEs.view(it.n_scan, 1, it.nz, 4), tgt, b.dtip)
        assert torch.equal(b.loss_of(i).reshape(1), loss)
        assert torch.equal(b.df_c[a:c], df.reshape(-1)) and torch.equal(b.dL[a:c], dL.reshape(-1, 4))
        ubar, dk, diag = gpu.adjoint_grid_state(grid, P, pts, PPs, dL.reshape(it.n_scan, it.nz, 4))
        assert torch.equal(b.ubar[a:c], ubar) and torch.equal(b.dk[a:c], dk) and torch.equal(b.diag[a:c], diag)
        p0, dA, dB, dC = spec.vectors()
        grad, dks = gpu.adjoint_grid_params(kind, it.atoms.astype(np.float32), it.params.astype(np.float32), p0, dA,
                                            dB, dC, spec.tipQs, spec.tipQZs, grid, P, PPs, ubar, dk)
        # node-major (MUFU rsqrt, FP32 pair terms) vs state-major (IEEE, FP64 per pair) sums
        torch.testing.assert_close(b.grad_of(i), grad, rtol=1e-4, atol=1e-5 * float(grad.abs().max()))
        dk_total += dks
    torch.testing.assert_close(b.dk_sum, dk_total, rtol=1e-9, atol=1e-14)


def test_batch_shapes_give_same_results(cuda):
    items = _items(0, n=5, seed=41)
    ref = AFMBatch(items)
    _target(ref)
    ref.forward_adjoint()
    L = _lib.lib()
    for kw in (dict(gb_ty=2, gb_zb=16, rx_threads=64, rx_tile_h=1, adj_chunk=1024, rx_sync=0, rx_regs=0),
               dict(gb_ty=8, gb_zb=8, rx_threads=256, rx_tile_h=32, rx_ctas_per_sm=1, adj_chunk=65536, rx_regs=1,
                    rx_sync=0),
               dict(rx_threads=128, rx_tile_h=4, rx_regs=2, rx_sync=0),
               dict(grid_layout=1, rx_sync=0), dict(grid_layout=1, rx_regs=2), dict(grid_layout=1, rx_regs=1, gb_zb=16),
               dict(rx_sync=1, rx_regs=0), dict(rx_sync=1, rx_tile_h=1, rx_threads=64, rx_regs=2),
               dict(rx_sync=1, rx_tile_h=32, rx_regs=1, grid_layout=1), dict(rx_regs=3, rx_tile_h=2),
               dict(rx_sync=0, rx_regs=3, grid_layout=1), dict(adj_ilp=2), dict(adj_ilp=2, adj_chunk=4096), dict(rx_sync=2),
               dict(adj_ilp=3), dict(adj_ilp=3, adj_chunk=4096),
               dict(rx_regs=3), dict(rx_regs=4, grid_layout=1), dict(rx_sync=0, rx_regs=4, rx_tile_h=4)):
        s = L.spm_batch_default_shape()
        for k, v in kw.items():
            setattr(s, k, v)
        b = AFMBatch(items, shape=s)
        b.set_target_states(ref.target)
        b.forward_adjoint()
        torch.cuda.synchronize()
        for i in range(len(items)):
            assert torch.equal(b.slab(i), ref.slab(i)), (kw, i)
            if b.shape.grid_layout == 1:  # xz-quads: the (x+1), (z+1), (x+1,z+1) neighbours
                full = ref.slab(i)
                assert torch.equal(b.slab(i, 1), torch.roll(full, -1, dims=2))
                assert torch.equal(b.slab(i, 2), torch.roll(full, -1, dims=0))
                assert torch.equal(b.slab(i, 3), torch.roll(full, (-1, -1), dims=(0, 2)))
        assert torch.equal(b.FEs, ref.FEs) and torch.equal(b.PPs, ref.PPs)
        assert torch.equal(b.loss, ref.loss) and torch.equal(b.ubar, ref.ubar)
        # adj_chunk regroups the staged nodes into other FP32 partial sums (FP64 across them)
        torch.testing.assert_close(b.grad, ref.grad, rtol=1e-5, atol=1e-6 * float(ref.grad.abs().max()))


def test_batch_graph_replay(cuda):
    b = AFMBatch(_items(0, n=4, seed=51))
    _target(b)
    b.forward_adjoint()
    torch.cuda.synchronize()
    eager = [t.clone() for t in (b.FEs, b.PPs, b.loss, b.grad)]
    g = b.capture(b.forward_adjoint)
    for t in (b.FEs, b.PPs, b.loss, b.grad, b.grid):
        t.zero_()
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    for e, t in zip(eager, (b.FEs, b.PPs, b.loss, b.grad)):
        assert torch.equal(e, t)


def test_failure_mask_kernel(cuda):
    """spm_batch_failure_mask = w_base * (status of s-1, s, s+1 all 0), cyclic."""
    n = 100003
    g = torch.Generator(device="cuda").manual_seed(3)
    diag = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    diag[:, 3] = (torch.rand(n, device="cuda", generator=g) < 0.05).float() * 3.0
    diag[0, 3] = 1.0  # a failure at the array's start masks the last state too
    w_base = torch.rand(n, dtype=torch.float64, device="cuda", generator=g)
    out = torch.empty_like(w_base)
    _lib.check(_lib.lib().spm_batch_failure_mask(n, _lib.ptr(diag), _lib.ptr(w_base), _lib.ptr(out),
                                                 _lib.stream_ptr()), "spm_batch_failure_mask")
    ok = diag[:, 3] == 0
    ok = ok & torch.roll(ok, 1) & torch.roll(ok, -1)
    assert torch.equal(out, w_base * ok) and out[-1] == 0.0


@pytest.mark.parametrize("sync", [0, 1])
def test_batch_unrastered_molecule(cuda, sync):
    """A molecule whose points are no full raster (raster_ny = 0) is relaxed in
    runs of 32 consecutive pixels, under both schedules; results equal the
    per-molecule path bit for bit."""
    items = _items(0, n=3, seed=91)
    s = _lib.lib().spm_batch_default_shape()
    s.rx_sync = sync
    b = AFMBatch(items, shape=s)
    b.plan.desc(1).raster_ny = 0
    b.set_shape(s)
    assert b.desc(1).raster_ny == 0
    b.forward()
    torch.cuda.synchronize()
    for i in range(len(items)):
        spec, grid, P, pts, FEs, PPs = _per_molecule(b, i)
        assert torch.equal(b.fes(i), FEs) and torch.equal(b.pps(i), PPs), i


def test_batch_with_empty_scan(cuda):
    """A molecule with no pixels contributes nothing: its loss and gradient are
    zero and the others' results are those of a batch without it."""
    import dataclasses
    items = _items(0, n=3, seed=93)
    empty = dataclasses.replace(items[1], xs=items[1].xs[:0], ys=items[1].ys[:0])
    b = AFMBatch([items[0], empty, items[2]])
    ref = AFMBatch([items[0], items[2]])
    rng = np.random.default_rng(5)
    t0, t2 = (rng.normal(0.0, 0.05, (len(it.xs), len(it.ys), it.nz)) for it in (items[0], items[2]))
    b.set_target(0, t0)
    b.set_target(2, t2)
    b.set_target(1, np.zeros((0, 0, empty.nz)))
    ref.set_target(0, t0)
    ref.set_target(1, t2)
    b.forward_adjoint()
    ref.forward_adjoint()
    torch.cuda.synchronize()
    for i, r in ((0, 0), (2, 1)):
        assert torch.equal(b.fes(i), ref.fes(r)) and torch.equal(b.loss_of(i), ref.loss_of(r))
        torch.testing.assert_close(b.grad_of(i), ref.grad_of(r), rtol=1e-5,
                                   atol=1e-6 * float(ref.grad.abs().max()))
    assert float(b.loss_of(1)) == 0.0 and not b.grad_of(1).any()


def test_batch_of_single_chunk_molecules(cuda):
    """Molecules of at most one 256-state loss chunk each, so one CTA of the
    loss and ubar-maxima kernels spans several molecules: every molecule's
    loss equals its batch-of-one loss bit for bit, its gradient to rounding."""
    items = synthetic.batch_molecules(11, seed=61, natoms=(6, 14), side=(5, 7), zside=(8, 10), npx=(2, 4),
                                      nzs=(8, 12))
    assert all(it.n_scan * it.nz <= 256 for it in items)
    rng = np.random.default_rng(8)
    tg = [rng.normal(0.0, 0.05, (len(it.xs), len(it.ys), it.nz)) for it in items]
    b = AFMBatch(items)
    for i in range(len(items)):
        b.set_target(i, tg[i])
    b.forward_adjoint()
    for i, it in enumerate(items):
        one = AFMBatch([it])
        one.set_target(0, tg[i])
        one.forward_adjoint()
        torch.cuda.synchronize()
        assert torch.equal(b.loss_of(i), one.loss_of(0)), i
        torch.testing.assert_close(b.grad_of(i), one.grad_of(0), rtol=1e-5,
                                   atol=1e-6 * float(one.grad.abs().max()))


@pytest.mark.parametrize("kind", [0, 1])
def test_adjoint_scratch_reuse_and_garbage(cuda, kind):
    """The node kernel leaves the adjoint grid cleared for the next call; a
    scratch buffer of arbitrary content (no clear marker) is cleared first.
    The ubar maxima come from the state adjoint (SPM_ADJ_STATE_MAXIMA) or, without it, from the params
    call itself: the same gradients."""
    b = AFMBatch(_items(kind, n=4, seed=71 + kind), kind=kind)
    _target(b)
    b.forward_adjoint()
    torch.cuda.synchronize()
    g1 = b.grad.clone()
    b.adjoint_params()
    torch.cuda.synchronize()
    assert torch.equal(b.grad, g1)
    for fill in ("random", "zero"):  # all-zero buffer: no marker either
        if fill == "random":
            b.adj_scratch.view(torch.uint8).random_(0, 256)
        else:
            b.adj_scratch.view(torch.uint8).fill_(0)
        b._state_maxima = False  # the maxima were overwritten: the params call computes them
        b.adjoint_params()
        torch.cuda.synchronize()
        assert torch.equal(b.grad, g1), fill
        b.adj_scratch.view(torch.uint8).random_(0, 256)
        b.adjoint_state()  # maxima from the state adjoint, the adjoint grid left as garbage
        b.adjoint_params()
        torch.cuda.synchronize()
        assert torch.equal(b.grad, g1), fill
    # garbage under the clear marker of another buffer with the same layout (memory handed out again can
    # hold one exactly where this buffer's marker sits): the marker is the buffer's own, so it is cleared
    other = AFMBatch(_items(kind, n=4, seed=71 + kind), kind=kind)
    _target(other)
    other.forward_adjoint()
    torch.cuda.synchronize()
    at = _adj_mark_offset(b) // 8
    assert at == _adj_mark_offset(other) // 8
    b.adj_scratch.view(torch.uint8).random_(0, 256)
    b.adj_scratch.view(torch.int64).reshape(-1)[at] = other.adj_scratch.view(torch.int64).reshape(-1)[at]
    b._state_maxima = False
    b.adjoint_params()
    torch.cuda.synchronize()
    assert torch.equal(b.grad, g1)
    # a new scratch in memory that held this one (same address and layout, so its own marker) and was written
    # by other tensors since: AFMBatch zero-fills a new scratch
    torch.cuda.synchronize()
    clean = b.adj_scratch.view(torch.int64).reshape(-1)[at].clone()
    nbytes = b.adj_scratch.numel() * 8
    b.adj_scratch = None
    junk = torch.empty((nbytes,), dtype=torch.uint8, device="cuda").random_(0, 256)
    junk.view(torch.int64)[at] = clean
    del junk
    b._ensure_adj_scratch()
    b._state_maxima = False
    b.adjoint_params()
    torch.cuda.synchronize()
    assert torch.equal(b.grad, g1)


@pytest.mark.parametrize("kind", [0, 1])
def test_adjoint_without_pair_parameter_columns(cuda, kind):
    """Without SPM_ADJ_PAIR_PARAMS the node kernel drops the pair-parameter
    terms: columns 3-4 are 0, the position and charge columns are the full
    adjoint's bit for bit (their arithmetic is the same)."""
    b = AFMBatch(_items(kind, n=4, seed=73 + kind), kind=kind)
    _target(b)
    b.forward_adjoint()
    torch.cuda.synchronize()
    full = b.grad.clone()
    assert full[:, 3:5].abs().max() > 0
    b.pair_param_grads = False
    b.adjoint_params()
    torch.cuda.synchronize()
    assert torch.equal(b.grad[:, [0, 1, 2, 5]], full[:, [0, 1, 2, 5]])
    assert not b.grad[:, 3:5].any()
    with pytest.raises(ValueError):
        _lib.check(_lib.lib().spm_batch_adjoint_params(b.kind, b.n, _lib.ptr(b.mols_d), b.plan.totals,
                                                       ctypes.byref(b.shape), _lib.ptr(b.atoms), _lib.ptr(b.params),
                                                       _lib.hptr(b._Qs), _lib.hptr(b._QZs), _lib.ptr(b.PPs),
                                                       _lib.ptr(b.ubar), _lib.ptr(b.dk), _lib.ptr(b.grad),
                                                       _lib.ptr(b.dk_sum), 4, _lib.ptr(b.adj_scratch),
                                                       _lib.stream_ptr()), "spm_batch_adjoint_params")
    # without the spring terms (dk NULL in both calls): the same gradient, dk_sum = 0, dk left untouched
    dk_sum = b.dk_sum.clone()
    assert dk_sum.abs().max() > 0
    b.dk.fill_(7.0)
    b.stiffness_grads = False
    b.adjoint_state()
    b.adjoint_params()
    torch.cuda.synchronize()
    assert torch.equal(b.grad[:, [0, 1, 2, 5]], full[:, [0, 1, 2, 5]])
    assert not b.dk_sum.any() and bool((b.dk == 7.0).all())
    b.stiffness_grads = True
    b.adjoint_state()
    b.adjoint_params()
    torch.cuda.synchronize()
    assert torch.equal(b.dk_sum, dk_sum)


def test_batch_adam_reduces_loss(cuda):
    items = _items(0, n=4, seed=61)
    truth = AFMBatch(items)
    truth.forward_adjoint()  # target 0: df_c is the df image of the true structures
    b = AFMBatch(items)
    b.set_target_states(truth.df_c)
    rng = np.random.default_rng(2)
    for i, it in enumerate(items):
        a = it.atoms.copy()
        a[:, :3] += rng.normal(0.0, 0.05, (len(a), 3)).astype(np.float32)
        b.set_atoms(i, a)
    opt = BatchAdam(b, lr=0.005, cols=(0, 1, 2))
    b.forward_adjoint()
    loss0 = b.loss.clone()
    g = b.capture(opt.step, warmup=0)
    for _ in range(15):
        g.replay()
    b.forward_adjoint()
    torch.cuda.synchronize()
    assert torch.isfinite(b.loss).all()
    assert float(b.loss.sum()) < float(loss0.sum())


def test_batch_adam_graph_with_failure_mask_equals_eager(cuda):
    """With the failure mask on, a fitting step runs the mask beside the parameter adjoint on a side
    stream; a captured step replayed equals the same steps run eagerly bit for bit (atoms, the moment
    buffers and the next step's loss weights)."""
    items = _items(0, n=4, seed=64)
    truth = AFMBatch(items)
    truth.forward_adjoint()
    rng = np.random.default_rng(9)
    moved = [it.atoms.copy() for it in items]
    for a in moved:
        a[:, :3] += rng.normal(0.0, 0.05, (len(a), 3)).astype(np.float32)
    runs = []
    for graph in (False, True):
        b = AFMBatch(items).set_relax_options(polish=True, warm=True)
        b.set_target_states(truth.df_c)
        for i, a in enumerate(moved):
            b.set_atoms(i, a)
        b.enable_failure_mask()
        opt = BatchAdam(b, lr=0.005, cols=(0, 1, 2, 3))
        if graph:
            g = b.capture(opt.step, warmup=0)
            b.reset_warm_start()
            b.atoms.copy_(torch.as_tensor(b.plan.atoms, device="cuda"))
            for i, a in enumerate(moved):
                b.set_atoms(i, a)
            opt.reset()
            b.enable_failure_mask()  # a second call resets the weights in place
            for _ in range(4):
                g.replay()
        else:
            for _ in range(4):
                opt.step()
        torch.cuda.synchronize()
        runs.append((b.atoms.clone(), opt.m.clone(), b.weights.clone(), b.loss.clone()))
    for x, y in zip(*runs):
        assert torch.equal(x, y)


def test_stream_group_fit_equals_groups_run_one_after_another(cuda):
    """Fitting steps of two molecule groups captured on two streams in one graph equal the same
    groups' steps run eagerly one after another bit for bit (atoms, moments, next weights, losses);
    the first step's per-molecule losses equal those of one batch over all the molecules."""
    from spammm_b200.batch import StreamGroup, molecule_groups
    items = _items(0, n=5, seed=66)
    truth = AFMBatch(items)
    truth.forward_adjoint()
    rng = np.random.default_rng(12)
    moved = [it.atoms.copy() for it in items]
    for a in moved:
        a[:, :3] += rng.normal(0.0, 0.05, (len(a), 3)).astype(np.float32)
    groups = molecule_groups(len(items), 2)
    assert groups == [[0, 2, 4], [1, 3]]

    def setup(b, idx):
        b.set_relax_options(polish=True, warm=True)
        for j, i in enumerate(idx):
            lo, hi = truth._rows(i, "state")
            b.set_target(j, truth.df_c[lo:hi])
            b.set_atoms(j, moved[i])
        b.enable_failure_mask()
    whole = AFMBatch(items)
    setup(whole, list(range(len(items))))
    whole.forward_adjoint()
    runs = []
    for graph in (False, True):
        parts = [AFMBatch([items[i] for i in idx]) for idx in groups]
        for b, idx in zip(parts, groups):
            setup(b, idx)
        opts = [BatchAdam(b, lr=0.005, cols=(0, 1, 2, 3)) for b in parts]
        sg = StreamGroup([o.step for o in opts])
        if graph:
            g = sg.capture()
            for b, o, idx in zip(parts, opts, groups):
                b.reset_warm_start()
                setup(b, idx)  # a second enable_failure_mask resets the weights in place
                o.reset()
        first = None
        for k in range(3):
            if graph:
                g.replay()
            else:
                for o in opts:
                    o.step()
            if k == 0:
                torch.cuda.synchronize()
                first = [[b.loss_of(j).clone() for j in range(len(idx))] for b, idx in zip(parts, groups)]
        torch.cuda.synchronize()
        for ls, idx in zip(first, groups):
            for l0, i in zip(ls, idx):
                assert torch.equal(l0, whole.loss_of(i)), (i, graph)
        runs.append([(b.atoms.clone(), o.m.clone(), b.weights.clone(), b.loss.clone()) for b, o in zip(parts, opts)])
    for pa, pb in zip(*runs):
        for x, y in zip(pa, pb):
            assert torch.equal(x, y)


def test_autotune_returns_valid_shape(cuda):
    from spammm_b200 import autotune
    items = _items(0, n=5, seed=71)
    shape, report = autotune.tuned_shape(items, max_molecules=3, reps=1)
    assert {"grid", "relax", "adjoint"} <= set(report) <= {"grid", "relax", "adjoint", "relax_adjoint_layout"}
    ref = AFMBatch(items)
    ref.forward()
    b = AFMBatch(items, shape=shape)
    b.forward()
    torch.cuda.synchronize()
    assert torch.equal(ref.FEs, b.FEs) and torch.equal(ref.PPs, b.PPs)


def test_batch_polished_relaxation_matches_per_molecule(cuda):
    """SPM_FLAG_POLISH in the batched (z-synchronised) relaxation: every molecule bit-identical to the
    per-molecule relax_pp with the polish, for both slab layouts and both register variants of the default
    tile shape; the polish moves the equilibria and lowers the residual."""
    items = _items(0, n=4, seed=61)
    base = _lib.lib().spm_batch_default_shape()
    for layout, regs in ((0, 4), (1, 2), (0, 0)):
        shape = _lib.BatchShape(*base.key())
        shape.grid_layout, shape.rx_regs, shape.rx_sync = layout, regs, 1
        b = AFMBatch(items, shape=shape).set_relax_options(polish=True)
        b.forward()
        torch.cuda.synchronize()
        for i, it in enumerate(b.items):
            spec = it.spec(b.kind, b.probe, b.dtip)
            spec.polish = True
            p0, dA, dB, dC = spec.vectors()
            grid = gpu.grid_build(b.kind, it.atoms.astype(np.float32), it.params.astype(np.float32), spec.ngrid, p0,
                                  dA, dB, dC, spec.tipQs, spec.tipQZs)
            P = spec.scan_params(b.probe.stiffness)
            FEs, PPs = gpu.relax_pp(grid, P, torch.as_tensor(spec.points, device="cuda"))
            assert torch.equal(b.fes(i), FEs) and torch.equal(b.pps(i), PPs), (layout, regs, i)


def test_batch_warm_start_reaches_the_cold_equilibria(cuda):
    """SPM_FLAG_WARM with the polish: after the atoms move by ~5e-3 A (an Adam step of the fit is <= 0.01 A),
    a relaxation started from the previous equilibria reaches the equilibria of a cold start to the float32
    floor, in fewer FIRE steps; a warm start with no previous equilibria (NaN) is the cold relaxation."""
    items = _items(0, n=4, seed=62)
    b = AFMBatch(items).set_relax_options(polish=True, warm=True)
    b.forward()  # PPs NaN: every state starts from its stroke
    cold = AFMBatch(items).set_relax_options(polish=True)
    cold.forward()
    torch.cuda.synchronize()
    assert torch.equal(b.PPs, cold.PPs) and torch.equal(b.FEs, cold.FEs)
    it_cold0 = int(cold.iter_count.sum())
    rng = np.random.default_rng(3)
    moved = b.atoms.clone()
    moved[:, :3] += torch.as_tensor(rng.normal(0, 5e-3, (b.total_atoms, 3)), dtype=moved.dtype, device="cuda")
    b.atoms.copy_(moved)
    cold.atoms.copy_(moved)
    b.forward()
    cold.forward()
    torch.cuda.synchronize()
    ok = (b.PPs[:, 3] > 0) & (cold.PPs[:, 3] > 0)
    assert float(ok.float().mean()) > 0.99
    dq = (b.PPs[ok, :3] - cold.PPs[ok, :3]).abs().max(dim=1).values
    print(f"\nwarm vs cold polished equilibria: max |dq| {float(dq.max()):.2e} A, 99.9% below "
          f"{float(torch.quantile(dq.float(), 0.999)):.2e} A; FIRE steps warm {int(b.iter_count.sum())} vs cold "
          f"{int(cold.iter_count.sum())} (first cold {it_cold0})")
    assert float(torch.quantile(dq.float(), 0.999)) < 1e-4
    assert int(b.iter_count.sum()) < 0.6 * int(cold.iter_count.sum())
    b.reset_warm_start()
    assert bool(torch.isnan(b.PPs).all())


@pytest.mark.parametrize("kind", [0, 1])
def test_batch_two_pass_schedule_is_bit_identical(cuda, kind):
    """rx_sync = 2 (warm polished calls): the Newton-only prefix pass in z-synchronised tiles, then the FIRE
    pass over the strokes that stopped, gives the one-pass schedule's FEs, PPs and step counts bit for bit --
    on the cold first call (every stroke goes to the second pass at its first z-step) and after the atoms
    move (strokes stop part-way down, at z-steps that need FIRE); LJ and Morse grids."""
    items = _items(kind, n=5, seed=66)
    base = _lib.lib().spm_batch_default_shape()
    mid_stroke = 0
    for layout, regs in ((0, 4), (1, 2), (0, 0)):
        shapes = []
        for sync in (1, 2):
            sh = _lib.BatchShape(*base.key())
            sh.grid_layout, sh.rx_regs, sh.rx_sync = layout, regs, sync
            shapes.append(sh)
        one = AFMBatch(items, kind=kind, shape=shapes[0]).set_relax_options(polish=True, warm=True)
        two = AFMBatch(items, kind=kind, shape=shapes[1]).set_relax_options(polish=True, warm=True)
        rng = np.random.default_rng(7)
        for step, sigma in enumerate((0.0, 5e-3, 5e-3, 0.1, 5e-3, 0.3, 0.5)):
            if sigma:
                d = torch.as_tensor(rng.normal(0, sigma, (one.total_atoms, 3)), dtype=one.atoms.dtype, device="cuda")
                one.atoms[:, :3] += d
                two.atoms[:, :3] += d
            one.forward()
            two.forward()
            torch.cuda.synchronize()
            assert torch.equal(one.FEs, two.FEs) and torch.equal(one.PPs, two.PPs), (layout, regs, step)
            assert torch.equal(one.iter_count, two.iter_count), (layout, regs, step)
            ws = two.workspace.cpu().numpy()
            n_tail = int(ws[2])
            if step == 0:
                assert n_tail == two.total_pixels  # no previous equilibria: every stroke from its first z-step
            else:
                assert n_tail < two.total_pixels
                iz = ws[4:4 + 12 * n_tail].reshape(-1, 12)[:, 2]
                mid_stroke += int((iz > 0).sum())
            print(f"layout {layout} regs {regs} call {step}: {n_tail} of {two.total_pixels} strokes in the FIRE pass")
    if kind == 0:  # the LJ batch has strokes that stop part-way down (the Morse case checks the same identity)
        assert mid_stroke > 0


def test_batch_polish_and_warm_need_the_synchronised_schedule(cuda):
    items = _items(0, n=2, seed=63)
    shape = _lib.BatchShape(*_lib.lib().spm_batch_default_shape().key())
    shape.rx_sync = 0
    b = AFMBatch(items, shape=shape).set_relax_options(polish=True)
    b.build_grids()
    with pytest.raises((ValueError, RuntimeError), match="rx_sync"):
        b.relax()


def test_batch_staged_relaxation_is_bit_identical(cuda):
    """rx_regs = 5: each warp's z-slab staged in shared memory by bulk copies; every tile shape gives the
    default kernel's FEs, PPs and step counts bit for bit, and no staging wait timed out."""
    items = _items(0, n=5, seed=64)
    base = _lib.lib().spm_batch_default_shape()
    ref = AFMBatch(items)
    ref.forward()
    for h in (2, 4, 8, 16):
        shape = _lib.BatchShape(*base.key())
        shape.rx_regs, shape.grid_layout, shape.rx_sync, shape.rx_threads, shape.rx_tile_h = 5, 0, 1, 128, h
        b = AFMBatch(items, shape=shape)
        b.forward()
        torch.cuda.synchronize()
        assert torch.equal(b.FEs, ref.FEs) and torch.equal(b.PPs, ref.PPs), h
        assert torch.equal(b.iter_count, ref.iter_count), h
        assert int(b.workspace[1]) == 0, "a staging wait timed out"


def test_batch_adjoint_bulk_staged_node_blocks(cuda):
    """adj_stage = 1: the node kernel fetches each block of adjoint-grid nodes by a bulk copy into
    shared memory.  The same pair terms; blocks of 256 instead of 512 nodes put the non-zero nodes in
    another order within a compute phase, so the FP32 partial sums round differently: within 1e-6 of
    the plain-load kernel's gradients (relative to the largest), and repeatable call after call."""
    items = _items(0, n=5, seed=67)
    out = []
    for stage in (0, 1):
        shape = _lib.BatchShape(*_lib.lib().spm_batch_default_shape().key())
        shape.adj_stage = stage
        b = AFMBatch(items, shape=shape)
        _target(b)
        b.forward_adjoint()
        g1 = b.grad.clone()
        b.adjoint_params()
        torch.cuda.synchronize()
        assert torch.equal(g1, b.grad)
        out.append(g1)
    scale = float(out[0].abs().max())
    torch.testing.assert_close(out[1], out[0], rtol=1e-6, atol=1e-6 * scale)


def test_batch_shape_change_drops_the_state_maxima(cuda):
    """A launch shape whose adjoint scratch differs (adj_chunk) reallocates the scratch: the next params
    call must compute the ubar maxima itself, not take the new buffer's content for them."""
    items = _items(0, n=4, seed=69)
    b = AFMBatch(items)
    _target(b)
    b.forward_adjoint()
    torch.cuda.synchronize()
    g1 = b.grad.clone()
    shape = _lib.BatchShape(*b.shape.key())
    shape.adj_chunk = 4096 if shape.adj_chunk != 4096 else 65536
    b.set_shape(shape)
    b.build_grids()
    b.adjoint_params()  # same states, ubar unchanged; the scratch is new
    torch.cuda.synchronize()
    torch.testing.assert_close(b.grad, g1, rtol=1e-6, atol=1e-6 * float(g1.abs().max()))


def test_batch_adjoint_aggregated_scatter_is_bit_identical(cuda):
    """adj_agg = 1 (the scatter merges each CTA's corner sums in shared memory first) and 2 (a warp walks a
    pixel tile down its strokes and merges its lanes' shared nodes): the same exact integer sums, so the
    gradients and spring terms equal the direct scatter's bit for bit, call after call, for every tile
    height."""
    items = _items(0, n=5, seed=65)
    out = []
    for agg, h in ((0, 8), (1, 8), (2, 8), (2, 1), (2, 4), (2, 32)):
        shape = _lib.BatchShape(*_lib.lib().spm_batch_default_shape().key())
        shape.adj_agg, shape.rx_tile_h = agg, h
        b = AFMBatch(items, shape=shape)
        _target(b)
        b.forward_adjoint()
        g1 = b.grad.clone()
        b.forward_adjoint()  # the scratch kept from the first call (cleared adjoint grid) gives the same
        torch.cuda.synchronize()
        assert torch.equal(g1, b.grad)
        out.append((g1, b.dk_sum.clone()))
    for g, dks in out[1:]:
        assert torch.equal(out[0][0], g) and torch.equal(out[0][1], dks)


def test_batch_tight_z_margin_keeps_every_state(cuda):
    """Slab layers for 1 nN of vertical spring give (0.5 A beyond the tip's z-range at the default 20 N/m,
    against 1.5 A): on molecules of the fitting distribution scanned down to 3 A above the molecule plane the
    relaxation, df and loss are the wide slabs' bit for bit (no probe leaves the thinner slab) and the
    gradients agree to rounding (node partials are grouped by slab layout)."""
    items = synthetic.batch_molecules(4, seed=5, z_end=3.0)
    tight, wide = AFMBatch(items), AFMBatch(items, slab_margin_z=1.5)
    assert tight.grid_float4 < 0.85 * wide.grid_float4
    _target(tight)
    _target(wide)
    for b in (tight, wide):
        b.set_relax_options(polish=True)
        b.forward_adjoint()
    torch.cuda.synchronize()
    assert bool((tight.PPs[:, 3] > 0).all())
    assert torch.equal(tight.FEs, wide.FEs) and torch.equal(tight.PPs, wide.PPs)
    assert torch.equal(tight.df_c, wide.df_c) and torch.equal(tight.loss, wide.loss)
    assert torch.equal(tight.ubar, wide.ubar)
    torch.testing.assert_close(tight.grad, wide.grad, rtol=1e-5, atol=1e-6 * float(wide.grad.abs().max()))


def _adj_mark_offset(b):
    """Byte offset of the adjoint scratch's 16-byte marker slot: the scratch's last 16 bytes."""
    return int(_lib.lib().spm_batch_adjoint_scratch_bytes(b.plan.totals, b.n)) - 16


def test_batch_adam_step_matches_the_adam_formula(cuda):
    """spm_batch_adam_step against Adam written out with tensor ops (FP32), two steps in a row, a
    column mask without y: the masked column and its moments stay untouched."""
    from spammm_b200._lib import check, lib, ptr, stream_ptr
    gen = torch.Generator(device="cuda").manual_seed(5)
    n = 3001
    grad = torch.randn((n, 6), dtype=torch.float64, device="cuda", generator=gen)
    atoms = torch.randn((n, 4), dtype=torch.float32, device="cuda", generator=gen) * 5
    m = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    v = torch.zeros_like(m)
    t = torch.zeros((), dtype=torch.float32, device="cuda")
    ra, rm, rv = atoms.clone(), m.clone(), v.clone()
    lr, b1, b2, eps, cols = 0.01, 0.9, 0.999, 1e-8, (0, 2, 3)
    mask = torch.zeros(4, dtype=torch.float32, device="cuda")
    mask[list(cols)] = 1.0
    for k in range(1, 3):
        check(lib().spm_batch_adam_step(n, ptr(grad), ptr(atoms), ptr(m), ptr(v), ptr(t), lr, b1, b2, eps,
                                        sum(1 << c for c in cols), stream_ptr()), "spm_batch_adam_step")
        g = torch.stack([grad[:, 0], grad[:, 1], grad[:, 2], grad[:, 5]], 1).float() * mask
        rm = rm * b1 + (1 - b1) * g
        rv = rv * b2 + (1 - b2) * g * g
        upd = (rm / (1 - b1 ** k)) / ((rv / (1 - b2 ** k)).sqrt() + eps)
        ra = ra - lr * upd
        grad = grad * 0.5 + 0.1  # the next step sees another gradient
        torch.cuda.synchronize()
        assert float(t) == k
        torch.testing.assert_close(m, rm, rtol=1e-6, atol=1e-7)
        torch.testing.assert_close(v, rv, rtol=1e-6, atol=1e-9)
        torch.testing.assert_close(atoms, ra, rtol=1e-6, atol=1e-6)
    assert torch.equal(m[:, 1], torch.zeros(n, device="cuda")) and torch.equal(atoms[:, 1], ra[:, 1])
