"""Batched probe-particle AFM: many molecules per launch, replayed as a CUDA graph.

The reference's AFMulator (spammm/SPM/AFM.py) images one molecule per call:
make_forcefield -> run_scan -> df.  ``AFMBatch`` runs the same grid path for a
whole batch of molecules with uneven atom counts, grid sizes and scan windows,
each stage ONE launch over the batch (the spm_batch_* entry points of
include/spm_b200.h):

  spm_batch_grid_build     force-grid slabs of every molecule
  spm_batch_relax          persistent SPM_RELAX_PP relaxation; warps draw
                           pixel tiles from one device counter and step
                           down the z-steps together
  spm_batch_df_amp         amplitude-averaged df of every stroke
  spm_batch_df_loss_seed   per-molecule df loss and dL/dFEs
  spm_batch_adjoint_state  implicit-function adjoint of every state
  spm_batch_adjoint_params gather through the grid build: d(loss)/d(atoms)

Per molecule the results are those of the per-molecule calls (grid_build ->
relax_pp -> adjoint on the same GridScanSpec): forward values bit for bit.
Only the nodes the probe can reach -- the scan window's columns and rows
widened by ``slab_margin`` on both sides, the tip's z-range by
``slab_margin_z`` (the spring's vertical give, ``z_margin``) -- are built and
stored; a probe that leaves them is reported as not converged instead of
sampling the missing nodes.

Molecules are laid out in descending order of relaxation work (longest
first), so the persistent relaxation ends with small molecules filling in.
All accessors take and return molecules in the caller's order.
"""
import ctypes
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import BatchMol, BatchShape, check, f4, hostvec, hptr, lib, ptr, stream_ptr
from .diff import GridScanSpec

F32 = torch.float32
F64 = torch.float64


@dataclass
class BatchItem:
    """One molecule: atoms, force-grid geometry and scan raster."""
    atoms: np.ndarray     # (na,4) x,y,z,Q
    params: np.ndarray    # (na,2) LJ c6,c12 or (na,4) Morse R0,E0,K,-
    origin: np.ndarray    # (3,) grid origin [A]
    step: float           # node spacing [A]
    ngrid: tuple          # (nx,ny,nz)
    xs: np.ndarray        # raster x coordinates
    ys: np.ndarray        # raster y coordinates
    z_top: float          # first tip z
    nz: int               # z-steps per stroke

    @property
    def n_scan(self):
        return len(self.xs) * len(self.ys)

    def points(self):
        """(n_scan,4) tip start points, ix-major raster."""
        X, Y = np.meshgrid(np.asarray(self.xs, np.float32), np.asarray(self.ys, np.float32), indexing="ij")
        pts = np.zeros((X.size, 4), np.float32)
        pts[:, 0] = X.ravel()
        pts[:, 1] = Y.ravel()
        pts[:, 2] = np.float32(self.z_top)
        return pts

    def spec(self, kind, probe, dtip):
        """The per-molecule GridScanSpec of this item (the unbatched path)."""
        return GridScanSpec(kind=kind, ngrid=tuple(int(v) for v in self.ngrid), origin=np.asarray(self.origin),
                            step=float(self.step), points=self.points(), nz=int(self.nz), dtip=float(dtip),
                            tipQs=hostvec(probe.tipQs), tipQZs=hostvec(probe.tipQZs), dpos0=hostvec(probe.dpos0),
                            relax_params=hostvec(probe.relax_params), max_iter=int(probe.max_iter),
                            f2conv=float(probe.f2conv), raster_ny=len(self.ys), strict=False)


def _default_stiffness():
    from .AFM import stiffness_Nm_to_eVA2
    kxy, kz = stiffness_Nm_to_eVA2(0.25), stiffness_Nm_to_eVA2(20.0)
    return np.array([-kxy, -kxy, -kz, 0.0], np.float32)


@dataclass
class ProbeSpec:
    """Probe shared by a batch: spring (eV/A^2, negative = restoring), tip
    charges, FIRE settings."""
    stiffness: np.ndarray = field(default_factory=_default_stiffness)
    dpos0: np.ndarray = field(default_factory=lambda: np.zeros(4, np.float32))
    tipQs: np.ndarray = field(default_factory=lambda: np.array([-0.05, 0, 0, 0], np.float32))
    tipQZs: np.ndarray = field(default_factory=lambda: np.zeros(4, np.float32))
    relax_params: np.ndarray = field(default_factory=lambda: np.array([0.5, 0.1, 0.02, 0.5], np.float32))
    max_iter: int = 1000
    f2conv: float = 1e-10


def lateral_range(item, probe, margin, axis):
    """Stored columns (axis 0) or rows (axis 1) [lo, lo + n) of the item's
    grid: every node a trilinear sample can touch while the probe stays within
    `margin` A of the scan window (the raster's tip positions + dpos0).  The
    whole axis when that range reaches an edge (the periodic wrap then needs
    both ends) or the scan is empty."""
    n = int(item.ngrid[axis])
    c = np.asarray(item.xs if axis == 0 else item.ys, np.float64)
    if c.size == 0:
        return 0, n
    d0 = float(probe.dpos0[axis])
    o, h = float(item.origin[axis]), float(item.step)
    t_lo, t_hi = (float(c.min()) + d0 - margin - o) / h, (float(c.max()) + d0 + margin - o) / h
    lo = int(math.floor(t_lo))
    hi = int(math.floor(t_hi)) + 2
    if lo < 0 or hi > n:
        return 0, n
    return lo, hi - lo


# The probe's vertical offset from its tip is F_z / k_z on a Cartesian spring: slab layers are built
# for |F_z| up to 1 nN (0.624 eV/A) -- 0.5 A at the default k_z of 20 N/m, where the batch
# distributions' states stay within 0.06 A of the tip's z -- and at most the lateral margin.
Z_FORCE_BOUND = 0.624
Z_MARGIN_MIN = 0.3


def z_margin(probe, margin):
    """Default margin (A) of the stored layers beyond the tip's z-range:
    Z_FORCE_BOUND / k_z, between Z_MARGIN_MIN and `margin` (the lateral
    one); `margin` itself for a radial spring (stiffness[3] != 0) or a
    probe without a restoring k_z."""
    k = np.asarray(probe.stiffness, np.float64)
    kz = -float(k[2])
    if float(k[3]) != 0.0 or not kz > 0.0:
        return float(margin)
    return min(float(margin), max(Z_MARGIN_MIN, Z_FORCE_BOUND / kz))


def slab_range(item, probe, dtip, margin):
    """Stored layers [z_lo, z_lo + nz_slab) of the item's grid: every layer a
    trilinear sample can touch while the probe stays within `margin` A of the
    tip's z-range (+ dpos0.z).  The full grid when that range reaches an edge
    (the periodic wrap then needs both ends)."""
    nzg = int(item.ngrid[2])
    z_first = float(item.z_top) + float(probe.dpos0[2])
    z_last = z_first + (int(item.nz) - 1) * float(dtip)
    lo_z, hi_z = min(z_first, z_last) - margin, max(z_first, z_last) + margin
    oz, h = float(item.origin[2]), float(item.step)
    t_lo, t_hi = (lo_z - oz) / h, (hi_z - oz) / h
    z_lo = int(math.floor(t_lo))
    z_hi = int(math.floor(t_hi)) + 2
    if z_lo < 0 or z_hi > nzg:
        return 0, nzg
    return z_lo, z_hi - z_lo


class BatchPlan:
    """Host side of a batch: descriptors in work order and the concatenated
    atom / parameter / point arrays (no device memory; see AFMBatch)."""

    def __init__(self, items, kind=0, probe=None, dtip=-0.1, slab_margin=1.5, order="lpt", slab_margin_z=None):
        if not items:
            raise ValueError("a batch needs at least one molecule")
        if dtip >= 0:
            raise ValueError(f"dtip must be < 0 (approach), got {dtip}")
        self.kind = int(kind)
        self.probe = probe or ProbeSpec()
        self.dtip = float(dtip)
        self.items = list(items)
        n = len(items)
        self.n = n
        cost = np.array([it.n_scan * it.nz for it in items], np.int64)
        self.order = np.argsort(-cost, kind="stable") if order == "lpt" else np.arange(n)
        self.pos = np.empty(n, np.int64)
        self.pos[self.order] = np.arange(n)
        pcols = 2 if self.kind == _lib.SPM_KIND_LJ else 4
        self.slab_margin = float(slab_margin)
        self.slab_margin_z = z_margin(self.probe, slab_margin) if slab_margin_z is None else float(slab_margin_z)
        self.mols = (BatchMol * n)()
        atoms_l, params_l, pts_l = [], [], []
        ao = po = so = go = 0
        for j, i in enumerate(self.order):
            it = items[i]
            a = np.asarray(it.atoms, np.float32).reshape(-1, 4)
            p = np.asarray(it.params, np.float32).reshape(len(a), -1)
            if p.shape[1] != pcols:
                raise ValueError(f"molecule {i}: params need {pcols} columns for kind {kind}")
            spec = it.spec(self.kind, self.probe, self.dtip)
            p0, dA, dB, dC = spec.vectors()
            dinv = spec.dinv()
            nx, ny, nzg = (int(v) for v in it.ngrid)
            z_lo, nzs = slab_range(it, self.probe, self.dtip, self.slab_margin_z)
            x_lo, nxs = lateral_range(it, self.probe, slab_margin, 0)
            y_lo, nys = lateral_range(it, self.probe, slab_margin, 1)
            D = self.mols[j]
            D.grid_off, D.state_off = go, so
            D.atom_off, D.n_atoms = ao, len(a)
            D.pix_off, D.n_scan = po, it.n_scan
            D.nx, D.ny, D.nz = nx, ny, nzg
            D.z_lo, D.nz_slab = z_lo, nzs
            D.x_lo, D.nx_slab, D.y_lo, D.ny_slab = x_lo, nxs, y_lo, nys
            D.nz_steps, D.raster_ny = int(it.nz), len(it.ys)
            D.p0, D.dA, D.dB, D.dC = f4(p0), f4(dA), f4(dB), f4(dC)
            D.dinvA, D.dinvB, D.dinvC = f4(dinv[0]), f4(dinv[1]), f4(dinv[2])
            atoms_l.append(a)
            params_l.append(p)
            pts_l.append(it.points())
            ao += len(a)
            po += it.n_scan
            so += it.n_scan * int(it.nz)
            go += nxs * nys * nzs
        self.atoms = np.ascontiguousarray(np.concatenate(atoms_l))
        self.params = np.ascontiguousarray(np.concatenate(params_l))
        self.points = np.ascontiguousarray(np.concatenate(pts_l))
        self.total_atoms, self.total_pixels, self.total_states, self.grid_float4 = ao, po, so, go
        self.shape = None

    def prepare(self, shape):
        """spm_batch_prepare for `shape`: fills the work prefixes; returns the totals."""
        shape = BatchShape(*shape.key())
        totals = (ctypes.c_longlong * _lib.SPM_BATCH_TOTALS)()
        check(lib().spm_batch_prepare(self.mols, self.n, ctypes.byref(shape), totals), "spm_batch_prepare")
        self.shape = shape
        self.totals = totals
        (self.n_tiles, self.n_slots, self.n_units, self.n_chunks) = list(totals)[:4]
        self.n_rows = totals[8]
        return list(totals)

    def desc(self, i):
        """Descriptor of molecule i (caller's order)."""
        return self.mols[int(self.pos[i])]


class AFMBatch:
    """A batch of molecules resident on one GPU (see the module docstring).

    items: list of BatchItem; kind: 0 LJ / 1 Morse (one kind per batch);
    probe: ProbeSpec; dtip: z-step (< 0: approach); slab_margin: A beyond the
    scan window (x, y) whose nodes are built; slab_margin_z: A beyond the
    tip's z-range (None: ``z_margin(probe, slab_margin)``, 0.5 A for the
    default probe); shape: BatchShape (None = library default;
    ``spammm_b200.autotune`` searches better ones)."""

    def __init__(self, items, kind=0, probe=None, dtip=-0.1, slab_margin=1.5, shape=None, order="lpt",
                 slab_margin_z=None):
        _lib.require_cuda()
        plan = BatchPlan(items, kind, probe, dtip, slab_margin, order, slab_margin_z)
        self.plan = plan
        self.dev = torch.device("cuda", torch.cuda.current_device())
        self.kind, self.probe, self.dtip, self.items, self.n = plan.kind, plan.probe, plan.dtip, plan.items, plan.n
        self.order, self.pos, self.mols = plan.order, plan.pos, plan.mols
        ao, po, so, go = plan.total_atoms, plan.total_pixels, plan.total_states, plan.grid_float4
        self.total_atoms, self.total_pixels, self.total_states, self.grid_float4 = ao, po, so, go
        dev = self.dev
        self.atoms = torch.as_tensor(plan.atoms, device=dev).contiguous()
        self.params = torch.as_tensor(plan.params, device=dev).contiguous()
        self.points = torch.as_tensor(plan.points, device=dev).contiguous()
        self.grid = None  # slabs: 2 (x-pairs) or 4 (xz-quads) float4 per node, allocated by set_shape
        self.FEs = torch.empty((so, 4), dtype=F32, device=dev)
        # NaN: no previous equilibrium (a warm-started relaxation then starts every state from its stroke)
        self.PPs = torch.full((so, 4), float("nan"), dtype=F32, device=dev)
        self.iter_count = torch.empty((po,), dtype=torch.int32, device=dev)
        self.df = torch.empty((so,), dtype=F32, device=dev)
        self.workspace = None  # sized for the launch shape by set_shape
        # loss / adjoint buffers: allocated by the first loss or adjoint call
        self.target = self.weights = self.df_c = self.dL = self.ubar = self.dk = self.diag = None
        self.grad = self.dk_sum = None
        # grad columns 3-4 (pair parameters): computed unless a caller that never reads them turns them off
        self.pair_param_grads = True
        self.stiffness_grads = True  # False: no spring-parameter terms (dk, dk_sum = 0)
        self.loss = torch.empty((self.n,), dtype=F64, device=dev)
        self._Qs = hostvec(self.probe.tipQs)
        self._QZs = hostvec(self.probe.tipQZs)
        self.polish = self.warm = False
        self.set_relax_options()
        self.shape = None
        self.set_shape(shape if shape is not None else lib().spm_batch_default_shape())

    def set_relax_options(self, polish=None, warm=None):
        """polish: Newton-polish every equilibrium (SPM_FLAG_POLISH); warm: start each z-step from the
        previous relaxation's equilibrium of the state (SPM_FLAG_WARM) -- for fits, whose atoms move a
        little per step; with the polish both starts reach the same equilibrium.  Both need the
        z-synchronised schedules (shape.rx_sync = 1 or 2).  The flags are read at launch time from the
        scan-parameter struct held here, so a captured graph keeps the options it was captured with."""
        if polish is not None:
            self.polish = bool(polish)
        if warm is not None:
            self.warm = bool(warm)
        self.scan_params = _lib.make_scan_params(tipC=[0, 0, 1, self.dtip], stiffness=self.probe.stiffness,
                                                 dpos0=self.probe.dpos0, relax_params=self.probe.relax_params,
                                                 nz=0, max_iter=self.probe.max_iter, f2conv=self.probe.f2conv,
                                                 fire=True, polish=self.polish, warm=self.warm)
        return self

    def reset_warm_start(self):
        """Forget the previous equilibria: the next warm-started relaxation starts every state from its
        stroke (call after changing atoms by more than a fit step)."""
        self.PPs.fill_(float("nan"))

    # ------------------------------------------------------------ planning
    def set_shape(self, shape):
        """Number the work items for `shape` and upload the descriptors."""
        totals = self.plan.prepare(shape)
        self.shape = self.plan.shape
        per_node = self.node_stride
        if self.grid is None or self.grid.shape[0] != per_node * self.grid_float4:
            self.grid = None  # release the old layout's buffer before allocating the new one
            self.grid = torch.empty((per_node * self.grid_float4, 4), dtype=F32, device=self.dev)
        (self.n_tiles, self.n_slots, self.n_units, self.n_chunks, states, atoms, pixels, gend, self.n_rows) = totals
        ws = int(lib().spm_batch_relax_workspace_bytes(self.n_slots, ctypes.byref(self.shape)))
        if self.workspace is None or self.workspace.numel() * 4 < ws:
            self.workspace = torch.zeros(((ws + 15) // 16 * 4,), dtype=torch.int32, device=self.dev)
        assert (states, atoms, pixels, gend) == (self.total_states, self.total_atoms, self.total_pixels,
                                                 self.grid_float4)
        raw = bytes(memoryview(self.mols).cast("B"))
        self.mols_d = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(self.dev)
        self.loss_scratch = torch.empty((max(1, lib().spm_batch_loss_scratch_bytes(self.n_chunks, self.n) // 8),),
                                        dtype=F64, device=self.dev)
        self._adj_bytes = int(lib().spm_batch_adjoint_scratch_bytes(self.plan.totals, self.n))
        self.adj_scratch = None  # allocated by the first adjoint (it holds the adjoint grid: 32 B per slab node)
        self._state_maxima = False  # a new scratch holds no maxima until the next adjoint_state
        return self

    def desc(self, i):
        """Descriptor of molecule i (caller's order)."""
        return self.plan.desc(i)

    @property
    def node_stride(self):
        """float4 stored per slab node: 2 (x-pairs) or 4 (xz-quads)."""
        return 4 if self.shape.grid_layout else 2

    # ------------------------------------------------------------ stages
    def build_grids(self):
        rc = lib().spm_batch_grid_build(self.kind, self.n, ptr(self.mols_d), self.n_tiles, ctypes.byref(self.shape),
                                        ptr(self.atoms), ptr(self.params), hptr(self._Qs), hptr(self._QZs),
                                        ptr(self.grid), stream_ptr())
        check(rc, "spm_batch_grid_build")

    def relax(self):
        rc = lib().spm_batch_relax(self.n, ptr(self.mols_d), self.n_slots, ctypes.byref(self.shape), ptr(self.grid),
                                   ptr(self.points), ctypes.byref(self.scan_params), ptr(self.FEs), ptr(self.PPs),
                                   ptr(self.iter_count), ptr(self.workspace), self.workspace.numel() * 4,
                                   stream_ptr())
        check(rc, "spm_batch_relax")

    def df_amp(self, amp=1.0):
        rc = lib().spm_batch_df_amp(self.n, ptr(self.mols_d), self.total_pixels, ptr(self.FEs), self.dtip,
                                    float(amp), ptr(self.df), stream_ptr())
        check(rc, "spm_batch_df_amp")

    def _ensure_loss_buffers(self):
        if self.target is None:
            so, dev = self.total_states, self.dev
            self.target = torch.zeros((so,), dtype=F64, device=dev)
            self.df_c = torch.empty((so,), dtype=F64, device=dev)
            self.dL = torch.empty((so, 4), dtype=F32, device=dev)

    def _ensure_adjoint_buffers(self):
        self._ensure_loss_buffers()
        if self.ubar is None:
            so, dev = self.total_states, self.dev
            self.ubar = torch.empty((so, 4), dtype=F32, device=dev)
            self.dk = torch.empty((so, 4), dtype=F32, device=dev)
            self.diag = torch.empty((so, 4), dtype=F32, device=dev)
            self.grad = torch.empty((self.total_atoms, 6), dtype=F64, device=dev)
            self.dk_sum = torch.empty((4,), dtype=F64, device=dev)

    def loss_seed(self):
        self._ensure_loss_buffers()
        rc = lib().spm_batch_df_loss_seed(self.n, ptr(self.mols_d), self.n_chunks, ptr(self.FEs), ptr(self.target),
                                          ptr(self.weights), self.dtip, ptr(self.df_c), ptr(self.dL), ptr(self.loss),
                                          ptr(self.loss_scratch), stream_ptr())
        check(rc, "spm_batch_df_loss_seed")

    def _ensure_adj_scratch(self):
        if self.adj_scratch is None:
            # zero-filled: memory handed out again by the caching allocator can hold an earlier scratch's
            # clear marker (same address, same layout) over an adjoint grid that other tensors overwrote
            self.adj_scratch = torch.zeros(((self._adj_bytes + 15) // 16, 2), dtype=F64, device=self.dev)

    def adjoint_state(self):
        """State adjoint; also leaves the per-molecule ubar maxima and touched boxes in the adjoint scratch
        for adjoint_params (SPM_ADJ_STATE_MAXIMA)."""
        self._ensure_adjoint_buffers()
        self._ensure_adj_scratch()
        rc = lib().spm_batch_adjoint_state(self.n, ptr(self.mols_d), self.total_states, ctypes.byref(self.shape),
                                           ptr(self.grid),
                                           ptr(self.points), ctypes.byref(self.scan_params), ptr(self.PPs),
                                           ptr(self.dL), ptr(self.ubar),
                                           ptr(self.dk) if self.stiffness_grads else None, ptr(self.diag),
                                           self.plan.totals, ptr(self.adj_scratch), stream_ptr())
        check(rc, "spm_batch_adjoint_state")
        self._state_maxima = True

    _state_maxima = False  # the adjoint scratch holds the maxima of the current ubar (from adjoint_state)

    def adjoint_params(self):
        self._ensure_adjoint_buffers()
        self._ensure_adj_scratch()
        rc = lib().spm_batch_adjoint_params(self.kind, self.n, ptr(self.mols_d), self.plan.totals,
                                            ctypes.byref(self.shape), ptr(self.atoms), ptr(self.params),
                                            hptr(self._Qs), hptr(self._QZs), ptr(self.PPs), ptr(self.ubar),
                                            ptr(self.dk) if self.stiffness_grads else None, ptr(self.grad),
                                            ptr(self.dk_sum),
                                            (_lib.SPM_ADJ_PAIR_PARAMS if self.pair_param_grads else 0) |
                                            (_lib.SPM_ADJ_STATE_MAXIMA if self._state_maxima else 0),
                                            ptr(self.adj_scratch), stream_ptr())
        check(rc, "spm_batch_adjoint_params")

    def forward(self, amp=None):
        """Grid slabs + relaxation (+ amplitude df when amp is given)."""
        self.build_grids()
        self.relax()
        if amp is not None:
            self.df_amp(amp)

    def forward_adjoint(self):
        """Forward, per-molecule df loss against self.target, adjoint ->
        self.loss (n, work order), self.grad (total_atoms,6), self.dk_sum."""
        self.build_grids()
        self.relax()
        self.loss_seed()
        self.adjoint_state()
        if not self._mask_failed:
            self.adjoint_params()
            return
        # the next call's loss weights from this call's adjoint status, on a side stream beside the
        # parameter adjoint (which neither reads nor writes them; graph capture keeps the fork and join)
        main = torch.cuda.current_stream()
        if self._side is None:
            self._side = torch.cuda.Stream(device=self.dev)
        self._side.wait_stream(main)
        with torch.cuda.stream(self._side):
            self._update_mask()
        self.adjoint_params()
        main.wait_stream(self._side)

    _mask_failed = False
    _side = None

    def enable_failure_mask(self):
        """Keep the loss consistent with its gradient: after each
        forward_adjoint, states whose adjoint failed (not converged, unstable
        -- where the probe flips --, singular, capped) and their z-neighbours,
        whose central-difference df sees them, get weight 0 in the next call's
        loss.  Their gradient is zero already; without the mask their share of
        the loss would move in ways the gradient cannot see.  Calling it again
        clears the mask in place (captured graphs keep their buffers)."""
        if self._mask_failed:
            self.weights.copy_(self.w_base)
            return
        w = np.ones(self.total_states, np.float64)
        for i in range(self.n):
            D = self.mols[i]
            if D.nz_steps > 0:
                v = w[D.state_off:D.state_off + D.n_scan * D.nz_steps].reshape(D.n_scan, D.nz_steps)
                v[:, 0] = 0.0
                v[:, -1] = 0.0
        self._ensure_adjoint_buffers()
        self.w_base = torch.as_tensor(w, device=self.dev)
        self.weights = self.w_base.clone()
        self._mask_failed = True

    def _update_mask(self):
        # neighbours are taken cyclically over the whole state array: they cross strokes only at
        # the strokes' first and last z-steps, whose base weight is 0
        check(lib().spm_batch_failure_mask(self.total_states, ptr(self.diag), ptr(self.w_base), ptr(self.weights),
                                           stream_ptr()), "spm_batch_failure_mask")

    # ------------------------------------------------------------ data in/out
    def _rows(self, i, what):
        D = self.desc(i)
        if what == "state":
            return D.state_off, D.state_off + D.n_scan * D.nz_steps
        if what == "pixel":
            return D.pix_off, D.pix_off + D.n_scan
        return D.atom_off, D.atom_off + D.n_atoms

    def slab(self, i, slot=0):
        """(nz_slab, ny_slab, nx_slab, 4) view of molecule i's stored box (slot
        0: the nodes' own values; [0, 0, 0] is the full grid's node (x_lo, y_lo,
        z_lo)).  Other slots hold the (x+1), (z+1) and (x+1, z+1) neighbours of
        the layout, wrapped inside the box."""
        D = self.desc(i)
        n = D.nx_slab * D.ny_slab * D.nz_slab
        k = self.node_stride
        return self.grid.view(-1, k, 4)[D.grid_off:D.grid_off + n, slot].reshape(D.nz_slab, D.ny_slab, D.nx_slab, 4)

    def slab_of_full(self, i, full):
        """The part of a full (nz, ny, nx, ...) grid of molecule i that its slab stores."""
        D = self.desc(i)
        return full[D.z_lo:D.z_lo + D.nz_slab, D.y_lo:D.y_lo + D.ny_slab, D.x_lo:D.x_lo + D.nx_slab]

    def fes(self, i):
        a, b = self._rows(i, "state")
        D = self.desc(i)
        return self.FEs[a:b].view(D.n_scan, D.nz_steps, 4)

    def pps(self, i):
        a, b = self._rows(i, "state")
        D = self.desc(i)
        return self.PPs[a:b].view(D.n_scan, D.nz_steps, 4)

    def df_image(self, i):
        """(nx_r, ny_r, nz) amplitude df of molecule i (stroke order: z-step 0 highest)."""
        a, b = self._rows(i, "state")
        it = self.items[i]
        return self.df[a:b].view(len(it.xs), len(it.ys), it.nz)

    def df_central(self, i):
        a, b = self._rows(i, "state")
        it = self.items[i]
        return self.df_c[a:b].view(len(it.xs), len(it.ys), it.nz)

    def atoms_of(self, i):
        a, b = self._rows(i, "atom")
        return self.atoms[a:b]

    def grad_of(self, i):
        """(na,6) d(loss_i)/d(x, y, z, P1, P2, Q) of molecule i."""
        a, b = self._rows(i, "atom")
        return self.grad[a:b]

    def loss_of(self, i):
        return self.loss[int(self.pos[i])]

    def set_atoms(self, i, atoms):
        a, b = self._rows(i, "atom")
        self.atoms[a:b].copy_(torch.as_tensor(np.asarray(atoms, np.float32).reshape(-1, 4), device=self.dev))

    def set_target_states(self, t):
        """Target df of every state at once ((total_states,) in the batch's state order)."""
        self._ensure_loss_buffers()
        self.target.copy_(t.reshape(-1).to(F64))

    def set_target(self, i, df_target):
        """Target df (nx_r, ny_r, nz) of molecule i for the loss."""
        self._ensure_loss_buffers()
        a, b = self._rows(i, "state")
        self.target[a:b].copy_(torch.as_tensor(np.asarray(df_target, np.float64).ravel(), device=self.dev)
                               if not isinstance(df_target, torch.Tensor) else df_target.reshape(-1).to(F64))

    def capture(self, fn, warmup=1):
        """CUDA graph of fn() (launches on the capture stream); returns the graph."""
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(warmup):
                fn()
        torch.cuda.current_stream().wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            fn()
        return g


class BatchAdam:
    """Adam (Kingma & Ba, 2015) on the batch's atom positions and charges,
    one kernel (spm_batch_adam_step) on fixed buffers with the step count on
    the device, so one fitting step -- forward, df loss, adjoint, update --
    captures into one CUDA graph.
    Summing the per-molecule losses makes each molecule's update depend on its
    own loss only.  The update reads gradient columns 0-2 and 5 only, so the
    batch's adjoint skips the pair-parameter columns and the spring terms."""

    def __init__(self, batch, lr=0.01, betas=(0.9, 0.999), eps=1e-8, cols=(0, 1, 2, 3)):
        self.b = batch
        batch.pair_param_grads = False
        batch.stiffness_grads = False
        self.lr, self.b1, self.b2, self.eps = float(lr), float(betas[0]), float(betas[1]), float(eps)
        self.cols = list(cols)
        dev = batch.dev
        na = batch.total_atoms
        self.m = torch.zeros((na, 4), dtype=F32, device=dev)
        self.v = torch.zeros((na, 4), dtype=F32, device=dev)
        self.t = torch.zeros((), dtype=F32, device=dev)  # steps taken (device-side, for graph replays)
        self.col_bits = sum(1 << int(c) for c in set(self.cols))
        if not 0 <= self.col_bits < 16:
            raise ValueError(f"BatchAdam: cols={cols} (0-3: x, y, z, charge)")

    def reset(self):
        self.m.zero_()
        self.v.zero_()
        self.t.zero_()

    def step(self):
        """One fitting step on the current stream (graph-capturable): forward + adjoint, then the
        update in one launch (spm_batch_adam_step)."""
        b = self.b
        b.forward_adjoint()
        check(lib().spm_batch_adam_step(b.total_atoms, ptr(b.grad), ptr(b.atoms), ptr(self.m), ptr(self.v),
                                        ptr(self.t), self.lr, self.b1, self.b2, self.eps, self.col_bits,
                                        stream_ptr()), "spm_batch_adam_step")


class StreamGroup:
    """Independent calls -- typically the ``BatchAdam.step`` of batches over
    disjoint molecule groups, each AFMBatch with its own buffers -- each on a
    stream of its own, forked from and joined back to the caller's stream.
    Captured into one CUDA graph (``capture``), the groups' kernels overlap:
    one group's launches fill the SMs that another group's kernel boundaries
    (its last wave, the dependent launch after it) leave idle.  The calls must
    share no buffer they write; each group's results are those of running it
    alone."""

    def __init__(self, calls, device=None):
        self.calls = list(calls)
        self.streams = [torch.cuda.Stream(device=device) for _ in self.calls]

    def __call__(self):
        main = torch.cuda.current_stream()
        for s in self.streams:
            s.wait_stream(main)
        for fn, s in zip(self.calls, self.streams):
            with torch.cuda.stream(s):
                fn()
        for s in self.streams:
            main.wait_stream(s)

    def capture(self):
        """CUDA graph of one call of every group (the fork and join included)."""
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self()
        return g


def molecule_groups(n, k):
    """Indices of n molecules dealt round-robin into k groups (sizes within one
    of each other; the batch distribution's large and small molecules spread
    evenly)."""
    k = max(1, min(int(k), n)) if n > 0 else 1
    return [list(range(j, n, k)) for j in range(k)]
