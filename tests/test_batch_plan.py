"""Host-side planning of batches (no GPU): descriptor layout, work numbering,
slab ranges and argument validation of spm_batch_prepare."""
import ctypes

import numpy as np
import pytest

from spammm_b200 import _lib, synthetic
from spammm_b200.batch import BatchPlan, ProbeSpec, lateral_range, slab_range


def small_items(n=7, seed=5, kind=0):
    return synthetic.batch_molecules(n, seed=seed, kind=kind, natoms=(10, 40), side=(5, 9), zside=(8, 14),
                                     npx=(5, 21), nzs=(8, 16))


def test_struct_layout():
    # spm_batch_mol: 7 int64 offsets, 16 int32 fields, 7 float[4] vectors
    assert ctypes.sizeof(_lib.BatchMol) == 7 * 8 + 16 * 4 + 7 * 16
    assert ctypes.sizeof(_lib.BatchShape) == 12 * 4


@pytest.mark.parametrize("shape_kw", [{}, dict(gb_ty=2, gb_zb=16, rx_tile_h=1, adj_chunk=1024),
                                      dict(gb_ty=8, rx_tile_h=32, rx_threads=256, adj_chunk=65536)])
def test_prepare_totals(shape_kw):
    items = small_items()
    plan = BatchPlan(items)
    shape = _lib.lib().spm_batch_default_shape()
    for k, v in shape_kw.items():
        setattr(shape, k, v)
    tot = plan.prepare(shape)
    tiles = slots = units = chunks = rows = 0
    th = shape.rx_tile_h
    tw = 32 // th
    for j in range(plan.n):
        D = plan.mols[j]
        assert (D.tile_off, D.slot_off, D.unit_off, D.chunk_off, D.row_off) == (tiles, slots, units, chunks, rows)
        tiles += -(-(D.nx_slab * D.ny_slab) // (32 * shape.gb_ty)) * -(-D.nz_slab // shape.gb_zb)
        nst = D.n_scan * D.nz_steps
        nxr = D.n_scan // D.raster_ny
        slots += -(-nxr // tw) * -(-D.raster_ny // th) * 32
        u = -(-(D.nx_slab * D.ny_slab * D.nz_slab) // shape.adj_chunk)
        units += u
        rows += u * D.n_atoms
        chunks += -(-nst // 256)
    assert tot[:4] == [tiles, slots, units, chunks]
    assert tot[4:7] == [plan.total_states, plan.total_atoms, plan.total_pixels]
    assert tot[7:] == [plan.grid_float4, rows]


def test_order_and_offsets():
    items = small_items(9)
    plan = BatchPlan(items)
    cost = [items[i].n_scan * items[i].nz for i in plan.order]
    assert cost == sorted(cost, reverse=True)
    assert sorted(plan.order.tolist()) == list(range(len(items)))
    for i, it in enumerate(items):
        D = plan.desc(i)
        a = plan.atoms[D.atom_off:D.atom_off + D.n_atoms]
        np.testing.assert_array_equal(a, np.asarray(it.atoms, np.float32))
        pts = plan.points[D.pix_off:D.pix_off + D.n_scan]
        np.testing.assert_array_equal(pts, it.points())
        assert D.nz_steps == it.nz and D.raster_ny == len(it.ys)


def test_slab_covers_probe_range():
    probe = ProbeSpec()
    for it in small_items(12, seed=9):
        z_lo, nzs = slab_range(it, probe, -0.1, 1.5)
        oz, h = float(it.origin[2]), float(it.step)
        for z in (it.z_top + 1.5, it.z_top - (it.nz - 1) * 0.1 - 1.5):
            t = (z - oz) / h
            assert z_lo <= np.floor(t) and np.floor(t) + 1 < z_lo + nzs
        assert 0 <= z_lo and z_lo + nzs <= it.ngrid[2]
    # a range reaching the grid edge keeps the whole grid (periodic wrap)
    it = small_items(1)[0]
    it.z_top = float(it.origin[2]) + 0.05
    assert slab_range(it, probe, -0.1, 1.5) == (0, it.ngrid[2])


def test_z_margin_follows_the_spring():
    """The stored layers' margin beyond the tip's z-range: 1 nN over k_z (0.5 A at 20 N/m), between 0.3 A and
    the lateral margin; the lateral margin itself for a radial spring or no restoring k_z.  A plan's slabs
    use it unless slab_margin_z is given."""
    import dataclasses
    from spammm_b200.batch import z_margin
    probe = ProbeSpec()
    assert abs(z_margin(probe, 1.5) - 0.5) < 1e-3
    assert z_margin(probe, 0.4) == 0.4
    soft = dataclasses.replace(probe, stiffness=probe.stiffness * np.float32(0.01))
    assert z_margin(soft, 1.5) == 1.5
    stiff = dataclasses.replace(probe, stiffness=probe.stiffness * np.float32(100.0))
    assert z_margin(stiff, 1.5) == 0.3
    radial = dataclasses.replace(probe, stiffness=np.array([*probe.stiffness[:3], -0.5], np.float32))
    assert z_margin(radial, 1.5) == 1.5
    items = small_items(5, seed=8)
    tight, wide = BatchPlan(items), BatchPlan(items, slab_margin_z=1.5)
    assert tight.slab_margin_z == z_margin(probe, 1.5) and wide.slab_margin_z == 1.5
    for i, it in enumerate(items):
        Dt, Dw = tight.desc(i), wide.desc(i)
        assert (Dt.z_lo, Dt.nz_slab) == slab_range(it, probe, -0.1, tight.slab_margin_z)
        assert (Dt.x_lo, Dt.nx_slab, Dt.y_lo, Dt.ny_slab) == (Dw.x_lo, Dw.nx_slab, Dw.y_lo, Dw.ny_slab)
        assert Dw.z_lo <= Dt.z_lo and Dt.z_lo + Dt.nz_slab <= Dw.z_lo + Dw.nz_slab
    assert tight.grid_float4 < wide.grid_float4


def test_lateral_range_covers_scan_window():
    """Stored columns and rows hold every texel a sample within the margin of
    the scan window needs; a window whose margin reaches the grid edge keeps
    the whole axis (periodic wrap)."""
    probe = ProbeSpec()
    items = synthetic.batch_molecules(12, seed=9)
    for it in items:
        for axis, c in ((0, it.xs), (1, it.ys)):
            lo, n = lateral_range(it, probe, 1.5, axis)
            o, h = float(it.origin[axis]), float(it.step)
            for v in (float(c.min()) - 1.5, float(c.max()) + 1.5):
                t = (v - o) / h
                assert lo <= np.floor(t) and np.floor(t) + 1 < lo + n
            assert 0 <= lo and lo + n <= it.ngrid[axis]
    assert any(lateral_range(it, probe, 1.5, 0)[1] < it.ngrid[0] for it in items)  # boxes are smaller than grids
    plan = BatchPlan(items)
    assert plan.grid_float4 == sum(D.nx_slab * D.ny_slab * D.nz_slab for D in plan.mols)
    it = items[0]
    assert lateral_range(it, probe, float(it.ngrid[0]) * it.step, 0) == (0, it.ngrid[0])
    import dataclasses
    assert lateral_range(dataclasses.replace(it, xs=it.xs[:0]), probe, 1.5, 0) == (0, it.ngrid[0])


def test_prepare_rejects_bad_descriptors():
    L = _lib.lib()
    shape = L.spm_batch_default_shape()
    totals = (ctypes.c_longlong * _lib.SPM_BATCH_TOTALS)()
    plan = BatchPlan(small_items(4))
    assert L.spm_batch_prepare(plan.mols, plan.n, ctypes.byref(shape), totals) == _lib.SPM_OK
    # rows that do not follow the previous molecule's
    plan.mols[2].atom_off += 1
    assert L.spm_batch_prepare(plan.mols, plan.n, ctypes.byref(shape), totals) == _lib.SPM_ERR_ARG
    assert b"follow" in L.spm_last_error()
    plan.mols[2].atom_off -= 1
    # slab outside the grid
    plan.mols[1].nz_slab = plan.mols[1].nz + 1
    assert L.spm_batch_prepare(plan.mols, plan.n, ctypes.byref(shape), totals) == _lib.SPM_ERR_ARG
    plan.mols[1].nz_slab = 4
    # columns / rows outside the grid
    for field, bad in (("x_lo", -1), ("nx_slab", 0), ("y_lo", -1), ("ny_slab", 0)):
        old = getattr(plan.mols[0], field)
        setattr(plan.mols[0], field, bad)
        assert L.spm_batch_prepare(plan.mols, plan.n, ctypes.byref(shape), totals) == _lib.SPM_ERR_ARG, field
        setattr(plan.mols[0], field, old)
    plan.mols[0].x_lo = plan.mols[0].nx - plan.mols[0].nx_slab + 1
    assert L.spm_batch_prepare(plan.mols, plan.n, ctypes.byref(shape), totals) == _lib.SPM_ERR_ARG
    assert b"outside" in L.spm_last_error()
    plan = BatchPlan(small_items(4))
    # overlapping slabs
    plan.mols[3].grid_off = plan.mols[2].grid_off
    assert L.spm_batch_prepare(plan.mols, plan.n, ctypes.byref(shape), totals) == _lib.SPM_ERR_ARG
    plan = BatchPlan(small_items(4))
    for field, bad in (("gb_ty", 3), ("gb_zb", 4), ("rx_threads", 96), ("rx_tile_h", 6), ("adj_chunk", 1000), ("rx_regs", 6), ("grid_layout", 2),
                       ("rx_sync", 3), ("adj_ilp", 4), ("adj_stage", 2), ("adj_agg", 3)):
        s = L.spm_batch_default_shape()
        setattr(s, field, bad)
        assert L.spm_batch_prepare(plan.mols, plan.n, ctypes.byref(s), totals) == _lib.SPM_ERR_ARG, field


def test_partial_raster_falls_back_to_1d():
    plan = BatchPlan(small_items(3))
    plan.mols[0].raster_ny = 7 if plan.mols[0].n_scan % 7 else 11
    if plan.mols[0].n_scan % plan.mols[0].raster_ny == 0:
        pytest.skip("raster size divisible")
    tot = plan.prepare(_lib.lib().spm_batch_default_shape())
    assert plan.mols[0].raster_ny == 0
    assert plan.mols[1].slot_off == -(-plan.mols[0].n_scan // 32) * 32  # a warp's 32 slots stay in one molecule
    assert tot[1] > 0


def test_relax_workspace_sizes_and_shape_combinations():
    """spm_batch_relax_workspace_bytes: the counters alone for the one-pass schedules, plus one 48-byte tail
    entry per slot for the two-pass one; shape combinations the kernels do not have are refused."""
    L = _lib.lib()
    s = L.spm_batch_default_shape()
    for sync, extra in ((0, 0), (1, 0), (2, 48)):
        s.rx_sync = sync
        assert L.spm_batch_relax_workspace_bytes(1000, ctypes.byref(s)) == 16 + extra * 1000
    assert L.spm_batch_relax_workspace_bytes(-1, ctypes.byref(s)) < 0
    totals = (ctypes.c_longlong * _lib.SPM_BATCH_TOTALS)()
    plan = BatchPlan(small_items(3))
    for kw, ok in ((dict(adj_stage=1, adj_ilp=1), True), (dict(adj_stage=1, adj_ilp=2), False),
                   (dict(adj_agg=2), True), (dict(rx_sync=2, rx_regs=4), True)):
        s = L.spm_batch_default_shape()
        for k, v in kw.items():
            setattr(s, k, v)
        rc = L.spm_batch_prepare(plan.mols, plan.n, ctypes.byref(s), totals)
        assert (rc == _lib.SPM_OK) == ok, kw


def test_autotune_shape_text():
    from spammm_b200 import autotune
    base = _lib.lib().spm_batch_default_shape()
    s = autotune._parse_shape("rx_regs=2,rx_tile_h=4,adj_stage=1", base)
    assert (s.rx_regs, s.rx_tile_h, s.adj_stage) == (2, 4, 1)
    assert s.gb_ty == base.gb_ty  # the other fields keep the base's values
    with pytest.raises(ValueError, match="unknown"):
        autotune._parse_shape("rx_bogus=1", base)
    # every candidate list names real fields
    for cands in (autotune.GRID_CANDIDATES, autotune.RELAX_CANDIDATES, autotune.ADJOINT_CANDIDATES):
        for kw in cands:
            assert all(hasattr(base, k) for k in kw), kw


def test_molecule_groups_deal_round_robin():
    from spammm_b200.batch import molecule_groups
    assert molecule_groups(10, 4) == [[0, 4, 8], [1, 5, 9], [2, 6], [3, 7]]
    assert molecule_groups(3, 8) == [[0], [1], [2]]  # no empty group
    assert molecule_groups(5, 1) == [list(range(5))]
    assert molecule_groups(5, 0) == [list(range(5))]
    g = molecule_groups(64, 4)
    assert sorted(i for grp in g for i in grp) == list(range(64)) and {len(x) for x in g} == {16}
