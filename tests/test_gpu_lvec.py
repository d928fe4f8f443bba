"""Periodic skew cell through the drop-in (setup_grid_lvec, spammm/SPM/AFM.py:
839-893): a NaCl-like layer with a molecule in a 60-degree cell read by
load_molecule from an .xyz with an "lvs" line (the fixture of
tests/golden/xyz_golden.npz), LJ grid on the skew node lattice against the FP64
oracle (grid-build tolerance of test_gpu_scale.py: 2e-5 |ref| + 2e-6 max|ref| +
1e-5 S + the node-position rounding term), and run_scan
(relaxStrokesTilted) over a window larger than the cell -- probes sample across
the periodic seam through the skew sampling transform -- bit-identical to the
canonical-FP32 oracle on the same grid; unrelaxed samples of a window shifted
by a period of the sampling transform equal the unshifted ones.

The sampling transform is the reference's: dinvA/B/C are the rows of inv(M)^T
(AFM.py:883-884 with _make_dinv_lvec, AFM.py:288-294), M = [a | b | Lz e_z]
by columns, and the kernel takes u = dot(pos, dinvA) (kernels/AFM.cl:100-104).
For a skew cell those are the columns of inv(M), not its rows, so the sampled
field repeats along the rows of M -- (a_x, b_x, 0) and (a_y, b_y, 0) -- not
along a and b.  The drop-in keeps that mapping bit for bit; the test checks
the periods it has.
"""
import os
import tempfile

import numpy as np
import pytest

from oracle import oracle as O
from spammm_b200.AFM import AFMulator

pytestmark = pytest.mark.gpu


def test_skew_periodic_cell_grid_and_scan(cuda, golden):
    g = golden("xyz_golden.npz")
    d = tempfile.mkdtemp(prefix="spm_lvec_")
    fn = os.path.join(d, "cell.xyz")
    with open(fn, "w") as f:
        f.write(str(g["lvs_skew_text"]))
    afm = AFMulator(use_morse=False)
    afm.load_molecule(fn)
    afm.assign_params()
    afm.setup_grid_lvec(n=(60, 52, 230), margin_z=2.0, z_top=12.0)
    afm.make_forcefield()
    nx, ny, nz = (int(v) for v in afm.n)
    grid = afm.img_FF.cpu().numpy()
    ref = O.grid_build(0, afm.atoms_arr, afm.cLJs_arr, afm.n, afm.p0, afm.dA, afm.dB, afm.dC, afm.tipQs, afm.tipQZs,
                       prec="f64")
    # node positions of the skew lattice, and each node's sum of contribution magnitudes S (FP32 sums err in
    # proportion to S; the cell's +-0.8 e ions cancel)
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    dA, dB, dC = (np.asarray(v, np.float64) for v in (afm.dA, afm.dB, afm.dC))
    q = (ix[..., None] * dA[:3] + iy[..., None] * dB[:3] + iz[..., None] * dC[:3]).reshape(-1, 3)
    a64, p64 = afm.atoms_arr.astype(np.float64), afm.cLJs_arr.astype(np.float64)
    raw = O.pair_fe(0, a64, p64, q, afm.tipQs, afm.tipQZs)
    S = O.pair_fe_abs(0, a64, p64, q, afm.tipQs, afm.tipQZs) * np.minimum(1.0, 100.0 / np.abs(raw[:, 3]))[:, None]
    ref = ref.reshape(-1, 4)
    scale = np.abs(ref).max(axis=0)
    err = np.abs(grid.reshape(-1, 4).astype(np.float64) - ref)
    from test_gpu_scale import pos_term
    assert not (err > 2e-5 * np.abs(ref) + 2e-6 * scale + 1e-5 * S + pos_term(q, a64, ref)).any()
    # a scan window of 9 x 8 A over a 6 A skew cell: the probes cross the periodic seam
    nxy, nzs, dtip = (36, 32), 20, -0.1
    p0 = np.array([-1.5, -1.0, 3.0 + afm.mol_z + 3.5], np.float32)
    da = np.array([0.25, 0.0, 0.0], np.float32)
    db = np.array([0.0, 0.25, 0.0], np.float32)
    FEs, pts = afm.run_scan(nxy=nxy, nz=nzs, dtip=dtip, scan_p0=p0, scan_da=da, scan_db=db)
    assert np.isfinite(FEs).all()
    p4 = np.zeros((nxy[0] * nxy[1], 4), np.float32)
    p4[:, :3] = pts.reshape(-1, 3)
    tipC = afm.tipC.copy()
    tipC[3] = dtip
    o = O.relax_tilted(grid, (afm.dinvA, afm.dinvB, afm.dinvC), p4, nzs, afm.tipA, afm.tipB, tipC, afm.stiffness,
                       afm.dpos0, afm.relax_pars, afm.surfFF, afm.n_relax_max, afm.f2conv)
    assert np.array_equal(FEs.reshape(-1, nzs, 4), o)
    # unrelaxed samples of a window shifted by a period of the sampling transform (a row of M) equal the
    # unshifted ones; a shift by the cell vector b is not a period of the reference's skew mapping
    raw1, _ = afm.get_raw_FE(nxy=nxy, nz=nzs, dtip=dtip, scan_p0=p0, scan_da=da, scan_db=db)
    # (the upper heights, where |F| < 1 eV/A: nearer the atoms a sample at a texel edge may round into
    # the neighbouring cell in one window and not the other, which the capped cores turn into O(1) jumps)
    far = np.abs(raw1[..., :3]).max(axis=(0, 1, 3)) < 1.0
    assert far.sum() >= 2
    lv = afm.mol.lvec.astype(np.float32)
    M = np.stack([lv[0, :3], lv[1, :3], np.array([0., 0., afm.L[2]], np.float32)], axis=1)
    for period in (M[0], M[1]):
        raw2, _ = afm.get_raw_FE(nxy=nxy, nz=nzs, dtip=dtip, scan_p0=p0 + np.array([period[0], period[1], 0.0],
                                                                                    np.float32),
                                 scan_da=da, scan_db=db)
        assert np.abs(raw2[:, :, far] - raw1[:, :, far]).max() < 1e-4 * np.abs(raw1[:, :, far]).max()
    raw3, _ = afm.get_raw_FE(nxy=nxy, nz=nzs, dtip=dtip, scan_p0=p0 + np.array([lv[1, 0], lv[1, 1], 0.0], np.float32),
                             scan_da=da, scan_db=db)
    assert np.abs(raw3[:, :, far] - raw1[:, :, far]).max() > 1e-2 * np.abs(raw1[:, :, far]).max()
