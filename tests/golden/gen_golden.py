"""Generates tests/golden/*.npz from the SPAMMM reference's own Python code.

Run where the reference tree is available, giving its root with --ref or
the SPAMMM_REF environment variable:

    python tests/golden/gen_golden.py --ref PATH

The reference imports pyopencl and matplotlib at module level; only its CPU
(NumPy/SciPy) functions are called here, so both are replaced by inert stub
modules written to a temporary directory.  The fixtures pin the oracle and the
CUDA kernels to the reference's own outputs:

  df_golden.npz        compute_df / compute_df_amp / compute_df_dir /
                       compute_df_amp_dir   (spammm/SPM/AFM.py:3048-3236)
  loss_golden.npz      df_loss_seed         (spammm/SPM/AFM.py:3125-3200)
  diss_golden.npz      compute_dissipation  (spammm/SPM/AFM.py:3238-3277),
                       afm_df_height_stacks (spammm/SPM/AFM_utils.py:653-681),
                       shared_postprocess   (spammm/SPM/AFM_utils.py:3363-3414)
  frame_golden.npz     AFMulator._make_dinv_axis_aligned (AFM.py:274-285),
                       _morse_atoms_from_Z mixing (AFM_utils.py:3993-4017)
  pair_golden.npz      _cpu_pair_fe / _cpu_pair_partials
                       (tests/SPM/test_afm_morse.py:451-545)
  direct_golden.npz    _cpu_relax_direct    (tests/SPM/test_afm_morse.py:548-604)
                       and _cpu_vjp_oracle  (tests/SPM/test_afm_morse.py:1240-1310)
  gridrelax_golden.npz Morse grid = _cpu_pair_fe at the nodes + the |E|>100 cap
                       of evalMorseC_QZs_toImg (kernels/AFM.cl:1053-1054), relaxed
                       with the reference's _cpu_tipForce/_cpu_update_FIRE in the
                       relaxStrokes / relaxStrokesTilted / getFEinStrokesTilted
                       loop structure (kernels/AFM.cl:210-233, 345-394, 478-562),
                       FP64, exact trilinear sampling with periodic wrap.
"""
import argparse
import os
import sys
import tempfile

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))

_STUB_PYOPENCL = "class _S:\n    def __getattr__(self, k): return _S()\n    def __call__(self, *a, **k): return _S()\n" \
                 "def __getattr__(name): return _S()\n"
_STUB_MPL = "def use(*a, **k): pass\ndef __getattr__(name):\n    import types\n    return types.SimpleNamespace()\n"
_STUB_MPL_SUB = "def __getattr__(name):\n    return lambda *a, **k: None\n"


def _install_stubs():
    d = tempfile.mkdtemp(prefix="spm_stub_")
    os.makedirs(os.path.join(d, "pyopencl"))
    os.makedirs(os.path.join(d, "matplotlib"))
    with open(os.path.join(d, "pyopencl", "__init__.py"), "w") as f:
        f.write(_STUB_PYOPENCL)
    with open(os.path.join(d, "matplotlib", "__init__.py"), "w") as f:
        f.write(_STUB_MPL)
    for m in ("pyplot", "collections", "colors", "cm", "patches", "gridspec", "ticker"):
        with open(os.path.join(d, "matplotlib", m + ".py"), "w") as f:
            f.write(_STUB_MPL_SUB)
    sys.path.insert(0, d)


def _trilin_periodic(grid, dinv, p):
    """Exact trilinear sample of an (nz,ny,nx,4) grid with REPEAT addressing."""
    nz, ny, nx = grid.shape[:3]
    idx, frac = [], []
    for d, n in zip(range(3), (nx, ny, nz)):
        u = p[0] * dinv[d][0] + p[1] * dinv[d][1] + p[2] * dinv[d][2] + dinv[d][3]
        s = u - np.floor(u)
        t = s * n - 0.5
        i0 = int(np.floor(t))
        a = t - np.floor(t)
        i0 %= n
        idx.append((i0, (i0 + 1) % n))
        frac.append(a)
    (x0, x1), (y0, y1), (z0, z1) = idx
    ax, ay, az = frac
    c00 = grid[z0, y0, x0] * (1 - ax) + grid[z0, y0, x1] * ax
    c10 = grid[z0, y1, x0] * (1 - ax) + grid[z0, y1, x1] * ax
    c01 = grid[z1, y0, x0] * (1 - ax) + grid[z1, y0, x1] * ax
    c11 = grid[z1, y1, x0] * (1 - ax) + grid[z1, y1, x1] * ax
    c0 = c00 * (1 - ay) + c10 * ay
    c1 = c01 * (1 - ay) + c11 * ay
    return c0 * (1 - az) + c1 * az


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SPAMMM_REF"),
                    help="root of the SPAMMM reference tree (default: $SPAMMM_REF)")
    ap.add_argument("--only", choices=["xyz"], default=None,
                    help="write only one fixture file (xyz: xyz_golden.npz)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference tree with --ref PATH or SPAMMM_REF")
    _install_stubs()
    sys.path.insert(0, args.ref)
    from spammm.SPM import AFM as A
    if args.only == "xyz":
        xyz_fixtures(A)
        return
    from spammm.SPM import AFM_utils as U
    import tests.SPM.test_afm_morse as T

    rng = np.random.default_rng(20261203)

    # ---------------- df functions
    df = {}
    cases = [
        ((6, 5, 21), np.float32, (0.3, 0.2, 0.1), (0., 0., 1.), 1.0),
        ((6, 5, 21), np.float64, (0.3, 0.2, 0.1), (0., 0., 1.), 0.4),
        ((7, 6, 15), np.float32, (0.25, 0.25, 0.1), (1., 0., 0.), 0.5),
        ((7, 6, 15), np.float64, 0.2, (1., 2., 3.), 0.7),
        ((5, 7, 17), np.float32, (0.1, 0.15, 0.1), (0.3, 0., 1.), 1.0),
        ((4, 4, 9), np.float64, (0.1, 0.1, 0.1), (0., -1., 0.), 0.25),
    ]
    for i, (shp, dt, sp, od, amp) in enumerate(cases):
        FEs = rng.standard_normal(shp + (4,)).astype(dt)
        df[f"c{i}_FEs"] = FEs
        df[f"c{i}_spacing"] = np.asarray(sp, dtype=np.float64)
        df[f"c{i}_osc"] = np.asarray(od, dtype=np.float64)
        df[f"c{i}_amp"] = np.float64(amp)
        df[f"c{i}_amp_dir"] = A.compute_df_amp_dir(FEs, sp, od, amp)
        df[f"c{i}_dir"] = A.compute_df_dir(FEs, sp, od)
    Fz = rng.standard_normal((5, 4, 19)).astype(np.float32)
    df["Fz"] = Fz
    df["compute_df"] = A.compute_df(Fz, 0.1)
    df["compute_df_amp"] = A.compute_df_amp(Fz, 0.1, 0.6)
    df["n_cases"] = np.int64(len(cases))
    np.savez_compressed(os.path.join(OUT, "df_golden.npz"), **df)

    # ---------------- df_loss_seed
    ls = {}
    for i, (shp, dtip, weighted) in enumerate([((3, 4, 9), -0.1, False), ((2, 3, 7), -0.15, True),
                                               ((4, 2, 12), -0.2, False)]):
        FEs = rng.standard_normal(shp + (4,))
        tgt = rng.standard_normal(shp)
        w = None
        if weighted:
            w = rng.uniform(0.1, 1.0, shp)
            w[:, :, 0] = 0
            w[:, :, -1] = 0
        loss, dfv, dL = A.df_loss_seed(FEs, tgt, dtip, w)
        ls[f"c{i}_FEs"] = FEs
        ls[f"c{i}_tgt"] = tgt
        ls[f"c{i}_w"] = w if w is not None else np.zeros(0)
        ls[f"c{i}_dtip"] = np.float64(dtip)
        ls[f"c{i}_loss"] = np.float64(loss)
        ls[f"c{i}_df"] = dfv
        ls[f"c{i}_dL"] = dL
    ls["n_cases"] = np.int64(3)
    np.savez_compressed(os.path.join(OUT, "loss_golden.npz"), **ls)

    # ---------------- dissipation, height stacks, shared_postprocess
    ds = {}
    h_df, h_Fz, h_scan = U.afm_df_height_stacks(3.7, 4.7, 0.1, amp=1.0)
    ds["h_df"], ds["h_Fz"], ds["h_scan"] = h_df, h_Fz, h_scan
    h2 = U.afm_df_height_stacks(3.0, 4.0, 0.2, amp=0.5, osc_dir=(1., 0., 1.))
    ds["h2_df"], ds["h2_Fz"], ds["h2_scan"] = h2
    h3 = U.afm_df_height_stacks(3.7, 4.7, 0.1, amp=1.0, osc_dir=(1., 0., 0.))
    ds["h3_df"], ds["h3_Fz"], ds["h3_scan"] = h3
    nzs = len(h_scan)
    Ff = rng.standard_normal((4, 3, nzs, 4)).astype(np.float32)
    Fb = (Ff + 0.05 * rng.standard_normal(Ff.shape)).astype(np.float32)
    ds["Ff"], ds["Fb"] = Ff, Fb
    ds["E_z"] = A.compute_dissipation(Ff, Fb, h_scan, h_df, 1.0, (0., 0., 1.))
    ds["E_t"] = A.compute_dissipation(Ff, Fb, h_scan, h_df, 0.6, (0.5, 0., 1.))
    spec = U.ScanSpec(scan_xs=np.arange(4, dtype=np.float32) * 0.1, scan_ys=np.arange(3, dtype=np.float32) * 0.1,
                      h_df=h_df, h_Fz=h_Fz, h_scan=h_scan, amplitude=1.0, osc_dir=(0., 0., 1.),
                      K_LAT=0.03, K_RAD=20.0, bond_length=3.0)
    res = U.shared_postprocess(Ff, spec, FEs_bwd=Fb)
    ds["pp_df"], ds["pp_Fz"], ds["pp_E"] = res.df, res.Fz, res.E_diss
    np.savez_compressed(os.path.join(OUT, "diss_golden.npz"), **ds)

    # ---------------- frames and mixing rules
    fr = {}
    for i, (L, o, n) in enumerate([((10., 20., 30.), (0., 0., 0.), (50, 100, 150)),
                                   ((10., 20., 30.), (-5., 3., 1.), (50, 100, 150)),
                                   ((48., 48., 24.), (-3., -3., -6.), (480, 480, 240))]):
        d = A.AFMulator._make_dinv_axis_aligned(np.array(L), np.array(o, dtype=np.float32), n)
        fr[f"c{i}_L"], fr[f"c{i}_o"], fr[f"c{i}_n"] = np.array(L), np.array(o), np.array(n)
        fr[f"c{i}_dinv"] = np.stack(d)
    Zs = np.array([1, 6, 7, 8, 11, 17], dtype=np.int32)
    pos = rng.standard_normal((len(Zs), 3))
    at, cm = U._morse_atoms_from_Z(pos, Zs, params_path=os.path.join(args.ref, "data", "ElementTypes.dat"))
    fr["mix_Z"], fr["mix_pos"], fr["mix_atoms"], fr["mix_cMs"] = Zs, pos, at, cm
    np.savez_compressed(os.path.join(OUT, "frame_golden.npz"), **fr)

    # ---------------- pair law
    pr = {}
    for i, (na, seed) in enumerate([(3, 11), (4, 17), (5, 29)]):
        atoms, cMs, tQ, tQZ = T._make_toy_system(n_atoms=na, seed=seed)
        q = np.random.default_rng(seed + 1).uniform(-2.0, 2.0, (12, 3))
        pr[f"c{i}_atoms"], pr[f"c{i}_cMs"], pr[f"c{i}_q"] = atoms, cMs, q
        pr[f"c{i}_Qs"], pr[f"c{i}_QZs"] = tQ, tQZ
        pr[f"c{i}_fe"] = T._cpu_pair_fe(atoms, cMs, q, tQ, tQZ)
        pr[f"c{i}_part"] = T._cpu_pair_partials(atoms, cMs, q, tQ, tQZ)
    pr["n_cases"] = np.int64(3)
    np.savez_compressed(os.path.join(OUT, "pair_golden.npz"), **pr)

    # ---------------- direct relaxation and VJP (reference CPU64 oracles)
    dr = {}
    AF = A.AFMulator
    atoms, cMs, tQ, tQZ = T._make_toy_system(n_atoms=2, seed=97)
    pts, p0, da, db = T._make_toy_scan(atoms, nxy=(3, 3), nz=5, dtip=-0.2)
    FEs, PPs = T._cpu_relax_direct(atoms, cMs, pts, 5, -0.2, AF.DEFAULT_tipA, AF.DEFAULT_tipB, AF.DEFAULT_tipC,
                                   AF.DEFAULT_stiffness, AF.DEFAULT_dpos0, AF.DEFAULT_relax_pars, AF.DEFAULT_surfFF,
                                   tQ, tQZ)
    dr.update(r_atoms=atoms, r_cMs=cMs, r_Qs=tQ, r_QZs=tQZ, r_pts=pts, r_p0=p0, r_da=da, r_db=db, r_FEs=FEs,
              r_PPs=PPs)
    atoms, cMs, tQ, tQZ = T._make_toy_system(n_atoms=2, seed=31)
    pts, p0, da, db = T._make_toy_scan(atoms, nxy=(3, 3), nz=5)
    tipC = AF.DEFAULT_tipC.copy()
    tipC[3] = -0.2
    FEs, PPs = T._cpu_relax_direct(atoms, cMs, pts, 5, -0.2, AF.DEFAULT_tipA, AF.DEFAULT_tipB, tipC,
                                   AF.DEFAULT_stiffness, AF.DEFAULT_dpos0, AF.DEFAULT_relax_pars, AF.DEFAULT_surfFF,
                                   tQ, tQZ, n_steps=2000, f2conv=1e-16)
    tgt = np.random.default_rng(33).standard_normal((3, 3, 5))
    loss, _, dL = A.df_loss_seed(FEs.reshape(3, 3, 5, 4), tgt, -0.2)
    grad, diag = T._cpu_vjp_oracle(atoms, cMs, PPs.reshape(3, 3, 5, 4), pts.reshape(3, 3, 3), -0.2, dL,
                                   AF.DEFAULT_tipA, AF.DEFAULT_tipB, tipC, AF.DEFAULT_stiffness, AF.DEFAULT_dpos0,
                                   AF.DEFAULT_surfFF, tQ, tQZ)
    dr.update(v_atoms=atoms, v_cMs=cMs, v_Qs=tQ, v_QZs=tQZ, v_pts=pts, v_p0=p0, v_da=da, v_db=db, v_FEs=FEs,
              v_PPs=PPs, v_tgt=tgt, v_dL=dL, v_grad=grad, v_loss=np.float64(loss))
    np.savez_compressed(os.path.join(OUT, "direct_golden.npz"), **dr)

    # ---------------- grid relaxation (FP64, reference helper functions)
    gr = {}
    atoms, cMs, tQ, tQZ = T._make_toy_system(n_atoms=3, seed=5)
    atoms[:, 2] *= 0.2
    n = (24, 22, 30)
    step = 0.25
    origin = np.array([-3.0, -2.75, -2.0])
    L = np.array(n) * step
    ia, ib, ic = np.meshgrid(np.arange(n[0]), np.arange(n[1]), np.arange(n[2]), indexing="ij")
    nodes = np.stack([origin[0] + ia * step, origin[1] + ib * step, origin[2] + ic * step], axis=-1).reshape(-1, 3)
    fe = T._cpu_pair_fe(atoms, cMs, nodes, tQ, tQZ)
    renorm = 100.0 / np.abs(fe[:, 3])
    cap = renorm < 1.0
    fe[cap] *= renorm[cap, None]
    grid = fe.reshape(n[0], n[1], n[2], 4).transpose(2, 1, 0, 3).copy()  # (nz,ny,nx,4)
    dinv = [np.asarray(v, dtype=np.float64) for v in
            A.AFMulator._make_dinv_axis_aligned(L, origin.astype(np.float32), n)]
    gr.update(atoms=atoms, cMs=cMs, Qs=tQ, QZs=tQZ, n=np.array(n), step=np.float64(step), origin=origin, grid=grid,
              dinv=np.stack(dinv))
    pts = np.zeros((9, 4), dtype=np.float32)
    k = 0
    for x in (-0.6, 0.0, 0.7):
        for y in (-0.5, 0.1, 0.6):
            pts[k, :3] = (x, y, 4.6)
            k += 1
    nzs = 6
    # kernel arguments are float4 in the reference: use float32-representable values
    stiff = np.array([-0.02, -0.02, -0.8, 0.0], np.float32).astype(np.float64)
    d0 = np.zeros(4)
    relax = AF.DEFAULT_relax_pars.astype(np.float64)
    dTip = np.array([0.0, 0.0, -0.1, 0.0], np.float32).astype(np.float64)

    def fire_stroke(pt, post_eval, tilted, tipC=None):
        a, b = np.array([1., 0, 0]), np.array([0., 1, 0])
        c = np.array([0., 0, 1])
        if tilted:
            a, b, c = (np.asarray(AF.DEFAULT_tipA[:3], np.float64), np.asarray(AF.DEFAULT_tipB[:3], np.float64),
                       np.asarray(tipC[:3], np.float64))
        dT = c * float(tipC[3]) if tilted else dTip[:3]
        d0r = T._rotMatT(d0[:3], a, b, c) if tilted else d0[:3]
        tip = pt[:3].astype(np.float64).copy()
        pos = tip + d0r
        dt, damp = float(relax[0]), float(relax[1])
        dtmax, dtmin, damp0 = dt, dt * 0.1, damp
        out_fe, out_d = [], []
        for iz in range(nzs):
            v = np.zeros(3)
            fe = np.zeros(4)
            for it in range(128):
                fe = _trilin_periodic(grid, dinv, pos)
                f = fe[:3].copy()
                dl = T._rotMat(pos - tip, a, b, c) if tilted else pos - tip
                ft = T._cpu_tipForce(dl, stiff, d0)
                f = f + (T._rotMatT(ft, a, b, c) if tilted else ft)
                v, dt, damp = T._cpu_update_FIRE(f, v, dt, damp, dtmin, dtmax, damp0)
                v = v + f * dt
                pos = pos + v * dt
                if float(np.dot(f, f)) < 1e-8:
                    break
            if post_eval:
                fe = _trilin_periodic(grid, dinv, pos)
                r = T._rotMat(fe[:3], a, b, c)
                fe = np.array([r[0], r[1], r[2], fe[3]])
            out_fe.append(fe.copy())
            out_d.append(np.array([*(pos - (tip + d0r)), 0.0]))
            tip = tip + dT
            pos = pos + dT
        return np.array(out_fe), np.array(out_d)

    FE_s, D_s, FE_t = [], [], []
    tipC = np.array([0., 0., 1., -0.1], np.float32).astype(np.float64)
    for p in pts:
        fe_, d_ = fire_stroke(p, False, False)
        FE_s.append(fe_)
        D_s.append(d_)
        FE_t.append(fire_stroke(p, True, True, tipC)[0])
    raw = []
    for p in pts:
        pos = p[:3].astype(np.float64) + d0[:3]
        row = []
        for iz in range(nzs):
            row.append(_trilin_periodic(grid, dinv, pos))
            pos = pos + dTip[:3]
        raw.append(row)
    gr.update(pts=pts, nzs=np.int64(nzs), stiffness=stiff, dpos0=d0, relax=relax, dTip=dTip, tipC=tipC,
              strokes_FEs=np.array(FE_s), strokes_disps=np.array(D_s), tilted_FEs=np.array(FE_t), raw_FEs=np.array(raw))
    np.savez_compressed(os.path.join(OUT, "gridrelax_golden.npz"), **gr)
    print("wrote fixtures to", OUT)


# xyz inputs for the loader fixture: element names or atomic numbers, an
# optional charge column, a count line and an "lvs" comment line (the periodic
# cell of setup_grid_lvec); written here, parsed by the reference.
XYZ_TEXTS = {
    "names_charges": "5\nmolecule with charges\nC 0.0 0.0 0.0 -0.12\nH 1.09 0.0 0.0 0.03\n"
                     "O -0.7 1.1 0.05 -0.4\nN 0.6 -1.2 -0.02 0.25\nH -0.5 -0.9 0.1 0.24\n",
    "numbers_no_charge": "4\n\n6 0.1 0.2 0.3\n1 1.2 0.2 0.3\n8 -1.0 0.4 0.2\n7 0.0 1.5 -0.1\n",
    "lvs_skew": "6\nlvs 6.0 0.0 0.0   3.0 5.196152422706632 0.0   0.0 0.0 20.0\n"
                "Na 0.0 0.0 0.0 0.8\nCl 2.0 0.0 0.0 -0.8\nNa 1.5 2.598 0.0 0.8\nCl 3.5 2.598 0.0 -0.8\n"
                "C 2.2 1.3 3.0 0.1\nH 3.1 1.3 3.0 -0.1\n",
}


def xyz_fixtures(A):
    """xyz_golden.npz: AFMulator.load_molecule's loader (spammm/AtomicSystem.py:35-90 ->
    atomicUtils.load_xyz :1212) and setup_grid_lvec (spammm/SPM/AFM.py:839-893) on a skew cell."""
    from types import SimpleNamespace
    from spammm.AtomicSystem import AtomicSystem
    out = {}
    d = tempfile.mkdtemp(prefix="spm_xyz_")
    for key, text in XYZ_TEXTS.items():
        fn = os.path.join(d, key + ".xyz")
        with open(fn, "w") as f:
            f.write(text)
        mol = AtomicSystem(fname=fn)
        out[f"{key}_text"] = np.array(text)
        out[f"{key}_apos"] = np.asarray(mol.apos, np.float64)
        out[f"{key}_enames"] = np.array(list(mol.enames))
        out[f"{key}_qs"] = np.asarray(mol.qs, np.float64)
        out[f"{key}_lvec"] = np.asarray(mol.lvec, np.float64) if mol.lvec is not None else np.zeros(0)
        if mol.lvec is not None:
            atoms = np.zeros((len(mol.apos), 4), np.float32)
            atoms[:, :3] = mol.apos
            atoms[:, 3] = mol.qs
            fake = SimpleNamespace(atoms_arr=atoms.copy(), mol=mol, _make_dinv_lvec=A.AFMulator._make_dinv_lvec,
                                   _max_alloc=1 << 40)
            n, margin_z, z_top = (60, 52, 230), 2.0, 12.0
            L = A.AFMulator.setup_grid_lvec(fake, n, margin_z, z_top)
            out.update({f"{key}_lvec_n": np.array(n), f"{key}_lvec_margin_z": np.float64(margin_z),
                        f"{key}_lvec_z_top": np.float64(z_top), f"{key}_lvec_L": L,
                        f"{key}_lvec_atoms": fake.atoms_arr, f"{key}_lvec_mol_shift": fake.mol_shift,
                        f"{key}_lvec_dA": fake.dA, f"{key}_lvec_dB": fake.dB, f"{key}_lvec_dC": fake.dC,
                        f"{key}_lvec_dinv": np.stack([fake.dinvA, fake.dinvB, fake.dinvC])})
    out["keys"] = np.array(list(XYZ_TEXTS))
    np.savez_compressed(os.path.join(OUT, "xyz_golden.npz"), **out)
    print("wrote xyz_golden.npz to", OUT)


if __name__ == "__main__":
    main()
