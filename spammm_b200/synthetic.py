"""Seeded synthetic workloads for the probe-particle AFM path.

No public dataset is involved: the benchmark configurations are synthetic
molecules/slabs with fixed seeds.  Shapes, sizes and value distributions:

  plain_small   38-atom planar molecule (C24 O6 H8) on a honeycomb lattice
                (1.4 A bonds, z=0, sigma=0.02 A jitter), charges U(-0.3,0.3)
                shifted to zero sum, LJ parameters from the element table;
                grid 20 A cube at 0.1 A (200^3); 100x100 pixels, 40 z-steps of
                0.1 A from 9 A above the molecule plane.
  plain_large   3-layer NaCl(100) slab (a=5.64 A, +-0.8 e) of 1140 ions under a
                60-atom C/N/H planar molecule at 3.0 A; grid 48x48x24 A at
                0.1 A (480x480x240); 480x480 pixels, 60 z-steps of 0.1 A.
  batch         molecules with U{10..120} C/N/O/H atoms, grids 12-32 A per
                side at 0.1 A (at least the molecule + 3 A on each side),
                scan windows of 64^2-256^2 pixels over the molecule, 30-60
                z-steps of 0.1 A ending 4 A above the molecule plane.

Probe (all configs): k_xy = 0.25 N/m, k_z = 20 N/m (harmonic, no radial
bond), Q = -0.05 e at the probe position; FIRE <= 1000 steps, |F| < 1e-5 eV/A.
"""
from dataclasses import dataclass

import numpy as np

from .AFM import stiffness_Nm_to_eVA2
from .AFM_utils import _lj_atoms_from_Z, _morse_atoms_from_Z

Z_OF = {"H": 1, "C": 6, "N": 7, "O": 8, "Na": 11, "Cl": 17}


def honeycomb_sites(n, bond=1.4):
    """The n honeycomb-lattice sites closest to the origin (bond length `bond`)."""
    a1 = np.array([1.5 * bond, np.sqrt(3) / 2 * bond])
    a2 = np.array([1.5 * bond, -np.sqrt(3) / 2 * bond])
    R = int(np.ceil(np.sqrt(n))) + 3
    pts = []
    for i in range(-R, R + 1):
        for j in range(-R, R + 1):
            base = i * a1 + j * a2
            pts.append(base)
            pts.append(base + np.array([bond, 0.0]))
    pts = np.array(pts)
    c = pts.mean(axis=0)
    d = np.linalg.norm(pts - c, axis=1)
    order = np.lexsort((pts[:, 1], pts[:, 0], np.round(d, 6)))
    return pts[order[:n]] - pts[order[:n]].mean(axis=0)


def planar_molecule(counts, seed, sigma=0.02, bond=1.4, qmax=0.3):
    """Planar molecule: element counts {'C':24,...} on honeycomb sites, H outermost.

    Returns (pos (n,3) float64, Z (n,) int32, q (n,) float64, zero-sum)."""
    rng = np.random.default_rng(seed)
    n = int(sum(counts.values()))
    xy = honeycomb_sites(n, bond)
    r = np.linalg.norm(xy, axis=1)
    order = np.argsort(r, kind="stable")
    names = []
    heavy = [e for e in ("C", "N", "O") for _ in range(counts.get(e, 0))]
    rng.shuffle(heavy)
    names_by_rank = heavy + ["H"] * counts.get("H", 0)
    Z = np.zeros(n, np.int32)
    for rank, idx in enumerate(order):
        Z[idx] = Z_OF[names_by_rank[rank]]
        names.append(names_by_rank[rank])
    pos = np.zeros((n, 3))
    pos[:, :2] = xy
    pos += rng.normal(0.0, sigma, pos.shape)
    q = rng.uniform(-qmax, qmax, n)
    q -= q.mean()
    return pos, Z, q


def nacl_slab(nx_ions=20, ny_ions=19, layers=3, a=5.64, charge=0.8):
    """NaCl(100) slab: ions on a square lattice of pitch a/2, alternating in
    x, y and layer; top layer at z=0, layers below at -a/2, -a, ..."""
    h = a / 2.0
    pos, Z, q = [], [], []
    for L in range(layers):
        for i in range(nx_ions):
            for j in range(ny_ions):
                s = (i + j + L) % 2
                pos.append((i * h, j * h, -L * h))
                Z.append(11 if s == 0 else 17)
                q.append(charge if s == 0 else -charge)
    pos = np.array(pos, dtype=np.float64)
    pos[:, 0] -= pos[:, 0].mean()
    pos[:, 1] -= pos[:, 1].mean()
    return pos, np.array(Z, np.int32), np.array(q, np.float64)


@dataclass
class PlainConfig:
    """One plain-path workload: atoms + grid + scan + probe."""
    name: str
    atoms: np.ndarray        # (na,4) float32 x,y,z,Q
    params: np.ndarray       # (na,2) LJ or (na,4) Morse float32
    kind: int                # 0 LJ, 1 Morse
    origin: np.ndarray       # (3,) grid origin
    step: float
    ngrid: tuple
    scan_xs: np.ndarray
    scan_ys: np.ndarray
    z_top: float             # first (highest) probe z
    nz: int
    dz: float
    stiffness: np.ndarray    # (4,) eV/A^2
    dpos0: np.ndarray
    tipQs: np.ndarray
    tipQZs: np.ndarray
    max_iter: int = 1000
    f2conv: float = 1e-10    # |F| < 1e-5 eV/A
    amp: float = 1.0

    @property
    def n_pix(self):
        return len(self.scan_xs) * len(self.scan_ys)

    @property
    def pxz(self):
        return self.n_pix * self.nz

    @property
    def pairs(self):
        return int(np.prod(self.ngrid)) * len(self.atoms)


def probe_params():
    k_xy = stiffness_Nm_to_eVA2(0.25)
    k_z = stiffness_Nm_to_eVA2(20.0)
    return (np.array([-k_xy, -k_xy, -k_z, 0.0], np.float32), np.zeros(4, np.float32),
            np.array([-0.05, 0, 0, 0], np.float32), np.zeros(4, np.float32))


def plain_small(seed=0, n_pix=100, nz=40, kind=0, ngrid=200):
    """38-atom molecule, 20 A grid at 0.1 A, n_pix^2 pixels x nz z-steps."""
    pos, Z, q = planar_molecule({"C": 24, "O": 6, "H": 8}, seed)
    atoms, prm = (_lj_atoms_from_Z if kind == 0 else _morse_atoms_from_Z)(pos, Z)
    atoms[:, 3] = q.astype(np.float32)
    step = 20.0 / ngrid
    origin = np.array([-10.0, -10.0, -6.0])
    span = 0.1 * n_pix
    xs = (-span / 2 + 0.1 * np.arange(n_pix)).astype(np.float32)
    k, d0, Qs, QZs = probe_params()
    return PlainConfig("plain_small", atoms, prm, kind, origin, step, (ngrid, ngrid, ngrid), xs, xs.copy(),
                       9.0, nz, 0.1, k, d0, Qs, QZs)


def plain_large(seed=1, kind=0, n_pix=480, nz=60):
    """1140-ion NaCl slab + 60-atom molecule at 3 A; 480x480x240 grid; n_pix^2 x nz."""
    spos, sZ, sq = nacl_slab()
    mpos, mZ, mq = planar_molecule({"C": 40, "N": 6, "H": 14}, seed)
    mpos[:, 2] += 3.0
    pos = np.concatenate([spos, mpos])
    Z = np.concatenate([sZ, mZ])
    q = np.concatenate([sq, mq])
    atoms, prm = (_lj_atoms_from_Z if kind == 0 else _morse_atoms_from_Z)(pos, Z)
    atoms[:, 3] = q.astype(np.float32)
    origin = np.array([-24.0, -24.0, -8.0])
    xs = (-24.0 + 0.1 * np.arange(n_pix)).astype(np.float32)
    k, d0, Qs, QZs = probe_params()
    return PlainConfig("plain_large", atoms, prm, kind, origin, 0.1, (480, 480, 240), xs, xs.copy(), 3.0 + 9.0, nz,
                       0.1, k, d0, Qs, QZs)


def batch_molecules(n_mol=512, seed=3, kind=0, z_end=4.0, dz=0.1, natoms=(10, 120), side=(12.0, 32.0),
                    zside=(12.0, 32.0), npx=(64, 256), nzs=(30, 60), pad=3.0):
    """n_mol BatchItems of the batch distribution: U{10..120} C/N/O/H atoms on
    honeycomb fragments, grids of U(12,32) A per side (x = y; at least the
    molecule's extent + 2*pad, so the periodic seam of the grid stays `pad` A
    away from every atom) and U(12,32) A in z at 0.1 A, square rasters of
    U{64..256}^2 pixels over the molecule's extent + 1 A on each side,
    U{30..60} z-steps of dz ending z_end A above the molecule plane.  The grid
    top sits 2 A above the first tip position.  The ranges are parameters
    (smaller ones make test batches)."""
    from .batch import BatchItem
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n_mol):
        na = int(rng.integers(natoms[0], natoms[1] + 1))
        nH = max(1, int(round(na * rng.uniform(0.15, 0.3))))
        nN = int(rng.integers(0, max(1, na // 10) + 1))
        nO = int(rng.integers(0, max(1, na // 10) + 1))
        nC = max(1, na - nH - nN - nO)
        pos, Z, q = planar_molecule({"C": nC, "N": nN, "O": nO, "H": nH}, seed * 100003 + m)
        atoms, prm = (_lj_atoms_from_Z if kind == 0 else _morse_atoms_from_Z)(pos, Z)
        atoms[:, 3] = q.astype(np.float32)
        half = float(np.abs(pos[:, :2]).max())  # molecule centred at the origin
        cell = max(float(rng.uniform(*side)), 2.0 * (half + pad))
        n = int(np.ceil(cell / 0.1))
        nzg = int(round(float(rng.uniform(*zside)) / 0.1))
        n_px = int(rng.integers(npx[0], npx[1] + 1))
        n_z = int(rng.integers(nzs[0], nzs[1] + 1))
        cell = n * 0.1
        z_top = z_end + (n_z - 1) * dz
        origin = np.array([-cell / 2, -cell / 2, z_top + 2.0 - nzg * 0.1])
        win = half + 1.0
        xs = (-win + (np.arange(n_px) + 0.5) * (2.0 * win / n_px)).astype(np.float32)
        out.append(BatchItem(atoms=atoms, params=prm, origin=origin, step=0.1, ngrid=(n, n, nzg), xs=xs,
                             ys=xs.copy(), z_top=float(z_top), nz=n_z))
    return out
