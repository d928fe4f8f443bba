"""Input adapters on the CPU against the reference's own outputs
(tests/golden/xyz_golden.npz, written by tests/golden/gen_golden.py --only xyz):

  * load_xyz_molecule (AFMulator.load_molecule) against the reference's loader
    (spammm/AtomicSystem.py:35-90 -> spammm/atomicUtils.py:1212 load_xyz, and
    the "lvs" comment line of a periodic cell): positions, element names,
    charges and the cell vectors;
  * setup_grid_lvec on a skew (60 degree) cell against the reference's
    (spammm/SPM/AFM.py:839-893): node vectors dA, dB, dC, the sampling
    transform dinvA..C, the z shift of the atoms and the cell lengths, bit for
    bit.
"""
import os
import tempfile
from types import SimpleNamespace

import numpy as np

from spammm_b200.AFM import AFMulator, load_xyz_molecule


def _molecule(g, key):
    d = tempfile.mkdtemp(prefix="spm_xyz_")
    fn = os.path.join(d, key + ".xyz")
    with open(fn, "w") as f:
        f.write(str(g[f"{key}_text"]))
    return load_xyz_molecule(fn)


def test_load_xyz_matches_reference_loader(golden):
    g = golden("xyz_golden.npz")
    for key in g["keys"]:
        key = str(key)
        mol = _molecule(g, key)
        assert np.array_equal(mol.apos, g[f"{key}_apos"])
        assert list(mol.enames) == [str(e) for e in g[f"{key}_enames"]]
        assert np.array_equal(mol.qs, g[f"{key}_qs"])
        ref_lvec = g[f"{key}_lvec"]
        if ref_lvec.size == 0:
            assert mol.lvec is None
        else:
            assert np.array_equal(mol.lvec, ref_lvec)


def test_setup_grid_lvec_matches_reference_on_a_skew_cell(golden):
    g = golden("xyz_golden.npz")
    key = "lvs_skew"
    mol = _molecule(g, key)
    atoms = np.zeros((mol.natoms, 4), np.float32)
    atoms[:, :3] = mol.apos
    atoms[:, 3] = mol.qs
    fake = SimpleNamespace(atoms_arr=atoms, mol=mol, _make_dinv_lvec=AFMulator._make_dinv_lvec)
    n = tuple(int(v) for v in g[f"{key}_lvec_n"])
    L = AFMulator.setup_grid_lvec(fake, n, float(g[f"{key}_lvec_margin_z"]), float(g[f"{key}_lvec_z_top"]))
    assert np.array_equal(L, g[f"{key}_lvec_L"])
    assert np.array_equal(fake.atoms_arr, g[f"{key}_lvec_atoms"])
    assert np.array_equal(fake.mol_shift, g[f"{key}_lvec_mol_shift"])
    for k in ("dA", "dB", "dC"):
        assert np.array_equal(getattr(fake, k), g[f"{key}_lvec_{k}"]), k
    assert np.array_equal(np.stack([fake.dinvA, fake.dinvB, fake.dinvC]), g[f"{key}_lvec_dinv"])
    assert fake.dB[0] != 0.0  # the cell is skew: grid rows are not axis-aligned
