"""Drop-in replacement of the hot-path callers in ``spammm.SPM.AFM_utils``.

Scan contract (``ScanSpec`` / ``ScanResult`` / ``shared_postprocess``,
spammm/SPM/AFM_utils.py:3307-3414), height ladders (``afm_df_height_stacks``,
:653-681), Morse mixing from atomic numbers (``_morse_atoms_from_Z``,
:3993-4017) and the Morse+Q PP-AFM driver ``run_morse_pp_afm`` (:4020-4153).
The df / Fz / dissipation post-processing runs on the GPU and takes the force
volume straight from device memory; plotting arguments are accepted and
ignored (plots are not part of this path).
"""
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import AFM as afm
from . import gpu
from .FFparams import read_element_types, z_map


def afm_df_height_stacks(h_min, h_max, h_step, amp=1.0, amp_align=True, osc_dir=(0., 0., 1.)):
    """(h_df, h_Fz, h_scan) height ladders (AFM_utils.py:653-681)."""
    def _h_stack(h0, h1, dz):
        n = int(round((float(h1) - float(h0)) / float(dz))) + 1
        return (float(h0) + np.arange(n, dtype=np.float64) * float(dz)).astype(np.float32)

    h_df = _h_stack(h_min, h_max, h_step)
    amp = float(amp)
    osc_n = np.asarray(osc_dir, dtype=np.float64)
    osc_norm = float(np.linalg.norm(osc_n))
    if osc_n.shape != (3,) or not np.isfinite(osc_norm) or osc_norm <= 0.0:
        raise ValueError(f"afm_df_height_stacks: osc_dir must be a finite non-zero vector, got {osc_dir!r}")
    osc_n /= osc_norm
    amp_z = amp * abs(float(osc_n[2]))
    h_Fz = (h_df.astype(np.float64) - amp_z).astype(np.float32) if amp_align else h_df.copy()
    h_scan = _h_stack(float(h_df[0]) - amp_z, float(h_df[-1]) + amp_z, h_step)
    if len(h_scan) < 3:
        raise ValueError(f"afm_df_height_stacks: need denser heights for amp={amp}: n_scan={len(h_scan)}")
    return h_df, h_Fz, h_scan


@dataclass
class ScanSpec:
    """Scan/grid contract shared by the backends (AFM_utils.py:3307-3327)."""
    scan_xs: np.ndarray
    scan_ys: np.ndarray
    h_df: np.ndarray
    h_Fz: np.ndarray
    h_scan: np.ndarray
    amplitude: float
    osc_dir: tuple
    K_LAT: float
    K_RAD: float
    bond_length: float
    scan_margin: float = 2.0


@dataclass
class ScanResult:
    """Backend-independent scan result (AFM_utils.py:3330-3361)."""
    df: np.ndarray
    Fz: np.ndarray
    heights: np.ndarray
    heights_Fz: np.ndarray
    scan_xs: np.ndarray
    scan_ys: np.ndarray
    amp_align: bool
    FEs: np.ndarray
    tip_disp: dict
    E_diss: np.ndarray
    backend_name: str = "unknown"
    fft_path: str = "none"

    def __getitem__(self, key):
        return getattr(self, key)

    def __contains__(self, key):
        return hasattr(self, key)

    def get(self, key, default=None):
        return getattr(self, key, default)


def _nearest_indices(h_scan, h_sel):
    h_scan = np.asarray(h_scan)
    return [int(np.argmin(np.abs(h_scan - h))) for h in h_sel]


def shared_postprocess(FEs_full, scan_spec, *, FEs_bwd=None, tip_disp=None, backend_name="unknown", fft_path="none",
                       return_device=False, E_diss=None):
    """df / Fz / E_diss from a relaxed (nx,ny,nz_scan,4) volume (AFM_utils.py:3363-3414).

    ``FEs_full`` / ``FEs_bwd`` may be CUDA tensors (kept on the device) or
    host arrays.  df is evaluated on the GPU only at the h_df slices.
    E_diss: the dissipation already integrated (the paired relaxation's fused
    epilogue, scan_fdbm_pair(dissipation=...)); then FEs_bwd is not read."""
    on_dev = isinstance(FEs_full, torch.Tensor)
    F = FEs_full if on_dev else np.asarray(FEs_full, dtype=np.float32)
    nx, ny, nz_scan = (int(s) for s in F.shape[:3])
    sx = float(scan_spec.scan_xs[1] - scan_spec.scan_xs[0]) if len(scan_spec.scan_xs) > 1 else 0.0
    sy = float(scan_spec.scan_ys[1] - scan_spec.scan_ys[0]) if len(scan_spec.scan_ys) > 1 else 0.0
    sz = float(scan_spec.h_scan[1] - scan_spec.h_scan[0]) if len(scan_spec.h_scan) > 1 else 0.0
    osc_n = np.asarray(scan_spec.osc_dir, dtype=np.float64)
    osc_n = osc_n / np.linalg.norm(osc_n)
    idx_df = _nearest_indices(scan_spec.h_scan, scan_spec.h_df)
    idx_Fz = _nearest_indices(scan_spec.h_scan, scan_spec.h_Fz)
    df = gpu.df_amp_dir(F, (sx, sy, sz), osc_n, float(scan_spec.amplitude), out_iz=idx_df)
    Fv = F if on_dev else torch.from_numpy(F).to(df.device)
    Fz = Fv[..., 2][:, :, idx_Fz]
    if E_diss is not None:
        E_diss = E_diss if isinstance(E_diss, torch.Tensor) else torch.as_tensor(np.asarray(E_diss), device=df.device)
    elif FEs_bwd is not None:
        E_diss = gpu.dissipation(Fv, FEs_bwd, scan_spec.h_scan, scan_spec.h_df, float(scan_spec.amplitude), osc_n)
    else:
        E_diss = torch.zeros((nx, ny, len(scan_spec.h_df)), dtype=torch.float32, device=df.device)
    if tip_disp is None:
        tip_disp = {k: np.zeros((nx, ny, nz_scan), dtype=np.float32) for k in ("dx", "dy", "dz")}
    amp_align = bool(abs(float(osc_n[2])) > 1e-12)
    if not return_device:
        df, Fz, E_diss = gpu.to_host(df), gpu.to_host(Fz), gpu.to_host(E_diss)
        F = gpu.to_host(F) if on_dev else F
    return ScanResult(df=df, Fz=Fz, heights=np.asarray(scan_spec.h_df, dtype=np.float32),
                      heights_Fz=np.asarray(scan_spec.h_Fz, dtype=np.float32),
                      scan_xs=np.asarray(scan_spec.scan_xs, dtype=np.float32),
                      scan_ys=np.asarray(scan_spec.scan_ys, dtype=np.float32), amp_align=amp_align, FEs=F,
                      tip_disp=tip_disp, E_diss=E_diss, backend_name=backend_name, fft_path=fft_path)


def compose_and_relax_total(F_total, scan_xs, scan_ys, heights, origin, step, atomPos, K_LAT=None, K_RAD=20.0,
                            bond_length=4.0, use_gpu_relax=True, ppm_mode=False, afmulator=None,
                            reuse_fdbm_grid=False, osc_dir=(0., 0., 1.), base_pos=(0., 0., 0.)):
    """FDBM stage 4 (AFM_utils.py:3111-3201): relax the probe in a total force
    field F_total (nx,ny,nz,4) and convert to df.

    ppm_mode=True: relaxStrokes with the spherical PPM bond (scan_fdbm);
    ppm_mode=False: 2-D lateral-only relaxStrokes2D (scan_fdbm_2d).  Returns
    (df (nx_s,ny_s,nz_s), tip_disp, FEs_relax (nx_s,ny_s,nz_s,4)).  The
    reference's legacy SciPy CPU relaxation (use_gpu_relax=False) is not part
    of this implementation."""
    if not use_gpu_relax:
        raise NotImplementedError("compose_and_relax_total: the CPU SciPy relaxation is not provided; "
                                  "use_gpu_relax must be True")
    if K_LAT is None:
        K_LAT = afm.K_LAT_HAPALA_EV_A2
    mol_z = float(np.asarray(atomPos)[:, 2].max())
    if ppm_mode:
        if afmulator is None:
            afmulator = afm.AFMulator(use_morse=False, nloc=32, use_fire=True)
        if not reuse_fdbm_grid:
            afmulator.setup_fdbm_grid(F_total, origin, step)
        FEs_relax, tip_disp = afmulator.scan_fdbm(scan_xs, scan_ys, heights, mol_z=mol_z, K_LAT=K_LAT, K_RAD=K_RAD,
                                                  bond_length=bond_length, ppm_mode=True, use_fire=True,
                                                  osc_dir=osc_dir, base_pos=base_pos)
    else:
        if afmulator is None:
            afmulator = afm.AFMulator(use_morse=False, nloc=32, use_fire=False)
        if not reuse_fdbm_grid:
            afmulator.setup_fdbm_grid(F_total, origin, step)
        FEs_relax, tip_disp = afmulator.scan_fdbm_2d(scan_xs, scan_ys, heights, mol_z=mol_z, K_LAT=K_LAT)
    spacing = (float(scan_xs[1] - scan_xs[0]), float(scan_ys[1] - scan_ys[0]), float(heights[1] - heights[0]))
    df = afm.compute_df_dir(FEs_relax, spacing, osc_dir=osc_dir)
    return df, tip_disp, FEs_relax


def _morse_atoms_from_Z(atomPos, atomTypes, params_path=None, tip_R=1.452, tip_E=0.0006808, tip_alpha=-1.8):
    """(atoms (na,4), cMs (na,4)) Morse parameters from atomic numbers (AFM_utils.py:3993-4017)."""
    zm = z_map(read_element_types(params_path))
    na = len(atomPos)
    atoms = np.zeros((na, 4), dtype=np.float32)
    atoms[:, :3] = np.asarray(atomPos, dtype=np.float32)[:, :3]
    cMs = np.zeros((na, 4), dtype=np.float32)
    for ia in range(na):
        z = int(atomTypes[ia])
        e = zm.get(z)
        assert e is not None, f"_morse_atoms_from_Z: no ElementTypes entry for Z={z}"
        R0 = tip_R + e.RvdW
        E0 = np.sqrt(abs(tip_E * e.EvdW))
        cMs[ia] = [R0, E0, tip_alpha, 0.]
    return atoms, cMs


def _lj_atoms_from_Z(atomPos, atomTypes, params_path=None, tip_R=1.452, tip_E=0.0006808):
    """(atoms (na,4), cLJs (na,2)) LJ (c6,c12) with the assign_params mixing (AFM.py:758-765)."""
    zm = z_map(read_element_types(params_path))
    na = len(atomPos)
    atoms = np.zeros((na, 4), dtype=np.float32)
    atoms[:, :3] = np.asarray(atomPos, dtype=np.float32)[:, :3]
    cLJs = np.zeros((na, 2), dtype=np.float32)
    for ia in range(na):
        e = zm.get(int(atomTypes[ia]))
        assert e is not None, f"_lj_atoms_from_Z: no ElementTypes entry for Z={int(atomTypes[ia])}"
        R0 = tip_R + e.RvdW
        E0 = np.sqrt(abs(tip_E * e.EvdW))
        cLJs[ia] = [2. * E0 * R0 ** 6, E0 * R0 ** 12]
    return atoms, cLJs


def run_morse_pp_afm(tag, atomPos, atomTypes, origin, step, ngrid, outdir=None, *, scan_spec, params_path=None,
                     margin=4.0, plots=None, df_cmap="gray", cmap="seismic", stage_height=4.2, charges=None):
    """Morse+Q PP-AFM through ScanSpec/ScanResult (AFM_utils.py:4020-4153).

    Grid build, forward and backward relaxation strokes, df and dissipation
    all run on the GPU; the returned ScanResult holds host arrays."""
    atomPos = np.asarray(atomPos, dtype=np.float64)
    atomTypes = np.asarray(atomTypes, dtype=np.int32)
    origin = np.asarray(origin, dtype=np.float64).ravel()[:3]
    step = float(step)
    ngrid = tuple(int(x) for x in ngrid[:3])
    if outdir:
        os.makedirs(outdir, exist_ok=True)
    afmulator = afm.AFMulator(use_morse=True, nloc=32, use_fire=True)
    atoms_arr, cLJs_arr = _morse_atoms_from_Z(atomPos, atomTypes, params_path=params_path)
    if charges is not None:
        atoms_arr[:, 3] = np.asarray(charges, dtype=np.float32)
    afmulator.atoms_arr = atoms_arr
    afmulator.cLJs_arr = cLJs_arr
    nx, ny, nz = ngrid
    L = np.array([nx * step, ny * step, nz * step], dtype=np.float32)
    afmulator.setup_grid_world(origin, L, ngrid)
    afmulator.make_forcefield()
    afmulator.setup_fdbm_grid_from_img(afmulator.img_FF, ngrid, origin, step)
    osc_n = np.asarray(scan_spec.osc_dir, dtype=np.float64)
    osc_n = osc_n / np.linalg.norm(osc_n)
    amp = float(scan_spec.amplitude)
    pad_x = int(np.ceil(abs(amp * osc_n[0]) / step - 1e-12))
    pad_y = int(np.ceil(abs(amp * osc_n[1]) / step - 1e-12))
    scan_xs = np.asarray(scan_spec.scan_xs, dtype=np.float32)
    scan_ys = np.asarray(scan_spec.scan_ys, dtype=np.float32)
    scan_xs_full = (float(scan_xs[0]) + (np.arange(len(scan_xs) + 2 * pad_x, dtype=np.float64) - pad_x) * step
                    ).astype(np.float32)
    scan_ys_full = (float(scan_ys[0]) + (np.arange(len(scan_ys) + 2 * pad_y, dtype=np.float64) - pad_y) * step
                    ).astype(np.float32)
    required = np.array([scan_spec.scan_margin + pad_x * step, scan_spec.scan_margin + pad_y * step])
    if np.any(required > float(margin) + 1e-9):
        raise ValueError(f"lateral amplitude leaves the force-field grid: required xy margins={required} A exceed "
                         f"margin={margin} A")
    mol_z = float(atomPos[:, 2].max())
    h_scan = np.asarray(scan_spec.h_scan, dtype=np.float32)
    kw = dict(mol_z=mol_z, K_LAT=float(scan_spec.K_LAT), K_RAD=float(scan_spec.K_RAD),
              bond_length=float(scan_spec.bond_length), ppm_mode=True, use_fire=True, osc_dir=scan_spec.osc_dir,
              base_pos=(0., 0., 0.), return_device=True)
    # forward and backward strokes and their dissipation in one relaxation launch (the reference's two
    # scan_fdbm calls and compute_dissipation)
    (FEs_full, tip_disp_full), (FEs_bwd_full, _), E_full = afmulator.scan_fdbm_pair(
        scan_xs_full, scan_ys_full, h_scan, dissipation=(scan_spec.h_scan, scan_spec.h_df, float(scan_spec.amplitude)),
        **kw)
    sx = slice(pad_x, pad_x + len(scan_xs))
    sy = slice(pad_y, pad_y + len(scan_ys))
    FEs = FEs_full[sx, sy].contiguous()
    tip_disp = {k: gpu.to_host(v[sx, sy]) for k, v in tip_disp_full.items()}
    result = shared_postprocess(FEs, scan_spec, tip_disp=tip_disp, backend_name="morse", fft_path="none",
                                E_diss=E_full[sx, sy].contiguous())
    result.tag = tag
    result.atomPos = atomPos
    result.origin = origin
    result.step = step
    result.h_scan = h_scan
    result.osc_dir = osc_n.copy()
    result.path = "Morse"
    result.afmulator = afmulator
    return result
