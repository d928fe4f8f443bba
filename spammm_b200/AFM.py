"""Drop-in replacement of SPAMMM's ``spammm.SPM.AFM`` probe-particle AFM path.

``AFMulator`` keeps the reference's constructor, attributes, method names,
argument meaning, return shapes/dtypes, z-ordering and raised exception types
(spammm/SPM/AFM.py:265-2600), but every computation runs in the sm_100a
kernels of ``libspmb200.so`` through its C ABI.  Host NumPy arrays go in and
come out exactly as in the reference; device-resident variants live in
``spammm_b200.gpu``.  The module-level df functions mirror
``compute_df*`` / ``df_loss_seed`` / ``compute_dissipation``
(AFM.py:3048-3277) and run on the GPU as well.

Differences from the reference, all deliberate:
  * the grid is a torch CUDA tensor (nz,ny,nx,4) instead of a cl.Image and is
    sampled with exact FP32 trilinear weights (the OpenCL texture filter uses
    8-bit fixed-point weights);
  * the FIRE step cap and convergence threshold, compile-time constants in the
    reference (N_RELAX_STEP_MAX=128, F2CONV=1e-8, kernels/AFM.cl:121-122), are
    the instance attributes ``n_relax_max`` / ``f2conv`` with those defaults;
  * plotting / FDBM / contact-surface methods are not part of this path.
"""
import os

import numpy as np
import torch

from . import _lib, gpu
from .FFparams import read_element_types

COULOMB_CONST = 14.3996448915  # [eV*Ang/e^2]
EV_A2_PER_N_M = 1.0 / 16.02176634
N_M_PER_EV_A2 = 16.02176634
K_LAT_HAPALA_N_M = 0.5
K_LAT_HAPALA_EV_A2 = K_LAT_HAPALA_N_M * EV_A2_PER_N_M

N_RELAX_STEP_MAX = 128   # kernels/AFM.cl:121
F2CONV = 1e-8            # kernels/AFM.cl:122
DIRECT_MAX_ATOMS = 128   # spammm/SPM/AFM.py:2105

verbosity = int(os.environ.get("SPAMMM_VERBOSITY", "0") or 0)


def _log(level, msg):
    if verbosity >= level:
        print(msg)


def stiffness_Nm_to_eVA2(k_Nm):
    """Spring constant N/m -> eV/A^2 (AFM.py:73-75)."""
    return float(k_Nm) * EV_A2_PER_N_M


def stiffness_eVA2_to_Nm(k_eVA2):
    return float(k_eVA2) * N_M_PER_EV_A2


def build_scan_xy_points_vectorized(scan_p0, scan_da, scan_db, nx, ny):
    """(nx*ny,4) float32 scan starts p0 + da*ix + db*iy, ix-major (AFM.py:82-95)."""
    p0 = np.asarray(scan_p0, dtype=np.float32).reshape(3)
    da = np.asarray(scan_da, dtype=np.float32).reshape(3)
    db = np.asarray(scan_db, dtype=np.float32).reshape(3)
    ix = np.arange(int(nx), dtype=np.float32)[:, None]
    iy = np.arange(int(ny), dtype=np.float32)[None, :]
    xyz = p0 + da * ix[..., None] + db * iy[..., None]
    pts = np.zeros((int(nx) * int(ny), 4), dtype=np.float32)
    pts[:, :3] = xyz.reshape(-1, 3)
    return pts


def build_scan_points_vectorized(scan_xs, scan_ys, h_scan):
    """(nx*ny*nz,4) float32 (x,y,z,0) grid, C order over (nx,ny,nz) (AFM.py:98-123)."""
    scan_xs = np.asarray(scan_xs, dtype=np.float32)
    scan_ys = np.asarray(scan_ys, dtype=np.float32)
    h_scan = np.asarray(h_scan, dtype=np.float32)
    gx, gy, gz = np.meshgrid(scan_xs, scan_ys, h_scan, indexing="ij")
    pts = np.stack([gx.ravel(), gy.ravel(), gz.ravel(), np.zeros(gx.size, dtype=np.float32)], axis=1)
    return np.ascontiguousarray(pts, dtype=np.float32)


def _raster_points(scan_p0, scan_da, scan_db, nx, ny):
    """p0 + da*ix + db*iy with the reference loop's dtype semantics (AFM.py:993-997)."""
    p0 = np.asarray(scan_p0)
    da = np.asarray(scan_da)
    db = np.asarray(scan_db)
    ix = np.arange(nx, dtype=np.float32)[:, None, None]
    iy = np.arange(ny, dtype=np.float32)[None, :, None]
    xyz = (p0 + da * ix) + db * iy
    pts = np.zeros((nx * ny, 4), dtype=np.float32)
    pts[:, :3] = xyz.reshape(-1, 3)
    return pts


class _Queue:
    """Stand-in for the reference's cl.CommandQueue: ``finish()`` synchronises."""

    def finish(self):
        torch.cuda.synchronize()


# The reference kernels (kernels/AFM.cl, kernels/contact_surface.cl) this library implements, by the
# reference's names: callers introspect AFMulator.prg.all_kernels() for them.
IMPLEMENTED_KERNELS = (
    "evalLJC_QZs_toImg", "evalMorseC_QZs_toImg", "relaxStrokes", "relaxStrokesTilted", "relaxStrokes2D",
    "getFEinStrokesTilted", "convolveZ", "izoZ", "relaxStrokesTiltedMorseDirect", "morseDirectStateAdjoint",
    "morseDirectParamPartials", "reduceMorseDirectParamPartials", "cs_brute_afm_morse_c_points")


class _Kernel:
    def __init__(self, name):
        self.function_name = name


class _Program:
    """Stand-in for the reference's compiled cl.Program (AFMulator.prg): all_kernels() lists the reference
    kernels whose work this library's CUDA kernels do."""

    def all_kernels(self):
        return [_Kernel(n) for n in IMPLEMENTED_KERNELS]


class _Device:
    def __init__(self, index):
        props = torch.cuda.get_device_properties(index)
        self.name = props.name
        self.vendor = "NVIDIA Corporation"
        self.opencl_c_version = "none (CUDA sm_100a kernels)"
        self.max_compute_units = props.multi_processor_count
        self.global_mem_size = props.total_memory


class _Context:
    """Stand-in for the reference's cl.Context (AFMulator.ctx): devices[0] describes the CUDA device."""

    def __init__(self, index):
        self.devices = [_Device(index)]


class _Molecule:
    def __init__(self, apos, enames, qs, lvec=None):
        self.apos = apos
        self.enames = enames
        self.qs = qs
        self.natoms = len(enames)
        self.lvec = lvec


# Chemical element symbols in order of atomic number (Z = index + 1).
ELEMENT_SYMBOLS = (
    "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar", "K", "Ca",
    "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y",
    "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I", "Xe", "Cs", "Ba", "La", "Ce",
    "Pr", "Nd", "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W", "Re", "Os", "Ir",
    "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th", "Pa", "U", "Np", "Pu", "Am", "Cm",
    "Bk", "Cf", "Es", "Fm", "Md", "No", "Lr", "Rf", "Db", "Sg", "Bh", "Hs", "Mt", "Ds", "Rg", "Cn", "Nh", "Fl", "Mc",
    "Lv", "Ts", "Og")
_Z_OF_SYMBOL = {e: i + 1 for i, e in enumerate(ELEMENT_SYMBOLS)}


def load_xyz_molecule(xyz_path, nmax=10000):
    """.xyz reader with the line rules of the reference's loader (AtomicSystem(fname) ->
    atomicUtils.load_xyz with bReadN, spammm/AtomicSystem.py:35-90, spammm/atomicUtils.py:1212):
    an atom line is "element x y z [q]" where the element is an atomic number or a chemical
    symbol; any other line before the first atom either gives the atom count (an integer first
    word) or is the comment; reading stops after the count.  A comment starting with "lvs" holds
    the periodic cell vectors (the first nine numbers on it, row-major)."""
    apos, enames, qs = [], [], []
    comment = None
    with open(xyz_path) as f:
        for line in f:
            w = line.split()
            atom = None
            try:
                xyz = (float(w[1]), float(w[2]), float(w[3]))
                try:
                    q = float(w[4])
                except (IndexError, ValueError):
                    q = 0.0
                try:
                    name = ELEMENT_SYMBOLS[int(w[0]) - 1]
                except ValueError:
                    name = w[0]
                    if name not in _Z_OF_SYMBOL:
                        raise KeyError(name)
                atom = (xyz, name, q)
            except (IndexError, ValueError, KeyError):
                if not apos:
                    try:
                        nmax = int(w[0])
                    except (IndexError, ValueError):
                        comment = line.strip()
            if atom is not None:
                apos.append(atom[0])
                enames.append(atom[1])
                qs.append(atom[2])
            if len(apos) >= nmax:
                break
    lvec = None
    if comment is not None and comment[:3] == "lvs":
        nums = []
        for tok in comment.split():
            try:
                nums.append(float(tok))
            except ValueError:
                continue
        if len(nums) < 9:
            raise ValueError(f"{xyz_path}: 'lvs' line holds {len(nums)} numbers, need 9")
        lvec = np.array(nums[:9], dtype=np.float64).reshape(3, 3)
    return _Molecule(np.array(apos, dtype=np.float64).reshape(-1, 3), enames, np.array(qs, dtype=np.float64), lvec)


class AFMulator:
    """GPU probe-particle AFM simulator (LJ/Morse + point charges), sm_100a.

    Mirrors ``spammm.SPM.AFM.AFMulator`` (spammm/SPM/AFM.py:265).  Coordinate
    convention: grid node i sits at origin + i*L/n; normalized grid
    coordinates carry the +0.5/n texel-centre offset.
    """

    @staticmethod
    def _make_dinv_axis_aligned(L, origin, n):
        """(dinvA,dinvB,dinvC) with the half-texel offset (AFM.py:274-285)."""
        nx, ny, nz = n
        dinvA = np.array([1. / L[0], 0., 0., -origin[0] / L[0] + 0.5 / nx], dtype=np.float32)
        dinvB = np.array([0., 1. / L[1], 0., -origin[1] / L[1] + 0.5 / ny], dtype=np.float32)
        dinvC = np.array([0., 0., 1. / L[2], -origin[2] / L[2] + 0.5 / nz], dtype=np.float32)
        return dinvA, dinvB, dinvC

    @staticmethod
    def _make_dinv_lvec(invMT, n):
        nx, ny, nz = n
        dinvA = np.array([invMT[0, 0], invMT[0, 1], invMT[0, 2], 0.5 / nx], dtype=np.float32)
        dinvB = np.array([invMT[1, 0], invMT[1, 1], invMT[1, 2], 0.5 / ny], dtype=np.float32)
        dinvC = np.array([invMT[2, 0], invMT[2, 1], invMT[2, 2], 0.5 / nz], dtype=np.float32)
        return dinvA, dinvB, dinvC

    DEFAULT_tipA = np.array([1., 0., 0., 0.], dtype=np.float32)
    DEFAULT_tipB = np.array([0., 1., 0., 0.], dtype=np.float32)
    DEFAULT_tipC = np.array([0., 0., 1., -0.1], dtype=np.float32)
    DEFAULT_stiffness = np.array([-0.03, -0.03, -0.03, -1.0], dtype=np.float32)
    DEFAULT_dpos0 = np.array([0., 0., -4.0, 4.0], dtype=np.float32)
    DEFAULT_relax_pars = np.array([0.5, 0.1, 0.02, 0.5], dtype=np.float32)
    DEFAULT_surfFF = np.array([0., 0., 0., 0.], dtype=np.float32)
    DEFAULT_tipQs = np.array([0., -0.1, 0.1, 0.], dtype=np.float32)
    DEFAULT_tipQZs = np.array([0., 1.8, 3.6, 0.], dtype=np.float32)

    def __init__(self, cl_src_dir=None, use_morse=False, nloc=32, use_fire=True):
        _lib.require_cuda()
        self.use_morse = use_morse
        self.use_fire = bool(use_fire)
        self.nloc = nloc
        self.cl_src_dir = cl_src_dir
        self.queue = _Queue()
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.prg = _Program()
        self.ctx = _Context(self.device.index)
        props = torch.cuda.get_device_properties(self.device)
        self._max_alloc = int(props.total_memory)
        self._global_mem = int(props.total_memory)
        self._vram_bytes = 0
        self.n_relax_max = N_RELAX_STEP_MAX
        self.f2conv = F2CONV
        # not in the reference: Newton-polish every relaxed state (SPM_FLAG_POLISH) so that FEs and
        # displacements sit at the equilibrium of the interpolated field instead of FIRE's stopping point
        self.newton_polish = False
        self.mol = self.elem_types = None
        self.atoms_arr = self.cLJs_arr = None
        self.img_FF = self.n = self.p0 = self.L = None
        self.dA = self.dB = self.dC = None
        self.dinvA = self.dinvB = self.dinvC = None
        self.mol_shift = np.zeros(3, dtype=np.float32)
        self.tipA = self.DEFAULT_tipA.copy()
        self.tipB = self.DEFAULT_tipB.copy()
        self.tipC = self.DEFAULT_tipC.copy()
        self.stiffness = self.DEFAULT_stiffness.copy()
        self.dpos0 = self.DEFAULT_dpos0.copy()
        self.relax_pars = self.DEFAULT_relax_pars.copy()
        self.surfFF = self.DEFAULT_surfFF.copy()
        self.tipQs = self.DEFAULT_tipQs.copy()
        self.tipQZs = self.DEFAULT_tipQZs.copy()
        self.img_FF_fdbm = None
        self.fdbm_dinvA = self.fdbm_dinvB = self.fdbm_dinvC = None
        self.fdbm_origin = self.fdbm_step = self.fdbm_shape = None
        self._morse_direct_fwd_state = None

    # ---------------------------------------------------------------- buffers
    def realloc_forcefield_buffers(self, na):
        """Kept for API compatibility: device buffers come from torch's allocator."""
        self._na_alloc = int(na)

    def realloc_scan_buffers(self, n_scan, nz):
        self._scan_alloc = (int(n_scan), int(nz))

    def _check_alloc(self, nbytes, what):
        if nbytes > self._max_alloc:
            raise MemoryError(f"{what} needs {nbytes} bytes ({nbytes / 1024 ** 3:.3f} GB) > device memory "
                              f"{self._max_alloc / 1024 ** 3:.3f} GB")

    def _flags_params(self, **kw):
        kw.setdefault("max_iter", self.n_relax_max)
        kw.setdefault("f2conv", self.f2conv)
        kw.setdefault("fire", self.use_fire)
        kw.setdefault("polish", self.newton_polish)
        return _lib.make_scan_params(**kw)

    # ---------------------------------------------------------------- FDBM grid
    def setup_fdbm_grid(self, F_total, origin, step):
        """Upload an (nx,ny,nz,4) force field (AFM.py:387-411)."""
        F_total = np.asarray(F_total)
        nx, ny, nz = F_total.shape[:3]
        Lx, Ly, Lz = nx * step, ny * step, nz * step
        F_img = np.ascontiguousarray(F_total.transpose(2, 1, 0, 3), dtype=np.float32)
        self._check_alloc(F_img.nbytes, "setup_fdbm_grid")
        self.img_FF_fdbm = torch.from_numpy(F_img).to(self.device)
        self.fdbm_dinvA, self.fdbm_dinvB, self.fdbm_dinvC = self._make_dinv_axis_aligned(
            np.array([Lx, Ly, Lz]), np.asarray(origin, dtype=np.float32), (nx, ny, nz))
        self.fdbm_origin = np.asarray(origin, dtype=np.float32)
        self.fdbm_step = float(step)
        self.fdbm_shape = (nx, ny, nz)
        _log(1, f"AFMulator.setup_fdbm_grid: grid={nx}x{ny}x{nz} step={step:.3f}")

    def setup_fdbm_grid_from_img(self, img_F, shape, origin, step):
        """Device-side grid copy (AFM.py:413-429); img_F is a (nz,ny,nx,4) CUDA tensor."""
        nx, ny, nz = [int(x) for x in shape[:3]]
        Lx, Ly, Lz = nx * step, ny * step, nz * step
        if self.img_FF_fdbm is None or self.fdbm_shape != (nx, ny, nz):
            self.img_FF_fdbm = torch.empty((nz, ny, nx, 4), dtype=torch.float32, device=self.device)
        self.img_FF_fdbm.copy_(img_F.reshape(nz, ny, nx, 4))
        self.fdbm_dinvA, self.fdbm_dinvB, self.fdbm_dinvC = self._make_dinv_axis_aligned(
            np.array([Lx, Ly, Lz]), np.asarray(origin, dtype=np.float32), (nx, ny, nz))
        self.fdbm_origin = np.asarray(origin, dtype=np.float32)
        self.fdbm_step = float(step)
        self.fdbm_shape = (nx, ny, nz)

    def download_image_rgba_xyz(self, img, shape):
        """(nz,ny,nx,4) device grid -> (nx,ny,nz,4) host array (AFM.py:474-481)."""
        nx, ny, nz = [int(x) for x in shape[:3]]
        host = gpu.to_host(img.reshape(nz, ny, nx, 4))
        return np.ascontiguousarray(host.transpose(2, 1, 0, 3))

    # ---------------------------------------------------------------- scans
    def _scan_fdbm_points(self, scan_xs, scan_ys, probe_heights, mol_z, bond_length, base, reverse):
        nx_s, ny_s, nz_s = len(scan_xs), len(scan_ys), len(probe_heights)
        heights_sorted = np.sort(probe_heights)
        dh = float(heights_sorted[-1] - heights_sorted[0]) / max(nz_s - 1, 1) if nz_s > 1 else 0.
        if reverse:
            dTip = np.array([0., 0., +dh, 0.], dtype=np.float32)
            z_start = float(heights_sorted[0]) + mol_z + bond_length + float(base[2])
        else:
            dTip = np.array([0., 0., -dh, 0.], dtype=np.float32)
            z_start = float(heights_sorted[-1]) + mol_z + bond_length + float(base[2])
        gx, gy = np.meshgrid(scan_xs, scan_ys, indexing="ij")
        pts = np.zeros((nx_s * ny_s, 4), dtype=np.float32)
        pts[:, 0] = gx.ravel() + base[0]
        pts[:, 1] = gy.ravel() + base[1]
        pts[:, 2] = z_start
        return pts, dTip

    def scan_fdbm(self, scan_xs, scan_ys, probe_heights, mol_z=0.0, ppm_mode=True, use_fire=True,
                  K_LAT=0.03, K_RAD=20.0, bond_length=3.0, stiffness=None, dpos0=None, relax_pars=None,
                  osc_dir=(0., 0., 1.), base_pos=(0., 0., 0.), reverse=False, return_device=False):
        """relaxStrokes over a 2D scan (AFM.py:493-642).

        Returns (FEs_relax (nx,ny,nz,4) float32 with iz=0 the lowest height,
        tip_disp {'dx','dy','dz'} each (nx,ny,nz)).  With ``return_device`` the
        arrays stay CUDA tensors.
        """
        base, stiffness_v, dpos0_v, relax_pars_v = self._scan_fdbm_setup(osc_dir, base_pos, use_fire, K_LAT, K_RAD,
                                                                         bond_length, stiffness, dpos0, relax_pars)
        nx_s, ny_s, nz_s = len(scan_xs), len(scan_ys), len(probe_heights)
        pts, dTip = self._scan_fdbm_points(scan_xs, scan_ys, probe_heights, mol_z, bond_length, base, reverse)
        n_scan = nx_s * ny_s
        self._check_alloc(n_scan * nz_s * 16, "scan_fdbm FEs")
        self.realloc_scan_buffers(n_scan, nz_s)
        P = self._flags_params(dinv=(self.fdbm_dinvA, self.fdbm_dinvB, self.fdbm_dinvC), dTip=dTip,
                               stiffness=stiffness_v, dpos0=dpos0_v, relax_params=relax_pars_v, nz=nz_s,
                               flip_z=not reverse, raster_ny=ny_s)
        FEs, disps = gpu.relax_strokes(self.img_FF_fdbm, P, torch.from_numpy(pts).to(self.device))
        return self._scan_outputs(FEs, disps, (nx_s, ny_s, nz_s), return_device)

    def scan_fdbm_pair(self, scan_xs, scan_ys, probe_heights, mol_z=0.0, ppm_mode=True, use_fire=True,
                       K_LAT=0.03, K_RAD=20.0, bond_length=3.0, stiffness=None, dpos0=None, relax_pars=None,
                       osc_dir=(0., 0., 1.), base_pos=(0., 0., 0.), return_device=False, dissipation=None):
        """The forward and the backward (reverse=True) strokes of scan_fdbm in
        one relaxation launch (SPM_FLAG_PAIRED), as run_morse_pp_afm and
        run_fdbm_pp_from_density (AFM_utils.py:3537-3553, 4091-4108) take them
        for the dissipation.  Each stroke's arithmetic is that of the separate
        calls, so the results are theirs bit for bit.

        Returns ((FEs_fwd, tip_disp_fwd), (FEs_bwd, tip_disp_bwd)), both with
        iz=0 the lowest height, as two scan_fdbm calls return them.
        dissipation=(h_scan, h_df, amp): also compute_dissipation(FEs_fwd,
        FEs_bwd, h_scan, h_df, amp, osc_dir) in the same launch (the lane that
        finishes a pixel's second stroke integrates it; spm_dissipation's
        arithmetic, bit for bit) and return it third, (nx, ny, len(h_df))."""
        base, stiffness_v, dpos0_v, relax_pars_v = self._scan_fdbm_setup(osc_dir, base_pos, use_fire, K_LAT, K_RAD,
                                                                         bond_length, stiffness, dpos0, relax_pars)
        nx_s, ny_s, nz_s = len(scan_xs), len(scan_ys), len(probe_heights)
        pts_f, dTip = self._scan_fdbm_points(scan_xs, scan_ys, probe_heights, mol_z, bond_length, base, False)
        pts_b, _ = self._scan_fdbm_points(scan_xs, scan_ys, probe_heights, mol_z, bond_length, base, True)
        n_scan = nx_s * ny_s
        self._check_alloc(2 * n_scan * nz_s * 16, "scan_fdbm_pair FEs")
        self.realloc_scan_buffers(2 * n_scan, nz_s)
        # the two point sets form one (2 nx) x ny raster: forward strokes, then backward ones
        P = self._flags_params(dinv=(self.fdbm_dinvA, self.fdbm_dinvB, self.fdbm_dinvC), dTip=dTip,
                               stiffness=stiffness_v, dpos0=dpos0_v, relax_params=relax_pars_v, nz=nz_s,
                               flip_z=True, raster_ny=ny_s, paired=True)
        pts = torch.from_numpy(np.concatenate([pts_f, pts_b])).to(self.device)
        shape = (nx_s, ny_s, nz_s)
        if dissipation is None:
            FEs, disps = gpu.relax_strokes(self.img_FF_fdbm, P, pts)
            return (self._scan_outputs(FEs[:n_scan], disps[:n_scan], shape, return_device),
                    self._scan_outputs(FEs[n_scan:], disps[n_scan:], shape, return_device))
        h_scan, h_df, amp = dissipation
        FEs, disps, E = gpu.relax_pair_dissipation(self.img_FF_fdbm, P, pts, h_scan, h_df, amp, osc_dir)
        E = E.view(nx_s, ny_s, -1)
        return (self._scan_outputs(FEs[:n_scan], disps[:n_scan], shape, return_device),
                self._scan_outputs(FEs[n_scan:], disps[n_scan:], shape, return_device),
                E if return_device else gpu.to_host(E))

    def _scan_fdbm_setup(self, osc_dir, base_pos, use_fire, K_LAT, K_RAD, bond_length, stiffness, dpos0,
                         relax_pars):
        """Validated scan frame and probe vectors of scan_fdbm (AFM.py:548-575)."""
        if self.img_FF_fdbm is None:
            raise AssertionError("call setup_fdbm_grid() first")
        osc_n = np.asarray(osc_dir, dtype=np.float32)
        osc_norm = float(np.linalg.norm(osc_n))
        if osc_n.shape != (3,) or not np.isfinite(osc_norm) or osc_norm <= 0.0:
            raise ValueError(f"osc_dir must be a finite non-zero vector, got {osc_dir!r}")
        base = np.asarray(base_pos, dtype=np.float32)
        if base.shape != (3,) or not np.isfinite(base).all():
            raise ValueError(f"base_pos must contain three finite coordinates, got {base_pos!r}")
        stiffness_v = (np.array([-K_LAT, -K_LAT, -K_LAT, -K_RAD], dtype=np.float32) if stiffness is None
                       else np.array(stiffness, dtype=np.float32))
        dpos0_v = (np.array([0., 0., -bond_length, bond_length], dtype=np.float32) if dpos0 is None
                   else np.array(dpos0, dtype=np.float32))
        if relax_pars is not None:
            relax_pars_v = np.array(relax_pars, dtype=np.float32)
        elif use_fire:
            relax_pars_v = self.relax_pars.copy()
        else:
            relax_pars_v = np.array([0.3, 0.2, 0.03, 0.3], dtype=np.float32)
        return base, stiffness_v, dpos0_v, relax_pars_v

    @staticmethod
    def _scan_outputs(FEs, disps, shape, return_device):
        FEs = FEs.reshape(*shape, 4)
        disps = disps.reshape(*shape, 4)
        if not return_device:
            FEs = gpu.to_host(FEs)
            disps = gpu.to_host(disps[..., :3].contiguous())  # the fourth channel is 0: not copied
        return FEs, {"dx": disps[..., 0], "dy": disps[..., 1], "dz": disps[..., 2]}

    def scan_fdbm_2d(self, scan_xs, scan_ys, probe_heights, mol_z=0.0, K_LAT=0.03, dt=0.3, damp=0.2,
                     return_device=False):
        """relaxStrokes2D over a 2D scan (AFM.py:644-704): z fixed per height
        slice, x,y relaxed by damped MD from the anchor (reset per slice).

        Returns (FEs_relax (nx,ny,nz,4) float32 with iz=0 the lowest height,
        tip_disp {'dx','dy','dz'} each (nx,ny,nz); dz = 0)."""
        if self.img_FF_fdbm is None:
            raise AssertionError("call setup_fdbm_grid() first")
        nx_s, ny_s, nz_s = len(scan_xs), len(scan_ys), len(probe_heights)
        heights_desc = np.sort(np.asarray(probe_heights, dtype=np.float64))[::-1]
        dh = float(heights_desc[0] - heights_desc[-1]) / max(nz_s - 1, 1) if nz_s > 1 else 0.
        z_start = float(heights_desc[0]) + mol_z
        gx, gy = np.meshgrid(scan_xs, scan_ys, indexing="ij")
        pts = np.zeros((nx_s * ny_s, 4), dtype=np.float32)
        pts[:, 0] = gx.ravel()
        pts[:, 1] = gy.ravel()
        pts[:, 2] = z_start
        self._check_alloc(nx_s * ny_s * nz_s * 16, "scan_fdbm_2d FEs")
        self.realloc_scan_buffers(nx_s * ny_s, nz_s)
        P = self._flags_params(dinv=(self.fdbm_dinvA, self.fdbm_dinvB, self.fdbm_dinvC), dTip=[0., 0., -dh, 0.],
                               stiffness=[K_LAT, 0., 0., 0.], relax_params=[dt, damp, 0., 0.], nz=nz_s, fire=False,
                               flip_z=True, raster_ny=ny_s, polish=False)
        FEs, disps = gpu.relax_2d(self.img_FF_fdbm, P, torch.from_numpy(pts).to(self.device))
        FEs = FEs.reshape(nx_s, ny_s, nz_s, 4)
        disps = disps.reshape(nx_s, ny_s, nz_s, 4)
        _log(1, f"AFMulator.scan_fdbm_2d: Fz min={float(FEs[..., 2].min()):.4f}  max={float(FEs[..., 2].max()):.4f}"
                f"  mean={float(FEs[..., 2].mean()):.4f} eV/Ang")
        if not return_device:
            FEs = gpu.to_host(FEs)
            disps = gpu.to_host(disps)
        tip_disp = {"dx": disps[..., 0], "dy": disps[..., 1], "dz": disps[..., 2]}
        return FEs, tip_disp

    # ---------------------------------------------------------------- molecule
    def load_molecule(self, xyz_path):
        self.mol = load_xyz_molecule(xyz_path)
        _log(1, f"AFMulator.load_molecule: {self.mol.natoms} atoms")
        return self.mol

    def assign_params(self, params_path=None, tip_R=1.452, tip_E=0.0006808, tip_alpha=-1.8):
        """LJ (c6,c12) or Morse (R0,E0,alpha) from ElementTypes.dat (AFM.py:730-768):
        R0 = tip_R + RvdW, E0 = sqrt(|tip_E*EvdW|); LJ c6 = 2 E0 R0^6, c12 = E0 R0^12."""
        assert self.mol is not None, "call load_molecule() first"
        et = read_element_types(params_path)
        self.elem_types = et
        na = self.mol.natoms
        atoms = np.zeros((na, 4), dtype=np.float32)
        atoms[:, :3] = self.mol.apos[:na, :3].astype(np.float32)
        if self.mol.qs is not None:
            atoms[:, 3] = self.mol.qs[:na].astype(np.float32)
        if self.use_morse:
            cMs = np.zeros((na, 4), dtype=np.float32)
            for ia, ename in enumerate(self.mol.enames[:na]):
                e = et.get(ename)
                assert e is not None, f"Element '{ename}' not in ElementTypes.dat"
                R0 = tip_R + e.RvdW
                E0 = np.sqrt(abs(tip_E * e.EvdW))
                cMs[ia] = [R0, E0, tip_alpha, 0.]
            self.cLJs_arr = cMs
        else:
            cLJs = np.zeros((na, 2), dtype=np.float32)
            for ia, ename in enumerate(self.mol.enames[:na]):
                e = et.get(ename)
                assert e is not None, f"Element '{ename}' not in ElementTypes.dat"
                R0 = tip_R + e.RvdW
                E0 = np.sqrt(abs(tip_E * e.EvdW))
                cLJs[ia] = [2. * E0 * R0 ** 6, E0 * R0 ** 12]
            self.cLJs_arr = cLJs
        self.atoms_arr = atoms
        return atoms, self.cLJs_arr

    # ---------------------------------------------------------------- grid frames
    def setup_grid(self, n=(100, 100, 60), L=None, margin=3.0, z_top=12.0, shift_atoms=True):
        """Grid around the molecule (AFM.py:772-811)."""
        assert self.atoms_arr is not None, "call assign_params() first"
        apos = self.atoms_arr[:, :3]
        mn, mx = apos.min(axis=0), apos.max(axis=0)
        if L is None:
            L = np.array([(mx[0] - mn[0]) + 2 * margin, (mx[1] - mn[1]) + 2 * margin,
                          (mx[2] - mn[2]) + margin + z_top], dtype=np.float32)
        else:
            L = np.array(L, dtype=np.float32)
        self.n = np.array(n, dtype=np.int32)
        nx, ny, nz = n
        p0_raw = np.array([mn[0] - margin, mn[1] - margin, mn[2] - margin / 2], dtype=np.float32)
        if shift_atoms:
            self.mol_shift = -p0_raw
            self.atoms_arr[:, :3] += self.mol_shift
            self.p0 = np.zeros(4, dtype=np.float32)
            ox, oy, oz = 0., 0., 0.
        else:
            self.mol_shift = np.zeros(3, dtype=np.float32)
            self.p0 = np.array([p0_raw[0], p0_raw[1], p0_raw[2], 0.], dtype=np.float32)
            ox, oy, oz = float(p0_raw[0]), float(p0_raw[1]), float(p0_raw[2])
        self.dA = np.array([L[0] / nx, 0., 0., 0.], dtype=np.float32)
        self.dB = np.array([0., L[1] / ny, 0., 0.], dtype=np.float32)
        self.dC = np.array([0., 0., L[2] / nz, 0.], dtype=np.float32)
        self.dinvA, self.dinvB, self.dinvC = self._make_dinv_axis_aligned(
            L, np.array([ox, oy, oz], dtype=np.float32), (nx, ny, nz))
        self.L = L
        self._grid_bytes = int(nx * ny * nz * 16)
        return L

    def setup_grid_world(self, p0_xyz, L_xyz, n):
        """World-frame grid box, no atom shift (AFM.py:813-837)."""
        assert self.atoms_arr is not None, "call assign_params() first"
        nx, ny, nz = [int(v) for v in n]
        p0 = np.asarray(p0_xyz, dtype=np.float32).reshape(3)
        L = np.asarray(L_xyz, dtype=np.float32).reshape(3)
        if np.any(L <= 0) or min(nx, ny, nz) < 2:
            raise ValueError(f"setup_grid_world: invalid p0={p0} L={L} n={n}")
        self.n = np.array([nx, ny, nz], dtype=np.int32)
        self.mol_shift = np.zeros(3, dtype=np.float32)
        self.p0 = np.array([p0[0], p0[1], p0[2], 0.], dtype=np.float32)
        self.dA = np.array([L[0] / nx, 0., 0., 0.], dtype=np.float32)
        self.dB = np.array([0., L[1] / ny, 0., 0.], dtype=np.float32)
        self.dC = np.array([0., 0., L[2] / nz, 0.], dtype=np.float32)
        self.dinvA, self.dinvB, self.dinvC = self._make_dinv_axis_aligned(L, p0, (nx, ny, nz))
        self.L = L
        self._grid_bytes = int(nx * ny * nz * 16)
        return L

    def setup_grid_lvec(self, n=(100, 100, 60), margin_z=2.0, z_top=12.0):
        """Primitive-cell grid along mol.lvec (AFM.py:839-893)."""
        assert self.atoms_arr is not None, "call assign_params() first"
        assert self.mol is not None and getattr(self.mol, "lvec", None) is not None, \
            "setup_grid_lvec requires mol.lvec (periodic system)"
        nx, ny, nz = [int(x) for x in n]
        if nx <= 1 or ny <= 1 or nz <= 1:
            raise ValueError(f"setup_grid_lvec: invalid n={n}")
        a = self.mol.lvec[0, :3].astype(np.float32)
        b = self.mol.lvec[1, :3].astype(np.float32)
        apos = self.atoms_arr[:, :3]
        zmin = float(apos[:, 2].min())
        zmax = float(apos[:, 2].max())
        Lz = (zmax - zmin) + float(margin_z) + float(z_top)
        if Lz <= 0:
            raise ValueError(f"setup_grid_lvec: invalid Lz={Lz}")
        p0z = zmin - 0.5 * float(margin_z)
        self.mol_shift = np.array([0., 0., -p0z], dtype=np.float32)
        self.atoms_arr[:, :3] += self.mol_shift[None, :]
        self.n = np.array([nx, ny, nz], dtype=np.int32)
        self.p0 = np.zeros(4, dtype=np.float32)
        self.dA = np.array([a[0] / nx, a[1] / nx, a[2] / nx, 0.], dtype=np.float32)
        self.dB = np.array([b[0] / ny, b[1] / ny, b[2] / ny, 0.], dtype=np.float32)
        self.dC = np.array([0., 0., Lz / nz, 0.], dtype=np.float32)
        M = np.stack([a, b, np.array([0., 0., Lz], dtype=np.float32)], axis=1).astype(np.float64)
        det = float(np.linalg.det(M))
        if abs(det) < 1e-12:
            raise ValueError(f"setup_grid_lvec: singular cell matrix det={det}")
        invMT = np.linalg.inv(M).T.astype(np.float32)
        self.dinvA, self.dinvB, self.dinvC = self._make_dinv_lvec(invMT, (nx, ny, nz))
        self.L = np.array([np.linalg.norm(a), np.linalg.norm(b), Lz], dtype=np.float32)
        self._grid_bytes = int(nx * ny * nz * 16)
        return self.L

    # ---------------------------------------------------------------- stage (a)
    def make_forcefield(self, bAlloc=True):
        """Build the LJ/Morse + Coulomb grid on the GPU (AFM.py:897-946)."""
        assert self.n is not None, "call setup_grid() first"
        nx, ny, nz = (int(v) for v in self.n)
        self._check_alloc(nx * ny * nz * 16, "FF image")
        if bAlloc:
            self.realloc_forcefield_buffers(len(self.atoms_arr))
        if self.img_FF is None or tuple(self.img_FF.shape) != (nz, ny, nx, 4):
            self.img_FF = torch.empty((nz, ny, nx, 4), dtype=torch.float32, device=self.device)
        kind = _lib.SPM_KIND_MORSE if self.use_morse else _lib.SPM_KIND_LJ
        atoms = torch.from_numpy(np.ascontiguousarray(self.atoms_arr, dtype=np.float32)).to(self.device)
        prm = torch.from_numpy(np.ascontiguousarray(self.cLJs_arr, dtype=np.float32)).to(self.device)
        gpu.grid_build(kind, atoms, prm, (nx, ny, nz), self.p0, self.dA, self.dB, self.dC, self.tipQs, self.tipQZs,
                       out=self.img_FF)

    # ---------------------------------------------------------------- stage (b)
    def _auto_scan_box(self, nx_s, ny_s):
        apos = self.atoms_arr[:, :3]
        mn, mx = apos.min(axis=0), apos.max(axis=0)
        x0 = mn[0] + (mx[0] - mn[0]) * 0.05
        y0 = mn[1] + (mx[1] - mn[1]) * 0.05
        clearance = 5.0
        z0 = float(mx[2]) + clearance + abs(float(self.dpos0[2]))
        scan_p0 = np.array([x0, y0, z0], dtype=np.float32)
        scan_da = np.array([(mx[0] - mn[0]) * 0.9 / max(nx_s - 1, 1), 0., 0.], dtype=np.float32)
        scan_db = np.array([0., (mx[1] - mn[1]) * 0.9 / max(ny_s - 1, 1), 0.], dtype=np.float32)
        return scan_p0, scan_da, scan_db

    def run_scan(self, nxy=(50, 50), nz=60, dtip=-0.1, scan_p0=None, scan_da=None, scan_db=None, bAlloc=True,
                 osc_dir=(0., 0., 1.), return_device=False):
        """relaxStrokesTilted scan (AFM.py:950-1010) -> (FEs (nx,ny,nz,4), pts (nx,ny,3))."""
        assert self.img_FF is not None, "call make_forcefield() first"
        nx_s, ny_s = nxy
        n_scan = nx_s * ny_s
        if scan_p0 is None:
            scan_p0, scan_da, scan_db = self._auto_scan_box(nx_s, ny_s)
        pts = _raster_points(scan_p0, scan_da, scan_db, nx_s, ny_s)
        self._check_alloc(n_scan * nz * 16, "run_scan: FEs buffer")
        osc_n = np.asarray(osc_dir, dtype=np.float32)
        osc_norm = float(np.linalg.norm(osc_n))
        if osc_n.shape != (3,) or not np.isfinite(osc_norm) or osc_norm <= 0.0:
            raise ValueError(f"osc_dir must be a finite non-zero vector, got {osc_dir!r}")
        tipC = self.tipC.copy()
        tipC[3] = np.float32(dtip)
        nxg, nyg, nzg = (int(v) for v in self.n)
        P = self._flags_params(dinv=(self.dinvA, self.dinvB, self.dinvC), tipA=self.tipA, tipB=self.tipB, tipC=tipC,
                               stiffness=self.stiffness, dpos0=self.dpos0, relax_params=self.relax_pars,
                               surfFF=self.surfFF, nz=nz, raster_ny=ny_s)
        FEs = gpu.relax_strokes_tilted(self.img_FF, P, torch.from_numpy(pts).to(self.device))
        FEs = FEs.reshape(nx_s, ny_s, nz, 4)
        if not return_device:
            FEs = gpu.to_host(FEs)
        return FEs, pts[:, :3].reshape(nx_s, ny_s, 3)

    def get_raw_FE(self, nxy=(60, 60), nz=21, dtip=-0.2, scan_p0=None, scan_da=None, scan_db=None, bAlloc=True,
                   osc_dir=(0., 0., 1.)):
        """Unrelaxed sampling (AFM.py:2523-2580) -> (FEs (nx,ny,nz,4), pts (nx,ny,3))."""
        assert self.img_FF is not None, "call make_forcefield() first"
        nx_s, ny_s = nxy
        n_scan = nx_s * ny_s
        if scan_p0 is None:
            scan_p0, scan_da, scan_db = self._auto_scan_box(nx_s, ny_s)
        pts = _raster_points(scan_p0, scan_da, scan_db, nx_s, ny_s)
        self._check_alloc(n_scan * nz * 16, "get_raw_FE: FEs buffer")
        osc_n = np.asarray(osc_dir, dtype=np.float32)
        osc_norm = float(np.linalg.norm(osc_n))
        if osc_n.shape != (3,) or not np.isfinite(osc_norm) or osc_norm <= 0.0:
            raise ValueError(f"osc_dir must be a finite non-zero vector, got {osc_dir!r}")
        dTip = np.array([0., 0., dtip, 0.], dtype=np.float32)
        P = self._flags_params(dinv=(self.dinvA, self.dinvB, self.dinvC), tipA=self.tipA, tipB=self.tipB,
                               tipC=self.tipC, dTip=dTip, dpos0=self.dpos0, nz=nz, raster_ny=ny_s, polish=False)
        FEs = gpu.fe_in_strokes_tilted(self.img_FF, P, torch.from_numpy(pts).to(self.device))
        return gpu.to_host(FEs.reshape(nx_s, ny_s, nz, 4)), pts[:, :3].reshape(nx_s, ny_s, 3)

    def _brute_afm_morse_c_queries(self, queries):
        """Uncapped Morse + Coulomb sums at arbitrary (n,3) points -> (E (n,), F (n,3)) float32
        (AFM.py:1051-1067, the direct reference of the grid builder)."""
        assert self.use_morse and self.atoms_arr is not None and self.cLJs_arr is not None
        q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, 3)
        out = gpu.to_host(gpu.pair_fe_points(_lib.SPM_KIND_MORSE, self.atoms_arr, self.cLJs_arr,
                                             torch.from_numpy(q).to(self.device), self.tipQs, self.tipQZs))
        return out[:, 3], out[:, :3]

    @property
    def mol_z(self):
        if self.atoms_arr is None:
            return 0.0
        return float(self.atoms_arr[:, 2].max())

    def get_df(self, FEs, k_tip=1800.0):
        """-mean_z(dFz/dz)/(2 k_tip) with unit z spacing (AFM.py:2591-2599) -> (nx,ny)."""
        FEs = np.asarray(FEs)
        vol = np.zeros(FEs.shape[:3] + (4,), dtype=np.float32)
        vol[..., 2] = FEs[..., 2]
        mdf = gpu.to_host(gpu.df_dir(vol, (1.0, 1.0, 1.0), (0., 0., 1.)))  # = -dFz/dz
        return mdf.mean(axis=2) / (2.0 * k_tip)

    # ---------------------------------------------------------------- direct Morse
    def run_scan_morse_direct(self, nxy=(50, 50), nz=60, dtip=-0.1, scan_p0=None, scan_da=None, scan_db=None, *,
                              workgroup_size=64, bAlloc=True, return_pp=True, return_device=False):
        """Grid-free Morse+Coulomb scan (AFM.py:2063-2233) -> (FEs, points_xyz[, PPs])."""
        assert self.use_morse, "run_scan_morse_direct requires use_morse=True (call AFMulator(use_morse=True))"
        assert self.atoms_arr is not None and self.cLJs_arr is not None, \
            "run_scan_morse_direct: call assign_params() first"
        nAtoms = int(len(self.atoms_arr))
        if not (1 <= nAtoms <= DIRECT_MAX_ATOMS):
            raise ValueError(f"run_scan_morse_direct: nAtoms={nAtoms} out of range [1,{DIRECT_MAX_ATOMS}]; "
                             f"limit is {DIRECT_MAX_ATOMS} (no silent grid fallback)")
        assert self.atoms_arr.shape == (nAtoms, 4) and self.atoms_arr.dtype == np.float32, \
            f"atoms_arr must be (nAtoms,4) float32, got {self.atoms_arr.shape} {self.atoms_arr.dtype}"
        assert self.cLJs_arr.shape == (nAtoms, 4) and self.cLJs_arr.dtype == np.float32, \
            f"cLJs_arr (Morse) must be (nAtoms,4) float32, got {self.cLJs_arr.shape} {self.cLJs_arr.dtype}"
        if scan_p0 is None or scan_da is None or scan_db is None:
            raise ValueError("run_scan_morse_direct: scan_p0, scan_da, scan_db are MANDATORY "
                             "(no bbox auto-derive during fitting)")
        scan_p0 = np.asarray(scan_p0, dtype=np.float32).reshape(3)
        scan_da = np.asarray(scan_da, dtype=np.float32).reshape(3)
        scan_db = np.asarray(scan_db, dtype=np.float32).reshape(3)
        assert np.isfinite(scan_p0).all() and np.isfinite(scan_da).all() and np.isfinite(scan_db).all(), \
            "run_scan_morse_direct: scan_p0/da/db must be finite"
        if not (float(dtip) < 0.0):
            raise ValueError(f"run_scan_morse_direct: dtip must be <0 for the MVP, got dtip={dtip}")
        try:
            nx_s, ny_s = (int(nxy[0]), int(nxy[1]))
        except Exception as e:
            raise ValueError(f"run_scan_morse_direct: nxy must be a 2-tuple of positive ints, got {nxy!r}") from e
        nz = int(nz)
        assert nx_s > 0 and ny_s > 0 and nz > 0, f"run_scan_morse_direct: nx,ny,nz must be positive, got {nxy} nz={nz}"
        workgroup_size = int(workgroup_size)
        assert workgroup_size > 0, f"run_scan_morse_direct: workgroup_size must be positive, got {workgroup_size}"
        n_scan = nx_s * ny_s
        pts = _raster_points(scan_p0, scan_da, scan_db, nx_s, ny_s)
        self._check_alloc(n_scan * nz * 16, "run_scan_morse_direct: FEs buffer")
        tipC = self.tipC.copy()
        tipC[3] = np.float32(dtip)
        P = self._flags_params(tipA=self.tipA, tipB=self.tipB, tipC=tipC, stiffness=self.stiffness, dpos0=self.dpos0,
                               relax_params=self.relax_pars, surfFF=self.surfFF, nz=nz, raster_ny=ny_s, fire=True,
                               polish=False)
        FEs_t, PPs_t = gpu.relax_direct_morse(self.atoms_arr, self.cLJs_arr, pts, P, self.tipQs, self.tipQZs)
        FEs = gpu.to_host(FEs_t.reshape(nx_s, ny_s, nz, 4))
        PPs = gpu.to_host(PPs_t.reshape(nx_s, ny_s, nz, 4))
        points_xyz = pts[:, :3].reshape(nx_s, ny_s, 3)
        finite_mask = np.isfinite(PPs).all(axis=-1)
        bad_mask = (~finite_mask) | (PPs[..., 3] < 0.0)
        if bad_mask.any():
            ix, iy, iz = np.unravel_index(np.argmax(bad_mask), bad_mask.shape)
            pp = PPs[ix, iy, iz]
            reason = "nonfinite" if not finite_mask[ix, iy, iz] else f"non-converged (iters={int(abs(pp[3]))})"
            raise RuntimeError(
                f"run_scan_morse_direct: PP telemetry failed at (ix={ix},iy={iy},iz={iz}): {reason}  "
                f"PP.xyz=({pp[0]:.6f},{pp[1]:.6f},{pp[2]:.6f}) PP.w={pp[3]:.1f}  "
                f"FE=({FEs[ix, iy, iz, 0]:.6f},{FEs[ix, iy, iz, 1]:.6f},{FEs[ix, iy, iz, 2]:.6f},{FEs[ix, iy, iz, 3]:.6f})")
        self._morse_direct_fwd_state = {
            "nAtoms": nAtoms, "nx": nx_s, "ny": ny_s, "nz": nz, "dtip": float(dtip),
            "scan_p0": scan_p0.copy(), "scan_da": scan_da.copy(), "scan_db": scan_db.copy(),
            "atoms_hash": hash(self.atoms_arr.tobytes()), "cLJs_hash": hash(self.cLJs_arr.tobytes()),
            "tipA": self.tipA.copy(), "tipB": self.tipB.copy(), "stiffness": self.stiffness.copy(),
            "dpos0": self.dpos0.copy(), "tipQs": self.tipQs.copy(), "tipQZs": self.tipQZs.copy(),
            "surfFF": self.surfFF.copy(),
        }
        if return_pp:
            return FEs, points_xyz, PPs
        return FEs, points_xyz

    def vjp_scan_morse_direct(self, PPs, points_xyz, dtip, dL_dFEs, *, workgroup_size=64, bAlloc=True):
        """Implicit-equilibrium VJP (AFM.py:2241-2519) -> (grad_theta (nAtoms,6) f64, diagnostics)."""
        assert self.use_morse, "vjp_scan_morse_direct requires use_morse=True"
        assert self.atoms_arr is not None and self.cLJs_arr is not None, \
            "vjp_scan_morse_direct: call assign_params() first"
        nAtoms = int(len(self.atoms_arr))
        if not (1 <= nAtoms <= DIRECT_MAX_ATOMS):
            raise ValueError(f"vjp_scan_morse_direct: nAtoms={nAtoms} out of range [1,{DIRECT_MAX_ATOMS}]")
        PPs = np.asarray(PPs)
        points_xyz = np.asarray(points_xyz)
        dL_dFEs = np.asarray(dL_dFEs)
        if PPs.ndim != 4 or PPs.shape[3] != 4:
            raise ValueError(f"vjp_scan_morse_direct: PPs must be (nx,ny,nz,4), got {PPs.shape}")
        if PPs.dtype != np.float32:
            raise ValueError(f"vjp_scan_morse_direct: PPs must be float32, got {PPs.dtype}")
        if points_xyz.ndim != 3 or points_xyz.shape[2] != 3:
            raise ValueError(f"vjp_scan_morse_direct: points_xyz must be (nx,ny,3), got {points_xyz.shape}")
        if points_xyz.dtype != np.float32:
            raise ValueError(f"vjp_scan_morse_direct: points_xyz must be float32, got {points_xyz.dtype}")
        if dL_dFEs.shape != PPs.shape:
            raise ValueError(f"vjp_scan_morse_direct: dL_dFEs shape {dL_dFEs.shape} != PPs shape {PPs.shape}")
        if dL_dFEs.dtype != np.float32:
            raise ValueError(f"vjp_scan_morse_direct: dL_dFEs must be float32, got {dL_dFEs.dtype}")
        nx, ny, nz = PPs.shape[:3]
        if points_xyz.shape[:2] != (nx, ny):
            raise ValueError(f"vjp_scan_morse_direct: points_xyz ({points_xyz.shape[:2]}) != PPs ({nx},{ny})")
        if not np.isfinite(PPs).all():
            raise ValueError("vjp_scan_morse_direct: PPs contains nonfinite values")
        if not np.isfinite(dL_dFEs).all():
            raise ValueError("vjp_scan_morse_direct: dL_dFEs contains nonfinite values")
        if (PPs[..., 3] <= 0.0).any():
            bad = np.argmax(PPs[..., 3] <= 0.0)
            ix, iy, iz = np.unravel_index(bad, (nx, ny, nz))
            raise ValueError(f"vjp_scan_morse_direct: PPs[{ix},{iy},{iz}].w={PPs[ix, iy, iz, 3]:.1f} <= 0 "
                             f"(non-converged); VJP requires all converged states")
        dtip = float(dtip)
        if dtip >= 0.0:
            raise ValueError(f"vjp_scan_morse_direct: dtip must be <0, got dtip={dtip}")
        workgroup_size = int(workgroup_size)
        assert workgroup_size > 0, f"vjp_scan_morse_direct: workgroup_size must be positive, got {workgroup_size}"
        fwd = self._morse_direct_fwd_state
        if fwd is None:
            raise RuntimeError("vjp_scan_morse_direct: no prior run_scan_morse_direct forward state recorded "
                               "(call run_scan_morse_direct first); cannot validate VJP inputs")
        mismatches = []
        if fwd["nAtoms"] != nAtoms:
            mismatches.append(f"nAtoms fwd={fwd['nAtoms']} vs vjp={nAtoms}")
        if fwd["nx"] != nx or fwd["ny"] != ny or fwd["nz"] != nz:
            mismatches.append(f"scan shape fwd=({fwd['nx']},{fwd['ny']},{fwd['nz']}) vs vjp=({nx},{ny},{nz})")
        if abs(fwd["dtip"] - dtip) > 1e-12:
            mismatches.append(f"dtip fwd={fwd['dtip']!r} vs vjp={dtip!r}")
        if (fwd["nx"], fwd["ny"]) == (nx, ny):
            fwd_pts = _raster_points(fwd["scan_p0"], fwd["scan_da"], fwd["scan_db"], nx, ny)[:, :3].reshape(nx, ny, 3)
            if not np.array_equal(fwd_pts, points_xyz):
                mismatches.append("points_xyz does not match the forward scan raster "
                                  f"(max|diff|={np.abs(fwd_pts - points_xyz).max():.6e})")
        if hash(self.atoms_arr.tobytes()) != fwd["atoms_hash"]:
            mismatches.append("atoms_arr content changed since forward (atoms_hash mismatch)")
        if hash(self.cLJs_arr.tobytes()) != fwd["cLJs_hash"]:
            mismatches.append("cLJs_arr content changed since forward (cLJs_hash mismatch)")
        for nm in ("tipA", "tipB", "stiffness", "dpos0", "tipQs", "tipQZs", "surfFF"):
            if not np.array_equal(getattr(self, nm), fwd[nm]):
                mismatches.append(f"{nm} changed since forward (fwd={fwd[nm]} vs cur={getattr(self, nm)})")
        if mismatches:
            raise RuntimeError("vjp_scan_morse_direct: stale or mismatched forward state:\n  - " +
                               "\n  - ".join(mismatches))
        tipC = self.tipC.copy()
        tipC[3] = np.float32(dtip)
        P = self._flags_params(tipA=self.tipA, tipB=self.tipB, tipC=tipC, stiffness=self.stiffness, dpos0=self.dpos0,
                               relax_params=self.relax_pars, surfFF=self.surfFF, nz=nz, fire=True, polish=False)
        pts = np.zeros((nx * ny, 4), dtype=np.float32)
        pts[:, :3] = points_xyz.reshape(-1, 3)
        lam, diag = gpu.adjoint_direct_state(self.atoms_arr, self.cLJs_arr, pts, P, self.tipQs, self.tipQZs,
                                             PPs.reshape(-1, 4), dL_dFEs.reshape(-1, 4))
        adjoint_diag = gpu.to_host(diag.reshape(nx, ny, nz, 4))
        if not np.isfinite(adjoint_diag).all():
            flat_idx = int(np.argmax(~np.isfinite(adjoint_diag).all(axis=-1)))
            ix, iy, iz = np.unravel_index(flat_idx, (nx, ny, nz))
            raise RuntimeError(f"vjp_scan_morse_direct: adjoint_diag nonfinite at (ix={ix},iy={iy},iz={iz}): "
                               f"diag={adjoint_diag[ix, iy, iz]}")
        residual_norms = adjoint_diag[..., 0].astype(np.float64)
        lambda_mins = adjoint_diag[..., 1].astype(np.float64)
        condition_estimates = adjoint_diag[..., 2].astype(np.float64)
        status_codes = adjoint_diag[..., 3].astype(np.int64)
        bad_mask = status_codes != 0
        if bad_mask.any():
            flat_idx = int(np.argmax(bad_mask))
            ix, iy, iz = np.unravel_index(flat_idx, (nx, ny, nz))
            raise RuntimeError(
                f"vjp_scan_morse_direct: adjoint failed at (ix={ix},iy={iy},iz={iz}): "
                f"status_code={int(status_codes[ix, iy, iz])} residual_norm={residual_norms[ix, iy, iz]:.6e} "
                f"lambda_min={lambda_mins[ix, iy, iz]:.6e} condition_estimate={condition_estimates[ix, iy, iz]:.6e}")
        grad = gpu.adjoint_direct_params(self.atoms_arr, self.cLJs_arr, pts, P, self.tipQs, self.tipQZs,
                                         PPs.reshape(-1, 4), dL_dFEs.reshape(-1, 4), lam)
        grad_theta = grad.cpu().numpy().astype(np.float64)
        if not np.isfinite(grad_theta).all():
            bad = int(np.argmax(~np.isfinite(grad_theta).all(axis=-1)))
            raise RuntimeError(f"vjp_scan_morse_direct: grad_theta nonfinite at atom {bad}: {grad_theta[bad]}")
        diagnostics = {"residual_norms": residual_norms, "lambda_mins": lambda_mins,
                       "condition_estimates": condition_estimates, "status_codes": status_codes}
        return grad_theta, diagnostics


# ---------------------------------------------------------------- stage (c)
def _to_np(t):
    return gpu.to_host(t)


def _volume(FEs, ncopy=3):
    """(nx,ny,nz,4) float32/float64 volume holding the first ncopy channels of FEs
    (FEs itself when it already is one: the kernels read channels 0-2 only)."""
    dt = np.float64 if FEs.dtype == np.float64 else np.float32
    if FEs.dtype == dt and FEs.shape[-1] == 4 and FEs.flags.c_contiguous:
        return FEs
    vol = np.zeros(FEs.shape[:3] + (4,), dtype=dt)
    vol[..., :ncopy] = FEs[..., :ncopy]
    return vol


def _zvolume(Fz):
    dt = np.float64 if Fz.dtype == np.float64 else np.float32
    vol = np.zeros(Fz.shape + (4,), dtype=dt)
    vol[..., 2] = Fz
    return vol


def compute_df(Fz, dz):
    """df = -dFz/dz (AFM.py:3048-3050); Fz (nx,ny,nz)."""
    Fz = np.asarray(Fz)
    vol = _zvolume(Fz)
    out = _to_np(gpu.df_dir(vol, (1.0, 1.0, abs(float(dz))), (0., 0., 1.)))
    return out.astype(np.float32) if Fz.dtype == np.float32 else out


def compute_df_amp(Fz, dz, amp=1.0):
    """Finite-amplitude df along z (AFM.py:3052-3089) -> float32 (nx,ny,nz)."""
    Fz = np.asarray(Fz)
    vol = _zvolume(Fz)
    return _to_np(gpu.df_amp_dir(vol, (1.0, 1.0, abs(float(dz))), (0., 0., 1.), amp))


def compute_df_dir(FEs, spacing, osc_dir=(0., 0., 1.)):
    """df = -n.grad(F.n) on an xyz volume (AFM.py:3105-3123) -> float64."""
    FEs = np.asarray(FEs)
    if FEs.ndim != 4 or FEs.shape[-1] < 3:
        raise ValueError(f"FEs must have shape (nx,ny,nz,>=3), got {FEs.shape}")
    return _to_np(gpu.df_dir(_volume(FEs), spacing, osc_dir))


def compute_df_amp_dir(FEs, spacing, osc_dir=(0., 0., 1.), amp=1.0):
    """Finite-amplitude df for any oscillation direction (AFM.py:3203-3236) -> float32."""
    FEs = np.asarray(FEs)
    if FEs.ndim != 4 or FEs.shape[-1] < 3:
        raise ValueError(f"FEs must have shape (nx,ny,nz,>=3), got {FEs.shape}")
    return _to_np(gpu.df_amp_dir(_volume(FEs), spacing, osc_dir, amp))


def df_loss_seed(FEs, target_df, dtip, weights=None):
    """Central-difference df loss and its exact adjoint (AFM.py:3125-3200).

    Returns (loss float, df (nx,ny,nz) f64, dL_dFEs (nx,ny,nz,4) f64)."""
    FEs = np.asarray(FEs)
    target_df = np.asarray(target_df, dtype=np.float64)
    if FEs.ndim != 4 or FEs.shape[3] < 3:
        raise ValueError(f"df_loss_seed: FEs must be (nx,ny,nz,>=4), got {FEs.shape}")
    nx, ny, nz = FEs.shape[:3]
    if target_df.shape != (nx, ny, nz):
        raise ValueError(f"df_loss_seed: target_df must be ({nx},{ny},{nz}), got {target_df.shape}")
    dtip = float(dtip)
    if dtip >= 0.0:
        raise ValueError(f"df_loss_seed: dtip must be <0, got dtip={dtip}")
    if nz < 3:
        raise ValueError(f"df_loss_seed: need nz>=3 for central difference, got nz={nz}")
    w = None
    if weights is not None:
        w = np.asarray(weights, dtype=np.float64)
        if w.shape != (nx, ny, nz):
            raise ValueError(f"df_loss_seed: weights must be ({nx},{ny},{nz}), got {w.shape}")
        if float(w.sum()) <= 0.0:
            raise ValueError("df_loss_seed: sum(weights) must be > 0")
    loss, df, dL = gpu.df_loss_seed(_zvolume(np.asarray(FEs[..., 2])), target_df, dtip, w)
    dL_dFEs = np.zeros((nx, ny, nz, 4), dtype=np.float64)
    dL_dFEs[..., 2] = _to_np(dL[..., 2]).astype(np.float64)
    return float(_to_np(loss)[0]), _to_np(df), dL_dFEs


def compute_dissipation(FEs_fwd, FEs_bwd, h_scan, h_df, amp, osc_dir=(0., 0., 1.)):
    """E_diss = |int (F_fwd - F_bwd).n dz| per cycle (AFM.py:3238-3277) -> float32 (nx,ny,nz_df)."""
    Ff = np.asarray(FEs_fwd)
    Fb = np.asarray(FEs_bwd)
    return _to_np(gpu.dissipation(_volume(Ff), _volume(Fb), h_scan, h_df, amp, osc_dir))


def df_to_hz(df, f0=30300.0, k0=1800.0):
    """Stiffness-proxy df [eV/A^2] -> frequency shift [Hz]: -(f0/(2 k0)) * 16.0218 * df."""
    return -(float(f0) / (2.0 * float(k0))) * N_M_PER_EV_A2 * np.asarray(df)
