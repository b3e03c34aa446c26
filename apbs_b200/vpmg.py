"""Host-side mirror of the reference Vpmg interface over the CUDA C ABI.

``Vpmg`` follows the call sequence of APBS's C API for one mg-manual
calculation (src/mg/vpmg.h):

    pmg = Vpmg(params)            # Vpmg_ctor    (vpmg.h:226)
    pmg.fillco(molecule)          # Vpmg_fillco  (vpmg.h:281)
    pmg.solve()                   # Vpmg_solve   (vpmg.h:306)
    e = pmg.energy()              # Vpmg_energy  (vpmg.h:334), kT
    u = pmg.u                     # thee->u after the solve

Every call goes to ``libapbs_b200.so`` (include/apbs_b200.h).  There is no
CPU implementation behind this module: if the library or a CUDA device is
missing, construction raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .synth import PmgbParams

FP64 = 0
MIXED = 1

K_GS7_FP64, K_GS27_WAVE, K_RESID_FP64, K_GS7_FP32, K_CG_COARSE = 0, 1, 2, 3, 4
K_VCYCLE_TAIL = 7
K_GS7_SWEEP_FP64, K_GS7_SWEEP_FP32 = 8, 9
DX_POT, DX_CHARGE, DX_KAPPA, DX_DIELX, DX_DIELY, DX_DIELZ = range(6)
MAP_DIELX, MAP_DIELY, MAP_DIELZ, MAP_KAPPA, MAP_CHARGE, MAP_POT = range(6)
TUNE_MIXED_CHEBYSHEV = 0
TUNE_GS27_LAG = 1
TUNE_GS27_CLUSTER = 2
TUNE_BAND_ALWAYS = 4
TUNE_GS7_COLOUR_PASSES = 5
TUNE_GS7_SWEEP_KCHUNK, TUNE_GS27_CLUSTER_MID, TUNE_TAIL_MAX_POINTS = 6, 7, 8
TUNE_MC_COOPERATIVE = 9
TUNE_MIXED_COARSE_SWEEPS, TUNE_MIXED_FINE_SWEEPS = 10, 11
TUNE_GS7_SWEEP_SHAPE = 12
TUNE_GS27_PLANES = 13
TUNE_CG_CLUSTER = 14
TUNE_GS27_PLANES_POLL = 15
TUNE_NKEYS = 16
NOALLOC_MAX_DIM = 1025   # PMGB_NOALLOC_MAX_DIM

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libapbs_b200.so")
_lib = None


class PmgbStats(ctypes.Structure):
    """Mirror of ``pmgb_stats`` in include/apbs_b200.h."""

    _fields_ = [
        ("vcycles", ctypes.c_int), ("newton_iters", ctypes.c_int),
        ("refinements", ctypes.c_int), ("coarse_method", ctypes.c_int),
        ("rel_residual", ctypes.c_double),
        ("t_fill_ms", ctypes.c_double), ("t_setup_ms", ctypes.c_double),
        ("t_solve_ms", ctypes.c_double), ("t_energy_ms", ctypes.c_double),
        ("energy_kT", ctypes.c_double), ("qf", ctypes.c_double),
        ("diel", ctypes.c_double), ("qm", ctypes.c_double),
        ("sas_points", ctypes.c_int), ("status", ctypes.c_int),
        ("ext_qf", ctypes.c_double), ("ext_diel", ctypes.c_double),
        ("ext_qm", ctypes.c_double), ("converged", ctypes.c_int),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class PmgbError(RuntimeError):
    pass


def lib():
    """Load the CUDA library; raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PmgbError("libapbs_b200.so is not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        vp = ctypes.c_void_p
        L.pmgb_create.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp)]
        L.pmgb_fillco.argtypes = [vp, ctypes.c_int, dp, dp, dp]
        L.pmgb_set_stream.argtypes = [vp, vp]
        L.pmgb_fillco_device.argtypes = [vp, ctypes.c_int, vp, vp, vp]
        L.pmgb_set_coefficients.argtypes = [vp, dp, dp, dp, dp, dp, dp, dp, dp]
        L.pmgb_focus.argtypes = [vp, vp, ctypes.c_int]
        L.pmgb_solve.argtypes = [vp]
        L.pmgb_energy.argtypes = [vp, dp]
        L.pmgb_forces.argtypes = [vp, dp, dp, dp]
        L.pmgb_debug_shift_wave_counter.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.pmgb_write_dx.argtypes = [vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p,
                                    ctypes.c_char_p]
        L.pmgb_set_map.argtypes = [vp, ctypes.c_int] + [ctypes.c_int] * 3 + \
            [ctypes.c_double] * 6 + [dp]
        L.pmgb_read_dx_host.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), dp, dp,
                                        dp]
        L.pmgb_write_dx_host.argtypes = [ctypes.c_char_p] + [ctypes.c_int] * 3 + \
            [ctypes.c_double] * 6 + [dp, dp, ctypes.c_char_p, ctypes.c_char_p]
        L.pmgb_get_potential.argtypes = [vp, dp]
        L.pmgb_get_maps.argtypes = [vp, dp, dp]
        L.pmgb_get_stats.argtypes = [vp, ctypes.POINTER(PmgbStats)]
        L.pmgb_get_residual_history.argtypes = [vp, dp, ctypes.c_int]
        L.pmgb_destroy.argtypes = [vp]
        L.pmgb_destroy.restype = None
        L.pmgb_solve_molecule.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp,
                                          ctypes.POINTER(PmgbStats)]
        L.pmgb_time_kernel.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, dp]
        L.pmgb_time_kernel.restype = ctypes.c_int
        L.pmgb_batch_solve.argtypes = [ctypes.POINTER(vp), ctypes.c_int, vp]
        L.pmgb_batch_solve.restype = ctypes.c_int
        L.pmgb_solver_set_tuning.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.pmgb_solver_set_tuning.restype = ctypes.c_int
        L.pmgb_solver_get_tuning.argtypes = [vp, ctypes.c_int]
        L.pmgb_solver_get_tuning.restype = ctypes.c_int
        L.pmgb_set_tuning.argtypes = [ctypes.c_int, ctypes.c_int]
        L.pmgb_set_tuning.restype = ctypes.c_int
        L.pmgb_get_tuning.argtypes = [ctypes.c_int]
        L.pmgb_get_tuning.restype = ctypes.c_int
        L.pmgb_energy_noalloc.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, dp]
        L.pmgb_energy_noalloc.restype = ctypes.c_int
        L.pmgb_last_error.restype = ctypes.c_char_p
        L.pmgb_launch_count.argtypes = [ctypes.c_int]
        L.pmgb_launch_count.restype = ctypes.c_longlong
        for name in ("pmgb_create", "pmgb_fillco", "pmgb_fillco_device", "pmgb_set_coefficients",
                     "pmgb_solve", "pmgb_energy", "pmgb_get_potential", "pmgb_get_maps",
                     "pmgb_get_stats", "pmgb_get_residual_history", "pmgb_solve_molecule",
                     "pmgb_set_stream"):
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def set_tuning(key: int, value: int) -> None:
    _check(lib().pmgb_set_tuning(key, value), "pmgb_set_tuning")


def get_tuning(key: int) -> int:
    return int(lib().pmgb_get_tuning(key))


def last_error() -> str:
    return lib().pmgb_last_error().decode(errors="replace")


def _dp(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(rc, what):
    if rc != 1:
        raise PmgbError("%s failed: %s" % (what, last_error()))


def _atoms(mol):
    xyz = np.ascontiguousarray(mol.xyz, dtype=np.float64).reshape(-1)
    q = np.ascontiguousarray(mol.charge, dtype=np.float64)
    r = np.ascontiguousarray(mol.radius, dtype=np.float64)
    return xyz, q, r


class Vpmg:
    """One PMG calculation held on the current CUDA device."""

    def __init__(self, params: PmgbParams, precision: int = FP64):
        self.params = params
        self.precision = precision
        self._h = ctypes.c_void_p()
        _check(lib().pmgb_create(ctypes.byref(params), precision, ctypes.byref(self._h)),
               "pmgb_create")

    @property
    def shape(self):
        p = self.params
        return (p.nz, p.ny, p.nx)

    def set_stream(self, stream_handle: int):
        """Issue all device work on this cudaStream_t (e.g. torch stream.cuda_stream)."""
        _check(lib().pmgb_set_stream(self._h, ctypes.c_void_p(stream_handle)), "pmgb_set_stream")

    def fillco_device(self, natoms, d_xyz, d_q, d_r):
        """Fill from atom arrays already in device memory (raw pointers)."""
        self._natoms = int(natoms)
        _check(lib().pmgb_fillco_device(self._h, natoms, ctypes.c_void_p(d_xyz),
                                        ctypes.c_void_p(d_q), ctypes.c_void_p(d_r)),
               "pmgb_fillco_device")

    def fillco(self, mol):
        xyz, q, r = _atoms(mol)
        self._keep = (xyz, q, r)
        self._natoms = int(mol.natoms)
        _check(lib().pmgb_fillco(self._h, mol.natoms, _dp(xyz), _dp(q), _dp(r)), "pmgb_fillco")

    def focus(self, coarse: "Vpmg", calc_energy: bool = True):
        """Boundary values (and, with calc_energy, the external energy) from
        a solved coarse calculation: Vpmg_ctor with focusFlag = 1.  Call
        before fillco; this calculation must use bcfl focus."""
        _check(lib().pmgb_focus(self._h, coarse._h, 1 if calc_energy else 0), "pmgb_focus")

    def set_coefficients(self, charge, epsx, epsy, epsz, kappa, faces):
        p = self.params
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
                for a in (charge, epsx, epsy, epsz, kappa)]
        faces = np.ascontiguousarray(faces, dtype=np.float64)
        fx, fy = 2 * p.ny * p.nz, 2 * p.nx * p.nz
        gx, gy, gz = faces[:fx], faces[fx:fx + fy], faces[fx + fy:]
        self._keep = (arrs, gx, gy, gz)
        _check(lib().pmgb_set_coefficients(self._h, *[_dp(a) for a in arrs], _dp(gx), _dp(gy),
                                           _dp(gz)), "pmgb_set_coefficients")

    def solve(self):
        _check(lib().pmgb_solve(self._h), "pmgb_solve")
        return 1

    def energy(self) -> float:
        e = np.zeros(1)
        _check(lib().pmgb_energy(self._h, _dp(e)), "pmgb_energy")
        return float(e[0])

    def set_map(self, which: int, data, h, origin):
        """Use a map (MAP_DIELX..MAP_CHARGE) given on its own grid, as the
        deck's "usemap": data (nz, ny, nx), spacing h, origin; data None
        stops using it.  Takes effect at the next fillco."""
        if data is None:
            _check(lib().pmgb_set_map(self._h, which, 0, 0, 0, 0, 0, 0, 0, 0, 0, None),
                   "pmgb_set_map")
            return
        d = np.ascontiguousarray(data, dtype=np.float64)
        nz, ny, nx = d.shape
        _check(lib().pmgb_set_map(self._h, which, nx, ny, nz, *[float(v) for v in h],
                                  *[float(v) for v in origin], _dp(d.reshape(-1))),
               "pmgb_set_map")

    def write_dx(self, path, which: int = 0, title: str | None = None,
                 package: str | None = None):
        """Write one map (DX_POT, DX_CHARGE, DX_KAPPA, DX_DIELX/Y/Z) as the
        OpenDX file writedataMG writes."""
        _check(lib().pmgb_write_dx(self._h, which, str(path).encode(),
                                   title.encode() if title else None,
                                   package.encode() if package else None), "pmgb_write_dx")

    def forces(self, boundary: bool = True) -> dict:
        """Per-atom forces of the last solve in kT/A, as Vpmg_force builds
        them per atom: ``qf`` (charge field) and, with ``boundary`` (needs
        srfm spl2), ``db`` (dielectric boundary) and ``ib`` (ionic
        boundary); each an (natoms, 3) array."""
        n = getattr(self, "_natoms", 0)
        qf = np.zeros((n, 3))
        db = np.zeros((n, 3)) if boundary else None
        ib = np.zeros((n, 3)) if boundary else None
        _check(lib().pmgb_forces(self._h, _dp(qf), _dp(db) if boundary else None,
                                 _dp(ib) if boundary else None), "pmgb_forces")
        out = {"qf": qf}
        if boundary:
            out.update(db=db, ib=ib)
        return out

    @property
    def u(self) -> np.ndarray:
        out = np.empty(self.shape)
        _check(lib().pmgb_get_potential(self._h, _dp(out)), "pmgb_get_potential")
        return out

    def potential_into(self, out: np.ndarray) -> np.ndarray:
        """Copy the potential into a caller's float64 array of nx*ny*nz
        values (pinned host memory makes the copy a direct DMA)."""
        if out.dtype != np.float64 or out.size != int(np.prod(self.shape)) or \
                not out.flags.c_contiguous:
            raise ValueError("potential_into: need a contiguous float64 array of nx*ny*nz")
        _check(lib().pmgb_get_potential(self._h, _dp(out)), "pmgb_get_potential")
        return out

    def maps(self):
        p = self.params
        n = p.nx * p.ny * p.nz
        m = np.empty(5 * n)
        f = np.empty(2 * (p.ny * p.nz + p.nx * p.nz + p.nx * p.ny))
        _check(lib().pmgb_get_maps(self._h, _dp(m), _dp(f)), "pmgb_get_maps")
        m = m.reshape(5, *self.shape)
        return dict(charge=m[0], epsx=m[1], epsy=m[2], epsz=m[3], kappa=m[4], faces=f)

    def stats(self) -> dict:
        st = PmgbStats()
        lib().pmgb_get_stats(self._h, ctypes.byref(st))
        return st.as_dict()

    def residual_history(self) -> np.ndarray:
        buf = np.zeros(8192)
        n = lib().pmgb_get_residual_history(self._h, _dp(buf), buf.size)
        return buf[:min(n, buf.size)].copy()

    def set_tuning(self, key: int, value: int):
        """Launch-shape tunable of this calculation only (PMGB_TUNE_*)."""
        _check(lib().pmgb_solver_set_tuning(self._h, key, value), "pmgb_solver_set_tuning")

    def get_tuning(self, key: int) -> int:
        return int(lib().pmgb_solver_get_tuning(self._h, key))

    def time_kernel(self, which: int, reps: int = 20):
        """Mean device ms per launch and algorithmic bytes per launch."""
        ms, b = np.zeros(1), np.zeros(1)
        _check(lib().pmgb_time_kernel(self._h, which, reps, _dp(ms), _dp(b)), "pmgb_time_kernel")
        return float(ms[0]), float(b[0])

    def close(self):
        if self._h:
            lib().pmgb_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def energy_noalloc(params, d_u, d_charge, d_epsx=0, d_epsy=0, d_epsz=0, d_kappa=0,
                   stream=0) -> float:
    """Energy (kT) from device arrays the caller owns, with no device
    allocation (pmgb_energy_noalloc).  Pointers are raw device addresses
    (e.g. torch tensor.data_ptr()); stream is a cudaStream_t handle or 0."""
    e = np.zeros(1)
    _check(lib().pmgb_energy_noalloc(ctypes.byref(params), ctypes.c_void_p(d_u),
                                     ctypes.c_void_p(d_charge), ctypes.c_void_p(d_epsx or None),
                                     ctypes.c_void_p(d_epsy or None), ctypes.c_void_p(d_epsz or None),
                                     ctypes.c_void_p(d_kappa or None), ctypes.c_void_p(stream or None),
                                     _dp(e)), "pmgb_energy_noalloc")
    return float(e[0])


def batch_solve(calcs, stream_handle: int = 0) -> None:
    """Solve filled mixed-precision LPBE calculations in one persistent
    kernel launch (pmgb_batch_solve); each is then solved as by Vpmg.solve."""
    arr = (ctypes.c_void_p * len(calcs))(*[c._h.value for c in calcs])
    _check(lib().pmgb_batch_solve(arr, len(calcs), ctypes.c_void_p(stream_handle or None)),
           "pmgb_batch_solve")


def solve_molecule(params, mol, precision=FP64, want_u=False):
    """One host-buffer call: fill + solve + energy (pmgb_solve_molecule)."""
    xyz, q, r = _atoms(mol)
    e = np.zeros(1)
    u = np.empty((params.nz, params.ny, params.nx)) if want_u else None
    st = PmgbStats()
    _check(lib().pmgb_solve_molecule(ctypes.byref(params), precision, mol.natoms, _dp(xyz),
                                     _dp(q), _dp(r), _dp(e), _dp(u), ctypes.byref(st)),
           "pmgb_solve_molecule")
    return float(e[0]), u, st.as_dict()


def read_dx(path):
    """OpenDX file -> (data (nz, ny, nx), h (3,), origin (3,)), as
    Vgrid_readDX reads it."""
    dims = (ctypes.c_int * 3)()
    h, origin = np.zeros(3), np.zeros(3)
    _check(lib().pmgb_read_dx_host(str(path).encode(), dims, _dp(h), _dp(origin), None),
           "pmgb_read_dx_host")
    data = np.zeros((dims[2], dims[1], dims[0]))
    _check(lib().pmgb_read_dx_host(str(path).encode(), dims, _dp(h), _dp(origin), _dp(data)),
           "pmgb_read_dx_host")
    return data, h, origin


def write_dx(path, data, h, origin, title="", package=None, pvec=None):
    """(nz, ny, nx) array -> OpenDX file, byte for byte as Vgrid_writeDX."""
    d = np.ascontiguousarray(data, dtype=np.float64)
    nz, ny, nx = d.shape
    pv = None if pvec is None else np.ascontiguousarray(pvec, dtype=np.float64)
    _check(lib().pmgb_write_dx_host(str(path).encode(), nx, ny, nz, *[float(v) for v in h],
                                    *[float(v) for v in origin], _dp(d.reshape(-1)), _dp(pv),
                                    title.encode(), package.encode() if package else None),
           "pmgb_write_dx_host")
