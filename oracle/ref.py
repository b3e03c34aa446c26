"""ctypes binding of oracle/_ref/libapbsref.so: the reference APBS PMG path
compiled unchanged (see oracle/Makefile).  TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libapbsref.so")
# the same reference objects and driver with Vpmg_solve replaced by the
# drop-in binding apbs_b200/dropin/vpmg_b200.c (solve on the GPU)
DROPIN_PATH = os.path.join(_HERE, "_ref", "libapbsref_b200.so")
_libs = {}


def available() -> bool:
    return os.path.exists(LIB_PATH)


def dropin_available() -> bool:
    return os.path.exists(DROPIN_PATH)


def lib(dropin=False):
    path = DROPIN_PATH if dropin else LIB_PATH
    if path not in _libs:
        _lib = ctypes.CDLL(path)
        _libs[path] = _lib
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.ref_pmg_run.restype = ctypes.c_int
        _lib.ref_pmg_run.argtypes = [ctypes.c_void_p, ctypes.c_int, dp, dp, dp,
                                     dp, dp, dp, dp, dp, ctypes.c_int, ctypes.c_int,
                                     dp, ctypes.POINTER(ctypes.c_int)]
        _lib.ref_pmg_run_maps.restype = ctypes.c_int
        _lib.ref_pmg_run_maps.argtypes = [ctypes.c_void_p, ctypes.c_int, dp, dp, dp,
                                          ctypes.POINTER(ctypes.c_int), dp,
                                          ctypes.POINTER(dp), dp, dp, dp]
        _lib.ref_write_dx.restype = ctypes.c_int
        _lib.ref_write_dx.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 6 + [
            dp, dp, ctypes.c_char_p, ctypes.c_char_p]
        _lib.ref_pmg_focus.restype = ctypes.c_int
        _lib.ref_pmg_focus.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, dp, dp, dp,
                                     dp, dp, dp, dp, ctypes.c_int, ctypes.c_int]
        _lib.ref_pmg_chain.restype = ctypes.c_int
        _lib.ref_pmg_chain.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp, dp, dp,
                                       dp, dp]
    return _libs[path]


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def run(params, mol, want_maps=False, want_faces=False, verbose=0, reslog_cap=4096,
        want_forces=False, dropin=False):
    """Run ctor+fillco+solve+energy of the reference on one calculation
    (with dropin=True, the same sequence with Vpmg_solve on the GPU).

    Returns a dict with u (nz,ny,nx), energy_kT, progress-message count,
    residual log, phase timings and, on request, the fill maps and faces and
    the per-atom forces (qf, db, ib: (natoms, 3) each, and their status).
    """
    n = params.nx * params.ny * params.nz
    u = np.zeros(n)
    maps = np.zeros(5 * n) if want_maps else None
    nfaces = 2 * (params.ny * params.nz + params.nx * params.nz + params.nx * params.ny)
    faces = np.zeros(nfaces) if want_faces else None
    out = np.zeros(16)
    reslog = np.zeros(reslog_cap)
    xyz = np.ascontiguousarray(mol.xyz, dtype=np.float64).reshape(-1)
    q = np.ascontiguousarray(mol.charge, dtype=np.float64)
    r = np.ascontiguousarray(mol.radius, dtype=np.float64)
    forces = np.zeros(9 * mol.natoms) if want_forces else None
    fstatus = np.zeros(mol.natoms, dtype=np.int32) if want_forces else None
    rc = lib(dropin).ref_pmg_run(ctypes.byref(params), mol.natoms, _ptr(xyz), _ptr(q), _ptr(r),
                           _ptr(u), _ptr(maps), _ptr(faces), _ptr(out), _ptr(reslog),
                           reslog_cap, verbose, _ptr(forces),
                           fstatus.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
                           if fstatus is not None else None)
    if rc != 1:
        raise RuntimeError("reference PMG run failed")
    shape = (params.nz, params.ny, params.nx)
    res = {
        "u": u.reshape(shape),
        "energy_kT": out[0],
        "progress_msgs": int(out[1]),
        "reslog": reslog[: min(int(out[2]), reslog_cap)].copy(),
        "t_ctor": out[3], "t_fillco": out[4], "t_solve": out[5], "t_energy": out[6],
        "qf": out[7], "diel": out[8], "qm": out[9],
    }
    if maps is not None:
        m = maps.reshape(5, *shape)
        res.update(charge=m[0], epsx=m[1], epsy=m[2], epsz=m[3], kappa=m[4])
    if faces is not None:
        res["faces"] = faces
    if forces is not None:
        f = forces.reshape(mol.natoms, 3, 3)
        res.update(qf=f[:, 0].copy(), db=f[:, 1].copy(), ib=f[:, 2].copy(), fstatus=fstatus)
    return res


def focus(coarse, fine, mol, want_faces=False, reslog_cap=8192, dropin=False):
    """Two-block focusing chain (coarse solve, then the bcfl-focus block whose
    faces and external energy come from it), computed by the reference.

    Returns the fine block's u, energy (with the external terms), faces on
    request, the external energies and the coarse energy."""
    xyz = np.ascontiguousarray(mol.xyz, dtype=np.float64).reshape(-1)
    q = np.ascontiguousarray(mol.charge, dtype=np.float64)
    r = np.ascontiguousarray(mol.radius, dtype=np.float64)
    n = fine.nx * fine.ny * fine.nz
    u = np.zeros(n)
    nfaces = 2 * (fine.ny * fine.nz + fine.nx * fine.nz + fine.nx * fine.ny)
    faces = np.zeros(nfaces) if want_faces else None
    out = np.zeros(16)
    reslog = np.zeros(reslog_cap)
    rc = lib(dropin).ref_pmg_focus(ctypes.byref(coarse), ctypes.byref(fine), mol.natoms, _ptr(xyz), _ptr(q),
                  _ptr(r), _ptr(u), _ptr(faces), _ptr(out), _ptr(reslog), reslog_cap, 0)
    if rc != 1:
        raise RuntimeError("reference focusing run failed")
    res = {
        "u": u.reshape(fine.nz, fine.ny, fine.nx), "energy_kT": out[0],
        "progress_msgs": int(out[1]), "reslog": reslog[: min(int(out[2]), reslog_cap)].copy(),
        "t_ctor": out[3], "t_fillco": out[4], "t_solve": out[5], "t_energy": out[6],
        "qf": out[7], "diel": out[8], "qm": out[9],
        "ext_qf": out[12], "ext_diel": out[13], "ext_qm": out[14], "coarse_energy_kT": out[15],
    }
    if faces is not None:
        res["faces"] = faces
    return res


def write_dx(path, data, h, origin, pvec=None, title="POTENTIAL (kT/e)"):
    """The reference's Vgrid_writeDX on data (nz, ny, nx): the OpenDX file
    writedataMG writes.  PACKAGE_STRING of this build is
    "APBS 3.4.1 (reference oracle build)"."""
    d = np.ascontiguousarray(data, dtype=np.float64)
    nz, ny, nx = d.shape
    pv = None if pvec is None else np.ascontiguousarray(pvec, dtype=np.float64)
    rc = lib().ref_write_dx(nx, ny, nz, h[0], h[1], h[2], origin[0], origin[1], origin[2],
                            _ptr(d.reshape(-1)), _ptr(None if pv is None else pv.reshape(-1)),
                            str(path).encode(), title.encode())
    if rc != 1:
        raise RuntimeError("reference DX write failed")


def run_maps(params, mol, maps):
    """The reference with "usemap" maps: maps is {index 0..5 (dielx, diely,
    dielz, kappa, charge, pot): (data (nz, ny, nx), h (3,), origin (3,))}.
    Returns u, energy_kT and the fill maps as run() does."""
    n = params.nx * params.ny * params.nz
    u = np.zeros(n)
    fill = np.zeros(5 * n)
    out = np.zeros(16)
    dims = (ctypes.c_int * 18)()
    geom = np.zeros(36)
    ptrs = (ctypes.POINTER(ctypes.c_double) * 6)()
    keep = []
    for m in range(6):
        if m in maps:
            data, h, origin = maps[m]
            d = np.ascontiguousarray(data, dtype=np.float64)
            keep.append(d)
            dims[3 * m], dims[3 * m + 1], dims[3 * m + 2] = d.shape[2], d.shape[1], d.shape[0]
            geom[6 * m:6 * m + 3] = h
            geom[6 * m + 3:6 * m + 6] = origin
            ptrs[m] = _ptr(d.reshape(-1))
    xyz = np.ascontiguousarray(mol.xyz, dtype=np.float64).reshape(-1)
    q = np.ascontiguousarray(mol.charge, dtype=np.float64)
    r = np.ascontiguousarray(mol.radius, dtype=np.float64)
    rc = lib().ref_pmg_run_maps(ctypes.byref(params), mol.natoms, _ptr(xyz), _ptr(q), _ptr(r),
                                dims, _ptr(geom), ptrs, _ptr(u), _ptr(fill), _ptr(out))
    if rc != 1:
        raise RuntimeError("reference PMG run with maps failed")
    shape = (params.nz, params.ny, params.nx)
    f = fill.reshape(5, *shape)
    return {"u": u.reshape(shape), "energy_kT": out[0], "charge": f[0], "epsx": f[1],
            "epsy": f[2], "epsz": f[3], "kappa": f[4]}


def chain(levels, mol, dropin=False):
    """An mg-auto focusing chain (a list of pmgb_params, coarse first, the
    later ones bcfl focus) run by the reference as main.c runs it.  Returns
    the total energy (kT) of every level and the finest potential."""
    from apbs_b200.synth import PmgbParams
    arr = (PmgbParams * len(levels))(*levels)
    xyz = np.ascontiguousarray(mol.xyz, dtype=np.float64).reshape(-1)
    q = np.ascontiguousarray(mol.charge, dtype=np.float64)
    r = np.ascontiguousarray(mol.radius, dtype=np.float64)
    e = np.zeros(len(levels))
    f = levels[-1]
    u = np.zeros(f.nx * f.ny * f.nz)
    rc = lib(dropin).ref_pmg_chain(ctypes.byref(arr), len(levels), mol.natoms, _ptr(xyz), _ptr(q),
                                   _ptr(r), _ptr(e), _ptr(u))
    if rc != 1:
        raise RuntimeError("reference focusing chain failed")
    return {"energies_kT": e, "u": u.reshape(f.nz, f.ny, f.nx)}
