"""Seeded synthetic molecules and mg-manual calculation descriptions.

The benchmark configurations describe globular clusters of atoms (no public
dataset is involved).  A cluster of ``natoms`` atoms is drawn from a seed:
positions uniform in a ball of radius ``radius`` with a minimum pairwise
separation (random sequential rejection), charges from
{-1, -0.5, 0, +0.5, +1} with weights {.1, .2, .4, .2, .1} shifted so the net
charge equals ``net_charge``, radii uniform in [1.2, 2.0] Angstrom.

``mg_manual`` builds the plain-C parameter block (``pmgb_params``) that both
the CUDA library and the CPU oracle consume, with the grid centred on the
molecule the way ``gcent mol 1`` does (midpoint of the atom-coordinate
bounding box, Valist_getStatistics in src/generic/valist.c).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

PMGB_MAXION = 8
SRFM_MOL, SRFM_SMOL, SRFM_SPL2, SRFM_SPL3, SRFM_SPL4 = 0, 1, 2, 3, 4
CHGM_TRIL, CHGM_SPL2, CHGM_SPL4 = 0, 1, 2
BCFL_ZERO, BCFL_SDH, BCFL_MDH, BCFL_FOCUS, BCFL_MAP = 0, 1, 2, 4, 6


class PmgbParams(ctypes.Structure):
    """Mirror of ``pmgb_params`` in include/pmgb_params.h."""

    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("nlev", ctypes.c_int),
        ("hx", ctypes.c_double), ("hy", ctypes.c_double), ("hz", ctypes.c_double),
        ("center", ctypes.c_double * 3),
        ("nonlin", ctypes.c_int), ("srfm", ctypes.c_int),
        ("chgm", ctypes.c_int), ("bcfl", ctypes.c_int),
        ("pdie", ctypes.c_double), ("sdie", ctypes.c_double),
        ("srad", ctypes.c_double), ("sdens", ctypes.c_double),
        ("temp", ctypes.c_double), ("etol", ctypes.c_double),
        ("nion", ctypes.c_int),
        ("ion_q", ctypes.c_double * PMGB_MAXION),
        ("ion_conc", ctypes.c_double * PMGB_MAXION),
        ("ion_radius", ctypes.c_double * PMGB_MAXION),
        ("swin", ctypes.c_double),
        ("itmax", ctypes.c_int),
    ]


@dataclass
class Molecule:
    xyz: np.ndarray      # (n, 3) float64, Angstrom
    charge: np.ndarray   # (n,) float64, e
    radius: np.ndarray   # (n,) float64, Angstrom

    @property
    def natoms(self) -> int:
        return int(self.xyz.shape[0])

    def center(self) -> np.ndarray:
        """Bounding-box midpoint of the atom coordinates (gcent mol)."""
        return 0.5 * (self.xyz.max(axis=0) + self.xyz.min(axis=0))


def cluster(natoms: int, radius: float, seed: int, net_charge: float = 0.0,
            min_sep: float = 1.5, center=(0.0, 0.0, 0.0)) -> Molecule:
    """Globular cluster by random sequential rejection inside a ball."""
    rng = np.random.default_rng(seed)
    cell = min_sep
    ncell = int(np.ceil(2 * radius / cell)) + 3
    grid: dict = {}
    pts = np.empty((natoms, 3))
    count = 0
    tries = 0
    sep2 = min_sep * min_sep
    while count < natoms:
        batch = rng.uniform(-radius, radius, size=(4096, 3))
        batch = batch[np.einsum("ij,ij->i", batch, batch) <= radius * radius]
        for p in batch:
            tries += 1
            c = tuple(((p + radius) / cell).astype(int) + 1)
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        lst = grid.get((c[0] + dx, c[1] + dy, c[2] + dz))
                        if lst:
                            for q in lst:
                                d = p - pts[q]
                                if d @ d < sep2:
                                    ok = False
                                    break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                pts[count] = p
                grid.setdefault(c, []).append(count)
                count += 1
                if count == natoms:
                    break
        if tries > 2000 * natoms + 100000:
            raise RuntimeError("cluster: packing too dense for min_sep")
    vals = np.array([-1.0, -0.5, 0.0, 0.5, 1.0])
    q = rng.choice(vals, size=natoms, p=[0.1, 0.2, 0.4, 0.2, 0.1])
    q = q + (net_charge - q.sum()) / natoms
    r = rng.uniform(1.2, 2.0, size=natoms)
    return Molecule(pts + np.asarray(center, dtype=float), q, r)


def mgparm_nlev(n: int) -> int:
    """Level count chosen by MGparm_check (src/generic/mgparm.c:263-330)."""
    ti = n - 1
    nlev = 0
    while ti % 2 == 0 and ti > 0:
        nlev += 1
        ti = int(np.ceil(0.5 * ti))
    nlev -= 1
    if n > 65 and nlev < 4:
        raise ValueError("dime %d needs rounding to c*2^5+1 as MGparm_check does" % n)
    return nlev


def mg_manual(dime, grid, center, *, npbe=False, srfm=SRFM_SMOL, bcfl=BCFL_SDH,
              pdie=2.0, sdie=78.54, srad=1.4, sdens=10.0, temp=298.15,
              ions=((1.0, 0.15, 2.0), (-1.0, 0.15, 2.0)), etol=0.0,
              nlev=None) -> PmgbParams:
    """Parameter block of one mg-manual ELEC calculation."""
    if np.isscalar(dime):
        dime = (int(dime),) * 3
    if np.isscalar(grid):
        grid = (float(grid),) * 3
    p = PmgbParams()
    p.nx, p.ny, p.nz = (int(d) for d in dime)
    p.nlev = int(nlev) if nlev else min(mgparm_nlev(d) for d in dime)
    p.hx, p.hy, p.hz = (float(h) for h in grid)
    for i in range(3):
        p.center[i] = float(center[i])
    p.nonlin = 1 if npbe else 0
    p.srfm = srfm
    p.chgm = CHGM_SPL2
    p.bcfl = bcfl
    p.pdie, p.sdie, p.srad, p.sdens, p.temp = pdie, sdie, srad, sdens, temp
    p.etol = etol
    p.nion = len(ions)
    for i, (qq, cc, rr) in enumerate(ions):
        p.ion_q[i], p.ion_conc[i], p.ion_radius[i] = qq, cc, rr
    return p


def config0(seed: int = 0):
    """65^3 LPBE, 500 atoms in a 12 A ball, 0.15 M 1:1 salt, spl2/smol/sdh."""
    mol = cluster(500, 12.0, seed)
    return mol, mg_manual(65, 0.5, mol.center())


def config1(seed: int = 1):
    """161^3 NPBE, 5000 atoms in a 25 A ball, net +12, 0.1 M 1:1 salt."""
    mol = cluster(5000, 25.0, seed, net_charge=12.0)
    return mol, mg_manual(161, 0.4, mol.center(), npbe=True,
                          ions=((1.0, 0.1, 2.0), (-1.0, 0.1, 2.0)))


def subregion_center(mol: Molecule, nsub: int, seed: int) -> np.ndarray:
    """Bounding-box midpoint of a seeded sub-region: one atom drawn from the
    seed and its ``nsub - 1`` nearest neighbours."""
    rng = np.random.default_rng(seed)
    a = int(rng.integers(mol.natoms))
    d = np.einsum("ij,ij->i", mol.xyz - mol.xyz[a], mol.xyz - mol.xyz[a])
    sel = mol.xyz[np.argsort(d, kind="stable")[:nsub]]
    return 0.5 * (sel.max(axis=0) + sel.min(axis=0))


def focus_pair(mol: Molecule, coarse_dime, coarse_h, fine_dime, fine_h, fine_center,
               **kw):
    """Coarse (bcfl sdh) and fine (bcfl focus) mg-manual blocks of one focusing
    chain.  The fine centre is moved inside the coarse box where needed, as
    the mg-auto setup keeps the fine domain inside the coarse one."""
    pc = mg_manual(coarse_dime, coarse_h, mol.center(), bcfl=BCFL_SDH, **kw)
    half_c = 0.5 * (coarse_dime - 1) * coarse_h
    half_f = 0.5 * (fine_dime - 1) * fine_h
    c0 = mol.center()
    fc = np.clip(np.asarray(fine_center, dtype=float), c0 - half_c + half_f, c0 + half_c - half_f)
    pf = mg_manual(fine_dime, fine_h, fc, bcfl=BCFL_FOCUS, **kw)
    return pc, pf


def config2(seed: int = 1):
    """Focusing on the 161^3 molecule: coarse 97^3 at 1.0 A, then fine 129^3 at
    0.35 A centred on a 30-atom sub-region; LPBE, 0.1 M 1:1 salt."""
    mol = cluster(5000, 25.0, seed, net_charge=12.0)
    pc, pf = focus_pair(mol, 97, 1.0, 129, 0.35, subregion_center(mol, 30, seed + 100),
                        ions=((1.0, 0.1, 2.0), (-1.0, 0.1, 2.0)))
    return mol, pc, pf


def _rotation(rng) -> np.ndarray:
    """Uniform random rotation (QR of a Gaussian matrix, sign-fixed)."""
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def binding_sweep(npose: int = 64, seed: int = 3, rec_atoms: int = 3000, rec_radius: float = 20.0,
                  lig_atoms: int = 40, lig_radius: float = 5.0, rec_dime: int = 129,
                  lig_dimes=(33, 49, 65), h: float = 0.55,
                  ions=((1.0, 0.15, 2.0), (-1.0, 0.15, 2.0)), etol: float = 0.0):
    """Binding-energy sweep: a receptor cluster and `npose` seeded rigid poses
    of a ligand cluster (net charge -1) placed on the receptor surface.

    Returns (receptor job, [(complex job, ligand job)] * npose), each job a
    (params, molecule) pair, all LPBE.  The receptor and every complex use
    the same grid (rec_dime^3 at spacing h centred on the receptor); each
    ligand grid has the same spacing, a dimension drawn from `lig_dimes`, and
    a centre on the same lattice, so the three energies of a pose share the
    grid placement and dG = E_complex - E_receptor - E_ligand.  etol is the
    solver tolerance of every job (0: the default 1e-6)."""
    rng = np.random.default_rng(seed)
    rec = cluster(rec_atoms, rec_radius, seed)
    lig0 = cluster(lig_atoms, lig_radius, seed + 1, net_charge=-1.0)
    lig0 = Molecule(lig0.xyz - lig0.xyz.mean(axis=0), lig0.charge, lig0.radius)
    c = rec.center()
    rec_job = (mg_manual(rec_dime, h, c, ions=ions, etol=etol), rec)
    half = 0.5 * (rec_dime - 1) * h
    pairs = []
    for _ in range(npose):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        pos = c + d * (rec_radius + lig_radius + 1.5)
        lig = Molecule(lig0.xyz @ _rotation(rng).T + pos, lig0.charge, lig0.radius)
        cplx = Molecule(np.vstack([rec.xyz, lig.xyz]), np.concatenate([rec.charge, lig.charge]),
                        np.concatenate([rec.radius, lig.radius]))
        assert np.all(np.abs(cplx.xyz - c) < half - 2.0), "complex leaves the grid"
        dime = int(rng.choice(lig_dimes))
        # ligand grid centre on the receptor lattice nearest the ligand centre
        lc = c + np.round((lig.center() - c) / h) * h
        pairs.append(((mg_manual(rec_dime, h, c, ions=ions, etol=etol), cplx),
                      (mg_manual(dime, h, lc, ions=ions, etol=etol), lig)))
    return rec_job, pairs
