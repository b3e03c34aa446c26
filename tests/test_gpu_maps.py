"""Coefficient and charge maps given on their own grids ("usemap diel",
"usemap kappa", "usemap charge") on the device against the reference
compiled from source with the same maps: the fill maps bitwise, the
potential and energy to 1e-9.  The maps are those of another calculation
over a larger box, written to OpenDX and read back, as a user would make
them."""
import numpy as np
import pytest

from apbs_b200 import synth, vpmg
from apbs_b200.vpmg import FP64, MAP_DIELX, MAP_KAPPA, MAP_POT, PmgbError, Vpmg
from oracle import ref

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")]

REL_U = 1e-9
REL_E = 1e-9
IONS = ((1.0, 0.15, 2.0), (-1.0, 0.15, 2.0))


def _source_maps(tmp_path, mol, kappa_scale=1.0):
    """Maps of a 49^3, 0.8 A calculation around the molecule, through DX files."""
    p = synth.mg_manual(49, 0.8, mol.center(), srfm=synth.SRFM_SPL2, ions=IONS)
    r = ref.run(p, mol, want_maps=True)
    h = (p.hx, p.hy, p.hz)
    origin = [p.center[d] - 0.5 * (n - 1) * hd for d, (n, hd) in
              enumerate(zip((p.nx, p.ny, p.nz), h))]
    out = {}
    for m, key, scale in ((0, "epsx", 1.0), (1, "epsy", 1.0), (2, "epsz", 1.0),
                          (3, "kappa", kappa_scale), (4, "charge", 1e-3)):
        path = tmp_path / ("%s.dx" % key)
        vpmg.write_dx(path, r[key] * scale, h, origin)
        out[m] = vpmg.read_dx(path)
    return out


@pytest.mark.parametrize("which", ["coef", "coef_charge", "coef_kappa_scaled", "charge"])
def test_usemap_matches_reference(tmp_path, which):
    mol = synth.cluster(150, 8.0, seed=13, net_charge=1.0)
    maps = _source_maps(tmp_path, mol, kappa_scale=2.5 if which == "coef_kappa_scaled" else 1.0)
    use = {"coef": (0, 1, 2, 3), "coef_charge": (0, 1, 2, 3, 4),
           "coef_kappa_scaled": (0, 1, 2, 3), "charge": (4,)}[which]
    sel = {m: maps[m] for m in use}
    p = synth.mg_manual(33, 0.9, mol.center(), ions=IONS)
    want = ref.run_maps(p, mol, sel)
    with Vpmg(p, FP64) as pmg:
        for m, (data, h, origin) in sel.items():
            pmg.set_map(m, data, h, origin)
        pmg.fillco(mol)
        got = pmg.maps()
        pmg.solve()
        u, e = pmg.u, pmg.energy()
    for k in ("epsx", "epsy", "epsz", "kappa", "charge"):
        if k == "charge" and 4 not in use:
            continue  # atom charges: scattered with atomics, checked elsewhere
        assert np.array_equal(got[k], want[k]), k
    assert np.abs(u - want["u"]).max() <= REL_U * np.abs(want["u"]).max()
    assert abs(e - want["energy_kT"]) <= REL_E * abs(want["energy_kT"])


def test_usemap_needs_every_dielectric_map(tmp_path):
    mol = synth.cluster(80, 6.0, seed=2)
    maps = _source_maps(tmp_path, mol)
    p = synth.mg_manual(33, 0.9, mol.center(), ions=IONS)
    with Vpmg(p, FP64) as pmg:
        pmg.set_map(MAP_DIELX, *maps[MAP_DIELX])
        with pytest.raises(PmgbError):
            pmg.fillco(mol)
        pmg.set_map(MAP_DIELX, None, None, None)
        pmg.fillco(mol)  # back to the surface of the atoms


def test_usemap_off_the_map_fails(tmp_path):
    mol = synth.cluster(80, 6.0, seed=2)
    maps = _source_maps(tmp_path, mol)
    p = synth.mg_manual(65, 0.9, mol.center(), ions=IONS)  # wider than the maps
    with Vpmg(p, FP64) as pmg:
        for m in (0, 1, 2, MAP_KAPPA):
            pmg.set_map(m, *maps[m])
        with pytest.raises(PmgbError):
            pmg.fillco(mol)


def test_bcfl_map_matches_reference(tmp_path):
    """bcfl map: the faces interpolated from a potential map (a coarse
    solve over a larger box, through a DX file), as focusFillBound does with
    the map in place of the coarse grid."""
    mol = synth.cluster(150, 8.0, seed=13, net_charge=1.0)
    pc = synth.mg_manual(49, 1.0, mol.center(), ions=IONS)
    rc = ref.run(pc, mol)
    h = (pc.hx, pc.hy, pc.hz)
    origin = [pc.center[d] - 0.5 * (n - 1) * hd for d, (n, hd) in
              enumerate(zip((pc.nx, pc.ny, pc.nz), h))]
    vpmg.write_dx(tmp_path / "pot.dx", rc["u"], h, origin, title="POTENTIAL (kT/e)")
    pot = vpmg.read_dx(tmp_path / "pot.dx")
    p = synth.mg_manual(33, 0.9, mol.center(), ions=IONS, bcfl=synth.BCFL_MAP)
    want = ref.run_maps(p, mol, {MAP_POT: pot})
    with Vpmg(p, FP64) as pmg:
        pmg.set_map(MAP_POT, *pot)
        pmg.fillco(mol)
        pmg.solve()
        u, e = pmg.u, pmg.energy()
    assert np.abs(u - want["u"]).max() <= REL_U * np.abs(want["u"]).max()
    assert abs(e - want["energy_kT"]) <= REL_E * abs(want["energy_kT"])
    # the boundary is the map's, not a Debye-Hueckel one
    assert np.abs(u[0] - want["u"][0]).max() <= 1e-12 * np.abs(want["u"][0]).max()
