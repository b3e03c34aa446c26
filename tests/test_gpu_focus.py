"""Focusing on the device (pmgb_focus): fine-grid faces from the coarse
potential and the external energy, against the reference's own focusing
chain compiled from source (Vpmg_ctor with focusFlag, focusFillBound,
extEnergy)."""
import numpy as np
import pytest

from apbs_b200 import synth
from apbs_b200.vpmg import FP64, MIXED, PmgbError, Vpmg
from oracle import port, ref

pytestmark = pytest.mark.gpu

REL_U = 1e-9       # FP64 drop-in bar, relative to max |u|
REL_E = 1e-9
REL_MIXED_E = 1e-6  # mixed precision against FP64


def _checker():
    return ref if ref.available() else port


def _cases():
    m = synth.cluster(200, 9.0, seed=5, net_charge=2.0)
    c = synth.subregion_center(m, 30, 7)
    m2 = synth.cluster(150, 8.0, seed=9, net_charge=-1.0)
    m3 = synth.cluster(1000, 14.0, seed=3, net_charge=4.0)
    return [
        ("lpbe33", m, *synth.focus_pair(m, 33, 1.0, 33, 0.45, c)),
        ("npbe33", m, *synth.focus_pair(m, 33, 1.0, 33, 0.45, c, npbe=True,
                                        ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))),
        ("lpbe49to33_mol_2to1", m2, *synth.focus_pair(
            m2, 49, 0.9, 33, 0.5, synth.subregion_center(m2, 30, 3), srfm=synth.SRFM_MOL,
            ions=((2, 0.05, 2.0), (-1, 0.1, 1.8)))),
        ("lpbe65to65", m3, *synth.focus_pair(m3, 65, 1.0, 65, 0.35,
                                             synth.subregion_center(m3, 30, 11))),
    ]


CASES = _cases()


def _run(mol, pc, pf, precision):
    with Vpmg(pc, precision) as coarse, Vpmg(pf, precision) as fine:
        coarse.fillco(mol)
        coarse.solve()
        e_coarse = coarse.energy()
        fine.focus(coarse, calc_energy=True)
        fine.fillco(mol)
        faces = fine.maps()["faces"]
        fine.solve()
        return dict(energy_kT=fine.energy(), u=fine.u, faces=faces, stats=fine.stats(),
                    hist=fine.residual_history(), coarse_energy_kT=e_coarse)


@pytest.mark.parametrize("name,mol,pc,pf", CASES, ids=[c[0] for c in CASES])
def test_focus_matches_reference(name, mol, pc, pf):
    want = _checker().focus(pc, pf, mol, want_faces=True)
    got = _run(mol, pc, pf, FP64)
    fscale = np.abs(want["faces"]).max()
    assert np.abs(got["faces"] - want["faces"]).max() <= 1e-12 * fscale
    st = got["stats"]
    for k, w in (("ext_qf", "ext_qf"), ("ext_diel", "ext_diel"), ("ext_qm", "ext_qm")):
        assert abs(st[k] - want[w]) <= 1e-10 * max(abs(want[w]), 1e-30), k
    assert abs(got["coarse_energy_kT"] - want["coarse_energy_kT"]) <= REL_E * abs(
        want["coarse_energy_kT"])
    scale = np.abs(want["u"]).max()
    assert np.abs(got["u"] - want["u"]).max() <= REL_U * scale
    assert abs(got["energy_kT"] - want["energy_kT"]) <= REL_E * abs(want["energy_kT"])


def test_focus_config2_mixed_and_fp64():
    """The 97^3 -> 129^3 focusing workload: FP64 against the reference and
    mixed precision against FP64."""
    mol, pc, pf = synth.config2()
    want = _checker().focus(pc, pf, mol)
    g64 = _run(mol, pc, pf, FP64)
    assert abs(g64["energy_kT"] - want["energy_kT"]) <= REL_E * abs(want["energy_kT"])
    assert np.abs(g64["u"] - want["u"]).max() <= REL_U * np.abs(want["u"]).max()
    gmx = _run(mol, pc, pf, MIXED)
    assert abs(gmx["energy_kT"] - g64["energy_kT"]) <= REL_MIXED_E * abs(g64["energy_kT"])
    assert np.abs(gmx["u"] - g64["u"]).max() <= 1e-5 * np.abs(g64["u"]).max()


def test_focus_errors():
    m = synth.cluster(100, 6.0, seed=2)
    pc, pf = synth.focus_pair(m, 33, 0.5, 33, 0.3, m.center())
    with Vpmg(pc, FP64) as coarse, Vpmg(pf, FP64) as fine:
        # a focus block cannot be filled before it has a parent (initMG refuses)
        with pytest.raises(PmgbError):
            fine.fillco(m)
        # the parent must have been solved
        coarse.fillco(m)
        with pytest.raises(PmgbError):
            fine.focus(coarse)
    # a fine box reaching outside the coarse one is refused (the reference asserts)
    far = synth.mg_manual(33, 0.3, m.center() + np.array([6.0, 0.0, 0.0]), bcfl=synth.BCFL_FOCUS)
    with Vpmg(pc, FP64) as coarse, Vpmg(far, FP64) as fine:
        coarse.fillco(m)
        coarse.solve()
        with pytest.raises(PmgbError):
            fine.focus(coarse)
