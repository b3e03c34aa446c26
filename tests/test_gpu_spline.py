"""Spline-based surfaces (srfm spl2, spl3 and spl4: fillcoCoefSpline,
fillcoCoefSpline3, fillcoCoefSpline4), the charge discretisations (chgm
spl0, spl2 and spl4: fillcoChargeSpline1/2, fillcoPermanentMultipole with
atomic charges) and the per-atom forces (Vpmg_qfForce, Vpmg_dbForce,
Vpmg_ibForce) on the device against the reference compiled from source
(oracle/_ref): the kappa and dielectric maps bitwise, the potential and
energy to 1e-9, every force component to 1e-8 of the largest force of its
kind (the forces difference the potential, whose two solves agree to
round-off, not bit for bit)."""
import numpy as np
import pytest

from apbs_b200 import synth
from apbs_b200.vpmg import FP64, PmgbError, Vpmg
from oracle import ref

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")]

REL_U = 1e-9
REL_E = 1e-9
REL_F = 1e-8

IONS = ((1.0, 0.15, 2.0), (-1.0, 0.15, 2.0))


def _cases():
    m1 = synth.cluster(200, 9.0, seed=3, net_charge=2.0)
    p1 = synth.mg_manual(65, 0.5, m1.center(), srfm=synth.SRFM_SPL2, ions=IONS)
    p2 = synth.mg_manual(65, 0.5, m1.center(), srfm=synth.SRFM_SPL2, npbe=True, ions=IONS)
    m3 = synth.cluster(120, 7.0, seed=9, net_charge=-1.0)
    p3 = synth.mg_manual((49, 65, 57), (0.45, 0.4, 0.5), m3.center(), srfm=synth.SRFM_SPL2,
                         ions=((2.0, 0.05, 2.0), (-1.0, 0.1, 1.8)))
    p3.chgm = synth.CHGM_TRIL
    p4 = synth.mg_manual(49, 0.55, m3.center(), srfm=synth.SRFM_SPL2, ions=())
    p4.swin = 0.4
    p5 = synth.mg_manual(65, 0.5, m1.center(), srfm=synth.SRFM_SPL4, ions=IONS)
    p6 = synth.mg_manual(57, 0.5, m3.center(), srfm=synth.SRFM_SPL4, npbe=True, ions=IONS)
    p7 = synth.mg_manual(65, 0.5, m1.center(), srfm=synth.SRFM_SPL3, ions=IONS)
    p8 = synth.mg_manual(57, 0.5, m3.center(), srfm=synth.SRFM_SPL3, npbe=True, ions=IONS)
    p9 = synth.mg_manual(49, 0.55, m3.center(), srfm=synth.SRFM_SPL3, ions=())
    p9.swin = 0.4
    p10 = synth.mg_manual(65, 0.5, m1.center(), srfm=synth.SRFM_SPL2, ions=IONS)
    p10.chgm = synth.CHGM_SPL4
    p11 = synth.mg_manual(57, 0.5, m3.center(), srfm=synth.SRFM_SPL4, npbe=True, ions=IONS)
    p11.chgm = synth.CHGM_SPL4
    return [("lpbe65_chgm_spl4", m1, p10), ("npbe57_spl4_chgm_spl4", m3, p11),
            ("lpbe65", m1, p1), ("npbe65", m1, p2), ("lpbe_box_spl0", m3, p3),
            ("lpbe49_noions_swin04", m3, p4), ("lpbe65_spl4", m1, p5), ("npbe57_spl4", m3, p6),
            ("lpbe65_spl3", m1, p7), ("npbe57_spl3", m3, p8),
            ("lpbe49_spl3_noions_swin04", m3, p9)]


CASES = _cases()


@pytest.mark.parametrize("name,mol,params", CASES, ids=[c[0] for c in CASES])
def test_spline_surface_solve_and_forces(name, mol, params):
    want = ref.run(params, mol, want_maps=True, want_forces=True)
    assert want["fstatus"].min() == 1
    with Vpmg(params, FP64) as pmg:
        pmg.fillco(mol)
        maps = pmg.maps()
        pmg.solve()
        u = pmg.u
        e = pmg.energy()
        f = pmg.forces()
    for k in ("epsx", "epsy", "epsz", "kappa"):
        assert np.array_equal(maps[k], want[k]), k
    assert np.abs(u - want["u"]).max() <= REL_U * np.abs(want["u"]).max()
    assert abs(e - want["energy_kT"]) <= REL_E * abs(want["energy_kT"])
    for k in ("qf", "db", "ib"):
        scale = np.abs(want[k]).max()
        assert np.abs(f[k] - want[k]).max() <= REL_F * max(scale, 1e-30), k
    # the boundary forces are not identically zero where they should not be
    assert np.abs(want["db"]).max() > 0.0
    if params.nion:
        assert np.abs(want["ib"]).max() > 0.0


def test_boundary_forces_need_spline_surfaces():
    """As the reference: the dielectric and ionic boundary forces are only
    defined for spline surfaces; the charge-field force is not."""
    m = synth.cluster(100, 6.0, seed=2)
    p = synth.mg_manual(33, 0.6, m.center())
    with Vpmg(p, FP64) as pmg:
        pmg.fillco(m)
        pmg.solve()
        qf = pmg.forces(boundary=False)["qf"]
        with pytest.raises(PmgbError):
            pmg.forces(boundary=True)
    want = ref.run(p, m, want_forces=True)
    assert np.abs(qf - want["qf"]).max() <= REL_F * np.abs(want["qf"]).max()
