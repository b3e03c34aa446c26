"""Pins the C restatement (oracle/pmg_oracle.c) against the reference APBS
sources compiled unchanged (oracle/_ref).  CPU only."""
import numpy as np
import pytest

from apbs_b200 import synth
from oracle import port, ref

pytestmark = pytest.mark.skipif(not (ref.available() and port.available()),
                                reason="oracle libraries not built")


def _cases():
    m0, p0 = synth.config0()
    m1 = synth.cluster(300, 10.0, seed=5, net_charge=3.0)
    p1 = synth.mg_manual(65, 0.5, m1.center(), npbe=True, ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    m2 = synth.cluster(400, 12.0, seed=7)
    p2 = synth.mg_manual(97, 0.4, m2.center())
    p3 = synth.mg_manual(49, 0.8, m2.center(), srfm=synth.SRFM_MOL)
    m4 = synth.cluster(120, 6.0, seed=11, net_charge=-2.0)
    p4 = synth.mg_manual(33, 0.6, m4.center(), npbe=True, ions=((2, 0.05, 2.0), (-1, 0.1, 1.8)))
    m5 = synth.cluster(150, 8.0, seed=11, net_charge=2.0)
    p5 = synth.mg_manual(33, 0.6, m5.center(), bcfl=synth.BCFL_MDH)
    p6 = synth.mg_manual(33, 0.6, m5.center(), bcfl=synth.BCFL_MDH, npbe=True)
    p6.chgm = synth.CHGM_TRIL
    p7 = synth.mg_manual(33, 0.6, m5.center(), ions=())
    p7.chgm = synth.CHGM_TRIL
    return [("config0", m0, p0), ("npbe65", m1, p1), ("lpbe97_band", m2, p2),
            ("lpbe49_mol", m2, p3), ("npbe33_2to1", m4, p4), ("lpbe33_mdh", m5, p5),
            ("npbe33_mdh_spl0", m5, p6), ("lpbe33_spl0_noions", m5, p7)]


@pytest.mark.parametrize("name,mol,params", _cases(), ids=lambda c: c if isinstance(c, str) else "")
def test_restatement_matches_reference(name, mol, params):
    a = ref.run(params, mol, want_maps=True, want_faces=True)
    b = port.run(params, mol, want_maps=True, want_faces=True)
    # fill maps and faces: bitwise (identical expression trees)
    for k in ("charge", "epsx", "epsy", "epsz", "kappa"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(a["faces"], b["faces"])
    # same iteration history (the reference log is printed with 7 digits)
    assert len(a["reslog"]) == len(b["reslog"])
    np.testing.assert_allclose(b["reslog"], a["reslog"], rtol=2e-6)
    # potential and energy to the round-off level
    scale = np.abs(a["u"]).max()
    assert np.abs(a["u"] - b["u"]).max() <= 1e-12 * scale
    assert abs(a["energy_kT"] - b["energy_kT"]) <= 1e-12 * abs(a["energy_kT"])


def _focus_cases():
    m = synth.cluster(200, 9.0, seed=5, net_charge=2.0)
    c = synth.subregion_center(m, 30, 7)
    lp = synth.focus_pair(m, 33, 1.0, 33, 0.45, c)
    np_ = synth.focus_pair(m, 33, 1.0, 33, 0.45, c, npbe=True,
                           ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    m2 = synth.cluster(150, 8.0, seed=9, net_charge=-1.0)
    lp2 = synth.focus_pair(m2, 49, 0.9, 33, 0.5, synth.subregion_center(m2, 30, 3),
                           srfm=synth.SRFM_MOL, ions=((2, 0.05, 2.0), (-1, 0.1, 1.8)))
    return [("lpbe33_focus", m, *lp), ("npbe33_focus", m, *np_), ("lpbe49to33_mol_2to1", m2, *lp2)]


@pytest.mark.parametrize("name,mol,pc,pf", _focus_cases(), ids=lambda c: c if isinstance(c, str) else "")
def test_focusing_restatement_matches_reference(name, mol, pc, pf):
    a = ref.focus(pc, pf, mol, want_faces=True)
    b = port.focus(pc, pf, mol, want_faces=True)
    # the faces interpolate coarse potentials that agree to round-off
    fscale = np.abs(a["faces"]).max()
    assert np.abs(a["faces"] - b["faces"]).max() <= 1e-13 * fscale
    for k in ("ext_qf", "ext_diel", "ext_qm", "coarse_energy_kT"):
        assert abs(a[k] - b[k]) <= 1e-12 * max(abs(a[k]), 1e-30), k
    assert len(a["reslog"]) == len(b["reslog"])
    np.testing.assert_allclose(b["reslog"], a["reslog"], rtol=2e-6)
    scale = np.abs(a["u"]).max()
    assert np.abs(a["u"] - b["u"]).max() <= 1e-12 * scale
    assert abs(a["energy_kT"] - b["energy_kT"]) <= 1e-12 * abs(a["energy_kT"])
    # the focused energy differs from the plain one by the external term
    assert a["ext_qf"] != 0.0


@pytest.mark.parametrize("npbe", [False, True], ids=["lpbe", "npbe"])
def test_iteration_limit_restated(npbe):
    """itmax below what convergence needs: the reference stops after itmax
    V-cycles (LPBE) or Newton steps (NPBE) and returns its iterate; the
    restatement stops at the same point."""
    m = synth.cluster(120, 6.0, seed=11, net_charge=-2.0)
    p = synth.mg_manual(33, 0.6, m.center(), npbe=npbe, ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    p.itmax = 1
    a = ref.run(p, m)
    b = port.run(p, m)
    assert len(a["reslog"]) == len(b["reslog"])
    assert a["reslog"][-1] > 1e-6          # not converged
    np.testing.assert_allclose(b["reslog"], a["reslog"], rtol=2e-6)
    scale = np.abs(a["u"]).max()
    assert np.abs(a["u"] - b["u"]).max() <= 1e-12 * scale
