"""The reference's unchanged call sequence (Vpmg_ctor -> Vpmg_fillco ->
Vpmg_solve -> Vpmg_setPart -> Vpmg_energy, oracle/ref_driver.c, as
initMG/solveMG/setPartMG/energyMG run it) with Vpmg_solve routed to the GPU
by the drop-in binding (apbs_b200/dropin/vpmg_b200.c), against the same
sequence with the reference's own Vpmg_solve: thee->u after the solve and
the energies computed from it by the reference's host code agree to 1e-9,
for an LPBE and an NPBE block and for a focusing chain (both solves on the
GPU, the fine faces interpolated by the reference from the GPU's coarse
potential).  APBS_B200_PRECISION=mixed runs the mixed-precision solver
behind the same symbol (1e-6 in energy)."""
import numpy as np
import pytest

from apbs_b200 import synth
from oracle import ref

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (ref.available() and ref.dropin_available()),
                                 reason="reference or drop-in not built")]

REL = 1e-9


def _cases():
    m0, p0 = synth.config0()
    m1 = synth.cluster(300, 10.0, seed=5, net_charge=3.0)
    p1 = synth.mg_manual(65, 0.5, m1.center(), npbe=True, ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    m2 = synth.cluster(400, 12.0, seed=7)
    p2 = synth.mg_manual(97, 0.4, m2.center())
    return [("config0_lpbe65", m0, p0), ("npbe65", m1, p1), ("lpbe97", m2, p2)]


@pytest.mark.parametrize("name,mol,params", _cases(), ids=[c[0] for c in _cases()])
def test_dropin_sequence_matches_reference(name, mol, params):
    want = ref.run(params, mol)
    got = ref.run(params, mol, dropin=True)
    scale = np.abs(want["u"]).max()
    assert np.abs(got["u"] - want["u"]).max() <= REL * scale
    assert abs(got["energy_kT"] - want["energy_kT"]) <= REL * abs(want["energy_kT"])
    for k in ("qf", "diel", "qm"):
        assert abs(got[k] - want[k]) <= REL * max(abs(want[k]), 1e-300), k


def test_dropin_focusing_chain_matches_reference():
    mol, pc, pf = synth.config2()
    want = ref.focus(pc, pf, mol)
    got = ref.focus(pc, pf, mol, dropin=True)
    scale = np.abs(want["u"]).max()
    assert np.abs(got["u"] - want["u"]).max() <= REL * scale
    assert abs(got["energy_kT"] - want["energy_kT"]) <= REL * abs(want["energy_kT"])
    assert abs(got["coarse_energy_kT"] - want["coarse_energy_kT"]) <= \
        REL * abs(want["coarse_energy_kT"])
    for k in ("ext_qf", "ext_diel", "ext_qm"):
        assert abs(got[k] - want[k]) <= REL * max(abs(want[k]), 1e-300), k


def test_dropin_mixed_precision(monkeypatch):
    monkeypatch.setenv("APBS_B200_PRECISION", "mixed")
    m1 = synth.cluster(300, 10.0, seed=5, net_charge=3.0)
    p1 = synth.mg_manual(65, 0.5, m1.center(), npbe=True, ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    want = ref.run(p1, m1)
    got = ref.run(p1, m1, dropin=True)
    assert abs(got["energy_kT"] - want["energy_kT"]) <= 1e-6 * abs(want["energy_kT"])
    assert np.abs(got["u"] - want["u"]).max() <= 1e-5 * np.abs(want["u"]).max()
