"""The allocation-free energy entry point (pmgb_energy_noalloc) against the
allocating one (pmgb_energy) on the same solved state.

Callers that cannot allocate device memory when they need the energy --
code inside another framework's memory pool, or with a fixed device
footprint -- hand in device arrays they already hold; the
result must equal what the solver's own energy call reports.  Two calls in
a row check that the shared scratch array carries nothing over.  This file
is collected last so a failure here never hides another test's result."""
import numpy as np
import pytest

from apbs_b200 import synth, vpmg

pytestmark = pytest.mark.gpu

REL = 1e-12


def _cases():
    m0, p0 = synth.config0()
    m1 = synth.cluster(120, 6.0, seed=11, net_charge=-2.0)
    p1 = synth.mg_manual(33, 0.6, m1.center(), npbe=True, ions=((2, 0.05, 2.0), (-1, 0.1, 1.8)))
    return [("lpbe65", m0, p0), ("npbe33", m1, p1)]


@pytest.mark.parametrize("name,mol,params", _cases(), ids=["lpbe65", "npbe33"])
def test_energy_noalloc_matches_pmgb_energy(name, mol, params):
    import torch

    with vpmg.Vpmg(params, vpmg.FP64) as pmg:
        pmg.fillco(mol)
        pmg.solve()
        e_ref = pmg.energy()
        u = pmg.u
        maps = pmg.maps()
    dev = torch.device("cuda", 0)
    t = {k: torch.tensor(np.ascontiguousarray(v), dtype=torch.float64, device=dev)
         for k, v in (("u", u), ("charge", maps["charge"]), ("epsx", maps["epsx"]),
                      ("epsy", maps["epsy"]), ("epsz", maps["epsz"]), ("kappa", maps["kappa"]))}
    torch.cuda.synchronize()
    got = []
    for _ in range(2):
        got.append(vpmg.energy_noalloc(params, t["u"].data_ptr(), t["charge"].data_ptr(),
                                       t["epsx"].data_ptr(), t["epsy"].data_ptr(),
                                       t["epsz"].data_ptr(), t["kappa"].data_ptr()))
    for e in got:
        assert abs(e - e_ref) <= REL * abs(e_ref), (e, e_ref)
