"""The reference's regression decks ([born], [ionize], [solv] of its
tests/test_cases.cfg; fixtures in tests/golden/) solved on the GPU through
the C ABI: every calculation of an mg-auto block is a level of a focusing
chain (pmgb_focus from the level before, then fill, solve, energy), an
mg-manual block one calculation.  Every energy APBS publishes for these
decks must pass the reference's own check (6 significant figures, 1e-4
relative), in FP64 and in mixed precision."""
import pytest

import golden_decks as gd
from apbs_b200.vpmg import FP64, MIXED, Vpmg

pytestmark = pytest.mark.gpu


def _gpu_chain(precision):
    def run(levels, mol):
        energies, prev = [], None
        try:
            for p in levels:
                pmg = Vpmg(p, precision)
                if prev is not None:
                    pmg.focus(prev, calc_energy=True)
                    prev.close()
                pmg.fillco(mol)
                pmg.solve()
                energies.append(pmg.energy())
                prev = pmg
        finally:
            if prev is not None:
                prev.close()
        return energies
    return run


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", gd.FIXTURES)
def test_published_energies_on_the_gpu(name, precision):
    fx = gd.load(name)
    got = gd.deck_values(fx, _gpu_chain(precision))
    bad = gd.mismatches(got, fx["expected_kJ_per_mol"])
    assert not bad, bad
