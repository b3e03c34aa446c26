"""The reference's regression decks ([born], [ionize], [solv] of its
tests/test_cases.cfg, fixtures in tests/golden/) run by the reference
compiled here (oracle/_ref) through the harness in golden_decks.py: this
pins the harness -- deck reading, mg-auto focusing geometry, unit
conversion -- against the energies APBS publishes for those decks, so the
GPU run of the same decks (test_gpu_golden.py) is checked against published
numbers, not only against this build's oracle.  CPU only."""
import pytest

import golden_decks as gd
from oracle import ref

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def _ref_chain(levels, mol):
    return list(ref.chain(levels, mol)["energies_kT"])


@pytest.mark.parametrize("name", gd.FIXTURES)
def test_reference_reproduces_published_energies(name):
    fx = gd.load(name)
    got = gd.deck_values(fx, _ref_chain)
    assert not gd.mismatches(got, fx["expected_kJ_per_mol"]), gd.mismatches(
        got, fx["expected_kJ_per_mol"])
