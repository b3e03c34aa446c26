"""The potential and fill maps of a calculation written to OpenDX on the
device path (pmgb_write_dx): the header of writedataMG, the values in
x-major order equal to the calculation's arrays at the file's six digits."""
import numpy as np
import pytest

from apbs_b200 import synth
from apbs_b200.vpmg import DX_KAPPA, DX_POT, FP64, Vpmg

pytestmark = pytest.mark.gpu


def _read_dx(path):
    lines = open(path).read().splitlines()
    i = next(n for n, l in enumerate(lines) if l.startswith("object 3"))
    counts = [int(v) for v in lines[4].split()[-3:]]
    vals = []
    for l in lines[i + 1:]:
        if l.startswith("attribute"):
            break
        vals.extend(float(v) for v in l.split())
    return lines, counts, np.array(vals)


def test_potential_and_kappa_dx(tmp_path):
    m, p = synth.config0()
    with Vpmg(p, FP64) as pmg:
        pmg.fillco(m)
        pmg.solve()
        u = pmg.u
        kappa = pmg.maps()["kappa"]
        pmg.write_dx(tmp_path / "pot.dx", DX_POT)
        pmg.write_dx(tmp_path / "kappa.dx", DX_KAPPA)
    for name, arr, title in (("pot.dx", u, "POTENTIAL (kT/e)"), ("kappa.dx", kappa, "KAPPA MAP")):
        lines, counts, vals = _read_dx(tmp_path / name)
        assert lines[0] == "# Data from APBS 3.4.1" and lines[2] == "# " + title
        assert counts == [p.nx, p.ny, p.nz]
        want = np.transpose(arr, (2, 1, 0)).reshape(-1)  # x-major, z fastest
        assert vals.shape == want.shape
        assert np.all(np.abs(vals - want) <= 5e-7 * np.abs(want) + 1e-300)
