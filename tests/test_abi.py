"""C-ABI checks that need no GPU: the library loads and exports every entry
point the public header declares; without a device the API fails cleanly."""
import ctypes
import os
import re

import pytest

from apbs_b200 import synth, vpmg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in ("apbs_b200.h",):
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names.update(re.findall(r"\b(pmgb_[a-z_0-9]+)\s*\(", txt))
    return sorted(names)


def test_header_declares_entry_points():
    names = _declared()
    for n in ("pmgb_create", "pmgb_fillco", "pmgb_solve", "pmgb_energy", "pmgb_destroy"):
        assert n in names


@pytest.mark.skipif(not os.path.exists(vpmg.LIB_PATH), reason="library not built")
def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(vpmg.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, missing


@pytest.mark.skipif(not os.path.exists(vpmg.LIB_PATH), reason="library not built")
def test_create_fails_loudly_without_device(gpu_available):
    if gpu_available:
        pytest.skip("a GPU is present")
    _, p = synth.config0()
    with pytest.raises(vpmg.PmgbError):
        vpmg.Vpmg(p)


def test_nlev_rule():
    # MGparm_check (src/generic/mgparm.c:263-330)
    assert synth.mgparm_nlev(65) == 5
    assert synth.mgparm_nlev(161) == 4
    assert synth.mgparm_nlev(129) == 6
    assert synth.mgparm_nlev(97) == 4
    assert synth.mgparm_nlev(33) == 4
    assert synth.mgparm_nlev(49) == 3
    assert synth.mgparm_nlev(225) == 4


@pytest.mark.skipif(not os.path.exists(vpmg.LIB_PATH), reason="library not built")
@pytest.mark.parametrize("what,edit,msg", [
    ("axis over the limit", lambda p: setattr(p, "nx", vpmg.NOALLOC_MAX_DIM + 2), "points per axis"),
    ("axis too small", lambda p: setattr(p, "nz", 2), "points per axis"),
    ("chgm spl0", lambda p: setattr(p, "chgm", synth.CHGM_TRIL), "chgm spl2"),
    ("nion over the table", lambda p: setattr(p, "nion", 9), "ion species"),
    ("negative nion", lambda p: setattr(p, "nion", -1), "ion species"),
])
def test_energy_noalloc_rejects_bad_arguments(what, edit, msg):
    """pmgb_energy_noalloc checks its arguments before any CUDA call, so the
    rejections run on a machine without a GPU (dummy device addresses are
    never touched)."""
    _, p = synth.config0()
    edit(p)
    with pytest.raises(vpmg.PmgbError, match=msg):
        vpmg.energy_noalloc(p, 0x1000, 0x2000, 0x3000, 0x4000, 0x5000, 0x6000)


@pytest.mark.skipif(not os.path.exists(vpmg.LIB_PATH), reason="library not built")
def test_energy_noalloc_rejects_npbe_without_maps():
    m = synth.cluster(50, 5.0, seed=1)
    p = synth.mg_manual(33, 0.6, m.center(), npbe=True)
    with pytest.raises(vpmg.PmgbError, match="NPBE needs"):
        vpmg.energy_noalloc(p, 0x1000, 0x2000)
