"""The Vpmg_solve drop-in (apbs_b200/dropin/vpmg_b200.c), linked with the
reference's own objects as APBS would link it (oracle/Makefile, target
dropin).  CPU side: the library exports the Vpmg entry points with the
binding's definitions, and without a GPU the unchanged reference sequence
fails loudly at Vpmg_solve instead of solving on the CPU."""
import ctypes
import os
import subprocess

import pytest

from apbs_b200 import synth
from oracle import ref

pytestmark = pytest.mark.skipif(not ref.dropin_available(), reason="drop-in not built")


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_dropin_exports_the_vpmg_entry_points():
    L = ctypes.CDLL(ref.DROPIN_PATH)
    for name in ("Vpmg_ctor", "Vpmg_ctor2", "Vpmg_dtor", "Vpmg_dtor2", "Vpmg_fillco",
                 "Vpmg_solve", "Vpmg_energy", "Vpmg_setPart", "Vpmg_qfEnergy"):
        assert hasattr(L, name), name
    # the reference's own definitions are still there under the _host names
    for name in ("Vpmg_solve_host", "Vpmg_ctor_host", "Vpmg_dtor_host"):
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", ref.DROPIN_PATH], capture_output=True,
                         text=True).stdout
    assert " T Vpmg_solve\n" in out


@pytest.mark.skipif(_have_gpu(), reason="a GPU is present")
def test_dropin_fails_loudly_without_a_device():
    m, p = synth.config0()
    with pytest.raises(RuntimeError):
        ref.run(p, m, dropin=True)
