"""OpenDX output (pmgb_write_dx_host) against the reference's Vgrid_writeDX
compiled from source: byte-for-byte equal files, with and without partition
weights, on values that exercise the "%12.6e" rounding (ties, tiny and huge
exponents, signed zeros).  Host-only: no GPU is needed."""
import ctypes

import numpy as np
import pytest

from apbs_b200 import vpmg
from oracle import ref

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")

PACKAGE = b"APBS 3.4.1 (reference oracle build)"


def _ours(path, data, h, origin, pvec=None, title=b"POTENTIAL (kT/e)"):
    L = vpmg.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    L.pmgb_write_dx_host.restype = ctypes.c_int
    L.pmgb_write_dx_host.argtypes = [ctypes.c_char_p] + [ctypes.c_int] * 3 + \
        [ctypes.c_double] * 6 + [dp, dp, ctypes.c_char_p, ctypes.c_char_p]
    d = np.ascontiguousarray(data, dtype=np.float64)
    nz, ny, nx = d.shape
    pv = None if pvec is None else np.ascontiguousarray(pvec, dtype=np.float64)
    rc = L.pmgb_write_dx_host(str(path).encode(), nx, ny, nz, h[0], h[1], h[2], *origin,
                              d.ctypes.data_as(dp),
                              None if pv is None else pv.ctypes.data_as(dp), title, PACKAGE)
    assert rc == 1, vpmg.last_error()


def _values(shape, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(shape) * 10.0 ** rng.integers(-12, 12, size=shape)
    flat = v.reshape(-1)
    special = [0.0, -0.0, 1.0, -1.0, 1.2345675, 9.9999995, 9.9999994999, 1e-300, -1e300,
               2.5e-7, 123456.5, 0.5, 1.0000005, 5e-324]
    flat[: len(special)] = special
    return v


@pytest.mark.parametrize("shape", [(5, 7, 9), (33, 17, 11), (4, 4, 4)])
def test_dx_file_matches_reference(tmp_path, shape):
    data = _values(shape, sum(shape))
    h, origin = (0.5, 0.4, 0.45), (-12.25, 3.5, -0.125)
    _ours(tmp_path / "ours.dx", data, h, origin)
    ref.write_dx(tmp_path / "ref.dx", data, h, origin)
    assert (tmp_path / "ours.dx").read_bytes() == (tmp_path / "ref.dx").read_bytes()


def test_dx_partition_subset_matches_reference(tmp_path):
    shape = (13, 11, 9)
    data = _values(shape, 5)
    nz, ny, nx = shape
    wx = np.zeros(nx); wx[2:7] = 1.0; wx[2] = 0.5
    wy = np.zeros(ny); wy[1:9] = 1.0
    wz = np.ones(nz); wz[-1] = 0.0
    pvec = wz[:, None, None] * wy[None, :, None] * wx[None, None, :]
    h, origin = (0.6, 0.6, 0.6), (1.0, 2.0, 3.0)
    _ours(tmp_path / "ours.dx", data, h, origin, pvec)
    ref.write_dx(tmp_path / "ref.dx", data, h, origin, pvec)
    assert (tmp_path / "ours.dx").read_bytes() == (tmp_path / "ref.dx").read_bytes()


def test_dx_read_round_trip(tmp_path):
    """The reader returns the values the writer printed (six digits), the
    grid counts, spacings and origin."""
    data = _values((6, 5, 7), 3)
    h, origin = (0.5, 0.25, 0.75), (-3.0, 1.5, 2.25)
    vpmg.write_dx(tmp_path / "m.dx", data, h, origin, title="KAPPA MAP")
    got, gh, go = vpmg.read_dx(tmp_path / "m.dx")
    assert got.shape == data.shape
    printed = np.array([float("%12.6e" % v) for v in data.reshape(-1)]).reshape(data.shape)
    assert np.array_equal(got, printed)
    assert np.allclose(gh, h) and np.allclose(go, origin)
