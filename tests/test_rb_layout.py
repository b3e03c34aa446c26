"""Host model of the single-pass red-black sweep (apbs_b200/csrc/gs7_rb.cuh):
the same slot arithmetic, loop bounds and tests, run CTA by CTA on small
grids, checked three ways before any of it runs on a GPU:

* every flat index the kernel reads lies inside the arrays, and every ring
  slot it reads lies inside [0, E) and was written for that plane;
* the operator it is given has zero couplings and zero f on boundary points
  and D = 1 there (as the solver builds it), and the sweep then equals the
  two colour passes of Vgsrb7x (src/pmgc/gsd.c:95-164) exactly, boundary
  values included;
* every interior point is written by exactly one CTA (boundary points of
  interior planes may be written as 0 by the CTA whose range holds them).
"""
import numpy as np
import pytest

SHAPES = [(9, 7, 5), (17, 9, 11), (33, 33, 9), (13, 21, 7)]


def gs7_rb_core(nx, S, E):
    core = 2 * (E - nx - 3)
    if core < 2:
        return 0
    return ((S + 1) & ~1) if core > S else core


def model(nx, ny, nz, E, kchunk, c1, oE, oN, uC, D, f, xin):
    S = nx * ny
    N = S * nz
    core = gs7_rb_core(nx, S, E)
    assert core > 0
    xout = np.zeros(N)
    writes = np.zeros(N, dtype=int)
    nrange = (S + core - 1) // core
    nchunk = (nz - 2 + kchunk - 1) // kchunk
    C2 = 1 - c1

    def rd(a, p):
        assert 0 <= p < N, p
        return a[p]

    for bx in range(nrange):
        for by in range(nchunk):
            c0 = bx * core
            c1e = min(c0 + core, S)
            k0 = 1 + by * kchunk
            k1 = min(k0 + kchunk, nz - 1)
            R = np.full((3, E), np.nan)
            written = {}
            base = lambda k: (k * S + c0 - nx - 1) >> 1

            def phase_a(k):
                m0 = base(k)
                lo, hi = k * S, k * S + S
                bp = k == 0 or k == nz - 1
                for e in range(E):
                    p = 2 * (m0 + e) + c1
                    v = 0.0
                    if not bp and lo <= p < hi:
                        v = (rd(f, p) + rd(oN, p) * rd(xin, p + nx) +
                             rd(oN, p - nx) * rd(xin, p - nx) + rd(oE, p) * rd(xin, p + 1) +
                             rd(oE, p - 1) * rd(xin, p - 1) + rd(uC, p - S) * rd(xin, p - S) +
                             rd(uC, p) * rd(xin, p + S)) / rd(D, p)
                    R[k % 3, e] = v
                written[k % 3] = k

            phase_a(k0 - 1)
            phase_a(k0)
            dW, dE = (C2 - c1 - 1) // 2, (C2 - c1 + 1) // 2
            dS, dN = (C2 - c1 - nx) // 2, (C2 - c1 + nx) // 2
            for k in range(k0, k1):
                phase_a(k + 1)

                def ring(slot_plane, e):
                    assert 0 <= e < E, (e, E)
                    assert written[slot_plane % 3] == slot_plane
                    return R[slot_plane % 3, e]

                m0 = base(k)
                dD = m0 + (C2 - c1 - S) // 2 - base(k - 1)
                dU = m0 + (C2 - c1 + S) // 2 - base(k + 1)
                lo, hi = k * S + c0, k * S + c1e
                for e in range(E):
                    m = m0 + e
                    p2, p1 = 2 * m + C2, 2 * m + c1
                    in2, in1 = lo <= p2 < hi, lo <= p1 < hi
                    if not in1 and not in2:
                        continue
                    v1 = ring(k, e)
                    if in2:
                        v2 = (rd(f, p2) + rd(oN, p2) * ring(k, e + dN) +
                              rd(oN, p2 - nx) * ring(k, e + dS) + rd(oE, p2) * ring(k, e + dE) +
                              rd(oE, p2 - 1) * ring(k, e + dW) +
                              rd(uC, p2 - S) * ring(k - 1, e + dD) +
                              rd(uC, p2) * ring(k + 1, e + dU)) / rd(D, p2)
                        xout[p2] = v2
                        writes[p2] += 1
                    if in1:
                        xout[p1] = v1
                        writes[p1] += 1
    return xout, writes


def operator(nx, ny, nz, seed):
    """Random symmetric 7-point operator with the fine level's boundary
    structure: couplings to and from boundary points zero, f zero there,
    D = oC + cc inside and 1 on the boundary."""
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    inner = (i > 0) & (i < nx - 1) & (j > 0) & (j < ny - 1) & (k > 0) & (k < nz - 1)
    oE = np.where(inner & (i < nx - 2), rng.uniform(0.5, 1.5, inner.shape), 0.0)
    oN = np.where(inner & (j < ny - 2), rng.uniform(0.5, 1.5, inner.shape), 0.0)
    uC = np.where(inner & (k < nz - 2), rng.uniform(0.5, 1.5, inner.shape), 0.0)
    D = np.where(inner, rng.uniform(6.0, 9.0, inner.shape), 1.0)
    f = np.where(inner, rng.normal(size=inner.shape), 0.0)
    x = np.where(inner, rng.normal(size=inner.shape), 0.0)
    return [a.reshape(-1) for a in (oE, oN, uC, D, f, x)] + [inner.reshape(-1)]


def colour_passes(nx, ny, nz, c1, oE, oN, uC, D, f, x):
    x = x.copy()
    S = nx * ny
    for par in (c1, 1 - c1):
        for k in range(1, nz - 1):
            for j in range(1, ny - 1):
                for i in range(1, nx - 1):
                    if (i + j + k) & 1 != par:
                        continue
                    p = (k * ny + j) * nx + i
                    x[p] = (f[p] + oN[p] * x[p + nx] + oN[p - nx] * x[p - nx] +
                            oE[p] * x[p + 1] + oE[p - 1] * x[p - 1] + uC[p - S] * x[p - S] +
                            uC[p] * x[p + S]) / D[p]
    return x


@pytest.mark.parametrize("nx,ny,nz", SHAPES)
@pytest.mark.parametrize("E,kchunk", [(24, 1), (40, 2), (64, 3), (200, 4)])
@pytest.mark.parametrize("c1", [0, 1])
def test_model_equals_colour_passes(nx, ny, nz, E, kchunk, c1):
    S = nx * ny
    if gs7_rb_core(nx, S, E) == 0:
        pytest.skip("range narrower than the ring")
    oE, oN, uC, D, f, x, inner = operator(nx, ny, nz, nx * 7 + ny + E)
    want = colour_passes(nx, ny, nz, c1, oE, oN, uC, D, f, x)
    got, writes = model(nx, ny, nz, E, kchunk, c1, oE, oN, uC, D, f, x)
    assert np.array_equal(got, want)          # bitwise, boundary zeros included
    assert np.all(writes[inner] == 1)
    assert np.all(writes <= 1)


def test_flat_parity_is_colour():
    for nx, ny, nz in SHAPES + [(161, 161, 161)]:
        k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        assert np.array_equal((((k * ny + j) * nx + i) & 1), (i + j + k) & 1)
