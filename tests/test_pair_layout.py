"""Index identities behind the pair sweep kernels (gs7_pairs.cuh, gs7_bulk.cuh),
checked on the host for the PMG grid shapes.

On a grid with odd nx and ny the flat index (k*ny + j)*nx + i has the parity
of i + j + k, so the aligned pair (2m, 2m+1) holds one point of each colour
of the red-black sweep (src/pmgc/gsd.c:95-164).  In row (j, k) with
s = (j + k) & 1, pair q covers i = 2q - s and 2q - s + 1; the neighbour of
element e in the next row or plane is element 1 - e of pair q - s + e; and the
pair rows jb .. jb+n-1 of one plane form one contiguous range whose pair
offsets are ((r*nx - s_r + s_0) >> 1) + q.
"""
import numpy as np
import pytest

SHAPES = [(33, 33, 33), (65, 65, 65), (161, 161, 161), (225, 225, 225), (17, 9, 33)]


def pair_base(nx, ny, j, k, q):
    return (k * ny + j) * nx + 2 * q - ((j + k) & 1)


@pytest.mark.parametrize("nx,ny,nz", SHAPES)
def test_flat_parity_is_colour(nx, ny, nz):
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    flat = (k * ny + j) * nx + i
    assert np.array_equal(flat & 1, (i + j + k) & 1)


@pytest.mark.parametrize("nx,ny,nz", SHAPES)
def test_pairs_cover_each_row_once(nx, ny, nz):
    w = (nx + 1) // 2
    for k in (0, 1, nz // 2, nz - 1):
        for j in range(ny):
            s = (j + k) & 1
            i = np.concatenate([2 * np.arange(w) - s, 2 * np.arange(w) - s + 1])
            inrow = np.sort(i[(i >= 0) & (i < nx)])
            assert np.array_equal(inrow, np.arange(nx))
            b = pair_base(nx, ny, j, k, 0)
            assert b % 2 == 0 and b >= 0


@pytest.mark.parametrize("nx,ny,nz", SHAPES)
def test_neighbour_pair_formula(nx, ny, nz):
    w = (nx + 1) // 2
    rng = np.random.default_rng(1)
    for _ in range(2000):
        j, k = int(rng.integers(1, ny - 2)), int(rng.integers(1, nz - 2))
        q, e = int(rng.integers(0, w)), int(rng.integers(0, 2))
        s = (j + k) & 1
        i = 2 * q - s + e
        if not 1 <= i <= nx - 2:
            continue
        flat = (k * ny + j) * nx + i
        qn = q - s + e
        assert 0 <= qn < w
        for dj, dk in ((1, 0), (-1, 0), (0, 1), (0, -1)):
            nb = pair_base(nx, ny, j + dj, k + dk, qn) + (1 - e)
            assert nb == flat + dj * nx + dk * nx * ny


@pytest.mark.parametrize("nx,ny,nz", SHAPES)
def test_cta_rows_are_one_contiguous_range(nx, ny, nz):
    w = (nx + 1) // 2
    for nrow in (3, 6, 8):
        sp = ((nrow - 1) * nx + 1) // 2 + w
        for k in (0, 1, nz - 2):
            for jb in range(0, ny - nrow + 1, max(1, nrow - 2)):
                start = pair_base(nx, ny, jb, k, 0)
                covered = []
                for r in range(nrow):
                    for q in range(w):
                        off = ((r * nx - ((jb + r + k) & 1) + ((jb + k) & 1)) >> 1) + q
                        assert start + 2 * off == pair_base(nx, ny, jb + r, k, q)
                        assert 0 <= off < sp
                        covered.append(off)
                # no gaps between rows: the copied range is exactly the pairs used
                assert max(covered) - min(covered) + 1 <= len(set(covered)) + nrow
