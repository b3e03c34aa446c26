"""Host model of the bulk-staged single-pass red-black sweep
(apbs_b200/csrc/gs7_rb_bulk.cuh): its stage schedule, ring slots, window
offsets, copy ranges and barrier phases, run CTA by CTA on small grids and
checked before any of it runs on a GPU:

* every bulk copy starts on a 16-byte boundary, has a length that is a
  multiple of 16 bytes and lies inside its array; every guarded load is
  bounds-checked as in the kernel;
* every shared-memory read lies inside its window and hits a slot that holds
  the plane it is meant to hold, filled by a stage the CTA has already
  waited for; no slot is refilled while a later step still reads it;
* at most P + 1 stages are in flight, and a barrier is re-armed only after
  its previous phase was waited for;
* the results equal the two colour passes of Vgsrb7x (src/pmgc/gsd.c:95-164)
  bit for bit, and every interior point is written by exactly one CTA;
* the launch shape the host picks fits the shared memory for the benchmark
  grids in FP32 and, up to 161^3, in FP64.
"""
import numpy as np
import pytest

from test_rb_layout import colour_passes, operator

P = 2
NC, NU, NX, NB = P + 2, P + 3, P + 3, P + 1
SMEM_MAX = 220 * 1024


def smem_bytes(Lw, E, tsize):
    return 64 + (4 * NC + NU + NX) * Lw * tsize + 3 * E * tsize


def shape(nx, S, nz, sms, tsize, smem_max=SMEM_MAX):
    """gs7_bulk_shape: (core, kchunk, Lw, E, nranges, nchunks, smem)."""
    AL = 16 // tsize
    best, best_cost = None, None
    for nr in range(1, 4097):
        core = (S + nr - 1) // nr
        core = (core + 1) & ~1
        Lw = ((core + 4 * nx + 6 + 2 * AL + AL - 1) // AL) * AL
        E = core // 2 + nx + 3
        sm = smem_bytes(Lw, E, tsize)
        if sm <= smem_max and (nr - 1) * core < S:
            planes = nz - 2
            nc = max(1, sms // nr)
            nc = min(nc, planes)
            kchunk = (planes + nc - 1) // nc
            nc = (planes + kchunk - 1) // kchunk
            waves = (nr * nc + sms - 1) // sms
            cost = waves * (kchunk + 2) * Lw
            if best is None or cost < best_cost:
                best, best_cost = (core, kchunk, Lw, E, nr, nc, sm), cost
        if core <= 2 * (nx + 2):
            break
    return best


def model(nx, ny, nz, c1, arrays, tsize, core, kchunk):
    """The kernel for one launch, with the checks of the module docstring."""
    oE, oN, uC, D, f, xin = arrays
    S = nx * ny
    ntot = S * nz
    AL = 16 // tsize
    E = core // 2 + nx + 3
    Lw = ((core + 4 * nx + 6 + 2 * AL + AL - 1) // AL) * AL
    C2 = 1 - c1
    xout = np.zeros(ntot)
    writes = np.zeros(ntot, dtype=int)
    nrange = (S + core - 1) // core
    nchunk = (nz - 2 + kchunk - 1) // kchunk
    coef = (oE, oN, D, f)

    for bx in range(nrange):
        for by in range(nchunk):
            c0 = bx * core
            c1e = min(c0 + core, S)
            k0 = 1 + by * kchunk
            k1 = min(k0 + kchunk, nz - 1)
            t0 = k0 - 1

            def off(q):
                v = q * S + c0 - 2 * nx - 2
                al = (v // AL) * AL  # floor also for negative v
                return al - q * S

            # slot contents: (plane, stage) per ring slot; data per slot
            cslots = [[None] * 4 for _ in range(NC)]
            cdata = np.full((NC, 4, Lw), np.nan)
            uslots, udata = [None] * NU, np.full((NU, Lw), np.nan)
            xslots, xdata = [None] * NX, np.full((NX, Lw), np.nan)
            waited = set()
            issued = []
            bar_uses = [0] * NB       # arms so far
            bar_waited = [0] * NB     # phases waited so far
            live_reads = {}           # (ring, slot) -> last step that reads it

            def fill(src, g0, dst):
                bulk = g0 >= 0 and g0 + Lw <= ntot
                if bulk:
                    assert (g0 * tsize) % 16 == 0 and (Lw * tsize) % 16 == 0
                    dst[:] = src[g0:g0 + Lw]
                else:
                    for e in range(Lw):
                        g = g0 + e
                        dst[e] = src[g] if 0 <= g < ntot else 0.0

            def issue(j, step):
                u = j - (t0 - 2)
                b = u % NB
                assert bar_uses[b] == bar_waited[b], "barrier re-armed before its wait"
                bar_uses[b] += 1
                assert len([s for s in issued if s not in waited]) < NB
                issued.append(j)
                has_c = j >= t0 and 0 <= j <= nz - 1
                has_u = j >= t0 - 1 and 0 <= j <= nz - 1
                has_x = j + 1 >= t0 - 1 and 0 <= j + 1 <= nz - 1
                gj, gx = j * S + off(j), (j + 1) * S + off(j + 1)
                for ring, ok, slot in (("c", has_c, j % NC), ("u", has_u, j % NU),
                                       ("x", has_x, (j + 1) % NX)):
                    if ok:
                        last = live_reads.get((ring, slot), -10)
                        assert last < step, (ring, slot, last, step)
                if has_c:
                    for a in range(4):
                        fill(coef[a], gj, cdata[j % NC, a])
                        cslots[j % NC][a] = (j, j)
                if has_u:
                    fill(uC, gj, udata[j % NU])
                    uslots[j % NU] = (j, j)
                if has_x:
                    fill(xin, gx, xdata[(j + 1) % NX])
                    xslots[(j + 1) % NX] = (j + 1, j)

            def wait(j):
                u = j - (t0 - 2)
                b = u % NB
                assert bar_waited[b] < bar_uses[b]
                assert (bar_waited[b] & 1) == ((u // NB) & 1)
                bar_waited[b] += 1
                waited.add(j)

            def read(ring, q, l, step):
                assert 0 <= l < Lw, (ring, q, l, Lw)
                if ring == "x":
                    slot = q % NX
                    plane, stage = xslots[slot]
                    val = xdata[slot, l]
                elif ring == "u":
                    slot = q % NU
                    plane, stage = uslots[slot]
                    val = udata[slot, l]
                else:
                    slot = q % NC
                    plane, stage = cslots[slot][ring]
                    val = cdata[slot, ring, l]
                assert plane == q and stage in waited, (ring, q, plane, stage)
                key = ("c" if isinstance(ring, int) else ring, slot)
                live_reads[key] = max(live_reads.get(key, -10), step)
                return val

            R = np.full((3, E), np.nan)
            rplane = [None] * 3

            def base(k):
                return (k * S + c0 - nx - 1) >> 1

            issue(t0 - 2, t0 - 1)
            issue(t0 - 1, t0 - 1)
            wait(t0 - 2)
            wait(t0 - 1)
            for j in range(t0, min(t0 + P, k1 + 1)):
                issue(j, t0 - 1)
            dW, dE = (C2 - c1 - 1) // 2, (C2 - c1 + 1) // 2
            dS, dN = (C2 - c1 - nx) // 2, (C2 - c1 + nx) // 2
            for t in range(t0, k1 + 1):
                if t + P <= k1:
                    issue(t + P, t)
                wait(t)
                m0 = base(t)
                if t == 0 or t == nz - 1:
                    R[t % 3, :] = 0.0
                else:
                    o0, om, op = off(t), off(t - 1), off(t + 1)
                    for e in range(E):
                        ip = 2 * (m0 + e) + c1 - t * S
                        v = 0.0
                        if 0 <= ip < S:
                            l, lm, lp = ip - o0, ip - om, ip - op
                            v = (read(3, t, l, t) + read(1, t, l, t) * read("x", t, l + nx, t) +
                                 read(1, t, l - nx, t) * read("x", t, l - nx, t) +
                                 read(0, t, l, t) * read("x", t, l + 1, t) +
                                 read(0, t, l - 1, t) * read("x", t, l - 1, t) +
                                 read("u", t - 1, lm, t) * read("x", t - 1, lm, t) +
                                 read("u", t, l, t) * read("x", t + 1, lp, t)) / read(2, t, l, t)
                        R[t % 3, e] = v
                rplane[t % 3] = t
                k = t - 1
                if k < k0:
                    continue

                def ring_r(q, e):
                    assert 0 <= e < E and rplane[q % 3] == q
                    return R[q % 3, e]

                m0 = base(k)
                dD = m0 + (C2 - c1 - S) // 2 - base(k - 1)
                dU = m0 + (C2 - c1 + S) // 2 - base(k + 1)
                lo, hi = k * S + c0, k * S + c1e
                o0, om = off(k), off(k - 1)
                for e in range(E):
                    m = m0 + e
                    p2, p1 = 2 * m + C2, 2 * m + c1
                    in2, in1 = lo <= p2 < hi, lo <= p1 < hi
                    if not in1 and not in2:
                        continue
                    v1 = ring_r(k, e)
                    if in2:
                        l, lm = p2 - k * S - o0, p2 - k * S - om
                        v2 = (read(3, k, l, t) + read(1, k, l, t) * ring_r(k, e + dN) +
                              read(1, k, l - nx, t) * ring_r(k, e + dS) +
                              read(0, k, l, t) * ring_r(k, e + dE) +
                              read(0, k, l - 1, t) * ring_r(k, e + dW) +
                              read("u", k - 1, lm, t) * ring_r(k - 1, e + dD) +
                              read("u", k, l, t) * ring_r(k + 1, e + dU)) / read(2, k, l, t)
                        xout[p2] = v2
                        writes[p2] += 1
                    if in1:
                        xout[p1] = v1
                        writes[p1] += 1
            assert set(issued) == waited  # nothing left in flight at exit
    return xout, writes


SHAPES = [(9, 7, 5), (17, 9, 11), (33, 33, 9), (13, 21, 7), (21, 15, 13)]


@pytest.mark.parametrize("nx,ny,nz", SHAPES)
@pytest.mark.parametrize("core,kchunk", [(2, 1), (6, 2), (40, 3), (128, 5), (1000, 4)])
@pytest.mark.parametrize("c1", [0, 1])
@pytest.mark.parametrize("tsize", [4, 8])
def test_bulk_model_equals_colour_passes(nx, ny, nz, core, kchunk, c1, tsize):
    S = nx * ny
    core = min(core, (S + 1) & ~1)
    oE, oN, uC, D, f, x, inner = operator(nx, ny, nz, nx * 3 + ny + core + kchunk)
    want = colour_passes(nx, ny, nz, c1, oE, oN, uC, D, f, x)
    got, writes = model(nx, ny, nz, c1, (oE, oN, uC, D, f, x), tsize, core, kchunk)
    assert np.array_equal(got, want)
    assert np.all(writes[inner] == 1)
    assert np.all(writes <= 1)


@pytest.mark.parametrize("n", [33, 65, 97, 129, 161, 225])
@pytest.mark.parametrize("tsize", [4, 8])
def test_launch_shape_fits(n, tsize):
    sh = shape(n, n * n, n, 148, tsize)
    if sh is None:
        # FP64 windows of the widest grids do not fit: the caller runs the
        # unstaged single-pass sweep instead
        assert tsize == 8 and n >= 225
        return
    core, kchunk, Lw, E, nr, nc, sm = sh
    assert sm <= SMEM_MAX and core % 2 == 0 and core >= 2
    assert (nr - 1) * core < n * n <= nr * core
    assert (nc - 1) * kchunk < n - 2 <= nc * kchunk
    assert nr <= 2 ** 31 - 1 and nc <= 65535
    # the window covers the widened range and its neighbours
    AL = 16 // tsize
    assert Lw >= core + 4 * n + 6 + AL and Lw % AL == 0
