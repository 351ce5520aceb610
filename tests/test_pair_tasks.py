"""CPU model of the FP32 two-point pass-1 task order (pair_tasks in
csrc/lanczos.cu): block b takes sites [b kvol / nb, (b+1) kvol / nb), runs
its wall pairs (s = 0 and s = Ls-2 of each site and flavour) first, padded
to whole warps, then its interior pairs.  The model checks, for many
lattices and grid sizes, that
  * every (even point, flavour) pair of the lattice is evaluated exactly once;
  * wall tasks are exactly the pairs holding a wall point, and run with the
    wall code; interior tasks hold neither wall and have both s neighbours;
  * every warp (32 consecutive task slots of a 256-thread block) is either
    all wall or all interior, so no warp runs both code paths;
  * the precomputed division by Ls/2 - 2 (Granlund-Montgomery, as
    make_fastdiv / fdiv) agrees with integer division on every numerator used.
"""
import pytest

THREADS = 256


def make_fastdiv(d):
    l = 0
    while (1 << l) < d:
        l += 1
    m = (((1 << 32) * ((1 << l) - d)) // d + 1) & 0xFFFFFFFF
    return m, l


def fdiv(n, fd):
    m, l = fd
    t = (n * m) >> 32
    return ((t + n) & 0xFFFFFFFF) >> l


def tasks_of_block(L, Lt, Ls, nb, b):
    kvol = L * L * Lt
    S0, S1 = b * kvol // nb, (b + 1) * kvol // nb
    ns = S1 - S0
    nwps = 1 if Ls == 2 else 2
    Pi = Ls // 2 - nwps
    nwf = ns * nwps
    nw = 2 * nwf
    nw32 = (nw + 31) & ~31
    nif = ns * Pi
    ntask = nw32 + 2 * nif
    dPi = make_fastdiv(Pi if Ls >= 6 else 1)
    out = []
    for t in range(ntask):
        if t < nw32:
            if t >= nw:
                out.append((t, None))
                continue
            f = 1 if t >= nwf else 0
            r = t - f * nwf
            site = S0 + ((r >> 1) if nwps == 2 else r)
            s = Ls - 2 if (nwps == 2 and (r & 1)) else 0
            out.append((t, (True, s + Ls * site, f)))
        else:
            v = t - nw32
            f = 1 if v >= nif else 0
            r = v - f * nif
            qd = fdiv(r, dPi)
            assert qd == r // Pi
            out.append((t, (False, 2 * (1 + r - qd * Pi) + Ls * (S0 + qd), f)))
    return out


SHAPES = [(24, 24, 24), (16, 16, 16), (12, 12, 8), (8, 8, 8), (6, 4, 6), (4, 6, 4),
          (8, 8, 2), (5, 3, 10), (32, 32, 16), (3, 5, 12)]


@pytest.mark.parametrize("L,Lt,Ls", SHAPES)
def test_pair_tasks_cover_the_lattice_once(L, Lt, Ls):
    kvol = L * L * Lt
    for nb in sorted({1, 3, 7, 148, 444, max(1, kvol // 5), kvol}):
        if nb > kvol:
            continue
        seen = {}
        for b in range(nb):
            tl = tasks_of_block(L, Lt, Ls, nb, b)
            for w0 in range(0, len(tl), 32):
                kinds = {x[1][0] for x in tl[w0:w0 + 32] if x[1] is not None}
                assert len(kinds) <= 1, ("warp with both code paths", L, Lt, Ls, nb, b, w0)
            for _, task in tl:
                if task is None:
                    continue
                wall, p, f = task
                s = p % Ls
                assert s % 2 == 0 and 0 <= p < kvol * Ls
                holds_wall = s == 0 or s + 1 == Ls - 1
                assert wall == holds_wall
                if not wall:
                    assert s >= 2 and s + 2 <= Ls - 2
                assert (p, f) not in seen
                seen[(p, f)] = True
        assert len(seen) == kvol * Ls  # (Ls/2 pairs) x 2 flavours per site
