"""CPU model of the row-staged kernels' copy schedule (csrc/row_stage.cuh).

The producer (lane 0 of the block's last warp, issuing bulk copies of
window rows into one ring of slots and of the t+-1 rows into a second ring,
each after its slot's previous use has been released) and the consumers
(waiting for window loads u, u+1, u+2 and t entry k of the block's k-th
output row, then releasing what the next row does not read) are restated
here, and for many lattice shapes and grid sizes the model checks what the
GPU code relies on:
  * output row (f, t, y) reads window rows (f, t, y-1), (f, t, y), (f, t, y+1)
    with y periodic, and t rows (f, t+1, y), (f, t-1, y) with t periodic;
  * a slot is refilled only after every consumer released its previous use,
    so each slot has at most one copy in flight and the wait parities
    (use count & 1) are unambiguous;
  * the producer never waits for a release the consumers cannot give
    (no deadlock), however far ahead it runs;
  * every copy is in bounds and starts on a 16-byte boundary, and the
    expect-tx byte counts stay below the mbarrier's limit (2^20 - 1).
"""
import pytest

NS = 5   # kRowSlots
NT = 3   # kRowTEnt


def simulate(L, Lt, Ls, nb, elem):
    Lrow = L * Ls
    nrows = 2 * Lt * L
    cs = L * L * Lt * Ls
    kferm = 8 * cs
    assert (Lrow * elem) % 16 == 0
    assert 8 * Lrow * elem < 2 ** 20
    for b in range(nb):
        rho0, rho1 = b * nrows // nb, (b + 1) * nrows // nb
        nk = rho1 - rho0
        if nk <= 0:
            continue

        def rows_of(k):
            rho = rho0 + k
            run = rho // L
            return run // Lt, run % Lt, rho - run * L

        # the window base of every step, as both sides compute it
        u = [0] * nk
        for k in range(1, nk):
            u[k] = u[k - 1] + 1 + (2 if rows_of(k)[2] == 0 else 0)

        # producer state
        pr = {"ra": rho0, "o": 0, "len": min((rho0 // L + 1) * L, rho1) - rho0,
              "issued": 0, "tissued": 0, "k": 0}
        loads, tloads = [], []
        released_y, released_t = set(), set()
        slot_y, slot_t = {}, {}

        def producer_step():
            """Issue the next copy if its slot is free; False when blocked or done."""
            k = pr["k"]
            if k >= nk:
                return False
            if pr["issued"] <= u[k] + 2:
                w = pr["issued"]
                if w >= NS and (w - NS) not in released_y:
                    return False
                if w % NS in slot_y:
                    assert slot_y[w % NS] == w - NS
                slot_y[w % NS] = w
                ra, o = pr["ra"], pr["o"]
                run = ra // L
                f, t = run // Lt, run % Lt
                y = (ra - run * L - 1 + o) % L
                for d in range(4):
                    off = cs * (4 * f + d) + Lrow * (y + L * t)
                    assert 0 <= off and off + Lrow <= kferm
                    assert (off * elem) % 16 == 0
                loads.append((f, t, y))
                pr["issued"] += 1
                pr["o"] += 1
                if pr["o"] == pr["len"] + 2:
                    pr["ra"] += pr["len"]
                    pr["o"] = 0
                    if pr["ra"] < rho1:
                        pr["len"] = min((pr["ra"] // L + 1) * L, rho1) - pr["ra"]
                return True
            if k >= NT and (k - NT) not in released_t:
                return False
            slot_t[k % NT] = k
            f, t, y = rows_of(k)
            for tt in ((t + 1) % Lt, (t - 1) % Lt):
                for d in range(4):
                    off = cs * (4 * f + d) + Lrow * (y + L * tt)
                    assert 0 <= off and off + Lrow <= kferm
                    assert (off * elem) % 16 == 0
            tloads.append((f, (t + 1) % Lt, (t - 1) % Lt, y))
            pr["tissued"] += 1
            pr["k"] += 1
            return True

        for k in range(nk):
            # the producer runs as far ahead as its slots allow
            while producer_step():
                pass
            f, t, y = rows_of(k)
            w0 = u[k]
            assert w0 + 2 < pr["issued"] and k < pr["tissued"], ("consumer would wait forever", k)
            for w in range(w0, w0 + 3):
                assert slot_y[w % NS] == w
            assert slot_t[k % NT] == k
            assert loads[w0] == (f, t, (y - 1) % L)
            assert loads[w0 + 1] == (f, t, y)
            assert loads[w0 + 2] == (f, t, (y + 1) % L)
            assert tloads[k] == (f, (t + 1) % Lt, (t - 1) % Lt, y)
            if k + 1 < nk:
                nrel = 3 if (y + 1) == L else 1
                assert u[k + 1] == w0 + nrel
                released_y.update(range(w0, w0 + nrel))
            released_t.add(k)
        while producer_step():
            pass
        assert pr["k"] == nk and pr["issued"] == u[nk - 1] + 3


SHAPES = [(24, 24, 24), (16, 16, 16), (16, 16, 32), (12, 12, 8), (8, 8, 8), (4, 4, 4),
          (3, 5, 2), (6, 4, 7), (24, 24, 16), (32, 32, 16), (2, 2, 4), (5, 3, 8), (6, 6, 5),
          (1, 3, 4), (4, 1, 4)]


@pytest.mark.parametrize("L,Lt,Ls", SHAPES)
def test_row_schedule(L, Lt, Ls):
    nrows = 2 * Lt * L
    for elem in (16, 8, 4):
        if (L * Ls * elem) % 16:
            continue
        for nb in sorted({1, 2, 3, 7, 148, 296, max(1, nrows // 3), nrows}):
            if 1 <= nb <= nrows:
                simulate(L, Lt, Ls, nb, elem)
