"""CPU model of the row-staged kernels' copy schedule (csrc/row_stage.cuh).

The kernels' producer (thread 0 issuing bulk copies of window rows into a
ring of slots, and of the t+-1 rows into a second ring) and consumer (every
thread waiting for window rows u, u+1, u+2 and t entry k of its k-th output
row) are restated here line by line, and for many lattice shapes and grid
sizes the model checks what the GPU code relies on:
  * output row (f, t, y) reads window rows (f, t, y-1), (f, t, y), (f, t, y+1)
    with y periodic, and t rows (f, t+1, y), (f, t-1, y) with t periodic;
  * a slot of either ring is refilled only after every output row that
    reads it is done, so each slot has at most one copy in flight (its wait
    parity is unambiguous);
  * every wait is on a copy already issued, and every issued copy is waited
    on before the block ends (no copy in flight at exit);
  * every copy is in bounds and starts on a 16-byte boundary.
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
    for b in range(nb):
        rho0, rho1 = b * nrows // nb, (b + 1) * nrows // nb
        if rho0 >= rho1:
            continue

        def run_len(ra):
            return min((ra // L + 1) * L, rho1) - ra

        st = {"rho_a": rho0, "o": 0, "issued": 0, "len": run_len(rho0)}
        slots, loads, done = {}, [], set()

        def issue():
            run = st["rho_a"] // L
            f, t = run // Lt, run % Lt
            y = (st["rho_a"] - run * L - 1 + st["o"]) % L
            w = st["issued"]
            if w % NS in slots:
                assert slots[w % NS] in done, ("slot refilled before use ended", w)
            slots[w % NS] = w
            for d in range(4):
                off = cs * (4 * f + d) + Lrow * (y + L * t)
                assert 0 <= off and off + Lrow <= kferm
                assert (off * elem) % 16 == 0
            loads.append((f, t, y))
            st["issued"] += 1
            st["o"] += 1
            if st["o"] == st["len"] + 2:
                st["rho_a"] += st["len"]
                st["o"] = 0
                if st["rho_a"] < rho1:
                    st["len"] = run_len(st["rho_a"])

        nk = rho1 - rho0
        tslots, tloads = {}, []

        def issue_t():
            k = len(tloads)
            if k % NT in tslots:
                assert tslots[k % NT] in tdone, ("t slot refilled before use ended", k)
            tslots[k % NT] = k
            rho = rho0 + k
            run = rho // L
            f, t, y = run // Lt, run % Lt, rho - run * L
            for tt in ((t + 1) % Lt, (t - 1) % Lt):
                for d in range(4):
                    off = cs * (4 * f + d) + Lrow * (y + L * tt)
                    assert 0 <= off and off + Lrow <= kferm
                    assert (off * elem) % 16 == 0
            tloads.append((f, (t + 1) % Lt, (t - 1) % Lt, y))

        tdone = set()
        while st["issued"] < 3 and st["rho_a"] < rho1:
            issue()
        issue_t()
        while st["issued"] < NS and st["rho_a"] < rho1:
            issue()
        while len(tloads) < NT and len(tloads) < nk:
            issue_t()
        u, run_prev = 0, rho0 // L
        for k, rho in enumerate(range(rho0, rho1)):
            run = rho // L
            if run != run_prev:
                u += 2
                run_prev = run
            f, t, y = run // Lt, run % Lt, rho - run * L
            for w in range(3):
                assert u + w < st["issued"] and slots[(u + w) % NS] == u + w
            assert k < len(tloads) and tslots[k % NT] == k
            assert loads[u] == (f, t, (y - 1) % L)
            assert loads[u + 1] == (f, t, y)
            assert loads[u + 2] == (f, t, (y + 1) % L)
            assert tloads[k] == (f, (t + 1) % Lt, (t - 1) % Lt, y)
            u += 1
            next_u = u + 2 if (rho + 1 < rho1 and (rho + 1) // L != run) else u
            done.update(range(next_u))
            tdone.add(k)
            while st["rho_a"] < rho1 and st["issued"] < next_u + NS:
                issue()
            while len(tloads) < nk and len(tloads) < k + 1 + NT:
                issue_t()
        assert st["issued"] <= u + 2   # all issued copies were waited on
        assert len(tloads) == nk


SHAPES = [(24, 24, 24), (16, 16, 16), (16, 16, 32), (12, 12, 8), (8, 8, 8), (4, 4, 4),
          (3, 5, 2), (6, 4, 7), (24, 24, 16), (32, 32, 16), (2, 2, 4), (5, 3, 8), (6, 6, 5)]


@pytest.mark.parametrize("L,Lt,Ls", SHAPES)
def test_row_schedule(L, Lt, Ls):
    nrows = 2 * Lt * L
    for elem in (16, 8, 4):
        if (L * Ls * elem) % 16:
            continue
        for nb in sorted({1, 2, 3, 7, 148, 296, max(1, nrows // 3), nrows}):
            if 1 <= nb <= nrows:
                simulate(L, Lt, Ls, nb, elem)
