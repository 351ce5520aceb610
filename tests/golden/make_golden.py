"""Generate the golden fixtures under tests/golden/ from the reference tree.

Run here, where the reference checkout is readable:
    python tests/golden/make_golden.py [/path/to/chiralHeisenberg]

Writes:
  remez2, remez4, remez2g  -- the rational-approximation data files the
                              reference program reads (rhmc/remez*; format
                              a0, (a_k, sigma_k)*n, b0, (b_k, sigma_k)*n);
  con_12x12x12.bin         -- rhmc/_con: one Fortran unformatted record,
                              chi(1728,3) real*8 + seed real*8;
  con_sp_12x12x12.bin      -- rhmc/Ls_8/b_0.45/_con: a configuration of the
                              older single-precision format (chi REAL*4,
                              seed REAL*8), the input of rhmc/sp_to_dp.f;
  list_directed.json       -- the first 60 records of fort.11-14 (kept as
                              action, conds, suscs, condmod) of every
                              rhmc/Ls_8 run: list-directed output written by
                              the reference's gfortran build;
  out_1_b0.45.txt          -- rhmc/Ls_8/b_0.45/out_1, the 'output' file of
                              two runs (explicit formats 9001-9024);
  seed_pins.json           -- (seed read from 'con', seed after start-up)
                              pairs printed by the reference into
                              rhmc/Ls_8/<run>/out_1.  Between the two prints
                              the program makes exactly one start-up call of
                              rano (cheisdwf.f:125-130,:160-161), i.e. 196
                              RRANF draws, so each pair is a known-answer
                              test of the generator.
The GPU tests never read the reference tree; they read these files.
"""
import json
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    rhmc = os.path.join(ref_root, "rhmc")
    for name in ("remez2", "remez4", "remez2g"):
        shutil.copyfile(os.path.join(rhmc, name), os.path.join(HERE, name))
    shutil.copyfile(os.path.join(rhmc, "_con"), os.path.join(HERE, "con_12x12x12.bin"))
    shutil.copyfile(os.path.join(rhmc, "Ls_8", "b_0.45", "_con"),
                    os.path.join(HERE, "con_sp_12x12x12.bin"))
    shutil.copyfile(os.path.join(rhmc, "Ls_8", "b_0.45", "out_1"),
                    os.path.join(HERE, "out_1_b0.45.txt"))
    # write(11,*) isweep,gaction,paction; write(12,*) cond; write(13,*) susc;
    # write(14,*) condmod,susctot (cheisdwf.f:347, :387-389)
    kinds = {"action": "iff", "conds": "fff", "suscs": "fff", "condmod": "ff"}
    ld = []
    for run in sorted(os.listdir(os.path.join(rhmc, "Ls_8"))):
        for name, k in kinds.items():
            fn = os.path.join(rhmc, "Ls_8", run, name)
            if os.path.exists(fn):
                with open(fn) as f:
                    lines = [f.readline() for _ in range(60)]
                ld.append({"source": f"rhmc/Ls_8/{run}/{name}", "kinds": k,
                           "lines": [x for x in lines if x]})
    with open(os.path.join(HERE, "list_directed.json"), "w") as f:
        json.dump(ld, f, indent=0)
    pins = []
    runs_dir = os.path.join(rhmc, "Ls_8")
    for run in sorted(os.listdir(runs_dir)):
        out = os.path.join(runs_dir, run, "out_1")
        if not os.path.exists(out):
            continue
        lines = open(out).read().splitlines()
        seeds = []
        for ln, text in enumerate(lines, start=1):
            m = re.match(r"\s*seed:\s*([0-9.Ee+-]+)", text)
            if m:
                seeds.append((ln, float(m.group(1))))
            else:
                seeds.append((ln, None))
        # a start-up print is followed by the header block and then the
        # post-start-up print (the 'seed:' line right after 'Stopping residuals')
        for ln, text in enumerate(lines, start=1):
            if "Stopping residuals" in text and ln < len(lines):
                m_after = re.match(r"\s*seed:\s*([0-9.Ee+-]+)", lines[ln])
                # the last 'seed:' before the header is the value read from con
                before = [s for s in seeds[: ln - 1] if s[1] is not None]
                hdr = [i for i in range(ln - 1, -1, -1) if "ksize=" in lines[i]]
                if m_after and before and hdr:
                    b = [s for s in before if s[0] <= hdr[0]]
                    if b:
                        pins.append({"run": run, "seed_in": b[-1][1],
                                     "seed_after_startup": float(m_after.group(1)),
                                     "source": f"rhmc/Ls_8/{run}/out_1:{b[-1][0]},{ln + 1}"})
    with open(os.path.join(HERE, "seed_pins.json"), "w") as f:
        json.dump({"draws_between": 196, "pins": pins}, f, indent=1)
    print(f"wrote {len(pins)} seed pins")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
