"""Generate the golden fixtures under tests/golden/ from the reference tree.

Run here, where the reference checkout is readable:
    python tests/golden/make_golden.py [/path/to/chiralHeisenberg]

Writes:
  remez2, remez4, remez2g  -- the rational-approximation data files the
                              reference program reads (rhmc/remez*; format
                              a0, (a_k, sigma_k)*n, b0, (b_k, sigma_k)*n);
  con_12x12x12.bin         -- rhmc/_con: one Fortran unformatted record,
                              chi(1728,3) real*8 + seed real*8;
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
