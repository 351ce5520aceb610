"""Generate the rational-approximation files of the multi-pseudofermion
variant (chdwf_prog_set_ext) with chiralheisenberg_b200.remez.

    python chiralheisenberg_b200/data/make_remez.py

Writes, in the layout of the reference's remez files (a0; n lines
'a_k, sigma_k'; b0; n lines 'b_k, sigma_k'; read as rhmc/cheisdwf.f:140-159):
  remez4_20  a ~ x^(1/4),  b ~ x^(-1/4)   20 poles
  remez8_20  a ~ x^(1/8),  b ~ x^(-1/8)   20 poles
on [1e-4, 50], the spectral range of the reference's own sets (their
relative error equioscillates on that interval).  With two pseudofermion
fields the heatbath takes remez8_20's a-set and the action and force take
remez4_20's b-set.  Each approximation is the minimax one in relative error;
its level is printed.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from chiralheisenberg_b200.remez import remez, write_remez_file  # noqa: E402

LO, HI, N = 1e-4, 50.0, 20


def main():
    for name, power in (("remez4_20", "1/4"), ("remez8_20", "1/8")):
        r, rinv = remez(power, LO, HI, N, digits=120)
        write_remez_file(os.path.join(HERE, name), r, rinv)
        print(f"{name}: x^{power} on [{LO}, {HI}], {N} poles, relative error {r.error:.4e}",
              flush=True)


if __name__ == "__main__":
    main()
