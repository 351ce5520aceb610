"""Rational approximations for RHMC: the Remez exchange algorithm.

The reference reads its rational approximations from files made by an
external generator (bulk_rhmc.f:9-10 credits M.A. Clarke and A.D. Kennedy's
Remez code; rhmc/cheisdwf.f:140-159 reads remez2, remez4, remez2g).  This
module generates such sets: the minimax approximation of f(x) = x^(p/q) on
[lo, hi] in RELATIVE error by a rational function of type (n, n),

    r(x) = a0 + sum_k a_k / (x + sigma_k),   sigma_k > 0,

in the partial-fraction form the multi-shift solver consumes, together with
the same form of 1/r(x), the minimax approximation of x^(-p/q).

Method (the classical second Remez algorithm for rational functions, as
described by Clarke & Kennedy, "Accelerating dynamical fermion computations
using the rational hybrid Monte Carlo (RHMC) algorithm with multiple
pseudofermion fields", Phys. Rev. Lett. 98 (2007) 051601):
  1. On 2n+2 reference points x_i solve the nonlinear system
         P(x_i) - f(x_i) (1 + (-1)^i E) Q(x_i) = 0,   Q monic of degree n,
     for the 2n+1 coefficients of P and Q and the level E (Newton's method;
     the first solve interpolates with E = 0 on 2n+1 points).
  2. Locate the 2n+1 zeros of e(x) = r(x)/f(x) - 1 between consecutive
     reference points and the extremum of |e| in each of the 2n+2 intervals
     they bound; these become the new reference points.
  3. Repeat until the extrema are level: (max|e| - min|e|) / max|e| < tol.
     The iteration is continued in the width of the interval: it converges
     on [lo, lo*R] for a small R, then widens R step by step to hi/lo,
     carrying the reference points over at the same relative positions in
     log x (a direct start on a wide interval lets the first interpolant
     put poles inside the interval).
  4. Factor Q (its n roots are real and negative for x^(p/q), p/q in (-1, 1))
     and form the residues: a_k = P(-sigma_k) / Q'(-sigma_k), a0 = P's leading
     coefficient.  The same for 1/r with the roots of P.
Everything runs in decimal arithmetic with `digits` significant digits (the
monomial basis on [1e-4, 50] at degree 25 spans more than 100 orders of
magnitude), then the coefficients are rounded to double precision.
"""
from __future__ import annotations

import decimal
from decimal import Decimal as D
from fractions import Fraction
import math
from typing import List, Tuple

__all__ = ["remez", "RationalApprox", "write_remez_file", "read_remez_file"]


class RationalApprox:
    """a0 + sum a_k / (x + sigma_k), with the relative-error level it reaches."""

    def __init__(self, a0: float, a: List[float], sigma: List[float], error: float,
                 power: Fraction, lo: float, hi: float):
        self.a0, self.a, self.sigma = a0, list(a), list(sigma)
        self.error, self.power, self.lo, self.hi = error, power, lo, hi
        self.spread = None

    @property
    def n(self) -> int:
        return len(self.a)

    def __call__(self, x):
        import numpy as np
        x = np.asarray(x, dtype=np.float64)
        return self.a0 + sum(ak / (x + sk) for ak, sk in zip(self.a, self.sigma))

    def as_set(self):
        """(num[0..n], den[0..n-1]) as the solver takes them."""
        import numpy as np
        return (np.array([self.a0] + self.a, dtype=np.float64),
                np.array(self.sigma, dtype=np.float64))


def _horner(c: List[D], x: D) -> D:
    v = D(0)
    for ck in reversed(c):
        v = v * x + ck
    return v


def _solve(A: List[List[D]], b: List[D]) -> List[D]:
    """Gaussian elimination with partial pivoting in the current context."""
    n = len(b)
    M = [row[:] + [bi] for row, bi in zip(A, b)]
    for k in range(n):
        piv = max(range(k, n), key=lambda i: abs(M[i][k]))
        if M[piv][k] == 0:
            raise ArithmeticError("singular Remez system")
        M[k], M[piv] = M[piv], M[k]
        pk = M[k][k]
        for i in range(k + 1, n):
            fct = M[i][k] / pk
            if fct:
                Mi, Mk = M[i], M[k]
                for j in range(k, n + 1):
                    Mi[j] -= fct * Mk[j]
    x = [D(0)] * n
    for k in range(n - 1, -1, -1):
        s = M[k][n]
        for j in range(k + 1, n):
            s -= M[k][j] * x[j]
        x[k] = s / M[k][k]
    return x


class _Remez:
    def __init__(self, power: Fraction, lo: D, hi: D, n: int):
        self.power, self.lo, self.hi, self.n = power, lo, hi, n
        self.pw = D(power.numerator) / D(power.denominator)

    def f(self, x: D) -> D:
        return x ** self.pw

    def coeffs(self, z: List[D]):
        n = self.n
        return z[:n + 1], z[n + 1:2 * n + 1] + [D(1)]

    def err(self, p, q, x: D) -> D:
        return _horner(p, x) / (_horner(q, x) * self.f(x)) - 1

    def newton(self, xs: List[D], z: List[D], E: D, it_max=40):
        """Solve P(x_i) - f_i (1 + s_i E) Q(x_i) = 0 on 2n+2 points."""
        n = self.n
        fs = [self.f(x) for x in xs]
        pows = [[x ** j for j in range(n + 1)] for x in xs]
        tiny = D(10) ** (-(decimal.getcontext().prec - 20))
        for _ in range(it_max):
            p, q = self.coeffs(z)
            F, J = [], []
            for i in range(len(xs)):
                s = 1 if i % 2 == 0 else -1
                g = fs[i] * (1 + s * E)
                Qx = sum(q[j] * pows[i][j] for j in range(n + 1))
                Px = sum(p[j] * pows[i][j] for j in range(n + 1))
                F.append(Px - g * Qx)
                J.append([pows[i][j] for j in range(n + 1)] +
                         [-g * pows[i][j] for j in range(n)] + [-fs[i] * s * Qx])
            dz = _solve(J, [-v for v in F])
            z = [a + b for a, b in zip(z, dz[:2 * n + 1])]
            E = E + dz[2 * n + 1]
            scale = max(abs(v) for v in z) or D(1)
            if max(abs(v) for v in dz[:2 * n + 1]) <= scale * tiny:
                break
        return z, E

    def initial(self, xs: List[D]) -> List[D]:
        """Interpolation with E = 0 on the first 2n+1 points."""
        n = self.n
        A, b = [], []
        for x in xs[:2 * n + 1]:
            fx = self.f(x)
            A.append([x ** j for j in range(n + 1)] + [-fx * x ** j for j in range(n)])
            b.append(fx * x ** n)
        return _solve(A, b)

    def _zero(self, p, q, a: D, b: D, ea: D, iters=200) -> D:
        """A zero of e between a and b (e changes sign), bisection in log x."""
        la, lb = a.ln(), b.ln()
        for _ in range(iters):
            lm = (la + lb) / 2
            em = self.err(p, q, lm.exp())
            if (em > 0) == (ea > 0):
                la, ea = lm, em
            else:
                lb = lm
            if lb - la < D(10) ** -12:
                break
        return ((la + lb) / 2).exp()

    def _extremum(self, p, q, a: D, b: D, sign: int) -> Tuple[D, D]:
        """Point of max sign*e on [a, b]: golden section in log x after a scan."""
        la, lb = a.ln(), b.ln()
        m = 24
        grid = [la + (lb - la) * k / m for k in range(m + 1)]
        vals = [sign * self.err(p, q, g.exp()) for g in grid]
        bi = max(range(m + 1), key=lambda k: vals[k])
        lo_, hi_ = grid[max(bi - 1, 0)], grid[min(bi + 1, m)]
        gr = (D(5).sqrt() - 1) / 2
        c = hi_ - gr * (hi_ - lo_)
        d = lo_ + gr * (hi_ - lo_)
        fc = sign * self.err(p, q, c.exp())
        fd = sign * self.err(p, q, d.exp())
        for _ in range(80):
            if fc > fd:
                hi_, d, fd = d, c, fc
                c = hi_ - gr * (hi_ - lo_)
                fc = sign * self.err(p, q, c.exp())
            else:
                lo_, c, fc = c, d, fd
                d = lo_ + gr * (hi_ - lo_)
                fd = sign * self.err(p, q, d.exp())
            if hi_ - lo_ < D(10) ** -12:
                break
        xm = (lo_ + hi_) / 2
        vm = sign * self.err(p, q, xm.exp())
        for cand in (la, lb):          # an endpoint may be the extremum
            v = sign * self.err(p, q, cand.exp())
            if v > vm:
                xm, vm = cand, v
        return xm.exp(), vm

    def iterate(self, xs: List[D], z: List[D], E: D, tol: float, max_iter: int):
        """Exchange until the extrema of e on [lo, hi] are level."""
        N = 2 * self.n + 2
        spread = 1.0
        for _ in range(max_iter):
            z, E = self.newton(xs, z, E)
            p, q = self.coeffs(z)
            es = [self.err(p, q, x) for x in xs]
            zeros = [self._zero(p, q, xs[i], xs[i + 1], es[i]) for i in range(N - 1)]
            bounds = [self.lo] + zeros + [self.hi]
            new, mags = [], []
            for i in range(N):
                x, v = self._extremum(p, q, bounds[i], bounds[i + 1], 1 if es[i] > 0 else -1)
                new.append(x)
                mags.append(v)
            mx, mn = max(mags), min(mags)
            spread = float((mx - mn) / mx) if mx > 0 else 1.0
            xs = new
            if spread < tol:
                z, E = self.newton(xs, z, E)
                break
        return xs, z, E, spread

    def run(self, tol=1e-8, max_iter=40):
        n = self.n
        N = 2 * n + 2
        lo, hi = self.lo, self.hi
        llo = lo.ln()
        L_target = hi.ln() - llo
        Lw = min(L_target, D(2))
        # Chebyshev-like positions in log x on the first interval
        tpos = [(1 - D(math.cos(math.pi * i / (N - 1)))) / 2 for i in range(N)]
        z, E, spread = None, D(0), 1.0
        while True:
            self.hi = (llo + Lw).exp()
            xs = [(llo + Lw * t).exp() for t in tpos]
            if z is None:
                z = self.initial(xs)
            xs, z, E, spread = self.iterate(xs, z, E, tol if Lw >= L_target else 1e-3, max_iter)
            tpos = [(x.ln() - llo) / Lw for x in xs]
            if Lw >= L_target:
                break
            Lw = min(L_target, Lw * D("1.6"))
        self.hi = hi
        p, q = self.coeffs(z)
        return p, q, abs(E), spread


def _real_roots(c: List[D], lo: D, hi: D, count: int) -> List[D]:
    """The `count` real roots of the polynomial c on the negative axis
    -hi..-lo, by sign changes on a log grid and bisection."""
    llo, lhi = lo.ln(), hi.ln()
    m = 6000
    roots = []
    prev_x = -(llo.exp())
    prev_v = _horner(c, prev_x)
    eps = D(10) ** (-(decimal.getcontext().prec - 10))
    for k in range(1, m + 1):
        x = -((llo + (lhi - llo) * k / m).exp())
        v = _horner(c, x)
        if (v > 0) != (prev_v > 0):
            a, b, va = prev_x, x, prev_v
            for _ in range(400):
                mid = (a + b) / 2
                vm = _horner(c, mid)
                if (vm > 0) == (va > 0):
                    a, va = mid, vm
                else:
                    b = mid
                if abs(b - a) <= abs(mid) * eps:
                    break
            roots.append((a + b) / 2)
        prev_x, prev_v = x, v
    if len(roots) != count:
        raise ArithmeticError(f"found {len(roots)} of {count} real roots")
    return roots


def _partial_fractions(num: List[D], den: List[D], lo: D, hi: D):
    """num/den (den of degree n with real negative roots) as
    a0 + sum a_k/(x + sigma_k)."""
    n = len(den) - 1
    roots = _real_roots(den, lo * D(10) ** -12, hi * D(10) ** 12, n)
    dden = [den[j] * j for j in range(1, n + 1)]
    a0 = num[-1] / den[-1] if len(num) == len(den) else D(0)
    a = [_horner(num, r) / _horner(dden, r) for r in roots]
    return a0, a, [-r for r in roots]


def remez(power, lo: float, hi: float, n: int, digits: int = 150, tol: float = 1e-8):
    """Minimax relative approximation of x^power on [lo, hi] by a type (n, n)
    rational function.  power: a Fraction or a string like "-1/4".  Returns
    (r, rinv): r ~ x^power and rinv = 1/r ~ x^-power, both RationalApprox."""
    pw = Fraction(power)
    ctx = decimal.Context(prec=digits, Emin=-10 ** 6, Emax=10 ** 6)
    with decimal.localcontext(ctx):
        lo_d, hi_d = D(repr(float(lo))), D(repr(float(hi)))
        rm = _Remez(pw, lo_d, hi_d, n)
        p, q, E, spread = rm.run(tol=tol)
        a0, a, s = _partial_fractions(p, q, lo_d, hi_d)
        b0, b, t = _partial_fractions(q, p, lo_d, hi_d)
        oa = sorted(range(n), key=lambda k: s[k])
        ob = sorted(range(n), key=lambda k: t[k])
        r = RationalApprox(float(a0), [float(a[k]) for k in oa], [float(s[k]) for k in oa],
                           float(E), pw, lo, hi)
        rinv = RationalApprox(float(b0), [float(b[k]) for k in ob], [float(t[k]) for k in ob],
                              float(E), -pw, lo, hi)
    r.spread = rinv.spread = spread
    return r, rinv


def write_remez_file(path: str, a: RationalApprox, b: RationalApprox) -> None:
    """The reference's remez file layout (read at rhmc/cheisdwf.f:140-159):
    a0; n lines 'a_k, sigma_k'; b0; n lines 'b_k, sigma_k'."""
    with open(path, "w") as fh:
        fh.write(f"{a.a0:.17e}\n")
        for ak, sk in zip(a.a, a.sigma):
            fh.write(f"{ak:.17e}, {sk:.17e}\n")
        fh.write(f"{b.a0:.17e}\n")
        for bk, tk in zip(b.a, b.sigma):
            fh.write(f"{bk:.17e}, {tk:.17e}\n")


def read_remez_file(path: str, n: int):
    """(anum[0..n], aden, bnum[0..n], bden) from a remez file."""
    import numpy as np
    vals = []
    for line in open(path):
        line = line.replace(",", " ").replace("d", "e").replace("D", "e").strip()
        if line:
            vals.append([float(t) for t in line.split()])
    an = [vals[0][0]] + [v[0] for v in vals[1:n + 1]]
    ad = [v[1] for v in vals[1:n + 1]]
    bn = [vals[n + 1][0]] + [v[0] for v in vals[n + 2:2 * n + 2]]
    bd = [v[1] for v in vals[n + 2:2 * n + 2]]
    return (np.array(an), np.array(ad), np.array(bn), np.array(bd))
