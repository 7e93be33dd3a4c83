"""Generate zig_tables.inc: the 256-layer ziggurat tables of Exp(1).

Marsaglia & Tsang's ziggurat for the exponential density f(x) = e^-x with
n = 256 layers of equal area v.  With r the base-layer edge:
    v        = (r + 1) e^-r                 (base strip r f(r) + tail f(r))
    x[0]     = v / f(r) = r + 1,  x[1] = r
    x[i+1]   = -ln(e^-x[i] + v / x[i])      (equal-area recurrence)
    x[256]   = 0,  y[i] = e^-x[i] (i >= 1),  y[0] = 0,  y[256] = 1
r is fixed by closing the recurrence at the top (x[256] = 0), found here by
bisection in 90-digit decimal arithmetic; every entry is then rounded once to
the nearest double.  These are the tables the ProbMinHash exponential sampler
indexes with the low byte of a random word (Boost exponential_table layout).
"""
import os
import sys
from decimal import Decimal as D, getcontext

N = 256


def _chain(r):
    v = (r + 1) * (-r).exp()
    xs = [r + 1, r]
    x = r
    for _ in range(1, N - 1):
        t = (-x).exp() + v / x
        if t >= 1:
            return None, None
        x = -(t.ln())
        xs.append(x)
    return xs, (-x).exp() + v / x - 1


def tables():
    getcontext().prec = 90
    lo, hi = D("7.6"), D("7.8")
    for _ in range(280):
        mid = (lo + hi) / 2
        xs, close = _chain(mid)
        if xs is None or close >= 0:
            lo = mid
        else:
            hi = mid
    xs, _ = _chain((lo + hi) / 2)
    xs.append(D(0))
    ys = [D(0)] + [(-x).exp() for x in xs[1:N]] + [D(1)]
    return [float(x) for x in xs], [float(y) for y in ys]


def main(out_path):
    tx, ty = tables()
    with open(out_path, "w") as f:
        f.write("// Generated by gen_zig_tables.py (ziggurat recurrence, 90-digit decimal).\n")
        f.write("static const double kZigX[257] = {\n")
        f.write(",\n".join(f"  {x!r}" for x in tx))
        f.write("\n};\nstatic const double kZigY[257] = {\n")
        f.write(",\n".join(f"  {y!r}" for y in ty))
        f.write("\n};\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else
         os.path.join(os.path.dirname(os.path.abspath(__file__)), "zig_tables.inc"))
