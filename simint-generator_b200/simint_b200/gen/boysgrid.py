"""Tabulated Boys function for the Taylor-grid evaluation.

F_n(x) = int_0^1 t^(2n) exp(-x t^2) dt = gamma(n+1/2, x) / (2 x^(n+1/2)).

The table layout and grid follow the reference's Boys scheme
(skel/simint/boys/boys_shortgrid.h:3-8, boys_taylor.h:14-39): grid points
x_i = 0.1 i for i = 0..365 (x < 36.5 is handled by the grid), orders
n = 0..31, and a 7th-order Taylor expansion around the nearest grid point
F_n(x) = sum_k F_{n+k}(x_i) (x_i - x)^k / k!, k = 0..7.
Above 36.5 the asymptotic form F_n(x) = (2n-1)!!/2^(n+1) sqrt(pi / x^(2n+1))
is used with the factor table boys_longfac[n] = sqrt(pi) (2n-1)!! / 2^(n+1)
(boys_longfac.h:13-49).

The values are computed here with mpmath at 60 significant digits (the same
recipe as python/boys/boys_common/boys.py:10-21, our own code) and rounded
to double; the generated C include is shared by the CUDA kernels and the CPU
oracle.  Generation takes a few seconds and is cached next to the output.
"""

import os

NPOINT = 366
MAXN = 31
SPACE = 0.1
MAXX = 36.5


def boys_value(n, x, mp):
    if x == 0:
        return mp.mpf(1) / (2 * n + 1)
    x = mp.mpf(x)
    a = mp.mpf(n) + mp.mpf(1) / 2
    return mp.gammainc(a, 0, x) / (2 * mp.power(x, a))


def make_table():
    import mpmath as mp
    mp.mp.dps = 60
    rows = []
    for i in range(NPOINT):
        x = mp.mpf(i) / 10          # exact decimal grid point
        rows.append([float(boys_value(n, x, mp)) for n in range(MAXN + 1)])
    longfac = []
    for n in range(MAXN + 1):
        df = mp.mpf(1)
        for k in range(2 * n - 1, 0, -2):
            df *= k
        longfac.append(float(mp.sqrt(mp.pi) * df / mp.power(2, n + 1)))
    return rows, longfac


def write_include(path):
    rows, longfac = make_table()
    lines = ["/* Boys function grid: F_n(0.1 i), i = 0..365, n = 0..31, and the",
             " * asymptotic factors sqrt(pi)(2n-1)!!/2^(n+1).  Generated by",
             " * simint_b200/gen/boysgrid.py (mpmath, 60 digits). */",
             "#define SIMINT_B200_BOYS_NPOINT %d" % NPOINT,
             "#define SIMINT_B200_BOYS_MAXN %d" % MAXN,
             "#define SIMINT_B200_BOYS_MAXX %r" % MAXX,
             "static const double simint_b200_boys_grid_host[%d][%d] = {" % (NPOINT, MAXN + 1)]
    for r in rows:
        lines.append("  {" + ", ".join(repr(v) for v in r) + "},")
    lines.append("};")
    lines.append("static const double simint_b200_boys_longfac_host[%d] = {" % (MAXN + 1))
    lines.append("  " + ", ".join(repr(v) for v in longfac))
    lines.append("};")
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write("\n".join(lines) + "\n")
    os.replace(tmp, path)


def ensure_include(path):
    if not os.path.exists(path):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        write_include(path)
    return path


if __name__ == "__main__":
    import sys
    write_include(sys.argv[1])
