"""Derive the float32 Rys tables (rys_table_f.inc) from the float64 ones.

The float32 pass of mixed precision needs roots and weights to float32
accuracy only, so its tables are smaller than the float64 tables of
gen_rys_table.py in two ways:
  1. each degree-13 piece polynomial (piece width 1 in T, local variable
     x in [-1, 1]) is re-expanded in Chebyshev polynomials and truncated to
     degree DEG_F; the dropped Chebyshev coefficients bound the truncation
     error, which is far below float32 rounding at DEG_F = 7;
  2. the large-T limit  u_i = x_i^2 / T,  w_i = W_i / sqrt(T)  (positive
     nodes/weights of the 2n-point Gauss-Hermite rule) is taken from the
     smallest integer T_asym_f(n) beyond which it agrees with the float64
     table to TOL_F (absolute on u, relative to F_0 = sum_i w_i on w).

Rows hold DEG_F + 1 = 8 float32 coefficients (two aligned 16-byte vectors).
The header of the output records the largest deviation from the float64
table over a grid of test points, coefficient rounding included.

Run:  python pyscf_b200/csrc/gen_rys_table_f.py   (seconds; reads rys_table.inc)
"""
import os
import re
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEG_F = 7
TOL_F = 3e-8
NTEST = 41


def parse(src):
    def lst(name, conv):
        m = re.search(r'#define %s (.*)' % name, src)
        return [conv(x) for x in m.group(1).split(',')]
    deg = int(re.search(r'#define RYS_DEG (\d+)', src).group(1))
    nmax = int(re.search(r'#define RYS_NMAX (\d+)', src).group(1))
    t_asym = lst('RYS_T_ASYM_LIST', int)
    off = lst('RYS_TABLE_OFFSET_LIST', int)
    x2 = lst('RYS_HERMITE_X2_LIST', float)
    w = lst('RYS_HERMITE_W_LIST', float)
    m = re.search(r'rys_table_data\[[^\]]*\]\s*=\s*\{(.*?)\};', src, re.S)
    data = np.array([float(v) for v in m.group(1).split(',') if v.strip()])
    return deg, nmax, t_asym, off, x2, w, data


def main():
    src = open(os.path.join(HERE, 'rys_table.inc')).read()
    deg, nmax, t_asym, off, x2, hw, data = parse(src)
    P = np.polynomial
    xs = np.linspace(-1.0, 1.0, NTEST)

    def piece(n, p):
        o = off[n] + p * 2 * n * (deg + 1)
        return data[o:o + 2 * n * (deg + 1)].reshape(2 * n, deg + 1)

    t_asym_f = [0] * (nmax + 1)
    rows_f = {}
    errs = {}
    for n in range(1, nmax + 1):
        k0 = n * (n - 1) // 2
        # smallest integer T from which the large-T limit is within TOL_F
        ta = t_asym[n]
        for p in range(t_asym[n] - 1, -1, -1):
            R = piece(n, p)
            T = p + (xs + 1.0) / 2.0
            u = np.array([P.polynomial.polyval(xs, R[i]) for i in range(n)])
            w = np.array([P.polynomial.polyval(xs, R[n + i]) for i in range(n)])
            F0 = w.sum(axis=0)
            ua = np.array([x2[k0 + i] / T for i in range(n)])
            wa = np.array([hw[k0 + i] / np.sqrt(T) for i in range(n)])
            if np.abs(u - ua).max() > TOL_F or (np.abs(w - wa) / F0).max() > TOL_F:
                break
            ta = p
        t_asym_f[n] = ta
        worst = 0.0
        out = []
        for p in range(ta):
            R = piece(n, p)
            F0 = sum(P.polynomial.polyval(xs, R[n + i]) for i in range(n))
            for r in range(2 * n):
                c = P.chebyshev.poly2cheb(R[r])
                c[DEG_F + 1:] = 0.0
                cf = P.chebyshev.cheb2poly(c)[:DEG_F + 1].astype(np.float32)
                v = P.polynomial.polyval(xs, R[r])
                vf = P.polynomial.polyval(xs, cf.astype(np.float64))
                e = np.abs(v - vf) / (F0 if r >= n else 1.0)
                worst = max(worst, float(e.max()))
                out.append(cf)
        rows_f[n] = out
        errs[n] = worst

    offs = [0] * (nmax + 2)
    for n in range(1, nmax + 1):
        offs[n + 1] = offs[n] + len(rows_f[n]) * (DEG_F + 1)
    size = offs[nmax + 1]
    lines = ['// Generated by gen_rys_table_f.py from rys_table.inc -- do not edit.',
             '// float32 Rys roots u_i and weights w_i for the float32 pass of mixed',
             '// precision.  Same pieces as the float64 table (piece p covers T in',
             '// [p, p+1), x = 2 (T - p) - 1), Chebyshev-truncated to degree %d; rows of' % DEG_F,
             '// %d ascending power-basis coefficients, u_0..u_{n-1}, w_0..w_{n-1}.' % (DEG_F + 1),
             '// Largest deviation from the float64 table (|du|, |dw|/F_0), coefficient',
             '// rounding included, and the T from which the large-T limit is used:']
    for n in range(1, nmax + 1):
        lines.append('//   n=%d: %.2e (asymptotic from T=%d)' % (n, errs[n], t_asym_f[n]))
    lines += ['#define RYS_F_DEG %d' % DEG_F,
              '#define RYS_F_ROW %d' % (DEG_F + 1),
              '#define RYS_F_T_ASYM_LIST %s' % ', '.join(str(t) for t in t_asym_f),
              '#define RYS_F_OFFSET_LIST %s' % ', '.join(str(o) for o in offs[:nmax + 1]),
              '#define RYS_F_SIZE %d' % size,
              '#ifdef RYS_TABLE_QUALIFIER',
              'RYS_TABLE_QUALIFIER float rys_table_f_data[RYS_F_SIZE] = {']
    vals = []
    for n in range(1, nmax + 1):
        for cf in rows_f[n]:
            vals += ['%.9ef' % float(v) for v in cf]
    for i in range(0, len(vals), 6):
        lines.append('        ' + ', '.join(vals[i:i + 6]) + ',')
    lines.append('};')
    lines.append('#endif')
    with open(os.path.join(HERE, 'rys_table_f.inc'), 'w') as fh:
        fh.write('\n'.join(lines) + '\n')
    print('rys_table_f.inc: %d floats; errors %s; T_asym_f %s' % (
        size, ' '.join('%.1e' % errs[n] for n in range(1, nmax + 1)), t_asym_f[1:]))


if __name__ == '__main__':
    main()
