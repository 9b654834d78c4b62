"""Generate the Rys-quadrature root/weight tables used by the CUDA kernels.

The Rys quadrature of order n for argument T is the n-point Gauss rule of the
measure  dmu(u) = exp(-T u) / (2 sqrt(u)) du  on u in [0, 1]  (u = t^2).  Its
moments are Boys functions,  int u^k dmu = F_k(T),  so the rule follows from
F_0..F_{2n-1} (Rys, Dupuis & King, J. Comput. Chem. 4, 154 (1983)).

This script computes the rules at 60 significant digits with mpmath:
  1. F_k(T) = gamma_lower(k+1/2, T) / (2 T^(k+1/2))  (F_k(0) = 1/(2k+1));
  2. recurrence coefficients of the orthogonal polynomials from the moments
     by Gautschi's Chebyshev algorithm (W. Gautschi, "Orthogonal Polynomials:
     Computation and Approximation", 2004, sec. 2.1.7);
  3. nodes and weights from the Jacobi matrix (Golub & Welsch, 1969).

Tables.  For each order n the interval [0, T_asym(n)) is cut into pieces of
width 1/PIECES_PER_UNIT; on each piece every root u_i(T) and weight w_i(T) is
a polynomial of degree DEG in the local variable x in [-1, 1], fitted by
Chebyshev interpolation and stored as power-basis coefficients for a Horner
evaluation.  Beyond T_asym(n) the rule is the large-T limit
   u_i = x_i^2 / T,  w_i = W_i / sqrt(T),
with (x_i, W_i) the positive nodes / weights of the 2n-point Gauss-Hermite rule;
T_asym(n) is the smallest grid point where that limit agrees with the exact
rule to 1e-15 relative.

The float64 Horner evaluation is replayed here with numpy on random test
points and compared with the 60-digit rule; the largest relative error is
written into the header.

Output: rys_table.inc (C++ arrays), committed next to this script.
Run:    python pyscf_b200/csrc/gen_rys_table.py   (a few minutes, 8 processes)
"""
import os
import sys
import multiprocessing as mp
import numpy as np
import mpmath

NMAX = 8               # up to 8 roots: (ff|ff) needs 7, its first derivative 7
PIECES_PER_UNIT = 1
DEG = 13               # polynomial degree per piece
T_GRID_MAX = 120
DPS = 60

HERE = os.path.dirname(os.path.abspath(__file__))


def boys_moments(T, kmax):
    T = mpmath.mpf(T)
    if T == 0:
        return [mpmath.mpf(1) / (2 * k + 1) for k in range(kmax + 1)]
    return [mpmath.gammainc(k + mpmath.mpf(1) / 2, 0, T) / (2 * T ** (k + mpmath.mpf(1) / 2))
            for k in range(kmax + 1)]


def chebyshev_algorithm(mom, n):
    """alpha_k, beta_k (k < n) of the monic orthogonal polynomials from the
    ordinary moments mom[0..2n-1]."""
    sig_prev = [mpmath.mpf(0)] * (2 * n)
    sig = list(mom[:2 * n])
    alpha = [mom[1] / mom[0]]
    beta = [mom[0]]
    for k in range(1, n):
        sig_new = [mpmath.mpf(0)] * (2 * n)
        for l in range(k, 2 * n - k):
            sig_new[l] = sig[l + 1] - alpha[k - 1] * sig[l] - beta[k - 1] * sig_prev[l]
        alpha.append(sig_new[k + 1] / sig_new[k] - sig[k] / sig[k - 1])
        beta.append(sig_new[k] / sig[k - 1])
        sig_prev, sig = sig, sig_new
    return alpha, beta


def gauss_rule(alpha, beta, n):
    J = mpmath.zeros(n, n)
    for i in range(n):
        J[i, i] = alpha[i]
        if i + 1 < n:
            J[i, i + 1] = J[i + 1, i] = mpmath.sqrt(beta[i + 1])
    E, Q = mpmath.eigsy(J)
    nodes = [E[i] for i in range(n)]
    weights = [beta[0] * Q[0, i] ** 2 for i in range(n)]
    order = sorted(range(n), key=lambda i: nodes[i])
    return [nodes[i] for i in order], [weights[i] for i in order]


def rys_rules(T):
    """(roots, weights) for n = 1..NMAX at one T, from one moment set."""
    mpmath.mp.dps = DPS
    mom = boys_moments(T, 2 * NMAX - 1)
    alpha, beta = chebyshev_algorithm(mom, NMAX)
    out = {}
    for n in range(1, NMAX + 1):
        r, w = gauss_rule(alpha, beta, n)
        out[n] = ([float(x) for x in r], [float(x) for x in w], r, w)
    return out


def hermite_half(n):
    """positive nodes x_i and weights W_i of the 2n-point Gauss-Hermite rule"""
    mpmath.mp.dps = DPS
    # Jacobi matrix of physicists' Hermite polynomials: alpha=0, beta_k = k/2
    m = 2 * n
    J = mpmath.zeros(m, m)
    for i in range(m - 1):
        J[i, i + 1] = J[i + 1, i] = mpmath.sqrt(mpmath.mpf(i + 1) / 2)
    E, Q = mpmath.eigsy(J)
    pairs = sorted([(E[i], mpmath.sqrt(mpmath.pi) * Q[0, i] ** 2) for i in range(m)])
    pos = [(x, w) for x, w in pairs if x > 0]
    return [p[0] for p in pos], [p[1] for p in pos]


def cheb_nodes(a, b, deg):
    k = np.arange(deg + 1)
    x = np.cos(np.pi * (k + 0.5) / (deg + 1))
    return x, a + (b - a) * (x + 1) / 2


def _eval_point(T):
    r = rys_rules(T)
    return T, {n: (r[n][2], r[n][3]) for n in r}


def fit_piece(values_mp, xnodes, deg):
    """power-basis coefficients (ascending) of the Chebyshev interpolant"""
    mpmath.mp.dps = DPS
    # Chebyshev coefficients c_j = 2/(N) sum_k f_k T_j(x_k)
    N = deg + 1
    c = []
    for j in range(N):
        s = mpmath.mpf(0)
        for k in range(N):
            s += values_mp[k] * mpmath.cos(mpmath.pi * j * (k + mpmath.mpf(1) / 2) / N)
        c.append(s * 2 / N)
    c[0] /= 2
    # convert sum c_j T_j(x) to power basis
    power = [mpmath.mpf(0)] * N
    Tprev = [mpmath.mpf(1)] + [mpmath.mpf(0)] * (N - 1)
    Tcur = [mpmath.mpf(0), mpmath.mpf(1)] + [mpmath.mpf(0)] * (N - 2)
    for j in range(N):
        Tj = Tprev if j == 0 else Tcur if j == 1 else None
        if j >= 2:
            Tnext = [mpmath.mpf(0)] * N
            for i in range(N):
                if i >= 1:
                    Tnext[i] += 2 * Tcur[i - 1]
                Tnext[i] -= Tprev[i]
            Tprev, Tcur = Tcur, Tnext
            Tj = Tcur
        for i in range(N):
            power[i] += c[j] * Tj[i]
    return [float(p) for p in power]


def horner(coef, x):
    r = np.zeros_like(x) + coef[-1]
    for c in coef[-2::-1]:
        r = r * x + c
    return r


def main():
    mpmath.mp.dps = DPS
    npiece = T_GRID_MAX * PIECES_PER_UNIT
    h = 1.0 / PIECES_PER_UNIT
    xk, _ = cheb_nodes(-1.0, 1.0, DEG)
    points = []
    for p in range(npiece):
        a = p * h
        for x in xk:
            points.append(a + h * (x + 1) / 2)
    # asymptotic check points (integer T)
    check_T = [float(t) for t in range(5, T_GRID_MAX + 1)]
    with mp.get_context('spawn').Pool(min(8, os.cpu_count() or 1)) as pool:
        vals = dict(pool.map(_eval_point, points + check_T, chunksize=16))
    herm = {n: hermite_half(n) for n in range(1, NMAX + 1)}
    # asymptotic thresholds
    t_asym = {}
    for n in range(1, NMAX + 1):
        xs, Ws = herm[n]
        ok_from = None
        for T in check_T:
            r, w = vals[T][n]
            err = 0
            for i in range(n):
                ua = xs[i] ** 2 / T
                wa = Ws[i] / mpmath.sqrt(T)
                err = max(err, abs(ua / r[i] - 1), abs(wa / w[i] - 1))
            if err < 1e-15:
                if ok_from is None:
                    ok_from = T
            else:
                ok_from = None
        if ok_from is None:
            raise SystemExit('asymptotic limit not reached for n=%d within T<%d' % (n, T_GRID_MAX))
        t_asym[n] = int(ok_from)
    # fit pieces
    tables = {}
    maxerr = {}
    rng = np.random.default_rng(7)
    for n in range(1, NMAX + 1):
        npc = t_asym[n] * PIECES_PER_UNIT
        tab = np.zeros((npc, 2 * n, DEG + 1))
        for p in range(npc):
            a = p * h
            Ts = [a + h * (x + 1) / 2 for x in xk]
            for i in range(n):
                tab[p, i] = fit_piece([vals[T][n][0][i] for T in Ts], xk, DEG)
                tab[p, n + i] = fit_piece([vals[T][n][1][i] for T in Ts], xk, DEG)
        tables[n] = tab
    # validate the float64 Horner evaluation on random points
    ntest = 60
    testT = np.concatenate([rng.uniform(0, t_asym[NMAX], ntest), rng.uniform(0, 2, 10)])
    with mp.get_context('spawn').Pool(min(8, os.cpu_count() or 1)) as pool:
        tv = dict(pool.map(_eval_point, [float(t) for t in testT], chunksize=4))
    for n in range(1, NMAX + 1):
        e = 0.0
        xs, Ws = herm[n]
        for T in testT:
            T = float(T)
            r, w = tv[T][n]
            if T >= t_asym[n]:
                ue = np.array([float(xs[i] ** 2) / T for i in range(n)])
                we = np.array([float(Ws[i]) / np.sqrt(T) for i in range(n)])
            else:
                p = int(T * PIECES_PER_UNIT)
                x = np.array([2 * (T - p * h) / h - 1])
                ue = np.array([horner(tables[n][p, i], x)[0] for i in range(n)])
                we = np.array([horner(tables[n][p, n + i], x)[0] for i in range(n)])
            for i in range(n):
                e = max(e, abs(ue[i] / float(r[i]) - 1), abs(we[i] / float(w[i]) - 1))
        maxerr[n] = e
        print('n=%d  T_asym=%d  max rel err %.2e' % (n, t_asym[n], e))
    write_inc(tables, t_asym, herm, maxerr)


def write_inc(tables, t_asym, herm, maxerr):
    """Write rys_table.inc.  The includer defines RYS_TABLE_QUALIFIER (for
    example `__device__ const` or `static const`) before including it."""
    out = os.path.join(HERE, 'rys_table.inc')
    with open(out, 'w') as f:
        f.write('// Generated by gen_rys_table.py -- do not edit.\n')
        f.write('// Rys roots u_i = t_i^2 and weights w_i (sum_i w_i = F_0(T)).\n')
        f.write('// Piece p covers T in [p, p+1); x = 2 (T - p) - 1; each row holds DEG+1\n')
        f.write('// power-basis coefficients (ascending) of u_0..u_{n-1}, w_0..w_{n-1}.\n')
        f.write('// Largest relative error of the float64 Horner evaluation against\n')
        f.write('// 60-digit rules on random test points:\n')
        for n in sorted(maxerr):
            f.write('//   n=%d: %.2e (asymptotic from T=%d)\n' % (n, maxerr[n], t_asym[n]))
        f.write('#define RYS_NMAX %d\n#define RYS_DEG %d\n#define RYS_PIECES_PER_UNIT %d\n'
                % (NMAX, DEG, PIECES_PER_UNIT))
        f.write('#define RYS_T_ASYM_LIST 0, %s\n' % ', '.join(str(t_asym[n]) for n in range(1, NMAX + 1)))
        offs = [0]
        for n in range(1, NMAX + 1):
            offs.append(offs[-1] + tables[n].size)
        f.write('#define RYS_TABLE_OFFSET_LIST 0, %s\n' % ', '.join(str(o) for o in offs[:NMAX]))
        f.write('#define RYS_TABLE_SIZE %d\n' % offs[-1])
        x2 = []
        ws = []
        for n in range(1, NMAX + 1):
            xs, Ws = herm[n]
            x2 += ['%.17e' % float(x ** 2) for x in xs]
            ws += ['%.17e' % float(w) for w in Ws]
        f.write('#define RYS_HERMITE_X2_LIST %s\n' % ', '.join(x2))
        f.write('#define RYS_HERMITE_W_LIST %s\n' % ', '.join(ws))
        f.write('#ifdef RYS_TABLE_QUALIFIER\n')
        f.write('RYS_TABLE_QUALIFIER double rys_table_data[RYS_TABLE_SIZE] = {\n')
        for n in range(1, NMAX + 1):
            flat = tables[n].reshape(-1)
            for i in range(0, flat.size, 4):
                f.write('  ' + ', '.join('%.17e' % v for v in flat[i:i + 4]) + ',\n')
        f.write('};\n#endif\n')
    print('wrote', out)


if __name__ == '__main__':
    main()
