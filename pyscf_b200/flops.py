"""Operation-count model of the J/K build (FP64 flops), used for the roofline.

Counts follow the arithmetic of the kernels in csrc/ (an FMA is 2 flops,
other operations 1), per primitive quartet of class (la lb|lc ld) with
n = L/2+1 Rys roots, NE = la+lb+1, NF = lc+ld+1, NG Cartesian components:
  setup        40                     centres, T, prefactor
  roots        4 n DEG                Horner evaluation of 2n polynomials of degree DEG
  per root     15                     recurrence coefficients
               3 * 4 NE NF            vertical recurrence, three directions
               3 * hrr(la,lb,lc,ld)   horizontal transfer, three directions
               3 NG                   I_x I_y I_z products accumulated into the block
and per contracted shell quartet and density
  12 NG                               J (2 FMA) and K (4 FMA) contractions.
Algorithmic flops of a build = sum over classes of
  prim_quartets * F_prim + quartets * n_dm * 12 NG.
"""
RYS_DEG = 13


def ncart(l):
    return (l + 1) * (l + 2) // 2


def hrr_flops(la, lb, lc, ld):
    nf = lc + ld + 1
    bra = sum(2 * (b + 1) for a in range(la + 1) for b in range(lb + 1)) * nf
    ket = sum(2 * (d + 1) for c in range(lc + 1) for d in range(ld + 1)) * (la + 1) * (lb + 1)
    return bra + ket


def prim_quartet_flops(la, lb, lc, ld):
    n = (la + lb + lc + ld) // 2 + 1
    ng = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    ne, nf = la + lb + 1, lc + ld + 1
    per_root = 15 + 3 * 4 * ne * nf + 3 * hrr_flops(la, lb, lc, ld) + 3 * ng
    return 40 + 4 * n * RYS_DEG + n * per_root


def contraction_flops(la, lb, lc, ld, n_dm=1):
    return 12 * ncart(la) * ncart(lb) * ncart(lc) * ncart(ld) * n_dm


def build_flops(class_stats, n_dm=1):
    """Total modelled flops of a build from Plan.class_stats()."""
    tot = 0.0
    for c in class_stats:
        key = (c['la'], c['lb'], c['lc'], c['ld'])
        tot += c['prim_quartets'] * prim_quartet_flops(*key) + c['quartets'] * contraction_flops(*key, n_dm=n_dm)
    return tot


def class_flops(c, n_dm=1):
    key = (c['la'], c['lb'], c['lc'], c['ld'])
    return c['prim_quartets'] * prim_quartet_flops(*key) + c['quartets'] * contraction_flops(*key, n_dm=n_dm)
