"""The kernels' integral arithmetic, replayed on the host, against the oracle.

b200jk_hostcheck_cart_quartet[_fp32] evaluate one shell quartet with the same
templates the CUDA kernels instantiate (Rys tables, recurrences, assembly),
compiled for the CPU.  The oracle's Obara-Saika/HGP integrals are an
independent formulation, so agreement pins the tables and recurrences of both
precisions for every (la lb | lc ld) orientation with l <= 3, without a GPU.
"""
import itertools

import numpy
import pytest

import oracle

SP = [0.282094791773878143, 0.488602511902919921, 1.0, 1.0]   # libcint's s/p factors


def _basis(offset):
    rng = numpy.random.default_rng(3)
    atm = numpy.zeros((4, 6), numpy.int32)
    env = [0.0] * 20
    bas = []
    for a in range(4):
        atm[a, 0] = 1
        atm[a, 1] = len(env)
        env += list(rng.uniform(-1, 1, 3) + offset)
    for a in range(4):
        for l in range(4):
            nprim = int(rng.integers(1, 3))
            pe = len(env)
            env += list(rng.uniform(0.2, 3.0, nprim))
            pc = len(env)
            env += list(rng.uniform(0.2, 1.0, nprim))
            bas.append([a, l, nprim, 1, 0, pe, pc, 0])
    return atm, numpy.array(bas, numpy.int32), numpy.array(env)


@pytest.mark.parametrize('fp32,tol', [(False, 1e-12), (True, 1e-5)])
def test_all_orientations(fp32, tol):
    from pyscf_b200 import lib
    # far from the origin: the float32 pass works relative to the first centre
    atm, bas, env = _basis(numpy.array([10.0, -7.0, 4.0]))
    worst = 0.0
    for ls in itertools.product(range(4), repeat=4):
        shls = [ls[0], 4 + ls[1], 8 + ls[2], 12 + ls[3]]
        ref = oracle.int2e_cart(atm, bas, env, shls) / (SP[ls[0]] * SP[ls[1]] * SP[ls[2]] * SP[ls[3]])
        got = lib.hostcheck_cart_quartet(atm, bas, env, shls, fp32=fp32)
        worst = max(worst, abs(got - ref).max() / max(abs(ref).max(), 1e-300))
    assert worst < tol
