"""CPU oracle for the direct-SCF J/K path.

ORACLE / TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py may import this package, and only as the checker
or the timed CPU baseline; the product (pyscf_b200) never does.

* ``liboracle.so`` (built by oracle/build.py): this project's restatement of
  libcint's int2e/int1e integrals (cint/cint_shim.c) and of PySCF's
  CVHFnr_direct_drv J/K driver (jk_direct.c).
* ``oracle/_ref`` (built only where the reference tree is readable): PySCF's
  own C drivers compiled from the reference sources against the same integral
  library.

Parity of the integral library is pinned against the reference's own golden
values (see tests/test_oracle_golden.py and tests/golden/README.md).
"""
import ctypes
import os

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'liboracle.so')
REF_LIBDIR = os.path.join(HERE, '_ref', 'pyext', 'pyscf', 'lib')

_lib = None


def ensure_built():
    import importlib
    importlib.import_module(__name__ + '.build').build_all()


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            ensure_built()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_get_jk.restype = ctypes.c_int
        _lib.oracle_grad_jk.restype = ctypes.c_int
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _arrays(atm, bas, env):
    return (numpy.ascontiguousarray(atm, dtype=numpy.int32), numpy.ascontiguousarray(bas, dtype=numpy.int32),
            numpy.array(env, dtype=numpy.double, order='C', copy=True))


def nao(bas, cart=False):
    bas = numpy.asarray(bas)
    l = bas[:, 1]
    nf = (l + 1) * (l + 2) // 2 if cart else 2 * l + 1
    return int((nf * bas[:, 3]).sum())


def ao_loc(bas, cart=False):
    bas = numpy.asarray(bas)
    l = bas[:, 1]
    nf = (l + 1) * (l + 2) // 2 if cart else 2 * l + 1
    return numpy.concatenate([[0], numpy.cumsum(nf * bas[:, 3])]).astype(numpy.int32)


def q_cond(atm, bas, env, cart=False, direct_scf_tol=1e-13):
    """CVHFnr_int2e_q_cond under mol.with_integral_screen(tol**2)."""
    lib = load()
    atm, bas, env = _arrays(atm, bas, env)
    nbas = bas.shape[0]
    q = numpy.empty((nbas, nbas))
    cut = -numpy.log(direct_scf_tol ** 2) if direct_scf_tol > 0 else 0.0
    lib.oracle_q_cond(_p(q), _p(atm), ctypes.c_int(atm.shape[0]), _p(bas), ctypes.c_int(nbas), _p(env),
                      ctypes.c_int(int(cart)), ctypes.c_double(cut))
    return q


def dm_cond(dms, bas, cart=False):
    lib = load()
    bas = numpy.ascontiguousarray(bas, dtype=numpy.int32)
    dms = numpy.ascontiguousarray(dms, dtype=numpy.double)
    n = dms.shape[-1]
    dms = dms.reshape(-1, n, n)
    out = numpy.empty((bas.shape[0], bas.shape[0]))
    lib.oracle_dm_cond(_p(out), _p(dms), ctypes.c_int(dms.shape[0]), _p(bas), ctypes.c_int(bas.shape[0]),
                       ctypes.c_int(int(cart)))
    return out


def get_jk(dms, atm, bas, env, hermi=1, cart=False, direct_scf_tol=1e-13, screen=True):
    """J/K of the restated direct-SCF driver.  screen=False is vhfopt=None.
    Returns (vj, vk, n_quartets_evaluated)."""
    lib = load()
    atm, bas, env = _arrays(atm, bas, env)
    dms = numpy.ascontiguousarray(dms, dtype=numpy.double)
    shape = dms.shape
    n = shape[-1]
    dms = dms.reshape(-1, n, n)
    vj = numpy.empty_like(dms)
    vk = numpy.empty_like(dms)
    qc = dc = None
    if screen:
        qc = q_cond(atm, bas, env, cart, direct_scf_tol)
        dc = dm_cond(dms, bas, cart)
    nq = ctypes.c_longlong(0)
    rc = lib.oracle_get_jk(_p(dms), ctypes.c_int(dms.shape[0]), _p(vj), _p(vk), ctypes.c_int(hermi),
                           _p(atm), ctypes.c_int(atm.shape[0]), _p(bas), ctypes.c_int(bas.shape[0]), _p(env),
                           ctypes.c_int(int(cart)), _p(qc) if screen else None, _p(dc) if screen else None,
                           ctypes.c_double(direct_scf_tol), ctypes.byref(nq))
    if rc != 0:
        raise RuntimeError('oracle_get_jk failed')
    if hermi == 2:
        for k in vk:
            iu = numpy.triu_indices(n, 1)
            k[iu] = -k.T[iu]
    return vj.reshape(shape), vk.reshape(shape), nq.value


def int2e_cart(atm, bas, env, shls):
    """Cartesian block (ab|cd) of one shell quartet, Fortran order [i,j,k,l],
    with libcint's 'sp' factors on s and p shells."""
    lib = load()
    atm, bas, env = _arrays(atm, bas, env)
    shls = numpy.asarray(shls, dtype=numpy.int32)
    dims = [((int(bas[s, 1]) + 1) * (int(bas[s, 1]) + 2) // 2) * int(bas[s, 3]) for s in shls]
    out = numpy.zeros(int(numpy.prod(dims)))
    lib.int2e_cart(_p(out), None, _p(shls), _p(atm), ctypes.c_int(atm.shape[0]), _p(bas),
                   ctypes.c_int(bas.shape[0]), _p(env), None, None)
    return out.reshape(dims, order='F')


def grad_q_cond(atm, bas, env, cart=False, direct_scf_tol=1e-14):
    """The two screening planes of grad.rhf.get_jk: (2, nbas, nbas), plane 0
    from int2e_ip1ip2 (CVHFnr_int2e_pp_q_cond), plane 1 from int2e, both under
    mol.with_integral_screen(tol**2) (pyscf/grad/rhf.py:155-169)."""
    lib = load()
    atm, bas, env = _arrays(atm, bas, env)
    nbas = bas.shape[0]
    q = numpy.empty((2, nbas, nbas))
    cut = -numpy.log(direct_scf_tol ** 2)
    lib.oracle_grad_q_cond(_p(q), _p(atm), ctypes.c_int(atm.shape[0]), _p(bas), ctypes.c_int(nbas), _p(env),
                           ctypes.c_int(int(cart)), ctypes.c_double(cut))
    return q


def dm_cond1(dm, bas, cart=False):
    """CVHFnr_dm_cond1: max |D| over each shell block, not symmetrised."""
    lib = load()
    bas = numpy.ascontiguousarray(bas, dtype=numpy.int32)
    dm = numpy.ascontiguousarray(dm, dtype=numpy.double)
    out = numpy.empty((bas.shape[0], bas.shape[0]))
    lib.oracle_dm_cond1(_p(out), _p(dm), ctypes.c_int(1), _p(bas), ctypes.c_int(bas.shape[0]),
                        ctypes.c_int(int(cart)))
    return out


def grad_jk(dm, atm, bas, env, cart=False, direct_scf_tol=1e-14, screen=True):
    """grad.rhf.get_jk restated: (vj, vk), each (3, nao, nao), already negated
    as the reference returns them (pyscf/grad/rhf.py:149-178)."""
    lib = load()
    atm, bas, env = _arrays(atm, bas, env)
    dm = numpy.ascontiguousarray(dm, dtype=numpy.double)
    n = dm.shape[-1]
    vj = numpy.empty((3, n, n))
    vk = numpy.empty((3, n, n))
    qc = dc = None
    if screen:
        qc = grad_q_cond(atm, bas, env, cart, direct_scf_tol)
        dc = dm_cond1(dm, bas, cart)
    rc = lib.oracle_grad_jk(_p(dm), _p(vj), _p(vk), _p(atm), ctypes.c_int(atm.shape[0]), _p(bas),
                            ctypes.c_int(bas.shape[0]), _p(env), ctypes.c_int(int(cart)),
                            _p(qc) if screen else None, _p(dc) if screen else None, ctypes.c_double(direct_scf_tol))
    if rc != 0:
        raise RuntimeError('oracle_grad_jk failed')
    return vj, vk
