"""Call the reference's own direct-SCF C driver without importing PySCF.

ORACLE / TEST INFRASTRUCTURE: the timed CPU baseline (bench.py) and tests use
it; the product never does.

oracle/_ref/pyext/pyscf/lib/libcvhf.so is PySCF's libcvhf compiled from the
reference sources (oracle/build.py) on the oracle integral library.  This
module repeats, with ctypes, what pyscf.scf._vhf does around it:
  * _VHFOpt(mol, 'int2e', 'CVHFnrs8_prescreen', 'CVHFnr_int2e_q_cond',
    'CVHFnr_dm_cond', tol): the _CVHFOpt structure (pyscf/scf/_vhf.py:302-310),
    q_cond from CVHFnr_int2e_q_cond under env[PTR_EXPCUTOFF] = -log(tol^2)
    (pyscf/scf/_vhf.py:184-206, gto/mole.py:3055-3068), dm_cond from
    CVHFnr_dm_cond (pyscf/scf/_vhf.py:208-230);
  * direct(): jkscripts 'ji->s2kl' and 'li->s2kj' (hermi=1) / 'li->s1kj',
    nr_direct_drv -> CVHFnr_direct_drv(int2e_sph, CVHFdot_nrs8, ...)
    (pyscf/scf/_vhf.py:405-464, 540-639), then hermi_triu on J (and K when
    hermi != 0) (pyscf/lib/numpy_helper.py:480).
"""
import ctypes
import os

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, '_ref', 'pyext', 'pyscf', 'lib')
PTR_EXPCUTOFF = 0

_libs = {}


def available():
    return os.path.exists(os.path.join(LIBDIR, 'libcvhf.so'))


def _load():
    if 'cvhf' not in _libs:
        if not available():
            raise RuntimeError('oracle/_ref is not built (needs the reference sources; see oracle/build.py)')
        # dependencies resolve through the libraries' $ORIGIN rpath
        _libs['cvhf'] = ctypes.CDLL(os.path.join(LIBDIR, 'libcvhf.so'))
    return _libs['cvhf']


class _CVHFOpt(ctypes.Structure):
    _fields_ = [('nbas', ctypes.c_int), ('ngrids', ctypes.c_int), ('direct_scf_tol', ctypes.c_double),
                ('q_cond', ctypes.c_void_p), ('dm_cond', ctypes.c_void_p),
                ('fprescreen', ctypes.c_void_p), ('r_vkscreen', ctypes.c_void_p)]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _fptr(lib, name):
    return ctypes.cast(getattr(lib, name), ctypes.c_void_p)


def ao_loc_nr(bas, cart=False):
    bas = numpy.asarray(bas)
    l = bas[:, 1]
    nf = (l + 1) * (l + 2) // 2 if cart else 2 * l + 1
    return numpy.concatenate([[0], numpy.cumsum(nf * bas[:, 3])]).astype(numpy.int32)


class RefVHFOpt:
    """The reference's _VHFOpt for int2e with the s8 prescreen."""

    def __init__(self, atm, bas, env, direct_scf_tol=1e-13, cart=False):
        lib = _load()
        self.atm = numpy.ascontiguousarray(atm, dtype=numpy.int32)
        self.bas = numpy.ascontiguousarray(bas, dtype=numpy.int32)
        self.env = numpy.array(env, dtype=numpy.double, order='C', copy=True)
        self.cart = cart
        self.intor = 'int2e_cart' if cart else 'int2e_sph'
        self.ao_loc = ao_loc_nr(self.bas, cart)
        nbas = self.bas.shape[0]
        self.q_cond = numpy.empty((nbas, nbas))
        saved = self.env[PTR_EXPCUTOFF]
        self.env[PTR_EXPCUTOFF] = abs(numpy.log(direct_scf_tol ** 2))
        lib.CVHFnr_int2e_q_cond(getattr(lib, self.intor), None, _p(self.q_cond), _p(self.ao_loc),
                                _p(self.atm), ctypes.c_int(self.atm.shape[0]), _p(self.bas),
                                ctypes.c_int(nbas), _p(self.env))
        self.env[PTR_EXPCUTOFF] = saved
        self.opt = _CVHFOpt()
        self.opt.nbas = nbas
        self.opt.direct_scf_tol = direct_scf_tol
        self.opt.fprescreen = _fptr(lib, 'CVHFnrs8_prescreen')
        self.opt.r_vkscreen = _fptr(lib, 'CVHFr_vknoscreen')
        self.opt.q_cond = self.q_cond.ctypes.data
        self.dm_cond = None

    def set_dm(self, dms):
        lib = _load()
        nbas = self.bas.shape[0]
        self.dm_cond = numpy.empty((nbas, nbas))
        lib.CVHFnr_dm_cond(_p(self.dm_cond), _p(dms), ctypes.c_int(dms.shape[0]), _p(self.ao_loc),
                           _p(self.atm), ctypes.c_int(self.atm.shape[0]), _p(self.bas),
                           ctypes.c_int(nbas), _p(self.env))
        self.opt.dm_cond = self.dm_cond.ctypes.data


def _hermi_triu(m, hermi):
    n = m.shape[0]
    iu = numpy.triu_indices(n, 1)
    if hermi == 2:
        m[iu] = -m.T[iu]
    else:
        m[iu] = m.T[iu]


def direct(dms, vhfopt, hermi=1, with_j=True, with_k=True):
    """The reference J/K (pyscf/scf/_vhf.py:405-464) with the given RefVHFOpt."""
    lib = _load()
    dms = numpy.ascontiguousarray(dms, dtype=numpy.double)
    shape = dms.shape
    nao = shape[-1]
    dms = dms.reshape(-1, nao, nao)
    n_dm = dms.shape[0]
    vhfopt.set_dm(dms)
    scripts = []
    if with_j:
        scripts += ['nrs8_ji_s2kl'] * n_dm
    if with_k:
        scripts += (['nrs8_li_s2kj'] if hermi == 1 else ['nrs8_li_s1kj']) * n_dm
    nd = len(scripts)
    dm_list = [dms[i % n_dm] for i in range(nd)]
    out = numpy.empty((nd, nao, nao))
    fjk = (ctypes.c_void_p * nd)(*[_fptr(lib, 'CVHF' + s).value for s in scripts])
    dmsptr = (ctypes.c_void_p * nd)(*[d.ctypes.data for d in dm_list])
    vjkptr = (ctypes.c_void_p * nd)(*[out[i].ctypes.data for i in range(nd)])
    nbas = vhfopt.bas.shape[0]
    shls_slice = (ctypes.c_int * 8)(*([0, nbas] * 4))
    lib.CVHFnr_direct_drv(getattr(lib, vhfopt.intor), getattr(lib, 'CVHFdot_nrs8'), fjk, dmsptr, vjkptr,
                          ctypes.c_int(nd), ctypes.c_int(1), shls_slice, _p(vhfopt.ao_loc), None,
                          ctypes.byref(vhfopt.opt), _p(vhfopt.atm), ctypes.c_int(vhfopt.atm.shape[0]),
                          _p(vhfopt.bas), ctypes.c_int(nbas), _p(vhfopt.env))
    vj = vk = None
    if with_j:
        vj = out[:n_dm]
        for m in vj:
            _hermi_triu(m, 1)
        vj = vj.reshape(shape)
    if with_k:
        vk = out[n_dm:] if with_j else out
        if hermi != 0:
            for m in vk:
                _hermi_triu(m, hermi)
        vk = vk.reshape(shape)
    return vj, vk
