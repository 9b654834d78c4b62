"""Drop-in for the direct-SCF entry points of ``pyscf.scf._vhf``.

Same names, arguments and return conventions as PySCF 2.12.1:

* ``direct(dms, atm, bas, env, vhfopt=None, hermi=0, cart=False, with_j=True,
  with_k=True, out=None, optimize_sr=False) -> (vj, vk)``
  (pyscf/scf/_vhf.py:405-464): J = 'ji->s2kl', K = 'li->s2kj' (hermi=1) or
  'li->s1kj' (otherwise), then hermi_triu.  Here the whole build runs in
  libb200jk on the GPU.
* ``VHFOpt`` mirrors ``_VHFOpt(mol, 'int2e', 'CVHFnrs8_prescreen',
  'CVHFnr_int2e_q_cond', 'CVHFnr_dm_cond', direct_scf_tol)`` as created by
  ``SCF.init_direct_scf`` (pyscf/scf/hf.py:2045-2054): it owns the device plan
  (shell pairs, primitive pairs, q_cond).

Errors follow the reference: shape mismatches raise RuntimeError
(pyscf/scf/_vhf.py:594-597); inputs the engine does not implement raise
NotImplementedError; CUDA failures raise lib.B200JKError.
"""
import hashlib

import numpy

from . import lib

_plan_cache = {}
_PLAN_CACHE_MAX = 8


def _key(atm, bas, env, cart, tol, device):
    h = hashlib.sha1()
    for a in (atm, bas, env):
        h.update(numpy.ascontiguousarray(a).tobytes())
    return (h.hexdigest(), bool(cart), float(tol), int(device))


def cached_plan(atm, bas, env, cart=False, direct_scf_tol=0.0, device=0):
    """A Plan for these arrays, reused across calls with the same molecule."""
    k = _key(atm, bas, env, cart, direct_scf_tol, device)
    p = _plan_cache.get(k)
    if p is None:
        if len(_plan_cache) >= _PLAN_CACHE_MAX:
            _plan_cache.pop(next(iter(_plan_cache))).close()
        p = lib.Plan(atm, bas, env, cart=cart, direct_scf_tol=direct_scf_tol, device=device)
        _plan_cache[k] = p
    return p


PTR_RANGE_OMEGA = 8   # pyscf/gto/mole.py:76


def _omega(env):
    env = numpy.asarray(env)
    return float(env[PTR_RANGE_OMEGA]) if env.size > PTR_RANGE_OMEGA else 0.0


def _with_omega(env, omega):
    env = numpy.array(env, dtype=numpy.double, copy=True)
    env[PTR_RANGE_OMEGA] = omega
    return env


class ShortRangePlan:
    """J/K of the short-range operator erfc(w r12)/r12 (env[PTR_RANGE_OMEGA]
    = -w < 0, as mol.with_short_range_coulomb sets it): the full-range build
    minus the long-range erf(w r12)/r12 build, erfc = 1 - erf, each on its own
    device plan with its own Schwarz bounds.  The reference evaluates the
    erfc integrals directly (libcint, through the same CVHFnr_direct_drv,
    pyscf/scf/_vhf.py:611-627 without optimize_sr)."""

    def __init__(self, atm, bas, env, cart=False, direct_scf_tol=1e-13, device=0):
        w = -_omega(env)
        self.full = cached_plan(atm, bas, _with_omega(env, 0.0), cart, direct_scf_tol, device)
        self.lr = cached_plan(atm, bas, _with_omega(env, w), cart, direct_scf_tol, device)
        self.nao, self.nbas = self.full.nao, self.full.nbas
        self.device = self.full.device

    def set_prescreen(self, screen=lib.SCREEN_NRS8):
        self.full.set_prescreen(screen)
        self.lr.set_prescreen(screen)

    def get_jk(self, dms, hermi=1, with_j=True, with_k=True, out_j=None, out_k=None, precision=lib.PREC_FP64,
               stream=None):
        fj, fk = self.full.get_jk(dms, hermi, with_j, with_k, precision=precision)
        lj, lk = self.lr.get_jk(dms, hermi, with_j, with_k, precision=precision)
        vj = vk = None
        if with_j:
            vj = fj - lj
            if out_j is not None:
                out_j[...] = vj.reshape(out_j.shape)
                vj = out_j
        if with_k:
            vk = fk - lk
            if out_k is not None:
                out_k[...] = vk.reshape(out_k.shape)
                vk = out_k
        return vj, vk

    def get_jk_device(self, dms, hermi=1, with_j=True, with_k=True, precision=lib.PREC_FP64):
        fj, fk = self.full.get_jk_device(dms, hermi, with_j, with_k, precision)
        lj, lk = self.lr.get_jk_device(dms, hermi, with_j, with_k, precision)
        return (fj - lj if with_j else None), (fk - lk if with_k else None)

    def int2e_s8(self, device=True):
        eri = self.full.int2e_s8(device)
        eri -= self.lr.int2e_s8(device)
        return eri

    def grad_jk(self, dms, with_j=True, with_k=True, direct_scf_tol=1e-14):
        fj, fk = self.full.grad_jk(dms, with_j, with_k, direct_scf_tol)
        lj, lk = self.lr.grad_jk(dms, with_j, with_k, direct_scf_tol)
        return (fj - lj if with_j else None), (fk - lk if with_k else None)

    def close(self):
        pass


def make_plan(atm, bas, env, cart=False, direct_scf_tol=1e-13, device=0, cached=True):
    """The device plan of a molecule: long range (omega > 0) and full range
    run in the kernels; short range (omega < 0) as full minus long range."""
    if _omega(env) < 0:
        return ShortRangePlan(atm, bas, env, cart, direct_scf_tol, device)
    if cached:
        return cached_plan(atm, bas, env, cart, direct_scf_tol, device)
    return lib.Plan(atm, bas, env, cart=cart, direct_scf_tol=direct_scf_tol, device=device)


class VHFOpt:
    """Direct-SCF optimizer: holds the device plan for one molecule.

    ``mol`` is a PySCF Mole or any object with ``_atm``, ``_bas``, ``_env``
    and ``cart``."""

    def __init__(self, mol, intor='int2e', prescreen='CVHFnrs8_prescreen',
                 qcondname='CVHFnr_int2e_q_cond', dmcondname='CVHFnr_dm_cond',
                 direct_scf_tol=1e-13, device=0):
        if intor not in ('int2e', 'int2e_sph', 'int2e_cart'):
            raise NotImplementedError('VHFOpt supports the int2e Coulomb kernel only, not %s' % intor)
        if prescreen not in _SCREENS and prescreen not in ('CVHFnoscreen', None):
            raise NotImplementedError('prescreen %s is not implemented' % prescreen)
        self.mol = mol
        self._intor = intor
        self._prescreen = prescreen
        self._qcondname = qcondname
        self._dmcondname = dmcondname
        tol = direct_scf_tol if prescreen in _SCREENS else 0.0
        # the molecule's current operator: full, long range (omega > 0) or
        # short range (omega < 0), as SCF.get_jk builds one _VHFOpt per omega
        self.plan = make_plan(mol._atm, mol._bas, mol._env, getattr(mol, 'cart', False), tol, device,
                              cached=False)
        self._arrays = (numpy.array(mol._atm, dtype=numpy.int32), numpy.array(mol._bas, dtype=numpy.int32),
                        numpy.array(mol._env, dtype=numpy.double), bool(getattr(mol, 'cart', False)))
        self._direct_scf_tol = direct_scf_tol

    @property
    def direct_scf_tol(self):
        return self._direct_scf_tol

    @property
    def prescreen(self):
        """Name of the per-quartet screen (the reference's _VHFOpt.prescreen,
        pyscf/scf/_vhf.py:219-226).  SCF.get_jk swaps in the J-only or K-only
        screen with lib.temporary_env when only one of J, K is built
        (pyscf/scf/hf.py:2069-2077); each build uses the current value."""
        return self._prescreen

    @prescreen.setter
    def prescreen(self, v):
        if v not in _SCREENS:
            if self._prescreen in (None, 'CVHFnoscreen') and v in (None, 'CVHFnoscreen'):
                self._prescreen = v
                return
            raise NotImplementedError('prescreen %s is not implemented' % v)
        if self._prescreen in (None, 'CVHFnoscreen'):
            raise NotImplementedError('an unscreened VHFOpt cannot switch to %s' % v)
        self._prescreen = v

    @property
    def q_cond(self):
        return self.plan.q_cond

    def matches(self, atm, bas, env, cart):
        a, b, e, c = self._arrays
        return (a.shape == numpy.shape(atm) and b.shape == numpy.shape(bas) and numpy.array_equal(a, atm)
                and numpy.array_equal(b, bas) and e.shape == numpy.shape(env) and numpy.array_equal(e, env)
                and c == bool(cart))


# the reference's per-quartet screens and the engine's modes for them
_SCREENS = {'CVHFnrs8_prescreen': lib.SCREEN_NRS8, 'CVHFnrs8_vj_prescreen': lib.SCREEN_VJ,
            'CVHFnrs8_vk_prescreen': lib.SCREEN_VK}


def _resolve_plan(vhfopt, atm, bas, env, cart):
    if isinstance(vhfopt, VHFOpt) and vhfopt.matches(atm, bas, env, cart):
        vhfopt.plan.set_prescreen(_SCREENS.get(vhfopt.prescreen, lib.SCREEN_NRS8))
        return vhfopt.plan
    if vhfopt is None:
        # the reference runs CVHFnr_direct_drv without any screening here
        return make_plan(atm, bas, env, cart, 0.0)
    tol = getattr(vhfopt, 'direct_scf_tol', 1e-13)
    plan = make_plan(atm, bas, env, cart, tol)
    plan.set_prescreen(_SCREENS.get(getattr(vhfopt, 'prescreen', None), lib.SCREEN_NRS8))
    return plan


def direct(dms, atm, bas, env, vhfopt=None, hermi=0, cart=False,
           with_j=True, with_k=True, out=None, optimize_sr=False):
    """J and K of one or several densities (pyscf/scf/_vhf.py:405-464);
    env[PTR_RANGE_OMEGA] selects the operator as in the reference (0 full,
    > 0 erf(w r)/r, < 0 erfc(|w| r)/r)."""
    try:
        import torch
        is_torch = isinstance(dms, torch.Tensor)
    except ImportError:
        is_torch = False
    if not with_j and not with_k:
        return None, None
    if is_torch and dms.is_cuda:
        plan = _resolve_plan(vhfopt, atm, bas, env, cart)
        return plan.get_jk_device(dms.to(torch.float64), hermi=hermi, with_j=with_j, with_k=with_k)
    dms = numpy.asarray(dms, order='C', dtype=numpy.double)
    dms_shape = dms.shape
    nao = dms_shape[-1]
    dms = dms.reshape(-1, nao, nao)
    plan = _resolve_plan(vhfopt, atm, bas, env, cart)
    if plan.nao != nao:
        raise RuntimeError('dm shape %s is inconsistent with nao=%d of the basis' % (dms_shape, plan.nao))
    n_dm = dms.shape[0]
    out_j = out_k = None
    if out is not None:
        out = numpy.asarray(out)
        n_jk = int(bool(with_j)) + int(bool(with_k))
        if out.shape != (n_jk * n_dm, nao, nao) or out.dtype != numpy.double or not out.flags.c_contiguous:
            raise RuntimeError('out must be a C-contiguous float64 array of shape %s'
                               % ((n_jk * n_dm, nao, nao),))
        if with_j:
            out_j = out[:n_dm]
        if with_k:
            out_k = out[n_dm:] if with_j else out[:n_dm]
    vj, vk = plan.get_jk(dms, hermi=hermi, with_j=with_j, with_k=with_k, out_j=out_j, out_k=out_k)
    if with_j:
        vj = vj.reshape(dms_shape)
    if with_k:
        vk = vk.reshape(dms_shape)
    return vj, vk
