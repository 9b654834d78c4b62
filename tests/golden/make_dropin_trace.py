"""Record every J/K call an unmodified PySCF run makes, with the reference's answers.

Runs only where the reference checkout is readable (this container): the
unmodified PySCF 2.12.1 package from the reference tree on the reference's own
C drivers (oracle/build.py).  It runs, with nothing patched,

    mf = scf.RHF(mol); mf.max_memory = 0; mf.kernel()      (direct SCF, as
        pyscf/scf/test/test_h2o_vdz.py:94-98)
    mf.get_j(); mf.get_k()                                  (J-only and K-only
        builds: SCF.get_jk switches to CVHFnrs8_vj/vk_prescreen,
        pyscf/scf/hf.py:2069-2077)
    grad.RHF(mf).kernel()                                   (pyscf/grad/rhf.py)

and wraps the two functions those runs reach through module lookups --
pyscf.scf._vhf.direct (looked up by hf.get_jk, pyscf/scf/hf.py:1007) and
pyscf.grad.rhf.get_jk (looked up by GradientsBase.get_jk,
pyscf/grad/rhf.py:321) -- with recorders that store each call's arguments
(density, hermi, with_j, with_k, the vhfopt's prescreen) and the reference's
own result.  tests/test_gpu_dropin_replay.py replays the calls through
pyscf_b200's drop-ins on the GPU, where PySCF itself cannot be imported.

    python tests/golden/make_dropin_trace.py
"""
import os
import sys

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build as oracle_build  # noqa: E402

oracle_build.build_all()
_env = oracle_build.reference_env()
for k in ('PYSCF_EXT_PATH', 'PYSCF_CONFIG_FILE'):
    os.environ[k] = _env[k]
for p in reversed(_env['PYTHONPATH'].split(':')):
    if p and p not in sys.path:
        sys.path.insert(0, p)

from pyscf import gto, scf, grad  # noqa: E402
import pyscf.scf._vhf as ref_vhf  # noqa: E402
import pyscf.grad.rhf as ref_grad  # noqa: E402

SCREENS = ('CVHFnrs8_prescreen', 'CVHFnrs8_vj_prescreen', 'CVHFnrs8_vk_prescreen', 'CVHFnoscreen')


def screen_name(vhfopt):
    if vhfopt is None:
        return 'none'
    ptr = ctypes_addr(vhfopt.prescreen)
    for s in SCREENS:
        if ptr == ctypes_addr(ref_vhf._fpointer(s)):
            return s
    return 'other'


def ctypes_addr(f):
    import ctypes
    return ctypes.cast(f, ctypes.c_void_p).value


def main():
    mol = gto.M(atom='O 0 0 0; H 0 -0.757 0.587; H 0 0.757 0.587', basis='cc-pvdz', verbose=0)
    calls = []
    direct0, gjk0 = ref_vhf.direct, ref_grad.get_jk

    def direct_rec(dms, atm, bas, env, vhfopt=None, hermi=0, cart=False, with_j=True, with_k=True, out=None,
                   optimize_sr=False):
        vj, vk = direct0(dms, atm, bas, env, vhfopt, hermi, cart, with_j, with_k, out, optimize_sr)
        calls.append(dict(kind='jk', dm=numpy.array(dms, copy=True), hermi=hermi, with_j=bool(with_j),
                          with_k=bool(with_k), screen=screen_name(vhfopt),
                          vj=None if vj is None else numpy.array(vj, copy=True),
                          vk=None if vk is None else numpy.array(vk, copy=True)))
        return vj, vk

    def gjk_rec(mol_, dm):
        vj, vk = gjk0(mol_, dm)
        calls.append(dict(kind='grad', dm=numpy.array(dm, copy=True), vj=numpy.array(vj), vk=numpy.array(vk)))
        return vj, vk

    ref_vhf.direct, ref_grad.get_jk = direct_rec, gjk_rec
    try:
        mf = scf.RHF(mol)
        mf.max_memory = 0
        mf.conv_tol = 1e-11
        e = mf.kernel()
        assert mf.converged
        n_scf = len(calls)
        dm = mf.make_rdm1()
        mf.get_j(mol, dm)
        mf.get_k(mol, dm)
        g = grad.RHF(mf).kernel()
    finally:
        ref_vhf.direct, ref_grad.get_jk = direct0, gjk0
    out = dict(atm=mol._atm, bas=mol._bas, env=mol._env, cart=numpy.int32(mol.cart), e_rhf=e, grad=g,
               e_nuc=mol.energy_nuc(), hcore=mf.get_hcore(), dm_final=dm, n_scf_calls=n_scf,
               ncalls=len(calls))
    for i, c in enumerate(calls):
        for k, v in c.items():
            if v is None:
                continue
            out['c%02d_%s' % (i, k)] = numpy.asarray(v)
    path = os.path.join(HERE, 'dropin_trace_h2o_vdz.npz')
    numpy.savez_compressed(path, **out)
    print('%d calls (%d during the SCF), E = %.12f -> %s' % (len(calls), n_scf, e, path))
    for i, c in enumerate(calls):
        print(i, c['kind'], c.get('screen', ''), c.get('hermi', ''), c.get('with_j', ''), c.get('with_k', ''),
              c['dm'].shape)


if __name__ == '__main__':
    main()
