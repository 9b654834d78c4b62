"""Generate the golden fixtures of tests/golden from the reference.

Runs only where the reference checkout is readable (this container): it
imports the unmodified PySCF 2.12.1 Python package from the reference tree,
on top of the reference's own C drivers (libcvhf/libcgto/libnp_helper)
compiled by oracle/build.py against the oracle integral library (upstream
libcint v6.1.3 is not available; see oracle/build.py).  The GPU box never
runs this script; it only reads the .npz files it writes.

For every workload of geometry.workloads() it stores PySCF's own
atm/bas/env arrays; for the small ones also
  * dm_rand  a seeded random symmetric density, with the reference J/K through
             scf.hf.get_jk(mol, dm, hermi=1, vhfopt=mf.init_direct_scf())
             (screened, direct_scf_tol=1e-13) and through _vhf.direct(...,
             vhfopt=None) (unscreened), and a non-symmetric density with hermi=0;
  * the converged RHF density and energy (max_memory=0, i.e. the direct path,
    as pyscf/scf/test/test_h2o_vdz.py:94-98), hcore and overlap, so that an
    SCF can be replayed on the GPU box without PySCF;
and for the SCF_ONLY workloads (C20H42/cc-pVDZ) the RHF energy, hcore and
overlap only.

    python tests/golden/make_golden.py [names...]
"""
import os
import sys
import time

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from oracle import build as oracle_build  # noqa: E402

oracle_build.build_all()
_env = oracle_build.reference_env()
for k in ('PYSCF_EXT_PATH', 'PYSCF_CONFIG_FILE'):
    os.environ[k] = _env[k]
for p in reversed(_env['PYTHONPATH'].split(':')):
    if p and p not in sys.path:
        sys.path.insert(0, p)

from pyscf import gto, scf, lib  # noqa: E402
from pyscf.scf import _vhf  # noqa: E402
import geometry  # noqa: E402

SMALL = ('h2o_631g', 'h2o_vdz', 'h2o2_vtz', 'h2o8_vdz')
# workloads that get an SCF replay (energy, hcore, overlap) but no J/K matrices
SCF_ONLY = ('c20h42_vdz',)
SCF_TOL = {'h2o_631g': 1e-11, 'h2o_vdz': 1e-11, 'h2o2_vtz': 1e-10, 'h2o8_vdz': 1e-10, 'c20h42_vdz': 1e-10}


def build_mol(name):
    atoms, basis = geometry.workloads()[name]
    return gto.M(atom=[(s, tuple(float(x) for x in r)) for s, r in atoms], basis=basis, verbose=0)


def make(name):
    t0 = time.time()
    mol = build_mol(name)
    out = dict(atm=mol._atm, bas=mol._bas, env=mol._env, cart=numpy.int32(mol.cart),
               nelec=numpy.int32(mol.nelectron), nao=numpy.int32(mol.nao), e_nuc=mol.energy_nuc())
    if name in SMALL:
        nao = mol.nao
        rng = numpy.random.default_rng(1234)
        a = rng.uniform(-1, 1, (nao, nao))
        dm_rand = (a + a.T) * 0.5
        dm_ns = rng.uniform(-1, 1, (nao, nao))
        mf = scf.RHF(mol)
        mf.max_memory = 0
        mf.conv_tol = SCF_TOL[name]
        e = mf.kernel()
        assert mf.converged
        opt = mf.init_direct_scf()
        vj, vk = scf.hf.get_jk(mol, dm_rand, hermi=1, vhfopt=opt)
        vj0, vk0 = _vhf.direct(dm_rand, mol._atm, mol._bas, mol._env, None, hermi=1)
        vjn, vkn = scf.hf.get_jk(mol, dm_ns, hermi=0, vhfopt=opt)
        dm_conv = mf.make_rdm1()
        vjc, vkc = scf.hf.get_jk(mol, dm_conv, hermi=1, vhfopt=opt)
        out.update(dm_rand=dm_rand, vj_rand=vj, vk_rand=vk, vj_rand_noscreen=vj0, vk_rand_noscreen=vk0,
                   dm_ns=dm_ns, vj_ns=vjn, vk_ns=vkn, dm_conv=dm_conv, vj_conv=vjc, vk_conv=vkc,
                   e_rhf=e, hcore=mf.get_hcore(), ovlp=mf.get_ovlp(), q_cond=opt.q_cond,
                   scf_conv_tol=SCF_TOL[name])
    if name in SCF_ONLY:
        mf = scf.RHF(mol)
        mf.max_memory = 0
        mf.conv_tol = SCF_TOL[name]
        e = mf.kernel()
        assert mf.converged
        out.update(e_rhf=e, hcore=mf.get_hcore(), ovlp=mf.get_ovlp(), scf_conv_tol=SCF_TOL[name])
    path = os.path.join(HERE, 'mol_%s.npz' % name)
    numpy.savez_compressed(path, **out)
    print('%-12s nao=%4d nbas=%4d  %.1fs -> %s' % (name, mol.nao, mol.nbas, time.time() - t0, path))


if __name__ == '__main__':
    names = sys.argv[1:] or list(geometry.workloads())
    for n in names:
        make(n)
