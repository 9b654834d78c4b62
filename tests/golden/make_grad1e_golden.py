"""One-electron part of the reference's RHF nuclear gradient, for the fixtures
grad_h2o_631g.npz, grad_h2o2_vtz.npz and grad_h2o16_vdz.npz.

Runs only where the reference checkout is readable (this container), on the
unmodified PySCF package over the reference's C drivers compiled by
oracle/build.py (as make_grad_golden.py).  For each fixture, with its
atm/bas/env and converged density dm0:
  * dme0 = 1/2 dm0 F dm0, F = mf.get_fock(dm=dm0): the energy-weighted
    density make_rdm1e builds from the orbitals, 2 C_occ e_occ C_occ^T, at
    convergence (F C = S C e);
  * de_1e: the one-electron lines of grad_elec (pyscf/grad/rhf.py:57-66),
    de[k] += einsum('xij,ij->x', hcore_deriv(k), dm0)  (hcore_generator,
    :121-143: int1e_ipkin + int1e_ipnuc and int1e_iprinv at every nucleus)
    de[k] -= 2 einsum('xij,ij->x', s1[:, p0:p1], dme0[p0:p1])  (get_ovlp,
    :145-146: -int1e_ipovlp);
  * de_nuc = grad_nuc(mol) (:86-107).
Written to grad1e_<name>.npz.

    python tests/golden/make_grad1e_golden.py
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

from pyscf import gto, scf  # noqa: E402
from pyscf.grad import rhf as grad_rhf  # noqa: E402

NAMES = ('h2o_631g', 'h2o2_vtz', 'h2o16_vdz')


def mol_of(f):
    mol = gto.Mole()
    mol._atm = numpy.asarray(f['atm'], dtype=numpy.int32)
    mol._bas = numpy.asarray(f['bas'], dtype=numpy.int32)
    mol._env = numpy.asarray(f['env'], dtype=numpy.double)
    mol.cart = bool(f['cart'])
    mol._built = True
    return mol


def make(name):
    f = dict(numpy.load(os.path.join(HERE, 'grad_%s.npz' % name)))
    mol = mol_of(f)
    mf = scf.RHF(mol)
    mf.max_memory = 0
    dm0 = f['dm0']
    fock = mf.get_fock(dm=dm0)
    dme0 = 0.5 * dm0 @ fock @ dm0
    g = grad_rhf.Gradients(mf)
    hcore_deriv = grad_rhf.hcore_generator(g, mol)
    s1 = grad_rhf.get_ovlp(mol)
    aoslices = mol.aoslice_by_atom()
    de = numpy.zeros((mol.natm, 3))
    for k in range(mol.natm):
        p0, p1 = aoslices[k, 2:]
        de[k] += numpy.einsum('xij,ij->x', hcore_deriv(k), dm0)
        de[k] -= numpy.einsum('xij,ij->x', s1[:, p0:p1], dme0[p0:p1]) * 2
    out = dict(dme0=dme0, de_1e=de, de_nuc=grad_rhf.grad_nuc(mol))
    path = os.path.join(HERE, 'grad1e_%s.npz' % name)
    numpy.savez_compressed(path, **out)
    total = de + f['de_2e'] + out['de_nuc']
    print('%-10s natm=%3d  |de_1e + de_2e + de_nuc - de| = %.2e -> %s'
          % (name, mol.natm, abs(total - f['de']).max(), path), flush=True)


if __name__ == '__main__':
    for n in (sys.argv[1:] or NAMES):
        make(n)
