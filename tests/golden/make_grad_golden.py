"""Generate the gradient fixtures tests/golden/grad_*.npz from the reference.

Like make_golden.py, this runs only where the reference checkout is readable:
it imports the unmodified PySCF 2.12.1 package on top of the reference's own
C drivers compiled by oracle/build.py against the oracle integral library.

For each molecule it stores
  * atm/bas/env and the converged RHF density dm0 (direct SCF, max_memory=0);
  * gq_cond: the two screening planes grad.rhf.get_jk builds
    (CVHFnr_int2e_pp_q_cond over int2e_ip1ip2, CVHFnr_int2e_q_cond over int2e;
    pyscf/grad/rhf.py:149-178);
  * gvj/gvk: grad.rhf.get_jk(mol, D) for D = dm0 and, where listed, for a
    seeded non-symmetric density (gvj_ns/gvk_ns), each (3, nao, nao);
  * de: grad.RHF(mf).kernel() (pyscf/grad/rhf.py:33-76) and de_2e, its
    two-electron part  2 sum_x einsum(vhf[:, p0:p1], dm0[p0:p1])  with
    vhf = vj - vk/2 (grad_elec, pyscf/grad/rhf.py:67-69), so that
    de - de_2e is the one-electron part the GPU does not compute;
  * aoslice: the AO range of every atom;
  * for a seeded subset of coordinates: RHF energies at +-h Bohr (conv_tol
    1e-12, started from dm0).

    python tests/golden/make_grad_golden.py [names...]
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

from pyscf import gto, scf, grad  # noqa: E402
from pyscf.grad import rhf as grad_rhf  # noqa: E402
import geometry  # noqa: E402

# name -> (store vj/vk, store a non-symmetric case, number of FD coordinates)
CASES = {
    'h2o_631g': (True, True, 9),
    'h2o2_vtz': (True, False, 0),
    'h2o16_vdz': (False, False, 12),
}
FD_H = 1e-4          # Bohr
FD_SEED = 506


def build_mol(name, coords_bohr=None):
    atoms, basis = geometry.workloads()[name]
    if coords_bohr is None:
        return gto.M(atom=[(s, tuple(float(x) for x in r)) for s, r in atoms], basis=basis, verbose=0)
    return gto.M(atom=[(s, tuple(float(x) for x in r)) for (s, _), r in zip(atoms, coords_bohr)],
                 basis=basis, unit='Bohr', verbose=0)


def grad_q_cond(mol):
    """The two planes of grad.rhf.get_jk's screening (pyscf/grad/rhf.py:155-169)."""
    import ctypes
    from pyscf.scf import _vhf
    from pyscf import lib
    libcvhf = _vhf.libcvhf
    ao_loc = mol.ao_loc_nr()
    nbas = mol.nbas
    q = numpy.empty((2, nbas, nbas))
    with mol.with_integral_screen(1e-14 ** 2):
        libcvhf.CVHFnr_int2e_pp_q_cond(getattr(libcvhf, mol._add_suffix('int2e_ip1ip2')), lib.c_null_ptr(),
                                       q[0].ctypes, ao_loc.ctypes, mol._atm.ctypes, ctypes.c_int(mol.natm),
                                       mol._bas.ctypes, ctypes.c_int(nbas), mol._env.ctypes)
        libcvhf.CVHFnr_int2e_q_cond(getattr(libcvhf, mol._add_suffix('int2e')), lib.c_null_ptr(),
                                    q[1].ctypes, ao_loc.ctypes, mol._atm.ctypes, ctypes.c_int(mol.natm),
                                    mol._bas.ctypes, ctypes.c_int(nbas), mol._env.ctypes)
    return q


def rhf(mol, conv_tol, dm_init=None):
    mf = scf.RHF(mol)
    mf.max_memory = 0
    mf.conv_tol = conv_tol
    mf.max_cycle = 200
    e = mf.kernel(dm0=dm_init)
    assert mf.converged
    return mf, e


def make(name):
    t0 = time.time()
    store_jk, store_ns, nfd = CASES[name]
    mol = build_mol(name)
    mf, e = rhf(mol, 1e-12)
    dm0 = mf.make_rdm1()
    vj, vk = grad_rhf.get_jk(mol, dm0)
    vhf = vj - 0.5 * vk
    aoslice = mol.aoslice_by_atom()[:, 2:4].astype(numpy.int32)
    de_2e = numpy.array([2 * numpy.einsum('xij,ij->x', vhf[:, p0:p1], dm0[p0:p1]) for p0, p1 in aoslice])
    de = grad.RHF(mf).kernel()
    out = dict(atm=mol._atm, bas=mol._bas, env=mol._env, cart=numpy.int32(mol.cart), nao=numpy.int32(mol.nao),
               nelec=numpy.int32(mol.nelectron), e_rhf=e, dm0=dm0, gq_cond=grad_q_cond(mol),
               de=de, de_2e=de_2e, aoslice=aoslice, coords=mol.atom_coords())
    if store_jk:
        out.update(gvj=vj, gvk=vk)
    if store_ns:
        rng = numpy.random.default_rng(4321)
        dm_ns = rng.uniform(-1, 1, (mol.nao, mol.nao))
        vjn, vkn = grad_rhf.get_jk(mol, dm_ns)
        out.update(dm_ns=dm_ns, gvj_ns=vjn, gvk_ns=vkn)
    if nfd:
        rng = numpy.random.default_rng(FD_SEED)
        picks = rng.choice(3 * mol.natm, size=min(nfd, 3 * mol.natm), replace=False)
        c0 = mol.atom_coords()
        efd = numpy.empty((len(picks), 2))
        for n, t in enumerate(picks):
            for s, sign in enumerate((1, -1)):
                c = c0.copy()
                c[t // 3, t % 3] += sign * FD_H
                _, efd[n, s] = rhf(build_mol(name, c), 1e-12, dm0)
        out.update(fd_coords=picks.astype(numpy.int32), fd_energies=efd, fd_h=FD_H)
    path = os.path.join(HERE, 'grad_%s.npz' % name)
    numpy.savez_compressed(path, **out)
    print('%-12s nao=%4d natm=%3d  %.1fs -> %s' % (name, mol.nao, mol.natm, time.time() - t0, path))


if __name__ == '__main__':
    for n in sys.argv[1:] or list(CASES):
        make(n)
