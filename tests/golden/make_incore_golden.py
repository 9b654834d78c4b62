"""Reference s8 integral tensors and in-core J/K for tests/test_gpu_incore.py.

Runs only where the reference checkout is readable (this container): it
imports the unmodified PySCF Python package from the reference tree on the
reference's C drivers compiled by oracle/build.py against the oracle
integral library (as make_golden.py does).  For the molecules of
mol_h2o_631g.npz, mol_h2o2_vtz.npz and mol_h2o8_vdz.npz (same atm/bas/env):

  * eri = mol.intor('int2e', aosym='s8')   (GTO2e_cart_or_sph,
    pyscf/lib/vhf/fill_nr_s8.c:110-138): stored whole for H2O/6-31G; for the
    larger ones PySCF's fingerprint lib.fp(eri), the number of exact zeros
    (quartets under the Schwarz cutoff), the largest entry and 20000 entries
    at seeded random positions (numpy.random.default_rng(7));
  * scf.hf.dot_eri_dm(eri, dm, hermi) -> _vhf.incore (pyscf/scf/_vhf.py:
    318-401) for the fixture's dm_rand (hermi=1), dm_ns (hermi=0) and
    dm_anti = (dm_ns - dm_ns^T)/2 (hermi=2); for H2O/6-31G also from the s4
    tensor ao2mo.restore(4, eri, nao);
  * make_variants(): H2O/cc-pVDZ in the Cartesian basis and under the erf
    and erfc operators (incore_h2o_vdz_variants.npz).

    OMP_NUM_THREADS=8 python tests/golden/make_incore_golden.py
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

from pyscf import gto, scf, lib, ao2mo  # noqa: E402

NAMES = ('h2o_631g', 'h2o2_vtz', 'h2o8_vdz')
NSAMPLE = 20000


def mol_of(f):
    mol = gto.Mole()
    mol._atm = numpy.asarray(f['atm'], dtype=numpy.int32)
    mol._bas = numpy.asarray(f['bas'], dtype=numpy.int32)
    mol._env = numpy.asarray(f['env'], dtype=numpy.double)
    mol.cart = bool(f['cart'])
    mol._built = True
    return mol


def make(name):
    t0 = time.time()
    f = dict(numpy.load(os.path.join(HERE, 'mol_%s.npz' % name)))
    mol = mol_of(f)
    nao = mol.nao_nr()
    eri = mol.intor('int2e', aosym='s8')
    t_fill = time.time() - t0
    dm_rand, dm_ns = f['dm_rand'], f['dm_ns']
    dm_anti = (dm_ns - dm_ns.T) * 0.5
    out = {'nao': numpy.int32(nao), 'eri_fp': lib.fp(eri), 'eri_nzero': numpy.int64((eri == 0).sum()),
           'eri_max': float(abs(eri).max()), 'eri_size': numpy.int64(eri.size)}
    if eri.size <= 10000:
        out['eri'] = eri
    rng = numpy.random.default_rng(7)
    idx = rng.integers(0, eri.size, NSAMPLE)
    out['sample_idx'] = idx
    out['sample_val'] = eri[idx]
    t1 = time.time()
    for tag, dm, hermi in (('rand', dm_rand, 1), ('ns', dm_ns, 0), ('anti', dm_anti, 2)):
        vj, vk = scf.hf.dot_eri_dm(eri, dm, hermi)
        out['vj_%s' % tag] = vj
        out['vk_%s' % tag] = vk
    t_jk = (time.time() - t1) / 3
    if eri.size <= 10000:
        eri4 = ao2mo.restore(4, eri, nao)
        for tag, dm, hermi in (('rand', dm_rand, 1), ('ns', dm_ns, 0), ('anti', dm_anti, 2)):
            vj, vk = scf.hf.dot_eri_dm(eri4, dm, hermi)
            out['s4_vj_%s' % tag] = vj
            out['s4_vk_%s' % tag] = vk
    out['dm_anti'] = dm_anti
    path = os.path.join(HERE, 'incore_%s.npz' % name)
    numpy.savez_compressed(path, **out)
    print('%-10s nao=%4d s8 %d entries (%d zero), fill %.1fs, J/K %.2fs -> %s'
          % (name, nao, eri.size, out['eri_nzero'], t_fill, t_jk, path), flush=True)


def make_variants():
    """H2O/cc-pVDZ (d shells): the whole s8 tensor of the spherical and of
    the Cartesian basis (int2e_cart), and of the spherical basis under
    env[PTR_RANGE_OMEGA] = 0.5 (erf, long range) and -0.5 (erfc, short
    range), as mol.intor('int2e', aosym='s8') returns them; with the in-core
    J/K (hermi=1) of a symmetric density of U(-1, 1) entries
    (numpy.random.default_rng(11)).  Written to incore_h2o_vdz_variants.npz."""
    f = dict(numpy.load(os.path.join(HERE, 'mol_h2o_vdz.npz')))
    out = {}
    for tag, cart, omega in (('full', False, 0.0), ('cart', True, 0.0), ('lr', False, 0.5), ('sr', False, -0.5)):
        g = dict(f)
        g['cart'] = numpy.int32(cart)
        env = numpy.array(f['env'], dtype=numpy.double)
        env[8] = omega   # PTR_RANGE_OMEGA (pyscf/gto/mole.py:76)
        g['env'] = env
        mol = mol_of(g)
        nao = mol.nao_nr()
        eri = mol.intor('int2e', aosym='s8')
        rng = numpy.random.default_rng(11)
        a = rng.uniform(-1, 1, (nao, nao))
        dm = (a + a.T) * 0.5
        vj, vk = scf.hf.dot_eri_dm(eri, dm, 1)
        out.update({'%s_eri' % tag: eri, '%s_env' % tag: env, '%s_dm' % tag: dm, '%s_vj' % tag: vj,
                    '%s_vk' % tag: vk, '%s_nao' % tag: numpy.int32(nao)})
        print(tag, nao, eri.size, flush=True)
    numpy.savez_compressed(os.path.join(HERE, 'incore_h2o_vdz_variants.npz'), **out)


if __name__ == '__main__':
    for n in (sys.argv[1:] or NAMES + ('variants',)):
        if n == 'variants':
            make_variants()
        else:
            make(n)
