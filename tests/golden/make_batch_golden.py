"""Generate tests/golden/batch_h2o_vdz512.npz: the batched-molecule workload.

512 water clusters (H2O)_n, n uniform in [1, 16] (numpy default_rng(404)),
each on n sites drawn without replacement from a 3x3x2 cubic lattice (3.0 A
spacing) with the rigid monomer, seeded random rotations and +-0.2 A jitter
of geometry.water_cluster (seed 404000 + index), basis cc-pVDZ.  PySCF's own
gto.M (reference package, importable here) builds the _atm/_bas/_env arrays;
the file stores them concatenated with per-molecule offsets, so the GPU box
needs no PySCF.

    python tests/golden/make_batch_golden.py
"""
import os
import sys

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

from pyscf import gto  # noqa: E402
import geometry  # noqa: E402

NMOL = 512
SHAPE = (3, 3, 2)


def main():
    rng = numpy.random.default_rng(404)
    lattice = [(i, j, k) for i in range(SHAPE[0]) for j in range(SHAPE[1]) for k in range(SHAPE[2])]
    atm, bas, env, nw, nao = [], [], [], [], []
    atm_off, bas_off, env_off = [0], [0], [0]
    for m in range(NMOL):
        n = int(rng.integers(1, 17))
        sites = [lattice[s] for s in rng.choice(len(lattice), size=n, replace=False)]
        atoms = geometry.water_cluster(SHAPE, 0.2, 404000 + m, sites=sites)
        mol = gto.M(atom=[(s, tuple(float(x) for x in r)) for s, r in atoms], basis='cc-pvdz', verbose=0)
        atm.append(mol._atm)
        bas.append(mol._bas)
        env.append(mol._env)
        nw.append(n)
        nao.append(mol.nao)
        atm_off.append(atm_off[-1] + mol._atm.shape[0])
        bas_off.append(bas_off[-1] + mol._bas.shape[0])
        env_off.append(env_off[-1] + mol._env.shape[0])
    numpy.savez_compressed(os.path.join(HERE, 'batch_h2o_vdz512.npz'),
                           atm=numpy.concatenate(atm), bas=numpy.concatenate(bas), env=numpy.concatenate(env),
                           atm_off=numpy.array(atm_off), bas_off=numpy.array(bas_off),
                           env_off=numpy.array(env_off), nwater=numpy.array(nw), nao=numpy.array(nao))
    print('%d molecules, waters %d..%d, total nao %d' % (NMOL, min(nw), max(nw), sum(nao)))


if __name__ == '__main__':
    main()
