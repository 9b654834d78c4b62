"""Reference RHF energies of 8 molecules of the 512-molecule batch workload.

Runs only where the reference checkout is readable (this container): the
unmodified PySCF package from the reference tree on the reference's own C
drivers (oracle/build.py), scf.RHF with the direct path (max_memory = 0, as
pyscf/scf/test/test_h2o_vdz.py:94-98), conv_tol 1e-10, on the first eight
molecules of tests/golden/batch_h2o_vdz512.npz with at most 5 waters
(nao <= 120, so that the CPU reference finishes in minutes).  The batched GPU
SCF (pyscf_b200/batch_scf.py) is checked against these energies.

    python tests/golden/make_batch_scf_golden.py
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
sys.path.insert(0, HERE)
import geometry  # noqa: E402
from make_batch_golden import NMOL, SHAPE  # noqa: E402


def molecules():
    """The batch workload's molecules, regenerated as make_batch_golden.py
    draws them (same generator, same order)."""
    rng = numpy.random.default_rng(404)
    lattice = [(i, j, k) for i in range(SHAPE[0]) for j in range(SHAPE[1]) for k in range(SHAPE[2])]
    for m in range(NMOL):
        n = int(rng.integers(1, 17))
        sites = [lattice[s] for s in rng.choice(len(lattice), size=n, replace=False)]
        yield m, n, geometry.water_cluster(SHAPE, 0.2, 404000 + m, sites=sites)


def main():
    f = dict(numpy.load(os.path.join(HERE, 'batch_h2o_vdz512.npz')))
    picks = [m for m in range(len(f['nao'])) if f['nwater'][m] <= 5][:8]
    energies = []
    for m, n, atoms in molecules():
        if m not in picks:
            continue
        mol = gto.M(atom=[(s, tuple(float(x) for x in r)) for s, r in atoms], basis='cc-pvdz', verbose=0)
        # the same nuclei as the workload's arrays (env layouts may differ)
        a0, a1 = f['atm_off'][m], f['atm_off'][m + 1]
        e0 = f['env_off'][m]
        xyz = numpy.array([f['env'][e0 + p: e0 + p + 3] for p in f['atm'][a0:a1, 1]])
        assert abs(xyz - mol.atom_coords()).max() < 1e-12
        mf = scf.RHF(mol)
        mf.max_memory = 0
        mf.conv_tol = 1e-10
        e = mf.kernel()
        assert mf.converged
        energies.append(e)
        print(m, n, e, flush=True)
    numpy.savez_compressed(os.path.join(HERE, 'batch_scf_sample.npz'), sample=numpy.array(picks),
                           e_rhf=numpy.array(energies))


if __name__ == '__main__':
    main()
