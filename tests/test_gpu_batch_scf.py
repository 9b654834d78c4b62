"""Batched SCF of the 512-molecule workload's molecules, whole iterations on
the GPU and replayed as one CUDA graph (pyscf_b200/batch_scf.py).

The first 24 molecules of tests/golden/batch_h2o_vdz512.npz (1 to 16 waters,
cc-pVDZ) run together; the eight of them with at most 5 waters have
reference RHF energies (the unmodified reference, direct SCF, conv_tol 1e-10;
tests/golden/make_batch_scf_golden.py).  Tolerance 1e-8 Eh (the reference's
own convergence is 1e-10 in the energy change per cycle).
"""
import os

import numpy
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def e_nuc(atm, env):
    z = atm[:, 0].astype(float)
    xyz = numpy.array([env[p:p + 3] for p in atm[:, 1]])
    r = numpy.linalg.norm(xyz[:, None] - xyz[None], axis=-1)
    iu = numpy.triu_indices(len(z), 1)
    return float((z[:, None] * z[None] / numpy.where(r > 0, r, 1.0))[iu].sum())


def molecules(b2, count):
    f = dict(numpy.load(os.path.join(GOLDEN, 'batch_h2o_vdz512.npz')))
    plans, nelec, enuc = [], [], []
    for m in range(count):
        a0, a1 = f['atm_off'][m], f['atm_off'][m + 1]
        b0, b1 = f['bas_off'][m], f['bas_off'][m + 1]
        e0, e1 = f['env_off'][m], f['env_off'][m + 1]
        atm, env = f['atm'][a0:a1], f['env'][e0:e1]
        plans.append(b2.Plan(atm, f['bas'][b0:b1], env, direct_scf_tol=1e-13))
        nelec.append(10 * int(f['nwater'][m]))
        enuc.append(e_nuc(atm, env))
    return plans, nelec, enuc


def test_batch_scf_graph_matches_reference():
    from pyscf_b200 import lib, batch_scf
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    path = os.path.join(GOLDEN, 'batch_scf_sample.npz')
    if not os.path.exists(path):
        pytest.skip('batch_scf_sample.npz missing (tests/golden/make_batch_scf_golden.py)')
    ref = dict(numpy.load(path))
    plans, nelec, enuc = molecules(lib, 24)
    scf = batch_scf.BatchRHF(plans, nelec, enuc)
    scf.start()
    scf.capture()
    e, de = scf.run(40)
    assert (de < 1e-9).all(), de.max()
    assert scf.idem_err.max().item() < 1e-10
    for m, er in zip(ref['sample'], ref['e_rhf']):
        assert abs(e[m] - er) < 1e-8, (m, e[m], er)
    # an eager iteration continues from the graph's state without moving it
    e2, _ = scf.run(1, use_graph=False)
    assert abs(e2 - e).max() < 1e-9
