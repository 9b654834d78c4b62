"""FP64 parity on the bench workload itself: (H2O)64/cc-pVTZ (nao 3712) and
its 16- and 32-water samples, with the bench density D = C C^T.

The expected values are the reference drivers' J/K of the same density
(PySCF's CVHFnr_direct_drv with CVHFnrs8_prescreen at 1e-13, compiled from
the reference sources on the oracle integral library;
tests/golden/make_h2o64_golden.py): all columns of the rows of eight sampled
shells (every shell type, centre and corner waters), the two-electron energy
E2 = 1/2 tr(D J) - 1/4 tr(D K), PySCF's fingerprints and the column sums of
the whole matrices.  The density is regenerated here from its seed.

Tolerances: sampled elements 1e-10 (the J/K parity bar); E2 and the
fingerprints, sums over 0.9-14 million elements of magnitude up to ~10,
1e-8 relative; column sums 1e-9.
"""
import os

import numpy
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _density(nao):
    rng = numpy.random.default_rng(304)
    c = rng.standard_normal((nao, min(320, nao))) / numpy.sqrt(nao)
    return c @ c.T


def _fp(a):
    a = numpy.asarray(a)
    return float(numpy.dot(numpy.cos(numpy.arange(a.size)), a.ravel()))


@pytest.mark.parametrize('name', ['h2o64_vtz_sub16', 'h2o64_vtz_sub32', 'h2o64_vtz'])
def test_bench_workload_matches_reference(name):
    import torch
    from pyscf_b200 import lib
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    ref_path = os.path.join(GOLDEN, 'jk_%s.npz' % name)
    if not os.path.exists(ref_path):
        pytest.skip('reference fixture %s missing (tests/golden/make_h2o64_golden.py)' % os.path.basename(ref_path))
    g = dict(numpy.load(ref_path))
    f = dict(numpy.load(os.path.join(GOLDEN, 'mol_%s.npz' % name)))
    nao = int(f['nao'])
    dm = _density(nao)
    plan = lib.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13)
    vj, vk = plan.get_jk_device(torch.tensor(dm, device='cuda:0'), hermi=1)
    vj = vj.cpu().numpy()
    vk = vk.cpu().numpy()
    rows = g['rows']
    assert abs(vj[rows] - g['vj_rows']).max() < 1e-10
    assert abs(vk[rows] - g['vk_rows']).max() < 1e-10
    e2 = 0.5 * numpy.sum(dm * vj) - 0.25 * numpy.sum(dm * vk)
    assert abs(e2 - float(g['e2'])) < 1e-8 * abs(float(g['e2']))
    assert abs(_fp(vj) - float(g['fp_j'])) < 1e-8 * max(1.0, abs(float(g['fp_j'])))
    assert abs(_fp(vk) - float(g['fp_k'])) < 1e-8 * max(1.0, abs(float(g['fp_k'])))
    assert abs(vj.sum(axis=0) - g['colsum_j']).max() < 1e-9
    assert abs(vk.sum(axis=0) - g['colsum_k']).max() < 1e-9
