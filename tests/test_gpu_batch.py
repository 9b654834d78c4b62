"""Batched J/K (b200jk_batch_*): many molecules in one launch per quartet class.

The batch runs the same kernels over a global quartet queue; each molecule's
J/K must equal the reference's (tests/golden, PySCF's own direct-SCF drivers)
and its own single-molecule build.  Tolerance: the J/K parity bar, 1e-10.
"""
import numpy
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu

TOL_JK = 1e-10


@pytest.fixture(scope='module')
def b2():
    from pyscf_b200 import lib
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    return lib


def _plans(b2, names):
    fs = [load_fixture(n) for n in names]
    return fs, [b2.Plan(f['atm'], f['bas'], f['env'], cart=bool(f['cart']), direct_scf_tol=1e-13) for f in fs]


def test_batch_matches_reference(b2):
    import torch
    names = ['h2o_631g', 'h2o_vdz', 'h2o2_vtz', 'h2o8_vdz', 'h2o_vdz']
    fs, plans = _plans(b2, names)
    batch = b2.Batch(plans)
    dms = [torch.tensor(f['dm_rand'], device='cuda:0') for f in fs]
    vj, vk = batch.get_jk_device(dms, hermi=1)
    torch.cuda.synchronize()
    for f, j, k in zip(fs, vj, vk):
        assert abs(j.cpu().numpy() - f['vj_rand']).max() < TOL_JK
        assert abs(k.cpu().numpy() - f['vk_rand']).max() < TOL_JK
    st = batch.stats()
    single = 0
    for p, d in zip(plans, dms):
        p.get_jk_device(d, hermi=1)
        single += p.stats()['quartets']
    assert st['quartets'] == single


def test_batch_general_density_and_mixed(b2):
    import torch
    names = ['h2o2_vtz', 'h2o8_vdz']
    fs, plans = _plans(b2, names)
    batch = b2.Batch(plans)
    dms = [torch.tensor(f['dm_ns'], device='cuda:0') for f in fs]
    vj, vk = batch.get_jk_device(dms, hermi=0)
    for f, j, k in zip(fs, vj, vk):
        assert abs(j.cpu().numpy() - f['vj_ns']).max() < TOL_JK
        assert abs(k.cpu().numpy() - f['vk_ns']).max() < TOL_JK
    for p in plans:
        p.set_mixed_threshold(1e30)
    vj, vk = batch.get_jk_device(dms, hermi=0, precision=b2.PREC_MIXED)
    st = batch.stats()
    assert st['fp32_quartets'] == st['quartets'] > 0
    for f, j, k in zip(fs, vj, vk):
        assert abs(j.cpu().numpy() - f['vj_ns']).max() < 2e-5 * abs(f['vj_ns']).max()
        assert abs(k.cpu().numpy() - f['vk_ns']).max() < 2e-5 * abs(f['vk_ns']).max()


def test_batch_cuda_graph(b2):
    """A batched build captured in a CUDA graph: replays give the reference
    J/K, also after the densities are refilled in place."""
    import torch
    names = ['h2o_vdz', 'h2o8_vdz', 'h2o2_vtz']
    fs, plans = _plans(b2, names)
    batch = b2.Batch(plans)
    dms = [torch.tensor(f['dm_rand'], device='cuda:0') for f in fs]
    batch.get_jk_device(dms, hermi=1)          # sizes every buffer
    vj = [torch.empty_like(d) for d in dms]
    vk = [torch.empty_like(d) for d in dms]
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        batch.get_jk_device_async(dms, vj, vk, hermi=1)
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        batch.get_jk_device_async(dms, vj, vk, hermi=1)
    for key in ('rand', 'conv'):
        for f, d in zip(fs, dms):
            d.copy_(torch.tensor(f['dm_' + key], device='cuda:0'))
        g.replay()
        torch.cuda.synchronize()
        for f, j, k in zip(fs, vj, vk):
            assert abs(j.cpu().numpy() - f['vj_' + key]).max() < TOL_JK
            assert abs(k.cpu().numpy() - f['vk_' + key]).max() < TOL_JK


def test_batch512_sample_matches_reference(b2):
    """The 512-molecule batch workload (bench's batch line), built in one
    batched build: 16 sampled molecules against the reference drivers' J/K of
    the same densities (tests/golden/make_batch_jk_golden.py): rows of their
    first three shells element-wise, PySCF fingerprints and E2."""
    import os
    import torch
    from conftest import GOLDEN
    path = os.path.join(GOLDEN, 'batch_jk_sample.npz')
    if not os.path.exists(path):
        pytest.skip('batch_jk_sample.npz missing (tests/golden/make_batch_jk_golden.py)')
    g = dict(numpy.load(path))
    f = dict(numpy.load(os.path.join(GOLDEN, 'batch_h2o_vdz512.npz')))
    rng = numpy.random.default_rng(405)
    plans, dms = [], []
    for m in range(len(f['nao'])):
        a0, a1 = f['atm_off'][m], f['atm_off'][m + 1]
        b0, b1 = f['bas_off'][m], f['bas_off'][m + 1]
        e0, e1 = f['env_off'][m], f['env_off'][m + 1]
        plans.append(b2.Plan(f['atm'][a0:a1], f['bas'][b0:b1], f['env'][e0:e1], direct_scf_tol=1e-13))
        nao, nocc = int(f['nao'][m]), 5 * int(f['nwater'][m])
        c = rng.standard_normal((nao, nocc)) / numpy.sqrt(nao)
        dms.append(torch.tensor(c @ c.T, device='cuda:0'))
    batch = b2.Batch(plans)
    vj, vk = batch.get_jk_device(dms, hermi=1)
    torch.cuda.synchronize()
    for m in g['sample']:
        j = vj[m].cpu().numpy()
        k = vk[m].cpu().numpy()
        d = dms[m].cpu().numpy()
        rows = g['m%03d_rows' % m]
        assert abs(j[rows] - g['m%03d_vj_rows' % m]).max() < TOL_JK, m
        assert abs(k[rows] - g['m%03d_vk_rows' % m]).max() < TOL_JK, m
        e2 = 0.5 * numpy.sum(d * j) - 0.25 * numpy.sum(d * k)
        assert abs(e2 - float(g['m%03d_e2' % m])) < 1e-9 * max(1.0, abs(e2)), m
        fpj = float(numpy.dot(numpy.cos(numpy.arange(j.size)), j.ravel()))
        fpk = float(numpy.dot(numpy.cos(numpy.arange(k.size)), k.ravel()))
        assert abs(fpj - float(g['m%03d_fp_j' % m])) < 1e-8 * max(1.0, abs(fpj)), m
        assert abs(fpk - float(g['m%03d_fp_k' % m])) < 1e-8 * max(1.0, abs(fpk)), m
