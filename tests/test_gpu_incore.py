"""The in-core path on the GPU against the reference's own outputs.

  * the s8 tensor of b200jk_int2e_s8 against mol.intor('int2e', aosym='s8')
    (GTO2e_cart_or_sph, pyscf/lib/vhf/fill_nr_s8.c:110-138): whole for
    H2O/6-31G; for (H2O)2/cc-pVTZ (f shells) and (H2O)8/cc-pVDZ by PySCF's
    fingerprint lib.fp over all entries and 20000 seeded entries, and the
    entries the reference leaves at zero (Schwarz cutoff) stay below 1e-12;
  * J/K of b200jk_incore_jk against scf.hf.dot_eri_dm -> _vhf.incore
    (pyscf/scf/_vhf.py:318-401) for a symmetric (hermi=1), a general
    (hermi=0) and an antisymmetric (hermi=2) density, from the s8 tensor the
    GPU filled, from host arrays and from the s4 matrix;
  * an RHF of (H2O)8/cc-pVDZ on in-core builds reproduces the reference
    energy.
Fixtures: tests/golden/make_incore_golden.py.  Tolerances: 1e-12 per
integral, 1e-10 (relative to the largest element) for J and K, 1e-8 Eh for
the energy.
"""
import os

import numpy
import pytest

from conftest import GOLDEN, load_fixture

pytestmark = pytest.mark.gpu

NAMES = ['h2o_631g', 'h2o2_vtz', 'h2o8_vdz']


def _golden(name):
    path = os.path.join(GOLDEN, 'incore_%s.npz' % name)
    if not os.path.exists(path):
        pytest.skip('incore_%s.npz missing (tests/golden/make_incore_golden.py)' % name)
    return dict(numpy.load(path))


def _plan(lib, f):
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    return lib.Plan(f['atm'], f['bas'], f['env'], cart=bool(f['cart']), direct_scf_tol=1e-13)


def _close(a, b, rel=1e-10):
    a, b = numpy.asarray(a), numpy.asarray(b)
    err = abs(a - b).max()
    assert err <= rel * max(1.0, abs(b).max()), err


@pytest.mark.parametrize('name', NAMES)
def test_int2e_s8_matches_reference(name):
    import torch
    from pyscf_b200 import lib
    f, g = load_fixture(name), _golden(name)
    plan = _plan(lib, f)
    eri = plan.int2e_s8(device=True)
    assert eri.numel() == int(g['eri_size'])
    idx = torch.as_tensor(g['sample_idx'], device=eri.device)
    got = eri[idx].cpu().numpy()
    assert abs(got - g['sample_val']).max() < 1e-12
    w = torch.cos(torch.arange(eri.numel(), device=eri.device, dtype=torch.float64))
    fp = float(torch.dot(w, eri))
    assert abs(fp - float(g['eri_fp'])) < 1e-9 * max(1.0, abs(float(g['eri_fp']))), (fp, float(g['eri_fp']))
    assert float(eri.abs().max()) == pytest.approx(float(g['eri_max']), rel=1e-12)
    if 'eri' in g:
        assert abs(eri.cpu().numpy() - g['eri']).max() < 1e-12
        zero = g['eri'] == 0
        assert abs(eri.cpu().numpy()[zero]).max() < 1e-12
    del eri, w
    torch.cuda.empty_cache()


@pytest.mark.parametrize('name', NAMES)
def test_incore_jk_from_gpu_tensor(name):
    import torch
    from pyscf_b200 import lib, incore
    f, g = load_fixture(name), _golden(name)
    plan = _plan(lib, f)
    eri = plan.int2e_s8(device=True)
    for tag, dm, hermi in (('rand', f['dm_rand'], 1), ('ns', f['dm_ns'], 0), ('anti', g['dm_anti'], 2)):
        vj, vk = incore.incore(eri, dm, hermi=hermi)
        _close(vj, g['vj_%s' % tag])
        _close(vk, g['vk_%s' % tag])
    # device densities in, device results out; two densities at once
    d = torch.as_tensor(numpy.stack([f['dm_rand'], f['dm_rand'] * 0.5]), device=eri.device)
    vj, vk = incore.incore(eri, d, hermi=1)
    assert vj.is_cuda and vj.shape == d.shape
    _close(vj[0].cpu().numpy(), g['vj_rand'])
    _close(vk[1].cpu().numpy(), 0.5 * g['vk_rand'])
    # J only, K only
    vj, vk = incore.incore(eri, f['dm_rand'], hermi=1, with_k=False)
    assert vk is None
    _close(vj, g['vj_rand'])
    vj, vk = incore.incore(eri, f['dm_rand'], hermi=1, with_j=False)
    assert vj is None
    _close(vk, g['vk_rand'])
    del eri
    torch.cuda.empty_cache()


def test_incore_host_arrays_and_s4():
    from pyscf_b200 import incore
    g = _golden('h2o_631g')
    f = load_fixture('h2o_631g')
    eri = g['eri']
    nao = int(g['nao'])
    npair = nao * (nao + 1) // 2
    # s4 matrix from the s8 vector (the reference's ao2mo.restore(4, ...))
    eri4 = numpy.empty((npair, npair))
    for p in range(npair):
        for q in range(p + 1):
            eri4[p, q] = eri4[q, p] = eri[p * (p + 1) // 2 + q]
    for tag, dm, hermi in (('rand', f['dm_rand'], 1), ('ns', f['dm_ns'], 0), ('anti', g['dm_anti'], 2)):
        vj, vk = incore.incore(eri, dm, hermi=hermi)
        assert isinstance(vj, numpy.ndarray)
        _close(vj, g['vj_%s' % tag])
        _close(vk, g['vk_%s' % tag])
        vj, vk = incore.incore(eri4, dm, hermi=hermi)
        _close(vj, g['s4_vj_%s' % tag])
        _close(vk, g['s4_vk_%s' % tag])


def test_incore_matches_direct_build():
    from pyscf_b200 import lib, incore
    f = load_fixture('h2o8_vdz')
    plan = _plan(lib, f)
    eri = plan.int2e_s8(device=True)
    vj, vk = incore.incore(eri, f['dm_conv'], hermi=1)
    _close(vj, f['vj_conv'])
    _close(vk, f['vk_conv'])


def test_rhf_on_incore_builds():
    from pyscf_b200 import lib, incore, rhf
    f = load_fixture('h2o8_vdz')
    plan = _plan(lib, f)
    eri = plan.int2e_s8(device=True)
    conv, e, *_ = rhf.kernel(f['hcore'], f['ovlp'], int(f['nelec']), float(f['e_nuc']),
                             lambda dm: incore.incore(eri, dm, hermi=1), conv_tol=1e-10)
    assert conv
    assert abs(e - float(f['e_rhf'])) < 1e-8, (e, float(f['e_rhf']))


@pytest.mark.parametrize('tag', ['full', 'cart', 'lr', 'sr'])
def test_int2e_s8_cartesian_and_range_separated(tag):
    """The GPU fill in the Cartesian basis (int2e_cart) and under the erf and
    erfc operators (env[PTR_RANGE_OMEGA] = 0.5, -0.5; erfc as full minus long
    range) against the reference's whole tensors of H2O/cc-pVDZ, 1e-12 per
    entry, and the in-core J/K of each against the reference's."""
    import torch
    from pyscf_b200 import lib, incore
    path = os.path.join(GOLDEN, 'incore_h2o_vdz_variants.npz')
    if not os.path.exists(path):
        pytest.skip('incore_h2o_vdz_variants.npz missing (tests/golden/make_incore_golden.py)')
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    g = dict(numpy.load(path))
    f = load_fixture('h2o_vdz')

    class Mol:
        _atm, _bas, _env, cart = f['atm'], f['bas'], g['%s_env' % tag], tag == 'cart'
    eri = incore.int2e_s8(Mol(), device=True)
    ref = g['%s_eri' % tag]
    assert eri.numel() == ref.size
    assert abs(eri.cpu().numpy() - ref).max() < 1e-12
    vj, vk = incore.incore(eri, g['%s_dm' % tag], hermi=1)
    _close(vj, g['%s_vj' % tag])
    _close(vk, g['%s_vk' % tag])
    del eri
    torch.cuda.empty_cache()
