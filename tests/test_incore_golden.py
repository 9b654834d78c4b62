"""The in-core fixtures and the contraction's decomposition, on the CPU.

tests/golden/incore_h2o_631g.npz holds the reference's s8 tensor of
H2O/6-31G (mol.intor('int2e', aosym='s8')) and its _vhf.incore J/K
(pyscf/scf/_vhf.py:318-401) for hermi = 1, 0, 2.  Checked here:
  * the fixtures against their definition, J = einsum('ijkl,ji->kl'),
    K = einsum('ijkl,jk->il') over the unpacked tensor, then hermi_triu;
  * the decomposition the GPU kernel uses (pyscf_b200/csrc/incore.cu): per
    stored entry the four pair-order images with weight 1/(coinciding
    images), K = A(D) + A(D^T)^T for s8, packed J from the row and column
    sums of the packed matrix, written as plain loops;
  * the in-core J/K of (H2O)8/cc-pVDZ against the direct J/K of the same
    density (mol_h2o8_vdz.npz, screened at 1e-13).
"""
import os

import numpy
import pytest

from conftest import GOLDEN, load_fixture


def _golden(name):
    path = os.path.join(GOLDEN, 'incore_%s.npz' % name)
    if not os.path.exists(path):
        pytest.skip('incore_%s.npz missing' % name)
    return dict(numpy.load(path))


def _pair(i, j):
    return i * (i + 1) // 2 + j if i >= j else j * (j + 1) // 2 + i


def _unpack(eri, nao):
    full = numpy.empty((nao,) * 4)
    for i in range(nao):
        for j in range(nao):
            for k in range(nao):
                for l in range(nao):
                    p, q = _pair(i, j), _pair(k, l)
                    hi, lo = max(p, q), min(p, q)
                    full[i, j, k, l] = eri[hi * (hi + 1) // 2 + lo]
    return full


def _hermi_triu(m, hermi):
    m = m.copy()
    iu = numpy.triu_indices(m.shape[0], 1)
    m[iu] = -m.T[iu] if hermi == 2 else m.T[iu]
    return m


def _kernel_decomposition(eri, dm, nao):
    """A(D) and packed J from the stored s8 entries, as incore_pass_kernel."""
    npair = nao * (nao + 1) // 2
    t = numpy.array([dm[i, j] + dm[j, i] if i != j else dm[i, i]
                     for i in range(nao) for j in range(i + 1)])
    A = numpy.zeros((nao, nao))
    Jp = numpy.zeros(npair)
    pairs = [(i, j) for i in range(nao) for j in range(i + 1)]
    for p, (i, j) in enumerate(pairs):
        for q in range(p + 1):
            k, l = pairs[q]
            v = eri[p * (p + 1) // 2 + q]
            wpq = 0.5 if p == q else 1.0
            w = wpq * (0.5 if i == j else 1.0) * (0.5 if k == l else 1.0)
            A[i, l] += w * v * dm[j, k]
            A[j, l] += w * v * dm[i, k]
            A[i, k] += w * v * dm[j, l]
            A[j, k] += w * v * dm[i, l]
            Jp[q] += wpq * v * t[p]
            Jp[p] += wpq * v * t[q]
    J = numpy.array([[Jp[_pair(x, y)] for y in range(nao)] for x in range(nao)])
    return A, J


def test_fixture_matches_definition():
    g = _golden('h2o_631g')
    f = load_fixture('h2o_631g')
    nao = int(g['nao'])
    full = _unpack(g['eri'], nao)
    for tag, dm, hermi in (('rand', f['dm_rand'], 1), ('ns', f['dm_ns'], 0), ('anti', g['dm_anti'], 2)):
        vj = _hermi_triu(numpy.einsum('ijkl,ji->kl', full, dm), 1)
        vk = numpy.einsum('ijkl,jk->il', full, dm)
        if hermi:
            vk = _hermi_triu(vk, hermi)
        assert abs(vj - g['vj_%s' % tag]).max() < 1e-12
        assert abs(vk - g['vk_%s' % tag]).max() < 1e-12
        assert abs(g['s4_vj_%s' % tag] - g['vj_%s' % tag]).max() < 1e-12
        assert abs(g['s4_vk_%s' % tag] - g['vk_%s' % tag]).max() < 1e-12


def test_kernel_decomposition_matches_fixture():
    g = _golden('h2o_631g')
    f = load_fixture('h2o_631g')
    nao = int(g['nao'])
    for tag, dm, hermi in (('rand', f['dm_rand'], 1), ('ns', f['dm_ns'], 0), ('anti', g['dm_anti'], 2)):
        A, J = _kernel_decomposition(g['eri'], dm, nao)
        if hermi == 1:
            K = A + A.T
        elif hermi == 2:
            K = A - A.T
        else:
            At, _ = _kernel_decomposition(g['eri'], dm.T.copy(), nao)
            K = A + At.T
        if hermi:
            K = _hermi_triu(K, hermi)
        assert abs(J - g['vj_%s' % tag]).max() < 1e-12
        assert abs(K - g['vk_%s' % tag]).max() < 1e-12


def test_incore_fixture_matches_direct_fixture():
    g = _golden('h2o8_vdz')
    f = load_fixture('h2o8_vdz')
    scale = max(1.0, abs(f['vj_rand']).max())
    assert abs(g['vj_rand'] - f['vj_rand']).max() < 1e-9 * scale
    assert abs(g['vk_rand'] - f['vk_rand']).max() < 1e-9 * scale


def test_range_separated_fixtures_add_up():
    """erf + erfc = 1: the reference's long- and short-range s8 tensors of
    H2O/cc-pVDZ add up to the full-range one (to the Schwarz cutoff, 1e-14,
    under which each operator leaves its own entries at zero)."""
    path = os.path.join(GOLDEN, 'incore_h2o_vdz_variants.npz')
    if not os.path.exists(path):
        pytest.skip('incore_h2o_vdz_variants.npz missing')
    g = dict(numpy.load(path))
    assert abs(g['lr_eri'] + g['sr_eri'] - g['full_eri']).max() < 1e-12
    assert g['cart_eri'].size > g['full_eri'].size   # 25 Cartesian AOs against 24
