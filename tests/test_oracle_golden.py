"""Pin the CPU oracle against the reference's own golden values.

The oracle is this project's restatement of libcint's integrals and of
CVHFnr_direct_drv (oracle/).  The fixtures hold J/K produced by the
reference's own C drivers (pyscf/lib/vhf/nr_direct.c and friends, compiled
from the reference sources) running on the oracle integral library, and the
reference tests' published fingerprints are checked here too."""
import numpy
import pytest

from conftest import load_fixture, lib_fp
import oracle


def test_h2o_vdz_identity_density_fingerprints():
    # pyscf/scf/test/test_rhf.py:909-916: dm = I, fp(vj), fp(vk)
    f = load_fixture('h2o_vdz')
    nao = int(f['nao'])
    vj, vk, _ = oracle.get_jk(numpy.eye(nao), f['atm'], f['bas'], f['env'], hermi=1)
    assert abs(lib_fp(vj) - 1.6593323222866125) < 1e-9
    assert abs(lib_fp(vk) - -1.4662135224053987) < 1e-9


def test_h2o_vdz_random_density_norm_and_k():
    # pyscf/scf/test/test_rhf.py:890-901 (|vj| = 77.035779188661465) and
    # :918-928 (fp(vk, hermi=0) = -12.365527167710301), numpy.random.seed(1)
    f = load_fixture('h2o_vdz')
    nao = int(f['nao'])
    numpy.random.seed(1)
    dm = numpy.random.random((nao, nao))
    vj, _, _ = oracle.get_jk(dm, f['atm'], f['bas'], f['env'], hermi=1)
    assert abs(numpy.linalg.norm(vj) - 77.035779188661465) < 1e-9
    _, vk, _ = oracle.get_jk(dm, f['atm'], f['bas'], f['env'], hermi=0)
    assert abs(lib_fp(vk) - -12.365527167710301) < 1e-11


def test_h2o_631g_direct_fingerprints():
    # pyscf/scf/test/test_vhf.py:158-174: dm = r + r^T, numpy.random.seed(1),
    # K by 'jk->s1il' (=(ij|kl) D_jk) and J by 'ji->s1kl', unscreened
    f = load_fixture('h2o_631g')
    nao = int(f['nao'])
    numpy.random.seed(1)
    dm = numpy.random.random((nao, nao))
    dm = dm + dm.T
    vj, vk, _ = oracle.get_jk(dm, f['atm'], f['bas'], f['env'], hermi=1, screen=False)
    assert abs(lib_fp(vk) - 5.0067176755619975) < 1e-11
    assert abs(lib_fp(vj) - 48.61070262547175) < 1e-11


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o_vdz', 'h2o2_vtz'])
def test_restated_driver_matches_reference_drivers(name):
    f = load_fixture(name)
    vj, vk, nq = oracle.get_jk(f['dm_rand'], f['atm'], f['bas'], f['env'], hermi=1)
    assert nq > 0
    assert abs(vj - f['vj_rand']).max() < 1e-11
    assert abs(vk - f['vk_rand']).max() < 1e-11
    vj, vk, _ = oracle.get_jk(f['dm_ns'], f['atm'], f['bas'], f['env'], hermi=0)
    assert abs(vj - f['vj_ns']).max() < 1e-11
    assert abs(vk - f['vk_ns']).max() < 1e-11
    vj, vk, _ = oracle.get_jk(f['dm_rand'], f['atm'], f['bas'], f['env'], hermi=1, screen=False)
    assert abs(vj - f['vj_rand_noscreen']).max() < 1e-11
    assert abs(vk - f['vk_rand_noscreen']).max() < 1e-11


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o_vdz', 'h2o2_vtz'])
def test_q_cond_matches_reference(name):
    f = load_fixture(name)
    q = oracle.q_cond(f['atm'], f['bas'], f['env'])
    assert abs(q - f['q_cond']).max() < 1e-13


def test_reference_energies_in_fixture():
    # pyscf/scf/test/test_h2o_vdz.py:45 and :98 (9 decimals)
    f = load_fixture('h2o_vdz')
    assert abs(float(f['e_rhf']) - -76.026765673120565) < 1e-9
    assert abs(float(f['e_rhf']) - -76.026765673119627) < 1e-9


def _grad_fixture(name):
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'grad_%s.npz' % name)
    return dict(numpy.load(path))


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o2_vtz'])
def test_grad_oracle_matches_reference(name):
    """The oracle's restatement of grad.rhf.get_jk (driver, screen, derivative
    conditioner) against the reference's own output."""
    f = _grad_fixture(name)
    q = oracle.grad_q_cond(f['atm'], f['bas'], f['env'])
    assert abs(q - f['gq_cond']).max() <= 1e-12 * abs(f['gq_cond']).max()
    vj, vk = oracle.grad_jk(f['dm0'], f['atm'], f['bas'], f['env'])
    assert abs(vj - f['gvj']).max() < 1e-11
    assert abs(vk - f['gvk']).max() < 1e-11


def test_grad_reference_fingerprint():
    """The fixture's RHF gradient reproduces the reference test's value
    (pyscf/grad/test/test_rhf.py:148-153, 6 places) and its own finite
    differences."""
    f = _grad_fixture('h2o_631g')
    assert abs(lib_fp(f['de']) - 0.0055115512502467556) < 5e-7
    h = float(f['fd_h'])
    fd = (f['fd_energies'][:, 0] - f['fd_energies'][:, 1]) / (2 * h)
    assert abs(f['de'].ravel()[f['fd_coords']] - fd).max() < 5e-6


def test_h2o_vdz_long_range_fingerprints():
    # pyscf/scf/test/test_rhf.py:930-952: numpy.random.seed(1) dm (nao, nao),
    # mf.get_j(mol, dm, omega=1.5) and mf.get_k(mol, dm, hermi=0, omega=1.5):
    # erf(omega r12)/r12 (env[PTR_RANGE_OMEGA] = 1.5) pins the oracle's
    # attenuated integrals
    f = load_fixture('h2o_vdz')
    nao = int(f['nao'])
    numpy.random.seed(1)
    dm = numpy.random.random((nao, nao))
    env = f['env'].copy()
    env[8] = 1.5
    vj, _, _ = oracle.get_jk(dm, f['atm'], f['bas'], env, hermi=1)
    assert abs(lib_fp(vj) - -10.015956161068031) < 1e-11
    _, vk, _ = oracle.get_jk(dm, f['atm'], f['bas'], env, hermi=0)
    assert abs(lib_fp(vk) - -11.399103957754445) < 1e-11


def test_short_range_is_full_minus_long_range():
    # erfc(w r)/r = 1/r - erf(w r)/r, element by element of the oracle's J/K
    f = load_fixture('h2o_631g')
    dm = f['dm_rand']
    full = oracle.get_jk(dm, f['atm'], f['bas'], f['env'], hermi=1, screen=False)
    e_lr, e_sr = f['env'].copy(), f['env'].copy()
    e_lr[8], e_sr[8] = 0.3, -0.3
    lr = oracle.get_jk(dm, f['atm'], f['bas'], e_lr, hermi=1, screen=False)
    sr = oracle.get_jk(dm, f['atm'], f['bas'], e_sr, hermi=1, screen=False)
    for i in range(2):
        assert abs(lr[i] + sr[i] - full[i]).max() < 1e-12
