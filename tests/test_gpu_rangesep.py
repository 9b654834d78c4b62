"""Range-separated Coulomb on the GPU: env[PTR_RANGE_OMEGA] = omega selects
erf(omega r12)/r12 (omega > 0, evaluated in the kernels) or
erfc(|omega| r12)/r12 (omega < 0, full minus long range), as
mol.with_range_coulomb / with_short_range_coulomb do for libcint
(pyscf/scf/hf.py:1006, pyscf/scf/_vhf.py:611-627).

Expected values: the reference's published long-range fingerprints
(pyscf/scf/test/test_rhf.py:930-952, omega = 1.5) and the oracle, whose
attenuated integrals are pinned to those fingerprints
(tests/test_oracle_golden.py).  Tolerance: the J/K parity bar, 1e-10.
"""
import numpy
import pytest

from conftest import load_fixture, lib_fp

pytestmark = pytest.mark.gpu

TOL_JK = 1e-10


class _Mol:
    def __init__(self, f, omega=0.0):
        self._atm, self._bas = f['atm'], f['bas']
        self._env = f['env'].copy()
        self._env[8] = omega
        self.cart = bool(f['cart'])


@pytest.fixture(scope='module')
def b2():
    from pyscf_b200 import lib
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    return lib


def test_long_range_reference_fingerprints(b2):
    # mf.get_j(mol, dm, omega=1.5), mf.get_k(mol, dm, hermi=0, omega=1.5)
    from pyscf_b200 import scf as b2scf, _vhf
    f = load_fixture('h2o_vdz')
    nao = int(f['nao'])
    numpy.random.seed(1)
    dm = numpy.random.random((nao, nao))
    mol = _Mol(f)
    opt = _vhf.VHFOpt(_Mol(f, 1.5), direct_scf_tol=1e-13)
    opt.prescreen = 'CVHFnrs8_vj_prescreen'
    vj, _ = b2scf.get_jk(mol, dm, 1, opt, True, False, omega=1.5)
    assert abs(lib_fp(vj) - -10.015956161068031) < 1e-10
    opt.prescreen = 'CVHFnrs8_vk_prescreen'
    _, vk = b2scf.get_jk(mol, dm, 0, opt, False, True, omega=1.5)
    assert abs(lib_fp(vk) - -11.399103957754445) < 1e-10


@pytest.mark.parametrize('name,omega', [('h2o2_vtz', 0.3), ('h2o8_vdz', 0.3), ('h2o_vdz', -0.4),
                                        ('h2o2_vtz', -0.25)])
def test_range_separated_matches_oracle(b2, name, omega):
    import oracle
    from pyscf_b200 import _vhf
    f = load_fixture(name)
    env = f['env'].copy()
    env[8] = omega
    rj, rk, _ = oracle.get_jk(f['dm_rand'], f['atm'], f['bas'], env, hermi=1)
    opt = _vhf.VHFOpt(_Mol(f, omega), direct_scf_tol=1e-13)
    vj, vk = _vhf.direct(f['dm_rand'], f['atm'], f['bas'], env, opt, hermi=1)
    assert abs(vj - rj).max() < TOL_JK
    assert abs(vk - rk).max() < TOL_JK
    # non-symmetric density (K by 'li->s1kj')
    rj, rk, _ = oracle.get_jk(f['dm_ns'], f['atm'], f['bas'], env, hermi=0)
    vj, vk = _vhf.direct(f['dm_ns'], f['atm'], f['bas'], env, opt, hermi=0)
    assert abs(vj - rj).max() < TOL_JK
    assert abs(vk - rk).max() < TOL_JK


def test_long_range_q_cond_and_mixed(b2):
    """The plan's Schwarz bound is that of the attenuated integrals (the
    reference computes it under with_range_coulomb); mixed precision works
    for them too."""
    import oracle
    f = load_fixture('h2o8_vdz')
    env = f['env'].copy()
    env[8] = 0.3
    p = b2.Plan(f['atm'], f['bas'], env, direct_scf_tol=1e-13)
    q = oracle.q_cond(f['atm'], f['bas'], env, False, 1e-13)
    assert abs(p.q_cond - q).max() <= 1e-10 * abs(q).max()
    assert (p.q_cond <= b2.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13).q_cond + 1e-15).all()
    vj, vk = p.get_jk(f['dm_rand'], hermi=1)
    p.set_mixed_threshold(1e-6)
    mj, mk = p.get_jk(f['dm_rand'], hermi=1, precision=b2.PREC_MIXED)
    assert p.stats()['fp32_quartets'] > 0
    assert abs(mj - vj).max() < 1e-8 and abs(mk - vk).max() < 1e-8


@pytest.mark.parametrize('omega', [0.3, -0.3])
def test_range_separated_gradient_jk(b2, omega):
    """grad.rhf.get_jk under with_range_coulomb(omega): int2e_ip1 of the
    attenuated operator, against the oracle's."""
    import oracle
    from pyscf_b200 import _vhf
    f = load_fixture('h2o_vdz')
    env = f['env'].copy()
    env[8] = omega
    d = f['dm_conv']
    rj, rk = oracle.grad_jk(d, f['atm'], f['bas'], env, False, 1e-14)
    plan = _vhf.make_plan(f['atm'], f['bas'], env, False, 1e-13)
    vj, vk = plan.grad_jk(d, direct_scf_tol=1e-14)
    assert abs(vj - rj).max() < TOL_JK
    assert abs(vk - rk).max() < TOL_JK
