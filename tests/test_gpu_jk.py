"""Parity of the CUDA J/K build with the reference (the -m gpu suite).

Every expected value comes from the reference: J/K produced by PySCF's own
direct-SCF C drivers (compiled from the reference sources on the oracle
integral library) and stored in tests/golden, PySCF's published
fingerprints and energies, or the oracle restatement run here.  The GPU path
is called through the C ABI (libb200jk.so via ctypes).

Tolerances: FP64 path max|dJ|, max|dK| <= 1e-10 and |dE_SCF| <= 1e-9 Eh.
"""
import numpy
import pytest

from conftest import load_fixture, lib_fp

pytestmark = pytest.mark.gpu

TOL_JK = 1e-10
TOL_E = 1e-9


@pytest.fixture(scope='module')
def b2():
    from pyscf_b200 import lib
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    return lib


def plan_for(b2, f, tol=1e-13):
    return b2.Plan(f['atm'], f['bas'], f['env'], cart=bool(f['cart']), direct_scf_tol=tol)


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o_vdz', 'h2o2_vtz', 'h2o8_vdz'])
def test_q_cond(b2, name):
    f = load_fixture(name)
    p = plan_for(b2, f)
    q = p.q_cond
    ref = f['q_cond']
    # q only steers the screen; the spherical diagonal of an (ff|ff) block is
    # a long alternating sum, so agreement is ~1e-12 relative
    assert abs(q - ref).max() <= 1e-10 * max(1.0, abs(ref).max())


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o_vdz', 'h2o2_vtz', 'h2o8_vdz'])
def test_jk_symmetric_density(b2, name):
    f = load_fixture(name)
    p = plan_for(b2, f)
    vj, vk = p.get_jk(f['dm_rand'], hermi=1)
    assert abs(vj - f['vj_rand']).max() < TOL_JK
    assert abs(vk - f['vk_rand']).max() < TOL_JK
    st = p.stats()
    assert st['quartets'] > 0


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o_vdz', 'h2o2_vtz'])
def test_jk_unscreened(b2, name):
    from pyscf_b200 import _vhf
    f = load_fixture(name)
    vj, vk = _vhf.direct(f['dm_rand'], f['atm'], f['bas'], f['env'], None, hermi=1)
    assert abs(vj - f['vj_rand_noscreen']).max() < TOL_JK
    assert abs(vk - f['vk_rand_noscreen']).max() < TOL_JK


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o_vdz', 'h2o2_vtz', 'h2o8_vdz'])
def test_jk_general_density(b2, name):
    f = load_fixture(name)
    p = plan_for(b2, f)
    vj, vk = p.get_jk(f['dm_ns'], hermi=0)
    assert abs(vj - f['vj_ns']).max() < TOL_JK
    assert abs(vk - f['vk_ns']).max() < TOL_JK


@pytest.mark.parametrize('name', ['h2o_vdz', 'h2o8_vdz'])
def test_jk_converged_density(b2, name):
    f = load_fixture(name)
    p = plan_for(b2, f)
    vj, vk = p.get_jk(f['dm_conv'], hermi=1)
    assert abs(vj - f['vj_conv']).max() < TOL_JK
    assert abs(vk - f['vk_conv']).max() < TOL_JK


def test_reference_fingerprints(b2):
    # pyscf/scf/test/test_rhf.py:909-916 and :918-928
    f = load_fixture('h2o_vdz')
    nao = int(f['nao'])
    p = plan_for(b2, f)
    vj, vk = p.get_jk(numpy.eye(nao), hermi=1)
    assert abs(lib_fp(vj) - 1.6593323222866125) < 1e-9
    assert abs(lib_fp(vk) - -1.4662135224053987) < 1e-9
    numpy.random.seed(1)
    dm = numpy.random.random((nao, nao))
    _, vk = p.get_jk(dm, hermi=0)
    assert abs(lib_fp(vk) - -12.365527167710301) < 1e-11


def test_631g_direct_fingerprints(b2):
    # pyscf/scf/test/test_vhf.py:158-174 (unscreened)
    from pyscf_b200 import _vhf
    f = load_fixture('h2o_631g')
    nao = int(f['nao'])
    numpy.random.seed(1)
    dm = numpy.random.random((nao, nao))
    dm = dm + dm.T
    vj, vk = _vhf.direct(dm, f['atm'], f['bas'], f['env'], None, hermi=1)
    assert abs(lib_fp(vk) - 5.0067176755619975) < 1e-11
    assert abs(lib_fp(vj) - 48.61070262547175) < 1e-11


def test_multiple_densities_and_antisymmetric(b2):
    from pyscf_b200 import _vhf
    f = load_fixture('h2o2_vtz')
    dms = numpy.stack([f['dm_rand'], f['dm_ns']])
    vj, vk = _vhf.direct(dms, f['atm'], f['bas'], f['env'], None, hermi=0)
    assert abs(vj[0] - f['vj_rand_noscreen']).max() < TOL_JK
    assert abs(vk[0] - f['vk_rand_noscreen']).max() < TOL_JK
    # antisymmetric density: J vanishes, K is antisymmetric (hermi=2)
    a = f['dm_ns'] - f['dm_ns'].T
    vj2, vk2 = _vhf.direct(a, f['atm'], f['bas'], f['env'], None, hermi=2)
    vj0, vk0 = _vhf.direct(a, f['atm'], f['bas'], f['env'], None, hermi=0)
    assert abs(vj2).max() < 1e-10
    assert abs(vk2 + vk2.T).max() < 1e-12
    assert abs(vk2 - vk0).max() < TOL_JK


def test_linearity_and_symmetry(b2):
    f = load_fixture('h2o8_vdz')
    p = plan_for(b2, f, tol=0.0)
    d1, d2 = f['dm_rand'], f['dm_conv']
    j1, k1 = p.get_jk(d1, hermi=1)
    j2, k2 = p.get_jk(d2, hermi=1)
    j3, k3 = p.get_jk(d1 + 0.5 * d2, hermi=1)
    assert abs(j3 - (j1 + 0.5 * j2)).max() < 1e-10
    assert abs(k3 - (k1 + 0.5 * k2)).max() < 1e-10
    assert abs(j1 - j1.T).max() < 1e-12
    assert abs(k1 - k1.T).max() < 1e-12


def test_device_pointer_path(b2):
    import torch
    f = load_fixture('h2o2_vtz')
    p = plan_for(b2, f)
    d = torch.tensor(f['dm_rand'], device='cuda:0')
    vj, vk = p.get_jk_device(d, hermi=1)
    torch.cuda.synchronize()
    assert abs(vj.cpu().numpy() - f['vj_rand']).max() < TOL_JK
    assert abs(vk.cpu().numpy() - f['vk_rand']).max() < TOL_JK


@pytest.mark.parametrize('name,ref', [('h2o_vdz', -76.026765673120565), ('h2o8_vdz', None)])
def test_scf_energy(b2, name, ref):
    """A full RHF on the GPU J/K build reproduces the reference energy."""
    from pyscf_b200 import rhf
    f = load_fixture(name)
    p = plan_for(b2, f)

    def get_jk(dm):
        return p.get_jk(dm, hermi=1)
    conv, e, dm, *_ = rhf.kernel(f['hcore'], f['ovlp'], int(f['nelec']), float(f['e_nuc']), get_jk,
                                 conv_tol=min(1e-11, float(f['scf_conv_tol'])))
    assert conv
    assert abs(e - float(f['e_rhf'])) < TOL_E
    if ref is not None:
        assert abs(e - ref) < TOL_E


def test_sharded_plans_sum_to_full_build(b2):
    """Two plans sharded (0, 2) and (1, 2), as two GPUs would run them, sum to
    the unsharded build (here both on one GPU, one after the other)."""
    f = load_fixture('h2o2_vtz')
    parts = []
    for r in range(2):
        p = plan_for(b2, f)
        p.set_shard(r, 2)
        parts.append(p.get_jk(f['dm_ns'], hermi=0))
        assert 0 < p.stats()['quartets']
    vj = parts[0][0] + parts[1][0]
    vk = parts[0][1] + parts[1][1]
    assert abs(vj - f['vj_ns']).max() < TOL_JK
    assert abs(vk - f['vk_ns']).max() < TOL_JK


def test_autotune_keeps_results(b2):
    """The autotuner only switches launch variants: J/K stay the reference's."""
    f = load_fixture('h2o8_vdz')
    p = plan_for(b2, f)
    tun = p.autotune(f['dm_conv'])
    tun32 = p.tuning(b2.PREC_MIXED)
    assert len(tun) == len(tun32) == 55 and set(tun) <= {0, 1, 2} and set(tun32) <= {0, 1}
    for dm, rj, rk in [(f['dm_rand'], f['vj_rand'], f['vk_rand']), (f['dm_conv'], f['vj_conv'], f['vk_conv'])]:
        vj, vk = p.get_jk(dm, hermi=1)
        assert abs(vj - rj).max() < TOL_JK
        assert abs(vk - rk).max() < TOL_JK
    vj, vk = p.get_jk(f['dm_conv'], hermi=1, precision=b2.PREC_MIXED)
    assert abs(vj - f['vj_conv']).max() < 1e-8
    assert abs(vk - f['vk_conv']).max() < 1e-8


def test_set_tuning_every_variant(b2):
    """Every class that has a second variant, forced to it in both
    precisions, reproduces the reference J/K; a variant a class lacks is
    refused."""
    f = load_fixture('h2o2_vtz')
    p = plan_for(b2, f)
    p.autotune(f['dm_rand'])
    have = [0] * 55
    for t in range(55):
        one = [0] * 55
        one[t] = 1
        try:
            p.set_tuning(one)
            have[t] = 1
        except RuntimeError:
            pass
    assert sum(have) > 0
    with pytest.raises(RuntimeError):
        p.set_tuning([1] * 55)
    with pytest.raises(RuntimeError):
        p.set_tuning([0] * 54)
    p.set_tuning(have)
    p.set_tuning(have, b2.PREC_MIXED)
    assert p.tuning() == have and p.tuning(b2.PREC_MIXED) == have
    vj, vk = p.get_jk(f['dm_rand'], hermi=1)
    assert abs(vj - f['vj_rand']).max() < TOL_JK
    assert abs(vk - f['vk_rand']).max() < TOL_JK
    p.set_mixed_threshold(1e30)
    vj, vk = p.get_jk(f['dm_rand'], hermi=1, precision=b2.PREC_MIXED)
    assert abs(vj - f['vj_rand']).max() < 2e-5 * abs(f['vj_rand']).max()
    assert abs(vk - f['vk_rand']).max() < 2e-5 * abs(f['vk_rand']).max()


def test_untuned_default_variants(b2):
    """A plan that was never tuned runs variant 0 below 1500 AOs and the
    measured defaults from there on (bra runs for eight s/p-ket classes,
    half-width groups for (21|20) and (22|10)); float32 passes stay at 0 and
    an explicit tuning replaces the defaults.  Parity of builds with the
    defaults is covered by the 32-water sample (nao 1856) against the
    reference drivers' J/K."""
    small = plan_for(b2, load_fixture('h2o8_vdz'))
    assert small.tuning() == [0] * 55
    big = plan_for(b2, load_fixture('h2o64_vtz_sub32'))
    expect = [0] * 55
    for t in (0, 1, 2, 3, 4, 6, 7, 21):
        expect[t] = 2
    expect[13] = expect[16] = 1
    assert big.tuning() == expect
    assert big.tuning(b2.PREC_MIXED) == [0] * 55
    big.set_tuning([0] * 55)
    assert big.tuning() == [0] * 55


@pytest.mark.parametrize('name', ['h2o8_vdz', 'h2o2_vtz'])
def test_bra_run_variant(b2, name):
    """Variant 2 of the register family (bra runs: K[a,*] and ket-side J
    carried across four bra pairs) on every class that has it reproduces the
    reference J/K in FP64, in the float64 pass of mixed builds, and falls back
    to the plain kernels for non-symmetric densities; float32 passes refuse it."""
    f = load_fixture(name)
    p = plan_for(b2, f)
    two = [0] * 55
    for t in range(55):
        one = [0] * 55
        one[t] = 2
        try:
            p.set_tuning(one)
            two[t] = 2
        except RuntimeError:
            pass
    assert sum(two) > 0
    with pytest.raises(RuntimeError):
        p.set_tuning(two, b2.PREC_MIXED)
    p.set_tuning(two)
    vj, vk = p.get_jk(f['dm_rand'], hermi=1)
    assert abs(vj - f['vj_rand']).max() < TOL_JK
    assert abs(vk - f['vk_rand']).max() < TOL_JK
    vj, vk = p.get_jk(f['dm_ns'], hermi=0)
    assert abs(vj - f['vj_ns']).max() < TOL_JK
    assert abs(vk - f['vk_ns']).max() < TOL_JK
    if 'dm_conv' in f:
        p.set_mixed_threshold(1e-6)
        vj, vk = p.get_jk(f['dm_conv'], hermi=1, precision=b2.PREC_MIXED)
        assert abs(vj - f['vj_conv']).max() < 1e-8
        assert abs(vk - f['vk_conv']).max() < 1e-8
