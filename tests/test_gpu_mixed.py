"""Mixed precision (B200JK_PREC_MIXED) of the CUDA J/K build.

Quartets whose Schwarz bound times max|D| is below tau are evaluated in
float32 (roots, recurrences, assembly) and contracted and accumulated in
float64; the rest run the float64 kernels.  Reference values are the
reference's own J/K (tests/golden, PySCF's direct-SCF drivers) and RHF
energy.  The float64 path of the same plan is the baseline for the error.

Tolerances: the RHF energy with mixed builds stays within 1e-6 Eh of the
reference's (the accuracy target of the mixed mode); single builds are
bounded relative to max|J|, max|K|.
"""
import numpy
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu

TOL_E_MIXED = 1e-6


@pytest.fixture(scope='module')
def b2():
    from pyscf_b200 import lib
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    return lib


def plan_for(b2, f, tol=1e-13):
    return b2.Plan(f['atm'], f['bas'], f['env'], cart=bool(f['cart']), direct_scf_tol=tol)


def test_mixed_tau_zero_is_fp64(b2):
    f = load_fixture('h2o8_vdz')
    p = plan_for(b2, f)
    p.set_mixed_threshold(0.0)
    vj, vk = p.get_jk(f['dm_conv'], hermi=1, precision=b2.PREC_MIXED)
    assert p.stats()['fp32_quartets'] == 0
    assert abs(vj - f['vj_conv']).max() < 1e-10
    assert abs(vk - f['vk_conv']).max() < 1e-10


@pytest.mark.parametrize('name', ['h2o8_vdz', 'h2o2_vtz'])
def test_mixed_all_fp32(b2, name):
    """tau above every bound: every quartet class (s..f) runs its float32
    kernel; the result keeps float32 accuracy against the reference."""
    f = load_fixture(name)
    p = plan_for(b2, f)
    p.set_mixed_threshold(1e30)
    vj, vk = p.get_jk(f['dm_rand'], hermi=1, precision=b2.PREC_MIXED)
    st = p.stats()
    assert st['fp32_quartets'] == st['quartets'] > 0
    assert abs(vj - f['vj_rand']).max() < 2e-5 * abs(f['vj_rand']).max()
    assert abs(vk - f['vk_rand']).max() < 2e-5 * abs(f['vk_rand']).max()
    # the split is exact: all quartets are still there
    p.set_mixed_threshold(0.0)
    p.get_jk(f['dm_rand'], hermi=1, precision=b2.PREC_MIXED)
    assert p.stats()['quartets'] == st['quartets']


def test_mixed_default_threshold(b2):
    f = load_fixture('h2o8_vdz')
    p = plan_for(b2, f)
    vj, vk = p.get_jk(f['dm_conv'], hermi=1, precision=b2.PREC_MIXED)
    st = p.stats()
    assert 0 < st['fp32_quartets'] < st['quartets']
    assert abs(vj - f['vj_conv']).max() < 1e-8
    assert abs(vk - f['vk_conv']).max() < 1e-8


def test_mixed_general_density(b2):
    f = load_fixture('h2o2_vtz')
    p = plan_for(b2, f)
    p.set_mixed_threshold(1e30)
    vj, vk = p.get_jk(f['dm_ns'], hermi=0, precision=b2.PREC_MIXED)
    assert abs(vj - f['vj_ns']).max() < 2e-5 * abs(f['vj_ns']).max()
    assert abs(vk - f['vk_ns']).max() < 2e-5 * abs(f['vk_ns']).max()


def test_mixed_scf_energy(b2):
    """RHF with incremental mixed-precision builds: as the density change
    shrinks, more quartets move to float32; the energy stays within 1e-6 Eh."""
    from pyscf_b200 import rhf
    f = load_fixture('h2o8_vdz')
    p = plan_for(b2, f)
    frac = []

    def get_jk(dm):
        r = p.get_jk(dm, hermi=1, precision=b2.PREC_MIXED)
        st = p.stats()
        frac.append(st['fp32_quartets'] / st['quartets'])
        return r
    conv, e, *_ = rhf.kernel(f['hcore'], f['ovlp'], int(f['nelec']), float(f['e_nuc']), get_jk, conv_tol=1e-10)
    assert conv
    assert abs(e - float(f['e_rhf'])) < TOL_E_MIXED
    assert frac[-1] > frac[0]


def test_c20h42_mixed_scf_report(b2):
    """C20H42/cc-pVDZ: FP64 and mixed-precision RHF with incremental builds;
    per build the mixed J/K against the FP64 J/K of the same density change,
    per iteration the energy against the FP64 SCF, and both final energies
    against the reference's RHF energy."""
    from pyscf_b200 import rhf
    f = load_fixture('c20h42_vdz')
    if 'hcore' not in f:
        pytest.skip('fixture without hcore (run tests/golden/make_golden.py c20h42_vdz)')
    p = plan_for(b2, f)
    rows, e64, e32, c64, c32 = rhf.mixed_precision_report(f['hcore'], f['ovlp'], int(f['nelec']), float(f['e_nuc']),
                                                          p, tau=1e-6, conv_tol=1e-10)
    assert c64 and c32
    assert abs(e64 - float(f['e_rhf'])) < 1e-9
    assert abs(e32 - float(f['e_rhf'])) < TOL_E_MIXED
    assert max(r['max_dJ'] for r in rows) < 1e-8
    assert max(r['max_dK'] for r in rows) < 1e-8
    assert rows[-1]['fp32_fraction'] > rows[0]['fp32_fraction']


def test_class_thresholds_and_mixed_tuner():
    """Per-class float32 thresholds: all zero is the FP64 build; the tuner's
    choice keeps E2 within its budget of the FP64 build and of the
    reference's J/K."""
    import numpy
    from pyscf_b200 import lib
    from conftest import load_fixture
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    f = load_fixture('h2o8_vdz')
    p = lib.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13)
    d = f['dm_conv']
    p.set_class_thresholds(numpy.zeros(55))
    vj, vk = p.get_jk(d, hermi=1, precision=lib.PREC_MIXED)
    assert p.stats()['fp32_quartets'] == 0
    assert abs(vj - f['vj_conv']).max() < 1e-10 and abs(vk - f['vk_conv']).max() < 1e-10
    with pytest.raises(RuntimeError):
        p.set_class_thresholds(numpy.zeros(54))
    res = p.autotune_mixed(d, budget=1e-7)
    tau = p.class_thresholds()
    assert res['tau'] in (0.0, 1e-2, 1e-3, 1e-4, 1e-5, 1e-6, 1e-7, 1e-8)
    assert set(numpy.unique(tau)) <= {0.0, res['tau']}
    assert abs(res['dE2']) <= 1e-7
    vj, vk = p.get_jk(d, hermi=1, precision=lib.PREC_MIXED)
    e2 = 0.5 * numpy.sum(d * vj) - 0.25 * numpy.sum(d * vk)
    e2_ref = 0.5 * numpy.sum(d * f['vj_conv']) - 0.25 * numpy.sum(d * f['vk_conv'])
    assert abs(e2 - e2_ref) <= 2e-7
    # back to the single threshold
    p.set_mixed_threshold(1e-6)
    assert (p.class_thresholds() == 1e-6).all()
