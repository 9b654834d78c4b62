"""One-electron integrals on the GPU (b200jk_int1e): overlap and core
Hamiltonian (kinetic + nuclear attraction) against the reference's
SCF.get_ovlp / get_hcore (pyscf/scf/hf.py:315-347), stored in the fixtures
by tests/golden/make_golden.py; and a full RHF whose every integral is
computed on the GPU reproduces the reference energy
(pyscf/scf/test/test_h2o_vdz.py:98, forced direct).
"""
import numpy
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def b2():
    from pyscf_b200 import lib
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    return lib


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o_vdz', 'h2o2_vtz', 'h2o8_vdz', 'c20h42_vdz'])
def test_overlap_and_core_hamiltonian(b2, name):
    f = load_fixture(name)
    p = b2.Plan(f['atm'], f['bas'], f['env'], cart=bool(f['cart']), direct_scf_tol=1e-13)
    S, H = p.int1e()
    assert abs(S - f['ovlp']).max() < 1e-12
    assert abs(H - f['hcore']).max() < 1e-10 * max(1.0, abs(f['hcore']).max())
    import torch
    Sd, Hd = p.int1e(device=True)
    assert abs(Sd.cpu().numpy() - S).max() == 0.0 and abs(Hd.cpu().numpy() - H).max() == 0.0


def test_rhf_with_gpu_integrals(b2):
    from pyscf_b200 import rhf
    f = load_fixture('h2o_vdz')
    p = b2.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13)
    S, H = p.int1e()
    conv, e, *_ = rhf.kernel(H, S, int(f['nelec']), float(f['e_nuc']), lambda d: p.get_jk(d, hermi=1),
                             conv_tol=1e-11)
    assert conv
    assert abs(e - -76.026765673120565) < 1e-9
