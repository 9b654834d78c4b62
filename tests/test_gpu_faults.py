"""Fault handling on a GPU, without faulting the GPU.

* An out-of-memory condition is forced by the library's test hook
  (b200jk_debug_fail_alloc) instead of exhausting the device: plan creation
  and a build must return B200JK_ENOMEM, leave nothing behind, and the next
  calls must work.
* Host memory passed where device memory is declared is rejected on the host
  (cudaPointerGetAttributes) before any kernel could dereference it.
* A NaN density element propagates into J/K, as in the reference, and does
  not poison the plan for the next build.
"""
import ctypes

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
    yield lib
    lib.load().b200jk_debug_fail_alloc(0)


@pytest.mark.parametrize('nth', [1, 3, 7])
def test_forced_enomem_in_plan_create(b2, nth):
    f = load_fixture('h2o_vdz')
    b2.load().b200jk_debug_fail_alloc(nth)
    try:
        with pytest.raises(b2.B200JKError) as e:
            b2.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13)
        assert e.value.code == b2.B200JK_ENOMEM
        assert 'cudaMalloc' in str(e.value)
    finally:
        b2.load().b200jk_debug_fail_alloc(0)
    p = b2.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13)
    vj, vk = p.get_jk(f['dm_rand'], hermi=1)
    assert abs(vj - f['vj_rand']).max() < TOL_JK
    assert abs(vk - f['vk_rand']).max() < TOL_JK


def test_forced_enomem_in_first_build(b2):
    """The first build allocates the workspace: a failure there is reported
    and the plan builds correctly on the next call."""
    f = load_fixture('h2o_vdz')
    p = b2.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13)
    b2.load().b200jk_debug_fail_alloc(2)
    try:
        with pytest.raises(b2.B200JKError) as e:
            p.get_jk(f['dm_rand'], hermi=1)
        assert e.value.code == b2.B200JK_ENOMEM
    finally:
        b2.load().b200jk_debug_fail_alloc(0)
    vj, vk = p.get_jk(f['dm_rand'], hermi=1)
    assert abs(vj - f['vj_rand']).max() < TOL_JK
    assert abs(vk - f['vk_rand']).max() < TOL_JK


def test_host_memory_as_device_pointers_rejected(b2):
    f = load_fixture('h2o_631g')
    p = b2.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13)
    dm = numpy.ascontiguousarray(f['dm_rand'])
    vj = numpy.empty_like(dm)
    vk = numpy.empty_like(dm)
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    rc = b2.load().b200jk_get_jk(p._h, ptr(dm), 1, 1, 1, 1, ptr(vj), ptr(vk), 1, 0, None)
    assert rc == b2.B200JK_EINVAL
    rc = b2.load().b200jk_grad_jk(p._h, ptr(dm), 1, 1, 1, ptr(vj), ptr(vk), 1, 1e-14, None)
    assert rc == b2.B200JK_EINVAL
    # the same arrays as host arrays (dev_ptrs = 0) are fine
    vj2, vk2 = p.get_jk(dm, hermi=1)
    assert abs(vj2 - f['vj_rand']).max() < TOL_JK


def test_nan_density_propagates_and_plan_recovers(b2):
    f = load_fixture('h2o_vdz')
    p = b2.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13)
    dm = f['dm_rand'].copy()
    dm[0, 0] = float('nan')
    vj, vk = p.get_jk(dm, hermi=1)
    # J_ab = sum_cd (ab|cd) D_cd: every J element that meets D_00 is NaN, as
    # numpy would make it in the reference's driver
    assert numpy.isnan(vj).any()
    assert numpy.isnan(vj[0, 0]) and numpy.isnan(vk[0, 0])
    vj, vk = p.get_jk(f['dm_rand'], hermi=1)
    assert abs(vj - f['vj_rand']).max() < TOL_JK
    assert abs(vk - f['vk_rand']).max() < TOL_JK
