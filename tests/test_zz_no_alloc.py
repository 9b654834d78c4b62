"""The allocation-free J/K entry point, b200jk_get_jk_noalloc.

It exists for callers that cannot let a library allocate device memory:
code running under a framework's caching allocator or a fixed device-memory
budget, where a cudaMalloc inside the call can fail (the pool holds the
memory) or stall the device.  It keeps all intermediates in one fixed
32 MiB scratch array inside the library.  Here it is called through the C ABI
and its J/K are compared with those of the regular entry point,
b200jk_get_jk, on two calls in a row (the scratch array keeps the previous
call's contents, so the second call checks that nothing stale leaks in).

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu

TOL_JK = 1e-10


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _noalloc(lib, plan, dm, hermi):
    import torch
    vj = torch.full_like(dm, float('nan'))
    vk = torch.full_like(dm, float('nan'))
    stream = torch.cuda.current_stream(dm.device).cuda_stream
    rc = lib.load().b200jk_get_jk_noalloc(plan._h, _ptr(dm), 1, hermi, 1, 1, _ptr(vj), _ptr(vk),
                                          ctypes.c_void_p(stream))
    lib.check(rc)
    torch.cuda.synchronize()
    return vj.cpu().numpy(), vk.cpu().numpy()


def test_noalloc_matches_get_jk_on_two_calls():
    import torch
    from pyscf_b200 import lib
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    f = load_fixture('h2o8_vdz')
    plan = lib.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13, device=0)
    for dm_host, hermi in ((f['dm_rand'], 1), (f['dm_ns'], 0)):
        dm = torch.tensor(dm_host, device='cuda:0')
        ref_j, ref_k = plan.get_jk(dm_host, hermi=hermi)
        for _ in range(2):
            vj, vk = _noalloc(lib, plan, dm, hermi)
            assert numpy.isfinite(vj).all() and numpy.isfinite(vk).all()
            assert abs(vj - ref_j).max() < TOL_JK
            assert abs(vk - ref_k).max() < TOL_JK
    # and against the reference drivers' output for the same density
    vj, vk = _noalloc(lib, plan, torch.tensor(f['dm_rand'], device='cuda:0'), 1)
    assert abs(vj - f['vj_rand']).max() < TOL_JK
    assert abs(vk - f['vk_rand']).max() < TOL_JK


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from pyscf_b200 import lib
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    f = load_fixture('h2o64_vtz_sub16')
    plan = lib.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13, device=0)
    dm = torch.zeros((plan.nao, plan.nao), dtype=torch.float64, device='cuda:0')
    with pytest.raises(lib.B200JKError) as e:
        _noalloc(lib, plan, dm, 1)
    assert e.value.code == lib.B200JK_EINVAL
    assert 'scratch' in str(e.value)
