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


def _noalloc(lib, plan, dm, hermi, with_j=True, with_k=True):
    """dm: (nao, nao) or (n_dm, nao, nao) CUDA tensor -> host vj, vk (None
    for what is not requested)."""
    import torch
    n_dm = 1 if dm.dim() == 2 else dm.shape[0]
    vj = torch.full_like(dm, float('nan'))
    vk = torch.full_like(dm, float('nan'))
    stream = torch.cuda.current_stream(dm.device).cuda_stream
    rc = lib.load().b200jk_get_jk_noalloc(plan._h, _ptr(dm), n_dm, hermi, int(with_j), int(with_k),
                                          _ptr(vj) if with_j else None, _ptr(vk) if with_k else None,
                                          ctypes.c_void_p(stream))
    lib.check(rc)
    torch.cuda.synchronize()
    return (vj.cpu().numpy() if with_j else None), (vk.cpu().numpy() if with_k else None)


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


@pytest.mark.parametrize('case', ['two_dms_hermi0', 'hermi2', 'j_only', 'k_only'])
def test_noalloc_variants_match_get_jk(case):
    """The scratch offsets depend on n_dm, hermi, with_j and with_k: every
    layout is compared with b200jk_get_jk, twice in a row."""
    import torch
    from pyscf_b200 import lib
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    f = load_fixture('h2o8_vdz')
    plan = lib.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13, device=0)
    wj = wk = True
    if case == 'two_dms_hermi0':
        dm_host, hermi = numpy.stack([f['dm_ns'], f['dm_rand']]), 0
    elif case == 'hermi2':
        dm_host, hermi = f['dm_ns'] - f['dm_ns'].T, 2
    elif case == 'j_only':
        dm_host, hermi, wk = f['dm_rand'], 1, False
    else:
        dm_host, hermi, wj = f['dm_rand'], 1, False
    ref_j, ref_k = plan.get_jk(dm_host, hermi=hermi, with_j=wj, with_k=wk)
    dm = torch.tensor(dm_host, device='cuda:0')
    for _ in range(2):
        vj, vk = _noalloc(lib, plan, dm, hermi, wj, wk)
        if wj:
            assert abs(vj.reshape(ref_j.shape) - ref_j).max() < TOL_JK
        if wk:
            assert abs(vk.reshape(ref_k.shape) - ref_k).max() < TOL_JK


def test_noalloc_rejects_host_memory():
    """Host arrays handed to the device-only entry point are an error, not a
    GPU fault."""
    from pyscf_b200 import lib
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    f = load_fixture('h2o_631g')
    plan = lib.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13, device=0)
    dm = numpy.ascontiguousarray(f['dm_rand'])
    vj = numpy.empty_like(dm)
    vk = numpy.empty_like(dm)
    rc = lib.load().b200jk_get_jk_noalloc(plan._h, dm.ctypes.data_as(ctypes.c_void_p), 1, 1, 1, 1,
                                          vj.ctypes.data_as(ctypes.c_void_p), vk.ctypes.data_as(ctypes.c_void_p),
                                          None)
    assert rc == lib.B200JK_EINVAL
    assert b'device memory' in lib.load().b200jk_last_error() or b'CUDA pointer' in lib.load().b200jk_last_error()


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
    # the message states the bytes needed against the 32 MiB the array holds
    import re
    m = re.search(r'needs (\d+) bytes .* holds (\d+) bytes', str(e.value))
    assert m, str(e.value)
    need, have = int(m.group(1)), int(m.group(2))
    assert have == 32 << 20 and need > have
