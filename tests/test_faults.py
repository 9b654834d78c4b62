"""Host-side fault handling of the C ABI (no GPU needed).

The reference reports these conditions by assert/exit in C
(pyscf/lib/vhf/optimizer.c:396-400, pyscf/lib/vhf/nr_direct_dot.c:24-25) or by
RuntimeError in Python (pyscf/scf/_vhf.py:594-597); the engine returns a
status code and a message instead, and checks the molecule arrays on the host
before it touches a GPU, so every case here runs on a CPU-only machine.
The device-side counterparts (an allocation failure forced by the test hook,
host memory passed as device memory, NaN densities) are in
tests/test_gpu_faults.py.
"""
import ctypes

import numpy
import pytest

from conftest import load_fixture


def _create(atm, bas, env, tol=1e-13):
    from pyscf_b200 import lib
    l = lib.load()
    h = ctypes.c_void_p()
    atm = numpy.ascontiguousarray(atm, dtype=numpy.int32)
    bas = numpy.ascontiguousarray(bas, dtype=numpy.int32)
    env = numpy.ascontiguousarray(env, dtype=numpy.double)
    rc = l.b200jk_plan_create(atm.ctypes.data_as(ctypes.c_void_p), atm.shape[0],
                              bas.ctypes.data_as(ctypes.c_void_p), bas.shape[0],
                              env.ctypes.data_as(ctypes.c_void_p), env.size, 0, tol, 0, ctypes.byref(h))
    msg = l.b200jk_last_error().decode()
    if rc == lib.B200JK_OK:
        l.b200jk_plan_destroy(h)
    return rc, msg


@pytest.fixture(scope='module')
def h2o():
    return load_fixture('h2o_631g')


def test_g_shell_is_unsupported(h2o):
    from pyscf_b200 import lib
    bas = h2o['bas'].copy()
    bas[0, 1] = 4            # l = 4 (g): beyond the l <= 3 kernels
    rc, msg = _create(h2o['atm'], bas, h2o['env'])
    assert rc == lib.B200JK_EUNSUPPORTED
    assert 'l > 3' in msg


def test_short_range_coulomb_is_not_a_plan(h2o):
    """env[PTR_RANGE_OMEGA] < 0 (erfc) has no plan of its own: the Python
    layer builds it as full minus long range; the C ABI says so."""
    from pyscf_b200 import lib
    env = h2o['env'].copy()
    env[8] = -0.3            # env[PTR_RANGE_OMEGA] (pyscf/gto/mole.py:76)
    rc, msg = _create(h2o['atm'], h2o['bas'], env)
    assert rc == lib.B200JK_EUNSUPPORTED
    assert 'short-range' in msg
    env[8] = float('nan')
    rc, msg = _create(h2o['atm'], h2o['bas'], env)
    assert rc == lib.B200JK_EINVAL


@pytest.mark.parametrize('slot, value, text', [
    (0, 99, 'atom index'),          # ATOM_OF beyond natm
    (0, -1, 'atom index'),
    (1, -1, 'negative angular'),    # ANG_OF
    (2, 0, 'empty shell'),          # NPRIM_OF
    (3, 0, 'empty shell'),          # NCTR_OF
    (5, 10 ** 6, 'outside env'),    # PTR_EXP
    (6, -5, 'outside env'),         # PTR_COEFF
])
def test_bad_bas_rows_rejected(h2o, slot, value, text):
    from pyscf_b200 import lib
    bas = h2o['bas'].copy()
    bas[1, slot] = value
    rc, msg = _create(h2o['atm'], bas, h2o['env'])
    assert rc == lib.B200JK_EINVAL, msg
    assert text in msg


def test_bad_coordinate_pointer_rejected(h2o):
    from pyscf_b200 import lib
    atm = h2o['atm'].copy()
    atm[0, 1] = h2o['env'].size     # PTR_COORD past the end of env
    rc, msg = _create(atm, h2o['bas'], h2o['env'])
    assert rc == lib.B200JK_EINVAL
    assert 'coordinate' in msg


def test_valid_molecule_passes_the_host_checks(h2o):
    """A valid molecule gets past the host checks: without a GPU the first
    failure is the missing device, not the arrays."""
    from pyscf_b200 import lib
    rc, msg = _create(h2o['atm'], h2o['bas'], h2o['env'])
    if lib.device_count() > 0:
        assert rc == lib.B200JK_OK
    else:
        assert rc == lib.B200JK_ECUDA and 'device' in msg


def test_alloc_hook_arguments():
    from pyscf_b200 import lib
    l = lib.load()
    assert l.b200jk_debug_fail_alloc(-1) == lib.B200JK_EINVAL
    assert l.b200jk_debug_fail_alloc(0) == lib.B200JK_OK


def test_python_layer_rejects_other_intors_and_screens(h2o):
    """VHFOpt accepts what the engine implements -- the int2e Coulomb family
    (full, long and short range through env[PTR_RANGE_OMEGA]) with the
    reference's s8, J-only and K-only screens -- and refuses the rest before
    any device work."""
    from pyscf_b200 import _vhf

    class Mol:
        _atm, _bas, _env, cart = h2o['atm'], h2o['bas'], h2o['env'], False
    with pytest.raises(NotImplementedError):
        _vhf.VHFOpt(Mol(), intor='int2e_ip1')
    with pytest.raises(NotImplementedError):
        _vhf.VHFOpt(Mol(), prescreen='CVHFgrad_jk_prescreen')


def test_incore_shape_checks_before_any_device_work():
    """_vhf.incore raises RuntimeError when the tensor fits neither symmetry
    (pyscf/scf/_vhf.py:397-399); the C ABI returns EINVAL with the same text
    before it looks for a GPU."""
    from pyscf_b200 import lib, incore
    l = lib.load()
    nao = 4
    dm = numpy.eye(nao)
    out = numpy.empty((nao, nao))
    bad = numpy.zeros(7)
    rc = l.b200jk_incore_jk(lib._ptr(bad), bad.size, nao, lib._ptr(dm), 1, 1, 1, 1, lib._ptr(out), lib._ptr(out),
                            0, 0, None)
    assert rc == lib.B200JK_EINVAL
    assert 'Array shape not consistent' in l.b200jk_last_error().decode()
    with pytest.raises(RuntimeError, match='Array shape not consistent'):
        incore.incore(bad, dm, hermi=1)
    rc = l.b200jk_incore_jk(lib._ptr(bad), bad.size, nao, lib._ptr(dm), 1, 3, 1, 1, lib._ptr(out), lib._ptr(out),
                            0, 0, None)
    assert rc == lib.B200JK_EINVAL
    assert incore.incore(bad, dm, with_j=False, with_k=False) == (None, None)
