"""The C-ABI library builds, loads and exports every symbol of include/b200jk.h;
host-side argument checks behave without a GPU."""
import ctypes
import os
import re
import subprocess

import numpy
import pytest

from conftest import ROOT


def header_symbols():
    text = open(os.path.join(ROOT, 'include', 'b200jk.h')).read()
    return sorted(set(re.findall(r'^\s*(?:int|const char \*)\s*(b200jk_\w+)\s*\(', text, re.M)))


def test_header_declares_the_abi():
    syms = header_symbols()
    for s in ('b200jk_plan_create', 'b200jk_plan_destroy', 'b200jk_get_jk', 'b200jk_get_q_cond',
              'b200jk_last_error', 'b200jk_stats'):
        assert s in syms


def test_library_exports_every_header_symbol():
    from pyscf_b200 import lib
    lib.load()
    out = subprocess.run(['nm', '-D', '--defined-only', lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if l.strip())
    missing = [s for s in header_symbols() if s not in exported]
    assert not missing, missing
    assert set(lib.EXPORTS) == set(header_symbols())


def test_library_is_sm100a():
    from pyscf_b200 import lib
    out = subprocess.run(['cuobjdump', '--list-elf', lib.LIB_PATH], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip('cuobjdump unavailable')
    assert 'sm_100a' in out.stdout


def test_version_and_errors_without_device():
    from pyscf_b200 import lib
    l = lib.load()
    assert l.b200jk_version() >= 1
    if lib.device_count() > 0:
        pytest.skip('a GPU is visible; covered by the gpu tests')
    atm = numpy.zeros((1, 6), numpy.int32)
    bas = numpy.zeros((1, 8), numpy.int32)
    env = numpy.zeros(30)
    with pytest.raises(lib.B200JKError) as e:
        lib.Plan(atm, bas, env)
    assert e.value.code in (lib.B200JK_ECUDA, lib.B200JK_EINVAL)


def test_null_arguments_rejected():
    from pyscf_b200 import lib
    l = lib.load()
    h = ctypes.c_void_p()
    rc = l.b200jk_plan_create(None, 0, None, 0, None, 0, 0, 1e-13, 0, ctypes.byref(h))
    assert rc == lib.B200JK_EINVAL
    assert b'NULL' in l.b200jk_last_error() or b'empty' in l.b200jk_last_error()
    rc = l.b200jk_get_jk(None, None, 0, 1, 1, 1, None, None, 0, 0, None)
    assert rc == lib.B200JK_EINVAL
