import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, 'tests', 'golden')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200); parity tests of the CUDA path')


def load_fixture(name):
    import numpy
    path = os.path.join(GOLDEN, 'mol_%s.npz' % name)
    if not os.path.exists(path):
        pytest.skip('fixture %s missing (run tests/golden/make_golden.py)' % name)
    return dict(numpy.load(path))


def lib_fp(a):
    """PySCF's fingerprint lib.fp (pyscf/lib/misc.py:1259-1263)."""
    import numpy
    a = numpy.asarray(a)
    return numpy.dot(numpy.cos(numpy.arange(a.size)), a.ravel())
