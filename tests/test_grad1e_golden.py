"""The one-electron gradient fixtures (tests/golden/make_grad1e_golden.py)
against the reference's whole RHF gradient: de_1e + de_2e + de_nuc = grad.RHF
(grad_*.npz).  The energy-weighted density of the fixtures is 1/2 D F D of
the converged density, equal to the orbital one up to the SCF convergence,
so the sum agrees to 5e-8 Eh/Bohr."""
import os

import numpy
import pytest

from conftest import GOLDEN


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o2_vtz', 'h2o16_vdz'])
def test_grad1e_fixture_sums_to_reference_gradient(name):
    p1 = os.path.join(GOLDEN, 'grad1e_%s.npz' % name)
    p2 = os.path.join(GOLDEN, 'grad_%s.npz' % name)
    if not (os.path.exists(p1) and os.path.exists(p2)):
        pytest.skip('fixtures missing')
    g1, g = dict(numpy.load(p1)), dict(numpy.load(p2))
    total = g1['de_1e'] + g['de_2e'] + g1['de_nuc']
    assert abs(total - g['de']).max() < 5e-8
    # the energy-weighted density is symmetric, as the GPU kernel assumes
    assert abs(g1['dme0'] - g1['dme0'].T).max() < 1e-10
