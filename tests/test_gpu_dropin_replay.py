"""Every J/K call an unmodified PySCF makes, answered by the GPU engine.

PySCF cannot be imported on the GPU box, so the unmodified reference runs
where it can (tests/golden/make_dropin_trace.py): scf.RHF(H2O/cc-pVDZ) with
the direct path, mf.get_j / mf.get_k, and grad.RHF(mf).kernel(), with
recorders on pyscf.scf._vhf.direct and pyscf.grad.rhf.get_jk -- the two
module attributes patch_pyscf() / patch_pyscf_grad() rebind.  Here each
recorded call is replayed through the drop-ins those patches install
(pyscf_b200.scf.get_jk -> pyscf_b200._vhf.direct with a pyscf_b200 VHFOpt
carrying the recorded prescreen, and pyscf_b200.grad.get_jk) and compared
with the reference's own result: J/K and gradient J/K to 1e-10, and the RHF
energy rebuilt from the final density to 1e-9 Eh.
"""
import os

import numpy
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL_JK = 1e-10
TOL_E = 1e-9


class _Mol:
    """The attributes of a PySCF Mole that the drop-ins read."""

    def __init__(self, f):
        self._atm, self._bas, self._env = f['atm'], f['bas'], f['env']
        self.cart = bool(f['cart'])


@pytest.fixture(scope='module')
def trace():
    from pyscf_b200 import lib
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    path = os.path.join(GOLDEN, 'dropin_trace_h2o_vdz.npz')
    if not os.path.exists(path):
        pytest.skip('trace missing (run tests/golden/make_dropin_trace.py)')
    return dict(numpy.load(path))


def _calls(f):
    for i in range(int(f['ncalls'])):
        c = {k[4:]: v for k, v in f.items() if k.startswith('c%02d_' % i)}
        c['kind'] = str(c['kind'])
        yield i, c


def test_every_recorded_call_matches_the_reference(trace):
    from pyscf_b200 import _vhf, scf as b2scf, grad as b2grad
    mol = _Mol(trace)
    opt = _vhf.VHFOpt(mol, 'int2e', 'CVHFnrs8_prescreen', 'CVHFnr_int2e_q_cond', 'CVHFnr_dm_cond', 1e-13)
    kinds = []
    for i, c in _calls(trace):
        kinds.append(c['kind'])
        if c['kind'] == 'jk':
            opt.prescreen = str(c['screen'])
            wj, wk = bool(c['with_j']), bool(c['with_k'])
            vj, vk = b2scf.get_jk(mol, c['dm'], int(c['hermi']), opt, wj, wk)
            if wj:
                assert abs(vj - c['vj']).max() < TOL_JK, i
            if wk:
                assert abs(vk - c['vk']).max() < TOL_JK, i
            opt.prescreen = 'CVHFnrs8_prescreen'
        else:
            vj, vk = b2grad.get_jk(mol, c['dm'])
            assert abs(vj - c['vj']).max() < TOL_JK, i
            assert abs(vk - c['vk']).max() < TOL_JK, i
    # the trace covers the SCF builds, the J-only / K-only screens and the gradient
    assert kinds.count('jk') >= 10 and 'grad' in kinds


def test_energy_from_the_final_density(trace):
    from pyscf_b200 import _vhf, scf as b2scf
    mol = _Mol(trace)
    opt = _vhf.VHFOpt(mol, direct_scf_tol=1e-13)
    d = trace['dm_final']
    vj, vk = b2scf.get_jk(mol, d, 1, opt)
    e = float(trace['e_nuc'] + numpy.sum(trace['hcore'] * d) + 0.5 * numpy.sum(d * (vj - 0.5 * vk)))
    assert abs(e - float(trace['e_rhf'])) < TOL_E
    # pyscf/scf/test/test_h2o_vdz.py:98 (forced direct)
    assert abs(e - (-76.026765673120565)) < TOL_E
