"""The drop-in boundary on an unmodified PySCF (CPU; needs the reference).

tests/dropin/run_patched_pyscf.py runs the reference's own scf.RHF and
grad.RHF with pyscf_b200.patch_pyscf() / patch_pyscf_grad(), with the engine
underneath replaced by the oracle (no GPU here): the run must go through
pyscf_b200's entry points (_vhf.direct, VHFOpt, grad.get_jk) and reproduce
the unpatched reference energy and gradient.  Skipped where the reference is
not importable (the GPU box).
"""
import json
import os
import subprocess
import sys

import numpy
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _env():
    sys.path.insert(0, ROOT)
    from oracle import build as ob
    if not ob.ref_available():
        pytest.skip('the reference package is not importable here')
    ob.build_all()
    return ob.reference_env()


def test_unmodified_pyscf_runs_through_pyscf_b200():
    env = _env()
    r = subprocess.run([sys.executable, os.path.join(ROOT, 'tests', 'dropin', 'run_patched_pyscf.py')],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert all(out['routed']) and all(out['restored'])
    assert out['calls']['get_jk'] > 5 and out['calls']['grad_jk'] >= 1
    assert abs(out['e_patched'] - out['e_ref']) < 1e-9
    assert abs(numpy.array(out['g_patched']) - numpy.array(out['g_ref'])).max() < 1e-7
