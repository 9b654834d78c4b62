"""Run an unmodified PySCF with pyscf_b200 patched in (driver of tests/test_dropin.py).

Executed in a subprocess with the reference importable (this container).  No
GPU exists here, so the engine underneath the patched entry points --
pyscf_b200.lib.Plan, the one class that talks to libb200jk -- is replaced by a
CPU stand-in that answers from the oracle.  Everything above it is the real
code path: pyscf.scf._vhf.direct rebound to pyscf_b200._vhf.direct,
SCF.init_direct_scf returning pyscf_b200's VHFOpt, RHF.get_jk taking the direct
branch, pyscf.grad.rhf.get_jk rebound to pyscf_b200.grad.get_jk.  Prints one
JSON line: energies and gradients with and without the patch, and how many
times the stand-in engine was called.
"""
import json
import os
import sys

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from pyscf import gto, scf, grad  # noqa: E402
import pyscf_b200  # noqa: E402
from pyscf_b200 import lib as b2lib, grad as b2grad  # noqa: E402

calls = {'get_jk': 0, 'grad_jk': 0}


class OraclePlan:
    """CPU stand-in for lib.Plan with the attributes the Python layer uses."""

    def __init__(self, atm, bas, env, cart=False, direct_scf_tol=1e-13, device=0):
        self.atm = numpy.asarray(atm, dtype=numpy.int32)
        self.bas = numpy.asarray(bas, dtype=numpy.int32)
        self.env = numpy.asarray(env, dtype=numpy.double)
        self.cart = bool(cart)
        self.direct_scf_tol = float(direct_scf_tol)
        self.nao = oracle.nao(self.bas, self.cart)
        self.nbas = self.bas.shape[0]

    def close(self):
        pass

    def set_prescreen(self, screen=0):
        # the oracle always applies the s8 screen; the J-only / K-only screens
        # drop only quartets below the threshold, far under this test's tolerance
        self.screen = screen

    @property
    def q_cond(self):
        return oracle.q_cond(self.atm, self.bas, self.env, self.cart, self.direct_scf_tol)

    def get_jk(self, dms, hermi=1, with_j=True, with_k=True, out_j=None, out_k=None, precision=0, stream=None):
        calls['get_jk'] += 1
        tol = self.direct_scf_tol
        vj, vk, _ = oracle.get_jk(dms, self.atm, self.bas, self.env, hermi=hermi, cart=self.cart,
                                  direct_scf_tol=tol if tol > 0 else 1e-13, screen=tol > 0)
        if out_j is not None and with_j:
            out_j[...] = vj.reshape(out_j.shape)
            vj = out_j
        if out_k is not None and with_k:
            out_k[...] = vk.reshape(out_k.shape)
            vk = out_k
        return (vj if with_j else None), (vk if with_k else None)

    def grad_jk(self, dm, with_j=True, with_k=True, direct_scf_tol=1e-14):
        calls['grad_jk'] += 1
        return oracle.grad_jk(dm, self.atm, self.bas, self.env, self.cart, direct_scf_tol)


def main():
    mol = gto.M(atom='O 0 0 0; H 0 -0.757 0.587; H 0 0.757 0.587', basis='631g', verbose=0)
    # reference, unpatched, forced direct as pyscf/scf/test/test_h2o_vdz.py:94-98
    mf0 = scf.RHF(mol)
    mf0.max_memory = 0
    mf0.conv_tol = 1e-11
    e0 = mf0.kernel()
    g0 = grad.RHF(mf0).kernel()
    # patched: an unmodified SCF and gradient run
    b2lib.Plan = OraclePlan
    pyscf_b200.patch_pyscf()
    b2grad.patch_pyscf_grad()
    import pyscf.scf._vhf as ref_vhf
    import pyscf.grad.rhf as ref_grad
    routed = (ref_vhf.direct is pyscf_b200._vhf.direct, ref_grad.get_jk is b2grad.get_jk)
    mf1 = scf.RHF(mol)
    mf1.conv_tol = 1e-11
    e1 = mf1.kernel()
    g1 = grad.RHF(mf1).kernel()
    pyscf_b200.unpatch_pyscf()
    b2grad.unpatch_pyscf_grad()
    print(json.dumps({'e_ref': e0, 'e_patched': e1, 'g_ref': g0.tolist(), 'g_patched': g1.tolist(),
                      'calls': calls, 'routed': routed,
                      'restored': (ref_vhf.direct is not pyscf_b200._vhf.direct,
                                   ref_grad.get_jk is not b2grad.get_jk)}))


if __name__ == '__main__':
    main()
