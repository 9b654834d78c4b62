"""Closed-shell SCF loop on top of the GPU J/K build.

A compact restatement of pyscf.scf.hf.kernel (pyscf/scf/hf.py:47-242) for
callers that have the one-electron matrices but not PySCF itself (the GPU
parity tests and the benchmark replay the reference SCF this way):
  * Fock F = h + V, V built incrementally from the density change,
    V_n = V_{n-1} + J[dD] - K[dD]/2  (RHF.get_veff, pyscf/scf/hf.py:2416-2427);
  * commutator DIIS on F with error F D S - S D F (CDIIS, pyscf/scf/diis.py);
  * aufbau occupation of the lowest nelec/2 orbitals, D = 2 C_occ C_occ^T;
  * converged when |dE| < conv_tol and |grad| < sqrt(conv_tol)
    (pyscf/scf/hf.py:194-200).
"""
import numpy
import scipy.linalg


class _DIIS:
    def __init__(self, space=8):
        self.space = space
        self.vecs = []
        self.errs = []

    def update(self, f, err):
        self.vecs.append(f.copy())
        self.errs.append(err.ravel().copy())
        if len(self.vecs) > self.space:
            self.vecs.pop(0)
            self.errs.pop(0)
        n = len(self.vecs)
        if n < 2:
            return f
        B = numpy.empty((n + 1, n + 1))
        B[-1, :] = B[:, -1] = -1
        B[-1, -1] = 0
        for i in range(n):
            for j in range(i + 1):
                B[i, j] = B[j, i] = numpy.dot(self.errs[i], self.errs[j])
        rhs = numpy.zeros(n + 1)
        rhs[-1] = -1
        try:
            c = numpy.linalg.solve(B, rhs)
        except numpy.linalg.LinAlgError:
            return f
        return sum(ci * v for ci, v in zip(c[:n], self.vecs))


def kernel(h1e, s1e, nelec, e_nuc, get_jk, conv_tol=1e-10, max_cycle=100, diis_space=8, dm0=None):
    """Returns (converged, e_tot, dm, mo_energy, mo_coeff, ncycle).

    get_jk(dm) -> (vj, vk) for one symmetric density."""
    nocc = int(nelec) // 2
    if dm0 is None:
        e, c = scipy.linalg.eigh(h1e, s1e)
        dm = 2 * c[:, :nocc] @ c[:, :nocc].T
    else:
        dm = numpy.asarray(dm0)
    vj, vk = get_jk(dm)
    vhf = vj - 0.5 * vk
    e_tot = numpy.einsum('ij,ji->', dm, h1e) + 0.5 * numpy.einsum('ij,ji->', dm, vhf) + e_nuc
    diis = _DIIS(diis_space)
    conv = False
    mo_e = mo_c = None
    cycle = 0
    for cycle in range(1, max_cycle + 1):
        f = h1e + vhf
        err = f @ dm @ s1e
        err = err - err.T
        f = diis.update(f, err)
        mo_e, mo_c = scipy.linalg.eigh(f, s1e)
        dm_new = 2 * mo_c[:, :nocc] @ mo_c[:, :nocc].T
        vj, vk = get_jk(dm_new - dm)
        vhf = vhf + vj - 0.5 * vk
        dm = dm_new
        e_last = e_tot
        e_tot = numpy.einsum('ij,ji->', dm, h1e) + 0.5 * numpy.einsum('ij,ji->', dm, vhf) + e_nuc
        fock = h1e + vhf
        g = mo_c[:, nocc:].T @ fock @ mo_c[:, :nocc]
        if abs(e_tot - e_last) < conv_tol and numpy.linalg.norm(g) < numpy.sqrt(conv_tol):
            conv = True
            break
    return conv, e_tot, dm, mo_e, mo_c, cycle
