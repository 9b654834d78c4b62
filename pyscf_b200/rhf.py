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


def kernel(h1e, s1e, nelec, e_nuc, get_jk, conv_tol=1e-10, max_cycle=100, diis_space=8, dm0=None, energies=None):
    """Returns (converged, e_tot, dm, mo_energy, mo_coeff, ncycle).

    get_jk(dm) -> (vj, vk) for one symmetric density.  If `energies` is a
    list, the energy after every J/K build is appended to it."""
    nocc = int(nelec) // 2
    if dm0 is None:
        e, c = scipy.linalg.eigh(h1e, s1e)
        dm = 2 * c[:, :nocc] @ c[:, :nocc].T
    else:
        dm = numpy.asarray(dm0)
    vj, vk = get_jk(dm)
    vhf = vj - 0.5 * vk
    e_tot = numpy.einsum('ij,ji->', dm, h1e) + 0.5 * numpy.einsum('ij,ji->', dm, vhf) + e_nuc
    if energies is not None:
        energies.append(e_tot)
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
        if energies is not None:
            energies.append(e_tot)
        fock = h1e + vhf
        g = mo_c[:, nocc:].T @ fock @ mo_c[:, :nocc]
        if abs(e_tot - e_last) < conv_tol and numpy.linalg.norm(g) < numpy.sqrt(conv_tol):
            conv = True
            break
    return conv, e_tot, dm, mo_e, mo_c, cycle


def mixed_precision_report(h1e, s1e, nelec, e_nuc, plan, tau, conv_tol=1e-10, max_cycle=100):
    """Run the SCF twice on the GPU J/K build, in FP64 and in mixed precision
    (quartets with q_ij q_kl max|dD| < tau in float32), both with incremental
    Fock builds on the density change.  For every mixed build the FP64 build
    of the same dD is made too, so each build reports max|dJ|, max|dK| and the
    float32 fraction, and each iteration the energy difference to the FP64
    SCF at the same iteration.  Returns (rows, e_fp64, e_mixed,
    converged_fp64, converged_mixed)."""
    from . import lib

    def jk64(dm):
        plan.set_mixed_threshold(0.0)
        return plan.get_jk(dm, hermi=1, precision=lib.PREC_FP64)

    energies64 = []
    conv64, e64, *_ = kernel(h1e, s1e, nelec, e_nuc, jk64, conv_tol=conv_tol, max_cycle=max_cycle,
                             energies=energies64)
    rows = []

    def jk_mixed(dm):
        plan.set_mixed_threshold(tau)
        vj, vk = plan.get_jk(dm, hermi=1, precision=lib.PREC_MIXED)
        st = plan.stats()
        rj, rk = jk64(dm)
        rows.append({'build': len(rows), 'max_dJ': float(abs(vj - rj).max()), 'max_dK': float(abs(vk - rk).max()),
                     'fp32_fraction': st['fp32_quartets'] / max(1, st['quartets']),
                     'max_abs_dD': float(abs(dm).max())})
        return vj, vk
    energies32 = []
    conv32, e32, *_ = kernel(h1e, s1e, nelec, e_nuc, jk_mixed, conv_tol=conv_tol, max_cycle=max_cycle,
                             energies=energies32)
    for i, r in enumerate(rows):
        r['E_mixed'] = energies32[i] if i < len(energies32) else None
        r['E_fp64'] = energies64[i] if i < len(energies64) else None
        if r['E_mixed'] is not None and r['E_fp64'] is not None:
            r['dE'] = r['E_mixed'] - r['E_fp64']
    return rows, e64, e32, conv64, conv32
