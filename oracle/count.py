"""Count the s8-unique shell quartets that pass PySCF's direct-SCF screens.

ORACLE / TEST INFRASTRUCTURE.  Restates CVHFnrs8_prescreen
(pyscf/lib/vhf/optimizer.c:90-117) over the canonical quartet set of
CVHFdot_nrs8 (pyscf/lib/vhf/nr_direct.c:182-230) with numpy, to give the
CPU baseline the same work-unit count the GPU engine reports.
"""
import numpy


def count_quartets(q_cond, dm_cond, tol=1e-13, screen=0):
    """screen 0: CVHFnrs8_prescreen; 1: CVHFnrs8_vj_prescreen (the two J
    terms); 2: CVHFnrs8_vk_prescreen (the four K terms) -- optimizer.c:90-167."""
    n = q_cond.shape[0]
    i, j = numpy.tril_indices(n)
    qp = q_cond[i, j]
    total = 0
    step = max(1, 4000000 // max(1, len(qp)))
    for s in range(0, len(qp), step):
        ij = numpy.arange(s, min(len(qp), s + step))
        kl = numpy.arange(len(qp))
        I, J = i[ij][:, None], j[ij][:, None]
        K, L = i[kl][None, :], j[kl][None, :]
        qq = qp[ij][:, None] * qp[None, :]
        d = numpy.zeros(qq.shape)
        if screen != 2:
            d = numpy.maximum(4 * dm_cond[J, I], 4 * dm_cond[L, K])
        if screen != 1:
            d = numpy.maximum(d, numpy.maximum(dm_cond[J, K], dm_cond[J, L]))
            d = numpy.maximum(d, numpy.maximum(dm_cond[I, K], dm_cond[I, L]))
        ok = (qq > tol) & (d * qq > tol) & (kl[None, :] <= ij[:, None])
        total += int(ok.sum())
    return total
