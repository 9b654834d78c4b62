"""Reference J/K of 16 molecules of the 512-molecule batch workload.

Runs only where the reference checkout is readable (this container): the
reference's direct-SCF driver (PySCF's CVHFnr_direct_drv, CVHFnrs8_prescreen
at 1e-13, compiled from the reference sources on the oracle integral library,
oracle.ref_driver) on molecules 0, 32, 64, ..., 480 of
tests/golden/batch_h2o_vdz512.npz, each with the density the batch bench
gives it: D_m = C_m C_m^T, C_m (nao_m x 5 n_m) with N(0,1)/sqrt(nao_m)
entries drawn in molecule order from numpy.random.default_rng(405).
Stored per sampled molecule: its index, PySCF's fingerprints of vj and vk,
E2 = 1/2 tr(D J) - 1/4 tr(D K), and full vj/vk rows of its first three
shells (J/K of the whole batch are built on the GPU and these molecules
compared, tests/test_gpu_batch.py).

    OMP_NUM_THREADS=8 python tests/golden/make_batch_jk_golden.py
"""
import os
import sys

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref_driver  # noqa: E402

SAMPLE = list(range(0, 512, 32))


def densities(f):
    rng = numpy.random.default_rng(405)
    out = []
    for m in range(len(f['nao'])):
        nao, nocc = int(f['nao'][m]), 5 * int(f['nwater'][m])
        c = rng.standard_normal((nao, nocc)) / numpy.sqrt(nao)
        out.append(c @ c.T)
    return out


def lib_fp(a):
    a = numpy.asarray(a)
    return float(numpy.dot(numpy.cos(numpy.arange(a.size)), a.ravel()))


def main():
    f = dict(numpy.load(os.path.join(HERE, 'batch_h2o_vdz512.npz')))
    dms = densities(f)
    out = {'sample': numpy.array(SAMPLE)}
    for m in SAMPLE:
        a0, a1 = f['atm_off'][m], f['atm_off'][m + 1]
        b0, b1 = f['bas_off'][m], f['bas_off'][m + 1]
        e0, e1 = f['env_off'][m], f['env_off'][m + 1]
        opt = ref_driver.RefVHFOpt(f['atm'][a0:a1], f['bas'][b0:b1], f['env'][e0:e1], 1e-13)
        vj, vk = ref_driver.direct(dms[m], opt, hermi=1)
        rows = numpy.arange(opt.ao_loc[0], opt.ao_loc[3])
        d = dms[m]
        out['m%03d_fp_j' % m] = lib_fp(vj)
        out['m%03d_fp_k' % m] = lib_fp(vk)
        out['m%03d_e2' % m] = float(0.5 * numpy.sum(d * vj) - 0.25 * numpy.sum(d * vk))
        out['m%03d_rows' % m] = rows
        out['m%03d_vj_rows' % m] = vj[rows]
        out['m%03d_vk_rows' % m] = vk[rows]
        print(m, int(f['nwater'][m]), vj.shape[0], out['m%03d_e2' % m], flush=True)
    numpy.savez_compressed(os.path.join(HERE, 'batch_jk_sample.npz'), **out)


if __name__ == '__main__':
    main()
