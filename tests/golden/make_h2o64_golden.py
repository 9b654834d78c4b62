"""Reference J/K of the (H2O)64/cc-pVTZ bench workload and its 16/32-water samples.

Runs only where the reference checkout is readable (this container): the
reference's own direct-SCF driver, PySCF's CVHFnr_direct_drv with
CVHFdot_nrs8, CVHFnrs8_prescreen (direct_scf_tol = 1e-13) and the
'ji->s2kl' / 'li->s2kj' scripts (pyscf/scf/_vhf.py:405-464,
pyscf/lib/vhf/nr_direct.c:355-476), compiled from the reference sources by
oracle/build.py on the oracle integral library, through oracle.ref_driver.

The density is the bench density D = C C^T, C (nao x min(320, nao)) with
N(0,1)/sqrt(nao) entries from numpy.random.default_rng(304), regenerated on
the GPU box from the same seed (bench.load_workload).  The full matrices are
too large to commit (110 MB each at nao = 3712), so each fixture keeps:

  rows            AO indices of sampled shells (all shell types, centre and
                  corner waters), the reference vj/vk on those rows (all
                  columns), vj_rows / vk_rows;
  fp_j, fp_k      PySCF's lib.fp fingerprints of the whole vj, vk
                  (pyscf/lib/misc.py:1259-1263), a checksum over every element;
  e2              1/2 tr(D vj) - 1/4 tr(D vk), the two-electron energy of D;
  colsum_j/k      column sums of vj and vk (every element enters one of them);
  wall_s, threads time and OpenMP threads of the reference build.

    OMP_NUM_THREADS=8 python tests/golden/make_h2o64_golden.py [sub16 sub32 full]

The full workload is about 1.8e10 quartets: ~2 h on 8 cores, run once.
"""
import os
import sys
import time

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref_driver  # noqa: E402

NAMES = {'sub16': 'h2o64_vtz_sub16', 'sub32': 'h2o64_vtz_sub32', 'full': 'h2o64_vtz'}
# per water (cc-pVTZ, PySCF shell order): O  s[nctr 2] s s p p p d d f, then
# two H  s s s p p d
SHELLS_PER_WATER = 21
# (water, shell within the water): O contracted s, O p, O d, O f, H p, H d
SAMPLE = [(0, 0), (0, 12), (-1, 3), (-1, 8), ('mid', 6), ('mid', 8), ('mid', 14), ('mid', 20)]


def density(nao):
    rng = numpy.random.default_rng(304)
    c = rng.standard_normal((nao, min(320, nao))) / numpy.sqrt(nao)
    return c @ c.T


def lib_fp(a):
    a = numpy.asarray(a)
    return float(numpy.dot(numpy.cos(numpy.arange(a.size)), a.ravel()))


def sample_rows(bas, ao_loc):
    nw = bas.shape[0] // SHELLS_PER_WATER
    shells = []
    for w, s in SAMPLE:
        w = nw // 2 if w == 'mid' else (w % nw)
        shells.append(w * SHELLS_PER_WATER + s)
    rows = numpy.concatenate([numpy.arange(ao_loc[i], ao_loc[i + 1]) for i in shells])
    return numpy.array(shells, dtype=numpy.int32), rows.astype(numpy.int32)


def make(tag):
    name = NAMES[tag]
    f = dict(numpy.load(os.path.join(HERE, 'mol_%s.npz' % name)))
    nao = int(f['nao'])
    dm = density(nao)
    opt = ref_driver.RefVHFOpt(f['atm'], f['bas'], f['env'], 1e-13)
    t0 = time.time()
    vj, vk = ref_driver.direct(dm, opt, hermi=1)
    wall = time.time() - t0
    shells, rows = sample_rows(f['bas'], opt.ao_loc)
    out = dict(workload=name, shells=shells, rows=rows, vj_rows=vj[rows], vk_rows=vk[rows],
               fp_j=lib_fp(vj), fp_k=lib_fp(vk), e2=float(0.5 * numpy.sum(dm * vj) - 0.25 * numpy.sum(dm * vk)),
               colsum_j=vj.sum(axis=0), colsum_k=vk.sum(axis=0), wall_s=wall,
               threads=int(os.environ.get('OMP_NUM_THREADS', '0')), direct_scf_tol=1e-13,
               density='C C^T, C nao x min(320, nao) N(0,1)/sqrt(nao), numpy default_rng(304)')
    path = os.path.join(HERE, 'jk_%s.npz' % name)
    numpy.savez_compressed(path, **out)
    print('%s nao=%d  %.0f s  fp_j=%.12g fp_k=%.12g e2=%.12f -> %s' % (name, nao, wall, out['fp_j'], out['fp_k'],
                                                                        out['e2'], path), flush=True)


if __name__ == '__main__':
    for t in sys.argv[1:] or ['sub16', 'sub32', 'full']:
        make(t)
