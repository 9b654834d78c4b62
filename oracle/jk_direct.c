/*
 * jk_direct.c — CPU restatement of PySCF's direct-SCF J/K build.
 *
 * ORACLE / TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it, and only as the checker.
 *
 * What it restates (PySCF 2.12.1):
 *   - Schwarz conditioner q_cond = sqrt(max |(ij|ij)|), floor 1e-100
 *     (CVHFnr_int2e_q_cond, pyscf/lib/vhf/optimizer.c:408-454);
 *   - density conditioner dm_cond_IJ = 1/2 max over sets and a in I, b in J of
 *     |D_ab| + |D_ba| (CVHFnr_dm_cond, optimizer.c:494-518);
 *   - the per-quartet screen (CVHFnrs8_prescreen, optimizer.c:90-117);
 *   - the canonical s8 quartet set i>=j, k>=l, ij>=kl
 *     (CVHFdot_nrs8, pyscf/lib/vhf/nr_direct.c:182-230);
 *   - the J script 'ji->s2kl' and K scripts 'li->s2kj' (hermi=1) /
 *     'li->s1kj' (hermi=0) of pyscf/scf/_vhf.py:427-437, i.e.
 *       vj[k,l] = sum_ij (ij|kl) D[j,i],   vk[k,j] = sum_il (ij|kl) D[l,i],
 *     followed by the hermi_triu mirroring of _vhf.py:454-463;
 *   - the gradient twin pyscf/grad/rhf.py:149-178 (int2e_ip1, s2kl,
 *     'lk->s1ij' and 'jk->s1il', CVHFgrad_jk_prescreen
 *     pyscf/lib/vhf/hessian_screen.c:44-68, q_cond planes from
 *     CVHFnr_int2e_pp_q_cond hessian_screen.c:70-123 and CVHFnr_int2e_q_cond).
 *
 * Here each unique quartet's integrals are scattered to all of their
 * symmetry images with weight 1/deg (deg = number of coinciding images), into
 * thread-private full matrices that are summed at the end.  The reference
 * accumulates triangles in 64-AO tiles and mirrors them; the two give the
 * same matrices up to summation order.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>
#include "cint/cint.h"

int int2e_sph(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
              double *env, CINTOpt *opt, double *cache);
int int2e_cart(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
               double *env, CINTOpt *opt, double *cache);
int int2e_ip1_sph(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
                  double *env, CINTOpt *opt, double *cache);
int int2e_ip1_cart(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
                   double *env, CINTOpt *opt, double *cache);
int int2e_ip1ip2_sph(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
                     double *env, CINTOpt *opt, double *cache);
int int2e_ip1ip2_cart(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
                      double *env, CINTOpt *opt, double *cache);
void oracle_boys(int mmax, double t, double *f);

typedef int (*intor_t)(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);

static void make_ao_loc(int *ao_loc, const int *bas, int nbas, int cart)
{
        ao_loc[0] = 0;
        for (int i = 0; i < nbas; i++) {
                int l = bas(ANG_OF, i);
                int nf = cart ? (l + 1) * (l + 2) / 2 : 2 * l + 1;
                ao_loc[i + 1] = ao_loc[i] + nf * bas(NCTR_OF, i);
        }
}

int oracle_nao(const int *bas, int nbas, int cart)
{
        int *ao_loc = malloc(sizeof(int) * (nbas + 1));
        make_ao_loc(ao_loc, bas, nbas, cart);
        int n = ao_loc[nbas];
        free(ao_loc);
        return n;
}

/* shared diagonal-quartet conditioner: q[ij] = sqrt(max over comps in
 * comp_sel of |(ij|ij)|), floor 1e-100.  ordered=0: pairs i >= j, mirrored
 * (CVHFnr_int2e_q_cond); ordered=1: every (i, j) on its own, not mirrored, as
 * the derivative conditioner is not symmetric (CVHFnr_int2e_pp_q_cond,
 * hessian_screen.c:70-123) */
static void q_cond_generic(double *q_cond, intor_t intor, int ncomp, const int *comp_sel, int nsel,
                           int *atm, int natm, int *bas, int nbas, double *env, int cart, int ordered)
{
        int *ao_loc = malloc(sizeof(int) * (nbas + 1));
        make_ao_loc(ao_loc, bas, nbas, cart);
        int dmax = 0;
        for (int i = 0; i < nbas; i++) dmax = MAX(dmax, ao_loc[i + 1] - ao_loc[i]);
        size_t npair = ordered ? (size_t)nbas * nbas : (size_t)nbas * (nbas + 1) / 2;
#pragma omp parallel
{
        double *buf = malloc(sizeof(double) * (size_t)dmax * dmax * dmax * dmax * ncomp);
#pragma omp for schedule(dynamic, 4)
        for (size_t ij = 0; ij < npair; ij++) {
                int ish, jsh;
                if (ordered) {
                        ish = (int)(ij / nbas);
                        jsh = (int)(ij - (size_t)ish * nbas);
                } else {
                        ish = (int)(sqrt(2 * (double)ij + .25) - .5 + 1e-7);
                        jsh = (int)(ij - (size_t)ish * (ish + 1) / 2);
                }
                int di = ao_loc[ish + 1] - ao_loc[ish];
                int dj = ao_loc[jsh + 1] - ao_loc[jsh];
                int shls[4] = {ish, jsh, ish, jsh};
                double qtmp = 1e-100;
                if ((*intor)(buf, NULL, shls, atm, natm, bas, nbas, env, NULL, NULL)) {
                        size_t n4 = (size_t)di * dj * di * dj;
                        for (int s = 0; s < nsel; s++) {
                                const double *b = buf + n4 * comp_sel[s];
                                for (int i = 0; i < di; i++)
                                for (int j = 0; j < dj; j++) {
                                        double t = fabs(b[i + (size_t)di * j + (size_t)di * dj * i + (size_t)di * dj * di * j]);
                                        qtmp = MAX(qtmp, t);
                                }
                        }
                        qtmp = sqrt(qtmp);
                }
                q_cond[(size_t)ish * nbas + jsh] = qtmp;
                if (!ordered) q_cond[(size_t)jsh * nbas + ish] = qtmp;
        }
        free(buf);
}
        free(ao_loc);
}

/* CVHFnr_int2e_q_cond restated (optimizer.c:408-454).  expcutoff mirrors
 * mol.with_integral_screen(direct_scf_tol**2) (pyscf/scf/_vhf.py:199). */
void oracle_q_cond(double *q_cond, int *atm, int natm, int *bas, int nbas, double *env,
                   int cart, double expcutoff)
{
        double saved = env[PTR_EXPCUTOFF];
        env[PTR_EXPCUTOFF] = expcutoff;
        int sel0[1] = {0};
        q_cond_generic(q_cond, cart ? int2e_cart : int2e_sph, 1, sel0, 1,
                       atm, natm, bas, nbas, env, cart, 0);
        env[PTR_EXPCUTOFF] = saved;
}

/* gradient conditioner: plane 0 from int2e_ip1ip2 diagonal comps (xx, yy, zz),
 * plane 1 from int2e (hessian_screen.c:70-123, pyscf/grad/rhf.py:160-171) */
void oracle_grad_q_cond(double *q_cond, int *atm, int natm, int *bas, int nbas, double *env,
                        int cart, double expcutoff)
{
        double saved = env[PTR_EXPCUTOFF];
        env[PTR_EXPCUTOFF] = expcutoff;
        int seld[3] = {0, 4, 8};
        q_cond_generic(q_cond, cart ? int2e_ip1ip2_cart : int2e_ip1ip2_sph, 9, seld, 3,
                       atm, natm, bas, nbas, env, cart, 1);
        int sel0[1] = {0};
        q_cond_generic(q_cond + (size_t)nbas * nbas, cart ? int2e_cart : int2e_sph, 1, sel0, 1,
                       atm, natm, bas, nbas, env, cart, 0);
        env[PTR_EXPCUTOFF] = saved;
}

/* CVHFnr_dm_cond restated (optimizer.c:494-518) */
void oracle_dm_cond(double *dm_cond, const double *dms, int n_dm, const int *bas, int nbas, int cart)
{
        int *ao_loc = malloc(sizeof(int) * (nbas + 1));
        make_ao_loc(ao_loc, bas, nbas, cart);
        size_t nao = ao_loc[nbas];
        for (int ish = 0; ish < nbas; ish++) {
        for (int jsh = 0; jsh <= ish; jsh++) {
                double dmax = 0;
                for (int s = 0; s < n_dm; s++) {
                        const double *d = dms + nao * nao * s;
                        for (int i = ao_loc[ish]; i < ao_loc[ish + 1]; i++)
                        for (int j = ao_loc[jsh]; j < ao_loc[jsh + 1]; j++) {
                                double t = fabs(d[i * nao + j]) + fabs(d[j * nao + i]);
                                dmax = MAX(dmax, t);
                        }
                }
                dm_cond[(size_t)ish * nbas + jsh] = .5 * dmax;
                dm_cond[(size_t)jsh * nbas + ish] = .5 * dmax;
        } }
        free(ao_loc);
}

/* CVHFdm_cond1-like plain max |D| per shell block, used by the gradient screen
 * (CVHFnr_dm_cond1, optimizer.c:472-492) */
void oracle_dm_cond1(double *dm_cond, const double *dms, int n_dm, const int *bas, int nbas, int cart)
{
        int *ao_loc = malloc(sizeof(int) * (nbas + 1));
        make_ao_loc(ao_loc, bas, nbas, cart);
        size_t nao = ao_loc[nbas];
        for (int ish = 0; ish < nbas; ish++) {
        for (int jsh = 0; jsh < nbas; jsh++) {
                double dmax = 0;
                for (int s = 0; s < n_dm; s++) {
                        const double *d = dms + nao * nao * s;
                        for (int i = ao_loc[ish]; i < ao_loc[ish + 1]; i++)
                        for (int j = ao_loc[jsh]; j < ao_loc[jsh + 1]; j++)
                                dmax = MAX(dmax, fabs(d[i * nao + j]));
                }
                dm_cond[(size_t)ish * nbas + jsh] = dmax;
        } }
        free(ao_loc);
}

/* CVHFnrs8_prescreen restated (optimizer.c:90-117) */
static int nrs8_prescreen(int i, int j, int k, int l, const double *q, const double *dmc,
                          size_t n, double tol)
{
        double qijkl = q[i * n + j] * q[k * n + l];
        return qijkl > tol
            && ((4 * dmc[j * n + i] * qijkl > tol)
             || (4 * dmc[l * n + k] * qijkl > tol)
             || (dmc[j * n + k] * qijkl > tol)
             || (dmc[j * n + l] * qijkl > tol)
             || (dmc[i * n + k] * qijkl > tol)
             || (dmc[i * n + l] * qijkl > tol));
}

/*
 * J/K over the s8-unique quartets.
 *   dms     (n_dm, nao, nao) C order
 *   vj, vk  (n_dm, nao, nao) outputs, overwritten (either may be NULL)
 *   q_cond, dm_cond  (nbas, nbas) or NULL for no screening (vhfopt=None)
 * Returns the number of quartets evaluated (after screening) in *nquartets.
 */
int oracle_get_jk(const double *dms, int n_dm, double *vj, double *vk, int hermi,
                  int *atm, int natm, int *bas, int nbas, double *env, int cart,
                  const double *q_cond, const double *dm_cond, double tol,
                  long long *nquartets)
{
        int *ao_loc = malloc(sizeof(int) * (nbas + 1));
        make_ao_loc(ao_loc, bas, nbas, cart);
        size_t nao = ao_loc[nbas];
        size_t nn = nao * nao;
        int dmax = 0;
        for (int i = 0; i < nbas; i++) dmax = MAX(dmax, ao_loc[i + 1] - ao_loc[i]);
        intor_t intor = cart ? int2e_cart : int2e_sph;
        size_t npair = (size_t)nbas * (nbas + 1) / 2;
        int nthreads = omp_get_max_threads();
        double *priv = calloc((size_t)nthreads * n_dm * 2 * nn, sizeof(double));
        if (!priv) return -1;
        long long count = 0;
#pragma omp parallel reduction(+:count)
{
        int tid = omp_get_thread_num();
        double *pj = priv + (size_t)tid * n_dm * 2 * nn;
        double *pk = pj + (size_t)n_dm * nn;
        double *buf = malloc(sizeof(double) * (size_t)dmax * dmax * dmax * dmax);
#pragma omp for schedule(dynamic, 1)
        for (size_t ij = 0; ij < npair; ij++) {
                int ish = (int)(sqrt(2 * (double)ij + .25) - .5 + 1e-7);
                int jsh = (int)(ij - (size_t)ish * (ish + 1) / 2);
                for (size_t kl = 0; kl <= ij; kl++) {
                        int ksh = (int)(sqrt(2 * (double)kl + .25) - .5 + 1e-7);
                        int lsh = (int)(kl - (size_t)ksh * (ksh + 1) / 2);
                        if (q_cond && !nrs8_prescreen(ish, jsh, ksh, lsh, q_cond, dm_cond, nbas, tol)) continue;
                        int shls[4] = {ish, jsh, ksh, lsh};
                        if (!(*intor)(buf, NULL, shls, atm, natm, bas, nbas, env, NULL, NULL)) continue;
                        count++;
                        double fac = 1;
                        if (ish == jsh) fac *= .5;
                        if (ksh == lsh) fac *= .5;
                        if (ij == kl) fac *= .5;
                        int i0 = ao_loc[ish], j0 = ao_loc[jsh], k0 = ao_loc[ksh], l0 = ao_loc[lsh];
                        int di = ao_loc[ish + 1] - i0, dj = ao_loc[jsh + 1] - j0;
                        int dk = ao_loc[ksh + 1] - k0, dl = ao_loc[lsh + 1] - l0;
                        for (int s = 0; s < n_dm; s++) {
                                const double *D = dms + nn * s;
                                double *J = pj + nn * s, *K = pk + nn * s;
                                for (int l = 0; l < dl; l++)
                                for (int k = 0; k < dk; k++)
                                for (int j = 0; j < dj; j++)
                                for (int i = 0; i < di; i++) {
                                        double v = fac * buf[i + di * (j + dj * (k + (size_t)dk * l))];
                                        size_t a = i0 + i, b = j0 + j, c = k0 + k, d = l0 + l;
                                        /* images (pq|rs) of (ab|cd):
                                         * J[r,s] += v D[q,p];  K[r,q] += v D[s,p]  ('li->kj') */
                                        double dab = D[b * nao + a] + D[a * nao + b];
                                        double dcd = D[d * nao + c] + D[c * nao + d];
                                        J[c * nao + d] += v * dab;
                                        J[d * nao + c] += v * dab;
                                        J[a * nao + b] += v * dcd;
                                        J[b * nao + a] += v * dcd;
                                        /* (ab|cd): K[c,b] += v D[d,a] */
                                        K[c * nao + b] += v * D[d * nao + a];
                                        /* (ba|cd): K[c,a] += v D[d,b] */
                                        K[c * nao + a] += v * D[d * nao + b];
                                        /* (ab|dc): K[d,b] += v D[c,a] */
                                        K[d * nao + b] += v * D[c * nao + a];
                                        /* (ba|dc): K[d,a] += v D[c,b] */
                                        K[d * nao + a] += v * D[c * nao + b];
                                        /* (cd|ab): K[a,d] += v D[b,c] */
                                        K[a * nao + d] += v * D[b * nao + c];
                                        /* (dc|ab): K[a,c] += v D[b,d] */
                                        K[a * nao + c] += v * D[b * nao + d];
                                        /* (cd|ba): K[b,d] += v D[a,c] */
                                        K[b * nao + d] += v * D[a * nao + c];
                                        /* (dc|ba): K[b,c] += v D[a,d] */
                                        K[b * nao + c] += v * D[a * nao + d];
                                }
                        }
                }
        }
        free(buf);
}
        for (int s = 0; s < n_dm; s++) {
                if (vj) {
                        double *o = vj + nn * s;
                        memset(o, 0, sizeof(double) * nn);
                        for (int t = 0; t < nthreads; t++) {
                                const double *p = priv + ((size_t)t * n_dm * 2 + s) * nn;
                                for (size_t x = 0; x < nn; x++) o[x] += p[x];
                        }
                }
                if (vk) {
                        double *o = vk + nn * s;
                        memset(o, 0, sizeof(double) * nn);
                        for (int t = 0; t < nthreads; t++) {
                                const double *p = priv + ((size_t)t * n_dm * 2 + n_dm + s) * nn;
                                for (size_t x = 0; x < nn; x++) o[x] += p[x];
                        }
                }
        }
        free(priv);
        free(ao_loc);
        if (nquartets) *nquartets = count;
        (void)hermi;
        return 0;
}

/*
 * Gradient J/K (pyscf/grad/rhf.py:149-178): for one density D,
 *   vj[x,i,j] = -sum_kl (d_x i j|kl) D[l,k],   vk[x,i,l] = -sum_jk (d_x i j|kl) D[j,k],
 * over quartets with k >= l (s2kl), screened by CVHFgrad_jk_prescreen when
 * q_cond (2 planes) and dm_cond (plain max, CVHFnr_dm_cond1) are given.
 */
int oracle_grad_jk(const double *dm, double *vj, double *vk,
                   int *atm, int natm, int *bas, int nbas, double *env, int cart,
                   const double *q_cond, const double *dm_cond, double tol)
{
        int *ao_loc = malloc(sizeof(int) * (nbas + 1));
        make_ao_loc(ao_loc, bas, nbas, cart);
        size_t nao = ao_loc[nbas];
        size_t nn = nao * nao;
        int dmax = 0;
        for (int i = 0; i < nbas; i++) dmax = MAX(dmax, ao_loc[i + 1] - ao_loc[i]);
        intor_t intor = cart ? int2e_ip1_cart : int2e_ip1_sph;
        int nthreads = omp_get_max_threads();
        double *priv = calloc((size_t)nthreads * 6 * nn, sizeof(double));
        if (!priv) return -1;
        const double *qkl = q_cond ? q_cond + (size_t)nbas * nbas : NULL;
#pragma omp parallel
{
        int tid = omp_get_thread_num();
        double *pj = priv + (size_t)tid * 6 * nn;
        double *pk = pj + 3 * nn;
        double *buf = malloc(sizeof(double) * (size_t)dmax * dmax * dmax * dmax * 3);
#pragma omp for schedule(dynamic, 1) collapse(2)
        for (int ish = 0; ish < nbas; ish++) {
        for (int jsh = 0; jsh < nbas; jsh++) {
                for (int ksh = 0; ksh < nbas; ksh++) {
                for (int lsh = 0; lsh <= ksh; lsh++) {
                        if (q_cond) {
                                double qijkl = q_cond[(size_t)ish * nbas + jsh] * qkl[(size_t)ksh * nbas + lsh];
                                double dmin = tol / qijkl;
                                if (!(qijkl > tol && ((2 * dm_cond[(size_t)lsh * nbas + ksh] > dmin)
                                                   || (dm_cond[(size_t)jsh * nbas + ksh] > dmin)
                                                   || (dm_cond[(size_t)jsh * nbas + lsh] > dmin)))) continue;
                        }
                        int shls[4] = {ish, jsh, ksh, lsh};
                        if (!(*intor)(buf, NULL, shls, atm, natm, bas, nbas, env, NULL, NULL)) continue;
                        int i0 = ao_loc[ish], j0 = ao_loc[jsh], k0 = ao_loc[ksh], l0 = ao_loc[lsh];
                        int di = ao_loc[ish + 1] - i0, dj = ao_loc[jsh + 1] - j0;
                        int dk = ao_loc[ksh + 1] - k0, dl = ao_loc[lsh + 1] - l0;
                        size_t n4 = (size_t)di * dj * dk * dl;
                        for (int x = 0; x < 3; x++) {
                                double *J = pj + x * nn, *K = pk + x * nn;
                                const double *bx = buf + x * n4;
                                for (int l = 0; l < dl; l++)
                                for (int k = 0; k < dk; k++)
                                for (int j = 0; j < dj; j++)
                                for (int i = 0; i < di; i++) {
                                        double v = bx[i + di * (j + dj * (k + (size_t)dk * l))];
                                        size_t a = i0 + i, b = j0 + j, c = k0 + k, d = l0 + l;
                                        if (ksh == lsh) {
                                                /* k, l range over the same shell: one image */
                                                J[a * nao + b] += v * dm[d * nao + c];
                                                K[a * nao + d] += v * dm[b * nao + c];
                                        } else {
                                                J[a * nao + b] += v * (dm[d * nao + c] + dm[c * nao + d]);
                                                K[a * nao + d] += v * dm[b * nao + c];
                                                K[a * nao + c] += v * dm[b * nao + d];
                                        }
                                }
                        }
                } }
        } }
        free(buf);
}
        memset(vj, 0, sizeof(double) * 3 * nn);
        memset(vk, 0, sizeof(double) * 3 * nn);
        for (int t = 0; t < nthreads; t++) {
                const double *p = priv + (size_t)t * 6 * nn;
                for (size_t x = 0; x < 3 * nn; x++) { vj[x] -= p[x]; vk[x] -= p[3 * nn + x]; }
        }
        free(priv);
        free(ao_loc);
        return 0;
}
