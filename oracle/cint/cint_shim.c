/*
 * cint_shim.c — CPU Gaussian-integral library with the libcint ABI.
 *
 * ORACLE / TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py use it, always as the checker.
 *
 * PySCF 2.12.1 evaluates its integrals in libcint v6.1.3, an un-vendored
 * ExternalProject dependency (pyscf/lib/CMakeLists.txt:175-199).  This file
 * restates the integrals the direct-SCF J/K path and its gradient need, from
 * published mathematics, behind libcint's calling convention:
 *
 *   int intor(double *out, int *dims, int *shls, int *atm, int natm,
 *             int *bas, int nbas, double *env, CINTOpt *opt, double *cache)
 *
 *   - out == NULL: return a scratch size (the GTOmax_cache_size protocol,
 *     pyscf/lib/gto/fill_int2e.c:42-62);
 *   - output in Fortran order [i,j,(k,l),comp]; dims (if given) are the
 *     leading dimensions of a larger array (pyscf/lib/gto/fill_int2c.c GTOint2c);
 *   - returns 0 when every primitive product is screened out (callers skip the
 *     contraction then, pyscf/lib/vhf/nr_direct.c:65-92).
 *
 * Methods:
 *   - Boys function: power series + downward recursion for T <= 40,
 *     erf + upward recursion above (both exact recurrences of F_m).
 *   - two-electron: Obara & Saika, J. Chem. Phys. 84, 3963 (1986) vertical
 *     recurrence on [e0|f0]^(m), contracted, then the Head-Gordon & Pople,
 *     J. Chem. Phys. 89, 5777 (1988) horizontal recurrence.  The GPU engine
 *     uses Rys quadrature instead, so the two are independent formulations.
 *   - one-electron: Obara-Saika 1D overlap recurrences (overlap, kinetic) and
 *     the nuclear-attraction recurrence with the Boys function.
 *   - derivative integrals (int2e_ip1, int2e_ip1ip2, int1e_ip*): d/dx of a
 *     Cartesian Gaussian  x^a e^{-alpha x^2}  is  a x^{a-1} - 2 alpha x^{a+1}.
 *   - real solid harmonics: Helgaker, Jorgensen & Olsen, "Molecular
 *     Electronic-Structure Theory" eqs. 6.4.47-6.4.50, rescaled by
 *     sqrt((2l+1)/4pi) so that they are r^l Y_lm with unit-normalised Y_lm;
 *     p functions ordered (x, y, z), l >= 2 ordered m = -l..l
 *     (pyscf/symm/sph.py:83-103 documents this ordering).
 *   - primitive radial normalisation is already folded into env by
 *     pyscf/gto/mole.py:988-1031; s and p carry the factors
 *     0.282094791773878143 and 0.488602511902919921 (pyscf/gto/mole.py:157-187).
 */
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <stdlib.h>
#include "cint.h"

#define LDEG 20            /* largest Cartesian degree the tables cover   */
#define NCUM_MAX 1771      /* ncum(LDEG+1) = 21*22*23/6                   */
#define MMAX 48            /* largest Boys order                          */

static int CX[NCUM_MAX], CY[NCUM_MAX], CZ[NCUM_MAX];

static inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }
static inline int ncum(int l) { return l * (l + 1) * (l + 2) / 6; }
static inline int cidx(int lx, int ly, int lz)
{
        int r = ly + lz;
        return ncum(lx + ly + lz) + r * (r + 1) / 2 + lz;
}

/* c2s[l] : (2l+1) x ncart(l) row-major coefficients of r^l Y_lm */
#define C2S_LMAX 15
static double *C2S[C2S_LMAX + 1];

static double fact(int n) { double r = 1; for (int i = 2; i <= n; i++) r *= i; return r; }
static double binom(int n, int k)
{
        if (k < 0 || k > n) return 0;
        return fact(n) / (fact(k) * fact(n - k));
}

static void build_c2s(int l)
{
        int nc = ncart(l), ns = 2 * l + 1;
        double *c = calloc((size_t)nc * ns, sizeof(double));
        double scale = sqrt((2 * l + 1) / (4 * M_PI));
        for (int m = -l; m <= l; m++) {
                int am = abs(m);
                /* v runs over v_m, v_m+1, ..., with v_m = 0 (m>=0) or 1/2 (m<0);
                 * use w = 2v (an integer of the right parity). */
                int wm = (m < 0) ? 1 : 0;
                double nlm = 1.0 / (pow(2, am) * fact(l)) *
                        sqrt(2 * fact(l + am) * fact(l - am) / (m == 0 ? 2.0 : 1.0));
                int row;
                if (l == 1) {
                        row = (m == 1) ? 0 : (m == -1) ? 1 : 2;
                } else {
                        row = m + l;
                }
                for (int t = 0; t <= (l - am) / 2; t++) {
                for (int u = 0; u <= t; u++) {
                        int wmax = 2 * ((am - wm) / 2) + wm;   /* 2*(floor(|m|/2 - v_m) + v_m) */
                        for (int w = wm; w <= wmax; w += 2) {
                                int sgn = ((t + (w - wm) / 2) % 2) ? -1 : 1;
                                double cf = sgn * pow(0.25, t) * binom(l, t) * binom(l - t, am + t)
                                          * binom(t, u) * binom(am, w);
                                int px = 2 * t + am - 2 * u - w;
                                int py = 2 * u + w;
                                int pz = l - 2 * t - am;
                                if (px < 0 || py < 0 || pz < 0) continue;
                                c[row * nc + (cidx(px, py, pz) - ncum(l))] += scale * nlm * cf;
                        }
                } }
        }
        C2S[l] = c;
}

__attribute__((constructor)) static void shim_init(void)
{
        for (int L = 0; L <= LDEG; L++) {
                for (int lx = L; lx >= 0; lx--) {
                for (int ly = L - lx; ly >= 0; ly--) {
                        int lz = L - lx - ly;
                        int n = cidx(lx, ly, lz);
                        CX[n] = lx; CY[n] = ly; CZ[n] = lz;
                } }
        }
        for (int l = 0; l <= C2S_LMAX; l++) build_c2s(l);
}

/* ------------------------------------------------------------------ */
/* counting helpers                                                    */

int CINTlen_cart(int l) { return ncart(l); }
int CINTlen_spinor(int bas_id, const int *bas)
{
        int l = bas(ANG_OF, bas_id), kappa = bas(KAPPA_OF, bas_id);
        if (kappa == 0) return 4 * l + 2;
        if (kappa < 0) return 2 * l + 2;
        return 2 * l;
}
int CINTcgtos_cart(int bas_id, const int *bas) { return ncart(bas(ANG_OF, bas_id)) * bas(NCTR_OF, bas_id); }
int CINTcgto_cart(int bas_id, const int *bas) { return CINTcgtos_cart(bas_id, bas); }
int CINTcgtos_spheric(int bas_id, const int *bas) { return (2 * bas(ANG_OF, bas_id) + 1) * bas(NCTR_OF, bas_id); }
int CINTcgto_spheric(int bas_id, const int *bas) { return CINTcgtos_spheric(bas_id, bas); }
int CINTcgtos_spinor(int bas_id, const int *bas) { return CINTlen_spinor(bas_id, bas) * bas(NCTR_OF, bas_id); }
int CINTcgto_spinor(int bas_id, const int *bas) { return CINTcgtos_spinor(bas_id, bas); }
int CINTtot_pgto_spheric(const int *bas, int nbas)
{
        int s = 0;
        for (int i = 0; i < nbas; i++) s += (2 * bas(ANG_OF, i) + 1) * bas(NPRIM_OF, i);
        return s;
}
int CINTtot_pgto_spinor(const int *bas, int nbas)
{
        int s = 0;
        for (int i = 0; i < nbas; i++) s += CINTlen_spinor(i, bas) * bas(NPRIM_OF, i);
        return s;
}
int CINTtot_cgto_cart(const int *bas, int nbas)
{
        int s = 0;
        for (int i = 0; i < nbas; i++) s += CINTcgto_cart(i, bas);
        return s;
}
int CINTtot_cgto_spheric(const int *bas, int nbas)
{
        int s = 0;
        for (int i = 0; i < nbas; i++) s += CINTcgto_spheric(i, bas);
        return s;
}
int CINTtot_cgto_spinor(const int *bas, int nbas)
{
        int s = 0;
        for (int i = 0; i < nbas; i++) s += CINTcgto_spinor(i, bas);
        return s;
}
void CINTshells_cart_offset(int ao_loc[], const int *bas, int nbas)
{
        ao_loc[0] = 0;
        for (int i = 0; i < nbas; i++) ao_loc[i + 1] = ao_loc[i] + CINTcgto_cart(i, bas);
}
void CINTshells_spheric_offset(int ao_loc[], const int *bas, int nbas)
{
        ao_loc[0] = 0;
        for (int i = 0; i < nbas; i++) ao_loc[i + 1] = ao_loc[i] + CINTcgto_spheric(i, bas);
}
void CINTshells_spinor_offset(int ao_loc[], const int *bas, int nbas)
{
        ao_loc[0] = 0;
        for (int i = 0; i < nbas; i++) ao_loc[i + 1] = ao_loc[i] + CINTcgto_spinor(i, bas);
}

/* radial normalisation 1/sqrt(int r^(2n+2) e^{-2a r^2} dr), as gto_norm */
double CINTgto_norm(int n, double a)
{
        double nn = n + 1.5;   /* (2n+2+1)/2 */
        double gi = tgamma(nn) / (2 * pow(2 * a, nn));
        return 1 / sqrt(gi);
}

double CINTcommon_fac_sp(int l)
{
        if (l == 0) return 0.282094791773878143;
        if (l == 1) return 0.488602511902919921;
        return 1;
}

double *CINTc2s_ket_sph(double *gsph, int nket, double *gcart, int l)
{
        int nc = ncart(l);
        if (l < 2) {
                memcpy(gsph, gcart, sizeof(double) * nket * nc);
                return gsph + nket * nc;
        }
        const double *c = C2S[l];
        for (int m = 0; m < 2 * l + 1; m++) {
                for (int i = 0; i < nket; i++) {
                        double s = 0;
                        for (int k = 0; k < nc; k++) s += gcart[i + nket * k] * c[m * nc + k];
                        gsph[i + nket * m] = s;
                }
        }
        return gsph + nket * (2 * l + 1);
}

double *CINTc2s_ket_sph1(double *gsph, double *gcart, int lds, int ldc, int l)
{
        int nc = ncart(l);
        if (l < 2) {
                for (int k = 0; k < nc; k++)
                        for (int i = 0; i < lds; i++) gsph[i + lds * k] = gcart[i + ldc * k];
                return gsph;
        }
        const double *c = C2S[l];
        for (int m = 0; m < 2 * l + 1; m++) {
                for (int i = 0; i < lds; i++) {
                        double s = 0;
                        for (int k = 0; k < nc; k++) s += gcart[i + ldc * k] * c[m * nc + k];
                        gsph[i + lds * m] = s;
                }
        }
        return gsph;
}

/* gsph[m + nsph*j] = sum_c Y(m; c) gcart[c + nc*j] */
double *CINTc2s_bra_sph(double *gsph, int nket, double *gcart, int l)
{
        int nc = ncart(l);
        if (l < 2) {
                memcpy(gsph, gcart, sizeof(double) * nket * nc);
                return gsph + nket * nc;
        }
        int ns = 2 * l + 1;
        const double *c = C2S[l];
        for (int j = 0; j < nket; j++) {
                for (int m = 0; m < ns; m++) {
                        double s = 0;
                        for (int k = 0; k < nc; k++) s += c[m * nc + k] * gcart[k + nc * j];
                        gsph[m + ns * j] = s;
                }
        }
        return gsph + nket * ns;
}

void CINTdel_optimizer(CINTOpt **opt) { if (opt) *opt = NULL; }
void CINTOpt_set_log_maxc(CINTOpt *opt, int *atm, int natm, int *bas, int nbas, double *env) {}
void CINTOpt_log_max_pgto_coeff(double *log_maxc, double *coeff, int nprim, int nctr)
{
        for (int ip = 0; ip < nprim; ip++) {
                double m = 0;
                for (int i = 0; i < nctr; i++) m = MAX(m, fabs(coeff[i * nprim + ip]));
                log_maxc[ip] = log(m);
        }
}

/* ------------------------------------------------------------------ */
/* Boys function F_m(T), m = 0..mmax                                   */

void oracle_boys(int mmax, double t, double *f)
{
        if (t <= 40.0) {
                double e = exp(-t);
                double term = 1.0 / (2 * mmax + 1);
                double sum = term;
                for (int k = 1; k < 2000; k++) {
                        term *= 2 * t / (2 * mmax + 2 * k + 1);
                        sum += term;
                        if (term < sum * 1e-18) break;
                }
                f[mmax] = e * sum;
                for (int m = mmax - 1; m >= 0; m--) {
                        f[m] = (2 * t * f[m + 1] + e) / (2 * m + 1);
                }
        } else {
                double e = exp(-t);
                double st = sqrt(t);
                f[0] = 0.5 * sqrt(M_PI) / st * erf(st);
                for (int m = 0; m < mmax; m++) {
                        f[m + 1] = ((2 * m + 1) * f[m] - e) / (2 * t);
                }
        }
}

/* ------------------------------------------------------------------ */
/* scratch                                                             */

static __thread double *tls_buf = NULL;
static __thread size_t tls_cap = 0;
static double *scratch(size_t n)
{
        if (n > tls_cap) {
                free(tls_buf);
                tls_cap = n + n / 2 + 1024;
                tls_buf = malloc(sizeof(double) * tls_cap);
                if (!tls_buf) { fprintf(stderr, "oracle cint: out of memory\n"); exit(1); }
        }
        return tls_buf;
}

/* ------------------------------------------------------------------ */
/* Head-Gordon-Pople horizontal recurrence
 *   (a, b+1_i| = (a+1_i, b| + AB_i (a, b|
 * X holds (e| for e of degrees [la, la+lb] at rows (cidx(e) - ncum(la)),
 * each row NF doubles.  Y receives (a,b| for deg a = la, deg b = lb, rows
 * a*ncart(lb)+b.                                                      */
static void hrr(double *Y, const double *X, int la, int lb, const double AB[3], int NF, double *work)
{
        int e0 = ncum(la);
        if (lb == 0) {
                memcpy(Y, X, sizeof(double) * ncart(la) * NF);
                return;
        }
        /* level k: rows (e_local, b) with deg e in [la, la+lb-k], deg b = k */
        size_t ne0 = ncum(la + lb + 1) - e0;
        const double *prev = X;
        int nb_prev = 1;
        size_t cap = ne0 * ncart(lb) * (size_t)NF;
        double *bufA = work, *bufB = work + cap;
        double *cur = bufA;
        for (int k = 1; k <= lb; k++) {
                int emax = la + lb - k;
                size_t ne = ncum(emax + 1) - e0;
                int nbk = ncart(k);
                double *dst = (k == lb) ? Y : cur;
                size_t ne_out = (k == lb) ? (size_t)ncart(la) : ne;
                for (size_t el = 0; el < ne_out; el++) {
                        int e = (int)el + e0;
                        int ex = CX[e], ey = CY[e], ez = CZ[e];
                        for (int b = 0; b < nbk; b++) {
                                int bc = ncum(k) + b;
                                int bx = CX[bc], by = CY[bc], bz = CZ[bc];
                                int dir = bx > 0 ? 0 : (by > 0 ? 1 : 2);
                                int pbx = bx - (dir == 0), pby = by - (dir == 1), pbz = bz - (dir == 2);
                                int pb = cidx(pbx, pby, pbz) - ncum(k - 1);
                                int e1 = cidx(ex + (dir == 0), ey + (dir == 1), ez + (dir == 2)) - e0;
                                const double *s1 = prev + ((size_t)e1 * nb_prev + pb) * NF;
                                const double *s0 = prev + (el * nb_prev + pb) * NF;
                                double *d = dst + (el * nbk + b) * NF;
                                double ab = AB[dir];
                                for (int f = 0; f < NF; f++) d[f] = s1[f] + ab * s0[f];
                        }
                }
                prev = dst;
                nb_prev = nbk;
                cur = (cur == bufA) ? bufB : bufA;
        }
}

/* Apply the sph (or sp-scaled cart) transform to one index of a block.
 * Block layout: [outer][n_in][inner]  ->  [outer][n_out][inner]        */
static void transform_index(double *dst, const double *src, int l, int sph,
                            size_t outer, size_t inner)
{
        int nc = ncart(l);
        if (!sph || l < 2) {
                double f = CINTcommon_fac_sp(l);
                size_t n = outer * nc * inner;
                for (size_t i = 0; i < n; i++) dst[i] = src[i] * f;
                return;
        }
        int ns = 2 * l + 1;
        const double *c = C2S[l];
        for (size_t o = 0; o < outer; o++) {
                for (int m = 0; m < ns; m++) {
                        double *d = dst + (o * ns + m) * inner;
                        for (size_t i = 0; i < inner; i++) d[i] = 0;
                        for (int k = 0; k < nc; k++) {
                                double cf = c[m * nc + k];
                                if (cf == 0) continue;
                                const double *s = src + (o * nc + k) * inner;
                                for (size_t i = 0; i < inner; i++) d[i] += cf * s[i];
                        }
                }
        }
}

static double expcutoff_of(const double *env)
{
        double c = env[PTR_EXPCUTOFF];
        if (c == 0) return 60.0;
        return MAX(20.0, c);
}

/* ------------------------------------------------------------------ */
/* two-electron integrals                                              */

enum { D2_NONE = 0, D2_IP1 = 1, D2_IP1IP2 = 2 };

typedef struct {
        int l, np, nc;
        const double *r, *exp, *coef;
} Shell;

static void load_shell(Shell *s, int sh, const int *atm, const int *bas, const double *env)
{
        s->l = bas(ANG_OF, sh);
        s->np = bas(NPRIM_OF, sh);
        s->nc = bas(NCTR_OF, sh);
        s->exp = env + bas(PTR_EXP, sh);
        s->coef = env + bas(PTR_COEFF, sh);
        s->r = env + atm(PTR_COORD, bas(ATOM_OF, sh));
}

/* Obara-Saika VRR.  V[(m*NE + e)*NF + f], e < NE = ncum(Ea+1), f < NF = ncum(Fc+1).
 * fm[m] already multiplied by the prefactor.                          */
static void vrr2e(double *V, int Ea, int Fc, const double *fm,
                  const double PA[3], const double WP[3], const double QC[3], const double WQ[3],
                  double p, double q)
{
        int L = Ea + Fc;
        int NE = ncum(Ea + 1), NF = ncum(Fc + 1);
        double rho = p * q / (p + q);
        double o2p = 0.5 / p, o2q = 0.5 / q, o2pq = 0.5 / (p + q);
        double rp = rho / p, rq = rho / q;
#define VV(m, e, f) V[((size_t)(m) * NE + (e)) * NF + (f)]
        for (int m = 0; m <= L; m++) VV(m, 0, 0) = fm[m];
        for (int e = 1; e < NE; e++) {
                int ex = CX[e], ey = CY[e], ez = CZ[e];
                int de = ex + ey + ez;
                int dir = ex > 0 ? 0 : (ey > 0 ? 1 : 2);
                int n1 = (dir == 0 ? ex : dir == 1 ? ey : ez) - 1;   /* quanta left in e' */
                int e1 = cidx(ex - (dir == 0), ey - (dir == 1), ez - (dir == 2));
                int e2 = n1 > 0 ? cidx(ex - 2 * (dir == 0), ey - 2 * (dir == 1), ez - 2 * (dir == 2)) : -1;
                for (int m = 0; m <= L - de; m++) {
                        double v = PA[dir] * VV(m, e1, 0) + WP[dir] * VV(m + 1, e1, 0);
                        if (e2 >= 0) v += n1 * o2p * (VV(m, e2, 0) - rp * VV(m + 1, e2, 0));
                        VV(m, e, 0) = v;
                }
        }
        for (int f = 1; f < NF; f++) {
                int fx = CX[f], fy = CY[f], fz = CZ[f];
                int df = fx + fy + fz;
                int dir = fx > 0 ? 0 : (fy > 0 ? 1 : 2);
                int n1 = (dir == 0 ? fx : dir == 1 ? fy : fz) - 1;
                int f1 = cidx(fx - (dir == 0), fy - (dir == 1), fz - (dir == 2));
                int f2 = n1 > 0 ? cidx(fx - 2 * (dir == 0), fy - 2 * (dir == 1), fz - 2 * (dir == 2)) : -1;
                for (int e = 0; e < NE; e++) {
                        int ex = CX[e], ey = CY[e], ez = CZ[e];
                        int de = ex + ey + ez;
                        int ne = (dir == 0 ? ex : dir == 1 ? ey : ez);
                        int em = ne > 0 ? cidx(ex - (dir == 0), ey - (dir == 1), ez - (dir == 2)) : -1;
                        for (int m = 0; m <= L - de - df; m++) {
                                double v = QC[dir] * VV(m, e, f1) + WQ[dir] * VV(m + 1, e, f1);
                                if (f2 >= 0) v += n1 * o2q * (VV(m, e, f2) - rq * VV(m + 1, e, f2));
                                if (em >= 0) v += ne * o2pq * VV(m + 1, em, f1);
                                VV(m, e, f) = v;
                        }
                }
        }
#undef VV
}

/* contracted Cartesian block (a,b|c,d) for degrees la,lb,lc,ld from the
 * contracted [e0|f0] accumulator acc (rows e in [emin..Ea], cols f in [fmin..Fc]) */
static void block_from_acc(double *out, const double *acc, int emin, int Ea, int fmin, int Fc,
                           int la, int lb, int lc, int ld, const double AB[3], const double CD[3],
                           double *work)
{
        int NEr = ncum(Ea + 1) - ncum(emin);
        int NFr = ncum(Fc + 1) - ncum(fmin);
        int nab = ncart(la) * ncart(lb);
        int ncd = ncart(lc) * ncart(ld);
        /* gather rows e in [la, la+lb], cols f in [lc, lc+ld] */
        int ne = ncum(la + lb + 1) - ncum(la);
        int nf = ncum(lc + ld + 1) - ncum(lc);
        double *X = work;                      /* ne * nf */
        double *Y = X + (size_t)ne * nf;       /* nab * nf */
        double *Yt = Y + (size_t)nab * nf;     /* nf * nab */
        double *Z = Yt + (size_t)nab * nf;     /* ncd * nab */
        double *hw = Z + (size_t)ncd * nab;
        for (int e = 0; e < ne; e++) {
                int er = e + ncum(la) - ncum(emin);
                for (int f = 0; f < nf; f++) {
                        int fr = f + ncum(lc) - ncum(fmin);
                        X[e * nf + f] = acc[(size_t)er * NFr + fr];
                }
        }
        (void)NEr;
        hrr(Y, X, la, lb, AB, nf, hw);
        for (int ab = 0; ab < nab; ab++)
                for (int f = 0; f < nf; f++) Yt[f * nab + ab] = Y[ab * nf + f];
        hrr(Z, Yt, lc, ld, CD, nab, hw);
        /* out[ab*ncd + cd] */
        for (int cd = 0; cd < ncd; cd++)
                for (int ab = 0; ab < nab; ab++) out[(size_t)ab * ncd + cd] = Z[(size_t)cd * nab + ab];
}

static size_t hrr_work_size(int la, int lb, int lc, int ld)
{
        size_t ne = ncum(la + lb + 1) - ncum(la);
        size_t nf = ncum(lc + ld + 1) - ncum(lc);
        size_t nab = ncart(la) * ncart(lb), ncd = ncart(lc) * ncart(ld);
        size_t h1 = ne * ncart(lb) * nf, h2 = nf * ncart(ld) * nab;
        return ne * nf + 2 * nab * nf + ncd * nab + 2 * MAX(h1, h2) + 64;
}

static int int2e_generic(double *out, const int *dims, const int *shls,
                         const int *atm, int natm, const int *bas, int nbas,
                         const double *env, int deriv, int sph)
{
        Shell s[4];
        for (int n = 0; n < 4; n++) load_shell(&s[n], shls[n], atm, bas, env);
        int la = s[0].l, lb = s[1].l, lc = s[2].l, ld = s[3].l;
        int ncomp = deriv == D2_NONE ? 1 : deriv == D2_IP1 ? 3 : 9;
        int nfi = sph ? 2 * la + 1 : ncart(la), nfj = sph ? 2 * lb + 1 : ncart(lb);
        int nfk = sph ? 2 * lc + 1 : ncart(lc), nfl = sph ? 2 * ld + 1 : ncart(ld);
        int di = nfi * s[0].nc, dj = nfj * s[1].nc, dk = nfk * s[2].nc, dl = nfl * s[3].nc;
        if (out == NULL) {
                return 64;
        }
        int d0 = dims ? dims[0] : di, d1 = dims ? dims[1] : dj;
        int d2 = dims ? dims[2] : dk, d3 = dims ? dims[3] : dl;
        size_t cstride = (size_t)d0 * d1 * d2 * d3;

        int raise_a = deriv >= D2_IP1, raise_c = deriv == D2_IP1IP2;
        int Ea = la + raise_a + lb, Fc = lc + raise_c + ld;
        int emin = MAX(0, la - raise_a), fmin = MAX(0, lc - raise_c);
        int nw = deriv == D2_NONE ? 1 : deriv == D2_IP1 ? 2 : 4;
        int nctr = s[0].nc * s[1].nc * s[2].nc * s[3].nc;
        int NE = ncum(Ea + 1), NF = ncum(Fc + 1);
        int NEr = NE - ncum(emin), NFr = NF - ncum(fmin);
        size_t accsz = (size_t)nw * nctr * NEr * NFr;
        int L = Ea + Fc;
        size_t vsz = (size_t)(L + 1) * NE * NF;

        const double *A = s[0].r, *B = s[1].r, *C = s[2].r, *D = s[3].r;
        double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
        double CD[3] = {C[0] - D[0], C[1] - D[1], C[2] - D[2]};
        double rrab = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
        double rrcd = CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2];
        double cutoff = expcutoff_of(env);
        /* range-separated Coulomb (libcint's env[PTR_RANGE_OMEGA], set by
         * mol.with_range_coulomb): omega > 0 is erf(omega r)/r, omega < 0
         * erfc(|omega| r)/r.  The Obara-Saika recurrence is a polynomial in
         * the Rys variable t^2, so attenuating the operator only changes the
         * auxiliary integrals: F_m(T) -> theta^(m+1/2) F_m(theta T) with
         * theta = omega^2 / (omega^2 + rho) for erf, F_m - that for erfc. */
        const double omega = env[PTR_RANGE_OMEGA];

        int nab_c = ncart(la + raise_a) * ncart(lb);
        int ncd_c = ncart(lc + raise_c) * ncart(ld);
        size_t blk = (size_t)nab_c * ncd_c;
        size_t hw = hrr_work_size(la + raise_a, lb, lc + raise_c, ld);
        size_t nab0 = (size_t)ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
        size_t tsz = (size_t)nctr * ncomp * nab0;
        size_t total = accsz + vsz + 4 * blk + hw + 2 * tsz + 64;
        double *work = scratch(total);
        double *acc = work;
        double *V = acc + accsz;
        double *blkbuf = V + vsz;           /* 4 blocks */
        double *hwork = blkbuf + 4 * blk;
        double *cart = hwork + hw;          /* [comp][ctr][a][b][c][d] */
        double *tmp = cart + tsz;
        memset(acc, 0, sizeof(double) * accsz);

        double fm[MMAX + 1];
        int nonzero = 0;
        for (int ip = 0; ip < s[0].np; ip++) {
        for (int jp = 0; jp < s[1].np; jp++) {
                double ai = s[0].exp[ip], aj = s[1].exp[jp];
                double p = ai + aj;
                double muab = ai * aj / p;
                if (muab * rrab > cutoff) continue;
                double Kab = exp(-muab * rrab);
                double P[3], PA[3];
                for (int x = 0; x < 3; x++) { P[x] = (ai * A[x] + aj * B[x]) / p; PA[x] = P[x] - A[x]; }
                for (int kp = 0; kp < s[2].np; kp++) {
                for (int lp = 0; lp < s[3].np; lp++) {
                        double ak = s[2].exp[kp], al = s[3].exp[lp];
                        double q = ak + al;
                        double mucd = ak * al / q;
                        if (mucd * rrcd > cutoff) continue;
                        nonzero = 1;
                        double Kcd = exp(-mucd * rrcd);
                        double Q[3], QC[3], W[3], WP[3], WQ[3], PQ[3];
                        for (int x = 0; x < 3; x++) {
                                Q[x] = (ak * C[x] + al * D[x]) / q;
                                QC[x] = Q[x] - C[x];
                                W[x] = (p * P[x] + q * Q[x]) / (p + q);
                                WP[x] = W[x] - P[x];
                                WQ[x] = W[x] - Q[x];
                                PQ[x] = P[x] - Q[x];
                        }
                        double rho = p * q / (p + q);
                        double T = rho * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
                        double pref = 2 * pow(M_PI, 2.5) / (p * q * sqrt(p + q)) * Kab * Kcd;
                        oracle_boys(L, T, fm);
                        if (omega != 0) {
                                double gm[MMAX + 1];
                                const double theta = omega * omega / (omega * omega + rho);
                                oracle_boys(L, theta * T, gm);
                                double tp = sqrt(theta);
                                for (int m = 0; m <= L; m++) {
                                        gm[m] *= tp;
                                        tp *= theta;
                                        fm[m] = omega > 0 ? gm[m] : fm[m] - gm[m];
                                }
                        }
                        for (int m = 0; m <= L; m++) fm[m] *= pref;
                        vrr2e(V, Ea, Fc, fm, PA, WP, QC, WQ, p, q);
                        /* accumulate contracted rows */
                        for (int w = 0; w < nw; w++) {
                                double wf = 1;
                                if (w & 1) wf *= ai;
                                if (w & 2) wf *= ak;
                                int ic = 0;
                                for (int cl = 0; cl < s[3].nc; cl++) {
                                for (int ck = 0; ck < s[2].nc; ck++) {
                                for (int cj = 0; cj < s[1].nc; cj++) {
                                for (int ci = 0; ci < s[0].nc; ci++, ic++) {
                                        double cf = wf * s[0].coef[ci * s[0].np + ip] * s[1].coef[cj * s[1].np + jp]
                                                  * s[2].coef[ck * s[2].np + kp] * s[3].coef[cl * s[3].np + lp];
                                        if (cf == 0) continue;
                                        double *a = acc + ((size_t)w * nctr + ic) * NEr * NFr;
                                        for (int e = ncum(emin); e < NE; e++) {
                                                const double *v = V + (size_t)e * NF + ncum(fmin);
                                                double *ar = a + (size_t)(e - ncum(emin)) * NFr;
                                                for (int f = 0; f < NFr; f++) ar[f] += cf * v[f];
                                        }
                                } } } }
                        }
                } }
        } }

        if (!nonzero) {
                for (int c = 0; c < ncomp; c++)
                        for (int l = 0; l < dl; l++) for (int k = 0; k < dk; k++)
                        for (int j = 0; j < dj; j++) for (int i = 0; i < di; i++)
                                out[c * cstride + i + (size_t)d0 * (j + (size_t)d1 * (k + (size_t)d2 * l))] = 0;
                return 0;
        }

        int na = ncart(la), nb = ncart(lb), nc_ = ncart(lc), nd = ncart(ld);
        /* cart[comp][ctr][a][b][c][d] */
        for (int ic = 0; ic < nctr; ic++) {
                if (deriv == D2_NONE) {
                        block_from_acc(cart + (size_t)ic * nab0, acc + (size_t)ic * NEr * NFr,
                                       emin, Ea, fmin, Fc, la, lb, lc, ld, AB, CD, hwork);
                } else if (deriv == D2_IP1) {
                        const double *acc0 = acc + ((size_t)0 * nctr + ic) * NEr * NFr;
                        const double *acc1 = acc + ((size_t)1 * nctr + ic) * NEr * NFr;
                        double *hp = blkbuf, *hm = blkbuf + blk;
                        block_from_acc(hp, acc1, emin, Ea, fmin, Fc, la + 1, lb, lc, ld, AB, CD, hwork);
                        if (la > 0) block_from_acc(hm, acc0, emin, Ea, fmin, Fc, la - 1, lb, lc, ld, AB, CD, hwork);
                        int nbcd = nb * nc_ * nd;
                        for (int x = 0; x < 3; x++) {
                                double *o = cart + ((size_t)x * nctr + ic) * nab0;
                                for (int a = 0; a < na; a++) {
                                        int ac = ncum(la) + a;
                                        int ax = CX[ac], ay = CY[ac], az = CZ[ac];
                                        int up = cidx(ax + (x == 0), ay + (x == 1), az + (x == 2)) - ncum(la + 1);
                                        int nq = x == 0 ? ax : x == 1 ? ay : az;
                                        int dn = nq > 0 ? cidx(ax - (x == 0), ay - (x == 1), az - (x == 2)) - ncum(la - 1) : -1;
                                        for (int r = 0; r < nbcd; r++) {
                                                double v = -2 * hp[(size_t)up * nbcd + r];
                                                if (dn >= 0) v += nq * hm[(size_t)dn * nbcd + r];
                                                o[(size_t)a * nbcd + r] = v;
                                        }
                                }
                        }
                } else {
                        /* weights: 0 plain, 1 alpha_i, 2 alpha_k, 3 alpha_i alpha_k */
                        double *hpp = blkbuf, *hpm = blkbuf + blk, *hmp = blkbuf + 2 * blk, *hmm = blkbuf + 3 * blk;
                        const double *aw[4];
                        for (int w = 0; w < 4; w++) aw[w] = acc + ((size_t)w * nctr + ic) * NEr * NFr;
                        block_from_acc(hpp, aw[3], emin, Ea, fmin, Fc, la + 1, lb, lc + 1, ld, AB, CD, hwork);
                        if (lc > 0) block_from_acc(hpm, aw[1], emin, Ea, fmin, Fc, la + 1, lb, lc - 1, ld, AB, CD, hwork);
                        if (la > 0) block_from_acc(hmp, aw[2], emin, Ea, fmin, Fc, la - 1, lb, lc + 1, ld, AB, CD, hwork);
                        if (la > 0 && lc > 0) block_from_acc(hmm, aw[0], emin, Ea, fmin, Fc, la - 1, lb, lc - 1, ld, AB, CD, hwork);
                        int ncp = ncart(lc + 1), ncm = lc > 0 ? ncart(lc - 1) : 0;
                        for (int x = 0; x < 3; x++) {
                        for (int y = 0; y < 3; y++) {
                                double *o = cart + ((size_t)(x * 3 + y) * nctr + ic) * nab0;
                                for (int a = 0; a < na; a++) {
                                        int ac = ncum(la) + a;
                                        int ax = CX[ac], ay = CY[ac], az = CZ[ac];
                                        int aup = cidx(ax + (x == 0), ay + (x == 1), az + (x == 2)) - ncum(la + 1);
                                        int anq = x == 0 ? ax : x == 1 ? ay : az;
                                        int adn = anq > 0 ? cidx(ax - (x == 0), ay - (x == 1), az - (x == 2)) - ncum(la - 1) : -1;
                                        for (int b = 0; b < nb; b++) {
                                        for (int c = 0; c < nc_; c++) {
                                                int cc = ncum(lc) + c;
                                                int cx = CX[cc], cy = CY[cc], cz = CZ[cc];
                                                int cup = cidx(cx + (y == 0), cy + (y == 1), cz + (y == 2)) - ncum(lc + 1);
                                                int cnq = y == 0 ? cx : y == 1 ? cy : cz;
                                                int cdn = cnq > 0 ? cidx(cx - (y == 0), cy - (y == 1), cz - (y == 2)) - ncum(lc - 1) : -1;
                                                for (int d = 0; d < nd; d++) {
                                                        double v = 4 * hpp[(((size_t)aup * nb + b) * ncp + cup) * nd + d];
                                                        if (cdn >= 0) v -= 2 * cnq * hpm[(((size_t)aup * nb + b) * ncm + cdn) * nd + d];
                                                        if (adn >= 0) v -= 2 * anq * hmp[(((size_t)adn * nb + b) * ncp + cup) * nd + d];
                                                        if (adn >= 0 && cdn >= 0) v += anq * cnq * hmm[(((size_t)adn * nb + b) * ncm + cdn) * nd + d];
                                                        o[(((size_t)a * nb + b) * nc_ + c) * nd + d] = v;
                                                }
                                        } }
                                }
                        } }
                }
        }

        /* transform indices: cart[comp*ctr][a][b][c][d] -> [comp*ctr][ia][jb][kc][ld] */
        size_t NO = (size_t)ncomp * nctr;
        double *t0 = cart, *t1 = tmp;
        transform_index(t1, t0, la, sph, NO, (size_t)nb * nc_ * nd);
        transform_index(t0, t1, lb, sph, NO * nfi, (size_t)nc_ * nd);
        transform_index(t1, t0, lc, sph, NO * nfi * nfj, (size_t)nd);
        transform_index(t0, t1, ld, sph, NO * nfi * nfj * nfk, 1);
        /* t0[comp][ctr (ci fastest ... cl slowest)][i][j][k][l] -> out */
        for (int c = 0; c < ncomp; c++) {
                int ic = 0;
                for (int cl = 0; cl < s[3].nc; cl++)
                for (int ck = 0; ck < s[2].nc; ck++)
                for (int cj = 0; cj < s[1].nc; cj++)
                for (int ci = 0; ci < s[0].nc; ci++, ic++) {
                        const double *src = t0 + ((size_t)c * nctr + ic) * nfi * nfj * nfk * nfl;
                        for (int i = 0; i < nfi; i++)
                        for (int j = 0; j < nfj; j++)
                        for (int k = 0; k < nfk; k++)
                        for (int l = 0; l < nfl; l++) {
                                size_t I = ci * nfi + i, J = cj * nfj + j, K = ck * nfk + k, Lx = cl * nfl + l;
                                out[c * cstride + I + d0 * (J + d1 * (K + d2 * Lx))] =
                                        src[((i * nfj + j) * nfk + k) * nfl + l];
                        }
                }
        }
        return 1;
}

#define INT2E(NAME, DERIV, SPH) \
int NAME(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas, \
         double *env, CINTOpt *opt, double *cache) \
{ return int2e_generic(out, dims, shls, atm, natm, bas, nbas, env, DERIV, SPH); }

INT2E(int2e_sph, D2_NONE, 1)
INT2E(int2e_cart, D2_NONE, 0)
INT2E(int2e_ip1_sph, D2_IP1, 1)
INT2E(int2e_ip1_cart, D2_IP1, 0)
INT2E(int2e_ip1ip2_sph, D2_IP1IP2, 1)
INT2E(int2e_ip1ip2_cart, D2_IP1IP2, 0)

/* ------------------------------------------------------------------ */
/* one-electron integrals                                              */

enum { OP_OVLP = 0, OP_KIN, OP_NUC, OP_RINV };

/* 1D overlap table S[a][b] for a <= amax, b <= bmax (row stride bmax+1) */
static void overlap1d(double *S, int amax, int bmax, double PA, double PB, double p, double s00)
{
        int nb = bmax + 1;
        double o2p = 0.5 / p;
        S[0] = s00;
        for (int b = 1; b <= bmax; b++) {
                double v = PB * S[b - 1];
                if (b > 1) v += (b - 1) * o2p * S[b - 2];
                S[b] = v;
        }
        for (int a = 1; a <= amax; a++) {
                for (int b = 0; b <= bmax; b++) {
                        double v = PA * S[(a - 1) * nb + b];
                        if (a > 1) v += (a - 1) * o2p * S[(a - 2) * nb + b];
                        if (b > 0) v += b * o2p * S[(a - 1) * nb + b - 1];
                        S[a * nb + b] = v;
                }
        }
}

/* nuclear-attraction style [e|C|0]^(m): T[m*NE + e], then HRR to (a|b) */
static void vrr1e(double *T, int Ea, const double *fm, const double PA[3], const double PC[3], double p)
{
        int NE = ncum(Ea + 1);
        double o2p = 0.5 / p;
        for (int m = 0; m <= Ea; m++) T[m * NE] = fm[m];
        for (int e = 1; e < NE; e++) {
                int ex = CX[e], ey = CY[e], ez = CZ[e];
                int de = ex + ey + ez;
                int dir = ex > 0 ? 0 : (ey > 0 ? 1 : 2);
                int n1 = (dir == 0 ? ex : dir == 1 ? ey : ez) - 1;
                int e1 = cidx(ex - (dir == 0), ey - (dir == 1), ez - (dir == 2));
                int e2 = n1 > 0 ? cidx(ex - 2 * (dir == 0), ey - 2 * (dir == 1), ez - 2 * (dir == 2)) : -1;
                for (int m = 0; m <= Ea - de; m++) {
                        double v = PA[dir] * T[m * NE + e1] - PC[dir] * T[(m + 1) * NE + e1];
                        if (e2 >= 0) v += n1 * o2p * (T[m * NE + e2] - T[(m + 1) * NE + e2]);
                        T[m * NE + e] = v;
                }
        }
}

static int int1e_generic(double *out, const int *dims, const int *shls,
                         const int *atm, int natm, const int *bas, int nbas,
                         const double *env, int op, int deriv, int sph)
{
        Shell s[2];
        load_shell(&s[0], shls[0], atm, bas, env);
        load_shell(&s[1], shls[1], atm, bas, env);
        int la = s[0].l, lb = s[1].l;
        int ncomp = deriv ? 3 : 1;
        int nfi = sph ? 2 * la + 1 : ncart(la), nfj = sph ? 2 * lb + 1 : ncart(lb);
        int di = nfi * s[0].nc, dj = nfj * s[1].nc;
        if (out == NULL) return 64;
        int d0 = dims ? dims[0] : di, d1 = dims ? dims[1] : dj;
        size_t cstride = (size_t)d0 * d1;
        int na = ncart(la), nb = ncart(lb);
        int nctr = s[0].nc * s[1].nc;
        size_t nab = (size_t)na * nb;
        const double *A = s[0].r, *B = s[1].r;
        double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
        double rr = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];

        int amax = la + deriv, bmax = lb + 2;
        int Ea = la + deriv + lb;
        size_t hw = hrr_work_size(la + deriv, lb, 0, 0);
        size_t need = (size_t)ncomp * nctr * nab * 3 + 3 * (amax + 1) * (bmax + 1) * 2
                      + (size_t)(Ea + 1) * ncum(Ea + 1) + 4 * ncart(la + 1) * nb + hw + 64;
        double *work = scratch(need);
        double *acc = work;                                   /* [comp][ctr][a][b] */
        double *S1 = acc + (size_t)ncomp * nctr * nab;        /* 3 dims of 1D tables */
        double *T = S1 + 3 * (amax + 1) * (bmax + 1) * 2;
        double *hp = T + (size_t)(Ea + 1) * ncum(Ea + 1);     /* (a+1|b) block */
        double *hm = hp + 2 * ncart(la + 1) * nb;             /* (a-1|b) block */
        double *h0 = hm + ncart(la + 1) * nb;
        double *hwork = h0 + ncart(la + 1) * nb;
        double *prim = hwork + hw;                            /* reuse tail for primitive block */
        (void)prim;
        memset(acc, 0, sizeof(double) * ncomp * nctr * nab);
        double cutoff = expcutoff_of(env);
        int nonzero = 0;
        double *pb = malloc(sizeof(double) * ncomp * nab);

        for (int ip = 0; ip < s[0].np; ip++) {
        for (int jp = 0; jp < s[1].np; jp++) {
                double ai = s[0].exp[ip], aj = s[1].exp[jp];
                double p = ai + aj, mu = ai * aj / p;
                if (mu * rr > cutoff) continue;
                nonzero = 1;
                double P[3], PA[3], PB[3];
                for (int x = 0; x < 3; x++) {
                        P[x] = (ai * A[x] + aj * B[x]) / p;
                        PA[x] = P[x] - A[x];
                        PB[x] = P[x] - B[x];
                }
                if (op == OP_OVLP || op == OP_KIN) {
                        int nbb = bmax + 1;
                        double *Sd[3];
                        for (int x = 0; x < 3; x++) {
                                Sd[x] = S1 + x * (amax + 1) * nbb;
                                double s00 = sqrt(M_PI / p) * exp(-mu * AB[x] * AB[x]);
                                overlap1d(Sd[x], amax, bmax, PA[x], PB[x], p, s00);
                        }
                        /* 1D factor functions:  f(a,b) = S or K for one axis */
#define S_(x, a, b) (Sd[x][(a) * nbb + (b)])
#define K_(x, a, b) ((b) * ((b) - 1) * ((b) >= 2 ? S_(x, a, (b) - 2) : 0) - 2 * aj * (2 * (b) + 1) * S_(x, a, b) + 4 * aj * aj * S_(x, a, (b) + 2))
                        for (int a = 0; a < na; a++) {
                                int ac = ncum(la) + a;
                                int av[3] = {CX[ac], CY[ac], CZ[ac]};
                                for (int b = 0; b < nb; b++) {
                                        int bc = ncum(lb) + b;
                                        int bv[3] = {CX[bc], CY[bc], CZ[bc]};
                                        for (int c = 0; c < ncomp; c++) {
                                                /* for each axis compute S factor and K factor,
                                                 * with the bra derivative on axis c when deriv */
                                                double sf[3], kf[3];
                                                for (int x = 0; x < 3; x++) {
                                                        int a0 = av[x], b0 = bv[x];
                                                        if (deriv && x == c) {
                                                                sf[x] = -2 * ai * S_(x, a0 + 1, b0);
                                                                kf[x] = -2 * ai * K_(x, a0 + 1, b0);
                                                                if (a0 > 0) {
                                                                        sf[x] += a0 * S_(x, a0 - 1, b0);
                                                                        kf[x] += a0 * K_(x, a0 - 1, b0);
                                                                }
                                                        } else {
                                                                sf[x] = S_(x, a0, b0);
                                                                kf[x] = (op == OP_KIN) ? K_(x, a0, b0) : 0;
                                                        }
                                                }
                                                double v;
                                                if (op == OP_OVLP) {
                                                        v = sf[0] * sf[1] * sf[2];
                                                } else {
                                                        v = -0.5 * (kf[0] * sf[1] * sf[2] + sf[0] * kf[1] * sf[2] + sf[0] * sf[1] * kf[2]);
                                                }
                                                pb[(size_t)c * nab + a * nb + b] = v;
                                        }
                                }
                        }
#undef S_
#undef K_
                } else {
                        /* nuclear attraction / rinv: sum over centres */
                        memset(pb, 0, sizeof(double) * ncomp * nab);
                        int ncentre = (op == OP_NUC) ? natm : 1;
                        double Kab = exp(-mu * rr);
                        for (int ia = 0; ia < ncentre; ia++) {
                                double charge;
                                const double *Cc;
                                if (op == OP_NUC) {
                                        if (atm(NUC_MOD_OF, ia) == FRAC_CHARGE_NUC) {
                                                charge = env[atm(PTR_FRAC_CHARGE, ia)];
                                        } else {
                                                charge = atm(CHARGE_OF, ia);
                                        }
                                        if (atm(NUC_MOD_OF, ia) == GAUSSIAN_NUC) {
                                                fprintf(stderr, "oracle cint: Gaussian nuclear model not supported\n");
                                                exit(1);
                                        }
                                        charge = -charge;
                                        Cc = env + atm(PTR_COORD, ia);
                                } else {
                                        charge = 1;
                                        Cc = env + PTR_RINV_ORIG;
                                        if (env[PTR_RINV_ZETA] != 0) {
                                                fprintf(stderr, "oracle cint: smeared rinv not supported\n");
                                                exit(1);
                                        }
                                }
                                if (charge == 0) continue;
                                double PC[3] = {P[0] - Cc[0], P[1] - Cc[1], P[2] - Cc[2]};
                                double Tb = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
                                double fm[MMAX + 1];
                                oracle_boys(Ea, Tb, fm);
                                double pref = 2 * M_PI / p * Kab * charge;
                                for (int m = 0; m <= Ea; m++) fm[m] *= pref;
                                vrr1e(T, Ea, fm, PA, PC, p);
                                if (!deriv) {
                                        /* T rows are m=0: e in [la, la+lb] */
                                        hrr(h0, T + ncum(la), la, lb, AB, 1, hwork);
                                        for (size_t r = 0; r < nab; r++) pb[r] += h0[r];
                                } else {
                                        hrr(hp, T + ncum(la + 1), la + 1, lb, AB, 1, hwork);
                                        if (la > 0) hrr(hm, T + ncum(la - 1), la - 1, lb, AB, 1, hwork);
                                        for (int x = 0; x < 3; x++) {
                                                for (int a = 0; a < na; a++) {
                                                        int ac = ncum(la) + a;
                                                        int ax = CX[ac], ay = CY[ac], az = CZ[ac];
                                                        int up = cidx(ax + (x == 0), ay + (x == 1), az + (x == 2)) - ncum(la + 1);
                                                        int nq = x == 0 ? ax : x == 1 ? ay : az;
                                                        int dn = nq > 0 ? cidx(ax - (x == 0), ay - (x == 1), az - (x == 2)) - ncum(la - 1) : -1;
                                                        for (int b = 0; b < nb; b++) {
                                                                double v = -2 * ai * hp[up * nb + b];
                                                                if (dn >= 0) v += nq * hm[dn * nb + b];
                                                                pb[(size_t)x * nab + a * nb + b] += v;
                                                        }
                                                }
                                        }
                                }
                        }
                }
                int ic = 0;
                for (int cj = 0; cj < s[1].nc; cj++)
                for (int ci = 0; ci < s[0].nc; ci++, ic++) {
                        double cf = s[0].coef[ci * s[0].np + ip] * s[1].coef[cj * s[1].np + jp];
                        for (int c = 0; c < ncomp; c++) {
                                double *a = acc + ((size_t)c * nctr + ic) * nab;
                                const double *v = pb + (size_t)c * nab;
                                for (size_t r = 0; r < nab; r++) a[r] += cf * v[r];
                        }
                }
        } }
        free(pb);

        if (!nonzero) {
                for (int c = 0; c < ncomp; c++)
                        for (int j = 0; j < dj; j++) for (int i = 0; i < di; i++)
                                out[c * cstride + i + (size_t)d0 * j] = 0;
                return 0;
        }
        size_t NO = (size_t)ncomp * nctr;
        double *t1 = malloc(sizeof(double) * NO * MAX(nab, (size_t)nfi * nfj) * 2 + 16);
        double *t0 = acc;
        transform_index(t1, t0, la, sph, NO, nb);
        transform_index(t0, t1, lb, sph, NO * nfi, 1);
        for (int c = 0; c < ncomp; c++) {
                int ic = 0;
                for (int cj = 0; cj < s[1].nc; cj++)
                for (int ci = 0; ci < s[0].nc; ci++, ic++) {
                        const double *src = t0 + ((size_t)c * nctr + ic) * nfi * nfj;
                        for (int i = 0; i < nfi; i++)
                        for (int j = 0; j < nfj; j++) {
                                out[c * cstride + (ci * nfi + i) + (size_t)d0 * (cj * nfj + j)] = src[i * nfj + j];
                        }
                }
        }
        free(t1);
        return 1;
}

#define INT1E(NAME, OP, DERIV, SPH) \
int NAME(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas, \
         double *env, CINTOpt *opt, double *cache) \
{ return int1e_generic(out, dims, shls, atm, natm, bas, nbas, env, OP, DERIV, SPH); }

INT1E(int1e_ovlp_sph, OP_OVLP, 0, 1)
INT1E(int1e_ovlp_cart, OP_OVLP, 0, 0)
INT1E(int1e_kin_sph, OP_KIN, 0, 1)
INT1E(int1e_kin_cart, OP_KIN, 0, 0)
INT1E(int1e_nuc_sph, OP_NUC, 0, 1)
INT1E(int1e_nuc_cart, OP_NUC, 0, 0)
INT1E(int1e_rinv_sph, OP_RINV, 0, 1)
INT1E(int1e_rinv_cart, OP_RINV, 0, 0)
INT1E(int1e_ipovlp_sph, OP_OVLP, 1, 1)
INT1E(int1e_ipovlp_cart, OP_OVLP, 1, 0)
INT1E(int1e_ipkin_sph, OP_KIN, 1, 1)
INT1E(int1e_ipkin_cart, OP_KIN, 1, 0)
INT1E(int1e_ipnuc_sph, OP_NUC, 1, 1)
INT1E(int1e_ipnuc_cart, OP_NUC, 1, 0)
INT1E(int1e_iprinv_sph, OP_RINV, 1, 1)
INT1E(int1e_iprinv_cart, OP_RINV, 1, 0)

/* CINTOpt is never built: every optimizer hands back NULL */
#define OPTIMIZER(NAME) \
void NAME(CINTOpt **opt, int *atm, int natm, int *bas, int nbas, double *env) { *opt = NULL; }
OPTIMIZER(int2e_optimizer)
OPTIMIZER(int2e_sph_optimizer)
OPTIMIZER(int2e_cart_optimizer)
OPTIMIZER(int2e_ip1_optimizer)
OPTIMIZER(int2e_ip1ip2_optimizer)
OPTIMIZER(int1e_ovlp_optimizer)
OPTIMIZER(int1e_kin_optimizer)
OPTIMIZER(int1e_nuc_optimizer)
OPTIMIZER(int1e_rinv_optimizer)
OPTIMIZER(int1e_ipovlp_optimizer)
OPTIMIZER(int1e_ipkin_optimizer)
OPTIMIZER(int1e_ipnuc_optimizer)
OPTIMIZER(int1e_iprinv_optimizer)
