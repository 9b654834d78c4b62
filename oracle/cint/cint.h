/*
 * cint.h — the libcint ABI as PySCF's C drivers see it, declared by this
 * project for its CPU oracle.
 *
 * ORACLE / TEST INFRASTRUCTURE.  Nothing in the product package links this.
 *
 * PySCF 2.12.1 fetches its integral engine, libcint v6.1.3, as a CMake
 * ExternalProject (pyscf/lib/CMakeLists.txt:175-199).  That dependency is not
 * vendored, so this header declares only what the reference drivers
 * (pyscf/lib/vhf/nr_direct.c, optimizer.c, hessian_screen.c,
 * pyscf/lib/gto/fill_int2e.c, fill_int2c.c and pyscf/lib/np_helper) name:
 *   - the slot layout of _atm/_bas/_env, as mirrored in Python by
 *     pyscf/gto/mole.py:58-88;
 *   - CART_MAX = 136 (the size of one (ff) Cartesian pair block squared is
 *     assumed by pyscf/lib/vhf/nr_direct.c:254 "136*136");
 *   - an opaque CINTOpt;
 *   - the integral entry-point signature used by every caller
 *     (pyscf/lib/vhf/nr_direct.c:72,75; pyscf/lib/gto/fill_int2c.c).
 * The functions themselves are implemented from published mathematics in
 * cint_shim.c of this directory.
 */
#ifndef ORACLE_CINT_H
#define ORACLE_CINT_H

#include <stdint.h>
#include <stdlib.h>

#define CINT_VERSION_MAJOR 6
#define CINT_VERSION_MINOR 1
#define CINT_VERSION_PATCH 3

#define CHARGE_OF       0
#define PTR_COORD       1
#define NUC_MOD_OF      2
#define PTR_ZETA        3
#define PTR_FRAC_CHARGE 4
#define PTR_RADIUS      5
#define ATM_SLOTS       6
#define RESERVE_ATMSLOT 7

#define ATOM_OF         0
#define ANG_OF          1
#define NPRIM_OF        2
#define NCTR_OF         3
#define RADI_POWER      3
#define KAPPA_OF        4
#define SO_TYPE_OF      4
#define PTR_EXP         5
#define PTR_COEFF       6
#define RESERVE_BASLOT  7
#define BAS_SLOTS       8

#define PTR_EXPCUTOFF   0
#define PTR_COMMON_ORIG 1
#define PTR_RINV_ORIG   4
#define PTR_RINV_ZETA   7
#define PTR_RANGE_OMEGA 8
#define PTR_F12_ZETA    9
#define PTR_GTG_ZETA    10
#define NGRIDS          11
#define PTR_GRIDS       12
#define AS_RINV_ORIG_ATOM 17
#define AS_ECPBAS_OFFSET 18
#define AS_NECPBAS      19
#define PTR_ENV_START   20

#define POINT_NUC       1
#define GAUSSIAN_NUC    2
#define FRAC_CHARGE_NUC 3

#define bas(SLOT, I)    bas[BAS_SLOTS * (I) + (SLOT)]
#define atm(SLOT, I)    atm[ATM_SLOTS * (I) + (SLOT)]

/* largest angular momentum the Cartesian tables cover; CART_MAX is the number
 * of Cartesian components for l = 15 */
#define ANG_MAX         15
#define CART_MAX        136
#define LMAX1           16

#ifndef M_PI
#define M_PI            3.14159265358979323846
#endif

#ifndef MIN
#define MIN(X,Y) ((X)<(Y)?(X):(Y))
#endif
#ifndef MAX
#define MAX(X,Y) ((X)>(Y)?(X):(Y))
#endif

typedef int FINT;

/* Opaque to every caller; this oracle never allocates one (the *_optimizer
 * entry points return NULL). */
typedef struct CINTOpt_s CINTOpt;

#ifdef __cplusplus
extern "C" {
#endif

/* number of spherical / Cartesian functions of shell bas_id (nctr included) */
int CINTlen_cart(int l);
int CINTlen_spinor(int bas_id, const int *bas);
int CINTcgtos_cart(int bas_id, const int *bas);
int CINTcgtos_spheric(int bas_id, const int *bas);
int CINTcgtos_spinor(int bas_id, const int *bas);
int CINTcgto_cart(int bas_id, const int *bas);
int CINTcgto_spheric(int bas_id, const int *bas);
int CINTcgto_spinor(int bas_id, const int *bas);
int CINTtot_pgto_spheric(const int *bas, int nbas);
int CINTtot_pgto_spinor(const int *bas, int nbas);
int CINTtot_cgto_cart(const int *bas, int nbas);
int CINTtot_cgto_spheric(const int *bas, int nbas);
int CINTtot_cgto_spinor(const int *bas, int nbas);
void CINTshells_cart_offset(int ao_loc[], const int *bas, int nbas);
void CINTshells_spheric_offset(int ao_loc[], const int *bas, int nbas);
void CINTshells_spinor_offset(int ao_loc[], const int *bas, int nbas);

double CINTgto_norm(int n, double a);
double CINTcommon_fac_sp(int l);

/* gsph[i + nket*m] = sum_c gcart[i + nket*c] * Y(l,m; c) */
double *CINTc2s_ket_sph(double *gsph, int nket, double *gcart, int l);
double *CINTc2s_ket_sph1(double *gsph, double *gcart, int lds, int ldc, int l);
double *CINTc2s_bra_sph(double *gsph, int nket, double *gcart, int l);

void CINTdel_optimizer(CINTOpt **opt);
void CINTOpt_set_log_maxc(CINTOpt *opt, int *atm, int natm, int *bas, int nbas, double *env);
void CINTOpt_log_max_pgto_coeff(double *log_maxc, double *coeff, int nprim, int nctr);

#ifdef __cplusplus
}
#endif

#endif
