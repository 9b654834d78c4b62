/*
 * b200jk.h — C ABI of the B200 direct-SCF Coulomb/exchange (J/K) engine.
 *
 * Every entry point returns an int status (B200JK_OK = 0); on failure
 * b200jk_last_error() gives a message for the calling thread.  No torch or
 * CUDA types appear in the signatures: densities and outputs are plain
 * double arrays, either host memory or device memory of the plan's GPU
 * (flag dev_ptrs), and a stream is passed as void* (NULL = the plan's own).
 *
 * The entry points replace PySCF 2.12.1's direct-SCF path:
 *
 *   b200jk_plan_create     SCF.init_direct_scf / _vhf._VHFOpt(mol, 'int2e',
 *                          'CVHFnrs8_prescreen', 'CVHFnr_int2e_q_cond',
 *                          'CVHFnr_dm_cond', direct_scf_tol)
 *                          (pyscf/scf/hf.py:2045-2054, pyscf/scf/_vhf.py:151-206);
 *                          the Schwarz conditioner is CVHFnr_int2e_q_cond
 *                          (pyscf/lib/vhf/optimizer.c:408-454)
 *   b200jk_get_q_cond      _VHFOpt.q_cond (pyscf/scf/_vhf.py:240-249)
 *   b200jk_get_jk          _vhf.direct(dms, atm, bas, env, vhfopt, hermi, cart,
 *                          with_j, with_k) (pyscf/scf/_vhf.py:405-464), i.e.
 *                          CVHFnr_direct_drv + CVHFdot_nrs8 + int2e_sph +
 *                          CVHFnrs8_ji_s2kl / CVHFnrs8_li_s2kj (hermi=1) or
 *                          CVHFnrs8_li_s1kj (hermi=0), followed by
 *                          lib.hermi_triu (pyscf/lib/vhf/nr_direct.c:355-476,
 *                          pyscf/lib/vhf/nr_direct_dot.c:1293-1647)
 *   b200jk_plan_destroy    CVHFdel_optimizer (pyscf/lib/vhf/optimizer.c:48-62)
 *
 * Input arrays use PySCF's own layout: atm int32 [natm][6], bas int32
 * [nbas][8], env float64 (pyscf/gto/mole.py:58-88, 965-1031).  Densities
 * and outputs are C-ordered (n_dm, nao, nao) float64 in PySCF's AO order
 * (spherical unless cart=1).
 */
#ifndef B200JK_H
#define B200JK_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B200JK_OK            0
#define B200JK_EINVAL        1   /* bad argument */
#define B200JK_EUNSUPPORTED  2   /* input outside what the engine implements */
#define B200JK_ECUDA         3   /* CUDA runtime error */
#define B200JK_ENOMEM        4   /* device allocation failed */
#define B200JK_ENOTBUILT     5   /* library built without device code */

#define B200JK_PREC_FP64     0   /* all quartets in float64 */
#define B200JK_PREC_MIXED    1   /* quartets with q_ij q_kl max|D| < tau evaluated in
                                    float32, all contraction and accumulation in
                                    float64; tau set by b200jk_set_mixed_threshold */

#define B200JK_SCREEN_NRS8   0   /* CVHFnrs8_prescreen (J and K terms) */
#define B200JK_SCREEN_VJ     1   /* CVHFnrs8_vj_prescreen (J terms only) */
#define B200JK_SCREEN_VK     2   /* CVHFnrs8_vk_prescreen (K terms only) */

typedef struct b200jk_plan b200jk_plan;
typedef struct b200jk_batch b200jk_batch;

typedef struct {
    int64_t quartets;            /* shell quartets evaluated by the last build */
    int64_t prim_quartets;       /* primitive quartets evaluated by the last build */
    int64_t shell_pairs;         /* significant shell pairs in the plan */
    int64_t prim_pairs;          /* primitive pairs in the plan */
    double  flops;               /* modelled FP64 flops of the last build */
    double  last_build_ms;       /* device time of the last J/K build */
    int32_t nao, nao_cart, nbas, nseg;
    int64_t kernel_launches;     /* kernels this library launched in the last build */
    int64_t fp32_quartets;       /* of quartets, those evaluated in float32 (mixed mode) */
    int64_t fp32_prim_quartets;  /* of prim_quartets, those evaluated in float32 */
} b200jk_stats_t;

typedef struct {
    int32_t la, lb, lc, ld;      /* quartet class (la lb | lc ld) */
    int64_t quartets;            /* shell quartets evaluated in the last build */
    int64_t prim_quartets;       /* primitive quartets evaluated in the last build */
    double  ms;                  /* kernel time of the class (profiling on), else 0 */
    int32_t family;              /* 0 thread-per-quartet, 1 warp-per-quartet */
    int32_t pad;
    int64_t fp32_quartets;       /* of quartets, those evaluated in float32 */
} b200jk_class_stat_t;

/* Library version, (major << 16) | minor. */
int b200jk_version(void);

/* Message of the last failure on this thread ("" if none). */
const char *b200jk_last_error(void);

/* Number of CUDA devices visible to the library (0 when none). */
int b200jk_device_count(int *count);

/* Build a plan for one molecule/basis: shell pairs, primitive pairs and the
 * Schwarz conditioner q_cond on GPU `device`.  direct_scf_tol <= 0 disables
 * screening (the reference's vhfopt=None).  The molecule arrays are checked
 * on the host before any device work: atom indices and env pointers out of
 * range give B200JK_EINVAL, l > 3 and env[PTR_RANGE_OMEGA] < 0 (the
 * short-range erfc operator: the long-range plan's build subtracted from the
 * full one gives it) give B200JK_EUNSUPPORTED, without touching a GPU.
 * env[PTR_RANGE_OMEGA] > 0 plans the long-range operator erf(omega r12)/r12
 * (mol.with_range_coulomb(omega), pyscf/scf/_vhf.py:611-627). */
int b200jk_plan_create(const int32_t *atm, int natm, const int32_t *bas, int nbas,
                       const double *env, int env_len, int cart, double direct_scf_tol,
                       int device, b200jk_plan **out);

int b200jk_plan_destroy(b200jk_plan *plan);

/* Move the plan to a new geometry: env is the molecule's env array with new
 * coordinates (same atoms and basis as at creation).  The shell pairs,
 * primitive pairs and q_cond are planned again; workspaces, stream, tuning,
 * shard, screen and mixed threshold are kept, so a geometry scan or an
 * autograd forward pass reuses the plan instead of creating one per point.
 * Graphs captured from batched builds of the plan become invalid (the next
 * b200jk_batch_get_jk_async refuses until b200jk_batch_get_jk ran).  The
 * reference rebuilds its _VHFOpt per geometry (SCF.init_direct_scf,
 * pyscf/scf/hf.py:2045-2054, after mol.set_geom_). */
int b200jk_plan_update_coords(b200jk_plan *plan, const double *env, int env_len);

/* nao in the output basis, nbas. */
int b200jk_plan_dims(const b200jk_plan *plan, int *nao, int *nbas);

/* One-electron integrals of the plan's basis in the output AO basis,
 * (nao, nao) C order, host or device memory as dev_ptrs (either may be NULL):
 *   ovlp   the overlap matrix, int1e_ovlp (SCF.get_ovlp, pyscf/scf/hf.py:341)
 *   hcore  kinetic energy + nuclear attraction of the point (or fractional)
 *          nuclear charges of atm, int1e_kin + int1e_nuc (get_hcore,
 *          pyscf/scf/hf.py:315-340, without ECP and finite-nucleus terms:
 *          atoms with those give B200JK_EUNSUPPORTED).
 * No Schwarz screening; primitive pairs as in the J/K build (exp(-ab/(a+b)
 * |AB|^2) >= e^-60). */
int b200jk_int1e(b200jk_plan *plan, double *ovlp, double *hcore, int dev_ptrs, void *stream);

/* One-electron part of the RHF nuclear gradient, contracted on the GPU:
 * de[natm][3] (overwritten) = the hcore and overlap lines of grad_elec
 * (pyscf/grad/rhf.py:57-66),
 *   de[k] = einsum('xij,ij->x', hcore_deriv(k), dm)
 *         - 2 einsum('xij,ij->x', s1[:, p0:p1], dme[p0:p1]),
 * hcore_deriv the int1e_ipkin + int1e_ipnuc + int1e_iprinv derivatives of
 * hcore_generator (:121-143) and s1 = -int1e_ipovlp (:145-146).  dm and dme
 * (the energy-weighted density, make_rdm1e) are symmetric (nao, nao); the
 * nuclear repulsion term (grad_nuc) and the two-electron term
 * (b200jk_grad_contract) are separate.  Host or device memory as dev_ptrs.
 * Point or fractional charges only (as b200jk_int1e). */
int b200jk_grad_int1e(b200jk_plan *plan, const double *dm, const double *dme, double *de, int dev_ptrs, void *stream);

/* The s8-packed two-electron integral tensor of the plan's basis, the array
 * mol.intor('int2e', aosym='s8') returns (GTO2e_cart_or_sph,
 * pyscf/lib/vhf/fill_nr_s8.c:110-138): entry (ij|kl), i >= j, k >= l, pair
 * index ij = i(i+1)/2 + j >= kl, at ij(ij+1)/2 + kl; len must be
 * npair(npair+1)/2 with npair = nao(nao+1)/2.  Quartets of shells with
 * q_ij q_kl <= 1e-14 are zero, as in the reference (CVHFnr_schwarz_cond with
 * the optimizer's default cutoff, pyscf/lib/vhf/optimizer.c:40, :71-88).
 * eri is device memory of the plan's GPU (dev_ptr = 1) or host memory; it is
 * overwritten.  The long-range operator of the plan (env[PTR_RANGE_OMEGA] > 0)
 * applies. */
int b200jk_int2e_s8(b200jk_plan *plan, double *eri, long long len, int dev_ptr, void *stream);

/* J/K from a stored integral tensor: the in-core path _vhf.incore
 * (pyscf/scf/_vhf.py:318-401, CVHFnrs8_incore_drv / CVHFnrs4_incore_drv with
 * pyscf/lib/vhf/nr_incore.c).  eri is the s8 tensor (eri_len =
 * npair(npair+1)/2) or the s4 matrix (eri_len = npair^2, row ij, column kl);
 * any other length is B200JK_EINVAL ("Array shape not consistent", as the
 * reference's RuntimeError).  dms (n_dm, nao, nao); vj, vk outputs of the same
 * shape, overwritten: J = einsum('ijkl,ji->kl'), K = einsum('ijkl,jk->il')
 * over the full tensor, then the reference's hermi_triu (vj always, vk for
 * hermi != 0).  hermi = 1 (2) takes the densities to be symmetric
 * (antisymmetric), as the reference's s2il (s1il + hermi_triu) kernels do.
 * All arrays are device memory of `device` (dev_ptrs = 1) or host memory (the
 * tensor is then copied to the GPU on every call).  No plan is needed. */
int b200jk_incore_jk(const double *eri, long long eri_len, int nao, const double *dms, int n_dm, int hermi,
                     int with_j, int with_k, double *vj, double *vk, int dev_ptrs, int device, void *stream);

/* Copy q_cond (nbas x nbas, C order) to host memory. */
int b200jk_get_q_cond(const b200jk_plan *plan, double *q_cond);

/* J/K for n_dm densities.  dms, vj, vk are (n_dm, nao, nao) C-ordered;
 * vj / vk may be NULL when with_j / with_k is 0.  Outputs are overwritten.
 * hermi: 1 symmetric densities, 0 general, 2 antisymmetric (as PySCF).
 * dev_ptrs: 0 host arrays, 1 device arrays on the plan's GPU (other memory is
 * rejected with B200JK_EINVAL).  stream: a cudaStream_t or NULL.
 * Non-finite density entries are not rejected (nor are they by the
 * reference): the screening bound ignores them and they propagate into the
 * J/K elements of every quartet that contracts with them; the plan stays
 * usable for the next build. */
int b200jk_get_jk(b200jk_plan *plan, const double *dms, int n_dm, int hermi,
                  int with_j, int with_k, double *vj, double *vk,
                  int dev_ptrs, int precision_mode, void *stream);

/* J/K like b200jk_get_jk, for callers that cannot let the library allocate
 * device memory (code running under a framework's caching allocator or a
 * fixed memory budget, where a cudaMalloc can fail or stall the device).  It
 * has no counterpart in the reference.  dms, vj, vk must be device arrays on
 * the plan's GPU (anything else is rejected with B200JK_EINVAL); nothing is
 * allocated: all intermediates live in one fixed 32 MiB scratch array that
 * every GPU loading the library holds until exit, which bounds the size
 * (roughly nao_cart <= 600 for one density); larger inputs are rejected with
 * B200JK_EINVAL and a message giving the bytes needed.  The first call on a
 * device also resolves the scratch array's device address (a one-time
 * set-up); make that first call before any stream capture begins.  The call
 * returns after `stream` has finished the build.  All calls share the one
 * array: calls that overlap on the GPU (other streams, other threads) race
 * and must be serialised by the caller.  A sharded plan (b200jk_set_shard)
 * gives its partial J/K, as b200jk_get_jk does.  The plan itself is created
 * (and allocated) by b200jk_plan_create beforehand. */
int b200jk_get_jk_noalloc(b200jk_plan *plan, const double *dms, int n_dm, int hermi,
                          int with_j, int with_k, double *vj, double *vk, void *stream);

/* Counters of the last build. */
int b200jk_stats(const b200jk_plan *plan, b200jk_stats_t *stats);

/* Per-quartet-class counters of the last build; *n receives the number of
 * classes (at most max are written).  With profiling on (b200jk_set_profiling)
 * each class kernel is bracketed by CUDA events and ms is filled in. */
int b200jk_class_stats(const b200jk_plan *plan, b200jk_class_stat_t *out, int max, int *n);
int b200jk_set_profiling(b200jk_plan *plan, int on);

/* Autotuner: for every quartet class with more than one launch variant (the
 * register family with one or several kets per lane, or bra runs; the shared-memory
 * family with full- or half-width lane groups per quartet), time each variant
 * on FP64 J/K builds of the density dm (nao x nao, symmetric; host array, or
 * device array with dev_ptrs = 1), then the float32 pass's variants on mixed
 * builds at the plan's threshold, and keep the faster for later builds of
 * this plan (and of batches whose first plan it is; a batch runs bra runs
 * as variant 0).  Five builds.  No
 * reference counterpart (PySCF has no kernel variants to tune). */
int b200jk_autotune(b200jk_plan *plan, const double *dm, int dev_ptrs, void *stream);

/* Chunk order of the class kernels: tiles of tile_b bra pairs walked
 * ket-chunk-major, so warps running together share ket data (default 64);
 * 0 = bra-major order.  Sharded plans always use bra-major order. */
int b200jk_set_tile(b200jk_plan *plan, int tile_b);

/* The chosen variant per quartet class (55 classes, bra class >= ket class)
 * for float64 quartets (precision B200JK_PREC_FP64) or for the float32 pass
 * of mixed builds (B200JK_PREC_MIXED).  Before any tuning: 0 everywhere on
 * plans of fewer than 1500 AOs; from 1500 AOs on, the float64 pass uses the
 * autotuner's measured choices on a large cc-pVTZ workload (bra runs for
 * eight classes of s and p kets, half-width groups for (21|20) and (22|10)). */
int b200jk_get_tuning(const b200jk_plan *plan, int precision, int *variants, int max, int *n);

/* Set the variants directly (n = 55; 0 everywhere, 1 or 2 only where the
 * class has that variant, 2 only for B200JK_PREC_FP64, else B200JK_EINVAL):
 * replays a tuning without timing.  Variant 2 (register family, bra runs: a
 * warp keeps its kets for 4 consecutive bra pairs and carries their K[a,*]
 * and ket-side J sums in registers) applies to the float64 pass of unsharded
 * builds of one symmetric density; other builds run such classes as 0. */
int b200jk_set_tuning(b200jk_plan *plan, int precision, const int *variants, int n);

/* Nuclear-gradient J/K: the drop-in for pyscf.grad.rhf.get_jk(mol, dm)
 * (pyscf/grad/rhf.py:149-178, i.e. _vhf.direct_mapdm('int2e_ip1', 's2kl',
 * ('lk->s1ij', 'jk->s1il'), dm, 3, ...) with CVHFgrad_jk_prescreen,
 * pyscf/lib/vhf/hessian_screen.c:44-123).  For each of the n_dm densities
 * (nao x nao, C order, need not be symmetric)
 *     vj[s][x][i][j] = -sum_kl (d_x i j|kl) D[l][k]
 *     vk[s][x][i][l] = -sum_jk (d_x i j|kl) D[j][k]
 * with d_x the x derivative acting on function i (libcint's int2e_ip1,
 * nabla on the electron coordinate); outputs (n_dm, 3, nao, nao)
 * are overwritten.  direct_scf_tol is the gradient screen's threshold (the
 * reference uses 1e-14); <= 0 disables screening.  dev_ptrs: 0 host arrays,
 * 1 device arrays on the plan's GPU.  The first call builds the derivative
 * Schwarz bound of the plan (int2e_ip1ip2 diagonal) on the GPU. */
int b200jk_grad_jk(b200jk_plan *plan, const double *dms, int n_dm, int with_j, int with_k,
                   double *vj, double *vk, int dev_ptrs, double direct_scf_tol, void *stream);

/* The two-electron part of the RHF nuclear gradient, contracted on the GPU
 * without forming vj/vk: for one symmetric density dm (nao x nao, C order)
 *     de[A][x] = 2 sum_{i in A} sum_j (vj - vk/2)[x][i][j] dm[i][j]
 * with vj, vk those of b200jk_grad_jk, i.e. the term grad_elec adds from
 * get_veff (pyscf/grad/rhf.py:62-68, get_veff :180-183 -> get_jk :149-178).
 * Each quartet contributes sum_abcd (d_x ab|cd) W_abcd with
 * W = 2 D_ab (D_cd + D_dc) - D_ac D_bd - D_ad D_bc, summed over the warp that
 * owns the bra pair before one atomic per atom and direction: no
 * (3, nao, nao) arrays are materialised.  de is (natm, 3), overwritten; host
 * or device memory as dev_ptrs; the screen is b200jk_grad_jk's. */
int b200jk_grad_contract(b200jk_plan *plan, const double *dm, double *de, int dev_ptrs,
                         double direct_scf_tol, void *stream);

/* Counters of the last gradient build: shell quartets (bra sides), primitive
 * quartets, device time (ms), kernels launched by this library. */
int b200jk_grad_stats(const b200jk_plan *plan, int64_t *quartets, int64_t *prim_quartets, double *ms,
                      int64_t *kernel_launches);

/* Per (bra class, ket class) counters of the last gradient build (100
 * entries; quartets = bra sides), with kernel times when profiling is on. */
int b200jk_grad_class_stats(const b200jk_plan *plan, b200jk_class_stat_t *out, int max, int *n);

/* The two screening planes of the gradient (2, nbas, nbas): plane 0 the
 * derivative bound sqrt(max |(d_x i j|d_x i j)|) with the derivative on the
 * row shell (CVHFnr_int2e_pp_q_cond), plane 1 q_cond. */
int b200jk_get_grad_q_cond(b200jk_plan *plan, double *q_cond);

/* Batches of molecules: the J/K builds of many plans (one per molecule, all
 * on one GPU, not sharded) in one launch per quartet class over a global
 * quartet queue, instead of one set of launches per molecule.  No reference
 * counterpart: PySCF builds J/K one molecule at a time.  The plans must
 * outlive the batch. */
int b200jk_batch_create(b200jk_plan *const *plans, int nmol, b200jk_batch **out);
int b200jk_batch_destroy(b200jk_batch *batch);

/* J/K of one density per molecule: dms[m], vj[m], vk[m] are DEVICE pointers to
 * C-ordered (nao_m, nao_m) float64 arrays (outputs overwritten; vj or vk may
 * be NULL with with_j / with_k 0).  hermi and precision_mode as in
 * b200jk_get_jk; the mixed threshold is the first plan's. */
int b200jk_batch_get_jk(b200jk_batch *batch, const double *const *dms, int hermi, int with_j, int with_k,
                        double *const *vj, double *const *vk, int precision_mode, void *stream);

/* The same launches as b200jk_batch_get_jk with nothing else: no
 * allocation, no host synchronisation, no statistics read-back, so that the
 * caller can capture them in a CUDA graph (stream capture of `stream`) and
 * replay the whole batched build; the graph reads dms[m] and writes vj[m],
 * vk[m] at the addresses given here.  Needs one b200jk_batch_get_jk call
 * with the same arguments first (it sizes every buffer); one captured graph
 * per batch at a time (they share the pinned argument staging).  A captured
 * graph holds the addresses of the plans' workspaces: a later build on one
 * of the plans that grows its workspace (b200jk_get_jk with more densities)
 * or destroying a plan invalidates it.  This call detects the first case and
 * returns B200JK_EINVAL until b200jk_batch_get_jk has run again; the caller
 * must not replay graphs captured before.  No reference counterpart. */
int b200jk_batch_get_jk_async(b200jk_batch *batch, const double *const *dms, int hermi, int with_j, int with_k,
                              double *const *vj, double *const *vk, int precision_mode, void *stream);

/* Counters of the last batched build: quartets (all molecules), of them in
 * float32, device time (ms), kernels launched by this library. */
int b200jk_batch_stats(const b200jk_batch *batch, int64_t *quartets, int64_t *fp32_quartets, double *ms,
                       int64_t *kernel_launches);

/* Multi-GPU sharding: the plan's J/K and gradient builds evaluate only the
 * bra shell pairs ij = index (mod count) of every quartet class, so count
 * plans (one per GPU, same molecule) produce partial results whose sum is the
 * full build; the caller sums them (an all-reduce).  Default index 0, count 1.
 * Replaces the reference's OpenMP split of CVHFnr_direct_drv's block loop
 * (pyscf/lib/vhf/nr_direct.c:355-476) across GPUs. */
int b200jk_set_shard(b200jk_plan *plan, int index, int count);

/* Density part of the per-quartet screen for the plan's later builds:
 * B200JK_SCREEN_NRS8 (default) keeps a quartet when
 * max(4 D_ji, 4 D_lk, D_jk, D_jl, D_ik, D_il) q_ij q_kl > tol, _VJ uses the
 * two J terms only, _VK the four K terms only.  The reference sets these on
 * its _VHFOpt (CVHFnrs8_prescreen / CVHFnrs8_vj_prescreen /
 * CVHFnrs8_vk_prescreen, pyscf/lib/vhf/optimizer.c:90-167); SCF.get_jk
 * switches to the J or K screen when only one of J, K is built
 * (pyscf/scf/hf.py:2069-2077). */
int b200jk_set_prescreen(b200jk_plan *plan, int screen);

/* Threshold tau of B200JK_PREC_MIXED (default 1e-6): a shell quartet whose
 * Schwarz bound times the largest density element, q_ij q_kl max|D|, is below
 * tau is evaluated in float32.  The bound uses the density passed to each
 * build, so incremental (difference-density) builds move more quartets to
 * float32 as the SCF converges.  tau <= 0 makes mixed mode all-float64.
 * No reference counterpart: PySCF evaluates every quartet in float64. */
int b200jk_set_mixed_threshold(b200jk_plan *plan, double tau);   /* also clears per-class thresholds */

/* Per-class float32 thresholds of B200JK_PREC_MIXED (n = 55, one per quartet
 * class in the order of b200jk_class_stats; >= 0, 0 keeps the class in
 * float64); tau NULL or n = 0 returns to the plan's single threshold, as
 * b200jk_set_mixed_threshold does.  Batches use their first plan's. */
int b200jk_set_class_thresholds(b200jk_plan *plan, const double *tau, int n);
int b200jk_get_class_thresholds(const b200jk_plan *plan, double *tau, int max, int *n);

/* Mixed-precision tuner: picks the float32 threshold of every quartet class
 * for the density dm (nao x nao, symmetric; host, or device with dev_ptrs).
 * Classes whose float32 kernels are not faster than their float64 ones (class
 * CUDA events of an all-float64 and an all-float32 build) stay in float64;
 * the others get the largest threshold of the ladder 1e-2 ... 1e-8 for which
 * the two-electron energy E2 = 1/2 tr(D J) - 1/4 tr(D K) of the mixed build
 * stays within `budget` (Eh) of the all-float64 build's.  The thresholds are
 * kept for later builds (b200jk_get_class_thresholds).  result, if not NULL,
 * receives {chosen threshold, dE2, max|dJ|, max|dK|} of the accepted build
 * against the float64 one.  At most 9 builds.  No reference counterpart
 * (PySCF evaluates every quartet in float64). */
int b200jk_autotune_mixed(b200jk_plan *plan, const double *dm, int dev_ptrs, double budget, double *result,
                          void *stream);

/* Measured FP64 FMA throughput of device `device` (TFLOP/s), from a
 * register-resident FMA loop over all SMs: the denominator of the FP64
 * roofline fraction. */
int b200jk_measure_fp64_peak(int device, double *tflops);

/* Test hook, no reference counterpart: the nth device allocation made by
 * the library from now on fails as an out-of-memory condition would (the
 * call returns B200JK_ENOMEM and frees what it had taken); 0 turns it off. */
int b200jk_debug_fail_alloc(int nth);

/* Host replay of the device integral code for one shell quartet (no GPU is
 * used): the Cartesian block (ab|cd) of shells shls[0..3] of the given
 * basis, primitives contracted with env's coefficients, without angular
 * normalisation; out is C-ordered [a][b][c][d] (cart components in PySCF
 * order).  For validating the kernels' arithmetic against a CPU reference. */
int b200jk_hostcheck_cart_quartet(const int32_t *atm, int natm, const int32_t *bas, int nbas,
                                  const double *env, const int32_t *shls, double *out);

/* The same block evaluated in float32 with the float32 tables, as the float32
 * pass of B200JK_PREC_MIXED does (coordinates relative to the first centre);
 * out is float64.  No reference counterpart (validation only). */
int b200jk_hostcheck_cart_quartet_fp32(const int32_t *atm, int natm, const int32_t *bas, int nbas,
                                       const double *env, const int32_t *shls, double *out);

#ifdef __cplusplus
}
#endif

#endif
