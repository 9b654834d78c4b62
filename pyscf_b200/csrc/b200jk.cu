// b200jk.cu — host planner, kernel dispatch and C ABI of the B200 J/K engine.
//
// The ABI (include/b200jk.h) is the drop-in for PySCF's direct-SCF path
// (pyscf/scf/_vhf.py:405-464 -> pyscf/lib/vhf/nr_direct.c:355-476).  The
// planner turns PySCF's _atm/_bas/_env (pyscf/gto/mole.py:58-88, 965-1031)
// into device tables:
//   segments      one per (shell, contraction column); a generally contracted
//                 shell (nctr > 1) becomes nctr segments sharing its exponents;
//   shell pairs   unordered segment pairs, oriented la >= lb, grouped into 10
//                 angular classes, sorted by the parent-shell Schwarz bound;
//   prim pairs    (P, p, K_ab c_a c_b, 1/(2p)) per surviving primitive pair
//                 (exp(-ab/(a+b) |AB|^2) >= e^-60, the libcint default cutoff);
//   q_cond        CVHFnr_int2e_q_cond on parent shells, computed on the GPU.
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>
#include <stdint.h>
#include <string.h>
#include <stdio.h>
#include <math.h>
#include <string>
#include <vector>
#include <algorithm>
#include <numeric>
#include <mutex>
#include <atomic>

#define RYS_TABLE_QUALIFIER static const
#include "rys_math.cuh"
#include "jk_launch.h"
#include "grad_launch.h"
#include "int1e_kernels.cuh"
#include "fill_launch.h"
#include "incore_launch.h"
#include "../../include/b200jk.h"

using namespace b200jk;

// ---------------------------------------------------------------------------
// errors

static thread_local std::string g_last_error;

static int fail(int code, const std::string &msg)
{
        g_last_error = msg;
        return code;
}

#define CUDA_TRY(expr)                                                                 \
        do {                                                                           \
                cudaError_t _e = (expr);                                               \
                if (_e != cudaSuccess)                                                 \
                        return fail(B200JK_ECUDA, std::string(#expr) + ": " +          \
                                                      cudaGetErrorString(_e));         \
        } while (0)

// A pointer the caller declares to be device memory must be memory the
// kernels of `device` can address: device (or managed) memory of that GPU.
// Host memory handed to a kernel would fault the GPU instead of returning an
// error, so it is rejected here.
static int check_dev_ptr(const void *p, int device, const char *what)
{
        if (!p) return B200JK_OK;
        cudaPointerAttributes at;
        const cudaError_t e = cudaPointerGetAttributes(&at, p);
        if (e != cudaSuccess) {
                cudaGetLastError();
                return fail(B200JK_EINVAL, std::string(what) + " is not a CUDA pointer");
        }
        if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
                return fail(B200JK_EINVAL, std::string(what) + " is not device memory (pass dev_ptrs = 0 for host arrays)");
        if (at.type == cudaMemoryTypeDevice && at.device != device)
                return fail(B200JK_EINVAL, std::string(what) + " lives on cuda:" + std::to_string(at.device) +
                                                   ", the plan on cuda:" + std::to_string(device));
        return B200JK_OK;
}

// Test hook: when positive, the n-th device allocation from now on fails as
// an out-of-memory condition would (b200jk_debug_fail_alloc).  0 = off.
static std::atomic<long long> g_fail_alloc_countdown{0};
static bool alloc_should_fail()
{
        long long v = g_fail_alloc_countdown.load();
        while (v > 0) {
                if (g_fail_alloc_countdown.compare_exchange_weak(v, v - 1)) return v == 1;
        }
        return false;
}

static inline unsigned grid_for(long long n, int block) { return (unsigned)((n + block - 1) / block); }

// slot layout of PySCF's _atm/_bas/_env (pyscf/gto/mole.py:58-88)
enum { CHARGE_OF = 0, PTR_COORD = 1, ATM_SLOTS = 6 };
enum { ATOM_OF = 0, ANG_OF = 1, NPRIM_OF = 2, NCTR_OF = 3, PTR_EXP = 5, PTR_COEFF = 6, BAS_SLOTS = 8 };
enum { PTR_RANGE_OMEGA = 8 };

static const int LMAX = 3;
static const int NPAIRCLASS = (LMAX + 1) * (LMAX + 2) / 2;
static inline int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }

__device__ __align__(32) double d_rys_table[rys_padded_size()];
// the float32 tables (degree 7, earlier large-T limit) of the float32 pass of
// mixed precision
__device__ __align__(32) float d_rys_table_f[RYS_F_SIZE];

// ---------------------------------------------------------------------------
// real solid harmonics r^l Y_lm (unit-normalised Y_lm), rows m = -l..l
// (p ordered x, y, z), columns Cartesian components in PySCF order.
// Helgaker, Jorgensen & Olsen, Molecular Electronic-Structure Theory,
// eqs. 6.4.47-6.4.50, times sqrt((2l+1)/(4 pi)).

static double factd(int n) { double r = 1; for (int i = 2; i <= n; i++) r *= i; return r; }
static double binomd(int n, int k) { return (k < 0 || k > n) ? 0.0 : factd(n) / (factd(k) * factd(n - k)); }

static void solid_harmonics(int l, double *rows /* [2l+1][ncart(l)] */)
{
        const int nc = ncart(l);
        for (int i = 0; i < (2 * l + 1) * nc; i++) rows[i] = 0;
        const double scale = sqrt((2 * l + 1) / (4 * M_PI));
        for (int m = -l; m <= l; m++) {
                const int am = abs(m);
                const int wm = m < 0 ? 1 : 0;   // 2*v_m
                const double nlm = 1.0 / (pow(2.0, am) * factd(l)) *
                                   sqrt(2 * factd(l + am) * factd(l - am) / (m == 0 ? 2.0 : 1.0));
                const int row = (l == 1) ? (m == 1 ? 0 : (m == -1 ? 1 : 2)) : m + l;
                for (int t = 0; t <= (l - am) / 2; t++)
                        for (int u = 0; u <= t; u++) {
                                const int wmax = 2 * ((am - wm) / 2) + wm;
                                for (int w = wm; w <= wmax; w += 2) {
                                        const int sgn = ((t + (w - wm) / 2) % 2) ? -1 : 1;
                                        const double cf = sgn * pow(0.25, t) * binomd(l, t) * binomd(l - t, am + t) *
                                                          binomd(t, u) * binomd(am, w);
                                        const int px = 2 * t + am - 2 * u - w, py = 2 * u + w, pz = l - 2 * t - am;
                                        if (px < 0 || py < 0 || pz < 0) continue;
                                        int idx = -1;
                                        for (int k = 0; k < nc; k++)
                                                if (cart_lx(l, k) == px && cart_ly(l, k) == py) idx = k;
                                        rows[row * nc + idx] += scale * nlm * cf;
                                }
                        }
        }
}

// c2s[l][row][cart] with 10x10 slots per l: output-basis rows of the Cartesian map
static std::vector<double> build_c2s(int cart)
{
        std::vector<double> t((LMAX + 1) * 100, 0.0);
        for (int l = 0; l <= LMAX; l++) {
                const int nc = ncart(l);
                if (cart || l < 2) {
                        const double f = l == 0 ? 0.282094791773878143 : (l == 1 ? 0.488602511902919921 : 1.0);
                        for (int k = 0; k < nc; k++) t[l * 100 + k * 10 + k] = f;
                } else {
                        std::vector<double> rows((2 * l + 1) * nc);
                        solid_harmonics(l, rows.data());
                        for (int m = 0; m < 2 * l + 1; m++)
                                for (int k = 0; k < nc; k++) t[l * 100 + m * 10 + k] = rows[m * nc + k];
                }
        }
        return t;
}

// ---------------------------------------------------------------------------
// plan

struct Seg {
        int parent, l, nprim, ctr;
        const double *exp;
        std::vector<double> coef;
        double R[3];
        int out_off, cart_off;
};

template <typename T>
struct DevArr {
        T *p = nullptr;
        size_t n = 0;
        void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
};

template <typename T>
static int dev_upload(DevArr<T> &d, const std::vector<T> &h)
{
        d.release();
        d.n = h.size();
        if (d.n == 0) return B200JK_OK;
        if (alloc_should_fail() || cudaMalloc(&d.p, sizeof(T) * d.n) != cudaSuccess) {
                d.p = nullptr;
                return fail(B200JK_ENOMEM, "cudaMalloc failed for a plan table");
        }
        CUDA_TRY(cudaMemcpy(d.p, h.data(), sizeof(T) * d.n, cudaMemcpyHostToDevice));
        return B200JK_OK;
}

template <typename T>
static int dev_alloc(DevArr<T> &d, size_t n)
{
        if (d.n >= n && d.p) return B200JK_OK;
        d.release();
        if (n == 0) return B200JK_OK;
        if (alloc_should_fail() || cudaMalloc(&d.p, sizeof(T) * n) != cudaSuccess) {
                d.p = nullptr;
                return fail(B200JK_ENOMEM, "cudaMalloc failed for a workspace buffer");
        }
        d.n = n;
        return B200JK_OK;
}

struct PairClassDev {
        int la = 0, lb = 0, n = 0;
        int boff[B2_NBUCKET + 1] = {0, 0, 0, 0, 0};
        DevArr<int4> sh;
        DevArr<int2> pr;
        DevArr<double> q, qs;
        DevArr<double4> A, AB;
        PairView view() const
        {
                PairView v;
                v.sh = sh.p; v.pr = pr.p; v.q = q.p; v.qs = qs.p; v.A = A.p; v.AB = AB.p; v.n = n;
                for (int b = 0; b <= B2_NBUCKET; b++) v.boff[b] = boff[b];
                return v;
        }
        void release() { sh.release(); pr.release(); q.release(); qs.release(); A.release(); AB.release(); n = 0; }
};

// what the gradient set-up keeps of the planner's segments and pairs
struct SegLite {
        int parent, l, cart_off;
        double R[3];
};
struct PairLite {
        int i, j;              // segments, l_i >= l_j
        int prim0, nprim;      // primitive pairs
};

// Gradient J/K state of a plan (built on the first gradient call): the
// derivative Schwarz bound q0 and the bra/ket pair lists of the gradient
// screen, plus the per-call workspace.
struct GradPlan {
        bool q0_ready = false, lists_ready = false;
        double tol = 0;
        PairClassDev bra[NPAIRCLASS], ket[NPAIRCLASS];
        DevArr<double> q0;
        DevArr<int2> goff;
        std::vector<size_t> goff_at;   // [X * NPAIRCLASS + Y], then NPAIRCLASS^2 + X for q0
        std::vector<double> h_q0;
        DevArr<double> D, Dc, Ds, V, out, dmc, fac, de;
        DevArr<int> shell_atom;
        DevArr<unsigned long long> dmax, stats;
        DevArr<int> nkl, kst;
        DevArr<long long> nchunk, chunk_off;
        DevArr<unsigned char> cub_tmp;
        int64_t quartets = 0, prim_quartets = 0, launches = 0;
        double last_ms = 0;
        std::vector<b200jk_class_stat_t> cls;   // per (bra class, ket class)
        std::vector<cudaEvent_t> cls_ev;
        void release()
        {
                for (auto e : cls_ev) cudaEventDestroy(e);
                cls_ev.clear();
                for (auto &c : bra) c.release();
                for (auto &c : ket) c.release();
                q0.release(); goff.release(); D.release(); Dc.release(); Ds.release(); V.release(); out.release();
                de.release(); shell_atom.release();
                dmc.release(); fac.release(); dmax.release(); stats.release(); nkl.release(); kst.release();
                nchunk.release(); chunk_off.release(); cub_tmp.release();
        }
};

struct b200jk_plan {
        int device = 0, cart = 0, natm = 0, nbas = 0, nao = 0, naoc = 0, nseg = 0;
        double tol = 0;
        // mixed precision: quartets with q_ij q_kl max|D| below fp32_tau run in
        // float32; tau_class (when set: one per quartet class, from
        // b200jk_set_class_thresholds or b200jk_autotune_mixed) replaces it per class
        double fp32_tau = 1e-6;
        std::vector<double> tau_class;
        // multi-GPU: this plan evaluates the bra pairs ij = shard (mod nshard)
        int shard = 0, nshard = 1;
        // launch variant per quartet class (register family: 0 = one ket per
        // lane, 1 = family_ket_run kets per lane; shared-memory family: 0 =
        // family_group lanes per quartet, 1 = half as many), chosen by
        // b200jk_autotune: kvar for float64 quartets, kvar32 for the float32
        // pass of mixed builds
        std::vector<int> kvar, kvar32;
        // bra pairs per tile of the tiled chunk order (0: bra-major order)
        int tile_b = 64;
        // density part of the quartet screen (B200JK_SCREEN_*)
        int screen = B200JK_SCREEN_NRS8;
        // omega^2 of the long-range operator erf(omega r12)/r12 (0: Coulomb)
        double omega2 = 0.0;
        // packed ket blocks for the J contraction: class X's blocks start at
        // pk_off[X] (entries, in ket-list order); pk_src maps entries to the
        // Cartesian matrix
        std::vector<long long> pk_off;
        long long pk_total = 0;
        DevArr<long long> pk_src;
        DevArr<double> Dpk, Jpk;
        std::vector<int> ao_loc;
        std::vector<int> shell_atom;   // atom of every PySCF shell (bas[:, ATOM_OF])
        std::vector<int32_t> h_atm, h_bas;   // the molecule's atm / bas (for b200jk_plan_update_coords)
        // nuclei of the one-electron integrals: (x, y, z, Z); nuc_model_ok is
        // false when an atom has a finite-nucleus model or an ECP core
        std::vector<double4> h_atoms;
        bool nuc_model_ok = true;
        // one-electron integrals: pair list and buffers (built on first use)
        DevArr<int4> i1_pair;
        DevArr<long long> i1_off;
        DevArr<double4> i1_seg, i1_atoms;
        DevArr<int> i1_seg_cart, i1_seg_atom;
        DevArr<double> i1_S, i1_H, i1_zero, i1_out, i1_de;
        int i1_npair = -1;
        // s8 integral fill: the pair lists of its Schwarz cutoff and the
        // count/scan workspace (built on first use)
        bool fill_ready = false;
        PairClassDev fill_pc[NPAIRCLASS];
        DevArr<double> fill_one;
        DevArr<int> fill_nkl, fill_kst;
        DevArr<long long> fill_nchunk, fill_chunk_off;
        DevArr<unsigned char> fill_cub;
        void release_fill()
        {
                for (auto &c : fill_pc) c.release();
                fill_one.release(); fill_nkl.release(); fill_kst.release();
                fill_nchunk.release(); fill_chunk_off.release(); fill_cub.release();
                fill_ready = false;
        }
        std::vector<double> h_qcond;
        PairClassDev pc[NPAIRCLASS];
        DevArr<double4> PP;
        DevArr<double2> PK;
        DevArr<double2> PE;            // primitive exponents (alpha of i, beta of j) per primitive pair
        std::vector<SegLite> segl;
        std::vector<PairLite> all_pairs[NPAIRCLASS];   // before screening
        GradPlan grad;
        DevArr<double> c2s, qcond, dm_cond;
        DevArr<int> goff_all;
        std::vector<size_t> goff_at;   // per quartet class
        DevArr<int4> seg_info;
        DevArr<int> out_seg, out_comp, cart_seg, cart_comp, ao_loc_d;
        // workspace; ws_gen counts the times its buffers moved
        int ws_ndm = 0;
        long long ws_gen = 0;
        DevArr<double> D, Dc, Ds, Jacc, Kacc, outJ, outK;
        DevArr<unsigned long long> dmax, stats;
        DevArr<int> nkl, kst;
        DevArr<long long> nchunk, chunk_off;
        DevArr<unsigned char> cub_tmp;
        cudaStream_t stream = nullptr;
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        int nsm = 148;
        int64_t shell_pairs = 0, prim_pairs = 0;
        b200jk_stats_t st;
        int profiling = 0;
        std::vector<b200jk_class_stat_t> cls;
        std::vector<cudaEvent_t> cls_ev;
        ~b200jk_plan()
        {
                for (auto &c : pc) c.release();
                PP.release(); PK.release(); PE.release(); grad.release(); c2s.release();
                pk_src.release(); Dpk.release(); Jpk.release(); qcond.release(); dm_cond.release();
                goff_all.release(); seg_info.release(); out_seg.release(); out_comp.release();
                cart_seg.release(); cart_comp.release(); ao_loc_d.release();
                D.release(); Dc.release(); Ds.release(); Jacc.release(); Kacc.release(); outJ.release(); outK.release();
                i1_pair.release(); i1_off.release(); i1_seg.release(); i1_atoms.release(); i1_seg_cart.release();
                i1_seg_atom.release(); i1_de.release();
                i1_S.release(); i1_H.release(); i1_zero.release(); i1_out.release();
                release_fill();
                dmax.release(); stats.release(); nkl.release(); kst.release(); nchunk.release(); chunk_off.release(); cub_tmp.release();
                for (auto e : cls_ev) cudaEventDestroy(e);
                if (ev0) cudaEventDestroy(ev0);
                if (ev1) cudaEventDestroy(ev1);
                if (stream) cudaStreamDestroy(stream);
        }
};

// ---------------------------------------------------------------------------
// quartet classes: bra class X >= ket class Y

struct QClass { int X, Y; };
static std::vector<QClass> quartet_classes()
{
        std::vector<QClass> v;
        for (int X = 0; X < NPAIRCLASS; X++)
                for (int Y = 0; Y <= X; Y++) v.push_back({X, Y});
        return v;
}
static void class_l(int X, int &la, int &lb)
{
        for (int a = 0; a <= LMAX; a++)
                for (int b = 0; b <= a; b++)
                        if (pair_class(a, b) == X) { la = a; lb = b; return; }
}

typedef int (*jk_launcher_t)(const JKArgs &, cudaStream_t, int, int, int, const JKArgs *, const long long *, int,
                             std::string &);

// the launch variant of class t in precision pass `pass` (1: float32 quartets)
// Launch variant of a float64 pass in a plan the autotuner has not timed:
// the autotuner's choices on the FP64 build of (H2O)64/cc-pVTZ, where each
// won by 15-25% per class -- bra runs (2) for eight register-family
// classes of s and p kets, half-width groups (1) for (21|20) and (22|10).
// Callers that never tune (a drop-in SCF, whose first builds would pay for
// the timing) get them on plans of DEFAULT_VARIANT_MIN_NAO or more AOs.
// Smaller plans keep variant 0: bra runs give a warp four bra pairs, too
// few warps for a small molecule (warm FP64 builds, defaults vs variant 0:
// nao 192 22.7 vs 11.8 ms, 464 73.0 vs 61.0, 928 263.8 vs 254.8, 1856
// 1975 vs 2022 ms).
static const int DEFAULT_VARIANT_MIN_NAO = 1500;
static int default_fp64_variant(size_t t)
{
        // index = position in quartet_classes(): bra pair class X (00, 10, 11,
        // 20, 21, 22, 30, ...) major, ket pair class Y <= X minor
        static const int table[] = {
                2,                   // (00|00)
                2, 2,                // (10|00) (10|10)
                2, 2, 0,             // (11|00) (11|10) (11|11)
                2, 2, 0, 0,          // (20|00) (20|10) (20|11) (20|20)
                0, 0, 0, 1, 0,       // (21|00) (21|10) (21|11) (21|20) (21|21)
                0, 1, 0, 0, 0, 0,    // (22|00) (22|10) ...
                2,                   // (30|00)
        };
        return t < sizeof(table) / sizeof(table[0]) ? table[t] : 0;
}

static int class_variant(const b200jk_plan *P, size_t t, int pass)
{
        const std::vector<int> &v = pass == 1 ? P->kvar32 : P->kvar;
        if (v.empty()) return pass == 1 || P->nao < DEFAULT_VARIANT_MIN_NAO ? 0 : default_fp64_variant(t);
        return t < v.size() ? v[t] : 0;
}

// the float32 threshold of quartet class t in mixed builds
static double class_tau(const b200jk_plan *P, size_t t)
{
        if (P->tau_class.size() > t) return P->tau_class[t];
        return P->fp32_tau;
}

// the parts of the register family of every class, as its unit was built
int b200jk::family_thread_parts(int la, int lb, int lc, int ld)
{
        typedef int (*np_fn)();
        struct Entry { int la, lb, lc, ld; np_fn fn; };
        static const Entry table[] = {
                {0, 0, 0, 0, launch_jk_0000_np},
                {1, 0, 0, 0, launch_jk_1000_np},
                {1, 0, 1, 0, launch_jk_1010_np},
                {1, 1, 0, 0, launch_jk_1100_np},
                {1, 1, 1, 0, launch_jk_1110_np},
                {1, 1, 1, 1, launch_jk_1111_np},
                {2, 0, 0, 0, launch_jk_2000_np},
                {2, 0, 1, 0, launch_jk_2010_np},
                {2, 0, 1, 1, launch_jk_2011_np},
                {2, 0, 2, 0, launch_jk_2020_np},
                {2, 1, 0, 0, launch_jk_2100_np},
                {2, 1, 1, 0, launch_jk_2110_np},
                {2, 1, 1, 1, launch_jk_2111_np},
                {2, 1, 2, 0, launch_jk_2120_np},
                {2, 1, 2, 1, launch_jk_2121_np},
                {2, 2, 0, 0, launch_jk_2200_np},
                {2, 2, 1, 0, launch_jk_2210_np},
                {2, 2, 1, 1, launch_jk_2211_np},
                {2, 2, 2, 0, launch_jk_2220_np},
                {2, 2, 2, 1, launch_jk_2221_np},
                {2, 2, 2, 2, launch_jk_2222_np},
                {3, 0, 0, 0, launch_jk_3000_np},
                {3, 0, 1, 0, launch_jk_3010_np},
                {3, 0, 1, 1, launch_jk_3011_np},
                {3, 0, 2, 0, launch_jk_3020_np},
                {3, 0, 2, 1, launch_jk_3021_np},
                {3, 0, 2, 2, launch_jk_3022_np},
                {3, 0, 3, 0, launch_jk_3030_np},
                {3, 1, 0, 0, launch_jk_3100_np},
                {3, 1, 1, 0, launch_jk_3110_np},
                {3, 1, 1, 1, launch_jk_3111_np},
                {3, 1, 2, 0, launch_jk_3120_np},
                {3, 1, 2, 1, launch_jk_3121_np},
                {3, 1, 2, 2, launch_jk_3122_np},
                {3, 1, 3, 0, launch_jk_3130_np},
                {3, 1, 3, 1, launch_jk_3131_np},
                {3, 2, 0, 0, launch_jk_3200_np},
                {3, 2, 1, 0, launch_jk_3210_np},
                {3, 2, 1, 1, launch_jk_3211_np},
                {3, 2, 2, 0, launch_jk_3220_np},
                {3, 2, 2, 1, launch_jk_3221_np},
                {3, 2, 2, 2, launch_jk_3222_np},
                {3, 2, 3, 0, launch_jk_3230_np},
                {3, 2, 3, 1, launch_jk_3231_np},
                {3, 2, 3, 2, launch_jk_3232_np},
                {3, 3, 0, 0, launch_jk_3300_np},
                {3, 3, 1, 0, launch_jk_3310_np},
                {3, 3, 1, 1, launch_jk_3311_np},
                {3, 3, 2, 0, launch_jk_3320_np},
                {3, 3, 2, 1, launch_jk_3321_np},
                {3, 3, 2, 2, launch_jk_3322_np},
                {3, 3, 3, 0, launch_jk_3330_np},
                {3, 3, 3, 1, launch_jk_3331_np},
                {3, 3, 3, 2, launch_jk_3332_np},
                {3, 3, 3, 3, launch_jk_3333_np}};
        for (const Entry &e : table)
                if (e.la == la && e.lb == lb && e.lc == lc && e.ld == ld) return e.fn();
        return 0;
}

static int dispatch_jk(b200jk_plan *P, int la, int lb, int lc, int ld, const JKArgs &a, int fp32, cudaStream_t s,
                       const JKArgs *margs = nullptr, const long long *mchunk = nullptr, int nmol = 0, int variant = 0)
{
        struct Entry { int la, lb, lc, ld; jk_launcher_t fn; };
        static const Entry table[] = {
                {0, 0, 0, 0, launch_jk_0000},
                {1, 0, 0, 0, launch_jk_1000},
                {1, 0, 1, 0, launch_jk_1010},
                {1, 1, 0, 0, launch_jk_1100},
                {1, 1, 1, 0, launch_jk_1110},
                {1, 1, 1, 1, launch_jk_1111},
                {2, 0, 0, 0, launch_jk_2000},
                {2, 0, 1, 0, launch_jk_2010},
                {2, 0, 1, 1, launch_jk_2011},
                {2, 0, 2, 0, launch_jk_2020},
                {2, 1, 0, 0, launch_jk_2100},
                {2, 1, 1, 0, launch_jk_2110},
                {2, 1, 1, 1, launch_jk_2111},
                {2, 1, 2, 0, launch_jk_2120},
                {2, 1, 2, 1, launch_jk_2121},
                {2, 2, 0, 0, launch_jk_2200},
                {2, 2, 1, 0, launch_jk_2210},
                {2, 2, 1, 1, launch_jk_2211},
                {2, 2, 2, 0, launch_jk_2220},
                {2, 2, 2, 1, launch_jk_2221},
                {2, 2, 2, 2, launch_jk_2222},
                {3, 0, 0, 0, launch_jk_3000},
                {3, 0, 1, 0, launch_jk_3010},
                {3, 0, 1, 1, launch_jk_3011},
                {3, 0, 2, 0, launch_jk_3020},
                {3, 0, 2, 1, launch_jk_3021},
                {3, 0, 2, 2, launch_jk_3022},
                {3, 0, 3, 0, launch_jk_3030},
                {3, 1, 0, 0, launch_jk_3100},
                {3, 1, 1, 0, launch_jk_3110},
                {3, 1, 1, 1, launch_jk_3111},
                {3, 1, 2, 0, launch_jk_3120},
                {3, 1, 2, 1, launch_jk_3121},
                {3, 1, 2, 2, launch_jk_3122},
                {3, 1, 3, 0, launch_jk_3130},
                {3, 1, 3, 1, launch_jk_3131},
                {3, 2, 0, 0, launch_jk_3200},
                {3, 2, 1, 0, launch_jk_3210},
                {3, 2, 1, 1, launch_jk_3211},
                {3, 2, 2, 0, launch_jk_3220},
                {3, 2, 2, 1, launch_jk_3221},
                {3, 2, 2, 2, launch_jk_3222},
                {3, 2, 3, 0, launch_jk_3230},
                {3, 2, 3, 1, launch_jk_3231},
                {3, 2, 3, 2, launch_jk_3232},
                {3, 3, 0, 0, launch_jk_3300},
                {3, 3, 1, 0, launch_jk_3310},
                {3, 3, 1, 1, launch_jk_3311},
                {3, 3, 2, 0, launch_jk_3320},
                {3, 3, 2, 1, launch_jk_3321},
                {3, 3, 2, 2, launch_jk_3322},
                {3, 3, 3, 0, launch_jk_3330},
                {3, 3, 3, 1, launch_jk_3331},
                {3, 3, 3, 2, launch_jk_3332},
                {3, 3, 3, 3, launch_jk_3333},
        };
        for (const Entry &e : table) {
                if (e.la == la && e.lb == lb && e.lc == lc && e.ld == ld) {
                        std::string err;
                        if (e.fn(a, s, P->nsm, fp32, variant, margs, mchunk, nmol, err)) return fail(B200JK_ECUDA, err);
                        return B200JK_OK;
                }
        }
        return fail(B200JK_EUNSUPPORTED, "quartet class outside l <= 3");
}

// packed 2D-integral offsets for every Cartesian component of a class
static void class_goff(int la, int lb, int lc, int ld, std::vector<int> &out)
{
        const int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
        auto hidx = [&](int a, int b, int c, int d) { return ((a * (lb + 1) + b) * (lc + 1) + c) * (ld + 1) + d; };
        for (int a = 0; a < na; a++)
                for (int b = 0; b < nb; b++)
                        for (int c = 0; c < nc; c++)
                                for (int d = 0; d < nd; d++) {
                                        const int ox = hidx(cart_lx(la, a), cart_lx(lb, b), cart_lx(lc, c), cart_lx(ld, d));
                                        const int oy = hidx(cart_ly(la, a), cart_ly(lb, b), cart_ly(lc, c), cart_ly(ld, d));
                                        const int oz = hidx(cart_lz(la, a), cart_lz(lb, b), cart_lz(lc, c), cart_lz(ld, d));
                                        out.push_back(ox | (oy << 10) | (oz << 20));
                                }
}

static std::once_flag g_table_once[64];
static int g_table_status[64];

static int ensure_tables(int device)
{
        if (device < 0 || device >= 64) return fail(B200JK_EINVAL, "device index out of range");
        std::call_once(g_table_once[device], [device]() {
                std::vector<double> padded(rys_padded_size());
                rys_pad_table(rys_table_data, padded.data());
                g_table_status[device] =
                        (cudaMemcpyToSymbol(d_rys_table, padded.data(), sizeof(double) * padded.size()) == cudaSuccess &&
                         cudaMemcpyToSymbol(d_rys_table_f, rys_table_f_data, sizeof(float) * RYS_F_SIZE) == cudaSuccess)
                                ? 0 : 1;
        });
        if (g_table_status[device]) return fail(B200JK_ECUDA, "could not upload the Rys tables");
        return B200JK_OK;
}

// eight independent FMA chains per thread; the result is stored so the
// chains cannot be removed
__global__ void fp64_fma_kernel(double *sink, int iters, double m)
{
        double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-9, a2 = a0 + 2e-9, a3 = a0 + 3e-9;
        double a4 = a0 + 4e-9, a5 = a0 + 5e-9, a6 = a0 + 6e-9, a7 = a0 + 7e-9;
        const double c = 1e-12;
        for (int i = 0; i < iters; i++) {
                a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
                a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
        }
        sink[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}

static const double *table_ptr()
{
        void *p = nullptr;
        cudaGetSymbolAddress(&p, d_rys_table);
        return (const double *)p;
}

static const float *table_f_ptr()
{
        void *p = nullptr;
        cudaGetSymbolAddress(&p, d_rys_table_f);
        return (const float *)p;
}

// ---------------------------------------------------------------------------
// C ABI

extern "C" {

int b200jk_version(void) { return (0 << 16) | 1; }

const char *b200jk_last_error(void) { return g_last_error.c_str(); }

int b200jk_device_count(int *count)
{
        if (!count) return fail(B200JK_EINVAL, "count is NULL");
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess) n = 0;
        *count = n;
        return B200JK_OK;
}

int b200jk_plan_dims(const b200jk_plan *plan, int *nao, int *nbas)
{
        if (!plan) return fail(B200JK_EINVAL, "plan is NULL");
        if (nao) *nao = plan->nao;
        if (nbas) *nbas = plan->nbas;
        return B200JK_OK;
}

int b200jk_plan_destroy(b200jk_plan *plan)
{
        if (!plan) return B200JK_OK;
        cudaSetDevice(plan->device);
        delete plan;
        return B200JK_OK;
}

static int build_segments(b200jk_plan *P, const int32_t *atm, int natm, const int32_t *bas, int nbas,
                          const double *env, int env_len, std::vector<Seg> &segs)
{
        P->ao_loc.assign(nbas + 1, 0);
        P->shell_atom.assign(nbas, 0);
        int cart_off = 0;
        for (int I = 0; I < nbas; I++) {
                const int32_t *b = bas + (size_t)I * BAS_SLOTS;
                const int ia = b[ATOM_OF], l = b[ANG_OF], np = b[NPRIM_OF], nc = b[NCTR_OF];
                if (ia < 0 || ia >= natm) return fail(B200JK_EINVAL, "bas: atom index out of range");
                P->shell_atom[I] = ia;
                if (l < 0) return fail(B200JK_EINVAL, "bas: negative angular momentum");
                if (l > LMAX) return fail(B200JK_EUNSUPPORTED, "angular momentum above f (l > 3) is not implemented");
                if (np <= 0 || nc <= 0) return fail(B200JK_EINVAL, "bas: empty shell");
                if (b[PTR_EXP] < 0 || b[PTR_EXP] + np > env_len || b[PTR_COEFF] < 0 || b[PTR_COEFF] + np * nc > env_len)
                        return fail(B200JK_EINVAL, "bas: exponent/coefficient pointer outside env");
                const int pc = atm[(size_t)ia * ATM_SLOTS + PTR_COORD];
                if (pc < 0 || pc + 3 > env_len) return fail(B200JK_EINVAL, "atm: coordinate pointer outside env");
                const int nf = P->cart ? ncart(l) : 2 * l + 1;
                P->ao_loc[I + 1] = P->ao_loc[I] + nf * nc;
                for (int c = 0; c < nc; c++) {
                        Seg s;
                        s.parent = I; s.l = l; s.nprim = np; s.ctr = c;
                        s.exp = env + b[PTR_EXP];
                        s.coef.assign(env + b[PTR_COEFF] + c * np, env + b[PTR_COEFF] + (c + 1) * np);
                        for (int x = 0; x < 3; x++) s.R[x] = env[pc + x];
                        s.out_off = P->ao_loc[I] + c * nf;
                        s.cart_off = cart_off;
                        cart_off += ncart(l);
                        segs.push_back(std::move(s));
                }
        }
        P->nao = P->ao_loc[nbas];
        P->naoc = cart_off;
        P->nseg = (int)segs.size();
        return B200JK_OK;
}

struct HostPair {
        int i, j;              // segments, l_i >= l_j
        int prim0, nprim;
        double q;
        double qs = 0;         // prefix-search key (maximum of q over its band)
        int band = 0;
};

int b200jk_plan_create(const int32_t *atm, int natm, const int32_t *bas, int nbas,
                       const double *env, int env_len, int cart, double direct_scf_tol,
                       int device, b200jk_plan **out)
{
        if (!out) return fail(B200JK_EINVAL, "out is NULL");
        *out = nullptr;
        if (!atm || !bas || !env || natm <= 0 || nbas <= 0 || env_len <= PTR_RANGE_OMEGA)
                return fail(B200JK_EINVAL, "empty or NULL molecule arrays");
        // env[PTR_RANGE_OMEGA] > 0: the long-range operator erf(omega r12)/r12,
        // as libcint evaluates it under mol.with_range_coulomb(omega); < 0
        // (short range, erfc) is built by callers as full minus long range
        const double omega = env[PTR_RANGE_OMEGA];
        if (!(omega == omega)) return fail(B200JK_EINVAL, "env[PTR_RANGE_OMEGA] is NaN");
        if (omega < 0.0)
                return fail(B200JK_EUNSUPPORTED, "short-range Coulomb (env[PTR_RANGE_OMEGA] < 0) is not a plan of its own: "
                                                 "subtract the long-range build (omega = |omega|) from the full one");
        b200jk_plan *P = new b200jk_plan();
        P->device = device;
        P->omega2 = omega > 0 ? omega * omega : 0.0;
        P->cart = cart ? 1 : 0;
        P->natm = natm;
        P->nbas = nbas;
        P->tol = direct_scf_tol > 0 ? direct_scf_tol : 0.0;
        auto bail = [&](int code) { delete P; return code; };
        // the molecule arrays are checked on the host before any device work:
        // indices, pointers into env, l <= 3 (the plan object holds no device
        // memory yet, so bailing out here touches no GPU)
        std::vector<Seg> segs;
        int rc = build_segments(P, atm, natm, bas, nbas, env, env_len, segs);
        if (rc) return bail(rc);
        // nuclei (libcint's int1e_nuc reads the same slots, pyscf/gto/mole.py:58-94)
        for (int ia = 0; ia < natm; ia++) {
                const int32_t *ar = atm + (size_t)ia * ATM_SLOTS;
                const int pc = ar[PTR_COORD], model = ar[2];   // NUC_MOD_OF
                if (pc < 0 || pc + 3 > env_len) return bail(fail(B200JK_EINVAL, "atm: coordinate pointer outside env"));
                double z = (double)ar[CHARGE_OF];
                if (model == 3) {   // NUC_FRAC_CHARGE: the charge is env[atm[PTR_FRAC_CHARGE]]
                        const int pz = ar[4];
                        if (pz < 0 || pz >= env_len) return bail(fail(B200JK_EINVAL, "atm: fractional-charge pointer outside env"));
                        z = env[pz];
                } else if (model != 0 && model != 1) {
                        P->nuc_model_ok = false;   // NUC_GAUSS or NUC_ECP
                }
                P->h_atoms.push_back(make_double4(env[pc], env[pc + 1], env[pc + 2], z));
        }
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
                cudaGetLastError();
                return bail(fail(B200JK_ECUDA, "no CUDA device is available"));
        }
        if (device < 0 || device >= ndev) return bail(fail(B200JK_EINVAL, "device index out of range"));
        if (cudaSetDevice(device) != cudaSuccess) return bail(fail(B200JK_ECUDA, "cudaSetDevice failed"));
        if ((rc = ensure_tables(device))) return bail(rc);
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return bail(fail(B200JK_ECUDA, "cudaGetDeviceProperties failed"));
        P->nsm = prop.multiProcessorCount;
        if (cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&P->ev0) != cudaSuccess || cudaEventCreate(&P->ev1) != cudaSuccess)
                return bail(fail(B200JK_ECUDA, "stream/event creation failed"));

        // segment info and basis maps
        std::vector<int4> seg_info(segs.size());
        std::vector<int> out_seg(P->nao), out_comp(P->nao), cart_seg(P->naoc), cart_comp(P->naoc);
        for (size_t s = 0; s < segs.size(); s++) {
                const Seg &g = segs[s];
                seg_info[s] = make_int4(g.l, g.out_off, g.cart_off, g.parent);
                const int nf = P->cart ? ncart(g.l) : 2 * g.l + 1;
                for (int k = 0; k < nf; k++) { out_seg[g.out_off + k] = (int)s; out_comp[g.out_off + k] = k; }
                for (int k = 0; k < ncart(g.l); k++) { cart_seg[g.cart_off + k] = (int)s; cart_comp[g.cart_off + k] = k; }
        }
        if ((rc = dev_upload(P->seg_info, seg_info)) || (rc = dev_upload(P->out_seg, out_seg)) ||
            (rc = dev_upload(P->out_comp, out_comp)) || (rc = dev_upload(P->cart_seg, cart_seg)) ||
            (rc = dev_upload(P->cart_comp, cart_comp)) || (rc = dev_upload(P->ao_loc_d, P->ao_loc)) ||
            (rc = dev_upload(P->c2s, build_c2s(P->cart))))
                return bail(rc);

        // shell pairs and primitive pairs
        std::vector<HostPair> pairs[NPAIRCLASS];
        std::vector<double4> hPP;
        std::vector<double2> hPK, hPE;
        const double expcut = 60.0;
        for (int si = 0; si < (int)segs.size(); si++) {
                for (int sj = 0; sj <= si; sj++) {
                        int i = si, j = sj;
                        if (segs[j].l > segs[i].l) std::swap(i, j);
                        const Seg &A = segs[i], &B = segs[j];
                        double AB[3], rr = 0;
                        for (int x = 0; x < 3; x++) { AB[x] = A.R[x] - B.R[x]; rr += AB[x] * AB[x]; }
                        HostPair hp;
                        hp.i = i; hp.j = j; hp.prim0 = (int)hPP.size(); hp.nprim = 0; hp.q = 0;
                        for (int pa = 0; pa < A.nprim; pa++) {
                                for (int pb = 0; pb < B.nprim; pb++) {
                                        const double a = A.exp[pa], b = B.exp[pb], p = a + b;
                                        const double mu = a * b / p;
                                        if (mu * rr > expcut) continue;
                                        const double cc = A.coef[pa] * B.coef[pb];
                                        if (cc == 0.0) continue;
                                        double4 P4;
                                        P4.x = (a * A.R[0] + b * B.R[0]) / p;
                                        P4.y = (a * A.R[1] + b * B.R[1]) / p;
                                        P4.z = (a * A.R[2] + b * B.R[2]) / p;
                                        P4.w = p;
                                        hPP.push_back(P4);
                                        hPK.push_back(make_double2(cc * exp(-mu * rr), 0.5 / p));
                                        hPE.push_back(make_double2(a, b));
                                        hp.nprim++;
                                }
                        }
                        if (hp.nprim == 0) continue;
                        pairs[pair_class(A.l, B.l)].push_back(hp);
                }
        }
        P->prim_pairs = (int64_t)hPP.size();
        if ((rc = dev_upload(P->PP, hPP)) || (rc = dev_upload(P->PK, hPK)) || (rc = dev_upload(P->PE, hPE)))
                return bail(rc);
        // the gradient set-up re-screens the unpruned pairs with its own bounds
        P->segl.resize(segs.size());
        for (size_t t = 0; t < segs.size(); t++) {
                P->segl[t].parent = segs[t].parent;
                P->segl[t].l = segs[t].l;
                P->segl[t].cart_off = segs[t].cart_off;
                for (int x = 0; x < 3; x++) P->segl[t].R[x] = segs[t].R[x];
        }
        for (int X = 0; X < NPAIRCLASS; X++) {
                P->all_pairs[X].clear();
                for (const HostPair &h : pairs[X]) P->all_pairs[X].push_back({h.i, h.j, h.prim0, h.nprim});
        }

        // Cartesian offset tables of all quartet classes (also used by q_cond)
        {
                std::vector<int> all;
                auto qcs = quartet_classes();
                P->goff_at.assign(qcs.size(), 0);
                for (size_t t = 0; t < qcs.size(); t++) {
                        int la, lb, lc, ld;
                        class_l(qcs[t].X, la, lb);
                        class_l(qcs[t].Y, lc, ld);
                        P->goff_at[t] = all.size();
                        class_goff(la, lb, lc, ld, all);
                }
                if ((rc = dev_upload(P->goff_all, all))) return bail(rc);
        }

        // upload unsorted pairs, compute q_cond on the GPU
        auto upload_class = [&](int X, const std::vector<HostPair> &hv) -> int {
                PairClassDev &c = P->pc[X];
                class_l(X, c.la, c.lb);
                c.n = (int)hv.size();
                for (int b = 0; b <= B2_NBUCKET; b++) c.boff[b] = 0;
                for (const HostPair &p : hv) c.boff[prim_bucket(p.nprim) + 1]++;
                for (int b = 0; b < B2_NBUCKET; b++) c.boff[b + 1] += c.boff[b];
                std::vector<int4> sh(hv.size());
                std::vector<int2> pr(hv.size());
                std::vector<double> q(hv.size()), qs(hv.size());
                std::vector<double4> Av(hv.size()), ABv(hv.size());
                for (size_t t = 0; t < hv.size(); t++) {
                        const Seg &A = segs[hv[t].i], &B = segs[hv[t].j];
                        sh[t] = make_int4(A.cart_off, B.cart_off, A.parent, B.parent);
                        pr[t] = make_int2(hv[t].prim0, hv[t].nprim);
                        q[t] = hv[t].q;
                        qs[t] = hv[t].qs;
                        Av[t] = make_double4(A.R[0], A.R[1], A.R[2], hv[t].i == hv[t].j ? 1.0 : 0.0);
                        ABv[t] = make_double4(A.R[0] - B.R[0], A.R[1] - B.R[1], A.R[2] - B.R[2], 0.0);
                }
                int r;
                if ((r = dev_upload(c.sh, sh)) || (r = dev_upload(c.pr, pr)) || (r = dev_upload(c.q, q)) ||
                    (r = dev_upload(c.qs, qs)) || (r = dev_upload(c.A, Av)) || (r = dev_upload(c.AB, ABv)))
                        return r;
                return B200JK_OK;
        };
        for (int X = 0; X < NPAIRCLASS; X++)
                if ((rc = upload_class(X, pairs[X]))) return bail(rc);

        std::vector<double> h_q((size_t)nbas * nbas, 1e-100);
        if ((rc = dev_upload(P->qcond, h_q))) return bail(rc);
        {
                auto qcs = quartet_classes();
                for (int X = 0; X < NPAIRCLASS; X++) {
                        QArgs qa;
                        qa.omega2 = P->omega2;
                        qa.pairs = P->pc[X].view();
                        qa.PP = P->PP.p; qa.PK = P->PK.p;
                        qa.table = table_ptr();
                        size_t gi = 0;
                        for (size_t t = 0; t < qcs.size(); t++) if (qcs[t].X == X && qcs[t].Y == X) gi = t;
                        qa.goff = P->goff_all.p + P->goff_at[gi];
                        qa.c2s = P->c2s.p;
                        qa.qcond = (unsigned long long *)P->qcond.p;
                        qa.nbas = nbas;
                        qa.cart = P->cart;
                        {
                                std::string err;
                                if (launch_qcond(P->pc[X].la, P->pc[X].lb, qa, P->stream, err)) return bail(fail(B200JK_ECUDA, err));
                        }
                }
                if (cudaStreamSynchronize(P->stream) != cudaSuccess)
                        return bail(fail(B200JK_ECUDA, std::string("q_cond kernels: ") + cudaGetErrorString(cudaGetLastError())));
                if (cudaMemcpy(h_q.data(), P->qcond.p, sizeof(double) * h_q.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
                        return bail(fail(B200JK_ECUDA, "q_cond download failed"));
        }
        P->h_qcond = h_q;

        // keep pairs that can pass q_ij q_kl > tol for some kl; sort by q
        double qmax = 0;
        for (double v : h_q) qmax = std::max(qmax, v);
        P->shell_pairs = 0;
        for (int X = 0; X < NPAIRCLASS; X++) {
                std::vector<HostPair> &hv = pairs[X];
                for (auto &p : hv) p.q = h_q[(size_t)segs[p.i].parent * nbas + segs[p.j].parent];
                if (P->tol > 0) {
                        hv.erase(std::remove_if(hv.begin(), hv.end(),
                                                [&](const HostPair &p) { return !(p.q * qmax > P->tol); }),
                                 hv.end());
                }
                // Order inside a bucket: bands of the bound (factor 2, largest
                // first), inside a band by first then second segment.  The
                // prefix screen searches the band maxima qs (a superset of the
                // passing kets; the exact test is per quartet).  Consecutive
                // kets then mostly share their first segment, which the
                // register family uses to carry K[., c] sums across the kets
                // of a lane.
                const double qcls = std::accumulate(hv.begin(), hv.end(), 0.0,
                                                    [](double m, const HostPair &p) { return std::max(m, p.q); });
                for (auto &p : hv)
                        p.band = (p.q > 0 && qcls > 0) ? std::min(2000, (int)std::floor(std::log2(qcls / p.q))) : 2000;
                std::stable_sort(hv.begin(), hv.end(), [&](const HostPair &a, const HostPair &b) {
                        const int ba = prim_bucket(a.nprim), bb = prim_bucket(b.nprim);
                        if (ba != bb) return ba < bb;
                        if (a.band != b.band) return a.band < b.band;
                        if (segs[a.i].cart_off != segs[b.i].cart_off) return segs[a.i].cart_off < segs[b.i].cart_off;
                        return segs[a.j].cart_off < segs[b.j].cart_off;
                });
                for (size_t t = 0; t < hv.size();) {
                        size_t e = t;
                        double m = 0;
                        while (e < hv.size() && prim_bucket(hv[e].nprim) == prim_bucket(hv[t].nprim) &&
                               hv[e].band == hv[t].band)
                                m = std::max(m, hv[e++].q);
                        for (size_t u = t; u < e; u++) hv[u].qs = m;
                        t = e;
                }
                P->shell_pairs += (int64_t)hv.size();
                if ((rc = upload_class(X, hv))) return bail(rc);
        }
        {
                std::vector<long long> src;
                P->pk_off.assign(NPAIRCLASS + 1, 0);
                for (int X = 0; X < NPAIRCLASS; X++) {
                        P->pk_off[X] = (long long)src.size();
                        for (const HostPair &hp : pairs[X]) {
                                const Seg &A = segs[hp.i], &B = segs[hp.j];
                                const int na = ncart(A.l), nb = ncart(B.l);
                                for (int x = 0; x < na; x++)
                                        for (int y = 0; y < nb; y++)
                                                src.push_back((long long)(A.cart_off + x) * P->naoc + B.cart_off + y);
                        }
                }
                P->pk_off[NPAIRCLASS] = (long long)src.size();
                P->pk_total = (long long)src.size();
                if ((rc = dev_upload(P->pk_src, src))) return bail(rc);
        }
        memset(&P->st, 0, sizeof(P->st));
        P->st.nao = P->nao; P->st.nao_cart = P->naoc; P->st.nbas = nbas; P->st.nseg = P->nseg;
        P->st.shell_pairs = P->shell_pairs; P->st.prim_pairs = P->prim_pairs;
        P->h_atm.assign(atm, atm + (size_t)natm * ATM_SLOTS);
        P->h_bas.assign(bas, bas + (size_t)nbas * BAS_SLOTS);
        *out = P;
        return B200JK_OK;
}

int b200jk_plan_update_coords(b200jk_plan *P, const double *env, int env_len)
{
        if (!P) return fail(B200JK_EINVAL, "plan is NULL");
        // the geometry-dependent tables are planned afresh for the new env
        // (same atoms and basis), then moved into this plan; its workspaces,
        // stream, tuning, shard, screen and threshold stay
        b200jk_plan *T = nullptr;
        int rc = b200jk_plan_create(P->h_atm.data(), P->natm, P->h_bas.data(), P->nbas, env, env_len, P->cart,
                                    P->tol > 0 ? P->tol : 0.0, P->device, &T);
        if (rc) return rc;
        if (T->nao != P->nao || T->naoc != P->naoc || T->nseg != P->nseg) {
                b200jk_plan_destroy(T);
                return fail(B200JK_EINVAL, "the new env changes the basis dimensions");
        }
        std::swap(P->PP, T->PP);
        std::swap(P->PK, T->PK);
        std::swap(P->PE, T->PE);
        std::swap(P->segl, T->segl);
        for (int X = 0; X < NPAIRCLASS; X++) {
                std::swap(P->pc[X], T->pc[X]);
                std::swap(P->all_pairs[X], T->all_pairs[X]);
        }
        std::swap(P->qcond, T->qcond);
        std::swap(P->h_qcond, T->h_qcond);
        std::swap(P->pk_off, T->pk_off);
        std::swap(P->pk_total, T->pk_total);
        std::swap(P->pk_src, T->pk_src);
        std::swap(P->grad, T->grad);   // derivative bounds belong to the old geometry
        std::swap(P->h_atoms, T->h_atoms);
        P->nuc_model_ok = T->nuc_model_ok;
        P->i1_npair = -1;              // the one-electron pair list is planned again on next use
        P->release_fill();             // so are the integral fill's pair lists
        P->shell_pairs = T->shell_pairs;
        P->prim_pairs = T->prim_pairs;
        P->st = T->st;
        // captured batched builds hold the old tables' addresses
        P->ws_gen++;
        b200jk_plan_destroy(T);
        return B200JK_OK;
}

// the one-electron pair list: every segment pair with a primitive pair (no
// Schwarz screening), element offsets, segments and atoms on the device
static int ensure_i1(b200jk_plan *P)
{
        if (P->i1_npair >= 0) return B200JK_OK;
        const size_t nc = (size_t)P->naoc * P->naoc, nn = (size_t)P->nao * P->nao;
        int rc;
        std::vector<int4> hp;
        std::vector<long long> off(1, 0);
        for (int X = 0; X < NPAIRCLASS; X++)
                for (const PairLite &q : P->all_pairs[X]) {
                        hp.push_back(make_int4(q.i, q.j, q.prim0, q.nprim));
                        off.push_back(off.back() + (long long)ncart(P->segl[q.i].l) * ncart(P->segl[q.j].l));
                }
        std::vector<double4> hs(P->segl.size());
        std::vector<int> hc(P->segl.size()), ha(P->segl.size());
        for (size_t t = 0; t < P->segl.size(); t++) {
                hs[t] = make_double4(P->segl[t].R[0], P->segl[t].R[1], P->segl[t].R[2], (double)P->segl[t].l);
                hc[t] = P->segl[t].cart_off;
                ha[t] = P->shell_atom[P->segl[t].parent];
        }
        if ((rc = dev_upload(P->i1_pair, hp)) || (rc = dev_upload(P->i1_off, off)) || (rc = dev_upload(P->i1_seg, hs)) ||
            (rc = dev_upload(P->i1_seg_cart, hc)) || (rc = dev_upload(P->i1_seg_atom, ha)) ||
            (rc = dev_upload(P->i1_atoms, P->h_atoms)) ||
            (rc = dev_alloc(P->i1_S, nc)) || (rc = dev_alloc(P->i1_H, nc)) || (rc = dev_alloc(P->i1_zero, nc)) ||
            (rc = dev_alloc(P->i1_out, 2 * nn)))
                return rc;
        CUDA_TRY(cudaMemset(P->i1_zero.p, 0, sizeof(double) * nc));
        P->i1_npair = (int)hp.size();
        return B200JK_OK;
}

int b200jk_int1e(b200jk_plan *P, double *ovlp, double *hcore, int dev_ptrs, void *stream)
{
        if (!P) return fail(B200JK_EINVAL, "plan is NULL");
        if (!ovlp && !hcore) return fail(B200JK_EINVAL, "no output requested");
        if (hcore && !P->nuc_model_ok)
                return fail(B200JK_EUNSUPPORTED, "finite-nucleus models and ECP atoms are not implemented in the "
                                                 "nuclear-attraction integrals");
        CUDA_TRY(cudaSetDevice(P->device));
        int rc;
        if (dev_ptrs && ((ovlp && (rc = check_dev_ptr(ovlp, P->device, "ovlp"))) ||
                         (hcore && (rc = check_dev_ptr(hcore, P->device, "hcore")))))
                return rc;
        const size_t nc = (size_t)P->naoc * P->naoc, nn = (size_t)P->nao * P->nao;
        if ((rc = ensure_i1(P))) return rc;
        cudaStream_t s = stream ? (cudaStream_t)stream : P->stream;
        CUDA_TRY(cudaMemsetAsync(P->i1_S.p, 0, sizeof(double) * nc, s));
        CUDA_TRY(cudaMemsetAsync(P->i1_H.p, 0, sizeof(double) * nc, s));
        long long nelem = 0;
        CUDA_TRY(cudaMemcpy(&nelem, P->i1_off.p + P->i1_npair, sizeof(long long), cudaMemcpyDeviceToHost));
        if (nelem > 0) {
                Int1eArgs a;
                a.pair = P->i1_pair.p; a.elem_off = P->i1_off.p; a.npair = P->i1_npair;
                a.seg = P->i1_seg.p; a.seg_cart = P->i1_seg_cart.p;
                a.PP = P->PP.p; a.PK = P->PK.p; a.PE = P->PE.p;
                a.atoms = P->i1_atoms.p; a.natm = (int)P->h_atoms.size(); a.naoc = P->naoc;
                a.table = table_ptr();
                a.S = P->i1_S.p; a.H = P->i1_H.p;
                int1e_kernel<<<grid_for(nelem, 128), 128, 0, s>>>(a);
                CUDA_TRY(cudaGetLastError());
        }
        double *os = dev_ptrs ? ovlp : P->i1_out.p, *oh = dev_ptrs ? hcore : P->i1_out.p + nn;
        if (ovlp) {
                cart_to_out_kernel<<<grid_for((long long)nn, 256), 256, 0, s>>>(P->i1_S.p, P->i1_zero.p, P->nao, P->naoc,
                                                                               P->out_seg.p, P->out_comp.p, P->seg_info.p,
                                                                               P->c2s.p, P->cart, 1, os);
                CUDA_TRY(cudaGetLastError());
        }
        if (hcore) {
                cart_to_out_kernel<<<grid_for((long long)nn, 256), 256, 0, s>>>(P->i1_H.p, P->i1_zero.p, P->nao, P->naoc,
                                                                               P->out_seg.p, P->out_comp.p, P->seg_info.p,
                                                                               P->c2s.p, P->cart, 1, oh);
                CUDA_TRY(cudaGetLastError());
        }
        if (!dev_ptrs) {
                if (ovlp) CUDA_TRY(cudaMemcpyAsync(ovlp, os, sizeof(double) * nn, cudaMemcpyDeviceToHost, s));
                if (hcore) CUDA_TRY(cudaMemcpyAsync(hcore, oh, sizeof(double) * nn, cudaMemcpyDeviceToHost, s));
        }
        CUDA_TRY(cudaStreamSynchronize(s));
        return B200JK_OK;
}

int b200jk_grad_int1e(b200jk_plan *P, const double *dm, const double *dme, double *de, int dev_ptrs, void *stream)
{
        if (!P) return fail(B200JK_EINVAL, "plan is NULL");
        if (!dm || !dme || !de) return fail(B200JK_EINVAL, "NULL argument");
        if (!P->nuc_model_ok)
                return fail(B200JK_EUNSUPPORTED, "finite-nucleus models and ECP atoms are not implemented in the "
                                                 "nuclear-attraction integrals");
        CUDA_TRY(cudaSetDevice(P->device));
        int rc;
        if (dev_ptrs && ((rc = check_dev_ptr(dm, P->device, "dm")) || (rc = check_dev_ptr(dme, P->device, "dme")) ||
                         (rc = check_dev_ptr(de, P->device, "de"))))
                return rc;
        if ((rc = ensure_i1(P))) return rc;
        const size_t nn = (size_t)P->nao * P->nao;
        const int natm = (int)P->h_atoms.size();
        if ((rc = dev_alloc(P->i1_de, 3 * (size_t)natm))) return rc;
        cudaStream_t s = stream ? (cudaStream_t)stream : P->stream;
        // the Cartesian D and W live in the overlap/hcore scratch
        const double *dD = dm, *dW = dme;
        if (!dev_ptrs) {
                CUDA_TRY(cudaMemcpyAsync(P->i1_out.p, dm, sizeof(double) * nn, cudaMemcpyHostToDevice, s));
                CUDA_TRY(cudaMemcpyAsync(P->i1_out.p + nn, dme, sizeof(double) * nn, cudaMemcpyHostToDevice, s));
                dD = P->i1_out.p;
                dW = P->i1_out.p + nn;
        }
        const long long nc = (long long)P->naoc * P->naoc;
        out_to_cart_kernel<<<grid_for(nc, 256), 256, 0, s>>>(dD, P->nao, P->naoc, P->cart_seg.p, P->cart_comp.p,
                                                             P->seg_info.p, P->c2s.p, P->cart, P->i1_S.p, nullptr, nullptr);
        CUDA_TRY(cudaGetLastError());
        out_to_cart_kernel<<<grid_for(nc, 256), 256, 0, s>>>(dW, P->nao, P->naoc, P->cart_seg.p, P->cart_comp.p,
                                                             P->seg_info.p, P->c2s.p, P->cart, P->i1_H.p, nullptr, nullptr);
        CUDA_TRY(cudaGetLastError());
        double *out = dev_ptrs ? de : P->i1_de.p;
        CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double) * 3 * natm, s));
        long long nelem = 0;
        CUDA_TRY(cudaMemcpy(&nelem, P->i1_off.p + P->i1_npair, sizeof(long long), cudaMemcpyDeviceToHost));
        if (nelem > 0) {
                Int1eGradArgs ga;
                Int1eArgs &a = ga.g;
                a.pair = P->i1_pair.p; a.elem_off = P->i1_off.p; a.npair = P->i1_npair;
                a.seg = P->i1_seg.p; a.seg_cart = P->i1_seg_cart.p;
                a.PP = P->PP.p; a.PK = P->PK.p; a.PE = P->PE.p;
                a.atoms = P->i1_atoms.p; a.natm = natm; a.naoc = P->naoc;
                a.table = table_ptr();
                a.S = nullptr; a.H = nullptr;
                ga.seg_atom = P->i1_seg_atom.p;
                ga.D = P->i1_S.p;
                ga.W = P->i1_H.p;
                ga.de = out;
                int1e_grad_kernel<<<grid_for(nelem, 128), 128, 0, s>>>(ga);
                CUDA_TRY(cudaGetLastError());
        }
        if (!dev_ptrs) CUDA_TRY(cudaMemcpyAsync(de, out, sizeof(double) * 3 * natm, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        return B200JK_OK;
}

int b200jk_get_q_cond(const b200jk_plan *plan, double *q_cond)
{
        if (!plan || !q_cond) return fail(B200JK_EINVAL, "NULL argument");
        memcpy(q_cond, plan->h_qcond.data(), sizeof(double) * plan->h_qcond.size());
        return B200JK_OK;
}

// the addresses of a plan's build workspace: a change means that work
// recorded with the old addresses (a captured batched build) is stale
static std::vector<const void *> workspace_key(const b200jk_plan *P)
{
        return {P->D.p, P->Dc.p, P->Ds.p, P->Jacc.p, P->Kacc.p, P->outJ.p, P->outK.p, P->dm_cond.p, P->dmax.p,
                P->stats.p, P->Dpk.p, P->Jpk.p, P->nkl.p, P->kst.p, P->nchunk.p, P->chunk_off.p, P->cub_tmp.p};
}

static int ensure_workspace(b200jk_plan *P, int n_dm)
{
        const size_t nn = (size_t)P->nao * P->nao, nc = (size_t)P->naoc * P->naoc;
        const std::vector<const void *> key0 = workspace_key(P);
        int rc;
        if ((rc = dev_alloc(P->D, nn * n_dm)) || (rc = dev_alloc(P->Dc, nc * n_dm * 2)) ||
            (rc = dev_alloc(P->Ds, nc * n_dm)) || (rc = dev_alloc(P->Jacc, nc * n_dm)) ||
            (rc = dev_alloc(P->Kacc, nc * n_dm * 2)) || (rc = dev_alloc(P->outJ, nn * n_dm)) ||
            (rc = dev_alloc(P->outK, nn * n_dm)) || (rc = dev_alloc(P->dm_cond, (size_t)P->nbas * P->nbas)) ||
            (rc = dev_alloc(P->dmax, 1)) || (rc = dev_alloc(P->stats, 4 * 64)) ||
            (rc = dev_alloc(P->Dpk, (size_t)std::max<long long>(1, P->pk_total) * n_dm)) ||
            (rc = dev_alloc(P->Jpk, (size_t)std::max<long long>(1, P->pk_total) * n_dm)))
                return rc;
        int maxn = 1;
        for (auto &c : P->pc) maxn = std::max(maxn, c.n * B2_NBUCKET);
        if ((rc = dev_alloc(P->nkl, maxn)) || (rc = dev_alloc(P->kst, maxn)) || (rc = dev_alloc(P->nchunk, maxn + 1)) ||
            (rc = dev_alloc(P->chunk_off, maxn + 1)))
                return rc;
        size_t tmp = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tmp, P->nchunk.p, P->chunk_off.p, maxn + 1);
        if ((rc = dev_alloc(P->cub_tmp, tmp + 16))) return rc;
        P->ws_ndm = std::max(P->ws_ndm, n_dm);
        if (workspace_key(P) != key0) P->ws_gen++;
        return B200JK_OK;
}


int b200jk_get_jk(b200jk_plan *P, const double *dms, int n_dm, int hermi, int with_j, int with_k,
                  double *vj, double *vk, int dev_ptrs, int precision_mode, void *stream)
{
        if (!P) return fail(B200JK_EINVAL, "plan is NULL");
        if (!dms || n_dm <= 0) return fail(B200JK_EINVAL, "no density matrices");
        if (hermi < 0 || hermi > 2) return fail(B200JK_EINVAL, "hermi must be 0, 1 or 2");
        if (with_j && !vj) return fail(B200JK_EINVAL, "vj is NULL while with_j is set");
        if (with_k && !vk) return fail(B200JK_EINVAL, "vk is NULL while with_k is set");
        if (precision_mode != B200JK_PREC_FP64 && precision_mode != B200JK_PREC_MIXED)
                return fail(B200JK_EUNSUPPORTED, "precision_mode must be 0 (FP64) or 1 (mixed FP32/FP64)");
        const int mixed = precision_mode == B200JK_PREC_MIXED;
        CUDA_TRY(cudaSetDevice(P->device));
        int rc;
        if (dev_ptrs && ((rc = check_dev_ptr(dms, P->device, "dms")) || (with_j && (rc = check_dev_ptr(vj, P->device, "vj"))) ||
                         (with_k && (rc = check_dev_ptr(vk, P->device, "vk")))))
                return rc;
        if ((rc = ensure_workspace(P, n_dm))) return rc;
        cudaStream_t s = stream ? (cudaStream_t)stream : P->stream;
        const size_t nn = (size_t)P->nao * P->nao, nc = (size_t)P->naoc * P->naoc;
        const int nk = hermi == 1 ? 1 : 2;
        CUDA_TRY(cudaEventRecord(P->ev0, s));
        const double *dD = dms;
        if (!dev_ptrs) {
                CUDA_TRY(cudaMemcpyAsync(P->D.p, dms, sizeof(double) * nn * n_dm, cudaMemcpyHostToDevice, s));
                dD = P->D.p;
        }
        // screening data
        CUDA_TRY(cudaMemsetAsync(P->dmax.p, 0, sizeof(unsigned long long), s));
        CUDA_TRY(cudaMemsetAsync(P->stats.p, 0, 4 * 64 * sizeof(unsigned long long), s));
        {
                const long long npair = (long long)P->nbas * (P->nbas + 1) / 2;
                dm_cond_kernel<<<grid_for(npair, 256), 256, 0, s>>>(dD, n_dm, P->nao, P->ao_loc_d.p, P->nbas,
                                                                  P->dm_cond.p, P->dmax.p);
                CUDA_TRY(cudaGetLastError());
        }
        // densities in the Cartesian basis
        for (int d = 0; d < n_dm; d++) {
                double *Dc = P->Dc.p + (size_t)d * nk * nc;
                out_to_cart_kernel<<<grid_for((long long)nc, 256), 256, 0, s>>>(
                        dD + (size_t)d * nn, P->nao, P->naoc, P->cart_seg.p, P->cart_comp.p, P->seg_info.p,
                        P->c2s.p, P->cart, Dc, nk == 2 ? Dc + nc : nullptr, nullptr);
                CUDA_TRY(cudaGetLastError());
                sym_sum_kernel<<<grid_for((long long)nc, 256), 256, 0, s>>>(Dc, P->naoc, P->Ds.p + (size_t)d * nc);
                CUDA_TRY(cudaGetLastError());
                if (with_j && P->pk_total > 0) {
                        pack_gather_kernel<<<grid_for(P->pk_total, 256), 256, 0, s>>>(
                                P->Ds.p + (size_t)d * nc, P->pk_src.p, P->pk_total, P->Dpk.p + (size_t)d * P->pk_total);
                        CUDA_TRY(cudaGetLastError());
                }
        }
        if (with_j && P->pk_total > 0)
                CUDA_TRY(cudaMemsetAsync(P->Jpk.p, 0, sizeof(double) * P->pk_total * n_dm, s));
        if (with_j) CUDA_TRY(cudaMemsetAsync(P->Jacc.p, 0, sizeof(double) * nc * n_dm, s));
        if (with_k) CUDA_TRY(cudaMemsetAsync(P->Kacc.p, 0, sizeof(double) * nc * n_dm * nk, s));

        const double *tbl = table_ptr();
        const float *tbl_f = table_f_ptr();
        auto qcs = quartet_classes();
        // dm_cond, to-Cartesian + symmetrise (+ J block gather) per density
        int64_t launches = 1 + (2 + (with_j && P->pk_total > 0 ? 1 : 0)) * n_dm;
        if (P->cls.size() != qcs.size()) {
                P->cls.assign(qcs.size(), b200jk_class_stat_t());
                for (size_t t = 0; t < qcs.size(); t++) {
                        int la, lb, lc, ld;
                        class_l(qcs[t].X, la, lb);
                        class_l(qcs[t].Y, lc, ld);
                        P->cls[t].la = la; P->cls[t].lb = lb; P->cls[t].lc = lc; P->cls[t].ld = ld;
                        P->cls[t].family = family_is_thread(la, lb, lc, ld) ? 0 : 1;
                }
        }
        if (P->profiling && P->cls_ev.empty()) {
                P->cls_ev.resize(2 * qcs.size());
                for (auto &e : P->cls_ev) CUDA_TRY(cudaEventCreate(&e));
        }
        std::vector<char> ran(qcs.size(), 0);
        {
                for (size_t t = 0; t < qcs.size(); t++) {
                        const PairClassDev &bra = P->pc[qcs[t].X], &ket = P->pc[qcs[t].Y];
                        if (bra.n == 0 || ket.n == 0) continue;
                        int la = bra.la, lb = bra.lb, lc = ket.la, ld = ket.lb;
                        const int same = qcs[t].X == qcs[t].Y;
                        const int nseg = bra.n * B2_NBUCKET;
                        if (P->profiling) CUDA_TRY(cudaEventRecord(P->cls_ev[2 * t], s));
                        // pass 0: float64 quartets (all of them unless mixed);
                        // pass 1: the float32 quartets of mixed precision
                        const double tau_c = mixed ? class_tau(P, t) : 0.0;
                        for (int pass = 0; pass < (tau_c > 0 ? 2 : 1); pass++) {
                                // tiled chunk order for unsharded plans (with shards the
                                // stride over bra pairs would leave tile slots idle)
                                const int tiled = P->nshard == 1 && P->tile_b > 0;
                                // chunk size of the family the dispatcher will pick; bra
                                // runs (variant 2) need the tiled float64 pass of one
                                // symmetric density, else the class runs variant 0
                                int variant = class_variant(P, t, pass);
                                const int brun = family_bra_run(la, lb, lc, ld);
                                if (variant == 2 && (pass == 1 || !tiled || n_dm != 1 || nk != 1 || brun <= 1 ||
                                                     P->tile_b % brun != 0))
                                        variant = 0;
                                const int chunk = family_chunk(la, lb, lc, ld, variant);
                                count_kernel<<<grid_for(nseg, 256), 256, 0, s>>>(
                                        bra.view(), ket.view(), same, P->tol > 0 ? P->tol : 0.0, (const double *)P->dmax.p,
                                        chunk, tau_c, pass, P->shard, P->nshard, P->nkl.p, P->kst.p,
                                        P->nchunk.p);
                                CUDA_TRY(cudaGetLastError());
                                const int ntb = (bra.n + P->tile_b - 1) / std::max(1, P->tile_b);
                                const int nscan = tiled ? B2_NBUCKET * ntb : nseg;
                                if (tiled) {
                                        const int nslot = variant == 2 ? P->tile_b / brun : P->tile_b;
                                        tile_count_kernel<<<grid_for(nscan, 256), 256, 0, s>>>(P->nkl.p, bra.n, chunk, P->tile_b,
                                                                                             ntb, nslot, P->nchunk.p);
                                        CUDA_TRY(cudaGetLastError());
                                }
                                CUDA_TRY(cudaMemsetAsync(P->nchunk.p + nscan, 0, sizeof(long long), s));
                                size_t tmp = P->cub_tmp.n;
                                CUDA_TRY(cub::DeviceScan::ExclusiveSum(P->cub_tmp.p, tmp, P->nchunk.p, P->chunk_off.p,
                                                                       nscan + 1, s));
                                JKArgs a;
                                a.tiled = tiled;
                                a.tile_b = P->tile_b;
                                a.ntile = nscan;
                                a.ntb = ntb;
                                a.bra = bra.view();
                                a.ket = ket.view();
                                a.PP = P->PP.p; a.PK = P->PK.p;
                                a.chunk_off = P->chunk_off.p;
                                a.nkl = P->nkl.p;
                                a.kst = P->kst.p;
                                a.dm_cond = P->dm_cond.p;
                                a.table = tbl;
                                a.table_f = tbl_f;
                                a.goff = P->goff_all.p + P->goff_at[t];
                                a.Jacc = P->Jacc.p; a.Kacc = P->Kacc.p;
                                a.Ds = P->Ds.p; a.Dk = P->Dc.p;
                                a.Dpk = P->Dpk.p + P->pk_off[qcs[t].Y];
                                a.Jpk = P->Jpk.p + P->pk_off[qcs[t].Y];
                                a.pk_stride = P->pk_total;
                                a.stats = P->stats.p + 2 * (64 * pass + t);
                                a.tol = P->tol > 0 ? P->tol : -1.0;
                                a.nbas = P->nbas; a.naoc = P->naoc; a.n_dm = n_dm; a.nk = nk;
                                a.with_j = with_j; a.with_k = with_k; a.same = same;
                                a.screen = P->screen;
                                a.omega2 = P->omega2;
                                if ((rc = dispatch_jk(P, la, lb, lc, ld, a, pass, s, nullptr, nullptr, 0, variant))) return rc;
                                launches += 2;   // count + class kernel (the scan is a CUB library kernel)
                        }
                        if (P->profiling) CUDA_TRY(cudaEventRecord(P->cls_ev[2 * t + 1], s));
                        ran[t] = 1;
                }
        }
        // ket-side J from the packed blocks, then back to the output basis
        if (with_j && P->pk_total > 0) {
                for (int d = 0; d < n_dm; d++) {
                        pack_scatter_add_kernel<<<grid_for(P->pk_total, 256), 256, 0, s>>>(
                                P->Jpk.p + (size_t)d * P->pk_total, P->pk_src.p, P->pk_total, P->Jacc.p + (size_t)d * nc);
                        CUDA_TRY(cudaGetLastError());
                        launches++;
                }
        }
        for (int d = 0; d < n_dm; d++) {
                if (with_j) {
                        const double *J = P->Jacc.p + (size_t)d * nc;
                        double *o = dev_ptrs ? vj + (size_t)d * nn : P->outJ.p + (size_t)d * nn;
                        cart_to_out_kernel<<<grid_for((long long)nn, 256), 256, 0, s>>>(
                                J, J, P->nao, P->naoc, P->out_seg.p, P->out_comp.p, P->seg_info.p, P->c2s.p,
                                P->cart, 1, o);
                        CUDA_TRY(cudaGetLastError());
                }
                if (with_k) {
                        const double *K1 = P->Kacc.p + (size_t)d * nk * nc;
                        const double *K2 = nk == 2 ? K1 + nc : K1;
                        double *o = dev_ptrs ? vk + (size_t)d * nn : P->outK.p + (size_t)d * nn;
                        cart_to_out_kernel<<<grid_for((long long)nn, 256), 256, 0, s>>>(
                                K1, K2, P->nao, P->naoc, P->out_seg.p, P->out_comp.p, P->seg_info.p, P->c2s.p,
                                P->cart, hermi, o);
                        CUDA_TRY(cudaGetLastError());
                }
        }
        launches += (with_j ? n_dm : 0) + (with_k ? n_dm : 0);
        CUDA_TRY(cudaEventRecord(P->ev1, s));
        if (!dev_ptrs) {
                if (with_j) CUDA_TRY(cudaMemcpyAsync(vj, P->outJ.p, sizeof(double) * nn * n_dm, cudaMemcpyDeviceToHost, s));
                if (with_k) CUDA_TRY(cudaMemcpyAsync(vk, P->outK.p, sizeof(double) * nn * n_dm, cudaMemcpyDeviceToHost, s));
        }
        unsigned long long hs[4 * 64];
        CUDA_TRY(cudaMemcpyAsync(hs, P->stats.p, sizeof(hs), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, P->ev0, P->ev1));
        P->st.quartets = 0;
        P->st.prim_quartets = 0;
        P->st.fp32_quartets = 0;
        P->st.fp32_prim_quartets = 0;
        for (size_t t = 0; t < qcs.size(); t++) {
                const unsigned long long *h64 = hs + 2 * t, *h32 = hs + 2 * (64 + t);
                P->cls[t].quartets = (int64_t)(h64[0] + h32[0]);
                P->cls[t].prim_quartets = (int64_t)(h64[1] + h32[1]);
                P->cls[t].fp32_quartets = (int64_t)h32[0];
                P->st.quartets += P->cls[t].quartets;
                P->st.prim_quartets += P->cls[t].prim_quartets;
                P->st.fp32_quartets += (int64_t)h32[0];
                P->st.fp32_prim_quartets += (int64_t)h32[1];
                P->cls[t].ms = 0;
                if (P->profiling && ran[t]) {
                        float cm = 0;
                        CUDA_TRY(cudaEventElapsedTime(&cm, P->cls_ev[2 * t], P->cls_ev[2 * t + 1]));
                        P->cls[t].ms = cm;
                }
        }
        P->st.last_build_ms = ms;
        P->st.kernel_launches = launches;
        return B200JK_OK;
}

int b200jk_set_shard(b200jk_plan *plan, int index, int count)
{
        if (!plan) return fail(B200JK_EINVAL, "plan is NULL");
        if (count < 1 || index < 0 || index >= count) return fail(B200JK_EINVAL, "shard index must be in [0, count)");
        plan->shard = index;
        plan->nshard = count;
        return B200JK_OK;
}

int b200jk_set_prescreen(b200jk_plan *plan, int screen)
{
        if (!plan) return fail(B200JK_EINVAL, "plan is NULL");
        if (screen != B200JK_SCREEN_NRS8 && screen != B200JK_SCREEN_VJ && screen != B200JK_SCREEN_VK)
                return fail(B200JK_EINVAL, "screen must be B200JK_SCREEN_NRS8, _VJ or _VK");
        plan->screen = screen;
        return B200JK_OK;
}

int b200jk_set_class_thresholds(b200jk_plan *plan, const double *tau, int n)
{
        if (!plan) return fail(B200JK_EINVAL, "plan is NULL");
        const int nclass = (int)quartet_classes().size();
        if (!tau || n == 0) {
                plan->tau_class.clear();
                return B200JK_OK;
        }
        if (n != nclass) return fail(B200JK_EINVAL, "one threshold per quartet class (55) is required");
        for (int t = 0; t < n; t++)
                if (!(tau[t] >= 0)) return fail(B200JK_EINVAL, "thresholds must be >= 0");
        plan->tau_class.assign(tau, tau + n);
        return B200JK_OK;
}

int b200jk_get_class_thresholds(const b200jk_plan *plan, double *tau, int max, int *n)
{
        if (!plan || !n) return fail(B200JK_EINVAL, "NULL argument");
        const int nclass = (int)quartet_classes().size();
        *n = nclass;
        for (int t = 0; t < nclass && t < max && tau; t++) tau[t] = class_tau(plan, t);
        return B200JK_OK;
}

int b200jk_set_mixed_threshold(b200jk_plan *plan, double tau)
{
        if (!plan) return fail(B200JK_EINVAL, "plan is NULL");
        if (!(tau == tau)) return fail(B200JK_EINVAL, "tau is NaN");
        plan->fp32_tau = tau;
        plan->tau_class.clear();
        return B200JK_OK;
}

// sums[0] += sum D*J, sums[1] += sum D*K; dmax_bits: max |A - B| over n as
// bits of a non-negative double (for the mixed-precision tuner)
static __global__ void e2_terms_kernel(const double *D, const double *J, const double *K, long long n, double *sums)
{
        double sj = 0.0, sk = 0.0;
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
                sj += D[i] * J[i];
                sk += D[i] * K[i];
        }
        sj = warp_sum(sj);
        sk = warp_sum(sk);
        if ((threadIdx.x & 31) == 0) {
                atomicAdd(sums, sj);
                atomicAdd(sums + 1, sk);
        }
}

static __global__ void max_abs_diff_kernel(const double *A, const double *B, long long n, unsigned long long *bits)
{
        double m = 0.0;
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
                m = fmax(m, fabs(A[i] - B[i]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) atomicMax(bits, (unsigned long long)__double_as_longlong(m));
}

int b200jk_autotune_mixed(b200jk_plan *P, const double *dm, int dev_ptrs, double budget, double *result,
                          void *stream)
{
        if (!P || !dm) return fail(B200JK_EINVAL, "NULL argument");
        if (!(budget > 0)) return fail(B200JK_EINVAL, "the error budget must be > 0");
        CUDA_TRY(cudaSetDevice(P->device));
        int rc = ensure_workspace(P, 1);
        if (rc) return rc;
        cudaStream_t s = stream ? (cudaStream_t)stream : P->stream;
        const int nclass = (int)quartet_classes().size();
        const size_t nn = (size_t)P->nao * P->nao;
        // reference J/K of the FP64 build, the density on the device, reduction slots
        DevArr<double> ref, dd, sums;
        DevArr<unsigned long long> bits;
        auto cleanup = [&]() { ref.release(); dd.release(); sums.release(); bits.release(); };
        if ((rc = dev_alloc(ref, 2 * nn)) || (rc = dev_alloc(dd, nn)) || (rc = dev_alloc(sums, 2)) ||
            (rc = dev_alloc(bits, 2))) {
                cleanup();
                return rc;
        }
        const int saved_prof = P->profiling;
        const std::vector<double> saved_tau = P->tau_class;
        P->profiling = 1;
        double *oj = P->outJ.p, *ok = P->outK.p;
        if (cudaMemcpyAsync(dd.p, dm, sizeof(double) * nn, dev_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            s) != cudaSuccess) {
                P->profiling = saved_prof;
                cleanup();
                return fail(B200JK_ECUDA, "copy of the density failed");
        }
        const unsigned grid = (unsigned)std::min<long long>(4 * P->nsm, (long long)(nn + 255) / 256);
        std::vector<double> t64(nclass), t32(nclass), tau(nclass, 0.0);
        double e64 = 0, chosen = 0, de = 0, dj = 0, dk = 0;
        auto build = [&](int prec) -> int {
                return b200jk_get_jk(P, dd.p, 1, 1, 1, 1, oj, ok, 1, prec, stream);
        };
        auto e2_and_diff = [&](double &e2, double &maxj, double &maxk) -> int {
                CUDA_TRY(cudaMemsetAsync(sums.p, 0, 2 * sizeof(double), s));
                CUDA_TRY(cudaMemsetAsync(bits.p, 0, 2 * sizeof(unsigned long long), s));
                e2_terms_kernel<<<grid, 256, 0, s>>>(dd.p, oj, ok, (long long)nn, sums.p);
                max_abs_diff_kernel<<<grid, 256, 0, s>>>(oj, ref.p, (long long)nn, bits.p);
                max_abs_diff_kernel<<<grid, 256, 0, s>>>(ok, ref.p + nn, (long long)nn, bits.p + 1);
                CUDA_TRY(cudaGetLastError());
                double hs[2];
                unsigned long long hb[2];
                CUDA_TRY(cudaMemcpyAsync(hs, sums.p, sizeof(hs), cudaMemcpyDeviceToHost, s));
                CUDA_TRY(cudaMemcpyAsync(hb, bits.p, sizeof(hb), cudaMemcpyDeviceToHost, s));
                CUDA_TRY(cudaStreamSynchronize(s));
                e2 = 0.5 * hs[0] - 0.25 * hs[1];
                memcpy(&maxj, &hb[0], sizeof(double));
                memcpy(&maxk, &hb[1], sizeof(double));
                return B200JK_OK;
        };
        // 1. FP64 build: reference J/K and per-class times
        if ((rc = build(B200JK_PREC_FP64))) goto done;
        if (cudaMemcpyAsync(ref.p, oj, sizeof(double) * nn, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(ref.p + nn, ok, sizeof(double) * nn, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
                rc = fail(B200JK_ECUDA, "copy of the FP64 J/K failed");
                goto done;
        }
        for (int t = 0; t < nclass; t++) t64[t] = P->cls.size() > (size_t)t ? P->cls[t].ms : 0.0;
        {
                double a, b;
                if ((rc = e2_and_diff(e64, a, b))) goto done;
        }
        // 2. every quartet in float32: per-class times of the float32 kernels
        P->tau_class.assign(nclass, 1e300);
        if ((rc = build(B200JK_PREC_MIXED))) goto done;
        for (int t = 0; t < nclass; t++) t32[t] = P->cls.size() > (size_t)t ? P->cls[t].ms : 0.0;
        // 3. the largest threshold of the ladder, applied to the classes whose
        // float32 pass is faster, whose two-electron energy stays within budget
        {
                const double ladder[] = {1e-2, 1e-3, 1e-4, 1e-5, 1e-6, 1e-7, 1e-8};
                bool ok_found = false;
                for (double tv : ladder) {
                        for (int t = 0; t < nclass; t++) tau[t] = (t32[t] > 0 && t32[t] < 0.97 * t64[t]) ? tv : 0.0;
                        P->tau_class = tau;
                        if ((rc = build(B200JK_PREC_MIXED))) goto done;
                        double e2;
                        if ((rc = e2_and_diff(e2, dj, dk))) goto done;
                        de = e2 - e64;
                        if (fabs(de) <= budget) {
                                chosen = tv;
                                ok_found = true;
                                break;
                        }
                }
                if (!ok_found) {
                        std::fill(tau.begin(), tau.end(), 0.0);
                        P->tau_class = tau;
                        chosen = 0;
                }
        }
        if (result) {
                result[0] = chosen;
                result[1] = de;
                result[2] = dj;
                result[3] = dk;
        }
done:
        P->profiling = saved_prof;
        if (rc) P->tau_class = saved_tau;
        cleanup();
        return rc;
}

int b200jk_autotune(b200jk_plan *P, const double *dm, int dev_ptrs, void *stream)
{
        if (!P || !dm) return fail(B200JK_EINVAL, "NULL argument");
        CUDA_TRY(cudaSetDevice(P->device));
        int rc = ensure_workspace(P, 1);
        if (rc) return rc;
        auto qcs = quartet_classes();
        const int nclass = (int)qcs.size();
        std::vector<int> best(nclass, 0);
        std::vector<double> best_ms(nclass, 1e300);
        const int saved_prof = P->profiling;
        P->profiling = 1;
        // the builds write into the plan's own output buffers
        double *oj = dev_ptrs ? P->outJ.p : nullptr, *ok = dev_ptrs ? P->outK.p : nullptr;
        std::vector<double> hj, hk;
        if (!dev_ptrs) {
                hj.resize((size_t)P->nao * P->nao);
                hk.resize((size_t)P->nao * P->nao);
                oj = hj.data();
                ok = hk.data();
        }
        P->kvar.assign(nclass, 0);
        P->kvar32.assign(nclass, 0);
        if ((rc = b200jk_get_jk(P, dm, 1, 1, 1, 1, oj, ok, dev_ptrs, B200JK_PREC_FP64, stream))) goto done;   // warm-up
        // float64 variants on FP64 builds, then the float32 pass's variants on
        // mixed builds (class times there include the float64 pass, whose
        // variant is already fixed, so the comparison is the float32 pass's)
        for (int prec = 0; prec < 2; prec++) {
                std::vector<int> &kv = prec ? P->kvar32 : P->kvar;
                std::fill(best_ms.begin(), best_ms.end(), 1e300);
                std::fill(best.begin(), best.end(), 0);
                for (int v = 0; v < 3; v++) {
                        if (v == 2 && prec == 1) break;   // bra runs: float64 pass only
                        kv.assign(nclass, v);
                        if ((rc = b200jk_get_jk(P, dm, 1, 1, 1, 1, oj, ok, dev_ptrs,
                                                prec ? B200JK_PREC_MIXED : B200JK_PREC_FP64, stream)))
                                goto done;
                        for (int t = 0; t < nclass; t++) {
                                int la, lb, lc, ld;
                                class_l(qcs[t].X, la, lb);
                                class_l(qcs[t].Y, lc, ld);
                                if (!family_has_variant_n(la, lb, lc, ld, v)) continue;   // no such variant
                                if (P->cls[t].ms < best_ms[t]) { best_ms[t] = P->cls[t].ms; best[t] = v; }
                        }
                }
                kv = best;
        }
done:
        P->profiling = saved_prof;
        if (rc) {
                P->kvar.assign(nclass, 0);
                P->kvar32.assign(nclass, 0);
        }
        return rc;
}

int b200jk_set_tile(b200jk_plan *P, int tile_b)
{
        if (!P) return fail(B200JK_EINVAL, "plan is NULL");
        if (tile_b < 0 || tile_b > 4096) return fail(B200JK_EINVAL, "tile width must be in [0, 4096]");
        P->tile_b = tile_b;
        return B200JK_OK;
}

int b200jk_get_tuning(const b200jk_plan *P, int precision, int *variants, int max, int *n)
{
        if (!P || !n) return fail(B200JK_EINVAL, "NULL argument");
        if (precision != B200JK_PREC_FP64 && precision != B200JK_PREC_MIXED)
                return fail(B200JK_EINVAL, "precision must be B200JK_PREC_FP64 or B200JK_PREC_MIXED");
        *n = (int)quartet_classes().size();
        const int pass = precision == B200JK_PREC_MIXED ? 1 : 0;
        for (int t = 0; t < *n && t < max && variants; t++) variants[t] = class_variant(P, t, pass);
        return B200JK_OK;
}

int b200jk_set_tuning(b200jk_plan *P, int precision, const int *variants, int n)
{
        if (!P || !variants) return fail(B200JK_EINVAL, "NULL argument");
        if (precision != B200JK_PREC_FP64 && precision != B200JK_PREC_MIXED)
                return fail(B200JK_EINVAL, "precision must be B200JK_PREC_FP64 or B200JK_PREC_MIXED");
        auto qcs = quartet_classes();
        if (n != (int)qcs.size()) return fail(B200JK_EINVAL, "one variant per quartet class (55) is required");
        for (int t = 0; t < n; t++) {
                int la, lb, lc, ld;
                class_l(qcs[t].X, la, lb);
                class_l(qcs[t].Y, lc, ld);
                if (variants[t] < 0 || variants[t] > 2 || !family_has_variant_n(la, lb, lc, ld, variants[t]) ||
                    (variants[t] == 2 && precision == B200JK_PREC_MIXED))
                        return fail(B200JK_EINVAL, "variant not available for this quartet class");
        }
        (precision == B200JK_PREC_MIXED ? P->kvar32 : P->kvar).assign(variants, variants + n);
        return B200JK_OK;
}

int b200jk_set_profiling(b200jk_plan *plan, int on)
{
        if (!plan) return fail(B200JK_EINVAL, "plan is NULL");
        plan->profiling = on ? 1 : 0;
        return B200JK_OK;
}

int b200jk_class_stats(const b200jk_plan *plan, b200jk_class_stat_t *out, int max, int *n)
{
        if (!plan || !n) return fail(B200JK_EINVAL, "NULL argument");
        *n = (int)plan->cls.size();
        for (int t = 0; t < *n && t < max && out; t++) out[t] = plan->cls[t];
        return B200JK_OK;
}

int b200jk_measure_fp64_peak(int device, double *tflops)
{
        if (!tflops) return fail(B200JK_EINVAL, "tflops is NULL");
        CUDA_TRY(cudaSetDevice(device));
        cudaDeviceProp prop;
        CUDA_TRY(cudaGetDeviceProperties(&prop, device));
        const int block = 256, iters = 4096;
        const int grid = prop.multiProcessorCount * 8;
        DevArr<double> sink;
        int rc = dev_alloc(sink, (size_t)grid * block);
        if (rc) return rc;
        cudaEvent_t e0, e1;
        CUDA_TRY(cudaEventCreate(&e0));
        CUDA_TRY(cudaEventCreate(&e1));
        fp64_fma_kernel<<<grid, block>>>(sink.p, iters, 1.0000001);   // warm-up
        CUDA_TRY(cudaEventRecord(e0));
        for (int r = 0; r < 5; r++) fp64_fma_kernel<<<grid, block>>>(sink.p, iters, 1.0000001);
        CUDA_TRY(cudaEventRecord(e1));
        CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        sink.release();
        const double flops = 5.0 * grid * block * (double)iters * 8 * 2;
        *tflops = flops / (ms * 1e-3) / 1e12;
        return B200JK_OK;
}

int b200jk_debug_fail_alloc(int nth)
{
        if (nth < 0) return fail(B200JK_EINVAL, "nth must be >= 0");
        g_fail_alloc_countdown.store(nth);
        return B200JK_OK;
}

int b200jk_stats(const b200jk_plan *plan, b200jk_stats_t *stats)
{
        if (!plan || !stats) return fail(B200JK_EINVAL, "NULL argument");
        *stats = plan->st;
        return B200JK_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Nuclear-gradient J/K (pyscf/grad/rhf.py:149-178).

// packed offsets/exponents of the gradient classes (GClass in grad_kernels.cuh)
static void grad_goff(int la, int lb, int lc, int ld, int mode, std::vector<int2> &out)
{
        const int EB = lb + 2, EC = lc + 1 + mode, ED = ld + 1 + mode;
        auto eidx = [&](int a, int b, int c, int d) { return ((a * EB + b) * EC + c) * ED + d; };
        auto ex = [](int l, int n) { return cart_lx(l, n) | (cart_ly(l, n) << 2) | (cart_lz(l, n) << 4); };
        const int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
        for (int a = 0; a < na; a++)
                for (int b = 0; b < nb; b++)
                        for (int c = 0; c < nc; c++)
                                for (int d = 0; d < nd; d++) {
                                        const int ox = eidx(cart_lx(la, a), cart_lx(lb, b), cart_lx(lc, c), cart_lx(ld, d));
                                        const int oy = eidx(cart_ly(la, a), cart_ly(lb, b), cart_ly(lc, c), cart_ly(ld, d));
                                        const int oz = eidx(cart_lz(la, a), cart_lz(lb, b), cart_lz(lc, c), cart_lz(ld, d));
                                        out.push_back(make_int2(ox | (oy << 10) | (oz << 20),
                                                                ex(la, a) | (ex(lb, b) << 6) | (ex(lc, c) << 12) | (ex(ld, d) << 18)));
                                }
}

typedef int (*grad_launcher_t)(int, int, const GradArgs &, cudaStream_t, int, std::string &);
typedef int (*gq0_launcher_t)(const GradQArgs &, cudaStream_t, std::string &);
static const grad_launcher_t g_grad_launch[NPAIRCLASS] = {
        launch_grad_00, launch_grad_10, launch_grad_11, launch_grad_20, launch_grad_21,
        launch_grad_22, launch_grad_30, launch_grad_31, launch_grad_32, launch_grad_33};
static const gq0_launcher_t g_gq0_launch[NPAIRCLASS] = {
        launch_gq0_00, launch_gq0_10, launch_gq0_11, launch_gq0_20, launch_gq0_21,
        launch_gq0_22, launch_gq0_30, launch_gq0_31, launch_gq0_32, launch_gq0_33};

// upload one class of pairs in the given order, q per pair
static int upload_pairs(const b200jk_plan *P, PairClassDev &c, int X, const std::vector<PairLite> &hv,
                        const std::vector<double> &q)
{
        class_l(X, c.la, c.lb);
        c.n = (int)hv.size();
        for (int b = 0; b <= B2_NBUCKET; b++) c.boff[b] = 0;
        for (const PairLite &p : hv) c.boff[prim_bucket(p.nprim) + 1]++;
        for (int b = 0; b < B2_NBUCKET; b++) c.boff[b + 1] += c.boff[b];
        std::vector<int4> sh(hv.size());
        std::vector<int2> pr(hv.size());
        std::vector<double4> Av(hv.size()), ABv(hv.size());
        for (size_t t = 0; t < hv.size(); t++) {
                const SegLite &A = P->segl[hv[t].i], &B = P->segl[hv[t].j];
                sh[t] = make_int4(A.cart_off, B.cart_off, A.parent, B.parent);
                pr[t] = make_int2(hv[t].prim0, hv[t].nprim);
                Av[t] = make_double4(A.R[0], A.R[1], A.R[2], hv[t].i == hv[t].j ? 1.0 : 0.0);
                ABv[t] = make_double4(A.R[0] - B.R[0], A.R[1] - B.R[1], A.R[2] - B.R[2], 0.0);
        }
        int r;
        if ((r = dev_upload(c.sh, sh)) || (r = dev_upload(c.pr, pr)) || (r = dev_upload(c.q, q)) ||
            (r = dev_upload(c.qs, q)) || (r = dev_upload(c.A, Av)) || (r = dev_upload(c.AB, ABv)))
                return r;
        return B200JK_OK;
}

// q0 (once per plan) and the gradient pair lists (per screening tolerance)
static int ensure_grad(b200jk_plan *P, double tol)
{
        GradPlan &g = P->grad;
        const int nbas = P->nbas;
        const size_t n2 = (size_t)nbas * nbas;
        int rc;
        if (!g.q0_ready) {
                std::vector<int2> all;
                g.goff_at.assign(NPAIRCLASS * NPAIRCLASS + NPAIRCLASS, 0);
                for (int X = 0; X < NPAIRCLASS; X++) {
                        int la, lb;
                        class_l(X, la, lb);
                        for (int Y = 0; Y < NPAIRCLASS; Y++) {
                                int lc, ld;
                                class_l(Y, lc, ld);
                                g.goff_at[X * NPAIRCLASS + Y] = all.size();
                                grad_goff(la, lb, lc, ld, 0, all);
                        }
                }
                for (int X = 0; X < NPAIRCLASS; X++) {
                        int la, lb;
                        class_l(X, la, lb);
                        g.goff_at[NPAIRCLASS * NPAIRCLASS + X] = all.size();
                        grad_goff(la, lb, la, lb, 1, all);
                }
                if ((rc = dev_upload(g.goff, all))) return rc;
                std::vector<double> init(n2, 1e-100);
                if ((rc = dev_upload(g.q0, init))) return rc;
                for (int X = 0; X < NPAIRCLASS; X++) {
                        const std::vector<PairLite> &hv = P->all_pairs[X];
                        if (hv.empty()) continue;
                        PairClassDev tmp;
                        if ((rc = upload_pairs(P, tmp, X, hv, std::vector<double>(hv.size(), 0.0)))) return rc;
                        GradQArgs q;
                        q.omega2 = P->omega2;
                        q.pairs = tmp.view();
                        q.PP = P->PP.p; q.PK = P->PK.p; q.PE = P->PE.p;
                        q.table = table_ptr();
                        q.goff = g.goff.p + g.goff_at[NPAIRCLASS * NPAIRCLASS + X];
                        q.c2s = P->c2s.p;
                        q.q0 = (unsigned long long *)g.q0.p;
                        q.nbas = nbas;
                        q.cart = P->cart;
                        std::string err;
                        if (g_gq0_launch[X](q, P->stream, err)) { tmp.release(); return fail(B200JK_ECUDA, err); }
                        const cudaError_t e = cudaStreamSynchronize(P->stream);
                        tmp.release();
                        if (e != cudaSuccess) return fail(B200JK_ECUDA, std::string("gradient q_cond: ") + cudaGetErrorString(e));
                }
                g.h_q0.resize(n2);
                CUDA_TRY(cudaMemcpy(g.h_q0.data(), g.q0.p, sizeof(double) * n2, cudaMemcpyDeviceToHost));
                g.q0_ready = true;
                g.lists_ready = false;
        }
        if (g.lists_ready && g.tol == tol) return B200JK_OK;
        const std::vector<double> &q1 = P->h_qcond, &q0 = g.h_q0;
        double q0max = 0, q1max = 0;
        for (size_t t = 0; t < n2; t++) { q0max = std::max(q0max, q0[t]); q1max = std::max(q1max, q1[t]); }
        for (int X = 0; X < NPAIRCLASS; X++) {
                std::vector<PairLite> hb, hk;
                std::vector<double> qb, qk;
                for (const PairLite &p : P->all_pairs[X]) {
                        const size_t pi = P->segl[p.i].parent, pj = P->segl[p.j].parent;
                        const double b = std::max(q0[pi * nbas + pj], q0[pj * nbas + pi]);
                        const double k = q1[pi * nbas + pj];
                        if (!(tol > 0) || b * q1max > tol) { hb.push_back(p); qb.push_back(b); }
                        if (!(tol > 0) || k * q0max > tol) { hk.push_back(p); qk.push_back(k); }
                }
                // bucket-major, descending bound inside a bucket
                auto order = [](std::vector<PairLite> &v, std::vector<double> &q) {
                        std::vector<size_t> idx(v.size());
                        std::iota(idx.begin(), idx.end(), 0);
                        std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
                                const int ba = prim_bucket(v[a].nprim), bb = prim_bucket(v[b].nprim);
                                if (ba != bb) return ba < bb;
                                return q[a] > q[b];
                        });
                        std::vector<PairLite> v2(v.size());
                        std::vector<double> q2(v.size());
                        for (size_t t = 0; t < idx.size(); t++) { v2[t] = v[idx[t]]; q2[t] = q[idx[t]]; }
                        v.swap(v2);
                        q.swap(q2);
                };
                order(hb, qb);
                order(hk, qk);
                g.bra[X].release();
                g.ket[X].release();
                if ((rc = upload_pairs(P, g.bra[X], X, hb, qb)) || (rc = upload_pairs(P, g.ket[X], X, hk, qk))) return rc;
        }
        g.tol = tol;
        g.lists_ready = true;
        return B200JK_OK;
}

// The gradient build: vj/vk (de == nullptr) or, for one symmetric density,
// the fused force contraction into de[natm][3] (host or device, as dev_ptrs).
static int grad_build(b200jk_plan *P, const double *dms, int n_dm, int with_j, int with_k, double *vj, double *vk,
                      double *de, int dev_ptrs, double direct_scf_tol, void *stream)
{
        if (!P) return fail(B200JK_EINVAL, "plan is NULL");
        if (!dms || n_dm <= 0) return fail(B200JK_EINVAL, "no density matrices");
        if (!de && with_j && !vj) return fail(B200JK_EINVAL, "vj is NULL while with_j is set");
        if (!de && with_k && !vk) return fail(B200JK_EINVAL, "vk is NULL while with_k is set");
        if (!(direct_scf_tol == direct_scf_tol)) return fail(B200JK_EINVAL, "direct_scf_tol is NaN");
        const bool fused = de != nullptr;
        if (fused) {
                n_dm = 1;
                with_j = with_k = 1;
                vj = vk = nullptr;
        }
        CUDA_TRY(cudaSetDevice(P->device));
        int rc;
        if (dev_ptrs && ((rc = check_dev_ptr(dms, P->device, "dms")) || (with_j && (rc = check_dev_ptr(vj, P->device, "vj"))) ||
                         (with_k && (rc = check_dev_ptr(vk, P->device, "vk"))) || (rc = check_dev_ptr(de, P->device, "de"))))
                return rc;
        const double tol = direct_scf_tol > 0 ? direct_scf_tol : 0.0;
        if ((rc = ensure_grad(P, tol))) return rc;
        GradPlan &g = P->grad;
        const size_t nn = (size_t)P->nao * P->nao, nc = (size_t)P->naoc * P->naoc;
        int maxn = 1;
        for (auto &c : g.bra) maxn = std::max(maxn, c.n * B2_NBUCKET);
        if (fused && ((rc = dev_alloc(g.de, (size_t)3 * P->natm)) || (!g.shell_atom.p && (rc = dev_upload(g.shell_atom, P->shell_atom)))))
                return rc;
        if ((rc = dev_alloc(g.D, nn * n_dm)) || (rc = dev_alloc(g.Dc, nc * n_dm)) || (rc = dev_alloc(g.Ds, nc * n_dm)) ||
            (rc = dev_alloc(g.V, fused ? 1 : 6 * nc * n_dm)) || (rc = dev_alloc(g.out, dev_ptrs || fused ? 1 : 6 * nn * n_dm)) ||
            (rc = dev_alloc(g.dmc, (size_t)P->nbas * P->nbas)) || (rc = dev_alloc(g.fac, 1)) ||
            (rc = dev_alloc(g.dmax, 1)) || (rc = dev_alloc(g.stats, 2 * NPAIRCLASS * NPAIRCLASS)) || (rc = dev_alloc(g.nkl, maxn)) ||
            (rc = dev_alloc(g.kst, maxn)) || (rc = dev_alloc(g.nchunk, maxn + 1)) || (rc = dev_alloc(g.chunk_off, maxn + 1)))
                return rc;
        size_t cub_bytes = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, g.nchunk.p, g.chunk_off.p, maxn + 1);
        if ((rc = dev_alloc(g.cub_tmp, cub_bytes + 16))) return rc;

        cudaStream_t s = stream ? (cudaStream_t)stream : P->stream;
        CUDA_TRY(cudaEventRecord(P->ev0, s));
        const double *dD = dms;
        if (!dev_ptrs) {
                CUDA_TRY(cudaMemcpyAsync(g.D.p, dms, sizeof(double) * nn * n_dm, cudaMemcpyHostToDevice, s));
                dD = g.D.p;
        }
        CUDA_TRY(cudaMemsetAsync(g.dmax.p, 0, sizeof(unsigned long long), s));
        CUDA_TRY(cudaMemsetAsync(g.stats.p, 0, 2 * NPAIRCLASS * NPAIRCLASS * sizeof(unsigned long long), s));
        if (P->profiling && g.cls_ev.empty()) {
                g.cls_ev.resize(2 * NPAIRCLASS * NPAIRCLASS);
                for (auto &e : g.cls_ev) CUDA_TRY(cudaEventCreate(&e));
        }
        std::vector<char> ran(NPAIRCLASS * NPAIRCLASS, 0);
        int64_t launches = 0;
        dm_cond1_kernel<<<grid_for((long long)P->nbas * P->nbas, 256), 256, 0, s>>>(dD, n_dm, P->nao, P->ao_loc_d.p,
                                                                                  P->nbas, g.dmc.p, g.dmax.p);
        CUDA_TRY(cudaGetLastError());
        grad_dm_factor_kernel<<<1, 1, 0, s>>>(g.dmax.p, g.fac.p);
        CUDA_TRY(cudaGetLastError());
        launches += 2;
        for (int d = 0; d < n_dm; d++) {
                double *Dc = g.Dc.p + (size_t)d * nc;
                out_to_cart_kernel<<<grid_for((long long)nc, 256), 256, 0, s>>>(
                        dD + (size_t)d * nn, P->nao, P->naoc, P->cart_seg.p, P->cart_comp.p, P->seg_info.p, P->c2s.p,
                        P->cart, Dc, nullptr, nullptr);
                CUDA_TRY(cudaGetLastError());
                sym_sum_kernel<<<grid_for((long long)nc, 256), 256, 0, s>>>(Dc, P->naoc, g.Ds.p + (size_t)d * nc);
                CUDA_TRY(cudaGetLastError());
                launches += 2;
        }
        if (fused) CUDA_TRY(cudaMemsetAsync(g.de.p, 0, sizeof(double) * 3 * P->natm, s));
        else CUDA_TRY(cudaMemsetAsync(g.V.p, 0, sizeof(double) * 6 * nc * n_dm, s));
        double *Vj = fused ? nullptr : g.V.p, *Vk = fused ? nullptr : g.V.p + 3 * nc * n_dm;
        for (int X = 0; X < NPAIRCLASS; X++) {
                const PairClassDev &bra = g.bra[X];
                if (bra.n == 0) continue;
                for (int Y = 0; Y < NPAIRCLASS; Y++) {
                        const PairClassDev &ket = g.ket[Y];
                        if (ket.n == 0) continue;
                        const int nseg = bra.n * B2_NBUCKET;
                        const int chunk = grad_chunk(bra.la, bra.lb, ket.la, ket.lb, fused);
                        count_kernel<<<grid_for(nseg, 256), 256, 0, s>>>(bra.view(), ket.view(), 0, tol, g.fac.p, chunk,
                                                                        0.0, 0, P->shard, P->nshard, g.nkl.p, g.kst.p,
                                                                        g.nchunk.p);
                        CUDA_TRY(cudaGetLastError());
                        CUDA_TRY(cudaMemsetAsync(g.nchunk.p + nseg, 0, sizeof(long long), s));
                        size_t tmp = g.cub_tmp.n;
                        CUDA_TRY(cub::DeviceScan::ExclusiveSum(g.cub_tmp.p, tmp, g.nchunk.p, g.chunk_off.p, nseg + 1, s));
                        GradArgs a;
                        a.bra = bra.view();
                        a.ket = ket.view();
                        a.PP = P->PP.p; a.PK = P->PK.p; a.PE = P->PE.p;
                        a.chunk_off = g.chunk_off.p;
                        a.nkl = g.nkl.p;
                        a.kst = g.kst.p;
                        a.q0 = g.q0.p;
                        a.q1 = P->qcond.p;
                        a.dmc = g.dmc.p;
                        a.table = table_ptr();
                        a.goff = g.goff.p + g.goff_at[X * NPAIRCLASS + Y];
                        a.Vj = Vj; a.Vk = Vk;
                        a.Ds = g.Ds.p; a.Dc = g.Dc.p;
                        a.stats = g.stats.p + 2 * (X * NPAIRCLASS + Y);
                        a.tol = tol > 0 ? tol : -1.0;
                        a.nbas = P->nbas; a.naoc = P->naoc; a.n_dm = n_dm;
                        a.with_j = with_j; a.with_k = with_k;
                        a.de = fused ? g.de.p : nullptr;
                        a.omega2 = P->omega2;
                        a.shell_atom = fused ? g.shell_atom.p : nullptr;
                        std::string err;
                        if (P->profiling) CUDA_TRY(cudaEventRecord(g.cls_ev[2 * (X * NPAIRCLASS + Y)], s));
                        if (g_grad_launch[X](ket.la, ket.lb, a, s, P->nsm, err)) return fail(B200JK_ECUDA, err);
                        if (P->profiling) CUDA_TRY(cudaEventRecord(g.cls_ev[2 * (X * NPAIRCLASS + Y) + 1], s));
                        ran[X * NPAIRCLASS + Y] = 1;
                        launches += 2;   // count + class kernel (the scan is a CUB library kernel)
                }
        }
        // to the output basis.  The kernels differentiate with respect to the
        // centre (d/dA = -nabla_r of int2e_ip1), so the accumulators already
        // hold the negated contraction grad.rhf.get_jk returns
        double *oj = dev_ptrs ? vj : g.out.p, *ok = dev_ptrs ? vk : g.out.p + 3 * nn * n_dm;
        const long long nout = (long long)3 * n_dm * nn;
        if (fused) {
                // the forces are complete: no accumulators to transform
                if (dev_ptrs) CUDA_TRY(cudaMemcpyAsync(de, g.de.p, sizeof(double) * 3 * P->natm, cudaMemcpyDeviceToDevice, s));
                with_j = with_k = 0;
        }
        if (with_j) {
                grad_cart_to_out_kernel<<<grid_for(nout, 256), 256, 0, s>>>(Vj, 3 * n_dm, P->nao, P->naoc, P->out_seg.p,
                                                                          P->out_comp.p, P->seg_info.p, P->c2s.p, 1.0, oj);
                CUDA_TRY(cudaGetLastError());
                launches++;
        }
        if (with_k) {
                grad_cart_to_out_kernel<<<grid_for(nout, 256), 256, 0, s>>>(Vk, 3 * n_dm, P->nao, P->naoc, P->out_seg.p,
                                                                          P->out_comp.p, P->seg_info.p, P->c2s.p, 1.0, ok);
                CUDA_TRY(cudaGetLastError());
                launches++;
        }
        CUDA_TRY(cudaEventRecord(P->ev1, s));
        if (!dev_ptrs) {
                if (with_j) CUDA_TRY(cudaMemcpyAsync(vj, oj, sizeof(double) * nout, cudaMemcpyDeviceToHost, s));
                if (with_k) CUDA_TRY(cudaMemcpyAsync(vk, ok, sizeof(double) * nout, cudaMemcpyDeviceToHost, s));
                if (fused) CUDA_TRY(cudaMemcpyAsync(de, g.de.p, sizeof(double) * 3 * P->natm, cudaMemcpyDeviceToHost, s));
        }
        std::vector<unsigned long long> hs(2 * NPAIRCLASS * NPAIRCLASS);
        CUDA_TRY(cudaMemcpyAsync(hs.data(), g.stats.p, sizeof(unsigned long long) * hs.size(), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, P->ev0, P->ev1));
        g.quartets = g.prim_quartets = 0;
        g.cls.assign(NPAIRCLASS * NPAIRCLASS, b200jk_class_stat_t());
        for (int X = 0; X < NPAIRCLASS; X++)
                for (int Y = 0; Y < NPAIRCLASS; Y++) {
                        const int t = X * NPAIRCLASS + Y;
                        b200jk_class_stat_t &c = g.cls[t];
                        class_l(X, c.la, c.lb);
                        class_l(Y, c.lc, c.ld);
                        c.quartets = (int64_t)hs[2 * t];
                        c.prim_quartets = (int64_t)hs[2 * t + 1];
                        c.family = grad_register_family(c.la, c.lb, c.lc, c.ld, fused) ? 0 : 1;
                        c.ms = 0;
                        if (P->profiling && ran[t]) {
                                float cm = 0;
                                CUDA_TRY(cudaEventElapsedTime(&cm, g.cls_ev[2 * t], g.cls_ev[2 * t + 1]));
                                c.ms = cm;
                        }
                        g.quartets += c.quartets;
                        g.prim_quartets += c.prim_quartets;
                }
        g.last_ms = ms;
        g.launches = launches;
        return B200JK_OK;
}

extern "C" int b200jk_grad_jk(b200jk_plan *P, const double *dms, int n_dm, int with_j, int with_k, double *vj,
                              double *vk, int dev_ptrs, double direct_scf_tol, void *stream)
{
        return grad_build(P, dms, n_dm, with_j, with_k, vj, vk, nullptr, dev_ptrs, direct_scf_tol, stream);
}

extern "C" int b200jk_grad_contract(b200jk_plan *P, const double *dm, double *de, int dev_ptrs,
                                    double direct_scf_tol, void *stream)
{
        if (!de) return fail(B200JK_EINVAL, "de is NULL");
        return grad_build(P, dm, 1, 1, 1, nullptr, nullptr, de, dev_ptrs, direct_scf_tol, stream);
}

extern "C" int b200jk_grad_stats(const b200jk_plan *P, int64_t *quartets, int64_t *prim_quartets, double *ms,
                                 int64_t *kernel_launches)
{
        if (!P) return fail(B200JK_EINVAL, "plan is NULL");
        if (quartets) *quartets = P->grad.quartets;
        if (prim_quartets) *prim_quartets = P->grad.prim_quartets;
        if (ms) *ms = P->grad.last_ms;
        if (kernel_launches) *kernel_launches = P->grad.launches;
        return B200JK_OK;
}

extern "C" int b200jk_grad_class_stats(const b200jk_plan *P, b200jk_class_stat_t *out, int max, int *n)
{
        if (!P || !n) return fail(B200JK_EINVAL, "NULL argument");
        *n = (int)P->grad.cls.size();
        for (int t = 0; t < *n && t < max && out; t++) out[t] = P->grad.cls[t];
        return B200JK_OK;
}

extern "C" int b200jk_get_grad_q_cond(b200jk_plan *P, double *q_cond)
{
        if (!P || !q_cond) return fail(B200JK_EINVAL, "NULL argument");
        CUDA_TRY(cudaSetDevice(P->device));
        int rc = ensure_grad(P, P->grad.lists_ready ? P->grad.tol : 1e-14);
        if (rc) return rc;
        const size_t n2 = (size_t)P->nbas * P->nbas;
        memcpy(q_cond, P->grad.h_q0.data(), sizeof(double) * n2);
        memcpy(q_cond + n2, P->h_qcond.data(), sizeof(double) * n2);
        return B200JK_OK;
}


// ---------------------------------------------------------------------------
// Batches of molecules (one launch per quartet class for all of them).

struct b200jk_batch {
        std::vector<b200jk_plan *> plans;
        int device = 0, nsm = 148;
        cudaStream_t stream = nullptr;
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        DevArr<JKArgs> args;
        DevArr<int> segoff, nkl, kst;
        DevArr<long long> nchunk, chunk_off, mchunk;
        DevArr<unsigned char> cub_tmp;
        DevArr<unsigned long long> stats;
        JKArgs *h_args = nullptr;       // pinned staging of the per-class argument arrays
        int *h_segoff = nullptr;
        size_t h_cap_args = 0, h_cap_seg = 0;
        // staging of the asynchronous entry (read by captured graphs at replay)
        JKArgs *h_args_async = nullptr;
        int *h_segoff_async = nullptr;
        // workspace generation of every plan when the last synchronous build
        // sized the buffers; the asynchronous entry refuses to run when a
        // plan's workspace has moved since (its captured graphs would use the
        // freed buffers)
        std::vector<long long> ws_gen;
        const double *tbl = nullptr;
        const float *tbl_f = nullptr;
        int64_t quartets = 0, prim_quartets = 0, fp32_quartets = 0, launches = 0;
        double last_ms = 0;
        ~b200jk_batch()
        {
                args.release(); segoff.release(); nkl.release(); kst.release(); nchunk.release();
                chunk_off.release(); mchunk.release(); cub_tmp.release(); stats.release();
                if (h_args) cudaFreeHost(h_args);
                if (h_segoff) cudaFreeHost(h_segoff);
                if (h_args_async) cudaFreeHost(h_args_async);
                if (h_segoff_async) cudaFreeHost(h_segoff_async);
                if (ev0) cudaEventDestroy(ev0);
                if (ev1) cudaEventDestroy(ev1);
                if (stream) cudaStreamDestroy(stream);
        }
};

extern "C" int b200jk_batch_create(b200jk_plan *const *plans, int nmol, b200jk_batch **out)
{
        if (!out) return fail(B200JK_EINVAL, "out is NULL");
        *out = nullptr;
        if (!plans || nmol <= 0) return fail(B200JK_EINVAL, "no plans");
        for (int m = 0; m < nmol; m++) {
                if (!plans[m]) return fail(B200JK_EINVAL, "a plan of the batch is NULL");
                if (plans[m]->device != plans[0]->device) return fail(B200JK_EINVAL, "the plans of a batch must share one GPU");
                if (plans[m]->nshard != 1) return fail(B200JK_EUNSUPPORTED, "sharded plans cannot be batched");
        }
        CUDA_TRY(cudaSetDevice(plans[0]->device));
        b200jk_batch *B = new b200jk_batch();
        B->plans.assign(plans, plans + nmol);
        B->device = plans[0]->device;
        B->nsm = plans[0]->nsm;
        if (cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&B->ev0) != cudaSuccess || cudaEventCreate(&B->ev1) != cudaSuccess) {
                delete B;
                return fail(B200JK_ECUDA, "stream/event creation failed");
        }
        B->tbl = table_ptr();
        B->tbl_f = table_f_ptr();
        *out = B;
        return B200JK_OK;
}

extern "C" int b200jk_batch_destroy(b200jk_batch *B)
{
        delete B;
        return B200JK_OK;
}

// async: no allocation (every buffer must exist from an earlier synchronous
// call), no host synchronisation, no statistics read-back, its own pinned
// staging of the argument arrays -- the launches alone, so that a caller can
// capture them in a CUDA graph
static int batch_build(b200jk_batch *B, const double *const *dms, int hermi, int with_j, int with_k,
                       double *const *vj, double *const *vk, int precision_mode, void *stream, bool async)
{
        if (!B) return fail(B200JK_EINVAL, "batch is NULL");
        if (!dms) return fail(B200JK_EINVAL, "dms is NULL");
        if (hermi < 0 || hermi > 2) return fail(B200JK_EINVAL, "hermi must be 0, 1 or 2");
        if ((with_j && !vj) || (with_k && !vk)) return fail(B200JK_EINVAL, "output pointer array is NULL");
        if (precision_mode != B200JK_PREC_FP64 && precision_mode != B200JK_PREC_MIXED)
                return fail(B200JK_EUNSUPPORTED, "precision_mode must be 0 (FP64) or 1 (mixed FP32/FP64)");
        const int nmol = (int)B->plans.size();
        for (int m = 0; m < nmol; m++)
                if (!dms[m] || (with_j && !vj[m]) || (with_k && !vk[m])) return fail(B200JK_EINVAL, "NULL device pointer in the batch");
        // thresholds of the first plan (per class when it has them)
        const int mixed = precision_mode == B200JK_PREC_MIXED;
        CUDA_TRY(cudaSetDevice(B->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : B->stream;
        const int nk = hermi == 1 ? 1 : 2;
        int rc;
        for (int m = 0; m < nmol; m++) {
                if (async) {
                        if (B->plans[m]->ws_ndm < 1 || B->ws_gen.size() != (size_t)nmol)
                                return fail(B200JK_EINVAL, "b200jk_batch_get_jk_async needs one b200jk_batch_get_jk call first");
                        if (B->plans[m]->ws_gen != B->ws_gen[m])
                                return fail(B200JK_EINVAL, "a plan's workspace moved since the last b200jk_batch_get_jk "
                                                           "(a larger build on it); call b200jk_batch_get_jk again");
                } else {
                        if ((rc = check_dev_ptr(dms[m], B->device, "dms[m]")) ||
                            (with_j && (rc = check_dev_ptr(vj[m], B->device, "vj[m]"))) ||
                            (with_k && (rc = check_dev_ptr(vk[m], B->device, "vk[m]"))))
                                return rc;
                        if ((rc = ensure_workspace(B->plans[m], 1))) return rc;
                }
        }
        if (!async) {
                B->ws_gen.resize(nmol);
                for (int m = 0; m < nmol; m++) B->ws_gen[m] = B->plans[m]->ws_gen;
        }
        auto qcs = quartet_classes();
        const int nclass = (int)qcs.size();
        // argument arrays of every (class, pass): only molecules with work in the class
        std::vector<size_t> at(2 * nclass + 1, 0), sat(2 * nclass + 1, 0);
        std::vector<int> ncnt(2 * nclass, 0);
        size_t tot_args = 0, tot_seg = 0;
        int max_segs = 1;
        for (int t = 0; t < nclass; t++) {
                int cnt = 0, segs = 0;
                for (int m = 0; m < nmol; m++) {
                        const PairClassDev &bra = B->plans[m]->pc[qcs[t].X], &ket = B->plans[m]->pc[qcs[t].Y];
                        if (bra.n == 0 || ket.n == 0) continue;
                        cnt++;
                        segs += bra.n * B2_NBUCKET;
                }
                max_segs = std::max(max_segs, segs);
                for (int pass = 0; pass < 2; pass++) {
                        at[2 * t + pass] = tot_args;
                        sat[2 * t + pass] = tot_seg;
                        ncnt[2 * t + pass] = cnt;
                        tot_args += cnt;
                        tot_seg += cnt + 1;
                }
        }
        if (async) {
                if (tot_args > B->h_cap_args || tot_seg > B->h_cap_seg || !B->h_args_async || B->args.n < tot_args)
                        return fail(B200JK_EINVAL, "b200jk_batch_get_jk_async needs one b200jk_batch_get_jk call first");
        } else {
                if (tot_args > B->h_cap_args || !B->h_args_async) {
                        if (B->h_args) cudaFreeHost(B->h_args);
                        if (B->h_args_async) cudaFreeHost(B->h_args_async);
                        B->h_args = B->h_args_async = nullptr;
                        CUDA_TRY(cudaMallocHost(&B->h_args, sizeof(JKArgs) * tot_args));
                        CUDA_TRY(cudaMallocHost(&B->h_args_async, sizeof(JKArgs) * tot_args));
                        B->h_cap_args = tot_args;
                }
                if (tot_seg > B->h_cap_seg || !B->h_segoff_async) {
                        if (B->h_segoff) cudaFreeHost(B->h_segoff);
                        if (B->h_segoff_async) cudaFreeHost(B->h_segoff_async);
                        B->h_segoff = B->h_segoff_async = nullptr;
                        CUDA_TRY(cudaMallocHost(&B->h_segoff, sizeof(int) * tot_seg));
                        CUDA_TRY(cudaMallocHost(&B->h_segoff_async, sizeof(int) * tot_seg));
                        B->h_cap_seg = tot_seg;
                }
                if ((rc = dev_alloc(B->args, std::max<size_t>(1, tot_args))) ||
                    (rc = dev_alloc(B->segoff, std::max<size_t>(1, tot_seg))) || (rc = dev_alloc(B->nkl, max_segs)) ||
                    (rc = dev_alloc(B->kst, max_segs)) || (rc = dev_alloc(B->nchunk, max_segs + 1)) ||
                    (rc = dev_alloc(B->chunk_off, max_segs + 1)) || (rc = dev_alloc(B->mchunk, nmol + 1)) ||
                    (rc = dev_alloc(B->stats, 4 * 64)))
                        return rc;
                size_t cub_bytes = 0;
                cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, B->nchunk.p, B->chunk_off.p, max_segs + 1);
                if ((rc = dev_alloc(B->cub_tmp, cub_bytes + 16))) return rc;
        }
        JKArgs *h_args = async ? B->h_args_async : B->h_args;
        int *h_segoff = async ? B->h_segoff_async : B->h_segoff;

        if (!async) CUDA_TRY(cudaEventRecord(B->ev0, s));
        int64_t launches = 0;
        // per molecule: screening data, Cartesian densities, cleared accumulators
        for (int m = 0; m < nmol; m++) {
                b200jk_plan *P = B->plans[m];
                const size_t nc = (size_t)P->naoc * P->naoc;
                CUDA_TRY(cudaMemsetAsync(P->dmax.p, 0, sizeof(unsigned long long), s));
                const long long npair = (long long)P->nbas * (P->nbas + 1) / 2;
                dm_cond_kernel<<<grid_for(npair, 256), 256, 0, s>>>(dms[m], 1, P->nao, P->ao_loc_d.p, P->nbas,
                                                                  P->dm_cond.p, P->dmax.p);
                CUDA_TRY(cudaGetLastError());
                out_to_cart_kernel<<<grid_for((long long)nc, 256), 256, 0, s>>>(
                        dms[m], P->nao, P->naoc, P->cart_seg.p, P->cart_comp.p, P->seg_info.p, P->c2s.p, P->cart,
                        P->Dc.p, nk == 2 ? P->Dc.p + nc : nullptr, nullptr);
                CUDA_TRY(cudaGetLastError());
                sym_sum_kernel<<<grid_for((long long)nc, 256), 256, 0, s>>>(P->Dc.p, P->naoc, P->Ds.p);
                CUDA_TRY(cudaGetLastError());
                if (with_j && P->pk_total > 0) {
                        pack_gather_kernel<<<grid_for(P->pk_total, 256), 256, 0, s>>>(P->Ds.p, P->pk_src.p, P->pk_total,
                                                                                   P->Dpk.p);
                        CUDA_TRY(cudaGetLastError());
                        CUDA_TRY(cudaMemsetAsync(P->Jpk.p, 0, sizeof(double) * P->pk_total, s));
                        launches++;
                }
                if (with_j) CUDA_TRY(cudaMemsetAsync(P->Jacc.p, 0, sizeof(double) * nc, s));
                if (with_k) CUDA_TRY(cudaMemsetAsync(P->Kacc.p, 0, sizeof(double) * nc * nk, s));
                launches += 3;
        }
        CUDA_TRY(cudaMemsetAsync(B->stats.p, 0, 4 * 64 * sizeof(unsigned long long), s));
        const double *tbl = B->tbl;
        const float *tbl_f = B->tbl_f;
        // argument arrays (pointers only depend on the workspaces): fill and upload once
        for (int t = 0; t < nclass; t++) {
                for (int pass = 0; pass < 2; pass++) {
                        JKArgs *ha = h_args + at[2 * t + pass];
                        int *hs = h_segoff + sat[2 * t + pass];
                        int k = 0, seg = 0;
                        for (int m = 0; m < nmol; m++) {
                                b200jk_plan *P = B->plans[m];
                                const PairClassDev &bra = P->pc[qcs[t].X], &ket = P->pc[qcs[t].Y];
                                if (bra.n == 0 || ket.n == 0) continue;
                                JKArgs a{};
                                a.bra = bra.view();
                                a.ket = ket.view();
                                a.PP = P->PP.p; a.PK = P->PK.p;
                                a.chunk_off = B->chunk_off.p + seg;
                                a.nkl = B->nkl.p + seg;
                                a.kst = B->kst.p + seg;
                                a.dm_cond = P->dm_cond.p;
                                a.table = tbl;
                                a.table_f = tbl_f;
                                a.goff = P->goff_all.p + P->goff_at[t];
                                a.Jacc = P->Jacc.p; a.Kacc = P->Kacc.p;
                                a.Ds = P->Ds.p; a.Dk = P->Dc.p;
                                a.Dpk = P->Dpk.p + P->pk_off[qcs[t].Y];
                                a.Jpk = P->Jpk.p + P->pk_off[qcs[t].Y];
                                a.pk_stride = P->pk_total;
                                a.stats = B->stats.p + 2 * (64 * pass + t);
                                a.dmax4 = (const double *)P->dmax.p;
                                a.tol = P->tol > 0 ? P->tol : -1.0;
                                a.nbas = P->nbas; a.naoc = P->naoc; a.n_dm = 1; a.nk = nk;
                                a.with_j = with_j; a.with_k = with_k; a.same = qcs[t].X == qcs[t].Y;
                                a.screen = P->screen;
                                a.omega2 = P->omega2;
                                ha[k] = a;
                                hs[k] = seg;
                                k++;
                                seg += bra.n * B2_NBUCKET;
                        }
                        hs[k] = seg;
                }
        }
        CUDA_TRY(cudaMemcpyAsync(B->args.p, h_args, sizeof(JKArgs) * tot_args, cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(B->segoff.p, h_segoff, sizeof(int) * tot_seg, cudaMemcpyHostToDevice, s));
        for (int t = 0; t < nclass; t++) {
                int la, lb, lc, ld;
                class_l(qcs[t].X, la, lb);
                class_l(qcs[t].Y, lc, ld);
                const double tau = mixed ? class_tau(B->plans[0], t) : 0.0;
                for (int pass = 0; pass < (tau > 0 ? 2 : 1); pass++) {
                        const int nm = ncnt[2 * t + pass];
                        if (nm == 0) continue;
                        // bra runs (variant 2) need the tiled pass of one plan: a batch
                        // runs those classes as variant 0
                        int variant = class_variant(B->plans[0], t, pass);
                        if (variant == 2) variant = 0;
                        const int chunk = family_chunk(la, lb, lc, ld, variant);
                        const JKArgs *dargs = B->args.p + at[2 * t + pass];
                        const int *dseg = B->segoff.p + sat[2 * t + pass];
                        const int segs = h_segoff[sat[2 * t + pass] + nm];
                        count_kernel_multi<<<grid_for(segs, 256), 256, 0, s>>>(dargs, dseg, nm, chunk, tau,
                                                                              pass, B->nkl.p, B->kst.p, B->nchunk.p);
                        CUDA_TRY(cudaGetLastError());
                        CUDA_TRY(cudaMemsetAsync(B->nchunk.p + segs, 0, sizeof(long long), s));
                        size_t tmp = B->cub_tmp.n;
                        CUDA_TRY(cub::DeviceScan::ExclusiveSum(B->cub_tmp.p, tmp, B->nchunk.p, B->chunk_off.p, segs + 1, s));
                        batch_chunk_starts<<<grid_for(nm + 1, 128), 128, 0, s>>>(B->chunk_off.p, dseg, nm, B->mchunk.p);
                        CUDA_TRY(cudaGetLastError());
                        const JKArgs &a0 = h_args[at[2 * t + pass]];
                        if ((rc = dispatch_jk(B->plans[0], la, lb, lc, ld, a0, pass, s, dargs, B->mchunk.p, nm, variant)))
                                return rc;
                        launches += 3;
                }
        }
        // back to the output basis, per molecule
        for (int m = 0; m < nmol; m++) {
                b200jk_plan *P = B->plans[m];
                const size_t nn = (size_t)P->nao * P->nao, nc = (size_t)P->naoc * P->naoc;
                if (with_j && P->pk_total > 0) {
                        pack_scatter_add_kernel<<<grid_for(P->pk_total, 256), 256, 0, s>>>(P->Jpk.p, P->pk_src.p,
                                                                                        P->pk_total, P->Jacc.p);
                        CUDA_TRY(cudaGetLastError());
                        launches++;
                }
                if (with_j) {
                        cart_to_out_kernel<<<grid_for((long long)nn, 256), 256, 0, s>>>(
                                P->Jacc.p, P->Jacc.p, P->nao, P->naoc, P->out_seg.p, P->out_comp.p, P->seg_info.p, P->c2s.p,
                                P->cart, 1, vj[m]);
                        CUDA_TRY(cudaGetLastError());
                        launches++;
                }
                if (with_k) {
                        const double *K2 = nk == 2 ? P->Kacc.p + nc : P->Kacc.p;
                        cart_to_out_kernel<<<grid_for((long long)nn, 256), 256, 0, s>>>(
                                P->Kacc.p, K2, P->nao, P->naoc, P->out_seg.p, P->out_comp.p, P->seg_info.p, P->c2s.p,
                                P->cart, hermi, vk[m]);
                        CUDA_TRY(cudaGetLastError());
                        launches++;
                }
        }
        if (async) return B200JK_OK;
        CUDA_TRY(cudaEventRecord(B->ev1, s));
        unsigned long long hs[4 * 64];
        CUDA_TRY(cudaMemcpyAsync(hs, B->stats.p, sizeof(hs), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, B->ev0, B->ev1));
        B->quartets = B->prim_quartets = B->fp32_quartets = 0;
        for (int t = 0; t < nclass; t++) {
                B->quartets += (int64_t)(hs[2 * t] + hs[2 * (64 + t)]);
                B->prim_quartets += (int64_t)(hs[2 * t + 1] + hs[2 * (64 + t) + 1]);
                B->fp32_quartets += (int64_t)hs[2 * (64 + t)];
        }
        B->last_ms = ms;
        B->launches = launches;
        return B200JK_OK;
}

extern "C" int b200jk_batch_get_jk(b200jk_batch *B, const double *const *dms, int hermi, int with_j, int with_k,
                                   double *const *vj, double *const *vk, int precision_mode, void *stream)
{
        return batch_build(B, dms, hermi, with_j, with_k, vj, vk, precision_mode, stream, false);
}

extern "C" int b200jk_batch_get_jk_async(b200jk_batch *B, const double *const *dms, int hermi, int with_j,
                                         int with_k, double *const *vj, double *const *vk, int precision_mode,
                                         void *stream)
{
        return batch_build(B, dms, hermi, with_j, with_k, vj, vk, precision_mode, stream, true);
}

extern "C" int b200jk_batch_stats(const b200jk_batch *B, int64_t *quartets, int64_t *fp32_quartets, double *ms,
                                  int64_t *kernel_launches)
{
        if (!B) return fail(B200JK_EINVAL, "batch is NULL");
        if (quartets) *quartets = B->quartets;
        if (fp32_quartets) *fp32_quartets = B->fp32_quartets;
        if (ms) *ms = B->last_ms;
        if (kernel_launches) *kernel_launches = B->launches;
        return B200JK_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free J/K build.
//
// Some callers cannot let a library call cudaMalloc: code that runs under a
// framework's caching allocator or a fixed device-memory budget (a cudaMalloc
// there can fail because the pool holds the memory, and it synchronises the
// device in the middle of the caller's stream work).  b200jk_get_jk_noalloc
// serves them: it runs the same kernels as b200jk_get_jk, but every
// intermediate (Cartesian densities, J/K accumulators, screening and chunk
// arrays, scan storage) lives in the file-scope array below, of fixed size
// B200JK_NOALLOC_SCRATCH_BYTES, which each GPU that loads this library holds
// until the process exits.  The plan must exist already (creating it
// allocates); the call itself allocates nothing.

#define B200JK_NOALLOC_SCRATCH_BYTES (32ull << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[B200JK_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch on each device, resolved by the first
// no-alloc call on that device that succeeds in doing so (with that device
// current).  A failed attempt is not remembered: the next call tries again.
static std::mutex g_noalloc_mu;
static unsigned char *g_noalloc_ptr[64];

static size_t noalloc_align(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" int b200jk_get_jk_noalloc(b200jk_plan *P, const double *dms, int n_dm, int hermi, int with_j,
                                     int with_k, double *vj, double *vk, void *stream)
{
        if (!P) return fail(B200JK_EINVAL, "plan is NULL");
        if (!dms || n_dm <= 0) return fail(B200JK_EINVAL, "no density matrices");
        if (hermi < 0 || hermi > 2) return fail(B200JK_EINVAL, "hermi must be 0, 1 or 2");
        if (with_j && !vj) return fail(B200JK_EINVAL, "vj is NULL while with_j is set");
        if (with_k && !vk) return fail(B200JK_EINVAL, "vk is NULL while with_k is set");
        const int dev = P->device;
        if (dev < 0 || dev >= 64) return fail(B200JK_EINVAL, "device index out of range");
        CUDA_TRY(cudaSetDevice(dev));
        // the kernels read and write these arrays directly: host memory would
        // fault the GPU, so anything but device memory of the plan's GPU is an error
        int rc;
        if ((rc = check_dev_ptr(dms, dev, "dms")) || (with_j && (rc = check_dev_ptr(vj, dev, "vj"))) ||
            (with_k && (rc = check_dev_ptr(vk, dev, "vk"))))
                return rc;
        unsigned char *base = nullptr;
        {
                std::lock_guard<std::mutex> lk(g_noalloc_mu);
                if (!g_noalloc_ptr[dev]) {
                        void *p = nullptr;
                        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
                        if (e != cudaSuccess || !p)
                                return fail(B200JK_ECUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") +
                                                                  cudaGetErrorString(e));
                        g_noalloc_ptr[dev] = (unsigned char *)p;
                }
                base = g_noalloc_ptr[dev];
        }

        // carve the scratch array; reject sizes beyond it before any work
        const size_t nn = (size_t)P->nao * P->nao, nc = (size_t)P->naoc * P->naoc;
        const int nk = hermi == 1 ? 1 : 2;
        int maxn = 1;
        for (auto &c : P->pc) maxn = std::max(maxn, c.n * B2_NBUCKET);
        size_t cub_bytes = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, (long long *)nullptr, (long long *)nullptr, maxn + 1);
        size_t off = 0;
        auto take = [&](size_t bytes) { size_t o = off; off += noalloc_align(bytes); return o; };
        const size_t o_Dc = take(sizeof(double) * nc * n_dm * nk);
        const size_t o_Ds = take(sizeof(double) * nc * n_dm);
        const size_t o_J = take(with_j ? sizeof(double) * nc * n_dm : 0);
        const size_t o_K = take(with_k ? sizeof(double) * nc * n_dm * nk : 0);
        const size_t o_dmc = take(sizeof(double) * (size_t)P->nbas * P->nbas);
        const size_t o_dmax = take(sizeof(unsigned long long));
        const size_t o_stats = take(sizeof(unsigned long long) * 2 * 64);
        const size_t o_nkl = take(sizeof(int) * (size_t)maxn);
        const size_t o_kst = take(sizeof(int) * (size_t)maxn);
        const size_t o_nchunk = take(sizeof(long long) * (size_t)(maxn + 1));
        const size_t o_off = take(sizeof(long long) * (size_t)(maxn + 1));
        const size_t o_cub = take(cub_bytes + 16);
        if (off > B200JK_NOALLOC_SCRATCH_BYTES) {
                char msg[256];
                snprintf(msg, sizeof(msg),
                         "b200jk_get_jk_noalloc needs %zu bytes of scratch for nao_cart=%d, n_dm=%d, hermi=%d; "
                         "the fixed scratch holds %llu bytes (use b200jk_get_jk)",
                         off, P->naoc, n_dm, hermi, (unsigned long long)B200JK_NOALLOC_SCRATCH_BYTES);
                return fail(B200JK_EINVAL, msg);
        }
        double *Dc = (double *)(base + o_Dc), *Ds = (double *)(base + o_Ds);
        double *Jacc = (double *)(base + o_J), *Kacc = (double *)(base + o_K);
        double *dmc = (double *)(base + o_dmc);
        unsigned long long *dmax = (unsigned long long *)(base + o_dmax);
        unsigned long long *stats = (unsigned long long *)(base + o_stats);
        int *nkl = (int *)(base + o_nkl), *kst = (int *)(base + o_kst);
        long long *nchunk = (long long *)(base + o_nchunk), *chunk_off = (long long *)(base + o_off);
        void *cub_tmp = base + o_cub;

        cudaStream_t s = stream ? (cudaStream_t)stream : P->stream;
        // the array keeps the previous call's contents: clear what accumulates
        CUDA_TRY(cudaMemsetAsync(dmax, 0, sizeof(unsigned long long), s));
        CUDA_TRY(cudaMemsetAsync(stats, 0, 2 * 64 * sizeof(unsigned long long), s));
        if (with_j) CUDA_TRY(cudaMemsetAsync(Jacc, 0, sizeof(double) * nc * n_dm, s));
        if (with_k) CUDA_TRY(cudaMemsetAsync(Kacc, 0, sizeof(double) * nc * n_dm * nk, s));
        {
                const long long npair = (long long)P->nbas * (P->nbas + 1) / 2;
                dm_cond_kernel<<<grid_for(npair, 256), 256, 0, s>>>(dms, n_dm, P->nao, P->ao_loc_d.p, P->nbas, dmc, dmax);
                CUDA_TRY(cudaGetLastError());
        }
        for (int d = 0; d < n_dm; d++) {
                double *dc = Dc + (size_t)d * nk * nc;
                out_to_cart_kernel<<<grid_for((long long)nc, 256), 256, 0, s>>>(
                        dms + (size_t)d * nn, P->nao, P->naoc, P->cart_seg.p, P->cart_comp.p, P->seg_info.p,
                        P->c2s.p, P->cart, dc, nk == 2 ? dc + nc : nullptr, nullptr);
                CUDA_TRY(cudaGetLastError());
                sym_sum_kernel<<<grid_for((long long)nc, 256), 256, 0, s>>>(dc, P->naoc, Ds + (size_t)d * nc);
                CUDA_TRY(cudaGetLastError());
        }
        const double *tbl = table_ptr();
        auto qcs = quartet_classes();
        for (size_t t = 0; t < qcs.size(); t++) {
                const PairClassDev &bra = P->pc[qcs[t].X], &ket = P->pc[qcs[t].Y];
                if (bra.n == 0 || ket.n == 0) continue;
                const int la = bra.la, lb = bra.lb, lc = ket.la, ld = ket.lb;
                const int same = qcs[t].X == qcs[t].Y;
                const int nseg = bra.n * B2_NBUCKET;
                count_kernel<<<grid_for(nseg, 256), 256, 0, s>>>(bra.view(), ket.view(), same, P->tol > 0 ? P->tol : 0.0,
                                                                (const double *)dmax, family_chunk(la, lb, lc, ld),
                                                                0.0, 0, P->shard, P->nshard, nkl, kst, nchunk);
                CUDA_TRY(cudaGetLastError());
                CUDA_TRY(cudaMemsetAsync(nchunk + nseg, 0, sizeof(long long), s));
                size_t tmp = cub_bytes;
                CUDA_TRY(cub::DeviceScan::ExclusiveSum(cub_tmp, tmp, nchunk, chunk_off, nseg + 1, s));
                JKArgs a;
                a.bra = bra.view();
                a.ket = ket.view();
                a.PP = P->PP.p; a.PK = P->PK.p;
                a.chunk_off = chunk_off;
                a.nkl = nkl;
                a.kst = kst;
                a.dm_cond = dmc;
                a.table = tbl;
                a.goff = P->goff_all.p + P->goff_at[t];
                a.Jacc = Jacc; a.Kacc = Kacc;
                a.Ds = Ds; a.Dk = Dc;
                a.stats = stats + 2 * t;
                a.tol = P->tol > 0 ? P->tol : -1.0;
                a.nbas = P->nbas; a.naoc = P->naoc; a.n_dm = n_dm; a.nk = nk;
                a.with_j = with_j; a.with_k = with_k; a.same = same;
                a.screen = P->screen;
                                a.omega2 = P->omega2;
                if ((rc = dispatch_jk(P, la, lb, lc, ld, a, 0, s))) return rc;
        }
        for (int d = 0; d < n_dm; d++) {
                if (with_j) {
                        const double *J = Jacc + (size_t)d * nc;
                        cart_to_out_kernel<<<grid_for((long long)nn, 256), 256, 0, s>>>(
                                J, J, P->nao, P->naoc, P->out_seg.p, P->out_comp.p, P->seg_info.p, P->c2s.p,
                                P->cart, 1, vj + (size_t)d * nn);
                        CUDA_TRY(cudaGetLastError());
                }
                if (with_k) {
                        const double *K1 = Kacc + (size_t)d * nk * nc;
                        const double *K2 = nk == 2 ? K1 + nc : K1;
                        cart_to_out_kernel<<<grid_for((long long)nn, 256), 256, 0, s>>>(
                                K1, K2, P->nao, P->naoc, P->out_seg.p, P->out_comp.p, P->seg_info.p, P->c2s.p,
                                P->cart, hermi, vk + (size_t)d * nn);
                        CUDA_TRY(cudaGetLastError());
                }
        }
        CUDA_TRY(cudaStreamSynchronize(s));
        return B200JK_OK;
}

// ---------------------------------------------------------------------------
// The s8 two-electron integral tensor (mol.intor('int2e', aosym='s8'),
// GTO2e_cart_or_sph, pyscf/lib/vhf/fill_nr_s8.c:110-138) and J/K from a
// stored tensor (_vhf.incore, pyscf/scf/_vhf.py:318-401).

typedef int (*fill_launcher_t)(int, int, const FillArgs &, cudaStream_t, int, std::string &);
static const fill_launcher_t g_fill_launch[NPAIRCLASS] = {
        launch_fill_00, launch_fill_10, launch_fill_11, launch_fill_20, launch_fill_21,
        launch_fill_22, launch_fill_30, launch_fill_31, launch_fill_32, launch_fill_33};

// pair lists of the fill: every pair that can pass q_ij q_kl > 1e-14 with
// some kl (the plan's own lists drop pairs at its direct_scf_tol)
static int ensure_fill(b200jk_plan *P)
{
        if (P->fill_ready) return B200JK_OK;
        const int nbas = P->nbas;
        double qmax = 0;
        for (double v : P->h_qcond) qmax = std::max(qmax, v);
        size_t maxn = 1;
        int rc;
        for (int X = 0; X < NPAIRCLASS; X++) {
                std::vector<PairLite> hv;
                std::vector<double> q;
                for (const PairLite &p : P->all_pairs[X]) {
                        const double v = P->h_qcond[(size_t)P->segl[p.i].parent * nbas + P->segl[p.j].parent];
                        if (v * qmax > B2_FILL_CUTOFF) { hv.push_back(p); q.push_back(v); }
                }
                // bucket-major, descending bound inside a bucket (the count
                // kernel's prefix search)
                std::vector<size_t> idx(hv.size());
                std::iota(idx.begin(), idx.end(), 0);
                std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
                        const int ba = prim_bucket(hv[a].nprim), bb = prim_bucket(hv[b].nprim);
                        if (ba != bb) return ba < bb;
                        return q[a] > q[b];
                });
                std::vector<PairLite> h2(hv.size());
                std::vector<double> q2(hv.size());
                for (size_t t = 0; t < idx.size(); t++) { h2[t] = hv[idx[t]]; q2[t] = q[idx[t]]; }
                P->fill_pc[X].release();
                if ((rc = upload_pairs(P, P->fill_pc[X], X, h2, q2))) return rc;
                maxn = std::max(maxn, h2.size());
        }
        const size_t nseg = maxn * B2_NBUCKET;
        if ((rc = dev_upload(P->fill_one, std::vector<double>(1, 1.0))) || (rc = dev_alloc(P->fill_nkl, nseg)) ||
            (rc = dev_alloc(P->fill_kst, nseg)) || (rc = dev_alloc(P->fill_nchunk, nseg + 1)) ||
            (rc = dev_alloc(P->fill_chunk_off, nseg + 1)))
                return rc;
        size_t tmp = 0;
        CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp, P->fill_nchunk.p, P->fill_chunk_off.p, (int)nseg + 1));
        if ((rc = dev_alloc(P->fill_cub, std::max<size_t>(tmp, 1)))) return rc;
        P->fill_ready = true;
        return B200JK_OK;
}

int b200jk_int2e_s8(b200jk_plan *P, double *eri, long long len, int dev_ptr, void *stream)
{
        if (!P) return fail(B200JK_EINVAL, "plan is NULL");
        if (!eri) return fail(B200JK_EINVAL, "eri is NULL");
        const long long npair = (long long)P->nao * (P->nao + 1) / 2;
        const long long need = npair * (npair + 1) / 2;
        if (len != need)
                return fail(B200JK_EINVAL, "eri holds " + std::to_string(len) + " entries; the s8 tensor of nao = " +
                                                   std::to_string(P->nao) + " has " + std::to_string(need));
        CUDA_TRY(cudaSetDevice(P->device));
        int rc;
        if (dev_ptr && (rc = check_dev_ptr(eri, P->device, "eri"))) return rc;
        if ((rc = ensure_fill(P))) return rc;
        cudaStream_t s = stream ? (cudaStream_t)stream : P->stream;
        DevArr<double> tmp;
        double *out = eri;
        if (!dev_ptr) {
                if ((rc = dev_alloc(tmp, (size_t)need))) return rc;
                out = tmp.p;
        }
        auto run = [&]() -> int {
                CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double) * need, s));
                auto qcs = quartet_classes();
                for (size_t t = 0; t < qcs.size(); t++) {
                        const PairClassDev &bra = P->fill_pc[qcs[t].X], &ket = P->fill_pc[qcs[t].Y];
                        if (bra.n == 0 || ket.n == 0) continue;
                        const int la = bra.la, lb = bra.lb, lc = ket.la, ld = ket.lb;
                        const int same = qcs[t].X == qcs[t].Y;
                        const int nseg = bra.n * B2_NBUCKET;
                        const int chunk = fill_chunk(la, lb, lc, ld);
                        count_kernel<<<grid_for(nseg, 256), 256, 0, s>>>(
                                bra.view(), ket.view(), same, B2_FILL_CUTOFF, P->fill_one.p, chunk, 0.0, 0, 0, 1,
                                P->fill_nkl.p, P->fill_kst.p, P->fill_nchunk.p);
                        CUDA_TRY(cudaGetLastError());
                        CUDA_TRY(cudaMemsetAsync(P->fill_nchunk.p + nseg, 0, sizeof(long long), s));
                        size_t tb = P->fill_cub.n;
                        CUDA_TRY(cub::DeviceScan::ExclusiveSum(P->fill_cub.p, tb, P->fill_nchunk.p, P->fill_chunk_off.p,
                                                               nseg + 1, s));
                        FillArgs f = FillArgs();
                        JKArgs &a = f.jk;
                        a.tiled = 0;
                        a.bra = bra.view();
                        a.ket = ket.view();
                        a.PP = P->PP.p; a.PK = P->PK.p;
                        a.chunk_off = P->fill_chunk_off.p;
                        a.nkl = P->fill_nkl.p;
                        a.kst = P->fill_kst.p;
                        a.table = table_ptr();
                        a.table_f = table_f_ptr();
                        a.goff = P->goff_all.p + P->goff_at[t];
                        a.tol = B2_FILL_CUTOFF;
                        a.nbas = P->nbas; a.naoc = P->naoc; a.same = same;
                        a.omega2 = P->omega2;
                        f.cart_seg = P->cart_seg.p;
                        f.seg_info = P->seg_info.p;
                        f.c2s = P->c2s.p;
                        f.cart = P->cart;
                        f.eri = out;
                        std::string err;
                        if (g_fill_launch[qcs[t].X](lc, ld, f, s, P->nsm, err)) return fail(B200JK_ECUDA, err);
                }
                if (!dev_ptr) CUDA_TRY(cudaMemcpyAsync(eri, out, sizeof(double) * need, cudaMemcpyDeviceToHost, s));
                CUDA_TRY(cudaStreamSynchronize(s));
                return B200JK_OK;
        };
        rc = run();
        tmp.release();
        return rc;
}

// workspace of the in-core contraction, one per device (calls are serialised)
struct IncoreWS {
        std::mutex mu;
        DevArr<double> A1, A2, Jp, t, Dt, eri, dms, vj, vk;
        DevArr<int4> items;
        std::vector<int4> h_items;     // the fast kernel's four item lists, then the general ones
        int nf[4] = {0, 0, 0, 0};
        int items_nao = -1, items_s8 = -1;
};
static IncoreWS g_incore_ws[64];

int b200jk_incore_jk(const double *eri, long long eri_len, int nao, const double *dms, int n_dm, int hermi,
                     int with_j, int with_k, double *vj, double *vk, int dev_ptrs, int device, void *stream)
{
        if (!eri) return fail(B200JK_EINVAL, "eri is NULL");
        if (nao <= 0) return fail(B200JK_EINVAL, "nao must be positive");
        if (!dms || n_dm <= 0) return fail(B200JK_EINVAL, "no density matrices");
        if (hermi < 0 || hermi > 2) return fail(B200JK_EINVAL, "hermi must be 0, 1 or 2");
        if (with_j && !vj) return fail(B200JK_EINVAL, "vj is NULL while with_j is set");
        if (with_k && !vk) return fail(B200JK_EINVAL, "vk is NULL while with_k is set");
        if (device < 0 || device >= 64) return fail(B200JK_EINVAL, "device index out of range");
        const long long npair = (long long)nao * (nao + 1) / 2;
        int s8;
        if (eri_len == npair * (npair + 1) / 2) s8 = 1;
        else if (eri_len == npair * npair) s8 = 0;
        else
                return fail(B200JK_EINVAL, "Array shape not consistent: eri has " + std::to_string(eri_len) +
                                                   " entries, neither the s8 (" + std::to_string(npair * (npair + 1) / 2) +
                                                   ") nor the s4 (" + std::to_string(npair * npair) +
                                                   ") tensor of nao = " + std::to_string(nao));
        if (incore_block(nao) == 0) return fail(B200JK_EUNSUPPORTED, "nao too large for the in-core contraction");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
                cudaGetLastError();
                return fail(B200JK_ECUDA, "no CUDA device is available");
        }
        if (device >= ndev) return fail(B200JK_EINVAL, "device index out of range");
        CUDA_TRY(cudaSetDevice(device));
        int rc;
        if (dev_ptrs && ((rc = check_dev_ptr(eri, device, "eri")) || (rc = check_dev_ptr(dms, device, "dms")) ||
                         (with_j && (rc = check_dev_ptr(vj, device, "vj"))) ||
                         (with_k && (rc = check_dev_ptr(vk, device, "vk")))))
                return rc;
        if (!with_j && !with_k) return B200JK_OK;
        IncoreWS &W = g_incore_ws[device];
        std::lock_guard<std::mutex> lk(W.mu);
        const size_t nn = (size_t)nao * nao;
        const int twopass = s8 && hermi == 0 && with_k;
        if ((rc = dev_alloc(W.A1, nn)) || (rc = dev_alloc(W.Jp, (size_t)npair)) || (rc = dev_alloc(W.t, (size_t)npair)) ||
            (twopass && ((rc = dev_alloc(W.A2, nn)) || (rc = dev_alloc(W.Dt, nn)))))
                return rc;
        const double *E = eri, *Dd = dms;
        double *oj = vj, *ok = vk;
        cudaStream_t s = stream ? (cudaStream_t)stream : 0;
        if (!dev_ptrs) {
                if ((rc = dev_alloc(W.eri, (size_t)eri_len)) || (rc = dev_alloc(W.dms, nn * n_dm)) ||
                    (with_j && (rc = dev_alloc(W.vj, nn * n_dm))) || (with_k && (rc = dev_alloc(W.vk, nn * n_dm))))
                        return rc;
                CUDA_TRY(cudaMemcpyAsync(W.eri.p, eri, sizeof(double) * eri_len, cudaMemcpyHostToDevice, s));
                CUDA_TRY(cudaMemcpyAsync(W.dms.p, dms, sizeof(double) * nn * n_dm, cudaMemcpyHostToDevice, s));
                E = W.eri.p; Dd = W.dms.p; oj = W.vj.p; ok = W.vk.p;
        }
        const int B = incore_block(nao);
        if (W.items_nao != nao || W.items_s8 != s8) {
                std::vector<int4> fast[4], general;
                incore_items(nao, s8, B, 2048, fast, general);
                W.h_items.clear();
                for (int v = 0; v < 4; v++) {
                        W.nf[v] = (int)fast[v].size();
                        W.h_items.insert(W.h_items.end(), fast[v].begin(), fast[v].end());
                }
                W.h_items.insert(W.h_items.end(), general.begin(), general.end());
                if ((rc = dev_upload(W.items, W.h_items))) return rc;
                W.items_nao = nao;
                W.items_s8 = s8;
        }
        std::string err;
        for (int d = 0; d < n_dm; d++) {
                const double *D = Dd + (size_t)d * nn;
                CUDA_TRY(cudaMemsetAsync(W.A1.p, 0, sizeof(double) * nn, s));
                CUDA_TRY(cudaMemsetAsync(W.Jp.p, 0, sizeof(double) * npair, s));
                if (launch_incore_tridm(D, nao, W.t.p, s, err)) return fail(B200JK_ECUDA, err);
                IncoreArgs a;
                a.eri = E; a.s8 = s8; a.nao = nao; a.npair = npair;
                a.D = D; a.t = W.t.p; a.A = W.A1.p; a.Jp = with_j ? W.Jp.p : nullptr;
                int off = 0;
                for (int v = 0; v < 4; v++) {
                        a.fitems[v] = W.items.p + off;
                        a.nf[v] = W.nf[v];
                        off += W.nf[v];
                }
                a.items = W.items.p + off; a.nitems = (int)W.h_items.size() - off;
                // one read of the tensor gives J and the K images (a J-only
                // call drops the images: the pass is bound by the read)
                if (launch_incore_pass(a, s, err)) return fail(B200JK_ECUDA, err);
                if (twopass) {
                        // the pair-swapped images of a general density: A(D^T)^T
                        CUDA_TRY(cudaMemsetAsync(W.A2.p, 0, sizeof(double) * nn, s));
                        if (launch_incore_transpose(D, nao, W.Dt.p, s, err)) return fail(B200JK_ECUDA, err);
                        IncoreArgs b = a;
                        b.D = W.Dt.p; b.A = W.A2.p; b.Jp = nullptr;
                        if (launch_incore_pass(b, s, err)) return fail(B200JK_ECUDA, err);
                }
                if (with_j && launch_incore_unpack_j(W.Jp.p, nao, oj + (size_t)d * nn, s, err))
                        return fail(B200JK_ECUDA, err);
                if (with_k) {
                        const int mode = !s8 ? 3 : (hermi == 0 ? 0 : (hermi == 1 ? 1 : 2));
                        if (launch_incore_finish_k(W.A1.p, twopass ? W.A2.p : nullptr, nao, mode, hermi,
                                                   ok + (size_t)d * nn, s, err))
                                return fail(B200JK_ECUDA, err);
                }
        }
        if (!dev_ptrs) {
                if (with_j) CUDA_TRY(cudaMemcpyAsync(vj, W.vj.p, sizeof(double) * nn * n_dm, cudaMemcpyDeviceToHost, s));
                if (with_k) CUDA_TRY(cudaMemcpyAsync(vk, W.vk.p, sizeof(double) * nn * n_dm, cudaMemcpyDeviceToHost, s));
        }
        CUDA_TRY(cudaStreamSynchronize(s));
        return B200JK_OK;
}
