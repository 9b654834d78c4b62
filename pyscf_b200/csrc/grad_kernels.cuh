// grad_kernels.cuh — sm_100a kernels of the nuclear-gradient J/K build.
//
// The reference path is pyscf.grad.rhf.get_jk (pyscf/grad/rhf.py:149-178):
//     vj_x[i,j] = -sum_kl (d_x i j|kl) D[l,k],   vk_x[i,l] = -sum_jk (d_x i j|kl) D[j,k]
// over all ordered bra shell pairs (i,j) and ket pairs k >= l ('s2kl'), with
// libcint's int2e_ip1 (derivative of the first bra function) and the screen
// CVHFgrad_jk_prescreen (pyscf/lib/vhf/hessian_screen.c:44-68).
//
// Work decomposition.  Bra pairs are the planner's unordered segment pairs
// (A,B); one evaluation of the quartet (AB|CD) yields both bra derivatives,
// side A = (d A, B|CD) and side B = (A, d B|CD) = the reference's (d B, A|CD),
// so the ordered pairs (i,j) and (j,i) share roots and recurrences.  A pair
// of one segment has side A only.  Ket pairs are the unordered segment pairs
// with both images (CD) and (DC) (weight 1/2 for a pair of one segment), as in
// the energy build.  Classes: every bra class X with every ket class Y.
//
// Arithmetic.  The 2D Rys integrals are built with the bra indices extended by
// one (a <= la+1, b <= lb+1), then per primitive quartet
//     d/dA_x : 2 alpha I_x(a+1, b) - a_x I_x(a-1, b)
//     d/dB_x : 2 beta  I_x(a, b+1) - b_x I_x(a, b-1)
// replace the x factor of the product I_x I_y I_z (alpha, beta the bra
// primitive exponents).  These are derivatives with respect to the centres,
// d/dA = -nabla_r on the function (libcint's ip1 is nabla_r), so the
// accumulated contraction is the negated one grad.rhf.get_jk returns.
// Mode 1 of the same machinery also extends the ket indices and
// differentiates bra and ket together, which gives the diagonal blocks
// (d_x a b|d_x a b) of int2e_ip1ip2 for the derivative Schwarz bound
// (CVHFnr_int2e_pp_q_cond, hessian_screen.c:70-123).
#pragma once
#include "jk_kernels.cuh"

namespace b200jk {

template <int LA, int LB, int LC, int LD, int MODE>
struct GClass {
        using K = Class4<LA, LB, LC, LD>;
        // extended 2D integral dimensions
        static constexpr int EA = LA + 2, EB = LB + 2, EC = LC + 1 + MODE, ED = LD + 1 + MODE;
        static constexpr int SE = EA * EB * EC * ED;
        static constexpr int STEP_A = EB * EC * ED, STEP_B = EC * ED, STEP_C = ED, STEP_D = 1;
        static constexpr int NE = LA + LB + 2, NF = LC + LD + 1 + MODE;
        static constexpr int NR = rys_nroots(LA + LB + LC + LD + 1 + MODE);
        static constexpr int NG = K::NG;
        // derivative components: side A x,y,z then side B x,y,z; NCP of them
        // are accumulated per pass over the primitives (all six when they fit)
        static constexpr int NCP = 6 * NG <= 8192 ? 6 : (3 * NG <= 8192 ? 3 : 1);
        static constexpr int NPASS = 6 / NCP;
        B2_HD static constexpr int eidx(int a, int b, int c, int d) { return ((a * EB + b) * EC + c) * ED + d; }
};

// shared-memory layout of one group (doubles); WONLY: the fused force
// contraction, whose G area holds the NG weights instead of NCP blocks
template <int LA, int LB, int LC, int LD, int MODE, bool WONLY = false>
struct GradSmem {
        using GC = GClass<LA, LB, LC, LD, MODE>;
        using K = Class4<LA, LB, LC, LD>;
        static constexpr int G = 0;                                  // [NCP][NG] (WONLY: [NG])
        static constexpr int E = G + (WONLY ? 1 : GC::NCP) * GC::NG; // [3][NR][SE]
        static constexpr int DSAB = E + 3 * GC::NR * GC::SE;
        static constexpr int DSCD = DSAB + K::NAB;
        static constexpr int XBC = DSCD + K::NCD;
        static constexpr int XBD = XBC + K::NB * K::NC;
        static constexpr int XAC = XBD + K::NB * K::ND;
        static constexpr int XAD = XAC + K::NA * K::NC;
        static constexpr int SIZE = ((XAD + K::NA * K::ND) + 3) & ~3;
};

// One (root, direction) slice of the extended 2D integrals:
// h[((a*EB + b)*EC + c)*ED + d] for a < EA, b < EB, c < EC, d < ED with
// a + b < NE and c + d < NF (the other entries are never read).
template <int LA, int LB, int LC, int LD, int MODE>
__device__ __forceinline__ void grad_slice(double *h, double g00, const RysCoef<double> &rc, int dir, double ab,
                                           double cd)
{
        using GC = GClass<LA, LB, LC, LD, MODE>;
        constexpr int NE = GC::NE, NF = GC::NF, EA = GC::EA, EB = GC::EB, EC = GC::EC, ED = GC::ED;
        double g[NE * NF];
        const double c00 = dir == 0 ? rc.c00[0] : (dir == 1 ? rc.c00[1] : rc.c00[2]);
        const double c00p = dir == 0 ? rc.c00p[0] : (dir == 1 ? rc.c00p[1] : rc.c00p[2]);
        vrr2d<NE, NF, double>(g, g00, c00, c00p, rc.b10, rc.b01, rc.b00);
        constexpr int NCD1 = EC * ED;
        double u[NE * NCD1];
        double cdp[ED];
        cdp[0] = 1.0;
#pragma unroll
        for (int k = 1; k < ED; k++) cdp[k] = cdp[k - 1] * cd;
#pragma unroll
        for (int e = 0; e < NE; e++)
#pragma unroll
        for (int c = 0; c < EC; c++)
#pragma unroll
        for (int d = 0; d < ED; d++) {
                double v = 0.0;
                if (c + d < NF) {
#pragma unroll
                        for (int k = 0; k <= d; k++) v += (double)binom(d, k) * cdp[d - k] * g[e * NF + c + k];
                }
                u[e * NCD1 + c * ED + d] = v;
        }
        double abp[EB];
        abp[0] = 1.0;
#pragma unroll
        for (int k = 1; k < EB; k++) abp[k] = abp[k - 1] * ab;
#pragma unroll
        for (int a = 0; a < EA; a++)
#pragma unroll
        for (int b = 0; b < EB; b++)
#pragma unroll
        for (int t = 0; t < NCD1; t++) {
                double v = 0.0;
                if (a + b < NE) {
#pragma unroll
                        for (int k = 0; k <= b; k++) v += (double)binom(b, k) * abp[b - k] * u[(a + k) * NCD1 + t];
                }
                h[(a * EB + b) * NCD1 + t] = v;
        }
}

// Per Cartesian component of a class, packed by the planner:
//   x: extended offsets ox | oy << 10 | oz << 20
//   y: exponents of a, b, c, d, 6 bits each (x | y << 2 | z << 4)
__device__ __forceinline__ int gexp(int packed, int fn, int dir) { return (packed >> (6 * fn + 2 * dir)) & 3; }

struct GradArgs {
        PairView bra, ket;
        const double4 *PP;           // primitive pair (P, p)
        const double2 *PK;           // primitive pair (K_ab c_i c_j, 1/(2p))
        const double2 *PE;           // primitive pair exponents (alpha of A, beta of B)
        const long long *chunk_off;
        const int *nkl, *kst;
        const double *q0;            // nbas x nbas derivative Schwarz bound (ordered, derivative on the row shell)
        const double *q1;            // nbas x nbas Schwarz bound
        const double *dmc;           // nbas x nbas max |D| per block (not symmetrised)
        const double *table;
        const int2 *goff;
        double *Vj, *Vk;             // [n_dm][3][naoc][naoc] Cartesian accumulators
        const double *Ds, *Dc;       // [n_dm][naoc][naoc]: D + D^T and D (Cartesian)
        unsigned long long *stats;   // [0] quartets (sides), [1] primitive quartets
        double tol;
        int nbas, naoc, n_dm, with_j, with_k;
        // fused force contraction (b200jk_grad_contract): de[atom][x] of the
        // parent shells' atoms (shell_atom[parent shell]); one symmetric density
        double *de = nullptr;
        const int *shell_atom = nullptr;
        // omega^2 of the long-range operator erf(omega r12)/r12, 0 = Coulomb
        double omega2 = 0.0;
};

// Weight of one Cartesian element (ab|cd) in the two-electron force of a
// symmetric density D (Cartesian, Ds = D + D^T): grad_elec adds
// 2 sum_{i in A} sum_j (vj - vk/2)_x[i,j] D[i,j] (pyscf/grad/rhf.py:62-68), which
// per quartet side is sum_abcd (d_x ab|cd) W[abcd] with
//     W = 2 D_ab Ds_cd - D_bc D_ad - D_bd D_ac
// for the derivative on a and, D being symmetric, the same W for b.
__device__ __forceinline__ double grad_force_weight(double dab, double dcd, double xbc, double xad, double xbd,
                                                    double xac)
{
        return 2.0 * dab * dcd - xbc * xad - xbd * xac;
}

// the per-lane side sums s[0..2] (derivative on a) and s[3..5] (on b) of a
// warp that worked on one bra pair: summed over the warp, one atomic per
// atom and direction
__device__ __forceinline__ void grad_force_flush(const GradArgs &a, int4 sb, double s[6], int lane)
{
#pragma unroll
        for (int q = 0; q < 6; q++) s[q] = warp_sum(s[q]);
        if (lane == 0) {
                const int atA = __ldg(a.shell_atom + sb.z), atB = __ldg(a.shell_atom + sb.w);
#pragma unroll
                for (int x = 0; x < 3; x++) {
                        if (s[x] != 0.0) atomicAdd(a.de + 3 * atA + x, s[x]);
                        if (s[3 + x] != 0.0) atomicAdd(a.de + 3 * atB + x, s[3 + x]);
                }
        }
}

// CVHFgrad_jk_prescreen for bra shells (i, j) (derivative on i) and ket
// shells k >= l
__device__ __forceinline__ bool grad_side_passes(const GradArgs &a, int i, int j, int k, int l)
{
        const size_t n = (size_t)a.nbas;
        const double qq = __ldg(a.q0 + i * n + j) * __ldg(a.q1 + k * n + l);
        if (!(qq > a.tol)) return false;
        const double dmin = a.tol / qq;
        return 2 * __ldg(a.dmc + l * n + k) > dmin || __ldg(a.dmc + j * n + k) > dmin || __ldg(a.dmc + j * n + l) > dmin;
}

// Accumulate derivative components [c0, c0 + GC::NCP) of one quartet into G.
// Mode 0: components 0..2 = d/dA_{x,y,z}, 3..5 = d/dB_{x,y,z}.  Mode 1 (bra =
// ket pair): components 0..2 = d/dA_x d/dC_x (same x), 3..5 = d/dB_x d/dD_x.
// P and Q are taken relative to the origin O; A = 0, C relative to O.
template <int LA, int LB, int LC, int LD, int MODE, int GS>
__device__ __forceinline__ void grad_eval_pass(double *sm, const GradArgs &a, int2 pb, int2 pk, const double4 O,
                                               const double AB[3], const double C[3], const double CD[3], double fac,
                                               int c0, int gl, unsigned gmask)
{
        using GC = GClass<LA, LB, LC, LD, MODE>;
        using S = GradSmem<LA, LB, LC, LD, MODE>;
        constexpr int NR = GC::NR, SE = GC::SE, NG = GC::NG, NCP = GC::NCP;
        double *G = sm + S::G;
        double *E = sm + S::E;
        const double *table = a.table + rys_padded_offset(NR);
        const double A[3] = {0.0, 0.0, 0.0};
        for (int t = gl; t < NCP * NG; t += GS) G[t] = 0.0;
        for (int ip = 0; ip < pb.y; ip++) {
                const double4 P = a.PP[pb.x + ip];
                const double2 KP = a.PK[pb.x + ip];
                const double2 EP = a.PE[pb.x + ip];
                const double Kab = KP.x * fac;
                const double Pv[3] = {P.x - O.x, P.y - O.y, P.z - O.z};
                const double ta = 2.0 * EP.x, tb = 2.0 * EP.y;
                for (int kp = 0; kp < pk.y; kp++) {
                        const double4 Q = a.PP[pk.x + kp];
                        const double2 KQ = a.PK[pk.x + kp];
                        const double2 EQ = a.PE[pk.x + kp];
                        const double Qv[3] = {Q.x - O.x, Q.y - O.y, Q.z - O.z};
                        const double tc = 2.0 * EQ.x, td = 2.0 * EQ.y;
                        __syncwarp(gmask);
                        for (int task = gl; task < 3 * NR; task += GS) {
                                const int r = task / 3, dir = task - 3 * r;
                                PrimQ<double> sq;
                                prim_setup<double>(sq, P.w, KP.y, Pv, Q.w, KQ.y, Qv, A, C, Kab * KQ.x, a.omega2);
                                double ur, wr;
                                rys_root_one<NR, double>(sq.T, table, r, ur, wr);
                                RysCoef<double> rc;
                                rys_coef<double>(rc, ur, sq);
                                const double g00 = dir == 2 ? sq.pref * wr : 1.0;
                                const double abx = dir == 0 ? AB[0] : (dir == 1 ? AB[1] : AB[2]);
                                const double cdx = dir == 0 ? CD[0] : (dir == 1 ? CD[1] : CD[2]);
                                grad_slice<LA, LB, LC, LD, MODE>(E + (dir * NR + r) * SE, g00, rc, dir, abx, cdx);
                        }
                        __syncwarp(gmask);
                        for (int t = gl; t < NG; t += GS) {
                                const int2 o = __ldg(a.goff + t);
                                const int oo[3] = {o.x & 1023, (o.x >> 10) & 1023, o.x >> 20};
                                for (int cc = 0; cc < NCP; cc++) {
                                        const int comp = c0 + cc;
                                        const int side = comp / 3, dir = comp - 3 * side;
                                        const int d1 = dir == 0 ? 1 : 0, d2 = dir == 2 ? 1 : 2;
                                        const int od = oo[dir], o1 = oo[d1], o2 = oo[d2];
                                        double v = 0.0;
                                        if (MODE == 0) {
                                                const int n = gexp(o.y, side, dir);   // a_x (side A) or b_x (side B)
                                                const int st = side == 0 ? GC::STEP_A : GC::STEP_B;
                                                const double tw = side == 0 ? ta : tb;
                                                for (int r = 0; r < NR; r++) {
                                                        const double *Ed = E + (dir * NR + r) * SE;
                                                        double dv = tw * Ed[od + st];
                                                        if (n) dv -= n * Ed[od - st];
                                                        v += dv * E[(d1 * NR + r) * SE + o1] * E[(d2 * NR + r) * SE + o2];
                                                }
                                        } else {
                                                // bra function (a or b) and its ket partner (c or d)
                                                const int n1 = gexp(o.y, side, dir), n2 = gexp(o.y, 2 + side, dir);
                                                const int s1 = side == 0 ? GC::STEP_A : GC::STEP_B;
                                                const int s2 = side == 0 ? GC::STEP_C : GC::STEP_D;
                                                const double w1 = side == 0 ? ta : tb, w2 = side == 0 ? tc : td;
                                                for (int r = 0; r < NR; r++) {
                                                        const double *Ed = E + (dir * NR + r) * SE;
                                                        double dv = w1 * w2 * Ed[od + s1 + s2];
                                                        if (n2) dv -= w1 * n2 * Ed[od + s1 - s2];
                                                        if (n1) dv -= n1 * w2 * Ed[od - s1 + s2];
                                                        if (n1 && n2) dv += n1 * n2 * Ed[od - s1 - s2];
                                                        v += dv * E[(d1 * NR + r) * SE + o1] * E[(d2 * NR + r) * SE + o2];
                                                }
                                        }
                                        G[cc * NG + t] += v;
                                }
                        }
                }
        }
        __syncwarp(gmask);
}

// The fused force contraction's pass of the shared-memory family: instead
// of building NCP derivative blocks in shared memory and contracting them
// afterwards, each lane assembles all six derivative components of its
// Cartesian components straight into fq[6] with the quartet's weights w
// (shared memory, NG doubles): no block to clear or update, one pass.
template <int LA, int LB, int LC, int LD, int GS>
__device__ __forceinline__ void grad_eval_force(double *sm, const GradArgs &a, int2 pb, int2 pk, const double4 O,
                                                const double AB[3], const double C[3], const double CD[3],
                                                double fac, const double *w, int gl, unsigned gmask, double fq[6])
{
        using GC = GClass<LA, LB, LC, LD, 0>;
        using S = GradSmem<LA, LB, LC, LD, 0, true>;
        constexpr int NR = GC::NR, SE = GC::SE, NG = GC::NG;
        constexpr int SA = GC::STEP_A, SB = GC::STEP_B;
        double *E = sm + S::E;
        const double *table = a.table + rys_padded_offset(NR);
        const double A[3] = {0.0, 0.0, 0.0};
        for (int ip = 0; ip < pb.y; ip++) {
                const double4 P = a.PP[pb.x + ip];
                const double2 KP = a.PK[pb.x + ip];
                const double2 EP = a.PE[pb.x + ip];
                const double Kab = KP.x * fac;
                const double Pv[3] = {P.x - O.x, P.y - O.y, P.z - O.z};
                const double ta = 2.0 * EP.x, tb = 2.0 * EP.y;
                for (int kp = 0; kp < pk.y; kp++) {
                        const double4 Q = a.PP[pk.x + kp];
                        const double2 KQ = a.PK[pk.x + kp];
                        const double Qv[3] = {Q.x - O.x, Q.y - O.y, Q.z - O.z};
                        __syncwarp(gmask);
                        for (int task = gl; task < 3 * NR; task += GS) {
                                const int r = task / 3, dir = task - 3 * r;
                                PrimQ<double> sq;
                                prim_setup<double>(sq, P.w, KP.y, Pv, Q.w, KQ.y, Qv, A, C, Kab * KQ.x, a.omega2);
                                double ur, wr;
                                rys_root_one<NR, double>(sq.T, table, r, ur, wr);
                                RysCoef<double> rc;
                                rys_coef<double>(rc, ur, sq);
                                const double g00 = dir == 2 ? sq.pref * wr : 1.0;
                                const double abx = dir == 0 ? AB[0] : (dir == 1 ? AB[1] : AB[2]);
                                const double cdx = dir == 0 ? CD[0] : (dir == 1 ? CD[1] : CD[2]);
                                grad_slice<LA, LB, LC, LD, 0>(E + (dir * NR + r) * SE, g00, rc, dir, abx, cdx);
                        }
                        __syncwarp(gmask);
                        for (int t = gl; t < NG; t += GS) {
                                const int2 o = __ldg(a.goff + t);
                                const int ox = o.x & 1023, oy = (o.x >> 10) & 1023, oz = o.x >> 20;
                                const int axn = gexp(o.y, 0, 0), ayn = gexp(o.y, 0, 1), azn = gexp(o.y, 0, 2);
                                const int bxn = gexp(o.y, 1, 0), byn = gexp(o.y, 1, 1), bzn = gexp(o.y, 1, 2);
                                const double wt = w[t];
                                double f[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
                                for (int r = 0; r < NR; r++) {
                                        const double *Ex = E + r * SE, *Ey = E + (NR + r) * SE, *Ez = E + (2 * NR + r) * SE;
                                        const double ex = Ex[ox], ey = Ey[oy], ez = Ez[oz];
                                        double dax = ta * Ex[ox + SA], day = ta * Ey[oy + SA], daz = ta * Ez[oz + SA];
                                        if (axn) dax -= axn * Ex[ox - SA];
                                        if (ayn) day -= ayn * Ey[oy - SA];
                                        if (azn) daz -= azn * Ez[oz - SA];
                                        double dbx = tb * Ex[ox + SB], dby = tb * Ey[oy + SB], dbz = tb * Ez[oz + SB];
                                        if (bxn) dbx -= bxn * Ex[ox - SB];
                                        if (byn) dby -= byn * Ey[oy - SB];
                                        if (bzn) dbz -= bzn * Ez[oz - SB];
                                        const double eyz = ey * ez, exz = ex * ez, exy = ex * ey;
                                        f[0] += dax * eyz;
                                        f[1] += day * exz;
                                        f[2] += daz * exy;
                                        f[3] += dbx * eyz;
                                        f[4] += dby * exz;
                                        f[5] += dbz * exy;
                                }
#pragma unroll
                                for (int q = 0; q < 6; q++) fq[q] += wt * f[q];
                        }
                }
        }
        __syncwarp(gmask);
}

template <int LA, int LB, int LC, int LD>
__host__ __device__ constexpr int grad_group_size()
{
        using K = Class4<LA, LB, LC, LD>;
        return K::NG <= 100 ? 8 : (K::NG <= 400 ? 16 : 32);
}

// The gradient J/K kernel of class (LA LB | LC LD): groups of GS lanes walk
// chunks of chunk_q quartets of one bra pair.
// FUSED: the force contraction with one symmetric density instead of the
// vj/vk accumulators (b200jk_grad_contract).
template <int LA, int LB, int LC, int LD, bool FUSED = false>
__global__ void __launch_bounds__(128) grad_jk_kernel(GradArgs a, int chunk_q)
{
        using K = Class4<LA, LB, LC, LD>;
        using GC = GClass<LA, LB, LC, LD, 0>;
        using S = GradSmem<LA, LB, LC, LD, 0, FUSED>;
        constexpr int GS = grad_group_size<LA, LB, LC, LD>();
        constexpr int NGRP = 32 / GS;
        constexpr int NG = K::NG;
        extern __shared__ __align__(32) double smem_dyn[];
        const int lane = threadIdx.x & 31;
        const int grp = lane / GS, gl = lane % GS;
        const unsigned gmask = GS == 32 ? 0xffffffffu : (((1u << GS) - 1u) << (grp * GS));
        const int wib = threadIdx.x >> 5;
        double *sm = smem_dyn + (size_t)(wib * NGRP + grp) * S::SIZE;
        const int nseg = a.bra.n * B2_NBUCKET;
        const long long total = a.chunk_off[nseg];
        const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
        const size_t n = (size_t)a.naoc, nn = n * n;
        unsigned long long nq = 0, npq = 0;
        for (long long chunk = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; chunk < total;
             chunk += nwarps) {
                const int sgi = find_bra(a.chunk_off, nseg, chunk);
                const int ij = sgi / B2_NBUCKET;
                const int kb = a.ket.boff[sgi % B2_NBUCKET] + a.kst[sgi];
                const int kl0 = kb + (int)(chunk - a.chunk_off[sgi]) * chunk_q;
                const int kl1 = kb + min((int)(chunk - a.chunk_off[sgi]) * chunk_q + chunk_q, a.nkl[sgi]);
                const int4 sb = a.bra.sh[ij];
                const int2 pb = a.bra.pr[ij];
                const double4 Ab = a.bra.A[ij];
                const double4 ABb = a.bra.AB[ij];
                const double AB[3] = {ABb.x, ABb.y, ABb.z};
                const int ia = sb.x, ib = sb.y;
                const bool bra_one_segment = Ab.w != 0.0;
                double fs[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                for (int kl = kl0 + grp; kl < kl1; kl += NGRP) {
                        const int4 sk = a.ket.sh[kl];
                        const int kk = max(sk.z, sk.w), ll = min(sk.z, sk.w);
                        const bool sideA = grad_side_passes(a, sb.z, sb.w, kk, ll);
                        const bool sideB = !bra_one_segment && grad_side_passes(a, sb.w, sb.z, kk, ll);
                        if (!sideA && !sideB) continue;
                        const int2 pk = a.ket.pr[kl];
                        const double4 Ak = a.ket.A[kl];
                        const double4 CDk = a.ket.AB[kl];
                        const double fac = Ak.w != 0.0 ? 0.5 : 1.0;
                        const double C[3] = {Ak.x - Ab.x, Ak.y - Ab.y, Ak.z - Ab.z};
                        const double CD[3] = {CDk.x, CDk.y, CDk.z};
                        if (gl == 0) {
                                nq += (unsigned long long)sideA + (unsigned long long)sideB;
                                npq += (unsigned long long)pb.y * pk.y;
                        }
                        const int ic = sk.x, id = sk.y;
                        if constexpr (FUSED) {
                                // weights of the quartet's elements into the G area, then one
                                // pass assembling all six derivative sums from them
                                const double *X = a.Dc;
                                double *w = sm + S::G;
                                double *dsab = sm + S::DSAB, *dscd = sm + S::DSCD;
                                double *xbc = sm + S::XBC, *xbd = sm + S::XBD;
                                double *xac = sm + S::XAC, *xad = sm + S::XAD;
                                for (int t = gl; t < K::NAB; t += GS) dsab[t] = __ldg(X + (ia + t / K::NB) * n + ib + t % K::NB);
                                for (int t = gl; t < K::NCD; t += GS) dscd[t] = __ldg(a.Ds + (ic + t / K::ND) * n + id + t % K::ND);
                                for (int t = gl; t < K::NB * K::NC; t += GS) xbc[t] = __ldg(X + (ib + t / K::NC) * n + ic + t % K::NC);
                                for (int t = gl; t < K::NB * K::ND; t += GS) xbd[t] = __ldg(X + (ib + t / K::ND) * n + id + t % K::ND);
                                for (int t = gl; t < K::NA * K::NC; t += GS) xac[t] = __ldg(X + (ia + t / K::NC) * n + ic + t % K::NC);
                                for (int t = gl; t < K::NA * K::ND; t += GS) xad[t] = __ldg(X + (ia + t / K::ND) * n + id + t % K::ND);
                                __syncwarp(gmask);
                                for (int t = gl; t < NG; t += GS) {
                                        const int d = t % K::ND, c = (t / K::ND) % K::NC;
                                        const int b = (t / K::NCD) % K::NB, xa = t / (K::NCD * K::NB);
                                        w[t] = grad_force_weight(dsab[xa * K::NB + b], dscd[c * K::ND + d], xbc[b * K::NC + c],
                                                                 xad[xa * K::ND + d], xbd[b * K::ND + d], xac[xa * K::NC + c]);
                                }
                                __syncwarp(gmask);
                                double fq[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                                grad_eval_force<LA, LB, LC, LD, GS>(sm, a, pb, pk, Ab, AB, C, CD, fac, w, gl, gmask, fq);
#pragma unroll
                                for (int q = 0; q < 6; q++)
                                        if (q < 3 ? sideA : sideB) fs[q] += fq[q];
                                continue;
                        }
                        // (the fused contraction never gets here: its group holds no blocks)
                        for (int pass = 0; pass < (FUSED ? 0 : GC::NPASS); pass++) {
                                const int c0 = pass * GC::NCP;
                                // skip a pass whose components all belong to a failing side
                                const bool needA = sideA && c0 < 3, needB = sideB && c0 + GC::NCP > 3;
                                if (!needA && !needB) continue;
                                grad_eval_pass<LA, LB, LC, LD, 0, GS>(sm, a, pb, pk, Ab, AB, C, CD, fac, c0, gl, gmask);
                                const double *G = sm + S::G;
                                for (int s = 0; s < a.n_dm; s++) {
                                        const double *Ds = a.Ds + s * nn;
                                        const double *X = a.Dc + s * nn;
                                        double *dsab = sm + S::DSAB, *dscd = sm + S::DSCD;
                                        double *xbc = sm + S::XBC, *xbd = sm + S::XBD;
                                        double *xac = sm + S::XAC, *xad = sm + S::XAD;
                                        for (int t = gl; t < K::NCD; t += GS) dscd[t] = __ldg(Ds + (ic + t / K::ND) * n + id + t % K::ND);
                                        for (int t = gl; t < K::NB * K::NC; t += GS) xbc[t] = __ldg(X + (ib + t / K::NC) * n + ic + t % K::NC);
                                        for (int t = gl; t < K::NB * K::ND; t += GS) xbd[t] = __ldg(X + (ib + t / K::ND) * n + id + t % K::ND);
                                        for (int t = gl; t < K::NA * K::NC; t += GS) xac[t] = __ldg(X + (ia + t / K::NC) * n + ic + t % K::NC);
                                        for (int t = gl; t < K::NA * K::ND; t += GS) xad[t] = __ldg(X + (ia + t / K::ND) * n + id + t % K::ND);
                                        (void)dsab;
                                        __syncwarp(gmask);
                                        for (int cc = 0; cc < GC::NCP; cc++) {
                                                const int comp = c0 + cc;
                                                const int side = comp / 3, x = comp - 3 * side;
                                                if (side == 0 ? !sideA : !sideB) continue;
                                                const double *Gc = G + cc * NG;
                                                double *Vj = a.Vj + ((size_t)s * 3 + x) * nn;
                                                double *Vk = a.Vk + ((size_t)s * 3 + x) * nn;
                                                if (a.with_j) {
                                                        // side A: Vj[a,b];  side B: Vj[b,a]
                                                        for (int t = gl; t < K::NAB; t += GS) {
                                                                double v = 0.0;
                                                                for (int u = 0; u < K::NCD; u++) v += Gc[t * K::NCD + u] * dscd[u];
                                                                const int xa = t / K::NB, yb = t % K::NB;
                                                                if (side == 0) atomicAdd(Vj + (ia + xa) * n + ib + yb, v);
                                                                else atomicAdd(Vj + (ib + yb) * n + ia + xa, v);
                                                        }
                                                }
                                                if (a.with_k) {
                                                        if (side == 0) {
                                                                // Vk[a,d] += G X[b,c];  Vk[a,c] += G X[b,d]
                                                                for (int t = gl; t < K::NA * K::ND; t += GS) {
                                                                        const int xa = t / K::ND, d = t % K::ND;
                                                                        double v = 0.0;
                                                                        for (int b = 0; b < K::NB; b++)
                                                                                for (int c = 0; c < K::NC; c++)
                                                                                        v += Gc[((xa * K::NB + b) * K::NC + c) * K::ND + d] * xbc[b * K::NC + c];
                                                                        atomicAdd(Vk + (ia + xa) * n + id + d, v);
                                                                }
                                                                for (int t = gl; t < K::NA * K::NC; t += GS) {
                                                                        const int xa = t / K::NC, c = t % K::NC;
                                                                        double v = 0.0;
                                                                        for (int b = 0; b < K::NB; b++)
                                                                                for (int d = 0; d < K::ND; d++)
                                                                                        v += Gc[((xa * K::NB + b) * K::NC + c) * K::ND + d] * xbd[b * K::ND + d];
                                                                        atomicAdd(Vk + (ia + xa) * n + ic + c, v);
                                                                }
                                                        } else {
                                                                // Vk[b,d] += G X[a,c];  Vk[b,c] += G X[a,d]
                                                                for (int t = gl; t < K::NB * K::ND; t += GS) {
                                                                        const int b = t / K::ND, d = t % K::ND;
                                                                        double v = 0.0;
                                                                        for (int xa = 0; xa < K::NA; xa++)
                                                                                for (int c = 0; c < K::NC; c++)
                                                                                        v += Gc[((xa * K::NB + b) * K::NC + c) * K::ND + d] * xac[xa * K::NC + c];
                                                                        atomicAdd(Vk + (ib + b) * n + id + d, v);
                                                                }
                                                                for (int t = gl; t < K::NB * K::NC; t += GS) {
                                                                        const int b = t / K::NC, c = t % K::NC;
                                                                        double v = 0.0;
                                                                        for (int xa = 0; xa < K::NA; xa++)
                                                                                for (int d = 0; d < K::ND; d++)
                                                                                        v += Gc[((xa * K::NB + b) * K::NC + c) * K::ND + d] * xad[xa * K::ND + d];
                                                                        atomicAdd(Vk + (ib + b) * n + ic + c, v);
                                                                }
                                                        }
                                                }
                                        }
                                        __syncwarp(gmask);
                                }
                        }
                }
                if constexpr (FUSED) grad_force_flush(a, sb, fs, lane);
        }
        if (a.stats && gl == 0 && nq) {
                atomicAdd(a.stats + 0, nq);
                atomicAdd(a.stats + 1, npq);
        }
}

// ---------------------------------------------------------------------------
// Register family of the gradient for small classes: one ket per lane, the
// six derivative blocks in registers, assembly offsets at compile time.

template <int LA, int LB, int LC, int LD>
__host__ __device__ constexpr bool grad_thread_family()
{
        using GC = GClass<LA, LB, LC, LD, 0>;
        return 6 * GC::NG + 3 * GC::SE <= 104;
}

// component T of the block: G[c*NG + T] += (derivative c of) I_x I_y I_z
template <int LA, int LB, int LC, int LD, int T>
__device__ __forceinline__ void grad_assemble_one(double *G, const double *Ex, const double *Ey, const double *Ez,
                                                  double ta, double tb)
{
        using K = Class4<LA, LB, LC, LD>;
        using GC = GClass<LA, LB, LC, LD, 0>;
        constexpr int NG = K::NG;
        constexpr int id = T % K::ND, ic = (T / K::ND) % K::NC, ib = (T / K::NCD) % K::NB, ia = T / (K::NCD * K::NB);
        constexpr int ax = cart_lx(LA, ia), ay = cart_ly(LA, ia), az = cart_lz(LA, ia);
        constexpr int bx = cart_lx(LB, ib), by = cart_ly(LB, ib), bz = cart_lz(LB, ib);
        constexpr int ox = GC::eidx(ax, bx, cart_lx(LC, ic), cart_lx(LD, id));
        constexpr int oy = GC::eidx(ay, by, cart_ly(LC, ic), cart_ly(LD, id));
        constexpr int oz = GC::eidx(az, bz, cart_lz(LC, ic), cart_lz(LD, id));
        constexpr int SA = GC::STEP_A, SB = GC::STEP_B;
        const double ex = Ex[ox], ey = Ey[oy], ez = Ez[oz];
        double dax = ta * Ex[ox + SA], day = ta * Ey[oy + SA], daz = ta * Ez[oz + SA];
        if constexpr (ax > 0) dax -= ax * Ex[ox - SA];
        if constexpr (ay > 0) day -= ay * Ey[oy - SA];
        if constexpr (az > 0) daz -= az * Ez[oz - SA];
        double dbx = tb * Ex[ox + SB], dby = tb * Ey[oy + SB], dbz = tb * Ez[oz + SB];
        if constexpr (bx > 0) dbx -= bx * Ex[ox - SB];
        if constexpr (by > 0) dby -= by * Ey[oy - SB];
        if constexpr (bz > 0) dbz -= bz * Ez[oz - SB];
        G[0 * NG + T] += dax * ey * ez;
        G[1 * NG + T] += ex * day * ez;
        G[2 * NG + T] += ex * ey * daz;
        G[3 * NG + T] += dbx * ey * ez;
        G[4 * NG + T] += ex * dby * ez;
        G[5 * NG + T] += ex * ey * dbz;
}

template <int LA, int LB, int LC, int LD, int... Ts>
__device__ __forceinline__ void grad_assemble(double *G, const double *Ex, const double *Ey, const double *Ez,
                                              double ta, double tb, std::integer_sequence<int, Ts...>)
{
        (grad_assemble_one<LA, LB, LC, LD, Ts>(G, Ex, Ey, Ez, ta, tb), ...);
}

template <int LA, int LB, int LC, int LD, bool FUSED = false>
__global__ void __launch_bounds__(128) grad_thread_kernel(GradArgs a)
{
        using K = Class4<LA, LB, LC, LD>;
        using GC = GClass<LA, LB, LC, LD, 0>;
        constexpr int NG = K::NG, NR = GC::NR, SE = GC::SE;
        const int lane = threadIdx.x & 31;
        const int nseg = a.bra.n * B2_NBUCKET;
        const long long total = a.chunk_off[nseg];
        const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
        const size_t n = (size_t)a.naoc, nn = n * n;
        const double *table = a.table + rys_padded_offset(NR);
        unsigned long long nq = 0, npq = 0;
        for (long long chunk = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; chunk < total;
             chunk += nwarps) {
                const int sgi = find_bra(a.chunk_off, nseg, chunk);
                const int ij = sgi / B2_NBUCKET;
                const int pos = (int)(chunk - a.chunk_off[sgi]) * 32 + lane;
                const int kl = a.ket.boff[sgi % B2_NBUCKET] + a.kst[sgi] + pos;
                const int4 sb = a.bra.sh[ij];
                const int2 pb = a.bra.pr[ij];
                const double4 Ab = a.bra.A[ij];
                const double4 ABb = a.bra.AB[ij];
                const double AB[3] = {ABb.x, ABb.y, ABb.z};
                int4 sk = make_int4(0, 0, 0, 0);
                bool sideA = false, sideB = false;
                if (pos < a.nkl[sgi]) {
                        sk = a.ket.sh[kl];
                        const int kk = max(sk.z, sk.w), ll = min(sk.z, sk.w);
                        sideA = grad_side_passes(a, sb.z, sb.w, kk, ll);
                        sideB = Ab.w == 0.0 && grad_side_passes(a, sb.w, sb.z, kk, ll);
                }
                const bool active = sideA || sideB;
                double G[6 * NG];
#pragma unroll
                for (int t = 0; t < 6 * NG; t++) G[t] = 0.0;
                if (active) {
                        const int2 pk = a.ket.pr[kl];
                        const double4 Ak = a.ket.A[kl];
                        const double4 CDk = a.ket.AB[kl];
                        const double fac = Ak.w != 0.0 ? 0.5 : 1.0;
                        const double A0[3] = {0.0, 0.0, 0.0};
                        const double C[3] = {Ak.x - Ab.x, Ak.y - Ab.y, Ak.z - Ab.z};
                        const double CD[3] = {CDk.x, CDk.y, CDk.z};
                        nq += (unsigned long long)sideA + (unsigned long long)sideB;
                        npq += (unsigned long long)pb.y * pk.y;
                        for (int ip = 0; ip < pb.y; ip++) {
                                const double4 P = a.PP[pb.x + ip];
                                const double2 KP = a.PK[pb.x + ip];
                                const double2 EP = a.PE[pb.x + ip];
                                const double Kab = KP.x * fac;
                                const double Pv[3] = {P.x - Ab.x, P.y - Ab.y, P.z - Ab.z};
                                const double ta = 2.0 * EP.x, tb = 2.0 * EP.y;
                                for (int kp = 0; kp < pk.y; kp++) {
                                        const double4 Q = a.PP[pk.x + kp];
                                        const double2 KQ = a.PK[pk.x + kp];
                                        const double Qv[3] = {Q.x - Ab.x, Q.y - Ab.y, Q.z - Ab.z};
                                        PrimQ<double> sq;
                                        prim_setup<double>(sq, P.w, KP.y, Pv, Q.w, KQ.y, Qv, A0, C, Kab * KQ.x, a.omega2);
                                        double u[NR], w[NR];
                                        rys_roots_slice<NR, double>(sq.T, table, u, w);
#pragma unroll
                                        for (int r = 0; r < NR; r++) {
                                                RysCoef<double> rc;
                                                rys_coef<double>(rc, u[r], sq);
                                                double Ex[SE], Ey[SE], Ez[SE];
                                                grad_slice<LA, LB, LC, LD, 0>(Ex, 1.0, rc, 0, AB[0], CD[0]);
                                                grad_slice<LA, LB, LC, LD, 0>(Ey, 1.0, rc, 1, AB[1], CD[1]);
                                                grad_slice<LA, LB, LC, LD, 0>(Ez, sq.pref * w[r], rc, 2, AB[2], CD[2]);
                                                grad_assemble<LA, LB, LC, LD>(G, Ex, Ey, Ez, ta, tb,
                                                                              std::make_integer_sequence<int, NG>{});
                                        }
                                }
                        }
                }
                const int ia = sb.x, ib = sb.y, ic = sk.x, id = sk.y;
                if constexpr (FUSED) {
                        double fs[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                        if (active) {
                                const double *X = a.Dc;
                                double dab[K::NAB], dcd[K::NCD], xbc[K::NB * K::NC], xbd[K::NB * K::ND];
                                double xac[K::NA * K::NC], xad[K::NA * K::ND];
#pragma unroll
                                for (int t = 0; t < K::NAB; t++) dab[t] = __ldg(X + (ia + t / K::NB) * n + ib + t % K::NB);
#pragma unroll
                                for (int t = 0; t < K::NCD; t++) dcd[t] = __ldg(a.Ds + (ic + t / K::ND) * n + id + t % K::ND);
#pragma unroll
                                for (int t = 0; t < K::NB * K::NC; t++) xbc[t] = __ldg(X + (ib + t / K::NC) * n + ic + t % K::NC);
#pragma unroll
                                for (int t = 0; t < K::NB * K::ND; t++) xbd[t] = __ldg(X + (ib + t / K::ND) * n + id + t % K::ND);
#pragma unroll
                                for (int t = 0; t < K::NA * K::NC; t++) xac[t] = __ldg(X + (ia + t / K::NC) * n + ic + t % K::NC);
#pragma unroll
                                for (int t = 0; t < K::NA * K::ND; t++) xad[t] = __ldg(X + (ia + t / K::ND) * n + id + t % K::ND);
#pragma unroll
                                for (int t = 0; t < NG; t++) {
                                        const int d = t % K::ND, c = (t / K::ND) % K::NC;
                                        const int b = (t / K::NCD) % K::NB, xa = t / (K::NCD * K::NB);
                                        const double w = grad_force_weight(dab[xa * K::NB + b], dcd[c * K::ND + d], xbc[b * K::NC + c],
                                                                           xad[xa * K::ND + d], xbd[b * K::ND + d], xac[xa * K::NC + c]);
#pragma unroll
                                        for (int q = 0; q < 6; q++) fs[q] += G[q * NG + t] * w;
                                }
                                if (!sideA) fs[0] = fs[1] = fs[2] = 0.0;
                                if (!sideB) fs[3] = fs[4] = fs[5] = 0.0;
                        }
                        grad_force_flush(a, sb, fs, lane);
                        continue;
                }
                for (int s = 0; s < a.n_dm; s++) {
                        const double *Ds = a.Ds + s * nn;
                        const double *X = a.Dc + s * nn;
                        double dcd[K::NCD];
#pragma unroll
                        for (int t = 0; t < K::NCD; t++)
                                dcd[t] = active ? __ldg(Ds + (ic + t / K::ND) * n + id + t % K::ND) : 0.0;
#pragma unroll
                        for (int x = 0; x < 3; x++) {
                                double *Vj = a.Vj + ((size_t)s * 3 + x) * nn;
                                double *Vk = a.Vk + ((size_t)s * 3 + x) * nn;
                                if (a.with_j) {
                                        // the bra block is the warp's: sum over the lanes, one atomic
#pragma unroll
                                        for (int t = 0; t < K::NAB; t++) {
                                                double vA = 0.0, vB = 0.0;
#pragma unroll
                                                for (int u = 0; u < K::NCD; u++) {
                                                        vA += G[x * NG + t * K::NCD + u] * dcd[u];
                                                        vB += G[(3 + x) * NG + t * K::NCD + u] * dcd[u];
                                                }
                                                vA = warp_sum(sideA ? vA : 0.0);
                                                vB = warp_sum(sideB ? vB : 0.0);
                                                const int xa = t / K::NB, yb = t % K::NB;
                                                if (lane == 0 && vA != 0.0) atomicAdd(Vj + (ia + xa) * n + ib + yb, vA);
                                                if (lane == 0 && vB != 0.0) atomicAdd(Vj + (ib + yb) * n + ia + xa, vB);
                                        }
                                }
                                if (a.with_k && sideA) {
                                        // Vk[a,d] += G X[b,c];  Vk[a,c] += G X[b,d]
#pragma unroll
                                        for (int xa = 0; xa < K::NA; xa++) {
#pragma unroll
                                                for (int d = 0; d < K::ND; d++) {
                                                        double v = 0.0;
#pragma unroll
                                                        for (int b = 0; b < K::NB; b++)
#pragma unroll
                                                                for (int c = 0; c < K::NC; c++)
                                                                        v += G[x * NG + ((xa * K::NB + b) * K::NC + c) * K::ND + d] *
                                                                             __ldg(X + (ib + b) * n + ic + c);
                                                        atomicAdd(Vk + (ia + xa) * n + id + d, v);
                                                }
#pragma unroll
                                                for (int c = 0; c < K::NC; c++) {
                                                        double v = 0.0;
#pragma unroll
                                                        for (int b = 0; b < K::NB; b++)
#pragma unroll
                                                                for (int d = 0; d < K::ND; d++)
                                                                        v += G[x * NG + ((xa * K::NB + b) * K::NC + c) * K::ND + d] *
                                                                             __ldg(X + (ib + b) * n + id + d);
                                                        atomicAdd(Vk + (ia + xa) * n + ic + c, v);
                                                }
                                        }
                                }
                                if (a.with_k && sideB) {
                                        // Vk[b,d] += G X[a,c];  Vk[b,c] += G X[a,d]
#pragma unroll
                                        for (int b = 0; b < K::NB; b++) {
#pragma unroll
                                                for (int d = 0; d < K::ND; d++) {
                                                        double v = 0.0;
#pragma unroll
                                                        for (int xa = 0; xa < K::NA; xa++)
#pragma unroll
                                                                for (int c = 0; c < K::NC; c++)
                                                                        v += G[(3 + x) * NG + ((xa * K::NB + b) * K::NC + c) * K::ND + d] *
                                                                             __ldg(X + (ia + xa) * n + ic + c);
                                                        atomicAdd(Vk + (ib + b) * n + id + d, v);
                                                }
#pragma unroll
                                                for (int c = 0; c < K::NC; c++) {
                                                        double v = 0.0;
#pragma unroll
                                                        for (int xa = 0; xa < K::NA; xa++)
#pragma unroll
                                                                for (int d = 0; d < K::ND; d++)
                                                                        v += G[(3 + x) * NG + ((xa * K::NB + b) * K::NC + c) * K::ND + d] *
                                                                             __ldg(X + (ia + xa) * n + id + d);
                                                        atomicAdd(Vk + (ib + b) * n + ic + c, v);
                                                }
                                        }
                                }
                        }
                }
        }
        if (a.stats) {
                for (int o = 16; o > 0; o >>= 1) {
                        nq += __shfl_xor_sync(0xffffffffu, nq, o);
                        npq += __shfl_xor_sync(0xffffffffu, npq, o);
                }
                if (lane == 0 && nq) {
                        atomicAdd(a.stats + 0, nq);
                        atomicAdd(a.stats + 1, npq);
                }
        }
}

// ---------------------------------------------------------------------------
// Derivative Schwarz bound: one warp per shell pair evaluates the diagonal
// blocks (d_x a b|d_x a b) (derivative on the first function of bra and ket,
// x = y = z components of int2e_ip1ip2) for both orientations of the pair,
// transforms them to the output basis and folds sqrt(max |.|) into the
// parent-shell entries q0[A,B] (derivative on A) and q0[B,A].
struct GradQArgs {
        double omega2;               // as GradArgs::omega2
        PairView pairs;
        const double4 *PP;
        const double2 *PK;
        const double2 *PE;
        const double *table;
        const int2 *goff;
        const double *c2s;
        unsigned long long *q0;
        int nbas, cart;
};

template <int LA, int LB>
__global__ void __launch_bounds__(32) grad_q0_kernel(GradQArgs q)
{
        using K = Class4<LA, LB, LA, LB>;
        using GC = GClass<LA, LB, LA, LB, 1>;
        using S = GradSmem<LA, LB, LA, LB, 1>;
        extern __shared__ __align__(32) double smem_dyn[];
        double *sm = smem_dyn;
        const int lane = threadIdx.x & 31;
        const int ij = blockIdx.x;
        if (ij >= q.pairs.n) return;
        GradArgs a;
        a.PP = q.PP;
        a.PK = q.PK;
        a.PE = q.PE;
        a.table = q.table;
        a.goff = q.goff;
        a.omega2 = q.omega2;
        const int4 sh = q.pairs.sh[ij];
        const int2 pr = q.pairs.pr[ij];
        const double4 Av = q.pairs.A[ij];
        const double4 ABv = q.pairs.AB[ij];
        const double AB[3] = {ABv.x, ABv.y, ABv.z}, C0[3] = {0.0, 0.0, 0.0};
        const int nsa = q.cart ? K::NA : 2 * LA + 1, nsb = q.cart ? K::NB : 2 * LB + 1;
        const double *ca = q.c2s + LA * 100, *cb = q.c2s + LB * 100;
        double mA = 0.0, mB = 0.0;
        for (int pass = 0; pass < GC::NPASS; pass++) {
                const int c0 = pass * GC::NCP;
                grad_eval_pass<LA, LB, LA, LB, 1, 32>(sm, a, pr, pr, Av, AB, C0, AB, 1.0, c0, lane, 0xffffffffu);
                const double *G = sm + S::G;
                for (int cc = 0; cc < GC::NCP; cc++) {
                        const int side = (c0 + cc) / 3;
                        const double *Gc = G + cc * GC::NG;
                        double m = 0.0;
                        for (int t = lane; t < nsa * nsb; t += 32) {
                                const int mi = t / nsb, ni = t % nsb;
                                double v = 0.0;
                                for (int x = 0; x < K::NA; x++) {
                                        const double c1 = ca[mi * 10 + x];
                                        if (c1 == 0.0) continue;
                                        for (int y = 0; y < K::NB; y++) {
                                                const double c2 = cb[ni * 10 + y];
                                                if (c2 == 0.0) continue;
                                                for (int x2 = 0; x2 < K::NA; x2++) {
                                                        const double c3 = ca[mi * 10 + x2];
                                                        if (c3 == 0.0) continue;
                                                        for (int y2 = 0; y2 < K::NB; y2++) {
                                                                const double c4 = cb[ni * 10 + y2];
                                                                if (c4 == 0.0) continue;
                                                                v += c1 * c2 * c3 * c4 * Gc[((x * K::NB + y) * K::NA + x2) * K::NB + y2];
                                                        }
                                                }
                                        }
                                }
                                m = fmax(m, fabs(v));
                        }
                        if (side == 0) mA = fmax(mA, m);
                        else mB = fmax(mB, m);
                }
                __syncwarp();
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
                mA = fmax(mA, __shfl_xor_sync(0xffffffffu, mA, o));
                mB = fmax(mB, __shfl_xor_sync(0xffffffffu, mB, o));
        }
        if (lane == 0) {
                const unsigned long long bA = (unsigned long long)__double_as_longlong(sqrt(fmax(mA, 1e-100)));
                const unsigned long long bB = (unsigned long long)__double_as_longlong(sqrt(fmax(mB, 1e-100)));
                atomicMax(q.q0 + (size_t)sh.z * q.nbas + sh.w, bA);
                atomicMax(q.q0 + (size_t)sh.w * q.nbas + sh.z, bB);
        }
}

// ---------------------------------------------------------------------------
// helpers of the gradient build

// CVHFnr_dm_cond1 (pyscf/lib/vhf/optimizer.c:472-492): max |D| over each
// parent-shell block, all n_dm densities, not symmetrised; and the global max.
static __global__ void dm_cond1_kernel(const double *dms, int n_dm, int nao, const int *ao_loc, int nbas,
                                       double *dm_cond, unsigned long long *dmax_bits)
{
        const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= (long long)nbas * nbas) return;
        const int I = (int)(t / nbas), J = (int)(t % nbas);
        const size_t n = nao;
        double m = 0.0;
        for (int s = 0; s < n_dm; s++) {
                const double *D = dms + (size_t)s * n * n;
                for (int a = ao_loc[I]; a < ao_loc[I + 1]; a++)
                        for (int b = ao_loc[J]; b < ao_loc[J + 1]; b++) m = fmax(m, fabs(D[a * n + b]));
        }
        dm_cond[t] = m;
        atomicMax(dmax_bits, (unsigned long long)__double_as_longlong(m));
}

// density factor of the ket-prefix bound: the screen needs
// q0 q1 > tol and q0 q1 max(2 D_lk, D_jk, D_jl) > tol, so q1 > tol / (q0 min(1, 2 max|D|))
static __global__ void grad_dm_factor_kernel(const unsigned long long *dmax_bits, double *factor)
{
        const double m = __longlong_as_double((long long)*dmax_bits);
        *factor = fmin(1.0, 2.0 * m);
}

// out[x][mu][nu] = scale sum_ab C[mu,a] V[x][a,b] C[nu,b], for nv blocks
static __global__ void grad_cart_to_out_kernel(const double *V, int nv, int nao, int naoc, const int *out_seg,
                                               const int *out_comp, const int4 *seg_info, const double *c2s,
                                               double scale, double *out)
{
        const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        const long long nn = (long long)nao * nao;
        if (t >= nn * nv) return;
        const long long blk = t / nn, r = t - blk * nn;
        const int mu = (int)(r / nao), nu = (int)(r % nao);
        const double *A = V + (size_t)blk * naoc * naoc;
        const int sm = out_seg[mu], sn = out_seg[nu];
        const int4 im = seg_info[sm], in_ = seg_info[sn];
        const int km = out_comp[mu], kn = out_comp[nu];
        const int ncm = (im.x + 1) * (im.x + 2) / 2, ncn = (in_.x + 1) * (in_.x + 2) / 2;
        const double *cm = c2s + im.x * 100 + km * 10, *cn = c2s + in_.x * 100 + kn * 10;
        double v = 0.0;
        for (int x = 0; x < ncm; x++) {
                const double f1 = cm[x];
                if (f1 == 0.0) continue;
                const size_t a = im.z + x;
                double s = 0.0;
                for (int y = 0; y < ncn; y++) {
                        const double f2 = cn[y];
                        if (f2 == 0.0) continue;
                        s += f2 * A[a * naoc + in_.z + y];
                }
                v += f1 * s;
        }
        out[t] = scale * v;
}

// ---------------------------------------------------------------------------
// Register family of the fused force contraction (b200jk_grad_contract) for
// mid-size classes.  A quartet's contribution to the forces is six numbers,
// fs[q] = sum_t G[q, t] w[t], with w[t] = 2 D_ab Ds_cd - X_bc X_ad - X_bd X_ac
// fixed by the density blocks.  So the lane computes w once per quartet and
// assembles each root's derivative integrals straight into fs: NG weights
// and the three 2D slices live in registers, not the six derivative blocks
// of grad_thread_kernel, which brings classes up to NG + 3 SE <= 102 (those of
// one p or d shell with two s or p shells) from the shared-memory family to
// one ket per lane.  Of grad_thread_kernel's own classes it takes those of 9
// or more components ((10|10): 254 -> 164 registers, 14.0 -> 12.7 ms on
// (H2O)16/cc-pVDZ); for the smaller ones the six blocks cost no occupancy
// and the two kernels were within 4% either way.
template <int LA, int LB, int LC, int LD>
__host__ __device__ constexpr bool grad_force_regs()
{
        using GC = GClass<LA, LB, LC, LD, 0>;
        return GC::NG + 3 * GC::SE <= 102 && (!grad_thread_family<LA, LB, LC, LD>() || GC::NG >= 9);
}

template <int LA, int LB, int LC, int LD, int T>
__device__ __forceinline__ void grad_force_one(double fs[6], const double *w, const double *Ex, const double *Ey,
                                               const double *Ez, double ta, double tb)
{
        using K = Class4<LA, LB, LC, LD>;
        using GC = GClass<LA, LB, LC, LD, 0>;
        constexpr int id = T % K::ND, ic = (T / K::ND) % K::NC, ib = (T / K::NCD) % K::NB, ia = T / (K::NCD * K::NB);
        constexpr int ax = cart_lx(LA, ia), ay = cart_ly(LA, ia), az = cart_lz(LA, ia);
        constexpr int bx = cart_lx(LB, ib), by = cart_ly(LB, ib), bz = cart_lz(LB, ib);
        constexpr int ox = GC::eidx(ax, bx, cart_lx(LC, ic), cart_lx(LD, id));
        constexpr int oy = GC::eidx(ay, by, cart_ly(LC, ic), cart_ly(LD, id));
        constexpr int oz = GC::eidx(az, bz, cart_lz(LC, ic), cart_lz(LD, id));
        constexpr int SA = GC::STEP_A, SB = GC::STEP_B;
        const double wt = w[T];
        const double ex = Ex[ox] * wt, ey = Ey[oy], ez = Ez[oz];
        double dax = ta * Ex[ox + SA], day = ta * Ey[oy + SA], daz = ta * Ez[oz + SA];
        if constexpr (ax > 0) dax -= ax * Ex[ox - SA];
        if constexpr (ay > 0) day -= ay * Ey[oy - SA];
        if constexpr (az > 0) daz -= az * Ez[oz - SA];
        double dbx = tb * Ex[ox + SB], dby = tb * Ey[oy + SB], dbz = tb * Ez[oz + SB];
        if constexpr (bx > 0) dbx -= bx * Ex[ox - SB];
        if constexpr (by > 0) dby -= by * Ey[oy - SB];
        if constexpr (bz > 0) dbz -= bz * Ez[oz - SB];
        const double eyz = ey * ez;
        fs[0] += wt * dax * eyz;
        fs[1] += ex * day * ez;
        fs[2] += ex * ey * daz;
        fs[3] += wt * dbx * eyz;
        fs[4] += ex * dby * ez;
        fs[5] += ex * ey * dbz;
}

template <int LA, int LB, int LC, int LD, int... Ts>
__device__ __forceinline__ void grad_force_assemble(double fs[6], const double *w, const double *Ex,
                                                    const double *Ey, const double *Ez, double ta, double tb,
                                                    std::integer_sequence<int, Ts...>)
{
        (grad_force_one<LA, LB, LC, LD, Ts>(fs, w, Ex, Ey, Ez, ta, tb), ...);
}


template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(128) grad_force_kernel(GradArgs a)
{
        using K = Class4<LA, LB, LC, LD>;
        using GC = GClass<LA, LB, LC, LD, 0>;
        constexpr int NG = K::NG, NR = GC::NR, SE = GC::SE;
        const int lane = threadIdx.x & 31;
        const int nseg = a.bra.n * B2_NBUCKET;
        const long long total = a.chunk_off[nseg];
        const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
        const size_t n = (size_t)a.naoc;
        const double *table = a.table + rys_padded_offset(NR);
        unsigned long long nq = 0, npq = 0;
        for (long long chunk = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; chunk < total;
             chunk += nwarps) {
                const int sgi = find_bra(a.chunk_off, nseg, chunk);
                const int ij = sgi / B2_NBUCKET;
                const int pos = (int)(chunk - a.chunk_off[sgi]) * 32 + lane;
                const int kl = a.ket.boff[sgi % B2_NBUCKET] + a.kst[sgi] + pos;
                const int4 sb = a.bra.sh[ij];
                const int2 pb = a.bra.pr[ij];
                const double4 Ab = a.bra.A[ij];
                const double4 ABb = a.bra.AB[ij];
                const double AB[3] = {ABb.x, ABb.y, ABb.z};
                int4 sk = make_int4(0, 0, 0, 0);
                bool sideA = false, sideB = false;
                if (pos < a.nkl[sgi]) {
                        sk = a.ket.sh[kl];
                        const int kk = max(sk.z, sk.w), ll = min(sk.z, sk.w);
                        sideA = grad_side_passes(a, sb.z, sb.w, kk, ll);
                        sideB = Ab.w == 0.0 && grad_side_passes(a, sb.w, sb.z, kk, ll);
                }
                const bool active = sideA || sideB;
                double fs[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                if (active) {
                        // the weights of the quartet's Cartesian components
                        const int ia = sb.x, ib = sb.y, ic = sk.x, id = sk.y;
                        const double *X = a.Dc;
                        double w[NG];
#pragma unroll
                        for (int t = 0; t < NG; t++) {
                                const int d = t % K::ND, c = (t / K::ND) % K::NC;
                                const int b = (t / K::NCD) % K::NB, xa = t / (K::NCD * K::NB);
                                w[t] = grad_force_weight(__ldg(X + (ia + xa) * n + ib + b), __ldg(a.Ds + (ic + c) * n + id + d),
                                                         __ldg(X + (ib + b) * n + ic + c), __ldg(X + (ia + xa) * n + id + d),
                                                         __ldg(X + (ib + b) * n + id + d), __ldg(X + (ia + xa) * n + ic + c));
                        }
                        const int2 pk = a.ket.pr[kl];
                        const double4 Ak = a.ket.A[kl];
                        const double4 CDk = a.ket.AB[kl];
                        const double fac = Ak.w != 0.0 ? 0.5 : 1.0;
                        const double A0[3] = {0.0, 0.0, 0.0};
                        const double C[3] = {Ak.x - Ab.x, Ak.y - Ab.y, Ak.z - Ab.z};
                        const double CD[3] = {CDk.x, CDk.y, CDk.z};
                        nq += (unsigned long long)sideA + (unsigned long long)sideB;
                        npq += (unsigned long long)pb.y * pk.y;
                        for (int ip = 0; ip < pb.y; ip++) {
                                const double4 P = a.PP[pb.x + ip];
                                const double2 KP = a.PK[pb.x + ip];
                                const double2 EP = a.PE[pb.x + ip];
                                const double Kab = KP.x * fac;
                                const double Pv[3] = {P.x - Ab.x, P.y - Ab.y, P.z - Ab.z};
                                const double ta = 2.0 * EP.x, tb = 2.0 * EP.y;
                                for (int kp = 0; kp < pk.y; kp++) {
                                        const double4 Q = a.PP[pk.x + kp];
                                        const double2 KQ = a.PK[pk.x + kp];
                                        const double Qv[3] = {Q.x - Ab.x, Q.y - Ab.y, Q.z - Ab.z};
                                        PrimQ<double> sq;
                                        prim_setup<double>(sq, P.w, KP.y, Pv, Q.w, KQ.y, Qv, A0, C, Kab * KQ.x, a.omega2);
                                        double u[NR], wr[NR];
                                        rys_roots_slice<NR, double>(sq.T, table, u, wr);
#pragma unroll
                                        for (int r = 0; r < NR; r++) {
                                                RysCoef<double> rc;
                                                rys_coef<double>(rc, u[r], sq);
                                                double Ex[SE], Ey[SE], Ez[SE];
                                                grad_slice<LA, LB, LC, LD, 0>(Ex, 1.0, rc, 0, AB[0], CD[0]);
                                                grad_slice<LA, LB, LC, LD, 0>(Ey, 1.0, rc, 1, AB[1], CD[1]);
                                                grad_slice<LA, LB, LC, LD, 0>(Ez, sq.pref * wr[r], rc, 2, AB[2], CD[2]);
                                                grad_force_assemble<LA, LB, LC, LD>(fs, w, Ex, Ey, Ez, ta, tb,
                                                                                    std::make_integer_sequence<int, NG>{});
                                        }
                                }
                        }
                        if (!sideA) fs[0] = fs[1] = fs[2] = 0.0;
                        if (!sideB) fs[3] = fs[4] = fs[5] = 0.0;
                }
                grad_force_flush(a, sb, fs, lane);
        }
        if (a.stats) {
                for (int o = 16; o > 0; o >>= 1) {
                        nq += __shfl_xor_sync(0xffffffffu, nq, o);
                        npq += __shfl_xor_sync(0xffffffffu, npq, o);
                }
                if (lane == 0 && nq) {
                        atomicAdd(a.stats + 0, nq);
                        atomicAdd(a.stats + 1, npq);
                }
        }
}

} // namespace b200jk
