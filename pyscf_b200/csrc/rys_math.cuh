// rys_math.cuh — electron-repulsion integrals by Rys quadrature.
//
// Everything here is __host__ __device__ so that the exact code the CUDA
// kernels run can also be replayed on the host (b200jk_hostcheck_* in
// b200jk.cu) and compared with the CPU oracle without a GPU.
//
// Conventions (shared with PySCF/libcint, pyscf/gto/mole.py:157-187 and
// pyscf/symm/sph.py:83-103):
//   Cartesian components of degree l are ordered lx descending, then ly
//   descending (xx, xy, xz, yy, yz, zz for l = 2).
//   A primitive Cartesian Gaussian is (x-Ax)^ax (y-Ay)^ay (z-Az)^az e^{-a r_A^2}
//   with no angular normalisation; the contraction coefficients (already
//   radially normalised by PySCF) and the real-solid-harmonic transform are
//   applied outside these routines.
//
// Method (Rys, Dupuis & King, J. Comput. Chem. 4, 154 (1983)):
//   (ab|cd) = 2 pi^{5/2} / (p q sqrt(p+q)) K_ab K_cd
//             * sum_r w_r I_x(r) I_y(r) I_z(r)
//   with roots u_r = t_r^2 and weights w_r of the Rys rule of order
//   n = floor(L/2) + 1, L = la+lb+lc+ld.  Per root and Cartesian direction the
//   2D integrals obey, with rho = pq/(p+q),
//     I(e+1,f) = C00 I(e,f) + e B10 I(e-1,f) + f B00 I(e,f-1)
//     I(e,f+1) = C00' I(e,f) + f B01 I(e,f-1) + e B00 I(e-1,f)
//     C00 = PA - (q/(p+q)) u PQ,  C00' = QC + (p/(p+q)) u PQ,
//     B00 = u / (2(p+q)),  B10 = (1 - q u/(p+q)) / (2p),  B01 = (1 - p u/(p+q)) / (2q),
//   and the transfer to the second centre of each pair is the binomial
//   expansion (x-B)^b = sum_k C(b,k) (x-A)^k (A-B)^{b-k}.
#pragma once
#include <math.h>
#include <utility>

#ifdef __CUDACC__
#define B2_HD __host__ __device__ __forceinline__
#define B2_HDC __host__ __device__ constexpr
#else
#define B2_HD inline
#define B2_HDC constexpr
#endif

#if defined(__CUDA_ARCH__)
#define B2_LDG(p) __ldg(p)
#else
#define B2_LDG(p) (*(p))
#endif

#include "rys_table.inc"
#include "rys_table_f.inc"

namespace b200jk {

// arithmetic helpers for the two compute types (double: FP64 path, float:
// FP32 evaluation of the mixed-precision path)
B2_HD double b2fma(double a, double b, double c) { return fma(a, b, c); }
B2_HD float b2fma(float a, float b, float c) { return fmaf(a, b, c); }
B2_HD double b2sqrt(double a) { return sqrt(a); }
B2_HD float b2sqrt(float a) { return sqrtf(a); }

B2_HDC int ncart(int l) { return (l + 1) * (l + 2) / 2; }
B2_HDC int nsph(int l) { return 2 * l + 1; }

// Cartesian component n of degree l
B2_HDC int cart_lx(int l, int n)
{
        int lx = l;
        while (n > l - lx) { n -= l - lx + 1; lx--; }
        return lx;
}
B2_HDC int cart_ly(int l, int n)
{
        int lx = l;
        while (n > l - lx) { n -= l - lx + 1; lx--; }
        return l - lx - n;
}
B2_HDC int cart_lz(int l, int n) { return l - cart_lx(l, n) - cart_ly(l, n); }

B2_HDC int binom(int n, int k)
{
        int r = 1;
        for (int i = 1; i <= k; i++) r = r * (n - k + i) / i;
        return r;
}

B2_HDC int rys_nroots(int L) { return L / 2 + 1; }

B2_HDC int rys_t_asym(int n)
{
        constexpr int t[] = {RYS_T_ASYM_LIST};
        return t[n];
}
B2_HDC int rys_table_offset(int n)
{
        constexpr int t[] = {RYS_TABLE_OFFSET_LIST};
        return t[n];
}
B2_HDC double rys_herm_x2(int k)
{
        constexpr double t[] = {RYS_HERMITE_X2_LIST};
        return t[k];
}
B2_HDC double rys_herm_w(int k)
{
        constexpr double t[] = {RYS_HERMITE_W_LIST};
        return t[k];
}

// Device layout of the tables: every polynomial row padded from RYS_DEG+1 to
// RYS_ROW coefficients so that a row is four aligned 32-byte vectors.
#define RYS_ROW 16
B2_HDC int rys_padded_offset(int n)
{
        int o = 0;
        for (int m = 1; m < n; m++) o += rys_t_asym(m) * 2 * m * RYS_ROW;
        return o;
}
B2_HDC int rys_padded_size() { return rys_padded_offset(RYS_NMAX + 1); }

// packed generator table -> padded layout
inline void rys_pad_table(const double *packed, double *out)
{
        for (int n = 1; n <= RYS_NMAX; n++) {
                const double *src = packed + rys_table_offset(n);
                double *dst = out + rys_padded_offset(n);
                for (int row = 0; row < rys_t_asym(n) * 2 * n; row++) {
                        for (int k = 0; k < RYS_ROW; k++)
                                dst[row * RYS_ROW + k] = k <= RYS_DEG ? src[row * (RYS_DEG + 1) + k] : 0.0;
                }
        }
}

template <typename R>
struct alignas(4 * sizeof(R)) RysVec4 {
        R v[4];
};

// Layout of the device tables per compute type.  float64: rows of RYS_ROW
// (degree RYS_DEG, padded), large-T limit from rys_t_asym(n).  float32 (the
// float32 pass of mixed precision): rows of RYS_F_ROW (degree RYS_F_DEG),
// large-T limit from the smaller rys_f_t_asym(n).
B2_HDC int rys_f_t_asym(int n)
{
        constexpr int t[] = {RYS_F_T_ASYM_LIST};
        return t[n];
}
B2_HDC int rys_f_offset(int n)
{
        constexpr int t[] = {RYS_F_OFFSET_LIST};
        return t[n];
}

template <typename R> struct RysLayout;
template <> struct RysLayout<double> {
        static constexpr int ROW = RYS_ROW;
        static B2_HDC int t_asym(int n) { return rys_t_asym(n); }
        static B2_HDC int offset(int n) { return rys_padded_offset(n); }
};
template <> struct RysLayout<float> {
        static constexpr int ROW = RYS_F_ROW;
        static B2_HDC int t_asym(int n) { return rys_f_t_asym(n); }
        static B2_HDC int offset(int n) { return rys_f_offset(n); }
};

// elements of the order-n slice of the table of type R
template <typename R>
B2_HDC int rys_slice_elems(int n) { return RysLayout<R>::t_asym(n) * 2 * n * RysLayout<R>::ROW; }

// Horner evaluation of one row at x
template <typename R>
B2_HD R rys_poly(const R *__restrict__ row, R x);

template <>
B2_HD double rys_poly<double>(const double *__restrict__ row, double x)
{
        const RysVec4<double> *q = reinterpret_cast<const RysVec4<double> *>(row);
        const RysVec4<double> q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
        double r = q3.v[1];
        r = b2fma(r, x, q3.v[0]);
        r = b2fma(r, x, q2.v[3]); r = b2fma(r, x, q2.v[2]); r = b2fma(r, x, q2.v[1]); r = b2fma(r, x, q2.v[0]);
        r = b2fma(r, x, q1.v[3]); r = b2fma(r, x, q1.v[2]); r = b2fma(r, x, q1.v[1]); r = b2fma(r, x, q1.v[0]);
        r = b2fma(r, x, q0.v[3]); r = b2fma(r, x, q0.v[2]); r = b2fma(r, x, q0.v[1]); r = b2fma(r, x, q0.v[0]);
        return r;
}

template <>
B2_HD float rys_poly<float>(const float *__restrict__ row, float x)
{
        const RysVec4<float> *q = reinterpret_cast<const RysVec4<float> *>(row);
        const RysVec4<float> q0 = q[0], q1 = q[1];
        float r = q1.v[3];
        r = b2fma(r, x, q1.v[2]); r = b2fma(r, x, q1.v[1]); r = b2fma(r, x, q1.v[0]);
        r = b2fma(r, x, q0.v[3]); r = b2fma(r, x, q0.v[2]); r = b2fma(r, x, q0.v[1]); r = b2fma(r, x, q0.v[0]);
        return r;
}

// Roots u[i] and weights w[i] of the order-NR Rys rule at argument T, with
// `tab` pointing at the order-NR slice of the table of type R (global memory
// or a copy in shared memory).  NaN or huge T take the asymptotic branch, so
// the table is never indexed out of range.
template <int NR, typename R>
B2_HD void rys_roots_slice(R T, const R *__restrict__ tab, R *u, R *w)
{
        using L = RysLayout<R>;
        if (!(T < (R)L::t_asym(NR))) {
                const R it = (R)1 / T;
                const R st = b2sqrt(it);
#pragma unroll
                for (int i = 0; i < NR; i++) {
                        u[i] = (R)rys_herm_x2(NR * (NR - 1) / 2 + i) * it;
                        w[i] = (R)rys_herm_w(NR * (NR - 1) / 2 + i) * st;
                }
                return;
        }
        const int p = (int)T;
        const R x = (R)2 * (T - (R)p) - (R)1;
        const R *c = tab + p * (2 * NR * L::ROW);
#pragma unroll
        for (int f = 0; f < NR; f++) {
                u[f] = rys_poly<R>(c + f * L::ROW, x);
                w[f] = rys_poly<R>(c + (NR + f) * L::ROW, x);
        }
}

// doubles in the order-NR slice of the padded float64 table
B2_HDC int rys_slice_size(int nr) { return rys_slice_elems<double>(nr); }

// Root r (and its weight) of the order-NR rule only; `tab` points at the
// order-NR slice of the table of type R.
template <int NR, typename R>
B2_HD void rys_root_one(R T, const R *__restrict__ tab, int r, R &u, R &w)
{
        using L = RysLayout<R>;
        if (!(T < (R)L::t_asym(NR))) {
                const R it = (R)1 / T;
                double x2 = rys_herm_x2(NR * (NR - 1) / 2), wh = rys_herm_w(NR * (NR - 1) / 2);
#pragma unroll
                for (int i = 1; i < NR; i++)
                        if (r == i) { x2 = rys_herm_x2(NR * (NR - 1) / 2 + i); wh = rys_herm_w(NR * (NR - 1) / 2 + i); }
                u = (R)x2 * it;
                w = (R)wh * b2sqrt(it);
                return;
        }
        const int p = (int)T;
        const R x = (R)2 * (T - (R)p) - (R)1;
        const R *c = tab + p * (2 * NR * L::ROW);
        u = rys_poly<R>(c + r * L::ROW, x);
        w = rys_poly<R>(c + (NR + r) * L::ROW, x);
}

// 2D vertical recurrence: g[e*NF + f], e < NE, f < NF.
template <int NE, int NF, typename R>
B2_HD void vrr2d(R *g, R g00, R c00, R c00p, R b10, R b01, R b00)
{
        g[0] = g00;
        if (NE > 1) g[NF] = c00 * g00;
#pragma unroll
        for (int e = 1; e < NE - 1; e++) g[(e + 1) * NF] = c00 * g[e * NF] + (R)e * b10 * g[(e - 1) * NF];
        if (NF > 1) {
#pragma unroll
                for (int e = 0; e < NE; e++) {
                        R v = c00p * g[e * NF];
                        if (e > 0) v += (R)e * b00 * g[(e - 1) * NF];
                        g[e * NF + 1] = v;
                }
#pragma unroll
                for (int f = 1; f < NF - 1; f++) {
#pragma unroll
                        for (int e = 0; e < NE; e++) {
                                R v = c00p * g[e * NF + f] + (R)f * b01 * g[e * NF + f - 1];
                                if (e > 0) v += (R)e * b00 * g[(e - 1) * NF + f];
                                g[e * NF + f + 1] = v;
                        }
                }
        }
}

// 2D horizontal transfer: from g[e][f] (e <= LA+LB, f <= LC+LD) to
// h[((a*(LB+1) + b)*(LC+1) + c)*(LD+1) + d].
template <int LA, int LB, int LC, int LD, typename R>
B2_HD void hrr2d(const R *g, R *h, R ab, R cd)
{
        constexpr int NF = LC + LD + 1;
        R abp[LB + 1], cdp[LD + 1];
        abp[0] = (R)1;
#pragma unroll
        for (int k = 1; k <= LB; k++) abp[k] = abp[k - 1] * ab;
        cdp[0] = (R)1;
#pragma unroll
        for (int k = 1; k <= LD; k++) cdp[k] = cdp[k - 1] * cd;
        // t[(a*(LB+1)+b)*NF + f]
        R t[(LA + 1) * (LB + 1) * NF];
#pragma unroll
        for (int a = 0; a <= LA; a++) {
#pragma unroll
                for (int b = 0; b <= LB; b++) {
#pragma unroll
                        for (int f = 0; f < NF; f++) {
                                R v = (R)0;
#pragma unroll
                                for (int k = 0; k <= b; k++)
                                        v += (R)binom(b, k) * abp[b - k] * g[(a + k) * NF + f];
                                t[(a * (LB + 1) + b) * NF + f] = v;
                        }
                }
        }
#pragma unroll
        for (int ab_ = 0; ab_ < (LA + 1) * (LB + 1); ab_++) {
#pragma unroll
                for (int c = 0; c <= LC; c++) {
#pragma unroll
                        for (int d = 0; d <= LD; d++) {
                                R v = (R)0;
#pragma unroll
                                for (int k = 0; k <= d; k++)
                                        v += (R)binom(d, k) * cdp[d - k] * t[ab_ * NF + c + k];
                                h[(ab_ * (LC + 1) + c) * (LD + 1) + d] = v;
                        }
                }
        }
}

template <int LA, int LB, int LC, int LD>
struct Class4 {
        static constexpr int NR = rys_nroots(LA + LB + LC + LD);
        static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
        static constexpr int NAB = NA * NB, NCD = NC * ND, NG = NAB * NCD;
        static constexpr int NE = LA + LB + 1, NF = LC + LD + 1;
        static constexpr int SA = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
        B2_HD static constexpr int hidx(int a, int b, int c, int d)
        {
                return ((a * (LB + 1) + b) * (LC + 1) + c) * (LD + 1) + d;
        }
};

// Scalars of one primitive quartet shared by all roots.  Primitive pairs
// carry 1/(2p), so a quartet needs one division and one square root.  R is
// the compute type (double, or float for the FP32 quartets of the mixed path).
template <typename R>
struct PrimQ {
        R PA[3], QC[3], PQ[3];
        R ipq;          // 1/(p+q)
        R qf0, pf0;     // q/(p+q), p/(p+q)
        R i2p, i2q;     // 1/(2p), 1/(2q)
        R T;            // rho |PQ|^2 (times theta for erf-attenuated Coulomb)
        R pref;         // 2 pi^{5/2} K_ab K_cd / (p q sqrt(p+q)) (times sqrt(theta))
        R theta;        // 1, or omega^2 / (omega^2 + rho) for erf(omega r12)/r12
};

// omega2 > 0: the long-range operator erf(omega r12)/r12 (omega2 = omega^2).
// Its Rys representation is the Coulomb one with the t-integral cut at
// t^2 = theta = omega^2 / (omega^2 + rho): with t = sqrt(theta) s, the
// quadrature is that of T' = theta T, roots t^2 = theta s_i^2, weights
// sqrt(theta) w_i (rys_coef applies theta to the root).
template <typename R>
B2_HD void prim_setup(PrimQ<R> &s, R p, R i2p, const R P[3], R q, R i2q, const R Q[3], const R A[3],
                      const R C[3], R kk, R omega2 = (R)0)
{
        s.ipq = (R)1 / (p + q);
        s.qf0 = q * s.ipq;
        s.pf0 = p * s.ipq;
        s.i2p = i2p;
        s.i2q = i2q;
#pragma unroll
        for (int x = 0; x < 3; x++) {
                s.PA[x] = P[x] - A[x];
                s.QC[x] = Q[x] - C[x];
                s.PQ[x] = P[x] - Q[x];
        }
        s.T = p * s.qf0 * (s.PQ[0] * s.PQ[0] + s.PQ[1] * s.PQ[1] + s.PQ[2] * s.PQ[2]);
        s.pref = (R)34.98683665524972497 * kk * ((R)4 * i2p * i2q) * b2sqrt(s.ipq);
        s.theta = (R)1;
        if (omega2 > (R)0) {
                const R rho = p * s.qf0;
                s.theta = omega2 / (omega2 + rho);
                s.T *= s.theta;
                s.pref *= b2sqrt(s.theta);
        }
}

// Root-dependent recurrence coefficients of one primitive quartet.
template <typename R>
struct RysCoef {
        R c00[3], c00p[3], b10, b01, b00;
};

template <typename R>
B2_HD void rys_coef(RysCoef<R> &rc, R u, const PrimQ<R> &s)
{
        u *= s.theta;
        const R qf = s.qf0 * u, pf = s.pf0 * u;
        rc.b00 = (R)0.5 * u * s.ipq;
        rc.b10 = s.i2p * ((R)1 - qf);
        rc.b01 = s.i2q * ((R)1 - pf);
#pragma unroll
        for (int x = 0; x < 3; x++) {
                rc.c00[x] = s.PA[x] - qf * s.PQ[x];
                rc.c00p[x] = s.QC[x] + pf * s.PQ[x];
        }
}

// Components [BASE, BASE + N) of the block, into Gp[0..N): G[T] += I_x I_y I_z
// for Cartesian component T.  The offsets into the 2D integrals are constant
// expressions, so the whole assembly unrolls into register operations.
template <int LA, int LB, int LC, int LD, int T, typename R>
B2_HD void assemble_one_to(R &g, const R *hx, const R *hy, const R *hz)
{
        using K = Class4<LA, LB, LC, LD>;
        constexpr int id = T % K::ND, ic = (T / K::ND) % K::NC, ib = (T / K::NCD) % K::NB, ia = T / (K::NCD * K::NB);
        constexpr int ox = K::hidx(cart_lx(LA, ia), cart_lx(LB, ib), cart_lx(LC, ic), cart_lx(LD, id));
        constexpr int oy = K::hidx(cart_ly(LA, ia), cart_ly(LB, ib), cart_ly(LC, ic), cart_ly(LD, id));
        constexpr int oz = K::hidx(cart_lz(LA, ia), cart_lz(LB, ib), cart_lz(LC, ic), cart_lz(LD, id));
        g += hx[ox] * hy[oy] * hz[oz];
}

template <int LA, int LB, int LC, int LD, int BASE, typename R, int... Ts>
B2_HD void assemble_part(R *Gp, const R *hx, const R *hy, const R *hz, std::integer_sequence<int, Ts...>)
{
        (assemble_one_to<LA, LB, LC, LD, BASE + Ts, R>(Gp[Ts], hx, hy, hz), ...);
}

// One primitive quartet into components [BASE, BASE + N) of the block.
// `tab` is the order-NR slice of the padded table of type R.
template <int LA, int LB, int LC, int LD, int BASE, int N, typename R>
B2_HD void add_prim_quartet_part(R *Gp, const R *tab, const PrimQ<R> &s, const R AB[3], const R CD[3])
{
        using K = Class4<LA, LB, LC, LD>;
        R u[K::NR], w[K::NR];
        rys_roots_slice<K::NR, R>(s.T, tab, u, w);
#pragma unroll
        for (int r = 0; r < K::NR; r++) {
                RysCoef<R> rc;
                rys_coef<R>(rc, u[r], s);
                R g[K::NE * K::NF];
                R hx[K::SA], hy[K::SA], hz[K::SA];
                vrr2d<K::NE, K::NF, R>(g, (R)1, rc.c00[0], rc.c00p[0], rc.b10, rc.b01, rc.b00);
                hrr2d<LA, LB, LC, LD, R>(g, hx, AB[0], CD[0]);
                vrr2d<K::NE, K::NF, R>(g, (R)1, rc.c00[1], rc.c00p[1], rc.b10, rc.b01, rc.b00);
                hrr2d<LA, LB, LC, LD, R>(g, hy, AB[1], CD[1]);
                vrr2d<K::NE, K::NF, R>(g, s.pref * w[r], rc.c00[2], rc.c00p[2], rc.b10, rc.b01, rc.b00);
                hrr2d<LA, LB, LC, LD, R>(g, hz, AB[2], CD[2]);
                assemble_part<LA, LB, LC, LD, BASE, R>(Gp, hx, hy, hz, std::make_integer_sequence<int, N>{});
        }
}

// Add one primitive quartet to the Cartesian block G[((a*NB+b)*NC+c)*ND+d]
// (host replay of the kernels' arithmetic); `tab` is the order-NR slice of
// the table of type R.
template <int LA, int LB, int LC, int LD, typename R>
B2_HD void add_prim_quartet(R *G, const R *tab, const PrimQ<R> &s, const R AB[3], const R CD[3])
{
        using K = Class4<LA, LB, LC, LD>;
        R u[K::NR], w[K::NR];
        rys_roots_slice<K::NR, R>(s.T, tab, u, w);
        for (int r = 0; r < K::NR; r++) {
                RysCoef<R> rc;
                rys_coef<R>(rc, u[r], s);
                R g[K::NE * K::NF];
                R hx[K::SA], hy[K::SA], hz[K::SA];
                vrr2d<K::NE, K::NF, R>(g, (R)1, rc.c00[0], rc.c00p[0], rc.b10, rc.b01, rc.b00);
                hrr2d<LA, LB, LC, LD, R>(g, hx, AB[0], CD[0]);
                vrr2d<K::NE, K::NF, R>(g, (R)1, rc.c00[1], rc.c00p[1], rc.b10, rc.b01, rc.b00);
                hrr2d<LA, LB, LC, LD, R>(g, hy, AB[1], CD[1]);
                vrr2d<K::NE, K::NF, R>(g, s.pref * w[r], rc.c00[2], rc.c00p[2], rc.b10, rc.b01, rc.b00);
                hrr2d<LA, LB, LC, LD, R>(g, hz, AB[2], CD[2]);
                // same operations in the same order as assemble_one_to
                for (int ia = 0; ia < K::NA; ia++)
                for (int ib = 0; ib < K::NB; ib++)
                for (int ic = 0; ic < K::NC; ic++)
                for (int id = 0; id < K::ND; id++) {
                        const int ox = K::hidx(cart_lx(LA, ia), cart_lx(LB, ib), cart_lx(LC, ic), cart_lx(LD, id));
                        const int oy = K::hidx(cart_ly(LA, ia), cart_ly(LB, ib), cart_ly(LC, ic), cart_ly(LD, id));
                        const int oz = K::hidx(cart_lz(LA, ia), cart_lz(LB, ib), cart_lz(LC, ic), cart_lz(LD, id));
                        G[((ia * K::NB + ib) * K::NC + ic) * K::ND + id] += hx[ox] * hy[oy] * hz[oz];
                }
        }
}

// One (root, direction) slice of the 2D integrals after the transfer,
// written to h (used by the warp-cooperative kernels).
template <int LA, int LB, int LC, int LD, typename R>
B2_HD void rys_2d_slice(R *h, R g00, const RysCoef<R> &rc, int dir, R ab, R cd)
{
        using K = Class4<LA, LB, LC, LD>;
        R g[K::NE * K::NF];
        vrr2d<K::NE, K::NF, R>(g, g00, rc.c00[dir], rc.c00p[dir], rc.b10, rc.b01, rc.b00);
        hrr2d<LA, LB, LC, LD, R>(g, h, ab, cd);
}

} // namespace b200jk
