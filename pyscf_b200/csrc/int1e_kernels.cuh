// int1e_kernels.cuh — one-electron integrals on the GPU: overlap, kinetic
// energy and nuclear attraction of the plan's basis, the matrices PySCF's
// SCF.get_ovlp / get_hcore build from libcint's int1e_ovlp, int1e_kin and
// int1e_nuc (pyscf/scf/hf.py:315-347).
//
// One thread per Cartesian element (a, b) of a segment pair (i >= j; the
// mirror element is written too).  Over the primitive pairs of the segment
// pair (the planner's (P, p), (K_ab c_a c_b, 1/2p), (alpha, beta)):
//   overlap   Obara-Saika 1D recurrence s(i, j) with PA, PB, 1/2p:
//             S = (pi/p)^{3/2} K s_x s_y s_z;
//   kinetic   T_x(i, j) = beta (2j + 1) s(i, j) - 2 beta^2 s(i, j + 2)
//                         - j (j - 1)/2 s(i, j - 2),
//             T = (pi/p)^{3/2} K (T_x s_y s_z + s_x T_y s_z + s_x s_y T_z);
//   nuclear   for every atom C of charge Z, Rys quadrature of the weight
//             exp(-p |PC|^2 t^2) on [0, 1] with (la + lb)/2 + 1 roots, 1D
//             recurrence I(i + 1, 0) = (PA - u PC) I(i, 0) + i (1 - u)/(2p) I(i - 1, 0)
//             and transfer I(i, j + 1) = I(i + 1, j) + AB I(i, j):
//             V = -Z (2 pi / p) K sum_r w_r I_x I_y I_z.
// The Cartesian matrices are then mapped to the output basis with the same
// real-solid-harmonic transform as the J/K build.
#pragma once
#include "rys_math.cuh"

namespace b200jk {

struct Int1eArgs {
        const int4 *pair;            // (segment i, segment j, first primitive pair, count), i >= j
        const long long *elem_off;   // first element of pair t; elem_off[npair] = total
        int npair;
        const double4 *seg;          // (centre x, y, z, l) per segment
        const int *seg_cart;         // Cartesian AO offset per segment
        const double4 *PP;           // (P, p)
        const double2 *PK;           // (K_ab c_a c_b, 1/(2p))
        const double2 *PE;           // (alpha, beta)
        const double4 *atoms;        // (x, y, z, Z)
        int natm, naoc;
        const double *table;         // Rys tables (float64)
        double *S, *H;               // Cartesian naoc x naoc
};

__device__ __forceinline__ int i1e_find(const long long *off, int n, long long e)
{
        int lo = 0, hi = n;
        while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (off[mid] <= e) lo = mid;
                else hi = mid;
        }
        return lo;
}

// the Cartesian exponents (x, y, z) of component c of angular momentum l in
// PySCF order (lx descending, then ly descending)
__device__ __forceinline__ void i1e_cart(int l, int c, int e[3])
{
        int k = 0;
        for (int lx = l; lx >= 0; lx--)
                for (int ly = l - lx; ly >= 0; ly--, k++)
                        if (k == c) {
                                e[0] = lx; e[1] = ly; e[2] = l - lx - ly;
                                return;
                        }
        e[0] = e[1] = e[2] = 0;
}

// 1D overlap s(i, j) for i <= ia, j <= jb, Obara-Saika
template <int NI, int NJ>
__device__ __forceinline__ void i1e_overlap_1d(double pa, double pb, double i2p, int ia, int jb, double (&s)[NI][NJ])
{
        for (int i = 0; i <= ia; i++)
                for (int j = 0; j <= jb; j++) {
                        double v;
                        if (i == 0 && j == 0) v = 1.0;
                        else if (i > 0) {
                                v = pa * s[i - 1][j];
                                if (i > 1) v += (i - 1) * i2p * s[i - 2][j];
                                if (j > 0) v += j * i2p * s[i - 1][j - 1];
                        } else {
                                v = pb * s[i][j - 1];
                                if (j > 1) v += (j - 1) * i2p * s[i][j - 2];
                        }
                        s[i][j] = v;
                }
}

template <int NR>
__device__ __forceinline__ double i1e_nuclear_roots(const Int1eArgs &a, const double P[3], double p, double i2p,
                                                    const double PA[3], const double AB[3], const int ea[3],
                                                    const int eb[3])
{
        const double *tab = a.table + RysLayout<double>::offset(NR);
        double v = 0.0;
        for (int c = 0; c < a.natm; c++) {
                const double4 C = a.atoms[c];
                const double PC[3] = {P[0] - C.x, P[1] - C.y, P[2] - C.z};
                const double T = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
                double u[NR], w[NR];
                rys_roots_slice<NR, double>(T, tab, u, w);
                double sum = 0.0;
#pragma unroll
                for (int r = 0; r < NR; r++) {
                        const double b10 = (1.0 - u[r]) * i2p;
                        double prod = w[r];
#pragma unroll
                        for (int x = 0; x < 3; x++) {
                                // I(i, 0) for i <= ea + eb, then transfer to (ea, eb)
                                const int n = ea[x] + eb[x];
                                double g[7];
                                const double c00 = PA[x] - u[r] * PC[x];
                                g[0] = 1.0;
                                if (n > 0) g[1] = c00;
                                for (int i = 1; i < n; i++) g[i + 1] = c00 * g[i] + i * b10 * g[i - 1];
                                // transfer: I(i, j) = sum_k binom(j, k) AB^(j-k) I(i + k, 0)
                                double t = 0.0, abp = 1.0;
                                for (int k = eb[x]; k >= 0; k--) {   // term k carries AB^(eb - k)
                                        t += binom(eb[x], k) * abp * g[ea[x] + k];
                                        abp *= AB[x];
                                }
                                prod *= t;
                        }
                        sum += prod;
                }
                v -= C.w * sum;
        }
        return v;
}

static __global__ void int1e_kernel(Int1eArgs a)
{
        const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (e >= a.elem_off[a.npair]) return;
        const int t = i1e_find(a.elem_off, a.npair, e);
        const int4 pr = a.pair[t];
        const double4 Si = a.seg[pr.x], Sj = a.seg[pr.y];
        const int li = (int)Si.w, lj = (int)Sj.w;
        const int nb = (lj + 1) * (lj + 2) / 2;
        const int loc = (int)(e - a.elem_off[t]);
        const int ca = loc / nb, cb = loc % nb;
        int ea[3], eb[3];
        i1e_cart(li, ca, ea);
        i1e_cart(lj, cb, eb);
        const double A[3] = {Si.x, Si.y, Si.z}, B[3] = {Sj.x, Sj.y, Sj.z};
        const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
        const int nr = (li + lj) / 2 + 1;
        double s_sum = 0.0, t_sum = 0.0, v_sum = 0.0;
        for (int ip = 0; ip < pr.w; ip++) {
                const double4 P4 = a.PP[pr.z + ip];
                const double2 K2 = a.PK[pr.z + ip];
                const double2 E2 = a.PE[pr.z + ip];
                const double p = P4.w, i2p = K2.y, K = K2.x, beta = E2.y;
                const double P[3] = {P4.x, P4.y, P4.z};
                const double PA[3] = {P[0] - A[0], P[1] - A[1], P[2] - A[2]};
                const double PB[3] = {P[0] - B[0], P[1] - B[1], P[2] - B[2]};
                double sx[3], tx[3];
                for (int x = 0; x < 3; x++) {
                        double s[4][6];
                        i1e_overlap_1d(PA[x], PB[x], i2p, ea[x], eb[x] + 2, s);
                        const int j = eb[x];
                        sx[x] = s[ea[x]][j];
                        double tk = beta * (2 * j + 1) * s[ea[x]][j] - 2.0 * beta * beta * s[ea[x]][j + 2];
                        if (j > 1) tk -= 0.5 * j * (j - 1) * s[ea[x]][j - 2];
                        tx[x] = tk;
                }
                const double pre = K * M_PI / p * sqrt(M_PI / p);
                s_sum += pre * sx[0] * sx[1] * sx[2];
                t_sum += pre * (tx[0] * sx[1] * sx[2] + sx[0] * tx[1] * sx[2] + sx[0] * sx[1] * tx[2]);
                const double pv = K * 2.0 * M_PI / p;
                double v;
                switch (nr) {
                case 1: v = i1e_nuclear_roots<1>(a, P, p, i2p, PA, AB, ea, eb); break;
                case 2: v = i1e_nuclear_roots<2>(a, P, p, i2p, PA, AB, ea, eb); break;
                case 3: v = i1e_nuclear_roots<3>(a, P, p, i2p, PA, AB, ea, eb); break;
                default: v = i1e_nuclear_roots<4>(a, P, p, i2p, PA, AB, ea, eb); break;
                }
                v_sum += pv * v;
        }
        const size_t n = (size_t)a.naoc;
        const int ci = a.seg_cart[pr.x] + ca, cj = a.seg_cart[pr.y] + cb;
        const double h = t_sum + v_sum;
        a.S[ci * n + cj] = s_sum;
        a.H[ci * n + cj] = h;
        a.S[cj * n + ci] = s_sum;
        a.H[cj * n + ci] = h;
}

// ---------------------------------------------------------------------------
// One-electron part of the RHF nuclear gradient, contracted in the kernel:
// the lines of grad_elec (pyscf/grad/rhf.py:57-66)
//   de[k] += einsum('xij,ij->x', hcore_deriv(k), D)          (:121-143)
//   de[k] -= 2 einsum('xij,ij->x', s1[:, p0:p1], W[p0:p1])    (:145-146)
// written as the derivative of  E1 = sum_ab D_ab h_ab - W_ab S_ab  over the
// Cartesian block of every segment pair (D, W symmetric, Cartesian basis).
// A basis function's centre derivative raises and lowers its exponent:
//   d/dA_x phi_a = 2 alpha phi_{a+1x} - a_x phi_{a-1x},
// so S and T use the 1D Obara-Saika overlaps up to a_x + 1 and b_x + 2, and
// V_C = -Z_C <a|1/r_C|b> uses Rys quadrature with (la + lb + 1)/2 + 1 roots
// for both centre derivatives; the nucleus C gets -(d/dA + d/dB) of its own
// operator (translational invariance).  Overlap and kinetic energy depend on
// A - B only: d/dB = -d/dA.
struct Int1eGradArgs {
        Int1eArgs g;                 // pairs, segments, primitive pairs, atoms, table (S, H unused)
        const int *seg_atom;         // atom of every segment
        const double *D, *W;         // Cartesian naoc x naoc, symmetric
        double *de;                  // natm x 3, accumulated
};

template <int NR>
__device__ __forceinline__ void i1e_grad_nuclear(const double *table, const double P[3], double p, double i2p,
                                                 const double PA[3], const double AB[3], const double4 C,
                                                 const int ea[3], const int eb[3], double alpha, double beta,
                                                 double fac, double vA[3], double vB[3])
{
        const double *tab = table + RysLayout<double>::offset(NR);
        const double PC[3] = {P[0] - C.x, P[1] - C.y, P[2] - C.z};
        const double T = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
        double u[NR], w[NR];
        rys_roots_slice<NR, double>(T, tab, u, w);
#pragma unroll
        for (int r = 0; r < NR; r++) {
                const double b10 = (1.0 - u[r]) * i2p;
                double I0[3], IA[3], IB[3];
#pragma unroll
                for (int x = 0; x < 3; x++) {
                        const int n = ea[x] + eb[x] + 1;
                        double g[8];
                        const double c00 = PA[x] - u[r] * PC[x];
                        g[0] = 1.0;
                        g[1] = c00;
                        for (int i = 1; i < n; i++) g[i + 1] = c00 * g[i] + i * b10 * g[i - 1];
                        // I(i, j) = sum_k binom(j, k) AB^(j-k) I(i + k, 0)
                        auto tr = [&](int i, int j) {
                                double t = 0.0, abp = 1.0;
                                for (int k = j; k >= 0; k--) {
                                        t += binom(j, k) * abp * g[i + k];
                                        abp *= AB[x];
                                }
                                return t;
                        };
                        I0[x] = tr(ea[x], eb[x]);
                        IA[x] = 2.0 * alpha * tr(ea[x] + 1, eb[x]) - (ea[x] > 0 ? ea[x] * tr(ea[x] - 1, eb[x]) : 0.0);
                        IB[x] = 2.0 * beta * tr(ea[x], eb[x] + 1) - (eb[x] > 0 ? eb[x] * tr(ea[x], eb[x] - 1) : 0.0);
                }
                const double fw = fac * w[r];
                vA[0] += fw * IA[0] * I0[1] * I0[2];
                vA[1] += fw * I0[0] * IA[1] * I0[2];
                vA[2] += fw * I0[0] * I0[1] * IA[2];
                vB[0] += fw * IB[0] * I0[1] * I0[2];
                vB[1] += fw * I0[0] * IB[1] * I0[2];
                vB[2] += fw * I0[0] * I0[1] * IB[2];
        }
}

// kinetic 1D factor T(i, j) of the Obara-Saika table s
template <int NI, int NJ>
__device__ __forceinline__ double i1e_kin_1d(const double (&s)[NI][NJ], int i, int j, double beta)
{
        double t = beta * (2 * j + 1) * s[i][j] - 2.0 * beta * beta * s[i][j + 2];
        if (j > 1) t -= 0.5 * j * (j - 1) * s[i][j - 2];
        return t;
}

// One thread per Cartesian element of a segment pair.  The loop over nuclei
// is the same for every lane, so each nucleus's share is summed over the
// warp before one atomic per component.
static __global__ void int1e_grad_kernel(Int1eGradArgs ga)
{
        const Int1eArgs &a = ga.g;
        const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        const bool active = e < a.elem_off[a.npair];
        const int lane = threadIdx.x & 31;
        int4 pr = make_int4(0, 0, 0, 0);
        int ea[3] = {0, 0, 0}, eb[3] = {0, 0, 0};
        int li = 0, lj = 0;
        double A[3] = {0, 0, 0}, AB[3] = {0, 0, 0};
        double fd = 0.0, fw = 0.0;
        if (active) {
                const int t = i1e_find(a.elem_off, a.npair, e);
                pr = a.pair[t];
                const double4 Si = a.seg[pr.x], Sj = a.seg[pr.y];
                li = (int)Si.w;
                lj = (int)Sj.w;
                const int nb = (lj + 1) * (lj + 2) / 2;
                const int loc = (int)(e - a.elem_off[t]);
                const int ca = loc / nb, cb = loc % nb;
                i1e_cart(li, ca, ea);
                i1e_cart(lj, cb, eb);
                A[0] = Si.x; A[1] = Si.y; A[2] = Si.z;
                AB[0] = Si.x - Sj.x; AB[1] = Si.y - Sj.y; AB[2] = Si.z - Sj.z;
                const size_t n = (size_t)a.naoc;
                const int ci = a.seg_cart[pr.x] + ca, cj = a.seg_cart[pr.y] + cb;
                // a pair of two segments stands for the elements (a, b) and (b, a)
                const double f = pr.x == pr.y ? 1.0 : 2.0;
                fd = f * ga.D[ci * n + cj];
                fw = f * ga.W[ci * n + cj];
        }
        double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0};
        if (active) {
                for (int ip = 0; ip < pr.w; ip++) {
                        const double4 P4 = a.PP[pr.z + ip];
                        const double2 K2 = a.PK[pr.z + ip];
                        const double2 E2 = a.PE[pr.z + ip];
                        const double p = P4.w, i2p = K2.y, alpha = E2.x, beta = E2.y;
                        const double PA[3] = {P4.x - A[0], P4.y - A[1], P4.z - A[2]};
                        const double PB[3] = {PA[0] + AB[0], PA[1] + AB[1], PA[2] + AB[2]};
                        const double pre = K2.x * M_PI / p * sqrt(M_PI / p);
                        double sx[3], tx[3], dsx[3], dtx[3];
                        for (int x = 0; x < 3; x++) {
                                double s[5][6];
                                i1e_overlap_1d(PA[x], PB[x], i2p, ea[x] + 1, eb[x] + 2, s);
                                const int i = ea[x], j = eb[x];
                                sx[x] = s[i][j];
                                tx[x] = i1e_kin_1d(s, i, j, beta);
                                dsx[x] = 2.0 * alpha * s[i + 1][j] - (i > 0 ? i * s[i - 1][j] : 0.0);
                                dtx[x] = 2.0 * alpha * i1e_kin_1d(s, i + 1, j, beta) -
                                         (i > 0 ? i * i1e_kin_1d(s, i - 1, j, beta) : 0.0);
                        }
                        for (int x = 0; x < 3; x++) {
                                const int y = (x + 1) % 3, z = (x + 2) % 3;
                                const double dS = pre * dsx[x] * sx[y] * sx[z];
                                const double dT = pre * (dtx[x] * sx[y] * sx[z] + dsx[x] * (tx[y] * sx[z] + sx[y] * tx[z]));
                                const double v = fd * dT - fw * dS;
                                gA[x] += v;
                                gB[x] -= v;
                        }
                }
        }
        for (int c = 0; c < a.natm; c++) {
                const double4 C = a.atoms[c];
                double vA[3] = {0, 0, 0}, vB[3] = {0, 0, 0};
                if (active) {
                        const int nr = (li + lj + 1) / 2 + 1;
                        for (int ip = 0; ip < pr.w; ip++) {
                                const double4 P4 = a.PP[pr.z + ip];
                                const double2 K2 = a.PK[pr.z + ip];
                                const double2 E2 = a.PE[pr.z + ip];
                                const double p = P4.w, i2p = K2.y;
                                const double P[3] = {P4.x, P4.y, P4.z};
                                const double PA[3] = {P4.x - A[0], P4.y - A[1], P4.z - A[2]};
                                const double fac = -C.w * K2.x * 2.0 * M_PI / p;
                                switch (nr) {
                                case 1: i1e_grad_nuclear<1>(a.table, P, p, i2p, PA, AB, C, ea, eb, E2.x, E2.y, fac, vA, vB); break;
                                case 2: i1e_grad_nuclear<2>(a.table, P, p, i2p, PA, AB, C, ea, eb, E2.x, E2.y, fac, vA, vB); break;
                                case 3: i1e_grad_nuclear<3>(a.table, P, p, i2p, PA, AB, C, ea, eb, E2.x, E2.y, fac, vA, vB); break;
                                default: i1e_grad_nuclear<4>(a.table, P, p, i2p, PA, AB, C, ea, eb, E2.x, E2.y, fac, vA, vB); break;
                                }
                        }
                }
#pragma unroll
                for (int x = 0; x < 3; x++) {
                        gA[x] += fd * vA[x];
                        gB[x] += fd * vB[x];
                        double gc = -fd * (vA[x] + vB[x]);
                        for (int o = 16; o > 0; o >>= 1) gc += __shfl_xor_sync(0xffffffffu, gc, o);
                        if (lane == 0 && gc != 0.0) atomicAdd(ga.de + 3 * c + x, gc);
                }
        }
        if (active) {
                const int ia = ga.seg_atom[pr.x], ib = ga.seg_atom[pr.y];
                for (int x = 0; x < 3; x++) {
                        atomicAdd(ga.de + 3 * ia + x, gA[x]);
                        atomicAdd(ga.de + 3 * ib + x, gB[x]);
                }
        }
}

} // namespace b200jk
