// fill_kernels.cuh — the s8-packed two-electron integral tensor of a plan's
// basis: the array mol.intor('int2e', aosym='s8') returns
// (GTO2e_cart_or_sph, pyscf/lib/vhf/fill_nr_s8.c:110-138, entries written by
// store_ij, :72-106).  Element (ij|kl) with i >= j, k >= l and pair indices
// ij = i(i+1)/2 + j >= kl sits at ij(ij+1)/2 + kl.  The reference leaves the
// quartets whose Schwarz bound q_ij q_kl is at most 1e-14 at zero
// (CVHFnr_schwarz_cond, pyscf/lib/vhf/optimizer.c:71-88, with the default
// cutoff of CVHFinit_optimizer, :40); so does this fill (the caller zeroes
// the array first).
//
// One group of GS lanes per quartet, as the shared-memory J/K family: the
// Cartesian block is evaluated into shared memory by group_eval_block (with
// no s8 degeneracy factor), transformed index by index to the output basis
// with the planner's [l][10][10] rows, and scattered to the packed array.
// Every location is written by exactly one lane: inside a segment pair of one
// segment only a >= b is stored, inside a quartet of one pair only ij >= kl.
#pragma once
#include "jk_kernels.cuh"

namespace b200jk {

// Schwarz cutoff of the reference's s8 fill
#define B2_FILL_CUTOFF 1e-14

struct FillArgs {
        JKArgs jk;                  // pairs, primitive pairs, Rys table, chunk lists, tol = cutoff
        const int *cart_seg;        // segment of every Cartesian AO
        const int4 *seg_info;       // (l, output offset, Cartesian offset, parent shell) per segment
        const double *c2s;          // [l][10][10] rows of the output basis
        int cart;                   // output basis Cartesian (1) or real spherical (0)
        double *eri;                // s8 packed, nao_pair (nao_pair + 1) / 2 entries
};

template <int LA, int LB, int LC, int LD>
struct FillSmem {
        using K = Class4<LA, LB, LC, LD>;
        using W = WarpSmem<LA, LB, LC, LD, double>;
        // G (the block) at 0 as in WarpSmem; the transform's second buffer
        // at NG, over the 2D slices, which are dead once the block is done
        static constexpr int T = K::NG;
        static constexpr int SIZE0 = 2 * K::NG > W::SIZE ? 2 * K::NG : W::SIZE;
        static constexpr int SIZE = (SIZE0 + 3) & ~3;
};

__device__ __forceinline__ int fill_nout(int l, int cart) { return cart ? (l + 1) * (l + 2) / 2 : 2 * l + 1; }

// out[a][m][c] = sum_k rows[m][k] in[a][k][c]: one index (n Cartesian
// components -> m output components) between `outer` and `inner` dims
__device__ __forceinline__ void fill_transform(const double *in, double *out, int outer, int n, int m, int inner,
                                               const double *__restrict__ rows, int gl, int gs)
{
        const int total = outer * m * inner;
        for (int e = gl; e < total; e += gs) {
                const int c = e % inner;
                const int t = e / inner;
                const int mi = t % m, a = t / m;
                const double *src = in + (size_t)a * n * inner + c;
                double v = 0.0;
                for (int k = 0; k < n; k++) v += __ldg(rows + mi * 10 + k) * src[k * inner];
                out[e] = v;
        }
}

__device__ __forceinline__ long long fill_pair(int i, int j)
{
        return i >= j ? (long long)i * (i + 1) / 2 + j : (long long)j * (j + 1) / 2 + i;
}

template <int LA, int LB, int LC, int LD, int GS>
__device__ __forceinline__ void fill_store(double *sm, const FillArgs &f, int4 sb, int4 sk, bool same_pair, int gl,
                                           unsigned gmask)
{
        using K = Class4<LA, LB, LC, LD>;
        using S = FillSmem<LA, LB, LC, LD>;
        double *G = sm, *T = sm + S::T;
        const int ma = fill_nout(LA, f.cart), mb = fill_nout(LB, f.cart);
        const int mc = fill_nout(LC, f.cart), md = fill_nout(LD, f.cart);
        fill_transform(G, T, K::NA * K::NB * K::NC, K::ND, md, 1, f.c2s + LD * 100, gl, GS);
        __syncwarp(gmask);
        fill_transform(T, G, K::NA * K::NB, K::NC, mc, md, f.c2s + LC * 100, gl, GS);
        __syncwarp(gmask);
        fill_transform(G, T, K::NA, K::NB, mb, mc * md, f.c2s + LB * 100, gl, GS);
        __syncwarp(gmask);
        fill_transform(T, G, 1, K::NA, ma, mb * mc * md, f.c2s + LA * 100, gl, GS);
        __syncwarp(gmask);
        const int oa = f.seg_info[f.cart_seg[sb.x]].y, ob = f.seg_info[f.cart_seg[sb.y]].y;
        const int oc = f.seg_info[f.cart_seg[sk.x]].y, od = f.seg_info[f.cart_seg[sk.y]].y;
        const bool same_ab = sb.x == sb.y, same_cd = sk.x == sk.y;
        const int total = ma * mb * mc * md;
        for (int e = gl; e < total; e += GS) {
                const int d = e % md, c = (e / md) % mc, b = (e / (md * mc)) % mb, a = e / (md * mc * mb);
                const int ia = oa + a, ib = ob + b, ic = oc + c, id = od + d;
                if (same_ab && ia < ib) continue;
                if (same_cd && ic < id) continue;
                const long long p = fill_pair(ia, ib), q = fill_pair(ic, id);
                if (same_pair && p < q) continue;
                const long long hi = p >= q ? p : q, lo = p >= q ? q : p;
                f.eri[hi * (hi + 1) / 2 + lo] = G[e];
        }
        __syncwarp(gmask);
}

// The chunk walk of the shared-memory J/K family (bra-major order), the
// Schwarz test alone per quartet.
template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(128) fill_kernel(FillArgs f, int chunk_q)
{
        using S = FillSmem<LA, LB, LC, LD>;
        constexpr int GS = group_size<LA, LB, LC, LD>();
        constexpr int NGRP = 32 / GS;
        extern __shared__ __align__(32) double smem_dyn[];
        const JKArgs &a = f.jk;
        const int lane = threadIdx.x & 31;
        const int grp = lane / GS, gl = lane % GS;
        const unsigned gmask = GS == 32 ? 0xffffffffu : (((1u << GS) - 1u) << (grp * GS));
        const int wib = threadIdx.x >> 5;
        double *sm = smem_dyn + (size_t)(wib * NGRP + grp) * S::SIZE;
        const long long total = a.chunk_off[a.bra.n * B2_NBUCKET];
        const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
        int goff_r[group_goff_regs<LA, LB, LC, LD, GS, double>()];
        group_load_goff<LA, LB, LC, LD, GS, double>(a.goff, gl, goff_r);
        for (long long chunk = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; chunk < total;
             chunk += nwarps) {
                int sgi, kc;
                if (!map_chunk(a, chunk, chunk_q, sgi, kc)) continue;
                const int ij = sgi / B2_NBUCKET;
                const int kb = a.ket.boff[sgi % B2_NBUCKET] + a.kst[sgi];
                const int kl0 = kb + kc * chunk_q;
                const int kl1 = kb + min(kc * chunk_q + chunk_q, a.nkl[sgi]);
                const int4 sb = a.bra.sh[ij];
                const int2 pb = a.bra.pr[ij];
                const double qij = a.bra.q[ij];
                const double4 Ab = a.bra.A[ij];
                const double4 ABb = a.bra.AB[ij];
                const double A[3] = {0.0, 0.0, 0.0}, AB[3] = {ABb.x, ABb.y, ABb.z};
                for (int kl = kl0 + grp; kl < kl1; kl += NGRP) {
                        const int4 sk = a.ket.sh[kl];
                        if (!(qij * a.ket.q[kl] > a.tol)) continue;
                        const int2 pk = a.ket.pr[kl];
                        const double4 Ak = a.ket.A[kl];
                        const double4 CDk = a.ket.AB[kl];
                        const double C[3] = {Ak.x - Ab.x, Ak.y - Ab.y, Ak.z - Ab.z};
                        const double CD[3] = {CDk.x, CDk.y, CDk.z};
                        group_eval_block<LA, LB, LC, LD, GS, double>(sm, a, pb, pk, Ab, A, AB, C, CD, 1.0, gl, gmask,
                                                                     goff_r);
                        fill_store<LA, LB, LC, LD, GS>(sm, f, sb, sk, a.same && ij == kl, gl, gmask);
                }
        }
}

} // namespace b200jk
