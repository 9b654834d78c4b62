// jk_kernels.cuh — sm_100a kernels of the direct-SCF J/K build.
//
// Work decomposition.  Shell pairs (i,j) are grouped into angular classes
// (la >= lb) and, inside a class, sorted by descending Schwarz bound q_ij.
// A quartet class (X|Y) pairs bra class X with ket class Y (X >= Y).  For a
// bra pair ij the ket pairs that can survive the screen
//     q_ij q_kl max(4 D_ji, 4 D_lk, D_jk, D_jl, D_ik, D_il) > tol
// (CVHFnrs8_prescreen, pyscf/lib/vhf/optimizer.c:90-117) form a prefix of the
// sorted ket list, so the work of a class is  sum_ij nkl(ij)  quartets; it is
// cut into chunks (32 quartets for the thread-per-quartet family, 8 for the
// warp-per-quartet family) and a grid-stride loop of warps walks the chunks
// (warp -> chunk -> bra pair by binary search of the chunk prefix sum).  The
// exact per-quartet test is then applied with the parent-shell density bound.
//
// Arithmetic.  Integrals are Cartesian; the density enters in the Cartesian
// AO basis D_c = C^T D C and the results leave as C J_c C^T (C the block
// diagonal real-solid-harmonic map), so no per-quartet transform is done.
// Each unique quartet scatters to its symmetry images with weight 1/deg:
//     Jacc[c,d] += v Ds[a,b],  Jacc[a,b] += v Ds[c,d]      (Ds = D + D^T)
//     Kacc[a,d] += v X[b,c],  Kacc[a,c] += v X[b,d],
//     Kacc[b,d] += v X[a,c],  Kacc[b,c] += v X[a,d]
// and  J = Jacc + Jacc^T,  K = Kacc[D] + Kacc[D^T]^T  (Kacc[D] + Kacc[D]^T for
// symmetric D).  These are the images PySCF's 'ji->s2kl' and 'li->s2kj' /
// 'li->s1kj' scripts accumulate (pyscf/lib/vhf/nr_direct_dot.c:1293-1647).
#pragma once
#include <type_traits>
#include <utility>
#include "rys_math.cuh"

namespace b200jk {

// Pairs of one angular class are stored bucket by bucket (buckets of equal
// primitive-pair count, so the lanes of a warp run loops of equal length),
// each bucket sorted by descending q.  Pair order inside a class is
// (bucket, rank); it defines the canonical ij >= kl of same-class quartets.
#define B2_NBUCKET 4
__host__ __device__ inline int prim_bucket(int nprim_pairs)
{
        return nprim_pairs <= 1 ? 0 : (nprim_pairs <= 4 ? 1 : (nprim_pairs <= 16 ? 2 : 3));
}

struct PairView {
        const int4 *sh;      // (cart AO of i, cart AO of j, parent shell i, parent shell j)
        const int2 *pr;      // (first primitive pair, number of primitive pairs)
        const double *q;     // parent-shell Schwarz bound
        const double *qs;    // prefix-search key: non-increasing inside a bucket, >= q
        const double4 *A;    // (A, 1 if i == j else 0)
        const double4 *AB;   // (A - B, 0)
        int n;
        int boff[B2_NBUCKET + 1];   // bucket b holds pairs [boff[b], boff[b+1])
};

struct JKArgs {
        PairView bra, ket;
        const double4 *PP;           // primitive pair (P, p)
        const double2 *PK;           // primitive pair (K_ab c_i c_j, 1/(2p))
        const long long *chunk_off;  // bra.n * B2_NBUCKET + 1 entries
        const int *nkl;              // per (bra pair, ket bucket)
        const double *dm_cond;       // nbas x nbas (parent shells)
        const double *table;         // Rys tables (padded layout), float64
        const float *table_f;        // the same tables in float32
        const int *kst;              // per (bra pair, ket bucket): first ket of this pass
        const int *goff;             // packed (ox, oy, oz) per Cartesian component (warp family)
        double *Jacc, *Kacc;
        const double *Ds, *Dk;
        unsigned long long *stats;   // [0] quartets, [1] primitive quartets
        const double *dmax4;         // 4 max|D| of the molecule (count kernel of a batch)
        // Ket-side J in packed form (optional): Dpk[kl*NCD + t] holds Ds of ket
        // pair kl's block and Jpk[kl*NCD + t] accumulates its J, density s at
        // + s*pk_stride.  Consecutive lanes work on consecutive kets, so the
        // reads and atomics are contiguous and the arrays stay in L2; nullptr
        // = read Ds and add into Jacc directly.
        const double *Dpk = nullptr;
        double *Jpk = nullptr;
        long long pk_stride = 0;
        // Tiled chunk order (optional): chunk_off then holds the offsets of
        // ntile tiles; tile t covers the bra pairs [(t % ntb)*tile_b, +tile_b)
        // of ket bucket t / ntb, walked ket-chunk-major (chunk k of all its
        // bra pairs, then chunk k + 1), so concurrent warps share ket data and
        // the K rows of few bra pairs.  0 = bra-major chunk order.
        int tiled = 0, tile_b = 16, ntile = 0, ntb = 0;
        double tol;
        int nbas, naoc, n_dm, nk;
        int with_j, with_k, same;
        // density part of the quartet screen: 0 the s8 screen (J and K),
        // 1 its J terms only, 2 its K terms only (B200JK_SCREEN_*)
        int screen = 0;
        // omega^2 of the long-range operator erf(omega r12)/r12, 0 = Coulomb
        double omega2 = 0.0;
};

// Packed ket blocks: src[e] is the Cartesian matrix offset of packed entry e
// (ket pair blocks of every class, in ket-list order).
static __global__ void pack_gather_kernel(const double *__restrict__ Ds, const long long *__restrict__ src,
                                          long long ne, double *__restrict__ Dpk)
{
        const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (e < ne) Dpk[e] = Ds[src[e]];
}

static __global__ void pack_scatter_add_kernel(const double *__restrict__ Jpk, const long long *__restrict__ src,
                                               long long ne, double *__restrict__ Jacc)
{
        const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (e < ne) Jacc[src[e]] += Jpk[e];   // entries are distinct: no atomics
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        return v;
}

__device__ __forceinline__ int find_bra(const long long *off, int n, long long chunk)
{
        int lo = 0, hi = n;  // off[lo] <= chunk < off[hi]
        while (hi - lo > 1) {
                int mid = (lo + hi) >> 1;
                if (__ldg(off + mid) <= chunk) lo = mid;
                else hi = mid;
        }
        return lo;
}

// The reference's per-quartet screens (pyscf/lib/vhf/optimizer.c):
//   s8 (CVHFnrs8_prescreen, :90-117)  q_ij q_kl > tol and
//        max(4 D_ji, 4 D_lk, D_jk, D_jl, D_ik, D_il) q_ij q_kl > tol
//   J  (CVHFnrs8_vj_prescreen, :119-141)  the 4 D_ji, 4 D_lk terms only
//   K  (CVHFnrs8_vk_prescreen, :143-167)  the D_jk, D_jl, D_ik, D_il terms only
// (SCF.get_jk picks J or K when only one is built, pyscf/scf/hf.py:2069-2077).
// The OR of the reference's comparisons equals one comparison of the
// maximum: rounding of d * qq is monotone in d and 4 d is exact.
__device__ __forceinline__ bool quartet_passes(const JKArgs &a, int4 sb, double qij, int4 sk, double qkl)
{
        const double qq = qij * qkl;
        if (!(qq > a.tol)) return false;
        const size_t n = (size_t)a.nbas;
        const double *dc = a.dm_cond;
        const int pi = sb.z, pj = sb.w, pk = sk.z, pl = sk.w;
        double d = 0.0;
        if (a.screen != 2) d = 4.0 * fmax(__ldg(dc + pj * n + pi), __ldg(dc + pl * n + pk));
        if (a.screen != 1) {
                d = fmax(d, fmax(__ldg(dc + pj * n + pk), __ldg(dc + pj * n + pl)));
                d = fmax(d, fmax(__ldg(dc + pi * n + pk), __ldg(dc + pi * n + pl)));
        }
        return d * qq > a.tol;
}

// 2 pi^{5/2}
#define B2_TWO_PI_2P5 34.98683665524972497

// ---------------------------------------------------------------------------
// Count kernel: for bra pair ij and ket bucket b, the prefix of the bucket
// that can pass the screen, split at the mixed-precision threshold: kets with
// q_ij q_kl max|D| >= tau32 form the FP64 part [0, n64), the rest the FP32
// part [n64, n).  pass 0 writes the FP64 part, pass 1 the FP32 part (start in
// kst, length in nkl) with its chunks of `chunk` quartets.  tau32 = 0 keeps
// every quartet in FP64.  Same-class quartets keep kl <= ij in the
// (bucket, rank) order.  Sharded over nshard GPUs, rank `shard` takes the bra
// pairs ij = shard (mod nshard): pairs are sorted by their bound inside a
// bucket, so striding spreads the cost evenly.
// Tiled chunk order: tile t gets tile_b x (the most chunks of its bra pairs)
// chunk slots; slots past a bra pair's own chunks stay idle.
// nslot chunk slots per ket chunk of a tile: tile_b (one bra pair per slot)
// or tile_b / BR (bra runs of the register family's variant 2)
static __global__ void tile_count_kernel(const int *__restrict__ nkl, int nbra, int chunk, int tile_b, int ntb,
                                         int nslot, long long *tile_cnt)
{
        const int t = blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= B2_NBUCKET * ntb) return;
        const int b = t / ntb, t0 = (t % ntb) * tile_b;
        int m = 0;
        for (int ij = t0; ij < min(nbra, t0 + tile_b); ij++) m = max(m, (nkl[ij * B2_NBUCKET + b] + chunk - 1) / chunk);
        tile_cnt[t] = (long long)m * nslot;
}

// chunk -> (segment, chunk of the segment); false for an idle slot
__device__ __forceinline__ bool map_chunk(const JKArgs &a, long long chunk, int chunk_len, int &sgi, int &kc)
{
        if (!a.tiled) {
                sgi = find_bra(a.chunk_off, a.bra.n * B2_NBUCKET, chunk);
                kc = (int)(chunk - a.chunk_off[sgi]);
                return true;
        }
        const int t = find_bra(a.chunk_off, a.ntile, chunk);
        const int l = (int)(chunk - a.chunk_off[t]);
        kc = l / a.tile_b;
        const int ij = (t % a.ntb) * a.tile_b + l % a.tile_b;
        if (ij >= a.bra.n) return false;
        sgi = ij * B2_NBUCKET + t / a.ntb;
        return kc * chunk_len < a.nkl[sgi];
}

// one (bra pair, ket bucket) segment t of a class: its ket range and chunks
__device__ __forceinline__ void count_segment(const PairView &bra, const PairView &ket, int same, double tol,
                                              double dm, int chunk, double tau32, int pass, int shard, int nshard,
                                              int t, int &nkl_out, int &kst_out, long long &nchunk_out)
{
        const int ij = t / B2_NBUCKET, b = t % B2_NBUCKET;
        const double qij = bra.q[ij];
        int cnt = 0, n64 = 0;
        const int lo0 = ket.boff[b], hi0 = ket.boff[b + 1];
        // with nshard > 1 this rank keeps the bra pairs ij = shard (mod nshard)
        const bool mine = nshard <= 1 || ij % nshard == shard;
        if (mine && dm > 0 && qij > 0 && hi0 > lo0) {
                const double thr = tol / (qij * dm);
                int lo = lo0, hi = hi0;
                while (lo < hi) {
                        int mid = (lo + hi) >> 1;
                        if (ket.qs[mid] > thr) lo = mid + 1;
                        else hi = mid;
                }
                cnt = lo - lo0;
                if (same) {
                        int bi = 0;
                        while (bi < B2_NBUCKET - 1 && ij >= bra.boff[bi + 1]) bi++;
                        if (b > bi) cnt = 0;
                        else if (b == bi) cnt = min(cnt, ij - lo0 + 1);
                }
                n64 = cnt;
                if (tau32 > 0) {
                        const double thr32 = tau32 / (qij * dm);
                        lo = lo0;
                        hi = lo0 + cnt;
                        while (lo < hi) {
                                int mid = (lo + hi) >> 1;
                                if (ket.qs[mid] >= thr32) lo = mid + 1;
                                else hi = mid;
                        }
                        n64 = lo - lo0;
                }
        }
        const int start = pass == 0 ? 0 : n64;
        const int len = pass == 0 ? n64 : cnt - n64;
        nkl_out = len;
        kst_out = start;
        nchunk_out = (len + chunk - 1) / chunk;
}

static __global__ void count_kernel(PairView bra, PairView ket, int same, double tol, const double *dmax4,
                                    int chunk, double tau32, int pass, int shard, int nshard, int *nkl, int *kst,
                                    long long *nchunk)
{
        const int t = blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= bra.n * B2_NBUCKET) return;
        count_segment(bra, ket, same, tol, *dmax4, chunk, tau32, pass, shard, nshard, t, nkl[t], kst[t], nchunk[t]);
}

// Count kernel of a batch of molecules: one thread per segment of the batch;
// molecule m owns segments [segoff[m], segoff[m+1]) of the concatenated
// nkl/kst/nchunk arrays.
static __global__ void count_kernel_multi(const JKArgs *__restrict__ margs, const int *__restrict__ segoff, int nmol,
                                          int chunk, double tau32, int pass, int *nkl, int *kst, long long *nchunk)
{
        const int t = blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= segoff[nmol]) return;
        int lo = 0, hi = nmol;   // segoff[lo] <= t < segoff[hi]
        while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (segoff[mid] <= t) lo = mid;
                else hi = mid;
        }
        const JKArgs &a = margs[lo];
        count_segment(a.bra, a.ket, a.same, a.tol > 0 ? a.tol : 0.0, *a.dmax4, chunk, tau32, pass, 0, 1,
                      t - segoff[lo], nkl[t], kst[t], nchunk[t]);
}

// first chunk of every molecule of a batch: mchunk[m] = chunk_off[segoff[m]]
static __global__ void batch_chunk_starts(const long long *chunk_off, const int *segoff, int nmol, long long *mchunk)
{
        const int m = blockIdx.x * blockDim.x + threadIdx.x;
        if (m <= nmol) mchunk[m] = chunk_off[segoff[m]];
}

// ---------------------------------------------------------------------------
// Thread-per-quartet family: one quartet per lane, the Cartesian block in
// registers.  Mid-size classes keep one part of the block at a time: the
// block is cut into NP parts along the first (bra) index; each part re-runs
// the primitive loop (roots and recurrences are cheap next to the assembly)
// and is contracted before the next, so only NG/NP integrals are live.

template <typename F, int... Ps>
__device__ __forceinline__ void for_parts(F &&f, std::integer_sequence<int, Ps...>)
{
        (f(std::integral_constant<int, Ps>{}), ...);
}

template <typename R> __device__ __forceinline__ const R *table_of(const JKArgs &a);
// whether the register family stages the order-nr table slice in shared memory
template <typename R> __host__ __device__ constexpr bool stage_table(int nr)
{
        return sizeof(R) == 4 || nr <= 4;
}
template <> __device__ __forceinline__ const double *table_of<double>(const JKArgs &a) { return a.table; }
template <> __device__ __forceinline__ const float *table_of<float>(const JKArgs &a) { return a.table_f; }

// Kets per lane of the register family (the autotuner picks 1 or ket_run<>
// per class).  With M > 1 a lane evaluates M
// consecutive kets of its bra pair; kets of one bound band are ordered by
// first segment, so consecutive kets mostly share it, and the lane carries
// its K[a,c] and K[b,c] sums in registers while the segment stays the same
// (one atomic per run instead of one per quartet: the contraction is bound
// by the number of L2 atomics).  Classes kept whole in registers (NP = 1)
// whose carried sums are at most 24 doubles.
template <int LA, int LB, int LC, int LD, int NP>
__host__ __device__ constexpr int ket_run()
{
        using K = Class4<LA, LB, LC, LD>;
        return (NP == 1 && K::NA * K::NC + K::NB * K::NC <= 24) ? 4 : 1;
}

// MULTI: one launch for a batch of molecules (b200jk_batch_get_jk).
// margs[m] holds the arguments of molecule m (its pair tables, matrices and
// slices of the batch's chunk arrays, whose chunk numbers are global) and
// mchunk[m] its first chunk in the batch's chunk queue, mchunk[nmol] the end;
// a0 carries the shared fields (tables, statistics).
// Blocks per SM the register family's kernels are compiled for (a
// translation-unit flag, set per class by the build from measured times):
// 0 leaves register allocation to the compiler (an explicit 1 does not: it
// lets the allocator use far more registers); 4 caps a thread at 128
// registers and 3 at 168, trading a few spills for 16 or 12 resident warps
// instead of 8 on the latency-bound classes whose blocks need more.  Float64 kernels only:
// the float32 ones need far fewer registers, and a cap above their natural
// count would only let them grow.
#ifndef B2_THREAD_MINB
#define B2_THREAD_MINB 0
#endif

template <int LA, int LB, int LC, int LD, int NP, typename R, bool MULTI, int KR>
__global__ void __launch_bounds__(128, (sizeof(R) == 8 ? B2_THREAD_MINB : 0)) jk_thread_kernel(JKArgs a0, const JKArgs *__restrict__ margs,
                                                        const long long *__restrict__ mchunk, int nmol)
{
        using K = Class4<LA, LB, LC, LD>;
        static_assert(K::NA % NP == 0, "parts must divide the bra components");
        constexpr int NAP = K::NA / NP;            // bra components per part
        constexpr int NGP = NAP * K::NB * K::NCD;  // integrals per part
        const int lane = threadIdx.x & 31;
        // the order-NR slice of the Rys table: staged in shared memory when
        // small (float64 up to four roots, <= 59 KB; float32 always, <= 27 KB),
        // read from global memory otherwise
        extern __shared__ __align__(32) double smem_dyn[];
        const R *tab = table_of<R>(a0) + RysLayout<R>::offset(K::NR);
        if constexpr (stage_table<R>(K::NR)) {
                constexpr int NS = rys_slice_elems<R>(K::NR);
                const RysVec4<R> *src = reinterpret_cast<const RysVec4<R> *>(tab);
                RysVec4<R> *dst = reinterpret_cast<RysVec4<R> *>(smem_dyn);
                for (int t = threadIdx.x; t < NS / 4; t += blockDim.x) dst[t] = src[t];
                __syncthreads();
                tab = reinterpret_cast<const R *>(smem_dyn);
        }
        const long long total = MULTI ? mchunk[nmol] : a0.chunk_off[a0.tiled ? a0.ntile : a0.bra.n * B2_NBUCKET];
        const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
        unsigned long long nq = 0, npq = 0;
        for (long long chunk = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; chunk < total;
             chunk += nwarps) {
              auto body = [&](const JKArgs &a) {
                const int nseg = a.bra.n * B2_NBUCKET;
                const size_t n = (size_t)a.naoc, nn = n * n;
                constexpr int M = KR;
                int sgi, kc;
                if (!map_chunk(a, chunk, 32 * M, sgi, kc)) return;
                (void)nseg;
                const int ij = sgi / B2_NBUCKET;
                const bool carry = M > 1 && a.n_dm == 1 && a.nk == 1 && a.with_k;
                double acc_a[K::NA * K::NC], acc_b[K::NB * K::NC];
                int cur_c = -1;
                const int4 sb0 = a.bra.sh[ij];
                auto flush = [&]() {
                        if (cur_c < 0) return;
#pragma unroll
                        for (int x = 0; x < K::NA; x++)
#pragma unroll
                                for (int c = 0; c < K::NC; c++)
                                        atomicAdd(a.Kacc + (sb0.x + x) * n + cur_c + c, acc_a[x * K::NC + c]);
#pragma unroll
                        for (int b = 0; b < K::NB; b++)
#pragma unroll
                                for (int c = 0; c < K::NC; c++)
                                        atomicAdd(a.Kacc + (sb0.y + b) * n + cur_c + c, acc_b[b * K::NC + c]);
                };
              for (int jk = 0; jk < M; jk++) {
                const int pos = kc * (32 * M) + lane * M + jk;
                const int kl = a.ket.boff[sgi % B2_NBUCKET] + a.kst[sgi] + pos;
                const int4 sb = a.bra.sh[ij];
                const int2 pb = a.bra.pr[ij];
                const double qij = a.bra.q[ij];
                const double4 Ab = a.bra.A[ij];
                const double4 ABb = a.bra.AB[ij];
                bool active = pos < a.nkl[sgi];
                int4 sk = make_int4(0, 0, 0, 0);
                if (active) {
                        sk = a.ket.sh[kl];
                        active = quartet_passes(a, sb, qij, sk, a.ket.q[kl]);
                }
                int2 pk = make_int2(0, 0);
                R fac = (R)1;
                // coordinates relative to the bra centre A, differenced in
                // float64: keeps the float32 pass accurate for quartets far
                // from the origin
                R C[3] = {0, 0, 0}, CD[3] = {0, 0, 0};
                const R A[3] = {(R)0, (R)0, (R)0}, AB[3] = {(R)ABb.x, (R)ABb.y, (R)ABb.z};
                if (active) {
                        pk = a.ket.pr[kl];
                        const double4 Ak = a.ket.A[kl];
                        const double4 CDk = a.ket.AB[kl];
                        if (Ab.w != 0.0) fac *= (R)0.5;
                        if (Ak.w != 0.0) fac *= (R)0.5;
                        if (a.same && ij == kl) fac *= (R)0.5;
                        C[0] = (R)(Ak.x - Ab.x); C[1] = (R)(Ak.y - Ab.y); C[2] = (R)(Ak.z - Ab.z);
                        CD[0] = (R)CDk.x; CD[1] = (R)CDk.y; CD[2] = (R)CDk.z;
                        nq++;
                        npq += (unsigned long long)pb.y * pk.y;
                }
                const int ia = sb.x, ib = sb.y, ic = sk.x, id = sk.y;
                if (carry && active && ic != cur_c) {
                        flush();
                        cur_c = ic;
#pragma unroll
                        for (int t = 0; t < K::NA * K::NC; t++) acc_a[t] = 0.0;
#pragma unroll
                        for (int t = 0; t < K::NB * K::NC; t++) acc_b[t] = 0.0;
                }
                for_parts([&](auto part_tag) {
                        constexpr int PART = decltype(part_tag)::value;
                        constexpr int A0 = PART * NAP;
                        R Gp[NGP];
#pragma unroll
                        for (int t = 0; t < NGP; t++) Gp[t] = (R)0;
                        if (active) {
                                for (int ip = 0; ip < pb.y; ip++) {
                                        const double4 P = a.PP[pb.x + ip];
                                        const double2 KP = a.PK[pb.x + ip];
                                        const R Kab = (R)KP.x * fac;
                                        const R Pv[3] = {(R)(P.x - Ab.x), (R)(P.y - Ab.y), (R)(P.z - Ab.z)};
                                        for (int kp = 0; kp < pk.y; kp++) {
                                                const double4 Q = a.PP[pk.x + kp];
                                                const double2 KQ = a.PK[pk.x + kp];
                                                const R Qv[3] = {(R)(Q.x - Ab.x), (R)(Q.y - Ab.y), (R)(Q.z - Ab.z)};
                                                PrimQ<R> sq;
                                                prim_setup<R>(sq, (R)P.w, (R)KP.y, Pv, (R)Q.w, (R)KQ.y, Qv, A, C,
                                                              Kab * (R)KQ.x, (R)a.omega2);
                                                add_prim_quartet_part<LA, LB, LC, LD, PART * NGP, NGP, R>(Gp, tab, sq, AB, CD);
                                        }
                                }
                        }
                        // Gp[((x*NB + b)*NC + c)*ND + d] holds bra component A0 + x
                        for (int s = 0; s < a.n_dm; s++) {
                                if (a.with_j) {
                                        const double *Ds = a.Ds + s * nn;
                                        double *J = a.Jacc + s * nn;
                                        if (active) {
                                                double dab[NAP * K::NB];
#pragma unroll
                                                for (int x = 0; x < NAP; x++)
#pragma unroll
                                                        for (int y = 0; y < K::NB; y++)
                                                                dab[x * K::NB + y] = __ldg(Ds + (ia + A0 + x) * n + ib + y);
#pragma unroll
                                                for (int x = 0; x < K::NC; x++)
#pragma unroll
                                                for (int y = 0; y < K::ND; y++) {
                                                        double v = 0.0;
#pragma unroll
                                                        for (int t = 0; t < NAP * K::NB; t++) v += (double)Gp[t * K::NCD + x * K::ND + y] * dab[t];
                                                        if (a.Jpk) atomicAdd(a.Jpk + s * a.pk_stride + (long long)kl * K::NCD + x * K::ND + y, v);
                                                        else atomicAdd(J + (ic + x) * n + id + y, v);
                                                }
                                        }
                                        double dcd[K::NCD];
#pragma unroll
                                        for (int x = 0; x < K::NC; x++)
#pragma unroll
                                                for (int y = 0; y < K::ND; y++)
                                                        dcd[x * K::ND + y] = !active ? 0.0
                                                                : (a.Dpk ? __ldg(a.Dpk + s * a.pk_stride + (long long)kl * K::NCD + x * K::ND + y)
                                                                         : __ldg(Ds + (ic + x) * n + id + y));
#pragma unroll
                                        for (int t = 0; t < NAP * K::NB; t++) {
                                                double v = 0.0;
#pragma unroll
                                                for (int u = 0; u < K::NCD; u++) v += (double)Gp[t * K::NCD + u] * dcd[u];
                                                v = warp_sum(v);
                                                if (lane == 0 && v != 0.0)
                                                        atomicAdd(J + (ia + A0 + t / K::NB) * n + ib + t % K::NB, v);
                                        }
                                }
                                if (a.with_k && active) {
                                        for (int tk = 0; tk < a.nk; tk++) {
                                                const double *X = a.Dk + (s * a.nk + tk) * nn;
                                                double *Kt = a.Kacc + (s * a.nk + tk) * nn;
                                                // K[a,d] += G X[b,c]
                                                {
                                                        double x_[K::NB * K::NC];
#pragma unroll
                                                        for (int b = 0; b < K::NB; b++)
#pragma unroll
                                                                for (int c = 0; c < K::NC; c++) x_[b * K::NC + c] = __ldg(X + (ib + b) * n + ic + c);
#pragma unroll
                                                        for (int x = 0; x < NAP; x++)
#pragma unroll
                                                        for (int d = 0; d < K::ND; d++) {
                                                                double v = 0.0;
#pragma unroll
                                                                for (int b = 0; b < K::NB; b++)
#pragma unroll
                                                                        for (int c = 0; c < K::NC; c++)
                                                                                v += (double)Gp[((x * K::NB + b) * K::NC + c) * K::ND + d] * x_[b * K::NC + c];
                                                                atomicAdd(Kt + (ia + A0 + x) * n + id + d, v);
                                                        }
                                                }
                                                // K[a,c] += G X[b,d]
                                                {
                                                        double x_[K::NB * K::ND];
#pragma unroll
                                                        for (int b = 0; b < K::NB; b++)
#pragma unroll
                                                                for (int d = 0; d < K::ND; d++) x_[b * K::ND + d] = __ldg(X + (ib + b) * n + id + d);
#pragma unroll
                                                        for (int x = 0; x < NAP; x++)
#pragma unroll
                                                        for (int c = 0; c < K::NC; c++) {
                                                                double v = 0.0;
#pragma unroll
                                                                for (int b = 0; b < K::NB; b++)
#pragma unroll
                                                                        for (int d = 0; d < K::ND; d++)
                                                                                v += (double)Gp[((x * K::NB + b) * K::NC + c) * K::ND + d] * x_[b * K::ND + d];
                                                                if (carry) acc_a[(A0 + x) * K::NC + c] += v;
                                                                else atomicAdd(Kt + (ia + A0 + x) * n + ic + c, v);
                                                        }
                                                }
                                                // K[b,d] += G X[a,c]  (this part's a only)
                                                {
                                                        double x_[NAP * K::NC];
#pragma unroll
                                                        for (int x = 0; x < NAP; x++)
#pragma unroll
                                                                for (int c = 0; c < K::NC; c++) x_[x * K::NC + c] = __ldg(X + (ia + A0 + x) * n + ic + c);
#pragma unroll
                                                        for (int b = 0; b < K::NB; b++)
#pragma unroll
                                                        for (int d = 0; d < K::ND; d++) {
                                                                double v = 0.0;
#pragma unroll
                                                                for (int x = 0; x < NAP; x++)
#pragma unroll
                                                                        for (int c = 0; c < K::NC; c++)
                                                                                v += (double)Gp[((x * K::NB + b) * K::NC + c) * K::ND + d] * x_[x * K::NC + c];
                                                                atomicAdd(Kt + (ib + b) * n + id + d, v);
                                                        }
                                                }
                                                // K[b,c] += G X[a,d]  (this part's a only)
                                                {
                                                        double x_[NAP * K::ND];
#pragma unroll
                                                        for (int x = 0; x < NAP; x++)
#pragma unroll
                                                                for (int d = 0; d < K::ND; d++) x_[x * K::ND + d] = __ldg(X + (ia + A0 + x) * n + id + d);
#pragma unroll
                                                        for (int b = 0; b < K::NB; b++)
#pragma unroll
                                                        for (int c = 0; c < K::NC; c++) {
                                                                double v = 0.0;
#pragma unroll
                                                                for (int x = 0; x < NAP; x++)
#pragma unroll
                                                                        for (int d = 0; d < K::ND; d++)
                                                                                v += (double)Gp[((x * K::NB + b) * K::NC + c) * K::ND + d] * x_[x * K::ND + d];
                                                                if (carry) acc_b[b * K::NC + c] += v;
                                                                else atomicAdd(Kt + (ib + b) * n + ic + c, v);
                                                        }
                                                }
                                        }
                                }
                        }
                }, std::make_integer_sequence<int, NP>{});
              }
                if (carry) flush();
              };
                if constexpr (MULTI) body(margs[find_bra(mchunk, nmol, chunk)]);
                else body(a0);
        }
        if (a0.stats) {
                for (int o = 16; o > 0; o >>= 1) {
                        nq += __shfl_xor_sync(0xffffffffu, nq, o);
                        npq += __shfl_xor_sync(0xffffffffu, npq, o);
                }
                if (lane == 0 && nq) {
                        atomicAdd(a0.stats + 0, nq);
                        atomicAdd(a0.stats + 1, npq);
                }
        }
}

// Bra-run length of the register family's launch variant 2 (1: the class
// has none): whole blocks in registers (NP = 1) and at most 32 carried
// doubles per lane (K[a,c], K[a,d] and the ket's J block).
template <int LA, int LB, int LC, int LD, int NP>
__host__ __device__ constexpr int bra_run()
{
        using K = Class4<LA, LB, LC, LD>;
        return (NP == 1 && K::NA * (K::NC + K::ND) + K::NCD <= 32) ? 4 : 1;
}

// Register family, bra runs (launch variant 2, float64 pass of unsharded
// tiled builds with one symmetric density).  A warp takes one chunk of 32
// kets (one per lane) and the BR consecutive bra pairs of one run of its
// tile: kets of the chunk are the same positions of the ket bucket for every
// bra pair of the run (kst = 0 in the float64 pass), so each lane keeps its
// ket's J block and, while consecutive bra pairs share their first segment a
// (pairs of a bound band are ordered by first segment), its K[a,c] and
// K[a,d] sums in registers: one atomic per run instead of one per quartet for
// those images.  K[b,c], K[b,d] still take one atomic per quartet and J[a,b]
// one per bra pair and warp.
template <int LA, int LB, int LC, int LD, int BR>
__global__ void __launch_bounds__(128, B2_THREAD_MINB) jk_thread_run_kernel(JKArgs a)
{
        using K = Class4<LA, LB, LC, LD>;
        constexpr int NG = K::NG;
        const int lane = threadIdx.x & 31;
        extern __shared__ __align__(32) double smem_dyn[];
        const double *tab = a.table + RysLayout<double>::offset(K::NR);
        if constexpr (stage_table<double>(K::NR)) {
                constexpr int NS = rys_slice_elems<double>(K::NR);
                const RysVec4<double> *src = reinterpret_cast<const RysVec4<double> *>(tab);
                RysVec4<double> *dst = reinterpret_cast<RysVec4<double> *>(smem_dyn);
                for (int t = threadIdx.x; t < NS / 4; t += blockDim.x) dst[t] = src[t];
                __syncthreads();
                tab = reinterpret_cast<const double *>(smem_dyn);
        }
        const size_t n = (size_t)a.naoc;
        const int nrun = a.tile_b / BR;   // runs per tile
        const long long total = a.chunk_off[a.ntile];
        const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
        unsigned long long nq = 0, npq = 0;
        for (long long chunk = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; chunk < total;
             chunk += nwarps) {
                const int t = find_bra(a.chunk_off, a.ntile, chunk);
                const int l = (int)(chunk - a.chunk_off[t]);
                const int kc = l / nrun, run = l % nrun;
                const int bucket = t / a.ntb;
                const int ij0 = (t % a.ntb) * a.tile_b + run * BR;
                const int pos = kc * 32 + lane;
                const int kl = a.ket.boff[bucket] + pos;
                const bool ket_ok = kl < a.ket.boff[bucket + 1];
                int4 sk = make_int4(0, 0, 0, 0);
                int2 pk = make_int2(0, 0);
                double4 Ak = make_double4(0, 0, 0, 0), CDk = make_double4(0, 0, 0, 0);
                double qkl = 0.0;
                if (ket_ok) {
                        sk = a.ket.sh[kl];
                        pk = a.ket.pr[kl];
                        Ak = a.ket.A[kl];
                        CDk = a.ket.AB[kl];
                        qkl = a.ket.q[kl];
                }
                const int ic = sk.x, id = sk.y;
                double accj[K::NCD], acc_c[K::NA * K::NC], acc_d[K::NA * K::ND];
#pragma unroll
                for (int u = 0; u < K::NCD; u++) accj[u] = 0.0;
                bool anyj = false, anyk = false;
                int cur_a = -1;
                auto flush_k = [&]() {
                        if (!anyk) return;
#pragma unroll
                        for (int x = 0; x < K::NA; x++) {
#pragma unroll
                                for (int c = 0; c < K::NC; c++) atomicAdd(a.Kacc + (cur_a + x) * n + ic + c, acc_c[x * K::NC + c]);
#pragma unroll
                                for (int d = 0; d < K::ND; d++) atomicAdd(a.Kacc + (cur_a + x) * n + id + d, acc_d[x * K::ND + d]);
                        }
                        anyk = false;
                };
                for (int r = 0; r < BR; r++) {
                        const int ij = ij0 + r;
                        if (ij >= a.bra.n) break;
                        const int sgi = ij * B2_NBUCKET + bucket;
                        const int nk = a.nkl[sgi];
                        if (kc * 32 >= nk) continue;   // warp-uniform
                        const int4 sb = a.bra.sh[ij];
                        const int2 pb = a.bra.pr[ij];
                        const double qij = a.bra.q[ij];
                        const double4 Ab = a.bra.A[ij];
                        const double4 ABb = a.bra.AB[ij];
                        const bool active = pos < nk && quartet_passes(a, sb, qij, sk, qkl);
                        if (sb.x != cur_a) {   // warp-uniform: the bra pair is the warp's
                                flush_k();
                                cur_a = sb.x;
#pragma unroll
                                for (int u = 0; u < K::NA * K::NC; u++) acc_c[u] = 0.0;
#pragma unroll
                                for (int u = 0; u < K::NA * K::ND; u++) acc_d[u] = 0.0;
                        }
                        double G[NG];
#pragma unroll
                        for (int u = 0; u < NG; u++) G[u] = 0.0;
                        if (active) {
                                double fac = 1.0;
                                if (Ab.w != 0.0) fac *= 0.5;
                                if (Ak.w != 0.0) fac *= 0.5;
                                if (a.same && ij == kl) fac *= 0.5;
                                const double A0[3] = {0.0, 0.0, 0.0}, AB[3] = {ABb.x, ABb.y, ABb.z};
                                const double C[3] = {Ak.x - Ab.x, Ak.y - Ab.y, Ak.z - Ab.z};
                                const double CD[3] = {CDk.x, CDk.y, CDk.z};
                                for (int ip = 0; ip < pb.y; ip++) {
                                        const double4 P = a.PP[pb.x + ip];
                                        const double2 KP = a.PK[pb.x + ip];
                                        const double Kab = KP.x * fac;
                                        const double Pv[3] = {P.x - Ab.x, P.y - Ab.y, P.z - Ab.z};
                                        for (int kp = 0; kp < pk.y; kp++) {
                                                const double4 Q = a.PP[pk.x + kp];
                                                const double2 KQ = a.PK[pk.x + kp];
                                                const double Qv[3] = {Q.x - Ab.x, Q.y - Ab.y, Q.z - Ab.z};
                                                PrimQ<double> sq;
                                                prim_setup<double>(sq, P.w, KP.y, Pv, Q.w, KQ.y, Qv, A0, C, Kab * KQ.x, a.omega2);
                                                add_prim_quartet_part<LA, LB, LC, LD, 0, NG, double>(G, tab, sq, AB, CD);
                                        }
                                }
                                nq++;
                                npq += (unsigned long long)pb.y * pk.y;
                                anyk = a.with_k != 0;
                        }
                        const int ia = sb.x, ib = sb.y;
                        // J: bra block summed over the warp, ket block carried
                        if (a.with_j) {
                                double dcd[K::NCD];
#pragma unroll
                                for (int u = 0; u < K::NCD; u++)
                                        dcd[u] = !active ? 0.0
                                                : (a.Dpk ? __ldg(a.Dpk + (long long)kl * K::NCD + u)
                                                         : __ldg(a.Ds + (ic + u / K::ND) * n + id + u % K::ND));
                                if (active) {
                                        anyj = true;
#pragma unroll
                                        for (int x = 0; x < K::NA; x++)
#pragma unroll
                                                for (int y = 0; y < K::NB; y++) {
                                                        const double dab = __ldg(a.Ds + (ia + x) * n + ib + y);
#pragma unroll
                                                        for (int u = 0; u < K::NCD; u++) accj[u] += G[(x * K::NB + y) * K::NCD + u] * dab;
                                                }
                                }
#pragma unroll
                                for (int tt = 0; tt < K::NAB; tt++) {
                                        double v = 0.0;
#pragma unroll
                                        for (int u = 0; u < K::NCD; u++) v += G[tt * K::NCD + u] * dcd[u];
                                        v = warp_sum(v);
                                        if (lane == 0 && v != 0.0) atomicAdd(a.Jacc + (ia + tt / K::NB) * n + ib + tt % K::NB, v);
                                }
                        }
                        if (a.with_k && active) {
                                const double *X = a.Dk;
                                double *Kt = a.Kacc;
#pragma unroll
                                for (int x = 0; x < K::NA; x++) {
                                        // K[a,d] += G X[b,c], K[a,c] += G X[b,d]: carried
#pragma unroll
                                        for (int b = 0; b < K::NB; b++) {
#pragma unroll
                                                for (int c = 0; c < K::NC; c++) {
                                                        const double xbc = __ldg(X + (ib + b) * n + ic + c);
#pragma unroll
                                                        for (int d = 0; d < K::ND; d++)
                                                                acc_d[x * K::ND + d] += G[((x * K::NB + b) * K::NC + c) * K::ND + d] * xbc;
                                                }
#pragma unroll
                                                for (int d = 0; d < K::ND; d++) {
                                                        const double xbd = __ldg(X + (ib + b) * n + id + d);
#pragma unroll
                                                        for (int c = 0; c < K::NC; c++)
                                                                acc_c[x * K::NC + c] += G[((x * K::NB + b) * K::NC + c) * K::ND + d] * xbd;
                                                }
                                        }
                                }
                                // K[b,d] += G X[a,c], K[b,c] += G X[a,d]: one atomic per element
#pragma unroll
                                for (int b = 0; b < K::NB; b++) {
#pragma unroll
                                        for (int d = 0; d < K::ND; d++) {
                                                double v = 0.0;
#pragma unroll
                                                for (int x = 0; x < K::NA; x++)
#pragma unroll
                                                        for (int c = 0; c < K::NC; c++)
                                                                v += G[((x * K::NB + b) * K::NC + c) * K::ND + d] * __ldg(X + (ia + x) * n + ic + c);
                                                atomicAdd(Kt + (ib + b) * n + id + d, v);
                                        }
#pragma unroll
                                        for (int c = 0; c < K::NC; c++) {
                                                double v = 0.0;
#pragma unroll
                                                for (int x = 0; x < K::NA; x++)
#pragma unroll
                                                        for (int d = 0; d < K::ND; d++)
                                                                v += G[((x * K::NB + b) * K::NC + c) * K::ND + d] * __ldg(X + (ia + x) * n + id + d);
                                                atomicAdd(Kt + (ib + b) * n + ic + c, v);
                                        }
                                }
                        }
                }
                if (a.with_k) flush_k();
                if (a.with_j && anyj) {
#pragma unroll
                        for (int u = 0; u < K::NCD; u++) {
                                if (a.Jpk) atomicAdd(a.Jpk + (long long)kl * K::NCD + u, accj[u]);
                                else atomicAdd(a.Jacc + (ic + u / K::ND) * n + id + u % K::ND, accj[u]);
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

// Parts of the register family for a class: 0 = class goes to the shared-
// memory family.  Budget: live integrals of a part plus the three 2D slices
// of one root.  B2_THREAD_PARTS (a translation-unit flag of a class unit,
// set by the build from measured times) replaces the budget's choice for
// that unit's class, which must be a register-family class; it must divide
// the bra's Cartesian components.
template <int LA, int LB, int LC, int LD>
__host__ __device__ constexpr int thread_parts()
{
        using K = Class4<LA, LB, LC, LD>;
#if defined(B2_THREAD_PARTS) && defined(B2_KET_LD)
        if (LA == B2_BRA_LA && LB == B2_BRA_LB && LC == B2_KET_LC && LD == B2_KET_LD) return B2_THREAD_PARTS;
#endif
        if (K::SA > 18 || K::NR > 4) return (K::NG + 3 * K::SA <= 80) ? 1 : 0;
        for (int np = 1; np <= K::NA && np <= 5; np++)
                if (K::NA % np == 0 && K::NG / np + 3 * K::SA <= (np == 1 ? 80 : 72)) return np;
        return 0;
}

// ---------------------------------------------------------------------------
// Warp-per-quartet family: 2D integrals and the Cartesian block in shared
// memory, components spread over the lanes.
template <int LA, int LB, int LC, int LD, typename R = double>
struct WarpSmem {
        using K = Class4<LA, LB, LC, LD>;
        // G[NG] and H[3][NR][SA] in the compute type, then float64 staging
        static constexpr int G = 0;                              // in R units
        static constexpr int H = G + K::NG;                      // in R units
        static constexpr int NRV = K::NG + 3 * K::NR * K::SA;
        static constexpr int DSAB = (int)((NRV * sizeof(R) + 7) / 8);   // doubles from here
        static constexpr int DSCD = DSAB + K::NAB;
        static constexpr int XBC = DSCD + K::NCD;
        static constexpr int XBD = XBC + K::NB * K::NC;
        static constexpr int XAC = XBD + K::NB * K::ND;
        static constexpr int XAD = XAC + K::NA * K::NC;
        static constexpr int SIZE = ((XAD + K::NA * K::ND) + 3) & ~3;   // doubles per group
};

template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void warp_slice_to_smem(R *h, R g00, const RysCoef<R> &rc, int dir, R ab, R cd)
{
        using K = Class4<LA, LB, LC, LD>;
        R g[K::NE * K::NF];
        const R c00 = dir == 0 ? rc.c00[0] : (dir == 1 ? rc.c00[1] : rc.c00[2]);
        const R c00p = dir == 0 ? rc.c00p[0] : (dir == 1 ? rc.c00p[1] : rc.c00p[2]);
        vrr2d<K::NE, K::NF, R>(g, g00, c00, c00p, rc.b10, rc.b01, rc.b00);
        // ket transfer first: u[e][c][d]
        constexpr int NCD1 = (LC + 1) * (LD + 1);
        R u[K::NE * NCD1];
        R cdp[LD + 1];
        cdp[0] = (R)1;
#pragma unroll
        for (int k = 1; k <= LD; k++) cdp[k] = cdp[k - 1] * cd;
#pragma unroll
        for (int e = 0; e < K::NE; e++)
#pragma unroll
        for (int c = 0; c <= LC; c++)
#pragma unroll
        for (int d = 0; d <= LD; d++) {
                R v = (R)0;
#pragma unroll
                for (int k = 0; k <= d; k++) v += (R)binom(d, k) * cdp[d - k] * g[e * K::NF + c + k];
                u[e * NCD1 + c * (LD + 1) + d] = v;
        }
        R abp[LB + 1];
        abp[0] = (R)1;
#pragma unroll
        for (int k = 1; k <= LB; k++) abp[k] = abp[k - 1] * ab;
#pragma unroll
        for (int x = 0; x <= LA; x++)
#pragma unroll
        for (int b = 0; b <= LB; b++)
#pragma unroll
        for (int t = 0; t < NCD1; t++) {
                R v = (R)0;
#pragma unroll
                for (int k = 0; k <= b; k++) v += (R)binom(b, k) * abp[b - k] * u[(x + k) * NCD1 + t];
                h[(x * (LB + 1) + b) * NCD1 + t] = v;
        }
}

// Lanes of one group (GS consecutive lanes of a warp) evaluate one quartet:
// the (root, direction) slices of the 2D integrals are spread over the group,
// then the Cartesian block is accumulated with components spread over it.
// `gl` is the lane index inside the group, `gmask` the group's lane mask.
// A, C, and the P, Q read here are relative to the origin O (the bra centre)
// Components per lane of a group of GS lanes, and whether their packed
// 2D-integral offsets are kept in registers (loaded once per kernel; the
// assembly then reads only the three 2D values from shared memory per
// component and root, instead of a fourth access for the offset).
template <int LA, int LB, int LC, int LD, int GS>
__host__ __device__ constexpr int group_nt()
{
        return (Class4<LA, LB, LC, LD>::NG + GS - 1) / GS;
}
// packed offsets kept in registers for at most this many components a lane
#ifndef B2_GOFF_REGS
#define B2_GOFF_REGS 8
#endif

// (float64 kernels only: the float32 ones are register-bound already)
template <int LA, int LB, int LC, int LD, int GS, typename R>
__host__ __device__ constexpr bool group_goff_in_regs()
{
        return sizeof(R) == 8 && group_nt<LA, LB, LC, LD, GS>() <= B2_GOFF_REGS;
}
template <int LA, int LB, int LC, int LD, int GS, typename R>
__host__ __device__ constexpr int group_goff_regs()
{
        return group_goff_in_regs<LA, LB, LC, LD, GS, R>() ? group_nt<LA, LB, LC, LD, GS>() : 1;
}
template <int LA, int LB, int LC, int LD, int GS, typename R>
__device__ __forceinline__ void group_load_goff(const int *goff, int gl, int *goff_r)
{
        constexpr int NT = group_nt<LA, LB, LC, LD, GS>();
        if constexpr (group_goff_in_regs<LA, LB, LC, LD, GS, R>()) {
#pragma unroll
                for (int i = 0; i < NT; i++) {
                        const int t = gl + i * GS;
                        goff_r[i] = t < Class4<LA, LB, LC, LD>::NG ? __ldg(goff + t) : 0;
                }
        }
}

template <int LA, int LB, int LC, int LD, int GS, typename R>
__device__ __forceinline__ void group_eval_block(double *sm, const JKArgs &a, int2 pb, int2 pk, const double4 O,
                                                 const R A[3], const R AB[3], const R C[3], const R CD[3],
                                                 R fac, int gl, unsigned gmask, const int *goff_r)
{
        using K = Class4<LA, LB, LC, LD>;
        using S = WarpSmem<LA, LB, LC, LD, R>;
        R *G = reinterpret_cast<R *>(sm) + S::G;
        R *H = reinterpret_cast<R *>(sm) + S::H;
        const R *table = table_of<R>(a) + RysLayout<R>::offset(K::NR);
        // the first primitive quartet stores the block, later ones add to it
        // (every pair has at least one primitive pair)
        bool first = true;
        for (int ip = 0; ip < pb.y; ip++) {
                const double4 P = a.PP[pb.x + ip];
                const double2 KP = a.PK[pb.x + ip];
                const R Kab = (R)KP.x * fac;
                const R Pv[3] = {(R)(P.x - O.x), (R)(P.y - O.y), (R)(P.z - O.z)};
                for (int kp = 0; kp < pk.y; kp++) {
                        const double4 Q = a.PP[pk.x + kp];
                        const double2 KQ = a.PK[pk.x + kp];
                        const R Qv[3] = {(R)(Q.x - O.x), (R)(Q.y - O.y), (R)(Q.z - O.z)};
                        __syncwarp(gmask);
                        // one task per root (all three directions) when the slices
                        // are small, else one per (root, direction)
                        constexpr bool PER_ROOT = K::SA <= 16;
                        constexpr int NTASK = PER_ROOT ? K::NR : 3 * K::NR;
                        for (int task = gl; task < NTASK; task += GS) {
                                const int r = PER_ROOT ? task : task / 3;
                                PrimQ<R> sq;
                                prim_setup<R>(sq, (R)P.w, (R)KP.y, Pv, (R)Q.w, (R)KQ.y, Qv, A, C, Kab * (R)KQ.x, (R)a.omega2);
                                R ur, wr;
                                rys_root_one<K::NR, R>(sq.T, table, r, ur, wr);
                                RysCoef<R> rc;
                                rys_coef<R>(rc, ur, sq);
                                const R pref = sq.pref;
                                if constexpr (PER_ROOT) {
                                        warp_slice_to_smem<LA, LB, LC, LD, R>(H + (0 * K::NR + r) * K::SA, (R)1, rc, 0, AB[0], CD[0]);
                                        warp_slice_to_smem<LA, LB, LC, LD, R>(H + (1 * K::NR + r) * K::SA, (R)1, rc, 1, AB[1], CD[1]);
                                        warp_slice_to_smem<LA, LB, LC, LD, R>(H + (2 * K::NR + r) * K::SA, pref * wr, rc, 2, AB[2], CD[2]);
                                } else {
                                        const int dir = task - 3 * r;
                                        const R g00 = dir == 2 ? pref * wr : (R)1;
                                        const R abx = dir == 0 ? AB[0] : (dir == 1 ? AB[1] : AB[2]);
                                        const R cdx = dir == 0 ? CD[0] : (dir == 1 ? CD[1] : CD[2]);
                                        warp_slice_to_smem<LA, LB, LC, LD, R>(H + (dir * K::NR + r) * K::SA, g00, rc, dir, abx, cdx);
                                }
                        }
                        __syncwarp(gmask);
                        constexpr int NT = group_nt<LA, LB, LC, LD, GS>();
                        if constexpr (group_goff_in_regs<LA, LB, LC, LD, GS, R>()) {
#pragma unroll
                                for (int i = 0; i < NT; i++) {
                                        const int t = gl + i * GS;
                                        if (K::NG % GS == 0 || t < K::NG) {
                                                const int o = goff_r[i];
                                                const int ox = o & 1023, oy = (o >> 10) & 1023, oz = o >> 20;
                                                R v = (R)0;
#pragma unroll
                                                for (int r = 0; r < K::NR; r++)
                                                        v += H[r * K::SA + ox] * H[(K::NR + r) * K::SA + oy] * H[(2 * K::NR + r) * K::SA + oz];
                                                G[t] = first ? v : G[t] + v;
                                        }
                                }
                        } else {
                                for (int t = gl; t < K::NG; t += GS) {
                                        const int o = __ldg(a.goff + t);
                                        const int ox = o & 1023, oy = (o >> 10) & 1023, oz = o >> 20;
                                        R v = (R)0;
#pragma unroll
                                        for (int r = 0; r < K::NR; r++)
                                                v += H[r * K::SA + ox] * H[(K::NR + r) * K::SA + oy] * H[(2 * K::NR + r) * K::SA + oz];
                                        G[t] = first ? v : G[t] + v;
                                }
                        }
                        first = false;
                }
        }
        __syncwarp(gmask);
}

// group size (lanes per quartet) of the shared-memory family for a class
template <int LA, int LB, int LC, int LD>
__host__ __device__ constexpr int group_size()
{
        using K = Class4<LA, LB, LC, LD>;
        return K::NG <= 100 ? 8 : (K::NG <= 400 ? 16 : 32);
}

// Blocks per SM the shared-memory family's float64 kernels are compiled for:
// 4 (at most 128 registers a thread) where the groups' shared memory admits 4
// blocks of the launch's size, so that registers do not lower the residency
// the shared memory allows; 0 (compiler's choice) otherwise and for the
// float32 kernels.  Must agree with the
// launch configuration in jk_classes.cu (warps per block, bytes per warp).
template <int LA, int LB, int LC, int LD, typename R, int GS_>
__host__ __device__ constexpr int warp_min_blocks()
{
        constexpr int GS = GS_ > 0 ? GS_ : group_size<LA, LB, LC, LD>();
        constexpr long per_warp = 8L * WarpSmem<LA, LB, LC, LD, R>::SIZE * (32 / GS);
        constexpr long wpb0 = (200L * 1024) / per_warp;
        constexpr long wpb = wpb0 < 1 ? 1 : (wpb0 > 4 ? 4 : wpb0);
        constexpr long by_smem = (227L * 1024) / (per_warp * wpb);
        // float32 kernels: the compiler's choice (0, not 1, which lets the
        // allocator take far more registers)
        if (sizeof(R) == 4) return 0;
#if defined(B2_WARP_MINB) && defined(B2_KET_LD)
        // build-time override of a class unit (build.py WARP_MINB)
        if (LA == B2_BRA_LA && LB == B2_BRA_LB && LC == B2_KET_LC && LD == B2_KET_LD) return B2_WARP_MINB;
#endif
        return by_smem >= 4 ? 4 : 0;
}

// GS_: lanes per quartet (0: group_size<>; the autotuner may pick half of it)
template <int LA, int LB, int LC, int LD, typename R, bool MULTI, int GS_ = 0>
__global__ void __launch_bounds__(128, (warp_min_blocks<LA, LB, LC, LD, R, GS_>())) jk_warp_kernel(JKArgs a0, int chunk_q, const JKArgs *__restrict__ margs,
                                                      const long long *__restrict__ mchunk, int nmol)
{
        using K = Class4<LA, LB, LC, LD>;
        using S = WarpSmem<LA, LB, LC, LD, R>;
        constexpr int GS = GS_ > 0 ? GS_ : group_size<LA, LB, LC, LD>();
        constexpr int NGRP = 32 / GS;
        extern __shared__ __align__(32) double smem_dyn[];
        const int lane = threadIdx.x & 31;
        const int grp = lane / GS, gl = lane % GS;
        const unsigned gmask = GS == 32 ? 0xffffffffu : (((1u << GS) - 1u) << (grp * GS));
        const int wib = threadIdx.x >> 5;
        double *sm = smem_dyn + (size_t)(wib * NGRP + grp) * S::SIZE;
        const long long total = MULTI ? mchunk[nmol] : a0.chunk_off[a0.tiled ? a0.ntile : a0.bra.n * B2_NBUCKET];
        const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
        unsigned long long nq = 0, npq = 0;
        // offsets of this lane's components (the same for every molecule of a batch)
        int goff_r[group_goff_regs<LA, LB, LC, LD, GS, R>()];
        group_load_goff<LA, LB, LC, LD, GS, R>(a0.goff, gl, goff_r);
        // bra-side J of one density: all kets of a chunk share its bra pair, so
        // each lane sums its J[a,b] components over the chunk and the groups
        // of the warp combine them before one atomic per element
        constexpr int NJB = sizeof(R) == 8 ? (K::NAB + GS - 1) / GS : 1;
        for (long long chunk = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; chunk < total;
             chunk += nwarps) {
              auto body = [&](const JKArgs &a) {
                const int nseg = a.bra.n * B2_NBUCKET;
                const size_t n = (size_t)a.naoc, nn = n * n;
                int sgi, kc;
                if (!map_chunk(a, chunk, chunk_q, sgi, kc)) return;
                (void)nseg;
                const int ij = sgi / B2_NBUCKET;
                const int kb = a.ket.boff[sgi % B2_NBUCKET] + a.kst[sgi];
                const int kl0 = kb + kc * chunk_q;
                const int kl1 = kb + min(kc * chunk_q + chunk_q, a.nkl[sgi]);
                const int4 sb = a.bra.sh[ij];
                const int2 pb = a.bra.pr[ij];
                const double qij = a.bra.q[ij];
                const double4 Ab = a.bra.A[ij];
                const double4 ABb = a.bra.AB[ij];
                const R A[3] = {(R)0, (R)0, (R)0}, AB[3] = {(R)ABb.x, (R)ABb.y, (R)ABb.z};
                const int ia = sb.x, ib = sb.y;
                // (float64 kernels only: the float32 ones are register-bound)
                const bool jab_sum = sizeof(R) == 8 && a.with_j && a.n_dm == 1;
                double jab[sizeof(R) == 8 ? NJB : 1];
#pragma unroll
                for (int i = 0; i < NJB; i++) jab[i] = 0.0;
                if (jab_sum) {
                        // the chunk's bra block of Ds, staged once
                        double *dsab = sm + S::DSAB;
                        for (int t = gl; t < K::NAB; t += GS) dsab[t] = __ldg(a.Ds + (ia + t / K::NB) * n + ib + t % K::NB);
                }
                for (int kl = kl0 + grp; kl < kl1; kl += NGRP) {
                        const int4 sk = a.ket.sh[kl];
                        if (!quartet_passes(a, sb, qij, sk, a.ket.q[kl])) continue;
                        const int2 pk = a.ket.pr[kl];
                        const double4 Ak = a.ket.A[kl];
                        const double4 CDk = a.ket.AB[kl];
                        R fac = (R)1;
                        if (Ab.w != 0.0) fac *= (R)0.5;
                        if (Ak.w != 0.0) fac *= (R)0.5;
                        if (a.same && ij == kl) fac *= (R)0.5;
                        const R C[3] = {(R)(Ak.x - Ab.x), (R)(Ak.y - Ab.y), (R)(Ak.z - Ab.z)};
                        const R CD[3] = {(R)CDk.x, (R)CDk.y, (R)CDk.z};
                        group_eval_block<LA, LB, LC, LD, GS, R>(sm, a, pb, pk, Ab, A, AB, C, CD, fac, gl, gmask, goff_r);
                        if (gl == 0) {
                                nq++;
                                npq += (unsigned long long)pb.y * pk.y;
                        }
                        const R *G = reinterpret_cast<const R *>(sm) + S::G;
                        const int ic = sk.x, id = sk.y;
                        for (int s = 0; s < a.n_dm; s++) {
                                if (a.with_j) {
                                        const double *Ds = a.Ds + s * nn;
                                        double *J = a.Jacc + s * nn;
                                        double *dsab = sm + S::DSAB, *dscd = sm + S::DSCD;
                                        if (!jab_sum)
                                                for (int t = gl; t < K::NAB; t += GS) dsab[t] = __ldg(Ds + (ia + t / K::NB) * n + ib + t % K::NB);
                                        for (int t = gl; t < K::NCD; t += GS)
                                                dscd[t] = a.Dpk ? __ldg(a.Dpk + s * a.pk_stride + (long long)kl * K::NCD + t)
                                                                : __ldg(Ds + (ic + t / K::ND) * n + id + t % K::ND);
                                        __syncwarp(gmask);
                                        for (int t = gl; t < K::NCD; t += GS) {
                                                double v = 0.0;
                                                for (int u = 0; u < K::NAB; u++) v += (double)G[u * K::NCD + t] * dsab[u];
                                                if (a.Jpk) atomicAdd(a.Jpk + s * a.pk_stride + (long long)kl * K::NCD + t, v);
                                                else atomicAdd(J + (ic + t / K::ND) * n + id + t % K::ND, v);
                                        }
                                        if (jab_sum) {
#pragma unroll
                                                for (int i = 0; i < NJB; i++) {
                                                        const int t = gl + i * GS;
                                                        if (t < K::NAB) {
                                                                double v = 0.0;
                                                                for (int u = 0; u < K::NCD; u++) v += (double)G[t * K::NCD + u] * dscd[u];
                                                                jab[i] += v;
                                                        }
                                                }
                                        } else {
                                                for (int t = gl; t < K::NAB; t += GS) {
                                                        double v = 0.0;
                                                        for (int u = 0; u < K::NCD; u++) v += (double)G[t * K::NCD + u] * dscd[u];
                                                        atomicAdd(J + (ia + t / K::NB) * n + ib + t % K::NB, v);
                                                }
                                        }
                                        __syncwarp(gmask);
                                }
                                if (a.with_k) {
                                        for (int tk = 0; tk < a.nk; tk++) {
                                                const double *X = a.Dk + (s * a.nk + tk) * nn;
                                                double *Kt = a.Kacc + (s * a.nk + tk) * nn;
                                                double *xbc = sm + S::XBC, *xbd = sm + S::XBD;
                                                double *xac = sm + S::XAC, *xad = sm + S::XAD;
                                                for (int t = gl; t < K::NB * K::NC; t += GS) xbc[t] = __ldg(X + (ib + t / K::NC) * n + ic + t % K::NC);
                                                for (int t = gl; t < K::NB * K::ND; t += GS) xbd[t] = __ldg(X + (ib + t / K::ND) * n + id + t % K::ND);
                                                for (int t = gl; t < K::NA * K::NC; t += GS) xac[t] = __ldg(X + (ia + t / K::NC) * n + ic + t % K::NC);
                                                for (int t = gl; t < K::NA * K::ND; t += GS) xad[t] = __ldg(X + (ia + t / K::ND) * n + id + t % K::ND);
                                                __syncwarp(gmask);
                                                // K[a,d] += G X[b,c]
                                                for (int t = gl; t < K::NA * K::ND; t += GS) {
                                                        const int x = t / K::ND, d = t % K::ND;
                                                        double v = 0.0;
                                                        for (int b = 0; b < K::NB; b++)
                                                                for (int c = 0; c < K::NC; c++)
                                                                        v += (double)G[((x * K::NB + b) * K::NC + c) * K::ND + d] * xbc[b * K::NC + c];
                                                        atomicAdd(Kt + (ia + x) * n + id + d, v);
                                                }
                                                // K[a,c] += G X[b,d]
                                                for (int t = gl; t < K::NA * K::NC; t += GS) {
                                                        const int x = t / K::NC, c = t % K::NC;
                                                        double v = 0.0;
                                                        for (int b = 0; b < K::NB; b++)
                                                                for (int d = 0; d < K::ND; d++)
                                                                        v += (double)G[((x * K::NB + b) * K::NC + c) * K::ND + d] * xbd[b * K::ND + d];
                                                        atomicAdd(Kt + (ia + x) * n + ic + c, v);
                                                }
                                                // K[b,d] += G X[a,c]
                                                for (int t = gl; t < K::NB * K::ND; t += GS) {
                                                        const int b = t / K::ND, d = t % K::ND;
                                                        double v = 0.0;
                                                        for (int x = 0; x < K::NA; x++)
                                                                for (int c = 0; c < K::NC; c++)
                                                                        v += (double)G[((x * K::NB + b) * K::NC + c) * K::ND + d] * xac[x * K::NC + c];
                                                        atomicAdd(Kt + (ib + b) * n + id + d, v);
                                                }
                                                // K[b,c] += G X[a,d]
                                                for (int t = gl; t < K::NB * K::NC; t += GS) {
                                                        const int b = t / K::NC, c = t % K::NC;
                                                        double v = 0.0;
                                                        for (int x = 0; x < K::NA; x++)
                                                                for (int d = 0; d < K::ND; d++)
                                                                        v += (double)G[((x * K::NB + b) * K::NC + c) * K::ND + d] * xad[x * K::ND + d];
                                                        atomicAdd(Kt + (ib + b) * n + ic + c, v);
                                                }
                                                __syncwarp(gmask);
                                        }
                                }
                        }
                }
                if (jab_sum) {
#pragma unroll
                        for (int i = 0; i < NJB; i++) {
                                double v = jab[i];
                                for (int o = GS; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                                const int t = gl + i * GS;
                                if (grp == 0 && t < K::NAB && v != 0.0) atomicAdd(a.Jacc + (ia + t / K::NB) * n + ib + t % K::NB, v);
                        }
                }
              };
                if constexpr (MULTI) body(margs[find_bra(mchunk, nmol, chunk)]);
                else body(a0);
        }
        if (a0.stats && gl == 0 && nq) {
                atomicAdd(a0.stats + 0, nq);
                atomicAdd(a0.stats + 1, npq);
        }
}

// ---------------------------------------------------------------------------
// Schwarz conditioner: one warp per shell pair evaluates (ij|ij), transforms
// the diagonal to the output basis and folds sqrt(max |(ab|ab)|) into the
// parent-shell entry (CVHFnr_int2e_q_cond, pyscf/lib/vhf/optimizer.c:408-454).
struct QArgs {
        double omega2;               // as JKArgs::omega2
        PairView pairs;
        const double4 *PP;
        const double2 *PK;
        const double *table;
        const int *goff;
        const double *c2s;           // [l][10][10] transform rows for the output basis
        unsigned long long *qcond;   // parent nbas x nbas, as bit patterns of positive doubles
        int nbas, cart;
};

template <int LA, int LB>
__global__ void __launch_bounds__(32) qcond_kernel(QArgs q)
{
        using K = Class4<LA, LB, LA, LB>;
        using S = WarpSmem<LA, LB, LA, LB, double>;
        extern __shared__ __align__(32) double smem_dyn[];
        double *sm = smem_dyn;
        const int lane = threadIdx.x & 31;
        const int ij = blockIdx.x;
        if (ij >= q.pairs.n) return;
        JKArgs a;
        a.PP = q.PP;
        a.PK = q.PK;
        a.table = q.table;
        a.goff = q.goff;
        a.omega2 = q.omega2;
        const int4 sh = q.pairs.sh[ij];
        const int2 pr = q.pairs.pr[ij];
        const double4 Av = q.pairs.A[ij];
        const double4 ABv = q.pairs.AB[ij];
        const double A[3] = {0.0, 0.0, 0.0}, AB[3] = {ABv.x, ABv.y, ABv.z};
        int goff_r[group_goff_regs<LA, LB, LA, LB, 32, double>()];
        group_load_goff<LA, LB, LA, LB, 32, double>(q.goff, lane, goff_r);
        group_eval_block<LA, LB, LA, LB, 32, double>(sm, a, pr, pr, Av, A, AB, A, AB, 1.0, lane, 0xffffffffu, goff_r);
        const double *G = sm + S::G;
        const int nsa = q.cart ? K::NA : 2 * LA + 1, nsb = q.cart ? K::NB : 2 * LB + 1;
        const double *ca = q.c2s + LA * 100, *cb = q.c2s + LB * 100;
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
                                                v += c1 * c2 * c3 * c4 * G[((x * K::NB + y) * K::NA + x2) * K::NB + y2];
                                        }
                                }
                        }
                }
                m = fmax(m, fabs(v));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) {
                const double qv = sqrt(fmax(m, 1e-100));
                const unsigned long long bits = (unsigned long long)__double_as_longlong(qv);
                atomicMax(q.qcond + (size_t)sh.z * q.nbas + sh.w, bits);
                atomicMax(q.qcond + (size_t)sh.w * q.nbas + sh.z, bits);
        }
}

// ---------------------------------------------------------------------------
// Density conditioner on parent shells (CVHFnr_dm_cond, optimizer.c:494-518)
// and its global maximum.
static __global__ void dm_cond_kernel(const double *dms, int n_dm, int nao, const int *ao_loc, int nbas,
                               double *dm_cond, unsigned long long *dmax_bits)
{
        const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        const long long npair = (long long)nbas * (nbas + 1) / 2;
        if (t >= npair) return;
        const int I = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
        int Ii = I;
        // guard rounding of the triangular inverse
        while ((long long)Ii * (Ii + 1) / 2 > t) Ii--;
        while ((long long)(Ii + 1) * (Ii + 2) / 2 <= t) Ii++;
        const int J = (int)(t - (long long)Ii * (Ii + 1) / 2);
        const size_t n = nao;
        double m = 0.0;
        for (int s = 0; s < n_dm; s++) {
                const double *D = dms + (size_t)s * n * n;
                for (int a = ao_loc[Ii]; a < ao_loc[Ii + 1]; a++)
                        for (int b = ao_loc[J]; b < ao_loc[J + 1]; b++)
                                m = fmax(m, fabs(D[a * n + b]) + fabs(D[b * n + a]));
        }
        m *= 0.5;
        dm_cond[(size_t)Ii * nbas + J] = m;
        dm_cond[(size_t)J * nbas + Ii] = m;
        atomicMax(dmax_bits, (unsigned long long)__double_as_longlong(4.0 * m));
}

// ---------------------------------------------------------------------------
// Basis maps.  For output-basis AO mu: segment, component; for Cartesian AO:
// segment, component.  seg_info[s] = (l, out offset, cart offset, 0).
static __global__ void out_to_cart_kernel(const double *D, int nao, int naoc, const int *cart_seg,
                                   const int *cart_comp, const int4 *seg_info, const double *c2s,
                                   int cart, double *Dc, double *DcT, double *Ds)
{
        const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= (long long)naoc * naoc) return;
        const int c = (int)(t / naoc), d = (int)(t % naoc);
        const int sc = cart_seg[c], sd = cart_seg[d];
        const int4 ic = seg_info[sc], id = seg_info[sd];
        const int xc = cart_comp[c], xd = cart_comp[d];
        const int nsc = cart ? (ic.x + 1) * (ic.x + 2) / 2 : 2 * ic.x + 1;
        const int nsd = cart ? (id.x + 1) * (id.x + 2) / 2 : 2 * id.x + 1;
        const double *cc = c2s + ic.x * 100, *cd = c2s + id.x * 100;
        double v = 0.0;
        for (int m = 0; m < nsc; m++) {
                const double f1 = cc[m * 10 + xc];
                if (f1 == 0.0) continue;
                const double *row = D + (size_t)(ic.y + m) * nao + id.y;
                double s = 0.0;
                for (int k = 0; k < nsd; k++) s += row[k] * cd[k * 10 + xd];
                v += f1 * s;
        }
        Dc[t] = v;
        if (DcT) DcT[(size_t)d * naoc + c] = v;
        (void)Ds;
}

static __global__ void sym_sum_kernel(const double *X, int n, double *Y)
{
        const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= (long long)n * n) return;
        const int i = (int)(t / n), j = (int)(t % n);
        Y[t] = X[t] + X[(size_t)j * n + i];
}

// out[mu,nu] = sum_ab C[mu,a] (A1[a,b] + A2[b,a]) C[nu,b];  hermi == 2 makes
// the upper triangle the negative of the lower one (lib.hermi_triu).
static __global__ void cart_to_out_kernel(const double *A1, const double *A2, int nao, int naoc,
                                   const int *out_seg, const int *out_comp, const int4 *seg_info,
                                   const double *c2s, int cart, int hermi, double *out)
{
        const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= (long long)nao * nao) return;
        int mu = (int)(t / nao), nu = (int)(t % nao);
        double sign = 1.0;
        if (hermi == 2 && mu < nu) { const int tmp = mu; mu = nu; nu = tmp; sign = -1.0; }
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
                        const size_t b = in_.z + y;
                        s += f2 * (A1[a * naoc + b] + A2[b * naoc + a]);
                }
                v += f1 * s;
        }
        out[t] = sign * v;
        (void)cart;
}

} // namespace b200jk
