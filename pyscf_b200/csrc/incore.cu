// incore.cu — J and K from a stored two-electron integral tensor: the in-core
// path of the reference, _vhf.incore (pyscf/scf/_vhf.py:318-401) driving
// CVHFnrs8_incore_drv / CVHFnrs4_incore_drv with the contractions of
// pyscf/lib/vhf/nr_incore.c (CVHFics8_tridm_vj :389, CVHFics8_jk_s2il :422,
// CVHFics8_jk_s1il :413, CVHFics4_kl_s2ij :461, CVHFics4_il_s1jk :438).
//
// Tensor layouts (pair index ij = i(i+1)/2 + j, i >= j; npair pairs):
//   s8  entry (ij|kl), ij >= kl, at ij(ij+1)/2 + kl;
//   s4  entry (ij|kl) at ij * npair + kl.
// A stored entry v = (ij|kl) stands for its symmetry images (a,b,c,d); image
// (a,b,c,d) adds v D[b,c] to K[a,d] and v D[a,b] to J[c,d].  A pass
// accumulates, with weight w = 1/(number of images that coincide),
//   A[i,l] += w v D[j,k]   A[j,l] += w v D[i,k]
//   A[i,k] += w v D[j,l]   A[j,k] += w v D[i,l]
// (the images that keep the order of the two pairs) and packed J
//   Jp[kl] += v t[ij]      Jp[ij] += v t[kl]  (s8 only; weight 1/2 if ij == kl)
// with t[ij] = D[i,j] + D[j,i] (D[i,i] on the diagonal).  The pair-swapped
// images are then, for s8, A(D^T)^T (so K = A(D) + A(D)^T for symmetric D),
// and for s4 the swapped entries are stored themselves (K = A(D)).
//
// Work decomposition: a thread block owns the packed rows ij of one pair of
// AO blocks (i in block I, j in block J, I >= J, B AOs a block) and a window
// of packed columns kl.  Each thread takes one column kl of a 256-column
// chunk and walks the block's rows, so every row's chunk is one coalesced
// 2 KB read and each entry is read from HBM once.  Two kernels share the
// windows: incore_fast_kernel takes every full block, in one launch of four
// variants -- the interior of the packed matrix (blocks I > J, columns
// before the block's rows: no per-entry test or weight), the windows of such
// blocks that reach their rows (EDGE: q <= p tested per entry), and the same
// two for the diagonal blocks I == J (DIAG: rows j > i skipped, the K images
// of j == i halved) -- and incore_pass_kernel the blocks of the partial last
// block row with every test.  The fast kernel sends the K images and J row
// sums of a lane's register sums straight to the accumulators with float64
// reductions (after a warp reduction where all lanes share k); the general
// one stages them in shared-memory slabs.  J row sums are reduce-scattered
// across the warp.  The bound is HBM: 8 bytes per stored entry.
#include <vector>
#include "incore_launch.h"

namespace b200jk {

namespace {

constexpr int NT = 256;   // threads per block = packed columns per chunk

__device__ __forceinline__ void pair_of(long long q, int &k, int &l)
{
        // k = floor((sqrt(8q + 1) - 1) / 2), corrected for rounding
        int kk = (int)((sqrt(8.0 * (double)q + 1.0) - 1.0) * 0.5);
        while ((long long)kk * (kk + 1) / 2 > q) kk--;
        while ((long long)(kk + 1) * (kk + 2) / 2 <= q) kk++;
        k = kk;
        l = (int)(q - (long long)kk * (kk + 1) / 2);
}

// N values a lane -> each value summed over the warp; lane gets the sum of
// value `row` (lanes that share `row` hold the same sum; the one with
// (lane & (32 / N - 1)) == 0 writes it)
template <int N>
__device__ __forceinline__ double reduce_scatter(double (&v)[N], int lane, int &row)
{
        int base = 0;
        int off = 16;
#pragma unroll
        for (int h = N / 2; h >= 1; h /= 2) {
                const bool up = (lane & off) != 0;
#pragma unroll
                for (int m = 0; m < h; m++) {
                        const double send = up ? v[m] : v[m + h];
                        const double keep = up ? v[m + h] : v[m];
                        v[m] = keep + __shfl_xor_sync(0xffffffffu, send, off);
                }
                if (up) base += h;
                off >>= 1;
        }
        double s = v[0];
        for (; off >= 1; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        row = base;
        return s;
}

__device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        return v;
}

template <int B, bool S8>
__global__ void __launch_bounds__(NT, 2) incore_pass_kernel(IncoreArgs a)
{
        extern __shared__ __align__(16) double sm[];
        const int nao = a.nao;
        double *DI = sm, *DJ = DI + B * nao, *SI = DJ + B * nao, *SJ = SI + B * nao, *RJ = SJ + B * nao;
        const int4 it = a.items[blockIdx.x];
        const int i0 = it.x * B, j0 = it.y * B;
        const int ni = min(B, nao - i0), nj = min(B, nao - j0);
        const int tid = threadIdx.x, lane = tid & 31;
        for (int e = tid; e < B * nao; e += NT) {
                const int r = e / nao, x = e % nao;
                DI[e] = r < ni ? a.D[(size_t)(i0 + r) * nao + x] : 0.0;
                DJ[e] = r < nj ? a.D[(size_t)(j0 + r) * nao + x] : 0.0;
                SI[e] = 0.0;
                SJ[e] = 0.0;
        }
        for (int e = tid; e < B * B; e += NT) RJ[e] = 0.0;
        __syncthreads();
        const long long c0 = it.z, c1 = it.w;
        for (long long qb = c0; qb < c1; qb += NT) {
                const long long q = qb + tid;
                const bool active = q < c1;
                int k = 0, l = 0;
                if (active) pair_of(q, k, l);
                const double tq = active ? a.t[q] : 0.0;
                const double wkl = k == l ? 0.5 : 1.0;
                // whether all lanes of the warp share k (images into column k)
                const int k0 = __shfl_sync(0xffffffffu, k, 0);
                const bool kuni = __all_sync(0xffffffffu, !active || k == k0);
                double acc2[B], acc4[B];
#pragma unroll
                for (int jj = 0; jj < B; jj++) {
                        acc2[jj] = 0.0;
                        acc4[jj] = 0.0;
                }
                double colj = 0.0;
                for (int ii = 0; ii < ni; ii++) {
                        const int i = i0 + ii;
                        const long long pbase = (long long)i * (i + 1) / 2;
                        // s8: rows before the chunk hold none of its columns
                        if (S8 && pbase + min(i, j0 + nj - 1) < qb) continue;
                        const double dik = DI[ii * nao + k], dil = DI[ii * nao + l];
                        double v[B];
#pragma unroll
                        for (int jj = 0; jj < B; jj++) {
                                const int j = j0 + jj;
                                const long long p = pbase + j;
                                const bool ok = active && jj < nj && j <= i && (!S8 || q <= p);
                                v[jj] = ok ? __ldg(a.eri + (S8 ? p * (p + 1) / 2 + q : p * a.npair + q)) : 0.0;
                        }
                        double acc1 = 0.0, acc3 = 0.0, rp[B];
#pragma unroll
                        for (int jj = 0; jj < B; jj++) rp[jj] = 0.0;
#pragma unroll
                        for (int jj = 0; jj < B; jj++) {
                                const int j = j0 + jj;
                                const long long p = pbase + j;
                                const double wpq = (S8 && p == q) ? 0.5 : 1.0;
                                const double vj = v[jj] * wpq;
                                const double vw = vj * (i == j ? 0.5 : 1.0) * wkl;
                                acc1 += vw * DJ[jj * nao + k];
                                acc3 += vw * DJ[jj * nao + l];
                                acc2[jj] += vw * dik;
                                acc4[jj] += vw * dil;
                                if (a.Jp) {
                                        const bool rowok = jj < nj && j <= i;
                                        colj += vj * (rowok ? __ldg(a.t + p) : 0.0);
                                        rp[jj] = vj * tq;
                                }
                        }
                        if (active) atomicAdd(SI + ii * nao + l, acc1);
                        if (kuni) {
                                acc3 = warp_sum_d(acc3);
                                if (lane == 0) atomicAdd(SI + ii * nao + k0, acc3);
                        } else if (active) {
                                atomicAdd(SI + ii * nao + k, acc3);
                        }
                        if (S8 && a.Jp) {
                                int row;
                                const double s = reduce_scatter<B>(rp, lane, row);
                                if ((lane & (32 / B - 1)) == 0 && s != 0.0) atomicAdd(RJ + ii * B + row, s);
                        }
                }
#pragma unroll
                for (int jj = 0; jj < B; jj++)
                        if (active && acc2[jj] != 0.0) atomicAdd(SJ + jj * nao + l, acc2[jj]);
                if (kuni) {
                        int row;
                        const double s = reduce_scatter<B>(acc4, lane, row);
                        if ((lane & (32 / B - 1)) == 0 && s != 0.0) atomicAdd(SJ + row * nao + k0, s);
                } else if (active) {
#pragma unroll
                        for (int jj = 0; jj < B; jj++)
                                if (acc4[jj] != 0.0) atomicAdd(SJ + jj * nao + k, acc4[jj]);
                }
                if (a.Jp && active && colj != 0.0) atomicAdd(a.Jp + q, colj);
        }
        __syncthreads();
        for (int e = tid; e < B * nao; e += NT) {
                const int r = e / nao, x = e % nao;
                if (r < ni && SI[e] != 0.0) atomicAdd(a.A + (size_t)(i0 + r) * nao + x, SI[e]);
                if (r < nj && SJ[e] != 0.0) atomicAdd(a.A + (size_t)(j0 + r) * nao + x, SJ[e]);
        }
        if (S8 && a.Jp)
                for (int e = tid; e < B * B; e += NT) {
                        const int ii = e / B, jj = e % B;
                        const int i = i0 + ii, j = j0 + jj;
                        if (ii < ni && jj < nj && j <= i && RJ[e] != 0.0)
                                atomicAdd(a.Jp + (long long)i * (i + 1) / 2 + j, RJ[e]);
                }
}

// The interior of the packed matrix: full AO blocks I > J (so i > j for
// every row) and, for s8, columns before the block's first row (so q < p for
// every entry).  No entry needs a validity test, rows follow each other by
// their length, and the only symmetry weight is the column's own k == l,
// applied once to the K sums of a lane.  The K images and the J row sums go
// straight to the (L2-resident) accumulators with fire-and-forget float64
// reductions, about one per four entries, so the block keeps only the two
// density slabs in shared memory and needs no flush.
// EDGE: the windows of such a block that reach its rows (s8): an entry is
// stored only for q <= p and counts half on the packed diagonal q == p.
// DIAG: a diagonal block I == J, whose rows are the pairs j <= i (the others
// are skipped, uniformly over the block) and count half for j == i.
template <int B, bool S8, bool EDGE, bool DIAG>
__device__ __forceinline__ void incore_fast_body(const IncoreArgs &a, const int4 it)
{
        extern __shared__ __align__(16) double sm[];
        const int nao = a.nao;
        double *DI = sm, *DJ = DI + B * nao;
        const int i0 = it.x * B, j0 = it.y * B;
        const int tid = threadIdx.x, lane = tid & 31;
        for (int e = tid; e < B * nao; e += NT) {
                const int r = e / nao, x = e % nao;
                DI[e] = a.D[(size_t)(i0 + r) * nao + x];
                DJ[e] = a.D[(size_t)(j0 + r) * nao + x];
        }
        __syncthreads();
        double *AI = a.A + (size_t)i0 * nao, *AJ = a.A + (size_t)j0 * nao;
        const long long c0 = it.z, c1 = it.w;
        for (long long qb = c0; qb < c1; qb += NT) {
                const long long q = qb + tid;
                const bool active = q < c1;
                int k = 0, l = 0;
                if (active) pair_of(q, k, l);
                const double tq = active ? a.t[q] : 0.0;
                const double wkl = k == l ? 0.5 : 1.0;
                const int k0 = __shfl_sync(0xffffffffu, k, 0);
                const bool kuni = __all_sync(0xffffffffu, !active || k == k0);
                double acc2[B], acc4[B];
#pragma unroll
                for (int jj = 0; jj < B; jj++) {
                        acc2[jj] = 0.0;
                        acc4[jj] = 0.0;
                }
                double colj = 0.0;
                for (int ii = 0; ii < B; ii++) {
                        const int i = i0 + ii;
                        const long long p0 = (long long)i * (i + 1) / 2 + j0;
                        // edge windows: rows before the chunk hold none of its columns
                        if (EDGE && p0 + B - 1 < qb) continue;
                        const double *row = a.eri + (S8 ? p0 * (p0 + 1) / 2 : p0 * a.npair) + q;
                        double v[B];
#pragma unroll
                        for (int jj = 0; jj < B; jj++) {
                                // DIAG rows j > i do not exist
                                const bool rowok = !DIAG || jj <= ii;
                                if (EDGE) {
                                        const long long p = p0 + jj;
                                        v[jj] = rowok && active && q <= p ? __ldg(row) * (q == p ? 0.5 : 1.0) : 0.0;
                                } else {
                                        v[jj] = rowok && active ? __ldg(row) : 0.0;
                                }
                                row += S8 ? p0 + jj + 1 : a.npair;   // next row: p + 1 entries on (s8)
                        }
                        const double dik = DI[ii * nao + k], dil = DI[ii * nao + l];
                        double acc1 = 0.0, acc3 = 0.0, rp[B];
#pragma unroll
                        for (int jj = 0; jj < B; jj++) {
                                // the K images of a row j == i count half (DIAG)
                                const double vk = DIAG && jj == ii ? 0.5 * v[jj] : v[jj];
                                acc1 += vk * DJ[jj * nao + k];
                                acc3 += vk * DJ[jj * nao + l];
                                acc2[jj] += vk * dik;
                                acc4[jj] += vk * dil;
                                colj += v[jj] * __ldg(a.t + p0 + jj);
                                rp[jj] = v[jj] * tq;
                        }
                        if (active && acc1 != 0.0) atomicAdd(AI + (size_t)ii * nao + l, wkl * acc1);
                        if (kuni) {
                                acc3 = warp_sum_d(wkl * acc3);
                                if (lane == 0 && acc3 != 0.0) atomicAdd(AI + (size_t)ii * nao + k0, acc3);
                        } else if (active && acc3 != 0.0) {
                                atomicAdd(AI + (size_t)ii * nao + k, wkl * acc3);
                        }
                        if (S8 && a.Jp) {
                                int rrow;
                                const double s = reduce_scatter<B>(rp, lane, rrow);
                                if ((lane & (32 / B - 1)) == 0 && s != 0.0) atomicAdd(a.Jp + p0 + rrow, s);
                        }
                }
#pragma unroll
                for (int jj = 0; jj < B; jj++) {
                        acc2[jj] *= wkl;
                        acc4[jj] *= wkl;
                        if (active && acc2[jj] != 0.0) atomicAdd(AJ + (size_t)jj * nao + l, acc2[jj]);
                }
                if (kuni) {
                        int rrow;
                        const double s = reduce_scatter<B>(acc4, lane, rrow);
                        if ((lane & (32 / B - 1)) == 0 && s != 0.0) atomicAdd(AJ + (size_t)rrow * nao + k0, s);
                } else if (active) {
#pragma unroll
                        for (int jj = 0; jj < B; jj++)
                                if (acc4[jj] != 0.0) atomicAdd(AJ + (size_t)jj * nao + k, acc4[jj]);
                }
                if (a.Jp && active && colj != 0.0) atomicAdd(a.Jp + q, colj);
        }
}

// One launch for the four variants: blocks take the items of variant 0
// (the bulk of the tensor) first, then those of 1, 2 and 3, which fill the
// tail of the launch.
template <int B, bool S8>
__global__ void __launch_bounds__(NT, 2) incore_fast_kernel(IncoreArgs a)
{
        // (the item lists are selected by constant indices: a run-time index
        // into the parameter array would copy it to local memory)
        int b = blockIdx.x;
        if (b < a.nf[0]) {
                incore_fast_body<B, S8, false, false>(a, a.fitems[0][b]);
                return;
        }
        b -= a.nf[0];
        if (b < a.nf[1]) {
                incore_fast_body<B, S8, true, false>(a, a.fitems[1][b]);
                return;
        }
        b -= a.nf[1];
        if (b < a.nf[2]) {
                incore_fast_body<B, S8, false, true>(a, a.fitems[2][b]);
                return;
        }
        b -= a.nf[2];
        incore_fast_body<B, S8, true, true>(a, a.fitems[3][b]);
}

__global__ void tridm_kernel(const double *__restrict__ D, int nao, double *__restrict__ t)
{
        const long long np = (long long)nao * (nao + 1) / 2;
        const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (p >= np) return;
        int i, j;
        pair_of(p, i, j);
        t[p] = i == j ? D[(size_t)i * nao + i] : D[(size_t)i * nao + j] + D[(size_t)j * nao + i];
}

__global__ void unpack_j_kernel(const double *__restrict__ Jp, int nao, double *__restrict__ vj)
{
        const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (e >= (long long)nao * nao) return;
        const int x = (int)(e / nao), y = (int)(e % nao);
        const int hi = x >= y ? x : y, lo = x >= y ? y : x;
        vj[e] = Jp[(long long)hi * (hi + 1) / 2 + lo];
}

__global__ void finish_k_kernel(const double *__restrict__ A1, const double *__restrict__ A2, int nao, int mode,
                                int hermi, double *__restrict__ vk)
{
        const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (e >= (long long)nao * nao) return;
        int x = (int)(e / nao), y = (int)(e % nao);
        double sign = 1.0;
        // hermi_triu: the upper triangle is the (negated) mirror of the lower
        if (hermi != 0 && x < y) {
                const int t = x; x = y; y = t;
                if (hermi == 2) sign = -1.0;
        }
        const size_t xy = (size_t)x * nao + y, yx = (size_t)y * nao + x;
        double v;
        switch (mode) {
        case 0: v = A1[xy] + A2[yx]; break;
        case 1: v = A1[xy] + A1[yx]; break;
        case 2: v = A1[xy] - A1[yx]; break;
        default: v = A1[xy]; break;
        }
        vk[e] = sign * v;
}

__global__ void transpose_kernel(const double *__restrict__ D, int nao, double *__restrict__ Dt)
{
        const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (e >= (long long)nao * nao) return;
        const int x = (int)(e / nao), y = (int)(e % nao);
        Dt[e] = D[(size_t)y * nao + x];
}

inline unsigned blocks_for(long long n, int b) { return (unsigned)((n + b - 1) / b); }

int check(const char *what, std::string &err)
{
        const cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) return 0;
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return 1;
}

template <int B, bool S8>
int launch_pass(const IncoreArgs &a, cudaStream_t s, std::string &err)
{
        const size_t smem = sizeof(double) * (4 * (size_t)B * a.nao + B * B);
        cudaError_t e = cudaFuncSetAttribute(incore_pass_kernel<B, S8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        const size_t smem_fast = sizeof(double) * 2 * (size_t)B * a.nao;
        if (e == cudaSuccess)
                e = cudaFuncSetAttribute(incore_fast_kernel<B, S8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_fast);
        if (e != cudaSuccess) {
                err = std::string("in-core kernel configuration: ") + cudaGetErrorString(e);
                return 1;
        }
        const int nfast = a.nf[0] + a.nf[1] + a.nf[2] + a.nf[3];
        if (nfast > 0) {
                incore_fast_kernel<B, S8><<<nfast, NT, smem_fast, s>>>(a);
                if (check("in-core kernel launch", err)) return 1;
        }
        if (a.nitems > 0) {
                incore_pass_kernel<B, S8><<<a.nitems, NT, smem, s>>>(a);
                if (check("in-core kernel launch", err)) return 1;
        }
        return 0;
}

} // namespace

// 8 AO rows per block: a lane keeps 4 x B doubles in registers (the J-row
// image sums, one row of entries and its row-J parts), which B = 8 keeps
// under the 128 registers of two resident blocks; the shared memory of a block is 4 slabs of B x nao
// doubles (+ B^2), so nao up to 880
int incore_block(int nao)
{
        const size_t limit = 227 * 1024;
        if (sizeof(double) * (4 * 8 * (size_t)nao + 64) <= limit) return 8;
        return 0;
}

void incore_items(int nao, int s8, int B, long long window, std::vector<int4> (&fast)[4],
                  std::vector<int4> &general)
{
        for (auto &v : fast) v.clear();
        general.clear();
        const long long npair = (long long)nao * (nao + 1) / 2;
        const int nb = (nao + B - 1) / B;
        auto split = [&](std::vector<int4> &v, int I, int J, long long c0, long long c1) {
                for (long long c = c0; c < c1; c += window)
                        v.push_back(make_int4(I, J, (int)c, (int)std::min(c1, c + window)));
        };
        for (int I = 0; I < nb; I++)
                for (int J = 0; J <= I; J++) {
                        const int imax = std::min(nao, (I + 1) * B) - 1;
                        const int jmax = std::min(std::min(nao, (J + 1) * B) - 1, imax);
                        const long long pmax = (long long)imax * (imax + 1) / 2 + jmax;
                        const long long ncol = s8 ? pmax + 1 : npair;
                        const bool full = (I + 1) * B <= nao;
                        const int diag = I == J ? 2 : 0;
                        if (!full) {
                                split(general, I, J, 0, ncol);
                        } else if (!s8) {
                                split(fast[diag], I, J, 0, ncol);
                        } else {
                                // the block's first row (i0, j0): columns
                                // before it are below the packed diagonal for
                                // every row of the block
                                const long long i0 = (long long)I * B;
                                const long long pmin = i0 * (i0 + 1) / 2 + (long long)J * B;
                                split(fast[diag], I, J, 0, pmin);
                                split(fast[diag + 1], I, J, pmin, ncol);
                        }
                }
}

int launch_incore_pass(const IncoreArgs &a, cudaStream_t s, std::string &err)
{
        const int B = incore_block(a.nao);
        if (B == 8) return a.s8 ? launch_pass<8, true>(a, s, err) : launch_pass<8, false>(a, s, err);
        err = "in-core contraction: nao too large for the shared-memory slabs";
        return 1;
}

int launch_incore_tridm(const double *D, int nao, double *t, cudaStream_t s, std::string &err)
{
        const long long np = (long long)nao * (nao + 1) / 2;
        tridm_kernel<<<blocks_for(np, 256), 256, 0, s>>>(D, nao, t);
        return check("in-core pair density", err);
}

int launch_incore_unpack_j(const double *Jp, int nao, double *vj, cudaStream_t s, std::string &err)
{
        unpack_j_kernel<<<blocks_for((long long)nao * nao, 256), 256, 0, s>>>(Jp, nao, vj);
        return check("in-core J unpack", err);
}

int launch_incore_finish_k(const double *A1, const double *A2, int nao, int mode, int hermi, double *vk,
                           cudaStream_t s, std::string &err)
{
        finish_k_kernel<<<blocks_for((long long)nao * nao, 256), 256, 0, s>>>(A1, A2, nao, mode, hermi, vk);
        return check("in-core K finish", err);
}

int launch_incore_transpose(const double *D, int nao, double *Dt, cudaStream_t s, std::string &err)
{
        transpose_kernel<<<blocks_for((long long)nao * nao, 256), 256, 0, s>>>(D, nao, Dt);
        return check("in-core transpose", err);
}

} // namespace b200jk
