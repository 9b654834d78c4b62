// incore_launch.h — interface between the host ABI (b200jk.cu) and the
// kernels of the in-core J/K contraction (incore.cu).
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <vector>

namespace b200jk {

// One contraction pass over a stored integral tensor for one density D.
struct IncoreArgs {
        const double *eri;      // s8: ij(ij+1)/2 + kl (ij >= kl); s4: ij * npair + kl
        int s8;                 // 1: s8 packed, 0: s4 matrix
        int nao;
        long long npair;        // nao (nao + 1) / 2
        const double *D;        // nao x nao (row-major) density of this pass
        const double *t;        // npair: D_ij + D_ji (i > j), D_ii (i == j)
        double *A;              // nao x nao accumulator of the pair-order K images (zeroed by the caller)
        double *Jp;             // npair accumulator of packed J, or nullptr (zeroed by the caller)
        const int4 *items;      // general items: (I block, J block, first column, end column) per thread block
        int nitems;
        // items of the fast kernel's variants, index EDGE + 2 DIAG: full blocks
        // (I > J, or I == J for DIAG), windows before the block's rows or (s8,
        // EDGE) the ones that reach them
        const int4 *fitems[4];
        int nf[4];
};

// AO rows per block of the contraction for a basis of nao functions (0 when
// the shared-memory slabs would not fit)
int incore_block(int nao);
// the work items of a pass: AO-block pairs I >= J crossed with column windows
// of at most `window` packed columns (s8: only the columns <= the block's
// last row).  fast[v], v = EDGE + 2 DIAG, gets the windows of full blocks
// (DIAG: I == J, else I > J): for s8 the columns before the block's first
// row (EDGE = 0: no entry there needs a validity test) and the rest (EDGE =
// 1: q <= p tested per entry, half weight on q == p); for s4 every window
// (EDGE = 0).  `general` gets the blocks of the partial last block row.
void incore_items(int nao, int s8, int B, long long window, std::vector<int4> (&fast)[4],
                  std::vector<int4> &general);

int launch_incore_pass(const IncoreArgs &a, cudaStream_t s, std::string &err);
// t = packed D + D^T (diagonal once) of a nao x nao density
int launch_incore_tridm(const double *D, int nao, double *t, cudaStream_t s, std::string &err);
// vj (nao x nao) from packed J; nullptr skips
int launch_incore_unpack_j(const double *Jp, int nao, double *vj, cudaStream_t s, std::string &err);
// vk from the accumulators: mode 0  K = A1 + A2^T,  1  K = A1 + A1^T,
// 2  K = A1 - A1^T,  3  K = A1; then the reference's hermi_triu for
// hermi != 0 (upper triangle from the lower, negated for hermi = 2)
int launch_incore_finish_k(const double *A1, const double *A2, int nao, int mode, int hermi, double *vk,
                           cudaStream_t s, std::string &err);
// Dt = D^T
int launch_incore_transpose(const double *D, int nao, double *Dt, cudaStream_t s, std::string &err);

} // namespace b200jk
