// fill_launch.h — interface between the host planner (b200jk.cu) and the
// translation units of the s8 integral fill (fill_classes.cu, compiled once
// per bra angular class).
#pragma once
#include <cuda_runtime.h>
#include <string>
#include "fill_kernels.cuh"

namespace b200jk {

// quartets per chunk of a warp for class (la lb | lc ld): 8 per group of the
// shared-memory family's size
inline int fill_chunk(int la, int lb, int lc, int ld)
{
        const int ng = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
        const int gs = ng <= 100 ? 8 : (ng <= 400 ? 16 : 32);
        return 8 * (32 / gs);
}

// one launcher per bra class (la, lb), la >= lb; the ket class (lc, ld),
// lc >= ld and not after (la, lb) in pair-class order, is a run-time argument
#define B2_FILL_DECL(LA, LB) \
        int launch_fill_##LA##LB(int lc, int ld, const FillArgs &f, cudaStream_t s, int nsm, std::string &err);
B2_FILL_DECL(0, 0)
B2_FILL_DECL(1, 0)
B2_FILL_DECL(1, 1)
B2_FILL_DECL(2, 0)
B2_FILL_DECL(2, 1)
B2_FILL_DECL(2, 2)
B2_FILL_DECL(3, 0)
B2_FILL_DECL(3, 1)
B2_FILL_DECL(3, 2)
B2_FILL_DECL(3, 3)
#undef B2_FILL_DECL

} // namespace b200jk
