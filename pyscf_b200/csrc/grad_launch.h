// grad_launch.h — interface between the host planner (b200jk.cu) and the
// translation units of the gradient kernels (grad_classes.cu, compiled once
// per bra angular class).
#pragma once
#include <cuda_runtime.h>
#include <string>
#include "grad_kernels.cuh"

namespace b200jk {

// whether class (la lb | lc ld) runs in a register family (one ket per lane):
// host twin of grad_thread_family and, for the fused force contraction, of
// grad_force_regs
inline bool grad_register_family(int la, int lb, int lc, int ld, bool fused = false)
{
        const int ng = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
        const int se = (la + 2) * (lb + 2) * (lc + 1) * (ld + 1);
        return 6 * ng + 3 * se <= 104 || (fused && ng + 3 * se <= 102);
}

// quartets per chunk of a warp for class (la lb | lc ld): one per lane in a
// register family, 8 per group otherwise
inline int grad_chunk(int la, int lb, int lc, int ld, bool fused = false)
{
        if (grad_register_family(la, lb, lc, ld, fused)) return 32;
        const int ng = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
        const int gs = ng <= 100 ? 8 : (ng <= 400 ? 16 : 32);
        return 8 * (32 / gs);
}

// one launcher per bra class (la, lb), la >= lb; the ket class (lc, ld),
// lc >= ld, is a run-time argument
#define B2_GRAD_DECL(LA, LB)                                                                              \
        int launch_grad_##LA##LB(int lc, int ld, const GradArgs &a, cudaStream_t s, int nsm, std::string &err); \
        int launch_gq0_##LA##LB(const GradQArgs &q, cudaStream_t s, std::string &err);
B2_GRAD_DECL(0, 0)
B2_GRAD_DECL(1, 0)
B2_GRAD_DECL(1, 1)
B2_GRAD_DECL(2, 0)
B2_GRAD_DECL(2, 1)
B2_GRAD_DECL(2, 2)
B2_GRAD_DECL(3, 0)
B2_GRAD_DECL(3, 1)
B2_GRAD_DECL(3, 2)
B2_GRAD_DECL(3, 3)
#undef B2_GRAD_DECL

} // namespace b200jk
