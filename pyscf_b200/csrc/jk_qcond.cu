// jk_qcond.cu — Schwarz-conditioner kernels, one per pair class.
#include "jk_launch.h"

namespace b200jk {

template <int LA, int LB>
static int launch_q(const QArgs &q, cudaStream_t s, std::string &err)
{
        const size_t smem = sizeof(double) * WarpSmem<LA, LB, LA, LB>::SIZE;
        cudaError_t e = cudaFuncSetAttribute(qcond_kernel<LA, LB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess && q.pairs.n > 0) {
                qcond_kernel<LA, LB><<<q.pairs.n, 32, smem, s>>>(q);
                e = cudaGetLastError();
        }
        if (e != cudaSuccess) {
                err = std::string("q_cond kernel: ") + cudaGetErrorString(e);
                return 1;
        }
        return 0;
}

int launch_qcond(int la, int lb, const QArgs &q, cudaStream_t s, std::string &err)
{
#define B2_QQ(LA, LB) if (la == LA && lb == LB) return launch_q<LA, LB>(q, s, err);
        B2_QQ(0, 0) B2_QQ(1, 0) B2_QQ(1, 1) B2_QQ(2, 0) B2_QQ(2, 1) B2_QQ(2, 2)
        B2_QQ(3, 0) B2_QQ(3, 1) B2_QQ(3, 2) B2_QQ(3, 3)
#undef B2_QQ
        err = "pair class outside l <= 3";
        return 1;
}

} // namespace b200jk
