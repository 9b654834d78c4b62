// grad_classes.cu — gradient kernels of one bra class (la lb | * *), compiled
// once per bra class with -DB2_BRA_LA -DB2_BRA_LB, so the ten translation
// units build in parallel.
#include <algorithm>
#include <mutex>
#include "grad_launch.h"

#ifndef B2_BRA_LB
#error "compile with -DB2_BRA_LA -DB2_BRA_LB"
#endif

#define B2_CAT2(a, b, c) a##b##c
#define B2_CAT(a, b, c) B2_CAT2(a, b, c)

namespace b200jk {

namespace {

struct GradCfg {
        int grid = 0, block = 32;
        size_t smem = 0;
        bool ready = false;
        cudaError_t status = cudaSuccess;
};

// largest dynamic shared memory a block may request on sm_100
constexpr size_t SMEM_MAX = 227 * 1024;

template <int LA, int LB, int LC, int LD, bool FUSED>
int launch_grad_impl(const GradArgs &a, cudaStream_t s, int nsm, std::string &err)
{
        using S = GradSmem<LA, LB, LC, LD, 0, FUSED>;
        constexpr int GS = grad_group_size<LA, LB, LC, LD>();
        static GradCfg cfg;
        static std::mutex mu;
        if constexpr (FUSED && grad_force_regs<LA, LB, LC, LD>()) {
                // the fused contraction's register family (one ket per lane)
                {
                        std::lock_guard<std::mutex> lk(mu);
                        if (!cfg.ready) {
                                int nb = 0;
                                cfg.block = 128;
                                cfg.status = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                        &nb, grad_force_kernel<LA, LB, LC, LD>, 128, 0);
                                cfg.grid = (nb > 0 ? nb : 1) * nsm;
                                cfg.ready = true;
                        }
                }
                if (cfg.status != cudaSuccess) {
                        err = std::string("gradient kernel configuration: ") + cudaGetErrorString(cfg.status);
                        return 1;
                }
                grad_force_kernel<LA, LB, LC, LD><<<cfg.grid, cfg.block, 0, s>>>(a);
                cudaError_t e = cudaGetLastError();
                if (e != cudaSuccess) {
                        err = std::string("gradient kernel launch: ") + cudaGetErrorString(e);
                        return 1;
                }
                return 0;
        } else if constexpr (grad_thread_family<LA, LB, LC, LD>()) {
                {
                        std::lock_guard<std::mutex> lk(mu);
                        if (!cfg.ready) {
                                int nb = 0;
                                cfg.block = 128;
                                cfg.status = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                        &nb, grad_thread_kernel<LA, LB, LC, LD, FUSED>, 128, 0);
                                cfg.grid = (nb > 0 ? nb : 1) * nsm;
                                cfg.ready = true;
                        }
                }
                if (cfg.status != cudaSuccess) {
                        err = std::string("gradient kernel configuration: ") + cudaGetErrorString(cfg.status);
                        return 1;
                }
                grad_thread_kernel<LA, LB, LC, LD, FUSED><<<cfg.grid, cfg.block, 0, s>>>(a);
                cudaError_t e = cudaGetLastError();
                if (e != cudaSuccess) {
                        err = std::string("gradient kernel launch: ") + cudaGetErrorString(e);
                        return 1;
                }
                return 0;
        }
        {
                std::lock_guard<std::mutex> lk(mu);
                if (!cfg.ready) {
                        const size_t per_warp = sizeof(double) * S::SIZE * (32 / GS);
                        if (per_warp > SMEM_MAX) {
                                cfg.status = cudaErrorInvalidConfiguration;
                        } else {
                                const int wpb = (int)std::min<size_t>(4, std::max<size_t>(1, (200 * 1024) / per_warp));
                                cfg.block = 32 * wpb;
                                cfg.smem = per_warp * wpb;
                                cfg.status = cudaFuncSetAttribute(grad_jk_kernel<LA, LB, LC, LD, FUSED>,
                                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem);
                                int nb = 0;
                                if (cfg.status == cudaSuccess)
                                        cfg.status = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                                &nb, grad_jk_kernel<LA, LB, LC, LD, FUSED>, cfg.block, cfg.smem);
                                cfg.grid = (nb > 0 ? nb : 1) * nsm;
                        }
                        cfg.ready = true;
                }
        }
        if (cfg.status != cudaSuccess) {
                err = std::string("gradient kernel configuration: ") + cudaGetErrorString(cfg.status);
                return 1;
        }
        grad_jk_kernel<LA, LB, LC, LD, FUSED><<<cfg.grid, cfg.block, cfg.smem, s>>>(a, 8 * (32 / GS));
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
                err = std::string("gradient kernel launch: ") + cudaGetErrorString(e);
                return 1;
        }
        return 0;
}

// the vj/vk build, or the fused force contraction when a.de is set
template <int LA, int LB, int LC, int LD>
int launch_grad_one(const GradArgs &a, cudaStream_t s, int nsm, std::string &err)
{
        if (a.de) return launch_grad_impl<LA, LB, LC, LD, true>(a, s, nsm, err);
        return launch_grad_impl<LA, LB, LC, LD, false>(a, s, nsm, err);
}

template <int LA, int LB>
int launch_gq0_one(const GradQArgs &q, cudaStream_t s, std::string &err)
{
        using S = GradSmem<LA, LB, LA, LB, 1>;
        static GradCfg cfg;
        static std::mutex mu;
        {
                std::lock_guard<std::mutex> lk(mu);
                if (!cfg.ready) {
                        cfg.smem = sizeof(double) * S::SIZE;
                        cfg.status = cfg.smem > SMEM_MAX ? cudaErrorInvalidConfiguration
                                                         : cudaFuncSetAttribute(grad_q0_kernel<LA, LB>,
                                                                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                                                (int)cfg.smem);
                        cfg.ready = true;
                }
        }
        if (cfg.status != cudaSuccess) {
                err = std::string("gradient q_cond configuration: ") + cudaGetErrorString(cfg.status);
                return 1;
        }
        if (q.pairs.n == 0) return 0;
        grad_q0_kernel<LA, LB><<<q.pairs.n, 32, cfg.smem, s>>>(q);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
                err = std::string("gradient q_cond launch: ") + cudaGetErrorString(e);
                return 1;
        }
        return 0;
}

} // namespace

int B2_CAT(launch_grad_, B2_BRA_LA, B2_BRA_LB)(int lc, int ld, const GradArgs &a, cudaStream_t s, int nsm,
                                               std::string &err)
{
        constexpr int LA = B2_BRA_LA, LB = B2_BRA_LB;
        switch (lc * 4 + ld) {
        case 0: return launch_grad_one<LA, LB, 0, 0>(a, s, nsm, err);
        case 4: return launch_grad_one<LA, LB, 1, 0>(a, s, nsm, err);
        case 5: return launch_grad_one<LA, LB, 1, 1>(a, s, nsm, err);
        case 8: return launch_grad_one<LA, LB, 2, 0>(a, s, nsm, err);
        case 9: return launch_grad_one<LA, LB, 2, 1>(a, s, nsm, err);
        case 10: return launch_grad_one<LA, LB, 2, 2>(a, s, nsm, err);
        case 12: return launch_grad_one<LA, LB, 3, 0>(a, s, nsm, err);
        case 13: return launch_grad_one<LA, LB, 3, 1>(a, s, nsm, err);
        case 14: return launch_grad_one<LA, LB, 3, 2>(a, s, nsm, err);
        case 15: return launch_grad_one<LA, LB, 3, 3>(a, s, nsm, err);
        default: err = "ket class out of range"; return 1;
        }
}

int B2_CAT(launch_gq0_, B2_BRA_LA, B2_BRA_LB)(const GradQArgs &q, cudaStream_t s, std::string &err)
{
        return launch_gq0_one<B2_BRA_LA, B2_BRA_LB>(q, s, err);
}

} // namespace b200jk
