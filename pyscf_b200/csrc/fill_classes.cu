// fill_classes.cu — s8 integral fill kernels of one bra class (la lb | * *),
// compiled once per bra class with -DB2_BRA_LA -DB2_BRA_LB.
#include <algorithm>
#include <mutex>
#include "fill_launch.h"

#ifndef B2_BRA_LB
#error "compile with -DB2_BRA_LA -DB2_BRA_LB"
#endif

#define B2_CAT2(a, b, c) a##b##c
#define B2_CAT(a, b, c) B2_CAT2(a, b, c)

namespace b200jk {

namespace {

struct FillCfg {
        int grid = 0, block = 32;
        size_t smem = 0;
        bool ready = false;
        cudaError_t status = cudaSuccess;
};

constexpr size_t SMEM_MAX = 227 * 1024;

template <int LA, int LB, int LC, int LD>
int launch_fill_one(const FillArgs &f, cudaStream_t s, int nsm, std::string &err)
{
        constexpr int GS = group_size<LA, LB, LC, LD>();
        static FillCfg cfg;
        static std::mutex mu;
        {
                std::lock_guard<std::mutex> lk(mu);
                if (!cfg.ready) {
                        const size_t per_warp = sizeof(double) * FillSmem<LA, LB, LC, LD>::SIZE * (32 / GS);
                        if (per_warp > SMEM_MAX) {
                                cfg.status = cudaErrorInvalidConfiguration;
                        } else {
                                const int wpb = (int)std::min<size_t>(4, std::max<size_t>(1, (200 * 1024) / per_warp));
                                cfg.block = 32 * wpb;
                                cfg.smem = per_warp * wpb;
                                cfg.status = cudaFuncSetAttribute(fill_kernel<LA, LB, LC, LD>,
                                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem);
                                int nb = 0;
                                if (cfg.status == cudaSuccess)
                                        cfg.status = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                                &nb, fill_kernel<LA, LB, LC, LD>, cfg.block, cfg.smem);
                                cfg.grid = (nb > 0 ? nb : 1) * nsm;
                        }
                        cfg.ready = true;
                }
        }
        if (cfg.status != cudaSuccess) {
                err = std::string("integral fill kernel configuration: ") + cudaGetErrorString(cfg.status);
                return 1;
        }
        fill_kernel<LA, LB, LC, LD><<<cfg.grid, cfg.block, cfg.smem, s>>>(f, 8 * (32 / GS));
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
                err = std::string("integral fill kernel launch: ") + cudaGetErrorString(e);
                return 1;
        }
        return 0;
}

constexpr int pair_index(int la, int lb) { return la * (la + 1) / 2 + lb; }

template <int LA, int LB, int LC, int LD>
int launch_if_ordered(const FillArgs &f, cudaStream_t s, int nsm, std::string &err)
{
        if constexpr (pair_index(LC, LD) <= pair_index(LA, LB)) {
                return launch_fill_one<LA, LB, LC, LD>(f, s, nsm, err);
        } else {
                err = "integral fill: ket class after the bra class";
                return 1;
        }
}

} // namespace

int B2_CAT(launch_fill_, B2_BRA_LA, B2_BRA_LB)(int lc, int ld, const FillArgs &f, cudaStream_t s, int nsm,
                                               std::string &err)
{
        constexpr int LA = B2_BRA_LA, LB = B2_BRA_LB;
        switch (lc * 4 + ld) {
        case 0: return launch_if_ordered<LA, LB, 0, 0>(f, s, nsm, err);
        case 4: return launch_if_ordered<LA, LB, 1, 0>(f, s, nsm, err);
        case 5: return launch_if_ordered<LA, LB, 1, 1>(f, s, nsm, err);
        case 8: return launch_if_ordered<LA, LB, 2, 0>(f, s, nsm, err);
        case 9: return launch_if_ordered<LA, LB, 2, 1>(f, s, nsm, err);
        case 10: return launch_if_ordered<LA, LB, 2, 2>(f, s, nsm, err);
        case 12: return launch_if_ordered<LA, LB, 3, 0>(f, s, nsm, err);
        case 13: return launch_if_ordered<LA, LB, 3, 1>(f, s, nsm, err);
        case 14: return launch_if_ordered<LA, LB, 3, 2>(f, s, nsm, err);
        case 15: return launch_if_ordered<LA, LB, 3, 3>(f, s, nsm, err);
        default: err = "integral fill: bad ket class"; return 1;
        }
}

} // namespace b200jk
