// jk_classes.cu — the kernel of one quartet class (la lb | lc ld), compiled
// once per class with -DB2_BRA_LA -DB2_BRA_LB -DB2_KET_LC -DB2_KET_LD so the
// 55 classes of l <= 3 build in parallel.
#include <mutex>
#include "jk_launch.h"

#ifndef B2_KET_LD
#error "compile with -DB2_BRA_LA -DB2_BRA_LB -DB2_KET_LC -DB2_KET_LD"
#endif

namespace b200jk {

namespace {

struct LaunchCfg {
        int grid = 0, block = 128;
        size_t smem = 0;
        bool ready = false;
        cudaError_t status = cudaSuccess;
};

// R is the evaluation type: double for the FP64 pass, float for the FP32 pass
// of mixed precision (accumulation stays in float64 either way).  MULTI: one
// launch over a batch of molecules (margs, mchunk, nmol on the device).
template <int LA, int LB, int LC, int LD, typename R, bool MULTI, int KR, int GSV = 0>
int launch_one(const JKArgs &a, const JKArgs *margs, const long long *mchunk, int nmol, cudaStream_t s, int nsm,
               std::string &err)
{
        // GSV > 0: lanes per quartet of the shared-memory family (a variant)
        constexpr int GSX = GSV > 0 ? GSV : group_size<LA, LB, LC, LD>();
        using K = Class4<LA, LB, LC, LD>;
        constexpr int NP = thread_parts<LA, LB, LC, LD>();
        constexpr bool thread = NP > 0;
        static LaunchCfg cfg;
        static std::mutex mu;
        {
                std::lock_guard<std::mutex> lk(mu);
                if (!cfg.ready) {
                        int nb = 0;
                        if constexpr (thread) {
                                cfg.block = 128;
                                cfg.smem = stage_table<R>(K::NR) ? sizeof(R) * rys_slice_elems<R>(K::NR) : 0;
                                cfg.status = cudaFuncSetAttribute(jk_thread_kernel<LA, LB, LC, LD, (NP > 0 ? NP : 1), R, MULTI, KR>,
                                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem);
                                if (cfg.status == cudaSuccess)
                                        cfg.status = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                                &nb, jk_thread_kernel<LA, LB, LC, LD, (NP > 0 ? NP : 1), R, MULTI, KR>, 128, cfg.smem);
                        } else {
                                const size_t per_warp = sizeof(double) * WarpSmem<LA, LB, LC, LD, R>::SIZE *
                                                        (32 / GSX);
                                const int wpb = (int)std::min<size_t>(4, std::max<size_t>(1, (200 * 1024) / per_warp));
                                cfg.block = 32 * wpb;
                                cfg.smem = per_warp * wpb;
                                cfg.status = cudaFuncSetAttribute(jk_warp_kernel<LA, LB, LC, LD, R, MULTI, GSX>,
                                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem);
                                if (cfg.status == cudaSuccess)
                                        cfg.status = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, jk_warp_kernel<LA, LB, LC, LD, R, MULTI, GSX>,
                                                                                                   cfg.block, cfg.smem);
                        }
                        cfg.grid = (nb > 0 ? nb : 1) * nsm;
                        cfg.ready = true;
                }
        }
        if (cfg.status != cudaSuccess) {
                err = std::string("kernel configuration: ") + cudaGetErrorString(cfg.status);
                return 1;
        }
        if constexpr (thread) {
                jk_thread_kernel<LA, LB, LC, LD, NP, R, MULTI, KR><<<cfg.grid, cfg.block, cfg.smem, s>>>(a, margs, mchunk, nmol);
        } else {
                jk_warp_kernel<LA, LB, LC, LD, R, MULTI, GSX><<<cfg.grid, cfg.block, cfg.smem, s>>>(
                        a, 8 * (32 / GSX), margs, mchunk, nmol);
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
                err = std::string("kernel launch: ") + cudaGetErrorString(e);
                return 1;
        }
        return 0;
}

// variant 2 of the register family: bra runs of BR pairs (float64 pass,
// tiled chunk order, one symmetric density; the host checks these)
template <int LA, int LB, int LC, int LD, int BR>
int launch_run(const JKArgs &a, cudaStream_t s, int nsm, std::string &err)
{
        using K = Class4<LA, LB, LC, LD>;
        static LaunchCfg cfg;
        static std::mutex mu;
        {
                std::lock_guard<std::mutex> lk(mu);
                if (!cfg.ready) {
                        int nb = 0;
                        cfg.block = 128;
                        cfg.smem = stage_table<double>(K::NR) ? sizeof(double) * rys_slice_elems<double>(K::NR) : 0;
                        cfg.status = cudaFuncSetAttribute(jk_thread_run_kernel<LA, LB, LC, LD, BR>,
                                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem);
                        if (cfg.status == cudaSuccess)
                                cfg.status = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                        &nb, jk_thread_run_kernel<LA, LB, LC, LD, BR>, 128, cfg.smem);
                        cfg.grid = (nb > 0 ? nb : 1) * nsm;
                        cfg.ready = true;
                }
        }
        if (cfg.status != cudaSuccess) {
                err = std::string("kernel configuration: ") + cudaGetErrorString(cfg.status);
                return 1;
        }
        jk_thread_run_kernel<LA, LB, LC, LD, BR><<<cfg.grid, cfg.block, cfg.smem, s>>>(a);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
                err = std::string("kernel launch: ") + cudaGetErrorString(e);
                return 1;
        }
        return 0;
}

} // namespace

// B2_FN_NAME is launch_jk_<la><lb><lc><ld>, declared in jk_launch.h
int B2_FN_NAME(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant, const JKArgs *margs,
               const long long *mchunk, int nmol, std::string &err)
{
        constexpr int NP = thread_parts<B2_BRA_LA, B2_BRA_LB, B2_KET_LC, B2_KET_LD>();
        constexpr int KRUN = NP > 0 ? ket_run<B2_BRA_LA, B2_BRA_LB, B2_KET_LC, B2_KET_LD, NP>() : 1;
        // the shared-memory family's variant 1: half as many lanes per quartet
        // (only where one warp's groups still fit the 200 KB a block may use here)
        constexpr int GSH0 = NP > 0 ? 0 : group_size<B2_BRA_LA, B2_BRA_LB, B2_KET_LC, B2_KET_LD>() / 2;
        constexpr int GSH = (GSH0 >= 8 && sizeof(double) * WarpSmem<B2_BRA_LA, B2_BRA_LB, B2_KET_LC, B2_KET_LD>::SIZE *
                                                  (32 / (GSH0 > 0 ? GSH0 : 1)) <= 200 * 1024) ? GSH0 : 0;
        constexpr int BRUN = NP > 0 ? bra_run<B2_BRA_LA, B2_BRA_LB, B2_KET_LC, B2_KET_LD, NP>() : 1;
        if constexpr (BRUN > 1) {
                if (variant == 2) {
                        if (nmol > 0 || fp32 || !a.tiled || a.n_dm != 1 || a.nk != 1) {
                                err = "launch variant 2 (bra runs) needs the tiled float64 pass of one symmetric density";
                                return 1;
                        }
                        return launch_run<B2_BRA_LA, B2_BRA_LB, B2_KET_LC, B2_KET_LD, BRUN>(a, s, nsm, err);
                }
        }
#define B2_L(R, M, KR) launch_one<B2_BRA_LA, B2_BRA_LB, B2_KET_LC, B2_KET_LD, R, M, KR>(a, margs, mchunk, nmol, s, nsm, err)
#define B2_LG(R, M) launch_one<B2_BRA_LA, B2_BRA_LB, B2_KET_LC, B2_KET_LD, R, M, 1, GSH>(a, margs, mchunk, nmol, s, nsm, err)
        if constexpr (GSH >= 8) {
                if (variant == 1) {
                        if (nmol > 0) return fp32 ? B2_LG(float, true) : B2_LG(double, true);
                        return fp32 ? B2_LG(float, false) : B2_LG(double, false);
                }
        }
#undef B2_LG
        if constexpr (KRUN > 1) {
                if (variant == 1) {
                        if (nmol > 0) return fp32 ? B2_L(float, true, KRUN) : B2_L(double, true, KRUN);
                        return fp32 ? B2_L(float, false, KRUN) : B2_L(double, false, KRUN);
                }
        }
        if (nmol > 0) return fp32 ? B2_L(float, true, 1) : B2_L(double, true, 1);
        return fp32 ? B2_L(float, false, 1) : B2_L(double, false, 1);
#undef B2_L
}

// B2_NP_NAME is launch_jk_<la><lb><lc><ld>_np: the parts of the register
// family this unit's class was built with (0: shared-memory family), which
// the host planner reads instead of recomputing the budget
int B2_NP_NAME() { return thread_parts<B2_BRA_LA, B2_BRA_LB, B2_KET_LC, B2_KET_LD>(); }

} // namespace b200jk
