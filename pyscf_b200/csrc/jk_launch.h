// jk_launch.h — interface between the host planner (b200jk.cu) and the
// translation units that hold the per-class kernels (jk_classes.cu, compiled
// once per bra angular class, and jk_qcond.cu).
#pragma once
#include <cuda_runtime.h>
#include <string>
#include "jk_kernels.cuh"

namespace b200jk {

// parts of the register family of class (la lb | lc ld) as its translation
// unit was built (thread_parts<> in jk_kernels.cuh with the build's
// per-class choice), 0 for the shared-memory family; defined in b200jk.cu
// from the units' launch_jk_*_np
int family_thread_parts(int la, int lb, int lc, int ld);
inline int family_is_thread(int la, int lb, int lc, int ld) { return family_thread_parts(la, lb, lc, ld) > 0; }
// lanes per quartet of the shared-memory family (group_size<> in jk_kernels.cuh)
inline int family_group(int la, int lb, int lc, int ld)
{
        const int ng = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
        return ng <= 100 ? 8 : (ng <= 400 ? 16 : 32);
}
// kets per lane of variant 1 of the register family (host twin of ket_run<>);
// 1 where the class has no such variant
inline int family_ket_run(int la, int lb, int lc, int ld)
{
        const int np = family_thread_parts(la, lb, lc, ld);
        const int na = ncart(la), nb = ncart(lb), nc = ncart(lc);
        return (np == 1 && na * nc + nb * nc <= 24) ? 4 : 1;
}
// whether a class has a launch variant 1 for the autotuner to try: more kets
// per lane (register family) or half as many lanes per quartet (shared-memory
// family with groups of 16 or 32 lanes)
// doubles of one group's shared memory (host twin of WarpSmem<..., double>::SIZE)
inline int family_group_smem(int la, int lb, int lc, int ld)
{
        const int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
        const int ng = na * nb * nc * nd, sa = (la + 1) * (lb + 1) * (lc + 1) * (ld + 1);
        const int nr = (la + lb + lc + ld) / 2 + 1;
        const int x = ng + 3 * nr * sa + na * nb + nc * nd + nb * nc + nb * nd + na * nc + na * nd;
        return (x + 3) & ~3;
}
// half-width groups (variant 1 of the shared-memory family: 32 -> 16 or
// 16 -> 8 lanes) where one warp's groups fit the 200 KB a block may use
inline bool family_half_groups(int la, int lb, int lc, int ld)
{
        const int gs = family_group(la, lb, lc, ld);
        return gs >= 16 && 8.0 * family_group_smem(la, lb, lc, ld) * (32 / (gs / 2)) <= 200 * 1024;
}
inline bool family_has_variant(int la, int lb, int lc, int ld)
{
        if (family_thread_parts(la, lb, lc, ld) > 0) return family_ket_run(la, lb, lc, ld) > 1;
        return family_half_groups(la, lb, lc, ld);
}
// bra pairs per run of the register family's variant 2 (host twin of
// bra_run<>); 1 where the class has no such variant
inline int family_bra_run(int la, int lb, int lc, int ld)
{
        const int np = family_thread_parts(la, lb, lc, ld);
        const int na = ncart(la), nc = ncart(lc), nd = ncart(ld);
        return (np == 1 && na * (nc + nd) + nc * nd <= 32) ? 4 : 1;
}
// launch variants of a class: 0 always, 1 (more kets per lane or half-width
// groups) and 2 (bra runs) where the class has them
inline bool family_has_variant_n(int la, int lb, int lc, int ld, int v)
{
        if (v == 0) return true;
        if (v == 1) return family_has_variant(la, lb, lc, ld);
        if (v == 2) return family_bra_run(la, lb, lc, ld) > 1;
        return false;
}
// quartets per chunk: 32 x kets per lane in the register family (variant 0:
// one ket per lane, 1: family_ket_run), 8 per group of the warp otherwise
inline int family_chunk(int la, int lb, int lc, int ld, int variant = 0)
{
        if (family_thread_parts(la, lb, lc, ld) > 0)
                return 32 * (variant == 1 ? family_ket_run(la, lb, lc, ld) : 1);   // bra runs: 32 kets too
        const int gs = family_group(la, lb, lc, ld);
        return 8 * (32 / (variant == 1 && family_half_groups(la, lb, lc, ld) ? gs / 2 : gs));   // 8 quartets per group
}

// one launcher per quartet class (la lb | lc ld), (lc, ld) <= (la, lb)
int launch_jk_0000(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_1000(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_1010(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_1100(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_1110(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_1111(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2000(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2010(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2011(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2020(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2100(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2110(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2111(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2120(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2121(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2200(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2210(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2211(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2220(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2221(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_2222(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3000(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3010(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3011(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3020(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3021(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3022(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3030(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3100(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3110(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3111(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3120(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3121(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3122(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3130(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3131(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3200(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3210(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3211(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3220(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3221(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3222(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3230(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3231(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3232(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3300(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3310(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3311(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3320(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3321(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3322(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3330(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3331(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3332(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
int launch_jk_3333(const JKArgs &a, cudaStream_t s, int nsm, int fp32, int variant,
                   const JKArgs *margs, const long long *mchunk, int nmol, std::string &err);
// the parts each class unit was built with (see family_thread_parts)
int launch_jk_0000_np();
int launch_jk_1000_np();
int launch_jk_1010_np();
int launch_jk_1100_np();
int launch_jk_1110_np();
int launch_jk_1111_np();
int launch_jk_2000_np();
int launch_jk_2010_np();
int launch_jk_2011_np();
int launch_jk_2020_np();
int launch_jk_2100_np();
int launch_jk_2110_np();
int launch_jk_2111_np();
int launch_jk_2120_np();
int launch_jk_2121_np();
int launch_jk_2200_np();
int launch_jk_2210_np();
int launch_jk_2211_np();
int launch_jk_2220_np();
int launch_jk_2221_np();
int launch_jk_2222_np();
int launch_jk_3000_np();
int launch_jk_3010_np();
int launch_jk_3011_np();
int launch_jk_3020_np();
int launch_jk_3021_np();
int launch_jk_3022_np();
int launch_jk_3030_np();
int launch_jk_3100_np();
int launch_jk_3110_np();
int launch_jk_3111_np();
int launch_jk_3120_np();
int launch_jk_3121_np();
int launch_jk_3122_np();
int launch_jk_3130_np();
int launch_jk_3131_np();
int launch_jk_3200_np();
int launch_jk_3210_np();
int launch_jk_3211_np();
int launch_jk_3220_np();
int launch_jk_3221_np();
int launch_jk_3222_np();
int launch_jk_3230_np();
int launch_jk_3231_np();
int launch_jk_3232_np();
int launch_jk_3300_np();
int launch_jk_3310_np();
int launch_jk_3311_np();
int launch_jk_3320_np();
int launch_jk_3321_np();
int launch_jk_3322_np();
int launch_jk_3330_np();
int launch_jk_3331_np();
int launch_jk_3332_np();
int launch_jk_3333_np();

int launch_qcond(int la, int lb, const QArgs &q, cudaStream_t s, std::string &err);

} // namespace b200jk
