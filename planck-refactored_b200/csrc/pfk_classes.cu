// pfk_classes.cu -- launchers of quartet classes PFK_CLASS_BEGIN ..
// PFK_CLASS_END - 1 (the build compiles this file once per class range so the
// 55 class instantiations build in parallel).
#include "pfk_internal.h"
#include "pfk_kernels.cuh"
#include "pfk_os.cuh"

#if !defined(PFK_CLASS_BEGIN) || !defined(PFK_CLASS_END)
#error "PFK_CLASS_BEGIN and PFK_CLASS_END must be defined (0 <= begin < end <= 55)"
#endif

namespace pfk {
namespace {

constexpr int kRegMaxComponents = 81;   // register path up to (pp|pp)-sized blocks

template <int LA, int LB, int LC, int LD>
void launch_class(const uint2 *q, long long n, const JKArgs &a, int nk, int flags, cudaStream_t st)
{
    using S = ClassShape<LA, LB, LC, LD>;
    using SS = SplitShape<LA, LB, LC, LD>;
    using TS = TeamShape<LA, LB, LC, LD>;
    const int fp32 = flags & kLaunchFP32;
    if constexpr (LA + LB + LC + LD <= kOSMaxL) {
        if (flags & kLaunchOS) {
            if (n <= 0) return;
            const long long grid = (n + 127) / 128;
            const bool dense = flags & kLaunchDense;
            // the denser build: blocks per SM its register cap must allow.  Up
            // to L = 2 the kernels need at most 104 registers, so 4 blocks would
            // change nothing; there 8 (L <= 1: 64 registers) and 6 (L = 2: 80)
            // trade a few spilled values for occupancy.  The autotuner keeps
            // whichever build is faster on the molecule's lists.
            constexpr int L = LA + LB + LC + LD;
            constexpr int MB = L <= 1 ? 8 : L == 2 ? 6 : 4;
            if (nk == 2) eri_os_kernel<LA, LB, LC, LD, 2><<<(unsigned)grid, 128, 0, st>>>(q, n, a);
            else if (fp32 && dense) eri_os_kernel<LA, LB, LC, LD, 1, float, MB><<<(unsigned)grid, 128, 0, st>>>(q, n, a);
            else if (fp32) eri_os_kernel<LA, LB, LC, LD, 1, float><<<(unsigned)grid, 128, 0, st>>>(q, n, a);
            else if (dense) eri_os_kernel<LA, LB, LC, LD, 1, double, MB><<<(unsigned)grid, 128, 0, st>>>(q, n, a);
            else eri_os_kernel<LA, LB, LC, LD, 1><<<(unsigned)grid, 128, 0, st>>>(q, n, a);
            return;
        }
    }
    if constexpr (S::N <= kRegMaxComponents) {
        if (n <= 0) return;
        const long long grid = (n + 127) / 128;
        if (nk == 2) eri_reg_kernel<LA, LB, LC, LD, 2><<<(unsigned)grid, 128, 0, st>>>(q, n, a);
        else if (fp32) eri_reg_kernel<LA, LB, LC, LD, 1, float><<<(unsigned)grid, 128, 0, st>>>(q, n, a);
        else eri_reg_kernel<LA, LB, LC, LD, 1><<<(unsigned)grid, 128, 0, st>>>(q, n, a);
    } else if constexpr (SS::OK) {
        using SF = SplitShape<LA, LB, LC, LD, float>;
        if (n < 0) {  // configure the current device (shared-memory opt-in)
            cudaFuncSetAttribute(eri_split_kernel<LA, LB, LC, LD, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SS::SMEM);
            cudaFuncSetAttribute(eri_split_kernel<LA, LB, LC, LD, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SS::SMEM);
            cudaFuncSetAttribute(eri_split_kernel<LA, LB, LC, LD, 1, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SF::SMEM);
            return;
        }
        if (n == 0) return;
        const long long grid = (n + SS::TEAMS - 1) / SS::TEAMS;
        if (nk == 2) eri_split_kernel<LA, LB, LC, LD, 2><<<(unsigned)grid, 128, SS::SMEM, st>>>(q, n, a);
        else if (fp32) eri_split_kernel<LA, LB, LC, LD, 1, float><<<(unsigned)grid, 128, SF::SMEM, st>>>(q, n, a);
        else eri_split_kernel<LA, LB, LC, LD, 1><<<(unsigned)grid, 128, SS::SMEM, st>>>(q, n, a);
    } else {
        using TF = TeamShape<LA, LB, LC, LD, float>;
        if (n < 0) {
            cudaFuncSetAttribute(eri_team_kernel<LA, LB, LC, LD, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS::SMEM);
            cudaFuncSetAttribute(eri_team_kernel<LA, LB, LC, LD, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS::SMEM);
            cudaFuncSetAttribute(eri_team_kernel<LA, LB, LC, LD, 1, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)TF::SMEM);
            return;
        }
        if (n == 0) return;
        const long long grid = (n + TS::TEAMS - 1) / TS::TEAMS;
        if (nk == 2) eri_team_kernel<LA, LB, LC, LD, 2><<<(unsigned)grid, TS::BLOCK, TS::SMEM, st>>>(q, n, a);
        else if (fp32) eri_team_kernel<LA, LB, LC, LD, 1, float><<<(unsigned)grid, TF::BLOCK, TF::SMEM, st>>>(q, n, a);
        else eri_team_kernel<LA, LB, LC, LD, 1><<<(unsigned)grid, TS::BLOCK, TS::SMEM, st>>>(q, n, a);
    }
}

// class index -> (bra pair class, ket pair class)
constexpr int cls_bra(int c)
{
    int x = 0;
    while ((x + 1) * (x + 2) / 2 <= c) ++x;
    return x;
}
constexpr int cls_ket(int c) { return c - cls_bra(c) * (cls_bra(c) + 1) / 2; }

template <int C>
void reg_range(ClassLauncher *table)
{
    constexpr int X = cls_bra(C), Y = cls_ket(C);
    table[C] = &launch_class<pc_la(X), pc_lb(X), pc_la(Y), pc_lb(Y)>;
    if constexpr (C + 1 < PFK_CLASS_END) reg_range<C + 1>(table);
}

// Runs at library load: puts this unit's launchers into the shared table.
struct Registrar {
    Registrar() { reg_range<PFK_CLASS_BEGIN>(g_class_launchers); }
};
const Registrar registrar;

}  // namespace
}  // namespace pfk
