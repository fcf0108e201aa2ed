// pfk_classes.cu -- launchers of the quartet-class kernels whose bra pair
// class is PFK_BRA_CLASS (compiled once per bra class, 0..9, so the 55
// class instantiations build in parallel).
#include "pfk_internal.h"
#include "pfk_kernels.cuh"

#ifndef PFK_BRA_CLASS
#error "PFK_BRA_CLASS must be defined (0..9)"
#endif

namespace pfk {
namespace {

constexpr int kRegMaxComponents = 81;   // register path up to (pp|pp)-sized blocks

template <int LA, int LB, int LC, int LD>
void launch_class(const uint2 *q, long long n, const JKArgs &a, int nk, cudaStream_t st)
{
    using S = ClassShape<LA, LB, LC, LD>;
    using SS = SplitShape<LA, LB, LC, LD>;
    using TS = TeamShape<LA, LB, LC, LD>;
    if constexpr (S::N <= kRegMaxComponents) {
        if (n <= 0) return;
        const long long grid = (n + 127) / 128;
        if (nk == 2) eri_reg_kernel<LA, LB, LC, LD, 2><<<(unsigned)grid, 128, 0, st>>>(q, n, a);
        else eri_reg_kernel<LA, LB, LC, LD, 1><<<(unsigned)grid, 128, 0, st>>>(q, n, a);
    } else if constexpr (SS::OK) {
        if (n < 0) {  // configure the current device (shared-memory opt-in)
            cudaFuncSetAttribute(eri_split_kernel<LA, LB, LC, LD, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SS::SMEM);
            cudaFuncSetAttribute(eri_split_kernel<LA, LB, LC, LD, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SS::SMEM);
            return;
        }
        if (n == 0) return;
        const long long grid = (n + SS::TEAMS - 1) / SS::TEAMS;
        if (nk == 2) eri_split_kernel<LA, LB, LC, LD, 2><<<(unsigned)grid, 128, SS::SMEM, st>>>(q, n, a);
        else eri_split_kernel<LA, LB, LC, LD, 1><<<(unsigned)grid, 128, SS::SMEM, st>>>(q, n, a);
    } else {
        if (n < 0) {
            cudaFuncSetAttribute(eri_team_kernel<LA, LB, LC, LD, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS::SMEM);
            cudaFuncSetAttribute(eri_team_kernel<LA, LB, LC, LD, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS::SMEM);
            return;
        }
        if (n == 0) return;
        const long long grid = (n + TS::TEAMS - 1) / TS::TEAMS;
        if (nk == 2) eri_team_kernel<LA, LB, LC, LD, 2><<<(unsigned)grid, 128, TS::SMEM, st>>>(q, n, a);
        else eri_team_kernel<LA, LB, LC, LD, 1><<<(unsigned)grid, 128, TS::SMEM, st>>>(q, n, a);
    }
}

template <int X, int Y>
void reg_one(ClassLauncher *table)
{
    table[quartet_class(X, Y)] = &launch_class<pc_la(X), pc_lb(X), pc_la(Y), pc_lb(Y)>;
    if constexpr (Y > 0) reg_one<X, Y - 1>(table);
}

}  // namespace

}  // namespace pfk

#define PFK_CAT2(a, b) a##b
#define PFK_CAT(a, b) PFK_CAT2(a, b)

namespace pfk {
void PFK_CAT(register_bra_class_, PFK_BRA_CLASS)(ClassLauncher *table)
{
    reg_one<PFK_BRA_CLASS, PFK_BRA_CLASS>(table);
}
}  // namespace pfk
