// pfk_internal.h -- shared host-side declarations of the Fock engine.
#pragma once
#include <string>

#include <cuda_runtime.h>

#include "pfk_device.cuh"
#include "planck_fock.h"

namespace pfk {

// Ten shell-pair classes (LA >= LB) in order ss, ps, pp, ds, dp, dd, fs, fp, fd, ff.
constexpr int kPairClasses = 10;
constexpr int kQuartetClasses = 55;
__host__ __device__ constexpr int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }
__host__ __device__ constexpr int pc_la(int pc) { return pc >= 6 ? 3 : pc >= 3 ? 2 : pc >= 1 ? 1 : 0; }
__host__ __device__ constexpr int pc_lb(int pc) { return pc - pc_la(pc) * (pc_la(pc) + 1) / 2; }
__host__ __device__ constexpr int quartet_class(int bra_pc, int ket_pc) { return bra_pc * (bra_pc + 1) / 2 + ket_pc; }
// Total angular momentum LA+LB+LC+LD of quartet class c.
__host__ __device__ constexpr int quartet_class_L(int c)
{
    int x = 0;
    while ((x + 1) * (x + 2) / 2 <= c) ++x;
    const int y = c - x * (x + 1) / 2;
    return pc_la(x) + pc_lb(x) + pc_la(y) + pc_lb(y);
}

// Launch flags.  kLaunchFP32 asks for the FP32-arithmetic variant (every
// kernel family has one for nk == 1; builds with two exchange densities run
// FP64).  kLaunchOS asks for the Obara-Saika kernel, which exists
// for classes with LA+LB+LC+LD <= kOSMaxL; the other classes run Rys.
// kLaunchDense picks the Obara-Saika kernel compiled for 4 blocks of 128
// per SM (single exchange density only).
constexpr int kLaunchFP32 = 1, kLaunchOS = 2, kLaunchDense = 4;
constexpr int kOSMaxL = 4;

// One launcher per quartet class.  nk = number of exchange densities (1 or 2).
using ClassLauncher = void (*)(const uint2 *quartets, long long n, const JKArgs &args, int nk, int flags,
                               cudaStream_t st);

// Launchers of the 55 classes, filled at library load by the pfk_classes.cu
// units (each compiled for a range of classes).  A launcher called with
// n < 0 only configures the current device for its kernels.
extern ClassLauncher g_class_launchers[kQuartetClasses];

// Context internals for the other units: its CUDA device, and recording a
// failure message (returns s).
int ctx_device(const pfk_ctx *ctx);
pfk_status ctx_fail(pfk_ctx *ctx, pfk_status s, const std::string &msg);

// One-electron integrals S, T, V of a validated basis on `device` (pfk_onee.cu);
// on failure `what` names the step.
cudaError_t one_electron_run(const pfk_basis_desc *basis, int natom, const double *nuclei, double *S, double *T,
                             double *V, int device, std::string &what);

}  // namespace pfk
