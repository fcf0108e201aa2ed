// pfk_setup.h -- host wrappers of the setup and finishing kernels (pfk_setup.cu).
#pragma once
#include <cuda_runtime.h>

#include "pfk_device.cuh"

namespace pfk {

void launch_schwarz(int pc, const int *ids, int n, const PairInfo *pairs, const PrimPair *prims, double *Q, int nb,
                    cudaStream_t st);
void launch_prim_bounds(int pc, const int *ids, int n, const PairInfo *pairs, PrimPair *prims, cudaStream_t st);
cudaError_t count_quartets(const double *qX, int nX, const double *qY, int nY, int diag, double tol, double bound,
                           long long *cnt_hi, long long *cnt_lo, cudaStream_t st);
cudaError_t exclusive_scan(const long long *in, long long *out, int n, void *tmp, size_t &tmp_bytes, cudaStream_t st);
cudaError_t fill_quartets(const int *idX, int nX, const int *idY, int diag, const long long *off_hi,
                          const long long *cnt_hi, const long long *off_lo, const long long *cnt_lo, uint2 *out_hi,
                          uint2 *out_lo, cudaStream_t st);
cudaError_t census(const uint2 *q, long long nq, const PairInfo *pairs, const int *pair_la, const int *pair_lb,
                   const double *Qao, int nb, double tol, unsigned long long *counters, int *out, long long cap,
                   cudaStream_t st);
// out = cj * 2 (J + J^T) + ck * (K + K^T) from fixed-point accumulators
// (2 nb^2 words each; either may be null).
cudaError_t combine(const FxWord *J, const FxWord *K, double cj, double ck, double *out, int nb, cudaStream_t st);
cudaError_t add(const double *a, const double *b, double *out, long long n, cudaStream_t st);
cudaError_t bra_work(const int *idX, int nX, int diag, const long long *cnt_hi, const long long *cnt_lo,
                     const long long *kprefY, const PairInfo *pairs, long long *work_hi, long long *work_lo,
                     cudaStream_t st);
cudaError_t measure_fma_peak(int device, double *fp64, double *fp32);
// D[first bf(s1) * nb + first bf(s2)] = max |P| over the (s1, s2) block of
// every non-null density P0..P2 (rounded up to FP32), for density screening.
cudaError_t shell_block_max(int nshell, const int *bf_off, const int *nbf, const double *P0, const double *P1,
                            const double *P2, int nb, float *D, cudaStream_t st);
cudaError_t sort_quartets(uint2 *q, long long n, const PairInfo *pairs, unsigned *keys_a, unsigned *keys_b,
                          uint2 *vals_b, void *temp, size_t &temp_bytes, cudaStream_t st);

}  // namespace pfk
