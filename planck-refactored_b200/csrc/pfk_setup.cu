// pfk_setup.cu -- per-geometry setup kernels (Schwarz table, screened quartet
// lists, quartet census) and the per-build finishing kernels.
#include <cub/device/device_scan.cuh>

#include "pfk_internal.h"
#include "pfk_kernels.cuh"
#include "pfk_setup.h"

namespace pfk {

// ---------------------------------------------------------------------------
// Schwarz table
// ---------------------------------------------------------------------------
template <int PC>
static void launch_schwarz_pc(const int *ids, int n, const PairInfo *pairs, const PrimPair *prims, double *Q, int nb,
                              cudaStream_t st)
{
    if (n <= 0) return;
    schwarz_kernel<pc_la(PC), pc_lb(PC)><<<(n + 63) / 64, 64, 0, st>>>(ids, n, pairs, prims, Q, nb);
}

template <int PC>
static void launch_prim_bounds_pc(const int *ids, int n, const PairInfo *pairs, PrimPair *prims, cudaStream_t st)
{
    if (n <= 0) return;
    prim_bound_kernel<pc_la(PC), pc_lb(PC)><<<(n + 63) / 64, 64, 0, st>>>(ids, n, pairs, prims);
}

void launch_prim_bounds(int pc, const int *ids, int n, const PairInfo *pairs, PrimPair *prims, cudaStream_t st)
{
    switch (pc) {
    case 0: launch_prim_bounds_pc<0>(ids, n, pairs, prims, st); break;
    case 1: launch_prim_bounds_pc<1>(ids, n, pairs, prims, st); break;
    case 2: launch_prim_bounds_pc<2>(ids, n, pairs, prims, st); break;
    case 3: launch_prim_bounds_pc<3>(ids, n, pairs, prims, st); break;
    case 4: launch_prim_bounds_pc<4>(ids, n, pairs, prims, st); break;
    case 5: launch_prim_bounds_pc<5>(ids, n, pairs, prims, st); break;
    case 6: launch_prim_bounds_pc<6>(ids, n, pairs, prims, st); break;
    case 7: launch_prim_bounds_pc<7>(ids, n, pairs, prims, st); break;
    case 8: launch_prim_bounds_pc<8>(ids, n, pairs, prims, st); break;
    case 9: launch_prim_bounds_pc<9>(ids, n, pairs, prims, st); break;
    default: break;
    }
}

void launch_schwarz(int pc, const int *ids, int n, const PairInfo *pairs, const PrimPair *prims, double *Q, int nb,
                    cudaStream_t st)
{
    switch (pc) {
    case 0: launch_schwarz_pc<0>(ids, n, pairs, prims, Q, nb, st); break;
    case 1: launch_schwarz_pc<1>(ids, n, pairs, prims, Q, nb, st); break;
    case 2: launch_schwarz_pc<2>(ids, n, pairs, prims, Q, nb, st); break;
    case 3: launch_schwarz_pc<3>(ids, n, pairs, prims, Q, nb, st); break;
    case 4: launch_schwarz_pc<4>(ids, n, pairs, prims, Q, nb, st); break;
    case 5: launch_schwarz_pc<5>(ids, n, pairs, prims, Q, nb, st); break;
    case 6: launch_schwarz_pc<6>(ids, n, pairs, prims, Q, nb, st); break;
    case 7: launch_schwarz_pc<7>(ids, n, pairs, prims, Q, nb, st); break;
    case 8: launch_schwarz_pc<8>(ids, n, pairs, prims, Q, nb, st); break;
    case 9: launch_schwarz_pc<9>(ids, n, pairs, prims, Q, nb, st); break;
    default: break;
    }
}

// ---------------------------------------------------------------------------
// Screened shell-quartet lists.  Bra pairs of class X and ket pairs of class Y
// are each sorted by qmax (descending), so the kets a bra keeps are a prefix:
// the ket b survives when qX[a] * qY[b] >= tol.  For X == Y only b >= a is
// kept (each unordered pair of shell pairs once).  A second threshold splits
// each bra's run at the FP32 bound: kets [a0, c_hi) are FP64, [c_hi, c) FP32.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int count_prefix(const double *__restrict__ qY, int nY, double qa, double thr)
{
    // largest c with qa * qY[c-1] >= thr (qY descending)
    int lo = 0, hi = nY;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (qa * qY[mid] >= thr) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__global__ void quartet_count_kernel(const double *__restrict__ qX, int nX, const double *__restrict__ qY, int nY,
                                     int diag, double tol, double bound, long long *cnt_hi, long long *cnt_lo)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nX) return;
    const double qa = qX[a];
    const int start = diag ? a : 0;
    int c = count_prefix(qY, nY, qa, tol);
    int ch = bound > tol ? count_prefix(qY, nY, qa, bound) : c;
    if (ch > c) ch = c;
    c = c > start ? c - start : 0;
    ch = ch > start ? ch - start : 0;
    cnt_hi[a] = ch;
    cnt_lo[a] = c - ch;
}

// One warp per bra: writes its FP64 run into out_hi and its FP32 run into out_lo.
__global__ void quartet_fill_kernel(const int *__restrict__ idX, int nX, const int *__restrict__ idY, int diag,
                                    const long long *__restrict__ off_hi, const long long *__restrict__ cnt_hi,
                                    const long long *__restrict__ off_lo, const long long *__restrict__ cnt_lo,
                                    uint2 *out_hi, uint2 *out_lo)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nX) return;
    const int a = warp;
    const unsigned bra = idX[a];
    const int start = diag ? a : 0;
    const long long nh = cnt_hi[a], nl = cnt_lo[a];
    const long long oh = off_hi[a], ol = off_lo[a];
    for (long long b = lane; b < nh; b += 32) out_hi[oh + b] = make_uint2(bra, (unsigned)idY[start + b]);
    for (long long b = lane; b < nl; b += 32) out_lo[ol + b] = make_uint2(bra, (unsigned)idY[start + nh + b]);
}

cudaError_t count_quartets(const double *qX, int nX, const double *qY, int nY, int diag, double tol, double bound,
                           long long *cnt_hi, long long *cnt_lo, cudaStream_t st)
{
    if (nX > 0) quartet_count_kernel<<<(nX + 127) / 128, 128, 0, st>>>(qX, nX, qY, nY, diag, tol, bound, cnt_hi, cnt_lo);
    return cudaGetLastError();
}

cudaError_t exclusive_scan(const long long *in, long long *out, int n, void *tmp, size_t &tmp_bytes, cudaStream_t st)
{
    return cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, in, out, n, st);
}

cudaError_t fill_quartets(const int *idX, int nX, const int *idY, int diag, const long long *off_hi,
                          const long long *cnt_hi, const long long *off_lo, const long long *cnt_lo, uint2 *out_hi,
                          uint2 *out_lo, cudaStream_t st)
{
    if (nX > 0)
        quartet_fill_kernel<<<(nX * 32 + 127) / 128, 128, 0, st>>>(idX, nX, idY, diag, off_hi, cnt_hi, off_lo, cnt_lo,
                                                                   out_hi, out_lo);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Census of the canonical AO quartets the lists stand for (the reference's
// screened set, os.cpp:1458-1476): same duplicate rules and AO-level mask as
// the integral kernels.  Counts, sums mix64 of the canonical code, and
// optionally writes the quartets.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long mix64(unsigned long long x)
{
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebULL;
    x ^= x >> 31;
    return x;
}

__global__ void census_kernel(const uint2 *__restrict__ quartets, long long nq, const PairInfo *__restrict__ pairs,
                              const int *__restrict__ pair_la, const int *__restrict__ pair_lb,
                              const double *__restrict__ Qao, int nb, double tol, unsigned long long *counters,
                              int *out, long long cap)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long cnt = 0, dig = 0;
    if (t < nq) {
        const uint2 qd = quartets[t];
        const PairInfo pb = pairs[qd.x], pk = pairs[qd.y];
        const int NA = ncart(pair_la[qd.x]), NB = ncart(pair_lb[qd.x]);
        const int NC = ncart(pair_la[qd.y]), ND = ncart(pair_lb[qd.y]);
        const bool same_ab = pb.bf_a == pb.bf_b, same_cd = pk.bf_a == pk.bf_b, same_bk = qd.x == qd.y;
        for (int ia = 0; ia < NA; ++ia)
            for (int ib = 0; ib < NB; ++ib)
                for (int ic = 0; ic < NC; ++ic)
                    for (int id = 0; id < ND; ++id) {
                        int i = pb.bf_a + ia, j = pb.bf_b + ib, k = pk.bf_a + ic, l = pk.bf_b + id;
                        if (quartet_weight(same_ab, same_cd, same_bk, ia, ib, ic, id, NB, ND, true, Qao, nb, i, j, k,
                                           l, tol) == 0.0)
                            continue;
                        if (i > j) { const int x = i; i = j; j = x; }
                        if (k > l) { const int x = k; k = l; l = x; }
                        if (i > k || (i == k && j > l)) {
                            int x = i; i = k; k = x;
                            x = j; j = l; l = x;
                        }
                        ++cnt;
                        dig += mix64(((unsigned long long)i << 48) | ((unsigned long long)j << 32) |
                                     ((unsigned long long)k << 16) | (unsigned long long)l);
                        if (out) {
                            const unsigned long long pos = atomicAdd(counters + 2, 1ULL);
                            if ((long long)pos < cap) {
                                out[4 * pos] = i;
                                out[4 * pos + 1] = j;
                                out[4 * pos + 2] = k;
                                out[4 * pos + 3] = l;
                            }
                        }
                    }
    }
    // warp reduction, then one atomic per warp
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
        dig += __shfl_down_sync(0xffffffffu, dig, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(counters, cnt);
        atomicAdd(counters + 1, dig);
    }
}

cudaError_t census(const uint2 *q, long long nq, const PairInfo *pairs, const int *pair_la, const int *pair_lb,
                   const double *Qao, int nb, double tol, unsigned long long *counters, int *out, long long cap,
                   cudaStream_t st)
{
    if (nq > 0)
        census_kernel<<<(unsigned)((nq + 255) / 256), 256, 0, st>>>(q, nq, pairs, pair_la, pair_lb, Qao, nb, tol,
                                                                    counters, out, cap);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Finishing kernels (O(nb^2))
// ---------------------------------------------------------------------------
// A + A^T of a fixed-point accumulator (fx_add) at (i, j), summed as
// integers (exact) before the one conversion to double.
__device__ __forceinline__ double fx_sym(const FxWord *__restrict__ A, size_t ij, size_t ji)
{
    const long long hi = (long long)(A[2 * ij] + A[2 * ji]);
    const long long lo = (long long)(A[2 * ij + 1] + A[2 * ji + 1]);
    return fx_value(hi, lo);
}

// out = cj * 2 (J + J^T) + ck * (K + K^T)   (either accumulator may be null)
__global__ void combine_kernel(const FxWord *__restrict__ J, const FxWord *__restrict__ K, double cj, double ck,
                               double *out, int nb)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nb * nb) return;
    const int i = (int)(t / nb), j = (int)(t % nb);
    const size_t ij = (size_t)i * nb + j, ji = (size_t)j * nb + i;
    double v = 0.0;
    if (J) v += cj * 2.0 * fx_sym(J, ij, ji);
    if (K) v += ck * fx_sym(K, ij, ji);
    out[ij] = v;
}

__global__ void add_kernel(const double *__restrict__ a, const double *__restrict__ b, double *out, long long n)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = a[t] + b[t];
}

cudaError_t combine(const FxWord *J, const FxWord *K, double cj, double ck, double *out, int nb, cudaStream_t st)
{
    const long long n = (long long)nb * nb;
    combine_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(J, K, cj, ck, out, nb);
    return cudaGetLastError();
}

cudaError_t add(const double *a, const double *b, double *out, long long n, cudaStream_t st)
{
    add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, b, out, n);
    return cudaGetLastError();
}

}  // namespace pfk

namespace pfk {

// Primitive-quartet work of each bra's FP64 and FP32 ket runs:
// K_bra * (sum of K_ket over the run) with all primitives counted (the
// algorithmic yardstick), from the ket class's nprim_full prefix.
__global__ void bra_work_kernel(const int *__restrict__ idX, int nX, int diag, const long long *__restrict__ cnt_hi,
                                const long long *__restrict__ cnt_lo, const long long *__restrict__ kprefY,
                                const PairInfo *__restrict__ pairs, long long *work_hi, long long *work_lo)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nX) return;
    const long long kb = pairs[idX[a]].nprim_full;
    const long long s = diag ? a : 0, nh = cnt_hi[a], nl = cnt_lo[a];
    work_hi[a] = kb * (kprefY[s + nh] - kprefY[s]);
    work_lo[a] = kb * (kprefY[s + nh + nl] - kprefY[s + nh]);
}

cudaError_t bra_work(const int *idX, int nX, int diag, const long long *cnt_hi, const long long *cnt_lo,
                     const long long *kprefY, const PairInfo *pairs, long long *work_hi, long long *work_lo,
                     cudaStream_t st)
{
    if (nX > 0)
        bra_work_kernel<<<(nX + 127) / 128, 128, 0, st>>>(idX, nX, diag, cnt_hi, cnt_lo, kprefY, pairs, work_hi,
                                                          work_lo);
    return cudaGetLastError();
}

// FMA throughput probe: eight independent dependency chains per thread,
// all in registers.
template <typename T>
__global__ void __launch_bounds__(256) fma_chain_kernel(T *out, int iters, T a, T b)
{
    T x0 = T(threadIdx.x) * T(1e-3), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
    T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

__global__ void shell_block_max_kernel(int nshell, const int *__restrict__ bf_off, const int *__restrict__ nbf,
                                       const double *__restrict__ P0, const double *__restrict__ P1,
                                       const double *__restrict__ P2, int nb, float *__restrict__ D)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nshell * nshell) return;
    const int s1 = (int)(t / nshell), s2 = (int)(t % nshell);
    const int i0 = bf_off[s1], j0 = bf_off[s2], ni = nbf[s1], nj = nbf[s2];
    double m = 0.0;
    for (int i = 0; i < ni; ++i)
        for (int j = 0; j < nj; ++j) {
            const size_t k = (size_t)(i0 + i) * nb + j0 + j;
            m = fmax(m, fabs(P0[k]));
            if (P1) m = fmax(m, fabs(P1[k]));
            if (P2) m = fmax(m, fabs(P2[k]));
        }
    D[(size_t)i0 * nb + j0] = __double2float_ru(m);
}

cudaError_t shell_block_max(int nshell, const int *bf_off, const int *nbf, const double *P0, const double *P1,
                            const double *P2, int nb, float *D, cudaStream_t st)
{
    const long long n = (long long)nshell * nshell;
    shell_block_max_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(nshell, bf_off, nbf, P0, P1, P2, nb, D);
    return cudaGetLastError();
}

template <typename T>
static cudaError_t time_fma(int device, double *tflops)
{
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return e;
    const int blocks = prop.multiProcessorCount * 8, threads = 256, iters = 4096;
    T *out = nullptr;
    e = cudaMalloc(&out, sizeof(T) * blocks * threads);
    if (e != cudaSuccess) return e;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    fma_chain_kernel<T><<<blocks, threads>>>(out, iters / 8, T(0.9999999), T(1e-7));   // warm-up
    cudaEventRecord(a);
    fma_chain_kernel<T><<<blocks, threads>>>(out, iters, T(0.9999999), T(1e-7));
    cudaEventRecord(b);
    e = cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    if (e != cudaSuccess) return e;
    const double flops = 2.0 * 64.0 * (double)iters * blocks * threads;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return cudaGetLastError();
}

cudaError_t measure_fma_peak(int device, double *fp64, double *fp32)
{
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess && fp64) e = time_fma<double>(device, fp64);
    if (e == cudaSuccess && fp32) e = time_fma<float>(device, fp32);
    return e;
}

}  // namespace pfk

#include <cub/device/device_radix_sort.cuh>

namespace pfk {

// Sort key of a shell quartet: (evaluated bra primitives, evaluated ket
// primitives), so that a warp's lanes run the same primitive loop lengths.
__global__ void quartet_key_kernel(const uint2 *__restrict__ q, long long n, const PairInfo *__restrict__ pairs,
                                   unsigned *keys)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint2 v = q[t];
    keys[t] = (unsigned)pairs[v.x].nprim * 4096u + (unsigned)pairs[v.y].nprim;
}

// Stable sort of one list segment by its key; tmp buffers sized by the caller
// (keys_a/keys_b: n unsigned, vals_b: n uint2, temp: temp_bytes).
cudaError_t sort_quartets(uint2 *q, long long n, const PairInfo *pairs, unsigned *keys_a, unsigned *keys_b,
                          uint2 *vals_b, void *temp, size_t &temp_bytes, cudaStream_t st)
{
    if (!temp) {
        return cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys_a, keys_b,
                                               reinterpret_cast<unsigned long long *>(q),
                                               reinterpret_cast<unsigned long long *>(vals_b), n, 0, 24, st);
    }
    if (n <= 1) return cudaSuccess;
    quartet_key_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(q, n, pairs, keys_a);
    cudaError_t e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_a, keys_b,
                                                    reinterpret_cast<unsigned long long *>(q),
                                                    reinterpret_cast<unsigned long long *>(vals_b), n, 0, 24, st);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(q, vals_b, sizeof(uint2) * n, cudaMemcpyDeviceToDevice, st);
}

}  // namespace pfk
