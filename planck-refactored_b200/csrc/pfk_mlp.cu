// pfk_mlp.cu -- the learned-guess network: a small multilayer perceptron
// trained and evaluated by this file's kernels on the GPU.
//
//   H_0 = bf16(X);  Z_l = H_{l-1} W_l + b_l;  H_l = bf16(SiLU(Z_l)) (l < L);
//   Y = Z_L (FP32).
//
// Every matrix product runs on the fifth-generation tensor cores as BF16 x
// BF16 with FP32 accumulation in tensor memory (tcgen05.mma, M 128, N 64,
// K 16); weights are kept in FP32 (Adam's master copy) and rounded to BF16
// for the products.  Training minimises the mean
// squared error against targets T with Adam.  The backward pass:
//   dZ_L = 2 (Y - T) / (n d_L);  dW_l = H_{l-1}^T bf16(dZ_l);
//   db_l = column sums of dZ_l;  dH_{l-1} = bf16(dZ_l) W_l^T;
//   dZ_{l-1} = dH_{l-1} * SiLU'(Z_{l-1}).
// The reference has no counterpart: it is the learned part of the guess
// hook (scf.cpp:206-240 selects the guess; a learned density enters the SCF
// as a ReadDensity guess does, scf.cpp:213-216).
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "planck_fock.h"

namespace {

thread_local std::string g_mlp_error;

// ---------------------------------------------------------------------------
// GEMM on the fifth-generation tensor cores: C[m][n] = sum_k A(m, k) B(k, n),
// A(m,k) = A[m*lda + k] (or A[k*lda + m] when TA), B(k,n) = B[k*ldb + n] (or
// B[n*ldb + k] when TB); BF16 operands, FP32 accumulation in tensor memory;
// the epilogue adds bias[n] and writes C (FP32) and/or H = bf16(SiLU(C)).
//
// One CTA of 128 threads per 128 x 64 tile of C.  Per round of 64 in K the
// threads stage the A tile (128 x 64) and the B tile (64 x 64, as N rows of
// K) in shared memory, K-major in the no-swizzle core-matrix layout (8 rows x
// 16 bytes per 128-byte core matrix), zero-filled outside the matrices; one
// thread issues four tcgen05.mma (M 128, N 64, K 16) into the tile's
// accumulator in tensor memory and commits them to an mbarrier that every
// thread waits on before the tiles are overwritten.  The epilogue reads the
// accumulator back with tcgen05.ld, warp w taking rows 32w .. 32w+31 (the
// tensor-memory lanes a warp may access).  Waits are bounded (2 s of
// %globaltimer); a wait that runs out sets *err, the CTA stops issuing,
// waits (bounded again) for the round in flight and frees its columns.
// ---------------------------------------------------------------------------
constexpr int TC_M = 128, TC_N = 64, TC_K = 64;
constexpr int TC_A_BYTES = TC_M * TC_K * 2, TC_B_BYTES = TC_N * TC_K * 2;
// 24 KB of tiles, requested as 28 KB so that at most 8 CTAs share an SM and
// their 8 x 64 accumulator columns fit the SM's 512 tensor-memory columns
constexpr int TC_SMEM = 28 * 1024;
static_assert(TC_A_BYTES + TC_B_BYTES <= TC_SMEM, "staged tiles exceed the shared-memory request");
constexpr uint32_t TC_TMEM_COLS = 64;
constexpr unsigned long long TC_WAIT_NS = 2000000000ull;
// instruction descriptor (kind::f16): D F32 (bits 4-5 = 1), A and B BF16
// (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bits
// 17-22, M >> 4 at bits 24-28
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of the 16-byte segment (row, K chunk kc of 8 elements) in a
// staged tile: K chunks of a row group are adjacent core matrices (128 B
// apart), row groups of 8 are TC_K / 8 core matrices apart.
__device__ __forceinline__ uint32_t tc_off(int row, int kc)
{
    return (uint32_t)(((row >> 3) * (TC_K / 8) + kc) * 128 + (row & 7) * 16);
}

// Shared-memory matrix descriptor of a K-major, no-swizzle operand whose
// first core matrix is at saddr: leading byte offset 128 (the next K chunk),
// stride byte offset TC_K / 8 * 128 (the next group of 8 rows), descriptor
// version 1 (bit 46), base offset 0, layout type 0 (no swizzle).
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
           ((uint64_t)((TC_K / 8 * 128u) >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits until phase `parity` of the mbarrier at bar completes; false after
// TC_WAIT_NS without completion.
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity)
{
    const unsigned long long t0 = global_ns();
    while (true) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(bar), "r"(parity)
                     : "memory");
        if (done) return true;
        if (global_ns() - t0 > TC_WAIT_NS) return false;
    }
}

__device__ __forceinline__ unsigned pack2(__nv_bfloat16 lo, __nv_bfloat16 hi)
{
    return (unsigned)__bfloat16_as_ushort(lo) | ((unsigned)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z)
{
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// Stages rows row0 .. row0 + ROWS - 1 of a K-major operand tile: element
// (r, k) = get(row0 + r, k0 + k), zero outside rows < nrows and k < K.  T:
// the source is stored with the row index contiguous (then consecutive
// threads take consecutive rows, else consecutive K chunks of a row).
template <int ROWS, bool T>
__device__ __forceinline__ void tc_stage(uint32_t sbase, const __nv_bfloat16 *__restrict__ src, int ld, int row0,
                                         int nrows, int k0, int K)
{
    constexpr int CH = TC_K / 8;
    for (int c = threadIdx.x; c < ROWS * CH; c += 128) {
        const int r = T ? c % ROWS : c / CH, kc = T ? c / ROWS : c % CH;
        const int gr = row0 + r;
        unsigned w[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int ka = k0 + kc * 8 + 2 * e, kb = ka + 1;
            __nv_bfloat16 lo = __float2bfloat16(0.0f), hi = lo;
            if (gr < nrows) {
                if (ka < K) lo = T ? src[(size_t)ka * ld + gr] : src[(size_t)gr * ld + ka];
                if (kb < K) hi = T ? src[(size_t)kb * ld + gr] : src[(size_t)gr * ld + kb];
            }
            w[e] = pack2(lo, hi);
        }
        asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sbase + tc_off(r, kc)), "r"(w[0]), "r"(w[1]),
                     "r"(w[2]), "r"(w[3])
                     : "memory");
    }
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(128) gemm_tc_kernel(int M, int N, int K, const __nv_bfloat16 *__restrict__ A,
                                                      int lda, const __nv_bfloat16 *__restrict__ B, int ldb,
                                                      const float *__restrict__ bias, float *C, __nv_bfloat16 *H,
                                                      int ldc, int *err)
{
    extern __shared__ __align__(128) unsigned char tc_tiles[];
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TC_M, n0 = blockIdx.x * TC_N;
    const uint32_t sA = smem_u32(tc_tiles), sB = sA + TC_A_BYTES, sbar = smem_u32(&mbar);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    const int nk = (K + TC_K - 1) / TC_K;
    uint32_t parity = 0;
    bool failed = false;
    for (int kt = 0; kt < nk; ++kt) {
        const int k0 = kt * TC_K;
        tc_stage<TC_M, TA>(sA, A, lda, m0, M, k0, K);
        tc_stage<TC_N, !TB>(sB, B, ldb, n0, N, k0, K);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // staged tiles visible to the tensor cores
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int s = 0; s < TC_K / 16; ++s) {
                const uint64_t da = tc_desc(sA + s * 256), db = tc_desc(sB + s * 256);
                const uint32_t accumulate = (kt > 0 || s > 0) ? 1u : 0u;
                asm volatile("{\n\t.reg .pred p;\n\t"
                             "setp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                             "l"(da), "l"(db), "r"(TC_IDESC), "r"(accumulate)
                             : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(sbar)
                         : "memory");
        }
        const bool ok = tc_wait(sbar, parity);
        parity ^= 1u;
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (failed) {
        if (tid == 0) atomicExch(err, 1);
        // the round whose wait ran out may still complete: wait for it once
        // more (bounded) before its accumulator columns are released below
        tc_wait(sbar, parity ^ 1u);
    } else {
        const int m = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c = 0; c < TC_N; c += 8) {
            uint32_t v[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
            if (nk > 0) {
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                             : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                               "=r"(v[7])
                             : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            }
            if (m < M) {
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const int n = n0 + c + e;
                    if (n >= N) continue;
                    float x = __uint_as_float(v[e]);
                    if (bias) x += bias[n];
                    if (C) C[(size_t)m * ldc + n] = x;
                    if (H) H[(size_t)m * ldc + n] = __float2bfloat16(silu(x));
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS) : "memory");
}

__global__ void to_bf16_kernel(const float *__restrict__ x, __nv_bfloat16 *__restrict__ y, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16(x[i]);
}

// dZ = 2 (Y - T) / (n d) (FP32 and BF16), loss += sum (Y - T)^2 / (n d)
__global__ void mse_grad_kernel(const float *__restrict__ Y, const float *__restrict__ T, long long n, float scale,
                                float *__restrict__ dZ, __nv_bfloat16 *__restrict__ G, double *loss)
{
    double part = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float r = Y[i] - T[i];
        const float d = 2.0f * r * scale;
        dZ[i] = d;
        G[i] = __float2bfloat16(d);
        part += (double)r * r * scale;
    }
    for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, part);
}

// dZ = dH * SiLU'(Z) (FP32 and BF16)
__global__ void silu_back_kernel(const float *__restrict__ dH, const float *__restrict__ Z, long long n,
                                 float *__restrict__ dZ, __nv_bfloat16 *__restrict__ G)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float d = dH[i] * silu_grad(Z[i]);
        dZ[i] = d;
        G[i] = __float2bfloat16(d);
    }
}

// db[c] = sum_r dZ[r][c]
__global__ void colsum_kernel(const float *__restrict__ dZ, int rows, int cols, float *__restrict__ db)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.0f;
    for (int r = 0; r < rows; ++r) s += dZ[(size_t)r * cols + c];
    db[c] = s;
}

// Adam (bias-corrected) on the FP32 master parameters (the next forward pass
// rounds the weights to BF16 again).
__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ grad, float *__restrict__ m,
                            float *__restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                            float c2)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float g = grad[i];
        const float mi = b1 * m[i] + (1.0f - b1) * g, vi = b2 * v[i] + (1.0f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

unsigned blocks_for(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 148 * 16); }

}  // namespace

struct pfk_mlp {
    int device = 0, nl = 0, max_batch = 0;
    std::vector<int> dims;
    std::vector<long long> w_off, b_off;      // offsets in the parameter vector
    long long nparam = 0;
    float *p = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;   // FP32 params, grads, Adam moments
    __nv_bfloat16 *wb = nullptr;              // BF16 copy of the parameter vector (weights used)
    std::vector<float *> Z;                   // pre-activations per layer [max_batch x d_l]
    std::vector<__nv_bfloat16 *> Hb;          // BF16 activations per layer (H_0 = input)
    float *dA = nullptr, *dB = nullptr;       // FP32 scratch for dZ / dH
    __nv_bfloat16 *G = nullptr;               // BF16 dZ
    double *loss = nullptr;
    int *tc_err = nullptr;                    // set by a tensor-core wait that ran out
    long long step = 0;
    std::string err;
};

namespace {

pfk_status mlp_fail(pfk_mlp *m, const std::string &msg, pfk_status s)
{
    if (m) m->err = msg;
    g_mlp_error = msg;
    return s;
}

#define MLP_CK(call)                                                                            \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) return mlp_fail(m, std::string(#call) + ": " + cudaGetErrorString(e_), PFK_ERR_CUDA); \
    } while (0)

template <bool TA, bool TB>
void gemm(pfk_mlp *m, int M, int N, int K, const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb,
          const float *bias, float *C, __nv_bfloat16 *H, int ldc, cudaStream_t st)
{
    dim3 grid((N + TC_N - 1) / TC_N, (M + TC_M - 1) / TC_M);
    gemm_tc_kernel<TA, TB><<<grid, 128, TC_SMEM, st>>>(M, N, K, A, lda, B, ldb, bias, C, H, ldc, m->tc_err);
}

// Forward pass of n rows already in m->Hb[0]; leaves Y in m->Z[nl-1].
void forward(pfk_mlp *m, int n, cudaStream_t st)
{
    to_bf16_kernel<<<blocks_for(m->nparam), 256, 0, st>>>(m->p, m->wb, m->nparam);
    for (int l = 0; l < m->nl; ++l) {
        const int din = m->dims[l], dout = m->dims[l + 1];
        const bool last = l == m->nl - 1;
        gemm<false, false>(m, n, dout, din, m->Hb[l], din, m->wb + m->w_off[l], dout, m->p + m->b_off[l], m->Z[l],
                           last ? nullptr : m->Hb[l + 1], dout, st);
    }
}

// Gradients of the mean squared error for n rows (inputs in Hb[0], targets T).
void backward(pfk_mlp *m, int n, const float *T, cudaStream_t st)
{
    const int L = m->nl;
    const long long ny = (long long)n * m->dims[L];
    cudaMemsetAsync(m->loss, 0, sizeof(double), st);
    mse_grad_kernel<<<blocks_for(ny), 256, 0, st>>>(m->Z[L - 1], T, ny, 1.0f / (float)ny, m->dA, m->G, m->loss);
    for (int l = L - 1; l >= 0; --l) {
        const int din = m->dims[l], dout = m->dims[l + 1];
        // dW_l = H_{l-1}^T G  (din x dout), db_l = colsum(dZ)
        gemm<true, false>(m, din, dout, n, m->Hb[l], din, m->G, dout, nullptr, m->grad + m->w_off[l], nullptr, dout, st);
        colsum_kernel<<<(dout + 127) / 128, 128, 0, st>>>(m->dA, n, dout, m->grad + m->b_off[l]);
        if (l == 0) break;
        // dH_{l-1} = G W_l^T (n x din), then dZ_{l-1} = dH * SiLU'(Z_{l-1})
        gemm<false, true>(m, n, din, dout, m->G, dout, m->wb + m->w_off[l], dout, nullptr, m->dB, nullptr, din, st);
        const long long nh = (long long)n * din;
        silu_back_kernel<<<blocks_for(nh), 256, 0, st>>>(m->dB, m->Z[l - 1], nh, m->dA, m->G);
    }
}

// After a synchronised call: PFK_ERR_CUDA if a GEMM's tensor-core wait ran out.
pfk_status check_tc(pfk_mlp *m)
{
    int e = 0;
    MLP_CK(cudaMemcpy(&e, m->tc_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return mlp_fail(m, "tensor-core GEMM: an mbarrier wait ran out (2 s)", PFK_ERR_CUDA);
    return PFK_OK;
}

pfk_status check_batch(pfk_mlp *m, const void *X, int n)
{
    if (!m) return mlp_fail(nullptr, "null network", PFK_ERR_STATE);
    if (!X || n <= 0 || n > m->max_batch) return mlp_fail(m, "null input or batch size outside 1..max_batch", PFK_ERR_INVALID);
    cudaSetDevice(m->device);
    return PFK_OK;
}

}  // namespace

extern "C" {

pfk_status pfk_mlp_create(int nlayers, const int *dims, int max_batch, int device, pfk_mlp **out)
{
    pfk_mlp *m = nullptr;
    if (!out) return mlp_fail(nullptr, "pfk_mlp_create: out is null", PFK_ERR_INVALID);
    *out = nullptr;
    if (nlayers < 1 || nlayers > 8 || !dims || max_batch <= 0)
        return mlp_fail(nullptr, "pfk_mlp_create: need 1..8 layers, dims and max_batch > 0", PFK_ERR_INVALID);
    for (int l = 0; l <= nlayers; ++l)
        if (dims[l] <= 0 || dims[l] > 4096 || dims[l] % 8)
            return mlp_fail(nullptr, "pfk_mlp_create: layer widths must be positive multiples of 8, at most 4096",
                            PFK_ERR_INVALID);
    m = new pfk_mlp();
    m->device = device;
    m->nl = nlayers;
    m->max_batch = max_batch;
    m->dims.assign(dims, dims + nlayers + 1);
    for (int l = 0; l < nlayers; ++l) {
        m->w_off.push_back(m->nparam);
        m->nparam += (long long)dims[l] * dims[l + 1];
        m->b_off.push_back(m->nparam);
        m->nparam += dims[l + 1];
    }
    auto bail = [&](pfk_status s) {
        g_mlp_error = m->err;
        pfk_mlp_destroy(m);
        return s;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(mlp_fail(m, "cudaSetDevice failed", PFK_ERR_CUDA));
    int widest = 0;
    for (int d : m->dims) widest = std::max(widest, d);
    bool ok = cudaMalloc(&m->p, sizeof(float) * m->nparam) == cudaSuccess &&
              cudaMalloc(&m->grad, sizeof(float) * m->nparam) == cudaSuccess &&
              cudaMalloc(&m->m, sizeof(float) * m->nparam) == cudaSuccess &&
              cudaMalloc(&m->v, sizeof(float) * m->nparam) == cudaSuccess &&
              cudaMalloc(&m->wb, sizeof(__nv_bfloat16) * m->nparam) == cudaSuccess &&
              cudaMalloc(&m->dA, sizeof(float) * (size_t)max_batch * widest) == cudaSuccess &&
              cudaMalloc(&m->dB, sizeof(float) * (size_t)max_batch * widest) == cudaSuccess &&
              cudaMalloc(&m->G, sizeof(__nv_bfloat16) * (size_t)max_batch * widest) == cudaSuccess &&
              cudaMalloc(&m->loss, sizeof(double)) == cudaSuccess &&
              cudaMalloc(&m->tc_err, sizeof(int)) == cudaSuccess;
    m->Z.assign(nlayers, nullptr);
    m->Hb.assign(nlayers, nullptr);
    for (int l = 0; ok && l < nlayers; ++l)
        ok = cudaMalloc(&m->Z[l], sizeof(float) * (size_t)max_batch * dims[l + 1]) == cudaSuccess &&
             cudaMalloc(&m->Hb[l], sizeof(__nv_bfloat16) * (size_t)max_batch * dims[l]) == cudaSuccess;
    if (!ok) return bail(mlp_fail(m, "pfk_mlp_create: device allocation failed", PFK_ERR_NOMEM));
    cudaMemset(m->tc_err, 0, sizeof(int));
    cudaMemset(m->p, 0, sizeof(float) * m->nparam);
    cudaMemset(m->m, 0, sizeof(float) * m->nparam);
    cudaMemset(m->v, 0, sizeof(float) * m->nparam);
    *out = m;
    return PFK_OK;
}

pfk_status pfk_mlp_destroy(pfk_mlp *m)
{
    if (!m) return PFK_OK;
    cudaSetDevice(m->device);
    cudaDeviceSynchronize();
    for (void *x : {(void *)m->p, (void *)m->grad, (void *)m->m, (void *)m->v, (void *)m->wb, (void *)m->dA,
                    (void *)m->dB, (void *)m->G, (void *)m->loss, (void *)m->tc_err})
        if (x) cudaFree(x);
    for (float *z : m->Z)
        if (z) cudaFree(z);
    for (__nv_bfloat16 *h : m->Hb)
        if (h) cudaFree(h);
    delete m;
    return PFK_OK;
}

const char *pfk_mlp_last_error(const pfk_mlp *m) { return m ? m->err.c_str() : g_mlp_error.c_str(); }

long long pfk_mlp_param_count(const pfk_mlp *m) { return m ? m->nparam : 0; }

pfk_status pfk_mlp_set_params(pfk_mlp *m, const float *params)
{
    if (!m || !params) return mlp_fail(m, "null network or parameters", PFK_ERR_INVALID);
    cudaSetDevice(m->device);
    MLP_CK(cudaMemcpy(m->p, params, sizeof(float) * m->nparam, cudaMemcpyHostToDevice));
    MLP_CK(cudaMemset(m->m, 0, sizeof(float) * m->nparam));
    MLP_CK(cudaMemset(m->v, 0, sizeof(float) * m->nparam));
    m->step = 0;
    return PFK_OK;
}

pfk_status pfk_mlp_get_params(pfk_mlp *m, float *params)
{
    if (!m || !params) return mlp_fail(m, "null network or parameters", PFK_ERR_INVALID);
    cudaSetDevice(m->device);
    MLP_CK(cudaMemcpy(params, m->p, sizeof(float) * m->nparam, cudaMemcpyDeviceToHost));
    return PFK_OK;
}

pfk_status pfk_mlp_forward(pfk_mlp *m, const float *dX, int n, float *dY, void *stream)
{
    pfk_status s = check_batch(m, dX, n);
    if (s != PFK_OK) return s;
    if (!dY) return mlp_fail(m, "null output", PFK_ERR_INVALID);
    cudaStream_t st = (cudaStream_t)stream;
    const long long nx = (long long)n * m->dims[0];
    to_bf16_kernel<<<blocks_for(nx), 256, 0, st>>>(dX, m->Hb[0], nx);
    forward(m, n, st);
    MLP_CK(cudaMemcpyAsync(dY, m->Z[m->nl - 1], sizeof(float) * (size_t)n * m->dims[m->nl], cudaMemcpyDeviceToDevice,
                           st));
    MLP_CK(cudaStreamSynchronize(st));
    MLP_CK(cudaGetLastError());
    return check_tc(m);
}

pfk_status pfk_mlp_gradients(pfk_mlp *m, const float *dX, const float *dT, int n, float *grads, double *loss,
                             void *stream)
{
    pfk_status s = check_batch(m, dX, n);
    if (s != PFK_OK) return s;
    if (!dT) return mlp_fail(m, "null targets", PFK_ERR_INVALID);
    cudaStream_t st = (cudaStream_t)stream;
    const long long nx = (long long)n * m->dims[0];
    to_bf16_kernel<<<blocks_for(nx), 256, 0, st>>>(dX, m->Hb[0], nx);
    forward(m, n, st);
    backward(m, n, dT, st);
    if (grads) MLP_CK(cudaMemcpyAsync(grads, m->grad, sizeof(float) * m->nparam, cudaMemcpyDeviceToHost, st));
    if (loss) MLP_CK(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    MLP_CK(cudaStreamSynchronize(st));
    MLP_CK(cudaGetLastError());
    return check_tc(m);
}

pfk_status pfk_mlp_train_step(pfk_mlp *m, const float *dX, const float *dT, int n, float lr, double *loss,
                              void *stream)
{
    pfk_status s = check_batch(m, dX, n);
    if (s != PFK_OK) return s;
    if (!dT || !(lr > 0.0f)) return mlp_fail(m, "null targets or non-positive learning rate", PFK_ERR_INVALID);
    cudaStream_t st = (cudaStream_t)stream;
    const long long nx = (long long)n * m->dims[0];
    to_bf16_kernel<<<blocks_for(nx), 256, 0, st>>>(dX, m->Hb[0], nx);
    forward(m, n, st);
    backward(m, n, dT, st);
    m->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f / (1.0f - powf(b1, (float)m->step)), c2 = 1.0f / (1.0f - powf(b2, (float)m->step));
    adam_kernel<<<blocks_for(m->nparam), 256, 0, st>>>(m->p, m->grad, m->m, m->v, m->nparam, lr, b1, b2, 1e-8f, c1,
                                                       c2);
    if (loss) MLP_CK(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    MLP_CK(cudaStreamSynchronize(st));
    MLP_CK(cudaGetLastError());
    return check_tc(m);
}

}  // extern "C"
