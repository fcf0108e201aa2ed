// pfk_mlp.cu -- the learned-guess network: a small multilayer perceptron
// trained and evaluated by this file's kernels on the GPU.
//
//   H_0 = bf16(X);  Z_l = H_{l-1} W_l + b_l;  H_l = bf16(SiLU(Z_l)) (l < L);
//   Y = Z_L (FP32).
//
// Every matrix product runs on the tensor cores as BF16 x BF16 with FP32
// accumulation (mma.sync m16n8k16); weights are kept in FP32 (Adam's master
// copy) and rounded to BF16 for the products.  Training minimises the mean
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
// GEMM: C[m][n] = sum_k A(m, k) B(k, n), A(m,k) = A[m*lda + k] (or A[k*lda + m]
// when TA), B(k,n) = B[k*ldb + n] (or B[n*ldb + k] when TB); BF16 operands,
// FP32 accumulation; epilogue adds bias[n] and writes C (FP32) and/or
// H = bf16(SiLU(C)).  Tile 64 x 64 per block of 128 threads (four warps, a
// 32 x 32 sub-tile each), K in steps of 16 staged in shared memory with
// bounds checks (out-of-range elements read as zero).
// ---------------------------------------------------------------------------
constexpr int BM = 64, BN = 64, BK = 16;

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

template <bool TA, bool TB>
__global__ void __launch_bounds__(128) gemm_bf16_kernel(int M, int N, int K, const __nv_bfloat16 *__restrict__ A,
                                                        int lda, const __nv_bfloat16 *__restrict__ B, int ldb,
                                                        const float *__restrict__ bias, float *C,
                                                        __nv_bfloat16 *H, int ldc)
{
    __shared__ __nv_bfloat16 As[BM][BK + 8];   // [m][k]
    __shared__ __nv_bfloat16 Bs[BN][BK + 8];   // [n][k]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int g = lane >> 2, q = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0f;

    for (int k0 = 0; k0 < K; k0 += BK) {
        // stage A (64 x 16) and B^T (64 x 16): 1024 elements each, 8 per thread
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int idx = tid + e * 128;
            const int r = idx / BK, c = idx % BK;       // r: m or n, c: k
            const int gm = m0 + r, gk = k0 + c, gn = n0 + r;
            __nv_bfloat16 va = __float2bfloat16(0.0f), vb = __float2bfloat16(0.0f);
            if (gm < M && gk < K) va = TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
            if (gn < N && gk < K) vb = TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
            As[r][c] = va;
            Bs[r][c] = vb;
        }
        __syncthreads();
        unsigned af[2][4], bf[4][2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r = wm + i * 16 + g;
            af[i][0] = pack2(As[r][2 * q], As[r][2 * q + 1]);
            af[i][1] = pack2(As[r + 8][2 * q], As[r + 8][2 * q + 1]);
            af[i][2] = pack2(As[r][2 * q + 8], As[r][2 * q + 9]);
            af[i][3] = pack2(As[r + 8][2 * q + 8], As[r + 8][2 * q + 9]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int cidx = wn + j * 8 + g;
            bf[j][0] = pack2(Bs[cidx][2 * q], Bs[cidx][2 * q + 1]);
            bf[j][1] = pack2(Bs[cidx][2 * q + 8], Bs[cidx][2 * q + 9]);
        }
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                asm volatile(
                    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                    "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                    : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
                    : "r"(af[i][0]), "r"(af[i][1]), "r"(af[i][2]), "r"(af[i][3]), "r"(bf[j][0]), "r"(bf[j][1]));
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int m = m0 + wm + i * 16 + g + (r >= 2 ? 8 : 0);
                const int n = n0 + wn + j * 8 + 2 * q + (r & 1);
                if (m < M && n < N) {
                    float v = acc[i][j][r];
                    if (bias) v += bias[n];
                    if (C) C[(size_t)m * ldc + n] = v;
                    if (H) H[(size_t)m * ldc + n] = __float2bfloat16(silu(v));
                }
            }
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
void gemm(int M, int N, int K, const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, const float *bias,
          float *C, __nv_bfloat16 *H, int ldc, cudaStream_t st)
{
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    gemm_bf16_kernel<TA, TB><<<grid, 128, 0, st>>>(M, N, K, A, lda, B, ldb, bias, C, H, ldc);
}

// Forward pass of n rows already in m->Hb[0]; leaves Y in m->Z[nl-1].
void forward(pfk_mlp *m, int n, cudaStream_t st)
{
    to_bf16_kernel<<<blocks_for(m->nparam), 256, 0, st>>>(m->p, m->wb, m->nparam);
    for (int l = 0; l < m->nl; ++l) {
        const int din = m->dims[l], dout = m->dims[l + 1];
        const bool last = l == m->nl - 1;
        gemm<false, false>(n, dout, din, m->Hb[l], din, m->wb + m->w_off[l], dout, m->p + m->b_off[l], m->Z[l],
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
        gemm<true, false>(din, dout, n, m->Hb[l], din, m->G, dout, nullptr, m->grad + m->w_off[l], nullptr, dout, st);
        colsum_kernel<<<(dout + 127) / 128, 128, 0, st>>>(m->dA, n, dout, m->grad + m->b_off[l]);
        if (l == 0) break;
        // dH_{l-1} = G W_l^T (n x din), then dZ_{l-1} = dH * SiLU'(Z_{l-1})
        gemm<false, true>(n, din, dout, m->G, dout, m->wb + m->w_off[l], dout, nullptr, m->dB, nullptr, din, st);
        const long long nh = (long long)n * din;
        silu_back_kernel<<<blocks_for(nh), 256, 0, st>>>(m->dB, m->Z[l - 1], nh, m->dA, m->G);
    }
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
              cudaMalloc(&m->loss, sizeof(double)) == cudaSuccess;
    m->Z.assign(nlayers, nullptr);
    m->Hb.assign(nlayers, nullptr);
    for (int l = 0; ok && l < nlayers; ++l)
        ok = cudaMalloc(&m->Z[l], sizeof(float) * (size_t)max_batch * dims[l + 1]) == cudaSuccess &&
             cudaMalloc(&m->Hb[l], sizeof(__nv_bfloat16) * (size_t)max_batch * dims[l]) == cudaSuccess;
    if (!ok) return bail(mlp_fail(m, "pfk_mlp_create: device allocation failed", PFK_ERR_NOMEM));
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
                    (void *)m->dB, (void *)m->G, (void *)m->loss})
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
    return PFK_OK;
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
    return PFK_OK;
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
    return PFK_OK;
}

}  // extern "C"
