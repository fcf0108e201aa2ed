// pfk_scf.cu -- the RHF loop on the device behind the C ABI (pfk_scf_rhf).
//
// The steps of the reference's run_rhf (src/scf/scf.cpp:175-441) with the
// two-electron part from the context's Fock build, launched directly on the
// loop's own stream (no graph capture, so that several loops, one per
// context, can run at once from host threads; capturing in several threads
// at once failed with cudaStreamWaitEvent "invalid argument" there):
//   * symmetric orthogonaliser X = S^-1/2 (scf.cpp:15-20);
//   * default guess from the eigenvectors of X^T H X (scf.cpp:33-45), or the
//     caller's density, which enters like a ReadDensity guess
//     (scf.cpp:213-216);
//   * per iteration F = H + G(P), E = 1/2 sum P (H + F) + E_nuc, Pulay DIIS
//     over the last 8 Fock matrices with error X^T (F P S - S P F) X
//     (types.h:759-837), diagonalisation of X^T F X, P = 2 C_occ C_occ^T;
//   * converged when |dE| < 1e-10 and the rms and max of dP are below 1e-10,
//     not before the second iteration (scf.cpp:126-135); at most 50, 100,
//     200 or 300 iterations by basis size (types.h:356-363).
// Everything stays FP64 on the device: the products are cuBLAS DGEMMs, the
// diagonalisations cuSOLVER's Dsyevd, the sums this file's fixed-order
// reductions (so a run is bitwise reproducible).  The DIIS system, at most
// 9 x 9, is solved on the host by Householder QR with column pivoting and a
// relative rank cut-off, the least-squares solver the reference uses there
// (types.h:813).  Not in the reference: optional FP32 builds on the
// difference density between full builds (a second context), with a full
// build at least every `full_every` iterations and for the final energy.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cublas_v2.h>
#include <cusolverDn.h>

#include "../../include/planck_fock.h"
#include "pfk_internal.h"

namespace pfk {

// The RHF build G(dP) on stream st launched directly, without capturing a
// graph (pfk_api.cu; pfk_fock_rhf_device captures one per (dP, dG, stream)).
pfk_status fock_rhf_direct(pfk_ctx *ctx, const double *dP, double *dG, cudaStream_t st);

namespace {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 256;   // fixed partial count: the reduction order does not depend on the GPU

// Fixed-order partial sums of sum(a .* b) (b == nullptr: sum(a .* a)) and
// max |a| over n elements: block k reduces the elements k, k + kRedBlocks *
// kRedThreads, ... in a fixed tree; the host adds the kRedBlocks partials in
// index order.
__global__ void __launch_bounds__(kRedThreads) dot_max_kernel(const double *__restrict__ a,
                                                              const double *__restrict__ b, long long n,
                                                              double *part_sum, double *part_max)
{
    __shared__ double ss[kRedThreads], sm[kRedThreads];
    double s = 0.0, m = 0.0;
    for (long long i = (long long)blockIdx.x * kRedThreads + threadIdx.x; i < n;
         i += (long long)kRedBlocks * kRedThreads) {
        const double x = a[i];
        s += x * (b ? b[i] : x);
        m = fmax(m, fabs(x));
    }
    ss[threadIdx.x] = s;
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            ss[threadIdx.x] += ss[threadIdx.x + w];
            sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part_sum[blockIdx.x] = ss[0];
        part_max[blockIdx.x] = sm[0];
    }
}

// out = a + s * b (elementwise; out may alias a)
__global__ void axpby_kernel(const double *a, double s, const double *b, double *out, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[i] + s * b[i];
}

// out = M - M^T (row-major n x n)
__global__ void antisym_kernel(const double *__restrict__ M, double *out, int n)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * n) return;
    const int i = (int)(t / n), j = (int)(t % n);
    out[t] = M[t] - M[(size_t)j * n + i];
}

// columns of U scaled by f(s_j): out[i][j] = U[i][j] * s_j^-1/2 (column-major U)
__global__ void scale_cols_kernel(const double *__restrict__ U, const double *__restrict__ s, double *out, int n)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * n) return;
    const int j = (int)(t / n);   // column-major: t = j * n + i
    out[t] = U[t] / sqrt(s[j]);
}

// Householder QR with column pivoting of the m x m system B x = rhs (row-major
// B), least-squares solution with the rank cut-off |R_kk| > m eps |R_00|;
// unknowns beyond the rank are zero.
std::vector<double> lstsq_pivoted(std::vector<double> A, std::vector<double> b, int m)
{
    std::vector<int> piv(m);
    for (int j = 0; j < m; ++j) piv[j] = j;
    std::vector<double> norms(m);
    for (int j = 0; j < m; ++j) {
        double s = 0.0;
        for (int i = 0; i < m; ++i) s += A[i * m + j] * A[i * m + j];
        norms[j] = s;
    }
    for (int k = 0; k < m; ++k) {
        // pivot: the remaining column of largest norm below row k
        int best = k;
        double bn = -1.0;
        for (int j = k; j < m; ++j) {
            double s = 0.0;
            for (int i = k; i < m; ++i) s += A[i * m + j] * A[i * m + j];
            if (s > bn) {
                bn = s;
                best = j;
            }
        }
        if (best != k) {
            for (int i = 0; i < m; ++i) std::swap(A[i * m + k], A[i * m + best]);
            std::swap(piv[k], piv[best]);
        }
        // Householder reflector for column k, rows k..m-1
        double alpha = 0.0;
        for (int i = k; i < m; ++i) alpha += A[i * m + k] * A[i * m + k];
        alpha = std::sqrt(alpha);
        if (alpha == 0.0) continue;
        if (A[k * m + k] > 0) alpha = -alpha;
        std::vector<double> v(m, 0.0);
        for (int i = k; i < m; ++i) v[i] = A[i * m + k];
        v[k] -= alpha;
        double vn = 0.0;
        for (int i = k; i < m; ++i) vn += v[i] * v[i];
        if (vn == 0.0) continue;
        for (int j = k; j < m; ++j) {
            double d = 0.0;
            for (int i = k; i < m; ++i) d += v[i] * A[i * m + j];
            const double f = 2.0 * d / vn;
            for (int i = k; i < m; ++i) A[i * m + j] -= f * v[i];
        }
        double d = 0.0;
        for (int i = k; i < m; ++i) d += v[i] * b[i];
        const double f = 2.0 * d / vn;
        for (int i = k; i < m; ++i) b[i] -= f * v[i];
    }
    const double r00 = std::fabs(A[0]);
    int rank = 0;
    while (rank < m && std::fabs(A[rank * m + rank]) > m * 2.220446049250313e-16 * r00) ++rank;
    std::vector<double> y(m, 0.0), x(m, 0.0);
    for (int k = rank - 1; k >= 0; --k) {
        double s = b[k];
        for (int j = k + 1; j < rank; ++j) s -= A[k * m + j] * y[j];
        y[k] = s / A[k * m + k];
    }
    for (int k = 0; k < rank; ++k) x[piv[k]] = y[k];
    return x;
}

struct Dev {
    std::vector<void *> ptrs;
    ~Dev()
    {
        for (void *p : ptrs) cudaFree(p);
    }
    cudaError_t get(double **p, size_t n)
    {
        cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), sizeof(double) * std::max<size_t>(n, 1));
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
};

struct Handles {
    cublasHandle_t blas = nullptr;
    cusolverDnHandle_t sol = nullptr;
    ~Handles()
    {
        if (blas) cublasDestroy(blas);
        if (sol) cusolverDnDestroy(sol);
    }
};

}  // namespace
}  // namespace pfk

using namespace pfk;

extern "C" pfk_status pfk_scf_rhf(pfk_ctx *ctx, const double *H, const double *S, double enuc, int nocc,
                                  const double *P0, const double *G0, const pfk_scf_options *opt,
                                  pfk_scf_result *res, double *P_out, double *C_out, double *eps_out)
{
    if (!ctx) return PFK_ERR_STATE;
    const int nb = pfk_nbasis(ctx);
    if (!H || !S || !res) return ctx_fail(ctx, PFK_ERR_INVALID, "pfk_scf_rhf: H, S and res must be given");
    if (nocc < 1 || nocc > nb) return ctx_fail(ctx, PFK_ERR_INVALID, "pfk_scf_rhf: need 1 <= nocc <= nbasis");
    if (G0 && !P0) return ctx_fail(ctx, PFK_ERR_INVALID, "pfk_scf_rhf: G0 needs P0");
    pfk_scf_options o{};
    o.max_iter = 0;
    o.tol_energy = 1e-10;
    o.tol_density = 1e-10;
    o.diis_depth = 8;
    o.incremental = nullptr;
    o.incremental_below = 1e-4;
    o.incremental_floor = 1e-8;
    o.full_every = 8;
    o.history = nullptr;
    if (opt) o = *opt;
    if (o.diis_depth < 1 || o.diis_depth > 32) return ctx_fail(ctx, PFK_ERR_INVALID, "pfk_scf_rhf: diis_depth 1..32");
    if (o.incremental && pfk_nbasis(o.incremental) != nb)
        return ctx_fail(ctx, PFK_ERR_INVALID, "pfk_scf_rhf: the incremental context has another basis");
    const int max_iter = o.max_iter > 0 ? o.max_iter : nb > 1000 ? 300 : nb > 500 ? 200 : nb > 250 ? 100 : 50;
    const auto t_start = std::chrono::steady_clock::now();
    std::memset(res, 0, sizeof(*res));

    cudaSetDevice(ctx_device(ctx));
    const size_t n2 = (size_t)nb * nb, bytes = sizeof(double) * n2;
    const int D = o.diis_depth;
#define SCF_CK(call)                                                                        \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return ctx_fail(ctx, PFK_ERR_CUDA, std::string("pfk_scf_rhf: " #call ": ") + cudaGetErrorString(e_)); \
    } while (0)
#define SCF_BL(call)                                                                        \
    do {                                                                                    \
        if ((call) != CUBLAS_STATUS_SUCCESS)                                                \
            return ctx_fail(ctx, PFK_ERR_CUDA, "pfk_scf_rhf: cuBLAS call failed: " #call);  \
    } while (0)
#define SCF_SO(call)                                                                        \
    do {                                                                                    \
        if ((call) != CUSOLVER_STATUS_SUCCESS)                                              \
            return ctx_fail(ctx, PFK_ERR_CUDA, "pfk_scf_rhf: cuSOLVER call failed: " #call); \
    } while (0)

    cudaStream_t st = nullptr;
    SCF_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{st};
    Handles h;
    Dev dv;
    // the libraries' own choices pinned, so that a run's bits depend only on
    // its inputs: no atomics in cuBLAS, a fixed cuBLAS workspace (its kernel
    // choice can depend on the workspace it finds), cuSOLVER's deterministic
    // mode
    constexpr size_t kBlasWorkspace = size_t(32) << 20;
    double *dBlasWs = nullptr;
    SCF_CK(dv.get(&dBlasWs, kBlasWorkspace / sizeof(double)));
    SCF_BL(cublasCreate(&h.blas));
    SCF_BL(cublasSetStream(h.blas, st));
    SCF_BL(cublasSetAtomicsMode(h.blas, CUBLAS_ATOMICS_NOT_ALLOWED));
    SCF_BL(cublasSetWorkspace(h.blas, dBlasWs, kBlasWorkspace));
    SCF_SO(cusolverDnCreate(&h.sol));
    SCF_SO(cusolverDnSetStream(h.sol, st));
    SCF_SO(cusolverDnSetDeterministicMode(h.sol, CUSOLVER_DETERMINISTIC_RESULTS));

    double *dH, *dS, *dX, *dP, *dPb, *dG, *dGd, *dF, *dT1, *dT2, *dE, *dW, *dPart, *dFs, *dEs, *dDP;
    for (double **p : {&dH, &dS, &dX, &dP, &dPb, &dG, &dGd, &dF, &dT1, &dT2, &dE, &dDP}) SCF_CK(dv.get(p, n2));
    SCF_CK(dv.get(&dW, nb));
    SCF_CK(dv.get(&dPart, 2 * kRedBlocks));
    SCF_CK(dv.get(&dFs, n2 * D));
    SCF_CK(dv.get(&dEs, n2 * D));
    int lwork = 0, *dInfo = nullptr;
    SCF_SO(cusolverDnDsyevd_bufferSize(h.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nb, dT1, nb, dW,
                                       &lwork));
    double *dWork;
    SCF_CK(dv.get(&dWork, (size_t)lwork));
    SCF_CK(dv.get(reinterpret_cast<double **>(&dInfo), 1));
    SCF_CK(cudaMemcpyAsync(dH, H, bytes, cudaMemcpyHostToDevice, st));
    SCF_CK(cudaMemcpyAsync(dS, S, bytes, cudaMemcpyHostToDevice, st));

    const unsigned g2 = (unsigned)((n2 + 255) / 256);
    const double one = 1.0, zero = 0.0, two = 2.0;
    std::vector<double> hpart(2 * kRedBlocks);
    // sum(a .* b) (b null: a .* a) and max |a|, in a fixed order
    auto reduce = [&](const double *a, const double *b, double &sum, double &mx) -> cudaError_t {
        dot_max_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(a, b, (long long)n2, dPart, dPart + kRedBlocks);
        cudaError_t e = cudaMemcpyAsync(hpart.data(), dPart, sizeof(double) * 2 * kRedBlocks, cudaMemcpyDeviceToHost,
                                        st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        sum = 0.0;
        mx = 0.0;
        for (int k = 0; k < kRedBlocks; ++k) {
            sum += hpart[k];
            mx = std::max(mx, hpart[kRedBlocks + k]);
        }
        return e;
    };
    // eigenvectors of the symmetric matrix in dT1 (overwritten by them, column
    // major), eigenvalues in dW
    auto syevd = [&]() -> pfk_status {
        SCF_SO(cusolverDnDsyevd(h.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nb, dT1, nb, dW, dWork,
                                lwork, dInfo));
        int info = 0;
        SCF_CK(cudaMemcpyAsync(&info, dInfo, sizeof(int), cudaMemcpyDeviceToHost, st));
        SCF_CK(cudaStreamSynchronize(st));
        if (info != 0) return ctx_fail(ctx, PFK_ERR_CUDA, "pfk_scf_rhf: Dsyevd did not converge");
        return PFK_OK;
    };
    // The matrices are symmetric, so row- and column-major storage coincide
    // for H, S, F, P and G; X is symmetric as well.  C (column-major, from
    // the eigenvectors) is the one non-symmetric matrix.
    // X = U s^-1/2 U^T
    SCF_CK(cudaMemcpyAsync(dT1, dS, bytes, cudaMemcpyDeviceToDevice, st));
    if (pfk_status s = syevd(); s != PFK_OK) return s;
    scale_cols_kernel<<<g2, 256, 0, st>>>(dT1, dW, dT2, nb);
    SCF_BL(cublasDgemm(h.blas, CUBLAS_OP_N, CUBLAS_OP_T, nb, nb, nb, &one, dT2, nb, dT1, nb, &zero, dX, nb));

    // new density from a Fock matrix in dF: T1 = X^T F X, eigenvectors, C = X C',
    // P = 2 C_occ C_occ^T (into dst); C stays in dT2 (column-major)
    auto density_from = [&](const double *Fm, double *dst) -> pfk_status {
        SCF_BL(cublasDgemm(h.blas, CUBLAS_OP_N, CUBLAS_OP_N, nb, nb, nb, &one, Fm, nb, dX, nb, &zero, dT2, nb));
        SCF_BL(cublasDgemm(h.blas, CUBLAS_OP_T, CUBLAS_OP_N, nb, nb, nb, &one, dX, nb, dT2, nb, &zero, dT1, nb));
        if (pfk_status s = syevd(); s != PFK_OK) return s;
        SCF_BL(cublasDgemm(h.blas, CUBLAS_OP_N, CUBLAS_OP_N, nb, nb, nb, &one, dX, nb, dT1, nb, &zero, dT2, nb));
        SCF_BL(cublasDgemm(h.blas, CUBLAS_OP_N, CUBLAS_OP_T, nb, nb, nocc, &two, dT2, nb, dT2, nb, &zero, dst, nb));
        return PFK_OK;
    };
    if (P0) {
        SCF_CK(cudaMemcpyAsync(dP, P0, bytes, cudaMemcpyHostToDevice, st));
    } else {
        if (pfk_status s = density_from(dH, dP); s != PFK_OK) return s;
    }
    if (G0) SCF_CK(cudaMemcpyAsync(dG, G0, bytes, cudaMemcpyHostToDevice, st));

    std::vector<double> B((size_t)(D + 1) * (D + 1), 0.0);   // error overlaps of the stored vectors
    int nvec = 0, head = 0;                                   // ring of the last D (F, e)
    double E_prev = 0.0, E = 0.0, build_ms = 0.0;
    int since_full = 0, full_builds = 0, diff_builds = 0;
    bool have_G = false, converged = false;
    int it = 0;
    cudaEvent_t ev0, ev1;
    SCF_CK(cudaEventCreate(&ev0));
    SCF_CK(cudaEventCreate(&ev1));
    struct EventGuard {
        cudaEvent_t a, b;
        ~EventGuard()
        {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } eg{ev0, ev1};
    auto build = [&](pfk_ctx *c, const double *src, double *dst) -> pfk_status {
        SCF_CK(cudaEventRecord(ev0, st));
        pfk_status s = fock_rhf_direct(c, src, dst, st);
        if (s != PFK_OK) return ctx_fail(ctx, s, std::string("pfk_scf_rhf: build: ") + pfk_last_error(c));
        SCF_CK(cudaEventRecord(ev1, st));
        SCF_CK(cudaEventSynchronize(ev1));
        float ms = 0.f;
        SCF_CK(cudaEventElapsedTime(&ms, ev0, ev1));
        build_ms += ms;
        return PFK_OK;
    };
    for (it = 1; it <= max_iter; ++it) {
        // G(P): the caller's first build, a difference build, or a full build
        double dmax_built = 0.0;
        if (o.incremental && have_G && since_full + 1 < o.full_every) {
            axpby_kernel<<<g2, 256, 0, st>>>(dP, -1.0, dPb, dDP, (long long)n2);
            double dummy;
            SCF_CK(reduce(dDP, nullptr, dummy, dmax_built));
        }
        if (it == 1 && G0) {
            since_full = 0;
        } else if (o.incremental && have_G && since_full + 1 < o.full_every && dmax_built >= o.incremental_floor &&
                   dmax_built < o.incremental_below) {
            if (pfk_status s = build(o.incremental, dDP, dGd); s != PFK_OK) return s;
            axpby_kernel<<<g2, 256, 0, st>>>(dG, 1.0, dGd, dG, (long long)n2);
            ++since_full;
            ++diff_builds;
        } else {
            if (pfk_status s = build(ctx, dP, dG); s != PFK_OK) return s;
            since_full = 0;
            ++full_builds;
        }
        have_G = true;
        SCF_CK(cudaMemcpyAsync(dPb, dP, bytes, cudaMemcpyDeviceToDevice, st));
        // F = H + G, E = 1/2 (P.H + P.F) + E_nuc
        axpby_kernel<<<g2, 256, 0, st>>>(dH, 1.0, dG, dF, (long long)n2);
        double pH, pF, mx;
        SCF_CK(reduce(dP, dH, pH, mx));
        SCF_CK(reduce(dP, dF, pF, mx));
        E = 0.5 * (pH + pF) + enuc;
        if (it == 1) res->first_energy = E;
        // error X^T (F P S - S P F) X = X^T (M - M^T) X with M = F P S
        SCF_BL(cublasDgemm(h.blas, CUBLAS_OP_N, CUBLAS_OP_N, nb, nb, nb, &one, dF, nb, dP, nb, &zero, dT1, nb));
        SCF_BL(cublasDgemm(h.blas, CUBLAS_OP_N, CUBLAS_OP_N, nb, nb, nb, &one, dT1, nb, dS, nb, &zero, dT2, nb));
        antisym_kernel<<<g2, 256, 0, st>>>(dT2, dT1, nb);
        SCF_BL(cublasDgemm(h.blas, CUBLAS_OP_N, CUBLAS_OP_N, nb, nb, nb, &one, dT1, nb, dX, nb, &zero, dT2, nb));
        double *e_slot = dEs + n2 * head, *f_slot = dFs + n2 * head;
        SCF_BL(cublasDgemm(h.blas, CUBLAS_OP_N, CUBLAS_OP_N, nb, nb, nb, &one, dX, nb, dT2, nb, &zero, e_slot, nb));
        SCF_CK(cudaMemcpyAsync(f_slot, dF, bytes, cudaMemcpyDeviceToDevice, st));
        // DIIS: overlaps of the new error with every stored one (slot order
        // = age order: oldest first, as the reference's deque)
        nvec = std::min(nvec + 1, D);
        std::vector<int> order(nvec);
        for (int k = 0; k < nvec; ++k) order[k] = ((head - (nvec - 1) + k) % D + D) % D;
        std::vector<double> ov(D, 0.0);
        for (int k = 0; k < nvec; ++k) {
            double s;
            SCF_CK(reduce(e_slot, dEs + n2 * order[k], s, mx));
            ov[order[k]] = s;
        }
        // B holds overlaps by slot; refresh the new slot's row and column
        for (int k = 0; k < D; ++k) B[(size_t)head * D + k] = B[(size_t)k * D + head] = ov[k];
        const double *Fx = dF;
        if (nvec >= 2) {
            const int m = nvec;
            std::vector<double> A((size_t)(m + 1) * (m + 1), -1.0), rhs(m + 1, 0.0);
            for (int a = 0; a < m; ++a)
                for (int b = 0; b < m; ++b) A[(size_t)a * (m + 1) + b] = B[(size_t)order[a] * D + order[b]];
            A[(size_t)m * (m + 1) + m] = 0.0;
            rhs[m] = -1.0;
            const std::vector<double> c = lstsq_pivoted(A, rhs, m + 1);
            SCF_CK(cudaMemsetAsync(dT1, 0, bytes, st));
            for (int a = 0; a < m; ++a)
                axpby_kernel<<<g2, 256, 0, st>>>(dT1, c[a], dFs + n2 * order[a], dT1, (long long)n2);
            SCF_CK(cudaMemcpyAsync(dE, dT1, bytes, cudaMemcpyDeviceToDevice, st));
            Fx = dE;
        }
        head = (head + 1) % D;
        // new density; convergence on dE and the rms / max of dP
        if (pfk_status s = density_from(Fx, dDP); s != PFK_OK) return s;   // dDP <- P_new
        axpby_kernel<<<g2, 256, 0, st>>>(dDP, -1.0, dP, dT1, (long long)n2);   // dP step
        double ss, dmax;
        SCF_CK(reduce(dT1, nullptr, ss, dmax));
        const double drms = std::sqrt(ss / (double)n2), dE = std::fabs(E - E_prev);
        SCF_CK(cudaMemcpyAsync(dP, dDP, bytes, cudaMemcpyDeviceToDevice, st));
        E_prev = E;
        if (o.history) {
            double *hrow = o.history + 6 * (size_t)(it - 1);
            hrow[0] = it;
            hrow[1] = E;
            hrow[2] = dE;
            hrow[3] = drms;
            hrow[4] = dmax;
            hrow[5] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
        }
        if (it > 1 && dE < o.tol_energy && drms < o.tol_density && dmax < o.tol_density) {
            converged = true;
            break;
        }
    }
    if (converged && o.incremental && since_full > 0) {
        // report the energy of a full build at the converged density
        if (pfk_status s = build(ctx, dP, dG); s != PFK_OK) return s;
        ++full_builds;
        axpby_kernel<<<g2, 256, 0, st>>>(dH, 1.0, dG, dF, (long long)n2);
        double pH, pF, mx;
        SCF_CK(reduce(dP, dH, pH, mx));
        SCF_CK(reduce(dP, dF, pF, mx));
        E_prev = 0.5 * (pH + pF) + enuc;
    }
    res->energy = E_prev;
    res->iterations = converged ? it : max_iter;
    res->converged = converged ? 1 : 0;
    res->full_builds = full_builds;
    res->difference_builds = diff_builds;
    res->build_ms = build_ms;
    if (P_out) SCF_CK(cudaMemcpyAsync(P_out, dP, bytes, cudaMemcpyDeviceToHost, st));
    if (C_out) SCF_CK(cudaMemcpyAsync(C_out, dT2, bytes, cudaMemcpyDeviceToHost, st));
    if (eps_out) SCF_CK(cudaMemcpyAsync(eps_out, dW, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
    SCF_CK(cudaStreamSynchronize(st));
    res->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
#undef SCF_CK
#undef SCF_BL
#undef SCF_SO
    return PFK_OK;
}
