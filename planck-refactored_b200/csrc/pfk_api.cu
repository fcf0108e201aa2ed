// pfk_api.cu -- the C ABI (include/planck_fock.h): context, per-geometry
// setup, and the per-iteration Fock builds.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include <cublas_v2.h>

#include "../../include/planck_fock.h"
#include "pfk_internal.h"
#include "pfk_setup.h"

using namespace pfk;

namespace pfk {
ClassLauncher g_class_launchers[kQuartetClasses];   // constant-initialised; filled by the class units
}

namespace {

thread_local std::string g_last_error;   // for failures without a context

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }   // the temporaries of list building are freed on every path
    cudaError_t alloc(size_t count)
    {
        release();
        n = count;
        if (count == 0) return cudaSuccess;
        return cudaMalloc(reinterpret_cast<void **>(&p), sizeof(T) * count);
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

struct GraphEntry {
    const void *in;
    void *out;
    cudaStream_t stream;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

}  // namespace

constexpr int kMaxLanes = 4;

struct pfk_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    // concurrent class launches: lanes - 1 side streams forked from the
    // build's stream (fork_ev) and joined back (join_ev) around the classes
    int lanes = kMaxLanes;
    cudaStream_t side[kMaxLanes - 1] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[kMaxLanes - 1] = {};
    cublasHandle_t blas = nullptr;   // created by the first pfk_mo_transform
    double mo_ms[3] = {0.0, 0.0, 0.0};   // last pfk_mo_transform: AO tensor, GEMMs, copy out
    // two pinned staging chunks for copying MO blocks into pageable host memory
    void *pin[2] = {nullptr, nullptr};
    cudaEvent_t pin_ev[2] = {nullptr, nullptr};

    int nshell = 0, nb = 0;
    std::vector<int> L, bf_off;
    DevBuf<int> d_shell_bf, d_shell_nbf;      // per shell: first basis function, function count
    double dscreen_tol = 0.0;                 // density screening threshold (0: off)
    DevBuf<float> d_Dsh;                      // per shell-pair block max |P| (nb x nb, block corners)

    int npairs = 0;
    std::vector<PairInfo> pairs;
    std::vector<int> pair_pc, pair_la, pair_lb;
    std::vector<PrimPair> prims;
    DevBuf<PairInfo> d_pairs;
    DevBuf<PrimPair> d_prims;
    DevBuf<int> d_pair_la, d_pair_lb;

    std::vector<double> Q;
    DevBuf<double> d_Q;

    std::vector<int> cls_ids[kPairClasses];
    DevBuf<int> d_cls_ids[kPairClasses];
    DevBuf<double> d_cls_q[kPairClasses];
    DevBuf<long long> d_cls_kpref[kPairClasses];   // prefix of nprim over the sorted class list

    long long prim_cnt[kQuartetClasses] = {};   // primitive quartets (all primitives), per class
    long long prim32_cnt[kQuartetClasses] = {}; // the part of prim_cnt on the FP32 list
    int shard_rank = 0, shard_n = 1;             // builds evaluate every shard_n-th quartet

    double tol = 1e-10, fp32_bound = 1e-8;
    double prim_tol = kPrimQuartetTol;   // primitive-quartet bound below which builds skip it
    int engine = PFK_ENGINE_OS, precision = PFK_PREC_FP64;

    DevBuf<uint2> d_quart;
    long long q_off[kQuartetClasses] = {}, q_cnt[kQuartetClasses] = {};
    long long q32_off[kQuartetClasses] = {}, q32_cnt[kQuartetClasses] = {};
    ClassLauncher launch[kQuartetClasses] = {};
    float class_ms[kQuartetClasses] = {};
    // engine auto: launch flags per class (kLaunchOS / kLaunchDense or 0 for
    // Rys); the static rule until pfk_autotune measures the candidates
    int auto_flags[kQuartetClasses] = {};

    DevBuf<double> d_P, d_Pb, d_Pt, d_G, d_Gb;
    DevBuf<FxWord> d_J, d_K0, d_K1;   // fixed-point accumulators, 2 nb^2 words each
    std::vector<GraphEntry> graphs;

    pfk_status fail(pfk_status s, const std::string &msg)
    {
        err = msg;
        return s;
    }
    pfk_status cuda_fail(const char *what, cudaError_t e)
    {
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return PFK_ERR_CUDA;
    }
};

#define PFK_CK(call)                                                    \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return ctx->cuda_fail(#call, e_);        \
    } while (0)

namespace {

constexpr double kPi = 3.14159265358979323846;

// Basis checks before any device work.  check_nbasis: contexts index basis
// functions with 16 bits in the quartet codes (ERI batches do not).
pfk_status validate(const pfk_basis_desc *b, std::string &why, bool check_nbasis = true)
{
    if (!b || b->nshell <= 0 || !b->L || !b->nprim || !b->center || !b->expo || !b->coef || !b->norm) {
        why = "basis descriptor is null or empty";
        return PFK_ERR_INVALID;
    }
    long long nb = 0, np = 0;
    for (int s = 0; s < b->nshell; ++s) {
        if (b->L[s] < 0) {
            why = "negative angular momentum";
            return PFK_ERR_INVALID;
        }
        if (b->L[s] > 3) {
            why = "angular momentum above f (L=3) is not supported";
            return PFK_ERR_UNSUPPORTED;
        }
        if (b->nprim[s] <= 0 || b->nprim[s] > 64) {
            why = "primitive count per shell must be 1..64";
            return PFK_ERR_INVALID;
        }
        for (int d = 0; d < 3; ++d)
            if (!std::isfinite(b->center[3 * s + d])) {
                why = "non-finite shell centre";
                return PFK_ERR_INVALID;
            }
        nb += ncart(b->L[s]);
        np += b->nprim[s];
    }
    for (long long i = 0; i < np; ++i)
        if (!(b->expo[i] > 0.0) || !std::isfinite(b->expo[i]) || !std::isfinite(b->coef[i]) || !std::isfinite(b->norm[i])) {
            why = "exponents must be positive and finite; coefficients and norms finite";
            return PFK_ERR_INVALID;
        }
    if (check_nbasis && nb >= 65536) {
        why = "more than 65535 basis functions";
        return PFK_ERR_UNSUPPORTED;
    }
    return PFK_OK;
}

// Shell pairs a <= b with primitive-pair data (src/base/types.h:631-674),
// oriented so that L(A) >= L(B).
//
// One oriented pair (A, B), L(A) >= L(B): appends its PairInfo and its
// primitive pairs (qp left at `qp`) to the vectors.  poff: first primitive
// of each shell.
void append_pair(const pfk_basis_desc *b, const std::vector<int> &poff, int A, int B, int bf_a, int bf_b, double qp,
                 std::vector<PairInfo> &pairs, std::vector<PrimPair> &prims)
{
    const double *ca = b->center + 3 * A, *cb = b->center + 3 * B;
    PairInfo pi{};
    pi.prim_off = (int)prims.size();
    pi.bf_a = bf_a;
    pi.bf_b = bf_b;
    pi.ABx = ca[0] - cb[0];
    pi.ABy = ca[1] - cb[1];
    pi.ABz = ca[2] - cb[2];
    const double R2 = pi.ABx * pi.ABx + pi.ABy * pi.ABy + pi.ABz * pi.ABz;
    for (int ia = 0; ia < b->nprim[A]; ++ia)
        for (int ib = 0; ib < b->nprim[B]; ++ib) {
            const double alpha = b->expo[poff[A] + ia], beta = b->expo[poff[B] + ib];
            const double zeta = alpha + beta, iz = 1.0 / zeta;
            PrimPair p{};
            p.zeta = zeta;
            p.inv_zeta = iz;
            p.Px = (alpha * ca[0] + beta * cb[0]) * iz;
            p.Py = (alpha * ca[1] + beta * cb[1]) * iz;
            p.Pz = (alpha * ca[2] + beta * cb[2]) * iz;
            p.PAx = p.Px - ca[0];
            p.PAy = p.Py - ca[1];
            p.PAz = p.Pz - ca[2];
            const double K = std::pow(kPi * iz, 1.5) * std::exp(-alpha * beta * iz * R2) * b->coef[poff[A] + ia] *
                             b->coef[poff[B] + ib] * b->norm[poff[A] + ia] * b->norm[poff[B] + ib];
            p.Kz = K * std::sqrt(zeta);
            p.qp = qp;
            prims.push_back(p);
        }
    pi.nprim_full = pi.nprim = (int)prims.size() - pi.prim_off;
    pairs.push_back(pi);
}

void build_pairs(pfk_ctx *ctx, const pfk_basis_desc *b)
{
    std::vector<int> poff(b->nshell + 1, 0);
    for (int s = 0; s < b->nshell; ++s) poff[s + 1] = poff[s] + b->nprim[s];
    ctx->pairs.clear();
    ctx->prims.clear();
    for (int sa = 0; sa < b->nshell; ++sa)
        for (int sb = sa; sb < b->nshell; ++sb) {
            const int A = b->L[sa] >= b->L[sb] ? sa : sb;
            const int B = A == sa ? sb : sa;
            // qp: prim_bounds sets it and orders the pair's primitives
            append_pair(b, poff, A, B, ctx->bf_off[A], ctx->bf_off[B], 0.0, ctx->pairs, ctx->prims);
            ctx->pair_pc.push_back(pair_class(b->L[A], b->L[B]));
            ctx->pair_la.push_back(b->L[A]);
            ctx->pair_lb.push_back(b->L[B]);
        }
    ctx->npairs = (int)ctx->pairs.size();
}

// Primitive Schwarz bounds (prim_bound_kernel) of the pairs build_pairs made:
// uploads the pairs, their primitives and the pair ids grouped by pair class
// (d_ids, npairs entries; cls_begin gets the class starts), computes every
// qp on the device, brings the primitives back, orders each pair's
// primitives by qp (descending), keeps in nprim those that can reach
// kPrimPairFloor with the largest qp of the basis, and uploads the result.
cudaError_t prim_bounds(pfk_ctx *h, PairInfo *d_pairs, PrimPair *d_prims, int *d_ids, std::vector<int> &cls_begin,
                        cudaStream_t st)
{
    std::vector<int> ids;
    cls_begin.assign(kPairClasses + 1, 0);
    for (int x = 0; x < kPairClasses; ++x) {
        cls_begin[x] = (int)ids.size();
        for (int p = 0; p < h->npairs; ++p)
            if (h->pair_pc[p] == x) ids.push_back(p);
    }
    cls_begin[kPairClasses] = (int)ids.size();
    const size_t np = h->prims.size();
    cudaError_t e = cudaMemcpyAsync(d_pairs, h->pairs.data(), sizeof(PairInfo) * h->npairs, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_prims, h->prims.data(), sizeof(PrimPair) * np, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_ids, ids.data(), sizeof(int) * ids.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    for (int x = 0; x < kPairClasses; ++x)
        launch_prim_bounds(x, d_ids + cls_begin[x], cls_begin[x + 1] - cls_begin[x], d_pairs, d_prims, st);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->prims.data(), d_prims, sizeof(PrimPair) * np, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    double qmax = 0.0;
    for (const PrimPair &p : h->prims) qmax = std::max(qmax, p.qp);
    for (PairInfo &pi : h->pairs) {
        PrimPair *b = h->prims.data() + pi.prim_off;
        std::stable_sort(b, b + pi.nprim_full, [](const PrimPair &x, const PrimPair &y) { return x.qp > y.qp; });
        pi.nprim = 0;
        while (pi.nprim < pi.nprim_full && b[pi.nprim].qp * qmax >= kPrimPairFloor) ++pi.nprim;
    }
    e = cudaMemcpyAsync(d_pairs, h->pairs.data(), sizeof(PairInfo) * h->npairs, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_prims, h->prims.data(), sizeof(PrimPair) * np, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

pfk_status upload_pairs(pfk_ctx *ctx)
{
    PFK_CK(ctx->d_pairs.alloc(ctx->npairs));
    PFK_CK(cudaMemcpyAsync(ctx->d_pairs.p, ctx->pairs.data(), sizeof(PairInfo) * ctx->npairs, cudaMemcpyHostToDevice,
                           ctx->stream));
    return PFK_OK;
}

// Screened shell-quartet lists for the current tol / FP32 bound.
// Releases the captured RHF builds; the next device call captures again.
void drop_graphs(pfk_ctx *ctx)
{
    for (auto &g : ctx->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    ctx->graphs.clear();
}

// Pair classes from fs on hold an f shell.  Quartet classes with one keep
// their whole list in FP64: on the ERI class microbenchmark's random shells
// the FP32 variants of those classes lose up to 1e-5 (fd|fd) and more
// (ff|ff), where the s..d classes stay within 1e-7 relative.
constexpr int kFirstFPairClass = 6;

pfk_status build_lists(pfk_ctx *ctx)
{
    const double bound = ctx->precision == PFK_PREC_MIXED ? ctx->fp32_bound : 0.0;
    int maxn = 1;
    for (int x = 0; x < kPairClasses; ++x) maxn = std::max(maxn, (int)ctx->cls_ids[x].size());
    DevBuf<long long> cnt_hi, cnt_lo, off_hi, off_lo, work_hi, work_lo;
    PFK_CK(work_hi.alloc(maxn));
    PFK_CK(work_lo.alloc(maxn));
    PFK_CK(cnt_hi.alloc(maxn));
    PFK_CK(cnt_lo.alloc(maxn));
    PFK_CK(off_hi.alloc(maxn));
    PFK_CK(off_lo.alloc(maxn));
    size_t tmp_bytes = 0;
    PFK_CK(exclusive_scan(cnt_hi.p, off_hi.p, maxn, nullptr, tmp_bytes, ctx->stream));
    DevBuf<char> tmp;
    PFK_CK(tmp.alloc(tmp_bytes + 16));

    // pass 1: counts
    long long total = 0;
    for (int x = 0; x < kPairClasses; ++x)
        for (int y = 0; y <= x; ++y) {
            const int cls = quartet_class(x, y);
            const int nX = (int)ctx->cls_ids[x].size(), nY = (int)ctx->cls_ids[y].size();
            ctx->q_cnt[cls] = ctx->q32_cnt[cls] = 0;
            ctx->prim_cnt[cls] = ctx->prim32_cnt[cls] = 0;
            if (nX == 0 || nY == 0) continue;
            PFK_CK(count_quartets(ctx->d_cls_q[x].p, nX, ctx->d_cls_q[y].p, nY, x == y, ctx->tol,
                                  x >= kFirstFPairClass ? 0.0 : bound, cnt_hi.p, cnt_lo.p, ctx->stream));
            size_t tb = tmp_bytes;
            PFK_CK(exclusive_scan(cnt_hi.p, off_hi.p, nX, tmp.p, tb, ctx->stream));
            tb = tmp_bytes;
            PFK_CK(exclusive_scan(cnt_lo.p, off_lo.p, nX, tmp.p, tb, ctx->stream));
            long long h[4];
            PFK_CK(cudaMemcpyAsync(&h[0], off_hi.p + nX - 1, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
            PFK_CK(cudaMemcpyAsync(&h[1], cnt_hi.p + nX - 1, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
            PFK_CK(cudaMemcpyAsync(&h[2], off_lo.p + nX - 1, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
            PFK_CK(cudaMemcpyAsync(&h[3], cnt_lo.p + nX - 1, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
            PFK_CK(cudaStreamSynchronize(ctx->stream));
            ctx->q_cnt[cls] = h[0] + h[1];
            ctx->q32_cnt[cls] = h[2] + h[3];
            total += ctx->q_cnt[cls] + ctx->q32_cnt[cls];
        }
    long long pos = 0;
    for (int c = 0; c < kQuartetClasses; ++c) {
        ctx->q_off[c] = pos;
        pos += ctx->q_cnt[c];
        ctx->q32_off[c] = pos;
        pos += ctx->q32_cnt[c];
    }
    PFK_CK(ctx->d_quart.alloc((size_t)std::max(total, 1LL)));
    // pass 2: fill
    for (int x = 0; x < kPairClasses; ++x)
        for (int y = 0; y <= x; ++y) {
            const int cls = quartet_class(x, y);
            const int nX = (int)ctx->cls_ids[x].size(), nY = (int)ctx->cls_ids[y].size();
            if (nX == 0 || nY == 0 || ctx->q_cnt[cls] + ctx->q32_cnt[cls] == 0) continue;
            PFK_CK(count_quartets(ctx->d_cls_q[x].p, nX, ctx->d_cls_q[y].p, nY, x == y, ctx->tol,
                                  x >= kFirstFPairClass ? 0.0 : bound, cnt_hi.p, cnt_lo.p, ctx->stream));
            size_t tb = tmp_bytes;
            PFK_CK(exclusive_scan(cnt_hi.p, off_hi.p, nX, tmp.p, tb, ctx->stream));
            tb = tmp_bytes;
            PFK_CK(exclusive_scan(cnt_lo.p, off_lo.p, nX, tmp.p, tb, ctx->stream));
            PFK_CK(fill_quartets(ctx->d_cls_ids[x].p, nX, ctx->d_cls_ids[y].p, x == y, off_hi.p, cnt_hi.p, off_lo.p,
                                 cnt_lo.p, ctx->d_quart.p + ctx->q_off[cls], ctx->d_quart.p + ctx->q32_off[cls],
                                 ctx->stream));
            PFK_CK(bra_work(ctx->d_cls_ids[x].p, nX, x == y, cnt_hi.p, cnt_lo.p, ctx->d_cls_kpref[y].p,
                            ctx->d_pairs.p, work_hi.p, work_lo.p, ctx->stream));
            std::vector<long long> h(2 * (size_t)nX);
            PFK_CK(cudaMemcpyAsync(h.data(), work_hi.p, sizeof(long long) * nX, cudaMemcpyDeviceToHost, ctx->stream));
            PFK_CK(cudaMemcpyAsync(h.data() + nX, work_lo.p, sizeof(long long) * nX, cudaMemcpyDeviceToHost, ctx->stream));
            PFK_CK(cudaStreamSynchronize(ctx->stream));
            long long w = 0, w32 = 0;
            for (size_t a = 0; a < h.size(); ++a) w += h[a];
            for (int a = 0; a < nX; ++a) w32 += h[(size_t)nX + a];
            ctx->prim_cnt[cls] = w;
            ctx->prim32_cnt[cls] = w32;
        }
    // order each list by its primitive loop lengths (stable: bra-major within a key)
    long long maxseg = 1;
    for (int c = 0; c < kQuartetClasses; ++c) maxseg = std::max(maxseg, std::max(ctx->q_cnt[c], ctx->q32_cnt[c]));
    {
        DevBuf<unsigned> ka, kb;
        DevBuf<uint2> vb;
        PFK_CK(ka.alloc(maxseg));
        PFK_CK(kb.alloc(maxseg));
        PFK_CK(vb.alloc(maxseg));
        size_t sort_bytes = 0;
        PFK_CK(sort_quartets(ctx->d_quart.p, maxseg, ctx->d_pairs.p, ka.p, kb.p, vb.p, nullptr, sort_bytes, ctx->stream));
        DevBuf<char> st;
        PFK_CK(st.alloc(sort_bytes + 16));
        for (int c = 0; c < kQuartetClasses; ++c) {
            size_t b1 = sort_bytes, b2 = sort_bytes;
            PFK_CK(sort_quartets(ctx->d_quart.p + ctx->q_off[c], ctx->q_cnt[c], ctx->d_pairs.p, ka.p, kb.p, vb.p, st.p,
                                 b1, ctx->stream));
            PFK_CK(sort_quartets(ctx->d_quart.p + ctx->q32_off[c], ctx->q32_cnt[c], ctx->d_pairs.p, ka.p, kb.p, vb.p,
                                 st.p, b2, ctx->stream));
        }
        PFK_CK(cudaStreamSynchronize(ctx->stream));
    }
    PFK_CK(cudaStreamSynchronize(ctx->stream));
    drop_graphs(ctx);   // captured builds refer to the old lists
    return PFK_OK;
}

pfk_status schwarz_and_sort(pfk_ctx *ctx)
{
    const int nb = ctx->nb;
    PFK_CK(ctx->d_Q.alloc((size_t)nb * nb));
    PFK_CK(cudaMemsetAsync(ctx->d_Q.p, 0, sizeof(double) * nb * nb, ctx->stream));
    std::vector<int> ids[kPairClasses];
    for (int p = 0; p < ctx->npairs; ++p) ids[ctx->pair_pc[p]].push_back(p);
    DevBuf<int> d_ids[kPairClasses];
    for (int x = 0; x < kPairClasses; ++x) {
        if (ids[x].empty()) continue;
        PFK_CK(d_ids[x].alloc(ids[x].size()));
        PFK_CK(cudaMemcpyAsync(d_ids[x].p, ids[x].data(), sizeof(int) * ids[x].size(), cudaMemcpyHostToDevice,
                               ctx->stream));
        launch_schwarz(x, d_ids[x].p, (int)ids[x].size(), ctx->d_pairs.p, ctx->d_prims.p, ctx->d_Q.p, nb, ctx->stream);
        PFK_CK(cudaGetLastError());
    }
    ctx->Q.assign((size_t)nb * nb, 0.0);
    PFK_CK(cudaMemcpyAsync(ctx->Q.data(), ctx->d_Q.p, sizeof(double) * nb * nb, cudaMemcpyDeviceToHost, ctx->stream));
    PFK_CK(cudaStreamSynchronize(ctx->stream));
    for (int x = 0; x < kPairClasses; ++x) ids[x].clear();
    // per-pair bound over components
    for (int p = 0; p < ctx->npairs; ++p) {
        PairInfo &pi = ctx->pairs[p];
        const int na = ncart(ctx->pair_la[p]), nbb = ncart(ctx->pair_lb[p]);
        double qmax = 0.0, qmin = INFINITY;
        for (int a = 0; a < na; ++a)
            for (int c = 0; c < nbb; ++c) {
                const double q = ctx->Q[(size_t)(pi.bf_a + a) * nb + pi.bf_b + c];
                qmax = std::max(qmax, q);
                qmin = std::min(qmin, q);
            }
        pi.qmax = qmax;
        pi.qmin = qmin;
    }
    pfk_status s = upload_pairs(ctx);
    if (s != PFK_OK) return s;
    // per-class lists sorted by qmax, descending (ties by pair index)
    for (int p = 0; p < ctx->npairs; ++p) ids[ctx->pair_pc[p]].push_back(p);
    for (int x = 0; x < kPairClasses; ++x) {
        auto &v = ids[x];
        std::stable_sort(v.begin(), v.end(), [&](int a, int b) { return ctx->pairs[a].qmax > ctx->pairs[b].qmax; });
        ctx->cls_ids[x] = v;
        std::vector<double> q(v.size());
        for (size_t i = 0; i < v.size(); ++i) q[i] = ctx->pairs[v[i]].qmax;
        if (v.empty()) continue;
        PFK_CK(ctx->d_cls_ids[x].alloc(v.size()));
        PFK_CK(ctx->d_cls_q[x].alloc(v.size()));
        PFK_CK(cudaMemcpyAsync(ctx->d_cls_ids[x].p, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice, ctx->stream));
        PFK_CK(cudaMemcpyAsync(ctx->d_cls_q[x].p, q.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice, ctx->stream));
        std::vector<long long> kp(v.size() + 1, 0);
        for (size_t i = 0; i < v.size(); ++i) kp[i + 1] = kp[i] + ctx->pairs[v[i]].nprim_full;
        PFK_CK(ctx->d_cls_kpref[x].alloc(kp.size()));
        PFK_CK(cudaMemcpyAsync(ctx->d_cls_kpref[x].p, kp.data(), sizeof(long long) * kp.size(), cudaMemcpyHostToDevice,
                               ctx->stream));
        PFK_CK(cudaStreamSynchronize(ctx->stream));
    }
    return PFK_OK;
}

// Kernel choice of class c.  engine os: the Obara-Saika kernel for the
// classes that have one (L <= kOSMaxL, where the reference's per-quartet auto
// choice is OS for every component quartet), Rys for the rest; engine rys:
// Rys; engine auto: the per-class choice of pfk_autotune (the os rule until
// it has run).
int class_flags(const pfk_ctx *ctx, int c)
{
    if (ctx->engine == PFK_ENGINE_RYS) return 0;
    if (ctx->engine == PFK_ENGINE_AUTO) return ctx->auto_flags[c];
    return quartet_class_L(c) <= kOSMaxL ? kLaunchOS : 0;
}

// Cartesian component quartets of class c (the launch-order cost weight).
static int class_components(int c)
{
    int x = 0;
    while ((x + 1) * (x + 2) / 2 <= c) ++x;
    const int y = c - x * (x + 1) / 2;
    return ncart(pc_la(x)) * ncart(pc_lb(x)) * ncart(pc_la(y)) * ncart(pc_lb(y));
}

// Launch every class kernel over the screened lists.  Jacc/K accumulators are
// zeroed first.  eri_out selects the dense-tensor mode.
pfk_status run_classes(pfk_ctx *ctx, const double *Pj, const double *Pk0, const double *Pk1, int nk, FxWord *Jacc,
                       FxWord *K0, FxWord *K1, double *eri_out, cudaStream_t st, bool timed)
{
    const size_t nb2 = (size_t)ctx->nb * ctx->nb;
    if (!eri_out) {
        PFK_CK(cudaMemsetAsync(Jacc, 0, sizeof(FxWord) * 2 * nb2, st));
        if (K0) PFK_CK(cudaMemsetAsync(K0, 0, sizeof(FxWord) * 2 * nb2, st));
        if (K1) PFK_CK(cudaMemsetAsync(K1, 0, sizeof(FxWord) * 2 * nb2, st));
    }
    JKArgs a{};
    if (ctx->dscreen_tol > 0.0 && !eri_out) {
        PFK_CK(shell_block_max(ctx->nshell, ctx->d_shell_bf.p, ctx->d_shell_nbf.p, Pj, Pk0 != Pj ? Pk0 : nullptr, Pk1,
                               ctx->nb, ctx->d_Dsh.p, st));
        a.Dsh = ctx->d_Dsh.p;
        a.dtol = ctx->dscreen_tol;
    }
    a.pairs = ctx->d_pairs.p;
    a.prims = ctx->d_prims.p;
    a.Qao = ctx->d_Q.p;
    a.Pj = Pj;
    a.Pk0 = Pk0;
    a.Pk1 = Pk1;
    a.Jacc = Jacc;
    a.Kacc0 = K0;
    a.Kacc1 = K1;
    a.eri_out = eri_out;
    a.tol = ctx->tol;
    a.ptol = ctx->prim_tol;
    a.nb = ctx->nb;
    a.qstride = ctx->shard_n;
    a.qoffset = ctx->shard_rank;
    auto local = [&](long long n) -> long long {
        return n > ctx->shard_rank ? (n - ctx->shard_rank + ctx->shard_n - 1) / ctx->shard_n : 0;
    };
    cudaEvent_t ev[2] = {nullptr, nullptr};
    if (timed) {
        PFK_CK(cudaEventCreate(&ev[0]));
        PFK_CK(cudaEventCreate(&ev[1]));
    }
    // lanes: the classes go, largest estimated cost first, to the lane with
    // the least work so far; a per-class timed pass stays on one stream
    const int nlanes = timed ? 1 : ctx->lanes;
    cudaStream_t lane_st[kMaxLanes] = {st};
    if (nlanes > 1) {
        PFK_CK(cudaEventRecord(ctx->fork_ev, st));
        for (int i = 1; i < nlanes; ++i) {
            lane_st[i] = ctx->side[i - 1];
            PFK_CK(cudaStreamWaitEvent(lane_st[i], ctx->fork_ev, 0));
        }
    }
    int order[kQuartetClasses];
    double cost[kQuartetClasses];
    for (int c = 0; c < kQuartetClasses; ++c) {
        order[c] = c;
        cost[c] = (double)ctx->prim_cnt[c] * class_components(c);
    }
    if (nlanes > 1)
        std::stable_sort(order, order + kQuartetClasses, [&](int x, int y) { return cost[x] > cost[y]; });
    double load[kMaxLanes] = {};
    for (int oc = 0; oc < kQuartetClasses; ++oc) {
        const int c = order[oc];
        const long long nh = local(ctx->q_cnt[c]), nl = local(ctx->q32_cnt[c]);
        if (nh + nl == 0) continue;
        if (timed) PFK_CK(cudaEventRecord(ev[0], st));
        const int os = class_flags(ctx, c);
        const int fp32 = ctx->precision == PFK_PREC_MIXED ? kLaunchFP32 : 0;
        int ln = 0;
        for (int i = 1; i < nlanes; ++i)
            if (load[i] < load[ln]) ln = i;
        load[ln] += cost[c];
        if (nh) ctx->launch[c](ctx->d_quart.p + ctx->q_off[c], nh, a, nk, os, lane_st[ln]);
        if (nl) ctx->launch[c](ctx->d_quart.p + ctx->q32_off[c], nl, a, nk, os | fp32, lane_st[ln]);
        PFK_CK(cudaGetLastError());
        if (timed) {
            PFK_CK(cudaEventRecord(ev[1], st));
            PFK_CK(cudaEventSynchronize(ev[1]));
            float ms = 0.f;
            PFK_CK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
            ctx->class_ms[c] = ms;
        }
    }
    if (timed) {
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
    }
    for (int i = 1; i < nlanes; ++i) {
        PFK_CK(cudaEventRecord(ctx->join_ev[i - 1], lane_st[i]));
        PFK_CK(cudaStreamWaitEvent(st, ctx->join_ev[i - 1], 0));
    }
    return PFK_OK;
}

pfk_status rhf_sequence(pfk_ctx *ctx, const double *dP, double *dG, cudaStream_t st)
{
    pfk_status s = run_classes(ctx, dP, dP, nullptr, 1, ctx->d_J.p, ctx->d_K0.p, nullptr, nullptr, st, false);
    if (s != PFK_OK) return s;
    PFK_CK(combine(ctx->d_J.p, ctx->d_K0.p, 1.0, -0.5, dG, ctx->nb, st));
    return PFK_OK;
}

pfk_status ensure_work(pfk_ctx *ctx)
{
    const size_t nb2 = (size_t)ctx->nb * ctx->nb;
    if (ctx->d_J.p) return PFK_OK;
    for (DevBuf<double> *b : {&ctx->d_P, &ctx->d_Pb, &ctx->d_Pt, &ctx->d_G, &ctx->d_Gb})
        PFK_CK(b->alloc(nb2));
    for (DevBuf<FxWord> *b : {&ctx->d_J, &ctx->d_K0, &ctx->d_K1})
        PFK_CK(b->alloc(2 * nb2));
    return PFK_OK;
}

// max |P(i,j) - P(j,i)| against 1e-10 max(1, max |P|), and every element
// finite.  The transposed pairs are compared tile by tile (32 x 32), so both
// tiles stay in cache: a row-against-column sweep of an 800 x 800 matrix
// missed the cache on every transposed load and took milliseconds.
pfk_status check_symmetric(pfk_ctx *ctx, const double *P)
{
    const int nb = ctx->nb;
    constexpr int kTile = 32;
    double amax = 0.0, dmax = 0.0, nonfinite = 0.0;   // v - v: 0 if v is finite, NaN otherwise
    for (size_t k = 0; k < (size_t)nb * nb; ++k) {
        amax = std::max(amax, std::fabs(P[k]));
        nonfinite += P[k] - P[k];
    }
    for (int i0 = 0; i0 < nb; i0 += kTile)
        for (int j0 = i0; j0 < nb; j0 += kTile) {
            const int i1 = std::min(i0 + kTile, nb), j1 = std::min(j0 + kTile, nb);
            for (int i = i0; i < i1; ++i)
                for (int j = std::max(j0, i + 1); j < j1; ++j)
                    dmax = std::max(dmax, std::fabs(P[(size_t)i * nb + j] - P[(size_t)j * nb + i]));
        }
    if (nonfinite != 0.0 || !(dmax <= 1e-10 * std::max(1.0, amax)))
        return ctx->fail(PFK_ERR_INVALID, "density matrix is not symmetric (or not finite)");
    return PFK_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

pfk_status pfk_create(const pfk_basis_desc *basis, int device, pfk_ctx **out)
{
    if (!out) {
        g_last_error = "pfk_create: out is null";
        return PFK_ERR_INVALID;
    }
    *out = nullptr;
    std::string why;
    pfk_status vs = validate(basis, why);
    if (vs != PFK_OK) {
        g_last_error = "pfk_create: " + why;
        return vs;
    }
    pfk_ctx *ctx = nullptr;
    try {
        ctx = new pfk_ctx();
    } catch (const std::bad_alloc &) {
        g_last_error = "pfk_create: host allocation failed";
        return PFK_ERR_NOMEM;
    }
    auto bail = [&](pfk_status s) {
        g_last_error = ctx->err;
        pfk_destroy(ctx);
        return s;
    };
    try {
        ctx->device = device;
        cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) return bail(ctx->cuda_fail("cudaSetDevice", e));
        e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return bail(ctx->cuda_fail("cudaStreamCreate", e));
        e = cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return bail(ctx->cuda_fail("cudaEventCreate", e));
        for (int i = 0; i < kMaxLanes - 1; ++i) {
            e = cudaStreamCreateWithFlags(&ctx->side[i], cudaStreamNonBlocking);
            if (e != cudaSuccess) return bail(ctx->cuda_fail("cudaStreamCreate", e));
            e = cudaEventCreateWithFlags(&ctx->join_ev[i], cudaEventDisableTiming);
            if (e != cudaSuccess) return bail(ctx->cuda_fail("cudaEventCreate", e));
        }
        ctx->nshell = basis->nshell;
        ctx->L.assign(basis->L, basis->L + basis->nshell);
        ctx->bf_off.resize(basis->nshell);
        int nb = 0;
        for (int s = 0; s < basis->nshell; ++s) {
            ctx->bf_off[s] = nb;
            nb += ncart(basis->L[s]);
        }
        ctx->nb = nb;
        build_pairs(ctx, basis);
        e = ctx->d_prims.alloc(ctx->prims.size());
        if (e != cudaSuccess) return bail(ctx->cuda_fail("cudaMalloc(prims)", e));
        e = cudaMemcpyAsync(ctx->d_prims.p, ctx->prims.data(), sizeof(PrimPair) * ctx->prims.size(),
                            cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return bail(ctx->cuda_fail("cudaMemcpy(prims)", e));
        e = ctx->d_pair_la.alloc(ctx->npairs);
        if (e == cudaSuccess) e = ctx->d_pair_lb.alloc(ctx->npairs);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ctx->d_pair_la.p, ctx->pair_la.data(), sizeof(int) * ctx->npairs, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ctx->d_pair_lb.p, ctx->pair_lb.data(), sizeof(int) * ctx->npairs, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return bail(ctx->cuda_fail("pair tables", e));
        pfk_status s = upload_pairs(ctx);
        if (s != PFK_OK) return bail(s);
        {
            DevBuf<int> ids;
            std::vector<int> cls_begin;
            e = ids.alloc(std::max(ctx->npairs, 1));
            if (e == cudaSuccess) e = prim_bounds(ctx, ctx->d_pairs.p, ctx->d_prims.p, ids.p, cls_begin, ctx->stream);
            if (e != cudaSuccess) return bail(ctx->cuda_fail("primitive bounds", e));
        }
        for (int c = 0; c < kQuartetClasses; ++c) {
            if (!g_class_launchers[c]) {
                ctx->err = "class kernel table incomplete (library built without every class unit)";
                return bail(PFK_ERR_STATE);
            }
            ctx->launch[c] = g_class_launchers[c];
            ctx->auto_flags[c] = quartet_class_L(c) <= kOSMaxL ? kLaunchOS : 0;
        }
        JKArgs none{};
        for (int c = 0; c < kQuartetClasses; ++c) ctx->launch[c](nullptr, -1, none, 1, 0, ctx->stream);
        e = cudaGetLastError();
        if (e != cudaSuccess) return bail(ctx->cuda_fail("kernel configuration", e));
        s = schwarz_and_sort(ctx);
        if (s != PFK_OK) return bail(s);
        s = build_lists(ctx);
        if (s != PFK_OK) return bail(s);
        s = ensure_work(ctx);
        if (s != PFK_OK) return bail(s);
    } catch (const std::bad_alloc &) {
        ctx->err = "host allocation failed";
        return bail(PFK_ERR_NOMEM);
    }
    *out = ctx;
    return PFK_OK;
}

pfk_status pfk_destroy(pfk_ctx *ctx)
{
    if (!ctx) return PFK_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto &g : ctx->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    ctx->d_pairs.release();
    ctx->d_prims.release();
    ctx->d_pair_la.release();
    ctx->d_pair_lb.release();
    ctx->d_Q.release();
    for (int x = 0; x < kPairClasses; ++x) {
        ctx->d_cls_ids[x].release();
        ctx->d_cls_q[x].release();
        ctx->d_cls_kpref[x].release();
    }
    ctx->d_quart.release();
    ctx->d_shell_bf.release();
    ctx->d_shell_nbf.release();
    ctx->d_Dsh.release();
    for (DevBuf<double> *b : {&ctx->d_P, &ctx->d_Pb, &ctx->d_Pt, &ctx->d_G, &ctx->d_Gb}) b->release();
    for (DevBuf<FxWord> *b : {&ctx->d_J, &ctx->d_K0, &ctx->d_K1}) b->release();
    for (int i = 0; i < kMaxLanes - 1; ++i) {
        if (ctx->side[i]) cudaStreamDestroy(ctx->side[i]);
        if (ctx->join_ev[i]) cudaEventDestroy(ctx->join_ev[i]);
    }
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    if (ctx->blas) cublasDestroy(ctx->blas);
    for (int k = 0; k < 2; ++k) {
        if (ctx->pin[k]) cudaFreeHost(ctx->pin[k]);
        if (ctx->pin_ev[k]) cudaEventDestroy(ctx->pin_ev[k]);
    }
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return PFK_OK;
}

int pfk_nbasis(const pfk_ctx *ctx) { return ctx ? ctx->nb : 0; }

const char *pfk_last_error(const pfk_ctx *ctx) { return ctx ? ctx->err.c_str() : g_last_error.c_str(); }

pfk_status pfk_set_options(pfk_ctx *ctx, double tol_eri, int engine, int precision, double fp32_bound)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!(tol_eri >= 0.0) || !std::isfinite(tol_eri)) return ctx->fail(PFK_ERR_INVALID, "tol_eri must be finite and >= 0");
    if (engine < PFK_ENGINE_OS || engine > PFK_ENGINE_AUTO) return ctx->fail(PFK_ERR_INVALID, "unknown engine");
    if (precision != PFK_PREC_FP64 && precision != PFK_PREC_MIXED) return ctx->fail(PFK_ERR_INVALID, "unknown precision");
    if (precision == PFK_PREC_MIXED && !(fp32_bound > 0.0 && std::isfinite(fp32_bound)))
        return ctx->fail(PFK_ERR_INVALID, "fp32_bound must be positive");
    cudaSetDevice(ctx->device);
    const bool rebuild = tol_eri != ctx->tol || precision != ctx->precision ||
                         (precision == PFK_PREC_MIXED && fp32_bound != ctx->fp32_bound);
    if (engine != ctx->engine) drop_graphs(ctx);   // captured builds hold the old engine's kernels
    ctx->tol = tol_eri;
    ctx->engine = engine;
    ctx->precision = precision;
    if (precision == PFK_PREC_MIXED) ctx->fp32_bound = fp32_bound;
    return rebuild ? build_lists(ctx) : PFK_OK;
}

pfk_status pfk_schwarz(pfk_ctx *ctx, double *Q)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!Q) return ctx->fail(PFK_ERR_INVALID, "Q is null");
    std::memcpy(Q, ctx->Q.data(), sizeof(double) * ctx->Q.size());
    return PFK_OK;
}

static pfk_status run_census(pfk_ctx *ctx, long long *n_ao, uint64_t *digest, long long *n_shell, int *out, long long cap)
{
    cudaSetDevice(ctx->device);
    DevBuf<unsigned long long> cnt;
    PFK_CK(cnt.alloc(3));
    PFK_CK(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long) * 3, ctx->stream));
    DevBuf<int> d_out;
    if (out && cap > 0) PFK_CK(d_out.alloc((size_t)cap * 4));
    long long nsh = 0;
    for (int c = 0; c < kQuartetClasses; ++c) {
        const long long n = ctx->q_cnt[c] + ctx->q32_cnt[c];
        nsh += n;
        if (n == 0) continue;
        PFK_CK(census(ctx->d_quart.p + ctx->q_off[c], n, ctx->d_pairs.p, ctx->d_pair_la.p, ctx->d_pair_lb.p,
                      ctx->d_Q.p, ctx->nb, ctx->tol, cnt.p, d_out.p, cap, ctx->stream));
    }
    unsigned long long h[3];
    PFK_CK(cudaMemcpyAsync(h, cnt.p, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    PFK_CK(cudaStreamSynchronize(ctx->stream));
    if (out && cap > 0) {
        const long long m = std::min<long long>(cap, (long long)h[2]);
        PFK_CK(cudaMemcpy(out, d_out.p, sizeof(int) * 4 * m, cudaMemcpyDeviceToHost));
    }
    if (n_ao) *n_ao = (long long)h[0];
    if (digest) *digest = h[1];
    if (n_shell) *n_shell = nsh;
    return PFK_OK;
}

pfk_status pfk_quartet_count(pfk_ctx *ctx, long long *n_ao_quartets, uint64_t *digest, long long *n_shell_quartets)
{
    if (!ctx) return PFK_ERR_STATE;
    return run_census(ctx, n_ao_quartets, digest, n_shell_quartets, nullptr, 0);
}

pfk_status pfk_quartet_list(pfk_ctx *ctx, int *out, long long cap, long long *n)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!out || cap < 0) return ctx->fail(PFK_ERR_INVALID, "output buffer is null");
    return run_census(ctx, n, nullptr, nullptr, out, cap);
}

// Captured-graph replay of the RHF build for a (dP, dG, stream) triple.
static pfk_status rhf_graph(pfk_ctx *ctx, const double *dP, double *dG, cudaStream_t st)
{
    GraphEntry *ge = nullptr;
    for (auto &g : ctx->graphs)
        if (g.in == dP && g.out == dG && g.stream == st) ge = &g;
    if (!ge) {
        GraphEntry g{dP, dG, st};
        PFK_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        pfk_status s = rhf_sequence(ctx, dP, dG, st);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &graph);
        if (s != PFK_OK) {
            if (graph) cudaGraphDestroy(graph);
            return s;
        }
        if (e != cudaSuccess) return ctx->cuda_fail("cudaStreamEndCapture", e);
        g.graph = graph;
        e = cudaGraphInstantiate(&g.exec, graph, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(graph);
            return ctx->cuda_fail("cudaGraphInstantiate", e);
        }
        ctx->graphs.push_back(g);
        ge = &ctx->graphs.back();
    }
    PFK_CK(cudaGraphLaunch(ge->exec, st));
    return PFK_OK;
}

pfk_status pfk_fock_rhf(pfk_ctx *ctx, const double *P, double *G)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!P || !G) return ctx->fail(PFK_ERR_INVALID, "null matrix");
    pfk_status s = check_symmetric(ctx, P);
    if (s != PFK_OK) return s;
    cudaSetDevice(ctx->device);
    const size_t bytes = sizeof(double) * ctx->nb * ctx->nb;
    PFK_CK(cudaMemcpyAsync(ctx->d_P.p, P, bytes, cudaMemcpyHostToDevice, ctx->stream));
    s = rhf_graph(ctx, ctx->d_P.p, ctx->d_G.p, ctx->stream);
    if (s != PFK_OK) return s;
    PFK_CK(cudaMemcpyAsync(G, ctx->d_G.p, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    PFK_CK(cudaStreamSynchronize(ctx->stream));
    return PFK_OK;
}

pfk_status pfk_fock_rhf_device(pfk_ctx *ctx, const double *dP, double *dG, void *stream)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!dP || !dG) return ctx->fail(PFK_ERR_INVALID, "null matrix");
    cudaSetDevice(ctx->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    return rhf_graph(ctx, dP, dG, st);
}

pfk_status pfk_fock_uhf(pfk_ctx *ctx, const double *Pa, const double *Pb, double *Ga, double *Gb)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!Pa || !Pb || !Ga || !Gb) return ctx->fail(PFK_ERR_INVALID, "null matrix");
    pfk_status s = check_symmetric(ctx, Pa);
    if (s == PFK_OK) s = check_symmetric(ctx, Pb);
    if (s != PFK_OK) return s;
    cudaSetDevice(ctx->device);
    const size_t nb2 = (size_t)ctx->nb * ctx->nb, bytes = sizeof(double) * nb2;
    cudaStream_t st = ctx->stream;
    PFK_CK(cudaMemcpyAsync(ctx->d_P.p, Pa, bytes, cudaMemcpyHostToDevice, st));
    PFK_CK(cudaMemcpyAsync(ctx->d_Pb.p, Pb, bytes, cudaMemcpyHostToDevice, st));
    PFK_CK(add(ctx->d_P.p, ctx->d_Pb.p, ctx->d_Pt.p, (long long)nb2, st));
    s = run_classes(ctx, ctx->d_Pt.p, ctx->d_P.p, ctx->d_Pb.p, 2, ctx->d_J.p, ctx->d_K0.p, ctx->d_K1.p, nullptr, st, false);
    if (s != PFK_OK) return s;
    PFK_CK(combine(ctx->d_J.p, ctx->d_K0.p, 1.0, -1.0, ctx->d_G.p, ctx->nb, st));
    PFK_CK(combine(ctx->d_J.p, ctx->d_K1.p, 1.0, -1.0, ctx->d_Gb.p, ctx->nb, st));
    PFK_CK(cudaMemcpyAsync(Ga, ctx->d_G.p, bytes, cudaMemcpyDeviceToHost, st));
    PFK_CK(cudaMemcpyAsync(Gb, ctx->d_Gb.p, bytes, cudaMemcpyDeviceToHost, st));
    PFK_CK(cudaStreamSynchronize(st));
    return PFK_OK;
}

pfk_status pfk_jk(pfk_ctx *ctx, const double *P, const double *Pk, double *J, double *K, double k_scale)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!P || !J) return ctx->fail(PFK_ERR_INVALID, "null matrix");
    if (!Pk) Pk = P;
    pfk_status s = check_symmetric(ctx, P);
    if (s == PFK_OK && Pk != P) s = check_symmetric(ctx, Pk);
    if (s != PFK_OK) return s;
    cudaSetDevice(ctx->device);
    const size_t nb2 = (size_t)ctx->nb * ctx->nb, bytes = sizeof(double) * nb2;
    cudaStream_t st = ctx->stream;
    PFK_CK(cudaMemcpyAsync(ctx->d_P.p, P, bytes, cudaMemcpyHostToDevice, st));
    const double *dPk = ctx->d_P.p;
    if (Pk != P) {
        PFK_CK(cudaMemcpyAsync(ctx->d_Pb.p, Pk, bytes, cudaMemcpyHostToDevice, st));
        dPk = ctx->d_Pb.p;
    }
    s = run_classes(ctx, ctx->d_P.p, dPk, nullptr, 1, ctx->d_J.p, K ? ctx->d_K0.p : nullptr, nullptr, nullptr, st, false);
    if (s != PFK_OK) return s;
    PFK_CK(combine(ctx->d_J.p, nullptr, 1.0, 0.0, ctx->d_G.p, ctx->nb, st));
    PFK_CK(cudaMemcpyAsync(J, ctx->d_G.p, bytes, cudaMemcpyDeviceToHost, st));
    if (K) {
        PFK_CK(combine(nullptr, ctx->d_K0.p, 0.0, k_scale, ctx->d_Gb.p, ctx->nb, st));
        PFK_CK(cudaMemcpyAsync(K, ctx->d_Gb.p, bytes, cudaMemcpyDeviceToHost, st));
    }
    PFK_CK(cudaStreamSynchronize(st));
    return PFK_OK;
}

pfk_status pfk_eri_tensor(pfk_ctx *ctx, double *eri)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!eri) return ctx->fail(PFK_ERR_INVALID, "eri is null");
    if (ctx->nb > 180) return ctx->fail(PFK_ERR_UNSUPPORTED, "dense tensor limited to 180 basis functions (8.4 GB)");
    cudaSetDevice(ctx->device);
    const size_t n4 = (size_t)ctx->nb * ctx->nb * ctx->nb * ctx->nb;
    DevBuf<double> d;
    PFK_CK(d.alloc(n4));
    PFK_CK(cudaMemsetAsync(d.p, 0, sizeof(double) * n4, ctx->stream));
    pfk_status s = run_classes(ctx, ctx->d_P.p, ctx->d_P.p, nullptr, 1, ctx->d_J.p, nullptr, nullptr, d.p, ctx->stream, false);
    if (s != PFK_OK) return s;
    PFK_CK(cudaMemcpyAsync(eri, d.p, sizeof(double) * n4, cudaMemcpyDeviceToHost, ctx->stream));
    PFK_CK(cudaStreamSynchronize(ctx->stream));
    return PFK_OK;
}

// AO -> MO transform of the stored tensor (transform_eri,
// src/post_hf/integrals.cpp:63-134): the dense AO tensor from the class
// kernels' tensor mode, then the four quarter transforms as FP64 GEMMs on
// the device.  Row-major tensors; the C_k are nb x n_k column-major.
//   T1[i][nls]  = sum_m C1(m,i) E[m][nls]     one GEMM, (nb^3 x nb)(nb x n1)
//   T2[i][a][ls] = sum_n C2(n,a) T1[i][n][ls] n1 GEMMs, (nb^2 x nb)(nb x n2)
//   T3[ia][j][s] = sum_l C3(l,j) T2[ia][l][s] n1 n2 GEMMs, (nb x nb)(nb x n3)
//   out[iaj][b]  = sum_s T3[iaj][s] C4(s,b)  one GEMM, (n4 x nb)(nb x n1 n2 n3)
// MP2 sums over an (ov|ov) block O[i][a][j][b] (dimensions n1 n2 n3 n4) in
// device memory, with D = e1_i + e2_j - e1_{n1+a} - e2_{n3+b} (e1 and e2 the
// orbital energies of the two spins, occupied first):
//   kMp2R    O (2 O - O_ibja) / D       RMP2 (run_rmp2, src/post_hf/mp2.cpp:
//                                       25-35; mp2_gradient.cpp:216-230)
//   kMp2Same (O - O_ibja)^2 / (4 D)     UMP2 same spin (mp2.cpp:93-124)
//   kMp2Opp  O^2 / D                    UMP2 opposite spin (mp2.cpp:126-139)
// O_ibja needs n1 = n3 and n2 = n4.  Grid-stride over the block, a
// warp-shuffle and shared-memory reduction per block into out[blockIdx.x];
// the host adds the per-block sums in block order, so the result does not
// depend on the order in which blocks finish.
constexpr int kMp2R = 0, kMp2Same = 1, kMp2Opp = 2;
__global__ void __launch_bounds__(256) mp2_sum_kernel(const double *__restrict__ O, const double *__restrict__ e1,
                                                      const double *__restrict__ e2, int n1, int n2, int n3, int n4,
                                                      int mode, double *out)
{
    const long long n = (long long)n1 * n2 * n3 * n4;
    double sum = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t % n4);
        const long long r = t / n4;
        const int j = (int)(r % n3);
        const long long r2 = r / n3;
        const int a = (int)(r2 % n2), i = (int)(r2 / n2);
        const double v = O[t];
        const double D = e1[i] + e2[j] - e1[n1 + a] - e2[n3 + b];
        if (mode == kMp2Opp) {
            sum += v * v / D;
        } else {
            const double w = O[(((long long)i * n2 + b) * n3 + j) * n4 + a];
            sum += mode == kMp2R ? v * (2.0 * v - w) / D : 0.25 * (v - w) * (v - w) / D;
        }
    }
    for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    __shared__ double part[8];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += part[w];
        out[blockIdx.x] = tot;
    }
}

// The transform behind pfk_mo_transform and the MP2 entry points: the
// result goes to the host buffer `out`, or, with eps1 set (blocks occ, vir,
// occ, vir; eps1 and eps2 the nbasis orbital energies of the first and the
// second pair's spin), into the MP2 sum of `mode` in *e_corr without leaving
// the device.  shared_E: an AO tensor (nbasis^4) kept across calls -- built
// by the first call that gets it empty, then reused and left intact (the
// second quarter's result then gets its own buffer instead of overwriting
// the tensor); null: a tensor of this call only.
static pfk_status mo_run(pfk_ctx *ctx, const double *C1, int n1, const double *C2, int n2, const double *C3, int n3,
                         const double *C4, int n4, double *out, const double *eps1, const double *eps2, int mode,
                         double *e_corr, DevBuf<double> *shared_E = nullptr)
{
    const int nb = ctx->nb;
    if (n1 < 1 || n2 < 1 || n3 < 1 || n4 < 1 || n1 > nb || n2 > nb || n3 > nb || n4 > nb)
        return ctx->fail(PFK_ERR_INVALID, "need 1 <= n_k <= nbasis");
    if (nb > 180) return ctx->fail(PFK_ERR_UNSUPPORTED, "dense tensor limited to 180 basis functions (8.4 GB)");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    if (!ctx->blas) {
        if (cublasCreate(&ctx->blas) != CUBLAS_STATUS_SUCCESS) return ctx->fail(PFK_ERR_CUDA, "cublasCreate failed");
    }
    if (cublasSetStream(ctx->blas, st) != CUBLAS_STATUS_SUCCESS) return ctx->fail(PFK_ERR_CUDA, "cublasSetStream failed");
    const size_t b = nb, b2 = b * b, b3 = b2 * b;
    // buffers allocated before the timed work: the AO tensor E and T1; T2
    // (n1 n2 nb^2 <= nb^4) then reuses E (or, with a shared tensor, a buffer
    // of its own), T3 (n1 n2 n3 nb <= n1 nb^3) reuses T1, and the result
    // (n1 n2 n3 n4 <= n1 n2 nb^2) reuses T2's buffer
    DevBuf<double> own_E, T1, T2buf, dC[4];
    DevBuf<double> &E = shared_E ? *shared_E : own_E;
    const bool build_E = E.p == nullptr;
    const double *hC[4] = {C1, C2, C3, C4};
    const int nk[4] = {n1, n2, n3, n4};
    for (int k = 0; k < 4; ++k) {
        PFK_CK(dC[k].alloc(b * nk[k]));
        PFK_CK(cudaMemcpyAsync(dC[k].p, hC[k], sizeof(double) * b * nk[k], cudaMemcpyHostToDevice, st));
    }
    cudaEvent_t ev[4] = {};
    struct EvFree {
        cudaEvent_t *e;
        ~EvFree() { for (int k = 0; k < 4; ++k) if (e[k]) cudaEventDestroy(e[k]); }
    } ev_free{ev};
    for (auto &x : ev) PFK_CK(cudaEventCreate(&x));
    if (build_E) PFK_CK(E.alloc(b2 * b2));
    PFK_CK(T1.alloc(b3 * n1));
    if (shared_E) PFK_CK(T2buf.alloc(b2 * (size_t)n1 * n2));
    PFK_CK(cudaEventRecord(ev[0], st));
    pfk_status s = PFK_OK;
    if (build_E) {
        PFK_CK(cudaMemsetAsync(E.p, 0, sizeof(double) * b2 * b2, st));
        s = run_classes(ctx, ctx->d_P.p, ctx->d_P.p, nullptr, 1, ctx->d_J.p, nullptr, nullptr, E.p, st, false);
        if (s != PFK_OK) return s;
    }
    PFK_CK(cudaEventRecord(ev[1], st));
    const double one = 1.0, zero = 0.0;
    auto ck = [&](cublasStatus_t r, const char *what) {
        return r == CUBLAS_STATUS_SUCCESS ? PFK_OK : ctx->fail(PFK_ERR_CUDA, std::string(what) + " failed");
    };
    double *T2 = shared_E ? T2buf.p : E.p, *T3 = T1.p, *O = T2;
    s = ck(cublasDgemm(ctx->blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)b3, n1, nb, &one, E.p, (int)b3, dC[0].p, nb, &zero,
                       T1.p, (int)b3),
           "quarter transform 1 (cublasDgemm)");
    if (s != PFK_OK) return s;
    s = ck(cublasDgemmStridedBatched(ctx->blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)b2, n2, nb, &one, T1.p, (int)b2,
                                     (long long)b3, dC[1].p, nb, 0, &zero, T2, (int)b2, (long long)b2 * n2, n1),
           "quarter transform 2 (cublasDgemmStridedBatched)");
    if (s != PFK_OK) return s;
    s = ck(cublasDgemmStridedBatched(ctx->blas, CUBLAS_OP_N, CUBLAS_OP_N, nb, n3, nb, &one, T2, nb, (long long)b2,
                                     dC[2].p, nb, 0, &zero, T3, nb, (long long)b * n3, n1 * n2),
           "quarter transform 3 (cublasDgemmStridedBatched)");
    if (s != PFK_OK) return s;
    const size_t no = (size_t)n1 * n2 * n3 * n4;
    s = ck(cublasDgemm(ctx->blas, CUBLAS_OP_T, CUBLAS_OP_N, n4, n1 * n2 * n3, nb, &one, dC[3].p, nb, T3, nb, &zero,
                       O, n4),
           "quarter transform 4 (cublasDgemm)");
    if (s != PFK_OK) return s;
    PFK_CK(cudaEventRecord(ev[2], st));
    if (eps1) {
        int nsm = 0;
        PFK_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device));
        const int grid = 8 * std::max(nsm, 1);   // 8 blocks of 256 per SM
        DevBuf<double> d_eps, d_sum;
        PFK_CK(d_eps.alloc(2 * b));
        PFK_CK(d_sum.alloc(grid));
        PFK_CK(cudaMemcpyAsync(d_eps.p, eps1, sizeof(double) * nb, cudaMemcpyHostToDevice, st));
        PFK_CK(cudaMemcpyAsync(d_eps.p + nb, eps2, sizeof(double) * nb, cudaMemcpyHostToDevice, st));
        mp2_sum_kernel<<<grid, 256, 0, st>>>(O, d_eps.p, d_eps.p + nb, n1, n2, n3, n4, mode, d_sum.p);
        PFK_CK(cudaGetLastError());
        std::vector<double> part(grid);
        PFK_CK(cudaMemcpyAsync(part.data(), d_sum.p, sizeof(double) * grid, cudaMemcpyDeviceToHost, st));
        PFK_CK(cudaEventRecord(ev[3], st));
        PFK_CK(cudaStreamSynchronize(st));
        double tot = 0.0;
        for (int k = 0; k < grid; ++k) tot += part[k];
        *e_corr = tot;
    } else {
        // the caller's buffer is pageable: stage it through two pinned chunks,
        // so the device copy runs at pinned speed and the host copy of one
        // chunk overlaps the device copy of the next
        constexpr size_t kChunk = size_t(16) << 20;   // bytes per chunk
        for (int k = 0; k < 2; ++k) {
            if (!ctx->pin[k]) PFK_CK(cudaHostAlloc(&ctx->pin[k], kChunk, cudaHostAllocDefault));
            if (!ctx->pin_ev[k]) PFK_CK(cudaEventCreateWithFlags(&ctx->pin_ev[k], cudaEventDisableTiming));
        }
        const size_t bytes = sizeof(double) * no;
        const char *src = reinterpret_cast<const char *>(O);
        char *dst = reinterpret_cast<char *>(out);
        size_t prev_off = 0, prev_n = 0;
        int k = 0;
        for (size_t off = 0; off < bytes; off += kChunk, ++k) {
            const int bi = k & 1;
            const size_t n = std::min(kChunk, bytes - off);
            PFK_CK(cudaMemcpyAsync(ctx->pin[bi], src + off, n, cudaMemcpyDeviceToHost, st));
            PFK_CK(cudaEventRecord(ctx->pin_ev[bi], st));
            if (k > 0) {   // the previous chunk, in the other buffer
                PFK_CK(cudaEventSynchronize(ctx->pin_ev[1 - bi]));
                std::memcpy(dst + prev_off, ctx->pin[1 - bi], prev_n);
            }
            prev_off = off;
            prev_n = n;
        }
        PFK_CK(cudaEventRecord(ev[3], st));
        if (k > 0) {
            PFK_CK(cudaEventSynchronize(ctx->pin_ev[(k - 1) & 1]));
            std::memcpy(dst + prev_off, ctx->pin[(k - 1) & 1], prev_n);
        }
    }
    PFK_CK(cudaStreamSynchronize(st));
    for (int k = 0; k < 3; ++k) {
        float ms = 0.f;
        PFK_CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
        ctx->mo_ms[k] = ms;
    }
    return PFK_OK;
}

pfk_status pfk_mo_transform(pfk_ctx *ctx, const double *C1, int n1, const double *C2, int n2, const double *C3,
                            int n3, const double *C4, int n4, double *out)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!C1 || !C2 || !C3 || !C4 || !out) return ctx->fail(PFK_ERR_INVALID, "null argument");
    return mo_run(ctx, C1, n1, C2, n2, C3, n3, C4, n4, out, nullptr, nullptr, 0, nullptr);
}

pfk_status pfk_rmp2_energy(pfk_ctx *ctx, const double *C, const double *eps, int nocc, double *e_corr)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!C || !eps || !e_corr) return ctx->fail(PFK_ERR_INVALID, "null argument");
    const int nb = ctx->nb, nv = nb - nocc;
    if (nocc < 1 || nv < 1) return ctx->fail(PFK_ERR_INVALID, "no occupied or virtual orbitals");
    const double *Cv = C + (size_t)nb * nocc;   // column-major: the virtual columns follow
    return mo_run(ctx, C, nocc, Cv, nv, C, nocc, Cv, nv, nullptr, eps, eps, kMp2R, e_corr);
}

pfk_status pfk_ump2_energy(pfk_ctx *ctx, const double *Ca, const double *eps_a, const double *Cb, const double *eps_b,
                           int n_alpha, int n_beta, double *e_corr)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!Ca || !eps_a || !Cb || !eps_b || !e_corr) return ctx->fail(PFK_ERR_INVALID, "null argument");
    const int nb = ctx->nb, nva = nb - n_alpha, nvb = nb - n_beta;
    if (n_alpha < 1 || nva < 1 || n_beta < 1 || nvb < 1)
        return ctx->fail(PFK_ERR_INVALID, "no occupied or virtual orbitals in a spin channel");
    const double *Cav = Ca + (size_t)nb * n_alpha, *Cbv = Cb + (size_t)nb * n_beta;
    double e_aa = 0.0, e_bb = 0.0, e_ab = 0.0;
    DevBuf<double> E;   // the AO tensor, built by the first transform and shared by all three
    pfk_status s =
        mo_run(ctx, Ca, n_alpha, Cav, nva, Ca, n_alpha, Cav, nva, nullptr, eps_a, eps_a, kMp2Same, &e_aa, &E);
    if (s == PFK_OK)
        s = mo_run(ctx, Cb, n_beta, Cbv, nvb, Cb, n_beta, Cbv, nvb, nullptr, eps_b, eps_b, kMp2Same, &e_bb, &E);
    if (s == PFK_OK)
        s = mo_run(ctx, Ca, n_alpha, Cav, nva, Cb, n_beta, Cbv, nvb, nullptr, eps_a, eps_b, kMp2Opp, &e_ab, &E);
    if (s == PFK_OK) *e_corr = e_aa + e_bb + e_ab;
    return s;
}

pfk_status pfk_mo_transform_times(const pfk_ctx *ctx, double *ms3)
{
    if (!ctx || !ms3) return PFK_ERR_STATE;
    for (int k = 0; k < 3; ++k) ms3[k] = ctx->mo_ms[k];
    return PFK_OK;
}

pfk_status pfk_class_stats(pfk_ctx *ctx, long long *quartets55, long long *prim_quartets55, double *ms55)
{
    if (!ctx) return PFK_ERR_STATE;
    cudaSetDevice(ctx->device);
    if (ms55) {
        for (int c = 0; c < kQuartetClasses; ++c) ctx->class_ms[c] = 0.f;
        pfk_status s = run_classes(ctx, ctx->d_P.p, ctx->d_P.p, nullptr, 1, ctx->d_J.p, ctx->d_K0.p, nullptr, nullptr,
                                   ctx->stream, true);
        if (s != PFK_OK) return s;
        for (int c = 0; c < kQuartetClasses; ++c) ms55[c] = ctx->class_ms[c];
    }
    for (int c = 0; c < kQuartetClasses; ++c) {
        if (quartets55) quartets55[c] = ctx->q_cnt[c] + ctx->q32_cnt[c];
        if (prim_quartets55) prim_quartets55[c] = ctx->prim_cnt[c];
    }
    return PFK_OK;
}

pfk_status pfk_precision_stats(pfk_ctx *ctx, long long *fp32_quartets55, long long *fp32_prim_quartets55)
{
    if (!ctx) return PFK_ERR_STATE;
    for (int c = 0; c < kQuartetClasses; ++c) {
        const bool mixed = ctx->precision == PFK_PREC_MIXED;
        if (fp32_quartets55) fp32_quartets55[c] = mixed ? ctx->q32_cnt[c] : 0;
        if (fp32_prim_quartets55) fp32_prim_quartets55[c] = mixed ? ctx->prim32_cnt[c] : 0;
    }
    return PFK_OK;
}

pfk_status pfk_autotune(pfk_ctx *ctx, int *choice55, double *ms55x3)
{
    if (!ctx) return PFK_ERR_STATE;
    cudaSetDevice(ctx->device);
    pfk_status s = ensure_work(ctx);
    if (s != PFK_OK) return s;
    const size_t nb2 = (size_t)ctx->nb * ctx->nb;
    PFK_CK(cudaMemsetAsync(ctx->d_P.p, 0, sizeof(double) * nb2, ctx->stream));   // timing only needs a density
    // candidates: Rys, Obara-Saika, Obara-Saika built for more blocks per SM
    // (8, 6 or 4 by class; L <= kOSMaxL only)
    const int candidates[3] = {0, kLaunchOS, kLaunchOS | kLaunchDense};
    double t[kQuartetClasses][3] = {};
    const int engine = ctx->engine;
    int chosen[kQuartetClasses];
    for (int c = 0; c < kQuartetClasses; ++c) chosen[c] = ctx->auto_flags[c];
    ctx->engine = PFK_ENGINE_AUTO;
    for (int v = 0; v < 3 && s == PFK_OK; ++v) {
        for (int c = 0; c < kQuartetClasses; ++c)
            ctx->auto_flags[c] = quartet_class_L(c) <= kOSMaxL ? candidates[v] : 0;
        for (int rep = 0; rep < 3 && s == PFK_OK; ++rep) {   // a warm-up pass, then the faster of two
            s = run_classes(ctx, ctx->d_P.p, ctx->d_P.p, nullptr, 1, ctx->d_J.p, ctx->d_K0.p, nullptr, nullptr,
                            ctx->stream, true);
            if (rep == 0) continue;
            for (int c = 0; c < kQuartetClasses; ++c)
                if (t[c][v] == 0.0 || ctx->class_ms[c] < t[c][v]) t[c][v] = ctx->class_ms[c];
        }
    }
    for (int c = 0; c < kQuartetClasses && s == PFK_OK; ++c) {
        if (ctx->q_cnt[c] + ctx->q32_cnt[c] == 0) continue;
        const int nv = quartet_class_L(c) <= kOSMaxL ? 3 : 1;
        int best = 0;
        for (int v = 1; v < nv; ++v)
            if (t[c][v] < t[c][best]) best = v;
        chosen[c] = candidates[best];
    }
    for (int c = 0; c < kQuartetClasses; ++c) {
        ctx->auto_flags[c] = chosen[c];
        if (choice55) choice55[c] = chosen[c];
        if (ms55x3)
            for (int v = 0; v < 3; ++v)
                ms55x3[3 * c + v] = (v == 0 || quartet_class_L(c) <= kOSMaxL) ? t[c][v] : 0.0;
    }
    ctx->engine = engine;
    drop_graphs(ctx);   // captured builds hold the old choices
    return s;
}

pfk_status pfk_set_density_screening(pfk_ctx *ctx, double dtol)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!(dtol >= 0.0) || !std::isfinite(dtol)) return ctx->fail(PFK_ERR_INVALID, "dtol must be finite and >= 0");
    cudaSetDevice(ctx->device);
    if (dtol > 0.0 && !ctx->d_Dsh.p) {
        std::vector<int> nbf(ctx->nshell);
        for (int s = 0; s < ctx->nshell; ++s) nbf[s] = ncart(ctx->L[s]);
        PFK_CK(ctx->d_shell_bf.alloc(ctx->nshell));
        PFK_CK(ctx->d_shell_nbf.alloc(ctx->nshell));
        PFK_CK(cudaMemcpy(ctx->d_shell_bf.p, ctx->bf_off.data(), sizeof(int) * ctx->nshell, cudaMemcpyHostToDevice));
        PFK_CK(cudaMemcpy(ctx->d_shell_nbf.p, nbf.data(), sizeof(int) * ctx->nshell, cudaMemcpyHostToDevice));
        PFK_CK(ctx->d_Dsh.alloc((size_t)ctx->nb * ctx->nb));
        PFK_CK(cudaMemset(ctx->d_Dsh.p, 0, sizeof(float) * (size_t)ctx->nb * ctx->nb));
    }
    if (dtol != ctx->dscreen_tol) drop_graphs(ctx);   // captured builds hold the old setting
    ctx->dscreen_tol = dtol;
    return PFK_OK;
}

pfk_status pfk_set_shard(pfk_ctx *ctx, int rank, int nranks)
{
    if (!ctx) return PFK_ERR_STATE;
    if (nranks < 1 || rank < 0 || rank >= nranks) return ctx->fail(PFK_ERR_INVALID, "need 0 <= rank < nranks");
    ctx->shard_rank = rank;
    ctx->shard_n = nranks;
    drop_graphs(ctx);
    return PFK_OK;
}

pfk_status pfk_set_primitive_tol(pfk_ctx *ctx, double ptol)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!(ptol >= 0.0 && ptol <= 1e-10)) return ctx->fail(PFK_ERR_INVALID, "need 0 <= ptol <= 1e-10");
    if (ptol != ctx->prim_tol) drop_graphs(ctx);   // captured builds hold the old value
    ctx->prim_tol = ptol;
    return PFK_OK;
}

pfk_status pfk_set_lanes(pfk_ctx *ctx, int lanes)
{
    if (!ctx) return PFK_ERR_STATE;
    if (lanes < 1 || lanes > kMaxLanes) return ctx->fail(PFK_ERR_INVALID, "need 1 <= lanes <= 4");
    if (lanes != ctx->lanes) drop_graphs(ctx);   // captured builds hold the old fork
    ctx->lanes = lanes;
    return PFK_OK;
}

pfk_status pfk_one_electron(const pfk_basis_desc *basis, int natom, const double *nuclei, double *S, double *T,
                            double *V, int device)
{
    std::string why;
    pfk_status vs = validate(basis, why);
    if (vs != PFK_OK) {
        g_last_error = "pfk_one_electron: " + why;
        return vs;
    }
    if (natom < 0 || (natom > 0 && !nuclei) || !S || !T || !V) {
        g_last_error = "pfk_one_electron: null output or nuclei pointer, or natom < 0";
        return PFK_ERR_INVALID;
    }
    for (int c = 0; c < 4 * natom; ++c)
        if (!std::isfinite(nuclei[c])) {
            g_last_error = "pfk_one_electron: non-finite nuclear coordinate or charge";
            return PFK_ERR_INVALID;
        }
    std::string what;
    cudaError_t e = one_electron_run(basis, natom, nuclei, S, T, V, device, what);
    if (e != cudaSuccess) {
        g_last_error = "pfk_one_electron: " + what + ": " + cudaGetErrorString(e);
        return PFK_ERR_CUDA;
    }
    return PFK_OK;
}

pfk_status pfk_measure_fma_peak(int device, double *fp64_tflops, double *fp32_tflops)
{
    cudaError_t e = measure_fma_peak(device, fp64_tflops, fp32_tflops);
    if (e != cudaSuccess) {
        g_last_error = std::string("pfk_measure_fma_peak: ") + cudaGetErrorString(e);
        return PFK_ERR_CUDA;
    }
    return PFK_OK;
}

}  // extern "C"

// ===========================================================================
// Allocation-free RHF build (pfk_fock_rhf_noalloc).
//
// For callers that may not allocate device memory -- code that runs inside a
// host application whose GPU memory is owned by another allocator or pool,
// or whose memory budget is fixed up front -- every device buffer the build
// needs (shell-pair and primitive-pair data, the Schwarz table, the screened
// quartet list, the J and K accumulators) is carved out of one file-scope
// array of PFK_NOALLOC_SCRATCH_BYTES.  Every GPU that loads this library
// holds that array until the process exits.
// ===========================================================================
static __device__ __align__(256) unsigned char g_noalloc_scratch[PFK_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char *g_noalloc_ptr[kNoallocMaxDevices] = {};

// Device address of the scratch array on the current device.  The name
// g_noalloc_scratch in host code is only a host-side stand-in, so the
// address is looked up once per device (with that device current) and
// cached; the same first call also sets the class kernels' shared-memory
// limits on that device.
pfk_status noalloc_setup(int dev, unsigned char **out, std::string &why)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (dev < 0 || dev >= kNoallocMaxDevices) {
        why = "device ordinal out of range for the allocation-free build";
        return PFK_ERR_UNSUPPORTED;
    }
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            why = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e);
            return PFK_ERR_CUDA;
        }
        JKArgs none{};
        for (int c = 0; c < kQuartetClasses; ++c) {
            if (!g_class_launchers[c]) {
                why = "class kernel table incomplete";
                return PFK_ERR_STATE;
            }
            g_class_launchers[c](nullptr, -1, none, 1, 0, nullptr);
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) {
            why = std::string("kernel configuration: ") + cudaGetErrorString(e);
            return PFK_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return PFK_OK;
}

// Bump allocation inside the scratch array (256-byte aligned pieces).
struct ScratchCarver {
    unsigned char *base;
    size_t used = 0;
    template <typename T>
    T *take(size_t count)
    {
        const size_t off = (used + 255) & ~size_t(255);
        used = off + sizeof(T) * count;
        return reinterpret_cast<T *>(base + off);
    }
};

template <typename T>
size_t carve_size(size_t used, size_t count)
{
    return ((used + 255) & ~size_t(255)) + sizeof(T) * count;
}

}  // namespace

extern "C" pfk_status pfk_fock_rhf_noalloc(const pfk_basis_desc *basis, const double *dP, double *dG, double tol_eri,
                                           void *stream)
{
    std::string why;
    pfk_status vs = validate(basis, why);
    if (vs != PFK_OK) {
        g_last_error = "pfk_fock_rhf_noalloc: " + why;
        return vs;
    }
    if (!dP || !dG || !(tol_eri >= 0.0) || !std::isfinite(tol_eri)) {
        g_last_error = "pfk_fock_rhf_noalloc: null matrix or bad tol_eri";
        return PFK_ERR_INVALID;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        g_last_error = std::string("pfk_fock_rhf_noalloc: cudaGetDevice: ") + cudaGetErrorString(e);
        return PFK_ERR_CUDA;
    }
    unsigned char *scratch = nullptr;
    vs = noalloc_setup(dev, &scratch, why);
    if (vs != PFK_OK) {
        g_last_error = "pfk_fock_rhf_noalloc: " + why;
        return vs;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // host-side shell-pair data, as pfk_create builds it
    pfk_ctx h;
    h.nshell = basis->nshell;
    h.bf_off.resize(basis->nshell);
    int nb = 0;
    for (int s = 0; s < basis->nshell; ++s) {
        h.bf_off[s] = nb;
        nb += ncart(basis->L[s]);
    }
    h.nb = nb;
    build_pairs(&h, basis);
    const size_t nb2 = (size_t)nb * nb;

    // everything but the quartet list, checked before the device is touched
    size_t need = 0;
    need = carve_size<PairInfo>(need, h.npairs);
    need = carve_size<PrimPair>(need, h.prims.size());
    need = carve_size<int>(need, h.npairs);
    need = carve_size<double>(need, nb2);
    need = carve_size<FxWord>(need, 2 * nb2);
    need = carve_size<FxWord>(need, 2 * nb2);
    if (need > PFK_NOALLOC_SCRATCH_BYTES) {
        g_last_error = "pfk_fock_rhf_noalloc: basis needs " + std::to_string(need) +
                       " bytes of scratch before the quartet list; the limit is " +
                       std::to_string((size_t)PFK_NOALLOC_SCRATCH_BYTES) + " bytes";
        return PFK_ERR_UNSUPPORTED;
    }
    ScratchCarver cv{scratch};
    PairInfo *d_pairs = cv.take<PairInfo>(h.npairs);
    PrimPair *d_prims = cv.take<PrimPair>(h.prims.size());
    int *d_ids = cv.take<int>(h.npairs);
    double *d_Q = cv.take<double>(nb2);
    FxWord *d_J = cv.take<FxWord>(2 * nb2);
    FxWord *d_K = cv.take<FxWord>(2 * nb2);

#define PFK_NA_CK(call)                                                                           \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            g_last_error = std::string("pfk_fock_rhf_noalloc: " #call ": ") + cudaGetErrorString(e_); \
            return PFK_ERR_CUDA;                                                                 \
        }                                                                                        \
    } while (0)

    // primitive bounds (uploads pairs, primitives and the class-grouped pair
    // ids), then the Schwarz table (the array keeps the previous call's
    // contents: clear it)
    std::vector<int> cls_begin;
    PFK_NA_CK(prim_bounds(&h, d_pairs, d_prims, d_ids, cls_begin, st));
    PFK_NA_CK(cudaMemsetAsync(d_Q, 0, sizeof(double) * nb2, st));
    for (int x = 0; x < kPairClasses; ++x)
        launch_schwarz(x, d_ids + cls_begin[x], cls_begin[x + 1] - cls_begin[x], d_pairs, d_prims, d_Q, nb, st);
    PFK_NA_CK(cudaGetLastError());
    std::vector<double> Q(nb2);
    PFK_NA_CK(cudaMemcpyAsync(Q.data(), d_Q, sizeof(double) * nb2, cudaMemcpyDeviceToHost, st));
    PFK_NA_CK(cudaStreamSynchronize(st));

    // per-pair bounds, Q-sorted class lists, screened shell-quartet lists
    std::vector<int> sorted[kPairClasses];
    for (int p = 0; p < h.npairs; ++p) {
        PairInfo &pi = h.pairs[p];
        const int na = ncart(h.pair_la[p]), nbb = ncart(h.pair_lb[p]);
        double qmax = 0.0, qmin = INFINITY;
        for (int a = 0; a < na; ++a)
            for (int c = 0; c < nbb; ++c) {
                const double q = Q[(size_t)(pi.bf_a + a) * nb + pi.bf_b + c];
                qmax = std::max(qmax, q);
                qmin = std::min(qmin, q);
            }
        pi.qmax = qmax;
        pi.qmin = qmin;
        sorted[h.pair_pc[p]].push_back(p);
    }
    for (auto &v : sorted)
        std::stable_sort(v.begin(), v.end(), [&](int a, int b) { return h.pairs[a].qmax > h.pairs[b].qmax; });
    std::vector<uint2> quart;
    long long cls_off[kQuartetClasses + 1] = {};
    for (int x = 0; x < kPairClasses; ++x)
        for (int y = 0; y <= x; ++y) {
            const int cls = quartet_class(x, y);
            cls_off[cls] = (long long)quart.size();
            const auto &X = sorted[x], &Y = sorted[y];
            for (size_t a = 0; a < X.size(); ++a) {
                const double qa = h.pairs[X[a]].qmax;
                size_t lo = 0, hi = Y.size();   // kets kept: a prefix of the Q-sorted list
                while (lo < hi) {
                    const size_t mid = (lo + hi) / 2;
                    if (qa * h.pairs[Y[mid]].qmax >= tol_eri) lo = mid + 1;
                    else hi = mid;
                }
                for (size_t b = (x == y ? a : 0); b < lo; ++b)
                    quart.push_back(make_uint2((unsigned)X[a], (unsigned)Y[b]));
            }
        }
    // (x, y) visits the classes in increasing class index, so cls_off holds
    // each class's start and the next class's start is its end
    cls_off[kQuartetClasses] = (long long)quart.size();
    const size_t total = carve_size<uint2>(cv.used, quart.size());
    if (total > PFK_NOALLOC_SCRATCH_BYTES) {
        g_last_error = "pfk_fock_rhf_noalloc: basis needs " + std::to_string(total) +
                       " bytes of scratch with its screened quartet list; the limit is " +
                       std::to_string((size_t)PFK_NOALLOC_SCRATCH_BYTES) + " bytes";
        return PFK_ERR_UNSUPPORTED;
    }
    uint2 *d_q = cv.take<uint2>(quart.size());
    PFK_NA_CK(cudaMemcpyAsync(d_pairs, h.pairs.data(), sizeof(PairInfo) * h.npairs, cudaMemcpyHostToDevice, st));
    if (!quart.empty())
        PFK_NA_CK(cudaMemcpyAsync(d_q, quart.data(), sizeof(uint2) * quart.size(), cudaMemcpyHostToDevice, st));

    // the build: accumulators start at zero on every call
    PFK_NA_CK(cudaMemsetAsync(d_J, 0, sizeof(FxWord) * 2 * nb2, st));
    PFK_NA_CK(cudaMemsetAsync(d_K, 0, sizeof(FxWord) * 2 * nb2, st));
    JKArgs a{};
    a.pairs = d_pairs;
    a.prims = d_prims;
    a.Qao = d_Q;
    a.Pj = dP;
    a.Pk0 = dP;
    a.Jacc = d_J;
    a.Kacc0 = d_K;
    a.tol = tol_eri;
    a.ptol = kPrimQuartetTol;
    a.nb = nb;
    a.qstride = 1;
    a.qoffset = 0;
    for (int c = 0; c < kQuartetClasses; ++c) {
        const long long n = cls_off[c + 1] - cls_off[c];
        if (n > 0) g_class_launchers[c](d_q + cls_off[c], n, a, 1, 0, st);
    }
    PFK_NA_CK(cudaGetLastError());
    PFK_NA_CK(combine(d_J, d_K, 1.0, -0.5, dG, nb, st));
    PFK_NA_CK(cudaStreamSynchronize(st));
#undef PFK_NA_CK
    return PFK_OK;
}

// ===========================================================================
// ERI batches (pfk_eri_batch_*): the contracted, normalised Cartesian block
// of every listed shell quartet, from the same class kernels the Fock builds
// use, written out instead of digested.  For the per-class measurements and
// accuracy tables of the integral kernels (the reference's per-quartet
// contracted integrals, os.cpp:994-1010 and rys.cpp:489-505).
// ===========================================================================
struct pfk_eri_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    std::vector<int> L;        // per shell
    std::vector<int> pair_pc;  // per pair
    DevBuf<PairInfo> d_pairs;
    DevBuf<PrimPair> d_prims;
    DevBuf<uint2> d_quart;
    long long nq = 0;
    int cls = -1;              // class of the listed quartets

    pfk_status fail(pfk_status s, const std::string &msg)
    {
        err = msg;
        return s;
    }
    pfk_status cuda_fail(const char *what, cudaError_t e)
    {
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return PFK_ERR_CUDA;
    }
};

extern "C" {

pfk_status pfk_eri_batch_create(const pfk_basis_desc *basis, int npairs, const int *pair_shells, int device,
                                pfk_eri_batch **out)
{
    if (!out) {
        g_last_error = "pfk_eri_batch_create: out is null";
        return PFK_ERR_INVALID;
    }
    *out = nullptr;
    std::string why;
    pfk_status vs = validate(basis, why, false);
    if (vs != PFK_OK) {
        g_last_error = "pfk_eri_batch_create: " + why;
        return vs;
    }
    if (npairs <= 0 || !pair_shells) {
        g_last_error = "pfk_eri_batch_create: no shell pairs";
        return PFK_ERR_INVALID;
    }
    std::vector<int> poff(basis->nshell + 1, 0);
    for (int s = 0; s < basis->nshell; ++s) poff[s + 1] = poff[s] + basis->nprim[s];
    std::vector<PairInfo> pairs;
    std::vector<PrimPair> prims;
    std::vector<int> pc;
    try {
        pairs.reserve(npairs);
        pc.reserve(npairs);
        for (int p = 0; p < npairs; ++p) {
            const int A = pair_shells[2 * p], B = pair_shells[2 * p + 1];
            if (A < 0 || B < 0 || A >= basis->nshell || B >= basis->nshell) {
                g_last_error = "pfk_eri_batch_create: pair " + std::to_string(p) + " names a shell out of range";
                return PFK_ERR_INVALID;
            }
            if (basis->L[A] < basis->L[B]) {
                g_last_error = "pfk_eri_batch_create: pair " + std::to_string(p) +
                               " must list the shell of higher angular momentum first";
                return PFK_ERR_INVALID;
            }
            if ((long long)prims.size() + (long long)basis->nprim[A] * basis->nprim[B] > INT32_MAX) {
                g_last_error = "pfk_eri_batch_create: more than 2^31 primitive pairs";
                return PFK_ERR_UNSUPPORTED;
            }
            // qp = 1 and no primitive floor: every primitive quartet is evaluated
            append_pair(basis, poff, A, B, 0, 0, 1.0, pairs, prims);
            pairs.back().qmax = pairs.back().qmin = 1.0;
            pc.push_back(pair_class(basis->L[A], basis->L[B]));
        }
    } catch (const std::bad_alloc &) {
        g_last_error = "pfk_eri_batch_create: host allocation failed";
        return PFK_ERR_NOMEM;
    }
    pfk_eri_batch *ctx = new (std::nothrow) pfk_eri_batch();
    if (!ctx) {
        g_last_error = "pfk_eri_batch_create: host allocation failed";
        return PFK_ERR_NOMEM;
    }
    auto bail = [&](pfk_status s) {
        g_last_error = "pfk_eri_batch_create: " + ctx->err;
        pfk_eri_batch_destroy(ctx);
        return s;
    };
    ctx->device = device;
    ctx->L.assign(basis->L, basis->L + basis->nshell);
    ctx->pair_pc = std::move(pc);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return bail(ctx->cuda_fail("cudaSetDevice", e));
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(ctx->cuda_fail("cudaStreamCreate", e));
    // the split and team kernels' shared-memory limits on this device
    JKArgs none{};
    for (int c = 0; c < kQuartetClasses; ++c) {
        if (!g_class_launchers[c]) return bail(ctx->fail(PFK_ERR_STATE, "class kernel table incomplete"));
        g_class_launchers[c](nullptr, -1, none, 1, 0, nullptr);
    }
    if ((e = ctx->d_pairs.alloc(pairs.size())) != cudaSuccess) return bail(ctx->cuda_fail("cudaMalloc(pairs)", e));
    if ((e = ctx->d_prims.alloc(prims.size())) != cudaSuccess) return bail(ctx->cuda_fail("cudaMalloc(prims)", e));
    e = cudaMemcpyAsync(ctx->d_pairs.p, pairs.data(), sizeof(PairInfo) * pairs.size(), cudaMemcpyHostToDevice,
                        ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ctx->d_prims.p, prims.data(), sizeof(PrimPair) * prims.size(), cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return bail(ctx->cuda_fail("upload of pair data", e));
    *out = ctx;
    return PFK_OK;
}

pfk_status pfk_eri_batch_destroy(pfk_eri_batch *b)
{
    if (!b) return PFK_OK;
    cudaSetDevice(b->device);
    b->d_pairs.release();
    b->d_prims.release();
    b->d_quart.release();
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return PFK_OK;
}

const char *pfk_eri_batch_last_error(const pfk_eri_batch *b) { return b ? b->err.c_str() : g_last_error.c_str(); }

pfk_status pfk_eri_batch_set_quartets(pfk_eri_batch *ctx, const int *quartets, long long n, int *cls, int *ncomp)
{
    if (!ctx) return PFK_ERR_STATE;
    if (!quartets || n <= 0) return ctx->fail(PFK_ERR_INVALID, "no quartets");
    const int npairs = (int)ctx->pair_pc.size();
    int c0 = -1;
    std::vector<uint2> q;
    try {
        q.resize((size_t)n);
    } catch (const std::bad_alloc &) {
        return ctx->fail(PFK_ERR_NOMEM, "host allocation failed");
    }
    for (long long t = 0; t < n; ++t) {
        const int x = quartets[2 * t], y = quartets[2 * t + 1];
        if (x < 0 || y < 0 || x >= npairs || y >= npairs)
            return ctx->fail(PFK_ERR_INVALID, "quartet " + std::to_string(t) + " names a pair out of range");
        const int px = ctx->pair_pc[x], py = ctx->pair_pc[y];
        if (px < py)
            return ctx->fail(PFK_ERR_INVALID, "quartet " + std::to_string(t) +
                                                  ": the bra pair's class must not be below the ket pair's");
        const int c = quartet_class(px, py);
        if (c0 < 0) c0 = c;
        if (c != c0)
            return ctx->fail(PFK_ERR_INVALID, "quartet " + std::to_string(t) + " is of another class than quartet 0");
        q[(size_t)t] = make_uint2((unsigned)x, (unsigned)y);
    }
    cudaSetDevice(ctx->device);
    PFK_CK(ctx->d_quart.alloc((size_t)n));
    PFK_CK(cudaMemcpyAsync(ctx->d_quart.p, q.data(), sizeof(uint2) * n, cudaMemcpyHostToDevice, ctx->stream));
    PFK_CK(cudaStreamSynchronize(ctx->stream));
    ctx->nq = n;
    ctx->cls = c0;
    int x = 0;
    while ((x + 1) * (x + 2) / 2 <= c0) ++x;
    const int y = c0 - x * (x + 1) / 2;
    if (cls) *cls = c0;
    if (ncomp) *ncomp = ncart(pc_la(x)) * ncart(pc_lb(x)) * ncart(pc_la(y)) * ncart(pc_lb(y));
    return PFK_OK;
}

pfk_status pfk_eri_batch_run(pfk_eri_batch *ctx, long long first, long long count, int engine, int precision,
                             double *d_out, void *stream)
{
    if (!ctx) return PFK_ERR_STATE;
    if (ctx->cls < 0) return ctx->fail(PFK_ERR_STATE, "no quartets set");
    if (!d_out) return ctx->fail(PFK_ERR_INVALID, "output is null");
    if (first < 0 || count <= 0 || first + count > ctx->nq) return ctx->fail(PFK_ERR_INVALID, "quartet range out of bounds");
    if (engine != PFK_ENGINE_OS && engine != PFK_ENGINE_RYS)
        return ctx->fail(PFK_ERR_INVALID, "engine must be PFK_ENGINE_OS or PFK_ENGINE_RYS");
    if (precision != PFK_PREC_FP64 && precision != PFK_PREC_MIXED)
        return ctx->fail(PFK_ERR_INVALID, "precision must be PFK_PREC_FP64 or PFK_PREC_MIXED");
    if (engine == PFK_ENGINE_OS && quartet_class_L(ctx->cls) > kOSMaxL)
        return ctx->fail(PFK_ERR_UNSUPPORTED, "no Obara-Saika kernel above LA+LB+LC+LD = 4 (engine os runs Rys there)");
    cudaSetDevice(ctx->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    JKArgs a{};
    a.pairs = ctx->d_pairs.p;
    a.prims = ctx->d_prims.p;
    a.blk_out = d_out;
    a.tol = 0.0;
    a.ptol = 0.0;
    a.nb = 0;
    a.qstride = 1;
    a.qoffset = 0;
    const int flags = (engine == PFK_ENGINE_OS ? kLaunchOS : 0) | (precision == PFK_PREC_MIXED ? kLaunchFP32 : 0);
    g_class_launchers[ctx->cls](ctx->d_quart.p + first, count, a, 1, flags, st);
    PFK_CK(cudaGetLastError());
    return PFK_OK;
}

}  // extern "C"

namespace pfk {
int ctx_device(const pfk_ctx *ctx) { return ctx->device; }
pfk_status fock_rhf_direct(pfk_ctx *ctx, const double *dP, double *dG, cudaStream_t st)
{
    cudaSetDevice(ctx->device);
    return rhf_sequence(ctx, dP, dG, st);
}
pfk_status ctx_fail(pfk_ctx *ctx, pfk_status s, const std::string &msg) { return ctx->fail(s, msg); }
}  // namespace pfk
