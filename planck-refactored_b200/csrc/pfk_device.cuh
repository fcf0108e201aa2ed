// pfk_device.cuh -- device-side building blocks of the Fock engine (sm_100a).
//
// Integral method: Rys quadrature (the reference's RysQuad path,
// src/integrals/rys.cpp:250-485), reorganised for the GPU:
//   * one shell quartet (all Cartesian components) per thread or per team,
//     instead of one Cartesian component quartet per call;
//   * roots/weights from piecewise Chebyshev tables generated offline in
//     80-digit arithmetic (gen_rys_table.py) instead of a per-primitive
//     long-double moment/eigensolver construction (rys_roots.cpp:88-235);
//   * the A->B and C->D transfer (rys.cpp:293-363) applied per Cartesian
//     axis to the 2D integrals of each root, so the 6D product is formed
//     only for the output components;
//   * J/K digestion fused into the integral kernel (os.cpp:1512-1520 does it
//     as a separate O(nb^4) pass over a stored tensor).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pfk {

// ---------------------------------------------------------------------------
// Shapes
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int ncart(int L) { return (L + 1) * (L + 2) / 2; }
__host__ __device__ constexpr int cart_block(int i)
{
    int n = 0;
    while ((n + 1) * (n + 2) / 2 <= i) ++n;
    return n;
}
// Cartesian component i of a shell of angular momentum L, in the reference's
// order (lx descending, then ly descending; src/basis/basis.cpp:20-37).
__host__ __device__ constexpr int cart_lx(int L, int i) { return L - cart_block(i); }
__host__ __device__ constexpr int cart_lz(int L, int i)
{
    return i - cart_block(i) * (cart_block(i) + 1) / 2;
}
__host__ __device__ constexpr int cart_ly(int L, int i) { return L - cart_lx(L, i) - cart_lz(L, i); }
// Iterative (not recursive) so that calls with unrolled-loop indices inline
// and fold to constants instead of becoming device-side calls.
__host__ __device__ constexpr int dfact(int n)
{
    int r = 1;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}
// 1/sqrt((2lx-1)!!(2ly-1)!!(2lz-1)!!) (src/basis/gaussian.cpp:283-296); the
// double factorials for L <= 3 are 1, 1, 3, 15, so the square roots below are
// of small integers.
__host__ __device__ constexpr double inv_sqrt_small(int d)
{
    return d == 1 ? 1.0 : d == 3 ? 0.57735026918962576451 : d == 9 ? 1.0 / 3.0
         : d == 15 ? 0.25819888974716112568 : 0.0;
}
__host__ __device__ constexpr double cart_norm(int L, int i)
{
    return inv_sqrt_small(dfact(2 * cart_lx(L, i) - 1) * dfact(2 * cart_ly(L, i) - 1) *
                          dfact(2 * cart_lz(L, i) - 1));
}

// ---------------------------------------------------------------------------
// Data layout in HBM
// ---------------------------------------------------------------------------
// One primitive pair of an (oriented) shell pair: Gaussian product data.
// K = (pi/zeta)^1.5 exp(-alpha beta |AB|^2 / zeta) c_a c_b N_a N_b
// (src/base/types.h:631-674 without the component norms, which are applied
// per Cartesian component after contraction), stored as Kz = K sqrt(zeta),
// the factor the quartet prefactor 2 sqrt(rho/pi) K_ab K_cd needs.
// qp is the pair's primitive Schwarz bound: the largest over its Cartesian
// components of sqrt|(ab|ab)| for this primitive pair alone, contraction
// coefficients and component norms included.  By the Cauchy-Schwarz
// inequality of the Coulomb metric, qp_ab qp_cd bounds what the primitive
// quartet adds to any normalised component integral of the shell quartet.
struct __align__(16) PrimPair {
    double zeta, inv_zeta;
    double Px, Py, Pz;
    double PAx, PAy, PAz;   // P - A (A = first centre of the oriented pair)
    double Kz, qp;
};

// Shell pair a <= b (shell order), oriented so that L(A) >= L(B).  Its
// primitive pairs are stored by decreasing qp; the first nprim have
// qp * (largest qp of the basis) >= kPrimPairFloor and are the ones the Fock
// build may evaluate, all nprim_full of them enter the Schwarz table.
struct __align__(16) PairInfo {
    int prim_off, nprim;     // range in the PrimPair array
    int bf_a, bf_b;          // first basis function of A and of B
    double ABx, ABy, ABz;    // A - B
    double qmax, qmin;       // max / min of Q(i,j) over the pair's components
    int nprim_full, pad_;
};

// Primitive pairs that cannot reach 1e-21 with any partner are dropped when
// the pairs are built.  Each build skips the primitive quartets with
// qp_ab qp_cd below JKArgs::ptol (kPrimQuartetTol unless the context sets
// another value): each adds less than ptol to every integral it touches.
constexpr double kPrimPairFloor = 1e-21;
constexpr double kPrimQuartetTol = 1e-16;

struct JKArgs {
    const PairInfo *__restrict__ pairs;
    const PrimPair *__restrict__ prims;
    const double *__restrict__ Qao;    // nb x nb Schwarz table
    const double *__restrict__ Pj;     // density for J
    const double *__restrict__ Pk0;    // densities for K (Pk1 used when NK == 2)
    const double *__restrict__ Pk1;
    // nb x nb fixed-point accumulators (unsymmetrised), two 64-bit words
    // per element (fx_add); the sums do not depend on the order of the adds
    unsigned long long *Jacc;
    unsigned long long *Kacc0;
    unsigned long long *Kacc1;
    double *eri_out;                    // dense tensor mode (nb^4) when non-null
    // block mode when non-null: list entry t writes its normalised Cartesian
    // block, unscreened, to blk_out[t * N ...] (no digestion, no tensor)
    double *blk_out;
    double tol;
    int nb;
    // this launch evaluates quartets[t * qstride + qoffset], t < nq (one
    // shard of a list split across GPUs; 1 and 0 for the whole list)
    int qstride, qoffset;
    // density screening (builds on a difference density): when Dsh is set,
    // a shell quartet is skipped if qmax(bra) qmax(ket) max|D| < dtol, with
    // Dsh[first bf of shell 1 * nb + first bf of shell 2] = max |P| over
    // that shell-pair block of every density of the build
    const float *__restrict__ Dsh;
    double dtol;
    // primitive quartets with qp_ab qp_cd < ptol are skipped (0: none)
    double ptol;
};

// ---------------------------------------------------------------------------
// Rys roots and weights
// ---------------------------------------------------------------------------
#define PFK_RYS_CONST_STORAGE static __constant__ const
#define PFK_RYS_TABLE_STORAGE static __device__ const
#include "rys_table_data.inc"

// Clenshaw evaluation of one root's u and w series together.  c points at
// the (u_0, w_0) pair of this root and interval; consecutive degrees are
// `stride` pairs apart (table layout: [k][root][interval][u, w]).
__device__ __forceinline__ void clenshaw_pair(const double *__restrict__ c, int stride, double x, double &u,
                                              double &w)
{
    const double2 *c2 = reinterpret_cast<const double2 *>(c);
    double bu1 = 0.0, bu2 = 0.0, bw1 = 0.0, bw2 = 0.0;
    const double x2 = 2.0 * x;
#pragma unroll
    for (int k = PFK_RYS_DEG; k >= 1; --k) {
        const double2 ck = __ldg(c2 + k * stride);
        const double tu = fma(x2, bu1, ck.x - bu2);
        const double tw = fma(x2, bw1, ck.y - bw2);
        bu2 = bu1;
        bu1 = tu;
        bw2 = bw1;
        bw1 = tw;
    }
    const double2 c0 = __ldg(c2);
    u = fma(x, bu1, c0.x - bu2);
    w = fma(x, bw1, c0.y - bw2);
}

// All NR roots u_r = t_r^2 and weights of the measure exp(-T u) u^-1/2 / 2 du.
template <int NR>
__device__ __forceinline__ void rys_roots(double T, double *u, double *w)
{
    if (T < kRysTmax[NR]) {
        const int iv = (int)(T * (1.0 / PFK_RYS_H));
        const double x = (T - iv * PFK_RYS_H) * (2.0 / PFK_RYS_H) - 1.0;
        const int nint = kRysNint[NR];
        const double *base = kRysCheb + kRysOffset[NR] + 2 * iv;
#pragma unroll
        for (int r = 0; r < NR; ++r) clenshaw_pair(base + 2 * r * nint, NR * nint, x, u[r], w[r]);
    } else {
        const double iT = 1.0 / T;
        const double isT = sqrt(iT);
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            u[r] = kRysAsymU[NR][r] * iT;
            w[r] = kRysAsymW[NR][r] * isT;
        }
    }
}

template <int NR>
__device__ __forceinline__ void rys_root_one(double T, int r, double &u, double &w)
{
    if (T < kRysTmax[NR]) {
        const int iv = (int)(T * (1.0 / PFK_RYS_H));
        const double x = (T - iv * PFK_RYS_H) * (2.0 / PFK_RYS_H) - 1.0;
        const int nint = kRysNint[NR];
        clenshaw_pair(kRysCheb + kRysOffset[NR] + 2 * iv + 2 * r * nint, NR * nint, x, u, w);
    } else {
        const double iT = 1.0 / T;
        u = kRysAsymU[NR][r] * iT;
        w = kRysAsymW[NR][r] * sqrt(iT);
    }
}

// ---------------------------------------------------------------------------
// Per-axis 2D integrals of one root (rys.cpp:250-280 recurrence), then the
// A->B and C->D transfers on that axis (rys.cpp:293-363 applied per axis):
// out[a*AST + b*BST + c*(LD+1) + d] = I_axis(a, b, c, d).  The default strides
// pack the table densely; shared-memory tables pass padded strides so that
// lanes reading different a (or a, b) slices hit different banks.
// ---------------------------------------------------------------------------
template <int LA, int LB, int LC, int LD, typename R, int BST = (LC + 1) * (LD + 1), int AST = (LB + 1) * BST>
__device__ __forceinline__ void axis_table(R C00, R D00, R B00, R B10, R B01, R AB, R CD, R scale,
                                           R *__restrict__ out)
{
    constexpr int E = LA + LB, F = LC + LD;
    R I[E + 1][F + 1];
    I[0][0] = scale;
    if constexpr (E > 0) I[1][0] = C00 * scale;
#pragma unroll
    for (int a = 1; a < E; ++a) I[a + 1][0] = C00 * I[a][0] + R(a) * B10 * I[a - 1][0];
#pragma unroll
    for (int c = 0; c < F; ++c) {
        I[0][c + 1] = D00 * I[0][c];
        if (c > 0) I[0][c + 1] += R(c) * B01 * I[0][c - 1];
#pragma unroll
        for (int a = 1; a <= E; ++a) {
            R v = D00 * I[a][c] + R(a) * B00 * I[a - 1][c];
            if (c > 0) v += R(c) * B01 * I[a][c - 1];
            I[a][c + 1] = v;
        }
    }
    // A -> B: G[a][b][c] with G(a, b+1) = G(a+1, b) + AB G(a, b)
    R G[E + 1][LB + 1][F + 1];
#pragma unroll
    for (int a = 0; a <= E; ++a)
#pragma unroll
        for (int c = 0; c <= F; ++c) G[a][0][c] = I[a][c];
#pragma unroll
    for (int b = 0; b < LB; ++b)
#pragma unroll
        for (int a = 0; a < E - b; ++a)
#pragma unroll
            for (int c = 0; c <= F; ++c) G[a][b + 1][c] = G[a + 1][b][c] + AB * G[a][b][c];
    // C -> D on the (a <= LA, b <= LB) slice
#pragma unroll
    for (int a = 0; a <= LA; ++a)
#pragma unroll
        for (int b = 0; b <= LB; ++b) {
            R H[F + 1][LD + 1];
#pragma unroll
            for (int c = 0; c <= F; ++c) H[c][0] = G[a][b][c];
#pragma unroll
            for (int d = 0; d < LD; ++d)
#pragma unroll
                for (int c = 0; c < F - d; ++c) H[c][d + 1] = H[c + 1][d] + CD * H[c][d];
#pragma unroll
            for (int c = 0; c <= LC; ++c)
#pragma unroll
                for (int d = 0; d <= LD; ++d) out[a * AST + b * BST + c * (LD + 1) + d] = H[c][d];
        }
}

// Per-primitive-quartet scalars shared by all roots.
struct QuartetScalars {
    double T, pref, rdelta, rho;
    double zinv, einv;
    double WPx, WPy, WPz, WQx, WQy, WQz;
};

__device__ __forceinline__ QuartetScalars quartet_scalars(const PrimPair &p, const PrimPair &q)
{
    QuartetScalars s;
    const double delta = p.zeta + q.zeta;
    const double rs = rsqrt(delta);          // 1/sqrt(zeta + eta)
    s.rdelta = rs * rs;
    s.rho = p.zeta * q.zeta * s.rdelta;
    const double PQx = p.Px - q.Px, PQy = p.Py - q.Py, PQz = p.Pz - q.Pz;
    s.T = s.rho * (PQx * PQx + PQy * PQy + PQz * PQz);
    // 2 sqrt(rho / pi) K_ab K_cd  (rys.cpp:415), sqrt(rho) = sqrt(zeta) sqrt(eta) / sqrt(delta),
    // with sqrt(zeta) and sqrt(eta) folded into Kz
    s.pref = 1.1283791670955125739 * (p.Kz * q.Kz) * rs;
    s.zinv = p.inv_zeta;
    s.einv = q.inv_zeta;
    const double fp = -q.zeta * s.rdelta, fq = p.zeta * s.rdelta;  // W-P = fp PQ, W-Q = fq PQ
    s.WPx = fp * PQx; s.WPy = fp * PQy; s.WPz = fp * PQz;
    s.WQx = fq * PQx; s.WQy = fq * PQy; s.WQz = fq * PQz;
    return s;
}

__device__ __forceinline__ PrimPair load_prim(const PrimPair *__restrict__ a, int i)
{
    const double2 *v = reinterpret_cast<const double2 *>(a + i);
    const double2 x0 = __ldg(v), x1 = __ldg(v + 1), x2 = __ldg(v + 2), x3 = __ldg(v + 3), x4 = __ldg(v + 4);
    PrimPair p;
    p.zeta = x0.x; p.inv_zeta = x0.y; p.Px = x1.x; p.Py = x1.y; p.Pz = x2.x;
    p.PAx = x2.y; p.PAy = x3.x; p.PAz = x3.y; p.Kz = x4.x; p.qp = x4.y;
    return p;
}

// ---------------------------------------------------------------------------
// Deterministic accumulation.  Every J/K contribution v is rounded to the
// nearest multiple of 2^-60, X = rint(v 2^60), and added as an integer split
// over two 64-bit words of the element: X = hi 2^36 + lo with |lo| <= 2^35,
// so contributions below 2^-25 in magnitude touch only lo.  Integer
// addition is associative, so the accumulated value is the same whatever
// order the threads, warps, streams and kernels add in, and a build is
// bitwise reproducible (FP64 atomics are not: their rounding depends on
// arrival order).  The value is hi_sum 2^-24 + lo_sum 2^-60 whichever way
// each X was split.  Range: |v| < 2^27 per contribution, |sum| < 2^29 per
// element; lo holds 2^28 full-size adds per element.  Resolution: 2^-61
// rounding per add, below the last bit of any FP64 value above 2^-8.
//
// The split needs no float-to-integer conversion: a double in [2^52, 2^53)
// has a unit in the last place of 1, so fma(v, 2^24, 1.5 2^52), rounded
// once, is 1.5 2^52 + rint(v 2^24) for |v| < 2^27, and its bit pattern minus
// that of 1.5 2^52 is the integer hi = rint(v 2^24) (1.5 2^52 is even, so
// ties still go to even).  The remainder r = v 2^24 - hi is exact (one more
// fma), and lo = rint(r 2^36) comes out the same way.  hi 2^36 + lo =
// rint(v 2^60), because hi 2^36 is an even integer and so shifts neither the
// rounding nor its ties.  Zero contributions (empty blocks) add nothing, and
// hi is added only when it is non-zero.
// ---------------------------------------------------------------------------
using FxWord = unsigned long long;
constexpr double kFxHiScale = 16777216.0;                 // 2^24: units of hi
constexpr double kFxLoScale = 68719476736.0;              // 2^36: lo units per hi unit
constexpr long long kFxSplit = 1LL << 36;
constexpr double kFxHiUnit = 1.0 / 16777216.0;             // 2^-24
constexpr double kFxLoUnit = 1.0 / 1152921504606846976.0;  // 2^-60
constexpr double kFxMagic = 6755399441055744.0;            // 1.5 2^52

__device__ __forceinline__ void fx_add(FxWord *acc, size_t idx, double v)
{
    if (v == 0.0) return;
    const double a = fma(v, kFxHiScale, kFxMagic);   // 1.5 2^52 + hi
    const double h = a - kFxMagic;                   // hi, exact
    const double r = fma(v, kFxHiScale, -h);         // v 2^24 - hi, exact, |r| <= 1/2
    const double b = fma(r, kFxLoScale, kFxMagic);   // 1.5 2^52 + lo, |lo| <= 2^35
    FxWord *p = acc + 2 * idx;
    if (h != 0.0) atomicAdd(p, (FxWord)(__double_as_longlong(a) - __double_as_longlong(kFxMagic)));
    atomicAdd(p + 1, (FxWord)(__double_as_longlong(b) - __double_as_longlong(kFxMagic)));
}

// Value of an accumulated (hi, lo) word pair: lo's multiples of 2^36 move
// into hi, so both parts convert to double exactly and one rounding remains.
__host__ __device__ __forceinline__ double fx_value(long long hi, long long lo)
{
    const long long rem = lo & (kFxSplit - 1);   // in [0, 2^36)
    const long long carry = (lo - rem) / kFxSplit;
    return (double)(hi + carry) * kFxHiUnit + (double)rem * kFxLoUnit;
}

// Contribution of one canonical AO quartet to the J/K accumulators:
// Jacc(i,j) += s v Pj(k,l), Jacc(k,l) += s v Pj(i,j),
// Kacc(i,k) += s v Pk(j,l), Kacc(j,k) += s v Pk(i,l),
// Kacc(i,l) += s v Pk(j,k), Kacc(j,l) += s v Pk(i,k);
// J = 2 (Jacc + Jacc^T), K = Kacc + Kacc^T.  This is the sum over the
// distinct members of the 8-fold permutation orbit that the reference
// writes into its tensor (os.cpp:137-163) and then contracts
// (os.cpp:1514-1520), with s = 1/|stabiliser| removing the duplicates.

// 8-fold scatter of one AO quartet into a dense tensor (os.cpp:137-163).
__device__ __forceinline__ void scatter8(double *eri, int nb, int i, int j, int k, int l, double v)
{
    const size_t n = nb, n2 = n * n, n3 = n2 * n;
    eri[i * n3 + j * n2 + k * n + l] = v;
    eri[j * n3 + i * n2 + k * n + l] = v;
    eri[i * n3 + j * n2 + l * n + k] = v;
    eri[j * n3 + i * n2 + l * n + k] = v;
    eri[k * n3 + l * n2 + i * n + j] = v;
    eri[l * n3 + k * n2 + i * n + j] = v;
    eri[k * n3 + l * n2 + j * n + i] = v;
    eri[l * n3 + k * n2 + j * n + i] = v;
}

}  // namespace pfk
