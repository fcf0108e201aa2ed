// pfk_os.cuh -- Obara-Saika engine: the reference's OS path (os.cpp:618-924,
// _eri_vrr + _eri_hrr_ab + _os_eri_primitive) restated per shell quartet.
//
// The reference runs the vertical recurrence once per Cartesian component
// quartet and primitive, then a horizontal recurrence.  Here one thread owns
// a whole shell quartet of class (LA LB | LC LD), L = LA+LB+LC+LD <= 4:
//   * Boys values F_0..F_L (boys_fm) in registers, from a Taylor series for
//     small T and from erf/exp with upward recursion otherwise -- no table
//     reads, so these kernels do not compete for L1 with the Rys tables;
//   * the vertical recurrence (Obara-Saika / Head-Gordon-Pople form) builds
//     [e0|f0] for e in [LA, LA+LB], f in [LC, LC+LD] per primitive quartet
//     and accumulates them contracted;
//   * the horizontal recurrences (ab| = (a+1 b-1| + AB (a b-1| and the same
//     on the ket run once per shell quartet on the contracted values;
//   * the J/K digestion is the one the Rys register path uses.
#pragma once
#include <type_traits>

#include "pfk_kernels.cuh"

namespace pfk {

// Cartesian component index of exponents (x, y, z), the inverse of
// cart_lx/ly/lz (lx descending, then ly descending).
__host__ __device__ constexpr int cart_index(int x, int y, int z)
{
    return (y + z) * (y + z + 1) / 2 + z;
}
__host__ __device__ constexpr int cart_l(int L, int i, int axis)
{
    return axis == 0 ? cart_lx(L, i) : axis == 1 ? cart_ly(L, i) : cart_lz(L, i);
}
// First axis with a non-zero exponent: the direction the recurrences step in.
__host__ __device__ constexpr int cart_dir(int L, int i)
{
    return cart_lx(L, i) > 0 ? 0 : cart_ly(L, i) > 0 ? 1 : 2;
}
// Index of component i of shell L with exponent `axis` changed by `delta`.
__host__ __device__ constexpr int cart_step(int L, int i, int axis, int delta)
{
    return cart_index(cart_lx(L, i) + (axis == 0 ? delta : 0), cart_ly(L, i) + (axis == 1 ? delta : 0),
                      cart_lz(L, i) + (axis == 2 ? delta : 0));
}

// Taylor coefficient (-1)^k / (k! (2M + 2k + 1)) of F_M(T).
__host__ __device__ constexpr double boys_series_coef(int M, int k)
{
    double f = 1.0;
    for (int j = 2; j <= k; ++j) f *= j;
    return (k % 2 ? -1.0 : 1.0) / (f * (2 * M + 2 * k + 1));
}

// The series coefficients as a constant-memory table: the FMAs of the series
// then read them as constant-bank operands instead of materialising each
// 64-bit literal in registers.
struct BoysSeriesTable {
    double c[7][32];
};
__host__ __device__ constexpr BoysSeriesTable make_boys_series_table()
{
    BoysSeriesTable t{};
    for (int M = 0; M < 7; ++M)
        for (int k = 0; k < 32; ++k) t.c[M][k] = boys_series_coef(M, k);
    return t;
}
static __constant__ const BoysSeriesTable kBoysSeries = make_boys_series_table();

// Boys function F_m(T), m = 0..M (M <= 6).  T below TS: the Taylor series of
// F_M and downward recursion F_m = (2T F_{m+1} + e^-T) / (2m+1), which is
// stable.  T >= TS: F_0 = sqrt(pi)/2 erf(sqrt T)/sqrt T (with erf(sqrt T) =
// 1 - e^-T erfcx(sqrt T), so one exponential serves all m) and the upward
// recursion F_{m+1} = ((2m+1) F_m - e^-T) / (2T); its error growth stays
// below ~10x for m <= 4 at T >= 2 (~2x for m <= 1 at T >= 1; TS = 3 for
// m = 5, 6).  T >= TA: the large-T limit F_0 = sqrt(pi / 4T), F_{m+1} =
// (2m+1) F_m / (2T), with no erf or exp; TA = 34, 38, 42, 44, 46 for
// M = 0..4 is where the limit's relative error (the dropped e^-T terms)
// falls to its own rounding level against 40-digit values, 60 above M = 4.
// Measured against 40-digit values: max relative error 1e-15 (M <= 1),
// 8e-15 (M = 4), 2e-14 (M = 6).
template <int M>
__device__ __forceinline__ void boys_fm(double T, double *F)
{
    constexpr double TS = M <= 1 ? 1.0 : M <= 4 ? 2.0 : 3.0;
    constexpr int NT = M <= 1 ? 18 : M <= 4 ? 25 : 32;   // terms: last term < 1e-17 at T = TS
    constexpr double TA = M == 0 ? 34.0 : M == 1 ? 38.0 : M == 2 ? 42.0 : M == 3 ? 44.0 : M == 4 ? 46.0 : 60.0;
    if (T < TS) {
        double s = kBoysSeries.c[M][NT - 1];
#pragma unroll
        for (int k = NT - 2; k >= 0; --k) s = fma(s, T, kBoysSeries.c[M][k]);
        F[M] = s;
        if constexpr (M > 0) {
            const double e = exp(-T);
#pragma unroll
            for (int m = M - 1; m >= 0; --m) F[m] = fma(2.0 * T, F[m + 1], e) * (1.0 / (2 * m + 1));
        }
    } else if (T < TA) {
        // erf(sqrt T) = 1 - e^-T erfcx(sqrt T): one exponential serves both
        // F_0 and the recursion (erfc(sqrt T) <= erfc(1) = 0.16, no cancellation)
        const double ist = rsqrt(T);
        const double e = exp(-T);
        F[0] = 0.88622692545275801365 * fma(-e, erfcx(T * ist), 1.0) * ist;   // sqrt(pi)/2
        if constexpr (M > 0) {
            const double h = 0.5 * ist * ist;                     // 1/(2T)
#pragma unroll
            for (int m = 0; m < M; ++m) F[m + 1] = fma(double(2 * m + 1), F[m], -e) * h;
        }
    } else {
        // erfc(sqrt T) and e^-T are below 1e-17 of every (2m+1) F_m here
        const double ist = rsqrt(T);
        F[0] = 0.88622692545275801365 * ist;
        const double h = 0.5 * ist * ist;
#pragma unroll
        for (int m = 0; m < M; ++m) F[m + 1] = double(2 * m + 1) * h * F[m];
    }
}

// Index bookkeeping of one class (all constexpr).
template <int LA, int LB, int LC, int LD>
struct OSShape {
    static constexpr int E = LA + LB, F = LC + LD, L = E + F;
    // bra-only values [a0|00]^(m): la <= E, m <= L - la
    __host__ __device__ static constexpr int aoff(int la)
    {
        int o = 0;
        for (int l = 0; l < la; ++l) o += ncart(l) * (L - l + 1);
        return o;
    }
    // ket level lc >= 1 keeps la in [lo(lc), E] and m in [0, F - lc]
    __host__ __device__ static constexpr int lo(int lc) { return LA - (F - lc) > 0 ? LA - (F - lc) : 0; }
    __host__ __device__ static constexpr int rowoff(int lc, int la)
    {
        int o = 0;
        for (int l = lo(lc); l < la; ++l) o += ncart(l);
        return o;
    }
    __host__ __device__ static constexpr int level_size(int lc) { return rowoff(lc, E + 1) * ncart(lc) * (F - lc + 1); }
    __host__ __device__ static constexpr int koff(int lc)
    {
        int o = aoff(E + 1);
        for (int l = 1; l < lc; ++l) o += level_size(l);
        return o;
    }
    static constexpr int NV = koff(F + 1);
    __host__ __device__ static constexpr int vi(int lc, int la, int ia, int ic, int m)
    {
        return lc == 0 ? aoff(la) + ia * (L - la + 1) + m
                       : koff(lc) + (rowoff(lc, la) + ia) * (ncart(lc) * (F - lc + 1)) + ic * (F - lc + 1) + m;
    }
    // contracted [e0|f0]: rows (la in [LA, E], ia), columns (lc in [LC, F], ic)
    __host__ __device__ static constexpr int row(int la)
    {
        int o = 0;
        for (int l = LA; l < la; ++l) o += ncart(l);
        return o;
    }
    __host__ __device__ static constexpr int col(int lc)
    {
        int o = 0;
        for (int l = LC; l < lc; ++l) o += ncart(l);
        return o;
    }
    static constexpr int NROW = row(E + 1), NCOL = col(F + 1), NACC = NROW * NCOL;
};

// Compile-time loop: fn(std::integral_constant<int, I>{}) for I = B .. E-1,
// so that every index computed inside is a constant expression.
template <int B, int E, typename Fn>
__device__ __forceinline__ void static_for(Fn &&fn)
{
    if constexpr (B < E) {
        fn(std::integral_constant<int, B>{});
        static_for<B + 1, E>(fn);
    }
}
#define PFK_CI(x) decltype(x)::value

// Vertical recurrence of one primitive quartet, added into the contracted
// [e0|f0] accumulator.  F0m[m] = 2 sqrt(rho/pi) K_ab K_cd F_m(T).
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void os_vrr(const double *F0m, const PrimPair &p, const PrimPair &q,
                                       const QuartetScalars &s, R *__restrict__ acc)
{
    using O = OSShape<LA, LB, LC, LD>;
    constexpr int E = O::E, F = O::F, L = O::L;
    R v[O::NV];
    const R PA[3] = {R(p.PAx), R(p.PAy), R(p.PAz)};
    const R QC[3] = {R(q.PAx), R(q.PAy), R(q.PAz)};
    const R WP[3] = {R(s.WPx), R(s.WPy), R(s.WPz)};
    const R WQ[3] = {R(s.WQx), R(s.WQy), R(s.WQz)};
    const R h_z = R(0.5 * s.zinv), h_e = R(0.5 * s.einv), h_ze = R(0.5 * s.rdelta);
    const R r_z = R(s.rho * s.zinv), r_e = R(s.rho * s.einv);      // rho/zeta, rho/eta
    static_for<0, L + 1>([&](auto m_) {
        constexpr int m = PFK_CI(m_);
        v[O::vi(0, 0, 0, 0, m)] = R(F0m[m]);
    });
    // bra: [a|00]^(m) = PA_d [a-1]^(m) + WP_d [a-1]^(m+1) + (a_d-1)/(2 zeta) ([a-2]^(m) - rho/zeta [a-2]^(m+1))
    static_for<1, E + 1>([&](auto la_) {
        constexpr int la = PFK_CI(la_);
        static_for<0, ncart(la)>([&](auto ia_) {
            constexpr int ia = PFK_CI(ia_);
            constexpr int d = cart_dir(la, ia), ad = cart_l(la, ia, d), ip = cart_step(la, ia, d, -1);
            static_for<0, L - la + 1>([&](auto m_) {
                constexpr int m = PFK_CI(m_);
                constexpr int i0 = O::vi(0, la - 1, ip, 0, m), i1 = O::vi(0, la - 1, ip, 0, m + 1);
                R x = PA[d] * v[i0] + WP[d] * v[i1];
                if constexpr (ad >= 2) {
                    constexpr int ig = cart_step(la - 1, ip, d, -1);
                    constexpr int g0 = O::vi(0, la - 2, ig, 0, m), g1 = O::vi(0, la - 2, ig, 0, m + 1);
                    x += R(ad - 1) * h_z * (v[g0] - r_z * v[g1]);
                }
                v[O::vi(0, la, ia, 0, m)] = x;
            });
        });
    });
    // ket: [a|c]^(m) = QC_d [a|c-1]^(m) + WQ_d [a|c-1]^(m+1)
    //                + (c_d-1)/(2 eta) ([a|c-2]^(m) - rho/eta [a|c-2]^(m+1))
    //                + a_d/(2(zeta+eta)) [a-1|c-1]^(m+1)
    static_for<1, F + 1>([&](auto lc_) {
        constexpr int lc = PFK_CI(lc_);
        static_for<O::lo(lc), E + 1>([&](auto la_) {
            constexpr int la = PFK_CI(la_);
            static_for<0, ncart(la)>([&](auto ia_) {
                constexpr int ia = PFK_CI(ia_);
                static_for<0, ncart(lc)>([&](auto ic_) {
                    constexpr int ic = PFK_CI(ic_);
                    constexpr int d = cart_dir(lc, ic), cd = cart_l(lc, ic, d), ad = cart_l(la, ia, d);
                    constexpr int cp = cart_step(lc, ic, d, -1);
                    static_for<0, F - lc + 1>([&](auto m_) {
                        constexpr int m = PFK_CI(m_);
                        constexpr int i0 = O::vi(lc - 1, la, ia, cp, m), i1 = O::vi(lc - 1, la, ia, cp, m + 1);
                        R x = QC[d] * v[i0] + WQ[d] * v[i1];
                        if constexpr (cd >= 2) {
                            constexpr int cg = cart_step(lc - 1, cp, d, -1);
                            constexpr int g0 = O::vi(lc - 2, la, ia, cg, m), g1 = O::vi(lc - 2, la, ia, cg, m + 1);
                            x += R(cd - 1) * h_e * (v[g0] - r_e * v[g1]);
                        }
                        if constexpr (ad >= 1) {
                            constexpr int am = cart_step(la, ia, d, -1);
                            constexpr int a1 = O::vi(lc - 1, la - 1, am, cp, m + 1);
                            x += R(ad) * h_ze * v[a1];
                        }
                        v[O::vi(lc, la, ia, ic, m)] = x;
                    });
                });
            });
        });
    });
    static_for<LA, E + 1>([&](auto la_) {
        constexpr int la = PFK_CI(la_);
        static_for<0, ncart(la)>([&](auto ia_) {
            constexpr int ia = PFK_CI(ia_);
            static_for<LC, F + 1>([&](auto lc_) {
                constexpr int lc = PFK_CI(lc_);
                static_for<0, ncart(lc)>([&](auto ic_) {
                    constexpr int ic = PFK_CI(ic_);
                    constexpr int k = (O::row(la) + ia) * O::NCOL + O::col(lc) + ic, src = O::vi(lc, la, ia, ic, 0);
                    acc[k] += v[src];
                });
            });
        });
    });
}

// Horizontal recurrences on the contracted [e0|f0] block: bra
// (a, b+1_d| = (a+1_d, b| + AB_d (a, b|, then the same on the ket with CD.
// out is the (ia, ib, ic, id) block of the class.
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void os_hrr(const R *__restrict__ acc, const R AB[3], const R CD[3], R *__restrict__ out)
{
    using O = OSShape<LA, LB, LC, LD>;
    constexpr int E = O::E, F = O::F, NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr int NCOL = O::NCOL;
    R x[NA * NB * NCOL];
    // bra, per ket column: hb[lb][la - LA][ia][ib] for la <= E - lb
    static_for<0, NCOL>([&](auto cc_) {
        constexpr int cc = PFK_CI(cc_);
        R hb[LB + 1][E - LA + 1][ncart(E)][ncart(LB)];
        static_for<LA, E + 1>([&](auto la_) {
            constexpr int la = PFK_CI(la_);
            static_for<0, ncart(la)>([&](auto ia_) {
                constexpr int ia = PFK_CI(ia_);
                hb[0][la - LA][ia][0] = acc[(O::row(la) + ia) * NCOL + cc];
            });
        });
        static_for<0, LB>([&](auto lb_) {
            constexpr int lb = PFK_CI(lb_);
            static_for<LA, E - lb>([&](auto la_) {
                constexpr int la = PFK_CI(la_);
                static_for<0, ncart(la)>([&](auto ia_) {
                    constexpr int ia = PFK_CI(ia_);
                    static_for<0, ncart(lb + 1)>([&](auto ib_) {
                        constexpr int ib = PFK_CI(ib_);
                        constexpr int d = cart_dir(lb + 1, ib), bp = cart_step(lb + 1, ib, d, -1);
                        constexpr int au = cart_step(la, ia, d, +1);
                        hb[lb + 1][la - LA][ia][ib] = hb[lb][la + 1 - LA][au][bp] + AB[d] * hb[lb][la - LA][ia][bp];
                    });
                });
            });
        });
        static_for<0, NA * NB>([&](auto ab_) {
            constexpr int ab = PFK_CI(ab_);
            x[ab * NCOL + cc] = hb[LB][0][ab / NB][ab % NB];
        });
    });
    // ket, per bra component pair
    static_for<0, NA * NB>([&](auto ab_) {
        constexpr int ab = PFK_CI(ab_);
        R hk[LD + 1][F - LC + 1][ncart(F)][ncart(LD)];
        static_for<LC, F + 1>([&](auto lc_) {
            constexpr int lc = PFK_CI(lc_);
            static_for<0, ncart(lc)>([&](auto ic_) {
                constexpr int ic = PFK_CI(ic_);
                hk[0][lc - LC][ic][0] = x[ab * NCOL + O::col(lc) + ic];
            });
        });
        static_for<0, LD>([&](auto ld_) {
            constexpr int ld = PFK_CI(ld_);
            static_for<LC, F - ld>([&](auto lc_) {
                constexpr int lc = PFK_CI(lc_);
                static_for<0, ncart(lc)>([&](auto ic_) {
                    constexpr int ic = PFK_CI(ic_);
                    static_for<0, ncart(ld + 1)>([&](auto id_) {
                        constexpr int id = PFK_CI(id_);
                        constexpr int d = cart_dir(ld + 1, id), dp = cart_step(ld + 1, id, d, -1);
                        constexpr int cu = cart_step(lc, ic, d, +1);
                        hk[ld + 1][lc - LC][ic][id] = hk[ld][lc + 1 - LC][cu][dp] + CD[d] * hk[ld][lc - LC][ic][dp];
                    });
                });
            });
        });
        static_for<0, NC * ND>([&](auto cd_) {
            constexpr int cd = PFK_CI(cd_);
            out[ab * NC * ND + cd] = hk[LD][0][cd / ND][cd % ND];
        });
    });
}

// One thread per shell quartet of an L <= 4 class, Obara-Saika integrals.
// R as in eri_reg_kernel: double, or float for the FP32 list (the Boys
// values and the per-primitive scalars stay FP64).  MINB: blocks of 128 per
// SM the register allocation must allow (1: the compiler's choice; the
// denser build of each class asks for 8, 6 or 4, at most 64, 80 or 128
// registers, for the autotuner to weigh occupancy against spills).
template <int LA, int LB, int LC, int LD, int NK, typename R = double, int MINB = 1>
__global__ void __launch_bounds__(128, MINB) eri_os_kernel(const uint2 *__restrict__ quartets, long long nq, JKArgs args)
{
    using O = OSShape<LA, LB, LC, LD>;
    constexpr int L = O::L;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    // lanes without a quartet stay with an empty primitive loop and a zero
    // block (finish_block needs the whole warp); a warp with none leaves
    const bool in_list = t < nq;
    if (!__any_sync(0xffffffffu, in_list)) return;
    const uint2 qd = quartets[(in_list ? t : nq - 1) * args.qstride + args.qoffset];
    const PairInfo pb = args.pairs[qd.x];
    const PairInfo pk = args.pairs[qd.y];
    const bool live = in_list && !density_negligible(pb, pk, args);

    R acc[O::NACC];
#pragma unroll
    for (int c = 0; c < O::NACC; ++c) acc[c] = R(0);
    // Primitive loops, ket outer (the lanes of a warp mostly share the bra
    // pair, so bra loads are broadcasts).  Loading the next bra primitive
    // ahead of the current one was measured slower: its registers cost more
    // occupancy than the latency it hides.
    const double qb0 = pb.nprim ? __ldg(&args.prims[pb.prim_off].qp) : 0.0;   // largest bra qp
    const int nket = live ? pk.nprim : 0;
    for (int jp = 0; jp < nket; ++jp) {
        const PrimPair q = load_prim(args.prims, pk.prim_off + jp);
        if (q.qp * qb0 < args.ptol) break;   // kets sorted by qp
        for (int ip = 0; ip < pb.nprim; ++ip) {
            const PrimPair p = load_prim(args.prims, pb.prim_off + ip);
            if (p.qp * q.qp < args.ptol) break;   // bras sorted by qp
            const QuartetScalars s = quartet_scalars(p, q);
            double Fm[L + 1];
            boys_fm<L>(s.T, Fm);
#pragma unroll
            for (int m = 0; m <= L; ++m) Fm[m] *= s.pref;
            os_vrr<LA, LB, LC, LD, R>(Fm, p, q, s, acc);
        }
    }
    constexpr int N = ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD);
    R blk[N];
    const R AB[3] = {R(pb.ABx), R(pb.ABy), R(pb.ABz)};
    const R CD[3] = {R(pk.ABx), R(pk.ABy), R(pk.ABz)};
    os_hrr<LA, LB, LC, LD, R>(acc, AB, CD, blk);
    finish_block<LA, LB, LC, LD, NK, R>(blk, qd, pb, pk, args, live, t);
}

}  // namespace pfk
