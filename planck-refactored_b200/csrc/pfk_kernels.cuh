// pfk_kernels.cuh -- per-angular-momentum-class ERI + J/K kernels.
//
// A class is (LA LB | LC LD) with LA >= LB, LC >= LD and (LA,LB) >= (LC,LD)
// in pair-class order; 55 classes cover (ss|ss)..(ff|ff).  Each kernel walks
// a list of screened shell quartets (bra pair, ket pair) of its class.
//
//   eri_reg_kernel   one thread per shell quartet; the contracted Cartesian
//                    block, the per-root axis tables and the J/K partial
//                    sums all live in registers.  Used for small classes.
//   eri_split_kernel a team of lanes per shell quartet sharing per-root
//                    tables in shared memory; each lane owns A-component
//                    slices of the block.  Larger classes.
//   eri_team_kernel  a team of TEAM threads (a warp or the whole block) per
//                    shell quartet; the per-root axis tables are built once
//                    per primitive quartet into shared memory and every
//                    thread accumulates a strided slice of the components.
#pragma once
#include "pfk_device.cuh"

namespace pfk {

template <int LA, int LB, int LC, int LD>
struct ClassShape {
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int N = NA * NB * NC * ND;
    static constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
    static constexpr int NI = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
    // offsets of component (ia, ib, ic, id) in the per-axis tables
    __host__ __device__ static constexpr int ax(int ia, int ib, int ic, int id)
    {
        return ((cart_lx(LA, ia) * (LB + 1) + cart_lx(LB, ib)) * (LC + 1) + cart_lx(LC, ic)) * (LD + 1) + cart_lx(LD, id);
    }
    __host__ __device__ static constexpr int ay(int ia, int ib, int ic, int id)
    {
        return ((cart_ly(LA, ia) * (LB + 1) + cart_ly(LB, ib)) * (LC + 1) + cart_ly(LC, ic)) * (LD + 1) + cart_ly(LD, id);
    }
    __host__ __device__ static constexpr int az(int ia, int ib, int ic, int id)
    {
        return ((cart_lz(LA, ia) * (LB + 1) + cart_lz(LB, ib)) * (LC + 1) + cart_lz(LC, ic)) * (LD + 1) + cart_lz(LD, id);
    }
    __host__ __device__ static constexpr double norm(int ia, int ib, int ic, int id)
    {
        return cart_norm(LA, ia) * cart_norm(LB, ib) * cart_norm(LC, ic) * cart_norm(LD, id);
    }
};

// Density screening of a whole shell quartet: every J and K contribution
// is a density block (kl, ij, jl, il, jk or ik) times integrals bounded by
// qmax(ij) qmax(kl).
__device__ __forceinline__ bool density_negligible(const PairInfo &pb, const PairInfo &pk, const JKArgs &a)
{
    if (!a.Dsh) return false;
    const size_t nb = a.nb;
    const int i = pb.bf_a, j = pb.bf_b, k = pk.bf_a, l = pk.bf_b;
    const float d = fmaxf(fmaxf(fmaxf(__ldg(a.Dsh + k * nb + l), __ldg(a.Dsh + i * nb + j)),
                                fmaxf(__ldg(a.Dsh + j * nb + l), __ldg(a.Dsh + i * nb + l))),
                          fmaxf(__ldg(a.Dsh + j * nb + k), __ldg(a.Dsh + i * nb + k)));
    return pb.qmax * pk.qmax * (double)d < a.dtol;
}

// Canonical-quartet bookkeeping for one Cartesian component quartet.
// Returns the weight s (0 when the component is a duplicate or screened out).
__device__ __forceinline__ double quartet_weight(bool same_ab, bool same_cd, bool same_bk, int ia, int ib,
                                                 int ic, int id, int NBc, int NDc, bool check,
                                                 const double *__restrict__ Qao, int nb, int i, int j,
                                                 int k, int l, double tol)
{
    double s = 1.0;
    if (same_ab) {
        if (ia > ib) return 0.0;
        if (ia == ib) s *= 0.5;
    }
    if (same_cd) {
        if (ic > id) return 0.0;
        if (ic == id) s *= 0.5;
    }
    if (same_bk) {
        const int pb = ia * NBc + ib, pk = ic * NDc + id;
        if (pb > pk) return 0.0;
        if (pb == pk) s *= 0.5;
    }
    if (check && __ldg(Qao + (size_t)i * nb + j) * __ldg(Qao + (size_t)k * nb + l) < tol) return 0.0;
    return s;
}


// J/K digestion of one weighted Cartesian block v (index ((ia*NB+ib)*NC+ic)*ND+id),
// one output block at a time so that only that block's density values and
// partial sums are live next to v:
//   J(i,j) += sum_kl v P(k,l)     J(k,l) += sum_ij v P(i,j)
//   K(i,k) += sum_jl v Pk(j,l)    K(j,k) += sum_il v Pk(i,l)
//   K(i,l) += sum_jk v Pk(j,k)    K(j,l) += sum_ik v Pk(i,k)
// (J = 2 (Jacc + Jacc^T) and K = Kacc + Kacc^T afterwards.)
// lead >= 0: every live lane of the warp digests a quartet of this same bra
// block (the others hold zero blocks), so the J(i,j) sums are first added
// across the warp and lane `lead` (the first live lane) issues each add
// instead of 32 lanes hitting the same address; lead < 0: each lane adds.
// SKIP: blocks the caller has already added (kSkipJij, kSkipJkl, kSkipKjk,
// kSkipKjl bits).
constexpr int kSkipJij = 1, kSkipJkl = 2, kSkipKjk = 4, kSkipKjl = 8;
template <int NA, int NB, int NC, int ND, int NK, int SKIP = 0, typename V>
__device__ __forceinline__ void digest_blocks(const V *v, int i0, int j0, int k0, int l0, const JKArgs &args,
                                              int lead = -1)
{
    const int nb = args.nb;
#define PFK_V(ia, ib, ic, id) double(v[(((ia) * NB + (ib)) * NC + (ic)) * ND + (id)])
    if constexpr (!(SKIP & kSkipJij)) {
        double p[NC * ND];
#pragma unroll
        for (int ic = 0; ic < NC; ++ic)
#pragma unroll
            for (int id = 0; id < ND; ++id) p[ic * ND + id] = __ldg(args.Pj + (size_t)(k0 + ic) * nb + l0 + id);
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int ib = 0; ib < NB; ++ib) {
                double s = 0.0;
#pragma unroll
                for (int ic = 0; ic < NC; ++ic)
#pragma unroll
                    for (int id = 0; id < ND; ++id) s += PFK_V(ia, ib, ic, id) * p[ic * ND + id];
                if (lead >= 0) {
#pragma unroll
                    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                    if ((int)(threadIdx.x & 31) == lead) fx_add(args.Jacc, (size_t)(i0 + ia) * nb + j0 + ib, s);
                } else {
                    fx_add(args.Jacc, (size_t)(i0 + ia) * nb + j0 + ib, s);
                }
            }
    }
    asm volatile("" ::: "memory");
    if constexpr (!(SKIP & kSkipJkl)) {
        double p[NA * NB];
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int ib = 0; ib < NB; ++ib) p[ia * NB + ib] = __ldg(args.Pj + (size_t)(i0 + ia) * nb + j0 + ib);
#pragma unroll
        for (int ic = 0; ic < NC; ++ic)
#pragma unroll
            for (int id = 0; id < ND; ++id) {
                double s = 0.0;
#pragma unroll
                for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                    for (int ib = 0; ib < NB; ++ib) s += PFK_V(ia, ib, ic, id) * p[ia * NB + ib];
                fx_add(args.Jacc, (size_t)(k0 + ic) * nb + l0 + id, s);
            }
    }
#pragma unroll
    for (int m = 0; m < NK; ++m) {
        FxWord *Kacc = m == 0 ? args.Kacc0 : args.Kacc1;
        const double *__restrict__ Pk = m == 0 ? args.Pk0 : args.Pk1;
        if (!Kacc) continue;
        asm volatile("" ::: "memory");
        {   // K(i,k) from Pk(j,l)
            double p[NB * ND];
#pragma unroll
            for (int ib = 0; ib < NB; ++ib)
#pragma unroll
                for (int id = 0; id < ND; ++id) p[ib * ND + id] = __ldg(Pk + (size_t)(j0 + ib) * nb + l0 + id);
#pragma unroll
            for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                for (int ic = 0; ic < NC; ++ic) {
                    double s = 0.0;
#pragma unroll
                    for (int ib = 0; ib < NB; ++ib)
#pragma unroll
                        for (int id = 0; id < ND; ++id) s += PFK_V(ia, ib, ic, id) * p[ib * ND + id];
                    fx_add(Kacc, (size_t)(i0 + ia) * nb + k0 + ic, s);
                }
        }
        asm volatile("" ::: "memory");
        if constexpr (!(SKIP & kSkipKjk)) {   // K(j,k) from Pk(i,l)
            double p[NA * ND];
#pragma unroll
            for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                for (int id = 0; id < ND; ++id) p[ia * ND + id] = __ldg(Pk + (size_t)(i0 + ia) * nb + l0 + id);
#pragma unroll
            for (int ib = 0; ib < NB; ++ib)
#pragma unroll
                for (int ic = 0; ic < NC; ++ic) {
                    double s = 0.0;
#pragma unroll
                    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                        for (int id = 0; id < ND; ++id) s += PFK_V(ia, ib, ic, id) * p[ia * ND + id];
                    fx_add(Kacc, (size_t)(j0 + ib) * nb + k0 + ic, s);
                }
        }
        asm volatile("" ::: "memory");
        {   // K(i,l) from Pk(j,k)
            double p[NB * NC];
#pragma unroll
            for (int ib = 0; ib < NB; ++ib)
#pragma unroll
                for (int ic = 0; ic < NC; ++ic) p[ib * NC + ic] = __ldg(Pk + (size_t)(j0 + ib) * nb + k0 + ic);
#pragma unroll
            for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                for (int id = 0; id < ND; ++id) {
                    double s = 0.0;
#pragma unroll
                    for (int ib = 0; ib < NB; ++ib)
#pragma unroll
                        for (int ic = 0; ic < NC; ++ic) s += PFK_V(ia, ib, ic, id) * p[ib * NC + ic];
                    fx_add(Kacc, (size_t)(i0 + ia) * nb + l0 + id, s);
                }
        }
        asm volatile("" ::: "memory");
        if constexpr (!(SKIP & kSkipKjl)) {   // K(j,l) from Pk(i,k)
            double p[NA * NC];
#pragma unroll
            for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                for (int ic = 0; ic < NC; ++ic) p[ia * NC + ic] = __ldg(Pk + (size_t)(i0 + ia) * nb + k0 + ic);
#pragma unroll
            for (int ib = 0; ib < NB; ++ib)
#pragma unroll
                for (int id = 0; id < ND; ++id) {
                    double s = 0.0;
#pragma unroll
                    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                        for (int ic = 0; ic < NC; ++ic) s += PFK_V(ia, ib, ic, id) * p[ia * NC + ic];
                    fx_add(Kacc, (size_t)(j0 + ib) * nb + l0 + id, s);
                }
        }
    }
#undef PFK_V
}

// The first live lane when every live lane of the warp digests a quartet of
// the same bra pair (the J(i,j) sums can then be added across the warp
// first), else -1.  Every lane of the warp calls it, in kernels where one
// thread owns a quartet and no sub-warp barrier precedes it (lanes without a
// quartet pass live = false and carry a zero block), so the answer depends
// only on the lists, never on which lanes happen to be converged -- part of
// what keeps a build bitwise reproducible.
__device__ __forceinline__ int warp_bra_lead(bool live, unsigned bra)
{
    const unsigned lv = __ballot_sync(0xffffffffu, live);
    if (lv == 0u) return -1;
    const int lead = __ffs(lv) - 1;
    const unsigned lead_bra = __shfl_sync(0xffffffffu, bra, lead);
    return __all_sync(0xffffffffu, !live || bra == lead_bra) ? lead : -1;
}

// Weights (duplicate components, AO-level screening), component norms and
// J/K digestion of a contracted Cartesian block acc[((ia*NB+ib)*NC+ic)*ND+id]
// of one shell quartet (list entry t); in dense-tensor mode the block is
// scattered instead, in block mode written out.  Every lane of the warp calls
// it; lanes with live = false hold a zero block (their digestion adds
// nothing) and write nothing in the tensor and block modes.
template <int LA, int LB, int LC, int LD, int NK, typename R>
__device__ __forceinline__ void finish_block(R *acc, const uint2 qd, const PairInfo &pb, const PairInfo &pk,
                                             const JKArgs &args, bool live, long long t)
{
    using S = ClassShape<LA, LB, LC, LD>;
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND;
    if (args.blk_out) {
        if (!live) return;
        double *o = args.blk_out + (size_t)t * S::N;
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int ib = 0; ib < NB; ++ib)
#pragma unroll
                for (int ic = 0; ic < NC; ++ic)
#pragma unroll
                    for (int id = 0; id < ND; ++id) {
                        const int c = ((ia * NB + ib) * NC + ic) * ND + id;
                        o[c] = double(acc[c]) * S::norm(ia, ib, ic, id);
                    }
        return;
    }
    const int nb = args.nb;
    const int i0 = pb.bf_a, j0 = pb.bf_b, k0 = pk.bf_a, l0 = pk.bf_b;
    const bool same_ab = (i0 == j0), same_cd = (k0 == l0), same_bk = (qd.x == qd.y);
    const bool check = pb.qmin * pk.qmin < args.tol;

    if (args.eri_out) {
        if (!live) return;
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int ib = 0; ib < NB; ++ib)
#pragma unroll
                for (int ic = 0; ic < NC; ++ic)
#pragma unroll
                    for (int id = 0; id < ND; ++id) {
                        const int c = ((ia * NB + ib) * NC + ic) * ND + id;
                        const double sw = quartet_weight(same_ab, same_cd, same_bk, ia, ib, ic, id, NB, ND, check,
                                                         args.Qao, nb, i0 + ia, j0 + ib, k0 + ic, l0 + id, args.tol);
                        if (sw != 0.0)
                            scatter8(args.eri_out, nb, i0 + ia, j0 + ib, k0 + ic, l0 + id,
                                     double(acc[c]) * S::norm(ia, ib, ic, id));
                    }
        return;
    }

    // weights (duplicates, AO-level screening) and component norms, in place
#pragma unroll
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
        for (int ib = 0; ib < NB; ++ib)
#pragma unroll
            for (int ic = 0; ic < NC; ++ic)
#pragma unroll
                for (int id = 0; id < ND; ++id) {
                    const int c = ((ia * NB + ib) * NC + ic) * ND + id;
                    const double sw = quartet_weight(same_ab, same_cd, same_bk, ia, ib, ic, id, NB, ND, check,
                                                     args.Qao, nb, i0 + ia, j0 + ib, k0 + ic, l0 + id, args.tol);
                    acc[c] = acc[c] * R(sw * S::norm(ia, ib, ic, id));
                }
    // lanes of a warp usually share the bra pair (lists are bra-major)
    const int lead = warp_bra_lead(live, qd.x);
    digest_blocks<NA, NB, NC, ND, NK>(acc, i0, j0, k0, l0, args, lead);
}

// ---------------------------------------------------------------------------
// Register path
// ---------------------------------------------------------------------------
// R is the arithmetic type of the 2D integrals, the transfer relations, the
// product and the contraction: double, or float for the mixed-precision list
// of quartets whose Schwarz bound is below the FP32 threshold.  Roots,
// weights and the per-primitive-quartet scalars stay FP64 in both, and so
// does the J/K digestion and accumulation.
template <int LA, int LB, int LC, int LD, int NK, typename R = double>
__global__ void __launch_bounds__(128) eri_reg_kernel(const uint2 *__restrict__ quartets, long long nq, JKArgs args)
{
    using S = ClassShape<LA, LB, LC, LD>;
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND, NR = S::NR, NI = S::NI;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    // Lanes past the end of the list, or whose quartet the density screen
    // drops, stay with an empty primitive loop and a zero block (see
    // finish_block); a warp with no quartet at all leaves.
    const bool in_list = t < nq;
    if (!__any_sync(0xffffffffu, in_list)) return;
    const uint2 qd = quartets[(in_list ? t : nq - 1) * args.qstride + args.qoffset];
    const PairInfo pb = args.pairs[qd.x];
    const PairInfo pk = args.pairs[qd.y];
    const bool live = in_list && !density_negligible(pb, pk, args);

    R acc[NA * NB * NC * ND];
#pragma unroll
    for (int c = 0; c < S::N; ++c) acc[c] = R(0);

    // ket primitives outer: a warp's lanes usually share the bra pair, so the
    // inner loads of bra primitives are broadcasts
    const double qb0 = pb.nprim ? __ldg(&args.prims[pb.prim_off].qp) : 0.0;   // largest bra qp
    const int nket = live ? pk.nprim : 0;
    for (int jp = 0; jp < nket; ++jp) {
        const PrimPair q = load_prim(args.prims, pk.prim_off + jp);
        if (q.qp * qb0 < args.ptol) break;   // kets sorted by qp
        for (int ip = 0; ip < pb.nprim; ++ip) {
            const PrimPair p = load_prim(args.prims, pb.prim_off + ip);
            if (p.qp * q.qp < args.ptol) break;   // bras sorted by qp
            const QuartetScalars s = quartet_scalars(p, q);
            double u[NR], w[NR];
            rys_roots<NR>(s.T, u, w);
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const double ur = u[r];
                const double B00 = 0.5 * s.rdelta * ur;
                const double B10 = 0.5 * s.zinv * (1.0 - s.rho * s.zinv * ur);
                const double B01 = 0.5 * s.einv * (1.0 - s.rho * s.einv * ur);
                R gx[NI], gy[NI], gz[NI];
                axis_table<LA, LB, LC, LD, R>(R(p.PAx + ur * s.WPx), R(q.PAx + ur * s.WQx), R(B00), R(B10),
                                              R(B01), R(pb.ABx), R(pk.ABx), R(w[r] * s.pref), gx);
                axis_table<LA, LB, LC, LD, R>(R(p.PAy + ur * s.WPy), R(q.PAy + ur * s.WQy), R(B00), R(B10),
                                              R(B01), R(pb.ABy), R(pk.ABy), R(1), gy);
                axis_table<LA, LB, LC, LD, R>(R(p.PAz + ur * s.WPz), R(q.PAz + ur * s.WQz), R(B00), R(B10),
                                              R(B01), R(pb.ABz), R(pk.ABz), R(1), gz);
#pragma unroll
                for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                    for (int ib = 0; ib < NB; ++ib)
#pragma unroll
                        for (int ic = 0; ic < NC; ++ic)
#pragma unroll
                            for (int id = 0; id < ND; ++id) {
                                const int c = ((ia * NB + ib) * NC + ic) * ND + id;
                                acc[c] += gx[S::ax(ia, ib, ic, id)] * gy[S::ay(ia, ib, ic, id)] *
                                          gz[S::az(ia, ib, ic, id)];
                            }
            }
        }
    }

    finish_block<LA, LB, LC, LD, NK, R>(acc, qd, pb, pk, args, live, t);
}

// ---------------------------------------------------------------------------
// Team path (TEAM = 8: four quartets per warp; TEAM = 32: one warp per
// quartet; TEAM = 128: the whole block per quartet).
// ---------------------------------------------------------------------------
// BLOCK threads per block: 128, or 256 for the classes above 4000
// components ((ff|fd), (ff|ff)), whose 128-thread teams held 63..79
// accumulators per thread and spilled them.
template <int LA, int LB, int LC, int LD, typename R = double>
struct TeamShape {
    using S = ClassShape<LA, LB, LC, LD>;
    static constexpr int TEAM = S::N <= 400 ? 8 : S::N <= 1300 ? 32 : S::N <= 4000 ? 128 : 256;
    static constexpr int BLOCK = TEAM > 128 ? TEAM : 128;
    static constexpr int TEAMS = BLOCK / TEAM;
    static constexpr int KPT = (S::N + TEAM - 1) / TEAM;
    static constexpr int TABLE = S::NR * 3 * S::NI;          // R values per team
    static constexpr size_t SMEM = sizeof(R) * TABLE * TEAMS;
};

template <int TEAM>
__device__ __forceinline__ void team_sync(unsigned mask)
{
    if constexpr (TEAM <= 32) __syncwarp(mask);
    else __syncthreads();
}

// R: the arithmetic type of the axis tables, the products and the
// contraction (double, or float for the FP32 list); roots, weights and the
// per-primitive scalars stay FP64, the digestion FP64 with fixed-point sums.
template <int LA, int LB, int LC, int LD, int NK, typename R = double>
__global__ void __launch_bounds__(TeamShape<LA, LB, LC, LD, R>::BLOCK) eri_team_kernel(const uint2 *__restrict__ quartets,
                                                                                  long long nq, JKArgs args)
{
    using S = ClassShape<LA, LB, LC, LD>;
    using TS = TeamShape<LA, LB, LC, LD, R>;
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND, NR = S::NR, NI = S::NI;
    constexpr int TEAM = TS::TEAM, KPT = TS::KPT;
    extern __shared__ __align__(16) unsigned char pfk_dyn_smem[];
    R *smem = reinterpret_cast<R *>(pfk_dyn_smem);
    const int team = threadIdx.x / TEAM, lane = threadIdx.x % TEAM;
    const long long t = (long long)blockIdx.x * TS::TEAMS + team;
    // Teams within a warp synchronise only their own lanes, so a team may
    // leave early; the block-wide team has exactly one quartet per block.
    if (t >= nq) return;
    const unsigned mask = TEAM >= 32 ? 0xffffffffu
                                     : (((1u << TEAM) - 1u) << ((threadIdx.x & 31) / TEAM * TEAM));
    R *g = smem + team * TS::TABLE;   // g[r][axis][NI]

    const uint2 qd = quartets[t * args.qstride + args.qoffset];
    const PairInfo pb = args.pairs[qd.x];
    const PairInfo pk = args.pairs[qd.y];
    if (density_negligible(pb, pk, args)) return;   // whole quartet (team-uniform)

    int off[KPT];
    R acc[KPT];
#pragma unroll
    for (int k = 0; k < KPT; ++k) {
        acc[k] = R(0);
        const int c = lane + k * TEAM;
        if (c < S::N) {
            const int id = c % ND, ic = (c / ND) % NC, ib = (c / (ND * NC)) % NB, ia = c / (ND * NC * NB);
            const int ox = ((cart_lx(LA, ia) * (LB + 1) + cart_lx(LB, ib)) * (LC + 1) + cart_lx(LC, ic)) * (LD + 1) + cart_lx(LD, id);
            const int oy = ((cart_ly(LA, ia) * (LB + 1) + cart_ly(LB, ib)) * (LC + 1) + cart_ly(LC, ic)) * (LD + 1) + cart_ly(LD, id);
            const int oz = ((cart_lz(LA, ia) * (LB + 1) + cart_lz(LB, ib)) * (LC + 1) + cart_lz(LC, ic)) * (LD + 1) + cart_lz(LD, id);
            off[k] = ox | (oy << 10) | (oz << 20);
        } else {
            off[k] = 0;
        }
    }

    // ket primitives outer: a warp's lanes usually share the bra pair, so the
    // inner loads of bra primitives are broadcasts
    const double qb0 = pb.nprim ? __ldg(&args.prims[pb.prim_off].qp) : 0.0;   // largest bra qp
    for (int jp = 0; jp < pk.nprim; ++jp) {
        const PrimPair q = load_prim(args.prims, pk.prim_off + jp);
        if (q.qp * qb0 < args.ptol) break;   // kets sorted by qp
        for (int ip = 0; ip < pb.nprim; ++ip) {
            const PrimPair p = load_prim(args.prims, pb.prim_off + ip);
            if (p.qp * q.qp < args.ptol) break;   // bras sorted by qp
            const QuartetScalars s = quartet_scalars(p, q);
            for (int task = lane; task < 3 * NR; task += TEAM) {
                const int r = task / 3, axis = task - 3 * r;
                double ur, wr;
                rys_root_one<NR>(s.T, r, ur, wr);
                const double B00 = 0.5 * s.rdelta * ur;
                const double B10 = 0.5 * s.zinv * (1.0 - s.rho * s.zinv * ur);
                const double B01 = 0.5 * s.einv * (1.0 - s.rho * s.einv * ur);
                double C00, D00, AB, CD, scale = 1.0;
                if (axis == 0) { C00 = p.PAx + ur * s.WPx; D00 = q.PAx + ur * s.WQx; AB = pb.ABx; CD = pk.ABx; scale = wr * s.pref; }
                else if (axis == 1) { C00 = p.PAy + ur * s.WPy; D00 = q.PAy + ur * s.WQy; AB = pb.ABy; CD = pk.ABy; }
                else { C00 = p.PAz + ur * s.WPz; D00 = q.PAz + ur * s.WQz; AB = pb.ABz; CD = pk.ABz; }
                axis_table<LA, LB, LC, LD, R>(R(C00), R(D00), R(B00), R(B10), R(B01), R(AB), R(CD), R(scale),
                                              g + (r * 3 + axis) * NI);
            }
            team_sync<TEAM>(mask);
#pragma unroll
            for (int k = 0; k < KPT; ++k) {
                const int ox = off[k] & 1023, oy = (off[k] >> 10) & 1023, oz = off[k] >> 20;
                R a = acc[k];
#pragma unroll
                for (int r = 0; r < NR; ++r)
                    a += g[(r * 3 + 0) * NI + ox] * g[(r * 3 + 1) * NI + oy] * g[(r * 3 + 2) * NI + oz];
                acc[k] = a;
            }
            team_sync<TEAM>(mask);
        }
    }

    if (args.blk_out) {
#pragma unroll
        for (int k = 0; k < KPT; ++k) {
            const int c = lane + k * TEAM;
            if (c >= S::N) continue;
            const int id = c % ND, ic = (c / ND) % NC, ib = (c / (ND * NC)) % NB, ia = c / (ND * NC * NB);
            args.blk_out[(size_t)t * S::N + c] =
                double(acc[k]) * cart_norm(LA, ia) * cart_norm(LB, ib) * cart_norm(LC, ic) * cart_norm(LD, id);
        }
        return;
    }
    const int nb = args.nb;
    const int i0 = pb.bf_a, j0 = pb.bf_b, k0 = pk.bf_a, l0 = pk.bf_b;
    const bool same_ab = (i0 == j0), same_cd = (k0 == l0), same_bk = (qd.x == qd.y);
    const bool check = pb.qmin * pk.qmin < args.tol;
#pragma unroll
    for (int k = 0; k < KPT; ++k) {
        const int c = lane + k * TEAM;
        if (c >= S::N) continue;
        const int id = c % ND, ic = (c / ND) % NC, ib = (c / (ND * NC)) % NB, ia = c / (ND * NC * NB);
        const int i = i0 + ia, j = j0 + ib, kk = k0 + ic, l = l0 + id;
        const double sw = quartet_weight(same_ab, same_cd, same_bk, ia, ib, ic, id, NB, ND, check, args.Qao, nb,
                                         i, j, kk, l, args.tol);
        if (sw == 0.0) continue;
        const double v =
            double(acc[k]) * sw * cart_norm(LA, ia) * cart_norm(LB, ib) * cart_norm(LC, ic) * cart_norm(LD, id);
        if (args.eri_out) {
            scatter8(args.eri_out, nb, i, j, kk, l, v / sw);
            continue;
        }
        fx_add(args.Jacc, (size_t)i * nb + j, v * __ldg(args.Pj + (size_t)kk * nb + l));
        fx_add(args.Jacc, (size_t)kk * nb + l, v * __ldg(args.Pj + (size_t)i * nb + j));
#pragma unroll
        for (int m = 0; m < NK; ++m) {
            FxWord *Kacc = m == 0 ? args.Kacc0 : args.Kacc1;
            const double *__restrict__ Pk = m == 0 ? args.Pk0 : args.Pk1;
            if (!Kacc) continue;
            fx_add(Kacc, (size_t)i * nb + kk, v * __ldg(Pk + (size_t)j * nb + l));
            fx_add(Kacc, (size_t)j * nb + kk, v * __ldg(Pk + (size_t)i * nb + l));
            fx_add(Kacc, (size_t)i * nb + l, v * __ldg(Pk + (size_t)j * nb + kk));
            fx_add(Kacc, (size_t)j * nb + l, v * __ldg(Pk + (size_t)i * nb + kk));
        }
    }
}

// ---------------------------------------------------------------------------
// Schwarz diagonal (ab|ab) per shell pair of class (LA, LB): Q(i,j) for all
// component pairs (os.cpp:1703-1752, rys.cpp:509-556).
// ---------------------------------------------------------------------------
// Adds the diagonal (ab|ab) of one primitive quartet (p, q) of shell pair pb
// to acc[ia * NB + ib] (unnormalised Cartesian components).
template <int LA, int LB>
__device__ __forceinline__ void diag_add(const PrimPair &p, const PrimPair &q, const PairInfo &pb, double *acc)
{
    using S = ClassShape<LA, LB, LA, LB>;
    constexpr int NA = S::NA, NB = S::NB, NR = S::NR, NI = S::NI;
    const QuartetScalars s = quartet_scalars(p, q);
    double u[NR], w[NR];
    rys_roots<NR>(s.T, u, w);
    for (int r = 0; r < NR; ++r) {
        const double ur = u[r];
        const double B00 = 0.5 * s.rdelta * ur;
        const double B10 = 0.5 * s.zinv * (1.0 - s.rho * s.zinv * ur);
        const double B01 = 0.5 * s.einv * (1.0 - s.rho * s.einv * ur);
        double gx[NI], gy[NI], gz[NI];
        axis_table<LA, LB, LA, LB, double>(p.PAx + ur * s.WPx, q.PAx + ur * s.WQx, B00, B10, B01, pb.ABx, pb.ABx, w[r] * s.pref, gx);
        axis_table<LA, LB, LA, LB, double>(p.PAy + ur * s.WPy, q.PAy + ur * s.WQy, B00, B10, B01, pb.ABy, pb.ABy, 1.0, gy);
        axis_table<LA, LB, LA, LB, double>(p.PAz + ur * s.WPz, q.PAz + ur * s.WQz, B00, B10, B01, pb.ABz, pb.ABz, 1.0, gz);
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int ib = 0; ib < NB; ++ib)
                acc[ia * NB + ib] += gx[S::ax(ia, ib, ia, ib)] * gy[S::ay(ia, ib, ia, ib)] * gz[S::az(ia, ib, ia, ib)];
    }
}

template <int LA, int LB>
__global__ void __launch_bounds__(64) schwarz_kernel(const int *__restrict__ pair_ids, int n, const PairInfo *__restrict__ pairs,
                                                     const PrimPair *__restrict__ prims, double *Qao, int nb)
{
    constexpr int NA = ncart(LA), NB = ncart(LB);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const PairInfo pb = pairs[pair_ids[t]];
    double acc[NA * NB];
#pragma unroll
    for (int c = 0; c < NA * NB; ++c) acc[c] = 0.0;
    for (int ip = 0; ip < pb.nprim_full; ++ip) {
        const PrimPair p = load_prim(prims, pb.prim_off + ip);
        for (int jp = 0; jp < pb.nprim_full; ++jp) diag_add<LA, LB>(p, load_prim(prims, pb.prim_off + jp), pb, acc);
    }
#pragma unroll
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
        for (int ib = 0; ib < NB; ++ib) {
            const double nrm = cart_norm(LA, ia) * cart_norm(LB, ib);
            const double q = sqrt(fabs(acc[ia * NB + ib] * nrm * nrm));
            const int i = pb.bf_a + ia, j = pb.bf_b + ib;
            Qao[(size_t)i * nb + j] = q;
            Qao[(size_t)j * nb + i] = q;
        }
}

// Primitive Schwarz bound of every primitive pair of the listed shell pairs:
// prims[k].qp = max over components of sqrt|N_a^2 N_b^2 (ab|ab)| for
// primitive pair k alone (one thread per shell pair; the pairs' primitive
// ranges are disjoint).
template <int LA, int LB>
__global__ void __launch_bounds__(64) prim_bound_kernel(const int *__restrict__ pair_ids, int n,
                                                        const PairInfo *__restrict__ pairs, PrimPair *prims)
{
    constexpr int NA = ncart(LA), NB = ncart(LB);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const PairInfo pb = pairs[pair_ids[t]];
    for (int ip = 0; ip < pb.nprim_full; ++ip) {
        const PrimPair p = prims[pb.prim_off + ip];
        double acc[NA * NB];
#pragma unroll
        for (int c = 0; c < NA * NB; ++c) acc[c] = 0.0;
        diag_add<LA, LB>(p, p, pb, acc);
        double m = 0.0;
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int ib = 0; ib < NB; ++ib) {
                const double nrm = cart_norm(LA, ia) * cart_norm(LB, ib);
                m = fmax(m, fabs(acc[ia * NB + ib] * nrm * nrm));
            }
        prims[pb.prim_off + ip].qp = sqrt(m);
    }
}

}  // namespace pfk

namespace pfk {

// ---------------------------------------------------------------------------
// Split path for mid-size classes.  A team of GROUP threads shares one shell
// quartet: per primitive quartet the 3*NR per-root axis tables are built
// once (the team's lanes take the (root, axis) tasks) into shared memory;
// thread g then owns every Cartesian component whose leading index is g --
// the A component (LEVEL 1) or the (A, B) component pair (LEVEL 2) -- so it
// needs only the matching slice of each table, which it copies to registers
// once per root, and accumulates its M components in registers.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int pow2ceil(int x) { return x <= 1 ? 1 : 2 * pow2ceil((x + 1) / 2); }

template <int LA, int LB, int LC, int LD, typename R = double>
struct SplitShape {
    using S = ClassShape<LA, LB, LC, LD>;
    static constexpr int LEVEL = (S::NB * S::NC * S::ND <= 64) ? 1 : 2;
    static constexpr int GROUP = LEVEL == 1 ? S::NA : S::NA * S::NB;
    static constexpr int M = S::N / GROUP;                    // components per thread
    static constexpr int NBT = LEVEL == 1 ? S::NB : 1;        // B components per thread
    static constexpr int TEAM = pow2ceil(GROUP) < 4 ? 4 : pow2ceil(GROUP);
    static constexpr int TEAMS = 128 / TEAM;
    static constexpr int SB = LEVEL == 1 ? (LB + 1) * (LC + 1) * (LD + 1) : (LC + 1) * (LD + 1);
    // table strides: a slice a (LEVEL 1) or (a, b) (LEVEL 2) is read by
    // different lanes at once, so slices start an odd number of doubles
    // apart (no two of them on the same shared-memory bank pair)
    static constexpr int BST = LEVEL == 2 ? (LC + 1) * (LD + 1) + ((LC + 1) * (LD + 1) + 1) % 2 : (LC + 1) * (LD + 1);
    static constexpr int AST = LEVEL == 1 ? (LB + 1) * BST + ((LB + 1) * BST + 1) % 2 : (LB + 1) * BST;
    static constexpr int NIP = (LA + 1) * AST;                 // padded table per (root, axis)
    // R values per team: an odd number of 8-byte words, so the teams of a
    // warp start on different bank pairs and every team's table (and the
    // FP64 reduction staged in it) is 8-byte aligned
    static constexpr int RAW = S::NR * 3 * NIP;
    static constexpr int TABLE = sizeof(R) == 8 ? RAW + (RAW + 1) % 2
                                                : 2 * ((RAW + 1) / 2 + ((RAW + 1) / 2 + 1) % 2);
    static constexpr size_t SMEM = sizeof(R) * TABLE * TEAMS;
    // team reduction of the blocks every owner adds to the same elements of
    // (LEVEL 1: J(k,l), K(j,k), K(j,l)), staged in the team's table after the
    // primitive loop: REDV partial sums per owner per exchange density
    static constexpr int REDV1 = S::NC * S::ND, REDVK = S::NB * S::NC + S::NB * S::ND;
    template <int NK>
    __host__ __device__ static constexpr int redv() { return REDV1 + NK * REDVK; }
    static constexpr bool TEAMRED =
        LEVEL == 1 && TEAM <= 32 && (REDV1 + 2 * REDVK) * GROUP * 8 <= TABLE * (int)sizeof(R);
    static constexpr bool OK = TEAM <= 128 && M <= 64;
};

template <int TEAM>
__device__ __forceinline__ void split_sync(unsigned mask, int team)
{
    if constexpr (TEAM <= 32) {
        __syncwarp(mask);
    } else if constexpr (TEAM == 64) {
        asm volatile("bar.sync %0, 64;" ::"r"(team + 1) : "memory");
    } else {
        __syncthreads();
    }
}

// Component norm for a runtime component index (same values as cart_norm).
template <int L>
__device__ __forceinline__ double cart_norm_rt(int i)
{
    double v = 1.0;
#pragma unroll
    for (int c = 0; c < ncart(L); ++c)
        if (c == i) v = cart_norm(L, c);
    return v;
}

template <int L>
__device__ __forceinline__ int cart_l_axis(int i, int axis)
{
    return axis == 0 ? cart_lx(L, i) : axis == 1 ? cart_ly(L, i) : cart_lz(L, i);
}

// R: the arithmetic type of the shared tables, the slices, the products and
// the contraction (double, or float for the FP32 list of quartets whose
// Schwarz bound is below the FP32 threshold); roots, weights and the
// per-primitive scalars stay FP64, and so does the digestion.
template <int LA, int LB, int LC, int LD, int NK, typename R = double>
__global__ void __launch_bounds__(128, 3) eri_split_kernel(const uint2 *__restrict__ quartets, long long nq, JKArgs args)
{
    using S = ClassShape<LA, LB, LC, LD>;
    using SS = SplitShape<LA, LB, LC, LD, R>;
    constexpr int NB = S::NB, NC = S::NC, ND = S::ND, NR = S::NR;
    constexpr int TEAM = SS::TEAM, LEVEL = SS::LEVEL, NBT = SS::NBT, SB = SS::SB, M = SS::M;
    extern __shared__ __align__(16) unsigned char pfk_dyn_smem[];
    R *smem = reinterpret_cast<R *>(pfk_dyn_smem);
    const int team = threadIdx.x / TEAM, lane = threadIdx.x % TEAM;
    const long long t = (long long)blockIdx.x * SS::TEAMS + team;
    // Whole teams leave together; every barrier below is per team.  No
    // full-warp intrinsic follows: the teams of a warp run different
    // primitive loops, each synchronising only its own lanes.
    if (t >= nq) return;
    const unsigned mask = TEAM >= 32 ? 0xffffffffu
                                     : (((1u << TEAM) - 1u) << ((threadIdx.x & 31) / TEAM * TEAM));
    R *g = smem + team * SS::TABLE;   // g[r][axis][NIP]

    const uint2 qd = quartets[t * args.qstride + args.qoffset];
    const PairInfo pb = args.pairs[qd.x];
    const PairInfo pk = args.pairs[qd.y];
    if (density_negligible(pb, pk, args)) return;   // whole quartet (team-uniform)
    const bool owner = lane < SS::GROUP;
    const int gi = owner ? lane : 0;
    const int ia = LEVEL == 1 ? gi : gi / NB;
    const int ib0 = LEVEL == 1 ? 0 : gi % NB;
    // slice base of each axis table for this thread's leading indices
    int base[3];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        const int la = cart_l_axis<LA>(ia, x);
        base[x] = LEVEL == 1 ? la * SS::AST : la * SS::AST + cart_l_axis<LB>(ib0, x) * SS::BST;
    }

    R acc[M];
#pragma unroll
    for (int c = 0; c < M; ++c) acc[c] = R(0);

    // ket primitives outer: a warp's lanes usually share the bra pair, so the
    // inner loads of bra primitives are broadcasts
    const double qb0 = pb.nprim ? __ldg(&args.prims[pb.prim_off].qp) : 0.0;   // largest bra qp
    for (int jp = 0; jp < pk.nprim; ++jp) {
        const PrimPair q = load_prim(args.prims, pk.prim_off + jp);
        if (q.qp * qb0 < args.ptol) break;   // kets sorted by qp
        for (int ip = 0; ip < pb.nprim; ++ip) {
            const PrimPair p = load_prim(args.prims, pb.prim_off + ip);
            if (p.qp * q.qp < args.ptol) break;   // bras sorted by qp
            const QuartetScalars s = quartet_scalars(p, q);
            for (int task = lane; task < 3 * NR; task += TEAM) {
                const int r = task / 3, axis = task - 3 * r;
                double ur, wr;
                rys_root_one<NR>(s.T, r, ur, wr);
                const double B00 = 0.5 * s.rdelta * ur;
                const double B10 = 0.5 * s.zinv * (1.0 - s.rho * s.zinv * ur);
                const double B01 = 0.5 * s.einv * (1.0 - s.rho * s.einv * ur);
                double C00, D00, AB, CD, scale = 1.0;
                if (axis == 0) { C00 = p.PAx + ur * s.WPx; D00 = q.PAx + ur * s.WQx; AB = pb.ABx; CD = pk.ABx; scale = wr * s.pref; }
                else if (axis == 1) { C00 = p.PAy + ur * s.WPy; D00 = q.PAy + ur * s.WQy; AB = pb.ABy; CD = pk.ABy; }
                else { C00 = p.PAz + ur * s.WPz; D00 = q.PAz + ur * s.WQz; AB = pb.ABz; CD = pk.ABz; }
                axis_table<LA, LB, LC, LD, R, SS::BST, SS::AST>(R(C00), R(D00), R(B00), R(B10), R(B01), R(AB),
                                                                  R(CD), R(scale), g + (r * 3 + axis) * SS::NIP);
            }
            split_sync<TEAM>(mask, team);
            if (owner) {
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    R tx[SB], ty[SB], tz[SB];
#pragma unroll
                    for (int e = 0; e < SB; ++e) {
                        tx[e] = g[(r * 3 + 0) * SS::NIP + base[0] + e];
                        ty[e] = g[(r * 3 + 1) * SS::NIP + base[1] + e];
                        tz[e] = g[(r * 3 + 2) * SS::NIP + base[2] + e];
                    }
#pragma unroll
                    for (int bl = 0; bl < NBT; ++bl)
#pragma unroll
                        for (int ic = 0; ic < NC; ++ic)
#pragma unroll
                            for (int id = 0; id < ND; ++id) {
                                const int c = (bl * NC + ic) * ND + id;
                                int ox, oy, oz;
                                if constexpr (LEVEL == 1) {
                                    ox = (cart_lx(LB, bl) * (LC + 1) + cart_lx(LC, ic)) * (LD + 1) + cart_lx(LD, id);
                                    oy = (cart_ly(LB, bl) * (LC + 1) + cart_ly(LC, ic)) * (LD + 1) + cart_ly(LD, id);
                                    oz = (cart_lz(LB, bl) * (LC + 1) + cart_lz(LC, ic)) * (LD + 1) + cart_lz(LD, id);
                                } else {
                                    ox = cart_lx(LC, ic) * (LD + 1) + cart_lx(LD, id);
                                    oy = cart_ly(LC, ic) * (LD + 1) + cart_ly(LD, id);
                                    oz = cart_lz(LC, ic) * (LD + 1) + cart_lz(LD, id);
                                }
                                acc[c] += tx[ox] * ty[oy] * tz[oz];
                            }
                }
            }
            split_sync<TEAM>(mask, team);
        }
    }
    // ---- digestion of this thread's components: A index ia, B indices
    // ib0 .. ib0 + NBT - 1, all C and D.  Non-owner lanes hold a zero block
    // (ia = 0) and take part only in the team reduction. ----
    const int nb = args.nb;
    const int i0 = pb.bf_a, j0 = pb.bf_b, k0 = pk.bf_a, l0 = pk.bf_b;
    const bool same_ab = (i0 == j0), same_cd = (k0 == l0), same_bk = (qd.x == qd.y);
    const bool check = pb.qmin * pk.qmin < args.tol;
    const int i = i0 + ia;

    if (args.blk_out) {
        if (!owner) return;
#pragma unroll
        for (int bl = 0; bl < NBT; ++bl)
#pragma unroll
            for (int ic = 0; ic < NC; ++ic)
#pragma unroll
                for (int id = 0; id < ND; ++id) {
                    const int ib = ib0 + bl;
                    const double nrm = cart_norm_rt<LA>(ia) * cart_norm_rt<LB>(ib) * cart_norm(LC, ic) * cart_norm(LD, id);
                    args.blk_out[(size_t)t * S::N + ((ia * NB + ib) * NC + ic) * ND + id] =
                        double(acc[(bl * NC + ic) * ND + id]) * nrm;
                }
        return;
    }
    if (args.eri_out) {
        if (!owner) return;
#pragma unroll
        for (int bl = 0; bl < NBT; ++bl)
#pragma unroll
            for (int ic = 0; ic < NC; ++ic)
#pragma unroll
                for (int id = 0; id < ND; ++id) {
                    const int ib = ib0 + bl;
                    const double sw = quartet_weight(same_ab, same_cd, same_bk, ia, ib, ic, id, NB, ND, check, args.Qao,
                                                     nb, i, j0 + ib, k0 + ic, l0 + id, args.tol);
                    if (sw != 0.0) {
                        const double nrm = cart_norm_rt<LA>(ia) * cart_norm_rt<LB>(ib) * cart_norm(LC, ic) * cart_norm(LD, id);
                        scatter8(args.eri_out, nb, i, j0 + ib, k0 + ic, l0 + id, double(acc[(bl * NC + ic) * ND + id]) * nrm);
                    }
                }
        return;
    }

#pragma unroll
    for (int bl = 0; bl < NBT; ++bl)
#pragma unroll
        for (int ic = 0; ic < NC; ++ic)
#pragma unroll
            for (int id = 0; id < ND; ++id) {
                const int ib = ib0 + bl;
                const double sw = quartet_weight(same_ab, same_cd, same_bk, ia, ib, ic, id, NB, ND, check, args.Qao, nb,
                                                 i, j0 + ib, k0 + ic, l0 + id, args.tol);
                acc[(bl * NC + ic) * ND + id] *=
                    R(sw * cart_norm_rt<LA>(ia) * cart_norm_rt<LB>(ib) * cart_norm(LC, ic) * cart_norm(LD, id));
            }
    // J(i, j0+ib0+bl): each owner adds its sums.  (A sum across the teams of
    // a warp would need a full-warp shuffle right after loops in which the
    // teams run different trip counts and synchronise only their own lanes;
    // measured on the GPU, that read lanes' registers before their teams had
    // written them.)
    {
        double p[NC * ND];
#pragma unroll
        for (int ic = 0; ic < NC; ++ic)
#pragma unroll
            for (int id = 0; id < ND; ++id) p[ic * ND + id] = __ldg(args.Pj + (size_t)(k0 + ic) * nb + l0 + id);
#pragma unroll
        for (int bl = 0; bl < NBT; ++bl) {
            double sj = 0.0;
#pragma unroll
            for (int ic = 0; ic < NC; ++ic)
#pragma unroll
                for (int id = 0; id < ND; ++id) sj += double(acc[(bl * NC + ic) * ND + id]) * p[ic * ND + id];
            if (owner) fx_add(args.Jacc, (size_t)i * nb + j0 + ib0 + bl, sj);
        }
    }
    if constexpr (SS::TEAMRED) {
        // owners stage their partial sums of J(k,l), K_m(j,k), K_m(j,l) in the
        // team's (now unused) table; the team then adds them up and one lane
        // per element issues the atomic
        constexpr int V = SS::template redv<NK>();
        double *red = reinterpret_cast<double *>(g);   // 8-byte aligned (SplitShape::TABLE)
        split_sync<TEAM>(mask, team);
        if (owner) {
            {
                double pij[NB];
#pragma unroll
                for (int bl = 0; bl < NB; ++bl) pij[bl] = __ldg(args.Pj + (size_t)i * nb + j0 + bl);
#pragma unroll
                for (int ic = 0; ic < NC; ++ic)
#pragma unroll
                    for (int id = 0; id < ND; ++id) {
                        double sj = 0.0;
#pragma unroll
                        for (int bl = 0; bl < NB; ++bl) sj += double(acc[(bl * NC + ic) * ND + id]) * pij[bl];
                        red[gi * V + ic * ND + id] = sj;
                    }
            }
#pragma unroll
            for (int m = 0; m < NK; ++m) {
                const double *__restrict__ Pk = m == 0 ? args.Pk0 : args.Pk1;
                double *r = red + gi * V + SS::REDV1 + m * SS::REDVK;
                if (!(m == 0 ? args.Kacc0 : args.Kacc1)) continue;
                double pil[ND], pik[NC];
#pragma unroll
                for (int id = 0; id < ND; ++id) pil[id] = __ldg(Pk + (size_t)i * nb + l0 + id);
#pragma unroll
                for (int ic = 0; ic < NC; ++ic) pik[ic] = __ldg(Pk + (size_t)i * nb + k0 + ic);
#pragma unroll
                for (int bl = 0; bl < NB; ++bl) {
#pragma unroll
                    for (int ic = 0; ic < NC; ++ic) {
                        double sk = 0.0;
#pragma unroll
                        for (int id = 0; id < ND; ++id) sk += double(acc[(bl * NC + ic) * ND + id]) * pil[id];
                        r[bl * NC + ic] = sk;                              // K(j,k)
                    }
#pragma unroll
                    for (int id = 0; id < ND; ++id) {
                        double sk = 0.0;
#pragma unroll
                        for (int ic = 0; ic < NC; ++ic) sk += double(acc[(bl * NC + ic) * ND + id]) * pik[ic];
                        r[NB * NC + bl * ND + id] = sk;                    // K(j,l)
                    }
                }
            }
        }
        split_sync<TEAM>(mask, team);
        for (int e = lane; e < V; e += TEAM) {
            double sum = 0.0;
            for (int o = 0; o < SS::GROUP; ++o) sum += red[o * V + e];
            if (e < SS::REDV1) {
                fx_add(args.Jacc, (size_t)(k0 + e / ND) * nb + l0 + e % ND, sum);
            } else {
                const int m = (e - SS::REDV1) / SS::REDVK, f = (e - SS::REDV1) % SS::REDVK;
                FxWord *Kacc = m == 0 ? args.Kacc0 : args.Kacc1;
                if (!Kacc) continue;
                if (f < NB * NC) fx_add(Kacc, (size_t)(j0 + f / NC) * nb + k0 + f % NC, sum);
                else fx_add(Kacc, (size_t)(j0 + (f - NB * NC) / ND) * nb + l0 + (f - NB * NC) % ND, sum);
            }
        }
    }
    if (!owner) return;
    digest_blocks<1, NBT, NC, ND, NK, kSkipJij | (SS::TEAMRED ? kSkipJkl | kSkipKjk | kSkipKjl : 0)>(
        acc, i, j0 + ib0, k0, l0, args);
}

}  // namespace pfk

