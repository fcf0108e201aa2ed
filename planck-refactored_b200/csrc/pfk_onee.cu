// pfk_onee.cu -- one-electron integrals on the device: overlap S, kinetic T
// and nuclear attraction V over the Cartesian basis (the reference computes
// them on the host with Obara-Saika, os.cpp:294-602).
//
// One thread per shell pair (a <= b in shell order), oriented so that
// L(A) >= L(B); the kernel is instantiated per (LA, LB) class:
//   * S and T from the one-dimensional Obara-Saika overlap recurrence per
//     axis, s(i+1, j) = PA s(i, j) + (i s(i-1, j) + j s(i, j-1)) / (2 zeta),
//     and T_x(i, j) = -1/2 [j(j-1) s(i, j-2) - 2 beta (2j+1) s(i, j)
//     + 4 beta^2 s(i, j+2)], T = T_x S_y S_z + S_x T_y S_z + S_x S_y T_z;
//   * V from the nuclear-attraction vertical recurrence
//     [a+1_d]^(m) = PA_d [a]^(m) - PC_d [a]^(m+1)
//                 + a_d / (2 zeta) ([a-1_d]^(m) - [a-1_d]^(m+1)),
//     [0]^(m) = -Z_C (2 pi / zeta) K F_m(zeta |PC|^2), summed over nuclei and
//     primitives, then the horizontal recurrence (a, b+1_d) = (a+1_d, b) +
//     AB_d (a, b) once per shell pair (os_hrr);
//   * the contracted normalisation c N (folded coefficients times primitive
//     norms) and the Cartesian component norms as in the ERI kernels.
#include <string>
#include <vector>

#include "pfk_internal.h"
#include "pfk_os.cuh"

namespace pfk {
namespace {

struct OneShell {
    double x, y, z;
    int L, nprim, prim_off, ao_off;
};

template <int LA, int LB>
__global__ void __launch_bounds__(128) onee_kernel(const int2 *__restrict__ pairs, int n,
                                                   const OneShell *__restrict__ sh, const double *__restrict__ expo,
                                                   const double *__restrict__ cn, int natom,
                                                   const double4 *__restrict__ nuc, int nb, double *S, double *T,
                                                   double *V)
{
    using O = OSShape<LA, LB, 0, 0>;
    constexpr int E = LA + LB, NA = ncart(LA), NB = ncart(LB);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int2 pr = pairs[t];
    const OneShell a = sh[pr.x], b = sh[pr.y];
    const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z};
    const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
    const double AB2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    double s_acc[NA * NB], t_acc[NA * NB], v_acc[O::NACC];
#pragma unroll
    for (int c = 0; c < NA * NB; ++c) s_acc[c] = t_acc[c] = 0.0;
#pragma unroll
    for (int c = 0; c < O::NACC; ++c) v_acc[c] = 0.0;

    for (int i = 0; i < a.nprim; ++i) {
        const double al = expo[a.prim_off + i], ca = cn[a.prim_off + i];
        for (int j = 0; j < b.nprim; ++j) {
            const double be = expo[b.prim_off + j], cb = cn[b.prim_off + j];
            const double zeta = al + be, iz = 1.0 / zeta, h = 0.5 * iz;
            const double K = ca * cb * exp(-al * be * iz * AB2);
            double P[3], PA[3], PB[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                P[d] = (al * A[d] + be * B[d]) * iz;
                PA[d] = P[d] - A[d];
                PB[d] = P[d] - B[d];
            }
            // one-dimensional overlaps s[d][i][j], i <= LA, j <= LB + 2
            double s1[3][LA + 1][LB + 3];
            const double s00 = sqrt(3.14159265358979323846 * iz);
#pragma unroll
            for (int d = 0; d < 3; ++d)
#pragma unroll
                for (int ii = 0; ii <= LA; ++ii)
#pragma unroll
                    for (int jj = 0; jj <= LB + 2; ++jj) {
                        double v;
                        if (ii == 0 && jj == 0) {
                            v = s00;
                        } else if (ii == 0) {
                            v = PB[d] * s1[d][0][jj - 1];
                            if (jj >= 2) v += h * (jj - 1) * s1[d][0][jj - 2];
                        } else {
                            v = PA[d] * s1[d][ii - 1][jj];
                            if (ii >= 2) v += h * (ii - 1) * s1[d][ii - 2][jj];
                            if (jj >= 1) v += h * jj * s1[d][ii - 1][jj - 1];
                        }
                        s1[d][ii][jj] = v;
                    }
            static_for<0, NA>([&](auto ia_) {
                constexpr int ia = PFK_CI(ia_);
                static_for<0, NB>([&](auto ib_) {
                    constexpr int ib = PFK_CI(ib_);
                    double sx[3], kx[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const int ea = cart_l(LA, ia, d), eb = cart_l(LB, ib, d);
                        sx[d] = s1[d][ea][eb];
                        double k = -2.0 * be * (2 * eb + 1) * s1[d][ea][eb] + 4.0 * be * be * s1[d][ea][eb + 2];
                        if (eb >= 2) k += eb * (eb - 1) * s1[d][ea][eb - 2];
                        kx[d] = -0.5 * k;
                    }
                    s_acc[ia * NB + ib] += K * sx[0] * sx[1] * sx[2];
                    t_acc[ia * NB + ib] +=
                        K * (kx[0] * sx[1] * sx[2] + sx[0] * kx[1] * sx[2] + sx[0] * sx[1] * kx[2]);
                });
            });
            for (int c = 0; c < natom; ++c) {
                const double4 C = nuc[c];
                const double PC[3] = {P[0] - C.x, P[1] - C.y, P[2] - C.z};
                double F[E + 1];
                boys_fm<E>(zeta * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]), F);
                const double pre = -C.w * 2.0 * 3.14159265358979323846 * iz * K;
                double v[O::NV];
                static_for<0, E + 1>([&](auto m_) {
                    constexpr int m = PFK_CI(m_);
                    v[O::vi(0, 0, 0, 0, m)] = pre * F[m];
                });
                static_for<1, E + 1>([&](auto la_) {
                    constexpr int la = PFK_CI(la_);
                    static_for<0, ncart(la)>([&](auto ia_) {
                        constexpr int ia = PFK_CI(ia_);
                        constexpr int d = cart_dir(la, ia), ad = cart_l(la, ia, d), ip = cart_step(la, ia, d, -1);
                        static_for<0, E - la + 1>([&](auto m_) {
                            constexpr int m = PFK_CI(m_);
                            double x = PA[d] * v[O::vi(0, la - 1, ip, 0, m)] - PC[d] * v[O::vi(0, la - 1, ip, 0, m + 1)];
                            if constexpr (ad >= 2) {
                                constexpr int ig = cart_step(la - 1, ip, d, -1);
                                x += (ad - 1) * h * (v[O::vi(0, la - 2, ig, 0, m)] - v[O::vi(0, la - 2, ig, 0, m + 1)]);
                            }
                            v[O::vi(0, la, ia, 0, m)] = x;
                        });
                    });
                });
                static_for<LA, E + 1>([&](auto la_) {
                    constexpr int la = PFK_CI(la_);
                    static_for<0, ncart(la)>([&](auto ia_) {
                        constexpr int ia = PFK_CI(ia_);
                        v_acc[O::row(la) + ia] += v[O::vi(0, la, ia, 0, 0)];
                    });
                });
            }
        }
    }
    double vblk[NA * NB];
    os_hrr<LA, LB, 0, 0, double>(v_acc, AB, AB, vblk);
#pragma unroll
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
        for (int ib = 0; ib < NB; ++ib) {
            const double nrm = cart_norm(LA, ia) * cart_norm(LB, ib);
            const size_t i = a.ao_off + ia, j = b.ao_off + ib;
            const double sv = s_acc[ia * NB + ib] * nrm, tv = t_acc[ia * NB + ib] * nrm, vv = vblk[ia * NB + ib] * nrm;
            S[i * nb + j] = sv;
            S[j * nb + i] = sv;
            T[i * nb + j] = tv;
            T[j * nb + i] = tv;
            V[i * nb + j] = vv;
            V[j * nb + i] = vv;
        }
}

using OneeLauncher = void (*)(const int2 *, int, const OneShell *, const double *, const double *, int,
                              const double4 *, int, double *, double *, double *, cudaStream_t);

template <int LA, int LB>
void launch_onee(const int2 *pairs, int n, const OneShell *sh, const double *expo, const double *cn, int natom,
                 const double4 *nuc, int nb, double *S, double *T, double *V, cudaStream_t st)
{
    onee_kernel<LA, LB><<<(n + 127) / 128, 128, 0, st>>>(pairs, n, sh, expo, cn, natom, nuc, nb, S, T, V);
}

// (LA, LB) with LA >= LB, index LA (LA + 1) / 2 + LB
const OneeLauncher kOnee[10] = {launch_onee<0, 0>, launch_onee<1, 0>, launch_onee<1, 1>, launch_onee<2, 0>,
                                launch_onee<2, 1>, launch_onee<2, 2>, launch_onee<3, 0>, launch_onee<3, 1>,
                                launch_onee<3, 2>, launch_onee<3, 3>};

template <typename X>
struct Dev {
    X *p = nullptr;
    ~Dev() { if (p) cudaFree(p); }
    cudaError_t put(const X *h, size_t n)
    {
        cudaError_t e = cudaMalloc(&p, sizeof(X) * (n ? n : 1));
        if (e != cudaSuccess || !n) return e;
        return cudaMemcpy(p, h, sizeof(X) * n, cudaMemcpyHostToDevice);
    }
};

}  // namespace

cudaError_t one_electron_run(const pfk_basis_desc *basis, int natom, const double *nuclei, double *S, double *T,
                             double *V, int device, std::string &what)
{
    auto fail = [&](const char *w, cudaError_t err) {
        what = w;
        return err;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail("cudaSetDevice", e);
    const int ns = basis->nshell;
    std::vector<OneShell> sh(ns);
    std::vector<double> expo, cn;
    int nb = 0, po = 0;
    for (int s = 0; s < ns; ++s) {
        sh[s] = {basis->center[3 * s], basis->center[3 * s + 1], basis->center[3 * s + 2], basis->L[s],
                 basis->nprim[s], po, nb};
        for (int k = 0; k < basis->nprim[s]; ++k) {
            expo.push_back(basis->expo[po + k]);
            cn.push_back(basis->coef[po + k] * basis->norm[po + k]);
        }
        po += basis->nprim[s];
        nb += ncart(basis->L[s]);
    }
    std::vector<int2> pairs[10];
    for (int a = 0; a < ns; ++a)
        for (int b = a; b < ns; ++b) {
            const int la = sh[a].L, lb = sh[b].L;
            if (la >= lb) pairs[la * (la + 1) / 2 + lb].push_back(make_int2(a, b));
            else pairs[lb * (lb + 1) / 2 + la].push_back(make_int2(b, a));
        }
    std::vector<double4> nuc(natom);
    for (int c = 0; c < natom; ++c) nuc[c] = make_double4(nuclei[4 * c], nuclei[4 * c + 1], nuclei[4 * c + 2], nuclei[4 * c + 3]);

    Dev<OneShell> d_sh;
    Dev<double> d_expo, d_cn, d_S, d_T, d_V;
    Dev<double4> d_nuc;
    Dev<int2> d_pairs[10];
    if ((e = d_sh.put(sh.data(), ns)) != cudaSuccess || (e = d_expo.put(expo.data(), expo.size())) != cudaSuccess ||
        (e = d_cn.put(cn.data(), cn.size())) != cudaSuccess || (e = d_nuc.put(nuc.data(), natom)) != cudaSuccess)
        return fail("upload of shell data", e);
    const size_t nb2 = (size_t)nb * nb;
    if ((e = cudaMalloc(&d_S.p, sizeof(double) * nb2)) != cudaSuccess ||
        (e = cudaMalloc(&d_T.p, sizeof(double) * nb2)) != cudaSuccess ||
        (e = cudaMalloc(&d_V.p, sizeof(double) * nb2)) != cudaSuccess)
        return fail("cudaMalloc(S, T, V)", e);
    for (int c = 0; c < 10; ++c) {
        if (pairs[c].empty()) continue;
        if ((e = d_pairs[c].put(pairs[c].data(), pairs[c].size())) != cudaSuccess) return fail("upload of pairs", e);
        kOnee[c](d_pairs[c].p, (int)pairs[c].size(), d_sh.p, d_expo.p, d_cn.p, natom, d_nuc.p, nb, d_S.p, d_T.p,
                 d_V.p, nullptr);
        if ((e = cudaGetLastError()) != cudaSuccess) return fail("one-electron kernel launch", e);
    }
    if ((e = cudaMemcpy(S, d_S.p, sizeof(double) * nb2, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(T, d_T.p, sizeof(double) * nb2, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(V, d_V.p, sizeof(double) * nb2, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return fail("copy of S, T, V", e);
    return cudaSuccess;
}

}  // namespace pfk
