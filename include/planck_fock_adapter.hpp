// planck_fock_adapter.hpp -- header-only C++ adapter: Planck's integral entry
// points on top of the C ABI of planck_fock.h.
//
// Planck's SCF, DFT and post-HF code reach the two-electron integrals through
// free functions in src/integrals/base.h (reference project paths):
//
//   _compute_2e            base.h:39-55   -> pfk_adapter::compute_2e
//   _compute_2e_fock       base.h:57-73   -> pfk_adapter::compute_2e_fock
//   _compute_2e_fock_uhf   base.h:75-93   -> pfk_adapter::compute_2e_fock_uhf
//   build_coulomb_from_eri / build_exchange_from_eri
//                          dft/driver.cpp:689-731 -> pfk_adapter::compute_jk
//
// The functions below take the same arguments as those, except that a
// pfk_adapter::Context (one per basis and geometry, built once after
// build_shellpairs) stands in for the std::vector<ShellPair>.  They are
// templates over Planck's own types so that this header needs neither Eigen
// nor Planck's headers:
//
//   Basis     has _shells, a range of shells with _shell (ShellType, S = 0 ..
//             F = 3), _center[0..2] (Bohr), nprimitives(), and _primitives,
//             _coefficients, _normalizations indexable by primitive
//             (HartreeFock::Basis / Shell, types.h:263-327);
//   Matrix    constructible as Matrix(rows, cols), with rows(), cols() and a
//             contiguous data() (Eigen::MatrixXd; column-major, but G, J and K
//             are symmetric so the layout does not matter);
//   Method    an enum whose values are ObaraSaika = 0, RysQuadrature = 1,
//             Auto = 2 (HartreeFock::IntegralMethod, types.h:95-100), the
//             order of pfk_engine;
//   SymOps    a container with size() (std::vector<SignedAOSymOp>).
//
// Errors: the reference's functions do not fail except by throwing
// std::bad_alloc; these throw pfk_adapter::Error (a std::runtime_error
// carrying the pfk_status) with the library's message.  A non-null sym_ops
// with more than one operation is rejected with PFK_ERR_UNSUPPORTED: the
// engine builds the full quartet set and has no symmetry-orbit filter
// (os.cpp:1478-1487).  A single operation is the identity and is accepted.
#ifndef PLANCK_FOCK_ADAPTER_HPP
#define PLANCK_FOCK_ADAPTER_HPP

#include <cstddef>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "planck_fock.h"

namespace pfk_adapter {

class Error : public std::runtime_error {
public:
    Error(pfk_status s, const std::string &what) : std::runtime_error(what), status_(s) {}
    pfk_status status() const noexcept { return status_; }

private:
    pfk_status status_;
};

// Shell data of a Planck basis in the C ABI's layout (pfk_basis_desc points
// into the vectors, so keep the ShellData alive while the descriptor is used).
struct ShellData {
    std::vector<int> L, nprim;
    std::vector<double> center, expo, coef, norm;
    pfk_basis_desc desc() const
    {
        return pfk_basis_desc{static_cast<int>(L.size()), L.data(), nprim.data(), center.data(),
                              expo.data(), coef.data(), norm.data()};
    }
};

template <class Basis>
ShellData shell_data(const Basis &basis)
{
    ShellData d;
    for (const auto &sh : basis._shells) {
        d.L.push_back(static_cast<int>(sh._shell));
        const int n = static_cast<int>(sh.nprimitives());
        d.nprim.push_back(n);
        for (int x = 0; x < 3; ++x) d.center.push_back(sh._center[x]);
        for (int i = 0; i < n; ++i) {
            d.expo.push_back(sh._primitives[i]);
            d.coef.push_back(sh._coefficients[i]);   // the contracted normalisation is already folded in
            d.norm.push_back(sh._normalizations[i]);
        }
    }
    return d;
}

// One engine context: the device memory, Schwarz table and screened quartet
// lists of one basis and geometry.  Not copyable; movable.
class Context {
public:
    template <class Basis>
    explicit Context(const Basis &basis, int device = 0)
    {
        const ShellData d = shell_data(basis);
        const pfk_basis_desc desc = d.desc();
        const pfk_status s = pfk_create(&desc, device, &ctx_);
        if (s != PFK_OK) throw Error(s, std::string("pfk_create: ") + pfk_last_error(nullptr));
    }
    ~Context()
    {
        if (ctx_) pfk_destroy(ctx_);
    }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;
    Context(Context &&o) noexcept : ctx_(o.ctx_), tol_(o.tol_), engine_(o.engine_) { o.ctx_ = nullptr; }
    Context &operator=(Context &&o) noexcept
    {
        if (this != &o) {
            if (ctx_) pfk_destroy(ctx_);
            ctx_ = o.ctx_;
            tol_ = o.tol_;
            engine_ = o.engine_;
            o.ctx_ = nullptr;
        }
        return *this;
    }

    pfk_ctx *get() const noexcept { return ctx_; }
    std::size_t nbasis() const noexcept { return static_cast<std::size_t>(pfk_nbasis(ctx_)); }

    void check(pfk_status s, const char *what) const
    {
        if (s != PFK_OK) throw Error(s, std::string(what) + ": " + pfk_last_error(ctx_));
    }

    // OptionsIntegral (types.h:408-412) for the next build: the engine and
    // tol_eri of the call.  pfk_set_options rebuilds the quartet lists when
    // tol_eri changes, so it is called only when either value changes.
    void configure(int engine, double tol_eri)
    {
        if (engine == engine_ && tol_eri == tol_) return;
        check(pfk_set_options(ctx_, tol_eri, engine, PFK_PREC_FP64, 1e-8), "pfk_set_options");
        engine_ = engine;
        tol_ = tol_eri;
    }

private:
    pfk_ctx *ctx_ = nullptr;
    double tol_ = -1.0;
    int engine_ = -1;
};

namespace detail {

template <class SymOps>
void check_sym_ops(const SymOps *sym_ops)
{
    if (sym_ops && sym_ops->size() > 1)
        throw Error(PFK_ERR_UNSUPPORTED, "integral symmetry operations are not supported by the GPU engine");
}

inline void check_nbasis(const Context &ctx, std::size_t nbasis)
{
    if (nbasis != ctx.nbasis())
        throw Error(PFK_ERR_INVALID, "nbasis " + std::to_string(nbasis) + " does not match the context's " +
                                         std::to_string(ctx.nbasis()));
}

template <class Matrix>
void check_square(const Matrix &M, std::size_t nbasis, const char *name)
{
    if (static_cast<std::size_t>(M.rows()) != nbasis || static_cast<std::size_t>(M.cols()) != nbasis)
        throw Error(PFK_ERR_INVALID, std::string(name) + " is not nbasis x nbasis");
}

struct NoSymOps {
    std::size_t size() const noexcept { return 0; }
};

}  // namespace detail

// _compute_2e_fock (base.h:57-73): G = J(P) - K(P)/2.
template <class Matrix, class Method, class SymOps = detail::NoSymOps>
Matrix compute_2e_fock(Context &ctx, const Matrix &density, std::size_t nbasis, const Method &engine,
                       double tol_eri = 1e-10, const SymOps *sym_ops = nullptr)
{
    detail::check_sym_ops(sym_ops);
    detail::check_nbasis(ctx, nbasis);
    detail::check_square(density, nbasis, "density");
    ctx.configure(static_cast<int>(engine), tol_eri);
    Matrix G(density.rows(), density.cols());
    ctx.check(pfk_fock_rhf(ctx.get(), density.data(), G.data()), "pfk_fock_rhf");
    return G;
}

// _compute_2e_fock_uhf (base.h:75-93): Ga = J(Pa+Pb) - K(Pa), Gb = J(Pa+Pb) - K(Pb).
template <class Matrix, class Method, class SymOps = detail::NoSymOps>
std::pair<Matrix, Matrix> compute_2e_fock_uhf(Context &ctx, const Matrix &Pa, const Matrix &Pb, std::size_t nbasis,
                                              const Method &engine, double tol_eri = 1e-10,
                                              const SymOps *sym_ops = nullptr)
{
    detail::check_sym_ops(sym_ops);
    detail::check_nbasis(ctx, nbasis);
    detail::check_square(Pa, nbasis, "Pa");
    detail::check_square(Pb, nbasis, "Pb");
    ctx.configure(static_cast<int>(engine), tol_eri);
    Matrix Ga(Pa.rows(), Pa.cols()), Gb(Pb.rows(), Pb.cols());
    ctx.check(pfk_fock_uhf(ctx.get(), Pa.data(), Pb.data(), Ga.data(), Gb.data()), "pfk_fock_uhf");
    return {std::move(Ga), std::move(Gb)};
}

// _compute_2e (base.h:39-55): the full nbasis^4 tensor, row-major
// i*nb^3 + j*nb^2 + k*nb + l with all 8 permutations (nbasis <= 180).
template <class Method, class SymOps = detail::NoSymOps>
std::vector<double> compute_2e(Context &ctx, std::size_t nbasis, const Method &engine, double tol_eri = 1e-10,
                               const SymOps *sym_ops = nullptr)
{
    detail::check_sym_ops(sym_ops);
    detail::check_nbasis(ctx, nbasis);
    ctx.configure(static_cast<int>(engine), tol_eri);
    std::vector<double> eri(nbasis * nbasis * nbasis * nbasis);
    ctx.check(pfk_eri_tensor(ctx.get(), eri.data()), "pfk_eri_tensor");
    return eri;
}

// RKS / UKS Coulomb and exact exchange (dft/driver.cpp:689-731, 3077-3118):
// J = J(P_total), K = k_scale K(P_spin), e.g. k_scale = -a_x / 2 for a hybrid.
template <class Matrix, class Method>
std::pair<Matrix, Matrix> compute_jk(Context &ctx, const Matrix &P_total, const Matrix &P_spin, double k_scale,
                                     const Method &engine, double tol_eri = 1e-10)
{
    const std::size_t nb = ctx.nbasis();
    detail::check_square(P_total, nb, "P_total");
    detail::check_square(P_spin, nb, "P_spin");
    ctx.configure(static_cast<int>(engine), tol_eri);
    Matrix J(P_total.rows(), P_total.cols()), K(P_spin.rows(), P_spin.cols());
    ctx.check(pfk_jk(ctx.get(), P_total.data(), P_spin.data(), J.data(), K.data(), k_scale), "pfk_jk");
    return {std::move(J), std::move(K)};
}

}  // namespace pfk_adapter

#endif  // PLANCK_FOCK_ADAPTER_HPP
