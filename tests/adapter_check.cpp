// adapter_check.cpp -- compiled by tests/test_adapter.py against
// include/planck_fock_adapter.hpp and libplanck_fock.so, with minimal
// stand-ins for Planck's HartreeFock::Shell / Basis / IntegralMethod types
// (src/base/types.h:46-54, 95-100, 263-327) and an Eigen-like matrix.
//
//   adapter_check cpu <basis.txt> [nogpu]    checks that need no GPU; with
//                                            nogpu, also that a context fails
//                                            with PFK_ERR_CUDA
//   adapter_check gpu <basis.txt> <P.bin> <out.bin>
//                                            G (RHF, OS and Rys), Ga/Gb (UHF),
//                                            J/K through the adapter
//
// basis.txt: nshell, then per shell "L nprim cx cy cz" followed by nprim
// lines "exponent coefficient normalisation".  P.bin: nb*nb doubles.
// Prints one "ok <check>" line per passed check; exits non-zero on failure.
#include <cmath>
#include <cstdio>
#include <deque>
#include <fstream>
#include <string>
#include <vector>

#include "planck_fock_adapter.hpp"

namespace HartreeFock {
enum class ShellType { S, P, D, F, G, H };
enum class IntegralMethod { ObaraSaika, RysQuadrature, Auto };
struct SignedAOSymOp {
    int dummy = 0;
};
struct Vec {
    std::vector<double> v;
    double operator[](std::size_t i) const { return v[i]; }
    std::size_t size() const { return v.size(); }
};
struct Shell {
    double _center[3] = {0.0, 0.0, 0.0};
    ShellType _shell = ShellType::S;
    Vec _primitives, _coefficients, _normalizations;
    std::size_t nprimitives() const noexcept { return _primitives.size(); }
};
struct Basis {
    std::deque<Shell> _shells;
};
}  // namespace HartreeFock

struct Mat {
    long r, c;
    std::vector<double> v;
    Mat(long rows, long cols) : r(rows), c(cols), v(static_cast<std::size_t>(rows * cols)) {}
    long rows() const { return r; }
    long cols() const { return c; }
    double *data() { return v.data(); }
    const double *data() const { return v.data(); }
};

static int fail(const std::string &what)
{
    std::printf("FAIL %s\n", what.c_str());
    return 1;
}

static bool read_basis(const char *path, HartreeFock::Basis &b)
{
    std::ifstream f(path);
    int ns = 0;
    if (!(f >> ns)) return false;
    for (int s = 0; s < ns; ++s) {
        HartreeFock::Shell sh;
        int L = 0, np = 0;
        f >> L >> np >> sh._center[0] >> sh._center[1] >> sh._center[2];
        sh._shell = static_cast<HartreeFock::ShellType>(L);
        for (int i = 0; i < np; ++i) {
            double e, c, n;
            f >> e >> c >> n;
            sh._primitives.v.push_back(e);
            sh._coefficients.v.push_back(c);
            sh._normalizations.v.push_back(n);
        }
        b._shells.push_back(sh);
    }
    return static_cast<bool>(f);
}

template <class F>
static bool throws_status(F &&fn, pfk_status want, std::string *msg = nullptr)
{
    try {
        fn();
    } catch (const pfk_adapter::Error &e) {
        if (msg) *msg = e.what();
        return e.status() == want;
    }
    return false;
}

int main(int argc, char **argv)
{
    if (argc < 3) return fail("usage");
    const std::string mode = argv[1];
    HartreeFock::Basis basis;
    if (!read_basis(argv[2], basis)) return fail("basis file");

    // shell data in the C ABI's layout
    const pfk_adapter::ShellData d = pfk_adapter::shell_data(basis);
    std::size_t np = 0, nb = 0;
    for (const auto &sh : basis._shells) {
        np += sh.nprimitives();
        const int L = static_cast<int>(sh._shell);
        nb += static_cast<std::size_t>((L + 1) * (L + 2) / 2);
    }
    if (d.L.size() != basis._shells.size() || d.expo.size() != np || d.center.size() != 3 * basis._shells.size())
        return fail("shell_data sizes");
    std::printf("ok shell_data nshell=%zu nprim=%zu nbasis=%zu\n", d.L.size(), np, nb);

    // a g shell is rejected by pfk_create before the device is touched
    {
        HartreeFock::Basis bad = basis;
        bad._shells.front()._shell = HartreeFock::ShellType::G;
        std::string msg;
        if (!throws_status([&] { pfk_adapter::Context c(bad); }, PFK_ERR_UNSUPPORTED, &msg))
            return fail("g shell not rejected");
        if (msg.find("angular momentum") == std::string::npos) return fail("g shell message: " + msg);
        std::printf("ok rejects_g_shell\n");
    }
    // a non-positive exponent is invalid
    {
        HartreeFock::Basis bad = basis;
        bad._shells.back()._primitives.v[0] = -1.0;
        if (!throws_status([&] { pfk_adapter::Context c(bad); }, PFK_ERR_INVALID)) return fail("bad exponent");
        std::printf("ok rejects_bad_exponent\n");
    }

    if (mode == "cpu") {
        if (argc < 4 || std::string(argv[3]) != "nogpu") return 0;
        // without a GPU, creating a context fails loudly with a CUDA status
        std::string msg;
        if (!throws_status([&] { pfk_adapter::Context c(basis); }, PFK_ERR_CUDA, &msg))
            return fail("context without a GPU did not fail with PFK_ERR_CUDA");
        std::printf("ok no_gpu_fails_loudly\n");
        return 0;
    }
    if (mode != "gpu" || argc < 5) return fail("mode");

    std::vector<double> P(nb * nb);
    {
        std::FILE *f = std::fopen(argv[3], "rb");
        if (!f || std::fread(P.data(), sizeof(double), P.size(), f) != P.size()) return fail("P file");
        std::fclose(f);
    }
    pfk_adapter::Context ctx(basis, 0);
    if (ctx.nbasis() != nb) return fail("nbasis");
    Mat Pm(static_cast<long>(nb), static_cast<long>(nb));
    Pm.v = P;
    using HartreeFock::IntegralMethod;
    std::vector<HartreeFock::SignedAOSymOp> one(1), two(2);

    const Mat G_os = pfk_adapter::compute_2e_fock(ctx, Pm, nb, IntegralMethod::ObaraSaika, 1e-10, &one);
    const Mat G_rys = pfk_adapter::compute_2e_fock(ctx, Pm, nb, IntegralMethod::RysQuadrature, 1e-10, &one);
    const auto GaGb = pfk_adapter::compute_2e_fock_uhf(ctx, Pm, Pm, nb, IntegralMethod::Auto, 1e-10, &one);
    const auto JK = pfk_adapter::compute_jk(ctx, Pm, Pm, -0.25, IntegralMethod::ObaraSaika);
    // a looser tol_eri reaches the library (fewer quartets, a different G)
    const Mat G_loose = pfk_adapter::compute_2e_fock(ctx, Pm, nb, IntegralMethod::ObaraSaika, 1e-3);
    std::printf("ok builds\n");

    if (!throws_status([&] { pfk_adapter::compute_2e_fock(ctx, Pm, nb, IntegralMethod::ObaraSaika, 1e-10, &two); },
                       PFK_ERR_UNSUPPORTED))
        return fail("two symmetry operations accepted (RHF)");
    if (!throws_status([&] { pfk_adapter::compute_2e_fock_uhf(ctx, Pm, Pm, nb, IntegralMethod::Auto, 1e-10, &two); },
                       PFK_ERR_UNSUPPORTED))
        return fail("two symmetry operations accepted (UHF)");
    if (!throws_status([&] { pfk_adapter::compute_2e_fock(ctx, Pm, nb + 1, IntegralMethod::ObaraSaika); },
                       PFK_ERR_INVALID))
        return fail("wrong nbasis accepted");
    std::printf("ok rejects_sym_ops_and_nbasis\n");

    std::FILE *f = std::fopen(argv[4], "wb");
    if (!f) return fail("out file");
    for (const Mat *M : {&G_os, &G_rys, &GaGb.first, &GaGb.second, &JK.first, &JK.second, &G_loose})
        std::fwrite(M->data(), sizeof(double), nb * nb, f);
    std::fclose(f);
    std::printf("ok wrote\n");
    return 0;
}
