// pfk_checkpoint.cu -- Planck checkpoint files (.hfchk, format version 6):
// a writer for densities made outside the reference's SCF (the learned guess)
// and the density-restart reader.  Host code only; nothing here touches a GPU.
//
// Byte layout (host byte order, IEEE-754 doubles), as Checkpoint::save writes
// it (src/io/checkpoint.cpp:347-489):
//   "PLNKCHK\0", uint32 version, uint64 nbasis, uint8 is_uhf,
//   uint8 is_converged, uint32 last_iter (always 0), double total_energy,
//   double nuclear_repulsion, uint64 natoms, int32 charge,
//   uint32 multiplicity, int32 Z[natoms], double xyz[natoms][3] (Bohr),
//   uint32 length + basis name bytes, uint8 has_opt_coords,
//   matrix S, matrix H, then per spin channel (alpha; beta when is_uhf)
//   matrix density, matrix fock, vector mo_energies, matrix mo_coefficients,
//   uint8 has_casscf_mos (+ matrix), uint8 has_basis = 1, uint64 nshells,
//   per shell {int32 L, uint32 nprim, double centre[3], double exps[nprim],
//   double coefs[nprim], double norms[nprim]}, uint64 nbf, per function
//   {uint64 shell, int32 lx, ly, lz, double component_norm},
//   uint8 has_casscf_active_densities (+ vector),
//   uint8 has_casscf_active_orbitals (+ int32 start, int32 count).
// A matrix is int64 rows, int64 cols, then rows*cols doubles column-major; a
// vector is an n x 1 matrix.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "planck_fock.h"

namespace {

thread_local std::string g_chk_error;

constexpr char kMagic[8] = {'P', 'L', 'N', 'K', 'C', 'H', 'K', '\0'};
constexpr uint32_t kVersion = 6;
// limits the reference's reader enforces (checkpoint.cpp:53-54)
constexpr uint32_t kMaxString = 4096;
constexpr uint64_t kMaxAtoms = 1000000;

pfk_status fail(pfk_status s, std::string msg)
{
    g_chk_error = std::move(msg);
    return s;
}

int dfact(int n)   // n!!, (-1)!! = 1
{
    int r = 1;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}

class Writer {
public:
    explicit Writer(const char *path) : out_(path, std::ios::binary | std::ios::trunc) {}
    bool open() const { return static_cast<bool>(out_); }
    bool good() const { return static_cast<bool>(out_); }
    template <typename T>
    void pod(T v) { out_.write(reinterpret_cast<const char *>(&v), sizeof(T)); }
    void bytes(const void *p, size_t n) { out_.write(static_cast<const char *>(p), static_cast<std::streamsize>(n)); }
    void matrix(const double *m, int64_t rows, int64_t cols)
    {
        pod<int64_t>(rows);
        pod<int64_t>(cols);
        bytes(m, sizeof(double) * static_cast<size_t>(rows * cols));
    }

private:
    std::ofstream out_;
};

// Reader with the reference's checks and messages (checkpoint.cpp:26-225).
class Reader {
public:
    explicit Reader(const char *path) : in_(path, std::ios::binary) {}
    bool open() const { return static_cast<bool>(in_); }
    std::string err;

    bool exact(void *p, size_t n, const std::string &label)
    {
        in_.read(static_cast<char *>(p), static_cast<std::streamsize>(n));
        if (!in_) err = "Checkpoint truncated while reading " + label;
        return static_cast<bool>(in_);
    }
    template <typename T>
    bool pod(T &v)
    {
        in_.read(reinterpret_cast<char *>(&v), sizeof(T));
        if (!in_) err = "Checkpoint truncated while reading " + std::to_string(sizeof(T)) + " bytes";
        return static_cast<bool>(in_);
    }
    bool string(std::string &s)
    {
        uint32_t len = 0;
        if (!exact(&len, 4, "string length")) return false;
        if (len > kMaxString) {
            err = "Checkpoint string length " + std::to_string(len) + " exceeds supported limit " +
                  std::to_string(kMaxString);
            return false;
        }
        s.assign(len, '\0');
        return len == 0 || exact(&s[0], len, "string data");
    }
    // A matrix of at most max_dim x max_dim; data may be null to skip it.
    // want_vector: an n x 1 vector, whose column count is checked first.
    bool matrix(std::vector<double> *data, int64_t &rows, int64_t &cols, uint64_t max_dim, const std::string &label,
                bool want_vector = false)
    {
        if (!exact(&rows, 8, label + " row count") || !exact(&cols, 8, label + " column count")) return false;
        if (want_vector && cols != 1) {
            err = "Checkpoint " + label + " is not stored as an n x 1 vector";
            return false;
        }
        if (rows < 0 || cols < 0) {
            err = "Checkpoint " + label + " has negative dimensions";
            return false;
        }
        if (static_cast<uint64_t>(rows) > max_dim || static_cast<uint64_t>(cols) > max_dim) {
            err = "Checkpoint " + label + " dimensions " + std::to_string(rows) + "x" + std::to_string(cols) +
                  " exceed supported limit " + std::to_string(max_dim);
            return false;
        }
        const size_t n = static_cast<size_t>(rows) * static_cast<size_t>(cols);
        std::vector<double> tmp;
        std::vector<double> &dst = data ? *data : tmp;
        dst.resize(n);
        return n == 0 || exact(dst.data(), n * sizeof(double), label + " data");
    }
    bool vector(int64_t &n, uint64_t max_dim, const std::string &label)
    {
        int64_t cols = 0;
        return matrix(nullptr, n, cols, max_dim, label, true);
    }

private:
    std::ifstream in_;
};

int count_functions(const pfk_basis_desc *b)
{
    int nb = 0;
    for (int s = 0; s < b->nshell; ++s) nb += (b->L[s] + 1) * (b->L[s] + 2) / 2;
    return nb;
}

bool channel_ok(const pfk_spin_channel *c)
{
    return c && c->density && c->fock && c->mo_energies && c->mo_coefficients;
}

}  // namespace

extern "C" {

const char *pfk_checkpoint_last_error(void) { return g_chk_error.c_str(); }

pfk_status pfk_checkpoint_write(const char *path, const pfk_checkpoint_meta *meta, const pfk_basis_desc *basis,
                                const double *S, const double *H, const pfk_spin_channel *alpha,
                                const pfk_spin_channel *beta)
{
    if (!path || !meta || !basis || !S || !H || !channel_ok(alpha) || (beta && !channel_ok(beta)))
        return fail(PFK_ERR_INVALID, "pfk_checkpoint_write: null argument");
    if (meta->natoms < 0 || (meta->natoms > 0 && (!meta->atomic_numbers || !meta->coords_bohr)))
        return fail(PFK_ERR_INVALID, "pfk_checkpoint_write: bad atom data");
    const std::string name = meta->basis_name ? meta->basis_name : "";
    if (name.size() > kMaxString) return fail(PFK_ERR_INVALID, "pfk_checkpoint_write: basis name too long");
    if (basis->nshell < 0 || (basis->nshell > 0 && (!basis->L || !basis->nprim || !basis->center || !basis->expo ||
                                                     !basis->coef || !basis->norm)))
        return fail(PFK_ERR_INVALID, "pfk_checkpoint_write: bad basis data");
    for (int s = 0; s < basis->nshell; ++s)
        if (basis->L[s] < 0 || basis->L[s] > 5 || basis->nprim[s] < 1)
            return fail(PFK_ERR_INVALID, "pfk_checkpoint_write: shell " + std::to_string(s) + " has a bad L or nprim");
    const int64_t nb = count_functions(basis);

    Writer w(path);
    if (!w.open()) return fail(PFK_ERR_INVALID, std::string("Cannot open checkpoint file for writing: ") + path);
    w.bytes(kMagic, 8);
    w.pod<uint32_t>(kVersion);
    w.pod<uint64_t>(static_cast<uint64_t>(nb));
    w.pod<uint8_t>(beta ? 1 : 0);
    w.pod<uint8_t>(meta->converged ? 1 : 0);
    w.pod<uint32_t>(0);   // last iteration: the reference stores 0
    w.pod<double>(meta->total_energy);
    w.pod<double>(meta->nuclear_repulsion);
    w.pod<uint64_t>(static_cast<uint64_t>(meta->natoms));
    w.pod<int32_t>(meta->charge);
    w.pod<uint32_t>(meta->multiplicity);
    for (int a = 0; a < meta->natoms; ++a) w.pod<int32_t>(meta->atomic_numbers[a]);
    for (int a = 0; a < 3 * meta->natoms; ++a) w.pod<double>(meta->coords_bohr[a]);
    w.pod<uint32_t>(static_cast<uint32_t>(name.size()));
    w.bytes(name.data(), name.size());
    w.pod<uint8_t>(meta->has_opt_coords ? 1 : 0);

    w.matrix(S, nb, nb);
    w.matrix(H, nb, nb);
    for (const pfk_spin_channel *c : {alpha, beta}) {
        if (!c) continue;
        w.matrix(c->density, nb, nb);
        w.matrix(c->fock, nb, nb);
        w.matrix(c->mo_energies, nb, 1);
        w.matrix(c->mo_coefficients, nb, nb);
    }
    w.pod<uint8_t>(0);   // no CASSCF orbitals

    // shell data and basis functions (format version 4)
    w.pod<uint8_t>(1);
    w.pod<uint64_t>(static_cast<uint64_t>(basis->nshell));
    long long p0 = 0;
    for (int s = 0; s < basis->nshell; ++s) {
        const int np = basis->nprim[s];
        w.pod<int32_t>(basis->L[s]);
        w.pod<uint32_t>(static_cast<uint32_t>(np));
        for (int x = 0; x < 3; ++x) w.pod<double>(basis->center[3 * s + x]);
        w.bytes(basis->expo + p0, sizeof(double) * np);
        w.bytes(basis->coef + p0, sizeof(double) * np);
        w.bytes(basis->norm + p0, sizeof(double) * np);
        p0 += np;
    }
    w.pod<uint64_t>(static_cast<uint64_t>(nb));
    for (int s = 0; s < basis->nshell; ++s) {
        const int L = basis->L[s];
        for (int lx = L; lx >= 0; --lx)           // lx descending, then ly descending
            for (int ly = L - lx; ly >= 0; --ly) {
                const int lz = L - lx - ly;
                w.pod<uint64_t>(static_cast<uint64_t>(s));
                w.pod<int32_t>(lx);
                w.pod<int32_t>(ly);
                w.pod<int32_t>(lz);
                w.pod<double>(1.0 / std::sqrt(static_cast<double>(dfact(2 * lx - 1) * dfact(2 * ly - 1) *
                                                                  dfact(2 * lz - 1))));
            }
    }
    w.pod<uint8_t>(0);   // no CASSCF active-space occupations (version 5)
    w.pod<uint8_t>(0);   // no CASSCF active-orbital window (version 6)
    if (!w.good()) return fail(PFK_ERR_INVALID, std::string("I/O error while writing checkpoint: ") + path);
    return PFK_OK;
}

pfk_status pfk_checkpoint_read_density(const char *path, int nbasis, int target_uhf, int n_alpha, int n_beta,
                                       double *Pa, double *Pb, double *total_energy, int *checkpoint_uhf)
{
    if (!path || !Pa || (target_uhf && !Pb) || nbasis <= 0)
        return fail(PFK_ERR_INVALID, "pfk_checkpoint_read_density: null argument or nbasis <= 0");
    Reader r(path);
    if (!r.open()) return fail(PFK_ERR_INVALID, std::string("Cannot open checkpoint file: ") + path);
    auto bad = [&]() { return fail(PFK_ERR_INVALID, r.err); };

    char magic[8] = {};
    if (!r.exact(magic, 8, "magic")) return bad();
    if (std::memcmp(magic, kMagic, 8) != 0) return fail(PFK_ERR_INVALID, "Not a valid Planck checkpoint file (bad magic)");
    uint32_t version = 0;
    if (!r.pod(version)) return bad();
    if (version < 2 || version > kVersion)
        return fail(PFK_ERR_INVALID, "Checkpoint version mismatch: file=" + std::to_string(version) +
                                         ", expected=" + std::to_string(kVersion));
    uint64_t nb = 0;
    uint8_t uhf = 0, conv = 0;
    uint32_t iters = 0;
    double etot = 0.0, enuc = 0.0;
    if (!r.pod(nb) || !r.pod(uhf) || !r.pod(conv) || !r.pod(iters) || !r.pod(etot) || !r.pod(enuc)) return bad();
    uint64_t natoms = 0;
    if (!r.pod(natoms)) return bad();
    if (natoms > kMaxAtoms)
        return fail(PFK_ERR_INVALID, "Checkpoint geometry block atom count " + std::to_string(natoms) +
                                         " exceeds supported limit " + std::to_string(kMaxAtoms));
    int32_t charge = 0;
    uint32_t mult = 0;
    if (!r.pod(charge) || !r.pod(mult)) return bad();
    for (uint64_t a = 0; a < natoms; ++a) {
        int32_t z = 0;
        if (!r.pod(z)) return bad();
    }
    for (uint64_t a = 0; a < 3 * natoms; ++a) {
        double x = 0.0;
        if (!r.pod(x)) return bad();
    }
    std::string basis_name;
    if (!r.string(basis_name)) return bad();
    uint8_t has_opt = 0;
    if (!r.pod(has_opt)) return bad();
    if (nb != static_cast<uint64_t>(nbasis))
        return fail(PFK_ERR_INVALID, "Checkpoint nbasis (" + std::to_string(nb) + ") does not match current nbasis (" +
                                         std::to_string(nbasis) +
                                         "); use the same basis set or remove the checkpoint file.");

    int64_t rows = 0, cols = 0;
    if (!r.matrix(nullptr, rows, cols, nb, "overlap matrix")) return bad();
    if (!r.matrix(nullptr, rows, cols, nb, "core Hamiltonian")) return bad();
    std::vector<double> dens[2], mo[2];
    int64_t mo_cols[2] = {0, 0};
    for (int ch = 0; ch < (uhf ? 2 : 1); ++ch) {
        const std::string label = ch ? "beta" : "alpha";
        if (!r.matrix(&dens[ch], rows, cols, nb, label + " density")) return bad();
        if (rows != nbasis || cols != nbasis)
            return fail(PFK_ERR_INVALID, "Checkpoint " + label + " density is " + std::to_string(rows) + "x" +
                                             std::to_string(cols) + ", not nbasis x nbasis");
        if (!r.matrix(nullptr, rows, cols, nb, label + " fock")) return bad();
        int64_t ne = 0;
        if (!r.vector(ne, nb, label + " orbital energies")) return bad();
        if (!r.matrix(&mo[ch], rows, mo_cols[ch], nb, label + " MO coefficients")) return bad();
        if (mo_cols[ch] > 0 && rows != nbasis)
            return fail(PFK_ERR_INVALID, "Checkpoint " + label + " MO coefficients have " + std::to_string(rows) +
                                             " rows, not nbasis");
    }
    if (version >= 3) {   // CASSCF orbitals are read past, as the reference does
        uint8_t has_cas = 0;
        if (!r.pod(has_cas)) return bad();
        if (has_cas && !r.matrix(nullptr, rows, cols, nb, "CASSCF MO coefficients")) return bad();
    }

    // spin adaptation to the target (checkpoint.cpp:294-336)
    const size_t n2 = static_cast<size_t>(nbasis) * nbasis;
    if (uhf) {
        if (target_uhf) {
            std::memcpy(Pa, dens[0].data(), sizeof(double) * n2);
            std::memcpy(Pb, dens[1].data(), sizeof(double) * n2);
        } else {
            for (size_t k = 0; k < n2; ++k) Pa[k] = dens[0][k] + dens[1][k];
        }
    } else if (!target_uhf) {
        std::memcpy(Pa, dens[0].data(), sizeof(double) * n2);
    } else {
        // an RHF checkpoint for a spin-resolved target: P_s = C_occ(s) C_occ(s)^T
        for (int s = 0; s < 2; ++s) {
            const int nocc = s ? n_beta : n_alpha;
            double *Ps = s ? Pb : Pa;
            std::memset(Ps, 0, sizeof(double) * n2);
            if (nocc <= 0 || mo_cols[0] == 0) continue;
            if (nocc > mo_cols[0])
                return fail(PFK_ERR_INVALID, "Checkpoint orbital block has " + std::to_string(mo_cols[0]) +
                                                 " columns but " + std::to_string(nocc) +
                                                 " occupied orbitals are required");
            const double *C = mo[0].data();   // column-major, nbasis rows
            for (int j = 0; j < nbasis; ++j)
                for (int i = 0; i < nbasis; ++i) {
                    double v = 0.0;
                    for (int o = 0; o < nocc; ++o) v += C[(size_t)o * nbasis + i] * C[(size_t)o * nbasis + j];
                    Ps[(size_t)j * nbasis + i] = v;
                }
        }
    }
    if (total_energy) *total_energy = etot;
    if (checkpoint_uhf) *checkpoint_uhf = uhf ? 1 : 0;
    return PFK_OK;
}

}  // extern "C"
