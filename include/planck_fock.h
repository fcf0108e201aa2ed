/*
 * planck_fock.h -- C ABI of the B200 direct-SCF Fock-build engine.
 *
 * Drop-in for the two-electron part of Planck's SCF: the entry points below
 * replace the functions callers reach through src/integrals/base.h
 * (reference project paths):
 *
 *   _compute_2e        base.h:39-55   -> pfk_eri_tensor
 *   _compute_2e_fock   base.h:57-73   -> pfk_fock_rhf   (G = J - K/2)
 *   _compute_2e_fock_uhf base.h:75-93 -> pfk_fock_uhf   (G_a, G_b)
 *   build_coulomb_from_eri / build_exchange_from_eri
 *                      src/dft/driver.cpp:689-731 -> pfk_jk
 *   _compute_schwarz_table os.cpp:1703-1752 / rys.cpp:509-556 -> pfk_schwarz
 *   the screened quartet loop os.cpp:1458-1476 -> pfk_quartet_count / _list
 *
 * Conventions
 *   - Basis data is the reference's Shell data (src/base/types.h:263-275):
 *     centre in Bohr, L, primitive exponents, contraction coefficients with
 *     the contracted normalisation already folded in (gaussian.cpp:273-281),
 *     and per-primitive normalisations (basis.cpp:39-48).  Shells appear in
 *     the reference's order; each shell expands to (L+1)(L+2)/2 Cartesian
 *     functions ordered lx descending, then ly descending (basis.cpp:20-37),
 *     with component norms 1/sqrt((2lx-1)!!(2ly-1)!!(2lz-1)!!)
 *     (gaussian.cpp:283-296).  0 <= L <= 3.
 *   - Matrices are nbasis x nbasis FP64.  Densities must be symmetric (every
 *     SCF density is); G, J and K come back symmetric, so row- and
 *     column-major storage coincide (the reference's Eigen matrices are
 *     column-major).
 *   - tol_eri screens canonical AO quartets exactly as the reference does:
 *     a quartet is skipped when Q(i,j)*Q(k,l) < tol_eri, Q = sqrt|(ij|ij)|.
 *   - Every call returns a status; nothing throws across the ABI.  A failed
 *     call leaves a message in pfk_last_error(ctx).
 *   - A context owns its device memory, stream and captured graphs.  It is
 *     single-threaded; use one context per molecule (several may coexist).
 */
#ifndef PLANCK_FOCK_H
#define PLANCK_FOCK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PFK_OK = 0,
    PFK_ERR_INVALID = 1,     /* bad argument or basis data */
    PFK_ERR_UNSUPPORTED = 2, /* e.g. L > 3, non-null symmetry operations */
    PFK_ERR_CUDA = 3,        /* CUDA runtime error (message in pfk_last_error) */
    PFK_ERR_NOMEM = 4,       /* device or host allocation failed */
    PFK_ERR_STATE = 5        /* call out of order (e.g. null context) */
} pfk_status;

/* IntegralMethod (src/base/types.h:88-100): OS, Rys, Auto. */
typedef enum { PFK_ENGINE_OS = 0, PFK_ENGINE_RYS = 1, PFK_ENGINE_AUTO = 2 } pfk_engine;

/* FP64 everywhere, or FP32 for quartets whose Schwarz bound is below
 * fp32_bound (Boys values, roots/weights, Fock accumulation stay FP64).
 * Classes with an f shell stay FP64 in either mode. */
typedef enum { PFK_PREC_FP64 = 0, PFK_PREC_MIXED = 1 } pfk_precision;

typedef struct {
    int nshell;
    const int *L;          /* [nshell] angular momentum, 0..3 */
    const int *nprim;      /* [nshell] primitives per shell */
    const double *center;  /* [3*nshell] Bohr */
    const double *expo;    /* [sum nprim] Shell::_primitives */
    const double *coef;    /* [sum nprim] Shell::_coefficients (Nc folded in) */
    const double *norm;    /* [sum nprim] Shell::_normalizations */
} pfk_basis_desc;

typedef struct pfk_ctx pfk_ctx;

/* Build the context on CUDA device `device`: uploads shell-pair data,
 * computes the Schwarz table and the screened quartet lists for tol_eri
 * = 1e-10 (OptionsIntegral default, types.h:408-412).  Replaces the
 * per-call Schwarz table of os.cpp:1447. */
pfk_status pfk_create(const pfk_basis_desc *basis, int device, pfk_ctx **out);
pfk_status pfk_destroy(pfk_ctx *ctx);

/* OptionsIntegral (types.h:408-412): tol_eri and engine.  precision and
 * fp32_bound select the mixed-precision path.  Rebuilds the quartet lists
 * when tol_eri or fp32_bound change. */
pfk_status pfk_set_options(pfk_ctx *ctx, double tol_eri, int engine, int precision,
                           double fp32_bound);

int pfk_nbasis(const pfk_ctx *ctx);
const char *pfk_last_error(const pfk_ctx *ctx);

/* Schwarz table Q(i,j) = sqrt|(ij|ij)|, nbasis x nbasis, host buffer.
 * Counterpart of _compute_schwarz_table (os.cpp:1703-1752). */
pfk_status pfk_schwarz(pfk_ctx *ctx, double *Q);

/* Screened canonical AO quartet set (os.cpp:1458-1476): count, an order-
 * independent 64-bit digest (sum over quartets of mix64 of the packed
 * i<<48|j<<32|k<<16|l code with i<=j, k<=l, (i,j)<=(k,l)), and the number
 * of shell quartets the kernels evaluate. */
pfk_status pfk_quartet_count(pfk_ctx *ctx, long long *n_ao_quartets, uint64_t *digest,
                             long long *n_shell_quartets);

/* The AO quartets themselves (4 ints each, canonical, unordered); up to cap. */
pfk_status pfk_quartet_list(pfk_ctx *ctx, int *out, long long cap, long long *n);

/* RHF: G = J(P) - K(P)/2.  _compute_2e_fock (base.h:57-73, os.cpp:1435-1523). */
pfk_status pfk_fock_rhf(pfk_ctx *ctx, const double *P, double *G);

/* UHF: Ga = J(Pa+Pb) - K(Pa), Gb = J(Pa+Pb) - K(Pb).
 * _compute_2e_fock_uhf (base.h:75-93, os.cpp:1533-1625). */
pfk_status pfk_fock_uhf(pfk_ctx *ctx, const double *Pa, const double *Pb, double *Ga, double *Gb);

/* RKS/UKS Coulomb and exchange: J = J(P), K = k_scale * K(Pk)
 * (dft/driver.cpp:689-731 builds them from the stored tensor; hybrids scale
 * K by the exact-exchange fraction).  Pk may equal P; K may be NULL. */
pfk_status pfk_jk(pfk_ctx *ctx, const double *P, const double *Pk, double *J, double *K,
                  double k_scale);

/* Device-pointer form of pfk_fock_rhf: dP and dG live on the context's
 * device; the call is asynchronous on `stream` (a cudaStream_t, NULL for the
 * context's own stream).  The first call with a given (dP, dG, stream)
 * captures the whole build in a CUDA graph and later calls replay it. */
pfk_status pfk_fock_rhf_device(pfk_ctx *ctx, const double *dP, double *dG, void *stream);

/* Conventional build: the full nbasis^4 tensor, row-major
 * i*nb^3 + j*nb^2 + k*nb + l, all 8 permutations written
 * (_compute_2e, os.cpp:1755-1829).  Host buffer of nb^4 doubles. */
pfk_status pfk_eri_tensor(pfk_ctx *ctx, double *eri);

/* AO -> MO transform of the stored tensor, the consumer behind MP2 and the
 * stability analysis (transform_eri, src/post_hf/integrals.cpp:63-134):
 *   out[i][a][j][b] = sum_{mu nu lam sig} C1(mu,i) C2(nu,a) C3(lam,j) C4(sig,b)
 *                     (mu nu|lam sig),
 * row-major n1 x n2 x n3 x n4 in a host buffer.  C_k are host nbasis x n_k
 * matrices, column-major (the reference's Eigen MO blocks), 1 <= n_k <=
 * nbasis.  The AO tensor is built on the device by the class kernels
 * (as pfk_eri_tensor, nbasis <= 180) and the four quarter transforms run
 * there as FP64 GEMMs (cuBLAS); nothing of size nbasis^4 crosses to the
 * host. */
pfk_status pfk_mo_transform(pfk_ctx *ctx, const double *C1, int n1, const double *C2, int n2, const double *C3,
                            int n3, const double *C4, int n4, double *out);

/* Device time in ms of the last pfk_mo_transform on this context, from CUDA
 * events on its stream: ms3[0] the AO tensor (clear + class kernels),
 * ms3[1] the four quarter-transform GEMMs, ms3[2] the copy of the result to
 * the host.  For measurement. */
pfk_status pfk_mo_transform_times(const pfk_ctx *ctx, double *ms3);

/* RMP2 correlation energy of a converged RHF (run_rmp2,
 * src/post_hf/mp2.cpp:10-38, with the amplitudes of mp2_gradient.cpp:203-232):
 *   E = sum_{iajb} (ia|jb) [2 (ia|jb) - (ib|ja)] / (e_i + e_j - e_a - e_b).
 * C: host nbasis x nbasis MO coefficients, column-major, the nocc occupied
 * orbitals first; eps: their nbasis orbital energies.  The (ov|ov) block is
 * made as by pfk_mo_transform and summed on the device, so it never crosses
 * to the host; pfk_mo_transform_times then reports the sum as its third
 * phase.  nbasis <= 180. */
pfk_status pfk_rmp2_energy(pfk_ctx *ctx, const double *C, const double *eps, int nocc, double *e_corr);

/* UMP2 correlation energy of a converged UHF (run_ump2,
 * src/post_hf/mp2.cpp:43-143): the alpha-alpha and beta-beta terms
 * 1/4 sum [(ia|jb) - (ib|ja)]^2 / D and the alpha-beta term sum (ia|jb)^2 / D
 * over three device-resident (ov|ov) blocks, transformed as by
 * pfk_mo_transform from one AO tensor built once, and summed where they were
 * made.  Ca, Cb: host nbasis x
 * nbasis MO coefficients per spin, column-major, occupied first; eps_a, eps_b
 * their orbital energies.  nbasis <= 180. */
pfk_status pfk_ump2_energy(pfk_ctx *ctx, const double *Ca, const double *eps_a, const double *Cb, const double *eps_b,
                           int n_alpha, int n_beta, double *e_corr);

/* Per-class work of one build over the 55 classes (ss|ss)..(ff|ff):
 * screened shell quartets, primitive quartets (sum of K_ab * K_cd), and --
 * when ms55 is non-null -- the device time of each class's kernel in a
 * timed RHF build on the context's current density, in milliseconds.
 * Any output pointer may be NULL.  For profiling and roofline reports. */
pfk_status pfk_class_stats(pfk_ctx *ctx, long long *quartets55, long long *prim_quartets55,
                           double *ms55);

/* The FP32 list of the mixed-precision builds per class: its screened shell
 * quartets and primitive quartets (zero in FP64 mode).  The rest of each
 * class (pfk_class_stats) runs in FP64.  Any output may be NULL. */
pfk_status pfk_precision_stats(pfk_ctx *ctx, long long *fp32_quartets55, long long *fp32_prim_quartets55);

/* Restrict every later build of this context to shard `rank` of `nranks`:
 * of each class's screened quartet list (ordered by primitive loop length)
 * only every nranks-th quartet starting at `rank` is evaluated, so the
 * shards carry equal mixes of work and the partial G (or J, K) of all ranks
 * sum to the full result.  nranks = 1 restores the whole list.  Used by
 * one-process-per-GPU runs, which sum the partial matrices with one
 * all-reduce. */
pfk_status pfk_set_shard(pfk_ctx *ctx, int rank, int nranks);

/* Density screening for builds on a difference density (incremental SCF):
 * with dtol > 0, every later build of this context first takes the largest
 * |P| of each shell-pair block over the densities it is given, and skips
 * every shell quartet whose Schwarz bound qmax(ab) qmax(cd) times the
 * largest of its six density blocks is below dtol.  A build on a full
 * density does not want this (its result would no longer be the
 * reference's); dtol = 0 turns it off.  Not in the reference. */
pfk_status pfk_set_density_screening(pfk_ctx *ctx, double dtol);

/* Concurrent class launches: every later build of this context issues its
 * class kernels on `lanes` streams (1 to 4; default 4) forked from the
 * build's stream and joined back before the J/K combine, so that one class's
 * tail and the small classes overlap the others.  Classes go, largest
 * (primitive quartets x component quartets) first, to the lane with the
 * least work.  lanes = 1 issues them in class order on the build's stream.
 * The results are bitwise identical for every lane count: the J/K
 * accumulation is in fixed-point integers, whose sums do not depend on the
 * order of the additions.
 * Not in the reference (its loop over quartets is one OpenMP region). */
pfk_status pfk_set_lanes(pfk_ctx *ctx, int lanes);

/* Primitive screening: every later build of this context skips the
 * primitive quartets whose bound qp(ab) qp(cd) is below ptol, where qp of a
 * primitive pair is the largest sqrt|(ab|ab)| over its Cartesian components
 * for that primitive pair alone (coefficients and norms included).  By the
 * Cauchy-Schwarz inequality a skipped primitive quartet adds less than ptol
 * to every integral it touches.  Default 1e-16; 0 evaluates every primitive
 * pair kept at setup (those that can reach 1e-21 with some partner).
 * 0 <= ptol <= 1e-10.  Not in the reference, which evaluates every
 * primitive quartet of a surviving shell quartet. */
pfk_status pfk_set_primitive_tol(pfk_ctx *ctx, double ptol);

/* Autotuner for engine auto: times every candidate kernel of every class on
 * this context's screened lists (a warm-up pass, then the faster of two timed
 * passes) and keeps the fastest per class for the builds made with engine
 * auto.  Candidates: 0 = Rys, 2 = Obara-Saika, 6 = Obara-Saika compiled for
 * more blocks of 128 threads per SM (8 for LA+LB+LC+LD <= 1, 6 for 2, 4
 * above: fewer registers per thread); the last two exist for classes with
 * LA+LB+LC+LD <= 4, the others always run Rys.  Until it runs, engine auto
 * uses the reference's outcome (OS for L <= 4, Rys above).  choice55 (may be
 * NULL) receives the chosen candidate per class, ms55x3 (may be NULL) the
 * measured milliseconds per class and candidate (0 when not applicable).
 * The reference chooses per component quartet from a cost model
 * (rys.cpp:195-236); this chooses per class from measurements. */
pfk_status pfk_autotune(pfk_ctx *ctx, int *choice55, double *ms55x3);

/* Measurement helper: sustained FP64 and FP32 fused-multiply-add throughput
 * of `device` in TFLOP/s (2 flops per FMA), from a register-resident FMA
 * loop over all SMs, timed with CUDA events.  The FP64 figure is the
 * roofline denominator of the integral kernels. */
pfk_status pfk_measure_fma_peak(int device, double *fp64_tflops, double *fp32_tflops);

/* ---- ERI batches --------------------------------------------------------
 * The contracted, normalised Cartesian block of every listed shell quartet,
 * from the class kernels of the Fock builds, written to device memory
 * instead of digested: the per-quartet integrals of the reference's
 * _contracted_eri (os.cpp:994-1010) and _rys_contracted_eri
 * (rys.cpp:489-505), all components of a shell quartet at once, every
 * primitive quartet evaluated, no Schwarz screening.  For the per-class
 * throughput and accuracy measurements of the integral kernels.
 *
 * pfk_eri_batch_create: shells as for pfk_create; pair_shells[2p], [2p+1]
 * are the shells (A, B) of pair p, with L(A) >= L(B).
 * pfk_eri_batch_set_quartets: host list of (bra pair, ket pair) ids, all of
 * one class with class(bra) >= class(ket) in the pair-class order ss, ps,
 * pp, ds, dp, dd, fs, fp, fd, ff; uploads it.  cls (may be NULL) receives
 * the quartet class (0..54), ncomp the components per quartet.
 * pfk_eri_batch_run: quartets first .. first+count-1 of the list into d_out
 * (device, count * ncomp doubles; quartet t's block at t * ncomp, component
 * ((ia*NB + ib)*NC + ic)*ND + id in the reference's Cartesian order),
 * asynchronous on `stream` (NULL: the batch's own).  engine: PFK_ENGINE_OS
 * (classes with LA+LB+LC+LD <= 4; PFK_ERR_UNSUPPORTED above) or
 * PFK_ENGINE_RYS; precision PFK_PREC_FP64, or PFK_PREC_MIXED for the FP32
 * variant (recurrences, transfers and contraction in FP32; Boys values, Rys
 * roots and weights and the per-primitive scalars in FP64). */
typedef struct pfk_eri_batch pfk_eri_batch;
pfk_status pfk_eri_batch_create(const pfk_basis_desc *basis, int npairs, const int *pair_shells, int device,
                                pfk_eri_batch **out);
pfk_status pfk_eri_batch_destroy(pfk_eri_batch *b);
const char *pfk_eri_batch_last_error(const pfk_eri_batch *b);
pfk_status pfk_eri_batch_set_quartets(pfk_eri_batch *b, const int *quartets, long long n, int *cls, int *ncomp);
pfk_status pfk_eri_batch_run(pfk_eri_batch *b, long long first, long long count, int engine, int precision,
                             double *d_out, void *stream);

/* ---- RHF on the device -------------------------------------------------
 * The loop of the reference's run_rhf (src/scf/scf.cpp:175-441) with the
 * context's Fock builds, all FP64 on the device: symmetric orthogonaliser
 * X = S^-1/2, the core-Hamiltonian guess (or the caller's P0, taken like the
 * reference's ReadDensity guess), F = H + G(P), E = 1/2 sum P (H + F) + E_nuc,
 * Pulay DIIS over the last diis_depth Fock matrices with error
 * X^T (F P S - S P F) X (types.h:759-837; the small DIIS system solved on
 * the host by column-pivoted QR), diagonalisation (cuSOLVER Dsyevd),
 * P = 2 C_occ C_occ^T; converged when |dE| < tol_energy and the rms and max
 * of the density change are below tol_density, not before iteration 2
 * (scf.cpp:126-135).  max_iter 0 takes the reference's limit by basis size
 * (types.h:356-363).  A non-null `incremental` (a second context on the same
 * basis, normally mixed precision with every quartet on the FP32 list and
 * density screening) builds G(P) = G(P_built) + G(P - P_built) while
 * incremental_floor <= max|P - P_built| < incremental_below, with a full
 * build at least every full_every iterations and one for the final energy;
 * not in the reference.  G0 (with P0) is the caller's build of the first
 * iteration (the learned-guess hook makes it).  H, S, P0, G0 and the outputs
 * P_out, C_out (MO coefficients, column-major), eps_out are host arrays and
 * may be NULL where optional; the sums are in a fixed order, so a run is
 * bitwise reproducible.  The loop runs on a stream of its own, launches its
 * builds directly (no graph capture) and returns when done, so calls on
 * different contexts may run at once from several host threads (one
 * context per thread). */
typedef struct {
    int max_iter;              /* 0: the reference's limit by basis size */
    double tol_energy;         /* 1e-10 */
    double tol_density;        /* 1e-10 */
    int diis_depth;            /* 8 */
    pfk_ctx *incremental;      /* NULL: full builds only */
    double incremental_below;  /* 1e-4 */
    double incremental_floor;  /* 1e-8 */
    int full_every;            /* 8 */
    double *history;           /* NULL, or 6 doubles per iteration (host): iteration, E, |dE|, rms dP,
                                  max dP, milliseconds since the call began */
} pfk_scf_options;

typedef struct {
    double energy, first_energy;
    int iterations, converged;
    int full_builds, difference_builds;
    double build_ms;           /* device time of the Fock builds (CUDA events) */
    double total_ms;           /* wall time of the call */
} pfk_scf_result;

pfk_status pfk_scf_rhf(pfk_ctx *ctx, const double *H, const double *S, double enuc, int nocc, const double *P0,
                       const double *G0, const pfk_scf_options *opt, pfk_scf_result *res, double *P_out,
                       double *C_out, double *eps_out);

/* One-electron integrals of the basis: overlap S, kinetic energy T and
 * nuclear attraction V (nbasis x nbasis, host buffers, symmetric), with
 * point nuclei nuclei[4*natom] = (x, y, z in Bohr, charge Z).  Needs no
 * context: runs on CUDA device `device` and returns when S, T, V are written.
 * Counterpart of the reference's host-side Obara-Saika one-electron code
 * (os.cpp:294-602), which the SCF setup calls before the first Fock build
 * (H = T + V, scf.cpp:175-205). */
pfk_status pfk_one_electron(const pfk_basis_desc *basis, int natom, const double *nuclei, double *S, double *T,
                            double *V, int device);

/* ---------------------------------------------------------------------------
 * Learned initial guess: the network.  A multilayer perceptron
 * (dims[0] -> dims[1] -> ... -> dims[nlayers], SiLU between layers, linear
 * output) whose matrix products run on the tensor cores in BF16 with FP32
 * accumulation, trained on the GPU with Adam on the mean squared error.  It
 * has no counterpart in the reference: it predicts the atom-pair density
 * blocks of the guess density that Planck's SCF takes like a ReadDensity
 * guess (scf.cpp:206-240, 213-216).  Parameters are one FP32 vector: per
 * layer the weight matrix W_l (dims[l] x dims[l+1], row-major, Z = H W + b)
 * then the bias b_l.  Widths must be multiples of 8.  X, T, Y are device
 * arrays of n rows (row-major FP32), n <= max_batch; the calls return when
 * their results are written.
 * ------------------------------------------------------------------------- */
typedef struct pfk_mlp pfk_mlp;
pfk_status pfk_mlp_create(int nlayers, const int *dims, int max_batch, int device, pfk_mlp **out);
pfk_status pfk_mlp_destroy(pfk_mlp *m);
const char *pfk_mlp_last_error(const pfk_mlp *m);
long long pfk_mlp_param_count(const pfk_mlp *m);
pfk_status pfk_mlp_set_params(pfk_mlp *m, const float *params);   /* host; resets Adam */
pfk_status pfk_mlp_get_params(pfk_mlp *m, float *params);         /* host */
/* Y = network(X). */
pfk_status pfk_mlp_forward(pfk_mlp *m, const float *X, int n, float *Y, void *stream);
/* Gradients (host vector in the parameter layout, may be NULL) and the loss
 * mean((Y - T)^2) of one batch, without an update. */
pfk_status pfk_mlp_gradients(pfk_mlp *m, const float *X, const float *T, int n, float *grads, double *loss,
                             void *stream);
/* One Adam step (beta 0.9, 0.999, eps 1e-8) with learning rate lr; loss as above. */
pfk_status pfk_mlp_train_step(pfk_mlp *m, const float *X, const float *T, int n, float lr, double *loss,
                              void *stream);

/* Size of the device scratch array behind pfk_fock_rhf_noalloc: 64 MiB,
 * held by every GPU that loads the library until the process exits. */
#define PFK_NOALLOC_SCRATCH_BYTES (64u << 20)

/* RHF build G = J(P) - K(P)/2 that allocates no device memory.  It has no
 * counterpart in the reference.  It is for callers that must not call
 * cudaMalloc or any allocator -- a host program whose GPU memory is owned by
 * another allocator or pool, or one whose memory budget is fixed up front.
 * Every device buffer the build needs (pair data, Schwarz table, screened
 * quartet list, J and K accumulators) lives in one static device array of
 * PFK_NOALLOC_SCRATCH_BYTES; a basis whose data does not fit is rejected with
 * PFK_ERR_UNSUPPORTED and a message giving the bytes needed (roughly up to
 * 200 basis functions of 6-31G** fit).
 *   basis   host shell data, as for pfk_create
 *   dP, dG  nbasis x nbasis densities / result on the current CUDA device
 *   stream  cudaStream_t for the work (NULL: the default stream); the call
 *           synchronises it and returns with dG written.
 * Every call rebuilds the pair data, the Schwarz table and the screened
 * quartet list on the host (it copies the Schwarz table back and
 * synchronises the stream to do so), so it costs host time per call and
 * must never be called inside a stream capture.  The first call on a device
 * also looks up the scratch array's device address and sets kernel
 * attributes on that device.  All calls on a device share the one array:
 * calls that overlap on the GPU (other host threads, other streams) race and
 * must be serialised by the caller.  Each call clears what it needs at zero. */
pfk_status pfk_fock_rhf_noalloc(const pfk_basis_desc *basis, const double *dP, double *dG, double tol_eri,
                                void *stream);

/* ---- Checkpoint files (.hfchk, format version 6) ----------------------
 * The reference's restart file (src/io/checkpoint.h:11-72), so that a density
 * made here -- a learned guess, or a converged GPU SCF -- restarts the
 * reference with `guess density`, and a reference checkpoint restarts this
 * library's driver.  Host code; no GPU is needed.  Files are host byte
 * order with IEEE-754 doubles, like the reference's.  Every nbasis x nbasis
 * array below is column-major (element (i, j) at i + nbasis * j), the layout
 * of the reference's Eigen matrices; for the symmetric ones it does not
 * matter. */

/* Molecule and run data of a checkpoint (the Calculator fields that
 * Checkpoint::save writes, checkpoint.cpp:356-379). */
typedef struct {
    int natoms;
    const int *atomic_numbers;    /* [natoms] */
    const double *coords_bohr;    /* [3*natoms]: x0 y0 z0 x1 y1 z1 ... */
    int charge;
    unsigned int multiplicity;
    const char *basis_name;       /* NUL-terminated, at most 4096 bytes */
    double total_energy;
    double nuclear_repulsion;
    int converged;                /* 0 or 1 */
    int has_opt_coords;           /* 0 or 1 */
} pfk_checkpoint_meta;

/* One spin channel (SpinChannel: density, Fock matrix, orbital energies
 * [nbasis], MO coefficients with MO j in column j). */
typedef struct {
    const double *density;
    const double *fock;
    const double *mo_energies;
    const double *mo_coefficients;
} pfk_spin_channel;

/* Write a checkpoint as Checkpoint::save does (checkpoint.cpp:347-489):
 * header, molecule, S, H, the alpha channel, the beta channel when beta is
 * non-NULL (UHF/ROHF), no CASSCF data, and the shell and basis-function
 * tables of `basis`, whose Cartesian function count is the file's nbasis.
 * An RHF channel holds the total density; a UHF or ROHF reader of an RHF
 * file builds its spin densities from the leading MO columns, so list the
 * occupied orbitals first. */
pfk_status pfk_checkpoint_write(const char *path, const pfk_checkpoint_meta *meta, const pfk_basis_desc *basis,
                                const double *S, const double *H, const pfk_spin_channel *alpha,
                                const pfk_spin_channel *beta);

/* Density restart, as Checkpoint::load with load_1e_matrices = false
 * (checkpoint.cpp:491-663): the same checks and error messages (magic,
 * version 2..6, nbasis, size limits, truncation), then the stored densities
 * adapted to the target like adapt_restart_spin_state
 * (checkpoint.cpp:294-336): UHF file and UHF target -> Pa, Pb as stored;
 * UHF file, RHF target -> Pa = P_alpha + P_beta; RHF file, RHF target -> Pa
 * = the stored density; RHF file, UHF target -> Pa, Pb from the first
 * n_alpha / n_beta MO columns.  Pb may be NULL for an RHF target.  The
 * stored total energy and whether the file is spin-resolved come back in
 * the optional last two arguments. */
pfk_status pfk_checkpoint_read_density(const char *path, int nbasis, int target_uhf, int n_alpha, int n_beta,
                                       double *Pa, double *Pb, double *total_energy, int *checkpoint_uhf);

/* Message of the last failed checkpoint call on this thread. */
const char *pfk_checkpoint_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* PLANCK_FOCK_H */
