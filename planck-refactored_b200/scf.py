"""RHF driver around the GPU Fock build: the loop Planck's run_rhf runs
(src/scf/scf.cpp:175-441), with the two-electron part from a FockEngine.

Steps, as the reference takes them:
  * symmetric orthogonaliser X = S^-1/2 (scf.cpp:15-20);
  * default guess: eigenvectors of X^T H X, P = 2 C_occ C_occ^T
    (scf.cpp:33-45, SCFGuess::HCore, types.h:329-347); a caller-supplied
    density enters like the reference's ReadDensity guess (scf.cpp:213-216);
  * per iteration F = H + G(P), E = 1/2 sum P (H + F) + E_nuc, Pulay DIIS over
    the last 8 Fock matrices with error X^T (F P S - S P F) X
    (types.h:759-837), diagonalisation of X^T F X, new P;
  * converged when |dE| < 1e-10 and the rms and max of dP are below 1e-10,
    not before the second iteration (scf.cpp:126-135); at most 50/100/200/300
    iterations by basis size (types.h:356-363).

Everything here is FP64 on the host, as the reference keeps DIIS and the
diagonalisation.  Options beyond the reference:
  * `incremental`: G(P_n) = G(P_{n-1}) + G(P_n - P_{n-1}) with the
    difference-density build in FP32 (a second context whose whole quartet
    list is on the FP32 path, with density screening at 1e-12: quartets
    whose Schwarz bound times the largest difference-density block they
    touch is below it are skipped) while the density steps are small but not
    yet near convergence (max|dP| between 1e-8 and 1e-4), a full FP64 build
    at least every `full_every` iterations, and one for the final energy;
  * the learned-guess hook (guess.py) supplies P0 and the acceptance rule.
"""
import numpy as np
import scipy.linalg as sla

from .basis import ANGSTROM_TO_BOHR  # noqa: F401  (re-exported for callers building geometries)


def nuclear_repulsion(coords, charges):
    e = 0.0
    n = len(charges)
    for i in range(n):
        for j in range(i):
            e += charges[i] * charges[j] / np.linalg.norm(coords[i] - coords[j])
    return e


def max_cycles(nb):
    """types.h:356-363"""
    return 300 if nb > 1000 else 200 if nb > 500 else 100 if nb > 250 else 50


def orthogonaliser(S):
    s, U = np.linalg.eigh(S)
    return (U * (1.0 / np.sqrt(s))) @ U.T


def hcore_density(H, X, nocc):
    _, Cp = np.linalg.eigh(X.T @ H @ X)
    C = X @ Cp[:, :nocc]
    return 2.0 * C @ C.T


def _lstsq_pivoted(A, b):
    """Least squares by column-pivoted QR with a relative rank cut-off of
    n * eps * |R_00| (the solver the reference's DIIS uses, types.h:813)."""
    Q, R, piv = sla.qr(A, pivoting=True)
    d = np.abs(np.diag(R))
    rank = int(np.count_nonzero(d > np.finfo(float).eps * len(d) * d[0]))
    x = np.zeros(A.shape[1])
    if rank:
        x[piv[:rank]] = sla.solve_triangular(R[:rank, :rank], (Q.T @ b)[:rank])
    return x


class Pulay:
    """DIIS over the last `depth` Fock matrices and error vectors."""

    def __init__(self, depth=8):
        self.depth, self.F, self.E = depth, [], []

    def add(self, F, e):
        self.F = (self.F + [F.copy()])[-self.depth:]
        self.E = (self.E + [e.copy()])[-self.depth:]

    def fock(self):
        m = len(self.F)
        if m < 2:
            return self.F[-1]
        B = -np.ones((m + 1, m + 1))
        B[m, m] = 0.0
        for i in range(m):
            for j in range(i, m):
                B[i, j] = B[j, i] = float(np.vdot(self.E[i], self.E[j]))
        rhs = np.zeros(m + 1)
        rhs[m] = -1.0
        c = _lstsq_pivoted(B, rhs)
        return sum(c[i] * self.F[i] for i in range(m))


def first_energy(H, enuc, P, G):
    """Energy of one Fock build on density P (the acceptance test of a guess)."""
    F = H + G
    return 0.5 * float(np.sum(P * (H + F))) + enuc


def rhf(engine, H, S, enuc, nocc, P0=None, G0=None, max_iter=None, tol_e=1e-10, tol_d=1e-10, diis_depth=8,
        incremental=None, full_every=8, incremental_below=1e-4, incremental_floor=1e-8):
    """Run RHF to convergence.  engine: FockEngine (its fock_rhf gives
    G = J - K/2).  P0: starting density (default: the core-Hamiltonian
    guess); G0: G(P0) if the caller already built it (the guess hook does).
    incremental: an optional second FockEngine on the same basis set to
    mixed precision with an fp32_bound above every Schwarz bound, used for
    the difference-density builds while incremental_floor <= max|P - P_built|
    < incremental_below
    (an FP32 build of a large difference would carry ~1e-7 relative errors
    into every later G until the next full build), with a full build at
    least every full_every iterations.  Below incremental_floor the steps are
    within reach of the 1e-10 tests, and the quartets the difference builds
    screen out (each under 1e-12) add up to errors of that order, so those
    last iterations use full builds.  Returns a dict with energy,
    iterations, converged, P, C, eps, history and the first-iteration
    energy."""
    nb = H.shape[0]
    X = orthogonaliser(S)
    P = hcore_density(H, X, nocc) if P0 is None else np.array(P0, dtype=np.float64)
    max_iter = max_iter or max_cycles(nb)
    diis = Pulay(diis_depth)
    E_prev, G, P_built, history, E_first, since_full = 0.0, None, None, [], None, 0
    for it in range(1, max_iter + 1):
        if it == 1 and G0 is not None:
            G = np.array(G0, dtype=np.float64)
            since_full = 0
        elif (incremental is not None and G is not None and since_full + 1 < full_every
              and incremental_floor <= float(np.abs(P - P_built).max()) < incremental_below):
            G = G + incremental.fock_rhf(P - P_built)
            since_full += 1
        else:
            G = engine.fock_rhf(P)
            since_full = 0
        P_built = P
        F = H + G
        E = 0.5 * float(np.sum(P * (H + F))) + enuc
        if E_first is None:
            E_first = E
        diis.add(F, X.T @ (F @ P @ S - S @ P @ F) @ X)
        eps, Cp = np.linalg.eigh(X.T @ diis.fock() @ X)
        C = X @ Cp
        Pn = 2.0 * C[:, :nocc] @ C[:, :nocc].T
        dP = Pn - P
        dE, dmax, drms = abs(E - E_prev), float(np.abs(dP).max()), float(np.sqrt(np.mean(dP * dP)))
        history.append((it, E, dE, drms, dmax))
        P, E_prev = Pn, E
        if it > 1 and dE < tol_e and drms < tol_d and dmax < tol_d:
            if incremental is not None:   # report the energy of a full build at the converged density
                E_prev = first_energy(H, enuc, P, engine.fock_rhf(P))
            return {"energy": E_prev, "iterations": it, "converged": True, "P": P, "C": C, "eps": eps,
                    "history": history, "first_energy": E_first}
    return {"energy": E_prev, "iterations": max_iter, "converged": False, "P": P, "C": C, "eps": eps,
            "history": history, "first_energy": E_first}


def rhf_device(engine, H, S, enuc, nocc, P0=None, max_iter=None, tol_e=1e-10, tol_d=1e-10, diis_depth=8):
    """The loop of rhf() with its linear algebra on the GPU: the density stays
    in HBM and feeds pfk_fock_rhf_device (one captured graph, replayed every
    iteration), and F, the DIIS errors and products, the diagonalisation
    (torch.linalg.eigh: cuSOLVER) and the convergence tests run there in
    FP64; only the DIIS system (at most 9 x 9) is solved on the host, with the
    same pivoted QR.  Not in the reference, which keeps this on the host; the
    steps are rhf()'s, so it converges to the same energy, though the
    eigensolver's rounding can move the iteration that first meets the 1e-10
    tests.  Returns rhf()'s dict (numpy arrays) plus build_seconds, the device
    time of the Fock builds."""
    import torch
    dev = torch.device("cuda", getattr(engine, "device", 0))
    f64 = dict(dtype=torch.float64, device=dev)
    nb = H.shape[0]
    Ht, St = torch.tensor(H, **f64), torch.tensor(S, **f64)
    X = torch.tensor(orthogonaliser(S), **f64)
    P = torch.tensor(hcore_density(H, orthogonaliser(S), nocc) if P0 is None else P0, **f64)
    dP, dG = torch.empty_like(P), torch.empty_like(P)
    # one non-default stream for torch's work and the build, so that they are
    # ordered (a null handle would send the build to the context's own stream)
    stream = torch.cuda.Stream(dev)
    with torch.cuda.stream(stream):
        return _rhf_device_loop(engine, Ht, St, X, P, dP, dG, stream, enuc, nocc, nb, max_iter, tol_e, tol_d,
                                diis_depth)


def _rhf_device_loop(engine, Ht, St, X, P, dP, dG, stream, enuc, nocc, nb, max_iter, tol_e, tol_d, diis_depth):
    import torch
    max_iter = max_iter or max_cycles(nb)
    Fs, Es = [], []
    E_prev, history, E_first, build_ms = 0.0, [], None, 0.0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for it in range(1, max_iter + 1):
        dP.copy_(P)
        ev[0].record(stream)
        engine.fock_rhf_device(dP.data_ptr(), dG.data_ptr(), stream.cuda_stream)
        ev[1].record(stream)
        F = Ht + dG
        E = 0.5 * float(torch.sum(P * (Ht + F))) + enuc
        build_ms += ev[0].elapsed_time(ev[1])
        if E_first is None:
            E_first = E
        err = X.T @ (F @ P @ St - St @ P @ F) @ X
        Fs, Es = (Fs + [F])[-diis_depth:], (Es + [err])[-diis_depth:]
        m = len(Fs)
        if m < 2:
            Fx = F
        else:
            Et = torch.stack([e.reshape(-1) for e in Es])
            B = -np.ones((m + 1, m + 1))
            B[m, m] = 0.0
            B[:m, :m] = (Et @ Et.T).cpu().numpy()
            rhs = np.zeros(m + 1)
            rhs[m] = -1.0
            c = _lstsq_pivoted(B, rhs)
            Fx = sum(float(c[i]) * Fs[i] for i in range(m))
        eps, Cp = torch.linalg.eigh(X.T @ Fx @ X)
        C = X @ Cp
        Pn = 2.0 * C[:, :nocc] @ C[:, :nocc].T
        d = Pn - P
        dE = abs(E - E_prev)
        dmax, drms = float(d.abs().max()), float(torch.sqrt(torch.mean(d * d)))
        history.append((it, E, dE, drms, dmax))
        P, E_prev = Pn, E
        if it > 1 and dE < tol_e and drms < tol_d and dmax < tol_d:
            return {"energy": E, "iterations": it, "converged": True, "P": P.cpu().numpy(), "C": C.cpu().numpy(),
                    "eps": eps.cpu().numpy(), "history": history, "first_energy": E_first,
                    "build_seconds": build_ms * 1e-3}
    return {"energy": E_prev, "iterations": max_iter, "converged": False, "P": P.cpu().numpy(), "C": C.cpu().numpy(),
            "eps": eps.cpu().numpy(), "history": history, "first_energy": E_first, "build_seconds": build_ms * 1e-3}


def uhf(engine, H, S, enuc, n_alpha, n_beta, P0=None, max_iter=None, tol_e=1e-10, tol_d=1e-10, diis_depth=8):
    """UHF to convergence (the loop of run_uhf, src/scf/scf.cpp:467-930) on
    FockEngine.fock_uhf (Ga = J(Pa+Pb) - K(Pa), Gb = J(Pa+Pb) - K(Pb)).
    Guess: per spin, the n_s lowest eigenvectors of X^T H X
    (scf.cpp:505-511), or P0 = (Pa, Pb).  Per iteration
    E = 1/2 sum[(Pa + Pb) H + Pa Fa + Pb Fb] + E_nuc; one Pulay extrapolation
    of (Fa, Fb) with the joint error (X^T (Fs Ps S - S Ps Fs) X)_s; converged
    when |dE| and the rms and max of both density steps are below the
    thresholds, not before the second iteration.  Returns energy,
    iterations, converged, Pa, Pb, Ca, Cb, eps_a, eps_b, history."""
    nb = H.shape[0]
    X = orthogonaliser(S)
    if P0 is None:
        _, Cp = np.linalg.eigh(X.T @ H @ X)
        C = X @ Cp
        Pa, Pb = C[:, :n_alpha] @ C[:, :n_alpha].T, C[:, :n_beta] @ C[:, :n_beta].T
    else:
        Pa, Pb = (np.array(p, dtype=np.float64) for p in P0)
    max_iter = max_iter or max_cycles(nb)
    diis = Pulay(diis_depth)
    E_prev, history = 0.0, []
    for it in range(1, max_iter + 1):
        Ga, Gb = engine.fock_uhf(Pa, Pb)
        Fa, Fb = H + Ga, H + Gb
        E = 0.5 * float(np.sum((Pa + Pb) * H + Pa * Fa + Pb * Fb)) + enuc
        err = np.stack([X.T @ (F @ Ps @ S - S @ Ps @ F) @ X for F, Ps in ((Fa, Pa), (Fb, Pb))])
        diis.add(np.stack([Fa, Fb]), err)
        Fx = diis.fock()
        out = []
        for F, n in ((Fx[0], n_alpha), (Fx[1], n_beta)):
            eps, Cp = np.linalg.eigh(X.T @ F @ X)
            C = X @ Cp
            out.append((eps, C, C[:, :n] @ C[:, :n].T))
        (eps_a, Ca, Pan), (eps_b, Cb, Pbn) = out
        dPa, dPb = Pan - Pa, Pbn - Pb
        dE = abs(E - E_prev)
        dmax = max(float(np.abs(dPa).max()), float(np.abs(dPb).max()))
        drms = max(float(np.sqrt(np.mean(dPa * dPa))), float(np.sqrt(np.mean(dPb * dPb))))
        history.append((it, E, dE, drms, dmax))
        Pa, Pb, E_prev = Pan, Pbn, E
        if it > 1 and dE < tol_e and drms < tol_d and dmax < tol_d:
            return {"energy": E, "iterations": it, "converged": True, "Pa": Pa, "Pb": Pb, "Ca": Ca, "Cb": Cb,
                    "eps_a": eps_a, "eps_b": eps_b, "history": history}
    return {"energy": E_prev, "iterations": max_iter, "converged": False, "Pa": Pa, "Pb": Pb, "Ca": Ca, "Cb": Cb,
            "eps_a": eps_a, "eps_b": eps_b, "history": history}


class System:
    """A molecule on one GPU: basis shells, one-electron matrices from the
    device (pfk_one_electron), nuclear repulsion and a FockEngine."""

    def __init__(self, atoms, basis_name, library, device=0, engine="os", precision="fp64", fp32_bound=1e-8):
        from . import FockEngine, one_electron, shells_for
        self.mol, self.shells = shells_for(atoms, basis_name, library)
        self.basis_name = basis_name
        S, T, V = one_electron(self.shells, self.mol.coords, self.mol.Z, device)
        self.S, self.H = S, T + V
        self.enuc = nuclear_repulsion(self.mol.coords, self.mol.Z)
        self.nocc = self.mol.nelectron() // 2
        self.engine = FockEngine(self.shells, device=device, engine=engine, precision=precision,
                                 fp32_bound=fp32_bound)
        self.device = device
        self._incr = None

    def incremental_engine(self):
        if self._incr is None:
            from . import FockEngine
            self._incr = FockEngine(self.shells, device=self.device, engine=self.engine.engine, precision="mixed",
                                    fp32_bound=1e300)
            self._incr.set_density_screening(1e-12)
        return self._incr

    def run(self, P0=None, incremental=False, linalg="host", **kw):
        """RHF to convergence.  linalg="host": rhf() (numpy linear algebra);
        "gpu": the whole loop behind the C ABI (pfk_scf_rhf: DIIS and
        diagonalisation on the device, no Python per iteration), with the
        difference-density builds when incremental is set; "device": the torch
        loop rhf_device."""
        if linalg == "gpu":
            G0 = kw.pop("G0", None)
            return self.engine.scf_rhf(self.H, self.S, self.enuc, self.nocc, P0=P0, G0=G0,
                                       incremental=self.incremental_engine() if incremental else None, **kw)
        if linalg == "device":
            if incremental:
                raise ValueError("the device loop has no difference-density builds")
            kw.pop("G0", None)   # the device loop makes its first build itself
            return rhf_device(self.engine, self.H, self.S, self.enuc, self.nocc, P0=P0, **kw)
        return rhf(self.engine, self.H, self.S, self.enuc, self.nocc, P0=P0,
                   incremental=self.incremental_engine() if incremental else None, **kw)

    def close(self):
        self.engine.close()
        if self._incr is not None:
            self._incr.close()
