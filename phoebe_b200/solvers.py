"""Exact phonon BTE solvers on top of the scattering matrix's products.

Host-side restatement of the solver loops of the reference's phonon
transport application (src/apps/phonon_transport_app.cpp:112-126, 197-383)
and of the vector algebra they use (src/bte/vector_bte.cpp:66-110, 160-290;
src/bte/drift.cpp:3-29; src/observable/phonon_thermal_cond.cpp:58-113,
148-240).  The products with the scattering matrix, which are where the time
goes, run on the GPU through the `PhScatteringMatrix` given (a stored matrix
costs one HBM read of it per product; without one, each product is a builder
pass); the loops themselves act on (nT, 3, numStates) vectors of a few MB.

Vectors follow the reference's VectorBTE: (nT, 3, numStates) with states
s = iq * nb + ib, and every operation leaves excluded states (E < 0.1 cm^-1)
at zero.  Conductivities are (nT, 3, 3) in atomic units; multiply by
constants.thConductivityAuToSi for W/(m K)."""
import numpy as np

from . import constants as C


class BteProblem:
    """Energies, velocities and temperatures of one solve, with the
    reference's derived vectors: the drift dn/dT v (BulkTDrift), n(n+1),
    the excluded states and the conductivity normalisation 1/(Nq V)."""

    def __init__(self, E, vg, temperatures_ry, num_q, volume):
        self.E = np.asarray(E, dtype=np.float64).ravel()
        self.vg = np.asarray(vg, dtype=np.float64).reshape(-1, 3)
        self.T = np.atleast_1d(np.asarray(temperatures_ry, dtype=np.float64))
        self.excluded = self.E < C.phExcludeCutoff
        self.norm = 1.0 / float(num_q) / float(volume)
        with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
            x = np.sinh(self.E[None, :] / 2.0 / self.T[:, None])
            self.popterm = 0.25 / x / x                                  # (nT, ns) n(n+1)
            dndt = self.popterm * self.E[None, :] / self.T[:, None] ** 2
            self.drift = self.clean(dndt[:, None, :] * self.vg.T[None, :, :])   # (nT, 3, ns)

    def clean(self, v):
        """Zero on excluded states (VectorBTE::baseOperator, vector_bte.cpp:171-173)."""
        v = np.array(v, dtype=np.float64, copy=True)
        v[..., self.excluded] = 0.0
        return v

    def vdot(self, a, b):
        """VectorBTE::dot (vector_bte.cpp:66-110): (nT, 3), excluded states skipped."""
        keep = ~self.excluded
        return np.einsum("cis,cis->ci", a[..., keep], b[..., keep])

    def relaxation_times(self, diagonal):
        """getTimesFromVectorBTE (scattering.cpp:484-513): n(n+1) / A_diag."""
        with np.errstate(divide="ignore", invalid="ignore"):
            return self.popterm / np.asarray(diagonal)

    def rta_population(self, diagonal):
        """popRTA = drift * tau (phonon_transport_app.cpp:115-117)."""
        with np.errstate(invalid="ignore"):
            return self.clean(self.drift * self.relaxation_times(diagonal)[:, None, :])

    def kappa_from_population(self, n):
        """PhononThermalConductivity::calcFromPopulation (:64-113): sum_s n_i v_j E / (Nq V)."""
        keep = ~self.excluded
        return np.einsum("cis,sj,s->cij", n[..., keep], self.vg[keep], self.E[keep]) * self.norm

    def kappa_from_canonical(self, f):
        """calcFromCanonicalPopulation (:58-62): n = n(n+1) f first."""
        return self.kappa_from_population(self.clean(f * self.popterm[:, None, :]))

    def kappa_variational(self, af, f, b):
        """calcVariational (:148-240): 2 y2 - y1, y1 = f (A f) T^2 / (Nq V), y2 = f b T^2 / (Nq V)."""
        keep = ~self.excluded
        w = self.norm * self.T[:, None, None] ** 2
        y1 = np.einsum("cis,cjs->cij", f[..., keep], af[..., keep]) * w
        y2 = np.einsum("cis,cjs->cij", f[..., keep], b[..., keep]) * w
        return 2.0 * y2 - y1


def relative_change(new, old):
    """findMaxRelativeDifference (src/utilities.cpp:80-102).  As in the
    reference, the SMALLEST |new - old| / |old| over the tensor components is
    returned (components with old = 0 give NaN or inf and are passed over)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        d = np.abs((new - old) / old).ravel()
    d = d[np.isfinite(d)]
    if d.size == 0:
        raise ValueError("no finite relative difference")
    return float(d.min())


class BteNotConverged(RuntimeError):
    """max_iter reached; .history holds the conductivity of every iteration."""

    def __init__(self, msg, history):
        super().__init__(msg)
        self.history = history


def iterative(problem, diagonal, off_diagonal_dot, threshold=1e-5, max_iter=50):
    """Omini-Sparavigna iterations (phonon_transport_app.cpp:197-247):
    f_{k+1} = f_RTA - (A_offdiag f_k) / A_diag.  diagonal: (nT, ns), the
    scattering matrix's diagonal; off_diagonal_dot(x): the product with its
    off-diagonal part.  Returns (kappa (nT, 3, 3), history of kappa), and
    raises BteNotConverged after max_iter iterations, as the reference."""
    P = problem
    pop_rta = P.rta_population(diagonal)
    kappa_old = P.kappa_from_population(pop_rta)
    with np.errstate(divide="ignore", invalid="ignore"):
        f_rta = P.clean(pop_rta / P.popterm[:, None, :])
        inv_diag = np.where(np.asarray(diagonal) != 0.0, 1.0 / np.asarray(diagonal), 0.0)
    f_old = f_rta
    history = [kappa_old]
    for _ in range(max_iter):
        f_next = P.clean(off_diagonal_dot(f_old) * inv_diag[:, None, :])
        f_next = P.clean(f_rta - f_next)
        kappa = P.kappa_from_canonical(f_next)
        history.append(kappa)
        if relative_change(kappa, kappa_old) < threshold:
            return kappa, history
        kappa_old, f_old = kappa, f_next
    raise BteNotConverged("Reached max BTE iterations without convergence", history)


def variational(problem, diagonal, dot, threshold=1e-5, max_iter=50):
    """Conjugate-gradient solve of A f = b, b the drift, started from the RTA
    solution (phonon_transport_app.cpp:249-383), one step size per
    temperature and direction.  As in the reference, the conductivity of an
    iteration is calcVariational(A f_new, f, b) with the previous f."""
    P = problem
    b = P.drift
    with np.errstate(divide="ignore", invalid="ignore"):
        f = P.clean(P.rta_population(diagonal) / P.popterm[:, None, :])
    kappa_old = P.kappa_from_population(P.rta_population(diagonal))
    w0 = P.clean(dot(f))
    r = P.clean(b - w0)
    d = P.clean(b - w0)
    history = [kappa_old]

    def ratio(num, den):
        with np.errstate(divide="ignore", invalid="ignore"):
            return np.where(den != 0.0, num / den, 0.0)

    for _ in range(max_iter):
        w = P.clean(dot(d))
        alpha = ratio(P.vdot(r, r), P.vdot(d, w))
        f_new = P.clean(d * alpha[:, :, None] + f)
        r_new = P.clean(r - w * alpha[:, :, None])
        beta = ratio(P.vdot(r_new, r_new), P.vdot(r, r))
        d_new = P.clean(d * beta[:, :, None] + r_new)
        af = P.clean(dot(f_new))
        kappa = P.kappa_variational(af, f, b)
        history.append(kappa)
        if relative_change(kappa, kappa_old) < threshold:
            return kappa, history
        kappa_old, f, r, d = kappa, f_new, r_new, d_new
    raise BteNotConverged("Reached max BTE iterations without convergence", history)


def relaxons(problem, relaxon_solve):
    """Relaxon conductivity without symmetries (PhononThermalConductivity::
    calcFromRelaxons, phonon_thermal_cond.cpp:242-445; the reference allows
    one temperature, the first).  relaxon_solve(x) = Theta diag(1/lambda+)
    Theta^T x for x (3, ns), Theta and lambda the eigenvectors and eigenvalues
    of Omega = a2Omega(A).  States with E > 0 take part, as in the reference:
    x = dn/dT v / sqrt(n(n+1)), and the result is rescaled by sqrt(n(n+1)) before
    calcFromPopulation.  Returns kappa (1, 3, 3)."""
    P = problem
    T = P.T[0]
    term = P.popterm[0]
    pos = P.E > 0.0
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        root = np.sqrt(term)
        dndt = term * P.E / T / T                                        # Particle::getDndt
        x = np.where(pos[None, :], (dndt / root)[None, :] * P.vg.T, 0.0)  # (3, ns)
    pop = relaxon_solve(x)
    pop = np.where(pos[None, :], pop * np.where(pos, root, 1.0)[None, :], pop)
    return P.kappa_from_population(pop[None])


def exact(problem, matrix):
    """Direct solve of A f = b on the included states (no reference
    counterpart; the fixed point both solvers approach), kappa from f."""
    P = problem
    keep = ~P.excluded
    A = np.asarray(matrix)[np.ix_(keep, keep)]
    out = []
    for c in range(len(P.T)):
        f = np.zeros((3, P.E.size))
        f[:, keep] = np.linalg.solve(A, P.drift[c][:, keep].T).T
        n = f * P.popterm[c][None, :]
        out.append(np.einsum("is,sj,s->ij", n[:, keep], P.vg[keep], P.E[keep]) * P.norm)
    return np.array(out)
