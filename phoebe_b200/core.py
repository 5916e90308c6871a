"""Host-side mirror of the reference's scattering-rate classes over libphx.

Class and method names follow mir-group/phoebe so that ports of its tests
read alike:

* ``PhononH0``            -- src/harmonic/phonon_h0.h (diagonalizeFromCoordinates,
                             diagonalizeVelocityFromCoordinates, populate)
* ``Interaction3Ph``      -- src/interaction/interaction_3ph.h (cacheD3,
                             getCouplingsSquared, estimateNumBatches)
* ``PhScatteringMatrix``  -- src/bte/ph_scattering.h / scattering.h (setup,
                             getLinewidths, getSingleModeTimes) plus the RTA
                             thermal conductivity of phonon_thermal_cond.cpp.

All arithmetic runs in libphx on the GPU; these classes only marshal arrays.
"""
import ctypes

import numpy as np

from . import _abi
from . import constants as C
from ._abi import c128, check, dptr, f64, i32, iptr


class Context:
    """One GPU and one CUDA stream (phx_ctx)."""

    def __init__(self, device=0):
        L = _abi.load()
        h = ctypes.c_void_p()
        check(L.phx_ctx_create(int(device), ctypes.byref(h)))
        self.h = h
        self.device = device

    def synchronize(self):
        check(_abi.load().phx_ctx_synchronize(self.h), self.h)

    def close(self):
        if getattr(self, "h", None):
            _abi.load().phx_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ws_reorder(crystal, fc2):
    """Host-only acoustic sum rule + Wigner-Seitz reorder (no GPU needed)."""
    L = _abi.load()
    nat = crystal.num_atoms
    cell, pos, fc = f64(crystal.direct_cell), f64(crystal.positions), f64(fc2)
    grid = i32(fc2.shape[2:5])
    n = ctypes.c_int(0)
    check(L.phx_ws_reorder(nat, dptr(cell), dptr(pos), iptr(grid), dptr(fc), ctypes.byref(n),
                           None, None, None))
    nb = 3 * nat
    R = np.zeros((n.value, 3))
    w = np.zeros(n.value)
    M = np.zeros((n.value, nb, nb))
    check(L.phx_ws_reorder(nat, dptr(cell), dptr(pos), iptr(grid), dptr(fc), ctypes.byref(n),
                           dptr(R), dptr(w), dptr(M)))
    return R, w, M


def q2_slice(rank, world, nq):
    """Contiguous q2 range [begin, end) of one rank: the reference splits the outer
    q2 loop over MPI ranks and sums the linewidth vector (ph_scattering.cpp:800)."""
    return rank * nq // world, (rank + 1) * nq // world


def finalize_linewidths(A, E, vg=None, temperatures=None, boundary_length=0.0):
    """What the builder's finalize step does, for partial results summed over
    ranks: degeneracy averaging of temperature row 0 (scattering.cpp:1168-1207),
    then boundary scattering |v|/L n(n+1) when boundary_length > 0
    (ph_scattering.cpp:819-860; needs vg (nq, nb, 3) and the temperatures),
    then zero for excluded states (scattering.cpp:30-50, ph_scattering.cpp:900-906).
    A (nT, nq*nb) summed over ranks, E (nq, nb); returns a new array."""
    E = np.asarray(E)
    nq, nb = E.shape
    out = np.array(A, dtype=np.float64).reshape(-1, nq, nb)
    row = out[0].copy()
    for b1 in range(nb):
        m = np.abs(E - E[:, b1:b1 + 1]) < C.degeneracyThreshold
        n = m.sum(axis=1).astype(np.float32).astype(np.float64)
        out[0][:, b1] = (row * m).sum(axis=1) / n
    if boundary_length and boundary_length > 0:
        speed = np.linalg.norm(np.asarray(vg), axis=-1)
        ok = E >= C.phExcludeCutoff
        for c, T in enumerate(np.atleast_1d(temperatures)):
            with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
                x = np.sinh(E / 2.0 / T)
                out[c][ok] += (speed / boundary_length * (0.25 / x / x))[ok]
    out[:, E < C.phExcludeCutoff] = 0.0
    return out.reshape(A.shape)


def isotope_coupling(crystal, mass_variance):
    """Per-atom isotope coupling of the builder: the isotope mass variance of
    each atom's species (dimensionless, e.g. 2.0164e-4 for natural Si) times
    the atom's mass squared -- the reference's massVariance
    (ph_scattering.cpp:27-38)."""
    g = np.asarray(mass_variance, dtype=np.float64)
    m = np.asarray(crystal.atomic_masses, dtype=np.float64)
    return g * m * m


class PhononH0:
    """Harmonic phonon Hamiltonian on the GPU (PhononH0)."""

    def __init__(self, ctx, crystal, fc2):
        L = _abi.load()
        self.ctx = ctx
        self.crystal = crystal
        self.nb = crystal.num_bands
        h = ctypes.c_void_p()
        cell, pos = f64(crystal.direct_cell), f64(crystal.positions)
        masses = f64(crystal.atomic_masses)
        grid = i32(fc2.shape[2:5])
        fc = f64(fc2)
        check(L.phx_ph_h0_create(ctx.h, crystal.num_atoms, dptr(cell), dptr(pos), dptr(masses),
                                 iptr(grid), dptr(fc), ctypes.byref(h)), ctx.h)
        self.h = h

    def diagonalizeFromCoordinates(self, q_cart, withMassScaling=True):
        q = f64(np.atleast_2d(q_cart))
        nq = q.shape[0]
        E = np.zeros((nq, self.nb))
        U = np.zeros((nq, self.nb, self.nb, 2))
        check(_abi.load().phx_ph_diag(self.h, nq, dptr(q), int(withMassScaling), dptr(E),
                                      dptr(U)), self.ctx.h)
        return E, U[..., 0] + 1j * U[..., 1]

    def diagonalizeWithVelocities(self, q_cart):
        q = f64(np.atleast_2d(q_cart))
        nq = q.shape[0]
        E = np.zeros((nq, self.nb))
        U = np.zeros((nq, self.nb, self.nb, 2))
        vg = np.zeros((nq, self.nb, 3))
        check(_abi.load().phx_ph_diag_velocities(self.h, nq, dptr(q), dptr(E), dptr(U), dptr(vg)),
              self.ctx.h)
        return E, U[..., 0] + 1j * U[..., 1], vg

    def populate(self, mesh, withVelocities=True):
        """Band structure on a full Gamma-centred mesh, resident on the GPU."""
        return BandStructure.from_h0(self, mesh, withVelocities)

    def close(self):
        if getattr(self, "h", None):
            _abi.load().phx_ph_h0_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BandStructure:
    """Device-resident energies / eigenvectors / velocities on a mesh (phx_bands)."""

    def __init__(self, ctx, h, mesh, nb, reciprocal_cell):
        self.ctx = ctx
        self.h = h
        self.mesh = tuple(int(x) for x in mesh)
        self.nb = nb
        self.nq = int(np.prod(self.mesh))
        self.reciprocal_cell = np.asarray(reciprocal_cell)

    @classmethod
    def from_h0(cls, h0, mesh, with_velocities=True):
        h = ctypes.c_void_p()
        m = i32(mesh)
        check(_abi.load().phx_bands_create_mesh(h0.h, iptr(m), int(with_velocities),
                                                ctypes.byref(h)), h0.ctx.h)
        return cls(h0.ctx, h, mesh, h0.nb, h0.crystal.reciprocal_cell)

    @classmethod
    def from_arrays(cls, ctx, mesh, reciprocal_cell, E, U, vg=None):
        h = ctypes.c_void_p()
        m = i32(mesh)
        rc = f64(reciprocal_cell)
        Ed = f64(E)
        Ud = c128(U)
        vd = f64(vg) if vg is not None else None
        nb = Ed.shape[-1]
        check(_abi.load().phx_bands_create_from_host(ctx.h, iptr(m), dptr(rc), nb, dptr(Ed),
                                                     dptr(Ud), dptr(vd) if vd is not None else None,
                                                     ctypes.byref(h)), ctx.h)
        return cls(ctx, h, mesh, nb, reciprocal_cell)

    def get(self, velocities=True):
        E = np.zeros((self.nq, self.nb))
        U = np.zeros((self.nq, self.nb, self.nb, 2))
        vg = np.zeros((self.nq, self.nb, 3)) if velocities else None
        check(_abi.load().phx_bands_get(self.h, dptr(E), dptr(U),
                                        dptr(vg) if velocities else None), self.ctx.h)
        return E, U[..., 0] + 1j * U[..., 1], vg

    def close(self):
        if getattr(self, "h", None):
            _abi.load().phx_bands_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


PRECISIONS = {"fp64": _abi.PHX_PREC_FP64, "split_bf16": _abi.PHX_PREC_SPLIT_BF16,
              "split_fp16": _abi.PHX_PREC_SPLIT_FP16}


class Interaction3Ph:
    """3-phonon vertex on the GPU (Interaction3Ph)."""

    def __init__(self, ctx, crystal, fc3, precision="fp64"):
        self.ctx = ctx
        self.nat = crystal.num_atoms
        self.nb = 3 * self.nat
        D3, R2, R3, w2, w3 = (f64(x) for x in (fc3.D3, fc3.R2, fc3.R3, fc3.w2, fc3.w3))
        self.nr3, self.nr2 = D3.shape[3], D3.shape[4]
        h = ctypes.c_void_p()
        check(_abi.load().phx_v3_create(ctx.h, self.nat, self.nr2, self.nr3, dptr(D3), dptr(R2),
                                        dptr(R3), dptr(w2), dptr(w3), ctypes.byref(h)), ctx.h)
        self.h = h
        self.setPrecision(precision)

    def setPrecision(self, precision):
        check(_abi.load().phx_v3_set_precision(self.h, PRECISIONS[precision]), self.ctx.h)
        self.precision = precision

    def cacheD3(self, q2):
        q = f64(q2)
        check(_abi.load().phx_v3_cache_d3(self.h, dptr(q)), self.ctx.h)

    def getCouplingsSquared(self, q1s, q2, ev1s, ev2, ev3Pluss, ev3Minss, nb1s=None, nb2=None,
                            nb3Pluss=None, nb3Minss=None):
        """Returns (couplingPlus, couplingMins): lists of (nb1,nb2,nb3) arrays."""
        q1 = f64(np.atleast_2d(q1s))
        nq1 = q1.shape[0]
        nb = self.nb

        def pad(evs):
            out = np.zeros((nq1, nb, nb), dtype=np.complex128)
            for i, e in enumerate(evs):
                e = np.asarray(e)
                out[i, :, :e.shape[1]] = e
            return out

        e1, e3p, e3m = pad(ev1s), pad(ev3Pluss), pad(ev3Minss)
        ev2 = np.asarray(ev2)
        e2 = np.zeros((nb, nb), dtype=np.complex128)
        e2[:, :ev2.shape[1]] = ev2
        nb1s = i32(nb1s if nb1s is not None else [np.asarray(e).shape[1] for e in ev1s])
        nb2 = int(nb2 if nb2 is not None else ev2.shape[1])
        nb3p = i32(nb3Pluss if nb3Pluss is not None else [np.asarray(e).shape[1] for e in ev3Pluss])
        nb3m = i32(nb3Minss if nb3Minss is not None else [np.asarray(e).shape[1] for e in ev3Minss])
        sizeP = int(np.sum(nb1s * nb2 * nb3p))
        sizeM = int(np.sum(nb1s * nb2 * nb3m))
        outP = np.zeros(max(sizeP, 1))
        outM = np.zeros(max(sizeM, 1))
        E1, E2, E3p, E3m = c128(e1), c128(e2), c128(e3p), c128(e3m)
        check(_abi.load().phx_v3_couplings_sq(self.h, nq1, dptr(q1), dptr(E1), iptr(nb1s), dptr(E2),
                                              nb2, dptr(E3p), iptr(nb3p), dptr(E3m), iptr(nb3m),
                                              dptr(outP), dptr(outM)), self.ctx.h)
        cp, cm = [], []
        oP = oM = 0
        for i in range(nq1):
            n = nb1s[i] * nb2 * nb3p[i]
            cp.append(outP[oP:oP + n].reshape(nb1s[i], nb2, nb3p[i]))
            oP += n
            n = nb1s[i] * nb2 * nb3m[i]
            cm.append(outM[oM:oM + n].reshape(nb1s[i], nb2, nb3m[i]))
            oM += n
        return cp, cm

    def estimateNumBatches(self, nq1, nb2):
        n = ctypes.c_int(0)
        check(_abi.load().phx_v3_estimate_num_batches(self.h, nq1, nb2, ctypes.byref(n)), self.ctx.h)
        return n.value

    def close(self):
        if getattr(self, "h", None):
            _abi.load().phx_v3_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PhScatteringMatrix:
    """Phonon scattering matrix on a full mesh (PhScatteringMatrix / ScatteringMatrix).

    Without in_memory, setup() runs the builder's linewidth mode and dot()
    its matrix-vector mode (one builder pass per product, nothing stored).
    With in_memory (the reference's scatteringMatrixInMemory; one
    temperature), setup() builds the whole matrix into device memory and dot()
    / offDiagonalDot() multiply with it."""

    def __init__(self, coupling3Ph, bands, temperatures_ry, smearing="adaptive", sigma=0.0, window=None,
                 isotope_coupling=None, boundary_length=0.0, in_memory=False):
        """window: optional (energy (nq), cut (nq)) per-q1 q2 window: the pair
        (q1, q2) counts only when energy[q2] <= cut[q1] (synth.q2_window).
        isotope_coupling: per-atom coupling (core.isotope_coupling) enables
        isotope scattering; boundary_length > 0 (Bohr) enables boundary
        scattering (the reference's withIsotopeScattering / boundaryLength)."""
        self.in_memory = bool(in_memory)
        self._m = None
        self.v3 = coupling3Ph
        self.bands = bands
        self.temperatures = f64(np.atleast_1d(temperatures_ry))
        self.smearing = smearing
        self.sigma = float(sigma)
        self.window = None if window is None else (f64(window[0]), f64(window[1]))
        self.isotope = None if isotope_coupling is None else f64(isotope_coupling)
        self.boundary_length = float(boundary_length)
        self.internalDiagonal = None
        self.stats = None

    def _params(self, q2_begin=0, q2_end=None, finalize=True):
        p = _abi.LwParams()
        p.num_temperatures = len(self.temperatures)
        p.temperatures = dptr(self.temperatures)
        p.smearing = _abi.PHX_SMEAR_GAUSSIAN if self.smearing == "gaussian" else _abi.PHX_SMEAR_ADAPTIVE
        p.sigma = self.sigma
        p.finalize = int(finalize)
        p.q2_begin = int(q2_begin)
        p.q2_end = int(self.bands.nq if q2_end is None else q2_end)
        if self.window is not None:
            p.window_energy = dptr(self.window[0])
            p.window_cut = dptr(self.window[1])
        if self.isotope is not None:
            p.isotope_coupling = dptr(self.isotope)
        p.boundary_length = self.boundary_length
        return p

    def setup(self, q2_begin=0, q2_end=None, finalize=True):
        """Builds A_out = linewidth * n(n+1) (internalDiagonal), shape (nT, nq*nb).
        In memory: builds the matrix too; its diagonal is not degeneracy-averaged."""
        if self.in_memory:
            return self._setup_matrix(q2_begin, q2_end, finalize)
        nT = len(self.temperatures)
        out = np.zeros((nT, self.bands.nq * self.bands.nb))
        p = self._params(q2_begin, q2_end, finalize)
        st = _abi.LwStats()
        check(_abi.load().phx_ph_linewidths(self.v3.h, self.bands.h, ctypes.byref(p), dptr(out),
                                            ctypes.byref(st)), self.v3.ctx.h)
        self.internalDiagonal = out
        self.stats = st
        return out

    def setup_screened(self, net, log10_threshold, q2_begin=0, q2_end=None, finalize=True):
        """setup() with learned screening (phx_ph_linewidths_screened): the vertices
        (q1, q2) that the network net (screening.ScreeningMLP with 12 pair inputs)
        predicts below log10_threshold are dropped; the rest are exact.
        self.stats.pairs_screened_out counts the dropped vertices."""
        nT = len(self.temperatures)
        out = np.zeros((nT, self.bands.nq * self.bands.nb))
        p = self._params(q2_begin, q2_end, finalize)
        st = _abi.LwStats()
        check(_abi.load().phx_ph_linewidths_screened(self.v3.h, self.bands.h, ctypes.byref(p), net.h,
                                                     float(log10_threshold), dptr(out), ctypes.byref(st)),
              self.v3.ctx.h)
        self.internalDiagonal = out
        self.stats = st
        return out

    def _setup_matrix(self, q2_begin, q2_end, finalize):
        if len(self.temperatures) != 1:
            raise ValueError("a stored scattering matrix holds one temperature")
        self.close()
        p = self._params(q2_begin, q2_end, finalize)
        st = _abi.LwStats()
        h = ctypes.c_void_p()
        L = _abi.load()
        check(L.phx_ph_smatrix_create(self.v3.h, self.bands.h, ctypes.byref(p), ctypes.byref(h), ctypes.byref(st)),
              self.v3.ctx.h)
        self._m = h
        ns = L.phx_smatrix_num_states(h)
        diag = np.zeros((1, ns))
        check(L.phx_smatrix_diagonal(h, dptr(diag)), self.v3.ctx.h)
        self.internalDiagonal = diag
        self.stats = st
        return diag

    @property
    def num_states(self):
        return self.bands.nq * self.bands.nb

    def _vectors(self, x):
        x = f64(x)
        single = x.ndim == 3
        x = x[None] if single else x
        if x.shape[1:] != (len(self.temperatures), 3, self.num_states):
            raise ValueError("vectors must be (nT, 3, numStates) or (nvec, nT, 3, numStates)")
        return x, single

    def dot(self, x, q2_begin=0, q2_end=None, finalize=True):
        """A x (ScatteringMatrix::dot) for x (nT, 3, ns) or (nvec, nT, 3, ns).
        In memory: rows and columns of excluded states left out; otherwise one
        matrix-vector pass of the builder (switchCase 1)."""
        x, single = self._vectors(x)
        y = np.zeros_like(x)
        L = _abi.load()
        if self.in_memory:
            if self._m is None:
                raise RuntimeError("setup() first")
            check(L.phx_smatrix_dot(self._m, x.shape[0], dptr(x), 0, dptr(y)), self.v3.ctx.h)
        else:
            p = self._params(q2_begin, q2_end, finalize)
            st = _abi.LwStats()
            check(L.phx_ph_smatrix_dot(self.v3.h, self.bands.h, ctypes.byref(p), x.shape[0], dptr(x), dptr(y),
                                       ctypes.byref(st)), self.v3.ctx.h)
            self.stats = st
        return y[0] if single else y

    def offDiagonalDot(self, x):
        """ScatteringMatrix::offDiagonalDot (scattering.cpp:180-265).  In memory:
        A x without the diagonal; otherwise, as the reference, dot(x) minus
        internalDiagonal * x with the internalDiagonal of setup() (averaged)."""
        x, single = self._vectors(x)
        if self.in_memory:
            if self._m is None:
                raise RuntimeError("setup() first")
            y = np.zeros_like(x)
            check(_abi.load().phx_smatrix_dot(self._m, x.shape[0], dptr(x), 1, dptr(y)), self.v3.ctx.h)
        else:
            if self.internalDiagonal is None:
                raise RuntimeError("setup() first")
            y = self.dot(x) - self.internalDiagonal[None, :, None, :] * x
        return y[0] if single else y

    def getMatrixRows(self, row0, nrows):
        """Rows row0 .. row0+nrows-1 of the stored matrix, (nrows, numStates)."""
        if self._m is None:
            raise RuntimeError("the matrix is stored only with in_memory=True, after setup()")
        out = np.zeros((nrows, self.num_states))
        check(_abi.load().phx_smatrix_get_rows(self._m, int(row0), int(nrows), dptr(out)), self.v3.ctx.h)
        return out

    def symmetrize(self):
        """A -> (A + A^T) / 2 for the stored matrix (ScatteringMatrix::symmetrize)."""
        if self._m is None:
            raise RuntimeError("the matrix is stored only with in_memory=True, after setup()")
        check(_abi.load().phx_smatrix_symmetrize(self._m), self.v3.ctx.h)

    def _stored(self):
        if self._m is None:
            raise RuntimeError("the matrix is stored only with in_memory=True, after setup()")
        return self._m

    def a2Omega(self):
        """ScatteringMatrix::a2Omega (scattering.cpp:366-434) in device memory:
        A(i, j) / sqrt(n_i(n_i+1) n_j(n_j+1)); internalDiagonal / n(n+1)."""
        L = _abi.load()
        check(L.phx_smatrix_a2omega(self._stored()), self.v3.ctx.h)
        diag = np.zeros((1, self.num_states))
        check(L.phx_smatrix_diagonal(self._m, dptr(diag)), self.v3.ctx.h)
        self.internalDiagonal = diag

    def diagonalize(self, numEigenvalues=0):
        """ScatteringMatrix::diagonalize (scattering.cpp:872-910): eigenvalues
        (ascending) of the matrix's upper triangle, all of them or the
        smallest numEigenvalues; the eigenvectors replace the matrix in device
        memory (getMatrixRows then returns their rows)."""
        ev = np.zeros(self.num_states)
        found = ctypes.c_int(0)
        check(_abi.load().phx_smatrix_diagonalize(self._stored(), int(numEigenvalues), dptr(ev),
                                                  ctypes.byref(found)), self.v3.ctx.h)
        self.eigenvalues = ev[:found.value].copy()
        return self.eigenvalues

    def relaxonSolve(self, x):
        """Theta diag(1/lambda, lambda > 0) Theta^T x for x (3, ns) or
        (nvec, 3, ns), after diagonalize() (calcFromRelaxons,
        phonon_thermal_cond.cpp:316-380)."""
        x = f64(x)
        single = x.ndim == 2
        x = x[None] if single else x
        if x.shape[1:] != (3, self.num_states):
            raise ValueError("vectors must be (3, numStates) or (nvec, 3, numStates)")
        y = np.zeros_like(x)
        check(_abi.load().phx_smatrix_relaxon_solve(self._stored(), x.shape[0], dptr(x), dptr(y)), self.v3.ctx.h)
        return y[0] if single else y

    def close(self):
        if getattr(self, "_m", None) is not None:
            _abi.load().phx_smatrix_destroy(self._m)
            self._m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def outputToJSON(self, path, crystal):
        """rta_ph_relaxation_times.json (ScatteringMatrix::outputToJSON, scattering.cpp:639-815)
        from the internalDiagonal of setup()."""
        from . import output
        if self.internalDiagonal is None:
            raise RuntimeError("setup() first")
        E, _, vg = self.bands.get()
        return output.relaxation_times_json(path, crystal, self.bands.mesh, E, vg, self.internalDiagonal,
                                            self.temperatures)

    def getLinewidths(self, E):
        """Gamma = A_out / (n(n+1)) (scattering.cpp:529-568)."""
        T = self.temperatures[:, None]
        x = np.sinh(np.asarray(E).reshape(1, -1) / 2.0 / T)
        with np.errstate(divide="ignore", invalid="ignore"):
            return self.internalDiagonal / (0.25 / x / x)

    def getSingleModeTimes(self, E):
        """tau = n(n+1) / A_out (scattering.cpp:484-513)."""
        T = self.temperatures[:, None]
        x = np.sinh(np.asarray(E).reshape(1, -1) / 2.0 / T)
        with np.errstate(divide="ignore", invalid="ignore"):
            return (0.25 / x / x) / self.internalDiagonal

    def thermalConductivity(self, volume):
        """RTA kappa (nT,3,3) in W/(m K)."""
        kappa = np.zeros((len(self.temperatures), 3, 3))
        A = f64(self.internalDiagonal)
        check(_abi.load().phx_ph_rta_kappa(self.bands.h, len(self.temperatures),
                                           dptr(self.temperatures), dptr(A), float(volume),
                                           dptr(kappa)), self.v3.ctx.h)
        return kappa * C.thConductivityAuToSi


# ---------------------------------------------------------------------------
# electron-phonon Wannier path
# ---------------------------------------------------------------------------

class ElectronH0Wannier:
    """Electronic Wannier Hamiltonian on the GPU (ElectronH0Wannier, no shifted vectors)."""

    def __init__(self, ctx, crystal, R, deg, H):
        L = _abi.load()
        self.ctx = ctx
        self.crystal = crystal
        self.nw = int(H.shape[1])
        h = ctypes.c_void_p()
        cell, Rd, dd, Hd = f64(crystal.direct_cell), f64(R), f64(deg), c128(H)
        check(L.phx_el_h0_create(ctx.h, self.nw, len(Rd), dptr(cell), dptr(Rd), dptr(dd), dptr(Hd),
                                 ctypes.byref(h)), ctx.h)
        self.h = h

    def _diag(self, k_cart, velocities):
        k = f64(np.atleast_2d(k_cart))
        nk = k.shape[0]
        E = np.zeros((nk, self.nw))
        U = np.zeros((nk, self.nw, self.nw, 2))
        vg = np.zeros((nk, self.nw, 3)) if velocities else None
        check(_abi.load().phx_el_diag(self.h, nk, dptr(k), dptr(E), dptr(U),
                                      dptr(vg) if velocities else None), self.ctx.h)
        return E, U[..., 0] + 1j * U[..., 1], vg

    def diagonalizeFromCoordinates(self, k_cart):
        E, U, _ = self._diag(k_cart, False)
        return E, U

    def diagonalizeWithVelocities(self, k_cart):
        return self._diag(k_cart, True)

    def populate(self, mesh, withVelocities=True):
        """Band structure on a full Gamma-centred k mesh, resident on the GPU."""
        h = ctypes.c_void_p()
        m = i32(mesh)
        check(_abi.load().phx_el_bands_create_mesh(self.h, iptr(m), int(withVelocities), ctypes.byref(h)),
              self.ctx.h)
        return BandStructure(self.ctx, h, mesh, self.nw, self.crystal.reciprocal_cell)

    def close(self):
        if getattr(self, "h", None):
            _abi.load().phx_el_h0_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class InteractionElPhWan:
    """Electron-phonon coupling in the Wannier basis on the GPU (InteractionElPhWan)."""

    def __init__(self, ctx, Re, degE, Rp, degP, g):
        L = _abi.load()
        self.ctx = ctx
        g = np.ascontiguousarray(g, dtype=np.complex64)
        self.nRe, self.nRp, self.nph, self.nw = g.shape[0], g.shape[1], g.shape[2], g.shape[3]
        gf = g.view(np.float32)
        h = ctypes.c_void_p()
        Re, degE, Rp, degP = f64(Re), f64(degE), f64(Rp), f64(degP)
        check(L.phx_elph_create(ctx.h, self.nw, self.nph, self.nRe, self.nRp, dptr(Re), dptr(degE), dptr(Rp),
                                dptr(degP), gf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(h)),
              ctx.h)
        self.h = h
        self.nb1 = 0

    def setPrecision(self, precision):
        """'fp64' or 'split_bf16' (tensor-core Rp transform in the linewidth builder)."""
        check(_abi.load().phx_elph_set_precision(self.h, PRECISIONS[precision]), self.ctx.h)
        self.precision = precision

    def cacheElPh(self, eigvec1, k1C):
        """eigvec1: (nw, nb1) complex (columns = bands at k1)."""
        U = c128(eigvec1)
        self.nb1 = int(np.asarray(eigvec1).shape[1])
        check(_abi.load().phx_elph_cache_k1(self.h, dptr(f64(k1C)), dptr(U), self.nb1), self.ctx.h)

    def calcCouplingSquared(self, eigvecs2, eigvecs3, q3Cs):
        """eigvecs2: list of (nw, nb2) complex; eigvecs3: list of (nph, nph); q3Cs: (nk2,3).
        Returns the list of |g|^2 tensors (nb1, nb2, nph), as getCouplingSquared."""
        nk2 = len(eigvecs2)
        nb2s = i32([np.asarray(u).shape[1] for u in eigvecs2])
        nb2max = int(nb2s.max()) if nk2 else 1
        U2 = np.zeros((nk2, self.nw, nb2max), dtype=np.complex128)
        for i, u in enumerate(eigvecs2):
            U2[i, :, :u.shape[1]] = u
        ev3 = np.ascontiguousarray(np.asarray(eigvecs3), dtype=np.complex128)
        out = np.zeros((nk2, self.nb1, nb2max, self.nph))
        check(_abi.load().phx_elph_couplings_sq(self.h, nk2, dptr(f64(q3Cs)), dptr(c128(U2)), iptr(nb2s), nb2max,
                                                dptr(c128(ev3)), dptr(out)), self.ctx.h)
        self.cacheCoupling = [out[i, :, :nb2s[i], :] for i in range(nk2)]
        return self.cacheCoupling

    def getCouplingSquared(self, ik2):
        return self.cacheCoupling[ik2]

    def close(self):
        if getattr(self, "h", None):
            _abi.load().phx_elph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ElScatteringMatrix:
    """Electron-phonon linewidths (ElScatteringMatrix::builder, linewidth mode) on the GPU.

    k2 = k1 + q runs over the q mesh of the phonon band structure (which must
    divide the electron k mesh); norm defaults to 1/N_q."""

    def __init__(self, elph, el_bands, ph_bands, temperatures_ry, chemical_potential, window, smearing="adaptive",
                 sigma=0.0, norm=None):
        self.elph, self.el, self.ph = elph, el_bands, ph_bands
        self.temperatures = f64(np.atleast_1d(temperatures_ry))
        self.mu, self.window = float(chemical_potential), float(window)
        self.smearing, self.sigma = smearing, float(sigma)
        self.norm = 1.0 / ph_bands.nq if norm is None else float(norm)

    def setup(self, k1_list=None):
        """Linewidths (nT, nk1, nw) of the outer k points (all k of the mesh by default)."""
        k1 = i32(np.arange(self.el.nq) if k1_list is None else k1_list)
        p = _abi.ElParams()
        p.num_temperatures = len(self.temperatures)
        p.temperatures = dptr(self.temperatures)
        p.chemical_potential = self.mu
        p.window = self.window
        p.smearing = _abi.PHX_SMEAR_GAUSSIAN if self.smearing == "gaussian" else _abi.PHX_SMEAR_ADAPTIVE
        p.sigma = self.sigma
        p.norm = self.norm
        p.num_k1 = len(k1)
        p.k1_list = iptr(k1)
        out = np.zeros((len(self.temperatures), len(k1), self.el.nb))
        st = _abi.LwStats()
        check(_abi.load().phx_el_linewidths(self.elph.h, self.el.h, self.ph.h, ctypes.byref(p), dptr(out),
                                            ctypes.byref(st)), self.elph.ctx.h)
        self.stats = st
        self.linewidths = out
        return out
