"""ctypes binding of the CPU FP64 oracle (test infrastructure only).

The oracle restates the reference's CPU algorithms for the scattering-rate
path (see the header of each C++ file for the reference lines it follows).
Only the tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of
``bench.py`` may import this package; the product library never uses it.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def build():
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_ws_reorder.restype = ctypes.c_int
        L.orc_ws_reorder.argtypes = [ctypes.c_int, _D, _D, _I, _D, _I, _D, _D, _D]
        L.orc_ph_diag.restype = ctypes.c_int
        L.orc_ph_diag.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, _D,
                                  ctypes.c_int, _D, _D]
        L.orc_ph_velocities.restype = ctypes.c_int
        L.orc_ph_velocities.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, ctypes.c_int,
                                        _D, _D, _D]
        L.orc_v3_create.restype = ctypes.c_void_p
        L.orc_v3_create.argtypes = [ctypes.c_int] * 3 + [_D] * 5
        L.orc_v3_destroy.argtypes = [ctypes.c_void_p]
        L.orc_v3_cache_d3.argtypes = [ctypes.c_void_p, _D]
        L.orc_v3_couplings.argtypes = [ctypes.c_void_p, ctypes.c_int] + [_D] * 7
        L.orc_symmetrize_coupling.argtypes = [_D, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _D,
                                              _D]
        L.orc_ph_linewidths.restype = ctypes.c_int
        L.orc_ph_linewidths.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _D, _D, _D, _D, _D,
                                        ctypes.c_int, _D, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_int, _I, ctypes.c_int, _D, _D, _D, _D, ctypes.c_double]
        L.orc_ph_smatrix.restype = ctypes.c_int
        L.orc_ph_smatrix.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _D, _D, _D, _D, _D, _D, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_int, _I, ctypes.c_int, _D, _D, _D, ctypes.c_double]
        L.orc_ph_smatrix_dot.restype = ctypes.c_int
        L.orc_ph_smatrix_dot.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _D, _D, _D, _D, _D, ctypes.c_int, _D,
                                         ctypes.c_int, ctypes.c_double, ctypes.c_int, _I, ctypes.c_int,
                                         ctypes.c_int, _D, _D, _D, ctypes.c_double]
        L.orc_smatrix_dot.argtypes = [ctypes.c_int, _D, _D, ctypes.c_int, _D, ctypes.c_int, _D]
        L.orc_rta_kappa.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, ctypes.c_long,
                                    ctypes.c_double, _D]
        L.orc_el_diag.restype = ctypes.c_int
        L.orc_el_diag.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, ctypes.c_int, _D, _D, _D, _D]
        _F = ctypes.POINTER(ctypes.c_float)
        L.orc_elph_cache.restype = ctypes.c_int
        L.orc_elph_cache.argtypes = [ctypes.c_int] * 4 + [_D, _D, _F, _D, _D, ctypes.c_int, _D]
        L.orc_elph_couplings.restype = ctypes.c_int
        L.orc_elph_couplings.argtypes = [ctypes.c_int] * 3 + [_D, _D, _D, ctypes.c_int, ctypes.c_int, _D, _D,
                                                               _I, ctypes.c_int, _D, _D]
        L.orc_el_linewidths.restype = ctypes.c_int
        L.orc_el_linewidths.argtypes = ([ctypes.c_int] * 4 + [_D, _D, _D, _D, _F, _I, _I, _D, _D, _D, _I, _I,
                                                              _D, _D, _D, _D, ctypes.c_int, _I, ctypes.c_int,
                                                              _D, ctypes.c_double, ctypes.c_int,
                                                              ctypes.c_double, ctypes.c_double, _D])
        _lib = L
    return _lib


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return a.ctypes.data_as(_D)


def ws_reorder(crystal, fc):
    """ASR "simple" + Wigner-Seitz reorder -> (R (nR,3), w (nR,), mat2R (nR,nb,nb))."""
    L = lib()
    nat = crystal.num_atoms
    cell = _d(crystal.direct_cell)
    pos = _d(crystal.positions)
    grid = np.ascontiguousarray(fc.shape[2:5], dtype=np.int32)
    fcc = _d(fc)
    n = ctypes.c_int(0)
    rc = L.orc_ws_reorder(nat, _p(cell), _p(pos), grid.ctypes.data_as(_I), _p(fcc),
                          ctypes.byref(n), None, None, None)
    if rc:
        raise RuntimeError("orc_ws_reorder failed: %d" % rc)
    nR = n.value
    nb = 3 * nat
    R = np.zeros((nR, 3))
    w = np.zeros(nR)
    M = np.zeros((nR, nb, nb))
    rc = L.orc_ws_reorder(nat, _p(cell), _p(pos), grid.ctypes.data_as(_I), _p(fcc),
                          ctypes.byref(n), _p(R), _p(w), _p(M))
    if rc:
        raise RuntimeError("orc_ws_reorder failed: %d" % rc)
    return R, w, M


class PhononH0:
    """Oracle harmonic Hamiltonian (CPU path of PhononH0)."""

    def __init__(self, crystal, fc):
        self.crystal = crystal
        self.R, self.w, self.mat2R = ws_reorder(crystal, fc)
        self.nb = crystal.num_bands
        self.masses = _d(np.repeat(crystal.atomic_masses, 3))

    def diagonalize(self, q_cart, mass_scaling=True):
        q = _d(np.atleast_2d(q_cart))
        nq = q.shape[0]
        E = np.zeros((nq, self.nb))
        U = np.zeros((nq, self.nb, self.nb, 2))
        rc = lib().orc_ph_diag(self.nb, len(self.w), _p(self.R), _p(self.w), _p(self.mat2R),
                               _p(self.masses), nq, _p(q), int(mass_scaling), _p(E), _p(U))
        if rc:
            raise RuntimeError("oracle eigensolver failed")
        return E, U[..., 0] + 1j * U[..., 1]

    def velocities(self, q_cart, full=False):
        q = _d(np.atleast_2d(q_cart))
        nq = q.shape[0]
        vg = np.zeros((nq, self.nb, 3))
        vf = np.zeros((nq, self.nb, self.nb, 3, 2)) if full else None
        rc = lib().orc_ph_velocities(self.nb, len(self.w), _p(self.R), _p(self.w),
                                     _p(self.mat2R), _p(self.masses), nq, _p(q), _p(vg),
                                     _p(vf) if full else None)
        if rc:
            raise RuntimeError("oracle eigensolver failed")
        if full:
            return vg, vf[..., 0] + 1j * vf[..., 1]
        return vg


def _c(a):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a.view(np.float64)


class Interaction3Ph:
    """Oracle 3-phonon vertex (Interaction3Ph CPU restatement)."""

    def __init__(self, crystal, fc3):
        self.nat = crystal.num_atoms
        self.nb = 3 * self.nat
        self._keep = [_d(fc3.D3), _d(fc3.R2), _d(fc3.R3), _d(fc3.w2), _d(fc3.w3)]
        nr3, nr2 = fc3.D3.shape[3], fc3.D3.shape[4]
        self.h = lib().orc_v3_create(self.nat, nr2, nr3, *[_p(x) for x in self._keep])

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_v3_destroy(self.h)
            self.h = None

    def cache_d3(self, q2):
        q = _d(q2)
        lib().orc_v3_cache_d3(self.h, _p(q))

    def couplings_squared(self, q1s, ev1s, ev2, ev3p, ev3m):
        q1s = _d(np.atleast_2d(q1s))
        nq1 = q1s.shape[0]
        nb = self.nb
        e1, e2, e3p, e3m = _c(ev1s), _c(ev2), _c(ev3p), _c(ev3m)
        outP = np.zeros((nq1, nb, nb, nb))
        outM = np.zeros((nq1, nb, nb, nb))
        lib().orc_v3_couplings(self.h, nq1, _p(q1s), _p(e1), _p(e2), _p(e3p), _p(e3m), _p(outP),
                               _p(outM))
        return outP, outM

    def linewidths(self, mesh, E, ev, vg, qcart, recip, temps_ry, smearing, sigma,
                   q2_list=None, finalize=True, out=None, window=None, isotope_coupling=None,
                   boundary_length=0.0):
        """window: optional (energy (nq), cut (nq)): pair (q1, q2) only when
        energy[q2] <= cut[q1].  isotope_coupling: per-atom massVariance (variance x
        mass^2); boundary_length: Bohr (0: none)."""
        nq, nb = E.shape
        m = np.ascontiguousarray(mesh, dtype=np.int32)
        T = _d(temps_ry)
        nT = len(T)
        if out is None:
            out = np.zeros((nT, nq * nb))
        Ed, evd, vgd, qd, rd = _d(E), _c(ev), _d(vg), _d(qcart), _d(recip)
        if q2_list is None:
            nq2, ql = nq, None
        else:
            ql_arr = np.ascontiguousarray(q2_list, dtype=np.int32)
            nq2, ql = len(ql_arr), ql_arr.ctypes.data_as(_I)
        we, wc = (None, None) if window is None else (_d(window[0]), _d(window[1]))
        gi = None if isotope_coupling is None else _d(isotope_coupling)
        rc = lib().orc_ph_linewidths(self.h, nq, m.ctypes.data_as(_I), _p(Ed), _p(evd), _p(vgd),
                                     _p(qd), _p(rd), nT, _p(T), 0 if smearing == "gaussian" else 1,
                                     float(sigma), nq2, ql, int(finalize), _p(out),
                                     _p(we) if we is not None else None,
                                     _p(wc) if wc is not None else None,
                                     _p(gi) if gi is not None else None, float(boundary_length))
        if rc:
            raise RuntimeError("oracle linewidth builder failed: %d" % rc)
        return out

    @staticmethod
    def _q2(q2_list, nq):
        if q2_list is None:
            return nq, None
        ql = np.ascontiguousarray(q2_list, dtype=np.int32)
        return len(ql), ql

    def scattering_matrix(self, mesh, E, ev, vg, qcart, recip, temp_ry, smearing, sigma, q2_list=None,
                          finalize=True, isotope_coupling=None, boundary_length=0.0):
        """switchCase 0 (one temperature): returns (matrix (ns, ns), linewidth row (ns))."""
        nq, nb = E.shape
        ns = nq * nb
        m = np.ascontiguousarray(mesh, dtype=np.int32)
        T = _d([temp_ry])
        mat = np.zeros((ns, ns))
        lw = np.zeros(ns)
        nq2, ql = self._q2(q2_list, nq)
        gi = None if isotope_coupling is None else _d(isotope_coupling)
        rc = lib().orc_ph_smatrix(self.h, nq, m.ctypes.data_as(_I), _p(_d(E)), _p(_c(ev)), _p(_d(vg)),
                                  _p(_d(qcart)), _p(_d(recip)), _p(T), 0 if smearing == "gaussian" else 1,
                                  float(sigma), nq2, None if ql is None else ql.ctypes.data_as(_I),
                                  int(finalize), _p(lw), _p(mat), None if gi is None else _p(gi),
                                  float(boundary_length))
        if rc:
            raise RuntimeError("oracle matrix builder failed: %d" % rc)
        return mat, lw

    def scattering_dot(self, mesh, E, ev, vg, qcart, recip, temps_ry, smearing, sigma, x, q2_list=None,
                       finalize=True, isotope_coupling=None, boundary_length=0.0):
        """switchCase 1: y = A x for x (nvec, nT, 3, ns), without storing A."""
        nq, nb = E.shape
        m = np.ascontiguousarray(mesh, dtype=np.int32)
        T = _d(temps_ry)
        x = _d(x)
        assert x.ndim == 4 and x.shape[1:] == (len(T), 3, nq * nb)
        y = np.zeros_like(x)
        nq2, ql = self._q2(q2_list, nq)
        gi = None if isotope_coupling is None else _d(isotope_coupling)
        rc = lib().orc_ph_smatrix_dot(self.h, nq, m.ctypes.data_as(_I), _p(_d(E)), _p(_c(ev)), _p(_d(vg)),
                                      _p(_d(qcart)), _p(_d(recip)), len(T), _p(T),
                                      0 if smearing == "gaussian" else 1, float(sigma), nq2,
                                      None if ql is None else ql.ctypes.data_as(_I), int(finalize), x.shape[0],
                                      _p(x), _p(y), None if gi is None else _p(gi), float(boundary_length))
        if rc:
            raise RuntimeError("oracle matrix-vector builder failed: %d" % rc)
        return y


def smatrix_dot(mat, E, x, off_diagonal=False):
    """ScatteringMatrix::dot / offDiagonalDot of a stored matrix; x (nvec, 3, ns)."""
    ns = mat.shape[0]
    x = _d(x)
    y = np.zeros_like(x)
    lib().orc_smatrix_dot(ns, _p(_d(mat)), _p(_d(E).ravel()), x.shape[0], _p(x), int(off_diagonal), _p(y))
    return y


# src/constants/constants.h: 0.1 cm^-1 in Ry, the phonon exclusion cut-off (scattering.cpp:37)
_TERAHERTZ_AU = 6.62607015e-34 / (2.0 * np.pi) / 4.359744650e-18 * 1.0e12
_RY_TO_CMM1 = 1.0e10 * (1.0 / _TERAHERTZ_AU / 2.0 / (2.0 * np.pi)) / 299792458.0
_PH_EXCLUDE_CUTOFF = 0.1 / _RY_TO_CMM1


def _poppm1(E, T):
    x = np.sinh(np.asarray(E, dtype=np.float64) / 2.0 / T)
    return 0.25 / x / x


def a2omega(mat, diag, E, T):
    """ScatteringMatrix::a2Omega (src/bte/scattering.cpp:366-434), without
    symmetries: for states i, j both outside excludeIndices (E < 0.1 cm^-1,
    :30-41), mat[i, j] /= sqrt(term_i term_j) and diag[i] /= term_i, term the
    n(n+1) of Particle::getPopPopPm1.  Returns copies."""
    mat = np.array(mat, dtype=np.float64, copy=True)
    diag = np.array(diag, dtype=np.float64, copy=True).ravel()
    E = np.asarray(E, dtype=np.float64).ravel()
    keep = E >= _PH_EXCLUDE_CUTOFF
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        term = _poppm1(E, T)
    idx = np.flatnonzero(keep)
    mat[np.ix_(idx, idx)] /= np.sqrt(np.outer(term[idx], term[idx]))
    diag[idx] /= term[idx]
    return mat, diag


def relaxons(mat, E, vg, T, num_q, volume, num_eigenvalues=0):
    """The relaxon solver without symmetries (src/apps/phonon_transport_app.cpp:
    386-420) on a stored matrix A (already a2omega'd): eigenvalues of the upper
    triangle, all or the smallest num_eigenvalues (ParallelMatrix::diagonalize,
    src/algebra/PMatrix.cpp:99-160, 266-404, uplo 'U'; LAPACK here), then
    PhononThermalConductivity::calcFromRelaxons (src/observable/
    phonon_thermal_cond.cpp:316-445):
        relaxonsPopulation(a, i) = sum_s [lambda_a > 0, E_s > 0]
                                   dndt_s / sqrt(term_s) v_si theta(s, a) / lambda_a
        population(i, s) = sum_a theta(s, a) relaxonsPopulation(a, i),
        times sqrt(term_s) where E_s > 0, then calcFromPopulation
    (:64-113; excluded states left out).  Returns (eigenvalues, eigenvectors, kappa (3, 3))."""
    E = np.asarray(E, dtype=np.float64).ravel()
    vg = np.asarray(vg, dtype=np.float64).reshape(-1, 3)
    lam, theta = np.linalg.eigh(np.asarray(mat, dtype=np.float64), UPLO="U")
    if 0 < num_eigenvalues < E.size:
        lam, theta = lam[:num_eigenvalues], theta[:, :num_eigenvalues]
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        term = _poppm1(E, T)
        dndt = term * E / T / T
        w = np.where((E > 0.0)[:, None], (dndt / np.sqrt(term))[:, None] * vg, 0.0)    # (ns, 3)
    good = lam > 0.0
    rpop = np.zeros((lam.size, 3))
    rpop[good] = (theta[:, good].T @ w) / lam[good][:, None]
    pop = theta[:, good] @ rpop[good]                                               # (ns, 3)
    with np.errstate(invalid="ignore"):
        pop = np.where((E > 0.0)[:, None], pop * np.sqrt(np.where(E > 0.0, term, 1.0))[:, None], pop)
    keep = E >= _PH_EXCLUDE_CUTOFF
    kappa = np.einsum("si,sj,s->ij", pop[keep], vg[keep], E[keep]) / float(num_q) / float(volume)
    return lam, theta, kappa


def symmetrize_coupling(c, e1, e2, e3):
    c = _d(c).copy()
    nb1, nb2, nb3 = c.shape
    lib().orc_symmetrize_coupling(_p(c), nb1, nb2, nb3, _p(_d(e1)), _p(_d(e2)), _p(_d(e3)))
    return c


def rta_kappa(E, vg, Aout, temps_ry, nqmesh, volume):
    ns = E.size
    T = _d(temps_ry)
    kappa = np.zeros((len(T), 3, 3))
    lib().orc_rta_kappa(ns, len(T), _p(T), _p(_d(E)), _p(_d(vg)), _p(_d(Aout)), int(nqmesh),
                        float(volume), _p(kappa))
    return kappa


def _ip(a):
    return np.ascontiguousarray(a, dtype=np.int32).ctypes.data_as(_I)


def _f32c(a):
    """complex64 array -> contiguous interleaved float32."""
    return np.ascontiguousarray(a, dtype=np.complex64).view(np.float32)


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class ElectronH0Wannier:
    """CPU FP64 restatement of ElectronH0Wannier (no shifted vectors)."""

    def __init__(self, R, deg, H):
        self.R, self.deg = _d(R), _d(deg)
        self.H = _c(H)
        self.nR, self.nw = H.shape[0], H.shape[1]

    def diagonalize(self, k_cart, velocities=False):
        k = _d(np.atleast_2d(k_cart))
        nk = k.shape[0]
        E = np.zeros((nk, self.nw))
        U = np.zeros((nk, self.nw, self.nw, 2))
        vg = np.zeros((nk, self.nw, 3)) if velocities else None
        rc = lib().orc_el_diag(self.nw, self.nR, _p(self.R), _p(self.deg), _p(self.H), nk, _p(k), _p(E),
                               _p(U), _p(vg) if velocities else None)
        assert rc == 0
        U = U[..., 0] + 1j * U[..., 1]
        return (E, U, vg) if velocities else (E, U)


class InteractionElPhWan:
    """CPU FP64 restatement of InteractionElPhWan (cacheElPh, calcCouplingSquared)."""

    def __init__(self, Re, degE, Rp, degP, g):
        self.Re, self.degE, self.Rp, self.degP = _d(Re), _d(degE), _d(Rp), _d(degP)
        self.g = _f32c(g)
        self.nRe, self.nRp, self.nph, self.nw = g.shape[0], g.shape[1], g.shape[2], g.shape[3]

    def cache_elph(self, U1, k1):
        U1 = np.asarray(U1)
        nb1 = U1.shape[1]
        out = np.zeros((self.nRp, self.nph, nb1, self.nw, 2))
        lib().orc_elph_cache(self.nw, self.nph, self.nRe, self.nRp, _p(self.Re), _p(self.degE), _fp(self.g),
                             _p(_d(k1)), _p(_c(U1)), nb1, _p(out))
        self.cached = out
        self.nb1 = nb1
        return out[..., 0] + 1j * out[..., 1]

    def calc_coupling_squared(self, U2s, nb2s, ev3s, q3s):
        nk2 = len(nb2s)
        nb2max = U2s.shape[2]
        out = np.zeros((nk2, self.nb1, nb2max, self.nph))
        lib().orc_elph_couplings(self.nw, self.nph, self.nRp, _p(self.Rp), _p(self.degP), _p(self.cached),
                                 self.nb1, nk2, _p(_d(q3s)), _p(_c(U2s)), _ip(nb2s),
                                 nb2max, _p(_c(ev3s)), _p(out))
        return out


def el_linewidths(elph, kmesh, qmesh, Ek, Uk, vk, lo, hi, Eq, evq, kcart, recipk, k1list, temps_ry, mu,
                  smearing, sigma, norm):
    """ElScatteringMatrix::builder (linewidth mode): returns (nT, nk1, nw)."""
    nk1 = len(k1list)
    nT = len(temps_ry)
    out = np.zeros((nT, nk1, elph.nw))
    vk_ = _d(vk) if vk is not None else _d(np.zeros((Ek.shape[0], Ek.shape[1], 3)))
    rc = lib().orc_el_linewidths(elph.nw, elph.nph, elph.nRe, elph.nRp, _p(elph.Re), _p(elph.degE), _p(elph.Rp),
                                 _p(elph.degP), _fp(elph.g), _ip(kmesh),
                                 _ip(qmesh), _p(_d(Ek)), _p(_c(Uk)),
                                 _p(vk_), _ip(lo),
                                 _ip(hi), _p(_d(Eq)), _p(_c(evq)),
                                 _p(_d(kcart)), _p(_d(recipk)), nk1, _ip(k1list),
                                 nT, _p(_d(temps_ry)), float(mu), 1 if smearing == "adaptive" else 0,
                                 float(sigma), float(norm), _p(out))
    assert rc == 0
    return out
