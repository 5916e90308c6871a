"""Seeded synthetic force constants with the shapes of the benchmark workloads.

No reference generator exists: the reference reads DFT force constants from
files (QE ``.fc`` for FC2, src/parser/qe_input_parser.cpp:385-560; ShengBTE
``FORCE_CONSTANTS_3RD`` for FC3, src/parser/ifc3_parser.cpp:648-840).  This
module produces arrays in exactly those in-memory layouts:

* FC2 as ``forceConstants(3,3,n1,n2,n3,nat,nat)`` in Ry/Bohr^2, element
  (i,j,m,na,nb) = Phi_ij(atom na in cell R_m; atom nb in cell 0);
* FC3 as the dense ``D3(nb,nb,nb,nr3,nr2)`` tensor in Ry/Bohr^3 with the list
  of distinct second/third cell vectors (Bohr) and unit weights, as the
  ShengBTE reader builds it.

Randomness comes from a counter-based generator (splitmix64 -> uniform in
(0,1] -> Box-Muller, FP64) so every consumer regenerates identical inputs.
"""
from dataclasses import dataclass
import itertools

import numpy as np

from . import constants as C
from .lattice import Crystal

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
SEED_BASE = 0x5048584B00000000


def _splitmix64(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
    return z ^ (z >> np.uint64(31))


class CounterRNG:
    """Stateless counter-based RNG: value i of stream s depends only on (seed, s, i)."""

    def __init__(self, seed):
        self.seed = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)

    def uniform(self, stream, n):
        with np.errstate(over="ignore"):
            ctr = np.arange(n, dtype=np.uint64) + (np.uint64(stream) << np.uint64(40))
            z = _splitmix64(self.seed ^ _splitmix64(ctr))
        return ((z >> np.uint64(11)).astype(np.float64) + 1.0) * (2.0 ** -53)

    def normal(self, stream, n):
        u = self.uniform(stream, 2 * n)
        u1, u2 = u[0::2], u[1::2]
        return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


# ---------------------------------------------------------------------------
# cells
# ---------------------------------------------------------------------------

def diamond_crystal(a_ang=5.43, mass_amu=28.0):
    """Diamond-structure cell: FCC lattice, 2 atoms, a=5.43 A, 28 amu."""
    a = a_ang / C.distanceBohrToAng
    cell = 0.5 * a * np.array([[0.0, 1.0, 1.0], [1.0, 0.0, 1.0], [1.0, 1.0, 0.0]]).T
    pos = np.array([[0.0, 0.0, 0.0], [0.25 * a, 0.25 * a, 0.25 * a]])
    return Crystal(cell, pos, np.array([0, 0]), np.array([mass_amu * C.massAmuToRy]))


def perovskite_crystal(a_ang=3.9, masses_amu=(137.0, 48.0, 16.0, 16.0, 16.0)):
    """5-atom cubic perovskite-like cell ABO3 (A at corner, B at centre)."""
    a = a_ang / C.distanceBohrToAng
    cell = a * np.eye(3)
    frac = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5],
                     [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
    pos = frac @ cell.T
    return Crystal(cell, pos, np.arange(5), np.array(masses_amu) * C.massAmuToRy)


def twelve_atom_crystal(seed, a_ang=5.43):
    """12-atom cubic cell (3x the diamond primitive basis along a cubic cell).

    Atoms sit on the 8 diamond sites of the conventional cubic cell plus 4
    octahedral interstitials; masses are drawn uniformly in [20, 80] amu.
    """
    a = a_ang / C.distanceBohrToAng
    cell = a * np.eye(3)
    fcc = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]])
    frac = np.vstack([fcc, fcc + 0.25, fcc + np.array([0.5, 0.0, 0.0])])
    pos = frac @ cell.T
    rng = CounterRNG(seed)
    masses = 20.0 + 60.0 * rng.uniform(7, 12)
    return Crystal(cell, pos, np.arange(12), masses * C.massAmuToRy)


# ---------------------------------------------------------------------------
# FC2: central springs on a coarse supercell grid
# ---------------------------------------------------------------------------

def spring_fc2(crystal, shells, grid=(4, 4, 4), tol=1e-6):
    """Central-spring harmonic force constants in the QE ``.fc`` layout.

    ``shells`` is a list of (radius_bohr, k_ry_per_bohr2, pair_filter) where
    pair_filter(na, nb) selects which atom pairs the shell connects (None =
    all).  Off-site blocks are -k * d d^T for every neighbour vector d; the
    on-site block is fixed by the acoustic sum rule.
    """
    nat = crystal.num_atoms
    g = np.array(grid)
    fc = np.zeros((3, 3, g[0], g[1], g[2], nat, nat))
    A = crystal.direct_cell
    rmax = max(s[0] for s in shells) + tol
    nmax = int(np.ceil(rmax / min(np.linalg.norm(A, axis=0)))) + 2
    rng = range(-nmax, nmax + 1)
    for na in range(nat):
        for nb in range(nat):
            for n1, n2, n3 in itertools.product(rng, rng, rng):
                R = A @ np.array([n1, n2, n3], dtype=np.float64)
                d = R + crystal.positions[na] - crystal.positions[nb]
                r = np.linalg.norm(d)
                if r < tol:
                    continue
                for radius, k, filt in shells:
                    if abs(r - radius) < tol and (filt is None or filt(na, nb)):
                        dd = d / r
                        fc[:, :, n1 % g[0], n2 % g[1], n3 % g[2], na, nb] += -k * np.outer(dd, dd)
    for na in range(nat):
        s = fc[:, :, :, :, :, na, :].sum(axis=(2, 3, 4, 5))
        fc[:, :, 0, 0, 0, na, na] -= s
    return fc


def _k_ry(k_ev_ang2):
    return k_ev_ang2 * C.distanceBohrToAng ** 2 / C.energyRyToEv


def diamond_fc2(crystal, k1=45.0, k2=5.0, grid=(4, 4, 4)):
    a = np.linalg.norm(crystal.direct_cell[:, 0]) * np.sqrt(2.0)
    shells = [(a * np.sqrt(3.0) / 4.0, _k_ry(k1), None), (a / np.sqrt(2.0), _k_ry(k2), None)]
    return spring_fc2(crystal, shells, grid)


def perovskite_fc2(crystal, grid=(4, 4, 4)):
    a = crystal.direct_cell[0, 0]
    shells = [(0.5 * a, _k_ry(12.0), None),                    # B-O
              (a / np.sqrt(2.0), _k_ry(3.0), None),            # A-O and O-O
              (a * np.sqrt(3.0) / 2.0, _k_ry(2.0), None),      # A-B
              (a, _k_ry(1.5), None)]                           # A-A, B-B, O-O
    return spring_fc2(crystal, shells, grid)


def twelve_atom_fc2(crystal, grid=(2, 2, 2)):
    a = crystal.direct_cell[0, 0]
    shells = [(a * np.sqrt(3.0) / 4.0, _k_ry(40.0), None),
              (0.5 * a, _k_ry(12.0), None),
              (a / np.sqrt(2.0), _k_ry(5.0), None)]
    return spring_fc2(crystal, shells, grid)


# ---------------------------------------------------------------------------
# FC3: (R2,R3) pairs closed under index permutations, symmetrised + ASR
# ---------------------------------------------------------------------------

def _orbit(p):
    """Images of the cell pair (R2,R3) under the 6 permutations of the triple
    (0, R2, R3), each translated so the first cell is 0, with the transpose
    that maps the (i1,i2,i3) block onto the image block."""
    R2, R3 = p
    neg = lambda v: tuple(-x for x in v)
    sub = lambda u, v: tuple(x - y for x, y in zip(u, v))
    return [((R2, R3), (0, 1, 2)),
            ((R3, R2), (0, 2, 1)),
            ((neg(R2), sub(R3, R2)), (1, 0, 2)),
            ((sub(R2, R3), neg(R3)), (2, 1, 0)),
            ((sub(R3, R2), neg(R2)), (1, 2, 0)),
            ((neg(R3), sub(R2, R3)), (2, 0, 1))]


@dataclass
class FC3:
    D3: np.ndarray        # (nb,nb,nb,nr3,nr2) Ry/Bohr^3
    R2: np.ndarray        # (nr2,3) Bohr
    R3: np.ndarray        # (nr3,3) Bohr
    w2: np.ndarray        # (nr2,nat,nat)
    w3: np.ndarray        # (nr3,nat,nat)
    num_pairs: int
    iterations: int = 0
    residual: float = 0.0


def random_fc3(crystal, num_pairs, seed, amp_ev=3.0, decay_ang=4.0,
               tol=1e-12, max_iter=500):
    """FC3 on ``num_pairs`` (R2,R3) lattice-vector pairs.

    Orbits of pairs under index permutation are added in order of increasing
    largest |R| among R2, R3, R3-R2 (ties broken by the seeded RNG), skipping
    an orbit that would overshoot, until exactly ``num_pairs`` pairs are in.
    Entries start as N(0,1)*amp*exp(-(|R2|+|R3|)/decay) (eV/A^3, A) and are
    then alternately permutation-symmetrised and projected onto the acoustic
    sum rule sum_{R3,c} Phi(0a,R2b,R3c) = 0 until both residuals are below
    tol relative to max|Phi| (at most max_iter rounds).
    """
    nat = crystal.num_atoms
    nb = 3 * nat
    A = crystal.direct_cell
    rng = CounterRNG(seed)
    nmax = 4
    vecs = [v for v in itertools.product(range(-nmax, nmax + 1), repeat=3)]
    length = {v: np.linalg.norm(A @ np.array(v, dtype=np.float64)) for v in vecs}
    vecset = set(vecs)
    # candidate orbits with all three vectors within the 9th distinct length
    # (further shells only when those cannot supply num_pairs pairs)
    dl = sorted(set(round(x, 6) for x in length.values()))
    pairs = []
    for shell in range(8, len(dl)):
        lim = dl[shell]
        orbits = {}
        short = [v for v in vecs if length[v] <= lim + 1e-9]
        for R2 in short:
            for R3 in short:
                R32 = tuple(x - y for x, y in zip(R3, R2))
                if R32 not in vecset or length[R32] > lim + 1e-9:
                    continue
                imgs = frozenset(q for q, _ in _orbit((R2, R3)))
                if imgs in orbits:
                    continue
                orbits[imgs] = max(length[R2], length[R3], length[R32])
        keys = list(orbits.keys())
        tie = rng.uniform(1, len(keys))
        order = sorted(range(len(keys)), key=lambda i: (round(orbits[keys[i]], 6), tie[i]))
        # greedy in that order; when the orbit sizes (1, 3, 6) cannot add up to
        # num_pairs with the single-pair orbit in, retry without it
        for min_size in (1, 2):
            pairs = []
            for i in order:
                orb = sorted(keys[i])
                if len(orb) >= min_size and len(pairs) + len(orb) <= num_pairs:
                    pairs.extend(orb)
                if len(pairs) == num_pairs:
                    break
            if len(pairs) == num_pairs:
                break
        if len(pairs) == num_pairs:
            break
    if len(pairs) != num_pairs:
        raise RuntimeError("could not assemble %d permutation-closed pairs" % num_pairs)
    pidx = {p: i for i, p in enumerate(pairs)}
    # initial random blocks
    scale = C.distanceBohrToAng ** 3 / C.energyRyToEv
    z = rng.normal(2, num_pairs * nb ** 3).reshape(num_pairs, nb, nb, nb)
    B = np.empty_like(z)
    for p, i in pidx.items():
        r2 = length[p[0]] * C.distanceBohrToAng
        r3 = length[p[1]] * C.distanceBohrToAng
        B[i] = z[i] * amp_ev * np.exp(-(r2 + r3) / decay_ang) * scale
    # precompute permutation maps and ASR groups
    perm_maps = [[(pidx[q], ax) for q, ax in _orbit(p)] for p in pairs]
    R2s = sorted(set(p[0] for p in pairs))
    groups = {R2: [pidx[p] for p in pairs if p[0] == R2] for R2 in R2s}

    # image k of every pair is a permutation of the pair set with one transpose
    jmap = np.array([[j for j, _ in imgs] for imgs in perm_maps])        # (num_pairs, 6)
    axes = [ax for _, ax in perm_maps[0]]

    def symmetrise(B):
        S = np.zeros_like(B)
        for k, ax in enumerate(axes):
            S[jmap[:, k]] += np.transpose(B, (0,) + tuple(1 + a for a in ax))
        return S / 6.0

    def asr_project(B):
        out = B.copy()
        for R2, idx in groups.items():
            blk = B[idx].reshape(len(idx), nb, nb, nat, 3)
            s = blk.sum(axis=(0, 3))  # (nb, nb, 3)
            cnt = len(idx) * nat
            out[idx] = (blk - s[None, :, :, None, :] / cnt).reshape(len(idx), nb, nb, nb)
        return out

    def asr_residual(B):
        r = 0.0
        for R2, idx in groups.items():
            blk = B[idx].reshape(len(idx), nb, nb, nat, 3)
            r = max(r, np.abs(blk.sum(axis=(0, 3))).max())
        return r

    if nb >= 24:
        # large cells (the 36-branch one): the same alternating projections,
        # vectorised with torch on a GPU when one is present
        B, it, res = _project_torch(B, jmap, axes, R2s, pairs, nat, nb, tol, max_iter)
    else:
        for it in range(max_iter):
            B = asr_project(symmetrise(B))
            ref = np.abs(B).max()
            res = max(np.abs(symmetrise(B) - B).max(), asr_residual(B)) / ref
            if res < tol:
                break
    # dense ShengBTE-style layout
    Rvecs = sorted(set(p[0] for p in pairs) | set(p[1] for p in pairs))
    ridx = {v: i for i, v in enumerate(Rvecs)}
    nr = len(Rvecs)
    D3 = np.zeros((nb, nb, nb, nr, nr))
    cols = np.empty(num_pairs, dtype=np.int64)
    for p, i in pidx.items():
        cols[i] = ridx[p[1]] * nr + ridx[p[0]]
    D3.reshape(nb ** 3, nr * nr)[:, cols] = B.reshape(num_pairs, nb ** 3).T
    Rcart = np.array([A @ np.array(v, dtype=np.float64) for v in Rvecs])
    w = np.ones((nr, nat, nat))
    return FC3(D3, Rcart.copy(), Rcart.copy(), w, w.copy(), num_pairs, it + 1, res)


def _project_torch(B, jmap, axes, R2s, pairs, nat, nb, tol, max_iter):
    """random_fc3's alternating projections (index-permutation symmetrisation,
    then the acoustic sum rule per R2 group) for large blocks, with torch
    index_add_ instead of numpy loops.  Returns (B, iterations, residual)."""
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    n = B.shape[0]
    gidx = {R2: g for g, R2 in enumerate(R2s)}
    gid = torch.tensor([gidx[p[0]] for p in pairs], dtype=torch.int64, device=dev)
    cnt = torch.bincount(gid, minlength=len(R2s)).to(torch.float64) * nat
    jm = torch.from_numpy(np.ascontiguousarray(jmap)).to(dev)
    X = torch.from_numpy(B).to(dev)

    def sym(Y):
        S = torch.zeros_like(Y)
        for k, ax in enumerate(axes):
            S.index_add_(0, jm[:, k], Y.permute((0,) + tuple(1 + a for a in ax)))
        return S / 6.0

    def group_sums(Y):
        ps = Y.reshape(n, nb, nb, nat, 3).sum(dim=3)
        return torch.zeros((len(R2s), nb, nb, 3), dtype=Y.dtype, device=dev).index_add_(0, gid, ps)

    def asr(Y):
        corr = (group_sums(Y) / cnt[:, None, None, None])[gid]
        return (Y.reshape(n, nb, nb, nat, 3) - corr[:, :, :, None, :]).reshape(n, nb, nb, nb)

    S = sym(X)
    res = float("inf")
    it = 0
    for it in range(max_iter):
        X = asr(S)
        S = sym(X)
        ref = X.abs().max()
        res = float(torch.maximum((S - X).abs().max(), group_sums(X).abs().max()) / ref)
        if res < tol:
            break
    out = X.cpu().numpy()
    del X, S
    if dev == "cuda":
        torch.cuda.empty_cache()
    return out, it, res


# ---------------------------------------------------------------------------
# benchmark workloads
# ---------------------------------------------------------------------------

@dataclass
class Workload:
    name: str
    crystal: Crystal
    fc2: np.ndarray
    fc3: FC3
    mesh: tuple
    temperatures_k: tuple
    smearing: str          # "gaussian" or "adaptive"
    sigma_ry: float        # Gaussian width (Ry); ignored for adaptive


def diamond_workload(mesh=(8, 8, 8), smearing="gaussian", temperatures_k=(300.0,),
                     num_pairs=400):
    """Diamond cell with spring FC2 and the seed-0 FC3 (shared by both diamond
    workloads, which differ only in mesh, smearing and temperatures)."""
    cr = diamond_crystal()
    fc2 = diamond_fc2(cr)
    fc3 = random_fc3(cr, num_pairs, SEED_BASE + 0)
    return Workload("diamond-%dx%dx%d" % tuple(mesh), cr, fc2, fc3, tuple(mesh),
                    tuple(temperatures_k), smearing, 0.3 / C.ryToTHz)


def config0():
    """Diamond, 8^3 mesh, Gaussian 0.3 THz, 300 K (CPU-runnable case)."""
    return diamond_workload((8, 8, 8), "gaussian", (300.0,))


def config1():
    """Diamond, 20^3 mesh, adaptive smearing, 100/300/600 K (headline case)."""
    return diamond_workload((20, 20, 20), "adaptive", (100.0, 300.0, 600.0))


def perovskite_workload(mesh=(24, 24, 24), num_pairs=1500, fc_grid=(7, 7, 7), smearing="adaptive",
                        temperatures_k=(300.0,)):
    """Batched uneven instances: the 5-atom perovskite-like cell (15 branches),
    spring FC2 on a 7x7x7 grid, 1500 FC3 pairs (seed of config 2)."""
    cr = perovskite_crystal()
    fc2 = perovskite_fc2(cr, fc_grid)
    fc3 = random_fc3(cr, num_pairs, SEED_BASE + 2)
    return Workload("perovskite-%dx%dx%d" % tuple(mesh), cr, fc2, fc3, tuple(mesh),
                    tuple(temperatures_k), smearing, 0.3 / C.ryToTHz)


def config2(mesh=(24, 24, 24)):
    """5-atom perovskite, 24^3 mesh, per-q1 q2 window (use q2_window on its bands)."""
    return perovskite_workload(mesh)


def twelve_atom_workload(mesh=(16, 16, 16), num_pairs=4000, smearing="adaptive", temperatures_k=(300.0,)):
    """The learned-screening cell: 12 atoms (36 branches), masses uniform in
    20-80 amu, spring FC2 on a 2x2x2 grid, num_pairs FC3 pairs (seed of config 4)."""
    cr = twelve_atom_crystal(SEED_BASE + 4)
    fc2 = twelve_atom_fc2(cr)
    fc3 = random_fc3(cr, num_pairs, SEED_BASE + 4)
    return Workload("twelve-atom-%dx%dx%d" % tuple(mesh), cr, fc2, fc3, tuple(mesh),
                    tuple(temperatures_k), smearing, 0.3 / C.ryToTHz)


def config4(mesh=(16, 16, 16)):
    """12-atom cell, 36 branches, 4000 FC3 pairs, 16^3 mesh."""
    return twelve_atom_workload(mesh)


def q2_window(E, mesh, seed=SEED_BASE + 2, keep_min=0.2, keep_max=1.0):
    """Per-q1 energy window on q2 (uneven work; no counterpart in the reference).

    The window energy of q2 is the largest phonon energy at q2 or at -q2, so
    q2 and -q2 always fall on the same side of a window.  Each q1 draws a kept
    fraction f uniform in [keep_min, keep_max] from the counter RNG (stream 7,
    counter q1); its cut is the window energy of rank ceil(f nq) - 1 in
    ascending order, and q2 is paired with q1 iff energy[q2] <= cut[q1] (ties
    kept).  Returns (energy (nq), cut (nq))."""
    E = np.asarray(E)
    nq = E.shape[0]
    n0, n1, n2 = mesh
    idx = np.arange(nq)
    ix, iy, iz = idx % n0, (idx // n0) % n1, idx // (n0 * n1)
    neg = ((n2 - iz) % n2) * n0 * n1 + ((n1 - iy) % n1) * n0 + (n0 - ix) % n0
    energy = np.maximum(E.max(axis=1), E[neg].max(axis=1))
    f = keep_min + (keep_max - keep_min) * CounterRNG(seed).uniform(7, nq)
    srt = np.sort(energy)
    rank = np.clip(np.ceil(f * nq).astype(np.int64) - 1, 0, nq - 1)
    return energy, srt[rank]


# ---------------------------------------------------------------------------
# electron-phonon Wannier model (workload of the el-ph path)
# ---------------------------------------------------------------------------

@dataclass
class ElPhModel:
    crystal: Crystal
    Re: np.ndarray      # (nRe,3) Bohr
    degE: np.ndarray    # (nRe,)
    H: np.ndarray       # (nRe,nw,nw) complex128, Ry; H(-R) = H(R)^dagger
    Rp: np.ndarray      # (nRp,3) Bohr
    degP: np.ndarray    # (nRp,)
    g: np.ndarray       # (nRe,nRp,nph,nw,nw) complex64, Ry/Bohr


def lattice_cube(crystal, n):
    """The (2n+1)^3 lattice vectors i a1 + j a2 + k a3 with |i|,|j|,|k| <= n
    (Cartesian, Bohr), each with degeneracy 1; index of -R is (count-1) - index of R."""
    r = np.arange(-n, n + 1)
    ijk = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
    R = ijk @ crystal.direct_cell.T
    return R, np.ones(len(R))


def wannier_hamiltonian(crystal, nw=8, ncell=3, seed=SEED_BASE + 3, amp_ev=2.0, decay_ang=3.0):
    """H(R) = (X(R) + X(-R)^dagger)/2 with X complex N(0,1) amp exp(-|R|/decay):
    Hermitian-consistent, so H(k) is Hermitian at every k."""
    R, deg = lattice_cube(crystal, ncell)
    nR = len(R)
    rng = CounterRNG(seed)
    x = rng.normal(0, 2 * nR * nw * nw).reshape(nR, nw, nw, 2)
    X = x[..., 0] + 1j * x[..., 1]
    dist = np.linalg.norm(R, axis=1) * C.distanceBohrToAng
    X *= (amp_ev / C.energyRyToEv * np.exp(-dist / decay_ang))[:, None, None]
    H = 0.5 * (X + np.conj(np.transpose(X[::-1], (0, 2, 1))))
    return R, deg, H


def elph_coupling(crystal, nRe_cell, nRp_cell, nph, nw, seed=SEED_BASE + 3, amp=0.1, decay_ang=4.0):
    """g(Re,Rp,nu,w1,w2) complex64 N(0,1) amp eV/A exp(-(|Re|+|Rp|)/decay), in Ry/Bohr;
    generated per Re (stream 1 + iRe of the counter RNG) to bound memory."""
    Re, degE = lattice_cube(crystal, nRe_cell)
    Rp, degP = lattice_cube(crystal, nRp_cell)
    rng = CounterRNG(seed)
    dE = np.linalg.norm(Re, axis=1) * C.distanceBohrToAng
    dP = np.linalg.norm(Rp, axis=1) * C.distanceBohrToAng
    unit = amp / C.energyRyToEv * C.distanceBohrToAng
    per = len(Rp) * nph * nw * nw
    g = np.empty((len(Re), len(Rp), nph, nw, nw), dtype=np.complex64)
    for ie in range(len(Re)):
        x = rng.normal(1 + ie, 2 * per).reshape(len(Rp), nph, nw, nw, 2)
        scale = (unit * np.exp(-(dE[ie] + dP) / decay_ang))[:, None, None, None]
        g[ie] = ((x[..., 0] + 1j * x[..., 1]) * scale).astype(np.complex64)
    return Re, degE, Rp, degP, g


def elph_model(crystal=None, nw=8, ncell_h=3, ncell_e=3, ncell_p=3, seed=SEED_BASE + 3):
    """Wannier Hamiltonian on (2 ncell_h + 1)^3 vectors and el-ph coupling on
    (2 ncell_e + 1)^3 x (2 ncell_p + 1)^3 vectors for the diamond cell (6 branches)."""
    cr = crystal if crystal is not None else diamond_crystal()
    Rh, degh, H = wannier_hamiltonian(cr, nw, ncell_h, seed)
    Re, degE, Rp, degP, g = elph_coupling(cr, ncell_e, ncell_p, cr.num_bands, nw, seed + (1 << 20))
    if ncell_e != ncell_h:
        raise ValueError("the Hamiltonian and the coupling share the electronic vectors")
    return ElPhModel(cr, Re, degE, H, Rp, degP, g)


def active_window(E, mu, window):
    """Active band range [lo, hi) of every k point: bands with |E - mu| <= window."""
    act = (E >= mu - window) & (E <= mu + window)
    nk, nw = E.shape
    lo = np.where(act.any(1), act.argmax(1), 0).astype(np.int32)
    hi = np.where(act.any(1), nw - act[:, ::-1].argmax(1), 0).astype(np.int32)
    return lo, hi
