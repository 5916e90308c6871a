"""Learned screening of 3-phonon triplets (no counterpart in the reference).

A small network (12 -> 256 -> 256 -> 256 -> 1, GELU, BF16 weights, FP32
accumulation; hand-written CUDA kernels in libphx) is trained on triplet
contributions that the exact GPU vertex generates, and predicts
log10(c / Gamma(q1, b1)) for a branch triplet (q1, q2, b1, b2, b3): its
contribution c to the linewidth of mode (q1, b1) relative to that linewidth.
Screening drops the live triplets predicted below a threshold; every retained
triplet keeps its exact value.

Features of a triplet (12): the fractional coordinates of q1 and q2, the three
frequencies divided by the largest frequency of the mesh, and the three
group-velocity norms divided by the largest one.

Triplet convention: the builder evaluates only the "+" vertex and lets each
(q1, q2, b1, b2, b3) carry the "+" process of (q1, q2) and the "-" processes of
(q1, -q2) (same q3 = q1 + q2, time reversal), so the contribution of a triplet
is |V+|^2 (symmetrised over degenerate blocks) times the sum of those rate
factors, at the first temperature.

Pair-level screening (the screened builder, phx_ph_linewidths_screened): the
same network shape with 12 pair inputs (pair_features) predicts, for a vertex
(q1, q2) -- one "triplet" in the benchmark's unit of work -- log10 of the
largest fraction it adds to the linewidth of any mode of q1
(pair_targets); the builder drops the vertices predicted below a threshold
and evaluates the rest exactly.  Training pairs come from the exact builder
itself, one q2 at a time (pair_contributions).
"""
import ctypes

import numpy as np

from . import _abi
from . import constants as C
from ._abi import check

NIN = 12
HIDDEN = 256
DEPTH = 3
FLOOR = 1e-12     # relative contributions are clamped here before the logarithm

_F = ctypes.POINTER(ctypes.c_float)


def _fp(a):
    return a.ctypes.data_as(_F)


def layer_dims(nin=NIN, hidden=HIDDEN, depth=DEPTH):
    return [nin] + [hidden] * depth + [1]


def init_params(nin=NIN, hidden=HIDDEN, depth=DEPTH, seed=0):
    """He-initialised weights, zero biases, flat FP32 vector (W (nout,nin) then b per layer)."""
    dims = layer_dims(nin, hidden, depth)
    rng = np.random.default_rng(seed)
    ps = []
    for l in range(len(dims) - 1):
        ps.append((rng.normal(size=(dims[l + 1], dims[l])) * np.sqrt(2.0 / dims[l])).ravel())
        ps.append(np.zeros(dims[l + 1]))
    return np.concatenate(ps).astype(np.float32)


class ScreeningMLP:
    """The screening network on the GPU (phx_mlp)."""

    def __init__(self, ctx, nin=NIN, hidden=HIDDEN, depth=DEPTH, params=None, seed=0):
        self.ctx = ctx
        self.dims = layer_dims(nin, hidden, depth)
        p = np.ascontiguousarray(params if params is not None else init_params(nin, hidden, depth, seed),
                                 dtype=np.float32)
        h = ctypes.c_void_p()
        check(_abi.load().phx_mlp_create(ctx.h, nin, hidden, depth, _fp(p), ctypes.byref(h)), ctx.h)
        self.h = h
        self.nparam = int(_abi.load().phx_mlp_num_params(h))
        assert self.nparam == p.size

    def params(self):
        p = np.zeros(self.nparam, dtype=np.float32)
        check(_abi.load().phx_mlp_get_params(self.h, _fp(p)), self.ctx.h)
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(_abi.load().phx_mlp_set_params(self.h, _fp(p)), self.ctx.h)

    def infer(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.zeros(X.shape[0], dtype=np.float32)
        check(_abi.load().phx_mlp_infer(self.h, X.shape[0], _fp(X), _fp(y)), self.ctx.h)
        return y

    def grad(self, X, t):
        X = np.ascontiguousarray(X, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(self.nparam, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        check(_abi.load().phx_mlp_grad(self.h, X.shape[0], _fp(X), _fp(t), _fp(g), _fp(loss)), self.ctx.h)
        return float(loss[0]), g

    def train(self, X, t, epochs=10, batch=1024, lr=1e-3, seed=1):
        X = np.ascontiguousarray(X, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        losses = np.zeros(max(1, epochs), dtype=np.float32)
        check(_abi.load().phx_mlp_train(self.h, X.shape[0], _fp(X), _fp(t), int(epochs), int(batch), float(lr),
                                        int(seed), _fp(losses)), self.ctx.h)
        return losses[:epochs]

    def close(self):
        if getattr(self, "h", None):
            _abi.load().phx_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# training data from the exact vertex
# ---------------------------------------------------------------------------

def _symmetrize(c, e1, e2, e3):
    """symmetrizeCoupling (scattering.cpp:1209-1318) on c (nq1, nb, nb, nb) with
    per-q1 energies e1 (nq1, nb), e2 (nb) and per-q1 e3 (nq1, nb); only the q1
    rows with a degenerate pair are touched."""
    nq1, nb = e1.shape
    out = c.copy()
    for axis, e in ((1, e1), (2, np.broadcast_to(e2, (nq1, nb))), (3, e3)):
        rows = np.nonzero((np.abs(np.diff(e, axis=1)) < 1e-6).any(axis=1))[0]
        for i in rows:
            b = 0
            while b < nb:
                d = 1
                while b + d < nb and abs(e[i, b] - e[i, b + d]) < 1e-6:
                    d += 1
                if d > 1:
                    sl = [i, slice(None), slice(None), slice(None)]
                    sl[axis] = slice(b, b + d)
                    blk = out[tuple(sl)]
                    m = blk.sum(axis=axis - 1, keepdims=True) / float(d)
                    out[tuple(sl)] = np.broadcast_to(m, blk.shape)
                b += d
    return out


def rate_factors(E, vg, iq2, iq3, iq2m, qT, nq, temperature, smearing="adaptive", sigma=0.0):
    """Rate factors F (nq1, b1, b2, b3) of the "+" process of (q1, q2) and the "-"
    processes of (q1, -q2) with q3 = q1 + q2 (ph_scattering.cpp:338-380, 466-518),
    times 0.5 (the linewidth convention), FP64."""
    e1 = E[:, :, None, None]
    e2 = E[iq2][None, None, :, None]
    e2m = E[iq2m][None, None, :, None]
    e3 = E[iq3][:, None, None, :]

    def sig(v):
        s = np.sqrt(((v @ qT.T) ** 2).sum(-1) / 6)
        return np.where((s != 0) & (s < C.adaptiveBroadeningCutoff), C.adaptiveBroadeningCutoff, s)

    def delta(e, s, vz):
        if smearing == "gaussian":
            x = e / sigma
            return np.where(x > 6, 0.0, np.exp(-x * x) / sigma / np.sqrt(np.pi))
        sd = np.where(s > 0, s, 1.0)
        x = e / sd
        d = np.where(np.abs(e) > 2 * s, 0.0, np.exp(-x * x) / np.sqrt(np.pi) / sd / C.erf2)
        d = np.where(s == 0, 0.0, d)
        return np.where(vz & (e == 0), 1.0, d)

    v2 = vg[iq2][None, None, :, None, :]
    v2m = vg[iq2m][None, None, :, None, :]
    v3 = vg[iq3][:, None, None, :, :]
    sp, sm = sig(v2 - v3), sig(v2m - v3)
    vzp, vzm = np.all(v2 == v3, -1), np.all(v2m == v3, -1)
    ok = (e1 >= C.phExcludeCutoff) & (e3 >= C.phEnergyCutoff)
    dp = np.where(ok & (e2 >= C.phExcludeCutoff), delta(e1 + e2 - e3, sp, vzp), 0.0)
    d1 = np.where(ok & (e2m >= C.phExcludeCutoff), delta(e1 + e3 - e2m, sm, vzm), 0.0)
    d2 = np.where(ok & (e2m >= C.phExcludeCutoff), delta(e2m + e3 - e1, sm, vzm), 0.0)

    def bose(e):
        return np.where(e > 0, 1.0 / np.expm1(np.maximum(e, 1e-300) / temperature), 0.0)

    n1, n2, n2m, n3 = bose(e1), bose(e2), bose(e2m), bose(e3)
    pre = np.pi / 4 * 0.5 / nq
    with np.errstate(divide="ignore", invalid="ignore"):
        fp = pre * dp / (e1 * e2 * e3) * n1 * n2 * (n3 + 1)
        fm = pre / (e1 * e2m * e3) * (n3 * n1 * (n2m + 1) * d1 + n2m * n3 * (n1 + 1) * d2)
    return np.nan_to_num(fp, posinf=0.0) + np.nan_to_num(fm, posinf=0.0)


def triplet_contributions(v3, mesh, q_cart, E, U, vg, recip, temperature, q2_list, smearing="adaptive",
                          sigma=0.0):
    """Contributions c (len(q2_list), nq1, b1, b2, b3) to the linewidths, from the
    couplings of the GPU vertex v3 (Interaction3Ph) and FP64 rate factors."""
    n0, n1, n2 = mesh
    nq, nb = E.shape
    idx = np.arange(nq)
    ix, iy, iz = idx % n0, (idx // n0) % n1, idx // (n0 * n1)
    qT = np.asarray(recip) / np.asarray(mesh)[:, None]
    out = np.zeros((len(q2_list), nq, nb, nb, nb))
    for k, iq2 in enumerate(q2_list):
        jx, jy, jz = iq2 % n0, (iq2 // n0) % n1, iq2 // (n0 * n1)
        iq3 = ((iz + jz) % n2) * n0 * n1 + ((iy + jy) % n1) * n0 + (ix + jx) % n0
        iq2m = ((n2 - jz) % n2) * n0 * n1 + ((n1 - jy) % n1) * n0 + (n0 - jx) % n0
        v3.cacheD3(q_cart[iq2])
        cp, _ = v3.getCouplingsSquared(q_cart, q_cart[iq2], list(U), U[iq2], list(U[iq3]), list(U[iq3]))
        W = _symmetrize(np.stack(cp), E, E[iq2], E[iq3])
        F = rate_factors(E, vg, iq2, iq3, iq2m, qT, nq, temperature, smearing, sigma)
        out[k] = W * F
    return out


def features(mesh, E, vg, q2_list):
    """Features (len(q2_list), nq1, b1, b2, b3, 12) of every triplet."""
    n0, n1, n2 = mesh
    nq, nb = E.shape
    idx = np.arange(nq)
    frac = np.stack([idx % n0 / n0, (idx // n0) % n1 / n1, idx // (n0 * n1) / n2], 1)
    ix, iy, iz = idx % n0, (idx // n0) % n1, idx // (n0 * n1)
    emax = E.max()
    vn = np.linalg.norm(vg, axis=-1)
    vmax = max(vn.max(), 1e-300)
    out = np.zeros((len(q2_list), nq, nb, nb, nb, NIN), dtype=np.float32)
    for k, iq2 in enumerate(q2_list):
        jx, jy, jz = iq2 % n0, (iq2 // n0) % n1, iq2 // (n0 * n1)
        iq3 = ((iz + jz) % n2) * n0 * n1 + ((iy + jy) % n1) * n0 + (ix + jx) % n0
        f = out[k]
        f[..., 0:3] = frac[:, None, None, None, :]
        f[..., 3:6] = frac[iq2][None, None, None, None, :]
        f[..., 6] = (E / emax)[:, :, None, None]
        f[..., 7] = (E[iq2] / emax)[None, None, :, None]
        f[..., 8] = (E[iq3] / emax)[:, None, None, :]
        f[..., 9] = (vn / vmax)[:, :, None, None]
        f[..., 10] = (vn[iq2] / vmax)[None, None, :, None]
        f[..., 11] = (vn[iq3] / vmax)[:, None, None, :]
    return out


def relative_targets(c, A):
    """log10 of the contribution relative to the linewidth A (nq1, nb) of its mode."""
    r = c / np.where(A > 0, A, np.inf)[None, :, :, None, None]
    return np.log10(np.maximum(r, FLOOR)).astype(np.float32)


# ---------------------------------------------------------------------------
# pair-level screening (the screened builder)
# ---------------------------------------------------------------------------

def pair_features(mesh, E, q2_list):
    """Features (len(q2_list), nq1, 12) of the vertices (q1, q2): fractional
    coordinates of q1, q2 and q3 = q1 + q2, and the lowest phonon energy at
    each over the largest of the mesh (as the builder's pair_features_kernel,
    in FP32)."""
    n0, n1, n2 = mesh
    nq = E.shape[0]
    idx = np.arange(nq)
    ix, iy, iz = idx % n0, (idx // n0) % n1, idx // (n0 * n1)
    frac = np.stack([ix / n0, iy / n1, iz / n2], 1).astype(np.float32)
    emin = (E.min(axis=1) / np.abs(E).max()).astype(np.float32)
    out = np.zeros((len(q2_list), nq, NIN), dtype=np.float32)
    for k, iq2 in enumerate(q2_list):
        jx, jy, jz = iq2 % n0, (iq2 // n0) % n1, iq2 // (n0 * n1)
        iq3 = ((iz + jz) % n2) * n0 * n1 + ((iy + jy) % n1) * n0 + (ix + jx) % n0
        out[k, :, 0:3] = frac
        out[k, :, 3:6] = frac[iq2]
        out[k, :, 6:9] = frac[iq3]
        out[k, :, 9] = emin
        out[k, :, 10] = emin[iq2]
        out[k, :, 11] = emin[iq3]
    return out


def pair_contributions(sm, q2_list, temperature_index=0):
    """Exact contributions u (len(q2_list), nq1, nb) of each vertex (q1, q2) to the
    linewidths of q1 (A_out units, one temperature), from the builder sm
    (core.PhScatteringMatrix) run on one q2 at a time without finalisation."""
    nq, nb = sm.bands.nq, sm.bands.nb
    out = np.zeros((len(q2_list), nq, nb))
    for k, iq2 in enumerate(q2_list):
        A = sm.setup(int(iq2), int(iq2) + 1, finalize=False)
        out[k] = A[temperature_index].reshape(nq, nb)
    return out


def pair_targets(u, A):
    """log10 of the largest fraction max_b1 u(q1, q2, b1) / A(q1, b1) of a vertex,
    with A (nq1, nb) the unscreened, unaveraged linewidths (A_out units)."""
    r = u / np.where(A > 0, A, np.inf)[None, :, :]
    return np.log10(np.maximum(r.max(axis=2), FLOOR)).astype(np.float32)
