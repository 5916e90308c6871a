"""CPU FP64 oracle of the screening network (TEST INFRASTRUCTURE ONLY).

Restates the network of the library's screening path in numpy: MLP
nin -> hidden (x depth, GELU tanh form) -> 1 with every weight and bias rounded
to BF16 (round to nearest even) before use, mean-squared-error loss, and its
exact gradient by back-propagation (checked against central finite
differences by the tests).  There is no reference counterpart: phoebe has no
learned screening.
"""
import numpy as np


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (a >> 16) & 1
    r = ((a + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def layer_dims(nin, hidden, depth):
    return [nin] + [hidden] * depth + [1]


def unpack(params, dims):
    """Split the flat parameter vector into [(W (nout,nin), b (nout))]."""
    out, o = [], 0
    for l in range(len(dims) - 1):
        nin, nout = dims[l], dims[l + 1]
        W = params[o:o + nout * nin].reshape(nout, nin)
        o += nout * nin
        b = params[o:o + nout]
        o += nout
        out.append((W, b))
    return out


def init_params(nin, hidden, depth, seed=0):
    """He-style initial parameters (FP32)."""
    dims = layer_dims(nin, hidden, depth)
    rng = np.random.default_rng(seed)
    ps = []
    for l in range(len(dims) - 1):
        ps.append((rng.normal(size=(dims[l + 1], dims[l])) * np.sqrt(2.0 / dims[l])).ravel())
        ps.append(np.zeros(dims[l + 1]))
    return np.concatenate(ps).astype(np.float32)


_K = np.sqrt(2.0 / np.pi)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(_K * (x + 0.044715 * x ** 3)))


def gelu_d(x):
    t = np.tanh(_K * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * _K * (1.0 + 3 * 0.044715 * x * x)


def forward(params, X, dims, rounded=True):
    """Returns the output (B,) and the per-layer (Z, A) caches, FP64 arithmetic."""
    p = bf16(params).astype(np.float64) if rounded else np.asarray(params, dtype=np.float64)
    layers = unpack(p, dims)
    A = np.asarray(X, dtype=np.float64)
    cache = [(None, A)]
    for l, (W, b) in enumerate(layers):
        Z = A @ W.T + b
        A = gelu(Z) if l + 1 < len(layers) else Z
        cache.append((Z, A))
    return A[:, 0], cache


def loss_and_grad(params, X, t, dims, rounded=True):
    """Mean squared error and its gradient with respect to the (rounded) parameters."""
    p = bf16(params).astype(np.float64) if rounded else np.asarray(params, dtype=np.float64)
    layers = unpack(p, dims)
    y, cache = forward(params, X, dims, rounded)
    B = len(t)
    d = y - np.asarray(t, dtype=np.float64)
    loss = np.mean(d * d)
    dZ = (2.0 * d / B)[:, None]
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        if l + 1 < len(layers):
            dZ = dZ * gelu_d(cache[l + 1][0])
        A_prev = cache[l][1]
        grads[l] = (dZ.T @ A_prev, dZ.sum(0))
        dZ = dZ @ W
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat
