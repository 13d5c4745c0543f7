"""Test infrastructure: the NumPy restatement of the learned-guess network that
the engine's kernels are checked against. It is not part of the engine and
nothing in the engine calls it.

The network has no counterpart in the reference (the reference starts every
implicit solve from its bisection warm start, koral/solve/implicit.zig:944);
it is pinned by a central finite-difference check of `loss_grad` in float64,
so the gradient it gives is the gradient of `forward`.

Blob layout (floats): input mean[16], input std[16], output mean[4], output
std[4], W1[64][16], b1[64], W2[64][64], b2[64], W3[4][64], b3[4], row-major
[out][in]. The forward pass rounds inputs, weights and hidden activations to
BF16 (round to nearest even), as the tensor-core inference does; `exact=True`
turns the rounding off.
"""
import numpy as np

IN, H, OUT = 16, 64, 4
OFF_IMEAN = 0
OFF_ISTD = OFF_IMEAN + IN
OFF_OMEAN = OFF_ISTD + IN
OFF_OSTD = OFF_OMEAN + OUT
OFF_W1 = OFF_OSTD + OUT
OFF_B1 = OFF_W1 + H * IN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + OUT * H
NW = OFF_B3 + OUT


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    return {
        "imean": w[OFF_IMEAN:OFF_ISTD], "istd": w[OFF_ISTD:OFF_OMEAN],
        "omean": w[OFF_OMEAN:OFF_OSTD], "ostd": w[OFF_OSTD:OFF_W1],
        "W1": w[OFF_W1:OFF_B1].reshape(H, IN), "b1": w[OFF_B1:OFF_W2],
        "W2": w[OFF_W2:OFF_B2].reshape(H, H), "b2": w[OFF_B2:OFF_W3],
        "W3": w[OFF_W3:OFF_B3].reshape(OUT, H), "b3": w[OFF_B3:NW],
    }


def _r(x, exact):
    return x if exact else bf16(x.astype(np.float32)).astype(np.float64)


def forward(w, x, exact=False):
    """Standardised features (n x 16) -> (outputs n x 4, hidden activations)."""
    p = unpack(w)
    x = _r(np.asarray(x, dtype=np.float64), exact)
    W1, W2, W3 = (_r(p[k], exact) for k in ("W1", "W2", "W3"))
    h1 = _r(np.maximum(x @ W1.T + p["b1"], 0.0), exact)
    h2 = _r(np.maximum(h1 @ W2.T + p["b2"], 0.0), exact)
    y = h2 @ W3.T + p["b3"]
    return y, (x, h1, h2, W1, W2, W3)


def loss_grad(w, x, t, exact=False):
    """Mean squared error over n x 4 outputs and its gradient with respect to
    the blob (straight through the BF16 rounding of weights and activations;
    the normalisation entries get zero)."""
    y, (xr, h1, h2, W1, W2, W3) = forward(w, x, exact)
    t = np.asarray(t, dtype=np.float64)
    n = y.shape[0]
    e = y - t
    loss = float((e * e).sum() / (n * OUT))
    dy = 2.0 * e / (n * OUT)
    dh2 = (dy @ W3) * (h2 > 0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    g = np.zeros(NW)
    g[OFF_W1:OFF_B1] = (dh1.T @ xr).ravel()
    g[OFF_B1:OFF_W2] = dh1.sum(0)
    g[OFF_W2:OFF_B2] = (dh2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = dh2.sum(0)
    g[OFF_W3:OFF_B3] = (dy.T @ h2).ravel()
    g[OFF_B3:NW] = dy.sum(0)
    return loss, g


def random_blob(seed, scale=1.0):
    """A blob with He-uniform weights, small random biases and unit
    normalisation (for checks)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NW, dtype=np.float32)
    w[OFF_ISTD:OFF_OMEAN] = 1.0
    w[OFF_OSTD:OFF_W1] = 1.0
    for off, rows, cols in ((OFF_W1, H, IN), (OFF_W2, H, H), (OFF_W3, OUT, H)):
        a = np.sqrt(6.0 / cols) * scale
        w[off:off + rows * cols] = rng.uniform(-a, a, rows * cols)
    for off, m in ((OFF_B1, H), (OFF_B2, H), (OFF_B3, OUT)):
        w[off:off + m] = rng.uniform(-0.1, 0.1, m)
    return w


def features_raw(pp, dt, gdet, alpha, gas_start):
    """Raw features of pre-solve primitives (n x 13 in the reference's VELR
    slot order: rho, u, v1-3, entropy, B1-3, E, F1-3)."""
    pp = np.asarray(pp, dtype=np.float64)
    f = np.empty((pp.shape[0], IN))
    f[:, 0] = np.log10(pp[:, 0])
    f[:, 1] = np.log10(pp[:, 1])
    f[:, 2:5] = np.arcsinh(pp[:, 2:5] * 1e3)
    f[:, 5] = np.where(gas_start, 1.0, -1.0)
    f[:, 6:9] = np.arcsinh(pp[:, 6:9] * 1e12)
    f[:, 9] = np.log10(pp[:, 9])
    f[:, 10:13] = np.arcsinh(pp[:, 10:13] * 1e3)
    f[:, 13] = np.log10(dt)
    f[:, 14] = np.log10(gdet)
    f[:, 15] = alpha
    return f
