"""The NumPy restatement of the learned-guess network (oracle/mlp_ref.py):
BF16 rounding on known values, and its analytic gradient against central
finite differences in float64 (the pin of the oracle that the GPU training
kernels are checked against)."""
import numpy as np

from oracle import mlp_ref as M


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0**-8, 1.0 + 3 * 2.0**-8, -2.5, 1.0 + 2.0**-7, 3.0e38, 0.0], dtype=np.float32)
    want = np.array([1.0, 1.0, 1.0 + 2.0**-6, -2.5, 1.0 + 2.0**-7, 2.9983e38, 0.0], dtype=np.float32)
    got = M.bf16(x)
    assert np.array_equal(got[:5], want[:5])
    assert got[6] == 0.0
    assert abs(got[5] / 3.0e38 - 1) < 2.0**-8


def test_blob_layout():
    assert M.NW == 5548
    assert (M.OFF_W1, M.OFF_B3) == (40, 5544)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    w = M.random_blob(7).astype(np.float64)
    x = rng.standard_normal((9, M.IN))
    t = rng.standard_normal((9, M.OUT))
    loss, g = M.loss_grad(w, x, t, exact=True)
    assert np.all(g[:M.OFF_W1] == 0.0)
    picks = np.concatenate([rng.integers(M.OFF_W1, M.NW, 60), [M.OFF_B1, M.OFF_B2 + 5, M.OFF_B3 + 3]])
    h = 1e-6
    for e in picks:
        wp, wm = w.copy(), w.copy()
        wp[e] += h
        wm[e] -= h
        fd = (M.loss_grad(wp, x, t, exact=True)[0] - M.loss_grad(wm, x, t, exact=True)[0]) / (2 * h)
        assert abs(fd - g[e]) <= 1e-6 * max(1.0, abs(g[e])), (e, fd, g[e])


def test_bf16_forward_close_to_exact():
    rng = np.random.default_rng(4)
    w = M.random_blob(8)
    x = rng.standard_normal((256, M.IN))
    y_b, _ = M.forward(w, x)
    y_e, _ = M.forward(w, x, exact=True)
    assert np.abs(y_b - y_e).max() < 0.05 * np.abs(y_e).max()
