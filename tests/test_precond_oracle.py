"""CPU checks of the preconditioner oracle (oracle/net_oracle.py): its network
gradient against finite differences, and the TPA factor's limits."""
import numpy as np

from oracle import net_oracle as N


def test_network_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    shape = (4, 5, 6)
    NL = int(np.prod(shape))
    gs = [rng.standard_normal(NL) + 1j * rng.standard_normal(NL) for _ in range(2)]
    ts = [rng.standard_normal(NL) + 1j * rng.standard_normal(NL) for _ in range(2)]
    w = N.identity_weights(noise=0.1, seed=1).astype(np.float64)
    loss, grad = N.loss_grad(gs, ts, shape, w, emulate_bf16=False)
    for idx in rng.choice(N.NET_NW, 25, replace=False):
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[idx] += h
        wm[idx] -= h
        fd = (N.loss_grad(gs, ts, shape, wp, False)[0] - N.loss_grad(gs, ts, shape, wm, False)[0]) / (2 * h)
        assert abs(fd - grad[idx]) <= 1e-6 * max(1.0, abs(fd)), (idx, fd, grad[idx])


def test_identity_weights_reproduce_the_input():
    rng = np.random.default_rng(4)
    shape = (4, 4, 6)
    g = rng.standard_normal(96) + 1j * rng.standard_normal(96)
    out = N.forward(g, shape, N.identity_weights(), emulate_bf16=False)[0]
    np.testing.assert_allclose(out, g, rtol=1e-12, atol=1e-12)


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159265, 65504.0], np.float32)
    r = N.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125   # ties to even, then up
    assert abs(r[3] - (-3.140625)) < 1e-7


def test_tpa_factor_limits():
    assert abs(N.tpa_factor(0.0) - 1.0) < 1e-15
    x = np.array([10.0, 100.0])
    np.testing.assert_allclose(N.tpa_factor(x), 8 * x ** 3 / (16 * x ** 4), rtol=0.2)   # ~ 1/(2x) for large x
