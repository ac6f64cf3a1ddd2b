"""The learned preconditioner's CPU oracle (oracle/gnn_oracle.py), checked
against itself: its hand-written backward pass equals central finite
differences of its forward pass (float64, no rounding)."""
import numpy as np

from alien_b200 import abi
from oracle import gnn_oracle as G


def test_backward_matches_finite_differences():
    P = abi.diffusion(6, 5, 4, sigma=1.5, smooth=2.0, seed=3)
    g = G.Graph.from_csr(P.row_ptr, P.cols, P.vals)
    p = G.init_params(1)
    rng = np.random.default_rng(0)
    r, e = rng.normal(size=P.n), rng.normal(size=P.n)
    L, grad = G.backward(p, g, r, e)
    assert abs(L - G.loss(p, g, r, e)) < 1e-12
    v, gv = p.flat(), grad.flat()
    scale = np.max(np.abs(gv))
    off = {"W0": 0, "b0": 128, "W": 192, "b": 192 + 4 * 8192, "u": 192 + 4 * 8192 + 256}
    idx = list(rng.choice(v.size, 60, replace=False)) + [off["u"], off["u"] + 3, off["u"] + 4, v.size - 2, v.size - 1, 5, 130]
    eps = 1e-6
    for k in idx:
        vp, vm = v.copy(), v.copy()
        vp[k] += eps
        vm[k] -= eps
        fd = (G.loss(G.Params.unflat(vp), g, r, e) - G.loss(G.Params.unflat(vm), g, r, e)) / (2 * eps)
        assert abs(fd - gv[k]) <= 1e-6 * scale + 1e-4 * abs(fd), (k, fd, gv[k])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0, 0.0], dtype=np.float32)
    assert np.array_equal(G.bf16(x), np.array([1.0, 1.0, 1.0078125, -3.0, 0.0], dtype=np.float32))


def test_skip_alone_is_jacobi_and_scaling_invariant():
    """w_d = 0, b_d = 0, w_s = 1 gives z = r / a_ii exactly; and the network
    output is equivariant under a positive scaling of the residual."""
    P = abi.diffusion(5, 4, 3, sigma=1.5, smooth=2.0, seed=5)
    g = G.Graph.from_csr(P.row_ptr, P.cols, P.vals)
    r = np.random.default_rng(1).normal(size=P.n)
    p = G.init_params(0)
    z, _ = G.forward(p, g, r)
    z2, _ = G.forward(p, g, 1e6 * r)
    np.testing.assert_allclose(z2, 1e6 * z, rtol=1e-12)
    p.wd[:] = 0.0
    p.bd, p.ws = 0.0, 1.0
    z, _ = G.forward(p, g, r)
    np.testing.assert_allclose(z, r / g.diag, rtol=1e-14)
