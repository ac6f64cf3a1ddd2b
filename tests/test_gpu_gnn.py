"""The learned preconditioner on the GPU vs its CPU oracle.

Forward and backward of libab2's kernels (BF16 tensor-core dense layers with
FP32 accumulation, BF16 activations) against oracle/gnn_oracle.py evaluated
with the same BF16 roundings and float64 accumulation: the network output and
every gradient block agree to BF16 accuracy.  Training on the GPU reduces the
loss; flexible CG with the network converges, with ILU(0) taking over when
the network's steps stall.
"""
import numpy as np
import pytest

from alien_b200 import abi
from oracle import gnn_oracle as G

pytestmark = pytest.mark.gpu


def blocks(v):
    off = [0, 128, 192, 192 + 4 * 8192, 192 + 4 * 8192 + 256, 192 + 4 * 8192 + 260, 192 + 4 * 8192 + 264,
           192 + 4 * 8192 + 328, 192 + 4 * 8192 + 329, v.size]
    names = ["W0", "b0", "W", "b", "u", "c", "wd", "bd", "ws"]
    return {nm: v[a:b] for nm, a, b in zip(names, off[:-1], off[1:])}


@pytest.fixture(scope="module")
def system():
    P = abi.diffusion(12, 11, 10, sigma=1.5, smooth=2.0, seed=4)
    rng = np.random.default_rng(1)
    return P, rng.normal(size=P.n), rng.normal(size=P.n)


@pytest.mark.parametrize("layer", ["grid", "gather"])
def test_forward_matches_oracle(ctx, system, layer):
    P, r, _ = system
    p = G.init_params(2)
    net = abi.Gnn(ctx, p.flat().astype(np.float32))
    net.set_layer(layer)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    net.bind(A)
    assert net.layer == layer
    vr, vz = ctx.vector(r), ctx.vector(P.n)
    net.apply(vr, vz)
    z = vz.download()
    zo, _ = G.forward(p, G.Graph.from_csr(P.row_ptr, P.cols, P.vals), r, bf16_round=True)
    assert np.linalg.norm(z - zo) / np.linalg.norm(zo) < 2e-2
    assert np.all(np.isfinite(z))


def test_jacobi_skip_alone_is_jacobi(ctx, system):
    """With the decoder's hidden weights and bias zero and the skip 1, the
    network is z = r / a_ii (the scaled residual passes through FP32)."""
    P, r, _ = system
    p = G.init_params(2)
    p.wd[:] = 0.0
    p.bd, p.ws = 0.0, 1.0
    net = abi.Gnn(ctx, p.flat().astype(np.float32))
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    net.bind(A)
    vr, vz = ctx.vector(r), ctx.vector(P.n)
    net.apply(vr, vz)
    d = G.Graph.from_csr(P.row_ptr, P.cols, P.vals).diag
    np.testing.assert_allclose(vz.download(), r / d, rtol=1e-6, atol=0)


@pytest.mark.parametrize("layer", ["grid", "gather"])
def test_gradient_matches_oracle(ctx, system, layer):
    P, r, e = system
    p = G.init_params(3)
    net = abi.Gnn(ctx, p.flat().astype(np.float32))
    net.set_layer(layer)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    net.bind(A)
    L, g = net.loss_grad(ctx.vector(r), ctx.vector(e))
    Lo, go = G.backward(p, G.Graph.from_csr(P.row_ptr, P.cols, P.vals), r, e, bf16_round=True)
    assert abs(L - Lo) <= 2e-2 * abs(Lo)
    gb, gob = blocks(g.astype(np.float64)), blocks(go.flat())
    for name in gb:
        a, b = gb[name], gob[name]
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        cos = a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30)
        assert err < 5e-2 and cos > 0.998, (name, err, cos)


@pytest.mark.parametrize("shape", [(12, 11, 10), (40, 36, 30), (128, 3, 3), (3, 3, 257), (5, 4, 3)])
def test_layer_kernels_agree(ctx, shape):
    """The grid layer (bulk-copied neighbour blocks, tcgen05 dense layer) and
    the gather layer (indexed neighbour rows, mma.sync) compute the same
    network: outputs within BF16 rounding of each other on grids with a
    ragged last tile, several tiles a CTA, fewer nodes than one tile, and
    neighbour blocks that start before the first or end after the last
    node."""
    nx, ny, nz = shape
    P = abi.diffusion(nx, ny, nz, sigma=1.5, smooth=2.0, seed=6)
    rng = np.random.default_rng(3)
    r = rng.normal(size=P.n)
    p = G.init_params(4, wd_scale=4.0).flat().astype(np.float32)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    out = {}
    for layer in ("grid", "gather"):
        net = abi.Gnn(ctx, p)
        net.set_layer(layer)
        net.bind(A)
        assert net.layer == layer
        vr, vz = ctx.vector(r), ctx.vector(P.n)
        net.apply(vr, vz)
        out[layer] = vz.download()
        net.close()
    assert np.all(np.isfinite(out["grid"]))
    rel = np.linalg.norm(out["grid"] - out["gather"]) / np.linalg.norm(out["gather"])
    assert rel < 1e-2, rel
    if P.n <= 2000:
        zo, _ = G.forward(G.Params.unflat(p.astype(np.float64)), G.Graph.from_csr(P.row_ptr, P.cols, P.vals), r,
                          bf16_round=True)
        assert np.linalg.norm(out["grid"] - zo) / np.linalg.norm(zo) < 2e-2


def test_layer_kernels_agree_on_gradients(ctx):
    """Training on the grid layer: its forward pass also stores m1..m4 and h5
    for the backward kernels.  On 43,200 nodes (several tiles a CTA) the loss
    and every gradient block agree with the gather layer's to BF16 accuracy."""
    P = abi.diffusion(40, 36, 30, sigma=1.5, smooth=2.0, seed=6)
    rng = np.random.default_rng(9)
    r, e = rng.normal(size=P.n), rng.normal(size=P.n)
    p = G.init_params(5).flat().astype(np.float32)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    out = {}
    for layer in ("grid", "gather"):
        net = abi.Gnn(ctx, p)
        net.set_layer(layer)
        net.bind(A)
        out[layer] = net.loss_grad(ctx.vector(r), ctx.vector(e))
        net.close()
    (Lg, gg), (La, ga) = out["grid"], out["gather"]
    assert np.isfinite(Lg) and abs(Lg - La) <= 1e-2 * abs(La), (Lg, La)
    bg, ba = blocks(gg.astype(np.float64)), blocks(ga.astype(np.float64))
    for name in bg:
        err = np.linalg.norm(bg[name] - ba[name]) / max(np.linalg.norm(ba[name]), 1e-30)
        assert err < 5e-2, (name, err)


def test_grid_layer_needs_a_3d_grid(ctx):
    """On a 2-D grid (no 3-D 7-point profile) AUTO takes the gather layer and
    an explicit grid request is refused."""
    P = abi.diffusion(31, 9, 1, sigma=1.5, smooth=3.0, seed=7)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    net = abi.Gnn(ctx, G.init_params(1).flat().astype(np.float32))
    net.bind(A)
    assert net.layer == "gather"
    net.set_layer("grid")
    with pytest.raises(abi.AB2Error) as e:
        net.bind(A)
    assert e.value.code == abi.AB2_ERR_UNSUPPORTED
    net.close()


def test_training_reduces_loss_and_fcg_converges(ctx):
    """Train on (residual, error) pairs from ILU0-CG iterates of a few seeded
    fields, then solve a held-out field with flexible CG."""
    from alien_b200 import gnn_train

    net = abi.Gnn(ctx, G.init_params(0).flat().astype(np.float32))
    hist = gnn_train.train(ctx, net, fields=6, side=16, steps_per_pair=4, lr=2e-3, seed=10)
    first, last = np.mean(hist[:8]), np.mean(hist[-8:])
    assert last < 0.9 * first, (first, last)
    P = abi.diffusion(16, 16, 16, sigma=1.5, smooth=3.0, seed=999)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    net.bind(A)
    ilu = abi.Precond(ctx, A, "ilu0")
    b = ctx.vector(P.b)
    x = ctx.vector(P.n)
    res = abi.fcg_solve(ctx, A, b, x, gnn=net, fallback=ilu, tol=1e-8, max_iter=2000)
    assert res.succeeded and res.true_residual < 1e-7
    assert res.gnn_steps >= 1
    x2 = ctx.vector(P.n)
    base = abi.fcg_solve(ctx, A, b, x2, gnn=None, fallback=ilu, tol=1e-8, max_iter=2000)
    assert base.succeeded and base.gnn_steps == 0
    # both judged against the plain solver's converged solution (CG + ILU(0) to 1e-13); the
    # coefficients span nine decades, so a 1e-8 residual leaves errors well above 1e-8
    xs = ctx.vector(P.n)
    abi.Solver(ctx, A, solver="cg", precond="ilu0", tol=1e-13, max_iter=5000).solve(b, xs)
    xs = xs.download()
    for v in (x, x2):
        assert np.linalg.norm(v.download() - xs) / np.linalg.norm(xs) < 1e-3


WEIGHTS = __import__("pathlib").Path(__file__).resolve().parents[1] / "alien_b200" / "gnn_weights.npy"


def test_trained_network_gains_over_its_jacobi_path(ctx):
    """What training gains: on a held-out field (not among the training
    seeds), flexible CG with the committed trained network against the same
    network with its learned part removed (decoder weights and bias zero: only
    the Jacobi skip remains, z = r / a_ii) -- fewer iterations to 1e-8.  The
    hybrid with ILU(0) for the step after each failed network step converges
    too; its counts are printed beside ILU(0) alone."""
    from alien_b200 import gnn_train

    trained = np.load(WEIGHTS)
    skip = trained.copy()
    o = 192 + 4 * 8192 + 264  # wd, bd
    skip[o:o + 65] = 0.0
    P = gnn_train.field(48, 5_000_019)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    b = ctx.vector(P.b)
    ilu = abi.Precond(ctx, A, "ilu0")
    res = {}
    for name, w, fb in (("trained", trained, None), ("skip_only", skip, None), ("hybrid", trained, ilu),
                        ("ilu0", None, ilu)):
        net = None
        if w is not None:
            net = abi.Gnn(ctx, w)
            net.bind(A)
        x = ctx.vector(P.n)
        r = abi.fcg_solve(ctx, A, b, x, gnn=net, fallback=fb, tol=1e-8, max_iter=3000)
        assert r.succeeded and r.true_residual < 1e-7, (name, r)
        res[name] = r.iterations
    print("flexible CG iterations, held-out 48^3 field:", res)
    assert res["trained"] <= 0.9 * res["skip_only"], res
