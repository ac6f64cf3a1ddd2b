"""CPU oracle of the learned preconditioner -- TEST INFRASTRUCTURE ONLY.

Imported by tests/ (and bench.py's CPU legs) to check libab2's GNN kernels
(alien_b200/csrc/gnn.cu); never by the product.  No reference counterpart:
Alien has no learned preconditioner, so this file defines the network and is
checked against finite differences of itself (float64) and against the GPU
(BF16 operands, FP32 accumulation) within BF16 tolerances.

Network (a message-passing network on the matrix graph, weights shared over
nodes).  It works on the symmetrically diagonal-scaled system
D^-1/2 A D^-1/2 (unit diagonal), so that neither its inputs nor its outputs
carry the coefficients' orders of magnitude:
  d_i    = sqrt(a_ii)
  t_i    = r_i / d_i,  s = sqrt(mean(t^2))       scaled residual and its scale
  x0_i   = [t_i / s, log(a_ii) / 10]            node features
  e_ij   = log|a_ij| - (log a_ii + log a_jj)/2  edge features (off-diagonal entries)
  h1     = relu(W0 x0 + b0)                     W0: 64 x 2
  layer l = 1..4:
    g_ij = sigmoid(u_l e_ij + c_l)              edge gate
    m_i  = sum_j g_ij h_l[j]                    aggregation over the row's neighbours
    h_l+1 = relu(W_l [h_l ; m] + b_l)           W_l: 64 x 128 (tensor cores on the GPU)
  y_i    = w_d . h5_i + b_d + w_s x0_i[0]       w_s: linear skip of the scaled residual
  z_i    = s * y_i / d_i                        z = M(r), the preconditioned residual
With w_d = 0, b_d = 0 and w_s = 1 the network is exactly Jacobi (z = r / a_ii);
the initialisation starts close to that and training learns the correction.
Loss for a (residual r, error e) pair: L = (z - e)^T A (z - e) / (e^T A e).

`bf16=True` rounds what the GPU rounds: the dense layers' weights and inputs
[h ; m], the aggregation's gates and the stored activations,
round-to-nearest-even (the backward pass treats the roundings as identity).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

H = 64
LAYERS = 4


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


@dataclass
class Params:
    W0: np.ndarray            # 64 x 2
    b0: np.ndarray            # 64
    W: list                   # LAYERS x (64 x 128)
    b: list                   # LAYERS x 64
    u: np.ndarray             # LAYERS
    c: np.ndarray             # LAYERS
    wd: np.ndarray            # 64
    bd: float = 0.0
    ws: float = 1.0

    def copy(self) -> "Params":
        return Params(self.W0.copy(), self.b0.copy(), [w.copy() for w in self.W], [v.copy() for v in self.b],
                      self.u.copy(), self.c.copy(), self.wd.copy(), float(self.bd), float(self.ws))

    def flat(self) -> np.ndarray:
        return np.concatenate([self.W0.ravel(), self.b0, *[w.ravel() for w in self.W], *self.b, self.u, self.c,
                               self.wd, [self.bd, self.ws]]).astype(np.float64)

    @staticmethod
    def unflat(v: np.ndarray) -> "Params":
        v = np.asarray(v, dtype=np.float64)
        o = 0

        def take(k, shape=None):
            nonlocal o
            a = v[o:o + k]
            o += k
            return a.reshape(shape) if shape else a

        W0 = take(2 * H, (H, 2))
        b0 = take(H)
        W = [take(H * 2 * H, (H, 2 * H)) for _ in range(LAYERS)]
        b = [take(H) for _ in range(LAYERS)]
        u = take(LAYERS)
        c = take(LAYERS)
        wd = take(H)
        bd = float(take(1)[0])
        ws = float(take(1)[0])
        return Params(W0, b0, W, b, u, c, wd, bd, ws)


def init_params(seed: int = 0, wd_scale: float = 1.0) -> Params:
    """He-style initialisation, seeded; w_s = 1 (the Jacobi skip)."""
    rng = np.random.default_rng(seed)
    W0 = rng.normal(0, np.sqrt(2 / 2), (H, 2)).astype(np.float32)
    W = [rng.normal(0, np.sqrt(2 / (2 * H)), (H, 2 * H)).astype(np.float32) for _ in range(LAYERS)]
    return Params(W0, np.zeros(H, np.float32), W, [np.full(H, 0.01, np.float32) for _ in range(LAYERS)],
                  np.full(LAYERS, 0.5, np.float32), np.zeros(LAYERS, np.float32),
                  (wd_scale * rng.normal(0, np.sqrt(1 / H), H)).astype(np.float32), 0.0, 1.0)


@dataclass
class Graph:
    """What the network reads from the matrix."""
    n: int
    rp: np.ndarray
    ci: np.ndarray
    vals: np.ndarray
    diag: np.ndarray
    edge_row: np.ndarray      # row of each off-diagonal entry
    edge_col: np.ndarray
    edge_feat: np.ndarray     # log|a_ij| - (log a_ii + log a_jj) / 2

    @staticmethod
    def from_csr(rp, ci, vals) -> "Graph":
        n = len(rp) - 1
        rows = np.repeat(np.arange(n), np.diff(rp))
        diag = np.zeros(n)
        on = ci == rows
        diag[rows[on]] = vals[on]
        off = ~on
        er, ec = rows[off], ci[off]
        ef = np.log(np.abs(vals[off])) - 0.5 * (np.log(diag[er]) + np.log(diag[ec]))
        return Graph(n, np.asarray(rp), np.asarray(ci), np.asarray(vals, np.float64), diag, er, ec, ef)

    def matvec(self, x):
        y = np.zeros(self.n)
        rows = np.repeat(np.arange(self.n), np.diff(self.rp))
        np.add.at(y, rows, self.vals * x[self.ci])
        return y


def _sig(t):
    return 1.0 / (1.0 + np.exp(-t))


def forward(p: Params, G: Graph, r: np.ndarray, bf16_round: bool = False):
    """Returns z and the activations the backward pass needs."""
    rd = (lambda a: bf16(a).astype(np.float64)) if bf16_round else (lambda a: np.asarray(a, np.float64))
    r = np.asarray(r, np.float64)
    sd = np.sqrt(G.diag)
    t = r / sd
    s = float(np.sqrt(np.mean(t * t)))
    x0 = np.stack([t / s if s > 0 else np.zeros_like(t), np.log(G.diag) / 10.0], axis=1)
    pre0 = x0 @ p.W0.astype(np.float64).T + p.b0
    h = rd(np.maximum(pre0, 0.0))
    cache = {"s": s, "x0": x0, "pre0": pre0, "h": [h], "m": [], "pre": [], "g": []}
    for l in range(LAYERS):
        g = _sig(float(p.u[l]) * G.edge_feat + float(p.c[l]))
        gm = rd(g) if bf16_round else g  # the GPU's aggregation is a BF16 x BF16 -> FP32 tensor-core product
        m = np.zeros((G.n, H))
        np.add.at(m, G.edge_row, gm[:, None] * h[G.edge_col])
        m = rd(m)
        inp = np.concatenate([h, m], axis=1)
        pre = inp @ rd(p.W[l]).T + p.b[l]
        h = rd(np.maximum(pre, 0.0))
        cache["m"].append(m)
        cache["pre"].append(pre)
        cache["g"].append(g)
        cache["h"].append(h)
    y = h @ p.wd.astype(np.float64) + p.bd + p.ws * x0[:, 0]
    z = s * y / sd
    return z, cache


def loss(p: Params, G: Graph, r, e, bf16_round: bool = False) -> float:
    z, _ = forward(p, G, r, bf16_round)
    d = z - e
    return float(d @ G.matvec(d) / (e @ G.matvec(e)))


def backward(p: Params, G: Graph, r, e, bf16_round: bool = False):
    """Loss and its gradient (a Params of gradients)."""
    z, C = forward(p, G, r, bf16_round)
    Ae = G.matvec(e)
    eAe = float(e @ Ae)
    d = z - e
    Ad = G.matvec(d)
    L = float(d @ Ad) / eAe
    dz = 2.0 * Ad / eAe
    s = C["s"]
    dy = dz * s / np.sqrt(G.diag)
    h5 = C["h"][-1]
    gwd = h5.T @ dy
    gbd = float(dy.sum())
    gws = float(dy @ C["x0"][:, 0])
    dh = np.outer(dy, p.wd.astype(np.float64))
    gW, gb, gu, gc = [None] * LAYERS, [None] * LAYERS, np.zeros(LAYERS), np.zeros(LAYERS)
    for l in reversed(range(LAYERS)):
        pre = C["pre"][l]
        h_in, m, g = C["h"][l], C["m"][l], C["g"][l]
        dpre = dh * (pre > 0)
        inp = np.concatenate([h_in, m], axis=1)
        Wl = bf16(p.W[l]).astype(np.float64) if bf16_round else p.W[l].astype(np.float64)
        gW[l] = dpre.T @ inp
        gb[l] = dpre.sum(axis=0)
        dinp = dpre @ Wl
        dh_in, dm = dinp[:, :H], dinp[:, H:]
        dh_new = dh_in.copy()
        np.add.at(dh_new, G.edge_col, g[:, None] * dm[G.edge_row])
        dg = np.sum(dm[G.edge_row] * h_in[G.edge_col], axis=1)
        ds = dg * g * (1 - g)
        gu[l] = float(ds @ G.edge_feat)
        gc[l] = float(ds.sum())
        dh = dh_new
    dpre0 = dh * (C["pre0"] > 0)
    gW0 = dpre0.T @ C["x0"]
    gb0 = dpre0.sum(axis=0)
    return L, Params(gW0, gb0, gW, gb, gu, gc, gwd, gbd, gws)
