"""Test infrastructure (oracle only): CPU restatement of the learned surrogate.

The reference (Uph) has no learned component; the message-passing network is
this project's addition, so this file is its specification.  It restates in
numpy float64 exactly what the GPU kernels compute:

* the neighbour graph: every node's partners within the radius R
  (DBL_EPSILON < r^2 < R^2, r^2 = dx*dx + dy*dy in double -- the pair
  predicate of the SPH search), sorted by node index (the GPU keeps its
  cell-list order, which changes only the order of FP32 sums);
* node features, edge features e_ij = ((x_j - x_i)/R, (y_j - y_i)/R, r/R,
  (rho_j - rho_i)/rho_unit) in FP32;
* the network (latent width 128, `rounds` message-passing rounds):
      h0   = Enc2 relu(Enc1 f + b) + b
      per round:
        [P | Q] = W_pq h + b_pq                              (128 -> 256)
        s_i  = sum_j relu(P_i + Q_j + W_e e_ij)              (edge MLP layer 1)
        m_i  = W_2 s_i                                       (edge MLP layer 2,
                                                              summed over j)
        h   <- h + N2 relu(N1 [h ; m] + b) + b               (node MLP, residual)
      out  = Dec2 relu(Dec1 h + b) + b                        (first 5 columns used)
  The message MLP is the 2-layer MLP relu(W_a h_i + W_b h_j + W_e e_ij + b)
  -> W_2, summed over partners; its second layer is linear, so the sum moves
  inside (sum_j W_2 r_ij = W_2 sum_j r_ij) and its first layer splits into
  per-node products P = W_a h, Q = W_b h.  Exact, not an approximation.
* the loss (mean squared error over the fluid rows' 5 outputs) and the
  backward pass of all of the above.

With ``emulate=True`` every value the GPU stores in BF16 is rounded to BF16
here at the same place (round to nearest even of the FP32 value) -- the
activations, the residual stream h after every residual add, P, Q, S, m --
and everything else is float64.  With ``emulate=False`` the whole network is float64 -- the
form the finite-difference check pins.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""
from __future__ import annotations

import math

import numpy as np

LATENT = 128
FEAT = 128      # input feature width (6 used, zero padded for the tensor-core K granule)
OUT_PAD = 128   # decoder output width (NOUT used)
NOUT = 5        # dx, dy, du, dv, drho increments (normalised)
NFEAT_USED = 6
DBL_EPSILON = np.finfo(np.float64).eps


# ---- parameter layout (offsets in floats; every block a multiple of 128) -----
def layout(rounds: int = 3):
    """[(name, shape)] in storage order; matrices are [out x in] row-major."""
    L = [("enc1.w", (LATENT, FEAT)), ("enc1.b", (LATENT,)), ("enc2.w", (LATENT, LATENT)), ("enc2.b", (LATENT,))]
    for r in range(rounds):
        L += [(f"r{r}.pq.w", (2 * LATENT, LATENT)), (f"r{r}.pq.b", (2 * LATENT,)), (f"r{r}.we", (LATENT, 4)),
              (f"r{r}.w2", (LATENT, LATENT)), (f"r{r}.n1.w", (LATENT, 2 * LATENT)), (f"r{r}.n1.b", (LATENT,)),
              (f"r{r}.n2.w", (LATENT, LATENT)), (f"r{r}.n2.b", (LATENT,))]
    L += [("dec1.w", (LATENT, LATENT)), ("dec1.b", (LATENT,)), ("dec2.w", (OUT_PAD, LATENT)), ("dec2.b", (OUT_PAD,))]
    return L


def offsets(rounds: int = 3):
    off, o = {}, 0
    for name, shape in layout(rounds):
        off[name] = (o, shape)
        o += int(np.prod(shape))
    return off, o


def unpack(flat: np.ndarray, rounds: int = 3) -> dict:
    off, _ = offsets(rounds)
    return {k: flat[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in off.items()}


# ---- rounding -------------------------------------------------------------
def bf16(x) -> np.ndarray:
    """Round to BF16 (nearest even) through FP32, returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float64).astype(np.float32))
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


# ---- graph and features --------------------------------------------------------
class Graph:
    """CSR neighbour lists (receiver-major, partners ascending) + edge features."""

    def __init__(self, x: np.ndarray, y: np.ndarray, radius: float, rho=None, rho_unit: float = 0.1):
        n = x.shape[0]
        r2cut = radius * radius
        indptr = [0]
        indices = []
        # cell binning keeps this O(n) for the test sizes
        cell = radius
        cx = np.floor((x - x.min()) / cell).astype(np.int64)
        cy = np.floor((y - y.min()) / cell).astype(np.int64)
        bins = {}
        for i in range(n):
            bins.setdefault((cx[i], cy[i]), []).append(i)
        for i in range(n):
            cand = []
            for ox in (-1, 0, 1):
                for oy in (-1, 0, 1):
                    cand.extend(bins.get((cx[i] + ox, cy[i] + oy), ()))
            cand = np.array(sorted(cand), dtype=np.int64)
            dx = x[cand] - x[i]
            dy = y[cand] - y[i]
            r2 = dx * dx + dy * dy
            keep = cand[(r2 > DBL_EPSILON) & (r2 < r2cut)]
            indices.extend(keep.tolist())
            indptr.append(len(indices))
        self.n = n
        self.indptr = np.array(indptr, np.int64)
        self.indices = np.array(indices, np.int64)
        self.recv = np.repeat(np.arange(n), np.diff(self.indptr))
        self.send = self.indices
        dx = x[self.send] - x[self.recv]
        dy = y[self.send] - y[self.recv]
        r = np.sqrt(dx * dx + dy * dy)
        dr = np.zeros_like(dx) if rho is None else (rho[self.send] - rho[self.recv]) / rho_unit
        self.e = np.stack([dx / radius, dy / radius, r / radius, dr], axis=1).astype(np.float32).astype(np.float64)

    def degree(self) -> np.ndarray:
        return np.diff(self.indptr)


def node_features(u, v, rho, itype, vel_scale: float, rho0: float, rho_scale: float) -> np.ndarray:
    """f = [u/U, v/U, (rho/rho0 - 1)/s_rho, fluid, fixed wall, moving wall, 0...]
    (itype 1 fluid, 3 moving boundary, anything else fixed), FP32 then BF16."""
    n = u.shape[0]
    F = np.zeros((n, FEAT), np.float64)
    F[:, 0] = np.float32(u / vel_scale)
    F[:, 1] = np.float32(v / vel_scale)
    F[:, 2] = np.float32((rho / rho0 - 1.0) / rho_scale)
    F[:, 3] = itype == 1
    F[:, 5] = itype == 3
    F[:, 4] = (itype != 1) & (itype != 3)
    return bf16(F)


def _segsum(vals: np.ndarray, idx: np.ndarray, n: int) -> np.ndarray:
    out = np.zeros((n,) + vals.shape[1:], np.float64)
    np.add.at(out, idx, vals)
    return out


# ---- network ------------------------------------------------------------------
def forward(flat: np.ndarray, F: np.ndarray, g: Graph, rounds: int = 3, emulate: bool = True):
    """Returns (out [n x 128], cache for backward)."""
    W = unpack(np.asarray(flat, np.float64), rounds)
    rb = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    Wm = {k: (rb(v) if (v.ndim == 2 and not k.endswith(".we")) else v) for k, v in W.items()}
    c = {"F": F}
    a1 = rb(np.maximum(F @ Wm["enc1.w"].T + W["enc1.b"], 0.0))
    h = rb(a1 @ Wm["enc2.w"].T + W["enc2.b"])
    c["a1"] = a1
    c["rounds"] = []
    for r in range(rounds):
        hb = rb(h)
        PQ = rb(hb @ Wm[f"r{r}.pq.w"].T + W[f"r{r}.pq.b"])
        P, Q = PQ[:, :LATENT], PQ[:, LATENT:]
        we = W[f"r{r}.we"]
        z = P[g.recv] + Q[g.send] + g.e @ we.T
        S = rb(_segsum(np.maximum(z, 0.0), g.recv, g.n))
        m = rb(S @ Wm[f"r{r}.w2"].T)
        cat = np.concatenate([hb, m], axis=1)
        u = rb(np.maximum(cat @ Wm[f"r{r}.n1.w"].T + W[f"r{r}.n1.b"], 0.0))
        h = rb(h + (u @ Wm[f"r{r}.n2.w"].T + W[f"r{r}.n2.b"]))
        c["rounds"].append(dict(hb=hb, PQ=PQ, z=z, S=S, m=m, cat=cat, u=u))
    hb = rb(h)
    d1 = rb(np.maximum(hb @ Wm["dec1.w"].T + W["dec1.b"], 0.0))
    out = d1 @ Wm["dec2.w"].T + W["dec2.b"]
    c.update(h3b=hb, d1=d1, Wm=Wm, W=W, g=g, emulate=emulate, rounds_n=rounds)
    return out, c


def loss_and_grad(out: np.ndarray, target: np.ndarray, n_fluid: int):
    """Mean squared error over rows [0, n_fluid) and the first NOUT columns."""
    d = out[:n_fluid, :NOUT] - target
    count = n_fluid * NOUT
    loss = float(np.sum(d * d) / count)
    dout = np.zeros_like(out)
    dout[:n_fluid, :NOUT] = 2.0 * d / count
    return loss, dout


def backward(c: dict, dout: np.ndarray) -> np.ndarray:
    """Gradient of the loss w.r.t. the flat parameter vector (float64)."""
    rounds = c["rounds_n"]
    W, Wm, g = c["W"], c["Wm"], c["g"]
    rb = bf16 if c["emulate"] else (lambda a: np.asarray(a, np.float64))
    G = {k: np.zeros_like(v, dtype=np.float64) for k, v in W.items()}
    dO = rb(dout)
    G["dec2.w"] = dO.T @ c["d1"]
    G["dec2.b"] = dO.sum(0)
    dz = rb((dO @ Wm["dec2.w"]) * (c["d1"] > 0))
    G["dec1.w"] = dz.T @ c["h3b"]
    G["dec1.b"] = dz.sum(0)
    dh = dz @ Wm["dec1.w"]
    for r in reversed(range(rounds)):
        R = c["rounds"][r]
        dhb = rb(dh)
        G[f"r{r}.n2.w"] = dhb.T @ R["u"]
        G[f"r{r}.n2.b"] = dhb.sum(0)
        dz = rb((dhb @ Wm[f"r{r}.n2.w"]) * (R["u"] > 0))
        G[f"r{r}.n1.w"] = dz.T @ R["cat"]
        G[f"r{r}.n1.b"] = dz.sum(0)
        dh = dh + dz @ Wm[f"r{r}.n1.w"][:, :LATENT]
        dm = rb(dz @ Wm[f"r{r}.n1.w"][:, LATENT:])
        G[f"r{r}.w2"] = dm.T @ R["S"]
        dS = dm @ Wm[f"r{r}.w2"]
        dze = dS[g.recv] * (R["z"] > 0)
        dP = _segsum(dze, g.recv, g.n)
        dQ = _segsum(dze, g.send, g.n)
        G[f"r{r}.we"] = dze.T @ g.e
        dPQ = rb(np.concatenate([dP, dQ], axis=1))
        G[f"r{r}.pq.w"] = dPQ.T @ R["hb"]
        G[f"r{r}.pq.b"] = dPQ.sum(0)
        dh = dh + dPQ @ Wm[f"r{r}.pq.w"]
    dhb = rb(dh)
    G["enc2.w"] = dhb.T @ c["a1"]
    G["enc2.b"] = dhb.sum(0)
    dz = rb((dhb @ Wm["enc2.w"]) * (c["a1"] > 0))
    G["enc1.w"] = dz.T @ c["F"]
    G["enc1.b"] = dz.sum(0)
    off, total = offsets(rounds)
    flat = np.zeros(total, np.float64)
    for k, (o, s) in off.items():
        flat[o:o + int(np.prod(s))] = G[k].ravel()
    return flat


def loss_of(flat, F, g, target, n_fluid, rounds=3, emulate=False) -> float:
    out, _ = forward(flat, F, g, rounds, emulate)
    return loss_and_grad(out, target, n_fluid)[0]
