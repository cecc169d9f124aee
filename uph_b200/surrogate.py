"""The learned surrogate (include/uph_surrogate.h) from Python.

A message-passing network over the SPH neighbour graph (radius R = 2h)
predicts how the fluid state changes over one macro step of `macro_steps`
SPH steps.  It is trained on the GPU, by the library's own BF16 tensor-core
forward and backward kernels and Adam, on pairs of states the plain solver
produces; `Surrogate.advance` then steps a simulation with it, re-running the
plain solver every `judge_every`-th macro step as the judge of its density
and free-surface error and handing control back to the plain solver for
`fallback_macro` macro steps whenever a threshold is exceeded.

Training data comes from batches of wave flumes (the workload's geometry,
shortened): flumes stacked in y in one simulation, each with its own piston
amplitude and period (per-particle wall motion), advanced by the plain WCSPH
solver; states are recorded in windows of consecutive macro steps after a
warm-up.  Device memory and random numbers for the training loop are torch
tensors; every network computation is the library's.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from . import deck as D
from ._capi import PREC_FP32_PAIR, PROFILE_WCSPH, SurConfig, SurJudge, SurNodes, SurReport

LATENT = 128
FEAT = 128
OUT_PAD = 128
NOUT = 5
NFEAT_USED = 6
OUTPUT_NAMES = ("dx", "dy", "du", "dv", "drho")


# ---- parameters ------------------------------------------------------------------
def param_layout(rounds: int = 3) -> List[Tuple[str, Tuple[int, ...]]]:
    """Storage order of the flat FP32 parameter vector (matrices [out x in])."""
    L = [("enc1.w", (LATENT, FEAT)), ("enc1.b", (LATENT,)), ("enc2.w", (LATENT, LATENT)), ("enc2.b", (LATENT,))]
    for r in range(rounds):
        L += [(f"r{r}.pq.w", (2 * LATENT, LATENT)), (f"r{r}.pq.b", (2 * LATENT,)), (f"r{r}.we", (LATENT, 4)),
              (f"r{r}.w2", (LATENT, LATENT)), (f"r{r}.n1.w", (LATENT, 2 * LATENT)), (f"r{r}.n1.b", (LATENT,)),
              (f"r{r}.n2.w", (LATENT, LATENT)), (f"r{r}.n2.b", (LATENT,))]
    L += [("dec1.w", (LATENT, LATENT)), ("dec1.b", (LATENT,)), ("dec2.w", (OUT_PAD, LATENT)), ("dec2.b", (OUT_PAD,))]
    return L


def init_params(seed: int, rounds: int = 3) -> np.ndarray:
    """Uniform(+-1/sqrt(fan_in)) weights and zero biases; the residual and
    output layers start 10x smaller, W_e's density-difference column at zero.
    Entries no input or output reaches (the padded feature columns, decoder
    rows past the 5 outputs) are zero and stay zero under training (their
    gradient is 0)."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in param_layout(rounds):
        if name.endswith(".b"):
            parts.append(np.zeros(shape, np.float32))
            continue
        fan_in = {"enc1.w": NFEAT_USED}.get(name, 4 if name.endswith(".we") else shape[1])
        bound = 1.0 / math.sqrt(fan_in)
        w = rng.uniform(-bound, bound, size=shape)
        if name.endswith(".n2.w") or name == "dec2.w":
            w *= 0.1
        if name.endswith(".we"):
            w[:, 3] = 0.0  # the density-difference feature starts unused
        if name == "enc1.w":
            w[:, NFEAT_USED:] = 0.0
        if name == "dec2.w":
            w[NOUT:, :] = 0.0
        parts.append(w.astype(np.float32))
    return np.concatenate([p.ravel() for p in parts])


@dataclasses.dataclass
class NetConfig:
    rounds: int = 3
    macro_steps: int = 40
    radius: float = 0.0        # 2h
    dt: float = 0.0
    rho0: float = 1000.0
    vel_scale: float = 0.1     # m/s
    rho_scale: float = 0.01    # relative density
    edge_rho_scale: float = 1e-3  # unit of the edge density difference, relative to rho0
    out_scale: Tuple[float, ...] = (1e-4, 1e-4, 1e-3, 1e-3, 1.0)

    @classmethod
    def for_params(cls, uph_params: dict, macro_steps: int, **kw) -> "NetConfig":
        """Radius 2h, dt and rho0 of a simulation (Deck.uph_params())."""
        return cls(macro_steps=macro_steps, radius=2.0 * uph_params["h"], dt=uph_params["time_step"],
                   rho0=uph_params["density0"], **kw)

    def c_struct(self) -> SurConfig:
        c = SurConfig()
        c.rounds = self.rounds
        c.macro_steps = self.macro_steps
        c.radius = self.radius
        c.dt = self.dt
        c.rho0 = self.rho0
        c.vel_scale = self.vel_scale
        c.rho_scale = self.rho_scale
        c.edge_rho_scale = self.edge_rho_scale
        for k in range(NOUT):
            c.out_scale[k] = float(self.out_scale[k])
        return c


@dataclasses.dataclass
class Judge:
    depth: float
    surface_x0: float
    surface_x1: float
    surface_bins: int = 100
    judge_every: int = 10
    fallback_macro: int = 10
    max_rho_err: float = 0.01
    max_surface_err: float = 0.02

    def c_struct(self) -> SurJudge:
        j = SurJudge()
        for f, _ in SurJudge._fields_:
            setattr(j, f, getattr(self, f))
        return j


class Nodes:
    """One graph's node arrays on the GPU (torch: float64 x, y, u, v, rho and
    int32 itype), fluid nodes first, and a box containing them."""

    def __init__(self, x, y, u, v, rho, itype, n_fluid: int, box: Tuple[float, float, float, float]):
        self.x, self.y, self.u, self.v, self.rho, self.itype = x, y, u, v, rho, itype
        self.n = int(x.shape[0])
        self.n_fluid = int(n_fluid)
        self.box = box

    @classmethod
    def from_state(cls, st: Dict[str, np.ndarray], n_fluid: int, box, device="cuda") -> "Nodes":
        import torch
        t = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=device)
        return cls(t(st["Position"][:, 0]), t(st["Position"][:, 1]), t(st["Velocity"][:, 0]),
                   t(st["Velocity"][:, 1]), t(st["density"]), t(st["itype"], torch.int32), n_fluid, box)

    def c_struct(self) -> SurNodes:
        s = SurNodes()
        s.n = self.n
        s.n_fluid = self.n_fluid
        for k in ("x", "y", "u", "v", "rho", "itype"):
            a = getattr(self, k)
            assert a.is_cuda and a.is_contiguous() and a.shape[0] == self.n
            setattr(s, k, a.data_ptr())
        s.lo_x, s.lo_y, s.hi_x, s.hi_y = (float(b) for b in self.box)
        return s


class Surrogate:
    """A network instance with its device buffers for up to `capacity` nodes."""

    def __init__(self, cfg: NetConfig, capacity: int, params: Optional[np.ndarray] = None, seed: int = 0):
        self.lib = _lib.lib()
        self.cfg = cfg
        self.capacity = int(capacity)
        h = C.c_void_p()
        c = cfg.c_struct()
        _lib.check(self.lib.uph_sur_create(C.byref(c), self.capacity, C.byref(h)), "uph_sur_create")
        self.handle = h
        self.count = int(self.lib.uph_sur_param_count(cfg.rounds))
        self.set_params(init_params(seed, cfg.rounds) if params is None else params)

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.uph_sur_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def set_stream(self, cuda_stream: int) -> None:
        _lib.check(self.lib.uph_sur_set_stream(self.handle, C.c_void_p(cuda_stream)), "uph_sur_set_stream")

    def set_params(self, flat: np.ndarray) -> None:
        a = np.ascontiguousarray(flat, dtype=np.float32)
        if a.size != self.count:
            raise ValueError(f"expected {self.count} parameters, got {a.size}")
        _lib.check(self.lib.uph_sur_set_params(self.handle, a.ctypes.data, a.size), "uph_sur_set_params")

    def get_params(self) -> np.ndarray:
        a = np.empty(self.count, np.float32)
        _lib.check(self.lib.uph_sur_get_params(self.handle, a.ctypes.data, a.size), "uph_sur_get_params")
        return a

    def set_fused(self, on: bool) -> None:
        """Fused node-chain kernels (True, default) or one GEMM per layer."""
        _lib.check(self.lib.uph_sur_set_fused(self.handle, int(bool(on))), "uph_sur_set_fused")

    def reset_optimizer(self) -> None:
        _lib.check(self.lib.uph_sur_reset_optimizer(self.handle), "uph_sur_reset_optimizer")

    def forward(self, nodes: Nodes):
        """Normalised outputs [n x 5] (torch, float32, on the GPU)."""
        import torch
        out = torch.empty((nodes.n, NOUT), dtype=torch.float32, device=nodes.x.device)
        s = nodes.c_struct()
        _lib.check(self.lib.uph_sur_forward(self.handle, C.byref(s), out.data_ptr()), "uph_sur_forward")
        return out

    def gradients(self, nodes: Nodes, target, want_grad: bool = True, want_loss: bool = True):
        """(loss or None, gradient torch tensor or None) of the mean squared
        error against target [n_fluid x 5] (normalised, float32, GPU)."""
        import torch
        assert target.dtype == torch.float32 and target.is_contiguous() and target.shape == (nodes.n_fluid, NOUT)
        grad = torch.empty(self.count, dtype=torch.float32, device=nodes.x.device) if want_grad else None
        loss = C.c_double()
        s = nodes.c_struct()
        _lib.check(self.lib.uph_sur_gradients(self.handle, C.byref(s), target.data_ptr(),
                                              grad.data_ptr() if want_grad else None,
                                              C.byref(loss) if want_loss else None), "uph_sur_gradients")
        return (loss.value if want_loss else None), grad

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8, clip: float = 1.0) -> None:
        _lib.check(self.lib.uph_sur_adam(self.handle, lr, beta1, beta2, eps, clip), "uph_sur_adam")

    def advance(self, sim, macro_steps: int, judge: Judge, report: Optional[SurReport] = None) -> SurReport:
        rep = report if report is not None else SurReport()
        j = judge.c_struct()
        _lib.check(self.lib.uph_sur_advance(self.handle, sim.handle, macro_steps, C.byref(j), C.byref(rep)),
                   "uph_sur_advance")
        return rep

    def save(self, path: str, **extra) -> None:
        c = dataclasses.asdict(self.cfg)
        np.savez(path, params=self.get_params(), config=np.array(repr(c)), **extra)

    @staticmethod
    def load_file(path: str) -> Tuple[NetConfig, np.ndarray]:
        z = np.load(path, allow_pickle=False)
        import ast
        c = ast.literal_eval(str(z["config"]))
        c["out_scale"] = tuple(c["out_scale"])
        return NetConfig(**c), z["params"]


# ---- training data ----------------------------------------------------------------
@dataclasses.dataclass
class FlumeBatch:
    deck: D.Deck
    state: Dict[str, np.ndarray]
    wall_table: Tuple[np.ndarray, np.ndarray, np.ndarray]
    pistons: List[Tuple[float, float]]
    box: Tuple[float, float, float, float]


def flume_batch(pistons: Sequence[Tuple[float, float]], length: float = 4.0, depth: float = 0.5, dx: float = 0.005,
                layers: int = 3, eta: float = 1.3, sponge_fraction: float = 0.7) -> FlumeBatch:
    """Wave flumes (D.wave_flume geometry) stacked in y, flume k driven by
    piston k = (amplitude A, period T): x = A (1 - cos(2 pi t / T)).  Each
    flume damps u in its last (1 - sponge_fraction) of length, like the
    workload's sponge at x >= 7 m of 10 m (System.c:333-335)."""
    decks = [D.wave_flume(length, depth, dx, layers, eta, amplitude=a, period=T, piston_layers=layers,
                          hydrostatic_walls=True) for a, T in pistons]
    amax = max(a for a, _ in pistons)
    pad = 4 * eta * dx + layers * dx + 2 * amax
    pitch = 2.0 * depth + 2 * pad
    fl, fx, mv, x0, hs, om = [], [], [], [], [], []
    for k, ((a, T), d) in enumerate(zip(pistons, decks)):
        off = k * pitch
        for blk, out in ((d.fluid, fl), (d.fixed, fx), (d.moving, mv)):
            b = blk.copy()
            b[:, 1] += off
            out.append(b)
        x0.append(d.wall_table[0])
        hs.append(d.wall_table[1])
        om.append(d.wall_table[2])
    p = dict(decks[0].params)
    deck = D.Deck(p, np.concatenate(fl), np.zeros((0, 12)), np.concatenate(fx), np.concatenate(mv), eta_override=eta)
    lo = (-pad, -pad)
    hi = (length + pad, (len(pistons) - 1) * pitch + 2.0 * depth + pad)
    deck.domain_lo, deck.domain_hi = lo, hi
    st = deck.initial_state()
    xf = st["Position"][:deck.n_fluid, 0]
    st["spongeFactor"][:] = np.where(xf >= sponge_fraction * length, p.get("sponge_factor0", 0.2), 0.0)
    return FlumeBatch(deck, st, (np.concatenate(x0), np.concatenate(hs), np.concatenate(om)), list(pistons),
                      (lo[0], lo[1], hi[0], hi[1]))


def raw_increments(cfg: NetConfig, s0: Dict[str, np.ndarray], s1: Dict[str, np.ndarray], nf: int) -> np.ndarray:
    """The fluid's macro-step increments the network predicts, unnormalised:
    (x1 - x0 - T u0, y1 - y0 - T v0, u1 - u0, v1 - v0, rho1 - rho0)."""
    T = cfg.macro_steps * cfg.dt
    p0, p1 = s0["Position"][:nf], s1["Position"][:nf]
    v0, v1 = s0["Velocity"][:nf], s1["Velocity"][:nf]
    return np.stack([p1[:, 0] - p0[:, 0] - T * v0[:, 0], p1[:, 1] - p0[:, 1] - T * v0[:, 1],
                     v1[:, 0] - v0[:, 0], v1[:, 1] - v0[:, 1],
                     s1["density"][:nf] - s0["density"][:nf]], axis=1)


@dataclasses.dataclass
class Frame:
    nodes: "Nodes"
    raw: object       # torch float64 [nf x 5] raw increments


def generate_frames(batch: FlumeBatch, cfg: NetConfig, warm_steps: int, windows: int, window_gap_steps: int,
                    pairs_per_window: int, precision: int = PREC_FP32_PAIR, graph_steps: int = 0,
                    device: str = "cuda") -> List[Frame]:
    """Plain-solver trajectories of the flume batch: after `warm_steps`,
    `windows` windows `window_gap_steps` apart, each `pairs_per_window`
    consecutive macro steps (state, increments) recorded."""
    import torch
    from .sim import Simulation
    K = cfg.macro_steps
    sim = Simulation(batch.deck.uph_params(PROFILE_WCSPH, precision))
    sim.upload(batch.state, 0)
    sim.set_wall_motion(*batch.wall_table)
    if graph_steps:
        sim.set_graph(graph_steps)
    nf = batch.deck.n_fluid
    frames = []
    sim.step(warm_steps)
    for w in range(windows):
        if w:
            sim.step(window_gap_steps)
        s0 = sim.download()
        for _ in range(pairs_per_window):
            sim.step(K)
            s1 = sim.download()
            raw = raw_increments(cfg, s0, s1, nf)
            frames.append(Frame(Nodes.from_state(s0, nf, batch.box, device),
                                torch.as_tensor(raw, dtype=torch.float64, device=device)))
            s0 = s1
    sim.close()
    return frames


def collect_rollout_frames(batch: FlumeBatch, sur: "Surrogate", warm_steps: int, windows: int, window_gap_steps: int,
                           horizons: Sequence[int], precision: int = PREC_FP32_PAIR,
                           device: str = "cuda") -> List[Frame]:
    """Frames from the network's own states: from plain states of the flume
    batch, the network advances `h` macro steps (for each h in horizons),
    then the plain solver takes one macro step from that network-made state
    (its leapfrog restarting, as after any network step); the pair is a
    training frame.  Teaches the network to correct the drift of its own
    rollouts (e.g. towards the walls)."""
    import torch
    from .sim import Simulation
    cfg = sur.cfg
    K = cfg.macro_steps
    nf = batch.deck.n_fluid
    p = batch.deck.uph_params(PROFILE_WCSPH, precision)
    length = batch.box[2]
    off = Judge(depth=1.0, surface_x0=batch.box[0], surface_x1=length, surface_bins=16, judge_every=1 << 30,
                fallback_macro=0)
    sim = Simulation(p)
    sim.upload(batch.state, 0)
    sim.set_wall_motion(*batch.wall_table)
    sim.step(warm_steps)
    frames = []
    for w in range(windows):
        if w:
            sim.step(window_gap_steps)
        st = sim.download()
        itime = int(sim.stats()["itime"])
        for h in horizons:
            s2 = Simulation(p)
            s2.upload(st, itime)
            s2.set_wall_motion(*batch.wall_table)
            sur.advance(s2, h, off)
            s_net = s2.download()
            s2.step(K)
            s_plain = s2.download()
            s2.close()
            frames.append(Frame(Nodes.from_state(s_net, nf, batch.box, device),
                                torch.as_tensor(raw_increments(cfg, s_net, s_plain, nf), dtype=torch.float64,
                                                device=device)))
    sim.close()
    return frames


def fit_output_scales(frames: List[Frame]) -> Tuple[float, ...]:
    """Root-mean-square of each raw increment over all frames."""
    import torch
    sq = torch.zeros(NOUT, dtype=torch.float64, device=frames[0].raw.device)
    n = 0
    for f in frames:
        sq += (f.raw * f.raw).sum(0)
        n += f.raw.shape[0]
    return tuple(float(math.sqrt(v / n)) if v > 0 else 1.0 for v in sq.tolist())


def train(sur: Surrogate, frames: List[Frame], iters: int, lr: float = 1e-3, lr_final: float = 2e-5,
          seed: int = 0, noise_vel: float = 0.0, noise_rho: float = 0.0, clip: float = 1.0,
          log_every: int = 100) -> List[Tuple[int, float]]:
    """Adam on random frames with a cosine learning-rate decay.  Optional
    input noise (velocity std noise_vel m/s, density std noise_rho kg/m^3) on
    the fluid nodes, with the targets corrected for it, so the network learns
    to undo small state errors of its own rollouts."""
    import torch
    cfg = sur.cfg
    T = cfg.macro_steps * cfg.dt
    scale = torch.tensor(cfg.out_scale, dtype=torch.float64, device=frames[0].raw.device)
    gen = torch.Generator(device=frames[0].raw.device).manual_seed(seed)
    rng = np.random.default_rng(seed)
    hist = []
    for it in range(iters):
        f = frames[int(rng.integers(len(frames)))]
        nodes, raw = f.nodes, f.raw
        nf = nodes.n_fluid
        if noise_vel > 0 or noise_rho > 0:
            du = torch.randn(nf, generator=gen, device=raw.device, dtype=torch.float64) * noise_vel
            dv = torch.randn(nf, generator=gen, device=raw.device, dtype=torch.float64) * noise_vel
            dr = torch.randn(nf, generator=gen, device=raw.device, dtype=torch.float64) * noise_rho
            u = nodes.u.clone()
            v = nodes.v.clone()
            rho = nodes.rho.clone()
            u[:nf] += du
            v[:nf] += dv
            rho[:nf] += dr
            nodes = Nodes(nodes.x, nodes.y, u, v, rho, nodes.itype, nf, nodes.box)
            raw = raw - torch.stack([T * du, T * dv, du, dv, dr], 1)
        target = (raw / scale).to(torch.float32).contiguous()
        want = (it % log_every == 0) or it == iters - 1
        loss, _ = sur.gradients(nodes, target, want_grad=False, want_loss=want)
        c = 0.5 * (1.0 + math.cos(math.pi * it / max(1, iters - 1)))
        sur.adam(lr_final + (lr - lr_final) * c, clip=clip)
        if want:
            hist.append((it, loss))
    return hist


# ---- comparison with the plain solver ------------------------------------------------
def surface_heights(pos: np.ndarray, x0: float, x1: float, bins: int) -> np.ndarray:
    """Highest fluid particle per x-bin (NaN for an empty bin)."""
    b = np.floor((pos[:, 0] - x0) * bins / (x1 - x0)).astype(np.int64)
    ok = (b >= 0) & (b < bins)
    out = np.full(bins, -np.inf)
    np.maximum.at(out, b[ok], pos[ok, 1])
    out[np.isinf(out)] = np.nan
    return out


def state_errors(a: Dict[str, np.ndarray], b: Dict[str, np.ndarray], nf: int, depth: float, x0: float, x1: float,
                 bins: int) -> dict:
    """Errors of state a against state b (same particles, reference order):
    RMS and largest relative density error, largest free-surface height
    difference as a fraction of depth."""
    ra, rb = a["density"][:nf], b["density"][:nf]
    rel = (ra - rb) / rb
    ha = surface_heights(a["Position"][:nf], x0, x1, bins)
    hb = surface_heights(b["Position"][:nf], x0, x1, bins)
    ok = ~np.isnan(ha) & ~np.isnan(hb)
    surf = float(np.max(np.abs(ha[ok] - hb[ok])) / depth) if ok.any() else 0.0
    return {"rho_rms": float(np.sqrt(np.mean(rel * rel))), "rho_max": float(np.max(np.abs(rel))), "surface": surf}


# ---- the wave-flume surrogate: data, training, evaluation ---------------------------------
def draw_pistons(seed: int, count: int) -> List[Tuple[float, float]]:
    """Piston (amplitude, period) pairs of the workload: A ~ U[0.02, 0.06] m,
    T ~ U[1.0, 1.6] s."""
    rng = np.random.default_rng(seed)
    return [(float(rng.uniform(0.02, 0.06)), float(rng.uniform(1.0, 1.6))) for _ in range(count)]


def train_flume(out_path: Optional[str] = None, seed: int = 0, n_flumes: int = 6, length: float = 4.0,
                depth: float = 0.5, dx: float = 0.005, macro_steps: int = 40, warm_time: float = 1.0,
                windows: int = 16, window_gap_time: float = 0.1, pairs_per_window: int = 10, iters: int = 3000,
                lr: float = 5e-4, noise_vel: float = 0.0, noise_rho: float = 0.0, dagger_rounds: int = 0,
                dagger_iters: int = 1500, dagger_horizons: Sequence[int] = (4, 12, 24), dagger_windows: int = 6,
                dagger_repeat: int = 3, edge_rho_scale: float = 1e-3, log=print) -> dict:
    """Generates flume trajectories with the plain FP32-pair WCSPH solver,
    trains a 3-round network on them (the last window held out), then for
    `dagger_rounds` rounds adds frames that start from the network's own
    rollouts (collect_rollout_frames, each repeated `dagger_repeat` times in
    the sampling pool) and trains on, and saves it.  Returns the training
    record (with the trained Surrogate)."""
    import time

    import torch
    t0 = time.time()
    pistons = draw_pistons(seed, n_flumes)
    batch = flume_batch(pistons, length, depth, dx)
    p = batch.deck.uph_params(PROFILE_WCSPH, PREC_FP32_PAIR)
    cfg = NetConfig.for_params(p, macro_steps, edge_rho_scale=edge_rho_scale)
    dt = cfg.dt
    frames = generate_frames(batch, cfg, int(round(warm_time / dt)), windows, int(round(window_gap_time / dt)),
                             pairs_per_window)
    torch.cuda.synchronize()
    t_gen = time.time() - t0
    held = frames[-pairs_per_window:] if windows > 1 else frames[-1:]
    train_frames = frames[:-pairs_per_window] if windows > 1 else frames
    cfg.out_scale = fit_output_scales(train_frames)
    nf = batch.deck.n_fluid
    u2 = sum(float((f.nodes.u[:nf] ** 2 + f.nodes.v[:nf] ** 2).mean()) for f in train_frames) / len(train_frames)
    cfg.vel_scale = max(math.sqrt(u2), 1e-3)
    log(f"frames {len(frames)} ({batch.deck.n_all} nodes each) in {t_gen:.1f} s; scales {cfg.out_scale}, "
        f"U {cfg.vel_scale:.4f}")
    sur = Surrogate(cfg, batch.deck.n_all, seed=seed)

    def held_loss():
        scale = torch.tensor(cfg.out_scale, dtype=torch.float64, device="cuda")
        tot = 0.0
        for f in held:
            l, _ = sur.gradients(f.nodes, (f.raw / scale).to(torch.float32).contiguous(), want_grad=False)
            tot += l
        return tot / len(held)

    l0 = held_loss()
    t1 = time.time()
    hist = train(sur, train_frames, iters, lr=lr, seed=seed, noise_vel=noise_vel, noise_rho=noise_rho,
                 log_every=max(1, iters // 20))
    for rnd in range(dagger_rounds):
        t2 = time.time()
        extra = collect_rollout_frames(batch, sur, int(round(warm_time / dt)), dagger_windows,
                                       int(round(2 * window_gap_time / dt)), dagger_horizons)
        train_frames = train_frames + extra * dagger_repeat
        log(f"rollout round {rnd}: {len(extra)} frames in {time.time() - t2:.1f} s; held-out {held_loss():.4f}")
        hist += train(sur, train_frames, dagger_iters, lr=lr * 0.3, seed=seed + 1 + rnd, noise_vel=noise_vel,
                      noise_rho=noise_rho, log_every=max(1, dagger_iters // 5))
    torch.cuda.synchronize()
    t_train = time.time() - t1
    l1 = held_loss()
    for it, l in hist:
        log(f"  iter {it:6d}  loss {l:.5f}")
    log(f"held-out loss {l0:.4f} -> {l1:.4f}; {iters} iterations in {t_train:.1f} s "
        f"({1e3 * t_train / max(1, iters):.2f} ms each)")
    rec = dict(pistons=np.array(pistons), history=np.array(hist), held_loss=np.array([l0, l1]),
               seconds=np.array([t_gen, t_train]), nodes=np.array(batch.deck.n_all))
    if out_path:
        sur.save(out_path, **rec)
    rec["surrogate"] = sur
    return rec


def evaluate_flume(sur: Surrogate, length: float = 4.0, depth: float = 0.5, dx: float = 0.005,
                   piston: Tuple[float, float] = (0.04, 1.3), warm_time: float = 0.5, steps: int = 2000,
                   judge: Optional[Judge] = None, precision: int = PREC_FP32_PAIR, plain_precision: int = None,
                   baselines: bool = True, log=print) -> dict:
    """One flume (the workload's geometry, `length` long) warmed up from rest
    by the plain solver, then advanced `steps` SPH steps (a) by the plain
    solver in `plain_precision` and (b) by the surrogate with its judge, from
    the same state.  Returns the errors of (b) against (a), the wall times and
    the judge's report; with `baselines` also the errors of the network alone
    (no judge) and of a zero network (x += T u, nothing else changes)."""
    import time

    import torch

    from ._capi import PREC_FP64
    from .sim import Simulation
    plain_precision = PREC_FP64 if plain_precision is None else plain_precision
    A, T = piston
    deck = D.wave_flume(length, depth, dx, amplitude=A, period=T, piston_layers=3, hydrostatic_walls=True)
    K = sur.cfg.macro_steps
    nmacro = steps // K
    steps = nmacro * K
    warm = int(round(warm_time / sur.cfg.dt))
    w = Simulation.from_deck(deck, PROFILE_WCSPH, precision)
    w.step(warm)
    st0 = w.download()
    w.close()
    nf = deck.n_fluid
    judge = judge or Judge(depth=depth, surface_x0=0.0, surface_x1=length, surface_bins=int(length / 0.05))
    bins = judge.surface_bins

    def new_sim(prec):
        sim = Simulation(deck.uph_params(PROFILE_WCSPH, prec))
        sim.upload(st0, warm)
        sim.set_wall_motion(*deck.wall_table)
        return sim

    def run_plain(prec):
        sim = new_sim(prec)
        sim.step(K)  # untimed: first-call allocations
        sim.upload(st0, warm)
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(nmacro):
            sim.step(K)
        torch.cuda.synchronize()
        el = time.perf_counter() - t
        out = sim.download()
        sim.close()
        return out, el

    def run_sur(net, jd):
        sim = new_sim(precision)
        torch.cuda.synchronize()
        t = time.perf_counter()
        rep = net.advance(sim, nmacro, jd)
        torch.cuda.synchronize()
        el = time.perf_counter() - t
        out = sim.download()
        sim.close()
        return out, el, rep

    ref, t_plain = run_plain(plain_precision)
    res = {"n_fluid": nf, "steps": steps, "macro_steps": K, "t_plain": t_plain}
    st, t_sur, rep = run_sur(sur, judge)
    res.update(t_surrogate=t_sur, report=rep.to_dict(), errors=state_errors(st, ref, nf, depth, 0.0, length, bins))
    res["speedup"] = t_plain / t_sur
    if baselines:
        off = dataclasses.replace(judge, judge_every=1 << 30)
        st_n, t_n, _ = run_sur(sur, off)
        res["network_only"] = state_errors(st_n, ref, nf, depth, 0.0, length, bins)
        res["t_network_only"] = t_n
        zero = Surrogate(sur.cfg, sur.capacity, np.zeros(sur.count, np.float32))
        st_z, _, _ = run_sur(zero, off)
        zero.close()
        res["zero_network"] = state_errors(st_z, ref, nf, depth, 0.0, length, bins)
        fs, t_fs = run_plain(precision)
        res["plain_same_precision"] = state_errors(fs, ref, nf, depth, 0.0, length, bins)
        res["t_plain_same_precision"] = t_fs
    log(res)
    return res


if __name__ == "__main__":
    import argparse
    import os
    ap = argparse.ArgumentParser(description="train the wave-flume surrogate on the GPU")
    ap.add_argument("--out", default="uph_b200/weights/flume_mpnn.npz")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--flumes", type=int, default=6)
    ap.add_argument("--length", type=float, default=4.0)
    ap.add_argument("--macro-steps", type=int, default=40)
    ap.add_argument("--warm-time", type=float, default=1.0)
    ap.add_argument("--windows", type=int, default=16)
    ap.add_argument("--pairs", type=int, default=10)
    ap.add_argument("--iters", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=5e-4)
    ap.add_argument("--noise-vel", type=float, default=0.0)
    ap.add_argument("--noise-rho", type=float, default=0.0)
    ap.add_argument("--dagger-rounds", type=int, default=2)
    a = ap.parse_args()
    os.makedirs(os.path.dirname(a.out) or ".", exist_ok=True)
    train_flume(a.out, a.seed, a.flumes, a.length, macro_steps=a.macro_steps, warm_time=a.warm_time,
                windows=a.windows, pairs_per_window=a.pairs, iters=a.iters, lr=a.lr, noise_vel=a.noise_vel,
                noise_rho=a.noise_rho, dagger_rounds=a.dagger_rounds)
