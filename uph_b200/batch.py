"""Batches of independent tanks advanced as one simulation.

The batched-tank workload: 256 dam-break and sloshing tanks drawn from a seed.
- Column width is uniform in [0.3, 1.5] m, height uniform in [0.5, 2.0] m,
  dx = 0.01 m, so each tank holds 1.5k-30k particles.
- Sloshing tanks are shaken horizontally with amplitude uniform in
  [0.01, 0.05] m and period uniform in [0.8, 2.0] s.

All tanks share one set of physical constants (dx, h, c0, dt), so they can be
one simulation:
- tanks are shelf-packed into one domain, separated by gaps wider than the
  interaction radius plus twice the largest wall stroke, so no pair ever
  crosses between tanks;
- fluid particles of all tanks form the fluid block;
- dam-break walls form the fixed block;
- sloshing walls form the moving block, shaken rigidly with their tank's own
  amplitude and period (uph_sim_set_wall_motion; the reference's sloshing
  walls, inputbp.c:244-276, generalised to whole tanks).

One step of the batch is one set of kernel launches for every tank; with
uph_sim_set_graph the whole multi-step call replays as one CUDA graph.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List

import numpy as np

from . import deck as D


@dataclasses.dataclass
class TankSpec:
    kind: str          # "dambreak" or "sloshing"
    width: float       # water column width (m)
    height: float      # water column height (m)
    amplitude: float   # sloshing: displacement amplitude A (x = A (1 - cos wt)); 0 for dam break
    period: float      # sloshing period (s)


def draw_tanks(seed: int = 0, count: int = 256) -> List[TankSpec]:
    """Half dam-break, half sloshing tanks, alternating, from one seed."""
    rng = np.random.default_rng(seed)
    tanks = []
    for k in range(count):
        w = float(rng.uniform(0.3, 1.5))
        h = float(rng.uniform(0.5, 2.0))
        a = float(rng.uniform(0.01, 0.05))
        T = float(rng.uniform(0.8, 2.0))
        if k % 2 == 0:
            tanks.append(TankSpec("dambreak", w, h, 0.0, 0.0))
        else:
            tanks.append(TankSpec("sloshing", w, h, a, T))
    return tanks


@dataclasses.dataclass
class Batch:
    deck: D.Deck
    tanks: List[TankSpec]
    fluid_ranges: List[tuple]      # per tank, [start, end) in the fluid block
    moving_ranges: List[tuple]     # per tank, [start, end) in the moving block (empty for dam breaks)
    offsets: List[tuple]           # per tank, (x, y) of its interior origin in the batch domain
    wall_x0: np.ndarray            # moving block: rest x
    wall_hs: np.ndarray            # moving block: half stroke (= amplitude A)
    wall_om: np.ndarray            # moving block: angular frequency


def _tank_rows(spec: TankSpec, dx: float, layers: int, p: dict):
    """Fluid rows and wall rows of one tank with its interior origin at (0, 0)."""
    nx, ny = int(round(spec.width / dx)), int(round(spec.height / dx))
    x, y = D.lattice(0.5 * dx, 0.5 * dx, nx, ny, dx)
    mass = p["density0"] * dx * dx
    fluid = D._rows(x, y, p["density0"], 0.0, mass, D.FLUID_ITYPE)
    if spec.kind == "dambreak":
        length, tank_h = 2.5 * spec.width, 1.3 * spec.height
    else:
        length, tank_h = spec.width, 1.5 * spec.height
    walls = D.tank_walls(length, tank_h, dx, layers, p["density0"], mass)
    return fluid, walls, length, tank_h


def build_batch(tanks: List[TankSpec], dx: float = 0.01, layers: int = 2, eta: float = 1.3,
                max_row_width: float = None) -> Batch:
    """One deck holding every tank; see the module docstring."""
    # shared constants: c0 from the tallest column (the workload's c0 = 10 sqrt(g H))
    hmax = max(t.height for t in tanks)
    p = D.base_params(dx, eta=eta, local_depth=hmax)
    h = eta * dx
    stroke_max = max(2.0 * t.amplitude for t in tanks)
    gap = 4.0 * h + 2.0 * stroke_max + (layers + 1) * dx
    built = [_tank_rows(t, dx, layers, p) for t in tanks]
    # shelf packing: tallest first, rows of about the square root of the total area
    order = sorted(range(len(tanks)), key=lambda k: -built[k][3])
    area = sum((b[2] + gap) * (b[3] + gap) for b in built)
    row_w = max_row_width or max(math.sqrt(area) * 1.2, max(b[2] for b in built) + gap)
    offsets = [None] * len(tanks)
    x, y, shelf_h = 0.0, 0.0, 0.0
    for k in order:
        length, tank_h = built[k][2], built[k][3]
        if x > 0.0 and x + length + gap > row_w:
            x, y = 0.0, y + shelf_h + gap
            shelf_h = 0.0
        offsets[k] = (x + layers * dx, y + layers * dx)
        x += length + 2 * layers * dx + gap
        shelf_h = max(shelf_h, tank_h + layers * dx)
    fluid_blocks, fixed_blocks, moving_blocks = [], [], []
    fluid_ranges, moving_ranges = [], []
    wx0, whs, wom = [], [], []
    nf = nm = 0
    for k, (spec, (fluid, walls, _, _)) in enumerate(zip(tanks, built)):
        ox, oy = offsets[k]
        f = fluid.copy()
        f[:, 0] += ox
        f[:, 1] += oy
        w = walls.copy()
        w[:, 0] += ox
        w[:, 1] += oy
        fluid_blocks.append(f)
        fluid_ranges.append((nf, nf + f.shape[0]))
        nf += f.shape[0]
        if spec.kind == "sloshing":
            moving_blocks.append(w)
            moving_ranges.append((nm, nm + w.shape[0]))
            nm += w.shape[0]
            wx0.append(w[:, 0].copy())
            whs.append(np.full(w.shape[0], spec.amplitude))
            wom.append(np.full(w.shape[0], 2.0 * math.pi / spec.period))
        else:
            fixed_blocks.append(w)
            moving_ranges.append((nm, nm))
    cat = lambda blocks: np.concatenate(blocks) if blocks else np.zeros((0, 12))
    deck = D.Deck(p, cat(fluid_blocks), np.zeros((0, 12)), cat(fixed_blocks), cat(moving_blocks), eta_override=eta)
    allrows = np.concatenate([deck.fluid, deck.fixed, deck.moving])
    lo = allrows[:, :2].min(axis=0) - (4 * h + stroke_max + dx)
    hi = allrows[:, :2].max(axis=0) + (4 * h + stroke_max + dx)
    hi[1] += 0.5 * hmax  # room for splashes above the tallest tank
    deck.domain_lo = (float(lo[0]), float(lo[1]))
    deck.domain_hi = (float(hi[0]), float(hi[1]))
    f = lambda parts: np.concatenate(parts) if parts else np.zeros(0)
    return Batch(deck, tanks, fluid_ranges, moving_ranges, offsets, f(wx0), f(whs), f(wom))


def tank_deck(batch: Batch, k: int) -> tuple:
    """The k-th tank alone as its own deck (same constants and positions),
    with its wall-shaking table: the per-tank "plain" run of the batch."""
    spec = batch.tanks[k]
    f0, f1 = batch.fluid_ranges[k]
    fluid = batch.deck.fluid[f0:f1]
    if spec.kind == "sloshing":
        m0, m1 = batch.moving_ranges[k]
        moving = batch.deck.moving[m0:m1]
        fixed = np.zeros((0, 12))
        table = (batch.wall_x0[m0:m1], batch.wall_hs[m0:m1], batch.wall_om[m0:m1])
    else:
        # fixed walls of dam-break tanks are stored in tank order
        counts = [b for b in range(k) if batch.tanks[b].kind == "dambreak"]
        start = sum(_wall_count(batch, b) for b in counts)
        fixed = batch.deck.fixed[start:start + _wall_count(batch, k)]
        moving = np.zeros((0, 12))
        table = None
    d = D.Deck(dict(batch.deck.params), fluid.copy(), np.zeros((0, 12)), fixed.copy(), moving.copy(),
               eta_override=batch.deck.eta_override)
    h = batch.deck.eta_override * batch.deck.params["dx"]
    rows = np.concatenate([d.fluid, d.fixed, d.moving])
    pad = 4 * h + 0.2
    d.domain_lo = (float(rows[:, 0].min() - pad), float(rows[:, 1].min() - pad))
    d.domain_hi = (float(rows[:, 0].max() + pad), float(rows[:, 1].max() + pad + spec.height))
    return d, table


def _wall_count(batch: Batch, k: int) -> int:
    spec = batch.tanks[k]
    dx = batch.deck.params["dx"]
    layers = 2
    length = 2.5 * spec.width if spec.kind == "dambreak" else spec.width
    tank_h = 1.3 * spec.height if spec.kind == "dambreak" else 1.5 * spec.height
    nxw = int(round(length / dx)) + 2 * layers
    ny = int(round(tank_h / dx))
    return layers * nxw + 2 * layers * ny


def free_surface_heights(positions: np.ndarray, x0: float, width: float, dx: float, nbins: int = 8) -> np.ndarray:
    """Height of the highest fluid particle in each of `nbins` equal x-bins
    over [x0, x0 + width] (empty bins give 0)."""
    x = positions[:, 0]
    y = positions[:, 1]
    edges = np.linspace(x0, x0 + width, nbins + 1)
    idx = np.clip(np.digitize(x, edges) - 1, 0, nbins - 1)
    out = np.zeros(nbins)
    np.maximum.at(out, idx, y)
    return out
