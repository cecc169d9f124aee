"""Deck formats and synthetic tanks.

The reference reads a case from fixed file names in the working directory:

* ``parameters.dat`` -- 34 whitespace-separated values read by one fscanf in
  CreateSystem (src/lib/System.c:60-94), in PARAM_ORDER below;
* ``FluidParticle.dat``, ``SolidParticle.dat``, ``FixedBoundaryParticle.dat``,
  ``MovingBoundaryParticle.dat``, ``FrozenParticle.dat`` -- a count line, then
  12 columns per particle: x y u v density DynamicPressure mass tempPosition
  tempPositionGate itype localVelocity_x localVelocity_y (input.c:59-71,
  inputbp.c:88-150).

This module reads and writes those files, applies the reference's derived
quantities (System.c:292-335, input.c:105-145, inputbp.c:285-290) and builds
the synthetic tanks used for parity tests and benchmarks.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, Optional

import numpy as np

from ._capi import PROFILE_REF, PREC_FP64, empty_state

# parameters.dat order and C type, System.c:60-94
PARAM_ORDER = [
    ("stroke", float), ("wave_period", float), ("local_depth", float), ("flat_bottom_length", float),
    ("density0", float), ("adiabatic_constant", float), ("gravity", float), ("dx", float), ("dy", float),
    ("dim", int), ("viscosity0", float), ("mach_number", float), ("peclet_number", float),
    ("epsilon", float), ("alpha", float), ("virtual_type", int), ("print_step", int),
    ("screen_step", int), ("time_step", float), ("lid_velocity", float), ("near_neighbor", int),
    ("select_boundary_force", int), ("lennard_select", float), ("spring_constant0", float),
    ("damping_constant0", float), ("flag_init_simul", int), ("gravity_flag", int),
    ("thermal_diffusivity0", float), ("moving_boundary", int),
    ("number_of_initialization_steps", int), ("pressure_probe_x", float),
    ("pressure_probe_y", float), ("stress_type", int), ("dissipation_control_volume", int),
]

PARTICLE_FILES = ["FluidParticle.dat", "SolidParticle.dat", "FixedBoundaryParticle.dat",
                  "MovingBoundaryParticle.dat", "FrozenParticle.dat"]

FLUID_ITYPE = 1
FIXED_WALL_ITYPE = 2


def derive_params(p: dict, eta_override: float = 0.0) -> dict:
    """Derived quantities of CreateSystem (System.c:292-335) and input.c:107."""
    p = dict(p)
    g, depth, mach = p["gravity"], p["local_depth"], p["mach_number"]
    if p["moving_boundary"] == 2:
        c0 = math.sqrt(2.0 * g * depth) / mach
    else:
        c0 = math.sqrt(g * depth) / mach
    p["speed_of_sound"] = c0
    p["compression_factor"] = (1.0 / p["adiabatic_constant"]) * p["density0"] * c0 * c0
    p["omega"] = 2.0 * math.pi / p["wave_period"] if p["wave_period"] != 0 else 0.0
    p["eta"] = math.sqrt(p["near_neighbor"] / (4.0 * math.pi))
    if eta_override > 0:
        p["eta"] = eta_override
    p["h"] = p["eta"] * p["dx"]
    p["lennard_coefficient"] = g * depth
    p["sponge_factor0"] = 0.2
    p["sponge_position0"] = 7.0
    p["wave_absorption"] = 1
    return p


def read_parameters(path: str) -> dict:
    with open(path) as f:
        toks = f.read().split()
    if len(toks) < len(PARAM_ORDER):
        raise ValueError(f"{path}: {len(toks)} values, {len(PARAM_ORDER)} expected")
    out = {}
    for (name, typ), tok in zip(PARAM_ORDER, toks):
        out[name] = int(float(tok)) if typ is int else float(tok)
    return out


def write_parameters(path: str, p: dict) -> None:
    with open(path, "w") as f:
        for name, typ in PARAM_ORDER:
            v = p[name]
            f.write(f"{int(v)}\n" if typ is int else f"{float(v)!r}\n")


def _read_particles(path: str) -> np.ndarray:
    if not os.path.exists(path):
        return np.zeros((0, 12))
    with open(path) as f:
        first = f.readline().split()
        n = int(first[0]) if first else 0
        if n == 0:
            return np.zeros((0, 12))
        data = np.loadtxt(f, max_rows=n, ndmin=2)
    if data.shape != (n, 12):
        raise ValueError(f"{path}: expected {n} rows of 12 columns, got {data.shape}")
    return data


def _write_particles(path: str, rows: np.ndarray) -> None:
    rows = np.asarray(rows, dtype=np.float64).reshape(-1, 12)
    with open(path, "w") as f:
        f.write(f"{rows.shape[0]}\n")
        if rows.shape[0]:
            fmt = " ".join(["%.17g"] * 9 + ["%d"] + ["%.17g"] * 2)
            np.savetxt(f, rows, fmt=fmt)


@dataclasses.dataclass
class Deck:
    """A case: parameters plus particle rows (12 columns) per block."""
    params: dict
    fluid: np.ndarray
    solid: np.ndarray
    fixed: np.ndarray
    moving: np.ndarray
    eta_override: float = 0.0
    domain_lo: tuple = (0.0, 0.0)
    domain_hi: tuple = (0.0, 0.0)
    # per-particle motion of the moving block (x0, half stroke, omega) for
    # uph_sim_set_wall_motion, or None for the reference's own wall motion
    wall_table: Optional[tuple] = None

    @property
    def n_fluid(self) -> int:
        return int(self.fluid.shape[0])

    @property
    def n_all(self) -> int:
        return int(self.fluid.shape[0] + self.solid.shape[0] + self.fixed.shape[0] + self.moving.shape[0])

    def write(self, directory: str) -> None:
        os.makedirs(directory, exist_ok=True)
        write_parameters(os.path.join(directory, "parameters.dat"), self.params)
        _write_particles(os.path.join(directory, "FluidParticle.dat"), self.fluid)
        _write_particles(os.path.join(directory, "SolidParticle.dat"), self.solid)
        _write_particles(os.path.join(directory, "FixedBoundaryParticle.dat"), self.fixed)
        _write_particles(os.path.join(directory, "MovingBoundaryParticle.dat"), self.moving)
        _write_particles(os.path.join(directory, "FrozenParticle.dat"), np.zeros((0, 12)))

    def uph_params(self, profile: int = PROFILE_REF, precision: int = PREC_FP64,
                   av_alpha: Optional[float] = None, knn_cap: int = 0) -> dict:
        """A dict for UphParams.from_dict: file fields, derived fields, counts.
        knn_cap = 40 is the reference's own 40-nearest cap (derivatives.c:1085)."""
        p = derive_params(self.params, self.eta_override)
        p.update(profile=profile, precision=precision, n_fluid=self.n_fluid,
                 n_solid=int(self.solid.shape[0]), n_fixed=int(self.fixed.shape[0]),
                 n_moving=int(self.moving.shape[0]), knn_cap=knn_cap,
                 av_alpha=self.params["alpha"] if av_alpha is None else av_alpha)
        lo, hi = self.domain()
        p["domain_lo"] = list(lo)
        p["domain_hi"] = list(hi)
        return p

    def domain(self):
        if self.domain_hi != (0.0, 0.0):
            return self.domain_lo, self.domain_hi
        rows = np.concatenate([self.fluid, self.solid, self.fixed, self.moving])
        lo = rows[:, :2].min(axis=0)
        hi = rows[:, :2].max(axis=0)
        pad = 4.0 * derive_params(self.params, self.eta_override)["h"]
        return (float(lo[0] - pad), float(lo[1] - pad)), (float(hi[0] + pad), float(hi[1] + pad + (hi[1] - lo[1])))

    def initial_state(self) -> Dict[str, np.ndarray]:
        """State arrays as the reference holds them at its first derivatives()
        call: fluid rows from input() (input.c:57-131), wall rows from
        inputbp() (inputbp.c:88-150, 285-290), rates zero, *_min copies
        (sph.cc:79-87), sponge factors from input.c:137-144."""
        p = derive_params(self.params, self.eta_override)
        rows = np.concatenate([self.fluid, self.solid, self.fixed, self.moving])
        nf, n = self.n_fluid, rows.shape[0]
        st = empty_state(nf, n)
        st["Position"][:] = rows[:, 0:2]
        st["Velocity"][:] = rows[:, 2:4]
        st["density"][:] = rows[:, 4]
        st["DynamicPressure"][:] = rows[:, 5]
        st["mass"][:] = rows[:, 6]
        st["itype"][:] = rows[:, 9].astype(np.int32)
        st["localVelocity"][:] = rows[:, 10:12]
        st["localDensity"][:] = p["density0"]
        st["localPressure"][:] = 0.0
        st["density_min"][:] = st["density"][:nf]
        st["DynamicPressure_min"][:] = st["DynamicPressure"][:nf]
        st["spongeFactor"][:] = np.where(st["Position"][:nf, 0] >= p["sponge_position0"], p["sponge_factor0"], 0.0)
        return st


    def dam_gate_flag(self) -> np.ndarray:
        """damGateFlag as input() sets it: fluid in the 0.38 m dam column 1,
        the rest of the fluid -1 (input.c:146-159), walls 0 (inputbp.c:311)."""
        flag = np.zeros(self.n_all, np.int32)
        flag[:self.n_fluid] = np.where(self.fluid[:, 0] <= 0.38, 1, -1)
        return flag


def read_deck(directory: str, eta_override: float = 0.0) -> Deck:
    p = read_parameters(os.path.join(directory, "parameters.dat"))
    blocks = [_read_particles(os.path.join(directory, name)) for name in PARTICLE_FILES[:4]]
    return Deck(p, *blocks, eta_override=eta_override)


# ---------------------------------------------------------------- synthetic --

def base_params(dx: float, local_depth: float = 2.0, dt: Optional[float] = None, eta: float = 1.3,
                **over) -> dict:
    """parameters.dat values for the synthetic tanks.  Physics constants not
    named by the workload (viscosity, diffusivity, spring and damping
    constants, epsilon, stress and wall-force modes) are those of the
    reference's hydrostatic deck (tests/hydrostaticPressure/parameters.dat)."""
    p = dict(
        stroke=0.0, wave_period=1.0, local_depth=local_depth, flat_bottom_length=1.0,
        density0=1000.0, adiabatic_constant=7.0, gravity=9.81, dx=dx, dy=dx, dim=2,
        viscosity0=1e-6, mach_number=0.1, peclet_number=12.5, epsilon=1.0, alpha=0.01,
        virtual_type=77, print_step=1000000, screen_step=1000000, time_step=0.0, lid_velocity=0.0,
        near_neighbor=19, select_boundary_force=3, lennard_select=0.01, spring_constant0=0.00589,
        damping_constant0=0.05345, flag_init_simul=1, gravity_flag=1, thermal_diffusivity0=0.015,
        moving_boundary=0, number_of_initialization_steps=1000000000, pressure_probe_x=0.0,
        pressure_probe_y=0.0, stress_type=1, dissipation_control_volume=1,
    )
    p.update(over)
    d = derive_params(p, eta)
    if dt is None:
        dt = 0.2 * d["h"] / d["speed_of_sound"]
    p["time_step"] = dt
    if "thermal_diffusivity0" not in over:
        # The REF profile's pressure / density diffusion (derivatives.c:1569-1672)
        # is explicit with coefficient gamma * kappa; the reference deck's
        # kappa = 0.015 m^2/s belongs to dx = 0.01 m, dt = 1e-5 s.  At the
        # workloads' finer spacings it would break the explicit diffusion
        # limit, so kappa keeps the diffusion number gamma kappa dt / h^2 at 0.02.
        p["thermal_diffusivity0"] = 0.02 * d["h"] ** 2 / (p["adiabatic_constant"] * dt)
    return p


def _rows(x, y, rho, p, mass, itype):
    n = x.size
    r = np.zeros((n, 12))
    r[:, 0] = x
    r[:, 1] = y
    r[:, 4] = rho
    r[:, 5] = p
    r[:, 6] = mass
    r[:, 9] = itype
    return r


def lattice(x0, y0, nx, ny, dx):
    ix, iy = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    return (x0 + ix.ravel() * dx), (y0 + iy.ravel() * dx)


def tank_walls(length, height, dx, layers, rho0, mass, open_top=True):
    """Wall particles outside the tank interior [0, length] x [0, height]:
    `layers` rows at (k + 1/2) dx outside each face; the bottom rows span the
    corners.  Fluid sits at dx/2 inside each face, so every fluid-wall gap is
    dx."""
    nxw = int(round(length / dx)) + 2 * layers
    xs, ys = [], []
    for k in range(layers):
        xb = -(layers - 0.5) * dx + np.arange(nxw) * dx
        xs.append(xb)
        ys.append(np.full_like(xb, -(k + 0.5) * dx))
    ny = int(round(height / dx))
    yside = 0.5 * dx + np.arange(ny) * dx
    for k in range(layers):
        xs.append(np.full_like(yside, -(k + 0.5) * dx))
        ys.append(yside)
        xs.append(np.full_like(yside, length + (k + 0.5) * dx))
        ys.append(yside)
    x = np.concatenate(xs)
    y = np.concatenate(ys)
    return _rows(x, y, rho0, 0.0, mass, FIXED_WALL_ITYPE)


def hydrostatic_fields(y, depth, p):
    """p = rho0 g (H - y) and rho from the inverse Tait law."""
    d = derive_params(p)
    pres = p["density0"] * p["gravity"] * (depth - y)
    rho = p["density0"] * (1.0 + pres / d["compression_factor"]) ** (1.0 / p["adiabatic_constant"])
    return rho, pres


def dam_break(tank=(4.0, 3.0), column=(1.0, 2.0), dx=0.02, layers=2, eta=1.3, hydrostatic=False,
              **over) -> Deck:
    """Water column at the left wall of an open tank (config 0 / config 2
    geometry).  Fluid on a lattice from (dx/2, dx/2), zero velocity, particle
    mass rho0 dx^2; `hydrostatic` sets p = rho0 g (H - y) and the matching
    Tait density instead of rho0 / 0."""
    p = base_params(dx, eta=eta, **over)
    nx, ny = int(round(column[0] / dx)), int(round(column[1] / dx))
    x, y = lattice(0.5 * dx, 0.5 * dx, nx, ny, dx)
    mass = p["density0"] * dx * dx
    if hydrostatic:
        rho, pres = hydrostatic_fields(y, column[1], p)
    else:
        rho, pres = p["density0"], 0.0
    fluid = _rows(x, y, rho, pres, mass, FLUID_ITYPE)
    walls = tank_walls(tank[0], tank[1], dx, layers, p["density0"], mass)
    deck = Deck(p, fluid, np.zeros((0, 12)), walls, np.zeros((0, 12)), eta_override=eta)
    pad = 4 * eta * dx + layers * dx
    deck.domain_lo = (-pad, -pad)
    deck.domain_hi = (tank[0] + pad, max(tank[1], column[1]) * 1.5 + pad)
    return deck


def hydrostatic_tank(width=2.0, depth=1.0, dx=0.002, layers=3, eta=1.3, tank_height=None, **over) -> Deck:
    """Config 1: still water filling the tank width, density set
    hydrostatically; the analytic answer is p = rho0 g (H - y)."""
    th = depth * 1.2 if tank_height is None else tank_height
    deck = dam_break(tank=(width, th), column=(width, depth), dx=dx, layers=layers, eta=eta,
                     hydrostatic=True, **over)
    # wall particles carry the hydrostatic state of their depth (zero gauge
    # pressure above the surface), so the walls push back as hard as the
    # water next to them
    yw = np.minimum(deck.fixed[:, 1], depth)
    deck.fixed[:, 4], deck.fixed[:, 5] = hydrostatic_fields(yw, depth, deck.params)
    return deck


def wave_flume(length=10.0, depth=0.5, dx=0.005, layers=3, eta=1.3, amplitude=0.04, period=1.3,
               piston_layers=1, hydrostatic_walls=False, **over) -> Deck:
    """Config 4 geometry: a flume whose left wall is a piston wavemaker, one
    column of moving particles (itype 3, as in the reference's wave deck) at
    x = S/2 (1 - cos wt) (inputbp.c:194-207, movingBoundary 1, S = 2A).  The
    sponge layer damps u for x >= 7 m (System.c:333-335, input.c:137-144).
    Fluid starts one spacing right of the piston; bottom and right walls have
    `layers` rows.

    For long runs: `piston_layers` > 1 makes the piston that many columns
    thick (at x = 0, -dx, ...), moved rigidly through `deck.wall_table`
    (x = x0 + A (1 - cos wt), the same displacement; the reference's own
    motion would put every column at one x), and `hydrostatic_walls` gives
    the wall particles the hydrostatic density and pressure of their depth.
    With one column and walls at rest density the fluid next to the piston
    leaks through it within a few hundred steps."""
    over = dict(over)
    over.setdefault("local_depth", depth)
    p = base_params(dx, eta=eta, stroke=2.0 * amplitude, wave_period=period, moving_boundary=1, **over)
    nx, ny = int(round(length / dx)), int(round(depth / dx))
    x, y = lattice(dx, 0.5 * dx, nx, ny, dx)
    mass = p["density0"] * dx * dx
    rho, pres = hydrostatic_fields(y, depth, p)
    fluid = _rows(x, y, rho, pres, mass, FLUID_ITYPE)
    xs, ys = [], []
    nxw = nx + 1 + 2 * layers
    for k in range(layers):
        xb = -layers * dx + np.arange(nxw) * dx
        xs.append(xb)
        ys.append(np.full_like(xb, -(k + 0.5) * dx))
    nyw = int(round(1.5 * depth / dx))
    yside = 0.5 * dx + np.arange(nyw) * dx
    for k in range(layers):
        xs.append(np.full_like(yside, (nx + 1 + k) * dx))
        ys.append(yside)
    fixed = _rows(np.concatenate(xs), np.concatenate(ys), p["density0"], 0.0, mass, FIXED_WALL_ITYPE)
    xp = np.concatenate([np.full_like(yside, -k * dx) for k in range(piston_layers)])
    yp = np.tile(yside, piston_layers)
    moving = _rows(xp, yp, p["density0"], 0.0, mass, 3)
    if hydrostatic_walls:
        for blk in (fixed, moving):
            blk[:, 4], blk[:, 5] = hydrostatic_fields(np.minimum(blk[:, 1], depth), depth, p)
    deck = Deck(p, fluid, np.zeros((0, 12)), fixed, moving, eta_override=eta)
    if piston_layers > 1:
        deck.wall_table = (xp.copy(), np.full(xp.size, amplitude), np.full(xp.size, 2.0 * math.pi / period))
    pad = 4 * eta * dx + max(layers, piston_layers) * dx + 2 * amplitude
    deck.domain_lo = (-pad, -pad)
    deck.domain_hi = (length + pad, depth * 2.0 + pad)
    return deck


def lid_cavity(size=0.4, dx=0.02, layers=2, eta=1.3, lid_velocity=1.0, **over) -> Deck:
    """A lid-driven cavity: water filling a size x size box whose top is a
    row of moving particles sliding at lid_velocity (movingBoundary 3,
    inputbp.c:209-223: x = tempPosition + U t).  Gravity off."""
    over = dict(over)
    over.setdefault("gravity_flag", 0)
    p = base_params(dx, eta=eta, moving_boundary=3, lid_velocity=lid_velocity, **over)
    n = int(round(size / dx))
    x, y = lattice(0.5 * dx, 0.5 * dx, n, n, dx)
    mass = p["density0"] * dx * dx
    fluid = _rows(x, y, p["density0"], 0.0, mass, FLUID_ITYPE)
    fixed = tank_walls(size, size, dx, layers, p["density0"], mass)
    nxl = n + 2 * layers
    xs = np.concatenate([-(layers - 0.5) * dx + np.arange(nxl) * dx for _ in range(layers)])
    ys = np.concatenate([np.full(nxl, size + (k + 0.5) * dx) for k in range(layers)])
    moving = _rows(xs, ys, p["density0"], 0.0, mass, 3)
    moving[:, 7] = xs  # tempPosition
    moving[:, 8] = ys  # tempPositionGate
    deck = Deck(p, fluid, np.zeros((0, 12)), fixed, moving, eta_override=eta)
    pad = 4 * eta * dx + layers * dx
    deck.domain_lo = (-pad - 0.5 * size, -pad)
    deck.domain_hi = (size + pad + 0.5 * size, size + pad + layers * dx)
    return deck


def gate_dam_break(tank=(1.0, 0.6), column=(0.3, 0.4), dx=0.02, layers=2, eta=1.3, gate_velocity=1.0,
                   **over) -> Deck:
    """A dam break released by a gate (movingBoundary 2, inputbp.c:224-243):
    a column of moving particles one spacing right of the water, lifted at
    gate_velocity until 1.5 (LocalDepth - 15 dx) / gate_velocity."""
    over = dict(over)
    over.setdefault("local_depth", column[1])
    d = dam_break(tank=tank, column=column, dx=dx, layers=layers, eta=eta, hydrostatic=True, moving_boundary=2,
                  lid_velocity=gate_velocity, **over)
    ny = int(round(column[1] / dx))
    ys = 0.5 * dx + np.arange(ny) * dx
    xs = np.full(ny, column[0] + 0.5 * dx)
    moving = _rows(xs, ys, d.params["density0"], 0.0, d.params["density0"] * dx * dx, 3)
    moving[:, 7] = xs
    moving[:, 8] = ys
    d.moving = moving
    return d

