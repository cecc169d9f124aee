"""Generates the golden vectors in this directory from the reference's own
solver, compiled from its sources by oracle/Makefile (oracle/_ref/libuph_ref.so).

    python tests/golden/make_golden.py

Each case is a small synthetic deck (written in the reference's file formats,
read by the reference's own CreateSystem / input / inputbp) advanced with the
reference's derivatives() and the sph.cc leapfrog for NSTEPS steps.  The
fluid fields after steps 1 and 3 and the pair list of step 1's derivatives()
call are stored.  Every case is checked to have at most 39 in-radius
neighbours per query, so the reference's 40-NN cap never binds and the pair
set does not depend on libnabo's tie order.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from uph_b200 import deck as D  # noqa: E402

NSTEPS = 3
STORED_STEPS = (1, 3)  # fields after these steps; pairs of step 1


def _perturb(deck: D.Deck, seed: int, vel: float = 0.05) -> D.Deck:
    """Random fluid velocities and local velocities so every pair term is non-zero."""
    rng = np.random.default_rng(seed)
    f = deck.fluid
    f[:, 2:4] = rng.uniform(-vel, vel, size=(f.shape[0], 2))
    f[:, 10:12] = f[:, 2:4] + rng.uniform(-0.1 * vel, 0.1 * vel, size=(f.shape[0], 2))
    f[:, 4] *= 1.0 + rng.uniform(-1e-3, 1e-3, size=f.shape[0])
    return deck


def cases():
    """name -> Deck"""
    out = {}
    K = dict(thermal_diffusivity0=0.015)  # the reference hydrostatic deck's value
    out["dambreak_h13"] = _perturb(D.dam_break(tank=(1.0, 1.0), column=(0.4, 0.6), dx=0.02, layers=2,
                                               hydrostatic=True, **K), seed=1)
    # the reference decks' own smoothing length eta = sqrt(19 / 4 pi)
    d = D.dam_break(tank=(0.8, 0.6), column=(0.5, 0.3), dx=0.02, layers=2, eta=0.0, hydrostatic=True, **K)
    d.params["near_neighbor"] = 19
    out["tank_nn19"] = _perturb(d, seed=2)
    out["flume_piston_sponge"] = _perturb(D.wave_flume(length=7.6, depth=0.2, dx=0.04, layers=2, amplitude=0.02,
                                                       period=1.2, **K), seed=3, vel=0.02)
    for mode in (1, 4, 5, 0):
        out[f"wallforce_mode{mode}"] = _perturb(D.dam_break(tank=(0.5, 0.5), column=(0.3, 0.3), dx=0.02, layers=2,
                                                            hydrostatic=True, select_boundary_force=mode, **K),
                                                seed=10 + mode)
    # no walls: ParticleBoundary = Nf - 1 excludes the last fluid particle as a partner
    d = D.dam_break(tank=(0.4, 0.4), column=(0.2, 0.2), dx=0.02, layers=2, hydrostatic=True, **K)
    d.fixed = np.zeros((0, 12))
    out["fluid_only"] = _perturb(d, seed=20)
    # ragged: irregular fluid positions, gravity off, a solid block
    d = D.dam_break(tank=(0.6, 0.6), column=(0.4, 0.4), dx=0.02, layers=2, hydrostatic=True, gravity_flag=0, **K)
    rng = np.random.default_rng(21)
    d.fluid[:, 0:2] += rng.uniform(-0.2, 0.2, size=(d.fluid.shape[0], 2)) * 0.02
    solid = d.fluid[-40:].copy()
    solid[:, 9] = 5
    d.fluid = d.fluid[:-40]
    d.solid = solid
    out["ragged_solid"] = _perturb(d, seed=22)
    return out


def run_case(name: str, deck: D.Deck) -> dict:
    tmp = tempfile.mkdtemp(prefix=f"uph_golden_{name}_")
    deck.write(tmp)
    eta = deck.eta_override
    run = O.RefRun(tmp, eta_override=eta)
    out = {"fluid": deck.fluid, "solid": deck.solid, "fixed": deck.fixed, "moving": deck.moving,
           "eta_override": np.float64(eta),
           "params": np.array([deck.params[k] for k, _ in D.PARAM_ORDER], dtype=np.float64),
           "domain_lo": np.array(deck.domain()[0]), "domain_hi": np.array(deck.domain()[1])}
    for step in range(1, NSTEPS + 1):
        run.step(1)
        if run.truncated_queries() or run.max_inradius() > 39:
            raise RuntimeError(f"{name}: the 40-NN cap binds (max in-radius {run.max_inradius()})")
        if step not in STORED_STEPS:
            continue
        for f in O.FLUID_FIELDS:
            out[f"s{step}_{f}"] = run.get(f)
        if step != 1:
            continue
        i, j = run.pairs()
        out[f"s{step}_i_pair"] = i
        out[f"s{step}_j_pair"] = j
        out[f"s{step}_rij2"] = run.get("rij2")
        out[f"s{step}_w"] = run.get("w")
        out[f"s{step}_dwcdx"] = run.get("dwcdx")
        out[f"s{step}_max_inradius"] = np.int64(run.max_inradius())
    run.close()
    return out


def deck_from_golden(g) -> D.Deck:
    params = {k: (int(v) if t is int else float(v)) for (k, t), v in zip(D.PARAM_ORDER, g["params"])}
    deck = D.Deck(params, g["fluid"], g["solid"], g["fixed"], g["moving"], eta_override=float(g["eta_override"]))
    deck.domain_lo = tuple(float(v) for v in g["domain_lo"])
    deck.domain_hi = tuple(float(v) for v in g["domain_hi"])
    return deck


def main():
    O.build(reference=True)
    for name, deck in cases().items():
        data = run_case(name, deck)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **data)
        print(f"{name}: nf={deck.n_fluid} n={deck.n_all} pairs={data['s1_i_pair'].size} "
              f"max_inradius={int(data['s1_max_inradius'])} -> {os.path.relpath(path, ROOT)} "
              f"({os.path.getsize(path) // 1024} KiB)")


if __name__ == "__main__":
    main()
