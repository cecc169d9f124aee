"""Batched tanks: many independent dam-break and sloshing tanks advanced as
one simulation (one set of launches per step, CUDA-graph replays, autotuned
cell / tile sizes) must reproduce each tank run on its own."""
import numpy as np
import pytest

from _util import compare_fields, rel_err
from oracle import oracle as O
from uph_b200 import batch as B

pytestmark = pytest.mark.gpu

SMALL = [
    B.TankSpec("dambreak", 0.30, 0.50, 0.0, 0.0),
    B.TankSpec("sloshing", 0.35, 0.55, 0.03, 1.1),
    B.TankSpec("dambreak", 0.42, 0.70, 0.0, 0.0),
    B.TankSpec("sloshing", 0.30, 0.80, 0.05, 0.9),
    B.TankSpec("dambreak", 0.36, 0.60, 0.0, 0.0),
    B.TankSpec("sloshing", 0.48, 0.50, 0.01, 1.7),
]
FIELDS = ["Position", "Velocity", "density", "DynamicPressure", "ddensitydt", "dvdt"]


def _run_batch(batch, steps, precision=0, graph=0, tuning=None):
    from uph_b200.sim import Simulation
    s = Simulation.from_deck(batch.deck, profile=1, precision=precision)
    if batch.wall_x0.size:
        s.set_wall_motion(batch.wall_x0, batch.wall_hs, batch.wall_om)
    if tuning:
        s.set_tuning(*tuning)
    if graph:
        s.step(1)
        s.set_graph(graph)
        for _ in range((steps - 1) // graph):
            s.step(graph)
        rest = (steps - 1) % graph
        if rest:
            s.step(rest)
    else:
        s.step(steps)
    st = s.download()
    s.close()
    return st


def _run_tank(batch, k, steps, precision=0):
    from uph_b200.sim import Simulation
    d, table = B.tank_deck(batch, k)
    s = Simulation.from_deck(d, profile=1, precision=precision)
    if table is not None:
        s.set_wall_motion(*table)
    s.step(steps)
    st = s.download()
    s.close()
    return d, st


def test_batch_matches_tanks_run_alone():
    batch = B.build_batch(SMALL)
    steps = 100
    st = _run_batch(batch, steps)
    for k in range(len(SMALL)):
        d, alone = _run_tank(batch, k, steps)
        f0, f1 = batch.fluid_ranges[k]
        got = {f: st[f][f0:f1] for f in FIELDS}
        compare_fields(got, alone, d.n_fluid, 1e-9, fields=FIELDS)


def test_sloshing_batch_matches_oracle():
    batch = B.build_batch(SMALL[:2])
    steps = 20
    o = O.Oracle(batch.deck.uph_params(profile=1), batch.deck.initial_state())
    o.set_wall_motion(batch.wall_x0, batch.wall_hs, batch.wall_om)
    o.step(steps)
    st = _run_batch(batch, steps)
    want = o.state()
    compare_fields(st, want, batch.deck.n_fluid, 1e-10, fields=FIELDS)
    # the shaken walls are where the table puts them
    m0 = batch.deck.n_fluid + batch.deck.fixed.shape[0]
    assert rel_err(st["Position"][m0:], want["Position"][m0:]) <= 1e-14


def test_graph_replay_matches_plain_stepping():
    """Graph windows re-sort the storage on their own schedule, so sums run in
    a different order: FP64 agreement far below the parity bar."""
    batch = B.build_batch(SMALL)
    a = _run_batch(batch, 161, precision=0, graph=40)
    b = _run_batch(batch, 161, precision=0, graph=0)
    compare_fields(a, b, batch.deck.n_fluid, 1e-9, fields=FIELDS)


def test_tuning_changes_nothing_but_speed():
    batch = B.build_batch(SMALL)
    a = _run_batch(batch, 60, tuning=(1, 4, 8))
    b = _run_batch(batch, 60, tuning=(3, 16, 32))
    compare_fields(a, b, batch.deck.n_fluid, 1e-9, fields=FIELDS)


def test_autotune_choice_and_cache():
    from uph_b200.sim import Simulation
    batch = B.build_batch(SMALL)
    s = Simulation.from_deck(batch.deck, profile=1, precision=1)
    s.set_wall_motion(batch.wall_x0, batch.wall_hs, batch.wall_om)
    choice, ms = s.autotune(trial_steps=5)
    assert choice[0] in (1, 2, 3) and choice[1] in (9, 11, 13) and choice[2] in (16, 64, 256)
    assert ms > 0.0
    s.step(10)
    assert np.all(np.isfinite(s.download()["Position"]))
    s.close()
    s2 = Simulation.from_deck(batch.deck, profile=1, precision=1)
    choice2, ms2 = s2.autotune(trial_steps=5)
    assert choice2 == choice and ms2 == 0.0  # same size class: taken from the cache
    s2.close()


def test_fp32_batch_against_fp64_tanks():
    """The batched FP32-pair run against each tank's FP64 run after 200
    steps: density within 1 % of rho0, free-surface height within 2 % of the
    column height."""
    batch = B.build_batch(SMALL)
    steps = 200
    st = _run_batch(batch, steps, precision=1, graph=50)
    rho0 = batch.deck.params["density0"]
    dx = batch.deck.params["dx"]
    for k, spec in enumerate(SMALL):
        d, alone = _run_tank(batch, k, steps)
        f0, f1 = batch.fluid_ranges[k]
        drho = np.abs(st["density"][f0:f1] - alone["density"][:d.n_fluid]).max() / rho0
        assert drho <= 0.01, f"tank {k}: density error {drho:.2e}"
        x0 = batch.offsets[k][0]
        length = 2.5 * spec.width if spec.kind == "dambreak" else spec.width
        hb = B.free_surface_heights(st["Position"][f0:f1], x0, length, dx)
        ha = B.free_surface_heights(alone["Position"][:d.n_fluid], x0, length, dx)
        err = np.abs(hb - ha).max() / spec.height
        assert err <= 0.02, f"tank {k}: free-surface error {err:.2e}"
