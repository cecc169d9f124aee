"""The resident simulation's diagnostics and output files against the
unmodified reference driver.

The compiled reference (oracle/_ref/sph) runs three steps with print_step 1
and writes out<k>.dat, TotalKineticEnergy.dat, PointPressure.dat,
PointPressureTwo.dat and FluidParticleInit.dat (output.c:19-140).  The
resident simulation runs the same steps on the GPU with its per-evaluation
diagnostics on (kinetic energy and pressure probes at the state each
derivatives() call sees) and writes the same files through
uph_write_output.  Values must agree to the last printed decimal; the
columns this path writes as 0 (approxVorticity, specificDissipationRate,
tempPosition, tempPositionGate) are left out."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from _util import deck_from_golden, load_golden, ref_env
from oracle import oracle as O
from uph_b200._capi import PREC_FP64, PROFILE_REF

pytestmark = pytest.mark.gpu

SPH = os.path.join(O.REF_DIR, "sph")
OUT_COLUMNS = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 11, 13]
INIT_COLUMNS = [0, 1, 2, 3, 4, 5, 6, 9, 10, 11]


def _decks():
    from uph_b200 import deck as D
    yield "tank_nn19", deck_from_golden(load_golden("tank_nn19"))
    d = D.wave_flume(length=7.6, depth=0.2, dx=0.04, layers=2, amplitude=0.02, period=1.2, eta=0.0,
                     near_neighbor=21)
    rng = np.random.default_rng(4)
    d.fluid[:, 2:4] = rng.uniform(-0.02, 0.02, size=(d.n_fluid, 2))
    yield "flume_nn21", d


def _close(a, b):
    # 10 printed decimals: one unit in the last place
    assert a.shape == b.shape
    assert np.max(np.abs(a - b)) <= 1.5e-10 * max(1.0, np.max(np.abs(a))), np.max(np.abs(a - b))


@pytest.mark.parametrize("case,deck", list(_decks()), ids=lambda v: v if isinstance(v, str) else "")
def test_resident_output_matches_reference_driver(case, deck):
    from uph_b200.sim import Simulation
    if not os.path.exists(SPH):
        pytest.skip(f"{SPH} not built (make -C oracle ref)")
    assert not deck.eta_override
    deck.params["print_step"] = 1
    deck.params["screen_step"] = 1000
    deck.params["number_of_initialization_steps"] = 2
    fl = deck.fluid
    deck.params["pressure_probe_x"] = float(np.median(fl[:, 0]))
    deck.params["pressure_probe_y"] = float(fl[:, 1].min() + 0.25 * np.ptp(fl[:, 1]))
    with tempfile.TemporaryDirectory() as ref_dir, tempfile.TemporaryDirectory() as gpu_dir:
        deck.write(ref_dir)
        r = subprocess.run([SPH, "3"], cwd=ref_dir, capture_output=True, text=True, timeout=300, env=ref_env())
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        gate = deck.dam_gate_flag()
        with Simulation.from_deck(deck, PROFILE_REF, PREC_FP64) as sim:
            sim.set_diagnostics(True)
            for k in (1, 2, 3):
                sim.step(1)
                d = sim.diagnostics()
                assert d["itime"] == k
                sim.write_output(gpu_dir, k, dam_gate_flag=gate)
        for k in (1, 2, 3):
            a = np.loadtxt(os.path.join(ref_dir, f"out{k}.dat"))[:, OUT_COLUMNS]
            b = np.loadtxt(os.path.join(gpu_dir, f"out{k}.dat"))[:, OUT_COLUMNS]
            _close(a, b)
        for name in ("TotalKineticEnergy.dat", "PointPressure.dat", "PointPressureTwo.dat"):
            a = np.loadtxt(os.path.join(ref_dir, name), ndmin=2)
            b = np.loadtxt(os.path.join(gpu_dir, name), ndmin=2)
            assert a.shape[0] == 3
            _close(a, b)
        pp = np.loadtxt(os.path.join(ref_dir, "PointPressure.dat"), ndmin=2)
        assert np.all(pp[:, 2] > 0)  # the first probe sits in the water
        a = np.loadtxt(os.path.join(ref_dir, "FluidParticleInit.dat"), skiprows=1)[:, INIT_COLUMNS]
        b = np.loadtxt(os.path.join(gpu_dir, "FluidParticleInit.dat"), skiprows=1)[:, INIT_COLUMNS]
        _close(a, b)


def test_diagnostics_follow_graph_replay_and_toggle():
    """Diagnostics inside replayed CUDA graphs equal those of plain calls, and
    turning them off makes the query fail instead of returning stale data."""
    from uph_b200 import deck as D
    from uph_b200._lib import UphError
    from uph_b200.sim import Simulation
    deck = D.dam_break(dx=0.02, hydrostatic=True)
    out = []
    for graph in (0, 4):
        with Simulation.from_deck(deck, PROFILE_REF, PREC_FP64) as sim:
            sim.set_diagnostics(True, probe=(0.1, 0.05))
            sim.set_graph(graph)
            vals = []
            for _ in range(3):
                sim.step(4)
                vals.append(sim.diagnostics())
            out.append(vals)
            sim.set_diagnostics(False)
            with pytest.raises(UphError, match="UPH_BAD_ARG"):
                sim.diagnostics()
    assert [v["itime"] for v in out[0]] == [4, 8, 12]
    for a, b in zip(*out):
        assert a == b
    assert out[0][-1]["point_neighbors"] > 0 and out[0][-1]["kinetic_energy"] > 0
