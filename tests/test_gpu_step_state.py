"""The step-to-step state: a loop that uploads only sim.STEP_INPUT_FIELDS and
downloads only sim.STEP_OUTPUT_FIELDS (the end-to-end pattern of bench.py)
advances exactly like one that moves the whole uph_state every step, on a
piston flume (moving walls) in the REF profile."""
import numpy as np
import pytest

from uph_b200 import deck as D

pytestmark = pytest.mark.gpu


def test_step_fields_round_trip_matches_full_state():
    from uph_b200._capi import empty_state
    from uph_b200.sim import STEP_INPUT_FIELDS, STEP_OUTPUT_FIELDS, Simulation

    deck = D.wave_flume(length=1.5, depth=0.2, dx=0.02, layers=2, amplitude=0.02, period=1.2)
    init = deck.initial_state()
    nf, n = deck.n_fluid, deck.n_all
    finals = []
    for lean in (False, True):
        with Simulation.from_deck(deck) as s:
            s.upload(init, 0)
            s.step(1)
            if lean:
                out = {k: v for k, v in empty_state(nf, n).items() if k in STEP_OUTPUT_FIELDS}
            else:
                out = empty_state(nf, n)
            s.download(out)
            for itime in range(1, 6):
                if lean:
                    upl = {k: (out[k] if k in out else init[k]) for k in STEP_INPUT_FIELDS}
                else:
                    upl = out
                s.upload(upl, itime)
                s.step(1)
                s.download(out)
            finals.append({k: out[k].copy() for k in STEP_OUTPUT_FIELDS})
    full, lean = finals
    for k in STEP_OUTPUT_FIELDS:
        assert np.array_equal(full[k], lean[k]), k
    assert np.abs(full["Velocity"][:nf]).max() > 0
