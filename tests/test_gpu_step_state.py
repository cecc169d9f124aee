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


def _fused_cases():
    from uph_b200._capi import PREC_FP32_PAIR, PREC_FP64, PROFILE_REF, PROFILE_WCSPH

    flume = D.wave_flume(length=1.5, depth=0.2, dx=0.02, layers=2, amplitude=0.02, period=1.2)
    # piston flume: moving walls, the sponge layer; graph replays and
    # frequent storage re-sorts in between; both profiles and precisions
    yield "flume_piston_ref", flume, PROFILE_REF, PREC_FP64, 0
    yield "flume_piston_wcsph_fp64", flume, PROFILE_WCSPH, PREC_FP64, 0
    yield "flume_piston_wcsph_fp32", flume, PROFILE_WCSPH, PREC_FP32_PAIR, 0
    # the lid of a driven cavity (movingBoundary 3) under the 40-nearest cap
    yield "lid_cavity_ref_knn40", D.lid_cavity(size=0.3, dx=0.015, layers=2), PROFILE_REF, PREC_FP64, 40
    # h = 1.5 dx: about 28 partners in radius, so the bulk's candidate lists
    # overflow (those particles walk the stencil) while the surface's fit
    yield "dambreak_ref_h15_overflow", D.dam_break(tank=(0.6, 0.5), column=(0.2, 0.3), dx=0.01, eta=1.5), \
        PROFILE_REF, PREC_FP64, 0


@pytest.mark.parametrize("case,deck,profile,precision,knn", list(_fused_cases()),
                         ids=lambda v: v if isinstance(v, str) else "")
def test_fused_step_matches_separate_corrector(case, deck, profile, precision, knn):
    """The rate pass that applies the leapfrog step in its epilogue (writing
    the other state buffer) leaves every field bit-identical to the pass
    followed by the stand-alone corrector, and the passes' per-particle
    candidate lists leave it bit-identical to walking the cell stencil at
    every pass, through multi-step calls, graph replays, storage re-sorts and
    downloads in between."""
    from uph_b200._capi import empty_state
    from uph_b200.sim import Simulation

    nf, n = deck.n_fluid, deck.n_all
    runs = []
    for fused, lists in ((False, True), (True, True), (True, False)):
        with Simulation.from_deck(deck, profile=profile, precision=precision, knn_cap=knn) as s:
            s.set_fused_step(fused)
            s.set_candidate_lists(lists)
            s.set_tuning(2, 8, 3)
            states = []
            for k, nsteps in enumerate([1, 4, 4, 3, 4, 1, 4]):
                if k == 2:
                    s.set_graph(4)
                s.step(nsteps)
                out = empty_state(nf, n)
                s.download(out)
                states.append(out)
            runs.append(states)
    for other in runs[1:]:
        for k, (a, b) in enumerate(zip(runs[0], other)):
            for f in a:
                assert np.array_equal(a[f], b[f], equal_nan=True), (k, f)
    last = runs[1][-1]
    assert np.abs(last["Velocity"][:nf]).max() > 0
