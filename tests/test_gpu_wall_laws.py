"""The lid (movingBoundary 3) and gate (movingBoundary 2) wall laws of the
reference's inputbp (inputbp.c:209-243) on the resident GPU path, against the
reference's solver compiled from its sources on the same decks: all 17 fluid
fields within 1e-10 after steps 1 and 3, and the moving particles where the
laws put them."""
import os
import tempfile

import numpy as np
import pytest

from _util import FLUID_FIELDS, REL_TOL_FP64, compare_fields
from oracle import oracle as O
from uph_b200 import deck as D

pytestmark = pytest.mark.gpu

DECKS = {
    "lid_cavity": lambda: D.lid_cavity(size=0.4, dx=0.02, layers=2, lid_velocity=1.0),
    "gate_dam_break": lambda: D.gate_dam_break(tank=(1.0, 0.6), column=(0.3, 0.4), dx=0.02, layers=2,
                                               gate_velocity=1.0),
}


@pytest.mark.parametrize("name", sorted(DECKS))
def test_wall_law_matches_compiled_reference(name):
    if not os.path.exists(os.path.join(O.REF_DIR, "libuph_ref.so")):
        pytest.skip("oracle/_ref/libuph_ref.so not built (make -C oracle ref)")
    from uph_b200.sim import Simulation

    deck = DECKS[name]()
    nf, n = deck.n_fluid, deck.n_all
    m0 = n - deck.moving.shape[0]
    with tempfile.TemporaryDirectory() as tmp:
        deck.write(tmp)
        run = O.RefRun(tmp, eta_override=deck.eta_override)
        try:
            run.step(1)
            ref1 = {f: run.get(f) for f in FLUID_FIELDS}
            run.step(2)
            ref3 = {f: run.get(f) for f in FLUID_FIELDS}
            ref_walls = run.get("Position", m0, n - m0)
        finally:
            run.close()
    with Simulation.from_deck(deck) as s:
        s.step(1)
        compare_fields(s.download(), ref1, nf, REL_TOL_FP64)
        s.step(2)
        st = s.download()
        compare_fields(st, ref3, nf, REL_TOL_FP64)
    # the walls at the third step's evaluation time, t = 3 dt
    t = 3 * deck.params["time_step"]
    U = deck.params["lid_velocity"]
    want = deck.moving[:, 0:2].copy()
    if name == "lid_cavity":
        want[:, 0] = deck.moving[:, 7] + U * t
    else:
        want[:, 1] = deck.moving[:, 8] + U * t
    assert np.allclose(st["Position"][m0:], want, rtol=0, atol=1e-15)
    assert np.allclose(ref_walls, want, rtol=0, atol=1e-15)
