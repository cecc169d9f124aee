"""Particle-packing initialisation (flagInitSimul == 0; derivatives.c:2948-3066,
4279-4288) against the reference's solver compiled from its sources.

In place of the physics the reference relaxes the particle arrangement: a
kernel-sum gradient per fluid particle, a momentum term that every pair of
the particle adds once more, a hydrostatic reset of density and pressure, and
the wall forces; no wall moves (inputbp.c:194-243 require flagInitSimul 1).
A dam break with a disturbed lattice, so that the gradient is not zero.
Bars: all 17 fluid fields within 1e-10 after steps 1 and 3, uncapped and
under the 40-nearest cap."""
import os
import tempfile

import numpy as np
import pytest

from _util import FLUID_FIELDS, REL_TOL_FP64, compare_fields
from oracle import oracle as O
from uph_b200 import deck as D

pytestmark = pytest.mark.gpu


def _deck(capped):
    d = D.dam_break(tank=(1.0, 1.0), column=(0.4, 0.6), dx=0.02, layers=2, hydrostatic=True,
                    eta=0.0 if capped else 1.3)
    if capped:
        d.params["near_neighbor"] = 91
    rng = np.random.default_rng(11)
    d.fluid[:, 0:2] += rng.uniform(-0.002, 0.002, size=(d.n_fluid, 2))
    d.params["flag_init_simul"] = 0
    return d


@pytest.mark.parametrize("capped", [False, True], ids=["h13", "nn91_capped"])
def test_packing_matches_compiled_reference(capped):
    if not os.path.exists(os.path.join(O.REF_DIR, "libuph_ref.so")):
        pytest.skip("oracle/_ref/libuph_ref.so not built (make -C oracle ref)")
    from uph_b200.sim import Simulation

    deck = _deck(capped)
    with tempfile.TemporaryDirectory() as tmp:
        deck.write(tmp)
        run = O.RefRun(tmp, eta_override=deck.eta_override)
        try:
            run.step(1)
            ref1 = {f: run.get(f) for f in FLUID_FIELDS}
            run.step(2)
            ref3 = {f: run.get(f) for f in FLUID_FIELDS}
        finally:
            run.close()
    assert np.abs(ref1["dvdt"]).max() > 0
    with Simulation.from_deck(deck, knn_cap=40 if capped else 0) as s:
        s.step(1)
        e1 = compare_fields(s.download(), ref1, deck.n_fluid, REL_TOL_FP64)
        s.step(2)
        e3 = compare_fields(s.download(), ref3, deck.n_fluid, REL_TOL_FP64)
    print(f"packing ({'capped' if capped else 'uncapped'}): max field error step 1 {max(e1.values()):.2e}, "
          f"step 3 {max(e3.values()):.2e}")
