"""Virtual mirror particles (derivatives.c:3194-4192) against the reference's
solver compiled from its sources.

The reference appends, every call, mirror copies of the fluid particles near
each wall line of the virtualType; they are points of its 40-nearest search
(so they can take a query's places) but never in a pair (j < Nf + Ns + Nb -
1).  The decks here make them matter: a still tank filling [0, W] x [0, D]
with FlatBottomLength = W and LocalDepth = D, so that the left, right,
bottom, top and corner mirrors all fire, and nearNeighbor 91 (a smoothing
length of 2.7 spacings), so that the 40-nearest cap binds and mirror points
do take places.  Type 1's slope starts inside the tank (FlatBottomLength
0.75 W) so that its mirror fires too.

Bars: the virtual particles' count and positions bit-identical; the step-1
pair list bit-identical; all 17 fluid fields within 1e-10 after step 1; and
the same pair set differs from the one without mirrors (they are exercised).
The drop-in's System rows are checked in test_gpu_dropin.py."""
import os
import tempfile

import numpy as np
import pytest

from _util import FLUID_FIELDS, REL_TOL_FP64, compare_fields
from oracle import oracle as O
from uph_b200 import deck as D

pytestmark = pytest.mark.gpu

TYPES = [1, 3, 4, 5, 7, 8]


def _deck(vt):
    d = D.hydrostatic_tank(width=0.4, depth=0.3, dx=0.02, layers=2, eta=0.0)
    d.params["near_neighbor"] = 91
    d.params["virtual_type"] = vt
    d.params["flat_bottom_length"] = 0.3 if vt == 1 else 0.4
    d.params["local_depth"] = 0.3
    return d


@pytest.mark.parametrize("vt", TYPES)
def test_virtual_particles_match_compiled_reference(vt):
    if not os.path.exists(os.path.join(O.REF_DIR, "libuph_ref.so")):
        pytest.skip("oracle/_ref/libuph_ref.so not built (make -C oracle ref)")
    from uph_b200.sim import Simulation

    deck = _deck(vt)
    nb = deck.n_all
    with tempfile.TemporaryDirectory() as tmp:
        deck.write(tmp)
        run = O.RefRun(tmp, eta_override=deck.eta_override)
        try:
            run.derivatives(deck.params["time_step"])
            nv = run.counts()["n_virtual"]
            vpos = run.get("Position", nb, nv)
            ri, rj = run.pairs()
            capped = run.truncated_queries()
        finally:
            run.close()
        run = O.RefRun(tmp, eta_override=deck.eta_override)
        try:
            run.step(1)
            ref1 = {f: run.get(f) for f in FLUID_FIELDS}
        finally:
            run.close()
    assert nv > 0 and capped > 0
    with Simulation.from_deck(deck, knn_cap=40) as s:
        s.derivatives(deck.params["time_step"])
        pos, src, kind = s.virtual()
        i, j, _, _, _ = s.pairs()
    assert pos.shape[0] == nv, f"{pos.shape[0]} virtual particles against the reference's {nv}"
    assert np.array_equal(pos, vpos), "virtual positions differ"
    assert np.array_equal(i, ri) and np.array_equal(j, rj), "capped pair list differs"
    with Simulation.from_deck(deck, knn_cap=40) as s:
        s.step(1)
        e1 = compare_fields(s.download(), ref1, deck.n_fluid, REL_TOL_FP64)
    deck.params["virtual_type"] = 77
    with Simulation.from_deck(deck, knn_cap=40) as s:
        s.derivatives(deck.params["time_step"])
        i0, j0, _, _, _ = s.pairs()
    assert not (np.array_equal(i0, ri) and np.array_equal(j0, rj)), "the mirrors changed no pair"
    print(f"virtualType {vt}: {nv} virtual particles ({sorted(set(kind.tolist()))}), {ri.size} capped pairs "
          f"bit-identical ({i0.size} without mirrors); max field error step 1 {max(e1.values()):.2e}")
