"""Pins the CPU oracle: the restatement oracle/uph_oracle.c against the golden
vectors produced by the reference's own solver (tests/golden/), and the
golden vectors against a fresh run of the compiled reference."""
import os
import tempfile

import numpy as np
import pytest

from _util import FLUID_FIELDS, GOLDEN_CASES, compare_fields, deck_from_golden, load_golden, rel_err
from oracle import oracle as O
from uph_b200 import deck as D

# the restatement keeps the reference's expressions and loop order, so it
# agrees far below the product's 1e-10 bar
ORACLE_TOL = 1e-13


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_oracle_matches_reference_golden(case):
    g = load_golden(case)
    deck = deck_from_golden(g)
    o = O.Oracle(deck.uph_params(), deck.initial_state())
    o.step(1)
    s1 = o.state()
    want1 = {f: g[f"s1_{f}"] for f in FLUID_FIELDS}
    compare_fields(s1, want1, deck.n_fluid, ORACLE_TOL)
    i, j, r2, w, dw = o.pairs()
    assert np.array_equal(i, g["s1_i_pair"]) and np.array_equal(j, g["s1_j_pair"])
    assert np.array_equal(r2, g["s1_rij2"]), "rij2 must be bit-identical"
    assert rel_err(w, g["s1_w"]) <= 1e-15
    assert rel_err(dw, g["s1_dwcdx"]) <= 1e-15
    o.step(2)
    s3 = o.state()
    compare_fields(s3, {f: g[f"s3_{f}"] for f in FLUID_FIELDS}, deck.n_fluid, ORACLE_TOL)


def _ref_available():
    return os.path.exists(os.path.join(O.REF_DIR, "libuph_ref.so"))


@pytest.mark.skipif(not _ref_available(), reason="compiled reference (oracle/_ref/libuph_ref.so) not built")
@pytest.mark.parametrize("case", ["dambreak_h13", "flume_piston_sponge", "fluid_only"])
def test_golden_reproduces_with_compiled_reference(case):
    """The committed fixtures are what the compiled reference produces now."""
    g = load_golden(case)
    deck = deck_from_golden(g)
    with tempfile.TemporaryDirectory() as tmp:
        deck.write(tmp)
        run = O.RefRun(tmp, eta_override=deck.eta_override)
        run.step(1)
        for f in FLUID_FIELDS:
            assert rel_err(run.get(f), g[f"s1_{f}"]) <= 1e-14, f
        i, j = run.pairs()
        assert np.array_equal(i, g["s1_i_pair"]) and np.array_equal(j, g["s1_j_pair"])
        run.close()


@pytest.mark.skipif(not _ref_available(), reason="compiled reference not built")
def test_reference_capacity_patch_changes_nothing():
    """The harness's smaller particle capacity (fluid_capacity_pct) leaves every
    result identical to the reference's own 100 Nf capacity."""
    g = load_golden("dambreak_h13")
    deck = deck_from_golden(g)
    with tempfile.TemporaryDirectory() as tmp:
        deck.write(tmp)
        a = O.RefRun(tmp, eta_override=deck.eta_override)
        b = O.RefRun(tmp, eta_override=deck.eta_override, fluid_capacity_pct=16)
        assert b.counts()["max_n"] < a.counts()["max_n"]
        a.step(2)
        b.step(2)
        for f in FLUID_FIELDS:
            assert np.array_equal(a.get(f), b.get(f)), f
        a.close()
        b.close()


def test_oracle_search_brute_force():
    """Radius search with the reference's filter against an O(n^2) scan."""
    rng = np.random.default_rng(5)
    n, nf = 700, 500
    pos = rng.uniform(0, 1, size=(n, 2))
    pos[10] = pos[11]  # a coincident pair: libnabo never returns d2 <= DBL_EPSILON
    dist = 0.06 ** 2
    pb = n - 1
    i, j, r2, mx = O.search(pos, nf, pb, dist)
    want = []
    for s in range(nf):
        for t in range(s + 1, pb):
            d = pos[s] - pos[t]
            d2 = d[0] * d[0] + d[1] * d[1]
            if np.finfo(float).eps < d2 < dist:
                want.append((s, t))
    assert list(zip(i.tolist(), j.tolist())) == want
    assert (10, 11) not in want


def test_wcsph_oracle_conserves_mass_and_momentum_pairwise():
    """The WCSPH restatement's pair forces are antisymmetric: without walls,
    gravity and wall forces the total momentum rate is zero."""
    deck = D.dam_break(tank=(0.4, 0.4), column=(0.2, 0.2), dx=0.02, hydrostatic=True, gravity_flag=0)
    deck.fixed = np.zeros((0, 12))
    rng = np.random.default_rng(3)
    deck.fluid[:, 2:4] = rng.uniform(-0.1, 0.1, size=(deck.n_fluid, 2))
    p = deck.uph_params(profile=1)
    o = O.Oracle(p, deck.initial_state())
    o.derivatives(0.0)
    s = o.state()
    m = s["mass"][:deck.n_fluid]
    mom = (m[:, None] * s["dvdt"]).sum(axis=0)
    scale = np.abs(m[:, None] * s["dvdt"]).sum()
    assert np.all(np.abs(mom) <= 1e-12 * scale)
