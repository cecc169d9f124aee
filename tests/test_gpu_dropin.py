"""The drop-in: the reference's own driver (src/bin/sph.cc) and libSPH host
files (input.c, inputbp.c, output.c, ...) relinked against libuph_sph.so in
place of derivatives.c + Search.cc, compared with the unmodified reference;
and the package's own host caller of derivatives() (libuph_driver.so).

Both builds live in oracle/_ref/ (made by `make -C oracle ref dropin` from
the reference's sources); a machine without those sources runs the prebuilt
files."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from _util import FLUID_FIELDS, REL_TOL_FP64, compare_fields, deck_from_golden, load_golden, ref_env, rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SPH = os.path.join(O.REF_DIR, "sph")
SPH_UPH = os.path.join(O.REF_DIR, "sph_uph")
DROPIN = os.path.join(O.REF_DIR, "libuph_dropin.so")


def _need(*paths):
    for p in paths:
        if not os.path.exists(p):
            pytest.skip(f"{p} not built (make -C oracle ref dropin)")


class DropInRun(O.RefRunInProcess):
    """The harness API over the reference host code + libuph_sph.so."""
    _lib = None

    def __init__(self, deck_dir, eta_override=0.0):
        import ctypes as C
        if DropInRun._lib is None:
            lib = C.CDLL(DROPIN)
            lib.ref_open.restype = C.c_void_p
            lib.ref_open.argtypes = [C.c_char_p, C.c_double, C.c_int]
            lib.ref_close.argtypes = [C.c_void_p]
            lib.ref_step.argtypes = [C.c_void_p, C.c_int]
            lib.ref_counts.argtypes = [C.c_void_p, C.c_void_p]
            lib.ref_get.restype = C.c_long
            lib.ref_get.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.c_void_p]
            lib.ref_pairs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
            DropInRun._lib = lib
        self.lib = DropInRun._lib
        self.h = self.lib.ref_open(os.fsencode(deck_dir), eta_override, 0)
        assert self.h


@pytest.mark.parametrize("case", ["dambreak_h13", "flume_piston_sponge", "tank_nn19", "ragged_solid"])
def test_dropin_derivatives_in_reference_driver_loop(case):
    """sph.cc's leapfrog (restated by the harness) calling the GPU
    derivatives() through the System struct, vs the reference's goldens."""
    _need(DROPIN)
    g = load_golden(case)
    deck = deck_from_golden(g)
    with tempfile.TemporaryDirectory() as tmp:
        deck.write(tmp)
        run = DropInRun(tmp, eta_override=deck.eta_override)
        run.step(1)
        got = {f: run.get(f) for f in FLUID_FIELDS}
        compare_fields(got, {f: g[f"s1_{f}"] for f in FLUID_FIELDS}, deck.n_fluid, REL_TOL_FP64)
        i, j = run.pairs()
        assert np.array_equal(i, g["s1_i_pair"]) and np.array_equal(j, g["s1_j_pair"])
        assert np.array_equal(run.get("rij2"), g["s1_rij2"])
        assert rel_err(run.get("w"), g["s1_w"]) <= 1e-13
        run.step(2)
        got = {f: run.get(f) for f in FLUID_FIELDS}
        compare_fields(got, {f: g[f"s3_{f}"] for f in FLUID_FIELDS}, deck.n_fluid, REL_TOL_FP64)
        run.close()


def _out_table(path):
    return np.loadtxt(path)


def _driver_decks():
    from uph_b200 import deck as D
    g = load_golden("tank_nn19")
    yield "tank_nn19", deck_from_golden(g)
    # nearNeighbor 21 gives eta = 1.293, close to the workloads' 1.3, without an override
    d = D.wave_flume(length=7.6, depth=0.2, dx=0.04, layers=2, amplitude=0.02, period=1.2, eta=0.0,
                     near_neighbor=21)
    rng = np.random.default_rng(4)
    d.fluid[:, 2:4] = rng.uniform(-0.02, 0.02, size=(d.n_fluid, 2))
    yield "flume_nn21", d
    # virtual mirror particles (virtualType 7) under a binding 40-nearest cap:
    # out<k>.dat prints the mirror rows the drop-in writes back
    t = D.hydrostatic_tank(width=0.4, depth=0.3, dx=0.02, layers=2, eta=0.0)
    t.params.update(near_neighbor=91, virtual_type=7, flat_bottom_length=0.4, local_depth=0.3)
    yield "tank_virtual7_nn91", t
    # particle packing (flagInitSimul 0) on a disturbed lattice
    k = D.dam_break(tank=(1.0, 1.0), column=(0.4, 0.6), dx=0.02, layers=2, hydrostatic=True, eta=0.0,
                    near_neighbor=21)
    k.fluid[:, 0:2] += np.random.default_rng(11).uniform(-0.002, 0.002, size=(k.n_fluid, 2))
    k.params["flag_init_simul"] = 0
    yield "dambreak_packing_nn21", k


# output.c:46-60 columns: i x y u v density mass hsml p damGateFlag approxVorticity
# itype specificDissipationRate localDensity.  specificDissipationRate (12) is
# left out: ComputeSpecificDissipationRate (derivatives.c:2573-2628, called at
# :4269) adds every call's bulk dissipation into it without resetting, a
# running sum over all calls that feeds no state, which the drop-in does not
# keep (it writes 0).
OUT_COLUMNS = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 13]


@pytest.mark.parametrize("case,deck", list(_driver_decks()), ids=lambda v: v if isinstance(v, str) else "")
def test_unmodified_sph_driver_with_dropin_library(case, deck):
    """The reference's own `sph` executable, relinked against the GPU
    library, writes the same out<step>.dat snapshots (10 decimals,
    output.c:46-60) and energy series as the unmodified reference."""
    _need(SPH, SPH_UPH)
    deck.params["print_step"] = 1
    deck.params["screen_step"] = 1000
    assert not deck.eta_override
    tables = []
    for exe in (SPH, SPH_UPH):
        with tempfile.TemporaryDirectory() as tmp:
            deck.write(tmp)
            r = subprocess.run([exe, "3"], cwd=tmp, capture_output=True, text=True, timeout=300, env=ref_env())
            assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
            tables.append([_out_table(os.path.join(tmp, f"out{k}.dat"))[:, OUT_COLUMNS] for k in (1, 2, 3)] +
                          [_out_table(os.path.join(tmp, "TotalKineticEnergy.dat"))])
    ref, gpu = tables
    for a, b in zip(ref, gpu):
        assert a.shape == b.shape
        # 10 printed decimals: allow one unit in the last place
        assert np.max(np.abs(a - b)) <= 1.5e-10 * max(1.0, np.max(np.abs(a)))


@pytest.mark.parametrize("case,pair_export", [("dambreak_h13", 2), ("flume_piston_sponge", 0), ("ragged_solid", 1)])
def test_driver_library_with_dropin(case, pair_export):
    """libuph_driver.so (the package's own host caller: sph.cc's leapfrog on
    the host around the drop-in derivatives()) against the reference's
    goldens after steps 1 and 3, with every pair-export level; the exported
    pair arrays equal the reference's where they are exported."""
    from uph_b200.dropin import DropInRun

    g = load_golden(case)
    deck = deck_from_golden(g)
    st = deck.initial_state()
    with DropInRun(deck.uph_params(), st, pair_export=pair_export) as run:
        run.step(1)
        compare_fields(run.state(), {f: g[f"s1_{f}"] for f in FLUID_FIELDS}, deck.n_fluid, REL_TOL_FP64)
        run.step(2)
        compare_fields(run.state(), {f: g[f"s3_{f}"] for f in FLUID_FIELDS}, deck.n_fluid, REL_TOL_FP64)
