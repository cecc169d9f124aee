"""uph_write_output against the reference's own output() (output.c:19-140).

The compiled reference (oracle/_ref/sph, built from its sources) runs a small
tank for two steps and prints its snapshots and diagnostics files.  Those
values, read back and written again through uph_write_output, must give the
same files character for character -- except the approxVorticity and
specificDissipationRate columns of out<k>.dat and the tempPosition /
tempPositionGate columns of FluidParticleInit.dat, which this path writes
as 0.  No GPU is involved: the writer is host code."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from _util import deck_from_golden, load_golden, ref_env
from oracle import oracle as O
from uph_b200._capi import empty_state
from uph_b200.sim import write_output

SPH = os.path.join(O.REF_DIR, "sph")


def _fields(line):
    """[field, separator, field, ...] of one text line (separators kept)."""
    return re.split(r"(\s+)", line.rstrip("\n"))


def _zero_columns(text, columns):
    out = []
    for line in text.splitlines(keepends=True):
        parts = _fields(line)
        vals = parts[0::2]
        if len(vals) > max(columns):
            for c in columns:
                parts[2 * c] = "0.0000000000"
        out.append("".join(parts) + "\n")
    return "".join(out)


def _read(path):
    with open(path) as f:
        return f.read()


def _case():
    deck = deck_from_golden(load_golden("tank_nn19"))
    deck.params["print_step"] = 1
    deck.params["screen_step"] = 1000
    deck.params["number_of_initialization_steps"] = 2
    fl = deck.fluid
    deck.params["pressure_probe_x"] = float(np.median(fl[:, 0]))
    deck.params["pressure_probe_y"] = float(fl[:, 1].min() + 0.25 * np.ptp(fl[:, 1]))
    return deck


def test_writer_reproduces_reference_files():
    if not os.path.exists(SPH):
        pytest.skip(f"{SPH} not built (make -C oracle ref)")
    deck = _case()
    assert not deck.eta_override
    params = deck.uph_params()
    nf, n = deck.n_fluid, deck.n_all
    with tempfile.TemporaryDirectory() as ref_dir, tempfile.TemporaryDirectory() as out_dir:
        deck.write(ref_dir)
        r = subprocess.run([SPH, "2"], cwd=ref_dir, capture_output=True, text=True, timeout=300, env=ref_env())
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        ke = np.loadtxt(os.path.join(ref_dir, "TotalKineticEnergy.dat"), ndmin=2)
        pp = np.loadtxt(os.path.join(ref_dir, "PointPressure.dat"), ndmin=2)
        pp2 = np.loadtxt(os.path.join(ref_dir, "PointPressureTwo.dat"), ndmin=2)
        assert ke.shape[0] == pp.shape[0] == pp2.shape[0] == 2
        assert int(pp[1, 2]) > 0  # the probe sits in the water
        init = np.loadtxt(os.path.join(ref_dir, "FluidParticleInit.dat"), skiprows=1)
        for k in (1, 2):
            tab = np.loadtxt(os.path.join(ref_dir, f"out{k}.dat"))
            assert tab.shape == (n, 14)
            assert np.all(tab[:, 7] == round(params["h"], 10))
            st = empty_state(nf, n)
            st["Position"][:] = tab[:, 1:3]
            st["Velocity"][:] = tab[:, 3:5]
            st["density"][:] = tab[:, 5]
            st["mass"][:] = tab[:, 6]
            st["DynamicPressure"][:] = tab[:, 8]
            st["itype"][:] = tab[:, 11].astype(np.int32)
            st["localDensity"][:] = tab[:, 13]
            if k == 2:
                st["localVelocity"][:nf] = init[:, 10:12]
            diag = dict(kinetic_energy=ke[k - 1, 1], potential_energy=ke[k - 1, 2], point_pressure=pp[k - 1, 1],
                        point_neighbors=int(pp[k - 1, 2]), pressure_norm=pp[k - 1, 3],
                        point_pressure_two=pp[k - 1, 4], point_neighbors_two=int(pp2[k - 1, 1]), itime=k)
            write_output(out_dir, params, st, diag, k, tab[:, 9].astype(np.int32))
            want = _zero_columns(_read(os.path.join(ref_dir, f"out{k}.dat")), [10, 12])
            assert _read(os.path.join(out_dir, f"out{k}.dat")) == want
        for name in ("TotalKineticEnergy.dat", "PointPressure.dat", "PointPressureTwo.dat"):
            assert _read(os.path.join(out_dir, name)) == _read(os.path.join(ref_dir, name)), name
        want = _read(os.path.join(ref_dir, "FluidParticleInit.dat"))
        got = _read(os.path.join(out_dir, "FluidParticleInit.dat"))
        assert got == _zero_columns(want, [7, 8])


def test_writer_rejects_missing_fields_and_bad_directory():
    from uph_b200._lib import UphError
    deck = _case()
    st = deck.initial_state()
    diag = dict(kinetic_energy=0.0, potential_energy=0.0, point_pressure=0.0, pressure_norm=1.0,
                point_pressure_two=0.0, point_neighbors=0, point_neighbors_two=0, itime=0)
    with tempfile.TemporaryDirectory() as tmp:
        with pytest.raises(UphError, match="UPH_IO_ERROR"):
            write_output(os.path.join(tmp, "missing", "dir"), deck.uph_params(), st, diag, 1)
        del st["mass"]
        with pytest.raises(UphError, match="UPH_BAD_ARG"):
            write_output(tmp, deck.uph_params(), st, diag, 1)


def test_dam_gate_flag_follows_input():
    deck = _case()
    flag = deck.dam_gate_flag()
    assert flag.shape == (deck.n_all,)
    assert np.all(flag[deck.n_fluid:] == 0)
    assert np.array_equal(flag[:deck.n_fluid] == 1, deck.fluid[:, 0] <= 0.38)
