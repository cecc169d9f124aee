"""CPU checks of the C ABI: the libraries load, export every declared
symbol, and their host-only entry points (parameters, decks, errors) work
without a GPU."""
import ctypes as C
import os
import re
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import oracle as O
from uph_b200 import _lib
from uph_b200 import deck as D
from uph_b200._capi import UphParams, empty_state, state_struct

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b((?:uph_\w+|derivatives|SearchNeighbors))\s*\(", text)))


def _exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_libuph_exports_every_declared_symbol():
    names = _declared("uph.h") + _declared("uph_surrogate.h")
    assert len(names) >= 30
    exported = _exported(_lib.LIB_PATH)
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    l = _lib.lib()  # loads and binds every signature
    for n in names:
        assert hasattr(l, n)
        assert n in _lib.SIGNATURES, n


def test_libuph_sph_exports_dropin_symbols():
    names = _declared("uph_system.h")
    assert names == ["SearchNeighbors", "derivatives", "uph_dropin_set_callbacks", "uph_dropin_set_pair_export"]
    assert set(names) <= _exported(_lib.LIB_SPH_PATH)


def test_libuph_driver_exports_its_symbols():
    names = _declared("uph_driver.h")
    assert names == ["uph_driver_create", "uph_driver_destroy", "uph_driver_state", "uph_driver_step"]
    exported = _exported(_lib.LIB_DRIVER_PATH)
    assert set(names) <= exported
    # its wall callbacks are handed to the drop-in, not exported under the
    # libSPH names a caller's own libSPH defines
    assert not {"inputbp", "inoutflow"} & exported


def test_status_strings():
    l = _lib.lib()
    assert l.uph_status_string(0) == b"UPH_OK"
    assert l.uph_status_string(2) == b"UPH_OUT_OF_DOMAIN"
    assert l.uph_status_string(10) == b"UPH_IO_ERROR"


def test_params_from_file_matches_python_derivation():
    deck = D.dam_break(dx=0.05, hydrostatic=True)
    with tempfile.TemporaryDirectory() as tmp:
        deck.write(tmp)
        p = UphParams()
        _lib.check(_lib.lib().uph_params_from_file(os.path.join(tmp, "parameters.dat").encode(), 1.3, C.byref(p)),
                   "params")
    want = D.derive_params(deck.params, 1.3)
    for k in ["speed_of_sound", "compression_factor", "omega", "eta", "h", "time_step", "density0",
              "spring_constant0", "thermal_diffusivity0", "lennard_coefficient"]:
        assert getattr(p, k) == pytest.approx(want[k], rel=0, abs=0), k
    assert p.select_boundary_force == 3 and p.stress_type == 1 and p.virtual_type == 77


def test_params_missing_file_is_io_error():
    p = UphParams()
    st = _lib.lib().uph_params_from_file(b"/nonexistent/parameters.dat", 0.0, C.byref(p))
    assert st == 10
    assert b"parameters" in _lib.lib().uph_last_error()


def test_deck_read_matches_python_initial_state():
    deck = D.wave_flume(length=1.0, depth=0.2, dx=0.05, layers=2)
    with tempfile.TemporaryDirectory() as tmp:
        deck.write(tmp)
        p = UphParams()
        l = _lib.lib()
        _lib.check(l.uph_deck_read(tmp.encode(), 1.3, C.byref(p), None), "deck_read counts")
        assert (p.n_fluid, p.n_solid, p.n_fixed, p.n_moving) == (deck.n_fluid, 0, deck.fixed.shape[0],
                                                                 deck.moving.shape[0])
        arrays = empty_state(p.n_fluid, deck.n_all)
        keep = []
        st = state_struct(arrays, keep)
        _lib.check(l.uph_deck_read(tmp.encode(), 1.3, C.byref(p), C.byref(st)), "deck_read")
    want = deck.initial_state()
    for k in ["Position", "Velocity", "localVelocity", "density", "localDensity", "DynamicPressure",
              "localPressure", "mass", "itype", "density_min", "DynamicPressure_min", "spongeFactor"]:
        assert np.array_equal(arrays[k], want[k]), k


def test_deck_read_bad_row_is_io_error():
    deck = D.dam_break(dx=0.1)
    with tempfile.TemporaryDirectory() as tmp:
        deck.write(tmp)
        with open(os.path.join(tmp, "FluidParticle.dat"), "a") as f:
            f.write("1 2 3\n")
        path = os.path.join(tmp, "FluidParticle.dat")
        lines = open(path).read().splitlines()
        lines[0] = str(int(lines[0]) + 1)
        open(path, "w").write("\n".join(lines) + "\n")
        p = UphParams()
        arrays = empty_state(deck.n_fluid + 1, deck.n_all + 1)
        keep = []
        st = state_struct(arrays, keep)
        assert _lib.lib().uph_deck_read(tmp.encode(), 0.0, C.byref(p), C.byref(st)) == 10


def test_deck_text_roundtrip():
    deck = D.dam_break(dx=0.05, hydrostatic=True)
    with tempfile.TemporaryDirectory() as tmp:
        deck.write(tmp)
        back = D.read_deck(tmp, eta_override=1.3)
    assert back.params == deck.params
    for blk in ("fluid", "solid", "fixed", "moving"):
        assert np.array_equal(getattr(back, blk), getattr(deck, blk)), blk


@pytest.mark.skipif(shutil.which("gcc") is None or not os.path.isdir(os.path.join(O.REFERENCE_TREE, "src", "lib")),
                    reason="needs gcc and the reference headers")
def test_system_layout_matches_reference():
    """include/uph_system.h declares the reference's struct with the same layout."""
    fields = ["dim", "itype", "NumberOfInteractingParticles", "MaxNumberOfParticles", "NumberOfFluidParticles",
              "Position", "Velocity", "mass", "Pressure", "hsml", "density", "ddensitydt", "dvdt", "density0",
              "DynamicPressure", "dpdt", "densityFluctuation", "velocityFluctuation", "localDensity",
              "localVelocity", "dwcdx", "timeStep", "virtualType", "selectBoundaryForce", "springConstant0",
              "thermalDiffusivity0", "movingBoundary", "spongeFactor", "waveAbsorption", "stressType",
              "ddensitydt_approx", "dvdt_approx", "SpeedOfSound", "stroke", "omega", "eta", "Gravity",
              "LocalDepth", "epsilon", "i_pair", "rij2", "w", "CompressionFactor", "AdiabaticConstant",
              "HowManyNeighbors"]
    src = "#include <stdio.h>\n#include <stddef.h>\n#include HDR\nint main(void){\n"
    src += 'printf("%zu\\n", sizeof(System));\n'
    for f in fields:
        src += f'printf("%zu\\n", offsetof(System, {f}));\n'
    src += "return 0;}\n"
    outs = []
    with tempfile.TemporaryDirectory() as tmp:
        c = os.path.join(tmp, "l.c")
        open(c, "w").write(src)
        for hdr, inc in [('"System.h"', os.path.join(O.REFERENCE_TREE, "src", "lib")), ('"uph_system.h"', os.path.join(ROOT, "include"))]:
            exe = os.path.join(tmp, "l")
            subprocess.run(["gcc", "-std=gnu99", f"-DHDR={hdr}", "-I", inc, c, "-o", exe], check=True)
            outs.append(subprocess.run([exe], capture_output=True, text=True, check=True).stdout)
    assert outs[0] == outs[1]


def test_sim_create_without_device_fails_cleanly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    deck = D.dam_break(dx=0.1)
    p = UphParams.from_dict(deck.uph_params())
    h = C.c_void_p()
    st = _lib.lib().uph_sim_create(C.byref(p), C.byref(h))
    assert st == 7  # UPH_NO_DEVICE
    assert not h.value


def test_sim_create_rejects_unsupported_modes():
    deck = D.dam_break(dx=0.1)
    # particle packing and stressType 2 exist for the REF profile only
    for over, status in [({"stress_type": 2, "profile": 1}, 8), ({"flag_init_simul": 0, "profile": 1}, 8),
                         ({"flag_init_simul": 2}, 8),
                         ({"precision": 1}, 8), ({"domain_hi": None}, 1)]:
        d = deck.uph_params()
        d.update(over)
        if d["domain_hi"] is None:
            d["domain_hi"] = list(d["domain_lo"])
        p = UphParams.from_dict(d)
        h = C.c_void_p()
        assert _lib.lib().uph_sim_create(C.byref(p), C.byref(h)) == status, over


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_python_structs_match_the_c_header():
    """The ctypes mirrors of include/uph.h's structs have the header's size
    and field offsets (a mismatch would let the library write past a Python
    buffer)."""
    from uph_b200._capi import UphDiagnostics, UphStats
    checks = [("uph_stats", UphStats), ("uph_params", UphParams), ("uph_diagnostics", UphDiagnostics)]
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"uph.h\"\nint main(void){\n"
    for cname, cls in checks:
        src += f'printf("%zu\\n", sizeof({cname}));\n'
        for field, _ in cls._fields_:
            src += f'printf("%zu\\n", offsetof({cname}, {field}));\n'
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as tmp:
        c = os.path.join(tmp, "s.c")
        open(c, "w").write(src)
        exe = os.path.join(tmp, "s")
        subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        got = [int(v) for v in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    want = []
    for _, cls in checks:
        want.append(C.sizeof(cls))
        want += [getattr(cls, field).offset for field, _ in cls._fields_]
    assert got == want
