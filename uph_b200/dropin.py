"""The reference-facing entry point from Python: the drop-in derivatives()
(libuph_sph.so, include/uph_system.h) called once per leapfrog step by the
host driver of libuph_driver.so (include/uph_driver.h), over a System with
the reference's layout.  Every step copies the state the reference's
derivatives() reads to the device and its outputs back, as a relinked
reference would.

There is no CPU fallback: the libraries must be built
(`python -m uph_b200.build`)."""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional

import numpy as np

from . import _lib
from ._capi import STATE_FIELDS, UphParams, empty_state, state_struct

_driver = None


def driver_lib() -> C.CDLL:
    global _driver
    if _driver is None:
        # loading the driver loads libuph_sph.so and libuph.so with it; the
        # drop-in's callbacks (inputbp, inoutflow) resolve to the driver's
        lib = C.CDLL(_lib.LIB_DRIVER_PATH)
        lib.uph_driver_create.restype = C.c_void_p
        lib.uph_driver_create.argtypes = [C.POINTER(UphParams), C.c_void_p, C.c_int32]
        lib.uph_driver_step.restype = C.c_int
        lib.uph_driver_step.argtypes = [C.c_void_p, C.c_int32]
        lib.uph_driver_state.restype = C.c_int
        lib.uph_driver_state.argtypes = [C.c_void_p, C.c_void_p]
        lib.uph_driver_destroy.restype = None
        lib.uph_driver_destroy.argtypes = [C.c_void_p]
        lib.uph_dropin_set_pair_export.restype = None
        lib.uph_dropin_set_pair_export.argtypes = [C.c_int]
        _driver = lib
    return _driver


class DropInRun:
    """A System advanced by the reference's leapfrog (src/bin/sph.cc:90-168)
    around derivatives(sys, t).  max_particles sizes the System's arrays (the
    reference's MaxNumberOfParticles): the pair arrays must hold every pair."""

    def __init__(self, params: dict, state: Dict[str, np.ndarray], max_particles: Optional[int] = None,
                 pair_export: int = 2):
        self.lib = driver_lib()
        self.nf = params["n_fluid"]
        self.n = params["n_fluid"] + params["n_solid"] + params["n_fixed"] + params["n_moving"]
        if max_particles is None:
            max_particles = self.n + 16 * self.nf
        self.params = UphParams.from_dict(params)
        keep = []
        st = state_struct({k: np.ascontiguousarray(v) for k, v in state.items()}, keep)
        self.handle = self.lib.uph_driver_create(C.byref(self.params), C.byref(st), int(max_particles))
        if not self.handle:
            raise RuntimeError("uph_driver_create failed (bad arguments or out of host memory)")
        self.set_pair_export(pair_export)

    def set_pair_export(self, level: int) -> None:
        """2: the full pair list (the reference's); 1: i, j, rij2; 0: the count."""
        self.lib.uph_dropin_set_pair_export(int(level))

    def step(self, nsteps: int = 1) -> None:
        _lib.check(self.lib.uph_driver_step(self.handle, int(nsteps)), "uph_driver_step")

    def state(self) -> Dict[str, np.ndarray]:
        out = empty_state(self.nf, self.n)
        keep = []
        st = state_struct(out, keep)
        _lib.check(self.lib.uph_driver_state(self.handle, C.byref(st)), "uph_driver_state")
        return out

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.uph_driver_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def bytes_per_step(nf: int, n: int, niac: int, pair_export: int) -> tuple:
        """(host-to-device, device-to-host) bytes one derivatives() call
        copies: the fields it reads of every particle; the rates,
        fluctuations and Tait pressure it returns; the pair arrays."""
        h2d = n * (3 * 16 + 5 * 8 + 4) + nf * 8  # Position, Velocity, localVelocity; 5 scalars; itype; sponge
        d2h = nf * (2 * 8 + 16 + 2 * 8 + 16 + 2 * 8 + 16) + n * 8  # rates, *_approx, fluctuations; Pressure
        d2h += niac * {0: 0, 1: 16, 2: 40}[pair_export]
        return h2d, d2h


__all__ = ["DropInRun", "driver_lib", "STATE_FIELDS"]
