"""Python host mirror of the reference's hot-path interface.

The reference drives its solver as

    sys = CreateSystem(...); input(sys)                 # System.c:38, input.c:22
    for itime in 1..N: ...; derivatives(sys, t); ...    # sph.cc:90-168
    SearchNeighbors(Position, i_pair, j_pair, rij2, Nf, N, PB, 40, dist)   # Search.cc:5

`Simulation` holds one case resident on the GPU and offers the same
operations -- `derivatives(t)` (one rate evaluation, derivatives.c:3137),
`step(n)` (the sph.cc leapfrog), `search_neighbors` (SearchNeighbors) --
through libuph.so.  Arrays are numpy, in the reference's particle order and
layout ([n][2] vectors).  Errors raise UphError with the library's status
instead of the reference's printf + exit(1).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional

import numpy as np

from . import _lib
from ._capi import (PREC_FP64, PROFILE_REF, STATE_FIELDS, UphDiagnostics, UphParams, UphStats, empty_state,
                    state_struct)
from .deck import Deck


# The fields a leapfrog step after the first reads from an upload, and so
# the state one step hands to the next: positions, velocities, density and
# pressure of every particle, mass, type and sponge (constant), and the
# fluid's predictor rates and fluctuations.  The step derives the rest
# (local and *_min fields from the predictor, the corrector rates and the
# equation of state from the rate pass), so an upload may leave them NULL.
STEP_INPUT_FIELDS = ["Position", "Velocity", "density", "DynamicPressure", "mass", "itype", "spongeFactor",
                     "ddensitydt_approx", "dpdt_approx", "dvdt_approx", "densityFluctuation",
                     "pressureFluctuation", "velocityFluctuation"]
STEP_OUTPUT_FIELDS = [f for f in STEP_INPUT_FIELDS if f not in ("mass", "itype", "spongeFactor")]


class Simulation:
    def __init__(self, params: dict):
        self.lib = _lib.lib()
        self.params = UphParams.from_dict(params)
        self.n_fluid = int(params["n_fluid"])
        self.n_all = int(params["n_fluid"] + params["n_solid"] + params["n_fixed"] + params["n_moving"])
        h = C.c_void_p()
        _lib.check(self.lib.uph_sim_create(C.byref(self.params), C.byref(h)), "uph_sim_create")
        self.handle = h

    @classmethod
    def from_deck(cls, deck: Deck, profile: int = PROFILE_REF, precision: int = PREC_FP64,
                  av_alpha: Optional[float] = None, knn_cap: int = 0) -> "Simulation":
        sim = cls(deck.uph_params(profile, precision, av_alpha, knn_cap))
        sim.upload(deck.initial_state(), 0)
        if deck.wall_table is not None:
            sim.set_wall_motion(*deck.wall_table)
        mb = deck.params.get("moving_boundary", 0)
        if mb in (2, 3) and deck.moving.shape[0]:
            # the decks' tempPosition (lid) / tempPositionGate (gate) columns
            sim.set_wall_base(deck.moving[:, 0 if mb == 3 else 8])
        return sim

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.uph_sim_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state ----------------------------------------------------------------
    def upload(self, state: Dict[str, np.ndarray], itime: int = 0) -> None:
        keep = []
        st = state_struct(state, keep)
        _lib.check(self.lib.uph_sim_upload(self.handle, C.byref(st), itime), "uph_sim_upload")

    def download(self, out: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        if out is None:
            out = empty_state(self.n_fluid, self.n_all)
        keep = []
        st = state_struct(out, keep)
        _lib.check(self.lib.uph_sim_download(self.handle, C.byref(st)), "uph_sim_download")
        return out

    state = download

    # -- the hot path ----------------------------------------------------------
    def step(self, nsteps: int = 1) -> None:
        _lib.check(self.lib.uph_sim_step(self.handle, nsteps), "uph_sim_step")

    def set_graph(self, steps_per_graph: int) -> None:
        """Record / replay `steps_per_graph`-step calls of step() as a CUDA graph."""
        _lib.check(self.lib.uph_sim_set_graph(self.handle, steps_per_graph), "uph_sim_set_graph")

    def set_fused_step(self, enable: bool) -> None:
        """Whether the rate pass applies the leapfrog step itself (default on)."""
        _lib.check(self.lib.uph_sim_set_fused_step(self.handle, 1 if enable else 0), "uph_sim_set_fused_step")

    def set_candidate_lists(self, enable: bool) -> None:
        """Whether the rate passes keep per-particle candidate lists between cell-list builds (default on)."""
        _lib.check(self.lib.uph_sim_set_candidate_lists(self.handle, 1 if enable else 0),
                   "uph_sim_set_candidate_lists")

    def set_tuning(self, reach: int, tile: int, reorder_interval: int) -> None:
        _lib.check(self.lib.uph_sim_set_tuning(self.handle, reach, tile, reorder_interval), "uph_sim_set_tuning")

    def autotune(self, trial_steps: int = 10):
        """Native autotuner; returns ((reach, tile, interval), best ms/step or 0 if cached)."""
        choice = (C.c_int32 * 3)()
        ms = C.c_double(0.0)
        _lib.check(self.lib.uph_sim_autotune(self.handle, trial_steps, C.byref(choice), C.byref(ms)),
                   "uph_sim_autotune")
        return tuple(choice), ms.value

    def set_wall_motion(self, x0, half_stroke, omega) -> None:
        """Shake each moving-boundary particle: x = x0 + hs (1 - cos(omega t))."""
        self._wall = [np.ascontiguousarray(a, dtype=np.float64) for a in (x0, half_stroke, omega)]
        _lib.check(self.lib.uph_sim_set_wall_motion(self.handle, *(a.ctypes.data for a in self._wall)),
                   "uph_sim_set_wall_motion")

    def set_wall_base(self, base) -> None:
        """Base coordinates of the lid (x) or gate (y) particles, reference order."""
        self._base = np.ascontiguousarray(base, dtype=np.float64)
        _lib.check(self.lib.uph_sim_set_wall_base(self.handle, self._base.ctypes.data), "uph_sim_set_wall_base")

    def derivatives(self, t: float) -> None:
        _lib.check(self.lib.uph_sim_derivatives(self.handle, t), "uph_sim_derivatives")

    def pairs(self):
        """(i_pair, j_pair, rij2, w, dwcdx) of the current positions."""
        n = C.c_int64(0)
        st = self.lib.uph_sim_pairs(self.handle, 0, None, None, None, None, None, C.byref(n))
        if st not in (0, 3):
            _lib.check(st, "uph_sim_pairs")
        k = n.value
        i = np.zeros(k, np.int32)
        j = np.zeros(k, np.int32)
        r2 = np.zeros(k)
        w = np.zeros(k)
        dw = np.zeros((k, 2))
        _lib.check(self.lib.uph_sim_pairs(self.handle, k, i.ctypes.data, j.ctypes.data, r2.ctypes.data,
                                          w.ctypes.data, dw.ctypes.data, C.byref(n)), "uph_sim_pairs")
        return i, j, r2, w, dw

    def virtual(self):
        """(position [k][2], source fluid index [k], mirror kind [k]) of the
        virtual mirror particles of the last evaluation (uph_sim_virtual)."""
        n = C.c_int64(0)
        _lib.check(self.lib.uph_sim_virtual(self.handle, 0, None, None, None, C.byref(n)), "uph_sim_virtual")
        k = n.value
        pos = np.zeros((k, 2))
        src = np.zeros(k, np.int32)
        kind = np.zeros(k, np.int32)
        if k:
            _lib.check(self.lib.uph_sim_virtual(self.handle, k, pos.ctypes.data, src.ctypes.data, kind.ctypes.data,
                                                C.byref(n)), "uph_sim_virtual")
        return pos, src, kind

    def stats(self) -> dict:
        s = UphStats()
        _lib.check(self.lib.uph_sim_stats(self.handle, C.byref(s)), "uph_sim_stats")
        return {name: getattr(s, name) for name, _ in UphStats._fields_}

    # -- diagnostics and output ----------------------------------------------------
    def set_diagnostics(self, enable: bool = True, probe: Optional[tuple] = None,
                        probe_two: tuple = (0.0, 0.0)) -> None:
        """Per-evaluation kinetic energy and pressure probes (derivatives.c:2254-2393).

        `probe` defaults to parameters.dat's pressureProbeX/Y; the reference
        never sets the second probe, so (0, 0) reproduces its files."""
        if probe is None:
            probe = (self.params.pressure_probe_x, self.params.pressure_probe_y)
        _lib.check(self.lib.uph_sim_set_diagnostics(self.handle, 1 if enable else 0, float(probe[0]),
                                                    float(probe[1]), float(probe_two[0]), float(probe_two[1])),
                   "uph_sim_set_diagnostics")

    def diagnostics(self) -> dict:
        d = UphDiagnostics()
        _lib.check(self.lib.uph_sim_diagnostics(self.handle, C.byref(d)), "uph_sim_diagnostics")
        return {name: getattr(d, name) for name, _ in UphDiagnostics._fields_}

    def write_output(self, directory: str, itime: Optional[int] = None, state: Optional[dict] = None,
                     dam_gate_flag: Optional[np.ndarray] = None) -> None:
        """output(sys, itime) of output.c:19-140 for the current (or a given
        downloaded) state, with the diagnostics of the last evaluation."""
        write_output(directory, self.params, self.download() if state is None else state,
                     self.diagnostics(), self.stats()["itime"] if itime is None else itime, dam_gate_flag)

    # -- measurement -----------------------------------------------------------
    def set_stream(self, cuda_stream: int) -> None:
        _lib.check(self.lib.uph_sim_set_stream(self.handle, C.c_void_p(cuda_stream)), "uph_sim_set_stream")

    def profile(self, enable: bool) -> None:
        _lib.check(self.lib.uph_sim_profile(self.handle, 1 if enable else 0), "uph_sim_profile")

    def kernel_times(self) -> Dict[str, tuple]:
        ms = np.zeros(16)
        cnt = np.zeros(16, np.int64)
        names = C.create_string_buffer(512)
        nw = C.c_int32(0)
        _lib.check(self.lib.uph_sim_kernel_times(self.handle, 16, ms.ctypes.data, cnt.ctypes.data, names, 512,
                                                 C.byref(nw)), "uph_sim_kernel_times")
        keys = names.value.decode().split(",")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(keys[:nw.value])}

    def launch_count(self) -> int:
        return int(self.lib.uph_sim_launch_count(self.handle))


def write_output(directory: str, params, state: dict, diagnostics: dict, itime: int,
                 dam_gate_flag: Optional[np.ndarray] = None) -> None:
    """uph_write_output: the reference's out<itime>.dat and diagnostics files.

    `params` is a UphParams or a dict of its fields; `diagnostics` a dict of
    UphDiagnostics fields (Simulation.diagnostics())."""
    lib = _lib.lib()
    p = params if isinstance(params, UphParams) else UphParams.from_dict(params)
    keep = []
    st = state_struct(state, keep)
    d = UphDiagnostics(**{k: diagnostics[k] for k, _ in UphDiagnostics._fields_})
    gate = None
    if dam_gate_flag is not None:
        gate = np.ascontiguousarray(dam_gate_flag, dtype=np.int32)
        keep.append(gate)
    _lib.check(lib.uph_write_output(os.fsencode(directory), int(itime), C.byref(p), C.byref(st),
                                    None if gate is None else gate.ctypes.data, C.byref(d)), "uph_write_output")


def search_neighbors(position: np.ndarray, n_fluid: int, particle_boundary: int, dist: float,
                     number_of_neighbors: int = 40):
    """SearchNeighbors (Search.cc:5): pairs (s, j), s < n_fluid < ..., j > s,
    DBL_EPSILON < rij2 < dist, j < particle_boundary; returns (i, j, rij2)."""
    l = _lib.lib()
    pos = np.ascontiguousarray(position, dtype=np.float64).reshape(-1, 2)
    n = C.c_int64(0)
    st = l.uph_search_neighbors(pos.ctypes.data, n_fluid, pos.shape[0], particle_boundary, number_of_neighbors,
                                dist, 0, None, None, None, C.byref(n))
    if st not in (0, 3):
        _lib.check(st, "uph_search_neighbors")
    k = n.value
    i = np.zeros(k, np.int32)
    j = np.zeros(k, np.int32)
    r2 = np.zeros(k)
    _lib.check(l.uph_search_neighbors(pos.ctypes.data, n_fluid, pos.shape[0], particle_boundary,
                                      number_of_neighbors, dist, k, i.ctypes.data, j.ctypes.data, r2.ctypes.data,
                                      C.byref(n)), "uph_search_neighbors")
    return i, j, r2


__all__ = ["Simulation", "search_neighbors", "STATE_FIELDS"]
