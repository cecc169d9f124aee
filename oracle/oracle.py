"""Test infrastructure (oracle only): Python access to the CPU checkers.

* ``Oracle`` wraps the CPU restatement oracle/uph_oracle.c
  (oracle/_ref/libuph_oracle.so).
* ``RefRun`` wraps the reference's own solver compiled from its sources
  (oracle/_ref/libuph_ref.so; oracle/ref_harness.c drives it).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  The product (uph_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from uph_b200._capi import (STATE_FIELDS, UphParams, empty_state, state_struct)

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def _reference_tree() -> str:
    """The reference's source tree: $UPH_REFERENCE, else the default of
    oracle/Makefile (its REF line is the one place the default is kept)."""
    env = os.environ.get("UPH_REFERENCE")
    if env:
        return env
    with open(os.path.join(HERE, "Makefile")) as f:
        for line in f:
            if line.startswith("REF ?="):
                return line.rsplit(",", 1)[-1].strip().rstrip(")")
    return ""


REFERENCE_TREE = _reference_tree()


def build(reference: bool = True) -> None:
    """make -C oracle (the compiled reference only when its sources exist)."""
    target = "all" if reference else "port"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def _load(name: str) -> C.CDLL:
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (make -C oracle)")
    return C.CDLL(path)


_oracle_lib = None


def oracle_lib() -> C.CDLL:
    global _oracle_lib
    if _oracle_lib is None:
        lib = _load("libuph_oracle.so")
        lib.uph_oracle_create.restype = C.c_void_p
        lib.uph_oracle_create.argtypes = [C.POINTER(UphParams)]
        lib.uph_oracle_destroy.argtypes = [C.c_void_p]
        lib.uph_oracle_set_state.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        lib.uph_oracle_get_state.argtypes = [C.c_void_p, C.c_void_p]
        lib.uph_oracle_derivatives.argtypes = [C.c_void_p, C.c_double]
        lib.uph_oracle_step.argtypes = [C.c_void_p, C.c_int]
        lib.uph_oracle_pairs.restype = C.c_int64
        lib.uph_oracle_pairs.argtypes = [C.c_void_p, C.c_int64] + [C.c_void_p] * 5
        lib.uph_oracle_max_neighbors.argtypes = [C.c_void_p]
        lib.uph_oracle_set_wall_motion.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.uph_oracle_energies.argtypes = [C.c_void_p, C.c_void_p]
        lib.uph_oracle_search.restype = C.c_int64
        lib.uph_oracle_search.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int64,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _oracle_lib = lib
    return _oracle_lib


class Oracle:
    """The CPU restatement holding one simulation."""

    def __init__(self, params: dict, state: dict, itime: int = 0):
        self.lib = oracle_lib()
        self.params = UphParams.from_dict(params)
        self.nf = params["n_fluid"]
        self.n = params["n_fluid"] + params["n_solid"] + params["n_fixed"] + params["n_moving"]
        self.h = self.lib.uph_oracle_create(C.byref(self.params))
        keep = []
        st = state_struct({k: np.ascontiguousarray(v) for k, v in state.items()}, keep)
        self.lib.uph_oracle_set_state(self.h, C.byref(st), itime)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.uph_oracle_destroy(self.h)
            self.h = None

    def step(self, nsteps: int = 1) -> None:
        self.lib.uph_oracle_step(self.h, nsteps)

    def derivatives(self, t: float) -> None:
        self.lib.uph_oracle_derivatives(self.h, t)

    def state(self) -> dict:
        out = empty_state(self.nf, self.n)
        keep = []
        st = state_struct(out, keep)
        self.lib.uph_oracle_get_state(self.h, C.byref(st))
        return out

    def pairs(self):
        n = self.lib.uph_oracle_pairs(self.h, 0, None, None, None, None, None)
        i = np.zeros(n, np.int32)
        j = np.zeros(n, np.int32)
        r2 = np.zeros(n)
        w = np.zeros(n)
        dw = np.zeros((n, 2))
        self.lib.uph_oracle_pairs(self.h, n, i.ctypes.data, j.ctypes.data, r2.ctypes.data, w.ctypes.data,
                                  dw.ctypes.data)
        return i, j, r2, w, dw

    def max_neighbors(self) -> int:
        return self.lib.uph_oracle_max_neighbors(self.h)

    def set_wall_motion(self, x0, half_stroke, omega) -> None:
        self._wall = [np.ascontiguousarray(a, dtype=np.float64) for a in (x0, half_stroke, omega)]
        self.lib.uph_oracle_set_wall_motion(self.h, *(a.ctypes.data for a in self._wall))

    def energies(self):
        out = np.zeros(3)
        self.lib.uph_oracle_energies(self.h, out.ctypes.data)
        return out


def search(pos: np.ndarray, n_fluid: int, particle_boundary: int, dist: float):
    """Radius search with SearchNeighbors' filter; returns (i, j, rij2, max_inradius)."""
    lib = oracle_lib()
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    n_all = pos.shape[0]
    mx = C.c_int(0)
    n = lib.uph_oracle_search(pos.ctypes.data, n_fluid, n_all, particle_boundary, dist, 0, None, None, None,
                              C.byref(mx))
    i = np.zeros(n, np.int32)
    j = np.zeros(n, np.int32)
    r2 = np.zeros(n)
    lib.uph_oracle_search(pos.ctypes.data, n_fluid, n_all, particle_boundary, dist, n, i.ctypes.data,
                          j.ctypes.data, r2.ctypes.data, C.byref(mx))
    return i, j, r2, mx.value


# --------------------------------------------------------- compiled reference

_ref_lib = None


def ref_lib() -> C.CDLL:
    global _ref_lib
    if _ref_lib is None:
        lib = _load("libuph_ref.so")
        lib.ref_open.restype = C.c_void_p
        lib.ref_open.argtypes = [C.c_char_p, C.c_double, C.c_int]
        lib.ref_close.argtypes = [C.c_void_p]
        lib.ref_step.argtypes = [C.c_void_p, C.c_int]
        lib.ref_derivatives.argtypes = [C.c_void_p, C.c_double]
        lib.ref_counts.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_scalars.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_get.restype = C.c_long
        lib.ref_get.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.c_void_p]
        lib.ref_set.restype = C.c_long
        lib.ref_set.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.c_void_p]
        lib.ref_get_itype.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        lib.ref_pairs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ref_time_inputbp.restype = C.c_double
        lib.ref_time_inputbp.argtypes = [C.c_void_p, C.c_int]
        lib.uph_standin_reset_stats.argtypes = []
        lib.uph_standin_truncated_queries.restype = C.c_long
        lib.uph_standin_max_inradius.restype = C.c_int
        _ref_lib = lib
    return _ref_lib


VECTOR_FIELDS = {"Position", "Velocity", "localVelocity", "Velocity_min", "dvdt", "dvdt_approx",
                 "velocityFluctuation", "dwcdx"}


class RefRunInProcess:
    """The reference solver (CreateSystem + input + sph.cc's loop) on a deck
    directory, in this process: what RefRun's child process runs, and the
    base of harnesses over the same API that must share this process (the
    drop-in build, whose derivatives() runs on this process's GPU).
    fluid_capacity_pct > 0 shrinks the reference's 100 Nf particle capacity
    (see oracle/ref_harness.c)."""

    def __init__(self, deck_dir: str, eta_override: float = 0.0, fluid_capacity_pct: int = 0):
        self.lib = ref_lib()
        self.lib.uph_standin_reset_stats()
        self.h = self.lib.ref_open(os.fsencode(deck_dir), eta_override, fluid_capacity_pct)
        if not self.h:
            raise FileNotFoundError(f"reference could not open deck {deck_dir}")

    def close(self):
        if self.h:
            self.lib.ref_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def counts(self) -> dict:
        c = np.zeros(9, np.int32)
        self.lib.ref_counts(self.h, c.ctypes.data)
        keys = ["n_fluid", "n_solid", "n_fixed", "n_moving", "n_boundary", "niac", "max_n", "itime", "n_virtual"]
        return dict(zip(keys, (int(v) for v in c)))

    def scalars(self) -> dict:
        s = np.zeros(16)
        self.lib.ref_scalars(self.h, s.ctypes.data)
        keys = ["dt", "c0", "B", "eta", "h", "rho0", "gamma", "g", "k_spring", "c_damp", "kappa", "mu",
                "epsilon", "dx", "omega", "stroke"]
        return dict(zip(keys, (float(v) for v in s)))

    def step(self, nsteps: int = 1) -> None:
        self.lib.ref_step(self.h, nsteps)

    def derivatives(self, t: float) -> None:
        self.lib.ref_derivatives(self.h, t)

    def get(self, name: str, first: int = 0, n: int = None) -> np.ndarray:
        c = self.counts()
        if n is None:
            n = c["niac"] if name in ("rij2", "w", "dwcdx") else c["n_fluid"]
        vec = name in VECTOR_FIELDS
        out = np.zeros((n, 2) if vec else n)
        got = self.lib.ref_get(self.h, name.encode(), first, n, out.ctypes.data)
        if got < 0:
            raise KeyError(name)
        return out

    def set(self, name: str, values: np.ndarray, first: int = 0) -> None:
        values = np.ascontiguousarray(values, dtype=np.float64)
        n = values.shape[0]
        if self.lib.ref_set(self.h, name.encode(), first, n, values.ctypes.data) < 0:
            raise KeyError(name)

    def itype(self, first: int = 0, n: int = None) -> np.ndarray:
        if n is None:
            c = self.counts()
            n = c["n_fluid"] + c["n_solid"] + c["n_boundary"]
        out = np.zeros(n, np.int32)
        self.lib.ref_get_itype(self.h, first, n, out.ctypes.data)
        return out

    def pairs(self):
        n = self.counts()["niac"]
        i = np.zeros(n, np.int32)
        j = np.zeros(n, np.int32)
        self.lib.ref_pairs(self.h, i.ctypes.data, j.ctypes.data)
        return i, j

    def time_inputbp(self, ncalls: int = 3) -> float:
        """Seconds per call of the reference's inputbp() (the boundary decks'
        per-step re-read and the wall-motion law) at the next step's time."""
        return float(self.lib.ref_time_inputbp(self.h, ncalls)) / max(ncalls, 1)

    def truncated_queries(self) -> int:
        return int(self.lib.uph_standin_truncated_queries())

    def max_inradius(self) -> int:
        return int(self.lib.uph_standin_max_inradius())


# The compiled reference runs in a child process of its own (spawned, never
# forked: the parent may hold a CUDA context).  There it shares no heap or
# OpenMP runtime with CUDA, torch or the GPU library, and a crash of the
# reference's C code ends the child, not the caller: the call raises
# ReferenceCrash.  Its heap blocks start zeroed (glibc's MALLOC_PERTURB_=255),
# so what the reference reads before writing is zero on every run, as on a
# fresh heap: CreateSystem leaves fields such as inflowParticles unset
# (System.c:195-250), which derivatives.c:3163 reads before :3172 sets it.

class ReferenceCrash(RuntimeError):
    pass


def _ref_worker_main(conn) -> None:
    runs = {}
    while True:
        try:
            msg = conn.recv()
        except EOFError:
            return
        h, method, args = msg
        try:
            if method == "open":
                run = RefRunInProcess(*args)
                runs[id(run)] = run
                val = id(run)
            elif method == "close":
                run = runs.pop(h, None)
                if run is not None:
                    run.close()
                val = None
            elif method == "exit":
                conn.send((True, None))
                return
            else:
                val = getattr(runs[h], method)(*args)
            conn.send((True, val))
        except Exception as e:  # the reference's own errors go back to the caller
            conn.send((False, e))


class _RefWorker:
    def __init__(self):
        import multiprocessing as mp
        ctx = mp.get_context("spawn")
        self.conn, child = ctx.Pipe()
        saved = {k: os.environ.get(k) for k in ("MALLOC_PERTURB_",)}
        os.environ["MALLOC_PERTURB_"] = "255"
        try:
            self.proc = ctx.Process(target=_ref_worker_main, args=(child,), daemon=True)
            self.proc.start()
        finally:
            for k, v in saved.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        child.close()

    def alive(self) -> bool:
        return self.proc.is_alive()

    def call(self, h, method, *args):
        try:
            self.conn.send((h, method, args))
            ok, val = self.conn.recv()
        except (EOFError, BrokenPipeError, ConnectionResetError):
            self.proc.join(5)
            raise ReferenceCrash(f"the compiled reference's process ended (exit code {self.proc.exitcode}) "
                                 f"in {method}{args}") from None
        if not ok:
            raise val
        return val


_worker = None


def _ref_worker() -> _RefWorker:
    global _worker
    if _worker is None or not _worker.alive():
        _worker = _RefWorker()
    return _worker


class RefRun:
    """The reference solver (CreateSystem + input + sph.cc's loop) on a deck
    directory, run in the reference's own child process (see above).
    fluid_capacity_pct > 0 shrinks the reference's 100 Nf particle capacity
    (see oracle/ref_harness.c)."""

    def __init__(self, deck_dir: str, eta_override: float = 0.0, fluid_capacity_pct: int = 0):
        self.w = _ref_worker()
        self.h = self.w.call(None, "open", os.path.abspath(deck_dir), float(eta_override), int(fluid_capacity_pct))

    def _call(self, method, *args):
        return self.w.call(self.h, method, *args)

    def close(self):
        if getattr(self, "h", None) is not None:
            h, self.h = self.h, None
            if self.w.alive():
                self.w.call(h, "close")

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def counts(self) -> dict:
        return self._call("counts")

    def scalars(self) -> dict:
        return self._call("scalars")

    def step(self, nsteps: int = 1) -> None:
        self._call("step", int(nsteps))

    def derivatives(self, t: float) -> None:
        self._call("derivatives", float(t))

    def get(self, name: str, first: int = 0, n: int = None) -> np.ndarray:
        return self._call("get", name, first, n)

    def set(self, name: str, values: np.ndarray, first: int = 0) -> None:
        self._call("set", name, np.ascontiguousarray(values, dtype=np.float64), first)

    def itype(self, first: int = 0, n: int = None) -> np.ndarray:
        return self._call("itype", first, n)

    def pairs(self):
        return self._call("pairs")

    def time_inputbp(self, ncalls: int = 3) -> float:
        return self._call("time_inputbp", ncalls)

    def truncated_queries(self) -> int:
        return self._call("truncated_queries")

    def max_inradius(self) -> int:
        return self._call("max_inradius")


# fields compared after a step (reference name -> uph_state name is the same)
FLUID_FIELDS = ["Position", "Velocity", "localVelocity", "density", "localDensity", "DynamicPressure",
                "localPressure", "ddensitydt", "dpdt", "dvdt", "ddensitydt_approx", "dpdt_approx", "dvdt_approx",
                "densityFluctuation", "pressureFluctuation", "velocityFluctuation", "Pressure"]

STATE_NAMES = [name for name, _, _ in STATE_FIELDS]
