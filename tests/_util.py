"""Shared helpers of the test suite."""
from __future__ import annotations

import glob
import os

import numpy as np

from uph_b200 import deck as D

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN_CASES = sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))

# fields compared after a step; the reference's System names
FLUID_FIELDS = ["Position", "Velocity", "localVelocity", "density", "localDensity", "DynamicPressure",
                "localPressure", "ddensitydt", "dpdt", "dvdt", "ddensitydt_approx", "dpdt_approx", "dvdt_approx",
                "densityFluctuation", "pressureFluctuation", "velocityFluctuation", "Pressure"]

# FP64 parity bound of the drop-in path: relative to the field's largest
# magnitude (norm-wise), so near-cancelling entries are judged on the field's
# own scale
REL_TOL_FP64 = 1e-10


def load_golden(name: str):
    return np.load(os.path.join(GOLDEN_DIR, name + ".npz"))


def deck_from_golden(g) -> D.Deck:
    params = {k: (int(v) if t is int else float(v)) for (k, t), v in zip(D.PARAM_ORDER, g["params"])}
    deck = D.Deck(params, g["fluid"].copy(), g["solid"].copy(), g["fixed"].copy(), g["moving"].copy(),
                  eta_override=float(g["eta_override"]))
    deck.domain_lo = tuple(float(v) for v in g["domain_lo"])
    deck.domain_hi = tuple(float(v) for v in g["domain_hi"])
    return deck


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """max |a - b| / max |b| (0 when both are identically zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = float(np.max(np.abs(b))) if b.size else 0.0
    diff = float(np.max(np.abs(a - b))) if b.size else 0.0
    if scale == 0.0:
        return diff
    return diff / scale


def compare_fields(got: dict, want: dict, n_fluid: int, tol: float, fields=FLUID_FIELDS):
    """Returns {field: rel_err} and asserts every one is <= tol."""
    errs = {}
    for f in fields:
        g = np.asarray(got[f])[:n_fluid]
        w = np.asarray(want[f])[:n_fluid]
        errs[f] = rel_err(g, w)
    bad = {k: v for k, v in errs.items() if not v <= tol}
    assert not bad, f"fields above {tol:g}: {bad}"
    return errs


def ref_env() -> dict:
    """The environment for the reference's own executables: at most 64
    OpenMP threads, the rows of its per-thread scratch (System.c:209); and
    heap blocks that start zeroed (glibc's MALLOC_PERTURB_=255 fills each new
    block with 0x00), because its first inoutflow() call reads
    sys->inflowParticles before anything sets it (derivatives.c:3163 before
    :3172; System.c never initialises it)."""
    import os
    return dict(os.environ, OMP_NUM_THREADS=str(min(64, os.cpu_count() or 1)), MALLOC_PERTURB_="255")
