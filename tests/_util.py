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


def compare_fields(got: dict, want: dict, n_fluid: int, tol: float, fields=FLUID_FIELDS, scales=None):
    """Returns {field: rel_err} and asserts every one is <= tol.  `scales`
    gives fields whose error is judged against a larger scale than their
    own largest magnitude (see velocity_fluctuation_scale)."""
    errs = {}
    for f in fields:
        g = np.asarray(got[f])[:n_fluid]
        w = np.asarray(want[f])[:n_fluid]
        errs[f] = rel_err(g, w)
        if scales and f in scales and w.size:
            errs[f] = float(np.max(np.abs(g - w))) / max(float(scales[f]), float(np.max(np.abs(w))))
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


def reference_state(run) -> dict:
    """The compiled reference's current state (oracle.RefRun) in the layout
    uph_sim_upload takes: every particle's kinematics and densities, the
    fluid's leapfrog and rate fields."""
    from uph_b200._capi import STATE_FIELDS
    c = run.counts()
    nf = c["n_fluid"]
    n = nf + c["n_solid"] + c["n_boundary"]
    out = {}
    for name, kind, _ in STATE_FIELDS:
        k = n if kind == "all" else nf
        out[name] = run.itype(0, k) if name == "itype" else run.get(name, 0, k)
    return out


def velocity_fluctuation_scale(run) -> float:
    """The scale velocityFluctuation's rounding is bounded by: over the fluid,
    the largest sum of the magnitudes of the two terms every pair adds,
    m_j (v_i - v_j) w / rhot_i and m_i (v_i - v_j) w / rhot_j
    (LocalVelocityFluctuation, derivatives.c:2060-2097).  The two nearly
    cancel where neighbouring densities agree, so the field can be far
    smaller than its terms; any summation order then leaves an error of about
    2^-52 times this scale, the reference's own included.  Read right after a
    derivatives() call of `run` (oracle.RefRun): its pairs, w and state."""
    c = run.counts()
    nf = c["n_fluid"]
    n = nf + c["n_solid"] + c["n_boundary"]
    i, j = run.pairs()
    w = run.get("w")
    v = run.get("Velocity", 0, n)
    rhot = run.get("localDensity", 0, n)
    m = run.get("mass", 0, n)
    avg = np.abs(v[i] - v[j]) * np.abs(w)[:, None]
    terms = avg * (m[j] / rhot[i] + m[i] / rhot[j])[:, None]
    s = np.zeros((nf, 2))
    np.add.at(s, i, terms)
    return float(s.max()) if s.size else 0.0
