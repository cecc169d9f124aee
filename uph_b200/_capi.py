"""ctypes mirrors of the C ABI structs in include/uph.h.

These are plain data descriptions shared by the host mirror (uph_b200.sim),
the tests and the oracle wrapper.  Loading the CUDA library itself happens in
uph_b200._lib.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

UPH_OK = 0
STATUS_NAMES = {
    0: "UPH_OK",
    1: "UPH_BAD_ARG",
    2: "UPH_OUT_OF_DOMAIN",
    3: "UPH_NEIGHBOR_OVERFLOW",
    4: "UPH_NAN",
    5: "UPH_TIMEOUT",
    6: "UPH_CUDA_ERROR",
    7: "UPH_NO_DEVICE",
    8: "UPH_UNSUPPORTED",
    9: "UPH_OUT_OF_MEMORY",
    10: "UPH_IO_ERROR",
}

PROFILE_REF = 0
PROFILE_WCSPH = 1
PREC_FP64 = 0
PREC_FP32_PAIR = 1

i32 = C.c_int32
f64 = C.c_double

# (name, ctype) in declaration order of struct uph_params
PARAM_FIELDS = [
    ("profile", i32), ("precision", i32),
    ("n_fluid", i32), ("n_solid", i32), ("n_fixed", i32), ("n_moving", i32),
    ("stroke", f64), ("wave_period", f64), ("local_depth", f64), ("flat_bottom_length", f64),
    ("density0", f64), ("adiabatic_constant", f64), ("gravity", f64), ("dx", f64), ("dy", f64),
    ("dim", i32),
    ("viscosity0", f64), ("mach_number", f64), ("peclet_number", f64), ("epsilon", f64), ("alpha", f64),
    ("virtual_type", i32), ("print_step", i32), ("screen_step", i32),
    ("time_step", f64), ("lid_velocity", f64),
    ("near_neighbor", i32), ("select_boundary_force", i32),
    ("lennard_select", f64), ("spring_constant0", f64), ("damping_constant0", f64),
    ("flag_init_simul", i32), ("gravity_flag", i32),
    ("thermal_diffusivity0", f64),
    ("moving_boundary", i32), ("number_of_initialization_steps", i32),
    ("pressure_probe_x", f64), ("pressure_probe_y", f64),
    ("stress_type", i32), ("dissipation_control_volume", i32),
    ("speed_of_sound", f64), ("compression_factor", f64), ("omega", f64), ("eta", f64), ("h", f64),
    ("lennard_coefficient", f64), ("sponge_factor0", f64), ("sponge_position0", f64),
    ("wave_absorption", i32),
    ("av_alpha", f64),
    ("knn_cap", i32),
    ("domain_lo", f64 * 2), ("domain_hi", f64 * 2),
]


class UphParams(C.Structure):
    _fields_ = PARAM_FIELDS

    def to_dict(self) -> dict:
        out = {}
        for name, ct in PARAM_FIELDS:
            v = getattr(self, name)
            out[name] = list(v) if isinstance(v, C.Array) else v
        return out

    @classmethod
    def from_dict(cls, d: dict) -> "UphParams":
        p = cls()
        for name, ct in PARAM_FIELDS:
            if name in d:
                v = d[name]
                if isinstance(getattr(p, name), C.Array):
                    arr = getattr(p, name)
                    for k, x in enumerate(v):
                        arr[k] = x
                else:
                    setattr(p, name, v)
        return p


DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int32)

# (name, kind, width) kind: "all" or "fluid"; width 2 = [n][2]
STATE_FIELDS = [
    ("Position", "all", 2), ("Velocity", "all", 2), ("localVelocity", "all", 2),
    ("density", "all", 1), ("localDensity", "all", 1), ("DynamicPressure", "all", 1),
    ("localPressure", "all", 1), ("mass", "all", 1), ("itype", "all", 1),
    ("Velocity_min", "fluid", 2), ("density_min", "fluid", 1), ("DynamicPressure_min", "fluid", 1),
    ("spongeFactor", "fluid", 1),
    ("ddensitydt", "fluid", 1), ("dpdt", "fluid", 1), ("dvdt", "fluid", 2),
    ("ddensitydt_approx", "fluid", 1), ("dpdt_approx", "fluid", 1), ("dvdt_approx", "fluid", 2),
    ("densityFluctuation", "fluid", 1), ("pressureFluctuation", "fluid", 1),
    ("velocityFluctuation", "fluid", 2),
    ("Pressure", "all", 1),
]


class UphState(C.Structure):
    _fields_ = [(name, IP if name == "itype" else DP) for name, _, _ in STATE_FIELDS]


class UphStats(C.Structure):
    _fields_ = [
        ("niac", C.c_int64), ("max_neighbors", i32), ("itime", i32),
        ("kinetic_energy", f64), ("potential_energy", f64), ("total_mass", f64),
        ("max_abs_density_error", f64), ("list_builds", C.c_int64),
    ]


class UphDiagnostics(C.Structure):
    _fields_ = [
        ("kinetic_energy", f64), ("potential_energy", f64),
        ("point_pressure", f64), ("pressure_norm", f64), ("point_pressure_two", f64),
        ("point_neighbors", i32), ("point_neighbors_two", i32), ("itime", i32),
    ]


def state_shapes(n_fluid: int, n_all: int) -> dict:
    out = {}
    for name, kind, width in STATE_FIELDS:
        n = n_all if kind == "all" else n_fluid
        out[name] = (n, 2) if width == 2 else (n,)
    return out


def empty_state(n_fluid: int, n_all: int) -> dict:
    """Zeroed numpy arrays for every uph_state field."""
    out = {}
    for name, shape in state_shapes(n_fluid, n_all).items():
        out[name] = np.zeros(shape, dtype=np.int32 if name == "itype" else np.float64)
    return out


def state_struct(arrays: dict, keepalive: list) -> UphState:
    """A UphState pointing at the numpy arrays in `arrays` (missing -> NULL).

    Arrays are made C-contiguous with the right dtype; the converted arrays are
    appended to `keepalive` so the pointers stay valid."""
    st = UphState()
    for name, _, _ in STATE_FIELDS:
        a = arrays.get(name)
        if a is None:
            continue
        dt = np.int32 if name == "itype" else np.float64
        if a.dtype != dt or not a.flags["C_CONTIGUOUS"]:
            raise ValueError(f"state field {name} must be a C-contiguous {np.dtype(dt).name} array")
        keepalive.append(a)
        setattr(st, name, a.ctypes.data_as(IP if name == "itype" else DP))
    return st


# ---- include/uph_surrogate.h -------------------------------------------------
class SurConfig(C.Structure):
    _fields_ = [("rounds", C.c_int32), ("macro_steps", C.c_int32), ("radius", C.c_double), ("dt", C.c_double),
                ("rho0", C.c_double), ("vel_scale", C.c_double), ("rho_scale", C.c_double),
                ("edge_rho_scale", C.c_double), ("out_scale", C.c_double * 5)]


class SurNodes(C.Structure):
    _fields_ = [("n", C.c_int32), ("n_fluid", C.c_int32)] + \
               [(k, C.c_void_p) for k in ("x", "y", "u", "v", "rho", "itype")] + \
               [(k, C.c_double) for k in ("lo_x", "lo_y", "hi_x", "hi_y")]


class SurJudge(C.Structure):
    _fields_ = [("judge_every", C.c_int32), ("fallback_macro", C.c_int32), ("max_rho_err", C.c_double),
                ("max_surface_err", C.c_double), ("depth", C.c_double), ("surface_x0", C.c_double),
                ("surface_x1", C.c_double), ("surface_bins", C.c_int32)]


class SurReport(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("macro_steps", "network_steps", "judged_steps", "failed_checks",
                                         "plain_steps", "graph_overflows", "rejected_steps")] + \
               [(k, C.c_double) for k in ("last_rho_err", "last_surface_err", "max_rho_err", "max_surface_err")]

    def to_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}
