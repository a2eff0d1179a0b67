"""ctypes mirror of ``simp_params`` (include/simp_gpu.h) and the run presets.

The reference holds every switch and constant as a compile-time Fortran
PARAMETER (fortran/src/modules/globals.f90:58-187 and
data_variables.f90:153-180).  ``reference_default()`` reproduces those shipped
values; ``basin_params()`` derives the parameter set of a synthetic sea-ice
basin (cubic-spline kernel, fixed smoothing length, fixed time step, chosen
forcing) used by the plain, mixed-precision, batched and served workloads.
"""
from __future__ import annotations

import ctypes
import struct

SKF_QUADRATIC = 1
SKF_GAUSSIAN = 2
SKF_QUINTIC = 3
SKF_WENDLAND_C2 = 4
SKF_WENDLAND_C4 = 5
SKF_WENDLAND_C6 = 6
SKF_MARQUIS = 7
SKF_MARQUIS2 = 8
SKF_CUBIC = 9
# kernel code -> the key of its known-answer fixture and its scale_h
KERNELS = {1: ("quadratic", 2), 2: ("gaussian", 3), 3: ("quintic", 3), 4: ("wendland_c2", 1),
           5: ("wendland_c4", 1), 6: ("wendland_c6", 1), 7: ("marquis", 3), 8: ("marquis2", 3),
           9: ("cubic", 2)}
PREC_FP64 = 0
PREC_MIXED = 1

# pair-pass implementations (include/simp_gpu.h, SIMP_PASSES_*)
PASSES_GATHER = 0        # gathers; the kinematic pass's kernel count chosen by size
PASSES_TILED = 1         # shared-memory tiles of a cell row with their halo
PASSES_GATHER_ONE = 2    # gathers, kinematic pass as one kernel
PASSES_GATHER_TWO = 3    # gathers, kinematic pass as pair finding + pair sums
WIND_UNIFORM = 0
WIND_VORTEX = 1

_INT_FIELDS = [
    "int_algorithm", "nnps_algorithm", "sle", "tse", "rheology", "eos_alg",
    "pa_sph", "skf", "den_alg", "bfa", "viscosity", "pressure_force",
    "wind_force", "water_force", "boundary_pressure", "boundary_friction",
    "mass_from_area", "max_ind_int", "hsml_multiplicity", "wind_kind",
    "precision", "reserved0",
]
_DBL_FIELDS = [
    "P_star", "c_eos", "e", "delta_min", "k_t",
    "rho_ice", "rho_air", "rho_water", "c_wind", "c_water",
    "b_length", "kappa_n", "kappa_t", "alpha",
    "wind_u", "wind_v", "current_u", "current_v",
    "vortex_x", "vortex_y", "vortex_umax", "vortex_radius",
    "dt", "max_hsml", "skin",
    "zeta_max", "eta_max", "phi",
    "xi", "Y", "nu",
]
# regularisation switches and constants (after the doubles above)
_TAIL_FIELDS = [
    ("artificial_visc", ctypes.c_int32), ("xsph_regularization", ctypes.c_int32),
    ("art_visc_alg", ctypes.c_int32), ("reserved1", ctypes.c_int32),
    ("alpha_pi", ctypes.c_double), ("beta_pi", ctypes.c_double), ("chi", ctypes.c_double),
]
ART_VISC_HK = 1     # Hernquist and Katz (regularization.f90:102-213)
ART_VISC_MON = 2    # Monaghan (regularization.f90:220-308)


class SimpParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in _INT_FIELDS] + [
        (n, ctypes.c_double) for n in _DBL_FIELDS] + _TAIL_FIELDS

    def copy(self) -> "SimpParams":
        out = SimpParams()
        ctypes.memmove(ctypes.byref(out), ctypes.byref(self), ctypes.sizeof(self))
        return out

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class SimpForcing(ctypes.Structure):
    """Per-basin forcing of a batch (``simp_forcing`` in include/simp_gpu.h)."""
    _fields_ = [("wind_kind", ctypes.c_int32), ("reserved0", ctypes.c_int32),
                ("wind_u", ctypes.c_double), ("wind_v", ctypes.c_double),
                ("vortex_x", ctypes.c_double), ("vortex_y", ctypes.c_double),
                ("vortex_umax", ctypes.c_double), ("vortex_radius", ctypes.c_double)]

    @classmethod
    def of(cls, p: "SimpParams") -> "SimpForcing":
        """The forcing a parameter set describes (its wind fields)."""
        f = cls()
        for name, _ in cls._fields_:
            if name != "reserved0":
                setattr(f, name, getattr(p, name))
        return f


class ServerConfig(ctypes.Structure):
    """``simp_server_config`` (include/simp_serve.h)."""
    _fields_ = [("hbm_budget_bytes", ctypes.c_double), ("max_instances", ctypes.c_int32),
                ("max_request_particles", ctypes.c_int32), ("quantum_steps", ctypes.c_int32),
                ("spot_every", ctypes.c_int32)]


class RequestStats(ctypes.Structure):
    """``simp_request_stats`` (include/simp_serve.h)."""
    _fields_ = [("arrival_s", ctypes.c_double), ("admitted_s", ctypes.c_double),
                ("completed_s", ctypes.c_double), ("steps", ctypes.c_int64), ("ntotal", ctypes.c_int32),
                ("status", ctypes.c_int32), ("spot_checked", ctypes.c_int32), ("reserved0", ctypes.c_int32),
                ("err_v", ctypes.c_double), ("err_h", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    """``simp_server_stats`` (include/simp_serve.h)."""
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("cancelled", ctypes.c_int64),
                ("particle_steps", ctypes.c_int64), ("batch_steps", ctypes.c_int64),
                ("peak_resident_particles", ctypes.c_int64), ("peak_resident_requests", ctypes.c_int32),
                ("reserved0", ctypes.c_int32), ("makespan_s", ctypes.c_double),
                ("capacity_particles", ctypes.c_double), ("admit_s", ctypes.c_double),
                ("step_s", ctypes.c_double), ("retire_s", ctypes.c_double)]


def _real4(v: float) -> float:
    """Value of a Fortran default-real (single precision) literal."""
    return struct.unpack("f", struct.pack("f", v))[0]


def reference_default() -> SimpParams:
    """The shipped PARAMETER values (globals.f90, data_variables.f90)."""
    p = SimpParams()
    p.int_algorithm = 2      # globals.f90:64
    p.nnps_algorithm = 2     # :73
    p.sle = 2                # :81
    p.tse = 2                # :89
    p.rheology = 1           # :96
    p.eos_alg = 3            # :127
    p.pa_sph = 1             # :134
    p.skf = SKF_WENDLAND_C6  # :147
    p.den_alg = 3            # :155
    p.bfa = 1                # :119
    p.viscosity = 1          # :180-187
    p.pressure_force = 1
    p.wind_force = 1
    p.water_force = 1
    p.boundary_pressure = 1
    p.boundary_friction = 0
    p.mass_from_area = 1
    p.max_ind_int = 200      # :24
    p.hsml_multiplicity = 3  # data_variables.f90:105
    p.wind_kind = WIND_UNIFORM
    p.precision = PREC_FP64
    # data_variables.f90:157-180; default-real literals keep single precision
    p.P_star = 2.75e4
    p.c_eos = 20.0
    p.e = 2.0                # 0.5 * (P_star + T_star) / S_star, T_star = 0
    p.delta_min = 2.0e-9
    p.k_t = 0.0              # T_star / P_star
    p.rho_ice = 900.0
    p.rho_air = _real4(1.3)
    p.rho_water = 1026.0
    p.c_wind = 1.2e-3
    p.c_water = 5.5e-3
    p.b_length = 8000.0
    p.kappa_n = 5.4e12
    p.kappa_t = 5.0e-8
    p.alpha = _real4(1.0 / 6.0)   # 1. / (2 * hsml_multiplicity)
    p.wind_u = 0.0               # wind_forcing.f90:36-37
    p.wind_v = _real4(-5.3)
    p.current_u = 0.0            # water_drag.f90:36-37
    p.current_v = 0.0
    p.vortex_x = p.vortex_y = p.vortex_umax = p.vortex_radius = 0.0
    p.dt = 0.0
    p.max_hsml = 0.0
    p.skin = -1.0
    p.zeta_max = 0.0          # data_variables.f90:154, declared without a value
    p.eta_max = 0.0
    p.phi = 45.0              # data_variables.f90:159 (mu = tan(phi pi / 180.), :180)
    p.xi = _real4(0.5225)     # data_variables.f90:175, a default-real literal
    p.Y = 1.0e9               # :157
    p.nu = _real4(0.3)        # :158
    p.artificial_visc = 0     # globals.f90:180-187
    p.xsph_regularization = 0
    p.art_visc_alg = ART_VISC_HK  # globals.f90:103
    p.alpha_pi = 1.0          # data_variables.f90:171
    p.beta_pi = 2.0           # :172
    p.chi = _real4(0.3)       # :173, a default-real literal
    return p


def basin_params(dx: float, *, skf: int = SKF_CUBIC, dt: float = 1.0,
                 wind=(10.0, 0.0), precision: int = PREC_FP64,
                 vortex=None) -> SimpParams:
    """Parameters of a synthetic basin with lattice spacing ``dx``.

    Cubic-spline kernel with SIMP support radius hsml = 2.4 dx (smoothing
    length 1.2 dx, support 2h); fixed hsml and constant mass (sle = 0 with the
    mass update off); fixed dt (tse = 0); wall interaction length
    b_length = 4 dx; Hibler VP rheology with the reference's constants.
    """
    p = reference_default()
    p.skf = skf
    p.sle = 0
    p.mass_from_area = 0
    p.tse = 0
    p.dt = dt
    p.b_length = 4.0 * dx
    p.precision = precision
    if vortex is None:
        p.wind_kind = WIND_UNIFORM
        p.wind_u, p.wind_v = float(wind[0]), float(wind[1])
    else:
        p.wind_kind = WIND_VORTEX
        p.vortex_x, p.vortex_y, p.vortex_umax, p.vortex_radius = (float(v) for v in vortex)
    return p
