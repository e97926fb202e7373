"""ctypes binding of the C ABI declared in include/vf_b200.h.

The library is loaded from this package directory (libvfb200.so, built by
``python -m virtualfluids_b200.build``).  There is no fallback: if the shared
library is missing or fails to load, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libvfb200.so"

VFB_OK = 0
VFB_ERR_INVALID_ARGUMENT = -1
VFB_ERR_CUDA = -2
VFB_ERR_UNSUPPORTED = -3
VFB_ERR_NOT_FINITE = -4
VFB_ERR_OUT_OF_RANGE = -5
VFB_ERR_CONFIGURATION = -6

FP32, FP64, FP16, BF16, FX16, FX16W = 0, 1, 2, 3, 4, 5
STORAGE_NAMES = {"fp32": FP32, "fp64": FP64, "fp16": FP16, "bf16": BF16, "fx16": FX16, "fx16w": FX16W}

TEMPLATE_DEFAULT, TEMPLATE_WRITE_MACRO_VARS, TEMPLATE_APPLY_BODY_FORCE, TEMPLATE_ALL_FEATURES = 0, 1, 2, 3

_u32p = ctypes.POINTER(ctypes.c_uint32)


class CollisionArgs(ctypes.Structure):
    """vfb_collision_args (include/vf_b200.h)."""

    _fields_ = [
        ("distributions", ctypes.c_void_p),
        ("numberOfLBnodes", ctypes.c_ulonglong),
        ("neighborX", ctypes.c_void_p),
        ("neighborY", ctypes.c_void_p),
        ("neighborZ", ctypes.c_void_p),
        ("fluidNodeIndices", ctypes.c_void_p),
        ("numberOfFluidNodes", ctypes.c_uint32),
        ("omega", ctypes.c_double),
        ("forces", ctypes.c_double * 3),
        ("forceFactor", ctypes.c_double),
        ("quadricLimiters", ctypes.c_double * 3),
        ("isEvenTimestep", ctypes.c_int),
        ("collisionTemplate", ctypes.c_int),
        ("rho", ctypes.c_void_p),
        ("vx", ctypes.c_void_p),
        ("vy", ctypes.c_void_p),
        ("vz", ctypes.c_void_p),
        ("bodyForceX", ctypes.c_void_p),
        ("bodyForceY", ctypes.c_void_p),
        ("bodyForceZ", ctypes.c_void_p),
    ]


class BcLattice(ctypes.Structure):
    """vfb_bc_lattice (include/vf_b200.h)."""

    _fields_ = [
        ("distributions", ctypes.c_void_p),
        ("numberOfLBnodes", ctypes.c_ulonglong),
        ("neighborX", ctypes.c_void_p),
        ("neighborY", ctypes.c_void_p),
        ("neighborZ", ctypes.c_void_p),
        ("omega", ctypes.c_double),
        ("isEvenTimestep", ctypes.c_int),
    ]


class BcList(ctypes.Structure):
    """vfb_bc_list (include/vf_b200.h)."""

    _fields_ = [
        ("k", ctypes.c_void_p),
        ("q", ctypes.c_void_p),
        ("Vx", ctypes.c_void_p),
        ("Vy", ctypes.c_void_p),
        ("Vz", ctypes.c_void_p),
        ("numberOfBCnodes", ctypes.c_uint32),
        ("locations", ctypes.c_void_p),
    ]


class StressList(ctypes.Structure):
    """vfb_stress_list (include/vf_b200.h)."""

    _fields_ = [(name, ctypes.c_void_p) for name in (
        "k", "kN", "q", "normalX", "normalY", "normalZ", "Vx", "Vy", "Vz", "Vx1", "Vy1", "Vz1", "samplingOffset",
        "z0", "uStar", "Fx", "Fy", "Fz")] + [("numberOfBCnodes", ctypes.c_uint32), ("locations", ctypes.c_void_p)]


class ScalingArgs(ctypes.Structure):
    """vfb_scaling_args (include/vf_b200.h)."""

    _fields_ = [
        ("distributionsCoarse", ctypes.c_void_p),
        ("distributionsFine", ctypes.c_void_p),
        ("neighborXcoarse", ctypes.c_void_p),
        ("neighborYcoarse", ctypes.c_void_p),
        ("neighborZcoarse", ctypes.c_void_p),
        ("neighborXfine", ctypes.c_void_p),
        ("neighborYfine", ctypes.c_void_p),
        ("neighborZfine", ctypes.c_void_p),
        ("numberOfLBnodesCoarse", ctypes.c_ulonglong),
        ("numberOfLBnodesFine", ctypes.c_ulonglong),
        ("isEvenTimestep", ctypes.c_int),
        ("coarseCells", ctypes.c_void_p),
        ("fineCells", ctypes.c_void_p),
        ("numberOfCells", ctypes.c_uint32),
        ("omegaCoarse", ctypes.c_double),
        ("omegaFine", ctypes.c_double),
        ("offsetX", ctypes.c_void_p),
        ("offsetY", ctypes.c_void_p),
        ("offsetZ", ctypes.c_void_p),
        ("fineWriteMask", ctypes.c_void_p),
        ("coarseBlocks", ctypes.c_void_p),
        ("fineBlocks", ctypes.c_void_p),
    ]


(BC_NOSLIP_INTERPOLATED, BC_NOSLIP_BOUNCE_BACK, BC_VELOCITY_INTERPOLATED, BC_VELOCITY_BOUNCE_BACK, BC_SLIP,
 BC_VELOCITY_WITH_PRESSURE, BC_STRESS_INTERPOLATED, BC_STRESS_BOUNCE_BACK, BC_STRESS_BOUNCE_BACK_PRESSURE) = range(9)

# (name, restype, argtypes) of every exported entry point
_SIGNATURES = [
    ("vfb_version", ctypes.c_int, []),
    ("vfb_last_error", ctypes.c_char_p, []),
    ("vfb_storage_bytes", ctypes.c_int, [ctypes.c_int]),
    ("vfb_k17_collision", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(CollisionArgs), ctypes.c_void_p]),
    ("vfb_bgk_collision", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(CollisionArgs), ctypes.c_void_p]),
    ("vfb_init_equilibrium", ctypes.c_int,
     [ctypes.c_int, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
      ctypes.c_void_p]),
    ("vfb_init_nonequilibrium", ctypes.c_int,
     [ctypes.c_int, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_double, ctypes.c_int, ctypes.c_void_p]),
    ("vfb_macroscopic", ctypes.c_int,
     [ctypes.c_int, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p]),
    ("vfb_mass_and_energy", ctypes.c_int,
     [ctypes.c_int, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    ("vfb_mass_and_energy_static", ctypes.c_int,
     [ctypes.c_int, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    ("vfb_bc_post", ctypes.c_int,
     [ctypes.c_int, ctypes.c_int, ctypes.POINTER(BcLattice), ctypes.POINTER(BcList), ctypes.c_void_p]),
    ("vfb_bc_stress", ctypes.c_int,
     [ctypes.c_int, ctypes.c_int, ctypes.POINTER(BcLattice), ctypes.POINTER(StressList), ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("vfb_bc_locations", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p]),
    ("vfb_bc_pressure_noneq", ctypes.c_int,
     [ctypes.c_int, ctypes.POINTER(BcLattice), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
      ctypes.c_int, ctypes.c_void_p]),
    ("vfb_bc_outflow_nonreflecting", ctypes.c_int,
     [ctypes.c_int, ctypes.POINTER(BcLattice), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int,
      ctypes.c_int, ctypes.c_double, ctypes.c_void_p]),
    ("vfb_sim_create", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]),
    ("vfb_sim_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("vfb_sim_levels", ctypes.c_int, [ctypes.c_void_p]),
    ("vfb_sim_init_level", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p]),
    ("vfb_sim_run", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p]),
    ("vfb_sim_macroscopic", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p]),
    ("vfb_sim_mass_and_energy", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    ("vfb_sim_kinetic_energy", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    ("vfb_sim_stress_list", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(StressList)]),
    ("vfb_sim_bc_epilogue_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    ("vfb_collision_plan_set_bc_epilogue", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_uint32,
      ctypes.c_void_p]),
    ("vfb_collision_plan_epilogue_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("vfb_copy_device_to_host", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    ("vfb_sim_level_state", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_ulonglong),
      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]),
    ("vfb_scale_coarse_to_fine", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ScalingArgs), ctypes.c_void_p]),
    ("vfb_scale_fine_to_coarse", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ScalingArgs), ctypes.c_void_p]),
    ("vfb_scaling_blocks", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p]),
    ("vfb_scale_interface", ctypes.c_int,
     [ctypes.c_int, ctypes.POINTER(ScalingArgs), ctypes.POINTER(ScalingArgs), ctypes.c_void_p]),
    ("vfb_scaling_independent", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_int)]),
    ("vfb_debug_scale_host", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ScalingArgs)]),
    ("vfb_scaling_write_mask", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulonglong,
      ctypes.c_void_p]),
    ("vfb_collision_plan_create", ctypes.c_int,
     [ctypes.c_int, ctypes.POINTER(CollisionArgs), ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]),
    ("vfb_collision_plan_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("vfb_collision_plan_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_ulonglong)]),
    ("vfb_collision_plan_check", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("vfb_k17_collision_planned", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(CollisionArgs), ctypes.c_void_p]),
    ("vfb_bgk_collision_planned", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(CollisionArgs), ctypes.c_void_p]),
    ("vfb_debug_collide_node", ctypes.c_int,
     [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.POINTER(ctypes.c_double),
      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    ("vfb_debug_k17_adjoint_node", ctypes.c_int,
     [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_double,
      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    ("vfb_sim_adjoint_forward", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    ("vfb_sim_adjoint_backward", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("vfb_sim_adjoint_schedule", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    ("vfb_saturated_populations", ctypes.c_int,
     [ctypes.c_int, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_void_p]),
    ("vfb_sim_saturated_populations", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_void_p]),
    ("vfb_sim_set_forces", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    ("vfb_sim_output", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("vfb_output_pass", ctypes.c_int,
     [ctypes.c_int, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    ("vfb_sim_set_velocity_bc", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("vfb_debug_init_nonequilibrium_node", ctypes.c_int,
     [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_double,
      ctypes.POINTER(ctypes.c_double)]),
    ("vfb_enstrophy", ctypes.c_int,
     [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulonglong,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    ("vfb_debug_enstrophy_nodes", ctypes.c_int,
     [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulonglong,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p]),
    ("vfb_sim_enstrophy", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                         ctypes.c_void_p]),
    ("vfb_debug_side_qs", ctypes.c_int,
     [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    ("vfb_grid_build", ctypes.c_void_p, [ctypes.POINTER(ctypes.c_double), ctypes.c_int]),
    ("vfb_grid_levels", ctypes.c_int, [ctypes.c_void_p]),
    ("vfb_grid_count", ctypes.c_longlong, [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p]),
    ("vfb_grid_elem_size", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p]),
    ("vfb_grid_copy", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p]),
    ("vfb_grid_free", None, [ctypes.c_void_p]),
    ("vfb_grid_create", ctypes.c_void_p, [ctypes.c_int]),
    ("vfb_grid_put", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p]),
]

_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    """The loaded native library; raises if it is missing."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m virtualfluids_b200.build` "
                    "(there is no CPU fallback)")
            L = ctypes.CDLL(str(LIB_PATH))
            for name, res, args in _SIGNATURES:
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
        return _lib


def exported_symbols() -> list[str]:
    return [s[0] for s in _SIGNATURES]


class VfbError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"vfb error {code}: {message}")
        self.code = code


def check(rc: int) -> None:
    if rc != VFB_OK:
        msg = lib().vfb_last_error()
        raise VfbError(rc, msg.decode() if msg else "")


def last_error() -> str:
    m = lib().vfb_last_error()
    return m.decode() if m else ""
