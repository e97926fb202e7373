"""The C ABI library loads, exports every entry point include/vf_b200.h
declares, and rejects invalid arguments without touching a GPU."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from virtualfluids_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "vf_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vfb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    assert "vfb_k17_collision" in declared_symbols()


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (vfb_[a-z0-9_]+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert set(declared_symbols()) <= set(_lib.exported_symbols())


def test_version_and_storage_sizes():
    L = _lib.lib()
    assert L.vfb_version() >= 100
    assert [L.vfb_storage_bytes(s) for s in (0, 1, 2, 3, 9)] == [4, 8, 2, 2, 0]


def test_null_args_rejected():
    L = _lib.lib()
    assert L.vfb_k17_collision(0, None, None) == _lib.VFB_ERR_INVALID_ARGUMENT
    assert "NULL" in _lib.last_error()


def test_invalid_omega_rejected():
    a = _lib.CollisionArgs()
    a.distributions = 1
    a.neighborX = a.neighborY = a.neighborZ = a.fluidNodeIndices = 1
    a.numberOfLBnodes = 10
    a.numberOfFluidNodes = 5
    a.omega = 2.5
    rc = _lib.lib().vfb_k17_collision(0, ctypes.byref(a), None)
    assert rc == _lib.VFB_ERR_INVALID_ARGUMENT
    assert "omega" in _lib.last_error()


def test_unknown_storage_rejected():
    a = _lib.CollisionArgs()
    rc = _lib.lib().vfb_k17_collision(7, ctypes.byref(a), None)
    assert rc == _lib.VFB_ERR_INVALID_ARGUMENT


def test_template_needs_macro_arrays():
    a = _lib.CollisionArgs()
    a.distributions = 1
    a.neighborX = a.neighborY = a.neighborZ = a.fluidNodeIndices = 1
    a.numberOfLBnodes = 10
    a.numberOfFluidNodes = 5
    a.omega = 1.5
    a.collisionTemplate = _lib.TEMPLATE_WRITE_MACRO_VARS
    assert _lib.lib().vfb_k17_collision(0, ctypes.byref(a), None) == _lib.VFB_ERR_INVALID_ARGUMENT


def test_empty_fluid_list_is_a_no_op():
    a = _lib.CollisionArgs()
    a.numberOfFluidNodes = 0
    assert _lib.lib().vfb_k17_collision(0, ctypes.byref(a), None) == _lib.VFB_OK


def test_grid_build_rejects_short_spec():
    s = (ctypes.c_double * 10)()
    assert not _lib.lib().vfb_grid_build(s, 10)
    assert "61" in _lib.last_error()


def test_init_nonequilibrium_rejects_bad_arguments():
    L = _lib.lib()
    p = [1] * 9  # placeholders: the checks return before any device access
    assert L.vfb_init_nonequilibrium(0, None, 10, *p[:9], 1.0, 1, None) == _lib.VFB_ERR_INVALID_ARGUMENT
    assert L.vfb_init_nonequilibrium(0, 1, 10, *p[:9], 2.0, 1, None) == _lib.VFB_ERR_INVALID_ARGUMENT
    assert "omega" in _lib.last_error()
    assert L.vfb_init_nonequilibrium(0, 1, 1, *p[:9], 1.0, 1, None) == _lib.VFB_ERR_OUT_OF_RANGE
    assert L.vfb_init_nonequilibrium(9, 1, 10, *p[:9], 1.0, 1, None) == _lib.VFB_ERR_INVALID_ARGUMENT


def test_outflow_rejects_bad_arguments():
    L = _lib.lib()
    t = _lib.BcLattice()
    t.distributions = t.neighborX = t.neighborY = t.neighborZ = 1
    t.numberOfLBnodes = 10
    assert L.vfb_bc_outflow_nonreflecting(0, ctypes.byref(t), 1, 1, 0, 1, 0, 0.0, None) == _lib.VFB_OK  # empty list
    assert L.vfb_bc_outflow_nonreflecting(0, ctypes.byref(t), 1, 1, 4, 7, 0, 0.0, None) == \
        _lib.VFB_ERR_INVALID_ARGUMENT
    assert "direction" in _lib.last_error()
    assert L.vfb_bc_outflow_nonreflecting(0, ctypes.byref(t), None, 1, 4, 1, 0, 0.0, None) == \
        _lib.VFB_ERR_INVALID_ARGUMENT
    assert L.vfb_bc_outflow_nonreflecting(0, ctypes.byref(t), 1, 1, 4, 1, 1, float("nan"), None) == \
        _lib.VFB_ERR_INVALID_ARGUMENT
    assert L.vfb_bc_outflow_nonreflecting(8, ctypes.byref(t), 1, 1, 4, 1, 0, 0.0, None) == \
        _lib.VFB_ERR_INVALID_ARGUMENT


def test_enstrophy_rejects_bad_arguments():
    L = _lib.lib()
    out = (ctypes.c_double * 2)()
    p = [1] * 9
    assert L.vfb_enstrophy(1, *p[:4], 10, *p[:5], None, None) == _lib.VFB_ERR_INVALID_ARGUMENT
    assert L.vfb_enstrophy(1, None, *p[:3], 10, *p[:5], out, None) == _lib.VFB_ERR_INVALID_ARGUMENT
    assert L.vfb_enstrophy(2, *p[:4], 10, *p[:5], out, None) == _lib.VFB_ERR_INVALID_ARGUMENT
    assert "precision" in _lib.last_error()
    assert L.vfb_enstrophy(1, *p[:4], 1, *p[:5], out, None) == _lib.VFB_ERR_OUT_OF_RANGE


def test_parameter_setters_of_the_new_options():
    from virtualfluids_b200.simulation import Parameter, PressureBC
    p = Parameter()
    assert p.use_init_neq is False and p.outflow_pressure_correction_factor == 0.0
    p.set_use_init_neq(True)
    p.set_outflow_pressure_correction_factor(0.25)
    assert p.use_init_neq is True and p.outflow_pressure_correction_factor == 0.25
    assert int(PressureBC.OutflowNonReflective) == 1 and int(PressureBC.OutflowNonReflectivePressureCorrection) == 2


def test_initial_condition_helpers():
    import numpy as np
    from virtualfluids_b200.simulation import Parameter
    p = Parameter()
    x = np.linspace(0.0, 10.0, 11)
    p.set_initial_condition_uniform(0.01, -0.02, 0.0)
    rho, vx, vy, vz = p.initial_condition(x, x, x)
    assert np.all(rho == 0) and np.all(vx == 0.01) and np.all(vy == -0.02) and np.all(vz == 0)
    p.set_initial_condition_log_law(0.3, 0.1, 10.0)
    _, vx, vy, _ = p.initial_condition(x, x, x - 1.0)
    assert vx[0] == 0.0 and vx[1] == 0.0  # z clipped at 0
    assert abs(vx[-1] - 0.3 / 0.4 * np.log(9.0 / 0.1 + 1.0) / 10.0) < 1e-15 and np.all(vy == 0)
    p.set_initial_condition_perturbed_log_law(0.3, 0.1, 100.0, 50.0, 20.0, 10.0)
    _, vx, vy, vz = p.initial_condition(x, x, x)
    assert np.all(np.isfinite(vx)) and np.all(np.isfinite(vz)) and np.abs(vy).max() > 0


def test_geometry_bc_setter_accepts_plain_ints():
    """set_geometry_boundary_condition takes either enum's members or their
    plain values: no-slip kinds first, then the velocity kinds."""
    from virtualfluids_b200.simulation import BoundaryConditionFactory, NoSlipBC, Parameter, VelocityBC
    bc = BoundaryConditionFactory()
    for kind in NoSlipBC:
        bc.set_geometry_boundary_condition(int(kind))
        assert bc.geometry is kind
    for kind in VelocityBC:
        bc.set_geometry_boundary_condition(int(kind))
        assert bc.geometry is kind
        bc.set_geometry_boundary_condition(kind)
        assert bc.geometry is kind
    with pytest.raises(ValueError):
        bc.set_geometry_boundary_condition(99)
    p = Parameter()
    assert p.velocity_ratio == 1.0
    p.set_velocity_ratio(2.5)
    assert p.velocity_ratio == 2.5
    with pytest.raises(ValueError):
        p.set_velocity_ratio(0.0)


def test_sim_params_layout_matches_header():
    """The ctypes mirror of vfb_sim_params lists the header's fields in order."""
    import re
    from pathlib import Path
    from virtualfluids_b200.simulation import VfbSimParams
    text = Path(__file__).resolve().parents[1].joinpath("include", "vf_b200.h").read_text()
    body = text[text.index("typedef struct vfb_sim_params {"):text.index("} vfb_sim_params;")]
    names = re.findall(r"^\s+(?:int|double)\s+(\w+)", body, re.M)
    assert names == [f[0] for f in VfbSimParams._fields_]


def test_stress_selection_and_wall_model_reader_exist():
    """The stress kinds, the simulation parameters' wall-model fields and the
    readers are bound (no GPU call)."""
    from virtualfluids_b200 import _lib
    from virtualfluids_b200.simulation import BoundaryConditionFactory, Parameter, StressBC, VfbSimParams

    L = _lib.lib()
    for name in ("vfb_bc_stress", "vfb_sim_stress_list", "vfb_copy_device_to_host"):
        assert hasattr(L, name)
    names = [f[0] for f in VfbSimParams._fields_]
    assert names[-3:] == ["stressBC", "hasWallModelMonitor", "bcEpilogue"]
    bc = BoundaryConditionFactory()
    assert bc.stress == StressBC.NotSpecified
    bc.set_stress_boundary_condition(StressBC.StressBounceBackPressureCompressible)
    assert int(bc.stress) == _lib.BC_STRESS_BOUNCE_BACK_PRESSURE == 8
    p = Parameter()
    p.set_has_wall_model_monitor(True)
    assert p.has_wall_model_monitor
    assert L.vfb_copy_device_to_host(None, None, 0, None) == 0


def test_stress_builder_api_errors():
    from virtualfluids_b200.grid import MultipleGridBuilder, SideType

    b = MultipleGridBuilder()
    b.addCoarseGrid(0, 0, 0, 7, 7, 7, 1.0)
    b.buildGrids()
    with pytest.raises(ValueError):
        b.setStressBoundaryCondition(SideType.GEOMETRY, 0, 0, 1, 2, 0.1, 1.0)
    with pytest.raises(ValueError):
        b.setStressBoundaryCondition(SideType.MZ, 0, 0, 1, 1.5, 0.1, 1.0)
    # a sampling node beyond the far side of the box is an error of the build
    b.setStressBoundaryCondition(SideType.MZ, 0, 0, 1, 40, 0.1, 1.0)
    with pytest.raises(_lib.VfbError):
        b.arrays()
