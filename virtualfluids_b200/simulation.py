"""pyfluids-style host API over the simulation C ABI.

Mirrors the names of the reference's Python bindings
(pythonbindings/src/gpu/submodules/simulation.cpp:52-79, parameter.cpp:60-143,
boundary_conditions.cpp:42-82): a ``Parameter``, a ``BoundaryConditionFactory``
and a ``Simulation(parameter, gridBuilder, bcFactory, gridScalingFactory)``
whose ``run`` crosses into the library once and runs the whole time loop in
C++ (the recursive per-level schedule of UpdateGrid27).
"""
from __future__ import annotations

import ctypes
import enum

import numpy as np

from . import _lib
from .grid import MultipleGridBuilder, export_level


class VfbSimParams(ctypes.Structure):
    """vfb_sim_params (include/vf_b200.h)."""

    _fields_ = [
        ("storage", ctypes.c_int),
        ("collisionKernel", ctypes.c_int),
        ("velocityBC", ctypes.c_int),
        ("noSlipBC", ctypes.c_int),
        ("geometryBC", ctypes.c_int),
        ("slipBC", ctypes.c_int),
        ("pressureBC", ctypes.c_int),
        ("viscosity", ctypes.c_double),
        ("forces", ctypes.c_double * 3),
        ("quadricLimiters", ctypes.c_double * 3),
        ("usePlan", ctypes.c_int),
        ("useGraphs", ctypes.c_int),
        ("useInitNeq", ctypes.c_int),
        ("outflowPressureCorrectionFactor", ctypes.c_double),
        ("velocityRatio", ctypes.c_double),
        ("stressBC", ctypes.c_int),
        ("hasWallModelMonitor", ctypes.c_int),
        ("bcEpilogue", ctypes.c_int),
    ]


class VelocityBC(enum.IntEnum):
    VelocityInterpolatedCompressible = _lib.BC_VELOCITY_INTERPOLATED
    VelocityBounceBack = _lib.BC_VELOCITY_BOUNCE_BACK
    VelocityWithPressureInterpolatedCompressible = _lib.BC_VELOCITY_WITH_PRESSURE


class NoSlipBC(enum.IntEnum):
    NoSlipDelayBounceBack = -1  # no kernel: bounce-back through the stopper nodes
    NoSlipInterpolatedCompressible = _lib.BC_NOSLIP_INTERPOLATED
    NoSlipBounceBack = _lib.BC_NOSLIP_BOUNCE_BACK


class SlipBC(enum.IntEnum):
    NotSpecified = -1
    SlipCompressible = _lib.BC_SLIP


class StressBC(enum.IntEnum):
    NotSpecified = -1
    StressCompressible = _lib.BC_STRESS_INTERPOLATED
    StressBounceBackCompressible = _lib.BC_STRESS_BOUNCE_BACK
    StressBounceBackPressureCompressible = _lib.BC_STRESS_BOUNCE_BACK_PRESSURE


class PressureBC(enum.IntEnum):
    NotSpecified = -1
    PressureNonEquilibriumCompressible = 0
    OutflowNonReflective = 1
    OutflowNonReflectivePressureCorrection = 2


KERNELS = {"K17CompressibleNavierStokes": 0, "BGKCompSP27": 1}


class BoundaryConditionFactory:
    """Selection of the BC kernels (BoundaryConditionFactory.h:75-162)."""

    def __init__(self):
        self.velocity = VelocityBC.VelocityInterpolatedCompressible
        self.no_slip = NoSlipBC.NoSlipDelayBounceBack
        self.geometry = NoSlipBC.NoSlipDelayBounceBack
        self.slip = SlipBC.NotSpecified
        self.stress = StressBC.NotSpecified
        self.pressure = PressureBC.NotSpecified

    def set_velocity_boundary_condition(self, boundary_condition_type: VelocityBC):
        self.velocity = VelocityBC(boundary_condition_type)

    def set_no_slip_boundary_condition(self, boundary_condition_type: NoSlipBC):
        self.no_slip = NoSlipBC(boundary_condition_type)

    def set_geometry_boundary_condition(self, boundary_condition_type):
        """A no-slip kind, or a velocity kind for a geometry given a velocity
        (setVelocityBoundaryCondition(SideType.GEOMETRY, ...)).  Plain ints are
        looked up among the no-slip kinds first, then the velocity kinds, as
        the reference's variant setter accepts either enum."""
        if isinstance(boundary_condition_type, (VelocityBC, NoSlipBC)):
            self.geometry = boundary_condition_type
            return
        try:
            self.geometry = NoSlipBC(boundary_condition_type)
        except ValueError:
            self.geometry = VelocityBC(boundary_condition_type)

    def set_slip_boundary_condition(self, boundary_condition_type: SlipBC):
        self.slip = SlipBC(boundary_condition_type)

    def set_stress_boundary_condition(self, boundary_condition_type: StressBC):
        self.stress = StressBC(boundary_condition_type)

    def set_pressure_boundary_condition(self, boundary_condition_type: PressureBC):
        self.pressure = PressureBC(boundary_condition_type)


class Parameter:
    """The subset of Parameter the time step reads (Parameter.cpp:69,395-420)."""

    def __init__(self):
        self.viscosity = 0.001
        self.forcing = (0.0, 0.0, 0.0)
        self.quadric_limiters = (0.01, 0.01, 0.01)
        self.main_kernel = "K17CompressibleNavierStokes"
        self.storage = "fp64"
        self.use_plan = True
        self.use_graphs = True
        self.use_init_neq = False
        # the reference leaves it unset; it matters only for
        # PressureBC.OutflowNonReflectivePressureCorrection
        self.outflow_pressure_correction_factor = 0.0
        # world-to-lattice velocity ratio; only the geometry list's velocities
        # are divided by it (GridGenerator.cpp:507-513)
        self.velocity_ratio = 1.0
        self.has_wall_model_monitor = False
        # True: the planned collision applies the post-collision BCs of its
        # wall nodes itself (the same result).  Off by default: measured slower
        # on B200 (an x-face wall puts one BC node in every row, so the
        # epilogue runs in one lane of most warps)
        self.use_bc_epilogue = False
        self.initial_condition = None

    def set_viscosity_LB(self, viscosity: float):
        self.viscosity = float(viscosity)

    def set_forcing(self, forcing_x: float, forcing_y: float, forcing_z: float):
        self.forcing = (float(forcing_x), float(forcing_y), float(forcing_z))

    def set_quadric_limiters(self, quadric_limiter_p: float, quadric_limiter_m: float, quadric_limiter_d: float):
        self.quadric_limiters = (float(quadric_limiter_p), float(quadric_limiter_m), float(quadric_limiter_d))

    def configure_main_kernel(self, kernel: str):
        if kernel not in KERNELS:
            raise ValueError(f"unknown kernel {kernel!r}; known: {sorted(KERNELS)}")
        self.main_kernel = kernel

    def set_storage(self, storage: str):
        """Population storage: "fp64", "fp32", or the 16-bit forms "fp16" /
        "bf16" / "fx16" / "fx16w" (fixed point relative to the weight over a
        quarter of it, or over a range that widens with the direction's
        non-zero components; see vf_b200.h)."""
        if storage not in _lib.STORAGE_NAMES:
            raise ValueError(f"unknown storage {storage!r}")
        self.storage = storage

    def set_use_init_neq(self, use_init_neq: bool):
        """Initialise with the equilibrium plus the first-order strain-rate
        part computed from the initial velocity field (Parameter::setUseInitNeq,
        InitNavierStokesCompressibleNonEquilibrium_Device) instead of the
        equilibrium alone."""
        self.use_init_neq = bool(use_init_neq)

    def set_outflow_pressure_correction_factor(self, correction_factor: float):
        """Parameter::setOutflowPressureCorrectionFactor: the density
        correction of OutflowNonReflectivePressureCorrection."""
        self.outflow_pressure_correction_factor = float(correction_factor)

    def set_velocity_ratio(self, velocity_ratio: float):
        """Parameter::setVelocityRatio.  The grid generator divides the
        geometry BC's velocities by it when it uploads them
        (GridGenerator.cpp:507-513); side velocity BCs are not scaled."""
        if not velocity_ratio > 0.0:
            raise ValueError("velocity ratio must be positive")
        self.velocity_ratio = float(velocity_ratio)

    def set_has_wall_model_monitor(self, has_wall_model_monitor: bool):
        """The stress kernels write u* and the wall momentum per entry
        (Parameter::setHasWallModelMonitor); read them with
        Simulation.wall_model()."""
        self.has_wall_model_monitor = bool(has_wall_model_monitor)

    def set_initial_condition(self, init_func):
        """init_func(x, y, z) -> (drho, vx, vy, vz), evaluated on numpy arrays of coordinates."""
        self.initial_condition = init_func

    # The pyfluids helpers (pythonbindings/src/gpu/submodules/parameter.cpp:98-133),
    # evaluated in FP64 on the coordinate arrays.
    def set_initial_condition_uniform(self, velocity_x: float, velocity_y: float, velocity_z: float):
        """drho = 0 and a uniform velocity."""
        v = (float(velocity_x), float(velocity_y), float(velocity_z))
        self.initial_condition = lambda x, y, z: (0.0 * x, v[0] + 0.0 * x, v[1] + 0.0 * x, v[2] + 0.0 * x)

    def set_initial_condition_log_law(self, u_star: float, z0: float, velocity_ratio: float):
        """vx = u_star / 0.4 * log(max(z, 0) / z0 + 1) / velocity_ratio (von Karman constant 0.4)."""
        def f(x, y, z):
            zc = np.maximum(z, 0.0)
            vx = u_star / 0.4 * np.log(zc / z0 + 1.0) / velocity_ratio
            return 0.0 * x, vx, 0.0 * x, 0.0 * x
        self.initial_condition = f

    def set_initial_condition_perturbed_log_law(self, u_star: float, z0: float, length_x: float, length_z: float,
                                                height: float, velocity_ratio: float):
        """The log law plus the sinusoidal perturbations of the reference's
        atmospheric boundary-layer set-up."""
        def f(x, y, z):
            zc = np.maximum(z, 0.0)
            bump = 2.0 * np.sin(np.pi * 16.0 * x / length_x) * np.sin(np.pi * 8.0 * zc / height) / \
                ((zc / height) ** 2 + 1.0)
            vx = (u_star / 0.4 * np.log(zc / z0 + 1.0) + bump) / velocity_ratio
            vy = bump / velocity_ratio
            vz = 8.0 * u_star / 0.4 * (np.sin(np.pi * 8.0 * y / height) * np.sin(np.pi * 8.0 * zc / height) +
                                       np.sin(np.pi * 8.0 * x / length_x)) / \
                ((0.5 * length_z - zc) ** 2 + 1.0) / velocity_ratio
            return 0.0 * x, vx, vy, vz
        self.initial_condition = f


def grid_from_arrays(levels) -> int:
    """A vfb_grid container holding the given levels (a list of dicts of named
    arrays, as MultipleGridBuilder.arrays() or another grid provider returns
    them, interface cells included).  The caller frees it with vfb_grid_free."""
    L = _lib.lib()
    h = L.vfb_grid_create(len(levels))
    if not h:
        raise _lib.VfbError(_lib.VFB_ERR_INVALID_ARGUMENT, _lib.last_error())
    try:
        for lvl, arrays in enumerate(levels):
            for name, a in arrays.items():
                a = np.ascontiguousarray(a)
                _lib.check(L.vfb_grid_put(h, lvl, name.encode(), a.itemsize, a.size, a.ctypes.data))
    except Exception:
        L.vfb_grid_free(h)
        raise
    return h


class Simulation:
    """Simulation(parameter, gridBuilder, bcFactory[, gridScalingFactory]).

    gridBuilder is a MultipleGridBuilder, or the list of per-level array dicts
    of another grid provider (e.g. a grid made by the reference's builder)."""

    def __init__(self, parameter: Parameter, gridBuilder: MultipleGridBuilder, bcFactory: BoundaryConditionFactory,
                 gridScalingFactory=None, stream=None):
        self.parameter = parameter
        self.stream = 0 if stream is None else int(stream)
        L = _lib.lib()
        p = VfbSimParams()
        p.storage = _lib.STORAGE_NAMES[parameter.storage]
        p.collisionKernel = KERNELS[parameter.main_kernel]
        p.velocityBC = int(bcFactory.velocity)
        p.noSlipBC = int(bcFactory.no_slip)
        p.geometryBC = int(bcFactory.geometry)
        p.slipBC = int(bcFactory.slip)
        p.pressureBC = int(bcFactory.pressure)
        p.viscosity = parameter.viscosity
        p.forces[:] = parameter.forcing
        p.quadricLimiters[:] = parameter.quadric_limiters
        p.usePlan = int(bool(parameter.use_plan))
        p.useGraphs = int(bool(parameter.use_graphs))
        p.useInitNeq = int(bool(parameter.use_init_neq))
        p.outflowPressureCorrectionFactor = parameter.outflow_pressure_correction_factor
        p.velocityRatio = parameter.velocity_ratio
        p.stressBC = int(bcFactory.stress)
        p.hasWallModelMonitor = int(bool(parameter.has_wall_model_monitor))
        p.bcEpilogue = int(bool(parameter.use_bc_epilogue))
        self._double = p.storage == _lib.FP64
        if isinstance(gridBuilder, MultipleGridBuilder):
            spec = gridBuilder.full_spec()
            grid = L.vfb_grid_build(spec.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(spec))
        else:
            grid = grid_from_arrays(gridBuilder)
        if not grid:
            raise _lib.VfbError(_lib.VFB_ERR_CONFIGURATION, _lib.last_error())
        try:
            self.levels = [export_level(L, grid, lvl, "vfb_grid") for lvl in range(L.vfb_grid_levels(grid))]
            h = ctypes.c_void_p()
            _lib.check(L.vfb_sim_create(ctypes.byref(p), grid, ctypes.byref(h), self.stream))
            self._h = h
        finally:
            L.vfb_grid_free(grid)
        if parameter.initial_condition is not None:
            for lvl, g in enumerate(self.levels):
                fields = parameter.initial_condition(g["coordX"], g["coordY"], g["coordZ"])
                solid = g["geo"] != 19
                arrays = []
                for f in fields:
                    a = np.array(np.broadcast_to(f, g["coordX"].shape), dtype=np.float64)
                    a[solid] = 0.0
                    arrays.append(a)
                self.init_level(lvl, *arrays)

    @property
    def real(self):
        return np.float64 if self._double else np.float32

    def init_level(self, level: int, drho, vx, vy, vz):
        a = [np.ascontiguousarray(x, dtype=self.real) for x in (drho, vx, vy, vz)]
        _lib.check(_lib.lib().vfb_sim_init_level(self._h, level, *[x.ctypes.data for x in a], self.stream))

    def run(self, steps: int = 1):
        _lib.check(_lib.lib().vfb_sim_run(self._h, int(steps), self.stream))

    def macroscopic(self, level: int = 0, out=None):
        """(drho, vx, vy, vz) host arrays of a level, into `out` (four
        contiguous arrays of the compute precision, e.g. views of pinned
        buffers for fast copies) when given."""
        N = len(self.levels[level]["geo"])
        if out is None:
            out = [np.zeros(N, self.real) for _ in range(4)]
        elif len(out) != 4 or any(o.dtype != self.real or o.size != N or not o.flags.c_contiguous for o in out):
            raise ValueError(f"out must be four contiguous {np.dtype(self.real).name} arrays of {N} elements")
        _lib.check(_lib.lib().vfb_sim_macroscopic(self._h, level, *[o.ctypes.data for o in out], self.stream))
        return out

    def mass_and_energy(self, level: int = 0):
        out = (ctypes.c_double * 3)()
        _lib.check(_lib.lib().vfb_sim_mass_and_energy(self._h, level, out, self.stream))
        return out[0], out[1], int(out[2])

    def kinetic_energy(self, level: int = 0):
        """KineticEnergyAnalyzer's value: mean (1 + drho) |u|^2 / 2 over the
        fluid nodes whose six axis neighbours are fluid (FP64 sum), and their number."""
        out = (ctypes.c_double * 2)()
        _lib.check(_lib.lib().vfb_sim_kinetic_energy(self._h, level, out, self.stream))
        return out[0], int(out[1])

    def enstrophy(self, level: int = 0):
        """EnstrophyAnalyzer's value: mean 1/2 (1 + drho) |curl u|^2 over the
        fluid nodes whose six axis neighbours are fluid (FP64 sum), and their
        number."""
        out = (ctypes.c_double * 2)()
        _lib.check(_lib.lib().vfb_sim_enstrophy(self._h, level, out, self.stream))
        return out[0], int(out[1])

    def output(self, level: int = 0, fields: bool = True):
        """The level's output in one pass over its populations: a dict of the
        FP64 sums (mass, energy, non-finite count over the fluid list), the
        kinetic-energy and enstrophy analyzers' means and node counts, and,
        with fields=True, the host arrays drho, vx, vy, vz."""
        out = (ctypes.c_double * 8)()
        N = len(self.levels[level]["geo"])
        arrays = [np.zeros(N, self.real) for _ in range(4)] if fields else [None] * 4
        ptrs = [None if a is None else a.ctypes.data for a in arrays]
        _lib.check(_lib.lib().vfb_sim_output(self._h, level, out, *ptrs, self.stream))
        r = {"mass": out[0], "energy": out[1], "nonfinite": int(out[2]), "kinetic_energy": out[3],
             "kinetic_energy_nodes": int(out[4]), "enstrophy": out[5], "enstrophy_nodes": int(out[6]),
             "fluid_nodes": int(out[7])}
        if fields:
            r["fields"] = arrays
        return r

    def set_forces(self, fx: float, fy: float, fz: float):
        """The global force of the following steps (Parameter::setForcing)."""
        g = (ctypes.c_double * 3)(float(fx), float(fy), float(fz))
        _lib.check(_lib.lib().vfb_sim_set_forces(self._h, g))

    def set_velocity_bc(self, vx, vy, vz, level: int = 0):
        """The velocities of every entry of a level's velocity list (in the
        list's order, levels[level]["velocity.k"]), from the next step on."""
        n = len(self.levels[level]["velocity.k"])
        a = [np.ascontiguousarray(np.broadcast_to(np.asarray(v, np.float64), (n,))) for v in (vx, vy, vz)]
        _lib.check(_lib.lib().vfb_sim_set_velocity_bc(self._h, level, *[x.ctypes.data for x in a], self.stream))
        for c, x in zip(("vx", "vy", "vz"), a):
            self.levels[level][f"velocity.{c}"] = x.copy()

    def adjoint_forward(self, steps: int, checkpoint_interval: int, nodes, wx, wy=None, wz=None) -> float:
        """Run `steps` steps (the state advances) keeping a checkpoint every
        `checkpoint_interval` steps, and return the objective
        J = sum_j wx[j] ux + wy[j] uy + wz[j] uz at the nodes `nodes` of the
        final state (single-level simulations; see vfb_sim_adjoint_forward)."""
        nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
        n = len(nodes)
        w = [np.ascontiguousarray(np.broadcast_to(np.asarray(0.0 if v is None else v, np.float64), (n,)))
             for v in (wx, wy, wz)]
        J = ctypes.c_double()
        _lib.check(_lib.lib().vfb_sim_adjoint_forward(self._h, int(steps), int(checkpoint_interval), nodes.ctypes.data,
                                                      *[x.ctypes.data for x in w], n, ctypes.byref(J), self.stream))
        return J.value

    def adjoint_backward(self, seed: float = 1.0):
        """Gradients of seed * J from the last adjoint_forward: (dJ/dU of the
        velocity list as an array of shape (3, n), dJ/d(global force) of shape (3,))."""
        n = len(self.levels[0]["velocity.k"])
        dv = np.zeros((3, n), np.float64)
        df = np.zeros(3, np.float64)
        _lib.check(_lib.lib().vfb_sim_adjoint_backward(self._h, float(seed), dv.ctypes.data, df.ctypes.data,
                                                       self.stream))
        return dv, df

    def saturated_populations(self, level: int = 0) -> int:
        """How many stored populations of the level sit at the ends of the FX16
        or FX16W range (deviations clipped on store); 0 for the other
        storages."""
        n = ctypes.c_ulonglong()
        _lib.check(_lib.lib().vfb_sim_saturated_populations(self._h, level, ctypes.byref(n), self.stream))
        return n.value

    def adjoint_schedule(self) -> dict:
        """The schedule of the last adjoint_forward: whether the BC lists run in
        one launch per step, and whether the forward pass taped its only
        segment (checkpoint_interval >= steps: no recomputation backwards)."""
        out = (ctypes.c_int * 2)()
        _lib.check(_lib.lib().vfb_sim_adjoint_schedule(self._h, out))
        return {"lists_together": bool(out[0]), "taped_forward": bool(out[1])}

    def bc_epilogue_stats(self, level: int = 0) -> tuple[int, int, int]:
        """(nodes, BC entries) the level's collision applies in its BC
        epilogue, and the entries left to the separate BC launches."""
        out = (ctypes.c_ulonglong * 3)()
        _lib.check(_lib.lib().vfb_sim_bc_epilogue_stats(self._h, level, out))
        return int(out[0]), int(out[1]), int(out[2])

    def wall_model(self, level: int = 0) -> dict[str, np.ndarray]:
        """The level's stress list and wall-model arrays as host copies: the
        filter states Vx, Vy, Vz (sampling node) and Vx1, Vy1, Vz1 (wall
        node) and, with the monitor, uStar, Fx, Fy, Fz; empty when the level
        has no stress list."""
        L = _lib.lib()
        lst = _lib.StressList()
        _lib.check(L.vfb_sim_stress_list(self._h, level, ctypes.byref(lst)))
        n = int(lst.numberOfBCnodes)
        out = {}
        if n == 0:
            return out
        names = ["Vx", "Vy", "Vz", "Vx1", "Vy1", "Vz1", "uStar", "Fx", "Fy", "Fz"]
        for name in names:
            ptr = getattr(lst, name)
            if not ptr:
                continue
            a = np.zeros(n, self.real)
            _lib.check(L.vfb_copy_device_to_host(a.ctypes.data, ptr, a.nbytes, self.stream))
            out[name] = a
        return out

    def level_state(self, level: int = 0):
        """(device pointer of the populations, N, isEvenTimestep, omega)."""
        ptr = ctypes.c_void_p()
        n = ctypes.c_ulonglong()
        ev = ctypes.c_int()
        om = ctypes.c_double()
        _lib.check(_lib.lib().vfb_sim_level_state(self._h, level, ctypes.byref(ptr), ctypes.byref(n), ctypes.byref(ev),
                                                  ctypes.byref(om)))
        return ptr.value, n.value, bool(ev.value), om.value

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().vfb_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
