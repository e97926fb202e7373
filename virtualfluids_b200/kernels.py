"""Thin Python access to the kernel entry points of the C ABI, on torch CUDA
tensors (torch provides device memory and the stream; the arithmetic is in
libvfb200.so).

This is the level of VirtualFluids' kernel launchers: one call is one launch of
a collision, init or macroscopic kernel on one level.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the environment
    torch = None

STORAGE_OF_DTYPE = {}
if torch is not None:
    STORAGE_OF_DTYPE = {torch.float32: _lib.FP32, torch.float64: _lib.FP64, torch.float16: _lib.FP16,
                        torch.bfloat16: _lib.BF16, torch.int16: _lib.FX16}


# FP16 storage holds the shifted populations times this power of two (so that
# deviations of order 1e-6 stay normal numbers); the kernels undo it on load
HALF_STORAGE_SCALE = 4096.0
# FX16 storage holds q = round((f_d - w_d) * 2^17 / w_d) as int16
WEIGHTS = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)
FX16_SCALE = 2.0 ** 17 / WEIGHTS


def storage_scale(storage_dtype):
    """Factor between a population and its stored number: a scalar (1 except
    FP16), or for FX16 an array of 27 per-slot factors (2^17 / w_d)."""
    if storage_dtype == torch.int16:
        return FX16_SCALE
    return HALF_STORAGE_SCALE if storage_dtype == torch.float16 else 1.0


def decode(dist) -> np.ndarray:
    """The populations f_d - w_d (FP64 host array, 27 * N) of a stored array."""
    a = dist.detach().cpu().to(torch.float64).numpy()
    s = storage_scale(dist.dtype)
    if np.ndim(s):
        return (a.reshape(27, -1) / s[:, None]).ravel()
    return a / s


def encode(values, storage_dtype, device="cuda"):
    """A stored array (27 * N) of the given populations f_d - w_d."""
    v = np.asarray(values, dtype=np.float64)
    s = storage_scale(storage_dtype)
    if np.ndim(s):
        q = np.clip(np.rint(v.reshape(27, -1) * s[:, None]), -32768, 32767).ravel()
        return torch.from_numpy(q.astype(np.int16)).to(device)
    return torch.from_numpy(v * s).to(device, storage_dtype)


def compute_dtype(storage_dtype):
    return torch.float64 if storage_dtype == torch.float64 else torch.float32


def _p(t) -> int | None:
    return None if t is None else t.data_ptr()


def _stream(stream) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


@dataclass
class DeviceLattice:
    """Index arrays of one grid level on the device (LBMSimulationParameter fields)."""

    N: int
    neighborX: "torch.Tensor"
    neighborY: "torch.Tensor"
    neighborZ: "torch.Tensor"
    geo: "torch.Tensor"
    fluid: "torch.Tensor"
    # the -x-y-z neighbour (neighborInverse / neighborWSB of the reference),
    # needed only by the non-equilibrium initialisation
    neighborInverse: "torch.Tensor | None" = None

    @staticmethod
    def from_arrays(g: dict[str, np.ndarray], device="cuda") -> "DeviceLattice":
        def u32(a):
            return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(device)
        inverse = u32(g["neighborNeg"]) if "neighborNeg" in g else None
        return DeviceLattice(len(g["geo"]), u32(g["neighborX"]), u32(g["neighborY"]), u32(g["neighborZ"]),
                             u32(g["geo"]), u32(g["fluid"]), inverse)

    @property
    def numberOfFluidNodes(self) -> int:
        return int(self.fluid.numel())


def new_distributions(lat: DeviceLattice, dtype, device="cuda"):
    return torch.zeros(27 * lat.N, dtype=dtype, device=device)


def collision_args(dist, lat: DeviceLattice, omega: float, is_even: bool, *, forces=(0.0, 0.0, 0.0),
                   force_factor: float = 1.0, limiters=(0.01, 0.01, 0.01), template: int = 0, macro=None, body=None,
                   fluid=None) -> _lib.CollisionArgs:
    nodes = lat.fluid if fluid is None else fluid
    a = _lib.CollisionArgs()
    a.distributions = dist.data_ptr() if dist is not None else None
    a.numberOfLBnodes = lat.N
    a.neighborX = lat.neighborX.data_ptr()
    a.neighborY = lat.neighborY.data_ptr()
    a.neighborZ = lat.neighborZ.data_ptr()
    a.fluidNodeIndices = nodes.data_ptr()
    a.numberOfFluidNodes = int(nodes.numel())
    a.omega = float(omega)
    a.forces[:] = [float(x) for x in forces]
    a.forceFactor = float(force_factor)
    a.quadricLimiters[:] = [float(x) for x in limiters]
    a.isEvenTimestep = int(bool(is_even))
    a.collisionTemplate = int(template)
    if macro is not None:
        a.rho, a.vx, a.vy, a.vz = [_p(t) for t in macro]
    if body is not None:
        a.bodyForceX, a.bodyForceY, a.bodyForceZ = [_p(t) for t in body]
    return a


def collision(kernel: str, dist, lat: DeviceLattice, omega: float, is_even: bool, *, plan=None, stream=None,
              **kw) -> None:
    """One fused collide + stream pass (``kernel`` is "K17" or "BGK"); with a
    CollisionPlan the planned (bulk-copy) kernel is used."""
    a = collision_args(dist, lat, omega, is_even, **kw)
    L = _lib.lib()
    if plan is not None:
        if plan.dtype != dist.dtype:
            raise ValueError("plan was built for another storage type")
        fn = L.vfb_k17_collision_planned if kernel.upper() == "K17" else L.vfb_bgk_collision_planned
        _lib.check(fn(plan.handle, ctypes.byref(a), _stream(stream)))
        return
    storage = STORAGE_OF_DTYPE[dist.dtype]
    fn = L.vfb_k17_collision if kernel.upper() == "K17" else L.vfb_bgk_collision
    _lib.check(fn(storage, ctypes.byref(a), _stream(stream)))


class CollisionPlan:
    """vfb_collision_plan for one level (fluid list and neighbour arrays)."""

    def __init__(self, dtype, lat: DeviceLattice, fluid=None, stream=None):
        self.dtype = dtype
        self.lat = lat
        self.fluid = lat.fluid if fluid is None else fluid
        a = collision_args(None, lat, 1.0, True, fluid=self.fluid)
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().vfb_collision_plan_create(STORAGE_OF_DTYPE[dtype], ctypes.byref(a), ctypes.byref(h),
                                                        _stream(stream)))
        self.handle = h

    def stats(self) -> dict[str, int]:
        out = (ctypes.c_ulonglong * 6)()
        _lib.check(_lib.lib().vfb_collision_plan_stats(self.handle, out))
        keys = ("tiles", "bulk_tiles", "lane_tiles", "bulk_nodes", "wrap_nodes", "lane_nodes")
        return dict(zip(keys, [int(x) for x in out]))

    def check(self, stream=None) -> None:
        _lib.check(_lib.lib().vfb_collision_plan_check(self.handle, _stream(stream)))

    def close(self) -> None:
        if getattr(self, "handle", None):
            _lib.lib().vfb_collision_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def init_equilibrium(dist, lat: DeviceLattice, rho, vx, vy, vz, is_even: bool, stream=None) -> None:
    storage = STORAGE_OF_DTYPE[dist.dtype]
    _lib.check(_lib.lib().vfb_init_equilibrium(storage, dist.data_ptr(), lat.N, lat.geo.data_ptr(),
                                               lat.neighborX.data_ptr(), lat.neighborY.data_ptr(),
                                               lat.neighborZ.data_ptr(), rho.data_ptr(), vx.data_ptr(),
                                               vy.data_ptr(), vz.data_ptr(), int(bool(is_even)), _stream(stream)))


def init_nonequilibrium(dist, lat: DeviceLattice, rho, vx, vy, vz, omega: float, is_even: bool,
                        stream=None) -> None:
    """InitNavierStokesCompressibleNonEquilibrium_Device: equilibrium plus the
    strain-rate part from central differences of (vx, vy, vz); the lattice
    needs its inverse neighbour array."""
    if lat.neighborInverse is None:
        raise _lib.VfbError(_lib.VFB_ERR_INVALID_ARGUMENT, "lattice has no inverse neighbour array (neighborNeg)")
    storage = STORAGE_OF_DTYPE[dist.dtype]
    _lib.check(_lib.lib().vfb_init_nonequilibrium(storage, dist.data_ptr(), lat.N, lat.geo.data_ptr(),
                                                  lat.neighborX.data_ptr(), lat.neighborY.data_ptr(),
                                                  lat.neighborZ.data_ptr(), lat.neighborInverse.data_ptr(),
                                                  rho.data_ptr(), vx.data_ptr(), vy.data_ptr(), vz.data_ptr(),
                                                  float(omega), int(bool(is_even)), _stream(stream)))


def enstrophy(lat: DeviceLattice, rho, vx, vy, vz, stream=None) -> tuple[float, int]:
    """EnstrophyAnalyzer's value over one level's macroscopic fields (device
    tensors of the compute precision): the mean of 1/2 (drho + 1) |curl u|^2
    over the fluid nodes whose axis neighbours are fluid, and their number."""
    if lat.neighborInverse is None:
        raise _lib.VfbError(_lib.VFB_ERR_INVALID_ARGUMENT, "lattice has no inverse neighbour array (neighborNeg)")
    precision = _lib.FP64 if rho.dtype == torch.float64 else _lib.FP32
    out = (ctypes.c_double * 2)()
    _lib.check(_lib.lib().vfb_enstrophy(precision, rho.data_ptr(), vx.data_ptr(), vy.data_ptr(), vz.data_ptr(), lat.N,
                                        lat.geo.data_ptr(), lat.neighborX.data_ptr(), lat.neighborY.data_ptr(),
                                        lat.neighborZ.data_ptr(), lat.neighborInverse.data_ptr(), out,
                                        _stream(stream)))
    return out[0], int(out[1])


def macroscopic(dist, lat: DeviceLattice, is_even: bool, stream=None):
    """(drho, vx, vy, vz) of every node from the populations of one parity."""
    storage = STORAGE_OF_DTYPE[dist.dtype]
    cd = compute_dtype(dist.dtype)
    out = [torch.empty(lat.N, dtype=cd, device=dist.device) for _ in range(4)]
    _lib.check(_lib.lib().vfb_macroscopic(storage, dist.data_ptr(), lat.N, lat.geo.data_ptr(),
                                          lat.neighborX.data_ptr(), lat.neighborY.data_ptr(),
                                          lat.neighborZ.data_ptr(), int(bool(is_even)), *[o.data_ptr() for o in out],
                                          _stream(stream)))
    return out


def mass_and_energy(dist, lat: DeviceLattice, is_even: bool, nodes=None, stream=None) -> tuple[float, float, int]:
    """FP64 sums over a node list: total drho, kinetic energy, non-finite count."""
    storage = STORAGE_OF_DTYPE[dist.dtype]
    idx = lat.fluid if nodes is None else nodes
    out = (ctypes.c_double * 3)()
    _lib.check(_lib.lib().vfb_mass_and_energy(storage, dist.data_ptr(), lat.N, lat.neighborX.data_ptr(),
                                              lat.neighborY.data_ptr(), lat.neighborZ.data_ptr(), idx.data_ptr(),
                                              int(idx.numel()), int(bool(is_even)), out, _stream(stream)))
    return out[0], out[1], int(out[2])


def _bc_lattice(dist, lat: DeviceLattice, omega: float, is_even: bool) -> _lib.BcLattice:
    t = _lib.BcLattice()
    t.distributions = dist.data_ptr()
    t.numberOfLBnodes = lat.N
    t.neighborX = lat.neighborX.data_ptr()
    t.neighborY = lat.neighborY.data_ptr()
    t.neighborZ = lat.neighborZ.data_ptr()
    t.omega = float(omega)
    t.isEvenTimestep = int(bool(is_even))
    return t


def bc_locations(lat: DeviceLattice, k, stream=None):
    """The location table of a BC list (8 * len(k) uint32 on the device)."""
    out = torch.empty(8 * int(k.numel()), dtype=torch.int32, device=k.device)
    _lib.check(_lib.lib().vfb_bc_locations(k.data_ptr(), int(k.numel()), lat.neighborX.data_ptr(),
                                           lat.neighborY.data_ptr(), lat.neighborZ.data_ptr(), out.data_ptr(),
                                           _stream(stream)))
    return out


def bc_post(kind: int, dist, lat: DeviceLattice, k, q, omega: float, is_even: bool, vx=None, vy=None, vz=None,
            stream=None, locations=None) -> None:
    """One post-collision BC kernel (``kind`` one of _lib.BC_*) over a list:
    ``k`` int32 node indices, ``q`` compute-precision array of 27 * len(k)
    (direction-major), ``vx``/``vy``/``vz`` per-node wall velocity,
    ``locations`` the list's location table (bc_locations) or None."""
    lst = _lib.BcList()
    lst.k = k.data_ptr()
    lst.q = q.data_ptr()
    lst.Vx, lst.Vy, lst.Vz = _p(vx), _p(vy), _p(vz)
    lst.numberOfBCnodes = int(k.numel())
    lst.locations = _p(locations)
    t = _bc_lattice(dist, lat, omega, is_even)
    _lib.check(_lib.lib().vfb_bc_post(int(kind), STORAGE_OF_DTYPE[dist.dtype], ctypes.byref(t), ctypes.byref(lst),
                                      _stream(stream)))


STRESS_ARRAYS = ("k", "kN", "q", "normalX", "normalY", "normalZ", "Vx", "Vy", "Vz", "Vx1", "Vy1", "Vz1",
                 "samplingOffset", "z0")
STRESS_MONITORS = ("uStar", "Fx", "Fy", "Fz")


def bc_stress(kind: int, dist, lat: DeviceLattice, lst: dict, omega: float, is_even: bool, vx, vy, vz,
              turbulent_viscosity=None, stream=None) -> None:
    """One wall-model (stress) BC kernel (``kind`` one of _lib.BC_STRESS_*)
    over a stress list: ``lst`` maps the vfb_stress_list names (k, kN, q,
    normalX.., Vx.. / Vx1.. the two filter states, samplingOffset, z0 and,
    for the monitor, uStar, Fx, Fy, Fz; optionally locations) to device
    tensors; ``vx``/``vy``/``vz`` are the level's macroscopic velocity."""
    s = _lib.StressList()
    for name in STRESS_ARRAYS:
        setattr(s, name, lst[name].data_ptr())
    for name in STRESS_MONITORS:
        setattr(s, name, _p(lst.get(name)))
    s.locations = _p(lst.get("locations"))
    s.numberOfBCnodes = int(lst["k"].numel())
    t = _bc_lattice(dist, lat, omega, is_even)
    _lib.check(_lib.lib().vfb_bc_stress(int(kind), STORAGE_OF_DTYPE[dist.dtype], ctypes.byref(t), ctypes.byref(s),
                                        _p(turbulent_viscosity), vx.data_ptr(), vy.data_ptr(), vz.data_ptr(),
                                        _stream(stream)))


def bc_outflow(dist, lat: DeviceLattice, k, kN, direction: int, is_even: bool, pressure_correction: bool = False,
               correction_factor: float = 0.0, stream=None) -> None:
    """The non-reflecting outflow (OutflowNonReflecting, or with
    pressure_correction OutflowNonReflectingPressureCorrection) of one
    directional list."""
    t = _bc_lattice(dist, lat, 1.0, is_even)
    _lib.check(_lib.lib().vfb_bc_outflow_nonreflecting(STORAGE_OF_DTYPE[dist.dtype], ctypes.byref(t), k.data_ptr(),
                                                       kN.data_ptr(), int(k.numel()), int(direction),
                                                       int(bool(pressure_correction)), float(correction_factor),
                                                       _stream(stream)))


def bc_pressure(dist, lat: DeviceLattice, k, kN, rho, direction: int, is_even: bool, stream=None) -> None:
    """The pre-collision non-equilibrium pressure BC of one directional list."""
    t = _bc_lattice(dist, lat, 1.0, is_even)
    _lib.check(_lib.lib().vfb_bc_pressure_noneq(STORAGE_OF_DTYPE[dist.dtype], ctypes.byref(t), k.data_ptr(),
                                                kN.data_ptr(), rho.data_ptr(), int(k.numel()), int(direction),
                                                _stream(stream)))
