"""Python binding of the oracle (TEST INFRASTRUCTURE ONLY).

Loads the CPU restatement (oracle/liboracle_{f32,f64}.so, built from
vf_oracle.c) and, when present, the reference's own sources compiled on the
host (oracle/_ref/libvfref_{f32,f64}.so).  Only tests/, the smoke check and
bench.py's CPU-baseline leg use this module; the product never imports it.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

_c = ctypes
_vp = _c.c_void_p


def build(with_ref: bool = False) -> None:
    """Build the oracle (and the reference libraries when the tree exists)."""
    subprocess.run(["make", "-C", str(HERE), "ref" if with_ref else "all", "-j8"], check=True,
                   capture_output=True, text=True)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_vp)


def _STRESS_ARGS(R, size_t, count_t):
    return [_c.c_int, _vp, size_t, _vp, _vp, _vp, _vp, _vp, _vp, count_t, R, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
            _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c.c_int, _vp, _vp, _vp, _vp, _c.c_int]


STRESS_STATE = ("vxEl", "vyEl", "vzEl", "vxWMean", "vyWMean", "vzWMean")
STRESS_MONITORS = ("uStar", "Fx", "Fy", "Fz")


def _stress_call(kind, dist, N, nx, ny, nz, lst, omega, vx, vy, vz, turb, monitor, is_even):
    n = len(lst["k"])
    return (kind, _ptr(dist), N, _ptr(nx), _ptr(ny), _ptr(nz), _ptr(lst["k"]), _ptr(lst["kN"]), _ptr(lst["q"]), n,
            omega, _ptr(turb), _ptr(vx), _ptr(vy), _ptr(vz), _ptr(lst["normalX"]), _ptr(lst["normalY"]),
            _ptr(lst["normalZ"]), *[_ptr(lst[a]) for a in STRESS_STATE], _ptr(lst["samplingOffset"]),
            _ptr(lst["z0"]), int(bool(monitor)), *[_ptr(lst.get(a)) for a in STRESS_MONITORS], int(is_even))


class _Lib:
    def __init__(self, path: Path, suffix: str, real):
        self.path = path
        self.L = _c.CDLL(str(path))
        self.sfx = suffix
        self.real = real

    def fn(self, name):
        return getattr(self.L, name + self.sfx)


class Oracle(_Lib):
    """The CPU restatement (vf_oracle.c) for one precision."""

    def __init__(self, precision: str = "f64"):
        real = np.float64 if precision == "f64" else np.float32
        super().__init__(HERE / f"liboracle_{precision}.so", "_" + precision, real)
        R = _c.c_double if precision == "f64" else _c.c_float
        self.R = R
        self.fn("vfo_k17_collide").argtypes = [_vp, R, _vp, R, R, R, _vp, _vp, _vp, _vp]
        self.fn("vfo_collision_k17").argtypes = [_vp, _c.c_uint64, _vp, _vp, _vp, _vp, _c.c_uint32, R, _vp, R, _vp,
                                                 _c.c_int, _c.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
        self.fn("vfo_bgk_collide").argtypes = [_vp, R]
        self.fn("vfo_collision_bgk").argtypes = [_vp, _c.c_uint64, _vp, _vp, _vp, _vp, R, _c.c_int]
        self.fn("vfo_init_eq").argtypes = [_vp, _c.c_uint64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c.c_int]
        self.fn("vfo_init_noneq").argtypes = [_vp, _c.c_uint64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, R,
                                              _c.c_int]
        self.fn("vfo_noneq_node").argtypes = [R, R, R, R, _vp, R, _vp]
        self.fn("vfo_bc_post").argtypes = [_c.c_int, _vp, _c.c_uint64, _vp, _vp, _vp, _vp, _vp, _c.c_uint32, R, _vp,
                                           _vp, _vp, _c.c_int]
        self.fn("vfo_bc_pressure_noneq").argtypes = [_vp, _c.c_uint64, _vp, _vp, _vp, _vp, _vp, _vp, _c.c_uint32,
                                                     _c.c_int, _c.c_int]
        self.fn("vfo_bc_outflow").argtypes = [_c.c_int, _vp, _c.c_uint64, _vp, _vp, _vp, _vp, _vp, _c.c_uint32,
                                              _c.c_int, R, _c.c_int]
        self.fn("vfo_bc_stress").argtypes = _STRESS_ARGS(R, _c.c_uint64, _c.c_uint32)
        self.fn("vfo_enstrophy_nodes").argtypes = [_vp, _vp, _vp, _vp, _c.c_uint64, _vp, _vp, _vp, _vp, _vp, _vp,
                                                   _vp]
        self.fn("vfo_macroscopic").argtypes = [_vp, _c.c_uint64, _vp, _vp, _vp, _vp, _c.c_int, _vp, _vp, _vp, _vp]

    # -- single node ----------------------------------------------------------
    def k17_node(self, f, omega, limiter=(0.01, 0.01, 0.01), force=(0.0, 0.0, 0.0)):
        f = np.ascontiguousarray(f, dtype=self.real).copy()
        lim = np.asarray(limiter, dtype=self.real)
        out = [self.R() for _ in range(4)]
        self.fn("vfo_k17_collide")(_ptr(f), omega, _ptr(lim), force[0], force[1], force[2],
                                   *[_c.byref(o) for o in out])
        return f, np.array([o.value for o in out], dtype=self.real)

    def bgk_node(self, f, omega):
        f = np.ascontiguousarray(f, dtype=self.real).copy()
        self.fn("vfo_bgk_collide")(_ptr(f), omega)
        return f

    def noneq_node(self, drho, vx, vy, vz, grad, omega):
        """Equilibrium plus non-equilibrium populations of one node (27,
        canonical direction order) from the velocity gradient grad[a][b] =
        d u_a / d x_b."""
        g = np.ascontiguousarray(grad, dtype=self.real).reshape(9)
        f = np.zeros(27, self.real)
        self.fn("vfo_noneq_node")(drho, vx, vy, vz, _ptr(g), omega, _ptr(f))
        return f

    # -- whole-lattice passes (arrays modified in place) ----------------------
    def collision_k17(self, dist, N, nx, ny, nz, fluid, omega, forces=(0, 0, 0), force_factor=1.0,
                      limiters=(0.01, 0.01, 0.01), is_even=True, flags=0, macro=None, body=None):
        forces = np.asarray(forces, dtype=self.real)
        lim = np.asarray(limiters, dtype=self.real)
        rho, vx, vy, vz = macro if macro is not None else (None,) * 4
        bx, by, bz = body if body is not None else (None,) * 3
        self.fn("vfo_collision_k17")(_ptr(dist), N, _ptr(nx), _ptr(ny), _ptr(nz), _ptr(fluid), len(fluid), omega,
                                     _ptr(forces), force_factor, _ptr(lim), int(is_even), flags, _ptr(rho), _ptr(vx),
                                     _ptr(vy), _ptr(vz), _ptr(bx), _ptr(by), _ptr(bz))

    def collision_bgk(self, dist, N, geo, nx, ny, nz, omega, is_even=True):
        self.fn("vfo_collision_bgk")(_ptr(dist), N, _ptr(geo), _ptr(nx), _ptr(ny), _ptr(nz), omega, int(is_even))

    def init_eq(self, dist, N, geo, nx, ny, nz, rho, ux, uy, uz, is_even):
        self.fn("vfo_init_eq")(_ptr(dist), N, _ptr(geo), _ptr(nx), _ptr(ny), _ptr(nz), _ptr(rho), _ptr(ux),
                               _ptr(uy), _ptr(uz), int(is_even))

    def init_noneq(self, dist, N, geo, nx, ny, nz, nneg, rho, ux, uy, uz, omega, is_even):
        self.fn("vfo_init_noneq")(_ptr(dist), N, _ptr(geo), _ptr(nx), _ptr(ny), _ptr(nz), _ptr(nneg), _ptr(rho),
                                  _ptr(ux), _ptr(uy), _ptr(uz), omega, int(is_even))

    def bc_post(self, kind, dist, N, nx, ny, nz, k, q, omega, vx=None, vy=None, vz=None, is_even=True):
        self.fn("vfo_bc_post")(kind, _ptr(dist), N, _ptr(nx), _ptr(ny), _ptr(nz), _ptr(k), _ptr(q), len(k), omega,
                               _ptr(vx), _ptr(vy), _ptr(vz), int(is_even))

    def bc_stress(self, kind, dist, N, nx, ny, nz, lst, omega, vx, vy, vz, turb=None, monitor=False, is_even=True):
        """Wall-model BC (kind 0 StressCompressible, 1 StressBounceBack, 2
        StressBounceBackPressure) over the list dict lst (its filter and
        monitor arrays are updated in place)."""
        self.fn("vfo_bc_stress")(*_stress_call(kind, dist, N, nx, ny, nz, lst, omega, vx, vy, vz, turb, monitor,
                                               is_even))

    def bc_pressure(self, dist, N, nx, ny, nz, k, kN, rho, direction, is_even=True):
        self.fn("vfo_bc_pressure_noneq")(_ptr(dist), N, _ptr(nx), _ptr(ny), _ptr(nz), _ptr(k), _ptr(kN), _ptr(rho),
                                         len(k), direction, int(is_even))

    def bc_outflow(self, dist, N, nx, ny, nz, k, kN, direction, correction=False, factor=0.0, is_even=True):
        self.fn("vfo_bc_outflow")(int(bool(correction)), _ptr(dist), N, _ptr(nx), _ptr(ny), _ptr(nz), _ptr(k), _ptr(kN),
                                  len(k), direction, factor, int(is_even))

    def enstrophy_nodes(self, rho, vx, vy, vz, geo, nx, ny, nz, nneg):
        """Per-node enstrophy values and the counted mask of EnstrophyAnalyzer."""
        N = len(geo)
        out = np.zeros(N, self.real)
        counted = np.zeros(N, np.uint32)
        args = [np.ascontiguousarray(a, dtype=self.real) for a in (rho, vx, vy, vz)]
        self.fn("vfo_enstrophy_nodes")(*[_ptr(a) for a in args], N, _ptr(geo), _ptr(nx), _ptr(ny), _ptr(nz),
                                       _ptr(nneg), _ptr(out), _ptr(counted))
        return out, counted.astype(bool)

    def macroscopic(self, dist, N, geo, nx, ny, nz, is_even):
        out = [np.zeros(N, self.real) for _ in range(4)]
        self.fn("vfo_macroscopic")(_ptr(dist), N, _ptr(geo), _ptr(nx), _ptr(ny), _ptr(nz), int(is_even),
                                   *[_ptr(o) for o in out])
        return out


def ref_available(precision: str = "f64") -> bool:
    return (REF_DIR / f"libvfref_{precision}.so").exists()


class Reference(_Lib):
    """The reference's own sources compiled on the host (oracle/_ref)."""

    def __init__(self, precision: str = "f64"):
        real = np.float64 if precision == "f64" else np.float32
        super().__init__(REF_DIR / f"libvfref_{precision}.so", "_" + precision, real)
        R = _c.c_double if precision == "f64" else _c.c_float
        self.R = R
        self.fn("vfref_k17_node").argtypes = [_vp, R, _vp, R, R, R, _vp]
        self.fn("vfref_collision_k17").argtypes = [_vp, _c.c_ulonglong, _vp, _vp, _vp, _vp, _c.c_uint, R, _vp, R, _vp,
                                                   _c.c_int, _c.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
        self.fn("vfref_collision_bgk").argtypes = [_vp, _c.c_ulonglong, _vp, _vp, _vp, _vp, R, _c.c_int]
        self.fn("vfref_init_eq").argtypes = [_vp, _c.c_ulonglong, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c.c_int]
        self.fn("vfref_init_noneq").argtypes = [_vp, _c.c_ulonglong, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                                R, _c.c_int]
        self.fn("vfref_bc_post").argtypes = [_c.c_int, _vp, _c.c_ulonglong, _vp, _vp, _vp, _vp, _vp, _c.c_uint, R, _vp,
                                             _vp, _vp, _c.c_int]
        self.fn("vfref_bc_pressure_noneq").argtypes = [_vp, _c.c_ulonglong, _vp, _vp, _vp, _vp, _vp, _vp, _c.c_uint,
                                                       _c.c_int, _c.c_int]
        self.fn("vfref_bc_outflow").argtypes = [_c.c_int, _vp, _c.c_ulonglong, _vp, _vp, _vp, _vp, _vp, _c.c_uint,
                                                _c.c_int, R, _c.c_int]
        self.fn("vfref_bc_stress").argtypes = _STRESS_ARGS(R, _c.c_ulonglong, _c.c_uint)
        self.fn("vfref_grid_build").restype = _vp
        self.fn("vfref_grid_build").argtypes = [_vp]
        self.fn("vfref_grid_levels").argtypes = [_vp]
        self.fn("vfref_grid_count").restype = _c.c_longlong
        self.fn("vfref_grid_count").argtypes = [_vp, _c.c_int, _c.c_char_p]
        self.fn("vfref_grid_elem_size").argtypes = [_vp, _c.c_int, _c.c_char_p]
        self.fn("vfref_grid_copy").argtypes = [_vp, _c.c_int, _c.c_char_p, _vp]
        self.fn("vfref_grid_free").argtypes = [_vp]
        self.fn("vfref_cpu_block_create").restype = _vp
        self.fn("vfref_cpu_block_create").argtypes = [_c.c_int, _c.c_int, _c.c_int]
        self.fn("vfref_cpu_block_create_tgv").restype = _vp
        self.fn("vfref_cpu_block_create_tgv").argtypes = [_c.c_int, _c.c_double]
        self.fn("vfref_cpu_block_free").argtypes = [_vp]
        self.fn("vfref_cpu_block_run").restype = _c.c_double
        self.fn("vfref_cpu_block_run").argtypes = [_vp, _c.c_int, R]
        for name in ("vfref_scale_cf", "vfref_scale_fc"):
            self.fn(name).argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c.c_ulonglong, _c.c_ulonglong, _c.c_int,
                                      _vp, _vp, _c.c_uint, R, R, _vp, _vp, _vp]

    def scale(self, coarse_to_fine, distC, distF, coarse, fine, is_even, cells_c, cells_f, omega_c, omega_f,
              off_x, off_y, off_z):
        """scaleCoarseToFineCompressible_Device<false> / scaleFineToCoarseCompressible_Device<false>
        over all cells; coarse / fine are dicts with neighborX/Y/Z."""
        name = "vfref_scale_cf" if coarse_to_fine else "vfref_scale_fc"
        self.fn(name)(_ptr(distC), _ptr(distF), _ptr(coarse["neighborX"]), _ptr(coarse["neighborY"]),
                      _ptr(coarse["neighborZ"]), _ptr(fine["neighborX"]), _ptr(fine["neighborY"]),
                      _ptr(fine["neighborZ"]), len(coarse["geo"]), len(fine["geo"]), int(is_even), _ptr(cells_c),
                      _ptr(cells_f), len(cells_c), omega_c, omega_f, _ptr(off_x), _ptr(off_y), _ptr(off_z))

    def k17_node(self, f, omega, limiter=(0.01, 0.01, 0.01), force=(0.0, 0.0, 0.0)):
        f = np.ascontiguousarray(f, dtype=self.real).copy()
        lim = np.asarray(limiter, dtype=self.real)
        out = np.zeros(4, self.real)
        self.fn("vfref_k17_node")(_ptr(f), omega, _ptr(lim), force[0], force[1], force[2], _ptr(out))
        return f, out

    def collision_k17(self, dist, N, nx, ny, nz, fluid, omega, forces=(0, 0, 0), force_factor=1.0,
                      limiters=(0.01, 0.01, 0.01), is_even=True, flags=0, macro=None, body=None):
        forces = np.asarray(forces, dtype=self.real)
        lim = np.asarray(limiters, dtype=self.real)
        rho, vx, vy, vz = macro if macro is not None else (None,) * 4
        bx, by, bz = body if body is not None else (None,) * 3
        self.fn("vfref_collision_k17")(_ptr(dist), N, _ptr(nx), _ptr(ny), _ptr(nz), _ptr(fluid), len(fluid), omega,
                                       _ptr(forces), force_factor, _ptr(lim), int(is_even), flags, _ptr(rho),
                                       _ptr(vx), _ptr(vy), _ptr(vz), _ptr(bx), _ptr(by), _ptr(bz))

    def collision_bgk(self, dist, N, geo, nx, ny, nz, omega, is_even=True):
        self.fn("vfref_collision_bgk")(_ptr(dist), N, _ptr(geo), _ptr(nx), _ptr(ny), _ptr(nz), omega, int(is_even))

    def init_eq(self, dist, N, geo, nx, ny, nz, rho, ux, uy, uz, is_even):
        self.fn("vfref_init_eq")(_ptr(dist), N, _ptr(geo), _ptr(nx), _ptr(ny), _ptr(nz), _ptr(rho), _ptr(ux),
                                 _ptr(uy), _ptr(uz), int(is_even))

    def init_noneq(self, dist, N, geo, nx, ny, nz, nneg, rho, ux, uy, uz, omega, is_even):
        self.fn("vfref_init_noneq")(_ptr(dist), N, _ptr(geo), _ptr(nx), _ptr(ny), _ptr(nz), _ptr(nneg), _ptr(rho),
                                    _ptr(ux), _ptr(uy), _ptr(uz), omega, int(is_even))

    def bc_post(self, kind, dist, N, nx, ny, nz, k, q, omega, vx=None, vy=None, vz=None, is_even=True):
        self.fn("vfref_bc_post")(kind, _ptr(dist), N, _ptr(nx), _ptr(ny), _ptr(nz), _ptr(k), _ptr(q), len(k), omega,
                                 _ptr(vx), _ptr(vy), _ptr(vz), int(is_even))

    def bc_stress(self, kind, dist, N, nx, ny, nz, lst, omega, vx, vy, vz, turb=None, monitor=False, is_even=True):
        self.fn("vfref_bc_stress")(*_stress_call(kind, dist, N, nx, ny, nz, lst, omega, vx, vy, vz, turb, monitor,
                                                 is_even))

    def bc_pressure(self, dist, N, nx, ny, nz, k, kN, rho, direction, is_even=True):
        self.fn("vfref_bc_pressure_noneq")(_ptr(dist), N, _ptr(nx), _ptr(ny), _ptr(nz), _ptr(k), _ptr(kN),
                                           _ptr(rho), len(k), direction, int(is_even))

    def bc_outflow(self, dist, N, nx, ny, nz, k, kN, direction, correction=False, factor=0.0, is_even=True):
        self.fn("vfref_bc_outflow")(int(bool(correction)), _ptr(dist), N, _ptr(nx), _ptr(ny), _ptr(nz), _ptr(k),
                                    _ptr(kN), len(k), direction, factor, int(is_even))

    def grid(self, spec):
        """Build a grid with the reference builder; returns {level: {name: array}}."""
        s = np.zeros(max(64, len(spec)))
        s[:len(spec)] = spec
        h = self.fn("vfref_grid_build")(_ptr(s))
        try:
            out = {}
            for level in range(self.fn("vfref_grid_levels")(h)):
                out[level] = _export_all(self, h, level, "vfref_grid")
            return out
        finally:
            self.fn("vfref_grid_free")(h)

    def cpu_tgv_block(self, n: int, u0: float = 0.05) -> "CpuBlock":
        """The reference CPU path's EsoSplit block holding the n^3 Taylor-Green
        vortex (created once; run passes on it with .run)."""
        return CpuBlock(self, self.fn("vfref_cpu_block_create_tgv")(n, u0), n)

    def cpu_block_mlups(self, n: int, steps: int, omega: float = 1.9) -> tuple[float, float]:
        """Run the reference CPU K17 loop on an n^3 block; returns (seconds, MLUPS)."""
        h = self.fn("vfref_cpu_block_create")(n, n, n)
        try:
            sec = self.fn("vfref_cpu_block_run")(h, steps, omega)
        finally:
            self.fn("vfref_cpu_block_free")(h)
        return sec, steps * n ** 3 / sec / 1e6


class CpuBlock:
    """An EsoSplit block of the reference CPU path kept between timed passes."""

    def __init__(self, ref: "Reference", handle, n: int):
        self.ref, self.h, self.n = ref, handle, n
        if not handle:
            raise MemoryError(f"could not create the {n}^3 CPU block")

    def run(self, steps: int, omega: float) -> float:
        """`steps` collision passes of the reference CPU K17 loop; seconds."""
        return self.ref.fn("vfref_cpu_block_run")(self.h, steps, omega)

    def close(self):
        if self.h:
            self.ref.fn("vfref_cpu_block_free")(self.h)
            self.h = None

    def __del__(self):
        self.close()


def ref_gpu_available(precision: str = "f64") -> bool:
    return (REF_DIR / f"libvfref_gpu_{precision}.so").exists()


def _dptr(t):
    """Device address of a tensor (or None)."""
    return None if t is None else _vp(t.data_ptr())


class ReferenceGpu(_Lib):
    """The reference's GPU kernel sources compiled unmodified by nvcc for
    sm_100a (oracle/_ref/libvfref_gpu_{f32,f64}.so, launchers in
    oracle/ref/ref_gpu_device.cu).  Arguments are CUDA tensors; every call is
    asynchronous on `stream` (a cudaStream_t address, 0 = legacy stream)."""

    def __init__(self, precision: str = "f64"):
        real = np.float64 if precision == "f64" else np.float32
        super().__init__(REF_DIR / f"libvfref_gpu_{precision}.so", "_" + precision, real)
        R = _c.c_double if precision == "f64" else _c.c_float
        self.R = R
        self.fn("vfref_gpu_collision_k17").argtypes = [_vp, _c.c_ulonglong, _vp, _vp, _vp, _vp, _c.c_uint, R, _vp, R,
                                                       _vp, _c.c_int, _vp]
        self.fn("vfref_gpu_collision_bgk").argtypes = [_vp, _c.c_ulonglong, _vp, _vp, _vp, _vp, R, _c.c_int, _vp]
        self.fn("vfref_gpu_bc_post").argtypes = [_c.c_int, _vp, _c.c_ulonglong, _vp, _vp, _vp, _vp, _vp, _c.c_uint, R,
                                                 _vp, _vp, _vp, _c.c_int, _vp]
        for name in ("vfref_gpu_scale_cf", "vfref_gpu_scale_fc"):
            self.fn(name).argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c.c_ulonglong, _c.c_ulonglong, _c.c_int,
                                      _vp, _vp, _c.c_uint, R, R, _vp, _vp, _vp, _vp]
        self.fn("vfref_gpu_enstrophy").argtypes = [_vp] * 11 + [_c.c_ulonglong, _vp]

    def enstrophy(self, vx, vy, vz, rho, nx, ny, nz, nneg, geo, enstrophy, is_fluid, stream=0):
        """enstrophyKernel of EnstrophyAnalyzer.cu over all nodes (device tensors;
        enstrophy and is_fluid zero-initialised)."""
        self._check(self.fn("vfref_gpu_enstrophy")(
            *[_dptr(t) for t in (vx, vy, vz, rho, nx, ny, nz, nneg, geo, enstrophy, is_fluid)], geo.numel(),
            _vp(stream)), "enstrophyKernel")

    @staticmethod
    def _check(rc: int, what: str) -> None:
        if rc != 0:
            raise RuntimeError(f"{what}: CUDA error {rc}")

    def collision_k17(self, dist, lat, omega, is_even, forces, limiters, force_factor=1.0, stream=0):
        """forces / limiters: device tensors of three values of the library's real type."""
        self._check(self.fn("vfref_gpu_collision_k17")(
            _dptr(dist), lat.N, _dptr(lat.neighborX), _dptr(lat.neighborY), _dptr(lat.neighborZ), _dptr(lat.fluid),
            lat.fluid.numel(), omega, _dptr(forces), force_factor, _dptr(limiters), int(is_even), _vp(stream)),
            "runCollision<K17>")

    def collision_bgk(self, dist, lat, omega, is_even, stream=0):
        self._check(self.fn("vfref_gpu_collision_bgk")(
            _dptr(dist), lat.N, _dptr(lat.geo), _dptr(lat.neighborX), _dptr(lat.neighborY), _dptr(lat.neighborZ),
            omega, int(is_even), _vp(stream)), "B92CompressibleNavierStokes_Device")

    def bc_post(self, kind, dist, lat, k, q, omega, is_even, vx=None, vy=None, vz=None, stream=0):
        rc = self.fn("vfref_gpu_bc_post")(
            kind, _dptr(dist), lat.N, _dptr(lat.neighborX), _dptr(lat.neighborY), _dptr(lat.neighborZ), _dptr(k),
            _dptr(q), k.numel(), omega, _dptr(vx), _dptr(vy), _dptr(vz), int(is_even), _vp(stream))
        self._check(rc, f"BC kernel kind {kind}")

    def scale(self, coarse_to_fine, distC, distF, latC, latF, is_even, cells_c, cells_f, omega_c, omega_f,
              off_x, off_y, off_z, stream=0):
        name = "vfref_gpu_scale_cf" if coarse_to_fine else "vfref_gpu_scale_fc"
        rc = self.fn(name)(_dptr(distC), _dptr(distF), _dptr(latC.neighborX), _dptr(latC.neighborY),
                           _dptr(latC.neighborZ), _dptr(latF.neighborX), _dptr(latF.neighborY), _dptr(latF.neighborZ),
                           latC.N, latF.N, int(is_even), _dptr(cells_c), _dptr(cells_f), cells_c.numel(), omega_c,
                           omega_f, _dptr(off_x), _dptr(off_y), _dptr(off_z), _vp(stream))
        self._check(rc, name)


_NAMES = ["coordX", "coordY", "coordZ", "neighborX", "neighborY", "neighborZ", "neighborNeg", "geo", "dims", "fluid",
          "velocity.k", "velocity.vx", "velocity.vy", "velocity.vz", "velocity.q", "slip.k", "slip.nx", "slip.ny",
          "slip.nz", "slip.q", "geometry.k", "geometry.q", "geometry.vx", "geometry.vy", "geometry.vz",
          "pressure.count", "stress.k", "stress.kN", "stress.nx", "stress.ny", "stress.nz", "stress.q",
          "stress.samplingOffset", "stress.z0", "cf.coarse", "cf.fine", "fc.coarse",
          "fc.fine", "cf.offX", "cf.offY", "cf.offZ", "fc.offX", "fc.offY", "fc.offZ"]
_INT_NAMES = {"velocity.k", "slip.k", "geometry.k", "pressure.count", "dims", "stress.samplingOffset"}


def _dtype_for(name: str, size: int):
    base = name.split(".")[-1]
    if name in _INT_NAMES or base in ("k", "kN", "dir", "count"):
        return np.int32
    if name in ("neighborX", "neighborY", "neighborZ", "neighborNeg", "geo", "fluid", "cf.coarse", "cf.fine",
                "fc.coarse", "fc.fine"):
        return np.uint32
    return np.float64 if size == 8 else np.float32


def _export_all(obj, h, level, prefix):
    count = obj.fn(prefix + "_count") if hasattr(obj, "fn") else getattr(obj, prefix + "_count")
    esize = obj.fn(prefix + "_elem_size")
    copy = obj.fn(prefix + "_copy")
    names = list(_NAMES)
    npc = count(h, level, b"pressure.count")
    if npc >= 0:
        tmp = np.zeros(1, np.int32)
        copy(h, level, b"pressure.count", _ptr(tmp))
        for i in range(int(tmp[0])):
            names += [f"pressure{i}.{s}" for s in ("k", "kN", "rho", "q", "dir")]
    out = {}
    for name in names:
        n = count(h, level, name.encode())
        if n < 0:
            continue
        es = esize(h, level, name.encode())
        a = np.zeros(n, _dtype_for(name, es))
        assert a.itemsize == es, (name, a.itemsize, es)
        copy(h, level, name.encode(), _ptr(a))
        out[name] = a
    return out
