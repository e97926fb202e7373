"""One randomized multi-level grid scenario built by the library's builder and
by the reference's builder (oracle/_ref), compared array by array.  Run as a
child process by tests/test_grid_builder.py: the reference's builder reads
outside its arrays in some scenarios (undefined behaviour that has crashed
it), so every case gets a fresh process and a crash of the reference skips
the case instead of ending the test run.

    python tests/grid_compare_case.py <seed>   ->  prints "ok", "diff ..." or "mine failed ..."
    (seed -1: the full-size wall-mounted cube benchmark grid)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

from oracle.pyoracle import Reference  # noqa: E402
from tests.test_grid_builder import build_mine  # noqa: E402


def random_spec(seed: int) -> np.ndarray:
    """A box refined to level 1 or 2 inside a coarse channel, random
    periodicity, layer counts, side BCs and (half the time) a solid cuboid or
    sphere strictly inside the box."""
    rng = np.random.default_rng(seed)
    s = np.zeros(64)
    n = rng.integers(16, 36, 3)
    s[0:7] = [0, 0, 0, n[0] - 1, n[1] - 1, n[2] - 1, 1.0]
    s[7:10] = rng.integers(0, 2, 3)
    lo = [int(rng.integers(0, int(n[a]) // 2)) for a in range(3)]
    hi = [lo[a] + int(rng.integers(4, max(5, int(n[a]) - lo[a]))) for a in range(3)]
    s[10] = 1
    s[11:17] = [lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]]
    s[61] = 1 if rng.random() < 0.7 else 2
    s[17:19] = [rng.integers(4, 12), rng.integers(4, 8)]
    if rng.random() < 0.5:
        c0 = [lo[a] + 1 for a in range(3)]
        c1 = [min(hi[a] - 1, c0[a] + 2 + int(rng.integers(0, 3))) for a in range(3)]
        if all(c1[a] > c0[a] for a in range(3)):
            s[19] = 1
            s[20:26] = [*c0, *c1]
            s[26] = 1
            if rng.random() < 0.5:
                # a sphere inside that cuboid instead (fractional q from the ray intersection)
                centre = [(c0[a] + c1[a]) / 2 + rng.uniform(-0.2, 0.2) for a in range(3)]
                radius = min(c1[a] - c0[a] for a in range(3)) / 2 * rng.uniform(0.6, 0.95)
                s[19] = 2
                s[20:26] = [*centre, radius, 0, 0]
    i = 0
    for side in rng.permutation(6):
        if s[7 + side // 2] > 0:
            continue
        kind = int(rng.choice([1, 2, 3, 4]))
        vals = {1: (0, 0, 0), 2: (0.03, 0.01, 0), 3: (0.0, 0, 0), 4: (0, 0, 1)}[kind]
        s[30 + 5 * i: 35 + 5 * i] = (side, kind, *vals)
        i += 1
    return s


def cube_benchmark_spec() -> np.ndarray:
    """The wall-mounted cube benchmark at full size: coarse 256 x 96 x 96,
    refined box x 48..128, y 24..72, z 0..40, cube of side 16 on the floor at
    x = 64 centred in y, inlet velocity, pressure outlet, no-slip floor, slip
    top, periodic span, no-slip geometry."""
    s = np.zeros(64)
    s[0:7] = [0, 0, 0, 255, 95, 95, 1.0]
    s[8] = 1
    s[10] = 1
    s[11:17] = [48, 24, 0, 128, 72, 40]
    s[19] = 1
    s[20:26] = [64, 40, 0, 80, 56, 16]
    s[26] = 1
    for i, b in enumerate([(0, 2, 0.04, 0, 0), (1, 3, 0.0, 0, 0), (4, 1, 0, 0, 0), (5, 4, 0, 0, 1)]):
        s[30 + 5 * i: 35 + 5 * i] = b
    return s


def main(seed: int) -> int:
    s = cube_benchmark_spec() if seed < 0 else random_spec(seed)
    ref = Reference("f64").grid(s)
    ref = [ref[lvl] for lvl in sorted(ref)]
    try:
        mine = build_mine(s)
    except Exception as e:  # noqa: BLE001
        print("mine failed", e)
        return 0
    if len(mine) != len(ref):
        print("diff levels", len(mine), len(ref))
        return 0
    for lvl, r in enumerate(ref):
        for name, v in r.items():
            m = mine[lvl].get(name)
            if m is None:
                if len(v):
                    print("diff missing", lvl, name)
                    return 0
                continue
            if name.startswith("coord"):
                same = m.shape == v.shape and np.allclose(m, v, rtol=0, atol=1e-9 * max(1.0, np.abs(v).max()))
            else:
                same = m.shape == v.shape and np.array_equal(m.astype(v.dtype), v)
            if not same:
                print("diff", lvl, name)
                return 0
    print("ok", len(ref), "levels")
    return 0


if __name__ == "__main__":
    sys.exit(main(int(sys.argv[1])))
