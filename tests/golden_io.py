"""Loader for the committed golden vectors (tests/golden/*.npz), produced by
tests/golden/make_golden.py from xFluid's own solver."""
from pathlib import Path

import numpy as np

from xfluid_b200.scenes import Scene

GOLDEN = Path(__file__).resolve().parent / "golden"
# the variational solver's cases (normal_*.npz belong to test_normal.py, steps_*.npz to test_steps.py,
# particles_*.npz to test_particles.py, full_*.npz to the full-size test in test_gpu_parity.py)
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz")
               if not p.stem.startswith(("normal_", "steps_", "particles_", "full_")))


def load(name):
    g = dict(np.load(GOLDEN / f"{name}.npz"))
    ni, nj, nk = (int(x) for x in g["dims"])
    sc = Scene(ni, nj, nk, g["mat"], g["u"], g["v"], g["w"], name=name)
    return sc, g


def bits_equal(a, b):
    """Bit-identical FP64 arrays, except that -0.0 and +0.0 compare equal (the
    reference keeps the sign of zero in rows without an unknown; the GPU
    output grid holds +0.0 there)."""
    a = np.ascontiguousarray(a, dtype=np.float64) + 0.0
    b = np.ascontiguousarray(b, dtype=np.float64) + 0.0
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))
