"""Stub for the ``trimesh`` import at the top of the reference's
sim/init_conditions.py; voxelisation is not emulated (test infrastructure
only)."""


class Trimesh:  # pragma: no cover - never used by the golden generator
    def __init__(self, *a, **k):
        raise RuntimeError("trimesh is not available; the delta-wing mask is built by the oracle")
