"""xfluid_b200: B200-native (sm_100a) pressure projection for xFluid's
FLIP/PIC water step -- the variational MAC-grid Poisson system, MIC(0)-PCG in
natural order and the pressure-gradient update -- behind xFluid's solver
interface.  The compute path is libxfp.so (include/xfp.h); see solver.py for
the Python mirror of VariationalPressureSolver.
"""
import importlib

__all__ = ["VariationalPressureSolver", "NormalPressureSolver", "project_scene", "scenes"]


def __getattr__(name):
    if name in ("VariationalPressureSolver", "NormalPressureSolver", "project_scene"):
        return getattr(importlib.import_module(__name__ + ".solver"), name)
    raise AttributeError(name)
