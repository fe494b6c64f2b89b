"""kratos_b200: B200-native (sm_100a) unsplit Godunov hydro / ideal-MHD step
with the Kratos plugin surface (parameter files, block layout, snapshots)."""
from .engine import Dynamics, KratosError  # noqa: F401
