"""bearing_b200: Bearing's contact-solve stage on NVIDIA B200 (sm_100a), behind Bearing's World API."""
from .world import Batch, World, BearingError, GpuSolver  # noqa: F401

__all__ = ["World", "Batch", "BearingError", "GpuSolver"]
