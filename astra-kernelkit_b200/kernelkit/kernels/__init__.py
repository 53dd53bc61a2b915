from .cone_fp import RayDrivenConeFP
from .cone_bp import VoxelDrivenConeBP

__all__ = ["RayDrivenConeFP", "VoxelDrivenConeBP"]
