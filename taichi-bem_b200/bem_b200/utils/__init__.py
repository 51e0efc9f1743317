from .types import CellFluxType, VertAttachType, KernelType, PanelsRelation, AssembleType, ScopeType
from .functions import get_gaussion_integration_points_and_weights
from .io import warp_tensor, unwarp_tensor

__all__ = ["CellFluxType", "VertAttachType", "KernelType", "PanelsRelation", "AssembleType", "ScopeType",
           "get_gaussion_integration_points_and_weights", "warp_tensor", "unwarp_tensor"]
