from .core_manager import CoreManager
from .mesh_manager import MeshManager
from .bem_manager import BEMManager

__all__ = ["CoreManager", "MeshManager", "BEMManager"]
